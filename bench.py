"""Benchmark: ray-steps/s of the B200 tracer on the 512^3 turbulent box with
1e7 rays, with the all-FP64 port and the error against it, end-to-end
throughput through the public API, the trace kernel's roofline and the CPU
baseline. Prints one JSON line (rank 0).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl sloth|reference]

One bench step = one trace of every ray of the workload (Morton pre-pass +
persistent tracer). Multi-GPU runs shard nothing across ranks: each rank
traces its own seeded 1e7-ray beam through its own copy of the grid (weak
scaling; rays are independent, there is no data-path collective).
"""
from __future__ import annotations

import argparse
import json
import math
import os
import re
import subprocess
import sys
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "ray-steps/s, 512³ turb box 1e7 rays, ≤1e-6 rel err vs all-FP64 kernel; p99 latency"
UNIT = "ray-steps/s"
BYTES_PER_RAY_STEP = 384          # 3 stages (4th-order Runge-Kutta-Nystrom) x 8 corners x 16-byte float4 voxels
L = 5e-3
LWL = 532e-9
TE, ZION = 20.0, 1.0


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=5)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", choices=["sloth", "reference"], default="sloth")
    ap.add_argument("--n", type=int, default=512, help="grid points per axis")
    ap.add_argument("--rays", type=float, default=1e7)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--no-fp64", action="store_true")
    ap.add_argument("--no-rk4", action="store_true")
    ap.add_argument("--no-e2e", action="store_true")
    ap.add_argument("--no-cpu", action="store_true")
    ap.add_argument("--cpu-seconds", type=float, default=15.0)
    ap.add_argument("--no-serving", action="store_true")
    ap.add_argument("--serving-requests", type=int, default=2000)
    ap.add_argument("--no-adjoint", action="store_true")
    ap.add_argument("--no-diagnostics", action="store_true")
    return ap.parse_args()


# ---------------------------------------------------------------------------
# helpers
# ---------------------------------------------------------------------------
def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            d = json.load(f)
        return float(d["hbm_gbs"]), "measured"
    return 6650.0, "fallback"


def committed_lane_ops():
    """FP32 lane-operations per ray-step of the trace kernel, from the committed
    ncu instruction-mix summary (scalar FFMA/FADD/FMUL plus two lanes per
    paired FFMA2/FADD2/FMUL2)."""
    p = os.path.join(ROOT, "profiles", "trace_kernel_kolmogorov512_1e7.md")
    if not os.path.exists(p):
        return None, None
    text = open(p).read()
    m = re.search(r"fp32_lane_ops_per_ray_step:\s*([0-9.eE+]+)", text)
    w = re.search(r"fp32_lane_ops_workload:\s*(.+)", text)
    return (float(m.group(1)) if m else None), (w.group(1).strip() if w else None)


def committed_backward_lane_ops():
    """FP32 lane-operations per ray-step of the adjoint backward kernel, from the
    committed ncu instruction-mix summary of the detector-image workload."""
    p = os.path.join(ROOT, "profiles", "adjoint_kernels_kolmogorov128_1e6.md")
    if not os.path.exists(p):
        return None, None
    text = open(p).read()
    m = re.search(r"backward_fp32_lane_ops_per_ray_step:\s*([0-9.eE+]+)", text)
    w = re.search(r"backward_lane_ops_workload:\s*(.+)", text)
    return (float(m.group(1)) if m else None), (w.group(1).strip() if w else None)


def committed_traffic(args):
    """DRAM bytes per trace launch from the committed ncu summary of the
    512^3 / 1e7-ray workload (None for any other workload)."""
    p = os.path.join(ROOT, "profiles", "trace_kernel_kolmogorov512_1e7.md")
    if (args.n, int(args.rays), args.seed) != (512, 10 ** 7, 2024) or not os.path.exists(p):
        return None
    m = re.search(r"traffic_bytes_per_launch:\s*([0-9.eE+]+)", open(p).read())
    return float(m.group(1)) if m else None


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms, written to
    clocks_rank<i>.csv in $SLOTH_CLOCKS_DIR (default: the temp directory)."""

    def __init__(self, index):
        import tempfile
        self.index = index
        self.proc = None
        folder = os.environ.get("SLOTH_CLOCKS_DIR") or tempfile.gettempdir()
        self.path = os.path.join(folder, f"clocks_rank{index}.csv")

    def __enter__(self):
        try:
            os.makedirs(os.path.dirname(self.path), exist_ok=True)
            self.f = open(self.path, "w")
            self.proc = subprocess.Popen(
                ["nvidia-smi", f"--id={self.index}",
                 "--query-gpu=index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
                 "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
                 "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap",
                 "--format=csv,noheader,nounits", "-lms", "200"], stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.proc = None
        return self

    def __exit__(self, *a):
        if self.proc is not None:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()
            self.f.close()

    def summary(self):
        if self.proc is None or not os.path.exists(self.path):
            return None
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for line in open(self.path):
            f = [x.strip() for x in line.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for name, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(name)
        if not sm:
            return None
        return {"sm_mhz": float(np.median(sm)), "sm_max_mhz": mx, "reasons": sorted(reasons),
                "samples": len(sm)}


def make_workload(n, nrays, seed, device):
    import torch
    from sloth_b200 import workloads
    ne = workloads.kolmogorov_box(n, L=L, mean=1e25, rms=0.2, seed=seed, device=device)
    rays = workloads.gaussian_beam(nrays, waist=1.5e-3, L=L, seed=seed + 1, device=device)
    torch.cuda.synchronize()
    return ne, rays


# ---------------------------------------------------------------------------
# reference arm: the oracle's C restatement of the reference on host cores
# ---------------------------------------------------------------------------
def cpu_sample(ne_host, rays_host, spacing, omega, dtau, n_steps, seconds, threads=0):
    """The bounded CPU sample of the workload: the first m rays of the beam, all
    their steps, with m sized from a short probe so that one trace of the
    sample takes about `seconds` on the host cores. Returns (run, m, threads),
    run() tracing the sample once and returning its ray-step count."""
    from oracle import oracle_c
    from oracle import ref_restated as rr
    grid = rr.Grid(ne_host.astype(np.float64), (-L / 2,) * 3, spacing, omega, Te=TE, Z=ZION)
    thr = threads or oracle_c.threads()
    kw = dict(dtau=dtau, first_save=n_steps, save_every=1, n_saves=1, project=True, plane=L / 2,
              inv_brems=True, threads=thr, want_state=False)
    probe = min(rays_host.shape[1], 256 * thr)
    t0 = time.perf_counter()
    r = oracle_c.trace_rays(grid, rays_host[:, :probe], **kw)
    dt = time.perf_counter() - t0
    per_ray_s = dt / probe
    m = int(min(rays_host.shape[1], max(probe, seconds / per_ray_s)))
    sub = np.ascontiguousarray(rays_host[:, :m])

    def run():
        return oracle_c.trace_rays(grid, sub, **kw)["total_steps"]
    run.grid = grid
    return run, m, thr


def cpu_oracle_rate(ne_host, rays_host, spacing, omega, dtau, n_steps, seconds, threads=0):
    """Time the oracle's FP64 C restatement on the bounded sample once;
    returns (ray-steps/s, sample description, threads, total_steps)."""
    run, m, thr = cpu_sample(ne_host, rays_host, spacing, omega, dtau, n_steps, seconds, threads)
    t0 = time.perf_counter()
    steps = run()
    dt = time.perf_counter() - t0
    return steps / dt, f"first {m} rays of the 1e7-ray beam, all steps", thr, steps, run.grid


def run_reference(args):
    """The reference arm: the oracle's FP64 C restatement of the reference
    propagator on every host core, each step one trace of the same bounded
    sample the sloth arm's cpu_baseline leg times (the first m rays of the
    beam, all steps), m sized so that the W + K steps take about three
    minutes (at most 15 s per step)."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from sloth_b200 import runtime, workloads
    from sloth_b200.core import physics
    n = args.n
    h = L / (n - 1)
    ne = workloads.kolmogorov_box(n, L=L, mean=1e25, rms=0.2, seed=args.seed, device="cpu").numpy()
    rays = workloads.gaussian_beam(int(args.rays), waist=1.5e-3, L=L, seed=args.seed + 1).double().numpy()
    omega = physics.omega_of(LWL)
    sched = runtime.schedule_times([math.sqrt(8.0) * L], (h, h, h))
    per_step_s = min(args.cpu_seconds, 180.0 / max(1, args.steps + args.warmup))
    run, m, thr = cpu_sample(ne, rays, (h, h, h), omega, sched.dtau, sched.first_save, per_step_s)
    times, steps = [], []
    for i in range(args.warmup + args.steps):
        t0 = time.perf_counter()
        st = run()
        dt = time.perf_counter() - t0
        if i >= args.warmup:
            times.append(dt)
            steps.append(st)
    value = float(np.sum(steps) / np.sum(times))
    sample = f"first {m} rays of the {int(args.rays):.0e}-ray beam, all steps, traced once per step"
    line = {
        "impl": "reference", "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": args.gpus,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * float(np.mean(times)),
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
        "config": {"workload": f"{n}^3 Kolmogorov turbulent box (mean 1e19 cm^-3, 20% RMS), {int(args.rays):.0e}-ray "
                               f"3 mm Gaussian beam, 532 nm, Te=20 eV, Z=1; each step the {m}-ray sample",
                   "integrator": "fixed-step 4th-order Runge-Kutta-Nystrom, ds = h/2",
                   "field_samples_per_ray_step": 3,
                   "note": "the reference (JAX/diffrax) cannot be installed on this image; its CPU path is "
                           "stood in for by the oracle's FP64 C restatement (the tracers' method)"},
        "cpu_baseline": {"value": value, "unit": UNIT, "cores": thr, "kind": "port", "sample": sample},
        "e2e": {"value": value, "unit": UNIT, "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------------------
# serving leg: 2000 requests, Poisson arrivals at 200/s, grids {64..384}^3
# (sinusoid or Kolmogorov by a fair coin), lognormal ray counts (median 2e5,
# sigma 1, clipped to [1e4, 4e6]), 120 GB admission budget
# ---------------------------------------------------------------------------
def run_serving(args):
    import torch
    from sloth_b200 import serving
    reqs = serving.request_stream(args.serving_requests, rate=200.0, seed=args.seed)
    fields = {}
    for r in reqs:
        k = serving.grid_key(r.kind, r.n, r.field_seed)
        if k not in fields:
            fields[k] = serving.field_for(r.kind, r.n, r.field_seed)
    torch.cuda.synchronize()
    out = {}
    # a first saturated replay warms the process's caching allocators (pinned
    # result buffers, request ray tensors) and is not reported; the measured
    # saturated replay and the live stream then see a warm server, as a
    # deployed one runs (the first replay's GPU sat idle 10-20% of its span
    # on those first-use host costs)
    with serving.RayServer(120 << 30) as srv:
        serving.replay(srv, reqs, fields=fields, realtime=False)
    with serving.RayServer(120 << 30) as srv:
        sat = serving.replay(srv, reqs, fields=fields, realtime=False)
    with serving.RayServer(120 << 30) as srv:
        live = serving.replay(srv, reqs, fields=fields, realtime=True)
    out = {"requests": live["requests"], "rate_per_s": 200.0, "p50_ms": live["p50_ms"], "p99_ms": live["p99_ms"],
           "mean_ms": live["mean_ms"], "ray_steps_per_s": live["ray_steps_per_s"], "ray_steps": live["ray_steps"],
           "seconds": live["seconds"],
           "saturated_ray_steps_per_s": sat["ray_steps_per_s"], "saturated_seconds": sat["seconds"],
           "iterations": live["stats"]["iterations"], "grid_packs": live["stats"]["grid_packs"],
           "gpu_busy_frac": live["stats"]["gpu_busy_ms"] / max(live["stats"]["gpu_span_ms"], 1e-9),
           "host_loop_max_ms": live["host_loop_max_ms"],
           "saturated_gpu_busy_frac": sat["stats"]["gpu_busy_ms"] / max(sat["stats"]["gpu_span_ms"], 1e-9),
           "budget_bytes": live["stats"]["budget_bytes"],
           "stream": f"{args.serving_requests} requests, Poisson 200/s, grids {{64,128,192,256,384}}^3 "
                     "sinusoid|Kolmogorov, "
                     "lognormal rays median 2e5 sigma 1 in [1e4, 4e6], 120 GB budget; latency = arrival to "
                     "results in pinned host memory; a first saturated replay (every request queued at once) "
                     "warms the host allocators and is not reported, then the saturated replay and the live "
                     "stream are measured"}
    del fields
    torch.cuda.empty_cache()
    return out


# ---------------------------------------------------------------------------
# diagnostics: the single-lens shadowgraphy chain and the transmission-
# weighted 3448 x 2574 histogram of every traced ray, one K6 launch
# ---------------------------------------------------------------------------
def run_diagnostics(outs):
    import torch
    from sloth_b200.processing import diagnostics as dg
    jv, amp = outs["jones"][-1], outs["amp"][-1]
    n = int(jv.shape[1])
    L = 400.0
    ops = [(dg.TRAVEL, 3 * L / 4, 0, 0), (dg.CIRCULAR_APERTURE, 25.0, 0, 0), (dg.LENS, L / 2, L / 2, 0),
           (dg.TRAVEL, 3 * L / 2, 0, 0)]
    H = torch.zeros((2574, 3448), dtype=torch.float64, device=jv.device)
    stream = torch.cuda.current_stream()
    times = []
    for it in range(8):
        H.zero_()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(stream)
        dg.run_optics(jv, ops, weights=amp, pos_scale=1e3, hist=(3448, 2574, (-9.0, 9.0), (-6.75, 6.75)), out_hist=H)
        e1.record(stream)
        torch.cuda.synchronize()
        if it >= 3:
            times.append(e0.elapsed_time(e1))
    ms = float(np.median(times))
    return {"workload": f"Shadowgraphy.single_lens_solve + histogram (3448 x 2574, transmission weights) of the "
                        f"{n:.0e} traced rays", "ms": ms, "rays_per_s": n / (ms / 1e3),
            "binned_weight": float(H.sum()), "launches": 1}


# ---------------------------------------------------------------------------
# adjoint: d loss / d ne for a 256^2 detector image of 1e6 rays through a
# 128^3 FP32 Kolmogorov grid (400 steps, checkpoints every 20, 2-pixel
# splat); loss = ||I - I_target||^2 with I_target from another seeded field
# ---------------------------------------------------------------------------
def run_adjoint(args):
    import torch
    from sloth_b200 import adjoint, workloads
    n, nrays = 128, 1_000_000
    h = L / (n - 1)
    spec = adjoint.box_detector(L, n_px=256, sigma_px=2.0, n_steps=400, ckpt_every=20)
    ne_t = workloads.kolmogorov_box(n, L=L, mean=1e25, rms=0.2, seed=args.seed + 41, device="cuda")
    ne = workloads.kolmogorov_box(n, L=L, mean=1e25, rms=0.2, seed=args.seed + 42, device="cuda")
    rays = workloads.gaussian_beam(nrays, waist=1.5e-3, L=L, seed=args.seed + 43, device="cuda")
    kw = dict(origin=(-L / 2,) * 3, spacing=(h,) * 3, lwl=LWL)
    with torch.no_grad():
        target = adjoint.detector_image(ne_t, rays, spec, **kw, precision="f64").double()
    stream = torch.cuda.current_stream()
    fwd_ms, bwd_ms, steps = [], [], 0
    for it in range(3 + max(args.steps, 3)):
        x = ne.detach().requires_grad_(True)
        st = {}
        e0, e1, e2 = (torch.cuda.Event(enable_timing=True) for _ in range(3))
        e0.record(stream)
        img = adjoint.detector_image(x, rays, spec, **kw, precision="f32", stats=st)
        e1.record(stream)
        loss = (img.double() - target).pow(2).sum()
        loss.backward()
        e2.record(stream)
        torch.cuda.synchronize()
        if it >= 3:
            fwd_ms.append(e0.elapsed_time(e1))
            bwd_ms.append(e1.elapsed_time(e2))
            steps = int(st["ray_steps"][0])
    g32 = x.grad.double()
    # central differences of the FP64 forward at 16 voxels of the beam's core
    rng = np.random.default_rng(args.seed)
    c = n // 2
    vox = [tuple(int(v) for v in rng.integers(c - 30, c + 30, 3)) for _ in range(16)]
    ne64, r64 = ne.double(), rays.double()

    def loss_at(v):
        with torch.no_grad():
            return float((adjoint.detector_image(v, r64, spec, **kw, precision="f64") - target).pow(2).sum())
    fd, ad = [], []
    for v in vox:
        eps = 1e-3 * float(ne64[v])
        y = ne64.clone()
        y[v] += eps
        lp = loss_at(y)
        y[v] -= 2 * eps
        fd.append((lp - loss_at(y)) / (2 * eps))
        ad.append(float(g32[v]))
    fd, ad = np.array(fd), np.array(ad)
    fms, bms = float(np.median(fwd_ms)), float(np.median(bwd_ms))
    out = {"workload": "128^3 FP32 Kolmogorov grid, 1e6 rays (3 mm Gaussian beam), 400 steps, checkpoints "
                       "every 20, 256^2 detector, 2-pixel Gaussian splat, L = ||I - I_target||^2",
           "ray_steps": steps, "forward_ms": fms, "backward_ms": bms,
           "forward_ray_steps_per_s": steps / (fms / 1e3), "backward_ray_steps_per_s": steps / (bms / 1e3),
           "grad_vs_fd": {"voxels": len(vox), "max_abs_err_rel_to_max": float(np.abs(ad - fd).max() / np.abs(fd).max()),
                          "fd": "central, eps = 1e-3 ne, FP64 forward"},
           "timing": "CUDA events; forward = pack + Morton pre-pass + trace + splat; backward = loss grad + "
                     "adjoint kernel + pack adjoint"}
    del ne_t, ne, rays, target, g32
    torch.cuda.empty_cache()
    return out


# ---------------------------------------------------------------------------
# error of the FP32 split kernel against the all-FP64 port (all rays)
# ---------------------------------------------------------------------------
def _q(t, p):
    import torch
    t = t.float() if t.numel() < 2 ** 24 else t[:: max(1, t.numel() // 2 ** 23)].float()
    return float(torch.quantile(t, p))


def accuracy(o32, o64, spread=None):
    """Per-output error of the FP32 kernel against the FP64 port on every ray;
    far-face rays (those crossing the far face inside the box's transverse
    extent) and side-exit rays (the others, leaving or missing the box
    through a side face at grazing incidence) are also reported apart.
    `spread` is the FP64 port's own change when its input positions move by
    one FP32 ulp (amp and phase, per ray): the conditioning of each ray."""
    j32, j64 = o32["jones"][-1].double(), o64["jones"][-1].double()
    ok = (o32["status"] != 2) & (o64["status"] != 2)
    far = ok & (j64[0].abs() <= L / 2) & (j64[2].abs() <= L / 2)
    side = ok & ~far
    dpos = torch_max(j32[0], j64[0], j32[2], j64[2])[ok] / L
    dang = torch_max(j32[1], j64[1], j32[3], j64[3])[ok]
    ph64 = o64["phase"][-1]
    scale = float(ph64[ok].abs().max())
    dph = (o32["phase"][-1] - ph64).abs()
    damp = (o32["amp"][-1].double() - o64["amp"][-1].double()).abs()
    acc = {"position_rel_L_max": float(dpos.max()), "position_rel_L_p99": _q(dpos, 0.99),
           "angle_abs_max_rad": float(dang.max()), "angle_abs_p99_rad": _q(dang, 0.99),
           "phase_abs_max_rad": float(dph[ok].max()), "phase_max_abs_rad": scale,
           "phase_rel_max": float(dph[ok].max()) / scale,
           "phase_rel_max_far_face": float(dph[far].max()) / scale,
           "phase_rel_p99": _q(dph[ok] / scale, 0.99),
           "amp_abs_max": float(damp[ok].max()), "amp_abs_max_far_face": float(damp[far].max()),
           "amp_abs_p99": _q(damp[ok], 0.99),
           "rays_compared": int(ok.sum()), "rays_far_face": int(far.sum()), "rays_side_exit": int(side.sum()),
           "status_mismatch": int((o32["status"] != o64["status"]).sum())}
    if side.any():
        acc["amp_abs_max_side_exit"] = float(damp[side].max())
        acc["phase_rel_max_side_exit"] = float(dph[side].max()) / scale
    if spread is not None and side.any():
        s_amp, s_ph = spread
        big = side & (damp > 1e-6)
        acc["fp64_one_ulp_input_spread"] = {
            "what": "the FP64 port's own change when the rays' x and y move by one FP32 ulp (max over +/-)",
            "amp_abs_max_side_exit": float(s_amp[side].max()), "amp_abs_max_far_face": float(s_amp[far].max()),
            "phase_rel_max_side_exit": float(s_ph[side].max()) / scale,
            "phase_rel_max_far_face": float(s_ph[far].max()) / scale,
            "side_exit_rays_amp_err_above_1e-6": int(big.sum()),
            "their_fp64_spread_min": float(s_amp[big].min()) if big.any() else None,
            "side_exit_rays_spread_above_1e-6": int((side & (s_amp > 1e-6)).sum())}
    return acc


def torch_max(a1, b1, a2, b2):
    import torch
    return torch.maximum((a1 - b1).abs(), (a2 - b2).abs())


# ---------------------------------------------------------------------------
# B200 arm
# ---------------------------------------------------------------------------
def run_sloth(args):
    import torch
    from sloth_b200 import _capi, runtime
    from sloth_b200.core import physics
    from sloth_b200.core.propagator import solve

    from sloth_b200 import replicas
    world, rank, local = replicas.rank_env()
    torch.cuda.set_device(local)
    dev = torch.device("cuda", local)
    dist = replicas.init(world, dev, "nccl")

    n, nrays = args.n, int(args.rays)
    h = L / (n - 1)
    omega = physics.omega_of(LWL)
    seed = replicas.rank_seed(args.seed, rank)
    ne, rays = make_workload(n, nrays, seed, dev)
    grid = runtime.pack_grid(ne, (-L / 2,) * 3, (h, h, h), omega, precision="f32")
    sched = runtime.schedule_times([math.sqrt(8.0) * L], (h, h, h))
    stream = torch.cuda.current_stream()
    outs = {}
    ws = None

    def step(ev=None):
        return runtime.trace(grid, rays, sched, project=True, plane=L / 2, inv_brems=True, Te=TE, Z=ZION,
                             want_status=True, want_steps=False, outputs=outs, events=ev)

    def barrier():
        replicas.barrier(dist)

    for _ in range(args.warmup):
        step()
    torch.cuda.synchronize()
    barrier()
    evs = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    kev = [(torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)) for _ in range(args.steps)]
    for a, b in kev:
        a.record()
        b.record()
    torch.cuda.synchronize()
    launches0 = _capi.launch_count()
    with ClockSampler(local) as clk:
        torch.cuda.synchronize()
        barrier()
        for i in range(args.steps):
            evs[i][0].record(stream)
            step(kev[i])
            evs[i][1].record(stream)
        torch.cuda.synchronize()
        barrier()
    launches = _capi.launch_count() - launches0
    per_step_ms = [a.elapsed_time(b) for a, b in evs]
    kernel_ms = [a.elapsed_time(b) for a, b in kev]
    total_ms = evs[0][0].elapsed_time(evs[-1][1])
    ray_steps = int(outs["total_steps"][0])
    total_ms, all_ray_steps = replicas.job_totals(dist, total_ms, ray_steps, dev)
    value = all_ray_steps * args.steps / (total_ms / 1e3)
    f32_out = {k: v.clone() for k, v in outs.items()}

    # ---- all-FP64 port of the same kernel on the same workload -------------
    tkw = dict(project=True, plane=L / 2, inv_brems=True, Te=TE, Z=ZION, want_steps=False)

    def timed(g, r, reps, integ, outputs):
        """Mean ms per trace and mean trace-kernel ms over `reps` traces (after one untimed)."""
        runtime.trace(g, r, sched, outputs=outputs, integrator=integ, **tkw)
        torch.cuda.synchronize()
        k2 = (torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True))
        k2[0].record()
        k2[1].record()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        ktimes = []
        e0.record(stream)
        for _ in range(reps):
            runtime.trace(g, r, sched, outputs=outputs, integrator=integ, events=k2, **tkw)
            e1.record(stream)
            torch.cuda.synchronize()
            ktimes.append(k2[0].elapsed_time(k2[1]))
        return e0.elapsed_time(e1) / reps, float(np.mean(ktimes))

    fp64 = None
    acc = None
    rk4 = None
    phase_first = None
    phase_ref = None
    if not args.no_fp64 and world == 1:
        g64 = runtime.pack_grid(ne, (-L / 2,) * 3, (h, h, h), omega, precision="f64")
        r64 = rays.double()
        o64 = {}
        ms64, kms64 = timed(g64, r64, 2, "rkn", o64)
        rs64 = int(o64["total_steps"][0])
        fp64 = {"value": rs64 / (ms64 / 1e3), "ms_per_step": ms64, "kernel_ms": kms64, "ray_steps": rs64}
        # the FP64 port's sensitivity to a one-ulp (FP32) move of the input positions
        s_amp = s_ph = None
        for d in (1.0, -1.0):
            rp = rays.clone()
            rp[0:2] = torch.nextafter(rp[0:2], torch.full_like(rp[0:2], d * math.inf))
            op = runtime.trace(g64, rp.double(), sched, **tkw)
            da = (op["amp"][-1] - o64["amp"][-1]).abs()
            dp = (op["phase"][-1] - o64["phase"][-1]).abs()
            s_amp = da if s_amp is None else torch.maximum(s_amp, da)
            s_ph = dp if s_ph is None else torch.maximum(s_ph, dp)
            del op
        acc = accuracy(f32_out, o64, (s_amp, s_ph))
        del s_amp, s_ph
        phase_first = {"rays": 100, "f64": o64["phase"][-1][:100].cpu().numpy(),
                       "f32": f32_out["phase"][-1][:100].cpu().numpy()}
        if not args.no_rk4:
            # the classical RK4 step the workload descriptions name: four field
            # samples per ray-step instead of three, FP32 split and FP64 port
            o4 = {}
            ms4, kms4 = timed(grid, rays, 3, "rk4", o4)
            rs4 = int(o4["total_steps"][0])
            o4_64 = {}
            ms4_64, kms4_64 = timed(g64, r64, 1, "rk4", o4_64)
            rk4 = {"integrator": "classical RK4, ds = h/2", "field_samples_per_ray_step": 4,
                   "value": rs4 / (ms4 / 1e3), "ms_per_step": ms4, "kernel_ms": kms4, "ray_steps": rs4,
                   "fp64_port": {"value": int(o4_64["total_steps"][0]) / (ms4_64 / 1e3), "ms_per_step": ms4_64,
                                 "kernel_ms": kms4_64},
                   "speedup_of_fp32": ms4_64 / ms4,
                   "fp32_vs_fp64": accuracy(o4, o4_64)}
            # the two integrators' FP64 results differ by their truncation error
            j4, jn = o4_64["jones"][-1], o64["jones"][-1]
            rk4["rkn_vs_rk4_fp64_position_rel_L_max"] = float(
                torch_max(j4[0], jn[0], j4[2], jn[2]).max() / L)
            del o4, o4_64
        del g64, r64, o64

    # ---- end to end through the public API (host buffers) -------------------
    e2e = None
    if not args.no_e2e:
        import types
        ne_host = ne.cpu().pin_memory()
        rays_host = rays.cpu().pin_memory()
        c1 = np.linspace(-L / 2, L / 2, n).astype(np.float32)
        dom = types.SimpleNamespace(ne=ne_host, x=c1, y=c1, z=c1, probing_direction='z',
                                    lengths=np.array([L] * 3, np.float32), dims=np.array([n] * 3),
                                    Np_total=None, inv_brems=True, Te=np.float32(TE), Z=np.float32(ZION),
                                    region_count=1, ray_batch_count=1)
        res = None
        # warm-up calls also fill PyTorch's caching host allocator with the
        # pinned result buffers (two sets: the previous result is still held)
        for _ in range(max(args.warmup, 3)):
            res = solve(rays_host, dom, L, lwl=LWL, verbose=False, detector_plane=L / 2, return_extras=True)
        torch.cuda.synchronize()
        reps = max(2, min(args.steps, 3))
        barrier()
        t0 = time.perf_counter()
        for _ in range(reps):
            res = solve(rays_host, dom, L, lwl=LWL, verbose=False, detector_plane=L / 2, return_extras=True)
        torch.cuda.synchronize()
        dt = (time.perf_counter() - t0) / reps
        rf, amp, _, ex = res
        d2h = rf.nbytes + amp.nbytes + ex["phase"].nbytes + ex["status"].nbytes + ex["steps"].nbytes
        h2d = ne_host.numel() * ne_host.element_size() + rays_host.numel() * rays_host.element_size()
        # solve() returns host arrays, so each call ends synchronised; the
        # per-rank time is host-measured and the job's is the max over ranks
        dt_ms, steps_all = replicas.job_totals(dist, dt * 1e3, float(ex["total_steps"]), dev)
        e2e = {"value": steps_all / (dt_ms / 1e3), "unit": UNIT, "h2d_bytes_per_step": int(h2d),
               "d2h_bytes_per_step": int(d2h), "ms_per_step": dt_ms,
               "path": "sloth_b200.core.propagator.solve (pinned host ne and rays, numpy outputs)"}

    # ---- diagnostics: shadowgraphy of the traced rays on a KAF-8300 ---------
    diag = None
    if not args.no_diagnostics and world == 1:
        diag = run_diagnostics(f32_out)

    # ---- serving: the mixed request stream (p50/p99 latency) ----------------
    serve = None
    if not args.no_serving and world == 1:
        serve = run_serving(args)

    # ---- adjoint: gradient of a detector-image loss -------------------------
    adj = None
    if not args.no_adjoint and world == 1:
        adj = run_adjoint(args)

    # ---- CPU baseline (rank 0, N = 1) ---------------------------------------
    cpu = None
    if rank == 0 and world == 1 and not args.no_cpu:
        rays_host = rays.double().cpu().numpy()
        rate, sample, thr, _, ogrid = cpu_oracle_rate(ne.cpu().numpy(), rays_host, (h, h, h), omega, sched.dtau,
                                                      sched.first_save, args.cpu_seconds)
        cpu = {"value": rate, "unit": UNIT, "cores": thr, "kind": "port", "sample": sample}
        if phase_first is not None:
            # the kernels' phase against the oracle's reference semantics (the
            # legacy solver's interpolated n, pinned to its own phase()) on
            # the first rays of the beam
            from oracle import ref_restated as rr
            k = phase_first["rays"]
            ref = rr.trace_rays(ogrid, rays_host[:, :k], dtau=sched.dtau, first_save=sched.first_save,
                                save_every=1, n_saves=1, project=True, plane=L / 2,
                                phase_mode="reference")["phase"][-1]
            dens = rr.trace_rays(ogrid, rays_host[:, :k], dtau=sched.dtau, first_save=sched.first_save,
                                 save_every=1, n_saves=1, project=True, plane=L / 2,
                                 phase_mode="density")["phase"][-1]
            sc = float(np.abs(ref).max())
            phase_ref = {"rays": k, "oracle": "numpy FP64, phase_mode 'reference' (interpolated n - 1)",
                         "fp64_port_rel_max": float(np.abs(phase_first["f64"] - ref).max() / sc),
                         "fp32_rel_max": float(np.abs(phase_first["f32"] - ref).max() / sc),
                         "density_form_gap_rel_max": float(np.abs(dens - ref).max() / sc)}
        del ogrid

    if rank == 0:
        hbm_peak, peak_kind = measured_peaks()
        kms = float(np.mean(kernel_ms))
        traffic = committed_traffic(args)
        lane_ops, lane_ops_where = committed_lane_ops()
        clocks = clk.summary()
        sms = torch.cuda.get_device_properties(dev).multi_processor_count
        sm_mhz = (clocks or {}).get("sm_mhz") or 1965.0
        # the FP32 pipe: 128 FP32 lanes per SM per clock (FFMA2 occupies both FMA pipes)
        pipe_peak = sms * 128 * sm_mhz * 1e6 / 1e12
        pipe_achieved = ray_steps * lane_ops / (kms / 1e3) / 1e12 if lane_ops else None
        gather_gbs = ray_steps * BYTES_PER_RAY_STEP / (kms / 1e3) / 1e9
        if adj:
            # the adjoint backward against the same FP32-pipe peak (its kernel is issue-bound; see
            # the profile the lane-operation count comes from)
            bl, bl_where = committed_backward_lane_ops()
            if bl:
                ach = adj["ray_steps"] * bl / (adj["backward_ms"] / 1e3) / 1e12
                adj["backward_roofline"] = {"bound": "fp32_pipe", "achieved": ach, "peak": pipe_peak,
                                            "unit": "T FP32 lane-ops/s", "frac": ach / pipe_peak,
                                            "lane_ops_per_ray_step": bl, "lane_ops_from": bl_where,
                                            "note": "backward_ms includes the loss gradient and the pack "
                                                    "adjoint; the peak uses the trace's sampled SM clock"}
        line = {
            "metric": METRIC, "value": value, "unit": UNIT, "n_gpus": world, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": total_ms / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": {"workload": f"{n}^3 Kolmogorov turbulent box (mean 1e19 cm^-3, 20% RMS, k^-11/3), "
                                   f"{nrays:.0e} rays, 3 mm Gaussian beam along +z, 532 nm, Te=20 eV, Z=1, "
                                   "detector plane z=+2.5 mm",
                       "integrator": "fixed-step 4th-order Runge-Kutta-Nystrom, ds = h/2",
                       "field_samples_per_ray_step": 3,
                       "unit_of_work": "one ray-step = one fixed step of one ray inside or near the grid; it "
                                       "samples the field 3 times (RK4 would sample it 4 times)",
                       "l2": f"inputs larger than L2 ({n ** 3 * 16 / 1e9:.2f} GB packed grid, "
                             f"{nrays * 24 / 1e6:.0f} MB rays)",
                       "precision": "FP32 state with compensated sums, FP64 phase accumulator, Kahan FP32 optical "
                                    "depth; the phase integrand n - 1 is interpolated from the packed grid",
                       "seed": args.seed, "ray_steps_per_trace": ray_steps},
            "latency_ms": {"p50": float(np.percentile(per_step_ms, 50)), "p99": float(np.percentile(per_step_ms, 99)),
                           "what": "one 1e7-ray trace per request"},
            "roofline": {"bound": "fp32_pipe", "achieved": pipe_achieved, "peak": pipe_peak,
                         "unit": "T FP32 lane-ops/s",
                         "frac": (pipe_achieved / pipe_peak) if pipe_achieved else None,
                         "traffic": traffic,
                         "peak_kind": f"{sms} SMs x 128 FP32 lanes x {sm_mhz:.0f} MHz (median SM clock sampled "
                                      "in the timed region)",
                         "lane_ops_per_ray_step": lane_ops, "lane_ops_from": lane_ops_where,
                         "kernel": "trace_kernel<PolF32>", "kernel_ms": kms,
                         "hbm": {"peak_gbs": hbm_peak, "peak_kind": f"{peak_kind} HBM copy bandwidth",
                                 "dram_achieved_gbs": (traffic / (kms / 1e3) / 1e9) if traffic else None,
                                 "dram_frac": (traffic / (kms / 1e3) / 1e9 / hbm_peak) if traffic else None,
                                 "logical_gather_bytes_per_ray_step": BYTES_PER_RAY_STEP,
                                 "logical_gather_gbs": gather_gbs},
                         "note": "achieved = ray-steps/s x FP32 lane-operations per ray-step (ncu instruction "
                                 "mix: scalar FFMA/FADD/FMUL + 2 x paired FFMA2/FADD2/FMUL2); the trace is bound "
                                 "by its FP32 pipes, not memory: DRAM traffic (traffic, from ncu) is ~1.5 B per "
                                 "ray-step against 384 logical gather bytes, which a register cell cache and L1 "
                                 "serve"},
            "cpu_baseline": cpu,
            "e2e": e2e,
            "gpu_launches": int(launches),
            "clocks": clocks,
            "fp64_port": fp64,
            "fp32_vs_fp64": acc,
            "phase_vs_reference_semantics": phase_ref,
            "rk4": rk4,
            "serving": serve,
            "adjoint": adj,
            "diagnostics": diag,
        }
        if fp64:
            line["fp64_port"]["speedup_of_fp32"] = value / world / fp64["value"]
        print(json.dumps(line), flush=True)
    replicas.finish(dist)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
    else:
        run_sloth(args)


if __name__ == "__main__":
    main()
