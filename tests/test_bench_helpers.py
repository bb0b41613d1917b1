"""Host-side helpers of bench.py that feed its roofline object: the DRAM
traffic per trace launch comes from the committed ncu summary of the 512^3 /
1e7-ray workload (and from nowhere for any other workload), it equals that
summary's read + write bytes, and it stays within a few bytes per ray-step of
the ray-steps that summary counts."""
import argparse
import importlib.util
import os
import re

from conftest import ROOT


def _bench():
    spec = importlib.util.spec_from_file_location("bench_under_test", os.path.join(ROOT, "bench.py"))
    mod = importlib.util.module_from_spec(spec)
    spec.loader.exec_module(mod)
    return mod


def test_committed_traffic_matches_the_profile():
    bench = _bench()
    args = argparse.Namespace(n=512, rays=1e7, seed=2024)
    traffic = bench.committed_traffic(args)
    text = open(os.path.join(ROOT, "profiles", "trace_kernel_kolmogorov512_1e7.md")).read()

    def count(label):
        m = re.search(r"\| " + re.escape(label) + r" \| ([0-9,]+)", text)
        return int(m.group(1).replace(",", ""))

    rd, wr, steps = count("dram__bytes_read.sum"), count("dram__bytes_write.sum"), count("ray-steps in the launch")
    assert traffic == rd + wr
    assert 0.5 < traffic / steps < 4.0          # a few bytes per ray-step, far below the 384 logical


def test_committed_traffic_only_for_the_profiled_workload():
    bench = _bench()
    for n, rays, seed in ((256, 1e6, 2024), (512, 1e6, 2024), (512, 1e7, 7)):
        assert bench.committed_traffic(argparse.Namespace(n=n, rays=rays, seed=seed)) is None


def test_logical_bytes_per_ray_step():
    """Three stage samples of eight 16-byte voxels."""
    assert _bench().BYTES_PER_RAY_STEP == 3 * 8 * 16


def test_committed_lane_ops_match_the_instruction_mix():
    """The FP32 lane-operations per ray-step that the roofline uses equal the
    summary's scalar FP32 count plus two lanes per paired instruction."""
    ops, where = _bench().committed_lane_ops()
    text = open(os.path.join(ROOT, "profiles", "trace_kernel_kolmogorov512_1e7.md")).read()
    m = re.search(r"\| FFMA2 / FADD2 / FMUL2 \(two FP32 lanes each\) \| ([0-9.]+) / ([0-9.]+) / ([0-9.]+)", text)
    s = re.search(r"\| FFMA / FADD / FMUL \| ([0-9.]+) / ([0-9.]+) / ([0-9.]+)", text)
    paired = sum(float(x) for x in m.groups())
    scalar = sum(float(x) for x in s.groups())
    assert abs(ops - (scalar + 2 * paired)) < 0.5
    assert where
