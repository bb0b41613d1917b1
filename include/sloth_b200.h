/*
 * sloth_b200.h — C ABI of the B200 (sm_100a) ray-propagation library.
 *
 * The library replaces the hot path of SLOTH's JAX propagator: the grid-level
 * precompute, the trilinear interpolator, the RHS and the vmapped diffrax solve,
 * and the Jones-vector projection at the end of a trace. Every entry point:
 *   - returns SLOTH_OK (0) or a negative SLOTH_ERR_* code (never throws, never
 *     exits, never aborts); sloth_strerror() turns a code into text;
 *   - takes caller-owned DEVICE buffers as plain pointers (e.g. torch
 *     tensor.data_ptr()); nothing here allocates device memory except the
 *     request server, which owns one arena sized by its HBM budget;
 *   - launches asynchronously on the caller's CUDA stream (`stream` is a
 *     cudaStream_t passed as void*; NULL = the legacy default stream).
 *
 * Units: positions in metres, velocities in m/s, densities in m^-3, time as
 * path length tau = c*t in metres. Ray arrays are row-major (6, N):
 * rows x, y, z, vx, vy, vz, exactly the layout of the reference's Beam.s0.
 */
#ifndef SLOTH_B200_H
#define SLOTH_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define SLOTH_ABI_VERSION 3

/* ---- return codes ------------------------------------------------------ */
#define SLOTH_OK                        0
#define SLOTH_ERR_INVALID_ARGUMENT     -1
#define SLOTH_ERR_NULL_POINTER         -2
#define SLOTH_ERR_MISALIGNED           -3
#define SLOTH_ERR_WORKSPACE_TOO_SMALL  -4
#define SLOTH_ERR_CUDA                 -5
#define SLOTH_ERR_NO_DEVICE            -6
#define SLOTH_ERR_TOO_LARGE            -7
#define SLOTH_ERR_OUT_OF_MEMORY        -8
#define SLOTH_ERR_NOT_FOUND            -9
#define SLOTH_ERR_BUSY                -10
#define SLOTH_ERR_UNSUPPORTED_DEVICE  -11

/* ---- per-ray status written by the tracers ---------------------------- */
#define SLOTH_RAY_EXITED          0  /* left the grid and can never re-enter   */
#define SLOTH_RAY_INSIDE_AT_END   1  /* still inside the grid at the last save */
#define SLOTH_RAY_NONFINITE       2  /* state became NaN/Inf; outputs are NaN  */

/* Uniform grid: point i of axis a sits at origin[a] + i*spacing[a].
 * Voxel (i, j, k) is element (i*n[1] + j)*n[2] + k (C order, z fastest),
 * which is numpy's layout of an (nx, ny, nz) array. */
typedef struct SlothGridDesc {
    int32_t n[3];        /* points per axis, each >= 2                        */
    int32_t reserved;    /* must be 0                                         */
    double  origin[3];   /* coordinate of point 0 per axis (m)                */
    double  spacing[3];  /* uniform spacing per axis (m), > 0                 */
} SlothGridDesc;

/* Integration methods of the tracers (SlothTraceParams::integrator). */
#define SLOTH_INTEGRATOR_RKN 0   /* Nystrom's 4th-order Runge-Kutta-Nystrom: 3 field samples per step */
#define SLOTH_INTEGRATOR_RK4 1   /* classical RK4 of the first-order system: 4 field samples per step */

/* Fixed-step schedule and physics of one trace (fourth-order Runge-Kutta-
 * Nystrom steps, three field samples per step, or classical RK4 steps, four
 * samples; `integrator`).
 * All steps have the same length dtau (tau = c*t, metres). Save j (0-based)
 * is taken after step first_save + j*save_every; the trace ends at the last
 * save. Rays that have left the grid for good are advanced to later saves by
 * exact straight-line drift (the RHS is zero outside the grid). */
typedef struct SlothTraceParams {
    double  omega;            /* laser angular frequency (rad/s)                    */
    double  dtau;             /* step length in c*t (m), > 0                        */
    int32_t first_save;       /* step index of save 0, >= 0                         */
    int32_t save_every;       /* steps between saves, >= 1 when n_saves > 1         */
    int32_t n_saves;          /* number of saves, 1 .. SLOTH_MAX_SAVES              */
    int32_t probing_axis;     /* 0 = x, 1 = y, 2 = z                                */
    int32_t project_to_plane; /* 0: Jones vector at the ray's current position
                                 (reference keep_current_plane=True); 1: the ray's
                                 straight line back-projected to `plane`
                                 (keep_current_plane=False, ne_extent = plane)      */
    int32_t inv_brems;        /* 1: accumulate inverse-bremsstrahlung optical depth */
    double  plane;            /* detector plane along probing_axis (m)              */
    double  kappa_q2;         /* kappa/c per (ne/nc)^2 with the Coulomb log factored
                                 out (1/m): 3.1e-5*Z*(nc_cc/omega)^2*Te^-1.5        */
    double  coulomb_log_w;    /* ln(v_the/(omega*b_min)): Coulomb log for ne < nc   */
    double  ope_ratio2;       /* (omega_pe/omega)^2 per unit ne/nc (NRL constants)  */
    double  q_max;            /* upper bound of ne/nc over the grid, or 0 if unknown;
                                 a bound selects faster exact paths (sub-critical
                                 kappa)                                           */
    double  q_min;            /* lower bound of ne/nc over the grid (0 for a density
                                 known to be >= 0). With q_max it bounds the ray's
                                 acceleration. Runs of steps that the bound proves
                                 interior skip the face test; when the bound also keeps
                                 every stage point of an interior step inside the grid,
                                 those steps skip the per-stage grid test as well
                                 (bitwise the same results in FP32, within 1e-12
                                 relative in FP64; fewer instructions). A value above
                                 the true minimum is an error of the caller. */
    int32_t integrator;       /* SLOTH_INTEGRATOR_RKN (0, default) or SLOTH_INTEGRATOR_RK4;
                                 the request server takes RKN steps only          */
    int32_t reserved;         /* must be 0                                          */
} SlothTraceParams;

#define SLOTH_MAX_SAVES 4096

/* Output buffers of a trace; element type follows the entry point
 * (float for *_f32, double for *_f64) unless stated. Arrays with a save axis
 * are [n_saves][rows][N] row-major. NULL skips an optional output. */
typedef struct SlothTraceOutputs {
    void*     jones;        /* [S][4][N] required: rows (pos1, angle1, pos2, angle2)
                               in the reference's ray_to_Jonesvector order          */
    void*     state;        /* [S][6][N] optional: x,y,z (m), vx,vy,vz (m/s)        */
    double*   phase;        /* [S][N] optional, always double: optical phase
                               integral of omega*(n-1) dt (rad)                     */
    void*     amp;          /* [S][N] optional: exp(-tau_ib); needs inv_brems       */
    uint8_t*  status;       /* [N] optional: SLOTH_RAY_*                            */
    int32_t*  steps;        /* [N] optional: steps taken before exit / end          */
    unsigned long long* total_steps; /* [1] optional device counter: sum of steps,
                               zeroed by the entry point before the launch          */
    void*     trace_event_begin; /* optional cudaEvent_t recorded on `stream` right
                               before the tracer kernel (after the sort pre-pass)   */
    void*     trace_event_end;   /* optional cudaEvent_t recorded right after it     */
} SlothTraceOutputs;

/* ---- library info ------------------------------------------------------ */
const char* sloth_strerror(int code);
int  sloth_abi_version(void);
/* Device properties of the current CUDA device. */
int  sloth_device_info(int* sm_count, int* cc_major, int* cc_minor);
/* Number of kernels this library has launched in this process. */
unsigned long long sloth_launch_count(void);

/* ---- K1: grid pack ------------------------------------------------------
 * Replaces precompute_gradients (src/core/propagator.py:39-93) and the
 * reference's per-grid kappa precompute (:116-164, folded into the tracer).
 * Writes one voxel-packed (q, dq/du, dq/dv, dq/dw) per grid point, where
 * q = ne * ne_scale (ne_scale = 1/nc) and d/du is the derivative per grid
 * cell: central differences inside, one-sided at the faces (jnp.gradient
 * semantics, :90-92). ne is float32 (ne_is_f64 = 0) or float64, C order.
 * grid_out must be 16-byte aligned (f32: float4) / 16-byte aligned (f64:
 * 2 x double2 per voxel). */
size_t sloth_grid_bytes(const SlothGridDesc* g, int real_bytes /* 4 or 8 */);
int sloth_grid_pack_f32(const SlothGridDesc* g, const void* ne, int ne_is_f64,
                        double ne_scale, void* grid_out, void* stream);
int sloth_grid_pack_f64(const SlothGridDesc* g, const void* ne, int ne_is_f64,
                        double ne_scale, void* grid_out, void* stream);
/* The trace layout, which the tracers (K2/K3) and the request server read:
 * as above, but channel 0 holds the refractive index minus one instead of
 * q, n - 1 = sqrt(1 - x) - 1 with x = ope_ratio2 * q = (omega_pe/omega)^2,
 * evaluated in FP64 as -x / (1 + sqrt(1 - x)) and -x where x > 1. The
 * tracers interpolate it for the optical phase, as the legacy solver
 * interpolates its n grid (src/legacy/full_solver.py:289, :342-345), and
 * rebuild q at the cell corners for the inverse-bremsstrahlung rate.
 * ope_ratio2 as in SlothTraceParams (> 0). */
int sloth_grid_pack_trace_f32(const SlothGridDesc* g, const void* ne, int ne_is_f64, double ne_scale,
                              double ope_ratio2, void* grid_out, void* stream);
int sloth_grid_pack_trace_f64(const SlothGridDesc* g, const void* ne, int ne_is_f64, double ne_scale,
                              double ope_ratio2, void* grid_out, void* stream);

/* ---- K0: trilinear sample -----------------------------------------------
 * Replaces RegularGridInterpolator (src/core/interpolator.py:15-105) on the
 * packed grid: for each point (3, N) row-major in metres, writes the four
 * interpolated channels (4, N): q and dq/du, dq/dv, dq/dw, with 0 outside
 * the grid (fill_value = 0, :85-87, :102-104). */
int sloth_sample_f32(const SlothGridDesc* g, const void* grid, const double* points,
                     int64_t n, float* out, void* stream);
int sloth_sample_f64(const SlothGridDesc* g, const void* grid, const double* points,
                     int64_t n, double* out, void* stream);

/* ---- K2/K3: tracers ------------------------------------------------------
 * Replace the vmapped diffrax solve of dsdt (src/core/propagator.py:723-793,
 * :1159-1198) and the Jones-vector projection of its result
 * (src/shared/propagation.py:4-90, propagator.py:316-327, :1210-1218).
 * _f32: FP32 state with compensated (Neumaier) position and velocity sums,
 * FP32 float4 grid, FP64 phase accumulator, Kahan FP32 optical depth.
 * _f64: the same kernel with every quantity in FP64 and a double grid.
 * grid: the trace layout (sloth_grid_pack_trace_f32 / _f64).
 * rays: (6, N) row-major, float (f32) or double (f64).
 * workspace: device scratch of at least sloth_trace_workspace_bytes(N) bytes,
 * 256-byte aligned; its contents need not be initialised. */
size_t sloth_trace_workspace_bytes(int64_t n_rays);
int sloth_trace_f32(const SlothGridDesc* g, const void* grid, const SlothTraceParams* p,
                    const float* rays, int64_t n, const SlothTraceOutputs* out,
                    void* workspace, size_t workspace_bytes, void* stream);
int sloth_trace_f64(const SlothGridDesc* g, const void* grid, const SlothTraceParams* p,
                    const double* rays, int64_t n, const SlothTraceOutputs* out,
                    void* workspace, size_t workspace_bytes, void* stream);

/* ---- request server -------------------------------------------------------
 * No counterpart in the reference (SLOTH traces one batch per call). Serves a
 * stream of trace jobs of different grids and ray counts by continuous
 * batching: one device arena of budget_bytes (allocated at create) holds the
 * packed grids -- an LRU cache keyed by the caller's 64-bit grid key -- and
 * each admitted job's rays, sort workspace and outputs. Jobs are admitted in
 * submission order as memory and job-table slots free up. Every
 * sloth_server_step() retires finished work, admits waiting jobs, and
 * launches one iteration -- a captured CUDA graph running the FP32 tracer's
 * persistent kernels over tiles handed out round-robin to all admitted jobs
 * (quantum tiles per job per round, at most tiles_per_step tiles) -- with up
 * to two iterations in flight. Results of a job do not depend on the other
 * jobs in its iterations. Lifecycle of a job:
 *   PENDING -> RUNNING (admitted) -> DONE -> fetch -> FETCHING -> FETCHED
 * (memory released), or a negative SLOTH_ERR_* state if admission failed,
 * or CANCELLED (sloth_server_cancel) from PENDING, RUNNING or DONE.
 * The caller keeps `ne` (needed until the job is admitted, and only if the
 * grid key is not resident) and `rays` valid until the job leaves PENDING.
 * A handle may be used from several host threads (calls are serialised). */
typedef struct SlothServer SlothServer;

typedef struct SlothServerConfig {
    size_t  budget_bytes;    /* device arena for grids and jobs (>= 16 MiB)      */
    int32_t max_jobs;        /* jobs admitted at the same time (table slots)     */
    int32_t tiles_per_step;  /* 1024-ray tiles per iteration                     */
    int32_t quantum;         /* tiles per job per round-robin round              */
    int32_t reserved;        /* must be 0                                        */
} SlothServerConfig;

typedef struct SlothServerStats {
    size_t    budget_bytes, arena_used;
    long long grids_resident, grid_packs, grid_evictions;
    long long jobs_submitted, jobs_admitted, jobs_done, jobs_failed;
    long long iterations, tiles, kernel_launches;
    double    gpu_busy_ms;   /* time some iteration was running on the GPU (union)  */
    double    gpu_span_ms;   /* first iteration start to last finished iteration end */
    long long jobs_cancelled;
    long long cancelled_pending_free;   /* cancelled jobs whose memory waits for in-flight iterations */
} SlothServerStats;

#define SLOTH_JOB_PENDING  0
#define SLOTH_JOB_RUNNING  1
#define SLOTH_JOB_DONE     2
#define SLOTH_JOB_FETCHING 3
#define SLOTH_JOB_FETCHED  4
#define SLOTH_JOB_CANCELLED 5

int sloth_server_create(const SlothServerConfig* cfg, SlothServer** out);
int sloth_server_destroy(SlothServer* s);
/* Queues a job. ne (device, float32 or float64 per ne_is_f64, m^-3) is packed
 * when the job is admitted unless grid_key is resident (then ne may be NULL).
 * rays: (6, n) float32, host memory (pinned) if rays_on_host, else device.
 * p as for sloth_trace_f32 (its q_max selects the fast exact paths).
 * SLOTH_ERR_TOO_LARGE if the job can never fit in the arena. */
int sloth_server_submit(SlothServer* s, uint64_t grid_key, const SlothGridDesc* g, const void* ne,
                        int ne_is_f64, const SlothTraceParams* p, const float* rays, int rays_on_host,
                        int64_t n, int* job_id);
/* One scheduling step; never blocks on the GPU. */
int sloth_server_step(SlothServer* s, int* n_running, int* n_pending);
int sloth_server_job_state(SlothServer* s, int job_id, int* state);
/* Starts the download of a DONE job's outputs into dst (host or device
 * pointers; NULL skips; element types as for sloth_trace_f32, no state);
 * the job's memory is released once the copy has finished (FETCHED). */
int sloth_server_fetch(SlothServer* s, int job_id, const SlothTraceOutputs* dst);
/* Forgets a DONE, FETCHED or CANCELLED job (a DONE job's memory is released
 * unread). */
int sloth_server_release(SlothServer* s, int job_id);
/* Cancels a job; never blocks on the GPU. A PENDING job leaves the queue; a
 * RUNNING job gets no further tiles, and its memory and table slot are
 * released once the iterations already holding its tiles have finished on
 * the GPU (stats.cancelled_pending_free counts such jobs); a DONE job's
 * memory is released unread. The job's state becomes CANCELLED at once.
 * CANCELLED, FETCHED and failed jobs are left as they are (SLOTH_OK);
 * a FETCHING job returns SLOTH_ERR_BUSY. No counterpart in the reference. */
int sloth_server_cancel(SlothServer* s, int job_id);
/* Fault injection for tests of the create path: the next
 * sloth_server_create reports the `nth` (1-based) of its device or pinned
 * host allocations as failed (cudaErrorMemoryAllocation) without making it,
 * releases what it had allocated and returns SLOTH_ERR_OUT_OF_MEMORY.
 * One-shot; 0 disarms. Returns the number of allocations create makes. */
int sloth_server_inject_alloc_failure(int nth);
int sloth_server_stats(SlothServer* s, SlothServerStats* st);
/* Waits for all work the server has launched. */
int sloth_server_sync(SlothServer* s);

/* ---- allocation-free FP32 tracer ------------------------------------------
 * No counterpart in the reference. Some callers cannot allocate device
 * memory: an XLA FFI handler inside a JAX program (the reference's own
 * runtime) is handed only its operand and result buffers, and XLA has
 * already reserved most of the GPU for itself; an embedded or real-time host
 * may forbid device allocation after start-up. sloth_trace_f32 needs a caller
 * workspace; this variant takes the same inputs and outputs and keeps its
 * scratch in a fixed device array inside the library instead, so it
 * allocates nothing (no cudaMalloc, no cudaFree, no allocating library call).
 * Limits and rules:
 *   - n <= SLOTH_NOALLOC_MAX_RAYS, else SLOTH_ERR_TOO_LARGE;
 *   - the array (about 13.6 MB) is held on every GPU that loads the library
 *     until the process exits;
 *   - every call looks up the array's device address on the current device
 *     with cudaGetSymbolAddress, so the address stays right after
 *     cudaDeviceReset; the first call on each device also loads the
 *     library's device code there: make that first call before any stream
 *     capture;
 *   - every call shares the array, so calls that overlap on the GPU (other
 *     streams, other host threads) race: serialise them.
 * Results equal sloth_trace_f32's for the same inputs. */
#define SLOTH_NOALLOC_MAX_RAYS (1 << 20)
int sloth_trace_f32_noalloc(const SlothGridDesc* g, const void* grid, const SlothTraceParams* p,
                            const float* rays, int64_t n, const SlothTraceOutputs* out, void* stream);

/* ---- K4/K5: detector image and its adjoint --------------------------------
 * No counterpart in the reference, which never differentiates. The forward
 * model maps the packed grid to a detector image:
 *   - fixed-step Runge-Kutta-Nystrom steps of the reference's ray equations (src/core/propagator.py
 *     168-243: dv/dt = -(c^2/2) grad(ne/nc), trilinear gradient, fill 0
 *     outside), at most n_steps steps of dtau, in the tracers' scaled scheme
 *     but without face clipping. A ray stops early once it is outside the
 *     grid on some axis and moving away from it along that axis.
 *   - projection of the final ray on a straight line to the plane
 *     `plane` along probing_axis (src/shared/propagation.py:92-134).
 *   - a Gaussian splat into an n_px[0] x n_px[1] image covering
 *     window = {u0, u1, v0, v1} (metres) on the two transverse axes in
 *     ascending order (probing z: u = x, v = y; image[i][j], i along u).
 *     A ray at pixel coordinates (a, b) (pixel i covers
 *     [u0 + i du, u0 + (i+1) du)) adds g(i - a) g(j - b) / (2 pi s^2), with
 *     g(d) = exp(-d^2 / 2s^2) times a taper that is 1 up to 3s and falls to 0
 *     at 4s as a C2 smoothstep; s = sigma_px.
 * The forward keeps each ray's state every ckpt_every steps in the workspace.
 * The backward needs that workspace unchanged, and the same grid, params and n:
 *   - it adds d L / d(packed grid) for the given d L / d image to grid_grad
 *     (same layout as the packed grid; the entry point zeroes it first;
 *     channel q stays 0);
 *   - it recomputes each checkpoint segment and runs the discrete adjoint of
 *     the steps in reverse.
 * sloth_grid_pack_adjoint_* maps d L / d(packed grid) to d L / d ne through
 * the transpose of sloth_grid_pack_*: ne_grad = ne_scale * (dq + sum over
 * axes of the transposed difference stencil of the gradient channels).
 * _f32: FP32 grid, rays, image and compensated FP32 state (as sloth_trace_f32);
 * grid_grad accumulates with FP32 atomics. _f64: all FP64. */
typedef struct SlothImageParams {
    double  dtau;            /* step c*dt (m)                                      */
    int32_t n_steps;         /* steps per ray, at most                             */
    int32_t ckpt_every;      /* steps per checkpoint segment, 1 .. 32              */
    int32_t probing_axis;    /* detector plane normal: 0, 1 or 2                   */
    int32_t n_px[2];         /* image size (pixels) along the two transverse axes  */
    int32_t reserved;        /* must be 0                                          */
    double  plane;           /* detector plane position along probing_axis (m)     */
    double  window[4];       /* u0, u1, v0, v1: detector extent (m)                */
    double  sigma_px;        /* splat Gaussian sigma (pixels), 0 < sigma <= 8       */
} SlothImageParams;

size_t sloth_image_workspace_bytes(const SlothImageParams* p, int64_t n_rays);
/* total_steps: device counter the forward adds every ray's step count to
 * (the caller zeroes it; NULL skips). */
int sloth_image_forward_f32(const SlothGridDesc* g, const void* grid, const SlothImageParams* p,
                            const float* rays, int64_t n, float* image, unsigned long long* total_steps,
                            void* workspace, size_t workspace_bytes, void* stream);
int sloth_image_forward_f64(const SlothGridDesc* g, const void* grid, const SlothImageParams* p,
                            const double* rays, int64_t n, double* image, unsigned long long* total_steps,
                            void* workspace, size_t workspace_bytes, void* stream);
int sloth_image_backward_f32(const SlothGridDesc* g, const void* grid, const SlothImageParams* p,
                             int64_t n, const float* image_grad, void* grid_grad, void* workspace,
                             size_t workspace_bytes, void* stream);
int sloth_image_backward_f64(const SlothGridDesc* g, const void* grid, const SlothImageParams* p,
                             int64_t n, const double* image_grad, void* grid_grad, void* workspace,
                             size_t workspace_bytes, void* stream);
int sloth_grid_pack_adjoint_f32(const SlothGridDesc* g, const void* grid_grad, double ne_scale,
                                float* ne_grad, void* stream);
int sloth_grid_pack_adjoint_f64(const SlothGridDesc* g, const void* grid_grad, double ne_scale,
                                double* ne_grad, void* stream);

/* ---- K6: ray-transfer-matrix diagnostics ----------------------------------
 * Replaces the optics and histogram of src/processing/diagnostics.py
 * (lens, travel, the apertures and stops, knife_edge, the lens_cutoff
 * prefilter, Diagnostic.histogram; :16-128, :176-268) on Jones vectors
 * (4, N) = (x, theta, y, phi), e.g. a trace's last save. Per ray:
 *   1. if prefilter: keep only rays with sqrt((L tan theta + x)^2 +
 *      (L tan phi + y)^2) <= R, on the input as given;
 *   2. rows 0 and 2 times pos_scale (1e3 for the reference's m -> mm),
 *      rounded in the input's precision;
 *   3. the optics in order, in FP64 (see SLOTH_OPTIC_*). Travel and lens
 *      are 4x4 matrix products in the reference, so a NaN in any component
 *      makes all four NaN. The stops set all four to NaN;
 *   4. if ccd_clip: keep |x| <= ccd_half[0] and |y| <= ccd_half[1];
 *   5. if hist != NULL: add the ray's weight (1 if weights is NULL) to
 *      hist[iy][ix] (ny x nx, doubles; the entry point adds, the caller
 *      zeroes). The bins are numpy.histogram2d's over x_range x y_range:
 *      numpy's linspace edges, the upper edge in the last bin, NaN and
 *      out-of-range values dropped. The reference's H is this transposed
 *      layout.
 * rays_out (4, N) doubles (optional) receives the rays after step 3, with
 * NaN for rejected rays. kept (N bytes, optional) receives 1 for rays the
 * prefilter keeps. */
#define SLOTH_OPTIC_TRAVEL             1  /* a = distance: x += a*theta, y += a*phi          */
#define SLOTH_OPTIC_LENS               2  /* a = f1, b = f2: theta -= x/f1, phi -= y/f2      */
#define SLOTH_OPTIC_CIRCULAR_APERTURE  3  /* a = R: rejects x^2 + y^2 > R^2                  */
#define SLOTH_OPTIC_CIRCULAR_STOP      4  /* a = R: rejects x^2 + y^2 < R^2                  */
#define SLOTH_OPTIC_RECT_APERTURE      5  /* a = Lx, b = Ly: rejects x^2 > Lx^2 AND y^2 > Ly^2
                                             (the reference's rect_aperture, as written)     */
#define SLOTH_OPTIC_KNIFE_EDGE         6  /* axis = 0 (x) or 2 (y), a = offset, b = direction:
                                             rejects v > a if b > 0, v < a if b < 0          */
#define SLOTH_OPTIC_ANNULAR_STOP       7  /* a = R1, b = R2: rejects R1^2 < r^2 < R2^2        */
#define SLOTH_MAX_OPTICS 32

typedef struct SlothOptic {
    int32_t kind;            /* SLOTH_OPTIC_*                                      */
    int32_t axis;            /* knife edge only                                    */
    double  a, b;
} SlothOptic;

typedef struct SlothDetectorParams {
    int32_t nx, ny;          /* histogram bins along x (row 0) and y (row 2)        */
    double  x_range[2];      /* histogram range along x                            */
    double  y_range[2];
    double  pos_scale;       /* factor on rows 0 and 2 before the optics           */
    int32_t prefilter;       /* 1: lens_cutoff prefilter with prefilter_L, _R      */
    int32_t ccd_clip;        /* 1: clip to |x| <= ccd_half[0], |y| <= ccd_half[1]  */
    double  prefilter_L, prefilter_R;
    double  ccd_half[2];
    int32_t reserved;        /* must be 0                                          */
    int32_t reserved2;
} SlothDetectorParams;

int sloth_optics_f32(const float* rays, int64_t n, const float* weights, const SlothOptic* optics,
                     int32_t n_optics, const SlothDetectorParams* d, double* hist, double* rays_out,
                     uint8_t* kept, void* stream);
int sloth_optics_f64(const double* rays, int64_t n, const double* weights, const SlothOptic* optics,
                     int32_t n_optics, const SlothDetectorParams* d, double* hist, double* rays_out,
                     uint8_t* kept, void* stream);

/* ---- K7: probing beam on the device --------------------------------------
 * The rays of the reference's Beam (src/core/beam.py:57-346), (6, n)
 * row-major as Beam.s0: start plane probing_axis = ne_extent, speed c,
 * polar angle divergence * N(0,1) from the probing axis, azimuth pi * U, and
 * positions per beam_type (circular: radius size[0] * sqrt(U); square:
 * size[0] * (2U - 1) on both axes; rectangular: size[0], size[1]; linear:
 * size[0] * (2U - 1) on axis 0, velocity in the axis-0 / axis-2 plane).
 * The random numbers are not numpy's RandomState stream: draw k of ray id is
 * a hash of (seed, id, k). The rays [first_id, first_id + n) of one seed
 * are the same whichever calls generate them. */
#define SLOTH_BEAM_CIRCULAR     0
#define SLOTH_BEAM_SQUARE       1
#define SLOTH_BEAM_RECTANGULAR  2   /* also rect_trackers */
#define SLOTH_BEAM_LINEAR       3

typedef struct SlothBeamParams {
    int32_t  beam_type;      /* SLOTH_BEAM_*                                       */
    int32_t  probing_axis;   /* 0, 1, 2                                            */
    double   size[2];        /* beam_size (m); size[1] for rectangular only        */
    double   divergence;     /* rad                                                */
    double   ne_extent;      /* start plane coordinate along probing_axis (m)      */
    uint64_t seed;
    uint64_t first_id;       /* id of the first ray generated by this call         */
    int32_t  reserved;       /* must be 0                                          */
    int32_t  reserved2;
} SlothBeamParams;

int sloth_beam_f32(const SlothBeamParams* p, int64_t n, float* s0, void* stream);
int sloth_beam_f64(const SlothBeamParams* p, int64_t n, double* s0, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* SLOTH_B200_H */
