// Device code shared by the tracer entry points (trace.cu) and the request
// server (server.cu): kernel arguments, samplers, the integration step, per-ray
// bookkeeping, the per-tile tracing loop and the Morton pre-pass.
//
// What the reference does (src/core/propagator.py):
//   dsdt (:168-243): ds/dt = (v, grad(G)(r) [, kappa(r)]), G = -c^2/2 * ne/nc,
//                    grad(G) from precomputed grids through the trilinear
//                    interpolator (fill 0 outside the grid);
//   solve / trace_and_save_depths (:723-793, :1159-1198): vmap of a diffrax
//                    solve from t = 0 to the save times; output through
//                    ray_to_Jonesvector (src/shared/propagation.py:4-90).
// What runs here: the same ODE with a fixed-step fourth-order Runge-Kutta-
// Nystrom method in scaled units (grid cells, cells per step; see rkn_step),
// one thread per ray, plus the optical phase integral of omega*(n - 1) with
// n - 1 interpolated from the trace layout's channel 0, as the legacy solver
// interpolates its n grid (src/legacy/full_solver.py:289, :341-347), and the
// inverse-bremsstrahlung optical depth, both as Simpson quadratures of the
// stage values, and the Jones-vector projection at each save.
//
// Grid faces: the RHS jumps to the outside fill there. A step whose
// straight-line prediction p + w crosses a face is cut to end on it (a step
// of a fraction phi) and the ray then leaves on a straight line; a
// step whose prediction ends within kFaceMargin cells of a face, or is cut,
// samples its stage points clamped into the grid, i.e. it integrates the
// field's limit from inside, so that no stage sits on the discontinuity.
//
// Launch structure (all on the caller's stream):
//   1. keys_kernel   : Morton key of each ray's entry cell + bucket histogram
//   2. scan_kernel   : exclusive scan of the bucket counts (one CTA)
//   3. scatter_kernel: rays into bucket order
//   4. trace_kernel  : persistent CTAs; each takes a tile of 1024 rays in
//                      bucket order, sorts it by full key in shared memory,
//                      and its warps trace the tile; lanes whose ray has
//                      finished are refilled from the tile with one warp
//                      ballot + one shared-memory atomic per refill.
#pragma once

#include <cmath>
#include <type_traits>

#include "common.cuh"

#ifndef SLOTH_TRACE_THREADS
#define SLOTH_TRACE_THREADS 256
#endif
#ifndef SLOTH_TRACE_MIN_BLOCKS
#define SLOTH_TRACE_MIN_BLOCKS 2
#endif
#ifndef SLOTH_PAIRED_F32
#define SLOTH_PAIRED_F32 1
#endif
#ifndef SLOTH_PAIRED_STEP
#define SLOTH_PAIRED_STEP 1
#endif

namespace sloth {

constexpr int kThreads = SLOTH_TRACE_THREADS;
constexpr double kFaceMargin = 0.02;     // cells

// Inverse-bremsstrahlung modes of the tracer.
enum { IB_OFF = 0, IB_SUBCRITICAL = 1, IB_GENERAL = 2 };

// Integration methods (SlothTraceParams::integrator): Nystrom's fourth-order
// Runge-Kutta-Nystrom step (3 field samples) or the classical RK4 step of
// the first-order system (4 samples).
enum { INTEG_RKN = SLOTH_INTEGRATOR_RKN, INTEG_RK4 = SLOTH_INTEGRATOR_RK4 };

// How a step samples its stage points: PLAIN tests each point against the
// grid (fill 0 outside); CLAMP moves it into the grid first (steps at a
// face); INTERIOR skips the test, for steps whose stage points are known to
// lie inside (see interior_bound_ok). Every mode clamps the cell index into
// the grid, so no mode can read outside the grid.
enum { SAMPLE_PLAIN = 0, SAMPLE_CLAMP = 1, SAMPLE_INTERIOR = 2 };

// Largest |acceleration| (cells per step^2) for which an interior step
// (ray inside, prediction p + w at least kFaceMargin inside on every axis)
// has every stage point inside: the stages sit at p + w/2 + A1/8 and
// p + w + A2/2, at least kFaceMargin/2 and kFaceMargin from the faces before
// the A terms, so |A| <= min(8 * kFaceMargin/2, 2 * kFaceMargin) = 0.04
// suffices; 0.03 keeps headroom for rounding.
constexpr double kInteriorAccel = 0.03;

// ---------------------------------------------------------------------------
// Kernel arguments.
// ---------------------------------------------------------------------------
struct TraceArgs {
    GridGeo geo;
    const void* grid;
    const void* rays;          // (6, N) of R
    long long n;
    const unsigned* perm;      // bucket-ordered ray ids
    const unsigned* skeys;     // their keys
    int* tile_counter;
    int n_tiles;      // n_big tiles of kTile rays, then tiles of kSmallTile rays
    int n_big;
    double origin[3], spacing[3];
    double w_of_v[3];          // w = v * w_of_v   (cells per step per m/s)
    double v_of_w[3];          // v = w * v_of_w
    double S[3];               // -(dtau/h)^2 / 2
    float Sf[3];               // the same, rounded to FP32 once here (the FP32 tracer reads these
                               // instead of converting the doubles inside its loop)
    float S4f[3], S2f[3], S6f[3];   // Sf/4, Sf/2 and fl(1/6)*Sf in FP32: the paired RKN step's
                                    // unit-step coefficients with S folded in
    float ope2f, cl_lof, cl_wf;
    float inv_ope2f;           // 1 / ope2 (q from x = ope2 * q)
    float accel_bound;         // bound on |acceleration| (cells per step^2), 0 when unknown
                               // (see interior_run and interior_sampling_ok)
    double phase_scale;        // (omega/c) * dtau / 6
    double tau_scale;          // kappa_q2 * dtau / 6
    double cl_w, cl_lo;        // Coulomb log below nc, and max(2, cl_w)
    double ope2;               // (omega_pe/omega)^2 per unit q
    double inv_ope2;
    double plane;
    int first_save, save_every, n_saves;
    int axis, t1, t2;
    int project;
    void* jones;
    void* state;
    double* phase;
    void* amp;
    uint8_t* status;
    int32_t* steps;
    unsigned long long* total_steps;
};

// Scalar parameters in the tracer's precision (FP32 copies made on the host).
template <class R> __device__ __forceinline__ R arg_S(const TraceArgs& a, int k);
template <> __device__ __forceinline__ float arg_S<float>(const TraceArgs& a, int k) { return a.Sf[k]; }
template <> __device__ __forceinline__ double arg_S<double>(const TraceArgs& a, int k) { return a.S[k]; }
template <class R> __device__ __forceinline__ R arg_ope2(const TraceArgs& a) {
    if constexpr (sizeof(R) == 4) return a.ope2f; else return a.ope2;
}
template <class R> __device__ __forceinline__ R arg_cl_lo(const TraceArgs& a) {
    if constexpr (sizeof(R) == 4) return a.cl_lof; else return a.cl_lo;
}
template <class R> __device__ __forceinline__ R arg_cl_w(const TraceArgs& a) {
    if constexpr (sizeof(R) == 4) return a.cl_wf; else return a.cl_w;
}
template <class R> __device__ __forceinline__ R arg_inv_ope2(const TraceArgs& a) {
    if constexpr (sizeof(R) == 4) return a.inv_ope2f; else return a.inv_ope2;
}

__device__ __forceinline__ double sel3(const double (&v)[3], int i) {
    return i == 0 ? v[0] : (i == 1 ? v[1] : v[2]);
}

template <class P>
struct Ray {
    typename P::Acc p[3];      // position (cells)
    typename P::Acc w[3];      // velocity (cells per step)
    typename P::Acc tau;       // sum of kappa stage combinations
    double ph;                 // sum of (n-1) stage combinations
    double lag;                // steps between the ray's time and `step` after an exit step
    int step, save_j, next_save;
    int run;                   // steps ahead that are certainly interior steps (fast path)
    unsigned id;
    bool exited;               // left the grid through a face-clipped step
};

template <class P>
struct CellCache {
    unsigned base;
    typename P::V c[8];
};

// One field sample: n - 1 (the trace layout's channel 0), the three gradient
// channels and the inverse-bremsstrahlung rate per kappa_q2.
template <class P>
struct Sample {
    typename P::R n1, g0, g1, g2, k;
};

// A cached cell as trilinear polynomials in the in-cell coordinates
// (fx, fy, fz): per channel T = a + bx fx + by fy + bz fz + cxy fx fy +
// cxz fx fz + cyz fy fz + cxyz fx fy fz, channels q, dq/du, dq/dv, dq/dw and
// (when NK = 5) the inverse-bremsstrahlung corner rate.
template <class P, int NK>
struct CellPoly {
    unsigned base;
    typename P::R t[NK][8];
};

template <class R>
__device__ __forceinline__ void poly_coeffs(R (&t)[8], R v0, R v1, R v2, R v3, R v4, R v5, R v6, R v7) {
    // corner index = 4*dx + 2*dy + dz
    const R bz = v1 - v0, by = v2 - v0, bx = v4 - v0;
    const R dyz = v3 - v2, dxz = v5 - v4, dxy = v6 - v4;
    t[0] = v0;
    t[1] = bx;
    t[2] = by;
    t[3] = bz;
    t[4] = dxy - by;                       // cxy
    t[5] = dxz - bz;                       // cxz
    t[6] = dyz - bz;                       // cyz
    t[7] = ((v7 - v6) - dxz) - (dyz - bz); // cxyz
}

__device__ __forceinline__ float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }

template <class R>
__device__ __forceinline__ R poly_eval(const R (&t)[8], R fx, R fy, R fz) {
    // explicit fused multiply-adds: every kernel that inlines this rounds alike
    const R cz = fma_rn(fy, fma_rn(fx, t[7], t[6]), fma_rn(fx, t[5], t[3]));   // coefficient of fz
    const R cy = fma_rn(fx, t[4], t[2]);                                         // of fy (without fz)
    return fma_rn(fz, cz, fma_rn(fy, cy, fma_rn(fx, t[1], t[0])));
}

// FP32 cell cache on paired instructions. The packed voxel is a float4
// (q, dq/du, dq/dv, dq/dw), so (q, dq/du) and (dq/dv, dq/dw) arrive in
// register pairs; each pair of trilinear polynomials is built and evaluated
// with sm_100's two-wide FP32 instructions (__fadd2/__ffma2: one instruction
// for two channels, each component rounded exactly as the scalar operation).
// The inverse-bremsstrahlung channel (NK = 5) stays scalar.
template <int NK>
struct CellPolyF2 {
    unsigned base;
    float2 t[2][8];
};

// The FP32 paired cache keeps the cell's kappa polynomial (NK == 5) in shared
// memory rather than registers: each thread owns one slot, [2][threads]
// float4 so that a warp's 16-byte loads do not conflict. This keeps 8 values
// out of the step's 128-register budget; the coefficients are written once
// per cell and read once per stage, off the step's critical path.
static __shared__ float4 s_kappa_coef[2][kThreads];

__device__ __forceinline__ void kappa_store(const float (&k)[8]) {
    s_kappa_coef[0][threadIdx.x] = make_float4(k[0], k[1], k[2], k[3]);
    s_kappa_coef[1][threadIdx.x] = make_float4(k[4], k[5], k[6], k[7]);
}

__device__ __forceinline__ float kappa_eval(float fx, float fy, float fz);

__device__ __forceinline__ float2 sub2(float2 a, float2 b) {
    return __ffma2_rn(b, make_float2(-1.0f, -1.0f), a);          // a - b, one rounding
}

__device__ __forceinline__ void poly_coeffs2(float2 (&t)[8], float2 v0, float2 v1, float2 v2, float2 v3, float2 v4,
                                             float2 v5, float2 v6, float2 v7) {
    const float2 bz = sub2(v1, v0), by = sub2(v2, v0), bx = sub2(v4, v0);
    const float2 dyz = sub2(v3, v2), dxz = sub2(v5, v4), dxy = sub2(v6, v4);
    t[0] = v0;
    t[1] = bx;
    t[2] = by;
    t[3] = bz;
    t[4] = sub2(dxy, by);
    t[5] = sub2(dxz, bz);
    t[6] = sub2(dyz, bz);
    t[7] = sub2(sub2(sub2(v7, v6), dxz), sub2(dyz, bz));
}

__device__ __forceinline__ float2 poly_eval2(const float2 (&t)[8], float2 fx, float2 fy, float2 fz) {
    const float2 cz = __ffma2_rn(fy, __ffma2_rn(fx, t[7], t[6]), __ffma2_rn(fx, t[5], t[3]));
    const float2 cy = __ffma2_rn(fx, t[4], t[2]);
    return __ffma2_rn(fz, cz, __ffma2_rn(fy, cy, __ffma2_rn(fx, t[1], t[0])));
}

template <class C> struct IsPairedCache : std::false_type {};
template <int NK> struct IsPairedCache<CellPolyF2<NK>> : std::true_type {};

// x = (omega_pe/omega)^2 of a grid point from its n - 1 (the trace layout):
// n - 1 = sqrt(1 - x) - 1 gives x = -(n - 1)(2 + (n - 1)) up to the critical
// density (n - 1 >= -1), and the layout stores -x above it.
template <class R>
__device__ __forceinline__ R x_of_n1(R n1) {
    if constexpr (sizeof(R) == 4)
        return n1 >= -1.0f ? -__fmul_rn(n1, __fadd_rn(2.0f, n1)) : -n1;
    else
        return n1 >= -1.0 ? -__dmul_rn(n1, __dadd_rn(2.0, n1)) : -n1;
}

// Inverse-bremsstrahlung rate of one grid point per kappa_q2: q^2 * CL(q),
// CL = max(2, cl_w - ln(max(omega_pe/omega, 1))) (src/core/propagator.py:155-162),
// with q rebuilt from the point's n - 1.
template <class P>
__device__ __forceinline__ typename P::R corner_kappa(const TraceArgs& a, typename P::R n1) {
    using R = typename P::R;
    const R x = x_of_n1<R>(n1);
    const R q = x * arg_inv_ope2<R>(a);
    const R cl = (x > R(1)) ? fmax(R(2), arg_cl_w<R>(a) - R(0.5) * P::log_(x)) : arg_cl_lo<R>(a);
    return q * q * cl;
}

// Below the critical density the rate is kappa_q2 * CL * q^2 with a constant
// CL, so the sub-critical corners carry x^2 = (ope2 * q)^2 and the optical
// depth's scale the constant factor cl_lo / ope2^2.
template <class R>
__device__ __forceinline__ R corner_x2(R n1) {
    const R x = x_of_n1<R>(n1);
    if constexpr (sizeof(R) == 4) return __fmul_rn(x, x); else return __dmul_rn(x, x);
}

// Loads cell b into the paired cache: its polynomial coefficients, two
// channels per instruction.
template <class P, int IB, int NK>
__device__ __forceinline__ void paired_fill(const TraceArgs& a, unsigned b, CellPolyF2<NK>& cc) {
    const GridGeo& g = a.geo;
    cc.base = b;
    const float4* gp = reinterpret_cast<const float4*>(a.grid);
    const float4 v0 = __ldg(gp + b), v1 = __ldg(gp + b + 1u);
    const float4 v2 = __ldg(gp + b + g.sy), v3 = __ldg(gp + b + g.sy + 1u);
    const float4 v4 = __ldg(gp + b + g.sx), v5 = __ldg(gp + b + g.sx + 1u);
    const float4 v6 = __ldg(gp + b + g.sx + g.sy), v7 = __ldg(gp + b + g.sx + g.sy + 1u);
#define SLOTH_LO(v) make_float2(v.x, v.y)
#define SLOTH_HI(v) make_float2(v.z, v.w)
    poly_coeffs2(cc.t[0], SLOTH_LO(v0), SLOTH_LO(v1), SLOTH_LO(v2), SLOTH_LO(v3), SLOTH_LO(v4), SLOTH_LO(v5),
                 SLOTH_LO(v6), SLOTH_LO(v7));
    poly_coeffs2(cc.t[1], SLOTH_HI(v0), SLOTH_HI(v1), SLOTH_HI(v2), SLOTH_HI(v3), SLOTH_HI(v4), SLOTH_HI(v5),
                 SLOTH_HI(v6), SLOTH_HI(v7));
#undef SLOTH_LO
#undef SLOTH_HI
    if constexpr (IB == IB_SUBCRITICAL) {
        float k[8];
        poly_coeffs<float>(k, corner_x2(v0.x), corner_x2(v1.x), corner_x2(v2.x), corner_x2(v3.x), corner_x2(v4.x),
                           corner_x2(v5.x), corner_x2(v6.x), corner_x2(v7.x));
        kappa_store(k);
    } else if constexpr (IB == IB_GENERAL) {
        float k[8];
        poly_coeffs<float>(k, corner_kappa<P>(a, v0.x), corner_kappa<P>(a, v1.x), corner_kappa<P>(a, v2.x),
                           corner_kappa<P>(a, v3.x), corner_kappa<P>(a, v4.x), corner_kappa<P>(a, v5.x),
                           corner_kappa<P>(a, v6.x), corner_kappa<P>(a, v7.x));
        kappa_store(k);
    }
}

__device__ __forceinline__ float kappa_eval(float fx, float fy, float fz) {
    const float4 a = s_kappa_coef[0][threadIdx.x], b = s_kappa_coef[1][threadIdx.x];
    const float k[8] = {a.x, a.y, a.z, a.w, b.x, b.y, b.z, b.w};
    return poly_eval<float>(k, fx, fy, fz);
}

// Trilinear sample of the packed grid (rules of src/core/interpolator.py:79-104:
// cell i = floor(p) clamped to [0, n-2], product weights, fill 0 outside)
// returning q, the three gradient channels and, when IB, the interpolated
// inverse-bremsstrahlung rate per kappa_q2. The reference interpolates a
// kappa grid computed at the grid points (src/core/propagator.py:239,
// :623-631); with uniform Te and Z that grid is q^2 * CL(q) per point, so its
// interpolant is the weighted sum of the corner values, formed here from the
// corners already loaded (CL is constant below the critical density).
//
// The point is hi + lo: hi is the ray's running position (large) and lo its
// compensation plus the stage offset (small). The cell index comes from the
// rounded sum; the weights from (hi - i) + lo, which resolves the position
// inside the cell to FP32 relative precision rather than FP32 precision of
// the absolute position. CLAMP moves the point into the grid first.
template <class P, int IB, int MODE, class Cache>
__device__ __forceinline__ void sample_c(const TraceArgs& a, const typename P::R (&hi)[3],
                                         const typename P::R (&lo)[3], Sample<P>& out, Cache& cc) {
    using R = typename P::R;
    using V = typename P::V;
    const GridGeo& g = a.geo;
    R h[3], l[3], p[3];
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        h[x] = hi[x];
        l[x] = lo[x];
        p[x] = h[x] + l[x];
        if constexpr (MODE == SAMPLE_CLAMP) {
            const R pc = fmin(fmax(p[x], R(0)), lim_of<R>(g, x));
            if (pc != p[x]) {
                h[x] = pc;
                l[x] = R(0);
                p[x] = pc;
            }
        }
    }
    int ix, iy, iz;
    if constexpr (MODE != SAMPLE_INTERIOR) {
        const bool in = (p[0] >= R(0)) & (p[0] <= lim_of<R>(g, 0)) & (p[1] >= R(0)) &
                        (p[1] <= lim_of<R>(g, 1)) & (p[2] >= R(0)) & (p[2] <= lim_of<R>(g, 2));
        if (!in) {
            out.n1 = out.g0 = out.g1 = out.g2 = out.k = R(0);
            return;
        }
        ix = min((int)p[0], g.n[0] - 2);
        iy = min((int)p[1], g.n[1] - 2);
        iz = min((int)p[2], g.n[2] - 2);
    } else {
        // one unsigned min clamps both ends (a negative index wraps to a large value)
        ix = (int)min((unsigned)(int)p[0], (unsigned)(g.n[0] - 2));
        iy = (int)min((unsigned)(int)p[1], (unsigned)(g.n[1] - 2));
        iz = (int)min((unsigned)(int)p[2], (unsigned)(g.n[2] - 2));
    }
    const R fx = (h[0] - (R)ix) + l[0], fy = (h[1] - (R)iy) + l[1], fz = (h[2] - (R)iz) + l[2];
    const unsigned b = (unsigned)ix * g.sx + (unsigned)iy * g.sy + (unsigned)iz;
    if constexpr (IsPairedCache<Cache>::value) {
        if (b != cc.base) paired_fill<P, IB>(a, b, cc);
        const float2 fx2 = make_float2(fx, fx), fy2 = make_float2(fy, fy), fz2 = make_float2(fz, fz);
        const float2 r0 = poly_eval2(cc.t[0], fx2, fy2, fz2);
        const float2 r1 = poly_eval2(cc.t[1], fx2, fy2, fz2);
        out.n1 = r0.x;
        out.g0 = r0.y;
        out.g1 = r1.x;
        out.g2 = r1.y;
        if constexpr (IB == IB_SUBCRITICAL) {
            out.k = kappa_eval(fx, fy, fz);   // cl_lo / ope2^2 is in tau_scale
        } else if constexpr (IB == IB_GENERAL) {
            out.k = kappa_eval(fx, fy, fz);
        } else {
            out.k = 0.0f;
        }
    } else if constexpr (P::cell_poly) {
        if (b != cc.base) {
            cc.base = b;
            const V v0 = P::load(a.grid, b), v1 = P::load(a.grid, b + 1u);
            const V v2 = P::load(a.grid, b + g.sy), v3 = P::load(a.grid, b + g.sy + 1u);
            const V v4 = P::load(a.grid, b + g.sx), v5 = P::load(a.grid, b + g.sx + 1u);
            const V v6 = P::load(a.grid, b + g.sx + g.sy), v7 = P::load(a.grid, b + g.sx + g.sy + 1u);
            poly_coeffs<R>(cc.t[0], v0.x, v1.x, v2.x, v3.x, v4.x, v5.x, v6.x, v7.x);
            poly_coeffs<R>(cc.t[1], v0.y, v1.y, v2.y, v3.y, v4.y, v5.y, v6.y, v7.y);
            poly_coeffs<R>(cc.t[2], v0.z, v1.z, v2.z, v3.z, v4.z, v5.z, v6.z, v7.z);
            poly_coeffs<R>(cc.t[3], v0.w, v1.w, v2.w, v3.w, v4.w, v5.w, v6.w, v7.w);
            if constexpr (IB == IB_SUBCRITICAL) {
                poly_coeffs<R>(cc.t[4 % (IB ? 5 : 4)], corner_x2(v0.x), corner_x2(v1.x), corner_x2(v2.x),
                               corner_x2(v3.x), corner_x2(v4.x), corner_x2(v5.x), corner_x2(v6.x), corner_x2(v7.x));
            } else if constexpr (IB == IB_GENERAL) {
                poly_coeffs<R>(cc.t[4 % (IB ? 5 : 4)], corner_kappa<P>(a, v0.x), corner_kappa<P>(a, v1.x),
                               corner_kappa<P>(a, v2.x), corner_kappa<P>(a, v3.x), corner_kappa<P>(a, v4.x),
                               corner_kappa<P>(a, v5.x), corner_kappa<P>(a, v6.x), corner_kappa<P>(a, v7.x));
            }
        }
        out.n1 = poly_eval<R>(cc.t[0], fx, fy, fz);
        out.g0 = poly_eval<R>(cc.t[1], fx, fy, fz);
        out.g1 = poly_eval<R>(cc.t[2], fx, fy, fz);
        out.g2 = poly_eval<R>(cc.t[3], fx, fy, fz);
        if constexpr (IB == IB_SUBCRITICAL) {
            out.k = poly_eval<R>(cc.t[4 % (IB ? 5 : 4)], fx, fy, fz);   // cl_lo / ope2^2 is in tau_scale
        } else if constexpr (IB == IB_GENERAL) {
            out.k = poly_eval<R>(cc.t[4 % (IB ? 5 : 4)], fx, fy, fz);
        } else {
            out.k = R(0);
        }
    } else {
        V c[8];
        if constexpr (P::cell_cache) {
            if (b != cc.base) {
                cc.base = b;
                cc.c[0] = P::load(a.grid, b);
                cc.c[1] = P::load(a.grid, b + 1u);
                cc.c[2] = P::load(a.grid, b + g.sy);
                cc.c[3] = P::load(a.grid, b + g.sy + 1u);
                cc.c[4] = P::load(a.grid, b + g.sx);
                cc.c[5] = P::load(a.grid, b + g.sx + 1u);
                cc.c[6] = P::load(a.grid, b + g.sx + g.sy);
                cc.c[7] = P::load(a.grid, b + g.sx + g.sy + 1u);
            }
    #pragma unroll
            for (int i = 0; i < 8; ++i) c[i] = cc.c[i];
        } else {
            c[0] = P::load(a.grid, b);
            c[1] = P::load(a.grid, b + 1u);
            c[2] = P::load(a.grid, b + g.sy);
            c[3] = P::load(a.grid, b + g.sy + 1u);
            c[4] = P::load(a.grid, b + g.sx);
            c[5] = P::load(a.grid, b + g.sx + 1u);
            c[6] = P::load(a.grid, b + g.sx + g.sy);
            c[7] = P::load(a.grid, b + g.sx + g.sy + 1u);
        }
        const R ex = R(1) - fx, ey = R(1) - fy, ez = R(1) - fz;
        const R w00 = ex * ey, w01 = ex * fy, w10 = fx * ey, w11 = fx * fy;
        const R w[8] = {w00 * ez, w00 * fz, w01 * ez, w01 * fz, w10 * ez, w10 * fz, w11 * ez, w11 * fz};
        R q = R(0), g0 = R(0), g1 = R(0), g2 = R(0);
    #pragma unroll
        for (int i = 0; i < 8; ++i) {
            q += c[i].x * w[i];
            g0 += c[i].y * w[i];
            g1 += c[i].z * w[i];
            g2 += c[i].w * w[i];
        }
        out.n1 = q;
        out.g0 = g0;
        out.g1 = g1;
        out.g2 = g2;
        if constexpr (IB == IB_SUBCRITICAL) {
            R k = R(0);
    #pragma unroll
            for (int i = 0; i < 8; ++i) k += w[i] * corner_x2(c[i].x);
            out.k = k;   // cl_lo / ope2^2 is in tau_scale
        } else if constexpr (IB == IB_GENERAL) {
            R k = R(0);
    #pragma unroll
            for (int i = 0; i < 8; ++i) k += w[i] * corner_kappa<P>(a, c[i].x);
            out.k = k;
        } else {
            out.k = R(0);
        }
    }
}

// One step of length phi (in steps; phi = 1 except for a step cut at a grid
// face) in scaled units; see the file header. The ray equation is second
// order with a position-only force, p'' = A(p), and the phase and optical
// depth integrate functions of the position only, so the step is Nystrom's
// fourth-order Runge-Kutta-Nystrom method, three samples of the field instead
// of RK4's four:
//   stage points p, p + phi*w/2 + phi^2 A1/8, p + phi*w + phi^2 A2/2,
//   p' = p + phi*w + phi^2 (A1 + 2 A2)/6,  w' = w + phi (A1 + 4 A2 + A3)/6,
// and the phase and depth take Simpson's weights (1, 4, 1)/6 on the stages.
// The position and velocity are fourth order; the two integrals are third
// order in the step (their middle stage point is second order), an error
// many orders below the FP32 rounding here. Stage sums are accumulated as the
// stages are produced to keep few values live.
// The phase integrand n - 1 is interpolated from the trace layout's channel 0
// (the legacy solver's interpolated n, src/legacy/full_solver.py:289, :342-345).
template <class P, int IB, int MODE, class Cache>
__device__ __forceinline__ void rkn_step(const TraceArgs& a, Ray<P>& r, Cache& cc, typename P::R phi) {
    using R = typename P::R;
    const R hphi = R(0.5) * phi, phi6 = phi * R(1.0 / 6.0), phi2_6 = phi * phi6;
    const R phi2_8 = R(0.125) * phi * phi, phi2_2 = R(0.5) * phi * phi;
    const R S0 = arg_S<R>(a, 0), S1 = arg_S<R>(a, 1), S2 = arg_S<R>(a, 2);
    R ph[3], pl[3], we[3], sA[3], sW[3], st[3];
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        ph[x] = r.p[x].hi();
        pl[x] = r.p[x].lo();
        we[x] = r.w[x].val();
    }
    Sample<P> s;
    // stage 1 at p
    sample_c<P, IB, MODE>(a, ph, pl, s, cc);
    R g = s.n1;
    R kq = s.k;
    {
        const R A[3] = {S0 * s.g0, S1 * s.g1, S2 * s.g2};
#pragma unroll
        for (int x = 0; x < 3; ++x) {
            sA[x] = A[x];
            sW[x] = A[x];
            st[x] = pl[x] + (hphi * we[x] + phi2_8 * A[x]);     // p + phi*w/2 + phi^2 A1/8
        }
    }
    // stage 2
    sample_c<P, IB, MODE>(a, ph, st, s, cc);
    {
        const R A[3] = {S0 * s.g0, S1 * s.g1, S2 * s.g2};
#pragma unroll
        for (int x = 0; x < 3; ++x) {
            sA[x] += R(2) * A[x];
            sW[x] += R(4) * A[x];
            st[x] = pl[x] + (phi * we[x] + phi2_2 * A[x]);      // p + phi*w + phi^2 A2/2
        }
    }
    g += R(4) * s.n1;
    kq += R(4) * s.k;
    // stage 3
    sample_c<P, IB, MODE>(a, ph, st, s, cc);
    sW[0] += S0 * s.g0; sW[1] += S1 * s.g1; sW[2] += S2 * s.g2;
    g += s.n1;
    kq += s.k;
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        const R dp = phi * r.w[x].hi() + (phi * r.w[x].lo() + phi2_6 * sA[x]);
        r.p[x].add(dp);
        r.w[x].add(phi6 * sW[x]);
    }
    r.ph += (double)(phi * g);
    if constexpr (IB != IB_OFF) r.tau.add(phi * kq);
}

// ---------------------------------------------------------------------------
// FP32 with the paired cell cache: the y and z components of every
// per-axis quantity of the step travel as one register pair and use sm_100's
// paired FP32 instructions (the cell polynomials already deliver dq/dv and
// dq/dw as a pair); x stays scalar. Each component is rounded exactly as the
// scalar step rounds it.
// ---------------------------------------------------------------------------
__device__ __forceinline__ float2 bc2(float v) { return make_float2(v, v); }

// sample at (hx + lx, hyz + lyz)
template <int IB, int MODE, int NK>
__device__ __forceinline__ void sample_f2(const TraceArgs& a, float hx, float lx, float2 hyz, float2 lyz,
                                          Sample<PolF32>& out, CellPolyF2<NK>& cc) {
    const GridGeo& g = a.geo;
    float px = hx + lx;
    float2 pyz = __fadd2_rn(hyz, lyz);
    if constexpr (MODE == SAMPLE_CLAMP) {
        const float cx = fminf(fmaxf(px, 0.0f), g.limf[0]);
        if (cx != px) { hx = cx; lx = 0.0f; px = cx; }
        const float cy = fminf(fmaxf(pyz.x, 0.0f), g.limf[1]);
        if (cy != pyz.x) { hyz.x = cy; lyz.x = 0.0f; pyz.x = cy; }
        const float cz = fminf(fmaxf(pyz.y, 0.0f), g.limf[2]);
        if (cz != pyz.y) { hyz.y = cz; lyz.y = 0.0f; pyz.y = cz; }
    }
    int ix, iy, iz;
    if constexpr (MODE != SAMPLE_INTERIOR) {
        const bool in = (px >= 0.0f) & (px <= g.limf[0]) & (pyz.x >= 0.0f) & (pyz.x <= g.limf[1]) &
                        (pyz.y >= 0.0f) & (pyz.y <= g.limf[2]);
        if (!in) {
            out.n1 = out.g0 = out.g1 = out.g2 = out.k = 0.0f;
            return;
        }
        ix = min((int)px, g.n[0] - 2);
        iy = min((int)pyz.x, g.n[1] - 2);
        iz = min((int)pyz.y, g.n[2] - 2);
    } else {
        ix = (int)min((unsigned)(int)px, (unsigned)(g.n[0] - 2));
        iy = (int)min((unsigned)(int)pyz.x, (unsigned)(g.n[1] - 2));
        iz = (int)min((unsigned)(int)pyz.y, (unsigned)(g.n[2] - 2));
    }
    const float fx = (hx - (float)ix) + lx;
    const float2 fyz = __fadd2_rn(__fadd2_rn(hyz, make_float2(-(float)iy, -(float)iz)), lyz);
    const unsigned b = (unsigned)ix * g.sx + (unsigned)iy * g.sy + (unsigned)iz;
    if (b != cc.base) paired_fill<PolF32, IB>(a, b, cc);
    const float2 fx2 = bc2(fx), fy2 = bc2(fyz.x), fz2 = bc2(fyz.y);
    const float2 r0 = poly_eval2(cc.t[0], fx2, fy2, fz2);
    const float2 r1 = poly_eval2(cc.t[1], fx2, fy2, fz2);
    out.n1 = r0.x;
    out.g0 = r0.y;
    out.g1 = r1.x;
    out.g2 = r1.y;
    if constexpr (IB == IB_SUBCRITICAL) {
        out.k = kappa_eval(fx, fyz.x, fyz.y);   // cl_lo / ope2^2 is in tau_scale
    } else if constexpr (IB == IB_GENERAL) {
        out.k = kappa_eval(fx, fyz.x, fyz.y);
    } else {
        out.k = 0.0f;
    }
}

// s + x with the compensation c (AccF::add on a pair)
__device__ __forceinline__ void kahan2(float2& s, float2& c, float2 x) {
    const float2 y = __fadd2_rn(x, c);
    const float2 t = __fadd2_rn(s, y);
    c = __fadd2_rn(y, __ffma2_rn(s, bc2(1.0f), make_float2(-t.x, -t.y)) );
    s = t;
}

// kahan2 of a * b, the product's rounding folded into the compensated add
__device__ __forceinline__ void kahan2_fma(float2& s, float2& c, float2 a, float2 b) {
    const float2 y = __ffma2_rn(a, b, c);
    const float2 t = __fadd2_rn(s, y);
    c = __fadd2_rn(y, __ffma2_rn(s, bc2(1.0f), make_float2(-t.x, -t.y)) );
    s = t;
}

// UNIT: phi is 1 (every step but a cut one); the multiplications by phi are
// left out, which gives bitwise the results of the general form at phi = 1
// (fma(1, a, b) rounds as a + b).
template <int IB, int MODE, bool UNIT, int NK>
__device__ __forceinline__ void rkn_step_f2(const TraceArgs& a, Ray<PolF32>& r, CellPolyF2<NK>& cc, float phi) {
    if constexpr (UNIT) phi = 1.0f;
    auto mphi = [&](float x) { return UNIT ? x : __fmul_rn(phi, x); };
    auto mphi2 = [&](float2 x) { return UNIT ? x : __fmul2_rn(bc2(phi), x); };
    const float hphi = 0.5f * phi, phi6 = phi * (1.0f / 6.0f), phi2_6 = phi * phi6;
    const float phi2_2 = 0.5f * phi * phi;
    // The accelerations enter the step only through the stage points and the
    // two weighted sums, so S multiplies the step's coefficients rather than
    // every stage's gradient: k4 = phi S/4 and k2 = phi^2 S/2 (stage points,
    // p + (phi/2)(w + k4 G1) and p + phi w + k2 G2), k6 = phi^2 S/6 (position),
    // kw = phi S/6 (velocity). Unit steps read them from the arguments, formed
    // there exactly as here at phi = 1.
    float k4x, k2x, k6x, kwx;
    float2 k4yz, k2yz, k6yz, kwyz;
    if constexpr (UNIT) {
        k4x = a.S4f[0];
        k2x = a.S2f[0];
        k6x = kwx = a.S6f[0];
        k4yz = make_float2(a.S4f[1], a.S4f[2]);
        k2yz = make_float2(a.S2f[1], a.S2f[2]);
        k6yz = kwyz = make_float2(a.S6f[1], a.S6f[2]);
    } else {
        const float S0 = a.Sf[0];
        const float2 S12 = make_float2(a.Sf[1], a.Sf[2]);
        k4x = __fmul_rn(0.25f * phi, S0);
        k2x = __fmul_rn(phi2_2, S0);
        k6x = __fmul_rn(phi2_6, S0);
        kwx = __fmul_rn(phi6, S0);
        k4yz = __fmul2_rn(bc2(0.25f * phi), S12);
        k2yz = __fmul2_rn(bc2(phi2_2), S12);
        k6yz = __fmul2_rn(bc2(phi2_6), S12);
        kwyz = __fmul2_rn(bc2(phi6), S12);
    }
    const float2 hphi2 = bc2(hphi), phi22 = bc2(phi);
    // Every rounding is explicit (intrinsics), so that each kernel that
    // inlines this step (the tracer's and the server's) rounds alike.
    const float phx = r.p[0].s, plx = r.p[0].c, wex = r.w[0].s + r.w[0].c;
    const float2 phyz = make_float2(r.p[1].s, r.p[2].s), plyz = make_float2(r.p[1].c, r.p[2].c);
    const float2 weyz = __fadd2_rn(make_float2(r.w[1].s, r.w[2].s), make_float2(r.w[1].c, r.w[2].c));
    Sample<PolF32> s;
    // stage 1 at p; gA = g1 + 2 g2 and gW = g1 + 4 g2 + g3 are the gradient
    // sums (S applied in the coefficients)
    sample_f2<IB, MODE>(a, phx, plx, phyz, plyz, s, cc);
    float g = s.n1;
    float kq = s.k;
    float gAx = s.g0;
    float2 gAyz = make_float2(s.g1, s.g2);
    float gWx = gAx;
    float2 gWyz = gAyz;
    // stage 2 at p + phi*w/2 + phi^2 A1/8 = p + (phi/2)(w + k4 G1)
    float stx = __fmaf_rn(hphi, __fmaf_rn(k4x, gAx, wex), plx);
    float2 styz = __ffma2_rn(hphi2, __ffma2_rn(k4yz, gAyz, weyz), plyz);
    sample_f2<IB, MODE>(a, phx, stx, phyz, styz, s, cc);
    {
        const float Gx = s.g0;
        const float2 Gyz = make_float2(s.g1, s.g2);
        gAx = __fmaf_rn(2.0f, Gx, gAx);
        gAyz = __ffma2_rn(bc2(2.0f), Gyz, gAyz);
        gWx = __fmaf_rn(4.0f, Gx, gWx);
        gWyz = __ffma2_rn(bc2(4.0f), Gyz, gWyz);
        // stage 3 at p + phi*w + phi^2 A2/2
        stx = __fadd_rn(plx, __fmaf_rn(k2x, Gx, mphi(wex)));
        styz = __fadd2_rn(plyz, __ffma2_rn(k2yz, Gyz, mphi2(weyz)));
    }
    g = __fmaf_rn(4.0f, s.n1, g);
    kq = __fmaf_rn(4.0f, s.k, kq);
    sample_f2<IB, MODE>(a, phx, stx, phyz, styz, s, cc);
    gWx = __fadd_rn(gWx, s.g0);
    gWyz = __fadd2_rn(gWyz, make_float2(s.g1, s.g2));
    g = __fadd_rn(g, s.n1);
    kq = __fadd_rn(kq, s.k);
    // x: the scalar update
    if constexpr (UNIT)
        r.p[0].add(__fadd_rn(r.w[0].hi(), __fmaf_rn(k6x, gAx, r.w[0].lo())));
    else
        r.p[0].add(__fmaf_rn(phi, r.w[0].hi(), __fmaf_rn(k6x, gAx, __fmul_rn(phi, r.w[0].lo()))));
    r.w[0].add_fma(kwx, gWx);
    // y, z: the same update on pairs
    {
        const float2 whi = make_float2(r.w[1].s, r.w[2].s), wlo = make_float2(r.w[1].c, r.w[2].c);
        const float2 dp = UNIT ? __fadd2_rn(whi, __ffma2_rn(k6yz, gAyz, wlo))
                               : __ffma2_rn(phi22, whi, __ffma2_rn(k6yz, gAyz, __fmul2_rn(phi22, wlo)));
        float2 ps = phyz, pc = plyz;
        kahan2(ps, pc, dp);
        r.p[1].s = ps.x; r.p[2].s = ps.y; r.p[1].c = pc.x; r.p[2].c = pc.y;
        float2 ws = whi, wc = wlo;
        kahan2_fma(ws, wc, kwyz, gWyz);
        r.w[1].s = ws.x; r.w[2].s = ws.y; r.w[1].c = wc.x; r.w[2].c = wc.y;
    }
    r.ph += (double)mphi(g);
    if constexpr (IB != IB_OFF) r.tau.add(mphi(kq));
}

// One classical RK4 step of the first-order system (p, w)' = (w, A(p)) of
// length phi, four samples of the field (the integrator the workload
// descriptions name; INTEG_RK4):
//   stage points p, p + phi*w/2, p + phi*w2/2, p + phi*w3
//   with w2 = w + phi*A1/2, w3 = w + phi*A2/2;
//   p' = p + phi*w + phi^2 (A1 + A2 + A3)/6,  w' = w + phi (A1 + 2A2 + 2A3 + A4)/6,
// and the phase and depth take RK4's weights (1, 2, 2, 1)/6 on the stages.
// The stage points lie within phi^2 |A|/4 and phi^2 |A|/2 of the segment
// from p to p + phi*w, as the RKN step's do, so the interior-sampling bound
// kInteriorAccel and the interior-run envelope hold for both methods.
template <class P, int IB, int MODE, class Cache>
__device__ __forceinline__ void rk4_step(const TraceArgs& a, Ray<P>& r, Cache& cc, typename P::R phi) {
    using R = typename P::R;
    const R two = R(2);
    const R hphi = R(0.5) * phi, phi6 = phi * R(1.0 / 6.0), phi2_6 = phi * phi6;
    const R S0 = arg_S<R>(a, 0), S1 = arg_S<R>(a, 1), S2 = arg_S<R>(a, 2);
    R ph[3], pl[3], we[3], sA[3], sW[3], w3[3], st[3];
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        ph[x] = r.p[x].hi();
        pl[x] = r.p[x].lo();
        we[x] = r.w[x].val();
    }
    Sample<P> s;
    // stage 1 at p
    sample_c<P, IB, MODE>(a, ph, pl, s, cc);
    R g = s.n1;
    R kq = s.k;
    sA[0] = S0 * s.g0; sA[1] = S1 * s.g1; sA[2] = S2 * s.g2;
    // stage 2 at p + phi*w/2
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        sW[x] = sA[x];
        st[x] = pl[x] + hphi * we[x];
    }
    sample_c<P, IB, MODE>(a, ph, st, s, cc);
#pragma unroll
    for (int x = 0; x < 3; ++x) st[x] = pl[x] + hphi * (we[x] + hphi * sA[x]);   // p + phi*w2/2
    {
        const R A[3] = {S0 * s.g0, S1 * s.g1, S2 * s.g2};
#pragma unroll
        for (int x = 0; x < 3; ++x) {
            w3[x] = we[x] + hphi * A[x];
            sA[x] += A[x];
            sW[x] += two * A[x];
        }
    }
    g += two * s.n1;
    kq += two * s.k;
    // stage 3 at p + phi*w2/2
    sample_c<P, IB, MODE>(a, ph, st, s, cc);
    {
        const R A[3] = {S0 * s.g0, S1 * s.g1, S2 * s.g2};
#pragma unroll
        for (int x = 0; x < 3; ++x) {
            sA[x] += A[x];
            sW[x] += two * A[x];
            st[x] = pl[x] + phi * w3[x];
        }
    }
    g += two * s.n1;
    kq += two * s.k;
    // stage 4 at p + phi*w3
    sample_c<P, IB, MODE>(a, ph, st, s, cc);
    sW[0] += S0 * s.g0; sW[1] += S1 * s.g1; sW[2] += S2 * s.g2;
    g += s.n1;
    kq += s.k;
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        const R dp = phi * r.w[x].hi() + (phi * r.w[x].lo() + phi2_6 * sA[x]);
        r.p[x].add(dp);
        r.w[x].add(phi6 * sW[x]);
    }
    r.ph += (double)(phi * g);
    if constexpr (IB != IB_OFF) r.tau.add(phi * kq);
}

// The RK4 step in the paired FP32 form (y and z components as register
// pairs), every rounding explicit.
template <int IB, int MODE, bool UNIT, int NK>
__device__ __forceinline__ void rk4_step_f2(const TraceArgs& a, Ray<PolF32>& r, CellPolyF2<NK>& cc, float phi) {
    if constexpr (UNIT) phi = 1.0f;
    auto mphi = [&](float x) { return UNIT ? x : __fmul_rn(phi, x); };
    auto mphi2 = [&](float2 x) { return UNIT ? x : __fmul2_rn(bc2(phi), x); };
    const float hphi = 0.5f * phi, phi6 = phi * (1.0f / 6.0f), phi2_6 = phi * phi6;
    const float S0 = a.Sf[0];
    const float2 S12 = make_float2(a.Sf[1], a.Sf[2]);
    const float2 hphi2 = bc2(hphi), two2 = bc2(2.0f);
    const float phx = r.p[0].s, plx = r.p[0].c, wex = __fadd_rn(r.w[0].s, r.w[0].c);
    const float2 phyz = make_float2(r.p[1].s, r.p[2].s), plyz = make_float2(r.p[1].c, r.p[2].c);
    const float2 weyz = __fadd2_rn(make_float2(r.w[1].s, r.w[2].s), make_float2(r.w[1].c, r.w[2].c));
    Sample<PolF32> s;
    // stage 1 at p
    sample_f2<IB, MODE>(a, phx, plx, phyz, plyz, s, cc);
    float g = s.n1;
    float kq = s.k;
    float sAx = __fmul_rn(S0, s.g0);
    float2 sAyz = __fmul2_rn(S12, make_float2(s.g1, s.g2));
    float sWx = sAx;
    float2 sWyz = sAyz;
    // stage 2 at p + phi*w/2
    float stx = __fmaf_rn(hphi, wex, plx);
    float2 styz = __ffma2_rn(hphi2, weyz, plyz);
    sample_f2<IB, MODE>(a, phx, stx, phyz, styz, s, cc);
    stx = __fmaf_rn(hphi, __fmaf_rn(hphi, sAx, wex), plx);                 // p + phi*w2/2
    styz = __ffma2_rn(hphi2, __ffma2_rn(hphi2, sAyz, weyz), plyz);
    float w3x;
    float2 w3yz;
    {
        const float Ax = __fmul_rn(S0, s.g0);
        const float2 Ayz = __fmul2_rn(S12, make_float2(s.g1, s.g2));
        w3x = __fmaf_rn(hphi, Ax, wex);
        w3yz = __ffma2_rn(hphi2, Ayz, weyz);
        sAx = __fadd_rn(sAx, Ax);
        sAyz = __fadd2_rn(sAyz, Ayz);
        sWx = __fmaf_rn(2.0f, Ax, sWx);
        sWyz = __ffma2_rn(two2, Ayz, sWyz);
    }
    g = __fmaf_rn(2.0f, s.n1, g);
    kq = __fmaf_rn(2.0f, s.k, kq);
    // stage 3 at p + phi*w2/2
    sample_f2<IB, MODE>(a, phx, stx, phyz, styz, s, cc);
    {
        const float Ax = __fmul_rn(S0, s.g0);
        const float2 Ayz = __fmul2_rn(S12, make_float2(s.g1, s.g2));
        sAx = __fadd_rn(sAx, Ax);
        sAyz = __fadd2_rn(sAyz, Ayz);
        sWx = __fmaf_rn(2.0f, Ax, sWx);
        sWyz = __ffma2_rn(two2, Ayz, sWyz);
        stx = __fadd_rn(plx, mphi(w3x));
        styz = __fadd2_rn(plyz, mphi2(w3yz));
    }
    g = __fmaf_rn(2.0f, s.n1, g);
    kq = __fmaf_rn(2.0f, s.k, kq);
    // stage 4 at p + phi*w3
    sample_f2<IB, MODE>(a, phx, stx, phyz, styz, s, cc);
    sWx = __fmaf_rn(S0, s.g0, sWx);
    sWyz = __ffma2_rn(S12, make_float2(s.g1, s.g2), sWyz);
    g = __fadd_rn(g, s.n1);
    kq = __fadd_rn(kq, s.k);
    // x: the scalar update
    if constexpr (UNIT)
        r.p[0].add(__fadd_rn(r.w[0].hi(), __fadd_rn(r.w[0].lo(), __fmul_rn(phi2_6, sAx))));
    else
        r.p[0].add(__fmaf_rn(phi, r.w[0].hi(), __fmaf_rn(phi, r.w[0].lo(), __fmul_rn(phi2_6, sAx))));
    r.w[0].add(__fmul_rn(phi6, sWx));
    // y, z: the same update on pairs
    {
        const float2 phi2 = bc2(phi);
        const float2 whi = make_float2(r.w[1].s, r.w[2].s), wlo = make_float2(r.w[1].c, r.w[2].c);
        const float2 dp = UNIT ? __fadd2_rn(whi, __fadd2_rn(wlo, __fmul2_rn(bc2(phi2_6), sAyz)))
                               : __ffma2_rn(phi2, whi, __ffma2_rn(phi2, wlo, __fmul2_rn(bc2(phi2_6), sAyz)));
        float2 ps = phyz, pc = plyz;
        kahan2(ps, pc, dp);
        r.p[1].s = ps.x; r.p[2].s = ps.y; r.p[1].c = pc.x; r.p[2].c = pc.y;
        float2 ws = whi, wc = wlo;
        kahan2(ws, wc, __fmul2_rn(bc2(phi6), sWyz));
        r.w[1].s = ws.x; r.w[2].s = ws.y; r.w[1].c = wc.x; r.w[2].c = wc.y;
    }
    r.ph += (double)mphi(g);
    if constexpr (IB != IB_OFF) r.tau.add(mphi(kq));
}

// One step: the paired FP32 form with the paired cell cache, the generic form
// otherwise; RKN unless INTEG selects RK4.
template <class P, int IB, int MODE, bool UNIT = false, int INTEG = INTEG_RKN, class Cache>
__device__ __forceinline__ void step_any(const TraceArgs& a, Ray<P>& r, Cache& cc, typename P::R phi) {
    if constexpr (INTEG == INTEG_RK4) {
        if constexpr (IsPairedCache<Cache>::value && SLOTH_PAIRED_STEP) {
            rk4_step_f2<IB, MODE, UNIT>(a, r, cc, phi);
        } else {
            rk4_step<P, IB, MODE>(a, r, cc, phi);
        }
    } else if constexpr (IsPairedCache<Cache>::value && SLOTH_PAIRED_STEP) {
        rkn_step_f2<IB, MODE, UNIT>(a, r, cc, phi);
    } else {
        rkn_step<P, IB, MODE>(a, r, cc, phi);
    }
}

// Kind of the next step of a ray: 0 plain step of a ray inside the grid whose
// prediction stays more than kFaceMargin inside; 1 full step sampled with
// clamped stage points (its prediction ends within kFaceMargin of a face);
// 2 step cut at the face its prediction crosses, length phi, after which the
// ray leaves; 3 plain step of a ray outside the grid (zero RHS).
template <class P>
__device__ __forceinline__ int step_kind(const TraceArgs& a, const Ray<P>& r, typename P::R& phi) {
    using R = typename P::R;
    const R margin = R(kFaceMargin);
    R p[3], w[3];
    bool in = true;
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        p[x] = r.p[x].val();
        w[x] = r.w[x].val();
        in = in & (p[x] >= R(0)) & (p[x] <= lim_of<R>(a.geo, x));
    }
    phi = R(1);
    if (!in) return 3;
    bool near = false;
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        const R pn = p[x] + w[x];
        const R lim = lim_of<R>(a.geo, x);
        if (pn > lim - margin) {
            near = true;
            // distance to the face from the compensated position
            if (pn > lim) phi = fmin(phi, ((lim - r.p[x].hi()) - r.p[x].lo()) / w[x]);
        }
        if (pn < margin) {
            near = true;
            if (pn < R(0)) phi = fmin(phi, (-r.p[x].hi() - r.p[x].lo()) / w[x]);
        }
    }
    phi = fmax(phi, R(0));
    return phi < R(1) ? 2 : (near ? 1 : 0);
}

// Number of steps after the current interior step (kind 0) that are certainly
// kind 0 too, for a trace whose accelerations are bounded by B =
// a.accel_bound: 127, 31, 7 or 0. From the state (p, w) now, after j steps
// |w_j - w| <= j B (each step adds a weighted mean of stage accelerations)
// and |p_j - p - j w| <= B j^2 / 2 (each step moves w_i + (A1 + A2 + A3) / 6),
// so the position p_j and the prediction p_j + w_j lie within
// B (j^2 / 2 + j) of the segment from p + w to p + (j + 1) w. If that segment,
// widened by the bound for j = m plus a rounding slack, keeps kFaceMargin from
// every face, the next m steps are interior steps, and step_kind need not run
// for them: the steps take the same path as with it, bit for bit.
template <class P>
__device__ __forceinline__ int interior_run(const TraceArgs& a, const Ray<P>& r) {
    using R = typename P::R;
    const R B = (R)a.accel_bound;
    const R margin = R(kFaceMargin) + R(0.25);       // face margin + rounding slack (cells)
    R p[3], w[3];
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        p[x] = r.p[x].val();
        w[x] = r.w[x].val();
    }
    auto fits = [&](int m) {
        const R dev = margin + B * R(0.5 * m * m + m);
        bool ok = true;
#pragma unroll
        for (int x = 0; x < 3; ++x) {
            const R e1 = p[x] + w[x], e2 = p[x] + R(m + 1) * w[x];
            ok = ok & (fmin(e1, e2) >= dev) & (fmax(e1, e2) <= lim_of<R>(a.geo, x) - dev);
        }
        return ok;
    };
    if (fits(127)) return 127;
    if (fits(31)) return 31;
    if (fits(7)) return 7;
    return 0;
}

// Whether a trace's interior steps may sample without the grid test: its
// accelerations are bounded by kInteriorAccel (accel_bound carries 0.1% of
// headroom over the bound).
__host__ __device__ __forceinline__ bool interior_sampling_ok(const TraceArgs& a) {
    return a.accel_bound > 0.0f && a.accel_bound <= (float)(kInteriorAccel * 1.001);
}

template <class P>
__device__ __forceinline__ bool ray_in_grid(const TraceArgs& a, const Ray<P>& r) {
    using R = typename P::R;
    bool in = true;
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        const R p = r.p[x].val();
        in = in & (p >= R(0)) & (p <= lim_of<R>(a.geo, x));
    }
    return in;
}

// True once the ray is outside the grid on an axis and moving away from it
// on that axis: its path is then a straight line that never re-enters.
template <class P>
__device__ __forceinline__ bool ray_gone(const TraceArgs& a, const Ray<P>& r) {
    using R = typename P::R;
    bool gone = false;
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        const R p = r.p[x].val(), w = r.w[x].val();
        gone = gone | ((p < R(0)) & (w <= R(0))) | ((p > lim_of<R>(a.geo, x)) & (w >= R(0)));
    }
    return gone;
}

// Writes save j of ray `id` from its state (cells, cells per step, FP64)
// `drift` unit steps before the save time (drift > 0 only for rays that have
// left the grid for good, whose path is a straight line).
template <class R>
__device__ __forceinline__ void emit_save(const TraceArgs& a, unsigned id, int j, double drift,
                                       double p0, double p1, double p2, double w0, double w1,
                                       double w2, double ph, double tau) {
    double x[3], v[3];
    const double p[3] = {p0, p1, p2}, w[3] = {w0, w1, w2};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        x[k] = a.origin[k] + (p[k] + drift * w[k]) * a.spacing[k];
        v[k] = w[k] * a.v_of_w[k];
    }
    const double xa = sel3(x, a.axis), va = sel3(v, a.axis);
    const double x1 = sel3(x, a.t1), v1 = sel3(v, a.t1);
    const double x2 = sel3(x, a.t2), v2 = sel3(v, a.t2);
    double pos1 = x1, pos2 = x2;
    if (a.project) {
        const double tbp = (xa - a.plane) / va;
        pos1 = x1 - v1 * tbp;
        pos2 = x2 - v2 * tbp;
    }
    const size_t n = (size_t)a.n;
    R* jo = reinterpret_cast<R*>(a.jones) + (size_t)j * 4u * n;
    jo[id] = (R)pos1;
    jo[n + id] = (R)atan(v1 / va);
    jo[2 * n + id] = (R)pos2;
    jo[3 * n + id] = (R)atan(v2 / va);
    if (a.state) {
        R* so = reinterpret_cast<R*>(a.state) + (size_t)j * 6u * n;
#pragma unroll
        for (int k = 0; k < 3; ++k) {
            so[k * n + id] = (R)x[k];
            so[(3 + k) * n + id] = (R)v[k];
        }
    }
    if (a.phase) a.phase[(size_t)j * n + id] = ph * a.phase_scale;
    if (a.amp) reinterpret_cast<R*>(a.amp)[(size_t)j * n + id] = (R)exp(-tau * a.tau_scale);
}

template <class P>
__device__ __forceinline__ void emit(const TraceArgs& a, const Ray<P>& r, double drift) {
    emit_save<typename P::R>(a, r.id, r.save_j, drift, r.p[0].vald(), r.p[1].vald(), r.p[2].vald(),
                             r.w[0].vald(), r.w[1].vald(), r.w[2].vald(), r.ph, r.tau.vald());
}

template <class P>
__device__ __forceinline__ void finish_ray(const TraceArgs& a, const Ray<P>& r, uint8_t st,
                                           unsigned long long& my_steps) {
    bool finite = isfinite(r.ph);
#pragma unroll
    for (int k = 0; k < 3; ++k) finite = finite & isfinite(r.p[k].vald()) & isfinite(r.w[k].vald());
    if (!finite) st = SLOTH_RAY_NONFINITE;
    if (a.status) a.status[r.id] = st;
    if (a.steps) a.steps[r.id] = r.step;
    my_steps += (unsigned long long)r.step;
}

// Saves due at the current step, then the end / exit checks. Returns true
// while the ray still needs steps. `check_gone` is false after a plain step
// taken from inside the grid with its prediction more than kFaceMargin inside
// (the ray cannot have left); the outside test is skipped then.
//
// Most steps need nothing here, which the first test decides with integer
// compares. The rest goes through one loop with a single emit call site: a
// save due now is taken at the ray's time (lag), and a ray that has left
// the grid for good takes all its remaining saves by straight-line drift.
// (Two emit call sites with the same arguments let the compiler hoist their
// common part, the state's FP64 conversions and the Jones angles, into
// every step.)
template <class P>
__device__ __forceinline__ bool settle(const TraceArgs& a, Ray<P>& r, unsigned long long& my_steps,
                                      bool check_gone = true) {
    const bool leaving = r.exited || (check_gone && ray_gone<P>(a, r));
    if (r.next_save != r.step && !leaving) return true;
    while (r.save_j < a.n_saves) {
        const bool due = r.next_save == r.step;
        if (!due && !leaving) break;
        const double drift = due ? r.lag : (double)(r.next_save - r.step) + r.lag;
        emit<P>(a, r, drift);
        ++r.save_j;
        r.next_save += a.save_every;
    }
    if (r.save_j >= a.n_saves) {
        finish_ray<P>(a, r, (!r.exited && ray_in_grid<P>(a, r)) ? SLOTH_RAY_INSIDE_AT_END : SLOTH_RAY_EXITED,
                      my_steps);
        return false;
    }
    return true;
}

template <class P>
__device__ __forceinline__ bool start_ray(const TraceArgs& a, unsigned id, Ray<P>& r,
                                          unsigned long long& my_steps) {
    using R = typename P::R;
    const R* rays = reinterpret_cast<const R*>(a.rays);
    const size_t n = (size_t)a.n;
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const double x = (double)rays[k * n + id];
        const double v = (double)rays[(3 + k) * n + id];
        r.p[k].set((x - a.origin[k]) / a.spacing[k]);
        r.w[k].set(v * a.w_of_v[k]);
    }
    r.tau.set(0.0);
    r.ph = 0.0;
    r.lag = 0.0;
    r.exited = false;
    r.step = 0;
    r.save_j = 0;
    r.next_save = a.first_save;
    r.run = 0;
    r.id = id;
    return settle<P>(a, r, my_steps);
}

// Shared-memory bitonic sort of `size` (a power of two, <= kTile) (key, id)
// pairs, ascending by key then id. `size` must be the same in every thread.
__device__ __forceinline__ void tile_sort(unsigned* key, unsigned* id, int size) {
    for (int k = 2; k <= size; k <<= 1) {
        for (int j = k >> 1; j > 0; j >>= 1) {
            for (int i = threadIdx.x; i < size; i += blockDim.x) {
                const int l = i ^ j;
                if (l > i) {
                    const unsigned ki = key[i], kl = key[l], ii = id[i], il = id[l];
                    const bool gt = (ki > kl) || (ki == kl && ii > il);
                    const bool up = (i & k) == 0;
                    if (gt == up) {
                        key[i] = kl; key[l] = ki;
                        id[i] = il; id[l] = ii;
                    }
                }
            }
            __syncthreads();
        }
    }
}

// Traces one tile of `cnt` rays (bucket-ordered ids perm[start..], keys
// skeys[start..]): sorts them by key in shared memory, then the block's warps
// trace them one thread per ray, refilling finished lanes from the tile
// (warp ballot + shared-memory atomic). *s_head must be 0 on entry and the
// block must be synchronised. Shared by the single-trace and serving kernels.
// FAST: 0 every step runs the face test; 1 steps proven interior by the
// acceleration bound skip it and sample without the grid test (bound at most
// kInteriorAccel); 2 they skip the face test but sample with the grid test
// (any finite bound). Every mode takes the same steps.
template <class P, int IB, int FAST, int INTEG = INTEG_RKN, class Cache>
__device__ __forceinline__ void trace_tile(const TraceArgs& a, long long start, int cnt, unsigned* s_key,
                                           unsigned* s_id, int* s_head, Cache& cc,
                                           unsigned long long& my_steps) {
    const unsigned FULL = 0xffffffffu;
    const int lane = threadIdx.x & 31;
    const unsigned lt_mask = (1u << lane) - 1u;
    int size = 32;                      // sort the smallest power of two that holds the tile
    while (size < cnt) size <<= 1;
    for (int i = threadIdx.x; i < size; i += blockDim.x) {
        if (i < cnt) {
            s_key[i] = a.skeys[start + i];
            s_id[i] = a.perm[start + i];
        } else {
            s_key[i] = 0xffffffffu;
            s_id[i] = 0xffffffffu;
        }
    }
    __syncthreads();
    tile_sort(s_key, s_id, size);

    Ray<P> r;
    bool active = false, qempty = false;
    for (;;) {
        const unsigned idle = __ballot_sync(FULL, !active);
        if (idle != 0u && !qempty) {
            const int nidle = __popc(idle);
            const int leader = __ffs(idle) - 1;
            int base = 0;
            if (lane == leader) base = atomicAdd(s_head, nidle);
            base = __shfl_sync(FULL, base, leader);
            if (base + nidle >= cnt) qempty = true;
            if (!active) {
                const int kk = base + __popc(idle & lt_mask);
                if (kk < cnt) active = start_ray<P>(a, s_id[kk], r, my_steps);
            }
        }
        if (__ballot_sync(FULL, active) == 0u) {
            if (qempty) break;
            continue;
        }
        typename P::R phi = typename P::R(1);
        int kind = -1;
        if (active) {
            if (FAST && r.run > 0) {
                --r.run;
                kind = 0;
            } else {
                kind = step_kind<P>(a, r, phi);
                if (FAST && kind == 0) r.run = interior_run<P>(a, r);
            }
        }
        // Fast path: when every lane takes an interior step, the warp takes
        // `extra` more of them in a uniform loop, as many as every lane's run
        // allows before its next save (so no save falls inside the loop and
        // no lane needs the face test, the refill or settle in between).
        int extra = 0;
        if (FAST) {
            const int mine = kind == 0 ? min(r.run, r.next_save - r.step - 1) : 0;
            extra = __reduce_min_sync(FULL, mine);
        }
        if (active) {
            if (FAST && kind == 0) {
#pragma unroll 1
                for (int e = 0;; ++e) {
                    step_any<P, IB, FAST == 1 ? SAMPLE_INTERIOR : SAMPLE_PLAIN, true, INTEG>(
                        a, r, cc, typename P::R(1));
                    if (e == extra) break;
                    ++r.step;
                }
                r.run -= extra;
            } else if (kind == 0 || kind == 3) {
                step_any<P, IB, SAMPLE_PLAIN, true, INTEG>(a, r, cc, typename P::R(1));
            } else {
                step_any<P, IB, SAMPLE_CLAMP, false, INTEG>(a, r, cc, phi);
                if (kind == 2) {
                    r.exited = true;
                    r.lag = 1.0 - (double)phi;
                }
            }
            ++r.step;
            active = settle<P>(a, r, my_steps, kind != 0);
        }
    }
    __syncthreads();
}

// Register cache of the last cell: polynomial coefficients or corners.
template <class P, int IB>
using CellCacheFor = typename std::conditional<
    P::cell_poly,
    typename std::conditional<std::is_same<typename P::R, float>::value && SLOTH_PAIRED_F32,
                              CellPolyF2<(IB != IB_OFF) ? 5 : 4>, CellPoly<P, (IB != IB_OFF) ? 5 : 4>>::type,
    CellCache<P>>::type;

// Sum of `v` over the block, added to *dst by one thread.
__device__ __forceinline__ void block_add(unsigned long long v, unsigned long long* s_acc,
                                          unsigned long long* dst) {
    const unsigned FULL = 0xffffffffu;
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(FULL, v, o);
    if ((threadIdx.x & 31) == 0 && v) atomicAdd(s_acc, v);
    __syncthreads();
    if (threadIdx.x == 0) {
        if (dst && *s_acc) atomicAdd(dst, *s_acc);
        *s_acc = 0;
    }
    __syncthreads();
}

// ---------------------------------------------------------------------------
// Morton bucket pre-pass.
// ---------------------------------------------------------------------------
struct KeyArgs {
    const void* rays;
    long long n;
    double origin[3], inv_h[3];
    int cmax[3];      // n - 2 per axis
    int shift[3];     // right shift to fit 10 bits
    int axis, t1, t2;
    int bucket_shift; // key >> bucket_shift = bucket
    unsigned* keys;
    unsigned* hist;
};

template <class R>
__global__ void __launch_bounds__(256) keys_kernel(const KeyArgs k) {
    const R* rays = reinterpret_cast<const R*>(k.rays);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < k.n; i += stride) {
        unsigned c[3];
#pragma unroll
        for (int a = 0; a < 3; ++a) {
            double u = floor(((double)rays[a * k.n + i] - k.origin[a]) * k.inv_h[a]);
            u = fmin(fmax(u, 0.0), (double)k.cmax[a]);   // NaN -> 0
            c[a] = ((unsigned)u) >> k.shift[a];
        }
        const unsigned c1 = k.t1 == 0 ? c[0] : c[1];
        const unsigned c2 = k.t2 == 1 ? c[1] : c[2];
        const unsigned ca = k.axis == 0 ? c[0] : (k.axis == 1 ? c[1] : c[2]);
        const unsigned key = morton_key(c1, c2, ca);
        k.keys[i] = key;
        atomicAdd(k.hist + (key >> k.bucket_shift), 1u);
    }
}

// Exclusive scan of nb (<= 2^18) counts by one CTA of 1024 threads, in
// passes of 16384 counts: each thread takes 16 consecutive counts (four
// 16-byte loads; hist is 256-byte aligned), the block scans the per-thread
// sums, and a running carry links the passes. The next pass's counts are
// loaded before this pass's block scan, so their latency overlaps it.
constexpr int kScanPer = 16;
constexpr int kScanPass = 1024 * kScanPer;

__device__ __forceinline__ void scan_load(const unsigned* hist, int nb, int i0, unsigned (&x)[kScanPer]) {
    if (i0 + kScanPer <= nb) {
        const uint4* h4 = reinterpret_cast<const uint4*>(hist + i0);
#pragma unroll
        for (int q = 0; q < kScanPer / 4; ++q) {
            const uint4 u = h4[q];
            x[4 * q] = u.x;
            x[4 * q + 1] = u.y;
            x[4 * q + 2] = u.z;
            x[4 * q + 3] = u.w;
        }
    } else {
#pragma unroll
        for (int j = 0; j < kScanPer; ++j) x[j] = i0 + j < nb ? hist[i0 + j] : 0u;
    }
}

static __global__ void __launch_bounds__(1024) scan_kernel(unsigned* hist, int nb) {
    __shared__ unsigned s_warp[32];
    const int t = threadIdx.x, lane = t & 31, wid = t >> 5;
    unsigned v[kScanPer], nx[kScanPer];
    scan_load(hist, nb, t * kScanPer, v);
    unsigned carry = 0;
    for (int base = 0; base < nb; base += kScanPass) {
        const int i0 = base + t * kScanPer;
        if (base + kScanPass < nb) scan_load(hist, nb, i0 + kScanPass, nx);
        unsigned sum = 0;
#pragma unroll
        for (int j = 0; j < kScanPer; ++j) {
            const unsigned c = v[j];
            v[j] = sum;
            sum += c;
        }
        unsigned inc = sum;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const unsigned y = __shfl_up_sync(0xffffffffu, inc, o);
            if (lane >= o) inc += y;
        }
        if (lane == 31) s_warp[wid] = inc;
        __syncthreads();
        if (wid == 0) {
            unsigned w = s_warp[lane];
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned y = __shfl_up_sync(0xffffffffu, w, o);
                if (lane >= o) w += y;
            }
            s_warp[lane] = w;
        }
        __syncthreads();
        const unsigned excl = carry + (inc - sum) + (wid > 0 ? s_warp[wid - 1] : 0u);
        carry += s_warp[31];
        if (i0 + kScanPer <= nb) {
            uint4* h4 = reinterpret_cast<uint4*>(hist + i0);
#pragma unroll
            for (int q = 0; q < kScanPer / 4; ++q)
                h4[q] = make_uint4(v[4 * q] + excl, v[4 * q + 1] + excl, v[4 * q + 2] + excl, v[4 * q + 3] + excl);
        } else {
#pragma unroll
            for (int j = 0; j < kScanPer; ++j)
                if (i0 + j < nb) hist[i0 + j] = v[j] + excl;
        }
        __syncthreads();   // s_warp is rewritten by the next pass
#pragma unroll
        for (int j = 0; j < kScanPer; ++j) v[j] = nx[j];
    }
}

static __global__ void __launch_bounds__(256) scatter_kernel(const unsigned* __restrict__ keys, long long n,
                                                      int bucket_shift, unsigned* offs,
                                                      unsigned* __restrict__ perm,
                                                      unsigned* __restrict__ skeys) {
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const unsigned key = keys[i];
        const unsigned pos = atomicAdd(offs + (key >> bucket_shift), 1u);
        perm[pos] = (unsigned)i;
        skeys[pos] = key;
    }
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
inline size_t align256(size_t x) { return (x + 255u) & ~(size_t)255u; }

constexpr size_t kHeaderBytes = 256;
constexpr size_t kHistBytes = (size_t)4 << kMaxBucketBits;

inline size_t workspace_bytes(long long n) {
    const size_t a = align256((size_t)(n > 0 ? n : 1) * 4u);
    return kHeaderBytes + kHistBytes + 3 * a;
}

inline int bucket_bits_for(long long n) {
    int bits = 0;
    while (bits < kMaxBucketBits && ((long long)1 << bits) * 32 < n) ++bits;
    return bits;
}


// Morton pre-pass of n rays into bucket order: keys, histogram (2^bbits
// buckets, zeroed by the caller), exclusive scan, scatter into perm/skeys.
// The buckets are the keys' top bbits bits; with fine_buckets, the top bbits
// of the bits the grid's keys use, so that a small grid's transverse cells
// get buckets of their own (for kernels that trace rays in bucket order
// without a further sort).
template <class R>
inline int launch_prepass(const SlothGridDesc* g, int axis, const R* rays, long long n, int bbits,
                          unsigned* keys, unsigned* hist, unsigned* perm, unsigned* skeys, int sms,
                          cudaStream_t s, bool fine_buckets = false) {
    const int t1 = axis == 0 ? 1 : 0;
    const int t2 = axis == 2 ? 1 : 2;
    KeyArgs ka;
    ka.rays = rays;
    ka.n = n;
    for (int k = 0; k < 3; ++k) {
        ka.origin[k] = g->origin[k];
        ka.inv_h[k] = 1.0 / g->spacing[k];
        ka.cmax[k] = g->n[k] - 2;
        int sh = 0;
        while (((g->n[k] - 2) >> sh) > 1023) ++sh;
        ka.shift[k] = sh;
    }
    ka.axis = axis;
    ka.t1 = t1;
    ka.t2 = t2;
    ka.bucket_shift = 30 - bbits;
    if (fine_buckets) {
        int tb = 0;   // bits of the largest transverse cell coordinate
        for (int t : {t1, t2})
            while (((g->n[t] - 2) >> ka.shift[t]) >> tb) ++tb;
        const int used = 2 * tb + 10;
        ka.bucket_shift = used > bbits ? used - bbits : 0;
    }
    ka.keys = keys;
    ka.hist = hist;
    const long long nblk = (n + 255) / 256;
    const int kb = (int)(nblk < (long long)sms * 8 ? nblk : (long long)sms * 8);
    keys_kernel<R><<<kb, 256, 0, s>>>(ka);
    note_launch();
    scan_kernel<<<1, 1024, 0, s>>>(hist, 1 << bbits);
    note_launch();
    scatter_kernel<<<kb, 256, 0, s>>>(keys, n, ka.bucket_shift, hist, perm, skeys);
    note_launch();
    return cuda_status(cudaGetLastError());
}

// Inverse-bremsstrahlung path of a trace: off, sub-critical (the grid's
// density stays below nc, so the Coulomb log is a constant), or general.
inline int trace_mode(const SlothTraceParams* p) {
    const double xmax = p->q_max > 0.0 ? p->q_max * p->ope_ratio2 : 1e300;
    return !p->inv_brems ? IB_OFF : (xmax <= 1.0 ? IB_SUBCRITICAL : IB_GENERAL);
}

// Largest |acceleration| (cells per step^2) the grid's density range allows:
// max_k |S_k| * (q_max - min(q_min, 0)); infinite when the range is unknown.
inline double interior_accel_bound(const SlothGridDesc* g, const SlothTraceParams* p) {
    if (!(p->q_max > 0.0) || !std::isfinite(p->q_min) || !(p->q_min <= p->q_max)) return INFINITY;
    double smax = 0.0;
    for (int k = 0; k < 3; ++k) {
        const double r = p->dtau / g->spacing[k];
        smax = fmax(smax, 0.5 * r * r);
    }
    return smax * (p->q_max - fmin(p->q_min, 0.0));
}

// Kernel arguments of one trace from the public descriptors.
inline void fill_trace_args(TraceArgs& ta, const SlothGridDesc* g, const void* grid, const SlothTraceParams* p,
                            const void* rays, long long n, const SlothTraceOutputs* out, const unsigned* perm,
                            const unsigned* skeys) {
    const int axis = p->probing_axis;
    ta.geo = make_geo(g);
    ta.grid = grid;
    ta.rays = rays;
    ta.n = n;
    ta.perm = perm;
    ta.skeys = skeys;
    ta.tile_counter = nullptr;
    ta.n_tiles = (int)((n + kTile - 1) / kTile);
    ta.n_big = ta.n_tiles;
    for (int k = 0; k < 3; ++k) {
        const double h = g->spacing[k];
        ta.origin[k] = g->origin[k];
        ta.spacing[k] = h;
        ta.w_of_v[k] = (p->dtau / h) / kC;
        ta.v_of_w[k] = kC * h / p->dtau;
        ta.S[k] = -0.5 * (p->dtau / h) * (p->dtau / h);
        ta.Sf[k] = (float)ta.S[k];
        // as the step forms them at phi = 1: exact scalings by 1/4 and 1/2, one
        // FP32 rounding of fl(1/6) * Sf
        ta.S4f[k] = 0.25f * ta.Sf[k];
        ta.S2f[k] = 0.5f * ta.Sf[k];
        ta.S6f[k] = (1.0f / 6.0f) * ta.Sf[k];
    }
    ta.phase_scale = (p->omega / kC) * p->dtau / 6.0;
    ta.tau_scale = p->kappa_q2 * p->dtau / 6.0;   // times cl_lo below for the sub-critical mode
    ta.cl_w = p->coulomb_log_w;
    ta.cl_lo = p->coulomb_log_w > 2.0 ? p->coulomb_log_w : 2.0;
    ta.ope2 = p->ope_ratio2;
    ta.ope2f = (float)ta.ope2;
    ta.inv_ope2 = 1.0 / p->ope_ratio2;
    ta.inv_ope2f = (float)ta.inv_ope2;
    ta.cl_lof = (float)ta.cl_lo;
    // Below the critical density the Coulomb log is the constant cl_lo and the
    // corners carry x^2 = (ope2 q)^2, so the optical depth's scale takes
    // cl_lo / ope2^2 once.
    if (trace_mode(p) == IB_SUBCRITICAL) ta.tau_scale *= ta.cl_lo * ta.inv_ope2 * ta.inv_ope2;
    ta.cl_wf = (float)ta.cl_w;
    {
        const double B = interior_accel_bound(g, p);
        ta.accel_bound = std::isfinite(B) ? (float)(B * 1.001) : 0.0f;
    }
    ta.plane = p->plane;
    ta.first_save = p->first_save;
    ta.save_every = p->n_saves > 1 ? p->save_every : 1;
    ta.n_saves = p->n_saves;
    ta.axis = axis;
    ta.t1 = axis == 0 ? 1 : 0;
    ta.t2 = axis == 2 ? 1 : 2;
    ta.project = p->project_to_plane ? 1 : 0;
    ta.jones = out->jones;
    ta.state = out->state;
    ta.phase = out->phase;
    ta.amp = out->amp;
    ta.status = out->status;
    ta.steps = out->steps;
    ta.total_steps = out->total_steps;
}

// Validation shared by the trace entry points (everything but buffers).
inline int check_trace_params(const SlothGridDesc* g, const SlothTraceParams* p, int64_t n) {
    int rc = check_grid(g);
    if (rc) return rc;
    if (!p) return SLOTH_ERR_NULL_POINTER;
    if (n < 0 || n > 2147483647LL) return n < 0 ? SLOTH_ERR_INVALID_ARGUMENT : SLOTH_ERR_TOO_LARGE;
    if (!(p->omega > 0.0) || !(p->dtau > 0.0) || !std::isfinite(p->dtau) || !std::isfinite(p->omega))
        return SLOTH_ERR_INVALID_ARGUMENT;
    if (p->n_saves < 1 || p->n_saves > SLOTH_MAX_SAVES || p->first_save < 0) return SLOTH_ERR_INVALID_ARGUMENT;
    if (p->n_saves > 1 && p->save_every < 1) return SLOTH_ERR_INVALID_ARGUMENT;
    if (p->probing_axis < 0 || p->probing_axis > 2) return SLOTH_ERR_INVALID_ARGUMENT;
    const long long last =
        (long long)p->first_save + (long long)(p->n_saves - 1) * (p->n_saves > 1 ? p->save_every : 0);
    if (last > 2000000000LL) return SLOTH_ERR_TOO_LARGE;
    if (p->inv_brems && !(p->kappa_q2 >= 0.0)) return SLOTH_ERR_INVALID_ARGUMENT;
    if (p->project_to_plane && !std::isfinite(p->plane)) return SLOTH_ERR_INVALID_ARGUMENT;
    if (!(p->ope_ratio2 > 0.0) || !std::isfinite(p->ope_ratio2)) return SLOTH_ERR_INVALID_ARGUMENT;
    if (!std::isfinite(p->q_max)) return SLOTH_ERR_INVALID_ARGUMENT;
    if (p->integrator != SLOTH_INTEGRATOR_RKN && p->integrator != SLOTH_INTEGRATOR_RK4)
        return SLOTH_ERR_INVALID_ARGUMENT;
    if (p->reserved != 0) return SLOTH_ERR_INVALID_ARGUMENT;
    return SLOTH_OK;
}

// True when interior steps may skip the per-stage grid test: the
// acceleration |S_k * dq/du_k| is at most max_k |S_k| * (q_max - min(q_min, 0))
// (a difference of q over at most one cell), and that is within
// kInteriorAccel. Needs q_max > 0 (known) and q_min <= q_max.
inline bool interior_bound_ok(const SlothGridDesc* g, const SlothTraceParams* p) {
    return interior_accel_bound(g, p) <= kInteriorAccel;
}


}  // namespace sloth
