// Detector-image forward model and its adjoint: the gradient of a loss on a
// synthetic detector image with respect to the density grid.
//
// No counterpart in the reference, which never differentiates. The model
// differentiates the reference's ray equations (src/core/propagator.py:
// 168-243, dr/dt = v, dv/dt = -(c^2/2) grad(ne/nc) from the precomputed
// gradient grid through the trilinear interpolator, src/core/interpolator.py:
// 79-104, fill 0 outside) through a detector image:
//
//   ne --pack (K1)--> (q, dq/du, dq/dv, dq/dw)
//      --fixed-step Runge-Kutta-Nystrom, at most n_steps steps--> final ray state
//      --straight line to the detector plane--> (X, Y)
//      --Gaussian splat--> image I
//
// The step is the tracer's (fourth-order Runge-Kutta-Nystrom, unit steps in
// grid cells) without face
// clipping: every stage samples the interpolant with fill 0 outside, so a
// ray's map is smooth except where a stage point crosses a grid face. A ray
// stops early once it is outside the grid on some axis and moving away from
// it along that axis: its remaining steps are straight lines, and the
// projection to the detector plane (src/shared/propagation.py:92-134) gives
// the same point from any point of that line.
//
// Splat: a ray at pixel coordinates (a, b) adds norm * g(i - a) * g(j - b)
// to pixel (i, j), with g(d) = exp(-d^2 / (2 s^2)) * taper(|d| / s), taper = 1
// up to 3 s and a C2 smoothstep from 1 to 0 between 3 s and 4 s, and norm =
// 1 / (2 pi s^2). The taper keeps the splat twice differentiable with a
// finite support of 4 s.
//
// Adjoint (backward): for each ray, d L / d(final state) from the image
// gradient through the splat and the projection; then, segment by segment
// from the last, the trajectory is recomputed from the segment's checkpoint
// (the forward stores one every ckpt_every steps) and the discrete adjoint of
// each step runs in reverse. Each stage's contribution to d L / d(grid
// gradient channels) is accumulated in registers for the 8 corners of the
// stage's cell and added to the grid-gradient buffer when the cell changes.
// pack_adjoint_kernel maps d L / d(packed grid) through the transposed
// difference stencil of K1 to d L / d ne.
#include <climits>
#include <cmath>

#include "tracer.cuh"

namespace sloth {

constexpr int kAdjThreads = 256;
// The backward's recompute of a checkpoint segment records where each stage
// of each step sampled the field (its cell and in-cell coordinates), and the
// step adjoints linearise there. Stages 1 and 2's in-cell coordinates go to
// shared memory, [step][word][thread] so that a warp's accesses are
// consecutive (5 words per step); the three cells and the other in-cell
// coordinates stay in a per-thread array. 128 threads per CTA: a 20-step
// segment takes 51 KB of shared memory in FP32, so four CTAs share an SM
// (16 warps; the kernel is latency-bound).
constexpr int kAdjBwdThreads = 128;
constexpr int kAdjStateWords = 5;
// Two FP32 builds of the backward: four CTAs per SM (128 registers) when
// four segment buffers fit an SM's shared memory (on B200, 228 KB per SM and
// 1 KB reserved per CTA: checkpoints at most every 21 steps), three (152
// registers) otherwise. FP64 runs one CTA per SM.
// The FP32 forward fits three 256-thread CTAs per SM (80 registers) without spilling.
template <class P> constexpr int adj_fwd_min_blocks() { return sizeof(typename P::R) == 4 ? 3 : 1; }
constexpr int kMaxCkptEvery = 32;
constexpr int kMaxTaps = 65;          // 2 * 4 * sigma + 1 pixels at sigma <= 8

struct ImageArgs {
    GridGeo geo;
    const void* grid;
    const void* rays;            // (6, n) of R, original order
    long long n;
    const unsigned* perm;        // slot -> ray id (bucket order)
    double origin[3], w_of_v[3], inv_h[3];
    double S[3];                 // -(dtau/h)^2 / 2
    float Sf[3];                 // S rounded to FP32 once on the host (the FP32 kernels' copy)
    int n_steps, ckpt_every, n_seg;
    int axis, t1, t2;
    double plane;                // detector plane (cells along axis)
    double px0[2], px_per_cell[2];
    int npx[2];
    int taps;                    // pixels per axis in a splat window
    double sigma, radius, norm;  // pixels
    void* ckpt;                  // [n_seg + 1][12 floats | 6 doubles][n]
    int* nsteps;                 // steps taken, per slot
    void* image;                 // forward: the image; backward: d L / d image
    void* ggrad;                 // backward: d L / d(packed grid)
    unsigned long long* total_steps;   // forward: steps of all rays are added here (may be null)
    const unsigned* accel_bound;       // float bits of max |S_k dq/du_k| over the grid (workspace)
};

// S_k in the kernel's precision: FP32 kernels read the host-rounded copy, so
// no step converts it.
template <class R> __device__ __forceinline__ R img_S(const ImageArgs& a, int k);
template <> __device__ __forceinline__ float img_S<float>(const ImageArgs& a, int k) { return a.Sf[k]; }
template <> __device__ __forceinline__ double img_S<double>(const ImageArgs& a, int k) { return a.S[k]; }

// ---------------------------------------------------------------------------
// Ray state and checkpoints.
// ---------------------------------------------------------------------------
template <class P>
struct MState {
    typename P::Acc p[3], w[3];
};

// A checkpoint is 48 bytes per ray: FP32 stores the value and compensation of
// each of the six sums, FP64 the six values; component-major for coalescing.
template <class P>
__device__ __forceinline__ void store_state(const ImageArgs& a, int k, long long slot, const MState<P>& r) {
    if constexpr (sizeof(typename P::R) == 4) {
        float* c = reinterpret_cast<float*>(a.ckpt) + (size_t)k * 12 * a.n + slot;
#pragma unroll
        for (int x = 0; x < 3; ++x) {
            c[(2 * x) * a.n] = r.p[x].s;
            c[(2 * x + 1) * a.n] = r.p[x].c;
            c[(6 + 2 * x) * a.n] = r.w[x].s;
            c[(7 + 2 * x) * a.n] = r.w[x].c;
        }
    } else {
        double* c = reinterpret_cast<double*>(a.ckpt) + (size_t)k * 6 * a.n + slot;
#pragma unroll
        for (int x = 0; x < 3; ++x) {
            c[x * a.n] = r.p[x].s;
            c[(3 + x) * a.n] = r.w[x].s;
        }
    }
}

template <class P>
__device__ __forceinline__ void load_state(const ImageArgs& a, int k, long long slot, MState<P>& r) {
    if constexpr (sizeof(typename P::R) == 4) {
        const float* c = reinterpret_cast<const float*>(a.ckpt) + (size_t)k * 12 * a.n + slot;
#pragma unroll
        for (int x = 0; x < 3; ++x) {
            r.p[x].s = c[(2 * x) * a.n];
            r.p[x].c = c[(2 * x + 1) * a.n];
            r.w[x].s = c[(6 + 2 * x) * a.n];
            r.w[x].c = c[(7 + 2 * x) * a.n];
        }
    } else {
        const double* c = reinterpret_cast<const double*>(a.ckpt) + (size_t)k * 6 * a.n + slot;
#pragma unroll
        for (int x = 0; x < 3; ++x) {
            r.p[x].s = c[x * a.n];
            r.w[x].s = c[(3 + x) * a.n];
        }
    }
}

// Outside the grid on some axis and moving away from it along that axis (or
// not finite): every later step is a straight line.
template <class P>
__device__ __forceinline__ bool ray_gone_model(const ImageArgs& a, const MState<P>& r) {
    using R = typename P::R;
    bool gone = false;
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        const R p = r.p[x].val(), w = r.w[x].val();
        gone |= (p < R(0) && w <= R(0)) || (p > lim_of<R>(a.geo, x) && w >= R(0)) || !(p == p) || !(w == w);
    }
    return gone;
}

// ---------------------------------------------------------------------------
// The gradient channels of one cell as trilinear polynomials.
// ---------------------------------------------------------------------------
template <class P>
struct GradCell {
    unsigned base;
    typename P::R t[3][8];
};

// Cell and in-cell coordinates of the point hi + lo (the tracer's split: the
// cell from the rounded sum, the fractions from (hi - i) + lo). False when
// the point is outside the grid (fill 0).
template <class P, bool INTERIOR = false>
__device__ __forceinline__ bool locate(const GridGeo& g, const typename P::R (&hi)[3],
                                       const typename P::R (&lo)[3], unsigned& base, typename P::R (&f)[3]) {
    using R = typename P::R;
    R p[3];
#pragma unroll
    for (int x = 0; x < 3; ++x) p[x] = hi[x] + lo[x];
    int ix, iy, iz;
    if constexpr (!INTERIOR) {
        const bool in = (p[0] >= R(0)) & (p[0] <= lim_of<R>(g, 0)) & (p[1] >= R(0)) &
                        (p[1] <= lim_of<R>(g, 1)) & (p[2] >= R(0)) & (p[2] <= lim_of<R>(g, 2));
        if (!in) return false;
        ix = min((int)p[0], g.n[0] - 2);
        iy = min((int)p[1], g.n[1] - 2);
        iz = min((int)p[2], g.n[2] - 2);
    } else {
        // a point of an interior step: inside by construction; one unsigned
        // min per axis keeps the index in the grid all the same
        ix = (int)min((unsigned)(int)p[0], (unsigned)(g.n[0] - 2));
        iy = (int)min((unsigned)(int)p[1], (unsigned)(g.n[1] - 2));
        iz = (int)min((unsigned)(int)p[2], (unsigned)(g.n[2] - 2));
    }
    f[0] = (hi[0] - (R)ix) + lo[0];
    f[1] = (hi[1] - (R)iy) + lo[1];
    f[2] = (hi[2] - (R)iz) + lo[2];
    base = (unsigned)ix * g.sx + (unsigned)iy * g.sy + (unsigned)iz;
    return true;
}

// FP32: the gradient channels as two polynomial pairs, (q, dq/du) and
// (dq/dv, dq/dw), in the float4 voxel's own register pairs, evaluated with
// sm_100's paired FP32 instructions (q is carried along at no cost).
struct GradCellF2 {
    unsigned base;
    float2 t[2][8];
};

__device__ __forceinline__ void load_cell_f2(const ImageArgs& a, unsigned b, GradCellF2& cc) {
    if (b == cc.base) return;
    cc.base = b;
    const GridGeo& g = a.geo;
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
}

template <class P>
__device__ __forceinline__ void load_cell(const ImageArgs& a, unsigned b, GradCell<P>& cc) {
    using R = typename P::R;
    if (b == cc.base) return;
    cc.base = b;
    const GridGeo& g = a.geo;
    const typename P::V v0 = P::load(a.grid, b), v1 = P::load(a.grid, b + 1u);
    const typename P::V v2 = P::load(a.grid, b + g.sy), v3 = P::load(a.grid, b + g.sy + 1u);
    const typename P::V v4 = P::load(a.grid, b + g.sx), v5 = P::load(a.grid, b + g.sx + 1u);
    const typename P::V v6 = P::load(a.grid, b + g.sx + g.sy), v7 = P::load(a.grid, b + g.sx + g.sy + 1u);
    poly_coeffs<R>(cc.t[0], v0.y, v1.y, v2.y, v3.y, v4.y, v5.y, v6.y, v7.y);
    poly_coeffs<R>(cc.t[1], v0.z, v1.z, v2.z, v3.z, v4.z, v5.z, v6.z, v7.z);
    poly_coeffs<R>(cc.t[2], v0.w, v1.w, v2.w, v3.w, v4.w, v5.w, v6.w, v7.w);
}

// Where one stage sampled the field: the cell (kNone when the point was
// outside the grid, fill 0) and the in-cell coordinates. The backward's
// recompute records the three stages of every step, and the step's adjoint
// linearises at exactly those points.
constexpr unsigned kNone = 0xffffffffu;

template <class P>
struct StageRec {
    unsigned b;
    typename P::R f[3];
};

// Acceleration S * grad(q) at hi + lo (zero outside); with rec, where it
// sampled.
template <class P, bool INTERIOR, class Cell>
__device__ __forceinline__ void accel(const ImageArgs& a, const typename P::R (&hi)[3], const typename P::R (&lo)[3],
                                      typename P::R (&A)[3], Cell& cc, StageRec<P>* rec = nullptr) {
    using R = typename P::R;
    unsigned b;
    R f[3];
    if (!locate<P, INTERIOR>(a.geo, hi, lo, b, f)) {
        A[0] = A[1] = A[2] = R(0);
        if (rec) {
            rec->b = kNone;
            rec->f[0] = rec->f[1] = rec->f[2] = R(0);
        }
        return;
    }
    if (rec) {
        rec->b = b;
        rec->f[0] = f[0];
        rec->f[1] = f[1];
        rec->f[2] = f[2];
    }
    if constexpr (std::is_same<Cell, GradCellF2>::value) {
        load_cell_f2(a, b, cc);
        const float2 fx = make_float2(f[0], f[0]), fy = make_float2(f[1], f[1]), fz = make_float2(f[2], f[2]);
        const float2 r0 = poly_eval2(cc.t[0], fx, fy, fz), r1 = poly_eval2(cc.t[1], fx, fy, fz);
        A[0] = img_S<R>(a, 0) * r0.y;
        A[1] = img_S<R>(a, 1) * r1.x;
        A[2] = img_S<R>(a, 2) * r1.y;
    } else {
        load_cell<P>(a, b, cc);
#pragma unroll
        for (int k = 0; k < 3; ++k) A[k] = img_S<R>(a, k) * poly_eval<R>(cc.t[k], f[0], f[1], f[2]);
    }
}

// One step (the tracer's Runge-Kutta-Nystrom step with phi = 1, without
// phase and depth):
//   p' = p + w + (A1 + 2 A2)/6,  w' = w + (A1 + 4 A2 + A3)/6,
//   stages at p, p + w/2 + A1/8, p + w + A2/2.
template <class P, bool INTERIOR = false, class Cell>
__device__ __forceinline__ void model_step(const ImageArgs& a, MState<P>& r, Cell& cc, StageRec<P>* rec = nullptr) {
    using R = typename P::R;
    R ph[3], pl[3], we[3], st[3], A1[3], A2[3], A3[3];
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        ph[x] = r.p[x].hi();
        pl[x] = r.p[x].lo();
        we[x] = r.w[x].val();
    }
    accel<P, INTERIOR>(a, ph, pl, A1, cc, rec);
#pragma unroll
    for (int x = 0; x < 3; ++x) st[x] = pl[x] + (R(0.5) * we[x] + R(0.125) * A1[x]);
    accel<P, INTERIOR>(a, ph, st, A2, cc, rec ? rec + 1 : nullptr);
#pragma unroll
    for (int x = 0; x < 3; ++x) st[x] = pl[x] + (we[x] + R(0.5) * A2[x]);
    accel<P, INTERIOR>(a, ph, st, A3, cc, rec ? rec + 2 : nullptr);
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        const R sA = A1[x] + R(2) * A2[x];
        const R sW = (A1[x] + R(4) * A2[x]) + A3[x];
        r.p[x].add(r.w[x].hi() + (r.w[x].lo() + sA * R(1.0 / 6.0)));
        r.w[x].add(sW * R(1.0 / 6.0));
    }
}

// ---------------------------------------------------------------------------
// Adjoint of one step.
// ---------------------------------------------------------------------------
template <class P>
struct CornerAcc {
    unsigned base;               // cell of the pending sums (kNone: none)
    typename P::R v[3][8];       // d L / d(channel k) at corner c
};

template <class P> struct AdjTypes { using Cell = GradCell<P>; using Acc = CornerAcc<P>; };
struct CornerAccF2;
template <> struct AdjTypes<PolF32> { using Cell = GradCellF2; using Acc = CornerAccF2; };

// Adds (x, y, z, w) to *p as one vector reduction that returns nothing
// (red.global.add.v4.f32, sm_90 and later). A float4 atomicAdd compiles to
// an atomic that sends each old value back through the crossbar; with about
// one flush of eight corners per three ray-steps that return traffic cost
// the backward 9% of its time.
__device__ __forceinline__ void red_add_v4(float4* p, float x, float y, float z, float w) {
    asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};"
                 :: "l"(p), "f"(x), "f"(y), "f"(z), "f"(w) : "memory");
}

template <class P>
__device__ __forceinline__ void flush(const ImageArgs& a, CornerAcc<P>& acc) {
    using R = typename P::R;
    if (acc.base == kNone) return;
    const GridGeo& g = a.geo;
    const unsigned b = acc.base;
    const unsigned off[8] = {b, b + 1u, b + g.sy, b + g.sy + 1u, b + g.sx, b + g.sx + 1u, b + g.sx + g.sy,
                             b + g.sx + g.sy + 1u};
#pragma unroll
    for (int c = 0; c < 8; ++c) {
        if constexpr (sizeof(R) == 4) {
            red_add_v4(reinterpret_cast<float4*>(a.ggrad) + off[c], 0.0f, acc.v[0][c], acc.v[1][c], acc.v[2][c]);
        } else {
            double* d = reinterpret_cast<double*>(a.ggrad) + 4 * (size_t)off[c];
            atomicAdd(d + 1, acc.v[0][c]);
            atomicAdd(d + 2, acc.v[1][c]);
            atomicAdd(d + 3, acc.v[2][c]);
        }
    }
    acc.base = kNone;
}

// FP32 corner sums as pairs: v[k][i] holds channel k + 1 at corners 2i and
// 2i + 1, which differ in z only, so that a pair is one sm_100 paired FP32
// operation and one pair of adjacent voxels in the flush.
struct CornerAccF2 {
    unsigned base;
    float2 v[3][4];
};

// The lanes of a warp that flush the same cell together first combine their
// corner sums in groups of up to four, and one lane per group of four issues
// the eight reductions. Rays of a warp share their entry cell and cross cell
// faces at the same steps, so a flush typically has most of the warp in one
// cell; 26 lanes issuing eight reductions each to the same eight voxels
// serialise in L2 (about a third of the backward's time before this). The
// combination is a tree over the members' ranks (the lanes that flush the same
// cell, in lane order): at stride d, rank r (r a multiple of 2d) adds the
// partial sum of rank r + d, found by pointer jumping (the member d ranks up
// is the member d/2 ranks up of the member d/2 ranks up). Two rounds measured
// best: 11.2 ms for the bench's backward, against 12.1 ms for a tree over the
// whole group (its shuffles cost more than the reductions they save) and
// 13.1 ms without combining. Every lane of `active` (the lanes that reached
// this call together) runs the same rounds, so the shuffles are matched.
constexpr int kFlushCombine = 4;   // lanes combined per reduction, a power of two
__device__ __forceinline__ void flush(const ImageArgs& a, CornerAccF2& acc) {
    const unsigned active = __activemask();
    const unsigned grp = __match_any_sync(active, acc.base);
    const int lane = threadIdx.x & 31;
    const unsigned above = grp & ~((2u << lane) - 1u);       // members above this lane
    int up = above ? __ffs(above) - 1 : lane;                // the member one rank up
    int has = above != 0u;
    const int rank = __popc(grp & ((1u << lane) - 1u));
    const int rounds = __reduce_max_sync(active, __popc(grp));
    int span = 1;   // after the rounds, rank r (a multiple of span) holds ranks r .. r + span - 1
    for (int d = 1; d < rounds && d < kFlushCombine; d <<= 1) {
        span = 2 * d;
        const float take = (has && (rank & (2 * d - 1)) == 0) ? 1.0f : 0.0f;
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const float tx = __shfl_sync(active, acc.v[k][i].x, up);
                const float ty = __shfl_sync(active, acc.v[k][i].y, up);
                acc.v[k][i].x = fmaf(take, tx, acc.v[k][i].x);
                acc.v[k][i].y = fmaf(take, ty, acc.v[k][i].y);
            }
        const int up2 = __shfl_sync(active, up, up);
        const int has2 = __shfl_sync(active, has, up);
        has = has && has2;
        up = has ? up2 : lane;   // no member that far up: read this lane's own sums (taken times 0)
    }
    if ((rank & (span - 1)) == 0 && acc.base != kNone) {
        const GridGeo& g = a.geo;
        const unsigned b = acc.base;
        const unsigned off[4] = {b, b + g.sy, b + g.sx, b + g.sx + g.sy};
        float4* gg = reinterpret_cast<float4*>(a.ggrad);
#pragma unroll
        for (int i = 0; i < 4; ++i) {
            red_add_v4(gg + off[i], 0.0f, acc.v[0][i].x, acc.v[1][i].x, acc.v[2][i].x);
            red_add_v4(gg + off[i] + 1u, 0.0f, acc.v[0][i].y, acc.v[1][i].y, acc.v[2][i].y);
        }
    }
    acc.base = kNone;
}

// Stage adjoint on the paired FP32 cache: channels 2 and 3 of the Jacobian
// transpose, the corner weights and the corner sums run as paired FP32
// operations (__ffma2_rn / __fmul2_rn), channel 1 scalar.
template <class P>
__device__ __forceinline__ void stage_adjoint(const ImageArgs& a, const StageRec<PolF32>& rec,
                                              const float (&Abar)[3], float (&q)[3], GradCellF2& cc,
                                              CornerAccF2& acc) {
    const unsigned b = rec.b;
    if (b == kNone) {
        q[0] = q[1] = q[2] = 0.0f;
        return;
    }
    const float f[3] = {rec.f[0], rec.f[1], rec.f[2]};
    load_cell_f2(a, b, cc);
    const float fx = f[0], fy = f[1], fz = f[2];
    const float2 fx2 = make_float2(fx, fx), fy2 = make_float2(fy, fy), fz2 = make_float2(fz, fz);
    float gb[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) gb[k] = img_S<float>(a, k) * Abar[k];
    // J^T gb. Channel 1 (dq/du) is the .y half of pair 0, channels 2 and 3 are pair 1.
    const float2* t0 = cc.t[0];
    const float2* t1 = cc.t[1];
    const float u76 = fmaf(fx, t0[7].y, t0[6].y);
    const float d1x = fmaf(fz, fmaf(fy, t0[7].y, t0[5].y), fmaf(fy, t0[4].y, t0[1].y));
    const float d1y = fmaf(fz, u76, fmaf(fx, t0[4].y, t0[2].y));
    const float d1z = fmaf(fy, u76, fmaf(fx, t0[5].y, t0[3].y));
    const float2 v76 = __ffma2_rn(fx2, t1[7], t1[6]);
    const float2 d2x = __ffma2_rn(fz2, __ffma2_rn(fy2, t1[7], t1[5]), __ffma2_rn(fy2, t1[4], t1[1]));
    const float2 d2y = __ffma2_rn(fz2, v76, __ffma2_rn(fx2, t1[4], t1[2]));
    const float2 d2z = __ffma2_rn(fy2, v76, __ffma2_rn(fx2, t1[5], t1[3]));
    q[0] = fmaf(gb[2], d2x.y, fmaf(gb[1], d2x.x, gb[0] * d1x));
    q[1] = fmaf(gb[2], d2y.y, fmaf(gb[1], d2y.x, gb[0] * d1y));
    q[2] = fmaf(gb[2], d2z.y, fmaf(gb[1], d2z.x, gb[0] * d1z));
    if (b != acc.base) {
        flush(a, acc);
        acc.base = b;
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int i = 0; i < 4; ++i) acc.v[k][i] = make_float2(0.0f, 0.0f);
    }
    // corner weights: pair i = (corner 2i, 2i + 1) = X * Y * (1 - fz, fz) with
    // X = 1 - fx or fx (i >> 1), Y = 1 - fy or fy (i & 1)
    const float2 one = make_float2(1.0f, 1.0f), neg = make_float2(-1.0f, -1.0f);
    const float2 ex2 = __ffma2_rn(fx2, neg, one), ey2 = __ffma2_rn(fy2, neg, one);
    const float2 zz = __ffma2_rn(fz2, make_float2(-1.0f, 1.0f), make_float2(1.0f, 0.0f));
    const float2 xz0 = __fmul2_rn(ex2, zz), xz1 = __fmul2_rn(fx2, zz);
    const float2 w[4] = {__fmul2_rn(xz0, ey2), __fmul2_rn(xz0, fy2), __fmul2_rn(xz1, ey2), __fmul2_rn(xz1, fy2)};
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const float2 g2 = make_float2(gb[k], gb[k]);
#pragma unroll
        for (int i = 0; i < 4; ++i) acc.v[k][i] = __ffma2_rn(g2, w[i], acc.v[k][i]);
    }
}

// Stage adjoint: with Abar = d L / d(stage acceleration), adds
// Abar_k * S_k * (corner weight) to the corners of the stage's cell and
// returns q = J^T (S * Abar), J = d grad(q) / d p at the stage point.
template <class P>
__device__ __forceinline__ void stage_adjoint(const ImageArgs& a, const StageRec<P>& rec,
                                              const typename P::R (&Abar)[3], typename P::R (&q)[3],
                                              GradCell<P>& cc, CornerAcc<P>& acc) {
    using R = typename P::R;
    const unsigned b = rec.b;
    if (b == kNone) {
        q[0] = q[1] = q[2] = R(0);
        return;
    }
    const R f[3] = {rec.f[0], rec.f[1], rec.f[2]};
    load_cell<P>(a, b, cc);
    const R fx = f[0], fy = f[1], fz = f[2];
    R gb[3];
#pragma unroll
    for (int k = 0; k < 3; ++k) gb[k] = img_S<R>(a, k) * Abar[k];
    // J^T gb: derivatives of the three trilinear polynomials
    q[0] = q[1] = q[2] = R(0);
#pragma unroll
    for (int k = 0; k < 3; ++k) {
        const R* t = cc.t[k];
        const R dx = (t[1] + fy * t[4]) + fz * (t[5] + fy * t[7]);
        const R dy = (t[2] + fx * t[4]) + fz * (t[6] + fx * t[7]);
        const R dz = (t[3] + fx * t[5]) + fy * (t[6] + fx * t[7]);
        q[0] += gb[k] * dx;
        q[1] += gb[k] * dy;
        q[2] += gb[k] * dz;
    }
    // corner weights, corner index 4*dx + 2*dy + dz
    if (b != acc.base) {
        flush<P>(a, acc);
        acc.base = b;
#pragma unroll
        for (int k = 0; k < 3; ++k)
#pragma unroll
            for (int c = 0; c < 8; ++c) acc.v[k][c] = R(0);
    }
    const R ex = R(1) - fx, ey = R(1) - fy, ez = R(1) - fz;
    const R w00 = ex * ey, w01 = ex * fy, w10 = fx * ey, w11 = fx * fy;
    const R w[8] = {w00 * ez, w00 * fz, w01 * ez, w01 * fz, w10 * ez, w10 * fz, w11 * ez, w11 * fz};
#pragma unroll
    for (int k = 0; k < 3; ++k)
#pragma unroll
        for (int c = 0; c < 8; ++c) acc.v[k][c] += gb[k] * w[c];
}

// Reverse of model_step from where its three stages sampled the field (the
// records of the recompute): (lp, lw) = adjoint of the output (p', w') on
// entry, of the input (p, w) on return. The step's stage points are
// p, p + w/2 + A1/8 and p + w + A2/2, so the chain through them needs only
// each stage's Jacobian transpose, not the step's p or w.
template <class P, class Cell, class Acc>
__device__ __forceinline__ void model_step_adjoint(const ImageArgs& a, const StageRec<P> (&rec)[3],
                                                   typename P::R (&lp)[3], typename P::R (&lw)[3], Cell& cc,
                                                   Acc& acc) {
    using R = typename P::R;
    // Direct terms of p' = p + w + (A1 + 2 A2)/6, w' = w + (A1 + 4 A2 + A3)/6:
    R a1[3], a2[3], a3[3], pb[3], wb[3], q[3];
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        a1[x] = (lp[x] + lw[x]) * R(1.0 / 6.0);
        a2[x] = lp[x] * R(1.0 / 3.0) + lw[x] * R(2.0 / 3.0);
        a3[x] = lw[x] * R(1.0 / 6.0);
        pb[x] = lp[x];
        wb[x] = lp[x] + lw[x];
    }
    // stage 3 at p + w + A2/2
    stage_adjoint<P>(a, rec[2], a3, q, cc, acc);
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        pb[x] += q[x];
        wb[x] += q[x];
        a2[x] += R(0.5) * q[x];
    }
    // stage 2 at p + w/2 + A1/8
    stage_adjoint<P>(a, rec[1], a2, q, cc, acc);
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        pb[x] += q[x];
        wb[x] += R(0.5) * q[x];
        a1[x] += R(0.125) * q[x];
    }
    // stage 1 at p
    stage_adjoint<P>(a, rec[0], a1, q, cc, acc);
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        lp[x] = pb[x] + q[x];
        lw[x] = wb[x];
    }
}

// ---------------------------------------------------------------------------
// Detector projection and splat.
// ---------------------------------------------------------------------------

// Splat profile g(d) and its derivative dg/dd (d and s in pixels).
template <class R>
__device__ __forceinline__ R splat_g(R d, R s, R& dg) {
    const R u = fabs(d) / s;
    if (u >= R(4)) {
        dg = R(0);
        return R(0);
    }
    R e;
    if constexpr (sizeof(R) == 4) e = expf(R(-0.5) * u * u);
    else e = exp(R(-0.5) * u * u);
    R t = R(1), dt = R(0);
    if (u > R(3)) {
        const R x = u - R(3);
        t = R(1) - x * x * x * (R(10) + x * (R(-15) + x * R(6)));
        dt = R(-30) * x * x * (R(1) - x) * (R(1) - x);
    }
    // d/dd [e(u) t(u)] with u = |d|/s
    const R sgn = d < R(0) ? R(-1) : R(1);
    dg = (e * (-u * t + dt)) * sgn / s;
    return e * t;
}

// Detector coordinates (pixels) of a final state; false if the ray never
// meets the plane or is not finite.
template <class P>
__device__ __forceinline__ bool detector_point(const ImageArgs& a, const MState<P>& r, double& pa, double& pb,
                                               double& t, double (&p)[3], double (&w)[3]) {
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        p[x] = r.p[x].vald();
        w[x] = r.w[x].vald();
    }
    const double wa = a.axis == 0 ? w[0] : (a.axis == 1 ? w[1] : w[2]);
    const double pax = a.axis == 0 ? p[0] : (a.axis == 1 ? p[1] : p[2]);
    if (!(wa != 0.0)) return false;
    t = (a.plane - pax) / wa;
    const double X = p[a.t1] + t * w[a.t1];
    const double Y = p[a.t2] + t * w[a.t2];
    pa = a.px0[0] + a.px_per_cell[0] * X;
    pb = a.px0[1] + a.px_per_cell[1] * Y;
    return isfinite(pa) && isfinite(pb) && fabs(pa) < 1e9 && fabs(pb) < 1e9;
}

template <class P>
__device__ __forceinline__ void splat(const ImageArgs& a, double pa, double pb) {
    using R = typename P::R;
    const int i0 = (int)floor(pa - a.radius) + 1;
    const int j0 = (int)floor(pb - a.radius) + 1;
    const R s = (R)a.sigma;
    R gy[kMaxTaps];
    for (int j = 0; j < a.taps; ++j) {
        R dg;
        gy[j] = splat_g<R>((R)((double)(j0 + j) - pb), s, dg);
    }
    R* img = reinterpret_cast<R*>(a.image);
    for (int i = 0; i < a.taps; ++i) {
        const int ii = i0 + i;
        if (ii < 0 || ii >= a.npx[0]) continue;
        R dg;
        const R gx = splat_g<R>((R)((double)ii - pa), s, dg) * (R)a.norm;
        if (gx == R(0)) continue;
        for (int j = 0; j < a.taps; ++j) {
            const int jj = j0 + j;
            if (jj < 0 || jj >= a.npx[1] || gy[j] == R(0)) continue;
            atomicAdd(img + (size_t)ii * a.npx[1] + jj, gx * gy[j]);
        }
    }
}

// A CTA's splats, formed in shared memory and added to the image once per
// pixel. The rays of a CTA share their entry cell, so their windows overlap
// on the detector; adding each ray's taps to the image directly (17 x 17
// reductions per ray at sigma = 2) made the image's L2 atomics a third of the
// forward's time. Here the CTA takes the box of its rays' windows (clipped to
// the image). When a window fits in the kSplatTile x kSplatTile tile at the
// box's low corner, the ray's separable weights g(i - a) * norm (rows) and
// g(j - b) (columns) over the tile go to shared memory, kSplatRays rays at a
// time, and every thread sums ray products for four pixels of the tile:
// pixel (r, c) = sum over rays of row_weight(r) * column_weight(c), a small
// matrix product. Windows that do not fit are splatted directly. Every thread
// of the CTA calls this (it synchronises the CTA).
constexpr int kSplatTile = 32;     // pixels per side of a CTA's tile
constexpr int kSplatRays = 64;     // rays staged per round
constexpr int kSplatPitch = kSplatTile + 1;   // shared row pitch (conflict-free stores and loads)

template <class P>
__device__ __forceinline__ void splat_block(const ImageArgs& a, bool has, double pa, double pb) {
    using R = typename P::R;
    __shared__ R s_row[kSplatRays * kSplatPitch], s_col[kSplatRays * kSplatPitch];
    __shared__ int s_box[2];
    const int t = threadIdx.x;
    int i0 = 0, j0 = 0, r0 = 0, r1 = -1, c0 = 0, c1 = -1;
    if (has) {
        i0 = (int)floor(pa - a.radius) + 1;
        j0 = (int)floor(pb - a.radius) + 1;
        r0 = max(i0, 0);
        r1 = min(i0 + a.taps - 1, a.npx[0] - 1);
        c0 = max(j0, 0);
        c1 = min(j0 + a.taps - 1, a.npx[1] - 1);
    }
    const bool in = r0 <= r1 && c0 <= c1;
    if (t == 0) s_box[0] = s_box[1] = INT_MAX;
    __syncthreads();
    if (in) {
        atomicMin(&s_box[0], r0);
        atomicMin(&s_box[1], c0);
    }
    __syncthreads();
    const int br = s_box[0], bc = s_box[1];
    const bool tiled = in && r1 < br + kSplatTile && c1 < bc + kSplatTile;
    if (in && !tiled) splat<P>(a, pa, pb);
    if (!__syncthreads_or(tiled)) return;
    // this thread's four pixels: column c, rows r, r + 8, r + 16, r + 24
    const int c = t & (kSplatTile - 1), rb = t >> 5;
    static_assert(kAdjThreads == 256 && kSplatTile == 32, "four pixels per thread");
    R acc[4] = {R(0), R(0), R(0), R(0)};
    const R s = (R)a.sigma;
    for (int base = 0; base < (int)blockDim.x; base += kSplatRays) {
        if (t >= base && t < base + kSplatRays) {
            R* rw = s_row + (t - base) * kSplatPitch;
            R* cw = s_col + (t - base) * kSplatPitch;
            for (int k = 0; k < kSplatTile; ++k) {
                R g = R(0), dg;
                const int ii = br + k;
                if (tiled && ii >= r0 && ii <= r1) g = splat_g<R>((R)((double)ii - pa), s, dg) * (R)a.norm;
                rw[k] = g;
                R h = R(0);
                const int jj = bc + k;
                if (tiled && jj >= c0 && jj <= c1) h = splat_g<R>((R)((double)jj - pb), s, dg);
                cw[k] = h;
            }
        }
        __syncthreads();
#pragma unroll 4
        for (int u = 0; u < kSplatRays; ++u) {
            const R h = s_col[u * kSplatPitch + c];
#pragma unroll
            for (int q = 0; q < 4; ++q) acc[q] += s_row[u * kSplatPitch + rb + 8 * q] * h;
        }
        __syncthreads();
    }
    R* img = reinterpret_cast<R*>(a.image);
#pragma unroll
    for (int q = 0; q < 4; ++q) {
        const int ii = br + rb + 8 * q, jj = bc + c;
        if (acc[q] != R(0) && ii < a.npx[0] && jj < a.npx[1]) atomicAdd(img + (size_t)ii * a.npx[1] + jj, acc[q]);
    }
}

// d L / d(pixel coordinates) from the image gradient.
template <class P>
__device__ __forceinline__ void splat_adjoint(const ImageArgs& a, double pa, double pb, double& ga, double& gb) {
    using R = typename P::R;
    const int i0 = (int)floor(pa - a.radius) + 1;
    const int j0 = (int)floor(pb - a.radius) + 1;
    const R s = (R)a.sigma;
    R gy[kMaxTaps], dgy[kMaxTaps];
    for (int j = 0; j < a.taps; ++j) gy[j] = splat_g<R>((R)((double)(j0 + j) - pb), s, dgy[j]);
    const R* gi = reinterpret_cast<const R*>(a.image);
    R sa = R(0), sb = R(0);
    for (int i = 0; i < a.taps; ++i) {
        const int ii = i0 + i;
        if (ii < 0 || ii >= a.npx[0]) continue;
        R dgx;
        const R gx = splat_g<R>((R)((double)ii - pa), s, dgx);
        if (gx == R(0) && dgx == R(0)) continue;
        R r0 = R(0), r1 = R(0);
        for (int j = 0; j < a.taps; ++j) {
            const int jj = j0 + j;
            if (jj < 0 || jj >= a.npx[1]) continue;
            const R v = gi[(size_t)ii * a.npx[1] + jj];
            r0 += v * gy[j];
            r1 += v * dgy[j];
        }
        // d/da g(i - a) = -g'(i - a)
        sa -= dgx * r0;
        sb -= gx * r1;
    }
    ga = (double)sa * a.norm;
    gb = (double)sb * a.norm;
}

// The tracer's interior-step test on the model state: inside the grid, and
// the prediction p + w at least kFaceMargin inside on every axis. With every
// stage acceleration below kInteriorAccel, all four stage points of the step
// are then inside, and locate needs no grid test.
template <class P>
__device__ __forceinline__ bool model_interior(const ImageArgs& a, const MState<P>& r) {
    using R = typename P::R;
    const R margin = R(kFaceMargin);
    bool ok = true;
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        const R p = r.p[x].val(), pn = p + r.w[x].val(), lim = lim_of<R>(a.geo, x);
        ok = ok & (p >= R(0)) & (p <= lim) & (pn >= margin) & (pn <= lim - margin);
    }
    return ok;
}

// Steps after an interior step that are certainly interior too (31, 7 or 0),
// for accelerations bounded by B; the argument of the tracer's interior_run:
// j steps on, the position and the prediction lie within B (j^2 / 2 + j) of
// the segment from p + w to p + (j + 1) w.
template <class P>
__device__ __forceinline__ int model_interior_run(const ImageArgs& a, const MState<P>& r, float B) {
    using R = typename P::R;
    const R margin = R(kFaceMargin) + R(0.25);
    R p[3], w[3];
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        p[x] = r.p[x].val();
        w[x] = r.w[x].val();
    }
    auto fits = [&](int m) {
        const R dev = margin + R(B) * R(0.5 * m * m + m);
        bool ok = true;
#pragma unroll
        for (int x = 0; x < 3; ++x) {
            const R e1 = p[x] + w[x], e2 = p[x] + R(m + 1) * w[x];
            ok = ok & (fmin(e1, e2) >= dev) & (fmax(e1, e2) <= lim_of<R>(a.geo, x) - dev);
        }
        return ok;
    };
    if (fits(31)) return 31;
    if (fits(7)) return 7;
    return 0;
}

// The acceleration bound of the fast path: infinity (no fast path) without one.
__device__ __forceinline__ float load_accel_bound(const ImageArgs& a) {
    if (!a.accel_bound) return INFINITY;
    const float b = __uint_as_float(*a.accel_bound);
    return b * 1.001f;
}

// Largest |S_k dq/du_k| over the packed grid's gradient channels. Trilinear
// interpolation stays within its corners' range, so this bounds every stage
// acceleration of the model. Non-negative floats order as their bit
// patterns, so the blocks combine with an unsigned atomicMax; a NaN channel
// gives infinity (no fast path).
template <class P>
__global__ void __launch_bounds__(256) accel_bound_kernel(const void* __restrict__ grid, size_t nvox,
                                                          double s0, double s1, double s2, unsigned* out) {
    __shared__ float s_max[8];
    float m = 0.0f;
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < nvox; i += (size_t)gridDim.x * blockDim.x) {
        double g0, g1, g2;
        if constexpr (sizeof(typename P::R) == 4) {
            const float4 v = reinterpret_cast<const float4*>(grid)[i];
            g0 = v.y; g1 = v.z; g2 = v.w;
        } else {
            const double* d = reinterpret_cast<const double*>(grid) + 4 * i;
            g0 = d[1]; g1 = d[2]; g2 = d[3];
        }
        const double x = fmax(fabs(s0 * g0), fmax(fabs(s1 * g1), fabs(s2 * g2)));
        const bool nan = !(g0 == g0) || !(g1 == g1) || !(g2 == g2);
        const float xf = nan ? INFINITY : __double2float_ru(x);
        m = xf > m ? xf : m;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_down_sync(0xffffffffu, m, o));
    if ((threadIdx.x & 31) == 0) s_max[threadIdx.x >> 5] = m;
    __syncthreads();
    if (threadIdx.x == 0) {
        for (int wi = 1; wi < (int)(blockDim.x >> 5); ++wi) m = fmaxf(m, s_max[wi]);
        atomicMax(out, __float_as_uint(m));
    }
}

// ---------------------------------------------------------------------------
// Kernels.
// ---------------------------------------------------------------------------
template <class P>
__global__ void __launch_bounds__(kAdjThreads, adj_fwd_min_blocks<P>()) image_forward_kernel(const __grid_constant__ ImageArgs a) {
    using R = typename P::R;
    __shared__ unsigned long long s_steps;
    if (threadIdx.x == 0) s_steps = 0;
    __syncthreads();
    const long long slot = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    int t = 0;
    bool has = false;     // the ray meets the detector plane at (pa, pb) pixels
    double pa = 0.0, pb = 0.0;
    if (slot < a.n) {
        const unsigned id = a.perm[slot];
        const R* rays = reinterpret_cast<const R*>(a.rays);
        MState<P> r;
#pragma unroll
        for (int x = 0; x < 3; ++x) {
            r.p[x].set(((double)rays[x * a.n + id] - a.origin[x]) * a.inv_h[x]);
            r.w[x].set((double)rays[(3 + x) * a.n + id] * a.w_of_v[x]);
        }
        typename AdjTypes<P>::Cell cc;
        cc.base = kNone;
        const float B = load_accel_bound(a);
        const bool fast = B <= (float)kInteriorAccel;
        int run = 0, ck = 0, seg = 0;    // ck: steps to the next checkpoint
        for (; t < a.n_steps; ++t) {
            bool interior = false;
            if (run > 0) {
                // proven interior: inside, so not gone either
                --run;
                interior = true;
            } else {
                if (ray_gone_model<P>(a, r)) break;
                if (fast && model_interior<P>(a, r)) {
                    interior = true;
                    run = model_interior_run<P>(a, r, B);
                }
            }
            if (ck == 0) {
                store_state<P>(a, seg++, slot, r);
                ck = a.ckpt_every;
            }
            --ck;
            if (interior)
                model_step<P, true>(a, r, cc);
            else
                model_step<P>(a, r, cc);
        }
        store_state<P>(a, a.n_seg, slot, r);
        a.nsteps[slot] = t;
        double tt, p[3], w[3];
        has = detector_point<P>(a, r, pa, pb, tt, p, w);
    }
    splat_block<P>(a, has, pa, pb);
    block_add((unsigned long long)t, &s_steps, a.total_steps);
}

// In-cell coordinates of stage 1 and the first two of stage 2 of step j of
// the current segment into / out of the shared buffer (`buf` points at this
// thread's column).
template <class P>
__device__ __forceinline__ void put_step(typename P::R* buf, int j, const StageRec<P> (&rec)[3]) {
    typename P::R* b = buf + (size_t)j * kAdjStateWords * kAdjBwdThreads;
#pragma unroll
    for (int x = 0; x < 3; ++x) b[x * kAdjBwdThreads] = rec[0].f[x];
    b[3 * kAdjBwdThreads] = rec[1].f[0];
    b[4 * kAdjBwdThreads] = rec[1].f[1];
}

template <class P>
__device__ __forceinline__ void get_step(const typename P::R* buf, int j, StageRec<P> (&rec)[3]) {
    const typename P::R* b = buf + (size_t)j * kAdjStateWords * kAdjBwdThreads;
#pragma unroll
    for (int x = 0; x < 3; ++x) rec[0].f[x] = b[x * kAdjBwdThreads];
    rec[1].f[0] = b[3 * kAdjBwdThreads];
    rec[1].f[1] = b[4 * kAdjBwdThreads];
}

template <class P, int MINB>
__global__ void __launch_bounds__(kAdjBwdThreads, MINB) image_backward_kernel(const __grid_constant__ ImageArgs a) {
    using R = typename P::R;
    extern __shared__ __align__(16) unsigned char s_dyn[];
    R* s_seg = reinterpret_cast<R*>(s_dyn) + threadIdx.x;   // this thread's column of the segment buffer
    const long long slot = (long long)blockIdx.x * blockDim.x + threadIdx.x;
    if (slot >= a.n) return;
    MState<P> r;
    load_state<P>(a, a.n_seg, slot, r);
    double pa, pb, t, p[3], w[3];
    if (!detector_point<P>(a, r, pa, pb, t, p, w)) return;
    double ga, gb;
    splat_adjoint<P>(a, pa, pb, ga, gb);
    // projection X = p1 + t w1, Y = p2 + t w2, t = (plane - pa) / wa
    const double Xb = ga * a.px_per_cell[0], Yb = gb * a.px_per_cell[1];
    const double wa = a.axis == 0 ? w[0] : (a.axis == 1 ? w[1] : w[2]);
    const double tb = Xb * w[a.t1] + Yb * w[a.t2];
    double lpd[3] = {0.0, 0.0, 0.0}, lwd[3] = {0.0, 0.0, 0.0};
    lpd[a.t1] = Xb;
    lwd[a.t1] = Xb * t;
    lpd[a.t2] = Yb;
    lwd[a.t2] = Yb * t;
    lpd[a.axis] = -tb / wa;
    lwd[a.axis] = -tb * t / wa;
    R lp[3], lw[3];
#pragma unroll
    for (int x = 0; x < 3; ++x) {
        lp[x] = (R)lpd[x];
        lw[x] = (R)lwd[x];
    }
    if (lp[0] == R(0) && lp[1] == R(0) && lp[2] == R(0) && lw[0] == R(0) && lw[1] == R(0) && lw[2] == R(0))
        return;
    const int T = a.nsteps[slot];
    typename AdjTypes<P>::Cell cc;
    cc.base = kNone;
    typename AdjTypes<P>::Acc acc;
    acc.base = kNone;
    // the three stage cells and the in-cell coordinates that the shared
    // buffer does not hold (stage 2's third, stage 3's) of each step
    unsigned segB[kMaxCkptEvery][3];
    R segF[kMaxCkptEvery][4];
    for (int s = (T + a.ckpt_every - 1) / a.ckpt_every - 1; s >= 0; --s) {
        load_state<P>(a, s, slot, r);
        const int j0 = s * a.ckpt_every;
        const int m = min(a.ckpt_every, T - j0);
        // recompute the segment from its checkpoint (bitwise the forward's
        // steps), recording where each stage sampled, then run its adjoint
        // in reverse
        for (int j = 0; j < m; ++j) {
            StageRec<P> rec[3];
            model_step<P>(a, r, cc, rec);
            put_step<P>(s_seg, j, rec);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                segB[j][k] = rec[k].b;
                segF[j][k] = rec[2].f[k];
            }
            segF[j][3] = rec[1].f[2];
        }
        // segB / segF live in local memory, mostly in L2: step j - 1's
        // records are loaded while step j's adjoint runs
        unsigned Bn[3];
        R Fn[4];
#pragma unroll
        for (int k = 0; k < 3; ++k) Bn[k] = segB[m - 1][k];
#pragma unroll
        for (int k = 0; k < 4; ++k) Fn[k] = segF[m - 1][k];
        for (int j = m - 1; j >= 0; --j) {
            StageRec<P> rec[3];
            get_step<P>(s_seg, j, rec);
#pragma unroll
            for (int k = 0; k < 3; ++k) {
                rec[k].b = Bn[k];
                rec[2].f[k] = Fn[k];
            }
            rec[1].f[2] = Fn[3];
            const int jn = j > 0 ? j - 1 : 0;
#pragma unroll
            for (int k = 0; k < 3; ++k) Bn[k] = segB[jn][k];
#pragma unroll
            for (int k = 0; k < 4; ++k) Fn[k] = segF[jn][k];
            model_step_adjoint<P>(a, rec, lp, lw, cc, acc);
        }
    }
    flush(a, acc);
}

// d L / d ne from d L / d(packed grid): the transpose of K1's per-axis
// stencil (one-sided differences on the faces, central inside), times
// ne_scale. Gathers from the 6 neighbours; no atomics.
template <class P>
__device__ __forceinline__ void load_gg(const void* gg, size_t i, double (&v)[4]) {
    if constexpr (sizeof(typename P::R) == 4) {
        const float4 x = reinterpret_cast<const float4*>(gg)[i];
        v[0] = x.x; v[1] = x.y; v[2] = x.z; v[3] = x.w;
    } else {
        const double* d = reinterpret_cast<const double*>(gg) + 4 * i;
        v[0] = d[0]; v[1] = d[1]; v[2] = d[2]; v[3] = d[3];
    }
}

// Transpose of one axis' stencil at index j of n: sum over the differences
// D[i] that use q[j] of d D[i] / d q[j] * Dbar[i], where Dbar[i] is channel
// `ch` of the neighbour at offset (i - j) * stride.
template <class P>
__device__ __forceinline__ double stencil_t(const void* gg, size_t v, int j, int n, size_t stride, int ch) {
    double r = 0.0, x[4];
    if (j >= 1) {          // D[j-1] holds +q[j] with weight 1 (face j-1 == 0) or 1/2
        load_gg<P>(gg, v - stride, x);
        r += (j - 1 == 0 ? 1.0 : 0.5) * x[ch];
    }
    if (j <= n - 2) {      // D[j+1] holds -q[j] with weight 1 (face j+1 == n-1) or 1/2
        load_gg<P>(gg, v + stride, x);
        r -= (j + 1 == n - 1 ? 1.0 : 0.5) * x[ch];
    }
    if (j == 0 || j == n - 1) {   // the one-sided differences on the faces use q[j] itself
        load_gg<P>(gg, v, x);
        r += (j == 0 ? -1.0 : 1.0) * x[ch];
    }
    return r;
}

template <class P, class Out>
__global__ void __launch_bounds__(256) pack_adjoint_kernel(const void* __restrict__ gg, Out* __restrict__ out,
                                                           GridGeo g, double scale) {
  // x over k (coalesced), y over j, z over i, as the pack kernel
  for (int i = blockIdx.z; i < g.n[0]; i += gridDim.z)
    for (int j = blockIdx.y; j < g.n[1]; j += gridDim.y)
      for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < g.n[2]; k += gridDim.x * blockDim.x) {
        const size_t vi = ((size_t)i * g.n[1] + j) * g.n[2] + k;
        double self[4];
        load_gg<P>(gg, vi, self);
        double r = self[0];
        r += stencil_t<P>(gg, vi, i, g.n[0], g.sx, 1);
        r += stencil_t<P>(gg, vi, j, g.n[1], g.sy, 2);
        r += stencil_t<P>(gg, vi, k, g.n[2], 1, 3);
        out[vi] = (Out)(r * scale);
      }
}

// ---------------------------------------------------------------------------
// Host side.
// ---------------------------------------------------------------------------
static int image_n_seg(const SlothImageParams* p) { return (p->n_steps + p->ckpt_every - 1) / p->ckpt_every; }

static size_t image_ws_bytes(const SlothImageParams* p, long long n) {
    const size_t nn = (size_t)(n > 0 ? n : 1);
    return workspace_bytes(n) + align256((size_t)(image_n_seg(p) + 1) * 48u * nn) + align256(4u * nn);
}

static int check_image_params(const SlothGridDesc* g, const SlothImageParams* p, int64_t n) {
    int rc = check_grid(g);
    if (rc) return rc;
    if (!p) return SLOTH_ERR_NULL_POINTER;
    if (n < 0) return SLOTH_ERR_INVALID_ARGUMENT;
    if (n > 2147483647LL) return SLOTH_ERR_TOO_LARGE;
    if (p->reserved != 0 || !(p->dtau > 0.0) || !std::isfinite(p->dtau)) return SLOTH_ERR_INVALID_ARGUMENT;
    if (p->n_steps < 1 || p->n_steps > 1000000) return SLOTH_ERR_INVALID_ARGUMENT;
    if (p->ckpt_every < 1 || p->ckpt_every > kMaxCkptEvery) return SLOTH_ERR_INVALID_ARGUMENT;
    if (p->probing_axis < 0 || p->probing_axis > 2) return SLOTH_ERR_INVALID_ARGUMENT;
    if (p->n_px[0] < 1 || p->n_px[1] < 1 || p->n_px[0] > 16384 || p->n_px[1] > 16384) return SLOTH_ERR_INVALID_ARGUMENT;
    if (!(p->sigma_px > 0.0) || !(p->sigma_px <= 8.0)) return SLOTH_ERR_INVALID_ARGUMENT;
    if (!std::isfinite(p->plane)) return SLOTH_ERR_INVALID_ARGUMENT;
    for (int k = 0; k < 4; ++k)
        if (!std::isfinite(p->window[k])) return SLOTH_ERR_INVALID_ARGUMENT;
    if (!(p->window[1] > p->window[0]) || !(p->window[3] > p->window[2])) return SLOTH_ERR_INVALID_ARGUMENT;
    return SLOTH_OK;
}

static void fill_image_args(ImageArgs& a, const SlothGridDesc* g, const void* grid, const SlothImageParams* p,
                            const void* rays, long long n, const unsigned* perm, void* ckpt, int* nsteps) {
    a.geo = make_geo(g);
    a.grid = grid;
    a.rays = rays;
    a.n = n;
    a.perm = perm;
    for (int k = 0; k < 3; ++k) {
        const double h = g->spacing[k];
        a.origin[k] = g->origin[k];
        a.inv_h[k] = 1.0 / h;
        a.w_of_v[k] = (p->dtau / h) / kC;
        a.S[k] = -0.5 * (p->dtau / h) * (p->dtau / h);
        a.Sf[k] = (float)a.S[k];
    }
    a.n_steps = p->n_steps;
    a.ckpt_every = p->ckpt_every;
    a.n_seg = image_n_seg(p);
    a.axis = p->probing_axis;
    a.t1 = a.axis == 0 ? 1 : 0;
    a.t2 = a.axis == 2 ? 1 : 2;
    a.plane = (p->plane - g->origin[a.axis]) / g->spacing[a.axis];
    const int tr[2] = {a.t1, a.t2};
    for (int d = 0; d < 2; ++d) {
        const double lo = p->window[2 * d], hi = p->window[2 * d + 1];
        const double pix = (hi - lo) / p->n_px[d];
        a.px_per_cell[d] = g->spacing[tr[d]] / pix;
        a.px0[d] = (g->origin[tr[d]] - lo) / pix - 0.5;
        a.npx[d] = p->n_px[d];
    }
    a.sigma = p->sigma_px;
    a.radius = 4.0 * p->sigma_px;
    a.taps = 2 * (int)ceil(a.radius) + 1;
    a.norm = 1.0 / (2.0 * 3.141592653589793 * p->sigma_px * p->sigma_px);
    a.ckpt = ckpt;
    a.nsteps = nsteps;
    a.image = nullptr;
    a.ggrad = nullptr;
    a.total_steps = nullptr;
    a.accel_bound = nullptr;
}

struct ImageWs {
    unsigned *hist, *keys, *perm, *skeys;
    void* ckpt;
    int* nsteps;
    unsigned* bound;    // acceleration bound of the forward (float bits), in the header's second half
};

static ImageWs carve(void* ws, const SlothImageParams* p, long long n) {
    ImageWs w;
    char* base = reinterpret_cast<char*>(ws);
    const size_t a = align256((size_t)(n > 0 ? n : 1) * 4u);
    w.bound = reinterpret_cast<unsigned*>(base + kHeaderBytes / 2);
    w.hist = reinterpret_cast<unsigned*>(base + kHeaderBytes);
    w.keys = reinterpret_cast<unsigned*>(base + kHeaderBytes + kHistBytes);
    w.perm = reinterpret_cast<unsigned*>(base + kHeaderBytes + kHistBytes + a);
    w.skeys = reinterpret_cast<unsigned*>(base + kHeaderBytes + kHistBytes + 2 * a);
    char* c = base + workspace_bytes(n);
    w.ckpt = c;
    w.nsteps = reinterpret_cast<int*>(c + align256((size_t)(image_n_seg(p) + 1) * 48u * (size_t)(n > 0 ? n : 1)));
    return w;
}

// The acceleration bound of the interior fast path into the workspace.
template <class P>
static int launch_accel_bound(const SlothGridDesc* g, const void* grid, const ImageArgs& a, unsigned* bound, int sms,
                              cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(bound, 0, sizeof(unsigned), s);
    if (e != cudaSuccess) return cuda_status(e);
    const size_t vox = (size_t)g->n[0] * g->n[1] * g->n[2];
    const size_t want = (vox + 255) / 256, cap = (size_t)sms * 8;
    accel_bound_kernel<P><<<(unsigned)(want < cap ? want : cap), 256, 0, s>>>(grid, vox, fabs(a.S[0]), fabs(a.S[1]),
                                                                               fabs(a.S[2]), bound);
    note_launch();
    return cuda_status(cudaGetLastError());
}

template <class P>
static int image_forward_impl(const SlothGridDesc* g, const void* grid, const SlothImageParams* p,
                              const typename P::R* rays, int64_t n, typename P::R* image,
                              unsigned long long* total_steps, void* ws, size_t ws_bytes, void* stream) {
    int rc = check_image_params(g, p, n);
    if (rc) return rc;
    if (!grid || !image || !ws || (n > 0 && !rays)) return SLOTH_ERR_NULL_POINTER;
    if (((uintptr_t)grid & 15u) || ((uintptr_t)ws & 255u) || ((uintptr_t)image & (sizeof(typename P::R) - 1)) ||
        ((uintptr_t)rays & (sizeof(typename P::R) - 1)))
        return SLOTH_ERR_MISALIGNED;
    if (ws_bytes < image_ws_bytes(p, n)) return SLOTH_ERR_WORKSPACE_TOO_SMALL;
    int sms = 148;
    if ((rc = device_sm_count(&sms)) != SLOTH_OK) return rc;
    cudaStream_t s = (cudaStream_t)stream;
    cudaError_t e = cudaMemsetAsync(image, 0, sizeof(typename P::R) * (size_t)p->n_px[0] * p->n_px[1], s);
    if (e != cudaSuccess) return cuda_status(e);
    if (n == 0) return SLOTH_OK;
    ImageWs w = carve(ws, p, n);
    // One thread per ray in bucket order, with no tile sort: buckets of one
    // transverse entry cell each (for grids of up to 513 points across the
    // probing axis) keep a warp's rays in few cells, so that its cell loads
    // and gradient flushes share addresses.
    const int bbits = kMaxBucketBits;
    if ((e = cudaMemsetAsync(w.hist, 0, (size_t)4 << bbits, s)) != cudaSuccess) return cuda_status(e);
    rc = launch_prepass<typename P::R>(g, p->probing_axis, rays, n, bbits, w.keys, w.hist, w.perm, w.skeys, sms, s,
                                       true);
    if (rc) return rc;
    ImageArgs a;
    fill_image_args(a, g, grid, p, rays, n, w.perm, w.ckpt, w.nsteps);
    a.image = image;
    a.total_steps = total_steps;
    if ((rc = launch_accel_bound<P>(g, grid, a, w.bound, sms, s)) != SLOTH_OK) return rc;
    a.accel_bound = w.bound;
    image_forward_kernel<P><<<(unsigned)((n + kAdjThreads - 1) / kAdjThreads), kAdjThreads, 0, s>>>(a);
    note_launch();
    return cuda_status(cudaGetLastError());
}

template <class P>
static int image_backward_impl(const SlothGridDesc* g, const void* grid, const SlothImageParams* p, int64_t n,
                               const typename P::R* image_grad, void* grid_grad, void* ws, size_t ws_bytes,
                               void* stream) {
    int rc = check_image_params(g, p, n);
    if (rc) return rc;
    if (!grid || !image_grad || !grid_grad || !ws) return SLOTH_ERR_NULL_POINTER;
    if (((uintptr_t)grid & 15u) || ((uintptr_t)grid_grad & 15u) || ((uintptr_t)ws & 255u) ||
        ((uintptr_t)image_grad & (sizeof(typename P::R) - 1)))
        return SLOTH_ERR_MISALIGNED;
    if (ws_bytes < image_ws_bytes(p, n)) return SLOTH_ERR_WORKSPACE_TOO_SMALL;
    cudaStream_t s = (cudaStream_t)stream;
    const size_t vox = (size_t)g->n[0] * g->n[1] * g->n[2];
    cudaError_t e = cudaMemsetAsync(grid_grad, 0, vox * 4 * sizeof(typename P::R), s);
    if (e != cudaSuccess) return cuda_status(e);
    if (n == 0) return SLOTH_OK;
    ImageWs w = carve(ws, p, n);
    ImageArgs a;
    fill_image_args(a, g, grid, p, nullptr, n, w.perm, w.ckpt, w.nsteps);
    a.image = const_cast<typename P::R*>(image_grad);
    a.ggrad = grid_grad;
    const size_t smem = (size_t)p->ckpt_every * kAdjStateWords * sizeof(typename P::R) * kAdjBwdThreads;
    const unsigned blocks = (unsigned)((n + kAdjBwdThreads - 1) / kAdjBwdThreads);
    auto launch = [&](auto kernel) {
        cudaError_t err = cudaFuncSetAttribute(kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (err == cudaSuccess) kernel<<<blocks, kAdjBwdThreads, smem, s>>>(a);
        return err;
    };
    if constexpr (sizeof(typename P::R) == 4) {
        int dev = 0, per_sm = 0, reserved = 0;
        if ((e = cudaGetDevice(&dev)) != cudaSuccess ||
            (e = cudaDeviceGetAttribute(&per_sm, cudaDevAttrMaxSharedMemoryPerMultiprocessor, dev)) != cudaSuccess ||
            (e = cudaDeviceGetAttribute(&reserved, cudaDevAttrReservedSharedMemoryPerBlock, dev)) != cudaSuccess)
            return cuda_status(e);
        if (4 * (smem + (size_t)reserved) <= (size_t)per_sm)
            e = launch(image_backward_kernel<P, 4>);
        else
            e = launch(image_backward_kernel<P, 3>);
    } else {
        e = launch(image_backward_kernel<P, 1>);
    }
    if (e != cudaSuccess) return cuda_status(e);
    note_launch();
    return cuda_status(cudaGetLastError());
}

template <class P, class Out>
static int pack_adjoint_impl(const SlothGridDesc* g, const void* grid_grad, double ne_scale, Out* ne_grad,
                             void* stream) {
    int rc = check_grid(g);
    if (rc) return rc;
    if (!grid_grad || !ne_grad) return SLOTH_ERR_NULL_POINTER;
    if (!(ne_scale > 0.0) || !std::isfinite(ne_scale)) return SLOTH_ERR_INVALID_ARGUMENT;
    if (((uintptr_t)grid_grad & 15u) || ((uintptr_t)ne_grad & (sizeof(Out) - 1))) return SLOTH_ERR_MISALIGNED;
    int sms = 148;
    if ((rc = device_sm_count(&sms)) != SLOTH_OK) return rc;
    const dim3 grid((unsigned)((g->n[2] + 255) / 256), (unsigned)(g->n[1] < 65535 ? g->n[1] : 65535),
                    (unsigned)(g->n[0] < 65535 ? g->n[0] : 65535));
    pack_adjoint_kernel<P, Out><<<grid, 256, 0, (cudaStream_t)stream>>>(grid_grad, ne_grad, make_geo(g), ne_scale);
    note_launch();
    return cuda_status(cudaGetLastError());
}

}  // namespace sloth

extern "C" {

size_t sloth_image_workspace_bytes(const SlothImageParams* p, int64_t n) {
    if (!p || p->ckpt_every < 1 || p->n_steps < 1 || n < 0) return 0;
    return sloth::image_ws_bytes(p, n);
}

int sloth_image_forward_f32(const SlothGridDesc* g, const void* grid, const SlothImageParams* p, const float* rays,
                            int64_t n, float* image, unsigned long long* total_steps, void* ws, size_t ws_bytes,
                            void* stream) {
    return sloth::image_forward_impl<sloth::PolF32>(g, grid, p, rays, n, image, total_steps, ws, ws_bytes, stream);
}

int sloth_image_forward_f64(const SlothGridDesc* g, const void* grid, const SlothImageParams* p, const double* rays,
                            int64_t n, double* image, unsigned long long* total_steps, void* ws, size_t ws_bytes,
                            void* stream) {
    return sloth::image_forward_impl<sloth::PolF64>(g, grid, p, rays, n, image, total_steps, ws, ws_bytes, stream);
}

int sloth_image_backward_f32(const SlothGridDesc* g, const void* grid, const SlothImageParams* p, int64_t n,
                             const float* image_grad, void* grid_grad, void* ws, size_t ws_bytes, void* stream) {
    return sloth::image_backward_impl<sloth::PolF32>(g, grid, p, n, image_grad, grid_grad, ws, ws_bytes, stream);
}

int sloth_image_backward_f64(const SlothGridDesc* g, const void* grid, const SlothImageParams* p, int64_t n,
                             const double* image_grad, void* grid_grad, void* ws, size_t ws_bytes, void* stream) {
    return sloth::image_backward_impl<sloth::PolF64>(g, grid, p, n, image_grad, grid_grad, ws, ws_bytes, stream);
}

int sloth_grid_pack_adjoint_f32(const SlothGridDesc* g, const void* grid_grad, double ne_scale, float* ne_grad,
                                void* stream) {
    return sloth::pack_adjoint_impl<sloth::PolF32, float>(g, grid_grad, ne_scale, ne_grad, stream);
}

int sloth_grid_pack_adjoint_f64(const SlothGridDesc* g, const void* grid_grad, double ne_scale, double* ne_grad,
                                void* stream) {
    return sloth::pack_adjoint_impl<sloth::PolF64, double>(g, grid_grad, ne_scale, ne_grad, stream);
}

}  // extern "C"
