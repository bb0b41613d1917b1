// Shared device code of the sloth_b200 library (sm_100a).
//
// Grid layout: one 16-byte voxel per grid point holding
//   (c0, dq/du, dq/dv, dq/dw),  q = ne/nc,  d/du = derivative per grid cell,
// in C order (z fastest), with c0 = q (the value layout) or c0 = n - 1, the
// plasma refractive index minus one (the trace layout the tracers read). The
// FP64 port stores the same four values as two double2 (32 bytes per voxel).
//
// Ray coordinates inside the tracers are in grid cells (p = (x - x0)/h) and
// the velocity in cells per step (w = (v/c) * dtau / h), so one integration step is a
// unit step and dw/dstep = S * dq/du with S = -(dtau/h)^2 / 2.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include "../../include/sloth_b200.h"

namespace sloth {

constexpr double kC = 299792458.0;          // speed of light (scipy.constants.c)
constexpr int kTile = 1024;                 // rays per shared-memory sorted tile
constexpr int kSmallTile = 256;             // rays per tile at the end of a trace's tile queue
#ifndef SLOTH_TAIL_WAVES
#define SLOTH_TAIL_WAVES 32
#endif
constexpr int kTailWaves = SLOTH_TAIL_WAVES;  // small tiles per CTA at the end of the queue
constexpr int kMaxBucketBits = 18;          // at most 2^18 Morton buckets

// Count of kernels launched by this library (defined in capi.cu).
void note_launch();

// ---------------------------------------------------------------------------
// Morton keys: transverse 2-D Morton code of the entry cell in the high 20
// bits, cell index along the probing axis in the low 10 bits.
// ---------------------------------------------------------------------------
__host__ __device__ inline unsigned spread_bits10(unsigned v) {
    v &= 0x3FFu;
    v = (v | (v << 8)) & 0x00FF00FFu;
    v = (v | (v << 4)) & 0x0F0F0F0Fu;
    v = (v | (v << 2)) & 0x33333333u;
    v = (v | (v << 1)) & 0x55555555u;
    return v;
}

__host__ __device__ inline unsigned morton_key(unsigned c1, unsigned c2, unsigned ca) {
    return (((spread_bits10(c1) << 1) | spread_bits10(c2)) << 10) | (ca & 0x3FFu);
}

// ---------------------------------------------------------------------------
// Precision policies.
// ---------------------------------------------------------------------------

// FP32 sum carried with a Kahan compensation term: the value is s + c, c
// holding the rounding error lost by the running sum. Used for positions,
// velocities and the optical depth so that ~10^3 small increments onto an
// O(1..10^3) running value keep FP64-like accuracy without FP64 arithmetic.
struct AccF {
    float s, c;
    __device__ __forceinline__ void set(double v) {
        s = (float)v;
        c = (float)(v - (double)s);
    }
    __device__ __forceinline__ void add(float x) {
        const float y = x + c;
        const float t = s + y;
        c = y - (t - s);
        s = t;
    }
    // add(a * b) with the product's rounding folded into the compensated add
    __device__ __forceinline__ void add_fma(float a, float b) {
        const float y = __fmaf_rn(a, b, c);
        const float t = s + y;
        c = y - (t - s);
        s = t;
    }
    __device__ __forceinline__ float val() const { return s + c; }
    __device__ __forceinline__ double vald() const { return (double)s + (double)c; }
    __device__ __forceinline__ float hi() const { return s; }
    __device__ __forceinline__ float lo() const { return c; }
};

struct AccD {
    double s;
    __device__ __forceinline__ void set(double v) { s = v; }
    __device__ __forceinline__ void add(double y) { s += y; }
    __device__ __forceinline__ double val() const { return s; }
    __device__ __forceinline__ double vald() const { return s; }
    __device__ __forceinline__ double hi() const { return s; }
    __device__ __forceinline__ double lo() const { return 0.0; }
};

struct Vox4F { float x, y, z, w; };
struct Vox4D { double x, y, z, w; };

#ifndef SLOTH_CELL_CACHE_F32
#define SLOTH_CELL_CACHE_F32 1
#endif
#ifndef SLOTH_CELL_CACHE_F64
#define SLOTH_CELL_CACHE_F64 1
#endif
#ifndef SLOTH_CELL_POLY_F32
#define SLOTH_CELL_POLY_F32 1
#endif
#ifndef SLOTH_CELL_POLY_F64
#define SLOTH_CELL_POLY_F64 0
#endif

struct PolF32 {
    using R = float;
    using V = Vox4F;
    using Acc = AccF;
    // keep the last cell's 8 corners in registers across stages and steps
    static constexpr bool cell_cache = SLOTH_CELL_CACHE_F32 != 0;
    // keep the cached cell as trilinear polynomial coefficients (7 FMAs per
    // channel per sample instead of 8 products and an 8-term sum)
    static constexpr bool cell_poly = SLOTH_CELL_POLY_F32 != 0;
    __device__ __forceinline__ static V load(const void* g, unsigned i) {
        const float4 v = __ldg(reinterpret_cast<const float4*>(g) + i);
        return V{v.x, v.y, v.z, v.w};
    }
    __device__ __forceinline__ static float log_(float x) { return __logf(x); }
};

struct PolF64 {
    using R = double;
    using V = Vox4D;
    using Acc = AccD;
    static constexpr bool cell_cache = SLOTH_CELL_CACHE_F64 != 0;
    static constexpr bool cell_poly = SLOTH_CELL_POLY_F64 != 0;
    __device__ __forceinline__ static V load(const void* g, unsigned i) {
        const double2* p = reinterpret_cast<const double2*>(g) + 2u * (size_t)i;
        const double2 a = __ldg(p), b = __ldg(p + 1);
        return V{a.x, a.y, b.x, b.y};
    }
    __device__ __forceinline__ static double log_(double x) { return log(x); }
};

// Geometry of the packed grid as the samplers see it.
struct GridGeo {
    int n[3];
    unsigned sx, sy;       // voxel strides of axes 0 and 1 (axis 2 stride is 1)
    float limf[3];         // n - 1 per axis (float)
    double limd[3];        // n - 1 per axis (double)
};

template <class R> __device__ __forceinline__ R lim_of(const GridGeo& g, int a);
template <> __device__ __forceinline__ float lim_of<float>(const GridGeo& g, int a) { return g.limf[a]; }
template <> __device__ __forceinline__ double lim_of<double>(const GridGeo& g, int a) { return g.limd[a]; }

// Trilinear sample of the packed grid at p (grid cells). Follows the
// reference interpolator (src/core/interpolator.py:79-104): cell index
// i = floor(p) clamped to [0, n-2], weight t = p - i, product weights over
// the 8 corners, and fill 0 when p < 0 or p > n-1 on any axis (NaN counts as
// outside). Returns false (and zeros) outside.
template <class P>
__device__ __forceinline__ bool sample(const void* __restrict__ grid, const GridGeo& g,
                                       typename P::R px, typename P::R py, typename P::R pz,
                                       typename P::V& out) {
    using R = typename P::R;
    const bool in = (px >= R(0)) & (px <= lim_of<R>(g, 0)) & (py >= R(0)) &
                    (py <= lim_of<R>(g, 1)) & (pz >= R(0)) & (pz <= lim_of<R>(g, 2));
    if (!in) {
        out = typename P::V{R(0), R(0), R(0), R(0)};
        return false;
    }
    const int ix = min((int)px, g.n[0] - 2);
    const int iy = min((int)py, g.n[1] - 2);
    const int iz = min((int)pz, g.n[2] - 2);
    const R fx = px - (R)ix, fy = py - (R)iy, fz = pz - (R)iz;
    const unsigned b = (unsigned)ix * g.sx + (unsigned)iy * g.sy + (unsigned)iz;
    const typename P::V c000 = P::load(grid, b);
    const typename P::V c001 = P::load(grid, b + 1u);
    const typename P::V c010 = P::load(grid, b + g.sy);
    const typename P::V c011 = P::load(grid, b + g.sy + 1u);
    const typename P::V c100 = P::load(grid, b + g.sx);
    const typename P::V c101 = P::load(grid, b + g.sx + 1u);
    const typename P::V c110 = P::load(grid, b + g.sx + g.sy);
    const typename P::V c111 = P::load(grid, b + g.sx + g.sy + 1u);
    const R ex = R(1) - fx, ey = R(1) - fy, ez = R(1) - fz;
    const R w00 = ex * ey, w01 = ex * fy, w10 = fx * ey, w11 = fx * fy;
    const R w000 = w00 * ez, w001 = w00 * fz, w010 = w01 * ez, w011 = w01 * fz;
    const R w100 = w10 * ez, w101 = w10 * fz, w110 = w11 * ez, w111 = w11 * fz;
#define SLOTH_TRI(ch)                                                                  \
    (c000.ch * w000 + c001.ch * w001 + c010.ch * w010 + c011.ch * w011 + c100.ch * w100 + \
     c101.ch * w101 + c110.ch * w110 + c111.ch * w111)
    out.x = SLOTH_TRI(x);
    out.y = SLOTH_TRI(y);
    out.z = SLOTH_TRI(z);
    out.w = SLOTH_TRI(w);
#undef SLOTH_TRI
    return true;
}

// Host helpers shared by the translation units.
int check_grid(const SlothGridDesc* g);
GridGeo make_geo(const SlothGridDesc* g);
int cuda_status(cudaError_t e);
int device_sm_count(int* sms);

}  // namespace sloth
