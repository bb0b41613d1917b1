// K1 grid pack and K0 trilinear sample.
//
// K1 follows precompute_gradients (src/core/propagator.py:72-93): the driving
// term is proportional to ne, and its gradient is taken with jnp.gradient
// semantics along each axis (second-order central differences inside,
// first-order one-sided differences on the two faces). Here the gradient is
// kept per grid cell and normalised to the critical density, q = ne/nc; the
// tracers fold the -c^2/2 and 1/h^2 factors into one per-axis constant.
// Channel 0 holds q itself (the value layout, read by the K0 sampler and the
// detector-image model) or, in the trace layout, the refractive index minus
// one, n - 1 = sqrt(1 - x) - 1 with x = (omega_pe/omega)^2 = ope_ratio2 * q,
// which the tracers interpolate for the optical phase as the legacy solver
// interpolates its n grid (src/legacy/full_solver.py:289, :292-296, :342-345).
// It is evaluated as -x / (1 + sqrt(1 - x)), free of cancellation, and is -x
// above the critical density (where the legacy n is not real).
// All arithmetic is FP64; the FP32 grid rounds the final values once.
#include "common.cuh"

namespace sloth {

// q = ne * scale, rounded on its own (__dmul_rn keeps the compiler from
// fusing it into the differences below, so the result is bit-identical to a
// plain IEEE evaluation of the same formula).
template <class In>
__device__ __forceinline__ double qat(const In* __restrict__ ne, size_t i, double scale) {
    return __dmul_rn((double)__ldg(ne + i), scale);
}

// Launch shape: x over k (contiguous, coalesced), y over j, z over i, each
// axis strided when the grid has more points than the launch dimension; no
// index arithmetic beyond a multiply-add per voxel.
// n - 1 of x = ope2 * q, every operation rounded on its own (no fused
// multiply-add), so that it equals a plain IEEE evaluation of the formula.
__device__ __forceinline__ double n_minus_1_of(double q, double ope2) {
    const double x = __dmul_rn(ope2, q);
    const double om = fmax(__dsub_rn(1.0, x), 0.0);
    return -__ddiv_rn(x, __dadd_rn(1.0, __dsqrt_rn(om)));
}

template <class In, bool F64OUT, bool NM1>
__global__ void __launch_bounds__(256) pack_kernel(const In* __restrict__ ne, void* __restrict__ out,
                                                   GridGeo g, double scale, double ope2) {
  for (int i = blockIdx.z; i < g.n[0]; i += gridDim.z)
    for (int j = blockIdx.y; j < g.n[1]; j += gridDim.y)
      for (int k = blockIdx.x * blockDim.x + threadIdx.x; k < g.n[2]; k += gridDim.x * blockDim.x) {
        const size_t vi = ((size_t)i * g.n[1] + j) * g.n[2] + k;
        const double q = qat(ne, vi, scale);
        double d0, d1, d2;
        if (i == 0)               d0 = qat(ne, vi + g.sx, scale) - q;
        else if (i == g.n[0] - 1) d0 = q - qat(ne, vi - g.sx, scale);
        else                      d0 = 0.5 * (qat(ne, vi + g.sx, scale) - qat(ne, vi - g.sx, scale));
        if (j == 0)               d1 = qat(ne, vi + g.sy, scale) - q;
        else if (j == g.n[1] - 1) d1 = q - qat(ne, vi - g.sy, scale);
        else                      d1 = 0.5 * (qat(ne, vi + g.sy, scale) - qat(ne, vi - g.sy, scale));
        if (k == 0)               d2 = qat(ne, vi + 1, scale) - q;
        else if (k == g.n[2] - 1) d2 = q - qat(ne, vi - 1, scale);
        else                      d2 = 0.5 * (qat(ne, vi + 1, scale) - qat(ne, vi - 1, scale));
        const double c0 = NM1 ? n_minus_1_of(q, ope2) : q;
        if (F64OUT) {
            double2* o = reinterpret_cast<double2*>(out) + 2 * vi;
            o[0] = make_double2(c0, d0);
            o[1] = make_double2(d1, d2);
        } else {
            reinterpret_cast<float4*>(out)[vi] = make_float4((float)c0, (float)d0, (float)d1, (float)d2);
        }
      }
}

// Launch shape of the grid-wide voxel kernels (pack, pack adjoint).
inline dim3 voxel_grid(const SlothGridDesc* gd) {
    return dim3((unsigned)((gd->n[2] + 255) / 256), (unsigned)(gd->n[1] < 65535 ? gd->n[1] : 65535),
                (unsigned)(gd->n[0] < 65535 ? gd->n[0] : 65535));
}

template <class P>
__global__ void __launch_bounds__(256) sample_kernel(const void* __restrict__ grid, GridGeo g,
                                                     double o0, double o1, double o2,
                                                     double ih0, double ih1, double ih2,
                                                     const double* __restrict__ pts, long long n,
                                                     typename P::R* __restrict__ out) {
    using R = typename P::R;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const R px = (R)((pts[i] - o0) * ih0);
        const R py = (R)((pts[n + i] - o1) * ih1);
        const R pz = (R)((pts[2 * n + i] - o2) * ih2);
        typename P::V v;
        sample<P>(grid, g, px, py, pz, v);
        out[i] = v.x;
        out[n + i] = v.y;
        out[2 * n + i] = v.z;
        out[3 * n + i] = v.w;
    }
}

static int grid_blocks(long long work, int per_sm) {
    int sms = 148;
    if (device_sm_count(&sms) != SLOTH_OK) sms = 148;
    long long b = (work + 255) / 256;
    long long cap = (long long)sms * per_sm;
    if (b > cap) b = cap;
    if (b < 1) b = 1;
    return (int)b;
}

template <bool F64OUT, bool NM1>
static int pack_impl(const SlothGridDesc* g, const void* ne, int ne_is_f64, double ne_scale, double ope2,
                     void* grid_out, void* stream) {
    int rc = check_grid(g);
    if (rc) return rc;
    if (!ne || !grid_out) return SLOTH_ERR_NULL_POINTER;
    if (!(ne_scale > 0.0) || !std::isfinite(ne_scale)) return SLOTH_ERR_INVALID_ARGUMENT;
    if (NM1 && (!(ope2 > 0.0) || !std::isfinite(ope2))) return SLOTH_ERR_INVALID_ARGUMENT;
    if (((uintptr_t)grid_out & 15u) != 0) return SLOTH_ERR_MISALIGNED;
    if (((uintptr_t)ne & (ne_is_f64 ? 7u : 3u)) != 0) return SLOTH_ERR_MISALIGNED;
    const GridGeo geo = make_geo(g);
    const long long total = (long long)g->n[0] * g->n[1] * g->n[2];
    cudaStream_t s = (cudaStream_t)stream;
    (void)total;
    const dim3 grid = voxel_grid(g);
    if (ne_is_f64)
        pack_kernel<double, F64OUT, NM1><<<grid, 256, 0, s>>>((const double*)ne, grid_out, geo, ne_scale, ope2);
    else
        pack_kernel<float, F64OUT, NM1><<<grid, 256, 0, s>>>((const float*)ne, grid_out, geo, ne_scale, ope2);
    note_launch();
    return cuda_status(cudaGetLastError());
}

template <class P>
static int sample_impl(const SlothGridDesc* g, const void* grid, const double* points, int64_t n,
                       typename P::R* out, void* stream) {
    int rc = check_grid(g);
    if (rc) return rc;
    if (n < 0) return SLOTH_ERR_INVALID_ARGUMENT;
    if (n == 0) return SLOTH_OK;
    if (!grid || !points || !out) return SLOTH_ERR_NULL_POINTER;
    if (((uintptr_t)grid & 15u) != 0) return SLOTH_ERR_MISALIGNED;
    const GridGeo geo = make_geo(g);
    cudaStream_t s = (cudaStream_t)stream;
    sample_kernel<P><<<grid_blocks(n, 8), 256, 0, s>>>(
        grid, geo, g->origin[0], g->origin[1], g->origin[2], 1.0 / g->spacing[0], 1.0 / g->spacing[1],
        1.0 / g->spacing[2], points, (long long)n, out);
    note_launch();
    return cuda_status(cudaGetLastError());
}

}  // namespace sloth

extern "C" {

size_t sloth_grid_bytes(const SlothGridDesc* g, int real_bytes) {
    if (sloth::check_grid(g) != SLOTH_OK) return 0;
    if (real_bytes != 4 && real_bytes != 8) return 0;
    return (size_t)g->n[0] * (size_t)g->n[1] * (size_t)g->n[2] * 4u * (size_t)real_bytes;
}

int sloth_grid_pack_f32(const SlothGridDesc* g, const void* ne, int ne_is_f64, double ne_scale,
                        void* grid_out, void* stream) {
    return sloth::pack_impl<false, false>(g, ne, ne_is_f64, ne_scale, 0.0, grid_out, stream);
}

int sloth_grid_pack_f64(const SlothGridDesc* g, const void* ne, int ne_is_f64, double ne_scale,
                        void* grid_out, void* stream) {
    return sloth::pack_impl<true, false>(g, ne, ne_is_f64, ne_scale, 0.0, grid_out, stream);
}

int sloth_grid_pack_trace_f32(const SlothGridDesc* g, const void* ne, int ne_is_f64, double ne_scale,
                              double ope_ratio2, void* grid_out, void* stream) {
    return sloth::pack_impl<false, true>(g, ne, ne_is_f64, ne_scale, ope_ratio2, grid_out, stream);
}

int sloth_grid_pack_trace_f64(const SlothGridDesc* g, const void* ne, int ne_is_f64, double ne_scale,
                              double ope_ratio2, void* grid_out, void* stream) {
    return sloth::pack_impl<true, true>(g, ne, ne_is_f64, ne_scale, ope_ratio2, grid_out, stream);
}

int sloth_sample_f32(const SlothGridDesc* g, const void* grid, const double* points, int64_t n,
                     float* out, void* stream) {
    return sloth::sample_impl<sloth::PolF32>(g, grid, points, n, out, stream);
}

int sloth_sample_f64(const SlothGridDesc* g, const void* grid, const double* points, int64_t n,
                     double* out, void* stream) {
    return sloth::sample_impl<sloth::PolF64>(g, grid, points, n, out, stream);
}

}  // extern "C"
