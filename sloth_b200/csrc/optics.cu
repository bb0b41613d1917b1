// Ray-transfer-matrix diagnostics: the reference's paraxial optics chain
// and detector histogram (src/processing/diagnostics.py:16-128, :176-268,
// :270-380) as one kernel over the Jones vectors a trace produced.
//
// Per ray (x, theta, y, phi), one thread:
//   1. optional lens-cutoff prefilter on the input (Diagnostic.__init__ with
//      prefilter_input, :223-231): keep sqrt((L tan theta + x)^2 +
//      (L tan phi + y)^2) <= R;
//   2. positions scaled (m_to_mm, :16-20: rows 0 and 2 times 1e3, rounded in
//      the input's precision as numpy does);
//   3. the optics in order, in FP64:
//        travel d    x = fma(d, theta, x), y = fma(d, phi, y)           (:47-61)
//        lens f1 f2  theta = (-1/f1)*x + theta, phi = (-1/f2)*y + phi   (:28-44)
//      each a 4x4 matrix product in the reference; np.matmul's BLAS sums a
//      row with fused multiply-adds in column order, which rounds travel
//      once and lens twice, as here. A NaN in any component makes all four
//      NaN. The stops set all four to NaN:
//        circular aperture R: x^2 + y^2 > R^2              (:63-71)
//        circular stop R:     x^2 + y^2 < R^2              (:73-81)
//        rectangular aperture: x^2 > Lx^2 AND y^2 > Ly^2   (:94-104, as written)
//        knife edge: x or y above (direction > 0) or below the offset (:106-123)
//        annular stop R1 R2: R1^2 < x^2 + y^2 < R2^2 (the helper at :83-92
//          only returns this mask; here it rejects);
//   4. optional CCD clip |x| <= hx, |y| <= hy (Diagnostic.histogram, :249-255);
//   5. the (weighted) histogram of (x, y) with numpy.histogram2d's bins
//      (:259, transposed: H[iy][ix]): edges linspace(lo, hi, n+1) computed
//      as numpy does (i*step + lo, last edge = hi), bin k holds
//      edges[k] <= v < edges[k+1], v == hi in the last bin, NaN and
//      out-of-range values dropped. Weights add with FP64 atomics.
#include <cmath>
#include <cstring>

#include "common.cuh"

namespace sloth {

struct OpticsArgs {
    const void* rays;
    long long n;
    const void* weights;
    SlothOptic op[SLOTH_MAX_OPTICS];
    double lens_c[SLOTH_MAX_OPTICS][2];   // -1/f1, -1/f2 for lens ops
    int n_ops;
    double pos_scale;
    int prefilter, ccd;
    double pre_L, pre_R, ccd_hx, ccd_hy;
    int nx, ny;
    double x0, x1, y0, y1, xstep, ystep;
    double* hist;
    double* rays_out;
    uint8_t* kept;
};

// numpy.linspace(lo, hi, n + 1)[i]
__device__ __forceinline__ double np_edge(int i, int n, double lo, double hi, double step) {
    return i < n ? __dadd_rn(__dmul_rn((double)i, step), lo) : hi;
}

// Bin of v in [lo, hi] with numpy.histogramdd's rule, or -1.
__device__ __forceinline__ int np_bin(double v, int n, double lo, double hi, double step) {
    if (!(v >= lo) || !(v <= hi)) return -1;
    if (v == hi) return n - 1;
    int k = (int)floor((v - lo) / step);
    k = min(max(k, 0), n - 1);
    // the estimate is within one bin of the answer; settle it on the edges
    for (int it = 0; it < 4 && k > 0 && v < np_edge(k, n, lo, hi, step); ++it) --k;
    for (int it = 0; it < 4 && k < n - 1 && v >= np_edge(k + 1, n, lo, hi, step); ++it) ++k;
    return k;
}

template <class T>
__global__ void __launch_bounds__(256) optics_kernel(const __grid_constant__ OpticsArgs a) {
    const T* rays = reinterpret_cast<const T*>(a.rays);
    const T* wts = reinterpret_cast<const T*>(a.weights);
    const double qnan = __longlong_as_double(0x7ff8000000000000LL);
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        const T rx = rays[i], rt = rays[a.n + i], ry = rays[2 * a.n + i], rp = rays[3 * a.n + i];
        bool keep = true;
        if (a.prefilter) {
            if constexpr (sizeof(T) == 4) {
                const float L = (float)a.pre_L;
                const float xp = __fadd_rn(__fmul_rn(L, tanf(rt)), rx);
                const float yp = __fadd_rn(__fmul_rn(L, tanf(rp)), ry);
                keep = sqrtf(__fadd_rn(__fmul_rn(xp, xp), __fmul_rn(yp, yp))) <= (float)a.pre_R;
            } else {
                const double xp = __dadd_rn(__dmul_rn(a.pre_L, tan(rt)), rx);
                const double yp = __dadd_rn(__dmul_rn(a.pre_L, tan(rp)), ry);
                keep = sqrt(__dadd_rn(__dmul_rn(xp, xp), __dmul_rn(yp, yp))) <= a.pre_R;
            }
        }
        if (a.kept) a.kept[i] = keep ? 1 : 0;
        double x, t, y, p;
        if (!keep) {
            x = t = y = p = qnan;
        } else {
            if constexpr (sizeof(T) == 4) {
                x = (double)__fmul_rn(rx, (float)a.pos_scale);
                y = (double)__fmul_rn(ry, (float)a.pos_scale);
            } else {
                x = __dmul_rn(rx, a.pos_scale);
                y = __dmul_rn(ry, a.pos_scale);
            }
            t = (double)rt;
            p = (double)rp;
            for (int k = 0; k < a.n_ops; ++k) {
                const SlothOptic& o = a.op[k];
                const bool anynan = isnan(x) || isnan(t) || isnan(y) || isnan(p);
                if (o.kind == SLOTH_OPTIC_TRAVEL || o.kind == SLOTH_OPTIC_LENS) {
                    if (anynan) {
                        x = t = y = p = qnan;
                    } else if (o.kind == SLOTH_OPTIC_TRAVEL) {
                        x = __fma_rn(o.a, t, x);
                        y = __fma_rn(o.a, p, y);
                    } else {
                        t = __dadd_rn(__dmul_rn(a.lens_c[k][0], x), t);
                        p = __dadd_rn(__dmul_rn(a.lens_c[k][1], y), p);
                    }
                    continue;
                }
                const double r2 = __dadd_rn(__dmul_rn(x, x), __dmul_rn(y, y));
                bool reject = false;
                switch (o.kind) {
                    case SLOTH_OPTIC_CIRCULAR_APERTURE: reject = r2 > __dmul_rn(o.a, o.a); break;
                    case SLOTH_OPTIC_CIRCULAR_STOP:     reject = r2 < __dmul_rn(o.a, o.a); break;
                    case SLOTH_OPTIC_RECT_APERTURE:
                        reject = (__dmul_rn(x, x) > __dmul_rn(o.a, o.a)) && (__dmul_rn(y, y) > __dmul_rn(o.b, o.b));
                        break;
                    case SLOTH_OPTIC_KNIFE_EDGE: {
                        const double v = o.axis == 0 ? x : y;
                        reject = o.b > 0.0 ? (v > o.a) : (v < o.a);
                        break;
                    }
                    case SLOTH_OPTIC_ANNULAR_STOP:
                        reject = (r2 > __dmul_rn(o.a, o.a)) && (r2 < __dmul_rn(o.b, o.b));
                        break;
                    default: break;
                }
                if (reject) x = t = y = p = qnan;
            }
        }
        if (a.rays_out) {
            a.rays_out[i] = x;
            a.rays_out[a.n + i] = t;
            a.rays_out[2 * a.n + i] = y;
            a.rays_out[3 * a.n + i] = p;
        }
        if (!a.hist || !keep || isnan(x) || isnan(y)) continue;
        if (a.ccd && !(fabs(x) <= a.ccd_hx && fabs(y) <= a.ccd_hy)) continue;
        const int ix = np_bin(x, a.nx, a.x0, a.x1, a.xstep);
        const int iy = np_bin(y, a.ny, a.y0, a.y1, a.ystep);
        if (ix < 0 || iy < 0) continue;
        const double w = wts ? (double)wts[i] : 1.0;
        atomicAdd(a.hist + (size_t)iy * a.nx + ix, w);
    }
}

template <class T>
static int optics_impl(const T* rays, int64_t n, const T* weights, const SlothOptic* optics, int32_t n_optics,
                       const SlothDetectorParams* d, double* hist, double* rays_out, uint8_t* kept, void* stream) {
    if (!d) return SLOTH_ERR_NULL_POINTER;
    if (n < 0 || n_optics < 0 || n_optics > SLOTH_MAX_OPTICS || d->reserved != 0) return SLOTH_ERR_INVALID_ARGUMENT;
    if (n > ((int64_t)1 << 40)) return SLOTH_ERR_TOO_LARGE;
    if (n_optics > 0 && !optics) return SLOTH_ERR_NULL_POINTER;
    if (!std::isfinite(d->pos_scale) || d->pos_scale == 0.0) return SLOTH_ERR_INVALID_ARGUMENT;
    if (d->prefilter && (!std::isfinite(d->prefilter_L) || !std::isfinite(d->prefilter_R)))
        return SLOTH_ERR_INVALID_ARGUMENT;
    if (d->ccd_clip && (!(d->ccd_half[0] >= 0.0) || !(d->ccd_half[1] >= 0.0))) return SLOTH_ERR_INVALID_ARGUMENT;
    if (hist) {
        if (d->nx < 1 || d->ny < 1 || d->nx > 65536 || d->ny > 65536) return SLOTH_ERR_INVALID_ARGUMENT;
        if (!std::isfinite(d->x_range[0]) || !std::isfinite(d->x_range[1]) || !std::isfinite(d->y_range[0]) ||
            !std::isfinite(d->y_range[1]) || !(d->x_range[1] > d->x_range[0]) || !(d->y_range[1] > d->y_range[0]))
            return SLOTH_ERR_INVALID_ARGUMENT;
    }
    OpticsArgs a;
    memset(&a, 0, sizeof(a));
    for (int k = 0; k < n_optics; ++k) {
        const SlothOptic& o = optics[k];
        if (!std::isfinite(o.a) || !std::isfinite(o.b)) return SLOTH_ERR_INVALID_ARGUMENT;
        switch (o.kind) {
            case SLOTH_OPTIC_TRAVEL: break;
            case SLOTH_OPTIC_LENS:
                if (o.a == 0.0 || o.b == 0.0) return SLOTH_ERR_INVALID_ARGUMENT;
                a.lens_c[k][0] = -1.0 / o.a;
                a.lens_c[k][1] = -1.0 / o.b;
                break;
            case SLOTH_OPTIC_CIRCULAR_APERTURE:
            case SLOTH_OPTIC_CIRCULAR_STOP:
            case SLOTH_OPTIC_RECT_APERTURE:
            case SLOTH_OPTIC_ANNULAR_STOP: break;
            case SLOTH_OPTIC_KNIFE_EDGE:
                if ((o.axis != 0 && o.axis != 2) || o.b == 0.0) return SLOTH_ERR_INVALID_ARGUMENT;
                break;
            default: return SLOTH_ERR_INVALID_ARGUMENT;
        }
        a.op[k] = o;
    }
    if (n == 0) return SLOTH_OK;
    if (!rays) return SLOTH_ERR_NULL_POINTER;
    const uintptr_t al = sizeof(T) - 1;
    if (((uintptr_t)rays & al) || ((uintptr_t)weights & al) || ((uintptr_t)hist & 7u) || ((uintptr_t)rays_out & 7u))
        return SLOTH_ERR_MISALIGNED;
    int sms = 148;
    int rc = device_sm_count(&sms);
    if (rc) return rc;
    a.rays = rays;
    a.n = n;
    a.weights = weights;
    a.n_ops = n_optics;
    a.pos_scale = d->pos_scale;
    a.prefilter = d->prefilter ? 1 : 0;
    a.ccd = d->ccd_clip ? 1 : 0;
    a.pre_L = d->prefilter_L;
    a.pre_R = d->prefilter_R;
    a.ccd_hx = d->ccd_half[0];
    a.ccd_hy = d->ccd_half[1];
    a.nx = d->nx;
    a.ny = d->ny;
    a.x0 = d->x_range[0];
    a.x1 = d->x_range[1];
    a.y0 = d->y_range[0];
    a.y1 = d->y_range[1];
    a.xstep = hist ? (a.x1 - a.x0) / a.nx : 1.0;
    a.ystep = hist ? (a.y1 - a.y0) / a.ny : 1.0;
    a.hist = hist;
    a.rays_out = rays_out;
    a.kept = kept;
    long long blocks = (n + 255) / 256;
    if (blocks > (long long)sms * 8) blocks = (long long)sms * 8;
    optics_kernel<T><<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(a);
    note_launch();
    return cuda_status(cudaGetLastError());
}

}  // namespace sloth

extern "C" {

int sloth_optics_f32(const float* rays, int64_t n, const float* weights, const SlothOptic* optics, int32_t n_optics,
                     const SlothDetectorParams* d, double* hist, double* rays_out, uint8_t* kept, void* stream) {
    return sloth::optics_impl<float>(rays, n, weights, optics, n_optics, d, hist, rays_out, kept, stream);
}

int sloth_optics_f64(const double* rays, int64_t n, const double* weights, const SlothOptic* optics,
                     int32_t n_optics, const SlothDetectorParams* d, double* hist, double* rays_out, uint8_t* kept,
                     void* stream) {
    return sloth::optics_impl<double>(rays, n, weights, optics, n_optics, d, hist, rays_out, kept, stream);
}

}  // extern "C"
