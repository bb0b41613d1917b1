// K7: probing-beam rays generated on the device.
//
// The ray layout and distributions of the reference's Beam.init_beam
// (src/core/beam.py:57-346): rays start on the plane probing_axis =
// ne_extent at speed c, with
//   circular     : radius size * sqrt(U) (numpy's power(2)), angle 2 pi U;
//   square       : (size * (2U - 1), size * (2U - 1));
//   rectangular / rect_trackers : (size0 * (2U - 1), size1 * (2U - 1));
//   linear       : (size * (2U - 1), 0), velocity in the (axis-0, axis-2)
//                  plane as in the host mirror;
// and the direction at polar angle chi = divergence * N(0, 1) from the
// probing axis, azimuth phi = pi U, with the reference's component order
// per probing direction (:115-145).
//
// The random numbers are NOT the reference's numpy RandomState stream: each
// draw k of ray `id` is a SplitMix64 hash of (seed, id, k), so ray id's
// values depend only on the seed and id. A batch or a rank generates rays
// [first_id, first_id + n) of the same beam, and the result is the same for
// any split. Normal draws use the Box-Muller transform of two such uniforms.
// Trigonometry is FP64; the _f32 entry point rounds the rays once.
#include <cmath>

#include "common.cuh"

namespace sloth {

__host__ __device__ __forceinline__ uint64_t splitmix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

// Uniform double in [0, 1) of draw k of ray id.
__device__ __forceinline__ double beam_uniform(uint64_t seed, uint64_t id, int k) {
    const uint64_t h = splitmix64(seed * 0x9e3779b97f4a7c15ULL + splitmix64(id * 8ULL + (uint64_t)k + 1ULL));
    return (double)(h >> 11) * 0x1.0p-53;
}

struct BeamArgs {
    int type, axis;
    double size0, size1, divergence, extent;
    uint64_t seed, first_id;
    long long n;
    void* out;
};

template <class T>
__global__ void __launch_bounds__(256) beam_kernel(const BeamArgs a) {
    T* s0 = reinterpret_cast<T*>(a.out);
    const double kPi = 3.141592653589793;
    const long long stride = (long long)gridDim.x * blockDim.x;
    for (long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x; i < a.n; i += stride) {
        const uint64_t id = a.first_id + (uint64_t)i;
        // draws: 0, 1 position; 2 azimuth; 3, 4 the normal for the polar angle
        const double u0 = beam_uniform(a.seed, id, 0), u1 = beam_uniform(a.seed, id, 1);
        const double u2 = beam_uniform(a.seed, id, 2), u3 = beam_uniform(a.seed, id, 3);
        const double u4 = beam_uniform(a.seed, id, 4);
        const double gauss = sqrt(-2.0 * log(1.0 - u3)) * cos(2.0 * kPi * u4);
        const double chi = a.divergence * gauss;
        double pa, pb, phi;
        if (a.type == SLOTH_BEAM_CIRCULAR) {
            const double t = 2.0 * kPi * u0, r = a.size0 * sqrt(u1);
            pa = r * cos(t);
            pb = r * sin(t);
        } else if (a.type == SLOTH_BEAM_LINEAR) {
            pa = a.size0 * (2.0 * u0 - 1.0);
            pb = 0.0;
        } else {
            pa = a.size0 * (2.0 * u1 - 1.0);
            pb = (a.type == SLOTH_BEAM_SQUARE ? a.size0 : a.size1) * (2.0 * u0 - 1.0);
        }
        phi = kPi * u2;
        double x, y, z, vx, vy, vz;
        const double C = kC;
        if (a.type == SLOTH_BEAM_LINEAR) {
            x = pa; y = 0.0; z = a.extent;
            vx = C * sin(chi); vy = 0.0; vz = C * cos(chi);
        } else {
            const double ca = C * cos(chi), s1 = C * sin(chi) * cos(phi), s2 = C * sin(chi) * sin(phi);
            if (a.axis == 0) {
                x = a.extent; y = pa; z = pb;
                vx = ca; vy = s1; vz = s2;
            } else if (a.axis == 2) {
                x = pa; y = pb; z = a.extent;
                vx = s1; vy = s2; vz = ca;
            } else {
                x = pa; y = a.extent; z = pb;
                vx = s1; vy = ca; vz = s2;
            }
        }
        s0[i] = (T)x;
        s0[a.n + i] = (T)y;
        s0[2 * a.n + i] = (T)z;
        s0[3 * a.n + i] = (T)vx;
        s0[4 * a.n + i] = (T)vy;
        s0[5 * a.n + i] = (T)vz;
    }
}

template <class T>
static int beam_impl(const SlothBeamParams* p, int64_t n, T* s0, void* stream) {
    if (!p) return SLOTH_ERR_NULL_POINTER;
    if (n < 0 || p->reserved != 0) return SLOTH_ERR_INVALID_ARGUMENT;
    if (p->beam_type < SLOTH_BEAM_CIRCULAR || p->beam_type > SLOTH_BEAM_LINEAR) return SLOTH_ERR_INVALID_ARGUMENT;
    if (p->probing_axis < 0 || p->probing_axis > 2) return SLOTH_ERR_INVALID_ARGUMENT;
    if (!std::isfinite(p->size[0]) || !std::isfinite(p->size[1]) || !std::isfinite(p->divergence) ||
        !std::isfinite(p->ne_extent))
        return SLOTH_ERR_INVALID_ARGUMENT;
    if (n == 0) return SLOTH_OK;
    if (!s0) return SLOTH_ERR_NULL_POINTER;
    if ((uintptr_t)s0 & (sizeof(T) - 1)) return SLOTH_ERR_MISALIGNED;
    int sms = 148;
    int rc = device_sm_count(&sms);
    if (rc) return rc;
    BeamArgs a;
    a.type = p->beam_type;
    a.axis = p->probing_axis;
    a.size0 = p->size[0];
    a.size1 = p->size[1];
    a.divergence = p->divergence;
    a.extent = p->ne_extent;
    a.seed = p->seed;
    a.first_id = p->first_id;
    a.n = n;
    a.out = s0;
    long long blocks = (n + 255) / 256;
    if (blocks > (long long)sms * 8) blocks = (long long)sms * 8;
    beam_kernel<T><<<(unsigned)blocks, 256, 0, (cudaStream_t)stream>>>(a);
    note_launch();
    return cuda_status(cudaGetLastError());
}

}  // namespace sloth

extern "C" {

int sloth_beam_f32(const SlothBeamParams* p, int64_t n, float* s0, void* stream) {
    return sloth::beam_impl<float>(p, n, s0, stream);
}

int sloth_beam_f64(const SlothBeamParams* p, int64_t n, double* s0, void* stream) {
    return sloth::beam_impl<double>(p, n, s0, stream);
}

}  // extern "C"
