// K2 (FP32 split) and K3 (FP64 port) tracer entry points: one trace of one
// ray set through one grid (the device code is in tracer.cuh).
#include <algorithm>

#include "tracer.cuh"

namespace sloth {

template <class P, int IB, int FAST, int INTEG>
__global__ void __launch_bounds__(kThreads, SLOTH_TRACE_MIN_BLOCKS)
trace_kernel(const __grid_constant__ TraceArgs a) {
    __shared__ unsigned s_key[kTile];
    __shared__ unsigned s_id[kTile];
    __shared__ int s_tile, s_head;
    __shared__ unsigned long long s_steps;
    unsigned long long my_steps = 0;
    if (threadIdx.x == 0) s_steps = 0;
    CellCacheFor<P, IB> cc;
    cc.base = 0xffffffffu;
    for (;;) {
        if (threadIdx.x == 0) {
            s_tile = atomicAdd(a.tile_counter, 1);
            s_head = 0;
        }
        __syncthreads();
        const int tile = s_tile;
        if (tile >= a.n_tiles) break;
        // Rays that start together in a tile have similar lifetimes, so a
        // kTile tile runs as kTile / kThreads waves. The queue ends in tiles
        // of one wave, so the CTAs finish within about one ray lifetime of
        // each other instead of one tile.
        long long start;
        int cnt;
        if (tile < a.n_big) {
            start = (long long)tile * kTile;
            cnt = kTile;
        } else {
            start = (long long)a.n_big * kTile + (long long)(tile - a.n_big) * kSmallTile;
            cnt = (int)min((long long)kSmallTile, a.n - start);
        }
        trace_tile<P, IB, FAST, INTEG>(a, start, cnt, s_key, s_id, &s_head, cc, my_steps);
    }
    // one atomic per CTA for the ray-step total
    block_add(my_steps, &s_steps, a.total_steps);
}

template <class P, int IB, int FAST, int INTEG>
static int launch_trace_k(const TraceArgs& ta, int sms, cudaStream_t s) {
    static int cached[64] = {0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_status(e);
    int per_sm = (dev >= 0 && dev < 64) ? cached[dev] : 0;
    if (per_sm <= 0) {
        if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, trace_kernel<P, IB, FAST, INTEG>, kThreads, 0) !=
                cudaSuccess || per_sm < 1)
            per_sm = 1;
        if (dev >= 0 && dev < 64) cached[dev] = per_sm;
    }
    long long blocks = (long long)sms * per_sm;
    // tile queue: big tiles, then the last kTailWaves small tiles per CTA
    TraceArgs t = ta;
    const long long small = std::min(ta.n, (long long)kTailWaves * blocks * kSmallTile);
    t.n_big = (int)((ta.n - small) / kTile);
    const long long rest = ta.n - (long long)t.n_big * kTile;
    t.n_tiles = t.n_big + (int)((rest + kSmallTile - 1) / kSmallTile);
    if (blocks > t.n_tiles) blocks = t.n_tiles;
    trace_kernel<P, IB, FAST, INTEG><<<(int)blocks, kThreads, 0, s>>>(t);
    note_launch();
    return cuda_status(cudaGetLastError());
}

template <class P, int IB, int INTEG>
static int launch_trace_i(const TraceArgs& ta, int sms, cudaStream_t s, int fast) {
    return fast == 1 ? launch_trace_k<P, IB, 1, INTEG>(ta, sms, s)
         : fast == 2 ? launch_trace_k<P, IB, 2, INTEG>(ta, sms, s)
                     : launch_trace_k<P, IB, 0, INTEG>(ta, sms, s);
}

template <class P, int IB>
static int launch_trace(const TraceArgs& ta, int sms, cudaStream_t s, int fast, int integ) {
    return integ == INTEG_RK4 ? launch_trace_i<P, IB, INTEG_RK4>(ta, sms, s, fast)
                              : launch_trace_i<P, IB, INTEG_RKN>(ta, sms, s, fast);
}

template <class P>
static int trace_impl(const SlothGridDesc* g, const void* grid, const SlothTraceParams* p,
                      const void* rays, int64_t n, const SlothTraceOutputs* out, void* ws,
                      size_t ws_bytes, void* stream) {
    using R = typename P::R;
    int rc = check_trace_params(g, p, n);
    if (rc) return rc;
    if (!out) return SLOTH_ERR_NULL_POINTER;
    if (n == 0) {
        if (out->total_steps) {
            cudaError_t e = cudaMemsetAsync(out->total_steps, 0, sizeof(unsigned long long), (cudaStream_t)stream);
            return cuda_status(e);
        }
        return SLOTH_OK;
    }
    if (!grid || !rays || !out->jones || !ws) return SLOTH_ERR_NULL_POINTER;
    if (((uintptr_t)grid & 15u) != 0 || ((uintptr_t)ws & 255u) != 0) return SLOTH_ERR_MISALIGNED;
    if (((uintptr_t)rays & (sizeof(R) - 1)) != 0 || ((uintptr_t)out->jones & (sizeof(R) - 1)) != 0)
        return SLOTH_ERR_MISALIGNED;
    if (ws_bytes < workspace_bytes(n)) return SLOTH_ERR_WORKSPACE_TOO_SMALL;

    cudaStream_t s = (cudaStream_t)stream;
    char* base = reinterpret_cast<char*>(ws);
    int* tile_counter = reinterpret_cast<int*>(base);
    unsigned* hist = reinterpret_cast<unsigned*>(base + kHeaderBytes);
    const size_t an = align256((size_t)n * 4u);
    unsigned* keys = reinterpret_cast<unsigned*>(base + kHeaderBytes + kHistBytes);
    unsigned* perm = reinterpret_cast<unsigned*>(base + kHeaderBytes + kHistBytes + an);
    unsigned* skeys = reinterpret_cast<unsigned*>(base + kHeaderBytes + kHistBytes + 2 * an);

    const int bbits = bucket_bits_for(n);
    cudaError_t e = cudaMemsetAsync(base, 0, kHeaderBytes + ((size_t)4 << bbits), s);
    if (e != cudaSuccess) return cuda_status(e);
    if (out->total_steps) {
        e = cudaMemsetAsync(out->total_steps, 0, sizeof(unsigned long long), s);
        if (e != cudaSuccess) return cuda_status(e);
    }
    int sms = 148;
    rc = device_sm_count(&sms);
    if (rc) return rc;
    rc = launch_prepass<R>(g, p->probing_axis, reinterpret_cast<const R*>(rays), n, bbits, keys, hist, perm,
                           skeys, sms, s);
    if (rc) return rc;

    TraceArgs ta;
    fill_trace_args(ta, g, grid, p, rays, n, out, perm, skeys);
    ta.tile_counter = tile_counter;
    const int ib = trace_mode(p);
    // interior runs with interior sampling, interior runs only, or neither
    const int fast = interior_bound_ok(g, p) ? 1 : (std::isfinite(interior_accel_bound(g, p)) ? 2 : 0);

    if (out->trace_event_begin) {
        e = cudaEventRecord((cudaEvent_t)out->trace_event_begin, s);
        if (e != cudaSuccess) return cuda_status(e);
    }
    const int integ = p->integrator;
    if (ib == IB_OFF)
        rc = launch_trace<P, IB_OFF>(ta, sms, s, fast, integ);
    else if (ib == IB_SUBCRITICAL)
        rc = launch_trace<P, IB_SUBCRITICAL>(ta, sms, s, fast, integ);
    else
        rc = launch_trace<P, IB_GENERAL>(ta, sms, s, fast, integ);
    if (rc) return rc;
    if (out->trace_event_end) {
        e = cudaEventRecord((cudaEvent_t)out->trace_event_end, s);
        if (e != cudaSuccess) return cuda_status(e);
    }
    return SLOTH_OK;
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the FP32 tracer: its scratch (tile counter,
// bucket histogram, keys, permutation) lives in one file-scope device array
// sized for SLOTH_NOALLOC_MAX_RAYS rays, so the caller passes only inputs and
// outputs and nothing here allocates. Host code cannot use the array's name
// as a device address; every call looks the current device's address up with
// cudaGetSymbolAddress (the first call on a device also loads the library's
// device code there). A cached address would dangle after cudaDeviceReset,
// which reloads the device code at a new address. All calls share the array,
// which keeps the previous call's contents (the tracer zeroes the parts that
// must start at zero), so calls that overlap on the GPU race.
// ---------------------------------------------------------------------------
constexpr size_t kNoAllocScratchBytes = kHeaderBytes + kHistBytes + 3 * (size_t)4 * SLOTH_NOALLOC_MAX_RAYS;
static_assert(kNoAllocScratchBytes % 256 == 0, "scratch sections must stay 256-byte aligned");

static __device__ __align__(256) unsigned char g_noalloc_scratch[kNoAllocScratchBytes];

static int noalloc_scratch(void** out) {
    void* addr = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&addr, g_noalloc_scratch);
    if (e != cudaSuccess) return cuda_status(e);
    if (addr == nullptr || ((uintptr_t)addr & 255u) != 0) return SLOTH_ERR_MISALIGNED;
    *out = addr;
    return SLOTH_OK;
}

}  // namespace sloth

extern "C" {

size_t sloth_trace_workspace_bytes(int64_t n_rays) { return sloth::workspace_bytes(n_rays); }

int sloth_trace_f32_noalloc(const SlothGridDesc* g, const void* grid, const SlothTraceParams* p,
                            const float* rays, int64_t n, const SlothTraceOutputs* out, void* stream) {
    if (n < 0) return SLOTH_ERR_INVALID_ARGUMENT;
    if (n > (int64_t)SLOTH_NOALLOC_MAX_RAYS) return SLOTH_ERR_TOO_LARGE;
    void* scratch = nullptr;
    const int rc = sloth::noalloc_scratch(&scratch);
    if (rc) return rc;
    return sloth::trace_impl<sloth::PolF32>(g, grid, p, rays, n, out, scratch, sloth::kNoAllocScratchBytes,
                                            stream);
}

int sloth_trace_f32(const SlothGridDesc* g, const void* grid, const SlothTraceParams* p, const float* rays,
                    int64_t n, const SlothTraceOutputs* out, void* workspace, size_t workspace_bytes,
                    void* stream) {
    return sloth::trace_impl<sloth::PolF32>(g, grid, p, rays, n, out, workspace, workspace_bytes, stream);
}

int sloth_trace_f64(const SlothGridDesc* g, const void* grid, const SlothTraceParams* p, const double* rays,
                    int64_t n, const SlothTraceOutputs* out, void* workspace, size_t workspace_bytes,
                    void* stream) {
    return sloth::trace_impl<sloth::PolF64>(g, grid, p, rays, n, out, workspace, workspace_bytes, stream);
}

}  // extern "C"
