// Library-level entry points and host helpers shared by the kernels' C ABI.
#include <atomic>
#include <cmath>

#include "common.cuh"

namespace sloth {

static std::atomic<unsigned long long> g_launches{0};

void note_launch() { g_launches.fetch_add(1, std::memory_order_relaxed); }

int cuda_status(cudaError_t e) {
    if (e == cudaSuccess) return SLOTH_OK;
    if (e == cudaErrorNoDevice || e == cudaErrorInsufficientDriver) return SLOTH_ERR_NO_DEVICE;
    if (e == cudaErrorMemoryAllocation) return SLOTH_ERR_OUT_OF_MEMORY;
    if (e == cudaErrorNoKernelImageForDevice || e == cudaErrorInvalidDeviceFunction)
        return SLOTH_ERR_UNSUPPORTED_DEVICE;
    return SLOTH_ERR_CUDA;
}

int device_sm_count(int* sms) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return cuda_status(e);
    static int cache[64] = {0};
    if (dev >= 0 && dev < 64 && cache[dev] > 0) {
        *sms = cache[dev];
        return SLOTH_OK;
    }
    int v = 0;
    e = cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev);
    if (e != cudaSuccess) return cuda_status(e);
    if (dev >= 0 && dev < 64) cache[dev] = v;
    *sms = v;
    return SLOTH_OK;
}

int check_grid(const SlothGridDesc* g) {
    if (!g) return SLOTH_ERR_NULL_POINTER;
    if (g->reserved != 0) return SLOTH_ERR_INVALID_ARGUMENT;
    double total = 1.0;
    for (int a = 0; a < 3; ++a) {
        if (g->n[a] < 2) return SLOTH_ERR_INVALID_ARGUMENT;
        if (!(g->spacing[a] > 0.0) || !std::isfinite(g->spacing[a]) || !std::isfinite(g->origin[a]))
            return SLOTH_ERR_INVALID_ARGUMENT;
        total *= (double)g->n[a];
    }
    // Voxel indices are 32-bit inside the kernels.
    if (total >= 2147483647.0) return SLOTH_ERR_TOO_LARGE;
    return SLOTH_OK;
}

GridGeo make_geo(const SlothGridDesc* g) {
    GridGeo k;
    for (int a = 0; a < 3; ++a) {
        k.n[a] = g->n[a];
        k.limd[a] = (double)(g->n[a] - 1);
        k.limf[a] = (float)(g->n[a] - 1);
    }
    k.sy = (unsigned)g->n[2];
    k.sx = (unsigned)g->n[1] * (unsigned)g->n[2];
    return k;
}

}  // namespace sloth

extern "C" {

const char* sloth_strerror(int code) {
    switch (code) {
        case SLOTH_OK: return "success";
        case SLOTH_ERR_INVALID_ARGUMENT: return "invalid argument";
        case SLOTH_ERR_NULL_POINTER: return "required pointer is NULL";
        case SLOTH_ERR_MISALIGNED: return "buffer is not aligned as required";
        case SLOTH_ERR_WORKSPACE_TOO_SMALL: return "workspace is smaller than required";
        case SLOTH_ERR_CUDA: return "CUDA runtime error";
        case SLOTH_ERR_NO_DEVICE: return "no usable CUDA device";
        case SLOTH_ERR_TOO_LARGE: return "size exceeds the supported maximum";
        case SLOTH_ERR_OUT_OF_MEMORY: return "out of device memory or budget";
        case SLOTH_ERR_NOT_FOUND: return "no such object";
        case SLOTH_ERR_BUSY: return "object is busy";
        case SLOTH_ERR_UNSUPPORTED_DEVICE: return "device is not sm_100 (B200); kernels are built for sm_100a only";
        default: return "unknown error code";
    }
}

int sloth_abi_version(void) { return SLOTH_ABI_VERSION; }

int sloth_device_info(int* sm_count, int* cc_major, int* cc_minor) {
    if (!sm_count || !cc_major || !cc_minor) return SLOTH_ERR_NULL_POINTER;
    int n = 0;
    cudaError_t e = cudaGetDeviceCount(&n);
    if (e != cudaSuccess || n == 0) {
        cudaGetLastError();
        return SLOTH_ERR_NO_DEVICE;
    }
    int dev = 0;
    e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return sloth::cuda_status(e);
    e = cudaDeviceGetAttribute(sm_count, cudaDevAttrMultiProcessorCount, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(cc_major, cudaDevAttrComputeCapabilityMajor, dev);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(cc_minor, cudaDevAttrComputeCapabilityMinor, dev);
    return sloth::cuda_status(e);
}

unsigned long long sloth_launch_count(void) {
    return sloth::g_launches.load(std::memory_order_relaxed);
}

}  // extern "C"
