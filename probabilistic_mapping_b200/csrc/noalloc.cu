// noalloc.cu -- depth-fusion step that allocates no device memory.
//
// pm_stage_depth_fuse needs a caller-provided z-buffer (8 bytes per pixel) next to its inputs
// and outputs.  Some callers cannot provide one at run time: a control loop on a robot or a
// drone that must not call the CUDA allocator once it is flying (cudaMalloc can block and
// synchronise the device), a plugin running inside a host framework that owns every device
// buffer, or code that records its work into a CUDA graph where no allocation may happen.
// This variant keeps the z-buffer in a file-scope __device__ array instead.  The array is part
// of the library image, so every GPU that loads the library holds it (4 MiB) until the process
// exits, and every call shares it: the kernels clear it at the start of each call, and calls
// that run at the same time on the GPU (two streams, two host threads) overwrite each other's
// z-buffer and give wrong results.
#include <cuda.h>

#include <mutex>

#include "pm_device.cuh"
#include "pm_stereo.h"

namespace {

// Largest image this entry point accepts: 2^19 pixels (e.g. 640 x 480, 752 x 480, 640 x 512).
constexpr size_t kNoAllocMaxPixels = size_t(1) << 19;
static __device__ __align__(256) unsigned long long g_noalloc_ztable[kNoAllocMaxPixels];

// Device address of the array per device ordinal, with the id of the context it was looked up
// in.  In host code the symbol g_noalloc_ztable only names a host-side stand-in, so its address
// must come from cudaGetSymbolAddress with the device current before a kernel may use it.  The
// address belongs to one context: after a cudaDeviceReset the device gets a new primary context
// (a new id) and the library image is loaded again, so the address is looked up again.
constexpr int kMaxDevices = 128;
std::mutex g_setup_mu;
struct Slot {
    unsigned long long ctx_id = 0;   // 0: not looked up yet (context ids start at 1)
    unsigned long long* ptr = nullptr;
};
Slot g_slot[kMaxDevices];

// The three driver calls used here, looked up through the runtime (cudaGetDriverEntryPoint-
// ByVersion) so that the library needs no link-time dependency on libcuda.
struct DriverCalls {
    CUresult (*ctx_get_current)(CUcontext*) = nullptr;
    CUresult (*ctx_get_id)(CUcontext, unsigned long long*) = nullptr;
    CUresult (*stream_get_ctx)(CUstream, CUcontext*) = nullptr;
    bool ok = false;
};
DriverCalls g_drv;   // filled under g_setup_mu

bool driver_calls() {
    if (g_drv.ok) return true;
    cudaDriverEntryPointQueryResult q;
    void* p = nullptr;
    if (cudaGetDriverEntryPointByVersion("cuCtxGetCurrent", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !p)
        return false;
    g_drv.ctx_get_current = reinterpret_cast<CUresult (*)(CUcontext*)>(p);
    if (cudaGetDriverEntryPointByVersion("cuCtxGetId", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !p)
        return false;
    g_drv.ctx_get_id = reinterpret_cast<CUresult (*)(CUcontext, unsigned long long*)>(p);
    if (cudaGetDriverEntryPointByVersion("cuStreamGetCtx", &p, 12000, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !p)
        return false;
    g_drv.stream_get_ctx = reinterpret_cast<CUresult (*)(CUstream, CUcontext*)>(p);
    g_drv.ok = true;
    return true;
}

// The current context and its id; null when the runtime has not made one current yet.
CUresult current_context(CUcontext* ctx, unsigned long long* id) {
    *ctx = nullptr;
    *id = 0;
    CUresult r = g_drv.ctx_get_current(ctx);
    if (r != CUDA_SUCCESS || !*ctx) return r;
    return g_drv.ctx_get_id(*ctx, id);
}

pm_status ztable_for_current_device(CUcontext* ctx_out, unsigned long long** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return PM_ERR_CUDA;
    if (dev < 0 || dev >= kMaxDevices) return PM_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!driver_calls()) return PM_ERR_CUDA;
    CUcontext ctx = nullptr;
    unsigned long long id = 0;
    if (current_context(&ctx, &id) != CUDA_SUCCESS) return PM_ERR_CUDA;
    if (!ctx || id != g_slot[dev].ctx_id) {
        // cudaGetSymbolAddress makes the device's primary context current if it is not yet
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_ztable) != cudaSuccess || !p) return PM_ERR_CUDA;
        if (current_context(&ctx, &id) != CUDA_SUCCESS || !ctx) return PM_ERR_CUDA;
        g_slot[dev].ctx_id = id;
        g_slot[dev].ptr = static_cast<unsigned long long*>(p);
    }
    *ctx_out = ctx;
    *out = g_slot[dev].ptr;
    return PM_OK;
}

// The stream must run in the current context: the array's address is that context's.
bool stream_in_context(void* stream, CUcontext ctx) {
    const uintptr_t s = reinterpret_cast<uintptr_t>(stream);
    if (s == 0 || s == reinterpret_cast<uintptr_t>(cudaStreamLegacy) ||
        s == reinterpret_cast<uintptr_t>(cudaStreamPerThread))
        return true;   // the default streams belong to the current context
    CUcontext sctx = nullptr;
    return g_drv.stream_get_ctx(static_cast<CUstream>(stream), &sctx) == CUDA_SUCCESS && sctx == ctx;
}

}  // namespace

extern "C" pm_status pm_stage_depth_fuse_noalloc(int W, int H, const float pose[12], const float cam[4],
                                                float* depth, float* const pre[4], float* const cur[4],
                                                int32_t* table, void* stream) {
    if (W <= 0 || H <= 0 || !pose || !cam || !depth || !pre || !cur) return PM_ERR_INVALID_ARGUMENT;
    if ((size_t)W * (size_t)H > kNoAllocMaxPixels) return PM_ERR_INVALID_ARGUMENT;   // beyond the array
    pm::FuseLaunch f{};   // value-initialised: no device-side step parameters
    f.W = W;
    f.H = H;
    for (int i = 0; i < 12; ++i) f.pose[i] = pose[i];
    for (int i = 0; i < 4; ++i) f.cam[i] = cam[i];
    f.depth = depth;
    for (int k = 0; k < 4; ++k) {
        if (!pre[k] || !cur[k]) return PM_ERR_INVALID_ARGUMENT;
        f.pre[k] = pre[k];
        f.cur[k] = cur[k];
    }
    f.table = table;
    f.variance = nullptr;
    CUcontext ctx = nullptr;
    pm_status st = ztable_for_current_device(&ctx, &f.ztable);
    if (st != PM_OK) return st;
    if (!stream_in_context(stream, ctx)) return PM_ERR_INVALID_ARGUMENT;
    // launch_fuse_gpu clears the z-buffer on `stream` before the kernels use it
    return pm::launch_fuse_gpu(f, (cudaStream_t)stream) == cudaSuccess ? PM_OK : PM_ERR_CUDA;
}
