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
#include <mutex>

#include "pm_device.cuh"
#include "pm_stereo.h"

namespace {

// Largest image this entry point accepts: 2^19 pixels (e.g. 640 x 480, 752 x 480, 640 x 512).
constexpr size_t kNoAllocMaxPixels = size_t(1) << 19;
static __device__ __align__(256) unsigned long long g_noalloc_ztable[kNoAllocMaxPixels];

// Device address of the array per device ordinal, looked up once per device.  In host code the
// symbol g_noalloc_ztable only names a host-side stand-in, so its address must come from
// cudaGetSymbolAddress with the device current before a kernel may use it.
constexpr int kMaxDevices = 128;
std::mutex g_setup_mu;
unsigned long long* g_ztable_dev[kMaxDevices] = {};

pm_status ztable_for_current_device(unsigned long long** out) {
    int dev = -1;
    if (cudaGetDevice(&dev) != cudaSuccess) return PM_ERR_CUDA;
    if (dev < 0 || dev >= kMaxDevices) return PM_ERR_UNSUPPORTED;
    std::lock_guard<std::mutex> lock(g_setup_mu);
    if (!g_ztable_dev[dev]) {
        void* p = nullptr;
        if (cudaGetSymbolAddress(&p, g_noalloc_ztable) != cudaSuccess || !p) return PM_ERR_CUDA;
        g_ztable_dev[dev] = static_cast<unsigned long long*>(p);
    }
    *out = g_ztable_dev[dev];
    return PM_OK;
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
    pm_status st = ztable_for_current_device(&f.ztable);
    if (st != PM_OK) return st;
    // launch_fuse_gpu clears the z-buffer on `stream` before the kernels use it
    return pm::launch_fuse_gpu(f, (cudaStream_t)stream) == cudaSuccess ? PM_OK : PM_ERR_CUDA;
}
