// imgproc.cu -- the image work of the sequence driver (evaluate.cc) on the GPU:
//   pyr_down_kernel   cv::pyrDown of a uint8 frame (evaluate.cc:176-178, 221-225);
//   depth_up2_kernel  depthUp, the nearest-neighbour 2x enlargement (evaluate.cc:121-135, 262-266);
//   range_mask_kernel the min/max depth masking (evaluate.cc:278-289);
//   minmax_kernel + colorize_kernel
//                     the debug view (evaluate.cc:291-307): cv::normalize(NORM_MINMAX, CV_8U),
//                     an 8-bit colour map, black where depth < 0.001.
//
// pyrDown is OpenCV's published Gaussian pyramid step: the 5x5 binomial kernel
// [1 4 6 4 1]^T [1 4 6 4 1] / 256 at every second pixel, borders mirrored without repeating the
// edge pixel (BORDER_REFLECT_101), result rounded half up, (sum + 128) >> 8.  All sums are exact
// integers, so any summation order gives OpenCV's bytes.
//
// The colour map is this library's own hue ramp, not OpenCV's COLORMAP_RAINBOW table: level v
// maps to t = 5 v, segment k = t / 256, f = t % 256, and (R, G, B) =
//   k 0: (255, f, 0)   red -> yellow        k 3: (0, 255 - f, 255)  cyan -> blue
//   k 1: (255 - f, 255, 0) yellow -> green  k 4: (f, 0, 255)        blue -> magenta
//   k 2: (0, 255, f)   green -> cyan
// stored B, G, R per pixel like an OpenCV 8UC3 image.
#include "pm_stereo.h"
#include "pm_device.cuh"

namespace pm {
namespace {

constexpr int kTx = 32, kTy = 8;                         // output tile of pyr_down_kernel
constexpr int kSx = 2 * kTx + 4, kSy = 2 * kTy + 4;      // source tile with the 2-pixel apron

// BORDER_REFLECT_101 index for any offset (iterated, so tiny images fold back correctly).
__device__ __forceinline__ int reflect101(int p, int n) {
    if (n == 1) return 0;
    while ((unsigned)p >= (unsigned)n) p = p < 0 ? -p : 2 * n - 2 - p;
    return p;
}

__global__ void __launch_bounds__(kTx * kTy) pyr_down_kernel(int W, int H, const uint8_t* __restrict__ src,
                                                            size_t sp, uint8_t* __restrict__ dst, size_t dp,
                                                            int dW, int dH) {
    __shared__ int s_src[kSy][kSx];
    __shared__ int s_row[kSy][kTx];
    const int ox0 = blockIdx.x * kTx, oy0 = blockIdx.y * kTy;
    const int sx0 = 2 * ox0 - 2, sy0 = 2 * oy0 - 2;
    const int tid = threadIdx.y * kTx + threadIdx.x;
    for (int i = tid; i < kSx * kSy; i += kTx * kTy) {
        const int r = i / kSx, c = i - r * kSx;
        s_src[r][c] = src[(size_t)reflect101(sy0 + r, H) * sp + reflect101(sx0 + c, W)];
    }
    __syncthreads();
    // horizontal pass for every source row of the tile
    for (int i = tid; i < kSy * kTx; i += kTx * kTy) {
        const int r = i / kTx, c = i - r * kTx;
        const int* p = &s_src[r][2 * c];
        s_row[r][c] = p[0] + 4 * p[1] + 6 * p[2] + 4 * p[3] + p[4];
    }
    __syncthreads();
    const int ox = ox0 + threadIdx.x, oy = oy0 + threadIdx.y;
    if (ox >= dW || oy >= dH) return;
    const int r = 2 * threadIdx.y, c = threadIdx.x;
    const int sum = s_row[r][c] + 4 * s_row[r + 1][c] + 6 * s_row[r + 2][c] + 4 * s_row[r + 3][c] + s_row[r + 4][c];
    dst[(size_t)oy * dp + ox] = (uint8_t)((sum + 128) >> 8);
}

__global__ void __launch_bounds__(256) depth_up2_kernel(int W, int H, const float* __restrict__ src, size_t sp,
                                                        float* __restrict__ dst, size_t dp) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= 2 * W) return;
    const float v = *reinterpret_cast<const float*>(reinterpret_cast<const char*>(src) + (size_t)(y >> 1) * sp +
                                                    (size_t)(x >> 1) * 4);
    *reinterpret_cast<float*>(reinterpret_cast<char*>(dst) + (size_t)y * dp + (size_t)x * 4) = v;
}

__global__ void __launch_bounds__(256) range_mask_kernel(int W, int H, float* depth, size_t pitch, float lo,
                                                         float hi) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    float* p = reinterpret_cast<float*>(reinterpret_cast<char*>(depth) + (size_t)y * pitch) + x;
    float d = *p;
    if (d < lo) d = 0.0f;
    if (d > hi) d = 0.0f;
    *p = d;
}

// float <-> unsigned key whose unsigned order is the float order (NaN excluded by the caller)
__device__ __forceinline__ unsigned f2key(float f) {
    const unsigned b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float key2f(unsigned k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7fffffffu) : ~k);
}

// cv::minMaxIdx over the map (NaNs skipped); keys[0] = min, keys[1] = max, cleared by the host.
__global__ void __launch_bounds__(256) minmax_kernel(int W, int H, const float* __restrict__ depth, size_t pitch,
                                                     unsigned* keys) {
    unsigned kmin = 0xffffffffu, kmax = 0u;
    const long n = (long)W * H;
    for (long i = (long)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x) {
        const int y = (int)(i / W), x = (int)(i - (long)y * W);
        const float d = *reinterpret_cast<const float*>(reinterpret_cast<const char*>(depth) + (size_t)y * pitch +
                                                        (size_t)x * 4);
        if (d != d) continue;
        const unsigned k = f2key(d);
        kmin = min(kmin, k);
        kmax = max(kmax, k);
    }
    kmin = __reduce_min_sync(kFull, kmin);
    kmax = __reduce_max_sync(kFull, kmax);
    if ((threadIdx.x & 31) == 0) {
        atomicMin(keys, kmin);
        atomicMax(keys + 1, kmax);
    }
}

__device__ __forceinline__ void hue_ramp(int v, uint8_t& r, uint8_t& g, uint8_t& b) {
    const int t = 5 * v, k = t >> 8, f = t & 255;
    switch (k) {
        case 0: r = 255; g = (uint8_t)f; b = 0; break;
        case 1: r = (uint8_t)(255 - f); g = 255; b = 0; break;
        case 2: r = 0; g = 255; b = (uint8_t)f; break;
        case 3: r = 0; g = (uint8_t)(255 - f); b = 255; break;
        default: r = (uint8_t)f; g = 0; b = 255; break;
    }
}

// cv::normalize(src, dst, 0, 255, NORM_MINMAX, CV_8U): scale = 255 / (max - min) (0 when the
// range is not above DBL_EPSILON) and shift = -min * scale in double, both rounded to float,
// then level = saturate(round-half-even(fma(d, scale, shift))), the fused multiply-add of
// OpenCV's vectorised float -> uint8 conversion.
__global__ void __launch_bounds__(256) colorize_kernel(int W, int H, const float* __restrict__ depth, size_t pitch,
                                                       const unsigned* __restrict__ keys, uint8_t* level,
                                                       size_t lp, uint8_t* bgr, size_t bp) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    if (x >= W) return;
    const double smin = keys[0] == 0xffffffffu ? 0.0 : (double)key2f(keys[0]);
    const double smax = keys[0] == 0xffffffffu ? 0.0 : (double)key2f(keys[1]);
    const double range = smax - smin;
    const double scale = range > 2.220446049250313e-16 ? 255.0 / range : 0.0;
    const double shift = 0.0 - smin * scale;
    const float a = (float)scale, b = (float)shift;
    const float d = *reinterpret_cast<const float*>(reinterpret_cast<const char*>(depth) + (size_t)y * pitch +
                                                    (size_t)x * 4);
    const float v = __fmaf_rn(d, a, b);
    int iv = (v != v) ? 0 : __float2int_rn(v);   // cvRound of NaN is INT_MIN -> saturates to 0
    iv = iv < 0 ? 0 : (iv > 255 ? 255 : iv);
    if (level) level[(size_t)y * lp + x] = (uint8_t)iv;
    if (bgr) {
        uint8_t r, g, bl;
        hue_ramp(iv, r, g, bl);
        if (d < 0.001f) r = g = bl = 0;
        uint8_t* o = bgr + (size_t)y * bp + 3 * (size_t)x;
        o[0] = bl;
        o[1] = g;
        o[2] = r;
    }
}

}  // namespace
}  // namespace pm

using namespace pm;

extern "C" {

pm_status pm_pyr_down_u8(int W, int H, const uint8_t* src, size_t src_pitch, uint8_t* dst, size_t dst_pitch,
                         void* stream) {
    if (W < 2 || H < 2 || !src || !dst) return PM_ERR_INVALID_ARGUMENT;
    const int dW = W / 2, dH = H / 2;
    if (src_pitch == 0) src_pitch = (size_t)W;
    if (dst_pitch == 0) dst_pitch = (size_t)dW;
    if (src_pitch < (size_t)W || dst_pitch < (size_t)dW) return PM_ERR_INVALID_ARGUMENT;
    const dim3 grid((dW + kTx - 1) / kTx, (dH + kTy - 1) / kTy);
    pyr_down_kernel<<<grid, dim3(kTx, kTy), 0, (cudaStream_t)stream>>>(W, H, src, src_pitch, dst, dst_pitch, dW, dH);
    return cudaGetLastError() == cudaSuccess ? PM_OK : PM_ERR_CUDA;
}

pm_status pm_depth_up2(int W, int H, const float* src, size_t src_pitch, float* dst, size_t dst_pitch,
                       void* stream) {
    if (W <= 0 || H <= 0 || !src || !dst) return PM_ERR_INVALID_ARGUMENT;
    if (src_pitch == 0) src_pitch = 4 * (size_t)W;
    if (dst_pitch == 0) dst_pitch = 8 * (size_t)W;
    if (src_pitch < 4 * (size_t)W || dst_pitch < 8 * (size_t)W || (src_pitch | dst_pitch) % 4)
        return PM_ERR_INVALID_ARGUMENT;
    const dim3 grid((2 * W + 255) / 256, 2 * H);
    depth_up2_kernel<<<grid, 256, 0, (cudaStream_t)stream>>>(W, H, src, src_pitch, dst, dst_pitch);
    return cudaGetLastError() == cudaSuccess ? PM_OK : PM_ERR_CUDA;
}

pm_status pm_depth_range_mask(int W, int H, float* depth, size_t pitch, float min_depth, float max_depth,
                              void* stream) {
    if (W <= 0 || H <= 0 || !depth) return PM_ERR_INVALID_ARGUMENT;
    if (pitch == 0) pitch = 4 * (size_t)W;
    if (pitch < 4 * (size_t)W || pitch % 4) return PM_ERR_INVALID_ARGUMENT;
    range_mask_kernel<<<dim3((W + 255) / 256, H), 256, 0, (cudaStream_t)stream>>>(W, H, depth, pitch, min_depth,
                                                                                 max_depth);
    return cudaGetLastError() == cudaSuccess ? PM_OK : PM_ERR_CUDA;
}

pm_status pm_colorize_depth(int W, int H, const float* depth, size_t pitch, uint8_t* level, size_t level_pitch,
                            uint8_t* bgr, size_t bgr_pitch, unsigned* scratch, void* stream) {
    if (W <= 0 || H <= 0 || !depth || !scratch || (!level && !bgr)) return PM_ERR_INVALID_ARGUMENT;
    if (pitch == 0) pitch = 4 * (size_t)W;
    if (level_pitch == 0) level_pitch = (size_t)W;
    if (bgr_pitch == 0) bgr_pitch = 3 * (size_t)W;
    if (pitch < 4 * (size_t)W || pitch % 4 || level_pitch < (size_t)W || bgr_pitch < 3 * (size_t)W)
        return PM_ERR_INVALID_ARGUMENT;
    cudaStream_t s = (cudaStream_t)stream;
    if (cudaMemsetAsync(scratch, 0xff, 4, s) != cudaSuccess || cudaMemsetAsync(scratch + 1, 0, 4, s) != cudaSuccess)
        return PM_ERR_CUDA;
    const long n = (long)W * H;
    const int blocks = (int)((n + 255) / 256 < 592 ? (n + 255) / 256 : 592);   // 4 per SM at most
    minmax_kernel<<<blocks, 256, 0, s>>>(W, H, depth, pitch, scratch);
    colorize_kernel<<<dim3((W + 255) / 256, H), 256, 0, s>>>(W, H, depth, pitch, scratch, level, level_pitch, bgr,
                                                             bgr_pitch);
    return cudaGetLastError() == cudaSuccess ? PM_OK : PM_ERR_CUDA;
}

}  // extern "C"
