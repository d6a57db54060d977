// convert.cu -- image conversions.
//   to_float_kernel: uint8 -> scaled float, the convertTo(CV_32F) + upload of
//                    StereoMapper::initReference / update (stereo_mapper.cpp:65-67,75-77);
//                    pitched, it fills the FP32 texels of the FP32 form's texture sampler.
//   to_half_kernel:  uint8 -> scaled FP16 (pitched texture storage of the FP16 form), or the
//                    same values widened to float (its reference image).
//   convert_kernel:  pitched <-> linear float copy (reference: convert.cu:4-45).  The pitch is
//                    taken in bytes; the reference received a byte step and indexed with it in
//                    floats (stereo_mapper.cpp:149-152 vs convert.cu:16-21), which reads past
//                    the end of the source for every row after the first quarter.
#include <cstring>

#include "pm_device.cuh"

namespace pm {
namespace {

__global__ void __launch_bounds__(256) to_float_kernel(int W, int H, const uint8_t* __restrict__ src,
                                                       size_t pitch, float* __restrict__ dst, size_t dst_pitch,
                                                       float scale) {
    const int y = blockIdx.y;
    const uint8_t* row = src + (size_t)y * pitch;
    float* out = reinterpret_cast<float*>(reinterpret_cast<char*>(dst) + (size_t)y * dst_pitch);
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < W; x += gridDim.x * blockDim.x)
        out[x] = __fmul_rn((float)row[x], scale);
}

__global__ void __launch_bounds__(256) to_quad_kernel(int W, int H, const uint8_t* __restrict__ src,
                                                      size_t pitch, float4* __restrict__ dst, float scale) {
    const int y = blockIdx.y;
    const uint8_t* r0 = src + (size_t)y * pitch;
    const uint8_t* r1 = r0 + pitch;
    const bool has1 = (y + 1) < H;
    float4* out = dst + (size_t)y * W;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < W; x += gridDim.x * blockDim.x) {
        const bool hasx = (x + 1) < W;
        float4 q;
        q.x = __fmul_rn((float)r0[x], scale);                                   // I(x, y)
        q.y = has1 ? __fmul_rn((float)r1[x], scale) : 0.0f;                     // I(x, y+1)
        q.z = hasx ? __fmul_rn((float)r0[x + 1], scale) : 0.0f;                 // I(x+1, y)
        q.w = (has1 && hasx) ? __fmul_rn((float)r1[x + 1], scale) : 0.0f;       // I(x+1, y+1)
        out[x] = q;
    }
}

__global__ void __launch_bounds__(256) to_half_kernel(int W, int H, const uint8_t* __restrict__ src, size_t pitch,
                                                      __half* __restrict__ dst, size_t dst_pitch, float scale,
                                                      int as_float) {
    const int y = blockIdx.y;
    const uint8_t* row = src + (size_t)y * pitch;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < W; x += gridDim.x * blockDim.x) {
        const __half v = __float2half_rn(__fmul_rn((float)row[x], scale));
        if (as_float)   // FP16-rounded values in float lanes, pitched (dst_pitch 0: packed rows)
            reinterpret_cast<float*>(reinterpret_cast<char*>(dst) + (size_t)y * (dst_pitch ? dst_pitch : 4 * (size_t)W))[x] =
                __half2float(v);
        else reinterpret_cast<__half*>(reinterpret_cast<char*>(dst) + (size_t)y * dst_pitch)[x] = v;
    }
}

// Quads for the FP16 form's sampler: the layout of to_quad_kernel with every value rounded to
// FP16 (the form's image precision), held in FP32 lanes so that a sample needs no conversion.
__global__ void __launch_bounds__(256) to_quad_half_kernel(int W, int H, const uint8_t* __restrict__ src,
                                                           size_t pitch, float4* __restrict__ dst, float scale) {
    const int y = blockIdx.y;
    const uint8_t* r0 = src + (size_t)y * pitch;
    const uint8_t* r1 = r0 + pitch;
    const bool has1 = (y + 1) < H;
    float4* out = dst + (size_t)y * W;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < W; x += gridDim.x * blockDim.x) {
        const bool hasx = (x + 1) < W;
        float4 q;
        q.x = __half2float(__float2half_rn(__fmul_rn((float)r0[x], scale)));                     // I(x, y)
        q.y = has1 ? __half2float(__float2half_rn(__fmul_rn((float)r1[x], scale))) : 0.0f;         // I(x, y+1)
        q.z = hasx ? __half2float(__float2half_rn(__fmul_rn((float)r0[x + 1], scale))) : 0.0f;     // I(x+1, y)
        q.w = (has1 && hasx) ? __half2float(__float2half_rn(__fmul_rn((float)r1[x + 1], scale))) : 0.0f;
        out[x] = q;
    }
}

__global__ void __launch_bounds__(256) convert_kernel(int W, int H, const float* __restrict__ in,
                                                      float* __restrict__ out, int flag, size_t pitch) {
    const int y = blockIdx.y;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < W; x += gridDim.x * blockDim.x) {
        if (flag) {   // linear -> pitched
            *reinterpret_cast<float*>(reinterpret_cast<char*>(out) + (size_t)y * pitch + (size_t)x * 4) =
                in[(size_t)y * W + x];
        } else {      // pitched -> linear
            out[(size_t)y * W + x] =
                *reinterpret_cast<const float*>(reinterpret_cast<const char*>(in) + (size_t)y * pitch + (size_t)x * 4);
        }
    }
}

}  // namespace

cudaError_t launch_to_float(int W, int H, const uint8_t* src, size_t src_pitch, float* dst, float scale,
                            cudaStream_t s) {
    const dim3 grid((W + 255) / 256, H);
    to_float_kernel<<<grid, 256, 0, s>>>(W, H, src, src_pitch, dst, 4 * (size_t)W, scale);
    return cudaGetLastError();
}

cudaError_t launch_to_float_pitched(int W, int H, const uint8_t* src, size_t src_pitch, float* dst,
                                    size_t dst_pitch, float scale, cudaStream_t s) {
    const dim3 grid((W + 255) / 256, H);
    to_float_kernel<<<grid, 256, 0, s>>>(W, H, src, src_pitch, dst, dst_pitch, scale);
    return cudaGetLastError();
}

cudaError_t launch_to_quad(int W, int H, const uint8_t* src, size_t src_pitch, float4* dst, float scale,
                           cudaStream_t s) {
    const dim3 grid((W + 255) / 256, H);
    to_quad_kernel<<<grid, 256, 0, s>>>(W, H, src, src_pitch, dst, scale);
    return cudaGetLastError();
}

cudaError_t launch_to_half(int W, int H, const uint8_t* src, size_t src_pitch, void* dst, size_t dst_pitch,
                           float scale, cudaStream_t s) {
    const dim3 grid((W + 255) / 256, H);
    to_half_kernel<<<grid, 256, 0, s>>>(W, H, src, src_pitch, reinterpret_cast<__half*>(dst), dst_pitch, scale, 0);
    return cudaGetLastError();
}

cudaError_t launch_to_float_h_pitched(int W, int H, const uint8_t* src, size_t src_pitch, float* dst,
                                     size_t dst_pitch, float scale, cudaStream_t s) {
    const dim3 grid((W + 255) / 256, H);
    to_half_kernel<<<grid, 256, 0, s>>>(W, H, src, src_pitch, reinterpret_cast<__half*>(dst), dst_pitch, scale, 1);
    return cudaGetLastError();
}

cudaError_t launch_to_float_h(int W, int H, const uint8_t* src, size_t src_pitch, float* dst, float scale,
                              cudaStream_t s) {
    const dim3 grid((W + 255) / 256, H);
    to_half_kernel<<<grid, 256, 0, s>>>(W, H, src, src_pitch, reinterpret_cast<__half*>(dst), 0, scale, 1);
    return cudaGetLastError();
}

cudaError_t launch_to_quad_half(int W, int H, const uint8_t* src, size_t src_pitch, float4* dst, float scale,
                                cudaStream_t s) {
    const dim3 grid((W + 255) / 256, H);
    to_quad_half_kernel<<<grid, 256, 0, s>>>(W, H, src, src_pitch, dst, scale);
    return cudaGetLastError();
}

cudaError_t make_source_texture(int W, int H, bool f32, void** buf, size_t* pitch, unsigned long long* tex) {
    cudaError_t e = cudaMallocPitch(buf, pitch, (f32 ? 4 : 2) * (size_t)W, (size_t)H);
    if (e != cudaSuccess) return e;
    cudaResourceDesc rd;
    std::memset(&rd, 0, sizeof rd);
    rd.resType = cudaResourceTypePitch2D;
    rd.res.pitch2D.devPtr = *buf;
    rd.res.pitch2D.desc = f32 ? cudaCreateChannelDesc<float>() : cudaCreateChannelDescHalf();
    rd.res.pitch2D.width = W;
    rd.res.pitch2D.height = H;
    rd.res.pitch2D.pitchInBytes = *pitch;
    cudaTextureDesc td;
    std::memset(&td, 0, sizeof td);
    td.addressMode[0] = td.addressMode[1] = cudaAddressModeBorder;
    td.filterMode = cudaFilterModeLinear;
    td.readMode = cudaReadModeElementType;
    td.normalizedCoords = 0;
    cudaTextureObject_t t = 0;
    e = cudaCreateTextureObject(&t, &rd, &td, nullptr);
    *tex = t;
    return e;
}

cudaError_t launch_convert(int W, int H, const float* in, float* out, int flag, size_t pitch, cudaStream_t s) {
    const dim3 grid((W + 255) / 256, H);
    convert_kernel<<<grid, 256, 0, s>>>(W, H, in, out, flag, pitch);
    return cudaGetLastError();
}

}  // namespace pm
