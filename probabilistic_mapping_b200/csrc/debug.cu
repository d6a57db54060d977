// debug.cu -- exhaustive self-check of the arithmetic shortcuts the FP32 kernels rely on for
// bit-exactness with IEEE operations:
//   [0] rcp_rn(w) == __frcp_rn(w)               for every positive finite float w
//   [1] floor_split(u) == floorf(u)              for every float u in [0, 2^22)
//   [2] div_small(x, d, RN(1/d)) == x / d (IEEE) for every non-negative finite float x and
//       every integer divisor d in [2, 33]
//   [3] rcp_warp2(w) follows its definition      for every float w (both elements)
#include "pm_device.cuh"
#include "pm_stereo.h"

namespace pm {

#ifdef PM_BOUNDS_CHECK
__device__ unsigned long long g_bounds_log[4];
__device__ bool bounds_fail(int site, long long idx, long long n) {
    if (atomicAdd(&g_bounds_log[0], 1ull) == 0) {
        g_bounds_log[1] = (unsigned long long)site;
        g_bounds_log[2] = (unsigned long long)idx;
        g_bounds_log[3] = (unsigned long long)n;
    }
    return false;
}
#endif

namespace {

// definition of rcp_warp2 (see pm_device.cuh)
__device__ float rcp_warp_spec(float w) {
    const float a = fabsf(w);
    if (!(a >= 1.17549435e-38f) || isinf(w)) return nan_f();
    if (a > 8.50705917e37f) return copysignf(0.0f, w);
    return __frcp_rn(w);
}

__device__ bool same_bits_or_nan(float a, float b) {
    return (a != a && b != b) || __float_as_uint(a) == __float_as_uint(b);
}

__global__ void __launch_bounds__(256) check_arith_kernel(uint32_t base, unsigned long long* bad) {
    const uint32_t bits = base + blockIdx.x * blockDim.x + threadIdx.x;
    const float x = __uint_as_float(bits);
    unsigned long long nb[4] = {0, 0, 0, 0};
    {
        const float2 r = rcp_warp2(make_float2(x, __uint_as_float(bits ^ 0x80000000u)));
        if (!same_bits_or_nan(r.x, rcp_warp_spec(x)) || !same_bits_or_nan(r.y, rcp_warp_spec(-x))) nb[3]++;
    }
    if (bits >= 0x7f800000u) {   // the other checks take positive finite floats and zero only
        if (nb[3]) atomicAdd(bad + 3, nb[3]);
        return;
    }
    if (bits != 0 && __float_as_uint(rcp_rn(x)) != __float_as_uint(__frcp_rn(x))) nb[0]++;
    if (x < 4194304.0f) {
        float fu;
        int i;
        floor_split(x, fu, i);
        if (fu != floorf(x) || i != (int)floorf(x)) nb[1]++;
    }
    for (int d = 2; d <= 33; ++d) {
        const float df = (float)d;
        if (__float_as_uint(div_small(x, df, __frcp_rn(df))) != __float_as_uint(__fdiv_rn(x, df))) nb[2]++;
    }
    for (int k = 0; k < 4; ++k)
        if (nb[k]) atomicAdd(bad + k, nb[k]);
}

}  // namespace
}  // namespace pm

extern "C" pm_status pm_debug_check_arith(uint64_t out[4], void* stream) {
    if (!out) return PM_ERR_INVALID_ARGUMENT;
    cudaStream_t s = (cudaStream_t)stream;
    unsigned long long* bad = nullptr;
    if (cudaMalloc(&bad, 4 * sizeof(unsigned long long)) != cudaSuccess) return PM_ERR_OUT_OF_MEMORY;
    pm_status st = PM_OK;
    if (cudaMemsetAsync(bad, 0, 4 * sizeof(unsigned long long), s) != cudaSuccess) st = PM_ERR_CUDA;
    // positive bit patterns; rcp_warp2 takes each one with both signs
    const uint32_t per = 1u << 26;
    for (uint32_t base = 0; st == PM_OK && base < 0x80000000u; base += per) {
        pm::check_arith_kernel<<<per / 256, 256, 0, s>>>(base, bad);
        if (cudaGetLastError() != cudaSuccess) st = PM_ERR_CUDA;
    }
    unsigned long long host[4] = {0, 0, 0, 0};
    if (st == PM_OK && (cudaMemcpyAsync(host, bad, sizeof host, cudaMemcpyDeviceToHost, s) != cudaSuccess ||
                        cudaStreamSynchronize(s) != cudaSuccess))
        st = PM_ERR_CUDA;
    cudaFree(bad);
    for (int k = 0; k < 4; ++k) out[k] = host[k];
    return st;
}

extern "C" pm_status pm_debug_bounds(uint64_t out[4], int reset) {
    if (!out) return PM_ERR_INVALID_ARGUMENT;
#ifdef PM_BOUNDS_CHECK
    unsigned long long host[4] = {0, 0, 0, 0};
    if (cudaDeviceSynchronize() != cudaSuccess ||
        cudaMemcpyFromSymbol(host, pm::g_bounds_log, sizeof host) != cudaSuccess)
        return PM_ERR_CUDA;
    for (int k = 0; k < 4; ++k) out[k] = host[k];
    if (reset) {
        const unsigned long long zero[4] = {0, 0, 0, 0};
        if (cudaMemcpyToSymbol(pm::g_bounds_log, zero, sizeof zero) != cudaSuccess) return PM_ERR_CUDA;
    }
    return PM_OK;
#else
    (void)reset;
    for (int k = 0; k < 4; ++k) out[k] = 0;
    return PM_ERR_UNSUPPORTED;   // the product library has no checks
#endif
}
