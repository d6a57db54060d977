// pm_device.cuh -- device helpers shared by the motion-stereo kernels (sm_100a).
//
// Every FP32 expression that the CPU oracle replays is written with explicit round-to-nearest
// intrinsics (__fmaf_rn, __fmul_rn, __fdiv_rn, __frcp_rn) and the library is compiled with
// -fmad=false, so no multiply-add is contracted behind our back: the FP32 results are
// reproducible bit-for-bit on the CPU.
#pragma once

#include <cuda_fp16.h>
#include <cuda_runtime.h>
#include <stdint.h>

#include "pm_internal.h"

namespace pm {

constexpr unsigned kFull = 0xffffffffu;

// ---- bounds-checked build ---------------------------------------------------------------
// libpm_stereo_checked.so is compiled with -DPM_BOUNDS_CHECK (and relocatable device code, so
// that every kernel shares one record).  In it each checked global access first tests its element
// index against the buffer's extent; a failing index is not accessed.  Every failure is counted,
// and the first failure's site (BoundsSite), index and extent are kept (pm_debug_bounds), so a
// wrong index shows up as a record instead of a fault.  In the product library the test is the
// constant true and compiles away.
#ifdef PM_BOUNDS_CHECK
extern __device__ unsigned long long g_bounds_log[4];   // failures, first site, its index, its extent
__device__ bool bounds_fail(int site, long long idx, long long n);
#define PM_IN_BOUNDS(idx, n, site)                                                        \
    (((unsigned long long)(long long)(idx) < (unsigned long long)(long long)(n)) ||       \
     ::pm::bounds_fail((site), (long long)(idx), (long long)(n)))
#else
#define PM_IN_BOUNDS(idx, n, site) true
#endif
// the elements [e, e + len) lie in [0, n)
#define PM_RANGE_IN_BOUNDS(e, len, n, site) PM_IN_BOUNDS((e), (long long)(n) - (long long)(len) + 1, (site))

__device__ __forceinline__ float nan_f() { return __int_as_float(0x7fffffff); }
__device__ __forceinline__ float inf_f() { return __int_as_float(0x7f800000); }

// pm_stats counters: adds one to each of a thread's words c0, c1, c2 (each in [0, N), or -1 for
// none) of the N global counters at g.  The block's counts meet in shared memory first, then one
// global add per word and block.  Every thread of the block calls it.
template <int N>
__device__ __forceinline__ void tally_block(unsigned* g, int c0, int c1 = -1, int c2 = -1) {
    __shared__ unsigned s[N];
    if (threadIdx.x < N) s[threadIdx.x] = 0u;
    __syncthreads();
    if (c0 >= 0) atomicAdd(&s[c0], 1u);
    if (c1 >= 0) atomicAdd(&s[c1], 1u);
    if (c2 >= 0) atomicAdd(&s[c2], 1u);
    __syncthreads();
    if (threadIdx.x < N && s[threadIdx.x]) atomicAdd(g + threadIdx.x, s[threadIdx.x]);
}

// Homography of one source frame as kernel arguments (the 12 floats of ad_calc_cost,
// calc_cost.cu:212-219).
struct Hom {
    float r11, r12, r13, r21, r22, r23, r31, r32, r33, t1, t2, t3;
};

// Correctly rounded 1/w.  For w in [2^-126, 2^126) one Newton-Raphson step from the hardware
// reciprocal estimate (r1 = r0 + r0 (1 - w r0)) gives exactly RN(1/w); this was checked for
// every float in that range against __frcp_rn (pm_debug_check_arith re-runs the check).
// Outside that range the estimate flushes to zero or infinity, so IEEE reciprocal is used.
__device__ __forceinline__ float rcp_rn(float w) {
    if (w >= 1.17549435e-38f && w < 8.50705917e37f) {
        float r0;
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r0) : "f"(w));
        return __fmaf_rn(r0, __fmaf_rn(-w, r0, 1.0f), r0);
    }
    return __frcp_rn(w);
}

// The warps' reciprocal, without a branch: rcp.approx.ftz plus the same Newton step.  Equal
// to RN(1/w) for 2^-126 <= |w| <= 2^126 (as rcp_rn); NaN for w = +-0, subnormal, infinite or NaN
// w (a warped sample from such a w is rejected); +-0 for larger finite |w|.  The FP32 oracle
// implements exactly this rule; pm_debug_check_arith checks it for every float.
__device__ __forceinline__ float2 rcp_warp2(float2 w) {
    float2 r0;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r0.x) : "f"(w.x));
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r0.y) : "f"(w.y));
    return __ffma2_rn(r0, __ffma2_rn(make_float2(-w.x, -w.y), r0, make_float2(1.0f, 1.0f)), r0);
}

// floor(u) for 0 <= u < 2^22 as (float, int) without a conversion instruction: adding
// 1.5 * 2^23 with rounding toward minus infinity leaves floor(u) in the low mantissa bits.
__device__ __forceinline__ void floor_split(float u, float& fu, int& i) {
    const float t = __fadd_rd(u, 12582912.0f);
    i = __float_as_int(t) - 0x4B400000;
    fu = __fsub_rn(t, 12582912.0f);
}

// Correctly rounded x / d for x >= 0 and an integer divisor d in [2, 33] with r = RN(1/d):
// q0 = RN(x r), then one correction with the exact residual fma(-q0, d, x) (Markstein).  Equal
// to IEEE division whenever x / d is a normal number; smaller x takes the IEEE path.
__device__ __forceinline__ float div_small(float x, float d, float r) {
    if (x != 0.0f && x < 1e-30f) return __fdiv_rn(x, d);
    const float q0 = __fmul_rn(x, r);
    return __fmaf_rn(__fmaf_rn(-q0, d, x), r, q0);
}

__device__ __forceinline__ void homog(const Hom& h, int qu, int qv, float& x, float& y, float& z) {
    const float fu = (float)qu, fv = (float)qv;
    x = __fmaf_rn(h.r11, fu, __fmaf_rn(h.r12, fv, h.r13));
    y = __fmaf_rn(h.r21, fu, __fmaf_rn(h.r22, fv, h.r23));
    z = __fmaf_rn(h.r31, fu, __fmaf_rn(h.r32, fv, h.r33));
}

// Bilinear fetch with texel centres at integer coordinates and zero border, the filtering of
// tex2D(t, u + 0.5f, v + 0.5f) with cudaFilterModeLinear / cudaAddressModeBorder
// (calc_cost.cu:93,230-237), evaluated with exact weights.  Caller guarantees
// 0 <= u <= W-1 and 0 <= v <= H-1, so only the +1 texels can fall outside.
__device__ __forceinline__ float bilinear(const float* __restrict__ img, int W, int H, float u, float v) {
    const float fu = floorf(u), fv = floorf(v);
    const int i = (int)fu, j = (int)fv;
    const float a = __fsub_rn(u, fu), b = __fsub_rn(v, fv);
    const float* row0 = img + (size_t)j * W;
    const bool in_i1 = (i + 1) < W, in_j1 = (j + 1) < H;
    const float t00 = __ldg(row0 + i);
    const float t10 = in_i1 ? __ldg(row0 + i + 1) : 0.0f;
    const float t01 = in_j1 ? __ldg(row0 + W + i) : 0.0f;
    const float t11 = (in_i1 && in_j1) ? __ldg(row0 + W + i + 1) : 0.0f;
    const float top = __fmaf_rn(a, __fsub_rn(t10, t00), t00);
    const float bot = __fmaf_rn(a, __fsub_rn(t11, t01), t01);
    return __fmaf_rn(b, __fsub_rn(bot, top), top);
}

// One warped sample (calc_cost.cu:85-93): w = z + t3*rho, u = (x + t1*rho)/w, v = (y + t2*rho)/w,
// computed as one correctly rounded reciprocal and two products.  Rejected samples (w < 0 or
// (u, v) outside [0, W-1] x [0, H-1], NaN included) return NaN, which then poisons the 9-term sum.
__device__ __forceinline__ float warp_fetch(const float* __restrict__ img, int W, int H, float x, float y,
                                            float z, const Hom& h, float rho) {
    const float w = __fmaf_rn(h.t3, rho, z);
    const float nx = __fmaf_rn(h.t1, rho, x);
    const float ny = __fmaf_rn(h.t2, rho, y);
    const float r = rcp_rn(w);
    const float u = __fmul_rn(nx, r), v = __fmul_rn(ny, r);
    const bool ok = (w >= 0.0f) && (u >= 0.0f) && (u <= (float)(W - 1)) && (v >= 0.0f) &&
                    (v <= (float)(H - 1));
    return ok ? bilinear(img, W, H, u, v) : nan_f();
}

// ---- warp reductions --------------------------------------------------------------------
__device__ __forceinline__ float warp_min_f32(float x) {
    float r;
    asm volatile("redux.sync.min.f32 %0, %1, 0xffffffff;" : "=f"(r) : "f"(x));
    return r;
}

// ---- cp.async (LDGSTS) helpers: a lane copies its own slice into its own shared slot ------
__device__ __forceinline__ uint32_t smem_addr(const void* p) {
    return (uint32_t)__cvta_generic_to_shared(p);
}
__device__ __forceinline__ void cp_async_16(void* smem, const void* gmem) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(smem_addr(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_8(void* smem, const void* gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(smem_addr(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_4(void* smem, const void* gmem) {
    asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(smem_addr(smem)), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N> __device__ __forceinline__ void cp_async_wait() {
    asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory");
}

// Copy BYTES from gmem to smem.  Lane slices start at lane*BYTES, so the piece size is the
// largest of 16/8/4 dividing BYTES: that keeps every piece naturally aligned on both sides.
template <int BYTES> __device__ __forceinline__ void cp_async_bytes(void* smem, const void* gmem) {
    static_assert(BYTES % 4 == 0, "cp.async copies at least 4 aligned bytes");
    constexpr int PIECE = (BYTES % 16 == 0) ? 16 : ((BYTES % 8 == 0) ? 8 : 4);
    char* s = (char*)smem;
    const char* g = (const char*)gmem;
#pragma unroll
    for (int off = 0; off < BYTES; off += PIECE) {
        if constexpr (PIECE == 16) cp_async_16(s + off, g + off);
        else if constexpr (PIECE == 8) cp_async_8(s + off, g + off);
        else cp_async_4(s + off, g + off);
    }
}

// ---- plane vectors: a lane owns PPL consecutive planes -----------------------------------
// CG: through L2 only (ld.global.cg), for data written earlier in the same launch by other blocks.
template <int PPL, bool CG = false> __device__ __forceinline__ void load_planes(float (&v)[PPL], const float* p) {
    if constexpr (PPL % 4 == 0) {
#pragma unroll
        for (int j = 0; j < PPL; j += 4) {
            const float4 t = CG ? __ldcg(reinterpret_cast<const float4*>(p + j)) : *reinterpret_cast<const float4*>(p + j);
            v[j] = t.x; v[j + 1] = t.y; v[j + 2] = t.z; v[j + 3] = t.w;
        }
    } else if constexpr (PPL % 2 == 0) {
#pragma unroll
        for (int j = 0; j < PPL; j += 2) {
            const float2 t = CG ? __ldcg(reinterpret_cast<const float2*>(p + j)) : *reinterpret_cast<const float2*>(p + j);
            v[j] = t.x; v[j + 1] = t.y;
        }
    } else {
#pragma unroll
        for (int j = 0; j < PPL; ++j) v[j] = CG ? __ldcg(p + j) : p[j];
    }
}
template <int PPL> __device__ __forceinline__ void store_planes(float* p, const float (&v)[PPL]) {
    if constexpr (PPL % 4 == 0) {
#pragma unroll
        for (int j = 0; j < PPL; j += 4)
            *reinterpret_cast<float4*>(p + j) = make_float4(v[j], v[j + 1], v[j + 2], v[j + 3]);
    } else if constexpr (PPL % 2 == 0) {
#pragma unroll
        for (int j = 0; j < PPL; j += 2) *reinterpret_cast<float2*>(p + j) = make_float2(v[j], v[j + 1]);
    } else {
#pragma unroll
        for (int j = 0; j < PPL; ++j) p[j] = v[j];
    }
}

}  // namespace pm
