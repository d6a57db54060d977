// cost_device.cuh -- device code of the plane-sweep cost stage (reference: calc_cost.cu:11-253):
// the tile function of cost_kernel and the per-warp rebase of the FP16 volume.  Included by
// cost.cu (the stand-alone kernels) and persist.cu (the batched form's persistent kernel).
#pragma once

#include <type_traits>

#include "pm_device.cuh"

namespace pm {
namespace {


constexpr int TXU = 30;                  // output columns per tile (lanes 1..30)
constexpr int TY = 8;                    // output rows per tile
constexpr int WARPS = 8;                 // one plane pair per warp
constexpr int PCB = 2 * WARPS;           // planes per CTA
constexpr int NT = 32 * WARPS;
constexpr int SP = PCB + 2;              // state pitch: even (8-byte pairs), conflict-free pairs
constexpr int NPIX = TXU * TY;

// Shared layout of a tile.  HC: the counts as FP16 (the FP16 form's first pass, whose counts are
// small integers, exact in FP16): fewer shared bytes per CTA leave more of the SM's L1 to the
// texture cache, which the texture samplers' speed depends on.
template <bool HC> struct SmemL {
    static constexpr size_t REF = 0;                                              // float2 [TY+2][32]
    static constexpr size_t ACC = REF + sizeof(float2) * (TY + 2) * 32;           // float [NPIX][SP]
    static constexpr size_t CNT = ACC + sizeof(float) * NPIX * SP;                // float or half [NPIX][SP]
    static constexpr size_t BYTES = CNT + (HC ? sizeof(__half) : sizeof(float)) * NPIX * SP;
};
using Smem = SmemL<false>;   // the larger layout

__device__ __forceinline__ float ref_at(const float* __restrict__ ref, int W, int H, int x, int y) {
    return (x < 0 || y < 0 || x >= W || y >= H) ? 0.0f : __ldg(ref + (size_t)y * W + x);
}

template <bool HALF> __device__ __forceinline__ void store_cost(void* base, size_t i, float v) {
    if constexpr (HALF) reinterpret_cast<__half*>(base)[i] = __float2half_rn(v);
    else reinterpret_cast<float*>(base)[i] = v;
}
template <bool HALF> __device__ __forceinline__ float load_cost(const void* base, size_t i) {
    if constexpr (HALF) return __half2float(reinterpret_cast<const __half*>(base)[i]);
    else return reinterpret_cast<const float*>(base)[i];
}

// ---- packed FP32x2 helpers --------------------------------------------------------------
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
// a - b as fma(b, -1, a): the product is exact, so this is RN(a - b) without a negation
__device__ __forceinline__ float2 sub2(float2 a, float2 b) { return __ffma2_rn(b, f2(-1.0f, -1.0f), a); }

__device__ __forceinline__ float2 shfl_up2(float2 v) {
    return f2(__shfl_up_sync(kFull, v.x, 1), __shfl_up_sync(kFull, v.y, 1));
}
__device__ __forceinline__ float2 shfl_down2(float2 v) {
    return f2(__shfl_down_sync(kFull, v.x, 1), __shfl_down_sync(kFull, v.y, 1));
}

// Source access: plain float rows, the quad layout (one 16-byte load per bilinear sample; in the
// FP16 form its values are rounded to FP16 but kept in FP32 lanes, since a per-sample conversion
// costs more issue slots than the wider loads cost bandwidth in this issue-bound kernel), or a
// texture object filtered by the texture unit: FP16 form (kTex, FP16 or FP16-rounded FP32 texels,
// hardware reciprocal estimate in the warp) or FP32 form (kTexF, FP32 texels of the images, the
// warp's Newton reciprocal: the reference's own sampler, calc_cost.cu:226-237).
enum { kPlain = 0, kQuad = 1, kTex = 2, kQuadH = 3, kTexF = 4 };
template <int SAMP> struct Src;
template <> struct Src<kPlain> {
    const float* __restrict__ p;
    int W, H;
};
template <> struct Src<kQuad> {
    const float4* __restrict__ q;
    int W, H;
    unsigned off;   // (1.5 * 2^23 bit pattern) * (W + 1), folded out of the quad index
};
template <> struct Src<kTex> {
    cudaTextureObject_t t;
    int W, H;
};
template <> struct Src<kTexF> {
    cudaTextureObject_t t;
    int W, H;
};
template <> struct Src<kQuadH> {   // FP16 form: quads of FP16-rounded values in FP32 lanes
    const float4* __restrict__ q;
    int W, H;
    unsigned off;
};

// Per-source constants of the warps, as packed pairs.
struct WarpConst {
    float2 t1, t2, t3;
    float W1, H1;
};

// The warped sample of one position (x, y, z) at two planes (calc_cost.cu:85-93):
// w = z + t3*rho, u = (x + t1*rho) * r, v = (y + t2*rho) * r with r = rcp_warp2(w) (FP16 form:
// the hardware reciprocal estimate); rejected (NaN) when w < 0 or (u, v) lies outside
// [0, W-1] x [0, H-1] (NaN coordinates included).
template <int SAMP>
__device__ __forceinline__ float2 sample2_core(const Src<SAMP>& src, const WarpConst& c, float2 w, float2 nx,
                                               float2 ny);
template <int SAMP>
__device__ __forceinline__ float2 sample2(const Src<SAMP>& src, const WarpConst& c, float x, float y, float z,
                                          float2 rho) {
    return sample2_core<SAMP>(src, c, __ffma2_rn(c.t3, rho, f2(z, z)), __ffma2_rn(c.t1, rho, f2(x, x)),
                              __ffma2_rn(c.t2, rho, f2(y, y)));
}
// The same from the denominator w and the numerators (nx, ny) of the plane pair.
template <int SAMP>
__device__ __forceinline__ float2 sample2_core(const Src<SAMP>& src, const WarpConst& c, float2 w, float2 nx,
                                               float2 ny) {
    float2 r;
    if constexpr (SAMP == kTex || SAMP == kQuadH) {
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r.x) : "f"(w.x));
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r.y) : "f"(w.y));
    } else {
        r = rcp_warp2(w);
    }
    const float2 u = __fmul2_rn(nx, r), v = __fmul2_rn(ny, r);
    // u + 0 turns -0 into +0 (which the reference's u < 0 accepts); then 0 <= u <= W-1 is one
    // unsigned compare of the bit patterns: negative values and NaN have patterns above W-1's.
    // The FP16 form's warps already use the reciprocal estimate, so it leaves out the +0: a
    // coordinate of exactly -0 (a numerator of -0, which needs rho = 0) is then rejected.
    constexpr bool EXACT = !(SAMP == kTex || SAMP == kQuadH);
    const float2 uz = EXACT ? __fadd2_rn(u, f2(0.0f, 0.0f)) : u, vz = EXACT ? __fadd2_rn(v, f2(0.0f, 0.0f)) : v;
    const unsigned Wb = __float_as_uint(c.W1), Hb = __float_as_uint(c.H1);
    const bool ok0 = (w.x >= 0.0f) && (__float_as_uint(uz.x) <= Wb) && (__float_as_uint(vz.x) <= Hb);
    const bool ok1 = (w.y >= 0.0f) && (__float_as_uint(uz.y) <= Wb) && (__float_as_uint(vz.y) <= Hb);
    if constexpr (SAMP == kTex || SAMP == kTexF) {
        // texel centres at +0.5, as the reference's tex2D(t, u + 0.5f, v + 0.5f) (calc_cost.cu:93),
        // both planes' coordinates in one packed add each
        const float2 uh = __fadd2_rn(u, f2(0.5f, 0.5f)), vh = __fadd2_rn(v, f2(0.5f, 0.5f));
        const float s0 = tex2D<float>(src.t, uh.x, vh.x);
        const float s1 = tex2D<float>(src.t, uh.y, vh.y);
        return f2(ok0 ? s0 : nan_f(), ok1 ? s1 : nan_f());
    } else if constexpr (SAMP == kQuad || SAMP == kQuadH) {
        // 0 <= u, v < 2^22: u + 1.5*2^23 rounded down is 1.5*2^23 + floor(u), exactly, and the
        // integer part sits in the low mantissa bits
        const float2 M = f2(12582912.0f, 12582912.0f);
        const float2 tu = __fadd2_rd(u, M), tv = __fadd2_rd(v, M);
        const float2 a = sub2(u, __fadd2_rn(tu, f2(-12582912.0f, -12582912.0f)));
        const float2 b = sub2(v, __fadd2_rn(tv, f2(-12582912.0f, -12582912.0f)));
        // floor(v) * W + floor(u) in 32-bit arithmetic (exact modulo 2^32, the true value is
        // below W * H); a rejected element reads quad 0 and is replaced by NaN below
        const unsigned i0 = __float_as_uint(tv.x) * (unsigned)src.W + __float_as_uint(tu.x) - src.off;
        const unsigned i1 = __float_as_uint(tv.y) * (unsigned)src.W + __float_as_uint(tu.y) - src.off;
        float2 lo0, hi0, lo1, hi1;
        {
            [[maybe_unused]] const long long nq = (long long)src.W * src.H;
            const bool in0 = !ok0 || PM_IN_BOUNDS(i0, nq, kSiteCostSource);
            const bool in1 = !ok1 || PM_IN_BOUNDS(i1, nq, kSiteCostSource);
            const float4 t0 = __ldg(src.q + (ok0 && in0 ? i0 : 0u));
            const float4 t1 = __ldg(src.q + (ok1 && in1 ? i1 : 0u));
            lo0 = f2(t0.x, t0.y); hi0 = f2(t0.z, t0.w);
            lo1 = f2(t1.x, t1.y); hi1 = f2(t1.z, t1.w);
        }
        // (top, bot) = fma(a, (I(x+1,y), I(x+1,y+1)) - (I(x,y), I(x,y+1)), (I(x,y), I(x,y+1)))
        const float2 p0 = __ffma2_rn(f2(a.x, a.x), sub2(hi0, lo0), lo0);
        const float2 p1 = __ffma2_rn(f2(a.y, a.y), sub2(hi1, lo1), lo1);
        const float s0 = __fmaf_rn(b.x, __fsub_rn(p0.y, p0.x), p0.x);
        const float s1 = __fmaf_rn(b.y, __fsub_rn(p1.y, p1.x), p1.x);
        return f2(ok0 ? s0 : nan_f(), ok1 ? s1 : nan_f());
    } else {
        return f2(ok0 ? bilinear(src.p, src.W, src.H, u.x, v.x) : nan_f(),
                  ok1 ? bilinear(src.p, src.W, src.H, u.y, v.y) : nan_f());
    }
}

__device__ __forceinline__ Hom load_hom(const CostLaunch& a, int s) {
    Hom h;
    if (a.hom_dev) {
        const float* p = a.hom_dev + 12 * s;
        h.r11 = __ldg(p + 0); h.r12 = __ldg(p + 1); h.r13 = __ldg(p + 2);
        h.r21 = __ldg(p + 3); h.r22 = __ldg(p + 4); h.r23 = __ldg(p + 5);
        h.r31 = __ldg(p + 6); h.r32 = __ldg(p + 7); h.r33 = __ldg(p + 8);
        h.t1 = __ldg(p + 9); h.t2 = __ldg(p + 10); h.t3 = __ldg(p + 11);
        return h;
    }
    h.r11 = a.hom[s][0]; h.r12 = a.hom[s][1]; h.r13 = a.hom[s][2];
    h.r21 = a.hom[s][3]; h.r22 = a.hom[s][4]; h.r23 = a.hom[s][5];
    h.r31 = a.hom[s][6]; h.r32 = a.hom[s][7]; h.r33 = a.hom[s][8];
    h.t1 = a.hom[s][9]; h.t2 = a.hom[s][10]; h.t3 = a.hom[s][11];
    return h;
}

// One source's 9-term sums folded into the running state of the two voxels of a plane pair,
// (cnt*last + tmp/9)/(cnt+1) and cnt+1 (calc_cost.cu:205-206); a NaN sum (a rejected sample)
// leaves its voxel unchanged (:89-91).  The first measurement of a voxel (last = -1, cnt = 0)
// comes out as tmp/9 exactly, which is the reference's separate branch (:200-203): every state
// this library writes has cnt = 0 exactly where last < 0.  Both divisions are a
// reciprocal-multiply with one FMA correction (RN(1/9) and the exact Newton reciprocal of
// cnt+1), equal to IEEE division for divisors up to 33 and dividends 0 or >= 1e-30 (the
// exhaustive check of pm_debug_check_arith); outside that the pair takes IEEE division.  A pass
// that starts from initReference (INC false) folds at most kMaxSources sources, so its divisors
// never exceed 33 and only the dividends are tested.
//
// The FP16 form (APPROX) stores the result in FP16, so it folds with one multiply by RN(1/9)
// and the hardware reciprocal estimate of cnt+1 (relative error ~1e-7, far below FP16's
// 4.9e-4) instead of the correctly rounded divisions.
template <bool INC, bool APPROX>
__device__ __forceinline__ void fold2(float2& acc, float2& cn, float2 tmp, float r9) {
    const float2 r9p = f2(r9, r9);
    if constexpr (APPROX) {
        const float2 n1 = __fadd2_rn(cn, f2(1.0f, 1.0f));
        float2 r;
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r.x) : "f"(n1.x));
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r.y) : "f"(n1.y));
        const float2 q = __fmul2_rn(__ffma2_rn(cn, acc, __fmul2_rn(tmp, r9p)), r);
        const bool v0 = tmp.x == tmp.x, v1 = tmp.y == tmp.y;
        acc = f2(v0 ? q.x : acc.x, v1 ? q.y : acc.y);
        cn = f2(v0 ? n1.x : cn.x, v1 ? n1.y : cn.y);
        return;
    }
    const float2 n1 = __fadd2_rn(cn, f2(1.0f, 1.0f));
    const float2 nn1 = __ffma2_rn(cn, f2(-1.0f, -1.0f), f2(-1.0f, -1.0f));   // -(cnt + 1), exact
    const float2 q0 = __fmul2_rn(tmp, r9p);
    const float2 m = __ffma2_rn(__ffma2_rn(q0, f2(-9.0f, -9.0f), tmp), r9p, q0);
    const float2 num = __ffma2_rn(cn, acc, m);
    const float2 r = rcp_warp2(n1);
    const float2 p0 = __fmul2_rn(num, r);
    float2 q = __ffma2_rn(__ffma2_rn(p0, nn1, num), r, p0);
    const bool fast = (!INC || (n1.x <= 33.0f && n1.y <= 33.0f)) && !(tmp.x != 0.0f && tmp.x < 1e-30f) &&
                      !(tmp.y != 0.0f && tmp.y < 1e-30f) && !(num.x != 0.0f && num.x < 1e-30f) &&
                      !(num.y != 0.0f && num.y < 1e-30f);
    if (!fast) {
        q.x = __fdiv_rn(__fmaf_rn(cn.x, acc.x, __fdiv_rn(tmp.x, 9.0f)), n1.x);
        q.y = __fdiv_rn(__fmaf_rn(cn.y, acc.y, __fdiv_rn(tmp.y, 9.0f)), n1.y);
    }
    const bool v0 = tmp.x == tmp.x, v1 = tmp.y == tmp.y;
    acc = f2(v0 ? q.x : acc.x, v1 ? q.y : acc.y);
    cn = f2(v0 ? n1.x : cn.x, v1 ? n1.y : cn.y);
}

// The FP16 form's first pass (from initReference): the state holds the SUM of the sources'
// tmp/9 terms and their count (FP16, exact for counts up to 2048), and the mean is formed once
// when the tile is stored (sum_to_mean); a rejected sum (NaN) adds nothing.  The reference's
// running mean (calc_cost.cu:200-207) and this mean differ only by FP32 rounding, far below the
// FP16 volume's step.
__device__ __forceinline__ void fold2_sum(float2& acc, __half2& cn, float2 tmp, float r9) {
    // a measured sum is >= +0 and a rejected one NaN, so fmaxf(tmp, 0) is the sum or 0 (the
    // maximum drops a NaN operand); 1 + 0 * tmp is 1 or NaN, and its maximum with 0 the count step
    acc = __ffma2_rn(make_float2(fmaxf(tmp.x, 0.0f), fmaxf(tmp.y, 0.0f)), make_float2(r9, r9), acc);
    const float2 one = __ffma2_rn(tmp, make_float2(0.0f, 0.0f), make_float2(1.0f, 1.0f));
    cn = __hadd2(cn, __floats2half2_rn(fmaxf(one.x, 0.0f), fmaxf(one.y, 0.0f)));
}
__device__ __forceinline__ float sum_to_mean(float sum, float cnt) {
    if (cnt == 0.0f) return -1.0f;   // never measured (initReference's -1, stereo_mapper.cpp:69)
    float r;
    asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r) : "f"(cnt));
    return __fmul_rn(sum, r);
}

// MODE 0: reference sample set (calc_cost.cu:83-199); MODE 1: corrected 3x3 patch.
// One CTA's tile (bx, by) and 16-plane block bz of the volume; smem_raw holds Smem::BYTES.
template <int MODE, bool HALF, int SAMP, bool INC>
__device__ __forceinline__ void cost_tile(const CostLaunch& a, int bx, int by, int bz, unsigned char* smem_raw) {
    constexpr bool HC = HALF && !INC;   // sums and FP16 counts
    constexpr bool PM = HALF;           // packed-pair warp coordinates (see the source loop)
    using SM = SmemL<HC>;
    using CntT = typename std::conditional<HC, __half, float>::type;
    float2* const refp = reinterpret_cast<float2*>(smem_raw + SM::REF);
    float* const accs = reinterpret_cast<float*>(smem_raw + SM::ACC);
    CntT* const cnts = reinterpret_cast<CntT*>(smem_raw + SM::CNT);

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int W = a.W, H = a.H, D = a.D;
    const int x0 = bx * TXU, y0 = by * TY, d0 = bz * PCB;
    const int x = x0 - 1 + lane;                              // this lane's column
    const bool out_col = lane >= 1 && lane <= TXU && x < W;   // an output column of the tile

    // reference tile + halo (border addressing -> 0, calc_cost.cu:230-231), each value
    // duplicated as the packed operand of both planes
    for (int i = tid; i < (TY + 2) * 32; i += NT) {
        const int r = i >> 5, l = i & 31;
        const float R = ref_at(a.ref, W, H, x0 - 1 + l, y0 - 1 + r);
        refp[i] = f2(R, R);
    }

    // running state of the tile's voxels, [pixel][plane] with pitch SP: from memory (the
    // state of earlier calls), or the initReference state cost = -1, count = 0
    if constexpr (INC) {
        for (int e = tid; e < NPIX * PCB; e += NT) {
            const int p = e / PCB, k = e - p * PCB;
            float c0 = -1.0f, n0 = 0.0f;   // running mean, count
            const int o = p / TXU, i = p - o * TXU;
            const int gx = x0 + i, gy = y0 + o;
            const size_t g = ((size_t)gy * W + gx) * D + d0 + k;
            if (gx < W && gy < H && PM_IN_BOUNDS(g, (long long)W * H * D, kSiteCostState)) {
                c0 = load_cost<HALF>(a.cost, g);
                if constexpr (HALF) c0 = __fadd_rn(c0, a.offset[(size_t)gy * W + gx]);
                n0 = a.cnt[g];
            }
            accs[p * SP + k] = c0;
            cnts[p * SP + k] = (CntT)n0;
        }
    } else {
        // the whole arrays, pitch padding included, in 16-byte stores: -1 (FP16 form: a sum of
        // 0) and a count of 0, whose FP32 and FP16 bit patterns are both zero
        static_assert((NPIX * SP * sizeof(float)) % 16 == 0 && (NPIX * SP * sizeof(CntT)) % 16 == 0 &&
                          SM::ACC % 16 == 0 && SM::CNT % 16 == 0, "16-byte state stores");
        const float c0 = HC ? 0.0f : -1.0f;
        float4* const av = reinterpret_cast<float4*>(accs);
        for (int i = tid; i < NPIX * SP / 4; i += NT) av[i] = make_float4(c0, c0, c0, c0);
        float4* const cv = reinterpret_cast<float4*>(cnts);
        for (int i = tid; i < (int)(NPIX * SP * sizeof(CntT) / 16); i += NT) cv[i] = make_float4(0.0f, 0.0f, 0.0f, 0.0f);
    }
    __syncthreads();

    const int da = d0 + 2 * warp;   // idep = i * DEP_SAMPLE (calc_cost.cu:81), plus rho0
    const float2 rho = f2(__fmaf_rn((float)da, a.drho, a.rho0), __fmaf_rn((float)(da + 1), a.drho, a.rho0));
    const float r9 = __frcp_rn(9.0f);
    // this lane's state slots (one 8-byte pair per row); lanes outside the output columns never
    // touch them
    float2* const accp = reinterpret_cast<float2*>(accs + (out_col ? lane - 1 : 0) * SP + 2 * warp);
    using CntPair = typename std::conditional<HC, __half2, float2>::type;
    CntPair* const cntp = reinterpret_cast<CntPair*>(cnts + (out_col ? lane - 1 : 0) * SP + 2 * warp);

    for (int s = 0; s < a.nsrc; ++s) {
        Src<SAMP> src;
        if constexpr (SAMP == kQuad || SAMP == kQuadH) {
            src.q = a.srcq + (size_t)s * W * H;
            src.off = 0x4B400000u * (unsigned)(W + 1);
        } else if constexpr (SAMP == kTex || SAMP == kTexF) {
            src.t = a.tex[s];
        } else {
            src.p = a.srcs + (size_t)s * W * H;
        }
        src.W = W;
        src.H = H;
        const Hom h = load_hom(a, s);
        WarpConst c;
        c.t1 = f2(h.t1, h.t1);
        c.t2 = f2(h.t2, h.t2);
        c.t3 = f2(h.t3, h.t3);
        c.W1 = (float)(W - 1);
        c.H1 = (float)(H - 1);
        // FP16 form (PM): the warped coordinates of the plane pair as packed pairs straight from
        // per-source constants.  At row y the denominator and numerators are R*y + A (one packed
        // FMA each: A holds the column's terms and t*rho), and MODE 0's corrupted neighbours 4
        // and 8 are the centre row's x plus constant pairs B and C (one packed add each).  The
        // association differs from the reference's expressions by rounding only, inside the FP16
        // form's tolerance; the FP32 forms keep the reference's expressions bit for bit.
        [[maybe_unused]] float Xc = 0.0f;
        [[maybe_unused]] float2 A1, A2, A3, R12, R22, R32, B1, B2, B3, C1, C2, C3;
        if constexpr (PM) {
            const float fx = (float)x;
            const float2 T1 = __fmul2_rn(c.t1, rho), T2 = __fmul2_rn(c.t2, rho), T3 = __fmul2_rn(c.t3, rho);
            Xc = __fmaf_rn(h.r11, fx, h.r13);
            const float Yc = __fmaf_rn(h.r21, fx, h.r23), Zc = __fmaf_rn(h.r31, fx, h.r33);
            A1 = __fadd2_rn(f2(Xc, Xc), T1);
            A2 = __fadd2_rn(f2(Yc, Yc), T2);
            A3 = __fadd2_rn(f2(Zc, Zc), T3);
            R12 = f2(h.r12, h.r12);
            R22 = f2(h.r22, h.r22);
            R32 = f2(h.r32, h.r32);
            if constexpr (MODE == 0) {
                B1 = __fadd2_rn(f2(h.r11, h.r11), T1);
                B2 = __fadd2_rn(f2(h.r21, h.r21), T2);
                B3 = __fadd2_rn(f2(h.r31, h.r31), T3);
                const float e1 = __fsub_rn(h.r11, h.r12), e2 = __fsub_rn(h.r11, h.r22), e3 = __fsub_rn(h.r11, h.r32);
                C1 = __fadd2_rn(f2(e1, e1), T1);
                C2 = __fadd2_rn(f2(e2, e2), T2);
                C3 = __fadd2_rn(f2(e3, e3), T3);
            }
        }

        // rows r-2 (up) and r-1 (centre) of this column (S) and of its left / right neighbour
        // columns (L / R); row r (down) is computed in the iteration
        float2 Su = f2(0.0f, 0.0f), Sc = Su, Lu = Su, Lc = Su, Ru = Su, Rc = Su;
        float hxc = 0.0f;
#pragma unroll   // unrolled, the rolling row registers are renamed instead of copied
        for (int r = 0; r < TY + 2; ++r) {
            float hx = 0.0f;   // the row's homogeneous x: MODE 0's neighbours of the next output row
            float2 Sd;
            if constexpr (PM) {
                const float fy = (float)(y0 - 1 + r);
                const float2 yy = f2(fy, fy);
                Sd = sample2_core<SAMP>(src, c, __ffma2_rn(R32, yy, A3), __ffma2_rn(R12, yy, A1),
                                        __ffma2_rn(R22, yy, A2));
                if constexpr (MODE == 0) hx = __fmaf_rn(h.r12, fy, Xc);
            } else {
                float hy, hz;
                homog(h, x, y0 - 1 + r, hx, hy, hz);
                Sd = sample2<SAMP>(src, c, hx, hy, hz, rho);
            }
            const float2 Ld = shfl_up2(Sd), Rd_ = shfl_down2(Sd);
            const int o = r - 2;   // output row y0 + o
            if (o >= 0 && out_col && y0 + o < H) {
                const float2* rp = refp + o * 32 + lane;   // up row, this column
                const float2 Ru_ = rp[0], Rc_ = rp[32], Rd = rp[64];
                const float2 Rl = rp[31], Rr = rp[33];
                const float2 Rul = rp[-1], Rru = rp[1], Rld = rp[63], Rdr = rp[65];
                float2 d[9];
                if constexpr (MODE == 0) {
                    // the corrupted neighbours (calc_cost.cu:49-51, 69-71) from the centre's x
                    float2 B4, B8;
                    if constexpr (PM) {
                        const float2 xc = f2(hxc, hxc);
                        B4 = sample2_core<SAMP>(src, c, __fadd2_rn(xc, B3), __fadd2_rn(xc, B1), __fadd2_rn(xc, B2));
                        B8 = sample2_core<SAMP>(src, c, __fadd2_rn(xc, C3), __fadd2_rn(xc, C1), __fadd2_rn(xc, C2));
                    } else {
                        const float xr = __fadd_rn(hxc, h.r11), yr = __fadd_rn(hxc, h.r21), zr = __fadd_rn(hxc, h.r31);
                        const float xru = __fsub_rn(xr, h.r12), yru = __fsub_rn(xr, h.r22), zru = __fsub_rn(xr, h.r32);
                        B4 = sample2<SAMP>(src, c, xr, yr, zr, rho);
                        B8 = sample2<SAMP>(src, c, xru, yru, zru, rho);
                    }
                    d[0] = sub2(Rc_, Sc);    // 0  (:93)
                    d[1] = sub2(Rd, Su);     // 1  warps (u, v-1), reads ref (u, v+1) (:106)
                    d[2] = sub2(Ru_, Sd);    // 2  warps (u, v+1), reads ref (u, v-1) (:119)
                    d[3] = sub2(Rl, Lc);     // 3  (:132)
                    d[4] = sub2(Rr, B4);     // 4  (:145)
                    d[5] = sub2(Rul, Lu);    // 5  (:159)
                    d[6] = sub2(Rdr, Rd_);   // 6  (:172)
                    d[7] = sub2(Rld, Ld);    // 7  (:185)
                    d[8] = sub2(Rru, B8);    // 8  (:198)
                } else {
                    d[0] = sub2(Rc_, Sc);
                    d[1] = sub2(Ru_, Su);
                    d[2] = sub2(Rd, Sd);
                    d[3] = sub2(Rl, Lc);
                    d[4] = sub2(Rr, Rc);
                    d[5] = sub2(Rul, Lu);
                    d[6] = sub2(Rdr, Rd_);
                    d[7] = sub2(Rld, Ld);
                    d[8] = sub2(Rru, Ru);
                }
                // the nine terms in the reference's order, both planes in one packed add each
                float2 t2 = f2(fabsf(d[0].x), fabsf(d[0].y));
#pragma unroll
                for (int k = 1; k < 9; ++k) t2 = __fadd2_rn(t2, f2(fabsf(d[k].x), fabsf(d[k].y)));
                const float tx = t2.x, ty = t2.y;
                float2* const ap = accp + o * (TXU * SP / 2);
                CntPair* const cp = cntp + o * (TXU * SP / 2);
                float2 av = *ap;
                CntPair nv = *cp;
                if constexpr (HC) fold2_sum(av, nv, f2(tx, ty), r9);
                else fold2<INC, HALF>(av, nv, f2(tx, ty), r9);
                *ap = av;
                *cp = nv;
            }
            Su = Sc; Sc = Sd;
            Lu = Lc; Lc = Ld;
            Ru = Rc; Rc = Rd_;
            hxc = hx;
        }
    }

    // store contiguous plane runs of the volume (plane-innermost layout): one thread per pixel
    // and 4 consecutive planes, the 4 threads of a pixel in consecutive lanes of one warp
    __syncthreads();
    constexpr int NQ = NPIX * (PCB / 4);
    static_assert(PCB % 4 == 0 && SP % 2 == 0 && NQ % 32 == 0, "whole warps per pass, 8-byte state pairs");
    // vector stores where the caller's buffers allow them (stage entry points take any pointer)
    const bool vcost = (reinterpret_cast<uintptr_t>(a.cost) & (HALF ? 7 : 15)) == 0;
    const bool vcnt = (reinterpret_cast<uintptr_t>(a.cnt) & 15) == 0;
    for (int e = tid; e < NQ; e += NT) {   // warp-uniform trip count
        const int p = e >> 2, k = (e & 3) * 4;
        const int o = p / TXU, i = p - o * TXU;
        const int gx = x0 + i, gy = y0 + o;
        const size_t g = ((size_t)gy * W + gx) * D + d0 + k;
        const float2 s01 = *reinterpret_cast<const float2*>(accs + p * SP + k);
        const float2 s23 = *reinterpret_cast<const float2*>(accs + p * SP + k + 2);
        float n[4];
        if constexpr (HC) {
            const float2 n01 = __half22float2(*reinterpret_cast<const __half2*>(cnts + p * SP + k));
            const float2 n23 = __half22float2(*reinterpret_cast<const __half2*>(cnts + p * SP + k + 2));
            n[0] = n01.x; n[1] = n01.y; n[2] = n23.x; n[3] = n23.y;
        } else {
            const float2 n01 = *reinterpret_cast<const float2*>(cnts + p * SP + k);
            const float2 n23 = *reinterpret_cast<const float2*>(cnts + p * SP + k + 2);
            n[0] = n01.x; n[1] = n01.y; n[2] = n23.x; n[3] = n23.y;
        }
        float v[4] = {s01.x, s01.y, s23.x, s23.y};
        if constexpr (HC) {   // sums and counts to means
#pragma unroll
            for (int j = 0; j < 4; ++j) v[j] = sum_to_mean(v[j], n[j]);
        }
        const bool in = gx < W && gy < H && PM_RANGE_IN_BOUNDS(g, 4, (long long)W * H * D, kSiteCostState);
        if constexpr (HALF) {
            // per pixel and 16-plane block: the smallest measured cost of the block (0 when none
            // is measured) is stored beside the block, and the half volume holds the differences
            float m = inf_f();
#pragma unroll
            for (int j = 0; j < 4; ++j) m = v[j] >= 0.0f ? fminf(m, v[j]) : m;
            m = fminf(m, __shfl_xor_sync(kFull, m, 1));
            m = fminf(m, __shfl_xor_sync(kFull, m, 2));
            m = m == inf_f() ? 0.0f : m;
            const size_t bo = ((size_t)gy * W + gx) * (D / PCB) + bz;
            if (k == 0 && gx < W && gy < H && PM_IN_BOUNDS(bo, (long long)W * H * (D / PCB), kSiteCostOffset))
                a.block_offset[bo] = m;
            if (in) {
                const __half2 h01 = __floats2half2_rn(__fsub_rn(v[0], m), __fsub_rn(v[1], m));
                const __half2 h23 = __floats2half2_rn(__fsub_rn(v[2], m), __fsub_rn(v[3], m));
                __half2* const dst = reinterpret_cast<__half2*>(reinterpret_cast<__half*>(a.cost) + g);
                if (vcost) {
                    uint2 u;
                    u.x = *reinterpret_cast<const unsigned*>(&h01);
                    u.y = *reinterpret_cast<const unsigned*>(&h23);
                    *reinterpret_cast<uint2*>(dst) = u;
                } else {
                    __half* const hd = reinterpret_cast<__half*>(dst);
                    hd[0] = __low2half(h01); hd[1] = __high2half(h01);
                    hd[2] = __low2half(h23); hd[3] = __high2half(h23);
                }
            }
        } else if (in) {
            float* const dst = reinterpret_cast<float*>(a.cost) + g;
            if (vcost) *reinterpret_cast<float4*>(dst) = make_float4(v[0], v[1], v[2], v[3]);
            else { dst[0] = v[0]; dst[1] = v[1]; dst[2] = v[2]; dst[3] = v[3]; }
        }
        if (in && a.cnt) {
            float* const cd = a.cnt + g;
            if (vcnt) *reinterpret_cast<float4*>(cd) = make_float4(n[0], n[1], n[2], n[3]);
            else { cd[0] = n[0]; cd[1] = n[1]; cd[2] = n[2]; cd[3] = n[3]; }
        }
    }
}

// Moves every 16-plane block of a pixel from its own offset to the pixel's: the smallest block
// offset, or 0 when some plane is unmeasured (negative).  One warp per RB consecutive pixels, lane
// l holding planes [l*PPL, (l+1)*PPL) of each as PPL/2 half pairs, rewritten in place; all RB
// pixels are loaded before any is reduced, to keep more bytes in flight.
constexpr int RB = 4;

// The RB pixels from pix0 on, by one warp.  LDCG: read the volume and block offsets through L2
// only (they were written earlier in the same launch by other CTAs).
template <int PPL, bool LDCG>
__device__ __forceinline__ void rebase_pixels(__half2* __restrict__ cost, const float* __restrict__ boff,
                                              float* __restrict__ off, long npix, int D, long pix0, int lane) {
    const int nb = D >> 4;
    __half2 h[RB][PPL / 2];
    float bl[RB];
#pragma unroll
    for (int r = 0; r < RB; ++r) {
        const long pix = pix0 + r < npix ? pix0 + r : npix - 1;   // a repeated last pixel is rewritten identically
        const __half2* c = cost + ((size_t)pix * D + lane * PPL) / 2;
        const bool in = PM_RANGE_IN_BOUNDS((long long)pix * D + lane * PPL, PPL, (long long)npix * D, kSiteRebase) &&
                        (lane >= nb || PM_IN_BOUNDS((long long)pix * nb + lane, (long long)npix * nb, kSiteRebase));
#pragma unroll
        for (int j = 0; j < PPL / 2; ++j) h[r][j] = !in ? __half2() : LDCG ? __ldcg(c + j) : c[j];
        bl[r] = lane < nb && in ? (LDCG ? __ldcg(boff + (size_t)pix * nb + lane) : __ldg(boff + (size_t)pix * nb + lane))
                                : inf_f();
    }
#pragma unroll
    for (int r = 0; r < RB; ++r) {
        if (pix0 + r >= npix) break;   // warp-uniform
        const long pix = pix0 + r;
        bool neg = false;
#pragma unroll
        for (int j = 0; j < PPL / 2; ++j) {
            const float2 v = __half22float2(h[r][j]);
            neg |= v.x < 0.0f || v.y < 0.0f;
        }
        const float g = __any_sync(kFull, neg) ? 0.0f : warp_min_f32(bl[r]);
        __half2* c = cost + ((size_t)pix * D + lane * PPL) / 2;
        const bool in = PM_RANGE_IN_BOUNDS((long long)pix * D + lane * PPL, PPL, (long long)npix * D, kSiteRebase);
#pragma unroll
        for (int j = 0; j < PPL / 2; ++j) {
            const float2 v = __half22float2(h[r][j]);
            const float s0 = __fsub_rn(__shfl_sync(kFull, bl[r], (lane * PPL + 2 * j) >> 4), g);
            const float s1 = __fsub_rn(__shfl_sync(kFull, bl[r], (lane * PPL + 2 * j + 1) >> 4), g);
            if (in) c[j] = __floats2half2_rn(__fadd_rn(v.x, s0), __fadd_rn(v.y, s1));
        }
        if (lane == 0) off[pix] = g;
    }
}

}  // namespace
}  // namespace pm
