// sgm_device.cuh -- device code of the SGM stage (reference: sgm.cu:5-135, filter_cost.cu:3-70):
// the path recurrences, the opposite-path pair block, and the pixel-range combine with the
// winner-take-all.  Included by sgm.cu (the stand-alone kernels) and persist.cu (the batched
// form's persistent kernel).
#pragma once

#include <climits>

#include "pm_device.cuh"

namespace pm {
namespace {

// Path r of the reference order (L->R, R->L, T->B, B->T, then TL->BR, BR->TL, TR->BL, BL->TR);
// pair p = paths (2p, 2p+1) runs along direction pair_dir(p) = the direction of path 2p.
__host__ __device__ inline void pair_dir(int p, int& dx, int& dy) {
    dx = p == 1 ? 0 : 1;
    dy = p == 0 ? 0 : 1;
    if (p == 3) dx = -1;
}

constexpr int PF = 8;      // prefetch distance in pixel steps

struct Chain {
    int x, y, n;
};

__host__ __device__ inline int num_chains(int dx, int dy, int W, int H) {
    return dy == 0 ? H : (dx == 0 ? W : W + H - 1);
}

// Start pixel of chain c: pixels whose predecessor (x-dx, y-dy) lies outside the image.
__device__ __forceinline__ Chain chain_start(int c, int dx, int dy, int W, int H) {
    int x, y;
    if (dy == 0) { x = dx > 0 ? 0 : W - 1; y = c; }
    else if (dx == 0) { x = c; y = dy > 0 ? 0 : H - 1; }
    else if (c < W) { x = c; y = dy > 0 ? 0 : H - 1; }
    else { x = dx > 0 ? 0 : W - 1; y = dy > 0 ? (c - W + 1) : (c - W); }
    const int nx = dx > 0 ? W - x : (dx < 0 ? x + 1 : INT_MAX);
    const int ny = dy > 0 ? H - y : (dy < 0 ? y + 1 : INT_MAX);
    return {x, y, nx < ny ? nx : ny};
}

__device__ __forceinline__ float min3f(float a, float b, float c) {
    float r;
    asm("min.f32 %0, %1, %2, %3;" : "=f"(r) : "f"(a), "f"(b), "f"(c));
    return r;
}

// value of plane d (warp-uniform) from the lane that owns it
template <int PPL> __device__ __forceinline__ float plane_value(const float (&s)[PPL], int d) {
    const int j = d % PPL;
    float v = s[0];
#pragma unroll
    for (int t = 1; t < PPL; ++t) v = (j == t) ? s[t] : v;
    return __shfl_sync(kFull, v, d / PPL);
}

// This lane's entries of the plane-order table, through shared memory.  Read straight from the
// kernel parameters with a lane-dependent index they become indexed constant-cache loads, which
// serialise per distinct address and which the compiler re-issues inside the pixel loop.
template <int PPL>
__device__ __forceinline__ void lane_order(const PlaneOrder& o, int lane, uint32_t& incl, uint16_t (&rk)[PPL]) {
    __shared__ uint32_t s_incl[32];
    __shared__ uint16_t s_rank[kMaxPlanes];
    for (int i = threadIdx.x; i < kMaxPlanes; i += blockDim.x) s_rank[i] = o.rank[i];
    if (threadIdx.x < 32) s_incl[threadIdx.x] = o.incl[threadIdx.x];
    __syncthreads();
    incl = s_incl[lane];
#pragma unroll
    for (int j = 0; j < PPL; ++j) rk[j] = s_rank[lane * PPL + j];
}

// |x| < FLOAT_EPS evaluated in double, as the reference's float-against-double compares
// (filter_cost.cu:37, stereo_mapper.cpp:651): RN_float(1e-5) = 9.99999974737875e-06 lies below
// 1e-5 and the next float above it, so (double)x < 1e-5 holds exactly when x <= that float.
constexpr float kFloatEpsBelow = 9.99999974737875e-06f;
__device__ __forceinline__ bool below_eps(float x) { return x <= kFloatEpsBelow; }
__device__ __forceinline__ bool within_eps(float x) { return x <= kFloatEpsBelow && x >= -kFloatEpsBelow; }

// Winner-take-all with the reference tree's tie-break, then the three rejection rules and
// the parabola subpixel refinement (filter_cost.cu:22-52), plus the optional uniqueness test.
template <int PPL>
__device__ __forceinline__ void wta_filter(const float (&s)[PPL], uint32_t incl, const uint16_t (&rk)[PPL],
                                           int lane, int D, const FilterParams& fp, float& depth_out,
                                           int& idx_out, int& cls_out) {
    float lmin = inf_f();
#pragma unroll
    for (int j = 0; j < PPL; ++j)
        if ((incl >> j) & 1u) lmin = fminf(lmin, s[j]);
    const float mn = warp_min_f32(lmin);
    unsigned lr = 0xffffffffu;
    int lj = 0;
#pragma unroll
    for (int j = 0; j < PPL; ++j)
        if (((incl >> j) & 1u) && s[j] == mn && rk[j] < lr) { lr = rk[j]; lj = j; }
    const unsigned r = __reduce_min_sync(kFull, lr);
    const unsigned ball = __ballot_sync(kFull, lr == r);
    const int idx = __shfl_sync(kFull, lane * PPL + lj, __ffs(ball) - 1);

    float depth;
    int cls = kWtaDepth;
    if (within_eps(mn)) {
        depth = kDepInf;                                   // non-overlap (:37-38)
        cls = kWtaNoOverlap;
    } else if (idx == 0 || idx == D - 1) {
        depth = 0.0f;                                      // border plane (:39-40)
        cls = kWtaBorder;
    } else {
        const float pre = plane_value(s, idx - 1), post = plane_value(s, idx + 1);
        if (__fadd_rn(pre, post) < __fmul_rn(__fmul_rn(2.0f, mn), fp.var_scale)) {
            depth = 0.0f;                                  // flat minimum (:41-42)
            cls = kWtaFlat;
        } else {
            bool reject = false;
            if (fp.uniq > 0.0f && fp.uniq < 1.0f) {
                float l2 = inf_f();
#pragma unroll
                for (int j = 0; j < PPL; ++j) {
                    const int d = lane * PPL + j;
                    if (((incl >> j) & 1u) && (d < idx - 1 || d > idx + 1)) l2 = fminf(l2, s[j]);
                }
                const float second = warp_min_f32(l2);
                reject = mn > __fmul_rn(fp.uniq, second);
            }
            if (reject) {
                depth = 0.0f;
                cls = kWtaAmbiguous;
            } else {                                       // parabola (:45-51)
                const float a2 = __fadd_rn(__fsub_rn(pre, __fmul_rn(2.0f, mn)), post);
                const float b = __fadd_rn(-pre, post);
                const float sub = __fsub_rn((float)idx, __fdiv_rn(b, __fmul_rn(2.0f, a2)));
                depth = rcp_rn(__fmaf_rn(sub, fp.drho, fp.rho0));
            }
        }
    }
    depth_out = depth;
    idx_out = idx;
    cls_out = cls;
}

// The debug winner-take-all of outputFusionCPU's CASE 0 and CASE 1 (stereo_mapper.cpp:636-660,
// 680-704): planes scanned in order from a minimum of 100000, the first strictly smaller value
// wins (so ties go to the lower plane); |min| < FLOAT_EPS gives 10000, the first and last plane
// give 0, otherwise the depth of the plane itself, 1 / (rho0 + d * drho), without subpixel
// refinement.  When no plane is below 100000 the reference leaves its index unset; plane 0 (and
// so 0) is reported here.
template <int PPL>
__device__ __forceinline__ void case_argmin(const float (&s)[PPL], int lane, int D, const FilterParams& fp,
                                            float& out, int& idx_out) {
    float m = 100000.0f;
    unsigned mi = 0xffffffffu;
#pragma unroll
    for (int j = 0; j < PPL; ++j)
        if (s[j] < m) { m = s[j]; mi = (unsigned)(lane * PPL + j); }
    const float mn = warp_min_f32(m);
    const unsigned r = __reduce_min_sync(kFull, m == mn ? mi : 0xffffffffu);
    const int idx = r < (unsigned)D ? (int)r : 0;
    float v;
    if (below_eps(mn)) v = kCaseInf;
    else if (idx == 0 || idx == D - 1) v = 0.0f;
    else v = rcp_rn(__fmaf_rn((float)idx, fp.drho, fp.rho0));
    out = v;
    idx_out = idx;
}

template <bool HALF> struct CostElem;
template <> struct CostElem<false> { using T = float; };
template <> struct CostElem<true> { using T = __half; };

// Ring stage of a warp: for each of its two chains the 32 lanes' cost slices of one step.
template <int PPL, bool HALF> struct Ring {
    static constexpr int CB = PPL * (int)sizeof(typename CostElem<HALF>::T);
    static constexpr int CHAIN_B = 32 * CB;
    static constexpr int STAGE_B = 2 * CHAIN_B;
};

template <int PPL, bool HALF, bool CG = false>
__device__ __forceinline__ void load_slice(float (&cv)[PPL], const unsigned char* p) {
    if constexpr (HALF) {
        const __half2* hp = reinterpret_cast<const __half2*>(p);
#pragma unroll
        for (int j = 0; j < PPL / 2; ++j) {
            const float2 v = __half22float2(CG ? __ldcg(hp + j) : hp[j]);
            cv[2 * j] = v.x;
            cv[2 * j + 1] = v.y;
        }
    } else {
        load_planes<PPL, CG>(cv, reinterpret_cast<const float*>(p));
    }
}

// Adds v to p[0..PPL) in global memory with vector float reductions (no result returned).
template <int PPL> __device__ __forceinline__ void red_planes(float* p, const float (&v)[PPL]) {
    if constexpr (PPL % 4 == 0) {
#pragma unroll
        for (int j = 0; j < PPL; j += 4)
            asm volatile("red.global.add.v4.f32 [%0], {%1, %2, %3, %4};" ::"l"(p + j), "f"(v[j]), "f"(v[j + 1]),
                         "f"(v[j + 2]), "f"(v[j + 3])
                         : "memory");
    } else if constexpr (PPL % 2 == 0) {
#pragma unroll
        for (int j = 0; j < PPL; j += 2)
            asm volatile("red.global.add.v2.f32 [%0], {%1, %2};" ::"l"(p + j), "f"(v[j]), "f"(v[j + 1]) : "memory");
    } else {
#pragma unroll
        for (int j = 0; j < PPL; ++j) asm volatile("red.global.add.f32 [%0], %1;" ::"l"(p + j), "f"(v[j]) : "memory");
    }
}

// The FP16 form's pair volumes: the lane's planes rounded to FP16 (round to nearest) and stored,
// or added to what is stored with packed FP16 reductions (the sum rounded to FP16, no flush).
template <int PPL> __device__ __forceinline__ void pack_h(uint32_t (&w)[PPL / 2], const float (&v)[PPL]) {
    static_assert(PPL % 2 == 0, "FP16 pair volumes need an even number of planes per lane");
#pragma unroll
    for (int j = 0; j < PPL / 2; ++j) {
        const __half2 h = __floats2half2_rn(v[2 * j], v[2 * j + 1]);
        w[j] = *reinterpret_cast<const uint32_t*>(&h);
    }
}
template <int PPL> __device__ __forceinline__ void store_planes_h(__half* p, const float (&v)[PPL]) {
    uint32_t w[PPL / 2];
    pack_h<PPL>(w, v);
    if constexpr (PPL == 8) {
        *reinterpret_cast<uint4*>(p) = make_uint4(w[0], w[1], w[2], w[3]);
    } else if constexpr (PPL == 4) {
        *reinterpret_cast<uint2*>(p) = make_uint2(w[0], w[1]);
    } else {
#pragma unroll
        for (int j = 0; j < PPL / 2; ++j) reinterpret_cast<uint32_t*>(p)[j] = w[j];
    }
}
template <int PPL> __device__ __forceinline__ void red_planes_h(__half* p, const float (&v)[PPL]) {
    uint32_t w[PPL / 2];
    pack_h<PPL>(w, v);
    if constexpr (PPL == 8) {
        asm volatile("red.global.add.noftz.v4.f16x2 [%0], {%1, %2, %3, %4};" ::"l"(p), "r"(w[0]), "r"(w[1]),
                     "r"(w[2]), "r"(w[3])
                     : "memory");
    } else if constexpr (PPL == 4) {
        asm volatile("red.global.add.noftz.v2.f16x2 [%0], {%1, %2};" ::"l"(p), "r"(w[0]), "r"(w[1]) : "memory");
    } else {
#pragma unroll
        for (int j = 0; j < PPL / 2; ++j)
            asm volatile("red.global.add.noftz.f16x2 [%0], %1;" ::"l"(p + 2 * j), "r"(w[j]) : "memory");
    }
}
// The meeting pixel of an odd chain in an FP16 pair volume: both paths' values rounded to FP16
// and added in FP16, as the reduction does for the other pixels.
template <int PPL> __device__ __forceinline__ void add_h(float (&o)[PPL], const float (&a)[PPL], const float (&b)[PPL]) {
#pragma unroll
    for (int j = 0; j < PPL; ++j) o[j] = __half2float(__hadd(__float2half_rn(a[j]), __float2half_rn(b[j])));
}

// Recurrence state of one path along one scanline, and the adaptive-penalty flags of the 32
// steps of the current batch (bit i: step k0 + i has a reference-image gradient below tau).
template <int PPL> struct PathState {
    float L[PPL];
    float mprev;
    unsigned qmask;
};

// a + b for the planes of a lane, two at a time on the packed FP32x2 pipe (each element rounds
// as the scalar add does).
template <int PPL>
__device__ __forceinline__ void add_planes(float (&o)[PPL], const float (&a)[PPL], const float (&b)[PPL]) {
#pragma unroll
    for (int j = 0; j + 1 < PPL; j += 2) {
        const float2 r = __fadd2_rn(make_float2(a[j], a[j + 1]), make_float2(b[j], b[j + 1]));
        o[j] = r.x;
        o[j + 1] = r.y;
    }
    if constexpr (PPL % 2) o[PPL - 1] = __fadd_rn(a[PPL - 1], b[PPL - 1]);
}
template <int PPL> __device__ __forceinline__ void add_planes(float (&o)[PPL], const float (&a)[PPL], float b) {
#pragma unroll
    for (int j = 0; j + 1 < PPL; j += 2) {
        const float2 r = __fadd2_rn(make_float2(a[j], a[j + 1]), make_float2(b, b));
        o[j] = r.x;
        o[j + 1] = r.y;
    }
    if constexpr (PPL % 2) o[PPL - 1] = __fadd_rn(a[PPL - 1], b);
}

// Smallest of the lane's planes that take part in the minimum (all of them when FULL).
template <int PPL, bool FULL> __device__ __forceinline__ float lane_min(const float (&v)[PPL], uint32_t incl) {
    if constexpr (FULL) {
        float m = v[0];
        int j = 1;
#pragma unroll
        for (; j + 1 < PPL; j += 2) m = min3f(m, v[j], v[j + 1]);
        if (j < PPL) m = fminf(m, v[j]);
        return m;
    } else {
        float m = inf_f();
#pragma unroll
        for (int j = 0; j < PPL; ++j)
            if ((incl >> j) & 1u) m = fminf(m, v[j]);
        return m;
    }
}

// Whether the pixel has a plane that was never measured (cost < 0): the path treats its cost as 0
// and outputs COST_INF = 0 there (sgm.cu:33-38, 67-71, 101-104).
template <int PPL, bool FULL> __device__ __forceinline__ bool pixel_invalid(const float (&cv)[PPL], uint32_t incl) {
    return __any_sync(kFull, lane_min<PPL, FULL>(cv, incl) < 0.0f);
}

// First pixel of a path: L = C, or 0 on an invalid pixel (sgm.cu:21-43).
template <int PPL, bool FULL>
__device__ __forceinline__ void path_first(PathState<PPL>& s, const float (&cv)[PPL], uint32_t incl, float (&o)[PPL]) {
    const bool inv = pixel_invalid<PPL, FULL>(cv, incl);
#pragma unroll
    for (int j = 0; j < PPL; ++j) s.L[j] = o[j] = inv ? 0.0f : cv[j];
    s.mprev = warp_min_f32(lane_min<PPL, FULL>(s.L, incl));
}

// One pixel step of a path (sgm.cu:57-108): L(p, d) = C(p, d) + min(L(p-r, d), L(p-r, d+-1) + P1,
// min_k L(p-r, k) + P2) - min_k L(p-r, k), P1/P2 scaled by q1/q2 when the flag q says the
// reference image's path gradient is below tau; a plane never measured makes the pixel invalid:
// its cost counts as 0 and the path's output there is COST_INF = 0.  o receives the output.
template <int PPL, bool FULL>
__device__ __forceinline__ void path_step(const SgmLaunch& a, PathState<PPL>& s, const float (&cv)[PPL], bool q,
                                          float p1q, float p2q, uint32_t incl, int lane, float (&o)[PPL]) {
    const bool inv = pixel_invalid<PPL, FULL>(cv, incl);
    const float P1 = q ? p1q : a.p1, P2 = q ? p2q : a.p2;
    const float mP2 = __fadd_rn(s.mprev, P2);
    float lm = __shfl_up_sync(kFull, s.L[PPL - 1], 1);
    float lp = __shfl_down_sync(kFull, s.L[0], 1);
    if (lane == 0) lm = inf_f();
    if (lane == 31) lp = inf_f();
    // min(L[d], minL + P2, L[d-1] + P1, L[d+1] + P1) (sgm.cu:85-92); min(a+P1, b+P1) is
    // min(a, b) + P1 exactly because rounding is monotonic
    float nb[PPL], cz[PPL], vv[PPL];
#pragma unroll
    for (int j = 0; j < PPL; ++j) {
        nb[j] = fminf(j == 0 ? lm : s.L[j - 1], j == PPL - 1 ? lp : s.L[j + 1]);
        cz[j] = inv ? 0.0f : cv[j];
    }
    add_planes<PPL>(nb, nb, P1);
#pragma unroll
    for (int j = 0; j < PPL; ++j) vv[j] = min3f(s.L[j], mP2, nb[j]);
    add_planes<PPL>(vv, cz, vv);               // C + val
    add_planes<PPL>(s.L, vv, -s.mprev);        // - minL (:98); the negation is exact
#pragma unroll
    for (int j = 0; j < PPL; ++j) o[j] = inv ? 0.0f : s.L[j];
    s.mprev = warp_min_f32(lane_min<PPL, FULL>(s.L, incl));
}

// Reference intensity of step k of a chain starting at pixel p0 (0 past its end).
__device__ __forceinline__ float chain_ref(const float* __restrict__ ref, long p0, long step, int k, int n,
                                           long npix) {
    return k < n && PM_IN_BOUNDS(p0 + (long)k * step, npix, kSitePairRef) ? __ldg(ref + p0 + (long)k * step) : 0.0f;
}

// The flags |I(k) - I(k-1)| < tau of the 32 steps k0 .. k0+31 of one chain as a ballot (bit i:
// step k0 + i).  Lane i holds I(k0 + i) in `cur` (read one batch ahead into `nxt`, which is
// then refilled with I(k0 + 64 + i)); `last` carries I(k0 - 1).
__device__ __forceinline__ unsigned penalty_flags(float& cur, float& nxt, const float* __restrict__ ref, long p0,
                                                  long step, int k0, int n, int lane, float tau, float& last,
                                                  long npix) {
    const float I = cur;
    cur = nxt;
    nxt = chain_ref(ref, p0, step, k0 + 64 + lane, n, npix);
    float prev = __shfl_up_sync(kFull, I, 1);
    if (lane == 0) prev = last;
    last = __shfl_sync(kFull, I, 31);
    return __ballot_sync(kFull, fabsf(__fsub_rn(I, prev)) < tau);
}

// A pair of opposite paths along the same scanlines: warp c takes scanline c of direction
// (dx, dy) and walks it from both ends at once into the pair's volume part[slot / 2]: while the
// two ends have not met, each stores its pixel's path values; after they have, each adds its
// values to what the other end stored there; at the meeting pixel of an odd chain the two are
// added in registers.  The two recurrences are independent, so each warp keeps two dependency
// chains in flight.  The cost slices of both ends are streamed PF steps ahead with cp.async into
// a per-warp shared ring; the reference pixels are read 32 steps at a time (one per lane, a batch
// ahead) and turned into one ballot of penalty flags.  The loop is split at the meeting point,
// so the store and the reduction phases run without a per-step branch.  HOUT: FP16 pair volume.
// One block of NW warps: scanlines bx*NW .. bx*NW + NW-1; `ring` holds NW * PF * STAGE_B bytes.
template <int PPL, bool HALF, int NW, bool FULL, bool HOUT>
__device__ __forceinline__ void sgm_pair_block(const SgmLaunch& a, int dx, int dy, int slot, int bx,
                                               unsigned char* ring) {
    using CT = typename CostElem<HALF>::T;
    using OT = typename CostElem<HOUT>::T;
    using RG = Ring<PPL, HALF>;
    constexpr int CB = RG::CB, CHAIN_B = RG::CHAIN_B, STAGE_B = RG::STAGE_B;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int W = a.W, H = a.H, D = a.D;
    const int c = bx * NW + warp;
    if (c >= num_chains(dx, dy, W, H)) return;        // warp-uniform; no block barriers below
    const Chain ch = chain_start(c, dx, dy, W, H);
    const int n = ch.n;
    const long step = (long)dy * W + dx;
    const long pf0 = (long)ch.y * W + ch.x;             // forward start
    const long pb0 = pf0 + (long)(n - 1) * step;        // backward start (the forward end)
    const long gstep = step * D;                         // elements per step in the volumes

    unsigned char* const wbase = ring + (size_t)warp * PF * STAGE_B;
    const CT* const cf0 = reinterpret_cast<const CT*>(a.cost) + (size_t)pf0 * D + lane * PPL;
    const CT* const cb0 = reinterpret_cast<const CT*>(a.cost) + (size_t)pb0 * D + lane * PPL;
    OT* const out = static_cast<OT*>(a.part[slot >> 1]);
    OT* qf = out + (size_t)pf0 * D + lane * PPL;        // the current step's output slices
    OT* qb = out + (size_t)pb0 * D + lane * PPL;
    const long npix = (long)W * H;
    [[maybe_unused]] const long long nvox = (long long)npix * D;
    auto put = [&](OT* q, const float (&v)[PPL]) {
        if (!PM_RANGE_IN_BOUNDS(q - out, PPL, nvox, kSitePairOut)) return;
        if constexpr (HOUT) store_planes_h<PPL>(q, v);
        else store_planes<PPL>(q, v);
    };
    auto add = [&](OT* q, const float (&v)[PPL]) {
        if (!PM_RANGE_IN_BOUNDS(q - out, PPL, nvox, kSitePairOut)) return;
        if constexpr (HOUT) red_planes_h<PPL>(q, v);
        else red_planes<PPL>(q, v);
    };
    auto meet = [](float (&o)[PPL], const float (&b)[PPL]) {   // o = o + b at the meeting pixel
        if constexpr (HOUT) {
            add_h<PPL>(o, o, b);
        } else {
#pragma unroll
            for (int j = 0; j < PPL; ++j) o[j] = __fadd_rn(o[j], b[j]);
        }
    };

    auto issue = [&](unsigned char* sb, int k) {
        [[maybe_unused]] const CT* const base = reinterpret_cast<const CT*>(a.cost);
        if (PM_RANGE_IN_BOUNDS(cf0 + (long)k * gstep - base, PPL, nvox, kSitePairLoad))
            cp_async_bytes<CB>(sb + lane * CB, cf0 + (long)k * gstep);
        if (PM_RANGE_IN_BOUNDS(cb0 - (long)k * gstep - base, PPL, nvox, kSitePairLoad))
            cp_async_bytes<CB>(sb + CHAIN_B + lane * CB, cb0 - (long)k * gstep);
    };
#pragma unroll 1
    for (int k = 0; k < PF; ++k) {
        if (k < n) issue(wbase + k * STAGE_B, k);
        cp_async_commit();
    }

    uint32_t incl = kFull;
    if constexpr (!FULL) incl = a.order.incl[lane];
    const float p1q = __fmul_rn(a.p1, a.q1), p2q = __fmul_rn(a.p2, a.q2);
    PathState<PPL> fs, bs;
    float lastf = 0.0f, lastb = 0.0f;
    // intensities of steps lane and 32 + lane of both chains; then the flags of steps 0..31
    float If = chain_ref(a.ref, pf0, step, lane, n, npix), Ifn = chain_ref(a.ref, pf0, step, 32 + lane, n, npix);
    float Ib = chain_ref(a.ref, pb0, -step, lane, n, npix), Ibn = chain_ref(a.ref, pb0, -step, 32 + lane, n, npix);
    fs.qmask = penalty_flags(If, Ifn, a.ref, pf0, step, 0, n, lane, a.tau, lastf, npix);
    bs.qmask = penalty_flags(Ib, Ibn, a.ref, pb0, -step, 0, n, lane, a.tau, lastb, npix);

    // step 0: the first pixel of both paths
    cp_async_wait<PF - 1>();
    {
        float cf[PPL], cb[PPL], of[PPL], ob[PPL];
        load_slice<PPL, HALF>(cf, wbase + lane * CB);
        load_slice<PPL, HALF>(cb, wbase + CHAIN_B + lane * CB);
        path_first<PPL, FULL>(fs, cf, incl, of);
        path_first<PPL, FULL>(bs, cb, incl, ob);
        if (n == 1) {
            meet(of, ob);
            put(qf, of);
        } else {
            put(qf, of);
            put(qb, ob);
        }
        if (PF < n) issue(wbase, PF);
        cp_async_commit();
    }
    int st = PF > 1 ? 1 : 0;

    // steps 1 .. n-1: the first visits (stores), the meeting pixel of an odd chain, then the
    // second visits (reductions)
    auto body = [&](int k, float (&of)[PPL], float (&ob)[PPL]) {
        qf += gstep;
        qb -= gstep;
        if ((k & 31) == 0) {
            fs.qmask = penalty_flags(If, Ifn, a.ref, pf0, step, k, n, lane, a.tau, lastf, npix);
            bs.qmask = penalty_flags(Ib, Ibn, a.ref, pb0, -step, k, n, lane, a.tau, lastb, npix);
        }
        cp_async_wait<PF - 1>();
        unsigned char* sb = wbase + st * STAGE_B;
        float cf[PPL], cb[PPL];
        load_slice<PPL, HALF>(cf, sb + lane * CB);
        load_slice<PPL, HALF>(cb, sb + CHAIN_B + lane * CB);
        const int bit = k & 31;
        path_step<PPL, FULL>(a, fs, cf, (fs.qmask >> bit) & 1u, p1q, p2q, incl, lane, of);
        path_step<PPL, FULL>(a, bs, cb, (bs.qmask >> bit) & 1u, p1q, p2q, incl, lane, ob);
        // refill this stage (consumed above) with step k + PF
        if (k + PF < n) issue(sb, k + PF);
        cp_async_commit();
        st = (st + 1 == PF) ? 0 : st + 1;
    };
    const int half = n >> 1;   // steps k < half are first visits of both ends
#pragma unroll 1
    for (int k = 1; k < half; ++k) {
        float of[PPL], ob[PPL];
        body(k, of, ob);
        put(qf, of);
        put(qb, ob);
    }
    int k = half > 1 ? half : 1;
    if ((n & 1) && n > 1) {   // both ends on the middle pixel (k == half)
        float of[PPL], ob[PPL];
        body(k, of, ob);
        meet(of, ob);
        put(qf, of);
        ++k;
    }
#pragma unroll 1
    for (; k < n; ++k) {   // second visits: the first ones were this warp's own stores
        float of[PPL], ob[PPL];
        body(k, of, ob);
        add(qf, of);
        add(qb, ob);
    }
    cp_async_wait<0>();
}

// Sum of the NP pair volumes (each P_2p + P_2p+1) in the order (P0 + P1) + (P2 + P3)
// [+ ((P4 + P5) + (P6 + P7))], then the winner-take-all filter (MODE kCombineFilter), the debug
// argmin (kCombineArgmin) or only a store of the sum (kCombineStore).  One warp per pixel: the
// calling warp takes pixels first, first + nw, ... below npix; the next pixel's slices are loaded
// before the current one is reduced.  Every thread of the block calls it (the plane-order table
// goes through shared memory).  CG: read the pair volumes and offsets through L2 only (written
// earlier in the same launch by other blocks).
template <int PPL, int MODE, int NP, bool HIN, bool CG>
__device__ __forceinline__ void combine_pixels(const SgmLaunch& a, long first, long nw, long npix) {
    const int lane = threadIdx.x & 31;
    const int D = a.D;
    uint32_t incl;
    uint16_t rk[PPL];
    lane_order<PPL>(a.order, lane, incl, rk);
    // raw 32-bit words of the lane's slice of each pair volume (FP16 pairs: two planes per word);
    // the FP16 volumes are half the bytes per pixel, so PD pixels are kept in flight instead of one
    constexpr int WPP = HIN ? PPL / 2 : PPL;
    constexpr int PD = HIN ? 3 : 1;
    [[maybe_unused]] const long long nvox = (long long)a.W * a.H * D;
    auto loadw = [&](long pix, uint32_t (&w)[NP][WPP], float& off) {
        const size_t e = (size_t)pix * D + lane * PPL;
        if (!PM_RANGE_IN_BOUNDS(e, PPL, nvox, kSiteCombineLoad)) {
#pragma unroll
            for (int g = 0; g < NP; ++g)
#pragma unroll
                for (int j = 0; j < WPP; ++j) w[g][j] = 0u;
            off = 0.0f;
            return;
        }
#pragma unroll
        for (int g = 0; g < NP; ++g) {
            const uint32_t* src = HIN ? reinterpret_cast<const uint32_t*>(static_cast<const __half*>(a.part[g]) + e)
                                      : reinterpret_cast<const uint32_t*>(static_cast<const float*>(a.part[g]) + e);
            if constexpr (WPP % 4 == 0) {
#pragma unroll
                for (int j = 0; j < WPP; j += 4) {
                    const uint4 t = CG ? __ldcg(reinterpret_cast<const uint4*>(src + j)) : *reinterpret_cast<const uint4*>(src + j);
                    w[g][j] = t.x; w[g][j + 1] = t.y; w[g][j + 2] = t.z; w[g][j + 3] = t.w;
                }
            } else if constexpr (WPP % 2 == 0) {
#pragma unroll
                for (int j = 0; j < WPP; j += 2) {
                    const uint2 t = CG ? __ldcg(reinterpret_cast<const uint2*>(src + j)) : *reinterpret_cast<const uint2*>(src + j);
                    w[g][j] = t.x; w[g][j + 1] = t.y;
                }
            } else {
#pragma unroll
                for (int j = 0; j < WPP; ++j) w[g][j] = CG ? __ldcg(src + j) : src[j];
            }
        }
        off = a.offset ? (CG ? __ldcg(a.offset + pix) : __ldg(a.offset + pix)) : 0.0f;
    };
    auto unpack = [](const uint32_t (&w)[WPP], float (&v)[PPL]) {
#pragma unroll
        for (int j = 0; j < WPP; ++j) {
            if constexpr (HIN) {
                const float2 f = __half22float2(*reinterpret_cast<const __half2*>(&w[j]));
                v[2 * j] = f.x;
                v[2 * j + 1] = f.y;
            } else {
                v[j] = __uint_as_float(w[j]);
            }
        }
    };
    uint32_t ring[PD + 1][NP][WPP];
    float offr[PD + 1];
    // up to four planes per lane, the pixel of the warp's step t sits in ring slot t % (PD + 1) and
    // the pixel loop is unrolled by PD + 1, so that every slot index is a constant and the ring
    // rotates without register moves
    const bool contiguous = a.depth_pitch == (size_t)a.W * sizeof(float);
    auto process = [&](long pix, const uint32_t (&w)[NP][WPP], float off) {
        float cur[NP][PPL];
#pragma unroll
        for (int g = 0; g < NP; ++g) unpack(w[g], cur[g]);
        float o[PPL];   // (P0 + P1) + (P2 + P3), two planes per packed add
        if constexpr (NP == 4) {
            float s01[PPL], s23[PPL];
            add_planes<PPL>(s01, cur[0], cur[1]);
            add_planes<PPL>(s23, cur[2], cur[3]);
            add_planes<PPL>(o, s01, s23);
        } else {
            add_planes<PPL>(o, cur[0], cur[1]);
        }
        if (a.offset) {   // every path carries the FP16 volume's per-pixel shift once
            add_planes<PPL>(o, o, __fmul_rn((float)(2 * NP), off));
        }

        if (a.total && PM_RANGE_IN_BOUNDS((size_t)pix * D + lane * PPL, PPL, nvox, kSiteCombineOut))
            store_planes<PPL>(a.total + (size_t)pix * D + lane * PPL, o);
        if constexpr (MODE != kCombineStore) {
            float depth;
            int idx;
            int cls = 0;
            if constexpr (MODE == kCombineFilter) wta_filter<PPL>(o, incl, rk, lane, D, a.fp, depth, idx, cls);
            else case_argmin<PPL>(o, lane, D, a.fp, depth, idx);
            if (lane == 0 && PM_IN_BOUNDS(pix, (long long)a.W * a.H, kSiteCombineOut)) {
                float* dp = a.depth + pix;
                if (!contiguous) {   // W * H < 2^32: 32-bit division
                    const unsigned up = (unsigned)pix, uw = (unsigned)a.W;
                    const unsigned y = up / uw, x = up - y * uw;
                    dp = reinterpret_cast<float*>(reinterpret_cast<char*>(a.depth) + (size_t)y * a.depth_pitch) + x;
                }
                *dp = depth;
                if (a.index) a.index[pix] = idx;
                if (a.wta_class) a.wta_class[pix] = (uint8_t)cls;
            }
        }
    };
#pragma unroll
    for (int i = 0; i < PD; ++i)
        if (first + i * nw < npix) loadw(first + i * nw, ring[i], offr[i]);
    if constexpr (PPL <= 4) {
        for (long pix = first; pix < npix;) {
#pragma unroll
            for (int u = 0; u <= PD; ++u) {   // slot u holds pix; slot (u + PD) % (PD + 1) takes pix + PD * nw
                if (pix >= npix) break;
                const int ld = (u + PD) % (PD + 1);
                if (pix + PD * nw < npix) loadw(pix + PD * nw, ring[ld], offr[ld]);
                process(pix, ring[u], offr[u]);
                pix += nw;
            }
        }
    } else {   // more planes per lane: one copy of the body, the ring shifted by register moves
        for (long pix = first; pix < npix; pix += nw) {
            if (pix + PD * nw < npix) loadw(pix + PD * nw, ring[PD], offr[PD]);
            process(pix, ring[0], offr[0]);
#pragma unroll
            for (int i = 0; i < PD; ++i) {
                offr[i] = offr[i + 1];
#pragma unroll
                for (int g = 0; g < NP; ++g)
#pragma unroll
                    for (int j = 0; j < WPP; ++j) ring[i][g][j] = ring[i + 1][g][j];
            }
        }
    }
}

}  // namespace
}  // namespace pm
