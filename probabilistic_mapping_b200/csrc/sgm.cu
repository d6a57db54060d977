// sgm.cu -- semi-global min-sum aggregation (reference: sgm.cu:5-135) and the
// winner-take-all / flatness / subpixel filter (reference: filter_cost.cu:3-70).
//
// The reference runs one block per scanline with one thread per plane and finds the two
// per-pixel minima with shared-memory tree reductions (~2 log2 D barriers per pixel step),
// one direction after the other.  Here:
//   * one WARP owns a scanline: lane l holds planes [l*PPL, (l+1)*PPL), the neighbour planes
//     d-1 / d+1 come from one shuffle each, and the minimum over planes is a single
//     redux.sync.min.f32;
//   * the per-pixel plane vector (contiguous in the plane-innermost layout) is streamed with
//     cp.async into a per-lane shared-memory ring PF steps ahead of the recurrence; the reference
//     pixels of a scanline are read 32 steps at a time, one per lane, and become one ballot of
//     adaptive-penalty flags, so a step costs a bit test instead of a load and a comparison;
//   * a step's arithmetic is the reference's, element for element, with the adds of two planes
//     on the packed FP32x2 pipe and no per-plane inclusion masks when every plane takes part in
//     the minima (D a power of two, or the exact minimum);
//   * opposite paths run as pairs: one warp walks a scanline from both ends at once, so it keeps
//     two independent recurrences in flight; the pairs (L/R, T/B and the two diagonals) run
//     concurrently on separate streams.  Each pair owns one volume: the path that reaches a pixel
//     first stores its values there and the other adds its own with a vector reduction, so the
//     volume ends up holding P_2p + P_2p+1 (float addition is commutative, so this is the same
//     sum in either order);
//   * a pixel-parallel combine kernel (one warp per pixel, full occupancy) adds the pair volumes,
//     (P0 + P1) + (P2 + P3) [+ ((P4 + P5) + (P6 + P7))], in registers and runs the
//     winner-take-all directly, so the complete sum need not be written.  The FP32 result
//     therefore differs from the reference's sequential path order only by rounding; the CPU
//     oracle replays this exact order.  (The reduction unit flushes subnormal sums to zero; path
//     values are costs plus penalties, never below 2^-126 unless exactly 0.)
//   * the FP16 form (FP16 cost volume) keeps its pair volumes in FP16 as well: each path's values
//     are rounded to FP16, the second end adds with packed FP16 reductions, and the combine adds
//     the pairs in FP32.  That halves the bytes of the pair volumes, which with FP32 pairs were
//     60 % of the stage's traffic; the FP16 form is held to its FP64 accuracy bound, not to bits.
#include <climits>
#include <vector>

#include "pm_device.cuh"

namespace pm {

void plane_order(int D, int compat, PlaneOrder& out) {
    // Merge order of `for (i = D>>1; i > 0; i >>= 1) if (d < i && d + i < D ...)`:
    // slot d keeps its element on ties, so the winner among equal values is the first in
    // the concatenated merge lists; planes never merged into slot 0 are dropped.
    std::vector<std::vector<int>> slot((size_t)D);
    for (int d = 0; d < D; ++d) slot[d].push_back(d);
    for (int i = D >> 1; i > 0; i >>= 1)
        for (int d = 0; d < i; ++d)
            if (d + i < D) {
                slot[d].insert(slot[d].end(), slot[d + i].begin(), slot[d + i].end());
                slot[d + i].clear();
            }
    std::vector<int> rank((size_t)D, 0);
    std::vector<char> incl((size_t)D, 0);
    int r = 0;
    for (int e : slot[0]) { rank[e] = r++; incl[e] = 1; }
    if (!compat)
        for (int d = 0; d < D; ++d)
            if (!incl[d]) { rank[d] = r++; incl[d] = 1; }
    const int ppl = D / 32;
    for (int l = 0; l < 32; ++l) {
        uint32_t bits = 0;
        for (int j = 0; j < ppl; ++j)
            if (incl[l * ppl + j]) bits |= 1u << j;
        out.incl[l] = bits;
    }
    for (int d = 0; d < kMaxPlanes; ++d) out.rank[d] = d < D ? (uint16_t)rank[d] : 0xffff;
}

namespace {

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

// Winner-take-all with the reference tree's tie-break, then the three rejection rules and
// the parabola subpixel refinement (filter_cost.cu:22-52), plus the optional uniqueness test.
template <int PPL>
__device__ __forceinline__ void wta_filter(const float (&s)[PPL], uint32_t incl, const uint16_t (&rk)[PPL],
                                           int lane, int D, const FilterParams& fp, float& depth_out,
                                           int& idx_out) {
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
    if ((double)mn < kFloatEps && (double)mn > -kFloatEps) {
        depth = kDepInf;                                   // non-overlap (:37-38)
    } else if (idx == 0 || idx == D - 1) {
        depth = 0.0f;                                      // border plane (:39-40)
    } else {
        const float pre = plane_value(s, idx - 1), post = plane_value(s, idx + 1);
        if (__fadd_rn(pre, post) < __fmul_rn(__fmul_rn(2.0f, mn), fp.var_scale)) {
            depth = 0.0f;                                  // flat minimum (:41-42)
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
            } else {                                       // parabola (:45-51)
                const float a2 = __fadd_rn(__fsub_rn(pre, __fmul_rn(2.0f, mn)), post);
                const float b = __fadd_rn(-pre, post);
                const float sub = __fsub_rn((float)idx, __fdiv_rn(b, __fmul_rn(2.0f, a2)));
                depth = __frcp_rn(__fmaf_rn(sub, fp.drho, fp.rho0));
            }
        }
    }
    depth_out = depth;
    idx_out = idx;
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
    if ((double)mn < kFloatEps) v = kCaseInf;
    else if (idx == 0 || idx == D - 1) v = 0.0f;
    else v = __frcp_rn(__fmaf_rn((float)idx, fp.drho, fp.rho0));
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

template <int PPL, bool HALF>
__device__ __forceinline__ void load_slice(float (&cv)[PPL], const unsigned char* p) {
    if constexpr (HALF) {
        const __half2* hp = reinterpret_cast<const __half2*>(p);
#pragma unroll
        for (int j = 0; j < PPL / 2; ++j) {
            const float2 v = __half22float2(hp[j]);
            cv[2 * j] = v.x;
            cv[2 * j + 1] = v.y;
        }
    } else {
        load_planes<PPL>(cv, reinterpret_cast<const float*>(p));
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
__device__ __forceinline__ float chain_ref(const float* __restrict__ ref, long p0, long step, int k, int n) {
    return k < n ? __ldg(ref + p0 + (long)k * step) : 0.0f;
}

// The flags |I(k) - I(k-1)| < tau of the 32 steps k0 .. k0+31 of one chain as a ballot (bit i:
// step k0 + i).  Lane i holds I(k0 + i) in `cur` (read one batch ahead into `nxt`, which is
// then refilled with I(k0 + 64 + i)); `last` carries I(k0 - 1).
__device__ __forceinline__ unsigned penalty_flags(float& cur, float& nxt, const float* __restrict__ ref, long p0,
                                                  long step, int k0, int n, int lane, float tau, float& last) {
    const float I = cur;
    cur = nxt;
    nxt = chain_ref(ref, p0, step, k0 + 64 + lane, n);
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
template <int PPL, bool HALF, int NW, bool FULL, bool HOUT>
__global__ void __launch_bounds__(NW * 32) sgm_pair_kernel(const SgmLaunch a, int dx, int dy, int slot) {
    using CT = typename CostElem<HALF>::T;
    using OT = typename CostElem<HOUT>::T;
    using RG = Ring<PPL, HALF>;
    constexpr int CB = RG::CB, CHAIN_B = RG::CHAIN_B, STAGE_B = RG::STAGE_B;
    extern __shared__ __align__(16) unsigned char ring[];

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int W = a.W, H = a.H, D = a.D;
    const int c = blockIdx.x * NW + warp;
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
    auto put = [](OT* q, const float (&v)[PPL]) {
        if constexpr (HOUT) store_planes_h<PPL>(q, v);
        else store_planes<PPL>(q, v);
    };
    auto add = [](OT* q, const float (&v)[PPL]) {
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
        cp_async_bytes<CB>(sb + lane * CB, cf0 + (long)k * gstep);
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
    float If = chain_ref(a.ref, pf0, step, lane, n), Ifn = chain_ref(a.ref, pf0, step, 32 + lane, n);
    float Ib = chain_ref(a.ref, pb0, -step, lane, n), Ibn = chain_ref(a.ref, pb0, -step, 32 + lane, n);
    fs.qmask = penalty_flags(If, Ifn, a.ref, pf0, step, 0, n, lane, a.tau, lastf);
    bs.qmask = penalty_flags(Ib, Ibn, a.ref, pb0, -step, 0, n, lane, a.tau, lastb);

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
            fs.qmask = penalty_flags(If, Ifn, a.ref, pf0, step, k, n, lane, a.tau, lastf);
            bs.qmask = penalty_flags(Ib, Ibn, a.ref, pb0, -step, k, n, lane, a.tau, lastb);
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
// argmin (kCombineArgmin) or only a store of the sum (kCombineStore).  One warp per pixel,
// grid-stride; the next pixel's slices are loaded before the current one is reduced.
template <int PPL, int MODE, int NP, bool HIN>
__global__ void __launch_bounds__(256) combine_kernel(const SgmLaunch a) {
    const int lane = threadIdx.x & 31;
    const long nw = (long)gridDim.x * (blockDim.x >> 5);
    const long npix = (long)a.W * a.H;
    const int D = a.D;
    uint32_t incl;
    uint16_t rk[PPL];
    lane_order<PPL>(a.order, lane, incl, rk);
    auto loadp = [&](long pix, float (&s)[NP][PPL]) {
        const size_t e = (size_t)pix * D + lane * PPL;
#pragma unroll
        for (int g = 0; g < NP; ++g) {
            if constexpr (HIN)
                load_slice<PPL, true>(s[g], reinterpret_cast<const unsigned char*>(static_cast<const __half*>(a.part[g]) + e));
            else
                load_planes<PPL>(s[g], static_cast<const float*>(a.part[g]) + e);
        }
    };
    long pix = (long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    float cur[NP][PPL], nxt[NP][PPL];
    if (pix < npix) loadp(pix, cur);
    for (; pix < npix; pix += nw) {
        if (pix + nw < npix) loadp(pix + nw, nxt);
        float o[PPL];
#pragma unroll
        for (int j = 0; j < PPL; ++j) {
            if constexpr (NP == 4)
                o[j] = __fadd_rn(__fadd_rn(cur[0][j], cur[1][j]), __fadd_rn(cur[2][j], cur[3][j]));
            else
                o[j] = __fadd_rn(cur[0][j], cur[1][j]);
        }
        if (a.offset) {   // every path carries the FP16 volume's per-pixel shift once
            const float sh = __fmul_rn((float)(2 * NP), __ldg(a.offset + pix));
#pragma unroll
            for (int j = 0; j < PPL; ++j) o[j] = __fadd_rn(o[j], sh);
        }

        if (a.total) store_planes<PPL>(a.total + (size_t)pix * D + lane * PPL, o);
        if constexpr (MODE != kCombineStore) {
            float depth;
            int idx;
            if constexpr (MODE == kCombineFilter) wta_filter<PPL>(o, incl, rk, lane, D, a.fp, depth, idx);
            else case_argmin<PPL>(o, lane, D, a.fp, depth, idx);
            if (lane == 0) {
                const int y = (int)(pix / a.W), x = (int)(pix - (long)y * a.W);
                *reinterpret_cast<float*>(reinterpret_cast<char*>(a.depth) + (size_t)y * a.depth_pitch +
                                          (size_t)x * 4) = depth;
                if (a.index) a.index[pix] = idx;
            }
        }
#pragma unroll
        for (int g = 0; g < NP; ++g)
#pragma unroll
            for (int j = 0; j < PPL; ++j) cur[g][j] = nxt[g][j];
    }
}

template <int PPL>
__global__ void __launch_bounds__(128) filter_kernel(const float* __restrict__ sum, int W, int H, int D,
                                                     const FilterParams fp, const PlaneOrder order,
                                                     float* depth, size_t pitch, int32_t* index) {
    const int lane = threadIdx.x & 31;
    const long pix = (long)blockIdx.x * 4 + (threadIdx.x >> 5);
    uint32_t incl;
    uint16_t rk[PPL];
    lane_order<PPL>(order, lane, incl, rk);
    if (pix >= (long)W * H) return;
    float s[PPL];
    load_planes<PPL>(s, sum + (size_t)pix * D + lane * PPL);
    float dep;
    int idx;
    wta_filter<PPL>(s, incl, rk, lane, D, fp, dep, idx);
    if (lane == 0) {
        const int y = (int)(pix / W), x = (int)(pix - (long)y * W);
        *reinterpret_cast<float*>(reinterpret_cast<char*>(depth) + (size_t)y * pitch + (size_t)x * 4) = dep;
        if (index) index[pix] = idx;
    }
}

// CASE 0 of outputFusionCPU: the debug argmin straight on the plane-sweep cost volume.
template <int PPL, bool HALF>
__global__ void __launch_bounds__(128) case_kernel(const void* __restrict__ vol, const float* __restrict__ offset,
                                                   int W, int H, int D, const FilterParams fp, float* depth,
                                                   size_t pitch, int32_t* index) {
    const int lane = threadIdx.x & 31;
    const long pix = (long)blockIdx.x * 4 + (threadIdx.x >> 5);
    if (pix >= (long)W * H) return;
    float s[PPL];
    if constexpr (HALF) {
        const __half* p = static_cast<const __half*>(vol) + (size_t)pix * D + lane * PPL;
        const float off = __ldg(offset + pix);
#pragma unroll
        for (int j = 0; j < PPL; ++j) s[j] = __fadd_rn(__half2float(p[j]), off);
    } else {
        load_planes<PPL>(s, static_cast<const float*>(vol) + (size_t)pix * D + lane * PPL);
    }
    float dep;
    int idx;
    case_argmin<PPL>(s, lane, D, fp, dep, idx);
    if (lane == 0) {
        const int y = (int)(pix / W), x = (int)(pix - (long)y * W);
        *reinterpret_cast<float*>(reinterpret_cast<char*>(depth) + (size_t)y * pitch + (size_t)x * 4) = dep;
        if (index) index[pix] = idx;
    }
}

// Path r of the reference order (L->R, R->L, T->B, B->T, then TL->BR, BR->TL, TR->BL, BL->TR);
// pair p = paths (2p, 2p+1) runs as one sgm_pair_kernel along direction kDirs[2p].
const int kDirs[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {-1, -1}, {-1, 1}, {1, -1}};

// A launch with an explicit priority attribute (recorded into graph nodes under capture), or a
// plain launch at the stream's priority.
template <typename... Args>
cudaError_t launch_with_priority(void (*kern)(Args...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                                 int priority, Args... args) {
    if (priority == 0) {
        kern<<<grid, block, smem, s>>>(args...);
        return cudaGetLastError();
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = grid;
    cfg.blockDim = block;
    cfg.dynamicSmemBytes = smem;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributePriority;
    attr[0].val.priority = priority;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, kern, args...);
}

template <int PPL, bool HALF, int NW>
cudaError_t launch_pair_nw(const SgmLaunch& a, int pair, cudaStream_t s) {
    const size_t smem = (size_t)NW * PF * Ring<PPL, HALF>::STAGE_B;
    // every plane takes part in the minima (D a power of two, or the exact minimum): no masks
    bool full = true;
    for (int l = 0; l < 32; ++l) full = full && a.order.incl[l] == (1u << PPL) - 1u;
    void (*kern)(SgmLaunch, int, int, int);
    if constexpr (HALF && PPL % 2 == 0) {
        if (a.part_half) kern = full ? sgm_pair_kernel<PPL, HALF, NW, true, true> : sgm_pair_kernel<PPL, HALF, NW, false, true>;
        else kern = full ? sgm_pair_kernel<PPL, HALF, NW, true, false> : sgm_pair_kernel<PPL, HALF, NW, false, false>;
    } else {
        if (a.part_half) return cudaErrorInvalidValue;   // FP16 pair volumes come with FP16 cost volumes
        kern = full ? sgm_pair_kernel<PPL, HALF, NW, true, false> : sgm_pair_kernel<PPL, HALF, NW, false, false>;
    }
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    const int dx = kDirs[2 * pair][0], dy = kDirs[2 * pair][1];
    const int nch = num_chains(dx, dy, a.W, a.H);
    return launch_with_priority(kern, dim3((nch + NW - 1) / NW), dim3(NW * 32), smem, s, a.priority, a, dx, dy,
                                2 * pair);
}

// scanlines (warps) per block: a.pair_warps in {2, 4, 8}, 2 when unset (the batched form's
// autotuner picks 2 for the 640x480x128 map too: smaller blocks spread one map's few scanlines
// over more SMs)
template <int PPL, bool HALF>
cudaError_t launch_pair(const SgmLaunch& a, int pair, cudaStream_t s) {
    switch (a.pair_warps) {
        case 4: return launch_pair_nw<PPL, HALF, 4>(a, pair, s);
        case 8: return launch_pair_nw<PPL, HALF, 8>(a, pair, s);
        default: return launch_pair_nw<PPL, HALF, 2>(a, pair, s);
    }
}

template <int PPL>
cudaError_t launch_combine(const SgmLaunch& a, int mode, cudaStream_t s) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long npix = (long)a.W * a.H;
    const long blocks_needed = (npix + 7) / 8;   // 8 warps per block
    const int blocks = (int)(blocks_needed < (long)sms * 8 ? blocks_needed : (long)sms * 8);
    const bool eight = a.num_paths == 8;
    void (*kern)(SgmLaunch) = nullptr;
    if (a.part_half) {
        if constexpr (PPL % 2 == 0) {
            if (mode == kCombineFilter)
                kern = eight ? combine_kernel<PPL, kCombineFilter, 4, true> : combine_kernel<PPL, kCombineFilter, 2, true>;
            else if (mode == kCombineArgmin)
                kern = eight ? combine_kernel<PPL, kCombineArgmin, 4, true> : combine_kernel<PPL, kCombineArgmin, 2, true>;
            else
                kern = eight ? combine_kernel<PPL, kCombineStore, 4, true> : combine_kernel<PPL, kCombineStore, 2, true>;
        } else {
            return cudaErrorInvalidValue;
        }
    } else if (mode == kCombineFilter) {
        kern = eight ? combine_kernel<PPL, kCombineFilter, 4, false> : combine_kernel<PPL, kCombineFilter, 2, false>;
    } else if (mode == kCombineArgmin) {
        kern = eight ? combine_kernel<PPL, kCombineArgmin, 4, false> : combine_kernel<PPL, kCombineArgmin, 2, false>;
    } else {
        kern = eight ? combine_kernel<PPL, kCombineStore, 4, false> : combine_kernel<PPL, kCombineStore, 2, false>;
    }
    return launch_with_priority(kern, dim3(blocks), dim3(256), 0, s, a.priority, a);
}

// Path pairs p = 0 .. num_paths/2 - 1: pairs 0..np-2 run on their own side streams when `side`
// is given, the last on `s`, which then joins the others and runs the combine kernel.
template <int PPL, bool HALF>
cudaError_t launch_sgm_t(const SgmLaunch& a, int mode, cudaStream_t s, const SgmStreams* side) {
    const int np = a.num_paths / 2;
    cudaError_t e = cudaSuccess;
    if (a.serial_pairs) side = nullptr;
    if (side) {
        if ((e = cudaEventRecord(side->fork, s)) != cudaSuccess) return e;
        for (int p = 0; p < np - 1; ++p) {
            if ((e = cudaStreamWaitEvent(side->stream[p], side->fork, 0)) != cudaSuccess) return e;
            if ((e = launch_pair<PPL, HALF>(a, p, side->stream[p])) != cudaSuccess) return e;
            if ((e = cudaEventRecord(side->join[p], side->stream[p])) != cudaSuccess) return e;
        }
    } else {
        for (int p = 0; p < np - 1 && e == cudaSuccess; ++p) e = launch_pair<PPL, HALF>(a, p, s);
        if (e != cudaSuccess) return e;
    }
    if ((e = launch_pair<PPL, HALF>(a, np - 1, s)) != cudaSuccess) return e;
    if (side)
        for (int p = 0; p < np - 1; ++p)
            if ((e = cudaStreamWaitEvent(s, side->join[p], 0)) != cudaSuccess) return e;
    return launch_combine<PPL>(a, mode, s);
}

template <int PPL>
cudaError_t launch_filter_t(const float* sum, int W, int H, int D, const FilterParams& fp,
                            const PlaneOrder& order, float* depth, size_t pitch, int32_t* index,
                            cudaStream_t s) {
    const long n = (long)W * H;
    filter_kernel<PPL><<<(unsigned)((n + 3) / 4), 128, 0, s>>>(sum, W, H, D, fp, order, depth, pitch, index);
    return cudaGetLastError();
}

}  // namespace

cudaError_t launch_sgm(const SgmLaunch& a, int mode, cudaStream_t s, const SgmStreams* side) {
    const int ppl = a.D / 32;
    // FP16 volumes need an even number of planes per lane (4-byte cp.async pieces)
    if (a.cost_half && (ppl % 2)) return cudaErrorInvalidValue;
    switch (ppl) {
        case 1: return launch_sgm_t<1, false>(a, mode, s, side);
        case 2: return a.cost_half ? launch_sgm_t<2, true>(a, mode, s, side)
                                   : launch_sgm_t<2, false>(a, mode, s, side);
        case 3: return launch_sgm_t<3, false>(a, mode, s, side);
        case 4: return a.cost_half ? launch_sgm_t<4, true>(a, mode, s, side)
                                   : launch_sgm_t<4, false>(a, mode, s, side);
        case 5: return launch_sgm_t<5, false>(a, mode, s, side);
        case 6: return a.cost_half ? launch_sgm_t<6, true>(a, mode, s, side)
                                   : launch_sgm_t<6, false>(a, mode, s, side);
        case 7: return launch_sgm_t<7, false>(a, mode, s, side);
        case 8: return a.cost_half ? launch_sgm_t<8, true>(a, mode, s, side)
                                   : launch_sgm_t<8, false>(a, mode, s, side);
        default: return cudaErrorInvalidValue;
    }
}

cudaError_t launch_filter(const float* sum, int W, int H, int D, const FilterParams& fp,
                          const PlaneOrder& order, float* depth, size_t pitch, int32_t* index,
                          cudaStream_t s) {
    switch (D / 32) {
        case 1: return launch_filter_t<1>(sum, W, H, D, fp, order, depth, pitch, index, s);
        case 2: return launch_filter_t<2>(sum, W, H, D, fp, order, depth, pitch, index, s);
        case 3: return launch_filter_t<3>(sum, W, H, D, fp, order, depth, pitch, index, s);
        case 4: return launch_filter_t<4>(sum, W, H, D, fp, order, depth, pitch, index, s);
        case 5: return launch_filter_t<5>(sum, W, H, D, fp, order, depth, pitch, index, s);
        case 6: return launch_filter_t<6>(sum, W, H, D, fp, order, depth, pitch, index, s);
        case 7: return launch_filter_t<7>(sum, W, H, D, fp, order, depth, pitch, index, s);
        case 8: return launch_filter_t<8>(sum, W, H, D, fp, order, depth, pitch, index, s);
        default: return cudaErrorInvalidValue;
    }
}

template <int PPL, bool HALF>
cudaError_t launch_case_t(const void* vol, const float* offset, int W, int H, int D, const FilterParams& fp,
                          float* depth, size_t pitch, int32_t* index, cudaStream_t s) {
    const long n = (long)W * H;
    case_kernel<PPL, HALF><<<(unsigned)((n + 3) / 4), 128, 0, s>>>(vol, offset, W, H, D, fp, depth, pitch, index);
    return cudaGetLastError();
}

cudaError_t launch_case_argmin(const void* vol, int half, const float* offset, int W, int H, int D,
                               const FilterParams& fp, float* depth, size_t pitch, int32_t* index, cudaStream_t s) {
    if (half && !offset) return cudaErrorInvalidValue;
    switch (D / 32) {
#define PM_CASE_PPL(P) \
        case P: return half ? launch_case_t<P, true>(vol, offset, W, H, D, fp, depth, pitch, index, s) \
                            : launch_case_t<P, false>(vol, offset, W, H, D, fp, depth, pitch, index, s);
        PM_CASE_PPL(1) PM_CASE_PPL(2) PM_CASE_PPL(3) PM_CASE_PPL(4)
        PM_CASE_PPL(5) PM_CASE_PPL(6) PM_CASE_PPL(7) PM_CASE_PPL(8)
#undef PM_CASE_PPL
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace pm
