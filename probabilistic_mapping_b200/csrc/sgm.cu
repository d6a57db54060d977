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
//     cp.async into a per-lane shared-memory ring PF steps ahead of the recurrence;
//   * the paths run as four concurrent groups {r, r+4} (an axis direction and a diagonal),
//     each accumulating into its own partial-sum volume, so four times as many scanlines are
//     in flight as in a one-direction-at-a-time schedule;
//   * a pixel-parallel combine kernel (one warp per pixel, full occupancy) adds the partials
//     as (S0 + S1) + (S2 + S3) in registers and runs the winner-take-all directly, so the
//     complete sum is never written.  The FP32 result therefore differs from the reference's
//     sequential path order only by rounding; the CPU oracle replays this exact order.
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

constexpr int WARPS = 4;   // scanlines per block
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

template <bool HALF> struct CostElem;
template <> struct CostElem<false> { using T = float; };
template <> struct CostElem<true> { using T = __half; };

enum { FIRST = 0, ACC = 1 };

// Bytes one lane moves per pixel step: the cost slice, the group's partial sum (ACC), and the
// reference pixel for the path gradient.
template <int PPL, int MODE, bool HALF> struct Slots {
    static constexpr int CB = PPL * (int)sizeof(typename CostElem<HALF>::T);
    static constexpr int SB = MODE == ACC ? PPL * 4 : 0;
    static constexpr int LANE_B = CB + SB + 4;
    static constexpr int STAGE_B = 32 * LANE_B;
};

// One direction pass accumulating into the partial-sum volume of its group.
template <int PPL, int MODE, bool HALF>
__global__ void __launch_bounds__(WARPS * 32) sgm_dir_kernel(const SgmLaunch a, int dx, int dy, int group) {
    using CT = typename CostElem<HALF>::T;
    using SL = Slots<PPL, MODE, HALF>;
    constexpr int CB = SL::CB, SB = SL::SB, STAGE_B = SL::STAGE_B;
    extern __shared__ __align__(16) unsigned char ring[];

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int W = a.W, H = a.H, D = a.D;
    const int c = blockIdx.x * WARPS + warp;
    if (c >= num_chains(dx, dy, W, H)) return;        // warp-uniform; no block barriers below
    const Chain ch = chain_start(c, dx, dy, W, H);

    // stage layout: [cost slices of 32 lanes][partial slices of 32 lanes][32 ref values]
    unsigned char* wbase = ring + (size_t)warp * PF * STAGE_B;
    const int off_c = lane * CB;
    const int off_s = 32 * CB + lane * SB;
    const int off_i = 32 * (CB + SB) + lane * 4;

    float* const part = a.part[group];
    const CT* __restrict__ cost = reinterpret_cast<const CT*>(a.cost);
    const long pstep = (long)dy * W + dx;
    long pix = (long)ch.y * W + ch.x;

    auto issue = [&](unsigned char* sb, long q) {
        const size_t e = (size_t)q * D + lane * PPL;
        cp_async_bytes<CB>(sb + off_c, cost + e);
        if constexpr (MODE == ACC) cp_async_bytes<SB>(sb + off_s, part + e);
        cp_async_4(sb + off_i, a.ref + q);
    };
#pragma unroll 1
    for (int k = 0; k < PF; ++k) {
        if (k < ch.n) issue(wbase + k * STAGE_B, pix + k * pstep);
        cp_async_commit();
    }

    const uint32_t incl = a.order.incl[lane];
    float L[PPL];
#pragma unroll
    for (int j = 0; j < PPL; ++j) L[j] = 0.0f;
    float mprev = 0.0f, Iprev = 0.0f;
    int st = 0;

#pragma unroll 1
    for (int k = 0; k < ch.n; ++k) {
        cp_async_wait<PF - 1>();
        unsigned char* sb = wbase + st * STAGE_B;
        float cv[PPL];
        if constexpr (HALF) {
            const __half* hp = reinterpret_cast<const __half*>(sb + off_c);
#pragma unroll
            for (int j = 0; j < PPL; ++j) cv[j] = __half2float(hp[j]);
        } else {
            load_planes<PPL>(cv, reinterpret_cast<const float*>(sb + off_c));
        }
        float sv[PPL];
        if constexpr (MODE == ACC) load_planes<PPL>(sv, reinterpret_cast<const float*>(sb + off_s));
        const float I = *reinterpret_cast<const float*>(sb + off_i);

        // a plane never measured (cost -1) marks the pixel invalid (sgm.cu:33,67)
        bool neg = false;
#pragma unroll
        for (int j = 0; j < PPL; ++j) neg |= (((incl >> j) & 1u) && cv[j] < 0.0f);
        const bool inv = __any_sync(kFull, neg);

        float Ln[PPL];
        if (k == 0) {
#pragma unroll
            for (int j = 0; j < PPL; ++j) Ln[j] = inv ? 0.0f : cv[j];
        } else {
            // adaptive penalties from the path gradient of the reference image (sgm.cu:75-82)
            const float D1 = fabsf(__fsub_rn(I, Iprev));
            float P1 = a.p1, P2 = a.p2;
            if (D1 < a.tau) { P1 = __fmul_rn(P1, a.q1); P2 = __fmul_rn(P2, a.q2); }
            const float mP2 = __fadd_rn(mprev, P2);
            float lm = __shfl_up_sync(kFull, L[PPL - 1], 1);
            float lp = __shfl_down_sync(kFull, L[0], 1);
            if (lane == 0) lm = inf_f();
            if (lane == 31) lp = inf_f();
            // min(L[d], minL + P2, L[d-1] + P1, L[d+1] + P1) (sgm.cu:85-92); min(a+P1, b+P1) is
            // min(a, b) + P1 exactly because rounding is monotonic
#pragma unroll
            for (int j = 0; j < PPL; ++j) {
                const float left = (j == 0) ? lm : L[j - 1];
                const float right = (j == PPL - 1) ? lp : L[j + 1];
                const float vv = min3f(L[j], mP2, __fadd_rn(fminf(left, right), P1));
                Ln[j] = __fsub_rn(__fadd_rn(inv ? 0.0f : cv[j], vv), mprev);   // (:98)
            }
        }
        Iprev = I;
        float lmin = inf_f();
#pragma unroll
        for (int j = 0; j < PPL; ++j) {
            L[j] = Ln[j];
            if ((incl >> j) & 1u) lmin = fminf(lmin, Ln[j]);
        }
        mprev = warp_min_f32(lmin);

        // the output is set to COST_INF = 0 at an invalid pixel, else accumulated (:101-108)
        float o[PPL];
        if constexpr (MODE == FIRST) {
#pragma unroll
            for (int j = 0; j < PPL; ++j) o[j] = inv ? 0.0f : Ln[j];
        } else {
#pragma unroll
            for (int j = 0; j < PPL; ++j) o[j] = inv ? 0.0f : __fadd_rn(sv[j], Ln[j]);
        }
        store_planes<PPL>(part + (size_t)pix * D + lane * PPL, o);
        // refill this stage (consumed above) with step k + PF
        if (k + PF < ch.n) issue(sb, pix + PF * pstep);
        cp_async_commit();
        pix += pstep;
        st = (st + 1 == PF) ? 0 : st + 1;
    }
    cp_async_wait<0>();
}

// Sum of the four group partials, (S0 + S1) + (S2 + S3), then (FILTER) the winner-take-all or
// (!FILTER) a store of the sum.  One warp per pixel, grid-stride; the next pixel's partials are
// loaded before the current one is reduced.
template <int PPL, bool FILTER>
__global__ void __launch_bounds__(256) combine_kernel(const SgmLaunch a) {
    const int lane = threadIdx.x & 31;
    const long nw = (long)gridDim.x * (blockDim.x >> 5);
    const long npix = (long)a.W * a.H;
    const int D = a.D;
    uint32_t incl;
    uint16_t rk[PPL];
    lane_order<PPL>(a.order, lane, incl, rk);
    auto load4 = [&](long pix, float (&s)[4][PPL]) {
        const size_t e = (size_t)pix * D + lane * PPL;
#pragma unroll
        for (int g = 0; g < 4; ++g) load_planes<PPL>(s[g], a.part[g] + e);
    };
    long pix = (long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    float cur[4][PPL], nxt[4][PPL];
    if (pix < npix) load4(pix, cur);
    for (; pix < npix; pix += nw) {
        if (pix + nw < npix) load4(pix + nw, nxt);
        float o[PPL];
#pragma unroll
        for (int j = 0; j < PPL; ++j) o[j] = __fadd_rn(__fadd_rn(cur[0][j], cur[1][j]), __fadd_rn(cur[2][j], cur[3][j]));
        if (a.total) store_planes<PPL>(a.total + (size_t)pix * D + lane * PPL, o);
        if constexpr (FILTER) {
            float depth;
            int idx;
            wta_filter<PPL>(o, incl, rk, lane, D, a.fp, depth, idx);
            if (lane == 0) {
                const int y = (int)(pix / a.W), x = (int)(pix - (long)y * a.W);
                *reinterpret_cast<float*>(reinterpret_cast<char*>(a.depth) + (size_t)y * a.depth_pitch +
                                          (size_t)x * 4) = depth;
                if (a.index) a.index[pix] = idx;
            }
        }
#pragma unroll
        for (int g = 0; g < 4; ++g)
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

const int kDirs[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {-1, -1}, {-1, 1}, {1, -1}};

template <int PPL, int MODE, bool HALF>
cudaError_t launch_dir(const SgmLaunch& a, int dir, int group, cudaStream_t s) {
    const size_t smem = (size_t)WARPS * PF * Slots<PPL, MODE, HALF>::STAGE_B;
    auto kern = sgm_dir_kernel<PPL, MODE, HALF>;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    const int dx = kDirs[dir][0], dy = kDirs[dir][1];
    const int nch = num_chains(dx, dy, a.W, a.H);
    kern<<<(nch + WARPS - 1) / WARPS, WARPS * 32, smem, s>>>(a, dx, dy, group);
    return cudaGetLastError();
}

template <int PPL>
cudaError_t launch_combine(const SgmLaunch& a, bool fuse_filter, cudaStream_t s) {
    int dev = 0, sms = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const long npix = (long)a.W * a.H;
    const long blocks_needed = (npix + 7) / 8;   // 8 warps per block
    const int blocks = (int)(blocks_needed < (long)sms * 8 ? blocks_needed : (long)sms * 8);
    if (fuse_filter) combine_kernel<PPL, true><<<blocks, 256, 0, s>>>(a);
    else combine_kernel<PPL, false><<<blocks, 256, 0, s>>>(a);
    return cudaGetLastError();
}

// Groups g = 0..3 hold paths {g} (4-path mode) or {g, g+4} (8-path mode).  Groups 0..2 run on
// their own streams when `side` is given; group 3 runs on `s`, which then joins the others and
// runs the combine / winner-take-all kernel.
template <int PPL, bool HALF>
cudaError_t launch_sgm_t(const SgmLaunch& a, bool fuse_filter, cudaStream_t s, const SgmStreams* side) {
    const bool eight = a.num_paths == 8;
    cudaError_t e = cudaSuccess;
    auto group_passes = [&](int g, cudaStream_t gs) -> cudaError_t {
        cudaError_t r = launch_dir<PPL, FIRST, HALF>(a, g, g, gs);
        if (r == cudaSuccess && eight) r = launch_dir<PPL, ACC, HALF>(a, g + 4, g, gs);
        return r;
    };
    if (side) {
        if ((e = cudaEventRecord(side->fork, s)) != cudaSuccess) return e;
        for (int g = 0; g < 3; ++g) {
            if ((e = cudaStreamWaitEvent(side->stream[g], side->fork, 0)) != cudaSuccess) return e;
            if ((e = group_passes(g, side->stream[g])) != cudaSuccess) return e;
            if ((e = cudaEventRecord(side->join[g], side->stream[g])) != cudaSuccess) return e;
        }
    } else {
        for (int g = 0; g < 3 && e == cudaSuccess; ++g) e = group_passes(g, s);
        if (e != cudaSuccess) return e;
    }
    if ((e = group_passes(3, s)) != cudaSuccess) return e;
    if (side)
        for (int g = 0; g < 3; ++g)
            if ((e = cudaStreamWaitEvent(s, side->join[g], 0)) != cudaSuccess) return e;
    return launch_combine<PPL>(a, fuse_filter, s);
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

cudaError_t launch_sgm(const SgmLaunch& a, bool fuse_filter, cudaStream_t s, const SgmStreams* side) {
    const int ppl = a.D / 32;
    // FP16 volumes need an even number of planes per lane (4-byte cp.async pieces)
    if (a.cost_half && (ppl % 2)) return cudaErrorInvalidValue;
    switch (ppl) {
        case 1: return launch_sgm_t<1, false>(a, fuse_filter, s, side);
        case 2: return a.cost_half ? launch_sgm_t<2, true>(a, fuse_filter, s, side)
                                   : launch_sgm_t<2, false>(a, fuse_filter, s, side);
        case 3: return launch_sgm_t<3, false>(a, fuse_filter, s, side);
        case 4: return a.cost_half ? launch_sgm_t<4, true>(a, fuse_filter, s, side)
                                   : launch_sgm_t<4, false>(a, fuse_filter, s, side);
        case 5: return launch_sgm_t<5, false>(a, fuse_filter, s, side);
        case 6: return a.cost_half ? launch_sgm_t<6, true>(a, fuse_filter, s, side)
                                   : launch_sgm_t<6, false>(a, fuse_filter, s, side);
        case 7: return launch_sgm_t<7, false>(a, fuse_filter, s, side);
        case 8: return a.cost_half ? launch_sgm_t<8, true>(a, fuse_filter, s, side)
                                   : launch_sgm_t<8, false>(a, fuse_filter, s, side);
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

}  // namespace pm
