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
#include <vector>

#include "sgm_device.cuh"

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

template <int PPL, bool HALF, int NW, bool FULL, bool HOUT>
__global__ void __launch_bounds__(NW * 32) sgm_pair_kernel(const SgmLaunch a, int dx, int dy, int slot) {
    extern __shared__ __align__(16) unsigned char ring[];
    sgm_pair_block<PPL, HALF, NW, FULL, HOUT>(a, dx, dy, slot, blockIdx.x, ring);
}

// Blocks per SM that the combine kernel is held to (0: no bound): D = 192 in FP32, D = 256 in FP16
// with four paths and D = 128 in FP16 with eight, where the compiler's default register choice
// leaves one block per SM fewer.
constexpr int combine_min_blocks(int ppl, int np, bool hin) {
    return ppl == 6 && !hin ? (np == 2 ? 4 : 3) : ppl == 8 && hin && np == 2 ? 3 : ppl == 4 && hin && np == 4 ? 4 : 0;
}

// grid-stride over the image's pixels, one warp per pixel
template <int PPL, int MODE, int NP, bool HIN>
__global__ void __launch_bounds__(256, combine_min_blocks(PPL, NP, HIN)) combine_kernel(const SgmLaunch a) {
    combine_pixels<PPL, MODE, NP, HIN, false>(a, (long)blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5),
                                              (long)gridDim.x * (blockDim.x >> 5), (long)a.W * a.H);
}

// pm_stats: the histogram of a per-pixel class array (classes below n <= 8), one ballot per class
// and 32 pixels, summed per block in shared memory
__global__ void __launch_bounds__(256) count_classes_kernel(const uint8_t* __restrict__ cls, long npix, int n,
                                                            unsigned* g) {
    __shared__ unsigned s[8];
    if (threadIdx.x < 8) s[threadIdx.x] = 0u;
    __syncthreads();
    for (long base = (long)blockIdx.x * blockDim.x; base < npix; base += (long)gridDim.x * blockDim.x) {
        const long i = base + threadIdx.x;
        const int v = i < npix && PM_IN_BOUNDS(i, npix, kSiteClassCount) ? (int)cls[i] : -1;
        for (int c = 0; c < n; ++c) {
            const unsigned m = __ballot_sync(kFull, v == c);
            if ((threadIdx.x & 31) == 0 && m) atomicAdd(&s[c], (unsigned)__popc(m));
        }
    }
    __syncthreads();
    if (threadIdx.x < n && s[threadIdx.x]) atomicAdd(g + threadIdx.x, s[threadIdx.x]);
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
    int idx, cls;
    wta_filter<PPL>(s, incl, rk, lane, D, fp, dep, idx, cls);
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
    int dx, dy;
    pair_dir(pair, dx, dy);
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

cudaError_t launch_count_classes(const uint8_t* cls, long npix, int n, unsigned* g, cudaStream_t s) {
    if (n < 1 || n > 8 || npix < 0) return cudaErrorInvalidValue;
    if (npix == 0) return cudaSuccess;
    const long blocks = (npix + 255) / 256;
    count_classes_kernel<<<(unsigned)(blocks < 592 ? blocks : 592), 256, 0, s>>>(cls, npix, n, g);
    return cudaGetLastError();
}

}  // namespace pm
