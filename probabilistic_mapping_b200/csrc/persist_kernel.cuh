// persist_kernel.cuh -- the persistent kernel of the batched form (see persist.cu), included by
// one file per form so that the instantiations compile in parallel.
#pragma once

#include "cost_device.cuh"
#include "pm_persist.h"
#include "sgm_device.cuh"

namespace pm {
namespace {

constexpr int kThreads = 256;          // 8 warps: a cost tile's warps, eight SGM scanlines
constexpr long kSpinLimit = 1L << 20;  // polls of a completion counter before giving up

// Waits until *c >= target (acquire).  False when the wait ran out or another block gave up.
__device__ bool wait_counter(const unsigned* c, unsigned target, unsigned* err) {
    unsigned ns = 32;
    for (long it = 0; it < kSpinLimit; ++it) {
        unsigned v;
        asm volatile("ld.acquire.gpu.global.u32 %0, [%1];" : "=r"(v) : "l"(c) : "memory");
        if (v >= target) return true;
        if (*reinterpret_cast<volatile unsigned*>(err)) return false;
        __nanosleep(ns);
        if (ns < 1024) ns <<= 1;
    }
    atomicExch(err, 1u);
    return false;
}

template <int PPL, bool HALF, bool FULL>
__device__ __forceinline__ void sgm_item(const PersistSeq& q, int pair, int bx, unsigned char* smem) {
    int dx, dy;
    pair_dir(pair, dx, dy);
    sgm_pair_block<PPL, HALF, 8, FULL, HALF>(q.sgm, dx, dy, 2 * pair, bx, smem);
}

template <int PPL, bool HALF>
__device__ __forceinline__ void sgm_item_ppl(const PersistSeq& q, int pair, int bx, unsigned char* smem) {
    if (q.full) sgm_item<PPL, HALF, true>(q, pair, bx, smem);
    else sgm_item<PPL, HALF, false>(q, pair, bx, smem);
}

template <int PPL, bool HALF>
__device__ __forceinline__ void combine_item(const PersistSeq& q, long p0, long p1) {
    const long first = p0 + (threadIdx.x >> 5);
    if (q.sgm.num_paths == 8) combine_pixels<PPL, kCombineFilter, 4, HALF, true>(q.sgm, first, kThreads / 32, p1);
    else combine_pixels<PPL, kCombineFilter, 2, HALF, true>(q.sgm, first, kThreads / 32, p1);
}

template <int PPL>
__device__ __forceinline__ void rebase_item(const PersistSeq& q, long p0, long p1) {
    const int lane = threadIdx.x & 31;
    __half2* cost = static_cast<__half2*>(q.cost.cost);
    for (long g = p0 + (long)(threadIdx.x >> 5) * RB; g < p1; g += (long)(kThreads / 32) * RB)
        rebase_pixels<PPL, true>(cost, q.cost.block_offset, q.cost.offset, p1, q.cost.D, g, lane);
}

// Dispatch on the sequence's planes per lane (D / 32); the FP16 form has an even number.
template <bool HALF, int MAXPPL>
__device__ __forceinline__ void run_ppl(int type, const PersistSeq& q, const PersistItem& it, unsigned char* smem) {
#define PM_PERSIST_CASE(P)                                                                        \
    case P:                                                                                       \
        if constexpr (P <= MAXPPL && (!HALF || P % 2 == 0)) {                                     \
            if (type == kItemSgm) sgm_item_ppl<P, HALF>(q, it.sub, (int)it.idx, smem);             \
            else if (type == kItemCombine) combine_item<P, HALF>(q, it.idx, it.end);               \
            else if constexpr (HALF) rebase_item<P>(q, it.idx, it.end);                           \
        }                                                                                         \
        break;
    switch (q.ppl) {
        PM_PERSIST_CASE(1) PM_PERSIST_CASE(2) PM_PERSIST_CASE(3) PM_PERSIST_CASE(4)
        PM_PERSIST_CASE(5) PM_PERSIST_CASE(6) PM_PERSIST_CASE(7) PM_PERSIST_CASE(8)
        default: break;
    }
#undef PM_PERSIST_CASE
}

// Three blocks per SM where every sequence has at most 128 planes (the cost tiles then run at the
// stand-alone kernel's occupancy; 618 against 554 maps/s with two blocks at 640x480x128), two
// where the 8-plane-per-lane bodies need the registers.
template <int MODE, bool HALF, int SAMP, int MAXPPL>
__global__ void __launch_bounds__(kThreads, MAXPPL <= 4 ? 3 : 2)
persist_kernel(const PersistSeq* __restrict__ seqs, const PersistItem* __restrict__ items, int n_items,
               unsigned* cnt, unsigned* head, unsigned* err) {
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ int s_item;
    __shared__ int s_ok;
    for (;;) {
        if (threadIdx.x == 0) s_item = (int)atomicAdd(head, 1u);
        __syncthreads();
        const int i = s_item;
        if (i >= n_items) return;   // the same i in every thread
        const PersistItem it = items[i];
        const PersistSeq& q = seqs[it.seq];
        if (threadIdx.x == 0) {
            bool ok = true;
            if (it.wait_kind >= 0) ok = wait_counter(cnt + 4 * it.seq + it.wait_kind, it.wait_target, err);
            __threadfence();
            s_ok = ok;
        }
        __syncthreads();
        if (s_ok) {
            if (it.type == kItemCost) {
                const int gx = q.gx, gy = q.gy;
                const int t = (int)it.idx;
                cost_tile<MODE, HALF, SAMP, false>(q.cost, t % gx, (t / gx) % gy, t / (gx * gy), smem);
            } else {
                run_ppl<HALF, MAXPPL>(it.type, q, it, smem);
            }
        }
        __syncthreads();   // every thread's stores of the item precede the signal
        if (threadIdx.x == 0) {
            __threadfence();
            atomicAdd(cnt + 4 * it.seq + it.type, 1u);
        }
    }
}

template <int MODE, bool HALF, int SAMP, int MAXPPL>
cudaError_t launch_t(const PersistLaunch& L, cudaStream_t s) {
    auto kern = persist_kernel<MODE, HALF, SAMP, MAXPPL>;
    cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)L.smem_bytes);
    if (e != cudaSuccess) return e;
    int dev = 0, sms = 0, per_sm = 0;
    if ((e = cudaGetDevice(&dev)) != cudaSuccess) return e;
    if ((e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev)) != cudaSuccess) return e;
    if ((e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kern, kThreads, L.smem_bytes)) != cudaSuccess)
        return e;
    if (per_sm < 1) return cudaErrorInvalidConfiguration;
    const int grid = L.max_blocks > 0 && L.max_blocks < sms * per_sm ? L.max_blocks : sms * per_sm;
    kern<<<grid, kThreads, L.smem_bytes, s>>>(L.seqs, L.items, L.n_items, L.counters, L.counters + 4 * L.n_seqs,
                                               L.counters + 4 * L.n_seqs + 1);
    return cudaGetLastError();
}

// The kernel of one form for the batch's cost mode and largest planes per lane.
template <bool HALF, int SAMP>
cudaError_t launch_form(const PersistLaunch& L, cudaStream_t s) {
    if (L.mode == 0) return L.max_ppl <= 4 ? launch_t<0, HALF, SAMP, 4>(L, s) : launch_t<0, HALF, SAMP, 8>(L, s);
    return L.max_ppl <= 4 ? launch_t<1, HALF, SAMP, 4>(L, s) : launch_t<1, HALF, SAMP, 8>(L, s);
}

}  // namespace
}  // namespace pm
