// persist.cu -- the batched form's persistent kernel: the cost volume, its FP16 rebase, the SGM
// path pairs and the combine + winner-take-all of EVERY sequence of a batch in one launch.
//
// The work of a batch step is a list of items -- a cost tile (30x8 pixels x 16 planes), a range of
// pixels to rebase (FP16 form), a block of eight scanlines of one opposite-path pair, a range of
// pixels to combine -- built once when the batch is created and kept in device memory.  A grid of
// as many 256-thread blocks as the GPU holds at once takes the items in list order from one
// atomic counter.  An item that needs the results of other items (the rebase needs every cost
// tile of its sequence, the path pairs the rebased volume, the combine every path pair) waits on
// a per-sequence completion counter, which the producing items raise when they finish.  The list
// puts every item after everything it waits for, so the earliest unfinished item never waits on
// a later one: the schedule makes progress whatever the number of resident blocks.  The list
// interleaves the cost tiles of sequence s with the latency-bound SGM work of sequence s - 1, so
// the ALU-bound tiles fill the issue slots the path recurrences leave idle.  Every wait has an
// iteration limit: when it runs out the block records an error word (read by
// pm_batch_synchronize), skips the item, and the waits after it give up at once, so a failure
// ends the launch instead of hanging it.
//
// Data made by one item and read by another in the same launch is read through L2 only
// (cp.async.cg, ld.global.cg); a producer's stores are ordered before its counter increment by a
// block barrier and a device-scope fence, a consumer's reads after its acquire load by a barrier.
#include "cost_device.cuh"
#include "pm_persist.h"
#include "sgm_device.cuh"

namespace pm {

size_t persist_smem_bytes(int ppl, bool half) {
    const size_t ring = (size_t)8 * PF * 2 * 32 * (size_t)ppl * (half ? 2 : 4);   // eight scanlines' rings
    return ring > Smem::BYTES ? ring : Smem::BYTES;
}

cudaError_t launch_persist(const PersistLaunch& L, cudaStream_t s) {
    if (L.n_items <= 0) return cudaSuccess;
    switch (L.form) {   // the kernels of each form are compiled in their own file
        case kPersistFp32Quad: return launch_persist_fp32_quad(L, s);
        case kPersistFp32Tex: return launch_persist_fp32_tex(L, s);
        case kPersistFp16Tex: return launch_persist_fp16_tex(L, s);
        case kPersistFp16Quad: return launch_persist_fp16_quad(L, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace pm
