// pm_persist.h -- the batched form's persistent kernel (persist.cu): its work list and launch.
#pragma once

#include "pm_internal.h"

namespace pm {

// Item kinds; also the index of the per-sequence completion counter each kind raises.
enum PersistItemType { kItemCost = 0, kItemRebase = 1, kItemSgm = 2, kItemCombine = 3 };

// One sequence as the persistent kernel sees it (device memory).
struct PersistSeq {
    CostLaunch cost;       // hom_dev points at the step's homographies
    SgmLaunch sgm;         // part_half = cost_half
    int gx, gy;            // cost tiles along x and y (planes: D / 16 along z)
    int ppl;               // planes per lane, D / 32
    int full;              // every plane takes part in the minima (no inclusion masks)
};

// One item of the work list.  idx: cost tile, SGM block of eight scanlines, or first pixel of a
// range [idx, end); sub: the path pair of an SGM item.  The item may start once counter
// wait_kind of its sequence has reached wait_target (wait_kind < 0: at once).
struct PersistItem {
    uint16_t type, seq;
    int8_t wait_kind;
    uint8_t sub;
    uint16_t pad;
    uint32_t wait_target;
    int32_t idx, end;
};

// The forms the persistent kernel is built for: every sequence of a batch shares one.
enum PersistForm { kPersistFp32Quad = 0, kPersistFp32Tex = 1, kPersistFp16Tex = 2, kPersistFp16Quad = 3 };

struct PersistLaunch {
    const PersistSeq* seqs;   // device, n_seqs
    const PersistItem* items; // device, n_items
    int n_seqs, n_items;
    unsigned* counters;       // device: 4 per sequence, then the list head, then the error word;
                              // zeroed before every launch
    int mode;                 // cost mode shared by the sequences
    int form;                 // PersistForm
    int max_ppl;              // largest D / 32 of the batch
    size_t smem_bytes;        // persist_smem_bytes of the batch
    int max_blocks;           // 0: as many blocks as fit on the GPU
};

// Dynamic shared memory of a block: a cost tile's, or the SGM ring of eight scanlines at ppl.
size_t persist_smem_bytes(int ppl, bool half);
cudaError_t launch_persist(const PersistLaunch& L, cudaStream_t s);
// one per form (persist_<form>.cu)
cudaError_t launch_persist_fp32_quad(const PersistLaunch& L, cudaStream_t s);
cudaError_t launch_persist_fp32_tex(const PersistLaunch& L, cudaStream_t s);
cudaError_t launch_persist_fp16_tex(const PersistLaunch& L, cudaStream_t s);
cudaError_t launch_persist_fp16_quad(const PersistLaunch& L, cudaStream_t s);

}  // namespace pm
