// batch.cu -- the batched form: many independent sequences (each its own pm_config: resolution,
// plane count, precision, parameters) stepped together.
//
// One pm_batch_run is one keyframe of every sequence -- initReference, num_sources updates and
// outputFusion, exactly as the StereoMapper calls (stereo_mapper.cpp:63-244) -- issued as ONE
// CUDA-graph launch.  The graph is captured once: every value that changes from step to step
// (homographies, the relative pose of the fusion step, the first-keyframe flag and the state
// ping-pong index) lives in a small parameter block that the graph copies from pinned host
// memory into device memory at its start, and the kernels read it from there.  The sequences are
// independent branches of the graph, so the ALU-bound cost volume of one sequence runs beside the
// latency-bound SGM passes of others.  Sequences of the same shape share a pool of `lanes` sets
// of cost and path volumes (the large buffers), chained by graph dependencies, which bounds the
// memory of a large batch.  Two graph instances alternate by step parity over double-buffered
// parameter blocks and frame buffers, so the host prepares step t+1 while step t runs.
// An optional autotuner times the SGM schedules (scanlines per block of the path-pair kernel,
// concurrent or serial path pairs) for each distinct shape and keeps the fastest.  With
// PM_BATCH_PRIORITY the SGM kernels carry the device's greatest launch priority, so the block
// dispatcher hands freed SM slots to one sequence's latency-bound SGM before the queued blocks
// of another sequence's cost kernel, and the two overlap instead of running back to back.
#include <cuda_fp16.h>

#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <map>
#include <string>
#include <tuple>
#include <vector>

#include "pm_internal.h"
#include "pm_persist.h"
#include "pm_stereo.h"

namespace pm {
pm_status validate_config(const pm_config* c);
}

using namespace pm;

namespace {

// Large buffers one sequence needs only while its cost volume and SGM are in flight.
struct LaneBufs {
    void* cost = nullptr;
    float* off = nullptr;    // FP16 volumes: the per-pixel shift (see CostLaunch::offset)
    float* boff = nullptr;   // FP16 volumes: block offsets before the rebase
    float* part[4] = {};
    int last_user = -1;   // sequence index that used this set last in the capture order
};

struct Seq {
    pm_config cfg{};
    int S = 0;
    size_t N = 0, V = 0;
    double K[9]{};
    bool have_K = false;
    float cam[4]{};
    // frames (1 + S uint8 images of W*H) and the step parameter block, per buffer set
    uint8_t* h_frames[2] = {};   // pinned host (host I/O)
    uint8_t* d_frames[2] = {};
    float* h_par[2] = {};        // pinned host
    float* d_par[2] = {};
    size_t par_floats = 0;       // 12*S homographies, 12 pose + 4 cam, 2 ints
    float* h_out[2] = {};        // pinned host: fused depth then variance (host I/O)
    // persistent device state
    float* d_ref = nullptr;
    float4* d_srcq = nullptr;
    // texture samplers: pitched source images and their texture objects
    void* d_srch[kMaxSources] = {};
    size_t srch_pitch = 0;
    cudaTextureObject_t tex[kMaxSources] = {};
    float* d_depth = nullptr;
    int32_t* d_idx = nullptr;
    float* d_state[2][4] = {};
    unsigned long long* d_ztable = nullptr;
    int32_t* d_table = nullptr;
    float* d_fused = nullptr;
    float* d_var = nullptr;
    unsigned* d_stats = nullptr;   // PM_BATCH_STATS: the step's pm_stats counters
    uint8_t* d_cls = nullptr;      // PM_BATCH_STATS: W*H winner-take-all class of each pixel
    PlaneOrder order{};
    int lane = -1;               // index into the batch's lane sets
    // host step state (stereo_mapper.cpp:128-156)
    bool first = true;
    int pre_index = 0;
    double R_prev[9]{}, t_prev[3]{};
    double R_ref[9]{}, T_ref[3]{};
    std::vector<double> R_src, T_src;
    bool have_pose = false;
    // SGM schedule
    int pair_warps = 4, serial_pairs = 0;
    float tuned_ms = 0.0f;
    // capture streams and events
    cudaStream_t st[4] = {};
    SgmStreams side{};
    cudaEvent_t done = nullptr, lane_free = nullptr;
};

}  // namespace

struct pm_batch {
    std::vector<Seq> seqs;
    std::vector<LaneBufs> lanes;
    int S = 0;
    int flags = 0;
    int device = 0;
    int sgm_priority = 0;   // launch priority of the SGM kernels (PM_BATCH_PRIORITY)
    cudaStream_t run = nullptr;
    cudaEvent_t root = nullptr;
    cudaEvent_t launched[2] = {};
    cudaGraph_t graph[2] = {};
    cudaGraphExec_t exec[2] = {};
    bool built = false;
    long step = 0;
    std::string err;
    // PM_BATCH_PERSISTENT: the work list and per-sequence descriptors of the persistent kernel
    bool persistent = false;
    PersistSeq* d_pseq[2] = {};   // per buffer set (the homographies' device block differs)
    PersistItem* d_items = nullptr;
    unsigned* d_counters = nullptr;
    size_t counter_bytes = 0;
    PersistLaunch plaunch{};
    cudaEvent_t persist_done = nullptr;
};

namespace {

pm_status bfail(pm_batch* b, pm_status s, const char* fmt, ...) {
    if (b) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        b->err = buf;
    }
    return s;
}

#define PB_CK(b, call)                                                                          \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return bfail((b), e_ == cudaErrorMemoryAllocation ? PM_ERR_OUT_OF_MEMORY : PM_ERR_CUDA, \
                         "%s: %s", #call, cudaGetErrorString(e_));                              \
    } while (0)

struct DevGuard {
    int prev = -1;
    explicit DevGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DevGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

using ShapeKey = std::tuple<int, int, int, int, int>;   // W, H, D, precision, num_paths
ShapeKey key_of(const pm_config& c) { return {c.width, c.height, c.num_planes, c.precision, c.num_paths}; }

void free_batch(pm_batch* b) {
    for (int k = 0; k < 2; ++k) {
        if (b->exec[k]) cudaGraphExecDestroy(b->exec[k]);
        if (b->graph[k]) cudaGraphDestroy(b->graph[k]);
        if (b->launched[k]) cudaEventDestroy(b->launched[k]);
    }
    for (auto& l : b->lanes) {
        cudaFree(l.cost);
        cudaFree(l.off);
        cudaFree(l.boff);
        for (auto* p : l.part) cudaFree(p);
    }
    for (auto& q : b->seqs) {
        for (int k = 0; k < 2; ++k) {
            cudaFreeHost(q.h_frames[k]);
            cudaFree(q.d_frames[k]);
            cudaFreeHost(q.h_par[k]);
            cudaFree(q.d_par[k]);
            cudaFreeHost(q.h_out[k]);
        }
        cudaFree(q.d_ref);
        cudaFree(q.d_srcq);
        for (int s = 0; s < kMaxSources; ++s) {
            if (q.tex[s]) cudaDestroyTextureObject(q.tex[s]);
            cudaFree(q.d_srch[s]);
        }
        cudaFree(q.d_depth);
        cudaFree(q.d_idx);
        for (auto& s : q.d_state)
            for (auto* p : s) cudaFree(p);
        cudaFree(q.d_ztable);
        cudaFree(q.d_table);
        cudaFree(q.d_fused);
        cudaFree(q.d_var);
        cudaFree(q.d_stats);
        cudaFree(q.d_cls);
        for (auto& s : q.st)
            if (s) cudaStreamDestroy(s);
        if (q.side.fork) cudaEventDestroy(q.side.fork);
        for (auto& e : q.side.join)
            if (e) cudaEventDestroy(e);
        if (q.done) cudaEventDestroy(q.done);
        if (q.lane_free) cudaEventDestroy(q.lane_free);
    }
    if (b->root) cudaEventDestroy(b->root);
    if (b->persist_done) cudaEventDestroy(b->persist_done);
    for (auto* p : b->d_pseq) cudaFree(p);
    cudaFree(b->d_items);
    cudaFree(b->d_counters);
    if (b->run) cudaStreamDestroy(b->run);
}

SgmLaunch sgm_launch(const Seq& q, const LaneBufs& l, int priority) {
    SgmLaunch a;
    std::memset(&a, 0, sizeof a);
    const pm_config& c = q.cfg;
    a.cost = l.cost;
    a.offset = l.off;
    a.cost_half = c.precision == PM_PREC_FP16;
    a.ref = q.d_ref;
    for (int r = 0; r < c.num_paths / 2; ++r) a.part[r] = l.part[r];
    a.part_half = a.cost_half;   // the FP16 form keeps its pair volumes in FP16
    a.W = c.width;
    a.H = c.height;
    a.D = c.num_planes;
    a.num_paths = c.num_paths;
    a.p1 = c.p1; a.p2 = c.p2; a.tau = c.tau_so; a.q1 = c.q1; a.q2 = c.q2;
    a.fp.var_scale = c.var_scale;
    a.fp.uniq = c.uniqueness_ratio;
    a.fp.rho0 = c.rho0;
    a.fp.drho = c.rho_step;
    a.depth = q.d_depth;
    a.depth_pitch = sizeof(float) * (size_t)c.width;
    a.index = q.d_idx;
    a.wta_class = q.d_cls;
    a.order = q.order;
    a.pair_warps = q.pair_warps;
    a.serial_pairs = q.serial_pairs;
    a.priority = priority;
    return a;
}

// The parameter block, the frames and their conversions of one sequence for buffer set k.
cudaError_t enqueue_inputs(pm_batch* b, int i, int k, cudaStream_t m) {
    Seq& q = b->seqs[i];
    const pm_config& c = q.cfg;
    const int W = c.width, H = c.height, S = q.S;
    const size_t N = q.N;
    const bool host = b->flags & PM_BATCH_HOST_IO;
    const bool half = c.precision == PM_PREC_FP16;
    cudaError_t e;
    if ((e = cudaMemcpyAsync(q.d_par[k], q.h_par[k], sizeof(float) * q.par_floats, cudaMemcpyHostToDevice, m)))
        return e;
    if (host && (e = cudaMemcpyAsync(q.d_frames[k], q.h_frames[k], (1 + S) * N, cudaMemcpyHostToDevice, m)))
        return e;
    const float sc = c.intensity_scale;
    e = half ? launch_to_float_h(W, H, q.d_frames[k], W, q.d_ref, sc, m)
             : launch_to_float(W, H, q.d_frames[k], W, q.d_ref, sc, m);
    if (e) return e;
    for (int s = 0; s < S; ++s) {
        const uint8_t* f = q.d_frames[k] + (1 + s) * N;
        if (c.sampler == PM_SAMPLER_TEXTURE)
            e = launch_to_half(W, H, f, W, q.d_srch[s], q.srch_pitch, sc, m);
        else if (c.sampler == PM_SAMPLER_TEXTURE_F32)
            e = half ? launch_to_float_h_pitched(W, H, f, W, (float*)q.d_srch[s], q.srch_pitch, sc, m)
                     : launch_to_float_pitched(W, H, f, W, (float*)q.d_srch[s], q.srch_pitch, sc, m);
        else
            e = half ? launch_to_quad_half(W, H, f, W, q.d_srcq + (size_t)s * N, sc, m)
                     : launch_to_quad(W, H, f, W, q.d_srcq + (size_t)s * N, sc, m);
        if (e) return e;
    }
    return cudaSuccess;
}

// The cost pass of one sequence (calc_cost.cu:212-253 for all its sources at once).
CostLaunch cost_launch(const Seq& q, const LaneBufs& l, int k) {
    const pm_config& c = q.cfg;
    CostLaunch a;
    std::memset(&a, 0, sizeof a);
    a.ref = q.d_ref;
    a.srcq = q.d_srcq;
    if (c.sampler != PM_SAMPLER_EXACT) {
        a.use_tex = 1;
        for (int s = 0; s < q.S; ++s) a.tex[s] = q.tex[s];
    }
    a.offset = l.off;
    a.block_offset = l.boff;
    a.W = c.width;
    a.H = c.height;
    a.D = c.num_planes;
    a.nsrc = q.S;
    a.rho0 = c.rho0;
    a.drho = c.rho_step;
    a.mode = c.cost_mode;
    a.hom_dev = q.d_par[k];
    a.cost = l.cost;
    a.cost_half = c.precision == PM_PREC_FP16;
    return a;
}

// The fusion step of one sequence (stereo_mapper.cpp:111-244) with the step's pose, flags and
// state index from its parameter block, and the host copies of its outputs.
cudaError_t enqueue_fusion(pm_batch* b, int i, int k, cudaStream_t m) {
    Seq& q = b->seqs[i];
    const size_t N = q.N;
    cudaError_t e;
    FuseLaunch f;
    std::memset(&f, 0, sizeof f);
    f.W = q.cfg.width;
    f.H = q.cfg.height;
    f.depth = q.d_fused;      // written from the WTA depth by the update kernel
    f.depth_in = q.d_depth;
    f.ztable = q.d_ztable;
    f.table = q.d_table;
    f.variance = q.d_var;
    f.params_dev = q.d_par[k] + 12 * q.S;
    f.flags_dev = reinterpret_cast<const int*>(q.d_par[k] + 12 * q.S + 16);
    for (int s = 0; s < 2; ++s)
        for (int j = 0; j < 4; ++j) f.state[s][j] = q.d_state[s][j];
    f.stats = q.d_stats;
    if ((e = launch_fuse_gpu(f, m))) return e;
    if (b->flags & PM_BATCH_HOST_IO) {
        if ((e = cudaMemcpyAsync(q.h_out[k], q.d_fused, 4 * N, cudaMemcpyDeviceToHost, m))) return e;
        if ((e = cudaMemcpyAsync(q.h_out[k] + N, q.d_var, 4 * N, cudaMemcpyDeviceToHost, m))) return e;
    }
    return cudaSuccess;
}

// PM_BATCH_STATS: the step's counters start from zero; the winner-take-all classes are counted
// once the combine kernel has written them.
cudaError_t clear_stats(const Seq& q, cudaStream_t m) {
    return q.d_stats ? cudaMemsetAsync(q.d_stats, 0, sizeof(unsigned) * kStatWords, m) : cudaSuccess;
}
cudaError_t count_wta_classes(const Seq& q, cudaStream_t m) {
    return q.d_stats ? launch_count_classes(q.d_cls, (long)q.N, kWtaClasses, q.d_stats + kStatWta, m) : cudaSuccess;
}

// The work of one sequence for buffer set k, on its own streams (captured into the graph).
cudaError_t enqueue_seq(pm_batch* b, int i, int k) {
    Seq& q = b->seqs[i];
    LaneBufs& l = b->lanes[q.lane];
    cudaStream_t m = q.st[0];
    cudaError_t e;
    if ((e = enqueue_inputs(b, i, k, m))) return e;
    if ((e = clear_stats(q, m))) return e;
    // the lane's volumes are free once the previous sequence in this lane has finished its SGM
    if (l.last_user >= 0 && (e = cudaStreamWaitEvent(m, b->seqs[l.last_user].lane_free, 0))) return e;
    l.last_user = i;
    if ((e = launch_cost(cost_launch(q, l, k), m))) return e;
    const SgmLaunch g = sgm_launch(q, l, b->sgm_priority);
    if ((e = launch_sgm(g, kCombineFilter, m, &q.side))) return e;
    if ((e = cudaEventRecord(q.lane_free, m))) return e;
    if ((e = count_wta_classes(q, m))) return e;
    return enqueue_fusion(b, i, k, m);
}

// ---- the persistent form -------------------------------------------------------------------
constexpr int kRebaseRange = 1024;    // pixels per rebase item (a multiple of 8 warps x RB)
constexpr int kCombineRange = 2048;   // pixels per combine item

// Blocks of eight scanlines of path pair p: rows (L/R), columns (T/B), diagonals.
int sgm_blocks(const pm_config& c, int pair) {
    const int n = pair == 0 ? c.height : (pair == 1 ? c.width : c.width + c.height - 1);
    return (n + 7) / 8;
}

// The work list: the cost tiles of sequence s interleaved with the rebase, SGM and combine items
// of sequence s - 1 (spread evenly among them), so every item comes after what it waits for.
std::vector<PersistItem> persist_items(const pm_batch* b) {
    const int n = (int)b->seqs.size();
    std::vector<std::vector<PersistItem>> C(n), P(n);
    auto item = [](int type, int seq, int wait_kind, unsigned target, int idx, int end, int sub) {
        PersistItem it{};
        it.type = (uint16_t)type;
        it.seq = (uint16_t)seq;
        it.wait_kind = (int8_t)wait_kind;
        it.wait_target = target;
        it.idx = idx;
        it.end = end;
        it.sub = (uint8_t)sub;
        return it;
    };
    for (int s = 0; s < n; ++s) {
        const pm_config& c = b->seqs[s].cfg;
        const int npix = c.width * c.height;
        const int ncost = ((c.width + 29) / 30) * ((c.height + 7) / 8) * (c.num_planes / 16);
        for (int t = 0; t < ncost; ++t) C[s].push_back(item(kItemCost, s, -1, 0, t, 0, 0));
        int wait_kind = kItemCost;
        unsigned target = (unsigned)ncost;
        if (c.precision == PM_PREC_FP16) {
            unsigned nr = 0;
            for (int p0 = 0; p0 < npix; p0 += kRebaseRange, ++nr)
                P[s].push_back(item(kItemRebase, s, kItemCost, ncost, p0, std::min(npix, p0 + kRebaseRange), 0));
            wait_kind = kItemRebase;
            target = nr;
        }
        unsigned ng = 0;
        for (int pair = 0; pair < c.num_paths / 2; ++pair)
            for (int bx = 0; bx < sgm_blocks(c, pair); ++bx, ++ng)
                P[s].push_back(item(kItemSgm, s, wait_kind, target, bx, 0, pair));
        for (int p0 = 0; p0 < npix; p0 += kCombineRange)
            P[s].push_back(item(kItemCombine, s, kItemSgm, ng, p0, std::min(npix, p0 + kCombineRange), 0));
    }
    std::vector<PersistItem> out(C[0]);
    for (int s = 1; s <= n; ++s) {
        const std::vector<PersistItem>& c = s < n ? C[s] : std::vector<PersistItem>();
        const std::vector<PersistItem>& p = P[s - 1];
        size_t j = 0;
        for (size_t i = 0; i < c.size(); ++i) {
            out.push_back(c[i]);
            const size_t upto = (i + 1) * p.size() / c.size();
            while (j < upto) out.push_back(p[j++]);
        }
        while (j < p.size()) out.push_back(p[j++]);
    }
    return out;
}

int persist_form(const pm_config& c) {
    if (c.precision == PM_PREC_FP16) return c.sampler == PM_SAMPLER_EXACT ? kPersistFp16Quad : kPersistFp16Tex;
    return c.sampler == PM_SAMPLER_EXACT ? kPersistFp32Quad : kPersistFp32Tex;
}

// Descriptors (both buffer sets), the work list and the counters; called once the plane
// spacings are known (at the first run).
pm_status setup_persist(pm_batch* b) {
    const int n = (int)b->seqs.size();
    std::vector<PersistSeq> h((size_t)n);
    int max_ppl = 1;
    size_t smem = 0;
    for (int k = 0; k < 2; ++k) {
        for (int i = 0; i < n; ++i) {
            const Seq& q = b->seqs[i];
            const LaneBufs& l = b->lanes[q.lane];
            PersistSeq& d = h[i];
            std::memset(&d, 0, sizeof d);
            d.cost = cost_launch(q, l, k);
            d.sgm = sgm_launch(q, l, 0);
            d.gx = (q.cfg.width + 29) / 30;
            d.gy = (q.cfg.height + 7) / 8;
            d.ppl = q.cfg.num_planes / 32;
            d.full = 1;
            for (int ln = 0; ln < 32; ++ln) d.full &= q.order.incl[ln] == (1u << d.ppl) - 1u;
            max_ppl = std::max(max_ppl, d.ppl);
            smem = std::max(smem, persist_smem_bytes(d.ppl, q.cfg.precision == PM_PREC_FP16));
        }
        if (!b->d_pseq[k]) PB_CK(b, cudaMalloc((void**)&b->d_pseq[k], sizeof(PersistSeq) * n));
        PB_CK(b, cudaMemcpy(b->d_pseq[k], h.data(), sizeof(PersistSeq) * n, cudaMemcpyHostToDevice));
    }
    const std::vector<PersistItem> items = persist_items(b);
    if (!b->d_items) PB_CK(b, cudaMalloc((void**)&b->d_items, sizeof(PersistItem) * items.size()));
    PB_CK(b, cudaMemcpy(b->d_items, items.data(), sizeof(PersistItem) * items.size(), cudaMemcpyHostToDevice));
    b->counter_bytes = sizeof(unsigned) * (4 * (size_t)n + 2);
    if (!b->d_counters) PB_CK(b, cudaMalloc((void**)&b->d_counters, b->counter_bytes));
    PB_CK(b, cudaMemset(b->d_counters, 0, b->counter_bytes));
    PersistLaunch& L = b->plaunch;
    L.items = b->d_items;
    L.n_seqs = n;
    L.n_items = (int)items.size();
    L.counters = b->d_counters;
    L.mode = b->seqs[0].cfg.cost_mode;
    L.form = persist_form(b->seqs[0].cfg);
    L.max_ppl = max_ppl;
    L.smem_bytes = smem;
    L.max_blocks = 0;
    return PM_OK;
}

// One step of the persistent form for buffer set k: the inputs of every sequence on its own
// stream, then the persistent kernel on the run stream, then every sequence's fusion step.
cudaError_t enqueue_persist(pm_batch* b, int k) {
    cudaError_t e;
    for (int i = 0; i < (int)b->seqs.size(); ++i) {
        Seq& q = b->seqs[i];
        if ((e = cudaStreamWaitEvent(q.st[0], b->root, 0))) return e;
        if ((e = enqueue_inputs(b, i, k, q.st[0]))) return e;
        if ((e = clear_stats(q, q.st[0]))) return e;
        if ((e = cudaEventRecord(q.side.fork, q.st[0]))) return e;
        if ((e = cudaStreamWaitEvent(b->run, q.side.fork, 0))) return e;
    }
    if ((e = cudaMemsetAsync(b->d_counters, 0, b->counter_bytes, b->run))) return e;
    PersistLaunch L = b->plaunch;
    L.seqs = b->d_pseq[k];
    if ((e = launch_persist(L, b->run))) return e;
    if ((e = cudaEventRecord(b->persist_done, b->run))) return e;
    for (int i = 0; i < (int)b->seqs.size(); ++i) {
        Seq& q = b->seqs[i];
        if ((e = cudaStreamWaitEvent(q.st[0], b->persist_done, 0))) return e;
        if ((e = count_wta_classes(q, q.st[0]))) return e;
        if ((e = enqueue_fusion(b, i, k, q.st[0]))) return e;
        if ((e = cudaEventRecord(q.done, q.st[0]))) return e;
        if ((e = cudaStreamWaitEvent(b->run, q.done, 0))) return e;
    }
    return cudaSuccess;
}

pm_status build_graphs(pm_batch* b) {
    if (b->persistent) {
        pm_status st = setup_persist(b);
        if (st != PM_OK) return st;
    }
    for (int k = 0; k < 2; ++k) {
        for (auto& l : b->lanes) l.last_user = -1;
        PB_CK(b, cudaStreamBeginCapture(b->run, cudaStreamCaptureModeThreadLocal));
        cudaError_t e = cudaEventRecord(b->root, b->run);
        if (b->persistent && e == cudaSuccess) e = enqueue_persist(b, k);
        for (int i = 0; !b->persistent && i < (int)b->seqs.size() && e == cudaSuccess; ++i) {
            Seq& q = b->seqs[i];
            e = cudaStreamWaitEvent(q.st[0], b->root, 0);
            if (e == cudaSuccess) e = enqueue_seq(b, i, k);
            if (e == cudaSuccess) e = cudaEventRecord(q.done, q.st[0]);
            if (e == cudaSuccess) e = cudaStreamWaitEvent(b->run, q.done, 0);
        }
        cudaGraph_t g = nullptr;
        const cudaError_t ee = cudaStreamEndCapture(b->run, &g);
        if (e != cudaSuccess || ee != cudaSuccess) {
            if (g) cudaGraphDestroy(g);
            cudaGetLastError();
            return bfail(b, PM_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e != cudaSuccess ? e : ee));
        }
        b->graph[k] = g;
        // with PM_BATCH_PRIORITY the SGM nodes keep their own (higher) priority
        PB_CK(b, cudaGraphInstantiateWithFlags(&b->exec[k], g,
                                               b->sgm_priority ? cudaGraphInstantiateFlagUseNodePriority : 0));
    }
    b->built = true;
    return PM_OK;
}

// Times the SGM stage of one sequence per distinct shape for every schedule candidate and keeps
// the fastest for all sequences of that shape.
pm_status autotune(pm_batch* b) {
    std::map<ShapeKey, int> done;
    cudaEvent_t t0, t1;
    PB_CK(b, cudaEventCreate(&t0));
    PB_CK(b, cudaEventCreate(&t1));
    pm_status st = PM_OK;
    for (int i = 0; i < (int)b->seqs.size() && st == PM_OK; ++i) {
        Seq& q = b->seqs[i];
        auto it = done.find(key_of(q.cfg));
        if (it != done.end()) {
            const Seq& t = b->seqs[it->second];
            q.pair_warps = t.pair_warps;
            q.serial_pairs = t.serial_pairs;
            q.tuned_ms = t.tuned_ms;
            continue;
        }
        LaneBufs& l = b->lanes[q.lane];
        const size_t esz = q.cfg.precision == PM_PREC_FP16 ? 2 : 4;
        float best = 1e30f;
        int bw = 4, bs = 0;
        const int warps[3] = {2, 4, 8};
        cudaError_t e = cudaMemsetAsync(l.cost, 0, esz * q.V, b->run);
        if (e == cudaSuccess) e = cudaMemsetAsync(q.d_ref, 0, 4 * q.N, b->run);
        for (int w : warps)
            for (int serial = 0; serial < 2 && e == cudaSuccess; ++serial) {
                q.pair_warps = w;
                q.serial_pairs = serial;
                const SgmLaunch g = sgm_launch(q, l, 0);
                e = launch_sgm(g, kCombineFilter, b->run, &q.side);   // warm-up
                if (e == cudaSuccess) e = cudaEventRecord(t0, b->run);
                for (int r = 0; r < 3 && e == cudaSuccess; ++r) e = launch_sgm(g, kCombineFilter, b->run, &q.side);
                if (e == cudaSuccess) e = cudaEventRecord(t1, b->run);
                if (e == cudaSuccess) e = cudaEventSynchronize(t1);
                float ms = 0.0f;
                if (e == cudaSuccess) e = cudaEventElapsedTime(&ms, t0, t1);
                ms /= 3.0f;
                if (e == cudaSuccess && ms < best) {
                    best = ms;
                    bw = w;
                    bs = serial;
                }
            }
        if (e != cudaSuccess) st = bfail(b, PM_ERR_CUDA, "autotune: %s", cudaGetErrorString(e));
        q.pair_warps = bw;
        q.serial_pairs = bs;
        q.tuned_ms = best;
        done[key_of(q.cfg)] = i;
    }
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    return st;
}

}  // namespace

extern "C" {

pm_status pm_batch_create(const pm_config* cfgs, int n, int num_sources, int lanes, int flags, pm_batch** out) {
    if (!out) return PM_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (!cfgs || n < 1 || num_sources < 1 || num_sources > kMaxSources || lanes < 0)
        return PM_ERR_INVALID_ARGUMENT;
    for (int i = 0; i < n; ++i) {
        if (validate_config(&cfgs[i]) != PM_OK) return PM_ERR_INVALID_ARGUMENT;
        if (cfgs[i].fusion_variant != PM_FUSION_GPU || cfgs[i].device != cfgs[0].device)
            return PM_ERR_UNSUPPORTED;
    }
    if (flags & PM_BATCH_PERSISTENT) {   // one form for all sequences, each with its own volumes
        if (lanes != 0) return PM_ERR_UNSUPPORTED;
        for (int i = 1; i < n; ++i)
            if (cfgs[i].precision != cfgs[0].precision || cfgs[i].sampler != cfgs[0].sampler ||
                cfgs[i].cost_mode != cfgs[0].cost_mode)
                return PM_ERR_UNSUPPORTED;
        if (n > 65535) return PM_ERR_UNSUPPORTED;
    }
    pm_batch* b = new pm_batch();
    b->S = num_sources;
    b->flags = flags;
    b->device = cfgs[0].device;
    b->persistent = (flags & PM_BATCH_PERSISTENT) != 0;
    DevGuard dg(b->device);
    if (flags & PM_BATCH_PRIORITY) {
        int least = 0, greatest = 0;
        if (cudaDeviceGetStreamPriorityRange(&least, &greatest) == cudaSuccess) b->sgm_priority = greatest;
    }
    cudaError_t first_err = cudaSuccess;
    auto note = [&](cudaError_t e) {
        if (e != cudaSuccess && first_err == cudaSuccess) first_err = e;
        return e == cudaSuccess;
    };
    auto alloc = [&](void** p, size_t bytes) { return note(cudaMalloc(p, bytes)); };
    bool ok = note(cudaStreamCreateWithFlags(&b->run, cudaStreamNonBlocking)) &&
              note(cudaEventCreateWithFlags(&b->root, cudaEventDisableTiming)) &&
              note(cudaEventCreateWithFlags(&b->launched[0], cudaEventDisableTiming)) &&
              note(cudaEventCreateWithFlags(&b->persist_done, cudaEventDisableTiming)) &&
              note(cudaEventCreateWithFlags(&b->launched[1], cudaEventDisableTiming));
    b->seqs.resize(n);
    // lanes: per distinct shape, `lanes` sets of cost + path volumes (0: one per sequence)
    std::map<ShapeKey, std::vector<int>> lane_of_shape;
    std::map<ShapeKey, int> count_of_shape;
    for (int i = 0; i < n && ok; ++i) {
        Seq& q = b->seqs[i];
        q.cfg = cfgs[i];
        q.S = num_sources;
        q.N = (size_t)q.cfg.width * q.cfg.height;
        q.V = q.N * q.cfg.num_planes;
        q.par_floats = 12 * (size_t)q.S + 16 + 2;
        q.R_src.assign(9 * (size_t)q.S, 0.0);
        q.T_src.assign(3 * (size_t)q.S, 0.0);
        plane_order(q.cfg.num_planes, q.cfg.tree_compat, q.order);
        const ShapeKey key = key_of(q.cfg);
        const int j = count_of_shape[key]++;
        std::vector<int>& pool = lane_of_shape[key];
        if (lanes == 0 || (int)pool.size() < lanes) {
            pool.push_back((int)b->lanes.size());
            LaneBufs l;
            const size_t esz = q.cfg.precision == PM_PREC_FP16 ? 2 : 4;
            ok = alloc(&l.cost, esz * q.V);
            if (ok && esz == 2)
                ok = alloc((void**)&l.off, 4 * q.N) && note(cudaMemset(l.off, 0, 4 * q.N)) &&
                     alloc((void**)&l.boff, 4 * q.N * (q.cfg.num_planes / 16));
            // the FP16 form keeps its pair volumes in FP16 (SgmLaunch::part_half)
            for (int r = 0; r < q.cfg.num_paths / 2 && ok; ++r) ok = alloc((void**)&l.part[r], esz * q.V);
            b->lanes.push_back(l);
            if (!ok) break;
        }
        q.lane = pool[lanes == 0 ? j : j % lanes];
        const size_t N = q.N;
        for (int k = 0; k < 2 && ok; ++k) {
            ok = note(cudaMallocHost((void**)&q.h_par[k], sizeof(float) * q.par_floats)) &&
                 alloc((void**)&q.d_par[k], sizeof(float) * q.par_floats) &&
                 alloc((void**)&q.d_frames[k], (1 + q.S) * N);
            if (ok && (flags & PM_BATCH_HOST_IO))
                ok = note(cudaMallocHost((void**)&q.h_frames[k], (1 + q.S) * N)) &&
                     note(cudaMallocHost((void**)&q.h_out[k], 2 * 4 * N));
            if (ok) std::memset(q.h_par[k], 0, sizeof(float) * q.par_floats);
        }
        ok = ok && alloc((void**)&q.d_ref, 4 * N) &&
             (q.cfg.sampler != PM_SAMPLER_EXACT || alloc((void**)&q.d_srcq, 16 * N * q.S)) &&
             alloc((void**)&q.d_depth, 4 * N) && alloc((void**)&q.d_idx, 4 * N) &&
             alloc((void**)&q.d_ztable, 8 * N) && alloc((void**)&q.d_table, 4 * N) &&
             alloc((void**)&q.d_fused, 4 * N) && alloc((void**)&q.d_var, 4 * N) &&
             (!(flags & PM_BATCH_STATS) ||
              (alloc((void**)&q.d_stats, sizeof(unsigned) * kStatWords) && alloc((void**)&q.d_cls, N) &&
               note(cudaMemset(q.d_stats, 0, sizeof(unsigned) * kStatWords))));
        for (int s = 0; s < 2 && ok; ++s)
            for (int k = 0; k < 4 && ok; ++k) ok = alloc((void**)&q.d_state[s][k], 4 * N);
        for (int s = 0; q.cfg.sampler != PM_SAMPLER_EXACT && s < q.S && ok; ++s)
            ok = note(make_source_texture(q.cfg.width, q.cfg.height, q.cfg.sampler == PM_SAMPLER_TEXTURE_F32,
                                          &q.d_srch[s], &q.srch_pitch, &q.tex[s]));
        for (int s = 0; s < 4 && ok; ++s) ok = note(cudaStreamCreateWithFlags(&q.st[s], cudaStreamNonBlocking));
        if (ok) {
            for (int s = 0; s < 3; ++s) q.side.stream[s] = q.st[1 + s];
            ok = note(cudaEventCreateWithFlags(&q.side.fork, cudaEventDisableTiming)) &&
                 note(cudaEventCreateWithFlags(&q.done, cudaEventDisableTiming)) &&
                 note(cudaEventCreateWithFlags(&q.lane_free, cudaEventDisableTiming));
            for (int s = 0; s < 3 && ok; ++s)
                ok = note(cudaEventCreateWithFlags(&q.side.join[s], cudaEventDisableTiming));
        }
    }
    pm_status tune = PM_OK;
    if (ok && (flags & PM_BATCH_AUTOTUNE) && !b->persistent) {
        tune = autotune(b);
        ok = tune == PM_OK;
    }
    if (ok) ok = note(cudaStreamSynchronize(b->run));
    if (!ok) {
        cudaGetLastError();
        free_batch(b);
        delete b;
        if (tune != PM_OK) return tune;
        return first_err == cudaErrorMemoryAllocation ? PM_ERR_OUT_OF_MEMORY : PM_ERR_CUDA;
    }
    *out = b;
    return PM_OK;
}

void pm_batch_destroy(pm_batch* b) {
    if (!b) return;
    DevGuard dg(b->device);
    if (b->run) cudaStreamSynchronize(b->run);
    free_batch(b);
    delete b;
}

pm_status pm_batch_init_intrinsic(pm_batch* b, int seq, const double K[9], float dep_sample) {
    if (!b) return PM_ERR_INVALID_ARGUMENT;
    if (seq < 0 || seq >= (int)b->seqs.size()) return bfail(b, PM_ERR_INVALID_ARGUMENT, "no sequence %d", seq);
    if (!K || !finite_n(K, 9) || K[0] == 0.0 || K[4] == 0.0 || K[3] != 0.0 || K[6] != 0.0 || K[7] != 0.0 ||
        K[8] != 1.0)
        return bfail(b, PM_ERR_INVALID_ARGUMENT, "K must be upper triangular with K[2][2] = 1 and nonzero fx, fy");
    if (!(dep_sample > 0.0f)) return bfail(b, PM_ERR_INVALID_ARGUMENT, "dep_sample must be positive");
    if (b->built && dep_sample != b->seqs[seq].cfg.rho_step)
        return bfail(b, PM_ERR_BAD_STATE, "the plane spacing is fixed once the batch has run");
    Seq& q = b->seqs[seq];
    std::memcpy(q.K, K, sizeof q.K);
    q.have_K = true;
    q.cfg.rho_step = dep_sample;
    q.cam[0] = (float)K[0];
    q.cam[1] = (float)K[4];
    q.cam[2] = (float)K[2];
    q.cam[3] = (float)K[5];
    return PM_OK;
}

pm_status pm_batch_frame(pm_batch* b, int seq, int frame, uint8_t** ptr) {
    if (!b || !ptr) return PM_ERR_INVALID_ARGUMENT;
    if (seq < 0 || seq >= (int)b->seqs.size() || frame < 0 || frame > b->S)
        return bfail(b, PM_ERR_INVALID_ARGUMENT, "no frame %d of sequence %d", frame, seq);
    DevGuard dg(b->device);
    const int k = (int)(b->step & 1);
    // the set is free once the launch two steps back (which read it) has completed
    if (b->step >= 2) PB_CK(b, cudaEventSynchronize(b->launched[k]));
    Seq& q = b->seqs[seq];
    uint8_t* base = (b->flags & PM_BATCH_HOST_IO) ? q.h_frames[k] : q.d_frames[k];
    *ptr = base + (size_t)frame * q.N;
    return PM_OK;
}

pm_status pm_batch_put_frame(pm_batch* b, int seq, int frame, const uint8_t* img, size_t pitch) {
    if (!b || !img) return PM_ERR_INVALID_ARGUMENT;
    uint8_t* dst = nullptr;
    pm_status st = pm_batch_frame(b, seq, frame, &dst);
    if (st != PM_OK) return st;
    const Seq& q = b->seqs[seq];
    const int W = q.cfg.width, H = q.cfg.height;
    if (pitch == 0) pitch = (size_t)W;
    if (pitch < (size_t)W) return bfail(b, PM_ERR_INVALID_ARGUMENT, "image pitch %zu < width %d", pitch, W);
    cudaPointerAttributes at;
    const bool dev_src = cudaPointerGetAttributes(&at, img) == cudaSuccess &&
                         (at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged);
    cudaGetLastError();
    DevGuard dg(b->device);
    if (b->flags & PM_BATCH_HOST_IO) {
        if (dev_src) {
            PB_CK(b, cudaMemcpy2D(dst, (size_t)W, img, pitch, (size_t)W, (size_t)H, cudaMemcpyDeviceToHost));
        } else {
            for (int y = 0; y < H; ++y) std::memcpy(dst + (size_t)y * W, img + (size_t)y * pitch, (size_t)W);
        }
    } else {
        PB_CK(b, cudaMemcpy2DAsync(dst, (size_t)W, img, pitch, (size_t)W, (size_t)H,
                                   dev_src ? cudaMemcpyDeviceToDevice : cudaMemcpyHostToDevice, b->run));
    }
    return PM_OK;
}

pm_status pm_batch_set_poses(pm_batch* b, int seq, const double R_ref[9], const double T_ref[3], const double* R_src,
                             const double* T_src) {
    if (!b) return PM_ERR_INVALID_ARGUMENT;
    if (seq < 0 || seq >= (int)b->seqs.size()) return bfail(b, PM_ERR_INVALID_ARGUMENT, "no sequence %d", seq);
    Seq& q = b->seqs[seq];
    if (!R_ref || !T_ref || !R_src || !T_src || !finite_n(R_ref, 9) || !finite_n(T_ref, 3) ||
        !finite_n(R_src, 9 * q.S) || !finite_n(T_src, 3 * q.S))
        return bfail(b, PM_ERR_INVALID_ARGUMENT, "poses must be finite");
    std::memcpy(q.R_ref, R_ref, sizeof q.R_ref);
    std::memcpy(q.T_ref, T_ref, sizeof q.T_ref);
    std::memcpy(q.R_src.data(), R_src, sizeof(double) * 9 * q.S);
    std::memcpy(q.T_src.data(), T_src, sizeof(double) * 3 * q.S);
    q.have_pose = true;
    return PM_OK;
}

pm_status pm_batch_run(pm_batch* b) {
    if (!b) return PM_ERR_INVALID_ARGUMENT;
    DevGuard dg(b->device);
    for (int i = 0; i < (int)b->seqs.size(); ++i) {
        const Seq& q = b->seqs[i];
        if (!q.have_K) return bfail(b, PM_ERR_BAD_STATE, "sequence %d: run before init_intrinsic", i);
        if (!q.have_pose) return bfail(b, PM_ERR_BAD_STATE, "sequence %d: run before set_poses", i);
    }
    if (!b->built) {
        pm_status st = build_graphs(b);
        if (st != PM_OK) return st;
    }
    const int k = (int)(b->step & 1);
    if (b->step >= 2) PB_CK(b, cudaEventSynchronize(b->launched[k]));
    for (auto& q : b->seqs) {
        float* par = q.h_par[k];
        for (int s = 0; s < q.S; ++s)   // initReference + update of every source (stereo_mapper.cpp:79-80)
            compose_homography(q.K, q.R_ref, q.T_ref, &q.R_src[9 * s], &q.T_src[3 * s], par + 12 * s);
        float* pose = par + 12 * q.S;
        int* flags = reinterpret_cast<int*>(pose + 16);
        std::memcpy(pose + 12, q.cam, sizeof q.cam);
        if (q.first) {   // stereo_mapper.cpp:128-146
            q.first = false;
            q.pre_index = 0;
            std::memset(pose, 0, 12 * sizeof(float));
            flags[0] = 1;
            flags[1] = 0;
        } else {
            fusion_pose(q.R_ref, q.T_ref, q.R_prev, q.t_prev, pose);
            flags[0] = 0;
            flags[1] = q.pre_index;
            q.pre_index ^= 1;   // stereo_mapper.cpp:237-241
        }
        std::memcpy(q.R_prev, q.R_ref, sizeof q.R_prev);
        std::memcpy(q.t_prev, q.T_ref, sizeof q.t_prev);
    }
    PB_CK(b, cudaGraphLaunch(b->exec[k], b->run));
    PB_CK(b, cudaEventRecord(b->launched[k], b->run));
    ++b->step;
    return PM_OK;
}

pm_status pm_batch_synchronize(pm_batch* b) {
    if (!b) return PM_ERR_INVALID_ARGUMENT;
    DevGuard dg(b->device);
    PB_CK(b, cudaStreamSynchronize(b->run));
    if (b->persistent && b->d_counters && b->step > 0) {   // the last step's error word
        unsigned err = 0;
        PB_CK(b, cudaMemcpy(&err, b->d_counters + 4 * b->seqs.size() + 1, sizeof err, cudaMemcpyDeviceToHost));
        if (err) return bfail(b, PM_ERR_CUDA, "persistent kernel: a dependency wait ran out; the step's outputs are invalid");
    }
    return PM_OK;
}

pm_status pm_batch_output(pm_batch* b, int seq, const float** depth, const float** variance) {
    if (!b) return PM_ERR_INVALID_ARGUMENT;
    if (seq < 0 || seq >= (int)b->seqs.size()) return bfail(b, PM_ERR_INVALID_ARGUMENT, "no sequence %d", seq);
    if (b->step == 0) return bfail(b, PM_ERR_BAD_STATE, "no step has run");
    const Seq& q = b->seqs[seq];
    const int k = (int)((b->step - 1) & 1);
    if (b->flags & PM_BATCH_HOST_IO) {
        if (depth) *depth = q.h_out[k];
        if (variance) *variance = q.h_out[k] + q.N;
    } else {
        if (depth) *depth = q.d_fused;
        if (variance) *variance = q.d_var;
    }
    return PM_OK;
}

pm_status pm_batch_copy_output(pm_batch* b, int seq, float* depth, size_t pitch, float* variance, size_t var_pitch) {
    if (!b) return PM_ERR_INVALID_ARGUMENT;
    const float* d = nullptr;
    const float* v = nullptr;
    pm_status st = pm_batch_output(b, seq, &d, &v);
    if (st != PM_OK) return st;
    const Seq& q = b->seqs[seq];
    const size_t row = sizeof(float) * (size_t)q.cfg.width;
    if (pitch == 0) pitch = row;
    if (var_pitch == 0) var_pitch = row;
    if (pitch < row || var_pitch < row) return bfail(b, PM_ERR_INVALID_ARGUMENT, "output pitch too small");
    DevGuard dg(b->device);
    PB_CK(b, cudaStreamSynchronize(b->run));
    if (depth) PB_CK(b, cudaMemcpy2D(depth, pitch, d, row, row, (size_t)q.cfg.height, cudaMemcpyDefault));
    if (variance) PB_CK(b, cudaMemcpy2D(variance, var_pitch, v, row, row, (size_t)q.cfg.height, cudaMemcpyDefault));
    return PM_OK;
}

pm_status pm_batch_wta_depth(pm_batch* b, int seq, const float** depth) {
    if (!b || !depth) return PM_ERR_INVALID_ARGUMENT;
    if (seq < 0 || seq >= (int)b->seqs.size()) return bfail(b, PM_ERR_INVALID_ARGUMENT, "no sequence %d", seq);
    *depth = b->seqs[seq].d_depth;
    return PM_OK;
}

pm_status pm_batch_copy_wta_depth(pm_batch* b, int seq, float* depth, size_t pitch) {
    const float* d = nullptr;
    pm_status st = pm_batch_wta_depth(b, seq, &d);
    if (st != PM_OK) return st;
    if (!depth) return bfail(b, PM_ERR_INVALID_ARGUMENT, "null destination");
    const Seq& q = b->seqs[seq];
    const size_t row = sizeof(float) * (size_t)q.cfg.width;
    if (pitch == 0) pitch = row;
    if (pitch < row) return bfail(b, PM_ERR_INVALID_ARGUMENT, "output pitch too small");
    DevGuard dg(b->device);
    PB_CK(b, cudaStreamSynchronize(b->run));
    PB_CK(b, cudaMemcpy2D(depth, pitch, d, row, row, (size_t)q.cfg.height, cudaMemcpyDefault));
    return PM_OK;
}

pm_status pm_batch_get_stats(pm_batch* b, int seq, pm_stats* out) {
    if (!b || !out) return PM_ERR_INVALID_ARGUMENT;
    if (seq < 0 || seq >= (int)b->seqs.size()) return bfail(b, PM_ERR_INVALID_ARGUMENT, "no sequence %d", seq);
    const Seq& q = b->seqs[seq];
    if (!q.d_stats) return bfail(b, PM_ERR_BAD_STATE, "the batch was created without PM_BATCH_STATS");
    DevGuard dg(b->device);
    PB_CK(b, cudaStreamSynchronize(b->run));
    PB_CK(b, cudaMemcpy(out, q.d_stats, sizeof(pm_stats), cudaMemcpyDeviceToHost));
    return PM_OK;
}

pm_status pm_batch_tuning(pm_batch* b, int seq, int* pair_warps, int* serial_pairs, float* ms) {
    if (!b) return PM_ERR_INVALID_ARGUMENT;
    if (seq < 0 || seq >= (int)b->seqs.size()) return bfail(b, PM_ERR_INVALID_ARGUMENT, "no sequence %d", seq);
    const Seq& q = b->seqs[seq];
    if (pair_warps) *pair_warps = q.pair_warps;
    if (serial_pairs) *serial_pairs = q.serial_pairs;
    if (ms) *ms = q.tuned_ms;
    return PM_OK;
}

void* pm_batch_stream(pm_batch* b) { return b ? (void*)b->run : nullptr; }

const char* pm_batch_last_error(const pm_batch* b) { return b ? b->err.c_str() : "null batch"; }

}  // extern "C"
