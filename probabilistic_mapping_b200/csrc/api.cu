// api.cu -- C ABI of libpm_stereo.so: the StereoMapper runtime (reference:
// motion_stereo/stereo_mapper.{h,cpp}) and the stage-level launch wrappers.
//
// A handle owns its device buffers (allocated once in pm_create, like the GpuMat members
// built in StereoMapper::StereoMapper, stereo_mapper.cpp:27-49), one CUDA stream, the
// intrinsics, and the queue of source frames of the current reference frame.  The cost
// volume is evaluated lazily: all queued sources are folded in one kernel pass when a
// result is requested, which equals the reference's per-update running mean.
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <string>
#include <vector>

#include <cuda_fp16.h>

#include "pm_internal.h"
#include "pm_stereo.h"

using namespace pm;

struct pm_mapper {
    pm_config cfg{};
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    double K[9]{};
    bool have_K = false;

    uint8_t* d_u8 = nullptr;    // upload staging, W*H bytes
    float* d_ref = nullptr;     // scaled reference image
    float4* d_srcq = nullptr;   // max_sources source frames in the quad layout (FP16 form: FP16-rounded values)
    void* d_srch[kMaxSources] = {};               // texture samplers: pitched FP16 or FP32 texels
    size_t srch_pitch = 0;
    cudaTextureObject_t tex[kMaxSources] = {};    // texture samplers: one texture object per slot
    int nsrc = 0;               // queued (not yet folded) sources
    std::vector<float> homs;    // 12 floats per queued source
    std::vector<float> all_homs;  // every source since initReference (inspection)
    bool have_ref = false;
    bool cost_valid = false;
    bool has_state = false;     // cost/cnt hold a folded running state

    void* d_cost = nullptr;     // W*H*D float or half
    float* d_off = nullptr;     // FP16 form: per-pixel shift of the half volume (W*H)
    float* d_boff = nullptr;    // FP16 form: block offsets before the rebase (W*H*D/16)
    float* d_cnt = nullptr;     // allocated on the first fold
    float* d_part[4] = {};      // SGM: one volume per opposite-path pair (num_paths / 2 of them)
    SgmStreams side{};          // concurrent path groups
    bool have_side = false;
    float* d_depth = nullptr;   // WTA depth, linear
    int32_t* d_idx = nullptr;   // WTA plane index
    bool store_sgm = false;

    float* d_state[2][4] = {};  // alpha, beta, mu, sigma ping-pong (stereo_mapper.h:48-49)
    unsigned long long* d_ztable = nullptr;
    int32_t* d_table = nullptr;
    float* d_fused = nullptr;
    float* d_var = nullptr;
    // CPU fusion variant scratch (allocated when the mapper is created with it)
    uint8_t* d_cmask = nullptr;
    float* d_corig = nullptr;
    int* d_chead = nullptr;
    int* d_cnext = nullptr;
    uint32_t* d_ctab = nullptr;
    int pre_index = 0;
    bool first_fusion = true;
    double R_prev[9]{}, t_prev[3]{};

    PlaneOrder order{};
    std::string err;

    bool timing = false;
    cudaEvent_t ev[PM_NUM_STAGES + 1] = {};
    bool ev_valid[PM_NUM_STAGES] = {};
    cudaEvent_t ev_cost_kernel = nullptr;   // end of the cost kernel alone (stage 0 minus the rebase)
    bool ev_cost_valid = false;

    unsigned* d_stats = nullptr;   // pm_stats counters (kStatWords), allocated by pm_enable_stats
    uint8_t* d_wta_class = nullptr;   // W*H winner-take-all class of each pixel (pm_stats)
    bool stats = false;
};

namespace pm {

void matmul3(const double* A, const double* B, double* C) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0;
            for (int k = 0; k < 3; ++k) s += A[3 * i + k] * B[3 * k + j];
            C[3 * i + j] = s;
        }
}
void matvec3(const double* A, const double* x, double* y) {
    for (int i = 0; i < 3; ++i) {
        double s = 0;
        for (int k = 0; k < 3; ++k) s += A[3 * i + k] * x[k];
        y[i] = s;
    }
}
void transpose3(const double* A, double* T) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) T[3 * j + i] = A[3 * i + j];
}
bool finite_n(const double* v, int n) {
    for (int i = 0; i < n; ++i)
        if (!std::isfinite(v[i])) return false;
    return true;
}

// H1 = K R_r^T R_l K^-1, H2 = K R_r^T (T_l - T_r) in FP64 (stereo_mapper.cpp:79-80), with the
// closed-form inverse of the upper-triangular K.
void compose_homography(const double* K, const double* Rl, const double* Tl, const double* Rr,
                        const double* Tr, float out[12]) {
    const double fx = K[0], s = K[1], cx = K[2], fy = K[4], cy = K[5];
    const double Ki[9] = {1.0 / fx, -s / (fx * fy), (s * cy - cx * fy) / (fx * fy), 0.0, 1.0 / fy, -cy / fy,
                          0.0, 0.0, 1.0};
    double RrT[9], A[9], B[9], H1[9];
    transpose3(Rr, RrT);
    matmul3(K, RrT, A);
    matmul3(A, Rl, B);
    matmul3(B, Ki, H1);
    const double dT[3] = {Tl[0] - Tr[0], Tl[1] - Tr[1], Tl[2] - Tr[2]};
    double H2[3];
    matvec3(A, dT, H2);
    for (int i = 0; i < 9; ++i) out[i] = (float)H1[i];
    for (int i = 0; i < 3; ++i) out[9 + i] = (float)H2[i];
}

// R_p2c = R^T R_prev, t_p2c = R^T (t_prev - t) (stereo_mapper.cpp:155-156, :766-767).
void fusion_pose_d(const double* R, const double* t, const double* R_prev, const double* t_prev, double out[12]) {
    double RT[9];
    transpose3(R, RT);
    matmul3(RT, R_prev, out);
    const double dt[3] = {t_prev[0] - t[0], t_prev[1] - t[1], t_prev[2] - t[2]};
    matvec3(RT, dt, out + 9);
}

void fusion_pose(const double* R, const double* t, const double* R_prev, const double* t_prev, float out[12]) {
    double d[12];
    fusion_pose_d(R, t, R_prev, t_prev, d);
    for (int i = 0; i < 12; ++i) out[i] = (float)d[i];
}

}  // namespace pm

namespace {

pm_status fail(pm_mapper* h, pm_status s, const char* fmt, ...) {
    if (h) {
        char buf[512];
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(buf, sizeof buf, fmt, ap);
        va_end(ap);
        h->err = buf;
    }
    return s;
}

#define PM_CK(h, call)                                                                          \
    do {                                                                                        \
        cudaError_t e_ = (call);                                                                \
        if (e_ != cudaSuccess)                                                                  \
            return fail((h), e_ == cudaErrorMemoryAllocation ? PM_ERR_OUT_OF_MEMORY : PM_ERR_CUDA, \
                        "%s: %s", #call, cudaGetErrorString(e_));                               \
    } while (0)

struct DeviceGuard {
    int prev = -1;
    explicit DeviceGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DeviceGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

bool is_device_ptr(const void* p) {
    cudaPointerAttributes at;
    if (cudaPointerGetAttributes(&at, p) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    return at.type == cudaMemoryTypeDevice || at.type == cudaMemoryTypeManaged;
}

pm_status check_config(const pm_config* c, pm_mapper* h) {
    if (!c) return fail(h, PM_ERR_INVALID_ARGUMENT, "config is NULL");
    if (c->width < 3 || c->height < 3) return fail(h, PM_ERR_INVALID_ARGUMENT, "image must be at least 3x3");
    if (c->num_planes < 32 || c->num_planes > kMaxPlanes || c->num_planes % 32)
        return fail(h, PM_ERR_INVALID_ARGUMENT, "num_planes must be a multiple of 32 in [32, %d]", kMaxPlanes);
    if (c->num_paths != 4 && c->num_paths != 8) return fail(h, PM_ERR_INVALID_ARGUMENT, "num_paths must be 4 or 8");
    if (c->cost_mode != PM_COST_REFERENCE && c->cost_mode != PM_COST_CORRECTED)
        return fail(h, PM_ERR_INVALID_ARGUMENT, "unknown cost_mode %d", c->cost_mode);
    if (c->precision != PM_PREC_FP32 && c->precision != PM_PREC_FP16)
        return fail(h, PM_ERR_INVALID_ARGUMENT, "unknown precision %d", c->precision);
    if (c->precision == PM_PREC_FP16 && c->num_planes % 64)
        return fail(h, PM_ERR_INVALID_ARGUMENT, "FP16 volumes need num_planes to be a multiple of 64");
    if (c->sampler != PM_SAMPLER_EXACT && c->sampler != PM_SAMPLER_TEXTURE && c->sampler != PM_SAMPLER_TEXTURE_F32)
        return fail(h, PM_ERR_INVALID_ARGUMENT, "unknown sampler %d", c->sampler);
    if (c->sampler == PM_SAMPLER_TEXTURE && c->precision != PM_PREC_FP16)
        return fail(h, PM_ERR_INVALID_ARGUMENT, "FP16 texels belong to the FP16 form");
    if (c->fusion_variant != PM_FUSION_GPU && c->fusion_variant != PM_FUSION_CPU_PATH)
        return fail(h, PM_ERR_INVALID_ARGUMENT, "unknown fusion_variant %d", c->fusion_variant);
    if (c->max_sources < 1 || c->max_sources > kMaxSources)
        return fail(h, PM_ERR_INVALID_ARGUMENT, "max_sources must be in [1, %d]", kMaxSources);
    if (!(c->rho_step > 0.0f) || !std::isfinite(c->rho0))
        return fail(h, PM_ERR_INVALID_ARGUMENT, "rho_step must be positive and rho0 finite");
    return PM_OK;
}

void fill_cost_launch(const pm_config& c, CostLaunch& a) {
    std::memset(&a, 0, sizeof a);
    a.W = c.width;
    a.H = c.height;
    a.D = c.num_planes;
    a.rho0 = c.rho0;
    a.drho = c.rho_step;
    a.mode = c.cost_mode;
    a.cost_half = c.precision == PM_PREC_FP16;
}

void fill_sgm_launch(const pm_config& c, const PlaneOrder& order, SgmLaunch& a) {
    std::memset(&a, 0, sizeof a);
    a.W = c.width;
    a.H = c.height;
    a.D = c.num_planes;
    a.num_paths = c.num_paths;
    a.p1 = c.p1; a.p2 = c.p2; a.tau = c.tau_so; a.q1 = c.q1; a.q2 = c.q2;
    a.fp.var_scale = c.var_scale;
    a.fp.uniq = c.uniqueness_ratio;
    a.fp.rho0 = c.rho0;
    a.fp.drho = c.rho_step;
    a.cost_half = c.precision == PM_PREC_FP16;
    a.order = order;
}

// Uploads a uint8 frame (host or device) and converts it to the scaled float image (dst) or,
// for source frame `slot` (>= 0), to the layout the cost kernel samples: quads (FP32) or the
// slot's FP16 texture storage (FP16 form).  The FP16 form also rounds the reference to FP16.
pm_status upload_image(pm_mapper* h, const uint8_t* img, size_t pitch, float* dst, int slot) {
    const int W = h->cfg.width, H = h->cfg.height;
    if (!img) return fail(h, PM_ERR_INVALID_ARGUMENT, "image pointer is NULL");
    if (pitch == 0) pitch = (size_t)W;
    if (pitch < (size_t)W) return fail(h, PM_ERR_INVALID_ARGUMENT, "image pitch %zu < width %d", pitch, W);
    const uint8_t* dev = img;
    if (!is_device_ptr(img)) {
        PM_CK(h, cudaMemcpy2DAsync(h->d_u8, (size_t)W, img, pitch, (size_t)W, (size_t)H, cudaMemcpyHostToDevice,
                                   h->stream));
        dev = h->d_u8;
        pitch = (size_t)W;
    }
    const float sc = h->cfg.intensity_scale;
    const bool half = h->cfg.precision == PM_PREC_FP16;
    if (slot >= 0 && !half && h->cfg.sampler == PM_SAMPLER_TEXTURE_F32)
        PM_CK(h, launch_to_float_pitched(W, H, dev, pitch, (float*)h->d_srch[slot], h->srch_pitch, sc, h->stream));
    else if (slot >= 0 && half && h->cfg.sampler == PM_SAMPLER_TEXTURE)
        PM_CK(h, launch_to_half(W, H, dev, pitch, h->d_srch[slot], h->srch_pitch, sc, h->stream));
    else if (slot >= 0 && half && h->cfg.sampler == PM_SAMPLER_TEXTURE_F32)
        PM_CK(h, launch_to_float_h_pitched(W, H, dev, pitch, (float*)h->d_srch[slot], h->srch_pitch, sc, h->stream));
    else if (slot >= 0 && half)
        PM_CK(h, launch_to_quad_half(W, H, dev, pitch, h->d_srcq + (size_t)slot * W * H, sc, h->stream));
    else if (slot >= 0)
        PM_CK(h, launch_to_quad(W, H, dev, pitch, h->d_srcq + (size_t)slot * W * H, sc, h->stream));
    else if (half)
        PM_CK(h, launch_to_float_h(W, H, dev, pitch, dst, sc, h->stream));
    else
        PM_CK(h, launch_to_float(W, H, dev, pitch, dst, sc, h->stream));
    return PM_OK;
}

// Folds the queued sources into the cost volume (fresh, or on top of the folded state).
pm_status evaluate_cost(pm_mapper* h, bool into_state) {
    if (h->cost_valid && !into_state) return PM_OK;
    const pm_config& c = h->cfg;
    CostLaunch a;
    fill_cost_launch(c, a);
    a.ref = h->d_ref;
    a.srcq = h->d_srcq;
    a.nsrc = h->nsrc;
    if (c.sampler != PM_SAMPLER_EXACT) {
        a.use_tex = 1;
        for (int s = 0; s < h->nsrc; ++s) a.tex[s] = h->tex[s];
    }
    for (int s = 0; s < h->nsrc; ++s)
        for (int i = 0; i < 12; ++i) a.hom[s][i] = h->homs[12 * s + i];
    a.cost = h->d_cost;
    a.offset = h->d_off;
    a.block_offset = h->d_boff;
    if (h->timing && !into_state) {
        a.kernel_done = h->ev_cost_kernel;
        h->ev_cost_valid = true;
    }
    if (into_state || h->has_state) {
        if (!h->d_cnt) PM_CK(h, cudaMalloc(&h->d_cnt, sizeof(float) * (size_t)c.width * c.height * c.num_planes));
        a.cnt = h->d_cnt;
        a.incremental = h->has_state ? 1 : 0;
        PM_CK(h, launch_cost(a, h->stream));
        h->has_state = true;
        h->nsrc = 0;
        h->homs.clear();
    } else {
        PM_CK(h, launch_cost(a, h->stream));
    }
    h->cost_valid = true;
    return PM_OK;
}

pm_status run_sgm_filter(pm_mapper* h) {
    const pm_config& c = h->cfg;
    SgmLaunch a;
    fill_sgm_launch(c, h->order, a);
    a.cost = h->d_cost;
    a.offset = h->d_off;
    a.ref = h->d_ref;
    for (int r = 0; r < c.num_paths / 2; ++r) a.part[r] = h->d_part[r];
    a.total = h->store_sgm ? h->d_part[0] : nullptr;   // combine reads part[0] of a pixel before writing it
    // the FP16 form keeps its pair volumes in FP16, unless the FP32 sum is to be stored over them
    a.part_half = a.cost_half && !h->store_sgm;
    a.depth = h->d_depth;
    a.depth_pitch = sizeof(float) * (size_t)c.width;
    a.index = h->d_idx;
    a.wta_class = h->stats ? h->d_wta_class : nullptr;
    PM_CK(h, launch_sgm(a, kCombineFilter, h->stream, h->have_side ? &h->side : nullptr));
    if (h->stats)
        PM_CK(h, launch_count_classes(h->d_wta_class, (long)c.width * c.height, kWtaClasses, h->d_stats + kStatWta,
                                      h->stream));
    return PM_OK;
}

// pm_stats: every output call starts from zero counters
pm_status clear_stats(pm_mapper* h) {
    if (h->stats) PM_CK(h, cudaMemsetAsync(h->d_stats, 0, sizeof(unsigned) * kStatWords, h->stream));
    return PM_OK;
}

// Stage timers: event i marks the start of stage i, event i+1 its end.
void mark(pm_mapper* h, int i) {
    if (h->timing && i >= 0 && i <= PM_NUM_STAGES) cudaEventRecord(h->ev[i], h->stream);
}
void mark_done(pm_mapper* h, int stage) {
    if (h->timing) {
        cudaEventRecord(h->ev[stage + 1], h->stream);
        h->ev_valid[stage] = true;
    }
}

pm_status copy_out(pm_mapper* h, float* dst, size_t pitch, const float* src) {
    const int W = h->cfg.width, H = h->cfg.height;
    if (pitch == 0) pitch = sizeof(float) * (size_t)W;
    if (pitch < sizeof(float) * (size_t)W) return fail(h, PM_ERR_INVALID_ARGUMENT, "output pitch too small");
    if (is_device_ptr(dst)) {
        PM_CK(h, cudaMemcpy2DAsync(dst, pitch, src, sizeof(float) * W, sizeof(float) * W, H,
                                   cudaMemcpyDeviceToDevice, h->stream));
    } else {
        PM_CK(h, cudaMemcpy2DAsync(dst, pitch, src, sizeof(float) * W, sizeof(float) * W, H,
                                   cudaMemcpyDeviceToHost, h->stream));
        PM_CK(h, cudaStreamSynchronize(h->stream));
    }
    return PM_OK;
}

void release(pm_mapper* h) {
    cudaFree(h->d_u8);
    cudaFree(h->d_ref);
    cudaFree(h->d_srcq);
    for (int s = 0; s < kMaxSources; ++s) {
        if (h->tex[s]) cudaDestroyTextureObject(h->tex[s]);
        cudaFree(h->d_srch[s]);
    }
    cudaFree(h->d_cost);
    cudaFree(h->d_off);
    cudaFree(h->d_boff);
    cudaFree(h->d_cnt);
    for (auto* p : h->d_part) cudaFree(p);
    cudaFree(h->d_depth);
    cudaFree(h->d_idx);
    for (auto& s : h->d_state)
        for (auto* p : s) cudaFree(p);
    cudaFree(h->d_ztable);
    cudaFree(h->d_table);
    cudaFree(h->d_fused);
    cudaFree(h->d_var);
    cudaFree(h->d_cmask);
    cudaFree(h->d_corig);
    cudaFree(h->d_chead);
    cudaFree(h->d_cnext);
    cudaFree(h->d_ctab);
    cudaFree(h->d_stats);
    cudaFree(h->d_wta_class);
    for (auto& e : h->ev)
        if (e) cudaEventDestroy(e);
    if (h->ev_cost_kernel) cudaEventDestroy(h->ev_cost_kernel);
    for (int g = 0; g < 3; ++g) {
        if (h->side.stream[g]) cudaStreamDestroy(h->side.stream[g]);
        if (h->side.join[g]) cudaEventDestroy(h->side.join[g]);
    }
    if (h->side.fork) cudaEventDestroy(h->side.fork);
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
}

}  // namespace

namespace pm {
pm_status validate_config(const pm_config* c) { return check_config(c, nullptr); }
}  // namespace pm

extern "C" {

void pm_config_default(pm_config* c, int width, int height, int num_planes) {
    if (!c) return;
    std::memset(c, 0, sizeof *c);
    c->width = width;
    c->height = height;
    c->num_planes = num_planes;
    c->rho0 = 0.0f;
    c->rho_step = (float)(1.0 / (0.15 * 160.0));   // evaluate.cc:345
    c->intensity_scale = 1.0f;
    c->num_paths = 4;
    c->p1 = 8.0f;       // parameters.cpp:12-16
    c->p2 = 24.0f;
    c->tau_so = 4.0f;
    c->q1 = 2.0f;
    c->q2 = 3.0f;
    c->var_scale = 1.02f;   // parameters.cpp:18
    c->uniqueness_ratio = 0.0f;
    c->cost_mode = PM_COST_REFERENCE;
    c->precision = PM_PREC_FP32;
    c->fusion_variant = PM_FUSION_GPU;
    c->tree_compat = 1;
    c->max_sources = 16;
    c->device = 0;
}

pm_status pm_create(const pm_config* cfg, pm_mapper** out) {
    if (!out) return PM_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    pm_status st = check_config(cfg, nullptr);
    if (st != PM_OK) return st;
    pm_mapper* h = new pm_mapper();
    h->cfg = *cfg;
    DeviceGuard g(cfg->device);
    const size_t N = (size_t)cfg->width * cfg->height;
    const size_t V = N * cfg->num_planes;
    const size_t esz = cfg->precision == PM_PREC_FP16 ? 2 : 4;
    cudaError_t first_err = cudaSuccess;
    auto note = [&](cudaError_t e) {
        if (e != cudaSuccess && first_err == cudaSuccess) first_err = e;
        return e == cudaSuccess;
    };
    auto alloc = [&](void** p, size_t bytes) { return note(cudaMalloc(p, bytes)); };
    bool ok = note(cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking));
    h->own_stream = ok;
    const bool half = cfg->precision == PM_PREC_FP16;
    ok = ok && alloc((void**)&h->d_u8, N) && alloc((void**)&h->d_ref, 4 * N) &&
         (cfg->sampler != PM_SAMPLER_EXACT || alloc((void**)&h->d_srcq, 16 * N * cfg->max_sources)) &&
         alloc(&h->d_cost, esz * V) && (!half || (alloc((void**)&h->d_off, 4 * N) && alloc((void**)&h->d_boff, 4 * N * (cfg->num_planes / 16)))) &&
         alloc((void**)&h->d_depth, 4 * N) &&
         alloc((void**)&h->d_idx, 4 * N) && alloc((void**)&h->d_ztable, 8 * N) &&
         alloc((void**)&h->d_table, 4 * N) && alloc((void**)&h->d_fused, 4 * N) &&
         alloc((void**)&h->d_var, 4 * N);
    // texture samplers: per-slot pitched images (FP16 form: FP16 texels, or FP16-rounded values in
    // FP32 texels; FP32 form: the images in FP32 texels) sampled through texture objects (linear
    // filter, zero border, unnormalised coordinates: the reference's texture setup,
    // calc_cost.cu:226-237)
    for (int s = 0; cfg->sampler != PM_SAMPLER_EXACT && s < cfg->max_sources && ok; ++s)
        ok = note(make_source_texture(cfg->width, cfg->height, cfg->sampler == PM_SAMPLER_TEXTURE_F32, &h->d_srch[s],
                                      &h->srch_pitch, &h->tex[s]));
    for (int r = 0; r < cfg->num_paths / 2 && ok; ++r) ok = alloc((void**)&h->d_part[r], 4 * V);
    if (ok && cfg->fusion_variant == PM_FUSION_CPU_PATH) {
        if (cfg->width >= 65536 || cfg->height >= 65536) ok = note(cudaErrorInvalidValue);
        ok = ok && alloc((void**)&h->d_cmask, N) && alloc((void**)&h->d_corig, 4 * N) &&
             alloc((void**)&h->d_chead, 4 * N) && alloc((void**)&h->d_cnext, 4 * N) && alloc((void**)&h->d_ctab, 4 * N);
    }
    for (int s = 0; s < 2 && ok; ++s)
        for (int k = 0; k < 4 && ok; ++k) ok = alloc((void**)&h->d_state[s][k], 4 * N);
    if (ok) {
        ok = note(cudaEventCreateWithFlags(&h->side.fork, cudaEventDisableTiming));
        for (int g3 = 0; g3 < 3 && ok; ++g3)
            ok = note(cudaStreamCreateWithFlags(&h->side.stream[g3], cudaStreamNonBlocking)) &&
                 note(cudaEventCreateWithFlags(&h->side.join[g3], cudaEventDisableTiming));
        h->have_side = ok;
    }
    if (ok) ok = cudaMemsetAsync(h->d_table, 0, 4 * N, h->stream) == cudaSuccess;
    for (int s = 0; s < 2 && ok; ++s)
        for (int k = 0; k < 4 && ok; ++k) ok = cudaMemsetAsync(h->d_state[s][k], 0, 4 * N, h->stream) == cudaSuccess;
    if (!ok) {
        cudaGetLastError();
        release(h);
        delete h;
        return first_err == cudaErrorMemoryAllocation ? PM_ERR_OUT_OF_MEMORY : PM_ERR_CUDA;
    }
    plane_order(cfg->num_planes, cfg->tree_compat, h->order);
    *out = h;
    return PM_OK;
}

void pm_destroy(pm_mapper* h) {
    if (!h) return;
    DeviceGuard g(h->cfg.device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    release(h);
    delete h;
}

pm_status pm_set_stream(pm_mapper* h, void* stream) {
    if (!h) return PM_ERR_INVALID_ARGUMENT;
    DeviceGuard g(h->cfg.device);
    if (h->stream) PM_CK(h, cudaStreamSynchronize(h->stream));
    if (h->own_stream && h->stream) cudaStreamDestroy(h->stream);
    h->stream = (cudaStream_t)stream;
    h->own_stream = false;
    return PM_OK;
}

pm_status pm_init_intrinsic(pm_mapper* h, const double K[9], float bf, float dep_sample) {
    (void)bf;   // unused by the reference as well (stereo_mapper.cpp:51-61)
    if (!h) return PM_ERR_INVALID_ARGUMENT;
    if (!K || !finite_n(K, 9)) return fail(h, PM_ERR_INVALID_ARGUMENT, "K must be 9 finite values");
    if (K[0] == 0.0 || K[4] == 0.0 || K[3] != 0.0 || K[6] != 0.0 || K[7] != 0.0 || K[8] != 1.0)
        return fail(h, PM_ERR_INVALID_ARGUMENT, "K must be upper triangular with K[2][2] = 1 and nonzero fx, fy");
    if (!(dep_sample > 0.0f)) return fail(h, PM_ERR_INVALID_ARGUMENT, "dep_sample must be positive");
    std::memcpy(h->K, K, sizeof h->K);
    h->have_K = true;
    h->cfg.rho_step = dep_sample;
    h->cost_valid = false;
    return PM_OK;
}

pm_status pm_init_reference(pm_mapper* h, const uint8_t* img, size_t pitch) {
    if (!h) return PM_ERR_INVALID_ARGUMENT;
    DeviceGuard g(h->cfg.device);
    pm_status st = upload_image(h, img, pitch, h->d_ref, -1);
    if (st != PM_OK) return st;
    h->have_ref = true;
    h->nsrc = 0;
    h->homs.clear();
    h->all_homs.clear();
    h->cost_valid = false;
    h->has_state = false;
    return PM_OK;
}

pm_status pm_update(pm_mapper* h, const uint8_t* img, size_t pitch, const double R_l[9], const double T_l[3],
                    const double R_r[9], const double T_r[3]) {
    if (!h) return PM_ERR_INVALID_ARGUMENT;
    if (!h->have_ref) return fail(h, PM_ERR_BAD_STATE, "update before initReference");
    if (!h->have_K) return fail(h, PM_ERR_BAD_STATE, "update before initIntrinsic");
    if (!R_l || !T_l || !R_r || !T_r || !finite_n(R_l, 9) || !finite_n(T_l, 3) || !finite_n(R_r, 9) ||
        !finite_n(T_r, 3))
        return fail(h, PM_ERR_INVALID_ARGUMENT, "poses must be finite");
    DeviceGuard g(h->cfg.device);
    if (h->nsrc == h->cfg.max_sources) {
        pm_status st = evaluate_cost(h, true);
        if (st != PM_OK) return st;
    }
    float hom[12];
    compose_homography(h->K, R_l, T_l, R_r, T_r, hom);
    pm_status st = upload_image(h, img, pitch, nullptr, h->nsrc);
    if (st != PM_OK) return st;
    h->homs.insert(h->homs.end(), hom, hom + 12);
    h->all_homs.insert(h->all_homs.end(), hom, hom + 12);
    ++h->nsrc;
    h->cost_valid = false;
    return PM_OK;
}

pm_status pm_output(pm_mapper* h, float* depth, size_t pitch) {
    if (!h) return PM_ERR_INVALID_ARGUMENT;
    if (!h->have_ref) return fail(h, PM_ERR_BAD_STATE, "output before initReference");
    if (!depth) return fail(h, PM_ERR_INVALID_ARGUMENT, "depth pointer is NULL");
    DeviceGuard g(h->cfg.device);
    for (bool& v : h->ev_valid) v = false;
    h->ev_cost_valid = false;
    pm_status st = clear_stats(h);
    if (st != PM_OK) return st;
    mark(h, 0);
    st = evaluate_cost(h, false);
    mark_done(h, 0);
    if (st == PM_OK) st = run_sgm_filter(h);
    mark_done(h, 1);
    mark(h, 3);
    if (st == PM_OK) st = copy_out(h, depth, pitch, h->d_depth);
    mark_done(h, 3);
    return st;
}

pm_status pm_output_case(pm_mapper* h, int output_case, float* result, size_t pitch) {
    if (!h) return PM_ERR_INVALID_ARGUMENT;
    if (output_case == PM_CASE_FILTERED) return pm_output(h, result, pitch);
    if (output_case != PM_CASE_RAW_ARGMIN && output_case != PM_CASE_SGM_ARGMIN)
        return fail(h, PM_ERR_INVALID_ARGUMENT, "output_case %d is not 0, 1 or 2", output_case);
    if (!h->have_ref) return fail(h, PM_ERR_BAD_STATE, "output before initReference");
    if (!result) return fail(h, PM_ERR_INVALID_ARGUMENT, "result pointer is NULL");
    DeviceGuard g(h->cfg.device);
    const pm_config& c = h->cfg;
    for (bool& v : h->ev_valid) v = false;
    h->ev_cost_valid = false;
    pm_status st = clear_stats(h);
    if (st != PM_OK) return st;
    mark(h, 0);
    st = evaluate_cost(h, false);
    mark_done(h, 0);
    if (st != PM_OK) return st;
    SgmLaunch a;
    fill_sgm_launch(c, h->order, a);
    if (output_case == PM_CASE_RAW_ARGMIN) {   // stereo_mapper.cpp:628-662
        PM_CK(h, launch_case_argmin(h->d_cost, a.cost_half, h->d_off, c.width, c.height, c.num_planes, a.fp, h->d_fused,
                                    sizeof(float) * (size_t)c.width, h->d_idx, h->stream));
    } else {                                   // stereo_mapper.cpp:668-706
        a.cost = h->d_cost;
        a.offset = h->d_off;
        a.ref = h->d_ref;
        for (int r = 0; r < c.num_paths / 2; ++r) a.part[r] = h->d_part[r];
        a.part_half = a.cost_half;
        a.depth = h->d_fused;
        a.depth_pitch = sizeof(float) * (size_t)c.width;
        a.index = h->d_idx;
        PM_CK(h, launch_sgm(a, kCombineArgmin, h->stream, h->have_side ? &h->side : nullptr));
    }
    mark_done(h, 1);
    mark(h, 3);
    st = copy_out(h, result, pitch, h->d_fused);
    mark_done(h, 3);
    return st;
}

pm_status pm_output_fusion(pm_mapper* h, float* depth, size_t depth_pitch, float* variance, size_t var_pitch,
                           const double R[9], const double t[3], float fx, float fy, float cx, float cy) {
    if (!h) return PM_ERR_INVALID_ARGUMENT;
    if (!h->have_ref) return fail(h, PM_ERR_BAD_STATE, "outputFusion before initReference");
    if (!depth) return fail(h, PM_ERR_INVALID_ARGUMENT, "depth pointer is NULL");
    if (!R || !t || !finite_n(R, 9) || !finite_n(t, 3)) return fail(h, PM_ERR_INVALID_ARGUMENT, "pose must be finite");
    DeviceGuard g(h->cfg.device);
    const int W = h->cfg.width, H = h->cfg.height;
    const size_t N = (size_t)W * H;
    for (bool& v : h->ev_valid) v = false;
    h->ev_cost_valid = false;
    pm_status st = clear_stats(h);
    if (st != PM_OK) return st;
    mark(h, 0);
    st = evaluate_cost(h, false);
    mark_done(h, 0);
    if (st == PM_OK) st = run_sgm_filter(h);
    mark_done(h, 1);
    if (st != PM_OK) return st;
    if (h->first_fusion) {   // stereo_mapper.cpp:128-146
        h->first_fusion = false;
        std::memcpy(h->R_prev, R, sizeof h->R_prev);
        std::memcpy(h->t_prev, t, sizeof h->t_prev);
        h->pre_index = 0;
        PM_CK(h, cudaMemsetAsync(h->d_state[0][0], 0, 4 * N, h->stream));
        PM_CK(h, cudaMemsetAsync(h->d_state[1][0], 0, 4 * N, h->stream));
        PM_CK(h, cudaMemsetAsync(h->d_fused, 0, 4 * N, h->stream));
        PM_CK(h, cudaMemsetAsync(h->d_var, 0, 4 * N, h->stream));
    } else if (h->cfg.fusion_variant == PM_FUSION_CPU_PATH) {   // outputFusionCPU (:741-804)
        FuseCpuLaunch f;
        std::memset(&f, 0, sizeof f);
        f.W = W;
        f.H = H;
        fusion_pose_d(R, t, h->R_prev, h->t_prev, f.pose);
        f.cam[0] = fx; f.cam[1] = fy; f.cam[2] = cx; f.cam[3] = cy;
        PM_CK(h, cudaMemcpyAsync(h->d_fused, h->d_depth, 4 * N, cudaMemcpyDeviceToDevice, h->stream));
        f.result = h->d_fused;
        for (int k = 0; k < 4; ++k) {
            f.pre[k] = h->d_state[h->pre_index][k];
            f.cur[k] = h->d_state[h->pre_index ^ 1][k];
        }
        f.table = reinterpret_cast<uint32_t*>(h->d_table);
        f.variance = h->d_var;
        f.mask = h->d_cmask;
        f.orig_mu = h->d_corig;
        f.head = h->d_chead;
        f.next = h->d_cnext;
        f.tab0 = h->d_ctab;
        f.stats = h->stats ? h->d_stats : nullptr;
        PM_CK(h, launch_fuse_cpu_variant(f, h->stream));
        std::memcpy(h->R_prev, R, sizeof h->R_prev);
        std::memcpy(h->t_prev, t, sizeof h->t_prev);
        h->pre_index ^= 1;
    } else {
        FuseLaunch f;
        std::memset(&f, 0, sizeof f);
        f.W = W;
        f.H = H;
        fusion_pose(R, t, h->R_prev, h->t_prev, f.pose);
        f.cam[0] = fx; f.cam[1] = fy; f.cam[2] = cx; f.cam[3] = cy;
        f.depth = h->d_fused;   // written from the WTA depth by the update kernel
        f.depth_in = h->d_depth;
        for (int k = 0; k < 4; ++k) {
            f.pre[k] = h->d_state[h->pre_index][k];
            f.cur[k] = h->d_state[h->pre_index ^ 1][k];
        }
        f.ztable = h->d_ztable;
        f.table = h->d_table;
        f.variance = h->d_var;
        f.stats = h->stats ? h->d_stats : nullptr;
        PM_CK(h, launch_fuse_gpu(f, h->stream));
        std::memcpy(h->R_prev, R, sizeof h->R_prev);
        std::memcpy(h->t_prev, t, sizeof h->t_prev);
        h->pre_index ^= 1;   // stereo_mapper.cpp:237-241
    }
    mark_done(h, 2);
    mark(h, 3);
    st = copy_out(h, depth, depth_pitch, h->d_fused);
    if (st == PM_OK && variance) st = copy_out(h, variance, var_pitch, h->d_var);
    mark_done(h, 3);
    return st;
}

pm_status pm_get_wta_depth(pm_mapper* h, float* depth, size_t pitch) {
    if (!h || !depth) return PM_ERR_INVALID_ARGUMENT;
    DeviceGuard g(h->cfg.device);
    return copy_out(h, depth, pitch, h->d_depth);
}

pm_status pm_get_wta_index(pm_mapper* h, int32_t* index) {
    if (!h || !index) return PM_ERR_INVALID_ARGUMENT;
    DeviceGuard g(h->cfg.device);
    const size_t bytes = sizeof(int32_t) * (size_t)h->cfg.width * h->cfg.height;
    PM_CK(h, cudaMemcpyAsync(index, h->d_idx, bytes, cudaMemcpyDefault, h->stream));
    PM_CK(h, cudaStreamSynchronize(h->stream));
    return PM_OK;
}

pm_status pm_get_state(pm_mapper* h, float* alpha, float* beta, float* mu, float* sigma) {
    if (!h) return PM_ERR_INVALID_ARGUMENT;
    DeviceGuard g(h->cfg.device);
    float* dst[4] = {alpha, beta, mu, sigma};
    for (int k = 0; k < 4; ++k) {
        if (!dst[k]) continue;
        pm_status st = copy_out(h, dst[k], 0, h->d_state[h->pre_index][k]);
        if (st != PM_OK) return st;
    }
    return PM_OK;
}

pm_status pm_set_state(pm_mapper* h, const float* alpha, const float* beta, const float* mu, const float* sigma,
                       const double R[9], const double t[3]) {
    if (!h || !alpha || !beta || !mu || !sigma || !R || !t) return PM_ERR_INVALID_ARGUMENT;
    DeviceGuard g(h->cfg.device);
    const size_t bytes = 4 * (size_t)h->cfg.width * h->cfg.height;
    const float* src[4] = {alpha, beta, mu, sigma};
    for (int k = 0; k < 4; ++k)
        PM_CK(h, cudaMemcpyAsync(h->d_state[h->pre_index][k], src[k], bytes, cudaMemcpyDefault, h->stream));
    PM_CK(h, cudaStreamSynchronize(h->stream));
    std::memcpy(h->R_prev, R, sizeof h->R_prev);
    std::memcpy(h->t_prev, t, sizeof h->t_prev);
    h->first_fusion = false;
    return PM_OK;
}

pm_status pm_get_buffers(pm_mapper* h, pm_buffers* out) {
    if (!h || !out) return PM_ERR_INVALID_ARGUMENT;
    out->cost = h->d_cost;
    out->cost_offset = h->d_off;
    out->sgm = h->d_part[0];
    out->wta_index = h->d_idx;
    out->wta_depth = h->d_depth;
    out->table = h->d_table;
    return PM_OK;
}

pm_status pm_debug_store_sgm(pm_mapper* h, int enable) {
    if (!h) return PM_ERR_INVALID_ARGUMENT;
    h->store_sgm = enable != 0;
    return PM_OK;
}

pm_status pm_get_homography(pm_mapper* h, int i, float out[12]) {
    if (!h || !out) return PM_ERR_INVALID_ARGUMENT;
    if (i < 0 || (size_t)(12 * (i + 1)) > h->all_homs.size())
        return fail(h, PM_ERR_INVALID_ARGUMENT, "no source frame %d", i);
    std::memcpy(out, h->all_homs.data() + 12 * i, 12 * sizeof(float));
    return PM_OK;
}

pm_status pm_enable_stage_timing(pm_mapper* h, int enable) {
    if (!h) return PM_ERR_INVALID_ARGUMENT;
    DeviceGuard g(h->cfg.device);
    if (enable && !h->ev[0]) {
        for (auto& e : h->ev) PM_CK(h, cudaEventCreate(&e));
        PM_CK(h, cudaEventCreate(&h->ev_cost_kernel));
    }
    h->timing = enable != 0;
    for (bool& v : h->ev_valid) v = false;
    h->ev_cost_valid = false;
    return PM_OK;
}

pm_status pm_get_stage_times(pm_mapper* h, float* ms, int n) {
    if (!h || !ms || n < 0) return PM_ERR_INVALID_ARGUMENT;
    if (!h->timing) return fail(h, PM_ERR_BAD_STATE, "stage timing is not enabled");
    DeviceGuard g(h->cfg.device);
    PM_CK(h, cudaStreamSynchronize(h->stream));
    for (int i = 0; i < n && i < PM_NUM_STAGES; ++i) {
        ms[i] = 0.0f;
        if (h->ev_valid[i]) PM_CK(h, cudaEventElapsedTime(&ms[i], h->ev[i], h->ev[i + 1]));
    }
    if (n > PM_NUM_STAGES) {
        ms[PM_NUM_STAGES] = 0.0f;
        if (h->ev_valid[0] && h->ev_cost_valid)
            PM_CK(h, cudaEventElapsedTime(&ms[PM_NUM_STAGES], h->ev[0], h->ev_cost_kernel));
    }
    return PM_OK;
}

static_assert(PM_STATS_WORDS == kStatWords && sizeof(pm_stats) == sizeof(unsigned) * kStatWords,
              "pm_stats mirrors the device counter block");

pm_status pm_enable_stats(pm_mapper* h, int enable) {
    if (!h) return PM_ERR_INVALID_ARGUMENT;
    DeviceGuard g(h->cfg.device);
    if (enable && !h->d_stats) {
        PM_CK(h, cudaMalloc(&h->d_wta_class, (size_t)h->cfg.width * h->cfg.height));
        PM_CK(h, cudaMalloc(&h->d_stats, sizeof(unsigned) * kStatWords));
        PM_CK(h, cudaMemsetAsync(h->d_stats, 0, sizeof(unsigned) * kStatWords, h->stream));
    }
    h->stats = enable != 0;
    return PM_OK;
}

pm_status pm_get_stats(pm_mapper* h, pm_stats* out) {
    if (!h || !out) return PM_ERR_INVALID_ARGUMENT;
    if (!h->stats) return fail(h, PM_ERR_BAD_STATE, "pixel counters are not enabled");
    DeviceGuard g(h->cfg.device);
    PM_CK(h, cudaMemcpyAsync(out, h->d_stats, sizeof(pm_stats), cudaMemcpyDeviceToHost, h->stream));
    PM_CK(h, cudaStreamSynchronize(h->stream));
    return PM_OK;
}

pm_status pm_synchronize(pm_mapper* h) {
    if (!h) return PM_ERR_INVALID_ARGUMENT;
    DeviceGuard g(h->cfg.device);
    PM_CK(h, cudaStreamSynchronize(h->stream));
    return PM_OK;
}

const char* pm_last_error(const pm_mapper* h) { return h ? h->err.c_str() : "null handle"; }

const char* pm_status_string(pm_status s) {
    switch (s) {
        case PM_OK: return "ok";
        case PM_ERR_INVALID_ARGUMENT: return "invalid argument";
        case PM_ERR_BAD_STATE: return "bad state";
        case PM_ERR_CUDA: return "CUDA error";
        case PM_ERR_OUT_OF_MEMORY: return "out of memory";
        case PM_ERR_UNSUPPORTED: return "unsupported";
        default: return "unknown status";
    }
}

// ---- stage-level wrappers -----------------------------------------------------------------

pm_status pm_stage_to_float(int W, int H, const uint8_t* src, size_t src_pitch, float* dst, float scale,
                            void* stream) {
    if (W <= 0 || H <= 0 || !src || !dst || src_pitch < (size_t)W) return PM_ERR_INVALID_ARGUMENT;
    return launch_to_float(W, H, src, src_pitch, dst, scale, (cudaStream_t)stream) == cudaSuccess ? PM_OK
                                                                                                  : PM_ERR_CUDA;
}

pm_status pm_stage_calc_cost(const pm_config* cfg, const float* ref, const float* srcs, int nsrc, const float* homs,
                             float* cost, float* cnt, uint8_t* invalid, void* stream) {
    if (check_config(cfg, nullptr) != PM_OK || !ref || !cost || nsrc < 0 || (nsrc > 0 && (!srcs || !homs)))
        return PM_ERR_INVALID_ARGUMENT;
    if (cfg->precision != PM_PREC_FP32) return PM_ERR_UNSUPPORTED;
    if (nsrc > kMaxSources && !cnt) return PM_ERR_INVALID_ARGUMENT;   // needs a running count
    const size_t N = (size_t)cfg->width * cfg->height;
    const int W = cfg->width, H = cfg->height;
    const bool tex = cfg->sampler == PM_SAMPLER_TEXTURE_F32;
    const cudaStream_t st = (cudaStream_t)stream;
    CostLaunch a;
    fill_cost_launch(*cfg, a);
    a.ref = ref;
    a.cost = cost;
    a.cnt = cnt;
    a.invalid = invalid;
    // texture sampler: pitched copies of one pass's sources behind texture objects, released
    // once the pass has finished
    void* buf[kMaxSources] = {};
    size_t pitch = 0;
    bool ok = true;
    int done = 0;
    do {
        const int n = std::min(nsrc - done, kMaxSources);
        a.srcs = srcs + N * done;
        a.nsrc = n;
        for (int s = 0; s < n; ++s)
            for (int i = 0; i < 12; ++i) a.hom[s][i] = homs[12 * (done + s) + i];
        for (int s = 0; tex && s < n && ok; ++s) {
            ok = make_source_texture(W, H, true, &buf[s], &pitch, &a.tex[s]) == cudaSuccess &&
                 cudaMemcpy2DAsync(buf[s], pitch, srcs + N * (done + s), 4 * (size_t)W, 4 * (size_t)W, (size_t)H,
                                   cudaMemcpyDeviceToDevice, st) == cudaSuccess;
        }
        a.use_tex = tex ? 1 : 0;
        // with a count buffer the call continues the running state, like repeated ad_calc_cost
        a.incremental = cnt ? 1 : 0;
        ok = ok && launch_cost(a, st) == cudaSuccess;
        if (tex) {
            ok = cudaStreamSynchronize(st) == cudaSuccess && ok;
            for (int s = 0; s < n; ++s) {
                if (a.tex[s]) cudaDestroyTextureObject(a.tex[s]);
                cudaFree(buf[s]);
                a.tex[s] = 0;
                buf[s] = nullptr;
            }
        }
        if (!ok) return PM_ERR_CUDA;
        done += n;
    } while (done < nsrc);
    return PM_OK;
}

pm_status pm_stage_sgm(const pm_config* cfg, const float* cost, const float* ref, float* out, float* scratch,
                       void* stream) {
    if (check_config(cfg, nullptr) != PM_OK || !cost || !ref || !out || !scratch) return PM_ERR_INVALID_ARGUMENT;
    if (cfg->precision != PM_PREC_FP32) return PM_ERR_UNSUPPORTED;
    PlaneOrder order;
    plane_order(cfg->num_planes, cfg->tree_compat, order);
    SgmLaunch a;
    fill_sgm_launch(*cfg, order, a);
    a.cost = cost;
    a.ref = ref;
    const size_t V = (size_t)cfg->width * cfg->height * cfg->num_planes;
    a.part[0] = out;   // the combine kernel reads part[0] of a pixel before it writes the total there
    for (int r = 1; r < cfg->num_paths / 2; ++r) a.part[r] = scratch + (r - 1) * V;
    a.total = out;
    return launch_sgm(a, kCombineStore, (cudaStream_t)stream, nullptr) == cudaSuccess ? PM_OK : PM_ERR_CUDA;
}

pm_status pm_stage_filter(const pm_config* cfg, const float* sgm, float* depth, size_t pitch, int32_t* index,
                          void* stream) {
    if (check_config(cfg, nullptr) != PM_OK || !sgm || !depth) return PM_ERR_INVALID_ARGUMENT;
    if (pitch == 0) pitch = sizeof(float) * (size_t)cfg->width;
    if (pitch < sizeof(float) * (size_t)cfg->width || pitch % 4) return PM_ERR_INVALID_ARGUMENT;
    PlaneOrder order;
    plane_order(cfg->num_planes, cfg->tree_compat, order);
    FilterParams fp{cfg->var_scale, cfg->uniqueness_ratio, cfg->rho0, cfg->rho_step};
    return launch_filter(sgm, cfg->width, cfg->height, cfg->num_planes, fp, order, depth, pitch, index,
                         (cudaStream_t)stream) == cudaSuccess
               ? PM_OK
               : PM_ERR_CUDA;
}

pm_status pm_stage_sgm_filter(const pm_config* cfg, const float* cost, const float* ref, float* scratch,
                              float* depth, size_t pitch, int32_t* index, void* stream) {
    if (check_config(cfg, nullptr) != PM_OK || !cost || !ref || !scratch || !depth) return PM_ERR_INVALID_ARGUMENT;
    if (cfg->precision != PM_PREC_FP32) return PM_ERR_UNSUPPORTED;
    if (pitch == 0) pitch = sizeof(float) * (size_t)cfg->width;
    if (pitch < sizeof(float) * (size_t)cfg->width || pitch % 4) return PM_ERR_INVALID_ARGUMENT;
    PlaneOrder order;
    plane_order(cfg->num_planes, cfg->tree_compat, order);
    SgmLaunch a;
    fill_sgm_launch(*cfg, order, a);
    a.cost = cost;
    a.ref = ref;
    const size_t V = (size_t)cfg->width * cfg->height * cfg->num_planes;
    for (int r = 0; r < cfg->num_paths / 2; ++r) a.part[r] = scratch + r * V;
    a.total = nullptr;
    a.depth = depth;
    a.depth_pitch = pitch;
    a.index = index;
    return launch_sgm(a, kCombineFilter, (cudaStream_t)stream, nullptr) == cudaSuccess ? PM_OK : PM_ERR_CUDA;
}

pm_status pm_stage_depth_fuse(int W, int H, const float pose[12], const float cam[4], float* depth,
                              float* const pre[4], float* const cur[4], uint64_t* ztable, int32_t* table,
                              void* stream) {
    if (W <= 0 || H <= 0 || !pose || !cam || !depth || !pre || !cur || !ztable) return PM_ERR_INVALID_ARGUMENT;
    FuseLaunch f;
    std::memset(&f, 0, sizeof f);
    f.W = W;
    f.H = H;
    for (int i = 0; i < 12; ++i) f.pose[i] = pose[i];
    for (int i = 0; i < 4; ++i) f.cam[i] = cam[i];
    f.depth = depth;
    for (int k = 0; k < 4; ++k) {
        if (!pre[k] || !cur[k]) return PM_ERR_INVALID_ARGUMENT;
        f.pre[k] = pre[k];
        f.cur[k] = cur[k];
    }
    f.ztable = reinterpret_cast<unsigned long long*>(ztable);
    f.table = table;
    return launch_fuse_gpu(f, (cudaStream_t)stream) == cudaSuccess ? PM_OK : PM_ERR_CUDA;
}

// Scratch of pm_stage_depth_fuse_cpu_path, W*H each: mask (u8), original mean (f32), list head
// and link (i32), initial table (u32); sections 256-byte aligned.
static size_t cpu_path_section(size_t n, size_t elem) { return (n * elem + 255) & ~(size_t)255; }

size_t pm_stage_depth_fuse_cpu_path_scratch(int W, int H) {
    if (W <= 0 || H <= 0) return 0;
    const size_t n = (size_t)W * H;
    return cpu_path_section(n, 1) + 4 * cpu_path_section(n, 4);
}

pm_status pm_stage_depth_fuse_cpu_path(int W, int H, const double pose[12], const float cam[4], float* result,
                                       float* const pre[4], float* const cur[4], uint32_t* table, void* scratch,
                                       void* stream) {
    if (W <= 0 || H <= 0 || W >= 65536 || H >= 65536 || !pose || !cam || !result || !pre || !cur || !scratch)
        return PM_ERR_INVALID_ARGUMENT;
    if (!finite_n(pose, 12)) return PM_ERR_INVALID_ARGUMENT;
    FuseCpuLaunch f;
    std::memset(&f, 0, sizeof f);
    f.W = W;
    f.H = H;
    for (int i = 0; i < 12; ++i) f.pose[i] = pose[i];
    for (int i = 0; i < 4; ++i) f.cam[i] = cam[i];
    f.result = result;
    for (int k = 0; k < 4; ++k) {
        if (!pre[k] || !cur[k]) return PM_ERR_INVALID_ARGUMENT;
        f.pre[k] = pre[k];
        f.cur[k] = cur[k];
    }
    f.table = table;
    const size_t n = (size_t)W * H;
    unsigned char* p = static_cast<unsigned char*>(scratch);
    f.mask = reinterpret_cast<uint8_t*>(p);
    p += cpu_path_section(n, 1);
    f.orig_mu = reinterpret_cast<float*>(p);
    p += cpu_path_section(n, 4);
    f.head = reinterpret_cast<int*>(p);
    p += cpu_path_section(n, 4);
    f.next = reinterpret_cast<int*>(p);
    p += cpu_path_section(n, 4);
    f.tab0 = reinterpret_cast<uint32_t*>(p);
    return launch_fuse_cpu_variant(f, (cudaStream_t)stream) == cudaSuccess ? PM_OK : PM_ERR_CUDA;
}

pm_status pm_stage_convert(int W, int H, const float* in, float* out, int flag, size_t pitch, void* stream) {
    if (W <= 0 || H <= 0 || !in || !out || pitch < sizeof(float) * (size_t)W || pitch % 4)
        return PM_ERR_INVALID_ARGUMENT;
    return launch_convert(W, H, in, out, flag, pitch, (cudaStream_t)stream) == cudaSuccess ? PM_OK : PM_ERR_CUDA;
}

}  // extern "C"
