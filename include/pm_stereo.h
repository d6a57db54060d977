/*
 * pm_stereo.h -- C ABI of the B200 motion-stereo library (libpm_stereo.so).
 *
 * Drop-in replacement for the StereoMapper class of HKUST-Aerial-Robotics/probabilistic_mapping
 * (motion_stereo/stereo_mapper.h:26-63) and for its five C-style launch wrappers
 * (ad_calc_cost, sgm2, filter_cost, depth_fuse, convert).  Plain pointers and sizes only.
 *
 * Conventions
 *   - Images are W x H, row-major, with an explicit row pitch in BYTES.
 *   - Cost volumes are plane-innermost float arrays: element ((y*W + x)*D + d), the INDEX()
 *     layout of motion_stereo/cuda_utils.h:34.
 *   - Matrices are row-major doubles; poses are camera-to-world (R, T) as in
 *     StereoMapper::update (stereo_mapper.cpp:73-91).
 *   - Pointers passed to the mapper-level calls may be host or device memory; the library
 *     tells them apart with cudaPointerGetAttributes.  Stage-level calls (pm_stage_*) take
 *     device pointers only and run on the given stream (NULL = legacy default stream).
 *   - Every call returns a pm_status; pm_last_error() holds the message of the last failure
 *     on a handle.  Nothing in the library exits or traps (the reference exits on error,
 *     cuda_utils.h:18-32).
 *   - A handle owns one CUDA stream; distinct handles may run concurrently; one handle must
 *     not be used from two threads at once.
 */
#ifndef PM_STEREO_H
#define PM_STEREO_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define PM_API __attribute__((visibility("default")))
#else
#define PM_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

typedef int pm_status;
#define PM_OK 0
#define PM_ERR_INVALID_ARGUMENT 1
#define PM_ERR_BAD_STATE 2
#define PM_ERR_CUDA 3
#define PM_ERR_OUT_OF_MEMORY 4
#define PM_ERR_UNSUPPORTED 5

#define PM_COST_REFERENCE 0 /* keeps the neighbour quirks of calc_cost.cu:50-51,70-71,106,119 */
#define PM_COST_CORRECTED 1 /* the intended 3x3 patch absolute difference */

#define PM_PREC_FP32 0 /* plain form: FP32 images, cost volume and aggregation */
#define PM_PREC_FP16 1 /* FP16 cost volume, FP32 SGM accumulators and fusion */

/* How source frames are sampled.  The FP32 form takes PM_SAMPLER_EXACT or PM_SAMPLER_TEXTURE_F32,
 * the FP16 form all three. */
#define PM_SAMPLER_EXACT 0   /* bilinear weights and interpolation in FP32 (FP16 form: of the
                                FP16-rounded images) */
#define PM_SAMPLER_TEXTURE 1 /* FP16 texels filtered by the texture unit (8-bit weights, as the
                                reference's own textures, calc_cost.cu:226-237; the unit filters
                                FP16 texels at reduced precision) */
#define PM_SAMPLER_TEXTURE_F32 2 /* FP32 texels filtered by the texture unit: 8-bit weights with
                                    FP32 filtering, at the speed of PM_SAMPLER_TEXTURE.  FP32 form:
                                    the images themselves, the reference's own sampler; FP16 form:
                                    the FP16-rounded images */

#define PM_FUSION_GPU 0      /* StereoMapper::outputFusion + depth_fusion.cu kernels */
#define PM_FUSION_CPU_PATH 1 /* the constants and masks of outputFusionCPU, run on the GPU */

typedef struct pm_config {
    int width, height;   /* WIDTH, HEIGHT (parameters.h:8-9), runtime here */
    int num_planes;      /* DEP_CNT (parameters.h:15); a multiple of 32, at most 256 */
    float rho0;          /* inverse depth of plane 0; 0 in the reference (calc_cost.cu:81) */
    float rho_step;      /* DEP_SAMPLE; pm_init_intrinsic overwrites it */
    float intensity_scale; /* image value = uint8 * scale; 1 in the reference (stereo_mapper.cpp:66) */
    int num_paths;       /* SGM paths: 4 (sgm.cu:119-133) or 8 (adds the four diagonals) */
    float p1, p2;        /* pi1, pi2 (parameters.cpp:12-13) */
    float tau_so;        /* parameters.cpp:14 */
    float q1, q2;        /* sgm_q1, sgm_q2 (parameters.cpp:15-16) */
    float var_scale;     /* flatness factor (parameters.cpp:18) */
    float uniqueness_ratio; /* extension: reject when best > ratio * second best; 0 disables */
    int cost_mode;       /* PM_COST_* */
    int precision;       /* PM_PREC_* */
    int fusion_variant;  /* PM_FUSION_* */
    int tree_compat;     /* 1: reproduce the reduction tree of sgm.cu:24-31 / filter_cost.cu:22-30
                            (drops planes when D is not a power of two); 0: exact minimum */
    int max_sources;     /* source frames kept per reference frame (lazy cost evaluation) */
    int device;          /* CUDA device ordinal */
    int sampler;         /* PM_SAMPLER_* */
} pm_config;

typedef struct pm_mapper pm_mapper;

/* Fills the reference's defaults (parameters.cpp:12-18, DEP_SAMPLE of evaluate.cc:345). */
PM_API void pm_config_default(pm_config* cfg, int width, int height, int num_planes);

/* StereoMapper::StereoMapper (stereo_mapper.cpp:27-49): allocates every device buffer. */
PM_API pm_status pm_create(const pm_config* cfg, pm_mapper** out);
PM_API void pm_destroy(pm_mapper* h);

/* Use the caller's stream instead of the handle's own one (e.g. a torch stream). */
PM_API pm_status pm_set_stream(pm_mapper* h, void* cuda_stream);

/* StereoMapper::initIntrinsic (stereo_mapper.cpp:51-61).  K row-major 3x3 (fy may be
 * negative, evaluate.cc:38); bf is unused, as in the reference; dep_sample sets rho_step. */
PM_API pm_status pm_init_intrinsic(pm_mapper* h, const double K[9], float bf, float dep_sample);

/* StereoMapper::initReference (stereo_mapper.cpp:63-71): uint8 W x H image; resets the
 * cost volume and the list of source frames. */
PM_API pm_status pm_init_reference(pm_mapper* h, const uint8_t* img, size_t pitch_bytes);

/* StereoMapper::update (stereo_mapper.cpp:73-91).  Composes H1 = K R_r^T R_l K^-1 and
 * H2 = K R_r^T (T_l - T_r) in FP64 and queues the source frame; the cost of all queued frames
 * is evaluated in one pass when the result is requested.  The result equals the reference's
 * per-call running mean.  A pageable host image may be reused as soon as the call returns;
 * page-locked host and device images must stay unchanged until the next pm_output* or
 * pm_synchronize call returns (the upload is asynchronous for them). */
PM_API pm_status pm_update(pm_mapper* h, const uint8_t* img, size_t pitch_bytes,
                    const double R_l[9], const double T_l[3],
                    const double R_r[9], const double T_r[3]);

/* StereoMapper::output (stereo_mapper.cpp:93-109): SGM + winner-take-all/subpixel; writes the
 * W x H depth (1000 = no overlap, 0 = rejected).  Synchronous for host destinations. */
PM_API pm_status pm_output(pm_mapper* h, float* depth, size_t pitch_bytes);

/* StereoMapper::outputFusion (stereo_mapper.cpp:111-244) or, with PM_FUSION_CPU_PATH,
 * outputFusionCPU (stereo_mapper.cpp:625-820).  R, t: current keyframe pose (camera-to-world,
 * row-major).  Writes the FUSED depth (the reference's GPU path returned the unfused map,
 * stereo_mapper.cpp:229-230; pm_get_wta_depth gives that one) and, when variance is not NULL,
 * the per-pixel variance sigma^2 of the fused state.  The first call only initialises the
 * state and writes zeros, as the reference does (stereo_mapper.cpp:128-146). */
PM_API pm_status pm_output_fusion(pm_mapper* h, float* depth, size_t depth_pitch, float* variance,
                           size_t variance_pitch, const double R[9], const double t[3],
                           float fx, float fy, float cx, float cy);

/* The debug outputs of outputFusionCPU, selected there by the global CASE (stereo_mapper.cpp:
 * 628-719; evaluate.cc:314-319 reads it from argv[1], default 0):
 *   PM_CASE_RAW_ARGMIN  argmin of the plane-sweep cost itself (:628-662);
 *   PM_CASE_SGM_ARGMIN  argmin of the SGM sum (:668-706);
 *   PM_CASE_FILTERED    the winner-take-all filter's depth, as pm_output (:712-719).
 * The argmin outputs scan the planes in order (first strict minimum below 100000 wins) and write
 * 10000 where |min| < 1e-5, 0 at the first and last plane, else 1 / (rho0 + d * rho_step) with no
 * subpixel refinement.  CASE >= 3 is pm_output_fusion with PM_FUSION_CPU_PATH.  pm_get_wta_index
 * afterwards gives the argmin's plane.  The fusion state is not touched. */
#define PM_CASE_RAW_ARGMIN 0
#define PM_CASE_SGM_ARGMIN 1
#define PM_CASE_FILTERED 2
PM_API pm_status pm_output_case(pm_mapper* h, int output_case, float* result, size_t pitch_bytes);

/* The winner-take-all depth of the last output call (the reference's `dep`). */
PM_API pm_status pm_get_wta_depth(pm_mapper* h, float* depth, size_t pitch_bytes);

/* The winner-take-all plane index (W*H int32, row-major) of the last output call. */
PM_API pm_status pm_get_wta_index(pm_mapper* h, int32_t* index);

/* Fusion state of the last fused frame (alpha, beta, mu, sigma^2: W*H floats each; any may
 * be NULL).  pm_set_state loads a state and pose, e.g. to resume a sequence. */
PM_API pm_status pm_get_state(pm_mapper* h, float* alpha, float* beta, float* mu, float* sigma);
PM_API pm_status pm_set_state(pm_mapper* h, const float* alpha, const float* beta, const float* mu,
                       const float* sigma, const double R[9], const double t[3]);

/* Device pointers of the internal buffers, for inspection and tests.  Valid until pm_destroy. */
typedef struct pm_buffers {
    const void* cost;      /* W*H*D: float (FP32) or half (FP16) */
    const float* sgm;      /* W*H*D float, filled only after pm_debug_store_sgm(h, 1) */
    const int32_t* wta_index; /* W*H winner-take-all plane index */
    const float* wta_depth;   /* W*H */
    const int32_t* table;  /* W*H propagation table of the last fusion step */
    const float* cost_offset; /* FP16 form: W*H; the half volume holds cost - cost_offset[pixel],
                                 the pixel's smallest measured cost (0 when some plane of the pixel
                                 is unmeasured); NULL in the FP32 form */
} pm_buffers;
PM_API pm_status pm_get_buffers(pm_mapper* h, pm_buffers* out);
PM_API pm_status pm_debug_store_sgm(pm_mapper* h, int enable);

/* Homography of source frame i as passed to the kernels (12 floats: H1 row-major, H2). */
PM_API pm_status pm_get_homography(pm_mapper* h, int i, float out[12]);

/* Opt-in CUDA-event timers around the stages of pm_output / pm_output_fusion (recorded on the
 * handle's stream).  pm_get_stage_times synchronises and returns, in milliseconds, the
 * time of the last call's stages: [0] cost volume, [1] SGM + winner-take-all, [2] fusion,
 * [3] copy-out.  n is the capacity of ms; returns PM_ERR_BAD_STATE when timing is off.
 * With n > PM_NUM_STAGES, ms[PM_NUM_STAGES] is the cost kernel alone: stage [0] without the
 * FP16 form's rebase pass (equal to [0] for the FP32 form). */
#define PM_NUM_STAGES 4
PM_API pm_status pm_enable_stage_timing(pm_mapper* h, int enable);
PM_API pm_status pm_get_stage_times(pm_mapper* h, float* ms, int n);

/* Per-map pixel counters (opt-in).  They replace the reference's debug prints and its
 * commented-out counters (stereo_mapper.cpp:56-60, 329, 431, 565).  Each pm_output,
 * pm_output_fusion and pm_output_case call clears them on the handle's stream.  Then:
 *   - The winner-take-all filter (filter_cost.cu:37-51; not pm_output_case's debug argmin)
 *     puts every pixel in one of five wta_* classes.
 *   - A non-first pm_output_fusion step adds the fusion classes.  tf_* follow transformMap
 *     (depth_fusion.cu:26-48, transformMapCPU stereo_mapper.cpp:274-326, cnt0..cnt4).
 *     pred_* follow depth_predict (:107-137, depthPreditCPU :405-421, cnt0/cnt1).
 *     upd_* follow depthUpdate (:161-219, depthUpdateCPU :466-556, cnt0..cnt4).
 * pm_get_stats waits for the handle's stream.  It returns PM_ERR_BAD_STATE while counting is off.
 * Counting adds a one-byte class store per pixel and a counting kernel (W*H bytes) to the
 * winner-take-all, and shared-memory tallies to the fusion kernels.  Outputs do not change. */
typedef struct pm_stats {
    uint32_t wta_depth;       /* sub-pixel depth written */
    uint32_t wta_no_overlap;  /* |min| < FLOAT_EPS: DEP_INF written */
    uint32_t wta_border;      /* minimum at the first or last plane: 0 */
    uint32_t wta_flat;        /* flat minimum (var_scale test): 0 */
    uint32_t wta_ambiguous;   /* uniqueness test failed: 0 */
    uint32_t tf_empty;        /* previous alpha < FLOAT_EPS */
    uint32_t tf_outlier;      /* previous inlier ratio below 0.4 (CPU variant: 0.5) */
    uint32_t tf_behind;       /* moved depth < FLOAT_EPS */
    uint32_t tf_outside;      /* projects outside the image */
    uint32_t tf_moved;        /* moved into the current keyframe */
    uint32_t pred_none;       /* cell without a predecessor after hole filling */
    uint32_t pred_copied;     /* cell that received a predicted state */
    uint32_t pred_filled;     /* of pred_copied: the predecessor came from hole filling */
    uint32_t upd_empty;       /* no prior state and no measurement */
    uint32_t upd_init;        /* no prior state; the measurement starts one */
    uint32_t upd_no_measurement; /* prior state, no measurement */
    uint32_t upd_output;      /* Bayesian update; inlier ratio above the output threshold */
    uint32_t upd_hidden;      /* Bayesian update; inlier ratio at or below it */
} pm_stats;
#define PM_STATS_WORDS 18
PM_API pm_status pm_enable_stats(pm_mapper* h, int enable);
PM_API pm_status pm_get_stats(pm_mapper* h, pm_stats* out);

PM_API pm_status pm_synchronize(pm_mapper* h);

/* Exhaustive self-check of the exact FP32 shortcuts in the kernels (no counterpart in the
 * reference): out[0] = floats w > 0 where the Newton reciprocal differs from the correctly
 * rounded 1/w, out[1] = floats u in [0, 2^22) where the add-based floor differs from floorf,
 * out[2] = (x, d) pairs, d in [2, 33], where the reciprocal-multiply division differs from IEEE
 * x / d, out[3] = floats w where the branch-free reciprocal of the warps differs from its
 * definition (RN(1/w) for 2^-126 <= |w| <= 2^126, NaN for zero, subnormal, infinite or NaN w,
 * +-0 above).  All four are 0 on a correct device.  Allocates 32 bytes of device memory. */
PM_API pm_status pm_debug_check_arith(uint64_t out[4], void* stream);
/* The bounds-checked library (libpm_stereo_checked.so, built from the same sources with
 * PM_BOUNDS_CHECK; no counterpart in the reference, which has no checks): the kernels test the
 * element index of their global accesses against the buffer and skip an access that is out of
 * range instead of faulting.  out[0] = accesses skipped since the last reset, out[1..3] = site,
 * index and extent of the first one.  Synchronises the device; reset = 1 clears the record.
 * The product library returns PM_ERR_UNSUPPORTED (and zeros). */
PM_API pm_status pm_debug_bounds(uint64_t out[4], int reset);
PM_API const char* pm_last_error(const pm_mapper* h);
PM_API const char* pm_status_string(pm_status s);

/* ---------------------------------------------------------------------------------------
 * Batched form (no counterpart in the reference): many independent sequences, each with its
 * own pm_config (resolution, planes, precision, parameters), stepped together.  One
 * pm_batch_run is one keyframe of every sequence -- initReference(frame 0), pm_update of frames
 * 1..num_sources with their poses, then outputFusion(R_ref, T_ref) -- exactly the StereoMapper
 * calls, issued as ONE CUDA-graph launch in which the sequences are independent branches.
 * Sequences of the same shape share `lanes` sets of cost and path volumes (0: one set each).
 * Two buffer sets alternate by step, so frames for step t+1 can be written while step t runs.
 * The CPU fusion variant is not available in a batch.
 * --------------------------------------------------------------------------------------- */
typedef struct pm_batch pm_batch;
#define PM_BATCH_HOST_IO 1  /* frames in and fused depth/variance out through batch-owned pinned
                               host buffers, copied inside the graph; else device buffers */
#define PM_BATCH_AUTOTUNE 2 /* time the SGM schedules for each distinct shape at creation */
#define PM_BATCH_PRIORITY 4 /* SGM kernels at the device's greatest launch priority, so they
                               overlap the other sequences' cost kernels */
#define PM_BATCH_PERSISTENT 8 /* the cost volumes, FP16 rebases, SGM path pairs and winner-take-all
                                 of all sequences in ONE persistent kernel launch (inside the
                                 graph), which takes the work items of every sequence from one
                                 list, interleaving one sequence's cost tiles with the previous
                                 one's SGM scanlines.  Needs lanes = 0 and one precision, sampler
                                 and cost mode for all sequences (else PM_ERR_UNSUPPORTED);
                                 PM_BATCH_AUTOTUNE and PM_BATCH_PRIORITY do not apply to it.
                                 pm_batch_synchronize reports PM_ERR_CUDA if a dependency wait
                                 of the last step ran out (its outputs are then invalid). */
#define PM_BATCH_STATS 16 /* per-sequence pm_stats counters of each step (pm_batch_get_stats) */
PM_API pm_status pm_batch_create(const pm_config* cfgs, int num_sequences, int num_sources, int lanes, int flags,
                                 pm_batch** out);
PM_API void pm_batch_destroy(pm_batch* b);
PM_API pm_status pm_batch_init_intrinsic(pm_batch* b, int seq, const double K[9], float dep_sample);
/* Buffer of frame f (0 = reference, 1..num_sources = sources) of sequence seq for the next
 * pm_batch_run: W*H uint8, row pitch W, host memory with PM_BATCH_HOST_IO, else device. */
PM_API pm_status pm_batch_frame(pm_batch* b, int seq, int frame, uint8_t** ptr);
/* Copies a W*H uint8 frame (host or device memory, row pitch in bytes, 0 = W) into that buffer. */
PM_API pm_status pm_batch_put_frame(pm_batch* b, int seq, int frame, const uint8_t* img, size_t pitch);
/* Poses of the next step: reference frame and the num_sources source frames (R_src 9 doubles
 * and T_src 3 doubles per source, row-major, as pm_update). */
PM_API pm_status pm_batch_set_poses(pm_batch* b, int seq, const double R_ref[9], const double T_ref[3],
                                    const double* R_src, const double* T_src);
PM_API pm_status pm_batch_run(pm_batch* b);
PM_API pm_status pm_batch_synchronize(pm_batch* b);
/* Fused depth and variance (W*H float) of the last step of sequence seq, after
 * pm_batch_synchronize: pinned host buffers with PM_BATCH_HOST_IO, device buffers otherwise. */
PM_API pm_status pm_batch_output(pm_batch* b, int seq, const float** depth, const float** variance);
/* Copies them into caller buffers (host or device, byte pitches, 0 = packed) after waiting for
 * the batch's stream. */
PM_API pm_status pm_batch_copy_output(pm_batch* b, int seq, float* depth, size_t pitch, float* variance,
                                      size_t var_pitch);
/* Winner-take-all depth (device, W*H float) of the last step of sequence seq. */
PM_API pm_status pm_batch_wta_depth(pm_batch* b, int seq, const float** depth);
/* Copies it into a caller buffer (host or device, byte pitch, 0 = packed) after waiting for the
 * batch's stream. */
PM_API pm_status pm_batch_copy_wta_depth(pm_batch* b, int seq, float* depth, size_t pitch);
/* SGM schedule of sequence seq: scanlines per block of the path-pair kernel, serial (1) or
 * concurrent (0) path pairs, and the stage time the autotuner measured (ms; 0 if untuned). */
PM_API pm_status pm_batch_tuning(pm_batch* b, int seq, int* pair_warps, int* serial_pairs, float* ms);
/* The pm_stats counters of sequence seq's last step (a batch created with PM_BATCH_STATS), after
 * waiting for the batch's stream; PM_ERR_BAD_STATE without the flag. */
PM_API pm_status pm_batch_get_stats(pm_batch* b, int seq, pm_stats* out);
PM_API void* pm_batch_stream(pm_batch* b);
PM_API const char* pm_batch_last_error(const pm_batch* b);

/* ---------------------------------------------------------------------------------------
 * Differentiation form (no counterpart in the reference): a differentiable depth loss over the
 * path and its hand-written adjoint.  Forward: corrected 3x3 cost averaged over the valid
 * sources, 8 SGM paths (their states kept, or recomputed per path in the backward), soft-argmin
 * rho_hat = sum_d softmax(-S/T)_d rho_d, loss = mean |rho_hat - rho_gt| over valid pixels with
 * rho_gt > 0.  Backward: gradients with respect to the source intensities and to the left se(3)
 * perturbation of every source pose (P_s -> exp([omega]) P_s + upsilon; omega first).
 * --------------------------------------------------------------------------------------- */
typedef struct pm_diff pm_diff;
typedef struct pm_diff_config {
    int width, height;
    int num_planes;      /* 32, 64, 128 or 256 */
    int num_sources;     /* 1 .. 4 */
    float rho0, rho_step;
    float temperature;   /* soft-argmin temperature in cost units */
    float p1, p2, tau_so, q1, q2;
    int store_paths;     /* 1: keep the 8 path-state volumes from the forward; 0: recompute */
    int device;
} pm_diff_config;
PM_API void pm_diff_config_default(pm_diff_config* c, int width, int height, int num_planes, int num_sources);
PM_API pm_status pm_diff_create(const pm_diff_config* c, pm_diff** out);
PM_API void pm_diff_destroy(pm_diff* d);
/* Device memory the handle holds (bytes). */
PM_API pm_status pm_diff_memory(const pm_diff* d, size_t* bytes);
/* ref (W*H), srcs (num_sources*W*H), rho_gt (W*H): device float images (scaled intensities,
 * ground-truth inverse depth, <= 0 where unknown); K without skew; R (9 per source) and t (3
 * per source): source-from-reference poses, row-major doubles; rho_hat: optional device W*H
 * output (0 outside the loss mask); *loss on the host.  The inputs must stay valid for the
 * backward. */
PM_API pm_status pm_diff_forward(pm_diff* d, const float* ref, const float* srcs, const double K[9], const double* R,
                                 const double* t, const float* rho_gt, float* rho_hat, double* loss, void* stream);
/* Gradients of the last forward's loss: grad_srcs (device, num_sources*W*H, overwritten) and
 * grad_pose (host, 6 per source: omega then upsilon). */
PM_API pm_status pm_diff_backward(pm_diff* d, float* grad_srcs, double* grad_pose, void* stream);
PM_API const char* pm_diff_last_error(const pm_diff* d);

/* ---------------------------------------------------------------------------------------
 * Stage-level calls: one call per reference launch wrapper.  Device pointers, caller-owned
 * buffers, asynchronous on `stream`.  Status codes report argument errors and launch errors.
 * --------------------------------------------------------------------------------------- */

/* uint8 -> scaled float image (the convertTo(CV_32F) + upload of stereo_mapper.cpp:66-67). */
PM_API pm_status pm_stage_to_float(int W, int H, const uint8_t* src, size_t src_pitch, float* dst,
                            float scale, void* stream);

/* ad_calc_cost (calc_cost.cu:212-253) for `nsrc` sources at once.  ref: W*H float; srcs: nsrc
 * consecutive W*H float images; homs: 12*nsrc floats in HOST memory.  cost: W*H*D float.
 * When cnt is NULL the volume starts from cost=-1, cnt=0 (initReference); otherwise cost and
 * cnt hold the running state and are updated in place, exactly as repeated ad_calc_cost
 * calls would.  invalid (optional, W*H bytes) receives 1 where some plane was never measured.
 * cfg->sampler PM_SAMPLER_TEXTURE_F32 samples the sources through textures, as the reference:
 * the call then allocates pitched copies of the sources and their texture objects, and returns
 * after the kernels have finished. */
PM_API pm_status pm_stage_calc_cost(const pm_config* cfg, const float* ref, const float* srcs, int nsrc,
                             const float* homs, float* cost, float* cnt, uint8_t* invalid,
                             void* stream);

/* sgm2 (sgm.cu:115-135): out := sum over cfg->num_paths paths; out needs no clearing.  Opposite
 * paths run pairwise in one kernel and each pair is aggregated into its own volume (out holds
 * pair 0, scratch the other num_paths/2 - 1: (num_paths/2 - 1)*W*H*D floats; a larger scratch,
 * such as the num_paths - 1 volumes earlier versions used, is fine), and the sum is
 * (P0 + P1) + (P2 + P3) [+ ((P4 + P5) + (P6 + P7))], paths in the reference's order. */
PM_API pm_status pm_stage_sgm(const pm_config* cfg, const float* cost, const float* ref, float* out,
                       float* scratch, void* stream);

/* filter_cost (filter_cost.cu:57-70): depth with a byte pitch; index (optional) W*H. */
PM_API pm_status pm_stage_filter(const pm_config* cfg, const float* sgm, float* depth, size_t pitch_bytes,
                          int32_t* index, void* stream);

/* sgm2 + filter_cost fused: the combine kernel adds the pair volumes in registers and runs the
 * winner-take-all; `scratch` holds the num_paths/2 pair volumes ((num_paths/2)*W*H*D floats). */
PM_API pm_status pm_stage_sgm_filter(const pm_config* cfg, const float* cost, const float* ref,
                              float* scratch, float* depth, size_t pitch_bytes, int32_t* index,
                              void* stream);

/* depth_fuse (depth_fusion.cu:229-280).  pose: R_p2c row-major then t_p2c (floats); cam: fx,
 * fy, cx, cy.  depth: W*H, in = WTA depth, out = fused depth.  pre/cur: alpha, beta, mu, sigma
 * (4 pointers each, W*H floats).  ztable: W*H uint64 scratch.  table (optional): W*H int32. */
PM_API pm_status pm_stage_depth_fuse(int W, int H, const float pose[12], const float cam[4],
                              float* depth, float* const pre[4], float* const cur[4],
                              uint64_t* ztable, int32_t* table, void* stream);

/* pm_stage_depth_fuse without the ztable argument, for callers that must not allocate device
 * memory at run time (a flight-control loop, a host framework that owns all device buffers,
 * work recorded into a CUDA graph).  No counterpart in the reference.  The z-buffer is a
 * library-owned __device__ array of 2^19 pixels (4 MiB, held by every GPU that loads the
 * library until exit); W*H above that returns PM_ERR_INVALID_ARGUMENT.  The array is cleared
 * at the start of each call and shared by all calls, so calls that overlap on the GPU race.
 * The call uses the array of the CURRENT device: `stream` must belong to the current device's
 * context (0 or the per-thread default stream are fine), else PM_ERR_INVALID_ARGUMENT.  The
 * first call in a context looks up the array's device address (cudaGetSymbolAddress); make
 * that first call before any stream capture.  After a cudaDeviceReset the device has a new
 * context, and the next call looks the address up again (again before any capture). */
PM_API pm_status pm_stage_depth_fuse_noalloc(int W, int H, const float pose[12], const float cam[4],
                                             float* depth, float* const pre[4], float* const cur[4],
                                             int32_t* table, void* stream);

/* The CPU fusion variant's step for a non-first keyframe, as outputFusionCPU runs it
 * (stereo_mapper.cpp:741-784): the masks of :743-760 on `result`, depthFuseCPU (:568-587:
 * transformMapCPU, holeFillingCPU, depthPreditCPU, depthUpdateCPU), then the re-mask of
 * :773-784.  pose: R_p2c row-major then t_p2c, doubles (the reference's Eigen types); cam: fx,
 * fy, cx, cy.  result: W*H, in = WTA depth, out = fused depth.  pre/cur: alpha, beta, mu, sigma
 * (4 device pointers each, W*H floats; pre is modified in place as transformMapCPU does).
 * table (optional): W*H uint32, the filled propagation table packed (y << 16) | x.  scratch:
 * pm_stage_depth_fuse_cpu_path_scratch(W, H) bytes of device memory.  W, H < 65536. */
PM_API size_t pm_stage_depth_fuse_cpu_path_scratch(int W, int H);
PM_API pm_status pm_stage_depth_fuse_cpu_path(int W, int H, const double pose[12], const float cam[4],
                                              float* result, float* const pre[4], float* const cur[4],
                                              uint32_t* table, void* scratch, void* stream);

/* convert (convert.cu:26-45).  flag != 0: linear -> pitched, else pitched -> linear.  The
 * pitch is in BYTES (the reference passed a byte step but indexed with it in floats). */
PM_API pm_status pm_stage_convert(int W, int H, const float* in, float* out, int flag,
                           size_t pitch_bytes, void* stream);

/* ---------------------------------------------------------------------------------------
 * Sequence tools: the image work and the output formats of the reference's driver
 * (evaluate.cc).  Kernels take device pointers and byte pitches (0 = packed) and run on
 * `stream`; the file functions take host memory.
 * --------------------------------------------------------------------------------------- */

/* cv::pyrDown(img, img, Size(W/2, H/2)) (evaluate.cc:176-178, 221-225): 5x5 binomial filter
 * [1 4 6 4 1]^T [1 4 6 4 1] / 256 at even pixels, mirrored borders (BORDER_REFLECT_101), rounded
 * half up.  dst is (W/2) x (H/2).  W, H >= 2. */
PM_API pm_status pm_pyr_down_u8(int W, int H, const uint8_t* src, size_t src_pitch, uint8_t* dst,
                                size_t dst_pitch, void* stream);

/* depthUp (evaluate.cc:121-135): each pixel of the W x H float map repeated in a 2x2 block of
 * the 2W x 2H dst. */
PM_API pm_status pm_depth_up2(int W, int H, const float* src, size_t src_pitch, float* dst, size_t dst_pitch,
                              void* stream);

/* The depth range mask of evaluate.cc:278-289, in place: depth < min_depth -> 0, then
 * depth > max_depth -> 0 (the driver uses 0.2 and 20). */
PM_API pm_status pm_depth_range_mask(int W, int H, float* depth, size_t pitch, float min_depth, float max_depth,
                                     void* stream);

/* The debug view of evaluate.cc:291-307.  level (optional, W x H bytes) receives
 * cv::normalize(depth, 0, 255, NORM_MINMAX, CV_8U); bgr (optional, 3 bytes per pixel, B G R)
 * receives a colour map of that level with pixels of depth < 0.001 black.  The colour map is
 * this library's own hue ramp (red, yellow, green, cyan, blue, magenta), not OpenCV's
 * COLORMAP_RAINBOW table.  scratch: 2 unsigned ints of device memory. */
PM_API pm_status pm_colorize_depth(int W, int H, const float* depth, size_t pitch, uint8_t* level,
                                   size_t level_pitch, uint8_t* bgr, size_t bgr_pitch, unsigned* scratch,
                                   void* stream);

/* The depth output message of evaluate.cc:271-276 (sensor_msgs/Image "32FC1", filled by
 * toImageMsg, src/tools/transport_util.h:103-132) becomes a file: PFM ("Pf", little-endian,
 * rows stored bottom-up as the format requires) or NPY (version 1.0, '<f4', shape (H, W)).
 * Host memory; pitch in bytes (0 = packed).  PM_ERR_INVALID_ARGUMENT when the file cannot be
 * written. */
PM_API pm_status pm_write_pfm(const char* path, int W, int H, const float* data, size_t pitch);
PM_API pm_status pm_write_npy(const char* path, int W, int H, const float* data, size_t pitch);
/* A B G R 8-bit image (pm_colorize_depth's bgr) as binary PPM (P6). */
PM_API pm_status pm_write_ppm(const char* path, int W, int H, const uint8_t* bgr, size_t pitch);

/* Reads an 8-bit frame for the driver: binary PGM/PPM (P5/P6), PNG (8-bit grey, grey+alpha,
 * palette, RGB, RGBA; 16-bit grey and RGB keep the high byte; not interlaced) or a 2-D uint8 NPY.
 * Colour becomes grey as cv::cvtColor(RGB2GRAY) does: (9798 R + 19235 G + 3735 B + 16384) >> 15.
 * Writes the size to *W, *H; with dst == NULL (or capacity too small, then
 * PM_ERR_INVALID_ARGUMENT) only the size.  dst rows are packed (pitch W). */
PM_API pm_status pm_read_image_u8(const char* path, int* W, int* H, uint8_t* dst, size_t capacity);

#ifdef __cplusplus
}
#endif
#endif /* PM_STEREO_H */
