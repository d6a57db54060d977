/*
 * pm_oracle.h -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * CPU restatement of the HKUST-Aerial-Robotics/probabilistic_mapping motion-stereo path
 * (motion_stereo/{calc_cost,sgm,filter_cost,depth_fusion,convert}.cu and the
 * StereoMapper orchestration in motion_stereo/stereo_mapper.cpp).  Only tests/,
 * __graft_entry__.smoke() and bench.py's cpu_baseline / reference arm may load it,
 * and only as the checker or the timed CPU baseline -- never as the product path.
 *
 * Every entry point exists in two instantiations:
 *   *_f64  -- the line-for-line FP64 transcription (parity target);
 *   *_f32  -- the same algorithm in FP32 with the op order of the B200 kernels, so that
 *             the GPU result can be compared bit-for-bit.
 *
 * Parity status: pinned against the reference's own CUDA (built unmodified through
 * oracle/ref_shim.h, run on a B200; outputs in tests/golden/ref_40x32x32.npz, generated by
 * tests/golden/make_ref_golden.py, checked by tests/test_golden.py): SGM, filter and convert
 * bit-exact, cost counts/validity exact and values within the texture-unit bilinear rounding,
 * fusion transform and z-buffer exact.  The CPU fusion variant (host C++ needing OpenCV and
 * Eigen) is checked by analytic known-answer tests only.
 *
 * Layouts: images are W*H row-major uint8; cost volumes are plane-innermost
 * ((y*W + x)*D + d), as INDEX() in motion_stereo/cuda_utils.h:34.
 */
#ifndef PM_ORACLE_H
#define PM_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_params {
    int W, H, D;
    double rho0;          /* inverse depth of plane 0 (reference: 0, calc_cost.cu:81) */
    double drho;          /* DEP_SAMPLE, plane spacing in inverse depth */
    double intensity_scale; /* image = uint8 * scale (reference: 1, stereo_mapper.cpp:66) */
    int cost_mode;        /* 0 = reference (keeps calc_cost.cu:50-51,70-71,106,119), 1 = corrected 3x3 */
    int bilinear_quant;   /* 1 = round bilinear weights to 1/256 like the texture unit */
    int num_paths;        /* 4 (sgm.cu:119-133) or 8 (adds the diagonals) */
    double p1, p2, tau_so, q1, q2;  /* parameters.cpp:12-16 */
    double var_scale;     /* parameters.cpp:18 */
    double uniqueness;    /* extension: reject when best > ratio * second best; <=0 or >=1 disables */
    int tree_compat;      /* 1 = reproduce the reduction tree of sgm.cu:24-31 for non power-of-two D */
    int sum_order;        /* 0 = reference path order, 1 = grouped order of the B200 kernels */
} orc_params;

/* a1: H1 = K R_r^T R_l K^-1, H2 = K R_r^T (T_l - T_r)  (stereo_mapper.cpp:79-80).
 * All matrices row-major doubles.  out[0..8] = H1, out[9..11] = H2. */
void orc_compose_homography(const double K[9], const double Rl[9], const double Tl[3],
                            const double Rr[9], const double Tr[3], double out[12]);

/* a12: relative pose for fusion, R_p2c = R^T R_prev, t_p2c = R^T (t_prev - t)
 * (stereo_mapper.cpp:155-156).  out[0..8] rotation, out[9..11] translation. */
void orc_relative_pose(const double R[9], const double t[3], const double Rprev[9],
                       const double tprev[3], double out[12]);

/* a3: plane-sweep cost volume over S sources (calc_cost.cu:11-210), running mean over the
 * sources in call order starting from cost=-1, cnt=0 (stereo_mapper.cpp:69-70).
 * homs: S*12 homography values as produced by orc_compose_homography. */
void orc_calc_cost_f64(const orc_params* p, const uint8_t* ref, const uint8_t* srcs, int S,
                       const double* homs, double* cost, double* cnt);
void orc_calc_cost_f32(const orc_params* p, const uint8_t* ref, const uint8_t* srcs, int S,
                       const double* homs, float* cost, float* cnt);

/* a4: SGM min-sum aggregation over num_paths directions (sgm.cu:5-135); sgm out = sum. */
void orc_sgm_f64(const orc_params* p, const uint8_t* ref, const double* cost, double* sgm);
void orc_sgm_f32(const orc_params* p, const uint8_t* ref, const float* cost, float* sgm);

/* a5: winner-take-all + flatness (+ optional uniqueness) + parabola subpixel
 * (filter_cost.cu:3-55).  depth: W*H, idx: W*H WTA plane index. */
void orc_filter_f64(const orc_params* p, const double* sgm, double* depth, int32_t* idx);
void orc_filter_f32(const orc_params* p, const float* sgm, float* depth, int32_t* idx);
/* The same with each pixel's outcome class: 0 depth, 1 non-overlap, 2 border plane, 3 flat,
 * 4 ambiguous (the pm_stats winner-take-all classes). */
void orc_filter_classes_f32(const orc_params* p, const float* sgm, float* depth, int32_t* idx, uint8_t* cls);

/* Plane priority of the WTA reduction tree (filter_cost.cu:22-30): rank[d] (0 = wins ties)
 * and incl[d] (0 when the tree never compares plane d). */
void orc_tree_order(int D, int tree_compat, int32_t* rank, int32_t* incl);

/* a6-a10: GPU depth-fusion step (depth_fusion.cu:8-225) with the races replaced by a
 * deterministic rule: the z-buffer keeps the smallest transformed depth, ties to the smaller
 * pixel index; hole filling takes the last occupied interior 3x3 neighbour in raster order.
 * depth: in = WTA depth, out = fused depth.  pre_* are modified in place like transformMap.
 * pose: float R_p2c[9], t_p2c[3]; cam: fx, fy, cx, cy. */
void orc_fuse_gpu_f64(int W, int H, const float pose[12], const float cam[4], double* depth,
                      double* pa, double* pb, double* pm, double* ps,
                      double* ca, double* cb, double* cm, double* cs, int32_t* table);
void orc_fuse_gpu_f32(int W, int H, const float pose[12], const float cam[4], float* depth,
                      float* pa, float* pb, float* pm, float* ps,
                      float* ca, float* cb, float* cm, float* cs, int32_t* table);
/* The same with the step's 13 pm_stats fusion counters: transform empty, outlier, behind,
 * outside, moved (transformMap :26-48); prediction none, copied, filled (depth_predict
 * :128-136, hole_filling); update empty, init, no measurement, output, hidden (:161-219). */
void orc_fuse_gpu_counts_f32(int W, int H, const float pose[12], const float cam[4], float* depth,
                             float* pa, float* pb, float* pm, float* ps,
                             float* ca, float* cb, float* cm, float* cs, int32_t* table, uint32_t* counts);

/* a13: CPU fusion variant (stereo_mapper.cpp:246-587) with the masking of
 * outputFusionCPU (stereo_mapper.cpp:743-784).  Sequential, as in the reference.
 * state: 2 * W*H each of alpha, beta, mu, sigma (the [2][H][W] statics); pre selects
 * the previous slot; pose is double R_p2c[9], t_p2c[3].  result: in = WTA depth, out = fused. */
void orc_fuse_cpu(int W, int H, const double pose[12], const float cam[4], int pre,
                  float* result, float* alpha, float* beta, float* mu, float* sigma,
                  uint32_t* table);
/* The same with the 13 counters of orc_fuse_gpu_counts_f32, classified as transformMapCPU,
 * depthPreditCPU and depthUpdateCPU count them (stereo_mapper.cpp:274-326, 405-421, 466-556). */
void orc_fuse_cpu_counts(int W, int H, const double pose[12], const float cam[4], int pre,
                         float* result, float* alpha, float* beta, float* mu, float* sigma,
                         uint32_t* table, uint32_t* counts);

/* a11: pitched <-> linear float copy (convert.cu:4-24), byte pitch. flag=1: linear->pitched. */
void orc_convert(int W, int H, const void* in, void* out, int flag, uint64_t pitch_bytes);

int orc_num_threads(void);
void orc_set_num_threads(int n);

/* Differentiable form (pm_oracle_diff.cpp): FP64 forward (cost over the corrected 3x3 patch, 8
 * SGM paths, soft-argmin at temperature T, L1 loss against rho_gt over valid pixels with
 * rho_gt > 0) and its adjoint.  ref: W*H, srcs: S*W*H scaled intensities; K: 3x3 without skew;
 * R: S*9, t: S*3 source-from-reference poses.  g_pose: S*6, the left se(3) perturbation
 * (omega, upsilon) of each source pose. */
typedef struct orc_diff_params {
    int W, H, D, S, num_paths;
    double rho0, drho, temperature;
    double p1, p2, tau_so, q1, q2;
} orc_diff_params;
double orc_diff_forward(const orc_diff_params* p, const double* ref, const double* srcs, const double* K,
                        const double* R, const double* t, const double* rho_gt, double* rho_hat, uint8_t* valid);
double orc_diff_backward(const orc_diff_params* p, const double* ref, const double* srcs, const double* K,
                         const double* R, const double* t, const double* rho_gt, double* g_srcs, double* g_pose);
/* The validity flag of each (pixel, plane, source) at a pose: ok[(pixel * D + d) * S + s] = 1
 * when all nine samples of the patch land inside the image with w >= 0.  The frozen forward
 * keeps those flags (the set of sources averaged into each voxel, and the pixel validity) while
 * the pose moves, so that central differences over a pose step see no border jumps. */
void orc_diff_source_validity(const orc_diff_params* p, const double* ref, const double* srcs, const double* K,
                              const double* R, const double* t, uint8_t* ok);
double orc_diff_forward_frozen(const orc_diff_params* p, const double* ref, const double* srcs, const double* K,
                               const double* R, const double* t, const double* rho_gt, const uint8_t* frozen);

#ifdef __cplusplus
}
#endif
#endif
