// pm_internal.h -- launch descriptors shared by the kernels and the C-ABI runtime.
#pragma once

#include <cuda_runtime.h>
#include <stddef.h>
#include <stdint.h>

namespace pm {

constexpr int kMaxSources = 32;   // source frames evaluated in one cost pass
constexpr int kMaxPlanes = 256;   // 32 lanes x up to 8 planes per lane
constexpr float kDepInf = 1000.0f;   // DEP_INF (parameters.h:29)
constexpr double kFloatEps = 1e-5;   // FLOAT_EPS (parameters.h:6)
constexpr float kCaseInf = 10000.0f; // no-overlap value of the CASE 0/1 debug outputs (stereo_mapper.cpp:651)

// Per-map pixel counters (pm_stats): word offsets of the classes in the device counter block.
enum WtaClass { kWtaDepth = 0, kWtaNoOverlap, kWtaBorder, kWtaFlat, kWtaAmbiguous, kWtaClasses };
enum TransformClass { kTfEmpty = 0, kTfOutlier, kTfBehind, kTfOutside, kTfMoved, kTfClasses };
enum UpdateClass { kUpdEmpty = 0, kUpdInit, kUpdNoMeasurement, kUpdOutput, kUpdHidden, kUpdClasses };
constexpr int kStatWta = 0;
constexpr int kStatTf = kStatWta + kWtaClasses;
constexpr int kStatPred = kStatTf + kTfClasses;   // none, copied, filled
constexpr int kStatUpd = kStatPred + 3;
constexpr int kStatWords = kStatUpd + kUpdClasses;

// Access sites of the bounds-checked build (PM_BOUNDS_CHECK): the site of a recorded failure.
enum BoundsSite {
    kSiteCostSource = 1,   // cost kernel: a source quad
    kSiteCostState,        // cost kernel: a voxel of the running state (load or store)
    kSiteCostOffset,       // cost kernel: a block offset or pixel offset of the FP16 form
    kSiteRebase,           // rebase of the FP16 volume
    kSitePairLoad,         // SGM pair kernel: a cost slice
    kSitePairRef,          // SGM pair kernel: a reference pixel
    kSitePairOut,          // SGM pair kernel: a pair-volume slice (store or reduction)
    kSiteCombineLoad,      // combine kernel: a pair-volume slice or a pixel offset
    kSiteCombineOut,       // combine kernel: depth, index or class of a pixel
    kSiteFuseTransform,    // fusion: the z-buffer cell of a moved pixel
    kSiteFuseGather,       // fusion: a neighbour or predecessor cell
    kSiteCpuList,          // CPU-variant fusion: a hitter list entry or the occupant of a cell
    kSiteCpuGather,        // CPU-variant fusion: a neighbour or predecessor cell
    kSiteClassCount,       // pm_stats class counting
};

// ---- plane-sweep cost volume (calc_cost.cu) ----------------------------------------------
struct CostLaunch {
    const float* ref;      // W*H scaled reference image
    const float* srcs;     // nsrc consecutive W*H scaled source images (used when srcq is null)
    // nsrc consecutive W*H quad images (2x2 bilinear footprints); in the FP16 form (cost_half)
    // their values are rounded to FP16
    const float4* srcq;
    // use_tex: the sources through these texture objects (pitched images, linear filtering, zero
    // border; FP16 form: FP16 or FP16-rounded FP32 texels, FP32 form: FP32 texels)
    unsigned long long tex[kMaxSources];
    int use_tex;
    int W, H, D, nsrc;
    float rho0, drho;
    int mode;              // 0 reference quirks, 1 corrected 3x3 patch
    float hom[kMaxSources][12];
    const float* hom_dev;  // batched form: the homographies (nsrc x 12) in device memory, or nullptr
    void* cost;            // W*H*D float, or __half when cost_half
    int cost_half;
    // FP16 volumes hold cost - offset[pixel], offset = the pixel's smallest measured cost (0 when
    // some plane is unmeasured, i.e. for a pixel the SGM treats as invalid), so that the values
    // near the minimum keep FP16's relative precision.  The SGM recurrences are unchanged by a
    // per-pixel shift; the winner-take-all adds it back once per path.  The kernel first writes
    // each 16-plane block relative to its own minimum (block_offset); a rebase pass then moves
    // every block to the pixel's offset.
    float* offset;         // W*H (cost_half only)
    float* block_offset;   // W*H*(D/16) scratch (cost_half only)
    float* cnt;            // running count (incremental mode) or nullptr
    uint8_t* invalid;      // W*H, 1 where a plane was never measured (optional)
    int incremental;       // start from (cost, cnt) in memory instead of (-1, 0)
    cudaEvent_t kernel_done = nullptr;   // recorded right after the cost kernel (before the rebase)
};
cudaError_t launch_cost(const CostLaunch& a, cudaStream_t s);

// ---- SGM aggregation + winner-take-all (sgm.cu, filter_cost.cu) ---------------------------
struct PlaneOrder {
    uint32_t incl[32];          // bit j of incl[l]: plane l*PPL+j takes part in the reduction tree
    uint16_t rank[kMaxPlanes];  // tie-break priority of each plane (0 wins)
};
// Priority of the reference reduction tree (filter_cost.cu:22-30); compat=0 keeps all planes.
void plane_order(int D, int compat, PlaneOrder& out);

struct FilterParams {
    float var_scale, uniq, rho0, drho;
};

struct SgmLaunch {
    const void* cost;      // W*H*D float or __half
    int cost_half;
    const float* ref;      // W*H scaled reference image (path gradient D1, sgm.cu:75)
    void* part[4];         // W*H*D volume of each opposite-path pair (num_paths / 2 of them): P_2p + P_2p+1,
                           // float, or __half when part_half
    int part_half;         // FP16 form: the pair volumes hold FP16 values (sums rounded to FP16)
    float* total;          // W*H*D complete sum (may alias part[0]); nullptr: not stored
    const float* offset;   // W*H per-pixel shift of an FP16 cost volume (see CostLaunch), or nullptr
    int W, H, D, num_paths;
    float p1, p2, tau, q1, q2;
    FilterParams fp;
    float* depth;          // W*H with byte pitch depth_pitch (fused filter only)
    size_t depth_pitch;
    int32_t* index;        // W*H (optional)
    PlaneOrder order;
    int pair_warps;        // scanlines per block of the path-pair kernel: 2, 4 or 8 (0: 2)
    int serial_pairs;      // 1: run the path pairs one after another on the caller's stream
    int priority;          // launch priority of the pair and combine kernels (0: the stream's)
    uint8_t* wta_class;    // W*H winner-take-all class of each pixel (WtaClass, fused filter only), or nullptr
};
// pm_stats: adds the per-pixel classes (values below n) of npix pixels to the n counters at g.
cudaError_t launch_count_classes(const uint8_t* cls, long npix, int n, unsigned* g, cudaStream_t s);
// Side streams for the concurrent path pairs: pairs 0..2 fork from the caller's stream and join
// back before the combine kernel.
struct SgmStreams {
    cudaStream_t stream[3];
    cudaEvent_t fork;
    cudaEvent_t join[3];
};
// What the combine kernel does with the summed path volumes.
enum CombineMode { kCombineStore = 0, kCombineFilter = 1, kCombineArgmin = 2 };
// Runs the opposite-path pairs (pair p into part[p]), then adds the pair volumes in registers
// and writes depth/index with the winner-take-all filter (kCombineFilter) or the debug argmin
// (kCombineArgmin); kCombineStore only writes `total`.  side == nullptr runs everything on s.
cudaError_t launch_sgm(const SgmLaunch& a, int mode, cudaStream_t s, const SgmStreams* side);
// The debug argmin over a float (half = 0) or __half (half = 1, shifted by offset) W*H*D volume.
cudaError_t launch_case_argmin(const void* vol, int half, const float* offset, int W, int H, int D,
                               const FilterParams& fp, float* depth, size_t pitch, int32_t* index, cudaStream_t s);
cudaError_t launch_filter(const float* sum, int W, int H, int D, const FilterParams& fp,
                          const PlaneOrder& order, float* depth, size_t pitch, int32_t* index,
                          cudaStream_t s);

// ---- image conversion (convert.cu + the uint8 -> float upload) ----------------------------
cudaError_t launch_to_float(int W, int H, const uint8_t* src, size_t src_pitch, float* dst,
                            float scale, cudaStream_t s);
// uint8 -> scaled float rows with a byte pitch (the FP32 form's texture storage).
cudaError_t launch_to_float_pitched(int W, int H, const uint8_t* src, size_t src_pitch, float* dst,
                                    size_t dst_pitch, float scale, cudaStream_t s);
// uint8 -> scaled FP16 image with a byte pitch (the FP16 form's texture storage).
cudaError_t launch_to_half(int W, int H, const uint8_t* src, size_t src_pitch, void* dst, size_t dst_pitch,
                           float scale, cudaStream_t s);
// uint8 -> FP16-rounded values in pitched float rows (the FP16 form's FP32-texel textures).
cudaError_t launch_to_float_h_pitched(int W, int H, const uint8_t* src, size_t src_pitch, float* dst,
                                     size_t dst_pitch, float scale, cudaStream_t s);
// uint8 -> quads of FP16-rounded values in FP32 lanes: the FP16 form's exact sampler.
cudaError_t launch_to_quad_half(int W, int H, const uint8_t* src, size_t src_pitch, float4* dst, float scale,
                                cudaStream_t s);
// uint8 -> scaled float image whose values are rounded to FP16 (the FP16 form's reference image).
cudaError_t launch_to_float_h(int W, int H, const uint8_t* src, size_t src_pitch, float* dst, float scale,
                              cudaStream_t s);
// uint8 -> scaled quad image: dst[y*W + x] = (I(x,y), I(x,y+1), I(x+1,y), I(x+1,y+1)), zero
// outside the image (the border addressing of the reference textures, calc_cost.cu:230-237).
cudaError_t launch_to_quad(int W, int H, const uint8_t* src, size_t src_pitch, float4* dst,
                           float scale, cudaStream_t s);
// A pitched W x H source image (FP16 texels, or FP32 texels when f32) and its texture object:
// linear filtering, zero border, unnormalised coordinates (the reference's texture setup,
// calc_cost.cu:226-237).
cudaError_t make_source_texture(int W, int H, bool f32, void** buf, size_t* pitch, unsigned long long* tex);
cudaError_t launch_convert(int W, int H, const float* in, float* out, int flag, size_t pitch_bytes,
                           cudaStream_t s);

// ---- depth fusion (depth_fusion.cu) --------------------------------------------------------
struct FuseLaunch {
    int W, H;
    float pose[12];        // R_p2c row-major, t_p2c
    float cam[4];          // fx, fy, cx, cy
    float* depth;          // in: WTA depth (unless depth_in is given), out: fused depth (W*H)
    const float* depth_in; // W*H WTA depth read instead of depth (nullptr: depth in place)
    float* pre[4];         // alpha, beta, mu, sigma of the previous keyframe (modified)
    float* cur[4];         // state of the current keyframe (written)
    unsigned long long* ztable;  // W*H scratch z-buffer
    int32_t* table;        // W*H filled propagation table (optional)
    float* variance;       // W*H sigma^2 of the current state (optional)
    // Batched form (values that change every step, read from device memory so that a captured
    // graph stays valid): params_dev = pose[12], cam[4]; flags_dev = {first, pre_index}; the
    // state sets are state[pre_index] (previous) and state[pre_index ^ 1] (current).  On the first
    // frame both state sets, the fused depth and the variance are cleared (stereo_mapper.cpp:128-146).
    const float* params_dev;
    const int* flags_dev;
    float* state[2][4];
    unsigned* stats;       // kStatWords counters (transform, predict and update classes added), or nullptr
};
cudaError_t launch_fuse_gpu(const FuseLaunch& a, cudaStream_t s);

// The CPU fusion variant (outputFusionCPU, stereo_mapper.cpp:625-820) run on the GPU.
struct FuseCpuLaunch {
    int W, H;              // both below 65536 (packed (y << 16) | x table)
    double pose[12];       // R_p2c row-major, t_p2c (double, as the reference's Eigen code)
    float cam[4];          // fx, fy, cx, cy
    float* result;         // in: WTA depth, out: fused and masked depth (W*H)
    float* pre[4];         // alpha, beta, mu, sigma of the previous keyframe (modified)
    float* cur[4];         // state of the current keyframe
    uint32_t* table;       // W*H filled propagation table, packed (y << 16) | x (optional)
    float* variance;       // W*H sigma^2 of the current state (optional)
    // scratch, W*H each
    uint8_t* mask;
    float* orig_mu;
    int* head;
    int* next;
    uint32_t* tab0;
    unsigned* stats;       // kStatWords counters, or nullptr
};
cudaError_t launch_fuse_cpu_variant(const FuseCpuLaunch& a, cudaStream_t s);

// ---- host-side geometry, FP64 (api.cu) -----------------------------------------------------
void matmul3(const double* A, const double* B, double* C);
void matvec3(const double* A, const double* x, double* y);
void transpose3(const double* A, double* T);
bool finite_n(const double* v, int n);
// H1 = K R_r^T R_l K^-1 and H2 = K R_r^T (T_l - T_r) (stereo_mapper.cpp:79-80) as 12 floats
void compose_homography(const double* K, const double* Rl, const double* Tl, const double* Rr,
                        const double* Tr, float out[12]);
// relative pose of the previous keyframe in the current one (stereo_mapper.cpp:155-156), 12 floats
void fusion_pose(const double* R, const double* t, const double* R_prev, const double* t_prev, float out[12]);
void fusion_pose_d(const double* R, const double* t, const double* R_prev, const double* t_prev, double out[12]);

}  // namespace pm
