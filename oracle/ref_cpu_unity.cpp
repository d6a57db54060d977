// ref_cpu_unity.cpp -- TEST INFRASTRUCTURE.  Compiles the reference's own
// motion_stereo/stereo_mapper.cpp (HKUST-Aerial-Robotics/probabilistic_mapping; included from
// where it lies, never copied) on the host, against the stand-in headers of oracle/ref_stubs/
// (Eigen, OpenCV, ROS) and the parameter names of oracle/ref_params.h, so that its CPU fusion
// variant -- outputFusionCPU (stereo_mapper.cpp:625-820) with transformMapCPU, holeFillingCPU,
// depthPreditCPU, depthUpdateCPU and depthFuseCPU (:246-587), and the CASE 0 / CASE 1 argmin
// outputs (:628-706) -- runs unmodified and can pin the CPU oracle and the GPU kernels.
//
// The reference's GPU stages are not part of this build.  Where outputFusionCPU calls them
// (sgm2, filter_cost) the harness's stand-ins below hand over the maps the GPU stages would have
// produced, which the caller supplies: the SGM volume for CASE 1, the winner-take-all depth for
// CASE >= 2.  GpuMat (oracle/ref_stubs) keeps its elements in host memory for this.  Built by
// oracle/build_ref.py (build_cpu) into oracle/_ref/libref_cpu_<W>x<H>x<D>.so.
#include "stereo_mapper.cpp"
#include "parameters.cpp"

#include <cstdint>

namespace {

const float* g_sgm_in = nullptr;   // CASE 1: the SGM volume sgm2 would write
const float* g_wta_in = nullptr;   // CASE >= 2: the depth filter_cost would write
StereoMapper* g_mapper = nullptr;

}  // namespace

// ---- stand-ins for the GPU launch wrappers (calc_cost.h, sgm.h, filter_cost.h, ...) ---------
void ad_calc_cost(unsigned char*, float, float, float, float, float, float, float, float, float, float, float,
                  float, unsigned char*, size_t, unsigned char*, size_t, unsigned char*, float) {}

void sgm2(unsigned char*, unsigned char* output) {
    if (g_sgm_in) std::memcpy(output, g_sgm_in, sizeof(float) * (size_t)WIDTH * HEIGHT * DEP_CNT);
}

void filter_cost(unsigned char*, unsigned char* dep, size_t pitch_dep, float) {
    if (!g_wta_in) return;
    for (int y = 0; y < HEIGHT; ++y)
        std::memcpy(dep + (size_t)y * pitch_dep, g_wta_in + (size_t)y * WIDTH, sizeof(float) * WIDTH);
}

void depth_fuse(float, float, float, float, float, float, float, float, float, float, float, float, float, float,
                float, float, unsigned char*, unsigned char*, unsigned char*, unsigned char*, unsigned char*,
                unsigned char*, unsigned char*, unsigned char*, unsigned char*, unsigned char*) {}

void convert(unsigned char*, unsigned char*, bool, size_t) {}

extern "C" {

int refcpu_shape(int* w, int* h, int* d) {
    *w = WIDTH;
    *h = HEIGHT;
    *d = DEP_CNT;
    return 0;
}

// A fresh StereoMapper (firstDepth = true): the start of a sequence.  K row-major 3x3.  The
// reference frame is set by the reference's own initReference with a blank 8-bit image (only
// its size matters to the fusion path, which sizes the first result by it).
int refcpu_reset(const double K[9], float dep_sample) {
    delete g_mapper;
    g_mapper = new StereoMapper();
    cv::Mat k(3, 3, CV_64F);
    for (int i = 0; i < 9; ++i) k.at<double>(i / 3, i % 3) = K[i];
    g_mapper->initIntrinsic(k, 0.0f, dep_sample);
    cv::Mat blank(HEIGHT, WIDTH, CV_8U);
    blank.setTo(0.0);
    g_mapper->initReference(blank);
    return 0;
}

// One StereoMapper::outputFusionCPU call with the global CASE = output_case.
//   raw_cost (CASE 0): the cost volume, W*H*D floats in the INDEX layout (cuda_utils.h:34);
//   sgm      (CASE 1): the SGM volume, same layout;
//   wta      (CASE >= 2): the winner-take-all depth, W*H;
//   R, t: the keyframe pose (row-major 3x3, 3-vector); fx, fy, cx, cy: the camera.
// result receives W*H floats.  state (may be NULL) receives alpha, beta, mu, sigma as 4 x 2
// planes of W*H floats (both ping-pong halves) and table the two W*H p_table planes.
int refcpu_output_fusion_cpu(int output_case, const float* raw_cost, const float* sgm, const float* wta,
                             const double R[9], const double t[3], float fx, float fy, float cx, float cy,
                             float* result, float* state, uint32_t* table) {
    if (!g_mapper) return 1;
    CASE = output_case;
    if (output_case == 0 && raw_cost)
        std::memcpy(g_mapper->raw_cost.data, raw_cost, sizeof(float) * (size_t)WIDTH * HEIGHT * DEP_CNT);
    g_sgm_in = sgm;
    g_wta_in = wta;
    Eigen::Matrix3d Rm;
    Eigen::Vector3d tv;
    for (int i = 0; i < 9; ++i) Rm(i / 3, i % 3) = R[i];
    for (int i = 0; i < 3; ++i) tv(i) = t[i];
    cv::Mat res;
    g_mapper->outputFusionCPU(res, Rm, tv, fx, fy, cx, cy);
    g_sgm_in = g_wta_in = nullptr;
    if (res.rows != HEIGHT || res.cols != WIDTH) return 2;
    for (int y = 0; y < HEIGHT; ++y) std::memcpy(result + (size_t)y * WIDTH, &res.at<float>(y, 0), sizeof(float) * WIDTH);
    const size_t N = (size_t)WIDTH * HEIGHT;
    if (state) {
        for (int k = 0; k < 2; ++k) {
            std::memcpy(state + (0 * 2 + k) * N, &alpha[k][0][0], sizeof(float) * N);
            std::memcpy(state + (1 * 2 + k) * N, &beta[k][0][0], sizeof(float) * N);
            std::memcpy(state + (2 * 2 + k) * N, &mu[k][0][0], sizeof(float) * N);
            std::memcpy(state + (3 * 2 + k) * N, &sigma[k][0][0], sizeof(float) * N);
        }
    }
    if (table)
        for (int k = 0; k < 2; ++k) std::memcpy(table + k * N, &p_table[k][0][0], sizeof(uint32_t) * N);
    return 0;
}

// The mapper's ping-pong index of the state the next call reads (pre_index).
int refcpu_pre_index() { return g_mapper ? g_mapper->pre_index : -1; }

}  // extern "C"
