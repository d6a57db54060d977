// pm_stereo_mapper.hpp -- C++ StereoMapper over the C ABI of libpm_stereo.so.
//
// Same class name and method names as the reference (motion_stereo/stereo_mapper.h:26-63), with
// raw pointers in place of cv::Mat / Eigen types (OpenCV is not a dependency):
//   cv::Mat 8UC1 image           -> const uint8_t* data + row pitch in bytes
//   cv::Mat 3x3 / 3x1 CV_64F     -> const double[9] row-major / const double[3]
//   Eigen::Matrix3d (col-major)  -> const double[9] row-major (use RowMajor maps or transpose)
//   cv::Mat& result (CV_32F)     -> float* + pitch (host or device memory)
// Failures throw pm::Error carrying the status code and the library's message.
#pragma once

#include <cstddef>
#include <cstdint>
#include <stdexcept>
#include <string>

#include "pm_stereo.h"

namespace pm {

class Error : public std::runtime_error {
public:
    Error(pm_status s, const std::string& what) : std::runtime_error(what), status(s) {}
    pm_status status;
};

class StereoMapper {
public:
    // StereoMapper::StereoMapper (stereo_mapper.cpp:27-49); the shape is a runtime argument.
    explicit StereoMapper(const pm_config& cfg) { check(pm_create(&cfg, &h_), "pm_create"); }
    StereoMapper(int width, int height, int num_planes) {
        pm_config cfg;
        pm_config_default(&cfg, width, height, num_planes);
        check(pm_create(&cfg, &h_), "pm_create");
    }
    ~StereoMapper() { pm_destroy(h_); }
    StereoMapper(const StereoMapper&) = delete;
    StereoMapper& operator=(const StereoMapper&) = delete;

    void initIntrinsic(const double K[9], float bf, float dep_sample) {
        check(pm_init_intrinsic(h_, K, bf, dep_sample), "initIntrinsic");
    }
    void initReference(const uint8_t* img, size_t pitch_bytes) {
        check(pm_init_reference(h_, img, pitch_bytes), "initReference");
    }
    void update(const uint8_t* img, size_t pitch_bytes, const double R_l[9], const double T_l[3],
                const double R_r[9], const double T_r[3]) {
        check(pm_update(h_, img, pitch_bytes, R_l, T_l, R_r, T_r), "update");
    }
    void output(float* depth, size_t pitch_bytes) { check(pm_output(h_, depth, pitch_bytes), "output"); }
    void outputFusion(float* depth, size_t depth_pitch, const double R[9], const double t[3], float fx, float fy,
                      float cx, float cy, float* variance = nullptr, size_t variance_pitch = 0) {
        check(pm_output_fusion(h_, depth, depth_pitch, variance, variance_pitch, R, t, fx, fy, cx, cy),
              "outputFusion");
    }
    // StereoMapper::outputFusionCPU (stereo_mapper.cpp:625-820): with CASE >= 3 the fused map of a
    // mapper created with fusion_variant = PM_FUSION_CPU_PATH, else the CASE 0/1/2 debug output.
    void outputFusionCPU(float* depth, size_t depth_pitch, const double R[9], const double t[3], float fx,
                         float fy, float cx, float cy, int output_case = 3) {
        if (output_case >= 3)
            check(pm_output_fusion(h_, depth, depth_pitch, nullptr, 0, R, t, fx, fy, cx, cy), "outputFusionCPU");
        else
            check(pm_output_case(h_, output_case, depth, depth_pitch), "outputFusionCPU");
    }
    void wtaDepth(float* depth, size_t pitch_bytes) { check(pm_get_wta_depth(h_, depth, pitch_bytes), "wtaDepth"); }
    // Pixel counters of the last output call (the reference's commented-out cnt0..cnt4 counters,
    // stereo_mapper.cpp:329, 431, 565, and the winner-take-all outcomes).
    void enableStats(bool on) { check(pm_enable_stats(h_, on ? 1 : 0), "enableStats"); }
    pm_stats stats() {
        pm_stats s;
        check(pm_get_stats(h_, &s), "stats");
        return s;
    }
    void setStream(void* cuda_stream) { check(pm_set_stream(h_, cuda_stream), "setStream"); }
    void synchronize() { check(pm_synchronize(h_), "synchronize"); }
    pm_mapper* handle() const { return h_; }

private:
    void check(pm_status s, const char* what) const {
        if (s != PM_OK) {
            std::string msg = std::string(what) + ": " + pm_status_string(s);
            if (h_ && pm_last_error(h_)[0]) msg += std::string(" (") + pm_last_error(h_) + ")";
            throw Error(s, msg);
        }
    }
    pm_mapper* h_ = nullptr;
};

}  // namespace pm
