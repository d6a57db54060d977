// Builds against include/pm_stereo_mapper.hpp and libpm_stereo.so the way a C++ host program
// (the reference's evaluate.cc) would, and exercises the error path: a bad configuration must
// raise pm::Error with PM_ERR_INVALID_ARGUMENT.  With a GPU present (argv[1] == "gpu") it also
// maps one synthetic frame pair and checks that the depth map is finite and that the pixel
// counters add up.
#include <cmath>
#include <cstdio>
#include <cstring>
#include <vector>

#include "pm_stereo_mapper.hpp"

int main(int argc, char** argv) {
    pm_config cfg;
    pm_config_default(&cfg, 64, 48, 48);   // 48 planes: not a multiple of 32
    try {
        pm::StereoMapper bad(cfg);
        std::printf("no error raised\n");
        return 1;
    } catch (const pm::Error& e) {
        if (e.status != PM_ERR_INVALID_ARGUMENT) {
            std::printf("wrong status %d\n", e.status);
            return 1;
        }
    }
    if (argc > 1 && std::strcmp(argv[1], "gpu") == 0) {
        const int W = 64, H = 48;
        pm::StereoMapper m(W, H, 64);
        const double K[9] = {50, 0, 32, 0, 50, 24, 0, 0, 1};
        m.initIntrinsic(K, 0.0f, 0.02f);
        std::vector<uint8_t> ref(W * H), src(W * H);
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                ref[y * W + x] = (uint8_t)(128 + 100 * std::sin(0.7 * x) * std::cos(0.5 * y));
                src[y * W + x] = (uint8_t)(128 + 100 * std::sin(0.7 * (x + 2)) * std::cos(0.5 * y));
            }
        const double I[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1}, T0[3] = {0, 0, 0}, T1[3] = {0.1, 0, 0};
        m.enableStats(true);
        m.initReference(ref.data(), W);
        m.update(src.data(), W, I, T0, I, T1);
        std::vector<float> depth(W * H);
        m.output(depth.data(), W * sizeof(float));
        const pm_stats st = m.stats();   // every pixel in one winner-take-all class
        if (st.wta_depth + st.wta_no_overlap + st.wta_border + st.wta_flat + st.wta_ambiguous != (uint32_t)(W * H)) {
            std::printf("winner-take-all counters do not add up to the pixels\n");
            return 1;
        }
        for (float d : depth)
            if (!std::isfinite(d)) {
                std::printf("non-finite depth\n");
                return 1;
            }
        // the CASE 2 debug output of outputFusionCPU is the filtered depth itself
        std::vector<float> case2(W * H);
        m.outputFusionCPU(case2.data(), W * sizeof(float), I, T0, 50, 50, 32, 24, 2);
        if (std::memcmp(case2.data(), depth.data(), depth.size() * sizeof(float)) != 0) {
            std::printf("CASE 2 differs from output\n");
            return 1;
        }
    }
    std::printf("ok\n");
    return 0;
}
