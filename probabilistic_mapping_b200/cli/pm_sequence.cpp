// pm_sequence -- headless sequence driver over libpm_stereo.so, in place of the reference's ROS
// node (evaluate.cc:137-361).
//
// Input is a TUM-style sequence: an image list ("timestamp file" per line, '#' comments) and a
// pose list ("timestamp tx ty tz qx qy qz qw", camera-to-world).  The node's callbacks push each
// image and pose to the front of two lists (evaluate.cc:87-116); replayed offline, the poses up
// to an image's time arrive before that image, and after every arrival processImg runs until it
// has nothing left to do.  processImg (evaluate.cc:137-309) is restated exactly:
//   * it waits until the image list holds more than lastSize frames (lastSize starts at
//     aggNum * interval = 18, evaluate.cc:348, and grows by one per keyframe);
//   * the newest image is the reference; it needs a pose with the same timestamp, searched from
//     the newest pose (evaluate.cc:183-205), and waits while the newest pose is older;
//   * the sources are the images interval, 2 interval, ... aggNum interval places older, with
//     the poses the same number of places older than the matched pose (evaluate.cc:213-231);
//   * the oldest image and pose are dropped (evaluate.cc:234-235), so in a steady stream a
//     keyframe is made for every second frame.
// Each keyframe runs initReference, aggNum updates and outputFusionCPU (CASE selects the output,
// stereo_mapper.cpp:628-719) through the C ABI, then depthUp for every pyramid level
// (evaluate.cc:262-266).  That depth -- the "32FC1" message of evaluate.cc:271-276 -- is written as
// PFM or NPY; the min/max-depth mask and the colour view (evaluate.cc:278-307) go to a PPM when
// asked for.  Frames are halved downsample times with cv::pyrDown's filter on the GPU and the
// intrinsics follow evaluate.cc:330-335.
//
// --dry-run prints the keyframe schedule (one JSON object per line) and touches no GPU.
// --associate T gives every image the pose nearest in time within T seconds, stamped with the
// image's time, before the replay (the reference needs poses stamped exactly like the images).
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <deque>
#include <fstream>
#include <sstream>
#include <string>
#include <vector>

#include "pm_stereo.h"

namespace {

struct Stamp {
    long long ns = 0;   // the decimal timestamp, exactly, in nanoseconds
    std::string text;
};

bool parse_stamp(const std::string& s, Stamp& out) {
    const size_t dot = s.find('.');
    const std::string ip = s.substr(0, dot), fp = dot == std::string::npos ? "" : s.substr(dot + 1);
    if (ip.empty() || ip.size() > 10 || fp.size() > 9) return false;
    for (char c : ip + fp)
        if (c < '0' || c > '9') return false;
    long long frac = 0;
    for (size_t i = 0; i < 9; ++i) frac = frac * 10 + (i < fp.size() ? fp[i] - '0' : 0);
    out.ns = std::stoll(ip) * 1000000000LL + frac;
    out.text = s;
    return true;
}

struct Frame {
    Stamp t;
    std::string file;
};
struct Pose {
    Stamp t;
    double tx, ty, tz, qx, qy, qz, qw;
};

bool read_lines(const std::string& path, std::vector<std::vector<std::string>>& rows) {
    std::ifstream f(path);
    if (!f) return false;
    std::string line;
    while (std::getline(f, line)) {
        const size_t h = line.find('#');
        if (h != std::string::npos) line.resize(h);
        std::istringstream ss(line);
        std::vector<std::string> tok;
        std::string w;
        while (ss >> w) tok.push_back(w);
        if (!tok.empty()) rows.push_back(tok);
    }
    return true;
}

// Eigen::Quaterniond::toRotationMatrix (evaluate.cc:190-195, 215-219): the unnormalised formula.
void quat_to_rot(double x, double y, double z, double w, double R[9]) {
    const double tx = 2 * x, ty = 2 * y, tz = 2 * z;
    const double twx = tx * w, twy = ty * w, twz = tz * w;
    const double txx = tx * x, txy = ty * x, txz = tz * x;
    const double tyy = ty * y, tyz = tz * y, tzz = tz * z;
    const double r[9] = {1 - (tyy + tzz), txy - twz, txz + twy, txy + twz, 1 - (txx + tzz),
                         tyz - twx, txz - twy, tyz + twx, 1 - (txx + tyy)};
    std::memcpy(R, r, sizeof r);
}

struct Keyframe {
    int ref;                 // index into the frame list
    int ref_pose;            // index into the pose list
    std::vector<int> src, src_pose;
};

// processImg's lists and counters (evaluate.cc:72-77, 100, 137-239).
struct Replay {
    int agg, interval;
    std::deque<int> images, poses;   // front = newest
    size_t last_size;
    const std::vector<Frame>& F;
    const std::vector<Pose>& P;
    int warnings = 0;
    Replay(int a, int iv, const std::vector<Frame>& f, const std::vector<Pose>& p)
        : agg(a), interval(iv), last_size((size_t)a * iv), F(f), P(p) {}

    bool process(Keyframe& kf) {
        if (images.size() <= last_size) return false;
        if (poses.empty() || P[poses.front()].t.ns < F[images.front()].t.ns) return false;
        size_t ip = 0;
        while (ip < poses.size() && P[poses[ip]].t.ns != F[images.front()].t.ns) ++ip;
        if (ip == poses.size()) {   // "can not find pose for the current Img"
            ++warnings;
            return false;
        }
        // the reference steps past the end of the pose list here (undefined behaviour); stop
        if (ip + (size_t)agg * interval >= poses.size()) {
            ++warnings;
            return false;
        }
        kf.ref = images.front();
        kf.ref_pose = poses[ip];
        kf.src.clear();
        kf.src_pose.clear();
        for (int i = 1; i <= agg; ++i) {
            kf.src.push_back(images[(size_t)i * interval]);
            kf.src_pose.push_back(poses[ip + (size_t)i * interval]);
        }
        ++last_size;
        images.pop_back();
        poses.pop_back();
        return true;
    }
};

std::vector<Keyframe> schedule(const std::vector<Frame>& F, const std::vector<Pose>& P, int agg, int interval,
                               int& warnings) {
    std::vector<int> fo(F.size()), po(P.size());
    for (size_t i = 0; i < F.size(); ++i) fo[i] = (int)i;
    for (size_t i = 0; i < P.size(); ++i) po[i] = (int)i;
    std::stable_sort(fo.begin(), fo.end(), [&](int a, int b) { return F[a].t.ns < F[b].t.ns; });
    std::stable_sort(po.begin(), po.end(), [&](int a, int b) { return P[a].t.ns < P[b].t.ns; });
    Replay r(agg, interval, F, P);
    std::vector<Keyframe> out;
    Keyframe kf;
    size_t pi = 0;
    for (int f : fo) {
        while (pi < po.size() && P[po[pi]].t.ns <= F[f].t.ns) r.poses.push_front(po[pi++]);
        r.images.push_front(f);
        while (r.process(kf)) out.push_back(kf);
    }
    while (pi < po.size()) r.poses.push_front(po[pi++]);
    while (r.process(kf)) out.push_back(kf);
    warnings = r.warnings;
    return out;
}

std::string json_str(const std::string& s) {
    std::string o = "\"";
    for (char c : s) {
        if (c == '"' || c == '\\') o += '\\';
        o += c;
    }
    return o + "\"";
}

struct Args {
    std::string images, poses, root, out = ".", format = "pfm";
    int planes = 64, paths = 4, downsample = 0, agg = 3, interval = 6, out_case = 0, device = 0;
    int precision = PM_PREC_FP32, cost_mode = PM_COST_REFERENCE, sampler = PM_SAMPLER_EXACT, color = 0, dry = 0;
    int limit = -1;
    double fx = 481.2017, fy = -480.0002, cx = 319.5, cy = 239.5;   // ICL-NUIM (evaluate.cc:36-39)
    double min_depth = 0.2, max_depth = 20.0, associate = -1.0;     // evaluate.cc:27-28
};

void usage() {
    std::fprintf(stderr,
                 "usage: pm_sequence --images LIST --poses LIST [--root DIR] [--out DIR]\n"
                 "  [--case N (0 raw-cost argmin, 1 SGM argmin, 2 filtered depth, >=3 fused; default 0)]\n"
                 "  [--planes 64] [--paths 4|8] [--fx F --fy F --cx F --cy F] [--downsample 0]\n"
                 "  [--agg 3] [--interval 6] [--min-depth 0.2] [--max-depth 20] [--format pfm|npy]\n"
                 "  [--color] [--precision fp32|fp16] [--sampler exact|texture (fp16)|texture_f32]\n"
                 "  [--cost reference|corrected] [--associate SECONDS]\n"
                 "  [--limit N] [--device 0] [--dry-run]\n");
}

bool parse_args(int argc, char** argv, Args& a) {
    for (int i = 1; i < argc; ++i) {
        const std::string k = argv[i];
        auto val = [&](void) -> const char* { return i + 1 < argc ? argv[++i] : nullptr; };
        const char* v = nullptr;
        if (k == "--dry-run") { a.dry = 1; continue; }
        if (k == "--color") { a.color = 1; continue; }
        if (!(v = val())) return false;
        if (k == "--images") a.images = v;
        else if (k == "--poses") a.poses = v;
        else if (k == "--root") a.root = v;
        else if (k == "--out") a.out = v;
        else if (k == "--format") a.format = v;
        else if (k == "--case") a.out_case = std::atoi(v);
        else if (k == "--planes") a.planes = std::atoi(v);
        else if (k == "--paths") a.paths = std::atoi(v);
        else if (k == "--downsample") a.downsample = std::atoi(v);
        else if (k == "--agg") a.agg = std::atoi(v);
        else if (k == "--interval") a.interval = std::atoi(v);
        else if (k == "--device") a.device = std::atoi(v);
        else if (k == "--limit") a.limit = std::atoi(v);
        else if (k == "--fx") a.fx = std::atof(v);
        else if (k == "--fy") a.fy = std::atof(v);
        else if (k == "--cx") a.cx = std::atof(v);
        else if (k == "--cy") a.cy = std::atof(v);
        else if (k == "--min-depth") a.min_depth = std::atof(v);
        else if (k == "--max-depth") a.max_depth = std::atof(v);
        else if (k == "--associate") a.associate = std::atof(v);
        else if (k == "--precision") a.precision = std::string(v) == "fp16" ? PM_PREC_FP16 : PM_PREC_FP32;
        else if (k == "--cost") a.cost_mode = std::string(v) == "corrected" ? PM_COST_CORRECTED : PM_COST_REFERENCE;
        else if (k == "--sampler") {
            const std::string m = v;
            if (m == "exact") a.sampler = PM_SAMPLER_EXACT;
            else if (m == "texture") a.sampler = PM_SAMPLER_TEXTURE;
            else if (m == "texture_f32") a.sampler = PM_SAMPLER_TEXTURE_F32;
            else return false;
        }
        else return false;
    }
    return !a.images.empty() && !a.poses.empty() && a.agg > 0 && a.interval > 0 && a.downsample >= 0 &&
           (a.format == "pfm" || a.format == "npy");
}

#define CK_CUDA(x)                                                                              \
    do {                                                                                        \
        cudaError_t e_ = (x);                                                                   \
        if (e_ != cudaSuccess) {                                                                \
            std::fprintf(stderr, "pm_sequence: %s failed: %s\n", #x, cudaGetErrorString(e_));   \
            return 3;                                                                           \
        }                                                                                       \
    } while (0)
#define CK_PM(h, x)                                                                                       \
    do {                                                                                                  \
        pm_status s_ = (x);                                                                               \
        if (s_ != PM_OK) {                                                                                \
            std::fprintf(stderr, "pm_sequence: %s failed: %s %s\n", #x, pm_status_string(s_),             \
                         (h) ? pm_last_error(h) : "");                                                    \
            return 3;                                                                                     \
        }                                                                                                 \
    } while (0)

// A frame in device memory: the file's size (fw, fh), ping-pong buffers for the pyramid steps,
// and the level the mapper sees (data, W x H).
struct DevFrame {
    uint8_t* buf[2] = {nullptr, nullptr};
    int fw = 0, fh = 0, W = 0, H = 0;
    uint8_t* data = nullptr;
};

}  // namespace

int main(int argc, char** argv) {
    Args a;
    if (!parse_args(argc, argv, a)) {
        usage();
        return 2;
    }
    std::vector<std::vector<std::string>> rows;
    std::vector<Frame> F;
    std::vector<Pose> P;
    if (!read_lines(a.images, rows)) { std::fprintf(stderr, "pm_sequence: cannot read %s\n", a.images.c_str()); return 2; }
    for (auto& r : rows) {
        Frame f;
        if (r.size() < 2 || !parse_stamp(r[0], f.t)) { std::fprintf(stderr, "pm_sequence: bad image line\n"); return 2; }
        f.file = r[1];
        F.push_back(f);
    }
    rows.clear();
    if (!read_lines(a.poses, rows)) { std::fprintf(stderr, "pm_sequence: cannot read %s\n", a.poses.c_str()); return 2; }
    for (auto& r : rows) {
        Pose p;
        if (r.size() < 8 || !parse_stamp(r[0], p.t)) { std::fprintf(stderr, "pm_sequence: bad pose line\n"); return 2; }
        double* v[7] = {&p.tx, &p.ty, &p.tz, &p.qx, &p.qy, &p.qz, &p.qw};
        for (int i = 0; i < 7; ++i) {
            char* end = nullptr;
            *v[i] = std::strtod(r[1 + i].c_str(), &end);
            if (end == r[1 + i].c_str() || *end != '\0' || !std::isfinite(*v[i])) {
                std::fprintf(stderr, "pm_sequence: bad pose value '%s'\n", r[1 + i].c_str());
                return 2;
            }
        }
        P.push_back(p);
    }
    if (a.associate >= 0.0) {   // restamp: each image gets its nearest pose within the tolerance
        std::vector<Pose> Q;
        const long long tol = (long long)std::llround(a.associate * 1e9);
        for (const Frame& f : F) {
            int best = -1;
            long long bd = 0;
            for (size_t i = 0; i < P.size(); ++i) {
                const long long d = std::llabs(P[i].t.ns - f.t.ns);
                if (d <= tol && (best < 0 || d < bd)) { best = (int)i; bd = d; }
            }
            if (best >= 0) {
                Pose q = P[best];
                q.t = f.t;
                Q.push_back(q);
            }
        }
        P.swap(Q);
    }
    int warnings = 0;
    std::vector<Keyframe> kfs = schedule(F, P, a.agg, a.interval, warnings);
    if (a.limit >= 0 && (size_t)a.limit < kfs.size()) kfs.resize((size_t)a.limit);
    if (a.dry) {
        for (const Keyframe& k : kfs) {
            std::printf("{\"ref\": %s, \"ref_file\": %s, \"ref_pose\": %s, \"sources\": [", json_str(F[k.ref].t.text).c_str(),
                        json_str(F[k.ref].file).c_str(), json_str(P[k.ref_pose].t.text).c_str());
            for (size_t i = 0; i < k.src.size(); ++i)
                std::printf("%s[%s, %s]", i ? ", " : "", json_str(F[k.src[i]].t.text).c_str(),
                            json_str(P[k.src_pose[i]].t.text).c_str());
            std::printf("]}\n");
        }
        std::printf("{\"keyframes\": %zu, \"warnings\": %d}\n", kfs.size(), warnings);
        return 0;
    }
    if (kfs.empty()) {
        std::printf("{\"keyframes\": 0, \"warnings\": %d}\n", warnings);
        return 0;
    }

    // intrinsics of the pyramid level (evaluate.cc:330-335) and initIntrinsic (:337-346)
    double fx = a.fx, fy = a.fy, cx = a.cx, cy = a.cy;
    for (int i = 0; i < a.downsample; ++i) {
        fx /= 2;
        fy /= 2;
        cx = (cx + 0.5) / 2.0 - 0.5;
        cy = (cy + 0.5) / 2.0 - 0.5;
    }
    const double K[9] = {fx, 0, cx, 0, fy, cy, 0, 0, 1};
    const float bf = (float)(0.02 * fx);
    const float dep_sample = 1.0f / (0.15 * 160.0);

    CK_CUDA(cudaSetDevice(a.device));
    cudaStream_t stream;
    CK_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    const std::string root = a.root.empty() ? "" : a.root + "/";
    std::vector<uint8_t> host;
    // uploads a frame and halves it `downsample` times; slot 0 = reference, 1.. = sources
    std::vector<DevFrame> slots((size_t)a.agg + 1);
    auto load = [&](int fi, DevFrame& df) -> int {
        int W = 0, H = 0;
        const std::string path = root + F[fi].file;
        if (pm_read_image_u8(path.c_str(), &W, &H, nullptr, 0) != PM_OK) {
            std::fprintf(stderr, "pm_sequence: cannot read image %s\n", path.c_str());
            return 2;
        }
        host.resize((size_t)W * H);
        if (pm_read_image_u8(path.c_str(), &W, &H, host.data(), host.size()) != PM_OK) return 2;
        if (df.fw != W || df.fh != H || !df.buf[0]) {
            cudaFree(df.buf[0]);
            cudaFree(df.buf[1]);
            CK_CUDA(cudaMalloc(&df.buf[0], (size_t)W * H));
            CK_CUDA(cudaMalloc(&df.buf[1], (size_t)W * H));
            df.fw = W;
            df.fh = H;
        }
        CK_CUDA(cudaMemcpyAsync(df.buf[0], host.data(), (size_t)W * H, cudaMemcpyHostToDevice, stream));
        int cur = 0, w = W, h = H;
        for (int l = 0; l < a.downsample; ++l) {
            if (w < 2 || h < 2) { std::fprintf(stderr, "pm_sequence: image too small to downsample\n"); return 2; }
            CK_PM((pm_mapper*)nullptr,
                  pm_pyr_down_u8(w, h, df.buf[cur], (size_t)w, df.buf[cur ^ 1], (size_t)(w / 2), stream));
            cur ^= 1;
            w /= 2;
            h /= 2;
        }
        df.data = df.buf[cur];
        df.W = w;
        df.H = h;
        CK_CUDA(cudaStreamSynchronize(stream));   // `host` is reused by the next load
        return 0;
    };

    pm_mapper* h = nullptr;
    int W = 0, H = 0;
    float *d_depth = nullptr, *d_up[2] = {nullptr, nullptr}, *d_mask = nullptr;
    uint8_t* d_bgr = nullptr;
    unsigned* d_scratch = nullptr;
    std::vector<float> h_depth;
    std::vector<uint8_t> h_bgr;
    double sum_ms = 0.0;
    std::vector<double> times;
    int rc;
    for (size_t n = 0; n < kfs.size(); ++n) {
        const Keyframe& k = kfs[n];
        double Rl[9], Tl[3];
        const Pose& pr = P[k.ref_pose];
        quat_to_rot(pr.qx, pr.qy, pr.qz, pr.qw, Rl);
        Tl[0] = pr.tx; Tl[1] = pr.ty; Tl[2] = pr.tz;
        if ((rc = load(k.ref, slots[0])) != 0) return rc;
        for (int i = 0; i < a.agg; ++i)
            if ((rc = load(k.src[i], slots[(size_t)i + 1])) != 0) return rc;
        if (!h) {   // the reference constructs its StereoMapper at start-up, outside the timed interval
            W = slots[0].W;
            H = slots[0].H;
            pm_config c;
            pm_config_default(&c, W, H, a.planes);
            c.num_paths = a.paths;
            c.precision = a.precision;
            c.sampler = a.sampler;   // the library rejects FP16 texels in the FP32 form
            c.cost_mode = a.cost_mode;
            c.fusion_variant = PM_FUSION_CPU_PATH;   // outputFusionCPU (evaluate.cc:260)
            c.device = a.device;
            c.max_sources = a.agg;
            CK_PM(h, pm_create(&c, &h));
            CK_PM(h, pm_set_stream(h, stream));
            CK_PM(h, pm_init_intrinsic(h, K, bf, dep_sample));
            const int up = 1 << a.downsample;
            CK_CUDA(cudaMalloc(&d_depth, 4 * (size_t)W * H));
            for (int b = 0; b < 2; ++b) CK_CUDA(cudaMalloc(&d_up[b], 4 * (size_t)W * H * up * up));
            CK_CUDA(cudaMalloc(&d_mask, 4 * (size_t)W * H * up * up));
            CK_CUDA(cudaMalloc(&d_bgr, 3 * (size_t)W * H * up * up));
            CK_CUDA(cudaMalloc(&d_scratch, 8));
        }
        for (const DevFrame& s : slots)
            if (s.W != W || s.H != H) { std::fprintf(stderr, "pm_sequence: frames differ in size\n"); return 2; }
        const auto t0 = std::chrono::steady_clock::now();   // evaluate.cc:244 (tc_sgm)
        CK_PM(h, pm_init_reference(h, slots[0].data, (size_t)W));
        for (int i = 0; i < a.agg; ++i) {
            double Rr[9], Tr[3];
            const Pose& ps = P[k.src_pose[i]];
            quat_to_rot(ps.qx, ps.qy, ps.qz, ps.qw, Rr);
            Tr[0] = ps.tx; Tr[1] = ps.ty; Tr[2] = ps.tz;
            CK_PM(h, pm_update(h, slots[(size_t)i + 1].data, (size_t)W, Rl, Tl, Rr, Tr));
        }
        if (a.out_case >= 3)
            CK_PM(h, pm_output_fusion(h, d_depth, 0, nullptr, 0, Rl, Tl, (float)fx, (float)fy, (float)cx, (float)cy));
        else
            CK_PM(h, pm_output_case(h, a.out_case, d_depth, 0));
        // depthUp per pyramid level (evaluate.cc:262-266)
        const float* cur = d_depth;
        int w = W, hh = H;
        for (int l = 0, b = 0; l < a.downsample; ++l, b ^= 1) {
            CK_PM(h, pm_depth_up2(w, hh, cur, 0, d_up[b], 0, stream));
            cur = d_up[b];
            w *= 2;
            hh *= 2;
        }
        h_depth.resize((size_t)w * hh);
        CK_CUDA(cudaMemcpyAsync(h_depth.data(), cur, 4 * (size_t)w * hh, cudaMemcpyDeviceToHost, stream));
        CK_CUDA(cudaStreamSynchronize(stream));
        const double ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        sum_ms += ms;
        times.push_back(ms);
        const std::string stem = a.out + "/depth_" + F[k.ref].t.text;
        const std::string dpath = stem + "." + a.format;
        if ((a.format == "pfm" ? pm_write_pfm(dpath.c_str(), w, hh, h_depth.data(), 0)
                               : pm_write_npy(dpath.c_str(), w, hh, h_depth.data(), 0)) != PM_OK) {
            std::fprintf(stderr, "pm_sequence: cannot write %s\n", dpath.c_str());
            return 2;
        }
        if (a.color) {   // evaluate.cc:278-307, on a copy: the written depth is unmasked
            CK_CUDA(cudaMemcpyAsync(d_mask, cur, 4 * (size_t)w * hh, cudaMemcpyDeviceToDevice, stream));
            CK_PM(h, pm_depth_range_mask(w, hh, d_mask, 0, (float)a.min_depth, (float)a.max_depth, stream));
            CK_PM(h, pm_colorize_depth(w, hh, d_mask, 0, nullptr, 0, d_bgr, 0, d_scratch, stream));
            h_bgr.resize(3 * (size_t)w * hh);
            CK_CUDA(cudaMemcpyAsync(h_bgr.data(), d_bgr, h_bgr.size(), cudaMemcpyDeviceToHost, stream));
            CK_CUDA(cudaStreamSynchronize(stream));
            const std::string cpath = a.out + "/color_" + F[k.ref].t.text + ".ppm";
            if (pm_write_ppm(cpath.c_str(), w, hh, h_bgr.data(), 0) != PM_OK) {
                std::fprintf(stderr, "pm_sequence: cannot write %s\n", cpath.c_str());
                return 2;
            }
        }
    }
    std::vector<double> sorted = times;
    std::sort(sorted.begin(), sorted.end());
    // the mean is the reference's "AVERAE CAL TIME" (evaluate.cc:268-270); the first keyframe also
    // pays the one-time loading of the library's kernels
    std::printf("{\"keyframes\": %zu, \"warnings\": %d, \"case\": %d, \"width\": %d, \"height\": %d, "
                "\"mean_ms_per_keyframe\": %.3f, \"median_ms_per_keyframe\": %.3f, \"first_ms\": %.3f}\n",
                kfs.size(), warnings, a.out_case, W << a.downsample, H << a.downsample, sum_ms / kfs.size(),
                sorted[sorted.size() / 2], times[0]);
    pm_destroy(h);
    for (DevFrame& s : slots) {
        cudaFree(s.buf[0]);
        cudaFree(s.buf[1]);
    }
    cudaFree(d_depth);
    cudaFree(d_up[0]);
    cudaFree(d_up[1]);
    cudaFree(d_mask);
    cudaFree(d_bgr);
    cudaFree(d_scratch);
    cudaStreamDestroy(stream);
    return 0;
}
