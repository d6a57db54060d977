// ref_unity.cu -- TEST INFRASTRUCTURE.  One translation unit that compiles the reference's own
// CUDA sources (motion_stereo/*.cu from HKUST-Aerial-Robotics/probabilistic_mapping, included
// from where they lie, never copied) with the compatibility header oracle/ref_shim.h, plus a
// small extern "C" harness that drives the reference's launch wrappers on host arrays.  Built
// by oracle/build_ref.py into oracle/_ref/; used only to produce the golden fixtures that pin
// the CPU oracle (tests/golden/make_ref_golden.py).
#include "calc_cost.cu"
#include "sgm.cu"
#include "filter_cost.cu"
#include "depth_fusion.cu"
#include "convert.cu"
#include "parameters.cpp"

#include <vector>

static const int pm_ref_slots_ready = (tex2Dleft.slot = &pm_ref_obj_tex2Dleft,
                                       tex2Dright.slot = &pm_ref_obj_tex2Dright, 0);

namespace {

struct Pitched {
    float* p = nullptr;
    size_t pitch = 0;
    Pitched() { cudaMallocPitch((void**)&p, &pitch, sizeof(float) * WIDTH, HEIGHT); }   // GpuMat
    ~Pitched() { cudaFree(p); }
    void upload(const float* h) {
        cudaMemcpy2D(p, pitch, h, sizeof(float) * WIDTH, sizeof(float) * WIDTH, HEIGHT, cudaMemcpyHostToDevice);
    }
    void download(float* h) const {
        cudaMemcpy2D(h, sizeof(float) * WIDTH, p, pitch, sizeof(float) * WIDTH, HEIGHT, cudaMemcpyDeviceToHost);
    }
};

template <class T> struct Lin {
    T* p = nullptr;
    size_t n;
    explicit Lin(size_t n_) : n(n_) { cudaMalloc((void**)&p, sizeof(T) * n); }
    ~Lin() { cudaFree(p); }
    void up(const T* h) { cudaMemcpy(p, h, sizeof(T) * n, cudaMemcpyHostToDevice); }
    void down(T* h) const { cudaMemcpy(h, p, sizeof(T) * n, cudaMemcpyDeviceToHost); }
};

}  // namespace

extern "C" {

int ref_shape(int* w, int* h, int* d) {
    *w = WIDTH;
    *h = HEIGHT;
    *d = DEP_CNT;
    return 0;
}

// The mutable parameters of parameters.cpp:12-18.
void ref_set_params(float p1, float p2, float tau, float q1, float q2, float vs) {
    pi1 = p1;
    pi2 = p2;
    tau_so = tau;
    sgm_q1 = q1;
    sgm_q2 = q2;
    var_scale = vs;
}

// initReference + S x update (stereo_mapper.cpp:63-91) with float images (already converted
// by the caller, as convertTo(CV_32F) does) and the 12 homography floats per source.
int ref_calc_cost(const float* ref_img, const float* src_imgs, int nsrc, const float* homs, float dep_sample,
                  float* cost_out, float* cnt_out) {
    const size_t V = (size_t)WIDTH * HEIGHT * DEP_CNT;
    Pitched l, r;
    l.upload(ref_img);
    Lin<float> cost(V), cnt(V);
    std::vector<float> init(V, -1.0f);
    cost.up(init.data());                                      // raw_cost.setTo(-1)
    cudaMemset(cnt.p, 0, sizeof(float) * V);                   // measurement_cnt.setTo(0)
    for (int s = 0; s < nsrc; ++s) {
        r.upload(src_imgs + (size_t)s * WIDTH * HEIGHT);
        const float* h = homs + 12 * s;
        ad_calc_cost((unsigned char*)cnt.p, h[0], h[1], h[2], h[3], h[4], h[5], h[6], h[7], h[8], h[9], h[10],
                     h[11], (unsigned char*)l.p, l.pitch, (unsigned char*)r.p, r.pitch,
                     (unsigned char*)cost.p, dep_sample);
    }
    cost.down(cost_out);
    cnt.down(cnt_out);
    return (int)cudaGetLastError();
}

// sgm_cost.setTo(0); sgm2(raw_cost, sgm_cost) (stereo_mapper.cpp:100-102); tex2Dleft bound to
// the reference image as ad_calc_cost leaves it.
int ref_sgm(const float* cost_in, const float* ref_img, float* out) {
    const size_t V = (size_t)WIDTH * HEIGHT * DEP_CNT;
    Pitched l;
    l.upload(ref_img);
    cudaUnbindTexture(tex2Dleft);
    tex2Dleft.addressMode[0] = cudaAddressModeBorder;
    tex2Dleft.addressMode[1] = cudaAddressModeBorder;
    tex2Dleft.filterMode = cudaFilterModeLinear;
    tex2Dleft.normalized = false;
    size_t off = 0;
    cudaChannelFormatDesc desc = cudaCreateChannelDesc<float>();
    cudaBindTexture2D(&off, tex2Dleft, l.p, desc, WIDTH, HEIGHT, l.pitch);
    Lin<float> in(V), o(V);
    in.up(cost_in);
    cudaMemset(o.p, 0, sizeof(float) * V);
    sgm2((unsigned char*)in.p, (unsigned char*)o.p);
    o.down(out);
    return (int)cudaGetLastError();
}

// filter_cost(sgm_cost, dep, dep.step, DEP_SAMPLE) (stereo_mapper.cpp:105-106); depth W*H.
int ref_filter(const float* sgm_in, float dep_sample, float* depth_out) {
    const size_t V = (size_t)WIDTH * HEIGHT * DEP_CNT;
    Lin<float> in(V);
    in.up(sgm_in);
    Pitched dep;
    filter_cost((unsigned char*)in.p, (unsigned char*)dep.p, dep.pitch, dep_sample);
    dep.download(depth_out);
    return (int)cudaGetLastError();
}

// depth_fuse (depth_fusion.cu:229-280) on linear W*H buffers: table zeroed first
// (stereo_mapper.cpp:163); depth: in WTA depth, out fused; pre/cur: alpha, beta, mu, sigma.
int ref_depth_fuse(const float* pose, const float* cam, float* depth, float* pre, float* cur, int* table_out) {
    const size_t N = (size_t)WIDTH * HEIGHT;
    Lin<float> d(N), tab(N);
    d.up(depth);
    cudaMemset(tab.p, 0, sizeof(int) * N);
    Lin<float> p[4] = {Lin<float>(N), Lin<float>(N), Lin<float>(N), Lin<float>(N)};
    Lin<float> c[4] = {Lin<float>(N), Lin<float>(N), Lin<float>(N), Lin<float>(N)};
    for (int k = 0; k < 4; ++k) {
        p[k].up(pre + k * N);
        c[k].up(cur + k * N);
    }
    depth_fuse(cam[0], cam[1], cam[2], cam[3], pose[0], pose[1], pose[2], pose[3], pose[4], pose[5], pose[6],
               pose[7], pose[8], pose[9], pose[10], pose[11], (unsigned char*)d.p, (unsigned char*)tab.p,
               (unsigned char*)p[0].p, (unsigned char*)p[1].p, (unsigned char*)p[2].p, (unsigned char*)p[3].p,
               (unsigned char*)c[0].p, (unsigned char*)c[1].p, (unsigned char*)c[2].p, (unsigned char*)c[3].p);
    d.down(depth);
    for (int k = 0; k < 4; ++k) {
        p[k].down(pre + k * N);
        c[k].down(cur + k * N);
    }
    cudaMemcpy(table_out, tab.p, sizeof(int) * N, cudaMemcpyDeviceToHost);
    return (int)cudaGetLastError();
}

// convert(input, output, flag, pitch) with the pitch in floats, the unit convertData indexes
// with (convert.cu:16-21).
int ref_convert(const float* in_lin, float* out_pitched, int pitch_floats) {
    const size_t N = (size_t)WIDTH * HEIGHT;
    Lin<float> a(N), b((size_t)pitch_floats * HEIGHT);
    a.up(in_lin);
    cudaMemset(b.p, 0, sizeof(float) * pitch_floats * HEIGHT);
    convert((unsigned char*)a.p, (unsigned char*)b.p, true, (size_t)pitch_floats);
    b.down(out_pitched);
    return (int)cudaGetLastError();
}

}  // extern "C"

extern "C" {

// Times the reference's own pipeline on device-resident data: initReference's two memsets,
// nsrc x ad_calc_cost, sgm_cost.setTo(0) + sgm2 and filter_cost (stereo_mapper.cpp:63-109),
// `reps` times; ms_out receives the mean milliseconds per depth map (CUDA events).
int ref_bench(const float* ref_img, const float* src_imgs, int nsrc, const float* homs, float dep_sample, int reps,
              float* ms_out) {
    const size_t V = (size_t)WIDTH * HEIGHT * DEP_CNT;
    Pitched l, dep;
    std::vector<Pitched> r((size_t)nsrc);
    l.upload(ref_img);
    for (int s = 0; s < nsrc; ++s) r[s].upload(src_imgs + (size_t)s * WIDTH * HEIGHT);
    Lin<float> cost(V), cnt(V), sg(V), minus1(V);
    std::vector<float> init(V, -1.0f);
    minus1.up(init.data());
    cudaEvent_t e0, e1;
    cudaEventCreate(&e0);
    cudaEventCreate(&e1);
    for (int it = -1; it < reps; ++it) {   // it = -1: warm-up
        if (it == 0) cudaEventRecord(e0);
        cudaMemcpy(cost.p, minus1.p, sizeof(float) * V, cudaMemcpyDeviceToDevice);   // raw_cost.setTo(-1)
        cudaMemset(cnt.p, 0, sizeof(float) * V);
        for (int s = 0; s < nsrc; ++s) {
            const float* h = homs + 12 * s;
            ad_calc_cost((unsigned char*)cnt.p, h[0], h[1], h[2], h[3], h[4], h[5], h[6], h[7], h[8], h[9], h[10],
                         h[11], (unsigned char*)l.p, l.pitch, (unsigned char*)r[s].p, r[s].pitch,
                         (unsigned char*)cost.p, dep_sample);
        }
        cudaMemset(sg.p, 0, sizeof(float) * V);
        sgm2((unsigned char*)cost.p, (unsigned char*)sg.p);
        filter_cost((unsigned char*)sg.p, (unsigned char*)dep.p, dep.pitch, dep_sample);
    }
    cudaEventRecord(e1);
    cudaEventSynchronize(e1);
    float ms = 0.0f;
    cudaEventElapsedTime(&ms, e0, e1);
    *ms_out = reps > 0 ? ms / reps : 0.0f;
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    return (int)cudaGetLastError();
}

}  // extern "C"
