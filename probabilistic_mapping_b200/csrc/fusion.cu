// fusion.cu -- Gaussian x uniform Bayesian depth fusion (reference: depth_fusion.cu:3-280).
//
// The reference runs four kernels with a device synchronisation after each (transformMap,
// hole_filling, depth_predict, depthUpdate) and resolves the z-buffer and the hole filling
// with racy atomicCAS loops, so its output depends on thread timing.  Here:
//   * fuse_transform_kernel forward-warps the confident previous state and resolves the
//     z-test with one 64-bit atomicMin on (depth bits << 32 | pixel index): the nearest
//     surface wins and ties go to the smaller index, independent of scheduling;
//   * fuse_update_kernel fuses hole filling (a gather over the 3x3 neighbourhood of the
//     unfilled table: the last occupied interior neighbour in raster order), the state
//     prediction and the Bayesian update, reading each previous-state entry once.
// Both rules are one legal outcome of the reference's races.  The double-precision
// promotions of the reference expressions (0.4, 0.6, 0.05, 0.01 and M_PI literals) are kept.
#include "pm_device.cuh"

namespace pm {
namespace {

constexpr unsigned long long kEmpty = ~0ull;

// The per-step view of a launch: by value (one mapper call) or from device memory (batched form).
struct FuseView {
    const float* pose;
    const float* cam;
    float* pre[4];
    float* cur[4];
    bool first;
};

__device__ __forceinline__ FuseView view(const FuseLaunch& a) {
    FuseView v;
    if (a.flags_dev) {
        const int idx = a.flags_dev[1] & 1;
        v.first = a.flags_dev[0] != 0;
        v.pose = a.params_dev;
        v.cam = a.params_dev + 12;
        for (int k = 0; k < 4; ++k) {
            v.pre[k] = a.state[idx][k];
            v.cur[k] = a.state[idx ^ 1][k];
        }
    } else {
        v.first = false;
        v.pose = a.pose;
        v.cam = a.cam;
        for (int k = 0; k < 4; ++k) {
            v.pre[k] = a.pre[k];
            v.cur[k] = a.cur[k];
        }
    }
    return v;
}

// transformMap of one pixel; returns its pm_stats class (-1: not counted)
__device__ __forceinline__ int transform_pixel(const FuseLaunch& a, const FuseView& v, int x, int y) {
    const int W = a.W, H = a.H;
    const int index = y * W + x;
    if (v.first) {   // first keyframe: both state sets start from zero (stereo_mapper.cpp:138-141)
        for (int k = 0; k < 4; ++k) a.state[0][k][index] = a.state[1][k][index] = 0.0f;
        return -1;
    }
    const float al = v.pre[0][index];
    if ((double)al < kFloatEps) return kTfEmpty;                           // (:26)
    const float be = v.pre[1][index];
    if ((double)__fdiv_rn(al, __fadd_rn(al, be)) < 0.4) return kTfOutlier; // (:30)
    const float dep = v.pre[2][index];
    const float fx = v.cam[0], fy = v.cam[1], cx = v.cam[2], cy = v.cam[3];
    const float px = __fmul_rn(__fdiv_rn(__fsub_rn((float)x, cx), fx), dep);   // (:34)
    const float py = __fmul_rn(__fdiv_rn(__fsub_rn((float)y, cy), fy), dep);
    const float pz = dep;
    const float* p = v.pose;
    // r11*px+r12*py+r13*pz + t1 (:37-39) with the multiply-add contraction of the reference's
    // nvcc build, so the transformed depth and the target pixel agree with it bit for bit
    const float px2 = __fadd_rn(__fmaf_rn(p[2], pz, __fmaf_rn(p[1], py, __fmul_rn(p[0], px))), p[9]);
    const float py2 = __fadd_rn(__fmaf_rn(p[5], pz, __fmaf_rn(p[4], py, __fmul_rn(p[3], px))), p[10]);
    const float pz2 = __fadd_rn(__fmaf_rn(p[8], pz, __fmaf_rn(p[7], py, __fmul_rn(p[6], px))), p[11]);
    if ((double)pz2 < kFloatEps) return kTfBehind;                         // (:40)
    const int x2 = __double2int_rz(__dadd_rn((double)__fmaf_rn(__fdiv_rn(px2, pz2), fx, cx), 0.5));   // (:43)
    const int y2 = __double2int_rz(__dadd_rn((double)__fmaf_rn(__fdiv_rn(py2, pz2), fy, cy), 0.5));
    if (x2 < 0 || x2 >= W || y2 < 0 || y2 >= H) return kTfOutside;
    v.pre[2][index] = pz2;                                                 // (:48)
    v.pre[3][index] = __double2float_rn(__dadd_rn((double)v.pre[3][index], __dmul_rn((double)pz2, 0.05)));
    if (index == 0) return kTfMoved;   // index 0 encodes "empty" in the reference's table
    const unsigned long long key = ((unsigned long long)__float_as_uint(pz2) << 32) | (unsigned)index;
    if (PM_IN_BOUNDS((long long)y2 * W + x2, (long long)W * H, kSiteFuseTransform))
        atomicMin(a.ztable + (size_t)y2 * W + x2, key);
    return kTfMoved;
}

__global__ void __launch_bounds__(256) fuse_transform_kernel(const FuseLaunch a) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const bool in = x < a.W && y < a.H;
    const int cls = in ? transform_pixel(a, view(a), x, y) : -1;
    if (a.stats) tally_block<kTfClasses>(a.stats + kStatTf, cls);
}

__device__ __forceinline__ float normpdf(float x, float mu, float sig) {   // (:3-6)
    const float d = __fsub_rn(x, mu);
    return __fmul_rn(expf(__fdiv_rn(__fmul_rn(-d, d), __fmul_rn(2.0f, sig))),
                     rsqrtf(__double2float_rn(__dmul_rn(2.0 * M_PI, (double)sig))));
}

// Hole filling, depth_predict and depthUpdate of one cell; returns its pm_stats classes
// (prediction: 0 none, 1 copied, 2 copied from hole filling; update: UpdateClass) or -1s.
__device__ __forceinline__ int2 update_pixel(const FuseLaunch& a, const FuseView& v, int x, int y) {
    const int W = a.W, H = a.H;
    const int e = y * W + x;
    if (v.first) {   // first keyframe: the fused map and its variance are zero
        a.depth[e] = 0.0f;
        if (a.variance) a.variance[e] = 0.0f;
        if (a.table) a.table[e] = 0;
        return make_int2(-1, -1);
    }

    // hole filling (:80-105): an empty cell takes the last occupied interior neighbour in
    // raster order, the writer whose own 3x3 loop (:96-103) reaches it first
    const unsigned long long k0 = a.ztable[e];
    int t = k0 == kEmpty ? 0 : (int)(unsigned)(k0 & 0xffffffffu);
    const bool direct = t != 0;
    if (t == 0) {
        for (int i = 1; i >= -1 && t == 0; --i)
            for (int j = 1; j >= -1; --j) {
                const int ny = y + i, nx = x + j;
                if (nx <= 0 || nx >= W - 1 || ny <= 0 || ny >= H - 1) continue;
                if (!PM_IN_BOUNDS((long long)ny * W + nx, (long long)W * H, kSiteFuseGather)) continue;
                const unsigned long long kk = a.ztable[ny * W + nx];
                if (kk != kEmpty) { t = (int)(unsigned)(kk & 0xffffffffu); break; }
            }
    }
    if (a.table) a.table[e] = t;

    // depth_predict (:107-137)
    float ca, cb = 0.0f, cm = 0.0f, cs = 0.0f;
    if (t == 0 || !PM_IN_BOUNDS(t, (long long)W * H, kSiteFuseGather)) {
        ca = -1.0f;
    } else {
        ca = v.pre[0][t]; cb = v.pre[1][t]; cm = v.pre[2][t]; cs = v.pre[3][t];
    }

    // depthUpdate (:139-225)
    const float d = a.depth_in ? a.depth_in[e] : a.depth[e];
    const float unc = __double2float_rn(__dmul_rn((double)__fmul_rn(d, d), 0.01));   // (:151)
    float out_d = d;
    bool write_all = (t != 0);   // predict copied the whole state
    int ucls;
    if ((double)ca < kFloatEps) {                                           // (:161)
        if ((double)d < kFloatEps) {
            out_d = 0.0f;
            ucls = kUpdEmpty;
        } else {
            ca = 10.0f; cb = 10.0f; cm = d; cs = 2500.0f;
            write_all = true;
            ucls = kUpdInit;
        }
    } else if ((double)d < kFloatEps) {                                     // (:176)
        out_d = ((double)__fdiv_rn(ca, __fadd_rn(ca, cb)) > 0.6) ? cm : 0.0f;
        ucls = kUpdNoMeasurement;
    } else {
        const float aa = ca, bb = cb, miu = cm, sq = cs;
        const float us = __fadd_rn(unc, sq);
        const float new_sq = __fdiv_rn(__fmul_rn(unc, sq), us);                           // (:195)
        const float new_miu = __fdiv_rn(__fmaf_rn(miu, unc, __fmul_rn(d, sq)), us);       // (:196)
        const float ab = __fadd_rn(aa, bb);
        float c1 = __fmul_rn(__fdiv_rn(aa, ab), normpdf(d, miu, us));                     // (:197)
        float c2 = __fdiv_rn(__fmul_rn(__fdiv_rn(bb, ab), 1.0f), 50.0f);                  // (:198)
        const float norm = __fadd_rn(c1, c2);
        c1 = __fdiv_rn(c1, norm);
        c2 = __fdiv_rn(c2, norm);
        const float a1 = __fadd_rn(aa, 1.0f), a2 = __fadd_rn(aa, 2.0f);
        const float ab1 = __fadd_rn(ab, 1.0f), ab2 = __fadd_rn(ab, 2.0f);
        // u*v + x*y -> fma(u, v, x*y) and X - u*v -> fma(-u, v, X): the contraction of the
        // reference's nvcc build (:203-208)
        const float f = __fmaf_rn(c1, __fdiv_rn(a1, ab1), __fmul_rn(c2, __fdiv_rn(aa, ab1)));
        const float den = __fmul_rn(ab1, ab2);
        const float ee = __fmaf_rn(c1, __fdiv_rn(__fmul_rn(a1, a2), den),
                                   __fmul_rn(c2, __fdiv_rn(__fmul_rn(aa, a1), den)));
        const float mu_p = __fmaf_rn(c1, new_miu, __fmul_rn(c2, miu));
        const float sig_p = __fmaf_rn(-mu_p, mu_p,
                                      __fmaf_rn(c1, __fmaf_rn(new_miu, new_miu, new_sq),
                                                __fmul_rn(c2, __fmaf_rn(miu, miu, sq))));
        const float a_p = __fdiv_rn(__fsub_rn(ee, f), __fsub_rn(f, __fdiv_rn(ee, f)));
        const float b_p = __fdiv_rn(__fmul_rn(a_p, __fsub_rn(1.0f, f)), f);
        ca = a_p; cb = b_p; cm = mu_p; cs = sig_p;
        write_all = true;
        const bool shown = (double)__fdiv_rn(aa, ab) > 0.6;                  // (:219)
        out_d = shown ? mu_p : 0.0f;
        ucls = shown ? kUpdOutput : kUpdHidden;
    }
    v.cur[0][e] = ca;
    if (write_all) { v.cur[1][e] = cb; v.cur[2][e] = cm; v.cur[3][e] = cs; }
    a.depth[e] = out_d;
    if (a.variance) a.variance[e] = write_all ? cs : v.cur[3][e];
    return make_int2(t == 0 ? 0 : direct ? 1 : 2, ucls);
}

__global__ void __launch_bounds__(256) fuse_update_kernel(const FuseLaunch a) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y;
    const bool in = x < a.W && y < a.H;
    const int2 cls = in ? update_pixel(a, view(a), x, y) : make_int2(-1, -1);
    // prediction words none, copied, filled, then the update classes (kStatUpd = kStatPred + 3)
    if (a.stats)
        tally_block<3 + kUpdClasses>(a.stats + kStatPred, cls.x < 0 ? -1 : cls.x == 0 ? 0 : 1,
                                     cls.x == 2 ? 2 : -1, cls.y < 0 ? -1 : 3 + cls.y);
}

}  // namespace

cudaError_t launch_fuse_gpu(const FuseLaunch& a, cudaStream_t s) {
    const dim3 block(256), grid((a.W + 255) / 256, a.H);
    cudaError_t e = cudaMemsetAsync(a.ztable, 0xff, sizeof(unsigned long long) * (size_t)a.W * a.H, s);
    if (e != cudaSuccess) return e;
    fuse_transform_kernel<<<grid, block, 0, s>>>(a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    fuse_update_kernel<<<grid, block, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace pm
