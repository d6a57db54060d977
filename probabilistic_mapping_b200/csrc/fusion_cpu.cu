// fusion_cpu.cu -- the reference's CPU fusion variant (outputFusionCPU, stereo_mapper.cpp:625-820,
// with depthFuseCPU :568-587) on the GPU.
//
// The reference runs it sequentially in raster order, and its z-buffer depends on that order:
// the first pixel to land on a cell takes it; a later pixel takes it over only when the
// occupant's moved depth is larger than the newcomer's ORIGINAL depth, and then the occupant's
// mean is overwritten with that original depth (transformMapCPU, :246-330).  Here every pixel is
// transformed in parallel and pushed onto a lock-free list of its target cell; one thread per
// cell then replays its hitters in pixel-index (raster) order with exactly that rule, so the
// result is the sequential one for any thread timing.  Hole filling (:332-389) becomes a gather:
// an empty cell takes the first originally occupied interior pixel, in raster order, whose 7x7
// window covers it -- which is what the sequential fill with its visited flags produces.
// Prediction and the update follow :391-566 with the CPU constants (inlier threshold 0.5 for the
// transform, measurement variance 64, initial variance 256, outlier density 1/16, beta += 1 on a
// missing measurement, output threshold 0.51 after the update, normpdfCPU multiplying by
// sqrt(2 pi sigma^2)), then the masks of :743-760 and :773-784.  The transform runs in double
// precision like the reference's Eigen code; the update in float without contractions.
#include "pm_device.cuh"

namespace pm {
namespace {

constexpr int kExpand = 3;   // expand_sz of holeFillingCPU (:334)

__device__ __forceinline__ uint32_t pack(int x, int y) { return ((uint32_t)y << 16) | (uint32_t)x; }

// masks (:743-760) and transformMapCPU's per-pixel part (:246-312); pushes the pixel onto its
// target cell's list.  Returns the pixel's pm_stats class (transformMapCPU's cnt0..cnt4).
__device__ __forceinline__ int cpu_transform_pixel(const FuseCpuLaunch& a, int x, int y) {
    const int i = y * a.W + x;
    float r = a.result[i];
    uint8_t m = 0;
    if (r > 100.0f) { r = 0.0f; m = 255; }
    if (r > 10.0f) r = 0.0f;
    a.result[i] = r;
    a.mask[i] = m;
    const float al = a.pre[0][i], be = a.pre[1][i];
    if ((double)al < kFloatEps) return kTfEmpty;
    if ((double)__fdiv_rn(al, __fadd_rn(al, be)) < 0.5) return kTfOutlier;
    const float depth = a.pre[2][i];
    const float fx = a.cam[0], fy = a.cam[1], cx = a.cam[2], cy = a.cam[3];
    const double p0 = (double)__fmul_rn(__fdiv_rn(__fsub_rn((float)x, cx), fx), depth);
    const double p1 = (double)__fmul_rn(__fdiv_rn(__fsub_rn((float)y, cy), fy), depth);
    const double p2 = (double)depth;
    double q[3];
    for (int k = 0; k < 3; ++k)
        q[k] = __dadd_rn(__dadd_rn(__dadd_rn(__dmul_rn(a.pose[3 * k], p0), __dmul_rn(a.pose[3 * k + 1], p1)),
                                   __dmul_rn(a.pose[3 * k + 2], p2)),
                         a.pose[9 + k]);
    if (q[2] < kFloatEps) return kTfBehind;
    const int x2 = __double2int_rz(__dadd_rn(__dadd_rn(__dmul_rn(__ddiv_rn(q[0], q[2]), (double)fx), (double)cx), 0.5));
    const int y2 = __double2int_rz(__dadd_rn(__dadd_rn(__dmul_rn(__ddiv_rn(q[1], q[2]), (double)fy), (double)cy), 0.5));
    if (x2 < 0 || x2 >= a.W || y2 < 0 || y2 >= a.H) return kTfOutside;
    a.orig_mu[i] = depth;
    a.pre[2][i] = __double2float_rn(q[2]);
    a.pre[3][i] = __double2float_rn(__dadd_rn((double)a.pre[3][i], __dmul_rn(q[2], 0.05)));
    const int cell = y2 * a.W + x2;
    a.next[i] = atomicExch(a.head + cell, i);
    return kTfMoved;
}

__global__ void __launch_bounds__(256) cpu_transform_kernel(const FuseCpuLaunch a) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    const int cls = x < a.W && y < a.H ? cpu_transform_pixel(a, x, y) : -1;
    if (a.stats) tally_block<kTfClasses>(a.stats + kStatTf, cls);
}

// The z-test of :313-328 replayed per cell in raster order of its hitters.
__global__ void __launch_bounds__(256) cpu_ztest_kernel(const FuseCpuLaunch a) {
    const int cell = blockIdx.x * blockDim.x + threadIdx.x;
    if (cell >= a.W * a.H) return;
    const int first = a.head[cell];
    uint32_t tab = 0;
    if (first >= 0) {
        int occ = -1;
        int last = -1;
        for (;;) {   // next hitter in index order: the smallest index above the last one
            int j = -1;
            for (int k = first; k >= 0 && PM_IN_BOUNDS(k, (long long)a.W * a.H, kSiteCpuList); k = a.next[k])
                if (k > last && (j < 0 || k < j)) j = k;
            if (j < 0) break;
            last = j;
            const uint32_t cur = occ < 0 ? 0u : pack(occ % a.W, occ / a.W);
            if (cur == 0) {           // an empty cell (pixel (0, 0) also reads as empty, :314)
                occ = j;
                continue;
            }
            const float nm = a.pre[2][occ];   // the occupant's moved depth
            if (nm <= a.orig_mu[j]) continue;
            a.pre[2][occ] = a.orig_mu[j];
            occ = j;
        }
        if (occ >= 0) tab = pack(occ % a.W, occ / a.W);
    }
    a.tab0[cell] = tab;
}

__device__ __forceinline__ float normpdf_cpu(float x, float mu, float var) {   // (:434-437)
    const float t = __fsub_rn(x, mu);
    const float arg = __fdiv_rn(__fmul_rn(-t, t), __fmul_rn(2.0f, var));
    return __double2float_rn(__dmul_rn((double)expf(arg), __dsqrt_rn(__dmul_rn(2.0 * M_PI, (double)var))));
}

// holeFillingCPU (gather), depthPreditCPU, depthUpdateCPU and the re-mask of one pixel.  Returns
// its pm_stats words relative to kStatPred: (none 0 / copied 1, filled 2 or -1, 3 + update class).
__device__ __forceinline__ int3 cpu_update_pixel(const FuseCpuLaunch& a, int x, int y) {
    const int i = y * a.W + x;
    uint32_t t = a.tab0[i];
    const bool direct = t != 0;
    if (t == 0) {
        for (int dy = -kExpand; dy <= kExpand && t == 0; ++dy)
            for (int dx = -kExpand; dx <= kExpand; ++dx) {
                const int sx = x + dx, sy = y + dy;
                if (sx < kExpand || sx >= a.W - kExpand || sy < kExpand || sy >= a.H - kExpand) continue;
                if (!PM_IN_BOUNDS((long long)sy * a.W + sx, (long long)a.W * a.H, kSiteCpuGather)) continue;
                const uint32_t v = a.tab0[sy * a.W + sx];
                if (v != 0) { t = v; break; }
            }
    }
    if (a.table) a.table[i] = t;
    // depthPreditCPU (:391-432)
    float ca, cb = a.cur[1][i], cm = a.cur[2][i], cs = a.cur[3][i];
    const int ts = (int)(t >> 16) * a.W + (int)(t & 0xffff);
    if (t == 0 || !PM_IN_BOUNDS(ts, (long long)a.W * a.H, kSiteCpuGather)) {
        ca = 0.0f;
    } else {
        ca = a.pre[0][ts]; cb = a.pre[1][ts]; cm = a.pre[2][ts]; cs = a.pre[3][ts];
    }
    // depthUpdateCPU (:439-566)
    const float d = a.result[i];
    const float unc = 64.0f;
    float res;
    int ucls;
    if ((double)ca < kFloatEps) {
        res = 0.0f;
        if ((double)d < kFloatEps) {
            cm = d;
            ucls = kUpdEmpty;
        } else {
            ca = 10.0f; cb = 10.0f; cm = d; cs = 256.0f;
            ucls = kUpdInit;
        }
    } else if ((double)d < kFloatEps) {
        cb = __double2float_rn(__dadd_rn((double)cb, 1.0));
        res = ((double)__fdiv_rn(ca, __fadd_rn(ca, cb)) > 0.51) ? cm : 0.0f;
        ucls = kUpdNoMeasurement;
    } else {
        const float aa = ca, bb = cb, miu = cm, sq = cs;
        const float us = __fadd_rn(unc, sq);
        const float new_sq = __fdiv_rn(__fmul_rn(unc, sq), us);
        const float new_miu = __fdiv_rn(__fadd_rn(__fmul_rn(d, sq), __fmul_rn(miu, unc)), us);
        const float ab = __fadd_rn(aa, bb);
        float c1 = __fmul_rn(__fdiv_rn(aa, ab), normpdf_cpu(d, miu, us));
        float c2 = __fdiv_rn(__fmul_rn(__fdiv_rn(bb, ab), 1.0f), 16.0f);
        const float norm = __fadd_rn(c1, c2);
        c1 = __fdiv_rn(c1, norm);
        c2 = __fdiv_rn(c2, norm);
        const float a1 = __fadd_rn(aa, 1.0f), a2 = __fadd_rn(aa, 2.0f);
        const float ab1 = __fadd_rn(ab, 1.0f), ab2 = __fadd_rn(ab, 2.0f);
        const float f = __fadd_rn(__fmul_rn(c1, __fdiv_rn(a1, ab1)), __fmul_rn(c2, __fdiv_rn(aa, ab1)));
        const float den = __fmul_rn(ab1, ab2);
        const float e = __fadd_rn(__fmul_rn(c1, __fdiv_rn(__fmul_rn(a1, a2), den)),
                                  __fmul_rn(c2, __fdiv_rn(__fmul_rn(aa, a1), den)));
        const float mu_p = __fadd_rn(__fmul_rn(c1, new_miu), __fmul_rn(c2, miu));
        const float sig_p = __fsub_rn(__fadd_rn(__fmul_rn(c1, __fadd_rn(new_sq, __fmul_rn(new_miu, new_miu))),
                                                __fmul_rn(c2, __fadd_rn(sq, __fmul_rn(miu, miu)))),
                                      __fmul_rn(mu_p, mu_p));
        const float a_p = __fdiv_rn(__fsub_rn(e, f), __fsub_rn(f, __fdiv_rn(e, f)));
        const float b_p = __fdiv_rn(__fmul_rn(a_p, __fsub_rn(1.0f, f)), f);
        ca = a_p; cb = b_p; cm = mu_p; cs = sig_p;
        const bool shown = (double)__fdiv_rn(a_p, __fadd_rn(a_p, b_p)) > 0.51;
        res = shown ? mu_p : 0.0f;
        ucls = shown ? kUpdOutput : kUpdHidden;
    }
    a.cur[0][i] = ca;
    a.cur[1][i] = cb;
    a.cur[2][i] = cm;
    a.cur[3][i] = cs;
    // re-mask (:773-784)
    if (a.mask[i] > 100) res = 0.0f;
    if ((double)res < 0.1) res = 0.0f;
    a.result[i] = res;
    if (a.variance) a.variance[i] = cs;
    return make_int3(t == 0 ? 0 : 1, t != 0 && !direct ? 2 : -1, 3 + ucls);
}

__global__ void __launch_bounds__(256) cpu_update_kernel(const FuseCpuLaunch a) {
    const int x = blockIdx.x * blockDim.x + threadIdx.x, y = blockIdx.y;
    const int3 c = x < a.W && y < a.H ? cpu_update_pixel(a, x, y) : make_int3(-1, -1, -1);
    if (a.stats) tally_block<3 + kUpdClasses>(a.stats + kStatPred, c.x, c.y, c.z);
}

}  // namespace

cudaError_t launch_fuse_cpu_variant(const FuseCpuLaunch& a, cudaStream_t s) {
    const size_t N = (size_t)a.W * a.H;
    if (a.W >= 65536 || a.H >= 65536) return cudaErrorInvalidValue;   // packed (y << 16) | x table
    cudaError_t e = cudaMemsetAsync(a.head, 0xff, sizeof(int) * N, s);
    if (e != cudaSuccess) return e;
    const dim3 grid((a.W + 255) / 256, a.H);
    cpu_transform_kernel<<<grid, 256, 0, s>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    cpu_ztest_kernel<<<(unsigned)((N + 255) / 256), 256, 0, s>>>(a);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    cpu_update_kernel<<<grid, 256, 0, s>>>(a);
    return cudaGetLastError();
}

}  // namespace pm
