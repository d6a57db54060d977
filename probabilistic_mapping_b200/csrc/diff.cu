// diff.cu -- the differentiation form: a differentiable depth loss over the motion-stereo path and
// its hand-written adjoint.
//
// Forward:  C = corrected 3x3 absolute-difference cost averaged over the valid sources (the cost
//           kernel of cost.cu, exact bilinear, FP32); 8 SGM paths (sgm.cu:57-108) whose internal
//           states L_r are kept (or recomputed per path in the backward); S = sum_r L_r;
//           rho_hat = sum_d softmax(-S/T)_d rho_d; loss = mean over valid pixels with rho_gt > 0 of
//           |rho_hat - rho_gt|.
// Backward: the soft-argmin Jacobian gives dS; each path is walked in reverse along its scanlines
//           and the adjoint is routed through the minima the forward took (same FP32 operations,
//           so ties resolve identically): to the same plane, the nearer neighbour plane (+P1) or
//           the path minimum (+P2), and minus the path minimum's plane for the subtracted minimum;
//           dC then flows through the absolute differences (their sign), into the source
//           intensities by the bilinear weights and into the 6-DoF pose of every source through
//           the spatial derivative of the bilinear sample and the projection, as the left se(3)
//           perturbation P_s -> exp([omega]) P_s + upsilon (omega first).
// One warp per scanline for the paths (lane l holds planes [l*PPL, (l+1)*PPL)), one thread per
// voxel for the cost adjoint with atomics into the intensity gradient and per-warp reductions of
// the pose gradient in double precision.
#include <cstring>
#include <string>
#include <vector>

#include "pm_device.cuh"
#include "pm_stereo.h"

namespace {

using namespace pm;

constexpr int kDirs8[8][2] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {-1, -1}, {-1, 1}, {1, -1}};

__host__ __device__ inline int nchains(int dx, int dy, int W, int H) {
    return dy == 0 ? H : (dx == 0 ? W : W + H - 1);
}

// start pixel and length of chain c of direction (dx, dy)
__device__ inline void chain_of(int c, int dx, int dy, int W, int H, int& x, int& y, int& n) {
    if (dy == 0) { x = dx > 0 ? 0 : W - 1; y = c; }
    else if (dx == 0) { x = c; y = dy > 0 ? 0 : H - 1; }
    else if (c < W) { x = c; y = dy > 0 ? 0 : H - 1; }
    else { x = dx > 0 ? 0 : W - 1; y = dy > 0 ? (c - W + 1) : (c - W); }
    const int nx = dx > 0 ? W - x : (dx < 0 ? x + 1 : 1 << 30);
    const int ny = dy > 0 ? H - y : (dy < 0 ? y + 1 : 1 << 30);
    n = nx < ny ? nx : ny;
}

__device__ inline float warp_sum(float v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(kFull, v, o);
    return v;
}

// lowest plane index holding the warp-wide minimum m of the lane vectors
template <int PPL> __device__ inline int argmin_plane(const float (&L)[PPL], float m, int lane) {
    int j = PPL;
#pragma unroll
    for (int t = PPL - 1; t >= 0; --t)
        if (L[t] == m) j = t;
    const unsigned b = __ballot_sync(kFull, j < PPL);
    const int src = __ffs(b) - 1;
    return src * PPL + __shfl_sync(kFull, j, src);
}

struct PathArgs {
    const float* C;          // V cost volume
    const uint8_t* invalid;  // N, 1 = pixel invalid (its cost counts as 0)
    const float* ref;        // N reference image (adaptive penalties)
    float* L;                // V path states (written by the forward, read by the backward)
    float* S;                // V sum of the paths (forward, accumulated) or nullptr
    const float* gS;         // V adjoint of S (backward)
    float* gC;               // V adjoint of C (backward, accumulated)
    int W, H, D, dx, dy;
    float p1, p2, tau, q1, q2;
};

__device__ inline void penalty(const PathArgs& a, long p, long pp, float& P1, float& P2) {
    P1 = a.p1;
    P2 = a.p2;
    if (fabsf(__fsub_rn(a.ref[p], a.ref[pp])) < a.tau) {
        P1 = __fmul_rn(P1, a.q1);
        P2 = __fmul_rn(P2, a.q2);
    }
}

// Forward of one path: L(p, d) = C'(p, d) + min(L(p', d), min(L(p', d-1), L(p', d+1)) + P1, m + P2) - m.
template <int PPL>
__global__ void __launch_bounds__(128) path_fwd_kernel(const PathArgs a) {
    const int lane = threadIdx.x & 31;
    const int c = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (c >= nchains(a.dx, a.dy, a.W, a.H)) return;
    int x, y, n;
    chain_of(c, a.dx, a.dy, a.W, a.H, x, y, n);
    const long step = (long)a.dy * a.W + a.dx;
    long p = (long)y * a.W + x;
    float L[PPL];
    float m = 0.0f;
    for (int k = 0; k < n; ++k, p += step) {
        const bool inv = a.invalid[p] != 0;
        float cv[PPL];
        load_planes<PPL>(cv, a.C + (size_t)p * a.D + lane * PPL);
        float Ln[PPL];
        if (k == 0) {
#pragma unroll
            for (int j = 0; j < PPL; ++j) Ln[j] = inv ? 0.0f : cv[j];
        } else {
            float P1, P2;
            penalty(a, p, p - step, P1, P2);
            const float mP2 = __fadd_rn(m, P2);
            float lm = __shfl_up_sync(kFull, L[PPL - 1], 1);
            float lp = __shfl_down_sync(kFull, L[0], 1);
            if (lane == 0) lm = inf_f();
            if (lane == 31) lp = inf_f();
#pragma unroll
            for (int j = 0; j < PPL; ++j) {
                const float left = j == 0 ? lm : L[j - 1];
                const float right = j == PPL - 1 ? lp : L[j + 1];
                const float vv = fminf(fminf(L[j], mP2), __fadd_rn(fminf(left, right), P1));
                Ln[j] = __fsub_rn(__fadd_rn(inv ? 0.0f : cv[j], vv), m);
            }
        }
        float lmin = inf_f();
#pragma unroll
        for (int j = 0; j < PPL; ++j) {
            L[j] = Ln[j];
            lmin = fminf(lmin, Ln[j]);
        }
        m = warp_min_f32(lmin);
        if (a.L) store_planes<PPL>(a.L + (size_t)p * a.D + lane * PPL, L);
        if (a.S) {
            float sv[PPL];
            load_planes<PPL>(sv, a.S + (size_t)p * a.D + lane * PPL);
#pragma unroll
            for (int j = 0; j < PPL; ++j) sv[j] = __fadd_rn(sv[j], L[j]);
            store_planes<PPL>(a.S + (size_t)p * a.D + lane * PPL, sv);
        }
    }
}

// Adjoint of one path, walking each scanline from its end: lambda = gS + routed adjoint;
// gC += lambda at valid pixels; lambda is routed to the predecessor's planes along the forward's
// minima.
template <int PPL>
__global__ void __launch_bounds__(128) path_bwd_kernel(const PathArgs a) {
    const int lane = threadIdx.x & 31;
    const int c = blockIdx.x * 4 + (threadIdx.x >> 5);
    if (c >= nchains(a.dx, a.dy, a.W, a.H)) return;
    int x, y, n;
    chain_of(c, a.dx, a.dy, a.W, a.H, x, y, n);
    const long step = (long)a.dy * a.W + a.dx;
    long p = (long)y * a.W + x + (long)(n - 1) * step;
    float mu[PPL];
#pragma unroll
    for (int j = 0; j < PPL; ++j) mu[j] = 0.0f;
    for (int k = n - 1; k >= 0; --k, p -= step) {
        float lam[PPL], g[PPL];
        load_planes<PPL>(g, a.gS + (size_t)p * a.D + lane * PPL);
#pragma unroll
        for (int j = 0; j < PPL; ++j) lam[j] = __fadd_rn(g[j], mu[j]);
        if (!a.invalid[p]) {
            float gc[PPL];
            load_planes<PPL>(gc, a.gC + (size_t)p * a.D + lane * PPL);
#pragma unroll
            for (int j = 0; j < PPL; ++j) gc[j] = __fadd_rn(gc[j], lam[j]);
            store_planes<PPL>(a.gC + (size_t)p * a.D + lane * PPL, gc);
        }
        if (k == 0) break;
        const long pp = p - step;
        float Lp[PPL];
        load_planes<PPL>(Lp, a.L + (size_t)pp * a.D + lane * PPL);
        float P1, P2;
        penalty(a, p, pp, P1, P2);
        float lmin = inf_f();
#pragma unroll
        for (int j = 0; j < PPL; ++j) lmin = fminf(lmin, Lp[j]);
        const float m = warp_min_f32(lmin);
        const int km = argmin_plane<PPL>(Lp, m, lane);
        const float mP2 = __fadd_rn(m, P2);
        float lm = __shfl_up_sync(kFull, Lp[PPL - 1], 1);
        float lp = __shfl_down_sync(kFull, Lp[0], 1);
        if (lane == 0) lm = inf_f();
        if (lane == 31) lp = inf_f();
        float same[PPL], toL[PPL], toR[PPL];
        float p2 = 0.0f, tot = 0.0f;
#pragma unroll
        for (int j = 0; j < PPL; ++j) {
            const float left = j == 0 ? lm : Lp[j - 1];
            const float right = j == PPL - 1 ? lp : Lp[j + 1];
            const float nb = __fadd_rn(fminf(left, right), P1);
            const float vmin = fminf(fminf(Lp[j], mP2), nb);
            same[j] = toL[j] = toR[j] = 0.0f;
            if (Lp[j] == vmin) same[j] = lam[j];
            else if (nb == vmin) { if (left <= right) toL[j] = lam[j]; else toR[j] = lam[j]; }
            else p2 = __fadd_rn(p2, lam[j]);
            tot = __fadd_rn(tot, lam[j]);
        }
        // contributions crossing lane boundaries: plane 0's "to d-1" goes to the previous lane's
        // last plane, the last plane's "to d+1" to the next lane's first plane
        const float fromR = __shfl_down_sync(kFull, toL[0], 1);        // lane+1's plane 0 -> my last
        const float fromL = __shfl_up_sync(kFull, toR[PPL - 1], 1);    // lane-1's last -> my plane 0
        const float kmadd = __fsub_rn(warp_sum(p2), warp_sum(tot));
#pragma unroll
        for (int j = 0; j < PPL; ++j) {
            float v = same[j];
            if (j + 1 < PPL) v = __fadd_rn(v, toL[j + 1]);
            else if (lane < 31) v = __fadd_rn(v, fromR);
            if (j > 0) v = __fadd_rn(v, toR[j - 1]);
            else if (lane > 0) v = __fadd_rn(v, fromL);
            if (lane * PPL + j == km) v = __fadd_rn(v, kmadd);
            mu[j] = v;
        }
    }
}

// Soft-argmin and the per-pixel loss terms; gS when grad is set (scale = 1 / |valid pixels|).
template <int PPL>
__global__ void __launch_bounds__(128) soft_kernel(const float* __restrict__ S, const float* __restrict__ rho_gt,
                                                   const uint8_t* __restrict__ invalid, int N, int D, float rho0,
                                                   float drho, float T, float* rho_hat, double* sums,
                                                   const double* count, float* gS) {
    const int lane = threadIdx.x & 31;
    const long p = (long)blockIdx.x * 4 + (threadIdx.x >> 5);
    if (p >= N) return;
    float s[PPL];
    load_planes<PPL>(s, S + (size_t)p * D + lane * PPL);
    float lmin = inf_f();
#pragma unroll
    for (int j = 0; j < PPL; ++j) lmin = fminf(lmin, s[j]);
    const float smin = warp_min_f32(lmin);
    float w[PPL], z = 0.0f, r = 0.0f;
#pragma unroll
    for (int j = 0; j < PPL; ++j) {
        w[j] = expf(-(s[j] - smin) / T);
        z += w[j];
        r += w[j] * (rho0 + (float)(lane * PPL + j) * drho);
    }
    z = warp_sum(z);
    r = warp_sum(r);
    const float rh = r / z;
    const bool in = !invalid[p] && rho_gt[p] > 0.0f;
    if (!gS) {
        if (lane == 0) {
            if (rho_hat) rho_hat[p] = in ? rh : 0.0f;
            if (in) {
                atomicAdd(sums, (double)fabsf(rh - rho_gt[p]));
                atomicAdd(sums + 1, 1.0);
            }
        }
        return;
    }
    float g = 0.0f;
    if (in && count[0] > 0.0) {
        const float diff = rh - rho_gt[p];
        g = (diff > 0.0f ? 1.0f : (diff < 0.0f ? -1.0f : 0.0f)) / (float)count[0];
    }
    float o[PPL];
#pragma unroll
    for (int j = 0; j < PPL; ++j)
        o[j] = g * (-1.0f / T) * (w[j] / z) * ((rho0 + (float)(lane * PPL + j) * drho) - rh);
    store_planes<PPL>(gS + (size_t)p * D + lane * PPL, o);
}

struct CostBwdArgs {
    const float* ref;
    const float* srcs;        // S x N
    const float* gC;          // V
    const uint8_t* invalid;
    float hom[kMaxSources][12];
    float fx, fy, cx, cy;
    int W, H, D, S;
    float rho0, drho;
    float* gI;                // S x N
    double* gP;               // S x 6
};

struct Smp {
    bool ok;
    float u, v, w, nx, ny, val, dIdu, dIdv, a, b;
    int i, j;
};

// One warped sample with the cost kernel's operations (homography FMAs, reciprocal, exact bilinear).
__device__ inline Smp warp_sample(const CostBwdArgs& A, int s, int qu, int qv, float rho) {
    const float* h = A.hom[s];
    const float fu = (float)qu, fv = (float)qv;
    const float x = __fmaf_rn(h[0], fu, __fmaf_rn(h[1], fv, h[2]));
    const float y = __fmaf_rn(h[3], fu, __fmaf_rn(h[4], fv, h[5]));
    const float z = __fmaf_rn(h[6], fu, __fmaf_rn(h[7], fv, h[8]));
    Smp r;
    r.w = __fmaf_rn(h[11], rho, z);
    r.nx = __fmaf_rn(h[9], rho, x);
    r.ny = __fmaf_rn(h[10], rho, y);
    const float2 rc = rcp_warp2(make_float2(r.w, r.w));
    r.u = __fmul_rn(r.nx, rc.x);
    r.v = __fmul_rn(r.ny, rc.x);
    r.ok = (r.w >= 0.0f) && (r.u >= 0.0f) && (r.u <= (float)(A.W - 1)) && (r.v >= 0.0f) && (r.v <= (float)(A.H - 1));
    if (!r.ok) return r;
    const float fu0 = floorf(r.u), fv0 = floorf(r.v);
    r.i = (int)fu0;
    r.j = (int)fv0;
    r.a = __fsub_rn(r.u, fu0);
    r.b = __fsub_rn(r.v, fv0);
    const float* img = A.srcs + (size_t)s * A.W * A.H;
    const bool i1 = r.i + 1 < A.W, j1 = r.j + 1 < A.H;
    const float t00 = img[(size_t)r.j * A.W + r.i];
    const float t10 = i1 ? img[(size_t)r.j * A.W + r.i + 1] : 0.0f;
    const float t01 = j1 ? img[(size_t)(r.j + 1) * A.W + r.i] : 0.0f;
    const float t11 = (i1 && j1) ? img[(size_t)(r.j + 1) * A.W + r.i + 1] : 0.0f;
    const float top = __fmaf_rn(r.a, __fsub_rn(t10, t00), t00);
    const float bot = __fmaf_rn(r.a, __fsub_rn(t11, t01), t01);
    r.val = __fmaf_rn(r.b, __fsub_rn(bot, top), top);
    r.dIdu = (1.0f - r.b) * (t10 - t00) + r.b * (t11 - t01);
    r.dIdv = (1.0f - r.a) * (t01 - t00) + r.a * (t11 - t10);
    return r;
}

__device__ inline float ref_px(const CostBwdArgs& A, int x, int y) {
    return (x < 0 || y < 0 || x >= A.W || y >= A.H) ? 0.0f : A.ref[(size_t)y * A.W + x];
}

__constant__ int kPatch[9][2] = {{0, 0}, {0, -1}, {0, 1}, {-1, 0}, {1, 0}, {-1, -1}, {1, 1}, {-1, 1}, {1, -1}};
constexpr int kMaxDiffSources = 4;

__global__ void __launch_bounds__(128) cost_bwd_kernel(const CostBwdArgs A) {
    const long e = (long)blockIdx.x * blockDim.x + threadIdx.x;
    const long V = (long)A.W * A.H * A.D;
    float gp[kMaxDiffSources][6];
#pragma unroll
    for (int s = 0; s < kMaxDiffSources; ++s)
#pragma unroll
        for (int i = 0; i < 6; ++i) gp[s][i] = 0.0f;
    if (e < V) {
        const long pix = e / A.D;
        const int d = (int)(e - pix * A.D);
        const int v = (int)(pix / A.W), u = (int)(pix - (long)v * A.W);
        const float g = A.gC[e];
        if (!A.invalid[pix] && g != 0.0f) {
            const float rho = __fmaf_rn((float)d, A.drho, A.rho0);
            int n = 0;
            for (int s = 0; s < A.S; ++s) {
                bool ok = true;
                for (int k = 0; k < 9 && ok; ++k) ok = warp_sample(A, s, u + kPatch[k][0], v + kPatch[k][1], rho).ok;
                n += ok;
            }
            if (n > 0) {
                for (int s = 0; s < A.S; ++s) {
                    bool ok = true;
                    for (int k = 0; k < 9 && ok; ++k) ok = warp_sample(A, s, u + kPatch[k][0], v + kPatch[k][1], rho).ok;
                    if (!ok) continue;
                    float* gi = A.gI + (size_t)s * A.W * A.H;
                    for (int k = 0; k < 9; ++k) {
                        const int qu = u + kPatch[k][0], qv = v + kPatch[k][1];
                        const Smp q = warp_sample(A, s, qu, qv, rho);
                        const float diff = ref_px(A, qu, qv) - q.val;
                        const float sg = diff > 0.0f ? 1.0f : (diff < 0.0f ? -1.0f : 0.0f);
                        const float c = -sg * g / (9.0f * (float)n);
                        if (c == 0.0f) continue;
                        atomicAdd(gi + (size_t)q.j * A.W + q.i, c * (1.0f - q.a) * (1.0f - q.b));
                        if (q.i + 1 < A.W) atomicAdd(gi + (size_t)q.j * A.W + q.i + 1, c * q.a * (1.0f - q.b));
                        if (q.j + 1 < A.H) atomicAdd(gi + (size_t)(q.j + 1) * A.W + q.i, c * (1.0f - q.a) * q.b);
                        if (q.i + 1 < A.W && q.j + 1 < A.H)
                            atomicAdd(gi + (size_t)(q.j + 1) * A.W + q.i + 1, c * q.a * q.b);
                        // pose: P = K^-1 (nx, ny, w); dP = omega x P + rho upsilon
                        const float Px = (q.nx - A.cx * q.w) / A.fx, Py = (q.ny - A.cy * q.w) / A.fy, Pz = q.w;
                        const float dP[6][3] = {{0.0f, -Pz, Py}, {Pz, 0.0f, -Px}, {-Py, Px, 0.0f},
                                                {rho, 0.0f, 0.0f}, {0.0f, rho, 0.0f}, {0.0f, 0.0f, rho}};
#pragma unroll
                        for (int i = 0; i < 6; ++i) {
                            const float du = (A.fx * dP[i][0] + (A.cx - q.u) * dP[i][2]) / q.w;
                            const float dv = (A.fy * dP[i][1] + (A.cy - q.v) * dP[i][2]) / q.w;
                            gp[s][i] += c * (q.dIdu * du + q.dIdv * dv);
                        }
                    }
                }
            }
        }
    }
    // pose gradient: warp sums, one double atomic per warp and component
    const int lane = threadIdx.x & 31;
    for (int s = 0; s < A.S; ++s)
        for (int i = 0; i < 6; ++i) {
            const float t = warp_sum(gp[s][i]);
            if (lane == 0 && t != 0.0f) atomicAdd(A.gP + 6 * s + i, (double)t);
        }
}

__global__ void to_quad_f_kernel(int W, int H, const float* __restrict__ img, float4* __restrict__ q) {
    const int y = blockIdx.y;
    for (int x = blockIdx.x * blockDim.x + threadIdx.x; x < W; x += gridDim.x * blockDim.x) {
        const float* r0 = img + (size_t)y * W;
        const bool hx = x + 1 < W, hy = y + 1 < H;
        q[(size_t)y * W + x] = make_float4(r0[x], hy ? r0[x + W] : 0.0f, hx ? r0[x + 1] : 0.0f,
                                           (hx && hy) ? r0[x + W + 1] : 0.0f);
    }
}

template <int PPL> cudaError_t launch_path(const PathArgs& a, bool fwd, cudaStream_t s) {
    const int nch = nchains(a.dx, a.dy, a.W, a.H);
    if (fwd) path_fwd_kernel<PPL><<<(nch + 3) / 4, 128, 0, s>>>(a);
    else path_bwd_kernel<PPL><<<(nch + 3) / 4, 128, 0, s>>>(a);
    return cudaGetLastError();
}

cudaError_t launch_path_any(const PathArgs& a, bool fwd, cudaStream_t s) {
    switch (a.D / 32) {
        case 1: return launch_path<1>(a, fwd, s);
        case 2: return launch_path<2>(a, fwd, s);
        case 4: return launch_path<4>(a, fwd, s);
        case 8: return launch_path<8>(a, fwd, s);
        default: return cudaErrorInvalidValue;
    }
}

template <int PPL>
cudaError_t launch_soft(const float* S, const float* rgt, const uint8_t* inv, int N, int D, float rho0, float drho,
                        float T, float* rho_hat, double* sums, const double* count, float* gS, cudaStream_t s) {
    soft_kernel<PPL><<<(N + 3) / 4, 128, 0, s>>>(S, rgt, inv, N, D, rho0, drho, T, rho_hat, sums, count, gS);
    return cudaGetLastError();
}

cudaError_t launch_soft_any(const float* S, const float* rgt, const uint8_t* inv, int N, int D, float rho0,
                            float drho, float T, float* rho_hat, double* sums, const double* count, float* gS,
                            cudaStream_t s) {
    switch (D / 32) {
        case 1: return launch_soft<1>(S, rgt, inv, N, D, rho0, drho, T, rho_hat, sums, count, gS, s);
        case 2: return launch_soft<2>(S, rgt, inv, N, D, rho0, drho, T, rho_hat, sums, count, gS, s);
        case 4: return launch_soft<4>(S, rgt, inv, N, D, rho0, drho, T, rho_hat, sums, count, gS, s);
        case 8: return launch_soft<8>(S, rgt, inv, N, D, rho0, drho, T, rho_hat, sums, count, gS, s);
        default: return cudaErrorInvalidValue;
    }
}

}  // namespace

struct pm_diff {
    pm_diff_config cfg{};
    size_t N = 0, V = 0;
    float4* quads = nullptr;
    float* C = nullptr;
    uint8_t* invalid = nullptr;
    float* S = nullptr;
    float* L = nullptr;       // 8 path volumes (store_paths) or 1
    float* gS = nullptr;
    float* gC = nullptr;
    double* sums = nullptr;   // [loss sum, valid count]
    double* gP = nullptr;     // S x 6
    float* rho_hat = nullptr;
    // inputs of the last forward
    const float* ref = nullptr;
    const float* srcs = nullptr;
    const float* rho_gt = nullptr;
    float hom[kMaxSources][12]{};
    float cam[4]{};
    bool have_forward = false;
    size_t bytes = 0;
    std::string err;
};

namespace {

pm_status dfail(pm_diff* d, pm_status s, const char* msg, cudaError_t e = cudaSuccess) {
    if (d) d->err = std::string(msg) + (e != cudaSuccess ? std::string(": ") + cudaGetErrorString(e) : "");
    return s;
}

#define PD_CK(d, call)                                                      \
    do {                                                                    \
        cudaError_t e_ = (call);                                            \
        if (e_ != cudaSuccess) return dfail((d), PM_ERR_CUDA, #call, e_);   \
    } while (0)

struct DGuard {
    int prev = -1;
    explicit DGuard(int dev) {
        if (cudaGetDevice(&prev) != cudaSuccess) prev = -1;
        if (prev != dev) cudaSetDevice(dev);
    }
    ~DGuard() {
        int cur = -1;
        if (prev >= 0 && cudaGetDevice(&cur) == cudaSuccess && cur != prev) cudaSetDevice(prev);
    }
};

void free_diff(pm_diff* d) {
    cudaFree(d->quads);
    cudaFree(d->C);
    cudaFree(d->invalid);
    cudaFree(d->S);
    cudaFree(d->L);
    cudaFree(d->gS);
    cudaFree(d->gC);
    cudaFree(d->sums);
    cudaFree(d->gP);
}

PathArgs path_args(const pm_diff* d, int r) {
    PathArgs a;
    std::memset(&a, 0, sizeof a);
    const pm_diff_config& c = d->cfg;
    a.C = d->C;
    a.invalid = d->invalid;
    a.ref = d->ref;
    a.W = c.width;
    a.H = c.height;
    a.D = c.num_planes;
    a.dx = kDirs8[r][0];
    a.dy = kDirs8[r][1];
    a.p1 = c.p1; a.p2 = c.p2; a.tau = c.tau_so; a.q1 = c.q1; a.q2 = c.q2;
    return a;
}

}  // namespace

extern "C" {

void pm_diff_config_default(pm_diff_config* c, int width, int height, int num_planes, int num_sources) {
    if (!c) return;
    std::memset(c, 0, sizeof *c);
    c->width = width;
    c->height = height;
    c->num_planes = num_planes;
    c->num_sources = num_sources;
    c->rho0 = 0.1f;
    c->rho_step = num_planes > 1 ? 1.9f / (float)(num_planes - 1) : 1.0f;
    c->temperature = 0.05f;
    c->p1 = 0.003f;
    c->p2 = 0.01f;
    c->tau_so = 3.5f / 255.0f;
    c->q1 = 2.0f;
    c->q2 = 3.0f;
    c->store_paths = 0;
    c->device = 0;
}

pm_status pm_diff_create(const pm_diff_config* c, pm_diff** out) {
    if (!c || !out) return PM_ERR_INVALID_ARGUMENT;
    *out = nullptr;
    if (c->width < 3 || c->height < 3 || c->num_planes < 32 || c->num_planes > kMaxPlanes ||
        (c->num_planes != 32 && c->num_planes != 64 && c->num_planes != 128 && c->num_planes != 256) ||
        c->num_sources < 1 || c->num_sources > kMaxDiffSources || !(c->temperature > 0.0f) || !(c->rho_step > 0.0f))
        return PM_ERR_INVALID_ARGUMENT;
    pm_diff* d = new pm_diff();
    d->cfg = *c;
    d->N = (size_t)c->width * c->height;
    d->V = d->N * c->num_planes;
    DGuard g(c->device);
    const size_t npaths = c->store_paths ? 8 : 1;
    bool ok = true;
    auto alloc = [&](void** p, size_t b) {
        if (!ok) return;
        ok = cudaMalloc(p, b) == cudaSuccess;
        d->bytes += b;
    };
    alloc((void**)&d->quads, 16 * d->N * c->num_sources);
    alloc((void**)&d->C, 4 * d->V);
    alloc((void**)&d->invalid, d->N);
    alloc((void**)&d->S, 4 * d->V);
    alloc((void**)&d->L, 4 * d->V * npaths);
    alloc((void**)&d->gS, 4 * d->V);
    alloc((void**)&d->gC, 4 * d->V);
    alloc((void**)&d->sums, 2 * sizeof(double));
    alloc((void**)&d->gP, 6 * sizeof(double) * c->num_sources);
    if (!ok) {
        cudaGetLastError();
        free_diff(d);
        delete d;
        return PM_ERR_OUT_OF_MEMORY;
    }
    *out = d;
    return PM_OK;
}

void pm_diff_destroy(pm_diff* d) {
    if (!d) return;
    DGuard g(d->cfg.device);
    cudaDeviceSynchronize();
    free_diff(d);
    delete d;
}

pm_status pm_diff_memory(const pm_diff* d, size_t* bytes) {
    if (!d || !bytes) return PM_ERR_INVALID_ARGUMENT;
    *bytes = d->bytes;
    return PM_OK;
}

pm_status pm_diff_forward(pm_diff* d, const float* ref, const float* srcs, const double K[9], const double* R,
                          const double* t, const float* rho_gt, float* rho_hat, double* loss, void* stream) {
    if (!d || !ref || !srcs || !K || !R || !t || !rho_gt || !loss) return PM_ERR_INVALID_ARGUMENT;
    if (!finite_n(K, 9) || K[1] != 0.0 || K[3] != 0.0 || K[6] != 0.0 || K[7] != 0.0 || K[8] != 1.0 || K[0] == 0.0 ||
        K[4] == 0.0)
        return dfail(d, PM_ERR_INVALID_ARGUMENT, "K must be [[fx, 0, cx], [0, fy, cy], [0, 0, 1]]");
    const pm_diff_config& c = d->cfg;
    const int S = c.num_sources, W = c.width, H = c.height, D = c.num_planes;
    if (!finite_n(R, 9 * S) || !finite_n(t, 3 * S)) return dfail(d, PM_ERR_INVALID_ARGUMENT, "poses must be finite");
    DGuard g(c.device);
    cudaStream_t st = (cudaStream_t)stream;
    d->ref = ref;
    d->srcs = srcs;
    d->rho_gt = rho_gt;
    d->rho_hat = rho_hat;
    // H1 = K R K^-1, H2 = K t for each source-from-reference pose
    const double Ki[9] = {1.0 / K[0], 0.0, -K[2] / K[0], 0.0, 1.0 / K[4], -K[5] / K[4], 0.0, 0.0, 1.0};
    for (int s = 0; s < S; ++s) {
        double A[9], B[9];
        matmul3(K, R + 9 * s, A);
        matmul3(A, Ki, B);
        double kt[3];
        matvec3(K, t + 3 * s, kt);
        for (int i = 0; i < 9; ++i) d->hom[s][i] = (float)B[i];
        for (int i = 0; i < 3; ++i) d->hom[s][9 + i] = (float)kt[i];
    }
    d->cam[0] = (float)K[0];
    d->cam[1] = (float)K[4];
    d->cam[2] = (float)K[2];
    d->cam[3] = (float)K[5];
    const dim3 qg((W + 255) / 256, H);
    for (int s = 0; s < S; ++s)
        to_quad_f_kernel<<<qg, 256, 0, st>>>(W, H, srcs + (size_t)s * d->N, d->quads + (size_t)s * d->N);
    PD_CK(d, cudaGetLastError());
    CostLaunch a;
    std::memset(&a, 0, sizeof a);
    a.ref = ref;
    a.srcq = d->quads;
    a.W = W;
    a.H = H;
    a.D = D;
    a.nsrc = S;
    a.rho0 = c.rho0;
    a.drho = c.rho_step;
    a.mode = PM_COST_CORRECTED;
    for (int s = 0; s < S; ++s)
        for (int i = 0; i < 12; ++i) a.hom[s][i] = d->hom[s][i];
    a.cost = d->C;
    a.invalid = d->invalid;
    PD_CK(d, launch_cost(a, st));
    PD_CK(d, cudaMemsetAsync(d->S, 0, 4 * d->V, st));
    for (int r = 0; r < 8; ++r) {
        PathArgs pa = path_args(d, r);
        pa.L = d->L + (c.store_paths ? (size_t)r * d->V : 0);
        pa.S = d->S;
        PD_CK(d, launch_path_any(pa, true, st));
    }
    PD_CK(d, cudaMemsetAsync(d->sums, 0, 2 * sizeof(double), st));
    PD_CK(d, launch_soft_any(d->S, rho_gt, d->invalid, (int)d->N, D, c.rho0, c.rho_step, c.temperature, rho_hat,
                             d->sums, nullptr, nullptr, st));
    double h[2];
    PD_CK(d, cudaMemcpyAsync(h, d->sums, sizeof h, cudaMemcpyDeviceToHost, st));
    PD_CK(d, cudaStreamSynchronize(st));
    *loss = h[1] > 0 ? h[0] / h[1] : 0.0;
    d->have_forward = true;
    return PM_OK;
}

pm_status pm_diff_backward(pm_diff* d, float* grad_srcs, double* grad_pose, void* stream) {
    if (!d || !grad_srcs || !grad_pose) return PM_ERR_INVALID_ARGUMENT;
    if (!d->have_forward) return dfail(d, PM_ERR_BAD_STATE, "backward before forward");
    const pm_diff_config& c = d->cfg;
    const int S = c.num_sources, D = c.num_planes;
    DGuard g(c.device);
    cudaStream_t st = (cudaStream_t)stream;
    PD_CK(d, launch_soft_any(d->S, d->rho_gt, d->invalid, (int)d->N, D, c.rho0, c.rho_step, c.temperature, nullptr,
                             nullptr, d->sums + 1, d->gS, st));
    PD_CK(d, cudaMemsetAsync(d->gC, 0, 4 * d->V, st));
    for (int r = 0; r < 8; ++r) {
        PathArgs pa = path_args(d, r);
        pa.L = d->L + (c.store_paths ? (size_t)r * d->V : 0);
        if (!c.store_paths) PD_CK(d, launch_path_any(pa, true, st));   // recompute this path's states
        pa.S = nullptr;
        pa.gS = d->gS;
        pa.gC = d->gC;
        PD_CK(d, launch_path_any(pa, false, st));
    }
    PD_CK(d, cudaMemsetAsync(grad_srcs, 0, 4 * d->N * S, st));
    PD_CK(d, cudaMemsetAsync(d->gP, 0, 6 * sizeof(double) * S, st));
    CostBwdArgs A;
    std::memset(&A, 0, sizeof A);
    A.ref = d->ref;
    A.srcs = d->srcs;
    A.gC = d->gC;
    A.invalid = d->invalid;
    for (int s = 0; s < S; ++s)
        for (int i = 0; i < 12; ++i) A.hom[s][i] = d->hom[s][i];
    A.fx = d->cam[0];
    A.fy = d->cam[1];
    A.cx = d->cam[2];
    A.cy = d->cam[3];
    A.W = c.width;
    A.H = c.height;
    A.D = D;
    A.S = S;
    A.rho0 = c.rho0;
    A.drho = c.rho_step;
    A.gI = grad_srcs;
    A.gP = d->gP;
    cost_bwd_kernel<<<(unsigned)((d->V + 127) / 128), 128, 0, st>>>(A);
    PD_CK(d, cudaGetLastError());
    PD_CK(d, cudaMemcpyAsync(grad_pose, d->gP, 6 * sizeof(double) * S, cudaMemcpyDeviceToHost, st));
    PD_CK(d, cudaStreamSynchronize(st));
    return PM_OK;
}

const char* pm_diff_last_error(const pm_diff* d) { return d ? d->err.c_str() : "null handle"; }

}  // extern "C"
