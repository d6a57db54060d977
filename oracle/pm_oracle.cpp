/*
 * pm_oracle.cpp -- TEST INFRASTRUCTURE, NOT PRODUCT CODE (see pm_oracle.h).
 *
 * CPU restatement of the motion-stereo path of HKUST-Aerial-Robotics/probabilistic_mapping.
 * Each function cites the reference lines it follows.  Written as one template over the
 * scalar type: Scalar=double is the FP64 parity oracle, Scalar=float reproduces the op order
 * of the B200 kernels (explicit fma, reciprocal-then-multiply warps) for bit-exact checks.
 *
 * Deliberate, documented differences from the literal reference:
 *  - neighbour homogeneous coordinates are evaluated from the neighbour pixel itself
 *    (x(q) = r11*qu + r12*qv + r13) instead of incrementally from the centre (x - r12, ...);
 *    the two bugged samples (calc_cost.cu:50-51, 70-71) keep their incremental form.
 *  - a warped sample with NaN coordinates (w == 0 and zero numerator) is rejected; the
 *    reference would fetch the texture at NaN.
 *  - the source bilinear is exact (texture-unit weight quantisation is opt-in).
 *  - the racy atomicCAS z-buffer / hole filling of depth_fusion.cu:53-104 are replaced by a
 *    deterministic rule that is one legal outcome of those races.
 */
#include "pm_oracle.h"

#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace {

const double kFloatEps = 1e-5;   // FLOAT_EPS, parameters.h:6
const float kDepInf = 1000.0f;   // DEP_INF, parameters.h:29

template <typename S> inline S fmaT(S a, S b, S c) { return std::fma(a, b, c); }

template <typename S> struct Plane {
    const S* p;
    int W, H;
    // border addressing of the reference textures (calc_cost.cu:230-231): outside -> 0
    inline S at(int x, int y) const {
        return (x < 0 || y < 0 || x >= W || y >= H) ? S(0) : p[(size_t)y * W + x];
    }
};

template <typename S> std::vector<S> to_scalar(const uint8_t* img, int n, double scale) {
    std::vector<S> out((size_t)n);
    const S sc = (S)scale;
    for (int i = 0; i < n; ++i) out[i] = (S)img[i] * sc;
    return out;
}

// Bilinear fetch with texel centres at integer coordinates: the reference samples
// tex2D(t, u + 0.5f, v + 0.5f) with cudaFilterModeLinear (calc_cost.cu:93,232), which is
// (1-a)(1-b)T[i,j] + a(1-b)T[i+1,j] + (1-a)b T[i,j+1] + ab T[i+1,j+1], i = floor(u), a = u - i.
template <typename S> inline S bilinear(const Plane<S>& im, S u, S v, int quant) {
    S fu = std::floor(u), fv = std::floor(v);
    int i = (int)fu, j = (int)fv;
    S a = u - fu, b = v - fv;
    if (quant) {
        a = std::nearbyint(a * (S)256) / (S)256;
        b = std::nearbyint(b * (S)256) / (S)256;
    }
    S t00 = im.at(i, j), t10 = im.at(i + 1, j), t01 = im.at(i, j + 1), t11 = im.at(i + 1, j + 1);
    S top = fmaT(a, t10 - t00, t00);
    S bot = fmaT(a, t11 - t01, t01);
    return fmaT(b, bot - top, top);
}

template <typename S> struct Hom {
    S r11, r12, r13, r21, r22, r23, r31, r32, r33, t1, t2, t3;
    explicit Hom(const double* h)
        : r11((S)h[0]), r12((S)h[1]), r13((S)h[2]), r21((S)h[3]), r22((S)h[4]), r23((S)h[5]),
          r31((S)h[6]), r32((S)h[7]), r33((S)h[8]), t1((S)h[9]), t2((S)h[10]), t3((S)h[11]) {}
};

// Reciprocal of a warp.  S = double: 1/w.  S = float: the kernels' branch-free reciprocal,
// RN(1/w) for 2^-126 <= |w| <= 2^126, NaN (sample rejected) for zero, subnormal, infinite or NaN
// w, +-0 for larger finite |w| -- outside the first range only for homogeneous coordinates no
// image-sized scene produces.
template <typename S> inline S rcp_warp(S w) { return (S)1 / w; }
template <> inline float rcp_warp<float>(float w) {
    const float a = std::fabs(w);
    if (!(a >= 1.17549435e-38f) || std::isinf(w)) return std::numeric_limits<float>::quiet_NaN();
    if (a > 8.50705917e37f) return std::copysign(0.0f, w);
    return 1.0f / w;
}

// One warped source sample (calc_cost.cu:85-93): w = z + t3*rho, u = (x + t1*rho)/w,
// v = (y + t2*rho)/w, rejected when w < 0 or (u, v) outside [0, W-1] x [0, H-1].
// Returns NaN for a rejected sample so that the 9-term sum carries the rejection.
template <typename S>
inline S warp_fetch(const Plane<S>& src, S x, S y, S z, const Hom<S>& h, S rho, int quant) {
    S w = fmaT(h.t3, rho, z);
    S nx = fmaT(h.t1, rho, x);
    S ny = fmaT(h.t2, rho, y);
    S r = rcp_warp(w);
    S u = nx * r, v = ny * r;
    bool ok = (w >= (S)0) && (u >= (S)0) && (u <= (S)(src.W - 1)) && (v >= (S)0) &&
              (v <= (S)(src.H - 1));
    if (!ok) return std::numeric_limits<S>::quiet_NaN();
    return bilinear(src, u, v, quant);
}

template <typename S> inline void homog(const Hom<S>& h, int qu, int qv, S& x, S& y, S& z) {
    S fu = (S)qu, fv = (S)qv;
    x = fmaT(h.r11, fu, fmaT(h.r12, fv, h.r13));
    y = fmaT(h.r21, fu, fmaT(h.r22, fv, h.r23));
    z = fmaT(h.r31, fu, fmaT(h.r32, fv, h.r33));
}

template <typename S> inline S warp_at(const Plane<S>& src, const Hom<S>& h, int qu, int qv, S rho,
                                       int quant) {
    S x, y, z;
    homog(h, qu, qv, x, y, z);
    return warp_fetch(src, x, y, z, h, rho, quant);
}

// a3 -- calc_cost.cu:11-210 (+ running mean of stereo_mapper.cpp:69-70 initial state).
template <typename S>
void calc_cost(const orc_params* p, const uint8_t* ref8, const uint8_t* srcs8, int nsrc,
               const double* homs, S* cost, S* cnt) {
    const int W = p->W, H = p->H, D = p->D;
    const size_t N = (size_t)W * H;
    std::vector<S> refv = to_scalar<S>(ref8, (int)N, p->intensity_scale);
    Plane<S> ref{refv.data(), W, H};
    std::vector<std::vector<S>> srcv((size_t)nsrc);
    for (int s = 0; s < nsrc; ++s) srcv[s] = to_scalar<S>(srcs8 + N * s, (int)N, p->intensity_scale);
    std::vector<Hom<S>> hs;
    for (int s = 0; s < nsrc; ++s) hs.emplace_back(homs + 12 * s);
    const S rho0 = (S)p->rho0, drho = (S)p->drho;
    const bool refmode = (p->cost_mode == 0);
    const int quant = p->bilinear_quant;

#pragma omp parallel for schedule(dynamic, 1)
    for (int v = 0; v < H; ++v) {
        for (int u = 0; u < W; ++u) {
            // reference-image samples of the 3x3 patch (border mode -> 0 outside)
            const S Rc = ref.at(u, v), Ru = ref.at(u, v - 1), Rd = ref.at(u, v + 1);
            const S Rl = ref.at(u - 1, v), Rr = ref.at(u + 1, v);
            const S Rul = ref.at(u - 1, v - 1), Rdr = ref.at(u + 1, v + 1);
            const S Rld = ref.at(u - 1, v + 1), Rru = ref.at(u + 1, v - 1);
            S* cp = cost + ((size_t)v * W + u) * D;
            S* np = cnt + ((size_t)v * W + u) * D;
            for (int d = 0; d < D; ++d) { cp[d] = (S)-1; np[d] = (S)0; }
            for (int s = 0; s < nsrc; ++s) {
                const Plane<S> src{srcv[s].data(), W, H};
                const Hom<S>& h = hs[s];
                S xc, yc, zc;
                homog(h, u, v, xc, yc, zc);
                // the two bugged neighbours of calc_cost.cu:49-51 and :69-71
                const S xr = xc + h.r11, yr = xc + h.r21, zr = xc + h.r31;
                const S xru = xr - h.r12, yru = xr - h.r22, zru = xr - h.r32;
                for (int d = 0; d < D; ++d) {
                    const S rho = fmaT((S)d, drho, rho0);   // idep = i * DEP_SAMPLE (:81)
                    const S W0 = warp_at(src, h, u, v, rho, quant);
                    const S Wu = warp_at(src, h, u, v - 1, rho, quant);
                    const S Wd = warp_at(src, h, u, v + 1, rho, quant);
                    const S Wl = warp_at(src, h, u - 1, v, rho, quant);
                    const S Wul = warp_at(src, h, u - 1, v - 1, rho, quant);
                    const S Wdr = warp_at(src, h, u + 1, v + 1, rho, quant);
                    const S Wld = warp_at(src, h, u - 1, v + 1, rho, quant);
                    S tmp = (S)0;
                    if (refmode) {
                        const S B4 = warp_fetch(src, xr, yr, zr, h, rho, quant);
                        const S B8 = warp_fetch(src, xru, yru, zru, h, rho, quant);
                        tmp += std::fabs(Rc - W0);    // 0 (:93)
                        tmp += std::fabs(Rd - Wu);    // 1: warps (u,v-1), reads ref (u,v+1) (:106)
                        tmp += std::fabs(Ru - Wd);    // 2: warps (u,v+1), reads ref (u,v-1) (:119)
                        tmp += std::fabs(Rl - Wl);    // 3 (:132)
                        tmp += std::fabs(Rr - B4);    // 4 (:145)
                        tmp += std::fabs(Rul - Wul);  // 5 (:159)
                        tmp += std::fabs(Rdr - Wdr);  // 6 (:172)
                        tmp += std::fabs(Rld - Wld);  // 7 (:185)
                        tmp += std::fabs(Rru - B8);   // 8 (:198)
                    } else {
                        const S Wr = warp_at(src, h, u + 1, v, rho, quant);
                        const S Wru = warp_at(src, h, u + 1, v - 1, rho, quant);
                        tmp += std::fabs(Rc - W0);
                        tmp += std::fabs(Ru - Wu);
                        tmp += std::fabs(Rd - Wd);
                        tmp += std::fabs(Rl - Wl);
                        tmp += std::fabs(Rr - Wr);
                        tmp += std::fabs(Rul - Wul);
                        tmp += std::fabs(Rdr - Wdr);
                        tmp += std::fabs(Rld - Wld);
                        tmp += std::fabs(Rru - Wru);
                    }
                    if (std::isnan(tmp)) continue;   // any rejected sample skips the voxel
                    const S last = cp[d], lcnt = np[d];
                    const S m = tmp / (S)9;
                    if (last < (S)0) {               // first measurement (:200-203)
                        cp[d] = m;
                        np[d] = (S)1;
                    } else {                         // (:205-206); /(cnt+1.0) is exact-rounded
                        cp[d] = fmaT(lcnt, last, m) / (lcnt + (S)1);
                        np[d] = lcnt + (S)1;
                    }
                }
            }
        }
    }
}

// Priority order of the in-place tree reduction `for (i = D>>1; i > 0; i >>= 1)
// if (d < i && d + i < D && c[d+i] < c[d]) c[d] = c[d+i]` (filter_cost.cu:22-30,
// sgm.cu:24-31).  Slot d keeps its element on ties, so the winner among equal values is the
// first one in the concatenation order of the merges; planes never merged into slot 0 drop out.
void tree_order(int D, int compat, std::vector<int>& rank, std::vector<int>& incl) {
    std::vector<std::vector<int>> slot((size_t)D);
    for (int d = 0; d < D; ++d) slot[d] = {d};
    for (int i = D >> 1; i > 0; i >>= 1)
        for (int d = 0; d < i; ++d)
            if (d + i < D) {
                slot[d].insert(slot[d].end(), slot[d + i].begin(), slot[d + i].end());
                slot[d + i].clear();
            }
    rank.assign((size_t)D, 0);
    incl.assign((size_t)D, 0);
    int r = 0;
    for (int e : slot[0]) { rank[e] = r++; incl[e] = 1; }
    if (!compat) {   // exact mode: every plane takes part, never-merged planes rank last
        for (int d = 0; d < D; ++d)
            if (!incl[d]) { rank[d] = r++; incl[d] = 1; }
    }
}

struct Dir { int dx, dy; };
// path order of the accumulation: sgm.cu:119-133 for the first four, then the diagonals
const Dir kDirs[8] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {-1, -1}, {-1, 1}, {1, -1}};

// a4 -- sgm.cu:5-113 (one scanline), host order sgm.cu:115-135.
// sum_order 0 accumulates the paths in the reference's order (L->R, R->L, T->B, B->T, then
// the diagonals) into one buffer.  sum_order 1 is the order of the B200 kernels, which write
// every path into its own volume P_r (paths in the order above) and add them pairwise:
// (P0 + P1) + (P2 + P3) for 4 paths, ((P0 + P1) + (P2 + P3)) + ((P4 + P5) + (P6 + P7)) for 8.
// The two differ only in FP rounding.
template <typename S>
void sgm_paths(const orc_params* p, const uint8_t* ref8, const S* C, const int* group_of, bool assign,
               std::vector<S*>& parts);

template <typename S>
void sgm(const orc_params* p, const uint8_t* ref8, const S* C, S* out) {
    const size_t V = (size_t)p->W * p->H * p->D;
    int group_of[8];
    std::vector<std::vector<S>> bufs;
    std::vector<S*> parts;
    if (p->sum_order == 0) {
        for (int r = 0; r < 8; ++r) group_of[r] = 0;
        parts.push_back(out);
        sgm_paths<S>(p, ref8, C, group_of, false, parts);
        return;
    }
    for (int r = 0; r < 8; ++r) group_of[r] = r;
    for (int r = 0; r < p->num_paths; ++r) {
        bufs.emplace_back(V);
        parts.push_back(bufs.back().data());
    }
    sgm_paths<S>(p, ref8, C, group_of, true, parts);
    const bool eight = p->num_paths == 8;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)V; ++i) {
        const S s4 = (parts[0][i] + parts[1][i]) + (parts[2][i] + parts[3][i]);
        out[i] = eight ? s4 + ((parts[4][i] + parts[5][i]) + (parts[6][i] + parts[7][i])) : s4;
    }
}

// assign: each path writes its own buffer (o = L at a valid pixel) instead of accumulating.
template <typename S>
void sgm_paths(const orc_params* p, const uint8_t* ref8, const S* C, const int* group_of, bool assign,
               std::vector<S*>& parts) {
    const int W = p->W, H = p->H, D = p->D;
    const size_t N = (size_t)W * H;
    std::vector<S> refv = to_scalar<S>(ref8, (int)N, p->intensity_scale);
    std::vector<int> rank, incl;
    tree_order(D, p->tree_compat, rank, incl);
    const S P1b = (S)p->p1, P2b = (S)p->p2, tau = (S)p->tau_so, q1 = (S)p->q1, q2 = (S)p->q2;
    for (S* part : parts) std::fill(part, part + N * D, (S)0);   // sgm_cost.setTo(0) (stereo_mapper.cpp:100)
    auto minincl = [&](const S* v) {
        S m = std::numeric_limits<S>::infinity();
        for (int d = 0; d < D; ++d)
            if (incl[d] && v[d] < m) m = v[d];
        return m;
    };
    for (int r = 0; r < p->num_paths; ++r) {
        const int dx = kDirs[r].dx, dy = kDirs[r].dy;
        S* const acc = parts[group_of[r]];
        // chain starts: pixels whose predecessor (x-dx, y-dy) lies outside the image
        std::vector<std::pair<int, int>> starts;
        for (int y = 0; y < H; ++y)
            for (int x = 0; x < W; ++x) {
                int px = x - dx, py = y - dy;
                if (px < 0 || py < 0 || px >= W || py >= H) starts.push_back({x, y});
            }
#pragma omp parallel for schedule(dynamic, 4)
        for (long ci = 0; ci < (long)starts.size(); ++ci) {
            std::vector<S> L((size_t)D), val((size_t)D);
            int x = starts[ci].first, y = starts[ci].second;
            S mprev = 0;
            for (int k = 0; x >= 0 && y >= 0 && x < W && y < H; ++k, x += dx, y += dy) {
                const S* c = C + ((size_t)y * W + x) * D;
                S* o = acc + ((size_t)y * W + x) * D;
                const bool invalid = minincl(c) < (S)0;   // (:33, :67) COST_INF = 0
                if (k == 0) {
                    for (int d = 0; d < D; ++d) {
                        L[d] = invalid ? (S)0 : c[d];
                        o[d] = invalid ? (S)0 : (assign ? L[d] : o[d] + L[d]);
                    }
                } else {
                    // D1 = |I(x,y) - I(x-dx,y-dy)| (:75); both inside the image here
                    const S D1 = std::fabs(refv[(size_t)y * W + x] - refv[(size_t)(y - dy) * W + (x - dx)]);
                    S P1 = P1b, P2 = P2b;
                    if (D1 < tau) { P1 *= q1; P2 *= q2; }
                    for (int d = 0; d < D; ++d) {
                        const S cd = invalid ? (S)0 : c[d];
                        S v = std::min(L[d], mprev + P2);
                        if (d - 1 >= 0) v = std::min(v, L[d - 1] + P1);
                        if (d + 1 < D) v = std::min(v, L[d + 1] + P1);
                        v = cd + v - mprev;     // (:98)
                        val[d] = v;
                        o[d] = invalid ? (S)0 : (assign ? v : o[d] + v);
                    }
                    L.swap(val);
                }
                mprev = minincl(L.data());
            }
        }
    }
}

// a5 -- filter_cost.cu:3-55 (+ the uniqueness extension after the flatness test).
// cls (optional): the pixel's outcome, 0 depth, 1 non-overlap, 2 border plane, 3 flat, 4 ambiguous
// (the pm_stats winner-take-all classes).
template <typename S>
void filter(const orc_params* p, const S* sgmv, S* depth, int32_t* idx, uint8_t* cls = nullptr) {
    const int W = p->W, H = p->H, D = p->D;
    std::vector<int> rank, incl;
    tree_order(D, p->tree_compat, rank, incl);
    const S vs = (S)p->var_scale, drho = (S)p->drho, rho0 = (S)p->rho0, ratio = (S)p->uniqueness;
    const bool uniq = p->uniqueness > 0 && p->uniqueness < 1;
#pragma omp parallel for schedule(static)
    for (long i = 0; i < (long)W * H; ++i) {
        const S* c = sgmv + (size_t)i * D;
        int best = -1;
        S mn = 0;
        for (int d = 0; d < D; ++d) {
            if (!incl[d]) continue;
            if (best < 0 || c[d] < mn || (c[d] == mn && rank[d] < rank[best])) { best = d; mn = c[d]; }
        }
        idx[i] = best;
        S out;
        uint8_t k = 0;
        if ((double)mn < kFloatEps && (double)mn > -kFloatEps) {
            out = (S)kDepInf;                                   // situation 1 (:37-38)
            k = 1;
        } else if (best == 0 || best == D - 1) {
            out = (S)0;                                         // situation 2 (:39-40)
            k = 2;
        } else if (c[best - 1] + c[best + 1] < (S)2 * mn * vs) {
            out = (S)0;                                         // situation 3 (:41-42)
            k = 3;
        } else {
            bool reject = false;
            if (uniq) {
                S second = std::numeric_limits<S>::infinity();
                for (int d = 0; d < D; ++d)
                    if (incl[d] && (d < best - 1 || d > best + 1) && c[d] < second) second = c[d];
                if (mn > ratio * second) reject = true;
            }
            if (reject) {
                out = (S)0;
                k = 4;
            } else {
                const S pre = c[best - 1], post = c[best + 1];
                const S a = pre - (S)2 * mn + post;            // (:48)
                const S b = -pre + post;                        // (:49)
                const S sub = (S)best - b / ((S)2 * a);         // (:50)
                out = (S)1 / fmaT(sub, drho, rho0);             // (:51) with rho0 = 0 -> sub*DEP_SAMPLE
            }
        }
        depth[i] = out;
        if (cls) cls[i] = k;
    }
}

// depth_fusion.cu:3-6
template <typename S> inline S normpdf(S x, S mu, S sig) {
    // rsqrtf(2.0f*M_PI*sigma_sq): the product is formed in double and rounded to the argument type
    return std::exp(-(x - mu) * (x - mu) / ((S)2 * sig)) *
           ((S)1 / std::sqrt((S)(2.0 * M_PI * (double)sig)));
}

// a6-a10 -- depth_fusion.cu:8-225 with the deterministic z-buffer / fill rule.
// counts (optional, 13 words, the pm_stats fusion classes): transform empty, outlier, behind,
// outside, moved; prediction none, copied, filled; update empty, init, no measurement, output,
// hidden.
template <typename S>
void fuse_gpu(int W, int H, const float pose[12], const float cam[4], S* depth, S* pa, S* pb,
              S* pm, S* ps, S* ca, S* cb, S* cm, S* cs, int32_t* table_out, uint32_t* counts = nullptr) {
    const size_t N = (size_t)W * H;
    uint32_t cnt[13] = {};
    const S r11 = pose[0], r12 = pose[1], r13 = pose[2], r21 = pose[3], r22 = pose[4],
            r23 = pose[5], r31 = pose[6], r32 = pose[7], r33 = pose[8], t1 = pose[9],
            t2 = pose[10], t3 = pose[11];
    const S fx = cam[0], fy = cam[1], cx = cam[2], cy = cam[3];
    // transformMap (:8-78): best (depth, index) per target cell
    std::vector<S> bestd(N, std::numeric_limits<S>::infinity());
    std::vector<int32_t> table(N, 0);
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const int index = y * W + x;
            const S a = pa[index];
            if ((double)a < kFloatEps) { ++cnt[0]; continue; }     // (:26)
            const S b = pb[index];
            if ((double)(a / (a + b)) < 0.4) { ++cnt[1]; continue; }   // (:30)
            const S dep = pm[index];
            const S px = ((S)x - cx) / fx * dep;                     // (:34)
            const S py = ((S)y - cy) / fy * dep;
            const S pz = dep;
            // r11*px+r12*py+r13*pz + t1 (:37-39) with the multiply-add contraction the reference's
            // nvcc build performs (matched against its outputs, tests/golden/)
            const S px2 = fmaT(r13, pz, fmaT(r12, py, r11 * px)) + t1;
            const S py2 = fmaT(r23, pz, fmaT(r22, py, r21 * px)) + t2;
            const S pz2 = fmaT(r33, pz, fmaT(r32, py, r31 * px)) + t3;
            if ((double)pz2 < kFloatEps) { ++cnt[2]; continue; }  // (:40)
            const int x2 = (int)((double)fmaT(px2 / pz2, fx, cx) + 0.5);   // (:43), truncation
            const int y2 = (int)((double)fmaT(py2 / pz2, fy, cy) + 0.5);
            if (x2 < 0 || x2 >= W || y2 < 0 || y2 >= H) { ++cnt[3]; continue; }
            ++cnt[4];
            pm[index] = pz2;                                         // (:48)
            ps[index] = (S)((double)ps[index] + (double)pz2 * 0.05); // (:49)
            if (index == 0) continue;   // table value 0 means empty: pixel 0 never propagates
            const int cell = y2 * W + x2;
            if (table[cell] == 0 || pz2 < bestd[cell] || (pz2 == bestd[cell] && index < table[cell])) {
                table[cell] = index;
                bestd[cell] = pz2;
            }
        }
    // hole_filling (:80-105): empty cells take the last occupied interior neighbour in raster
    // order -- the writer whose own 3x3 loop (:96-103) reaches the cell first, which is the
    // outcome when the writers run in lockstep
    std::vector<int32_t> filled(table);
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const int e = y * W + x;
            if (table[e] != 0) continue;
            for (int i = 1; i >= -1 && filled[e] == 0; --i)
                for (int j = 1; j >= -1; --j) {
                    const int ny = y + i, nx = x + j;
                    if (nx <= 0 || nx >= W - 1 || ny <= 0 || ny >= H - 1) continue;
                    const int t = table[ny * W + nx];
                    if (t != 0) { filled[e] = t; break; }
                }
        }
    if (table_out) std::memcpy(table_out, filled.data(), N * sizeof(int32_t));
    // depth_predict (:107-137)
    for (size_t e = 0; e < N; ++e) {
        const int t = filled[e];
        ++cnt[t == 0 ? 5 : 6];
        if (t != 0 && table[e] == 0) ++cnt[7];
        if (t == 0) {
            ca[e] = (S)-1.0;
        } else {
            ca[e] = pa[t]; cb[e] = pb[t]; cm[e] = pm[t]; cs[e] = ps[t];
        }
    }
    // depthUpdate (:139-225)
    for (size_t e = 0; e < N; ++e) {
        const S d = depth[e];
        const S unc = (S)((double)(d * d) * 0.01);                  // (:151)
        if ((double)ca[e] < kFloatEps) {                            // (:161)
            if ((double)d < kFloatEps) {
                depth[e] = (S)0;
                ++cnt[8];
            } else {
                ca[e] = (S)10; cb[e] = (S)10; cm[e] = d; cs[e] = (S)2500;
                ++cnt[9];
            }
            continue;
        }
        if ((double)d < kFloatEps) {                                // (:176)
            const S a = ca[e], b = cb[e];
            depth[e] = ((double)(a / (a + b)) > 0.6) ? cm[e] : (S)0;
            ++cnt[10];
            continue;
        }
        const S a = ca[e], b = cb[e], miu = cm[e], sq = cs[e];
        const S new_sq = unc * sq / (unc + sq);                               // (:195)
        const S new_miu = fmaT(miu, unc, d * sq) / (unc + sq);                // (:196)
        S c1 = (a / (a + b)) * normpdf(d, miu, unc + sq);                     // (:197)
        S c2 = (b / (a + b)) * (S)1 / (S)50;                                  // (:198)
        const S norm = c1 + c2;
        c1 = c1 / norm;
        c2 = c2 / norm;
        // u*v + x*y contracts to fma(u, v, x*y) and X - u*v to fma(-u, v, X), as in the
        // reference's nvcc build
        const S f = fmaT(c1, (a + (S)1) / (a + b + (S)1), c2 * (a / (a + b + (S)1)));
        const S ee = fmaT(c1, ((a + (S)1) * (a + (S)2)) / ((a + b + (S)1) * (a + b + (S)2)),
                          c2 * (a * (a + (S)1) / ((a + b + (S)1) * (a + b + (S)2))));
        const S mu_p = fmaT(c1, new_miu, c2 * miu);
        const S sig_p = fmaT(-mu_p, mu_p, fmaT(c1, fmaT(new_miu, new_miu, new_sq), c2 * fmaT(miu, miu, sq)));
        const S a_p = (ee - f) / (f - ee / f);
        const S b_p = a_p * ((S)1 - f) / f;
        ca[e] = a_p; cb[e] = b_p; cm[e] = mu_p; cs[e] = sig_p;
        const bool shown = (double)(a / (a + b)) > 0.6;                       // (:219)
        depth[e] = shown ? mu_p : (S)0;
        ++cnt[shown ? 11 : 12];
    }
    if (counts) std::memcpy(counts, cnt, sizeof cnt);
}

}  // namespace

extern "C" {

static void matmul3(const double* A, const double* B, double* C) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) {
            double s = 0;
            for (int k = 0; k < 3; ++k) s += A[3 * i + k] * B[3 * k + j];
            C[3 * i + j] = s;
        }
}
static void matvec3(const double* A, const double* x, double* y) {
    for (int i = 0; i < 3; ++i) {
        double s = 0;
        for (int k = 0; k < 3; ++k) s += A[3 * i + k] * x[k];
        y[i] = s;
    }
}
static void transpose3(const double* A, double* T) {
    for (int i = 0; i < 3; ++i)
        for (int j = 0; j < 3; ++j) T[3 * j + i] = A[3 * i + j];
}

void orc_compose_homography(const double K[9], const double Rl[9], const double Tl[3],
                            const double Rr[9], const double Tr[3], double out[12]) {
    // K = [fx s cx; 0 fy cy; 0 0 1]; closed-form inverse of the upper-triangular K
    const double fx = K[0], s = K[1], cx = K[2], fy = K[4], cy = K[5];
    const double Ki[9] = {1.0 / fx, -s / (fx * fy), (s * cy - cx * fy) / (fx * fy),
                          0.0,      1.0 / fy,       -cy / fy,
                          0.0,      0.0,            1.0};
    double RrT[9], A[9], B[9], H1[9];
    transpose3(Rr, RrT);
    matmul3(K, RrT, A);      // K * R_r^T
    matmul3(A, Rl, B);       // * R_l
    matmul3(B, Ki, H1);      // * K^-1   (stereo_mapper.cpp:79)
    const double dT[3] = {Tl[0] - Tr[0], Tl[1] - Tr[1], Tl[2] - Tr[2]};
    double H2[3];
    matvec3(A, dT, H2);      // K * R_r^T * (T_l - T_r)   (stereo_mapper.cpp:80)
    for (int i = 0; i < 9; ++i) out[i] = H1[i];
    for (int i = 0; i < 3; ++i) out[9 + i] = H2[i];
}

void orc_relative_pose(const double R[9], const double t[3], const double Rprev[9],
                       const double tprev[3], double out[12]) {
    double RT[9], Rpc[9];
    transpose3(R, RT);
    matmul3(RT, Rprev, Rpc);
    const double dt[3] = {tprev[0] - t[0], tprev[1] - t[1], tprev[2] - t[2]};
    double tpc[3];
    matvec3(RT, dt, tpc);
    for (int i = 0; i < 9; ++i) out[i] = Rpc[i];
    for (int i = 0; i < 3; ++i) out[9 + i] = tpc[i];
}

void orc_calc_cost_f64(const orc_params* p, const uint8_t* ref, const uint8_t* srcs, int S,
                       const double* homs, double* cost, double* cnt) {
    calc_cost<double>(p, ref, srcs, S, homs, cost, cnt);
}
void orc_calc_cost_f32(const orc_params* p, const uint8_t* ref, const uint8_t* srcs, int S,
                       const double* homs, float* cost, float* cnt) {
    calc_cost<float>(p, ref, srcs, S, homs, cost, cnt);
}
void orc_sgm_f64(const orc_params* p, const uint8_t* ref, const double* cost, double* out) {
    sgm<double>(p, ref, cost, out);
}
void orc_sgm_f32(const orc_params* p, const uint8_t* ref, const float* cost, float* out) {
    sgm<float>(p, ref, cost, out);
}
void orc_filter_f64(const orc_params* p, const double* s, double* depth, int32_t* idx) {
    filter<double>(p, s, depth, idx);
}
void orc_filter_f32(const orc_params* p, const float* s, float* depth, int32_t* idx) {
    filter<float>(p, s, depth, idx);
}
void orc_filter_classes_f32(const orc_params* p, const float* s, float* depth, int32_t* idx, uint8_t* cls) {
    filter<float>(p, s, depth, idx, cls);
}
void orc_tree_order(int D, int compat, int32_t* rank, int32_t* incl) {
    std::vector<int> r, in;
    tree_order(D, compat, r, in);
    for (int d = 0; d < D; ++d) { rank[d] = r[d]; incl[d] = in[d]; }
}
void orc_fuse_gpu_f64(int W, int H, const float pose[12], const float cam[4], double* depth,
                      double* pa, double* pb, double* pm, double* ps, double* ca, double* cb,
                      double* cm, double* cs, int32_t* table) {
    fuse_gpu<double>(W, H, pose, cam, depth, pa, pb, pm, ps, ca, cb, cm, cs, table);
}
void orc_fuse_gpu_f32(int W, int H, const float pose[12], const float cam[4], float* depth,
                      float* pa, float* pb, float* pm, float* ps, float* ca, float* cb,
                      float* cm, float* cs, int32_t* table) {
    fuse_gpu<float>(W, H, pose, cam, depth, pa, pb, pm, ps, ca, cb, cm, cs, table);
}
void orc_fuse_gpu_counts_f32(int W, int H, const float pose[12], const float cam[4], float* depth,
                             float* pa, float* pb, float* pm, float* ps, float* ca, float* cb,
                             float* cm, float* cs, int32_t* table, uint32_t* counts) {
    fuse_gpu<float>(W, H, pose, cam, depth, pa, pb, pm, ps, ca, cb, cm, cs, table, counts);
}

// a13 -- the CPU fusion variant that evaluate.cc:260 runs (outputFusionCPU, non-first frame):
// masks of stereo_mapper.cpp:743-760, depthFuseCPU (:568-587) = transformMapCPU (:246-330),
// holeFillingCPU (:332-389), depthPreditCPU (:391-432), depthUpdateCPU (:439-566), then the
// re-mask of :773-784.  Sequential, raster order, as in the reference.
// counts (optional): the 13 pm_stats fusion words, as fuse_gpu's, with transformMapCPU's
// inlier threshold 0.5 (:278) and depthUpdateCPU's output test (:552-556).
void orc_fuse_cpu_counts(int W, int H, const double pose[12], const float cam[4], int pre,
                         float* result, float* alpha, float* beta, float* mu, float* sigma,
                         uint32_t* table, uint32_t* counts) {
    const size_t N = (size_t)W * H;
    uint32_t cnt[13] = {};
    const int cur = pre ^ 1;
    float* aP = alpha + N * pre; float* bP = beta + N * pre; float* mP = mu + N * pre; float* sP = sigma + N * pre;
    float* aC = alpha + N * cur; float* bC = beta + N * cur; float* mC = mu + N * cur; float* sC = sigma + N * cur;
    uint32_t* tab = table + N * cur;
    const float fx = cam[0], fy = cam[1], cx = cam[2], cy = cam[3];
    // masks (:743-760)
    std::vector<uint8_t> mask(N, 0);
    for (size_t i = 0; i < N; ++i) {
        if (result[i] > 100) { result[i] = 0.0f; mask[i] = 255; }
        if (result[i] > 10) result[i] = 0.0f;
    }
    // transformMapCPU (:246-330)
    std::memset(tab, 0, N * sizeof(uint32_t));
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const size_t i = (size_t)y * W + x;
            if ((double)aP[i] < kFloatEps) { ++cnt[0]; continue; }
            if ((double)(aP[i] / (aP[i] + bP[i])) < 0.5) { ++cnt[1]; continue; }
            const float depth = mP[i];
            const double p0 = (double)(((float)x - cx) / fx * depth);
            const double p1 = (double)(((float)y - cy) / fy * depth);
            const double p2 = (double)depth;
            double q[3];
            for (int r = 0; r < 3; ++r)
                q[r] = pose[3 * r] * p0 + pose[3 * r + 1] * p1 + pose[3 * r + 2] * p2 + pose[9 + r];
            if (q[2] < kFloatEps) { ++cnt[2]; continue; }
            const int x2 = (int)(q[0] / q[2] * fx + cx + 0.5);
            const int y2 = (int)(q[1] / q[2] * fy + cy + 0.5);
            if (x2 < 0 || x2 >= W || y2 < 0 || y2 >= H) { ++cnt[3]; continue; }
            ++cnt[4];
            mP[i] = (float)q[2];
            sP[i] = (float)((double)sP[i] + q[2] * 0.05);
            uint32_t& cell = tab[(size_t)y2 * W + x2];
            if (cell == 0) {
                cell = ((uint32_t)y << 16) | (uint32_t)x;
            } else {
                const int nx = cell & 0xffff, ny = cell >> 16;
                float& nm = mP[(size_t)ny * W + nx];
                if (nm <= depth) continue;      // compares the occupant's moved depth (:318)
                nm = depth;
                cell = ((uint32_t)y << 16) | (uint32_t)x;
            }
        }
    // holeFillingCPU (:332-389), expand_sz = 3
    const int ex = 3;
    std::vector<uint8_t> vst(N, 0);
    std::vector<uint8_t> occupied(N);
    for (size_t i = 0; i < N; ++i) occupied[i] = tab[i] != 0;
    for (int y = ex; y < H - ex; ++y)
        for (int x = ex; x < W - ex; ++x) {
            const size_t i = (size_t)y * W + x;
            if (vst[i]) continue;
            if (tab[i] == 0) continue;
            for (int a = -ex; a <= ex; ++a)
                for (int b = -ex; b <= ex; ++b) {
                    const size_t k = (size_t)(y + a) * W + (x + b);
                    if (tab[k] == 0 && !vst[k]) { tab[k] = tab[i]; vst[k] = 1; }
                }
        }
    // depthPreditCPU (:391-432)
    for (size_t i = 0; i < N; ++i) {
        ++cnt[tab[i] == 0 ? 5 : 6];
        if (tab[i] != 0 && !occupied[i]) ++cnt[7];
        if (tab[i] == 0) {
            aC[i] = 0.0f;
        } else {
            const size_t t = (size_t)(tab[i] >> 16) * W + (tab[i] & 0xffff);
            aC[i] = aP[t]; bC[i] = bP[t]; mC[i] = mP[t]; sC[i] = sP[t];
        }
    }
    // depthUpdateCPU (:439-566), threshold 0.51 (:572)
    const double thr = 0.51;
    for (size_t i = 0; i < N; ++i) {
        const float d = result[i];
        const float unc = 64;
        if ((double)aC[i] < kFloatEps) {
            if ((double)d < kFloatEps) {
                result[i] = 0; mC[i] = d;
                ++cnt[8];
            } else {
                result[i] = 0; aC[i] = 10.0f; bC[i] = 10.0f; mC[i] = d; sC[i] = 256.0f;
                ++cnt[9];
            }
            continue;
        }
        if ((double)d < kFloatEps) {
            bC[i] = (float)((double)bC[i] + 1.0);
            result[i] = ((double)(aC[i] / (aC[i] + bC[i])) > thr) ? mC[i] : 0.0f;
            ++cnt[10];
            continue;
        }
        const float a = aC[i], b = bC[i], miu = mC[i], sq = sC[i];
        const float new_sq = unc * sq / (unc + sq);
        const float new_miu = (d * sq + miu * unc) / (unc + sq);
        // normpdfCPU (:434-437) multiplies by sqrt(2*pi*sigma^2)
        const float var = unc + sq;
        const float ex_arg = -(d - miu) * (d - miu) / (2.0f * var);
        const float npdf = (float)((double)std::exp(ex_arg) * std::sqrt(2.0f * M_PI * var));
        float c1 = (a / (a + b)) * npdf;
        float c2 = (b / (a + b)) * 1 / 16.0f;
        const float norm = c1 + c2;
        c1 = c1 / norm;
        c2 = c2 / norm;
        const float f = c1 * ((a + 1.0f) / (a + b + 1.0f)) + c2 * (a / (a + b + 1.0f));
        const float e = c1 * (((a + 1.0f) * (a + 2.0f)) / ((a + b + 1.0f) * (a + b + 2.0f))) +
                        c2 * (a * (a + 1.0f) / ((a + b + 1.0f) * (a + b + 2.0f)));
        const float mu_p = c1 * new_miu + c2 * miu;
        const float sig_p = c1 * (new_sq + new_miu * new_miu) + c2 * (sq + miu * miu) - mu_p * mu_p;
        const float a_p = (e - f) / (f - e / f);
        const float b_p = a_p * (1.0f - f) / f;
        aC[i] = a_p; bC[i] = b_p; mC[i] = mu_p; sC[i] = sig_p;
        const bool shown = (double)(a_p / (a_p + b_p)) > thr;
        result[i] = shown ? mu_p : 0.0f;
        ++cnt[shown ? 11 : 12];
    }
    // re-mask (:773-784)
    for (size_t i = 0; i < N; ++i) {
        if (mask[i] > 100) result[i] = 0.0f;
        if ((double)result[i] < 0.1) result[i] = 0.0f;
    }
    if (counts) std::memcpy(counts, cnt, sizeof cnt);
}

void orc_fuse_cpu(int W, int H, const double pose[12], const float cam[4], int pre,
                  float* result, float* alpha, float* beta, float* mu, float* sigma,
                  uint32_t* table) {
    orc_fuse_cpu_counts(W, H, pose, cam, pre, result, alpha, beta, mu, sigma, table, nullptr);
}

void orc_convert(int W, int H, const void* in, void* out, int flag, uint64_t pitch_bytes) {
    // convertData (convert.cu:4-24); the pitch is taken in bytes (the reference passes a
    // byte step but indexes with it in floats, stereo_mapper.cpp:149-152)
    const char* ib = (const char*)in;
    char* ob = (char*)out;
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            if (flag) {   // linear -> pitched
                std::memcpy(ob + y * pitch_bytes + 4 * (size_t)x, ib + 4 * ((size_t)y * W + x), 4);
            } else {
                std::memcpy(ob + 4 * ((size_t)y * W + x), ib + y * pitch_bytes + 4 * (size_t)x, 4);
            }
        }
}

int orc_num_threads(void) {
#ifdef _OPENMP
    return omp_get_max_threads();
#else
    return 1;
#endif
}
void orc_set_num_threads(int n) {
#ifdef _OPENMP
    if (n > 0) omp_set_num_threads(n);
#else
    (void)n;
#endif
}

}  // extern "C"
