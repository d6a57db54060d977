/*
 * pm_oracle_diff.cpp -- TEST INFRASTRUCTURE, NOT PRODUCT CODE (see pm_oracle.h).
 *
 * FP64 transcription of the differentiable form of the motion-stereo path and of its adjoint:
 *   cost      C(p,d) = mean over valid sources s of (1/9) sum over the 3x3 patch of
 *             |R(q) - I_s(pi_s(q, rho_d))|, the corrected patch of calc_cost.cu:11-210 with
 *             the running mean over sources (stereo_mapper.cpp:69-70 start state); a sample is
 *             valid when w >= 0 and it lands inside [0, W-1] x [0, H-1]; a pixel with a plane
 *             that no source measured is invalid (sgm.cu:33,67) and contributes cost 0;
 *   SGM       8 paths of sgm.cu:57-108 (adaptive P1/P2), S(p,d) = sum of the paths' states;
 *   subpixel  soft-argmin over the planes, rho_hat = sum_d softmax(-S/T)_d rho_d;
 *   loss      mean over valid pixels with rho_gt > 0 of |rho_hat - rho_gt|.
 * The adjoint follows the forward's choices exactly: the soft-argmin Jacobian, the SGM minima
 * as subgradients (ties to the same plane, then the nearer neighbour plane, then the P2 term;
 * the minimum over planes to its lowest index), the absolute differences through their sign,
 * and the bilinear samples through their weights (source intensities) and their spatial
 * derivative (pose).  Pose gradients are with respect to a left se(3) perturbation of each
 * source pose, P_s -> exp([omega]) P_s + upsilon with P_s = R_s P_ref + t_s, in the order
 * (omega_x, omega_y, omega_z, upsilon_x, upsilon_y, upsilon_z).
 */
#include <algorithm>
#include <cmath>
#include <cstring>
#include <limits>
#include <vector>

#include "pm_oracle.h"

namespace {

struct Dir {
    int dx, dy;
};
const Dir kDirs8[8] = {{1, 0}, {-1, 0}, {0, 1}, {0, -1}, {1, 1}, {-1, -1}, {-1, 1}, {1, -1}};

struct Model {
    const orc_diff_params* p;
    const double* ref;
    const double* srcs;
    // N*D*S source validity flags ((pixel * D + plane) * S + source) that replace the tests of
    // the warped samples, or nullptr.  A frozen-valid source is evaluated even where one of its
    // samples has moved out of [0, W-1] x [0, H-1]: the zero border keeps the bilinear value
    // continuous, so the loss has no jumps under a small pose change.
    const uint8_t* frozen = nullptr;
    double fx, fy, cx, cy;
    std::vector<double> H;   // S x 12: K R K^-1 row-major, then K t
    int W, H_, D, S;
    size_t N, V;
};

void homographies(const orc_diff_params* p, const double* K, const double* R, const double* t, std::vector<double>& Hs) {
    const double fx = K[0], cx = K[2], fy = K[4], cy = K[5];
    const double Ki[9] = {1.0 / fx, 0.0, -cx / fx, 0.0, 1.0 / fy, -cy / fy, 0.0, 0.0, 1.0};
    Hs.assign(12 * (size_t)p->S, 0.0);
    for (int s = 0; s < p->S; ++s) {
        const double* Rs = R + 9 * s;
        const double* ts = t + 3 * s;
        double A[9], B[9];
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double a = 0;
                for (int k = 0; k < 3; ++k) a += K[3 * i + k] * Rs[3 * k + j];
                A[3 * i + j] = a;
            }
        for (int i = 0; i < 3; ++i)
            for (int j = 0; j < 3; ++j) {
                double b = 0;
                for (int k = 0; k < 3; ++k) b += A[3 * i + k] * Ki[3 * k + j];
                B[3 * i + j] = b;
            }
        double* h = &Hs[12 * s];
        for (int i = 0; i < 9; ++i) h[i] = B[i];
        for (int i = 0; i < 3; ++i) h[9 + i] = K[3 * i] * ts[0] + K[3 * i + 1] * ts[1] + K[3 * i + 2] * ts[2];
    }
}

inline double at(const double* img, int W, int H, int x, int y) {
    return (x < 0 || y < 0 || x >= W || y >= H) ? 0.0 : img[(size_t)y * W + x];
}

// One warped sample of source s at position (qu, qv) and inverse depth rho.
struct Sample {
    bool ok;
    double u, v, w, val, dIdu, dIdv;
    int i, j;
    double a, b;
};

inline Sample sample(const Model& m, int s, int qu, int qv, double rho, bool force = false) {
    const double* h = &m.H[12 * s];
    Sample r{};
    const double x = h[0] * qu + h[1] * qv + h[2] + h[9] * rho;
    const double y = h[3] * qu + h[4] * qv + h[5] + h[10] * rho;
    const double w = h[6] * qu + h[7] * qv + h[8] + h[11] * rho;
    r.w = w;
    r.u = x / w;
    r.v = y / w;
    r.ok = w >= 0.0 && r.u >= 0.0 && r.u <= m.W - 1 && r.v >= 0.0 && r.v <= m.H_ - 1;
    if (!r.ok && !force) return r;
    const double* img = m.srcs + m.N * s;
    r.i = (int)std::floor(r.u);
    r.j = (int)std::floor(r.v);
    r.a = r.u - r.i;
    r.b = r.v - r.j;
    const double I00 = at(img, m.W, m.H_, r.i, r.j), I10 = at(img, m.W, m.H_, r.i + 1, r.j);
    const double I01 = at(img, m.W, m.H_, r.i, r.j + 1), I11 = at(img, m.W, m.H_, r.i + 1, r.j + 1);
    const double top = I00 + r.a * (I10 - I00), bot = I01 + r.a * (I11 - I01);
    r.val = top + r.b * (bot - top);
    r.dIdu = (1.0 - r.b) * (I10 - I00) + r.b * (I11 - I01);
    r.dIdv = (1.0 - r.a) * (I01 - I00) + r.a * (I11 - I10);
    return r;
}

const int kPatch[9][2] = {{0, 0}, {0, -1}, {0, 1}, {-1, 0}, {1, 0}, {-1, -1}, {1, 1}, {-1, 1}, {1, -1}};

// C (V), pixel validity (N); ok_out (optional): the N*D*S source validity flags of m.frozen
void cost_forward(const Model& m, std::vector<double>& C, std::vector<uint8_t>& valid, uint8_t* ok_out = nullptr) {
    const int W = m.W, H = m.H_, D = m.D;
    C.assign(m.V, 0.0);
    valid.assign(m.N, 1);
#pragma omp parallel for schedule(dynamic, 1)
    for (int v = 0; v < H; ++v)
        for (int u = 0; u < W; ++u) {
            bool pix_ok = true;
            for (int d = 0; d < D; ++d) {
                const double rho = m.p->rho0 + d * m.p->drho;
                double sum = 0.0;
                int n = 0;
                for (int s = 0; s < m.S; ++s) {
                    double tmp = 0.0;
                    const size_t fi = (((size_t)v * W + u) * D + d) * m.S + s;
                    bool ok = m.frozen ? m.frozen[fi] != 0 : true;
                    for (int k = 0; k < 9 && ok; ++k) {
                        const int qu = u + kPatch[k][0], qv = v + kPatch[k][1];
                        const Sample smp = sample(m, s, qu, qv, rho, m.frozen != nullptr);
                        if (!m.frozen) ok = smp.ok;
                        if (ok) tmp += std::fabs(at(m.ref, W, H, qu, qv) - smp.val);
                    }
                    if (ok_out) ok_out[fi] = ok;
                    if (ok) {
                        sum += tmp / 9.0;
                        ++n;
                    }
                }
                if (n == 0) pix_ok = false;
                C[((size_t)v * W + u) * D + d] = n ? sum / n : 0.0;
            }
            valid[(size_t)v * W + u] = pix_ok;
            if (!pix_ok)
                for (int d = 0; d < D; ++d) C[((size_t)v * W + u) * D + d] = 0.0;   // COST_INF = 0
        }
}

struct Chain {
    std::vector<size_t> pix;
};

std::vector<Chain> chains(int W, int H, int dx, int dy) {
    std::vector<Chain> out;
    for (int y = 0; y < H; ++y)
        for (int x = 0; x < W; ++x) {
            const int px = x - dx, py = y - dy;
            if (px >= 0 && py >= 0 && px < W && py < H) continue;
            Chain c;
            for (int xx = x, yy = y; xx >= 0 && yy >= 0 && xx < W && yy < H; xx += dx, yy += dy)
                c.pix.push_back((size_t)yy * W + xx);
            out.push_back(std::move(c));
        }
    return out;
}

inline void penalties(const orc_diff_params* p, const double* ref, size_t a, size_t b, double& P1, double& P2) {
    P1 = p->p1;
    P2 = p->p2;
    if (std::fabs(ref[a] - ref[b]) < p->tau_so) {
        P1 *= p->q1;
        P2 *= p->q2;
    }
}

inline int argmin_low(const double* v, int D) {
    int k = 0;
    for (int d = 1; d < D; ++d)
        if (v[d] < v[k]) k = d;
    return k;
}

// Path r's states L (V) along every chain of direction r.
void path_forward(const Model& m, const std::vector<double>& C, int r, std::vector<double>& L) {
    const int D = m.D;
    L.assign(m.V, 0.0);
    const auto ch = chains(m.W, m.H_, kDirs8[r].dx, kDirs8[r].dy);
#pragma omp parallel for schedule(dynamic, 8)
    for (long ci = 0; ci < (long)ch.size(); ++ci) {
        const auto& pix = ch[ci].pix;
        for (size_t k = 0; k < pix.size(); ++k) {
            const double* c = &C[pix[k] * D];
            double* l = &L[pix[k] * D];
            if (k == 0) {
                for (int d = 0; d < D; ++d) l[d] = c[d];
                continue;
            }
            const double* lp = &L[pix[k - 1] * D];
            double P1, P2;
            penalties(m.p, m.ref, pix[k], pix[k - 1], P1, P2);
            const double mp = lp[argmin_low(lp, D)];
            for (int d = 0; d < D; ++d) {
                double vv = std::min(lp[d], mp + P2);
                double nb = std::numeric_limits<double>::infinity();
                if (d > 0) nb = std::min(nb, lp[d - 1]);
                if (d + 1 < D) nb = std::min(nb, lp[d + 1]);
                vv = std::min(vv, nb + P1);
                l[d] = c[d] + vv - mp;
            }
        }
    }
}

// Adjoint of one path: lambda = gS + routed contributions, gC += lambda at valid pixels.
void path_backward(const Model& m, const std::vector<double>& L, const std::vector<double>& gS,
                   const std::vector<uint8_t>& valid, int r, std::vector<double>& gC) {
    const int D = m.D;
    const auto ch = chains(m.W, m.H_, kDirs8[r].dx, kDirs8[r].dy);
#pragma omp parallel for schedule(dynamic, 8)
    for (long ci = 0; ci < (long)ch.size(); ++ci) {
        const auto& pix = ch[ci].pix;
        std::vector<double> mu((size_t)D, 0.0), lam((size_t)D), nxt((size_t)D);
        for (size_t kk = pix.size(); kk-- > 0;) {
            for (int d = 0; d < D; ++d) lam[d] = gS[pix[kk] * D + d] + mu[d];
            if (valid[pix[kk]])
                for (int d = 0; d < D; ++d) gC[pix[kk] * D + d] += lam[d];
            std::fill(nxt.begin(), nxt.end(), 0.0);
            if (kk > 0) {
                const double* lp = &L[pix[kk - 1] * D];
                double P1, P2;
                penalties(m.p, m.ref, pix[kk], pix[kk - 1], P1, P2);
                const int km = argmin_low(lp, D);
                const double mp = lp[km];
                double total = 0.0;
                for (int d = 0; d < D; ++d) {
                    const double a = lp[d];
                    const double left = d > 0 ? lp[d - 1] : std::numeric_limits<double>::infinity();
                    const double right = d + 1 < D ? lp[d + 1] : std::numeric_limits<double>::infinity();
                    const double nb = std::min(left, right) + P1;
                    const double e = mp + P2;
                    const double vmin = std::min(std::min(a, e), nb);
                    if (a == vmin) nxt[d] += lam[d];
                    else if (nb == vmin) nxt[left <= right ? d - 1 : d + 1] += lam[d];
                    else nxt[km] += lam[d];
                    total += lam[d];
                }
                nxt[km] -= total;
            }
            mu.swap(nxt);
        }
    }
}

double soft_forward(const Model& m, const std::vector<double>& Ssum, const double* rho_gt,
                    const std::vector<uint8_t>& valid, double* rho_hat, std::vector<double>* gS) {
    const int D = m.D;
    const double T = m.p->temperature;
    long nvalid = 0;
    for (size_t i = 0; i < m.N; ++i) nvalid += valid[i] && rho_gt[i] > 0.0;
    double loss = 0.0;
    std::vector<double> w((size_t)D);
    for (size_t i = 0; i < m.N; ++i) {
        const double* s = &Ssum[i * D];
        const double smin = *std::min_element(s, s + D);
        double Z = 0.0;
        for (int d = 0; d < D; ++d) {
            w[d] = std::exp(-(s[d] - smin) / T);
            Z += w[d];
        }
        double rh = 0.0;
        for (int d = 0; d < D; ++d) {
            w[d] /= Z;
            rh += w[d] * (m.p->rho0 + d * m.p->drho);
        }
        const bool in = valid[i] && rho_gt[i] > 0.0;
        if (rho_hat) rho_hat[i] = in ? rh : 0.0;
        if (!in) continue;
        loss += std::fabs(rh - rho_gt[i]);
        if (gS) {
            const double diff = rh - rho_gt[i];
            const double g = (diff > 0 ? 1.0 : (diff < 0 ? -1.0 : 0.0)) / (double)nvalid;
            for (int d = 0; d < D; ++d)
                (*gS)[i * D + d] = g * (-1.0 / T) * w[d] * ((m.p->rho0 + d * m.p->drho) - rh);
        }
    }
    return nvalid ? loss / nvalid : 0.0;
}

void cost_backward(const Model& m, const std::vector<double>& gC, const std::vector<uint8_t>& valid, double* g_srcs,
                   double* g_pose) {
    const int W = m.W, H = m.H_, D = m.D, S = m.S;
    std::memset(g_srcs, 0, sizeof(double) * m.N * S);
    std::memset(g_pose, 0, sizeof(double) * 6 * S);
    for (int v = 0; v < H; ++v)
        for (int u = 0; u < W; ++u) {
            if (!valid[(size_t)v * W + u]) continue;
            for (int d = 0; d < D; ++d) {
                const double g = gC[((size_t)v * W + u) * D + d];
                if (g == 0.0) continue;
                const double rho = m.p->rho0 + d * m.p->drho;
                Sample smp[32][9];
                bool sok[32];
                int n = 0;
                for (int s = 0; s < S; ++s) {
                    sok[s] = true;
                    for (int k = 0; k < 9 && sok[s]; ++k) {
                        smp[s][k] = sample(m, s, u + kPatch[k][0], v + kPatch[k][1], rho);
                        sok[s] = smp[s][k].ok;
                    }
                    n += sok[s];
                }
                if (!n) continue;
                for (int s = 0; s < S; ++s) {
                    if (!sok[s]) continue;
                    double* gi = g_srcs + m.N * s;
                    for (int k = 0; k < 9; ++k) {
                        const Sample& q = smp[s][k];
                        const int qu = u + kPatch[k][0], qv = v + kPatch[k][1];
                        const double diff = at(m.ref, W, H, qu, qv) - q.val;
                        const double sg = diff > 0 ? 1.0 : (diff < 0 ? -1.0 : 0.0);
                        const double c = g / n / 9.0 * (-sg);   // dLoss / dI_hat
                        if (c == 0.0) continue;
                        const double wts[4] = {(1 - q.a) * (1 - q.b), q.a * (1 - q.b), (1 - q.a) * q.b, q.a * q.b};
                        const int tx[4] = {q.i, q.i + 1, q.i, q.i + 1}, ty[4] = {q.j, q.j, q.j + 1, q.j + 1};
                        for (int t4 = 0; t4 < 4; ++t4)
                            if (tx[t4] < W && ty[t4] < H) gi[(size_t)ty[t4] * W + tx[t4]] += c * wts[t4];
                        // pose: P = K^-1 (x, y, w), dP = omega x P + rho upsilon
                        const double x = q.u * q.w, y = q.v * q.w, w = q.w;
                        const double Px = (x - m.cx * w) / m.fx, Py = (y - m.cy * w) / m.fy, Pz = w;
                        const double dP[6][3] = {{0, -Pz, Py}, {Pz, 0, -Px}, {-Py, Px, 0},
                                                 {rho, 0, 0}, {0, rho, 0}, {0, 0, rho}};
                        for (int i = 0; i < 6; ++i) {
                            const double du = (m.fx * dP[i][0] + (m.cx - q.u) * dP[i][2]) / w;
                            const double dv = (m.fy * dP[i][1] + (m.cy - q.v) * dP[i][2]) / w;
                            g_pose[6 * s + i] += c * (q.dIdu * du + q.dIdv * dv);
                        }
                    }
                }
            }
        }
}

Model make_model(const orc_diff_params* p, const double* ref, const double* srcs, const double* K, const double* R,
                 const double* t) {
    Model m;
    m.p = p;
    m.ref = ref;
    m.srcs = srcs;
    m.fx = K[0];
    m.cx = K[2];
    m.fy = K[4];
    m.cy = K[5];
    m.W = p->W;
    m.H_ = p->H;
    m.D = p->D;
    m.S = p->S;
    m.N = (size_t)p->W * p->H;
    m.V = m.N * p->D;
    homographies(p, K, R, t, m.H);
    return m;
}

}  // namespace

extern "C" {

double orc_diff_forward(const orc_diff_params* p, const double* ref, const double* srcs, const double* K,
                        const double* R, const double* t, const double* rho_gt, double* rho_hat, uint8_t* valid_out) {
    const Model m = make_model(p, ref, srcs, K, R, t);
    std::vector<double> C, L, Ssum(m.V, 0.0);
    std::vector<uint8_t> valid;
    cost_forward(m, C, valid);
    for (int r = 0; r < p->num_paths; ++r) {
        path_forward(m, C, r, L);
        for (size_t i = 0; i < m.V; ++i) Ssum[i] += L[i];
    }
    if (valid_out) std::memcpy(valid_out, valid.data(), m.N);
    return soft_forward(m, Ssum, rho_gt, valid, rho_hat, nullptr);
}

void orc_diff_source_validity(const orc_diff_params* p, const double* ref, const double* srcs, const double* K,
                              const double* R, const double* t, uint8_t* ok) {
    const Model m = make_model(p, ref, srcs, K, R, t);
    std::vector<double> C;
    std::vector<uint8_t> valid;
    cost_forward(m, C, valid, ok);
}

double orc_diff_forward_frozen(const orc_diff_params* p, const double* ref, const double* srcs, const double* K,
                               const double* R, const double* t, const double* rho_gt, const uint8_t* frozen) {
    Model m = make_model(p, ref, srcs, K, R, t);
    m.frozen = frozen;
    std::vector<double> C, L, Ssum(m.V, 0.0);
    std::vector<uint8_t> valid;
    cost_forward(m, C, valid);
    for (int r = 0; r < p->num_paths; ++r) {
        path_forward(m, C, r, L);
        for (size_t i = 0; i < m.V; ++i) Ssum[i] += L[i];
    }
    return soft_forward(m, Ssum, rho_gt, valid, nullptr, nullptr);
}

double orc_diff_backward(const orc_diff_params* p, const double* ref, const double* srcs, const double* K,
                         const double* R, const double* t, const double* rho_gt, double* g_srcs, double* g_pose) {
    const Model m = make_model(p, ref, srcs, K, R, t);
    std::vector<double> C, L, Ssum(m.V, 0.0);
    std::vector<uint8_t> valid;
    cost_forward(m, C, valid);
    for (int r = 0; r < p->num_paths; ++r) {
        path_forward(m, C, r, L);
        for (size_t i = 0; i < m.V; ++i) Ssum[i] += L[i];
    }
    std::vector<double> gS(m.V, 0.0), gC(m.V, 0.0);
    const double loss = soft_forward(m, Ssum, rho_gt, valid, nullptr, &gS);
    for (int r = 0; r < p->num_paths; ++r) {   // the forward of each path recomputed
        path_forward(m, C, r, L);
        path_backward(m, L, gS, valid, r, gC);
    }
    cost_backward(m, gC, valid, g_srcs, g_pose);
    return loss;
}

}  // extern "C"
