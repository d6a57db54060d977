// cost.cu -- plane-sweep absolute-difference cost volume (reference: calc_cost.cu:11-253).
//
// The reference launches one thread per plane and walks D pixels per block, computing all
// nine projective warps of the 3x3 patch for every voxel and every source frame, with a
// read-modify-write of cost and count per call.  Here one CTA owns a 32x8 pixel tile and
// all planes of it, and for every chunk of 16 planes and every source frame runs three
// phases over shared memory:
//   A  warp the tile plus a one-pixel halo once (340 positions x 16 planes); the nine patch
//      samples of a voxel are read from this tile instead of being warped again;
//   A2 (reference mode) the two samples the reference computes from a corrupted neighbour
//      (calc_cost.cu:50-51 and :70-71) depend on the pixel itself, so each thread warps them
//      for its own pixel and stores the two absolute differences;
//   B  each thread sums the nine terms of its pixel in the reference's order and applies the
//      running-mean update in registers.
// All source frames queued since initReference are folded in one pass, so the volume is
// written once.  Further choices:
//   * source frames are stored as "quads": pixel (x, y) holds its 2x2 bilinear footprint
//     (I(x,y), I(x+1,y), I(x,y+1), I(x+1,y+1)) with the texture border (zero) applied, so a
//     bilinear sample is one aligned 16-byte load;
//   * floor() for addressing adds 1.5 * 2^23 with round-toward-minus-infinity, which leaves
//     the integer part in the mantissa, instead of float->int conversions;
//   * the divisions of the running mean use a reciprocal-multiply with one FMA correction
//     (Markstein), exhaustively checked to equal the correctly rounded quotient whenever the
//     quotient is a normal number; below that the code takes IEEE division;
//   * the tile is transposed through shared memory so the volume is stored in contiguous
//     plane runs of the plane-innermost layout (cuda_utils.h:34).
// All FP32 arithmetic uses explicit round-to-nearest intrinsics (see pm_device.cuh).
#include "pm_device.cuh"

namespace pm {
namespace {

constexpr int TX = 32, TY = 8;          // pixel tile
constexpr int PC = 16;                  // planes per chunk
constexpr int HX = TX + 2, HY = TY + 2; // tile + halo
constexpr int NPOS = HX * HY;           // 340 warped positions
constexpr int NT = TX * TY;             // 256 threads, one per pixel
constexpr int SP = PC + 1;              // transpose staging pitch (bank-conflict free)
constexpr int MAXCNT = kMaxSources + 2; // reciprocal table covers counts 0..kMaxSources+1

static_assert(NT * SP <= PC * NPOS, "staging must fit into the warp tile");
static_assert(TX == 32 && NT == TX * TY, "one warp per tile row, one thread per pixel");
static_assert((TX * PC) % 32 == 0, "the transposed block is moved in whole warp steps");
static_assert(MAXCNT <= NT && PC <= NT, "tables are filled by one thread per entry");

// shared-memory layout (floats)
template <int MODE> struct Smem {
    static constexpr int WT = 0;                       // [PC][NPOS] warped samples
    static constexpr int BUG = WT + PC * NPOS;         // [PC][2][NT] |R - B4|, |R - B8|
    static constexpr int HXo = BUG + (MODE == 0 ? PC * 2 * NT : 0);
    static constexpr int HYo = HXo + NPOS;
    static constexpr int HZo = HYo + NPOS;
    static constexpr int RHO = HZo + NPOS;             // [PC] plane inverse depths of the chunk
    static constexpr int RTAB = RHO + PC;              // [MAXCNT] RN(1/n)
    static constexpr int REF = RTAB + MAXCNT;          // [NPOS] reference image tile + halo
    static constexpr int TOTAL = REF + NPOS;
    static constexpr size_t BYTES = sizeof(float) * TOTAL;
};

__device__ __forceinline__ float ref_at(const float* __restrict__ ref, int W, int H, int x, int y) {
    return (x < 0 || y < 0 || x >= W || y >= H) ? 0.0f : __ldg(ref + (size_t)y * W + x);
}

template <bool HALF> __device__ __forceinline__ void store_cost(void* base, size_t i, float v) {
    if constexpr (HALF) reinterpret_cast<__half*>(base)[i] = __float2half_rn(v);
    else reinterpret_cast<float*>(base)[i] = v;
}
template <bool HALF> __device__ __forceinline__ float load_cost(const void* base, size_t i) {
    if constexpr (HALF) return __half2float(reinterpret_cast<const __half*>(base)[i]);
    else return reinterpret_cast<const float*>(base)[i];
}

// Source access: quad layout (one 16-byte load per bilinear sample) or plain float rows.
template <bool QUAD> struct Src;
template <> struct Src<true> {
    const float4* __restrict__ q;
    int W, H;
    // 0 <= u <= W-1 and 0 <= v <= H-1 (< 2^22): floor by the 1.5 * 2^23 round-down add
    __device__ __forceinline__ float fetch(float u, float v) const {
        float fu, fv;
        int i, j;
        floor_split(u, fu, i);
        floor_split(v, fv, j);
        const float a = __fsub_rn(u, fu), b = __fsub_rn(v, fv);
        const float4 t = __ldg(q + (size_t)j * W + i);
        const float top = __fmaf_rn(a, __fsub_rn(t.y, t.x), t.x);
        const float bot = __fmaf_rn(a, __fsub_rn(t.w, t.z), t.z);
        return __fmaf_rn(b, __fsub_rn(bot, top), top);
    }
};
template <> struct Src<false> {
    const float* __restrict__ p;
    int W, H;
    __device__ __forceinline__ float fetch(float u, float v) const { return bilinear(p, W, H, u, v); }
};

// warp_fetch of pm_device.cuh over either source layout
template <bool QUAD>
__device__ __forceinline__ float warp_sample(const Src<QUAD>& src, float x, float y, float z, const Hom& h,
                                             float rho) {
    const float w = __fmaf_rn(h.t3, rho, z);
    const float nx = __fmaf_rn(h.t1, rho, x);
    const float ny = __fmaf_rn(h.t2, rho, y);
    const float r = rcp_rn(w);
    const float u = __fmul_rn(nx, r), v = __fmul_rn(ny, r);
    const bool ok = (w >= 0.0f) && (u >= 0.0f) && (u <= (float)(src.W - 1)) && (v >= 0.0f) &&
                    (v <= (float)(src.H - 1));
    return ok ? src.fetch(u, v) : nan_f();
}

// ---- two samples at once on the packed FP32x2 pipe ----------------------------------------
// Each element follows exactly the scalar operation sequence above (every packed instruction
// rounds each element like its scalar counterpart), so the results are bit-identical; the pair
// only halves the instruction count.
__device__ __forceinline__ float2 f2(float a, float b) { return make_float2(a, b); }
__device__ __forceinline__ float2 neg2(float2 a) { return make_float2(-a.x, -a.y); }

__device__ __forceinline__ float2 rcp_rn2(float2 w) {
    const bool in0 = w.x >= 1.17549435e-38f && w.x < 8.50705917e37f;
    const bool in1 = w.y >= 1.17549435e-38f && w.y < 8.50705917e37f;
    if (in0 && in1) {
        float2 r0;
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r0.x) : "f"(w.x));
        asm("rcp.approx.ftz.f32 %0, %1;" : "=f"(r0.y) : "f"(w.y));
        return __ffma2_rn(r0, __ffma2_rn(neg2(w), r0, f2(1.0f, 1.0f)), r0);
    }
    return f2(rcp_rn(w.x), rcp_rn(w.y));
}

// bilinear from the quad layout for two in-range sample positions
__device__ __forceinline__ float2 fetch2(const float4* __restrict__ q, int W, float2 u, float2 v) {
    const float2 M = f2(12582912.0f, 12582912.0f);
    const float2 tu = __fadd2_rd(u, M), tv = __fadd2_rd(v, M);
    const int i0 = __float_as_int(tu.x) - 0x4B400000, i1 = __float_as_int(tu.y) - 0x4B400000;
    const int j0 = __float_as_int(tv.x) - 0x4B400000, j1 = __float_as_int(tv.y) - 0x4B400000;
    const float2 a = __fadd2_rn(u, neg2(__fadd2_rn(tu, neg2(M))));   // u - floor(u)
    const float2 b = __fadd2_rn(v, neg2(__fadd2_rn(tv, neg2(M))));
    const float4 t0 = __ldg(q + (size_t)j0 * W + i0);
    const float4 t1 = __ldg(q + (size_t)j1 * W + i1);
    // (top, bot) of each sample as one pair: fma(a, (t.y - t.x, t.w - t.z), (t.x, t.z))
    const float2 tb0 = __ffma2_rn(f2(a.x, a.x), __fadd2_rn(f2(t0.y, t0.w), neg2(f2(t0.x, t0.z))), f2(t0.x, t0.z));
    const float2 tb1 = __ffma2_rn(f2(a.y, a.y), __fadd2_rn(f2(t1.y, t1.w), neg2(f2(t1.x, t1.z))), f2(t1.x, t1.z));
    return __ffma2_rn(b, __fadd2_rn(f2(tb0.y, tb1.y), neg2(f2(tb0.x, tb1.x))), f2(tb0.x, tb1.x));
}

// warp_sample for two (x, y, z, rho) at once; a rejected element is NaN.
__device__ __forceinline__ float2 warp_sample2(const Src<true>& src, float2 x, float2 y, float2 z, const Hom& h,
                                               float2 rho) {
    const float2 w = __ffma2_rn(f2(h.t3, h.t3), rho, z);
    const float2 nx = __ffma2_rn(f2(h.t1, h.t1), rho, x);
    const float2 ny = __ffma2_rn(f2(h.t2, h.t2), rho, y);
    const float2 r = rcp_rn2(w);
    const float2 u = __fmul2_rn(nx, r), v = __fmul2_rn(ny, r);
    const float W1 = (float)(src.W - 1), H1 = (float)(src.H - 1);
    const bool ok0 = (w.x >= 0.0f) && (u.x >= 0.0f) && (u.x <= W1) && (v.x >= 0.0f) && (v.x <= H1);
    const bool ok1 = (w.y >= 0.0f) && (u.y >= 0.0f) && (u.y <= W1) && (v.y >= 0.0f) && (v.y <= H1);
    // positions of rejected elements are replaced by 0 so the fetch stays inside the image
    const float2 s = fetch2(src.q, src.W, f2(ok0 ? u.x : 0.0f, ok1 ? u.y : 0.0f), f2(ok0 ? v.x : 0.0f, ok1 ? v.y : 0.0f));
    return f2(ok0 ? s.x : nan_f(), ok1 ? s.y : nan_f());
}

__device__ __forceinline__ Hom load_hom(const CostLaunch& a, int s) {
    Hom h;
    h.r11 = a.hom[s][0]; h.r12 = a.hom[s][1]; h.r13 = a.hom[s][2];
    h.r21 = a.hom[s][3]; h.r22 = a.hom[s][4]; h.r23 = a.hom[s][5];
    h.r31 = a.hom[s][6]; h.r32 = a.hom[s][7]; h.r33 = a.hom[s][8];
    h.t1 = a.hom[s][9]; h.t2 = a.hom[s][10]; h.t3 = a.hom[s][11];
    return h;
}

// MODE 0: reference sample set (calc_cost.cu:83-199); MODE 1: corrected 3x3 patch.
template <int MODE, bool HALF, bool QUAD>
__global__ void __launch_bounds__(NT, 3) cost_kernel(const CostLaunch a) {
    using SM = Smem<MODE>;
    extern __shared__ __align__(16) float smem[];
    float* const wt = smem + SM::WT;
    float* const bug = smem + SM::BUG;
    float* const hx = smem + SM::HXo;
    float* const hy = smem + SM::HYo;
    float* const hz = smem + SM::HZo;
    float* const rho_s = smem + SM::RHO;
    float* const rtab = smem + SM::RTAB;

    const int tid = threadIdx.x, tx = tid & 31, ty = tid >> 5;
    const int x0 = blockIdx.x * TX, y0 = blockIdx.y * TY;
    const int u = x0 + tx, v = y0 + ty;
    const int W = a.W, H = a.H, D = a.D;
    const bool inside = (u < W) && (v < H);
    if (tid < MAXCNT) rtab[tid] = tid == 0 ? 0.0f : __frcp_rn((float)tid);

    // reference-image tile with halo (border addressing -> 0, calc_cost.cu:230-231); read per
    // phase from shared memory so it does not occupy registers across the phases
    float* const rt = smem + SM::REF;
    for (int p = tid; p < NPOS; p += NT) {
        const int py = p / HX, px = p - py * HX;
        rt[p] = ref_at(a.ref, W, H, x0 + px - 1, y0 + py - 1);
    }
    const float* const rc = rt + (ty + 1) * HX + (tx + 1);   // this pixel's centre
    const float r9 = __frcp_rn(9.0f);

    bool pix_invalid = false;

    for (int d0 = 0; d0 < D; d0 += PC) {
        float acc[PC], cn[PC];
        __syncthreads();   // previous chunk's staging reads are done
        if (tid < PC) rho_s[tid] = __fmaf_rn((float)(d0 + tid), a.drho, a.rho0);   // calc_cost.cu:81
        if (a.incremental) {
            // running state from memory, transposed through shared memory
            for (int pass = 0; pass < 2; ++pass) {
                __syncthreads();
                // warp ty moves the TX x PC block of its pixel row; lane-linear order keeps the
                // global accesses contiguous within each pixel's plane run
                for (int q = tx; q < TX * PC; q += 32) {
                    const int i = q / PC, k = q - i * PC;
                    const int pu = x0 + i, pv = y0 + ty;
                    float val = 0.0f;
                    if (pu < W && pv < H) {
                        const size_t e = ((size_t)pv * W + pu) * D + d0 + k;
                        val = pass == 0 ? load_cost<HALF>(a.cost, e) : a.cnt[e];
                    }
                    wt[(ty * TX + i) * SP + k] = val;
                }
                __syncthreads();
#pragma unroll
                for (int k = 0; k < PC; ++k) {
                    if (pass == 0) acc[k] = wt[tid * SP + k];
                    else cn[k] = wt[tid * SP + k];
                }
            }
        } else {
#pragma unroll
            for (int k = 0; k < PC; ++k) { acc[k] = -1.0f; cn[k] = 0.0f; }
        }

        for (int s = 0; s < a.nsrc; ++s) {
            Src<QUAD> src;
            if constexpr (QUAD) src.q = a.srcq + (size_t)s * W * H;
            else src.p = a.srcs + (size_t)s * W * H;
            src.W = W;
            src.H = H;
            const Hom h = load_hom(a, s);

            __syncthreads();   // previous consumers of wt / hx / bug are done
            for (int p = tid; p < NPOS; p += NT) {
                const int py = p / HX, px = p - py * HX;
                homog(h, x0 + px - 1, y0 + py - 1, hx[p], hy[p], hz[p]);
            }
            __syncthreads();
            // A: warped tile (quad sources: planes k and k + PC/2 of a position as one pair)
            if constexpr (QUAD) {
                constexpr int HALF_PC = PC / 2;
#pragma unroll 2
                for (int i = tid; i < HALF_PC * NPOS; i += NT) {
                    const int k = i / NPOS, p = i - k * NPOS;
                    const float x = hx[p], y = hy[p], z = hz[p];
                    const float2 s2 = warp_sample2(src, f2(x, x), f2(y, y), f2(z, z), h,
                                                   f2(rho_s[k], rho_s[k + HALF_PC]));
                    wt[i] = s2.x;
                    wt[i + HALF_PC * NPOS] = s2.y;
                }
            } else {
#pragma unroll 2
                for (int i = tid; i < PC * NPOS; i += NT) {
                    const int k = i / NPOS, p = i - k * NPOS;
                    wt[i] = warp_sample<QUAD>(src, hx[p], hy[p], hz[p], h, rho_s[k]);
                }
            }
            // A2: per-pixel samples of the corrupted neighbours (calc_cost.cu:49-51, 69-71)
            if (MODE == 0 && inside) {
                float xc, yc, zc;
                homog(h, u, v, xc, yc, zc);
                const float xr = __fadd_rn(xc, h.r11), yr = __fadd_rn(xc, h.r21), zr = __fadd_rn(xc, h.r31);
                const float xru = __fsub_rn(xr, h.r12), yru = __fsub_rn(xr, h.r22), zru = __fsub_rn(xr, h.r32);
                const float Rr = rc[1], Rru = rc[1 - HX];
#pragma unroll 2
                for (int k = 0; k < PC; ++k) {
                    const float rho = rho_s[k];
                    float B4, B8;
                    if constexpr (QUAD) {
                        const float2 b = warp_sample2(src, f2(xr, xru), f2(yr, yru), f2(zr, zru), h, f2(rho, rho));
                        B4 = b.x;
                        B8 = b.y;
                    } else {
                        B4 = warp_sample<QUAD>(src, xr, yr, zr, h, rho);
                        B8 = warp_sample<QUAD>(src, xru, yru, zru, h, rho);
                    }
                    bug[(2 * k) * NT + tid] = fabsf(__fsub_rn(Rr, B4));       // term 4 (:145)
                    bug[(2 * k + 1) * NT + tid] = fabsf(__fsub_rn(Rru, B8));  // term 8 (:198)
                }
            }
            __syncthreads();

            // B: nine-term sum in the reference order and the running mean
            if (inside) {
                const float* wc = wt + (ty + 1) * HX + (tx + 1);
                const float Rc = rc[0], Ru = rc[-HX], Rd = rc[HX], Rl = rc[-1], Rr = rc[1];
                const float Rul = rc[-HX - 1], Rdr = rc[HX + 1], Rld = rc[HX - 1], Rru = rc[1 - HX];
#pragma unroll
                for (int k = 0; k < PC; ++k) {
                    const float* w = wc + k * NPOS;
                    const float W0 = w[0], Wu = w[-HX], Wd = w[HX], Wl = w[-1];
                    const float Wul = w[-HX - 1], Wdr = w[HX + 1], Wld = w[HX - 1];
                    float tmp;
                    if constexpr (MODE == 0) {
                        const float t4 = bug[(2 * k) * NT + tid], t8 = bug[(2 * k + 1) * NT + tid];
                        tmp = fabsf(__fsub_rn(Rc, W0));                    // 0  (:93)
                        tmp = __fadd_rn(tmp, fabsf(__fsub_rn(Rd, Wu)));    // 1  (:106)
                        tmp = __fadd_rn(tmp, fabsf(__fsub_rn(Ru, Wd)));    // 2  (:119)
                        tmp = __fadd_rn(tmp, fabsf(__fsub_rn(Rl, Wl)));    // 3  (:132)
                        tmp = __fadd_rn(tmp, t4);                          // 4  (:145)
                        tmp = __fadd_rn(tmp, fabsf(__fsub_rn(Rul, Wul)));  // 5  (:159)
                        tmp = __fadd_rn(tmp, fabsf(__fsub_rn(Rdr, Wdr)));  // 6  (:172)
                        tmp = __fadd_rn(tmp, fabsf(__fsub_rn(Rld, Wld)));  // 7  (:185)
                        tmp = __fadd_rn(tmp, t8);                          // 8  (:198)
                    } else {
                        const float Wr = w[1], Wru = w[-HX + 1];
                        tmp = fabsf(__fsub_rn(Rc, W0));
                        tmp = __fadd_rn(tmp, fabsf(__fsub_rn(Ru, Wu)));
                        tmp = __fadd_rn(tmp, fabsf(__fsub_rn(Rd, Wd)));
                        tmp = __fadd_rn(tmp, fabsf(__fsub_rn(Rl, Wl)));
                        tmp = __fadd_rn(tmp, fabsf(__fsub_rn(Rr, Wr)));
                        tmp = __fadd_rn(tmp, fabsf(__fsub_rn(Rul, Wul)));
                        tmp = __fadd_rn(tmp, fabsf(__fsub_rn(Rdr, Wdr)));
                        tmp = __fadd_rn(tmp, fabsf(__fsub_rn(Rld, Wld)));
                        tmp = __fadd_rn(tmp, fabsf(__fsub_rn(Rru, Wru)));
                    }
                    if (tmp == tmp) {   // a rejected sample skips the voxel (calc_cost.cu:89-91)
                        const float m = div_small(tmp, 9.0f, r9);     // tmp / 9.0f
                        if (acc[k] < 0.0f) {                         // first measurement (:200-203)
                            acc[k] = m;
                            cn[k] = 1.0f;
                        } else {                                     // running mean (:205-206)
                            const float n1 = __fadd_rn(cn[k], 1.0f);
                            const float num = __fmaf_rn(cn[k], acc[k], m);
                            const int ni = (int)n1;   // counts beyond the table (long running states)
                            acc[k] = ni < MAXCNT ? div_small(num, n1, rtab[ni]) : __fdiv_rn(num, n1);
                            cn[k] = n1;
                        }
                    }
                }
            }
        }

        // transpose through shared memory and store contiguous plane runs of the volume
        for (int pass = 0; pass < (a.cnt ? 2 : 1); ++pass) {
            __syncthreads();
#pragma unroll
            for (int k = 0; k < PC; ++k) wt[tid * SP + k] = pass == 0 ? acc[k] : cn[k];
            __syncthreads();
            for (int q = tx; q < TX * PC; q += 32) {
                const int i = q / PC, k = q - i * PC;
                const int pu = x0 + i, pv = y0 + ty;
                if (pu < W && pv < H) {
                    const size_t e = ((size_t)pv * W + pu) * D + d0 + k;
                    const float val = wt[(ty * TX + i) * SP + k];
                    if (pass == 0) store_cost<HALF>(a.cost, e, val);
                    else a.cnt[e] = val;
                }
            }
        }
        if (inside) {
#pragma unroll
            for (int k = 0; k < PC; ++k) pix_invalid |= (cn[k] == 0.0f);
        }
    }
    if (a.invalid && inside) a.invalid[(size_t)v * W + u] = pix_invalid ? 1 : 0;
}

template <int MODE, bool HALF, bool QUAD>
cudaError_t launch_t(const CostLaunch& a, dim3 grid, cudaStream_t s) {
    auto kern = cost_kernel<MODE, HALF, QUAD>;
    constexpr size_t bytes = Smem<MODE>::BYTES;
    if (bytes > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
        if (e != cudaSuccess) return e;
    }
    kern<<<grid, NT, bytes, s>>>(a);
    return cudaGetLastError();
}

template <int MODE, bool HALF>
cudaError_t launch_q(const CostLaunch& a, dim3 grid, cudaStream_t s) {
    return a.srcq ? launch_t<MODE, HALF, true>(a, grid, s) : launch_t<MODE, HALF, false>(a, grid, s);
}

}  // namespace

cudaError_t launch_cost(const CostLaunch& a, cudaStream_t s) {
    if (a.nsrc > kMaxSources) return cudaErrorInvalidValue;
    const dim3 grid((a.W + TX - 1) / TX, (a.H + TY - 1) / TY);
    if (a.mode == 0) return a.cost_half ? launch_q<0, true>(a, grid, s) : launch_q<0, false>(a, grid, s);
    return a.cost_half ? launch_q<1, true>(a, grid, s) : launch_q<1, false>(a, grid, s);
}

}  // namespace pm
