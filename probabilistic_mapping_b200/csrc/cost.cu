// cost.cu -- plane-sweep absolute-difference cost volume (reference: calc_cost.cu:11-253).
//
// The reference launches one thread per plane and walks D pixels per block, computing all
// nine projective warps of the 3x3 patch for every voxel and every source frame, with a
// read-modify-write of cost and count per call.  Here a CTA owns a 30x8 pixel tile and 16
// planes; each warp owns two planes and streams the tile row by row:
//   * lane l warps the sample at column x0-1+l of the current row (lanes 0 and 31 are the halo
//     columns) for both planes at once on the packed FP32x2 pipe; the left and right
//     neighbours' samples arrive by one shuffle each and the rows above and below stay in
//     registers, so each warped position is computed once per plane instead of up to nine times;
//   * reference mode: the two samples the reference takes from a corrupted neighbour
//     (calc_cost.cu:49-51 and :69-71) depend on the pixel itself and are warped per output pixel;
//   * the nine terms are summed in the reference's order and folded into the running mean of
//     the tile's voxels, kept in shared memory in [pixel][plane] order, over all source frames
//     queued since initReference; the volume is then stored once, in contiguous plane runs of
//     the plane-innermost layout (cuda_utils.h:34).
// Source frames are "quads": pixel (x, y) holds I(x,y), I(x,y+1), I(x+1,y), I(x+1,y+1) with the
// texture border (zero) applied, so a bilinear sample is one aligned 16-byte load whose halves
// are the packed operands of the horizontal interpolation.  floor() adds 1.5 * 2^23 with
// round-toward-minus-infinity, leaving the integer part in the mantissa; the reciprocal is
// rcp.approx plus one Newton step without a range branch (rcp_warp2: RN(1/w) wherever an
// image-sized scene puts w, a stated value elsewhere); the divisions of the running mean are a
// reciprocal-multiply with one FMA correction.  Each is checked over every float against its
// definition (pm_debug_check_arith), and every packed instruction rounds each element like its
// scalar counterpart, so the FP32 oracle's scalar algorithm reproduces the volume bit for bit.
#include "cost_device.cuh"

namespace pm {
namespace {

// Three CTAs per SM; four for the FP16 form's texture sampler in a first pass, whose FP16 counts
// leave the smaller tile state (0.764 against 0.777 ms at 640x480x128, 5 sources; the FP32
// texture form loses 7 % at four, its larger state taking L1 from the texture cache).
template <int MODE, bool HALF, int SAMP, bool INC>
__global__ void __launch_bounds__(NT, (HALF && SAMP == kTex && !INC) ? 4 : 3) cost_kernel(const CostLaunch a) {
    extern __shared__ __align__(16) unsigned char smem_raw[];
    cost_tile<MODE, HALF, SAMP, INC>(a, blockIdx.x, blockIdx.y, blockIdx.z, smem_raw);
}

template <int PPL>
__global__ void __launch_bounds__(256) rebase_kernel(__half2* __restrict__ cost, const float* __restrict__ boff,
                                                     float* __restrict__ off, long npix, int D) {
    rebase_pixels<PPL, false>(cost, boff, off, npix, D, ((long)blockIdx.x * 8 + (threadIdx.x >> 5)) * RB,
                              threadIdx.x & 31);
}

// invalid[p] = 1 where some plane of pixel p was never measured (its cost is still -1); one
// warp per pixel.
template <bool HALF>
__global__ void __launch_bounds__(256) invalid_kernel(const void* cost, long npix, int D, uint8_t* invalid) {
    const long pix = (long)blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (pix >= npix) return;
    bool neg = false;
    for (int d = lane; d < D; d += 32) neg |= load_cost<HALF>(cost, (size_t)pix * D + d) < 0.0f;
    const bool any = __any_sync(kFull, neg);
    if (lane == 0) invalid[pix] = any ? 1 : 0;
}

template <int MODE, bool HALF, int SAMP>
cudaError_t launch_t(const CostLaunch& a, dim3 grid, cudaStream_t s) {
    auto kern = a.incremental ? cost_kernel<MODE, HALF, SAMP, true> : cost_kernel<MODE, HALF, SAMP, false>;
    const size_t smem = (HALF && !a.incremental) ? SmemL<true>::BYTES : SmemL<false>::BYTES;
    if (smem > 48 * 1024) {
        cudaError_t e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e != cudaSuccess) return e;
    }
    kern<<<grid, NT, smem, s>>>(a);
    return cudaGetLastError();
}

template <int MODE, bool HALF>
cudaError_t launch_q(const CostLaunch& a, dim3 grid, cudaStream_t s) {
    // FP16 volumes come from the FP16 form's samplers, FP32 volumes from the FP32 ones
    if constexpr (HALF) {
        if (a.use_tex) return launch_t<MODE, true, kTex>(a, grid, s);
        return a.srcq ? launch_t<MODE, true, kQuadH>(a, grid, s) : cudaErrorInvalidValue;
    } else {
        if (a.use_tex) return launch_t<MODE, false, kTexF>(a, grid, s);
        return a.srcq ? launch_t<MODE, false, kQuad>(a, grid, s) : launch_t<MODE, false, kPlain>(a, grid, s);
    }
}

}  // namespace

cudaError_t launch_cost(const CostLaunch& a, cudaStream_t s) {
    if (a.nsrc > kMaxSources || a.D % PCB || a.W < 1 || a.H < 1) return cudaErrorInvalidValue;
    if (a.cost_half && (!a.offset || !a.block_offset || (a.D / 32) % 2)) return cudaErrorInvalidValue;
    const dim3 grid((a.W + TXU - 1) / TXU, (a.H + TY - 1) / TY, a.D / PCB);
    cudaError_t e;
    if (a.mode == 0) e = a.cost_half ? launch_q<0, true>(a, grid, s) : launch_q<0, false>(a, grid, s);
    else e = a.cost_half ? launch_q<1, true>(a, grid, s) : launch_q<1, false>(a, grid, s);
    if (e != cudaSuccess) return e;
    if (a.kernel_done && (e = cudaEventRecord(a.kernel_done, s)) != cudaSuccess) return e;
    if (a.cost_half) {
        const long np = (long)a.W * a.H;
        const unsigned blocks = (unsigned)((np + 8 * RB - 1) / (8 * RB));
        __half2* c = static_cast<__half2*>(a.cost);
        switch (a.D / 32) {
            case 2: rebase_kernel<2><<<blocks, 256, 0, s>>>(c, a.block_offset, a.offset, np, a.D); break;
            case 4: rebase_kernel<4><<<blocks, 256, 0, s>>>(c, a.block_offset, a.offset, np, a.D); break;
            case 6: rebase_kernel<6><<<blocks, 256, 0, s>>>(c, a.block_offset, a.offset, np, a.D); break;
            case 8: rebase_kernel<8><<<blocks, 256, 0, s>>>(c, a.block_offset, a.offset, np, a.D); break;
            default: return cudaErrorInvalidValue;
        }
        if ((e = cudaGetLastError()) != cudaSuccess) return e;
    }
    if (!a.invalid) return cudaSuccess;
    const long npix = (long)a.W * a.H;
    if (a.cost_half) invalid_kernel<true><<<(unsigned)((npix + 7) / 8), 256, 0, s>>>(a.cost, npix, a.D, a.invalid);
    else invalid_kernel<false><<<(unsigned)((npix + 7) / 8), 256, 0, s>>>(a.cost, npix, a.D, a.invalid);
    return cudaGetLastError();
}

}  // namespace pm
