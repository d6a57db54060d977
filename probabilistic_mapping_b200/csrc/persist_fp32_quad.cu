// persist_fp32_quad.cu -- the persistent kernel's instantiations for one form (persist_kernel.cuh).
#include "persist_kernel.cuh"

namespace pm {
cudaError_t launch_persist_fp32_quad(const PersistLaunch& L, cudaStream_t s) { return launch_form<false, kQuad>(L, s); }
}  // namespace pm
