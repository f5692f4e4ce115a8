// k_z_step_c: the z pass with one lane per complex mode (the device code is
// in sf_zstep_c.cuh, which the ensemble kernels of sf_kernels.cu share).
#include "sf_zstep_c.cuh"

namespace sf {

template <bool IC>
__global__ void __launch_bounds__(kCW * 32, 3) k_z_step_c(StageArgs a) {
  z_step_c_body<IC>(a, blockIdx.x, blockIdx.z);
}

bool zstep_c_supported(const Geo& g) { return zc_fits(g.N3); }

int launch_z_step_c(const StageArgs& a, cudaStream_t st) {
  const Geo& g = a.g;
  const dim3 grid((g.P + 15) / 16, 1, g.nrun);
  k_z_step_c<true><<<grid, kCW * 32, zc_smem_bytes(g.N3), st>>>(a);
  return 1;
}

int prepare_zstep_c_kernels() {
  const int lim = 227 * 1024;
  return cudaFuncSetAttribute(k_z_step_c<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim) == cudaSuccess
             ? 0
             : -1;
}

}  // namespace sf
