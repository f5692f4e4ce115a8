// k_z_step_c: the z pass with one lane per complex mode (the device code is
// in sf_zstep_c.cuh, which the ensemble kernels of sf_kernels.cu share).
// CC z-chunks per block, two per warp: 16 (8 warps, 3 blocks per SM) by
// default, 32 (16 warps, one block per SM) for grids whose blocks leave SMs
// idle, as k_z_step takes 16 warps there.
#include "sf_zstep_c.cuh"

namespace sf {

template <int CC, bool IC>
__global__ void __launch_bounds__(CC * 16, CC == 16 ? 3 : 1) k_z_step_c(StageArgs a) {
  z_step_c_body<CC, IC>(a, blockIdx.x, blockIdx.z);
}

// chunks per block of a launch: 32 when the setting asks for 16 warps, or
// (setting 0) when one block per mode group leaves SMs without a block
static int zc_chunks(const StageArgs& a) {
  const Geo& g = a.g;
  const bool wide = a.zchunks == 16 || (a.zchunks == 0 && (long long)((g.P + 15) / 16) * g.nrun < 148);
  return (wide && zc_fits<32>(g.N3)) ? 32 : 16;
}

bool zstep_c_supported(const Geo& g) { return zc_fits<16>(g.N3); }

int launch_z_step_c(const StageArgs& a, cudaStream_t st) {
  const Geo& g = a.g;
  const dim3 grid((g.P + 15) / 16, 1, g.nrun);
  if (zc_chunks(a) == 32) k_z_step_c<32, true><<<grid, 32 * 16, zc_smem_bytes<32>(g.N3), st>>>(a);
  else k_z_step_c<16, true><<<grid, 16 * 16, zc_smem_bytes<16>(g.N3), st>>>(a);
  return 1;
}

int prepare_zstep_c_kernels() {
  const int lim = 227 * 1024;
  cudaError_t e = cudaFuncSetAttribute(k_z_step_c<16, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_z_step_c<32, true>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  return e == cudaSuccess ? 0 : -1;
}

}  // namespace sf
