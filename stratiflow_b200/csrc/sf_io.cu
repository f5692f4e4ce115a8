// Nodal fields of a solver's state: PopulateNodalVariables of one field
// (IMEXRK.h:141-162) read back in the reference's nodal layout, ToModal of
// a nodal field (Field.h:734-769, with Filter, Field.h:996-1021) into the
// state, and the velocity maxima of IMEXRK::CFL (IMEXRK.h:355-373). These
// serve .fields snapshots (IMEXRK.h:415-443) and the adaptive time step of
// FullEvolve (StateVector.cpp:3-84); they are called every hundred steps or
// once per file, not on the step's path.
#include <cuda_runtime.h>

#include <algorithm>
#include <cstring>
#include <string>
#include <vector>

#include "../../include/stratiflow_b200.h"
#include "sf_internal.cuh"

using namespace sf;

extern void sf_set_error_message(const std::string& msg);
extern const Geo& sf_solver_geo(const sf_solver* s);
extern float2* sf_solver_state(sf_solver* s, int run);
extern cudaStream_t sf_solver_stream(const sf_solver* s);
extern const float2* sf_solver_tw(const sf_solver* s);
extern const float* sf_solver_ubar(const sf_solver* s, int run);
extern void sf_solver_count_launches(sf_solver* s, int n);

namespace {

int iofail(int code, const std::string& m) {
  sf_set_error_message(m);
  return code;
}
#define ICK(call)                                                                                 \
  do {                                                                                            \
    cudaError_t e__ = (call);                                                                     \
    if (e__ != cudaSuccess) return iofail(SF_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e__)); \
  } while (0)

// max over all points of |nod + add[level]| (add may be null), as float bits
// (non-negative floats order like their bit patterns)
__global__ void k_nodal_absmax(const float* __restrict__ nod, const float* __restrict__ add, int N3,
                               size_t per_level, unsigned* out) {
  float m = 0.f;
  const size_t n = per_level * N3;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float v = nod[i] + (add ? add[i / per_level] : 0.f);
    m = fmaxf(m, fabsf(v));
  }
  for (int o = 16; o > 0; o >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, o));
  if ((threadIdx.x & 31) == 0) atomicMax(out, __float_as_uint(m));
}

// forward real transform along x of one nodal row per (level, y) (one warp):
// the kept modes k < K1, times `scale`
__global__ void k_fwd_x(Geo g, const float* __restrict__ nod, float2* __restrict__ out, long long stride_level,
                        long long stride_y, float scale, const float2* __restrict__ tw) {
  extern __shared__ float2 wsm[];
  const int t = blockIdx.x, y = blockIdx.y, lane = threadIdx.x;
  const float* src = nod + ((size_t)t * g.N2 + y) * g.N1;
  for (int x = lane; x < g.N1; x += 32) wsm[x] = make_float2(src[x], 0.f);
  __syncwarp();
  warp_fft(wsm, g.N1, g.logN1, tw, false, lane);
  float2* o = out + (size_t)t * stride_level + (size_t)y * stride_y;
  for (int k = lane; k < g.K1; k += 32) o[k] = make_float2(wsm[k].x * scale, wsm[k].y * scale);
}

// forward transform along y of the x-transformed rows [N3][N2][K1] per
// (level, kx) (one warp), the kept ky rows into the kept layout [N3][Pp]
__global__ void k_fwd_y(Geo g, const float2* __restrict__ mixed, float2* __restrict__ kept,
                        const float2* __restrict__ tw) {
  extern __shared__ float2 wsm[];
  const int t = blockIdx.x, j1 = blockIdx.y, lane = threadIdx.x;
  for (int y = lane; y < g.N2; y += 32) wsm[y] = mixed[((size_t)t * g.N2 + y) * g.K1 + j1];
  __syncwarp();
  warp_fft(wsm, g.N2, g.logN2, tw, false, lane);
  for (int q = lane; q < g.K2; q += 32) {
    const int n2 = q < g.Ky ? q : q + g.N2 - g.K2;
    kept[(size_t)t * g.Pp + (size_t)q * g.K1 + j1] = wsm[n2];
  }
}

// the nodal [N3][N2][N1] values of field f of one run's state
int nodal_of(sf_solver* s, int run, int f, float* nod, float* scratch) {
  const Geo& g = sf_solver_geo(s);
  const float2* src = sf_solver_state(s, run) + (size_t)f * g.fblk;
  sf_solver_count_launches(s, launch_base_nodal(g, src, f, nod, sf_solver_tw(s), scratch, sf_solver_stream(s)));
  ICK(cudaGetLastError());
  return SF_OK;
}

struct Scratch {
  float* nod = nullptr;
  float* mixed = nullptr;
  unsigned* mx = nullptr;
  ~Scratch() {
    cudaFree(nod);
    cudaFree(mixed);
    cudaFree(mx);
  }
};

int alloc(const Geo& g, Scratch& w) {
  if (cudaMalloc(&w.nod, sizeof(float) * (size_t)g.N3 * g.N2 * g.N1) != cudaSuccess)
    return iofail(SF_ENOMEM, "cudaMalloc nodal buffer");
  if (g.dim3 && cudaMalloc(&w.mixed, sizeof(float2) * g.mblk) != cudaSuccess)
    return iofail(SF_ENOMEM, "cudaMalloc mixed buffer");
  if (cudaMalloc(&w.mx, sizeof(unsigned) * 4) != cudaSuccess) return iofail(SF_ENOMEM, "cudaMalloc maxima");
  return SF_OK;
}

}  // namespace

extern "C" {

int sf_get_nodal(sf_solver* s, int run, int field, float* host) {
  if (!s || !host || field < 0 || field > 3) return iofail(SF_EINVAL, "bad argument");
  const Geo& g = sf_solver_geo(s);
  if (run < 0 || run >= g.nrun) return iofail(SF_EINVAL, "bad run");
  Scratch w;
  int rc = alloc(g, w);
  if (rc) return rc;
  const size_t n = (size_t)g.N3 * g.N2 * g.N1;
  if (field == 1 && !g.dim3) {
    std::fill(host, host + n, 0.f);
    return SF_OK;
  }
  rc = nodal_of(s, run, field, w.nod, w.mixed);
  if (rc) return rc;
  std::vector<float> h(n);
  ICK(cudaMemcpyAsync(h.data(), w.nod, sizeof(float) * n, cudaMemcpyDeviceToHost, sf_solver_stream(s)));
  ICK(cudaStreamSynchronize(sf_solver_stream(s)));
  // [N3][N2][N1] -> the reference's (N1 n2 + n1) N3 + n3 (Field.h:399-410)
  for (int t = 0; t < g.N3; t++)
    for (int y = 0; y < g.N2; y++)
      for (int x = 0; x < g.N1; x++)
        host[((size_t)g.N1 * y + x) * g.N3 + t] = h[((size_t)t * g.N2 + y) * g.N1 + x];
  return SF_OK;
}

int sf_set_nodal(sf_solver* s, int run, int field, const float* host) {
  if (!s || !host || field < 0 || field > 3) return iofail(SF_EINVAL, "bad argument");
  const Geo& g = sf_solver_geo(s);
  if (run < 0 || run >= g.nrun) return iofail(SF_EINVAL, "bad run");
  cudaStream_t st = sf_solver_stream(s);
  float2* dst = sf_solver_state(s, run) + (size_t)field * g.fblk;
  ICK(cudaMemsetAsync(dst, 0, sizeof(float2) * g.fblk, st));
  if (field == 1 && !g.dim3) return SF_OK;
  Scratch w;
  int rc = alloc(g, w);
  if (rc) return rc;
  const size_t n = (size_t)g.N3 * g.N2 * g.N1;
  std::vector<float> h(n);
  for (int t = 0; t < g.N3; t++)
    for (int y = 0; y < g.N2; y++)
      for (int x = 0; x < g.N1; x++)
        h[((size_t)t * g.N2 + y) * g.N1 + x] = host[((size_t)g.N1 * y + x) * g.N3 + t];
  ICK(cudaMemcpyAsync(w.nod, h.data(), sizeof(float) * n, cudaMemcpyHostToDevice, st));
  const float scale = 1.0f / ((float)g.N1 * (float)g.N2);   // ToModal's 1/(N1 N2) (Field.h:757)
  if (!g.dim3) {
    k_fwd_x<<<dim3(g.N3, 1), 32, sizeof(float2) * g.N1, st>>>(g, w.nod, dst, g.Pp, 0, scale, sf_solver_tw(s));
    sf_solver_count_launches(s, 1);
  } else {
    float2* mixed = reinterpret_cast<float2*>(w.mixed);
    k_fwd_x<<<dim3(g.N3, g.N2), 32, sizeof(float2) * g.N1, st>>>(g, w.nod, mixed, (long long)g.N2 * g.K1, g.K1,
                                                                  scale, sf_solver_tw(s));
    k_fwd_y<<<dim3(g.N3, g.K1), 32, sizeof(float2) * g.N2, st>>>(g, mixed, dst, sf_solver_tw(s));
    sf_solver_count_launches(s, 2);
  }
  ICK(cudaGetLastError());
  ICK(cudaStreamSynchronize(st));
  return SF_OK;
}

int sf_velocity_maxima(sf_solver* s, int run, double* out) {
  if (!s || !out) return iofail(SF_EINVAL, "bad argument");
  const Geo& g = sf_solver_geo(s);
  if (run < 0 || run >= g.nrun) return iofail(SF_EINVAL, "bad run");
  Scratch w;
  int rc = alloc(g, w);
  if (rc) return rc;
  cudaStream_t st = sf_solver_stream(s);
  ICK(cudaMemsetAsync(w.mx, 0, sizeof(unsigned) * 4, st));
  const size_t per_level = (size_t)g.N2 * g.N1;
  const unsigned blocks = (unsigned)std::min<size_t>((per_level * g.N3 + 255) / 256, 2048);
  for (int f = 0; f < 3; f++) {
    if (f == 1 && !g.dim3) continue;
    rc = nodal_of(s, run, f, w.nod, w.mixed);
    if (rc) return rc;
    // U1 + U_ (IMEXRK.h:359)
    k_nodal_absmax<<<blocks, 256, 0, st>>>(w.nod, f == 0 ? sf_solver_ubar(s, run) : nullptr, g.N3, per_level,
                                           w.mx + f);
    sf_solver_count_launches(s, 1);
    ICK(cudaGetLastError());
  }
  unsigned h[4];
  ICK(cudaMemcpyAsync(h, w.mx, sizeof(h), cudaMemcpyDeviceToHost, st));
  ICK(cudaStreamSynchronize(st));
  for (int f = 0; f < 3; f++) {
    float v;
    std::memcpy(&v, &h[f], sizeof(float));
    out[f] = v;
  }
  return SF_OK;
}

}  // extern "C"
