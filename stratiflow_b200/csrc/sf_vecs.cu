// Device-resident state vectors: the algebra of the reference's StateVector
// (StateVector.h:40-149, 415-421) on states in the kept layout, with FP64
// reductions. Used by the Newton-Krylov, Arnoldi and continuation drivers,
// whose Krylov bases live on the device.
#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <string>
#include <vector>

#include "../../include/stratiflow_b200.h"
#include "sf_internal.cuh"

using namespace sf;

extern void sf_set_error_message(const std::string& msg);
// geometry and coefficient access of a solver (sf_solver.cu)
extern const Geo& sf_solver_geo(const sf_solver* s);
extern const float* sf_solver_zc(const sf_solver* s);
extern float2* sf_solver_state(sf_solver* s, int run);
extern cudaStream_t sf_solver_stream(const sf_solver* s);
extern const std::vector<double>& sf_solver_z(const sf_solver* s, int which);

struct sf_vecs {
  Geo g{};
  int nvec = 0;
  float2* d = nullptr;      // [nvec][5][N3][Pp]
  double* red = nullptr;    // reduction scratch
  int cap_red = 0;
  double* coef = nullptr;   // block-update coefficients
  size_t cap_coef = 0;
  const float* zc = nullptr;
  cudaStream_t st = nullptr;
  std::vector<double> z, zf;
};

namespace {

int vfail(int code, const std::string& m) {
  sf_set_error_message(m);
  return code;
}
#define VCK(call)                                                                              \
  do {                                                                                         \
    cudaError_t e__ = (call);                                                                  \
    if (e__ != cudaSuccess) return vfail(SF_ECUDA, std::string(#call) + ": " + cudaGetErrorString(e__)); \
  } while (0)

inline size_t vstride(const Geo& g) { return (size_t)5 * g.fblk; }   // complex elements per vector

// y += alpha x over u1,u2,u3,b of `count` consecutive vectors
// (StateVector::MulAdd, StateVector.h:67-78); f4 = 4 fields, vs = vector stride
__global__ void k_axpy(float2* __restrict__ y, const float2* __restrict__ x, float alpha, size_t f4, size_t vs,
                       int count) {
  const size_t n = f4 * count;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const size_t o = (i / f4) * vs + (i % f4);
    float2 a = x[o], b = y[o];
    y[o] = make_float2(b.x + alpha * a.x, b.y + alpha * a.y);
  }
}
// y = a y + b x over all five fields
__global__ void k_lincomb(float2* __restrict__ y, const float2* __restrict__ x, float a, float b, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    float2 u = y[i], v = x[i];
    y[i] = make_float2(a * u.x + b * v.x, a * u.y + b * v.y);
  }
}

// out[k] = sum over fields f of w_f * InnerProd(v_k.f, x_k'.f) (Integration.h:282-311)
// for k < count; v_k at base + k*stride, x_k' = x + k*xstride (xstride 0:
// every v_k against one x). With `sum`, all k accumulate into out[0].
// Block (level, k, field).
__global__ void k_dots(Geo g, const float2* __restrict__ base, size_t stride, const float2* __restrict__ x,
                       size_t xstride, const float* __restrict__ zc, double wb, double* out, int sum) {
  const int j = blockIdx.x, k = blockIdx.y, f = blockIdx.z;
  if (f == 1 && !g.dim3) return;
  const float2* a = base + k * stride + ((size_t)f * g.N3 + j) * g.Pp;
  const float2* b = x + k * xstride + ((size_t)f * g.N3 + j) * g.Pp;
  double s = 0.0;
  for (int m = threadIdx.x; m < g.P; m += blockDim.x) {
    float2 u = a[m], v = b[m];
    double t = (double)u.x * v.x + (double)u.y * v.y;
    s += (m == 0) ? t : 2.0 * t;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
    const double wz = zc[(f == 2 ? ZC_WZD : ZC_WZN) * g.N3 + j];
    const double wf = (f == 3) ? wb : 1.0;
    if (wz != 0.0) atomicAdd(out + (sum ? 0 : k), t * wz * wf);
  }
}

// Block Gram matrix: part[c][i][k] = the share of level chunk c (kGramLevels
// levels of one field) of Dot(V_i, W_k), i < nv, k < nw <= kMaxBlock. One
// warp per (chunk, field, i): lanes stride over the modes and keep one FP64
// sum per k; the partial sums are added in a fixed order afterwards.
constexpr int kGramLevels = 8;
constexpr int kMaxBlock = 32;

template <int NW>
__global__ void __launch_bounds__(256) k_gram(Geo g, const float2* __restrict__ V, int nv,
                                               const float2* __restrict__ W, int nw, size_t stride,
                                               const float* __restrict__ zc, double Ri, double* __restrict__ part) {
  const int chunk = blockIdx.x, f = blockIdx.y, warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int i = blockIdx.z * 8 + warp;
  if (i >= nv) return;
  const int nch = gridDim.x;
  double acc[NW];
#pragma unroll
  for (int k = 0; k < NW; k++) acc[k] = 0.0;
  if (f != 1 || g.dim3) {
    for (int j = chunk * kGramLevels; j < min(g.N3, (chunk + 1) * kGramLevels); j++) {
      const double wz = (double)zc[(f == 2 ? ZC_WZD : ZC_WZN) * g.N3 + j] * (f == 3 ? Ri : 1.0);
      if (wz == 0.0) continue;
      const size_t row = ((size_t)f * g.N3 + j) * g.Pp;
      const float2* v = V + (size_t)i * stride + row;
      for (int m = lane; m < g.P; m += 32) {
        const float2 a = v[m];
        const double wm = (m == 0) ? wz : 2.0 * wz;
#pragma unroll
        for (int k = 0; k < NW; k++) {
          if (k < nw) {
            const float2 b = W[(size_t)k * stride + row + m];
            acc[k] += wm * ((double)a.x * b.x + (double)a.y * b.y);
          }
        }
      }
    }
  }
#pragma unroll
  for (int k = 0; k < NW; k++) {
    double t = acc[k];
    for (int o = 16; o > 0; o >>= 1) t += __shfl_xor_sync(0xffffffffu, t, o);
    acc[k] = t;
  }
  if (lane == 0) {
    double* out = part + (((size_t)f * nch + chunk) * nv + i) * nw;
#pragma unroll
    for (int k = 0; k < NW; k++)
      if (k < nw) out[k] = acc[k];
  }
}

// out[i][k] = sum over the 4 * nch partials, in order
__global__ void k_gram_sum(const double* __restrict__ part, int nparts, int nvw, double* __restrict__ out) {
  const int e = blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nvw) return;
  double s = 0.0;
  for (int c = 0; c < nparts; c++) s += part[(size_t)c * nvw + e];
  out[e] = s;
}

// W_k += alpha sum_i coef[i][k] V_i over u1,u2,u3,b, k < nw <= kMaxBlock
template <int NW>
__global__ void k_update(Geo g, float2* __restrict__ W, int nw, const float2* __restrict__ V, int nv, size_t stride,
                         const double* __restrict__ coef, double alpha) {
  const size_t n = (size_t)4 * g.fblk;
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x) {
    float2 acc[NW];
#pragma unroll
    for (int k = 0; k < NW; k++) acc[k] = make_float2(0.f, 0.f);
    for (int i = 0; i < nv; i++) {
      const float2 v = V[(size_t)i * stride + e];
      const double* c = coef + (size_t)i * nw;
#pragma unroll
      for (int k = 0; k < NW; k++) {
        if (k < nw) {
          const float ck = (float)(alpha * c[k]);
          acc[k].x += ck * v.x;
          acc[k].y += ck * v.y;
        }
      }
    }
#pragma unroll
    for (int k = 0; k < NW; k++) {
      if (k < nw) {
        float2& w = W[(size_t)k * stride + e];
        w = make_float2(w.x + acc[k].x, w.y + acc[k].y);
      }
    }
  }
}

// keep field f of mode m only if bit f of fieldmask is set and lo <= j1 < hi;
// p is zeroed
__global__ void k_band(Geo g, float2* v, int fieldmask, int lo, int hi) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= g.Pp) return;
  const int j1 = m % g.K1;
  for (int f = 0; f < 5; f++) {
    const bool keep = f < 4 && ((fieldmask >> f) & 1) && j1 >= lo && j1 < hi && m < g.P;
    if (keep) continue;
    for (int j = 0; j < g.N3; j++) v[((size_t)f * g.N3 + j) * g.Pp + m] = make_float2(0.f, 0.f);
  }
}

// StateVector::EnforceBCs (StateVector.h:415-421): u3 ZeroEnds, u1,u2,b
// NeumannEnds, on the kept modes
__global__ void k_enforce_bcs(Geo g, float2* v) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= g.P) return;
  const int N3 = g.N3;
  auto at = [&](int f, int j) -> float2& { return v[((size_t)f * N3 + j) * g.Pp + m]; };
  const float2 z = make_float2(0.f, 0.f);
  at(2, 0) = z; at(2, 1) = z; at(2, 2) = z; at(2, N3 - 2) = z; at(2, N3 - 1) = z;
  for (int f : {0, 1, 3}) {
    at(f, 0) = at(f, 1);
    at(f, N3 - 1) = at(f, N3 - 2);
  }
}

// ModalField::PhaseShift (Field.h:1168-1174) on u1,u2,u3,b: mode j1 times e^{i j1 shift}
__global__ void k_phase(Geo g, float2* v, double shift) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= g.P) return;
  const int j1 = m % g.K1;
  double sn, cs;
  sincos(j1 * shift, &sn, &cs);
  const float c = (float)cs, s = (float)sn;
  for (int f = 0; f < 4; f++)
    for (int j = 0; j < g.N3; j++) {
      float2& a = v[((size_t)f * g.N3 + j) * g.Pp + m];
      const float2 b = a;
      a = make_float2(b.x * c - b.y * s, b.x * s + b.y * c);
    }
}

// subtract a real constant from the (0,0) mode of one field (RemoveAverage)
__global__ void k_sub_mean(Geo g, float2* v, int f, float value) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= g.N3) return;
  v[((size_t)f * g.N3 + j) * g.Pp].x -= value;
}

inline unsigned nb(size_t n, int t) {
  size_t b = (n + t - 1) / t;
  return (unsigned)(b > 4096 ? 4096 : b);
}

}  // namespace

extern "C" {

int sf_vecs_create(sf_solver* like, int nvec, sf_vecs** out) {
  if (!like || nvec < 1 || !out) return vfail(SF_EINVAL, "bad argument");
  sf_vecs* v = new sf_vecs();
  v->g = sf_solver_geo(like);
  v->nvec = nvec;
  v->zc = sf_solver_zc(like);
  v->st = sf_solver_stream(like);
  v->z = sf_solver_z(like, 0);
  v->zf = sf_solver_z(like, 1);
  cudaError_t e = cudaMalloc(&v->d, sizeof(float2) * vstride(v->g) * nvec);
  if (e == cudaSuccess) e = cudaMemsetAsync(v->d, 0, sizeof(float2) * vstride(v->g) * nvec, v->st);
  v->cap_red = nvec;
  if (e == cudaSuccess) e = cudaMalloc(&v->red, sizeof(double) * v->cap_red);
  if (e != cudaSuccess) {
    if (v->d) cudaFree(v->d);
    if (v->red) cudaFree(v->red);
    delete v;
    return vfail(e == cudaErrorMemoryAllocation ? SF_ENOMEM : SF_ECUDA, cudaGetErrorString(e));
  }
  *out = v;
  return SF_OK;
}

int sf_vecs_destroy(sf_vecs* v) {
  if (!v) return SF_OK;
  // no use of the solver's stream here: the solver may be gone already;
  // cudaFree waits for the device work that may still read the memory
  cudaFree(v->d);
  cudaFree(v->red);
  cudaFree(v->coef);
  delete v;
  return SF_OK;
}

int sf_vecs_count(sf_vecs* v, int* n) {
  if (!v || !n) return vfail(SF_EINVAL, "bad argument");
  *n = v->nvec;
  return SF_OK;
}

int sf_vecs_device(sf_vecs* v, int i, void** ptr) {
  if (!v || i < 0 || i >= v->nvec || !ptr) return vfail(SF_EINVAL, "bad argument");
  *ptr = v->d + (size_t)i * vstride(v->g);
  return SF_OK;
}

int sf_vecs_from_run(sf_vecs* v, int i, sf_solver* s, int run, int count) {
  if (!v || !s || count < 1 || i < 0 || i + count > v->nvec || run < 0 || run + count > sf_solver_geo(s).nrun)
    return vfail(SF_EINVAL, "bad argument");
  VCK(cudaStreamSynchronize(sf_solver_stream(s)));
  VCK(cudaMemcpyAsync(v->d + (size_t)i * vstride(v->g), sf_solver_state(s, run),
                      sizeof(float2) * vstride(v->g) * count, cudaMemcpyDeviceToDevice, v->st));
  return SF_OK;
}

int sf_vecs_to_run(sf_vecs* v, int i, sf_solver* s, int run, int count) {
  if (!v || !s || count < 1 || i < 0 || i + count > v->nvec || run < 0 || run + count > sf_solver_geo(s).nrun)
    return vfail(SF_EINVAL, "bad argument");
  VCK(cudaStreamSynchronize(v->st));
  VCK(cudaMemcpyAsync(sf_solver_state(s, run), v->d + (size_t)i * vstride(v->g),
                      sizeof(float2) * vstride(v->g) * count, cudaMemcpyDeviceToDevice, sf_solver_stream(s)));
  VCK(cudaStreamSynchronize(sf_solver_stream(s)));
  return SF_OK;
}

int sf_vecs_copy(sf_vecs* v, int dst, sf_vecs* w, int src) {
  if (!v || !w || dst < 0 || dst >= v->nvec || src < 0 || src >= w->nvec) return vfail(SF_EINVAL, "bad argument");
  VCK(cudaMemcpyAsync(v->d + (size_t)dst * vstride(v->g), w->d + (size_t)src * vstride(w->g),
                      sizeof(float2) * vstride(v->g), cudaMemcpyDeviceToDevice, v->st));
  return SF_OK;
}

int sf_vecs_set_host(sf_vecs* v, int i, const float* host) {
  if (!v || !host || i < 0 || i >= v->nvec) return vfail(SF_EINVAL, "bad argument");
  VCK(cudaMemcpyAsync(v->d + (size_t)i * vstride(v->g), host, sizeof(float2) * vstride(v->g), cudaMemcpyHostToDevice,
                      v->st));
  VCK(cudaStreamSynchronize(v->st));
  return SF_OK;
}

int sf_vecs_get_host(sf_vecs* v, int i, float* host) {
  if (!v || !host || i < 0 || i >= v->nvec) return vfail(SF_EINVAL, "bad argument");
  VCK(cudaMemcpyAsync(host, v->d + (size_t)i * vstride(v->g), sizeof(float2) * vstride(v->g), cudaMemcpyDeviceToHost,
                      v->st));
  VCK(cudaStreamSynchronize(v->st));
  return SF_OK;
}

// v[y+k] += alpha w[x+k] on u1,u2,u3,b for k < count (MulAdd)
int sf_vecs_axpy(sf_vecs* v, int y, double alpha, sf_vecs* w, int x, int count) {
  if (!v || !w || count < 1 || y < 0 || y + count > v->nvec || x < 0 || x + count > w->nvec)
    return vfail(SF_EINVAL, "bad argument");
  const size_t f4 = (size_t)4 * v->g.fblk, vs = vstride(v->g);
  k_axpy<<<nb(f4 * count, 256), 256, 0, v->st>>>(v->d + (size_t)y * vs, w->d + (size_t)x * vs, (float)alpha, f4, vs,
                                                  count);
  VCK(cudaGetLastError());
  return SF_OK;
}

// v[y+k] = a v[y+k] + b w[x+k] on all five fields, k < count
int sf_vecs_lincomb(sf_vecs* v, int y, double a, double b, sf_vecs* w, int x, int count) {
  if (!v || !w || count < 1 || y < 0 || y + count > v->nvec || x < 0 || x + count > w->nvec)
    return vfail(SF_EINVAL, "bad argument");
  size_t n = vstride(v->g) * count;
  k_lincomb<<<nb(n, 256), 256, 0, v->st>>>(v->d + (size_t)y * vstride(v->g), w->d + (size_t)x * vstride(v->g),
                                            (float)a, (float)b, n);
  VCK(cudaGetLastError());
  return SF_OK;
}

int sf_vecs_scale(sf_vecs* v, int i, double alpha, int count) {
  if (!v || count < 1 || i < 0 || i + count > v->nvec) return vfail(SF_EINVAL, "bad argument");
  return sf_vecs_lincomb(v, i, alpha, 0.0, v, i, count);
}

static int ensure_red(sf_vecs* v, int count) {
  if (count > v->cap_red) {
    cudaFree(v->red);
    v->cap_red = count;
    VCK(cudaMalloc(&v->red, sizeof(double) * count));
  }
  return SF_OK;
}

// out[k] = StateVector::Dot(v[first + k], w[x]) for k < count, FP64
int sf_vecs_dots(sf_vecs* v, int first, int count, sf_vecs* w, int x, double Ri, double* out) {
  if (!v || !w || !out || first < 0 || count < 1 || first + count > v->nvec || x < 0 || x >= w->nvec)
    return vfail(SF_EINVAL, "bad argument");
  int rc = ensure_red(v, count);
  if (rc) return rc;
  VCK(cudaMemsetAsync(v->red, 0, sizeof(double) * count, v->st));
  k_dots<<<dim3(v->g.N3, count, 4), 256, 0, v->st>>>(v->g, v->d + (size_t)first * vstride(v->g), vstride(v->g),
                                                     w->d + (size_t)x * vstride(w->g), 0, v->zc, Ri, v->red, 0);
  VCK(cudaGetLastError());
  VCK(cudaMemcpyAsync(out, v->red, sizeof(double) * count, cudaMemcpyDeviceToHost, v->st));
  VCK(cudaStreamSynchronize(v->st));
  return SF_OK;
}

// *out = sum_k Dot(v[a + k], w[b + k]) for k < count, FP64
int sf_vecs_dot_sum(sf_vecs* v, int a, sf_vecs* w, int b, int count, double Ri, double* out) {
  if (!v || !w || !out || count < 1 || a < 0 || a + count > v->nvec || b < 0 || b + count > w->nvec)
    return vfail(SF_EINVAL, "bad argument");
  int rc = ensure_red(v, 1);
  if (rc) return rc;
  VCK(cudaMemsetAsync(v->red, 0, sizeof(double), v->st));
  k_dots<<<dim3(v->g.N3, count, 4), 256, 0, v->st>>>(v->g, v->d + (size_t)a * vstride(v->g), vstride(v->g),
                                                     w->d + (size_t)b * vstride(w->g), vstride(w->g), v->zc, Ri,
                                                     v->red, 1);
  VCK(cudaGetLastError());
  VCK(cudaMemcpyAsync(out, v->red, sizeof(double), cudaMemcpyDeviceToHost, v->st));
  VCK(cudaStreamSynchronize(v->st));
  return SF_OK;
}

int sf_vecs_enforce_bcs(sf_vecs* v, int i, int count) {
  if (!v || count < 1 || i < 0 || i + count > v->nvec) return vfail(SF_EINVAL, "bad argument");
  for (int k = 0; k < count; k++)
    k_enforce_bcs<<<(v->g.P + 127) / 128, 128, 0, v->st>>>(v->g, v->d + (size_t)(i + k) * vstride(v->g));
  VCK(cudaGetLastError());
  return SF_OK;
}

// StateVector::RemovePhaseShift (StateVector.h:103-120): shift = pi/2 -
// arg(u1(1,0,N3/2)) unless `shift` is given (use_given != 0); returns it
int sf_vecs_phase_shift(sf_vecs* v, int i, int use_given, double* shift) {
  if (!v || !shift || i < 0 || i >= v->nvec) return vfail(SF_EINVAL, "bad argument");
  if (!use_given) {
    float2 h;
    const float2* p = v->d + (size_t)i * vstride(v->g) + (size_t)(v->g.N3 / 2) * v->g.Pp + 1;   // u1, j1=1, j2=0
    VCK(cudaMemcpyAsync(&h, p, sizeof(float2), cudaMemcpyDeviceToHost, v->st));
    VCK(cudaStreamSynchronize(v->st));
    *shift = -std::atan2((double)h.y, (double)h.x) + 3.141592653589793238462 / 2;
  }
  k_phase<<<(v->g.P + 127) / 128, 128, 0, v->st>>>(v->g, v->d + (size_t)i * vstride(v->g), *shift);
  VCK(cudaGetLastError());
  return SF_OK;
}

// RemoveAverage(field, L3) (Integration.h:236-240) for field 0 (u1) or 3 (b):
// subtract IntegrateVertically(real (0,0) stack)/(2 L3) from the (0,0) stack
int sf_vecs_remove_average(sf_vecs* v, int i, int field, double L3) {
  if (!v || i < 0 || i >= v->nvec || (field != 0 && field != 3)) return vfail(SF_EINVAL, "bad argument");
  const Geo& g = v->g;
  std::vector<float2> col(g.N3);
  const float2* base = v->d + (size_t)i * vstride(g) + (size_t)field * g.fblk;
  VCK(cudaMemcpy2DAsync(col.data(), sizeof(float2), base, sizeof(float2) * g.Pp, sizeof(float2), g.N3,
                        cudaMemcpyDeviceToHost, v->st));
  VCK(cudaStreamSynchronize(v->st));
  double integ = 0.0;   // Neumann quadrature (Integration.h:8-21)
  for (int k = 1; k < g.N3 - 1; k++) integ += (v->z[k + 1] - v->z[k]) * (double)col[k].x;
  const float value = (float)(integ / L3 / 2);
  k_sub_mean<<<(g.N3 + 127) / 128, 128, 0, v->st>>>(g, v->d + (size_t)i * vstride(g), field, value);
  VCK(cudaGetLastError());
  return SF_OK;
}

// out[i * nb + k] = Dot(v[a + i], w[b + k]) (StateVector::Dot, FP64)
int sf_vecs_gram(sf_vecs* v, int a, int na, sf_vecs* w, int b, int nb, double Ri, double* out) {
  if (!v || !w || !out || na < 1 || nb < 1 || nb > kMaxBlock || a < 0 || a + na > v->nvec || b < 0 ||
      b + nb > w->nvec)
    return vfail(SF_EINVAL, "bad argument (1 <= nb <= 32)");
  const Geo& g = v->g;
  const int nch = (g.N3 + kGramLevels - 1) / kGramLevels;
  const size_t nvw = (size_t)na * nb, parts = (size_t)4 * nch;
  int rc = ensure_red(v, (int)(nvw * (parts + 1)));
  if (rc) return rc;
  double* part = v->red + nvw;
  dim3 grid(nch, 4, (na + 7) / 8);
  auto* wd = w->d + (size_t)b * vstride(w->g);
  auto* vd = v->d + (size_t)a * vstride(g);
  const size_t vs = vstride(g);
  if (nb <= 1) k_gram<1><<<grid, 256, 0, v->st>>>(g, vd, na, wd, nb, vs, v->zc, Ri, part);
  else if (nb <= 4) k_gram<4><<<grid, 256, 0, v->st>>>(g, vd, na, wd, nb, vs, v->zc, Ri, part);
  else if (nb <= 8) k_gram<8><<<grid, 256, 0, v->st>>>(g, vd, na, wd, nb, vs, v->zc, Ri, part);
  else if (nb <= 16) k_gram<16><<<grid, 256, 0, v->st>>>(g, vd, na, wd, nb, vs, v->zc, Ri, part);
  else k_gram<32><<<grid, 256, 0, v->st>>>(g, vd, na, wd, nb, vs, v->zc, Ri, part);
  VCK(cudaGetLastError());
  k_gram_sum<<<(unsigned)((nvw + 255) / 256), 256, 0, v->st>>>(part, (int)parts, (int)nvw, v->red);
  VCK(cudaGetLastError());
  VCK(cudaMemcpyAsync(out, v->red, sizeof(double) * nvw, cudaMemcpyDeviceToHost, v->st));
  VCK(cudaStreamSynchronize(v->st));
  return SF_OK;
}

// w[b + k] += alpha sum_i coef[i * nb + k] v[a + i] on u1..b (v and w ranges
// must not overlap)
int sf_vecs_update(sf_vecs* w, int b, int nb, double alpha, sf_vecs* v, int a, int na, const double* coef) {
  if (!v || !w || !coef || na < 1 || nb < 1 || nb > kMaxBlock || a < 0 || a + na > v->nvec || b < 0 ||
      b + nb > w->nvec)
    return vfail(SF_EINVAL, "bad argument (1 <= nb <= 32)");
  if (v == w && a < b + nb && b < a + na) return vfail(SF_EINVAL, "overlapping ranges");
  const size_t nc = (size_t)na * nb;
  if (nc > w->cap_coef) {
    cudaFree(w->coef);
    w->coef = nullptr;
    w->cap_coef = 0;
    VCK(cudaMalloc(&w->coef, sizeof(double) * nc));
    w->cap_coef = nc;
  }
  VCK(cudaMemcpyAsync(w->coef, coef, sizeof(double) * nc, cudaMemcpyHostToDevice, w->st));
  const Geo& g = w->g;
  const size_t n = (size_t)4 * g.fblk;
  const unsigned blocks = (unsigned)std::min<size_t>((n + 255) / 256, 4096);
  const size_t vs = vstride(g);
  float2* wd = w->d + (size_t)b * vs;
  const float2* vd = v->d + (size_t)a * vs;
  if (nb <= 1) k_update<1><<<blocks, 256, 0, w->st>>>(g, wd, nb, vd, na, vs, w->coef, alpha);
  else if (nb <= 4) k_update<4><<<blocks, 256, 0, w->st>>>(g, wd, nb, vd, na, vs, w->coef, alpha);
  else if (nb <= 8) k_update<8><<<blocks, 256, 0, w->st>>>(g, wd, nb, vd, na, vs, w->coef, alpha);
  else if (nb <= 16) k_update<16><<<blocks, 256, 0, w->st>>>(g, wd, nb, vd, na, vs, w->coef, alpha);
  else k_update<32><<<blocks, 256, 0, w->st>>>(g, wd, nb, vd, na, vs, w->coef, alpha);
  VCK(cudaGetLastError());
  return SF_OK;
}

// keep only the fields in field_mask (bit f: u1, u2, u3, b) and the modes
// with j1_lo <= j1 < j1_hi of vector i; p is zeroed
int sf_vecs_band(sf_vecs* v, int i, int field_mask, int j1_lo, int j1_hi) {
  if (!v || i < 0 || i >= v->nvec) return vfail(SF_EINVAL, "bad argument");
  k_band<<<(v->g.Pp + 127) / 128, 128, 0, v->st>>>(v->g, v->d + (size_t)i * vstride(v->g), field_mask, j1_lo, j1_hi);
  VCK(cudaGetLastError());
  return SF_OK;
}

// copy the z column of one mode of one field of vector i (N3 complex values)
// to the host (write = 0) or from it (write = 1)
int sf_vecs_column(sf_vecs* v, int i, int field, int mode, float* host, int write) {
  if (!v || !host || i < 0 || i >= v->nvec || field < 0 || field > 4 || mode < 0 || mode >= v->g.P)
    return vfail(SF_EINVAL, "bad argument");
  float2* col = v->d + (size_t)i * vstride(v->g) + (size_t)field * v->g.fblk + mode;
  const size_t pitch = sizeof(float2) * v->g.Pp;
  if (write) {
    VCK(cudaMemcpy2DAsync(col, pitch, host, sizeof(float2), sizeof(float2), v->g.N3, cudaMemcpyHostToDevice, v->st));
  } else {
    VCK(cudaMemcpy2DAsync(host, sizeof(float2), col, pitch, sizeof(float2), v->g.N3, cudaMemcpyDeviceToHost, v->st));
  }
  VCK(cudaStreamSynchronize(v->st));
  return SF_OK;
}

// zero the p field of vectors i..i+count-1
int sf_vecs_zero_pressure(sf_vecs* v, int i, int count) {
  if (!v || count < 1 || i < 0 || i + count > v->nvec) return vfail(SF_EINVAL, "bad argument");
  for (int k = 0; k < count; k++)
    VCK(cudaMemsetAsync(v->d + (size_t)(i + k) * vstride(v->g) + (size_t)4 * v->g.fblk, 0,
                        sizeof(float2) * v->g.fblk, v->st));
  return SF_OK;
}

int sf_vecs_synchronize(sf_vecs* v) {
  if (!v) return vfail(SF_EINVAL, "bad argument");
  VCK(cudaStreamSynchronize(v->st));
  return SF_OK;
}

}  // extern "C"
