// sf_remove_divergence_noalloc: the pressure projection (RemoveDivergence,
// IMEXRK.cpp:43-73) for callers that cannot allocate device memory.
//
// Who needs it: code that runs where cudaMalloc is not available or not
// allowed — a host that hands this library only pre-sized buffers from its
// own arena or pool, a real-time loop that must never enter the allocator
// after start-up, or a host framework that forbids allocation inside its
// callbacks. Such a caller cannot create an sf_solver (sf_create allocates
// its state, factors and scratch), but it can still project a velocity field
// it owns onto the divergence-free space with this one entry point.
//
// How it avoids allocation: everything the projection needs besides the
// caller's fields — the per-level grid coefficients, the Thomas factors of
// the Laplacian and the forward-sweep values of the solve — lives in the
// fixed-size array g_na_scratch below, a file-scope __device__ array that
// every GPU which loads this library holds until the process exits. The
// Laplacian factors are recomputed in FP64 inside the solve instead of being
// stored per mode, and the grid coefficients are computed on the device from
// N3 and L3, so no host-to-device copy is needed either.
//
// Limits and sharing: at most kNaMaxModeLevels = N3 * plane = 131072 complex
// values per call and N3 <= 1024, where plane = roundup(K1*K2, 16) is the
// kept modes of one level (a 2D grid of 256 x 1 x 1024 fits, as do
// 512 x 1 x 744 and the 3D grid 64 x 32 x 320); larger grids are rejected
// with SF_EINVAL. All calls on a device share the one array, which keeps the
// last call's contents; nothing in it has to start at zero (every value is
// written before it is read within a call). Calls whose GPU work overlaps — on two streams, or from two threads
// — race on that array and must be serialised by the caller.

#include <cuda_runtime.h>

#include <cmath>
#include <mutex>
#include <string>

#include "../../include/stratiflow_b200.h"
#include "sf_internal.cuh"

namespace sf {

constexpr int kNaMaxModeLevels = 131072;   // N3 * plane complex values per call
constexpr int kNaMaxN3 = 1024;
constexpr size_t kNaDBytes = sizeof(float2) * kNaMaxModeLevels;   // forward-sweep D_j
constexpr size_t kNaCBytes = sizeof(float) * kNaMaxModeLevels;    // Thomas factors C_j
constexpr int kNaCoef = 7;                                        // per-level FP64 arrays
constexpr size_t kNaCoefBytes = sizeof(double) * kNaCoef * kNaMaxN3;
constexpr size_t kNaKBytes = sizeof(float) * 2 * kMaxN;                  // kx, ky
constexpr size_t kNaScratchBytes = 2u << 20;   // 2 MiB
// layout: D_j | C_j | FP64 per-level coefficients | kx, ky
static_assert(kNaDBytes + kNaCBytes + kNaCoefBytes + kNaKBytes <= kNaScratchBytes, "scratch layout");

static __device__ __align__(256) unsigned char g_na_scratch[kNaScratchBytes];

enum { NA_LO, NA_DI, NA_UP, NA_DDN_DI, NA_DDN_UP, NA_DND_LO, NA_DND_DI };

// stretched grid of Field.cpp:3-83 in FP64, point by point
__device__ double na_zraw(int i, int N, double L) {   // before the rescaling, i >= 1
  double step = 2.0 / (double)(N - 2);
  double x = (i - 1 == N - 2) ? 1.0 : -1.0 + (i - 1) * step;
  return L * (2.0 * pow(x, 7.0) + x) / 3.0;
}
__device__ double na_z(int i, int N, double L) {
  double off = (na_zraw(1, N, L) + na_zraw(2, N, L)) / 2;
  return na_zraw(i, N, L) * (-L / off);
}
__device__ double na_zf_inner(int i, int N, double L) { return 0.5 * (na_z(i, N, L) + na_z(i + 1, N, L)); }
__device__ double na_zf(int i, int N, double L) {
  if (i == 0) return 2 * na_zf_inner(1, N, L) - na_zf_inner(2, N, L);
  if (i == N - 1) return 2 * na_zf_inner(N - 2, N, L) - na_zf_inner(N - 3, N, L);
  return na_zf_inner(i, N, L);
}
__device__ double na_DY(int i, int N, double L) { return na_zf(i, N, L) - na_zf(i - 1, N, L); }
__device__ double na_DYF(int i, int N, double L) {
  if (i == 0) i = 1;
  if (i == N - 1) i = N - 2;
  return na_z(i + 1, N, L) - na_z(i, N, L);
}

// per-level coefficients of Differentiation.cpp:6-61, one thread per level
__global__ void k_na_grid(int N, double L, double* __restrict__ coef) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= N) return;
  double lo = 0, di = 0, up = 0, ddi = 0, dup = 0, nlo = 0, ndi = 0;
  if (j >= 1 && j <= N - 2) {
    double DYj = na_DY(j, N, L), DYj1 = na_DY(j + 1, N, L), DYFj = na_DYF(j, N, L);
    lo = 1 / DYj / DYFj;
    di = -1 / DYj / DYFj - 1 / DYj1 / DYFj;
    up = 1 / DYj1 / DYFj;
  }
  if (j >= 1) {
    ddi = -1 / na_DYF(j, N, L);
    if (j < N - 1) dup = 1 / na_DYF(j, N, L);
  }
  if (j >= 2) {
    nlo = -1 / na_DY(j, N, L);
    ndi = 1 / na_DY(j, N, L);
  }
  coef[NA_LO * kNaMaxN3 + j] = lo;
  coef[NA_DI * kNaMaxN3 + j] = di;
  coef[NA_UP * kNaMaxN3 + j] = up;
  coef[NA_DDN_DI * kNaMaxN3 + j] = ddi;
  coef[NA_DDN_UP * kNaMaxN3 + j] = dup;
  coef[NA_DND_LO * kNaMaxN3 + j] = nlo;
  coef[NA_DND_DI * kNaMaxN3 + j] = ndi;
}

// The projection of k_z_proj_chunked on caller-owned fields [N3][plane] with the
// solve's scratch in the fixed array: the Laplacian rows (IMEXRK.h:55-78 with
// Neumannify) are factorised in FP64 during the forward sweep; D_j and C_j
// go to the scratch for the backward sweep. Thread per (mode, component);
// the two components of a mode are adjacent lanes and exchange q. No thread
// leaves before the shuffles.
__global__ void __launch_bounds__(128) k_na_proj(int N3, int K1, int Ky, int K2, int P, int Pp, int dim3,
                                                 double L1, double L2, const float* kx, const float* ky,
                                                 float* u1, float* u2, float* u3, const float* pin, float* pout,
                                                 float pm, unsigned char* scratch) {
  const int t = blockIdx.x * blockDim.x + threadIdx.x;
  const bool act = (t >> 1) < P;
  const int m = act ? (t >> 1) : 0, c = t & 1;
  const int kyint = (m / K1) < Ky ? (m / K1) : (m / K1) - K2;
  const int q = m / K1, j1 = m - q * K1;
  const float kxv = kx[j1], kyv = dim3 ? ky[q] : 0.f;
  // the factor rows use the FP64 wavenumbers (Differentiation.cpp:134-160)
  const double kxd = j1 * (2 * 3.141592653589793238462) / L1;
  const double kyd = dim3 ? kyint * (2 * 3.141592653589793238462) / L2 : 0.0;
  const double kk = -(kxd * kxd) + -(kyd * kyd);
  const float sc = c == 0 ? -1.f : 1.f;
  // D_j of this mode and component: [j][2*Pp] floats, mode m at 2m + c
  float* Dst = reinterpret_cast<float*>(scratch) + 2 * (size_t)m + c;
  float* Cst = reinterpret_cast<float*>(scratch + kNaDBytes);         // C_j
  const double* coef = reinterpret_cast<const double*>(scratch + kNaDBytes + kNaCBytes);
  const size_t s2 = 2 * (size_t)Pp;
  const float* u1o = u1 + 2 * (size_t)m + (1 - c);
  const float* u2o = dim3 ? u2 + 2 * (size_t)m + (1 - c) : nullptr;
  float* u1c = u1 + 2 * (size_t)m + c;
  float* u2c = dim3 ? u2 + 2 * (size_t)m + c : nullptr;
  float* u3c = u3 + 2 * (size_t)m + c;
  const float* pc = pin + 2 * (size_t)m + c;
  float* po = pout + 2 * (size_t)m + c;

  double Cprev = 0.0;
  float Dprev = 0.f;
  float w0 = u3c[0];
  for (int j = 0; j < N3; j++) {
    double aj = coef[NA_LO * kNaMaxN3 + j], bj = coef[NA_DI * kNaMaxN3 + j] + kk, cj = coef[NA_UP * kNaMaxN3 + j];
    if (j == 0) { bj = 1; cj = 0; }
    if (j == 1) { aj = 0; bj = 1; cj = (m == 0) ? 0.0 : -1.0; }   // (0,0) mode pinned
    if (j == N3 - 2) { aj = 1; bj = -1; cj = 0; }
    if (j == N3 - 1) { aj = 0; bj = 1; cj = 0; }
    if (j == 0) aj = 0;
    const double den = bj - aj * Cprev;
    Cprev = cj / den;
    // C_j as the step sequence uses it: float(c_j) * float(1/den_j)
    const float Cf = (float)cj * (float)(1.0 / den);
    const float w1 = (j + 1 < N3) ? u3c[(size_t)(j + 1) * s2] : 0.f;
    float dv = 0.f;
    if (j >= 2 && j <= N3 - 3) {
      const float a1 = u1o[(size_t)j * s2], a2 = dim3 ? u2o[(size_t)j * s2] : 0.f;
      dv = sc * (kxv * a1 + kyv * a2) +
           ((float)coef[NA_DDN_DI * kNaMaxN3 + j] * w0 + (float)coef[NA_DDN_UP * kNaMaxN3 + j] * w1);
    }
    const float inv = (float)(1.0 / den);
    const float D = (j == 0) ? dv * inv : (dv - (float)aj * Dprev) * inv;
    if (act) {
      Dst[(size_t)j * s2] = D;
      if (c == 0) Cst[(size_t)j * Pp + m] = Cf;
    }
    Dprev = D;
    w0 = w1;
  }
  __syncwarp();
  float qn = Dprev;   // q_{N3-1}
  {
    const int j = N3 - 1;
    const float qo = __shfl_xor_sync(0xffffffffu, qn, 1);
    if (act) {
      u1c[(size_t)j * s2] -= sc * kxv * qo;
      if (dim3) u2c[(size_t)j * s2] -= sc * kyv * qo;
      po[(size_t)j * s2] = pc[(size_t)j * s2] + pm * qn;
    }
  }
  for (int j = N3 - 2; j >= 0; j--) {
    const float Cj = Cst[(size_t)j * Pp + m];
    const float qj = Dst[(size_t)j * s2] - Cj * qn;
    const float qo = __shfl_xor_sync(0xffffffffu, qj, 1);
    if (act) {
      u1c[(size_t)j * s2] -= sc * kxv * qo;
      if (dim3) u2c[(size_t)j * s2] -= sc * kyv * qo;
      po[(size_t)j * s2] = pc[(size_t)j * s2] + pm * qj;
      const int jj = j + 1;   // u3_{j+1} -= ddz(q)_{j+1}, rows 2..N3-1
      if (jj >= 2)
        u3c[(size_t)jj * s2] -= (float)coef[NA_DND_LO * kNaMaxN3 + jj] * qj +
                                (float)coef[NA_DND_DI * kNaMaxN3 + jj] * qn;
    }
    qn = qj;
  }
}

// wavenumbers (Differentiation.cpp:113-160) of the kept modes, into the
// tail of the coefficient block
__global__ void k_na_wavenumbers(int N1, int N2, int K1, int K2, int Ky, double L1, double L2, float* kx,
                                 float* ky) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const double pi = 3.141592653589793238462;
  if (i < K1) kx[i] = (float)(i * (2 * pi) / L1);
  if (i < K2) {
    int kyint = N2 > 1 ? (i < Ky ? i : i - K2) : 0;
    ky[i] = N2 > 1 ? (float)(kyint * (2 * pi) / L2) : 0.f;
  }
}

static std::mutex g_na_mu;
static void* g_na_ptr[64] = {nullptr};

// device address of g_na_scratch on the current device, looked up once
static int na_scratch(void** out, std::string& err) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) { err = std::string("cudaGetDevice: ") + cudaGetErrorString(e); return SF_ECUDA; }
  if (dev < 0 || dev >= 64) { err = "device index out of range"; return SF_EINVAL; }
  std::lock_guard<std::mutex> lk(g_na_mu);
  if (!g_na_ptr[dev]) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_na_scratch);
    if (e != cudaSuccess || !p) {
      err = std::string("cudaGetSymbolAddress(g_na_scratch): ") + cudaGetErrorString(e);
      return SF_ECUDA;
    }
    g_na_ptr[dev] = p;
  }
  *out = g_na_ptr[dev];
  return SF_OK;
}

}  // namespace sf

using namespace sf;

// message storage shared with sf_last_error (sf_solver.cu)
extern void sf_set_error_message(const std::string& msg);

extern "C" int sf_remove_divergence_noalloc(const sf_grid* grid, const sf_flow* flow, double pressure_multiplier,
                                            void* u1, void* u2, void* u3, const void* p_in, void* p_out,
                                            void* stream) {
  auto bad = [](int code, const std::string& m) { sf_set_error_message(m); return code; };
  if (!grid || !flow || !u1 || !u3 || !p_in || !p_out) return bad(SF_EINVAL, "null argument");
  const int N1 = grid->N1, N2 = grid->N2, N3 = grid->N3;
  auto pow2 = [](int n) { return n > 0 && (n & (n - 1)) == 0; };
  if (grid->nrun != 1) return bad(SF_EINVAL, "sf_remove_divergence_noalloc projects one run (nrun must be 1)");
  if (!pow2(N1) || N1 < 16 || N1 > kMaxN || !(N2 == 1 || (pow2(N2) && N2 >= 16 && N2 <= 256)) || N3 % 4 != 0 ||
      N3 < 16)
    return bad(SF_EINVAL, "bad grid (N1, N2 powers of two; N3 % 4 == 0)");
  if (N2 > 1 && !u2) return bad(SF_EINVAL, "u2 is required in 3D");
  const int dim3 = N2 > 1;
  const int K1 = N1 / 3, Ky = dim3 ? N2 / 3 : 1, K2 = dim3 ? 2 * (N2 / 3) - 1 : 1;
  const int P = K1 * K2, Pp = (P + 15) / 16 * 16;
  if (N3 > kNaMaxN3 || (long long)N3 * Pp > kNaMaxModeLevels)
    return bad(SF_EINVAL, "grid too large for sf_remove_divergence_noalloc: N3*plane = " +
                              std::to_string((long long)N3 * Pp) + " > " + std::to_string(kNaMaxModeLevels) +
                              " or N3 > " + std::to_string(kNaMaxN3) + "; use sf_create + sf_remove_divergence");
  void* scratch = nullptr;
  std::string err;
  int rc = na_scratch(&scratch, err);
  if (rc != SF_OK) return bad(rc, err);
  cudaStream_t st = (cudaStream_t)stream;
  unsigned char* sc = static_cast<unsigned char*>(scratch);
  double* coef = reinterpret_cast<double*>(sc + kNaDBytes + kNaCBytes);
  float* kx = reinterpret_cast<float*>(sc + kNaDBytes + kNaCBytes + kNaCoefBytes);
  float* ky = kx + kMaxN;
  k_na_grid<<<(N3 + 255) / 256, 256, 0, st>>>(N3, flow->L3, coef);
  k_na_wavenumbers<<<1, kMaxN, 0, st>>>(N1, N2, K1, K2, Ky, flow->L1, flow->L2, kx, ky);
  k_na_proj<<<(2 * P + 127) / 128, 128, 0, st>>>(N3, K1, Ky, K2, P, Pp, dim3, flow->L1, flow->L2, kx, ky,
                                                  (float*)u1, (float*)u2, (float*)u3, (const float*)p_in,
                                                  (float*)p_out, (float)pressure_multiplier, sc);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return bad(SF_ECUDA, std::string("launch: ") + cudaGetErrorString(e));
  return SF_OK;
}
