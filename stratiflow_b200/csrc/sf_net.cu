// The learned predictor of pseudo-arclength continuation: a stack of 1D
// convolutions along z over the spectral coefficients of converged branch
// states (no counterpart in the reference, whose predictor is the secant of
// PseudoArclength.cpp:33-61). Training and inference run on the tensor
// cores with BF16 operands and FP32 accumulation; master weights, gradients
// and the Adam moments stay FP32.
//
// Tensors are channel-last: an activation is [batch][Z][C] (BF16), the
// weights of a layer W[Cout][tap][Cin] (tap < 5, zero padding of 2 levels at
// both ends of z) followed by its bias[Cout]. Every contraction is one
// implicit GEMM, C[m][n] = sum_k A(m,k) B(n,k):
//   forward          m = co, n = (b,z),        k = (tap,ci)
//   backward data    m = ci, n = (b,z),        k = (tap,co)
//   backward weights m = co, n = (tap,ci),     k = (b,z)
// tiled 64 x 64 x 32 through shared memory, with warp tiles of 32 x 32 issued
// as mma.sync m16n8k16 (bf16 x bf16 -> f32).
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <random>
#include <string>
#include <vector>

#include "../../include/stratiflow_b200.h"

extern void sf_set_error_message(const std::string& msg);

namespace {

constexpr int kTaps = 5, kPad = 2;
constexpr int BM = 64, BN = 64, BK = 32, SK = BK + 8;   // shared rows padded by 16 bytes
constexpr int kGemmThreads = 128;

enum GemmMode { G_FWD = 0, G_BWD_DATA = 1, G_BWD_W = 2 };

struct ConvGemm {
  int mode;
  int B, Z, Cin, Cout;
  int M, N, K;
  const __nv_bfloat16* W;    // [Cout][tap][Cin]
  const __nv_bfloat16* X;    // layer input [B][Z][Cin]
  const __nv_bfloat16* dP;   // gradient of the pre-activation [B][Z][Cout]
  const float* bias;         // forward
  float* outF;               // FP32 result (forward output layer, dW)
  __nv_bfloat16* outB;       // BF16 result (activation, dP of the layer below)
  int relu;                  // forward: ReLU on the BF16 result
  const __nv_bfloat16* mask; // backward data: keep where mask > 0 (ReLU')
};

__device__ __forceinline__ __nv_bfloat16 a_at(const ConvGemm& p, int m, int k) {
  const __nv_bfloat16 zero = __float2bfloat16(0.f);
  if (m >= p.M || k >= p.K) return zero;
  switch (p.mode) {
    case G_FWD: return p.W[(size_t)m * p.K + k];
    case G_BWD_DATA: {
      const int tap = k / p.Cout, co = k - tap * p.Cout;
      return p.W[((size_t)co * kTaps + tap) * p.Cin + m];
    }
    default: return p.dP[(size_t)k * p.Cout + m];
  }
}

__device__ __forceinline__ __nv_bfloat16 b_at(const ConvGemm& p, int n, int k) {
  const __nv_bfloat16 zero = __float2bfloat16(0.f);
  if (n >= p.N || k >= p.K) return zero;
  switch (p.mode) {
    case G_FWD: {
      const int b = n / p.Z, z = n - b * p.Z, tap = k / p.Cin, ci = k - tap * p.Cin, zz = z + tap - kPad;
      return (zz < 0 || zz >= p.Z) ? zero : p.X[((size_t)b * p.Z + zz) * p.Cin + ci];
    }
    case G_BWD_DATA: {
      const int b = n / p.Z, z = n - b * p.Z, tap = k / p.Cout, co = k - tap * p.Cout, zz = z - tap + kPad;
      return (zz < 0 || zz >= p.Z) ? zero : p.dP[((size_t)b * p.Z + zz) * p.Cout + co];
    }
    default: {
      const int tap = n / p.Cin, ci = n - tap * p.Cin, b = k / p.Z, z = k - b * p.Z, zz = z + tap - kPad;
      return (zz < 0 || zz >= p.Z) ? zero : p.X[((size_t)b * p.Z + zz) * p.Cin + ci];
    }
  }
}

__device__ __forceinline__ void mma_bf16(float (&c)[4], const unsigned (&a)[4], const unsigned (&b)[2]) {
  asm volatile(
      "mma.sync.aligned.m16n8k16.row.col.f32.bf16.bf16.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(c[0]), "+f"(c[1]), "+f"(c[2]), "+f"(c[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b[0]), "r"(b[1]));
}

// One 64 x 64 tile of C per block; 4 warps of 32 x 32
__global__ void __launch_bounds__(kGemmThreads) k_conv_gemm(ConvGemm p) {
  __shared__ __align__(16) __nv_bfloat16 As[BM][SK];
  __shared__ __align__(16) __nv_bfloat16 Bs[BN][SK];
  const int m0 = blockIdx.y * BM, n0 = blockIdx.x * BN;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int wm = (warp >> 1) * 32, wn = (warp & 1) * 32;
  const int g = lane >> 2, t = lane & 3;
  // which index runs fastest across threads when a tile is loaded: the one
  // that is contiguous in memory for this operand
  const bool a_mfast = p.mode != G_FWD, b_nfast = p.mode == G_BWD_W;
  float acc[2][4][4] = {};
  for (int k0 = 0; k0 < p.K; k0 += BK) {
    for (int i = tid; i < BM * BK; i += kGemmThreads) {
      const int r = a_mfast ? i % BM : i / BK, c = a_mfast ? i / BM : i % BK;
      As[r][c] = a_at(p, m0 + r, k0 + c);
    }
    for (int i = tid; i < BN * BK; i += kGemmThreads) {
      const int r = b_nfast ? i % BN : i / BK, c = b_nfast ? i / BN : i % BK;
      Bs[r][c] = b_at(p, n0 + r, k0 + c);
    }
    __syncthreads();
#pragma unroll
    for (int kk = 0; kk < BK; kk += 16) {
      unsigned af[2][4], bf[4][2];
#pragma unroll
      for (int i = 0; i < 2; i++) {
        const int r = wm + i * 16 + g;
        af[i][0] = *reinterpret_cast<const unsigned*>(&As[r][kk + 2 * t]);
        af[i][1] = *reinterpret_cast<const unsigned*>(&As[r + 8][kk + 2 * t]);
        af[i][2] = *reinterpret_cast<const unsigned*>(&As[r][kk + 2 * t + 8]);
        af[i][3] = *reinterpret_cast<const unsigned*>(&As[r + 8][kk + 2 * t + 8]);
      }
#pragma unroll
      for (int j = 0; j < 4; j++) {
        const int c = wn + j * 8 + g;
        bf[j][0] = *reinterpret_cast<const unsigned*>(&Bs[c][kk + 2 * t]);
        bf[j][1] = *reinterpret_cast<const unsigned*>(&Bs[c][kk + 2 * t + 8]);
      }
#pragma unroll
      for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 4; j++) mma_bf16(acc[i][j], af[i], bf[j]);
    }
    __syncthreads();
  }
  // epilogue: c0,c1 at (row g, cols 2t, 2t+1), c2,c3 at (row g+8, ...)
#pragma unroll
  for (int i = 0; i < 2; i++)
#pragma unroll
    for (int j = 0; j < 4; j++)
#pragma unroll
      for (int e = 0; e < 4; e++) {
        const int m = m0 + wm + i * 16 + g + (e >= 2 ? 8 : 0);
        const int n = n0 + wn + j * 8 + 2 * t + (e & 1);
        if (m >= p.M || n >= p.N) continue;
        float v = acc[i][j][e];
        if (p.mode == G_FWD) {
          v += p.bias[m];
          const size_t o = (size_t)n * p.M + m;
          if (p.outF) p.outF[o] = v;
          if (p.outB) p.outB[o] = __float2bfloat16(p.relu ? fmaxf(v, 0.f) : v);
        } else if (p.mode == G_BWD_DATA) {
          const size_t o = (size_t)n * p.M + m;
          if (p.mask && !(__bfloat162float(p.mask[o]) > 0.f)) v = 0.f;
          if (p.outF) p.outF[o] = v;
          if (p.outB) p.outB[o] = __float2bfloat16(v);
        } else {
          p.outF[(size_t)m * p.N + n] = v;
        }
      }
}

__global__ void k_to_bf16(const float* __restrict__ x, __nv_bfloat16* __restrict__ y, size_t n) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x)
    y[i] = __float2bfloat16(x[i]);
}

// loss = mean (out - target)^2; dP = bf16(2 (out - target) / count)
__global__ void k_mse(const float* __restrict__ out, const float* __restrict__ tgt, __nv_bfloat16* __restrict__ dP,
                      size_t n, double* loss) {
  double s = 0.0;
  const float inv = 2.0f / (float)n;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float d = out[i] - tgt[i];
    s += (double)d * d;
    dP[i] = __float2bfloat16(inv * d);
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double tsum = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) tsum += red[w];
    atomicAdd(loss, tsum / (double)n);
  }
}

// dbias[co] = sum over (b,z) of dP[b][z][co]
__global__ void k_bias_grad(const __nv_bfloat16* __restrict__ dP, int rows, int C, float* __restrict__ db) {
  const int co = blockIdx.x * blockDim.x + threadIdx.x;
  if (co >= C) return;
  float s = 0.f;
  for (int r = 0; r < rows; r++) s += __bfloat162float(dP[(size_t)r * C + co]);
  db[co] = s;
}

// Adam (Kingma & Ba 2015) on the FP32 master weights; refreshes the BF16
// copy of each weight (biases stay FP32)
__global__ void k_adam(float* __restrict__ w, const float* __restrict__ gr, float* __restrict__ m1,
                       float* __restrict__ m2, size_t n, float lr, float b1, float b2, float c1, float c2,
                       float eps) {
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const float gv = gr[i];
    const float a = b1 * m1[i] + (1.f - b1) * gv, b = b2 * m2[i] + (1.f - b2) * gv * gv;
    m1[i] = a;
    m2[i] = b;
    w[i] -= lr * (a / c1) / (sqrtf(b / c2) + eps);
  }
}

unsigned blocks_for(size_t n, int t) {
  size_t b = (n + t - 1) / t;
  return (unsigned)(b > 8192 ? 8192 : (b < 1 ? 1 : b));
}

}  // namespace

struct sf_net {
  int nl = 0, Z = 0, maxb = 0;
  std::vector<int> ch;               // ch[0] inputs .. ch[nl] outputs
  std::vector<size_t> woff, boff;    // offsets of W_l and b_l in the parameter vector
  size_t nparam = 0;
  float *w = nullptr, *gr = nullptr, *m1 = nullptr, *m2 = nullptr;
  __nv_bfloat16* wb = nullptr;       // BF16 copy of the whole parameter vector
  std::vector<__nv_bfloat16*> act;   // act[l]: input of layer l, [maxb][Z][ch[l]]
  std::vector<__nv_bfloat16*> dP;    // dP[l]: gradient of layer l's pre-activation
  float* out = nullptr;              // [maxb][Z][ch[nl]]
  float* xin = nullptr;              // FP32 staging of the input
  float* tgt = nullptr;              // training targets
  int nb_data = 0;                   // samples held in act[0] / tgt
  double* loss = nullptr;
  long long t = 0;                   // Adam steps taken
  cudaStream_t st = nullptr;
};

namespace {

int nfail(int code, const std::string& m) {
  sf_set_error_message(m);
  return code;
}

#define NCK(x)                                                                       \
  do {                                                                               \
    cudaError_t e_ = (x);                                                            \
    if (e_ != cudaSuccess) return nfail(SF_ECUDA, std::string(#x) + ": " + cudaGetErrorString(e_)); \
  } while (0)

int gemm(sf_net* n, ConvGemm p) {
  switch (p.mode) {
    case G_FWD: p.M = p.Cout; p.N = p.B * p.Z; p.K = kTaps * p.Cin; break;
    case G_BWD_DATA: p.M = p.Cin; p.N = p.B * p.Z; p.K = kTaps * p.Cout; break;
    default: p.M = p.Cout; p.N = kTaps * p.Cin; p.K = p.B * p.Z; break;
  }
  dim3 grid((p.N + BN - 1) / BN, (p.M + BM - 1) / BM);
  k_conv_gemm<<<grid, kGemmThreads, 0, n->st>>>(p);
  NCK(cudaGetLastError());
  return SF_OK;
}

int forward(sf_net* n, int B, bool keep_out) {
  for (int l = 0; l < n->nl; l++) {
    ConvGemm p{};
    p.mode = G_FWD;
    p.B = B; p.Z = n->Z; p.Cin = n->ch[l]; p.Cout = n->ch[l + 1];
    p.W = n->wb + n->woff[l];
    p.X = n->act[l];
    p.bias = n->w + n->boff[l];
    const bool last = l == n->nl - 1;
    p.outF = last ? n->out : nullptr;
    p.outB = last ? nullptr : n->act[l + 1];
    p.relu = last ? 0 : 1;
    int rc = gemm(n, p);
    if (rc) return rc;
  }
  (void)keep_out;
  return SF_OK;
}

// gradients of the mean-square loss against n->tgt into n->gr
int backward(sf_net* n, int B) {
  const size_t nout = (size_t)B * n->Z * n->ch[n->nl];
  NCK(cudaMemsetAsync(n->loss, 0, sizeof(double), n->st));
  k_mse<<<blocks_for(nout, 256), 256, 0, n->st>>>(n->out, n->tgt, n->dP[n->nl - 1], nout, n->loss);
  for (int l = n->nl - 1; l >= 0; l--) {
    ConvGemm p{};
    p.B = B; p.Z = n->Z; p.Cin = n->ch[l]; p.Cout = n->ch[l + 1];
    p.W = n->wb + n->woff[l];
    p.X = n->act[l];
    p.dP = n->dP[l];
    p.mode = G_BWD_W;
    p.outF = n->gr + n->woff[l];
    int rc = gemm(n, p);
    if (rc) return rc;
    k_bias_grad<<<(p.Cout + 127) / 128, 128, 0, n->st>>>(n->dP[l], B * n->Z, p.Cout, n->gr + n->boff[l]);
    if (l > 0) {   // dP of layer l-1 = (W^T * dP_l) where its ReLU was active
      ConvGemm q = p;
      q.mode = G_BWD_DATA;
      q.outF = nullptr;
      q.outB = n->dP[l - 1];
      q.mask = n->act[l];
      rc = gemm(n, q);
      if (rc) return rc;
    }
  }
  NCK(cudaGetLastError());
  return SF_OK;
}

int refresh_bf16(sf_net* n) {
  k_to_bf16<<<blocks_for(n->nparam, 256), 256, 0, n->st>>>(n->w, n->wb, n->nparam);
  NCK(cudaGetLastError());
  return SF_OK;
}

int upload_input(sf_net* n, const float* x, int B) {
  const size_t nin = (size_t)B * n->Z * n->ch[0];
  NCK(cudaMemcpyAsync(n->xin, x, sizeof(float) * nin, cudaMemcpyHostToDevice, n->st));
  k_to_bf16<<<blocks_for(nin, 256), 256, 0, n->st>>>(n->xin, n->act[0], nin);
  NCK(cudaGetLastError());
  return SF_OK;
}

}  // namespace

extern "C" {

int sf_net_create(int nlayers, const int* channels, int Z, int max_batch, unsigned long long seed, void* stream,
                  sf_net** out) {
  if (!out || nlayers < 1 || nlayers > 16 || !channels || Z < 1 || max_batch < 1)
    return nfail(SF_EINVAL, "bad argument");
  for (int l = 0; l <= nlayers; l++)
    if (channels[l] < 1 || channels[l] % 8) return nfail(SF_EINVAL, "channel counts must be positive multiples of 8");
  sf_net* n = new sf_net();
  n->nl = nlayers;
  n->Z = Z;
  n->maxb = max_batch;
  n->ch.assign(channels, channels + nlayers + 1);
  n->st = (cudaStream_t)stream;
  for (int l = 0; l < nlayers; l++) {
    n->woff.push_back(n->nparam);
    n->nparam += (size_t)n->ch[l + 1] * kTaps * n->ch[l];
    n->boff.push_back(n->nparam);
    n->nparam += (size_t)n->ch[l + 1];
  }
  // He-normal weights (std sqrt(2 / fan_in)), zero biases, from the seed;
  // the output layer starts at zero so that an untrained net predicts no
  // correction
  std::vector<float> h(n->nparam, 0.f);
  std::mt19937_64 rng(seed);
  for (int l = 0; l < nlayers - 1; l++) {
    std::normal_distribution<float> nd(0.f, std::sqrt(2.f / (kTaps * n->ch[l])));
    for (size_t i = 0; i < (size_t)n->ch[l + 1] * kTaps * n->ch[l]; i++) h[n->woff[l] + i] = nd(rng);
  }
  auto bail = [&](const char* what) {
    sf_net_destroy(n);
    return nfail(SF_ENOMEM, what);
  };
  if (cudaMalloc(&n->w, sizeof(float) * n->nparam) != cudaSuccess) return bail("cudaMalloc weights");
  if (cudaMalloc(&n->gr, sizeof(float) * n->nparam) != cudaSuccess) return bail("cudaMalloc gradients");
  if (cudaMalloc(&n->m1, sizeof(float) * n->nparam) != cudaSuccess) return bail("cudaMalloc moments");
  if (cudaMalloc(&n->m2, sizeof(float) * n->nparam) != cudaSuccess) return bail("cudaMalloc moments");
  if (cudaMalloc(&n->wb, sizeof(__nv_bfloat16) * n->nparam) != cudaSuccess) return bail("cudaMalloc bf16 weights");
  n->act.assign(nlayers, nullptr);
  n->dP.assign(nlayers, nullptr);
  const size_t rows = (size_t)max_batch * Z;
  for (int l = 0; l < nlayers; l++) {
    if (cudaMalloc(&n->act[l], sizeof(__nv_bfloat16) * rows * n->ch[l]) != cudaSuccess) return bail("cudaMalloc act");
    if (cudaMalloc(&n->dP[l], sizeof(__nv_bfloat16) * rows * n->ch[l + 1]) != cudaSuccess) return bail("cudaMalloc dP");
  }
  if (cudaMalloc(&n->out, sizeof(float) * rows * n->ch[nlayers]) != cudaSuccess) return bail("cudaMalloc out");
  if (cudaMalloc(&n->tgt, sizeof(float) * rows * n->ch[nlayers]) != cudaSuccess) return bail("cudaMalloc targets");
  if (cudaMalloc(&n->xin, sizeof(float) * rows * n->ch[0]) != cudaSuccess) return bail("cudaMalloc input");
  if (cudaMalloc(&n->loss, sizeof(double)) != cudaSuccess) return bail("cudaMalloc loss");
  if (cudaMemcpy(n->w, h.data(), sizeof(float) * n->nparam, cudaMemcpyHostToDevice) != cudaSuccess ||
      cudaMemset(n->m1, 0, sizeof(float) * n->nparam) != cudaSuccess ||
      cudaMemset(n->m2, 0, sizeof(float) * n->nparam) != cudaSuccess ||
      cudaMemset(n->gr, 0, sizeof(float) * n->nparam) != cudaSuccess) {
    sf_net_destroy(n);
    return nfail(SF_ECUDA, "initialising the weights");
  }
  int rc = refresh_bf16(n);
  if (rc) {
    sf_net_destroy(n);
    return rc;
  }
  *out = n;
  return SF_OK;
}

int sf_net_destroy(sf_net* n) {
  if (!n) return SF_OK;
  for (auto p : n->act) cudaFree(p);
  for (auto p : n->dP) cudaFree(p);
  for (void* p : {(void*)n->w, (void*)n->gr, (void*)n->m1, (void*)n->m2, (void*)n->wb, (void*)n->out,
                  (void*)n->tgt, (void*)n->xin, (void*)n->loss})
    cudaFree(p);
  delete n;
  return SF_OK;
}

int sf_net_num_params(sf_net* n, long long* count) {
  if (!n || !count) return nfail(SF_EINVAL, "bad argument");
  *count = (long long)n->nparam;
  return SF_OK;
}

int sf_net_get_params(sf_net* n, float* host) {
  if (!n || !host) return nfail(SF_EINVAL, "bad argument");
  NCK(cudaMemcpyAsync(host, n->w, sizeof(float) * n->nparam, cudaMemcpyDeviceToHost, n->st));
  NCK(cudaStreamSynchronize(n->st));
  return SF_OK;
}

int sf_net_set_params(sf_net* n, const float* host) {
  if (!n || !host) return nfail(SF_EINVAL, "bad argument");
  NCK(cudaMemcpyAsync(n->w, host, sizeof(float) * n->nparam, cudaMemcpyHostToDevice, n->st));
  NCK(cudaMemsetAsync(n->m1, 0, sizeof(float) * n->nparam, n->st));
  NCK(cudaMemsetAsync(n->m2, 0, sizeof(float) * n->nparam, n->st));
  n->t = 0;
  int rc = refresh_bf16(n);
  if (rc) return rc;
  NCK(cudaStreamSynchronize(n->st));
  return SF_OK;
}

int sf_net_forward(sf_net* n, const float* x, int batch, float* y) {
  if (!n || !x || !y || batch < 1 || batch > n->maxb) return nfail(SF_EINVAL, "bad argument");
  int rc = upload_input(n, x, batch);
  if (!rc) rc = forward(n, batch, true);
  if (rc) return rc;
  n->nb_data = 0;   // act[0] no longer holds the training inputs
  NCK(cudaMemcpyAsync(y, n->out, sizeof(float) * batch * n->Z * n->ch[n->nl], cudaMemcpyDeviceToHost, n->st));
  NCK(cudaStreamSynchronize(n->st));
  return SF_OK;
}

int sf_net_set_data(sf_net* n, const float* x, const float* target, int batch) {
  if (!n || !x || !target || batch < 1 || batch > n->maxb) return nfail(SF_EINVAL, "bad argument");
  int rc = upload_input(n, x, batch);
  if (rc) return rc;
  NCK(cudaMemcpyAsync(n->tgt, target, sizeof(float) * batch * n->Z * n->ch[n->nl], cudaMemcpyHostToDevice,
                      n->st));
  n->nb_data = batch;
  return SF_OK;
}

int sf_net_gradient(sf_net* n, float* grad, double* loss) {
  if (!n || n->nb_data < 1) return nfail(SF_ESTATE, "sf_net_set_data first");
  int rc = forward(n, n->nb_data, true);
  if (!rc) rc = backward(n, n->nb_data);
  if (rc) return rc;
  if (grad) NCK(cudaMemcpyAsync(grad, n->gr, sizeof(float) * n->nparam, cudaMemcpyDeviceToHost, n->st));
  if (loss) NCK(cudaMemcpyAsync(loss, n->loss, sizeof(double), cudaMemcpyDeviceToHost, n->st));
  NCK(cudaStreamSynchronize(n->st));
  return SF_OK;
}

int sf_net_train(sf_net* n, int steps, double lr, double* losses) {
  if (!n || steps < 0) return nfail(SF_EINVAL, "bad argument");
  if (n->nb_data < 1) return nfail(SF_ESTATE, "sf_net_set_data first");
  const float b1 = 0.9f, b2 = 0.999f, eps = 1e-8f;
  for (int s = 0; s < steps; s++) {
    int rc = forward(n, n->nb_data, true);
    if (!rc) rc = backward(n, n->nb_data);
    if (rc) return rc;
    n->t++;
    const float c1 = 1.f - std::pow(b1, (float)n->t), c2 = 1.f - std::pow(b2, (float)n->t);
    k_adam<<<blocks_for(n->nparam, 256), 256, 0, n->st>>>(n->w, n->gr, n->m1, n->m2, n->nparam, (float)lr, b1, b2,
                                                           c1, c2, eps);
    rc = refresh_bf16(n);
    if (rc) return rc;
    if (losses) NCK(cudaMemcpyAsync(losses + s, n->loss, sizeof(double), cudaMemcpyDeviceToHost, n->st));
  }
  NCK(cudaStreamSynchronize(n->st));
  return SF_OK;
}

}  // extern "C"
