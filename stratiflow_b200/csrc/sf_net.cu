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
// issued as tcgen05.mma on 128 x 128 tiles with the accumulator in tensor
// memory (k_conv_gemm_tc).
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

// ---------------------------------------------------------------- tcgen05 --
// The implicit GEMMs on the 5th-generation tensor cores: a CTA of four
// warps computes a 128 x 128 tile of C with tcgen05.mma (kind::f16, BF16 x
// BF16 -> FP32) issued by one thread, the accumulator in tensor memory (128
// lanes x 128 FP32 columns), A and B staged in shared memory as 64-wide K
// slices in the K-major layout with the 128-byte swizzle: each row's 64
// elements are one 128-byte line whose 16-byte chunk c sits at c ^ (row % 8),
// 8-row groups 1024 bytes apart (SBO); an instruction's K = 16 is the next 32
// bytes of every row (the descriptor's start address advances by 32 bytes).
// The 16-byte operand loads of one row then fill one line without bank
// conflicts.
// Two shared-memory stages: the loads of K slice t + 1 overlap the MMAs of
// slice t, and an mbarrier that the MMAs' commit arrives on frees a stage.
// Every wait is bounded; a wait that runs out sets *err and the block skips
// to freeing its tensor memory.
constexpr int TM = 128, TN = 128, TK = 64, kTcThreads = 128;
constexpr int kTcStageElems = (TM + TN) * TK;                      // bf16 per stage
// two stages, plus room to align the first to the swizzle's 1024-byte period
constexpr size_t kTcSmem = sizeof(__nv_bfloat16) * 2 * kTcStageElems + 1024;
constexpr long long kTcSpin = 1ll << 26;                           // bounded mbarrier waits

__device__ __forceinline__ uint32_t smem_u32(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

// K-major shared-memory matrix descriptor (sm_100) of the 128-byte swizzle:
// start address and the byte offsets in 16-byte units (LBO 16 bytes, unused
// by this layout; SBO 1024 bytes between 8-row groups), descriptor version 1,
// layout type 2 (SWIZZLE_128B)
__device__ __forceinline__ uint64_t umma_desc_sw128(uint32_t addr) {
  return (uint64_t)((addr >> 4) & 0x3FFF) | (1ull << 16) | ((uint64_t)(1024 >> 4) << 32) | (1ull << 46) |
         (2ull << 61);
}

// instruction descriptor of kind::f16: D FP32, A and B BF16, both K-major,
// N and M of the instruction
__host__ __device__ constexpr uint32_t umma_idesc_bf16(int M, int N) {
  return (1u << 4) | (1u << 7) | (1u << 10) | ((uint32_t)(N >> 3) << 17) | ((uint32_t)(M >> 4) << 24);
}

__device__ __forceinline__ bool mbar_wait(uint64_t* bar, uint32_t phase) {
  const uint32_t a = smem_u32(bar);
  for (long long i = 0; i < kTcSpin; i++) {
    uint32_t done;
    asm volatile(
        "{\n\t.reg .pred p;\n\t"
        "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
        "selp.u32 %0, 1, 0, p;\n\t}"
        : "=r"(done)
        : "r"(a), "r"(phase)
        : "memory");
    if (done) return true;
  }
  return false;
}

// 8 consecutive BF16 operands as one 16-byte load, zeros outside the matrix.
// Channel counts are multiples of 8, so a run of 8 along the contiguous index
// never crosses a tap or a row, and every run starts on a 16-byte boundary.
__device__ __forceinline__ uint4 ld8(const __nv_bfloat16* p) { return *reinterpret_cast<const uint4*>(p); }
__device__ __forceinline__ uint4 zero8() { return make_uint4(0u, 0u, 0u, 0u); }

// A(m, k..k+7) where k is contiguous (forward: W[m][k])
__device__ __forceinline__ uint4 a_k8(const ConvGemm& p, int m, int k) {
  return (m < p.M && k < p.K) ? ld8(p.W + (size_t)m * p.K + k) : zero8();
}
// A(m..m+7, k) where m is contiguous (backward data: W[co][tap][m];
// backward weights: dP[k][m])
__device__ __forceinline__ uint4 a_m8(const ConvGemm& p, int m, int k) {
  if (m >= p.M || k >= p.K) return zero8();
  if (p.mode == G_BWD_DATA) {
    const int tap = k / p.Cout, co = k - tap * p.Cout;
    return ld8(p.W + ((size_t)co * kTaps + tap) * p.Cin + m);
  }
  return ld8(p.dP + (size_t)k * p.Cout + m);
}
// B(n, k..k+7) where k is contiguous (forward: X rows; backward data: dP rows)
__device__ __forceinline__ uint4 b_k8(const ConvGemm& p, int n, int k) {
  if (n >= p.N || k >= p.K) return zero8();
  const int b = n / p.Z, z = n - b * p.Z;
  if (p.mode == G_FWD) {
    const int tap = k / p.Cin, ci = k - tap * p.Cin, zz = z + tap - kPad;
    return (zz < 0 || zz >= p.Z) ? zero8() : ld8(p.X + ((size_t)b * p.Z + zz) * p.Cin + ci);
  }
  const int tap = k / p.Cout, co = k - tap * p.Cout, zz = z - tap + kPad;
  return (zz < 0 || zz >= p.Z) ? zero8() : ld8(p.dP + ((size_t)b * p.Z + zz) * p.Cout + co);
}
// B(n..n+7, k) where n is contiguous (backward weights: X rows at z + tap)
__device__ __forceinline__ uint4 b_n8(const ConvGemm& p, int n, int k) {
  if (n >= p.N || k >= p.K) return zero8();
  const int tap = n / p.Cin, ci = n - tap * p.Cin, b = k / p.Z, z = k - b * p.Z, zz = z + tap - kPad;
  return (zz < 0 || zz >= p.Z) ? zero8() : ld8(p.X + ((size_t)b * p.Z + zz) * p.Cin + ci);
}

// element (r, c) of a [rows][TK = 64] tile in the 128-byte-swizzled layout
__device__ __forceinline__ int tc_off(int r, int c) {
  return ((r >> 3) << 9) + ((r & 7) << 6) + ((((c >> 3) ^ (r & 7))) << 3) + (c & 7);
}

__global__ void __launch_bounds__(kTcThreads) k_conv_gemm_tc(ConvGemm p, int* err) {
  extern __shared__ __align__(128) unsigned char tsm[];
  // the stages start on a 1024-byte boundary (the swizzle pattern's period)
  __nv_bfloat16* stage0 = reinterpret_cast<__nv_bfloat16*>(tsm + ((1024 - (smem_u32(tsm) & 1023)) & 1023));
  __shared__ __align__(8) uint64_t mbar[2];
  __shared__ uint32_t tmem_base;
  __shared__ int failed;
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int m0 = blockIdx.y * TM, n0 = blockIdx.x * TN;
  const bool a_mfast = p.mode != G_FWD, b_nfast = p.mode == G_BWD_W;
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(smem_u32(&tmem_base)),
                 "r"(TN));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  if (tid == 0) {
    failed = 0;
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[0])));
    asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(smem_u32(&mbar[1])));
    asm volatile("fence.mbarrier_init.release.cluster;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const uint32_t tmem = tmem_base;
  const int nk = (p.K + TK - 1) / TK;
  uint32_t phase[2] = {0, 0};
  constexpr uint32_t idesc = umma_idesc_bf16(TM, TN);
  for (int kt = 0; kt < nk && !failed; kt++) {
    const int s = kt & 1, k0 = kt * TK;
    __nv_bfloat16* As = stage0 + (size_t)s * kTcStageElems;
    __nv_bfloat16* Bs = As + TM * TK;
    if (kt >= 2) {   // the MMAs of slice kt - 2 read this stage
      if (!mbar_wait(&mbar[s], phase[s])) {
        if (tid == 0) { failed = 1; atomicExch(err, 1); }
      }
      phase[s] ^= 1;
    }
    __syncthreads();
    if (failed) break;
    // one 16-byte load per thread and pass: a core-matrix row when K is the
    // contiguous index, else 8 rows of one K column
    // K contiguous: 8 threads load one row's 128 bytes and fill its line;
    // M or N contiguous: a thread loads 8 rows of one K column, and the
    // threads of a warp take consecutive columns (conflict-free stores)
    if (!a_mfast) {
      for (int i = tid; i < TM * (TK / 8); i += kTcThreads) {
        const int r = i / (TK / 8), c = 8 * (i % (TK / 8));
        *reinterpret_cast<uint4*>(&As[tc_off(r, c)]) = a_k8(p, m0 + r, k0 + c);
      }
    } else {
      for (int i = tid; i < (TM / 8) * TK; i += kTcThreads) {
        const int c = i % TK, r = 8 * (i / TK);
        const uint4 v = a_m8(p, m0 + r, k0 + c);
        const __nv_bfloat16* e = reinterpret_cast<const __nv_bfloat16*>(&v);
#pragma unroll
        for (int j = 0; j < 8; j++) As[tc_off(r + j, c)] = e[j];
      }
    }
    if (!b_nfast) {
      for (int i = tid; i < TN * (TK / 8); i += kTcThreads) {
        const int r = i / (TK / 8), c = 8 * (i % (TK / 8));
        *reinterpret_cast<uint4*>(&Bs[tc_off(r, c)]) = b_k8(p, n0 + r, k0 + c);
      }
    } else {
      for (int i = tid; i < (TN / 8) * TK; i += kTcThreads) {
        const int c = i % TK, r = 8 * (i / TK);
        const uint4 v = b_n8(p, n0 + r, k0 + c);
        const __nv_bfloat16* e = reinterpret_cast<const __nv_bfloat16*>(&v);
#pragma unroll
        for (int j = 0; j < 8; j++) Bs[tc_off(r + j, c)] = e[j];
      }
    }
    // the generic-proxy stores must be visible to the tensor cores' async proxy
    asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
    __syncthreads();
    if (tid == 0) {
      asm volatile("tcgen05.fence::after_thread_sync;");
      const uint32_t a0 = smem_u32(As), b0 = smem_u32(Bs);
#pragma unroll
      for (int kk = 0; kk < TK / 16; kk++) {
        // K = 16 per instruction: bytes 32 kk .. 32 kk + 31 of every row
        const uint64_t da = umma_desc_sw128(a0 + 32 * kk);
        const uint64_t db = umma_desc_sw128(b0 + 32 * kk);
        const uint32_t acc = (kt > 0 || kk > 0) ? 1u : 0u;
        asm volatile(
            "{\n\t.reg .pred p;\n\t"
            "setp.ne.b32 p, %4, 0;\n\t"
            "tcgen05.mma.cta_group::1.kind::f16 [%0], %1, %2, %3, p;\n\t}"
            ::"r"(tmem), "l"(da), "l"(db), "r"(idesc), "r"(acc));
      }
      asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];" ::"r"(
                       smem_u32(&mbar[s]))
                   : "memory");
    }
  }
  // the last commit covers every MMA issued before it
  if (!failed && nk > 0) {
    const int s = (nk - 1) & 1;
    if (!mbar_wait(&mbar[s], phase[s]) && tid == 0) { failed = 1; atomicExch(err, 1); }
  }
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  if (!failed) {
    // warp w reads tensor-memory lanes 32w..32w+31: row m0 + 32w + lane
    const int m = m0 + 32 * warp + lane;
    for (int c = 0; c < TN; c += 8) {
      uint32_t v[8];
      asm volatile(
          "tcgen05.ld.sync.aligned.32x32b.x8.b32 {%0, %1, %2, %3, %4, %5, %6, %7}, [%8];"
          : "=r"(v[0]), "=r"(v[1]), "=r"(v[2]), "=r"(v[3]), "=r"(v[4]), "=r"(v[5]), "=r"(v[6]), "=r"(v[7])
          : "r"(tmem + ((uint32_t)(32 * warp) << 16) + (uint32_t)c));
      asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
      if (m >= p.M) continue;
#pragma unroll
      for (int e = 0; e < 8; e++) {
        const int n = n0 + c + e;
        if (n >= p.N) break;
        float x = __uint_as_float(v[e]);
        if (p.mode == G_FWD) {
          x += p.bias[m];
          const size_t o = (size_t)n * p.M + m;
          if (p.outF) p.outF[o] = x;
          if (p.outB) p.outB[o] = __float2bfloat16(p.relu ? fmaxf(x, 0.f) : x);
        } else if (p.mode == G_BWD_DATA) {
          const size_t o = (size_t)n * p.M + m;
          if (p.mask && !(__bfloat162float(p.mask[o]) > 0.f)) x = 0.f;
          if (p.outF) p.outF[o] = x;
          if (p.outB) p.outB[o] = __float2bfloat16(x);
        } else {
          p.outF[(size_t)m * p.N + n] = x;
        }
      }
    }
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (warp == 0) asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(tmem), "r"(TN));
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
  int* err = nullptr;                // set by a GEMM block whose bounded wait ran out
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
  dim3 grid((p.N + TN - 1) / TN, (p.M + TM - 1) / TM);
  k_conv_gemm_tc<<<grid, kTcThreads, kTcSmem, n->st>>>(p, n->err);
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

// after a synchronisation: a GEMM whose tensor-core wait ran out is an error
static int net_status(sf_net* n) {
  int h = 0;
  NCK(cudaMemcpy(&h, n->err, sizeof(int), cudaMemcpyDeviceToHost));
  if (h) {
    NCK(cudaMemset(n->err, 0, sizeof(int)));
    return nfail(SF_ECUDA, "a tensor-core GEMM block gave up waiting for its MMAs");
  }
  return SF_OK;
}

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
  if (cudaMalloc(&n->err, sizeof(int)) != cudaSuccess) return bail("cudaMalloc status");
  if (cudaMemset(n->err, 0, sizeof(int)) != cudaSuccess ||
      cudaFuncSetAttribute(k_conv_gemm_tc, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kTcSmem) != cudaSuccess) {
    sf_net_destroy(n);
    return nfail(SF_ECUDA, "setting up the tensor-core GEMM");
  }
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
                  (void*)n->tgt, (void*)n->xin, (void*)n->loss, (void*)n->err})
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
  return net_status(n);
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
  return net_status(n);
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
  return net_status(n);
}

}  // extern "C"
