// IMEXRK::TimeStepAdjoint (IMEXRK.h:86-126) for 2D batches: per RK substep
// the direct state interpolated between the two given snapshots (with U_ in
// its u1), UpdateAdjointVariables (IMEXRK.h:461-500: the mixing objective's
// forcing with K = 2), BuildRHSAdjoint (IMEXRK.cpp:260-379) in one x pass,
// then the CN and pressure solves of the other steps without the linear
// buoyancy terms of BuildRHS.
//
// The x pass (one block per slab of S output levels and run): 12 nodal rows
// per level are formed by inverse transforms, two rows per complex FFT —
// the adjoint U1, U3, B; the direct U1T (+U_), U3T, BT; their x derivatives;
// ddz of u1T and bT (Neumann -> Dirichlet) and of u3T (Dirichlet ->
// Neumann), taken on the modal rows before the transform. Nine products
// follow, each forward-transformed (two per complex FFT): U1 U1T, Bar(U1) U3T,
// Tilde(U1T) U3, Dir(U3) Dir(U3T), Bar(B) U3T, B U1T and the three forcings;
// the z stencils and x derivatives give r1, r3, rB.
#include <cuda_runtime.h>

#include <algorithm>

#include "sf_fft.cuh"
#include "sf_internal.cuh"

namespace sf {

namespace {

// the direct state of the substep, (1 - frac) above + frac below, with U_
// added to the (0,0) mode of u1 (ToNodal, + U_, ToModal of IMEXRK.h:101-106)
__global__ void k_adj_direct(Geo g, const float2* __restrict__ below, const float2* __restrict__ above, float frac,
                             const float* __restrict__ Ubar, float2* __restrict__ out) {
  const size_t per_run = (size_t)4 * g.fblk;
  const size_t n = per_run * g.nrun;
  for (size_t i = blockIdx.x * (size_t)blockDim.x + threadIdx.x; i < n; i += (size_t)gridDim.x * blockDim.x) {
    const size_t r = i / per_run, e = i - r * per_run;
    const size_t f = e / g.fblk, w = e - f * g.fblk;
    const size_t src = r * 5 * g.fblk + f * g.fblk + w;
    const float2 a = above[src], b = below[src];
    float2 v = make_float2((1.f - frac) * a.x + frac * b.x, (1.f - frac) * a.y + frac * b.y);
    const int m = (int)(w % g.Pp), t = (int)(w / g.Pp);
    if (f == 0 && m == 0) v.x += Ubar[r * g.N3 + t];
    out[i] = v;
  }
}

// nodal rows
enum { R_U1, R_U3, R_B, R_U1T, R_U3T, R_BT, R_DXU1T, R_DXU3T, R_DXBT, R_DZU1T, R_DZU3T, R_DZBT, R_COUNT };
// products, in hat-row order
enum { Q_P1, Q_P2, Q_P3, Q_P4, Q_P5, Q_P6, Q_F1, Q_F3, Q_FB, Q_COUNT };

__host__ __device__ __forceinline__ void adj_slots(int p, int S, int& first, int& count) {
  if (p == Q_P2 || p == Q_P5) { first = 1; count = S + 1; }
  else if (p == Q_P4) { first = 0; count = S + 1; }
  else { first = 1; count = S; }
}
__host__ __device__ __forceinline__ int adj_row(int p, int s, int S) {
  int base = 0;
  for (int q = 0; q < p; q++) {
    int f, c;
    adj_slots(q, S, f, c);
    base += c;
  }
  int f, c;
  adj_slots(p, S, f, c);
  return base + s - f;
}
__host__ __device__ inline int adj_rows(int S) { return adj_row(Q_COUNT - 1, S, S) + 1; }

constexpr int kAdjGroups = 8;
inline int adiv(long long a, long long b) { return (int)((a + b - 1) / b); }

struct AdjLayout {
  size_t stg_off, nod_off, buf_off, avg_off, bytes;
};
__host__ __device__ inline AdjLayout adj_layout(int S, int N1, int K1, int bufstride) {
  AdjLayout L;
  const int NS = S + 2;
  size_t off = 0;
  const size_t stg = sizeof(float2) * (size_t)6 * NS * K1, hat = sizeof(float2) * (size_t)adj_rows(S) * K1;
  L.stg_off = off; off += stg > hat ? stg : hat;   // the staged rows, then the transformed products
  L.nod_off = off; off += sizeof(float) * (size_t)R_COUNT * NS * N1;
  L.buf_off = off; off += sizeof(float2) * (size_t)kAdjGroups * bufstride;
  L.avg_off = off; off += sizeof(float) * (size_t)2 * NS;
  L.bytes = off;
  return L;
}

template <int N1>
__global__ void __launch_bounds__(kAdjGroups * 32) k_xpass_adj(StageArgs a, int S) {
  constexpr int G = FFTShape<N1>::G, E = FFTShape<N1>::E, BUF = fft_buf_stride<N1>();
  constexpr int NGB = kAdjGroups;
  const Geo g = a.g;
  extern __shared__ __align__(16) unsigned char xsm[];
  const AdjLayout L = adj_layout(S, N1, g.K1, BUF);
  float2* stg = reinterpret_cast<float2*>(xsm + L.stg_off);   // [6][NS][K1]: u1, u3, b, u1T, u3T, bT
  float2* hat = stg;
  float* nod = reinterpret_cast<float*>(xsm + L.nod_off);     // [R_COUNT][NS][N1]
  float* avg = reinterpret_cast<float*>(xsm + L.avg_off);     // [2][NS]: <bT>, <u3T>
  const int K1 = g.K1, N3 = g.N3, NS = S + 2;
  const int j0 = blockIdx.x * S;
  const int run = blockIdx.z;
  const int gid = threadIdx.x / G, l = threadIdx.x % G;
  float2* buf = reinterpret_cast<float2*>(xsm + L.buf_off) + (size_t)gid * BUF;
  const float* zc = a.zc;

  // ---- stage the modal rows of levels j0-1 .. j0+S ----
  for (int i = threadIdx.x; i < 6 * NS * K1; i += blockDim.x) {
    const int fb = i / (NS * K1), r = i - fb * NS * K1, s = r / K1, k = r - s * K1;
    const int t = j0 - 1 + s;
    float2 v = make_float2(0.f, 0.f);
    if (t >= 0 && t < N3) {
      if (fb < 3) {   // adjoint u1, u3, b (fields 0, 2, 3)
        const int f = fb == 0 ? 0 : fb + 1;
        v = a.S[((size_t)(run * 5 + f) * N3 + t) * g.Pp + k];
      } else {        // direct u1T, u3T, bT
        const int f = fb == 3 ? 0 : fb - 2;
        v = a.adir[((size_t)(run * 4 + f) * N3 + t) * g.Pp + k];
      }
    }
    stg[i] = v;
  }
  __syncthreads();
  auto SR = [&](int fb, int s) -> const float2* { return stg + ((size_t)fb * NS + s) * K1; };
  for (int s = threadIdx.x; s < NS; s += blockDim.x) {   // HorizontalAverage (Integration.h:38-42)
    avg[s] = SR(5, s)[0].x;
    avg[NS + s] = SR(4, s)[0].x;
  }

  // ---- phase A: 12 nodal rows per slot, two per inverse transform ----
  const int ntA = 6 * NS;
  for (int base = 0; base < ntA; base += NGB) {
    const int task = base + gid;
    const bool valid = task < ntA;
    const int s = valid ? task % NS : 0, pr = valid ? task / NS : 0;
    const int t = j0 - 1 + s;
    const bool tin = valid && t >= 0 && t < N3;
    int rA, rB;
    switch (pr) {
      case 0: rA = R_U1; rB = R_U3; break;
      case 1: rA = R_B; rB = R_DZBT; break;
      case 2: rA = R_U1T; rB = R_U3T; break;
      case 3: rA = R_BT; rB = R_DXU1T; break;
      case 4: rA = R_DXU3T; rB = R_DXBT; break;
      default: rA = R_DZU1T; rB = R_DZU3T; break;
    }
    // modal value of row r at mode k
    auto mval = [&](int r, int k) -> float2 {
      if (!tin) return make_float2(0.f, 0.f);
      const float kxv = a.kx[k];
      switch (r) {
        case R_U1: return SR(0, s)[k];
        case R_U3: return SR(1, s)[k];
        case R_B: return SR(2, s)[k];
        case R_U1T: return SR(3, s)[k];
        case R_U3T: return SR(4, s)[k];
        case R_BT: return SR(5, s)[k];
        case R_DXU1T: return cik(kxv, SR(3, s)[k]);
        case R_DXU3T: return cik(kxv, SR(4, s)[k]);
        case R_DXBT: return cik(kxv, SR(5, s)[k]);
        case R_DZU1T:   // Neumann -> Dirichlet (Differentiation.cpp:35-61), rows 2..N-1
          if (t < 2 || s < 1) return make_float2(0.f, 0.f);
          return cadd(cscale(SR(3, s - 1)[k], zc[ZC_DND_LO * N3 + t]), cscale(SR(3, s)[k], zc[ZC_DND_DI * N3 + t]));
        case R_DZBT:
          if (t < 2 || s < 1) return make_float2(0.f, 0.f);
          return cadd(cscale(SR(5, s - 1)[k], zc[ZC_DND_LO * N3 + t]), cscale(SR(5, s)[k], zc[ZC_DND_DI * N3 + t]));
        default: {   // R_DZU3T: Dirichlet -> Neumann, rows 1..N-1 (the last without the level above)
          if (t < 1 || s + 1 >= NS) return make_float2(0.f, 0.f);
          float2 v = cscale(SR(4, s)[k], zc[ZC_DDN_DI * N3 + t]);
          if (t < N3 - 1) v = cadd(v, cscale(SR(4, s + 1)[k], zc[ZC_DDN_UP * N3 + t]));
          return v;
        }
      }
    };
    float2 x[E];
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int n = l + G * e;
      float2 zz = make_float2(0.f, 0.f);
      if (n == 0) {
        zz = make_float2(mval(rA, 0).x, mval(rB, 0).x);   // c2r uses the real part of the k = 0 term
      } else if (n < K1) {
        const float2 A = mval(rA, n), B = mval(rB, n);
        zz = make_float2(A.x - B.y, A.y + B.x);            // A + iB
      } else if (n > N1 - K1) {
        const float2 A = mval(rA, N1 - n), B = mval(rB, N1 - n);
        zz = make_float2(A.x + B.y, B.x - A.y);            // conj(A) + i conj(B)
      }
      x[e] = zz;
    }
    reg_fft<N1, true>(x, buf, a.tw, l);
    if (valid) {
      float* pA = nod + ((size_t)rA * NS + s) * N1;
      float* pB = nod + ((size_t)rB * NS + s) * N1;
#pragma unroll
      for (int sl = 0; sl < E; sl++) {
        const int xo = reg_fft_out_index<N1>(l, sl);
        pA[xo] = x[sl].x;
        pB[xo] = x[sl].y;
      }
    }
  }
  __syncthreads();

  // ---- phase B: the nine products at their slots, two per forward transform ----
  const int nrows = adj_rows(S);
  const int ntB = (nrows + 1) / 2;
  const float sc = 0.5f * g.inv_n12;
  const float Ri = a.Ri[run], iK = a.adj_invK;
  auto R = [&](int r, int s, int x) -> float { return nod[((size_t)r * NS + s) * N1 + x]; };
  for (int base = 0; base < ntB; base += NGB) {
    const int task = base + gid;
    int pp[2] = {-1, -1}, ss[2] = {0, 0}, row[2] = {0, 0};
#pragma unroll
    for (int h = 0; h < 2; h++) {
      int r = 2 * task + h;
      if (task < ntB && r < nrows) {
        row[h] = r;
        for (int p = 0; p < Q_COUNT; p++) {
          int f0, c;
          adj_slots(p, S, f0, c);
          if (r < c) { pp[h] = p; ss[h] = f0 + r; break; }
          r -= c;
        }
      }
    }
    auto value = [&](int p, int s, int x) -> float {
      const int t = j0 - 1 + s;
      if (p < 0 || t < 0 || t >= N3) return 0.f;
      const bool lo = (t >= 1) && (s >= 1);
      const int sm = lo ? s - 1 : s;
      const bool top = t <= N3 - 2;
      const int sp = (top && s + 1 < NS) ? s + 1 : s;
      const float tp = (top && s + 1 < NS) ? 1.f : 0.f;
      const float lof = lo ? 1.f : 0.f;
      switch (p) {
        case Q_P1: return R(R_U1, s, x) * R(R_U1T, s, x);
        case Q_P2: return lof * 0.5f * (R(R_U1, s, x) + R(R_U1, sm, x)) * R(R_U3T, s, x);
        case Q_P3:
          return lof * (zc[ZC_TILDE_DI * N3 + t] * R(R_U1T, s, x) + zc[ZC_TILDE_LO * N3 + t] * R(R_U1T, sm, x)) *
                 R(R_U3, s, x);
        case Q_P4:
          return (0.5f * R(R_U3, s, x) + 0.5f * tp * R(R_U3, sp, x)) *
                 (0.5f * R(R_U3T, s, x) + 0.5f * tp * R(R_U3T, sp, x));
        case Q_P5: return lof * 0.5f * (R(R_B, s, x) + R(R_B, sm, x)) * R(R_U3T, s, x);
        case Q_P6: return R(R_B, s, x) * R(R_U1T, s, x);
        case Q_F1:   // -(ddx(u1T) U1 + Dir(ddx(u3T) U3) + ddx(bT) B)
          return -(R(R_DXU1T, s, x) * R(R_U1, s, x) +
                   0.5f * (R(R_DXU3T, s, x) * R(R_U3, s, x) + tp * R(R_DXU3T, sp, x) * R(R_U3, sp, x)) +
                   R(R_DXBT, s, x) * R(R_B, s, x));
        case Q_F3: {   // (BT - <bT>)/K - (ddz(u1T) Full(U1) + Full(ddz(u3T)) U3 + ddz(bT) Full(B))
          const float flo = lof * zc[ZC_FULL_LO * N3 + t], fdi = lof * zc[ZC_FULL_DI * N3 + t];
          return iK * (R(R_BT, s, x) - avg[s]) -
                 (R(R_DZU1T, s, x) * (flo * R(R_U1, sm, x) + fdi * R(R_U1, s, x)) +
                  (flo * R(R_DZU3T, sm, x) + fdi * R(R_DZU3T, s, x)) * R(R_U3, s, x) +
                  R(R_DZBT, s, x) * (flo * R(R_B, sm, x) + fdi * R(R_B, s, x)));
        }
        default:   // Q_FB: (U3T - <u3T>)/K + Ri Dir(U3)
          return iK * (R(R_U3T, s, x) - avg[NS + s]) + Ri * 0.5f * (R(R_U3, s, x) + tp * R(R_U3, sp, x));
      }
    };
    float2 x[E];
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int n = l + G * e;
      x[e] = make_float2(value(pp[0], ss[0], n), value(pp[1], ss[1], n));
    }
    reg_fft<N1, false>(x, buf, a.tw, l);
#pragma unroll
    for (int sl = 0; sl < E; sl++) buf[reg_fft_out_index<N1>(l, sl)] = x[sl];
    __syncwarp();
    for (int k = l; k < K1; k += G) {
      const float2 zk = buf[k];
      const float2 zc2 = cconj(buf[(N1 - k) & (N1 - 1)]);
      if (pp[0] >= 0) hat[(size_t)row[0] * K1 + k] = make_float2((zk.x + zc2.x) * sc, (zk.y + zc2.y) * sc);
      if (pp[1] >= 0) hat[(size_t)row[1] * K1 + k] = make_float2((zk.y - zc2.y) * sc, -(zk.x - zc2.x) * sc);
    }
    __syncwarp();
  }
  __syncthreads();

  // ---- phase D: r1, r3, rB (r += ..., IMEXRK.cpp:265-378) ----
  auto H = [&](int p, int s, int k) -> float2 { return hat[(size_t)adj_row(p, s, S) * K1 + k]; };
  for (int i = threadIdx.x; i < S * K1; i += blockDim.x) {
    const int si = i / K1, k = i - si * K1;
    const int t = j0 + si, s = si + 1;
    if (t >= N3) continue;
    const float kxv = a.kx[k];
    auto dzdn = [&](int p) -> float2 {
      if (t == 0) return make_float2(0.f, 0.f);
      float2 v = cscale(H(p, s, k), zc[ZC_DDN_DI * N3 + t]);
      if (t < N3 - 1) v = cadd(v, cscale(H(p, s + 1, k), zc[ZC_DDN_UP * N3 + t]));
      return v;
    };
    float2 dnd = make_float2(0.f, 0.f);
    if (t >= 2)
      dnd = cadd(cscale(H(Q_P4, s - 1, k), zc[ZC_DND_LO * N3 + t]), cscale(H(Q_P4, s, k), zc[ZC_DND_DI * N3 + t]));
    const float2 r1 = cadd(cadd(cik(kxv, H(Q_P1, s, k)), dzdn(Q_P2)), H(Q_F1, s, k));
    const float2 r3 = cadd(cadd(cik(kxv, H(Q_P3, s, k)), dnd), H(Q_F3, s, k));
    const float2 rb = cadd(cadd(dzdn(Q_P5), cik(kxv, H(Q_P6, s, k))), H(Q_FB, s, k));
    float2* r = a.rnl + (size_t)run * 4 * g.fblk + (size_t)t * g.Pp + k;
    r[0 * g.fblk] = r1;
    r[2 * g.fblk] = r3;
    r[3 * g.fblk] = rb;
  }
}

template <int N1>
void adj_launch(const StageArgs& a, cudaStream_t st) {
  const Geo& g = a.g;
  constexpr int G = FFTShape<N1>::G, BUF = fft_buf_stride<N1>();
  int S = 4;
  while (S > 1 && ((long long)adiv(g.N3, S) * g.nrun < 2 * 148 || adj_layout(S, N1, g.K1, BUF).bytes > 227 * 1024))
    S--;
  const size_t bytes = adj_layout(S, N1, g.K1, BUF).bytes;
  k_xpass_adj<N1><<<dim3(adiv(g.N3, S), 1, g.nrun), kAdjGroups * G, bytes, st>>>(a, S);
}

}  // namespace

size_t adjoint_smem_needed(const Geo& g) {
  int bufstride = 0;
  switch (g.N1) {
    case 16: bufstride = fft_buf_stride<16>(); break;
    case 32: bufstride = fft_buf_stride<32>(); break;
    case 64: bufstride = fft_buf_stride<64>(); break;
    case 128: bufstride = fft_buf_stride<128>(); break;
    case 256: bufstride = fft_buf_stride<256>(); break;
    default: bufstride = fft_buf_stride<512>(); break;
  }
  return adj_layout(4, g.N1, g.K1, bufstride).bytes;
}

int prepare_adjoint_kernels() {
  const int lim = 227 * 1024;
  cudaError_t e = cudaSuccess;
#define ADJ_ATTR(N) \
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_xpass_adj<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  ADJ_ATTR(16) ADJ_ATTR(32) ADJ_ATTR(64) ADJ_ATTR(128) ADJ_ATTR(256) ADJ_ATTR(512)
#undef ADJ_ATTR
  return e == cudaSuccess ? 0 : -1;
}

int launch_stage_adjoint(StageArgs a, const float2* below, const float2* above, float frac, float2* adir,
                         cudaStream_t st) {
  const Geo& g = a.g;
  const size_t n = (size_t)4 * g.fblk * g.nrun;
  k_adj_direct<<<(unsigned)std::min<size_t>((n + 255) / 256, 4096), 256, 0, st>>>(g, below, above, frac, a.Ubar,
                                                                                  adir);
  a.adir = adir;
  a.adjoint = 1;
  switch (g.N1) {
    case 16: adj_launch<16>(a, st); break;
    case 32: adj_launch<32>(a, st); break;
    case 64: adj_launch<64>(a, st); break;
    case 128: adj_launch<128>(a, st); break;
    case 256: adj_launch<256>(a, st); break;
    case 512: adj_launch<512>(a, st); break;
  }
  return 2 + launch_z_solves(a, st);
}

}  // namespace sf
