// IMEXRK::TimeStepAdjoint (IMEXRK.h:86-126) for 2D and 3D batches: per RK substep
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
// the z stencils and x derivatives give r1, r3, rB. In 3D, 12 fields are
// first transformed along y (the adjoint and direct fields and ddy of the
// direct ones), the x pass forms 20 rows and 16 products per level into the
// eight combinations of the forward pass, and the forward y transform of the
// forward step sums them with their i ky factors.
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
// lane groups of the 3D adjoint x pass: its 20 nodal rows leave room for one
// block per SM, so the block carries more groups (24 x 16 lanes at N1 = 256)
// to keep enough warps resident
constexpr int kAdj3Groups = 24;
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

// ---------------------------------------------------------------- 3D ----
// The 12 fields of the 3D adjoint x pass, inverse-transformed along y:
// the adjoint u1, u2, u3, b; the direct totals u1T, u2T, u3T, bT; and ddy of
// the direct totals (i ky applied on the modal rows). [nrun][12][N3][N2][K1]
constexpr int kYT = 128;
template <int N2>
__host__ __device__ constexpr int ycols_adj() { return (kYT / 32) * (32 / FFTShape<N2>::G); }

template <int N2>
__global__ void __launch_bounds__(kYT) k_ifft_y_adj(StageArgs a) {
  constexpr int G = FFTShape<N2>::G, E = FFTShape<N2>::E, BUF = fft_buf_stride<N2>();
  const Geo g = a.g;
  __shared__ float2 fbuf[(kYT / G) * BUF];
  const int grp = threadIdx.x / G, l = threadIdx.x % G;
  const int j1 = blockIdx.x * ycols_adj<N2>() + grp;
  const int j = blockIdx.y;
  const int run = blockIdx.z / 12, f = blockIdx.z % 12;
  const bool act = j1 < g.K1;
  const float2* src = f < 4 ? a.S + ((size_t)(run * 5 + f) * g.N3 + j) * g.Pp
                            : a.adir + ((size_t)(run * 4 + (f & 3)) * g.N3 + j) * g.Pp;
  float2 x[E];
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int n2 = l + G * e;
    int q = -1;
    if (n2 < g.Ky) q = n2;
    else if (n2 > N2 - g.Ky) q = n2 - (N2 - g.K2);
    float2 v = (act && q >= 0) ? src[q * g.K1 + j1] : make_float2(0.f, 0.f);
    if (f >= 8 && q >= 0) v = cik(a.ky[q], v);
    x[e] = v;
  }
  reg_fft<N2, true>(x, fbuf + grp * BUF, a.tw, l);
  if (act) {
    float2* dst = a.amix + ((size_t)(run * 12 + f) * g.N3 + j) * N2 * g.K1 + j1;
#pragma unroll
    for (int sl = 0; sl < E; sl++) dst[(size_t)reg_fft_out_index<N2>(l, sl) * g.K1] = x[sl];
  }
}

// nodal rows of the 3D adjoint x pass
enum { T_U1, T_U2, T_U3, T_B, T_U1T, T_U2T, T_U3T, T_BT, T_DX0, T_DY0 = T_DX0 + 4, T_DZU1T = T_DY0 + 4, T_DZU2T,
       T_DZU3T, T_DZBT, T_COUNT };
// products of the 3D adjoint, in hat-row order
enum { A_U1U1T, A_BU1_U3T, A_U1U2T, A_U2U2T, A_BU2_U3T, A_U2U1T, A_TU1T_U3, A_TU2T_U3, A_DU3DU3T, A_BB_U3T,
       A_BU2T, A_BU1T, A_F1, A_F2, A_F3, A_FB, A_COUNT };

__host__ __device__ __forceinline__ void adj3_slots(int p, int S, int& first, int& count) {
  if (p == A_BU1_U3T || p == A_BU2_U3T || p == A_BB_U3T) { first = 1; count = S + 1; }
  else if (p == A_DU3DU3T) { first = 0; count = S + 1; }
  else { first = 1; count = S; }
}
__host__ __device__ __forceinline__ int adj3_row(int p, int s, int S) {
  int base = 0;
  for (int q = 0; q < p; q++) {
    int f, c;
    adj3_slots(q, S, f, c);
    base += c;
  }
  int f, c;
  adj3_slots(p, S, f, c);
  return base + s - f;
}
__host__ __device__ inline int adj3_rows(int S) { return adj3_row(A_COUNT - 1, S, S) + 1; }

__host__ __device__ inline AdjLayout adj3_layout(int S, int N1, int K1, int bufstride) {
  AdjLayout L;
  const int NS = S + 2;
  size_t off = 0;
  const size_t stg = sizeof(float2) * (size_t)12 * NS * K1, hat = sizeof(float2) * (size_t)adj3_rows(S) * K1;
  L.stg_off = off; off += stg > hat ? stg : hat;
  L.nod_off = off; off += sizeof(float) * (size_t)T_COUNT * NS * N1;
  L.buf_off = off; off += sizeof(float2) * (size_t)kAdj3Groups * bufstride;
  L.avg_off = off; off += sizeof(float) * (size_t)2 * NS;
  L.bytes = off;
  return L;
}

// One block per (slab of S output levels, y row, run): the 20 nodal rows, the
// 16 products and the 8 combinations of the forward 3D pass (C_f, C_fy with
// r_f = Fy(C_f) + i ky Fy(C_fy)), into a.mixout
template <int N1>
__global__ void __launch_bounds__(kAdj3Groups * FFTShape<N1>::G) k_xpass_adj3(StageArgs a, int S) {
  constexpr int G = FFTShape<N1>::G, E = FFTShape<N1>::E, BUF = fft_buf_stride<N1>();
  constexpr int NGB = kAdj3Groups;
  const Geo g = a.g;
  extern __shared__ __align__(16) unsigned char xsm[];
  const AdjLayout L = adj3_layout(S, N1, g.K1, BUF);
  float2* stg = reinterpret_cast<float2*>(xsm + L.stg_off);   // [12][NS][K1]
  float2* hat = stg;
  float* nod = reinterpret_cast<float*>(xsm + L.nod_off);     // [T_COUNT][NS][N1]
  float* avg = reinterpret_cast<float*>(xsm + L.avg_off);     // [2][NS]: <bT>, <u3T>
  const int K1 = g.K1, N3 = g.N3, NS = S + 2;
  const int j0 = blockIdx.x * S;
  const int y = blockIdx.y;
  const int run = blockIdx.z;
  const int gid = threadIdx.x / G, l = threadIdx.x % G;
  float2* buf = reinterpret_cast<float2*>(xsm + L.buf_off) + (size_t)gid * BUF;
  const float* zc = a.zc;

  for (int i = threadIdx.x; i < 12 * NS * K1; i += blockDim.x) {
    const int fb = i / (NS * K1), r = i - fb * NS * K1, s = r / K1, k = r - s * K1;
    const int t = j0 - 1 + s;
    stg[i] = (t >= 0 && t < N3) ? a.amix[(((size_t)(run * 12 + fb) * N3 + t) * g.N2 + y) * K1 + k]
                                : make_float2(0.f, 0.f);
  }
  for (int s = threadIdx.x; s < NS; s += blockDim.x) {   // HorizontalAverage: the (0,0) modes
    const int t = j0 - 1 + s;
    const bool in = t >= 0 && t < N3;
    avg[s] = in ? a.adir[((size_t)(run * 4 + 3) * N3 + t) * g.Pp].x : 0.f;
    avg[NS + s] = in ? a.adir[((size_t)(run * 4 + 2) * N3 + t) * g.Pp].x : 0.f;
  }
  __syncthreads();
  auto SR = [&](int fb, int s) -> const float2* { return stg + ((size_t)fb * NS + s) * K1; };

  // ---- phase A: 20 nodal rows per slot, two per inverse transform ----
  const int ntA = 10 * NS;
  for (int base = 0; base < ntA; base += NGB) {
    const int task = base + gid;
    const bool valid = task < ntA;
    const int s = valid ? task % NS : 0, pr = valid ? task / NS : 0;
    const int t = j0 - 1 + s;
    const bool tin = valid && t >= 0 && t < N3;
    const int rA = 2 * pr, rB = 2 * pr + 1;
    auto mval = [&](int r, int k) -> float2 {
      if (!tin) return make_float2(0.f, 0.f);
      if (r < T_DX0) return SR(r, s)[k];                            // adjoint and direct fields
      if (r < T_DY0) return cik(a.kx[k], SR(4 + r - T_DX0, s)[k]);  // ddx of the direct fields
      if (r < T_DZU1T) return SR(8 + r - T_DY0, s)[k];              // ddy of the direct fields
      if (r == T_DZU3T) {                                          // Dirichlet -> Neumann
        if (t < 1 || s + 1 >= NS) return make_float2(0.f, 0.f);
        float2 v = cscale(SR(6, s)[k], zc[ZC_DDN_DI * N3 + t]);
        if (t < N3 - 1) v = cadd(v, cscale(SR(6, s + 1)[k], zc[ZC_DDN_UP * N3 + t]));
        return v;
      }
      const int fb = r == T_DZU1T ? 4 : (r == T_DZU2T ? 5 : 7);     // Neumann -> Dirichlet
      if (t < 2 || s < 1) return make_float2(0.f, 0.f);
      return cadd(cscale(SR(fb, s - 1)[k], zc[ZC_DND_LO * N3 + t]), cscale(SR(fb, s)[k], zc[ZC_DND_DI * N3 + t]));
    };
    float2 x[E];
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int n = l + G * e;
      float2 zz = make_float2(0.f, 0.f);
      if (n == 0) {
        zz = make_float2(mval(rA, 0).x, mval(rB, 0).x);
      } else if (n < K1) {
        const float2 A = mval(rA, n), B = mval(rB, n);
        zz = make_float2(A.x - B.y, A.y + B.x);
      } else if (n > N1 - K1) {
        const float2 A = mval(rA, N1 - n), B = mval(rB, N1 - n);
        zz = make_float2(A.x + B.y, B.x - A.y);
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

  // ---- phase B: the 16 products ----
  const int nrows = adj3_rows(S);
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
        for (int p = 0; p < A_COUNT; p++) {
          int f0, c;
          adj3_slots(p, S, f0, c);
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
      auto bar = [&](int r) { return lof * 0.5f * (R(r, s, x) + R(r, sm, x)); };
      auto dir = [&](int r) { return 0.5f * R(r, s, x) + 0.5f * tp * R(r, sp, x); };
      const float flo = lof * zc[ZC_FULL_LO * N3 + t], fdi = lof * zc[ZC_FULL_DI * N3 + t];
      auto full = [&](int r) { return flo * R(r, sm, x) + fdi * R(r, s, x); };
      auto tilde = [&](int r) {
        return lof * (zc[ZC_TILDE_DI * N3 + t] * R(r, s, x) + zc[ZC_TILDE_LO * N3 + t] * R(r, sm, x));
      };
      switch (p) {
        case A_U1U1T: return R(T_U1, s, x) * R(T_U1T, s, x);
        case A_BU1_U3T: return bar(T_U1) * R(T_U3T, s, x);
        case A_U1U2T: return R(T_U1, s, x) * R(T_U2T, s, x);
        case A_U2U2T: return R(T_U2, s, x) * R(T_U2T, s, x);
        case A_BU2_U3T: return bar(T_U2) * R(T_U3T, s, x);
        case A_U2U1T: return R(T_U2, s, x) * R(T_U1T, s, x);
        case A_TU1T_U3: return tilde(T_U1T) * R(T_U3, s, x);
        case A_TU2T_U3: return tilde(T_U2T) * R(T_U3, s, x);
        case A_DU3DU3T: return dir(T_U3) * dir(T_U3T);
        case A_BB_U3T: return bar(T_B) * R(T_U3T, s, x);
        case A_BU2T: return R(T_B, s, x) * R(T_U2T, s, x);
        case A_BU1T: return R(T_B, s, x) * R(T_U1T, s, x);
        case A_F1:
        case A_F2: {   // -(d(u1T) U1 + d(u2T) U2 + Dir(d(u3T) U3) + d(bT) B), d = ddx | ddy
          const int d0 = p == A_F1 ? T_DX0 : T_DY0;
          return -(R(d0, s, x) * R(T_U1, s, x) + R(d0 + 1, s, x) * R(T_U2, s, x) +
                   0.5f * (R(d0 + 2, s, x) * R(T_U3, s, x) + tp * R(d0 + 2, sp, x) * R(T_U3, sp, x)) +
                   R(d0 + 3, s, x) * R(T_B, s, x));
        }
        case A_F3:
          return iK * (R(T_BT, s, x) - avg[s]) -
                 (R(T_DZU1T, s, x) * full(T_U1) + R(T_DZU2T, s, x) * full(T_U2) + full(T_DZU3T) * R(T_U3, s, x) +
                  R(T_DZBT, s, x) * full(T_B));
        default:   // A_FB
          return iK * (R(T_U3T, s, x) - avg[NS + s]) + Ri * dir(T_U3);
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

  // ---- phase D: the 8 combinations ----
  auto H = [&](int p, int s, int k) -> float2 { return hat[(size_t)adj3_row(p, s, S) * K1 + k]; };
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
      dnd = cadd(cscale(H(A_DU3DU3T, s - 1, k), zc[ZC_DND_LO * N3 + t]),
                 cscale(H(A_DU3DU3T, s, k), zc[ZC_DND_DI * N3 + t]));
    float2* m = a.mixout + (((size_t)run * 8 * N3 + t) * g.N2 + y) * K1 + k;
    const size_t cs = g.mblk;
    m[0 * cs] = cadd(cadd(cik(kxv, H(A_U1U1T, s, k)), dzdn(A_BU1_U3T)), H(A_F1, s, k));
    m[1 * cs] = H(A_U1U2T, s, k);
    m[2 * cs] = cadd(cadd(cik(kxv, H(A_U2U1T, s, k)), dzdn(A_BU2_U3T)), H(A_F2, s, k));
    m[3 * cs] = H(A_U2U2T, s, k);
    m[4 * cs] = cadd(cadd(cik(kxv, H(A_TU1T_U3, s, k)), dnd), H(A_F3, s, k));
    m[5 * cs] = H(A_TU2T_U3, s, k);
    m[6 * cs] = cadd(cadd(dzdn(A_BB_U3T), cik(kxv, H(A_BU1T, s, k))), H(A_FB, s, k));
    m[7 * cs] = H(A_BU2T, s, k);
  }
}

template <int N1>
void adj3_launch(const StageArgs& a, cudaStream_t st) {
  const Geo& g = a.g;
  constexpr int G = FFTShape<N1>::G, BUF = fft_buf_stride<N1>();
  int S = 2;
  while (S > 1 && adj3_layout(S, N1, g.K1, BUF).bytes > 227 * 1024) S--;
  k_xpass_adj3<N1><<<dim3(adiv(g.N3, S), g.N2, g.nrun), kAdj3Groups * G, adj3_layout(S, N1, g.K1, BUF).bytes, st>>>(
      a, S);
}

template <int N2>
void ify_adj_launch(const StageArgs& a, cudaStream_t st) {
  k_ifft_y_adj<N2><<<dim3(adiv(a.g.K1, ycols_adj<N2>()), a.g.N3, a.g.nrun * 12), kYT, 0, st>>>(a);
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
#define ADJ_ATTR(N)                                                                                       \
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_xpass_adj<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim); \
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_xpass_adj3<N>, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
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
  if (g.dim3) {
    switch (g.N2) {
      case 16: ify_adj_launch<16>(a, st); break;
      case 32: ify_adj_launch<32>(a, st); break;
      case 64: ify_adj_launch<64>(a, st); break;
      case 128: ify_adj_launch<128>(a, st); break;
      case 256: ify_adj_launch<256>(a, st); break;
    }
    switch (g.N1) {
      case 16: adj3_launch<16>(a, st); break;
      case 32: adj3_launch<32>(a, st); break;
      case 64: adj3_launch<64>(a, st); break;
      case 128: adj3_launch<128>(a, st); break;
      case 256: adj3_launch<256>(a, st); break;
      case 512: adj3_launch<512>(a, st); break;
    }
    launch_fft_y_combos(a, st);
    return 4 + launch_z_solves(a, st);
  }
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
