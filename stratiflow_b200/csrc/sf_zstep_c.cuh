// The z pass of a stage (ExplicitRK, FinishRHS, CrankNicolson and the Thomas
// solves of every field, IMEXRK.cpp:75-134, then RemoveDivergence,
// IMEXRK.cpp:43-73) with one lane per complex mode.
//
// k_z_step (sf_kernels.cu) gives each lane one real component of a mode, so
// the two lanes of a mode load and multiply the same real coefficients (the
// inverse pivots 1/den_j, the diagonals a_j and c_j, the grid stencils) and
// each lane's chunk of the levels is one serial chain. Here a lane owns both
// components of its mode as a float2 and updates them with paired FP32
// instructions (FFMA2 / FMUL2 / FADD2: every Thomas coefficient is real, so a
// complex value times a coefficient is one packed instruction), and each warp
// carries two z-chunks of the same 16 modes (lanes 0-15 the chunk 2w, lanes
// 16-31 the chunk 2w+1): a block of 8 warps splits N3 into 16 chunks (16
// warps and 32 chunks for grids too small to fill the GPU), so each
// serial sweep is half as long and the warp instructions per level are about
// half of k_z_step's. The arithmetic of every term is k_z_step's, in the same
// order; the chunked scan over 16 chunks instead of 8 reassociates the
// recurrences, so the two kernels agree to rounding.
#pragma once
#include <climits>
#include <type_traits>
#include "sf_internal.cuh"
#include "sf_fft2.cuh"

namespace sf {

constexpr int kCC = 16;        // z-chunks per block (two per warp) of the default block of 8 warps;
                               // grids too small to fill the GPU take 32 (16 warps)
constexpr int kCU = 2;         // levels of every input loaded ahead in the first sweep
constexpr int kCI = 8;         // levels of inverse pivots loaded ahead in the later sweeps
constexpr int kCP = 4;         // levels of the fields loaded ahead in the projection's last sweep

__device__ __forceinline__ float2 cz() { return make_float2(0.f, 0.f); }
__device__ __forceinline__ float2 cmul(float a, float2 x) { return pmul(pk2(a), x); }             // a x
__device__ __forceinline__ float2 cfma(float a, float2 x, float2 y) { return pfma(pk2(a), x, y); }   // a x + y
// i k z, componentwise as k_z_step's (i k z)_c = sc k z_{1-c}
__device__ __forceinline__ float2 czik(float k, float2 z) { return make_float2(-(k * z.y), k * z.x); }

struct ZcShared {
  float2* D;     // [N3][16]: be_j, then D_j
  float* A;      // [CC][16]
  float2* B;     // [CC][16]
  float2* In;    // [CC][16]
};
template <int CC>
__device__ __forceinline__ ZcShared zc_shared(int N3) {
  extern __shared__ __align__(16) float zcsm[];
  ZcShared s;
  s.D = reinterpret_cast<float2*>(zcsm);
  s.B = s.D + (size_t)N3 * 16;
  s.In = s.B + CC * 16;
  s.A = reinterpret_cast<float*>(s.In + CC * 16);
  return s;
}

// the scan of the chunks' affine maps v -> A v + B over the CC chunks of a
// block, upward (D) or downward (x), one lane per mode of warp 0
template <int CC>
__device__ __forceinline__ float2 zc_scan(const ZcShared& sh, int ch, int ml, int w, int lane, float A, float2 B,
                                          bool up) {
  sh.A[ch * 16 + ml] = A;
  sh.B[ch * 16 + ml] = B;
  __syncthreads();
  if (w == 0 && lane < 16) {
    float2 v = cz();
    for (int i = 0; i < CC; i++) {
      const int k = up ? i : CC - 1 - i;
      sh.In[k * 16 + lane] = v;
      v = cfma(sh.A[k * 16 + lane], v, sh.B[k * 16 + lane]);
    }
  }
  __syncthreads();
  return sh.In[ch * 16 + ml];
}

template <int K>
__device__ __forceinline__ void zc_iden(float (&bi)[K], const float* __restrict__ iden, int Pp, int j0, int step,
                                        int lo, int hi) {
#pragma unroll
  for (int i = 0; i < K; i++) {
    const int j = j0 + step * i;
    bi[i] = (j >= lo && j < hi) ? iden[(size_t)j * Pp] : 0.f;
  }
}

// the chunk map of the backward sweep x_js = B + A x_je
struct ZcMap {
  float A;
  float2 B;
};

// the second sweep (D_j), composing the chunk map of the backward sweep; the
// scan of those maps follows at the caller, outside any branch, so that every
// thread of the block reaches its barriers through the same instructions
template <bool IN, class CofF>
__device__ __forceinline__ ZcMap zc_sweep2(const ZcShared& sh, int js, int je, int ml, float2 D,
                                           const float* __restrict__ fa, const float* __restrict__ iden, int Pp,
                                           CofF Cof) {
  float A = 1.f;
  float2 B = cz();
  for (int j0 = js; j0 < je; j0 += kCI) {
    float bi[kCI];
    zc_iden(bi, iden, Pp, j0, 1, IN ? INT_MIN : js, IN ? INT_MAX : je);
#pragma unroll
    for (int i = 0; i < kCI; i++) {
      const int j = j0 + i;
      if (!IN && j >= je) break;
      const float al = (!IN && j == 0) ? 0.f : -fa[j] * bi[i];
      D = cfma(al, D, sh.D[j * 16 + ml]);
      sh.D[j * 16 + ml] = D;
      B = cfma(A, D, B);
      A = -A * Cof(j, bi[i]);
    }
  }
  return ZcMap{A, B};
}

// the CN solve of field f of family FAM (0: u1, u2; 1: u3, Dirichlet; 2: b)
template <int CC, int FAM, bool IC>
__device__ __forceinline__ void zc_cn(const StageArgs& a, const int f, const int bx, const int bz) {
  const Geo g = a.g;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int ml = lane & 15, ch = 2 * w + (lane >> 4);
  const int m0 = bx * 16 + ml;
  const bool act = m0 < g.P;
  const int m = act ? m0 : 0;
  const int run = bz;
  const int N3 = g.N3, Pp = g.Pp;
  const int chunk = (N3 + CC - 1) / CC;
  const int js = min(N3, ch * chunk), je = min(N3, js + chunk);
  const ZcShared sh = zc_shared<CC>(N3);
  const int q = m / g.K1, j1 = m - q * g.K1;
  const float kxv = a.kx[j1], kyv = a.ky[q];
  const float d1 = -(kxv * kxv), d2 = -(kyv * kyv);
  constexpr bool dir = (FAM == 1);
  const int fs = (FAM == 2 ? 1 : (dir ? 2 : 0)) * 3 + a.stage;   // factor sets: velocity, buoyancy, u3
  const float* __restrict__ fa = a.fa + (size_t)fs * N3;
  const float* __restrict__ fc = a.fc + (size_t)fs * N3;
  const float* __restrict__ iden = a.inv_den + (size_t)fs * N3 * Pp + m;
  const float* __restrict__ zc = a.zc;
  const float* __restrict__ lo2 = zc + (dir ? ZC_D2D_LO : ZC_D2N_LO) * N3;
  const float* __restrict__ di2 = zc + (dir ? ZC_D2D_DI : ZC_D2N_DI) * N3;
  const float* __restrict__ up2 = zc + (dir ? ZC_D2D_UP : ZC_D2N_UP) * N3;
  const float* __restrict__ dnd_lo = zc + ZC_DND_LO * N3;
  const float* __restrict__ dnd_di = zc + ZC_DND_DI * N3;
  const float* __restrict__ full_lo = zc + ZC_FULL_LO * N3;
  const float* __restrict__ full_di = zc + ZC_FULL_DI * N3;
  const float cco = (FAM == 2) ? a.cb : a.cv;
  const float Ri = a.Ri[run];
  const float* __restrict__ dB = a.dBdz + (size_t)run * N3;
  const bool zmode = (m == 0);   // the (0,0) mode: no buoyancy force (IMEXRK.cpp:141-143)
  const size_t fo = (size_t)(run * 5 + f) * N3 * Pp + m;
  const float2* uc = a.S + fo;
  const float2* pc = a.S + (size_t)(run * 5 + 4) * N3 * Pp + m;
  const float2* bc = a.S + (size_t)(run * 5 + 3) * N3 * Pp + m;
  const float2* wc = a.S + (size_t)(run * 5 + 2) * N3 * Pp + m;
  const float2* rc = a.rnl + (size_t)(run * 4 + f) * N3 * Pp + m;
  float2* rold = a.rold + (size_t)(run * 4 + f) * N3 * Pp + m;
  float2* out = a.Sn + fo;
  const bool use_rold = (a.hz != 0.f);
  const float kgrad = (f == 0) ? kxv : kyv;
  const size_t S1 = (size_t)Pp;

  // ---- forward, pass 1: right-hand side, be_j, chunk map ----
  float2 um = js >= 1 && js < N3 ? uc[(js - 1) * S1] : cz();
  float2 u0 = js < N3 ? uc[js * S1] : cz();
  float2 pm1 = (FAM == 1 && js >= 1 && js < N3) ? pc[(js - 1) * S1] : cz();
  float2 bm1 = (FAM == 1 && js >= 1 && js < N3) ? bc[(js - 1) * S1] : cz();
  float2 w0 = (FAM == 2 && js < N3) ? wc[js * S1] : cz();
  float A = 1.f;
  float2 B = cz();
  // a warp whose two chunks are clear of both ends (levels 3..N3-4) and a
  // whole number of batches of each sweep takes the sweeps without the
  // per-level end tests. The choice is the whole warp's: the later sweep ends
  // in the chunk scan's block barriers, which both halves of the warp must
  // reach through the same code
  const bool interior =
      __all_sync(0xffffffffu, IC && js >= 3 && je <= N3 - 4 && (je - js) % kCI == 0);
  static_assert(kCI % kCU == 0, "the first sweep's batches tile the later sweeps'");
  auto sweep1 = [&](auto tag) {
    constexpr bool IN = decltype(tag)::value;
    for (int j0 = js; j0 < je; j0 += kCU) {
      float2 bu[kCU], br[kCU], bo[kCU], bp[kCU], bx[kCU];
      float bi[kCU];
#pragma unroll
      for (int i = 0; i < kCU; i++) {
        const int j = j0 + i;
        const bool in = IN || j < je, nx = IN || (j + 1 < N3 && in);
        bu[i] = nx ? uc[(j + 1) * S1] : cz();
        br[i] = in ? rc[j * S1] : cz();
        bo[i] = (in && use_rold) ? rold[j * S1] : cz();
        bi[i] = in ? iden[(size_t)j * Pp] : 0.f;
        bp[i] = cz();
        bx[i] = cz();
        if (FAM == 0 || FAM == 1) bp[i] = in ? pc[j * S1] : cz();
        if (FAM == 1) bx[i] = in ? bc[j * S1] : cz();
        if (FAM == 2) bx[i] = nx ? wc[(j + 1) * S1] : cz();
      }
#pragma unroll
      for (int i = 0; i < kCU; i++) {
        const int j = j0 + i;
        if (!IN && j >= je) break;
        const float2 up = bu[i];
        float2 rt = br[i];
        float2 gp = cz();
        if (FAM == 0) {
          gp = czik(kgrad, bp[i]);   // i k p
        } else if (FAM == 1) {
          if (IN || j >= 2) gp = cfma(dnd_lo[j], pm1, cmul(dnd_di[j], bp[i]));
          pm1 = bp[i];
          if ((IN || j >= 1) && !zmode && !a.adjoint)   // r3 += Ri Full(b - <b>)
            rt = cfma(Ri, cfma(full_lo[j], bm1, cmul(full_di[j], bx[i])), rt);
          bm1 = bx[i];
        } else {
          const float2 w1 = bx[i];
          const float2 dw = (IN || j + 1 < N3) ? cfma(0.5f, w0, cmul(0.5f, w1)) : cmul(0.5f, w0);
          if (!a.adjoint) rt = cfma(-dB[j], dw, rt);   // rB -= dB/dz ReinterpolateDirichlet(u3)
          w0 = w1;
        }
        float2 R = u0;
        if (use_rold) R = cfma(a.hz, bo[i], R);
        R = cfma(-a.h, gp, R);
        R = cfma(a.hb, rt, R);
        const bool band = IN || (dir ? (j >= 2 && j <= N3 - 2) : (j >= 1 && j <= N3 - 2));
        const float2 d2u = band ? cfma(up2[j], up, cfma(di2[j], u0, cmul(lo2[j], um))) : cz();
        R = cfma(cco, padd(cfma(d2, u0, cmul(d1, u0)), d2u), R);
        const bool zend = !IN && ((j <= 1) || (j >= N3 - 2) || (dir && j == 2));   // ZeroEnds (Field.h:475-486)
        if (zend) R = cz();
        const float2 be = cmul(bi[i], R);
        const float al = (!IN && j == 0) ? 0.f : -fa[j] * bi[i];
        sh.D[j * 16 + ml] = be;
        if (act) rold[j * S1] = rt;
        A = al * A;
        B = cfma(al, B, be);
        um = u0;
        u0 = up;
      }
    }
  };
  if (interior) sweep1(std::true_type{});
  else sweep1(std::false_type{});
  const float2 Din = zc_scan<CC>(sh, ch, ml, w, lane, A, B, true);
  auto Cof = [&](int j, float bij) { return fc[j] * bij; };
  const ZcMap bk = interior ? zc_sweep2<true>(sh, js, je, ml, Din, fa, iden, Pp, Cof)
                            : zc_sweep2<false>(sh, js, je, ml, Din, fa, iden, Pp, Cof);
  float2 x = zc_scan<CC>(sh, ch, ml, w, lane, bk.A, bk.B, false);
  // ---- backward: x_j = D_j - C_j x_{j+1} ----
  auto sweep3 = [&](auto tag) {
    constexpr bool IN = decltype(tag)::value;
    for (int j0 = je - 1; j0 >= js; j0 -= kCI) {
      float bi[kCI];
      zc_iden(bi, iden, Pp, j0, -1, IN ? INT_MIN : js, IN ? INT_MAX : je);
#pragma unroll
      for (int i = 0; i < kCI; i++) {
        const int j = j0 - i;
        if (!IN && j < js) break;
        x = cfma(-(fc[j] * bi[i]), x, sh.D[j * 16 + ml]);
        if (act) out[j * S1] = x;
      }
    }
  };
  if (interior) sweep3(std::true_type{});
  else sweep3(std::false_type{});
}

// RemoveDivergence on the new velocities: the divergence and the Laplacian
// factors upward, q downward, then u -= grad q and p += pm q (k_z_step's
// projection, one lane per complex mode)
template <int CC>
__device__ __forceinline__ void zc_proj(const StageArgs& a, const int bx, const int bz) {
  const Geo g = a.g;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int ml = lane & 15, ch = 2 * w + (lane >> 4);
  const int m0 = bx * 16 + ml;
  const bool act = m0 < g.P;
  const int m = act ? m0 : 0;
  const int run = bz;
  const int N3 = g.N3, Pp = g.Pp;
  const int chunk = (N3 + CC - 1) / CC;
  const int js = min(N3, ch * chunk), je = min(N3, js + chunk);
  const ZcShared sh = zc_shared<CC>(N3);
  const int q = m / g.K1, j1 = m - q * g.K1;
  const float kxv = a.kx[j1], kyv = g.dim3 ? a.ky[q] : 0.f;
  const size_t S1 = (size_t)Pp;
  float2* u1 = a.Sn + (size_t)(run * 5 + 0) * N3 * Pp + m;
  float2* u2 = a.Sn + (size_t)(run * 5 + 1) * N3 * Pp + m;
  float2* u3 = a.Sn + (size_t)(run * 5 + 2) * N3 * Pp + m;
  const float2* ps = a.S + (size_t)(run * 5 + 4) * N3 * Pp + m;
  float2* pd = a.Sn + (size_t)(run * 5 + 4) * N3 * Pp + m;
  const float* __restrict__ a_ = a.fa + (size_t)kFS_Lap * N3;
  const float* __restrict__ c_ = a.fc + (size_t)kFS_Lap * N3;
  const float* __restrict__ iden = a.inv_den + (size_t)kFS_Lap * N3 * Pp + m;
  const float* __restrict__ zc = a.zc;
  const float* __restrict__ ddn_di = zc + ZC_DDN_DI * N3;
  const float* __restrict__ ddn_up = zc + ZC_DDN_UP * N3;
  const float* __restrict__ dnd_lo = zc + ZC_DND_LO * N3;
  const float* __restrict__ dnd_di = zc + ZC_DND_DI * N3;

  // ---- forward, pass 1: divergence, be_j, chunk map ----
  float2 w0 = js < N3 ? u3[js * S1] : cz();
  float A = 1.f;
  float2 B = cz();
  for (int j0 = js; j0 < je; j0 += kCU) {
    float2 b1[kCU], b2[kCU], b3[kCU];
    float bi[kCU];
#pragma unroll
    for (int i = 0; i < kCU; i++) {
      const int j = j0 + i;
      const bool in = j < je;
      b1[i] = in ? u1[j * S1] : cz();
      b2[i] = (in && g.dim3) ? u2[j * S1] : cz();
      b3[i] = (in && j + 1 < N3) ? u3[(j + 1) * S1] : cz();
      bi[i] = in ? iden[(size_t)j * Pp] : 0.f;
    }
#pragma unroll
    for (int i = 0; i < kCU; i++) {
      const int j = j0 + i;
      if (j >= je) break;
      const float2 w1 = b3[i];
      float2 dv = cz();
      if (j >= 2 && j <= N3 - 3) {
        const float2 t = cfma(kyv, b2[i], cmul(kxv, b1[i]));   // kx u1 + ky u2
        dv = padd(make_float2(-t.y, t.x), cfma(ddn_up[j], w1, cmul(ddn_di[j], w0)));
      }
      const float2 be = cmul(bi[i], dv);
      const float al = (j == 0) ? 0.f : -a_[j] * bi[i];
      sh.D[j * 16 + ml] = be;
      A = al * A;
      B = cfma(al, B, be);
      w0 = w1;
    }
  }
  const float2 Din = zc_scan<CC>(sh, ch, ml, w, lane, A, B, true);
  auto Cof = [&](int j, float bij) {
    float Cj = c_[j] * bij;
    if (m == 0 && j == 1) Cj = 0.f;   // (0,0) mode: row 1 pinned (IMEXRK.h:68-74)
    return Cj;
  };
  const ZcMap bk = zc_sweep2<false>(sh, js, je, ml, Din, a_, iden, Pp, Cof);
  float2 qn = zc_scan<CC>(sh, ch, ml, w, lane, bk.A, bk.B, false);   // q at level je
  // ---- backward, pass 2: q_j, projection, p; every row of u1, u2, u3, p is
  // written once, by the step of one level, so the loads of a batch may all
  // go ahead of its stores ----
  const float pm = a.pm;
  for (int j0 = je - 1; j0 >= js; j0 -= kCP) {
    float bi[kCP];
    float2 pv[kCP], v1[kCP], v2[kCP], v3[kCP];
    zc_iden(bi, iden, Pp, j0, -1, js, je);
#pragma unroll
    for (int i = 0; i < kCP; i++) {
      const int j = j0 - i, jj = j + 1;
      const bool in = j >= js && act;
      pv[i] = in ? ps[j * S1] : cz();
      v1[i] = in ? u1[j * S1] : cz();
      v2[i] = (in && g.dim3) ? u2[j * S1] : cz();
      v3[i] = (in && jj >= 2 && jj <= N3 - 1) ? u3[jj * S1] : cz();
    }
#pragma unroll
    for (int i = 0; i < kCP; i++) {
      const int j = j0 - i;
      if (j < js) break;
      const float2 qj = cfma(-Cof(j, bi[i]), qn, sh.D[j * 16 + ml]);
      if (act) {
        u1[j * S1] = psub(v1[i], czik(kxv, qj));
        if (g.dim3) u2[j * S1] = psub(v2[i], czik(kyv, qj));
        pd[j * S1] = cfma(pm, qj, pv[i]);
        const int jj = j + 1;   // u3_{j+1} -= ddz(q)_{j+1}, rows 2..N-1
        if (jj >= 2 && jj <= N3 - 1) u3[jj * S1] = psub(v3[i], cfma(dnd_lo[jj], qj, cmul(dnd_di[jj], qn)));
      }
      qn = qj;
    }
  }
}

// the whole z pass of a stage for the 16 modes of block coordinate bx of run
// bz: the CN solves of every field, then RemoveDivergence on the new
// velocities, which the block has just written (visible to it after the
// barrier). Needs N3 >= 32 and zc_smem_bytes(N3) of dynamic shared memory.
template <int CC, bool IC>
__device__ __forceinline__ void z_step_c_body(const StageArgs& a, const int bx, const int bz) {
  if (a.g.dim3) {
    zc_cn<CC, 0, IC>(a, 0, bx, bz);
    zc_cn<CC, 0, IC>(a, 1, bx, bz);
  } else {
    zc_cn<CC, 0, IC>(a, 0, bx, bz);
  }
  zc_cn<CC, 1, IC>(a, 2, bx, bz);
  zc_cn<CC, 2, IC>(a, 3, bx, bz);
  __syncthreads();
  zc_proj<CC>(a, bx, bz);
}

template <int CC = kCC>
__host__ __device__ inline size_t zc_smem_bytes(int N3) {
  return sizeof(float2) * ((size_t)N3 * 16 + 2 * CC * 16) + sizeof(float) * CC * 16;
}
template <int CC = kCC>
__host__ __device__ inline bool zc_fits(int N3) { return N3 >= 2 * CC; }

}  // namespace sf
