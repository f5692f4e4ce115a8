// CUDA kernels of one IMEX-RK stage (IMEXRK.cpp:8-24 / 26-41) for sm_100a.
//
// A stage runs as
//   [3D] k_ifft_y   modal u1,u2,u3,b -> (kx, y) rows          (ModalField::ToNodal, y part)
//        k_xpass    per (y row, slab of z levels): c2r along x, the nodal
//                   products of BuildRHS / BuildRHSLinear, r2c along x,
//                   1/(N1 N2), 2/3 truncation and the z stencils and
//                   x-derivatives that follow each product
//   [3D] k_fft_y    (kx, y) -> (kx, ky), y-derivatives, sum into r
//        k_z_step   per group of 16 modes: for every field ExplicitRK + linear
//                   buoyancy terms + FinishRHS + CrankNicolson right-hand side +
//                   Thomas solve, then the divergence, Laplacian solve,
//                   projection and p update (k_z_proj_chunked alone serves
//                   RemoveDivergence outside a step)
// Every kernel touches only kept (dealiased) modes, which is all the reference's
// ModalField arithmetic touches (Field.h:1129-1166).

#include <algorithm>
#include <climits>
#include <type_traits>
#include "sf_internal.cuh"
#include "sf_fft.cuh"
#include "sf_fft2.cuh"
#include "sf_zstep_c.cuh"

namespace sf {

// ===================================================== y transforms (3D) ====
constexpr int kYThreads = 128;

__device__ __forceinline__ int n2_of_q(int q, int Ky, int K2, int N2) { return q < Ky ? q : q + N2 - K2; }

// kx columns handled by one block of the y transforms: one per lane group
template <int N2>
__host__ __device__ constexpr int ycols() { return (kYThreads / 32) * (32 / FFTShape<N2>::G); }

// modal [q][j1] of (run, field f, level j) -> mixed [y][j1], inverse c2c in y.
// One lane group per kx column; consecutive columns in consecutive groups so
// that a warp's loads of one y row cover whole 32-byte sectors.
template <int N2>
__global__ void __launch_bounds__(kYThreads, 8) k_ifft_y(StageArgs a) {
  constexpr int G = FFTShape<N2>::G, E = FFTShape<N2>::E, BUF = fft_buf_stride<N2>();
  const Geo g = a.g;
  __shared__ float2 fbuf[(kYThreads / G) * BUF];
  const int lane = threadIdx.x & 31, grp = threadIdx.x / G, l = threadIdx.x % G;
  const int j1 = blockIdx.x * ycols<N2>() + grp;
  const int j = blockIdx.y + a.lvl0;
  const int run = blockIdx.z >> 2, f = blockIdx.z & 3;
  const bool act = j1 < g.K1;
  const float2* src = a.S + ((size_t)(run * 5 + f) * g.N3 + j) * g.Pp;
  float2 x[E];
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int n2 = l + G * e;
    // kept rows: ky = 0..Ky-1 at n2 < Ky, ky = -(Ky-1)..-1 at n2 > N2 - Ky
    int q = -1;
    if (n2 < g.Ky) q = n2;
    else if (n2 > N2 - g.Ky) q = n2 - (N2 - g.K2);
    x[e] = (act && q >= 0) ? src[q * g.K1 + j1] : make_float2(0.f, 0.f);
  }
  (void)lane;
  reg_fft<N2, true>(x, fbuf + (threadIdx.x / G) * BUF, a.tw, l);
  if (act) {
    float2* dst = a.mixin + ((size_t)(run * 4 + f) * g.N3 + j) * N2 * g.K1 + j1;
#pragma unroll
    for (int sl = 0; sl < E; sl++) dst[(size_t)reg_fft_out_index<N2>(l, sl) * g.K1] = x[sl];
  }
}

// The same for fields (2p, 2p+1) of every run at once (blockIdx.z = 2 run +
// p): each lane group transforms its column of both fields as one packed pair
// of transforms (sf_fft2.cuh), half the FP32 instructions of two transforms.
template <int N2>
__global__ void __launch_bounds__(kYThreads) k_ifft_y2(StageArgs a) {
  constexpr int G = FFTShape<N2>::G, E = FFTShape<N2>::E;
  const Geo g = a.g;
  __shared__ float4 fbuf4[(kYThreads / G) * fft2_buf_elems<N2>()];
  __shared__ float4 tw4[E * G];
  __shared__ float2 tw2[E * G];
  fill_tw2<N2>(tw4, tw2, a.tw, threadIdx.x, kYThreads);
  __syncthreads();
  const int grp = threadIdx.x / G, l = threadIdx.x % G;
  const int j1 = blockIdx.x * ycols<N2>() + grp;
  const int j = blockIdx.y + a.lvl0;
  const int run = blockIdx.z >> 1, f0 = 2 * (blockIdx.z & 1);
  const bool act = j1 < g.K1;
  const float2* srcA = a.S + ((size_t)(run * 5 + f0) * g.N3 + j) * g.Pp + j1;
  const float2* srcB = srcA + (size_t)g.N3 * g.Pp;
  c2x x[E];
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int n2 = l + G * e;
    int q = -1;
    if (n2 < g.Ky) q = n2;
    else if (n2 > N2 - g.Ky) q = n2 - (N2 - g.K2);
    const bool in = act && q >= 0;
    const float2 A = in ? srcA[(size_t)q * g.K1] : make_float2(0.f, 0.f);
    const float2 B = in ? srcB[(size_t)q * g.K1] : make_float2(0.f, 0.f);
    x[e] = c2x{make_float2(A.x, B.x), make_float2(A.y, B.y)};
  }
  reg_fft2<N2, true>(x, fbuf4 + grp * fft2_buf_elems<N2>(), tw4, tw2, l);
  if (act) {
    float2* dA = a.mixin + ((size_t)(run * 4 + f0) * g.N3 + j) * N2 * g.K1 + j1;
    float2* dB = dA + (size_t)g.N3 * N2 * g.K1;
#pragma unroll
    for (int sl = 0; sl < E; sl++) {
      const size_t o = (size_t)reg_fft_out_index<N2>(l, sl) * g.K1;
      dA[o] = make_float2(x[sl].re.x, x[sl].im.x);
      dB[o] = make_float2(x[sl].re.y, x[sl].im.y);
    }
  }
}

// mixed combos (C_f, C_fy) [y][j1] -> r_f[q][j1] = Fy(C_f) + i ky Fy(C_fy)
template <int N2>
__global__ void __launch_bounds__(kYThreads) k_fft_y(StageArgs a) {
  constexpr int G = FFTShape<N2>::G, E = FFTShape<N2>::E;
  const Geo g = a.g;
  __shared__ float4 fbuf4[(kYThreads / G) * fft2_buf_elems<N2>()];
  __shared__ float4 tw4[E * G];
  __shared__ float2 tw2[E * G];
  fill_tw2<N2>(tw4, tw2, a.tw, threadIdx.x, kYThreads);
  __syncthreads();
  const int grp = threadIdx.x / G, l = threadIdx.x % G;
  const int j1 = blockIdx.x * ycols<N2>() + grp;
  const int j = blockIdx.y + a.lvl0;
  const int run = blockIdx.z >> 2, f = blockIdx.z & 3;
  const bool act = j1 < g.K1;
  const float2* cA = a.mixout + ((size_t)(run * 8 + 2 * f) * g.N3 + j) * N2 * g.K1 + j1;
  const float2* cB = a.mixout + ((size_t)(run * 8 + 2 * f + 1) * g.N3 + j) * N2 * g.K1 + j1;
  // (C_f, C_fy) as one packed pair of transforms (sf_fft2.cuh)
  c2x x[E];
#pragma unroll
  for (int e = 0; e < E; e++) {
    const size_t o = (size_t)(l + G * e) * g.K1;
    const float2 A = act ? cA[o] : make_float2(0.f, 0.f), B = act ? cB[o] : make_float2(0.f, 0.f);
    x[e] = c2x{make_float2(A.x, B.x), make_float2(A.y, B.y)};
  }
  reg_fft2<N2, false>(x, fbuf4 + grp * fft2_buf_elems<N2>(), tw4, tw2, l);
  if (act) {
    float2* dst = a.rnl + ((size_t)(run * 4 + f) * g.N3 + j) * g.Pp + j1;
#pragma unroll
    for (int sl = 0; sl < E; sl++) {
      const int n2 = reg_fft_out_index<N2>(l, sl);
      int q = -1;
      if (n2 < g.Ky) q = n2;
      else if (n2 > N2 - g.Ky) q = n2 - (N2 - g.K2);
      if (q >= 0) {   // Fy(C_f) + i ky Fy(C_fy)
        const float ky = a.ky[q];
        dst[(size_t)q * g.K1] = make_float2(x[sl].re.x - ky * x[sl].im.y, x[sl].im.x + ky * x[sl].re.y);
      }
    }
  }
}

// ============================================================= x pass ====
// product ids (BuildRHS, IMEXRK.cpp:155-192; BuildRHSLinear, :212-257)
enum Prod { P_S1, P_SB1, P_P3, P_Q1, P_QB, P_P4, P_S12, P_S22, P_SB2, P_Q2, P_P3Y, P_COUNT };

constexpr int kXMaxThreads = 512;

// slots s = 0..S+1 hold level j0-1+s; product p is formed at slots
// [first, first+count)
__host__ __device__ __forceinline__ void prod_slots(int p, int S, int& first, int& count) {
  if (p == P_Q1 || p == P_QB || p == P_Q2) { first = 1; count = S + 1; }
  else if (p == P_P4) { first = 0; count = S + 1; }
  else { first = 1; count = S; }
}
__host__ __device__ inline int prod_rows(int nprod, int S) {
  int n = 0;
  for (int p = 0; p < nprod; p++) { int f, c; prod_slots(p, S, f, c); n += c; }
  return n;
}

// row of the transformed product p at slot s; p is a compile-time constant at
// every call, so the loop folds
__device__ __forceinline__ int hat_row(int p, int s, int S) {
  int base = 0;
#pragma unroll
  for (int q = 0; q < P_COUNT; q++) {
    if (q == p) break;
    int f, c;
    prod_slots(q, S, f, c);
    base += c;
  }
  int f, c;
  prod_slots(p, S, f, c);
  return base + s - f;
}

// products whose first slot repeats the last (Q products) or next-to-last
// (P4) slot of the slab below; a block that walks up through several slabs
// keeps those transformed rows instead of forming them again
__host__ __device__ __forceinline__ bool carried(int p) {
  return p == P_Q1 || p == P_QB || p == P_Q2 || p == P_P4;
}

// row stride (floats) of the nodal rows in shared memory: N1 padded by one
// lane group, so the lane groups of a warp, which read the same field at
// consecutive slots, fall on different banks
__host__ __device__ constexpr int nod_row(int N1) { return N1 + (N1 >= 256 ? 16 : (N1 >= 64 ? 8 : 4)); }

struct XLayout {  // shared-memory carve-up of k_xpass
  int nprod, nrows;
  size_t hat_off, stage_off, buf_off, nod_off, base_off, carry_off, bytes;
};

__host__ __device__ inline XLayout x_layout(int S, int N1, int K1, int dim3, int linear, int bufstride, int ngroups,
                                            int tlm, int prefetch) {
  XLayout L;
  L.nprod = dim3 ? P_COUNT : 6;
  L.nrows = prod_rows(L.nprod, S);
  size_t off = 0;
  // transformed products, one row of K1 per (product, slot), and the staged
  // input rows of phase A (4 x (S+2) x K1, twice that when the base rows of
  // a tangent-linear batch come along): their own bytes when a block loads
  // the next slab's rows during this slab's work, else the same bytes
  auto al16 = [](size_t b) { return (b + 15) & ~(size_t)15; };   // 16-byte aligned regions
  size_t hat = al16(sizeof(float2) * (size_t)L.nrows * K1),
         stage = al16(sizeof(float2) * (size_t)(tlm ? 8 : 4) * (S + 2) * K1);
  L.hat_off = off;
  if (prefetch) {
    off += hat;
    L.stage_off = off; off += stage;
  } else {
    L.stage_off = off; off += (hat > stage ? hat : stage);
  }
  L.buf_off = off;  off += sizeof(float2) * (size_t)ngroups * bufstride;
  L.nod_off = off;  off += sizeof(float) * (size_t)4 * (S + 2) * nod_row(N1);
  L.base_off = off; if (linear) off += sizeof(float) * (size_t)4 * (S + 2) * nod_row(N1);
  L.carry_off = off; off += sizeof(float2) * (size_t)4 * K1;   // transformed rows kept for the next slab
  L.bytes = off;
  return L;
}

// ---- BuildRHS / BuildRHSLinear products by pair ----
// Each forward transform carries two real products; a pair kind fixes which
// two, so the rows each lane reads and the arithmetic are compile-time
// constants and the two products of a pair share their loads. Products at
// slot i + 1 of a slab (i < S): (S1, SB1), (P3, P4), (S12, S22), (SB2, P3Y);
// the Q products at slot i + 2: (Q1, QB) and (Q2 at i + 2, Q2 at i + 3); the
// slab's first halo rows, (Q1, QB) at slot 1 and (P4 at slot 0, Q2 at slot 1),
// when no slab below handed them over.
enum PairKind { K_SSB1, K_P34, K_S122, K_SB2P, K_QQB, K_Q2Q2, K_HALO };

struct HalfC {  // one product at one slot: its rows and coefficients
  int s, sm, sp;
  float ub, ubm, tlo, tdi, hb, lof, top;
  bool live;
};

__device__ __forceinline__ HalfC half_coeffs(int s, int j0, int N3, const float* Ub, const float* zc) {
  HalfC c;
  const int t = j0 - 1 + s;
  c.live = t >= 0 && t < N3;
  const int tc = c.live ? t : 0;
  const bool lo = c.live && (t >= 1) && (s >= 1);
  c.s = s;
  c.sm = lo ? s - 1 : s;
  c.top = (t <= N3 - 2) ? 1.f : 0.f;
  c.sp = (t <= N3 - 2) ? s + 1 : s;
  c.lof = lo ? 1.f : 0.f;
  c.tlo = c.lof * zc[ZC_TILDE_LO * N3 + tc];
  c.tdi = c.lof * zc[ZC_TILDE_DI * N3 + tc];
  c.hb = 0.5f * c.lof;
  c.ub = Ub[tc];
  c.ubm = lo ? Ub[tc - 1] : 0.f;
  return c;
}

// product P of BuildRHS at point n (IMEXRK.cpp:155-192; the U1t*U1t product
// leaves out its x-independent U_^2 part, which ddx multiplies by zero)
template <int P, int N1>
__device__ __forceinline__ float prod_at(const float* nod, int NS, const HalfC& c, int n) {
  auto u = [&](int f, int slot) { return nod[(f * NS + slot) * nod_row(N1) + n]; };
  float v;
  if constexpr (P == P_S1) { const float a = u(0, c.s); v = a * (a + 2.f * c.ub); }
  else if constexpr (P == P_SB1) v = (u(0, c.s) + c.ub) * u(3, c.s);
  else if constexpr (P == P_P3)
    v = (c.tdi * u(0, c.s) + c.tlo * u(0, c.sm) + (c.tlo * c.ubm + c.tdi * c.ub)) * (c.lof * u(2, c.s));
  else if constexpr (P == P_Q1)
    v = (c.hb * u(0, c.s) + c.hb * u(0, c.sm) + (c.hb * c.ubm + c.hb * c.ub)) * (c.lof * u(2, c.s));
  else if constexpr (P == P_QB) v = (c.hb * u(3, c.s) + c.hb * u(3, c.sm)) * (c.lof * u(2, c.s));
  else if constexpr (P == P_P4) { const float d = 0.5f * u(2, c.s) + 0.5f * c.top * u(2, c.sp); v = d * d; }
  else if constexpr (P == P_S12) v = (u(0, c.s) + c.ub) * u(1, c.s);
  else if constexpr (P == P_S22) { const float a = u(1, c.s); v = a * a; }
  else if constexpr (P == P_SB2) v = u(1, c.s) * u(3, c.s);
  else if constexpr (P == P_Q2) v = (c.hb * u(1, c.s) + c.hb * u(1, c.sm)) * (c.lof * u(2, c.s));
  else v = (c.tdi * u(1, c.s) + c.tlo * u(1, c.sm)) * (c.lof * u(2, c.s));   // P_P3Y
  return c.live ? v : 0.f;
}

// product P of BuildRHSLinear at point n (IMEXRK.cpp:212-257): the
// derivative of BuildRHS's product about the base, whose rows `bas` hold
// U1b + U_, U2b, U3b, Bb (so the U_ terms come with the base's u1)
template <int P, int N1>
__device__ __forceinline__ float prod_at_lin(const float* nod, const float* bas, int NS, const HalfC& c, int n) {
  auto u = [&](int f, int slot) { return nod[(f * NS + slot) * nod_row(N1) + n]; };
  auto U = [&](int f, int slot) { return bas[(f * NS + slot) * nod_row(N1) + n]; };
  float v;
  if constexpr (P == P_S1) v = (2.f * u(0, c.s)) * U(0, c.s);
  else if constexpr (P == P_SB1) v = u(3, c.s) * U(0, c.s) + U(3, c.s) * u(0, c.s);
  else if constexpr (P == P_P3)
    v = (c.tdi * u(0, c.s) + c.tlo * u(0, c.sm)) * (c.lof * U(2, c.s)) +
        (c.tdi * U(0, c.s) + c.tlo * U(0, c.sm)) * (c.lof * u(2, c.s));
  else if constexpr (P == P_Q1)
    v = (c.hb * u(0, c.s) + c.hb * u(0, c.sm)) * (c.lof * U(2, c.s)) +
        (c.hb * U(0, c.s) + c.hb * U(0, c.sm)) * (c.lof * u(2, c.s));
  else if constexpr (P == P_QB)
    v = (c.hb * u(3, c.s) + c.hb * u(3, c.sm)) * (c.lof * U(2, c.s)) +
        (c.hb * U(3, c.s) + c.hb * U(3, c.sm)) * (c.lof * u(2, c.s));
  else if constexpr (P == P_P4)   // 2 Dir(u3) Dir(U3b)
    v = (u(2, c.s) + c.top * u(2, c.sp)) * (0.5f * U(2, c.s) + 0.5f * c.top * U(2, c.sp));
  else if constexpr (P == P_S12) v = u(0, c.s) * U(1, c.s) + U(0, c.s) * u(1, c.s);
  else if constexpr (P == P_S22) v = (2.f * u(1, c.s)) * U(1, c.s);
  else if constexpr (P == P_SB2) v = u(3, c.s) * U(1, c.s) + U(3, c.s) * u(1, c.s);
  else if constexpr (P == P_Q2)
    v = (c.hb * u(1, c.s) + c.hb * u(1, c.sm)) * (c.lof * U(2, c.s)) +
        (c.hb * U(1, c.s) + c.hb * U(1, c.sm)) * (c.lof * u(2, c.s));
  else   // P_P3Y
    v = (c.tdi * u(1, c.s) + c.tlo * u(1, c.sm)) * (c.lof * U(2, c.s)) +
        (c.tdi * U(1, c.s) + c.tlo * U(1, c.sm)) * (c.lof * u(2, c.s));
  return c.live ? v : 0.f;
}

template <int P0, int P1, int N1, int E, int G, bool LINEAR>
__device__ __forceinline__ void pair_eval(float2 (&x)[E], const float* nod, const float* bas, int NS, const HalfC& c0,
                                          const HalfC& c1, bool two, int l) {
#pragma unroll
  for (int e = 0; e < E; e++) {
    const int n = l + G * e;
    if constexpr (LINEAR)
      x[e] = make_float2(prod_at_lin<P0, N1>(nod, bas, NS, c0, n), two ? prod_at_lin<P1, N1>(nod, bas, NS, c1, n) : 0.f);
    else
      x[e] = make_float2(prod_at<P0, N1>(nod, NS, c0, n), two ? prod_at<P1, N1>(nod, NS, c1, n) : 0.f);
  }
}

__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void cp_async_wait_all() { asm volatile("cp.async.wait_all;\n" ::); }
// 16-byte asynchronous copy (both addresses 16-byte aligned)
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem) {
  unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16;\n" ::"r"(s), "l"(gmem));
}

// One block per (`iters` consecutive slabs of S output levels, y row, run).
// Lane groups of G lanes each run one transform at a time; all groups of the
// block step through their task lists in lockstep so every lane reaches
// every warp sync. Walking up from one slab to the next, the block keeps the
// two top nodal levels and the top transformed rows of the carried products
// (their z stencils reach one level across the slab boundary), so each level
// is transformed once rather than once per slab that touches it.
// The body of one x-pass block: (bx, by, bz) = (level column, y row, run)
// relative to a.xcol0 and a.run_offset, so that a kernel over many solvers'
// work items can run it for any block of any of them.
template <int N1, bool LINEAR>
__device__ __forceinline__ void xpass_body(const StageArgs& a, int S, int iters, int bx, int by, int bz) {
  constexpr int G = FFTShape<N1>::G, E = FFTShape<N1>::E, BUF = fft_buf_stride<N1>();
  const int NGB = blockDim.x / G;   // lane groups per block
  const Geo g = a.g;
  extern __shared__ __align__(16) unsigned char xsm[];
  const int tlm = LINEAR ? a.tlm : 0;   // base rows from a live run of this batch
  const XLayout L = x_layout(S, N1, g.K1, g.dim3, LINEAR, BUF, NGB, tlm, iters > 1);
  float2* hat = reinterpret_cast<float2*>(xsm + L.hat_off);
  float2* stg = reinterpret_cast<float2*>(xsm + L.stage_off);  // phase A input rows [4 or 8][S+2][K1]
  constexpr int NR = nod_row(N1);   // nodal row stride
  float* nod = reinterpret_cast<float*>(xsm + L.nod_off);      // [4][S+2][NR]: U1, U2, U3, B
  float* bnod = reinterpret_cast<float*>(xsm + L.base_off);    // [4][S+2][NR]: U1b+Ubar, U2b, U3b, Bb
  constexpr int K1 = N1 / 3;   // kept x modes (the solver's K1), a compile-time constant here
  const int N3 = g.N3;
  const int y = by;
  const int run = bz + a.run_offset;
  const int brun = tlm ? (run - tlm) % tlm : run;   // run that holds the base state
  const int gid = threadIdx.x / G, l = threadIdx.x % G;
  float2* buf = reinterpret_cast<float2*>(xsm + L.buf_off) + (size_t)gid * BUF;
  const float* Ub = a.Ubar + (size_t)run * N3;
  const float* zc = a.zc;
  const int NS = S + 2;
  const int nf = tlm ? 8 : 4;   // own u1,u2,u3,b (and the base run's)
  float2* carry = reinterpret_cast<float2*>(xsm + L.carry_off);   // [4][K1]: Q1, QB, Q2, P4
  // this lane's twiddles, held in registers for every transform of the block
  // (read from the table at each transform when E = 32 would not fit)
  constexpr bool kTwReg = E <= 16;
  float2 twl[kTwReg ? E : 1];
  if constexpr (kTwReg) lane_twiddles<N1>(twl, a.tw, l);
  auto fft_inv = [&](float2 (&v)[E]) {
    if constexpr (kTwReg) reg_fft_w<N1, true>(v, buf, twl, l);
    else reg_fft<N1, true>(v, buf, a.tw, l);
  };
  auto fft_fwd = [&](float2 (&v)[E]) {
    if constexpr (kTwReg) reg_fft_w<N1, false>(v, buf, twl, l);
    else reg_fft<N1, false>(v, buf, a.tw, l);
  };

  // stage the input rows u1, u2, u3, b (and the base run's) at slots s0..S+1
  // (levels jj0-1+s0 .. jj0+S) with asynchronous copies, one warp per row
  auto stage_rows = [&](int jj0, int s0) {
    const int NSn = NS - s0, nw = blockDim.x >> 5, lane = threadIdx.x & 31;
    for (int row = threadIdx.x >> 5; row < nf * NSn; row += nw) {
      const int fb = row / NSn, s = s0 + row - fb * NSn;
      const int f = fb & 3, rr = fb < 4 ? run : brun;
      const int t = jj0 - 1 + s;
      float2* d = stg + ((size_t)fb * NS + s) * K1;
      if (t < 0 || t >= N3 || (f == 1 && !g.dim3)) {
        for (int k = lane; k < K1; k += 32) d[k] = make_float2(0.f, 0.f);
      } else {
        const float2* src = g.dim3 ? a.mixin + (((size_t)(rr * 4 + f) * N3 + t) * g.N2 + y) * K1
                                   : a.S + ((size_t)(rr * 5 + f) * N3 + t) * g.Pp;
        for (int k = lane; k < K1; k += 32) cp_async8(d + k, src + k);
      }
    }
  };
  const int col = bx + a.xcol0;   // level column of this block
  stage_rows(col * iters * S, 0);

  for (int it = 0; it < iters; it++) {
  const int j0 = (col * iters + it) * S;
  if (j0 >= N3) break;
  const int s0 = it == 0 ? 0 : 2;   // nodal slots 0, 1 come from the slab below
  const int NSn = NS - s0;

  if (LINEAR && !tlm) {  // frozen nodal base rows (IMEXRK.h:344-351), one warp per row
    const int nw = blockDim.x >> 5, lane = threadIdx.x & 31;
    for (int row = threadIdx.x >> 5; row < 4 * NS; row += nw) {
      const int f = row / NS, t = j0 - 1 + row - f * NS;
      float* d = bnod + (size_t)row * NR;
      if (t < 0 || t >= N3 || (f == 1 && !g.dim3)) {
        for (int x = lane; x < N1; x += 32) d[x] = 0.f;
      } else {
        const float* src = a.base + (((size_t)(run * 4 + f) * N3 + t) * g.N2 + y) * N1;
        for (int c = lane; c < N1 / 4; c += 32) cp_async16(d + 4 * c, src + 4 * c);
      }
    }
  }
  cp_async_wait_all();
  __syncthreads();
  if (LINEAR && !tlm) {   // U1b + U_ as nnTemp (phase A writes only the own rows meanwhile)
    for (int i = threadIdx.x; i < NS * N1; i += blockDim.x) {
      const int sl = i / N1, t = j0 - 1 + sl;
      if (t >= 0 && t < N3) bnod[sl * NR + (i - sl * N1)] += Ub[t];
    }
  }

  // ---- phase A: inverse transforms of (u1, u3) and (b, u2) (ToNodal) ----
  // (and of the base run's fields for a tangent-linear batch)
  const int ntA = NSn * (tlm ? 4 : 2);
  for (int base = 0; base < ntA; base += NGB) {
    const int task = base + gid;
    const bool valid = task < ntA;
    const int s = valid ? s0 + task % NSn : 0, pr4 = valid ? task / NSn : 0;
    const int pr = pr4 & 1, ofs = (pr4 >> 1) * 4;   // ofs 4: base rows
    const int fA = pr == 0 ? 0 : 3;       // u1 | b
    const int fB = pr == 0 ? 2 : 1;       // u3 | u2
    const float2* srcA = stg + ((size_t)(ofs + fA) * NS + s) * K1;
    const float2* srcB = stg + ((size_t)(ofs + fB) * NS + s) * K1;
    float2 x[E];
#pragma unroll
    for (int e = 0; e < E; e++) {
      const int n = l + G * e;
      float2 zz = make_float2(0.f, 0.f);
      if (n == 0) {
        zz = make_float2(srcA[0].x, srcB[0].x);   // c2r uses the real part of the k = 0 term
      } else if (n < K1) {
        const float2 A = srcA[n], B = srcB[n];
        zz = make_float2(A.x - B.y, A.y + B.x);            // A + iB
      } else if (n > N1 - K1) {
        const float2 A = srcA[N1 - n], B = srcB[N1 - n];
        zz = make_float2(A.x + B.y, B.x - A.y);            // conj(A) + i conj(B)
      }
      x[e] = zz;
    }
    fft_inv(x);
    if (valid) {
      float* rows = ofs ? bnod : nod;
      float* rA = rows + ((size_t)fA * NS + s) * NR;
      float* rB = rows + ((size_t)fB * NS + s) * NR;
      const int t = j0 - 1 + s;
      // the base's U1 row carries U_ (nnTemp = U1_tot + U_, IMEXRK.cpp:212)
      const float add = (ofs && fA == 0 && t >= 0 && t < N3) ? a.Ubar[(size_t)brun * N3 + t] : 0.f;
#pragma unroll
      for (int sl = 0; sl < E; sl++) {
        const int xo = reg_fft_out_index<N1>(l, sl);
        rA[xo] = x[sl].x + add;
        rB[xo] = x[sl].y;
      }
    }
  }
  __syncthreads();

  // the next slab's input rows load while this slab's products are formed
  if (it + 1 < iters && j0 + S < N3) stage_rows(j0 + S, 2);

  // rows carried over from the slab below
  if (it > 0)
    for (int i = threadIdx.x; i < 4 * K1; i += blockDim.x) {
      const int q = i / K1, k = i - q * K1;
      const int p = q == 0 ? P_Q1 : (q == 1 ? P_QB : (q == 2 ? P_Q2 : P_P4));
      if (p < L.nprod) hat[(size_t)hat_row(p, p == P_P4 ? 0 : 1, S) * K1 + k] = carry[i];
    }

  // ---- phase B/C: nodal products, forward transforms in pairs (ToModal) ----
  const int nprod = L.nprod;
  const float sc = 0.5f * g.inv_n12;
  const int NT = g.dim3 ? 5 : 3;   // pair kinds at every output level
  const int nmain = NT * S, nq2 = g.dim3 ? (S + 1) / 2 : 0, ntB = nmain + nq2 + (it == 0 ? 2 : 0);
  for (int base = 0; base < ntB; base += NGB) {
    const int task = base + gid;
    int kind = -1, i = 0;
    if (task < nmain) {
      const int q = task / S;
      kind = q < 2 ? q : (g.dim3 ? q : K_QQB);   // 2D: (S1, SB1), (P3, P4), (Q1, QB)
      i = task - q * S;
    } else if (task < nmain + nq2) {
      kind = K_Q2Q2;
      i = 2 * (task - nmain);
    } else if (task < ntB) {
      kind = task == nmain + nq2 ? K_QQB : K_HALO;
      i = -1;
    }
    int s0 = i + 1, s1 = i + 1, p0 = -1, p1 = -1;
    switch (kind) {
      case K_SSB1: p0 = P_S1; p1 = P_SB1; break;
      case K_P34: p0 = P_P3; p1 = P_P4; break;
      case K_S122: p0 = P_S12; p1 = P_S22; break;
      case K_SB2P: p0 = P_SB2; p1 = P_P3Y; break;
      case K_QQB: p0 = P_Q1; p1 = P_QB; s0 = s1 = i + 2; break;
      case K_Q2Q2: p0 = P_Q2; p1 = i + 1 < S ? P_Q2 : -1; s0 = i + 2; s1 = i + 3; break;
      case K_HALO: p0 = P_P4; p1 = g.dim3 ? P_Q2 : -1; s0 = 0; s1 = 1; break;
      default: break;
    }
    const HalfC c0 = half_coeffs(s0, j0, N3, Ub, zc), c1 = half_coeffs(s1, j0, N3, Ub, zc);
    const bool two = p1 >= 0;
    float2 x[E];
    switch (kind) {
      case K_SSB1: pair_eval<P_S1, P_SB1, N1, E, G, LINEAR>(x, nod, bnod, NS, c0, c1, true, l); break;
      case K_P34: pair_eval<P_P3, P_P4, N1, E, G, LINEAR>(x, nod, bnod, NS, c0, c1, true, l); break;
      case K_S122: pair_eval<P_S12, P_S22, N1, E, G, LINEAR>(x, nod, bnod, NS, c0, c1, true, l); break;
      case K_SB2P: pair_eval<P_SB2, P_P3Y, N1, E, G, LINEAR>(x, nod, bnod, NS, c0, c1, true, l); break;
      case K_QQB: pair_eval<P_Q1, P_QB, N1, E, G, LINEAR>(x, nod, bnod, NS, c0, c1, true, l); break;
      case K_Q2Q2: pair_eval<P_Q2, P_Q2, N1, E, G, LINEAR>(x, nod, bnod, NS, c0, c1, two, l); break;
      case K_HALO: pair_eval<P_P4, P_Q2, N1, E, G, LINEAR>(x, nod, bnod, NS, c0, c1, two, l); break;
      default:
#pragma unroll
        for (int e = 0; e < E; e++) x[e] = make_float2(0.f, 0.f);
    }
    fft_fwd(x);
#pragma unroll
    for (int sl = 0; sl < E; sl++) buf[reg_fft_out_index<N1>(l, sl)] = x[sl];
    __syncwarp();
    if (p0 >= 0) {
      float2* h0 = hat + (size_t)hat_row(p0, s0, S) * K1;
      float2* h1 = hat + (size_t)hat_row(two ? p1 : p0, s1, S) * K1;
#pragma unroll
      for (int q = 0; q < (K1 + G - 1) / G; q++) {
        const int k = l + q * G;
        if (k >= K1) break;
        const float2 zk = buf[k];
        const float2 zc2 = cconj(buf[(N1 - k) & (N1 - 1)]);
        h0[k] = make_float2((zk.x + zc2.x) * sc, (zk.y + zc2.y) * sc);          // (Zk + conj Z_{N-k}) / 2
        if (two) h1[k] = make_float2((zk.y - zc2.y) * sc, -(zk.x - zc2.x) * sc);  // (Zk - conj Z_{N-k}) / (2i)
      }
    }
    __syncwarp();
  }
  __syncthreads();

  // ---- phase D: z stencils of the products and x derivatives ----
  auto H = [&](int p, int s, int k) -> float2 { return hat[(size_t)hat_row(p, s, S) * K1 + k]; };
  for (int i = threadIdx.x; i < S * K1; i += blockDim.x) {
    const int si = i / K1, k = i - si * K1;
    const int t = j0 + si, s = si + 1;
    if (t >= N3) continue;
    const float kxv = a.kx[k];
    // ddz Dirichlet -> Neumann of a Q product (Differentiation.cpp:35-61)
    auto dzdn = [&](int p) -> float2 {
      if (t == 0) return make_float2(0.f, 0.f);
      float di = zc[ZC_DDN_DI * N3 + t];
      float2 v = cscale(H(p, s, k), di);
      if (t < N3 - 1) v = cadd(v, cscale(H(p, s + 1, k), zc[ZC_DDN_UP * N3 + t]));
      return v;
    };
    float2 dnd = make_float2(0.f, 0.f);  // ddz Neumann -> Dirichlet of P4
    if (t >= 2)
      dnd = cadd(cscale(H(P_P4, s - 1, k), zc[ZC_DND_LO * N3 + t]), cscale(H(P_P4, s, k), zc[ZC_DND_DI * N3 + t]));
    const float2 c1 = csub(cscale(cik(kxv, H(P_S1, s, k)), -1.f), dzdn(P_Q1));
    const float2 c3 = csub(cscale(cik(kxv, H(P_P3, s, k)), -1.f), dnd);
    const float2 cB = csub(cscale(cik(kxv, H(P_SB1, s, k)), -1.f), dzdn(P_QB));
    if (!g.dim3) {
      float2* r = a.rnl + (size_t)run * 4 * g.fblk + (size_t)t * g.Pp + k;
      r[0 * g.fblk] = c1;
      r[2 * g.fblk] = c3;
      r[3 * g.fblk] = cB;
    } else {
      const float2 c1y = cscale(H(P_S12, s, k), -1.f);
      const float2 c2 = csub(cscale(cik(kxv, H(P_S12, s, k)), -1.f), dzdn(P_Q2));
      const float2 c2y = cscale(H(P_S22, s, k), -1.f);
      const float2 c3y = cscale(H(P_P3Y, s, k), -1.f);
      const float2 cBy = cscale(H(P_SB2, s, k), -1.f);
      float2* m = a.mixout + (((size_t)run * 8 * N3 + t) * g.N2 + y) * K1 + k;
      const size_t cs = g.mblk;
      m[0 * cs] = c1; m[1 * cs] = c1y; m[2 * cs] = c2; m[3 * cs] = c2y;
      m[4 * cs] = c3; m[5 * cs] = c3y; m[6 * cs] = cB; m[7 * cs] = cBy;
    }
  }

  // ---- keep what the next slab shares with this one ----
  if (it + 1 < iters) {
    __syncthreads();
    for (int i = threadIdx.x; i < 4 * K1; i += blockDim.x) {
      const int q = i / K1, k = i - q * K1;
      const int p = q == 0 ? P_Q1 : (q == 1 ? P_QB : (q == 2 ? P_Q2 : P_P4));
      if (p < nprod) carry[i] = hat[(size_t)hat_row(p, p == P_P4 ? S : S + 1, S) * K1 + k];
    }
    for (int i = threadIdx.x; i < nf * 2 * N1; i += blockDim.x) {   // nodal slots S, S+1 -> 0, 1
      const int fb = i / (2 * N1), r = i - fb * 2 * N1, sl = r / N1, x = r - sl * N1;
      float* rows = fb < 4 ? nod : bnod;
      const int f = fb & 3;
      rows[((size_t)f * NS + sl) * NR + x] = rows[((size_t)f * NS + S + sl) * NR + x];
    }
    __syncthreads();
  }
  }   // slabs
}

template <int N1, bool LINEAR>
__global__ void __launch_bounds__(kXMaxThreads) k_xpass(StageArgs a, int S, int iters) {
  xpass_body<N1, LINEAR>(a, S, iters, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ============================================================ z pass ====
constexpr int kZU = 8;   // levels of every input loaded ahead per thread



// ------------------------------------------------ chunked z solves ----
// The Thomas sweeps are first-order affine recurrences: D_j = al_j D_{j-1} +
// be_j (al_j = -a_j/den_j, be_j = R_j/den_j) upward, x_j = D_j - C_j x_{j+1}
// downward. A block of ZW warps (8, or 16 for grids too small to fill the
// GPU) splits N3 into ZW z-chunks, one per warp,
// and covers 16 modes x {real, imag} per warp: every chunk composes its
// affine map, one warp scans the ZW maps in z order, and every chunk then
// replays its levels from the right incoming value. be_j and D_j stay in
// shared memory ([N3][32] floats per block). The result equals the sequential
// sweep up to rounding.
constexpr int kZU2 = 4;   // levels of every input loaded ahead in the chunked z kernels' first sweep
constexpr int kZI = 16;   // levels of inverse pivots loaded ahead in their later sweeps
constexpr int kZP = 4;    // levels of the fields loaded ahead in the projection's last sweep

template <int ZW>
__device__ __forceinline__ void zscan_up(float* sA, float* sB, float* sIn, int w, int lane, float A, float B) {
  sA[w * 32 + lane] = A;
  sB[w * 32 + lane] = B;
  __syncthreads();
  if (w == 0) {
    float v = 0.f;
    for (int k = 0; k < ZW; k++) {
      sIn[k * 32 + lane] = v;
      v = sA[k * 32 + lane] * v + sB[k * 32 + lane];
    }
  }
  __syncthreads();
}
template <int ZW>
__device__ __forceinline__ void zscan_down(float* sA, float* sB, float* sIn, int w, int lane, float A, float B) {
  sA[w * 32 + lane] = A;
  sB[w * 32 + lane] = B;
  __syncthreads();
  if (w == 0) {
    float v = 0.f;
    for (int k = ZW - 1; k >= 0; k--) {
      sIn[k * 32 + lane] = v;
      v = sA[k * 32 + lane] * v + sB[k * 32 + lane];
    }
  }
  __syncthreads();
}

// the inverse pivots of levels j0, j0 + step, ... (K of them, those in
// [lo, hi)) loaded ahead of their use in the serial sweeps
template <int K>
__device__ __forceinline__ void load_iden(float (&bi)[K], const float* __restrict__ iden, int Pp, int j0, int step,
                                          int lo, int hi) {
#pragma unroll
  for (int i = 0; i < K; i++) {
    const int j = j0 + step * i;
    bi[i] = (j >= lo && j < hi) ? iden[(size_t)j * Pp] : 0.f;
  }
}

// the CN solve of k_z_step for field f of family FAM (0: u1 and u2,
// 1: u3, Dirichlet; 2: b), so that each family's loads and terms are fixed
// at compile time; IC: chunks clear of the ends take sweeps without the
// per-level end tests
template <int ZW, int FAM, bool IC>
__device__ __forceinline__ void z_cn_body(const StageArgs& a, const int f, const int bx, const int bz) {
  const Geo g = a.g;
  extern __shared__ float zsm[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int m0 = bx * 16 + (lane >> 1), c = lane & 1;
  const bool act = m0 < g.P;
  const int m = act ? m0 : 0;
  const int run = bz;
  const int N3 = g.N3, Pp = g.Pp;
  const int chunk = (N3 + ZW - 1) / ZW;
  const int js = min(N3, w * chunk), je = min(N3, js + chunk);
  float* sD = zsm;                      // [N3][32]: be_j, then D_j
  float* sA = zsm + (size_t)N3 * 32;    // [ZW][32]
  float* sB = sA + ZW * 32;
  float* sIn = sB + ZW * 32;
  const int q = m / g.K1, j1 = m - q * g.K1;
  const float kxv = a.kx[j1], kyv = a.ky[q];
  const float d1 = -(kxv * kxv), d2 = -(kyv * kyv);
  const float sc = c == 0 ? -1.f : 1.f;   // (i k z)_c = sc * k * z_{1-c}
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
  const float* uc = reinterpret_cast<const float*>(a.S + fo) + c;
  const float* pc = reinterpret_cast<const float*>(a.S + (size_t)(run * 5 + 4) * N3 * Pp + m) + c;
  const float* po = reinterpret_cast<const float*>(a.S + (size_t)(run * 5 + 4) * N3 * Pp + m) + (1 - c);
  const float* bc = reinterpret_cast<const float*>(a.S + (size_t)(run * 5 + 3) * N3 * Pp + m) + c;
  const float* wc = reinterpret_cast<const float*>(a.S + (size_t)(run * 5 + 2) * N3 * Pp + m) + c;
  const float* rc = reinterpret_cast<const float*>(a.rnl + (size_t)(run * 4 + f) * N3 * Pp + m) + c;
  float* rold = reinterpret_cast<float*>(a.rold + (size_t)(run * 4 + f) * N3 * Pp + m) + c;
  float* out = reinterpret_cast<float*>(a.Sn + fo) + c;
  const bool use_rold = (a.hz != 0.f);
  const float kgrad = (f == 0) ? kxv : kyv;
  const size_t S2 = 2 * (size_t)Pp;

  // ---- forward, pass 1: right-hand side, be_j, chunk map ----
  float um = js >= 1 && js < N3 ? uc[(js - 1) * S2] : 0.f;
  float u0 = js < N3 ? uc[js * S2] : 0.f;
  float pm1 = (FAM == 1 && js >= 1 && js < N3) ? pc[(js - 1) * S2] : 0.f;
  float bm1 = (FAM == 1 && js >= 1 && js < N3) ? bc[(js - 1) * S2] : 0.f;
  float w0 = (FAM == 2 && js < N3) ? wc[js * S2] : 0.f;
  float A = 1.f, B = 0.f;
  // a chunk clear of both ends (levels 3..N3-4) and a whole number of batches
  // of each sweep takes the sweeps without the per-level end tests
  const bool interior = IC && js >= 3 && je <= N3 - 4 && (je - js) % kZI == 0;
  static_assert(kZI % kZU2 == 0, "the first sweep's batches tile the later sweeps'");
  auto sweep1 = [&](auto tag) {
  constexpr bool IN = decltype(tag)::value;
  for (int j0 = js; j0 < je; j0 += kZU2) {
    float bu[kZU2], br[kZU2], bo[kZU2], bp[kZU2], bx[kZU2], bi[kZU2];
#pragma unroll
    for (int i = 0; i < kZU2; i++) {
      const int j = j0 + i;
      const bool in = IN || j < je, nx = IN || (j + 1 < N3 && in);
      bu[i] = nx ? uc[(j + 1) * S2] : 0.f;
      br[i] = in ? rc[j * S2] : 0.f;
      bo[i] = (in && use_rold) ? rold[j * S2] : 0.f;
      bi[i] = in ? iden[(size_t)j * Pp] : 0.f;
      bp[i] = 0.f;
      bx[i] = 0.f;
      if (FAM == 0) bp[i] = in ? po[j * S2] : 0.f;
      if (FAM == 1) {
        bp[i] = in ? pc[j * S2] : 0.f;
        bx[i] = in ? bc[j * S2] : 0.f;
      }
      if (FAM == 2) bx[i] = nx ? wc[(j + 1) * S2] : 0.f;
    }
#pragma unroll
    for (int i = 0; i < kZU2; i++) {
      const int j = j0 + i;
      if (!IN && j >= je) break;
      const float up = bu[i];
      float rt = br[i];
      float gp = 0.f;
      if (FAM == 0) {
        gp = sc * kgrad * bp[i];   // (i k p)_c
      } else if (FAM == 1) {
        if (IN || j >= 2) gp = dnd_lo[j] * pm1 + dnd_di[j] * bp[i];
        pm1 = bp[i];
        if ((IN || j >= 1) && !zmode && !a.adjoint) rt += Ri * (full_lo[j] * bm1 + full_di[j] * bx[i]);   // r3 += Ri Full(b - <b>)
        bm1 = bx[i];
      } else {
        const float w1 = bx[i];
        const float dw = (IN || j + 1 < N3) ? 0.5f * w0 + 0.5f * w1 : 0.5f * w0;
        if (!a.adjoint) rt -= dB[j] * dw;   // rB -= dB/dz ReinterpolateDirichlet(u3)
        w0 = w1;
      }
      float R = u0;
      if (use_rold) R += a.hz * bo[i];
      R += -a.h * gp;
      R += a.hb * rt;
      const bool band = IN || (dir ? (j >= 2 && j <= N3 - 2) : (j >= 1 && j <= N3 - 2));
      const float d2u = band ? lo2[j] * um + di2[j] * u0 + up2[j] * up : 0.f;
      R += cco * ((d1 * u0 + d2 * u0) + d2u);
      const bool zend = !IN && ((j <= 1) || (j >= N3 - 2) || (dir && j == 2));   // ZeroEnds (Field.h:475-486)
      if (zend) R = 0.f;
      const float be = R * bi[i];
      const float al = (!IN && j == 0) ? 0.f : -fa[j] * bi[i];
      sD[j * 32 + lane] = be;
      if (act) rold[j * S2] = rt;
      A = al * A;
      B = al * B + be;
      um = u0;
      u0 = up;
    }
  }
  };
  if (interior) sweep1(std::true_type{});
  else sweep1(std::false_type{});
  zscan_up<ZW>(sA, sB, sIn, w, lane, A, B);
  // ---- forward, pass 2: D_j, and with it the chunk map of the backward
  // sweep x_j = D_j - C_j x_{j+1}, composed upwards: x_js = B + A x_je ----
  float D = sIn[w * 32 + lane];
  A = 1.f;
  B = 0.f;
  auto sweep2 = [&](auto tag) {
    constexpr bool IN = decltype(tag)::value;
    for (int j0 = js; j0 < je; j0 += kZI) {
      float bi[kZI];
      load_iden(bi, iden, Pp, j0, 1, IN ? INT_MIN : js, IN ? INT_MAX : je);
#pragma unroll
      for (int i = 0; i < kZI; i++) {
        const int j = j0 + i;
        if (!IN && j >= je) break;
        const float al = (!IN && j == 0) ? 0.f : -fa[j] * bi[i];
        D = al * D + sD[j * 32 + lane];
        sD[j * 32 + lane] = D;
        B = B + A * D;
        A = -A * (fc[j] * bi[i]);
      }
    }
  };
  if (interior) sweep2(std::true_type{});
  else sweep2(std::false_type{});
  __syncthreads();
  zscan_down<ZW>(sA, sB, sIn, w, lane, A, B);
  // ---- backward, pass 2: the solution ----
  float x = sIn[w * 32 + lane];
  auto sweep3 = [&](auto tag) {
    constexpr bool IN = decltype(tag)::value;
    for (int j0 = je - 1; j0 >= js; j0 -= kZI) {
      float bi[kZI];
      load_iden(bi, iden, Pp, j0, -1, IN ? INT_MIN : js, IN ? INT_MAX : je);
#pragma unroll
      for (int i = 0; i < kZI; i++) {
        const int j = j0 - i;
        if (!IN && j < js) break;
        const float Cj = fc[j] * bi[i];
        x = sD[j * 32 + lane] - Cj * x;
        if (act) out[j * S2] = x;
      }
    }
  };
  if (interior) sweep3(std::true_type{});
  else sweep3(std::false_type{});
}

// RemoveDivergence with the chunked solve, for 16 modes per block: the
// divergence and the Laplacian factors upward, q downward, then u -= grad q
// and p += pm q. The two components of a mode are adjacent lanes and
// exchange q; u3_{j+1} at a chunk's top uses the next chunk's q from the scan.
template <int ZW>
__device__ __forceinline__ void z_proj_body(const Geo& g, float2* U, const float2* Psrc, float2* Pdst,
                                            const float* zc, const float* fa, const float* fc,
                                            const float* inv_den, const float* kx, const float* ky, float pm,
                                            const int bx, const int bz) {
  extern __shared__ float zsm[];
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int m0 = bx * 16 + (lane >> 1), c = lane & 1;
  const bool act = m0 < g.P;
  const int m = act ? m0 : 0;
  const int run = bz;
  const int N3 = g.N3, Pp = g.Pp;
  const int chunk = (N3 + ZW - 1) / ZW;
  const int js = min(N3, w * chunk), je = min(N3, js + chunk);
  float* sD = zsm;
  float* sA = zsm + (size_t)N3 * 32;
  float* sB = sA + ZW * 32;
  float* sIn = sB + ZW * 32;
  const int q = m / g.K1, j1 = m - q * g.K1;
  const float kxv = kx[j1], kyv = g.dim3 ? ky[q] : 0.f;
  const float sc = c == 0 ? -1.f : 1.f;
  const size_t S2 = 2 * (size_t)Pp;
  float* u1 = reinterpret_cast<float*>(U + (size_t)(run * 5 + 0) * N3 * Pp + m);
  float* u2 = reinterpret_cast<float*>(U + (size_t)(run * 5 + 1) * N3 * Pp + m);
  float* u3 = reinterpret_cast<float*>(U + (size_t)(run * 5 + 2) * N3 * Pp + m) + c;
  const float* ps = reinterpret_cast<const float*>(Psrc + (size_t)(run * 5 + 4) * N3 * Pp + m) + c;
  float* pd = reinterpret_cast<float*>(Pdst + (size_t)(run * 5 + 4) * N3 * Pp + m) + c;
  const float* __restrict__ a_ = fa + (size_t)kFS_Lap * N3;
  const float* __restrict__ c_ = fc + (size_t)kFS_Lap * N3;
  const float* __restrict__ iden = inv_den + (size_t)kFS_Lap * N3 * Pp + m;
  const float* __restrict__ ddn_di = zc + ZC_DDN_DI * N3;
  const float* __restrict__ ddn_up = zc + ZC_DDN_UP * N3;
  const float* __restrict__ dnd_lo = zc + ZC_DND_LO * N3;
  const float* __restrict__ dnd_di = zc + ZC_DND_DI * N3;
  const float* u1o = u1 + (1 - c);   // u1_{1-c}
  const float* u2o = u2 + (1 - c);
  float* u1c = u1 + c;
  float* u2c = u2 + c;

  // ---- forward, pass 1: divergence, be_j, chunk map ----
  float w0 = js < N3 ? u3[js * S2] : 0.f;
  float A = 1.f, B = 0.f;
  for (int j0 = js; j0 < je; j0 += kZU) {
    float b1[kZU], b2[kZU], b3[kZU], bi[kZU];
#pragma unroll
    for (int i = 0; i < kZU; i++) {
      const int j = j0 + i;
      const bool in = j < je;
      b1[i] = in ? u1o[j * S2] : 0.f;
      b2[i] = (in && g.dim3) ? u2o[j * S2] : 0.f;
      b3[i] = (in && j + 1 < N3) ? u3[(j + 1) * S2] : 0.f;
      bi[i] = in ? iden[(size_t)j * Pp] : 0.f;
    }
#pragma unroll
    for (int i = 0; i < kZU; i++) {
      const int j = j0 + i;
      if (j >= je) break;
      const float w1 = b3[i];
      float dv = 0.f;
      if (j >= 2 && j <= N3 - 3) dv = sc * (kxv * b1[i] + kyv * b2[i]) + (ddn_di[j] * w0 + ddn_up[j] * w1);
      const float be = dv * bi[i];
      const float al = (j == 0) ? 0.f : -a_[j] * bi[i];
      sD[j * 32 + lane] = be;
      A = al * A;
      B = al * B + be;
      w0 = w1;
    }
  }
  zscan_up<ZW>(sA, sB, sIn, w, lane, A, B);
  // D_j, and with it the chunk map of the backward sweep, composed upwards
  auto Cof = [&](int j, float bij) {
    float Cj = c_[j] * bij;
    if (m == 0 && j == 1) Cj = 0.f;   // (0,0) mode: row 1 pinned (IMEXRK.h:68-74)
    return Cj;
  };
  float D = sIn[w * 32 + lane];
  A = 1.f;
  B = 0.f;
  for (int j0 = js; j0 < je; j0 += kZI) {
    float bi[kZI];
    load_iden(bi, iden, Pp, j0, 1, js, je);
#pragma unroll
    for (int i = 0; i < kZI; i++) {
      const int j = j0 + i;
      if (j >= je) break;
      const float al = (j == 0) ? 0.f : -a_[j] * bi[i];
      D = al * D + sD[j * 32 + lane];
      sD[j * 32 + lane] = D;
      B = B + A * D;
      A = -A * Cof(j, bi[i]);
    }
  }
  __syncthreads();
  zscan_down<ZW>(sA, sB, sIn, w, lane, A, B);
  // ---- backward, pass 2: q_j, projection, p ----
  float qn = sIn[w * 32 + lane];   // q at level je (0 above the top)
  // every row of u1, u2, u3, p is written once, by the step of one level,
  // so the loads of a batch may all go ahead of its stores
  for (int j0 = je - 1; j0 >= js; j0 -= kZP) {
    float bi[kZP], pv[kZP], v1[kZP], v2[kZP], v3[kZP];
    load_iden(bi, iden, Pp, j0, -1, js, je);
#pragma unroll
    for (int i = 0; i < kZP; i++) {
      const int j = j0 - i, jj = j + 1;
      const bool in = j >= js && act;
      pv[i] = in ? ps[j * S2] : 0.f;
      v1[i] = in ? u1c[j * S2] : 0.f;
      v2[i] = (in && g.dim3) ? u2c[j * S2] : 0.f;
      v3[i] = (in && jj >= 2 && jj <= N3 - 1) ? u3[jj * S2] : 0.f;
    }
#pragma unroll
    for (int i = 0; i < kZP; i++) {
      const int j = j0 - i;
      if (j < js) break;
      const float qj = sD[j * 32 + lane] - Cof(j, bi[i]) * qn;
      const float qo = __shfl_xor_sync(0xffffffffu, qj, 1);
      if (act) {
        u1c[j * S2] = v1[i] - sc * kxv * qo;
        if (g.dim3) u2c[j * S2] = v2[i] - sc * kyv * qo;
        pd[j * S2] = pv[i] + pm * qj;
        const int jj = j + 1;   // u3_{j+1} -= ddz(q)_{j+1}, rows 2..N-1
        if (jj >= 2 && jj <= N3 - 1) u3[jj * S2] = v3[i] - (dnd_lo[jj] * qj + dnd_di[jj] * qn);
      }
      qn = qj;
    }
  }
}

template <int ZW>
__global__ void __launch_bounds__(ZW * 32, ZW == 8 ? 3 : 1) k_z_proj_chunked(Geo g, float2* U, const float2* Psrc, float2* Pdst,
                                                           const float* zc, const float* fa, const float* fc,
                                                           const float* inv_den, const float* kx, const float* ky,
                                                           float pm) {
  z_proj_body<ZW>(g, U, Psrc, Pdst, zc, fa, fc, inv_den, kx, ky, pm, blockIdx.x, blockIdx.z);
}

// The whole z pass of a stage for 16 modes per block: the CN solves of every
// field (ExplicitRK, linear buoyancy terms, FinishRHS, CrankNicolson and the
// Thomas solve, IMEXRK.cpp:75-134), then RemoveDivergence on the new
// velocities (IMEXRK.cpp:43-73). The projection reads the velocities this
// block has just written (visible to the block after the barrier, and still
// in L2), so the pass makes one trip through HBM instead of two kernels'.
// Every field's solve uses the same shared-memory rows: a thread reads and
// writes only its own rows of sD, and the chunk scans synchronise the block.
template <int ZW, bool IC>
__device__ __forceinline__ void z_step_body(const StageArgs& a, const int bx, const int bz) {
  if (a.g.dim3) {
    z_cn_body<ZW, 0, IC>(a, 0, bx, bz);
    z_cn_body<ZW, 0, IC>(a, 1, bx, bz);
  } else {
    z_cn_body<ZW, 0, IC>(a, 0, bx, bz);
  }
  z_cn_body<ZW, 1, IC>(a, 2, bx, bz);
  z_cn_body<ZW, 2, IC>(a, 3, bx, bz);
  __syncthreads();
  z_proj_body<ZW>(a.g, a.Sn, a.S, a.Sn, a.zc, a.fa, a.fc, a.inv_den, a.kx, a.ky, a.pm, bx, bz);
}

template <int ZW, bool IC>
__global__ void __launch_bounds__(ZW * 32, ZW == 8 ? 3 : 1) k_z_step(StageArgs a) {
  z_step_body<ZW, IC>(a, blockIdx.x, blockIdx.z);
}


// ============================================================ ensembles ====
// Every member of an ensemble of 2D solvers (grids of different sizes, one
// run each) in one launch per kernel: a block reads its work item and its
// member's stage arguments and runs the same block body as the solver's own
// launch would. Blocks have kEnsThreads threads for every grid; the dynamic
// shared memory is the largest any member needs.
__global__ void __launch_bounds__(kEnsThreads, 2) k_xpass_ens(const StageArgs* __restrict__ args,
                                                              const EnsItem* __restrict__ items) {
  __shared__ StageArgs sa;
  const EnsItem it = items[blockIdx.x];
  if (threadIdx.x == 0) sa = args[it.run];
  __syncthreads();
  switch (sa.g.N1) {
    case 16: xpass_body<16, false>(sa, it.S, it.iters, it.x, 0, 0); break;
    case 32: xpass_body<32, false>(sa, it.S, it.iters, it.x, 0, 0); break;
    case 64: xpass_body<64, false>(sa, it.S, it.iters, it.x, 0, 0); break;
    case 128: xpass_body<128, false>(sa, it.S, it.iters, it.x, 0, 0); break;
    case 256: xpass_body<256, false>(sa, it.S, it.iters, it.x, 0, 0); break;
    case 512: xpass_body<512, false>(sa, it.S, it.iters, it.x, 0, 0); break;
    default: break;
  }
}

__global__ void __launch_bounds__(kEnsThreads, 2) k_zstep_ens(const StageArgs* __restrict__ args,
                                                              const EnsItem* __restrict__ items) {
  __shared__ StageArgs sa;
  const EnsItem it = items[blockIdx.x];
  if (threadIdx.x == 0) sa = args[it.run];
  __syncthreads();
  if (sa.zkernel == 2 && zc_fits(sa.g.N3)) z_step_c_body<kCC, true>(sa, it.x, 0);
  else if ((sa.g.N3 + 7) / 8 >= 48) z_step_body<8, true>(sa, it.x, 0);
  else z_step_body<8, false>(sa, it.x, 0);
}


// One RK stage of every member in one launch: blocks claim work items from
// counters[0] in order, all x-pass items first (largest members first), then
// all z-step items. A z-step item of member r starts once member r's x-pass
// items have all finished (counters[1 + r] reaches xneed[r]). A block claims
// its next item as it starts the current one, so the claim's latency hides
// behind the work; every wait still ends: an item claimed ahead always has a
// higher index than the claiming block's current item, so every x-pass item
// is being run or is next after an x-pass item being run, and x-pass items
// wait on nothing. The waits are bounded all the same: one that runs out
// sets *err and skips its item. The host clears the counters before each step.
constexpr long long kEnsSpin = 1ll << 24;   // x 64 ns: about a second

__global__ void __launch_bounds__(kEnsThreads, 2) k_ens_stage(const StageArgs* __restrict__ args,
                                                              const EnsItem* __restrict__ xitems, int nx,
                                                              const EnsItem* __restrict__ zitems, int nz,
                                                              int* counters, const int* __restrict__ xneed,
                                                              int* err) {
  __shared__ __align__(16) StageArgs sa;
  __shared__ int next, have, ok;
  static_assert(sizeof(StageArgs) % sizeof(int) == 0, "StageArgs copied as words");
  if (threadIdx.x == 0) {
    next = atomicAdd(&counters[0], 1);
    have = -1;
  }
  __syncthreads();
  for (;;) {
    const int i = next;
    if (i >= nx + nz) break;
    const bool xp = i < nx;
    const EnsItem it = xp ? xitems[i] : zitems[i - nx];
    const bool fresh = it.run != have;
    __syncthreads();   // everyone has read next and have
    if (threadIdx.x == 0) {
      next = atomicAdd(&counters[0], 1);
      have = it.run;
      ok = 1;
    }
    if (fresh) {   // this member's stage arguments, copied by the block's threads
      const int* src = reinterpret_cast<const int*>(args + it.run);
      int* dst = reinterpret_cast<int*>(&sa);
      for (int w = threadIdx.x; w < (int)(sizeof(StageArgs) / sizeof(int)); w += blockDim.x) dst[w] = src[w];
    }
    if (!xp && threadIdx.x == 0) {
      const volatile int* done = counters + 1 + it.run;
      long long n = 0;
      while (*done < xneed[it.run] && n < kEnsSpin) {
        __nanosleep(64);
        n++;
      }
      if (*done < xneed[it.run]) {
        ok = 0;
        atomicExch(err, 1);
      }
      __threadfence();   // the member's x-pass results before its z step reads them
    }
    __syncthreads();
    if (xp) {
      switch (sa.g.N1) {
        case 16: xpass_body<16, false>(sa, it.S, it.iters, it.x, 0, 0); break;
        case 32: xpass_body<32, false>(sa, it.S, it.iters, it.x, 0, 0); break;
        case 64: xpass_body<64, false>(sa, it.S, it.iters, it.x, 0, 0); break;
        case 128: xpass_body<128, false>(sa, it.S, it.iters, it.x, 0, 0); break;
        case 256: xpass_body<256, false>(sa, it.S, it.iters, it.x, 0, 0); break;
        case 512: xpass_body<512, false>(sa, it.S, it.iters, it.x, 0, 0); break;
        default: break;
      }
      __syncthreads();
      if (threadIdx.x == 0) {
        __threadfence();   // this item's r rows, before it counts as done
        atomicAdd(&counters[1 + it.run], 1);
      }
    } else if (ok) {   // the member's own z kernel: one lane per complex mode, or one per component
      if (sa.zkernel == 2 && zc_fits(sa.g.N3)) z_step_c_body<kCC, true>(sa, it.x, 0);
      else if ((sa.g.N3 + 7) / 8 >= 48) z_step_body<8, true>(sa, it.x, 0);
      else z_step_body<8, false>(sa, it.x, 0);
    }
    __syncthreads();
  }
}


// ====================================================== factorisation ====
// Thomas factors of every (factor set, mode) in FP64 (Tridiagonal.h:14-27):
// inv_den_j = 1/(b_j - a_j C_{j-1}), stored as float. Rows follow
// UpdateForTimestep (IMEXRK.h:502-545) and the Laplacian of the constructor
// (IMEXRK.h:55-78) with Neumannify / Dirichlify (Differentiation.h:17-59).
__global__ void k_factor(Geo g, const double* __restrict__ bands, const double* __restrict__ kx,
                         const double* __restrict__ ky, double h0, double h1, double h2, double Re,
                         double Pr, float* inv_den) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  const int fs = blockIdx.y;
  const int N = g.N3;
  if (m >= g.Pp) return;
  float* out = inv_den + (size_t)fs * N * g.Pp + m;
  if (m >= g.P) {
    for (int j = 0; j < N; j++) out[(size_t)j * g.Pp] = 0.f;
    return;
  }
  const int q = m / g.K1, j1 = m - q * g.K1;
  const double kk = -(kx[j1] * kx[j1]) + -(ky[q] * ky[q]);
  const bool lap = (fs == kFS_Lap);
  const int fam = lap ? 0 : fs / 3, k = lap ? 0 : fs % 3;
  const bool dir = (fam == 2);
  const double h = k == 0 ? h0 : (k == 1 ? h1 : h2);
  const double s = 0.5 * h;
  const double den_re = (fam == 1) ? Re * Pr : Re;
  const double* lo = bands + (dir ? 3 : 0) * N;
  const double* di = bands + (dir ? 4 : 1) * N;
  const double* up = bands + (dir ? 5 : 2) * N;
  double Cprev = 0.0;
  for (int j = 0; j < N; j++) {
    double aj, bj, cj;
    if (lap) {
      aj = lo[j]; bj = di[j] + kk; cj = up[j];
    } else {
      aj = -(s * lo[j]) / den_re; bj = 1.0 - (s * (di[j] + kk)) / den_re; cj = -(s * up[j]) / den_re;
    }
    if (!dir) {   // Neumannify
      if (j == 0) { bj = 1; cj = 0; }
      if (j == 1) { aj = 0; bj = 1; cj = -1; }
      if (j == N - 2) { aj = 1; bj = -1; cj = 0; }
      if (j == N - 1) { aj = 0; bj = 1; cj = 0; }
      if (lap && m == 0 && j == 1) cj = 0;   // (0,0) mode pinned
    } else {      // Dirichlify
      if (j <= 2) { aj = 0; bj = 1; cj = 0; }
      if (j >= N - 2) { aj = 0; bj = 1; cj = 0; }
    }
    if (j == N - 1) cj = 0;
    double den = (j == 0) ? bj : bj - aj * Cprev;
    out[(size_t)j * g.Pp] = (float)(1.0 / den);
    Cprev = cj / den;
  }
}

// ============================================== layout transposes ====
// reference layout [N2][M1][N3] (z fastest) <-> kept layout [N3][Pp]
__global__ void k_gather_ref(Geo g, const float2* __restrict__ ref, float2* __restrict__ kept) {
  __shared__ float2 tile[32][33];
  const int M1 = g.N1 / 2 + 1;
  const int m0 = blockIdx.x * 32, jz0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    int m = m0 + r, jz = jz0 + threadIdx.x;
    float2 v = make_float2(0.f, 0.f);
    if (m < g.P && jz < g.N3) {
      int q = m / g.K1, j1 = m - q * g.K1;
      int n2 = n2_of_q(q, g.Ky, g.K2, g.N2);
      v = ref[((size_t)M1 * n2 + j1) * g.N3 + jz];
    }
    tile[r][threadIdx.x] = v;
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    int jz = jz0 + r, m = m0 + threadIdx.x;
    if (jz < g.N3 && m < g.Pp) kept[(size_t)jz * g.Pp + m] = tile[threadIdx.x][r];
  }
}

__global__ void k_scatter_ref(Geo g, const float2* __restrict__ kept, float2* __restrict__ ref) {
  __shared__ float2 tile[32][33];
  const int M1 = g.N1 / 2 + 1;
  const int m0 = blockIdx.x * 32, jz0 = blockIdx.y * 32;
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    int jz = jz0 + r, m = m0 + threadIdx.x;
    tile[threadIdx.x][r] = (jz < g.N3 && m < g.P) ? kept[(size_t)jz * g.Pp + m] : make_float2(0.f, 0.f);
  }
  __syncthreads();
  for (int r = threadIdx.y; r < 32; r += blockDim.y) {
    int m = m0 + r, jz = jz0 + threadIdx.x;
    if (m < g.P && jz < g.N3) {
      int q = m / g.K1, j1 = m - q * g.K1;
      int n2 = n2_of_q(q, g.Ky, g.K2, g.N2);
      ref[((size_t)M1 * n2 + j1) * g.N3 + jz] = tile[r][threadIdx.x];
    }
  }
}

// ============================================================ energies ====
// InnerProd (Integration.h:282-311) of each field pair in FP64: per level the
// sum over kept modes of w_m Re(a conj b) with w = 1 for (0,0) and 2 otherwise,
// then the vertical quadrature. out[pair*4 + f] accumulates field f
// (0 u1, 1 u2, 2 u3, 3 b).
__global__ void k_inner(Geo g, const float2* __restrict__ Sa, const float2* __restrict__ Sb,
                        const float* __restrict__ zc, double* out) {
  const int j = blockIdx.x;
  const int pair = blockIdx.y;
  const int f = blockIdx.z;
  const float2* a = Sa + ((size_t)(pair * 5 + f) * g.N3 + j) * g.Pp;
  const float2* b = Sb + ((size_t)(pair * 5 + f) * g.N3 + j) * g.Pp;
  double s = 0.0;
  for (int m = threadIdx.x; m < g.P; m += blockDim.x) {
    float2 x = a[m], y = b[m];
    double v = (double)x.x * y.x + (double)x.y * y.y;
    s += (m == 0) ? v : 2.0 * v;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
    const float wz = zc[(f == 2 ? ZC_WZD : ZC_WZN) * g.N3 + j];
    if (wz != 0.f) atomicAdd(out + pair * 4 + f, t * (double)wz);
  }
}

// The squared-gradient integrals of the dissipation rates (sf_dissipation),
// InnerProd (Integration.h:282-311) of each gradient component at the
// location it lives on, in FP64: per level j the sum over kept modes of
// w_m [ (kx^2 + ky^2) |a_j|^2 wz(j) + |vertical difference|^2 / dz ], with
//   u1, u2, b (Neumann): ddz lands on Dirichlet rows, (a_j - a_{j-1}) / DY_j,
//                        integrated over rows 2..N3-2 with weights DY_j;
//   u3 (Dirichlet):      ddz lands on Neumann rows, (a_{j+1} - a_j) / DYF_j,
//                        integrated over rows 1..N3-2 with weights DYF_j
// (Differentiation.cpp:35-61, Integration.h:5-35). out[run*4 + f] accumulates.
__global__ void k_grad_sq(Geo g, const float2* __restrict__ S, const float* __restrict__ zc,
                          const double* __restrict__ kxd, const double* __restrict__ kyd, double* out) {
  const int j = blockIdx.x, run = blockIdx.y, f = blockIdx.z;
  const int N3 = g.N3;
  const bool dir = f == 2;
  const float2* a = S + ((size_t)(run * 5 + f) * N3 + j) * g.Pp;
  const double wz = (double)zc[(dir ? ZC_WZD : ZC_WZN) * N3 + j];
  int jn = -1;
  double iv = 0.0;
  if (!dir && j >= 2 && j <= N3 - 2) { jn = j - 1; iv = (double)zc[ZC_DND_DI * N3 + j]; }   // 1/DY_j
  if (dir && j >= 1 && j <= N3 - 2) { jn = j + 1; iv = (double)zc[ZC_DDN_UP * N3 + j]; }   // 1/DYF_j
  const float2* an = S + ((size_t)(run * 5 + f) * N3 + (jn >= 0 ? jn : j)) * g.Pp;
  double s = 0.0;
  for (int m = threadIdx.x; m < g.P; m += blockDim.x) {
    const int q = m / g.K1, j1 = m - q * g.K1;
    const double kk = kxd[j1] * kxd[j1] + (g.dim3 ? kyd[q] * kyd[q] : 0.0);
    const float2 x = a[m];
    double v = kk * ((double)x.x * x.x + (double)x.y * x.y) * wz;
    if (jn >= 0) {
      const float2 y = an[m];
      const double dx = (double)x.x - y.x, dy = (double)x.y - y.y;
      v += (dx * dx + dy * dy) * iv;
    }
    s += (m == 0) ? v : 2.0 * v;
  }
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  __shared__ double red[32];
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
  __syncthreads();
  if (threadIdx.x == 0) {
    double t = 0.0;
    for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
    if (t != 0.0) atomicAdd(out + run * 4 + f, t);
  }
}

// ======================================================== launchers ====
static inline unsigned cdiv(long long a, long long b) { return (unsigned)((a + b - 1) / b); }

struct XShape {
  int S, iters, threads;
  size_t bytes;
};

// launch shape of the x pass: slab height S, slabs per block, threads, bytes
template <int N1, bool LIN>
static XShape xpass_shape(const StageArgs& a, int nruns) {
  const Geo& g = a.g;
  const int tlm = LIN ? a.tlm : 0;
  constexpr int G = FFTShape<N1>::G, BUF = fft_buf_stride<N1>();
  const int nprod = g.dim3 ? P_COUNT : 6;
  // threads: enough lane groups for all phase-A transforms of a slab (one
  // round), at least two warps, at most kXMaxThreads
  auto threads = [&](int S) {
    int groups = a.xgroups > 0 ? a.xgroups : 2 * (S + 2);
    int t = ((groups * G + 31) / 32) * 32;
    return t < 64 ? 64 : (t > kXMaxThreads ? kXMaxThreads : t);
  };
  auto bytes = [&](int S, int pre) { return x_layout(S, N1, g.K1, g.dim3, LIN, BUF, threads(S) / G, tlm, pre).bytes; };
  (void)nprod;
  // largest slab whose shared memory lets two blocks share an SM, then
  // smaller slabs while the grid would leave SMs idle
  const int cand[] = {8, 6, 4, 3, 2};
  int S = 2;
  for (int c : cand)
    if (bytes(c, g.dim3) <= 112 * 1024) { S = c; break; }
  if (g.dim3 && S > 4) S = 4;
  for (int i = 0; i < 5; i++) {
    if (cand[i] >= S) continue;
    if ((long long)((g.N3 + S - 1) / S) * g.N2 * nruns >= 2 * 148) break;
    S = cand[i];
  }
  // slabs per block: in 3D as many as keep at least two waves of blocks, up
  // to 6 (measured at 256 x 128 x 384: 6 slabs 2.5% faster per step than 1,
  // 12 slower); in 2D one (carrying rows saves transforms but not lockstep
  // rounds there, and the extra barriers cost more)
  int iters = 1;
  while (g.dim3 && iters < 6 && S * (iters + 1) <= g.N3 &&
         (long long)cdiv(g.N3, S * (iters + 1)) * g.N2 * nruns >= 4 * 148)
    iters++;
  if (a.xslabs > 0) iters = std::min<int>(a.xslabs, (int)cdiv(g.N3, S));
  if (iters > 1 && bytes(S, 1) > 227 * 1024) iters = 1;   // no room for the prefetch buffer
  return XShape{S, iters, threads(S), bytes(S, iters > 1)};
}

// one launch over the level columns a.xcol0 .. a.xcol0 + a.xcols - 1 (all
// when a.xcols = 0); a column is the S * iters levels one block walks through
template <int N1, bool LIN>
static void xpass_launch(const StageArgs& a, int nruns, cudaStream_t st) {
  const Geo& g = a.g;
  const XShape x = xpass_shape<N1, LIN>(a, nruns);
  const int ncol = (int)cdiv(g.N3, x.S * x.iters);
  const int cols = a.xcols > 0 ? a.xcols : ncol - a.xcol0;
  dim3 grid(cols, g.N2, nruns);
  k_xpass<N1, LIN><<<grid, x.threads, x.bytes, st>>>(a, x.S, x.iters);
}

template <int N1>
static int xpass_col_levels(const StageArgs& a, bool L, int nruns) {
  const XShape x = L ? xpass_shape<N1, true>(a, nruns) : xpass_shape<N1, false>(a, nruns);
  return x.S * x.iters;
}

static int xpass_column_levels(const StageArgs& a, bool L, int nruns) {
  switch (a.g.N1) {
    case 16: return xpass_col_levels<16>(a, L, nruns);
    case 32: return xpass_col_levels<32>(a, L, nruns);
    case 64: return xpass_col_levels<64>(a, L, nruns);
    case 128: return xpass_col_levels<128>(a, L, nruns);
    case 256: return xpass_col_levels<256>(a, L, nruns);
    default: return xpass_col_levels<512>(a, L, nruns);
  }
}

static void launch_xpass_runs(const StageArgs& a, bool L, int nruns, cudaStream_t st) {
  switch (a.g.N1) {
    case 16: L ? xpass_launch<16, true>(a, nruns, st) : xpass_launch<16, false>(a, nruns, st); break;
    case 32: L ? xpass_launch<32, true>(a, nruns, st) : xpass_launch<32, false>(a, nruns, st); break;
    case 64: L ? xpass_launch<64, true>(a, nruns, st) : xpass_launch<64, false>(a, nruns, st); break;
    case 128: L ? xpass_launch<128, true>(a, nruns, st) : xpass_launch<128, false>(a, nruns, st); break;
    case 256: L ? xpass_launch<256, true>(a, nruns, st) : xpass_launch<256, false>(a, nruns, st); break;
    case 512: L ? xpass_launch<512, true>(a, nruns, st) : xpass_launch<512, false>(a, nruns, st); break;
  }
}

// the x pass of every run: one launch, or for a tangent-linear batch one
// nonlinear launch for the base runs and one linear launch for the rest
static int launch_xpass(const StageArgs& a, cudaStream_t st) {
  if (a.tlm > 0) {
    StageArgs b = a;
    b.run_offset = 0;
    launch_xpass_runs(b, false, a.tlm, st);
    b.run_offset = a.tlm;
    launch_xpass_runs(b, true, a.g.nrun - a.tlm, st);
    return 2;
  }
  StageArgs b = a;
  b.run_offset = 0;
  if (a.xkernel == 1 && xmarch_supported(a)) {
    // the same level columns as the slab kernel's launch would cover
    const int lv = xpass_column_levels(a, false, a.g.nrun);
    const int ncol = (int)cdiv(a.g.N3, lv);
    const int c1 = a.xcols > 0 ? a.xcol0 + a.xcols : ncol;
    return launch_xmarch(b, a.xcol0 * lv, std::min(a.g.N3, c1 * lv), st);
  }
  launch_xpass_runs(b, a.linear != 0, a.g.nrun, st);
  return 1;
}

// nz = runs x fields transformed (blockIdx.z = 4 run + field); a single
// field of a single run (nz = 1) reads and writes that field only
template <int N2>
static void ify_launch(const StageArgs& a, int nz, cudaStream_t st) {
  const int nl = a.nlvl > 0 ? a.nlvl : a.g.N3 - a.lvl0;
  if (nz % 4 == 0)   // whole runs: the fields in packed pairs
    k_ifft_y2<N2><<<dim3(cdiv(a.g.K1, ycols<N2>()), nl, nz / 2), kYThreads, 0, st>>>(a);
  else
    k_ifft_y<N2><<<dim3(cdiv(a.g.K1, ycols<N2>()), nl, nz), kYThreads, 0, st>>>(a);
}
template <int N2>
static void fy_launch(const StageArgs& a, cudaStream_t st) {
  const int nl = a.nlvl > 0 ? a.nlvl : a.g.N3 - a.lvl0;
  k_fft_y<N2><<<dim3(cdiv(a.g.K1, ycols<N2>()), nl, a.g.nrun * 4), kYThreads, 0, st>>>(a);
}
static void launch_ifft_y_z(const StageArgs& a, int nz, cudaStream_t st) {
  switch (a.g.N2) {
    case 16: ify_launch<16>(a, nz, st); break;
    case 32: ify_launch<32>(a, nz, st); break;
    case 64: ify_launch<64>(a, nz, st); break;
    case 128: ify_launch<128>(a, nz, st); break;
    case 256: ify_launch<256>(a, nz, st); break;
  }
}
static void launch_ifft_y(const StageArgs& a, int nrun, cudaStream_t st) { launch_ifft_y_z(a, nrun * 4, st); }
static void launch_fft_y(const StageArgs& a, cudaStream_t st) {
  switch (a.g.N2) {
    case 16: fy_launch<16>(a, st); break;
    case 32: fy_launch<32>(a, st); break;
    case 64: fy_launch<64>(a, st); break;
    case 128: fy_launch<128>(a, st); break;
    case 256: fy_launch<256>(a, st); break;
  }
}
int launch_fft_y_combos(const StageArgs& a, cudaStream_t st) {
  launch_fft_y(a, st);
  return 1;
}

// opt-in shared-memory limits of every kernel, set once per process before
// any launch (and outside stream capture)
int prepare_kernels() {
  const int lim = 227 * 1024;
  cudaError_t e = cudaSuccess;
#define ATTR(K) if (e == cudaSuccess) e = cudaFuncSetAttribute(K, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  ATTR((k_xpass<16, false>)) ATTR((k_xpass<32, false>)) ATTR((k_xpass<64, false>))
  ATTR((k_xpass<128, false>)) ATTR((k_xpass<256, false>)) ATTR((k_xpass<512, false>))
  ATTR((k_xpass<16, true>)) ATTR((k_xpass<32, true>)) ATTR((k_xpass<64, true>))
  ATTR((k_xpass<128, true>)) ATTR((k_xpass<256, true>)) ATTR((k_xpass<512, true>))
  ATTR(k_z_proj_chunked<8>) ATTR(k_z_proj_chunked<16>)
  ATTR((k_z_step<8, false>)) ATTR((k_z_step<8, true>)) ATTR((k_z_step<16, false>)) ATTR((k_z_step<16, true>))
#undef ATTR
  if (e == cudaSuccess && prepare_xmarch_kernels() != 0) return -1;
  if (e == cudaSuccess && prepare_zstep_tma_kernels() != 0) return -1;
  if (e == cudaSuccess && prepare_zstep_c_kernels() != 0) return -1;
  return e == cudaSuccess ? 0 : -1;
}

static size_t zchunk_smem(const Geo& g, int zw) { return sizeof(float) * ((size_t)g.N3 * 32 + 3 * zw * 32); }

// z chunks per block: 16 (shorter serial sweeps, one 16-warp block per SM)
// when the grid leaves SMs without a block, else 8 (three blocks per SM)
static int z_chunks(const Geo& g, int fields) {
  return (long long)cdiv(g.P, 16) * fields * g.nrun < 148 ? 16 : 8;
}

int launch_project(const StageArgs& a, cudaStream_t st) {
  const Geo& g = a.g;
  const dim3 grid(cdiv(g.P, 16), 1, g.nrun);
  if ((a.zchunks ? a.zchunks : z_chunks(g, 1)) == 16)
    k_z_proj_chunked<16><<<grid, 16 * 32, zchunk_smem(g, 16), st>>>(g, a.Sn, a.S, a.Sn, a.zc, a.fa, a.fc,
                                                                      a.inv_den, a.kx, a.ky, a.pm);
  else
    k_z_proj_chunked<8><<<grid, 8 * 32, zchunk_smem(g, 8), st>>>(g, a.Sn, a.S, a.Sn, a.zc, a.fa, a.fc, a.inv_den,
                                                                   a.kx, a.ky, a.pm);
  return 1;
}

// the merged z pass (CN solves of every field, then the projection): one
// block per 16 modes, so the chunk count follows from the mode groups alone;
// chunks of 48 levels or more take the variant with end-test-free interior
// sweeps (measured 7% faster at 384 levels in 8 chunks, and slower with
// 32-level chunks, where it is not used)
// the z pass as k_z_step_tma: where the solver asks for it, has its tensor
// maps, and the launch takes 8 chunks
bool z_step_takes_tma(const StageArgs& a) {
  const int zw = a.zchunks ? a.zchunks : z_chunks(a.g, 1);
  return a.zkernel == 1 && a.zmaps && zw == 8 && zstep_tma_supported(a.g);
}

// the z pass as k_z_step_c: where the solver asks for it and the grid has
// the levels for its 16 chunks (the chunk count is the kernel's own)
bool z_step_takes_c(const StageArgs& a) { return a.zkernel == 2 && zstep_c_supported(a.g); }

static void launch_z_step(const StageArgs& a, cudaStream_t st) {
  const Geo& g = a.g;
  const dim3 zgrid(cdiv(g.P, 16), 1, g.nrun);
  const int zw = a.zchunks ? a.zchunks : z_chunks(g, 1);
  if (z_step_takes_c(a) && launch_z_step_c(a, st)) return;
  if (z_step_takes_tma(a) && launch_z_step_tma(a, st)) return;
  const bool ic = cdiv(g.N3, zw) >= 48;
  if (zw == 16) {
    if (ic) k_z_step<16, true><<<zgrid, 16 * 32, zchunk_smem(g, 16), st>>>(a);
    else k_z_step<16, false><<<zgrid, 16 * 32, zchunk_smem(g, 16), st>>>(a);
  } else {
    if (ic) k_z_step<8, true><<<zgrid, 8 * 32, zchunk_smem(g, 8), st>>>(a);
    else k_z_step<8, false><<<zgrid, 8 * 32, zchunk_smem(g, 8), st>>>(a);
  }
}

const char* stage_kernel_name(const Geo& g, int i) {
  static const char* n3[] = {"k_ifft_y", "k_xpass", "k_fft_y", "k_z_step"};
  static const char* n2[] = {"k_xpass", "k_z_step"};
  return g.dim3 ? n3[i] : n2[i];
}
int stage_kernel_count(const Geo& g) { return g.dim3 ? 4 : 2; }

// The 3D x-y pass in level bands: band b's inverse y transforms (stream y1,
// all bands back to back), x pass (the stage's stream, after the inverse
// transforms of its own band and of the band above, whose lowest level its
// z stencils read) and forward y transforms (stream y2, after that band's x
// pass). The memory-bound y transforms of the other bands then run beside the
// compute-bound x pass instead of before and after it. Bands follow the x
// pass's block columns, so no block straddles two bands.
static int launch_xy_banded(const StageArgs& a, cudaStream_t st, const XYAux& aux) {
  const Geo& g = a.g;
  const int lv = xpass_column_levels(a, a.linear != 0, g.nrun);
  const int ncol = (int)cdiv(g.N3, lv);
  const int B = std::min(std::min(aux.bands, kMaxBands), ncol);
  auto c0 = [&](int b) { return (int)((long long)ncol * b / B); };
  auto band = [&](int b) {
    StageArgs y = a;
    y.lvl0 = c0(b) * lv;
    y.nlvl = std::min(g.N3, c0(b + 1) * lv) - y.lvl0;
    return y;
  };
  cudaEventRecord(aux.fork, st);
  cudaStreamWaitEvent(aux.y1, aux.fork, 0);
  cudaStreamWaitEvent(aux.y2, aux.fork, 0);
  for (int b = 0; b < B; b++) {
    launch_ifft_y(band(b), g.nrun, aux.y1);
    cudaEventRecord(aux.ev_ify[b], aux.y1);
  }
  for (int b = 0; b < B; b++) {
    cudaStreamWaitEvent(st, aux.ev_ify[std::min(b + 1, B - 1)], 0);
    StageArgs x = a;
    x.xcol0 = c0(b);
    x.xcols = c0(b + 1) - c0(b);
    launch_xpass(x, st);
    cudaEventRecord(aux.ev_x[b], st);
  }
  for (int b = 0; b < B; b++) {
    cudaStreamWaitEvent(aux.y2, aux.ev_x[b], 0);
    launch_fft_y(band(b), aux.y2);
  }
  cudaEventRecord(aux.join, aux.y2);
  cudaStreamWaitEvent(st, aux.join, 0);
  return 3 * B;
}

int launch_stage(const StageArgs& a, cudaStream_t st, cudaEvent_t* ev, const XYAux* aux) {
  const Geo& g = a.g;
  if (g.dim3 && aux && aux->bands > 1 && !ev && !a.tlm) {
    const int n = launch_xy_banded(a, st, *aux);
    launch_z_step(a, st);
    return n + 1;
  }
  int n = 0;
  auto mark = [&]() {
    if (ev) cudaEventRecord(ev[n], st);
    n++;
  };
  if (g.dim3) {
    launch_ifft_y(a, g.nrun, st);
    mark();
  }
  const int extra = launch_xpass(a, st) - 1;   // a tangent-linear batch launches the x pass twice
  mark();
  if (g.dim3) {
    launch_fft_y(a, st);
    mark();
  }
  launch_z_step(a, st);
  mark();
  return n + extra;
}

int launch_z_solves(const StageArgs& a, cudaStream_t st) {
  launch_z_step(a, st);
  return 1;
}

int launch_factor(const Geo& g, const double* bands, const double* kx, const double* ky, double h0, double h1,
                  double h2, double Re, double Pr, float* inv_den, cudaStream_t st) {
  k_factor<<<dim3(cdiv(g.Pp, 128), kNumFS), 128, 0, st>>>(g, bands, kx, ky, h0, h1, h2, Re, Pr, inv_den);
  return 1;
}

int launch_gather_ref(const Geo& g, const float2* ref, float2* kept, cudaStream_t st) {
  k_gather_ref<<<dim3(cdiv(g.Pp, 32), cdiv(g.N3, 32)), dim3(32, 8), 0, st>>>(g, ref, kept);
  return 1;
}

int launch_scatter_ref(const Geo& g, const float2* kept, float2* ref, cudaStream_t st) {
  k_scatter_ref<<<dim3(cdiv(g.P, 32), cdiv(g.N3, 32)), dim3(32, 8), 0, st>>>(g, kept, ref);
  return 1;
}

static int fft_G(int N) { return N >= 256 ? 16 : (N >= 64 ? 8 : 4); }
static int fft_bufstride(int N) {
  switch (N) {
    case 16: return fft_buf_stride<16>();
    case 32: return fft_buf_stride<32>();
    case 64: return fft_buf_stride<64>();
    case 128: return fft_buf_stride<128>();
    case 256: return fft_buf_stride<256>();
    default: return fft_buf_stride<512>();
  }
}

size_t ensemble_xpass_smem(int N1, int S) {
  return x_layout(S, N1, N1 / 3, 0, 0, fft_bufstride(N1), kEnsThreads / fft_G(N1), 0, 0).bytes;
}
size_t ensemble_zstep_smem(int N3) {
  return std::max(sizeof(float) * ((size_t)N3 * 32 + 3 * 8 * 32), zc_smem_bytes(N3));
}

int launch_xpass_ens(const StageArgs* args, const EnsItem* items, int nitems, size_t smem, cudaStream_t st) {
  k_xpass_ens<<<nitems, kEnsThreads, smem, st>>>(args, items);
  return 1;
}
int launch_zstep_ens(const StageArgs* args, const EnsItem* items, int nitems, size_t smem, cudaStream_t st) {
  k_zstep_ens<<<nitems, kEnsThreads, smem, st>>>(args, items);
  return 1;
}
int launch_ens_stage(const StageArgs* args, const EnsItem* xitems, int nx, const EnsItem* zitems, int nz,
                     int* counters, const int* xneed, int* err, int blocks, size_t smem, cudaStream_t st) {
  k_ens_stage<<<blocks, kEnsThreads, smem, st>>>(args, xitems, nx, zitems, nz, counters, xneed, err);
  return 1;
}
int ensemble_stage_blocks(size_t smem) {
  int per_sm = 0, sms = 0, dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess ||
      cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_ens_stage, kEnsThreads, smem) != cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return 148;
  return (per_sm < 1 ? 1 : per_sm) * sms;
}
int prepare_ensemble_kernels() {
  const int lim = 227 * 1024 - (int)sizeof(StageArgs) - 64;
  cudaError_t e = cudaFuncSetAttribute(k_xpass_ens, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_zstep_ens, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  if (e == cudaSuccess) e = cudaFuncSetAttribute(k_ens_stage, cudaFuncAttributeMaxDynamicSharedMemorySize, lim);
  return e == cudaSuccess ? 0 : -1;
}

int launch_grad_sq(const Geo& g, const float2* S, int nruns, const float* zc, const double* kxd, const double* kyd,
                   double* out, cudaStream_t st) {
  k_grad_sq<<<dim3(g.N3, nruns, 4), 256, 0, st>>>(g, S, zc, kxd, kyd, out);
  return 1;
}

int launch_energy(const Geo& g, const float2* Sa, const float2* Sb, int npairs, const float* zc, const float* Ri,
                  double* out, cudaStream_t st) {
  (void)Ri;
  k_inner<<<dim3(g.N3, npairs, 4), 256, 0, st>>>(g, Sa, Sb, zc, out);
  return 1;
}

// nodal field of one modal field (kept layout, one run) -> base [N3][N2][N1]
// via the same transforms as the x pass: used once per set_base.
__global__ void k_base_x(Geo g, const float2* __restrict__ rows, long long row_stride_level,
                         long long row_stride_y, float* __restrict__ out, const float2* __restrict__ tw) {
  extern __shared__ float2 wsm[];
  const int t = blockIdx.x, y = blockIdx.y;
  const int lane = threadIdx.x;
  float2* wk = wsm;
  const float2* src = rows + (size_t)t * row_stride_level + (size_t)y * row_stride_y;
  for (int x = lane; x < g.N1; x += 32) wk[x] = make_float2(0.f, 0.f);
  __syncwarp();
  for (int k = lane; k < g.K1; k += 32) {
    float2 A = src[k];
    if (k == 0) wk[0] = make_float2(A.x, 0.f);
    else { wk[k] = A; wk[g.N1 - k] = cconj(A); }
  }
  __syncwarp();
  warp_fft(wk, g.N1, g.logN1, tw, true, lane);
  float* o = out + ((size_t)t * g.N2 + y) * g.N1;
  for (int x = lane; x < g.N1; x += 32) o[x] = wk[x].x;
}

int launch_base_nodal(const Geo& g, const float2* kept_modal, int field, float* base_out, const float2* tw,
                      float* scratch_mixed, cudaStream_t st) {
  (void)field;
  if (!g.dim3) {
    k_base_x<<<dim3(g.N3, 1), 32, sizeof(float2) * g.N1, st>>>(g, kept_modal, g.Pp, 0, base_out, tw);
    return 1;
  }
  // 3D: inverse y transform into scratch [N3][N2][K1], then x
  StageArgs a = {};
  a.g = g;
  a.g.nrun = 1;
  a.S = kept_modal;   // treated as field 0 of a one-run state
  a.mixin = reinterpret_cast<float2*>(scratch_mixed);
  a.tw = tw;
  launch_ifft_y_z(a, 1, st);   // that field only: the input and the scratch hold one field
  k_base_x<<<dim3(g.N3, g.N2), 32, sizeof(float2) * g.N1, st>>>(g, a.mixin, (long long)g.N2 * g.K1, g.K1,
                                                                base_out, tw);
  return 2;
}

}  // namespace sf
