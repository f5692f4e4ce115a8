// The z pass of a stage (ExplicitRK, FinishRHS, CrankNicolson and the Thomas
// solves of every field, IMEXRK.cpp:75-134, then RemoveDivergence,
// IMEXRK.cpp:43-73) with its inputs brought in by the tensor-memory
// accelerator and its Thomas intermediates in tensor memory.
//
// Same decomposition and arithmetic as k_z_step (sf_kernels.cu): a block owns
// 16 modes x {re, im} (one lane each); 8 warps each own one z-chunk of the
// levels; every Thomas system is three sweeps joined by two scans of the
// chunks' affine maps. The first sweep of each system reads every level's
// inputs from HBM. Here each warp keeps the next tiles of its chunk's inputs
// (u_{j+1}, r, r_old, 1/den_j and the coupled fields: 4 levels x 16 modes per
// tile, one cp.async.bulk.tensor instruction each) in flight into a
// three-slot shared-memory ring of its own, each slot tracked by an mbarrier
// that the copies complete; a slot is refilled as soon as the warp has read
// it, with the next tiles of the same system or of the next one, so the first
// sweep reads shared memory at fixed offsets instead of computing global
// addresses. The be_j / D_j values the sweeps hand to each other live in the
// SM's tensor memory (64 columns of the warp's lane quarter per warp), so the
// shared memory holds the rings. Every mbarrier wait is bounded: one that
// runs out sets the solver's error word and the block carries on (its results
// are then wrong, and the host reports the error after its synchronisation).
#include <cstdint>
#include <type_traits>
#include <cuda.h>
#include <cudaTypedefs.h>
#include "sf_internal.cuh"

namespace sf {

constexpr int kZW = 8;                   // warps (z-chunks) per block
constexpr int kZThreads = kZW * 32;
constexpr int kZTL = 4;                  // levels per tile
constexpr int kZNA = 5;                  // full-width tiles (input arrays) per ring slot, at most
constexpr int kZNS = 3;                  // ring slots per chunk
constexpr int kZTCols = 64;              // tensor-memory columns (levels) per warp
constexpr int kZI2 = 16;                 // levels per tensor-memory load in the later sweeps
constexpr int kZP2 = 4;                  // levels loaded ahead in the projection's last sweep
constexpr long long kZWaitCycles = 1ll << 31;   // SM cycles (about a second) before a wait gives up
constexpr long long kZDrainCycles = 1ll << 25;  // the same for the block's last wait on its copies
constexpr int kZIden = kZNA * kZTL * 32;          // offset of the pivots' half-width tile in a slot
constexpr int kZSlotFloats = kZIden + kZTL * 16;

__device__ __forceinline__ uint32_t zs(const void* p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mb_init(uint64_t* b, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(zs(b)), "r"(count) : "memory");
}
__device__ __forceinline__ bool mb_try(uint32_t b, unsigned parity) {
  uint32_t ok;
  asm volatile(
      "{\n\t.reg .pred p;\n\tmbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\tselp.u32 %0, 1, 0, p;\n\t}"
      : "=r"(ok)
      : "r"(b), "r"(parity)
      : "memory");
  return ok != 0;
}
// wait for the phase of the given parity of the barrier at shared address b
// to complete, for at most `limit` SM cycles; a wait that runs out sets the
// block's `bad` word (after which the block's other waits give up at once,
// unless `drain`) and the solver's error word, and returns
__device__ __forceinline__ void mb_wait(uint32_t b, unsigned parity, int* err, int code, volatile int* bad,
                                        long long limit = kZWaitCycles, bool drain = false) {
  if (mb_try(b, parity)) return;
  const long long t0 = clock64();
  for (;;) {
    if (mb_try(b, parity)) return;
    if (!drain && *bad) return;
    if (clock64() - t0 > limit) {
      *bad = 1;
      if (err) atomicExch(err, code);
      return;
    }
  }
}
// the block's barrier for the chunk scans
__device__ __forceinline__ void zc_sync() { asm volatile("bar.sync 1, %0;" ::"n"(kZW * 32) : "memory"); }

__device__ __forceinline__ void tz_st4(uint32_t addr, const float (&v)[kZTL]) {
  static_assert(kZTL == 4, "one 4-column store per tile");
  asm volatile("tcgen05.st.sync.aligned.32x32b.x4.b32 [%0], {%1, %2, %3, %4};" ::"r"(addr), "f"(v[0]), "f"(v[1]),
               "f"(v[2]), "f"(v[3])
               : "memory");
}
__device__ __forceinline__ void tz_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;" ::: "memory"); }
__device__ __forceinline__ void tz_ld16(uint32_t addr, float (&v)[16]) {
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0, %1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15}, [%16];"
      : "=f"(v[0]), "=f"(v[1]), "=f"(v[2]), "=f"(v[3]), "=f"(v[4]), "=f"(v[5]), "=f"(v[6]), "=f"(v[7]),
        "=f"(v[8]), "=f"(v[9]), "=f"(v[10]), "=f"(v[11]), "=f"(v[12]), "=f"(v[13]), "=f"(v[14]), "=f"(v[15])
      : "r"(addr));
  asm volatile("tcgen05.wait::ld.sync.aligned;" ::: "memory");
}
__device__ __forceinline__ void tz_st16(uint32_t addr, const float (&v)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1, %2, %3, %4, %5, %6, %7, %8, %9, %10, %11, %12, %13, %14, "
      "%15, %16};" ::"r"(addr),
      "f"(v[0]), "f"(v[1]), "f"(v[2]), "f"(v[3]), "f"(v[4]), "f"(v[5]), "f"(v[6]), "f"(v[7]), "f"(v[8]), "f"(v[9]),
      "f"(v[10]), "f"(v[11]), "f"(v[12]), "f"(v[13]), "f"(v[14]), "f"(v[15])
      : "memory");
}

// shared memory of the block (the rings in the dynamic part)
struct ZShared {
  uint64_t full[kZW][kZNS];
  float sA[kZW * 32], sB[kZW * 32], sIn[kZW * 32];
  uint32_t tmem_base;
  int bad;   // a wait of this block ran out
};

// the chunks' scans (as k_z_step's), among the compute warps
__device__ __forceinline__ float zt_scan(ZShared& sh, int w, int lane, float A, float B, bool up) {
  sh.sA[w * 32 + lane] = A;
  sh.sB[w * 32 + lane] = B;
  zc_sync();
  if (w == 0) {
    float v = 0.f;
    for (int i = 0; i < kZW; i++) {
      const int k = up ? i : kZW - 1 - i;
      sh.sIn[k * 32 + lane] = v;
      v = sh.sA[k * 32 + lane] * v + sh.sB[k * 32 + lane];
    }
  }
  zc_sync();
  return sh.sIn[w * 32 + lane];
}

// chunk bounds of warp w
__device__ __forceinline__ void zt_chunk(int N3, int w, int& js, int& je) {
  const int chunk = (N3 + kZW - 1) / kZW;
  js = min(N3, w * chunk);
  je = min(N3, js + chunk);
}

// systems of the z pass, in order: 0 u1, 1 u2 (3D), 2 u3, 3 b, 4 the
// projection's first sweep
struct ZTiles {
  int n;            // tiles per ring slot
  unsigned bytes;   // bytes they bring
};
__device__ __forceinline__ ZTiles zt_tiles(int sys, bool use_rold, bool dim3) {
  if (sys == 4) return ZTiles{4, (dim3 ? 3u : 2u) * kZTL * 128 + kZTL * 64};   // U1, [U2], W, 1/den
  const unsigned o = use_rold ? kZTL * 128 : 0;   // r_old only when the stage reads it
  if (sys == 2) return ZTiles{6, 4u * kZTL * 128 + kZTL * 64 + o};
  return ZTiles{5, 3u * kZTL * 128 + kZTL * 64 + o};
}

// the tensor maps of one launch
struct ZTmaps {
  const CUtensorMap *S, *Sn, *R, *O, *I;
};

// a warp's ring: fill k (the k-th tile the warp reads) goes to slot k % kZNS;
// fills are numbered through the systems in order (u1, [u2], u3, b, the
// projection), nt tiles each. Every lane keeps the same copy of the
// counters; lane 0 issues the copies.
struct ZRing {
  float* slots;
  uint32_t sbase, bbase;   // shared addresses of slot 0 and of its barrier
  int kslot, kpar;         // slot and phase parity of the next fill to read
  int kc;                  // fills read
  int issued;              // fills issued
  int islot, it, isys;     // slot, tile and system of the next fill to issue
  int nt;                  // tiles per system of this chunk
};

__device__ __forceinline__ void tma2s(uint32_t dst, const CUtensorMap* map, int x, int y, uint32_t bar) {
  asm volatile(
      "cp.async.bulk.tensor.2d.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3}], [%4];" ::"r"(
          dst),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(bar)
      : "memory");
}
__device__ __forceinline__ void mb_expect_tx_s(uint32_t bar, unsigned bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(bytes) : "memory");
}

// issue the next fill (lane 0): the tile of levels js + 4 it .. + 3 of every
// input of system isys
__device__ __forceinline__ void zr_issue(const StageArgs& a, const ZRing& R, const ZTmaps& M, int js) {
  const Geo& g = a.g;
  const int N3 = g.N3, run = blockIdx.z;
  const int x32 = 32 * blockIdx.x, x16 = 16 * blockIdx.x;
  const bool use_rold = a.hz != 0.f;
  const int sys = g.dim3 ? R.isys : (R.isys == 0 ? 0 : R.isys + 1);   // 0 u1, 1 u2, 2 u3, 3 b, 4 projection
  const uint32_t bar = R.bbase + 8u * R.islot;
  const uint32_t r = R.sbase + (uint32_t)(R.islot * kZSlotFloats * 4);
  const uint32_t ri = r + kZIden * 4;
  constexpr uint32_t A = kZTL * 32 * 4;   // bytes of one full-width tile
  const int j = js + R.it * kZTL;         // the tile's first level
  const int s5 = run * 5 * N3 + j, s4 = run * 4 * N3 + j;
  mb_expect_tx_s(bar, zt_tiles(sys, use_rold, g.dim3 != 0).bytes);
  if (sys < 4) {
    const int fam = sys < 2 ? 0 : (sys == 2 ? 1 : 2);
    const int fs = (fam == 2 ? 1 : (fam == 1 ? 2 : 0)) * 3 + a.stage;
    tma2s(r, M.S, x32, s5 + sys * N3 + 1, bar);                        // u_{j+1}
    tma2s(r + A, M.R, x32, s4 + sys * N3, bar);                        // r
    if (use_rold) tma2s(r + 2 * A, M.O, x32, s4 + sys * N3, bar);      // r_old
    tma2s(ri, M.I, x16, fs * N3 + j, bar);                             // 1/den
    if (fam < 2) tma2s(r + 3 * A, M.S, x32, s5 + 4 * N3, bar);         // p
    if (fam == 1) tma2s(r + 4 * A, M.S, x32, s5 + 3 * N3, bar);        // b
    if (fam == 2) tma2s(r + 3 * A, M.S, x32, s5 + 2 * N3 + 1, bar);    // u3_{j+1}
  } else {
    tma2s(r, M.Sn, x32, s5, bar);                                      // u1 (new)
    if (g.dim3) tma2s(r + A, M.Sn, x32, s5 + N3, bar);                 // u2 (new)
    tma2s(r + 2 * A, M.Sn, x32, s5 + 2 * N3 + 1, bar);                 // u3_{j+1} (new)
    tma2s(ri, M.I, x16, kFS_Lap * N3 + j, bar);                        // 1/den of the Laplacian
  }
}

// issue every fill that has a free slot, up to fill `allowed` (the
// projection's fills wait until the block has written the new velocities);
// a slot is free once the warp has read the fill before it there
__device__ __forceinline__ void zr_top_up(const StageArgs& a, ZRing& R, const ZTmaps& M, int allowed, int js,
                                          int lane) {
  const int target = min(R.kc + kZNS, allowed);
  if (target <= R.issued) return;
  __syncwarp();
  if (lane == 0) asm volatile("fence.proxy.async.shared::cta;" ::: "memory");   // reads before the overwrite
  while (R.issued < target) {
    if (lane == 0) zr_issue(a, R, M, js);
    R.issued++;
    R.islot = R.islot == kZNS - 1 ? 0 : R.islot + 1;
    if (++R.it == R.nt) {
      R.it = 0;
      R.isys++;
    }
  }
}

// the warp's wait for its next fill; returns the slot's floats
__device__ __forceinline__ const float* zr_take(const StageArgs& a, ZShared& sh, ZRing& R) {
  mb_wait(R.bbase + 8u * R.kslot, R.kpar, a.zerr, 1, &sh.bad);
  return R.slots + R.kslot * kZSlotFloats;
}
// after the warp has read the fill: the next fills into the freed slot
__device__ __forceinline__ void zr_done(const StageArgs& a, ZRing& R, const ZTmaps& M, int allowed, int js,
                                        int lane) {
  R.kc++;
  if (++R.kslot == kZNS) {
    R.kslot = 0;
    R.kpar ^= 1;
  }
  zr_top_up(a, R, M, allowed, js, lane);
}

// the second sweep (D_j back into tensor memory) and both scans; returns the
// backward sweep's value at level je
template <class CofF>
__device__ __forceinline__ float zt_sweep2(ZShared& sh, uint32_t tc, int js, int je, float A, float B,
                                           const float* __restrict__ fa, const float* __restrict__ iden, int Pp, int w,
                                           int lane, CofF Cof) {
  tz_wait_st();
  float D = zt_scan(sh, w, lane, A, B, true);
  A = 1.f;
  B = 0.f;
  for (int b0 = 0; b0 < je - js; b0 += kZI2) {
    float v[kZI2], bi[kZI2];
#pragma unroll
    for (int i = 0; i < kZI2; i++) {
      const int j = js + b0 + i;
      bi[i] = j < je ? iden[(size_t)j * Pp] : 0.f;
    }
    tz_ld16(tc + b0, v);
#pragma unroll
    for (int i = 0; i < kZI2; i++) {
      const int j = js + b0 + i;
      if (j < je) {
        const float al = (j == 0) ? 0.f : -fa[j] * bi[i];
        D = al * D + v[i];
        v[i] = D;
        B = B + A * D;
        A = -A * Cof(j, bi[i]);
      }
    }
    tz_st16(tc + b0, v);
  }
  tz_wait_st();
  return zt_scan(sh, w, lane, A, B, false);
}

// the Crank-Nicolson solve of field f of family FAM (0: u1, u2; 1: u3; 2: b):
// k_z_step's z_cn_body with the first sweep read from the ring
template <int FAM>
__device__ __forceinline__ void zt_cn(const StageArgs& a, ZShared& sh, ZRing& R, const ZTmaps& M, int allowed,
                                      const int f, uint32_t tc) {
  const Geo g = a.g;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int m0 = blockIdx.x * 16 + (lane >> 1), c = lane & 1;
  const bool act = m0 < g.P;
  const int m = act ? m0 : 0;
  const int run = blockIdx.z;
  const int N3 = g.N3, Pp = g.Pp;
  int js, je;
  zt_chunk(N3, w, js, je);
  const int q = m / g.K1, j1 = m - q * g.K1;
  const float kxv = a.kx[j1], kyv = a.ky[q];
  const float d1 = -(kxv * kxv), d2 = -(kyv * kyv);
  const float sc = c == 0 ? -1.f : 1.f;   // (i k z)_c = sc * k * z_{1-c}
  constexpr bool dir = (FAM == 1);
  const int fs = (FAM == 2 ? 1 : (dir ? 2 : 0)) * 3 + a.stage;
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
  const float* bc = reinterpret_cast<const float*>(a.S + (size_t)(run * 5 + 3) * N3 * Pp + m) + c;
  const float* wc = reinterpret_cast<const float*>(a.S + (size_t)(run * 5 + 2) * N3 * Pp + m) + c;
  float* rold = reinterpret_cast<float*>(a.rold + (size_t)(run * 4 + f) * N3 * Pp + m) + c;
  float* out = reinterpret_cast<float*>(a.Sn + fo) + c;
  const bool use_rold = (a.hz != 0.f);
  const float kgrad = (f == 0) ? kxv : kyv;
  const size_t S2 = 2 * (size_t)Pp;
  const int ml = lane >> 1;   // this lane's mode within the tile's 16

  // ---- forward, pass 1: right-hand side, be_j, chunk map ----
  float um = js >= 1 && js < N3 ? uc[(js - 1) * S2] : 0.f;
  float u0 = js < N3 ? uc[js * S2] : 0.f;
  float pm1 = (FAM == 1 && js >= 1 && js < N3) ? pc[(js - 1) * S2] : 0.f;
  float bm1 = (FAM == 1 && js >= 1 && js < N3) ? bc[(js - 1) * S2] : 0.f;
  float w0 = (FAM == 2 && js < N3) ? wc[js * S2] : 0.f;
  float A = 1.f, B = 0.f;
  // a chunk clear of both ends (levels 3..N3-4) whose length is a whole number
  // of tiles takes the sweep without the per-level end tests
  const bool interior = js >= 3 && je <= N3 - 4 && (je - js) % kZTL == 0;
  auto sweep1 = [&](auto tag) {
    constexpr bool IN = decltype(tag)::value;
    for (int t0 = js; t0 < je; t0 += kZTL) {
      const float* r = zr_take(a, sh, R);
      float bev[kZTL] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
      for (int i = 0; i < kZTL; i++) {
        const int j = t0 + i;
        if (!IN && j >= je) break;
        const bool nx = IN || j + 1 < N3;
        const float up = nx ? r[(0 * kZTL + i) * 32 + lane] : 0.f;
        float rt = r[(1 * kZTL + i) * 32 + lane];
        const float bo = use_rold ? r[(2 * kZTL + i) * 32 + lane] : 0.f;
        const float bi = r[kZIden + i * 16 + ml];
        float gp = 0.f;
        if (FAM == 0) {
          gp = sc * kgrad * r[(3 * kZTL + i) * 32 + (lane ^ 1)];   // (i k p)_c
        } else if (FAM == 1) {
          const float bp = r[(3 * kZTL + i) * 32 + lane], bx_ = r[(4 * kZTL + i) * 32 + lane];
          if (IN || j >= 2) gp = dnd_lo[j] * pm1 + dnd_di[j] * bp;
          pm1 = bp;
          if ((IN || j >= 1) && !zmode && !a.adjoint) rt += Ri * (full_lo[j] * bm1 + full_di[j] * bx_);   // r3 += Ri Full(b - <b>)
          bm1 = bx_;
        } else {
          const float w1 = nx ? r[(3 * kZTL + i) * 32 + lane] : 0.f;
          const float dw = nx ? 0.5f * w0 + 0.5f * w1 : 0.5f * w0;
          if (!a.adjoint) rt -= dB[j] * dw;   // rB -= dB/dz ReinterpolateDirichlet(u3)
          w0 = w1;
        }
        float rhs = u0;
        if (use_rold) rhs += a.hz * bo;
        rhs += -a.h * gp;
        rhs += a.hb * rt;
        const bool band = IN || (dir ? (j >= 2 && j <= N3 - 2) : (j >= 1 && j <= N3 - 2));
        const float d2u = band ? lo2[j] * um + di2[j] * u0 + up2[j] * up : 0.f;
        rhs += cco * ((d1 * u0 + d2 * u0) + d2u);
        const bool zend = !IN && ((j <= 1) || (j >= N3 - 2) || (dir && j == 2));   // ZeroEnds (Field.h:475-486)
        if (zend) rhs = 0.f;
        const float be = rhs * bi;
        const float al = (!IN && j == 0) ? 0.f : -fa[j] * bi;
        bev[i] = be;
        if (act) rold[j * S2] = rt;
        A = al * A;
        B = al * B + be;
        um = u0;
        u0 = up;
      }
      tz_st4(tc + (uint32_t)(t0 - js), bev);
      zr_done(a, R, M, allowed, js, lane);
    }
  };
  if (interior) sweep1(std::true_type{});
  else sweep1(std::false_type{});
  float x = zt_sweep2(sh, tc, js, je, A, B, fa, iden, Pp, w, lane, [&](int j, float bij) { return fc[j] * bij; });
  // ---- backward: x_j = D_j - C_j x_{j+1} ----
  for (int b0 = ((je - js - 1) / kZI2) * kZI2; b0 >= 0; b0 -= kZI2) {
    float v[kZI2], bi[kZI2];
#pragma unroll
    for (int i = 0; i < kZI2; i++) {
      const int j = js + b0 + i;
      bi[i] = j < je ? iden[(size_t)j * Pp] : 0.f;
    }
    tz_ld16(tc + b0, v);
#pragma unroll
    for (int i = kZI2 - 1; i >= 0; i--) {
      const int j = js + b0 + i;
      if (j < je) {
        x = v[i] - fc[j] * bi[i] * x;
        if (act) out[j * S2] = x;
      }
    }
  }
}

// RemoveDivergence on the new velocities (k_z_step's z_proj_body), the first
// sweep read from the ring
__device__ __forceinline__ void zt_proj(const StageArgs& a, ZShared& sh, ZRing& R, const ZTmaps& M, int allowed,
                                        uint32_t tc) {
  const Geo g = a.g;
  const int lane = threadIdx.x & 31, w = threadIdx.x >> 5;
  const int m0 = blockIdx.x * 16 + (lane >> 1), c = lane & 1;
  const bool act = m0 < g.P;
  const int m = act ? m0 : 0;
  const int run = blockIdx.z;
  const int N3 = g.N3, Pp = g.Pp;
  int js, je;
  zt_chunk(N3, w, js, je);
  const int q = m / g.K1, j1 = m - q * g.K1;
  const float kxv = a.kx[j1], kyv = g.dim3 ? a.ky[q] : 0.f;
  const float sc = c == 0 ? -1.f : 1.f;
  const size_t S2 = 2 * (size_t)Pp;
  float2* U = a.Sn;
  float* u1 = reinterpret_cast<float*>(U + (size_t)(run * 5 + 0) * N3 * Pp + m);
  float* u2 = reinterpret_cast<float*>(U + (size_t)(run * 5 + 1) * N3 * Pp + m);
  float* u3 = reinterpret_cast<float*>(U + (size_t)(run * 5 + 2) * N3 * Pp + m) + c;
  const float* ps = reinterpret_cast<const float*>(a.S + (size_t)(run * 5 + 4) * N3 * Pp + m) + c;
  float* pd = reinterpret_cast<float*>(a.Sn + (size_t)(run * 5 + 4) * N3 * Pp + m) + c;
  const float* __restrict__ a_ = a.fa + (size_t)kFS_Lap * N3;
  const float* __restrict__ c_ = a.fc + (size_t)kFS_Lap * N3;
  const float* __restrict__ iden = a.inv_den + (size_t)kFS_Lap * N3 * Pp + m;
  const float* __restrict__ zc = a.zc;
  const float* __restrict__ ddn_di = zc + ZC_DDN_DI * N3;
  const float* __restrict__ ddn_up = zc + ZC_DDN_UP * N3;
  const float* __restrict__ dnd_lo = zc + ZC_DND_LO * N3;
  const float* __restrict__ dnd_di = zc + ZC_DND_DI * N3;
  float* u1c = u1 + c;
  float* u2c = u2 + c;
  const int ml = lane >> 1;

  // ---- forward, pass 1: divergence, be_j, chunk map ----
  float w0 = js < N3 ? u3[js * S2] : 0.f;
  float A = 1.f, B = 0.f;
  for (int t0 = js; t0 < je; t0 += kZTL) {
    const float* r = zr_take(a, sh, R);
    float bev[kZTL] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
    for (int i = 0; i < kZTL; i++) {
      const int j = t0 + i;
      if (j >= je) break;
      const float b1 = r[(0 * kZTL + i) * 32 + (lane ^ 1)];                   // u1_{1-c}
      const float b2 = g.dim3 ? r[(1 * kZTL + i) * 32 + (lane ^ 1)] : 0.f;    // u2_{1-c}
      const float w1 = j + 1 < N3 ? r[(2 * kZTL + i) * 32 + lane] : 0.f;
      const float bi = r[kZIden + i * 16 + ml];
      float dv = 0.f;
      if (j >= 2 && j <= N3 - 3) dv = sc * (kxv * b1 + kyv * b2) + (ddn_di[j] * w0 + ddn_up[j] * w1);
      const float be = dv * bi;
      const float al = (j == 0) ? 0.f : -a_[j] * bi;
      bev[i] = be;
      A = al * A;
      B = al * B + be;
      w0 = w1;
    }
    tz_st4(tc + (uint32_t)(t0 - js), bev);
    zr_done(a, R, M, allowed, js, lane);
  }
  auto Cof = [&](int j, float bij) {   // the (0,0) mode: row 1 pinned (IMEXRK.h:68-74)
    float Cj = c_[j] * bij;
    if (m == 0 && j == 1) Cj = 0.f;
    return Cj;
  };
  float qn = zt_sweep2(sh, tc, js, je, A, B, a_, iden, Pp, w, lane, Cof);   // q at level je
  // ---- backward: q_j, u -= grad q and p += pm q; every row of u1, u2, u3, p
  // is written once, by the step of one level, so the loads of a batch may
  // all go ahead of its stores ----
  const float pm = a.pm;
  for (int b0 = ((je - js - 1) / kZI2) * kZI2; b0 >= 0; b0 -= kZI2) {
    float v[kZI2], bi[kZI2];
#pragma unroll
    for (int i = 0; i < kZI2; i++) {
      const int j = js + b0 + i;
      bi[i] = j < je ? iden[(size_t)j * Pp] : 0.f;
    }
    tz_ld16(tc + b0, v);
#pragma unroll
    for (int i0 = kZI2 - 1; i0 >= 0; i0 -= kZP2) {
      float pv[kZP2], v1[kZP2], v2[kZP2], v3[kZP2];
#pragma unroll
      for (int k = 0; k < kZP2; k++) {
        const int j = js + b0 + i0 - k, jj = j + 1;
        const bool in = j < je && act;
        pv[k] = in ? ps[j * S2] : 0.f;
        v1[k] = in ? u1c[j * S2] : 0.f;
        v2[k] = (in && g.dim3) ? u2c[j * S2] : 0.f;
        v3[k] = (in && jj >= 2 && jj <= N3 - 1) ? u3[jj * S2] : 0.f;
      }
#pragma unroll
      for (int k = 0; k < kZP2; k++) {
        const int i = i0 - k, j = js + b0 + i;
        if (j >= je) continue;
        const float qj = v[i] - Cof(j, bi[i]) * qn;
        const float qo = __shfl_xor_sync(0xffffffffu, qj, 1);
        if (act) {
          u1c[j * S2] = v1[k] - sc * kxv * qo;
          if (g.dim3) u2c[j * S2] = v2[k] - sc * kyv * qo;
          pd[j * S2] = pv[k] + pm * qj;
          const int jj = j + 1;   // u3_{j+1} -= ddz(q)_{j+1}, rows 2..N-1
          if (jj >= 2 && jj <= N3 - 1) u3[jj * S2] = v3[k] - (dnd_lo[jj] * qj + dnd_di[jj] * qn);
        }
        qn = qj;
      }
    }
  }
}

// one block per 16 modes: 8 warps, one z-chunk each, run the CN solves of
// every field, then the projection
__global__ void __launch_bounds__(kZThreads, 3)
    k_z_step_tma(StageArgs a, const __grid_constant__ CUtensorMap mS, const __grid_constant__ CUtensorMap mSn,
                 const __grid_constant__ CUtensorMap mR, const __grid_constant__ CUtensorMap mO,
                 const __grid_constant__ CUtensorMap mI) {
  extern __shared__ __align__(128) float rings[];   // [kZW][kZNS slots][kZSlotFloats]
  __shared__ ZShared sh;
  const int w = threadIdx.x >> 5, lane = threadIdx.x & 31;
  if (threadIdx.x == 0) {
    sh.bad = 0;
    for (int i = 0; i < kZW; i++)
      for (int s = 0; s < kZNS; s++) mb_init(&sh.full[i][s], 1);
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  if (w == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;" ::"r"(zs(&sh.tmem_base)),
                 "r"(2 * kZTCols));
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;");
  }
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  asm volatile("tcgen05.fence::after_thread_sync;");
  const bool dim3 = a.g.dim3 != 0;
  const ZTmaps M{&mS, &mSn, &mR, &mO, &mI};
  int js, je;
  zt_chunk(a.g.N3, w, js, je);
  ZRing R;
  R.slots = rings + (size_t)w * kZNS * kZSlotFloats;
  R.sbase = zs(R.slots);
  R.bbase = zs(&sh.full[w][0]);
  R.kslot = 0;
  R.kpar = 0;
  R.kc = 0;
  R.issued = 0;
  R.islot = 0;
  R.it = 0;
  R.isys = 0;
  R.nt = (je - js + kZTL - 1) / kZTL;
  const int nsys = dim3 ? 5 : 4;
  const int ncn = (nsys - 1) * R.nt, ntot = nsys * R.nt;
  zr_top_up(a, R, M, ncn, js, lane);
  const uint32_t tc = sh.tmem_base + ((uint32_t)(32 * (w & 3)) << 16) + (uint32_t)((w >> 2) * kZTCols);
  zt_cn<0>(a, sh, R, M, ncn, 0, tc);
  if (dim3) zt_cn<0>(a, sh, R, M, ncn, 1, tc);
  zt_cn<1>(a, sh, R, M, ncn, 2, tc);
  zt_cn<2>(a, sh, R, M, ncn, 3, tc);
  // the projection's tiles of the new velocities are read by the tensor-memory
  // accelerator (the async proxy) after this block's stores of them
  asm volatile("fence.proxy.async.global;" ::: "memory");
  __syncthreads();
  zr_top_up(a, R, M, ntot, js, lane);
  zt_proj(a, sh, R, M, ntot, tc);
  tz_wait_st();
  // every copy has landed before the block can end (each was waited for,
  // unless a wait ran out)
  if (lane == 0)
    for (int k = max(0, R.issued - kZNS); k < R.issued; k++)
      mb_wait(R.bbase + 8u * (k % kZNS), (k / kZNS) & 1, a.zerr, 3, &sh.bad, kZDrainCycles, true);
  __syncwarp();
  asm volatile("tcgen05.fence::before_thread_sync;");
  __syncthreads();
  if (w == 0) {
    asm volatile("tcgen05.fence::after_thread_sync;");
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;" ::"r"(sh.tmem_base), "r"(2 * kZTCols));
  }
}

static size_t zstep_tma_smem() { return sizeof(float) * (size_t)kZW * kZNS * kZSlotFloats; }

bool zstep_tma_supported(const Geo& g) {
  const int chunk = (g.N3 + kZW - 1) / kZW;
  return chunk <= kZTCols && g.N3 >= 2 * kZW && g.Pp % 16 == 0;
}

// the tensor maps of the z pass's inputs: 2D views [rows][columns] of float
// data, box = 32 columns (16 modes x re/im) or 16 (one pivot per mode) x kZTL rows
static int encode_map(CUtensorMap* m, const void* base, unsigned long long cols, unsigned long long rows,
                      unsigned box_cols) {
  static PFN_cuTensorMapEncodeTiled encode = nullptr;
  if (!encode) {
    cudaDriverEntryPointQueryResult q;
    void* fn = nullptr;
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &fn, cudaEnableDefault, &q) != cudaSuccess ||
        q != cudaDriverEntryPointSuccess || !fn)
      return -1;
    encode = reinterpret_cast<PFN_cuTensorMapEncodeTiled>(fn);
  }
  const cuuint64_t dims[2] = {cols, rows};
  const cuuint64_t strides[1] = {cols * sizeof(float)};
  const cuuint32_t box[2] = {box_cols, (cuuint32_t)kZTL};
  const cuuint32_t es[2] = {1, 1};
  const CUresult r = encode(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 2, const_cast<void*>(base), dims, strides, box, es,
                            CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                            CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS ? 0 : -1;
}

int zstep_tma_maps(const Geo& g, const float2* S0, const float2* S1, const float2* rnl, const float2* rold,
                   const float* inv_den, ZMaps* out) {
  static_assert(sizeof(CUtensorMap) == sizeof(ZMap), "tensor map size");
  const unsigned long long w2 = 2ull * g.Pp, r5 = (unsigned long long)g.nrun * 5 * g.N3,
                           r4 = (unsigned long long)g.nrun * 4 * g.N3;
  int e = 0;
  out->sbase[0] = S0;
  out->sbase[1] = S1;
  out->rbase[0] = rnl;
  out->rbase[1] = rold;
  out->rbase[2] = inv_den;
  e |= encode_map(reinterpret_cast<CUtensorMap*>(&out->s[0]), S0, w2, r5, 32);
  e |= encode_map(reinterpret_cast<CUtensorMap*>(&out->s[1]), S1, w2, r5, 32);
  e |= encode_map(reinterpret_cast<CUtensorMap*>(&out->rnl), rnl, w2, r4, 32);
  e |= encode_map(reinterpret_cast<CUtensorMap*>(&out->rold), rold, w2, r4, 32);
  e |= encode_map(reinterpret_cast<CUtensorMap*>(&out->iden), inv_den, (unsigned long long)g.Pp,
                  (unsigned long long)kNumFS * g.N3, 16);
  return e ? -1 : 0;
}

int launch_z_step_tma(const StageArgs& a, cudaStream_t st) {
  const Geo& g = a.g;
  const ZMaps* zm = reinterpret_cast<const ZMaps*>(a.zmaps);
  const int cs = a.S == zm->sbase[0] ? 0 : (a.S == zm->sbase[1] ? 1 : -1);
  const int cn = a.Sn == zm->sbase[0] ? 0 : (a.Sn == zm->sbase[1] ? 1 : -1);
  if (cs < 0 || cn < 0 || cs == cn) return 0;   // not the solver's two state buffers
  if (a.rnl != zm->rbase[0] || a.rold != zm->rbase[1] || a.inv_den != zm->rbase[2]) return 0;
  const CUtensorMap* mS = reinterpret_cast<const CUtensorMap*>(&zm->s[cs]);
  const CUtensorMap* mSn = reinterpret_cast<const CUtensorMap*>(&zm->s[cn]);
  const dim3 grid((g.P + 15) / 16, 1, g.nrun);
  k_z_step_tma<<<grid, kZThreads, zstep_tma_smem(), st>>>(a, *mS, *mSn, *reinterpret_cast<const CUtensorMap*>(&zm->rnl),
                                                          *reinterpret_cast<const CUtensorMap*>(&zm->rold),
                                                          *reinterpret_cast<const CUtensorMap*>(&zm->iden));
  return 1;
}

int prepare_zstep_tma_kernels() {
  return cudaFuncSetAttribute(k_z_step_tma, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)zstep_tma_smem()) ==
                 cudaSuccess
             ? 0
             : -1;
}

}  // namespace sf
