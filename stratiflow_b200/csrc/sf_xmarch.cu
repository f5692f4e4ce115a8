// The 3D x pass of the nonlinear step as level-marching lane groups
// (BuildRHS, IMEXRK.cpp:136-193: ToNodal's x part, the nodal products, ToModal's
// x part with 1/(N1 N2) and the 2/3 truncation, then the x derivatives and the
// z stencils that follow each product).
//
// One lane group (XMT<N1>::G lanes: the whole warp at N1 = 256, else
// FFTShape<N1>::G lanes) owns one y row and walks up a range of z levels. At level t it inverse-transforms the four fields of level t
// (u1 + i u3 and b + i u2, packed as one two-transform pair, sf_fft2.cuh),
// keeps them in registers and the fields of level t-1 in its own shared
// memory, forms the eleven products of level t (with P4 of level t-1, the one
// product that needs u3 of the level above), forward-transforms them as three
// packed pairs and finishes the combinations:
//   level t-1: c1, cB, c2 get their ddz(D->N) term from Q1, QB, Q2 of level t,
//              c3 its ddz(N->D) term from P4 of level t-1; written out;
//   level t:   c1y, c2y, c3y, cBy written out; c1, cB, c2, c3 started and
//              carried in registers to the next level.
// The nodal values a lane forms after the inverse transform are those of the
// x positions it feeds into the forward transforms (x = l + G e), so the
// products need no exchange between lanes; the only shared memory traffic is
// the transforms' transposes, the level below and the staged input rows.
// No block-wide barrier after set-up: the groups of a warp share their level
// range (they own neighbouring y rows) and march in step; warps are
// independent.
#include <algorithm>
#include "sf_internal.cuh"
#include "sf_fft2.cuh"

namespace sf {

// Lane layout of the march for one grid width N1: G lanes per y row, E x
// points per lane (x = l + G e), W rows per warp, the output slots that hold
// the kept modes, and the packed transform pair.
template <int N1>
struct XMT {   // N1 = 64, 128: two-stage transforms over FFTShape<N1>::G lanes
  static constexpr int G = FFTShape<N1>::G, E = FFTShape<N1>::E, H = E / G, K1 = N1 / 3;
  static constexpr int W = 32 / G;                  // rows per warp
  static constexpr int WARPS = 6;                   // warps per block
  static constexpr int NK2 = (K1 - 1) / E + 1;
  static constexpr int NKS = H * NK2;               // output slots holding a kept mode for some lane
  static constexpr int TB = fft2_buf_elems<N1>();   // float4 per transpose buffer
  static constexpr int TWE = E * G;                 // twiddle table entries
  // output slot of the i-th kept candidate; slot h*G + k2 holds mode l + h*G + E*k2
  __host__ __device__ static constexpr int kslot(int i) { return (i / NK2) * G + i % NK2; }
  __device__ static int kmode(int l, int i) { return l + (kslot(i) / G) * G + E * (kslot(i) % G); }
  // x position index e (x = l + G e) of inverse output slot s
  __host__ __device__ static constexpr int pos(int s) { return s / G + H * (s % G); }
  // slot holding mode N1 - k at lane G - l (l >= 1) or at lane 0 (l = 0)
  __host__ __device__ static constexpr int partner(int i, bool lane0) {
    const int s = kslot(i), h = s / G, k2 = s % G;
    const int q = lane0 ? (E - h - H * k2) % E : E - 1 - h - H * k2;
    return (q % H) * G + q / H;
  }
  __device__ static void fill(float4* tw4, float2* tw2, const float2* tw, int tid, int nthr) {
    fill_tw2<N1>(tw4, tw2, tw, tid, nthr);
  }
  template <bool INV>
  __device__ static void fft(c2x (&x)[E], float4* buf, const float4* tw4, const float2* tw2, int l,
                             const float4 (&)[8]) {
    reg_fft2<N1, INV>(x, buf, tw4, tw2, l);
  }
};
template <>
struct XMT<256> {   // a whole warp per row: three stages, 8 x 8 x 4 (reg_fft2_256w)
  static constexpr int G = 32, E = 8, K1 = 85, W = 1, WARPS = 12;
  static constexpr int NKS = 3;                     // modes l, l + 32, l + 64
  static constexpr int TB = 8 * 33, TWE = 8 * 32;
  // slot of out[l + 32 j]: j = h + 2 q in slot h*4 + q
  __host__ __device__ static constexpr int jslot(int j) { return (j % 2) * 4 + j / 2; }
  __host__ __device__ static constexpr int kslot(int i) { return jslot(i); }
  __device__ static int kmode(int l, int i) { return l + 32 * i; }
  __host__ __device__ static constexpr int pos(int s) { return s / 4 + 2 * (s % 4); }
  __host__ __device__ static constexpr int partner(int i, bool lane0) { return jslot(lane0 ? (8 - i) % 8 : 7 - i); }
  __device__ static void fill(float4* tw4, float2* tw2, const float2* tw, int tid, int nthr) {
    fill_tw2_256w(tw4, tw2, tw, tid, nthr);
  }
  template <bool INV>
  __device__ static void fft(c2x (&x)[E], float4* buf, const float4* tw4, const float2* tw2, int l,
                             const float4 (&w1)[8]) {
    reg_fft2_256w<INV>(x, buf, tw4, tw2, l, w1);
  }
};

template <int N1>
struct XMShape : XMT<N1> {
  using T = XMT<N1>;
  // shared memory of one row: two levels of nodal values (float4 per x
  // point, a ring: this level and the one below), the transpose buffer, the
  // carried combinations ((c1, cB), (c2, c3) per kept slot and lane) and the
  // staged input rows of the next level (4 x K1)
  static constexpr size_t group_bytes =
      sizeof(float4) * (size_t)(2 * N1 + T::TB + 2 * T::NKS * T::G) + sizeof(float2) * 4 * T::K1;
  static constexpr size_t table_bytes = (sizeof(float4) + sizeof(float2)) * (size_t)T::TWE;
  static constexpr size_t smem_bytes = table_bytes + (size_t)T::WARPS * T::W * group_bytes;
  static_assert(group_bytes % 16 == 0 && table_bytes % 16 == 0, "16-byte aligned regions");
  static_assert(smem_bytes <= 227 * 1024, "one block fits an SM");
};

__device__ __forceinline__ void xm_cp8(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;\n" ::"r"(s), "l"(gmem));
}
__device__ __forceinline__ void xm_cp_wait() { asm volatile("cp.async.wait_all;\n" ::); }

__device__ __forceinline__ float4 c2x_f4(const c2x& v) { return make_float4(v.re.x, v.re.y, v.im.x, v.im.y); }

// levels t_lo .. t_hi - 1 of every (run, y row) of the launch; the units
// (run, block of W rows, level) are split evenly over the launch's warps
template <int N1>
__global__ void __launch_bounds__(XMT<N1>::WARPS * 32, 1) k_xmarch(StageArgs a, int t_lo, int t_hi) {
  using X = XMShape<N1>;
  using T = XMT<N1>;
  constexpr int G = T::G, E = T::E, K1 = T::K1, W = T::W, NKS = T::NKS, kXMWarps = T::WARPS;
  const Geo g = a.g;
  const int N3 = g.N3, N2 = g.N2;
  extern __shared__ __align__(16) unsigned char xsm[];
  float4* tw4 = reinterpret_cast<float4*>(xsm);
  float2* tw2 = reinterpret_cast<float2*>(xsm + sizeof(float4) * T::TWE);
  T::fill(tw4, tw2, a.tw, threadIdx.x, blockDim.x);
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int gw = lane / G, l = lane - gw * G;
  __builtin_assume(l >= 0 && l < G);
  unsigned char* gb = xsm + X::table_bytes + (size_t)(warp * W + gw) * X::group_bytes;
  float4* ring = reinterpret_cast<float4*>(gb);     // [2 levels][E slots][G lanes]: u1, b, u3, u2
  float4* tbuf = ring + 2 * N1;                     // transpose buffer
  float4* cbuf = tbuf + T::TB;                      // [2][NKS][G]: (c1, cB), (c2, c3) awaiting their z terms
  float2* stg = reinterpret_cast<float2*>(cbuf + 2 * NKS * G);   // [4][K1]: u1, u2, u3, b of the next level
  __syncthreads();

  const int partner_lane = (lane & ~(G - 1)) | ((G - l) & (G - 1));
  // the first-stage twiddles of the whole-warp transform, held in registers
  float4 w1[8];
#pragma unroll
  for (int k = 0; k < 8; k++) w1[k] = (N1 == 256) ? tw4[(k * 32 + l) % T::TWE] : make_float4(0.f, 0.f, 0.f, 0.f);
  // zero, but not known to the compiler: a batch's shared-memory reads take
  // (bits of the last batch's result) & rz as an offset, a true dependency
  // that keeps the compiler from starting one batch's products and
  // transform under the last one's, which would need both register sets
  const int rz = (int)(gridDim.x >> 30);
  int tok = 0;
  const float* __restrict__ zc = a.zc;
  const float sc = 0.5f * g.inv_n12;
  const float2 SC = make_float2(sc, sc);

  const int L = t_hi - t_lo;
  const long long NYB = N2 / W;
  const long long U = (long long)g.nrun * NYB * L;
  const long long NW = (long long)gridDim.x * kXMWarps;
  const long long wid = (long long)blockIdx.x * kXMWarps + warp;
  long long u = U * wid / NW;
  const long long uend = U * (wid + 1) / NW;

  while (u < uend) {
    const long long rb = u / L;
    const int ta = t_lo + (int)(u - rb * L);
    const int tb = (int)std::min<long long>((long long)t_hi, (long long)ta + (uend - u));
    u += tb - ta;
    const int run = (int)(rb / NYB), y = (int)(rb % NYB) * W + gw;
    const float* __restrict__ Ub = a.Ubar + (size_t)run * N3;
    const float2* __restrict__ src = a.mixin + ((size_t)run * 4 * N3 * N2 + y) * K1;   // + (f*N3 + t)*N2*K1
    const size_t fstride = (size_t)N3 * N2 * K1, tstride = (size_t)N2 * K1;
    float2* __restrict__ dst = a.mixout + ((size_t)run * 8 * N3 * N2 + y) * K1;        // + (c*N3 + t)*N2*K1

    // the four input rows of level t into the stage, 8-byte asynchronous
    // copies (a row of K1 complex values is not 16-byte aligned in general)
    auto prefetch = [&](int t) {
      if (t < 0 || t >= N3) return;
      const float2* s0 = src + (size_t)t * tstride + l;
#pragma unroll
      for (int f = 0; f < 4; f++) {
        const float2* sf = s0 + f * fstride;
#pragma unroll
        for (int j = 0; j < (K1 + G - 1) / G; j++)
          if (l + G * j < K1) xm_cp8(stg + f * K1 + l + G * j, sf + G * j);
      }
    };
    // this lane's kept mode in kept slot i
    auto kk = [&](int i) { return T::kmode(l, i); };
    // c1, cB and c2, c3 of the last level, awaiting their z terms, per kept slot
    auto Ca = [&](int i) -> float4& { return cbuf[i * G + l]; };
    auto Cb = [&](int i) -> float4& { return cbuf[(NKS + i) * G + l]; };
    auto store = [&](int c, int lvl, int i, float2 v) { dst[((size_t)c * N3 + lvl) * tstride + kk(i)] = v; };
    auto mikx = [&](float k, float2 v) { return make_float2(k * v.y, -k * v.x); };   // -(i k) v

    prefetch(ta - 1);
    // step t: the inverse transform of level t, then (ta <= t < tb) every
    // product of level t and P4 of level t-1, or (t = tb) only Q1, QB, Q2 of
    // level t and P4 of level t-1 (t = ta - 1 only transforms)
#pragma unroll 1
    for (int t = ta - 1; t <= tb; t++) {
      const bool lv = t >= 0 && t < N3;
      c2x x[E];
      if (lv) {
        xm_cp_wait();
        __syncwarp();
        const float2 *su1 = stg, *su2 = stg + K1, *su3 = stg + 2 * K1, *sb = stg + 3 * K1;
        // c2r input of the pair (u1 + i u3, b + i u2) at n = l + G e: A + iB
        // at n < K1 (real parts only at n = 0), conj(A) + i conj(B) of mode
        // N1 - n at n > N1 - K1, zero between; one load per field from the
        // mode index and a sign, so no position loads two rows
#pragma unroll
        for (int e = 0; e < E; e++) {
          if (G * e >= K1 && G * e + G - 1 <= N1 - K1) {   // zero at every lane
            x[e] = c2x{make_float2(0.f, 0.f), make_float2(0.f, 0.f)};
            continue;
          }
          const int n = l + G * e;
          const bool dir = n < K1, cnj = n > N1 - K1;
          const int m = (dir ? n : (cnj ? N1 - n : 0)) + tok;
          const float on = (dir || cnj) ? 1.f : 0.f;
          const float sg = dir ? -1.f : 1.f;                 // A.x + sg B.y, B.x - sg A.y
          const float im0 = (n == 0) ? 0.f : on;             // k = 0: real parts only
          const float2 A = su1[m], B = su3[m], C_ = sb[m], D = su2[m];
          const float2 re = make_float2(on * A.x + (sg * im0) * B.y, on * C_.x + (sg * im0) * D.y);
          const float2 im = make_float2(on * B.x - (sg * im0) * A.y, on * D.x - (sg * im0) * C_.y);
          x[e] = c2x{re, im};
        }
      }
      __syncwarp();   // the staged rows are read: the next level's copies may start
      if (t < tb) prefetch(t + 1);
      // level t into its ring slot (u1, b, u3, u2 per x point; zero outside 0..N3-1)
      float4* curl = ring + (size_t)(t & 1) * N1;
      const float4* prev = ring + (size_t)((t - 1) & 1) * N1;
      if (lv) {
        T::template fft<true>(x, tbuf, tw4, tw2, l, w1);
#pragma unroll
        for (int s = 0; s < E; s++) curl[s * G + l] = c2x_f4(x[s]);
        tok = __float_as_int(x[0].re.x) & rz;
      } else {
#pragma unroll
        for (int s = 0; s < E; s++) curl[s * G + l] = make_float4(0.f, 0.f, 0.f, 0.f);
      }
      if (t < ta) continue;

      // ---- coefficients of level t (products) and of the combinations ----
      const bool lo = lv && t >= 1, lvm = t >= 1 && t - 1 < N3;
      const float lof = lo ? 1.f : 0.f, hb = 0.5f * lof, lm = lvm ? 1.f : 0.f;
      const float ub = lv ? Ub[t] : 0.f, ubm = lo ? Ub[t - 1] : 0.f;
      const float tlo = lo ? zc[ZC_TILDE_LO * N3 + t] : 0.f, tdi = lo ? zc[ZC_TILDE_DI * N3 + t] : 0.f;
      const float topm = (t - 1 <= N3 - 2) ? 1.f : 0.f;   // Dir(u3) of level t-1 reaches level t
      const int tm = t - 1;
      const bool fin = tm >= ta;   // level t-1 belongs to this segment: finish it
      const float fu = (fin && tm >= 1 && tm < N3 - 1) ? zc[ZC_DDN_UP * N3 + tm] : 0.f;
      const float fd = (fin && tm >= 2) ? zc[ZC_DND_DI * N3 + tm] : 0.f;
      const float sd = (lv && t >= 1) ? zc[ZC_DDN_DI * N3 + t] : 0.f;
      const float sl = (lv && t >= 2) ? zc[ZC_DND_LO * N3 + t] : 0.f;

      // the forward transform pairs of the step, one batch at a time:
      //   b = 0: Q1 + i QB, Q2 + i P4 (level t-1)   [ta <= t <= tb]
      //   b = 1: S1 + i SB1, S12 + i S22            [t < tb]
      //   b = 2: P3 + i P3Y, SB2                    [t < tb]
      const int nb = t < tb ? 3 : 1;
#pragma unroll 1
      for (int b = 0; b < nb; b++) {
        c2x z[E];
        if (b == 0) {
#pragma unroll
          for (int s = 0; s < E; s++) {
            const float4 pv = prev[s * G + l + tok], cv = curl[s * G + l + tok];   // u1, b, u3, u2 of t-1, t
            const float U1 = cv.x, Bv = cv.y, U3 = cv.z, U2 = cv.w;
            const float w3 = lof * U3;
            const float q1 = (hb * U1 + hb * pv.x + (hb * ubm + hb * ub)) * w3;
            const float qb = (hb * Bv + hb * pv.y) * w3;
            const float q2 = (hb * U2 + hb * pv.w) * w3;
            const float d = 0.5f * pv.z + 0.5f * topm * U3;
            z[T::pos(s)] = c2x{make_float2(q1, q2), make_float2(qb, lm * (d * d))};
          }
        } else if (b == 1) {
#pragma unroll
          for (int s = 0; s < E; s++) {
            const float4 cv = curl[s * G + l + tok];
            const float U1 = cv.x, Bv = cv.y, U2 = cv.w;
            const float u1t = U1 + ub;
            z[T::pos(s)] = c2x{make_float2(U1 * (U1 + 2.f * ub), u1t * U2), make_float2(u1t * Bv, U2 * U2)};
          }
        } else {
#pragma unroll
          for (int s = 0; s < E; s++) {
            const float4 pv = prev[s * G + l + tok], cv = curl[s * G + l + tok];
            const float U1 = cv.x, Bv = cv.y, U3 = cv.z, U2 = cv.w;
            const float w3 = lof * U3;
            const float p3 = (tdi * U1 + tlo * pv.x + (tlo * ubm + tdi * ub)) * w3;
            const float p3y = (tdi * U2 + tlo * pv.w) * w3;
            z[T::pos(s)] = c2x{make_float2(p3, U2 * Bv), make_float2(p3y, 0.f)};
          }
        }
        T::template fft<false>(z, tbuf, tw4, tw2, l, w1);
        // split each transform of the pair into its two real products at
        // the kept modes: (Z_k + conj Z_{N-k}) / 2 and (Z_k - conj Z_{N-k}) / (2i),
        // times 1/(N1 N2)
#pragma unroll
        for (int i = 0; i < NKS; i++) {
          const int s = T::kslot(i);
          const c2x zs = z[s];
          const c2x po = z[T::partner(i, false)];
          c2x p;
          p.re.x = __shfl_sync(0xffffffffu, po.re.x, partner_lane);
          p.re.y = __shfl_sync(0xffffffffu, po.re.y, partner_lane);
          p.im.x = __shfl_sync(0xffffffffu, po.im.x, partner_lane);
          p.im.y = __shfl_sync(0xffffffffu, po.im.y, partner_lane);
          if (l == 0) p = z[T::partner(i, true)];
          if (kk(i) >= K1) continue;
          const float2 SR = pmul(padd(zs.re, p.re), SC), DI = pmul(psub(zs.im, p.im), SC);
          const float2 SI = pmul(padd(zs.im, p.im), SC), DR = pmul(psub(p.re, zs.re), SC);
          const float2 A1 = make_float2(SR.x, DI.x), A2 = make_float2(SI.x, DR.x);   // transform A's products
          const float2 B1 = make_float2(SR.y, DI.y), B2 = make_float2(SI.y, DR.y);   // transform B's
          if (b == 0) {   // A1 = Q1, A2 = QB, B1 = Q2, B2 = P4 of level t-1
            if (fin) {
              const float4 ca = Ca(i), cb = Cb(i);
              store(0, tm, i, make_float2(ca.x - fu * A1.x, ca.y - fu * A1.y));
              store(6, tm, i, make_float2(ca.z - fu * A2.x, ca.w - fu * A2.y));
              store(2, tm, i, make_float2(cb.x - fu * B1.x, cb.y - fu * B1.y));
              store(4, tm, i, make_float2(cb.z - fd * B2.x, cb.w - fd * B2.y));
            }
            Ca(i) = make_float4(-sd * A1.x, -sd * A1.y, -sd * A2.x, -sd * A2.y);
            Cb(i) = make_float4(-sd * B1.x, -sd * B1.y, -sl * B2.x, -sl * B2.y);
          } else if (b == 1) {   // S1, SB1, S12, S22
            const float k = __ldg(a.kx + kk(i));
            const float2 a1 = mikx(k, A1), aB = mikx(k, A2), a2 = mikx(k, B1);
            const float4 ca = Ca(i), cb = Cb(i);
            Ca(i) = make_float4(a1.x + ca.x, a1.y + ca.y, aB.x + ca.z, aB.y + ca.w);
            Cb(i) = make_float4(a2.x + cb.x, a2.y + cb.y, cb.z, cb.w);
            store(1, t, i, make_float2(-B1.x, -B1.y));
            store(3, t, i, make_float2(-B2.x, -B2.y));
          } else {   // P3, P3Y, SB2
            const float2 a3 = mikx(__ldg(a.kx + kk(i)), A1);
            const float4 cb = Cb(i);
            Cb(i) = make_float4(cb.x, cb.y, cb.z + a3.x, cb.w + a3.y);
            store(5, t, i, make_float2(-A2.x, -A2.y));
            store(7, t, i, make_float2(-B1.x, -B1.y));
          }
        }
        tok = __float_as_int(z[0].re.x) & rz;
      }
    }
  }
}

template <int N1>
static int xmarch_launch(const StageArgs& a, int t_lo, int t_hi, cudaStream_t st) {
  using X = XMShape<N1>;
  static int blocks = 0;   // resident blocks of the device this process runs on
  if (blocks == 0) {
    int dev = 0, nsm = 0, bps = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&bps, k_xmarch<N1>, X::WARPS * 32, X::smem_bytes);
    blocks = std::max(1, bps) * std::max(1, nsm);
  }
  k_xmarch<N1><<<blocks, X::WARPS * 32, X::smem_bytes, st>>>(a, t_lo, t_hi);
  return 1;
}

bool xmarch_supported(const StageArgs& a) {
  const Geo& g = a.g;
  if (!g.dim3 || a.linear || a.tlm || a.adjoint) return false;
  const int N1 = g.N1;
  if (N1 != 64 && N1 != 128 && N1 != 256) return false;
  const int W = N1 == 256 ? XMT<256>::W : 4;
  return g.N2 % W == 0;
}

int launch_xmarch(const StageArgs& a, int t_lo, int t_hi, cudaStream_t st) {
  switch (a.g.N1) {
    case 64: return xmarch_launch<64>(a, t_lo, t_hi, st);
    case 128: return xmarch_launch<128>(a, t_lo, t_hi, st);
    case 256: return xmarch_launch<256>(a, t_lo, t_hi, st);
  }
  return 0;
}

int prepare_xmarch_kernels() {
  cudaError_t e = cudaFuncSetAttribute(k_xmarch<64>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                       (int)XMShape<64>::smem_bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_xmarch<128>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)XMShape<128>::smem_bytes);
  if (e == cudaSuccess)
    e = cudaFuncSetAttribute(k_xmarch<256>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)XMShape<256>::smem_bytes);
  return e == cudaSuccess ? 0 : -1;
}

}  // namespace sf
