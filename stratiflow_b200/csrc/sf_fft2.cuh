// Register FFTs of two transforms at once, packed two-wide for sm_100's
// paired FP32 instructions (FADD2 / FMUL2 / FFMA2 through __fadd2_rn,
// __fmul2_rn, __ffma2_rn).
//
// A lane holds each complex point of transforms A and B as one c2x value,
// re = (re_A, re_B), im = (im_A, im_B). Every butterfly, twiddle and transpose
// then acts on both transforms with one packed instruction or one 128-bit
// shared-memory access, where the single-transform code (sf_fft.cuh) issues
// two. The split of the transform over the G lanes of a group, the twiddles,
// the padded transpose and the output order are those of reg_fft_body: on
// entry lane l holds in[l + G*e] in slot e; on exit slot h*G + k2 holds
// out[(l + h*G) + E*k2]. Unnormalised; forward e^{-2 pi i nk/N}, inverse
// e^{+2 pi i nk/N}.
#pragma once

#include "sf_fft.cuh"

namespace sf {

struct c2x {
  float2 re, im;   // (transform A, transform B)
};

__device__ __forceinline__ float2 pk2(float a) { return make_float2(a, a); }
__device__ __forceinline__ float2 padd(float2 a, float2 b) { return __fadd2_rn(a, b); }
// a - b (packed subtraction, sub.rn.f32x2)
__device__ __forceinline__ float2 psub(float2 a, float2 b) {
  unsigned long long x = *reinterpret_cast<const unsigned long long*>(&a), y = *reinterpret_cast<const unsigned long long*>(&b), d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(x), "l"(y));
  return *reinterpret_cast<float2*>(&d);
}
__device__ __forceinline__ float2 pmul(float2 a, float2 b) { return __fmul2_rn(a, b); }
__device__ __forceinline__ float2 pfma(float2 a, float2 b, float2 c) { return __ffma2_rn(a, b, c); }

__device__ __forceinline__ c2x c2add(c2x a, c2x b) { return c2x{padd(a.re, b.re), padd(a.im, b.im)}; }
__device__ __forceinline__ c2x c2sub(c2x a, c2x b) { return c2x{psub(a.re, b.re), psub(a.im, b.im)}; }

// the butterfly lo = ev + W_E^k od, hi = ev - W_E^k od (W conjugated for the
// inverse); k is a compile-time constant after unrolling, and the products
// with +-1 and +-i become sign and operand choices of the adds
template <int E, bool INV>
__device__ __forceinline__ void bfly2(c2x& lo, c2x& hi, const c2x ev, const c2x od, int k) {
  const int i = (k * (32 / E)) & 31;
  if (i == 0) {
    lo = c2add(ev, od);
    hi = c2sub(ev, od);
  } else if ((i == 8 && !INV) || (i == 24 && INV)) {   // W od = -i od = (od.im, -od.re)
    lo = c2x{padd(ev.re, od.im), psub(ev.im, od.re)};
    hi = c2x{psub(ev.re, od.im), padd(ev.im, od.re)};
  } else if ((i == 8 && INV) || (i == 24 && !INV)) {   // W od = i od = (-od.im, od.re)
    lo = c2x{psub(ev.re, od.im), padd(ev.im, od.re)};
    hi = c2x{padd(ev.re, od.im), psub(ev.im, od.re)};
  } else if (i == 16) {
    lo = c2sub(ev, od);
    hi = c2add(ev, od);
  } else {
    const float c = w32c(i), s = INV ? -w32s(i) : w32s(i);
    const c2x t{pfma(od.re, pk2(c), pmul(od.im, pk2(-s))), pfma(od.re, pk2(s), pmul(od.im, pk2(c)))};
    lo = c2add(ev, t);
    hi = c2sub(ev, t);
  }
}

// in-place DFT of E packed registers, natural order in and out (radix-2 DIT)
template <int E, bool INV>
__device__ __forceinline__ void dft2(c2x* v) {
  if constexpr (E == 2) {
    const c2x a = v[0], b = v[1];
    v[0] = c2add(a, b);
    v[1] = c2sub(a, b);
  } else {
    c2x ev[E / 2], od[E / 2];
#pragma unroll
    for (int i = 0; i < E / 2; i++) {
      ev[i] = v[2 * i];
      od[i] = v[2 * i + 1];
    }
    dft2<E / 2, INV>(ev);
    dft2<E / 2, INV>(od);
#pragma unroll
    for (int k = 0; k < E / 2; k++) bfly2<E, INV>(v[k], v[k + E / 2], ev[k], od[k], k);
  }
}

// Per-lane twiddle table of the packed transforms in shared memory, [k1][l]
// so that the lanes of a group read consecutive entries: tw4 = (wr, wr, wi,
// wi) and tw2 = (-wi, -wi), with wr + i wi = W_N^{l*k1} (forward sign).
template <int N>
__device__ __forceinline__ void fill_tw2(float4* tw4, float2* tw2, const float2* __restrict__ tw, int tid, int nthr) {
  constexpr int G = FFTShape<N>::G, E = FFTShape<N>::E;
  for (int i = tid; i < E * G; i += nthr) {
    const int k1 = i / G, l = i - k1 * G;
    const float2 w = tw[(l * k1) * (kMaxN / N)];
    tw4[i] = make_float4(w.x, w.x, w.y, w.y);
    tw2[i] = make_float2(-w.y, -w.y);
  }
}

// a * w (or a * conj(w) for the inverse), w from its table entry (wr, wr, wi,
// wi): one 128-bit shared load and five packed operations. The load and the
// arithmetic are one block of instructions, so that the compiler does not load
// a transform's twiddles ahead into registers (four per twiddle).
template <bool INV>
__device__ __forceinline__ void tw2_apply(c2x& a, const float4* t4, const float2* /*t2*/) {
  unsigned long long re = *reinterpret_cast<const unsigned long long*>(&a.re);
  unsigned long long im = *reinterpret_cast<const unsigned long long*>(&a.im);
  const unsigned s4 = (unsigned)__cvta_generic_to_shared(t4);
  if (INV)   // re' = re wr + im wi, im' = im wr - re wi
    asm volatile(
        "{\n\t.reg .b64 wr, wi, p, q;\n\t"
        "ld.shared.v2.b64 {wr, wi}, [%2];\n\t"
        "mul.rn.f32x2 p, %1, wi;\n\t"
        "mul.rn.f32x2 q, %1, wr;\n\t"
        "fma.rn.f32x2 p, %0, wr, p;\n\t"
        "mul.rn.f32x2 %1, %0, wi;\n\t"
        "sub.rn.f32x2 %1, q, %1;\n\t"
        "mov.b64 %0, p;\n\t}"
        : "+l"(re), "+l"(im)
        : "r"(s4));
  else       // re' = re wr - im wi, im' = re wi + im wr
    asm volatile(
        "{\n\t.reg .b64 wr, wi, p, q;\n\t"
        "ld.shared.v2.b64 {wr, wi}, [%2];\n\t"
        "mul.rn.f32x2 p, %1, wi;\n\t"
        "mul.rn.f32x2 q, %0, wr;\n\t"
        "sub.rn.f32x2 p, q, p;\n\t"
        "mul.rn.f32x2 q, %0, wi;\n\t"
        "fma.rn.f32x2 %1, %1, wr, q;\n\t"
        "mov.b64 %0, p;\n\t}"
        : "+l"(re), "+l"(im)
        : "r"(s4));
  a.re = *reinterpret_cast<float2*>(&re);
  a.im = *reinterpret_cast<float2*>(&im);
}

// elements (float4) of one group's transpose buffer
template <int N>
__host__ __device__ constexpr int fft2_buf_elems() {
  return FFTShape<N>::E * (FFTShape<N>::G + 1);
}

// The packed transform pair; buf is this group's fft2_buf_elems<N>() float4.
// Every lane of the warp must call it together (it syncs the warp).
template <int N, bool INV>
__device__ __forceinline__ void reg_fft2(c2x (&x)[FFTShape<N>::E], float4* buf, const float4* __restrict__ tw4,
                                         const float2* __restrict__ tw2, int l) {
  constexpr int G = FFTShape<N>::G, E = FFTShape<N>::E, H = E / G;
  dft2<E, INV>(x);
#pragma unroll
  for (int k1 = 1; k1 < E; k1++) tw2_apply<INV>(x[k1], tw4 + k1 * G + l, tw2 + k1 * G + l);
  __syncwarp();
#pragma unroll
  for (int k1 = 0; k1 < E; k1++) buf[k1 * (G + 1) + l] = make_float4(x[k1].re.x, x[k1].re.y, x[k1].im.x, x[k1].im.y);
  __syncwarp();
  c2x y[H][G];
#pragma unroll
  for (int h = 0; h < H; h++)
#pragma unroll
    for (int i = 0; i < G; i++) {
      const float4 v = buf[(l + h * G) * (G + 1) + i];
      y[h][i] = c2x{make_float2(v.x, v.y), make_float2(v.z, v.w)};
    }
  __syncwarp();
#pragma unroll
  for (int h = 0; h < H; h++) {
    dft2<G, INV>(y[h]);
#pragma unroll
    for (int k2 = 0; k2 < G; k2++) x[h * G + k2] = y[h][k2];
  }
}

// The packed transform pair of N = 256 points over a whole warp (32 lanes,
// 8 points each) in three stages: on entry lane l holds in[l + 32 e] in slot e
// (e < 8); an 8-point DFT over e and W_256^{l k1}; a transpose so that lane
// (k1 = l % 8, l0 = l / 8) holds column k1 at l0 + 4 l1 (l1 < 8); an 8-point
// DFT over l1 and W_32^{l0 m} (= W_256^{8 l0 m}, the same table); a transpose
// so that lane l holds the values l0 = 0..3 of (k1 = l % 8, m = l / 8 + 4 h),
// h = 0, 1; two 4-point DFTs over l0. On exit slot h*4 + q holds
// out[l + 32 h + 64 q], i.e. out[l + 32 j] with j = h + 2q. tw4 / tw2 are the
// table of fill_tw2_256w: [k1][l], W_256^{l k1}, k1 < 8, l < 32; tw2 its second-stage table. buf holds
// 8 x 33 float4 (padded columns: every access conflict-free).
__device__ __forceinline__ void fill_tw2_256w(float4* tw4, float2* tw2, const float2* __restrict__ tw, int tid,
                                              int nthr) {
  for (int i = tid; i < 8 * 32; i += nthr) {
    const int k1 = i / 32, l = i - k1 * 32;
    const float2 w = tw[(l * k1) * (kMaxN / 256)];
    tw4[i] = make_float4(w.x, w.x, w.y, w.y);
  }
  // the second stage's W_32^{l0 m} = W_256^{8 l0 m} as [m][l0], so that the
  // four distinct entries one warp reads lie in 64 contiguous bytes
  float4* t2 = reinterpret_cast<float4*>(tw2);
  for (int i = tid; i < 8 * 4; i += nthr) {
    const int m = i / 4, l0 = i - m * 4;
    const float2 w = tw[(8 * l0 * m) * (kMaxN / 256)];
    t2[i] = make_float4(w.x, w.x, w.y, w.y);
  }
}

__device__ __forceinline__ float4 c2x_to4(const c2x& v) { return make_float4(v.re.x, v.re.y, v.im.x, v.im.y); }
__device__ __forceinline__ c2x c2x_of4(const float4 v) { return c2x{make_float2(v.x, v.y), make_float2(v.z, v.w)}; }

// a * w (a * conj(w) for the inverse) with WR = (wr, wr), WI = (wi, wi) in registers
template <bool INV>
__device__ __forceinline__ c2x tw2_mul_reg(const c2x a, const float4 w) {
  const float2 WR = make_float2(w.x, w.y), WI = make_float2(w.z, w.w);
  if (INV) return c2x{pfma(a.re, WR, pmul(a.im, WI)), psub(pmul(a.im, WR), pmul(a.re, WI))};
  return c2x{psub(pmul(a.re, WR), pmul(a.im, WI)), pfma(a.im, WR, pmul(a.re, WI))};
}

template <bool INV>
__device__ __forceinline__ void reg_fft2_256w(c2x (&x)[8], float4* buf, const float4* __restrict__ tw4,
                                              const float2* __restrict__ tw2, int l, const float4 (&w1)[8]) {
  dft2<8, INV>(x);
#pragma unroll
  for (int k1 = 1; k1 < 8; k1++) x[k1] = tw2_mul_reg<INV>(x[k1], w1[k1]);
  __syncwarp();
#pragma unroll
  for (int k1 = 0; k1 < 8; k1++) buf[k1 * 33 + l] = c2x_to4(x[k1]);   // element (row l, column k1)
  __syncwarp();
  const int k1 = l & 7, l0 = l >> 3;
#pragma unroll
  for (int l1 = 0; l1 < 8; l1++) x[l1] = c2x_of4(buf[k1 * 33 + l0 + 4 * l1]);
  __syncwarp();
  dft2<8, INV>(x);
#pragma unroll
  for (int m = 1; m < 8; m++) tw2_apply<INV>(x[m], reinterpret_cast<const float4*>(tw2) + m * 4 + l0, tw2);
#pragma unroll
  for (int m = 0; m < 8; m++) buf[m * 33 + l] = c2x_to4(x[m]);         // element (lane l, m)
  __syncwarp();
  c2x y[2][4];
#pragma unroll
  for (int h = 0; h < 2; h++)
#pragma unroll
    for (int q = 0; q < 4; q++) y[h][q] = c2x_of4(buf[((l >> 3) + 4 * h) * 33 + (l & 7) + 8 * q]);
  __syncwarp();
#pragma unroll
  for (int h = 0; h < 2; h++) {
    dft2<4, INV>(y[h]);
#pragma unroll
    for (int q = 0; q < 4; q++) x[h * 4 + q] = y[h][q];
  }
}

}  // namespace sf
