// Register-resident FFTs for one group of G lanes of a warp.
//
// An N-point transform, N = G * E, is split as: lane l of the group holds the
// E points in[l + G*e]; an E-point DFT in registers; twiddles W_N^{l*k1}; one
// transpose through a padded shared buffer; a G-point DFT in registers over
// the G lanes' values of column k1, owned by lane k1 mod G. On exit register
// slot h*G + k2 of lane l holds out[(l + h*G) + E*k2] (h < E/G).
// Unnormalised; forward uses e^{-2 pi i nk/N}, inverse e^{+2 pi i nk/N} (the
// FFTW conventions the reference relies on).
#pragma once

#include "sf_internal.cuh"

namespace sf {

#include "sf_tw32.inc"

template <int N> struct FFTShape;
template <> struct FFTShape<16> { static constexpr int G = 4, E = 4; };
template <> struct FFTShape<32> { static constexpr int G = 4, E = 8; };
template <> struct FFTShape<64> { static constexpr int G = 8, E = 8; };
template <> struct FFTShape<128> { static constexpr int G = 8, E = 16; };
template <> struct FFTShape<256> { static constexpr int G = 16, E = 16; };
template <> struct FFTShape<512> { static constexpr int G = 16, E = 32; };

// float2 elements of one group's buffer: the E x (G+1) padded transpose, at
// least N (it also holds a whole output row), rounded so that the groups of
// one half-warp start on different banks
template <int N>
__host__ __device__ constexpr int fft_buf_stride() {
  constexpr int G = FFTShape<N>::G, E = FFTShape<N>::E;
  constexpr int s = (E * (G + 1) > N) ? E * (G + 1) : N;
  return s + (((G - s) % 16) + 16) % 16;
}

// a * W_E^k (forward) or a * conj(W_E^k) (inverse); k is a compile-time
// constant after unrolling, so the branches and constants fold
template <int E, bool INV>
__device__ __forceinline__ float2 twmul(float2 a, int k) {
  const int i = (k * (32 / E)) & 31;
  if (i == 0) return a;
  if (i == 8) return INV ? make_float2(-a.y, a.x) : make_float2(a.y, -a.x);
  if (i == 16) return make_float2(-a.x, -a.y);
  if (i == 24) return INV ? make_float2(a.y, -a.x) : make_float2(-a.y, a.x);
  const float c = w32c(i), s = INV ? -w32s(i) : w32s(i);
  return make_float2(a.x * c - a.y * s, a.x * s + a.y * c);
}

// in-place DFT of E registers, natural order in and out (radix-2 DIT)
template <int E, bool INV>
__device__ __forceinline__ void dft(float2* v) {
  if constexpr (E == 2) {
    const float2 a = v[0], b = v[1];
    v[0] = make_float2(a.x + b.x, a.y + b.y);
    v[1] = make_float2(a.x - b.x, a.y - b.y);
  } else {
    float2 ev[E / 2], od[E / 2];
#pragma unroll
    for (int i = 0; i < E / 2; i++) {
      ev[i] = v[2 * i];
      od[i] = v[2 * i + 1];
    }
    dft<E / 2, INV>(ev);
    dft<E / 2, INV>(od);
#pragma unroll
    for (int k = 0; k < E / 2; k++) {
      const float2 t = twmul<E, INV>(od[k], k);
      v[k] = make_float2(ev[k].x + t.x, ev[k].y + t.y);
      v[k + E / 2] = make_float2(ev[k].x - t.x, ev[k].y - t.y);
    }
  }
}

// x: in[l + G*e] on entry, out[(l + h*G) + E*k2] in slot h*G + k2 on exit.
// buf: this group's fft_buf_stride<N>() elements. twid(k1) gives W_N^{l*k1}
// (forward sign). Every lane of the warp must call it together (it syncs the
// warp).
template <int N, bool INV, class TW>
__device__ __forceinline__ void reg_fft_body(float2 (&x)[FFTShape<N>::E], float2* buf, const TW& twid, int l) {
  constexpr int G = FFTShape<N>::G, E = FFTShape<N>::E, H = E / G;
  dft<E, INV>(x);
#pragma unroll
  for (int k1 = 1; k1 < E; k1++) {
    float2 w = twid(k1);
    if (INV) w.y = -w.y;
    x[k1] = cmul(x[k1], w);
  }
  __syncwarp();
#pragma unroll
  for (int k1 = 0; k1 < E; k1++) buf[k1 * (G + 1) + l] = x[k1];
  __syncwarp();
  float2 y[H][G];
#pragma unroll
  for (int h = 0; h < H; h++)
#pragma unroll
    for (int i = 0; i < G; i++) y[h][i] = buf[(l + h * G) * (G + 1) + i];
  __syncwarp();
#pragma unroll
  for (int h = 0; h < H; h++) {
    dft<G, INV>(y[h]);
#pragma unroll
    for (int k2 = 0; k2 < G; k2++) x[h * G + k2] = y[h][k2];
  }
}

// the transform with the twiddles read from tw: e^{-2 pi i k/kMaxN}, k < kMaxN
template <int N, bool INV>
__device__ __forceinline__ void reg_fft(float2 (&x)[FFTShape<N>::E], float2* buf, const float2* __restrict__ tw,
                                        int l) {
  reg_fft_body<N, INV>(x, buf, [&](int k1) { return tw[(l * k1) * (kMaxN / N)]; }, l);
}

// lane l's twiddles W_N^{l*k1}, k1 < E, for a kernel that runs many
// transforms and keeps them in registers
template <int N>
__device__ __forceinline__ void lane_twiddles(float2 (&w)[FFTShape<N>::E], const float2* __restrict__ tw, int l) {
#pragma unroll
  for (int k1 = 0; k1 < FFTShape<N>::E; k1++) w[k1] = tw[(l * k1) * (kMaxN / N)];
}

// the transform with lane_twiddles' registers
template <int N, bool INV>
__device__ __forceinline__ void reg_fft_w(float2 (&x)[FFTShape<N>::E], float2* buf, const float2 (&w)[FFTShape<N>::E],
                                          int l) {
  reg_fft_body<N, INV>(x, buf, [&](int k1) { return w[k1]; }, l);
}

// output index of register slot `slot` of lane l
template <int N>
__device__ __forceinline__ int reg_fft_out_index(int l, int slot) {
  constexpr int G = FFTShape<N>::G, E = FFTShape<N>::E;
  return (l + (slot / G) * G) + E * (slot % G);
}

}  // namespace sf
