// CPU oracle for the Stratiflow IMEX-RK time step.
//
// TEST INFRASTRUCTURE ONLY. This file is the parity checker for the CUDA
// path and the timed CPU baseline of the benchmark. Nothing in the product
// library links, loads or calls it.
//
// It restates, in plain C++ templated on the precision (float = the
// reference's default build, double = its -DDOUBLE build), the algorithm of
// jeremypparker/Stratiflow's IMEXRK::TimeStep and TimeStepLinear:
//   grid            Field.cpp:3-83
//   operators       Differentiation.cpp:6-160, Differentiation.h:17-59
//   Thomas solver   Tridiagonal.h:14-53
//   FFT + filter    Field.h:734-769, 965-1021, 1129-1166
//   products        Stratiflow.h:51-164
//   scheme          IMEXRK.h:37-81, 128-162, 321-352, 395-411, 502-545,
//                   629-632; IMEXRK.cpp:8-258
//   norms           Integration.h:5-46, 118-146, 282-311
// Storage follows the reference exactly: a field is z-fastest with index
// (Nx*n2 + n1)*N3 + n3 (Field.h:399,410), Nx = N1 for nodal fields and
// N1/2+1 for modal fields. The dense N3xN3 vertical matrices of the
// reference are applied here as the 2- and 3-point bands they contain.
// FFTW is replaced by an own radix-2 FFT with FFTW's sign and scaling
// conventions (unnormalised forward e^{-i}, unnormalised inverse e^{+i}).
//
// Parity status: the reference ships no tests, golden vectors or fixtures,
// and it cannot be compiled in this environment (Eigen3 and FFTW are absent),
// so this restatement is pinned by (a) a literal dense-matrix transcription
// of the reference's operator construction in numpy, (b) numpy's FFT, and
// (c) known-answer tests; it is not pinned against outputs of the reference
// itself ("parity unpinned" by the reference).
//
// One generalisation, carried identically by the CUDA path: the reference
// hard-wires the background stratification dB/dz = 1 in BuildRHS
// (IMEXRK.cpp:145-147). Here it is a per-level array dBdz[N3] multiplying
// ReinterpolateDirichlet(u3); dBdz = 1 reproduces the reference exactly.

#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdint>
#include <cstring>
#include <vector>
#ifdef _OPENMP
#include <omp.h>
#endif

namespace sfo {

enum BC { Neumann = 0, Dirichlet = 1 };

// ---------------------------------------------------------------- FFT ----
template <class T>
struct FFT1 {
  using C = std::complex<T>;
  int n = 1;
  std::vector<C> tw;   // e^{-2 pi i k/n}, k < n/2
  std::vector<int> rev;
  void init(int n_) {
    n = n_;
    tw.resize(std::max(1, n / 2));
    for (int k = 0; k < n / 2; k++) {
      double a = -2.0 * M_PI * double(k) / double(n);
      tw[k] = C(T(std::cos(a)), T(std::sin(a)));
    }
    rev.assign(n, 0);
    int lg = 0;
    while ((1 << lg) < n) lg++;
    for (int i = 0; i < n; i++) {
      int r = 0;
      for (int b = 0; b < lg; b++)
        if (i & (1 << b)) r |= 1 << (lg - 1 - b);
      rev[i] = r;
    }
  }
  // in place, unnormalised; sign -1 forward, +1 inverse
  void run(C* a, bool inverse) const {
    if (n == 1) return;
    for (int i = 0; i < n; i++)
      if (i < rev[i]) std::swap(a[i], a[rev[i]]);
    for (int len = 2; len <= n; len <<= 1) {
      int half = len >> 1, step = n / len;
      for (int i = 0; i < n; i += len)
        for (int j = 0; j < half; j++) {
          C w = tw[j * step];
          if (inverse) w = std::conj(w);
          C u = a[i + j], v = a[i + j + half] * w;
          a[i + j] = u + v;
          a[i + j + half] = u - v;
        }
    }
  }
};

// ------------------------------------------------------------- solver ----
template <class T>
struct Solver {
  using C = std::complex<T>;
  // grid (Parameters.h:6-43 as runtime values)
  int N1, N2, N3, M1, K1;
  bool dim3;
  T L1, L2, L3, Re, Ri, Pr;
  T deltaT = T(0.01);
  T h[3];
  static constexpr double beta[3] = {1.0, 25.0 / 8.0, 9.0 / 4.0};   // IMEXRK.h:631
  static constexpr double zeta[3] = {0.0, -17.0 / 8.0, -5.0 / 4.0}; // IMEXRK.h:632

  // vertical grid (Field.cpp:3-83); index 0 of z and DY is unused there
  std::vector<T> z, zf, DY, DYF;
  // band coefficients (Differentiation.cpp:6-110)
  std::vector<T> d2n_lo, d2n_di, d2n_up, d2d_lo, d2d_di, d2d_up;
  std::vector<T> dnd_lo, dnd_di;  // ddz Neumann -> Dirichlet, rows 1..N-1
  std::vector<T> ddn_di, ddn_up;  // ddz Dirichlet -> Neumann, rows 1..N-1
  std::vector<T> full_lo, full_di, tilde_lo, tilde_di;
  // Fourier (Differentiation.cpp:113-160)
  std::vector<T> kx, ky, kx2, ky2;   // kx,ky: real part of i*k, i.e. 2 pi k/L
  std::vector<int> keptY;            // kept n2 indices (Field.h:1129-1166)

  // modal fields, (M1*n2+n1)*N3+n3
  std::vector<C> u1, u2, u3, b, p, R1, R2, R3, RB, r1, r2, r3, rB, ntmp, dtmp, div, q;
  // nodal fields, (N1*n2+n1)*N3+n3
  std::vector<T> U1, U2, U3, B, U1t, prod, prod2, Ubar, dBdz;
  // frozen base state of the linearisation (IMEXRK.h:334-352)
  std::vector<T> U1b, U2b, U3b, Bb;

  // Thomas factors: a and c are per row only, b and C per kept stack
  struct Fam {
    std::vector<T> a, c;          // N3
    std::vector<T> bb, CC;        // nkept * N3
  };
  Fam velN[3], velD[3], buoN[3], lap;

  FFT1<T> fx, fy;

  int nkept() const { return K1 * int(keptY.size()); }
  size_t midx(int n1, int n2) const { return (size_t(M1) * n2 + n1) * N3; }
  size_t nidx(int n1, int n2) const { return (size_t(N1) * n2 + n1) * N3; }

  void init(int n1, int n2, int n3, double l1, double l2, double l3, double re, double ri, double pr) {
    N1 = n1; N2 = n2; N3 = n3; M1 = N1 / 2 + 1; K1 = N1 / 3;
    dim3 = N2 > 1;
    L1 = T(l1); L2 = T(l2); L3 = T(l3); Re = T(re); Ri = T(ri); Pr = T(pr);
    build_grid();
    build_fourier();
    size_t ms = size_t(M1) * N2 * N3, ns = size_t(N1) * N2 * N3;
    for (auto* f : {&u1, &u2, &u3, &b, &p, &R1, &R2, &R3, &RB, &r1, &r2, &r3, &rB, &ntmp, &dtmp, &div, &q})
      f->assign(ms, C(0));
    for (auto* f : {&U1, &U2, &U3, &B, &U1t, &prod, &prod2, &U1b, &U2b, &U3b, &Bb}) f->assign(ns, T(0));
    Ubar.assign(N3, T(0));
    dBdz.assign(N3, T(1));
    fx.init(N1);
    fy.init(N2);
    build_laplacian();
    update_for_timestep();
  }

  // Field.cpp:3-19, 21-31, 62-83
  void build_grid() {
    int N = N3;
    z.assign(N, T(0)); zf.assign(N, T(0)); DY.assign(N, T(0)); DYF.assign(N, T(0));
    T cs = 2;
    // Eigen's LinSpaced(N-1, -1, 1): low + i*step, the last point exactly high
    T step = (T(1) - T(-1)) / T(N - 2);
    for (int i = 0; i < N - 1; i++) {
      T x = (i == N - 2) ? T(1) : T(-1) + T(i) * step;
      z[i + 1] = L3 * (cs * std::pow(x, T(7)) + x) / (cs + 1);
    }
    T offsetPoint = (z[1] + z[2]) / 2;
    for (int i = 1; i < N; i++) z[i] *= -L3 / offsetPoint;
    for (int i = 1; i <= N - 2; i++) zf[i] = T(0.5) * (z[i] + z[i + 1]);
    zf[0] = 2 * zf[1] - zf[2];
    zf[N - 1] = 2 * zf[N - 2] - zf[N - 3];
    for (int i = 1; i < N; i++) DY[i] = zf[i] - zf[i - 1];
    for (int i = 1; i <= N - 2; i++) DYF[i] = z[i + 1] - z[i];
    DYF[N - 1] = DYF[N - 2];
    DYF[0] = DYF[1];

    d2n_lo.assign(N, 0); d2n_di.assign(N, 0); d2n_up.assign(N, 0);
    d2d_lo.assign(N, 0); d2d_di.assign(N, 0); d2d_up.assign(N, 0);
    // Differentiation.cpp:6-33
    for (int j = 1; j < N - 1; j++) {
      d2n_lo[j] = 1 / DY[j] / DYF[j];
      d2n_di[j] = -1 / DY[j] / DYF[j] - 1 / DY[j + 1] / DYF[j];
      d2n_up[j] = 1 / DY[j + 1] / DYF[j];
    }
    for (int j = 2; j < N - 1; j++) {
      d2d_lo[j] = 1 / DYF[j - 1] / DY[j];
      d2d_di[j] = -1 / DYF[j - 1] / DY[j] - 1 / DYF[j] / DY[j];
      d2d_up[j] = 1 / DYF[j] / DY[j];
    }
    // Differentiation.cpp:35-61 (the last Dirichlet row's superdiagonal lies
    // outside the matrix and is absent)
    dnd_lo.assign(N, 0); dnd_di.assign(N, 0); ddn_di.assign(N, 0); ddn_up.assign(N, 0);
    for (int j = 2; j <= N - 1; j++) { dnd_lo[j] = -1 / DY[j]; dnd_di[j] = 1 / DY[j]; }
    for (int j = 1; j <= N - 1; j++) { ddn_di[j] = -1 / DYF[j]; if (j < N - 1) ddn_up[j] = 1 / DYF[j]; }
    // Differentiation.cpp:63-101
    full_lo.assign(N, 0); full_di.assign(N, 0); tilde_lo.assign(N, 0); tilde_di.assign(N, 0);
    for (int j = 1; j < N; j++) {
      full_lo[j] = DYF[j] / (2 * DY[j]);
      full_di[j] = DYF[j - 1] / (2 * DY[j]);
      tilde_lo[j] = DYF[j - 1] / (2 * DY[j]);
      tilde_di[j] = DYF[j] / (2 * DY[j]);
    }
  }

  static std::vector<double> kint(int n) {  // Differentiation.cpp:113-132
    std::vector<double> k(n, 0.0);
    if (n == 1) return k;
    int idx = 0;
    for (int v = 0; v <= n / 3; v++) k[idx++] = v;
    for (int v = 0; v < n - 2 * (n / 3) - 1; v++) k[idx++] = 0;
    for (int v = -n / 3; v <= -1; v++) k[idx++] = v;
    return k;
  }

  void build_fourier() {
    auto k1 = kint(N1), k2 = kint(N2);
    T pi = T(3.141592653589793238462);
    kx.assign(M1, 0); kx2.assign(M1, 0); ky.assign(N2, 0); ky2.assign(N2, 0);
    for (int j = 0; j < M1; j++) {
      kx[j] = T(k1[j]) * (2 * pi) / L1;
      kx2[j] = -(kx[j] * kx[j]);  // (i k)^2, FourierSecondDerivativeMatrix
    }
    for (int j = 0; j < N2; j++) {
      ky[j] = (N2 == 1) ? T(0) : T(k2[j]) * (2 * pi) / L2;
      ky2[j] = -(ky[j] * ky[j]);
    }
    keptY.clear();
    if (dim3) {
      for (int j = 0; j < N2 / 3; j++) keptY.push_back(j);
      for (int j = N2 - N2 / 3 + 1; j < N2; j++) keptY.push_back(j);
    } else {
      for (int j = 0; j < N2; j++) keptY.push_back(j);
    }
  }

  template <class F>
  void per_kept(F f) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int iy = 0; iy < int(keptY.size()); iy++)
      for (int n1 = 0; n1 < K1; n1++) f(n1, keptY[iy], iy * K1 + n1);
  }

  // ---- Thomas (Tridiagonal.h:14-53) ----
  // rows given as (a,b,c) per row; a[0] and c[N-1] unused
  static void factor(const T* a, const T* bb, const T* c, T* CC, int N) {
    for (int j = 0; j < N - 1; j++) CC[j] = c[j];
    CC[N - 1] = 0;
    CC[0] = CC[0] / bb[0];
    for (int j = 1; j < N - 1; j++) CC[j] = CC[j] / (bb[j] - a[j] * CC[j - 1]);
  }
  template <class X>
  static void thomas(const T* a, const T* bb, const T* CC, const X* d, X* x, X* D, int N) {
    D[0] = d[0] / bb[0];
    for (int j = 1; j < N; j++) D[j] = (d[j] - a[j] * D[j - 1]) / (bb[j] - a[j] * CC[j - 1]);
    x[N - 1] = D[N - 1];
    for (int j = N - 2; j >= 0; j--) x[j] = D[j] - CC[j] * x[j + 1];
  }

  // Neumannify / Dirichlify (Differentiation.h:17-59) on banded rows
  void neumannify(std::vector<T>& a, std::vector<T>& bb, std::vector<T>& c) const {
    int N = N3;
    bb[0] = 1; c[0] = 0;
    a[1] = 0; bb[1] = 1; c[1] = -1;
    a[N - 2] = 1; bb[N - 2] = -1; c[N - 2] = 0;
    a[N - 1] = 0; bb[N - 1] = 1;
  }
  void dirichlify(std::vector<T>& a, std::vector<T>& bb, std::vector<T>& c) const {
    int N = N3;
    bb[0] = 1; c[0] = 0;
    a[1] = 0; bb[1] = 1; c[1] = 0;
    a[2] = 0; bb[2] = 1; c[2] = 0;
    a[N - 1] = 0; bb[N - 1] = 1;
    bb[N - 2] = 1; c[N - 2] = 0; a[N - 2] = 0;
  }

  // IMEXRK.h:55-78
  void build_laplacian() {
    int N = N3, nk = nkept();
    lap.a.assign(N, 0); lap.c.assign(N, 0);
    lap.bb.assign(size_t(nk) * N, 0); lap.CC.assign(size_t(nk) * N, 0);
    std::vector<T> a(N), bb(N), c(N);
    for (int iy = 0; iy < int(keptY.size()); iy++)
      for (int n1 = 0; n1 < K1; n1++) {
        int n2 = keptY[iy], s = iy * K1 + n1;
        for (int j = 0; j < N; j++) {
          a[j] = d2n_lo[j];
          bb[j] = d2n_di[j] + kx2[n1] + ky2[n2];
          c[j] = d2n_up[j];
        }
        neumannify(a, bb, c);
        if (n1 == 0 && n2 == 0) {
          bb[0] = 1; c[0] = 0;
          a[1] = 0; bb[1] = 1; c[1] = 0;
        }
        // a is the same for every stack; c differs in row 1 for the (0,0)
        // stack but only enters through the per-stack factor CC
        lap.a = a;
        std::copy(bb.begin(), bb.end(), lap.bb.begin() + size_t(s) * N);
        factor(a.data(), bb.data(), c.data(), &lap.CC[size_t(s) * N], N);
      }
  }

  // IMEXRK.h:502-545
  void update_for_timestep() {
    h[0] = T(double(deltaT) * 8.0 / 15.0);
    h[1] = T(double(deltaT) * 2.0 / 15.0);
    h[2] = T(double(deltaT) * 5.0 / 15.0);
    int N = N3, nk = nkept();
    for (int k = 0; k < 3; k++) {
      T s = T(0.5 * double(h[k]));
      for (Fam* F : {&velN[k], &buoN[k], &velD[k]}) {
        F->a.assign(N, 0); F->c.assign(N, 0);
        F->bb.assign(size_t(nk) * N, 0); F->CC.assign(size_t(nk) * N, 0);
      }
      std::vector<T> a(N), bb(N), c(N);
      for (int iy = 0; iy < int(keptY.size()); iy++)
        for (int n1 = 0; n1 < K1; n1++) {
          int n2 = keptY[iy], st = iy * K1 + n1;
          T kk = kx2[n1] + ky2[n2];
          // velocity, Neumann
          for (int j = 0; j < N; j++) {
            a[j] = -(s * d2n_lo[j]) / Re;
            bb[j] = 1 - (s * (d2n_di[j] + kx2[n1] + ky2[n2])) / Re;
            c[j] = -(s * d2n_up[j]) / Re;
          }
          neumannify(a, bb, c);
          if (st == 0) { velN[k].a = a; velN[k].c = c; }
          std::copy(bb.begin(), bb.end(), velN[k].bb.begin() + size_t(st) * N);
          factor(a.data(), bb.data(), c.data(), &velN[k].CC[size_t(st) * N], N);
          // buoyancy, Neumann
          for (int j = 0; j < N; j++) {
            a[j] = -(s * d2n_lo[j]) / Re / Pr;
            bb[j] = 1 - (s * (d2n_di[j] + kx2[n1] + ky2[n2])) / Re / Pr;
            c[j] = -(s * d2n_up[j]) / Re / Pr;
          }
          neumannify(a, bb, c);
          if (st == 0) { buoN[k].a = a; buoN[k].c = c; }
          std::copy(bb.begin(), bb.end(), buoN[k].bb.begin() + size_t(st) * N);
          factor(a.data(), bb.data(), c.data(), &buoN[k].CC[size_t(st) * N], N);
          // velocity, Dirichlet
          for (int j = 0; j < N; j++) {
            a[j] = -(s * d2d_lo[j]) / Re;
            bb[j] = 1 - (s * (d2d_di[j] + kx2[n1] + ky2[n2])) / Re;
            c[j] = -(s * d2d_up[j]) / Re;
          }
          dirichlify(a, bb, c);
          if (st == 0) { velD[k].a = a; velD[k].c = c; }
          std::copy(bb.begin(), bb.end(), velD[k].bb.begin() + size_t(st) * N);
          factor(a.data(), bb.data(), c.data(), &velD[k].CC[size_t(st) * N], N);
          (void)kk;
        }
    }
  }

  // ---------------------------------------------------- FFT of fields ----
  // NodalField::ToModal (Field.h:734-769): r2c per level, 1/(N1 N2), filter
  void to_modal(const std::vector<T>& nod, std::vector<C>& mod) {
    T scale = 1 / static_cast<T>(N1 * N2);
#pragma omp parallel
    {
      std::vector<C> row(N1), col(N2), tmp(size_t(M1) * N2);
#pragma omp for schedule(static)
      for (int n3 = 0; n3 < N3; n3++) {
        for (int n2 = 0; n2 < N2; n2++) {
          for (int n1 = 0; n1 < N1; n1++) row[n1] = C(nod[nidx(n1, n2) + n3], 0);
          fx.run(row.data(), false);
          for (int n1 = 0; n1 < K1; n1++) tmp[size_t(n1) * N2 + n2] = row[n1];
        }
        for (int n1 = 0; n1 < K1; n1++) {
          for (int n2 = 0; n2 < N2; n2++) col[n2] = tmp[size_t(n1) * N2 + n2];
          fy.run(col.data(), false);
          for (int n2 = 0; n2 < N2; n2++) tmp[size_t(n1) * N2 + n2] = col[n2];
        }
        for (int n2 = 0; n2 < N2; n2++)
          for (int n1 = 0; n1 < M1; n1++) mod[midx(n1, n2) + n3] = C(0);
        for (int n2 : keptY)
          for (int n1 = 0; n1 < K1; n1++) mod[midx(n1, n2) + n3] = tmp[size_t(n1) * N2 + n2] * scale;
      }
    }
  }

  // ModalField::ToNodal (Field.h:965-994): c2r per level, unnormalised.
  // Only kept modes are non-zero in every field this is applied to.
  // ncols < M1 skips columns known to be zero (filtered fields)
  void to_nodal(const std::vector<C>& mod, std::vector<T>& nod, int ncols = -1) {
    if (ncols < 0) ncols = M1;
#pragma omp parallel
    {
      std::vector<C> row(N1), col(N2), tmp(size_t(M1) * N2, C(0));
#pragma omp for schedule(static)
      for (int n3 = 0; n3 < N3; n3++) {
        for (int n1 = 0; n1 < ncols; n1++) {
          for (int n2 = 0; n2 < N2; n2++) col[n2] = mod[midx(n1, n2) + n3];
          fy.run(col.data(), true);
          for (int n2 = 0; n2 < N2; n2++) tmp[size_t(n1) * N2 + n2] = col[n2];
        }
        for (int n2 = 0; n2 < N2; n2++) {
          row[0] = C(tmp[n2].real(), 0);
          for (int n1 = 1; n1 < N1 / 2; n1++) {
            row[n1] = tmp[size_t(n1) * N2 + n2];
            row[N1 - n1] = std::conj(row[n1]);
          }
          row[N1 / 2] = C(tmp[size_t(N1 / 2) * N2 + n2].real(), 0);
          fx.run(row.data(), true);
          for (int n1 = 0; n1 < N1; n1++) nod[nidx(n1, n2) + n3] = row[n1].real();
        }
      }
    }
  }

  // ------------------------------------------------- vertical stencils ----
  template <class X> X D2N(const X* f, int j) const {
    if (j < 1 || j > N3 - 2) return X(0);
    return d2n_lo[j] * f[j - 1] + d2n_di[j] * f[j] + d2n_up[j] * f[j + 1];
  }
  template <class X> X D2D(const X* f, int j) const {
    if (j < 2 || j > N3 - 2) return X(0);
    return d2d_lo[j] * f[j - 1] + d2d_di[j] * f[j] + d2d_up[j] * f[j + 1];
  }
  template <class X> X DzND(const X* f, int j) const {  // Neumann -> Dirichlet
    if (j < 2) return X(0);
    return dnd_lo[j] * f[j - 1] + dnd_di[j] * f[j];
  }
  template <class X> X DzDN(const X* f, int j) const {  // Dirichlet -> Neumann
    if (j < 1) return X(0);
    if (j == N3 - 1) return ddn_di[j] * f[j];
    return ddn_di[j] * f[j] + ddn_up[j] * f[j + 1];
  }
  template <class X> X Full(const X* f, int j) const {
    if (j < 1) return X(0);
    return full_lo[j] * f[j - 1] + full_di[j] * f[j];
  }
  template <class X> X Bar(const X* f, int j) const {
    if (j < 1) return X(0);
    return T(0.5) * f[j - 1] + T(0.5) * f[j];
  }
  template <class X> X Tilde(const X* f, int j) const {
    if (j < 1) return X(0);
    return tilde_lo[j] * f[j - 1] + tilde_di[j] * f[j];
  }
  template <class X> X Dir(const X* f, int j) const {
    if (j == N3 - 1) return T(0.5) * f[j];
    return T(0.5) * f[j] + T(0.5) * f[j + 1];
  }

  // nodal helpers: f(j) over each (n1,n2) stack of nodal arrays
  template <class F>
  void nodal_eval(std::vector<T>& out, F f) {
#pragma omp parallel for collapse(2) schedule(static)
    for (int n2 = 0; n2 < N2; n2++)
      for (int n1 = 0; n1 < N1; n1++) {
        size_t o = nidx(n1, n2);
        for (int j = 0; j < N3; j++) out[o + j] = f(o, j);
      }
  }

  // ------------------------------------------------------ the scheme ----
  void populate_nodal() {  // IMEXRK.h:141-162
    // the four fields are filtered before every call, so only the K1 kept
    // columns are non-zero
    to_nodal(u1, U1, K1);
    if (dim3) to_nodal(u2, U2, K1);
    to_nodal(u3, U3, K1);
    to_nodal(b, B, K1);
  }

  void zero_ends(std::vector<C>& f, BC bc, size_t o) const {  // Field.h:475-486
    f[o + 0] = C(0); f[o + 1] = C(0); f[o + N3 - 1] = C(0); f[o + N3 - 2] = C(0);
    if (bc == Dirichlet) f[o + 2] = C(0);
  }

  void solve_fam(const Fam& F, std::vector<C>& R, std::vector<C>& into, BC bc) {
    int N = N3;
    per_kept([&](int n1, int n2, int s) {
      size_t o = midx(n1, n2);
      zero_ends(R, bc, o);
      std::vector<T> dr(N), di(N), xr(N), xi(N), D(N);
      for (int j = 0; j < N; j++) { dr[j] = R[o + j].real(); di[j] = R[o + j].imag(); }
      const T* bb = &F.bb[size_t(s) * N];
      const T* CC = &F.CC[size_t(s) * N];
      thomas<T>(F.a.data(), bb, CC, dr.data(), xr.data(), D.data(), N);
      thomas<T>(F.a.data(), bb, CC, di.data(), xi.data(), D.data(), N);
      for (int j = 0; j < N; j++) into[o + j] = C(xr[j], xi[j]);
    });
  }

  // IMEXRK.cpp:43-73
  void remove_divergence(T pressureMultiplier) {
    int N = N3;
    per_kept([&](int n1, int n2, int s) {
      size_t o = midx(n1, n2);
      C ikx(0, kx[n1]), iky(0, ky[n2]);
      for (int j = 0; j < N; j++) {
        C d = ikx * u1[o + j];
        if (dim3) d += iky * u2[o + j];
        d += DzDN(&u3[o], j);
        div[o + j] = d;
      }
      zero_ends(div, Neumann, o);
      std::vector<T> dr(N), di(N), xr(N), xi(N), D(N);
      for (int j = 0; j < N; j++) { dr[j] = div[o + j].real(); di[j] = div[o + j].imag(); }
      const std::vector<T>& a = lap.a;
      thomas<T>(a.data(), &lap.bb[size_t(s) * N], &lap.CC[size_t(s) * N], dr.data(), xr.data(), D.data(), N);
      thomas<T>(a.data(), &lap.bb[size_t(s) * N], &lap.CC[size_t(s) * N], di.data(), xi.data(), D.data(), N);
      for (int j = 0; j < N; j++) q[o + j] = C(xr[j], xi[j]);
      std::vector<C> du3(N);
      for (int j = 0; j < N; j++) du3[j] = DzND(&q[o], j);
      for (int j = 0; j < N; j++) {
        u1[o + j] -= ikx * q[o + j];
        if (dim3) u2[o + j] -= iky * q[o + j];
        u3[o + j] -= du3[j];
        p[o + j] += pressureMultiplier * q[o + j];
      }
    });
  }

  // IMEXRK.cpp:119-134
  void explicit_rk(int k) {
    T hz = T(double(h[k]) * zeta[k]);
    T mh = -h[k];
    per_kept([&](int n1, int n2, int s) {
      size_t o = midx(n1, n2);
      C ikx(0, kx[n1]), iky(0, ky[n2]);
      for (int j = 0; j < N3; j++) {
        R1[o + j] = u1[o + j] + hz * r1[o + j] + mh * (ikx * p[o + j]);
        if (dim3) R2[o + j] = u2[o + j] + hz * r2[o + j] + mh * (iky * p[o + j]);
        R3[o + j] = u3[o + j] + hz * r3[o + j] + mh * DzND(&p[o], j);
        RB[o + j] = b[o + j] + hz * rB[o + j];
      }
    });
    for (auto* f : {&r1, &r2, &r3, &rB}) std::fill(f->begin(), f->end(), C(0));
  }

  // IMEXRK.cpp:107-117
  void finish_rhs(int k) {
    T hb = T(double(h[k]) * beta[k]);
    per_kept([&](int n1, int n2, int s) {
      size_t o = midx(n1, n2);
      for (int j = 0; j < N3; j++) {
        R1[o + j] += hb * r1[o + j];
        if (dim3) R2[o + j] += hb * r2[o + j];
        R3[o + j] += hb * r3[o + j];
        RB[o + j] += hb * rB[o + j];
      }
    });
  }

  // IMEXRK.cpp:75-105
  void crank_nicolson(int k) {
    T cv = T(0.5) * h[k] / Re;
    T cb = T(0.5) * h[k] / Re / Pr;
    per_kept([&](int n1, int n2, int s) {
      size_t o = midx(n1, n2);
      for (int j = 0; j < N3; j++) {
        R1[o + j] += cv * (kx2[n1] * u1[o + j] + ky2[n2] * u1[o + j] + D2N(&u1[o], j));
        if (dim3) R2[o + j] += cv * (kx2[n1] * u2[o + j] + ky2[n2] * u2[o + j] + D2N(&u2[o], j));
        R3[o + j] += cv * (kx2[n1] * u3[o + j] + ky2[n2] * u3[o + j] + D2D(&u3[o], j));
        RB[o + j] += cb * (kx2[n1] * b[o + j] + ky2[n2] * b[o + j] + D2N(&b[o], j));
      }
    });
    solve_fam(velN[cur_k], R1, u1, Neumann);
    if (dim3) solve_fam(velN[cur_k], R2, u2, Neumann);
    solve_fam(velD[cur_k], R3, u3, Dirichlet);
    solve_fam(buoN[cur_k], RB, b, Neumann);
  }
  int cur_k = 0;

  // linear buoyancy terms of BuildRHS (IMEXRK.cpp:140-147), generalised
  // background stratification dBdz (=1 in the reference)
  void linear_terms() {
    per_kept([&](int n1, int n2, int s) {
      size_t o = midx(n1, n2);
      bool zero_mode = (n1 == 0 && n2 == 0);
      for (int j = 0; j < N3; j++) {
        if (!zero_mode) r3[o + j] += Ri * Full(&b[o], j);
        rB[o + j] -= dBdz[j] * Dir(&u3[o], j);
      }
    });
  }

  // r (modal) op= mult * prod, mult applied per kept stack
  enum Mul { One, IKX, IKY };
  void accum(std::vector<C>& r, const std::vector<C>& m, Mul mul, T sign) {
    per_kept([&](int n1, int n2, int s) {
      size_t o = midx(n1, n2);
      C f = (mul == IKX) ? C(0, kx[n1]) : (mul == IKY) ? C(0, ky[n2]) : C(1, 0);
      for (int j = 0; j < N3; j++) r[o + j] += sign * (f * m[o + j]);
    });
  }
  void accum_dznd(std::vector<C>& r, const std::vector<C>& m, T sign) {
    per_kept([&](int n1, int n2, int s) {
      size_t o = midx(n1, n2);
      std::vector<C> t(N3);
      for (int j = 0; j < N3; j++) t[j] = DzND(&m[o], j);
      for (int j = 0; j < N3; j++) r[o + j] += sign * t[j];
    });
  }

  // IMEXRK.cpp:136-193 with the products of Stratiflow.h:112-139
  void build_rhs() {
    linear_terms();
    for (size_t i = 0; i < U1.size(); i++) U1t[i] = U1[i] + Ubar[i % N3];
    // U1t*U1t -> r1 -= ddx
    nodal_eval(prod, [&](size_t o, int j) { return U1t[o + j] * U1t[o + j]; });
    to_modal(prod, ntmp); accum(r1, ntmp, IKX, -1);
    // ddz(Bar(U1t)*U3) -> r1 -=
    product_bar_dz(U1t, U3); to_modal(prod, ntmp); accum(r1, ntmp, One, -1);
    // Tilde(U1t)*U3 -> dtmp ; Dir(U3)*Dir(U3) -> ntmp ; r3 -= ddx(dtmp) + ddz(ntmp)
    nodal_eval(prod, [&](size_t o, int j) { return Tilde(&U1t[o], j) * U3[o + j]; });
    to_modal(prod, dtmp);
    nodal_eval(prod, [&](size_t o, int j) { return Dir(&U3[o], j) * Dir(&U3[o], j); });
    to_modal(prod, ntmp);
    accum(r3, dtmp, IKX, -1); accum_dznd(r3, ntmp, -1);
    if (dim3) {
      nodal_eval(prod, [&](size_t o, int j) { return U2[o + j] * U2[o + j]; });
      to_modal(prod, ntmp); accum(r2, ntmp, IKY, -1);
      product_bar_dz(U2, U3); to_modal(prod, ntmp); accum(r2, ntmp, One, -1);
      nodal_eval(prod, [&](size_t o, int j) { return Tilde(&U2[o], j) * U3[o + j]; });
      to_modal(prod, dtmp); accum(r3, dtmp, IKY, -1);
      nodal_eval(prod, [&](size_t o, int j) { return U1t[o + j] * U2[o + j]; });
      to_modal(prod, ntmp); accum(r1, ntmp, IKY, -1); accum(r2, ntmp, IKX, -1);
    }
    product_bar_dz(B, U3); to_modal(prod, ntmp); accum(rB, ntmp, One, -1);
    if (dim3) {
      nodal_eval(prod, [&](size_t o, int j) { return U2[o + j] * B[o + j]; });
      to_modal(prod, ntmp); accum(rB, ntmp, IKY, -1);
    }
    nodal_eval(prod, [&](size_t o, int j) { return U1t[o + j] * B[o + j]; });
    to_modal(prod, ntmp); accum(rB, ntmp, IKX, -1);
  }

  // prod = ddz(Bar(A)*Bd) with Bd a Dirichlet nodal field (Stratiflow.h:119-124)
  void product_bar_dz(const std::vector<T>& A, const std::vector<T>& Bd) {
    nodal_eval(prod2, [&](size_t o, int j) { return Bar(&A[o], j) * Bd[o + j]; });
    nodal_eval(prod, [&](size_t o, int j) { return DzDN(&prod2[o], j); });
  }
  // prod = ddz(Bar(A1)*B1 + Bar(A2)*B2) (Stratiflow.h:149-156)
  void product_bar_dz2(const std::vector<T>& A1, const std::vector<T>& A2,
                       const std::vector<T>& B1, const std::vector<T>& B2) {
    nodal_eval(prod2, [&](size_t o, int j) {
      return Bar(&A1[o], j) * B1[o + j] + Bar(&A2[o], j) * B2[o + j];
    });
    nodal_eval(prod, [&](size_t o, int j) { return DzDN(&prod2[o], j); });
  }

  // IMEXRK.cpp:195-258
  void build_rhs_linear() {
    linear_terms();
    std::vector<T>& nn = U1t;  // nnTemp = U1_tot + U_
    for (size_t i = 0; i < U1b.size(); i++) nn[i] = U1b[i] + Ubar[i % N3];
    nodal_eval(prod, [&](size_t o, int j) { return U1[o + j] * nn[o + j]; });
    to_modal(prod, ntmp); accum(r1, ntmp, IKX, -2);
    product_bar_dz2(U1, nn, U3b, U3); to_modal(prod, ntmp); accum(r1, ntmp, One, -1);
    nodal_eval(prod, [&](size_t o, int j) {
      return Tilde(&U1[o], j) * U3b[o + j] + Tilde(&nn[o], j) * U3[o + j];
    });
    to_modal(prod, dtmp);
    nodal_eval(prod, [&](size_t o, int j) { return Dir(&U3[o], j) * Dir(&U3b[o], j); });
    to_modal(prod, ntmp);
    accum(r3, dtmp, IKX, -1); accum_dznd(r3, ntmp, -2);
    if (dim3) {
      product_bar_dz2(U2, U2b, U3b, U3); to_modal(prod, ntmp); accum(r2, ntmp, One, -1);
      nodal_eval(prod, [&](size_t o, int j) { return U2[o + j] * U2b[o + j]; });
      to_modal(prod, ntmp); accum(r2, ntmp, IKY, -2);
      nodal_eval(prod, [&](size_t o, int j) {
        return Tilde(&U2[o], j) * U3b[o + j] + Tilde(&U2b[o], j) * U3[o + j];
      });
      to_modal(prod, dtmp); accum(r3, dtmp, IKY, -1);
      nodal_eval(prod, [&](size_t o, int j) { return U1[o + j] * U2b[o + j] + nn[o + j] * U2[o + j]; });
      to_modal(prod, ntmp); accum(r1, ntmp, IKY, -1); accum(r2, ntmp, IKX, -1);
    }
    product_bar_dz2(B, Bb, U3b, U3); to_modal(prod, ntmp); accum(rB, ntmp, One, -1);
    if (dim3) {
      nodal_eval(prod, [&](size_t o, int j) { return B[o + j] * U2b[o + j] + Bb[o + j] * U2[o + j]; });
      to_modal(prod, ntmp); accum(rB, ntmp, IKY, -1);
    }
    nodal_eval(prod, [&](size_t o, int j) { return B[o + j] * nn[o + j] + Bb[o + j] * U1[o + j]; });
    to_modal(prod, ntmp); accum(rB, ntmp, IKX, -1);
  }

  // ---- adjoint step (IMEXRK.h:86-126, 461-500; IMEXRK.cpp:260-379) ----
  // direct total fields of the current RK substep, modal and nodal
  std::vector<C> u1T, u2T, u3T, bT, mtmp;
  std::vector<T> U1T, U2T, U3T, BT, U1F, U2F, U3F, BF, nd1, nd2;
  T adjK = T(2);

  void adjoint_alloc() {
    if (!u1T.empty()) return;
    for (auto* f : {&u1T, &u2T, &u3T, &bT, &mtmp}) f->assign(u1.size(), C(0));
    for (auto* f : {&U1T, &U2T, &U3T, &BT, &U1F, &U2F, &U3F, &BF, &nd1, &nd2}) f->assign(U1.size(), T(0));
  }

  // IMEXRK::UpdateAdjointVariables (IMEXRK.h:461-500), the mixing objective's
  // forcing; J itself is not needed by the step
  void update_adjoint_variables() {
    to_nodal(u1T, U1T);
    if (dim3) to_nodal(u2T, U2T); else std::fill(U2T.begin(), U2T.end(), T(0));
    to_nodal(u3T, U3T);
    to_nodal(bT, BT);
    const size_t o00 = midx(0, 0);
    std::vector<T> bave(N3), wave(N3);   // HorizontalAverage (Integration.h:38-42)
    for (int j = 0; j < N3; j++) { bave[j] = bT[o00 + j].real(); wave[j] = u3T[o00 + j].real(); }
    adjK = T(2);
    nodal_eval(U3F, [&](size_t o, int j) { return (T(1) / adjK) * (BT[o + j] - bave[j]); });
    nodal_eval(BF, [&](size_t o, int j) { return (T(1) / adjK) * (U3T[o + j] - wave[j]); });
    std::fill(U1F.begin(), U1F.end(), T(0));
    std::fill(U2F.begin(), U2F.end(), T(0));
  }

  // modal derivative of a direct field, to nodal: mul = IKX (ddx) or
  // DzND / DzDN (ddz), as in `neumannTemp = ddx(u1_tot); ...ToNodal`
  enum DerivKind { D_X, D_Y, DZ_ND, DZ_DN };
  void deriv_nodal(const std::vector<C>& f, DerivKind kd, std::vector<T>& out) {
    per_kept([&](int n1, int n2, int s) {
      (void)s;
      size_t o = midx(n1, n2);
      for (int j = 0; j < N3; j++) {
        C v;
        if (kd == D_X) v = C(0, kx[n1]) * f[o + j];
        else if (kd == D_Y) v = C(0, ky[n2]) * f[o + j];
        else if (kd == DZ_ND) v = DzND(&f[o], j);
        else v = DzDN(&f[o], j);
        mtmp[o + j] = v;
      }
    });
    to_nodal(mtmp, out);
  }

  // IMEXRK::BuildRHSAdjoint (IMEXRK.cpp:260-379), 2D and 3D
  void build_rhs_adjoint() {
    // adjoint buoyancy
    nodal_eval(prod, [&](size_t o, int j) { return BF[o + j] + Ri * Dir(&U3[o], j); });
    BF.swap(prod);
    // advection of adjoint quantities by the direct flow
    nodal_eval(prod, [&](size_t o, int j) { return U1[o + j] * U1T[o + j]; });
    to_modal(prod, ntmp); accum(r1, ntmp, IKX, 1);
    product_bar_dz(U1, U3T); to_modal(prod, ntmp); accum(r1, ntmp, One, 1);
    nodal_eval(prod, [&](size_t o, int j) { return Tilde(&U1T[o], j) * U3[o + j]; });
    to_modal(prod, dtmp);
    nodal_eval(prod, [&](size_t o, int j) { return Dir(&U3[o], j) * Dir(&U3T[o], j); });
    to_modal(prod, ntmp);
    accum(r3, dtmp, IKX, 1); accum_dznd(r3, ntmp, 1);
    if (dim3) {
      nodal_eval(prod, [&](size_t o, int j) { return U2[o + j] * U2T[o + j]; });
      to_modal(prod, ntmp); accum(r2, ntmp, IKY, 1);
      product_bar_dz(U2, U3T); to_modal(prod, ntmp); accum(r2, ntmp, One, 1);
      nodal_eval(prod, [&](size_t o, int j) { return Tilde(&U2T[o], j) * U3[o + j]; });
      to_modal(prod, dtmp); accum(r3, dtmp, IKY, 1);
      nodal_eval(prod, [&](size_t o, int j) { return U1[o + j] * U2T[o + j]; });
      to_modal(prod, ntmp); accum(r1, ntmp, IKY, 1);
      nodal_eval(prod, [&](size_t o, int j) { return U2[o + j] * U1T[o + j]; });
      to_modal(prod, ntmp); accum(r2, ntmp, IKX, 1);
    }
    product_bar_dz(B, U3T); to_modal(prod, ntmp); accum(rB, ntmp, One, 1);
    if (dim3) {
      nodal_eval(prod, [&](size_t o, int j) { return B[o + j] * U2T[o + j]; });
      to_modal(prod, ntmp); accum(rB, ntmp, IKY, 1);
    }
    nodal_eval(prod, [&](size_t o, int j) { return B[o + j] * U1T[o + j]; });
    to_modal(prod, ntmp); accum(rB, ntmp, IKX, 1);

    // extra adjoint terms: (grad u_tot)^T u-adjoint and grad b_tot b-adjoint
    deriv_nodal(u1T, D_X, nd1);                                   // ddx(u1_tot), Neumann
    nodal_eval(prod2, [&](size_t o, int j) { return nd1[o + j] * U1[o + j]; });
    if (dim3) {
      deriv_nodal(u2T, D_X, nd1);
      nodal_eval(prod2, [&](size_t o, int j) { return prod2[o + j] + nd1[o + j] * U2[o + j]; });
    }
    deriv_nodal(u3T, D_X, nd2);                                   // ddx(u3_tot), Dirichlet
    nodal_eval(prod, [&](size_t o, int j) { return nd2[o + j] * U3[o + j]; });
    nodal_eval(U1F, [&](size_t o, int j) { return U1F[o + j] - (prod2[o + j] + Dir(&prod[o], j)); });
    if (dim3) {
      deriv_nodal(u1T, D_Y, nd1);
      nodal_eval(prod2, [&](size_t o, int j) { return nd1[o + j] * U1[o + j]; });
      deriv_nodal(u2T, D_Y, nd1);
      nodal_eval(prod2, [&](size_t o, int j) { return prod2[o + j] + nd1[o + j] * U2[o + j]; });
      deriv_nodal(u3T, D_Y, nd2);
      nodal_eval(prod, [&](size_t o, int j) { return nd2[o + j] * U3[o + j]; });
      nodal_eval(U2F, [&](size_t o, int j) { return U2F[o + j] - (prod2[o + j] + Dir(&prod[o], j)); });
    }
    deriv_nodal(u1T, DZ_ND, nd2);                                // ddz(u1_tot), Dirichlet
    nodal_eval(prod2, [&](size_t o, int j) { return nd2[o + j] * Full(&U1[o], j); });
    if (dim3) {
      deriv_nodal(u2T, DZ_ND, nd2);
      nodal_eval(prod2, [&](size_t o, int j) { return prod2[o + j] + nd2[o + j] * Full(&U2[o], j); });
    }
    deriv_nodal(u3T, DZ_DN, nd1);                                // ddz(u3_tot), Neumann
    nodal_eval(U3F, [&](size_t o, int j) { return U3F[o + j] - (prod2[o + j] + Full(&nd1[o], j) * U3[o + j]); });
    deriv_nodal(bT, D_X, nd1);                                    // ddx(b_tot)
    nodal_eval(U1F, [&](size_t o, int j) { return U1F[o + j] - nd1[o + j] * B[o + j]; });
    if (dim3) {
      deriv_nodal(bT, D_Y, nd1);
      nodal_eval(U2F, [&](size_t o, int j) { return U2F[o + j] - nd1[o + j] * B[o + j]; });
    }
    deriv_nodal(bT, DZ_ND, nd2);                                 // ddz(b_tot), Dirichlet
    nodal_eval(U3F, [&](size_t o, int j) { return U3F[o + j] - nd2[o + j] * Full(&B[o], j); });
    // the forcing terms
    to_modal(U1F, ntmp); accum(r1, ntmp, One, 1);
    if (dim3) { to_modal(U2F, ntmp); accum(r2, ntmp, One, 1); }
    to_modal(U3F, dtmp); accum(r3, dtmp, One, 1);
    to_modal(BF, ntmp); accum(rB, ntmp, One, 1);
  }

  // IMEXRK::TimeStepAdjoint (IMEXRK.h:86-126): the direct state below (the
  // earlier time) and above (the later one), modal, reference layout
  void time_step_adjoint(const std::vector<C>* below, const std::vector<C>* above) {
    adjoint_alloc();
    T interpFrac = 0;
    for (int k = 0; k < 3; k++) {
      cur_k = k;
      std::vector<C>* tot[4] = {&u1T, &u2T, &u3T, &bT};
      for (int f = 0; f < 4; f++)
        for (size_t i = 0; i < u1.size(); i++) (*tot[f])[i] = (T(1) - interpFrac) * above[f][i] + interpFrac * below[f][i];
      // u1_tot += U_ through nodal space
      to_nodal(u1T, U1T);
      for (size_t i = 0; i < U1T.size(); i++) U1T[i] += Ubar[i % N3];
      to_modal(U1T, u1T);
      update_adjoint_variables();
      explicit_rk(k);
      build_rhs_adjoint();
      finish_rhs(k);
      stage_common_tail(k);
      interpFrac += h[k] / deltaT;
    }
  }

  void filter_all() {  // IMEXRK.h:128-139 with Field.h:996-1021
    std::vector<char> keep(N2, 0);
    for (int n2 : keptY) keep[n2] = 1;
    for (auto* f : {&u1, &u2, &u3, &b, &p})
      for (int n2 = 0; n2 < N2; n2++)
        for (int n1 = 0; n1 < M1; n1++)
          if (n1 >= K1 || !keep[n2])
            for (int j = 0; j < N3; j++) (*f)[midx(n1, n2) + j] = C(0);
    if (!dim3) std::fill(u2.begin(), u2.end(), C(0));
  }

  void stage_common_tail(int k) {
    crank_nicolson(k);
    remove_divergence(1 / h[k]);
    filter_all();
    populate_nodal();
  }

  void time_step() {  // IMEXRK.cpp:8-24
    for (int k = 0; k < 3; k++) {
      cur_k = k;
      explicit_rk(k);
      build_rhs();
      finish_rhs(k);
      stage_common_tail(k);
    }
  }
  void time_step_linear() {  // IMEXRK.cpp:26-41
    for (int k = 0; k < 3; k++) {
      cur_k = k;
      explicit_rk(k);
      build_rhs_linear();
      finish_rhs(k);
      stage_common_tail(k);
    }
  }

  // StateVector::FixedEvolve set-up (StateVector.cpp:85-105): FilterAll,
  // PopulateNodalVariables, RemoveDivergence(0), PrepareRun's populate
  void prepare() {
    filter_all();
    populate_nodal();
    remove_divergence(T(0));
    populate_nodal();
  }

  // Integration.h:5-35 (vertical quadrature)
  T integrate_vertically(const std::vector<T>& f, BC bc) const {
    T result = 0;
    if (bc == Neumann) {
      for (int k = 1; k < N3 - 1; k++) result += (z[k + 1] - z[k]) * f[k];
    } else {
      for (int k = 2; k < N3 - 1; k++) result += (zf[k] - zf[k - 1]) * f[k];
    }
    return result;
  }
  // Integration.h:282-311
  T inner_prod(const std::vector<C>& a, const std::vector<C>& bv, BC bc) const {
    std::vector<T> horz(N3, 0);
    for (int j3 = 0; j3 < N3; j3++) {
      T sum = 0;
      for (int j1 = 0; j1 < M1; j1++)
        for (int j2 = 0; j2 < N2; j2++) {
          size_t o = midx(j1, j2) + j3;
          T v = std::real(a[o] * std::conj(bv[o]));
          sum += (j1 == 0 && j2 == 0) ? v : 2 * v;
        }
      horz[j3] = sum;
    }
    return integrate_vertically(horz, bc);
  }
  T KE() const {  // IMEXRK.h:395-406
    T e = T(0.5) * (inner_prod(u1, u1, Neumann) + inner_prod(u3, u3, Dirichlet));
    if (dim3) e += T(0.5) * inner_prod(u2, u2, Neumann);
    return e;
  }
  T PE() const { return Ri * T(0.5) * inner_prod(b, b, Neumann); }  // IMEXRK.h:408-411

  // Dissipation rates in the normalisation of KE and PE (the reference has no
  // such diagnostic; it is the sink of KE and PE that the viscous and
  // diffusive terms of CrankNicolson, IMEXRK.cpp:75-105, produce):
  //   eps = (1/Re) sum_i InnerProd(grad u_i, grad u_i)
  //   chi = Ri/(Re Pr) InnerProd(grad b, grad b)
  // with ddx, ddy the Fourier multipliers (Differentiation.cpp:134-160) and
  // ddz the staggered bidiagonal operators (Differentiation.cpp:35-61), each
  // gradient component integrated by InnerProd at the location it lives on.
  T grad_sq(const std::vector<C>& f, BC bc) const {
    std::vector<C> d(f.size(), C(0));
    T s = 0;
    for (int dir = 0; dir < 3; dir++) {
      if (dir == 1 && !dim3) continue;
      for (int n2 = 0; n2 < N2; n2++)
        for (int n1 = 0; n1 < M1; n1++) {
          const size_t o = midx(n1, n2);
          for (int j = 0; j < N3; j++) {
            if (dir == 0) d[o + j] = C(0, kx[n1]) * f[o + j];
            else if (dir == 1) d[o + j] = C(0, ky[n2]) * f[o + j];
            else d[o + j] = (bc == Neumann) ? DzND(&f[o], j) : DzDN(&f[o], j);
          }
        }
      const BC at = (dir == 2) ? (bc == Neumann ? Dirichlet : Neumann) : bc;
      s += inner_prod(d, d, at);
    }
    return s;
  }
  void dissipation(T& eps, T& chi) const {
    T g = grad_sq(u1, Neumann) + grad_sq(u3, Dirichlet);
    if (dim3) g += grad_sq(u2, Neumann);
    eps = g / Re;
    chi = Ri / (Re * Pr) * grad_sq(b, Neumann);
  }

  // Nodal1D::SetValue for a Neumann profile (Field.h:661-682)
  void set_background(const double* U) {
    for (int j = 0; j < N3; j++) Ubar[j] = T(U[j]);
  }
};

template <class T> constexpr double Solver<T>::beta[3];
template <class T> constexpr double Solver<T>::zeta[3];

// ------------------------------------------------------------ helpers ----
static inline uint64_t splitmix64(uint64_t& s) {
  uint64_t z = (s += 0x9E3779B97F4A7C15ull);
  z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
  z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
  return z ^ (z >> 31);
}
static inline double unit01(uint64_t& s) {  // (0,1]
  return (double((splitmix64(s) >> 11) + 1)) * (1.0 / 9007199254740992.0);
}
static inline void gauss2(uint64_t& s, double& g0, double& g1) {  // Box-Muller
  double u1 = unit01(s), u2 = unit01(s);
  double r = std::sqrt(-2.0 * std::log(u1));
  g0 = r * std::cos(2.0 * M_PI * u2);
  g1 = r * std::sin(2.0 * M_PI * u2);
}

struct Handle {
  int prec;
  Solver<float>* sf = nullptr;
  Solver<double>* sd = nullptr;
};

}  // namespace sfo

using namespace sfo;

template <class T>
static std::vector<std::complex<T>>* field_ptr(Solver<T>* s, int f) {
  switch (f) {
    case 0: return &s->u1;
    case 1: return &s->u2;
    case 2: return &s->u3;
    case 3: return &s->b;
    case 4: return &s->p;
    case 5: return &s->r1;
    case 6: return &s->r2;
    case 7: return &s->r3;
    case 8: return &s->rB;
  }
  return nullptr;
}

#define DISPATCH(h, ...)                   \
  do {                                     \
    if ((h)->prec == 64) {                 \
      auto* S = (h)->sd;                   \
      __VA_ARGS__;                         \
    } else {                               \
      auto* S = (h)->sf;                   \
      __VA_ARGS__;                         \
    }                                      \
  } while (0)

extern "C" {

// Create an oracle solver. prec = 32 (reference default build) or 64
// (reference -DDOUBLE build). Mirrors IMEXRK::IMEXRK (IMEXRK.h:37-81) with
// runtime grid sizes.
void* sfo_create(int prec, int N1, int N2, int N3, double L1, double L2, double L3, double Re,
                 double Ri, double Pr, double dt) {
  // the own FFT is radix-2: N1 and N2 must be powers of two; N3 % 4 == 0
  // as asserted by VerticalPoints (Field.cpp:7)
  auto pow2 = [](int n) { return n > 0 && (n & (n - 1)) == 0; };
  if (!pow2(N1) || !pow2(N2) || N1 < 8 || N3 < 8 || N3 % 4 != 0) return nullptr;
  auto* h = new Handle();
  h->prec = prec;
  if (prec == 64) {
    h->sd = new Solver<double>();
    h->sd->deltaT = dt;
    h->sd->init(N1, N2, N3, L1, L2, L3, Re, Ri, Pr);
  } else {
    h->sf = new Solver<float>();
    h->sf->deltaT = float(dt);
    h->sf->init(N1, N2, N3, L1, L2, L3, Re, Ri, Pr);
  }
  return h;
}

void sfo_destroy(void* hv) {
  auto* h = (Handle*)hv;
  delete h->sf;
  delete h->sd;
  delete h;
}

void sfo_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n);
#endif
  (void)n;
}
int sfo_get_threads() {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

// IMEXRK::deltaT + UpdateForTimestep (IMEXRK.h:502-545)
void sfo_set_dt(void* hv, double dt) {
  auto* h = (Handle*)hv;
  DISPATCH(h, { S->deltaT = decltype(S->deltaT)(dt); S->update_for_timestep(); });
}
void sfo_set_ri(void* hv, double ri) {
  auto* h = (Handle*)hv;
  DISPATCH(h, { S->Ri = decltype(S->Ri)(ri); });
}

// IMEXRK::SetBackground (IMEXRK.h:321-332) plus the background
// stratification profile dB/dz at the Neumann levels.
void sfo_set_background(void* hv, const double* U, const double* dBdz) {
  auto* h = (Handle*)hv;
  DISPATCH(h, {
    S->set_background(U);
    for (int j = 0; j < S->N3; j++) S->dBdz[j] = decltype(S->Ri)(dBdz[j]);
  });
}

// grid arrays: which = 0 z, 1 zf, 2 DY, 3 DYF
void sfo_get_grid(void* hv, int which, double* out) {
  auto* h = (Handle*)hv;
  DISPATCH(h, {
    auto& v = which == 0 ? S->z : which == 1 ? S->zf : which == 2 ? S->DY : S->DYF;
    for (int j = 0; j < S->N3; j++) out[j] = double(v[j]);
  });
}

// Field raw data in the reference layout, complex as interleaved doubles,
// (M1*n2+n1)*N3+n3. field: 0 u1, 1 u2, 2 u3, 3 b, 4 p, 5..8 r1,r2,r3,rB.
void sfo_set_field(void* hv, int field, const double* ri) {
  auto* h = (Handle*)hv;
  DISPATCH(h, {
    auto* f = field_ptr(S, field);
    using Tt = decltype(S->Ri);
    for (size_t i = 0; i < f->size(); i++) (*f)[i] = std::complex<Tt>(Tt(ri[2 * i]), Tt(ri[2 * i + 1]));
  });
}
void sfo_get_field(void* hv, int field, double* ri) {
  auto* h = (Handle*)hv;
  DISPATCH(h, {
    auto* f = field_ptr(S, field);
    for (size_t i = 0; i < f->size(); i++) {
      ri[2 * i] = double((*f)[i].real());
      ri[2 * i + 1] = double((*f)[i].imag());
    }
  });
}
// nodal U1,U2,U3,B (which 0..3), (N1*n2+n1)*N3+n3
void sfo_get_nodal(void* hv, int which, double* out) {
  auto* h = (Handle*)hv;
  DISPATCH(h, {
    auto& v = which == 0 ? S->U1 : which == 1 ? S->U2 : which == 2 ? S->U3 : S->B;
    for (size_t i = 0; i < v.size(); i++) out[i] = double(v[i]);
  });
}

// FixedEvolve's set-up (StateVector.cpp:85-105)
void sfo_prepare(void* hv) {
  auto* h = (Handle*)hv;
  DISPATCH(h, S->prepare());
}
void sfo_step(void* hv, int n) {  // IMEXRK::TimeStep
  auto* h = (Handle*)hv;
  DISPATCH(h, { for (int i = 0; i < n; i++) S->time_step(); });
}
void sfo_step_linear(void* hv, int n) {  // IMEXRK::TimeStepLinear
  auto* h = (Handle*)hv;
  DISPATCH(h, { for (int i = 0; i < n; i++) S->time_step_linear(); });
}
void sfo_remove_divergence(void* hv, double pm) {
  auto* h = (Handle*)hv;
  DISPATCH(h, S->remove_divergence(decltype(S->Ri)(pm)));
}
void sfo_populate_nodal(void* hv) {
  auto* h = (Handle*)hv;
  DISPATCH(h, S->populate_nodal());
}
void sfo_filter_all(void* hv) {
  auto* h = (Handle*)hv;
  DISPATCH(h, S->filter_all());
}

// IMEXRK::TimeStepAdjoint (IMEXRK.h:86-126): below and above hold the direct
// state's u1, u2, u3, b (modal, reference layout, re/im interleaved), one
// field after the other
void sfo_step_adjoint(void* hv, const double* below, const double* above) {
  auto* h = (Handle*)hv;
  DISPATCH(h, {
    using Tt = decltype(S->Ri);
    using Cc = std::complex<Tt>;
    const size_t n = S->u1.size();
    std::vector<Cc> bl[4], ab[4];
    for (int f = 0; f < 4; f++) {
      bl[f].resize(n);
      ab[f].resize(n);
      for (size_t i = 0; i < n; i++) {
        bl[f][i] = Cc(Tt(below[2 * (f * n + i)]), Tt(below[2 * (f * n + i) + 1]));
        ab[f][i] = Cc(Tt(above[2 * (f * n + i)]), Tt(above[2 * (f * n + i) + 1]));
      }
    }
    S->time_step_adjoint(bl, ab);
  });
}

// IMEXRK::SetBackground(u1,u2,u3,b) (IMEXRK.h:334-352): the frozen base of
// TimeStepLinear, given as modal fields in the reference layout.
void sfo_set_base(void* hv, const double* u1, const double* u2, const double* u3, const double* bb) {
  auto* h = (Handle*)hv;
  DISPATCH(h, {
    using Tt = decltype(S->Ri);
    using Cc = std::complex<Tt>;
    std::vector<Cc> t(S->u1.size());
    auto load = [&](const double* src, std::vector<Tt>& dst) {
      for (size_t i = 0; i < t.size(); i++) t[i] = Cc(Tt(src[2 * i]), Tt(src[2 * i + 1]));
      S->to_nodal(t, dst);
    };
    load(u1, S->U1b);
    if (S->dim3) load(u2, S->U2b); else std::fill(S->U2b.begin(), S->U2b.end(), Tt(0));
    load(u3, S->U3b);
    load(bb, S->Bb);
  });
}

void sfo_energy(void* hv, double* ke, double* pe) {
  auto* h = (Handle*)hv;
  DISPATCH(h, { *ke = double(S->KE()); *pe = double(S->PE()); });
}

void sfo_dissipation(void* hv, double* eps, double* chi) {
  auto* h = (Handle*)hv;
  DISPATCH(h, {
    decltype(S->Ri) e, c;
    S->dissipation(e, c);
    *eps = double(e);
    *chi = double(c);
  });
}

// modal fields -> nodal and back (Field.h:734-769, 965-994) on a single
// field given in the reference layout; used by the FFT pinning tests.
void sfo_to_nodal(void* hv, const double* modal_ri, double* nodal) {
  auto* h = (Handle*)hv;
  DISPATCH(h, {
    using Tt = decltype(S->Ri);
    std::vector<std::complex<Tt>> t(S->u1.size());
    for (size_t i = 0; i < t.size(); i++) t[i] = std::complex<Tt>(Tt(modal_ri[2 * i]), Tt(modal_ri[2 * i + 1]));
    std::vector<Tt> o(S->U1.size());
    S->to_nodal(t, o);
    for (size_t i = 0; i < o.size(); i++) nodal[i] = double(o[i]);
  });
}
void sfo_to_modal(void* hv, const double* nodal, double* modal_ri) {
  auto* h = (Handle*)hv;
  DISPATCH(h, {
    using Tt = decltype(S->Ri);
    std::vector<Tt> t(S->U1.size());
    for (size_t i = 0; i < t.size(); i++) t[i] = Tt(nodal[i]);
    std::vector<std::complex<Tt>> o(S->u1.size());
    S->to_modal(t, o);
    for (size_t i = 0; i < o.size(); i++) { modal_ri[2 * i] = double(o[i].real()); modal_ri[2 * i + 1] = double(o[i].imag()); }
  });
}

// Seeded initial condition (no counterpart in the reference, whose random
// generators are unseeded, Field.h:1029-1031): Gaussian modal coefficients
// (splitmix64 + Box-Muller, FP64) on kept modes n1 < nx_lo and, in 3D,
// |ky| < ny_lo, times amp*exp(-z^2) at each field's staggered level;
// Hermitian on n1 = 0. fields_mask bit f perturbs field f (0 u1,1 u2,2 u3,3 b).
// Writes the four fields in the reference layout (p is left zero), after
// StateVector::EnforceBCs (StateVector.h:415-421).
void sfo_make_ic(void* hv, uint64_t seed, double amp, int nx_lo, int ny_lo, int fields_mask) {
  auto* h = (Handle*)hv;
  DISPATCH(h, {
    using Tt = decltype(S->Ri);
    using Cc = std::complex<Tt>;
    uint64_t st = seed;
    int N1 = S->N1, N2 = S->N2, N3 = S->N3, M1 = S->M1;
    auto kyint = Solver<double>::kint(N2);
    for (int f = 0; f < 4; f++) {
      auto* F = field_ptr(S, f);
      std::fill(F->begin(), F->end(), Cc(0));
      if (!(fields_mask & (1 << f))) continue;
      if (f == 1 && !S->dim3) continue;
      bool dir = (f == 2);
      std::vector<double> env(N3);
      for (int j = 0; j < N3; j++) {
        double zz = dir ? double(S->z[j]) : double(S->zf[j]);
        env[j] = amp * std::exp(-zz * zz);
      }
      for (int n2 : S->keptY) {
        int kyv = S->dim3 ? int(kyint[n2]) : 0;
        if (std::abs(kyv) >= ny_lo && S->dim3) continue;
        for (int n1 = 0; n1 < std::min(nx_lo, S->K1); n1++) {
          if (n1 == 0 && kyv < 0) continue;  // filled by symmetry below
          for (int j = 0; j < N3; j++) {
            double g0, g1;
            gauss2(st, g0, g1);
            if (n1 == 0 && kyv == 0) g1 = 0.0;
            (*F)[S->midx(n1, n2) + j] = Cc(Tt(env[j] * g0), Tt(env[j] * g1));
          }
        }
      }
      if (S->dim3) {  // Hermitian n1 = 0 column: X(0,-ky) = conj X(0,ky)
        for (int n2 : S->keptY) {
          int kyv = int(kyint[n2]);
          if (kyv <= 0) continue;
          int m2 = N2 - n2;
          for (int j = 0; j < N3; j++) (*F)[S->midx(0, m2) + j] = std::conj((*F)[S->midx(0, n2) + j]);
        }
      }
      (void)N1; (void)M1;
      // EnforceBCs
      for (int n2 = 0; n2 < N2; n2++)
        for (int n1 = 0; n1 < S->M1; n1++) {
          size_t o = S->midx(n1, n2);
          if (dir) {
            (*F)[o + 0] = (*F)[o + 1] = (*F)[o + 2] = Cc(0);
            (*F)[o + N3 - 1] = (*F)[o + N3 - 2] = Cc(0);
          } else {
            (*F)[o + 0] = (*F)[o + 1];
            (*F)[o + N3 - 1] = (*F)[o + N3 - 2];
          }
        }
    }
    std::fill(S->p.begin(), S->p.end(), Cc(0));
  });
}

}  // extern "C"
