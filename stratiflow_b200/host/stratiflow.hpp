// C++ front end of stratiflow_b200 over its C-ABI: the reference's solver
// and driver classes (IMEXRK, StateVector/ExtendedStateVector, NewtonKrylov,
// PseudoArclengthContinuation, FindPeriodic) with their device state on the
// GPU and FP64 Krylov numerics on the host.
//
// A state here is a multiple-shooting vector: M segments x_0..x_{M-1} of
// one trajectory (M = 1 is the reference's StateVector) plus one scalar
// parameter p (the reference's ExtendedStateVector::p: Ri in continuation, the
// period T in the periodic-orbit search). Every evaluation of the evolution
// map advances all M segments as the M runs of one batched solver, so one
// Jacobian action of GMRES costs one batched integration over T/M.
#pragma once

#include <algorithm>
#include <chrono>
#include <cstdio>
#include <cstdlib>
#include <cmath>
#include <complex>
#include <functional>
#include <memory>
#include <random>
#include <stdexcept>
#include <string>
#include <vector>

#include "stratiflow_b200.h"

namespace stratiflow {

// STRATIFLOW_VERBOSE=1 prints the Krylov and Newton progress to stderr, as
// the reference prints its Newton steps (NewtonKrylov.h:47)
inline bool verbose() {
  static const bool v = [] {
    const char* e = std::getenv("STRATIFLOW_VERBOSE");
    return e && *e && *e != '0';
  }();
  return v;
}

inline void check(int rc) {
  if (rc != SF_OK) throw std::runtime_error(std::string("stratiflow_b200: ") + sf_last_error());
}

// gridParams + flowParams (Parameters.h:6-43) and the background of the run
struct Params {
  int N1 = 256, N2 = 1, N3 = 256;
  double L1 = 2 * 3.141592653589793 / 0.44, L2 = 3.141592653589793 / 0.44, L3 = 10.0;
  double Re = 1000, Pr = 1, Ri = 0.12, dt = 0.01;
  int background = 0;   // 0: B = tanh z, 1: B = tanh 3z, 2: B = z (the reference)
};

// Field.cpp:21-31 in FP64
inline std::vector<double> vertical_points_fractional(double L, int N) {
  std::vector<double> z(N, 0.0), zf(N, 0.0);
  const double step = 2.0 / (N - 2);
  for (int i = 0; i < N - 1; i++) {
    double x = (i == N - 2) ? 1.0 : -1.0 + i * step;
    z[i + 1] = L * (2.0 * std::pow(x, 7) + x) / 3.0;
  }
  double off = (z[1] + z[2]) / 2;
  for (int i = 1; i < N; i++) z[i] *= -L / off;
  for (int i = 1; i <= N - 2; i++) zf[i] = 0.5 * (z[i] + z[i + 1]);
  zf[0] = 2 * zf[1] - zf[2];
  zf[N - 1] = 2 * zf[N - 2] - zf[N - 3];
  return zf;
}

// U_ = tanh z set as Nodal1D::SetValue does (Field.h:661-682), and dB/dz
inline void background_profiles(const Params& p, std::vector<double>& U, std::vector<double>& dB) {
  const int N = p.N3;
  auto zf = vertical_points_fractional(p.L3, N);
  U.resize(N);
  dB.resize(N);
  for (int j = 0; j < N; j++) {
    U[j] = std::tanh(zf[j]);
    double c1 = std::cosh(zf[j]), c3 = std::cosh(3 * zf[j]);
    dB[j] = p.background == 0 ? 1.0 / (c1 * c1) : (p.background == 1 ? 3.0 / (c3 * c3) : 1.0);
  }
  U[1] = U[2]; U[0] = U[1]; U[N - 2] = U[N - 3]; U[N - 1] = U[N - 2];
}

// IMEXRK (IMEXRK.h:31-670) for a batch of runs
class Solver {
 public:
  Solver(const Params& p, int nrun) : p_(p), nrun_(nrun), ri_(nrun, -1.0), dt_(p.dt) {
    sf_grid g{p.N1, p.N2, p.N3, nrun};
    sf_flow f{p.L1, p.L2, p.L3, p.Re, p.Pr};
    check(sf_create(&g, &f, p.dt, 0, &h_));
    std::vector<double> U, dB;
    background_profiles(p, U, dB);
    for (int r = 0; r < nrun; r++) {
      check(sf_set_background(h_, r, U.data(), dB.data()));
      set_ri(r, p.Ri);
    }
  }
  ~Solver() { sf_destroy(h_); }
  Solver(const Solver&) = delete;
  Solver& operator=(const Solver&) = delete;
  void set_dt(double dt) {
    if (std::fabs(dt - dt_) > 1e-14 * dt) {
      check(sf_set_dt(h_, dt));
      dt_ = dt;
    }
  }
  void set_ri(int run, double ri) {
    if (ri != ri_[run]) {
      check(sf_set_ri(h_, run, ri));
      ri_[run] = ri;
    }
  }
  sf_solver* h() const { return h_; }
  int nrun() const { return nrun_; }
  const Params& params() const { return p_; }
  double dt() const { return dt_; }

 private:
  Params p_;
  int nrun_;
  std::vector<double> ri_;
  double dt_;
  sf_solver* h_ = nullptr;
};

// M device states of one grid
class Store {
 public:
  Store(Solver& like, int n) : n_(n) { check(sf_vecs_create(like.h(), n, &v_)); }
  ~Store() { sf_vecs_destroy(v_); }
  Store(const Store&) = delete;
  Store& operator=(const Store&) = delete;
  sf_vecs* v() const { return v_; }
  int n() const { return n_; }

 private:
  int n_;
  sf_vecs* v_ = nullptr;
};

// The evolution context: parameters, the segment count M and the batched
// solver (the reference's static StateVector::solver, StateVector.h:546).
struct Context {
  Params p;
  int M = 1;
  std::unique_ptr<Solver> solver;   // nrun = M
  std::unique_ptr<Solver> tangent;  // nrun = 2M: M bases + M tangent-linear runs
  long long evolutions = 0;         // batched integrations performed
  double evolve_seconds = 0;
  Context(const Params& prm, int m) : p(prm), M(m), solver(new Solver(prm, m)) {}
  Solver& tangent_solver() {
    if (!tangent) {
      tangent.reset(new Solver(p, 2 * M));
      check(sf_set_tangent(tangent->h(), M));
    }
    return *tangent;
  }
  // one-run solvers for segment-wise evolutions: the nonlinear map, and
  // TimeStepLinear about a frozen base (LinearEvolve, StateVector.cpp:107-156)
  std::unique_ptr<Solver> single, linear;
  Solver& single_solver() {
    if (!single) single.reset(new Solver(p, 1));
    return *single;
  }
  Solver& linear_solver() {
    if (!linear) linear.reset(new Solver(p, 1));
    return *linear;
  }
  // one base and s tangent-linear runs (block Krylov methods, M = 1)
  std::unique_ptr<Solver> block_tangent;
  Solver& block_tangent_solver(int s) {
    if (!block_tangent || block_tangent->nrun() != s + 1) {
      block_tangent.reset(new Solver(p, s + 1));
      check(sf_set_tangent(block_tangent->h(), 1));
    }
    return *block_tangent;
  }
};

// Multiple-shooting state (StateVector for M = 1, plus the scalar of
// ExtendedStateVector, ExtendedStateVector.h:6-96)
class Vec {
 public:
  explicit Vec(Context& c) : c_(&c), s_(new Store(*c.solver, c.M)) {}
  Vec(const Vec& o) : p(o.p), q(o.q), c_(o.c_), s_(new Store(*o.c_->solver, o.c_->M)) {
    check(sf_vecs_copy_range(o));
  }
  Vec& operator=(const Vec& o) {
    if (this != &o) {
      check(sf_vecs_copy_range(o));
      p = o.p;
      q = o.q;
    }
    return *this;
  }
  double p = 0.0;
  double q = 0.0;   // a second scalar unknown (the Hopf frequency theta, HopfBifurcation.h:12-14); 0 elsewhere

  int M() const { return c_->M; }
  sf_vecs* v() const { return s_->v(); }
  Context& ctx() const { return *c_; }

  // MulAdd (StateVector.h:67-78, ExtendedStateVector.h:28-32), then EnforceBCs
  void MulAdd(double a, const Vec& x) {
    check(sf_vecs_axpy(v(), 0, a, x.v(), 0, M()));
    p += a * x.p;
    q += a * x.q;
    EnforceBCs();
  }
  Vec& operator+=(const Vec& x) { MulAdd(1.0, x); return *this; }
  Vec& operator-=(const Vec& x) { MulAdd(-1.0, x); return *this; }
  Vec& operator*=(double a) {
    check(sf_vecs_scale(v(), 0, a, M()));
    p *= a;
    q *= a;
    return *this;
  }
  // StateVector::Dot summed over the segments + p p' (ExtendedStateVector.h:12-15)
  double Dot(const Vec& o, bool with_p = true) const {
    double d = 0;
    check(sf_vecs_dot_sum(v(), 0, o.v(), 0, M(), c_->p.Ri, &d));
    return d + (with_p ? p * o.p + q * o.q : 0.0);
  }
  double Norm2() const { return Dot(*this); }
  double Norm() const { return std::sqrt(Norm2()); }
  void Zero() {
    check(sf_vecs_scale(v(), 0, 0.0, M()));
    p = 0;
    q = 0;
  }
  void EnforceBCs() { check(sf_vecs_enforce_bcs(v(), 0, M())); }
  // RemovePhaseShift of segment 0, the same shift applied to every segment
  double RemovePhaseShift() {
    double s = 0;
    check(sf_vecs_phase_shift(v(), 0, 0, &s));
    for (int i = 1; i < M(); i++) check(sf_vecs_phase_shift(v(), i, 1, &s));
    return s;
  }
  void RemoveAverage(int field) {
    for (int i = 0; i < M(); i++) check(sf_vecs_remove_average(v(), i, field, c_->p.L3));
  }
  void set_segment_host(int i, const float* kept) { check(sf_vecs_set_host(v(), i, kept)); }
  void get_segment_host(int i, float* kept) const { check(sf_vecs_get_host(v(), i, kept)); }

 private:
  int sf_vecs_copy_range(const Vec& o) {
    for (int i = 0; i < M(); i++) {
      int rc = sf_vecs_copy(v(), i, o.v(), i);
      if (rc) return rc;
    }
    return SF_OK;
  }
  Context* c_;
  std::unique_ptr<Store> s_;
};

// Evolve every segment of x over tau at the given Ri (FullEvolve with a fixed
// step, StateVector.cpp:3-84, 85-105): p is zeroed, the state projected
// (RemoveDivergence(0)), nsteps = ceil(tau/dt) equal steps, EnforceBCs on
// the result. If `extra` is given it receives the state one more step later
// (for the time derivative of the flow map).
inline void Evolve(const Vec& x, double tau, double Ri, Vec& out, Vec* extra = nullptr) {
  Context& c = x.ctx();
  auto t0 = std::chrono::steady_clock::now();
  const int nsteps = std::max(1, (int)std::ceil(tau / c.p.dt - 1e-9));
  c.solver->set_dt(tau / nsteps);
  for (int r = 0; r < c.M; r++) c.solver->set_ri(r, Ri);
  const double p = x.p;
  if (&out != &x) out = x;
  // p = 0 at the start of every integration: the map depends on u1..b only
  check(sf_vecs_zero_pressure(out.v(), 0, c.M));
  check(sf_vecs_to_run(out.v(), 0, c.solver->h(), 0, c.M));
  check(sf_prepare(c.solver->h()));
  check(sf_step(c.solver->h(), nsteps));
  check(sf_vecs_from_run(out.v(), 0, c.solver->h(), 0, c.M));
  if (extra) {
    check(sf_step(c.solver->h(), 1));
    check(sf_vecs_from_run(extra->v(), 0, c.solver->h(), 0, c.M));
    extra->EnforceBCs();
    extra->p = p;
  }
  out.EnforceBCs();
  out.p = p;
  check(sf_vecs_synchronize(out.v()));
  c.evolutions += 1;
  c.evolve_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// The derivative of Evolve at x applied to dx, exactly (to FP32 rounding):
// the bases x and the perturbations dx advance together in one batch, each
// perturbation by TimeStepLinear (IMEXRK.h:334-352) about its base's state
// at the same RK stage. The pressure of both is zeroed and both are
// projected first, as Evolve does; out.p = dx.p.
inline void EvolveTangent(const Vec& x, const Vec& dx, double tau, double Ri, Vec& out) {
  Context& c = x.ctx();
  auto t0 = std::chrono::steady_clock::now();
  Solver& s = c.tangent_solver();
  const int nsteps = std::max(1, (int)std::ceil(tau / c.p.dt - 1e-9));
  s.set_dt(tau / nsteps);
  for (int r = 0; r < 2 * c.M; r++) s.set_ri(r, Ri);
  const double p = dx.p;
  Vec b(x);
  if (&out != &dx) out = dx;
  check(sf_vecs_zero_pressure(b.v(), 0, c.M));
  check(sf_vecs_zero_pressure(out.v(), 0, c.M));
  check(sf_vecs_to_run(b.v(), 0, s.h(), 0, c.M));
  check(sf_vecs_to_run(out.v(), 0, s.h(), c.M, c.M));
  check(sf_prepare(s.h()));
  check(sf_step(s.h(), nsteps));
  check(sf_vecs_from_run(out.v(), 0, s.h(), c.M, c.M));
  out.EnforceBCs();
  out.p = p;
  check(sf_vecs_synchronize(out.v()));
  c.evolutions += 1;
  c.evolve_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// ------------------------------------------ dense FP64 helpers ----------
// min |b - A y| for A m x n (row-major, m >= n) by Householder QR; returns
// |b - A y| and y (zero where R's diagonal vanishes)
inline double lsq_householder(std::vector<double> A, int m, int n, std::vector<double> b, std::vector<double>& y) {
  for (int k = 0; k < n; k++) {
    double nrm = 0;
    for (int i = k; i < m; i++) nrm += A[(size_t)i * n + k] * A[(size_t)i * n + k];
    nrm = std::sqrt(nrm);
    if (nrm == 0) continue;
    const double a0 = A[(size_t)k * n + k];
    const double alpha = a0 > 0 ? -nrm : nrm;
    std::vector<double> v(m - k);
    for (int i = k; i < m; i++) v[i - k] = A[(size_t)i * n + k];
    v[0] -= alpha;
    double vn = 0;
    for (double t : v) vn += t * t;
    if (vn == 0) continue;
    for (int j = k; j < n; j++) {
      double d = 0;
      for (int i = k; i < m; i++) d += v[i - k] * A[(size_t)i * n + j];
      d = 2 * d / vn;
      for (int i = k; i < m; i++) A[(size_t)i * n + j] -= d * v[i - k];
    }
    double d = 0;
    for (int i = k; i < m; i++) d += v[i - k] * b[i];
    d = 2 * d / vn;
    for (int i = k; i < m; i++) b[i] -= d * v[i - k];
  }
  y.assign(n, 0.0);
  double rmax = 0;
  for (int k = 0; k < n; k++) rmax = std::max(rmax, std::fabs(A[(size_t)k * n + k]));
  for (int k = n - 1; k >= 0; k--) {
    double t = b[k];
    for (int j = k + 1; j < n; j++) t -= A[(size_t)k * n + j] * y[j];
    const double rk = A[(size_t)k * n + k];
    y[k] = std::fabs(rk) > 1e-13 * rmax ? t / rk : 0.0;
  }
  double r = 0;
  for (int i = n; i < m; i++) r += b[i] * b[i];
  return std::sqrt(r);
}

// lower Cholesky factor of the k x k SPD matrix G (row-major); false if G is
// not numerically positive definite
inline bool cholesky(const std::vector<double>& G, int k, std::vector<double>& L) {
  L.assign((size_t)k * k, 0.0);
  double dmax = 0;
  for (int i = 0; i < k; i++) dmax = std::max(dmax, G[(size_t)i * k + i]);
  for (int j = 0; j < k; j++) {
    double d = G[(size_t)j * k + j];
    for (int t = 0; t < j; t++) d -= L[(size_t)j * k + t] * L[(size_t)j * k + t];
    if (!(d > 1e-24 * dmax)) return false;
    L[(size_t)j * k + j] = std::sqrt(d);
    for (int i = j + 1; i < k; i++) {
      double v = G[(size_t)i * k + j];
      for (int t = 0; t < j; t++) v -= L[(size_t)i * k + t] * L[(size_t)j * k + t];
      L[(size_t)i * k + j] = v / L[(size_t)j * k + j];
    }
  }
  return true;
}

// FullEvolve's time loop (StateVector.cpp:3-84) on a solver's device state:
// RemoveDivergence(0), then every `interval` steps the CFL number (largest
// over the runs, IMEXRK::CFL, IMEXRK.h:355-373) resets dt to reach
// target_cfl, and when fewer than `interval` steps remain dt is shortened so
// that the run ends exactly at T. stats: steps, t, last dt, CFL checks, seconds.
inline void FullEvolveAdaptive(sf_solver* h, int nrun, double T, double target_cfl, int interval, double* stats) {
  auto t0 = std::chrono::steady_clock::now();
  double dt = 0;
  check(sf_get_dt(h, &dt));
  check(sf_prepare(h));
  double t = 0;
  long long steps = 0;
  int checks = 0;
  while (t + 1e-4 < T) {
    double cfl = 0;
    for (int r = 0; r < nrun; r++) {
      double c = 0;
      check(sf_cfl(h, r, &c));
      cfl = std::max(cfl, c);
    }
    checks++;
    if (cfl > 0) dt *= target_cfl / cfl;
    const double remaining = T - t;
    const int rs = (int)(remaining / dt) + 1;
    if (rs < interval) dt = remaining / rs;   // finish exactly at T
    check(sf_set_dt(h, dt));
    int k = std::min(interval, std::max(1, (int)std::ceil((T - 1e-4 - t) / dt)));
    check(sf_step(h, k));
    t += k * dt;
    steps += k;
  }
  check(sf_synchronize(h));
  if (stats) {
    stats[0] = (double)steps;
    stats[1] = t;
    stats[2] = dt;
    stats[3] = checks;
    stats[4] = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
  }
}

// ------------------------------------------------------------ FP64 SVD ----
// one-sided Jacobi SVD of an m x n matrix (m >= n), row-major A:
// A = U diag(S) V^T, U m x n, V n x n
inline void svd(std::vector<double> A, int m, int n, std::vector<double>& U, std::vector<double>& S,
                std::vector<double>& V) {
  V.assign((size_t)n * n, 0.0);
  for (int i = 0; i < n; i++) V[(size_t)i * n + i] = 1.0;
  for (int sweep = 0; sweep < 60; sweep++) {
    double off = 0;
    for (int p = 0; p < n - 1; p++)
      for (int q = p + 1; q < n; q++) {
        double a = 0, b = 0, d = 0;
        for (int i = 0; i < m; i++) {
          double x = A[(size_t)i * n + p], y = A[(size_t)i * n + q];
          a += x * x; b += y * y; d += x * y;
        }
        if (std::fabs(d) <= 1e-300 || std::fabs(d) <= 1e-15 * std::sqrt(a * b)) continue;
        off = std::max(off, std::fabs(d) / std::sqrt(a * b));
        double zeta = (b - a) / (2 * d);
        double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1 + zeta * zeta));
        double cs = 1 / std::sqrt(1 + t * t), sn = cs * t;
        for (int i = 0; i < m; i++) {
          double x = A[(size_t)i * n + p], y = A[(size_t)i * n + q];
          A[(size_t)i * n + p] = cs * x - sn * y;
          A[(size_t)i * n + q] = sn * x + cs * y;
        }
        for (int i = 0; i < n; i++) {
          double x = V[(size_t)i * n + p], y = V[(size_t)i * n + q];
          V[(size_t)i * n + p] = cs * x - sn * y;
          V[(size_t)i * n + q] = sn * x + cs * y;
        }
      }
    if (off < 1e-15) break;
  }
  S.assign(n, 0.0);
  U.assign((size_t)m * n, 0.0);
  for (int j = 0; j < n; j++) {
    double s = 0;
    for (int i = 0; i < m; i++) s += A[(size_t)i * n + j] * A[(size_t)i * n + j];
    s = std::sqrt(s);
    S[j] = s;
    for (int i = 0; i < m; i++) U[(size_t)i * n + j] = s > 0 ? A[(size_t)i * n + j] / s : 0.0;
  }
}

// ------------------------------------------------------- Newton-Krylov ----
struct NKOptions {
  int max_newton = 20;
  int krylov = 80;            // GMRES basis size (K, NewtonKrylov.h:237)
  double target = 1e-6;       // relative residual |F(x)| / |x|
  double gmres_tol = 0.01;    // relative GMRES residual (NewtonKrylov.h:96)
  double Delta = 100;         // initial trust region, relative to |x| (NewtonKrylov.h:29)
  double fd_eps = 3e-4;       // finite-difference step relative to |x|
  bool tangent = true;        // Jacobian actions by the tangent-linear batch, else by
                              // finite differences (NewtonKrylov.h:218-235)
  bool precondition = true;   // block solvers: the mean-flow preconditioner
  bool relative = false;      // block fixed point: the x shift as an unknown with a phase condition
};

struct NKStats {
  int newton_iterations = 0;
  int krylov_vectors = 0;       // Jacobian actions
  long long evolutions = 0;     // batched integrations
  double seconds = 0;
  double evolve_seconds = 0;
  double residual = 0;
  bool converged = false;
  std::vector<double> residuals;
  std::vector<double> gmres_residuals;   // relative GMRES residual of each Newton step
  std::vector<int> gmres_vectors;        // Jacobian actions of each Newton step
};

// NewtonKrylov<VectorType> (NewtonKrylov.h:1-241) with FP64 Gram-Schmidt,
// Hessenberg and least squares, EvalDerivative by finite differences, and
// the hookstep trust region whose acceptance test the reference leaves
// switched off (NewtonKrylov.h:48, 69): a step is taken only if it lowers
// the residual, otherwise Delta is halved and the constrained least-squares
// problem is solved again in the same Krylov basis.
class NewtonKrylov {
 public:
  explicit NewtonKrylov(const NKOptions& o) : opt(o) {}
  virtual ~NewtonKrylov() = default;
  NKOptions opt;

  virtual Vec EvalFunction(const Vec& at) = 0;
  virtual void EnforceConstraints(Vec& at) { (void)at; }
  // called after F has been evaluated at each accepted Newton iterate
  virtual void AtIterate(const Vec& x, const Vec& F) { (void)x; (void)F; }
  // J * dir about the current Newton iterate (x0, F0 = F(x0))
  virtual Vec EvalDerivative(const Vec& dir) {
    const double eps = opt.fd_eps * x0_->Norm() / std::max(dir.Norm(), 1e-300);
    Vec t(*x0_);
    t.MulAdd(eps, dir);
    Vec r = EvalFunction(t);
    r.MulAdd(-1.0, *F0_);
    r *= 1.0 / eps;
    return r;
  }

  NKStats Run(Vec& x) {
    NKStats st;
    auto t0 = std::chrono::steady_clock::now();
    Context& c = x.ctx();
    const long long ev0 = c.evolutions;
    const double es0 = c.evolve_seconds;
    std::unique_ptr<Vec> F(new Vec(EvalFunction(x)));
    double xn = std::max(x.Norm(), 1e-300);
    double res = F->Norm() / xn;
    double Delta = opt.Delta * xn;
    st.residuals.push_back(res);
    for (int it = 0; it < opt.max_newton && res >= opt.target; it++) {
      x0_ = &x;
      F0_ = F.get();
      AtIterate(x, *F);
      const int used = GMRES(*F);
      st.krylov_vectors += used;
      st.gmres_vectors.push_back(used);
      st.gmres_residuals.push_back(n_ > 0 ? ResidualQR() : 1.0);
      bool accepted = false;
      for (int attempt = 0; attempt < 8 && !accepted; attempt++) {
        double zn = 0;
        Vec dx = Hookstep(x, Delta, zn);
        Vec xt(x);
        xt.MulAdd(1.0, dx);
        EnforceConstraints(xt);
        EnforceConstraints(xt);
        EnforceConstraints(xt);
        std::unique_ptr<Vec> Ft(new Vec(EvalFunction(xt)));
        const double rt = Ft->Norm() / std::max(xt.Norm(), 1e-300);
        if (rt < res) {
          x = xt;
          F = std::move(Ft);
          if (zn >= 0.9 * Delta && rt < 0.5 * res) Delta *= 2;   // the step hit the region and worked
          res = rt;
          accepted = true;
        } else {
          Delta = 0.5 * std::min(Delta, zn);
        }
      }
      basis_.clear();
      st.newton_iterations++;
      st.residuals.push_back(res);
      if (!accepted) break;
    }
    st.residual = res;
    st.converged = res < opt.target;
    st.evolutions = c.evolutions - ev0;
    st.evolve_seconds = c.evolve_seconds - es0;
    st.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    x0_ = nullptr;
    F0_ = nullptr;
    return st;
  }

 protected:
  const Vec* x0_ = nullptr;
  const Vec* F0_ = nullptr;
  std::vector<std::unique_ptr<Vec>> basis_;
  std::vector<double> H_;   // (K) x (K-1), row-major with stride K-1
  double beta_ = 0;
  int n_ = 0;               // columns of the Hessenberg block in use

  // Arnoldi with modified Gram-Schmidt (NewtonKrylov.h:150-177) for A = -J
  // until the unconstrained least-squares residual is below gmres_tol or the
  // basis is full; keeps the basis for the hooksteps. Returns the number of
  // Jacobian actions.
  int GMRES(const Vec& rhs) {
    const int K = opt.krylov;
    basis_.clear();
    H_.assign((size_t)K * (K - 1), 0.0);
    basis_.emplace_back(new Vec(rhs));
    basis_[0]->EnforceBCs();
    beta_ = basis_[0]->Norm();
    n_ = 0;
    if (!(beta_ > 0)) return 0;
    *basis_[0] *= 1.0 / beta_;
    int used = 0;
    for (int k = 1; k < K; k++) {
      basis_.emplace_back(new Vec(EvalDerivative(*basis_[k - 1])));
      *basis_[k] *= -1.0;   // factor of -1 for the Newton iteration
      used++;
      for (int j = 0; j < k; j++) {
        const double h = basis_[j]->Dot(*basis_[k]);
        H_[(size_t)j * (K - 1) + (k - 1)] = h;
        basis_[k]->MulAdd(-h, *basis_[j]);
      }
      const double hn = basis_[k]->Norm();
      H_[(size_t)k * (K - 1) + (k - 1)] = hn;
      if (hn > 0) *basis_[k] *= 1.0 / hn;
      basis_[k]->EnforceBCs();
      n_ = k;
      const double rq = ResidualQR();
      if (verbose() && (k % 10 == 0)) std::fprintf(stderr, "GMRES: %d vectors, relative residual %.3e\n", k, rq);
      if (rq < opt.gmres_tol || !(hn > 1e-14 * beta_)) break;
    }
    return used;
  }

  // relative residual of the unconstrained least-squares problem (Householder QR)
  double ResidualQR() {
    const int K = opt.krylov, m = n_ + 1, n = n_;
    std::vector<double> A((size_t)m * n), b(m, 0.0), y;
    for (int i = 0; i < m; i++)
      for (int j = 0; j < n; j++) A[(size_t)i * n + j] = H_[(size_t)i * (K - 1) + j];
    b[0] = beta_;
    return lsq_householder(A, m, n, b, y) / beta_;
  }

  // min |beta e_0 - H y| with |y| <= Delta through the SVD of H (Chandler &
  // Kerswell 2013, as NewtonKrylov.h:179-216); returns the relative residual
  double LeastSquares(double Delta, double& znorm) {
    const int K = opt.krylov, m = n_ + 1, n = n_;
    std::vector<double> sub((size_t)m * n), U, S, V;
    for (int i = 0; i < m; i++)
      for (int j = 0; j < n; j++) sub[(size_t)i * n + j] = H_[(size_t)i * (K - 1) + j];
    svd(sub, m, n, U, S, V);
    std::vector<double> pv(n), z(n);
    for (int j = 0; j < n; j++) pv[j] = U[j] * beta_;   // U^T (beta e_0)
    auto zfor = [&](double mu) {
      double s = 0;
      for (int j = 0; j < n; j++) {
        const double d = S[j];
        z[j] = (d * d + mu) > 0 ? pv[j] * d / (d * d + mu) : 0.0;
        s += z[j] * z[j];
      }
      return std::sqrt(s);
    };
    double mu = 0;
    if (zfor(0) > Delta) {
      double lo = 0, hi = 1e-12;
      while (zfor(hi) > Delta) hi *= 4;
      for (int b = 0; b < 80; b++) {
        const double mid = 0.5 * (lo + hi);
        (zfor(mid) > Delta ? lo : hi) = mid;
      }
      mu = hi;
    }
    znorm = zfor(mu);
    y_.assign(n, 0.0);
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) y_[i] += V[(size_t)i * n + j] * z[j];
    double r2 = 0;
    for (int i = 0; i < m; i++) {
      double s = (i == 0) ? -beta_ : 0.0;
      for (int j = 0; j < n; j++) s += sub[(size_t)i * n + j] * y_[j];
      r2 += s * s;
    }
    return std::sqrt(r2) / beta_;
  }

  Vec Hookstep(const Vec& like, double Delta, double& znorm) {
    Vec dx(like);
    dx.Zero();
    if (n_ == 0) {
      znorm = 0;
      return dx;
    }
    LeastSquares(Delta, znorm);
    for (int k = 0; k < n_; k++) dx.MulAdd(y_[k], *basis_[k]);
    return dx;
  }

  std::vector<double> y_;
};

// ----------------------------------------------- block Krylov vectors ----
// n device vectors of one state (M = 1) plus the scalar of each
// (ExtendedStateVector::p, ExtendedStateVector.h:6-96)
class Block {
 public:
  Block(Context& c, int n) : n_(n), p(n, 0.0) { check(sf_vecs_create(c.solver->h(), n, &v_)); }
  ~Block() { sf_vecs_destroy(v_); }
  Block(const Block&) = delete;
  Block& operator=(const Block&) = delete;
  sf_vecs* v() const { return v_; }
  int n() const { return n_; }

 private:
  int n_;
  sf_vecs* v_ = nullptr;

 public:
  std::vector<double> p;
};

// G[i][k] = Dot(A[a+i], B[b+k]) + p products (ExtendedStateVector::Dot)
inline std::vector<double> block_gram(const Block& A, int a, int na, const Block& B, int b, int nb, double Ri) {
  std::vector<double> G((size_t)na * nb);
  check(sf_vecs_gram(A.v(), a, na, B.v(), b, nb, Ri, G.data()));
  for (int i = 0; i < na; i++)
    for (int k = 0; k < nb; k++) G[(size_t)i * nb + k] += A.p[a + i] * B.p[b + k];
  return G;
}

// B[b+k] += alpha sum_i C[i][k] A[a+i] (scalars too)
inline void block_update(Block& B, int b, int nb, double alpha, const Block& A, int a, int na,
                         const std::vector<double>& C) {
  check(sf_vecs_update(B.v(), b, nb, alpha, A.v(), a, na, C.data()));
  for (int k = 0; k < nb; k++) {
    double t = 0;
    for (int i = 0; i < na; i++) t += C[(size_t)i * nb + k] * A.p[a + i];
    B.p[b + k] += alpha * t;
  }
}

// dst[b..b+k) = src[a..a+k) L^-T with G = L L^T the Gram matrix of the
// source (FP64); false if it is rank deficient. R = L^T.
inline bool cholqr(const Block& src, int a, Block& dst, int b, int k, double Ri, std::vector<double>& R) {
  std::vector<double> G = block_gram(src, a, k, src, a, k, Ri), L;
  if (!cholesky(G, k, L)) return false;
  std::vector<double> C((size_t)k * k, 0.0);   // C = L^-T, column by column
  for (int j = 0; j < k; j++)
    for (int i = k - 1; i >= 0; i--) {
      double t = (i == j) ? 1.0 : 0.0;
      for (int m = i + 1; m < k; m++) t -= L[(size_t)m * k + i] * C[(size_t)m * k + j];
      C[(size_t)i * k + j] = t / L[(size_t)i * k + i];
    }
  check(sf_vecs_scale(dst.v(), b, 0.0, k));
  for (int i = 0; i < k; i++) dst.p[b + i] = 0.0;
  block_update(dst, b, k, 1.0, src, a, k, C);
  R.assign((size_t)k * k, 0.0);
  for (int i = 0; i < k; i++)
    for (int j = 0; j < k; j++) R[(size_t)i * k + j] = L[(size_t)j * k + i];
  return true;
}

// two passes of Cholesky QR: dst[b..b+k) orthonormal, src = dst R (R = R2 R1);
// src is overwritten
inline bool cholqr2(Block& src, int a, Block& dst, int b, int k, double Ri, std::vector<double>& R) {
  std::vector<double> R1, R2;
  if (!cholqr(src, a, dst, b, k, Ri, R1)) return false;
  if (!cholqr(dst, b, src, a, k, Ri, R2)) return false;
  for (int i = 0; i < k; i++) {
    check(sf_vecs_copy(dst.v(), b + i, src.v(), a + i));
    dst.p[b + i] = src.p[a + i];
  }
  R.assign((size_t)k * k, 0.0);
  for (int i = 0; i < k; i++)
    for (int j = 0; j < k; j++) {
      double t = 0;
      for (int m = 0; m < k; m++) t += R2[(size_t)i * k + m] * R1[(size_t)m * k + j];
      R[(size_t)i * k + j] = t;
    }
  return true;
}

// Evolve's derivative at x0 over tau applied to V[a..a+k) into W[b..b+k):
// one batched integration of the base and k tangent-linear runs
// (sf_set_tangent); the scalars of W are zeroed
inline void EvolveTangentBlock(const Vec& x0, double tau, double Ri, int s, const Block& V, int a, int k, Block& W,
                               int b) {
  Context& c = x0.ctx();
  auto t0 = std::chrono::steady_clock::now();
  Solver& S = c.block_tangent_solver(s);
  const int nsteps = std::max(1, (int)std::ceil(tau / c.p.dt - 1e-9));
  S.set_dt(tau / nsteps);
  for (int r = 0; r <= s; r++) S.set_ri(r, Ri);
  Vec base(x0);
  check(sf_vecs_zero_pressure(base.v(), 0, 1));
  check(sf_vecs_to_run(base.v(), 0, S.h(), 0, 1));
  check(sf_vecs_zero_pressure(V.v(), a, k));
  check(sf_vecs_to_run(V.v(), a, S.h(), 1, k));
  check(sf_prepare(S.h()));
  check(sf_step(S.h(), nsteps));
  check(sf_vecs_from_run(W.v(), b, S.h(), 1, k));
  check(sf_vecs_zero_pressure(W.v(), b, k));
  check(sf_vecs_enforce_bcs(W.v(), b, k));
  check(sf_vecs_synchronize(W.v()));
  for (int i = 0; i < k; i++) W.p[b + i] = 0.0;
  c.evolutions += 1;
  c.evolve_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// ------------------------------------------- mean-flow preconditioner ----
// The slowest directions of F(x) = Phi_T(x) - x in a stratified shear layer
// are the horizontally averaged profiles of u1 and b (the (0,0) modes): they
// relax by vertical diffusion alone, over L3^2 Re ~ 1e5 time units, so
// J = Phi_T' - I is nearly singular on them and GMRES needs many vectors to
// resolve them. This right preconditioner applies M = (I - E + Pi)^-1 to the
// (0,0) columns of u1 and b, with E = exp(T nu D2) the diffusion propagator
// of the mean profile (D2 the Neumann second derivative of
// Differentiation.cpp:6-33 with the ghost levels folded in, nu = 1/Re for u1
// and 1/(Re Pr) for b) and Pi the projection on constant profiles (weights
// DYF, which D2 conserves); everything else passes unchanged. Then J M is
// close to -I on the mean profiles, as it is on the fast decaying modes.
class MeanFlowPreconditioner {
 public:
  MeanFlowPreconditioner(const Params& p, double T) : N_(p.N3) {
    const int N = p.N3, n = N - 2;
    std::vector<double> z(N, 0.0), zf(N, 0.0), DY(N, 0.0), DYF(N, 0.0);
    const double step = 2.0 / (N - 2);
    for (int i = 0; i < N - 1; i++) {
      const double x = (i == N - 2) ? 1.0 : -1.0 + i * step;
      z[i + 1] = p.L3 * (2.0 * std::pow(x, 7) + x) / 3.0;
    }
    const double off = (z[1] + z[2]) / 2;
    for (int i = 1; i < N; i++) z[i] *= -p.L3 / off;
    for (int i = 1; i <= N - 2; i++) zf[i] = 0.5 * (z[i] + z[i + 1]);
    zf[0] = 2 * zf[1] - zf[2];
    zf[N - 1] = 2 * zf[N - 2] - zf[N - 3];
    for (int i = 1; i < N; i++) DY[i] = zf[i] - zf[i - 1];
    for (int i = 1; i <= N - 2; i++) DYF[i] = z[i + 1] - z[i];
    // D2 on the interior levels 1..N-2, ghosts f_0 = f_1, f_{N-1} = f_{N-2}
    std::vector<double> A((size_t)n * n, 0.0), w(n);
    for (int j = 1; j <= N - 2; j++) {
      const double lo = 1 / DY[j] / DYF[j], up = 1 / DY[j + 1] / DYF[j], r = j - 1;
      A[(size_t)r * n + r] += -lo - up;
      A[(size_t)r * n + (j == 1 ? r : r - 1)] += lo;
      A[(size_t)r * n + (j == N - 2 ? r : r + 1)] += up;
      w[r] = DYF[j];
    }
    const double nus[2] = {1.0 / p.Re, 1.0 / (p.Re * p.Pr)};
    for (int k = 0; k < 2; k++) {
      std::vector<double> E = expm(A, n, T * nus[k]);
      double ws = 0;
      for (double t : w) ws += t;
      for (int i = 0; i < n; i++)
        for (int j = 0; j < n; j++) E[(size_t)i * n + j] = (i == j ? 1.0 : 0.0) - E[(size_t)i * n + j] + w[j] / ws;
      Minv_[k] = inverse(E, n);
    }
  }

  // M applied in place to vectors a..a+k of a block (u1 and b (0,0) columns)
  void Apply(sf_vecs* v, int a, int k) const {
    const int N = N_, n = N - 2;
    std::vector<float> col(2 * (size_t)N);
    std::vector<double> f(n), g(n);
    for (int i = a; i < a + k; i++)
      for (int q = 0; q < 2; q++) {
        const int field = q == 0 ? 0 : 3;
        check(sf_vecs_column(v, i, field, 0, col.data(), 0));
        for (int r = 0; r < n; r++) f[r] = col[2 * (r + 1)];
        const std::vector<double>& M = Minv_[q];
        for (int r = 0; r < n; r++) {
          double t = 0;
          for (int c = 0; c < n; c++) t += M[(size_t)r * n + c] * f[c];
          g[r] = t;
        }
        for (int r = 0; r < n; r++) col[2 * (r + 1)] = (float)g[r];
        col[0] = col[2];
        col[2 * (N - 1)] = col[2 * (N - 2)];
        check(sf_vecs_column(v, i, field, 0, col.data(), 1));
      }
  }

 private:
  int N_;
  std::vector<double> Minv_[2];

  static std::vector<double> matmul(const std::vector<double>& X, const std::vector<double>& Y, int n) {
    std::vector<double> Z((size_t)n * n, 0.0);
    for (int i = 0; i < n; i++)
      for (int k = 0; k < n; k++) {
        const double x = X[(size_t)i * n + k];
        if (x == 0.0) continue;
        for (int j = 0; j < n; j++) Z[(size_t)i * n + j] += x * Y[(size_t)k * n + j];
      }
    return Z;
  }
  // exp(c A) by scaling and squaring of a degree-16 Taylor polynomial
  static std::vector<double> expm(const std::vector<double>& A, int n, double c) {
    double nrm = 0;
    for (int j = 0; j < n; j++) {
      double t = 0;
      for (int i = 0; i < n; i++) t += std::fabs(A[(size_t)i * n + j]);
      nrm = std::max(nrm, t);
    }
    nrm *= std::fabs(c);
    int sq = 0;
    while (nrm / std::ldexp(1.0, sq) > 0.25) sq++;
    const double scale = c / std::ldexp(1.0, sq);
    std::vector<double> X((size_t)n * n), E((size_t)n * n, 0.0), term((size_t)n * n, 0.0);
    for (size_t i = 0; i < X.size(); i++) X[i] = A[i] * scale;
    for (int i = 0; i < n; i++) E[(size_t)i * n + i] = term[(size_t)i * n + i] = 1.0;
    for (int k = 1; k <= 16; k++) {
      term = matmul(term, X, n);
      for (size_t i = 0; i < term.size(); i++) term[i] /= k;
      for (size_t i = 0; i < E.size(); i++) E[i] += term[i];
    }
    for (int i = 0; i < sq; i++) E = matmul(E, E, n);
    return E;
  }
  // Gauss-Jordan with partial pivoting
  static std::vector<double> inverse(std::vector<double> A, int n) {
    std::vector<double> B((size_t)n * n, 0.0);
    for (int i = 0; i < n; i++) B[(size_t)i * n + i] = 1.0;
    for (int c = 0; c < n; c++) {
      int piv = c;
      for (int r = c + 1; r < n; r++)
        if (std::fabs(A[(size_t)r * n + c]) > std::fabs(A[(size_t)piv * n + c])) piv = r;
      if (A[(size_t)piv * n + c] == 0.0) throw std::runtime_error("mean-flow preconditioner: singular matrix");
      if (piv != c)
        for (int j = 0; j < n; j++) {
          std::swap(A[(size_t)piv * n + j], A[(size_t)c * n + j]);
          std::swap(B[(size_t)piv * n + j], B[(size_t)c * n + j]);
        }
      const double d = 1.0 / A[(size_t)c * n + c];
      for (int j = 0; j < n; j++) {
        A[(size_t)c * n + j] *= d;
        B[(size_t)c * n + j] *= d;
      }
      for (int r = 0; r < n; r++) {
        if (r == c) continue;
        const double f = A[(size_t)r * n + c];
        if (f == 0.0) continue;
        for (int j = 0; j < n; j++) {
          A[(size_t)r * n + j] -= f * A[(size_t)c * n + j];
          B[(size_t)r * n + j] -= f * B[(size_t)c * n + j];
        }
      }
    }
    return B;
  }
};

// Newton-Krylov (NewtonKrylov.h:1-241) for single-shooting problems with a
// block Krylov solver: the residual is split into s pieces (fields x bands
// of j1), so the block Krylov space contains GMRES's Krylov space of the
// residual, and every Arnoldi step applies the Jacobian to s directions in
// one batched tangent-linear integration. Gram-Schmidt is classical, twice
// (CGS2), against the whole basis in FP64 on the device; each new block is
// orthonormalised by Cholesky QR, twice. The least-squares residual is
// checked after each block (Householder QR); the hookstep (trust region of
// NewtonKrylov.h:179-216) uses the SVD of the final block Hessenberg matrix.
class BlockNewtonKrylov {
 public:
  BlockNewtonKrylov(const NKOptions& o, int s) : opt(o), s_(std::max(1, std::min(s, 32))) {}
  virtual ~BlockNewtonKrylov() = default;
  NKOptions opt;

  virtual Vec EvalFunction(const Vec& at) = 0;
  virtual void EnforceConstraints(Vec& at) { (void)at; }
  virtual void AtIterate(const Vec& x, const Vec& F) { (void)x; (void)F; }
  // W[b..b+k) = J V[a..a+k) about x0 (including the scalar rows/columns)
  virtual void ApplyJ(const Vec& x0, const Block& V, int a, int k, Block& W, int b) = 0;
  // the time over which the mean-flow preconditioner relaxes (0: none)
  virtual double PreconditionerTime() const { return 0.0; }

  NKStats Run(Vec& x) {
    NKStats st;
    auto t0 = std::chrono::steady_clock::now();
    Context& c = x.ctx();
    if (c.M != 1) throw std::runtime_error("the block Newton-Krylov solver needs one segment (M = 1)");
    if (opt.precondition && PreconditionerTime() > 0 && !prec_)
      prec_.reset(new MeanFlowPreconditioner(c.p, PreconditionerTime()));
    const long long ev0 = c.evolutions;
    const double es0 = c.evolve_seconds;
    std::unique_ptr<Vec> F(new Vec(EvalFunction(x)));
    double xn = std::max(x.Norm(), 1e-300);
    double res = F->Norm() / xn;
    double Delta = opt.Delta * xn;
    st.residuals.push_back(res);
    for (int it = 0; it < opt.max_newton && res >= opt.target; it++) {
      x0_ = &x;
      AtIterate(x, *F);
      Vec rhs(*F);
      rhs *= -1.0;
      double gres = 1.0;
      const int used = GMRES(x, rhs, gres);
      st.krylov_vectors += used;
      st.gmres_vectors.push_back(used);
      st.gmres_residuals.push_back(gres);
      bool accepted = false;
      for (int attempt = 0; attempt < 8 && !accepted; attempt++) {
        double zn = 0;
        Vec dx = Hookstep(x, Delta, zn);
        Vec xt(x);
        xt.MulAdd(1.0, dx);
        EnforceConstraints(xt);
        EnforceConstraints(xt);
        EnforceConstraints(xt);
        std::unique_ptr<Vec> Ft(new Vec(EvalFunction(xt)));
        const double rt = Ft->Norm() / std::max(xt.Norm(), 1e-300);
        if (rt < res) {
          x = xt;
          F = std::move(Ft);
          if (zn >= 0.9 * Delta && rt < 0.5 * res) Delta *= 2;
          res = rt;
          accepted = true;
        } else {
          Delta = 0.5 * std::min(Delta, zn);
        }
      }
      st.newton_iterations++;
      st.residuals.push_back(res);
      if (verbose())
        std::fprintf(stderr, "NEWTON STEP %d: relative residual %.3e (GMRES %.3e, %d vectors)%s\n", it + 1, res,
                     gres, used, accepted ? "" : ", no step accepted");
      if (!accepted) break;
    }
    st.residual = res;
    st.converged = res < opt.target;
    st.evolutions = c.evolutions - ev0;
    st.evolve_seconds = c.evolve_seconds - es0;
    st.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    x0_ = nullptr;
    return st;
  }

 protected:
  const Vec* x0_ = nullptr;
  int s_;
  int bw_ = 0;                       // block width in use
  int n_ = 0;                        // basis vectors in the least-squares problem
  std::unique_ptr<Block> V_, W_, Z_;
  std::unique_ptr<MeanFlowPreconditioner> prec_;
  std::vector<double> H_;            // (cap + bw) x cap, row-major with stride cap
  std::vector<double> b0_;           // right-hand side in the basis
  int cap_ = 0;

  // rhs = sum of its pieces: u1, (u2,) u3, b, each split into bands of j1
  int Split(const Vec& rhs) {
    const Params& P = rhs.ctx().p;
    const int K1 = P.N1 / 3;
    std::vector<int> fields = P.N2 > 1 ? std::vector<int>{0, 1, 2, 3} : std::vector<int>{0, 2, 3};
    const int nbands = std::max(1, s_ / (int)fields.size());
    std::vector<int> edges{0};
    for (int q = 1; q < nbands; q++) edges.push_back(std::min(K1, 1 << (q - 1)));
    edges.push_back(K1);
    int n = 0;
    const double rn2 = rhs.Dot(rhs);
    for (int f : fields)
      for (int q = 0; q < nbands; q++) {
        if (edges[q] >= edges[q + 1]) continue;
        check(sf_vecs_copy(V_->v(), n, rhs.v(), 0));
        check(sf_vecs_band(V_->v(), n, 1 << f, edges[q], edges[q + 1]));
        V_->p[n] = 0.0;
        double d = 0;
        check(sf_vecs_dot_sum(V_->v(), n, V_->v(), n, 1, rhs.ctx().p.Ri, &d));
        if (d > 1e-20 * rn2) n++;   // pieces with no share of the residual are left out
      }
    if (rhs.p != 0.0 || n == 0) {   // the scalar row is a piece of its own
      check(sf_vecs_scale(V_->v(), n, 0.0, 1));
      V_->p[n] = rhs.p;
      n++;
    }
    return n;
  }

  // two passes of Cholesky QR from W[0..k) into V[at..at+k)
  bool CholQR2(int at, int k, double Ri, std::vector<double>& R) { return cholqr2(*W_, 0, *V_, at, k, Ri, R); }

  // least squares min |b0 - H y| over the first n columns
  double Residual(int n, std::vector<double>& y) {
    const int m = n + bw_;
    std::vector<double> A((size_t)m * n), b(b0_.begin(), b0_.begin() + m);
    for (int i = 0; i < m; i++)
      for (int j = 0; j < n; j++) A[(size_t)i * n + j] = H_[(size_t)i * cap_ + j];
    return lsq_householder(A, m, n, b, y);
  }

  // block Arnoldi for J y = rhs; returns the Jacobian actions
  int GMRES(const Vec& x0, const Vec& rhs, double& rel) {
    Context& c = rhs.ctx();
    const double Ri = c.p.Ri;
    cap_ = std::max(opt.krylov / s_, 1) * s_;
    if (!V_ || V_->n() < cap_ + s_ + 1) V_.reset(new Block(c, cap_ + s_ + 1));
    if (!W_ || W_->n() < s_ + 1) W_.reset(new Block(c, s_ + 1));
    if (prec_ && (!Z_ || Z_->n() < s_ + 1)) Z_.reset(new Block(c, s_ + 1));
    // the pieces of the residual, orthonormalised: rhs = V_1 R_1 (1,..,1)
    int k = Split(rhs);
    for (int i = 0; i < k; i++) {
      check(sf_vecs_copy(W_->v(), i, V_->v(), i));
      W_->p[i] = V_->p[i];
    }
    std::vector<double> R;
    while (k > 0 && !CholQR2(0, k, Ri, R)) k--;   // drop trailing pieces until independent
    bw_ = k;
    H_.assign((size_t)(cap_ + bw_) * cap_, 0.0);
    b0_.assign(cap_ + bw_, 0.0);
    for (int i = 0; i < bw_; i++)
      for (int j = 0; j < bw_; j++) b0_[i] += R[(size_t)i * bw_ + j];
    double bn = 0;
    for (double t : b0_) bn += t * t;
    bn = std::sqrt(bn);
    n_ = 0;
    rel = 1.0;
    if (!(bn > 0) || bw_ == 0) return 0;
    int used = 0;
    std::vector<double> y;
    for (int j = 0; (j + 1) * bw_ <= cap_; j++) {
      const int nb = (j + 1) * bw_;   // basis vectors so far
      if (prec_) {   // right preconditioning: the basis spans J M
        for (int i = 0; i < bw_; i++) {
          check(sf_vecs_copy(Z_->v(), i, V_->v(), j * bw_ + i));
          Z_->p[i] = V_->p[j * bw_ + i];
        }
        prec_->Apply(Z_->v(), 0, bw_);
        ApplyJ(x0, *Z_, 0, bw_, *W_, 0);
      } else {
        ApplyJ(x0, *V_, j * bw_, bw_, *W_, 0);
      }
      used += bw_;
      for (int pass = 0; pass < 2; pass++) {
        std::vector<double> C = block_gram(*V_, 0, nb, *W_, 0, bw_, Ri);
        for (int i = 0; i < nb; i++)
          for (int q = 0; q < bw_; q++) H_[(size_t)i * cap_ + j * bw_ + q] += C[(size_t)i * bw_ + q];
        block_update(*W_, 0, bw_, -1.0, *V_, 0, nb, C);
      }
      std::vector<double> Rn;
      const bool ok = nb + bw_ <= cap_ + bw_ && CholQR2(nb, bw_, Ri, Rn);
      if (ok)
        for (int i = 0; i < bw_; i++)
          for (int q = 0; q < bw_; q++) H_[(size_t)(nb + i) * cap_ + j * bw_ + q] = Rn[(size_t)i * bw_ + q];
      n_ = nb;
      rel = Residual(n_, y) / bn;
      if (verbose())
        std::fprintf(stderr, "block GMRES: %d vectors, relative residual %.3e%s\n", nb, rel,
                     ok ? "" : " (new block rank deficient)");
      if (!ok || rel < opt.gmres_tol) break;
    }
    return used;
  }

  // the trust-region step (NewtonKrylov.h:179-216) in the block basis
  Vec Hookstep(const Vec& like, double Delta, double& znorm) {
    Vec dx(like);
    dx.Zero();
    znorm = 0;
    if (n_ == 0) return dx;
    const int m = n_ + bw_, n = n_;
    std::vector<double> sub((size_t)m * n), U, S, Vv;
    for (int i = 0; i < m; i++)
      for (int j = 0; j < n; j++) sub[(size_t)i * n + j] = H_[(size_t)i * cap_ + j];
    svd(sub, m, n, U, S, Vv);
    std::vector<double> pv(n, 0.0), z(n);
    for (int j = 0; j < n; j++)
      for (int i = 0; i < m; i++) pv[j] += U[(size_t)i * n + j] * b0_[i];
    const double smax = *std::max_element(S.begin(), S.end());
    auto zfor = [&](double mu) {
      double t = 0;
      for (int j = 0; j < n; j++) {
        const double d = S[j];
        z[j] = (d > 1e-13 * smax) ? pv[j] * d / (d * d + mu) : 0.0;
        t += z[j] * z[j];
      }
      return std::sqrt(t);
    };
    double mu = 0;
    if (zfor(0) > Delta) {
      double lo = 0, hi = 1e-12;
      while (zfor(hi) > Delta) hi *= 4;
      for (int it = 0; it < 80; it++) {
        const double mid = 0.5 * (lo + hi);
        (zfor(mid) > Delta ? lo : hi) = mid;
      }
      mu = hi;
    }
    znorm = zfor(mu);
    std::vector<double> y(n, 0.0);
    for (int i = 0; i < n; i++)
      for (int j = 0; j < n; j++) y[i] += Vv[(size_t)i * n + j] * z[j];
    check(sf_vecs_update(dx.v(), 0, 1, 1.0, V_->v(), 0, n, y.data()));
    if (prec_) prec_->Apply(dx.v(), 0, 1);
    double p = 0;
    for (int i = 0; i < n; i++) p += y[i] * V_->p[i];
    dx.p = p;
    dx.EnforceBCs();
    return dx;
  }
};

// F_i = Phi(x_i) - x_{i+1 mod M} for every segment i
inline Vec ShootingResidual(const Vec& phi, const Vec& at) {
  Vec r(phi);
  const int M = at.M();
  for (int i = 0; i < M; i++) check(sf_vecs_axpy(r.v(), i, -1.0, at.v(), (i + 1) % M, 1));
  r.EnforceBCs();
  return r;
}

// Dot of segment `seg` of a and b (StateVector::Dot)
inline double SegmentDot(const Vec& a, const Vec& b, int seg) {
  double d = 0;
  check(sf_vecs_dot_sum(a.v(), seg, b.v(), seg, 1, a.ctx().p.Ri, &d));
  return d;
}

// FindPeriodic (FindPeriodic.cpp:4-28) by multiple shooting: unknowns
// (x_0..x_{M-1}, p = T); F_i = Phi_{T/M}(x_i) - x_{i+1 mod M},
// F_p = n . (x_0 - x_ref) with n the flow direction at the initial guess
// (the reference uses n . (Phi_T(x) - offset)).
class PeriodicOrbit : public NewtonKrylov {
 public:
  PeriodicOrbit(const NKOptions& o, const Vec& guess) : NewtonKrylov(o), ref_(guess), normal_(guess) {
    Context& c = guess.ctx();
    Vec e1(guess), e2(guess);
    Evolve(guess, c.p.dt, c.p.Ri, e1, &e2);
    normal_ = e2;
    normal_.MulAdd(-1.0, e1);
    normal_ *= 1.0 / c.p.dt;
    normal_.p = 0;
  }
  Vec EvalFunction(const Vec& at) override {
    Context& c = at.ctx();
    Vec phi(at), ext(at);
    Evolve(at, at.p / c.M, c.p.Ri, phi, &ext);
    Vec r = ShootingResidual(phi, at);
    Vec d(at);
    d.MulAdd(-1.0, ref_);
    r.p = SegmentDot(normal_, d, 0);
    ext.MulAdd(-1.0, phi);   // flow direction at the segment ends
    ext *= 1.0 / c.solver->dt();
    last_f_.reset(new Vec(ext));
    return r;
  }
  void AtIterate(const Vec& x, const Vec& F) override {
    (void)x; (void)F;
    f0_ = std::move(last_f_);
  }
  // J (dX, dT): Phi' dx_i - dx_{i+1}, plus dT/M times the flow direction at
  // the segment ends, and the phase condition n . dx_0
  Vec EvalDerivative(const Vec& dir) override {
    Vec d(dir);
    d.p = 0;
    Vec r(d);
    if (opt.tangent) {
      Context& c = d.ctx();
      Vec phi(d);
      EvolveTangent(*x0_, d, x0_->p / c.M, c.p.Ri, phi);
      r = ShootingResidual(phi, d);
    } else {
      r = NewtonKrylov::EvalDerivative(d);
    }
    if (f0_) r.MulAdd(dir.p / dir.ctx().M, *f0_);
    r.p = SegmentDot(normal_, d, 0);
    return r;
  }

 private:
  Vec ref_, normal_;
  std::unique_ptr<Vec> last_f_, f0_;
};

// PseudoArclengthContinuation (PseudoArclength.h:6-42) by multiple shooting:
// unknowns (x_0..x_{M-1}, p = Ri); F_i = Phi_{T/M}(x_i; Ri) - x_{i+1 mod M},
// F_p = ds - v . (X - X0); EnforceConstraints removes the phase shift and the
// averages of u1 and b (PseudoArclength.h:15-20).
class PseudoArclength : public NewtonKrylov {
 public:
  PseudoArclength(const NKOptions& o, const Vec& x0, const Vec& v, double ds, double T)
      : NewtonKrylov(o), x0c_(x0), v_(v), ds_(ds), T_(T) {}
  Vec EvalFunction(const Vec& at) override {
    Context& c = at.ctx();
    Vec phi(at);
    Evolve(at, T_ / c.M, at.p, phi);
    Vec r = ShootingResidual(phi, at);
    Vec d(at);
    d.MulAdd(-1.0, x0c_);
    r.p = ds_ - v_.Dot(d);
    last_phi_.reset(new Vec(phi));
    return r;
  }
  void EnforceConstraints(Vec& at) override {
    at.RemovePhaseShift();
    at.RemoveAverage(0);
    at.RemoveAverage(3);
  }
  // dPhi/dRi at the Newton iterate by a one-sided difference in Ri
  void AtIterate(const Vec& x, const Vec& F) override {
    (void)F;
    if (!opt.tangent || !last_phi_) return;
    const double e = std::max(1e-3 * std::fabs(x.p), 1e-5);
    Vec phi(x);
    Evolve(x, T_ / x.ctx().M, x.p + e, phi);
    phi.MulAdd(-1.0, *last_phi_);
    phi *= 1.0 / e;
    phi.p = 0;
    dphi_dri_.reset(new Vec(phi));
  }
  // J (dX, dRi) = Phi' dx_i + dRi dPhi/dRi - dx_{i+1}; -v . (dX, dRi)
  Vec EvalDerivative(const Vec& dir) override {
    if (!opt.tangent || !dphi_dri_) return NewtonKrylov::EvalDerivative(dir);
    Vec d(dir);
    d.p = 0;
    Vec phi(d);
    EvolveTangent(*x0_, d, T_ / d.ctx().M, x0_->p, phi);
    Vec r = ShootingResidual(phi, d);
    r.MulAdd(dir.p, *dphi_dri_);
    r.p = -v_.Dot(dir);
    return r;
  }

 private:
  Vec x0c_, v_;
  double ds_, T_;
  std::unique_ptr<Vec> last_phi_, dphi_dri_;
};

// ------------------------------------------ block single-shooting problems
// W_i -= V_i for i < k (the "- x" of F = Phi(x) - x)
inline void subtract_identity(const Block& V, int a, int k, Block& W, int b) {
  std::vector<double> I((size_t)k * k, 0.0);
  for (int i = 0; i < k; i++) I[(size_t)i * k + i] = 1.0;
  block_update(W, b, k, -1.0, V, a, k, I);
}

// BasicNewtonKrylov (BasicNewtonKrylov.h:5-14) for Phi_T(x) = x, with the
// phase and average constraints of PseudoArclength.h:15-20
//
// With NKOptions::relative the translation in x, which Phi_T commutes with
// and which makes J singular, becomes an unknown instead of being removed
// after each update: unknowns (x, p = sigma), F = S_sigma Phi_T(x) - x with
// S_sigma the phase shift of StateVector::RemovePhaseShift (mode j1 times
// e^{i j1 sigma}), and the phase condition F_p = t . (x - x_ref), t the
// direction of a shift of the initial guess x_ref (a relative equilibrium;
// sigma = 0 for a steady state).
class BlockFixedPoint : public BlockNewtonKrylov {
 public:
  BlockFixedPoint(const NKOptions& o, int s, double T, bool constrain)
      : BlockNewtonKrylov(o, s), T_(T), constrain_(constrain) {}
  void SetReference(const Vec& x) {
    if (!opt.relative) return;
    ref_.reset(new Vec(x));
    tref_.reset(new Vec(ShiftDerivative(x)));
    tref_->p = 0;
  }
  Vec EvalFunction(const Vec& at) override {
    Vec phi(at);
    Evolve(at, T_, at.ctx().p.Ri, phi);
    if (opt.relative && ref_) {
      double sh = at.p;
      for (int i = 0; i < phi.M(); i++) check(sf_vecs_phase_shift(phi.v(), i, 1, &sh));
      last_phi_.reset(new Vec(phi));
      Vec d(at);
      d.MulAdd(-1.0, *ref_);
      phi.MulAdd(-1.0, at);
      phi.p = SegmentDot(*tref_, d, 0);
      return phi;
    }
    phi.MulAdd(-1.0, at);
    phi.p = 0;
    return phi;
  }
  void EnforceConstraints(Vec& at) override {
    if (!constrain_) return;
    if (!opt.relative) at.RemovePhaseShift();   // else the phase condition fixes the phase
    at.RemoveAverage(0);
    at.RemoveAverage(3);
  }
  void AtIterate(const Vec& x, const Vec& F) override {
    (void)x; (void)F;
    if (opt.relative && last_phi_) {
      dsigma_.reset(new Vec(ShiftDerivative(*last_phi_)));
      dsigma_->p = 0;
    }
  }
  void ApplyJ(const Vec& x0, const Block& V, int a, int k, Block& W, int b) override {
    EvolveTangentBlock(x0, T_, x0.ctx().p.Ri, k, V, a, k, W, b);
    if (opt.relative && ref_) {
      double sh = x0.p;
      for (int i = 0; i < k; i++) check(sf_vecs_phase_shift(W.v(), b + i, 1, &sh));
    }
    subtract_identity(V, a, k, W, b);
    if (opt.relative && dsigma_) {
      check(sf_vecs_update(W.v(), b, k, 1.0, dsigma_->v(), 0, 1, &V.p[a]));
      std::vector<double> td(k);
      check(sf_vecs_gram(V.v(), a, k, tref_->v(), 0, 1, x0.ctx().p.Ri, td.data()));
      for (int i = 0; i < k; i++) W.p[b + i] = td[i];
    }
  }
  double PreconditionerTime() const override { return T_; }

 private:
  double T_;
  bool constrain_;
  std::unique_ptr<Vec> ref_, tref_, last_phi_, dsigma_;

  // d/dsigma of S_sigma y at sigma = 0 by a central difference of exact phase
  // shifts (i j1 y up to (j1 e)^2 / 6)
  static Vec ShiftDerivative(const Vec& y) {
    const double e = 1e-3;
    Vec a(y), b(y);
    double sp = e, sm = -e;
    for (int i = 0; i < y.M(); i++) {
      check(sf_vecs_phase_shift(a.v(), i, 1, &sp));
      check(sf_vecs_phase_shift(b.v(), i, 1, &sm));
    }
    check(sf_vecs_lincomb(a.v(), 0, 1.0 / (2 * e), -1.0 / (2 * e), b.v(), 0, y.M()));
    a.p = 0;
    return a;
  }
};

// FindPeriodic (FindPeriodic.cpp:4-28): unknowns (x, p = T); F = Phi_T(x) - x,
// F_p = n . (x - x_ref) with n the flow direction at the initial guess
class BlockPeriodicOrbit : public BlockNewtonKrylov {
 public:
  BlockPeriodicOrbit(const NKOptions& o, int s, const Vec& guess)
      : BlockNewtonKrylov(o, s), ref_(guess), normal_(guess) {
    Context& c = guess.ctx();
    Vec e1(guess), e2(guess);
    Evolve(guess, c.p.dt, c.p.Ri, e1, &e2);
    normal_ = e2;
    normal_.MulAdd(-1.0, e1);
    normal_ *= 1.0 / c.p.dt;
    normal_.p = 0;
  }
  Vec EvalFunction(const Vec& at) override {
    Context& c = at.ctx();
    Vec phi(at), ext(at);
    Evolve(at, at.p, c.p.Ri, phi, &ext);
    ext.MulAdd(-1.0, phi);
    ext *= 1.0 / c.solver->dt();
    ext.p = 0;
    last_f_.reset(new Vec(ext));
    Vec d(at);
    d.MulAdd(-1.0, ref_);
    phi.MulAdd(-1.0, at);
    phi.p = SegmentDot(normal_, d, 0);
    return phi;
  }
  void AtIterate(const Vec& x, const Vec& F) override {
    (void)x; (void)F;
    f0_ = std::move(last_f_);
  }
  double PreconditionerTime() const override { return ref_.p; }
  void ApplyJ(const Vec& x0, const Block& V, int a, int k, Block& W, int b) override {
    Context& c = x0.ctx();
    EvolveTangentBlock(x0, x0.p, c.p.Ri, k, V, a, k, W, b);
    subtract_identity(V, a, k, W, b);
    if (f0_) check(sf_vecs_update(W.v(), b, k, 1.0, f0_->v(), 0, 1, &V.p[a]));
    std::vector<double> nd(k);
    check(sf_vecs_gram(V.v(), a, k, normal_.v(), 0, 1, c.p.Ri, nd.data()));
    for (int i = 0; i < k; i++) W.p[b + i] = nd[i];
  }

 private:
  Vec ref_, normal_;
  std::unique_ptr<Vec> last_f_, f0_;
};

// PseudoArclengthContinuation (PseudoArclength.h:6-42): unknowns (x, p = Ri)
class BlockPseudoArclength : public BlockNewtonKrylov {
 public:
  BlockPseudoArclength(const NKOptions& o, int s, const Vec& x0, const Vec& v, double ds, double T)
      : BlockNewtonKrylov(o, s), x0c_(x0), v_(v), ds_(ds), T_(T) {}
  Vec EvalFunction(const Vec& at) override {
    Vec phi(at);
    Evolve(at, T_, at.p, phi);
    last_phi_.reset(new Vec(phi));
    phi.MulAdd(-1.0, at);
    Vec d(at);
    d.MulAdd(-1.0, x0c_);
    phi.p = ds_ - v_.Dot(d);
    return phi;
  }
  void EnforceConstraints(Vec& at) override {
    at.RemovePhaseShift();
    at.RemoveAverage(0);
    at.RemoveAverage(3);
  }
  // dPhi/dRi at the Newton iterate by a one-sided difference in Ri
  void AtIterate(const Vec& x, const Vec& F) override {
    (void)F;
    const double e = std::max(1e-3 * std::fabs(x.p), 1e-5);
    Vec phi(x);
    Evolve(x, T_, x.p + e, phi);
    phi.MulAdd(-1.0, *last_phi_);
    phi *= 1.0 / e;
    phi.p = 0;
    dphi_dri_.reset(new Vec(phi));
  }
  double PreconditionerTime() const override { return T_; }
  void ApplyJ(const Vec& x0, const Block& V, int a, int k, Block& W, int b) override {
    Context& c = x0.ctx();
    EvolveTangentBlock(x0, T_, x0.p, k, V, a, k, W, b);
    subtract_identity(V, a, k, W, b);
    check(sf_vecs_update(W.v(), b, k, 1.0, dphi_dri_->v(), 0, 1, &V.p[a]));
    std::vector<double> vd(k);
    check(sf_vecs_gram(V.v(), a, k, v_.v(), 0, 1, c.p.Ri, vd.data()));
    for (int i = 0; i < k; i++) W.p[b + i] = -(vd[i] + v_.p * V.p[a + i]);
  }

 private:
  Vec x0c_, v_;
  double ds_, T_;
  std::unique_ptr<Vec> last_phi_, dphi_dri_;
};

// -------------------------------------------------------------- Arnoldi ----
// eigenvalues of a real n x n matrix (row-major): Householder reduction to
// upper Hessenberg form, then the complex QR algorithm with Wilkinson shifts
// and deflation (Golub & Van Loan, Matrix Computations, 7.4-7.5)
inline std::vector<std::complex<double>> eigenvalues(std::vector<double> A, int n) {
  using cd = std::complex<double>;
  for (int k = 0; k + 2 < n; k++) {   // Hessenberg reduction
    double nrm = 0;
    for (int i = k + 1; i < n; i++) nrm += A[(size_t)i * n + k] * A[(size_t)i * n + k];
    nrm = std::sqrt(nrm);
    if (nrm == 0) continue;
    const double a0 = A[(size_t)(k + 1) * n + k];
    const double alpha = a0 > 0 ? -nrm : nrm;
    std::vector<double> v(n - k - 1);
    for (int i = k + 1; i < n; i++) v[i - k - 1] = A[(size_t)i * n + k];
    v[0] -= alpha;
    double vn = 0;
    for (double t : v) vn += t * t;
    if (vn == 0) continue;
    for (int j = 0; j < n; j++) {   // A = (I - 2vv'/v'v) A
      double d = 0;
      for (int i = k + 1; i < n; i++) d += v[i - k - 1] * A[(size_t)i * n + j];
      d = 2 * d / vn;
      for (int i = k + 1; i < n; i++) A[(size_t)i * n + j] -= d * v[i - k - 1];
    }
    for (int i = 0; i < n; i++) {   // A = A (I - 2vv'/v'v)
      double d = 0;
      for (int j = k + 1; j < n; j++) d += A[(size_t)i * n + j] * v[j - k - 1];
      d = 2 * d / vn;
      for (int j = k + 1; j < n; j++) A[(size_t)i * n + j] -= d * v[j - k - 1];
    }
  }
  std::vector<cd> H((size_t)n * n);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) H[(size_t)i * n + j] = (j >= i - 1) ? cd(A[(size_t)i * n + j], 0.0) : cd(0.0);
  std::vector<cd> ev;
  int hi = n - 1, iter = 0;
  while (hi >= 0) {
    if (hi == 0) {
      ev.push_back(H[0]);
      break;
    }
    int lo = hi;   // find the active block [lo, hi]
    while (lo > 0) {
      const double s = std::abs(H[(size_t)lo * n + lo]) + std::abs(H[(size_t)(lo - 1) * n + lo - 1]);
      if (std::abs(H[(size_t)lo * n + lo - 1]) <= 1e-15 * (s > 0 ? s : 1.0)) {
        H[(size_t)lo * n + lo - 1] = 0;
        break;
      }
      lo--;
    }
    if (lo == hi) {
      ev.push_back(H[(size_t)hi * n + hi]);
      hi--;
      iter = 0;
      continue;
    }
    // Wilkinson shift: the eigenvalue of the trailing 2 x 2 block closer to H(hi,hi)
    const cd a = H[(size_t)(hi - 1) * n + hi - 1], b = H[(size_t)(hi - 1) * n + hi];
    const cd c = H[(size_t)hi * n + hi - 1], d = H[(size_t)hi * n + hi];
    const cd tr = a + d, det = a * d - b * c;
    const cd disc = std::sqrt(tr * tr / 4.0 - det);
    const cd l1 = tr / 2.0 + disc, l2 = tr / 2.0 - disc;
    cd mu = std::abs(l1 - d) < std::abs(l2 - d) ? l1 : l2;
    if (++iter % 11 == 0) mu += std::abs(c);   // exceptional shift
    if (iter > 60 * n) throw std::runtime_error("eigenvalues: QR iteration did not converge");
    // one shifted QR step on the block by Givens rotations
    std::vector<cd> cs(hi - lo), sn(hi - lo);
    for (int k = lo; k <= hi; k++) H[(size_t)k * n + k] -= mu;
    for (int k = lo; k < hi; k++) {
      const cd x = H[(size_t)k * n + k], y = H[(size_t)(k + 1) * n + k];
      const double r = std::sqrt(std::norm(x) + std::norm(y));
      const cd cc = r > 0 ? x / r : cd(1.0), ss = r > 0 ? y / r : cd(0.0);
      cs[k - lo] = cc;
      sn[k - lo] = ss;
      for (int j = k; j < n; j++) {   // rows k, k+1 <- G^H [rows]
        const cd t1 = H[(size_t)k * n + j], t2 = H[(size_t)(k + 1) * n + j];
        H[(size_t)k * n + j] = std::conj(cc) * t1 + std::conj(ss) * t2;
        H[(size_t)(k + 1) * n + j] = -ss * t1 + cc * t2;
      }
    }
    for (int k = lo; k < hi; k++) {   // columns k, k+1 <- [cols] G
      const cd cc = cs[k - lo], ss = sn[k - lo];
      for (int i = 0; i <= std::min(k + 2, hi); i++) {
        const cd t1 = H[(size_t)i * n + k], t2 = H[(size_t)i * n + k + 1];
        H[(size_t)i * n + k] = t1 * cc + t2 * ss;
        H[(size_t)i * n + k + 1] = -t1 * std::conj(ss) + t2 * std::conj(cc);
      }
    }
    for (int k = lo; k <= hi; k++) H[(size_t)k * n + k] += mu;
  }
  return ev;
}

// a null vector of (A - lambda I), A real n x n, by inverse iteration with
// complex LU (partial pivoting); unit 2-norm
inline std::vector<std::complex<double>> eigenvector(const std::vector<double>& A, int n, std::complex<double> lambda) {
  using cd = std::complex<double>;
  std::vector<cd> M((size_t)n * n);
  double scale = 0;
  for (double t : A) scale = std::max(scale, std::fabs(t));
  const cd shift = lambda + cd(1e-10 * (scale > 0 ? scale : 1.0), 0.0);
  for (int i = 0; i < n; i++)
    for (int j = 0; j < n; j++) M[(size_t)i * n + j] = cd(A[(size_t)i * n + j], 0.0) - (i == j ? shift : cd(0.0));
  std::vector<int> piv(n);
  for (int k = 0; k < n; k++) {
    int p = k;
    for (int i = k + 1; i < n; i++)
      if (std::abs(M[(size_t)i * n + k]) > std::abs(M[(size_t)p * n + k])) p = i;
    piv[k] = p;
    if (p != k)
      for (int j = 0; j < n; j++) std::swap(M[(size_t)p * n + j], M[(size_t)k * n + j]);
    if (std::abs(M[(size_t)k * n + k]) == 0.0) M[(size_t)k * n + k] = 1e-300;
    for (int i = k + 1; i < n; i++) {
      const cd f = M[(size_t)i * n + k] / M[(size_t)k * n + k];
      M[(size_t)i * n + k] = f;
      for (int j = k + 1; j < n; j++) M[(size_t)i * n + j] -= f * M[(size_t)k * n + j];
    }
  }
  std::vector<cd> x(n, cd(1.0));
  for (int it = 0; it < 3; it++) {
    for (int k = 0; k < n; k++) std::swap(x[k], x[piv[k]]);
    for (int i = 0; i < n; i++)
      for (int j = 0; j < i; j++) x[i] -= M[(size_t)i * n + j] * x[j];
    for (int i = n - 1; i >= 0; i--) {
      for (int j = i + 1; j < n; j++) x[i] -= M[(size_t)i * n + j] * x[j];
      x[i] /= M[(size_t)i * n + i];
    }
    double nrm = 0;
    for (const cd& t : x) nrm += std::norm(t);
    nrm = std::sqrt(nrm);
    for (cd& t : x) t /= nrm;
  }
  return x;
}

struct ArnoldiResult {
  std::vector<std::complex<double>> eigenvalues;   // by decreasing modulus
  int vectors = 0;                                  // linearised integrations (directions)
  long long integrations = 0;                       // batched integrations
  double seconds = 0;
};

// Arnoldi (Arnoldi.h:15-193, BasicArnoldi): eigenvalues of the linearised
// evolution over T about a frozen base state (StateVector::LinearEvolve,
// StateVector.cpp:107-155), with s directions per batched integration
// (block Arnoldi; s = 1 is the reference's), FP64 block Gram-Schmidt (CGS2)
// and Cholesky QR, and the eigenvalues of the block Hessenberg matrix in
// FP64. It stops when the nev largest Ritz values change by less than tol
// (relative) from one block to the next, or after `krylov` vectors. With
// eig_re/eig_im it returns the real and imaginary parts of the leading
// eigenvector (the reference's eigReal / eigImag).
class BlockArnoldi {
 public:
  BlockArnoldi(int s, int krylov, double tol, int nev, unsigned long long seed = 1)
      : s_(std::max(1, std::min(s, 32))), K_(krylov), tol_(tol), nev_(nev), seed_(seed) {}

  ArnoldiResult Run(const Vec& about, double T, Vec* eig_re = nullptr, Vec* eig_im = nullptr) {
    Context& c = about.ctx();
    if (c.M != 1) throw std::runtime_error("Arnoldi needs one segment (M = 1)");
    auto t0 = std::chrono::steady_clock::now();
    const double Ri = c.p.Ri;
    const int cap = std::max(K_ / s_, 2) * s_;
    Block V(c, cap + s_), W(c, s_);
    Solver S(c.p, s_);
    void* base = nullptr;
    check(sf_vecs_device(about.v(), 0, &base));
    for (int r = 0; r < s_; r++) check(sf_set_base_device(S.h(), r, base));
    const int nsteps = std::max(1, (int)std::ceil(T / c.p.dt - 1e-9));
    S.set_dt(T / nsteps);
    // starting block: seeded low-wavenumber excitations (ExciteLowWavenumbers, StateVector.cpp:228-236)
    Seed(c, W);
    std::vector<double> R;
    if (!cholqr2(W, 0, V, 0, s_, Ri, R)) throw std::runtime_error("Arnoldi: degenerate starting block");
    std::vector<double> H((size_t)(cap + s_) * cap, 0.0);
    ArnoldiResult res;
    std::vector<std::complex<double>> prev;
    int n = 0;
    for (int j = 0; (j + 1) * s_ <= cap; j++) {
      const int nb = (j + 1) * s_;
      // W = L V_j: one batched linearised integration of s directions
      check(sf_vecs_zero_pressure(V.v(), j * s_, s_));
      check(sf_vecs_to_run(V.v(), j * s_, S.h(), 0, s_));
      check(sf_prepare(S.h()));
      check(sf_step_linear(S.h(), nsteps));
      check(sf_vecs_from_run(W.v(), 0, S.h(), 0, s_));
      check(sf_vecs_zero_pressure(W.v(), 0, s_));
      check(sf_vecs_enforce_bcs(W.v(), 0, s_));
      for (int i = 0; i < s_; i++) W.p[i] = 0;
      res.vectors += s_;
      res.integrations += 1;
      for (int pass = 0; pass < 2; pass++) {
        std::vector<double> C = block_gram(V, 0, nb, W, 0, s_, Ri);
        for (int i = 0; i < nb; i++)
          for (int q = 0; q < s_; q++) H[(size_t)i * cap + j * s_ + q] += C[(size_t)i * s_ + q];
        block_update(W, 0, s_, -1.0, V, 0, nb, C);
      }
      n = nb;
      std::vector<double> Rn;
      const bool ok = nb + s_ <= cap + s_ && cholqr2(W, 0, V, nb, s_, Ri, Rn);
      if (ok)
        for (int i = 0; i < s_; i++)
          for (int q = 0; q < s_; q++) H[(size_t)(nb + i) * cap + j * s_ + q] = Rn[(size_t)i * s_ + q];
      std::vector<double> Hn((size_t)n * n);
      for (int i = 0; i < n; i++)
        for (int q = 0; q < n; q++) Hn[(size_t)i * n + q] = H[(size_t)i * cap + q];
      std::vector<std::complex<double>> ev = eigenvalues(Hn, n);
      std::sort(ev.begin(), ev.end(), [](auto x, auto y) { return std::abs(x) > std::abs(y); });
      double change = 1.0;
      if (!prev.empty()) {
        change = 0;
        for (int k = 0; k < std::min<int>(nev_, (int)std::min(ev.size(), prev.size())); k++)
          change = std::max(change, std::abs(std::abs(ev[k]) - std::abs(prev[k])) / std::max(std::abs(ev[k]), 1e-300));
      }
      if (verbose())
        std::fprintf(stderr, "Arnoldi: %d vectors, largest |eigenvalue| %.8e, change %.2e\n", n, std::abs(ev[0]),
                     change);
      prev = ev;
      res.eigenvalues = ev;
      if (!ok || change < tol_) break;
    }
    if (eig_re || eig_im) {
      std::vector<double> Hn((size_t)n * n);
      for (int i = 0; i < n; i++)
        for (int q = 0; q < n; q++) Hn[(size_t)i * n + q] = H[(size_t)i * cap + q];
      std::vector<std::complex<double>> y = eigenvector(Hn, n, res.eigenvalues[0]);
      std::vector<double> yr(n), yi(n);
      for (int i = 0; i < n; i++) {
        yr[i] = y[i].real();
        yi[i] = y[i].imag();
      }
      if (eig_re) {
        eig_re->Zero();
        check(sf_vecs_update(eig_re->v(), 0, 1, 1.0, V.v(), 0, n, yr.data()));
      }
      if (eig_im) {
        eig_im->Zero();
        check(sf_vecs_update(eig_im->v(), 0, 1, 1.0, V.v(), 0, n, yi.data()));
      }
    }
    res.seconds = std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
    return res;
  }

 private:
  int s_, K_;
  double tol_;
  int nev_;
  unsigned long long seed_;

  void Seed(Context& c, Block& W) {
    const Params& p = c.p;
    const int K1 = p.N1 / 3, K2 = p.N2 > 1 ? 2 * (p.N2 / 3) - 1 : 1, Ky = p.N2 > 1 ? p.N2 / 3 : 1;
    const int plane = (K1 * K2 + 15) / 16 * 16;
    std::vector<float> h((size_t)2 * 5 * p.N3 * plane);
    std::mt19937_64 rng(seed_);
    std::normal_distribution<double> nd(0.0, 1.0);
    auto zf = vertical_points_fractional(p.L3, p.N3);
    for (int i = 0; i < W.n(); i++) {
      std::fill(h.begin(), h.end(), 0.f);
      for (int f = 0; f < 4; f++) {
        if (f == 1 && p.N2 == 1) continue;
        for (int j = 1; j < p.N3 - 1; j++)
          for (int q = 0; q < K2; q++) {
            const int ky = q < Ky ? q : q - K2;
            if (std::abs(ky) >= 8) continue;
            for (int j1 = 0; j1 < std::min(K1, 8); j1++) {
              const double w = std::exp(-zf[j] * zf[j]);
              const size_t o = 2 * (((size_t)f * p.N3 + j) * plane + (size_t)q * K1 + j1);
              h[o] = (float)(w * nd(rng));
              h[o + 1] = (j1 == 0 && ky == 0) ? 0.f : (float)(w * nd(rng));
            }
          }
      }
      check(sf_vecs_set_host(W.v(), i, h.data()));
      W.p[i] = 0;
    }
    check(sf_vecs_enforce_bcs(W.v(), 0, W.n()));
  }
};

// ====================================================== bifurcations ====
// The drivers of InverseIteration.cpp, FindCriticalPoint.cpp and FindHopf.cpp.
// Their extended states are one Vec whose segments are the state and its
// eigenvector(s): the reference's CriticalPoint (x, v, p) and
// HopfBifurcation (x, v1, v2, theta, p) have exactly the inner product, the
// MulAdd and the EnforceBCs of a Vec of two or three segments with p (and
// q = theta). The state segment evolves by FullEvolve and the eigenvector
// segments by LinearEvolve about the frozen state, one segment at a time.

inline int steps_over(const Context& c, double tau) { return std::max(1, (int)std::ceil(tau / c.p.dt - 1e-9)); }

// FullEvolve (StateVector.cpp:3-84) of segment i of x into segment o of out,
// as Evolve does for all segments: p zeroed, projected, equal steps of at
// most dt, EnforceBCs on the result
inline void EvolveSegment(const Vec& x, int i, double tau, double Ri, Vec& out, int o) {
  Context& c = x.ctx();
  auto t0 = std::chrono::steady_clock::now();
  Solver& s = c.single_solver();
  const int n = steps_over(c, tau);
  s.set_dt(tau / n);
  s.set_ri(0, Ri);
  if (&out != &x || o != i) check(sf_vecs_copy(out.v(), o, x.v(), i));
  check(sf_vecs_zero_pressure(out.v(), o, 1));
  check(sf_vecs_to_run(out.v(), o, s.h(), 0, 1));
  check(sf_prepare(s.h()));
  check(sf_step(s.h(), n));
  check(sf_vecs_from_run(out.v(), o, s.h(), 0, 1));
  check(sf_vecs_enforce_bcs(out.v(), o, 1));
  check(sf_vecs_synchronize(out.v()));
  c.evolutions += 1;
  c.evolve_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// LinearEvolve (StateVector.cpp:107-156): segment id of d advanced over tau
// by TimeStepLinear about the frozen base segment ia of `about`
// (SetBackground, IMEXRK.h:334-352), into segment o of out. The steps are
// those of EvolveSegment (the reference fixes deltaT = 0.01 here).
inline void LinearEvolveSegment(const Vec& about, int ia, const Vec& d, int id, double tau, double Ri, Vec& out,
                                int o) {
  Context& c = about.ctx();
  auto t0 = std::chrono::steady_clock::now();
  Solver& s = c.linear_solver();
  const int n = steps_over(c, tau);
  s.set_dt(tau / n);
  s.set_ri(0, Ri);
  void* base = nullptr;
  check(sf_vecs_device(about.v(), ia, &base));
  check(sf_set_base_device(s.h(), 0, base));
  if (&out != &d || o != id) check(sf_vecs_copy(out.v(), o, d.v(), id));
  check(sf_vecs_zero_pressure(out.v(), o, 1));
  check(sf_vecs_to_run(out.v(), o, s.h(), 0, 1));
  check(sf_prepare(s.h()));
  check(sf_step_linear(s.h(), n));
  check(sf_vecs_from_run(out.v(), o, s.h(), 0, 1));
  check(sf_vecs_enforce_bcs(out.v(), o, 1));
  check(sf_vecs_synchronize(out.v()));
  c.evolutions += 1;
  c.evolve_seconds += std::chrono::duration<double>(std::chrono::steady_clock::now() - t0).count();
}

// CopyToSolver, FilterAll, PopulateNodalVariables, RemoveDivergence(0),
// CopyFromSolver of segment i (the projection Rescale brackets its scaling
// with, StateVector.cpp:189-226); p is zeroed
inline void ProjectSegment(Vec& x, int i) {
  Solver& s = x.ctx().single_solver();
  check(sf_vecs_zero_pressure(x.v(), i, 1));
  check(sf_vecs_to_run(x.v(), i, s.h(), 0, 1));
  check(sf_prepare(s.h()));
  check(sf_vecs_from_run(x.v(), i, s.h(), 0, 1));
}

// StateVector::Rescale (StateVector.cpp:189-226) of segment i to `energy`
// (Energy = Dot / 2, StateVector.h:141-144)
inline void RescaleSegment(Vec& x, int i, double energy) {
  ProjectSegment(x, i);
  const double e = 0.5 * SegmentDot(x, x, i);
  check(sf_vecs_scale(x.v(), i, e != 0.0 ? std::sqrt(energy / e) : 0.0, 1));
  ProjectSegment(x, i);
}

// ddx of u1, u2, u3, b of segment i into segment o of out (i kx on every
// kept mode m = q K1 + j1, kx = 2 pi j1 / L1); p zero
inline void DdxSegment(const Vec& x, int i, Vec& out, int o) {
  const Params& P = x.ctx().p;
  const int K1 = P.N1 / 3, K2 = P.N2 > 1 ? 2 * (P.N2 / 3) - 1 : 1;
  const int plane = (K1 * K2 + 15) / 16 * 16;
  const size_t n = (size_t)5 * P.N3 * plane;
  std::vector<float> h(2 * n);
  x.get_segment_host(i, h.data());
  const double two_pi = 2.0 * std::acos(-1.0);
  for (int f = 0; f < 5; f++)
    for (int t = 0; t < P.N3; t++)
      for (int m = 0; m < plane; m++) {
        float* z = h.data() + 2 * (((size_t)f * P.N3 + t) * plane + m);
        if (f == 4 || m >= K1 * K2) {
          z[0] = z[1] = 0.f;
          continue;
        }
        const float kx = (float)(two_pi * (m % K1) / P.L1);
        const float re = z[0], im = z[1];
        z[0] = -kx * im;
        z[1] = kx * re;
      }
  out.set_segment_host(o, h.data());
}

// FindCriticalPoint (FindCriticalPoint.cpp:110-150): unknowns x (segment 0),
// v (segment 1) and p = Ri; F = (Phi_T(x) - x, L_T(x) v - v, Energy(v) -
// weight), L_T(x) the evolution linearised about the frozen x. The
// constraints take the component along ddx x (the shift symmetry) and the
// mean of u1 and b out of v and rescale it to the weight. Every evaluation
// sets the Ri of the inner products to p, as the reference sets flowParams.Ri.
class CriticalPointNK : public NewtonKrylov {
 public:
  CriticalPointNK(const NKOptions& o, double T, double weight) : NewtonKrylov(o), T_(T), weight_(weight) {}
  Vec EvalFunction(const Vec& at) override {
    Context& c = at.ctx();
    c.p.Ri = at.p;
    Vec r(at);
    EvolveSegment(at, 0, T_, at.p, r, 0);
    LinearEvolveSegment(at, 0, at, 1, T_, at.p, r, 1);
    r.MulAdd(-1.0, at);
    r.p = 0.5 * SegmentDot(at, at, 1) - weight_;
    r.q = 0;
    return r;
  }
  void EnforceConstraints(Vec& at) override {
    Context& c = at.ctx();
    c.p.Ri = at.p;
    Vec ps(at);
    DdxSegment(at, 0, ps, 0);
    const double n2 = SegmentDot(ps, ps, 0);
    if (n2 != 0) {
      double d = 0;
      check(sf_vecs_dots(at.v(), 1, 1, ps.v(), 0, c.p.Ri, &d));
      check(sf_vecs_axpy(at.v(), 1, -d / n2, ps.v(), 0, 1));
    }
    check(sf_vecs_remove_average(at.v(), 1, 0, c.p.L3));
    check(sf_vecs_remove_average(at.v(), 1, 3, c.p.L3));
    RescaleSegment(at, 1, weight_);
  }

 private:
  double T_, weight_;
};

// FindHopf (FindHopf.cpp:4-57): unknowns x, v1, v2 (segments 0, 1, 2),
// q = theta and p = Ri; F = (Phi_T(x) - x, L v1 - cos(theta) v1 + sin(theta)
// v2, L v2 - sin(theta) v1 - cos(theta) v2, v1.A - 1, v2.A), A the first
// eigenvector of the initial guess (segment 0 of `A`). The constraint turns
// (v1, v2) in their plane so that v1.A = 1 and v2.A = 0.
class HopfNK : public NewtonKrylov {
 public:
  HopfNK(const NKOptions& o, double T, const Vec& A) : NewtonKrylov(o), T_(T), A_(A) {}
  Vec EvalFunction(const Vec& at) override {
    Context& c = at.ctx();
    c.p.Ri = at.p;
    Vec r(at);
    EvolveSegment(at, 0, T_, at.p, r, 0);
    LinearEvolveSegment(at, 0, at, 1, T_, at.p, r, 1);
    LinearEvolveSegment(at, 0, at, 2, T_, at.p, r, 2);
    const double cs = std::cos(at.q), sn = std::sin(at.q);
    check(sf_vecs_axpy(r.v(), 0, -1.0, at.v(), 0, 1));
    check(sf_vecs_axpy(r.v(), 1, -cs, at.v(), 1, 1));
    check(sf_vecs_axpy(r.v(), 1, sn, at.v(), 2, 1));
    check(sf_vecs_axpy(r.v(), 2, -sn, at.v(), 1, 1));
    check(sf_vecs_axpy(r.v(), 2, -cs, at.v(), 2, 1));
    r.EnforceBCs();
    r.q = ADot(at, 1) - 1.0;
    r.p = ADot(at, 2);
    return r;
  }
  void EnforceConstraints(Vec& at) override {
    at.ctx().p.Ri = at.p;
    const double a1 = ADot(at, 1), a2 = ADot(at, 2);
    const double th = std::atan2(-a2, a1);
    const double r = 1.0 / (std::cos(th) * a1 - std::sin(th) * a2);
    Vec old(at);
    // v1 <- r cos v1 - r sin v2, v2 <- r sin v1 + r cos v2 (the old v1, v2)
    check(sf_vecs_lincomb(at.v(), 1, r * std::cos(th), -r * std::sin(th), old.v(), 2, 1));
    check(sf_vecs_lincomb(at.v(), 2, r * std::cos(th), r * std::sin(th), old.v(), 1, 1));
  }
  double ADot(const Vec& at, int seg) const {
    double d = 0;
    check(sf_vecs_dots(at.v(), seg, 1, A_.v(), 0, at.ctx().p.Ri, &d));
    return d;
  }

 private:
  double T_;
  Vec A_;
};

// The GMRES least-squares problem min |beta e_0 - H y| over the columns of the
// Hessenberg matrix H received so far, kept in QR form by Givens rotations:
// add() takes column k-1 (rows 0..k) and returns the relative residual of
// the k-column problem, solve() its minimiser. For H of full column rank
// this is the minimiser the reference computes by an SVD of H
// (InverseIteration.cpp:86-104).
class GivensLS {
 public:
  explicit GivensLS(double beta) : beta_(beta), g_(1, beta) {}
  double add(std::vector<double> h) {
    const int k = (int)R_.size() + 1;   // h has k + 1 entries
    for (int j = 0; j < k - 1; j++) {   // the earlier rotations
      const double a = h[j], b = h[j + 1];
      h[j] = cs_[j] * a + sn_[j] * b;
      h[j + 1] = -sn_[j] * a + cs_[j] * b;
    }
    const double r = std::hypot(h[k - 1], h[k]);
    const double c = r > 0 ? h[k - 1] / r : 1.0, sn = r > 0 ? h[k] / r : 0.0;
    cs_.push_back(c);
    sn_.push_back(sn);
    h[k - 1] = r;
    h[k] = 0;
    g_.push_back(-sn * g_[k - 1]);
    g_[k - 1] = c * g_[k - 1];
    R_.push_back(h);
    return std::fabs(g_[k]) / beta_;
  }
  std::vector<double> solve() const {   // back substitution R y = g
    const int n = (int)R_.size();
    std::vector<double> y(n, 0.0);
    for (int i = n - 1; i >= 0; i--) {
      double s = g_[i];
      for (int j = i + 1; j < n; j++) s -= R_[j][i] * y[j];
      y[i] = R_[i][i] != 0 ? s / R_[i][i] : 0.0;
    }
    return y;
  }
  double last_pivot() const { return R_.empty() ? 0.0 : R_.back()[R_.size() - 1]; }

 private:
  double beta_;
  std::vector<double> g_, cs_, sn_;
  std::vector<std::vector<double>> R_;   // reduced columns
};

struct InverseIterationResult {
  std::vector<double> mu;         // |L b| / |b| before each solve (muApprox)
  std::vector<double> residual;   // |L b - muApprox b| with |b| = 1
  std::vector<int> krylov;        // GMRES vectors of each solve
};

// InverseIteration (InverseIteration.cpp:1-124) about the frozen state
// `about` (one segment): each iteration reports muApprox = |L b| / |b| and
// the residual |L b - muApprox b|, solves (L - mu) y = b by GMRES (modified
// Gram-Schmidt, EnforceBCs on each basis vector) to relative residual eps
// with at most K vectors, and takes b = y / |y|. The reference solves each
// least-squares problem by an SVD of the Hessenberg block; Givens rotations
// give the same minimiser (the block has full rank while the basis grows)
// at O(k) work per vector instead of O(k^3).
inline InverseIterationResult InverseIteration(const Vec& about, Vec& b, double T, double mu, double eps, int iters,
                                               int K) {
  Context& c = about.ctx();
  const double Ri = c.p.Ri;
  InverseIterationResult out;
  b *= 1.0 / b.Norm();
  for (int it = 0; it < iters; it++) {
    Vec bT(b);
    LinearEvolveSegment(about, 0, b, 0, T, Ri, bT, 0);
    const double ma = bT.Norm() / b.Norm();
    bT.MulAdd(-ma, b);
    out.mu.push_back(ma);
    out.residual.push_back(bT.Norm());
    if (verbose()) std::fprintf(stderr, "Inverse iteration %d: eigenvalue %.8f, residual %.3e\n", it, ma, bT.Norm());
    std::vector<std::unique_ptr<Vec>> q;
    q.emplace_back(new Vec(b));
    q[0]->EnforceBCs();
    const double beta = q[0]->Norm();
    *q[0] *= 1.0 / beta;
    GivensLS ls(beta);   // the Hessenberg columns, reduced as they arrive
    int used = 0;
    for (int k = 1; k < K; k++) {
      q.emplace_back(new Vec(*q[k - 1]));
      LinearEvolveSegment(about, 0, *q[k - 1], 0, T, Ri, *q[k], 0);
      q[k]->MulAdd(-mu, *q[k - 1]);
      std::vector<double> h(k + 1, 0.0);
      for (int j = 0; j < k; j++) {
        h[j] = q[j]->Dot(*q[k]);
        q[k]->MulAdd(-h[j], *q[j]);
      }
      h[k] = q[k]->Norm();
      if (h[k] > 0) *q[k] *= 1.0 / h[k];
      q[k]->EnforceBCs();
      used = k;
      const double res = ls.add(h);
      if (verbose() && k % 10 == 0) std::fprintf(stderr, "GMRES STEP %d, RESIDUAL: %.3e\n", k, res);
      if (res < eps || !(ls.last_pivot() > 0)) break;
    }
    out.krylov.push_back(used);
    if (used == 0) continue;   // no vector to solve with (K < 2): b stays
    const std::vector<double> y = ls.solve();   // b = sum y_k q_k
    b.Zero();
    for (int k = 0; k < used; k++) b.MulAdd(y[k], *q[k]);
    b *= 1.0 / b.Norm();
  }
  return out;
}

}  // namespace stratiflow
