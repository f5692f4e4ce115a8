// C entry points of the host-side drivers (stratiflow.hpp), used by the
// Python front end and the benchmarks:
//   sfh_newton_fixed     BasicNewtonKrylov (BasicNewtonKrylov.h): Phi_T(x) = x
//   sfh_periodic_orbit   FindPeriodic (FindPeriodic.cpp): Phi_T(x) = x, T unknown
//   sfh_arclength        one corrector of PseudoArclength (PseudoArclength.cpp:63-68)
//   sfh_arnoldi          BasicArnoldi (Arnoldi.h:15-226): eigenvalues of the linearised evolution
//   sfh_linear_evolve    LinearEvolve (StateVector.cpp:107-156) about a frozen state
//   sfh_inverse_iteration  InverseIteration (InverseIteration.cpp)
//   sfh_critical_point   FindCriticalPoint (FindCriticalPoint.cpp)
//   sfh_find_hopf        FindHopf (FindHopf.cpp)
// States cross this interface in the kept layout of include/stratiflow_b200.h,
// M consecutive states (the shooting segments).
#include <cstring>
#include <exception>
#include <string>

#include "stratiflow.hpp"

using namespace stratiflow;

namespace {

thread_local std::string g_host_err;

Params params_from(const double* a) {
  Params p;
  p.N1 = (int)a[0]; p.N2 = (int)a[1]; p.N3 = (int)a[2];
  p.L1 = a[3]; p.L2 = a[4]; p.L3 = a[5]; p.Re = a[6]; p.Pr = a[7]; p.Ri = a[8]; p.dt = a[9];
  p.background = (int)a[10];
  return p;
}

NKOptions options_from(const double* o) {
  NKOptions n;
  if (!o) return n;
  n.max_newton = (int)o[0];
  n.krylov = (int)o[1];
  n.target = o[2];
  n.gmres_tol = o[3];
  n.Delta = o[4];
  n.fd_eps = o[5];
  n.tangent = o[6] == 0.0;   // 0: tangent-linear Jacobian actions, 1: finite differences
  n.precondition = o[8] != 0.0;
  n.relative = o[9] != 0.0;
  return n;
}

// directions per batched Jacobian action of the block solver (opts[7]); 0
// selects the one-direction solver
int block_from(const double* o) { return o ? (int)o[7] : 0; }

size_t kept_elems(const Params& p) {
  const int K1 = p.N1 / 3, K2 = p.N2 > 1 ? 2 * (p.N2 / 3) - 1 : 1;
  const int plane = (K1 * K2 + 15) / 16 * 16;
  return (size_t)5 * p.N3 * plane;   // complex values of one state
}

void load(Vec& x, const float* host, const Params& p) {
  for (int i = 0; i < x.M(); i++) x.set_segment_host(i, host + 2 * kept_elems(p) * i);
}
void store(const Vec& x, float* host, const Params& p) {
  for (int i = 0; i < x.M(); i++) x.get_segment_host(i, host + 2 * kept_elems(p) * i);
}

// stats layout: [0] newton iterations, [1] Jacobian actions, [2] batched
// integrations, [3] seconds, [4] seconds inside integrations, [5] final
// relative residual, [6] converged, [7] number of residuals n, [8..8+n)
// residuals, then per Newton step i < n-1 its relative GMRES residual and
// its Jacobian actions
void write_stats(const NKStats& s, double* out, int cap) {
  if (!out || cap < 8) return;
  out[0] = s.newton_iterations;
  out[1] = s.krylov_vectors;
  out[2] = (double)s.evolutions;
  out[3] = s.seconds;
  out[4] = s.evolve_seconds;
  out[5] = s.residual;
  out[6] = s.converged ? 1.0 : 0.0;
  const int n = std::min((int)s.residuals.size(), cap - 8);
  out[7] = n;
  for (int i = 0; i < n; i++) out[8 + i] = s.residuals[i];
  const int ng = std::min((int)s.gmres_residuals.size(), (cap - 8 - n) / 2);
  for (int i = 0; i < ng; i++) {
    out[8 + n + 2 * i] = s.gmres_residuals[i];
    out[8 + n + 2 * i + 1] = s.gmres_vectors[i];
  }
}

// BasicNewtonKrylov with the constraints of PseudoArclength (phase, averages)
class FixedPoint : public NewtonKrylov {
 public:
  FixedPoint(const NKOptions& o, double T, bool constrain) : NewtonKrylov(o), T_(T), constrain_(constrain) {}
  Vec EvalFunction(const Vec& at) override {
    Vec phi(at);
    Evolve(at, T_ / at.M(), at.ctx().p.Ri, phi);
    Vec r = ShootingResidual(phi, at);
    r.p = 0;
    return r;
  }
  void EnforceConstraints(Vec& at) override {
    if (!constrain_) return;
    at.RemovePhaseShift();
    at.RemoveAverage(0);
    at.RemoveAverage(3);
  }
  // Phi' d_i - d_{i+1}
  Vec EvalDerivative(const Vec& dir) override {
    if (!opt.tangent) return NewtonKrylov::EvalDerivative(dir);
    Vec phi(dir);
    EvolveTangent(*x0_, dir, T_ / dir.M(), dir.ctx().p.Ri, phi);
    Vec r = ShootingResidual(phi, dir);
    r.p = 0;
    return r;
  }

 private:
  double T_;
  bool constrain_;
};

}  // namespace

extern "C" {

const char* sfh_last_error(void) { return g_host_err.c_str(); }

// params: N1,N2,N3,L1,L2,L3,Re,Pr,Ri,dt,background; opts: max_newton, krylov,
// target, gmres_tol, Delta, fd_eps, jacobian (0 tangent-linear, 1 finite
// differences), block (directions per batched Jacobian action; 0: one, which
// also allows multiple shooting, M > 1; >= 1 needs M = 1), precondition (block
// solvers: 1 applies the mean-flow preconditioner), relative (block fixed
// point: 1 makes the x shift an unknown, p the shift)
int sfh_newton_fixed(const double* params, int M, double T, int constrain, const float* guess, const double* opts,
                     float* out, double* stats, int stats_cap) {
  try {
    Params p = params_from(params);
    Context c(p, M);
    Vec x(c);
    load(x, guess, p);
    x.EnforceBCs();
    NKStats s;
    if (block_from(opts) > 0) {
      BlockFixedPoint nk(options_from(opts), block_from(opts), T, constrain != 0);
      if (constrain) nk.EnforceConstraints(x);
      x.p = 0;
      nk.SetReference(x);
      s = nk.Run(x);
    } else {
      FixedPoint nk(options_from(opts), T, constrain != 0);
      if (constrain) nk.EnforceConstraints(x);
      s = nk.Run(x);
    }
    store(x, out, p);
    write_stats(s, stats, stats_cap);
    return 0;
  } catch (const std::exception& e) {
    g_host_err = e.what();
    return -1;
  }
}

int sfh_periodic_orbit(const double* params, int M, double T0, const float* guess, const double* opts, float* out,
                       double* T_out, double* stats, int stats_cap) {
  try {
    Params p = params_from(params);
    Context c(p, M);
    Vec x(c);
    load(x, guess, p);
    x.EnforceBCs();
    x.p = T0;
    NKStats s;
    if (block_from(opts) > 0) {
      BlockPeriodicOrbit nk(options_from(opts), block_from(opts), x);
      s = nk.Run(x);
    } else {
      PeriodicOrbit nk(options_from(opts), x);
      s = nk.Run(x);
    }
    store(x, out, p);
    if (T_out) *T_out = x.p;
    write_stats(s, stats, stats_cap);
    return 0;
  } catch (const std::exception& e) {
    g_host_err = e.what();
    return -1;
  }
}

// One pseudo-arclength corrector: x0 (M states, Ri0) is the last converged
// point, v (M states, v_Ri) the unit tangent in the extended norm, ds the
// step, guess (M states, Ri_guess) the predictor. Writes the converged point.
int sfh_arclength(const double* params, int M, double T, const float* x0, double Ri0, const float* v, double vRi,
                  double ds, const float* guess, double Ri_guess, const double* opts, float* out, double* Ri_out,
                  double* stats, int stats_cap) {
  try {
    Params p = params_from(params);
    Context c(p, M);
    Vec X0(c), V(c), X(c);
    load(X0, x0, p);
    X0.p = Ri0;
    load(V, v, p);
    V.p = vRi;
    load(X, guess, p);
    X.p = Ri_guess;
    X.EnforceBCs();
    NKStats s;
    if (block_from(opts) > 0) {
      BlockPseudoArclength nk(options_from(opts), block_from(opts), X0, V, ds, T);
      nk.EnforceConstraints(X);
      s = nk.Run(X);
    } else {
      PseudoArclength nk(options_from(opts), X0, V, ds, T);
      nk.EnforceConstraints(X);
      s = nk.Run(X);
    }
    store(X, out, p);
    if (Ri_out) *Ri_out = X.p;
    write_stats(s, stats, stats_cap);
    return 0;
  } catch (const std::exception& e) {
    g_host_err = e.what();
    return -1;
  }
}

// The tangent-linear action Phi'(x) dx of the M segments over tau each
int sfh_evolve_tangent(const double* params, int M, double tau, double Ri, const float* x, const float* dx,
                       float* out) {
  try {
    Params p = params_from(params);
    Context c(p, M);
    Vec a(c), d(c), y(c);
    load(a, x, p);
    load(d, dx, p);
    EvolveTangent(a, d, tau, Ri, y);
    store(y, out, p);
    return 0;
  } catch (const std::exception& e) {
    g_host_err = e.what();
    return -1;
  }
}

// Arnoldi (Arnoldi.h, BasicArnoldi) about the state `about` over T: up to
// nev_cap eigenvalues (by decreasing modulus) into ev_re/ev_im, their number
// into *nev_out; the leading eigenvector's real and imaginary parts into
// vec_re/vec_im (kept layout; may be NULL). stats: [0] directions integrated,
// [1] batched integrations, [2] seconds.
int sfh_arnoldi(const double* params, const float* about, double T, int block, int krylov, double tol, int nev,
                unsigned long long seed, double* ev_re, double* ev_im, int nev_cap, int* nev_out, float* vec_re,
                float* vec_im, double* stats) {
  try {
    Params p = params_from(params);
    Context c(p, 1);
    Vec x(c), er(c), ei(c);
    load(x, about, p);
    x.EnforceBCs();
    BlockArnoldi ar(block, krylov, tol, nev, seed);
    ArnoldiResult r = ar.Run(x, T, vec_re ? &er : nullptr, vec_im ? &ei : nullptr);
    const int n = std::min((int)r.eigenvalues.size(), nev_cap);
    for (int i = 0; i < n; i++) {
      ev_re[i] = r.eigenvalues[i].real();
      ev_im[i] = r.eigenvalues[i].imag();
    }
    if (nev_out) *nev_out = n;
    if (vec_re) store(er, vec_re, p);
    if (vec_im) store(ei, vec_im, p);
    if (stats) {
      stats[0] = r.vectors;
      stats[1] = (double)r.integrations;
      stats[2] = r.seconds;
    }
    return 0;
  } catch (const std::exception& e) {
    g_host_err = e.what();
    return -1;
  }
}

// LinearEvolve (StateVector.cpp:107-156): d advanced over T by TimeStepLinear
// about the frozen state `about`, into out (one state each, kept layout)
int sfh_linear_evolve(const double* params, const float* about, const float* d, double T, float* out) {
  try {
    Params p = params_from(params);
    Context c(p, 1);
    Vec a(c), x(c);
    load(a, about, p);
    load(x, d, p);
    LinearEvolveSegment(a, 0, x, 0, T, p.Ri, x, 0);
    store(x, out, p);
    return 0;
  } catch (const std::exception& e) {
    g_host_err = e.what();
    return -1;
  }
}

// InverseIteration (InverseIteration.cpp:1-124) about `about` at the Ri of
// params: b (one state) in and out, normalised; shift mu, GMRES tolerance
// eps, at most `krylov` vectors per solve. hist: [0] iterations n, then n
// eigenvalue estimates, n residuals, n GMRES vector counts.
int sfh_inverse_iteration(const double* params, const float* about, float* b, double T, double mu, double eps,
                          int iters, int krylov, double* hist, int cap) {
  try {
    Params p = params_from(params);
    Context c(p, 1);
    Vec a(c), x(c);
    load(a, about, p);
    load(x, b, p);
    x.EnforceBCs();
    InverseIterationResult r = InverseIteration(a, x, T, mu, eps, iters, krylov);
    store(x, b, p);
    const int n = (int)r.mu.size();
    if (hist && cap >= 1 + 3 * n) {
      hist[0] = n;
      for (int i = 0; i < n; i++) {
        hist[1 + i] = r.mu[i];
        hist[1 + n + i] = r.residual[i];
        hist[1 + 2 * n + i] = r.krylov[i];
      }
    }
    return 0;
  } catch (const std::exception& e) {
    g_host_err = e.what();
    return -1;
  }
}

// FindCriticalPoint (FindCriticalPoint.cpp:110-213): xv = (x, v), two states
// in and out; *Ri the parameter unknown p, in and out. mode 0: the
// constraints, then Newton-Krylov (the reference's main, :203-208); 1: the
// constraints only; 2: F(x, v, Ri) into xv and *Ri.
int sfh_critical_point(const double* params, int mode, double T, double weight, float* xv, double* Ri,
                       const double* opts, double* stats, int cap) {
  try {
    Params p = params_from(params);
    p.Ri = *Ri;
    Context c(p, 2);
    Vec x(c);
    load(x, xv, p);
    x.EnforceBCs();
    x.p = *Ri;
    CriticalPointNK nk(options_from(opts), T, weight);
    if (mode == 2) {
      Vec F = nk.EvalFunction(x);
      store(F, xv, p);
      *Ri = F.p;
      return 0;
    }
    nk.EnforceConstraints(x);
    if (mode == 0) {
      NKStats st = nk.Run(x);
      write_stats(st, stats, cap);
    }
    store(x, xv, p);
    *Ri = x.p;
    return 0;
  } catch (const std::exception& e) {
    g_host_err = e.what();
    return -1;
  }
}

// FindHopf (FindHopf.cpp:4-101): xv = (x, v1, v2), three states in and out;
// *Ri (p) and *theta (the eigenvalue's argument) in and out. v1 and v2 are
// first divided by |v1| and A is the resulting v1 (:88-93). mode 0: the
// constraints, then Newton-Krylov; 1: the constraints only; 2: F into xv,
// *theta (v1.A - 1) and *Ri (v2.A).
int sfh_find_hopf(const double* params, int mode, double T, float* xv, double* Ri, double* theta,
                  const double* opts, double* stats, int cap) {
  try {
    Params p = params_from(params);
    p.Ri = *Ri;
    Context c(p, 3);
    Vec x(c);
    load(x, xv, p);
    x.EnforceBCs();
    x.p = *Ri;
    x.q = *theta;
    const double n1 = std::sqrt(SegmentDot(x, x, 1));
    if (n1 > 0) check(sf_vecs_scale(x.v(), 1, 1.0 / n1, 2));
    Vec A(c);
    check(sf_vecs_copy(A.v(), 0, x.v(), 1));
    HopfNK nk(options_from(opts), T, A);
    if (mode == 2) {
      Vec F = nk.EvalFunction(x);
      store(F, xv, p);
      *Ri = F.p;
      *theta = F.q;
      return 0;
    }
    nk.EnforceConstraints(x);
    if (mode == 0) {
      NKStats st = nk.Run(x);
      write_stats(st, stats, cap);
    }
    store(x, xv, p);
    *Ri = x.p;
    *theta = x.q;
    return 0;
  } catch (const std::exception& e) {
    g_host_err = e.what();
    return -1;
  }
}

// FullEvolve with the adaptive time step on an existing solver (all its runs)
int sfh_full_evolve(sf_solver* solver, double T, double target_cfl, int interval, double* stats) {
  try {
    int nrun = 0;
    check(sf_get_runs(solver, &nrun));
    FullEvolveAdaptive(solver, nrun, T, target_cfl, interval, stats);
    return 0;
  } catch (const std::exception& e) {
    g_host_err = e.what();
    return -1;
  }
}

// Evolve M segments over T/M each (for the callers' own experiments)
int sfh_evolve(const double* params, int M, double tau, double Ri, const float* in, float* out) {
  try {
    Params p = params_from(params);
    Context c(p, M);
    Vec x(c), y(c);
    load(x, in, p);
    Evolve(x, tau, Ri, y);
    store(y, out, p);
    return 0;
  } catch (const std::exception& e) {
    g_host_err = e.what();
    return -1;
  }
}

}  // extern "C"
