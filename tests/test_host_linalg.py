"""CPU tests of the host drivers' FP64 dense numerics (stratiflow_b200/host/
stratiflow.hpp): the eigenvalues of the Arnoldi Hessenberg matrices, their
eigenvectors, the Householder least squares of the GMRES convergence check
and the one-sided Jacobi SVD of the hookstep, against numpy/LAPACK on seeded
random matrices. The header is compiled into a small program with g++ (its
device entry points are declared but never called)."""
import os
import subprocess
import tempfile

import numpy as np
import pytest

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))

PROG = r"""
#include <cstdio>
#include <vector>
#include "stratiflow.hpp"
using namespace stratiflow;
int main() {
  int n, m;
  // eigenvalues + eigenvector of the leading one
  if (std::scanf("%d", &n) != 1) return 1;
  std::vector<double> A((size_t)n * n);
  for (auto& a : A) if (std::scanf("%lf", &a) != 1) return 1;
  auto ev = eigenvalues(A, n);
  std::printf("%zu\n", ev.size());
  for (auto& e : ev) std::printf("%.17g %.17g\n", e.real(), e.imag());
  size_t best = 0;
  for (size_t i = 1; i < ev.size(); i++) if (std::abs(ev[i]) > std::abs(ev[best])) best = i;
  auto v = eigenvector(A, n, ev[best]);
  std::printf("%.17g %.17g\n", ev[best].real(), ev[best].imag());
  for (auto& e : v) std::printf("%.17g %.17g\n", e.real(), e.imag());
  // least squares and SVD of an m x n matrix
  if (std::scanf("%d %d", &m, &n) != 2) return 1;
  std::vector<double> B((size_t)m * n), b(m), y;
  for (auto& a : B) if (std::scanf("%lf", &a) != 1) return 1;
  for (auto& a : b) if (std::scanf("%lf", &a) != 1) return 1;
  double r = lsq_householder(B, m, n, b, y);
  std::printf("%.17g\n", r);
  for (double t : y) std::printf("%.17g\n", t);
  std::vector<double> U, S, V;
  svd(B, m, n, U, S, V);
  for (double t : S) std::printf("%.17g\n", t);
  return 0;
}
"""


@pytest.fixture(scope="module")
def prog():
    d = tempfile.mkdtemp()
    src, exe = os.path.join(d, "t.cpp"), os.path.join(d, "t")
    open(src, "w").write(PROG)
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "stratiflow_b200", "host"),
                    "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
    return exe


@pytest.mark.parametrize("n,seed", [(12, 1), (40, 2), (96, 3)])
def test_eigen_lsq_svd_against_lapack(prog, n, seed):
    rng = np.random.default_rng(seed)
    A = rng.normal(size=(n, n))
    A[np.tril_indices(n, -3)] *= 0.1     # block-Hessenberg-like decay, as from Arnoldi
    m, k = n + 8, n
    B = rng.normal(size=(m, k))
    b = rng.normal(size=m)
    inp = f"{n}\n" + " ".join(f"{v:.17g}" for v in A.ravel()) + f"\n{m} {k}\n" + \
        " ".join(f"{v:.17g}" for v in B.ravel()) + "\n" + " ".join(f"{v:.17g}" for v in b) + "\n"
    out = subprocess.run([prog], input=inp, capture_output=True, text=True, check=True).stdout.split("\n")
    cnt = int(out[0])
    ev = np.array([complex(*map(float, l.split())) for l in out[1:1 + cnt]])
    ref = np.linalg.eigvals(A)
    # every eigenvalue matched to LAPACK's (sorted by nearest)
    for e in ref:
        assert np.min(np.abs(ev - e)) <= 1e-9 * np.max(np.abs(ref))
    lam = complex(*map(float, out[1 + cnt].split()))
    v = np.array([complex(*map(float, l.split())) for l in out[2 + cnt:2 + cnt + n]])
    assert np.linalg.norm(A @ v - lam * v) <= 1e-8 * np.linalg.norm(A, 2)
    pos = 2 + cnt + n
    r = float(out[pos])
    y = np.array([float(v) for v in out[pos + 1:pos + 1 + k]])
    yref, res, *_ = np.linalg.lstsq(B, b, rcond=None)
    assert np.allclose(y, yref, rtol=1e-8, atol=1e-10)
    assert abs(r - np.linalg.norm(B @ yref - b)) <= 1e-9 * np.linalg.norm(b)
    S = np.sort(np.array([float(v) for v in out[pos + 1 + k:pos + 1 + 2 * k]]))[::-1]
    assert np.allclose(S, np.linalg.svd(B, compute_uv=False), rtol=1e-10)


GIVENS = r"""
#include <cstdio>
#include <vector>
#include "stratiflow.hpp"
using namespace stratiflow;
int main() {
  int n;
  double beta;
  if (std::scanf("%d %lf", &n, &beta) != 2) return 1;
  GivensLS ls(beta);
  for (int k = 1; k <= n; k++) {
    std::vector<double> h(k + 1);
    for (auto& a : h) if (std::scanf("%lf", &a) != 1) return 1;
    std::printf("%.17g\n", ls.add(h));
  }
  for (double t : ls.solve()) std::printf("%.17g\n", t);
  return 0;
}
"""


def test_givens_least_squares_matches_lstsq():
    """GivensLS (InverseIteration's GMRES least squares): after each new
    Hessenberg column the relative residual of min |beta e_0 - H y| and, at
    the end, the minimiser agree with LAPACK's least squares (which the
    reference's SVD solve equals for H of full rank) to 1e-10."""
    d = tempfile.mkdtemp()
    src, exe = os.path.join(d, "g.cpp"), os.path.join(d, "g")
    open(src, "w").write(GIVENS)
    subprocess.run(["g++", "-O2", "-std=c++17", "-I", os.path.join(ROOT, "stratiflow_b200", "host"),
                    "-I", os.path.join(ROOT, "include"), src, "-o", exe], check=True)
    rng = np.random.default_rng(7)
    n, beta = 24, 1.7
    H = np.triu(rng.standard_normal((n + 1, n)), -1)   # upper Hessenberg
    feed = [f"{n} {beta:.17g}"]
    for k in range(1, n + 1):
        feed.append(" ".join(f"{v:.17g}" for v in H[:k + 1, k - 1]))
    out = subprocess.run([exe], input="\n".join(feed), capture_output=True, text=True, check=True).stdout.split()
    vals = np.array([float(v) for v in out])
    res, y = vals[:n], vals[n:]
    e0 = np.zeros(n + 1)
    e0[0] = beta
    for k in range(1, n + 1):
        yk, *_ = np.linalg.lstsq(H[:k + 1, :k], e0[:k + 1], rcond=None)
        want = np.linalg.norm(H[:k + 1, :k] @ yk - e0[:k + 1]) / beta
        assert abs(res[k - 1] - want) <= 1e-10 * max(1.0, want), k
    ywant, *_ = np.linalg.lstsq(H, e0, rcond=None)
    assert np.linalg.norm(y - ywant) <= 1e-10 * np.linalg.norm(ywant)
