"""Literal dense-matrix transcription of jeremypparker/Stratiflow's IMEX-RK step.

TEST INFRASTRUCTURE ONLY (imported by ``tests/`` and by the fixture
generator in ``tests/golden/``). It pins the banded C++ oracle
(``sf_oracle.cpp``): where the oracle applies 2- and 3-point bands, this
module builds the full N3 x N3 matrices element by element exactly as the
reference does and multiplies them, uses numpy's FFT in place of FFTW, and
keeps the reference's class structure and method names so that each step
can be read against the C++ source:

  VerticalPoints/...Fractional/dz/dzFractional   Field.cpp:3-83
  Vertical(Second)DerivativeMatrix, Reinterpolation*, k, KVector
                                                  Differentiation.cpp:6-160
  Neumannify / Dirichlify                         Differentiation.h:17-59
  Tridiagonal::compute / solve                    Tridiagonal.h:14-53
  ToModal / ToNodal / Filter / ParallelPerStack   Field.h:734-769, 965-1021, 1129-1166
  product helpers                                 Stratiflow.h:112-164
  IMEXRK (constructor, TimeStep, TimeStepLinear, RemoveDivergence,
  CrankNicolson, FinishRHS, ExplicitRK, BuildRHS, BuildRHSLinear,
  UpdateForTimestep, KE, PE)                      IMEXRK.h:37-545, IMEXRK.cpp:8-258
  InnerProd / IntegrateVertically                 Integration.h:5-35, 282-311

It runs in float64 (the reference's -DDOUBLE build) and is meant for grids
of a few thousand points. The one deliberate generalisation is shared with
the oracle: BuildRHS's ``rB -= ReinterpolateDirichlet(u3)`` (IMEXRK.cpp:147)
is multiplied by a per-level profile ``dBdz`` (all ones = the reference).
"""
from __future__ import annotations

import numpy as np

NEU, DIR = 0, 1


# ------------------------------------------------------------ Field.cpp ----
def vertical_points(L, N):
    cs = 2.0
    assert N % 4 == 0
    # Eigen LinSpaced(N-1, -1, 1): low + i*step with the last point exactly high
    step = 2.0 / (N - 2)
    x = np.array([(-1.0 + i * step) if i < N - 2 else 1.0 for i in range(N - 1)])
    ret = np.zeros(N)
    ret[1:] = L * (cs * x ** 7 + x) / (cs + 1)
    offset = (ret[1] + ret[2]) / 2
    ret[1:] *= -L / offset
    return ret


def vertical_points_fractional(L, N):
    z = vertical_points(L, N)
    ret = np.zeros(N)
    ret[1:N - 1] = 0.5 * (z[1:N - 1] + z[2:])
    ret[0] = 2 * ret[1] - ret[2]
    ret[N - 1] = 2 * ret[N - 2] - ret[N - 3]
    return ret


def dz(L, N):
    zf = vertical_points_fractional(L, N)
    ret = np.zeros(N)
    ret[1:] = zf[1:] - zf[:-1]
    return ret


def dz_fractional(L, N):
    z = vertical_points(L, N)
    ret = np.zeros(N)
    ret[1:N - 1] = z[2:] - z[1:N - 1]
    ret[N - 1] = ret[N - 2]
    ret[0] = ret[1]
    return ret


# ------------------------------------------------- Differentiation.cpp ----
def vertical_second_derivative_matrix(L, N, bc):
    D = np.zeros((N, N))
    DY, DYF = dz(L, N), dz_fractional(L, N)
    if bc == NEU:
        for j in range(1, N - 1):
            D[j, j - 1] = 1 / DY[j] / DYF[j]
            D[j, j] = -1 / DY[j] / DYF[j] - 1 / DY[j + 1] / DYF[j]
            D[j, j + 1] = 1 / DY[j + 1] / DYF[j]
    else:
        for j in range(2, N - 1):
            D[j, j - 1] = 1 / DYF[j - 1] / DY[j]
            D[j, j] = -1 / DYF[j - 1] / DY[j] - 1 / DYF[j] / DY[j]
            D[j, j + 1] = 1 / DYF[j] / DY[j]
    return D


def vertical_derivative_matrix(L, N, bc):
    D = np.zeros((N, N))
    DY, DYF = dz(L, N), dz_fractional(L, N)
    if bc == NEU:
        for j in range(2, N):
            D[j, j - 1] = -1 / DY[j]
            D[j, j] = 1 / DY[j]
    else:
        for j in range(1, N):
            D[j, j] = -1 / DYF[j]
            if j + 1 < N:  # the reference writes D(N-1, N) outside the matrix
                D[j, j + 1] = 1 / DYF[j]
    return D


def _set_diag(D, offset, values):
    n = D.shape[0]
    for t, v in enumerate(values):
        i = t - offset if offset < 0 else t
        j = t if offset < 0 else t + offset
        D[i if offset >= 0 else t - offset, j] = v


def neumann_reinterpolation_full(L, N):
    diff, frac = dz(L, N), dz_fractional(L, N)
    D = np.zeros((N, N))
    for j in range(1, N):  # diagonal(-1) = frac.tail(N-1) / (2 diff.tail(N-1))
        D[j, j - 1] = frac[j] / (2 * diff[j])
    for j in range(1, N):  # diagonal(0).tail(N-1) = frac.head(N-1) / (2 diff.tail(N-1))
        D[j, j] = frac[j - 1] / (2 * diff[j])
    return D


def neumann_reinterpolation_bar(L, N):
    D = np.zeros((N, N))
    for j in range(1, N):
        D[j, j - 1] = 0.5
        D[j, j] = 0.5
    return D


def neumann_reinterpolation_tilde(L, N):
    diff, frac = dz(L, N), dz_fractional(L, N)
    D = np.zeros((N, N))
    for j in range(1, N):  # diagonal(-1) = frac.head(N-1) / (2 diff.tail(N-1))
        D[j, j - 1] = frac[j - 1] / (2 * diff[j])
    for j in range(1, N):  # diagonal(0).tail(N-1) = frac.tail(N-1) / (2 diff.tail(N-1))
        D[j, j] = frac[j] / (2 * diff[j])
    return D


def dirichlet_reinterpolation(L, N):
    D = np.zeros((N, N))
    for j in range(N):
        D[j, j] = 0.5
    for j in range(N - 1):
        D[j, j + 1] = 0.5
    return D


def k_of(n):
    if n == 1:
        return np.zeros(1)
    return np.concatenate([np.arange(0, n // 3 + 1, dtype=float),
                           np.zeros(n - 2 * (n // 3) - 1),
                           np.arange(-(n // 3), 0, dtype=float)])


def kvector(L, N, dimension):
    ret = 1j * (k_of(N) * (2 * np.pi) / L)
    return ret if dimension == 2 else ret[: N // 2 + 1]


def fourier_second_derivative(L, N, dimension):
    kv = kvector(L, N, dimension)
    return (kv * kv).real


def neumannify(M):
    N = M.shape[0]
    M[0, 0] = 1; M[0, 1] = 0; M[0, 2] = 0
    M[1, 0] = 0; M[1, 1] = 1; M[1, 2] = -1
    M[N - 2, N - 3] = 1; M[N - 2, N - 2] = -1; M[N - 2, N - 1] = 0
    M[N - 1, N - 3] = 0; M[N - 1, N - 2] = 0; M[N - 1, N - 1] = 1


def dirichlify(M):
    N = M.shape[0]
    M[0, 0] = 1; M[0, 1] = 0; M[0, 2] = 0
    M[1, 0] = 0; M[1, 1] = 1; M[1, 2] = 0
    M[2, 1] = 0; M[2, 2] = 1; M[2, 3] = 0
    M[N - 1, N - 2] = 0; M[N - 1, N - 1] = 1; M[N - 1, N - 3] = 0
    M[N - 2, N - 2] = 1; M[N - 2, N - 1] = 0; M[N - 2, N - 3] = 0; M[N - 2, N - 4] = 0


# ------------------------------------------------------- Tridiagonal.h ----
class Tridiagonal:
    def compute(self, A):
        N = A.shape[0]
        self.a = np.zeros(N); self.b = np.zeros(N); self.C = np.zeros(N)
        self.a[1:] = np.diag(A, -1)
        self.b[:] = np.diag(A, 0)
        self.C[:N - 1] = np.diag(A, 1)
        self.C[0] = self.C[0] / self.b[0]
        for j in range(1, N - 1):
            self.C[j] = self.C[j] / (self.b[j] - self.a[j] * self.C[j - 1])

    def solve(self, d):
        N = d.shape[0]
        a, b, C = self.a, self.b, self.C
        D = np.zeros(N, dtype=d.dtype)
        x = np.zeros(N, dtype=d.dtype)
        D[0] = d[0] / b[0]
        for j in range(1, N):
            D[j] = (d[j] - a[j] * D[j - 1]) / (b[j] - a[j] * C[j - 1])
        x[N - 1] = D[N - 1]
        for j in range(N - 2, -1, -1):
            x[j] = D[j] - C[j] * x[j + 1]
        return x


# -------------------------------------------------------------- IMEXRK ----
class IMEXRK:
    beta = (1.0, 25.0 / 8.0, 9.0 / 4.0)
    zeta = (0.0, -17.0 / 8.0, -5.0 / 4.0)

    def __init__(self, N1, N2, N3, L1, L2, L3, Re, Ri, Pr, dt):
        self.N1, self.N2, self.N3 = N1, N2, N3
        self.M1 = N1 // 2 + 1
        self.L1, self.L2, self.L3, self.Re, self.Ri, self.Pr = L1, L2, L3, Re, Ri, Pr
        self.dim3 = N2 > 1
        self.deltaT = dt
        L = L3
        self.D2N = vertical_second_derivative_matrix(L, N3, NEU)
        self.D2D = vertical_second_derivative_matrix(L, N3, DIR)
        self.DzN = vertical_derivative_matrix(L, N3, NEU)   # Neumann -> Dirichlet
        self.DzD = vertical_derivative_matrix(L, N3, DIR)   # Dirichlet -> Neumann
        self.Rfull = neumann_reinterpolation_full(L, N3)
        self.Rbar = neumann_reinterpolation_bar(L, N3)
        self.Rtilde = neumann_reinterpolation_tilde(L, N3)
        self.Rdir = dirichlet_reinterpolation(L, N3)
        self.d1 = fourier_second_derivative(L1, N1, 1)
        self.d2 = fourier_second_derivative(L2, N2, 2) if N2 > 1 else np.zeros(1)
        self.kx = kvector(L1, N1, 1)                          # i*k
        self.ky = kvector(L2, N2, 2) if N2 > 1 else np.zeros(1, complex)
        # kept stacks (Field.h:1129-1166)
        self.kept = np.zeros((N2, self.M1), dtype=bool)
        if self.dim3:
            for j2 in list(range(0, N2 // 3)) + list(range(N2 - N2 // 3 + 1, N2)):
                self.kept[j2, : N1 // 3] = True
        else:
            self.kept[:, : N1 // 3] = True
        ms = (N2, self.M1, N3)
        z = lambda: np.zeros(ms, complex)
        self.u1, self.u2, self.u3, self.b, self.p = z(), z(), z(), z(), z()
        self.r1, self.r2, self.r3, self.rB = z(), z(), z(), z()
        ns = (N2, N1, N3)
        self.U1 = np.zeros(ns); self.U2 = np.zeros(ns); self.U3 = np.zeros(ns); self.B = np.zeros(ns)
        self.U1b = np.zeros(ns); self.U2b = np.zeros(ns); self.U3b = np.zeros(ns); self.Bb = np.zeros(ns)
        self.U_ = np.zeros(N3)
        self.dBdz = np.ones(N3)
        # IMEXRK.h:55-78
        self.solveLaplacian = {}
        for j1 in range(self.M1):
            for j2 in range(N2):
                lap = self.D2N.copy()
                lap += self.d1[j1] * np.eye(N3)
                lap += self.d2[j2] * np.eye(N3)
                neumannify(lap)
                if j1 == 0 and j2 == 0:
                    lap[0, :] = 0; lap[0, 0] = 1
                    lap[1, :] = 0; lap[1, 1] = 1
                t = Tridiagonal(); t.compute(lap)
                self.solveLaplacian[(j1, j2)] = t
        self.UpdateForTimestep()

    # Field.h:1129-1166
    def stacks(self):
        return [(j1, j2) for j2 in range(self.N2) for j1 in range(self.M1) if self.kept[j2, j1]]

    # IMEXRK.h:502-545
    def UpdateForTimestep(self):
        dt = self.deltaT
        self.h = [dt * 8.0 / 15.0, dt * 2.0 / 15.0, dt * 5.0 / 15.0]
        N3 = self.N3
        I = np.eye(N3)
        self.vN, self.vD, self.bN = [{}, {}, {}], [{}, {}, {}], [{}, {}, {}]
        for j1 in range(self.M1):
            for j2 in range(self.N2):
                for k in range(3):
                    lap = self.D2N + self.d1[j1] * I + self.d2[j2] * I
                    s = I - 0.5 * self.h[k] * lap / self.Re
                    neumannify(s); t = Tridiagonal(); t.compute(s); self.vN[k][(j1, j2)] = t
                    s = I - 0.5 * self.h[k] * lap / self.Re / self.Pr
                    neumannify(s); t = Tridiagonal(); t.compute(s); self.bN[k][(j1, j2)] = t
                    lap = self.D2D + self.d1[j1] * I + self.d2[j2] * I
                    s = I - 0.5 * self.h[k] * lap / self.Re
                    dirichlify(s); t = Tridiagonal(); t.compute(s); self.vD[k][(j1, j2)] = t

    # ---- transforms (Field.h:734-769, 965-994) ----
    def ToModal(self, nod):
        N1, N2 = self.N1, self.N2
        # FFTW r2c over dims {N2, N1} per level, then 1/(N1 N2) and Filter
        out = np.fft.rfft2(np.moveaxis(nod, 2, 0), axes=(1, 2))  # [N3][N2][M1]
        out = np.moveaxis(out, 0, 2) / (N1 * N2)
        out[~self.kept] = 0
        return out

    def ToNodal(self, mod):
        N1, N2 = self.N1, self.N2
        a = np.moveaxis(mod, 2, 0)
        out = np.fft.irfft2(a, s=(N2, N1), axes=(1, 2)) * (N1 * N2)
        return np.moveaxis(out, 0, 2)

    @staticmethod
    def Z(M, f):  # Dim3MatMul per stack: (M * stack)
        return f @ M.T

    # ---- IMEXRK.h:128-162 ----
    def FilterAll(self):
        for f in (self.u1, self.u2, self.u3, self.b, self.p):
            f[~self.kept] = 0
        if not self.dim3:
            self.u2[:] = 0

    def PopulateNodalVariables(self):
        self.U1 = self.ToNodal(self.u1)
        if self.dim3:
            self.U2 = self.ToNodal(self.u2)
        self.U3 = self.ToNodal(self.u3)
        self.B = self.ToNodal(self.b)

    @staticmethod
    def ZeroEnds(f, bc):
        f[..., 0] = 0; f[..., 1] = 0; f[..., -1] = 0; f[..., -2] = 0
        if bc == DIR:
            f[..., 2] = 0

    def _solve(self, fam, R, into, bc):
        self.ZeroEnds(R, bc)
        for (j1, j2) in self.stacks():
            t = fam[(j1, j2)]
            into[j2, j1] = t.solve(R[j2, j1].real) + 1j * t.solve(R[j2, j1].imag)

    # IMEXRK.cpp:43-73
    def RemoveDivergence(self, pm):
        kxm = self.kx[None, :, None]
        kym = self.ky[:, None, None]
        div = np.zeros_like(self.u1)
        div_all = kxm * self.u1 + (kym * self.u2 if self.dim3 else 0) + self.Z(self.DzD, self.u3)
        div[self.kept] = div_all[self.kept]
        self.ZeroEnds(div, NEU)
        q = np.zeros_like(div)
        for (j1, j2) in self.stacks():
            t = self.solveLaplacian[(j1, j2)]
            q[j2, j1] = t.solve(div[j2, j1].real) + 1j * t.solve(div[j2, j1].imag)
        m = self.kept
        self.u1[m] -= (kxm * q)[m]
        if self.dim3:
            self.u2[m] -= (kym * q)[m]
        self.u3[m] -= self.Z(self.DzN, q)[m]
        self.p[m] += pm * q[m]

    # IMEXRK.cpp:119-134
    def ExplicitRK(self, k):
        h, z = self.h[k], self.zeta[k]
        m = self.kept
        kxm = self.kx[None, :, None]; kym = self.ky[:, None, None]
        self.R1 = np.zeros_like(self.u1); self.R2 = np.zeros_like(self.u1)
        self.R3 = np.zeros_like(self.u1); self.RB = np.zeros_like(self.u1)
        self.R1[m] = (self.u1 + (h * z) * self.r1 + (-h) * (kxm * self.p))[m]
        if self.dim3:
            self.R2[m] = (self.u2 + (h * z) * self.r2 + (-h) * (kym * self.p))[m]
        self.R3[m] = (self.u3 + (h * z) * self.r3 + (-h) * self.Z(self.DzN, self.p))[m]
        self.RB[m] = (self.b + (h * z) * self.rB)[m]
        for f in (self.r1, self.r2, self.r3, self.rB):
            f[:] = 0

    # IMEXRK.cpp:107-117
    def FinishRHS(self, k):
        hb = self.h[k] * self.beta[k]
        m = self.kept
        self.R1[m] += hb * self.r1[m]
        if self.dim3:
            self.R2[m] += hb * self.r2[m]
        self.R3[m] += hb * self.r3[m]
        self.RB[m] += hb * self.rB[m]

    # IMEXRK.cpp:75-105
    def CrankNicolson(self, k):
        h = self.h[k]
        m = self.kept
        d1 = self.d1[None, :, None]; d2 = self.d2[:, None, None]
        c = 0.5 * h / self.Re
        self.R1[m] += (c * (d1 * self.u1 + d2 * self.u1 + self.Z(self.D2N, self.u1)))[m]
        self._solve(self.vN[k], self.R1, self.u1, NEU)
        if self.dim3:
            self.R2[m] += (c * (d1 * self.u2 + d2 * self.u2 + self.Z(self.D2N, self.u2)))[m]
            self._solve(self.vN[k], self.R2, self.u2, NEU)
        self.R3[m] += (c * (d1 * self.u3 + d2 * self.u3 + self.Z(self.D2D, self.u3)))[m]
        self._solve(self.vD[k], self.R3, self.u3, DIR)
        cb = 0.5 * h / self.Re / self.Pr
        self.RB[m] += (cb * (d1 * self.b + d2 * self.b + self.Z(self.D2N, self.b)))[m]
        self._solve(self.bN[k], self.RB, self.b, NEU)

    def _acc(self, r, val):
        r[self.kept] += val[self.kept]

    def _linear_terms(self):
        # IMEXRK.cpp:140-147 (dBdz generalises the hard-wired 1)
        nt = self.b.copy(); nt[0, 0] = 0
        self._acc(self.r3, self.Ri * self.Z(self.Rfull, nt))
        self._acc(self.rB, -(self.dBdz * self.Z(self.Rdir, self.u3)))

    # IMEXRK.cpp:136-193
    def BuildRHS(self):
        Z, TM = self.Z, self.ToModal
        kxm = self.kx[None, :, None]; kym = self.ky[:, None, None]
        self._linear_terms()
        U1t = self.U1 + self.U_
        U3, B, U2 = self.U3, self.B, self.U2
        nt = TM(U1t * U1t); self._acc(self.r1, -(kxm * nt))
        nt = TM(Z(self.DzD, Z(self.Rbar, U1t) * U3)); self._acc(self.r1, -nt)
        dt_ = TM(Z(self.Rtilde, U1t) * U3)
        nt = TM(Z(self.Rdir, U3) * Z(self.Rdir, U3))
        self._acc(self.r3, -(kxm * dt_ + Z(self.DzN, nt)))
        if self.dim3:
            nt = TM(U2 * U2); self._acc(self.r2, -(kym * nt))
            nt = TM(Z(self.DzD, Z(self.Rbar, U2) * U3)); self._acc(self.r2, -nt)
            dt_ = TM(Z(self.Rtilde, U2) * U3); self._acc(self.r3, -(kym * dt_))
            nt = TM(U1t * U2); self._acc(self.r1, -(kym * nt)); self._acc(self.r2, -(kxm * nt))
        nt = TM(Z(self.DzD, Z(self.Rbar, B) * U3)); self._acc(self.rB, -nt)
        if self.dim3:
            nt = TM(U2 * B); self._acc(self.rB, -(kym * nt))
        nt = TM(U1t * B); self._acc(self.rB, -(kxm * nt))

    # IMEXRK.cpp:195-258
    def BuildRHSLinear(self):
        Z, TM = self.Z, self.ToModal
        kxm = self.kx[None, :, None]; kym = self.ky[:, None, None]
        self._linear_terms()
        nn = self.U1b + self.U_
        U1, U2, U3, B = self.U1, self.U2, self.U3, self.B
        U2b, U3b, Bb = self.U2b, self.U3b, self.Bb
        nt = TM(U1 * nn); self._acc(self.r1, -2.0 * (kxm * nt))
        nt = TM(Z(self.DzD, Z(self.Rbar, U1) * U3b + Z(self.Rbar, nn) * U3)); self._acc(self.r1, -nt)
        dt_ = TM(Z(self.Rtilde, U1) * U3b + Z(self.Rtilde, nn) * U3)
        nt = TM(Z(self.Rdir, U3) * Z(self.Rdir, U3b))
        self._acc(self.r3, -(kxm * dt_ + 2.0 * Z(self.DzN, nt)))
        if self.dim3:
            nt = TM(Z(self.DzD, Z(self.Rbar, U2) * U3b + Z(self.Rbar, U2b) * U3)); self._acc(self.r2, -nt)
            nt = TM(U2 * U2b); self._acc(self.r2, -2.0 * (kym * nt))
            dt_ = TM(Z(self.Rtilde, U2) * U3b + Z(self.Rtilde, U2b) * U3); self._acc(self.r3, -(kym * dt_))
            nt = TM(U1 * U2b + nn * U2); self._acc(self.r1, -(kym * nt)); self._acc(self.r2, -(kxm * nt))
        nt = TM(Z(self.DzD, Z(self.Rbar, B) * U3b + Z(self.Rbar, Bb) * U3)); self._acc(self.rB, -nt)
        if self.dim3:
            nt = TM(B * U2b + Bb * U2); self._acc(self.rB, -(kym * nt))
        nt = TM(B * nn + Bb * U1); self._acc(self.rB, -(kxm * nt))

    def _stage(self, k, linear):
        self.ExplicitRK(k)
        if linear:
            self.BuildRHSLinear()
        else:
            self.BuildRHS()
        self.FinishRHS(k)
        self.CrankNicolson(k)
        self.RemoveDivergence(1 / self.h[k])
        self.FilterAll()
        self.PopulateNodalVariables()

    def TimeStep(self):  # IMEXRK.cpp:8-24
        for k in range(3):
            self._stage(k, False)

    def TimeStepLinear(self):  # IMEXRK.cpp:26-41
        for k in range(3):
            self._stage(k, True)

    # IMEXRK.h:461-500 (the mixing objective's forcing; J itself is not needed)
    def UpdateAdjointVariables(self, u1t, u2t, u3t, bt):
        self.U1_tot = self.ToNodal(u1t)
        self.U2_tot = self.ToNodal(u2t) if self.dim3 else np.zeros_like(self.U1)
        self.U3_tot = self.ToNodal(u3t)
        self.B_tot = self.ToNodal(bt)
        bAve = bt[0, 0].real          # HorizontalAverage (Integration.h:38-42)
        wAve = u3t[0, 0].real
        K = 2.0
        self.u3Forcing = (1 / K) * (self.B_tot - bAve)
        self.bForcing = (1 / K) * (self.U3_tot - wAve)
        self.u1Forcing = np.zeros_like(self.U1)
        self.u2Forcing = np.zeros_like(self.U1)

    # IMEXRK.cpp:260-379
    def BuildRHSAdjoint(self, u1t, u2t, u3t, bt):
        Z, TM, TN = self.Z, self.ToModal, self.ToNodal
        kxm = self.kx[None, :, None]; kym = self.ky[:, None, None]
        U1, U2, U3, B = self.U1, self.U2, self.U3, self.B
        U1T, U2T, U3T = self.U1_tot, self.U2_tot, self.U3_tot
        self.bForcing = self.bForcing + self.Ri * Z(self.Rdir, U3)
        nt = TM(U1 * U1T); self._acc(self.r1, kxm * nt)
        nt = TM(Z(self.DzD, Z(self.Rbar, U1) * U3T)); self._acc(self.r1, nt)
        dt_ = TM(Z(self.Rtilde, U1T) * U3)
        nt = TM(Z(self.Rdir, U3) * Z(self.Rdir, U3T))
        self._acc(self.r3, kxm * dt_ + Z(self.DzN, nt))
        if self.dim3:
            nt = TM(U2 * U2T); self._acc(self.r2, kym * nt)
            nt = TM(Z(self.DzD, Z(self.Rbar, U2) * U3T)); self._acc(self.r2, nt)
            dt_ = TM(Z(self.Rtilde, U2T) * U3); self._acc(self.r3, kym * dt_)
            nt = TM(U1 * U2T); self._acc(self.r1, kym * nt)
            nt = TM(U2 * U1T); self._acc(self.r2, kxm * nt)
        nt = TM(Z(self.DzD, Z(self.Rbar, B) * U3T)); self._acc(self.rB, nt)
        if self.dim3:
            nt = TM(B * U2T); self._acc(self.rB, kym * nt)
        nt = TM(B * U1T); self._acc(self.rB, kxm * nt)
        # extra adjoint terms
        nn2 = TN(kxm * u1t) * U1
        if self.dim3:
            nn2 = nn2 + TN(kxm * u2t) * U2
        self.u1Forcing = self.u1Forcing - (nn2 + Z(self.Rdir, TN(kxm * u3t) * U3))
        if self.dim3:
            nn2 = TN(kym * u1t) * U1 + TN(kym * u2t) * U2
            self.u2Forcing = self.u2Forcing - (nn2 + Z(self.Rdir, TN(kym * u3t) * U3))
        nd2 = TN(Z(self.DzN, u1t)) * Z(self.Rfull, U1)
        if self.dim3:
            nd2 = nd2 + TN(Z(self.DzN, u2t)) * Z(self.Rfull, U2)
        self.u3Forcing = self.u3Forcing - (nd2 + Z(self.Rfull, TN(Z(self.DzD, u3t))) * U3)
        self.u1Forcing = self.u1Forcing - TN(kxm * bt) * B
        if self.dim3:
            self.u2Forcing = self.u2Forcing - TN(kym * bt) * B
        self.u3Forcing = self.u3Forcing - TN(Z(self.DzN, bt)) * Z(self.Rfull, B)
        self._acc(self.r1, TM(self.u1Forcing))
        if self.dim3:
            self._acc(self.r2, TM(self.u2Forcing))
        self._acc(self.r3, TM(self.u3Forcing))
        self._acc(self.rB, TM(self.bForcing))

    # IMEXRK.h:86-126; below / above: dicts of modal u1, u2, u3, b
    def TimeStepAdjoint(self, below, above):
        f = 0.0
        for k in range(3):
            tot = {n: (1 - f) * above[n] + f * below[n] for n in ("u1", "u2", "u3", "b")}
            U1T = self.ToNodal(tot["u1"]) + self.U_
            tot["u1"] = self.ToModal(U1T)
            self.UpdateAdjointVariables(tot["u1"], tot["u2"], tot["u3"], tot["b"])
            self.ExplicitRK(k)
            self.BuildRHSAdjoint(tot["u1"], tot["u2"], tot["u3"], tot["b"])
            self.FinishRHS(k)
            self.CrankNicolson(k)
            self.RemoveDivergence(1 / self.h[k])
            self.FilterAll()
            self.PopulateNodalVariables()
            f += self.h[k] / self.deltaT

    def SetBase(self, u1, u2, u3, b):  # IMEXRK.h:334-352
        self.U1b = self.ToNodal(u1)
        if self.dim3:
            self.U2b = self.ToNodal(u2)
        self.U3b = self.ToNodal(u3)
        self.Bb = self.ToNodal(b)

    def Prepare(self):  # StateVector.cpp:94-97 and PrepareRun
        self.FilterAll()
        self.PopulateNodalVariables()
        self.RemoveDivergence(0.0)
        self.PopulateNodalVariables()

    # Integration.h:5-35, 282-311
    def IntegrateVertically(self, f, bc):
        N3 = self.N3
        if bc == NEU:
            z = vertical_points(self.L3, N3)
            return sum((z[k + 1] - z[k]) * f[k] for k in range(1, N3 - 1))
        zf = vertical_points_fractional(self.L3, N3)
        return sum((zf[k] - zf[k - 1]) * f[k] for k in range(2, N3 - 1))

    def InnerProd(self, a, b, bc):
        w = np.full((self.N2, self.M1), 2.0)
        w[0, 0] = 1.0
        horz = np.einsum("ij,ijk->k", w, (a * np.conj(b)).real)
        return self.IntegrateVertically(horz, bc)

    def KE(self):
        e = 0.5 * (self.InnerProd(self.u1, self.u1, NEU) + self.InnerProd(self.u3, self.u3, DIR))
        if self.dim3:
            e += 0.5 * self.InnerProd(self.u2, self.u2, NEU)
        return e

    def PE(self):
        return self.Ri * 0.5 * self.InnerProd(self.b, self.b, NEU)
