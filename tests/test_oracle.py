"""CPU tests of the oracle: pinned to the dense transcription of the reference
(golden fixtures), to numpy's FFT, and to known answers of the operators."""
import os

import numpy as np
import pytest

from oracle import dense_ref as D
from oracle import oracle as O
from tests.helpers import CONFIGS, make_ic, make_oracle, rel_l2

GOLD = os.path.join(os.path.dirname(__file__), "golden")


@pytest.fixture(scope="module", autouse=True)
def _build():
    O.build()


@pytest.mark.parametrize("case", ["small2d", "small2d_tanh", "small3d"])
def test_oracle_matches_golden(case):
    g = np.load(os.path.join(GOLD, case + ".npz"))
    N1, N2, N3, L1, L2, L3, Re, Ri, Pr, dt = g["params"]
    o = O.Oracle(int(N1), int(N2), int(N3), L1, L2, L3, Re, Ri, Pr, dt, prec=64)
    o.set_background(g["U"], g["dBdz"])
    for k in ("u1", "u2", "u3", "b"):
        o.set_field(k, g["in_" + k])
    o.set_field("p", np.zeros_like(g["in_u1"]))
    o.prepare()
    for k in ("u1", "u2", "u3", "b", "p"):
        assert rel_l2(o.get_field(k), g["prep_" + k]) < 1e-12, k
    o.step(3)
    for k in ("u1", "u2", "u3", "b", "p"):
        assert rel_l2(o.get_field(k), g["step3_" + k]) < 1e-11, k
    ke, pe = o.energy()
    assert abs(ke - g["step3_energy"][0]) <= 1e-12 * abs(g["step3_energy"][0])
    assert abs(pe - g["step3_energy"][1]) <= 1e-11 * abs(g["step3_energy"][1]) + 1e-300
    st = o.get_state()
    o.set_base(st["u1"], st["u2"], st["u3"], st["b"])
    o.step_linear(2)
    for k in ("u1", "u2", "u3", "b", "p"):
        assert rel_l2(o.get_field(k), g["lin2_" + k]) < 1e-11, k
    # TimeStepAdjoint (IMEXRK.h:86-126) between the prepared input and the
    # 3-step state, from the fixture's adjoint input
    below = {k: g["prep_" + k] for k in ("u1", "u2", "u3", "b")}
    above = {k: g["step3_" + k] for k in ("u1", "u2", "u3", "b")}
    for k in ("u1", "u2", "u3", "b", "p"):
        o.set_field(k, g["adjin_" + k])
    o.populate_nodal()
    for _ in range(2):
        o.step_adjoint(below, above)
    for k in ("u1", "u2", "u3", "b", "p"):
        if k == "u2" and int(N2) == 1:
            continue
        assert rel_l2(o.get_field(k), g["adj2_" + k]) < 1e-10, k


@pytest.mark.parametrize("prec,tol", [(64, 1e-13), (32, 3e-6)])
@pytest.mark.parametrize("shape", [(32, 1, 16), (32, 16, 16)])
def test_fft_matches_numpy(prec, tol, shape):
    N1, N2, N3 = shape
    o = O.Oracle(N1, N2, N3, 1.0, 1.0, 10.0, 1000, 0.1, 1.0, 0.01, prec=prec)
    rng = np.random.default_rng(1)
    nod = rng.standard_normal((N2, N1, N3))
    mod = o.to_modal(nod)
    ref = np.moveaxis(np.fft.rfft2(np.moveaxis(nod, 2, 0), axes=(1, 2)), 0, 2) / (N1 * N2)
    kept = np.zeros((N2, N1 // 2 + 1), bool)
    ys = [0] if N2 == 1 else list(range(N2 // 3)) + list(range(N2 - N2 // 3 + 1, N2))
    for j2 in ys:
        kept[j2, : N1 // 3] = True
    ref[~kept] = 0
    assert rel_l2(mod, ref) < tol
    back = o.to_nodal(mod)
    ref_back = np.moveaxis(np.fft.irfft2(np.moveaxis(mod, 2, 0), s=(N2, N1), axes=(1, 2)), 0, 2) * N1 * N2
    assert rel_l2(back, ref_back) < tol


def test_fft_of_trig_polynomial():
    """cos(2 pi k x/L) transforms to 1/2 at mode k (Field.h:734-769 scaling)."""
    N1, N3 = 64, 16
    L1 = 3.0
    o = O.Oracle(N1, 1, N3, L1, 1.0, 10.0, 1000, 0.1, 1.0, 0.01, prec=64)
    x = np.arange(N1) * L1 / N1
    nod = np.zeros((1, N1, N3))
    nod[0] = np.cos(2 * np.pi * 5 * x / L1)[:, None] + 0.25
    mod = o.to_modal(nod)
    expect = np.zeros_like(mod)
    expect[0, 5, :] = 0.5
    expect[0, 0, :] = 0.25
    assert np.abs(mod - expect).max() < 1e-14


def test_operators_known_answers():
    """The banded operators equal the reference's dense matrices, and the
    second derivative is exact on quadratics away from the boundary rows."""
    N, L = 32, 10.0
    z = D.vertical_points(L, N)
    zf = D.vertical_points_fractional(L, N)
    # Neumann points are midpoints of Dirichlet points, so the Dirichlet
    # second difference is exact for z^2; the Neumann one is exact for linear
    # functions and a consistent approximation for z^2
    D2D = D.vertical_second_derivative_matrix(L, N, D.DIR)
    zz = z.copy(); zz[0] = 2 * z[1] - z[2]
    assert np.allclose((D2D @ zz ** 2)[2:N - 1], 2.0, rtol=1e-9)
    D2N = D.vertical_second_derivative_matrix(L, N, D.NEU)
    assert np.allclose((D2N @ (3 * zf + 1))[1:N - 1], 0.0, atol=1e-9)
    assert np.allclose((D2N @ zf ** 2)[2:N - 2], 2.0, rtol=0.1)
    # ddz of a linear function is exact on both staggerings
    DzN = D.vertical_derivative_matrix(L, N, D.NEU)
    assert np.allclose((DzN @ (3 * zf + 1))[2:], 3.0, rtol=1e-12)
    DzD = D.vertical_derivative_matrix(L, N, D.DIR)
    zz = z.copy(); zz[0] = 2 * z[1] - z[2]
    assert np.allclose((DzD @ (3 * zz + 1))[1:N - 1], 3.0, rtol=1e-12)
    # full reinterpolation is exact for linear functions at Dirichlet points
    R = D.neumann_reinterpolation_full(L, N)
    assert np.allclose((R @ zf)[2:N - 1], z[2:N - 1], rtol=1e-12, atol=1e-12)


def test_prepare_removes_divergence():
    cfg = CONFIGS["shear3d_small"]
    o = make_oracle(cfg, prec=64)
    o.make_ic(3, amp=1e-2, fields=("u1", "u2", "u3"))
    o.prepare()
    st = o.get_state()
    N1, N2, N3 = cfg["N1"], cfg["N2"], cfg["N3"]
    imex = D.IMEXRK(N1, N2, N3, cfg["L1"], cfg["L2"], cfg["L3"], cfg["Re"], cfg["Ri"], cfg["Pr"], cfg["dt"])
    div = imex.kx[None, :, None] * st["u1"] + imex.ky[:, None, None] * st["u2"] + imex.Z(imex.DzD, st["u3"])
    div[~imex.kept] = 0
    inner = div[..., 2:N3 - 2]
    assert np.abs(inner).max() < 1e-12 * max(1.0, np.abs(st["u1"]).max())


def test_fp32_tracks_fp64():
    """The FP32 build of the restatement stays within the FP32 noise floor of
    the FP64 build over 10 steps of the 2D Kelvin-Helmholtz case."""
    cfg = CONFIGS["kh2d"]
    ic = make_ic(cfg)
    o32, o64 = make_oracle(cfg, 32), make_oracle(cfg, 64)
    for o in (o32, o64):
        o.set_state(ic)
        o.prepare()
        o.step(10)
    for k in ("u1", "u3", "b"):
        assert rel_l2(o32.get_field(k), o64.get_field(k)) < 2e-5, k
    assert rel_l2(o32.get_field("p"), o64.get_field("p")) < 1e-3


def test_grid_helpers_match_oracle():
    from stratiflow_b200 import grid
    o = O.Oracle(32, 1, 64, 1.0, 1.0, 10.0, 1000, 0.1, 1.0, 0.01, prec=64)
    assert np.allclose(grid.vertical_points(10.0, 64)[1:], o.grid("z")[1:], rtol=1e-14)
    assert np.allclose(grid.vertical_points_fractional(10.0, 64), o.grid("zf"), rtol=1e-14)


@pytest.mark.parametrize("name", ["kh2d", "shear3d_small"])
def test_dissipation_matches_numpy_restatement(name):
    """The oracle's dissipation rates equal a numpy restatement written from
    the definitions: per field, sum over modes with the InnerProd weights
    (1 for (0,0), 2 otherwise; Integration.h:282-311) of (kx^2 + ky^2) |f|^2
    at the field's own quadrature rows, plus the squared staggered difference
    ddz f (Differentiation.cpp:35-61) at the other grid's quadrature rows
    (Integration.h:5-35)."""
    from stratiflow_b200.grid import vertical_points, vertical_points_fractional
    cfg = CONFIGS[name]
    st = make_ic(cfg, seed=5)
    st["b"] = 0.7 * st["u1"] + 0.2j * st["u3"]   # a non-zero buoyancy field
    o = make_oracle(cfg, 64)
    o.set_state(st)
    eps, chi = o.dissipation()
    N1, N2, N3 = cfg["N1"], cfg["N2"], cfg["N3"]
    z = vertical_points(cfg["L3"], N3)
    zf = vertical_points_fractional(cfg["L3"], N3)
    DY = np.zeros(N3); DY[1:] = zf[1:] - zf[:-1]
    DYF = np.zeros(N3); DYF[1:N3 - 1] = z[2:] - z[1:N3 - 1]

    def kint(n):
        if n == 1:
            return np.zeros(1)
        return np.array(list(range(n // 3 + 1)) + [0] * (n - 2 * (n // 3) - 1) + list(range(-(n // 3), 0)),
                        dtype=float)
    kx = kint(N1)[:N1 // 2 + 1] * 2 * np.pi / cfg["L1"]
    ky = kint(N2) * 2 * np.pi / cfg["L2"] if N2 > 1 else np.zeros(1)
    w = np.full((N2, N1 // 2 + 1), 2.0)
    w[0, 0] = 1.0
    k2 = (ky[:, None] ** 2 + kx[None, :] ** 2)[:, :, None]

    def grad_sq(f, neumann):
        f = np.asarray(f, dtype=np.complex128)
        a2 = np.abs(f) ** 2
        if neumann:
            hz = np.zeros(N3); hz[1:N3 - 1] = DYF[1:N3 - 1]          # Neumann rows 1..N3-2
            d = np.zeros_like(f); d[:, :, 2:] = (f[:, :, 2:] - f[:, :, 1:-1]) / DY[2:]
            vz = np.zeros(N3); vz[2:N3 - 1] = DY[2:N3 - 1]           # Dirichlet rows 2..N3-2
        else:
            hz = np.zeros(N3); hz[2:N3 - 1] = DY[2:N3 - 1]
            d = np.zeros_like(f)
            d[:, :, 1:N3 - 1] = (f[:, :, 2:] - f[:, :, 1:N3 - 1]) / DYF[1:N3 - 1]
            vz = np.zeros(N3); vz[1:N3 - 1] = DYF[1:N3 - 1]
        return float(np.sum(w[:, :, None] * (k2 * a2 * hz + np.abs(d) ** 2 * vz)))

    g = grad_sq(st["u1"], True) + grad_sq(st["u3"], False)
    if N2 > 1:
        g += grad_sq(st["u2"], True)
    assert abs(eps - g / cfg["Re"]) <= 1e-12 * abs(eps)
    c = cfg["Ri"] / (cfg["Re"] * cfg["Pr"]) * grad_sq(st["b"], True)
    assert abs(chi - c) <= 1e-12 * abs(chi)
