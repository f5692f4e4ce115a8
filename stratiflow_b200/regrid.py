"""StateVector::LoadAndInterpolate (StateVector.h:275-413): a 2D `.fields`
file of another resolution (K1 x 1 x K3) onto a solver's grid.

The file's four nodal fields go to modal space at their own resolution on
the GPU (a solver of that size, `IMEXRK.LoadFlow`); every x mode the new grid
keeps is then interpolated linearly in z from the old stretched grid to the
new one, Neumann fields (u1, u2, b) between the fractional points and u3
between the Dirichlet points, clamped at the ends, with the reference's
search for the bracketing points; the Neumann ghost levels copy their
neighbours and EnforceBCs (StateVector.h:415-421) finishes the state. The
file's grid has L3 = 10, as the reference assumes (StateVector.h:301-302).
"""
from __future__ import annotations

import numpy as np

from .grid import vertical_points, vertical_points_fractional


def _weights(old_pts, new_pts, last):
    """[new][old] interpolation matrix of the reference's loop: for each new
    point, the first old pair (k-1, k) with z_k >= z (k stops at `last`),
    weights clamped to [0, 1]."""
    W = np.zeros((len(new_pts), len(old_pts)))
    for j, z in enumerate(new_pts):
        ka = 0
        while True:
            ka += 1
            kb = ka - 1
            zb, za = old_pts[kb], old_pts[ka]
            if not (za < z and ka < last):
                break
        wa = (z - zb) / (za - zb)
        wb = (za - z) / (za - zb)
        if wa > 1:
            wa, wb = 1.0, 0.0
        if wb > 1:
            wa, wb = 0.0, 1.0
        W[j, kb] += wb
        W[j, ka] += wa
    return W


def load_and_interpolate(solver, run, filename, K1, K3, L3_file=10.0):
    """Load the 2D `.fields` file of a K1 x 1 x K3 grid into run `run` of
    `solver` (a 2D IMEXRK); p is set to zero."""
    import stratiflow_b200 as sf
    if solver.N2 != 1:
        raise sf.SFError("LoadAndInterpolate is two-dimensional (StateVector.h:307-309)")
    old = sf.IMEXRK(K1, 1, K3, solver.L1, solver.L2, L3_file, solver.Re, solver.Pr, solver.deltaT)
    old.LoadFlow(0, filename)
    N3 = solver.N3
    Wn = _weights(vertical_points_fractional(L3_file, K3), vertical_points_fractional(solver.L3, N3), K3 - 2)
    # u3 lives on the Dirichlet points 1..N3-1 (row 0 is unused)
    Wd = np.zeros((N3, K3))
    Wd[1:, :] = _weights(vertical_points(L3_file, K3), vertical_points(solver.L3, N3)[1:], K3 - 1)
    nm = min(K1 // 2 + 1, solver.N1 // 2 + 1)
    out = {}
    for name in ("u1", "u2", "u3", "b"):
        src = old.get_field(0, name)[0]          # [M1_old][K3]
        dst = np.zeros(solver.modal_shape, dtype=np.complex128)
        W = Wd if name == "u3" else Wn
        dst[0, :nm, :] = src[:nm, :] @ W.T
        if name != "u3":                          # Neumann ends (StateVector.h:355-362)
            dst[0, :, 0] = dst[0, :, 1]
            dst[0, :, N3 - 1] = dst[0, :, N3 - 2]
        out[name] = dst
    out["p"] = np.zeros(solver.modal_shape, dtype=np.complex128)
    solver.set_state(run, out)
    old.close()
    v = sf.Vecs(solver, 1)
    v.from_run(0, run)
    v.enforce_bcs(0)
    v.to_run(0, run)
    solver.synchronize()
