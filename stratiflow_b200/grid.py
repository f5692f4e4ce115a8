"""Host-side grid helpers: the stretched vertical grid of Field.cpp:3-31 and
the background profiles a caller hands to ``IMEXRK.SetBackground``."""
from __future__ import annotations

import numpy as np


def vertical_points(L3: float, N3: int) -> np.ndarray:
    """Dirichlet (w) levels z_j, j >= 1 (Field.cpp:3-19); z_0 is unused."""
    assert N3 % 4 == 0
    step = 2.0 / (N3 - 2)   # Eigen LinSpaced(N3-1, -1, 1)
    x = np.array([(-1.0 + i * step) if i < N3 - 2 else 1.0 for i in range(N3 - 1)])
    z = np.zeros(N3)
    z[1:] = L3 * (2.0 * x ** 7 + x) / 3.0
    z[1:] *= -L3 / ((z[1] + z[2]) / 2)
    return z


def vertical_points_fractional(L3: float, N3: int) -> np.ndarray:
    """Neumann (u, b, p) levels (Field.cpp:21-31)."""
    z = vertical_points(L3, N3)
    zf = np.zeros(N3)
    zf[1:N3 - 1] = 0.5 * (z[1:N3 - 1] + z[2:])
    zf[0] = 2 * zf[1] - zf[2]
    zf[N3 - 1] = 2 * zf[N3 - 2] - zf[N3 - 3]
    return zf


def neumann_profile(f, L3: float, N3: int) -> np.ndarray:
    """Nodal1D::SetValue for a Neumann profile (Field.h:661-682): f at the
    fractional levels, then the two ghost levels at each end copied inwards."""
    z = vertical_points_fractional(L3, N3)
    v = np.array([f(zz) for zz in z], dtype=np.float64)
    v[1] = v[2]
    v[0] = v[1]
    v[N3 - 2] = v[N3 - 3]
    v[N3 - 1] = v[N3 - 2]
    return v


def background_profile(kind: str, L3: float, N3: int):
    """(U_, dB/dz) at the Neumann levels for the named background:
    'tanh'  U = tanh z, B = tanh z       -> dB/dz = sech^2 z
    'holmboe' U = tanh z, B = tanh 3z    -> dB/dz = 3 sech^2 3z
    'linear' U = tanh z, B = z           -> dB/dz = 1 (the reference's BuildRHS)."""
    zf = vertical_points_fractional(L3, N3)
    U = neumann_profile(np.tanh, L3, N3)
    if kind == "tanh":
        dB = 1.0 / np.cosh(zf) ** 2
    elif kind == "holmboe":
        dB = 3.0 / np.cosh(3 * zf) ** 2
    elif kind == "linear":
        dB = np.ones(N3)
    else:
        raise ValueError(kind)
    return U, dB


def kept_modes(N1: int, N2: int):
    """(j1, j2) index lists of the kept modes in the device's mode order
    m = q*K1 + j1 (Field.h:1129-1166)."""
    K1 = N1 // 3
    if N2 == 1:
        ys = [0]
    else:
        ys = list(range(0, N2 // 3)) + list(range(N2 - N2 // 3 + 1, N2))
    return [(j1, j2) for j2 in ys for j1 in range(K1)]
