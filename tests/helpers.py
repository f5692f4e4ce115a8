"""Shared set-up of the parity tests: the benchmark configurations, seeded
initial conditions made by the oracle in FP64, and error norms."""
from __future__ import annotations

import numpy as np

from oracle import oracle as O
from stratiflow_b200.grid import background_profile

L1_DEFAULT = 2 * np.pi / 0.44

# (N1, N2, N3, L1, L2, L3, Re, Ri, Pr, dt, background, perturbed fields)
CONFIGS = {
    # plain 2D Kelvin-Helmholtz, 128 x 1 x 128
    "kh2d": dict(N1=128, N2=1, N3=128, L1=L1_DEFAULT, L2=L1_DEFAULT / 2, L3=10.0, Re=1000.0, Ri=0.1,
                 Pr=1.0, dt=0.01, bg="tanh", fields=("u1", "u3")),
    # 3D stratified shear layer, 256 x 128 x 384, Holmboe-type B = tanh(3z)
    "shear3d": dict(N1=256, N2=128, N3=384, L1=L1_DEFAULT, L2=L1_DEFAULT / 2, L3=10.0, Re=4000.0, Ri=0.16,
                    Pr=1.0, dt=0.005, bg="holmboe", fields=("u1", "u2", "u3")),
    # 2D 256 x 1 x 256 of the Newton-Krylov and continuation cases
    "nk2d": dict(N1=256, N2=1, N3=256, L1=L1_DEFAULT, L2=L1_DEFAULT / 2, L3=10.0, Re=1000.0, Ri=0.12,
                 Pr=1.0, dt=0.01, bg="tanh", fields=("u1", "u3")),
    # small 2D grid for eigenvalue checks against the oracle
    "lin2d": dict(N1=64, N2=1, N3=64, L1=L1_DEFAULT, L2=L1_DEFAULT / 2, L3=10.0, Re=1000.0, Ri=0.1,
                  Pr=1.0, dt=0.01, bg="tanh", fields=("u1", "u3")),
    # reduced 3D grid of the same flow, small enough for the oracle in seconds
    "shear3d_small": dict(N1=64, N2=32, N3=64, L1=L1_DEFAULT, L2=L1_DEFAULT / 2, L3=10.0, Re=4000.0,
                          Ri=0.16, Pr=1.0, dt=0.005, bg="holmboe", fields=("u1", "u2", "u3")),
}


def make_oracle(cfg, prec=32, Ri=None):
    c = cfg
    o = O.Oracle(c["N1"], c["N2"], c["N3"], c["L1"], c["L2"], c["L3"], c["Re"],
                 c["Ri"] if Ri is None else Ri, c["Pr"], c["dt"], prec=prec)
    U, dB = background_profile(c["bg"], c["L3"], c["N3"])
    o.set_background(U, dB)
    return o


def make_ic(cfg, seed=1234, amp=1e-3):
    """Seeded perturbation, made divergence-free by the FP64 oracle."""
    o = make_oracle(cfg, prec=64)
    o.make_ic(seed, amp=amp, nx_lo=8, ny_lo=8, fields=cfg["fields"])
    o.prepare()
    return o.get_state()


def rel_l2(a, b):
    a = np.asarray(a, dtype=np.complex128)
    b = np.asarray(b, dtype=np.complex128)
    n = np.linalg.norm(b)
    return float(np.linalg.norm(a - b) / (n if n > 0 else 1.0))


# measured relative L2 errors of the parity tests, by case; written as JSON to
# the path in SF_PARITY_TABLE at the end of the session (tests/conftest.py)
PARITY_TABLE: dict = {}


def record_parity(case: str, errs: dict, bounds: dict | None = None):
    """errs: {(oracle precision, field): relative L2}."""
    row = PARITY_TABLE.setdefault(case, {})
    for (prec, f), v in errs.items():
        row[f"{f} vs FP{prec}"] = float(v)
        if bounds is not None:
            row[f"{f} vs FP{prec} bound"] = float(bounds[(prec, f)])
