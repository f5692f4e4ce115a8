"""Launch planner of the time step: picks, per grid, the launch settings of
the step's kernels by timing them on the device, and caches the choice.

The reference's analogue is FFTW's planner: every transform site plans with
FFTW_PATIENT (Field.h:719-730, 949-960), which times candidate algorithms on
first use and keeps the fastest as wisdom. Here the candidates are the
kernels' launch shapes, which change no result (or only its rounding):

  xslabs    z-slabs one x-pass block walks through (sf_set_xpass_slabs;
            0 = the launcher's own choice)
  xgroups   lane groups per x-pass block (sf_set_xpass_groups; 0 = enough
            for one slab's inverse transforms in one round)
  xy_bands  level bands of the 3D x-y pass whose y transforms run beside the
            neighbouring bands' x passes (sf_set_xy_bands; 3D only)
  z_chunks  warps per block of the z solves, 8 or 16, each with one z-chunk
            (k_z_step) or two (k_z_step_c) (sf_set_z_chunks; 0 = the
            launcher's choice from the grid size)
  xkernel   the 3D nonlinear x pass as level-marching warps (1) or slab
            blocks (0) (sf_set_xpass_kernel; 3D only)
  zkernel   the z pass as k_z_step_c (2, one lane per complex mode),
            k_z_step (0) or k_z_step_tma (1, inputs brought in by
            tensor-map copies; applies with 8 z-chunks) (sf_set_z_kernel)

The search is coordinate descent from the launchers' defaults: each setting
in turn takes every candidate value with the others held, and a value
replaces the current one only if it is faster by more than the noise margin.
Plans are cached in memory and in a JSON file (SF_PLAN_CACHE, default
~/.cache/stratiflow_b200/plans.json) keyed by device name, grid, run count and
step kind.
"""
from __future__ import annotations

import json
import os
import time
from typing import Callable, Dict, List, Tuple

DEFAULTS = {"xkernel": 1, "xslabs": 0, "xy_bands": 1, "z_chunks": 0, "xgroups": 0, "zkernel": 2}
ORDER = ("xkernel", "xy_bands", "xslabs", "xgroups", "zkernel", "z_chunks")
MARGIN = 0.02   # a candidate must be 2% faster to replace the current value

_memory: Dict[str, dict] = {}


def space(N2: int, N3: int) -> Dict[str, List[int]]:
    """Candidate values of each setting for a grid."""
    return {
        "xkernel": [1, 0] if N2 > 1 else [DEFAULTS["xkernel"]],
        "xy_bands": [1, 2, 3, 4, 6, 8] if N2 > 1 else [DEFAULTS["xy_bands"]],
        "xslabs": [0, 1, 2, 3, 4, 6, 8],
        "z_chunks": [0] + [c for c in (8, 16) if N3 >= 2 * c],
        "xgroups": [0, 8, 16],
        "zkernel": [2, 0, 1],
    }


def search(measure: Callable[[dict], float], cand: Dict[str, List[int]], passes: int = 2,
           margin: float = MARGIN) -> Tuple[dict, List[Tuple[dict, float]]]:
    """Coordinate descent over the candidate values; `measure(settings)`
    returns seconds per step. Returns the best settings and every
    measurement made, in order."""
    cur = {k: (DEFAULTS[k] if DEFAULTS[k] in v else v[0]) for k, v in cand.items()}
    seen: Dict[Tuple, float] = {}
    log: List[Tuple[dict, float]] = []

    def t(settings):
        key = tuple(sorted(settings.items()))
        if key not in seen:
            seen[key] = float(measure(dict(settings)))
            log.append((dict(settings), seen[key]))
        return seen[key]

    best = t(cur)
    for _ in range(passes):
        changed = False
        for k in ORDER:
            if k not in cand:
                continue
            for v in cand[k]:
                if v == cur[k]:
                    continue
                trial = dict(cur, **{k: v})
                tv = t(trial)
                if tv < best * (1.0 - margin):
                    cur, best, changed = trial, tv, True
        if not changed:
            break
    return cur, log


def cache_path() -> str:
    return os.environ.get("SF_PLAN_CACHE",
                          os.path.join(os.path.expanduser("~"), ".cache", "stratiflow_b200", "plans.json"))


def plan_key(device: str, N1: int, N2: int, N3: int, nrun: int, mode: str) -> str:
    return f"{device}|{N1}x{N2}x{N3}|runs {nrun}|{mode}"


def load_cache(path: str | None = None) -> Dict[str, dict]:
    path = path or cache_path()
    try:
        with open(path) as f:
            d = json.load(f)
        return d if isinstance(d, dict) else {}
    except (OSError, ValueError):
        return {}


def store(key: str, settings: dict, path: str | None = None) -> None:
    _memory[key] = dict(settings)
    path = path or cache_path()
    d = load_cache(path)
    d[key] = dict(settings)
    try:
        os.makedirs(os.path.dirname(path), exist_ok=True)
        tmp = f"{path}.{os.getpid()}.tmp"   # processes sharing the cache (ranks) write their own
        with open(tmp, "w") as f:
            json.dump(d, f, indent=1, sort_keys=True)
        os.replace(tmp, path)
    except OSError:
        pass   # a read-only home keeps the plan in memory only


def lookup(key: str, path: str | None = None) -> dict | None:
    if key in _memory:
        return dict(_memory[key])
    d = load_cache(path).get(key)
    if isinstance(d, dict) and set(d) >= set(DEFAULTS):
        _memory[key] = {k: int(d[k]) for k in DEFAULTS}
        return dict(_memory[key])
    return None


def apply(solver, settings: dict) -> None:
    solver.set_xpass_kernel(int(settings.get("xkernel", DEFAULTS["xkernel"])))
    solver.set_xpass_slabs(int(settings["xslabs"]))
    if solver.N2 > 1:
        solver.set_xy_bands(int(settings["xy_bands"]))
    solver.set_z_chunks(int(settings["z_chunks"]))
    solver.set_xpass_groups(int(settings.get("xgroups", 0)))
    solver.set_z_kernel(int(settings.get("zkernel", DEFAULTS["zkernel"])))


def device_name(solver) -> str:
    try:
        import torch
        return torch.cuda.get_device_name(solver.device)
    except Exception:
        return "cuda"


def tune(solver, mode: str = "step", steps: int = 8, use_cache: bool = True, passes: int = 2):
    """Pick and apply the launch settings of `solver` for `mode` ("step":
    TimeStep, "linear": TimeStepLinear). The solver's state is saved before
    the timing steps and put back afterwards. Returns (settings, log)."""
    key = plan_key(device_name(solver), solver.N1, solver.N2, solver.N3, solver.nrun, mode)
    if use_cache:
        hit = lookup(key)
        if hit is not None:
            apply(solver, hit)
            return hit, []
    saved = solver.get_state_kept()
    advance = solver.TimeStepLinear if mode == "linear" else solver.TimeStep

    def measure(settings):
        apply(solver, settings)
        advance(2)   # captures the step graph of these settings
        solver.synchronize()
        t0 = time.perf_counter()
        advance(steps)
        solver.synchronize()
        dt = (time.perf_counter() - t0) / steps
        solver.set_state_kept(saved)
        return dt

    best, log = search(measure, space(solver.N2, solver.N3), passes=passes)
    apply(solver, best)
    solver.set_state_kept(saved)
    store(key, best)
    return best, log
