#!/usr/bin/env python
"""Benchmark of the IMEX-RK time step (IMEXRK::TimeStep, IMEXRK.cpp:8-24).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config shear3d|kh2d|nk2d|ensemble2d] [--xy-bands B]
    python bench.py --config continuation|predictor [--out DIR --points 40 --train 15 ...]

One "step" is one IMEX-RK time step (three RK stages) of every run of the
workload. The default workload is the 3D stratified shear layer
256 x 128 x 384 (Re 4000, Ri 0.16, Pr 1, U = tanh z, B = tanh 3z, dt 0.005)
with a seeded synthetic 1e-3 perturbation. Its state (5 x 21.7 MB) and the
per-step traffic exceed the 126 MB L2, so no L2 flush is needed between
steps. For N > 1 (torchrun) every rank advances its own replica (the step
does not shard on one GPU's workload: replicas only, weak scaling); the
value is the aggregate steps/s of all ranks over the max-over-ranks time.

Prints one JSON line on rank 0.
"""
from __future__ import annotations

import argparse
import ctypes as C
import json
import os
import subprocess
import sys
import tempfile
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

METRIC = "IMEX-RK steps/s (% HBM roofline); s per continuation point, learned vs plain"
L1_DEFAULT = 2 * np.pi / 0.44

WORKLOADS = {
    "shear3d": dict(N1=256, N2=128, N3=384, Re=4000.0, Ri=0.16, Pr=1.0, dt=0.005, bg="holmboe", nrun=1,
                    fields=("u1", "u2", "u3")),
    "kh2d": dict(N1=128, N2=1, N3=128, Re=1000.0, Ri=0.1, Pr=1.0, dt=0.01, bg="tanh", nrun=1,
                 fields=("u1", "u3")),
    "nk2d": dict(N1=256, N2=1, N3=256, Re=1000.0, Ri=0.12, Pr=1.0, dt=0.01, bg="tanh", nrun=1,
                 fields=("u1", "u3")),
    # 64 runs of the 256 x 256 2D case in one launch per kernel
    "ensemble2d": dict(N1=256, N2=1, N3=256, Re=1000.0, Ri=0.15, Pr=1.0, dt=0.01, bg="tanh", nrun=64,
                       fields=("u1", "u3")),
    # 64 independent 2D runs, N1 in {64, 128, 256}, N3 in {128, 256, 384} and
    # Ri uniform in [0.05, 0.25] drawn from a seed, one launch per kernel per
    # RK stage over all of them (sf_ensemble)
    "ensemble3": dict(N1=256, N2=1, N3=384, Re=1000.0, Ri=0.15, Pr=1.0, dt=0.01, bg="tanh", nrun=64,
                      fields=("u1", "u3"), mixed=True, seed=3),
}


def ensemble3_members(wl):
    """(N1, N3, Ri) of every run of the mixed ensemble, drawn from its seed."""
    rng = np.random.default_rng(wl["seed"])
    n1 = rng.choice([64, 128, 256], size=wl["nrun"])
    n3 = rng.choice([128, 256, 384], size=wl["nrun"])
    ri = rng.uniform(0.05, 0.25, size=wl["nrun"])
    return [(int(a), int(b), float(c)) for a, b, c in zip(n1, n3, ri)]


def peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        d = json.load(open(p))
        return float(d["hbm_gbs"]), float(d["bf16_tflops"]), "measured"
    return 6650.0, 1590.0, "fallback"


def seeded_state(s, cfg, seed):
    """Synthetic input: Gaussian modal coefficients (seeded) on kx < 8 (and
    |ky| < 8 in 3D) times 1e-3 exp(-z^2), Hermitian at kx = 0, ghost levels
    as StateVector::EnforceBCs leaves them; p = 0. Kept layout, all runs."""
    from stratiflow_b200.grid import vertical_points, vertical_points_fractional
    rng = np.random.default_rng(seed)
    N1, N2, N3 = s.N1, s.N2, s.N3
    z = vertical_points(10.0, N3)
    zf = vertical_points_fractional(10.0, N3)
    st = np.zeros(s.kept_shape, dtype=np.complex64)
    K1, K2 = s.K1, s.K2
    Ky = N2 // 3 if N2 > 1 else 1
    kyv = np.array([q if q < Ky else q - K2 for q in range(K2)]) if N2 > 1 else np.zeros(1, int)
    for r in range(s.nrun):
        for f, name in enumerate(("u1", "u2", "u3", "b")):
            if name not in cfg["fields"]:
                continue
            env = 1e-3 * np.exp(-(z if name == "u3" else zf) ** 2)
            for q in range(K2):
                if abs(kyv[q]) >= 8:
                    continue
                for j1 in range(min(8, K1)):
                    if j1 == 0 and kyv[q] < 0:
                        continue
                    c = rng.standard_normal(N3) + 1j * rng.standard_normal(N3)
                    if j1 == 0 and kyv[q] == 0:
                        c = c.real
                    st[r, f, :, q * K1 + j1] = env * c
                    if j1 == 0 and kyv[q] > 0:
                        qn = int(np.where(kyv == -kyv[q])[0][0])
                        st[r, f, :, qn * K1] = np.conj(env * c)
            if name == "u3":
                st[r, f, [0, 1, 2, N3 - 2, N3 - 1]] = 0
            else:
                st[r, f, 0] = st[r, f, 1]
                st[r, f, N3 - 1] = st[r, f, N3 - 2]
    return st


def make_solver(cfg, device, seed=2024):
    import stratiflow_b200 as sf
    from stratiflow_b200.grid import background_profile
    s = sf.IMEXRK(cfg["N1"], cfg["N2"], cfg["N3"], L1_DEFAULT, L1_DEFAULT / 2, 10.0, cfg["Re"], cfg["Pr"],
                  cfg["dt"], nrun=cfg["nrun"], device=device)
    U, dB = background_profile(cfg["bg"], 10.0, cfg["N3"])
    rng = np.random.default_rng(seed)
    for r in range(cfg["nrun"]):
        ri = cfg["Ri"] if cfg["nrun"] == 1 else float(rng.uniform(0.05, 0.25))
        s.set_ri(r, ri)
        s.SetBackground(r, U, dB)
    s.set_state_kept(seeded_state(s, cfg, seed))
    s.Prepare()
    s.synchronize()
    return s


class ClockSampler:
    """nvidia-smi clocks and throttle reasons sampled every 200 ms."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, device):
        self.device = device
        self.f = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
        self.p = None

    def __enter__(self):
        try:
            self.p = subprocess.Popen(["nvidia-smi", "-i", str(self.device), f"--query-gpu={self.Q}",
                                       "--format=csv,noheader,nounits", "-lms", "200"],
                                      stdout=self.f, stderr=subprocess.DEVNULL)
        except Exception:
            self.p = None
        time.sleep(0.3)
        return self

    def __exit__(self, *a):
        if self.p is not None:
            self.p.terminate()
            try:
                self.p.wait(timeout=5)
            except Exception:
                self.p.kill()

    def summary(self):
        self.f.flush()
        rows = []
        try:
            for line in open(self.f.name):
                parts = [x.strip() for x in line.split(",")]
                if len(parts) >= 9 and parts[1].replace(".", "").isdigit():
                    rows.append(parts)
        except Exception:
            pass
        if not rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unsampled"]}
        sm = np.array([float(r[1]) for r in rows])
        smax = max(float(r[2]) for r in rows)
        load = sm[sm > 0.5 * smax] if np.any(sm > 0.5 * smax) else sm
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = sorted({names[i] for r in rows for i in range(4) if r[5 + i].lower() == "active"})
        return {"sm_mhz": float(np.median(load)), "sm_max_mhz": smax, "reasons": reasons,
                "samples": len(rows)}


def ncu_traffic(config, kernel):
    """DRAM bytes (read + write) per launch of `kernel` on this workload from
    one ncu capture, as recorded in profiles/dram_traffic.json (None if the
    kernel has no capture there)."""
    path = os.path.join(os.path.dirname(os.path.abspath(__file__)), "profiles", "dram_traffic.json")
    try:
        with open(path) as f:
            rec = json.load(f).get(config, {}).get(kernel)
        return None if rec is None else float(rec["bytes_per_launch"])
    except (OSError, ValueError, KeyError):
        return None


def kernel_bytes(s, name):
    """Compulsory HBM bytes of one launch of a kernel in this decomposition:
    S = one kept-mode complex64 field (N3*K1*K2*8 B per run), M = one
    (kx, y) complex64 field (N3*N2*K1*8 B per run)."""
    S = s.N3 * s.K1 * s.K2 * 8 * s.nrun
    M = s.N3 * s.N2 * s.K1 * 8 * s.nrun
    nf = 4 if s.dim3 else 3
    if name == "k_ifft_y":
        return 4 * S + 4 * M
    if name in ("k_xpass", "k_xmarch"):
        return (4 * M + 8 * M) if s.dim3 else (3 * S + 3 * S)
    if name == "k_fft_y":
        return 8 * M + 4 * S
    if name in ("k_z_step", "k_z_step_tma", "k_z_step_c"):
        # in: u (nf fields), p, r_nl, r_old, and the per-mode factors 1/den_j
        # (float, half a complex field) of the velocity, u3, b and Laplacian
        # systems; out: u, p and r_old for the next stage
        return (3 * nf + 1 + 2) * S + (2 * nf + 1) * S
    return 0


def pass_of(name):
    """The pass of the step a kernel belongs to: the x-y pass (transforms,
    products, stencils) or the z pass (implicit solves and projection)."""
    return "z" if name.startswith("k_z") else "xy"


def pass_bytes(s, which):
    """Algorithmic bytes of one RK stage's pass, averaged over the three
    stages, from the compulsory traffic of kept-mode complex64 arrays (S per
    field): the x-y pass reads u and writes r (3D 8 S, 2D 6 S); the z pass
    reads u, p, r_old, r_new and writes u, p (3D 18 S, 2D 14 S; stage 0 has no
    r_old: 14 S, 11 S). Three stages sum to 74 S (3D) and 57 S (2D)."""
    S = s.N3 * s.K1 * s.K2 * 8 * s.nrun
    if which == "xy":
        return (8 if s.dim3 else 6) * S
    return ((14 + 18 + 18) if s.dim3 else (11 + 14 + 14)) * S / 3.0


def step_bytes_model(s):
    """Compulsory traffic per RK step of the fused step: 57 S in 2D and 74 S in
    3D (x-y pass reads u, writes r; z pass reads u, p, r_old, r_new and writes
    u, p; stage 0 has no r_old)."""
    S = s.N3 * s.K1 * s.K2 * 8 * s.nrun
    return (74 if s.dim3 else 57) * S


def cpu_baseline(wl, budget_s=20.0):
    """The FP32 oracle (CPU restatement of the reference, OpenMP on every host
    core) on a bounded sample of the same workload: whole steps of one run."""
    from oracle import oracle as O
    from stratiflow_b200.grid import background_profile
    O.build()
    cores = os.cpu_count() or 1
    O.set_threads(cores)
    cfg = wl
    o = O.Oracle(cfg["N1"], cfg["N2"], cfg["N3"], L1_DEFAULT, L1_DEFAULT / 2, 10.0, cfg["Re"], cfg["Ri"],
                 cfg["Pr"], cfg["dt"], prec=32)
    U, dB = background_profile(cfg["bg"], 10.0, cfg["N3"])
    o.set_background(U, dB)
    o.make_ic(7, amp=1e-3, fields=cfg["fields"])
    o.prepare()
    t0 = time.perf_counter()
    o.step(1)
    t1 = time.perf_counter() - t0
    n = int(max(1, min(200, budget_s / max(t1, 1e-6))))
    t0 = time.perf_counter()
    o.step(n)
    t = time.perf_counter() - t0
    runs = cfg["nrun"]
    return {"value": n / t / runs, "unit": "steps/s", "cores": O.get_threads(), "kind": "port",
            "sample": f"{n} whole steps of one run of the {cfg['N1']}x{cfg['N2']}x{cfg['N3']} workload"
                      + (f", scaled to the {runs}-run job" if runs > 1 else "")}


def dist_setup(args, backend="nccl"):
    """One process per GPU under torchrun (RANK / LOCAL_RANK / WORLD_SIZE /
    MASTER_* from the environment); a short process-group timeout so ranks
    that wait for one another end with an error. backend "gloo" (CPU tests of
    this host logic) leaves the GPUs alone."""
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    pg = None
    if ws > 1:
        import datetime
        import torch
        import torch.distributed as dist
        if backend == "nccl":
            torch.cuda.set_device(local)
            dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120),
                                    device_id=torch.device("cuda", local))
        else:
            dist.init_process_group(backend, timeout=datetime.timedelta(seconds=60))
        pg = dist
    return ws, rank, local, pg


def max_over_ranks(x, dist, device="cuda"):
    """The largest x over all ranks (every rank gets it); x itself on one rank."""
    if dist is None:
        return x
    import torch
    t = torch.tensor([float(x)], dtype=torch.float64, device=device)
    dist.all_reduce(t, op=dist.ReduceOp.MAX)
    return float(t.item())


def run_reference(args, wl, ws, rank):
    if rank != 0:
        return None
    if wl.get("mixed"):
        cb = ensemble_cpu_baseline(wl, ensemble3_members(wl), budget_s=60.0)
        return {"metric": METRIC, "value": cb["value"], "unit": "steps/s", "impl": "reference", "n_gpus": ws,
                "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 / cb["value"],
                "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
                "data": "synthetic", "config": {"workload": f"ensemble3: {wl['nrun']} mixed 2D runs (seed "
                                                            f"{wl['seed']})"},
                "cpu_baseline": cb,
                "e2e": {"value": cb["value"], "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    from oracle import oracle as O
    from stratiflow_b200.grid import background_profile
    O.build()
    cores = os.cpu_count() or 1
    O.set_threads(cores)
    o = O.Oracle(wl["N1"], wl["N2"], wl["N3"], L1_DEFAULT, L1_DEFAULT / 2, 10.0, wl["Re"], wl["Ri"], wl["Pr"],
                 wl["dt"], prec=32)
    U, dB = background_profile(wl["bg"], 10.0, wl["N3"])
    o.set_background(U, dB)
    o.make_ic(7, amp=1e-3, fields=wl["fields"])
    o.prepare()
    nw = min(args.warmup, 3)
    t0 = time.perf_counter()
    o.step(nw)
    tw = (time.perf_counter() - t0) / nw
    # bounded: at most ~90 s of timed CPU work
    n = int(max(1, min(args.steps, 90.0 / max(tw, 1e-6))))
    t0 = time.perf_counter()
    o.step(n)
    t = time.perf_counter() - t0
    v = n / t / wl["nrun"]
    return {"metric": METRIC, "value": v, "unit": "steps/s", "impl": "reference", "n_gpus": ws,
            "steps": n, "warmup": nw, "ms_per_step": 1e3 * t / n,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32",
            "data": "synthetic", "config": workload_config(args, wl),
            "cpu_baseline": {"value": v, "unit": "steps/s", "cores": O.get_threads(), "kind": "port",
                             "sample": f"{n} whole steps of one run (FP32 CPU restatement of "
                                       f"IMEXRK::TimeStep, OpenMP)"},
            "e2e": {"value": v, "unit": "steps/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}


# ---------------------------------------------------------------------------
# Newton-Krylov continuation along Ri (pseudo-arclength) and the learned predictor's
# study: `--config continuation` and `--config predictor` (2D 256 x 1 x 256,
# Re 1000, Pr 1, U = tanh z, B = tanh z, dt 0.01, T = 11 as NewtonKrylov.h:113).
#
# continuation: saturates the flow at Ri0 from a seeded synthetic input,
# converges two branch points with Newton-Krylov, runs a pseudo-arclength
# continuation in Ri with the secant predictor (PseudoArclength.cpp:33-68),
# trains the learned predictor on the first `train` converged points, and
# continues again from the same two points with the learned predictor (secant
# fallback after 6 Newton iterations). One JSON line per branch point goes to
# stderr and OUT/continuation.jsonl; the metric line (seconds, Newton
# iterations and linearised integrations per point, learned vs plain) to stdout.
# predictor: the learned and the secant guesses on a branch that needs no
# Newton solve (predictor_study).
# ---------------------------------------------------------------------------

def flow_at(Ri, N=256):
    from stratiflow_b200 import drivers as D
    return D.Flow(N, 1, N, L1_DEFAULT, L1_DEFAULT / 2, 10.0, 1000.0, 1.0, Ri, 0.01, "tanh")


def seeded(flow, seed=2024):
    """Gaussian modal coefficients on j1 < 8 times 1e-3 exp(-z^2) for u1 and
    u3, Hermitian at j1 = 0, made divergence-free by the solver."""
    import stratiflow_b200 as sf
    from stratiflow_b200.grid import background_profile, vertical_points, vertical_points_fractional
    s = sf.IMEXRK(flow.N1, 1, flow.N3, flow.L1, flow.L2, flow.L3, flow.Re, flow.Pr, flow.dt)
    U, dB = background_profile(flow.background, flow.L3, flow.N3)
    s.set_ri(0, flow.Ri)
    s.SetBackground(0, U, dB)
    rng = np.random.default_rng(seed)
    st = np.zeros(s.kept_shape, dtype=np.complex64)
    zf = vertical_points_fractional(flow.L3, flow.N3)
    z = vertical_points(flow.L3, flow.N3)
    for f, zz in ((0, zf), (2, z)):
        c = rng.normal(size=(flow.N3, 8)) + 1j * rng.normal(size=(flow.N3, 8))
        c[:, 0] = c[:, 0].real
        st[0, f, :, :8] = 1e-3 * np.exp(-zz[:, None] ** 2) * c
    s.set_state_kept(st)
    s.Prepare()
    return s


def saturate(flow, t_end, seed=2024):
    s = seeded(flow, seed)
    s.TimeStep(int(round(t_end / flow.dt)))
    s.synchronize()
    x = s.get_state_kept()[0]
    s.close()
    return x


def ext_dist(flow, a, b):
    from stratiflow_b200 import drivers as D
    (xa, ra), (xb, rb) = a, b
    d = xa.astype(np.complex128) - xb
    d[4] = 0
    return float(np.sqrt(D.ext_dot(flow, (d, 0.0), (d, 0.0), flow.Ri) + (ra - rb) ** 2))


def continuation_study(args):
    from stratiflow_b200 import drivers as D
    os.makedirs(args.out, exist_ok=True)
    log = open(os.path.join(args.out, "continuation.jsonl"), "w")

    def emit(rec):
        line = json.dumps(rec)
        print(line, file=sys.stderr, flush=True)
        log.write(line + "\n")
        log.flush()

    opts = D.NKOptions(max_newton=args.max_newton, krylov=args.krylov, target=args.target, gmres_tol=args.gmres_tol,
                       Delta=args.delta, block=args.block)
    Ri0 = args.ri0
    flow = flow_at(Ri0)
    t0 = time.perf_counter()
    x = saturate(flow, args.saturate)
    emit({"stage": "saturate", "Ri": Ri0, "t": args.saturate, "seconds": time.perf_counter() - t0})
    pts = []
    for Ri in (Ri0, Ri0 + args.dri):
        x, st = D.newton_fixed(flow_at(Ri), x, args.T, opts=opts)
        x = x.reshape(flow.state_shape)
        emit({"stage": "start point", "Ri": Ri, **{k: st[k] for k in ("converged", "residual", "newton_iterations",
                                                                           "jacobian_actions", "seconds")}})
        pts.append((x, Ri))
    ds = ext_dist(flow, pts[0], pts[1])
    emit({"stage": "step", "ds": ds})

    def run(tag, start, npoints, predictor):
        def cb(k, st):
            emit({"stage": tag, "point": k, **{key: st[key] for key in (
                "Ri", "predictor", "converged", "residual", "newton_iterations", "jacobian_actions",
                "integrations", "seconds", "wall_seconds")}, "residuals": st["residuals"]})
        return D.continuation(flow, start, ds, npoints, T=args.T, opts=opts, predictor=predictor, log=cb,
                              fallback_after=6)

    plain_pts, plain_stats = run("plain", pts, args.points, None)
    train = min(args.train, len(plain_pts) - 2)
    net = D.LearnedPredictor(flow, hidden=args.hidden, seed=1)
    t1 = time.perf_counter()
    losses = net.fit(plain_pts[:train + 2], ds, steps=args.train_steps, lr=args.lr)
    emit({"stage": "train", "samples": train, "params": net.net.num_params, "loss_first": float(losses[0]),
          "loss_last": float(losses[-1]), "heldout_secant": net.val_baseline, "heldout": net.val_losses,
          "uses_net": net.use_net, "seconds": time.perf_counter() - t1})
    start = plain_pts[train:train + 2]
    n_eval = len(plain_pts) - (train + 2)
    learned_pts, learned_stats = run("learned", start, n_eval, net)
    # the same branch points, plain vs learned
    ref = plain_stats[train:train + len(learned_stats)]
    summ = {"stage": "summary", "points_compared": len(learned_stats)}
    for tag, sts in (("plain", ref), ("learned", learned_stats)):
        conv = [s for s in sts if s["converged"]]
        summ[tag] = {
            "converged": len(conv),
            "newton_iterations_per_point": float(np.mean([s["newton_iterations"] for s in sts])) if sts else None,
            "jacobian_actions_per_point": float(np.mean([s["jacobian_actions"] for s in sts])) if sts else None,
            "integrations_per_point": float(np.mean([s["integrations"] for s in sts])) if sts else None,
            "seconds_per_point": float(np.mean([s["wall_seconds"] for s in sts])) if sts else None,
        }
    summ["learned_fallbacks"] = sum(1 for s in learned_stats if s["predictor"] != "learned")
    emit(summ)
    log.close()
    print(json.dumps({
        "metric": METRIC, "value": summ["learned"]["seconds_per_point"], "unit": "s per continuation point",
        "higher_is_better": False, "n_gpus": 1, "dtype": "f32 (FP64 Krylov numerics)", "data": "synthetic",
        "config": {"workload": f"continuation: 2D 256x1x256, Re 1000, Pr 1, Ri from {Ri0:g}, T {args.T:g}, "
                               f"{args.points} points, learned predictor trained on {train}",
                   "target_residual": args.target},
        "plain": summ["plain"], "learned": summ["learned"], "points_compared": summ["points_compared"],
        "learned_fallbacks": summ["learned_fallbacks"]}), flush=True)
    np.save(os.path.join(args.out, "branch_plain.npy"), np.stack([p[0] for p in plain_pts]))
    np.save(os.path.join(args.out, "branch_plain_ri.npy"), np.array([p[1] for p in plain_pts]))


def predictor_study(args):
    """The learned predictor against the secant on a branch generated by the
    solver without Newton: the saturated states x(Ri) at time t_sat of one
    seeded input, for Ri evenly spaced, phase shift and averages removed as
    PseudoArclength's constraints do (PseudoArclength.h:15-20). The network
    is trained on the first `train` points; for every later point k the
    guesses from points k-2, k-1 are compared with x(Ri_k) in the extended
    norm. All branch points are integrated together as the runs of one batch."""
    import stratiflow_b200 as sf
    from stratiflow_b200 import drivers as D
    from stratiflow_b200.grid import background_profile
    os.makedirs(args.out, exist_ok=True)
    Ris = np.linspace(args.ri0, args.ri1, args.points)
    flow = flow_at(float(Ris[0]))
    base = seeded(flow, args.seed).get_state_kept()[0]
    s = sf.IMEXRK(flow.N1, 1, flow.N3, flow.L1, flow.L2, flow.L3, flow.Re, flow.Pr, flow.dt, nrun=len(Ris))
    U, dB = background_profile(flow.background, flow.L3, flow.N3)
    for r, Ri in enumerate(Ris):
        s.set_ri(r, float(Ri))
        s.SetBackground(r, U, dB)
    s.set_state_kept(np.broadcast_to(base, s.kept_shape).copy())
    s.Prepare()
    t0 = time.perf_counter()
    s.TimeStep(int(round(args.saturate / flow.dt)))
    s.synchronize()
    t_int = time.perf_counter() - t0
    V = sf.Vecs(s, len(Ris))
    V.from_run(0, 0, len(Ris))
    pts = []
    for r, Ri in enumerate(Ris):
        V.phase_shift(r)
        V.remove_average(r, 0, flow.L3)
        V.remove_average(r, 3, flow.L3)
        x = V.get(r)
        x[4] = 0
        pts.append((x, float(Ri)))
    net = D.LearnedPredictor(flow, hidden=args.hidden, seed=1)
    dist = lambda a, b: ext_dist(flow, a, b)
    ds = dist(pts[0], pts[1])
    t1 = time.perf_counter()
    net.fit(pts[:args.train], ds, steps=args.train_steps, lr=args.lr)
    t_train = time.perf_counter() - t1
    rows = []
    for k in range(args.train, len(pts)):
        (gs, rs), _ = D.secant_predictor(flow, pts[k - 2], pts[k - 1], ds)
        gl, rl = net(pts[:k], ds)
        es = dist((gs, rs), pts[k])
        el = dist((gl, rl), pts[k])
        rows.append({"point": k, "Ri": pts[k][1], "secant_error": es, "learned_error": el,
                     "step": dist(pts[k - 1], pts[k])})
    ratio = [r["learned_error"] / r["secant_error"] for r in rows]
    summ = {"stage": "predictor summary", "points": len(pts), "train": args.train, "evaluated": len(rows),
            "t_saturate": args.saturate, "integration_seconds": t_int, "train_seconds": t_train,
            "params": net.net.num_params, "uses_net": net.use_net, "heldout_secant": net.val_baseline,
            "heldout_best": min(net.val_losses) if net.val_losses else None,
            "median_learned_over_secant_error": float(np.median(ratio)),
            "mean_learned_over_secant_error": float(np.mean(ratio)),
            "points_where_learned_is_better": int(sum(r < 1 for r in ratio))}
    with open(os.path.join(args.out, "predictor.jsonl"), "w") as f:
        for r in rows + [summ]:
            f.write(json.dumps(r) + "\n")
    print(json.dumps(summ), flush=True)



def make_ensemble(wl, device, seed):
    """The mixed-grid ensemble: every run's background, Ri and seeded input."""
    import stratiflow_b200 as sf
    from stratiflow_b200.grid import background_profile
    runs = ensemble3_members(wl)
    e = sf.Ensemble([(n1, n3) for n1, n3, _ in runs], (L1_DEFAULT, 10.0, wl["Re"], wl["Pr"]), wl["dt"],
                    device=device)
    for r, (m, (n1, n3, ri)) in enumerate(zip(e.members, runs)):
        U, dB = background_profile(wl["bg"], 10.0, n3)
        m.set_ri(0, ri)
        m.SetBackground(0, U, dB)
        m.set_state_kept(seeded_state(m, dict(wl, nrun=1), seed + r))
        m.Prepare()
        m.synchronize()
    return e, runs


def ensemble_bytes_per_step(runs):
    """The compulsory per-step traffic summed over the runs: 57 S per 2D run."""
    return sum(57 * n3 * (n1 // 3) * 8 for n1, n3, _ in runs)


def ensemble_cpu_baseline(wl, runs, budget_s=20.0):
    """The FP32 oracle (OpenMP, all host cores) on one run of every distinct
    grid of the ensemble, a few steps each; the job's steps/s is one over the
    sum of the runs' step times."""
    from oracle import oracle as O
    from stratiflow_b200.grid import background_profile
    O.build()
    O.set_threads(os.cpu_count() or 1)
    per = {}
    t_budget = budget_s / max(1, len({(a, b) for a, b, _ in runs}))
    for n1, n3 in sorted({(a, b) for a, b, _ in runs}):
        o = O.Oracle(n1, 1, n3, L1_DEFAULT, L1_DEFAULT / 2, 10.0, wl["Re"], 0.15, wl["Pr"], wl["dt"], prec=32)
        U, dB = background_profile(wl["bg"], 10.0, n3)
        o.set_background(U, dB)
        o.make_ic(7, amp=1e-3, fields=wl["fields"])
        o.prepare()
        t0 = time.perf_counter()
        o.step(1)
        t1 = time.perf_counter() - t0
        n = int(max(1, min(100, t_budget / max(t1, 1e-6))))
        t0 = time.perf_counter()
        o.step(n)
        per[(n1, n3)] = (time.perf_counter() - t0) / n
    total = sum(per[(a, b)] for a, b, _ in runs)
    return {"value": 1.0 / total, "unit": "steps/s", "cores": O.get_threads(), "kind": "port",
            "sample": f"whole steps of one run of each of the {len(per)} distinct grids, summed over the "
                      f"{len(runs)} runs"}


def run_ensemble3(args, wl, ws, rank, dist, local):
    import torch
    torch.cuda.set_device(local)
    e, runs = make_ensemble(wl, local, seed=2024 + rank)
    stream = torch.cuda.ExternalStream(e.stream(), device=torch.device("cuda", local))
    e.step(args.warmup)
    e.synchronize()
    n0 = e.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        e0.record(stream)
        e.step(args.steps)
        e1.record(stream)
        e.synchronize()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
    ms = max_over_ranks(e0.elapsed_time(e1), dist)
    launches = e.launch_count() - n0
    value = ws * args.steps / (ms / 1e3)
    clocks = clk.summary()
    # end to end: every step copies every run's kept state in from pinned host
    # memory and back out, through the members' C-ABI calls
    from stratiflow_b200 import load_library
    L = load_library()
    bufs = []
    for m in e.members:
        nb = 5 * m.N3 * m.plane * 8
        hi = torch.empty(nb, dtype=torch.uint8, pin_memory=True)
        ho = torch.empty(nb, dtype=torch.uint8, pin_memory=True)
        L.sf_get_state_kept(m.handle, C.c_void_p(hi.data_ptr()))
        bufs.append((hi, ho))
    nbytes = sum(b[0].numel() for b in bufs)
    n_e2e = max(3, min(args.steps, 20))
    if dist is not None:
        dist.barrier()
    t0 = time.perf_counter()
    for _ in range(n_e2e):
        for m, (hi, _ho) in zip(e.members, bufs):
            if L.sf_set_state_kept(m.handle, C.c_void_p(hi.data_ptr())):
                raise RuntimeError(L.sf_last_error().decode())
        e.step(1)
        e.synchronize()
        for m, (_hi, ho) in zip(e.members, bufs):
            if L.sf_get_state_kept(m.handle, C.c_void_p(ho.data_ptr())):
                raise RuntimeError(L.sf_last_error().decode())
    te = max_over_ranks(time.perf_counter() - t0, dist)
    e2e = {"value": ws * n_e2e / te, "unit": "steps/s", "h2d_bytes_per_step": nbytes, "d2h_bytes_per_step": nbytes,
           "api": "sf_set_state_kept + sf_ensemble_step + sf_get_state_kept per run"}
    mx, mz = e.profile(3)
    hbm, _, src = peaks()
    step_bytes = ensemble_bytes_per_step(runs)
    step_ach = step_bytes * (value / ws) / 1e9
    S_all = sum(n3 * (n1 // 3) * 8 for n1, n3, _ in runs)
    dom, dom_ms, dom_bytes = ("k_xpass_ens", mx, 6 * S_all) if mx >= mz else ("k_zstep_ens", mz, 13 * S_all)
    e.close()
    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return
    grids = {}
    for n1, n3, _ in runs:
        grids[f"{n1}x1x{n3}"] = grids.get(f"{n1}x1x{n3}", 0) + 1
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded tanh shear layers, 1e-3 perturbations)",
        "config": {"workload": f"ensemble3: {len(runs)} independent 2D runs, N1 in {{64,128,256}}, "
                               f"N3 in {{128,256,384}}, Ri in [0.05,0.25] (seed {wl['seed']}), Re {wl['Re']:g}, "
                               f"Pr {wl['Pr']:g}, dt {wl['dt']:g}, one launch per RK stage (persistent blocks over x-pass then z-solve work items)",
                   "grids": grids, "parallelism": f"replicas x{args.gpus}",
                   "l2": "L2-resident working set (launch-bound case)"},
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": dom_bytes / (dom_ms / 1e3) / 1e9, "peak": hbm,
                     "unit": "GB/s", "frac": dom_bytes / (dom_ms / 1e3) / 1e9 / hbm,
                     "peak_source": src, "traffic": None, "algorithmic_bytes_per_launch": dom_bytes,
                     "launch_ms": dom_ms},
        "step_roofline": {"bytes_per_step": step_bytes, "achieved": step_ach, "peak": hbm, "unit": "GB/s",
                          "frac": step_ach / hbm},
        "kernel_ms_per_step": {"k_xpass_ens": 3 * mx, "k_zstep_ens": 3 * mz},
        "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks,
    }
    if ws == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = ensemble_cpu_baseline(wl, runs)
    print(json.dumps(line), flush=True)


def profile_only(args, s):
    """Eager steps with per-kernel CUDA-event times, for profiler captures:
    step (TimeStep), linear (TimeStepLinear about the current state), adjoint
    (TimeStepAdjoint with the current state at both ends of the step) or net
    (the continuation predictor's forward and gradient passes, batch 16)."""
    import stratiflow_b200 as sf
    if args.z_kernel >= 0:
        s.set_z_kernel(args.z_kernel)
    if args.profile_mode == "step":
        s.TimeStep(args.warmup)
        s.synchronize()
        for name, t in s.profile_step(nsteps=max(1, args.steps)):
            print(f"{name} {t:.4f} ms")
    elif args.profile_mode == "linear":
        for r in range(s.nrun):
            st = s.get_state(r)
            s.SetBase(r, st["u1"], st["u2"], st["u3"], st["b"])
        s.TimeStepLinear(args.warmup)
        s.synchronize()
        for name, t in s.profile_step(nsteps=max(1, args.steps), linear=True):
            print(f"{name} {t:.4f} ms")
    elif args.profile_mode == "adjoint":
        v = sf.Vecs(s, s.nrun)
        v.from_run(0, 0, s.nrun)
        for _ in range(args.warmup + args.steps):
            s.TimeStepAdjoint((v, 0), (v, 0))
        s.synchronize()
    elif args.profile_mode == "net":
        import torch
        Z, batch, ch = 256, 16, [1024, 256, 256, 256, 512]
        net = sf.Net(ch, Z, batch, seed=1)
        rng = np.random.default_rng(0)
        x = rng.standard_normal((batch, Z, ch[0])).astype(np.float32)
        y = rng.standard_normal((batch, Z, ch[-1])).astype(np.float32)
        net.set_data(x, y)
        for _ in range(args.warmup):
            net.gradient()
        torch.cuda.synchronize()
        t0 = time.perf_counter()
        for _ in range(max(1, args.steps)):
            net.forward(x)
            net.set_data(x, y)   # a forward pass replaces the training inputs
            net.gradient()
        torch.cuda.synchronize()
        print(f"net forward + gradient {1e3 * (time.perf_counter() - t0) / max(1, args.steps):.3f} ms")
    s.synchronize()


def workload_config(args, wl):
    return {"workload": f"{args.config}: {wl['N1']}x{wl['N2']}x{wl['N3']} x {wl['nrun']} run(s), "
                        f"Re {wl['Re']:g}, Pr {wl['Pr']:g}, dt {wl['dt']:g}, background {wl['bg']}",
            "N1": wl["N1"], "N2": wl["N2"], "N3": wl["N3"], "runs_per_gpu": wl["nrun"],
            "parallelism": f"replicas x{args.gpus}",
            "l2": "state and per-step traffic exceed the 126 MB L2 (no flush)" if args.config == "shear3d"
                  else "L2-resident working set (launch-bound case)"}


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=50)
    ap.add_argument("--warmup", type=int, default=5)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--config", default="shear3d", choices=sorted(WORKLOADS) + ["continuation", "predictor"])
    ap.add_argument("--no-autotune", action="store_true", help="keep the launchers' default launch settings")
    ap.add_argument("--z-kernel", type=int, default=-1,
                    help="--profile-only: the z-pass kernel (sf_set_z_kernel; -1 keeps the solver's)")
    ap.add_argument("--xy-bands", type=int, default=0,
                    help="level bands of the 3D x-y pass (a launch setting; 0: the solver's default)")
    # continuation / predictor studies
    ap.add_argument("--out", default="bench_out")
    ap.add_argument("--ri0", type=float, default=0.05)
    ap.add_argument("--ri1", type=float, default=0.25)
    ap.add_argument("--dri", type=float, default=0.005, help="Ri step between the two start points")
    ap.add_argument("--points", type=int, default=40)
    ap.add_argument("--train", type=int, default=15)
    ap.add_argument("--saturate", type=float, default=400.0)
    ap.add_argument("--T", type=float, default=11.0)
    ap.add_argument("--target", type=float, default=1e-6)
    ap.add_argument("--max-newton", type=int, default=8)
    ap.add_argument("--krylov", type=int, default=320)
    ap.add_argument("--gmres-tol", type=float, default=1e-2)
    ap.add_argument("--delta", type=float, default=1.0)
    ap.add_argument("--block", type=int, default=16)
    ap.add_argument("--hidden", type=int, default=256)
    ap.add_argument("--train-steps", type=int, default=600)
    ap.add_argument("--lr", type=float, default=1e-3)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-only", action="store_true",
                    help="warm up, then print the per-kernel times of --steps eager steps (for ncu)")
    ap.add_argument("--profile-mode", default="step", choices=["step", "linear", "adjoint", "net"],
                    help="what --profile-only runs")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    if args.config == "continuation":
        continuation_study(args)
        return
    if args.config == "predictor":
        predictor_study(args)
        return
    wl = WORKLOADS[args.config]
    ws, rank, local, dist = dist_setup(args)
    if wl.get("mixed") and args.impl == "ours":
        run_ensemble3(args, wl, ws, rank, dist, local)
        return

    if args.impl == "reference":
        line = run_reference(args, wl, ws, rank)
        if rank == 0:
            print(json.dumps(line), flush=True)
        if dist is not None:
            dist.destroy_process_group()
        return

    import torch
    torch.cuda.set_device(local)
    s = make_solver(wl, local, seed=2024 + rank)
    if args.profile_only:
        profile_only(args, s)
        return
    stream = torch.cuda.ExternalStream(s.stream(), device=torch.device("cuda", local))

    # launch settings: the planner's choice for this grid (timed once per
    # device and grid, outside the timed region, then cached), unless given
    plan = None
    if not args.no_autotune:
        from stratiflow_b200 import autotune
        plan = autotune.tune(s)[0]
    if args.xy_bands > 0:
        s.set_xy_bands(args.xy_bands)
    # warm-up (also captures the step graph)
    s.TimeStep(args.warmup)
    s.synchronize()

    n0 = s.launch_count()
    e0 = torch.cuda.Event(enable_timing=True)
    e1 = torch.cuda.Event(enable_timing=True)
    with ClockSampler(local) as clk:
        if dist is not None:
            dist.barrier()
        torch.cuda.synchronize()
        s.synchronize()
        e0.record(stream)
        s.TimeStep(args.steps)
        e1.record(stream)
        s.synchronize()
        torch.cuda.synchronize()
        if dist is not None:
            dist.barrier()
    ms = max_over_ranks(e0.elapsed_time(e1), dist)
    launches = s.launch_count() - n0
    value = ws * args.steps / (ms / 1e3)
    clocks = clk.summary()

    # ---- end to end through the C-ABI with pinned host buffers ----
    nbytes = s.nrun * 5 * s.N3 * s.plane * 8
    host_in = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    host_out = torch.empty(nbytes, dtype=torch.uint8, pin_memory=True)
    s.synchronize()
    p_dev, _ = s.state_device_ptr()
    torch.cuda.synchronize()
    # seed the pinned input with the current state
    from stratiflow_b200 import load_library
    L = load_library()
    L.sf_get_state_kept(s.handle, C.c_void_p(host_in.data_ptr()))
    # a stream of steps long enough that filling and draining the copy
    # pipeline (the first input's copy, the last result's) is a small part
    n_e2e = max(100, args.steps)
    hin, hout = C.c_void_p(host_in.data_ptr()), C.c_void_p(host_out.data_ptr())

    def timed(body):
        if dist is not None:
            dist.barrier()
        t0 = time.perf_counter()
        body()
        return max_over_ranks(time.perf_counter() - t0, dist)

    def one_by_one():   # each call copies in, steps and copies out before the next
        for _ in range(n_e2e):
            rc = L.sf_set_state_kept(s.handle, hin)   # H2D of the step's input
            rc |= L.sf_step(s.handle, 1)
            rc |= L.sf_get_state_kept(s.handle, hout)  # D2H of the result
            if rc != 0:
                raise RuntimeError(L.sf_last_error().decode())

    def overlapped():   # sf_step_host_async: the same copies, overlapping the neighbouring steps
        rc = 0
        for _ in range(n_e2e):
            rc |= L.sf_step_host_async(s.handle, hin, hout, 1)
        rc |= L.sf_synchronize(s.handle)
        if rc != 0:
            raise RuntimeError(L.sf_last_error().decode())

    te_sync = timed(one_by_one)
    if L.sf_step_host_async(s.handle, hin, hout, 1) or L.sf_synchronize(s.handle):   # staging buffers
        raise RuntimeError(L.sf_last_error().decode())
    te = timed(overlapped)
    # the bound the copies alone set: one step's input in and result out over
    # PCIe at the same time, between pinned host and device buffers
    dev = torch.device("cuda", local)
    dev_in = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    dev_out = torch.empty(nbytes, dtype=torch.uint8, device=dev)
    cs_in, cs_out = torch.cuda.Stream(device=dev), torch.cuda.Stream(device=dev)

    def copies():
        for _ in range(5):
            with torch.cuda.stream(cs_in):
                dev_in.copy_(host_in, non_blocking=True)
            with torch.cuda.stream(cs_out):
                host_out.copy_(dev_out, non_blocking=True)
        torch.cuda.synchronize(dev)

    copies()
    tc = timed(copies) / 5
    del dev_in, dev_out
    e2e = {"value": ws * n_e2e / te, "unit": "steps/s", "h2d_bytes_per_step": nbytes,
           "d2h_bytes_per_step": nbytes, "api": "sf_step_host_async",
           "steps": n_e2e, "one_call_at_a_time": ws * n_e2e / te_sync,
           "copy_bound": {"value": ws / tc, "unit": "steps/s", "ms_per_step": tc * 1e3,
                          "what": "the step's input in and result out over PCIe concurrently, no compute"}}

    # ---- per-kernel profile of one step (eager, CUDA events) ----
    prof = s.profile_step(nsteps=3)
    per_kernel = {}
    for name, t in prof:
        k = name.split(":", 1)[1]
        per_kernel.setdefault(k, [0.0, 0])
        per_kernel[k][0] += t
        per_kernel[k][1] += 1
    total = sum(v[0] for v in per_kernel.values())
    dom = max(per_kernel, key=lambda k: per_kernel[k][0])
    dom_ms = per_kernel[dom][0] / per_kernel[dom][1]
    hbm, bf16, src = peaks()
    # the dominant kernel against the algorithmic bytes of the pass it belongs
    # to (a kernel that is part of a pass gets the whole pass's bytes: the
    # fraction then says how far that one kernel is from the pass's bound)
    achieved = pass_bytes(s, pass_of(dom)) / (dom_ms / 1e3) / 1e9
    traffic = ncu_traffic(args.config, dom)
    passes = {}
    for which in ("xy", "z"):
        ks = [k for k in per_kernel if pass_of(k) == which]
        ms_stage = sum(per_kernel[k][0] for k in ks) / 3.0   # per_kernel holds ms per step
        if ms_stage > 0:
            a = pass_bytes(s, which) / (ms_stage / 1e3) / 1e9
            passes[which] = {"kernels": sorted(ks), "bytes_per_stage": pass_bytes(s, which),
                             "ms_per_stage": ms_stage, "achieved": a, "frac": a / hbm}
    step_bytes = step_bytes_model(s)
    step_ach = step_bytes * (value / ws) / 1e9

    if dist is not None:
        dist.destroy_process_group()
    if rank != 0:
        return
    line = {
        "metric": METRIC, "value": value, "unit": "steps/s", "n_gpus": ws, "steps": args.steps,
        "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True, "scaling": "weak",
        "vs_baseline": None, "dtype": "f32", "data": "synthetic (seeded tanh shear layer, 1e-3 perturbation)",
        "config": dict(workload_config(args, wl), launch_plan=plan),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "peak_source": src + " (MEASURED_PEAKS.json hbm_gbs)"
                     if src == "measured" else src, "traffic": traffic,
                     "algorithmic_bytes_per_launch": pass_bytes(s, pass_of(dom)),
                     "decomposition_bytes_per_launch": kernel_bytes(s, dom), "launch_ms": dom_ms},
        "pass_roofline": passes,
        "step_roofline": {"bytes_per_step": step_bytes, "achieved": step_ach, "peak": hbm, "unit": "GB/s",
                          "frac": step_ach / hbm},
        "kernel_share": {k: round(v[0] / total, 4) for k, v in sorted(per_kernel.items())},
        "kernel_ms_per_step": {k: round(v[0], 4) for k, v in sorted(per_kernel.items())},
        "e2e": e2e, "gpu_launches": int(launches), "clocks": clocks,
    }
    if ws == 1 and not args.no_cpu_baseline:
        line["cpu_baseline"] = cpu_baseline(wl)
    print(json.dumps(line), flush=True)


if __name__ == "__main__":
    main()
