"""Newton-Krylov and continuation studies of the 2D stratified shear layer
(N1 = N3 = 256, Re = 1000, Pr = 1, U = tanh z, B = tanh z, dt = 0.01,
T = 11 as NewtonKrylov.h:113), run end to end on the GPU:

    python -m stratiflow_b200.experiments continuation --out DIR [--points 40 --train 15]
    python -m stratiflow_b200.experiments predictor --out DIR [--points 40 --train 15]

`continuation` saturates the flow at Ri0 from the seeded synthetic input,
converges two branch points with Newton-Krylov, runs a pseudo-arclength
continuation in Ri with the secant predictor (PseudoArclength.cpp:33-68),
trains the learned predictor on the first `train` converged points, and
continues again from the same two points with the learned predictor (secant
fallback after 6 Newton iterations). One JSON line per branch point and a
summary line go to stdout and to DIR/continuation.jsonl.

`predictor` compares the learned and the secant guesses on a branch that
needs no Newton solve (predictor_study).
"""
from __future__ import annotations

import argparse
import json
import os
import sys
import time

import numpy as np

from . import drivers as D

L1 = 2 * np.pi / 0.44


def flow_at(Ri, N=256):
    return D.Flow(N, 1, N, L1, L1 / 2, 10.0, 1000.0, 1.0, Ri, 0.01, "tanh")


def seeded(flow, seed=2024):
    """Gaussian modal coefficients on j1 < 8 times 1e-3 exp(-z^2) for u1 and
    u3, Hermitian at j1 = 0, made divergence-free by the solver."""
    import stratiflow_b200 as sf
    from .grid import background_profile, vertical_points, vertical_points_fractional
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
    (xa, ra), (xb, rb) = a, b
    d = xa.astype(np.complex128) - xb
    d[4] = 0
    return float(np.sqrt(D.ext_dot(flow, (d, 0.0), (d, 0.0), flow.Ri) + (ra - rb) ** 2))


def continuation_study(args):
    os.makedirs(args.out, exist_ok=True)
    log = open(os.path.join(args.out, "continuation.jsonl"), "w")

    def emit(rec):
        line = json.dumps(rec)
        print(line, flush=True)
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
    from .grid import background_profile
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
            line = json.dumps(r)
            print(line, flush=True)
            f.write(line + "\n")


def main(argv=None):
    ap = argparse.ArgumentParser(prog="python -m stratiflow_b200.experiments")
    sub = ap.add_subparsers(dest="cmd", required=True)
    c = sub.add_parser("continuation")
    c.add_argument("--out", required=True)
    c.add_argument("--ri0", type=float, default=0.05)
    c.add_argument("--dri", type=float, default=0.005, help="Ri step between the two start points")
    c.add_argument("--points", type=int, default=40)
    c.add_argument("--train", type=int, default=15)
    c.add_argument("--saturate", type=float, default=400.0)
    c.add_argument("--T", type=float, default=11.0)
    c.add_argument("--target", type=float, default=1e-6)
    c.add_argument("--max-newton", type=int, default=8)
    c.add_argument("--krylov", type=int, default=320)
    c.add_argument("--gmres-tol", type=float, default=1e-2)
    c.add_argument("--delta", type=float, default=1.0)
    c.add_argument("--block", type=int, default=16)
    c.add_argument("--hidden", type=int, default=256)
    c.add_argument("--train-steps", type=int, default=600)
    c.add_argument("--lr", type=float, default=1e-3)
    q = sub.add_parser("predictor")
    q.add_argument("--out", required=True)
    q.add_argument("--ri0", type=float, default=0.05)
    q.add_argument("--ri1", type=float, default=0.25)
    q.add_argument("--points", type=int, default=40)
    q.add_argument("--train", type=int, default=15)
    q.add_argument("--saturate", type=float, default=300.0)
    q.add_argument("--seed", type=int, default=2024)
    q.add_argument("--hidden", type=int, default=256)
    q.add_argument("--train-steps", type=int, default=600)
    q.add_argument("--lr", type=float, default=1e-3)
    args = ap.parse_args(argv)
    if args.cmd == "continuation":
        continuation_study(args)
    elif args.cmd == "predictor":
        predictor_study(args)


if __name__ == "__main__":
    sys.exit(main())
