#!/usr/bin/env python
"""Benchmark of the IMEX-RK time step (IMEXRK::TimeStep, IMEXRK.cpp:8-24).

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
                    [--config shear3d|kh2d|nk2d|ensemble2d]

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
}


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
    if name == "k_xpass":
        return (4 * M + 8 * M) if s.dim3 else (3 * S + 3 * S)
    if name == "k_fft_y":
        return 8 * M + 4 * S
    if name == "k_z_cn":
        # u, r_nl, r_old, p (and the b/u3 cross terms) in; u_new, r out; the
        # per-mode factor 1/den_j as float (half a complex field) per field
        return nf * (3 * S + S + 0.5 * S) + nf * 2 * S
    if name == "k_z_proj":
        return (nf - 1) * S + S + 0.5 * S + (nf - 1) * S + S
    return 0


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
    ap.add_argument("--config", default="shear3d", choices=sorted(WORKLOADS))
    ap.add_argument("--no-cpu-baseline", action="store_true")
    ap.add_argument("--profile-only", action="store_true",
                    help="warm up, then print the per-kernel times of --steps eager steps (for ncu)")
    args = ap.parse_args()
    args.warmup = max(3, args.warmup)
    wl = WORKLOADS[args.config]
    ws, rank, local, dist = dist_setup(args)

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
        s.TimeStep(args.warmup)
        s.synchronize()
        for name, t in s.profile_step(nsteps=max(1, args.steps)):
            print(f"{name} {t:.4f} ms")
        s.synchronize()
        return
    stream = torch.cuda.ExternalStream(s.stream(), device=torch.device("cuda", local))

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
    n_e2e = max(3, min(args.steps, 50))
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
    e2e = {"value": ws * n_e2e / te, "unit": "steps/s", "h2d_bytes_per_step": nbytes,
           "d2h_bytes_per_step": nbytes, "api": "sf_step_host_async",
           "one_call_at_a_time": ws * n_e2e / te_sync}

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
    achieved = kernel_bytes(s, dom) / (dom_ms / 1e3) / 1e9
    traffic = ncu_traffic(args.config, dom)
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
        "config": workload_config(args, wl),
        "roofline": {"bound": "hbm", "kernel": dom, "achieved": achieved, "peak": hbm, "unit": "GB/s",
                     "frac": achieved / hbm, "peak_source": src + " (MEASURED_PEAKS.json hbm_gbs)"
                     if src == "measured" else src, "traffic": traffic,
                     "algorithmic_bytes_per_launch": kernel_bytes(s, dom), "launch_ms": dom_ms},
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
