#!/usr/bin/env python
"""Benchmark: DSEM right-hand side + low-storage RK stage, FP64, p = 8.

Workload: the reference-scale Taylor-Green case (22^3 periodic hex elements on
[0,2pi]^3, p = 8, 729 Gauss points per element, 38,811,960 conserved
unknowns, Re = 1600, Mach 0.1, Carpenter-Kennedy 2N-storage RK with 5 stages,
dt = 0.5 x the inviscid limit).  A "step" is one RK time step (5 stages) of
the whole mesh.  Metric: DOF-RK-stages/s = unknowns x 5 x steps / seconds.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]
    python bench.py --workload ensemble [--steps K] [--warmup W]
    python bench.py --workload adjoint [--fd-check]
    python bench.py --workload cfg3 [--steps K] [--warmup W]

value : device-resident throughput, CUDA events on the library's stream
        around exactly K steps (CUDA graph per step), max over ranks.
e2e   : the same metric through the C-ABI with host buffers, one context:
        each step uploads the state from pinned host memory, advances one step
        and downloads it.  e2e_concurrent: three contexts (three copies of the
        case) on three host threads, whose copies overlap each other's steps.
At N = 1 the line also carries the other two parts of the metric: "ensemble"
(the cfg-4 64-case ensemble against the same cases one by one) and "adjoint"
(the cfg-5 adjoint/forward time ratio at 20 snapshots, the store-all variant
beside it, and GPU central differences along 8 seeded directions), each with
its own clock record.  --no-extras leaves them out.
Multi-GPU (torchrun): replicas only -- every rank advances its own copy of the
case, no data-path collective; value sums the ranks' unknowns.

--workload ensemble: 64 independent cases drawn from a seed (E in {4^3, 6^3,
8^3, 10^3, 12^3}, p in {4, 6, 8}, Re ~ U[400, 3200], Mach ~ U[0.05, 0.3] set
through the reference pressure, Taylor-Green or isotropic initial condition),
advanced together by one ensemble context (dsem_create_batch) against the same
64 cases run one after another through single-case contexts.

--workload adjoint: 12^3 elements at p = 6 (2,963,520 unknowns), Taylor-Green
with a seeded 5 % isotropic velocity perturbation (it removes the symmetries
at which the Roe flux's branches meet), Re = 1600, 400 steps; J = sum of eps * dt over the last 100 steps and its
exact discrete gradient with respect to the initial state and 1/Re
(dsem_adjoint), with every stage state kept in HBM and with 20 binomial
snapshots, timed against the 400 forward steps alone (dsem_step).
"""
import argparse
import json
import math
import os
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

NEX, P = 22, 8
RE = 1600.0
CFL = 0.5
STAGES = 5


def parse():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--nex", type=int, default=NEX)
    ap.add_argument("--p", type=int, default=P)
    ap.add_argument("--workload", default="tgv", choices=["tgv", "ensemble", "adjoint", "cfg3"])
    ap.add_argument("--fd-check", action="store_true")
    ap.add_argument("--no-extras", action="store_true",
                    help="default workload: leave out the ensemble and adjoint objects of the line")
    ap.add_argument("--ens-steps", type=int, default=10, help="ensemble object: timed steps")
    ap.add_argument("--cases", type=int, default=64)
    ap.add_argument("--seed", type=int, default=2024)
    ap.add_argument("--adj-steps", type=int, default=400, help="adjoint workload: steps of the run")
    ap.add_argument("--adj-window", type=int, default=100, help="adjoint workload: steps in the objective")
    ap.add_argument("--shape", type=int, default=-1,
                    help="default workload: the volume kernel's launch shape (0..4) instead of the autotuner's")
    return ap.parse_args()


# ---------------------------------------------------------------- op counts
# Counted from the kernel source (division and sqrt counted as one flop each;
# an FMA as two).  G = p+1 Gauss points, L = G+1 Lobatto points per direction.
VIS_FLOPS = 87     # one directional viscous flux vector (vis_flux_x/y/z)
EUL_FLOPS = 20     # one directional Euler flux vector
ROE_FLOPS = 161    # Roe flux + average + signed copies per mortar point
FVIS_FLOPS = 30    # viscous BR1 average per mortar point


def vol_flops(G):
    L, G2, NG = G + 1, G * G, G ** 3
    chain = lambda n: 2 * n - 1
    f = 5 * NG  # Q*jacob
    f += 3 * (5 * G2 * (L - 2) * chain(G) + 5 * G2 * G * chain(L) + 5 * NG)  # Lobatto, derivative, gradient
    f += 2 * 5 * NG  # Q*jacob reloads
    f += 3 * (5 * G2 * (L - 2) * chain(G) + 11 * G2 * L * chain(G))  # Lobatto rebuild, 11 gradient fields to grid
    f += 3 * (2 * G2 * (VIS_FLOPS + 5) + (L - 2) * G2 * (VIS_FLOPS + 5 + EUL_FLOPS + 5 + 10))  # fluxes
    f += 3 * 5 * G2 * G * chain(L - 2) + 2 * 5 * NG  # interior divergence + accumulation
    return f


def stage_flops(G):
    G2, NG = G * G, G ** 3
    upd = 30 * G2 * 2 + 5 * NG * 17 + 30 * G2 * (2 * G - 1)
    faces = 3 * G2 * (ROE_FLOPS + FVIS_FLOPS)  # three mortars per element
    return vol_flops(G) + upd + faces


def vol_bytes(G):
    L, G2, NG, NL = G + 1, G * G, G ** 3, (G + 1) * G * G
    return 8 * (5 * NG + NG + 3 * NG + 3 * NL + 30 * G2 + 30 * G2 + 5 * NG)


def stage_bytes(G):
    L, G2, NG, NL = G + 1, G * G, G ** 3, (G + 1) * G * G
    face_inv = 8 * (30 * G2 * 3 + 3 * G2 * 4)
    face_vis = 8 * (30 * G2 * 2 + 3 * G2)
    upd = 8 * (5 * NG * 5 + NG + 30 * G2 * 3)
    return face_inv + vol_bytes(G) + face_vis + upd


# ------------------------------------------------------------------- clocks
class Clocks:
    FIELDS = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
              "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
              "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, dev):
        self.dev = dev
        self.rows = []
        self.proc = None

    def __enter__(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", "-i", str(self.dev), f"--query-gpu={self.FIELDS}",
                                          "--format=csv,noheader,nounits", "-lms", "200"],
                                         stdout=subprocess.PIPE, stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None
        return self

    def _read(self):
        for line in self.proc.stdout:
            self.rows.append([x.strip() for x in line.split(",")])

    def __exit__(self, *a):
        if self.proc:
            self.proc.terminate()
            try:
                self.proc.wait(timeout=5)
            except Exception:
                self.proc.kill()

    def summary(self):
        if not self.rows:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["unavailable"], "samples": 0}
        sm = [float(r[1]) for r in self.rows if len(r) > 8 and r[1].replace(".", "").isdigit()]
        mx = [float(r[2]) for r in self.rows if len(r) > 8 and r[2].replace(".", "").isdigit()]
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        reasons = set()
        for r in self.rows:
            for k, n in enumerate(names):
                if len(r) > 5 + k and r[5 + k].lower() == "active":
                    reasons.add(n)
        return {"sm_mhz": float(np.median(sm)) if sm else None, "sm_max_mhz": max(mx) if mx else None,
                "reasons": sorted(reasons), "samples": len(self.rows)}


def fp64_gemm_peak(torch, dev):
    """cuBLAS FP64 GEMM throughput (burst), TFLOP/s: the FP64 arithmetic ceiling."""
    n = 8192
    a = torch.randn(n, n, dtype=torch.float64, device=dev)
    b = torch.randn(n, n, dtype=torch.float64, device=dev)
    for _ in range(2):
        torch.matmul(a, b)
    torch.cuda.synchronize(dev)
    best = 1e30
    for _ in range(5):
        s, e = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        s.record()
        torch.matmul(a, b)
        e.record()
        torch.cuda.synchronize(dev)
        best = min(best, s.elapsed_time(e))
    del a, b
    return 2.0 * n ** 3 / (best * 1e-3) / 1e12


def measured_peaks():
    p = os.path.join(ROOT, "MEASURED_PEAKS.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f), "measured"
    return {"hbm_gbs": 6650.0, "bf16_tflops": 1590.0}, "fallback"


def profiled_traffic():
    p = os.path.join(ROOT, "profiles", "k_vol_traffic.json")
    if os.path.exists(p):
        with open(p) as f:
            return json.load(f)
    return None


# ------------------------------------------------------------ CPU baseline
def cpu_baseline(desc, q, dt, dof):
    from oracle import oracle
    cores = oracle.set_threads(os.cpu_count() or 1)
    c = oracle.Case.from_desc(desc)
    c.set_phys(re=RE)
    c.set_q(q)
    t0 = time.perf_counter()
    for kk in range(1, STAGES + 1):
        c.stage(0.0, dt, kk, want_qt=False)
    t = time.perf_counter() - t0
    return {"value": dof * STAGES / t, "unit": "DOF-RK-stages/s", "cores": cores, "kind": "port",
            "sample": f"1 RK step (5 stages) of the same case ({int(desc['ngrid'])} elements, "
                      f"p={int(desc['ncg'][0]) - 1}), C++ oracle with OpenMP over elements"}


def run_reference(args):
    """Reference arm: the CPU restatement of DSEM's FP64 path on all host cores."""
    rank = int(os.environ.get("RANK", "0"))
    if rank != 0:
        return
    from dsem_b200 import mesh
    from oracle import oracle
    cores = oracle.set_threads(os.cpu_count() or 1)
    box = mesh.Box(args.nex, args.nex, args.nex, args.p)
    q = mesh.taylor_green(box)
    dt = CFL * mesh.dtcalc(box, q)
    dof = 5 * box.nel * (args.p + 1) ** 3
    c = oracle.Case.from_desc(box.desc())
    c.set_phys(re=RE)
    c.set_q(q)
    kk = 0
    for _ in range(args.warmup):
        kk = kk % STAGES + 1
        c.stage(0.0, dt, kk, want_qt=False)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        kk = kk % STAGES + 1
        c.stage(0.0, dt, kk, want_qt=False)
    t = time.perf_counter() - t0
    v = dof * args.steps / t
    line = {"metric": "DOF-RK-stages/s FP64 at p=8", "value": v, "unit": "DOF-RK-stages/s", "impl": "reference",
            "n_gpus": args.gpus, "steps": args.steps, "warmup": args.warmup, "ms_per_step": 1e3 * t / args.steps,
            "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64", "data": "synthetic",
            "config": {"workload": f"taylor-green {args.nex}^3 hex p={args.p}, Re=1600, Mach 0.1, 5-stage LSRK",
                       "unknowns": dof, "step": "one RK stage per sample"},
            "cpu_baseline": {"value": v, "unit": "DOF-RK-stages/s", "cores": cores, "kind": "port",
                             "sample": "one RK stage of the full case per step (C++ oracle, OpenMP)"},
            "e2e": {"value": v, "unit": "DOF-RK-stages/s", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0}}
    print(json.dumps(line), flush=True)


# ---------------------------------------------------------------- ensemble
ENS_SIZES = (4, 6, 8, 10, 12)
ENS_ORDERS = (4, 6, 8)


def ensemble_cases(n, seed):
    """(nex, p, Re, Mach, initial condition) of n cases drawn from seed."""
    rng = np.random.default_rng(seed)
    out = []
    for _ in range(n):
        nex = int(rng.choice(ENS_SIZES))
        p = int(rng.choice(ENS_ORDERS))
        re = float(rng.uniform(400.0, 3200.0))
        ma = float(rng.uniform(0.05, 0.3))
        ic = "tgv" if rng.random() < 0.5 else "iso"
        out.append((nex, p, re, ma, ic))
    return out


def ensemble_inputs(cases, seed):
    from dsem_b200 import mesh
    boxes, descs, qs, dts = {}, [], [], []
    for k, (nex, p, re, ma, ic) in enumerate(cases):
        if (nex, p) not in boxes:
            b = mesh.Box(nex, nex, nex, p)
            boxes[(nex, p)] = (b, b.desc())
        b, d = boxes[(nex, p)]
        twall = 1.0 / (ma * ma)  # rho0 = V0 = 1: Mach = V0 / sqrt(gamma p0 / rho0), p0 = twall / gamma
        q = mesh.taylor_green(b, twall=twall) if ic == "tgv" else \
            mesh.random_isotropic(b, seed=seed * 1000 + k, k0=2.0, mach_t=ma, twall=twall)
        descs.append(d)
        qs.append(q)
        dts.append(CFL * mesh.dtcalc(b, q))
    return descs, qs, np.array(dts)


def measure_ensemble(args, steps, warmup):
    """cfg 4: the 64-case ensemble in one context against the same cases run one by one.
    Returns the ensemble object of the bench line."""
    import torch
    from dsem_b200.solver import Ensemble, Solver
    cases = ensemble_cases(args.cases, args.seed)
    descs, qs, dts = ensemble_inputs(cases, args.seed)
    dof = np.array([5 * int(d["ngrid"]) * (c[1] + 1) ** 3 for d, c in zip(descs, cases)])
    work = float(dof.sum()) * STAGES * steps
    # one ensemble context
    ens = Ensemble(descs, [c[2] for c in cases])
    for k, q in enumerate(qs):
        ens.upload_case(k, q)
    shapes, _ = ens.autotune(reps=3)  # launch shape of the volume kernel per order (untimed)
    ens.step_batch(dts, warmup)
    torch.cuda.synchronize()
    with Clocks(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        ens.step_batch(dts, steps)
    ms_b, launches_b = ens.last_timing()
    ens.close()
    # the same cases one after another, each with the launch shape the ensemble's tuner chose for its order
    ms_s, launches_s = 0.0, 0
    for d, q, dt, c in zip(descs, qs, dts, cases):
        s = Solver(d, re=c[2])
        s.upload(q)
        s.set_vol_variant(c[1], shapes[c[1]])
        s.step(dt, warmup)
        s.step(dt, steps)
        m, n = s.last_timing()
        ms_s += m
        launches_s += n
        s.close()
    return {"metric": "DOF-RK-stages/s FP64, 64-case ensemble", "value": work / (ms_b * 1e-3),
            "unit": "DOF-RK-stages/s", "steps": steps, "warmup": warmup, "ms_per_step": ms_b / steps,
            "workload": f"ensemble of {len(cases)} cases, seed {args.seed}: E in 4^3..12^3, p in 4/6/8, "
                        "Re U[400,3200], Mach U[0.05,0.3]", "cases": len(cases),
            "unknowns": int(dof.sum()), "elements": int(sum(int(d["ngrid"]) for d in descs)),
            "volume_launch_shape_per_p": {str(k): v for k, v in shapes.items()},
            "sequential": {"value": work / (ms_s * 1e-3), "ms_per_step": ms_s / steps, "gpu_launches": launches_s},
            "speedup_vs_sequential": ms_s / ms_b, "gpu_launches": launches_b, "clocks": clk.summary()}


def run_ensemble(args):
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    e = measure_ensemble(args, args.steps, args.warmup)
    out = {"metric": e["metric"], "value": e["value"], "unit": e["unit"], "n_gpus": 1, "steps": args.steps,
           "warmup": args.warmup, "ms_per_step": e["ms_per_step"], "higher_is_better": True, "scaling": "weak",
           "vs_baseline": None, "dtype": "f64", "data": "synthetic (seeded Taylor-Green / isotropic initial conditions)",
           "config": {"workload": e["workload"], "cases": e["cases"], "unknowns": e["unknowns"],
                      "elements": e["elements"], "volume_launch_shape_per_p": e["volume_launch_shape_per_p"]},
           "sequential": e["sequential"], "speedup_vs_sequential": e["speedup_vs_sequential"],
           "gpu_launches": e["gpu_launches"], "clocks": e["clocks"]}
    print(json.dumps(out), flush=True)


def measure_adjoint(args, fd_check):
    """cfg 5: adjoint / forward time ratio at 20 step snapshots, two-level (segments)
    and binomial (revolve), and with every stage state kept; optional GPU central
    differences along 8 seeded directions and in 1/Re.  Returns the adjoint
    object of the bench line."""
    from dsem_b200 import mesh
    from dsem_b200.solver import Solver
    nex, p, nsteps, window = 12, 6, args.adj_steps, min(args.adj_window, args.adj_steps)
    box = mesh.Box(nex, nex, nex, p)
    q = mesh.perturbed_taylor_green(box, seed=args.seed)
    dt = CFL * mesh.dtcalc(box, q)
    s = Solver(box.desc(), re=RE)
    s.upload(q)
    s.step(dt, 3)  # warm-up (graph capture), then back to the initial state
    s.upload(q)
    dev = int(os.environ.get("LOCAL_RANK", "0"))
    out = {"metric": f"adjoint / forward time, {nsteps} steps, 20 step snapshots", "unit": "ratio",
           "higher_is_better": False,
           "workload": f"perturbed taylor-green {nex}^3 hex p={p}, Re=1600, {nsteps} steps, J = sum eps dt "
                       f"over the last {window}, checkpointing at 20 stored step states",
           "unknowns": 5 * box.nel * (p + 1) ** 3}
    res = {}
    with Clocks(dev) as clk:
        s.step(dt, nsteps)
        fwd_ms, _ = s.last_timing()
        out["forward_ms"] = fwd_ms
        for snaps, scheme, key in ((20, "segments", "segments_20"), (20, "revolve", "snapshots_20"),
                                   (0, "revolve", "snapshots_0")):
            s.upload(q)
            J, g, lr, ms = s.adjoint(dt, nsteps, window, snapshots=snaps, scheme=scheme)
            res[key] = (J, g, lr, ms)
            out[f"adjoint_ms_{key}"] = ms
            out[f"ratio_{key}"] = ms / fwd_ms
    out["clocks"] = clk.summary()
    out["value"] = out["ratio_segments_20"]
    out["scheme"] = ("20 step snapshots, two-level: the first sweep keeps the state at the start of each "
                     "20-step segment; the reverse sweep recomputes one segment at a time and keeps its "
                     "100 stage states and face traces in HBM while reversing it")
    out["revolve_variant"] = {"value": out["ratio_snapshots_20"],
                              "note": "20 step snapshots, binomial checkpointing (revolve order), nothing else kept"}
    out["store_all_variant"] = {"value": out["ratio_snapshots_0"],
                                "note": "every stage state and its face traces kept in HBM (snapshots = 0)"}
    J, g, lr, _ = res["segments_20"]
    out["J"] = J
    out["dJ_dinvRe"] = lr
    out["gradients_identical_across_checkpointing"] = bool(
        all(np.array_equal(res["snapshots_0"][1], res[k][1]) for k in ("segments_20", "snapshots_20")))
    if fd_check:  # central differences on the GPU along 8 seeded directions
        rng = np.random.default_rng(2024)
        G = p + 1
        rel = []
        for _ in range(8):
            d = rng.standard_normal(q.shape)
            d[:, :, G:] = 0.0
            d[:, :, :, G:] = 0.0
            d[:, :, :, :, G:] = 0.0
            h = 1e-6
            Jpm = []
            for sgn in (1.0, -1.0):
                s.upload(q + sgn * h * d)
                Jpm.append(s.adjoint(dt, nsteps, window, want_grad=False)[0])
            fd = (Jpm[0] - Jpm[1]) / (2 * h)
            rel.append(abs(float(np.sum(g * d)) - fd) / abs(fd))
        r0 = 1.0 / RE
        hr = 1e-4 * r0
        Jr = []
        for rr in (r0 + hr, r0 - hr):
            sr = Solver(box.desc(), re=1.0 / rr)
            sr.upload(q)
            Jr.append(sr.adjoint(dt, nsteps, window, want_grad=False)[0])
            sr.close()
        fdr = (Jr[0] - Jr[1]) / (2 * hr)
        out["fd_check"] = {"directions": 8, "step": h, "max_rel_err_q0": max(rel),
                           "rel_err_inv_re": abs(lr - fdr) / abs(fdr)}
    s.close()
    return out


def run_adjoint(args):
    import torch
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    a = measure_adjoint(args, args.fd_check)
    out = {"metric": a["metric"], "value": a["value"], "unit": "ratio", "n_gpus": 1, "higher_is_better": False,
           "dtype": "f64", "data": "synthetic (Taylor-Green + seeded 5% isotropic perturbation)",
           "config": {"workload": a["workload"], "unknowns": a["unknowns"]}}
    out.update({k: v for k, v in a.items() if k not in ("metric", "value", "unit", "higher_is_better", "workload",
                                                        "unknowns")})
    print(json.dumps(out), flush=True)


def run_cfg3(args):
    """cfg 3: decaying compressible isotropic turbulence, 16^3 periodic elements at p = 6 with the
    middle third in x at p = 8 (p-nonconforming band: 2,560 + 1,536 elements), seeded
    divergence-free field with E(k) ~ k^4 exp(-2 (k/4)^2) at turbulent Mach 0.3, Re = 115
    (Re_lambda ~ 100), entropy viscosity on.  DOF-RK-stages/s of the whole step (entropy
    viscosity included) and the volume kernel's FP64 rate per order."""
    import torch
    from dsem_b200 import mesh
    from dsem_b200.solver import Solver
    torch.cuda.set_device(int(os.environ.get("LOCAL_RANK", "0")))
    n = 16
    orders = np.full(n ** 3, 6)
    for iz in range(n):
        for ix in range(n):
            for iy in range(n):
                if n // 3 <= ix < n - n // 3:
                    orders[iy + n * (ix + n * iz)] = 8
    box = mesh.Box(n, n, n, orders)
    q = mesh.random_isotropic(box, seed=2024, k0=4.0, mach_t=0.3)
    s = Solver(box.desc(), re=115.0, cmu=1.0, mumax=0.5, shock=1)
    s.upload(q)
    dt = 0.3 * mesh.dtcalc(box, q)
    shapes, _ = s.autotune(reps=3)
    s.step(dt, args.warmup)
    torch.cuda.synchronize()
    with Clocks(int(os.environ.get("LOCAL_RANK", "0"))) as clk:
        s.step(dt, args.steps)
    ms, launches = s.last_timing()
    dof = int(sum(5 * (int(p) + 1) ** 3 for p in orders))
    prof = s.profile_rhs(5)
    nel = {p: int((orders == p).sum()) for p in (6, 8)}
    vol_fl = sum(nel[p] * vol_flops(p + 1) for p in nel)
    fp64_peak = fp64_gemm_peak(torch, "cuda")
    achieved = vol_fl / (prof[1] * 1e-3) / 1e12
    out = {"metric": "DOF-RK-stages/s FP64, cfg 3 (p-nonconforming band, entropy viscosity)",
           "value": dof * STAGES * args.steps / (ms * 1e-3), "unit": "DOF-RK-stages/s", "n_gpus": 1,
           "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms / args.steps, "higher_is_better": True,
           "dtype": "f64", "data": "synthetic (seeded isotropic field)",
           "config": {"workload": "isotropic turbulence 16^3 hex, p = 6 with a p = 8 band in the middle third of x, "
                                  "M_t 0.3, Re 115, entropy viscosity", "unknowns": dof, "elements": int(box.nel),
                      "elements_per_order": {str(k): v for k, v in nel.items()},
                      "volume_launch_shape_per_p": {str(k): v for k, v in shapes.items()}},
           "gpu_launches": launches, "clocks": clk.summary(),
           "roofline": {"bound": "fp64", "kernel": "k_vol_diag, entropy-viscosity variant, both orders",
                        "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s", "frac": achieved / fp64_peak,
                        "peak_source": "cuBLAS FP64 GEMM 8192^3 measured in this run",
                        "note": "counted flops exclude the entropy-viscosity prolongation (2 G-term chains per point)",
                        "kernel_ms": {"face_inv": prof[0], "vol": prof[1], "face_vis": prof[2], "update": prof[3]}}}
    s.close()
    print(json.dumps(out), flush=True)


def main():
    args = parse()
    if args.impl == "reference":
        run_reference(args)
        return
    if args.workload == "ensemble":
        if int(os.environ.get("RANK", "0")) == 0:
            run_ensemble(args)
        return
    if args.workload == "adjoint":
        if int(os.environ.get("RANK", "0")) == 0:
            run_adjoint(args)
        return
    if args.workload == "cfg3":
        if int(os.environ.get("RANK", "0")) == 0:
            run_cfg3(args)
        return
    import torch
    world = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    torch.cuda.set_device(local)
    dist = None
    if world > 1:
        import datetime

        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=300))
    from dsem_b200 import mesh
    from dsem_b200.solver import Solver

    box = mesh.Box(args.nex, args.nex, args.nex, args.p)
    desc = box.desc()
    q = mesh.taylor_green(box)
    dt = CFL * mesh.dtcalc(box, q)
    G = args.p + 1
    dof = 5 * box.nel * G ** 3
    s = Solver(desc, re=RE)
    s.upload(q)
    if args.shape >= 0:  # a given launch shape (profiling one shape), no tuning
        s.set_vol_variant(args.p, args.shape)
        shapes, shape_ms = {args.p: args.shape}, np.full((8, 5), -1.0)
    else:
        shapes, shape_ms = s.autotune(reps=3)  # launch shape of the volume kernel (untimed)

    def barrier():
        torch.cuda.synchronize()
        if dist:
            dist.barrier()

    # ---- device-resident throughput
    s.step(dt, args.warmup)
    barrier()
    with Clocks(local) as clk:
        s.step(dt, args.steps)
        barrier()
    ms, launches = s.last_timing()
    t = torch.tensor([ms], dtype=torch.float64, device="cuda")
    if dist:
        dist.all_reduce(t, op=dist.ReduceOp.MAX)
    ms_max = float(t.item())
    value = world * dof * STAGES * args.steps / (ms_max * 1e-3)

    # ---- end to end through the C-ABI with host buffers (pinned), ldx = nx = p+2: every step,
    # the state from pinned host memory to the device, one RK step, the state back to pinned
    # host memory.  Headline (e2e): one context, the drop-in's model (one context per rank),
    # where each step's copies and compute run one after another.  Beside it (e2e_concurrent):
    # NCTX contexts on NCTX host threads (the C-ABI's threading model), each its own copy of
    # the case, so that one context's copies overlap the others' compute.
    import threading
    NCTX = 3
    ldx = G + 1
    k_e2e = max(1, min(args.steps, 10))

    def serve(solver, hq_np, n):
        for _ in range(n):
            solver.upload(hq_np)
            solver.step(dt, 1)
            solver.download(out=hq_np)

    def timed_e2e(ctxs, hq_nps):
        barrier()
        t0 = time.perf_counter()
        workers = [threading.Thread(target=serve, args=(sv, h, k_e2e)) for sv, h in zip(ctxs, hq_nps)]
        for w in workers:
            w.start()
        for w in workers:
            w.join()
        barrier()
        te = torch.tensor([time.perf_counter() - t0], dtype=torch.float64, device="cuda")
        if dist:
            dist.all_reduce(te, op=dist.ReduceOp.MAX)
        return world * dof * STAGES * len(ctxs) * k_e2e / float(te.item())

    hqs = [torch.empty((box.nel, 5, ldx, ldx, ldx), dtype=torch.float64, pin_memory=True) for _ in range(NCTX)]
    hq_nps = [h.numpy() for h in hqs]
    s.download(out=hq_nps[0])
    serve(s, hq_nps[0], 1)  # warm-up of the host path
    e2e_single = timed_e2e([s], hq_nps[:1])
    ctxs = [s]
    for _ in range(NCTX - 1):
        sx = Solver(desc, re=RE)
        sx.upload(q)
        sx.set_vol_variant(args.p, shapes[args.p])
        ctxs.append(sx)
    for sv, h in zip(ctxs[1:], hq_nps[1:]):
        sv.download(out=h)
        serve(sv, h, 1)  # warm-up of the other contexts (graph capture)
    e2e_conc = timed_e2e(ctxs, hq_nps)
    nbytes = hq_nps[0].nbytes
    for sv in ctxs[1:]:
        sv.close()

    # ---- per-kernel device times (CUDA events on the library stream)
    prof = s.profile_rhs(5)
    t_vol = prof[1] * 1e-3
    peaks, src = measured_peaks()
    out = None
    if rank == 0:
        fp64_peak = fp64_gemm_peak(torch, "cuda")
        achieved = vol_flops(G) * box.nel / t_vol / 1e12
        hbm_ach = vol_bytes(G) * box.nel / t_vol / 1e9
        tr = profiled_traffic()
        roof = {"bound": "fp64", "pipe": "fp64 (DFMA, SIMT)", "achieved": achieved, "peak": fp64_peak, "unit": "TFLOP/s",
                "frac": achieved / fp64_peak, "kernel": "k_vol_diag (volume kernel, diagonal metrics)",
                "peak_source": "cuBLAS FP64 GEMM 8192^3 measured in this run (MEASURED_PEAKS.json has no FP64 figure)",
                "traffic": (tr["bytes_per_launch"] if tr else None),
                "hbm": {"achieved": hbm_ach, "peak": peaks["hbm_gbs"], "unit": "GB/s",
                        "frac": hbm_ach / peaks["hbm_gbs"], "peak_source": src},
                "kernel_ms": {"face_inv": prof[0], "vol": prof[1], "face_vis": prof[2], "update": prof[3]},
                "flops_per_element_stage": stage_flops(G), "vol_flops_per_element": vol_flops(G),
                "vol_bytes_per_element": vol_bytes(G)}
        stage_ms = ms_max / (args.steps * STAGES)
        step_tf = stage_flops(G) * box.nel / (stage_ms * 1e-3) / 1e12
        out = {"metric": "DOF-RK-stages/s FP64 at p=8", "value": value, "unit": "DOF-RK-stages/s",
               "n_gpus": world, "steps": args.steps, "warmup": args.warmup, "ms_per_step": ms_max / args.steps,
               "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f64",
               "data": "synthetic (analytic Taylor-Green initial condition)",
               "config": {"workload": f"taylor-green {args.nex}^3 hex p={args.p}, Re=1600, Mach 0.1, 5-stage LSRK",
                          "unknowns_per_gpu": dof, "elements": box.nel, "parallelism": f"replicas x{world}",
                          "l2": "inputs larger than L2 (state 310 MB + face buffers 620 MB)",
                          "stage_tflops_fp64": step_tf,
                          "volume_launch_shape": {"chosen": shapes[args.p],
                                                  "ms_per_shape": [round(float(x), 4) for x in shape_ms[args.p - 1]]}},
               "e2e": {"value": e2e_single, "unit": "DOF-RK-stages/s", "h2d_bytes_per_step": nbytes,
                       "d2h_bytes_per_step": nbytes, "steps": k_e2e,
                       "driver": "one context: upload + step + download per step, one after another"},
               "e2e_concurrent": {"value": e2e_conc, "unit": "DOF-RK-stages/s", "h2d_bytes_per_step": nbytes,
                                  "d2h_bytes_per_step": nbytes, "steps": NCTX * k_e2e,
                                  "driver": f"{NCTX} contexts (three copies of the case) on {NCTX} host threads, "
                                            "upload + step + download per step; copies overlap other contexts' steps"},
               "gpu_launches": launches, "clocks": clk.summary(), "roofline": roof}
        if world == 1:
            out["cpu_baseline"] = cpu_baseline(desc, q, dt, dof)
    s.close()
    if rank == 0 and world == 1 and not args.no_extras:
        # the other two parts of the metric: batched-ensemble speed-up (cfg 4) and the
        # adjoint/forward time ratio at 20 snapshots (cfg 5), each with its own clock record
        out["ensemble"] = measure_ensemble(args, args.ens_steps, args.warmup)
        out["adjoint"] = measure_adjoint(args, fd_check=True)
    if rank == 0:
        print(json.dumps(out), flush=True)
    if dist:
        dist.barrier()
        dist.destroy_process_group()


if __name__ == "__main__":
    main()
