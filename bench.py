#!/usr/bin/env python
"""Benchmark of the LBcuda hot path on B200.

Workload (one GPU): two-component colour-gradient spinodal decomposition,
128^3 periodic, rhoR = rhoB = 0.5 + U(-0.01, 0.01) per cell from seed 1,
tauR = tauB = 1, sigma = 0.02, beta = 0.7.  One bench step = 500 lattice
steps (nIterOut of the reference's own 128^3 deck, Tests/CPC_Tab2_128/
input.dat, the interval at which it prints Mlup/s); the default 20 timed
steps are the 10,000 steps of the workload.  Headline: MLUPS (interior
cells, 10^6 lattice-cell updates per second) with FP16 shifted storage;
the FP32-storage run, the errors against an FP64 run and the roofline are
reported beside it.

    python bench.py [--gpus N] [--steps K] [--warmup W] [--impl ours|reference]

N > 1 (torchrun): every rank advances its own independent box (replicas,
weak scaling, no data-path collective); the time is the max over ranks.
"""
import argparse
import json
import os
import statistics
import subprocess
import sys
import threading
import time

import numpy as np

ROOT = os.path.dirname(os.path.abspath(__file__))
sys.path.insert(0, ROOT)

L = 128
SEED = 1
SIGMA, BETA = 0.02, 0.7
LB_PER_STEP = 500
# DRAM bytes (read + write) of one k_cg_lean launch at 128^3, from the ncu
# captures summarised in profiles/ (None where no capture of that storage)
# DRAM read + write bytes of one launch of the fluid kernel at 128^3 (ncu
# dram__bytes_read.sum + dram__bytes_write.sum, the captures summarised in
# profiles/k_cg_lean_*_128cube.md); measured, so they change with the kernel
TRAFFIC = {"f16": 370.1e6, "f16sd": 368.9e6, "f16sdp": 393.7e6, "f32": 622.6e6}
BYTES_PER_CELL = {"f16": 160, "bf16": 160, "f16sd": 160, "bf16sd": 160, "f16sdp": 160, "bf16sdp": 160, "f32": 312,
                  "f64": 616}  # algorithmic bytes per cell-step
MINIMAL_BYTES = {"f16": 152, "bf16": 152, "f16sd": 152, "f16sdp": 160, "f32": 304, "f64": 608}  # bytes the kernel must move
METRIC = "MLUPS & HBM GB/s, FP16-store vs FP32 LB at stated FP64 error, 1\u00d7B200"
# closure weights for radius-4 spheres (the ensemble workload), written by
# `python bench.py --only ensemble-closure --save-weights <path>`
CLOSURE_R4 = os.path.join(ROOT, "lbcuda_b200", "data", "closure_r4_weights.npy")


def peaks():
    try:
        with open(os.path.join(ROOT, "MEASURED_PEAKS.json")) as fh:
            d = json.load(fh)
        return float(d["hbm_gbs"]), "measured"
    except Exception:
        return 6650.0, "fallback"


class Clocks:
    """nvidia-smi sampling of SM clocks and throttle reasons during the timed region."""
    Q = ("index,clocks.sm,clocks.max.sm,power.draw,clocks_event_reasons.active,"
         "clocks_event_reasons.hw_slowdown,clocks_event_reasons.hw_thermal_slowdown,"
         "clocks_event_reasons.sw_thermal_slowdown,clocks_event_reasons.sw_power_cap")

    def __init__(self, index):
        self.index = str(index)
        self.proc = None
        self.lines = []

    def start(self):
        try:
            self.proc = subprocess.Popen(["nvidia-smi", f"--query-gpu={self.Q}", "--format=csv,noheader,nounits",
                                          "-i", self.index, "-lms", "200"], stdout=subprocess.PIPE,
                                         stderr=subprocess.DEVNULL, text=True)
            self.t = threading.Thread(target=self._read, daemon=True)
            self.t.start()
        except Exception:
            self.proc = None

    def _read(self):
        for ln in self.proc.stdout:
            self.lines.append(ln.strip())

    def stop(self):
        if not self.proc:
            return {"sm_mhz": None, "sm_max_mhz": None, "reasons": ["nvidia-smi unavailable"]}
        self.proc.terminate()
        try:
            self.proc.wait(5)
        except Exception:
            self.proc.kill()
        sm, mx, reasons = [], None, set()
        names = ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown", "sw_power_cap"]
        for ln in self.lines:
            f = [x.strip() for x in ln.split(",")]
            if len(f) < 9:
                continue
            try:
                sm.append(float(f[1]))
                mx = float(f[2])
            except ValueError:
                continue
            for nm, v in zip(names, f[5:9]):
                if v.lower() == "active":
                    reasons.add(nm)
        return {"sm_mhz": statistics.median(sm) if sm else None, "sm_max_mhz": mx,
                "reasons": sorted(reasons), "samples": len(sm)}


def max_over_ranks(v, pg, device):
    """The largest of every rank's value (timings are reported as the slowest rank's)."""
    if pg is None:
        return v
    import torch
    t = torch.tensor([float(v)], dtype=torch.float64, device=device)
    pg.all_reduce(t, op=pg.ReduceOp.MAX)
    return float(t.item())


def dist_env():
    ws = int(os.environ.get("WORLD_SIZE", "1"))
    rank = int(os.environ.get("RANK", "0"))
    local = int(os.environ.get("LOCAL_RANK", "0"))
    return ws, rank, local


WORKLOAD = ("colour-gradient spinodal 128^3 periodic, rho=0.5+U(-0.01,0.01) seed 1, tau=1, sigma=0.02, beta=0.7, "
            "10,000 lattice steps")


def workload_config():
    """The `config` object both arms print (the timed sample of each arm is described beside it)."""
    return {"workload": WORKLOAD, "cells": L ** 3, "lattice_steps_total": 20 * LB_PER_STEP,
            "l2": "inputs larger than L2 (2 x 160 MB population buffers at FP16, 2 x 320 MB at FP32)"}


def reference_arm(args, ws, rank):
    """The oracle (CPU restatement of the reference) on all host cores; it imports nothing of the
    product package, only oracle/."""
    if rank != 0:
        return 0
    from oracle.orc import OracleSim, default_params, noise_fields, num_threads
    p = default_params(L, model="cg", sigma=SIGMA, beta=BETA)
    rR, rB = noise_fields(L, L, L, seed=SEED)
    o = OracleSim(p, "ref")
    o.set_fields(rR, rB)
    per = 2  # lattice steps per bench step: a bounded sample of the workload
    for _ in range(args.warmup):
        o.step(per)
    t0 = time.perf_counter()
    for _ in range(args.steps):
        o.step(per)
    dt = time.perf_counter() - t0
    mlups = args.steps * per * L ** 3 / dt / 1e6
    line = {
        "impl": "reference", "metric": METRIC, "value": mlups, "unit": "MLUPS", "n_gpus": ws,
        "steps": args.steps, "warmup": args.warmup, "ms_per_step": dt / args.steps * 1e3,
        "higher_is_better": True, "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
        "config": workload_config(),
        "storage": "f32 (the reference's only storage)", "lattice_steps_per_bench_step": per,
        "cpu_baseline": {"value": mlups, "unit": "MLUPS", "cores": num_threads(), "kind": "port",
                         "sample": f"{args.steps} x {per} lattice steps of 128^3 after {args.warmup} x {per} warm-up"},
        "e2e": {"value": mlups, "unit": "MLUPS", "h2d_bytes_per_step": 0, "d2h_bytes_per_step": 0},
    }
    print(json.dumps(line), flush=True)
    return 0


def cpu_baseline_sample():
    from oracle.orc import OracleSim, default_params, noise_fields, num_threads
    p = default_params(L, model="cg", sigma=SIGMA, beta=BETA)
    rR, rB = noise_fields(L, L, L, seed=SEED)
    o = OracleSim(p, "ref")
    o.set_fields(rR, rB)
    o.step(1)
    n = 0
    t0 = time.perf_counter()
    while time.perf_counter() - t0 < 10.0:
        o.step(1)
        n += 1
    dt = time.perf_counter() - t0
    return {"value": n * L ** 3 / dt / 1e6, "unit": "MLUPS", "cores": num_threads(), "kind": "port",
            "sample": f"{n} lattice steps of the 128^3 workload (about 10 s), FP32, OpenMP"}


def bgk_timing(Lb, steps, warm=20):
    """Plain BGK (D3Q19, FP32, tau = 1, rho = 1 + U(-1e-3, 1e-3) from seed 1, u = 0), one k_bgk launch
    per lattice step: ms per step, MLUPS and the kernel's HBM fraction at 152 B per cell-step."""
    from lbcuda_b200 import LBSim, make_params
    from lbcuda_b200.inputs import seeded_noise_fields
    rho = seeded_noise_fields(Lb, Lb, Lb, mean=1.0, amp=1e-3, seed=SEED, ncomp=1)[0]
    s = LBSim(make_params(Lb, model="bgk", storage="f32", tau=1.0))
    s.set_fields(rho, None)
    s.step(warm)
    s.sync()
    tot, k, nl = s.time_steps(steps, kernel_timing=True)
    code = s.status()[0]
    s.close()
    per_us = k / nl * 1e3
    gbs = 152 * Lb ** 3 / (per_us * 1e-6) / 1e9
    return {"box": Lb, "steps": steps, "ms_per_step": tot / steps, "mlups": Lb ** 3 * steps / (tot * 1e-3) / 1e6,
            "kernel": "k_bgk", "kernel_us": per_us, "achieved_gbs": gbs, "frac": gbs / peaks()[0],
            "l2_resident": bool(152 * Lb ** 3 < 126e6), "device_error": code}


def error_vs_f64(nsteps_list=(100, 1000, 10000), workload="spinodal"):
    """Relative L2 error of |u| and phi of each storage against the FP64-storage run.

    workload "spinodal": the bench's own field (chaotic: every storage decorrelates from FP64 with
    time); "droplet": the reference's initType-1 droplet (radius L/8) in a uniform flow
    u0 = (0.02, 0.01, 0.005), a smooth problem whose error grows with rounding only."""
    from lbcuda_b200 import LBSim, make_params
    from lbcuda_b200.inputs import initial_fields, seeded_noise_fields
    vel = (0.0, 0.0, 0.0)
    if workload == "droplet":
        rR, rB = initial_fields(1, L, L, L)
        vel = (0.02, 0.01, 0.005)
    else:
        rR, rB = seeded_noise_fields(L, L, L, seed=SEED)
    out = {"workload": workload}
    sims = {}
    for st in ("f64", "f32", "f16", "bf16", "f16sd", "bf16sd", "f16sdp", "bf16sdp"):
        s = LBSim(make_params(L, model="cg", storage=st, sigma=SIGMA, beta=BETA))
        s.set_fields(rR, rB, vel)
        sims[st] = s
    done = 0
    for n in nsteps_list:
        res = {}
        for st, s in sims.items():
            s.step(n - done)
            res[st] = s.get_fields(f64=True)
        done = n
        u64, p64 = res["f64"][2], res["f64"][3]
        m64 = res["f64"][0].sum() + res["f64"][1].sum()
        for st in ("f32", "f16", "bf16", "f16sd", "bf16sd", "f16sdp", "bf16sdp"):
            eu = float(np.linalg.norm(res[st][2] - u64) / np.linalg.norm(u64))
            ep = float(np.linalg.norm(res[st][3] - p64) / np.linalg.norm(p64))
            out.setdefault(st, {})[f"after_{n}"] = {"u_rel_l2": eu, "phi_rel_l2": ep}
        out.setdefault("f64", {})[f"after_{n}"] = {"mass": float(m64)}
    for s in sims.values():
        s.close()
    return out


COLLOID_L = 256
COLLOID_N = 1280


def small_colloid_positions(L=128, n=160, seed=5, min_dist=13.0):
    """Seeded non-overlapping centres (centre distance >= 2r + 2 for r = 5.5) in an L^3 box:
    the colloid workload's 5 % volume fraction at 1/8 of its size, for profiler captures."""
    rng = np.random.default_rng(seed)
    x = []
    while len(x) < n:
        c = rng.uniform(1, L, 3)
        ok = True
        for y in x:
            d = c - y
            d -= L * np.round(d / L)
            if np.dot(d, d) < min_dist ** 2:
                ok = False
                break
        if ok:
            x.append(c)
    return np.array(x)


def colloid_sim(storage, schedule=2, small=False):
    """Colloid workload: 256^3 CG fluid with 1280 spheres of radius 5.5 (the first 1280 of the
    reference's Tests/07-1280-Particle placement), density 1, neutral wetting, at rest.
    small=True: 128^3 with 160 seeded spheres moving at up to 0.01 (profiler captures)."""
    from lbcuda_b200 import LBSim, make_params
    from lbcuda_b200.inputs import read_input_xyz, seeded_noise_fields
    if small:
        L, n = 128, 160
        x = small_colloid_positions(L, n)
        v = np.random.default_rng(6).uniform(-0.01, 0.01, (n, 3))
        q = None
    else:
        L, n = COLLOID_L, COLLOID_N
        deck = os.path.join(ROOT, "tests", "golden", "decks", "07-1280.input.xyz.256cube.r5.5")
        x, _, q = read_input_xyz(deck, n, True)
        v = np.zeros_like(x)
    vol = 4.0 / 3.0 * np.pi * 5.5 ** 3
    p = make_params(L, model="cg", storage=storage, sigma=SIGMA, beta=BETA, max_particles=n, radius=5.5,
                    rmass=float(1.0 / vol), wetting="neutral", lrotate=1, max_vel=1.0)
    s = LBSim(p)
    s.set_schedule(schedule)
    rR, rB = seeded_noise_fields(L, L, L, seed=SEED)
    s.set_fields(rR, rB)
    s.set_particles(x, v, None, q)
    return s


def colloid_error_vs_f64(steps=(100, 1000)):
    """Colloid workload at 128^3 (160 spheres r = 5.5 moving at up to 0.01): relative L2 error of the velocity
    field, relative max and L2 errors of the particle forces and the largest position difference of each
    storage against the FP64 run of the same kernels."""
    sims = {st: colloid_sim(st, small=True) for st in ("f64", "f32", "f16", "f16sd")}
    out, done = {}, 0
    for n in steps:
        res = {}
        for st, sm in sims.items():
            sm.step(n - done)
            res[st] = (sm.get_fields(f64=True)[2], sm.get_particles())
        done = n
        u64, p64 = res["f64"]
        for st in ("f32", "f16", "f16sd"):
            u, pp = res[st]
            out.setdefault(st, {})[f"after_{n}"] = {
                "u_rel_l2": float(np.linalg.norm(u - u64) / np.linalg.norm(u64)),
                "force_rel_max": float(np.abs(pp["force"] - p64["force"]).max() / np.abs(p64["force"]).max()),
                "force_rel_l2": float(np.linalg.norm(pp["force"] - p64["force"]) / np.linalg.norm(p64["force"])),
                "x_abs_max": float(np.abs(pp["x"] - p64["x"]).max())}
    for sm in sims.values():
        sm.close()
    return out


def colloid_timing(storage, steps=50, warm=10, small=False):
    s = colloid_sim(storage, small=small)
    s.step(warm)
    s.sync()
    tot, k, nl = s.time_steps(steps, kernel_timing=True)
    code = s.status()[0]
    s.close()
    cells = (128 if small else COLLOID_L) ** 3
    mlups = cells * steps / (tot * 1e-3) / 1e6
    return {"storage": storage, "small": small, "fluid_kernel_us": k / nl * 1e3 if nl else None, "mlups": mlups,
            "ms_per_step": tot / steps, "steps": steps, "achieved_gbs_at_basis": mlups * 1e6 * BYTES_PER_CELL[storage] / 1e9,
            "frac_at_basis": mlups * 1e6 * BYTES_PER_CELL[storage] / 1e9 / peaks()[0], "device_error": code}


def variants_timing(storage, steps=100, warm=20):
    """The reference's compile-time variants as models (densR = 2, densB = 1 for the two-density ones,
    as in its namelist deck): the spinodal workload at 128^3 on the two-pass schedule (phase field /
    densities, then the collision), single density on D3Q19 beside them for scale."""
    from lbcuda_b200 import LBSim, make_params
    from lbcuda_b200.inputs import seeded_noise_fields
    rR, rB = seeded_noise_fields(L, L, L, seed=SEED)
    out = {"storage": storage, "densR": 2.0, "densB": 1.0, "schedule": "two-pass"}
    for model in ("cg", "cg-diffdens", "cg-d3q27", "cg-diffdens-d3q27"):
        s = LBSim(make_params(L, model=model, storage=storage, sigma=SIGMA, beta=BETA, densR=2.0, densB=1.0))
        s.set_schedule(0)
        s.set_fields((2.0 * rR).astype(np.float32) if "diffdens" in model else rR, rB)
        s.step(warm)
        s.sync()
        tot, _, _ = s.time_steps(steps, kernel_timing=False)
        out[model] = {"ms_per_step": tot / steps, "mlups": L ** 3 * steps / (tot * 1e-3) / 1e6,
                      "device_error": s.status()[0]}
        s.close()
    return out


def ensemble_timing(steps=100, err_steps=200, seed=7, weights=None):
    """Ensemble workload: 48 boxes, edges uniform from {32, 48, 64, 96}, 0-40 spheres of radius 4 each
    (seeded, min gap 1), FP16 sum / difference pairs, the learned closure on (with `weights`, trained for
    radius 4; without them every close pair takes the analytic lubrication fallback), advanced together
    by the persistent kernel under a CUDA graph after the autotuner.  Error: relative L2 of each box's
    velocity field against the same box advanced alone with FP32 storage (same closure), after err_steps
    steps."""
    import ctypes
    from lbcuda_b200 import LBSim, capi, make_params
    from lbcuda_b200.ensemble import Ensemble, random_boxes
    from lbcuda_b200.inputs import seeded_noise_fields
    spec = random_boxes(48, seed=seed)

    def params(L, n, storage):
        return make_params(L, model="cg", storage=storage, sigma=SIGMA, beta=BETA, max_particles=max(n, 1),
                           radius=4.0, wetting="neutral", lrotate=1, max_vel=1.0, exact_tiles=0,
                           hz_rmin=8.5, hz_rcap=7.0, closure=1, lubrication=1, lubric_rmin=1.0, lubric_rcap=0.2)

    wf = None if weights is None else np.ascontiguousarray(weights, np.float32)

    def load(sim, i, L, x):
        rR, rB = seeded_noise_fields(L, L, L, seed=100 + i)
        sim.set_fields(rR, rB)
        if len(x):
            sim.set_particles(x, np.zeros_like(x))
            if wf is not None:
                capi.check(capi.lib().lbx_closure_set(sim._h, wf.ctypes.data_as(ctypes.POINTER(ctypes.c_float))),
                           "lbx_closure_set")

    ens = Ensemble([params(L, len(x), "f16sd") for L, x in spec])
    for i, (L, x) in enumerate(spec):
        load(ens.boxes[i], i, L, x)
    tuned = ens.tune(trial=6)
    for i, (L, x) in enumerate(spec):
        load(ens.boxes[i], i, L, x)
    ens.step(err_steps)
    errs = []
    for i, (L, x) in enumerate(spec):
        ref = LBSim(params(L, len(x), "f32"))
        load(ref, i, L, x)
        ref.step(err_steps)
        u16, u32 = ens.boxes[i].get_fields()[2], ref.get_fields()[2]
        errs.append(float(np.linalg.norm(u16 - u32) / max(np.linalg.norm(u32), 1e-30)))
        ref.close()
    ens.step(10)
    ms = ens.time(steps)
    cells = ens.cells
    spheres = int(sum(len(x) for _, x in spec))
    ens.close()
    return {"boxes": len(spec), "cells": cells, "spheres": spheres, "storage": "f16sd", "tuned": tuned,
            "closure": "trained weights (R_lo = 4)" if weights is not None else "analytic fallback only",
            "ms_per_step": ms / steps, "mlups": cells * steps / (ms * 1e-3) / 1e6,
            "u_rel_l2_vs_f32_per_box": {"after_steps": err_steps, "max": max(errs), "median": float(np.median(errs))}}


def closure_experiment(R_hi=6, L_hi=48, R_lo=3, steps_hi=240, m=256, epochs=100, n_direct=64, seed=11,
                       return_weights=False):
    """Learned closure workload.  Training data: the resistance of every lattice class of R_lo pairs with
    gap/R in [0.05, 1.5] (121 classes at R_lo = 3; R_hi resolved in L_hi^3, R_lo in the box scaled by
    R_lo / R_hi; a rest run and nine unit pair-frame velocity runs per class and resolution, static force
    subtracted), m velocity vectors per class uniform in +-1e-3 (pair frame), training on the GPU by the
    library's kernels.  Held out: n_direct pairs run directly (gap/R log-uniform, random orientation,
    random velocities) and fresh velocities for every class.  Errors: relative L2 of the R_lo pair forces,
    corrected or not, against the scaled R_hi forces."""
    from lbcuda_b200 import LBSim, closure, make_params
    t0 = time.perf_counter()
    res = closure.resistance(R_hi=R_hi, L_hi=L_hi, R_lo=R_lo, steps_hi=steps_hi)
    t_res = time.perf_counter() - t0
    X, T, _ = closure.synthesize(res, m, seed=seed)
    t0 = time.perf_counter()
    w, loss = closure.train(X, T, epochs=epochs, lr=2e-3)
    t_train = time.perf_counter() - t0
    Xd, Td, info = closure.generate(n_direct, R_hi=R_hi, L_hi=L_hi, R_lo=R_lo, steps_hi=steps_hi, seed=seed + 1)
    Xv, Tv, bv = closure.synthesize(res, 16, seed=seed + 2)
    fidx = [0, 1, 2, 6, 7, 8]  # the two forces, pair frame

    def rel(Tt, base, corr):
        hi = (base + Tt)[:, fidx]
        err = (Tt - corr)[:, fidx]
        per_pair = np.linalg.norm(err, axis=1) / np.maximum(np.linalg.norm(hi, axis=1), 1e-30)
        return {"rel_l2": float(np.linalg.norm(err) / np.linalg.norm(hi)), "median_pair": float(np.median(per_pair)),
                "pairs_within_5pct": float(np.mean(per_pair <= 0.05))}

    def errors(Xt, Tt, base):
        return {"none": rel(Tt, base, np.zeros_like(Tt)),
                "analytic_lubrication": rel(Tt, base, closure.analytic_lubrication(Xt, float(R_lo))),
                "closure": rel(Tt, base, closure.infer(w, Xt))}

    # cost of a step at each resolution (same prescribed-motion pair runs)
    costs = {}
    for R, L in ((R_hi, L_hi), (R_lo, int(round(L_hi * R_lo / R_hi)))):
        p = make_params(L, model="cg", storage="f32", max_particles=2, radius=float(R), kinematic=1, lrotate=1,
                        wetting="neutral", max_vel=1.0, exact_tiles=0)
        sim = LBSim(p)
        one = np.ones((L, L, L), np.float32)
        sim.set_fields(one, np.zeros_like(one))
        c = np.full(3, (L + 1) / 2.0)
        sim.set_particles(np.stack([c - [1.2 * R, 0, 0], c + [1.2 * R, 0, 0]]), np.zeros((2, 3)))
        sim.step(10)
        tot, _, _ = sim.time_steps(100, kernel_timing=False)
        costs[R] = tot / 100
        sim.close()
    steps_lo = info["steps_lo"]
    out = {"R_hi": R_hi, "R_lo": R_lo, "L_hi": L_hi, "steps_hi": steps_hi, "steps_lo": steps_lo,
            "classes": int(len(res["gap"])), "train_samples": int(len(X)), "epochs": epochs,
            "resistance_s": t_res, "train_s": t_train, "final_loss": float(loss[-1]),
            "held_out_direct_pairs": n_direct, "error_direct": errors(Xd, Td, info["base"]),
            "error_fresh_velocities": errors(Xv, Tv, bv),
            "ms_per_step": {"R_hi": costs[R_hi], "R_lo": costs[R_lo]},
            "cost_ratio_same_physical_time": costs[R_hi] * steps_hi / (costs[R_lo] * steps_lo)}
    return (out, w) if return_weights else out


def suspension_positions(L, n, r, seed=9, min_gap=0.1):
    """Seeded non-overlapping centres (centre distance >= 2r + min_gap) in a periodic L^3 box."""
    rng = np.random.default_rng(seed)
    x = np.zeros((0, 3))
    while len(x) < n:
        c = rng.uniform(1, L, 3)
        d = x - c
        d -= L * np.round(d / L)
        if not len(x) or (d * d).sum(1).min() >= (2 * r + min_gap) ** 2:
            x = np.vstack([x, c])
    return x


def closure_suspension(w, L=256, n=4000, r=3.0, steps=50, warm=10, seed=9):
    """The trained closure deployed: L^3 one-colour fluid with n spheres of radius r (seeded, gaps >= 0.1),
    velocities uniform in +-5e-4 (pair-frame relative velocities inside the training envelope), FP16 sum /
    difference pairs.  ms per step with the network on every close pair inside its envelope (analytic
    lubrication outside it) and with the analytic lubrication alone."""
    import ctypes
    from lbcuda_b200 import LBSim, capi, make_params
    x = suspension_positions(L, n, r, seed)
    v = np.random.default_rng(seed + 1).uniform(-5e-4, 5e-4, (n, 3))
    vol = 4.0 / 3.0 * np.pi * r ** 3
    close = 0
    for i0 in range(0, n, 500):
        d = x[i0:i0 + 500, None, :] - x[None, :, :]
        d -= L * np.round(d / L)
        dist = np.sqrt((d * d).sum(-1))
        close += int(((dist > 0) & (dist <= (2.0 + 1.5) * r)).sum())
    close //= 2
    out = {"box": L, "spheres": n, "radius": r, "volume_fraction": n * vol / L ** 3, "pairs_gap_le_1.5R": close}
    for name, on in (("closure", 1), ("analytic_only", 0)):
        p = make_params(L, model="cg", storage="f16sd", max_particles=n, radius=r, rmass=float(1.0 / vol),
                        wetting="neutral", lrotate=1, max_vel=1.0, exact_tiles=0, hz_rmin=float(2 * r - 0.5),
                        hz_rcap=float(2 * r - 2.0), closure=on, lubrication=1, lubric_k=1.0 / 6.0, lubric_rmin=1.0,
                        lubric_rcap=float(0.05 * r))
        s = LBSim(p)
        if on:
            wf = np.ascontiguousarray(w, np.float32)
            capi.check(capi.lib().lbx_closure_set(s._h, wf.ctypes.data_as(ctypes.POINTER(ctypes.c_float))),
                       "lbx_closure_set")
        one = np.ones((L, L, L), np.float32)
        s.set_fields(one, np.zeros_like(one))
        s.set_particles(x, v)
        s.step(warm)
        s.sync()
        tot, _, _ = s.time_steps(steps, kernel_timing=False)
        out[name] = {"ms_per_step": tot / steps, "device_error": s.status()[0]}
        s.close()
    out["closure_overhead"] = out["closure"]["ms_per_step"] / out["analytic_only"]["ms_per_step"] - 1.0
    return out


def summary(line):
    """The key figures of every workload in a few hundred bytes, printed last."""
    c = line["colloid_256_1280"]
    e = line["error_vs_f64"]
    r3 = lambda v: float(f"{v:.3g}")
    out = {
        "spinodal_128_f16sd": {"mlups": r3(line["value"]), "frac": r3(line["roofline"]["frac"]),
                               "fp16_over_fp32": r3(line["fp16_over_fp32"]),
                               "u_err_vs_f64_100": r3(e["f16sd"]["after_100"]["u_rel_l2"]),
                               "u_err_vs_f64_1000": r3(e["f16sd"]["after_1000"]["u_rel_l2"])},
        "colloid_256_1280_f16sd": {"ms_per_step": r3(c["f16sd"]["ms_per_step"]),
                                   "frac_at_160B": r3(c["f16sd"]["frac_at_basis"]),
                                   "over_fp32": r3(c["f32"]["ms_per_step"] / c["f16sd"]["ms_per_step"]),
                                   "u_err_vs_f64_100": r3(line["colloid_error_vs_f64"]["f16sd"]["after_100"]["u_rel_l2"])},
        "bgk_f32": {k: {"mlups": r3(v["mlups"]), "frac": r3(v["frac"])} for k, v in line["bgk"].items()},
        "ensemble_48": {"mlups": r3(line["ensemble_48"]["mlups"]),
                        "u_err_vs_f32_max": r3(line["ensemble_48"]["u_rel_l2_vs_f32_per_box"]["max"])},
    }
    cl = line.get("closure")
    if cl:
        out["closure"] = {"R_hi": cl["R_hi"], "pair_rel_l2": r3(cl["error_direct"]["closure"]["rel_l2"]),
                          "pairs_within_5pct": r3(cl["error_direct"]["closure"]["pairs_within_5pct"]),
                          "pair_cost_ratio": r3(cl["cost_ratio_same_physical_time"])}
        win = cl.get("window")
        if win:
            out["closure"]["window_force_rel_l2"] = {k: r3(win[k]["force_rel_l2"]) for k in
                                                     ("plain", "analytic_lubrication", "closure")}
            out["closure"]["window_cost_ratio"] = r3(win["cost_ratio_same_physical_time"])
    return out


def only_region(args, local):
    import torch
    torch.cuda.set_device(local)
    from lbcuda_b200 import LBSim, make_params
    from lbcuda_b200.inputs import seeded_noise_fields
    if args.only == "closure":
        res, w = closure_experiment(return_weights=True)
        res["suspension"] = closure_suspension(w)
        print(json.dumps(res), flush=True)
        return 0
    if args.only == "closure12":
        from lbcuda_b200 import closure as _cl
        res, w = closure_experiment(R_hi=12, L_hi=96, steps_hi=960, return_weights=True)
        res["window"] = _cl.window_score(w)
        print(json.dumps(res), flush=True)
        return 0
    if args.only == "ensemble-closure":
        r4, w4 = closure_experiment(R_hi=8, L_hi=64, R_lo=4, steps_hi=432, n_direct=32, return_weights=True)
        if args.save_weights:
            np.save(args.save_weights, np.asarray(w4, np.float32))
        res = ensemble_timing(weights=w4)
        res["closure_r4"] = r4
        print(json.dumps(res), flush=True)
        return 0
    if args.only == "ensemble-profile":
        # the ensemble workload's 48 boxes (FP16 sum / difference pairs), a few eager steps: profiler captures
        from lbcuda_b200.ensemble import Ensemble, random_boxes
        import ctypes
        from lbcuda_b200 import capi
        spec = random_boxes(48, seed=7)
        ens = Ensemble([make_params(Lb, model="cg", storage="f16sd", sigma=SIGMA, beta=BETA, max_particles=max(len(x), 1),
                                    radius=4.0, wetting="neutral", lrotate=1, max_vel=1.0, exact_tiles=0,
                                    hz_rmin=8.5, hz_rcap=7.0, closure=1, lubrication=1, lubric_rmin=1.0,
                                    lubric_rcap=0.2) for Lb, x in spec])
        wf = np.ascontiguousarray(np.load(CLOSURE_R4), np.float32)
        for i, (Lb, x) in enumerate(spec):
            rR, rB = seeded_noise_fields(Lb, Lb, Lb, seed=100 + i)
            ens.boxes[i].set_fields(rR, rB)
            if len(x):
                ens.boxes[i].set_particles(x, np.zeros_like(x))
                capi.check(capi.lib().lbx_closure_set(ens.boxes[i]._h, wf.ctypes.data_as(ctypes.POINTER(ctypes.c_float))),
                           "lbx_closure_set")
        ms = ens.time(max(1, args.steps) * 2)
        print(json.dumps({"only": args.only, "cells": ens.cells, "ms_per_step": ms / (max(1, args.steps) * 2)}),
              flush=True)
        ens.close()
        return 0
    if args.only == "mlp-profile":
        # a short training and one inference batch of the closure network: profiler captures
        from lbcuda_b200 import closure as _cl
        rng = np.random.default_rng(0)
        X = rng.uniform(-1, 1, (2048, _cl.DIN)).astype(np.float32)
        T = np.tanh(X[:, :_cl.DOUT]).astype(np.float32)
        t0 = time.perf_counter()
        w, loss = _cl.train(X, T, epochs=max(1, args.steps), lr=2e-3)
        t1 = time.perf_counter()
        Y = _cl.infer(w, np.repeat(X, 2, axis=0))
        t2 = time.perf_counter()
        print(json.dumps({"only": args.only, "train_s": t1 - t0, "infer_s": t2 - t1, "loss": float(loss[-1]),
                          "finite": bool(np.isfinite(Y).all())}), flush=True)
        return 0
    if args.only == "bgk":
        print(json.dumps({"64": bgk_timing(64, 2000), "256": bgk_timing(256, 200), "512": bgk_timing(512, 40)}),
              flush=True)
        return 0
    if args.only == "bgk-256":
        print(json.dumps(bgk_timing(256, max(1, args.steps) * 5, warm=args.warmup)), flush=True)
        return 0
    if args.only == "ensemble":
        print(json.dumps(ensemble_timing()), flush=True)
        return 0
    if args.only == "errors":
        print(json.dumps({"spinodal": error_vs_f64((100, 1000)),
                          "droplet": error_vs_f64((100, 1000), workload="droplet"),
                          "colloid": colloid_error_vs_f64()}), flush=True)
        return 0
    if args.only == "variants":
        print(json.dumps({st: variants_timing(st) for st in ("f32", "f16")}), flush=True)
        return 0
    if args.only.startswith("colloid"):
        r = colloid_timing(args.only.split("-")[1], steps=max(1, args.steps) * 5, warm=args.warmup,
                           small=args.only.endswith("small"))
        print(json.dumps(r), flush=True)
        return 0
    Lb = args.box
    rR, rB = seeded_noise_fields(Lb, Lb, Lb, seed=SEED)
    s = LBSim(make_params(Lb, model="cg", storage=args.only, sigma=SIGMA, beta=BETA))
    s.set_schedule(args.schedule)
    if args.zlen or args.shape:
        s.set_lean_shape(args.shape, args.zlen)
    s.set_lean_copies(args.lean_copies)
    s.set_fields(rR, rB)
    s.step(args.warmup * args.lb_steps)
    s.sync()
    tot, k, nl = s.time_steps(args.steps * args.lb_steps, kernel_timing=args.schedule != 0)
    n = args.steps * args.lb_steps
    kus = (k / nl * 1e3) if nl else None
    print(json.dumps({"only": args.only, "box": Lb, "schedule": args.schedule, "zlen": args.zlen or "auto",
                      "lean_copies": args.lean_copies, "shape": args.shape,
                      "ms_per_lattice_step": tot / n,
                      "mlups": Lb ** 3 * n / (tot * 1e-3) / 1e6, "kernel_us": kus,
                      "frac_at_basis": (BYTES_PER_CELL[args.only] * Lb ** 3 / (kus * 1e-6) / 1e9 / peaks()[0])
                      if kus else None}), flush=True)
    s.close()
    return 0


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--gpus", type=int, default=1)
    ap.add_argument("--steps", type=int, default=20)
    ap.add_argument("--warmup", type=int, default=3)
    ap.add_argument("--impl", default="ours", choices=["ours", "reference"])
    ap.add_argument("--no-extras", action="store_true", help="skip the error runs, the colloid case and the CPU baseline")
    ap.add_argument("--only", choices=["f16", "f32", "bf16", "f64", "f16sd", "bf16sd", "f16sdp", "bf16sdp", "colloid-f16", "colloid-f32", "colloid-f16-small", "colloid-f16sd", "colloid-f16sd-small",
                                       "colloid-f32-small", "ensemble", "ensemble-closure", "ensemble-profile", "mlp-profile", "closure",
                                       "closure12", "variants", "errors", "bgk",
                                       "bgk-256"],
                    help="profiling aid: run one timed region only and print its timing")
    ap.add_argument("--lb-steps", type=int, default=LB_PER_STEP, help="lattice steps per bench step")
    ap.add_argument("--schedule", type=int, default=2, help="colour-gradient schedule (0, 1, 2)")
    ap.add_argument("--box", type=int, default=L, help="lattice edge of the --only storage runs")
    ap.add_argument("--zlen", type=int, default=0,
                    help="--only storage runs: equal z-segments of this length (0: automatic plan)")
    ap.add_argument("--decomp", default="replicas", choices=["replicas", "slab"],
                    help="headline with N GPUs: independent boxes (default) or z-slabs of one box, halo planes "
                         "exchanged over NCCL every lattice step")
    ap.add_argument("--shape", type=int, default=0, help="--only storage runs: lean kernel CTA, 0 = 32x8, 1 = 32x16")
    ap.add_argument("--lean-copies", type=int, default=1,
                    help="--only storage runs: 16-bit pulls as box granules (1) or one copy per pull (0)")
    ap.add_argument("--save-weights", default=None,
                    help="--only ensemble-closure: write the trained radius-4 closure weights (.npy) here")
    args = ap.parse_args()
    ws, rank, local = dist_env()
    if args.impl == "reference":
        return reference_arm(args, ws, rank)
    if args.only:
        return only_region(args, local)

    import torch
    torch.cuda.set_device(local)
    pg = None
    if ws > 1:
        import datetime
        import torch.distributed as dist
        dist.init_process_group("nccl", timeout=datetime.timedelta(seconds=120))
        pg = dist

    from lbcuda_b200 import LBSim, make_params
    from lbcuda_b200.inputs import seeded_noise_fields

    rR, rB = seeded_noise_fields(L, L, L, seed=SEED + rank)
    hbm, peak_kind = peaks()

    def barrier():
        torch.cuda.synchronize()
        if pg is not None:
            pg.barrier()

    def run_storage(storage, timed_steps, warm):
        s = LBSim(make_params(L, model="cg", storage=storage, sigma=SIGMA, beta=BETA))
        s.set_fields(rR, rB)
        for _ in range(warm):
            s.step(LB_PER_STEP)
        s.sync()
        barrier()
        clk = Clocks(local)
        clk.start()
        total_ms, kernel_ms, launches = s.time_steps(timed_steps * LB_PER_STEP, kernel_timing=True)
        clocks = clk.stop()
        barrier()
        code = s.status()[0]
        s.close()
        return total_ms, kernel_ms, launches, clocks, code

    def run_slab(storage, timed_steps, warm):
        """Rank r's 128^3 z-slab of a 128 x 128 x (128 N) periodic box: halo planes swapped with the
        neighbouring ranks every lattice step (NCCL; one rank: with itself), CUDA events on the slab's
        stream.  Returns the same tuple as run_storage (the kernel time is not split out)."""
        from lbcuda_b200.slabs import DistExchange, LocalExchange, Slab
        pg_ = make_params(L, L, L * ws, model="cg", storage=storage, sigma=SIGMA, beta=BETA)
        gR, gB = seeded_noise_fields(L, L, L * ws, seed=SEED)
        slab = Slab(pg_, rank, ws)
        slab.set_fields(gR, gB)
        ex = DistExchange(slab, "cuda") if pg is not None else LocalExchange([slab])
        for _ in range(warm):
            ex.step(LB_PER_STEP)
        slab.sync()
        barrier()
        clk = Clocks(local)
        clk.start()
        e0, e1 = torch.cuda.Event(enable_timing=True), torch.cuda.Event(enable_timing=True)
        e0.record(slab.stream)
        ex.step(timed_steps * LB_PER_STEP)
        e1.record(slab.stream)
        e1.synchronize()
        clocks_ = clk.stop()
        barrier()
        code = slab.sim.status()[0]
        slab.close()
        # one fluid kernel per lattice step (the halo copies are not kernels)
        return e0.elapsed_time(e1), 0.0, timed_steps * LB_PER_STEP, clocks_, code

    # headline: FP16 storage as sum / difference pairs (R + B - w (rho0R + rho0B), R - B); beside it the
    # FP16 (R, B) pairs the sphere path stores, and FP32
    if args.decomp == "slab":
        tot16, k16, n16, clocks, code16 = run_slab("f16sd", args.steps, args.warmup)
    else:
        tot16, k16, n16, clocks, code16 = run_storage("f16sd", args.steps, args.warmup)
    tot32, k32, n32, _, code32 = run_storage("f32", args.steps, args.warmup)
    totrb, krb, nrb, _, coderb = run_storage("f16", args.steps, args.warmup)
    totsp, ksp, nsp, _, codesp = run_storage("f16sdp", args.steps, args.warmup)

    def maxr(v):
        return max_over_ranks(v, pg, "cuda")

    tot16, tot32, totrb, totsp = maxr(tot16), maxr(tot32), maxr(totrb), maxr(totsp)
    cells = L ** 3
    lb_steps = args.steps * LB_PER_STEP
    mlups16 = ws * cells * lb_steps / (tot16 * 1e-3) / 1e6
    mlups32 = ws * cells * lb_steps / (tot32 * 1e-3) / 1e6
    mlupsrb = ws * cells * lb_steps / (totrb * 1e-3) / 1e6
    mlupssp = ws * cells * lb_steps / (totsp * 1e-3) / 1e6

    def roofline(storage, kernel_ms, launches):
        per_launch_ms = kernel_ms / max(launches, 1)
        alg = BYTES_PER_CELL[storage] * cells
        achieved = alg / (per_launch_ms * 1e-3) / 1e9
        return {"bound": "hbm", "achieved": achieved, "peak": hbm, "unit": "GB/s", "frac": achieved / hbm,
                "traffic": TRAFFIC.get(storage), "traffic_source": "ncu dram__bytes_read.sum + dram__bytes_write.sum, "
                "one launch at 128^3 (profiles/)", "peak_kind": peak_kind, "kernel": "k_cg_lean",
                "bytes_per_cell": BYTES_PER_CELL[storage],
                "kernel_us_per_launch": per_launch_ms * 1e3,
                "minimal_bytes_frac": MINIMAL_BYTES[storage] * cells / (per_launch_ms * 1e-3) / 1e9 / hbm}

    # e2e through the public API with host buffers, one continuous trajectory:
    # each bench step uploads the full population state from pinned host
    # memory (lbx_set_pops), runs one bench step of lattice steps and reads
    # the state back (lbx_get_pops), which the next step uploads again
    import ctypes
    pin = lambda shape: torch.empty(shape, dtype=torch.float32, pin_memory=True).numpy()
    s = LBSim(make_params(L, model="cg", storage="f16sd", sigma=SIGMA, beta=BETA))
    s.set_fields(rR, rB)
    hR, hB = pin((19, L, L, L)), pin((19, L, L, L))
    fp = lambda a: a.ctypes.data_as(ctypes.POINTER(ctypes.c_float))
    lib = s._L
    if lib.lbx_get_pops(s._h, fp(hR), fp(hB)):
        raise RuntimeError("lbx_get_pops")

    def e2e_step():
        rc = lib.lbx_set_pops(s._h, fp(hR), fp(hB))
        rc = rc or lib.lbx_step(s._h, LB_PER_STEP)
        rc = rc or lib.lbx_get_pops(s._h, fp(hR), fp(hB))
        if rc:
            raise RuntimeError(f"e2e step: lbx status {rc}")

    for _ in range(args.warmup):
        e2e_step()
    barrier()
    t0 = time.perf_counter()
    for _ in range(args.steps):
        e2e_step()
    barrier()
    e2e_wall = time.perf_counter() - t0
    e2e_ms = maxr(e2e_wall * 1e3)
    s.close()
    e2e_mlups = ws * cells * lb_steps / (e2e_ms * 1e-3) / 1e6

    extras = {}
    if rank == 0 and not args.no_extras:
        extras["error_vs_f64"] = error_vs_f64()
        extras["error_vs_f64_droplet"] = error_vs_f64((100, 1000), workload="droplet")
        extras["bgk"] = {"64": bgk_timing(64, 2000), "256": bgk_timing(256, 200), "512": bgk_timing(512, 40)}
        extras["colloid_256_1280"] = {st: colloid_timing(st) for st in ("f16sd", "f16", "f32")}
        extras["colloid_error_vs_f64"] = colloid_error_vs_f64()
        extras["variants_128"] = {st: variants_timing(st) for st in ("f32", "f16")}
        from lbcuda_b200 import closure as _cl
        # the task's closure: radius-3 pairs against radius-12 resolved ones
        extras["closure"], w = closure_experiment(R_hi=12, L_hi=96, steps_hi=960, return_weights=True)
        extras["closure"]["window"] = _cl.window_score(w)
        extras["closure"]["suspension"] = closure_suspension(w)
        # the ensemble's spheres have radius 4: its closure (R_lo = 4 trained against R_hi = 8 by
        # `bench.py --only ensemble-closure --save-weights ...`, the same pipeline as above) is an input
        # of the ensemble workload, loaded from the weights that run wrote
        extras["ensemble_48"] = ensemble_timing(weights=np.load(CLOSURE_R4))
        extras["ensemble_48"]["closure_weights"] = os.path.relpath(CLOSURE_R4, ROOT)
        extras["cpu_baseline"] = cpu_baseline_sample()

    if rank == 0:
        line = {
            "metric": METRIC, "value": mlups16, "unit": "MLUPS", "n_gpus": ws, "steps": args.steps,
            "warmup": args.warmup, "ms_per_step": tot16 / args.steps, "higher_is_better": True,
            "scaling": "weak", "vs_baseline": None, "dtype": "f32", "data": "synthetic",
            "config": workload_config(),
            "storage": "f16 sum / difference pairs (f_R + f_B - w*1, f_R - f_B), FP32 arithmetic",
            "lattice_steps_per_bench_step": LB_PER_STEP,
            "parallelism": ("z-slabs, halo planes over NCCL" if args.decomp == "slab" else "replicas")
            if ws > 1 else ("one z-slab exchanging with itself" if args.decomp == "slab" else "single"),
            "roofline": roofline("f16sd", k16, n16) if k16 > 0 else None,
            "fp32_storage": {"value": mlups32, "unit": "MLUPS", "ms_per_step": tot32 / args.steps,
                             "roofline": roofline("f32", k32, n32)},
            "fp16_over_fp32": mlups16 / mlups32,
            "f16_component_pairs": {"value": mlupsrb, "unit": "MLUPS", "ms_per_step": totrb / args.steps,
                                    "storage": "f16 (R - w rho0R, B - w rho0B) pairs",
                                    "roofline": roofline("f16", krb, nrb), "over_fp32": mlupsrb / mlups32},
            "f16_predicted_split": {"value": mlupssp, "unit": "MLUPS", "ms_per_step": totsp / args.steps,
                                    "storage": "f16 (total, colour difference less the receiving cell's predicted "
                                               "split) pairs + an FP32 phase field per cell",
                                    "roofline": roofline("f16sdp", ksp, nsp), "over_fp32": mlupssp / mlups32},
            "clocks": clocks,
            "e2e": {"value": e2e_mlups, "unit": "MLUPS", "h2d_bytes_per_step": 2 * 19 * 4 * cells,
                    "d2h_bytes_per_step": 2 * 19 * 4 * cells, "ms_per_step": e2e_ms / args.steps,
                    "timing": "host wall clock around the synchronous C-ABI calls (lbx_set_pops, lbx_step, "
                              "lbx_get_pops of the full FP32 state, one continuous trajectory), max over ranks",
                    "gpu_launches_per_step": LB_PER_STEP + 2},
            "gpu_launches": n16,
            "device_errors": [code16, code32, coderb, codesp],
        }
        line.update(extras)
        if extras:
            line["summary"] = summary(line)
        print(json.dumps(line), flush=True)
    if pg is not None:
        pg.destroy_process_group()
    return 0


if __name__ == "__main__":
    sys.exit(main())
