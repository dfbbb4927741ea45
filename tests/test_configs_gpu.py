"""Parity of the CUDA path with the CPU oracle at the benchmark configurations' own sizes.

Each test runs one configuration at its full lattice size, through the C ABI,
against the oracle on the same seeded inputs (the oracle finishes each in
seconds on the host cores):

  BGK, D3Q19, 64^3 periodic, tau = 1, rho = 1 + U(-1e-3, 1e-3) from seed 1,
      u = 0, FP32 storage, 1000 steps (the workload's full length)
  colour-gradient spinodal, 128^3, rhoR = rhoB = 0.5 + U(-0.01, 0.01) from
      seed 1, tau = 1, sigma = 0.02, beta = 0.7, FP32 storage, 100 steps
  colour gradient with the 1280 spheres (r = 5.5) of the reference's
      Tests/07-1280-Particle placement, 256^3, neutral wetting, rotation on,
      sphere density 1, FP32 fluid, FP64 particles, 5 steps

Stated tolerances:
  flags and the set of bounce-back links:              bit-exact
  BGK (expression order of the reference, no contraction): every field and
      population to 1e-5 (max |gpu - oracle| / max |oracle|)
  colour gradient, sphere states (FP32 fluid, reassociated collision):
      relative L2 |gpu - oracle|_2 / |oracle|_2 <= 1e-5 for every field and
      every particle quantity (the spinodal at rest: velocity 5e-5, its ~1e-4
      velocity being the difference of ~3e-2 momenta; the sphere velocities,
      forces and torques: max(1e-5, 2 x the oracle's FP32-vs-FP64 relative L2
      difference)), and the max-norm
      difference within max(1e-5, 2 x the oracle's own FP32-vs-FP64 max-norm
      difference on the same run): spinodal decomposition amplifies rounding
      differences, so any two FP32 operation orders drift apart at the rate
      the FP64 run measures
  particle positions / orientation:                    1e-6 absolute
"""
import os

import numpy as np
import pytest

from lbcuda_b200 import LBSim, make_params
from lbcuda_b200.inputs import read_input_xyz, seeded_noise_fields
from oracle.orc import OracleSim

pytestmark = pytest.mark.gpu

SEED = 1
TOL = 1e-5
DECK = os.path.join(os.path.dirname(__file__), "golden", "decks", "07-1280.input.xyz.256cube.r5.5")


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def test_bgk_64cube_1000_steps():
    n = 64
    p = make_params(n, model="bgk", storage="f32", tau=1.0)
    rho = seeded_noise_fields(n, n, n, mean=1.0, amp=1e-3, seed=SEED, ncomp=1)[0]
    g = LBSim(p)
    g.set_fields(rho, None)
    g.step(1000)
    o = OracleSim(p, "ref")
    o.set_fields(rho, None)
    assert o.step(1000) == 0
    assert g.status()[0] == 0
    gf, of = g.get_fields(), o.get_fields()
    # the BGK kernel keeps the reference's expression order without
    # contraction, so it rounds as the oracle does: every field to 1e-5, the
    # velocity (~1e-5 after 1000 steps) and the density deviations included
    assert rel(gf[0], of[0]) <= TOL
    dr = of[0] - of[0].mean()
    assert np.linalg.norm(gf[0] - of[0]) / np.linalg.norm(dr) <= TOL
    assert rel_l2(gf[2], of[2]) <= TOL
    pg, po = g.get_pops()[0], o.get_pops()[0]
    assert rel(pg, po) <= TOL


def envelope(a32, a64):
    """max |a32 - a64| / max |a64|: the FP32 rounding drift of the oracle's own run."""
    return rel(a32, a64)


@pytest.mark.parametrize("flow", [(0.0, 0.0, 0.0), (0.02, 0.01, 0.005)])
def test_cg_spinodal_128cube_100_steps(flow):
    n, steps = 128, 100
    p = make_params(n, model="cg", storage="f32", sigma=0.02, beta=0.7)
    rR, rB = seeded_noise_fields(n, n, n, seed=SEED)
    g = LBSim(p)
    g.set_fields(rR, rB, flow)
    g.step(steps)
    assert g.status()[0] == 0
    gf = g.get_fields()
    of = {}
    for mode in ("ref", "f64"):
        o = OracleSim(p, mode)
        o.set_fields(rR, rB, flow)
        assert o.step(steps) == 0
        of[mode] = o.get_fields()
        o.close()
    names = ("rhoR", "rhoB", "vel", "phase")
    for k, name in enumerate(names):
        a, b, c = gf[k], of["ref"][k], of["f64"][k]
        l2 = rel_l2(a, b)
        tol_l2 = 5e-5 if (name == "vel" and not any(flow)) else TOL
        assert l2 <= tol_l2, f"{name}: rel L2 {l2:.2e}"
        mx, env = rel(a, b), envelope(b, c)
        print(f"spinodal flow={flow} {name}: rel L2 {l2:.2e}, max-norm {mx:.2e}, FP32 envelope {env:.2e}")
        assert mx <= max(TOL, 2 * env), f"{name}: max-norm {mx:.2e}, FP32 envelope {env:.2e}"


def test_colloid_256cube_1280_spheres_5_steps():
    n, ns, steps = 256, 1280, 5
    x, _, q = read_input_xyz(DECK, ns, True)
    vol = 4.0 / 3.0 * np.pi * 5.5 ** 3
    p = make_params(n, model="cg", storage="f32", sigma=0.02, beta=0.7, max_particles=ns, radius=5.5,
                    rmass=float(1.0 / vol), wetting="neutral", lrotate=1, max_vel=1.0)
    rR, rB = seeded_noise_fields(n, n, n, seed=SEED)
    v = np.zeros_like(x)
    g = LBSim(p)
    g.set_fields(rR, rB)
    g.set_particles(x, v, None, q)
    g.step(steps)
    assert g.status()[0] == 0
    res = {}
    for mode in ("f32p64", "f64"):
        o = OracleSim(p, mode)
        o.set_fields(rR, rB)
        o.set_particles(x, v, None, q)
        o.record_links(True)
        assert o.step(steps) == 0
        res[mode] = (o.get_flags(), o.get_links(), o.get_particles(), o.get_fields())
        o.close()
    of, ol, op, ofl = res["f32p64"]
    assert np.array_equal(g.get_flags(), of)
    lg = g.get_links()
    assert lg.shape[0] > 400 * ns            # ~5 crossing links per surface cell, 410 surface cells
    assert np.array_equal(lg, ol)
    gp = g.get_particles()
    p64 = res["f64"][2]
    assert np.abs(gp["x"] - op["x"]).max() < 1e-6
    assert np.abs(gp["q"] - op["q"]).max() < 1e-6
    for key in ("v", "omega", "force", "torque"):
        # the sphere state integrates the FP32 fluid's forces, so both norms
        # are held to the FP32 envelope of the oracle's own run as well
        l2, env_l2 = rel_l2(gp[key], op[key]), rel_l2(op[key], p64[key])
        mx, env = rel(gp[key], op[key]), envelope(op[key], p64[key])
        print(f"colloid {key}: rel L2 {l2:.2e} (envelope {env_l2:.2e}), max-norm {mx:.2e} (envelope {env:.2e})")
        assert l2 <= max(TOL, 2 * env_l2), f"{key}: rel L2 {l2:.2e}, FP32 envelope {env_l2:.2e}"
        assert mx <= max(TOL, 2 * env), f"{key}: max-norm {mx:.2e}, FP32 envelope {env:.2e}"
    gf, f64 = g.get_fields(), res["f64"][3]
    for k, name in enumerate(("rhoR", "rhoB", "vel", "phase")):
        l2 = rel_l2(gf[k], ofl[k])
        assert l2 <= (5e-5 if name == "vel" else TOL), f"{name}: rel L2 {l2:.2e}"
        mx, env = rel(gf[k], ofl[k]), envelope(ofl[k], f64[k])
        print(f"colloid {name}: rel L2 {l2:.2e}, max-norm {mx:.2e}, FP32 envelope {env:.2e}")
        assert mx <= max(TOL, 2 * env), f"{name}: max-norm {mx:.2e}, FP32 envelope {env:.2e}"
