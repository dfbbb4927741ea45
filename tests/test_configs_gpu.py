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
  densities and phase field:                           1e-5 (max |gpu - oracle| / max |oracle|)
  velocity field:                                      1e-5 (relative L2) where the flow is
      resolved above FP32 rounding; the spinodal at rest holds 5e-5 (its velocity, ~1e-4, is the
      difference of momenta ~3e-2), and the same spinodal with a mean flow holds 1e-5
  particle positions / orientation:                    1e-6 absolute
  particle forces / torques / velocities:              1e-5 relative to the largest
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


@pytest.mark.parametrize("flow", [(0.0, 0.0, 0.0), (0.02, 0.01, 0.005)])
def test_cg_spinodal_128cube_100_steps(flow):
    n = 128
    p = make_params(n, model="cg", storage="f32", sigma=0.02, beta=0.7)
    rR, rB = seeded_noise_fields(n, n, n, seed=SEED)
    g = LBSim(p)
    g.set_fields(rR, rB, flow)
    g.step(100)
    o = OracleSim(p, "ref")
    o.set_fields(rR, rB, flow)
    assert o.step(100) == 0
    assert g.status()[0] == 0
    gf, of = g.get_fields(), o.get_fields()
    for name, a, b in zip(("rhoR", "rhoB", "phase"), (gf[0], gf[1], gf[3]), (of[0], of[1], of[3])):
        assert rel(a, b) <= TOL, name
    tol_u = TOL if any(flow) else 5e-5
    assert rel_l2(gf[2], of[2]) <= tol_u


def test_colloid_256cube_1280_spheres_5_steps():
    n, ns = 256, 1280
    x, _, q = read_input_xyz(DECK, ns, True)
    vol = 4.0 / 3.0 * np.pi * 5.5 ** 3
    p = make_params(n, model="cg", storage="f32", sigma=0.02, beta=0.7, max_particles=ns, radius=5.5,
                    rmass=float(1.0 / vol), wetting="neutral", lrotate=1, max_vel=1.0)
    rR, rB = seeded_noise_fields(n, n, n, seed=SEED)
    v = np.zeros_like(x)
    g = LBSim(p)
    g.set_fields(rR, rB)
    g.set_particles(x, v, None, q)
    o = OracleSim(p, "f32p64")
    o.set_fields(rR, rB)
    o.set_particles(x, v, None, q)
    o.record_links(True)
    g.step(5)
    assert o.step(5) == 0
    assert g.status()[0] == 0
    assert np.array_equal(g.get_flags(), o.get_flags())
    lg, lo = g.get_links(), o.get_links()
    assert lg.shape[0] > 400 * ns            # ~5 crossing links per surface cell, 410 surface cells
    assert np.array_equal(lg, lo)
    gp, op = g.get_particles(), o.get_particles()
    assert np.abs(gp["x"] - op["x"]).max() < 1e-6
    assert np.abs(gp["q"] - op["q"]).max() < 1e-6
    for key in ("v", "omega", "force", "torque"):
        assert rel(gp[key], op[key]) < TOL, key
    gf, of = g.get_fields(), o.get_fields()
    for name, a, b in zip(("rhoR", "rhoB", "phase"), (gf[0], gf[1], gf[3]), (of[0], of[1], of[3])):
        assert rel(a, b) <= TOL, name
    assert rel_l2(gf[2], of[2]) <= 5e-5
