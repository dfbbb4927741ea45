"""Parity of the CUDA particle path against the CPU oracle, through the C ABI.

The GPU keeps particle state in FP64, so it is compared with the oracle in
mode "f32p64" (FP32 fluid, FP64 particles).  Stated tolerances:
  flags (solid/fluid, surface, dead):      bit-exact
  fluid fields on fluid cells:             1e-5 relative (max-norm; velocity in L2)
  particle positions / orientation:        1e-6 absolute (FP32 fluid forces
                                           differ at 1e-7 and are integrated)
  particle velocities, forces, torques:    1e-5 relative to the largest
"""
import numpy as np
import pytest

from lbcuda_b200 import LBSim, make_params
from lbcuda_b200.inputs import seeded_noise_fields
from oracle.orc import OracleSim

pytestmark = pytest.mark.gpu


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def make_pair(n, x, v, omega=None, q=None, steps=0, fields=None, sched=2, **kw):
    kw.setdefault("max_vel", 1.0)
    p = make_params(n, model="cg", storage="f32", max_particles=len(x), **kw)
    if fields is None:
        r = np.full((n, n, n), 0.5, np.float32)
        fields = (r, r)
    g = LBSim(p)
    g.set_schedule(sched)
    g.set_fields(*fields)
    g.set_particles(x, v, omega, q)
    o = OracleSim(p, "f32p64")
    o.set_fields(*fields)
    o.set_particles(x, v, omega, q)
    if steps:
        g.step(steps)
        assert o.step(steps) == 0
    return g, o


def test_template_counts_r55():
    """spherical_template for rdim = 5.5: 410 surface, 328 dead cells + the centre."""
    g, o = make_pair(32, np.array([[16.0, 16.0, 16.0]]), np.zeros((1, 3)))
    t = o.template()
    assert (t == 2).sum() == 410 and (t == 4).sum() == 328 and (t == 5).sum() == 1
    f = g.get_flags()
    assert (f == 2).sum() == 410 and (f == 4).sum() == 328 and (f == 5).sum() == 1


def test_flags_bit_exact_with_periodic_wrap():
    x = np.array([[1.4, 16.2, 30.6], [20.5, 2.49, 17.0], [12.0, 25.7, 5.51], [28.3, 9.9, 25.2]])
    g, o = make_pair(32, x, np.zeros((4, 3)))
    assert np.array_equal(g.get_flags(), o.get_flags())


@pytest.mark.parametrize("sched", [2, 0])
@pytest.mark.parametrize("wetting", ["janus", "neutral"])
@pytest.mark.parametrize("lrotate", [0, 1])
def test_moving_spheres_match_oracle(wetting, lrotate, sched):
    """25 steps with fill/drain (the spheres cross cell boundaries), single-pass (2) and two-pass (0) fluid."""
    n = 32
    x = np.array([[8.3, 9.1, 10.2], [22.6, 20.4, 24.9], [15.2, 27.7, 3.1]])
    v = np.array([[0.04, -0.03, 0.02], [-0.05, 0.01, 0.03], [0.02, 0.04, -0.05]])
    om = np.array([[0.0, 0.0, 0.01], [0.005, -0.004, 0.0], [0.0, 0.006, 0.003]]) if lrotate else None
    rR, rB = seeded_noise_fields(n, n, n, seed=3)
    g, o = make_pair(n, x, v, om, None, steps=25, fields=(rR, rB), lrotate=lrotate, wetting=wetting,
                     sigma=0.02, beta=0.7, sched=sched)
    assert g.status()[0] == 0 and o.status()[0] == 0
    assert np.array_equal(g.get_flags(), o.get_flags())
    gp, op = g.get_particles(), o.get_particles()
    assert np.abs(gp["x"] - op["x"]).max() < 1e-6
    assert rel(gp["v"], op["v"]) < 1e-5
    assert rel(gp["force"], op["force"]) < 1e-5
    if lrotate:
        assert np.abs(gp["q"] - op["q"]).max() < 1e-6
        assert rel(gp["omega"], op["omega"]) < 1e-5
        assert rel(gp["torque"], op["torque"]) < 1e-5
    gf, of = g.get_fields(), o.get_fields()
    for name, a, b in zip(("rhoR", "rhoB", "vel", "phase"), gf, of):
        e = (np.linalg.norm(a - b) / np.linalg.norm(b)) if name == "vel" else rel(a, b)
        assert e <= 1e-5, (name, e)


def test_hertz_contact_pair():
    """Two overlapping spheres (Hertz force of addHertzian plus fluid forces) match the oracle."""
    x = np.array([[12.0, 16.0, 16.0], [22.2, 16.3, 16.1]])
    g, o = make_pair(32, x, np.zeros((2, 3)), steps=3, wetting="neutral")
    gp, op = g.get_particles(), o.get_particles()
    assert rel(gp["force"], op["force"]) < 1e-5
    assert np.abs(gp["x"] - op["x"]).max() < 1e-6


@pytest.mark.parametrize("exact", [1, 0])
def test_integer_radius_flags(exact):
    """Radius 4: the reference's tile lists (int(x +- r) boxes) miss template cells
    when frac(x) >= 0.5; exact_tiles = 1 reproduces that, 0 places every cell."""
    x = np.array([[10.7, 16.6, 12.2], [22.3, 9.5, 21.8]])
    g, o = make_pair(32, x, np.zeros((2, 3)), radius=4.0, exact_tiles=exact)
    fg, fo = g.get_flags(), o.get_flags()
    assert np.array_equal(fg, fo)
    solid = int((fg != 1).sum())
    if exact:
        assert solid < 2 * 257  # a full r = 4 sphere has 257 cells
    else:
        assert solid == 2 * 257


def test_reference_deck_placement_flags():
    """The first 16 spheres of the reference's 256^3 r=5.5 placement, shifted into 64^3 boxes."""
    import os
    from lbcuda_b200.inputs import read_input_xyz
    deck = os.path.join(os.path.dirname(__file__), "golden", "decks", "07-1280.input.xyz.256cube.r5.5")
    x, v, q = read_input_xyz(deck, 1280, True)
    sel = x[(x < 64).all(axis=1)][:16]
    g, o = make_pair(64, sel, np.zeros_like(sel), q=None)
    assert np.array_equal(g.get_flags(), o.get_flags())


@pytest.mark.parametrize("kinematic", [1, 2])
def test_kinematic_pair_parity(kinematic):
    """Prescribed-motion (1) and frozen-geometry (2) spheres, the closure's force probes, across the
    periodic boundary."""
    x = np.array([[4.0, 16.0, 16.0], [24.3, 16.5, 15.8]])   # periodic distance 11.71, gap 0.71
    v = np.array([[-0.01, 0.002, 0.0], [0.01, -0.002, 0.001]])
    om = np.array([[0.0, 0.0, 0.002], [0.001, 0.0, 0.0]])
    g, o = make_pair(32, x, v, om, steps=20, wetting="neutral", kinematic=kinematic, lrotate=1)
    gp, op = g.get_particles(), o.get_particles()
    assert np.array_equal(g.get_flags(), o.get_flags())
    assert np.abs(gp["x"] - op["x"]).max() < 1e-9
    assert rel(gp["force"], op["force"]) < 1e-5
    assert rel(gp["torque"], op["torque"]) < 1e-5


STAGES = ["lbx_make_list_atoms", "lbx_init_isfluid", "lbx_del_fluid", "lbx_init_rho", "lbx_make_fluid",
          "lbx_virtual_rho", "lbx_time_step_cg", "lbx_partbb", "lbx_partbb_p2n", "lbx_partbb_p2n2",
          "lbx_inter_force_particles", "lbx_time_step_force_particles"]


@pytest.mark.parametrize("sched", [2, 0])
def test_kernel_level_entries_equal_step(sched):
    """The reference's launch order (main.CUF:130-240) through the kernel-level entries gives lbx_step's state
    bit for bit, with spheres crossing cell boundaries (drain and fill active)."""
    from lbcuda_b200 import capi
    n = 32
    x = np.array([[10.3, 16.2, 15.7], [22.6, 15.1, 17.4]])
    v = np.array([[0.05, -0.01, 0.005], [-0.04, 0.03, 0.0]])
    om = np.array([[0.0, 0.01, 0.0], [0.005, 0.0, -0.01]])
    rR, rB = seeded_noise_fields(n, n, n, seed=4)
    sims = []
    for _ in range(2):
        p = make_params(n, model="cg", storage="f32", max_particles=2, max_vel=1.0, lrotate=1, sigma=0.02, beta=0.7)
        s = LBSim(p)
        s.set_schedule(sched)
        s.set_fields(rR, rB)
        s.set_particles(x, v, om, None)
        sims.append(s)
    a, b = sims
    a.step(16)
    L = capi.lib()
    for _ in range(16):
        for name in STAGES:
            assert getattr(L, name)(b._h) == 0, name
    assert a.status()[0] == 0 and b.status()[0] == 0
    assert a.steps_taken == b.steps_taken == 16
    assert np.array_equal(a.get_flags(), b.get_flags())
    pa, pb = a.get_pops(), b.get_pops()
    assert np.array_equal(pa[0], pb[0]) and np.array_equal(pa[1], pb[1])
    da, db = a.get_particles(), b.get_particles()
    for k in da:
        assert np.array_equal(da[k], db[k]), k
    assert (np.rint(da["x"]) != np.rint(x)).any()   # a sphere changed cell: drain and fill ran


def test_large_radius_spans_five_bins():
    """r = 12.5: a sphere's box (27 cells) touches five 8-cell bins per axis; flags bit-exact and the
    moving sphere's force and torque as in the oracle."""
    x = np.array([[20.3, 21.1, 19.6]])
    v = np.array([[0.02, -0.01, 0.015]])
    om = np.array([[0.0, 0.004, -0.003]])
    rR, rB = seeded_noise_fields(64, 64, 64, seed=8)
    g, o = make_pair(64, x, v, om, steps=6, fields=(rR, rB), radius=12.5, lrotate=1, wetting="neutral",
                     sigma=0.02, beta=0.7, rmass=1e-4)
    assert g.status()[0] == 0 and o.status()[0] == 0
    assert np.array_equal(g.get_flags(), o.get_flags())
    gp, op = g.get_particles(), o.get_particles()
    assert rel(gp["force"], op["force"]) < 1e-5
    assert rel(gp["torque"], op["torque"]) < 1e-5
