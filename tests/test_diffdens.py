"""Two fluid densities (the reference's DIFFDENS build, LBX_MODEL_CG_DIFFDENS).

CPU checks of the oracle restatement (kernels_fluid_CG.CUF:40-49, 163-177,
539-819; SetConstants main.CUF:1047-1083) and GPU parity of the two-pass
kernels against it.  Tolerances as for the single-density model: FP32
storage 1e-5 relative (max norm; velocity as relative L2), FP64 1e-12.
"""
import numpy as np
import pytest

from lbcuda_b200 import make_params
from lbcuda_b200.inputs import initial_fields, seeded_noise_fields
from oracle.orc import OracleSim


def rel(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.abs(a - b).max() / max(np.abs(b).max(), 1e-30))


def rel_l2(a, b):
    a = np.asarray(a, np.float64)
    b = np.asarray(b, np.float64)
    return float(np.linalg.norm(a - b) / max(np.linalg.norm(b), 1e-300))


def dd_params(n, densR, densB, storage="f32", **kw):
    return make_params(n, model="cg-diffdens", storage=storage, densR=densR, densB=densB, **kw)


@pytest.mark.parametrize("dens", [(1.0, 0.5), (2.0, 1.0)])
def test_uniform_mixture_at_rest_is_a_fixed_point(dens):
    """Uniform densities at rest: both density gradients vanish, so the
    equilibrium equilCG(rho_k, 0) set by set_fields is kept by the step."""
    n = 8
    p = dd_params(n, *dens)
    o = OracleSim(p, "f64")
    r = np.full((n, n, n), 0.6 * dens[0], np.float32)
    b = np.full((n, n, n), 0.4 * dens[1], np.float32)
    o.set_fields(r, b)
    p0 = o.get_pops()
    assert o.step(5) == 0
    p1 = o.get_pops()
    assert rel(p1[0], p0[0]) < 1e-13 and rel(p1[1], p0[1]) < 1e-13


def test_mass_conserved_and_fields_differ_from_single_density():
    """Each component's mass is conserved to rounding (the viscous correction
    sums to zero over the directions: Sum psi_l = -3 and Sum xi_l e_i^2 = 3/2)
    while no density is clamped at zero (a spinodal mixture; a pure phase
    with rho = 0 is clamped, as in init_rho*_CG, and then gains mass).  The
    droplet of the CPC_Tab2 deck (densR = 2, densB = 1) evolves differently
    from the single-density model."""
    n = 24
    rR, rB = seeded_noise_fields(n, n, n, seed=7)
    rR = (2.0 * rR).astype(np.float32)
    o = OracleSim(dd_params(n, 2.0, 1.0, sigma=0.05, beta=0.9), "f64")
    o.set_fields(rR, rB)
    m0 = o.get_pops()
    assert o.step(30) == 0
    m1 = o.get_pops()
    for c in (0, 1):
        assert abs(m1[c].sum() - m0[c].sum()) <= 1e-12 * m0[c].sum()
    rR, rB = initial_fields(1, n, n, n, dens=(2.0, 1.0))
    fields = []
    for p in (dd_params(n, 2.0, 1.0), make_params(n, model="cg", storage="f32")):
        s = OracleSim(p, "f64")
        s.set_fields(rR, rB, (0.01, 0.0, 0.02))
        s.step(30)
        fields.append(s.get_fields())
    assert rel(fields[0][2], fields[1][2]) > 1e-3


def test_initial_droplet_carries_the_densities():
    n = 16
    rR, rB = initial_fields(1, n, n, n, dens=(2.0, 1.0))
    r1, b1 = initial_fields(1, n, n, n)
    assert np.allclose(rR, 2.0 * r1) and np.allclose(rB, b1)


@pytest.mark.gpu
@pytest.mark.parametrize("dens,init", [((2.0, 1.0), "droplet"), ((1.0, 0.5), "noise")])
def test_diffdens_f32_matches_oracle(dens, init):
    from lbcuda_b200 import LBSim
    n = 32
    p = dd_params(n, *dens, sigma=0.05, beta=0.9)
    if init == "droplet":
        rR, rB = initial_fields(1, n, n, n, dens=dens)
        vel = (0.02, -0.01, 0.01)
    else:
        rR, rB = seeded_noise_fields(n, n, n, seed=4)
        rR = (rR * dens[0]).astype(np.float32)
        rB = (rB * dens[1]).astype(np.float32)
        vel = (0.0, 0.0, 0.0)
    g = LBSim(p)
    g.set_fields(rR, rB, vel)
    g.step(30)
    o = OracleSim(p, "ref")
    o.set_fields(rR, rB, vel)
    assert o.step(30) == 0
    gf, of = g.get_fields(), o.get_fields()
    for name, a, b in zip(("rhoR", "rhoB", "vel", "phase"), gf, of):
        e = rel_l2(a, b) if name == "vel" else rel(a, b)
        assert e <= (5e-5 if (name == "vel" and init == "noise") else 1e-5), (name, e)
    assert g.status()[0] == 0


@pytest.mark.gpu
def test_diffdens_f64_matches_oracle_f64():
    from lbcuda_b200 import LBSim
    n = 24
    p = dd_params(n, 1.0, 0.5, storage="f64", sigma=0.05, beta=0.9)
    rR, rB = initial_fields(1, n, n, n, dens=(1.0, 0.5))
    g = LBSim(p)
    g.set_fields(rR, rB, (0.01, 0.02, 0.0))
    g.step(20)
    o = OracleSim(p, "f64")
    o.set_fields(rR, rB, (0.01, 0.02, 0.0))
    o.step(20)
    for a, b in zip(g.get_fields(f64=True), o.get_fields()):
        assert rel(a, b) <= 1e-12


@pytest.mark.gpu
def test_diffdens_sphere_matches_oracle():
    """A moving sphere in a two-density fluid (particle two-pass schedule)."""
    from lbcuda_b200 import LBSim
    n = 32
    p = dd_params(n, 2.0, 1.0, max_particles=1, max_vel=1.0, wetting="neutral", lrotate=1)
    rR, rB = initial_fields(1, n, n, n, dens=(2.0, 1.0))
    x = np.array([[11.6, 16.3, 15.2]])
    v = np.array([[0.02, 0.01, -0.015]])
    g = LBSim(p)
    o = OracleSim(p, "f32p64")
    for s in (g, o):
        s.set_fields(rR, rB)
        s.set_particles(x, v)
    g.step(12)
    assert o.step(12) == 0
    assert np.array_equal(g.get_flags(), o.get_flags())
    assert rel(g.get_particles()["force"], o.get_particles()["force"]) <= 1e-5
    gf, of = g.get_fields(), o.get_fields()
    for a, b in zip(gf, of):
        assert rel_l2(a, b) <= 1e-5


@pytest.mark.gpu
def test_diffdens_arguments():
    from lbcuda_b200 import LBSim, LBXError
    with pytest.raises(LBXError):
        LBSim(dd_params(16, 2.0, 2.0))  # at least one density must be 1 (main.CUF:1059-1062)
    with pytest.raises(LBXError):
        LBSim(dd_params(16, 1.0, 0.0))
    g = LBSim(dd_params(16, 1.0, 0.5))
    with pytest.raises(LBXError):
        g.set_schedule(2)  # the two-density collision runs on the two-pass schedule
    g.set_schedule(0)
    g.close()


def test_namelist_deck_gives_the_densities(tmp_path):
    """The namelist deck (NEWINPUT build) is where densR / densB come from."""
    from lbcuda_b200.inputs import InputError, read_namelist_input
    deck = tmp_path / "deck.dat"
    deck.write_text("&simulation\nnIter=200   ! steps\nnIterOut=20\nnIterVTK=100\ninitType=1\n&end\n"
                    "&fluid\nDENSR=2.0\ndensB=1.0\nvx=0.0, vy=0.01, vz=0.0\ntauR=1.0\ntauB=1.0\n&end\n"
                    "&particle\nwithParticles=.false.\nnumAtoms=1\nlrotate=.false.\nmax_vel=1.0\n/\n")
    d = read_namelist_input(deck)
    assert d["densR"] == 2.0 and d["densB"] == 1.0 and d["vy"] == 0.01 and d["initType"] == 1
    assert d["withParticles"] is False and d["nIter"] == 200
    p = dd_params(16, d["densR"], d["densB"], tauR=d["tauR"], tauB=d["tauB"])
    assert p.densR == 2.0 and p.model == 2
    bad = tmp_path / "bad.dat"
    bad.write_text("&simulation\nnIter=1\nbogus=3\n&end\n&fluid\n&end\n&particle\n&end\n")
    with pytest.raises(InputError):
        read_namelist_input(bad)


def test_reference_namelist_deck():
    """The reference's own namelist deck (Tests/CPC_Tab2_128/newinput.dat):
    a droplet (initType 1) of density 2 in a fluid of density 1."""
    import os
    from lbcuda_b200.inputs import read_namelist_input
    deck = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden", "decks", "CPC_Tab2_128.newinput.dat")
    d = read_namelist_input(deck)
    assert (d["densR"], d["densB"]) == (2.0, 1.0)
    assert d["initType"] == 1 and d["withParticles"] is False
    assert (d["nIter"], d["nIterOut"]) == (5000, 500)
    assert (d["tauR"], d["tauB"]) == (1.0, 1.0)
