"""CPU checks of the oracle and of the host-side input logic (no GPU).

PARITY UNPINNED: the reference ships no golden outputs and cannot be built
here (CUDA Fortran), so the oracle is checked against analytic invariants of
the method and against identities between its own code paths.
"""
import ctypes
import os

import numpy as np
import pytest

from lbcuda_b200 import make_params
from lbcuda_b200 import inputs
from oracle.orc import OracleSim

DECKS = os.path.join(os.path.dirname(__file__), "golden", "decks")


def test_equilibrium_is_fixed_point():
    p = make_params(12, model="cg", sigma=0.02, beta=0.7)
    o = OracleSim(p, "f64")
    r = np.full((12, 12, 12), 0.5, np.float32)
    o.set_fields(r, r, (0.03, 0.0, -0.02))
    o.step(5)
    rR, rB, vel, ph = o.get_fields()
    assert np.abs(rR - 0.5).max() < 1e-14
    assert np.abs(vel - np.float32([0.03, 0.0, -0.02]).astype(np.float64)).max() < 1e-14
    assert np.abs(ph).max() < 1e-14


@pytest.mark.parametrize("mode", ["ref", "f64"])
def test_mass_conserved_per_component(mode):
    p = make_params(16, 12, 10, model="cg", sigma=0.02, beta=0.7)
    rR, rB = inputs.seeded_noise_fields(16, 12, 10, seed=4)
    o = OracleSim(p, mode)
    o.set_fields(rR, rB)
    m0 = np.array([rR.astype(np.float64).sum(), rB.astype(np.float64).sum()])
    o.step(30)
    a, b, _, _ = o.get_fields()
    m1 = np.array([a.sum(), b.sum()])
    tol = 1e-6 if mode == "ref" else 1e-13
    assert (np.abs(m1 - m0) / m0 < tol).all()


def test_cg_without_blue_is_bgk():
    """CG with rhoB = 0 has phase 1, no gradient, omega = 1/tauR: the BGK step."""
    n = 12
    r = (1 + np.random.default_rng(0).uniform(-1e-3, 1e-3, (n, n, n))).astype(np.float32)
    ob = OracleSim(make_params(n, model="bgk", tau=0.9), "ref")
    ob.set_fields(r, None, (0.01, 0.02, 0.0))
    ob.step(10)
    oc = OracleSim(make_params(n, model="cg", tauR=0.9, tauB=0.9), "ref")
    oc.set_fields(r, np.zeros_like(r), (0.01, 0.02, 0.0))
    oc.step(10)
    assert np.array_equal(ob.get_pops()[0], oc.get_pops()[0])
    assert np.abs(oc.get_pops()[1]).max() == 0.0


def test_momentum_conserved_bgk():
    n = 10
    r = (1 + np.random.default_rng(1).uniform(-1e-3, 1e-3, (n, n, n))).astype(np.float32)
    o = OracleSim(make_params(n, model="bgk"), "f64")
    o.set_fields(r, None, (0.02, 0.0, 0.01))
    _, _, v0, _ = o.get_fields()
    rho0, _, _, _ = o.get_fields()
    mom0 = (rho0[..., None] * v0).sum(axis=(0, 1, 2))
    o.step(20)
    rho1, _, v1, _ = o.get_fields()
    mom1 = (rho1[..., None] * v1).sum(axis=(0, 1, 2))
    assert np.abs(mom1 - mom0).max() < 1e-11


def test_periodic_translation_invariance():
    """Shifting the initial fields by a lattice vector shifts the result."""
    n = 12
    p = make_params(n, model="cg", sigma=0.02, beta=0.7)
    rR, rB = inputs.seeded_noise_fields(n, n, n, seed=7)
    o1 = OracleSim(p, "ref")
    o1.set_fields(rR, rB)
    o1.step(8)
    o2 = OracleSim(p, "ref")
    sh = (3, -5, 2)
    o2.set_fields(np.roll(rR, sh, (0, 1, 2)), np.roll(rB, sh, (0, 1, 2)))
    o2.step(8)
    a = o1.get_fields()[3]
    b = o2.get_fields()[3]
    assert np.array_equal(np.roll(a, sh, (0, 1, 2)), b)


def test_leclaire_constants():
    """Sum of B_l equals c_s^2 and sum_l w_l (e.psi)^2 = c_s^2 |psi|^2 (mass of the perturbation)."""
    b0 = -(2 + 2 * 0.5) / (3 * 0.5 + 12)
    b1 = 0.5 / (6 * 0.5 + 24)
    b2 = 1 / (6 * 0.5 + 24)
    assert abs(b0 + 6 * b1 + 12 * b2 - 1 / 3) < 1e-15


def test_input_dat_reference_decks():
    ok = inputs.read_input_dat(os.path.join(DECKS, "01.input.dat"))
    assert ok["nIter"] == 2000 and ok["initType"] == 1 and ok["vel"] == (0.05, 0.05, 0.05)
    assert not ok["withParticles"]
    t3 = inputs.read_input_dat(os.path.join(DECKS, "CPC_Tab3.input_3a.dat"))
    assert t3["withParticles"] and t3["numAtoms"] == 23 and t3["lrotate"] and t3["max_vel"] == 0.3
    p7 = inputs.read_input_dat(os.path.join(DECKS, "07-1280-Particle.input.dat"))
    assert p7["numAtoms"] == 4 and p7["nIterVTK"] == 1 and p7["max_vel"] == 1.75
    for stale in ("02", "03", "04"):  # 8-line decks without the initType line
        with pytest.raises(inputs.InputError):
            inputs.read_input_dat(os.path.join(DECKS, f"{stale}.input.dat"))


def test_input_xyz_and_eul2q():
    x, v, q = inputs.read_input_xyz(os.path.join(DECKS, "05-1Particle.input.xyz"), 1, True)
    assert np.allclose(x[0], [26.5, 6.5, 6.5]) and np.allclose(q[0], [1, 0, 0, 0])
    x, v, q = inputs.read_input_xyz(os.path.join(DECKS, "07-1280.input.xyz.256cube.r5.5"), 1280, True)
    assert x.shape == (1280, 3)
    assert np.allclose((q ** 2).sum(axis=1), 1.0, atol=1e-6)
    inputs.check_particles(x, 256, 256, 256, 5.5)  # the placement satisfies d >= 2r+1
    with pytest.raises(inputs.InputError):
        inputs.read_input_xyz(os.path.join(DECKS, "05-1Particle.input.xyz"), 2, False)


def test_fortran_field_roundtrip(tmp_path):
    a = np.random.default_rng(0).random((5, 4, 3), dtype=np.float32)
    f = tmp_path / "rhoR.init.bin"
    inputs.write_fortran_field(str(f), a)
    b = inputs.read_fortran_field(str(f), 3, 4, 5)
    assert np.array_equal(a, b)
    with pytest.raises(inputs.InputError):
        inputs.read_fortran_field(str(f), 4, 4, 5)


def test_initial_fields_shapes():
    for t in (1, 2, 5, 6):
        rR, rB = inputs.initial_fields(t, 16, 16, 16, seed=1)
        assert rR.shape == (16, 16, 16) and rR.dtype == np.float32
        assert np.allclose(rR + rB, 1.0, atol=1e-6)
    rR, _ = inputs.initial_fields(1, 32, 32, 32)
    assert rR[16, 16, 16] == 1.0 and rR[0, 0, 0] == 0.0  # droplet radius glz/8 at the centre


def test_oracle_binding_is_independent_of_the_product():
    """The oracle's params mirror, defaults and noise fields equal the product's,
    so the CPU arm of the benchmark needs nothing from lbcuda_b200."""
    from lbcuda_b200 import capi, make_params
    from lbcuda_b200.inputs import seeded_noise_fields
    from oracle import orc
    assert [f[0] for f in orc.Params._fields_] == [f[0] for f in capi.LbxParams._fields_]
    assert ctypes.sizeof(orc.Params) == ctypes.sizeof(capi.LbxParams)
    a = orc.default_params(24, 16, 8, model="bgk", tau=0.8, wetting="neutral")
    b = make_params(24, 16, 8, model="bgk", tau=0.8, wetting="neutral")
    assert bytes(a) == bytes(b)
    for x, y in zip(orc.noise_fields(8, 6, 4, seed=3), seeded_noise_fields(8, 6, 4, seed=3)):
        assert np.array_equal(x, y)


def test_init_pops_roundtrip(tmp_path):
    """initType 4's per-direction files: six-digit names (write_fmtnumb) and a lossless round trip."""
    rng = np.random.default_rng(0)
    pR = rng.normal(size=(19, 4, 3, 5)).astype(np.float32)
    pB = rng.normal(size=(19, 4, 3, 5)).astype(np.float32)
    inputs.write_init_pops(str(tmp_path), pR, pB, pR.sum(0), pB.sum(0))
    assert (tmp_path / "popR.000000.init.bin").exists() and (tmp_path / "popB.000018.init.bin").exists()
    a, b = inputs.read_init_pops(str(tmp_path), 5, 3, 4)
    assert np.array_equal(a, pR) and np.array_equal(b, pB)
    rR, rB = inputs.initial_fields(4, 5, 3, 4, path=str(tmp_path))
    assert np.array_equal(rR, pR.sum(0))
