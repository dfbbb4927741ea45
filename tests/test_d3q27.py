"""The D3Q27 lattice (the reference's D3Q27 build, dimensions_m.CUF:117-198).

CPU checks of the oracle restatement on 27 directions, and (gpu) parity of
the two-pass kernels against it: FP32 storage 1e-5 relative (velocity as
relative L2), FP64 1e-12.
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


def test_equilibrium_moments_and_fixed_point():
    """set_fields builds the D3Q27 equilibrium: its moments give back rho and
    u (sum p_l = 1, sum p_l e_l e_l = cs^2 I), and a uniform flow stays."""
    n = 8
    p = make_params(n, model="cg-d3q27", storage="f32")
    o = OracleSim(p, "f64")
    r = np.full((n, n, n), 0.7, np.float32)
    b = np.full((n, n, n), 0.3, np.float32)
    vel = (0.05, -0.02, 0.03)
    o.set_fields(r, b, vel)
    pops = o.get_pops()
    assert pops[0].shape[0] == 27
    rR, rB, u, ph = o.get_fields()
    assert np.abs(rR - 0.7).max() < 1e-6 and np.abs(rB - 0.3).max() < 1e-6
    assert np.abs(u - np.array(vel)).max() < 1e-6
    assert o.step(5) == 0
    rR, rB, u, ph = o.get_fields()
    assert np.abs(u - np.array(vel)).max() < 1e-6 and np.abs(rR - 0.7).max() < 1e-6


@pytest.mark.parametrize("model", ["cg-d3q27", "cg-diffdens-d3q27"])
def test_mass_and_momentum_conserved(model):
    n = 16
    p = make_params(n, model=model, storage="f32", sigma=0.05, beta=0.9, densR=1.0, densB=0.5)
    o = OracleSim(p, "f64")
    rR, rB = seeded_noise_fields(n, n, n, seed=3)
    o.set_fields(rR, rB, (0.01, 0.0, -0.02))
    p0 = o.get_pops()
    assert o.step(20) == 0
    p1 = o.get_pops()
    for c in (0, 1):
        assert abs(p1[c].sum() - p0[c].sum()) <= 1e-12 * p0[c].sum()
    ex = np.array([0, 1, -1, 0, 0, 0, 0, 1, -1, -1, 1, 1, -1, -1, 1, 0, 0, 0, 0, 1, -1, 1, -1, -1, 1, 1, -1])
    m0 = sum((ex[:, None, None, None] * p0[c]).sum() for c in (0, 1))
    m1 = sum((ex[:, None, None, None] * p1[c]).sum() for c in (0, 1))
    assert abs(m1 - m0) <= 1e-12 * abs(p0[0]).sum()


def test_d3q27_differs_from_d3q19():
    n = 16
    rR, rB = initial_fields(1, n, n, n)
    out = []
    for model in ("cg-d3q27", "cg"):
        o = OracleSim(make_params(n, model=model, storage="f32"), "f64")
        o.set_fields(rR, rB, (0.02, 0.01, 0.0))
        o.step(10)
        out.append(o.get_fields())
    assert rel(out[0][2], out[1][2]) > 1e-3


@pytest.mark.gpu
@pytest.mark.parametrize("model,init", [("cg-d3q27", "droplet"), ("cg-d3q27", "noise"),
                                        ("cg-diffdens-d3q27", "droplet")])
def test_d3q27_f32_matches_oracle(model, init):
    from lbcuda_b200 import LBSim
    n = 32
    dens = (2.0, 1.0) if "diffdens" in model else (1.0, 1.0)
    p = make_params(n, model=model, storage="f32", sigma=0.05, beta=0.9, densR=dens[0], densB=dens[1])
    if init == "droplet":
        rR, rB = initial_fields(1, n, n, n, dens=dens)
        vel = (0.02, -0.01, 0.01)
    else:
        rR, rB = seeded_noise_fields(n, n, n, seed=6)
        vel = (0.0, 0.0, 0.0)
    g = LBSim(p)
    g.set_fields(rR, rB, vel)
    g.step(30)
    o = OracleSim(p, "ref")
    o.set_fields(rR, rB, vel)
    assert o.step(30) == 0
    for name, a, b in zip(("rhoR", "rhoB", "vel", "phase"), g.get_fields(), o.get_fields()):
        e = rel_l2(a, b) if name == "vel" else rel(a, b)
        assert e <= (5e-5 if (name == "vel" and init == "noise") else 1e-5), (name, e)
    pg, po = g.get_pops(), o.get_pops()
    assert pg[0].shape[0] == 27
    assert rel(pg[0], po[0]) <= 1e-5 and rel(pg[1], po[1]) <= 1e-5
    assert g.status()[0] == 0


@pytest.mark.gpu
@pytest.mark.parametrize("storage,tol", [("f64", 1e-12), ("f16", 1e-2)])
def test_d3q27_other_storage(storage, tol):
    """FP64 storage against the FP64 oracle (1e-12); FP16 shifted storage
    against the FP64 oracle within its rounding (1e-2 on the phase field
    after 20 steps of a droplet)."""
    from lbcuda_b200 import LBSim
    n = 24
    p = make_params(n, model="cg-d3q27", storage=storage, sigma=0.05, beta=0.9)
    rR, rB = initial_fields(1, n, n, n)
    g = LBSim(p)
    g.set_fields(rR, rB, (0.01, 0.02, 0.0))
    g.step(20)
    o = OracleSim(p, "f64")
    o.set_fields(rR, rB, (0.01, 0.02, 0.0))
    o.step(20)
    gf, of = g.get_fields(f64=True), o.get_fields()
    if storage == "f64":
        for a, b in zip(gf, of):
            assert rel(a, b) <= tol
    else:
        assert rel_l2(gf[3], of[3]) <= tol


@pytest.mark.gpu
def test_d3q27_rejects_spheres_and_single_pass():
    from lbcuda_b200 import LBSim, LBXError
    with pytest.raises(LBXError):
        LBSim(make_params(32, model="cg-d3q27", storage="f32", max_particles=1))
    g = LBSim(make_params(16, model="cg-d3q27", storage="f32"))
    with pytest.raises(LBXError):
        g.set_schedule(2)
    g.close()


@pytest.mark.gpu
@pytest.mark.parametrize("storage,bound", [("f32", 2.5e-6), ("f64", 1e-12)])
def test_d3q27_mass(storage, bound):
    """FP64 sums of each component's mass over 20 steps.  The FP32 weights
    of the D3Q27 build sum to 1 + 1.08e-7 (the D3Q19 ones to 1 + 1.5e-8), so
    each BGK step at omega = 1 adds about 1.1e-7 of the mass in FP32, as the
    reference's FP32 tables do; FP64 storage and tables conserve it."""
    from lbcuda_b200 import LBSim
    g = LBSim(make_params(16, model="cg-d3q27", storage=storage))
    rR, rB = seeded_noise_fields(16, 16, 16, seed=1)
    g.set_fields(rR, rB)
    g.step(1)
    m0, _ = g.get_sums()
    g.step(20)
    m1, _ = g.get_sums()
    assert (np.abs(m1 - m0) / m0 <= bound).all(), np.abs(m1 - m0) / m0
    g.close()


@pytest.mark.gpu
def test_d3q27_noncubic_unequal_tau_matches_oracle():
    """A non-cubic box (48 x 20 x 16) with tauR != tauB and two densities."""
    from lbcuda_b200 import LBSim
    nx, ny, nz = 48, 20, 16
    p = make_params(nx, ny, nz, model="cg-diffdens-d3q27", storage="f32", tauR=0.8, tauB=1.3, sigma=0.05,
                    beta=0.9, densR=1.0, densB=0.5)
    rR, rB = seeded_noise_fields(nx, ny, nz, seed=12)
    rB = (0.5 * rB).astype(np.float32)
    g = LBSim(p)
    g.set_fields(rR, rB, (0.01, -0.02, 0.0))
    g.step(25)
    o = OracleSim(p, "ref")
    o.set_fields(rR, rB, (0.01, -0.02, 0.0))
    assert o.step(25) == 0
    for name, a, b in zip(("rhoR", "rhoB", "vel", "phase"), g.get_fields(), o.get_fields()):
        e = rel_l2(a, b) if name == "vel" else rel(a, b)
        assert e <= (5e-5 if name == "vel" else 1e-5), (name, e)


@pytest.mark.gpu
def test_d3q27_set_pops_roundtrip_bf16_shift():
    """27-plane population transfer both ways; BF16 storage keeps the D3Q27
    corner class's shift (w_3 rho0) in the round trip of an equilibrium."""
    from lbcuda_b200 import LBSim
    n = 12
    g = LBSim(make_params(n, model="cg-d3q27", storage="f32"))
    rng = np.random.default_rng(3)
    pR = rng.uniform(0.0, 0.1, (27, n, n, n)).astype(np.float32)
    pB = rng.uniform(0.0, 0.1, (27, n, n, n)).astype(np.float32)
    g.set_pops(pR, pB)
    a, b = g.get_pops()
    assert np.array_equal(a, pR) and np.array_equal(b, pB)
    g.close()
    g = LBSim(make_params(n, model="cg-d3q27", storage="bf16"))
    r = np.full((n, n, n), 0.5, np.float32)
    g.set_fields(r, r)
    a, b = g.get_pops()
    w = np.array([8 / 27] + [2 / 27] * 6 + [1 / 54] * 12 + [1 / 216] * 8)
    assert np.abs(a[:, 0, 0, 0] - 0.5 * w).max() < 1e-7
    g.close()
