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
