"""The two ways the single-pass kernel stages 16-bit pulls give the same bits.

With 16-bit storage the lean colour-gradient kernel copies the pulls of a plane into shared memory two planes
ahead of their collision, either as 16-byte granules of one box of rows per direction (the default when nx is
a multiple of 4; copied by some threads, read by all, ordered by per-slot mbarriers) or as one 4-byte copy per
pull (each thread copies what it reads).  The arithmetic after the copy is the same, so every stored pair,
particle record and flag must agree bit for bit between the two, on boxes whose columns wrap in x, y and z, on
both CTA shapes, with and without spheres, and on every 16-bit storage.
"""
import numpy as np
import pytest

from lbcuda_b200 import LBSim, make_params
from lbcuda_b200.inputs import seeded_noise_fields

pytestmark = pytest.mark.gpu


def _fluid_run(shape, storage, copies, cta, zlen, steps):
    nx, ny, nz = shape
    rR, rB = seeded_noise_fields(nx, ny, nz, seed=21)
    g = LBSim(make_params(nx, ny, nz, model="cg", storage=storage, sigma=0.02, beta=0.7))
    g.set_lean_copies(copies)
    g.set_lean_shape(cta, zlen)
    g.set_fields(rR, rB)
    g.step(steps)
    out = g.get_pops(), g.get_fields(), g.status()[0]
    g.close()
    return out


@pytest.mark.parametrize("storage", ["f16", "bf16", "f16sd", "bf16sd", "f16sdp", "bf16sdp"])
@pytest.mark.parametrize("shape,cta,zlen", [((40, 24, 20), 0, 7), ((64, 16, 24), 1, 0), ((32, 32, 72), 0, 0),
                                            ((8, 12, 10), 0, 4)])
def test_fluid_copies_bit_identical(storage, shape, cta, zlen):
    (pa, fa, sa), (pb, fb, sb) = (_fluid_run(shape, storage, m, cta, zlen, 12) for m in (1, 0))
    assert sa == 0 and sb == 0
    for a, b in zip(pa, pb):
        assert np.array_equal(a, b)
    for a, b in zip(fa, fb):
        assert np.array_equal(a, b)


def test_width_not_multiple_of_four_runs_per_pull():
    """nx = 30: the box granules would straddle the periodic x edge, so both settings take the 4-byte copies."""
    (pa, _, sa), (pb, _, sb) = (_fluid_run((30, 16, 12), "f16sd", m, 0, 0, 8) for m in (1, 0))
    assert sa == 0 and sb == 0
    assert all(np.array_equal(a, b) for a, b in zip(pa, pb))


def _sphere_run(storage, copies, n=32):
    x = np.array([[1.6, 16.3, 30.4], [18.2, 2.7, 16.9], [12.1, 24.8, 6.2]]) * (n / 32)
    v = np.array([[0.04, -0.03, 0.02], [-0.05, 0.01, 0.03], [0.02, 0.04, -0.05]])
    om = np.array([[0.0, 0.0, 0.01], [0.005, -0.004, 0.0], [0.0, 0.006, 0.003]])
    rR, rB = seeded_noise_fields(n, n, n, seed=5)
    g = LBSim(make_params(n, model="cg", storage=storage, max_particles=3, max_vel=1.0, lrotate=1,
                          wetting="neutral", sigma=0.02, beta=0.7))
    g.set_lean_copies(copies)
    g.set_fields(rR, rB)
    g.set_particles(x, v, om, None)
    g.step(20)
    out = g.get_pops(), g.get_particles(), g.get_flags(), g.status()[0]
    g.close()
    return out


@pytest.mark.parametrize("storage,n", [("f16", 32), ("f16sd", 32), ("bf16sd", 32), ("f16sd", 48)])
def test_moving_spheres_copies_bit_identical(storage, n):
    """With spheres the flag bytes and the side phase field are staged as box granules too (nx a multiple of
    16); 48^3 puts a column across the periodic x edge."""
    (pa, ra, fa, sa), (pb, rb, fb, sb) = (_sphere_run(storage, m, n) for m in (1, 0))
    assert sa == 0 and sb == 0
    assert np.array_equal(fa, fb)
    for a, b in zip(pa, pb):
        assert np.array_equal(a, b)
    for k in ra:
        assert np.array_equal(ra[k], rb[k]), k
