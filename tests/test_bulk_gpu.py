"""The lean kernel's two ways of moving 16-bit pulls into shared memory give the same bits.

With bulk copies one warp per plane copies whole rows of every direction
plane (cp.async.bulk on the TMA engine, split at the periodic x edge); with
per-thread copies every thread issues its own 4-byte cp.async.  The densities
and the collision read the same values in the same order, so every population
must agree exactly: boxes whose x extent is a multiple of 32, not a multiple
of 32 (a partial column), smaller than the copy window (the window wraps on
both sides), a single row of columns in y (the ring rows wrap onto the
column), with and without spheres.
"""
import numpy as np
import pytest

from lbcuda_b200 import LBSim, make_params
from lbcuda_b200.inputs import seeded_noise_fields

pytestmark = pytest.mark.gpu


def pair(shape, storage, steps, particles=None, **kw):
    nx, ny, nz = shape
    out = []
    for bulk in (True, False):
        p = make_params(nx, ny, nz, model="cg", storage=storage, sigma=0.02, beta=0.7, **kw)
        s = LBSim(p)
        s.set_lean_copies(bulk)
        rR, rB = seeded_noise_fields(nx, ny, nz, seed=9)
        s.set_fields(rR, rB, (0.01, -0.02, 0.005))
        if particles is not None:
            s.set_particles(*particles)
        s.step(steps)
        assert s.status()[0] == 0
        out.append(s)
    return out


@pytest.mark.parametrize("storage", ["f16", "bf16", "f16sd", "bf16sd"])
@pytest.mark.parametrize("shape", [(32, 32, 32), (48, 24, 20), (16, 8, 12), (128, 8, 40), (64, 16, 24)])
def test_fluid_bulk_equals_per_thread(shape, storage):
    a, b = pair(shape, storage, 30)
    pa, pb = a.get_pops(), b.get_pops()
    assert np.array_equal(pa[0], pb[0]) and np.array_equal(pa[1], pb[1])


@pytest.mark.parametrize("storage", ["f16", "f16sd"])
def test_particles_bulk_equals_per_thread(storage):
    """Three moving, rotating spheres (fill / drain within 25 steps), neutral wetting."""
    x = np.array([[8.3, 9.1, 10.2], [22.6, 20.4, 24.9], [15.2, 27.7, 3.1]])
    v = np.array([[0.04, -0.03, 0.02], [-0.05, 0.01, 0.03], [0.02, 0.04, -0.05]])
    om = np.array([[0.0, 0.0, 0.01], [0.005, -0.004, 0.0], [0.0, 0.006, 0.003]])
    a, b = pair((32, 32, 32), storage, 25, particles=(x, v, om, None), max_particles=3, lrotate=1,
                wetting="neutral", max_vel=1.0)
    pa, pb = a.get_pops(), b.get_pops()
    assert np.array_equal(pa[0], pb[0]) and np.array_equal(pa[1], pb[1])
    qa, qb = a.get_particles(), b.get_particles()
    for k in ("x", "v", "force", "torque"):
        assert np.array_equal(qa[k], qb[k]), k
    assert np.array_equal(a.get_flags(), b.get_flags())
