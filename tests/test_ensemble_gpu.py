"""The ensemble of uneven boxes gives, box by box, exactly what the same box
advanced alone gives (the multi-box kernel runs the same per-cell arithmetic;
only the work decomposition differs)."""
import numpy as np
import pytest

from lbcuda_b200 import LBSim, make_params
from lbcuda_b200.ensemble import Ensemble, random_boxes
from lbcuda_b200.inputs import seeded_noise_fields

pytestmark = pytest.mark.gpu


def _params(L, n, storage="f32"):
    return make_params(L, model="cg", storage=storage, sigma=0.02, beta=0.7, max_particles=max(n, 0),
                       radius=4.0, wetting="neutral", lrotate=1, max_vel=1.0, exact_tiles=0,
                       hz_rmin=7.5, hz_rcap=6.0)


@pytest.mark.parametrize("storage", ["f32", "f16", "f16sd"])
def test_ensemble_equals_boxes_alone(storage):
    spec = random_boxes(6, seed=3, edges=(32, 48), max_spheres=6)
    params = [_params(L, len(x), storage) for L, x in spec]
    ens = Ensemble(params)
    alone = []
    for i, ((L, x), p) in enumerate(zip(spec, params)):
        rR, rB = seeded_noise_fields(L, L, L, seed=10 + i)
        v = np.full_like(x, 0.01)
        for sim in (ens.boxes[i], None):
            if sim is None:
                sim = LBSim(p)
                alone.append(sim)
            sim.set_fields(rR, rB)
            if len(x):
                sim.set_particles(x, v)
    ens.step(7)  # graph (two steps) three times and one eager step
    for s in alone:
        s.step(7)
    for i, s in enumerate(alone):
        a, b = ens.boxes[i].get_fields(), s.get_fields()
        for fa, fb in zip(a, b):
            assert np.array_equal(fa, fb), i
        if len(spec[i][1]):
            pa, pb = ens.boxes[i].get_particles(), s.get_particles()
            assert np.array_equal(pa["x"], pb["x"]), i
    ens.close()


def test_ensemble_tuner_keeps_results_consistent():
    spec = random_boxes(4, seed=5, edges=(32, 64), max_spheres=3)
    ens = Ensemble([_params(L, len(x)) for L, x in spec])
    for i, (L, x) in enumerate(spec):
        rR, rB = seeded_noise_fields(L, L, L, seed=i)
        ens.boxes[i].set_fields(rR, rB)
        if len(x):
            ens.boxes[i].set_particles(x, np.zeros_like(x))
    choice = ens.tune(trial=4)
    assert choice["shape"] in ("32x8", "32x16") and choice["zlen"] in (4, 8, 16, 32, 64, 128)
    ens.step(4)
    for b in ens.boxes:
        assert b.status()[0] == 0
        m, _ = b.get_sums()
        assert np.isfinite(m).all()
    ens.close()


def test_ensemble_after_a_box_stepped_alone():
    """A box stepped by itself (the single-box step clears its spheres' owners at the end of the step and
    records that on the host) and then with the ensemble (whose captured graph replays its sphere stages
    without that record) still equals the same box advanced alone throughout; the spheres move across cells,
    so stale owners would change the flags."""
    spec = random_boxes(4, seed=11, edges=(32, 48), max_spheres=5)
    params = [_params(L, len(x), "f16sd") for L, x in spec]
    ens = Ensemble(params)
    alone = []
    for i, ((L, x), p) in enumerate(zip(spec, params)):
        rR, rB = seeded_noise_fields(L, L, L, seed=30 + i)
        v = np.full_like(x, 0.1)
        for sim in (ens.boxes[i], None):
            if sim is None:
                sim = LBSim(p)
                alone.append(sim)
            sim.set_fields(rR, rB)
            if len(x):
                sim.set_particles(x, v)
    for b in ens.boxes:
        b.step(3)
    ens.step(9)
    for s in alone:
        s.step(12)
    for i, s in enumerate(alone):
        assert ens.boxes[i].status()[0] == 0 and s.status()[0] == 0
        assert np.array_equal(ens.boxes[i].get_flags(), s.get_flags()), i
        for fa, fb in zip(ens.boxes[i].get_fields(), s.get_fields()):
            assert np.array_equal(fa, fb), i
        if len(spec[i][1]):
            assert np.array_equal(ens.boxes[i].get_particles()["x"], s.get_particles()["x"]), i
    ens.close()
    for s in alone:
        s.close()
