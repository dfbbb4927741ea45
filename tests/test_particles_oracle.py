"""CPU checks of the oracle's particle restatement (no GPU)."""
import numpy as np

from lbcuda_b200 import make_params
from oracle.orc import OracleSim


def _sim(n, x, v, **kw):
    kw.setdefault("max_vel", 1.0)
    p = make_params(n, model="cg", max_particles=len(x), **kw)
    o = OracleSim(p, "f32p64")
    r = np.full((n, n, n), 0.5, np.float32)
    o.set_fields(r, r)
    o.set_particles(np.asarray(x, float), np.asarray(v, float))
    return o


def independent_template(rdim):
    """spherical_template restated with numpy (main.CUF:1990-2130)."""
    rmax = int(rdim + 1)
    rmin = int(np.floor(rdim))
    k, j, i = np.meshgrid(*(np.arange(-rmax, rmax + 1),) * 3, indexing="ij")
    t = np.where(i * i + j * j + k * k <= rdim * rdim, 4, 1).astype(np.int8)
    e = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1), (1, 1, 0), (-1, -1, 0), (-1, 1, 0),
         (1, -1, 0), (1, 0, 1), (-1, 0, -1), (-1, 0, 1), (1, 0, -1), (0, 1, 1), (0, -1, -1), (0, -1, 1), (0, 1, -1)]
    out = t.copy()
    c = rmax
    for kk in range(-rmin, rmin + 1):
        for jj in range(-rmin, rmin + 1):
            for ii in range(-rmin, rmin + 1):
                if t[kk + c, jj + c, ii + c] != 4:
                    continue
                if any(t[kk + ez + c, jj + ey + c, ii + ex + c] == 1 for ex, ey, ez in e):
                    out[kk + c, jj + c, ii + c] = 2
    out[c, c, c] = 5
    return out


def test_template_matches_independent_restatement():
    for r in (5.5, 3.0, 4.0, 12.0):
        n = 32 if r < 10 else 32
        o = _sim(n, [[16.0, 16.0, 16.0]], [[0, 0, 0]], radius=r)
        assert np.array_equal(o.template(), independent_template(r)), r


def test_sphere_at_rest_in_quiescent_fluid_stays():
    """Neutral wetting: no colour gradient, no force (a Janus sphere would be pushed along its axis)."""
    o = _sim(32, [[16.2, 15.8, 16.4]], [[0, 0, 0]], wetting="neutral")
    o.step(10)
    d = o.get_particles()
    assert np.abs(d["v"]).max() < 1e-6
    assert np.abs(d["x"] - [16.2, 15.8, 16.4]).max() < 1e-5


def test_moving_sphere_is_decelerated_and_drags_fluid():
    o = _sim(32, [[12.2, 16.1, 16.3]], [[0.02, 0, 0]], wetting="neutral")
    v = []
    for _ in range(40):
        o.step(1)
        v.append(o.get_particles()["v"][0, 0])
    assert v[0] < 0.02 and all(b <= a + 1e-12 for a, b in zip(v, v[1:]))
    _, _, vel, _ = o.get_fields()
    assert vel[..., 0].sum() > 0  # momentum handed to the fluid


def test_fill_and_drain_keep_flags_consistent():
    """After crossing several cells the flags are those of the template at nint(x)."""
    o = _sim(32, [[10.4, 16.0, 16.0]], [[0.08, 0, 0]], wetting="neutral")
    o.step(30)
    x = o.get_particles()["x"][0]
    o2 = _sim(32, [x], [[0, 0, 0]], wetting="neutral")
    assert np.array_equal(o.get_flags(), o2.get_flags())


def test_kinematic_sphere_moves_with_set_velocity():
    """Prescribed motion: the centre advances by v each step, v is kept, the drag is recorded."""
    o = _sim(32, [[12.2, 16.1, 16.3]], [[0.02, 0.01, 0]], wetting="neutral", kinematic=1)
    o.step(25)
    d = o.get_particles()
    assert np.abs(d["x"][0] - [12.7, 16.35, 16.3]).max() < 1e-9
    assert np.array_equal(d["v"][0], [0.02, 0.01, 0.0])
    assert d["force"][0, 0] < 0 and d["force"][0, 1] < 0


def test_frozen_geometry_sphere_keeps_its_centre():
    """kinematic = 2: the centre stays while the wall moves with the set velocity (drag recorded)."""
    o = _sim(32, [[12.2, 16.1, 16.3]], [[0.02, 0.0, 0.0]], wetting="neutral", kinematic=2)
    o.step(20)
    d = o.get_particles()
    assert np.array_equal(d["x"][0], [12.2, 16.1, 16.3])
    assert np.array_equal(d["v"][0], [0.02, 0.0, 0.0])
    assert d["force"][0, 0] < 0
