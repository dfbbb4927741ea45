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


# D3Q19 directions 1..18 in the reference order (dimensions_m.CUF:211-218)
E19 = [(1, 0, 0), (-1, 0, 0), (0, 1, 0), (0, -1, 0), (0, 0, 1), (0, 0, -1), (1, 1, 0), (-1, -1, 0), (-1, 1, 0),
       (1, -1, 0), (1, 0, 1), (-1, 0, -1), (-1, 0, 1), (1, 0, -1), (0, 1, 1), (0, -1, -1), (0, -1, 1), (0, 1, -1)]


def independent_links(flags, owner_of):
    """The bounce-back link set restated from the flags with numpy: every
    surface cell and opposite pair (2i-1, 2i) with exactly one fluid end,
    as (sphere, cell, direction towards the fluid end)."""
    nz, ny, nx = flags.shape
    fluid = flags == 1
    rows = []
    zz, yy, xx = np.nonzero(flags == 2)
    for z, y, x in zip(zz, yy, xx):
        cell = x + nx * (y + ny * z)
        for it in range(9):
            lo, hi = 2 * it + 1, 2 * it + 2
            (ax, ay, az), (bx, by, bz) = E19[lo - 1], E19[hi - 1]
            fi = fluid[(z + az) % nz, (y + ay) % ny, (x + ax) % nx]
            fo = fluid[(z + bz) % nz, (y + by) % ny, (x + bx) % nx]
            if fi != fo:
                rows.append((owner_of(x, y, z), cell, hi if fo else lo))
    return np.array(sorted(rows), np.int64).reshape(-1, 3)


def test_oracle_links_match_independent_restatement():
    """Two spheres apart (one across the periodic edge): the links the oracle's
    node_to_particle_bounce_back_bc2 visits in a step are exactly the set
    restated from its flags."""
    n = 32
    x = np.array([[9.3, 10.6, 12.2], [24.7, 22.1, 1.4]])
    o = _sim(n, x, np.zeros((2, 3)), radius=5.5)
    o.record_links(True)
    assert o.step(1) == 0
    f = o.get_flags()

    def owner_of(cx, cy, cz):
        d = np.array([cx + 1, cy + 1, cz + 1], float) - x        # 1-based cell coordinates
        d -= n * np.round(d / n)
        return int(np.argmin((d * d).sum(axis=1)))

    ind = independent_links(f, owner_of)
    got = o.get_links().astype(np.int64)
    assert len(got) > 2 * 400
    assert np.array_equal(got, ind)
