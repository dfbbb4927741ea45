"""Learned pair closure: the network kernels against the numpy reference, its
use inside the particle step, and a small end-to-end gain check.

The closure has no counterpart in the reference; the numpy reference
(oracle/mlp_ref.py) is itself checked against finite differences.
Tolerances: GPU gradient vs numpy 1e-4 relative (FP32 vs FP64), inference
1e-5 relative to the output scale.
"""
import numpy as np
import pytest

from oracle import mlp_ref as M

RNG = np.random.default_rng(0)


def random_blob(seed=0, scale=0.3):
    rng = np.random.default_rng(seed)
    w = np.zeros(M.TOTAL, np.float32)
    w[:M.NPARAM] = rng.normal(0, scale, M.NPARAM)
    w[M.OFF["xmu"][0]:M.OFF["xmu"][0] + M.DIN] = rng.normal(0, 0.1, M.DIN)
    w[M.OFF["xsd"][0]:M.OFF["xsd"][0] + M.DIN] = rng.uniform(0.5, 2.0, M.DIN)
    w[M.OFF["ymu"][0]:M.OFF["ymu"][0] + 12] = rng.normal(0, 0.1, 12)
    w[M.OFF["ysd"][0]:M.OFF["ysd"][0] + 12] = rng.uniform(0.5, 2.0, 12)
    return w


def test_numpy_reference_gradient_matches_finite_differences():
    w = random_blob(1).astype(np.float64)
    X = RNG.normal(size=(24, M.DIN))
    T = RNG.normal(size=(24, 12))
    g = M.grad_std(w, X, T)
    for idx in (0, 7, 700, 790, 3000, 5000, 9000, M.NPARAM - 1):
        e = 1e-6
        wp, wm = w.copy(), w.copy()
        wp[idx] += e
        wm[idx] -= e
        fd = (M.loss_std(wp, X, T) - M.loss_std(wm, X, T)) / (2 * e)
        assert abs(fd - g[idx]) <= 1e-6 + 1e-5 * abs(fd)


def test_blob_layout_matches_the_header():
    import re
    from pathlib import Path
    from lbcuda_b200 import closure
    h = (Path(__file__).resolve().parents[1] / "include" / "lbx.h").read_text()
    nw = int(re.search(r"#define LBX_CLOSURE_NWEIGHTS (\d+)", h).group(1))
    assert nw == closure.NW == M.TOTAL and closure.NPARAM == M.NPARAM and closure.DIN == M.DIN


def test_pair_frame_and_features():
    from lbcuda_b200.closure import features, pair_frame
    for n in RNG.normal(size=(20, 3)):
        n /= np.linalg.norm(n)
        t1, t2 = pair_frame(n)
        F = np.stack([n, t1, t2])
        assert np.allclose(F @ F.T, np.eye(3), atol=1e-12)
    x, _ = features([10, 10, 10], [17.5, 10, 10], [0, 0, 0], [-1e-3, 0, 0], [0, 0, 0], [0, 0, 0], 3.0, (32,) * 3)
    # the gap of the rounded centres (the templates sit at 10 and NINT(17.5) = 18)
    assert abs(x[0] - 2.0 / 3.0) < 1e-12 and abs(x[1] + 1e-3) < 1e-15 and x[10] == 3.0
    assert x[11] == 0.0 and x[12] == 0.0          # on an axis: nc = (1, 0, 0)
    # periodic image: the pair across the boundary (NINT(31.5) = 32, one cell from 1)
    x, _ = features([1, 10, 10], [31.5, 10, 10], [0, 0, 0], [0, 0, 0], [0, 0, 0], [0, 0, 0], 3.0, (32,) * 3)
    assert abs(x[0] - (1.0 - 6) / 3) < 1e-12


def _signed_permutations():
    import itertools
    for perm in itertools.permutations(range(3)):
        for signs in itertools.product((1.0, -1.0), repeat=3):
            Q = np.zeros((3, 3))
            for r, k in enumerate(perm):
                Q[r, k] = signs[r]
            yield Q


def test_lattice_frame_is_fixed_by_the_cubic_group():
    """All 48 lattice images of a pair give the same inputs; outputs map back covariantly.

    Velocities map as Q v, angular velocities as det(Q) Q w (pseudovectors).
    Where |d| has equal or zero components some images are mirror images
    with the same separation (the class's own symmetry): those share the
    frame, give the same geometric inputs and mirrored velocity inputs, and
    the class's resistance carries that symmetry itself.
    """
    from lbcuda_b200.closure import features, lattice_frame
    rng = np.random.default_rng(4)
    ds = [np.array(d, float) for d in ((5, 3, 1), (4, 4, 2), (6, 0, 0), (5, 5, 5), (-3, 6, 2), (0, -7, 3),
                                       (2, -5, -7))]
    for d in ds:
        E, sign, nc = lattice_frame(d / np.linalg.norm(d))
        assert np.allclose(E @ E.T, np.eye(3), atol=1e-12)
        assert np.allclose(E[0], d / np.linalg.norm(d)) and abs(np.linalg.det(E) - sign) < 1e-12
        assert np.all(np.diff(nc) <= 0) and np.all(nc >= 0)
        xi = np.array([16.0, 16.0, 16.0])
        v = rng.uniform(-1e-3, 1e-3, (2, 3))
        om = rng.uniform(-1e-3, 1e-3, (2, 3))
        x0, (E0, s0) = features(xi, xi + d, v[0], v[1], om[0], om[1], 3.0, (64,) * 3)
        y = rng.normal(size=12)                        # any pair-frame output
        F0 = E0.T @ y[:3]
        T0 = s0 * (E0.T @ y[3:6])
        for Q in _signed_permutations():
            dq = np.linalg.det(Q)
            x, (Eq, sq) = features(xi, xi + Q @ d, Q @ v[0], Q @ v[1], dq * (Q @ om[0]), dq * (Q @ om[1]), 3.0,
                                   (64,) * 3)
            assert np.allclose(x[[0, 10, 11, 12]], x0[[0, 10, 11, 12]], rtol=0, atol=1e-15)
            a = np.abs(d)
            if len({a[0], a[1], a[2]}) == 3 and a.min() > 0:
                assert np.allclose(x, x0, rtol=0, atol=1e-15), (d, Q)
                assert np.allclose(Eq.T @ y[:3], Q @ F0, atol=1e-12)
                assert np.allclose(sq * (Eq.T @ y[3:6]), dq * (Q @ T0), atol=1e-12)


def test_lattice_classes_cover_the_envelope():
    from lbcuda_b200.closure import lattice_classes, nint
    cls = set(lattice_classes(3, (0.05, 1.5)))
    assert len(cls) == 121
    rng = np.random.default_rng(0)
    for _ in range(2000):
        d = nint(rng.normal(size=3) / 1.0 * 3)
        g = np.linalg.norm(d) / 3 - 2
        key = tuple(sorted(np.abs(d).astype(int), reverse=True))
        assert (key in cls) == (0.05 <= g <= 1.5)


def test_analytic_lubrication_is_repulsive_on_approach():
    from lbcuda_b200.closure import analytic_lubrication
    X = np.zeros((2, M.DIN))
    X[:, 0] = 0.1  # gap / R
    X[0, 1] = -1e-3  # approaching
    X[1, 1] = +1e-3  # separating
    F = analytic_lubrication(X, 3.0)
    assert F[0, 0] < 0 < F[0, 6]   # pushed apart
    assert F[1, 0] > 0 > F[1, 6]   # pulled together


@pytest.mark.gpu
def test_gpu_gradient_matches_numpy():
    from lbcuda_b200 import closure
    w = random_blob(2)
    Xs = RNG.normal(size=(64, M.DIN)).astype(np.float32)
    Ts = RNG.normal(size=(64, 12)).astype(np.float32)
    g_gpu = closure.grad(w, Xs, Ts)
    g_ref = M.grad_std(w.astype(np.float64), Xs, Ts)
    err = np.abs(g_gpu - g_ref).max() / np.abs(g_ref).max()
    assert err < 1e-4, err


@pytest.mark.gpu
def test_gpu_inference_matches_numpy():
    from lbcuda_b200 import closure
    w = random_blob(3)
    X = RNG.normal(size=(1000, M.DIN)).astype(np.float32)
    y = closure.infer(w, X)
    y_ref = M.infer(w.astype(np.float64), X)
    assert np.abs(y - y_ref).max() / np.abs(y_ref).max() < 1e-5


@pytest.mark.gpu
def test_gpu_training_fits_a_smooth_map():
    from lbcuda_b200 import closure
    X = RNG.uniform(-1, 1, size=(2048, M.DIN)).astype(np.float32)
    A = RNG.normal(size=(M.DIN, 12)) / 3
    T = (np.tanh(X @ A) + 0.1 * np.sin(3 * X[:, :1])).astype(np.float32)
    w, loss = closure.train(X[:1536], T[:1536], epochs=300, lr=3e-3)
    assert loss[-1] < 0.05 * loss[0]
    err = ((closure.infer(w, X[1536:]) - T[1536:]) ** 2).mean() / (T[1536:] ** 2).mean()
    assert err < 0.02, err


def _pair_sims(closure_on, lubrication, with_zero_net):
    from lbcuda_b200 import LBSim, make_params
    from oracle.orc import OracleSim
    n = 32
    kw = dict(max_particles=2, radius=4.0, max_vel=1.0, lrotate=1, wetting="neutral", hz_rmin=7.5, hz_rcap=6.0,
              lubrication=lubrication, lubric_k=1.0 / 6.0, lubric_rmin=1.0, lubric_rcap=0.2, closure=closure_on)
    p = make_params(n, model="cg", storage="f32", **kw)
    r = np.ones((n, n, n), np.float32)
    x = np.array([[11.3, 16.2, 15.8], [19.9, 16.6, 16.1]])
    v = np.array([[0.01, 0.0, 0.0], [-0.01, 0.002, 0.0]])
    g = LBSim(p)
    g.set_fields(r, np.zeros_like(r))
    g.set_particles(x, v)
    if with_zero_net:
        w = np.zeros(M.TOTAL, np.float32)
        w[M.OFF["xsd"][0]:M.OFF["xsd"][0] + M.DIN] = 1
        w[M.OFF["ysd"][0]:M.OFF["ysd"][0] + 12] = 1
        from lbcuda_b200 import capi
        import ctypes
        capi.check(capi.lib().lbx_closure_set(g._h, w.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
    o = OracleSim(p, "f32p64")
    o.set_fields(r, np.zeros_like(r))
    o.set_particles(x, v)
    return g, o


@pytest.mark.gpu
@pytest.mark.parametrize("closure_on", [0, 1])
def test_step_with_analytic_lubrication_matches_oracle(closure_on):
    """Closure off with lubrication, or closure on without weights (every pair falls back)."""
    g, o = _pair_sims(closure_on, 1, False)
    g.step(12)
    o.step(12)
    a, b = g.get_particles(), o.get_particles()
    assert np.abs(a["x"] - b["x"]).max() < 1e-6
    assert np.abs(a["force"] - b["force"]).max() <= 1e-5 * np.abs(b["force"]).max()


@pytest.mark.gpu
def test_zero_network_changes_nothing():
    g, o = _pair_sims(1, 0, True)
    g.step(12)
    o.step(12)
    a, b = g.get_particles(), o.get_particles()
    assert np.abs(a["x"] - b["x"]).max() < 1e-6
    assert np.abs(a["force"] - b["force"]).max() <= 1e-5 * np.abs(b["force"]).max()


@pytest.mark.gpu
def test_step_applies_the_network_in_the_lattice_frame():
    """The correction the particle step adds equals host features -> inference -> E^T (torques det P).

    Frozen geometry (kinematic = 2), so the fluid is the same with and without
    the network and the force difference is the correction itself; pairs in
    orientations that need every kind of class map (permutation, reflections).
    """
    import ctypes
    from lbcuda_b200 import LBSim, capi, closure, make_params
    rng = np.random.default_rng(9)
    w = random_blob(6)
    w[M.OFF["xmu"][0]:M.OFF["xmu"][0] + M.DIN] = 0.0
    w[M.OFF["xsd"][0]:M.OFF["xsd"][0] + M.DIN] = [0.5] + [1e-3] * 9 + [1.0, 0.3, 0.3]
    w[M.OFF["ymu"][0]:M.OFF["ymu"][0] + 12] = 0.0
    w[M.OFF["ysd"][0]:M.OFF["ysd"][0] + 12] = 1e-3
    n = 32
    kw = dict(max_particles=2, radius=3.0, max_vel=1.0, lrotate=1, wetting="neutral", kinematic=2,
              hz_rmin=5.5, hz_rcap=4.0, exact_tiles=0)
    on = LBSim(make_params(n, model="cg", storage="f32", closure=1, **kw))
    off = LBSim(make_params(n, model="cg", storage="f32", closure=0, **kw))
    capi.check(capi.lib().lbx_closure_set(on._h, w.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
    one = np.ones((n, n, n), np.float32)
    for d in ((5, 3, 2), (-3, 6, 2), (2, -5, -6), (-4, -4, 3), (0, 7, -1), (-6, -1, 3)):
        d = np.array(d, float)
        xi = np.array([14.0, 15.0, 16.0])
        x = np.stack([xi, xi + d])
        v = rng.uniform(-2.5e-4, 2.5e-4, (2, 3))     # inside the envelope: |pair-frame dv| <= 1e-3
        om = rng.uniform(-5e-4, 5e-4, (2, 3))
        res = []
        for sim in (on, off):
            sim.set_fields(one, np.zeros_like(one))
            sim.set_particles(x, v, om, None)
            sim.step(3)
            res.append(sim.get_particles())
        feat, (E, sign) = closure.features(x[0], x[1], v[0], v[1], om[0], om[1], 3.0, (n,) * 3)
        assert 0.05 <= feat[0] <= 1.5 and np.abs(feat[1:10]).max() <= 1e-3
        y = M.infer(w.astype(np.float64), feat[None, :].astype(np.float32))[0]
        want_f = np.stack([E.T @ y[0:3], E.T @ y[6:9]])
        want_t = np.stack([sign * (E.T @ y[3:6]), sign * (E.T @ y[9:12])])
        got_f = res[0]["force"] - res[1]["force"]
        got_t = res[0]["torque"] - res[1]["torque"]
        scale = np.abs(y).max()
        assert np.abs(got_f - want_f).max() <= 1e-4 * scale, (d, got_f, want_f)
        assert np.abs(got_t - want_t).max() <= 1e-4 * scale, (d, got_t, want_t)
    on.close()
    off.close()


@pytest.mark.gpu
def test_trained_closure_beats_plain_method_on_held_out_pairs():
    """Small end-to-end run: R_hi = 6 in 32^3 resolves, R_lo = 3 in 16^3 does not (gap/R in [0.05, 0.6]).

    Training data: the resistance of every lattice class in the envelope (32
    classes) with sampled velocities; held out: pairs run directly in random
    orientations with random velocities.  Relative L2 of the pair forces.
    """
    from lbcuda_b200 import closure
    gr = (0.05, 0.6)
    res = closure.resistance(R_hi=6, L_hi=32, R_lo=3, steps_hi=160, gap_range=gr)
    X, T, _ = closure.synthesize(res, 128, seed=1)
    w, loss = closure.train(X, T, epochs=100, lr=2e-3)
    Xh, Th, info = closure.generate(24, R_hi=6, L_hi=32, R_lo=3, steps_hi=160, seed=5, gap_range=gr)
    f = [0, 1, 2, 6, 7, 8]
    hi = np.linalg.norm((info["base"] + Th)[:, f])
    none = np.linalg.norm(Th[:, f]) / hi
    lub = np.linalg.norm((Th - closure.analytic_lubrication(Xh, 3.0))[:, f]) / hi
    net = np.linalg.norm((Th - closure.infer(w, Xh))[:, f]) / hi
    print(f"held-out pair-force error: none {none:.3f} analytic {lub:.3f} closure {net:.3f}; loss {loss[-1]:.2e}")
    assert net < 0.5 * min(none, lub)


@pytest.mark.gpu
def test_batched_pair_runs_equal_single_runs():
    """run_pairs (boxes advanced together in one ensemble) gives each configuration the bits of run_pair."""
    from lbcuda_b200 import closure
    z = np.zeros(3)
    cfgs = [dict(d=np.array([7.0, 1.0, 0.0]), dv=np.array([1e-3, 0, 0]), oi=z, oj=z),
            dict(d=np.array([6.0, 3.0, 2.0]), dv=z, oi=np.array([0, 5e-4, 0]), oj=z),
            dict(d=np.array([8.0, 0.0, 0.0]), dv=z, oi=z, oj=z)]
    batched = closure.run_pairs(cfgs, 3, 24, 40)
    for cfg, b in zip(cfgs, batched):
        single = closure.run_pair(cfg, 3, 24, 40)
        assert np.array_equal(b[0], single[0])
