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
    w[M.OFF["xmu"][0]:M.OFF["xmu"][0] + 11] = rng.normal(0, 0.1, 11)
    w[M.OFF["xsd"][0]:M.OFF["xsd"][0] + 11] = rng.uniform(0.5, 2.0, 11)
    w[M.OFF["ymu"][0]:M.OFF["ymu"][0] + 12] = rng.normal(0, 0.1, 12)
    w[M.OFF["ysd"][0]:M.OFF["ysd"][0] + 12] = rng.uniform(0.5, 2.0, 12)
    return w


def test_numpy_reference_gradient_matches_finite_differences():
    w = random_blob(1).astype(np.float64)
    X = RNG.normal(size=(24, 11))
    T = RNG.normal(size=(24, 12))
    g = M.grad_std(w, X, T)
    for idx in (0, 7, 700, 790, 3000, 5000, 9000, M.NPARAM - 1):
        e = 1e-6
        wp, wm = w.copy(), w.copy()
        wp[idx] += e
        wm[idx] -= e
        fd = (M.loss_std(wp, X, T) - M.loss_std(wm, X, T)) / (2 * e)
        assert abs(fd - g[idx]) <= 1e-6 + 1e-5 * abs(fd)


def test_pair_frame_and_features():
    from lbcuda_b200.closure import features, pair_frame
    for n in RNG.normal(size=(20, 3)):
        n /= np.linalg.norm(n)
        t1, t2 = pair_frame(n)
        F = np.stack([n, t1, t2])
        assert np.allclose(F @ F.T, np.eye(3), atol=1e-12)
    x, F = features([10, 10, 10], [17.5, 10, 10], [0, 0, 0], [-1e-3, 0, 0], [0, 0, 0], [0, 0, 0], 3.0, (32,) * 3)
    # the gap of the rounded centres (the templates sit at 10 and NINT(17.5) = 18)
    assert abs(x[0] - 2.0 / 3.0) < 1e-12 and abs(x[1] + 1e-3) < 1e-15 and x[10] == 3.0
    # periodic image: the pair across the boundary (NINT(31.5) = 32, one cell from 1)
    x, _ = features([1, 10, 10], [31.5, 10, 10], [0, 0, 0], [0, 0, 0], [0, 0, 0], [0, 0, 0], 3.0, (32,) * 3)
    assert abs(x[0] - (1.0 - 6) / 3) < 1e-12


def test_analytic_lubrication_is_repulsive_on_approach():
    from lbcuda_b200.closure import analytic_lubrication
    X = np.zeros((2, 11))
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
    Xs = RNG.normal(size=(64, 11)).astype(np.float32)
    Ts = RNG.normal(size=(64, 12)).astype(np.float32)
    g_gpu = closure.grad(w, Xs, Ts)
    g_ref = M.grad_std(w.astype(np.float64), Xs, Ts)
    err = np.abs(g_gpu - g_ref).max() / np.abs(g_ref).max()
    assert err < 1e-4, err


@pytest.mark.gpu
def test_gpu_inference_matches_numpy():
    from lbcuda_b200 import closure
    w = random_blob(3)
    X = RNG.normal(size=(1000, 11)).astype(np.float32)
    y = closure.infer(w, X)
    y_ref = M.infer(w.astype(np.float64), X)
    assert np.abs(y - y_ref).max() / np.abs(y_ref).max() < 1e-5


@pytest.mark.gpu
def test_gpu_training_fits_a_smooth_map():
    from lbcuda_b200 import closure
    X = RNG.uniform(-1, 1, size=(2048, 11)).astype(np.float32)
    A = RNG.normal(size=(11, 12)) / 3
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
        w[M.OFF["xsd"][0]:M.OFF["xsd"][0] + 11] = 1
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
def test_trained_closure_beats_plain_method_on_held_out_pairs():
    """Small end-to-end run: R_hi = 6 in 48^3 resolves, R_lo = 3 in 24^3 does not (gap/R up to 1.5)."""
    from lbcuda_b200 import closure
    X, T, info = closure.generate(192, R_hi=6, L_hi=48, R_lo=3, steps_hi=160, seed=5)
    ntr = 160
    w, loss = closure.train(X[:ntr], T[:ntr], epochs=300, lr=2e-3)
    pred = closure.infer(w, X[ntr:])
    base_err = np.linalg.norm(T[ntr:])                      # plain method: no correction
    lub_err = np.linalg.norm(T[ntr:] - closure.analytic_lubrication(X[ntr:], 4.0))
    net_err = np.linalg.norm(T[ntr:] - pred)
    print(f"targets |T| {np.abs(T).max(axis=0)}")
    print(f"held-out correction error: none {base_err:.3e} analytic {lub_err:.3e} closure {net_err:.3e}")
    assert net_err < base_err
