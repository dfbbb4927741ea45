"""CPU reference of the learned pair closure network (TEST INFRASTRUCTURE ONLY).

numpy FP64 forward pass and mean-squared-error gradient of the
11 -> 64 -> 64 -> 64 -> 12 SiLU network whose weights travel as the flat
blob described in include/lbx.h (LBX_CLOSURE_NWEIGHTS floats).  Used to check
the GPU kernels lbx_closure_infer / lbx_closure_grad.  The closure has no
counterpart in the reference, so this is checked against finite differences
in tests/test_closure.py.
"""
import numpy as np

DIN, H, DOUT = 13, 64, 12


def layout():
    off = {}
    o = 0
    for name, size in (("W0", H * DIN), ("b0", H), ("W1", H * H), ("b1", H), ("W2", H * H), ("b2", H),
                       ("W3", DOUT * H), ("b3", DOUT)):
        off[name] = (o, size)
        o += size
    nparam = o
    for name, size in (("xmu", DIN), ("xsd", DIN), ("ymu", DOUT), ("ysd", DOUT)):
        off[name] = (o, size)
        o += size
    return off, nparam, o


OFF, NPARAM, TOTAL = layout()


def unpack(w):
    w = np.asarray(w, np.float64)
    g = lambda k: w[OFF[k][0]:OFF[k][0] + OFF[k][1]]
    return dict(W0=g("W0").reshape(H, DIN), b0=g("b0"), W1=g("W1").reshape(H, H), b1=g("b1"),
                W2=g("W2").reshape(H, H), b2=g("b2"), W3=g("W3").reshape(DOUT, H), b3=g("b3"),
                xmu=g("xmu"), xsd=g("xsd"), ymu=g("ymu"), ysd=g("ysd"))


def silu(z):
    return z / (1.0 + np.exp(-z))


def dsilu(z):
    s = 1.0 / (1.0 + np.exp(-z))
    return s * (1.0 + z * (1.0 - s))


def forward_std(p, xs):
    """Standardised input -> standardised output, with the pre-activations."""
    z1 = xs @ p["W0"].T + p["b0"]
    z2 = silu(z1) @ p["W1"].T + p["b1"]
    z3 = silu(z2) @ p["W2"].T + p["b2"]
    y = silu(z3) @ p["W3"].T + p["b3"]
    return y, (z1, z2, z3)


def infer(w, X):
    p = unpack(w)
    xs = (np.asarray(X, np.float64) - p["xmu"]) / p["xsd"]
    y, _ = forward_std(p, xs)
    return y * p["ysd"] + p["ymu"]


def loss_std(w, Xs, Ts):
    p = unpack(w)
    y, _ = forward_std(p, np.asarray(Xs, np.float64))
    return float(((y - Ts) ** 2).mean())


def grad_std(w, Xs, Ts):
    """d(mean squared error)/d(params) on standardised data, flat NPARAM vector."""
    p = unpack(w)
    Xs = np.asarray(Xs, np.float64)
    Ts = np.asarray(Ts, np.float64)
    y, (z1, z2, z3) = forward_std(p, Xs)
    n = Xs.shape[0]
    dy = 2.0 * (y - Ts) / (n * DOUT)
    a3 = silu(z3)
    g = {}
    g["W3"] = dy.T @ a3
    g["b3"] = dy.sum(0)
    dz3 = (dy @ p["W3"]) * dsilu(z3)
    a2 = silu(z2)
    g["W2"] = dz3.T @ a2
    g["b2"] = dz3.sum(0)
    dz2 = (dz3 @ p["W2"]) * dsilu(z2)
    a1 = silu(z1)
    g["W1"] = dz2.T @ a1
    g["b1"] = dz2.sum(0)
    dz1 = (dz2 @ p["W1"]) * dsilu(z1)
    g["W0"] = dz1.T @ Xs
    g["b0"] = dz1.sum(0)
    out = np.zeros(NPARAM)
    for k in ("W0", "b0", "W1", "b1", "W2", "b2", "W3", "b3"):
        o, s = OFF[k]
        out[o:o + s] = g[k].ravel()
    return out
