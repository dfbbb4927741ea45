"""Learned pair closure: data generation, training and use (host side).

The closure corrects the force and torque of near-contact sphere pairs that
the lattice resolves poorly (small radius).  Its training data come from the
method itself: the same two-sphere configuration is run with prescribed
sphere motion (``kinematic`` contexts, frozen geometry) once well resolved
(radius R_hi in an L_hi^3 box) and once at the deployment radius R_lo (box,
gap and time scaled by s = R_lo/R_hi, s^2 for time; translational
velocities equal, angular velocities scaled by s so that the surface
velocities agree).  For such dynamically similar Stokes flows forces scale
as mu R U and torques as mu R^2 U, so the target is F_hi s - F_lo and
T_hi s^2 - T_lo.  Each force is the difference between the run with the
sampled motion and the same configuration at rest: two spheres closer than
a few cells hide some of each other's surface links, which leaves a static
pressure imbalance that does not depend on the motion.

Pairs are described in a pair frame fixed to the lattice (lattice_frame):
the lattice and a sphere template centred on a site are invariant under the
48 signed axis permutations, so every pair whose separation vector is one of
a class under that group has the same forces in that frame.  At R_lo the
rounded centres put every pair on one of finitely many classes (121 for
gap/R in [0.05, 1.5] at R_lo = 3); the flow is linear in the sphere
velocities at these Reynolds numbers, so per class a rest run and nine
unit-velocity runs at each resolution give the whole correction as a 12 x 9
matrix (resistance), from which training samples for any velocities follow
(synthesize).  Held-out pairs are run directly (generate) in random
orientations.  Training and inference run in the library's own kernels
(lbx_closure_train / lbx_closure_infer); the analytic lubrication of the
reference stays the fallback outside the training envelope and the judge of
the gain.
"""
import ctypes as C

import numpy as np

from . import capi
from .sim import LBSim, make_params

DIN, H, DOUT = 13, 64, 12  # inputs: gap/R, pair-frame dv, w_i, w_j, R, nc_1, nc_2
NW = 10046
NPARAM = 9996
XMU, XSD, YMU, YSD = NPARAM, NPARAM + DIN, NPARAM + 2 * DIN, NPARAM + 2 * DIN + DOUT


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def pair_frame(n):
    """(t1, t2) completing n: t1 = unit(n x e_k), e_k the axis least aligned with n."""
    n = np.asarray(n, np.float64)
    k = int(np.argmin(np.abs(n)))
    e = np.zeros(3)
    e[k] = 1.0
    t1 = np.cross(n, e)
    t1 /= np.linalg.norm(t1)
    return t1, np.cross(n, t1)


def nint(x):
    """Fortran NINT (half away from zero), the rounding that places a sphere's template."""
    x = np.asarray(x, np.float64)
    return np.sign(x) * np.floor(np.abs(x) + 0.5)


def lattice_frame(n):
    """(E, sign, nc): the closure's pair frame, fixed to the lattice (lattice_frame, lbx_closure.h).

    P, the signed axis permutation (stable order by descending |n|, ties to
    the lower axis, sign + for n_k >= 0) that takes n to nc = P n in the
    cubic fundamental domain; rows of E: n, P^T t1(nc), P^T t2(nc); sign =
    det P.  Pair-frame components: E v for velocities and forces, sign * E w
    for angular velocities and torques.
    """
    n = np.asarray(n, np.float64)
    a = np.abs(n)
    o = sorted(range(3), key=lambda k: (-a[k], k))
    sg = np.where(n >= 0.0, 1.0, -1.0)
    nc = a[o]
    t1, t2 = pair_frame(nc)
    E = np.zeros((3, 3))
    E[0] = n
    for r, k in enumerate(o):
        E[1, k] = sg[k] * t1[r]
        E[2, k] = sg[k] * t2[r]
    inv = int(o[0] > o[1]) + int(o[0] > o[2]) + int(o[1] > o[2])
    return E, (-1.0 if inv & 1 else 1.0) * sg[0] * sg[1] * sg[2], nc


def to_pair(out, E, sign):
    """(F_i, T_i, F_j, T_j) lab (4, 3) -> the 12 pair-frame components."""
    out = np.asarray(out, np.float64)
    return np.concatenate([E @ out[0], sign * (E @ out[1]), E @ out[2], sign * (E @ out[3])])


def features(xi, xj, vi, vj, oi, oj, R, box):
    """The 13 closure inputs of pair (i, j) (lab angular velocities) and (E, sign).

    Gap and frame come from the rounded centres, where the spheres'
    templates actually sit: an under-resolved pair's forces follow its
    discrete geometry, which can differ from the nominal one by a cell.
    """
    d = nint(xj) - nint(xi)
    box = np.asarray(box, np.float64)
    d = d - box * nint(d / box)
    r = np.linalg.norm(d)
    E, sign, nc = lattice_frame(d / r)
    dv = E @ (np.asarray(vj, np.float64) - np.asarray(vi, np.float64))
    x = np.concatenate([[(r - 2 * R) / R], dv, sign * (E @ np.asarray(oi, np.float64)),
                        sign * (E @ np.asarray(oj, np.float64)), [R], nc[1:]])
    return x, (E, sign)


def lattice_classes(R, gap_range=(0.05, 1.5)):
    """Separation vectors a >= b >= c >= 0 (one per lattice class) with gap/R in the range, by |d|."""
    hi = (2.0 + gap_range[1]) * R
    m = int(np.floor(hi)) + 1
    out = []
    for a in range(m + 1):
        for b in range(a + 1):
            for c in range(b + 1):
                g = np.sqrt(a * a + b * b + c * c) / R - 2.0
                if gap_range[0] <= g <= gap_range[1]:
                    out.append((a, b, c))
    return sorted(out, key=lambda t: (t[0] ** 2 + t[1] ** 2 + t[2] ** 2, t))


def sample_configs(n, seed=0, gap_range=(0.05, 1.5), vmax=1e-3):
    """gap/R log-uniform, pair-frame relative velocity and both angular velocities uniform in +-vmax."""
    rng = np.random.Generator(np.random.PCG64(seed))
    gaps = np.exp(rng.uniform(np.log(gap_range[0]), np.log(gap_range[1]), n))
    dirs = rng.normal(size=(n, 3))
    dirs /= np.linalg.norm(dirs, axis=1, keepdims=True)
    dv = rng.uniform(-vmax, vmax, (n, 3))
    oi = rng.uniform(-vmax, vmax, (n, 3))
    oj = rng.uniform(-vmax, vmax, (n, 3))
    return [dict(gap=g, n=d, dv=a, oi=b, oj=c) for g, d, a, b, c in zip(gaps, dirs, dv, oi, oj)]


def _pair_params(R, L, storage="f32", lubrication=False):
    """lbx_params of the closure's two-sphere runs: frozen geometry (kinematic = 2), rotation, neutral
    wetting, every template cell placed (exact_tiles = 0), Hertz only on overlap."""
    return make_params(L, model="cg", storage=storage, max_particles=2, radius=float(R), kinematic=2,
                       lrotate=1, wetting="neutral", max_vel=1.0,
                       hz_rmin=float(2 * R - 0.5), hz_rcap=float(2 * R - 2.0),
                       lubrication=1 if lubrication else 0, lubric_k=1.0 / 6.0, lubric_rmin=1.0,
                       lubric_rcap=float(0.05 * R), exact_tiles=0)


def _pair_state(cfg, L, mult=1):
    """Centres, velocities and angular velocities (lab frame) of a pair configuration."""
    d = np.asarray(cfg["d"], np.float64) * mult
    E, sign, _ = lattice_frame(d / np.linalg.norm(d))
    dv = E.T @ np.asarray(cfg["dv"], np.float64)
    oi = sign * (E.T @ np.asarray(cfg["oi"], np.float64))
    oj = sign * (E.T @ np.asarray(cfg["oj"], np.float64))
    c = np.full(3, float(L // 2))
    xj = (c + d - 1.0) % L + 1.0
    return np.stack([c, xj]), np.stack([-0.5 * dv, 0.5 * dv]), np.stack([oi, oj])


def run_pair(cfg, R, L, steps, average=0.25, storage="f32", lubrication=False, sim_cache=None, mult=1):
    """Forces / torques on both spheres of a prescribed-motion two-sphere run.

    Spheres of radius R on lattice sites, the second at mult * cfg['d'] (an
    integer lattice vector) from the first, velocities -dv/2 and +dv/2 and
    angular velocities oi, oj, all given in the lattice pair frame of d
    (body frame = lab, identity orientation).  The geometry is frozen
    (kinematic = 2): the spheres keep their place while their bounce-back
    walls move with the set velocities, so the forces belong to this
    configuration and no cell is filled or drained during the run.  Returns
    (F_i, T_i, F_j, T_j) in the lab frame, averaged over the last `average`
    fraction of the steps, and the configuration (x, v, omega).
    """
    x, v, om = _pair_state(cfg, L, mult)
    key = (R, L, storage, lubrication)
    sim = sim_cache.get(key) if sim_cache is not None else None
    if sim is None:
        sim = LBSim(_pair_params(R, L, storage, lubrication))
        if sim_cache is not None:
            sim_cache[key] = sim
    one = np.ones((L, L, L), np.float32)
    sim.set_fields(one, np.zeros_like(one))
    nav = max(1, int(round(steps * average)))
    sim.set_particles(x, v, om, None)
    sim.step(steps - nav)
    acc = np.zeros((4, 3))
    for _ in range(nav):
        sim.step(1)
        d = sim.get_particles()
        acc += np.stack([d["force"][0], d["torque"][0], d["force"][1], d["torque"][1]])
    return acc / nav, x, v, om


def run_pairs(cfgs, R, L, steps, average=0.25, storage="f32", mult=1, mem_bytes=60e9):
    """run_pair for many configurations: their boxes advance together, as many at a time as fit in
    mem_bytes of device memory, in one ensemble (one persistent fluid kernel per step, the sphere
    kernels of the boxes side by side); each box gives the bits of its own run_pair.  Returns the list
    of (forces (4, 3), x, v, omega)."""
    from .ensemble import Ensemble
    nav = max(1, int(round(steps * average)))
    per_box = L ** 3 * (19 * 2 * {"f32": 4, "f64": 8}.get(storage, 2) * 2 + 40)
    batch = max(1, min(len(cfgs), int(mem_bytes // per_box)))
    p = _pair_params(R, L, storage)
    one = np.ones((L, L, L), np.float32)
    zero = np.zeros_like(one)
    out = []
    for b0 in range(0, len(cfgs), batch):
        chunk = cfgs[b0:b0 + batch]
        ens = Ensemble([p] * len(chunk))
        states = []
        for box, cfg in zip(ens.boxes, chunk):
            x, v, om = _pair_state(cfg, L, mult)
            box.set_fields(one, zero)
            box.set_particles(x, v, om, None)
            states.append((x, v, om))
        ens.step(steps - nav)
        acc = np.zeros((len(chunk), 4, 3))
        for _ in range(nav):
            ens.step(1)
            for i, box in enumerate(ens.boxes):
                d = box.get_particles()
                acc[i] += np.stack([d["force"][0], d["torque"][0], d["force"][1], d["torque"][1]])
        ens.close()
        out.extend((acc[i] / nav,) + states[i] for i in range(len(chunk)))
    return out


def _scales(R_hi, L_hi, R_lo, steps_hi, gap_range):
    s = R_lo / R_hi
    L_lo = int(round(L_hi * s))
    steps_lo = max(8, int(round(steps_hi * s * s)))
    for L, R in ((L_hi, R_hi), (L_lo, R_lo)):
        if L < (4.0 + 2.0 * gap_range[1]) * R:
            raise ValueError(f"box {L} too small for radius {R} and gap/R up to {gap_range[1]}")
    if abs(R_hi / R_lo - round(R_hi / R_lo)) > 1e-12:
        raise ValueError("R_hi must be an integer multiple of R_lo")
    if L_hi % 8 or L_lo % 8:
        raise ValueError(f"boxes {L_hi} and {L_lo} must be multiples of 8 (the particle tile grid)")
    return s, L_lo, steps_lo, int(round(R_hi / R_lo))


# force and torque scaling from R_hi to R_lo (F_i, T_i, F_j, T_j in the 12 components)
def _out_scale(s):
    return np.repeat([s, s * s, s, s * s], 3)


def generate(n_samples, R_hi=12, L_hi=128, R_lo=3, steps_hi=300, seed=0, progress=None, gap_range=(0.05, 1.5),
             subtract_static=True):
    """(X, T, info) from direct runs: random pairs, features at R_lo and targets (resolved - under-resolved).

    Gap/R log-uniform in the range, separation direction uniform (so every
    lattice orientation occurs), velocities uniform in +-1e-3 in the pair
    frame.  The periodic box must keep each sphere's image farther away than
    its partner: L >= (4 + 2 gap_max) R, checked at both resolutions.
    """
    s, L_lo, steps_lo, mult = _scales(R_hi, L_hi, R_lo, steps_hi, gap_range)
    # separations on the R_lo lattice (R_hi: the same vector times R_hi / R_lo),
    # nearest to the sampled gap and direction, kept inside the gap range
    cfgs = []
    pool = sample_configs(8 * n_samples, seed, gap_range=gap_range)
    for cfg in pool:
        d = nint(np.asarray(cfg["n"]) * (2.0 + cfg["gap"]) * R_lo)
        gap = np.linalg.norm(d) / R_lo - 2.0
        if gap_range[0] <= gap <= gap_range[1]:
            cfgs.append(dict(cfg, d=d, gap=gap, n=d / np.linalg.norm(d)))
        if len(cfgs) == n_samples:
            break
    if len(cfgs) < n_samples:
        raise ValueError("gap range admits too few lattice separations")
    X = np.zeros((n_samples, DIN))
    T = np.zeros((n_samples, DOUT))
    base = np.zeros((n_samples, DOUT))
    z = np.zeros(3)
    cfg_hi = [dict(c, oi=np.asarray(c["oi"]) * s, oj=np.asarray(c["oj"]) * s) for c in cfgs]
    rest = [dict(c, dv=z, oi=z, oj=z) for c in cfgs]
    hi = run_pairs(cfg_hi + (rest if subtract_static else []), R_hi, L_hi, steps_hi, mult=mult)
    lo = run_pairs(cfgs + (rest if subtract_static else []), R_lo, L_lo, steps_lo)
    for k, cfg in enumerate(cfgs):
        f_hi, f_lo = hi[k][0], lo[k][0]
        x, v, om = lo[k][1:]
        if subtract_static:
            f_hi = f_hi - hi[n_samples + k][0]
            f_lo = f_lo - lo[n_samples + k][0]
        feat, (E, sign) = features(x[0], x[1], v[0], v[1], om[0], om[1], R_lo, (L_lo,) * 3)
        X[k] = feat
        T[k] = to_pair(f_hi, E, sign) * _out_scale(s) - to_pair(f_lo, E, sign)
        base[k] = to_pair(f_lo, E, sign)
        if progress and (k + 1) % progress == 0:
            print(f"closure data {k + 1}/{n_samples}", flush=True)
    return X, T, dict(base=base, cfgs=cfgs, steps_hi=steps_hi, steps_lo=steps_lo, L_lo=L_lo)


def resistance(R_hi=12, L_hi=96, R_lo=3, steps_hi=960, gap_range=(0.05, 1.5), amp=1e-3, progress=None):
    """Per lattice class: the pair-frame response of both resolutions to unit sphere velocities.

    For each class (lattice_classes, separation in the fundamental domain,
    so its frame needs no sign) a rest run and nine runs with one pair-frame
    velocity component (dv, w_i, w_j) set to amp, at R_lo and at R_hi
    (angular components times s there).  Returns dict with 'classes' (C, 3),
    'gap' (C,), 'M_lo' and 'M_hi' (C, 12, 9): pair-frame force and torque per
    unit R_lo-frame velocity, M_hi already scaled to R_lo units, so that a
    pair with velocities q has target (M_hi - M_lo) q.
    """
    s, L_lo, steps_lo, mult = _scales(R_hi, L_hi, R_lo, steps_hi, gap_range)
    classes = lattice_classes(R_lo, gap_range)
    C = len(classes)
    M_lo = np.zeros((C, DOUT, 9))
    M_hi = np.zeros((C, DOUT, 9))
    z = np.zeros(3)
    # per class: the rest run and the nine unit-velocity runs, every class's runs advanced together
    lo_cfgs, hi_cfgs = [], []
    for dcl in classes:
        d = np.asarray(dcl, np.float64)
        lo_cfgs.append(dict(d=d, dv=z, oi=z, oj=z))
        hi_cfgs.append(dict(d=d, dv=z, oi=z, oj=z))
        for k in range(9):
            e = np.zeros(9)
            e[k] = amp
            lo_cfgs.append(dict(d=d, dv=e[:3], oi=e[3:6], oj=e[6:]))
            hi_cfgs.append(dict(d=d, dv=e[:3], oi=e[3:6] * s, oj=e[6:] * s))
    lo = run_pairs(lo_cfgs, R_lo, L_lo, steps_lo)
    hi = run_pairs(hi_cfgs, R_hi, L_hi, steps_hi, mult=mult)
    for c, dcl in enumerate(classes):
        d = np.asarray(dcl, np.float64)
        E, sign, _ = lattice_frame(d / np.linalg.norm(d))
        r_lo = to_pair(lo[10 * c][0], E, sign)
        r_hi = to_pair(hi[10 * c][0], E, sign)
        for k in range(9):
            M_lo[c, :, k] = (to_pair(lo[10 * c + 1 + k][0], E, sign) - r_lo) / amp
            M_hi[c, :, k] = (to_pair(hi[10 * c + 1 + k][0], E, sign) - r_hi) / amp * _out_scale(s)
        if progress and (c + 1) % progress == 0:
            print(f"closure classes {c + 1}/{C}", flush=True)
    gap = np.array([np.linalg.norm(d) / R_lo - 2.0 for d in classes])
    return dict(classes=np.array(classes, np.float64), gap=gap, M_lo=M_lo, M_hi=M_hi, R_lo=float(R_lo),
                R_hi=float(R_hi), steps_hi=steps_hi, steps_lo=steps_lo, L_lo=L_lo)


def synthesize(res, m, seed=0, vmax=1e-3):
    """(X, T, base): m samples per class, pair-frame velocities uniform in +-vmax, targets from the matrices."""
    rng = np.random.Generator(np.random.PCG64(seed))
    C = len(res["gap"])
    Q = rng.uniform(-vmax, vmax, (C, m, 9))
    X = np.zeros((C, m, DIN))
    X[:, :, 0] = res["gap"][:, None]
    X[:, :, 1:10] = Q
    X[:, :, 10] = res["R_lo"]
    nc = res["classes"] / np.linalg.norm(res["classes"], axis=1, keepdims=True)
    X[:, :, 11:13] = nc[:, None, 1:3]
    T = np.einsum("cij,cmj->cmi", res["M_hi"] - res["M_lo"], Q)
    base = np.einsum("cij,cmj->cmi", res["M_lo"], Q)
    return X.reshape(C * m, DIN), T.reshape(C * m, DOUT), base.reshape(C * m, DOUT)


def init_weights(X, T, seed=0):
    w = np.zeros(NW, np.float32)
    capi.check(capi.lib().lbx_closure_init(_fp(w), int(seed)), "lbx_closure_init")
    w[XMU:XMU + DIN] = X.mean(0)
    w[XSD:XSD + DIN] = np.maximum(X.std(0), 1e-12)
    w[YMU:YMU + DOUT] = T.mean(0)
    w[YSD:YSD + DOUT] = np.maximum(T.std(0), 1e-12)
    return w


def train(X, T, epochs=500, lr=2e-3, seed=0, w=None):
    X = np.ascontiguousarray(X, np.float32)
    T = np.ascontiguousarray(T, np.float32)
    if w is None:
        w = init_weights(X, T, seed)
    loss = np.zeros(epochs, np.float32)
    capi.check(capi.lib().lbx_closure_train(_fp(w), _fp(X), _fp(T), X.shape[0], int(epochs), float(lr), int(seed),
                                            _fp(loss)), "lbx_closure_train")
    return w, loss


def infer(w, X):
    X = np.ascontiguousarray(X, np.float32)
    Y = np.zeros((X.shape[0], DOUT), np.float32)
    capi.check(capi.lib().lbx_closure_infer(_fp(np.ascontiguousarray(w, np.float32)), _fp(X), X.shape[0], _fp(Y)),
               "lbx_closure_infer")
    return Y


def grad(w, Xs, Ts):
    Xs = np.ascontiguousarray(Xs, np.float32)
    Ts = np.ascontiguousarray(Ts, np.float32)
    g = np.zeros(NPARAM, np.float32)
    capi.check(capi.lib().lbx_closure_grad(_fp(np.ascontiguousarray(w, np.float32)), _fp(Xs), _fp(Ts), Xs.shape[0],
                                           _fp(g)), "lbx_closure_grad")
    return g


def analytic_lubrication(X, R, mu=1.0 / 6.0, rcut_gap=1.0, rcap_gap=None):
    """The reference's normal squeeze force (addHertzian's lubrication branch) in the pair frame.

    F_j = -F_i = lubfactor n (n.(v_i - v_j)) (1/h - 1), h = max(gap, rcap) (lattice units),
    applied for gap <= rcut_gap; lubfactor = mu 6 pi R^4 / (2R)^2.
    """
    rcap_gap = 0.05 * R if rcap_gap is None else rcap_gap
    out = np.zeros((X.shape[0], DOUT))
    h = X[:, 0] * R
    lubfactor = mu * 6 * np.pi * R ** 4 / (2 * R) ** 2
    dvn = X[:, 1]                      # (v_j - v_i).n
    hh = np.maximum(h, rcap_gap)
    f = np.where(h <= rcut_gap, lubfactor * (-dvn) * (1.0 / hh - 1.0), 0.0)
    out[:, 0] = -f
    out[:, 6] = f
    return out


def window_positions(L, n, R, seed=0, min_gap=0.05, tries=200000):
    """n sphere centres of radius R on lattice sites of a periodic L^3 box, every centre distance at least
    (2 + min_gap) R (random sequential placement)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    dmin2 = ((2.0 + min_gap) * R) ** 2
    x = np.zeros((0, 3))
    for _ in range(tries):
        if len(x) == n:
            break
        c = rng.integers(1, L + 1, 3).astype(np.float64)
        d = x - c
        d -= L * np.round(d / L)
        if not len(x) or (d * d).sum(1).min() >= dmin2:
            x = np.vstack([x, c])
    return x


def _window_run(x, v, om, R, L, steps, average=0.25, closure=0, lubrication=0, weights=None):
    """Frozen-geometry suspension run: the spheres' forces and torques averaged over the last steps,
    and the ms per step."""
    n = len(x)
    p = make_params(L, model="cg", storage="f32", max_particles=n, radius=float(R), kinematic=2, lrotate=1,
                    wetting="neutral", max_vel=1.0, hz_rmin=float(2 * R - 0.5), hz_rcap=float(2 * R - 2.0),
                    lubrication=lubrication, lubric_k=1.0 / 6.0, lubric_rmin=1.0, lubric_rcap=float(0.05 * R),
                    exact_tiles=0, closure=closure)
    sim = LBSim(p)
    if weights is not None:
        wf = np.ascontiguousarray(weights, np.float32)
        capi.check(capi.lib().lbx_closure_set(sim._h, _fp(wf)), "lbx_closure_set")
    one = np.ones((L, L, L), np.float32)
    sim.set_fields(one, np.zeros_like(one))
    sim.set_particles(x, v, om, None)
    nav = max(1, int(round(steps * average)))
    sim.step(1)
    sim.sync()
    ms, _, _ = sim.time_steps(steps - nav - 1, kernel_timing=False)
    F = np.zeros((n, 3))
    T = np.zeros((n, 3))
    for _ in range(nav):
        sim.step(1)
        d = sim.get_particles()
        F += d["force"]
        T += d["torque"]
    code = sim.status()[0]
    sim.close()
    return F / nav, T / nav, ms / max(1, steps - nav - 1), code


def window_score(w, L_lo=64, R_lo=3, scale=4, n=460, steps_lo=60, vmax=5e-4, seed=21, gap_max=1.5):
    """A many-body check of the closure on a suspension window: n spheres of radius R_lo on lattice
    sites of an L_lo^3 box (volume fraction about 0.2, gaps from 0.05 R), translational and angular
    velocities uniform in +-vmax (frozen geometry, walls moving), and the same system resolved at
    R_hi = scale * R_lo: centres times scale in a (scale L_lo)^3 box, scale^2 times the steps, angular
    velocities divided by scale.  Each sphere's force and torque with motion minus those at rest,
    resolved and scaled to R_lo (F s, T s^2, s = 1/scale), is the target; the R_lo run is scored plain,
    with the reference's analytic lubrication, and with the closure (analytic outside its envelope).
    Returns relative L2 errors over all spheres and over the spheres with a partner within gap_max R,
    the median per-sphere error, the share within 5 %, and the cost of both resolutions."""
    s = 1.0 / scale
    rng = np.random.Generator(np.random.PCG64(seed + 1))
    x = window_positions(L_lo, n, R_lo, seed)
    n = len(x)
    v = rng.uniform(-vmax, vmax, (n, 3))
    om = rng.uniform(-vmax, vmax, (n, 3))
    L_hi, R_hi, steps_hi = L_lo * scale, R_lo * scale, steps_lo * scale * scale
    xh = scale * x
    z = np.zeros_like(v)
    Fm, Tm, ms_hi, c1 = _window_run(xh, v, om * s, R_hi, L_hi, steps_hi)
    Fr, Tr, _, c2 = _window_run(xh, z, z, R_hi, L_hi, steps_hi)
    tgt = np.concatenate([(Fm - Fr) * s, (Tm - Tr) * s * s], axis=1)
    F0, T0, _, c3 = _window_run(x, z, z, R_lo, L_lo, steps_lo)
    d = x[:, None, :] - x[None, :, :]
    d -= L_lo * np.round(d / L_lo)
    gap = np.sqrt((d * d).sum(-1)) / R_lo - 2.0
    np.fill_diagonal(gap, np.inf)
    close = (gap <= gap_max).any(axis=1)
    out = {"box_lo": L_lo, "R_lo": R_lo, "box_hi": L_hi, "R_hi": R_hi, "spheres": n,
           "volume_fraction": n * 4.0 / 3.0 * np.pi * R_lo ** 3 / L_lo ** 3, "steps_lo": steps_lo,
           "steps_hi": steps_hi, "spheres_with_close_partner": int(close.sum()),
           "close_pairs": int((gap[np.triu_indices(n, 1)] <= gap_max).sum()), "device_errors": [c1, c2, c3]}

    def score(pred):
        err = pred - tgt
        per = np.linalg.norm(err[:, :3], axis=1) / np.maximum(np.linalg.norm(tgt[:, :3], axis=1), 1e-30)
        return {"force_rel_l2": float(np.linalg.norm(err[:, :3]) / np.linalg.norm(tgt[:, :3])),
                "force_rel_l2_close": float(np.linalg.norm(err[close, :3]) / np.linalg.norm(tgt[close, :3])),
                "torque_rel_l2": float(np.linalg.norm(err[:, 3:]) / np.linalg.norm(tgt[:, 3:])),
                "median_sphere": float(np.median(per)), "spheres_within_5pct": float(np.mean(per <= 0.05))}

    runs = {"plain": dict(), "analytic_lubrication": dict(lubrication=1),
            "closure": dict(closure=1, lubrication=1, weights=w)}
    ms_lo = {}
    for name, kw in runs.items():
        F, T, ms, code = _window_run(x, v, om, R_lo, L_lo, steps_lo, **kw)
        out[name] = score(np.concatenate([F - F0, T - T0], axis=1))
        out[name]["device_error"] = code
        ms_lo[name] = ms
    out["ms_per_step"] = {"R_hi": ms_hi, "R_lo_closure": ms_lo["closure"], "R_lo_plain": ms_lo["plain"]}
    out["cost_ratio_same_physical_time"] = ms_hi * steps_hi / (ms_lo["closure"] * steps_lo)
    return out
