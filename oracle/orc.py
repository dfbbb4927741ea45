"""ctypes binding of the CPU oracle (oracle/lbx_oracle.cpp).

TEST INFRASTRUCTURE ONLY: imported by tests/, the smoke check and the
benchmark's CPU baseline / reference arm, never by the product package.
PARITY UNPINNED: see the header of lbx_oracle.cpp.
"""
import ctypes as C
import os

import numpy as np

_HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = os.path.join(_HERE, "liblbx_oracle.so")
Q = 19
MODES = {"ref": 0, "f32p64": 1, "f64": 2}
_lib = None


def lib():
    global _lib
    if _lib is None:
        if not os.path.exists(_LIB):
            from . import build
            build.build()
        L = C.CDLL(_LIB)
        P = C.c_void_p
        L.orc_create.restype = P
        L.orc_create.argtypes = [C.POINTER(Params), C.c_int]
        L.orc_default_params.argtypes = [C.POINTER(Params), C.c_int32, C.c_int32, C.c_int32]
        L.orc_destroy.argtypes = [P]
        L.orc_set_fields.argtypes = [P, C.POINTER(C.c_float), C.POINTER(C.c_float), C.c_float, C.c_float, C.c_float]
        L.orc_set_pops.argtypes = [P, C.POINTER(C.c_float), C.POINTER(C.c_float)]
        L.orc_step.argtypes = [P, C.c_int]
        D = C.POINTER(C.c_double)
        L.orc_get_fields.argtypes = [P, D, D, D, D]
        L.orc_get_pops.argtypes = [P, D, D]
        L.orc_get_flags.argtypes = [P, C.POINTER(C.c_int8)]
        L.orc_status.argtypes = [P, C.POINTER(C.c_int), C.POINTER(C.c_int), C.POINTER(C.c_int64)]
        L.orc_num_threads.restype = C.c_int
        L.orc_set_particles.argtypes = [P, C.c_int, D, D, D, D]
        L.orc_get_particles.argtypes = [P, D, D, D, D, D, D]
        L.orc_get_accumulators.argtypes = [P, D, D, D, D]
        L.orc_get_rho.argtypes = [P, D, D]
        L.orc_template.argtypes = [P, C.POINTER(C.c_int), C.POINTER(C.c_int8)]
        L.orc_record_links.argtypes = [P, C.c_int]
        L.orc_get_links.argtypes = [P, C.POINTER(C.c_int32), C.POINTER(C.c_int8), C.POINTER(C.c_int32), C.c_int64,
                                    C.POINTER(C.c_int64)]
        _lib = L
    return _lib


class Params(C.Structure):
    """lbx_params of include/lbx.h, mirrored here so that the oracle needs
    nothing of the product package (a CPU test checks both mirrors agree)."""
    _fields_ = [
        ("nx", C.c_int32), ("ny", C.c_int32), ("nz", C.c_int32),
        ("model", C.c_int32), ("storage", C.c_int32), ("wetting", C.c_int32),
        ("lrotate", C.c_int32), ("max_particles", C.c_int32),
        ("tau", C.c_float), ("tauR", C.c_float), ("tauB", C.c_float),
        ("sigma", C.c_float), ("beta", C.c_float),
        ("rho0R", C.c_float), ("rho0B", C.c_float),
        ("radius", C.c_float), ("rmass", C.c_float), ("max_vel", C.c_float),
        ("ext_force", C.c_float * 3), ("ext_torque", C.c_float * 3),
        ("hz_k", C.c_float), ("hz_rmin", C.c_float), ("hz_rcap", C.c_float),
        ("lubrication", C.c_int32),
        ("lubric_k", C.c_float), ("lubric_rmin", C.c_float), ("lubric_rcap", C.c_float),
        ("kinematic", C.c_int32), ("closure", C.c_int32),
        ("closure_gap_min", C.c_float), ("closure_gap_max", C.c_float), ("closure_vmax", C.c_float),
        ("exact_tiles", C.c_int32), ("densR", C.c_float), ("densB", C.c_float),
    ]


MODEL = {"bgk": 0, "cg": 1, "cg-diffdens": 2, "cg-d3q27": 3, "cg-diffdens-d3q27": 4}
WETTING = {"janus": 0, "neutral": 1}


def default_params(nx, ny=None, nz=None, model="cg", **kw):
    """The reference defaults (dimensions_m.CUF:50-99, restated by orc_default_params) with kw applied."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    p = Params()
    lib().orc_default_params(C.byref(p), nx, ny, nz)
    p.model = MODEL[model] if isinstance(model, str) else int(model)
    for k, v in kw.items():
        if k == "wetting" and isinstance(v, str):
            v = WETTING[v]
        if k in ("ext_force", "ext_torque"):
            getattr(p, k)[:] = list(v)
            continue
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def noise_fields(nx, ny, nz, mean=0.5, amp=0.01, seed=0, ncomp=2):
    """rho_k = mean + U(-amp, amp) per cell and component from numpy's PCG64
    with the given seed: the same fields the product's input helpers make."""
    rng = np.random.Generator(np.random.PCG64(seed))
    return [(np.float32(mean) + rng.uniform(-amp, amp, size=(nz, ny, nx))).astype(np.float32) for _ in range(ncomp)]


def _as_params(p):
    """Any structure with lbx_params' layout, as this module's Params."""
    if isinstance(p, Params):
        return p
    q = Params()
    if C.sizeof(p) != C.sizeof(q):
        raise TypeError("not an lbx_params layout")
    C.memmove(C.byref(q), C.byref(p), C.sizeof(q))
    return q


def num_threads():
    return lib().orc_num_threads()


def _p(a, t):
    return a.ctypes.data_as(C.POINTER(t)) if a is not None else None


class OracleSim:
    """Same surface as lbcuda_b200.LBSim, computed by the CPU restatement."""

    def __init__(self, params, mode="ref"):
        params = _as_params(params)
        self.params = params
        self.nx, self.ny, self.nz = params.nx, params.ny, params.nz
        self.ncomp = 1 if params.model == 0 else 2
        self.q = 27 if params.model in (3, 4) else Q  # the D3Q27 models
        self._L = lib()
        self._h = self._L.orc_create(C.byref(params), MODES[mode])
        if not self._h:
            raise RuntimeError("orc_create failed")

    @property
    def shape(self):
        return (self.nz, self.ny, self.nx)

    def close(self):
        if self._h:
            self._L.orc_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def set_fields(self, rhoR, rhoB=None, vel=(0.0, 0.0, 0.0)):
        rR = np.ascontiguousarray(rhoR, dtype=np.float32)
        rB = None if rhoB is None else np.ascontiguousarray(rhoB, dtype=np.float32)
        self._L.orc_set_fields(self._h, _p(rR, C.c_float), _p(rB, C.c_float), *map(float, vel))

    def set_pops(self, popsR, popsB=None):
        pR = np.ascontiguousarray(popsR, dtype=np.float32)
        pB = None if popsB is None else np.ascontiguousarray(popsB, dtype=np.float32)
        self._L.orc_set_pops(self._h, _p(pR, C.c_float), _p(pB, C.c_float))

    def step(self, n=1):
        return self._L.orc_step(self._h, int(n))

    def get_fields(self):
        rR = np.empty(self.shape)
        rB = np.empty(self.shape)
        vel = np.empty(self.shape + (3,))
        ph = np.empty(self.shape)
        D = C.c_double
        self._L.orc_get_fields(self._h, _p(rR, D), _p(rB, D), _p(vel, D), _p(ph, D))
        return rR, rB, vel, ph

    def get_pops(self):
        pR = np.empty((self.q,) + self.shape)
        pB = np.empty((self.q,) + self.shape)
        self._L.orc_get_pops(self._h, _p(pR, C.c_double), _p(pB, C.c_double))
        return pR, (pB if self.ncomp == 2 else None)

    def get_flags(self):
        f = np.empty(self.shape, np.int8)
        self._L.orc_get_flags(self._h, _p(f, C.c_int8))
        return f

    def set_particles(self, x, v=None, omega=None, q=None):
        x = np.ascontiguousarray(x, np.float64)
        n = x.shape[0]
        v = np.zeros((n, 3)) if v is None else np.ascontiguousarray(v, np.float64)
        om = None if omega is None else np.ascontiguousarray(omega, np.float64)
        q = None if q is None else np.ascontiguousarray(q, np.float64)
        D = C.c_double
        rc = self._L.orc_set_particles(self._h, n, _p(x, D), _p(v, D), _p(om, D), _p(q, D))
        if rc:
            raise RuntimeError(f"orc_set_particles {rc}")
        self.np = n

    def get_particles(self):
        n = self.np
        x, v, om = np.empty((n, 3)), np.empty((n, 3)), np.empty((n, 3))
        q, fo, to = np.empty((n, 4)), np.empty((n, 3)), np.empty((n, 3))
        D = C.c_double
        self._L.orc_get_particles(self._h, _p(x, D), _p(v, D), _p(om, D), _p(q, D), _p(fo, D), _p(to, D))
        return dict(x=x, v=v, omega=om, q=q, force=fo, torque=to)

    def get_rho(self):
        rR, rB = np.empty(self.shape), np.empty(self.shape)
        self._L.orc_get_rho(self._h, _p(rR, C.c_double), _p(rB, C.c_double))
        return rR, rB

    def record_links(self, on=True):
        """Record the bounce-back links of each particle step (off by default)."""
        self._L.orc_record_links(self._h, 1 if on else 0)

    def get_links(self):
        """Links of the last particle step: int32 (n, 3) rows (sphere, cell, direction), sorted."""
        n = C.c_int64()
        self._L.orc_get_links(self._h, None, None, None, 0, C.byref(n))
        m = n.value
        cell = np.empty(max(m, 1), np.int32)
        sph = np.empty(max(m, 1), np.int32)
        d = np.empty(max(m, 1), np.int8)
        self._L.orc_get_links(self._h, _p(cell, C.c_int32), _p(d, C.c_int8), _p(sph, C.c_int32), m, C.byref(n))
        return np.stack([sph[:m], cell[:m], d[:m].astype(np.int32)], axis=1)

    def template(self):
        rm = C.c_int()
        self._L.orc_template(self._h, C.byref(rm), None)
        w = 2 * rm.value + 1
        t = np.empty(w ** 3, np.int8)
        self._L.orc_template(self._h, C.byref(rm), _p(t, C.c_int8))
        return t.reshape(w, w, w)  # [k][j][i]

    def status(self):
        c, s, w = C.c_int(), C.c_int(), C.c_int64()
        self._L.orc_status(self._h, C.byref(c), C.byref(s), C.byref(w))
        return c.value, s.value, w.value
