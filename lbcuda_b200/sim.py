"""LBSim — the host-side object above the C ABI.

It plays the role of the reference's Fortran host for the hot path
(main.CUF:125-308): it owns one ``lbx`` context, sets the initial fields,
advances steps and reads moments back.  All arrays crossing the boundary are
numpy arrays in the reference's Fortran layout (x fastest): a field is
``(nz, ny, nx)`` in C order, populations ``(q, nz, ny, nx)`` (q = 19, or 27 for
the D3Q27 models).
"""
import ctypes as C

import numpy as np

from . import capi
from .capi import LbxParams, check

Q = 19


def make_params(nx, ny=None, nz=None, model="cg", storage="f32", **kw):
    """lbx_params with the reference defaults (lbx_default_params) overridden by kw."""
    ny = nx if ny is None else ny
    nz = nx if nz is None else nz
    p = LbxParams()
    capi.lib().lbx_default_params(C.byref(p), nx, ny, nz)
    p.model = capi.MODEL[model] if isinstance(model, str) else int(model)
    p.storage = capi.STORAGE[storage] if isinstance(storage, str) else int(storage)
    for k, v in kw.items():
        if k == "wetting" and isinstance(v, str):
            v = capi.WETTING[v]
        if k in ("ext_force", "ext_torque"):
            getattr(p, k)[:] = list(v)
            continue
        if not hasattr(p, k):
            raise KeyError(k)
        setattr(p, k, v)
    return p


def _fptr(a, ctype=C.c_float):
    return a.ctypes.data_as(C.POINTER(ctype)) if a is not None else None


class LBSim:
    """One simulation context on the current CUDA device."""

    def __init__(self, params):
        self.params = params
        self.nx, self.ny, self.nz = params.nx, params.ny, params.nz
        self.ncomp = 1 if params.model == capi.MODEL["bgk"] else 2
        self.q = 27 if params.model in (capi.MODEL["cg-d3q27"], capi.MODEL["cg-diffdens-d3q27"]) else Q
        self._L = capi.lib()
        h = C.c_void_p()
        check(self._L.lbx_create(C.byref(params), C.byref(h)), "lbx_create")
        self._h = h

    # -- lifetime ---------------------------------------------------------
    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            self._L.lbx_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    @property
    def shape(self):
        return (self.nz, self.ny, self.nx)

    # -- initial conditions ----------------------------------------------------
    def set_fields(self, rhoR, rhoB=None, vel=(0.0, 0.0, 0.0)):
        rR = np.ascontiguousarray(rhoR, dtype=np.float32).reshape(self.shape)
        rB = None if rhoB is None else np.ascontiguousarray(rhoB, dtype=np.float32).reshape(self.shape)
        check(self._L.lbx_set_fields(self._h, _fptr(rR), _fptr(rB), float(vel[0]), float(vel[1]), float(vel[2])),
              "lbx_set_fields")

    def set_pops(self, popsR, popsB=None):
        pR = np.ascontiguousarray(popsR, dtype=np.float32).reshape((self.q,) + self.shape)
        pB = None if popsB is None else np.ascontiguousarray(popsB, dtype=np.float32).reshape((self.q,) + self.shape)
        check(self._L.lbx_set_pops(self._h, _fptr(pR), _fptr(pB)), "lbx_set_pops")

    def set_particles(self, x, v=None, omega=None, q=None):
        x = np.ascontiguousarray(x, np.float64)
        n = x.shape[0]
        v = np.zeros((n, 3)) if v is None else np.ascontiguousarray(v, np.float64)
        om = None if omega is None else np.ascontiguousarray(omega, np.float64)
        q = None if q is None else np.ascontiguousarray(q, np.float64)
        D = C.c_double
        check(self._L.lbx_set_particles(self._h, n, _fptr(x, D), _fptr(v, D), _fptr(om, D), _fptr(q, D)),
              "lbx_set_particles")
        self.np = n

    def get_particles(self):
        n = self.np
        x, v, om = np.empty((n, 3)), np.empty((n, 3)), np.empty((n, 3))
        q, fo, to = np.empty((n, 4)), np.empty((n, 3)), np.empty((n, 3))
        D = C.c_double
        check(self._L.lbx_get_particles(self._h, _fptr(x, D), _fptr(v, D), _fptr(om, D), _fptr(q, D),
                                        _fptr(fo, D), _fptr(to, D)), "lbx_get_particles")
        return dict(x=x, v=v, omega=om, q=q, force=fo, torque=to)

    # -- stepping --------------------------------------------------------------
    def step(self, n=1):
        check(self._L.lbx_step(self._h, int(n)), "lbx_step")

    def sync(self):
        check(self._L.lbx_sync(self._h), "lbx_sync")

    def set_schedule(self, fused):
        """0 = two passes, 1 = first single-pass kernel, 2 = lean single-pass kernel (default)."""
        check(self._L.lbx_set_schedule(self._h, int(fused)), "lbx_set_schedule")

    def set_lean_shape(self, shape, zlen=0):
        check(self._L.lbx_set_lean_shape(self._h, int(shape), int(zlen)), "lbx_set_lean_shape")

    def set_lean_copies(self, mode):
        """16-bit pulls of the lean kernel: 1 = 16-byte box granules (default), 0 = one copy per pull."""
        check(self._L.lbx_set_lean_copies(self._h, int(mode)), "lbx_set_lean_copies")

    def time_steps(self, n, kernel_timing=True):
        """(total_ms, kernel_ms, kernel_launches) of n steps, CUDA events on the context stream."""
        t = C.c_double()
        k = C.c_double()
        nl = C.c_int64()
        check(self._L.lbx_time_steps(self._h, int(n), C.byref(t), C.byref(k) if kernel_timing else None,
                                     C.byref(nl)), "lbx_time_steps")
        return t.value, k.value, nl.value

    @property
    def steps_taken(self):
        s = C.c_int64()
        check(self._L.lbx_get_step(self._h, C.byref(s)))
        return s.value

    # -- readback ----------------------------------------------------------------
    def get_fields(self, f64=False):
        """moments2Fl: (rhoR, rhoB, vel[3], phase) of the post-streaming populations."""
        dt = np.float64 if f64 else np.float32
        ct = C.c_double if f64 else C.c_float
        rR = np.empty(self.shape, dt)
        rB = np.empty(self.shape, dt)
        vel = np.empty(self.shape + (3,), dt)
        ph = np.empty(self.shape, dt)
        fn = self._L.lbx_get_fields_f64 if f64 else self._L.lbx_get_fields
        check(fn(self._h, _fptr(rR, ct), _fptr(rB, ct), _fptr(vel, ct), _fptr(ph, ct)), "lbx_get_fields")
        return rR, rB, vel, ph

    def get_pops(self):
        pR = np.empty((self.q,) + self.shape, np.float32)
        pB = np.empty((self.q,) + self.shape, np.float32)
        check(self._L.lbx_get_pops(self._h, _fptr(pR), _fptr(pB)), "lbx_get_pops")
        return pR, (pB if self.ncomp == 2 else None)

    def get_flags(self):
        f = np.empty(self.shape, np.int8)
        check(self._L.lbx_get_flags(self._h, _fptr(f, C.c_int8)), "lbx_get_flags")
        return f

    def get_links(self):
        """Boundary links of the last step's bounce-back: int32 (n, 3) rows of
        (sphere, cell, direction), sorted (lbx_get_links)."""
        n = C.c_int64()
        check(self._L.lbx_get_links(self._h, None, None, None, 0, C.byref(n)), "lbx_get_links")
        m = n.value
        cell = np.empty(max(m, 1), np.int32)
        sph = np.empty(max(m, 1), np.int32)
        d = np.empty(max(m, 1), np.int8)
        check(self._L.lbx_get_links(self._h, _fptr(cell, C.c_int32), _fptr(d, C.c_int8), _fptr(sph, C.c_int32),
                                    m, C.byref(n)), "lbx_get_links")
        return np.stack([sph[:m], cell[:m], d[:m].astype(np.int32)], axis=1)

    def get_sums(self):
        m = np.zeros(2, np.float64)
        mom = np.zeros(3, np.float64)
        check(self._L.lbx_get_sums(self._h, _fptr(m, C.c_double), _fptr(mom, C.c_double)), "lbx_get_sums")
        return m, mom

    def status(self):
        code = C.c_int32()
        st = C.c_int32()
        wh = C.c_int64()
        check(self._L.lbx_status(self._h, C.byref(code), C.byref(st), C.byref(wh)), "lbx_status")
        return code.value, st.value, wh.value
