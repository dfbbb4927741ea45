"""Ensemble of uneven boxes advanced together (lbx_ensemble_*).

Each box is an ordinary context (an :class:`LBSim` view), so fields, spheres
and the closure are set and read box by box; ``step`` advances all boxes with
one persistent fluid kernel per step under a captured CUDA graph.
"""
import ctypes as C

import numpy as np

from . import capi
from .capi import LbxParams, check
from .sim import LBSim


class _BoxView(LBSim):
    """LBSim over a context owned by the ensemble (never destroyed by the view)."""

    def __init__(self, params, handle):  # noqa: D401 - no lbx_create here
        self.params = params
        self.nx, self.ny, self.nz = params.nx, params.ny, params.nz
        self.ncomp = 2
        self._L = capi.lib()
        self._h = handle

    def close(self):
        self._h = C.c_void_p()


class Ensemble:
    def __init__(self, params_list):
        self._L = capi.lib()
        arr = (LbxParams * len(params_list))(*params_list)
        h = C.c_void_p()
        check(self._L.lbx_ensemble_create(len(params_list), arr, C.byref(h)), "lbx_ensemble_create")
        self._h = h
        self.boxes = []
        for i, p in enumerate(params_list):
            bh = C.c_void_p()
            check(self._L.lbx_ensemble_box(self._h, i, C.byref(bh)), "lbx_ensemble_box")
            self.boxes.append(_BoxView(p, bh))

    def step(self, n=1):
        check(self._L.lbx_ensemble_step(self._h, int(n)), "lbx_ensemble_step")

    def time(self, n):
        ms = C.c_double()
        check(self._L.lbx_ensemble_time(self._h, int(n), C.byref(ms)), "lbx_ensemble_time")
        return ms.value

    def tune(self, trial=10):
        ch = (C.c_int32 * 2)()
        best = C.c_double()
        check(self._L.lbx_ensemble_tune(self._h, int(trial), ch, C.byref(best)), "lbx_ensemble_tune")
        return {"shape": "32x16" if ch[0] == 1 else "32x8", "zlen": int(ch[1]), "fused_kernel_ms": best.value}

    def close(self):
        if getattr(self, "_h", None) and self._h.value:
            for b in self.boxes:
                b.close()
            self._L.lbx_ensemble_destroy(self._h)
            self._h = C.c_void_p()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    @property
    def cells(self):
        return int(sum(b.nx * b.ny * b.nz for b in self.boxes))


def random_boxes(nbox=48, seed=0, edges=(32, 48, 64, 96), max_spheres=40, radius=4.0):
    """Box edges uniform from `edges`, 0..max_spheres spheres of `radius` placed without overlap (min gap 1)."""
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(nbox):
        L = int(rng.choice(edges))
        n_target = int(rng.integers(0, max_spheres + 1))
        xs = []
        tries = 0
        while len(xs) < n_target and tries < 20000:
            tries += 1
            x = rng.uniform(0.5, L + 0.5, 3)
            ok = True
            for y in xs:
                d = x - y
                d -= L * np.round(d / L)
                if np.linalg.norm(d) < 2 * radius + 1.0:
                    ok = False
                    break
            if ok:
                xs.append(x)
        out.append((L, np.array(xs).reshape(-1, 3)))
    return out
