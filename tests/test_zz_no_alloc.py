"""lbx_closure_infer_noalloc against lbx_closure_infer (GPU).

The no-allocation entry point stages its data in a fixed device array, so two
calls in a row must each give exactly the results of the allocating entry
point (same kernel, same launch shape), and sizes beyond the array are
rejected before any device work.  Collected last; passes alone as well.
"""
import ctypes as C

import numpy as np
import pytest

from lbcuda_b200 import capi
from lbcuda_b200.closure import DIN, DOUT, NPARAM, NW

pytestmark = pytest.mark.gpu

NMAX = 4096


def _fp(a):
    return a.ctypes.data_as(C.POINTER(C.c_float))


def _weights(seed):
    w = np.zeros(NW, np.float32)                                  # LBX_CLOSURE_NWEIGHTS
    assert capi.lib().lbx_closure_init(_fp(w), seed) == 0
    rng = np.random.default_rng(seed)
    npar = NPARAM
    w[npar:npar + DIN] = rng.normal(0, 0.5, DIN)                  # feature means
    w[npar + DIN:npar + 2 * DIN] = rng.uniform(0.5, 2.0, DIN)     # feature scales
    w[npar + 2 * DIN:npar + 2 * DIN + DOUT] = rng.normal(0, 0.1, DOUT)
    w[npar + 2 * DIN + DOUT:] = rng.uniform(0.5, 2.0, DOUT)
    return w


def _infer(name, w, X):
    Y = np.full((X.shape[0], DOUT), np.nan, np.float32)
    rc = getattr(capi.lib(), name)(_fp(w), _fp(X), X.shape[0], _fp(Y))
    return rc, Y


def test_two_calls_in_a_row_match_the_allocating_entry_point():
    rng = np.random.default_rng(11)
    cases = [(_weights(1), rng.normal(size=(NMAX, DIN)).astype(np.float32)),   # the full capacity
             (_weights(2), rng.normal(size=(37, DIN)).astype(np.float32))]     # then a short call
    got = []
    for w, X in cases:
        rc, Y = _infer("lbx_closure_infer_noalloc", w, X)
        assert rc == 0
        got.append(Y)
    for (w, X), Y in zip(cases, got):
        rc, ref = _infer("lbx_closure_infer", w, X)
        assert rc == 0
        assert np.isfinite(ref).all()
        assert np.array_equal(Y, ref)


def test_calls_leave_free_device_memory_unchanged():
    """After one warm-up call (module load, first lookup) the entry point must
    not allocate: the device's free memory stays the same over more calls."""
    import torch
    w = _weights(4)
    X = np.random.default_rng(4).normal(size=(NMAX, DIN)).astype(np.float32)
    rc, _ = _infer("lbx_closure_infer_noalloc", w, X)
    assert rc == 0
    torch.cuda.synchronize()
    free0 = torch.cuda.mem_get_info()[0]
    for n in (NMAX, 1, 513, NMAX):
        rc, Y = _infer("lbx_closure_infer_noalloc", w, X[:n])
        assert rc == 0 and np.isfinite(Y).all()
    torch.cuda.synchronize()
    assert torch.cuda.mem_get_info()[0] == free0


def test_sizes_beyond_the_scratch_are_rejected():
    w = _weights(3)
    X = np.zeros((NMAX + 1, DIN), np.float32)
    rc, Y = _infer("lbx_closure_infer_noalloc", w, X)
    assert rc == -2                      # LBX_ERR_ARG
    assert np.isnan(Y).all()             # nothing written back
    rc, _ = _infer("lbx_closure_infer_noalloc", w, X[:0])
    assert rc == -2
