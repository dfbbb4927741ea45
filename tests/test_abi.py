"""The C-ABI library loads and exports every symbol include/lbx.h declares.

No compute call here: these run without a GPU.
"""
import ctypes

from lbcuda_b200 import capi


def test_header_symbols_exported():
    syms = capi.header_symbols()
    assert len(syms) >= 20
    lib = ctypes.CDLL(capi.lib_path())
    missing = [s for s in syms if not hasattr(lib, s)]
    assert not missing, missing


def test_binding_covers_header():
    syms = set(capi.header_symbols())
    bound = set(capi.SIGNATURES)
    assert syms <= bound, sorted(syms - bound)


def test_default_params_and_error_strings():
    L = capi.lib()
    p = capi.LbxParams()
    L.lbx_default_params(ctypes.byref(p), 64, 32, 16)
    assert (p.nx, p.ny, p.nz) == (64, 32, 16)
    assert abs(p.sigma - 0.1) < 1e-7 and abs(p.beta - 0.999) < 1e-7  # dimensions_m.CUF:50
    assert abs(p.radius - 5.5) < 1e-7 and abs(p.rmass - 1 / 1500) < 1e-9
    assert L.lbx_error_string(1).startswith(b"density")
    assert L.lbx_error_string(-2) == b"invalid argument"


def test_invalid_arguments_rejected_without_gpu():
    L = capi.lib()
    p = capi.LbxParams()
    L.lbx_default_params(ctypes.byref(p), 2, 2, 2)  # below the 3-cell minimum
    h = ctypes.c_void_p()
    assert L.lbx_create(ctypes.byref(p), ctypes.byref(h)) == -2
    assert L.lbx_step(None, 1) == -2
    assert L.lbx_destroy(None) == -2
    for name in ("lbx_make_list_atoms", "lbx_init_isfluid", "lbx_del_fluid", "lbx_make_fluid", "lbx_virtual_rho",
                 "lbx_partbb", "lbx_partbb_p2n", "lbx_partbb_p2n2", "lbx_inter_force_particles",
                 "lbx_time_step_force_particles"):
        assert getattr(L, name)(None) == -2, name
    n = ctypes.c_int64(-1)
    assert L.lbx_get_links(None, None, None, None, 0, ctypes.byref(n)) == -2
