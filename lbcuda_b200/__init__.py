"""lbcuda_b200 — B200-native LBcuda hot path.

The compute lives in ``liblbx.so`` (hand-written sm_100a CUDA behind the C ABI
of ``include/lbx.h``); this package is the host side above that ABI:

* :mod:`lbcuda_b200.capi`   — ctypes binding of every ``lbx_*`` entry point;
* :mod:`lbcuda_b200.sim`    — :class:`LBSim`, the step-loop object a driver uses;
* :mod:`lbcuda_b200.inputs` — ``input.dat`` / ``input.xyz`` readers, initial
  fields of initType 1..6 and the Fortran-unformatted ``*.init.bin`` format.

The library is loaded eagerly on first use and a missing or unloadable
``liblbx.so`` raises immediately: there is no CPU fallback.
"""
from .capi import LBXError, lib, lib_path, LbxParams  # noqa: F401
from .sim import LBSim, make_params  # noqa: F401

__all__ = ["LBSim", "make_params", "LbxParams", "LBXError", "lib", "lib_path"]
