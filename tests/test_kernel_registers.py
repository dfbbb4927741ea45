"""The single-pass fluid kernels compile without register spills.

A spill in these kernels lands in the per-direction loops and their local
memory loads sit on the critical path: one of 8 bytes in the FP32 particle
variant once doubled its time (1.24 -> 2.67 ms per colloid step at 256^3).
The check compiles lbx_fused.cu with ptxas statistics (no GPU needed).
FP64 storage is exempt: its kernels run one CTA per SM at up to 255
registers and are not performance paths.
"""
import os
import re
import shutil
import subprocess

import pytest

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)


def test_lean_kernels_do_not_spill(tmp_path):
    from lbcuda_b200 import build as B
    nvcc = B.nvcc()
    if not (os.path.isabs(nvcc) and os.path.exists(nvcc)) and shutil.which(nvcc) is None:
        pytest.skip("nvcc not available")
    src = os.path.join(B.CSRC, "lbx_fused.cu")
    cmd = [nvcc] + B.NVCC_FLAGS + B.FILE_FLAGS.get("lbx_fused.cu", []) + ["-Xptxas", "-v", "-c", src, "-o",
                                                                          str(tmp_path / "f.o")]
    p = subprocess.run(cmd, capture_output=True, text=True)
    assert p.returncode == 0, p.stderr[-2000:]
    lines = p.stderr.splitlines()
    cur = None
    checked = 0
    bad = []
    for line in lines:
        m = re.search(r"Compiling entry function '(\S+)'", line)
        if m:
            cur = m.group(1)
            continue
        m = re.search(r"(\d+) bytes spill stores, (\d+) bytes spill loads", line)
        if m and cur and "k_cg_lean" in cur:
            if "IdLi" in cur:  # FP64 storage instantiations
                continue
            checked += 1
            if int(m.group(1)) or int(m.group(2)):
                bad.append((cur, m.group(1), m.group(2)))
    assert checked >= 8, "no k_cg_lean instantiations found in the ptxas output"
    assert not bad, f"register spills in single-pass kernels: {bad}"
