"""The input.dat workflow end to end: the command-line host lbx_run.

lbx_run reads a deck with the rules of readParameters (main.CUF:409-496),
steps through the C ABI, prints the reference's Mlup/s line every nIterOut
steps (main.CUF:284-289) and writes VTK image data (writeImageDataVTI,
write_output.f90:115-392) and particle VTK (writeParticleVTK,
write_output.f90:674-746) every nIterVTK steps.  These tests run it on the
reference's own decks (run lengths shortened), read its files back and compare
them with LBSim stepped through the same library on the same input: the same
kernels in the same order, so the fields agree bit for bit.  The restart path
is initType 4 (read_and_setPops, main.CUF:2489-2529): population files written
from one run start another, which must continue the first exactly.
"""
import os
import re
import subprocess

import numpy as np
import pytest

from lbcuda_b200 import LBSim, make_params
from lbcuda_b200.build import DRIVER
from lbcuda_b200.inputs import initial_fields, read_init_pops, read_input_xyz, write_init_pops

pytestmark = pytest.mark.gpu

DECKS = os.path.join(os.path.dirname(__file__), "golden", "decks")
LINE = re.compile(r"^Iter:\s*(\d+)\s+Time\(s\):\s*\S+\s+ms/it:\s*\S+\s+Mlup/s:\s*(\d+)\.?\s*$")


def deck_with(src, dst, n_iter, n_out, n_vtk, init_type=None, n_atoms=None):
    """A copy of a reference deck with the run lengths (and optionally initType / numAtoms) replaced."""
    lines = open(src).read().splitlines()
    vals = [n_iter, n_out, n_vtk]
    for k in range(3):
        lines[k] = f"{vals[k]}\t" + lines[k].split(None, 1)[1] if len(lines[k].split(None, 1)) > 1 else str(vals[k])
    if init_type is not None:
        lines[3] = f"{init_type}\t! init TYPE"
    if n_atoms is not None:
        lines[5] = f"YES {n_atoms}\t! with PARTICLES"
    with open(dst, "w") as fh:
        fh.write("\n".join(lines) + "\n")


def read_vti(path):
    """(dict name -> float32 array (nz, ny, nx[, 3]), extent) of a raw appended VTI file."""
    data = open(path, "rb").read()
    head, _, tail = data.partition(b"<AppendedData encoding=\"raw\">")
    xml = head.decode()
    ext = [int(v) for v in re.search(r'WholeExtent="([^"]+)"', xml).group(1).split()]
    nx, ny, nz = ext[1] - ext[0] + 1, ext[3] - ext[2] + 1, ext[5] - ext[4] + 1
    blob = tail[tail.index(b"_") + 1:]
    out = {}
    for m in re.finditer(r'<DataArray type="Float32" Name="(\w+)" NumberOfComponents="(\d)" format="appended" '
                         r'offset="(\d+)"', xml):
        name, nc, off = m.group(1), int(m.group(2)), int(m.group(3))
        size = int(np.frombuffer(blob, np.uint64, 1, off)[0])
        a = np.frombuffer(blob, np.float32, size // 4, off + 8)
        out[name] = a.reshape((nz, ny, nx, nc) if nc > 1 else (nz, ny, nx))
    return out, (nx, ny, nz)


def read_particle_vtk(path):
    lines = open(path).read().splitlines()
    n = int(lines[4].split()[1])
    x = np.array([[float(t) for t in ln.split()] for ln in lines[5:5 + n]])
    v = np.array([[float(t) for t in ln.split()] for ln in lines[7 + n:7 + 2 * n]])
    return x, v


def run_driver(cwd, args):
    r = subprocess.run([DRIVER] + args, cwd=cwd, capture_output=True, text=True, timeout=300)
    assert r.returncode == 0, r.stderr
    return [ln for ln in r.stdout.splitlines() if ln.startswith("Iter:")]


def test_droplet_deck(tmp_path):
    """Tests/01 (CG droplet, initType 1, flow 0.05) on 32^3: 20 steps, print every 10, VTK at 20."""
    n = 32
    deck_with(os.path.join(DECKS, "01.input.dat"), tmp_path / "input.dat", 20, 10, 20)
    out = run_driver(tmp_path, ["-L", str(n), "--out", "out", "input.dat"])
    assert len(out) == 2
    for k, ln in zip((10, 20), out):
        m = LINE.match(ln)
        assert m, ln
        assert int(m.group(1)) == k and int(m.group(2)) > 0
    f, ext = read_vti(tmp_path / "out" / "rho_0.00000020.vti")
    assert ext == (n, n, n)
    s = LBSim(make_params(n, model="cg", storage="f32"))
    rR, rB = initial_fields(1, n, n, n)
    s.set_fields(rR, rB, (0.05, 0.05, 0.05))
    s.step(20)
    gR, gB, gV, gP = s.get_fields()
    assert np.array_equal(f["rhoR"], gR) and np.array_equal(f["rhoB"], gB)
    assert np.array_equal(f["vel"], gV) and np.array_equal(f["phase"], gP)


def test_particle_deck(tmp_path):
    """Tests/07-1280-Particle's deck (rotation, MAX_PARTICLE_VEL) with 16 spheres of its placement in a
    128^3 box: particle VTK and fluid VTI after 6 steps against LBSim."""
    n = 128
    x, v, q = read_input_xyz(os.path.join(DECKS, "07-1280.input.xyz.256cube.r5.5"), 1280, True)
    # spheres of the placement inside [7, n - 7)^3: no periodic image of one
    # comes near another in the n^3 box
    keep = np.nonzero(((x >= 7) & (x < n - 7)).all(axis=1))[0][:16]
    k = len(keep)
    assert k == 16
    src = open(os.path.join(DECKS, "07-1280.input.xyz.256cube.r5.5")).read().splitlines()
    with open(tmp_path / "input.xyz", "w") as fh:
        fh.write("\n".join([str(k), src[1]] + [src[2 + i] for i in keep]) + "\n")
    deck_with(os.path.join(DECKS, "07-1280-Particle.input.dat"), tmp_path / "input.dat", 6, 3, 6, n_atoms=k)
    out = run_driver(tmp_path, ["-L", str(n), "--out", "out", "input.dat"])
    assert len(out) == 2 and all(LINE.match(ln) for ln in out)
    px, pv = read_particle_vtk(tmp_path / "out" / "particle_0.00000006.vtk")
    f, _ = read_vti(tmp_path / "out" / "rho_0.00000006.vti")
    p = make_params(n, model="cg", storage="f32", max_particles=k, lrotate=1, max_vel=1.75)
    s = LBSim(p)
    rR, rB = initial_fields(1, n, n, n)
    s.set_fields(rR, rB)
    s.set_particles(x[keep], v[keep], None, q[keep])
    s.step(6)
    d = s.get_particles()
    # the deck's Euler angles become quaternions in FP32 on both sides (eul2q,
    # main.CUF:1352-1370), by C's and numpy's cosf / sinf, which may differ in
    # the last bit; positions are printed with %g (6 significant digits)
    assert np.allclose(px, d["x"], rtol=0, atol=1e-4 * n)
    assert np.allclose(pv, d["v"], rtol=1e-4, atol=1e-9)
    gR, gB, gV, gP = s.get_fields()
    assert np.abs(f["rhoR"] - gR).max() <= 1e-5 * np.abs(gR).max()
    assert np.linalg.norm(f["vel"] - gV) <= 1e-5 * np.linalg.norm(gV)


def test_init_type_4_restart(tmp_path):
    """A run writes the initType-4 restart set; a second run started from it (initType 4) continues the
    first exactly: its VTI after 10 more steps equals LBSim run 20 steps straight."""
    n = 32
    a, b = tmp_path / "a", tmp_path / "b"
    a.mkdir()
    b.mkdir()
    deck_with(os.path.join(DECKS, "01.input.dat"), a / "input.dat", 10, 10, 10)
    run_driver(a, ["-L", str(n), "--out", "out", "--restart-out", str(b), "input.dat"])
    pR, pB = read_init_pops(str(b), n, n, n)
    s = LBSim(make_params(n, model="cg", storage="f32"))
    rR, rB = initial_fields(1, n, n, n)
    s.set_fields(rR, rB, (0.05, 0.05, 0.05))
    s.step(10)
    gR, gB = s.get_pops()
    assert np.array_equal(pR, gR) and np.array_equal(pB, gB)
    deck_with(os.path.join(DECKS, "01.input.dat"), b / "input.dat", 10, 10, 10, init_type=4)
    run_driver(b, ["-L", str(n), "--out", "out", "input.dat"])
    f, _ = read_vti(b / "out" / "rho_0.00000010.vti")
    s.step(10)
    gR, gB, gV, gP = s.get_fields()
    assert np.array_equal(f["rhoR"], gR) and np.array_equal(f["rhoB"], gB) and np.array_equal(f["vel"], gV)


def test_init_type_4_from_python_writer(tmp_path):
    """Population files written by the host-side writer start lbx_run exactly where LBSim.set_pops starts."""
    n = 24
    rng = np.random.default_rng(3)
    w = np.array([1 / 3] + [1 / 18] * 6 + [1 / 36] * 12, np.float32)[:, None, None, None]
    pR = (w * (0.5 + 0.01 * rng.uniform(-1, 1, (19, n, n, n)))).astype(np.float32)
    pB = (w * (0.5 + 0.01 * rng.uniform(-1, 1, (19, n, n, n)))).astype(np.float32)
    write_init_pops(str(tmp_path), pR, pB, pR.sum(0), pB.sum(0))
    deck_with(os.path.join(DECKS, "01.input.dat"), tmp_path / "input.dat", 5, 5, 5, init_type=4)
    run_driver(tmp_path, ["-L", str(n), "--out", "out", "input.dat"])
    f, _ = read_vti(tmp_path / "out" / "rho_0.00000005.vti")
    s = LBSim(make_params(n, model="cg", storage="f32"))
    s.set_pops(pR, pB)
    s.step(5)
    gR, gB, gV, gP = s.get_fields()
    assert np.array_equal(f["rhoR"], gR) and np.array_equal(f["phase"], gP)
