"""Input side of the reference workflow, restated on the host.

* :func:`read_input_dat`  — the positional ``input.dat`` of readParameters
  (main.CUF:409-496), with the same validation and messages;
* :func:`read_namelist_input` — the namelist deck of the NEWINPUT build
  (groups &simulation, &fluid, &particle; main.CUF:341-345, 356-408), the
  only input that carries the two fluid densities densR / densB;
* :func:`read_input_xyz`  — ``input.xyz`` of read_input_atom
  (main.CUF:1230-1350), Euler angles -> quaternion by eul2q
  (main.CUF:1352-1370) with the reference's (eul1, eul3, eul2) argument order;
* :func:`initial_fields`  — the density fields of initType 1, 2, 3, 5, 6
  (setup2, setup2_zplanes, read_and_setRed_Blue, setupCyl,
  set_random_dens_fluids: kernels_fluid_CG.CUF:140-311, main.CUF:2444-2684);
* :func:`read_fortran_field` / :func:`write_fortran_field` — the
  Fortran-unformatted ``rhoR.init.bin`` layout (header record
  minx,maxx,miny,maxy,minz,maxz then one FP32 record, main.CUF:2448-2470);
* :func:`read_init_pops` / :func:`write_init_pops` — initType 4's
  per-direction population files ``popR.NNNNNN.init.bin`` /
  ``popB.NNNNNN.init.bin`` (read_and_setPops, main.CUF:2489-2529), the
  restart set of a run;
* :func:`seeded_noise_fields` — the seeded synthetic inputs that stand in for
  the reference's unseeded Fortran RNG.
"""
import math
import os

import numpy as np


class InputError(ValueError):
    pass


def _tokens(line):
    line = line.split("!")[0]
    return line.split()


def read_input_dat(path):
    """Parse input.dat exactly like readParameters (main.CUF:409-496).

    Returns a dict with nIter, nIterOut, nIterVTK, initType, vel, withParticles,
    numAtoms, ext_force, max_vel, lrotate, ext_torque.  Raises InputError with
    the reference's messages when a required line is missing.
    """
    with open(path) as fh:
        lines = [ln for ln in fh.read().splitlines()]
    it = iter(lines)
    out = dict(nIter=5, nIterOut=1, nIterVTK=100000000, initType=-1, vel=(0.0, 0.0, 0.0),
               withParticles=False, numAtoms=1, ext_force=(0.0, 0.0, 0.0), max_vel=0.0,
               lrotate=False, ext_torque=(0.0, 0.0, 0.0))
    found = 0
    max_vel_found = 0

    def nxt():
        for ln in it:
            t = _tokens(ln)
            if t:
                return t
        raise StopIteration

    try:
        out["nIter"] = int(nxt()[0]); found = 1
        out["nIterOut"] = int(nxt()[0]); found = 2
        out["nIterVTK"] = int(nxt()[0]); found = 3
        out["initType"] = int(nxt()[0]); found = 4
        t = nxt()
        out["vel"] = tuple(float(v) for v in t[:3]); found = 5
        t = nxt()
        out["numAtoms"] = int(t[1]) if len(t) > 1 else 1
        found = 6
        if t[0][:3] == "YES":
            out["withParticles"] = True
        elif t[0][:3] == "NO":
            out["withParticles"] = False
        else:
            found = 5
        if out["withParticles"]:
            out["ext_force"] = tuple(float(v) for v in nxt()[:3]); found = 7
            t = nxt()
            out["max_vel"] = float(t[1]) if len(t) > 1 else 0.0
            found = 8
            # the reference compares string(1:3) with a 16-character literal,
            # which never matches; it only lowers `found` (main.CUF:457-462)
            if t[0][:3] == "MAX_PARTICLE_VEL":
                max_vel_found = 1
            else:
                found = 7
            t = nxt()
            found = 9
            if t[0][:3] == "YES":
                out["lrotate"] = True
            elif t[0][:3] == "NO":
                out["lrotate"] = False
            else:
                found = 8
            if out["lrotate"]:
                out["ext_torque"] = tuple(float(v) for v in nxt()[:3]); found = 10
    except (StopIteration, IndexError, ValueError):
        pass
    wp, lr = out["withParticles"], out["lrotate"]
    # main.CUF:478-493 (with the MAX_PARTICLE_VEL quirk: found stays 7 after
    # that line, then reaches 9/10 on the following lines)
    if (lr and found != 10) or (not lr and wp and found != 9) or (not wp and found != 6):
        msgs = []
        if found < 1: msgs.append("Number of iterations not found")
        if found < 2: msgs.append("nIterOut not found")
        if found < 3: msgs.append("nIterVTK not found")
        if found < 4: msgs.append("initType not found")
        if found < 5: msgs.append("vx,vy,vz,densR,densB not found")
        if found < 6: msgs.append("withParticles not found")
        if wp and found < 7: msgs.append("ext_fxx,ext_fyy,ext_fzz not found")
        if wp and max_vel_found < 1: msgs.append("MAX_PARTICLE_VEL not found")
        if wp and found < 9: msgs.append("lrotate not found")
        if lr and found < 10: msgs.append("ext_tqx,ext_tqy,ext_tqz not found")
        raise InputError("; ".join(msgs) or "input.dat incomplete")
    return out


_NAMELIST_GROUPS = {
    "simulation": ("nIter", "nIterOut", "nIterVTK", "initType"),
    "fluid": ("vx", "vy", "vz", "densR", "densB", "tauR", "tauB"),
    "particle": ("withParticles", "numAtoms", "lrotate", "ext_fxx", "ext_fyy", "ext_fzz", "ext_tqx", "ext_tqy",
                 "ext_tqz", "max_vel"),
}


def _namelist_value(text):
    t = text.strip().rstrip(",").strip()
    low = t.lower()
    if low in (".true.", "t", ".t.", "true"):
        return True
    if low in (".false.", "f", ".f.", "false"):
        return False
    try:
        return int(t)
    except ValueError:
        return float(t.lower().replace("d", "e"))


def read_namelist_input(path):
    """Read the namelist deck of the NEWINPUT build (main.CUF:341-345, 356-408).

    The three groups are read in order (simulation, fluid, particle) with
    list-directed namelist syntax: ``&group``, ``name=value`` entries
    (several per line allowed, ``!`` comments), closed by ``/`` or ``&end``.
    Names are matched without regard to case, as Fortran does; a name that
    is not in its group raises InputError, as a namelist read fails.
    Returns one dict of every name given (values int, float or bool); names
    not given keep the caller's defaults (the reference initialises them
    before the read: main.CUF:346-354).
    """
    with open(path) as fh:
        text = fh.read()
    out = {}
    pos = 0
    low = text.lower()
    for group, names in _NAMELIST_GROUPS.items():
        start = low.find("&" + group, pos)
        if start < 0:
            raise InputError(f"namelist group &{group} not found in {path}")
        body_start = start + 1 + len(group)
        ends = [e for e in (low.find("&end", body_start), low.find("/", body_start)) if e >= 0]
        if not ends:
            raise InputError(f"namelist group &{group} is not closed")
        end = min(ends)
        body = "\n".join(line.split("!")[0] for line in text[body_start:end].splitlines())
        canon = {n.lower(): n for n in names}
        for item in body.replace(",", " ").split():
            if "=" not in item:
                continue
            key, _, val = item.partition("=")
            key = key.strip().lower()
            if key not in canon:
                raise InputError(f"{key} is not in namelist &{group}")
            out[canon[key]] = _namelist_value(val)
        pos = end
    return out


def eul2q(phis, psis, thetas):
    """eul2q (main.CUF:1352-1370) in FP32 like the reference."""
    f = np.float32
    h = f(0.5)
    cy, sy = np.cos(f(phis) * h), np.sin(f(phis) * h)
    cp, sp = np.cos(f(psis) * h), np.sin(f(psis) * h)
    cr, sr = np.cos(f(thetas) * h), np.sin(f(thetas) * h)
    return np.array([cy * cp * cr + sy * sp * sr,
                     cy * cp * sr - sy * sp * cr,
                     sy * cp * sr + cy * sp * cr,
                     sy * cp * cr - cy * sp * sr], dtype=np.float32)


def read_input_xyz(path, num_atoms, lrotate):
    """read_input_atom (main.CUF:1230-1350): positions, velocities, quaternions."""
    with open(path) as fh:
        first = fh.readline()
        n_file = int(first.split()[0])
        if n_file < num_atoms:
            raise InputError("Input file:input.xyz contains less particles than needed. STOP")
        fh.readline()  # format line
        x = np.zeros((num_atoms, 3))
        v = np.zeros((num_atoms, 3))
        q = np.zeros((num_atoms, 4))
        q[:, 0] = 1.0
        for i in range(num_atoms):
            t = fh.readline().split()
            x[i] = [float(a) for a in t[1:4]]
            v[i] = [float(a) for a in t[4:7]]
            if lrotate:
                e = [float(a) for a in t[7:10]]
                q[i] = eul2q(e[0], e[2], e[1])  # call eul2q(eul(1),eul(3),eul(2),q)
    return x, v, q


def check_particles(x, nx, ny, nz, rdim):
    """SetupParts sanity checks (main.CUF:1187-1227), in FP32 like the reference."""
    xs = x.astype(np.float32)
    for i, p in enumerate(xs):
        if p[0] < 1 or p[0] > nx or p[1] < 1 or p[1] > ny or p[2] < 1 or p[2] > nz:
            raise InputError(f"Particle #{i + 1} out of bounds {p}")
    lim = np.float32(2 * rdim + 1)
    for i in range(len(xs)):
        d = np.sqrt(((xs[i + 1:] - xs[i]) ** 2).sum(axis=1))
        bad = np.nonzero(d < lim)[0]
        if bad.size:
            j = i + 1 + bad[0]
            raise InputError(f"Dist less than 2*rdim+1 {i + 1} {j + 1} {d[bad[0]]:.4f} < {lim:.4f}")


def _fcut(r, r1, r2):
    """fcut (kernels_fluid_CG.CUF:126-138), elementwise in FP32."""
    f = np.float32
    out = np.where(r <= r1, f(1.0), np.where(r > r2, f(0.0),
                   f(0.5) * np.cos((r - f(r1)) * f(math.pi) / (f(r2) - f(r1))).astype(f) + f(0.5)))
    return out.astype(f)


def _grid(nx, ny, nz):
    k, j, i = np.meshgrid(np.arange(1, nz + 1), np.arange(1, ny + 1), np.arange(1, nx + 1), indexing="ij")
    return i.astype(np.float32), j.astype(np.float32), k.astype(np.float32)


def initial_fields(init_type, nx, ny, nz, seed=0, path=".", dens=None):
    """(rhoR, rhoB) of initType 1, 2, 3, 5, 6 as float32 (nz, ny, nx) arrays.

    dens = (densR, densB) for the two-density model: the droplet of initType
    1 then carries densR inside and densB outside (setup2 with DIFFDENS,
    kernels_fluid_CG.CUF:163-169); the other types ignore it, as there."""
    f = np.float32
    if init_type == 1:  # setup2: droplet of radius glz/8 at the centre
        i, j, k = _grid(nx, ny, nz)
        radius = f(nz // 8)
        dx = i - f(nx // 2 + 0.5)
        dy = j - f(ny // 2 + 0.5)
        dz = k - f(nz // 2 + 0.5)
        r = np.sqrt(dx * dx + dy * dy + dz * dz).astype(f)
        t = _fcut(r, radius, radius + f(0.1))
        if dens is not None:
            return (t * f(dens[0])).astype(f), ((f(1.0) - t) * f(dens[1])).astype(f)
        return t, (f(1.0) - t).astype(f)
    if init_type == 2:  # setup2_zplanes: blue between glz/8 and 5glz/8
        i, j, k = _grid(nx, ny, nz)
        blue = (nz * 1 // 8 < k) & (k < nz * 5 // 8)
        t = np.where(blue, f(0.0), f(1.0)).astype(f)
        return t, (f(1.0) - t).astype(f)
    if init_type in (3, 4):  # read_and_setRed_Blue (initType 4 reads them before its populations)
        rR = read_fortran_field(os.path.join(path, "rhoR.init.bin"), nx, ny, nz)
        rB = read_fortran_field(os.path.join(path, "rhoB.init.bin"), nx, ny, nz)
        return rR, rB
    if init_type == 5:  # setupCyl: cylinder along z
        i, j, k = _grid(nx, ny, nz)
        radius = f(nz // 8)
        dx = i - f(nx // 2 + 0.5)
        dy = j - f(ny // 2 + 0.5)
        r = np.sqrt(dx * dx + dy * dy).astype(f)
        t = _fcut(r, radius, radius + f(0.1))
        return t, (f(1.0) - t).astype(f)
    if init_type == 6:  # set_random_dens_fluids: rhoR = 0.5 + 1e-4 U[0,1), rhoB = 1 - rhoR
        rng = np.random.Generator(np.random.PCG64(seed))
        rR = (f(0.5) + f(1.0e-4) * rng.random((nz, ny, nx), dtype=np.float32)).astype(f)
        return rR, (f(1.0) - rR).astype(f)
    raise InputError(f"Wront init type= {init_type}")


def seeded_noise_fields(nx, ny, nz, mean=0.5, amp=0.01, seed=0, ncomp=2):
    """rho_k = mean + U(-amp, amp), independently per cell and component (float32).

    PCG64 from numpy with the given seed; the synthetic stand-in for the
    reference's random initial conditions.
    """
    rng = np.random.Generator(np.random.PCG64(seed))
    out = []
    for _ in range(ncomp):
        out.append((np.float32(mean) + rng.uniform(-amp, amp, size=(nz, ny, nx))).astype(np.float32))
    return out


def read_fortran_field(path, nx, ny, nz):
    """Fortran unformatted sequential file: [6 x int32 header] [nx*ny*nz float32]."""
    with open(path, "rb") as fh:
        data = fh.read()
    off = 0

    def record():
        nonlocal off
        n = int(np.frombuffer(data, np.int32, 1, off)[0])
        body = data[off + 4: off + 4 + n]
        tail = int(np.frombuffer(data, np.int32, 1, off + 4 + n)[0])
        if tail != n:
            raise InputError(f"{path}: corrupt record marker")
        off += 8 + n
        return body

    hdr = np.frombuffer(record(), np.int32)
    if tuple(hdr) != (1, nx, 1, ny, 1, nz):
        raise InputError(f"Wrong start file {path} {tuple(hdr)}")
    body = np.frombuffer(record(), np.float32)
    if body.size != nx * ny * nz:
        raise InputError(f"{path}: {body.size} values, expected {nx * ny * nz}")
    return body.reshape(nz, ny, nx).copy()


def write_fortran_field(path, a):
    nz, ny, nx = a.shape
    hdr = np.array([1, nx, 1, ny, 1, nz], np.int32).tobytes()
    body = np.ascontiguousarray(a, np.float32).tobytes()
    with open(path, "wb") as fh:
        for rec in (hdr, body):
            n = np.array([len(rec)], np.int32).tobytes()
            fh.write(n + rec + n)


def pops_file(comp, l):
    """File name of direction l of one component in the initType-4 set: popR.NNNNNN.init.bin
    (write_fmtnumb's six zero-padded digits, write_output.f90:858-875)."""
    return f"pop{'RB'[comp]}.{l:06d}.init.bin"


def read_init_pops(path, nx, ny, nz, q=19):
    """initType 4 (read_and_setPops, main.CUF:2489-2529): the q per-direction files of each
    component in `path`, as float32 (q, nz, ny, nx) arrays (popsR, popsB)."""
    return tuple(np.stack([read_fortran_field(os.path.join(path, pops_file(c, l)), nx, ny, nz) for l in range(q)])
                 for c in (0, 1))


def write_init_pops(path, popsR, popsB, rhoR=None, rhoB=None):
    """The initType-4 restart set: popR/popB.NNNNNN.init.bin per direction ((q, nz, ny, nx) arrays)
    and, when given, rhoR/rhoB.init.bin, which the reference reads alongside (read_and_setRed_Blue)."""
    os.makedirs(path, exist_ok=True)
    for c, pops in enumerate((popsR, popsB)):
        for l in range(pops.shape[0]):
            write_fortran_field(os.path.join(path, pops_file(c, l)), pops[l])
    if rhoR is not None:
        write_fortran_field(os.path.join(path, "rhoR.init.bin"), rhoR)
        write_fortran_field(os.path.join(path, "rhoB.init.bin"), rhoB)
