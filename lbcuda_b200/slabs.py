"""z-slab decomposition of a periodic colour-gradient box.

The reference runs one MPI rank per z-slab and swaps halo planes of
populations between neighbouring ranks every step (main.CUF:504-1000;
rank layout setupMPI.CUF:26-30).  Here a slab is a context holding its own
planes plus HALO halo planes on each side (`lbx_set_zrange`): every step the
slabs first swap their boundary planes (`lbx_pack_planes` /
`lbx_unpack_planes`, packed device buffers), then each steps its own planes
on the single-pass kernel.  The step needs two halo planes: the phase field
of the plane next to the first own plane is summed from pulls that reach one
plane further.

Two transports move the packed planes:
  LocalExchange  several slabs in one process (device copies between their
                 contexts; one GPU can run a decomposed box this way),
  DistExchange   one slab per rank over torch.distributed: NCCL between GPUs
                 (NVLink / NVSwitch), gloo for host buffers.
Slab s sends its first HALO own planes to slab s - 1, which keeps them as its
upper halo, and its last HALO own planes to slab s + 1 (lower halo),
periodically.
"""
import copy

import numpy as np

from . import capi
from .sim import LBSim

HALO = 2


def own_planes(nz, nslabs):
    """Own planes per slab: nz split evenly (the reference requires the same)."""
    if nslabs < 1 or nz % nslabs:
        raise ValueError(f"nz = {nz} does not split into {nslabs} equal slabs")
    own = nz // nslabs
    if own < HALO:
        raise ValueError(f"a slab needs at least {HALO} own planes (has {own})")
    return own


class Slab:
    """Slab `index` of `nslabs` of the periodic box described by `params` (whole-box sizes)."""

    def __init__(self, params, index, nslabs):
        self.nz = int(params.nz)
        self.own = own_planes(self.nz, nslabs)
        self.index, self.nslabs = index, nslabs
        self.z0 = index * self.own  # first own plane in the whole box
        local = copy.copy(params)
        local.nz = self.own + 2 * HALO
        self.sim = LBSim(local)
        capi.check(self.sim._L.lbx_set_zrange(self.sim._h, HALO, HALO + self.own), "lbx_set_zrange")
        nb = capi.C.c_int64()
        capi.check(self.sim._L.lbx_plane_bytes(self.sim._h, HALO, capi.C.byref(nb)), "lbx_plane_bytes")
        self.halo_bytes = int(nb.value)

    # whole-box planes z0 - HALO .. z0 + own + HALO - 1 (periodic) of a field
    def _local(self, a):
        idx = (np.arange(self.z0 - HALO, self.z0 + self.own + HALO)) % self.nz
        return np.ascontiguousarray(np.asarray(a)[idx])

    def set_fields(self, rhoR, rhoB, vel=(0.0, 0.0, 0.0)):
        """Whole-box fields (nz, ny, nx); the halo planes are rewritten by the first exchange."""
        self.sim.set_fields(self._local(rhoR), self._local(rhoB), vel)

    # packed boundary planes: "low" = the first HALO own planes (sent down),
    # "high" = the last HALO own planes (sent up)
    def pack(self, which, buf):
        z = HALO if which == "low" else self.own
        capi.check(self.sim._L.lbx_pack_planes(self.sim._h, z, HALO, capi.C.c_void_p(buf.data_ptr())),
                   "lbx_pack_planes")

    # received halos: "low" = the planes below the own ones, "high" = above
    def unpack(self, which, buf):
        z = 0 if which == "low" else HALO + self.own
        capi.check(self.sim._L.lbx_unpack_planes(self.sim._h, z, HALO, capi.C.c_void_p(buf.data_ptr())),
                   "lbx_unpack_planes")

    def sync(self):
        self.sim.sync()

    @property
    def stream(self):
        """The context's CUDA stream, as a torch stream (packs, unpacks and steps are enqueued on it)."""
        import torch
        if getattr(self, "_stream", None) is None:
            ptr = capi.C.c_void_p()
            capi.check(self.sim._L.lbx_get_stream(self.sim._h, capi.C.byref(ptr)), "lbx_get_stream")
            self._stream = torch.cuda.ExternalStream(ptr.value or 0)
        return self._stream

    def step_own(self):
        self.sim.step(1)

    def own_fields(self):
        """(rhoR, rhoB, vel, phase) of the own planes."""
        f = self.sim.get_fields()
        return tuple(a[HALO:HALO + self.own] for a in f)

    def own_pops(self):
        pR, pB = self.sim.get_pops()
        return pR[:, HALO:HALO + self.own], pB[:, HALO:HALO + self.own]

    def close(self):
        self.sim.close()


class LocalExchange:
    """All slabs of a box in this process; packed planes move by device copies.

    Nothing waits on the host: slab i's stream records an event after its
    packs, and the two neighbours' streams wait on it before they unpack.  The
    buffers alternate between two sets, so a pack never overwrites a buffer a
    neighbour may not have unpacked yet (that unpack precedes, on the
    neighbour's stream, the pack this slab waited for one exchange later)."""

    def __init__(self, slabs):
        import torch
        self.slabs = slabs
        dev = torch.device("cuda", torch.cuda.current_device())
        mk = lambda s: torch.empty(s.halo_bytes, dtype=torch.uint8, device=dev)
        self.low = [[mk(s) for s in slabs] for _ in range(2)]
        self.high = [[mk(s) for s in slabs] for _ in range(2)]
        self.parity = 0

    def exchange(self):
        import torch
        n = len(self.slabs)
        lo, hi = self.low[self.parity], self.high[self.parity]
        self.parity ^= 1
        packed = []
        for i, s in enumerate(self.slabs):
            s.pack("low", lo[i])
            s.pack("high", hi[i])
            ev = torch.cuda.Event()
            ev.record(s.stream)
            packed.append(ev)
        for i, s in enumerate(self.slabs):
            up, down = (i + 1) % n, (i - 1) % n
            s.stream.wait_event(packed[up])
            s.stream.wait_event(packed[down])
            s.unpack("high", lo[up])  # the first own planes of the slab above
            s.unpack("low", hi[down])  # the last own planes of the slab below

    def step(self, nsteps=1):
        for _ in range(nsteps):
            self.exchange()
            for s in self.slabs:
                s.step_own()

    def sync(self):
        for s in self.slabs:
            s.sync()


class DistExchange:
    """One slab per rank of the default process group (rank r holds slab r).

    `slab` needs pack(which, tensor), unpack(which, tensor), sync() and
    halo_bytes; the buffers live on `device` (a CUDA device for NCCL, the CPU
    for gloo).  Every rank takes the same two sends and two receives per
    exchange, in the same order."""

    def __init__(self, slab, device):
        import torch
        import torch.distributed as dist
        self.dist = dist
        self.slab = slab
        self.rank, self.world = dist.get_rank(), dist.get_world_size()
        self.cuda = torch.device(device).type == "cuda"
        mk = lambda: torch.empty(slab.halo_bytes, dtype=torch.uint8, device=device)
        self.send_low, self.send_high, self.recv_low, self.recv_high = mk(), mk(), mk(), mk()

    def exchange(self):
        import torch
        s = self.slab
        if self.cuda:
            # every copy and transfer on the context's stream: the collectives
            # wait for the packs, the unpacks for the collectives
            with torch.cuda.stream(s.stream):
                self._swap()
        else:
            s.pack("low", self.send_low)
            s.pack("high", self.send_high)
            s.sync()
            self._swap(packed=True)
            s.sync()

    def _swap(self, packed=False):
        s = self.slab
        if not packed:
            s.pack("low", self.send_low)
            s.pack("high", self.send_high)
        if self.world == 1:  # periodic with itself
            self.recv_high.copy_(self.send_low)
            self.recv_low.copy_(self.send_high)
        else:
            d = self.dist
            down, up = (self.rank - 1) % self.world, (self.rank + 1) % self.world
            # tags keep the two messages between the same pair of ranks apart
            # (world size 2: down == up); NCCL matches them in issue order
            ops = [d.P2POp(d.isend, self.send_low, down, tag=1), d.P2POp(d.irecv, self.recv_high, up, tag=1),
                   d.P2POp(d.isend, self.send_high, up, tag=2), d.P2POp(d.irecv, self.recv_low, down, tag=2)]
            for w in d.batch_isend_irecv(ops):
                w.wait()
        s.unpack("high", self.recv_high)
        s.unpack("low", self.recv_low)

    def step(self, nsteps=1):
        for _ in range(nsteps):
            self.exchange()
            self.slab.step_own()
