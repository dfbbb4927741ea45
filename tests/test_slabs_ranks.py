"""The halo exchange of the z-slab decomposition across ranks, on CPU: gloo, world size 2 and 3.

Each rank holds slab r of a ring; after one exchange its upper halo must hold the first HALO own planes of
slab r + 1 and its lower halo the last HALO own planes of slab r - 1 (periodic), exactly the planes the
GPU slabs swap through lbx_pack_planes / lbx_unpack_planes (the same DistExchange code runs there over
NCCL).  A stand-in slab keeps its planes in a numpy array of byte rows.
"""
import os
import sys

import numpy as np
import torch
import torch.distributed as dist
import torch.multiprocessing as mp

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))


class FakeSlab:
    """own + 2 HALO planes of `row` bytes each; own plane k of rank r holds the value 100 r + k."""

    def __init__(self, rank, own, halo, row=24):
        self.own, self.halo, self.row = own, halo, row
        self.planes = np.full((own + 2 * halo, row), 255, np.uint8)
        for k in range(own):
            self.planes[halo + k] = 100 * rank + k
        self.halo_bytes = halo * row

    def pack(self, which, buf):
        z = self.halo if which == "low" else self.own
        buf.copy_(torch.from_numpy(self.planes[z:z + self.halo].reshape(-1).copy()))

    def unpack(self, which, buf):
        z = 0 if which == "low" else self.halo + self.own
        self.planes[z:z + self.halo] = buf.numpy().reshape(self.halo, self.row)

    def sync(self):
        pass


def _worker(rank, world, port, out):
    sys.path.insert(0, ROOT)
    from lbcuda_b200.slabs import HALO, DistExchange
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        s = FakeSlab(rank, own=5, halo=HALO)
        ex = DistExchange(s, "cpu")
        ex.exchange()
        out[rank] = [int(v) for v in s.planes[:, 0]]
    finally:
        dist.destroy_process_group()


def _run(world, port):
    ctx = mp.get_context("spawn")
    with ctx.Manager() as m:
        out = m.dict()
        mp.start_processes(_worker, args=(world, port, out), nprocs=world, join=True, start_method="spawn")
        return dict(out)


def _expected(rank, world, own=5, halo=2):
    lo, hi = (rank - 1) % world, (rank + 1) % world
    below = [100 * lo + k for k in range(own - halo, own)]  # last own planes of the slab below
    mine = [100 * rank + k for k in range(own)]
    above = [100 * hi + k for k in range(halo)]  # first own planes of the slab above
    return below + mine + above


def test_ring_of_two():
    out = _run(2, 29531)
    assert out == {r: _expected(r, 2) for r in range(2)}


def test_ring_of_three():
    out = _run(3, 29533)
    assert out == {r: _expected(r, 3) for r in range(3)}
