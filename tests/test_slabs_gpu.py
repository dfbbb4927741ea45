"""z-slab decomposition on one GPU: a box split into slabs, stepped with halo exchanges between the slabs'
contexts, equals the same box stepped whole, bit for bit.

Every cell's update depends only on the populations it pulls and on the phase field of its D3Q27
neighbourhood, so a slab whose two halo planes on each side hold its neighbours' boundary planes of the
last step computes exactly the whole box's values (the reference's MPI slabs, main.CUF:504-1000, keep the
same invariant).  One slab exchanges with itself (the periodic box); three slabs exchange around a ring.
"""
import numpy as np
import pytest

from lbcuda_b200 import LBSim, capi, make_params
from lbcuda_b200.inputs import seeded_noise_fields
from lbcuda_b200.slabs import HALO, LocalExchange, Slab

pytestmark = pytest.mark.gpu

LBX_ERR_ARG, LBX_ERR_STATE = -2, -4  # include/lbx.h


@pytest.mark.parametrize("storage", ["f32", "f16", "f16sd", "f16sdp", "bf16sd"])
@pytest.mark.parametrize("nslabs", [1, 3])
def test_slabs_equal_whole_box(storage, nslabs):
    nx, ny, nz, steps = 32, 24, 48, 12
    p = make_params(nx, ny, nz, model="cg", storage=storage, sigma=0.02, beta=0.7)
    rR, rB = seeded_noise_fields(nx, ny, nz, seed=4)
    whole = LBSim(p)
    whole.set_fields(rR, rB)
    whole.step(steps)
    ref_pops, ref_fields = whole.get_pops(), whole.get_fields()
    assert whole.status()[0] == 0
    whole.close()
    slabs = [Slab(p, i, nslabs) for i in range(nslabs)]
    for s in slabs:
        s.set_fields(rR, rB)
    ex = LocalExchange(slabs)
    ex.step(steps)
    ex.exchange()  # the readback pulls from the halo planes too
    for s in slabs:
        assert s.sim.status()[0] == 0
        z = slice(s.z0, s.z0 + s.own)
        for a, b in zip(s.own_pops(), ref_pops):
            assert np.array_equal(a, b[:, z])
        for a, b in zip(s.own_fields(), ref_fields):
            assert np.array_equal(a, b[z])
        s.close()


def test_zrange_arguments():
    """The own planes need two halo planes on each side; spheres and the other schedules are refused."""
    p = make_params(32, 24, 20, model="cg", storage="f16sd")
    g = LBSim(p)
    L = capi.lib()
    assert L.lbx_set_zrange(g._h, 1, 18) == LBX_ERR_ARG
    assert L.lbx_set_zrange(g._h, 2, 19) == LBX_ERR_ARG
    assert L.lbx_set_zrange(g._h, 5, 5) == LBX_ERR_ARG
    assert L.lbx_set_zrange(g._h, HALO, 20 - HALO) == 0
    assert L.lbx_set_schedule(g._h, 0) != 0
    assert L.lbx_set_zrange(g._h, 0, 0) == 0
    g.close()
    q = LBSim(make_params(32, 24, 24, model="cg", storage="f16", max_particles=1, radius=3.0))
    assert L.lbx_set_zrange(q._h, 2, 22) == LBX_ERR_STATE
    q.close()


def test_dist_exchange_single_rank_equals_whole_box():
    """DistExchange (the per-rank transport) with a process group of one: the slab exchanges with itself on
    its context's stream, and the periodic box comes out as stepped whole."""
    import os
    import socket

    import torch.distributed as dist

    from lbcuda_b200.slabs import DistExchange
    with socket.socket() as so:
        so.bind(("127.0.0.1", 0))
        port = so.getsockname()[1]
    os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
    dist.init_process_group("gloo", rank=0, world_size=1)
    try:
        nx, ny, nz, steps = 32, 16, 24, 9
        p = make_params(nx, ny, nz, model="cg", storage="f16sd", sigma=0.02, beta=0.7)
        rR, rB = seeded_noise_fields(nx, ny, nz, seed=8)
        whole = LBSim(p)
        whole.set_fields(rR, rB)
        whole.step(steps)
        ref = whole.get_pops()
        whole.close()
        s = Slab(p, 0, 1)
        s.set_fields(rR, rB)
        ex = DistExchange(s, "cuda")
        ex.step(steps)
        ex.exchange()
        for a, b in zip(s.own_pops(), ref):
            assert np.array_equal(a, b)
        s.close()
    finally:
        dist.destroy_process_group()
