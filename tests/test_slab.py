"""z slabs (one box split over GPUs): the split and the halo exchange
between ranks, on CPU ranks (gloo) with host buffers.  The device side is
compared with the whole box in test_gpu_slab.py."""
import os
import socket
import tempfile

import pytest
import torch
import torch.multiprocessing as mp

from hydropad_b200.slab import exchange_p2p, slab_bounds


def test_slab_bounds():
    assert slab_bounds(64, 1) == [(0, 64)]
    assert slab_bounds(64, 4) == [(0, 16), (16, 16), (32, 16), (48, 16)]
    assert slab_bounds(30, 4) == [(0, 8), (8, 8), (16, 7), (23, 7)]
    with pytest.raises(ValueError):
        slab_bounds(15, 4)


def _free_port():
    s = socket.socket()
    s.bind(("127.0.0.1", 0))
    p = s.getsockname()[1]
    s.close()
    return p


def _rank(rank, world, port, out):
    import torch.distributed as dist
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        plane = 6
        top4 = torch.full((5 * 4 * plane,), 100.0 + rank, dtype=torch.float64)
        bottom3 = torch.full((5 * 3 * plane,), 200.0 + rank, dtype=torch.float64)
        lower4 = torch.zeros(5 * 4 * plane, dtype=torch.float64)
        upper3 = torch.zeros(5 * 3 * plane, dtype=torch.float64)
        exchange_p2p(top4, bottom3, lower4, upper3, rank, world)
        ok = bool((lower4 == 100.0 + (rank - 1) % world).all()) and bool((upper3 == 200.0 + (rank + 1) % world).all())
        torch.save(ok, os.path.join(out, f"{rank}.pt"))
    finally:
        dist.destroy_process_group()


@pytest.mark.parametrize("world", [2, 3])
def test_halo_exchange_gloo(world):
    """Each rank's lower halo is the top of the rank below, its upper halo
    the bottom of the rank above, periodically (two ranks: the same peer)."""
    with tempfile.TemporaryDirectory() as d:
        mp.start_processes(_rank, args=(world, _free_port(), d), nprocs=world, join=True, start_method="spawn")
        assert all(torch.load(os.path.join(d, f"{r}.pt")) for r in range(world))


def test_halo_exchange_single_rank_is_periodic():
    top4, bottom3 = torch.arange(8.0), torch.arange(6.0)
    lower4, upper3 = torch.zeros(8), torch.zeros(6)
    exchange_p2p(top4, bottom3, lower4, upper3, 0, 1)
    assert torch.equal(lower4, top4) and torch.equal(upper3, bottom3)
