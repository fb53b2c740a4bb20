"""The multi-process gradient sum (ecsg_b200/distributed.py) on CPU ranks
(gloo, world size 2 and 3): every rank ends with the FP64 sum of all ranks'
gradient volumes, per grid, in the pack order, whatever each rank held."""
import ctypes
import os
import socket

import numpy as np
import pytest
import torch
import torch.distributed as dist
import torch.multiprocessing as mp


class HostGradients:
    """Stands in for a Simulation: the 22 volumes of each grid in host memory,
    packed and unpacked through raw pointers like the device calls."""

    def __init__(self, rank, sizes):
        self.ng = len(sizes)
        rng = np.random.default_rng(100 + rank)
        self.vols = [[rng.standard_normal(n) for n in grid] for grid in sizes]

    def gradient_elems(self, g):
        return sum(v.size for v in self.vols[g])

    def pack_gradient(self, g, ptr):
        out = np.ctypeslib.as_array((ctypes.c_double * self.gradient_elems(g)).from_address(ptr))
        out[:] = np.concatenate(self.vols[g])

    def unpack_gradient(self, g, ptr):
        src = np.ctypeslib.as_array((ctypes.c_double * self.gradient_elems(g)).from_address(ptr))
        off = 0
        for v in self.vols[g]:
            v[:] = src[off:off + v.size]
            off += v.size


SIZES = [[7 * (w + 1) for w in range(22)], [5 + w for w in range(22)]]


def _worker(rank, world, port, q):
    os.environ["MASTER_ADDR"] = "127.0.0.1"
    os.environ["MASTER_PORT"] = str(port)
    dist.init_process_group("gloo", rank=rank, world_size=world)
    try:
        from ecsg_b200.distributed import reduce_gradients_on
        sim = HostGradients(rank, SIZES)
        reduce_gradients_on(sim, None, "cpu")
        q.put((rank, [[v.copy() for v in grid] for grid in sim.vols]))
    finally:
        dist.destroy_process_group()


def _free_port():
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


@pytest.mark.parametrize("world", [2, 3])
def test_every_rank_gets_the_fp64_sum(world):
    ctx = mp.get_context("spawn")
    q = ctx.Queue()
    port = _free_port()
    procs = [ctx.Process(target=_worker, args=(r, world, port, q)) for r in range(world)]
    for p in procs:
        p.start()
    results = dict(q.get(timeout=120) for _ in range(world))
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    want = [[sum(HostGradients(r, SIZES).vols[g][w] for r in range(world)) for w in range(22)] for g in range(2)]
    for r in range(world):
        for g in range(2):
            for w in range(22):
                assert np.allclose(results[r][g][w], want[g][w], rtol=1e-15, atol=1e-15)
