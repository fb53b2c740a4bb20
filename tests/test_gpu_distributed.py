"""The device side of the gradient sum: the FP64 pack holds the volumes of
ecsg_get_gradient back to back, unpack writes a buffer back, and the NCCL
all-reduce on the library's stream leaves a one-rank gradient unchanged."""
import os
import socket

import numpy as np
import pytest
import torch

from ecsg_b200 import Simulation
from ecsg_b200.workloads import random_case_gen21, ricker

pytestmark = pytest.mark.gpu


def _sim_with_gradient(prec):
    nsteps = 12
    case = random_case_gen21(5, ratio=2, nx2=6, ny2=5, nz=(6, 5), aniso=0.3)
    for m in case.media:
        m["buoy"] = m["buoy"].astype(np.float64)
    n, h = case.grids[0]["n"], case.grids[0]["h"]
    case.src = {"xyz": (n[0] // 2 * h[0], n[1] // 2 * h[1], 2 * h[2]), "trace": ricker(nsteps, case.dt * 1e-3, 15.0),
                "scale": 1000.0, "comp": 0}
    case.rec = np.array([[(n[0] // 2 + 2) * h[0], n[1] // 2 * h[1], h[2]]], dtype=np.float32)
    s = Simulation(case, precision=prec)
    s.misfit_gradient(np.full((nsteps, 1), 0.01, np.float32), ckpt_every=4)
    return s


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_pack_unpack_and_one_rank_allreduce(prec):
    import torch.distributed as dist
    from ecsg_b200.distributed import allreduce_gradients
    s = _sim_with_gradient(prec)
    try:
        want = [np.concatenate([s.gradient(g, w).ravel() for w in range(22)]) for g in range(2)]
        assert all(np.abs(w).max() > 0 for w in want)
        dev = torch.device("cuda", 0)
        for g in range(2):
            buf = torch.empty(s.gradient_elems(g), dtype=torch.float64, device=dev)
            s.pack_gradient(g, buf.data_ptr())
            torch.cuda.synchronize()
            assert np.array_equal(buf.cpu().numpy(), want[g])
            buf *= 2.0
            torch.cuda.synchronize()
            s.unpack_gradient(g, buf.data_ptr())
            torch.cuda.synchronize()
            got = np.concatenate([s.gradient(g, w).ravel() for w in range(22)])
            assert np.array_equal(got, 2.0 * want[g])
        with socket.socket() as sk:
            sk.bind(("127.0.0.1", 0))
            port = sk.getsockname()[1]
        os.environ.update(MASTER_ADDR="127.0.0.1", MASTER_PORT=str(port))
        dist.init_process_group("nccl", rank=0, world_size=1)
        try:
            allreduce_gradients(s)
        finally:
            dist.destroy_process_group()
        for g in range(2):
            got = np.concatenate([s.gradient(g, w).ravel() for w in range(22)])
            assert np.array_equal(got, 2.0 * want[g])
    finally:
        s.close()
