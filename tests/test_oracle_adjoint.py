"""The FP64 CPU adjoint (oracle/adjoint_ad.cpp: reverse-mode differentiation
of the oracle's own time loop) against central differences of the oracle's
forward (oracle.py's OracleRun), before it is used to check the device
gradients.  No reference counterpart: the reference has no adjoint.

* its loss equals the oracle's forward misfit (the minimum Jacobi sweeps that
  make its solves exact move the loss by rounding only);
* d L / d m along seeded random directions of the node buoyancy and all 21
  slots of both grids matches central differences of the oracle forward to
  1e-6 relative (the differences' own truncation error is ~1e-8 at eps 1e-4),
  at ratios 2 (free surface) and 3 (rigid top).
"""
import copy

import numpy as np
import pytest

from ecsg_b200.workloads import random_case_gen21, ricker
from oracle.adjoint import misfit_gradient
from oracle.oracle import OracleRun


def loop_case(seed, ratio, top_bc, nsteps):
    case = random_case_gen21(seed, ratio=ratio, nx2=6, ny2=5, nz=(6, 5), top_bc=top_bc, aniso=0.3)
    case.mirror_fix = True
    for m in case.media:
        m["buoy"] = m["buoy"].astype(np.float64)
    h, n = case.grids[0]["h"], case.grids[0]["n"]
    case.src = {"xyz": (n[0] // 2 * h[0], n[1] // 2 * h[1], 2 * h[2]),
                "trace": ricker(nsteps, case.dt * 1e-3 * 2.0, 15.0), "scale": 1000.0, "comp": 0}
    case.rec = np.array([[(n[0] // 2 + 2) * h[0], n[1] // 2 * h[1], 1 * h[2]],
                         [(n[0] // 3) * h[0], (n[1] // 3) * h[1], (n[2] - 1) * h[2]],
                         [(n[0] // 2) * h[0], (n[1] // 2) * h[1], (n[2] + 3) * h[2]]], dtype=np.float32)
    case.rec_comp = 0
    return case


def oracle_loss(case, obs):
    rec = OracleRun(case).run(obs.shape[0])["rec"]      # receivers sample vx (rec_comp 0)
    return 0.5 * float(np.sum((rec.T - obs.astype(np.float64)) ** 2))


def perturbed(case, dirs, eps):
    c = copy.deepcopy(case)
    for g, m in enumerate(c.media):
        m["buoy"] = case.media[g]["buoy"] + eps * dirs[g][0]
        m["c21"] = [case.media[g]["c21"][k] + eps * dirs[g][1 + k] for k in range(21)]
    return c


def directions(case, rng):
    dirs = []
    for m in case.media:
        d = [m["buoy"] * rng.standard_normal(m["buoy"].shape)]
        scale = np.abs(m["c21"][0]).mean()
        d += [scale * rng.standard_normal(m["c21"][k].shape) for k in range(21)]
        dirs.append(d)
    return dirs


def gdot(grads, dirs):
    return sum(float(np.sum(grads[g][w] * dirs[g][w])) for g in range(len(dirs)) for w in range(22))


@pytest.mark.parametrize("ratio,top_bc", [(2, 1), (3, 0)])
def test_cpu_adjoint_matches_oracle_finite_differences(ratio, top_bc):
    nsteps = 30
    case = loop_case(11 + ratio, ratio, top_bc, nsteps)
    rng = np.random.default_rng(ratio)
    obs = (0.1 * rng.standard_normal((nsteps, len(case.rec)))).astype(np.float32)
    loss, grads, _ = misfit_gradient(case, obs)
    assert abs(loss - oracle_loss(case, obs)) <= 1e-13 * loss
    for _ in range(2):
        dirs = directions(case, rng)
        eps = 1e-4
        fd = (oracle_loss(perturbed(case, dirs, eps), obs) - oracle_loss(perturbed(case, dirs, -eps), obs)) / (2 * eps)
        an = gdot(grads, dirs)
        assert abs(fd - an) <= 1e-6 * abs(fd), (fd, an)
