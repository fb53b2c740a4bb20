"""Adjoint of the time loop on the device (no reference counterpart).

* Dot-product test per operator (FP64): <y, Op(s)> = <Op^T y, s> for random
  states s and adjoints y over every entry of the 9 fields of both grids
  (halos and ghosts included), for the velocity update with its mirrors, the
  21-Cij stress update (free surface on and off) and the three interface
  solves, at refinement ratios 2 and 3.  Tolerance 1e-12 of sum |y Op(s)|
  (1e-10 for the iterative sxz solve, whose forward stops at the reference's
  tolerance).
* Medium gradient per operator: d<y, Op_m(s)>/dm against central finite
  differences along a random direction of the node buoyancy and the 21 slots
  (the stencils are linear in the medium, the solves rational).
* The checkpointed misfit gradient: against central differences of the
  device forward (FP64) and of the FP64 CPU oracle along random medium
  directions (1e-5 relative), independent of the checkpoint interval, and the
  FP32 gradient within 2e-3 of the FP64 one.
"""
import copy
import zlib

import numpy as np
import pytest

from ecsg_b200 import SIM_POS, Simulation, field_shape
from ecsg_b200.workloads import CIJ21_POS, random_case_gen21, ricker
from oracle.oracle import OracleRun

pytestmark = pytest.mark.gpu


def _case(seed, ratio, top_bc, mirror_fix=True, nz=(6, 5)):
    case = random_case_gen21(seed, ratio=ratio, nx2=6, ny2=5, nz=nz, top_bc=top_bc, aniso=0.3)
    case.mirror_fix = mirror_fix
    for m in case.media:
        m["buoy"] = m["buoy"].astype(np.float64)
    return case


def _rand_state(case, rng):
    return {(g, k): rng.standard_normal(field_shape(case.grids[g]["n"], SIM_POS[k], case.radius))
            for g in range(len(case.grids)) for k in range(9)}


def _dot(a, b):
    return sum(float(np.sum(a[key] * b[key])) for key in a)


def _absdot(a, b):
    return sum(float(np.sum(np.abs(a[key] * b[key]))) for key in a)


def _forward(sim, op, idx):
    getattr(sim, {"vel": "update_vel", "stress": "update_stress", "vz": "ghost_vz", "sxz": "ghost_sxz",
                  "syz": "ghost_syz"}[op])(idx)


def _apply(case, s, op, idx, prec="f64"):
    with Simulation(case, precision=prec) as sim:
        for (g, k), a in s.items():
            sim.set_field(g, k, a)
        _forward(sim, op, idx)
        return {(g, k): sim.field(g, k) for (g, k) in s}


def _adjoint(case, s, y, op, idx):
    """Op^T y and the medium gradient of <y, Op(s)>."""
    with Simulation(case, precision="f64") as sim:
        for (g, k), a in s.items():
            sim.set_field(g, k, a)
        _forward(sim, op, idx)
        sim.adjoint_reset()
        for (g, k), a in y.items():
            sim.set_adjoint_field(g, k, a)
        sim.adjoint_op(op, idx)
        z = {(g, k): sim.adjoint_field(g, k) for (g, k) in y}
        grads = [[sim.gradient(g, w) for w in range(22)] for g in range(len(case.grids))]
    return z, grads


def _perturbed(case, dirs, eps):
    c = copy.deepcopy(case)
    for g, m in enumerate(c.media):
        m["buoy"] = case.media[g]["buoy"] + eps * dirs[g][0]
        m["c21"] = [case.media[g]["c21"][k] + eps * dirs[g][1 + k] for k in range(21)]
    return c


def _directions(case, rng):
    dirs = []
    for g, m in enumerate(case.media):
        d = [m["buoy"] * rng.standard_normal(m["buoy"].shape)]
        scale = np.abs(m["c21"][0]).mean()
        d += [scale * rng.standard_normal(m["c21"][k].shape) for k in range(21)]
        dirs.append(d)
    return dirs


def _gdot(grads, dirs):
    return sum(float(np.sum(grads[g][w] * dirs[g][w])) for g in range(len(dirs)) for w in range(22))


OPS = [("vel", 0), ("vel", 1), ("stress", 0), ("stress", 1), ("vz", 1), ("sxz", 1), ("syz", 1)]


@pytest.mark.parametrize("ratio,top_bc,mirror_fix", [(2, 1, True), (3, 0, False), (3, 1, True)])
@pytest.mark.parametrize("op,idx", OPS)
def test_operator_dot_product_and_medium_gradient(op, idx, ratio, top_bc, mirror_fix):
    case = _case(31 + ratio, ratio, top_bc, mirror_fix)
    rng = np.random.default_rng(zlib.crc32(repr((op, idx, ratio, top_bc)).encode()))
    s, y = _rand_state(case, rng), _rand_state(case, rng)
    out = _apply(case, s, op, idx)
    z, grads = _adjoint(case, s, y, op, idx)
    lhs, rhs = _dot(y, out), _dot(z, s)
    tol = (1e-10 if op == "sxz" else 1e-12) * _absdot(y, out)
    assert abs(lhs - rhs) <= tol, (lhs, rhs)
    # medium gradient along a random direction
    dirs = _directions(case, rng)
    eps = 1e-4
    fp = _dot(y, _apply(_perturbed(case, dirs, eps), s, op, idx))
    fm = _dot(y, _apply(_perturbed(case, dirs, -eps), s, op, idx))
    fd = (fp - fm) / (2 * eps)
    an = _gdot(grads, dirs)
    assert abs(fd - an) <= 1e-6 * max(abs(fd), 1e-3 * _absdot(y, out)), (fd, an)


def _loop_case(seed=7, ratio=2, top_bc=1, nsteps=30):
    case = _case(seed, ratio, top_bc, True, nz=(6, 5))
    h, n = case.grids[0]["h"], case.grids[0]["n"]
    case.src = {"xyz": (n[0] // 2 * h[0], n[1] // 2 * h[1], 2 * h[2]), "trace": ricker(nsteps, case.dt * 1e-3 * 2.0, 15.0),
                "scale": 1000.0, "comp": 0}
    case.rec = np.array([[(n[0] // 2 + 2) * h[0], n[1] // 2 * h[1], 1 * h[2]],
                         [(n[0] // 3) * h[0], (n[1] // 3) * h[1], (n[2] - 1) * h[2]],
                         [(n[0] // 2) * h[0], (n[1] // 2) * h[1], (n[2] + 3) * h[2]]], dtype=np.float32)
    case.rec_comp = 0
    return case


def _loss(case, obs, prec="f64"):
    with Simulation(case, precision=prec) as sim:
        return sim.misfit_gradient(obs, ckpt_every=obs.shape[0])


def _oracle_loss(case, obs):
    rec = OracleRun(case).run(obs.shape[0])["rec"]      # (n_rec, nsteps), FP64
    return 0.5 * float(np.sum((rec.T - obs.astype(np.float64)) ** 2))


@pytest.mark.parametrize("ratio,top_bc", [(2, 1), (3, 0)])
def test_misfit_gradient_matches_finite_differences(ratio, top_bc):
    nsteps = 30
    case = _loop_case(11 + ratio, ratio, top_bc, nsteps)
    rng = np.random.default_rng(ratio)
    obs = (0.1 * rng.standard_normal((nsteps, len(case.rec)))).astype(np.float32)
    with Simulation(case, precision="f64") as sim:
        loss = sim.misfit_gradient(obs, ckpt_every=7)
        grads = [[sim.gradient(g, w) for w in range(22)] for g in range(2)]
    assert np.isfinite(loss) and loss > 0
    assert abs(_oracle_loss(case, obs) - loss) <= 1e-10 * loss
    for trial in range(2):
        dirs = _directions(case, rng)
        eps = 1e-4
        an = _gdot(grads, dirs)
        fd_dev = (_loss(_perturbed(case, dirs, eps), obs) - _loss(_perturbed(case, dirs, -eps), obs)) / (2 * eps)
        fd_cpu = (_oracle_loss(_perturbed(case, dirs, eps), obs) - _oracle_loss(_perturbed(case, dirs, -eps), obs)) / (2 * eps)
        assert abs(fd_dev - an) <= 1e-5 * abs(fd_dev), (trial, fd_dev, an)
        assert abs(fd_cpu - an) <= 1e-5 * abs(fd_cpu), (trial, fd_cpu, an)


def test_gradient_independent_of_checkpoint_interval_and_fp32_close():
    nsteps = 24
    case = _loop_case(5, 3, 1, nsteps)
    obs = np.zeros((nsteps, len(case.rec)), np.float32)
    res = []
    for prec, k in (("f64", 1), ("f64", 5), ("f64", 24), ("f32", 5)):
        with Simulation(case, precision=prec) as sim:
            loss = sim.misfit_gradient(obs, ckpt_every=k)
            res.append((loss, [sim.gradient(g, w) for g in range(2) for w in range(22)]))
            # the fields are left at the final forward state
            final = sim.field(0, 0)
        if prec == "f64" and k == 5:
            with Simulation(case, precision="f64") as ref:
                ref.run(nsteps, graph=False)
                assert np.abs(final - ref.field(0, 0)).max() <= 1e-12 * np.abs(final).max()
    (l0, g0) = res[0]
    for l1, g1 in res[1:3]:
        assert abs(l1 - l0) <= 1e-13 * l0
        for a, b in zip(g0, g1):
            assert np.abs(a - b).max() <= 1e-10 * max(np.abs(a).max(), 1e-300)
    l32, g32 = res[3]
    assert abs(l32 - l0) <= 1e-4 * l0
    num = sum(float(np.sum((a - b) ** 2)) for a, b in zip(g0, g32))
    den = sum(float(np.sum(a ** 2)) for a in g0)
    assert np.sqrt(num / den) <= 2e-3


def test_torch_autograd_function_returns_the_device_gradient():
    torch = pytest.importorskip("torch")
    from ecsg_b200.autograd import misfit
    nsteps = 16
    case = _loop_case(9, 2, 1, nsteps)
    obs = np.zeros((nsteps, len(case.rec)), np.float32)
    medium = [[torch.tensor(m["buoy"], dtype=torch.float64, requires_grad=True)]
              + [torch.tensor(c, dtype=torch.float64, requires_grad=True) for c in m["c21"]] for m in case.media]
    loss = misfit(case, obs, medium, ckpt_every=4)
    loss.backward()
    with Simulation(case, precision="f64") as sim:
        ref = sim.misfit_gradient(obs, ckpt_every=4)
        want = [[sim.gradient(g, w) for w in range(22)] for g in range(2)]
    assert abs(loss.item() - ref) <= 1e-13 * ref
    for g in range(2):
        for w in range(22):
            got = medium[g][w].grad.numpy()
            assert np.abs(got - want[g][w]).max() <= 1e-10 * max(np.abs(want[g][w]).max(), 1e-300)


def test_misfit_loss_is_the_same_on_every_run():
    """The loss over many receiver samples (blocks of the residual kernel
    summed in a fixed order): identical on repeated runs, and equal to the sum
    of the squared device residuals to round-off."""
    nsteps = 40
    case = _loop_case(13, 2, 1, nsteps)
    h, n = case.grids[0]["h"], case.grids[0]["n"]
    xs, ys = np.meshgrid(np.arange(1, n[0] - 1), np.arange(1, n[1] - 1), indexing="ij")
    case.rec = np.stack([xs.ravel() * h[0], ys.ravel() * h[1], np.full(xs.size, 1 * h[2])], axis=1).astype(np.float32)
    obs = (1e-3 * np.random.default_rng(5).standard_normal((nsteps, len(case.rec)))).astype(np.float32)
    assert obs.size > 256 * 8
    losses = []
    for _ in range(3):
        with Simulation(case, precision="f32") as sim:
            losses.append(sim.misfit_gradient(obs, ckpt_every=10))
    assert losses[0] == losses[1] == losses[2], losses
    with Simulation(case, precision="f32") as sim:
        rec = sim.run(nsteps)["rec"].astype(np.float64)
    want = 0.5 * float(np.sum((rec.T - obs.astype(np.float64)) ** 2))
    assert abs(losses[0] - want) <= 1e-5 * abs(want), (losses[0], want)
