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
* Against the FP64 CPU adjoint (oracle/adjoint_ad.cpp, reverse-mode
  differentiation of the oracle's own loop): the device FP64 gradient equals
  it element by element to 1e-10 of the gradient's scale, on random 21-Cij
  composites (ratio 2 and 3, free surface and rigid top) and on a reduced
  copy of the shot-gradient workload (10 m over 30 m at ratio 3, smooth
  orthorhombic model, vz source and surface vz receivers, observed data from
  the same model with a 3 % vs blob).
* Central differences along 20 seeded random directions of the buoyancy and
  all 21 slots: the FP64 device gradient within 1e-6, the FP32 device
  gradient within 1e-3 (both relative to the difference quotient, which is
  taken on the FP64 CPU oracle's forward with its interface solves converged
  to rounding).
"""
import copy
import ctypes
import zlib

import numpy as np
import pytest

from ecsg_b200 import SIM_POS, Simulation, field_shape
from ecsg_b200.workloads import CIJ21_POS, random_case_gen21, ricker, tti_as_gen21, two_grid_adjoint_case
from oracle.adjoint import misfit_gradient as cpu_adjoint
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


def _assert_equal_to_cpu_adjoint(g_dev, g_cpu, tol=1e-10):
    """Element by element, relative to the largest gradient entry of the grid
    (the slots' gradients differ by orders of magnitude between positions),
    but to no less than 1e-3 of the largest entry of all grids (a grid the
    wavefield has barely reached has a gradient many orders below the
    others, whose last bits are noise of the grids' coupling)."""
    top = max(float(np.abs(a).max()) for gg in g_cpu for a in gg)
    for g in range(len(g_cpu)):
        scale = max(max(float(np.abs(a).max()) for a in g_cpu[g]), 1e-3 * top)
        assert scale > 0
        for w in range(22):
            err = float(np.abs(g_dev[g][w] - g_cpu[g][w]).max())
            assert err <= tol * scale, (g, w, err / scale)


@pytest.mark.parametrize("ratio,top_bc", [(2, 1), (3, 0), (3, 1)])
def test_device_gradient_equals_fp64_cpu_adjoint(ratio, top_bc):
    nsteps = 30
    case = _loop_case(21 + ratio, ratio, top_bc, nsteps)
    rng = np.random.default_rng(100 + ratio)
    obs = (0.1 * rng.standard_normal((nsteps, len(case.rec)))).astype(np.float32)
    loss_cpu, g_cpu, _ = cpu_adjoint(case, obs)
    with Simulation(case, precision="f64") as sim:
        loss = sim.misfit_gradient(obs, ckpt_every=7)
        g_dev = [[sim.gradient(g, w) for w in range(22)] for g in range(2)]
    assert abs(loss - loss_cpu) <= 1e-12 * loss
    _assert_equal_to_cpu_adjoint(g_dev, g_cpu)


def _reduced_shot_case(nsteps):
    """The shot-gradient workload's set-up at a reduced size: 19 x 19 x 11
    points at 10 m over 7 x 7 x 9 at 30 m (ratio 3), the smooth orthorhombic
    model, shot 5 of the 4 x 4 grid (vz force), surface vz receivers every
    third fine node; observed data from the blob model with the blob scaled
    into this volume (3 % vs, radius 40 m at 60 m depth)."""
    grids = [((18, 18, 10), 10.0), ((6, 6, 8), 30.0)]
    kw = dict(grids=grids, fpeak=40.0)
    case = tti_as_gen21(two_grid_adjoint_case(0, 5, nsteps, blob=False, **kw))
    truth = tti_as_gen21(two_grid_adjoint_case(0, 5, nsteps, blob=True, blob_depth=60.0, blob_radius=40.0, **kw))
    with Simulation(truth, precision="f64") as sim:
        obs = sim.run(nsteps, graph=False)["rec"].T.copy()
    return case, obs


def test_reduced_shot_workload_gradient_equals_cpu_adjoint():
    nsteps = 40
    case, obs = _reduced_shot_case(nsteps)
    loss_cpu, g_cpu, _ = cpu_adjoint(case, obs)
    assert loss_cpu > 0
    with Simulation(case, precision="f64") as sim:
        loss = sim.misfit_gradient(obs, ckpt_every=10)
        g_dev = [[sim.gradient(g, w) for w in range(22)] for g in range(2)]
    assert abs(loss - loss_cpu) <= 1e-12 * loss
    _assert_equal_to_cpu_adjoint(g_dev, g_cpu)


def _converged_oracle_loss(case, obs):
    """The misfit of the FP64 CPU oracle with every sxz Jacobi solve run to
    rounding (at least 200 sweeps).  The device forward and the oracle stop at
    the reference's tolerance, so their misfit moves by that tolerance when a
    medium perturbation changes a sweep count; central differences of it are
    then no check of a derivative.  With the solves converged the misfit is the
    smooth function of the medium whose gradient the adjoint computes."""
    from oracle.oracle import lib as olib
    flag = ctypes.c_int.in_dll(olib(), "o_jacobi_min_sweeps")
    flag.value = 200
    try:
        return _oracle_loss(case, obs)
    finally:
        flag.value = 0


@pytest.mark.parametrize("which", ["random", "reduced_shot"])
def test_gradients_on_twenty_directions(which):
    """FP64 within 1e-6 and FP32 within 1e-3 of central differences of the
    FP64 oracle forward with converged interface solves, on 20 seeded
    directions."""
    nsteps = 30 if which == "random" else 40
    if which == "random":
        case = _loop_case(41, 3, 1, nsteps)
        obs = (0.1 * np.random.default_rng(41).standard_normal((nsteps, len(case.rec)))).astype(np.float32)
    else:
        case, obs = _reduced_shot_case(nsteps)
    grads = {}
    for prec in ("f64", "f32"):
        with Simulation(case, precision=prec) as sim:
            sim.misfit_gradient(obs, ckpt_every=10)
            grads[prec] = [[sim.gradient(g, w) for w in range(22)] for g in range(2)]
    rng = np.random.default_rng(2024)
    worst = {"f64": 0.0, "f32": 0.0}
    for trial in range(20):
        dirs = _directions(case, rng)
        eps = 1e-6   # the quotient's truncation error is ~eps^2: 1e-4 leaves 1e-4 of it on the blob data
        fd = (_converged_oracle_loss(_perturbed(case, dirs, eps), obs)
              - _converged_oracle_loss(_perturbed(case, dirs, -eps), obs)) / (2 * eps)
        for prec in ("f64", "f32"):
            worst[prec] = max(worst[prec], abs(_gdot(grads[prec], dirs) - fd) / abs(fd))
    assert worst["f64"] <= 1e-6, worst
    assert worst["f32"] <= 1e-3, worst
