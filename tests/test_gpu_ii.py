"""Intuitive interpolation (imode 0) on the device against the oracle and the
reference itself.

* Each interface op, FP64: bitwise equal to the oracle over every entry of the
  9 fields of both grids (halos and ghosts included), on shapes where the far
  vz column reads past the coarse rows differently.
* Each op, FP32: bitwise equal to the reference's float build
  (oracle/_ref/libecsg_ref32.so), whose float and double sub-expressions the
  kernels reproduce.
* The time loop against the oracle (FP64 exact to round-off, FP32 1e-5).
* The reference's II golden traces (tests/golden/rec_ii_test{1,2,3}): full
  1172-step runs within 5e-5 rel-L2 with the golden-producing variant
  (ii_skip_end_column), as for the ECI goldens.
* Adjoints: dot-product tests of the three transposes and a misfit gradient
  against central differences.
"""
import copy
import os

import numpy as np
import pytest

from ecsg_b200 import SIM_POS, Simulation, field_shape
from ecsg_b200.workloads import eci_test_case, random_case, random_case_gen21, ricker
from oracle.oracle import OracleRun

pytestmark = pytest.mark.gpu
GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")
OPS = ("ghost_vz", "ghost_sxz", "ghost_syz")


def _ii(case, skip_end=False):
    case.imode = 0
    case.ii_skip_end_column = skip_end
    return case


def _fields(o):
    return [(g, k) for g in range(len(o.levels)) for k in range(9)]


@pytest.mark.parametrize("skip_end", [False, True])
@pytest.mark.parametrize("seed,nx2,ny2", [(1, 6, 5), (2, 3, 7), (3, 2, 2), (5, 33, 9)])
def test_ops_f64_bitwise_vs_oracle(seed, nx2, ny2, skip_end):
    case = _ii(random_case(seed, ratio=2, nx2=nx2, ny2=ny2, nz=(5, 4)), skip_end)
    o = OracleRun(case)
    rng = np.random.default_rng(seed)
    with Simulation(case, precision="f64") as s:
        for op in OPS:
            for g, k in _fields(o):
                a = rng.standard_normal(o.levels[g]["f"][k].shape)
                o.levels[g]["f"][k][...] = a
                s.set_field(g, k, a)
            getattr(o, op)(1)
            getattr(s, op)(1)
            for g, k in _fields(o):
                assert np.array_equal(o.levels[g]["f"][k], s.field(g, k)), (op, g, k)


@pytest.mark.parametrize("seed,nx2,ny2", [(1, 6, 5), (2, 3, 7), (5, 33, 9)])
def test_ops_f32_bitwise_vs_reference_float_build(seed, nx2, ny2):
    from oracle.ref import RefRun, available
    if not available(32):
        pytest.skip("reference float build (oracle/_ref/libecsg_ref32.so) absent")
    case = _ii(random_case(seed, ratio=2, nx2=nx2, ny2=ny2, nz=(5, 4)))
    r = RefRun(case, threads=2, bits=32)
    rng = np.random.default_rng(100 + seed)
    try:
        with Simulation(case, precision="f32") as s:
            for op in OPS:
                for g in range(2):
                    for k in range(9):
                        a = rng.standard_normal(r.shape(g, 0, k)[0]).astype(np.float32).astype(np.float64)
                        r.set(g, k, a)
                        s.set_field(g, k, a)
                getattr(r, op)(1)
                getattr(s, op)(1)
                for g in range(2):
                    for k in range(9):
                        assert np.array_equal(r.get(g, k), s.field(g, k)), (op, g, k)
    finally:
        r.close()


def _with_src_rec(case, nt):
    h, n = case.grids[0]["h"], case.grids[0]["n"]
    case.src = {"xyz": (n[0] // 2 * h[0], n[1] // 2 * h[1], 2 * h[2]), "trace": ricker(nt, case.dt * 1e-3 * 0.5, 15.0),
                "scale": 1000.0, "comp": 0}
    case.rec = np.array([[(n[0] // 2 + 3) * h[0], n[1] // 2 * h[1], 2 * h[2]],
                         [(n[0] - 1) * h[0], (n[1] // 3) * h[1], (n[2] - 1) * h[2]],
                         [(n[0] // 2) * h[0], (n[1] // 2) * h[1], (n[2] + 2) * h[2]]], dtype=np.float32)
    return case


@pytest.mark.parametrize("medium", ["iso", "gen21"])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_time_loop_vs_oracle(prec, medium):
    nsteps = 80
    if medium == "iso":
        case = random_case(41, ratio=2, nx2=9, ny2=8, nz=(8, 6))
    else:
        case = random_case_gen21(42, ratio=2, nx2=9, ny2=8, nz=(8, 6), aniso=0.3)
    case = _with_src_rec(_ii(case), nsteps)
    ref = OracleRun(case, energy=True).run(nsteps)
    with Simulation(case, precision=prec, energy=True) as s:
        out = s.run(nsteps, energy_every=1, graph=(prec == "f32"))
        assert s.status() == 0
    rel = np.linalg.norm(out["rec"] - ref["rec"], axis=1) / np.linalg.norm(ref["rec"], axis=1)
    erel = np.abs(out["energy"] - ref["energy"]).max() / np.abs(ref["energy"]).max()
    if prec == "f64":
        assert rel.max() < 1e-7 and erel < 1e-10, (rel, erel)   # traces are stored as float32
    else:
        assert rel.max() < 1e-5 and erel < 1e-5, (rel, erel)


@pytest.mark.parametrize("test", [1, 2, 3])
def test_reference_ii_golden_traces(test):
    """Full 1172-step II experiments of the reference's test suite, FP32 on the
    device, against its golden receiver traces."""
    case = _ii(eci_test_case(test, imode=0), skip_end=True)
    gold = np.load(os.path.join(GOLDEN, "rec_ii_test%d.npy" % test))
    with Simulation(case, precision="f32") as s:
        out = s.run(case.nsteps)
        assert s.status() == 0
    err = np.linalg.norm(out["rec"] - gold, axis=1) / np.linalg.norm(gold, axis=1)
    assert (err < 5e-5).all(), err


# ---------------------------------------------------------------------------
# adjoints
# ---------------------------------------------------------------------------
def _gen21_case(seed, top_bc=1):
    case = _ii(random_case_gen21(seed, ratio=2, nx2=6, ny2=5, nz=(6, 5), top_bc=top_bc, aniso=0.3))
    for m in case.media:
        m["buoy"] = m["buoy"].astype(np.float64)
    return case


def _rand_state(case, rng):
    return {(g, k): rng.standard_normal(field_shape(case.grids[g]["n"], SIM_POS[k], case.radius))
            for g in range(len(case.grids)) for k in range(9)}


@pytest.mark.parametrize("skip_end", [False, True])
@pytest.mark.parametrize("op", ["vz", "sxz", "syz"])
def test_adjoint_dot_product(op, skip_end):
    case = _gen21_case(7)
    case.ii_skip_end_column = skip_end
    rng = np.random.default_rng(len(op) + 10 * skip_end)
    s, y = _rand_state(case, rng), _rand_state(case, rng)
    with Simulation(case, precision="f64") as sim:
        for (g, k), a in s.items():
            sim.set_field(g, k, a)
        getattr(sim, "ghost_" + op)(1)
        out = {key: sim.field(*key) for key in s}
        sim.adjoint_reset()
        for (g, k), a in y.items():
            sim.set_adjoint_field(g, k, a)
        sim.adjoint_op(op, 1)
        z = {key: sim.adjoint_field(*key) for key in y}
    lhs = sum(float(np.sum(y[k] * out[k])) for k in y)
    rhs = sum(float(np.sum(z[k] * s[k])) for k in s)
    scale = sum(float(np.sum(np.abs(y[k] * out[k]))) for k in y)
    assert abs(lhs - rhs) <= 1e-12 * scale, (lhs, rhs)


def test_misfit_gradient_matches_finite_differences():
    nsteps = 24
    case = _with_src_rec(_gen21_case(13), nsteps)
    rng = np.random.default_rng(3)
    obs = (0.1 * rng.standard_normal((nsteps, len(case.rec)))).astype(np.float32)
    with Simulation(case, precision="f64") as sim:
        loss = sim.misfit_gradient(obs, ckpt_every=5)
        grads = [[sim.gradient(g, w) for w in range(22)] for g in range(2)]
    assert np.isfinite(loss) and loss > 0
    dirs = []
    for m in case.media:
        d = [m["buoy"] * rng.standard_normal(m["buoy"].shape)]
        scale = np.abs(m["c21"][0]).mean()
        d += [scale * rng.standard_normal(m["c21"][k].shape) for k in range(21)]
        dirs.append(d)

    def loss_at(eps):
        c = copy.deepcopy(case)
        for g, m in enumerate(c.media):
            m["buoy"] = case.media[g]["buoy"] + eps * dirs[g][0]
            m["c21"] = [case.media[g]["c21"][k] + eps * dirs[g][1 + k] for k in range(21)]
        with Simulation(c, precision="f64") as sim:
            return sim.misfit_gradient(obs, ckpt_every=nsteps)

    eps = 1e-4
    fd = (loss_at(eps) - loss_at(-eps)) / (2 * eps)
    an = sum(float(np.sum(grads[g][w] * dirs[g][w])) for g in range(2) for w in range(22))
    assert abs(fd - an) <= 1e-5 * abs(fd), (fd, an)
