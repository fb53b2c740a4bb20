"""Batches of instances (no reference counterpart) against the same instances
run one at a time: the batched step graph, shots sharing one medium, batched
misfit gradients with their FP64 sum, and the z-march autotuner."""
import numpy as np
import pytest

from ecsg_b200 import Simulation, batch_misfit_gradient, batch_run, sum_gradients
from ecsg_b200.workloads import random_case, random_case_gen21, ricker

pytestmark = pytest.mark.gpu


def _src_rec(case, nt, shift=0):
    h, n = case.grids[0]["h"], case.grids[0]["n"]
    case.src = {"xyz": ((n[0] // 2 + shift) * h[0], n[1] // 2 * h[1], 2 * h[2]),
                "trace": ricker(nt, case.dt * 1e-3 * 0.5, 15.0), "scale": 1000.0, "comp": 0}
    case.rec = np.array([[(n[0] // 2 + 3) * h[0], n[1] // 2 * h[1], 2 * h[2]],
                         [(n[0] // 3) * h[0], (n[1] // 3) * h[1], (n[2] - 1) * h[2]]], dtype=np.float32)
    return case


def _cases():
    return [_src_rec(random_case(81, ratio=2, nx2=9, ny2=8, nz=(8, 6)), 30),
            _src_rec(random_case(82, ratio=3, nx2=7, ny2=10, nz=(9, 5)), 30),
            _src_rec(random_case_gen21(83, ratio=2, nx2=11, ny2=6, nz=(7, 7), aniso=0.3), 30)]


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_batch_run_equals_one_at_a_time(prec):
    nsteps = 30
    alone = []
    for c in _cases():
        with Simulation(c, precision=prec) as s:
            r = s.run(nsteps, graph=False)
            alone.append((r["rec"], [s.field(g, k) for g in range(2) for k in range(9)]))
    sims = [Simulation(c, precision=prec) for c in _cases()]
    try:
        traces, ms = batch_run(sims, nsteps)
        fields = [[s.field(g, k) for g in range(2) for k in range(9)] for s in sims]
    finally:
        for s in sims:
            s.close()
    assert ms > 0
    for (rec, fa), tr, fb in zip(alone, traces, fields):
        assert np.array_equal(rec, tr)
        for a, b in zip(fa, fb):
            assert np.array_equal(a, b)


def test_shots_share_the_medium_and_batched_gradients_sum():
    nsteps = 20
    base = random_case_gen21(85, ratio=2, nx2=8, ny2=7, nz=(7, 6), aniso=0.3)
    for m in base.media:
        m["buoy"] = m["buoy"].astype(np.float64)
    shots = [_src_rec(random_case_gen21(85, ratio=2, nx2=8, ny2=7, nz=(7, 6), aniso=0.3), nsteps, shift=k)
             for k in (-2, 0, 3)]
    for c in shots:
        for m in c.media:
            m["buoy"] = m["buoy"].astype(np.float64)
    rng = np.random.default_rng(5)
    obs = [(0.05 * rng.standard_normal((nsteps, len(c.rec)))).astype(np.float32) for c in shots]
    # one at a time, each with its own medium copy
    want_loss, want_grad = [], []
    for c, o in zip(shots, obs):
        with Simulation(c, precision="f64") as s:
            want_loss.append(s.misfit_gradient(o, ckpt_every=6))
            want_grad.append([s.gradient(g, w) for g in range(2) for w in range(22)])
    model = Simulation(base, precision="f64")
    sims = [Simulation.shot(model, c) for c in shots]
    try:
        before = model.device_bytes()
        assert all(s.device_bytes() < before for s in sims)   # no medium copy of their own
        losses = batch_misfit_gradient(sims, obs, ckpt_every=6)
        got = [[s.gradient(g, w) for g in range(2) for w in range(22)] for s in sims]
        sum_gradients(sims[0], sims)
        total = [sims[0].gradient(g, w) for g in range(2) for w in range(22)]
    finally:
        for s in sims:
            s.close()
        model.close()
    assert np.array_equal(losses, np.array(want_loss))
    for gs, ws in zip(got, want_grad):
        for a, b in zip(gs, ws):
            assert np.abs(a - b).max() <= 1e-12 * max(np.abs(b).max(), 1e-300)
    for k, t in enumerate(total):
        ref = sum(w[k] for w in want_grad)
        assert np.abs(t - ref).max() <= 1e-12 * max(np.abs(ref).max(), 1e-300)


def test_autotune_changes_launch_shapes_not_results():
    case = _src_rec(random_case_gen21(87, ratio=3, nx2=12, ny2=10, nz=(40, 20), aniso=0.3), 25)
    with Simulation(case, precision="f32", energy=True) as s:
        a = s.run(25, energy_every=5, graph=True)
        fa = [s.field(g, k) for g in range(2) for k in range(9)]
    with Simulation(case, precision="f32", energy=True) as s:
        tuning = s.autotune(2)
        assert len(tuning) == 2 and all(len(t) == 2 for t in tuning)
        b = s.run(25, energy_every=5, graph=True)
        fb = [s.field(g, k) for g in range(2) for k in range(9)]
    assert np.array_equal(a["rec"], b["rec"])
    assert np.array_equal(a["energy"], b["energy"], equal_nan=True)
    for x, y in zip(fa, fb):
        assert np.array_equal(x, y)
