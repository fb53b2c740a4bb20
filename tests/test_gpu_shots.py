"""Shots in lockstep (ecsg_shots_misfit_gradient; no reference counterpart)
against the same shots one at a time (ecsg_misfit_gradient): three shots of
one 21-Cij model at ratios 2 and 3, each with its own source, sharing one
medium allocation.  The per-shot losses are bitwise the one-at-a-time losses
(the forward of each shot is the same arithmetic, the lockstep sxz solves
included), and the gradient left in the first instance equals the sum of the
one-at-a-time gradients to 1e-12 of the gradient's scale in FP64 and 1e-6 in
FP32 (the shots' terms are accumulated per step and point instead of per
shot).  Checkpointing with one level (the segment's states stored) and with
two (sub-checkpoints every 3 steps, the form used when the segment's states
of all shots do not fit in device memory) gives the same losses bitwise and
the same gradient to the same tolerance (the velocity adjoint adds with
atomics, in no fixed order).  Under a checkpoint budget that three shots do
not fit at one level, the call runs them as groups that do and sums the
groups' gradients: the same losses bitwise and the same gradient."""
import numpy as np
import pytest

from ecsg_b200 import Simulation, device_layout, shots_misfit_gradient
from ecsg_b200.workloads import random_case_gen21, ricker

pytestmark = pytest.mark.gpu


def _shot_case(seed, ratio, shift, nsteps):
    c = random_case_gen21(seed, ratio=ratio, nx2=8, ny2=7, nz=(7, 6), aniso=0.3)
    for m in c.media:
        m["buoy"] = m["buoy"].astype(np.float64)
    h, n = c.grids[0]["h"], c.grids[0]["n"]
    c.src = {"xyz": ((n[0] // 2 + shift) * h[0], (n[1] // 2 - shift) * h[1], 2 * h[2]),
             "trace": ricker(nsteps, c.dt * 1e-3 * 0.5, 15.0), "scale": 1000.0, "comp": 2}
    c.rec = np.array([[(n[0] // 2 + 3) * h[0], n[1] // 2 * h[1], 0.0],
                      [(n[0] // 3) * h[0], (n[1] // 3) * h[1], 0.0],
                      [(n[0] // 2) * h[0], (n[1] // 2) * h[1], (n[2] + 2) * h[2]]], dtype=np.float32)
    c.rec_comp = 2
    c.mirror_fix = True
    return c


def _close(a, b, tol, scale):
    return float(np.abs(a - b).max()) <= tol * scale


@pytest.mark.parametrize("ratio", [2, 3])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_shots_in_lockstep_equal_one_at_a_time(prec, ratio):
    nsteps, k = 22, 8
    seed = 90 + ratio
    cases = [_shot_case(seed, ratio, shift, nsteps) for shift in (-2, 0, 3)]
    rng = np.random.default_rng(ratio)
    obs = [(0.05 * rng.standard_normal((nsteps, len(c.rec)))).astype(np.float32) for c in cases]
    want_loss, want_grad = [], []
    for c, o in zip(cases, obs):
        with Simulation(c, precision=prec) as s:
            want_loss.append(s.misfit_gradient(o, ckpt_every=k))
            want_grad.append([s.gradient(g, w) for g in range(2) for w in range(22)])
    got = {}
    for sub in (0, 3):
        model = Simulation(cases[0], precision=prec)
        sims = [model] + [Simulation.shot(model, c) for c in cases[1:]]
        try:
            losses = shots_misfit_gradient(sims, obs, ckpt_every=k, sub_every=sub)
            got[sub] = (losses, [model.gradient(g, w) for g in range(2) for w in range(22)],
                        [x.status() for x in sims], [x.field(0, 2) for x in sims])
        finally:
            for x in sims[1:]:
                x.close()
            model.close()
    (l0, g0, st0, f0), (l1, g1, st1, f1) = got[0], got[3]
    assert st0 == [0, 0, 0] and st1 == [0, 0, 0]
    assert np.array_equal(l0, np.array(want_loss)), (l0, want_loss)
    assert np.array_equal(l0, l1)
    tol = 1e-12 if prec == "f64" else 1e-6
    scale = max(max(float(np.abs(gs[v]).max()) for v in range(44)) for gs in want_grad)
    for w in range(44):
        ref = sum(gs[w] for gs in want_grad)
        assert _close(g0[w], ref, tol, scale), (w, float(np.abs(g0[w] - ref).max()) / scale)
        assert _close(g1[w], g0[w], tol, scale), w
    # each shot is left at its own final forward state
    for c, fa, fb in zip(cases, f0, f1):
        with Simulation(c, precision=prec) as s:
            s.run(nsteps, graph=False)
            assert np.array_equal(fa, s.field(0, 2)) and np.array_equal(fb, fa)


def _state_bytes(case, prec):
    """Bytes of one saved state: the nine fields of every grid's box and the
    sxz warm starts of every interface (the plan's unit)."""
    tsize = 8 if prec == "f64" else 4
    b = 0
    for g in case.grids:
        px, py, pz = device_layout(g["n"], case.radius)["pitch"]
        b += 9 * px * py * pz * tsize
    for g in case.grids[1:]:
        b += 8 * (g["n"][0] + 1) * (g["n"][1] + 1)
    return b


@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_shots_in_groups_when_one_level_does_not_fit(monkeypatch, prec):
    """A checkpoint budget (ECSG_SHOTS_MEMORY) of 30 states in all:
    three shots need at least 36 states for one level at any interval up to
    the requested 8 steps (22 steps), two shots 26 at 8, so the call runs the
    shots as a group of two and a group of one, one level each, and sums the
    groups' gradients.  Losses bitwise and gradient to the one-at-a-time
    tolerance, as in the unconstrained call."""
    nsteps, k, ratio = 22, 8, 3
    cases = [_shot_case(93, ratio, shift, nsteps) for shift in (-2, 0, 3)]
    rng = np.random.default_rng(7)
    obs = [(0.05 * rng.standard_normal((nsteps, len(c.rec)))).astype(np.float32) for c in cases]
    want_loss, want_grad = [], []
    for c, o in zip(cases, obs):
        with Simulation(c, precision=prec) as s:
            want_loss.append(s.misfit_gradient(o, ckpt_every=k))
            want_grad.append([s.gradient(g, w) for g in range(2) for w in range(22)])
    monkeypatch.setenv("ECSG_SHOTS_MEMORY", str(30 * _state_bytes(cases[0], prec)))
    model = Simulation(cases[0], precision=prec)
    sims = [model] + [Simulation.shot(model, c) for c in cases[1:]]
    try:
        losses = shots_misfit_gradient(sims, obs, ckpt_every=k)
        grad = [model.gradient(g, w) for g in range(2) for w in range(22)]
        status = [x.status() for x in sims]
        final = [x.field(0, 2) for x in sims]
    finally:
        for x in sims[1:]:
            x.close()
        model.close()
    assert status == [0, 0, 0]
    assert np.array_equal(losses, np.array(want_loss)), (losses, want_loss)
    tol = 1e-12 if prec == "f64" else 1e-6
    scale = max(max(float(np.abs(gs[v]).max()) for v in range(44)) for gs in want_grad)
    for w in range(44):
        ref = sum(gs[w] for gs in want_grad)
        assert _close(grad[w], ref, tol, scale), (w, float(np.abs(grad[w] - ref).max()) / scale)
    for c, f in zip(cases, final):
        with Simulation(c, precision=prec) as s:
            s.run(nsteps, graph=False)
            assert np.array_equal(f, s.field(0, 2))


def test_shots_reject_instances_of_another_model():
    nsteps = 6
    a = _shot_case(95, 2, 0, nsteps)
    b = _shot_case(96, 2, 1, nsteps)
    obs = [np.zeros((nsteps, 3), np.float32)] * 2
    with Simulation(a, precision="f32") as sa, Simulation(b, precision="f32") as sb:
        with pytest.raises(Exception, match="share"):
            shots_misfit_gradient([sa, sb], obs, ckpt_every=3)
