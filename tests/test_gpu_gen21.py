"""21-Cij media on the device (ecsg_set_medium_cij21) against the oracle's
o_update_stress21 and its energy.

The device stress update follows the oracle's operation order, so the FP64
instantiation must match it exactly; interface solves and reductions differ
in summation order only (<= 1e-12 relative).  FP32: one operator <= 4e-6
relative to the field scale (21 products per normal stress instead of 3),
traces within 1e-5 rel-L2 of the FP64 oracle.
"""
import copy

import numpy as np
import pytest

from ecsg_b200 import Simulation
from ecsg_b200.workloads import ortho9_from_cij21, random_case_gen21, random_case_tti, ricker, tti_as_gen21
from oracle.oracle import OracleRun

pytestmark = pytest.mark.gpu


def _randomize(o, s, rng, prec):
    for g in range(len(o.levels)):
        for k in range(9):
            a = rng.standard_normal(o.levels[g]["f"][k].shape)
            if prec == "f32":
                a = a.astype(np.float32).astype(np.float64)
            o.levels[g]["f"][k][...] = a
            s.set_field(g, k, a)


def _err(o, s, comps=range(9)):
    worst = 0.0
    for g in range(len(o.levels)):
        for k in comps:
            a, b = o.levels[g]["f"][k], s.field(g, k)
            worst = max(worst, float(np.abs(a - b).max() / max(np.abs(a).max(), 1e-300)))
    return worst


def _with_src_rec(case, nt=60):
    h, n = case.grids[0]["h"], case.grids[0]["n"]
    case.src = {"xyz": (n[0] // 2 * h[0], n[1] // 2 * h[1], 2 * h[2]), "trace": ricker(nt, case.dt * 1e-3 * 0.5, 15.0),
                "scale": 1000.0, "comp": 0}
    case.rec = np.array([[(n[0] // 2 + 3) * h[0], n[1] // 2 * h[1], 2 * h[2]],
                         [(n[0] // 3) * h[0], (n[1] // 3) * h[1], (n[2] - 1) * h[2]],
                         [(n[0] // 2) * h[0], (n[1] // 2) * h[1], (n[2] + 2) * h[2]]], dtype=np.float32)
    return case


# (ratio, top_bc, nz): nz = 20 splits the fine grid's z-march into several chunks
CASES = [(2, 1, (6, 5)), (2, 0, (6, 5)), (3, 1, (6, 5)), (2, 1, (20, 12))]


@pytest.mark.parametrize("ratio,top_bc,nz", CASES)
def test_stress21_and_vz_f64(ratio, top_bc, nz):
    case = random_case_gen21(11 + ratio, ratio=ratio, nx2=7, ny2=6, nz=nz, top_bc=top_bc, aniso=0.3)
    o = OracleRun(case, energy=True)
    rng = np.random.default_rng(ratio + 10 * top_bc + nz[0])
    with Simulation(case, precision="f64", energy=True) as s:
        _randomize(o, s, rng, "f64")
        for g in range(2):
            o.update_stress(g)
            s.update_stress(g)
        assert _err(o, s) == 0.0
        # a second update adds onto the displacement sums of the first
        _randomize(o, s, rng, "f64")
        for g in range(2):
            o.update_stress(g)
            s.update_stress(g)
        assert _err(o, s) == 0.0
        _randomize(o, s, rng, "f64")
        o.ghost_vz(1)
        s.ghost_vz(1)
        assert _err(o, s) < 1e-12
        o.copy_vel()
        s.copy_vel()
        eo, es = o.energy(), s.energy()
        assert abs(eo - es) <= 1e-12 * abs(eo), (eo, es)


@pytest.mark.parametrize("ratio,top_bc,nz", CASES)
def test_stress21_and_vz_f32(ratio, top_bc, nz):
    case = random_case_gen21(21 + ratio, ratio=ratio, nx2=7, ny2=6, nz=nz, top_bc=top_bc, aniso=0.3)
    o = OracleRun(case)
    rng = np.random.default_rng(100 + ratio + 10 * top_bc + nz[0])
    with Simulation(case, precision="f32") as s:
        _randomize(o, s, rng, "f32")
        for g in range(2):
            o.update_stress(g)
            s.update_stress(g)
        assert _err(o, s) < 4e-6
        _randomize(o, s, rng, "f32")
        o.ghost_vz(1)
        s.ghost_vz(1)
        assert _err(o, s) < 4e-6


def test_off_block_zero_equals_orthorhombic_device_path():
    case = random_case_gen21(3, ratio=2, nx2=9, ny2=8, nz=(8, 6), top_bc=1)
    for m in case.media:
        for k in list(range(6, 15)) + [16, 17, 19]:
            m["c21"][k] = np.zeros_like(m["c21"][k])
        m["c9"] = ortho9_from_cij21(m["c21"])
    case = _with_src_rec(case)
    c9 = copy.copy(case)
    c9.medium = "ortho9"
    outs = []
    for cs in (case, c9):
        with Simulation(cs, precision="f64") as s:
            r = s.run(60, graph=False)
            outs.append((r["rec"], [s.field(g, k) for g in range(2) for k in range(9)]))
    assert np.abs(outs[0][0] - outs[1][0]).max() <= 1e-6 * np.abs(outs[1][0]).max()
    for a, b in zip(outs[0][1], outs[1][1]):
        assert np.abs(a - b).max() <= 1e-12 * max(np.abs(b).max(), 1e-300)


@pytest.mark.parametrize("ratio", [2, 3])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_time_loop_vs_oracle(ratio, prec):
    case = _with_src_rec(random_case_gen21(40 + ratio, ratio=ratio, nx2=9, ny2=8, nz=(8, 6), aniso=0.3))
    n = 80
    o = OracleRun(case, energy=True)
    ref = o.run(n)
    with Simulation(case, precision=prec, energy=True) as s:
        out = s.run(n, energy_every=1, graph=False)
    erel = np.abs(out["energy"] - ref["energy"]) / np.abs(ref["energy"]).max()
    if prec == "f64":
        ref32 = ref["rec"].astype(np.float32).astype(np.float64)
        rel32 = np.linalg.norm(out["rec"] - ref32, axis=1) / np.linalg.norm(ref32, axis=1)
        assert rel32.max() < 1e-7 and erel.max() < 1e-10, (rel32, erel.max())
    else:
        rel = np.linalg.norm(out["rec"] - ref["rec"], axis=1) / np.linalg.norm(ref["rec"], axis=1)
        assert rel.max() < 1e-5 and erel.max() < 1e-5, (rel, erel.max())


def test_graph_replay_is_bitwise_equal():
    case = _with_src_rec(random_case_gen21(50, ratio=3, nx2=9, ny2=8, nz=(8, 6), aniso=0.3))
    outs = []
    for graph in (False, True):
        with Simulation(case, precision="f32", energy=True) as s:
            r = s.run(40, energy_every=5, graph=graph)
            outs.append((r, [s.field(g, k) for g in range(2) for k in range(9)]))
    (ra, fa), (rb, fb) = outs
    assert np.array_equal(ra["rec"], rb["rec"])
    assert np.array_equal(ra["energy"], rb["energy"], equal_nan=True)
    for a, b in zip(fa, fb):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("prec,tol", [("f64", 1e-11), ("f32", 1e-5)])
@pytest.mark.parametrize("ratio,top_bc", [(2, 1), (3, 1), (3, 0)])
def test_energy_conserved_after_source(ratio, top_bc, prec, tol):
    case = random_case_gen21(60 + ratio, ratio=ratio, nx2=12, ny2=10, nz=(12, 8), top_bc=top_bc, aniso=0.3)
    case = _with_src_rec(case, nt=60)
    case.mirror_fix = True
    with Simulation(case, precision=prec, energy=True) as s:
        out = s.run(800, energy_every=10)
    e = out["energy"][100::10]   # the source acts during the first 60 steps
    drift = (e.max() - e.min()) / np.abs(e).mean()
    assert np.isfinite(e).all() and drift < tol, drift


@pytest.mark.parametrize("ratio", [2, 3])
def test_device_tti_medium_matches_host_slots(ratio):
    """ecsg_set_medium_tti (rotation and averaging on the device) against the
    same medium rotated and averaged on the host (ecsg_set_medium_cij21), and
    the FP32 run against the oracle on the host slots."""
    case = _with_src_rec(random_case_tti(7 + ratio, ratio=ratio, nx2=9, ny2=8, nz=(8, 6)))
    host = tti_as_gen21(case)
    runs = []
    for cs in (case, host):
        with Simulation(cs, precision="f64") as s:
            r = s.run(60, graph=False)
            runs.append((r["rec"], [s.field(g, k) for g in range(2) for k in range(9)]))
    assert np.abs(runs[0][0] - runs[1][0]).max() <= 1e-6 * np.abs(runs[1][0]).max()
    for a, b in zip(runs[0][1], runs[1][1]):
        assert np.abs(a - b).max() <= 1e-11 * max(np.abs(b).max(), 1e-300)
    ref = OracleRun(host).run(60)
    with Simulation(case, precision="f32") as s:
        out = s.run(60)
    rel = np.linalg.norm(out["rec"] - ref["rec"], axis=1) / np.linalg.norm(ref["rec"], axis=1)
    assert rel.max() < 1e-5, rel


@pytest.mark.parametrize("energy", [True, False])
@pytest.mark.parametrize("ratio,top_bc,nx2,ny2,nz", [(3, 1, 45, 11, (60, 30)), (2, 0, 67, 9, (20, 50)),
                                                    (2, 1, 64, 16, (49, 24))])
def test_tma_sweep_equals_scalar_sweep(monkeypatch, ratio, top_bc, nx2, ny2, nz, energy):
    """The FP32 TMA-staged sweep (stress21_tma.cu) against the plain FP32 sweep
    (stress21.cu, selected by ECSG_SCALAR_STENCILS=1): bitwise equal fields,
    traces and energies, on ragged tiles (x not a multiple of 32, y not of 8),
    several z-chunks per column, with and without the free surface and the
    displacement sums."""
    case = _with_src_rec(random_case_tti(70 + ratio + top_bc, ratio=ratio, nx2=nx2, ny2=ny2, nz=nz, top_bc=top_bc))
    from ecsg_b200 import SIM_POS, field_shape
    outs, ops = [], []
    for scalar in ("1", "0"):
        monkeypatch.setenv("ECSG_SCALAR_STENCILS", scalar)
        rng = np.random.default_rng(nx2)
        with Simulation(case, precision="f32", energy=energy) as s:
            for g in range(2):
                for k in range(9):
                    s.set_field(g, k, rng.standard_normal(field_shape(case.grids[g]["n"], SIM_POS[k], 1)))
            for g in range(2):
                s.update_stress(g)
            ops.append([s.field(g, k) for g in range(2) for k in range(9)])
        with Simulation(case, precision="f32", energy=energy) as s:
            r = s.run(30, energy_every=3 if energy else 0, graph=False)
            outs.append((r, [s.field(g, k) for g in range(2) for k in range(9)], s.status()))
    for a, b in zip(*ops):
        assert np.array_equal(a, b)
    (ra, fa, sa), (rb, fb, sb) = outs
    assert sa == 0 and sb == 0
    assert np.array_equal(ra["rec"], rb["rec"])
    if energy:
        assert np.array_equal(ra["energy"], rb["energy"], equal_nan=True)
    for a, b in zip(fa, fb):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("medium", ["tti", "iso"])
@pytest.mark.parametrize("ratio,top_bc,nx2,ny2,nz", [(3, 1, 45, 11, (60, 30)), (2, 0, 67, 9, (20, 50)),
                                                    (2, 1, 33, 16, (49, 24))])
def test_tma_velocity_sweep_equals_float4_sweep(monkeypatch, ratio, top_bc, nx2, ny2, nz, medium):
    """The FP32 TMA-staged velocity sweep (vel_tma.cu) against the float4 sweep
    (stencil_v4.cu, selected by ECSG_VEL_TMA=0): bitwise equal fields after one
    operator on random fields, and bitwise equal traces, energies and fields
    after 30 steps (energy copies every 3rd step), on tiles that do not divide
    the grid in x or y and with several z-chunks."""
    from ecsg_b200 import SIM_POS, field_shape
    from ecsg_b200.workloads import random_case
    if medium == "tti":
        case = random_case_tti(80 + ratio + top_bc, ratio=ratio, nx2=nx2, ny2=ny2, nz=nz, top_bc=top_bc)
    else:
        case = random_case(80 + ratio + top_bc, ratio=ratio, nx2=nx2, ny2=ny2, nz=nz, top_bc=top_bc)
    case = _with_src_rec(case)
    ops, outs = [], []
    for tma in ("0", "1"):
        monkeypatch.setenv("ECSG_VEL_TMA", tma)
        rng = np.random.default_rng(nx2 + ny2)
        with Simulation(case, precision="f32", energy=True) as s:
            for g in range(2):
                for k in range(9):
                    s.set_field(g, k, rng.standard_normal(field_shape(case.grids[g]["n"], SIM_POS[k], 1)))
            for g in range(2):
                s.update_vel(g)
            ops.append([s.field(g, k) for g in range(2) for k in range(3)])
        with Simulation(case, precision="f32", energy=True) as s:
            r = s.run(30, energy_every=3, graph=True)
            outs.append((r, [s.field(g, k) for g in range(2) for k in range(9)], s.status()))
    for a, b in zip(*ops):
        assert np.array_equal(a, b)
    (ra, fa, sa), (rb, fb, sb) = outs
    assert sa == 0 and sb == 0
    assert np.array_equal(ra["rec"], rb["rec"])
    assert np.array_equal(ra["energy"], rb["energy"], equal_nan=True)
    for a, b in zip(fa, fb):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("medium", ["tti", "iso"])
@pytest.mark.parametrize("graph", [False, True])
def test_side_stream_grids_equal_one_stream(monkeypatch, medium, graph):
    """The coarse grids' velocity and stress sweeps on side streams (the
    default for multi-grid runs) against every sweep on the library stream
    (ECSG_SIDE_GRIDS=0): bitwise equal traces, energies and fields on a
    three-grid ratio-3 composite, eager and as a CUDA graph."""
    from ecsg_b200.workloads import three_grid_case
    case = three_grid_case(seed=4, grids=[((72, 54, 12), 5.0), ((24, 18, 10), 15.0), ((8, 6, 8), 45.0)],
                           nsteps=40, medium=medium)
    outs = []
    for side in ("0", "1"):
        monkeypatch.setenv("ECSG_SIDE_GRIDS", side)
        with Simulation(case, precision="f32", energy=True) as s:
            r = s.run(40, energy_every=4, graph=graph)
            outs.append((r, [s.field(g, k) for g in range(3) for k in range(9)], s.status()))
    (ra, fa, sa), (rb, fb, sb) = outs
    assert sa == 0 and sb == 0
    assert np.abs(ra["rec"]).max() > 0
    assert np.array_equal(ra["rec"], rb["rec"])
    assert np.array_equal(ra["energy"], rb["energy"], equal_nan=True)
    for a, b in zip(fa, fb):
        assert np.array_equal(a, b)


@pytest.mark.parametrize("prec", ["f32", "f64"])
def test_fused_interface_solves_equal_one_launch_each(monkeypatch, prec):
    """The sxz solves of both interfaces of a three-grid composite in one
    cooperative launch (the default) against one launch per interface
    (ECSG_SXZ_FUSED=0): bitwise equal traces, fields and sweep counts, over
    enough steps for the wavefield to reach both interfaces (several sweeps
    per solve)."""
    from ecsg_b200.workloads import three_grid_case
    case = three_grid_case(seed=5, grids=[((72, 54, 6), 5.0), ((24, 18, 4), 15.0), ((8, 6, 8), 45.0)],
                           nsteps=160, medium="tti")
    outs = []
    for fused in ("0", "1"):
        monkeypatch.setenv("ECSG_SXZ_FUSED", fused)
        with Simulation(case, precision=prec, energy=True) as s:
            r = s.run(160, energy_every=8)
            totals = [s.sxz_state(i)[3] for i in (1, 2)]
            outs.append((r, [s.field(g, k) for g in range(3) for k in range(9)], s.status(), totals))
    (ra, fa, sa, ta), (rb, fb, sb, tb) = outs
    assert sa == 0 and sb == 0
    assert ta == tb and min(ta) > 160, ta   # both interfaces needed more than one sweep on some steps
    assert np.array_equal(ra["rec"], rb["rec"])
    assert np.array_equal(ra["energy"], rb["energy"], equal_nan=True)
    for a, b in zip(fa, fb):
        assert np.array_equal(a, b)
