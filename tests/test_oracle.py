"""Pins the C restatement (oracle/ecsg_oracle.c) to the reference.

1. Operator by operator against the reference's own functions (compiled from
   its sources into oracle/_ref) on random heterogeneous composites.
2. Whole time steps against the reference's loop.
3. Against the reference's golden receiver traces (tests/golden, recovered from
   the reference's SVN store by tests/golden/make_golden.py).
"""
import os

import numpy as np
import pytest

from conftest import ref_available
from ecsg_b200.workloads import eci_test_case, random_case
from oracle.oracle import OracleRun

GOLDEN = os.path.join(os.path.dirname(os.path.abspath(__file__)), "golden")

needs_ref = pytest.mark.skipif(not ref_available(64), reason="reference build (oracle/_ref) missing")


def _randomize(o, r, rng, scale=1.0):
    for g in range(len(o.levels)):
        for k in range(9):
            a = scale * rng.standard_normal(o.levels[g]["f"][k].shape)
            o.levels[g]["f"][k][...] = a
            r.set(g, k, a)


def _maxdiff(o, r):
    m = 0.0
    for g in range(len(o.levels)):
        for k in range(9):
            m = max(m, float(np.abs(o.levels[g]["f"][k] - r.get(g, k)).max()))
    return m


@needs_ref
@pytest.mark.parametrize("seed,top_bc", [(1, 1), (2, 0), (3, 1)])
def test_operators_match_reference(seed, top_bc):
    from oracle.ref import RefRun
    case = random_case(seed, ratio=2, nx2=6, ny2=5, nz=(5, 4), top_bc=top_bc)
    o = OracleRun(case, energy=True)
    r = RefRun(case, energy=True, threads=2)
    try:
        rng = np.random.default_rng(seed)
        for g in range(2):
            for k in range(9):
                assert np.array_equal(r.get(g, k, kind=1), o.levels[g]["c"][k]), (g, k)
        # stencils: same expression order, no FMA on either side -> bitwise
        _randomize(o, r, rng)
        for g in range(2):
            o.update_vel(g)
            r.update_vel(g)
        assert _maxdiff(o, r) == 0.0
        _randomize(o, r, rng)
        for g in range(2):
            o.update_stress(g)
            r.update_stress(g)
        assert _maxdiff(o, r) == 0.0
        # interface solves: same equations, general-ratio summation order
        _randomize(o, r, rng)
        o.ghost_vz(1)
        r.ghost_vz(1)
        assert _maxdiff(o, r) < 1e-13
        _randomize(o, r, rng)
        o.ghost_syz(1)
        r.ghost_syz(1)
        assert _maxdiff(o, r) < 1e-13
        _randomize(o, r, rng)
        o.ghost_sxz(1)
        r.ghost_sxz(1)
        assert _maxdiff(o, r) < 1e-12
        assert np.abs(o.X[0]["X"] - r.gsxz(0)).max() < 1e-12
        # energy and residues
        _randomize(o, r, rng)
        o.copy_vel()
        r.copy_vel()
        _randomize(o, r, rng)
        eo, er = o.energy(), r.energy()
        assert abs(eo - er) <= 1e-13 * abs(er)
        ro = o.residues(1)
        rr = r.residues(7)[0]   # the reference keeps residues as float32
        assert np.allclose(ro, rr, rtol=1e-6, atol=1e-6)
    finally:
        r.close()


@needs_ref
@pytest.mark.parametrize("top_bc", [1, 0])
@pytest.mark.parametrize("radius", [2, 3, 4, 5, 6])
def test_high_order_stencils_match_reference(radius, top_bc):
    from oracle.ref import RefRun
    case = random_case(7, ratio=2, nx2=8, ny2=7, nz=(9,), num_grids=1, radius=radius, top_bc=top_bc)
    o = OracleRun(case)
    r = RefRun(case, threads=2)
    try:
        rng = np.random.default_rng(radius)
        _randomize(o, r, rng)
        o.update_vel(0)
        r.update_vel(0)
        assert _maxdiff(o, r) == 0.0
        _randomize(o, r, rng)
        o.update_stress(0)
        r.update_stress(0)
        assert _maxdiff(o, r) == 0.0
    finally:
        r.close()


@needs_ref
def test_time_loop_matches_reference():
    """20 steps of main.cpp's loop with a source and receivers on a random composite."""
    from oracle.ref import RefRun
    case = random_case(11, ratio=2, nx2=8, ny2=6, nz=(6, 5))
    from ecsg_b200.workloads import ricker
    h = case.grids[0]["h"][0]
    case.src = {"xyz": (8 * h, 6 * h, 2 * h), "trace": ricker(40, case.dt / 1000.0 * 20, 15.0), "scale": 1000.0,
                "comp": 0}
    case.rec = np.array([[5 * h, 6 * h, 2 * h], [9 * h, 3 * h, 5 * h], [10 * h, 4 * h, 8 * h]], dtype=np.float32)
    o = OracleRun(case, energy=True)
    r = RefRun(case, energy=True, verb=False, threads=2)
    try:
        assert o.src == r.src_loc()[0]
        assert o.rec == r.rec_loc()
        for n in range(20):
            rec_o, e_o, _ = o.step(n)
            rec_r, e_r = r.step(n)
            assert np.abs(rec_o - rec_r).max() <= 1e-12 * max(1.0, np.abs(rec_r).max())
            assert abs(e_o - e_r) <= 1e-12 * abs(e_r)
        assert _maxdiff(o, r) <= 1e-10
    finally:
        r.close()


def test_golden_fixtures_present():
    for name in ("rec_eci_test1", "rec_eci_test2", "rec_eci_test3"):
        a = np.load(os.path.join(GOLDEN, name + ".npy"))
        assert a.shape == (4, 1172) and a.dtype == np.float32 and np.isfinite(a).all()
    geo = np.load(os.path.join(GOLDEN, "geo_eci_test1.npy"))
    case = eci_test_case(1)
    assert np.array_equal(geo.reshape(4, 3), case.rec)


def test_eci_case_geometry():
    """The rebuilt test1 inputs have the geometry the reference experiment reports."""
    case = eci_test_case(1)
    assert case.grids[0]["n"] == (384, 384, 72) and case.grids[1]["n"] == (192, 192, 59)
    assert case.nsteps == 1172 and abs(case.dt - 0.589378) < 1e-12
    o = OracleRun(case)
    assert o.src == (0, 192, 192, 14)
    assert o.rec == [(0, 210, 192, 14), (0, 230, 192, 14), (0, 248, 192, 14), (0, 268, 192, 14)]


def _rel_l2(a, b):
    return np.linalg.norm(a - b, axis=-1) / np.linalg.norm(b, axis=-1)


def test_oracle_reproduces_golden_prefix():
    """First 400 of 1172 steps of the test1 ECI experiment (receivers are causal,
    so a prefix of the golden trace is the golden trace of a shorter run)."""
    n = 400
    case = eci_test_case(1, nsteps=n)
    out = OracleRun(case).run(n)["rec"]
    gold = np.load(os.path.join(GOLDEN, "rec_eci_test1.npy"))[:, :n]
    err = _rel_l2(out, gold)
    assert (err < 5e-5).all(), err


@pytest.mark.slow
@pytest.mark.parametrize("test", [1, 2, 3])
def test_oracle_reproduces_golden_full(test):
    case = eci_test_case(test)
    out = OracleRun(case).run()["rec"]
    gold = np.load(os.path.join(GOLDEN, "rec_eci_test%d.npy" % test))
    err = _rel_l2(out, gold)
    assert (err < 5e-5).all(), err


def _energy_drift(case, nsteps=300, start=100):
    o = OracleRun(case, energy=True)
    e = np.array([o.step(n)[1] for n in range(nsteps)])[start:]
    return (e.max() - e.min()) / np.abs(e).mean()


def _small_energy_case(ratio):
    from ecsg_b200.workloads import ricker
    case = random_case(62, ratio=ratio, nx2=12, ny2=11, nz=(10, 8))
    n, h = case.grids[0]["n"], case.grids[0]["h"]
    case.src = {"xyz": (n[0] // 2 * h[0], n[1] // 2 * h[1], 2 * h[2]), "trace": ricker(60, case.dt * 5e-4, 15.0),
                "scale": 1000.0, "comp": 0}
    return case


@pytest.mark.parametrize("ratio", [2, 3])
def test_energy_exact_with_full_wall_mirrors(ratio):
    """With the vy wall mirrors covering the fine interface plane, the composite
    energy is conserved to round-off at ratio 2 and at the generalised ratio 3."""
    case = _small_energy_case(ratio)
    case.mirror_fix = True
    assert _energy_drift(case) < 1e-12


@needs_ref
def test_reference_wall_mirror_extent_leaks_energy():
    """The reference's vy y-wall mirrors run over vz's z-extent
    (update_vel.cpp:211-218, 239-246), one plane short of the fine grid's updated
    interface plane.  On a small two-grid case that leaks energy; the reference
    itself and the oracle agree step by step on the leaking energy."""
    from oracle.ref import RefRun
    case = _small_energy_case(2)
    assert _energy_drift(case) > 1e-6
    o = OracleRun(case, energy=True)
    r = RefRun(case, energy=True, threads=2)
    try:
        for n in range(150):
            eo = o.step(n)[1]
            er = r.step(n)[1]
            assert abs(eo - er) <= 1e-11 * abs(er)
    finally:
        r.close()


# ---------------------------------------------------------------------------
# Intuitive interpolation (imode 0)
# ---------------------------------------------------------------------------
@needs_ref
@pytest.mark.parametrize("seed,nx2,ny2", [(1, 6, 5), (2, 3, 7), (3, 2, 2), (4, 1, 3)])
def test_ii_operators_match_reference(seed, nx2, ny2):
    """update_ghost_{vz,sxz,syz}.cpp mode 0 on random fields (halos included):
    bitwise, including the far-column vz read past the end of the coarse rows."""
    from oracle.ref import RefRun
    case = random_case(seed, ratio=2, nx2=nx2, ny2=ny2, nz=(5, 4))
    case.imode = 0
    o = OracleRun(case)
    r = RefRun(case, threads=2)
    try:
        rng = np.random.default_rng(seed)
        for op in ("ghost_vz", "ghost_sxz", "ghost_syz"):
            _randomize(o, r, rng)
            getattr(o, op)(1)
            getattr(r, op)(1)
            assert _maxdiff(o, r) == 0.0, op
    finally:
        r.close()


@needs_ref
def test_ii_time_loop_matches_reference():
    from oracle.ref import RefRun
    from ecsg_b200.workloads import ricker
    case = random_case(11, ratio=2, nx2=8, ny2=6, nz=(6, 5))
    case.imode = 0
    h = case.grids[0]["h"][0]
    case.src = {"xyz": (8 * h, 6 * h, 2 * h), "trace": ricker(40, case.dt / 1000.0 * 20, 15.0), "scale": 1000.0,
                "comp": 0}
    case.rec = np.array([[5 * h, 6 * h, 2 * h], [9 * h, 3 * h, 5 * h], [10 * h, 4 * h, 8 * h]], dtype=np.float32)
    o = OracleRun(case, energy=True)
    r = RefRun(case, energy=True, threads=2)
    try:
        for n in range(25):
            rec_o, e_o, _ = o.step(n)
            rec_r, e_r = r.step(n)
            assert np.abs(rec_o - rec_r).max() <= 1e-12 * max(1.0, np.abs(rec_r).max())
            assert abs(e_o - e_r) <= 1e-12 * abs(e_r)
        assert _maxdiff(o, r) == 0.0
    finally:
        r.close()


def test_ii_oracle_reproduces_golden_prefix():
    """First 300 steps of the test1 II experiment against its golden traces."""
    n = 300
    case = eci_test_case(1, imode=0, nsteps=n)
    case.ii_skip_end_column = True
    out = OracleRun(case).run(n)["rec"]
    gold = np.load(os.path.join(GOLDEN, "rec_ii_test1.npy"))[:, :n]
    err = _rel_l2(out, gold)
    assert (err < 5e-5).all(), err


@pytest.mark.slow
@pytest.mark.parametrize("test", [1, 2, 3])
def test_oracle_reproduces_ii_golden_full(test):
    """The II goldens come from the revision of update_ghost_vz.cpp that left
    the last fine x column of vz ghosts untouched: with that variant the traces
    agree as closely as the ECI ones; with the current source they do not."""
    case = eci_test_case(test, imode=0)
    gold = np.load(os.path.join(GOLDEN, "rec_ii_test%d.npy" % test))
    case.ii_skip_end_column = True
    err = _rel_l2(OracleRun(case).run()["rec"], gold)
    assert (err < 5e-5).all(), err
    case.ii_skip_end_column = False
    err_now = _rel_l2(OracleRun(case).run()["rec"], gold)
    assert err_now.max() > 1e-4, err_now


def test_ii_energy_drifts_where_eci_is_flat():
    """The point of the reference's test1-cmp-eci-ii: after the source, the ECI
    energy is constant to round-off, the II energy is not."""
    drifts = {}
    for imode in (1, 0):
        case = _small_energy_case(2)
        case.mirror_fix = True
        case.imode = imode
        drifts[imode] = _energy_drift(case, nsteps=300)
    assert drifts[1] < 1e-12 and drifts[0] > 1e-3, drifts
