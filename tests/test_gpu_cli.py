"""ecsg_main (the reference's command line on the device) against the
reference's own driver (oracle/_ref/ecsg_ref_main) on the same RSF inputs:
receiver traces, energy trace, interface residues and vx/vz movies of both
grids, in both interface modes.

precision=f64 follows the reference's double build: traces and movie frames
(float32 in the files) agree to one float rounding, the energy to 1e-10, the
residues to the float precision of their traces.  precision=f32 (the default)
is held to 1e-5 rel-L2 on the traces and movies.
"""
import os

import numpy as np
import pytest

from ecsg_b200.workloads import random_case, ricker
from rsf_util import ECSG_MAIN, REF_MAIN, run_driver, write_inputs

pytestmark = pytest.mark.gpu
MOVIES = ("vx", "vz")


def _case(top_bc, nsteps):
    case = random_case(91 + top_bc, ratio=2, nx2=14, ny2=12, nz=(10, 8), top_bc=top_bc)
    n, h = case.grids[0]["n"], case.grids[0]["h"]
    case.src = {"xyz": (n[0] // 2 * h[0], n[1] // 2 * h[1], 3 * h[2]), "trace": ricker(nsteps, case.dt * 1e-3 * 0.5, 15.0),
                "scale": 1000.0, "comp": 0}
    case.rec = np.array([[(n[0] // 2 + 3) * h[0], n[1] // 2 * h[1], 3 * h[2]],
                         [(n[0] - 1) * h[0], (n[1] // 3) * h[1], (n[2] - 1) * h[2]],
                         [(n[0] // 2) * h[0], (n[1] // 2) * h[1], (n[2] + 3) * h[2]]], dtype=np.float32)
    return case


@pytest.mark.parametrize("precision", ["f64", "f32"])
@pytest.mark.parametrize("top_bc,imode", [(1, 1), (0, 1), (1, 0)])
def test_cli_matches_the_reference_driver(tmp_path, top_bc, imode, precision):
    if not (os.path.exists(REF_MAIN) and os.path.exists(ECSG_MAIN)):
        pytest.skip("reference driver build or ecsg_main absent")
    tmp = str(tmp_path)
    case = _case(top_bc, 46)
    args = write_inputs(tmp, case, 46, imode, movie_every=5, movies=MOVIES)
    ref, _ = run_driver(REF_MAIN, args, tmp, "ref", movies=MOVIES)
    got, stdout = run_driver(ECSG_MAIN, args, tmp, "dev", movies=MOVIES, extra=["precision=" + precision])
    assert "Total elapsed time" in stdout
    assert set(got) == set(ref)
    for key in ref:
        hr, hg = ref[key][0], got[key][0]
        for k in ("n1", "n2", "n3", "n4"):
            assert hr.get(k) == hg.get(k), (key, k)
        assert ref[key][1].shape == got[key][1].shape, key
    r, g = ref["rec_out"][1].reshape(3, -1), got["rec_out"][1].reshape(3, -1)
    assert np.abs(r).max() > 0
    e_r, e_g = ref["energy_trace"][1], got["energy_trace"][1]
    if precision == "f64":
        assert np.abs(g - r).max() <= 1e-6 * np.abs(r).max()
        assert np.abs(e_g - e_r).max() <= 1e-10 * np.abs(e_r).max() + 1e-30
        res_r, res_g = ref["res_trace"][1].reshape(9, -1), got["res_trace"][1].reshape(9, -1)
        for j in range(9):
            scale = max(np.abs(res_r[j]).max(), np.abs(res_r[3 * (j // 3) + 1]).max(), 1e-30)
            assert np.abs(res_g[j] - res_r[j]).max() <= 1e-5 * scale, j
    else:
        assert (np.linalg.norm(g - r, axis=1) <= 1e-5 * np.linalg.norm(r, axis=1)).all()
        assert np.abs(e_g - e_r).max() <= 1e-5 * np.abs(e_r).max()
    for m in MOVIES:
        for gi in (1, 2):
            key = "movie_%s_%d" % (m, gi)
            a, b = ref[key][1], got[key][1]
            assert a.size > 0 and np.abs(a).max() > 0, key
            tol = 1e-6 if precision == "f64" else 1e-5
            assert np.linalg.norm(a - b) <= tol * np.linalg.norm(a), key


def test_cli_separate_data_files(tmp_path):
    """Inputs with in= data files, outputs written under datapath=."""
    if not (os.path.exists(REF_MAIN) and os.path.exists(ECSG_MAIN)):
        pytest.skip("reference driver build or ecsg_main absent")
    tmp = str(tmp_path)
    case = _case(1, 25)
    args = write_inputs(tmp, case, 25, separate=True, movie_every=4, movies=("vz",))
    ref, _ = run_driver(REF_MAIN, args, tmp, "ref", movies=("vz",))
    os.makedirs(os.path.join(tmp, "data"))
    got, _ = run_driver(ECSG_MAIN, args, tmp, "dev", movies=("vz",),
                        extra=["precision=f64", "datapath=" + os.path.join(tmp, "data")])
    assert os.listdir(os.path.join(tmp, "data"))
    for key in ("rec_out", "movie_vz_1", "movie_vz_2"):
        a, b = ref[key][1], got[key][1]
        assert a.shape == b.shape and np.abs(a - b).max() <= 1e-6 * np.abs(a).max(), key


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_frame_is_the_field_domain(precision):
    from ecsg_b200 import Simulation
    case = _case(1, 20)
    with Simulation(case, precision=precision) as s:
        s.run(20)
        for g in range(2):
            for k in range(9):
                f = s.field(g, k)
                fr = s.frame(g, k)
                R = case.radius
                want = f[R:R + fr.shape[0], R:R + fr.shape[1], R:R + fr.shape[2]].astype(np.float32)
                assert fr.shape == tuple(d - 2 * R for d in f.shape)
                assert np.array_equal(fr, want), (g, k)


@pytest.mark.parametrize("precision", ["f32", "f64"])
def test_checkpoint_and_resume_match_an_uninterrupted_run(tmp_path, precision):
    """stop_after + checkpoint, then resume: rec_out, energy_trace and
    res_trace bitwise equal to one uninterrupted run; a checkpoint from a
    different set-up is refused."""
    if not os.path.exists(ECSG_MAIN):
        pytest.skip("ecsg_main absent")
    import subprocess
    tmp = str(tmp_path)
    case = _case(1, 41)
    args = write_inputs(tmp, case, 41)
    extra = ["precision=" + precision]
    full, _ = run_driver(ECSG_MAIN, args, tmp, "full", extra=extra)
    ck = os.path.join(tmp, "state.ckpt")
    _, out1 = run_driver(ECSG_MAIN, args, tmp, "part", extra=extra + ["checkpoint=" + ck, "checkpoint_every=7",
                                                                       "stop_after=17"])
    assert "Stopped after step 16" in out1 and os.path.exists(ck)
    resumed, out2 = run_driver(ECSG_MAIN, args, tmp, "res", extra=extra + ["resume=" + ck])
    assert "Resumed after step 16" in out2
    for key in ("rec_out", "energy_trace", "res_trace"):
        assert np.array_equal(full[key][1], resumed[key][1]), key
    # another precision is another set-up
    other = "f64" if precision == "f32" else "f32"
    cmd = [ECSG_MAIN] + args + ["rec_out=" + os.path.join(tmp, "x.rsf"), "precision=" + other, "resume=" + ck]
    p = subprocess.run(cmd, cwd=tmp, stdout=subprocess.PIPE, stderr=subprocess.PIPE, timeout=300)
    assert p.returncode != 0 and b"precision" in p.stderr


@pytest.mark.parametrize("medium", ["iso", "gen21"])
def test_save_and_load_state_continue_bit_for_bit(medium):
    from ecsg_b200 import Simulation
    from ecsg_b200.workloads import random_case_gen21
    if medium == "iso":
        case = _case(1, 30)
    else:
        case = random_case_gen21(8, ratio=2, nx2=10, ny2=9, nz=(8, 6), aniso=0.3)
        n, h = case.grids[0]["n"], case.grids[0]["h"]
        case.src = {"xyz": (n[0] // 2 * h[0], n[1] // 2 * h[1], 2 * h[2]), "trace": ricker(30, case.dt * 1e-3, 15.0),
                    "scale": 1000.0, "comp": 0}
        case.rec = np.array([[(n[0] // 2 + 2) * h[0], n[1] // 2 * h[1], 2 * h[2]]], dtype=np.float32)
    with Simulation(case, precision="f32", energy=True) as s:
        whole = s.run(30, energy_every=5)
    with Simulation(case, precision="f32", energy=True) as s:
        first = s.run(12, energy_every=5)
        state = s.save_state()
    with Simulation(case, precision="f32", energy=True) as s:
        s.load_state(state, step_index=12)
        second = s.run(18, energy_every=5)
    assert np.array_equal(whole["rec"], np.concatenate([first["rec"], second["rec"]], axis=1))
    assert np.array_equal(whole["energy"][12:], second["energy"], equal_nan=True)
