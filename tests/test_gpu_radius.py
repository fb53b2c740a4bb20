"""Stencil radius 2..6 on the device (stencil_r.cu) against the oracle, whose
radius loops are pinned bitwise to the reference (test_oracle.py).

* Each operator, FP64, single grid, isotropic and orthorhombic media, free and
  rigid top: bitwise equal over every entry of the 9 fields (halos included).
* 60-step runs with source, receivers and energy: FP64 traces at the float32
  output precision and energy to 1e-12; FP32 within 1e-5.
* The reference's own driver at radius 2 and 4 (one grid) through ecsg_main.
"""
import os

import numpy as np
import pytest

from ecsg_b200 import Simulation
from ecsg_b200.workloads import ortho9_from_cij21, random_case, random_case_gen21, ricker
from oracle.oracle import OracleRun

pytestmark = pytest.mark.gpu


def _case(radius, top_bc, medium, seed=3):
    if medium == "iso":
        case = random_case(seed, nx2=11, ny2=9, nz=(13,), num_grids=1, radius=radius, top_bc=top_bc)
    else:
        case = random_case_gen21(seed, nx2=11, ny2=9, nz=(13,), num_grids=1, top_bc=top_bc, aniso=0.3)
        for m in case.media:
            m["c9"] = ortho9_from_cij21(m["c21"])
        case.medium = "ortho9"
        case.radius = radius
    return case


@pytest.mark.parametrize("medium", ["iso", "ortho9"])
@pytest.mark.parametrize("top_bc", [1, 0])
@pytest.mark.parametrize("radius", [2, 3, 4, 5, 6])
def test_operators_f64_bitwise(radius, top_bc, medium):
    case = _case(radius, top_bc, medium)
    o = OracleRun(case)
    rng = np.random.default_rng(radius + 10 * top_bc)
    with Simulation(case, precision="f64") as s:
        for op in ("update_vel", "update_stress"):
            for k in range(9):
                a = rng.standard_normal(o.levels[0]["f"][k].shape)
                o.levels[0]["f"][k][...] = a
                s.set_field(0, k, a)
            getattr(o, op)(0)
            getattr(s, op)(0)
            for k in range(9):
                assert np.array_equal(o.levels[0]["f"][k], s.field(0, k)), (op, k)


def _with_src(case, nt):
    h, n = case.grids[0]["h"], case.grids[0]["n"]
    case.src = {"xyz": (n[0] // 2 * h[0], n[1] // 2 * h[1], 3 * h[2]), "trace": ricker(nt, case.dt * 1e-3, 15.0),
                "scale": 1000.0, "comp": 0}
    case.rec = np.array([[(n[0] // 2 + 3) * h[0], n[1] // 2 * h[1], 2 * h[2]],
                         [(n[0] - 1) * h[0], (n[1] // 3) * h[1], (n[2] - 1) * h[2]]], dtype=np.float32)
    return case


@pytest.mark.parametrize("prec", ["f64", "f32"])
@pytest.mark.parametrize("radius,top_bc", [(2, 1), (4, 0), (6, 1)])
def test_time_loop_vs_oracle(radius, top_bc, prec):
    nsteps = 60
    case = _with_src(_case(radius, top_bc, "iso", seed=5), nsteps)
    case.dt *= 0.7   # wider stencils: smaller stable step
    ref = OracleRun(case, energy=True).run(nsteps)
    with Simulation(case, precision=prec, energy=True) as s:
        out = s.run(nsteps, energy_every=1, graph=(prec == "f32"))
        assert s.status() == 0
    rel = np.linalg.norm(out["rec"] - ref["rec"], axis=1) / np.linalg.norm(ref["rec"], axis=1)
    erel = np.abs(out["energy"] - ref["energy"]).max() / np.abs(ref["energy"]).max()
    if prec == "f64":
        assert rel.max() < 1e-7 and erel < 1e-12, (rel, erel)
    else:
        assert rel.max() < 1e-5 and erel < 1e-5, (rel, erel)


@pytest.mark.parametrize("radius", [2, 4])
def test_reference_driver_at_radius(tmp_path, radius):
    from rsf_util import ECSG_MAIN, REF_MAIN, run_driver, write_inputs
    if not (os.path.exists(REF_MAIN) and os.path.exists(ECSG_MAIN)):
        pytest.skip("reference driver build or ecsg_main absent")
    tmp = str(tmp_path)
    case = _with_src(_case(radius, 1, "iso", seed=9), 40)
    args = [a if not a.startswith("radius=") else "radius=%d" % radius
            for a in write_inputs(tmp, case, 40, movie_every=4, movies=("vx",), verb=False)]
    ref, _ = run_driver(REF_MAIN, args, tmp, "ref", movies=("vx",), num_grids=1)
    got, _ = run_driver(ECSG_MAIN, args, tmp, "dev", movies=("vx",), num_grids=1, extra=["precision=f64"])
    r, g = ref["rec_out"][1], got["rec_out"][1]
    assert r.shape == g.shape and np.abs(r).max() > 0
    assert np.abs(g - r).max() <= 1e-6 * np.abs(r).max()
    e_r, e_g = ref["energy_trace"][1], got["energy_trace"][1]
    assert np.abs(e_g - e_r).max() <= 1e-10 * np.abs(e_r).max()
    a, b = ref["movie_vx_1"][1], got["movie_vx_1"][1]
    assert a.shape == b.shape and np.linalg.norm(a - b) <= 1e-6 * np.linalg.norm(a)
