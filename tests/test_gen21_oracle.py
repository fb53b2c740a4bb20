"""The 21-Cij stress update (no reference counterpart, oracle/ecsg_oracle.c
o_update_stress21) is pinned two ways: it reduces to the reference's
orthorhombic update when the 12 off-block entries vanish, and it conserves the
discrete energy 1/2 (rho v, v') + 1/2 (eps, sigma) to round-off with all 21
entries present, on single grids and on composites at ratio 2 and 3."""
import copy

import numpy as np
import pytest

from ecsg_b200.workloads import ortho9_from_cij21, random_case_gen21, ricker
from oracle.oracle import OracleRun


@pytest.mark.parametrize("top_bc", [0, 1])
def test_reduces_to_orthorhombic_update(top_bc):
    case = random_case_gen21(3, ratio=2, nx2=6, ny2=5, nz=(5, 4), top_bc=top_bc)
    for m in case.media:
        for k in list(range(6, 15)) + [16, 17, 19]:
            m["c21"][k] = np.zeros_like(m["c21"][k])
        m["c9"] = ortho9_from_cij21(m["c21"])
    o21 = OracleRun(case)
    c9 = copy.copy(case)
    c9.medium = "ortho9"
    o9 = OracleRun(c9)
    rng = np.random.default_rng(top_bc)
    for g in range(2):
        for k in range(9):
            a = rng.standard_normal(o21.levels[g]["f"][k].shape)
            o21.levels[g]["f"][k][...] = a
            o9.levels[g]["f"][k][...] = a
    for g in range(2):
        o21.update_stress(g)
        o9.update_stress(g)
    for g in range(2):
        for k in range(9):
            a, b = o21.levels[g]["f"][k], o9.levels[g]["f"][k]
            assert np.abs(a - b).max() <= 1e-14 * np.abs(b).max(), (g, k)


@pytest.mark.parametrize("ng,ratio,top_bc", [(1, 2, 1), (1, 2, 0), (2, 2, 1), (2, 3, 1), (2, 3, 0)])
def test_energy_conserved(ng, ratio, top_bc):
    nz = (8, 6) if ng == 2 else (10,)
    case = random_case_gen21(5, ratio=ratio, nx2=8, ny2=7, nz=nz, num_grids=ng, top_bc=top_bc, aniso=0.3)
    n, h = case.grids[0]["n"], case.grids[0]["h"]
    case.src = {"xyz": (n[0] // 2 * h[0], n[1] // 2 * h[1], 2 * h[2]), "trace": ricker(60, case.dt * 5e-4, 15.0),
                "scale": 1000.0, "comp": 0}
    case.mirror_fix = True
    o = OracleRun(case, energy=True)
    e = np.array([o.step(k)[1] for k in range(300)])[100:]
    assert (e.max() - e.min()) / np.abs(e).mean() < 1e-12
