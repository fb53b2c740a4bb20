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


def _strains_of_sums(U, k, n):
    """e1..e6 at the stress positions (R = 0 layout of the accumulators) as the
    strain differences (e*_at of the oracle) of velocity sums U with halo 1."""
    nx, ny, nz = n
    ux, uy, uz = U
    k0, k1, k2 = k
    e1 = k0 * (ux[1:nz + 2, 1:ny + 2, 2:nx + 2] - ux[1:nz + 2, 1:ny + 2, 1:nx + 1])
    e2 = k1 * (uy[1:nz + 2, 1:ny + 2, 1:nx + 1] - uy[1:nz + 2, 0:ny + 1, 1:nx + 1])
    e3 = k2 * (uz[1:nz + 2, 1:ny + 2, 1:nx + 1] - uz[0:nz + 1, 1:ny + 2, 1:nx + 1])
    e4 = k2 * (uy[2:nz + 2, 1:ny + 1, 1:nx + 1] - uy[1:nz + 1, 1:ny + 1, 1:nx + 1]) \
        + k1 * (uz[1:nz + 1, 2:ny + 2, 1:nx + 1] - uz[1:nz + 1, 1:ny + 1, 1:nx + 1])
    e5 = k2 * (ux[2:nz + 2, 1:ny + 2, 1:nx + 2] - ux[1:nz + 1, 1:ny + 2, 1:nx + 2]) \
        + k0 * (uz[1:nz + 1, 1:ny + 2, 1:nx + 2] - uz[1:nz + 1, 1:ny + 2, 0:nx + 1])
    e6 = k1 * (ux[1:nz + 2, 2:ny + 2, 1:nx + 2] - ux[1:nz + 2, 1:ny + 1, 1:nx + 2]) \
        + k0 * (uy[1:nz + 2, 1:ny + 1, 1:nx + 2] - uy[1:nz + 2, 1:ny + 1, 0:nx + 1])
    return [e1, e2, e3, e4, e5, e6]


@pytest.mark.parametrize("ratio,top_bc", [(2, 1), (3, 0)])
def test_accumulated_strains_are_strains_of_summed_velocities(ratio, top_bc):
    """The device keeps the velocities summed over the stress updates (three
    displacement sums) instead of six strain accumulators, and forms the
    strains at energy steps.  Here, on the oracle: the strain differences of
    the summed velocities equal the oracle's accumulated strains at every
    stress position of both grids, except the free-surface e3 (a condensed
    value), which the energy pairs with szz, held at 0 there; so the energy
    1/2 (eps, sigma) is the same."""
    case = random_case_gen21(17 + ratio, ratio=ratio, nx2=7, ny2=6, nz=(7, 5), top_bc=top_bc, aniso=0.3)
    n, h = case.grids[0]["n"], case.grids[0]["h"]
    case.src = {"xyz": (n[0] // 2 * h[0], n[1] // 2 * h[1], 2 * h[2]), "trace": ricker(40, case.dt * 1e-3, 15.0),
                "scale": 1000.0, "comp": 0}
    o = OracleRun(case, energy=True)
    U = [[np.zeros_like(o.levels[g]["f"][c]) for c in range(3)] for g in range(2)]
    update_stress = o.update_stress

    def summing_update_stress(g):
        for c in range(3):
            U[g][c] += o.levels[g]["f"][c]
        return update_stress(g)

    o.update_stress = summing_update_stress
    for step in range(40):
        o.step(step)
    for g in range(2):
        L = o.levels[g]
        es = _strains_of_sums(U[g], L["coeff"][:, 0], case.grids[g]["n"])
        for j in range(6):
            a, b = es[j], L["eps"][j]
            assert a.shape == b.shape, (g, j)
            if j == 2 and g == 0 and top_bc:
                a, b = a[1:], b[1:]
            assert np.abs(a - b).max() <= 1e-12 * np.abs(b).max(), (g, j)
        if top_bc and g == 0:
            assert np.abs(L["f"][5][1, 1:-1, 1:-1]).max() == 0.0   # szz on the free surface stays 0
