"""The drop-in: the reference's own driver (main.cpp) linked with
ecsg_b200/shim/sim_utils_shim.cpp in place of its hot-path sources
(oracle/_ref/ecsg_shim_main) against the same driver built unmodified
(oracle/_ref/ecsg_ref_main), on the same RSF inputs and command line.

The FP64 device operators reproduce the reference's stencil rounding and
solve the interfaces to its tolerance, so the receiver traces (float32, as
the driver writes them) agree to one float rounding, the energy to 1e-10 and
the interface residues to the float precision of their traces.
"""
import os

import numpy as np
import pytest

from ecsg_b200.workloads import random_case, ricker
from rsf_util import REF_MAIN, SHIM_MAIN, run_driver, write_inputs

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("top_bc,imode", [(1, 1), (0, 1), (1, 0)])
def test_reference_driver_through_the_shim(tmp_path, top_bc, imode):
    if not (os.path.exists(REF_MAIN) and os.path.exists(SHIM_MAIN)):
        pytest.skip("reference driver builds absent (built from the reference sources by __graft_entry__.build)")
    case = random_case(71 + top_bc, ratio=2, nx2=14, ny2=12, nz=(10, 8), top_bc=top_bc)
    n, h = case.grids[0]["n"], case.grids[0]["h"]
    nsteps = 40
    case.src = {"xyz": (n[0] // 2 * h[0], n[1] // 2 * h[1], 3 * h[2]), "trace": ricker(nsteps, case.dt * 1e-3 * 0.5, 15.0),
                "scale": 1000.0, "comp": 0}
    case.rec = np.array([[(n[0] // 2 + 3) * h[0], n[1] // 2 * h[1], 3 * h[2]],
                         [(n[0] // 3) * h[0], (n[1] // 3) * h[1], (n[2] - 1) * h[2]],
                         [(n[0] // 2) * h[0], (n[1] // 2) * h[1], (n[2] + 3) * h[2]]], dtype=np.float32)
    args = write_inputs(str(tmp_path), case, nsteps, imode)
    ref = {k: v[1] for k, v in run_driver(REF_MAIN, args, str(tmp_path), "ref")[0].items()}
    got = {k: v[1] for k, v in run_driver(SHIM_MAIN, args, str(tmp_path), "shim")[0].items()}
    assert ref["rec_out"].size == 3 * nsteps and np.abs(ref["rec_out"]).max() > 0
    assert np.abs(got["rec_out"] - ref["rec_out"]).max() <= 1e-6 * np.abs(ref["rec_out"]).max()
    assert np.abs(got["energy_trace"] - ref["energy_trace"]).max() <= 1e-10 * np.abs(ref["energy_trace"]).max() + 1e-30
    res_ref, res_got = ref["res_trace"].reshape(9, -1), got["res_trace"].reshape(9, -1)
    for j in range(9):
        scale = max(np.abs(res_ref[j]).max(), np.abs(res_ref[3 * (j // 3) + 1]).max(), 1e-30)
        assert np.abs(res_got[j] - res_ref[j]).max() <= 1e-5 * scale, j
