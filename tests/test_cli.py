"""The command-line driver (ecsg_b200/_lib/ecsg_main) without a GPU: it reads
the reference's RSF inputs (samples inline or in in= files) and its key=value
parameters, and with dryrun=y prints the set-up without touching the device.

Against the reference's own driver (oracle/_ref/ecsg_ref_main, run here on the
CPU): the same source and receiver lines on stdout and one movie frame per
step that main.cpp prints one at.
"""
import os
import subprocess

import numpy as np
import pytest

from ecsg_b200.workloads import random_case, ricker
from oracle.oracle import OracleRun
from rsf_util import ECSG_MAIN, REF_MAIN, read_rsf, run_driver, write_inputs, write_rsf

needs_cli = pytest.mark.skipif(not os.path.exists(ECSG_MAIN), reason="ecsg_main not built (ecsg_b200.build)")


def _case(nsteps=31):
    case = random_case(17, ratio=2, nx2=9, ny2=7, nz=(6, 5))
    n, h = case.grids[0]["n"], case.grids[0]["h"]
    case.src = {"xyz": (n[0] // 2 * h[0], n[1] // 2 * h[1], 2.4 * h[2]), "trace": ricker(nsteps, case.dt * 1e-3, 15.0),
                "scale": 1000.0, "comp": 0}
    z1 = n[2] * h[2]
    case.rec = np.array([[3.6 * h[0], 2 * h[1], 1.5 * h[2]],       # rounds half away from zero
                         [(n[0] - 1) * h[0], 5 * h[1], z1],          # on the interface: fine grid
                         [4 * h[0], 3 * h[1], z1 + 0.01],            # just below: coarse grid
                         [7 * h[0], 6 * h[1], z1 + 3 * case.grids[1]["h"][2]]], dtype=np.float32)
    return case


def _dry(args, tmp):
    out = subprocess.run([ECSG_MAIN] + args + ["dryrun=y", "rec_out=" + os.path.join(tmp, "r.rsf")],
                         check=True, stdout=subprocess.PIPE, timeout=120, cwd=tmp).stdout.decode()
    return out


@needs_cli
@pytest.mark.parametrize("separate", [False, True])
def test_dryrun_locations_match_the_oracle(tmp_path, separate):
    case = _case()
    args = write_inputs(str(tmp_path), case, 31, separate=separate)
    out = _dry(args, str(tmp_path))
    o = OracleRun(case)
    lines = out.splitlines()
    i = lines.index("== Source is placed at... ")
    g, ix, iy, iz = o.src
    assert lines[i + 1] == "(grid#%d, ix=%d, iy=%d, iz=%d)" % (g, ix, iy, iz)
    j = lines.index("== Record traces at... ")
    for k, (g, ix, iy, iz) in enumerate(o.rec):
        assert lines[j + 1 + k] == "(grid#%d, ix=%d,  iy=%d, iz=%d)" % (g, ix, iy, iz)
    assert "grid_1 size 18 14 6" in out and "grid_2 size 9 7 5" in out


@needs_cli
def test_missing_and_malformed_inputs_fail_with_a_message(tmp_path):
    case = _case()
    args = write_inputs(str(tmp_path), case, 31)
    bad = [a for a in args if not a.startswith("s13_2=")]
    p = subprocess.run([ECSG_MAIN] + bad + ["dryrun=y"], stdout=subprocess.PIPE, stderr=subprocess.PIPE, timeout=60)
    assert p.returncode != 0 and b"s13_2" in p.stderr
    # a medium whose size disagrees with the buoyancy
    m = case.media[1]["s11"][:-1]
    n, h = case.grids[1]["n"], case.grids[1]["h"]
    write_rsf(os.path.join(str(tmp_path), "s11_2.rsf"), m, n1=n[0] + 1, n2=n[1] + 1, n3=n[2], d1=h[0], d2=h[1], d3=h[2])
    p = subprocess.run([ECSG_MAIN] + args + ["dryrun=y"], stdout=subprocess.PIPE, stderr=subprocess.PIPE, timeout=60)
    assert p.returncode != 0 and b"size differs" in p.stderr
    p = subprocess.run([ECSG_MAIN] + [a for a in args if not a.startswith("dt=")] + ["dryrun=y"],
                       stdout=subprocess.PIPE, stderr=subprocess.PIPE, timeout=60)
    assert p.returncode != 0 and b"dt" in p.stderr


@needs_cli
@pytest.mark.skipif(not os.path.exists(REF_MAIN), reason="reference driver build (oracle/_ref) absent")
@pytest.mark.parametrize("every", [1, 3, 7])
def test_set_up_and_frames_match_the_reference_driver(tmp_path, every):
    """The reference's driver itself (CPU): same location lines on stdout, and
    as many movie frames as ecsg_main schedules."""
    case = _case()
    tmp = str(tmp_path)
    args = write_inputs(tmp, case, 31, movie_every=every, movies=("vz",), verb=False)
    outs, ref_stdout = run_driver(REF_MAIN, args, tmp, "ref", movies=("vz",))
    dry = _dry(args, tmp)
    ref_lines = [l for l in ref_stdout.splitlines() if l.startswith("(grid#") or l.startswith("== ")]
    dry_lines = [l for l in dry.splitlines() if l.startswith("(grid#") or l.startswith("== Source") or l.startswith("== Record")]
    assert ref_lines == dry_lines
    steps = [l for l in dry.splitlines() if l.startswith("== Steps")][0]
    nsteps = int(steps.split()[2].rstrip(","))
    nframes = int(steps.split()[4].rstrip(":"))
    hdr, rec = outs["rec_out"]
    assert int(hdr["n1"]) == nsteps
    for g in range(2):
        mh, mv = outs["movie_vz_%d" % (g + 1)]
        frame = int(mh["n1"]) * int(mh["n2"]) * int(mh["n3"])
        assert mv.size == nframes * frame
