"""RSF datasets for the driver tests: the inputs main.cpp reads (buoy_N,
s11_N, s13_N, src, rec_in) written from a workloads.Case, and a reader for
the outputs (header, then float32 samples after 0x0c 0x0c 0x04 or in the
in= file)."""
import os
import subprocess

import numpy as np

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
REF_MAIN = os.path.join(ROOT, "oracle", "_ref", "ecsg_ref_main")
SHIM_MAIN = os.path.join(ROOT, "oracle", "_ref", "ecsg_shim_main")
ECSG_MAIN = os.path.join(ROOT, "ecsg_b200", "_lib", "ecsg_main")


def write_rsf(path, data, separate=False, **hdr):
    """Header with the samples inline, or (separate=True) in path + '@' named by in=."""
    data = np.ascontiguousarray(data, dtype="<f4")
    with open(path, "wb") as fh:
        for k, v in hdr.items():
            fh.write(("%s=%s\n" % (k, repr(v) if isinstance(v, float) else v)).encode())
        if separate:
            fh.write(('data_format="native_float"\nesize=4\nin="%s@"\n' % path).encode())
        else:
            fh.write(b"\x0c\x0c\x04")
            fh.write(data.tobytes())
    if separate:
        with open(path + "@", "wb") as fh:
            fh.write(data.tobytes())


def read_rsf(path):
    raw = open(path, "rb").read()
    i = raw.find(b"\x0c\x0c\x04")
    text = raw[:i].decode() if i >= 0 else raw.decode()
    hdr = {}
    for tok in text.split():
        if "=" in tok:
            k, v = tok.split("=", 1)
            hdr[k] = v.strip('"')
    if i >= 0:
        data = np.frombuffer(raw[i + 3:], dtype="<f4")
    else:
        data = np.fromfile(hdr["in"], dtype="<f4")
    return hdr, data


def write_inputs(tmp, case, nsteps, imode=1, separate=False, movie_every=None, movies=(), verb=True):
    """Files and key=value arguments of main.cpp for a case.  The run has
    nsteps steps (nt = ceil(movie_dt * movie_nt / dt) + 1); with movie_every=k
    a frame is printed every k steps."""
    args = []
    for gi, g in enumerate(case.grids):
        n, h = g["n"], g["h"]
        for key in ("buoy", "s11", "s13"):
            p = os.path.join(tmp, "%s_%d.rsf" % (key, gi + 1))
            write_rsf(p, case.media[gi][key], separate, n1=n[0] + 1, n2=n[1] + 1, n3=n[2] + 1,
                      d1=float(h[0]), d2=float(h[1]), d3=float(h[2]))
            args.append("%s_%d=%s" % (key, gi + 1, p))
    x, y, z = case.src["xyz"]
    tr = np.asarray(case.src["trace"], np.float32)
    write_rsf(os.path.join(tmp, "src.rsf"), tr, separate, n1=tr.size, d1=float(case.dt) / 1000.0,
              o2=float(x), o3=float(y), o4=float(z))
    write_rsf(os.path.join(tmp, "rec.rsf"), case.rec, separate, n1=3, n2=len(case.rec))
    if movie_every:
        movie_dt, movie_nt = float(case.dt) * movie_every, (nsteps - 1) // movie_every
    else:
        movie_dt, movie_nt = float(case.dt), nsteps - 1
    args += ["src=" + os.path.join(tmp, "src.rsf"), "rec_in=" + os.path.join(tmp, "rec.rsf"),
             "num_threads=4", "num_grids=%d" % len(case.grids), "radius=1", "dt=%r" % float(case.dt),
             "imode=%d" % imode, "top_bc=%d" % case.top_bc, "check_energy=y", "verb=%s" % ("y" if verb else "n"),
             "movie_dt=%r" % movie_dt, "movie_nt=%d" % movie_nt]
    args += ["movie_%s_flag=y" % m for m in movies]
    return args


def run_driver(exe, args, tmp, tag, movies=(), num_grids=2, extra=()):
    outs = {k: os.path.join(tmp, "%s_%s.rsf" % (tag, k)) for k in ("rec_out", "energy_trace", "res_trace")}
    for m in movies:
        for g in range(num_grids):
            outs["movie_%s_%d" % (m, g + 1)] = os.path.join(tmp, "%s_movie_%s_%d.rsf" % (tag, m, g + 1))
    cmd = [exe] + list(args) + ["%s=%s" % (k, v) for k, v in outs.items()] + list(extra)
    proc = subprocess.run(cmd, check=True, cwd=tmp, stdout=subprocess.PIPE, stderr=subprocess.PIPE, timeout=600)
    res = {k: read_rsf(v) for k, v in outs.items() if os.path.exists(v)}
    return res, proc.stdout.decode()
