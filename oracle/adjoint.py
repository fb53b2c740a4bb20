"""FP64 CPU adjoint of the oracle's time loop (adjoint_ad.cpp).  TEST
INFRASTRUCTURE ONLY.

misfit_gradient(case, observed) runs the oracle's own C restatement of the
loop (main.cpp:165-261 order, as OracleRun.step) over observed.shape[0] steps
from rest with its arithmetic recorded on a tape, and returns the misfit
L = 1/2 sum (v_rec - observed)^2 with its exact reverse-mode gradient with
respect to the node buoyancy and the 21 stiffness slots of every grid: the
layout of the device's ecsg_get_gradient (which = 0: buoyancy, 1 + k: slot k).
21-Cij media (random_case_gen21 / tti_as_gen21 cases), radius 1, ECI mode.
"""
import ctypes
import os

import numpy as np

from oracle.oracle import fd_coeff, locate

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None
c_dp = ctypes.POINTER(ctypes.c_double)
c_fp = ctypes.POINTER(ctypes.c_float)
c_ip = ctypes.POINTER(ctypes.c_int)


class ADGrid(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int * 3), ("coeff", ctypes.c_double * 3), ("buoy", c_dp), ("c21", c_dp * 21),
                ("g_buoy", c_dp), ("g_c21", c_dp * 21)]


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "_build", "libecsg_oracle_ad.so")
        if not os.path.exists(path):
            raise RuntimeError("differentiated oracle missing: run `make -C oracle oracle`")
        L = ctypes.CDLL(path)
        L.ad_misfit_gradient.restype = ctypes.c_int
        L.ad_misfit_gradient.argtypes = [ctypes.c_int, ctypes.POINTER(ADGrid), ctypes.c_int, ctypes.c_int,
                                         ctypes.c_int, ctypes.c_int, c_ip, c_fp, ctypes.c_int, ctypes.c_float,
                                         ctypes.c_int, c_ip, ctypes.c_int, c_fp, ctypes.c_int, c_dp,
                                         ctypes.POINTER(ctypes.c_longlong)]
        _LIB = L
    return _LIB


def misfit_gradient(case, observed, jacobi_min_sweeps=200):
    """Returns (loss, grads, tape_len): grads[g][0] = dL/d buoyancy at the nodes,
    grads[g][1 + k] = dL/d slot k at CIJ21_POS[k], each without halo."""
    if case.medium != "gen21" or case.radius != 1 or case.imode != 1:
        raise ValueError("the differentiated oracle runs 21-Cij media at radius 1 in ECI mode")
    obs = np.ascontiguousarray(observed, dtype=np.float32)
    nsteps = obs.shape[0]
    ng = len(case.grids)
    fd = fd_coeff(1)
    keep = []
    grids = (ADGrid * ng)()
    grads = []
    for g, grid in enumerate(case.grids):
        n, h = grid["n"], grid["h"]
        m = case.media[g]
        G = grids[g]
        G.n[:] = list(n)
        G.coeff[:] = [fd[0] * case.dt / h[d] for d in range(3)]
        b = np.ascontiguousarray(m["buoy"], dtype=np.float64)
        cs = [np.ascontiguousarray(c, dtype=np.float64) for c in m["c21"]]
        gb = np.zeros_like(b)
        gc = [np.zeros_like(c) for c in cs]
        keep += [b, gb] + cs + gc
        G.buoy = b.ctypes.data_as(c_dp)
        G.g_buoy = gb.ctypes.data_as(c_dp)
        for k in range(21):
            G.c21[k] = cs[k].ctypes.data_as(c_dp)
            G.g_c21[k] = gc[k].ctypes.data_as(c_dp)
        grads.append([gb] + gc)
    origins, z0 = [], 0.0
    for grid in case.grids:
        origins.append((0.0, 0.0, z0))
        z0 += grid["n"][2] * grid["h"][2]
    src = None
    trace = np.zeros(1, np.float32)
    if case.src is not None:
        g, ix, iy, iz = locate(case.src["xyz"], case.grids, origins)
        src = (ctypes.c_int * 5)(g, ix, iy, iz, int(case.src.get("comp", 0)))
        trace = np.ascontiguousarray(case.src["trace"], dtype=np.float32)
    rec = np.array([locate(p, case.grids, origins) for p in case.rec], dtype=np.int32).reshape(-1, 4)
    rec = np.ascontiguousarray(rec)
    loss = ctypes.c_double()
    tape = ctypes.c_longlong()
    rc = lib().ad_misfit_gradient(ng, grids, case.ratio, case.top_bc, int(getattr(case, "mirror_fix", False)), nsteps,
                                  src, trace.ctypes.data_as(c_fp), len(trace) if src is not None else 0,
                                  float(case.src["scale"]) if src is not None else 0.0, len(rec),
                                  rec.ctypes.data_as(c_ip), int(getattr(case, "rec_comp", 0)),
                                  obs.ctypes.data_as(c_fp), int(jacobi_min_sweeps), ctypes.byref(loss),
                                  ctypes.byref(tape))
    if rc != 0:
        raise ValueError("ad_misfit_gradient: %s" % ("bad arguments" if rc == -1 else "tape too long"))
    return loss.value, grads, tape.value
