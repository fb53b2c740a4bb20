"""ecsg_ghost_sxz_noalloc against ecsg_ghost_sxz.

ecsg_ghost_sxz_noalloc is for callers that cannot allocate device memory: their
device memory belongs to another framework's allocator, or a fixed budget was
reserved up front.  Such a caller holds the two grids' fields itself and passes
them in; the solve's work space is a static device array inside the library.

Here torch plays that caller: it owns the field buffers, laid out in the
library's device layout and filled with the same random state as an ecsg_sim.
Two solves in a row (the second warm-started from the caller's X left by the
first, with the shared work space holding the first call's contents) must
match the allocating entry point within the tolerances of the other parity
tests (FP64 1e-12, FP32 2e-6 relative to the field scale).
"""
import ctypes

import numpy as np
import pytest

import ecsg_b200
from ecsg_b200 import XOFF, GridView, Simulation, device_layout, field_shape
from ecsg_b200.workloads import SIM_POS, random_case

pytestmark = pytest.mark.gpu


def _slices(n, R, arr_R, shape):
    l2, l1, l0 = shape
    o = R - arr_R
    return slice(o, o + l2), slice(o, o + l1), slice(XOFF - arr_R, XOFF - arr_R + l0)


def _to_device(torch, arr, n, R, arr_R, dtype):
    px, py, pz = device_layout(n, R)["pitch"]
    box = torch.zeros((pz, py, px), dtype=dtype)
    box[_slices(n, R, arr_R, arr.shape)] = torch.from_numpy(np.ascontiguousarray(arr)).to(dtype)
    return box.reshape(-1).cuda()


def _from_device(buf, n, R, shape):
    px, py, pz = device_layout(n, R)["pitch"]
    box = buf.detach().cpu().double().reshape(pz, py, px).numpy()
    return box[_slices(n, R, R, shape)]


def _view(g, bufs, buoy, R):
    v = GridView()
    v.size[:] = list(g["n"])
    v.step[:] = [float(h) for h in g["h"]]
    v.radius = R
    lay = device_layout(g["n"], R)
    v.pitch[:] = list(lay["pitch"])
    v.origin = lay["origin"]
    for k in range(9):
        v.field[k] = bufs[k].data_ptr()
    v.buoy = buoy.data_ptr()
    return v


@pytest.mark.parametrize("ratio", [2, 3])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_noalloc_matches_allocating_solve_twice(ratio, prec):
    torch = pytest.importorskip("torch")
    dtype = torch.float64 if prec == "f64" else torch.float32
    tol = 1e-12 if prec == "f64" else 2e-6
    case = random_case(100 + ratio, ratio=ratio, nx2=9, ny2=8, nz=(6, 5))
    R = case.radius
    rng = np.random.default_rng(7 * ratio + (prec == "f32"))
    L = ecsg_b200.lib()
    with Simulation(case, precision=prec) as sim:
        bufs, buoys = [], []
        for gi, g in enumerate(case.grids):
            bufs.append([])
            for k in range(9):
                a = rng.standard_normal(field_shape(g["n"], SIM_POS[k], R))
                if prec == "f32":
                    a = a.astype(np.float32).astype(np.float64)
                sim.set_field(gi, k, a)
                bufs[gi].append(_to_device(torch, a, g["n"], R, R, dtype))
            buoys.append(_to_device(torch, case.media[gi]["buoy"].astype(np.float64), g["n"], R, 0, dtype))
        views = [_view(g, bufs[gi], buoys[gi], R) for gi, g in enumerate(case.grids)]
        n2 = case.grids[1]["n"]
        X = torch.zeros((n2[0] + 1) * (n2[1] + 1), dtype=torch.float64, device="cuda")
        stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        err = ctypes.create_string_buffer(256)
        for call in range(2):
            if call == 1:
                # the same new state on both sides; X carries the warm start
                for gi, g in enumerate(case.grids):
                    for k in (0, 3, 7, 8):
                        a = rng.standard_normal(field_shape(g["n"], SIM_POS[k], R))
                        if prec == "f32":
                            a = a.astype(np.float32).astype(np.float64)
                        sim.set_field(gi, k, a)
                        bufs[gi][k].copy_(_to_device(torch, a, g["n"], R, R, dtype))
            sim.ghost_sxz(1)
            iters = ctypes.c_int(-1)
            rc = L.ecsg_ghost_sxz_noalloc(ctypes.byref(views[0]), ctypes.byref(views[1]), float(case.dt),
                                          ecsg_b200.ECSG_F64 if prec == "f64" else ecsg_b200.ECSG_F32,
                                          ctypes.c_void_p(X.data_ptr()), 0, stream, ctypes.byref(iters), err, 256)
            assert rc == ecsg_b200.ECSG_OK, err.value
            want_X, want_it, _, _ = sim.sxz_state(1)
            assert iters.value == want_it
            got_X = X.cpu().numpy()
            assert np.abs(got_X - want_X).max() <= tol * max(np.abs(want_X).max(), 1.0)
            for gi, g in enumerate(case.grids):
                for k in range(9):
                    want = sim.field(gi, k)
                    got = _from_device(bufs[gi][k], g["n"], R, want.shape)
                    assert np.abs(got - want).max() <= tol * np.abs(want).max(), (call, gi, k)


def test_noalloc_rejects_oversized_interface():
    L = ecsg_b200.lib()
    fine, coarse = GridView(), GridView()
    for v, n, h in ((fine, (800, 800, 10), 5.0), (coarse, (400, 400, 10), 10.0)):
        v.size[:] = list(n)
        v.step[:] = [h, h, h]
        v.radius = 1
    err = ctypes.create_string_buffer(256)
    dummy = ctypes.c_void_p(0x100)   # never dereferenced: the size check comes first
    rc = L.ecsg_ghost_sxz_noalloc(ctypes.byref(fine), ctypes.byref(coarse), 0.5, ecsg_b200.ECSG_F32, dummy, 0,
                                  None, None, err, 256)
    assert rc == -1 and b"exceeds the static work space" in err.value
