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
tests (FP64 1e-12, FP32 2e-6 relative to the field scale), and the second call
must leave the device's free memory unchanged.  The argument checks run
without a GPU; the solve, the sweep cap and the sticky status word need one.
"""
import ctypes

import numpy as np
import pytest

import ecsg_b200
from ecsg_b200 import XOFF, GridView, Simulation, device_layout, field_shape
from ecsg_b200.workloads import SIM_POS, random_case

ERR_INVALID, ERR_NOT_CONVERGED = -1, -5
ST_JACOBI_CAP = 1


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


class _Setup:
    """An ecsg_sim and torch-owned copies of the same random two-grid state."""

    def __init__(self, torch, ratio, prec, seed):
        self.torch, self.prec = torch, prec
        self.dtype = torch.float64 if prec == "f64" else torch.float32
        self.case = case = random_case(100 + ratio, ratio=ratio, nx2=9, ny2=8, nz=(6, 5))
        self.R = R = case.radius
        self.rng = np.random.default_rng(seed)
        self.sim = Simulation(case, precision=prec)
        self.bufs, buoys = [], []
        for gi, g in enumerate(case.grids):
            self.bufs.append([])
            for k in range(9):
                a = self.field_values(g, k)
                self.sim.set_field(gi, k, a)
                self.bufs[gi].append(_to_device(torch, a, g["n"], R, R, self.dtype))
            buoys.append(_to_device(torch, case.media[gi]["buoy"].astype(np.float64), g["n"], R, 0, self.dtype))
        self.buoys = buoys
        self.views = [_view(g, self.bufs[gi], buoys[gi], R) for gi, g in enumerate(case.grids)]
        n2 = case.grids[1]["n"]
        self.X = torch.zeros((n2[0] + 1) * (n2[1] + 1), dtype=torch.float64, device="cuda")
        self.stream = ctypes.c_void_p(torch.cuda.current_stream().cuda_stream)
        self.err = ctypes.create_string_buffer(256)

    def field_values(self, g, k):
        a = self.rng.standard_normal(field_shape(g["n"], SIM_POS[k], self.R))
        return a.astype(np.float32).astype(np.float64) if self.prec == "f32" else a

    def new_state(self):
        """The same new velocities and sxx/sxz/sxy on both sides."""
        for gi, g in enumerate(self.case.grids):
            for k in (0, 3, 7, 8):
                a = self.field_values(g, k)
                self.sim.set_field(gi, k, a)
                self.bufs[gi][k].copy_(_to_device(self.torch, a, g["n"], self.R, self.R, self.dtype))

    def call(self, max_iter=0, iters=None):
        return ecsg_b200.lib().ecsg_ghost_sxz_noalloc(
            ctypes.byref(self.views[0]), ctypes.byref(self.views[1]), float(self.case.dt),
            ecsg_b200.ECSG_F64 if self.prec == "f64" else ecsg_b200.ECSG_F32, ctypes.c_void_p(self.X.data_ptr()),
            max_iter, self.stream, ctypes.byref(iters) if iters is not None else None, self.err, 256)

    def sticky(self, clear):
        st = ctypes.c_int(-1)
        assert ecsg_b200.lib().ecsg_ghost_sxz_noalloc_status(self.stream, ctypes.byref(st), clear) == 0
        return st.value

    def close(self):
        self.sim.close()


@pytest.mark.gpu
@pytest.mark.parametrize("ratio", [2, 3, 4])
@pytest.mark.parametrize("prec", ["f64", "f32"])
def test_noalloc_matches_allocating_solve_twice(ratio, prec):
    torch = pytest.importorskip("torch")
    tol = 1e-12 if prec == "f64" else 2e-6
    S = _Setup(torch, ratio, prec, 7 * ratio + (prec == "f32"))
    try:
        S.sticky(clear=1)
        for call in range(2):
            if call == 1:
                S.new_state()   # X carries the warm start
            S.sim.ghost_sxz(1)
            iters = ctypes.c_int(-1)
            torch.cuda.synchronize()
            free0 = torch.cuda.mem_get_info()[0]
            rc = S.call(iters=iters)
            torch.cuda.synchronize()
            free1 = torch.cuda.mem_get_info()[0]
            assert rc == ecsg_b200.ECSG_OK, S.err.value
            if call == 1:   # the first call resolved the array's address; the second allocates nothing
                assert free1 == free0
            want_X, want_it, _, _ = S.sim.sxz_state(1)
            assert iters.value == want_it
            got_X = S.X.cpu().numpy()
            assert np.abs(got_X - want_X).max() <= tol * max(np.abs(want_X).max(), 1.0)
            for gi, g in enumerate(S.case.grids):
                for k in range(9):
                    want = S.sim.field(gi, k)
                    got = _from_device(S.bufs[gi][k], g["n"], S.R, want.shape)
                    assert np.abs(got - want).max() <= tol * np.abs(want).max(), (call, gi, k)
        assert S.sticky(clear=0) == 0   # converged solves leave the sticky word clear
    finally:
        S.close()


@pytest.mark.gpu
def test_noalloc_sweep_cap_reported_sync_and_async():
    """A cap of one sweep on a cold start: a waiting call returns
    ECSG_ERR_NOT_CONVERGED after 1 sweep; an asynchronous one (iters NULL)
    leaves ECSG_ST_JACOBI_CAP in the sticky word until it is cleared."""
    torch = pytest.importorskip("torch")
    S = _Setup(torch, 3, "f64", 11)
    try:
        S.sticky(clear=1)
        iters = ctypes.c_int(-1)
        assert S.call(max_iter=1, iters=iters) == ERR_NOT_CONVERGED
        assert iters.value == 1
        assert S.sticky(clear=1) & ST_JACOBI_CAP
        assert S.sticky(clear=0) == 0
        S.X.zero_()
        S.new_state()
        assert S.call(max_iter=1) == ecsg_b200.ECSG_OK   # does not wait: cannot know yet
        assert S.sticky(clear=1) & ST_JACOBI_CAP
        S.X.zero_()
        assert S.call() == ecsg_b200.ECSG_OK             # converges: nothing latched
        assert S.sticky(clear=0) == 0
    finally:
        S.close()


def _host_views(fine_n, fine_h, coarse_n, coarse_h):
    """Views with valid layouts and dummy pointers (the checks run first)."""
    vs = []
    for n, h in ((fine_n, fine_h), (coarse_n, coarse_h)):
        v = GridView()
        v.size[:] = list(n)
        v.step[:] = list(h)
        v.radius = 1
        lay = device_layout(n, 1)
        v.pitch[:] = list(lay["pitch"])
        v.origin = lay["origin"]
        for k in range(9):
            v.field[k] = 0x100
        v.buoy = 0x100
        vs.append(v)
    return vs


def _reject(fine, coarse):
    err = ctypes.create_string_buffer(256)
    rc = ecsg_b200.lib().ecsg_ghost_sxz_noalloc(ctypes.byref(fine), ctypes.byref(coarse), 0.5, ecsg_b200.ECSG_F32,
                                                ctypes.c_void_p(0x100), 0, None, None, err, 256)
    return rc, err.value


def test_noalloc_rejects_oversized_interface():
    fine, coarse = _host_views((800, 800, 10), (5.0,) * 3, (400, 400, 10), (10.0,) * 3)
    rc, msg = _reject(fine, coarse)
    assert rc == ERR_INVALID and b"exceeds the static work space" in msg


def test_noalloc_rejects_non_integer_or_unequal_ratios():
    # x steps 10 / 24: ratio 2.4 (sizes consistent with r = 2)
    fine, coarse = _host_views((20, 20, 6), (10.0, 10.0, 10.0), (10, 10, 5), (24.0, 20.0, 24.0))
    rc, msg = _reject(fine, coarse)
    assert rc == ERR_INVALID and b"ratio" in msg
    # x ratio 2, y ratio 3
    fine, coarse = _host_views((20, 20, 6), (10.0, 10.0, 10.0), (10, 10, 5), (20.0, 30.0, 20.0))
    rc, msg = _reject(fine, coarse)
    assert rc == ERR_INVALID and b"ratio" in msg
    # the valid pair passes the checks only with the right sizes
    fine, coarse = _host_views((21, 20, 6), (10.0, 10.0, 10.0), (10, 10, 5), (20.0, 20.0, 20.0))
    rc, msg = _reject(fine, coarse)
    assert rc == ERR_INVALID and b"ratio * coarse size" in msg


def test_noalloc_rejects_bad_layouts():
    fine, coarse = _host_views((20, 20, 6), (10.0,) * 3, (10, 10, 5), (20.0,) * 3)
    coarse.pitch[1] = coarse.size[1] + 2   # one row short of y in [-1, ny + 1]
    rc, msg = _reject(fine, coarse)
    assert rc == ERR_INVALID and b"pitch" in msg
    fine, coarse = _host_views((20, 20, 6), (10.0,) * 3, (10, 10, 5), (20.0,) * 3)
    fine.origin = 0                        # the x = -1 halo would sit before the buffer
    rc, msg = _reject(fine, coarse)
    assert rc == ERR_INVALID and b"origin" in msg
    fine, coarse = _host_views((20, 20, 6), (10.0,) * 3, (10, 10, 5), (20.0,) * 3)
    fine.origin = 1 << 40                  # would have been truncated to 32 bits
    rc, msg = _reject(fine, coarse)
    assert rc == ERR_INVALID and b"origin" in msg
    fine, coarse = _host_views((20, 20, 6), (10.0,) * 3, (10, 10, 5), (20.0,) * 3)
    coarse.field[4] = None
    rc, msg = _reject(fine, coarse)
    assert rc == ERR_INVALID and b"null" in msg
