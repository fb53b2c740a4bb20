"""ecsg_b200 -- B200 (sm_100a) implementation of ECSG's composite-staggered-grid time loop.

The compute path is libecsg_b200.so (hand-written CUDA kernels behind the C ABI
of include/ecsg_b200.h).  This module is a thin ctypes mirror of that ABI with
the reference's vocabulary: a Simulation holds the device state of one
composite run and exposes the reference's operators (UpdateVel, UpdateStress,
UpdateGhostVZ/SXZ/SYZ, ComputeEnergy, compute_res_*) and its time loop
(main.cpp:165-261).  There is no CPU fallback: without the built library or a
usable GPU every call raises.
"""
import ctypes
import math
import os

import numpy as np

from .workloads import SIM_POS, STIFF_POS, Case  # noqa: F401

HERE = os.path.dirname(os.path.abspath(__file__))
LIB_PATH = os.path.join(HERE, "_lib", "libecsg_b200.so")

ECSG_OK = 0
ECSG_F32, ECSG_F64 = 0, 1
ECSG_MEDIUM_ISO, ECSG_MEDIUM_ORTHO9, ECSG_MEDIUM_GEN21 = 0, 1, 2
_MEDIUM = {"iso": ECSG_MEDIUM_ISO, "ortho9": ECSG_MEDIUM_ORTHO9, "gen21": ECSG_MEDIUM_GEN21, "tti": ECSG_MEDIUM_GEN21}
ST_JACOBI_CAP, ST_BARRIER_TIMEOUT, ST_NONFINITE, ST_PIPE_TIMEOUT = 1, 2, 4, 8

c_dp = ctypes.POINTER(ctypes.c_double)
c_fp = ctypes.POINTER(ctypes.c_float)
c_ip = ctypes.POINTER(ctypes.c_int)


class GridDesc(ctypes.Structure):
    _fields_ = [("size", ctypes.c_int * 3), ("step", ctypes.c_double * 3)]


class Config(ctypes.Structure):
    _fields_ = [("num_grids", ctypes.c_int), ("radius", ctypes.c_int), ("dt", ctypes.c_double),
                ("imode", ctypes.c_int), ("top_bc", ctypes.c_int), ("precision", ctypes.c_int),
                ("medium", ctypes.c_int), ("energy", ctypes.c_int), ("jacobi_max_iter", ctypes.c_int),
                ("device", ctypes.c_int), ("mirror_fix", ctypes.c_int), ("ii_skip_end_column", ctypes.c_int)]


class GridView(ctypes.Structure):
    """ecsg_grid_view: one grid's device arrays in the library's device layout."""
    _fields_ = [("size", ctypes.c_int * 3), ("step", ctypes.c_double * 3), ("radius", ctypes.c_int),
                ("pitch", ctypes.c_int * 3), ("origin", ctypes.c_longlong), ("field", ctypes.c_void_p * 9),
                ("buoy", ctypes.c_void_p)]


XOFF = 32   # element x = 0 of every row sits 32 elements into the row (128-byte aligned rows)


def device_layout(n, R=1):
    """Padded device layout of a grid with n = (nx, ny, nz) cells and halo R:
    pitch (px, py, pz) and the index of element (0,0,0) (ecsg_device.cuh)."""
    px = ((XOFF + n[0] + 1 + max(R, 8)) + 31) // 32 * 32
    py = n[1] + 1 + 2 * R
    pz = n[2] + 1 + 2 * R
    return {"pitch": (px, py, pz), "origin": (R * py + R) * px + XOFF}


# (name, restype, argtypes) of every exported entry point of include/ecsg_b200.h
SIGNATURES = [
    ("ecsg_create", ctypes.c_int, [ctypes.POINTER(GridDesc), ctypes.POINTER(Config), ctypes.POINTER(ctypes.c_void_p)]),
    ("ecsg_destroy", ctypes.c_int, [ctypes.c_void_p]),
    ("ecsg_last_error", ctypes.c_char_p, [ctypes.c_void_p]),
    ("ecsg_device_count", ctypes.c_int, []),
    ("ecsg_set_medium_iso", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_fp, c_fp, c_fp]),
    ("ecsg_set_medium_ortho9", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_dp, ctypes.POINTER(c_dp)]),
    ("ecsg_set_medium_cij21", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_dp, ctypes.POINTER(c_dp)]),
    ("ecsg_set_medium_tti", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_fp, c_fp, c_fp, c_fp, c_fp,
                                           ctypes.c_double, ctypes.c_double, ctypes.c_double]),
    ("ecsg_set_field", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, c_dp]),
    ("ecsg_get_field", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, c_dp]),
    ("ecsg_domain_shape", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_int)]),
    ("ecsg_get_domain", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.POINTER(ctypes.c_float)]),
    ("ecsg_host_alloc", ctypes.c_int, [ctypes.c_size_t, ctypes.POINTER(ctypes.c_void_p)]),
    ("ecsg_host_free", ctypes.c_int, [ctypes.c_void_p]),
    ("ecsg_gradient_elems", ctypes.c_longlong, [ctypes.c_void_p, ctypes.c_int]),
    ("ecsg_pack_gradient", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    ("ecsg_unpack_gradient", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p]),
    ("ecsg_stream", ctypes.c_void_p, [ctypes.c_void_p]),
    ("ecsg_state_bytes", ctypes.c_longlong, [ctypes.c_void_p]),
    ("ecsg_save_state", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    ("ecsg_load_state", ctypes.c_int, [ctypes.c_void_p, ctypes.c_void_p]),
    ("ecsg_field_elems", ctypes.c_longlong, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    ("ecsg_update_vel", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("ecsg_update_stress", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("ecsg_ghost_vz", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("ecsg_ghost_sxz", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("ecsg_ghost_syz", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("ecsg_get_sxz_state", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_dp, c_ip, c_dp,
                                          ctypes.POINTER(ctypes.c_longlong)]),
    ("ecsg_set_sxz_state", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_dp]),
    ("ecsg_copy_vel", ctypes.c_int, [ctypes.c_void_p]),
    ("ecsg_energy", ctypes.c_int, [ctypes.c_void_p, c_dp]),
    ("ecsg_residues", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, c_dp]),
    ("ecsg_set_source", ctypes.c_int, [ctypes.c_void_p] + [ctypes.c_int] * 5 + [c_fp, ctypes.c_int, ctypes.c_float]),
    ("ecsg_set_receivers", ctypes.c_int, [ctypes.c_void_p, c_ip, ctypes.c_int, ctypes.c_int]),
    ("ecsg_locate", ctypes.c_int, [ctypes.c_void_p, c_dp, c_ip]),
    ("ecsg_run", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, c_fp, c_dp, ctypes.c_int, c_dp,
                                ctypes.c_int]),
    ("ecsg_last_run", ctypes.c_int, [ctypes.c_void_p, c_dp, ctypes.POINTER(ctypes.c_longlong)]),
    ("ecsg_timer_start", ctypes.c_int, [ctypes.c_void_p]),
    ("ecsg_timer_stop", ctypes.c_int, [ctypes.c_void_p, c_dp]),
    ("ecsg_time_kernels", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_dp]),
    ("ecsg_ghost_sxz_noalloc", ctypes.c_int, [ctypes.POINTER(GridView), ctypes.POINTER(GridView), ctypes.c_double,
                                              ctypes.c_int, ctypes.c_void_p, ctypes.c_int, ctypes.c_void_p, c_ip,
                                              ctypes.c_char_p, ctypes.c_size_t]),
    ("ecsg_ghost_sxz_noalloc_status", ctypes.c_int, [ctypes.c_void_p, c_ip, ctypes.c_int]),
    ("ecsg_synchronize", ctypes.c_int, [ctypes.c_void_p]),
    ("ecsg_get_status", ctypes.c_int, [ctypes.c_void_p, c_ip, ctypes.c_int]),
    ("ecsg_device_bytes", ctypes.c_longlong, [ctypes.c_void_p]),
    ("ecsg_update_vel_ex", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    ("ecsg_update_stress_ex", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, ctypes.c_int]),
    ("ecsg_set_coefficients", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_dp]),
    ("ecsg_create_shot", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p)]),
    ("ecsg_batch_run", ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_int, ctypes.c_int,
                                      ctypes.POINTER(c_fp), ctypes.POINTER(ctypes.c_double)]),
    ("ecsg_batch_misfit_gradient", ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_int,
                                                  ctypes.POINTER(c_fp), ctypes.c_int, c_dp]),
    ("ecsg_sum_gradients", ctypes.c_int, [ctypes.c_void_p, ctypes.POINTER(ctypes.c_void_p), ctypes.c_int]),
    ("ecsg_shots_misfit_gradient", ctypes.c_int, [ctypes.POINTER(ctypes.c_void_p), ctypes.c_int, ctypes.c_int,
                                                  ctypes.POINTER(c_fp), ctypes.c_int, ctypes.c_int, c_dp]),
    ("ecsg_autotune", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int]),
    ("ecsg_get_tuning", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_ip]),
    ("ecsg_adjoint_reset", ctypes.c_int, [ctypes.c_void_p]),
    ("ecsg_set_adjoint_field", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, c_dp]),
    ("ecsg_get_adjoint_field", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, c_dp]),
    ("ecsg_adjoint_op", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int]),
    ("ecsg_get_gradient", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, ctypes.c_int, c_dp]),
    ("ecsg_misfit_gradient", ctypes.c_int, [ctypes.c_void_p, ctypes.c_int, c_fp, ctypes.c_int,
                                            ctypes.POINTER(ctypes.c_double)]),
]
ECSG_ADJ_VEL, ECSG_ADJ_STRESS, ECSG_ADJ_GHOST_VZ, ECSG_ADJ_GHOST_SXZ, ECSG_ADJ_GHOST_SYZ = 0, 1, 2, 3, 4
_ADJ_OPS = {"vel": 0, "stress": 1, "vz": 2, "sxz": 3, "syz": 4}

_LIB = None


class EcsgError(RuntimeError):
    pass


def lib():
    """The loaded CUDA library; raises if it has not been built."""
    global _LIB
    if _LIB is None:
        if not os.path.exists(LIB_PATH):
            raise EcsgError("libecsg_b200.so is not built (python -m ecsg_b200.build); there is no CPU fallback")
        L = ctypes.CDLL(LIB_PATH)
        for name, res, args in SIGNATURES:
            fn = getattr(L, name)
            fn.restype = res
            fn.argtypes = args
        _LIB = L
    return _LIB


def field_shape(n, pos, R):
    """numpy shape (len2, len1, len0) of a component in Field layout."""
    return tuple((n[d] + 2 * R) if pos[d] else (n[d] + 1 + 2 * R) for d in (2, 1, 0))


class Simulation:
    """Device state of one composite run (ecsg_create .. ecsg_destroy)."""

    def __init__(self, case, precision="f32", energy=False, device=0, jacobi_max_iter=0):
        L = lib()
        self.case = case
        self.ng = len(case.grids)
        self.R = case.radius
        self.precision = precision
        self.energy_on = bool(energy)
        self.device = device
        descs = (GridDesc * self.ng)()
        for i, g in enumerate(case.grids):
            descs[i].size[:] = list(g["n"])
            descs[i].step[:] = [float(x) for x in g["h"]]
        cfg = Config(num_grids=self.ng, radius=case.radius, dt=float(case.dt), imode=case.imode,
                     top_bc=case.top_bc, precision=ECSG_F32 if precision == "f32" else ECSG_F64,
                     medium=_MEDIUM[case.medium],
                     energy=1 if energy else 0, jacobi_max_iter=jacobi_max_iter, device=device,
                     mirror_fix=1 if getattr(case, "mirror_fix", False) else 0,
                     ii_skip_end_column=1 if getattr(case, "ii_skip_end_column", False) else 0)
        h = ctypes.c_void_p()
        rc = L.ecsg_create(descs, ctypes.byref(cfg), ctypes.byref(h))
        if rc != ECSG_OK:
            raise EcsgError("ecsg_create failed (%d): %s" % (rc, L.ecsg_last_error(h).decode() if h.value else
                                                                  "no device or invalid configuration"))
        self.h = h
        for gi in range(self.ng):
            m = case.media[gi]
            if case.medium == "iso":
                b, s11, s13 = (np.ascontiguousarray(m[k], dtype=np.float32) for k in ("buoy", "s11", "s13"))
                self._ck(L.ecsg_set_medium_iso(h, gi, b.ctypes.data_as(c_fp), s11.ctypes.data_as(c_fp),
                                               s13.ctypes.data_as(c_fp)))
            elif case.medium == "tti":
                arrs = [np.ascontiguousarray(m[k], dtype=np.float32) for k in ("vp", "vs", "rho", "dip", "azi")]
                self._ck(L.ecsg_set_medium_tti(h, gi, *[a.ctypes.data_as(c_fp) for a in arrs],
                                               *[float(t) for t in case.thomsen]))
            else:
                key, nslot, fn = (("c21", 21, L.ecsg_set_medium_cij21) if case.medium == "gen21"
                                  else ("c9", 9, L.ecsg_set_medium_ortho9))
                b = np.ascontiguousarray(m["buoy"], dtype=np.float64)
                cs = [np.ascontiguousarray(a, dtype=np.float64) for a in m[key]]
                arr = (c_dp * nslot)(*[a.ctypes.data_as(c_dp) for a in cs])
                self._ck(fn(h, gi, b.ctypes.data_as(c_dp), arr))
        self._src_rec(case)

    def _src_rec(self, case):
        L, h = lib(), self.h
        self.src = None
        if case.src is not None:
            loc = self.locate(case.src["xyz"])
            tr = np.ascontiguousarray(case.src["trace"], dtype=np.float32)
            self._ck(L.ecsg_set_source(h, loc[0], loc[1], loc[2], loc[3], case.src.get("comp", 0),
                                       tr.ctypes.data_as(c_fp), tr.size, float(case.src["scale"])))
            self.src = loc
        self.rec = [self.locate(p) for p in case.rec]
        if self.rec:
            arr = np.ascontiguousarray(np.array(self.rec, dtype=np.int32).reshape(-1))
            self._ck(L.ecsg_set_receivers(h, arr.ctypes.data_as(c_ip), len(self.rec), case.rec_comp))
        self.step_index = 0
        self.graph_ok = True

    @classmethod
    def shot(cls, model, case):
        """A new instance sharing model's medium (ecsg_create_shot), with the
        source and receivers of case (same grids and medium as the model)."""
        self = cls.__new__(cls)
        self.case = case
        self.ng = model.ng
        self.R = model.R
        self.precision = model.precision
        self.energy_on = model.energy_on
        h = ctypes.c_void_p()
        rc = lib().ecsg_create_shot(model.h, ctypes.byref(h))
        if rc != ECSG_OK:
            raise EcsgError("ecsg_create_shot failed (%d)" % rc)
        self.h = h
        self._src_rec(case)
        return self

    def autotune(self, reps=3):
        self._ck(lib().ecsg_autotune(self.h, reps))
        return [self.tuning(g) for g in range(self.ng)]

    def tuning(self, g):
        c = (ctypes.c_int * 2)()
        self._ck(lib().ecsg_get_tuning(self.h, g, c))
        return tuple(c)

    # -- plumbing ------------------------------------------------------------
    def _ck(self, rc):
        if rc != ECSG_OK:
            raise EcsgError("ecsg call failed (%d): %s" % (rc, lib().ecsg_last_error(self.h).decode()))

    def close(self):
        if getattr(self, "h", None) is not None and self.h.value:
            lib().ecsg_destroy(self.h)
            self.h = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *a):
        self.close()

    def locate(self, xyz):
        p = (ctypes.c_double * 3)(*[float(v) for v in xyz])
        out = (ctypes.c_int * 4)()
        self._ck(lib().ecsg_locate(self.h, p, out))
        return tuple(out)

    def device_bytes(self):
        return lib().ecsg_device_bytes(self.h)

    # -- fields ---------------------------------------------------------------
    def field(self, g, k):
        n = self.case.grids[g]["n"]
        out = np.empty(field_shape(n, SIM_POS[k], self.R))
        self._ck(lib().ecsg_get_field(self.h, g, k, out.ctypes.data_as(c_dp)))
        return out

    def save_state(self):
        """The run state (fields, sxz warm starts, displacement sums) as bytes."""
        buf = np.empty(int(lib().ecsg_state_bytes(self.h)), np.uint8)
        self._ck(lib().ecsg_save_state(self.h, buf.ctypes.data_as(ctypes.c_void_p)))
        return buf

    def load_state(self, buf, step_index=None):
        """Restore a save_state() of a simulation with the same set-up; runs
        continue from step_index (the next step of the saved run)."""
        buf = np.ascontiguousarray(buf, dtype=np.uint8)
        if buf.size != int(lib().ecsg_state_bytes(self.h)):
            raise ValueError("state size does not match this simulation")
        self._ck(lib().ecsg_load_state(self.h, buf.ctypes.data_as(ctypes.c_void_p)))
        if step_index is not None:
            self.step_index = int(step_index)

    def gradient_elems(self, g):
        return int(lib().ecsg_gradient_elems(self.h, g))

    def pack_gradient(self, g, dst_ptr):
        """Enqueue the FP64 pack of grid g's 22 gradient volumes into device
        memory at dst_ptr (gradient_elems(g) doubles) on the library stream."""
        self._ck(lib().ecsg_pack_gradient(self.h, g, ctypes.c_void_p(dst_ptr)))

    def unpack_gradient(self, g, src_ptr):
        self._ck(lib().ecsg_unpack_gradient(self.h, g, ctypes.c_void_p(src_ptr)))

    def stream(self):
        """The library's cudaStream_t for this simulation (an integer handle)."""
        return lib().ecsg_stream(self.h)

    def frame(self, g, k):
        """Computational domain of field k of grid g as float32 (z, y, x), as a
        movie frame holds it (no halo)."""
        dims = (ctypes.c_int * 3)()
        self._ck(lib().ecsg_domain_shape(self.h, g, k, dims))
        out = np.empty((dims[2], dims[1], dims[0]), np.float32)
        self._ck(lib().ecsg_get_domain(self.h, g, k, out.ctypes.data_as(ctypes.POINTER(ctypes.c_float))))
        return out

    def set_field(self, g, k, arr):
        n = self.case.grids[g]["n"]
        arr = np.ascontiguousarray(arr, dtype=np.float64)
        if arr.shape != field_shape(n, SIM_POS[k], self.R):
            raise ValueError("field shape %s, expected %s" % (arr.shape, field_shape(n, SIM_POS[k], self.R)))
        self._ck(lib().ecsg_set_field(self.h, g, k, arr.ctypes.data_as(c_dp)))

    # -- operators (sim_utils.hpp:127-161) ----------------------------------
    def update_vel(self, g):
        self._ck(lib().ecsg_update_vel(self.h, g))

    def update_stress(self, g):
        self._ck(lib().ecsg_update_stress(self.h, g))

    def ghost_vz(self, i):
        self._ck(lib().ecsg_ghost_vz(self.h, i))

    def ghost_sxz(self, i):
        self._ck(lib().ecsg_ghost_sxz(self.h, i))

    def ghost_syz(self, i):
        self._ck(lib().ecsg_ghost_syz(self.h, i))

    def sxz_state(self, i):
        n2 = self.case.grids[i]["n"]
        X = np.zeros((n2[1] + 1) * (n2[0] + 1))
        it, tol, tot = ctypes.c_int(), ctypes.c_double(), ctypes.c_longlong()
        self._ck(lib().ecsg_get_sxz_state(self.h, i, X.ctypes.data_as(c_dp), ctypes.byref(it), ctypes.byref(tol),
                                          ctypes.byref(tot)))
        return X, it.value, tol.value, tot.value

    def set_sxz_state(self, i, X):
        X = np.ascontiguousarray(X, dtype=np.float64)
        self._ck(lib().ecsg_set_sxz_state(self.h, i, X.ctypes.data_as(c_dp)))

    def copy_vel(self):
        self._ck(lib().ecsg_copy_vel(self.h))

    def energy(self):
        e = ctypes.c_double()
        self._ck(lib().ecsg_energy(self.h, ctypes.byref(e)))
        return e.value

    def residues(self, i, which=7):
        out = np.zeros(9)
        self._ck(lib().ecsg_residues(self.h, i, which, out.ctypes.data_as(c_dp)))
        return out

    def last_run(self):
        """(device milliseconds of the last run's step loop, kernels it launched)"""
        ms, n = ctypes.c_double(), ctypes.c_longlong()
        self._ck(lib().ecsg_last_run(self.h, ctypes.byref(ms), ctypes.byref(n)))
        return ms.value, n.value

    def timer_start(self):
        self._ck(lib().ecsg_timer_start(self.h))

    def timer_stop(self):
        ms = ctypes.c_double()
        self._ck(lib().ecsg_timer_stop(self.h, ctypes.byref(ms)))
        return ms.value

    def time_kernels(self, nsteps=3):
        """Mean ms per step of each kernel class (see ecsg_time_kernels)."""
        out = np.zeros(7 * 8)
        self._ck(lib().ecsg_time_kernels(self.h, int(nsteps), out.ctypes.data_as(c_dp)))
        self.step_index += int(nsteps)
        o = out.reshape(7, 8)
        ng = self.ng
        return {"vel": o[0, :ng].tolist(), "vel_mirror": o[1, :ng].tolist(), "stress": o[2, :ng].tolist(),
                "ghost_vz": o[3, 1:ng].tolist(), "ghost_sxz": o[4, 1:ng].tolist(), "ghost_syz": o[5, 1:ng].tolist(),
                "src_rec": float(o[6, 0])}

    # -- adjoint (21-Cij media) ------------------------------------------------
    def adjoint_reset(self):
        self._ck(lib().ecsg_adjoint_reset(self.h))

    def set_adjoint_field(self, g, k, arr):
        a = np.ascontiguousarray(arr, dtype=np.float64)
        if a.shape != field_shape(self.case.grids[g]["n"], SIM_POS[k], self.R):
            raise ValueError("adjoint field %d of grid %d: shape %s" % (k, g, a.shape))
        self._ck(lib().ecsg_set_adjoint_field(self.h, g, k, a.ctypes.data_as(c_dp)))

    def adjoint_field(self, g, k):
        out = np.empty(field_shape(self.case.grids[g]["n"], SIM_POS[k], self.R))
        self._ck(lib().ecsg_get_adjoint_field(self.h, g, k, out.ctypes.data_as(c_dp)))
        return out

    def adjoint_op(self, op, index):
        """Transpose of one operator ("vel", "stress" on a grid; "vz", "sxz", "syz"
        on an interface); the fields must hold that operator's output state."""
        self._ck(lib().ecsg_adjoint_op(self.h, _ADJ_OPS[op], index))

    def gradient(self, g, which):
        """which = 0: buoyancy at the nodes; 1 + k: stiffness slot k (CIJ21_POS[k])."""
        from .workloads import CIJ21_POS
        n = self.case.grids[g]["n"]
        pos = (0, 0, 0) if which == 0 else CIJ21_POS[which - 1]
        out = np.empty(field_shape(n, pos, 0))
        self._ck(lib().ecsg_get_gradient(self.h, g, which, out.ctypes.data_as(c_dp)))
        return out

    def misfit_gradient(self, observed, ckpt_every=50):
        """L = 1/2 sum (receiver samples - observed)^2 over observed.shape[0] steps
        from rest; returns L, gradients via gradient()."""
        obs = np.ascontiguousarray(observed, dtype=np.float32)
        nsteps = obs.shape[0]
        loss = ctypes.c_double(0.0)
        self._ck(lib().ecsg_misfit_gradient(self.h, nsteps, obs.ctypes.data_as(c_fp), int(ckpt_every),
                                            ctypes.byref(loss)))
        self.step_index = nsteps
        return loss.value

    def status(self, clear=False):
        st = ctypes.c_int()
        self._ck(lib().ecsg_get_status(self.h, ctypes.byref(st), 1 if clear else 0))
        return st.value

    # -- the time loop (main.cpp:165-261) ------------------------------------
    def run(self, nsteps=None, energy_every=0, residues=False, graph=True, traces_out=None):
        """Advance nsteps steps on the device.  Returns dict(rec=(n_rec, nsteps)
        float32, energy=(nsteps,) with NaN on steps without energy, res=(nsteps,
        num_grids-1, 9))."""
        nsteps = self.case.nsteps if nsteps is None else int(nsteps)
        nrec = len(self.rec)
        tr = traces_out if traces_out is not None else np.zeros((nsteps, max(nrec, 1)), dtype=np.float32)
        en = np.zeros(nsteps) if energy_every else None
        rs = np.zeros((nsteps, max(self.ng - 1, 1), 9)) if residues else None
        args = (self.h, self.step_index, nsteps, tr.ctypes.data_as(c_fp) if nrec else None,
                en.ctypes.data_as(c_dp) if en is not None else None, int(energy_every),
                rs.ctypes.data_as(c_dp) if rs is not None else None)
        rc = lib().ecsg_run(*args, 1 if (graph and self.graph_ok) else 0)
        if rc != ECSG_OK and graph and self.graph_ok and b"graph" in lib().ecsg_last_error(self.h):
            # capture refused before any step ran: replay stream launches instead
            self.graph_ok = False
            rc = lib().ecsg_run(*args, 0)
        self._ck(rc)
        self.step_index += nsteps
        out = {"rec": tr[:, :nrec].T.copy()}
        if en is not None:
            out["energy"] = en
        if rs is not None:
            out["res"] = rs
        return out


def stability_dt(case_vmax, hmin, cfl=0.9):
    """dt bound of the reference tests (eci/SConstruct:108-113): h / vmax / sqrt(3) * cfl."""
    return hmin / case_vmax / math.sqrt(3) * cfl


def _handles(sims):
    return (ctypes.c_void_p * len(sims))(*[s.h.value for s in sims])


def batch_run(sims, nsteps, n0=0):
    """Advance every instance nsteps steps (ecsg_batch_run: one graph launch per
    step for all).  Returns (per-instance traces (n_rec, nsteps), device ms)."""
    bufs = [np.zeros((nsteps, max(len(s.rec), 1)), np.float32) for s in sims]
    ptrs = (c_fp * len(sims))(*[b.ctypes.data_as(c_fp) for b in bufs])
    ms = ctypes.c_double()
    rc = lib().ecsg_batch_run(_handles(sims), len(sims), int(n0), int(nsteps), ptrs, ctypes.byref(ms))
    if rc != ECSG_OK:
        raise EcsgError("ecsg_batch_run failed (%d): %s" % (rc, lib().ecsg_last_error(sims[0].h).decode()))
    for s in sims:
        s.step_index = n0 + nsteps
    return [b[:, :len(s.rec)].T.copy() for b, s in zip(bufs, sims)], ms.value


def batch_misfit_gradient(sims, observed, ckpt_every=50):
    """ecsg_misfit_gradient of every instance at once; returns the losses."""
    obs = [np.ascontiguousarray(o, dtype=np.float32) for o in observed]
    nsteps = obs[0].shape[0]
    ptrs = (c_fp * len(sims))(*[o.ctypes.data_as(c_fp) for o in obs])
    losses = np.zeros(len(sims))
    rc = lib().ecsg_batch_misfit_gradient(_handles(sims), len(sims), nsteps, ptrs, int(ckpt_every),
                                          losses.ctypes.data_as(c_dp))
    if rc != ECSG_OK:
        raise EcsgError("ecsg_batch_misfit_gradient failed (%d): %s" % (rc, lib().ecsg_last_error(sims[0].h).decode()))
    for s in sims:
        s.step_index = nsteps
    return losses


def shots_misfit_gradient(sims, observed, ckpt_every=50, sub_every=0):
    """The shots in lockstep (ecsg_shots_misfit_gradient): instances of one
    model; returns the per-shot losses and leaves the gradient of their sum in
    sims[0] (read with sims[0].gradient)."""
    obs = [np.ascontiguousarray(o, dtype=np.float32) for o in observed]
    nsteps = obs[0].shape[0]
    ptrs = (c_fp * len(sims))(*[o.ctypes.data_as(c_fp) for o in obs])
    losses = np.zeros(len(sims))
    rc = lib().ecsg_shots_misfit_gradient(_handles(sims), len(sims), nsteps, ptrs, int(ckpt_every), int(sub_every),
                                          losses.ctypes.data_as(c_dp))
    if rc != ECSG_OK:
        raise EcsgError("ecsg_shots_misfit_gradient failed (%d): %s" % (rc, lib().ecsg_last_error(sims[0].h).decode()))
    for s in sims:
        s.step_index = nsteps
    return losses


def sum_gradients(dst, srcs):
    """dst's gradients = sum over srcs, accumulated in FP64."""
    rc = lib().ecsg_sum_gradients(dst.h, _handles(srcs), len(srcs))
    if rc != ECSG_OK:
        raise EcsgError("ecsg_sum_gradients failed (%d): %s" % (rc, lib().ecsg_last_error(dst.h).decode()))
