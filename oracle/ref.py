"""ctypes front end of the reference itself (oracle/_ref/libecsg_ref{64,32}.so).

TEST INFRASTRUCTURE ONLY.  The library is the reference's own sources compiled
with the project RSF stand-in and oracle/ref_driver.cpp (see oracle/Makefile).
A RefRun sets the reference up through its own initialisers from in-memory RSF
inputs built from a workloads.Case, exactly as main.cpp would from files.
The driver keeps one global run per loaded library, so only one RefRun per
precision may be alive at a time.
"""
import ctypes
import os

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
_LIBS = {}
c_dp = ctypes.POINTER(ctypes.c_double)
c_ip = ctypes.POINTER(ctypes.c_int)


def available(bits=64):
    return os.path.exists(os.path.join(HERE, "_ref", "libecsg_ref%d.so" % bits))


def lib(bits=64):
    if bits not in _LIBS:
        path = os.path.join(HERE, "_ref", "libecsg_ref%d.so" % bits)
        if not os.path.exists(path):
            raise RuntimeError("reference build missing: run `make -C oracle ref` where the reference is mounted")
        L = ctypes.CDLL(path)
        L.ecsg_ref_setup.argtypes = [ctypes.c_int, ctypes.POINTER(ctypes.c_char_p)]
        L.ecsg_ref_field_shape.argtypes = [ctypes.c_int] * 3 + [c_ip] * 3
        L.ecsg_ref_get_field.argtypes = [ctypes.c_int] * 3 + [c_dp]
        L.ecsg_ref_set_field.argtypes = [ctypes.c_int] * 3 + [c_dp]
        L.ecsg_ref_get_coeff.argtypes = [ctypes.c_int, c_dp]
        L.ecsg_ref_get_gsxz.argtypes = [ctypes.c_int, c_dp]
        L.ecsg_ref_set_gsxz.argtypes = [ctypes.c_int, c_dp]
        L.ecsg_ref_src.argtypes = [c_ip, c_ip, c_ip]
        L.ecsg_ref_rec.argtypes = [c_ip, c_ip]
        L.ecsg_ref_energy.restype = ctypes.c_double
        L.ecsg_ref_residues.argtypes = [ctypes.c_int, c_dp]
        L.ecsg_ref_step.argtypes = [ctypes.c_int, c_dp, c_dp]
        L.ecsg_ref_run.argtypes = [ctypes.c_int, ctypes.c_int]
        L.ecsg_ref_run.restype = ctypes.c_double
        L.ecsg_rsf_register_memory.argtypes = [ctypes.c_char_p, ctypes.c_char_p,
                                               ctypes.POINTER(ctypes.c_float), ctypes.c_long]
        _LIBS[bits] = L
    return _LIBS[bits]


def _hdr(**kv):
    return " ".join("%s=%r" % (k, v) if isinstance(v, float) else "%s=%s" % (k, v) for k, v in kv.items()).encode()


class RefRun:
    """The reference's own code path on a workloads.Case (isotropic media)."""

    def __init__(self, case, energy=False, verb=False, threads=None, bits=64):
        if case.medium != "iso":
            raise ValueError("the reference reads isotropic media only (init_del_par_field.cpp:81-149)")
        self.L = lib(bits)
        self.case = case
        self.R = case.radius
        self._keep = []
        threads = threads or len(os.sched_getaffinity(0))
        for gi, g in enumerate(case.grids):
            n, h = g["n"], g["h"]
            for key in ("buoy", "s11", "s13"):
                arr = np.ascontiguousarray(case.media[gi][key], dtype=np.float32)
                self._keep.append(arr)
                hdr = _hdr(n1=n[0] + 1, n2=n[1] + 1, n3=n[2] + 1, d1=float(h[0]), d2=float(h[1]), d3=float(h[2]))
                self.L.ecsg_rsf_register_memory(("%s_%d" % (key, gi + 1)).encode(), hdr,
                                                arr.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), arr.size)
        args = ["ecsg_ref", "num_threads=%d" % threads, "num_grids=%d" % len(case.grids),
                "radius=%d" % case.radius, "dt=%r" % float(case.dt), "imode=%d" % case.imode,
                "top_bc=%d" % case.top_bc, "check_energy=%s" % ("y" if energy else "n"),
                "verb=%s" % ("y" if verb else "n")]
        if case.src is not None:
            tr = np.ascontiguousarray(case.src["trace"], dtype=np.float32)
            self._keep.append(tr)
            x, y, z = case.src["xyz"]
            hdr = _hdr(n1=tr.size, d1=float(case.dt) / 1000.0, o2=float(x), o3=float(y), o4=float(z))
            self.L.ecsg_rsf_register_memory(b"src", hdr, tr.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), tr.size)
            args.append("src=memory")
        if len(case.rec):
            rc = np.ascontiguousarray(case.rec, dtype=np.float32)
            self._keep.append(rc)
            self.L.ecsg_rsf_register_memory(b"rec_in", _hdr(n1=3, n2=rc.shape[0]),
                                            rc.ctypes.data_as(ctypes.POINTER(ctypes.c_float)), rc.size)
            args.append("rec_in=memory")
        argv = (ctypes.c_char_p * len(args))(*[a.encode() for a in args])
        rc = self.L.ecsg_ref_setup(len(args), argv)
        if rc != 0:
            raise RuntimeError("ecsg_ref_setup failed (%d)" % rc)
        self.n_rec = len(case.rec)

    def close(self):
        if self.L is not None:
            self.L.ecsg_ref_teardown()
            # the OpenMP runtime is shared with the oracle library: restore the thread count
            self.L.ecsg_ref_set_threads(len(os.sched_getaffinity(0)))
            self.L = None

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass

    def shape(self, g, kind, k):
        ln, pos, end = (ctypes.c_int * 3)(), (ctypes.c_int * 3)(), (ctypes.c_int * 3)()
        if self.L.ecsg_ref_field_shape(g, kind, k, ln, pos, end) != 0:
            raise KeyError((g, kind, k))
        return (ln[2], ln[1], ln[0]), tuple(pos), tuple(end)

    def get(self, g, k, kind=0):
        shp, _, _ = self.shape(g, kind, k)
        out = np.zeros(shp)
        self.L.ecsg_ref_get_field(g, kind, k, out.ctypes.data_as(c_dp))
        return out

    def set(self, g, k, arr, kind=0):
        arr = np.ascontiguousarray(arr, dtype=np.float64)
        shp, _, _ = self.shape(g, kind, k)
        assert arr.shape == shp, (arr.shape, shp)
        self.L.ecsg_ref_set_field(g, kind, k, arr.ctypes.data_as(c_dp))

    def coeff(self, g):
        out = np.zeros(3 * self.R)
        self.L.ecsg_ref_get_coeff(g, out.ctypes.data_as(c_dp))
        return out.reshape(3, self.R)

    def gsxz(self, i):
        n2 = self.case.grids[i + 1]["n"]
        out = np.zeros((n2[1] + 1) * (n2[0] + 1))
        self.L.ecsg_ref_get_gsxz(i, out.ctypes.data_as(c_dp))
        return out

    def set_gsxz(self, i, arr):
        arr = np.ascontiguousarray(arr, dtype=np.float64)
        self.L.ecsg_ref_set_gsxz(i, arr.ctypes.data_as(c_dp))

    def src_loc(self):
        g, ln = ctypes.c_int(), ctypes.c_int()
        loc = (ctypes.c_int * 3)()
        self.L.ecsg_ref_src(ctypes.byref(g), loc, ctypes.byref(ln))
        return (g.value, loc[0], loc[1], loc[2]), ln.value

    def rec_loc(self):
        n = ctypes.c_int()
        self.L.ecsg_ref_rec(ctypes.byref(n), None)
        loc = (ctypes.c_int * (4 * n.value))()
        self.L.ecsg_ref_rec(ctypes.byref(n), loc)
        return [tuple(loc[4 * i:4 * i + 4]) for i in range(n.value)]

    def update_vel(self, g):
        return self.L.ecsg_ref_update_vel(g)

    def update_stress(self, g):
        return self.L.ecsg_ref_update_stress(g)

    def ghost_vz(self, i):
        return self.L.ecsg_ref_ghost_vz(i)

    def ghost_sxz(self, i):
        return self.L.ecsg_ref_ghost_sxz(i)

    def ghost_syz(self, i):
        return self.L.ecsg_ref_ghost_syz(i)

    def copy_vel(self):
        return self.L.ecsg_ref_copy_vel()

    def energy(self):
        return self.L.ecsg_ref_energy()

    def residues(self, which=7):
        out = np.zeros(9 * (len(self.case.grids) - 1))
        self.L.ecsg_ref_residues(which, out.ctypes.data_as(c_dp))
        return out.reshape(-1, 9)

    def step(self, niter):
        rec = np.zeros(max(self.n_rec, 1))
        e = ctypes.c_double(0)
        self.L.ecsg_ref_step(niter, rec.ctypes.data_as(c_dp), ctypes.byref(e))
        return rec[: self.n_rec], e.value

    def run(self, nsteps, niter0=0):
        """Wall seconds for nsteps iterations of main.cpp's loop body."""
        return self.L.ecsg_ref_run(niter0, nsteps)
