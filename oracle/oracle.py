"""Python front end of the C restatement (ecsg_oracle.c).  TEST INFRASTRUCTURE ONLY.

Holds one composite run in double precision in the reference's Field layout
(field.cpp:85-149) and steps it in the order of main.cpp:165-261.  Set-up
helpers restate init_del_par_field.cpp (media), init_src.cpp (source),
init_del_rec_trace.cpp (receivers) and init_del_fdcoeff.cpp (coefficients).
"""
import ctypes
import math
import os

import numpy as np

from ecsg_b200.workloads import CIJ21_POS, SIM_POS, STIFF_POS

HERE = os.path.dirname(os.path.abspath(__file__))
_LIB = None

c_dp = ctypes.POINTER(ctypes.c_double)


class OField(ctypes.Structure):
    _fields_ = [("p", c_dp), ("len", ctypes.c_int * 3), ("R", ctypes.c_int),
                ("pos", ctypes.c_int * 3), ("end", ctypes.c_int * 3)]


class OGrid(ctypes.Structure):
    _fields_ = [("n", ctypes.c_int * 3), ("R", ctypes.c_int), ("f", OField * 9), ("buoy", OField),
                ("c", OField * 9), ("coeff", (ctypes.c_double * 6) * 3)]


def lib():
    global _LIB
    if _LIB is None:
        path = os.path.join(HERE, "_build", "libecsg_oracle.so")
        if not os.path.exists(path):
            raise RuntimeError("oracle library missing: run `make -C oracle oracle`")
        L = ctypes.CDLL(path)
        P = ctypes.POINTER
        L.o_update_vel.argtypes = [P(OGrid), ctypes.c_int, ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.o_update_stress.argtypes = [P(OGrid), ctypes.c_int, ctypes.c_int, ctypes.c_int]
        L.o_ghost_vz_eci.argtypes = [P(OGrid), P(OGrid), ctypes.c_int]
        L.o_ghost_vz_eci21.argtypes = [P(OGrid), P(OGrid), ctypes.c_int, P(OField), P(OField)]
        L.o_update_stress21.argtypes = [P(OGrid), P(OField), ctypes.c_int, ctypes.c_int, ctypes.c_int, P(OField)]
        L.o_ghost_syz_eci.argtypes = [P(OGrid), P(OGrid), ctypes.c_int]
        L.o_ghost_sxz_eci.argtypes = [P(OGrid), P(OGrid), ctypes.c_int, c_dp, c_dp, c_dp, c_dp,
                                      ctypes.c_int, c_dp]
        L.o_ghost_sxz_eci.restype = ctypes.c_int
        L.o_ghost_vz_ii.argtypes = [P(OGrid), P(OGrid), ctypes.c_int]
        L.o_ghost_sxz_ii.argtypes = [P(OGrid), P(OGrid)]
        L.o_ghost_syz_ii.argtypes = [P(OGrid), P(OGrid)]
        L.o_energy.argtypes = [P(OGrid), P(OField), P(OField), P(OField), c_dp]
        L.o_energy.restype = ctypes.c_double
        L.o_residues.argtypes = [P(OGrid), P(OGrid), ctypes.c_int, ctypes.c_int, c_dp]
        L.o_avgabs.argtypes = [P(OField)]
        L.o_avgabs.restype = ctypes.c_double
        _LIB = L
    return _LIB


# --------------------------------------------------------------------------
# Layout helpers (field.cpp:85-98)
# --------------------------------------------------------------------------
def field_shape(n, pos, R):
    """numpy shape (len2, len1, len0) of a Field with cells n and halo R."""
    return tuple((n[d] + 2 * R) if pos[d] else (n[d] + 1 + 2 * R) for d in (2, 1, 0))


def _ofield(arr, pos, R):
    assert arr.dtype == np.float64 and arr.flags.c_contiguous
    f = OField()
    f.p = arr.ctypes.data_as(c_dp)
    f.len[:] = [arr.shape[2], arr.shape[1], arr.shape[0]]
    f.R = R
    f.pos[:] = list(pos)
    f.end[:] = [arr.shape[2] - 1 - 2 * R, arr.shape[1] - 1 - 2 * R, arr.shape[0] - 1 - 2 * R]
    return f


def interior(arr, R):
    """View without the halo."""
    if R == 0:
        return arr
    return arr[R:-R, R:-R, R:-R]


# --------------------------------------------------------------------------
# Set-up restatements
# --------------------------------------------------------------------------
def fd_coeff(radius):
    """Staggered first-derivative coefficients, init_del_fdcoeff.cpp:38-85."""
    table = {1: [1.0], 2: [9 / 8, -1 / 24], 3: [75 / 64, -25 / 384, 3 / 640],
             4: [1225 / 1024, -245 / 3072, 49 / 5120, -5 / 7168],
             5: [711 / 587, -158 / 1761, 296 / 21383, -25 / 14159, 17 / 143243],
             6: [1225 / 1003, -338 / 3487, 35 / 2006, -127 / 42800, 19 / 52924, -6 / 274627]}
    if radius not in table:
        raise ValueError("FD coefficients of radius=%d have not been computed" % radius)
    return table[radius]


def reshape(f, pos):
    """Average a node field to a staggered position (field.cpp:428-476, same summation order)."""
    p0, p1, p2 = pos
    o2, o1, o0 = f.shape[0] - p2, f.shape[1] - p1, f.shape[2] - p0

    def s(a, b, c):
        return f[c:c + o2, b:b + o1, a:a + o0]

    return (s(0, 0, 0) + s(0, 0, p2) + s(0, p1, 0) + s(0, p1, p2)
            + s(p0, 0, 0) + s(p0, 0, p2) + s(p0, p1, 0) + s(p0, p1, p2)) / 8


def iso_stiffness(buoy, s11, s13):
    """Staggered 9-view of an isotropic medium (init_del_par_field.cpp:99-149).
    Returns (list of 9 arrays, list of the 5 distinct arrays)."""
    s11 = s11.astype(np.float64)
    s13 = s13.astype(np.float64)
    s44 = s11 - s13
    c11 = reshape(s11, STIFF_POS[0])
    c13 = reshape(s13, STIFF_POS[0])
    c55 = reshape(s44, STIFF_POS[7])
    c66 = reshape(s44, STIFF_POS[8])
    c44 = reshape(s44, STIFF_POS[6])
    nine = [c11, c11, c11, c13, c13, c13, c44, c55, c66]
    return nine


def energy_fields(buoy, nine, isotropic=True):
    """Densities at the velocity positions and compliances at the stress positions
    (InvertParameters, init_del_par_field.cpp:224-290).  For isotropic media the
    reference's closed form is used; otherwise the 3x3 normal block is inverted
    point by point."""
    b = buoy.astype(np.float64)
    dens = [1.0 / b, 1.0 / reshape(b, (1, 1, 0)), 1.0 / reshape(b, (1, 0, 1))]
    if isotropic:
        s11, s13 = nine[0], nine[4]
        base = s11 * s13 * s13 * 3 - s13 * s13 * s13 * 2 - s11 * s11 * s11
        base = 1.0 / base
        k11 = (s13 * s13 - s11 * s11) * base
        k13 = (s13 * s11 - s13 * s13) * base
        comp = [k11, k11, k11, k13, k13, k13, 1.0 / nine[6], 1.0 / nine[7], 1.0 / nine[8]]
    else:
        c11, c22, c33, c23, c13, c12 = nine[:6]
        M = np.stack([np.stack([c11, c12, c13], -1), np.stack([c12, c22, c23], -1),
                      np.stack([c13, c23, c33], -1)], -2)
        S = np.linalg.inv(M)
        comp = [S[..., 0, 0], S[..., 1, 1], S[..., 2, 2], S[..., 1, 2], S[..., 0, 2], S[..., 0, 1],
                1.0 / nine[6], 1.0 / nine[7], 1.0 / nine[8]]
    return [np.ascontiguousarray(a) for a in dens], [np.ascontiguousarray(a) for a in comp]


def c_round(x):
    """C round(): halves away from zero."""
    return int(math.floor(abs(x) + 0.5)) * (1 if x >= 0 else -1)


def locate(xyz, grids, origins):
    """Point -> (grid, ix, iy, iz), init_src.cpp:33-45 and init_del_rec_trace.cpp:82-93."""
    g = 0
    z = float(xyz[2])
    while z > grids[g]["h"][2] * grids[g]["n"][2]:
        z -= grids[g]["h"][2] * grids[g]["n"][2]
        g += 1
    if g >= len(grids):
        raise ValueError("point below the deepest grid")
    ix = c_round((float(xyz[0]) - origins[g][0]) / grids[g]["h"][0])
    iy = c_round((float(xyz[1]) - origins[g][1]) / grids[g]["h"][1])
    iz = c_round(z / grids[g]["h"][2])
    return g, ix, iy, iz


# --------------------------------------------------------------------------
# A composite run
# --------------------------------------------------------------------------
class OracleRun:
    """Double-precision composite run on the C restatement."""

    def __init__(self, case, energy=False):
        """case.ii_skip_end_column (imode 0 only) leaves the fine vz ghosts of
        the last x column untouched, as the revision of update_ghost_vz.cpp that
        produced the reference's II golden traces did."""
        self.case = case
        self.R = case.radius
        self.r = case.ratio
        self.imode = case.imode
        self.ii_end_column = not getattr(case, "ii_skip_end_column", False)
        if self.imode == 0 and len(case.grids) > 1 and self.r != 2:
            raise ValueError("intuitive interpolation (imode 0) is defined for ratio 2 only")
        self.energy_on = energy
        self.levels = []
        origins = []
        z0 = 0.0
        for gi, g in enumerate(case.grids):
            origins.append((0.0, 0.0, z0))
            z0 += g["n"][2] * g["h"][2]
        self.origins = origins
        fd = fd_coeff(self.R)
        for gi, g in enumerate(case.grids):
            n = g["n"]
            m = case.media[gi]
            L = {"n": n, "h": g["h"]}
            L["f"] = [np.zeros(field_shape(n, SIM_POS[k], self.R)) for k in range(9)]
            L["buoy"] = np.ascontiguousarray(m["buoy"].astype(np.float64))
            if case.medium == "iso":
                L["c"] = [np.ascontiguousarray(a) for a in iso_stiffness(m["buoy"], m["s11"], m["s13"])]
            elif case.medium == "ortho9":
                L["c"] = [np.ascontiguousarray(a.astype(np.float64)) for a in m["c9"]]
            elif case.medium == "gen21":
                L["c21"] = [np.ascontiguousarray(a.astype(np.float64)) for a in m["c21"]]
                L["c"] = [np.ascontiguousarray(a.astype(np.float64)) for a in m["c9"]]
            else:
                raise ValueError("oracle medium %r" % case.medium)
            coeff = np.zeros((3, 6))
            for d in range(3):
                for k in range(self.R):
                    coeff[d, k] = fd[k] * case.dt / g["h"][d]
            L["coeff"] = coeff
            if energy:
                L["dens"], L["comp"] = energy_fields(m["buoy"], L["c"], isotropic=(case.medium == "iso"))
                L["vcopy"] = [np.zeros_like(L["f"][k]) for k in range(3)]
                if case.medium == "gen21":
                    # accumulated strains at the stress positions: E_stress = 1/2 sum w eps.sigma
                    L["eps"] = [np.zeros(field_shape(n, SIM_POS[k], 0)) for k in range(3, 9)]
            self.levels.append(L)
        self._build_structs()
        ng = len(case.grids)
        self.X = []
        for i in range(1, ng):
            n2 = case.grids[i]["n"]
            self.X.append({"X": np.zeros((n2[1] + 1) * (n2[0] + 1)), "Xt": np.zeros((n2[1] + 1) * (n2[0] + 1)),
                           "A": np.zeros(9 * (n2[0] - 1) * (n2[1] - 1)), "B": np.zeros((n2[0] - 1) * (n2[1] - 1))})
        self.jacobi_iters = []
        self.src = None
        if case.src is not None:
            g, ix, iy, iz = locate(case.src["xyz"], case.grids, origins)
            self.src = (g, ix, iy, iz)
        self.rec = [locate(p, case.grids, origins) for p in case.rec]

    def _build_structs(self):
        self.structs = []
        for L in self.levels:
            s = OGrid()
            s.n[:] = list(L["n"])
            s.R = self.R
            for k in range(9):
                s.f[k] = _ofield(L["f"][k], SIM_POS[k], self.R)
                s.c[k] = _ofield(L["c"][k], STIFF_POS[k], 0)
            s.buoy = _ofield(L["buoy"], (0, 0, 0), 0)
            for d in range(3):
                for k in range(6):
                    s.coeff[d][k] = L["coeff"][d, k]
            self.structs.append(s)
            if "c21" in L:
                L["_c21"] = (OField * 21)(*[_ofield(L["c21"][k], CIJ21_POS[k], 0) for k in range(21)])
                L["_eps"] = (OField * 6)(*[_ofield(L["eps"][k], SIM_POS[k + 3], 0) for k in range(6)]) \
                    if "eps" in L else None
            if self.energy_on:
                L["_dens"] = (OField * 3)(*[_ofield(L["dens"][k], SIM_POS[k], 0) for k in range(3)])
                L["_comp"] = (OField * 9)(*[_ofield(L["comp"][k], STIFF_POS[k], 0) for k in range(9)])
                L["_vcopy"] = (OField * 3)(*[_ofield(L["vcopy"][k], SIM_POS[k], self.R) for k in range(3)])
                L["_h"] = (ctypes.c_double * 3)(*L["h"])

    # -- single operators ------------------------------------------------
    def update_vel(self, g):
        ng = len(self.levels)
        lib().o_update_vel(ctypes.byref(self.structs[g]), int(g == 0), int(g == ng - 1), self.case.top_bc,
                           int(getattr(self.case, "mirror_fix", False)))

    def update_stress(self, g):
        ng = len(self.levels)
        L = self.levels[g]
        if "c21" in L:
            lib().o_update_stress21(ctypes.byref(self.structs[g]), L["_c21"], int(g == 0), int(g == ng - 1),
                                    self.case.top_bc, L["_eps"])
        else:
            lib().o_update_stress(ctypes.byref(self.structs[g]), int(g == 0), int(g == ng - 1), self.case.top_bc)

    def ghost_vz(self, i):
        if self.imode == 0:
            lib().o_ghost_vz_ii(ctypes.byref(self.structs[i - 1]), ctypes.byref(self.structs[i]),
                                int(self.ii_end_column))
        elif "c21" in self.levels[i]:
            lib().o_ghost_vz_eci21(ctypes.byref(self.structs[i - 1]), ctypes.byref(self.structs[i]), self.r,
                                   self.levels[i - 1]["_c21"], self.levels[i]["_c21"])
        else:
            lib().o_ghost_vz_eci(ctypes.byref(self.structs[i - 1]), ctypes.byref(self.structs[i]), self.r)

    def ghost_syz(self, i):
        if self.imode == 0:
            lib().o_ghost_syz_ii(ctypes.byref(self.structs[i - 1]), ctypes.byref(self.structs[i]))
            return
        lib().o_ghost_syz_eci(ctypes.byref(self.structs[i - 1]), ctypes.byref(self.structs[i]), self.r)

    def ghost_sxz(self, i, max_iter=0):
        if self.imode == 0:
            lib().o_ghost_sxz_ii(ctypes.byref(self.structs[i - 1]), ctypes.byref(self.structs[i]))
            return 0, 0.0
        w = self.X[i - 1]
        tol = ctypes.c_double(0)
        it = lib().o_ghost_sxz_eci(ctypes.byref(self.structs[i - 1]), ctypes.byref(self.structs[i]), self.r,
                                   w["X"].ctypes.data_as(c_dp), w["Xt"].ctypes.data_as(c_dp),
                                   w["A"].ctypes.data_as(c_dp), w["B"].ctypes.data_as(c_dp),
                                   max_iter, ctypes.byref(tol))
        self.jacobi_iters.append(it)
        return it, tol.value

    def copy_vel(self):
        for L in self.levels:
            for k in range(3):
                L["vcopy"][k][...] = L["f"][k]

    def energy(self):
        e = 0.0
        for gi, L in enumerate(self.levels):
            if "c21" in L:
                e += self._energy21(L)
            else:
                e += lib().o_energy(ctypes.byref(self.structs[gi]), L["_vcopy"], L["_dens"], L["_comp"], L["_h"])
        return e

    def _energy21(self, L):
        """1/2 h^3 [sum w rho v v' + sum w eps.sigma] with the trapezoid weights of
        TriMulFields (field.cpp:502-515); eps are the accumulated strains."""
        R = self.R

        def w(shape, pos):
            m = np.ones(shape)
            for ax, d in ((0, 2), (1, 1), (2, 0)):
                if not pos[d]:
                    sl = [slice(None)] * 3
                    for idx in (0, shape[ax] - 1):
                        sl[ax] = idx
                        m[tuple(sl)] *= 0.5
            return m
        tot = 0.0
        for k in range(3):
            v = interior(L["f"][k], R)
            vc = interior(L["vcopy"][k], R)
            tot += float((w(v.shape, SIM_POS[k]) * L["dens"][k] * v * vc).sum())
        for k in range(6):
            sg = interior(L["f"][k + 3], R)
            tot += float((w(sg.shape, SIM_POS[k + 3]) * L["eps"][k] * sg).sum())
        h = L["h"]
        return 0.5 * h[0] * h[1] * h[2] * tot

    def residues(self, i, which=7):
        out = np.zeros(9)
        lib().o_residues(ctypes.byref(self.structs[i - 1]), ctypes.byref(self.structs[i]), self.r, which,
                         out.ctypes.data_as(c_dp))
        return out

    def field(self, g, k):
        return self.levels[g]["f"][k]

    # -- the time loop (main.cpp:165-261) ----------------------------------
    def step(self, niter, residues=False):
        ng = len(self.levels)
        res = np.zeros((max(ng - 1, 0), 9)) if residues else None
        if self.energy_on:
            self.copy_vel()
        for g in range(ng):
            self.update_vel(g)
        rc = getattr(self.case, "rec_comp", 0)   # the sampled component (main.cpp:182-184 samples vx)
        rec = np.array([self.levels[g]["f"][rc][iz + self.R, iy + self.R, ix + self.R]
                        for (g, ix, iy, iz) in self.rec])
        if residues:
            for i in range(1, ng):
                res[i - 1] = self.residues(i, 3)
        if self.src is not None and niter < len(self.case.src["trace"]):
            g, ix, iy, iz = self.src
            comp = self.case.src.get("comp", 0)
            amp = np.float32(self.case.src["scale"]) * np.float32(self.case.src["trace"][niter])
            self.levels[g]["f"][comp][iz + self.R, iy + self.R, ix + self.R] += float(amp)
        for i in range(1, ng):
            self.ghost_vz(i)
        if residues:
            for i in range(1, ng):
                res[i - 1, 6:] = self.residues(i, 4)[6:]
        e = self.energy() if self.energy_on else None
        for g in range(ng):
            self.update_stress(g)
        for i in range(1, ng):
            self.ghost_sxz(i)
            self.ghost_syz(i)
        return rec, e, res

    def run(self, nsteps=None, residues=False):
        nsteps = self.case.nsteps if nsteps is None else nsteps
        recs, es, rs = [], [], []
        for n in range(nsteps):
            rec, e, res = self.step(n, residues=residues)
            recs.append(rec)
            es.append(e)
            rs.append(res)
        out = {"rec": np.array(recs).T if self.rec else np.zeros((0, nsteps))}
        if self.energy_on:
            out["energy"] = np.array(es)
        if residues:
            out["res"] = np.array(rs)
        return out
