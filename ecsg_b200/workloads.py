"""Synthetic workloads: the reference's own experiment inputs and the benchmark media.

All generators are seeded numpy code; nothing is read from disk.

* ``eci_test_case(k)`` rebuilds the inputs of the reference experiment
  tests/test1-cmp-eci-ii (eci/SConstruct:26-195 with par1.py / par2.py /
  par3.py): a two-layer isotropic medium on a two-grid composite at refinement
  ratio 2.  Every number the reference script passes through a Madagascar
  command line is rounded through ``%f`` exactly as the script does, so the
  generated inputs are the ones the reference's golden traces were produced from.
* ``three_grid_vti(...)``: the three-grid ratio-3 tilted-VTI benchmark medium
  (1081x1081x121 @ 5 m, 361x361x161 @ 15 m, 121x121x101 @ 45 m by default).

Units follow the reference tests: metres, milliseconds, m/ms and g/cm^3.
"""
import math

import numpy as np

# Staggered positions (pos[d] = 1: staggered in dim d), init_del_sim.cpp:14-24.
SIM_POS = [(0, 0, 0), (1, 1, 0), (1, 0, 1), (1, 0, 0), (1, 0, 0), (1, 0, 0), (1, 1, 1), (0, 0, 1), (0, 1, 0)]
SIM_NAMES = ["vx", "vy", "vz", "sxx", "syy", "szz", "syz", "sxz", "sxy"]
# Stiffness order of update_stress.cpp:17-25 and their positions (init_del_par_field.cpp:82-88).
STIFF_NAMES = ["c11", "c22", "c33", "c23", "c13", "c12", "c44", "c55", "c66"]
STIFF_POS = [(1, 0, 0)] * 6 + [(1, 1, 1), (0, 0, 1), (0, 1, 0)]


def _f(x):
    """A value as it comes out of the reference script's '%f' formatting."""
    return float("%f" % x)


def ricker(nt, d1, fpeak, o1=0.0):
    """Ricker wavelet as the reference script asks sfmath for it (eci/SConstruct:118-147):
    (1-2a(t-t0)^2) exp(-a(t-t0)^2), a = pi^2 f^2 and t0 = 1/f, both '%f'-rounded."""
    pi = math.atan(1) * 4.0
    a = _f(pi ** 2 * fpeak ** 2)
    t0 = _f(1.0 / fpeak)
    t = o1 + np.arange(nt, dtype=np.float64) * d1
    arg = a * (t - t0) * (t - t0)
    return ((1.0 - 2.0 * arg) * np.exp(-arg)).astype(np.float32)


class Case:
    """Inputs of one composite-grid run.

    grids:   list of dicts with 'n' (cells, x,y,z) and 'h' (steps, x,y,z); grid 0 on top.
    media:   per grid, node-position float32 arrays (shape (nz+1, ny+1, nx+1)):
             'buoy', and either 's11','s13' (isotropic, the reference input form)
             or 'cij' (21 x node arrays in Voigt upper-triangle order).
    dt, nsteps, radius, top_bc, imode
    src:     dict(xyz=(x,y,z), trace=float32[nt], scale, comp) -- comp 0 = vx
    rec:     float32 (n_rec, 3) coordinates, plus rec_comp
    """

    def __init__(self, **kw):
        self.mirror_fix = False   # True: vy wall mirrors cover the updated interface plane (energy-exact)
        self.__dict__.update(kw)

    @property
    def ratio(self):
        if len(self.grids) < 2:
            return 1
        return int(round(self.grids[1]["h"][0] / self.grids[0]["h"][0]))

    def points(self):
        return sum((g["n"][0] + 1) * (g["n"][1] + 1) * (g["n"][2] + 1) for g in self.grids)


def eci_test_case(test=1, imode=1, nsteps=None):
    """Inputs of tests/test1-cmp-eci-ii/{eci,ii} with par{test}.py."""
    n_extra, src_option = {1: (5, 0), 2: (1, 0), 3: (5, 1)}[test]
    cfl, nspw, lx, ly, lz1, lz2, duration, fpeak = 0.98, 16, 1600, 1600, 300, 500, 700, 15.0
    layer1 = {"rho": 2.5, "cs": 1.0, "cp": 2.0}
    layer2 = {"rho": 2.65, "cs": 2.0, "cp": 4.0}
    for L in (layer1, layer2):
        L["buoy"] = 1.0 / L["rho"]
        L["s11"] = L["rho"] * L["cp"] ** 2
        L["s13"] = L["s11"] - 2 * L["rho"] * L["cs"] ** 2
    dx1 = layer1["cs"] * 1000 / fpeak / nspw
    dx2 = dx1 * 2
    nx2, ny2 = int(lx / dx2), int(ly / dx2)
    nx1, ny1 = 2 * nx2, 2 * ny2
    nz1 = int(lz1 / dx1 / 2) * 2
    nz2 = int(lz2 / dx2)
    g1 = {"n": (nx1, ny1, nz1), "h": (_f(dx1),) * 3}
    g2 = {"n": (nx2, ny2, nz2), "h": (_f(dx2),) * 3}

    def layered(nx, ny, nz, n2planes, key):
        a = np.empty((nz + 1, ny + 1, nx + 1), dtype=np.float32)
        a[: nz + 1 - n2planes] = np.float32(_f(layer1[key]))
        a[nz + 1 - n2planes:] = np.float32(_f(layer2[key]))
        return a

    media = [
        {k: layered(nx1, ny1, nz1, n_extra, k) for k in ("buoy", "s11", "s13")},
        {k: layered(nx2, ny2, nz2, nz2 + 1, k) for k in ("buoy", "s11", "s13")},
    ]
    dt = min(dx1, dx1, dx1) / max(layer1["cp"], layer2["cp"]) / math.sqrt(3) * cfl
    src_z = int(lz1 * 0.2 / dx2) * dx2 if src_option == 0 else (nz1 - 1) * dx1
    src_x = int(lx * 0.5 / dx2) * dx2
    src_y = int(ly * 0.5 / dx2) * dx2
    trace = ricker(700, _f(dt / 1000.0), fpeak)
    rec_z = int(lz1 * 0.2 / dx2) * dx2
    rec = np.array([[_f(int(lx * f / dx2) * dx2), _f(src_y), _f(rec_z)] for f in (0.55, 0.6, 0.65, 0.7)],
                   dtype=np.float32)
    movie_dt = _f(30 * dt)
    movie_nt = int(duration / (30 * dt))
    dtp = _f(dt)
    steps = int(math.ceil(movie_dt * movie_nt / dtp)) + 1
    return Case(name="eci_test%d" % test if imode else "ii_test%d" % test,
                grids=[g1, g2], media=media, medium="iso", dt=dtp,
                nsteps=steps if nsteps is None else nsteps, radius=1, top_bc=1, imode=imode,
                src={"xyz": (_f(src_x), _f(src_y), _f(src_z)), "trace": trace, "scale": 1000.0, "comp": 0},
                rec=rec, rec_comp=0)


def config1_case(ratio=3, nsteps=1500, fpeak=10.0, cfl=0.9):
    """The plain two-grid composite of the benchmark's accuracy configuration:
    fine top grid 91 x 91 x 31 points at 10 m (depth 0-300 m) over a coarse
    grid at 10 * ratio m reaching 1500 m (ratio 3: 31 x 31 x 41 points; the
    ratio-2 twin: 46 x 46 x 61), domain 900 x 900 m.  Isotropic media: top
    vp 1000, vs 500 m/s, rho 1800 kg/m^3; bottom vp 3000, vs 1700, rho 2300
    (in the reference tests' units m, ms, m/ms, g/cm^3: eci/SConstruct:34-40,
    buoy = 1/rho, s11 = rho vp^2, s13 = s11 - 2 rho vs^2).  Free surface,
    rigid sides and bottom.  A 10 Hz Ricker vz point force at (450, 450,
    150 m); dt = cfl * h / vmax / sqrt(3); 91 vz receivers on the surface
    line y = 450 m, x = 0, 10, ..., 900 m."""
    top = {"rho": 1.8, "cs": 0.5, "cp": 1.0}
    bot = {"rho": 2.3, "cs": 1.7, "cp": 3.0}
    for L in (top, bot):
        L["buoy"] = 1.0 / L["rho"]
        L["s11"] = L["rho"] * L["cp"] ** 2
        L["s13"] = L["s11"] - 2 * L["rho"] * L["cs"] ** 2
    h1, h2 = 10.0, 10.0 * ratio
    g1 = {"n": (90, 90, 30), "h": (h1,) * 3}
    g2 = {"n": (90 // ratio, 90 // ratio, int(round(1200.0 / h2))), "h": (h2,) * 3}
    media = []
    for g, L in ((g1, top), (g2, bot)):
        n = g["n"]
        media.append({k: np.full((n[2] + 1, n[1] + 1, n[0] + 1), np.float32(L[k]), dtype=np.float32)
                      for k in ("buoy", "s11", "s13")})
    dt = cfl * h1 / bot["cp"] / math.sqrt(3)
    rec = np.array([[10.0 * i, 450.0, 0.0] for i in range(91)], dtype=np.float32)
    return Case(name="config1_r%d" % ratio, grids=[g1, g2], media=media, medium="iso", dt=dt, nsteps=nsteps,
                radius=1, top_bc=1, imode=1,
                src={"xyz": (450.0, 450.0, 150.0), "trace": ricker(nsteps, dt * 1e-3, fpeak), "scale": 1.0, "comp": 2},
                rec=rec, rec_comp=2)


def random_case(seed, ratio=2, nx2=6, ny2=5, nz=(5, 4), radius=1, top_bc=1, num_grids=2, h1=10.0):
    """Small heterogeneous isotropic composite with random fields, for operator tests."""
    rng = np.random.default_rng(seed)
    grids = []
    nx, ny = nx2 * ratio ** (num_grids - 1), ny2 * ratio ** (num_grids - 1)
    h = h1
    for g in range(num_grids):
        grids.append({"n": (nx, ny, nz[g]), "h": (h, h, h)})
        nx //= ratio
        ny //= ratio
        h *= ratio
    media = []
    for g in grids:
        nx, ny, nzz = g["n"]
        shp = (nzz + 1, ny + 1, nx + 1)
        rho = rng.uniform(1.8, 2.6, shp)
        cs = rng.uniform(1.0, 1.6, shp)
        cp = cs * rng.uniform(1.7, 2.0, shp)
        s11 = rho * cp ** 2
        s13 = s11 - 2 * rho * cs ** 2
        media.append({"buoy": (1 / rho).astype(np.float32), "s11": s11.astype(np.float32),
                      "s13": s13.astype(np.float32)})
    vmax = max(float(np.sqrt(m["s11"] * m["buoy"]).max()) for m in media)
    dt = 0.5 * h1 / vmax / math.sqrt(3)
    return Case(name="random%d" % seed, grids=grids, media=media, medium="iso", dt=dt, nsteps=10,
                radius=radius, top_bc=top_bc, imode=1, src=None, rec=np.zeros((0, 3), np.float32), rec_comp=0)


# ---------------------------------------------------------------------------
# Three-grid ratio-3 benchmark model
# ---------------------------------------------------------------------------
THREE_GRID = [((1080, 1080, 120), 5.0), ((360, 360, 160), 15.0), ((120, 120, 100), 45.0)]


def _smooth_noise(rng, shape_m, corr_m, lattice_m=50.0):
    """Unit-variance Gaussian-filtered noise on a coarse lattice (correlation length
    corr_m), returned as a function that samples it at points (trilinear)."""
    from scipy.ndimage import gaussian_filter
    n = [int(math.ceil(s / lattice_m)) + 2 for s in shape_m]
    w = gaussian_filter(rng.standard_normal(n[::-1]), sigma=corr_m / lattice_m, mode="wrap")
    w = (w - w.mean()) / w.std()
    return w.astype(np.float32), lattice_m


def _sample(w, lattice_m, x, y, z):
    """Trilinear sample of lattice field w[z][y][x] at 1-D coordinate vectors x, y, z (m),
    done as three separable linear interpolations (x, then y, then z)."""
    def idx(c):
        f = c / lattice_m
        i = np.floor(f).astype(np.int64)
        return i, (f - i).astype(np.float32)
    ix, fx = idx(x)
    iy, fy = idx(y)
    iz, fz = idx(z)
    zlo, zhi = iz.min(), iz.max() + 2
    ylo, yhi = iy.min(), iy.max() + 2
    sub = w[zlo:zhi, ylo:yhi]
    a = sub[:, :, ix] * (1 - fx) + sub[:, :, ix + 1] * fx                       # (Z, Y, nx)
    b = a[:, iy - ylo, :] * (1 - fy)[None, :, None] + a[:, iy - ylo + 1, :] * fy[None, :, None]
    return (b[iz - zlo] * (1 - fz)[:, None, None] + b[iz - zlo + 1] * fz[:, None, None]).astype(np.float32)


def three_grid_model(seed=0, grids=None, pert=0.05, corr_m=200.0, tilt=False, max_dip_deg=30.0, tilt_corr_m=400.0):
    """Three-grid composite at ratio 3 (defaults: 1081x1081x121 @ 5 m over
    361x361x161 @ 15 m over 121x121x101 @ 45 m, 163,856,303 points).
    Background vp rises linearly 1.2 -> 5.0 m/ms with depth over the whole
    stack, vs = vp/1.8, rho from Gardner (0.31 vp[m/s]^0.25 g/cm^3), each with
    seeded 5 % Gaussian-filtered perturbations (200 m correlation length).
    Returns per-grid node arrays (vp, vs, rho) in float32; with tilt, also the
    symmetry-axis dip (smooth, 0 .. max_dip_deg) and azimuth (smooth, any
    angle), in radians, from two more seeded fields."""
    grids = grids or THREE_GRID
    rng = np.random.default_rng(seed)
    lx = grids[0][0][0] * grids[0][1]
    ly = grids[0][0][1] * grids[0][1]
    lz = sum(n[2] * h for n, h in grids)
    fields = [_smooth_noise(rng, (lx, ly, lz), corr_m) for _ in range(3)]
    if tilt:
        fields += [_smooth_noise(rng, (lx, ly, lz), tilt_corr_m, lattice_m=100.0) for _ in range(2)]
    out = []
    z0 = 0.0
    for (n, h) in grids:
        x = np.arange(n[0] + 1, dtype=np.float64) * h
        y = np.arange(n[1] + 1, dtype=np.float64) * h
        z = z0 + np.arange(n[2] + 1, dtype=np.float64) * h
        vp0 = (1.2 + (5.0 - 1.2) * (z / lz)).astype(np.float32)[:, None, None]
        p = [_sample(w, lat, x, y, z) for (w, lat) in fields]
        vp = vp0 * (1 + pert * p[0])
        vs = vp0 / np.float32(1.8) * (1 + pert * p[1])
        rho = (0.31 * (vp0 * 1000.0) ** 0.25).astype(np.float32) * (1 + pert * p[2])
        m = {"vp": vp, "vs": vs, "rho": rho, "n": n, "h": h}
        if tilt:
            w = _sample(*fields[3], x, y, z)
            m["dip"] = (np.float32(math.radians(max_dip_deg) * 0.5) * (1 + np.tanh(w))).astype(np.float32)
            m["azi"] = (np.float32(math.pi) * _sample(*fields[4], x, y, z)).astype(np.float32)
        out.append(m)
        z0 += n[2] * h
    return out


TTI_THOMSEN = (0.10, 0.05, 0.08)   # epsilon, delta, gamma of the benchmark medium


def three_grid_case(seed=0, grids=None, nsteps=2000, fpeak=15.0, cfl=0.9, medium="tti"):
    """Benchmark case on three_grid_model, free surface, a Ricker vz point force
    at the surface centre and a line of vz receivers along x at the surface
    centre line.  medium "tti": tilted VTI (Thomsen TTI_THOMSEN, seeded smooth
    dip <= 30 deg and azimuth), all 21 Cij, built on the device from the node
    arrays; "iso": isotropic stiffness from (vp, vs, rho)."""
    grids = grids or THREE_GRID
    model = three_grid_model(seed, grids, tilt=(medium == "tti"))
    if medium == "tti":
        eps = TTI_THOMSEN[0]
        vmax = max(float(m["vp"].max()) for m in model) * math.sqrt(1 + 2 * eps)
        media = [{k: m[k] for k in ("vp", "vs", "rho", "dip", "azi")} for m in model]
        return _surface_case("three_grid_r3_tti", grids, media, "tti", vmax, nsteps, fpeak, cfl)
    media = []
    vmax = 0.0
    for m in model:
        rho, vp, vs = m["rho"], m["vp"], m["vs"]
        s11 = rho * vp * vp
        s13 = s11 - 2 * rho * vs * vs
        media.append({"buoy": (1.0 / rho).astype(np.float32), "s11": s11.astype(np.float32),
                      "s13": s13.astype(np.float32)})
        vmax = max(vmax, float(vp.max()))
    return _surface_case("three_grid_r3", grids, media, "iso", vmax, nsteps, fpeak, cfl)


def _surface_case(name, grids, media, medium, vmax, nsteps, fpeak, cfl):
    h0 = grids[0][1]
    dt = h0 / vmax / math.sqrt(3) * cfl
    n0 = grids[0][0]
    cx, cy = n0[0] // 2 * h0, n0[1] // 2 * h0
    trace = ricker(int(3.0 / (fpeak * dt * 1e-3)) + 1, dt * 1e-3, fpeak)
    rec = np.stack([np.arange(n0[0] + 1) * h0, np.full(n0[0] + 1, cy), np.zeros(n0[0] + 1)], 1).astype(np.float32)
    case = Case(name=name, grids=[{"n": n, "h": (h, h, h)} for (n, h) in grids], media=media,
                medium=medium, dt=dt, nsteps=nsteps, radius=1, top_bc=1, imode=1,
                src={"xyz": (cx, cy, 0.0), "trace": trace, "scale": 1.0, "comp": 2}, rec=rec, rec_comp=2)
    if medium == "tti":
        case.thomsen = TTI_THOMSEN
    return case


# ---------------------------------------------------------------------------
# General anisotropic (21 Cij) media
# ---------------------------------------------------------------------------
# Slot order of the 21-Cij medium and the staggered position of each slot:
# 15 at the normal-stress position N (1,0,0), C44 C45 C46 at the syz position
# (1,1,1), C55 C56 at the sxz position (0,0,1), C66 at the sxy position (0,1,0).
CIJ21 = [(1, 1), (1, 2), (1, 3), (2, 2), (2, 3), (3, 3), (1, 4), (1, 5), (1, 6), (2, 4), (2, 5), (2, 6),
         (3, 4), (3, 5), (3, 6), (4, 4), (4, 5), (4, 6), (5, 5), (5, 6), (6, 6)]
CIJ21_POS = [(1, 0, 0)] * 15 + [(1, 1, 1)] * 3 + [(0, 0, 1)] * 2 + [(0, 1, 0)]


def stagger(f, pos):
    """Average a node field (nz+1, ny+1, nx+1) to a staggered position: the
    2-, 4- or 8-point mean of the reference's ReshapeField (field.cpp:428-476)."""
    p0, p1, p2 = pos
    o2, o1, o0 = f.shape[0] - p2, f.shape[1] - p1, f.shape[2] - p0

    def s(a, b, c):
        return f[c:c + o2, b:b + o1, a:a + o0]

    return (s(0, 0, 0) + s(0, 0, p2) + s(0, p1, 0) + s(0, p1, p2)
            + s(p0, 0, 0) + s(p0, 0, p2) + s(p0, p1, 0) + s(p0, p1, p2)) / 8


def cij_to_positions(C):
    """Node-position Voigt stiffness C (6, 6, nz+1, ny+1, nx+1) -> the 21
    staggered slot arrays (float64) of a 21-Cij medium."""
    return [np.ascontiguousarray(stagger(C[i - 1, j - 1].astype(np.float64), pos))
            for (i, j), pos in zip(CIJ21, CIJ21_POS)]


def ortho9_from_cij21(c21):
    """The orthorhombic part of a 21-Cij medium in the reference's 9-slot
    convention (c11 c22 c33 c23 c13 c12 c44 c55 c66, shear stored as 2 C44 etc.)."""
    return [c21[0], c21[3], c21[5], c21[4], c21[2], c21[1], 2 * c21[15], 2 * c21[18], 2 * c21[20]]


def random_anisotropic_C(rng, shape, rho, vp, vs, aniso=0.15):
    """Random symmetric positive-definite Voigt stiffness per point: an isotropic
    (lambda, mu) tensor plus a random symmetric perturbation of relative size aniso."""
    lam = rho * (vp * vp - 2 * vs * vs)
    mu = rho * vs * vs
    C = np.zeros((6, 6) + shape)
    for i in range(3):
        for j in range(3):
            C[i, j] = lam + (2 * mu if i == j else 0)
        C[i + 3, i + 3] = mu
    P = rng.uniform(-1, 1, (6, 6) + shape) * aniso * mu
    P = 0.5 * (P + P.transpose(1, 0, *range(2, P.ndim)))
    return C + P


def random_case_gen21(seed, ratio=2, nx2=6, ny2=5, nz=(5, 4), top_bc=1, num_grids=2, h1=10.0, aniso=0.15):
    """Small heterogeneous 21-Cij composite (random anisotropic stiffness per node)."""
    rng = np.random.default_rng(seed)
    grids = []
    nx, ny = nx2 * ratio ** (num_grids - 1), ny2 * ratio ** (num_grids - 1)
    h = h1
    for g in range(num_grids):
        grids.append({"n": (nx, ny, nz[g]), "h": (h, h, h)})
        nx //= ratio
        ny //= ratio
        h *= ratio
    media = []
    vmax = 0.0
    for g in grids:
        nxg, nyg, nzg = g["n"]
        shp = (nzg + 1, nyg + 1, nxg + 1)
        rho = rng.uniform(1.8, 2.6, shp)
        vs = rng.uniform(1.0, 1.6, shp)
        vp = vs * rng.uniform(1.7, 2.0, shp)
        C = random_anisotropic_C(rng, shp, rho, vp, vs, aniso)
        vmax = max(vmax, float(np.sqrt(np.max(np.linalg.eigvalsh(np.moveaxis(C, (0, 1), (-2, -1)))) / rho.min())))
        c21 = cij_to_positions(C)
        media.append({"buoy": (1 / rho).astype(np.float32), "c21": c21, "c9": ortho9_from_cij21(c21)})
    dt = 0.5 * h1 / vmax / math.sqrt(3)
    return Case(name="gen21_%d" % seed, grids=grids, media=media, medium="gen21", dt=dt, nsteps=10,
                radius=1, top_bc=top_bc, imode=1, src=None, rec=np.zeros((0, 3), np.float32), rec_comp=0)


# ---------------------------------------------------------------------------
# Tilted transversely isotropic media (rotated VTI)
# ---------------------------------------------------------------------------
VOIGT = [(0, 0), (1, 1), (2, 2), (1, 2), (2, 0), (0, 1)]


def rotation(dip, azi):
    """a = Rz(azi) Ry(dip): maps the symmetry-axis frame to the grid frame, so
    the axis is (sin dip cos azi, sin dip sin azi, cos dip).  Arrays broadcast;
    result (3, 3, ...)."""
    sd, cd, sa, ca = np.sin(dip), np.cos(dip), np.sin(azi), np.cos(azi)
    z = np.zeros_like(sd)
    return np.array([[ca * cd, -sa + z, ca * sd], [sa * cd, ca + z, sa * sd], [-sd, z, cd]])


def bond_matrix(a):
    """Bond stress matrix M of a rotation a (3, 3, ...): C' = M C M^T for Voigt
    stiffness with engineering shear strains (Auld, Acoustic Fields and Waves
    in Solids, ch. 3)."""
    M = np.zeros((6, 6) + a.shape[2:])
    for I, (i, j) in enumerate(VOIGT):
        for J, (k, l) in enumerate(VOIGT):
            M[I, J] = a[i, k] * a[j, k] if J < 3 else a[i, k] * a[j, l] + a[i, l] * a[j, k]
    return M


def vti_stiffness(vp, vs, rho, eps, delta, gamma):
    """Voigt stiffness (6, 6, ...) of a VTI medium from Thomsen's parameters
    (Thomsen 1986), float64."""
    vp, vs, rho = (np.asarray(v, dtype=np.float64) for v in (vp, vs, rho))
    c33, c44 = rho * vp * vp, rho * vs * vs
    c11, c66 = c33 * (1 + 2 * eps), c44 * (1 + 2 * gamma)
    c13 = np.sqrt((c33 - c44) * (c33 * (1 + 2 * delta) - c44)) - c44
    C = np.zeros((6, 6) + c33.shape)
    C[0, 0] = C[1, 1] = c11
    C[2, 2] = c33
    C[0, 1] = C[1, 0] = c11 - 2 * c66
    C[0, 2] = C[2, 0] = C[1, 2] = C[2, 1] = c13
    C[3, 3] = C[4, 4] = c44
    C[5, 5] = c66
    return C


def tti_stiffness(vp, vs, rho, dip, azi, thomsen):
    """Node stiffness (6, 6, ...) of a tilted VTI medium: vti_stiffness rotated
    by rotation(dip, azi) with the Bond matrix."""
    C = vti_stiffness(vp, vs, rho, *thomsen)
    M = bond_matrix(rotation(np.asarray(dip, np.float64), np.asarray(azi, np.float64)))
    return np.einsum("ik...,kl...,jl...->ij...", M, C, M)


def tti_as_gen21(case):
    """The same case with its TTI node medium turned into the 21 staggered slot
    arrays on the host (the oracle's input form), float64 buoyancy."""
    import copy
    out = copy.copy(case)
    out.media = []
    for m in case.media:
        C = tti_stiffness(m["vp"], m["vs"], m["rho"], m["dip"], m["azi"], case.thomsen)
        c21 = cij_to_positions(C)
        out.media.append({"buoy": 1.0 / m["rho"].astype(np.float64), "c21": c21, "c9": ortho9_from_cij21(c21)})
    out.medium = "gen21"
    return out


def random_case_tti(seed, ratio=2, nx2=6, ny2=5, nz=(5, 4), top_bc=1, num_grids=2, h1=10.0,
                    thomsen=(0.10, 0.05, 0.08)):
    """Small heterogeneous TTI composite: random node vp, vs, rho, dip (0..30 deg)
    and azimuth."""
    rng = np.random.default_rng(seed)
    grids = []
    nx, ny = nx2 * ratio ** (num_grids - 1), ny2 * ratio ** (num_grids - 1)
    h = h1
    for g in range(num_grids):
        grids.append({"n": (nx, ny, nz[g]), "h": (h, h, h)})
        nx //= ratio
        ny //= ratio
        h *= ratio
    media = []
    vmax = 0.0
    for g in grids:
        nxg, nyg, nzg = g["n"]
        shp = (nzg + 1, nyg + 1, nxg + 1)
        vs = rng.uniform(1.0, 1.6, shp).astype(np.float32)
        vp = (vs * rng.uniform(1.7, 2.0, shp)).astype(np.float32)
        media.append({"vp": vp, "vs": vs, "rho": rng.uniform(1.8, 2.6, shp).astype(np.float32),
                      "dip": rng.uniform(0, math.radians(30), shp).astype(np.float32),
                      "azi": rng.uniform(-math.pi, math.pi, shp).astype(np.float32)})
        vmax = max(vmax, float(vp.max()) * math.sqrt(1 + 2 * thomsen[0]))
    dt = 0.5 * h1 / vmax / math.sqrt(3)
    case = Case(name="tti_%d" % seed, grids=grids, media=media, medium="tti", dt=dt, nsteps=10,
                radius=1, top_bc=top_bc, imode=1, src=None, rec=np.zeros((0, 3), np.float32), rec_comp=0)
    case.thomsen = tuple(thomsen)
    return case


# ---------------------------------------------------------------------------
# Two-grid adjoint benchmark (shot gradients)
# ---------------------------------------------------------------------------
ADJOINT_GRIDS = [((360, 360, 60), 10.0), ((120, 120, 80), 30.0)]


def two_grid_adjoint_case(seed=0, shot=0, nsteps=1500, blob=False, grids=None, fpeak=10.0, cfl=0.9,
                          blob_depth=500.0, blob_radius=150.0):
    """Two grids at ratio 3 (default 361x361x61 @ 10 m over 121x121x81 @ 30 m,
    9,135,502 points), the smooth seeded model of three_grid_model made
    orthorhombic (VTI with a vertical axis: Thomsen TTI_THOMSEN, dip 0), free
    surface, one of 16 shots on a 4 x 4 surface grid (Ricker vz force), vz
    receivers on a surface grid of every third fine node (121 x 121 by
    default).  blob: the observed-data model, vs raised by a 3 % Gaussian
    (radius blob_radius, default 150 m) centred at blob_depth (500 m) below
    the middle of the surface."""
    grids = grids or ADJOINT_GRIDS
    model = three_grid_model(seed, grids)
    n0, h0 = grids[0]
    lx, ly = n0[0] * h0, n0[1] * h0
    media = []
    vmax = 0.0
    z0 = 0.0
    for m, (n, h) in zip(model, grids):
        vs = m["vs"]
        if blob:
            x = np.arange(n[0] + 1) * h - lx / 2
            y = np.arange(n[1] + 1) * h - ly / 2
            z = z0 + np.arange(n[2] + 1) * h - blob_depth
            r2 = z[:, None, None] ** 2 + y[None, :, None] ** 2 + x[None, None, :] ** 2
            vs = (vs * (1 + 0.03 * np.exp(-r2 / (2 * blob_radius ** 2)))).astype(np.float32)
        zero = np.zeros_like(m["vp"])
        media.append({"vp": m["vp"], "vs": vs, "rho": m["rho"], "dip": zero, "azi": zero})
        vmax = max(vmax, float(m["vp"].max()) * math.sqrt(1 + 2 * TTI_THOMSEN[0]))
        z0 += n[2] * h
    dt = h0 / vmax / math.sqrt(3) * cfl
    sx, sy = shot % 4, shot // 4
    src = ((0.2 + 0.2 * sx) * lx, (0.2 + 0.2 * sy) * ly, 0.0)
    trace = ricker(nsteps, dt * 1e-3, fpeak)
    nr = n0[0] // 3 + 1
    g = np.arange(nr) * 3 * h0
    rec = np.stack([np.tile(g, nr), np.repeat(g, nr), np.zeros(nr * nr)], 1).astype(np.float32)
    case = Case(name="two_grid_adjoint", grids=[{"n": n, "h": (h, h, h)} for (n, h) in grids], media=media,
                medium="tti", dt=dt, nsteps=nsteps, radius=1, top_bc=1, imode=1,
                src={"xyz": src, "trace": trace, "scale": 1.0, "comp": 2}, rec=rec, rec_comp=2)
    case.thomsen = TTI_THOMSEN
    return case


# ---------------------------------------------------------------------------
# Batch of uneven two-grid composites
# ---------------------------------------------------------------------------
def batch_instance_case(seed, nsteps=1000, fpeak=10.0, cfl=0.9):
    """One of the batch instances: fine nx, ny drawn from {61, 91, ..., 301}
    points with nz = 31 at 10 m over the matching coarse grid ((n-1)/3 + 1
    points) with 31..81 z points at 30 m; a seeded 3-layer tilted-VTI medium
    (vp 1.0..4.5 m/ms, vs = vp / 1.8, Gardner density, dip <= 30 deg per layer,
    Thomsen TTI_THOMSEN); one Ricker vz force at a random surface point; a
    line of 16 surface vz receivers."""
    rng = np.random.default_rng(10_000 + seed)
    nx = int(rng.choice(np.arange(61, 302, 30))) - 1
    ny = int(rng.choice(np.arange(61, 302, 30))) - 1
    nzc = int(rng.integers(31, 82)) - 1
    grids = [((nx, ny, 30), 10.0), ((nx // 3, ny // 3, nzc), 30.0)]
    depth = 30 * 10.0 + nzc * 30.0
    tops = np.sort(rng.uniform(0.15, 0.85, 2)) * depth
    vps = np.sort(rng.uniform(1.0, 4.5, 3))
    dips = np.radians(rng.uniform(0, 30, 3))
    azis = rng.uniform(-math.pi, math.pi, 3)
    media = []
    z0 = 0.0
    for (n, h) in grids:
        z = z0 + np.arange(n[2] + 1) * h
        layer = np.searchsorted(tops, z)
        shp = (n[2] + 1, n[1] + 1, n[0] + 1)
        vp = np.broadcast_to(vps[layer][:, None, None], shp).astype(np.float32)
        m = {"vp": vp, "vs": (vp / np.float32(1.8)).astype(np.float32),
             "rho": (0.31 * (vp * 1000.0) ** 0.25).astype(np.float32),
             "dip": np.broadcast_to(dips[layer][:, None, None], shp).astype(np.float32),
             "azi": np.broadcast_to(azis[layer][:, None, None], shp).astype(np.float32)}
        media.append({k: np.ascontiguousarray(v) for k, v in m.items()})
        z0 += n[2] * h
    h0 = grids[0][1]
    vmax = float(vps.max()) * math.sqrt(1 + 2 * TTI_THOMSEN[0])
    dt = h0 / vmax / math.sqrt(3) * cfl
    lx, ly = nx * h0, ny * h0
    src = (float(rng.uniform(0.1, 0.9)) * lx, float(rng.uniform(0.1, 0.9)) * ly, 0.0)
    rec = np.stack([np.linspace(0.1, 0.9, 16) * lx, np.full(16, 0.5 * ly), np.zeros(16)], 1).astype(np.float32)
    case = Case(name="batch_%d" % seed, grids=[{"n": n, "h": (h, h, h)} for (n, h) in grids], media=media,
                medium="tti", dt=dt, nsteps=nsteps, radius=1, top_bc=1, imode=1,
                src={"xyz": src, "trace": ricker(nsteps, dt * 1e-3, fpeak), "scale": 1.0, "comp": 2},
                rec=rec, rec_comp=2)
    case.thomsen = TTI_THOMSEN
    return case
