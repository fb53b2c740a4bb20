// sim_utils_shim.cpp -- the reference's hot-path entry points on the B200 library.
//
// Compiled in place of the reference's update_vel.cpp, update_stress.cpp,
// update_ghost_vz.cpp, update_ghost_sxz.cpp, update_ghost_syz.cpp,
// compute_energy.cpp and compute_res.cpp, this file gives the reference's own
// driver (main.cpp:165-261) the same functions with the same signatures
// (sim_utils.hpp:127-161), computed on the GPU through include/ecsg_b200.h:
//   UpdateVel, UpdateStress, UpdateGhostVZ, UpdateGhostSXZ, UpdateGhostSYZ,
//   ComputeEnergy, compute_res_sxz_vx, compute_res_syz_vy, compute_res_szz_vz.
// (Jacobi2D and Norm2D, helpers of the reference's sxz solve, are not used by
// the driver and are not provided.)
//
// Parity mode: every call uploads the Fields it reads from their host buffers
// (Field::GetPtr1, the reference layout), runs the operator on the device and
// downloads the Fields it changes, so host memory stays the source of truth
// and the driver's own host accesses (vel_copy, receivers, source, movies)
// need no change.  Device state per grid (a one-grid simulation for the grid
// operators and the energy) and per interface (a two-grid simulation for the
// ghost solves and residues) is created on first use and keyed by the address
// of the grid's sim[9] array.  The medium is taken from the pointers the
// driver passes (buoyancy to UpdateVel / UpdateGhostSXZ / UpdateGhostSYZ,
// stiffness to UpdateStress / UpdateGhostVZ); an operator only reads the part
// it was given.  Errors abort with a message, as the reference does
// (field.cpp:35-44).  Radius 1; both interface modes (imode 0 at ratio 2, imode 1).
#include "sim_utils.hpp"
#include "ecsg_b200.h"

#include <cstdio>
#include <cstdlib>
#include <map>
#include <type_traits>
#include <vector>

namespace {

[[noreturn]] void die(const char *what, const ecsg_sim *s = nullptr)
{
    std::fprintf(stderr, "ecsg_b200 shim: %s%s%s\n", what, s ? ": " : "", s ? ecsg_last_error(s) : "");
    std::abort();
}

void ck(int rc, const char *what, const ecsg_sim *s)
{
    if (rc != ECSG_OK) die(what, s);
}

// Field values as doubles (the reference's real is double unless built with
// its float macros, init.hpp:16-18)
const double *as_double(const Field &f, std::vector<double> &tmp)
{
    if (std::is_same<real, double>::value) return reinterpret_cast<const double *>(f.GetPtr1());
    const size_t n = (size_t)f.GetLen(0) * f.GetLen(1) * f.GetLen(2);
    tmp.resize(n);
    for (size_t i = 0; i < n; i++) tmp[i] = (double)f.GetPtr1()[i];
    return tmp.data();
}

void from_double(Field &f, const std::vector<double> &src)
{
    const size_t n = (size_t)f.GetLen(0) * f.GetLen(1) * f.GetLen(2);
    for (size_t i = 0; i < n; i++) f.GetPtr1()[i] = (real)src[i];
}

struct GridRec {
    int n[3] = {0, 0, 0};
    const Field *buoy = nullptr;
    Field *stiff[9] = {};
    bool have_stiff = false;
    double k[3] = {0, 0, 0};
    int version = 0;   // bumped when a medium pointer becomes known
};

struct SimRec {
    ecsg_sim *sim = nullptr;
    std::vector<const Field *> grids;   // members, top first
    std::vector<int> version;           // medium version uploaded per member
    std::vector<bool> kset;             // FD coefficients handed over per member
};

std::map<const Field *, GridRec> g_grids;
std::map<std::pair<std::vector<const Field *>, int>, SimRec> g_sims;   // (members, imode)
int g_top_bc = -1;

GridRec &grid_of(const Field *sim)
{
    GridRec &G = g_grids[sim];
    if (G.n[0] == 0) {
        const Field &vx = sim[0];   // position (0,0,0): end = grid size (field.cpp:88-97)
        for (int d = 0; d < 3; d++) G.n[d] = vx.GetEnd(d) - vx.GetStart(d);
        const int R = (vx.GetLen(0) - (vx.GetEnd(0) - vx.GetStart(0) + 1)) / 2;
        if (R != 1) die("radius must be 1 on the device path");
    }
    return G;
}

void note_coeff(GridRec &G, real **coeff)
{
    for (int d = 0; d < 3; d++) G.k[d] = (double)coeff[d][0];
}

// the simulation of one grid or of one interface (fine, coarse)
SimRec &sim_of(std::vector<const Field *> members, int imode = ECSG_MODE_ECI)
{
    SimRec &S = g_sims[{members, imode}];
    if (!S.sim) {
        S.grids = members;
        S.version.assign(members.size(), -1);
        S.kset.assign(members.size(), false);
        std::vector<ecsg_grid_desc> gd(members.size());
        int r = 1;
        for (size_t i = 0; i < members.size(); i++) {
            const GridRec &G = g_grids[members[i]];
            if (i == 1) r = g_grids[members[0]].n[0] / G.n[0];
            for (int d = 0; d < 3; d++) {
                gd[i].size[d] = G.n[d];
                gd[i].step[d] = (double)(i == 0 ? 1 : r);   // coefficients are set below
            }
        }
        ecsg_config cfg = {(int)members.size(), 1, 1.0, imode, g_top_bc < 0 ? 0 : g_top_bc, ECSG_F64,
                           ECSG_MEDIUM_ORTHO9, 1, 0, 0, 0};
        ck(ecsg_create(gd.data(), &cfg, &S.sim), "ecsg_create", S.sim);
    }
    for (size_t i = 0; i < members.size(); i++) {
        GridRec &G = g_grids[members[i]];
        if (G.k[0] > 0 && !S.kset[i]) {
            ck(ecsg_set_coefficients(S.sim, (int)i, G.k), "ecsg_set_coefficients", S.sim);
            S.kset[i] = true;
        }
        if (S.version[i] == G.version) continue;
        // medium: what is known so far; the rest zero (no operator reads it)
        const int n0 = G.n[0], n1 = G.n[1], n2 = G.n[2];
        static std::vector<double> zeros;
        zeros.assign((size_t)(n0 + 1) * (n1 + 1) * (n2 + 1), 0.0);
        std::vector<double> tb;
        const double *b = G.buoy ? as_double(*G.buoy, tb) : zeros.data();
        std::vector<double> tc[9];
        const double *c[9];
        for (int k = 0; k < 9; k++) c[k] = G.have_stiff ? as_double(*G.stiff[k], tc[k]) : zeros.data();
        ck(ecsg_set_medium_ortho9(S.sim, (int)i, b, c), "ecsg_set_medium_ortho9", S.sim);
        S.version[i] = G.version;
    }
    return S;
}

void upload(SimRec &S, int i, const Field *sim)
{
    std::vector<double> t;
    for (int k = 0; k < 9; k++) ck(ecsg_set_field(S.sim, i, k, as_double(sim[k], t)), "ecsg_set_field", S.sim);
}

void download(SimRec &S, int i, Field *sim, int k0 = 0, int k1 = 8)
{
    for (int k = k0; k <= k1; k++) {
        const size_t n = (size_t)sim[k].GetLen(0) * sim[k].GetLen(1) * sim[k].GetLen(2);
        if (std::is_same<real, double>::value) {
            ck(ecsg_get_field(S.sim, i, k, reinterpret_cast<double *>(sim[k].GetPtr1())), "ecsg_get_field", S.sim);
        } else {
            std::vector<double> t(n);
            ck(ecsg_get_field(S.sim, i, k, t.data()), "ecsg_get_field", S.sim);
            from_double(sim[k], t);
        }
    }
}

void set_top_bc(int top_bc)
{
    if (g_top_bc < 0) g_top_bc = top_bc;
    else if (g_top_bc != top_bc) die("top_bc changed between calls");
}

void learn_buoy(GridRec &G, const Field *b)
{
    if (G.buoy != b) { G.buoy = b; G.version++; }
}

void learn_stiff(GridRec &G, Field *const *st)
{
    bool same = G.have_stiff;
    for (int k = 0; k < 9 && same; k++) same = G.stiff[k] == st[k];
    if (!same) {
        for (int k = 0; k < 9; k++) G.stiff[k] = st[k];
        G.have_stiff = true;
        G.version++;
    }
}

SimRec &interface_of(Field *sim1, Field *sim2, int mode = ECSG_MODE_ECI)
{
    if (mode != ECSG_MODE_ECI && mode != ECSG_MODE_II) die("interface mode must be 0 or 1");
    grid_of(sim1);
    grid_of(sim2);
    return sim_of({sim1, sim2}, mode);
}

} // namespace

void UpdateVel(Field sim[9], const Field &buoy, real **coeff, int radius, int top, int bottom, int top_bc)
{
    if (radius != 1) die("UpdateVel: radius must be 1");
    set_top_bc(top_bc);
    GridRec &G = grid_of(sim);
    note_coeff(G, coeff);
    learn_buoy(G, &buoy);
    SimRec &S = sim_of({sim});
    upload(S, 0, sim);
    ck(ecsg_update_vel_ex(S.sim, 0, top, bottom), "UpdateVel", S.sim);
    download(S, 0, sim, 0, 2);
}

void UpdateStress(Field sim[9], Field *stiffness_ptr[9], real **coeffs, int radius, int top, int bottom, int top_bc)
{
    if (radius != 1) die("UpdateStress: radius must be 1");
    set_top_bc(top_bc);
    GridRec &G = grid_of(sim);
    note_coeff(G, coeffs);
    learn_stiff(G, stiffness_ptr);
    SimRec &S = sim_of({sim});
    upload(S, 0, sim);
    ck(ecsg_update_stress_ex(S.sim, 0, top, bottom), "UpdateStress", S.sim);
    download(S, 0, sim, 3, 8);
}

void UpdateGhostVZ(Field sim1[9], Field sim2[9], Field *stiff1[9], Field *stiff2[9], real **coeff1, real **coeff2,
                   Array &A, Array &B, int mode)
{
    (void)A; (void)B;   // the reference's work arrays; the device has its own
    GridRec &F = grid_of(sim1), &C = grid_of(sim2);
    note_coeff(F, coeff1);
    note_coeff(C, coeff2);
    learn_stiff(F, stiff1);
    learn_stiff(C, stiff2);
    SimRec &S = interface_of(sim1, sim2, mode);
    upload(S, 0, sim1);
    upload(S, 1, sim2);
    ck(ecsg_ghost_vz(S.sim, 1), "UpdateGhostVZ", S.sim);
    download(S, 0, sim1, 2, 2);
    download(S, 1, sim2, 2, 2);
}

void UpdateGhostSXZ(Field sim1[9], Field sim2[9], Field *buoy1, Field *buoy2, real **coeff1, real **coeff2,
                    Array &g_sxz2, Array &A, Array &B, Array &g_tmp, int mode)
{
    (void)A; (void)B; (void)g_tmp;
    GridRec &F = grid_of(sim1), &C = grid_of(sim2);
    note_coeff(F, coeff1);
    note_coeff(C, coeff2);
    learn_buoy(F, buoy1);
    learn_buoy(C, buoy2);
    SimRec &S = interface_of(sim1, sim2, mode);
    upload(S, 0, sim1);
    upload(S, 1, sim2);
    if (mode == ECSG_MODE_II) {   // explicit interpolation: g_sxz2 is not used (update_ghost_sxz.cpp:37-84)
        ck(ecsg_ghost_sxz(S.sim, 1), "UpdateGhostSXZ", S.sim);
        download(S, 0, sim1, 7, 7);
        download(S, 1, sim2, 7, 7);
        return;
    }
    // the Jacobi warm start lives in the caller's g_sxz2 ((nx2+1) x (ny2+1), x fastest)
    const size_t nxy = (size_t)(C.n[0] + 1) * (C.n[1] + 1);
    std::vector<double> X(nxy);
    for (size_t q = 0; q < nxy; q++) X[q] = (double)g_sxz2.GetPtr1()[q];
    ck(ecsg_set_sxz_state(S.sim, 1, X.data()), "UpdateGhostSXZ", S.sim);
    ck(ecsg_ghost_sxz(S.sim, 1), "UpdateGhostSXZ", S.sim);
    ck(ecsg_get_sxz_state(S.sim, 1, X.data(), nullptr, nullptr, nullptr), "UpdateGhostSXZ", S.sim);
    for (size_t q = 0; q < nxy; q++) g_sxz2.GetPtr1()[q] = (real)X[q];
    download(S, 0, sim1, 7, 7);
    download(S, 1, sim2, 7, 7);
}

void UpdateGhostSYZ(Field sim1[9], Field sim2[9], Field *buoy1, Field *buoy2, real **coeff1, real **coeff2, int mode)
{
    GridRec &F = grid_of(sim1), &C = grid_of(sim2);
    note_coeff(F, coeff1);
    note_coeff(C, coeff2);
    learn_buoy(F, buoy1);
    learn_buoy(C, buoy2);
    SimRec &S = interface_of(sim1, sim2, mode);
    upload(S, 0, sim1);
    upload(S, 1, sim2);
    ck(ecsg_ghost_syz(S.sim, 1), "UpdateGhostSYZ", S.sim);
    download(S, 0, sim1, 6, 6);
    download(S, 1, sim2, 6, 6);
}

// The device derives densities and compliances from the medium it holds
// (the same formulas as InitParField / InvertParameters), so density_ptr and
// compliance_ptr are not read; the grid's energy is scaled by its cell volume.
real ComputeEnergy(const Field sim[9], const Field vel_copy[3], Field *density_ptr[3], Field *compliance_ptr[9],
                   const real grid_size[3])
{
    (void)density_ptr; (void)compliance_ptr;
    GridRec &G = grid_of(sim);
    if (!G.buoy || !G.have_stiff) die("ComputeEnergy: the grid's medium has not been seen by an operator yet");
    SimRec &S = sim_of({sim});
    std::vector<double> t;
    for (int k = 0; k < 3; k++) ck(ecsg_set_field(S.sim, 0, k, as_double(vel_copy[k], t)), "ComputeEnergy", S.sim);
    ck(ecsg_copy_vel(S.sim), "ComputeEnergy", S.sim);
    upload(S, 0, sim);
    double e = 0.0;
    ck(ecsg_energy(S.sim, &e), "ComputeEnergy", S.sim);   // cell volume 1 (steps of 1)
    return (real)(e * (double)grid_size[0] * (double)grid_size[1] * (double)grid_size[2]);
}

namespace {
void residues(int group, int num_grids, Field **sim, std::vector<float> **res_vec)
{
    for (int i = 0; i + 1 < num_grids; i++) {
        SimRec &S = interface_of(sim[i], sim[i + 1]);
        upload(S, 0, sim[i]);
        upload(S, 1, sim[i + 1]);
        double out[9];
        ck(ecsg_residues(S.sim, 1, 1 << group, out), "compute_res", S.sim);
        for (int j = 0; j < 3; j++) res_vec[i][3 * group + j].push_back((float)out[3 * group + j]);
    }
}
} // namespace

void compute_res_sxz_vx(int num_grids, Grid grids[], Field **sim, std::vector<float> **res_vec)
{
    (void)grids;
    residues(0, num_grids, sim, res_vec);
}

void compute_res_syz_vy(int num_grids, Grid grids[], Field **sim, std::vector<float> **res_vec)
{
    (void)grids;
    residues(1, num_grids, sim, res_vec);
}

void compute_res_szz_vz(int num_grids, Grid grids[], Field **sim, std::vector<float> **res_vec)
{
    (void)grids;
    residues(2, num_grids, sim, res_vec);
}
