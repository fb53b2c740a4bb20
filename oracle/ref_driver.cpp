// ref_driver.cpp -- C-ABI harness around the reference's own functions.
//
// TEST INFRASTRUCTURE ONLY.  Compiled together with the unmodified reference
// sources (taken from where they lie, never copied into this repository) and
// the project RSF stand-in into oracle/_ref/libecsg_ref{64,32}.so.  Tests use it
// to pin the C restatement (ecsg_oracle.c) against the reference function by
// function, and bench.py's reference arm uses ecsg_ref_run() to time the
// reference's OpenMP time loop on the host cores.
//
// Set-up goes through the reference's own initialisers (InitParField,
// InitSim, InitGhostContainer, InitFDcoeff, InitSrc, InitRecTrace, InitRes;
// sim_utils.hpp:10-122) with the same key=value parameters as main.cpp:31-67.
// Media are handed over as in-memory RSF inputs (ecsg_rsf_register_memory).
// ecsg_ref_step() runs one iteration of main.cpp:165-261 in the same order.
#include "sim_utils.hpp"
#include "array.hpp"
#include <rsf.hh>
#include <omp.h>
#include <chrono>
#include <cmath>
#include <cstring>
#include <string>
#include <vector>

namespace {
struct RefState {
    bool ready = false;
    int num_grids = 0, radius = 1, imode = 1, top_bc = 0, num_threads = 1;
    bool check_energy = false, verb = false, has_src = false, has_rec = false;
    real dt = 0;
    Grid *grids = nullptr;
    Field *buoys = nullptr;
    Field **stiffs_obj = nullptr, **dens_obj = nullptr, **comp_obj = nullptr;
    Field ***stiffs_ptr = nullptr, ***dens_ptr = nullptr, ***comp_ptr = nullptr;
    Field **sim = nullptr, **vel_copy = nullptr;
    Array *g_sxz = nullptr, *g_tmp = nullptr, *A_sxz = nullptr, *B_sxz = nullptr, *A_vz = nullptr, *B_vz = nullptr;
    real ***coeff = nullptr;
    int src_grid = 0, src_loc[3] = {0, 0, 0};
    std::valarray<float> src_trace;
    int n_rec = 0;
    int **rec_loc = nullptr;
    std::vector<real> *rec_data = nullptr;
    std::vector<float> **res_vec = nullptr;
    std::vector<real> energy_vec;
} S;

Field *field_of(int g, int kind, int k)
{
    if (!S.ready || g < 0 || g >= S.num_grids) return nullptr;
    switch (kind) {
    case 0: return (k >= 0 && k < 9) ? &S.sim[g][k] : nullptr;      // simulation fields
    case 1: return (k >= 0 && k < 9) ? S.stiffs_ptr[g][k] : nullptr; // stiffness view
    case 2: return &S.buoys[g];                                       // buoyancy
    case 3: return (S.check_energy && k >= 0 && k < 3) ? S.dens_ptr[g][k] : nullptr;
    case 4: return (S.check_energy && k >= 0 && k < 9) ? S.comp_ptr[g][k] : nullptr;
    case 5: return (S.check_energy && k >= 0 && k < 3) ? &S.vel_copy[g][k] : nullptr;
    }
    return nullptr;
}
} // namespace

extern "C" {

int ecsg_ref_real_size(void) { return (int)sizeof(real); }

// argv holds key=value pairs exactly as main.cpp would receive them.
int ecsg_ref_setup(int argc, char **argv)
{
    if (S.ready) return -1;
    sf_init(argc, argv);
    iRSF par(0);
    par.get("num_threads", S.num_threads, 1);
    omp_set_num_threads(S.num_threads);
    par.get("check_energy", S.check_energy, false);
    par.get("radius", S.radius, 0);
    double dt = -1.0;
    par.get("dt", dt, -1.);
    S.dt = (real)dt;
    par.get("imode", S.imode, 1);
    par.get("verb", S.verb, false);
    par.get("top_bc", S.top_bc, 0);
    par.get("num_grids", S.num_grids, 1);
    if (S.radius <= 0 || S.dt <= 0 || S.num_grids < 1) return -2;
    std::string tmp;
    par.get("src", tmp, std::string(""));
    S.has_src = !tmp.empty();
    par.get("rec_in", tmp, std::string(""));
    S.has_rec = !tmp.empty();

    InitParField(S.num_grids, S.check_energy, S.grids, S.buoys, S.stiffs_obj, S.stiffs_ptr,
                 S.dens_obj, S.dens_ptr, S.comp_obj, S.comp_ptr);
    InitSim(S.num_grids, S.radius, S.check_energy, S.grids, S.sim, S.vel_copy);
    InitGhostContainer(S.num_grids, S.grids, S.num_threads, S.g_sxz, S.g_tmp, S.A_sxz, S.B_sxz, S.A_vz, S.B_vz);
    if (S.has_src) InitSrc(S.src_grid, S.src_loc, S.src_trace, S.grids, S.num_grids, S.dt);
    InitFDcoeff(S.num_grids, S.grids, S.radius, S.dt, S.coeff);
    if (S.has_rec) InitRecTrace(S.num_grids, S.grids, S.n_rec, S.rec_loc, S.rec_data);
    if (S.num_grids > 1) InitRes(S.num_grids, S.res_vec);
    if (S.check_energy)
        for (int i = 0; i < S.num_grids; i++)
            for (int j = 0; j < 3; j++) S.vel_copy[i][j] = S.sim[i][j];
    S.energy_vec.clear();
    S.ready = true;
    return 0;
}

void ecsg_ref_teardown(void)
{
    if (!S.ready) return;
    if (S.num_grids > 1) DelRes(S.num_grids, S.res_vec);
    if (S.has_rec) DelRecTrace(S.n_rec, S.rec_loc, S.rec_data);
    DelFDCoeff(S.num_grids, S.coeff);
    DelGhostContainer(S.g_sxz, S.g_tmp, S.A_sxz, S.B_sxz, S.A_vz, S.B_vz);
    DelSim(S.num_grids, S.check_energy, S.sim, S.vel_copy);
    DelParField(S.num_grids, S.check_energy, S.grids, S.buoys, S.stiffs_obj, S.stiffs_ptr,
                S.dens_obj, S.dens_ptr, S.comp_obj, S.comp_ptr);
    ecsg_rsf_clear_memory();
    S = RefState();
}

int ecsg_ref_set_threads(int n)
{
    omp_set_num_threads(n);
    return n;
}

// Shape of a stored field: len[3], pos[3], end[3].
int ecsg_ref_field_shape(int g, int kind, int k, int *len, int *pos, int *end)
{
    Field *f = field_of(g, kind, k);
    if (!f) return -1;
    for (int d = 0; d < 3; d++) { len[d] = f->GetLen(d); pos[d] = f->GetPos(d); end[d] = f->GetEnd(d); }
    return 0;
}

int ecsg_ref_get_field(int g, int kind, int k, double *out)
{
    Field *f = field_of(g, kind, k);
    if (!f) return -1;
    long n = (long)f->GetLen(0) * f->GetLen(1) * f->GetLen(2);
    const real *p = f->GetPtr1();
    for (long i = 0; i < n; i++) out[i] = (double)p[i];
    return 0;
}

int ecsg_ref_set_field(int g, int kind, int k, const double *in)
{
    Field *f = field_of(g, kind, k);
    if (!f) return -1;
    long n = (long)f->GetLen(0) * f->GetLen(1) * f->GetLen(2);
    real *p = f->GetPtr1();
    for (long i = 0; i < n; i++) p[i] = (real)in[i];
    return 0;
}

int ecsg_ref_get_coeff(int g, double *out)
{
    if (!S.ready || g < 0 || g >= S.num_grids) return -1;
    for (int d = 0; d < 3; d++)
        for (int k = 0; k < S.radius; k++) out[d * S.radius + k] = (double)S.coeff[g][d][k];
    return 0;
}

int ecsg_ref_grid(int g, int *size, double *step, double *origin)
{
    if (!S.ready || g < 0 || g >= S.num_grids) return -1;
    for (int d = 0; d < 3; d++) {
        size[d] = S.grids[g].size[d];
        step[d] = (double)S.grids[g].step[d];
        origin[d] = (double)S.grids[g].origin[d];
    }
    return 0;
}

// Warm-start buffer of the sxz Jacobi solve at interface i: (nx2+1)*(ny2+1).
int ecsg_ref_get_gsxz(int i, double *out)
{
    if (!S.ready || i < 0 || i >= S.num_grids - 1) return -1;
    int n0, n1;
    S.g_sxz[i].size(&n0, &n1);
    for (int b = 0; b < n1; b++)
        for (int a = 0; a < n0; a++) out[b * n0 + a] = (double)S.g_sxz[i].GetVal(a, b);
    return 0;
}
int ecsg_ref_set_gsxz(int i, const double *in)
{
    if (!S.ready || i < 0 || i >= S.num_grids - 1) return -1;
    int n0, n1;
    S.g_sxz[i].size(&n0, &n1);
    for (int b = 0; b < n1; b++)
        for (int a = 0; a < n0; a++) S.g_sxz[i].SetVal(a, b) = (real)in[b * n0 + a];
    return 0;
}

int ecsg_ref_src(int *grid, int *loc, int *len)
{
    if (!S.ready || !S.has_src) return -1;
    *grid = S.src_grid;
    for (int d = 0; d < 3; d++) loc[d] = S.src_loc[d];
    *len = (int)S.src_trace.size();
    return 0;
}

int ecsg_ref_rec(int *n, int *loc4)
{
    if (!S.ready || !S.has_rec) return -1;
    *n = S.n_rec;
    if (loc4)
        for (int i = 0; i < S.n_rec; i++)
            for (int j = 0; j < 4; j++) loc4[4 * i + j] = S.rec_loc[i][j];
    return 0;
}

// Individual reference calls (top/bottom flags as main.cpp:179-180, 228-229).
int ecsg_ref_update_vel(int g)
{
    if (!S.ready || g < 0 || g >= S.num_grids) return -1;
    UpdateVel(S.sim[g], S.buoys[g], S.coeff[g], S.radius, g == 0, g == S.num_grids - 1, S.top_bc);
    return 0;
}
int ecsg_ref_update_stress(int g)
{
    if (!S.ready || g < 0 || g >= S.num_grids) return -1;
    UpdateStress(S.sim[g], S.stiffs_ptr[g], S.coeff[g], S.radius, g == 0, g == S.num_grids - 1, S.top_bc);
    return 0;
}
int ecsg_ref_ghost_vz(int i)
{
    if (!S.ready || i < 1 || i >= S.num_grids) return -1;
    UpdateGhostVZ(S.sim[i - 1], S.sim[i], S.stiffs_ptr[i - 1], S.stiffs_ptr[i], S.coeff[i - 1], S.coeff[i],
                  S.A_vz[i - 1], S.B_vz[i - 1], S.imode);
    return 0;
}
int ecsg_ref_ghost_sxz(int i)
{
    if (!S.ready || i < 1 || i >= S.num_grids) return -1;
    UpdateGhostSXZ(S.sim[i - 1], S.sim[i], &S.buoys[i - 1], &S.buoys[i], S.coeff[i - 1], S.coeff[i],
                   S.g_sxz[i - 1], S.A_sxz[i - 1], S.B_sxz[i - 1], S.g_tmp[i - 1], S.imode);
    return 0;
}
int ecsg_ref_ghost_syz(int i)
{
    if (!S.ready || i < 1 || i >= S.num_grids) return -1;
    UpdateGhostSYZ(S.sim[i - 1], S.sim[i], &S.buoys[i - 1], &S.buoys[i], S.coeff[i - 1], S.coeff[i], S.imode);
    return 0;
}
int ecsg_ref_copy_vel(void)
{
    if (!S.ready || !S.check_energy) return -1;
    for (int i = 0; i < S.num_grids; i++)
        for (int j = 0; j < 3; j++) S.vel_copy[i][j] = S.sim[i][j];
    return 0;
}
double ecsg_ref_energy(void)
{
    if (!S.ready || !S.check_energy) return NAN;
    real e = 0;
    for (int i = 0; i < S.num_grids; i++)
        e += ComputeEnergy(S.sim[i], S.vel_copy[i], S.dens_ptr[i], S.comp_ptr[i], S.grids[i].step);
    return (double)e;
}
// Residues of the 3 interface pairs for interface 0..num_grids-2, in the
// res_trace order (compute_res.cpp:4-95).  which: bit0 vx-sxz, bit1 vy-syz, bit2 vz-szz.
int ecsg_ref_residues(int which, double *out)
{
    if (!S.ready || S.num_grids < 2) return -1;
    size_t n0 = S.res_vec[0][0].size(), n3 = S.res_vec[0][3].size(), n6 = S.res_vec[0][6].size();
    if (which & 1) compute_res_sxz_vx(S.num_grids, S.grids, S.sim, S.res_vec);
    if (which & 2) compute_res_syz_vy(S.num_grids, S.grids, S.sim, S.res_vec);
    if (which & 4) compute_res_szz_vz(S.num_grids, S.grids, S.sim, S.res_vec);
    for (int k = 0; k < S.num_grids - 1; k++) {
        for (int j = 0; j < 3; j++) {
            if (which & 1) out[9 * k + j] = S.res_vec[k][j][n0];
            if (which & 2) out[9 * k + 3 + j] = S.res_vec[k][3 + j][n3];
            if (which & 4) out[9 * k + 6 + j] = S.res_vec[k][6 + j][n6];
        }
    }
    return 0;
}

// One iteration of main.cpp:165-261 (movies excluded).  Receiver samples go to
// rec_out[n_rec] (may be null); the energy, if enabled, to *energy.
int ecsg_ref_step(int niter, double *rec_out, double *energy)
{
    if (!S.ready) return -1;
    if (S.check_energy)
        for (int i = 0; i < S.num_grids; i++)
            for (int j = 0; j < 3; j++) S.vel_copy[i][j] = S.sim[i][j];
    for (int i = 0; i < S.num_grids; i++)
        UpdateVel(S.sim[i], S.buoys[i], S.coeff[i], S.radius, i == 0, i == S.num_grids - 1, S.top_bc);
    for (int i = 0; i < S.n_rec; i++) {
        real v = S.sim[S.rec_loc[i][0]][0].GetVal(S.rec_loc[i][1], S.rec_loc[i][2], S.rec_loc[i][3]);
        S.rec_data[i].push_back(v);
        if (rec_out) rec_out[i] = (double)v;
    }
    if (S.verb && S.num_grids > 1) {
        compute_res_sxz_vx(S.num_grids, S.grids, S.sim, S.res_vec);
        compute_res_syz_vy(S.num_grids, S.grids, S.sim, S.res_vec);
    }
    if (S.has_src && niter < (int)S.src_trace.size())
        S.sim[S.src_grid][0].SetVal(S.src_loc[0], S.src_loc[1], S.src_loc[2]) += 1000 * S.src_trace[niter];
    for (int i = 1; i < S.num_grids; i++)
        UpdateGhostVZ(S.sim[i - 1], S.sim[i], S.stiffs_ptr[i - 1], S.stiffs_ptr[i], S.coeff[i - 1], S.coeff[i],
                      S.A_vz[i - 1], S.B_vz[i - 1], S.imode);
    if (S.verb && S.num_grids > 1) compute_res_szz_vz(S.num_grids, S.grids, S.sim, S.res_vec);
    if (S.check_energy) {
        real e = 0;
        for (int i = 0; i < S.num_grids; i++)
            e += ComputeEnergy(S.sim[i], S.vel_copy[i], S.dens_ptr[i], S.comp_ptr[i], S.grids[i].step);
        S.energy_vec.push_back(e);
        if (energy) *energy = (double)e;
    }
    for (int i = 0; i < S.num_grids; i++)
        UpdateStress(S.sim[i], S.stiffs_ptr[i], S.coeff[i], S.radius, i == 0, i == S.num_grids - 1, S.top_bc);
    for (int i = 1; i < S.num_grids; i++) {
        UpdateGhostSXZ(S.sim[i - 1], S.sim[i], &S.buoys[i - 1], &S.buoys[i], S.coeff[i - 1], S.coeff[i],
                       S.g_sxz[i - 1], S.A_sxz[i - 1], S.B_sxz[i - 1], S.g_tmp[i - 1], S.imode);
        UpdateGhostSYZ(S.sim[i - 1], S.sim[i], &S.buoys[i - 1], &S.buoys[i], S.coeff[i - 1], S.coeff[i], S.imode);
    }
    return 0;
}

// Runs nsteps iterations starting at niter0 and returns the wall time in
// seconds (std::chrono, not the reference's clock() CPU time).
double ecsg_ref_run(int niter0, int nsteps)
{
    if (!S.ready) return -1.0;
    auto t0 = std::chrono::steady_clock::now();
    for (int n = 0; n < nsteps; n++) ecsg_ref_step(niter0 + n, nullptr, nullptr);
    auto t1 = std::chrono::steady_clock::now();
    return std::chrono::duration<double>(t1 - t0).count();
}

} // extern "C"
