// adjoint_ad.cpp -- FP64 CPU adjoint of the oracle's time loop.
// TEST INFRASTRUCTURE ONLY: the checker for the device misfit gradients
// (ecsg_misfit_gradient); nothing under ecsg_b200/ links or calls it.
//
// The oracle's own restatement (ecsg_oracle.c: o_update_vel, the 21-Cij
// o_update_stress21 with its free-surface condensation and mirrors, the
// interface solves o_ghost_vz_eci21 / o_ghost_sxz_eci / o_ghost_syz_eci) is
// compiled here a second time with its arithmetic type replaced by the taped
// adouble of ad_tape.hpp.  Running the loop of main.cpp:165-261 (the order of
// oracle.py's OracleRun.step: velocities, receiver samples, source, vz ghosts,
// stresses, sxz and syz ghosts) records every operation; the misfit
// L = 1/2 sum_n sum_rec (v_rec(n) - d(n))^2 is then differentiated in reverse
// with respect to every node buoyancy and every one of the 21 stiffness slots
// of every grid.  The gradient is therefore the exact adjoint (in IEEE double)
// of the oracle's forward, obtained without deriving any transpose by hand:
// an independent check of the hand-written device adjoint kernels.
//
// The Jacobi solves of the sxz ghosts take at least `jacobi_min_sweeps`
// sweeps (o_jacobi_min_sweeps), enough to converge to rounding, so that their
// derivative is that of the exact solve X = A^-1 B, which is what the device
// adjoint transposes (a solve truncated at the reference's tolerance from a
// warm start has a different derivative).
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>

#include "ad_tape.hpp"

using adt::adouble;
using adt::fabs;
using adt::sqrt;

#define double adouble
#include "ecsg_oracle.c"
#undef double

namespace {

// Field shape of the oracle's layout (field.cpp:85-98): node dims n+1 points,
// staggered dims n, R halo cells each side.
struct Owned {
    std::vector<adouble> a;
    ofield f;
};

void make_field(Owned &o, const int n[3], const int pos[3], int R)
{
    int len[3];
    for (int d = 0; d < 3; d++) len[d] = (pos[d] ? n[d] : n[d] + 1) + 2 * R;
    o.a.assign((size_t)len[0] * len[1] * len[2], adouble());
    o.f.p = o.a.data();
    for (int d = 0; d < 3; d++) {
        o.f.len[d] = len[d];
        o.f.pos[d] = pos[d];
        o.f.end[d] = len[d] - 1 - 2 * R;
    }
    o.f.R = R;
}

const int kSimPos[9][3] = {{0, 0, 0}, {1, 1, 0}, {1, 0, 1}, {1, 0, 0}, {1, 0, 0},
                           {1, 0, 0}, {1, 1, 1}, {0, 0, 1}, {0, 1, 0}};
const int kStiffPos[9][3] = {{1, 0, 0}, {1, 0, 0}, {1, 0, 0}, {1, 0, 0}, {1, 0, 0},
                             {1, 0, 0}, {1, 1, 1}, {0, 0, 1}, {0, 1, 0}};
// 21-Cij slots: 0..14 at N (1,0,0), 15..17 at L4 (1,1,1), 18..19 at L5 (0,0,1), 20 at L6 (0,1,0)
const int *slot_pos(int k)
{
    static const int N[3] = {1, 0, 0}, L4[3] = {1, 1, 1}, L5[3] = {0, 0, 1}, L6[3] = {0, 1, 0};
    return k < 15 ? N : (k < 18 ? L4 : (k < 20 ? L5 : L6));
}

} // namespace

extern "C" {

// One grid of the problem: sizes, dt/h per dim (radius 1), the medium (node
// buoyancy and the 21 slots, without halo, x fastest) and the outputs.
typedef struct {
    int n[3];
    double coeff[3];
    const double *buoy;
    const double *c21[21];
    double *g_buoy;
    double *g_c21[21];
} ad_grid;

// Returns 0, -1 on bad arguments, -2 when the run needs a tape of more than
// 2^31 entries.  src = (grid, x, y, z, component), the
// source adds float(scale * trace[n]) for n < src_nt; rec = (grid, x, y, z)
// per receiver, sampling component rec_comp after the velocity update and
// before the source; obs[n * nrec + i].
int ad_misfit_gradient(int ng, ad_grid *G, int r, int top_bc, int mirror_fix, int nsteps, const int *src,
                       const float *src_trace, int src_nt, float src_scale, int nrec, const int *rec, int rec_comp,
                       const float *obs, int jacobi_min_sweeps, double *loss, long long *tape_len)
{
    if (ng < 1 || ng > 8 || nsteps < 1 || r < 2) return -1;
    adt::tape().clear();
    const int R = 1;
    std::vector<ogrid> og(ng);
    std::vector<Owned> fields(9 * ng), stiff(9 * ng), buoy(ng), c21(21 * ng);
    std::vector<std::vector<ofield>> c21f(ng, std::vector<ofield>(21));
    for (int g = 0; g < ng; g++) {
        ogrid &o = og[g];
        memset(&o, 0, sizeof o);
        for (int d = 0; d < 3; d++) o.n[d] = G[g].n[d];
        o.R = R;
        for (int k = 0; k < 9; k++) {
            make_field(fields[9 * g + k], G[g].n, kSimPos[k], R);
            o.f[k] = fields[9 * g + k].f;
            // the 9-slot form is read (and overridden) by the 21-Cij vz ghosts
            make_field(stiff[9 * g + k], G[g].n, kStiffPos[k], 0);
            o.c[k] = stiff[9 * g + k].f;
        }
        static const int node[3] = {0, 0, 0};
        make_field(buoy[g], G[g].n, node, 0);
        for (size_t q = 0; q < buoy[g].a.size(); q++) buoy[g].a[q] = adt::variable(G[g].buoy[q]);
        o.buoy = buoy[g].f;
        for (int k = 0; k < 21; k++) {
            Owned &c = c21[21 * g + k];
            make_field(c, G[g].n, slot_pos(k), 0);
            for (size_t q = 0; q < c.a.size(); q++) c.a[q] = adt::variable(G[g].c21[k][q]);
            c21f[g][k] = c.f;
        }
        for (int d = 0; d < 3; d++) o.coeff[d][0] = G[g].coeff[d];
    }
    // sxz solve work arrays per interface (X warm start kept across steps)
    std::vector<std::vector<adouble>> X(ng), Xt(ng), A(ng), B(ng);
    for (int i = 1; i < ng; i++) {
        const int nx2 = G[i].n[0], ny2 = G[i].n[1];
        X[i].assign((size_t)(nx2 + 1) * (ny2 + 1), adouble());
        Xt[i].assign((size_t)(nx2 + 1) * (ny2 + 1), adouble());
        A[i].assign((size_t)9 * (nx2 - 1) * (ny2 - 1), adouble());
        B[i].assign((size_t)(nx2 - 1) * (ny2 - 1), adouble());
    }
    o_jacobi_min_sweeps = jacobi_min_sweeps;
    adouble L(0.0);
    try {
    for (int n = 0; n < nsteps; n++) {
        for (int g = 0; g < ng; g++) o_update_vel(&og[g], g == 0, g == ng - 1, top_bc, mirror_fix);
        for (int i = 0; i < nrec; i++) {
            const int *p = rec + 4 * i;
            const adouble res = V(&og[p[0]].f[rec_comp], p[1], p[2], p[3]) - adouble((double)obs[(size_t)n * nrec + i]);
            L = L + adouble(0.5) * res * res;
        }
        if (src && n < src_nt) {
            const float amp = src_scale * src_trace[n];
            V(&og[src[0]].f[src[4]], src[1], src[2], src[3]) += adouble((double)amp);
        }
        for (int i = 1; i < ng; i++) o_ghost_vz_eci21(&og[i - 1], &og[i], r, c21f[i - 1].data(), c21f[i].data());
        for (int g = 0; g < ng; g++) o_update_stress21(&og[g], c21f[g].data(), g == 0, g == ng - 1, top_bc, nullptr);
        for (int i = 1; i < ng; i++) {
            o_ghost_sxz_eci(&og[i - 1], &og[i], r, X[i].data(), Xt[i].data(), A[i].data(), B[i].data(), 0, nullptr);
            o_ghost_syz_eci(&og[i - 1], &og[i], r);
        }
    }
    } catch (const std::exception &) {   // the tape outgrew 32-bit indices
        o_jacobi_min_sweeps = 0;
        adt::tape().clear();
        return -2;
    }
    o_jacobi_min_sweeps = 0;
    *loss = L.v;
    if (tape_len) *tape_len = (long long)adt::tape().e.size();
    const std::vector<double> adj = adt::reverse(L);
    for (int g = 0; g < ng; g++) {
        for (size_t q = 0; q < buoy[g].a.size(); q++) G[g].g_buoy[q] = adj[buoy[g].a[q].i];
        for (int k = 0; k < 21; k++) {
            const Owned &c = c21[21 * g + k];
            for (size_t q = 0; q < c.a.size(); q++) G[g].g_c21[k][q] = adj[c.a[q].i];
        }
    }
    adt::tape().clear();
    adt::tape().e.shrink_to_fit();
    return 0;
}

} // extern "C"
