/*
 * ecsg_oracle.c -- CPU restatement of the ECSG composite-staggered-grid time step.
 *
 * TEST INFRASTRUCTURE ONLY. This file is the checker for the CUDA product path.
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg load it;
 * nothing under ecsg_b200/ links, calls or falls back to it.
 *
 * Precision: IEEE double throughout (the reference's shipped precision,
 * init.hpp:16-18).  Build flags match the reference build (no -march, no FMA)
 * so that the straight-line stencil restatements round like the reference.
 *
 * Storage follows the reference Field layout (field.cpp:85-149): x fastest,
 * extents [0,n] on node dims and [0,n-1] on staggered dims, R halo cells on both
 * sides of every dim.  Component order of the 9 simulation fields follows
 * init_del_sim.cpp:14-24: vx vy vz sxx syy szz syz sxz sxy.  Stiffness order
 * follows update_stress.cpp:17-25: c11 c22 c33 c23 c13 c12 c44 c55 c66.
 *
 * Interface operators are written for a general odd-or-even refinement ratio r.
 * The reference hard-codes r = 2 (update_ghost_sxz.cpp:15, update_ghost_syz.cpp:5);
 * at r = 2 the general formulas here reduce to the reference's expressions
 * (same equations, different summation order).  The derivation:
 *   prolongation P per dim: node-type dims use linear interpolation from the
 *   interior coarse nodes (boundary coarse nodes count as zero); cell-type dims
 *   copy the coarse cell value into its r fine cells.
 *   The coarse interface value after an update equals the restriction
 *   R = P^T / r^2 of the fine interface values; the fine ghost is
 *   -(last fine interior) + P(coarse ghost + coarse first interior).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>
#include <stdint.h>

typedef struct {
    double *p;          /* address of element (-R,-R,-R) */
    int len[3];
    int R;
    int pos[3];
    int end[3];         /* start is 0 on every dim */
} ofield;

typedef struct {
    int n[3];
    int R;
    ofield f[9];        /* vx vy vz sxx syy szz syz sxz sxy */
    ofield buoy;        /* position (0,0,0), R = 0 */
    ofield c[9];        /* c11 c22 c33 c23 c13 c12 c44 c55 c66, staggered, R = 0 */
    double coeff[3][6]; /* coeff[d][k] = c_k * dt / h_d (init_del_fdcoeff.cpp:7-22) */
} ogrid;

static inline double *AT(const ofield *f, int i0, int i1, int i2)
{
    return f->p + ((int64_t)(i2 + f->R) * f->len[1] + (i1 + f->R)) * f->len[0] + (i0 + f->R);
}
#define V(f, a, b, c) (*AT((f), (a), (b), (c)))

/* ------------------------------------------------------------------------- */
/* Velocity update: update_vel.cpp:4-249                                      */
/* ------------------------------------------------------------------------- */
/* mirror_fix = 0 reproduces the reference exactly.  mirror_fix = 1 runs the vy
 * y-wall mirrors over vy's own z-extent [0, nz] instead of vz's [0, nz-1]
 * (update_vel.cpp:211-218, 239-246): on the fine side of an interface the
 * plane z = nz is updated (bottom = 0), and without its wall mirror the
 * summation-by-parts identity, hence the composite energy, leaks there. */
void o_update_vel(ogrid *g, int top, int bottom, int top_bc, int mirror_fix)
{
    ofield *vx = &g->f[0], *vy = &g->f[1], *vz = &g->f[2];
    ofield *sxx = &g->f[3], *syy = &g->f[4], *szz = &g->f[5];
    ofield *syz = &g->f[6], *sxz = &g->f[7], *sxy = &g->f[8];
    const ofield *b = &g->buoy;
    const int R = g->R;
    const double *c0 = g->coeff[0], *c1 = g->coeff[1], *c2 = g->coeff[2];

    if (top && top_bc == 1) /* free surface: the top plane is updated (update_vel.cpp:17-18) */
        top = 0;

    /* vx, walls in x and y excluded (update_vel.cpp:30-37) */
#pragma omp parallel for
    for (int iz = top; iz <= vx->end[2] - bottom; iz++)
        for (int iy = 1; iy < vx->end[1]; iy++)
            for (int ir = 0; ir < R; ir++)
                for (int ix = 1; ix < vx->end[0]; ix++)
                    V(vx, ix, iy, iz) += V(b, ix, iy, iz)
                        * (c0[ir] * (V(sxx, ix + ir, iy, iz) - V(sxx, ix - ir - 1, iy, iz))
                         + c1[ir] * (V(sxy, ix, iy + ir, iz) - V(sxy, ix, iy - ir - 1, iz))
                         + c2[ir] * (V(sxz, ix, iy, iz + ir) - V(sxz, ix, iy, iz - ir - 1)));

    /* vy, buoyancy averaged over 4 nodes in (x,y) (update_vel.cpp:43-53) */
#pragma omp parallel for
    for (int iz = top; iz <= vy->end[2] - bottom; iz++)
        for (int iy = 0; iy <= vy->end[1]; iy++)
            for (int ir = 0; ir < R; ir++)
                for (int ix = 0; ix <= vy->end[0]; ix++)
                    V(vy, ix, iy, iz) += 0.25 * (V(b, ix, iy, iz) + V(b, ix + 1, iy, iz)
                                               + V(b, ix, iy + 1, iz) + V(b, ix + 1, iy + 1, iz))
                        * (c0[ir] * (V(sxy, ix + ir + 1, iy, iz) - V(sxy, ix - ir, iy, iz))
                         + c2[ir] * (V(syz, ix, iy, iz + ir) - V(syz, ix, iy, iz - ir - 1))
                         + c1[ir] * (V(syy, ix, iy + ir + 1, iz) - V(syy, ix, iy - ir, iz)));

    /* vz, buoyancy averaged over 4 nodes in (x,z), y walls excluded (update_vel.cpp:59-69) */
#pragma omp parallel for
    for (int iz = 0; iz <= vz->end[2]; iz++)
        for (int iy = 1; iy < vz->end[1]; iy++)
            for (int ir = 0; ir < R; ir++)
                for (int ix = 0; ix <= vz->end[0]; ix++)
                    V(vz, ix, iy, iz) += 0.25 * (V(b, ix, iy, iz) + V(b, ix, iy, iz + 1)
                                               + V(b, ix + 1, iy, iz) + V(b, ix + 1, iy, iz + 1))
                        * (c0[ir] * (V(sxz, ix + ir + 1, iy, iz) - V(sxz, ix - ir, iy, iz))
                         + c2[ir] * (V(szz, ix, iy, iz + ir + 1) - V(szz, ix, iy, iz - ir))
                         + c1[ir] * (V(syz, ix, iy + ir, iz) - V(syz, ix, iy - ir - 1, iz)));

    /* Odd mirrors into the halos, in the reference's order (update_vel.cpp:73-246).
     * Several loops use vz's extents for vx/vy; kept as in the reference. */
    if (top) {
        for (int iy = 0; iy <= vz->end[1]; iy++)
            for (int ir = 1; ir <= R - top_bc; ir++)
                for (int ix = 0; ix <= vz->end[0]; ix++)
                    V(vz, ix, iy, -ir) = -V(vz, ix, iy, ir - 1);
        for (int iy = 0; iy <= vx->end[1]; iy++)
            for (int ir = 1; ir < R; ir++)
                for (int ix = 0; ix <= vz->end[0]; ix++)
                    V(vx, ix, iy, -ir) = -V(vx, ix, iy, ir);
        for (int iy = 0; iy <= vy->end[1]; iy++)
            for (int ir = 1; ir < R; ir++)
                for (int ix = 0; ix <= vz->end[0]; ix++)
                    V(vy, ix, iy, -ir) = -V(vy, ix, iy, ir);
    }
    if (bottom) {
        int iz = vz->end[2];
        for (int iy = 0; iy <= vz->end[1]; iy++)
            for (int ir = 1; ir <= R; ir++)
                for (int ix = 0; ix <= vz->end[0]; ix++)
                    V(vz, ix, iy, iz + ir) = -V(vz, ix, iy, iz - ir + 1);
        iz = vx->end[2];
        for (int iy = 0; iy <= vx->end[1]; iy++)
            for (int ir = 1; ir < R; ir++)
                for (int ix = 0; ix <= vz->end[0]; ix++)
                    V(vx, ix, iy, iz + ir) = -V(vx, ix, iy, iz - ir);
        iz = vy->end[2];
        for (int iy = 0; iy <= vy->end[1]; iy++)
            for (int ir = 1; ir < R; ir++)
                for (int ix = 0; ix <= vz->end[0]; ix++)
                    V(vy, ix, iy, iz + ir) = -V(vy, ix, iy, iz - ir);
    }
    /* x start */
    for (int iz = 0; iz <= vz->end[2]; iz++)
        for (int ir = 1; ir <= R; ir++)
            for (int iy = 0; iy <= vz->end[1]; iy++)
                V(vz, -ir, iy, iz) = -V(vz, ir - 1, iy, iz);
    for (int iz = 0; iz <= vx->end[2]; iz++)
        for (int ir = 1; ir < R; ir++)
            for (int iy = 0; iy <= vz->end[1]; iy++)
                V(vx, -ir, iy, iz) = -V(vx, ir, iy, iz);
    for (int iz = 0; iz <= vy->end[2]; iz++)
        for (int ir = 1; ir <= R; ir++)
            for (int iy = 0; iy <= vz->end[1]; iy++)
                V(vy, -ir, iy, iz) = -V(vy, ir - 1, iy, iz);
    /* x end */
    {
        int ix = vz->end[0];
        for (int iz = 0; iz <= vz->end[2]; iz++)
            for (int ir = 1; ir <= R; ir++)
                for (int iy = 0; iy <= vz->end[1]; iy++)
                    V(vz, ix + ir, iy, iz) = -V(vz, ix - ir + 1, iy, iz);
        ix = vx->end[0];
        for (int iz = 0; iz <= vx->end[2]; iz++)
            for (int ir = 1; ir < R; ir++)
                for (int iy = 0; iy <= vz->end[1]; iy++)
                    V(vx, ix + ir, iy, iz) = -V(vx, ix - ir, iy, iz);
        ix = vy->end[0];
        for (int iz = 0; iz <= vy->end[2]; iz++)
            for (int ir = 1; ir <= R; ir++)
                for (int iy = 0; iy <= vz->end[1]; iy++)
                    V(vy, ix + ir, iy, iz) = -V(vy, ix - ir + 1, iy, iz);
    }
    /* y start */
    for (int iz = 0; iz <= vz->end[2]; iz++)
        for (int ir = 1; ir < R; ir++)
            for (int ix = 0; ix <= vz->end[0]; ix++)
                V(vz, ix, -ir, iz) = -V(vz, ix, ir, iz);
    for (int iz = 0; iz <= vz->end[2]; iz++)
        for (int ir = 1; ir < R; ir++)
            for (int ix = 0; ix <= vx->end[0]; ix++)
                V(vx, ix, -ir, iz) = -V(vx, ix, ir, iz);
    for (int iz = 0; iz <= (mirror_fix ? vy->end[2] : vz->end[2]); iz++)
        for (int ir = 1; ir <= R; ir++)
            for (int ix = 0; ix <= vy->end[0]; ix++)
                V(vy, ix, -ir, iz) = -V(vy, ix, ir - 1, iz);
    /* y end */
    {
        int iy = vz->end[1];
        for (int iz = 0; iz <= vz->end[2]; iz++)
            for (int ir = 1; ir < R; ir++)
                for (int ix = 0; ix <= vz->end[0]; ix++)
                    V(vz, ix, iy + ir, iz) = -V(vz, ix, iy - ir, iz);
        iy = vx->end[1];
        for (int iz = 0; iz <= vz->end[2]; iz++)
            for (int ir = 1; ir < R; ir++)
                for (int ix = 0; ix <= vx->end[0]; ix++)
                    V(vx, ix, iy + ir, iz) = -V(vx, ix, iy - ir, iz);
        iy = vy->end[1];
        for (int iz = 0; iz <= (mirror_fix ? vy->end[2] : vz->end[2]); iz++)
            for (int ir = 1; ir <= R; ir++)
                for (int ix = 0; ix <= vy->end[0]; ix++)
                    V(vy, ix, iy + ir, iz) = -V(vy, ix, iy - ir + 1, iz);
    }
}

/* ------------------------------------------------------------------------- */
/* Stress update (orthorhombic 9-Cij form): update_stress.cpp:4-311          */
/* ------------------------------------------------------------------------- */
void o_update_stress(ogrid *g, int top, int bottom, int top_bc)
{
    ofield *vx = &g->f[0], *vy = &g->f[1], *vz = &g->f[2];
    ofield *sxx = &g->f[3], *syy = &g->f[4], *szz = &g->f[5];
    ofield *syz = &g->f[6], *sxz = &g->f[7], *sxy = &g->f[8];
    const ofield *c11 = &g->c[0], *c22 = &g->c[1], *c33 = &g->c[2];
    const ofield *c23 = &g->c[3], *c13 = &g->c[4], *c12 = &g->c[5];
    const ofield *c44 = &g->c[6], *c55 = &g->c[7], *c66 = &g->c[8];
    const int R = g->R;
    const double *k0 = g->coeff[0], *k1 = g->coeff[1], *k2 = g->coeff[2];
    const int flag = (top && top_bc) ? 1 : 0;

    /* free-surface row: szz held, reduced moduli c_ij - c_i3 c_j3 / c33 (update_stress.cpp:36-65) */
    if (flag) {
        int i2 = 0;
#pragma omp parallel for
        for (int i1 = 0; i1 <= szz->end[1]; i1++)
            for (int ir = 0; ir < R; ir++)
                for (int i0 = 0; i0 <= szz->end[0]; i0++) {
                    V(sxx, i0, i1, i2) +=
                        (V(c11, i0, i1, i2) - V(c13, i0, i1, i2) * V(c13, i0, i1, i2) / V(c33, i0, i1, i2))
                            * k0[ir] * (V(vx, i0 + ir + 1, i1, i2) - V(vx, i0 - ir, i1, i2))
                        + (V(c12, i0, i1, i2) - V(c13, i0, i1, i2) * V(c23, i0, i1, i2) / V(c33, i0, i1, i2))
                            * k1[ir] * (V(vy, i0, i1 + ir, i2) - V(vy, i0, i1 - ir - 1, i2));
                    V(syy, i0, i1, i2) +=
                        (V(c12, i0, i1, i2) - V(c23, i0, i1, i2) * V(c13, i0, i1, i2) / V(c33, i0, i1, i2))
                            * k0[ir] * (V(vx, i0 + ir + 1, i1, i2) - V(vx, i0 - ir, i1, i2))
                        + (V(c22, i0, i1, i2) - V(c23, i0, i1, i2) * V(c23, i0, i1, i2) / V(c33, i0, i1, i2))
                            * k1[ir] * (V(vy, i0, i1 + ir, i2) - V(vy, i0, i1 - ir - 1, i2));
                }
    }
    /* normal stresses (update_stress.cpp:69-97) */
#pragma omp parallel for
    for (int i2 = flag; i2 <= szz->end[2]; i2++)
        for (int i1 = 0; i1 <= szz->end[1]; i1++)
            for (int ir = 0; ir < R; ir++)
                for (int i0 = 0; i0 <= szz->end[0]; i0++) {
                    double dvx = V(vx, i0 + ir + 1, i1, i2) - V(vx, i0 - ir, i1, i2);
                    double dvy = V(vy, i0, i1 + ir, i2) - V(vy, i0, i1 - ir - 1, i2);
                    double dvz = V(vz, i0, i1, i2 + ir) - V(vz, i0, i1, i2 - ir - 1);
                    V(sxx, i0, i1, i2) += V(c11, i0, i1, i2) * k0[ir] * dvx
                                        + V(c12, i0, i1, i2) * k1[ir] * dvy
                                        + V(c13, i0, i1, i2) * k2[ir] * dvz;
                    V(syy, i0, i1, i2) += V(c12, i0, i1, i2) * k0[ir] * dvx
                                        + V(c22, i0, i1, i2) * k1[ir] * dvy
                                        + V(c23, i0, i1, i2) * k2[ir] * dvz;
                    V(szz, i0, i1, i2) += V(c13, i0, i1, i2) * k0[ir] * dvx
                                        + V(c23, i0, i1, i2) * k1[ir] * dvy
                                        + V(c33, i0, i1, i2) * k2[ir] * dvz;
                }
    /* shear stresses, stored shear modulus is 2*mu hence the 0.5 (update_stress.cpp:103-133) */
#pragma omp parallel for
    for (int i2 = 0; i2 <= syz->end[2]; i2++)
        for (int i1 = 0; i1 <= syz->end[1]; i1++)
            for (int ir = 0; ir < R; ir++)
                for (int i0 = 0; i0 <= syz->end[0]; i0++)
                    V(syz, i0, i1, i2) += 0.5 * V(c44, i0, i1, i2)
                        * (k2[ir] * (V(vy, i0, i1, i2 + ir + 1) - V(vy, i0, i1, i2 - ir))
                         + k1[ir] * (V(vz, i0, i1 + ir + 1, i2) - V(vz, i0, i1 - ir, i2)));
#pragma omp parallel for
    for (int i2 = 0; i2 <= sxz->end[2]; i2++)
        for (int i1 = 0; i1 <= sxz->end[1]; i1++)
            for (int ir = 0; ir < R; ir++)
                for (int i0 = 0; i0 <= sxz->end[0]; i0++)
                    V(sxz, i0, i1, i2) += 0.5 * V(c55, i0, i1, i2)
                        * (k2[ir] * (V(vx, i0, i1, i2 + ir + 1) - V(vx, i0, i1, i2 - ir))
                         + k0[ir] * (V(vz, i0 + ir, i1, i2) - V(vz, i0 - ir - 1, i1, i2)));
#pragma omp parallel for
    for (int i2 = 0; i2 <= sxy->end[2]; i2++)
        for (int i1 = 0; i1 <= sxy->end[1]; i1++)
            for (int ir = 0; ir < R; ir++)
                for (int i0 = 0; i0 <= sxy->end[0]; i0++)
                    V(sxy, i0, i1, i2) += 0.5 * V(c66, i0, i1, i2)
                        * (k1[ir] * (V(vx, i0, i1 + ir + 1, i2) - V(vx, i0, i1 - ir, i2))
                         + k0[ir] * (V(vy, i0 + ir, i1, i2) - V(vy, i0 - ir - 1, i1, i2)));

    /* Even mirrors into the halos (update_stress.cpp:135-309). */
    { int i0 = 0;
      for (int i2 = 0; i2 <= szz->end[2]; i2++) for (int ir = 1; ir < R; ir++) for (int i1 = 0; i1 <= szz->end[1]; i1++)
          V(sxx, i0 - ir, i1, i2) = V(sxx, i0 + ir - 1, i1, i2);
      for (int i2 = 0; i2 <= sxz->end[2]; i2++) for (int ir = 1; ir < R; ir++) for (int i1 = 0; i1 <= sxz->end[1]; i1++)
          V(sxz, i0 - ir, i1, i2) = V(sxz, i0 + ir, i1, i2);
      for (int i2 = 0; i2 <= sxy->end[2]; i2++) for (int ir = 1; ir < R; ir++) for (int i1 = 0; i1 <= sxy->end[1]; i1++)
          V(sxy, i0 - ir, i1, i2) = V(sxy, i0 + ir, i1, i2);
    }
    { int i0 = szz->end[0];
      for (int i2 = 0; i2 <= szz->end[2]; i2++) for (int ir = 1; ir < R; ir++) for (int i1 = 0; i1 <= szz->end[1]; i1++)
          V(sxx, i0 + ir, i1, i2) = V(sxx, i0 - ir + 1, i1, i2);
      i0 = sxz->end[0];
      for (int i2 = 0; i2 <= sxz->end[2]; i2++) for (int ir = 1; ir < R; ir++) for (int i1 = 0; i1 <= sxz->end[1]; i1++)
          V(sxz, i0 + ir, i1, i2) = V(sxz, i0 - ir, i1, i2);
      i0 = sxy->end[0];
      for (int i2 = 0; i2 <= sxy->end[2]; i2++) for (int ir = 1; ir < R; ir++) for (int i1 = 0; i1 <= sxy->end[1]; i1++)
          V(sxy, i0 + ir, i1, i2) = V(sxy, i0 - ir, i1, i2);
    }
    { int i1 = 0;
      for (int i2 = 0; i2 <= szz->end[2]; i2++) for (int ir = 1; ir < R; ir++) for (int i0 = 0; i0 <= szz->end[0]; i0++)
          V(syy, i0, i1 - ir, i2) = V(syy, i0, i1 + ir, i2);
      for (int i2 = 0; i2 <= syz->end[2]; i2++) for (int ir = 1; ir < R; ir++) for (int i0 = 0; i0 <= syz->end[0]; i0++)
          V(syz, i0, i1 - ir, i2) = V(syz, i0, i1 + ir - 1, i2);
      for (int i2 = 0; i2 <= sxy->end[2]; i2++) for (int ir = 1; ir < R; ir++) for (int i0 = 0; i0 <= sxy->end[0]; i0++)
          V(sxy, i0, i1 - ir, i2) = V(sxy, i0, i1 + ir - 1, i2);
    }
    { int i1 = szz->end[1];
      for (int i2 = 0; i2 <= szz->end[2]; i2++) for (int ir = 1; ir < R; ir++) for (int i0 = 0; i0 <= szz->end[0]; i0++)
          V(syy, i0, i1 + ir, i2) = V(syy, i0, i1 - ir, i2);
      i1 = syz->end[1];
      for (int i2 = 0; i2 <= syz->end[2]; i2++) for (int ir = 1; ir < R; ir++) for (int i0 = 0; i0 <= syz->end[0]; i0++)
          V(syz, i0, i1 + ir, i2) = V(syz, i0, i1 - ir + 1, i2);
      i1 = sxy->end[1];
      for (int i2 = 0; i2 <= sxy->end[2]; i2++) for (int ir = 1; ir < R; ir++) for (int i0 = 0; i0 <= sxy->end[0]; i0++)
          V(sxy, i0, i1 + ir, i2) = V(sxy, i0, i1 - ir + 1, i2);
    }
    if (top) {
        for (int i1 = 1; i1 < szz->end[1]; i1++) for (int ir = 1; ir < R; ir++) for (int i0 = 0; i0 <= szz->end[0]; i0++)
            V(szz, i0, i1, -ir) = V(szz, i0, i1, ir);
        for (int i1 = 0; i1 <= syz->end[1]; i1++) for (int ir = 1; ir < R + flag; ir++) for (int i0 = 0; i0 <= syz->end[0]; i0++)
            V(syz, i0, i1, -ir) = (1 - 2 * flag) * V(syz, i0, i1, ir - 1);
        for (int i1 = 1; i1 < sxz->end[1]; i1++) for (int ir = 1; ir < R + flag; ir++) for (int i0 = 1; i0 < sxz->end[0]; i0++)
            V(sxz, i0, i1, -ir) = (1 - 2 * flag) * V(sxz, i0, i1, ir - 1);
    }
    if (bottom) {
        int i2 = szz->end[2];
        for (int i1 = 1; i1 < szz->end[1]; i1++) for (int ir = 1; ir < R; ir++) for (int i0 = 0; i0 <= szz->end[0]; i0++)
            V(szz, i0, i1, i2 + ir) = V(szz, i0, i1, i2 - ir);
        i2 = syz->end[2];
        for (int i1 = 0; i1 <= syz->end[1]; i1++) for (int ir = 1; ir < R; ir++) for (int i0 = 0; i0 <= syz->end[0]; i0++)
            V(syz, i0, i1, i2 + ir) = V(syz, i0, i1, i2 - ir + 1);
        i2 = sxz->end[2];
        for (int i1 = 1; i1 < sxz->end[1]; i1++) for (int ir = 1; ir < R; ir++) for (int i0 = 1; i0 < sxz->end[0]; i0++)
            V(sxz, i0, i1, i2 + ir) = V(sxz, i0, i1, i2 - ir + 1);
    }
}

/* ------------------------------------------------------------------------- */
/* 1-D prolongation weights.                                                  */
/* Node-type dim: fine node i = r*j + k takes (1-k/r) of coarse node j and    */
/* k/r of node j+1; coarse boundary nodes (0 and n2) contribute nothing.      */
/* Cell-type dim: fine cell i takes all of coarse cell i/r.                   */
/* ------------------------------------------------------------------------- */
static inline double pw_node(int i, int j, int r, int n2)
{
    if (j <= 0 || j >= n2) return 0.0;
    int d = i - r * j;
    if (d <= -r || d >= r) return 0.0;
    return 1.0 - (double)abs(d) / (double)r;
}
/* Same weights without the boundary mask: the reference's vz operators read
 * the coarse boundary y-nodes as they are (update_ghost_vz.cpp:177-178, 244-245);
 * vz vanishes there in every run (update_vel.cpp:60). */
static inline double pw_node_all(int i, int j, int r)
{
    int d = i - r * j;
    if (d <= -r || d >= r) return 0.0;
    return 1.0 - (double)abs(d) / (double)r;
}
static inline double pw_cell(int i, int j, int r)
{
    return (i / r == j) ? 1.0 : 0.0;
}

/* szz-rate terms of a 21-Cij medium at an interface-plane N point beyond the
 * orthorhombic ones (defined with the 21-Cij update below). */
static double gen21_szz_extra(ogrid *g, const ofield *c21, int x, int y, int z);
static void gen21_c3(const ofield *c21, int x, int y, int z, double *c13, double *c23, double *c33);

/* ------------------------------------------------------------------------- */
/* Ghost vz (energy-conserving): update_ghost_vz.cpp:124-249, general ratio  */
/* Unknown: vz2(j0, j1, -1), j0 in [0,nx2), j1 in [1,ny2-1]; one tridiagonal */
/* system along y per coarse x-cell, solved by the Thomas algorithm.          */
/* scratch: 4*(ny2+1) doubles per thread (a, b, c, d).                        */
/* ------------------------------------------------------------------------- */
void o_ghost_vz_eci21(ogrid *g1, ogrid *g2, int r, const ofield *c21_1, const ofield *c21_2);
void o_ghost_vz_eci(ogrid *g1, ogrid *g2, int r) { o_ghost_vz_eci21(g1, g2, r, NULL, NULL); }

/* c21_1/c21_2: the two grids' 21-Cij media, or NULL for the 9-Cij form. */
void o_ghost_vz_eci21(ogrid *g1, ogrid *g2, int r, const ofield *c21_1, const ofield *c21_2)
{
    ofield *vx1 = &g1->f[0], *vy1 = &g1->f[1], *vz1 = &g1->f[2], *szz1 = &g1->f[5];
    ofield *vx2 = &g2->f[0], *vy2 = &g2->f[1], *vz2 = &g2->f[2], *szz2 = &g2->f[5];
    const ofield *c33_1 = &g1->c[2], *c23_1 = &g1->c[3], *c13_1 = &g1->c[4];
    const ofield *c33_2 = &g2->c[2], *c23_2 = &g2->c[3], *c13_2 = &g2->c[4];
    const int nx2 = vz2->end[0] + 1;   /* coarse x cells */
    const int ny2 = vz2->end[1];       /* coarse y cells */
    const int nz1 = vz1->end[2] + 1;
    const double k1x = g1->coeff[0][0], k1y = g1->coeff[1][0], k1z = g1->coeff[2][0];
    const double k2x = g2->coeff[0][0], k2y = g2->coeff[1][0], k2z = g2->coeff[2][0];
    const double rr = (double)r, r3 = rr * rr * rr;
    const int m = ny2 - 1;             /* unknowns per line */

#pragma omp parallel
    {
        double *a = (double *)malloc(sizeof(double) * (m + 1));
        double *d = (double *)malloc(sizeof(double) * (m + 1));
        double *c = (double *)malloc(sizeof(double) * (m + 1));
        double *rhs = (double *)malloc(sizeof(double) * (m + 1));
#pragma omp for
        for (int j0 = 0; j0 < nx2; j0++) {
            for (int j1 = 1; j1 <= m; j1++) {
                /* coarse prediction of szz2(j0,j1,0) without the ghost term */
                double q13 = V(c13_2, j0, j1, 0), q23 = V(c23_2, j0, j1, 0), q33 = V(c33_2, j0, j1, 0), qx = 0.0;
                if (c21_2) { gen21_c3(c21_2, j0, j1, 0, &q13, &q23, &q33); qx = gen21_szz_extra(g2, c21_2, j0, j1, 0); }
                double pc = V(szz2, j0, j1, 0)
                          + q13 * k2x * (V(vx2, j0 + 1, j1, 0) - V(vx2, j0, j1, 0))
                          + q23 * k2y * (V(vy2, j0, j1, 0) - V(vy2, j0, j1 - 1, 0))
                          + q33 * k2z * V(vz2, j0, j1, 0) + qx;
                double diag = r3 * k2z * q33;
                double lo = 0.0, up = 0.0, fsum = 0.0;
                for (int i0 = r * j0; i0 < r * j0 + r; i0++) {
                    for (int i1 = r * (j1 - 1) + 1; i1 <= r * (j1 + 1) - 1; i1++) {
                        double w = pw_node(i1, j1, r, ny2);
                        double wl = pw_node(i1, j1 - 1, r, ny2), wu = pw_node(i1, j1 + 1, r, ny2);
                        double f13 = V(c13_1, i0, i1, nz1), f23 = V(c23_1, i0, i1, nz1), f33 = V(c33_1, i0, i1, nz1), fx = 0.0;
                        if (c21_1) { gen21_c3(c21_1, i0, i1, nz1, &f13, &f23, &f33); fx = gen21_szz_extra(g1, c21_1, i0, i1, nz1); }
                        double cz = f33 * k1z;
                        /* P(vz2(.,.,0)) at fine node i1 */
                        int jl = i1 / r, ju = jl + 1;
                        double pv0 = pw_node_all(i1, jl, r) * V(vz2, j0, jl, 0)
                                   + (ju <= ny2 ? pw_node_all(i1, ju, r) * V(vz2, j0, ju, 0) : 0.0);
                        double pf = V(szz1, i0, i1, nz1)
                                  + f13 * k1x * (V(vx1, i0 + 1, i1, nz1) - V(vx1, i0, i1, nz1))
                                  + f23 * k1y * (V(vy1, i0, i1, nz1) - V(vy1, i0, i1 - 1, nz1))
                                  + cz * (pv0 - 2.0 * V(vz1, i0, i1, nz1 - 1)) + fx;
                        diag += rr * w * w * cz;
                        lo += rr * w * wl * cz;
                        up += rr * w * wu * cz;
                        fsum += rr * w * pf;
                    }
                }
                a[j1] = lo; d[j1] = diag; c[j1] = up;
                rhs[j1] = r3 * pc - fsum;
            }
            /* Thomas algorithm (update_ghost_vz.cpp:209-220) */
            for (int j1 = 2; j1 <= m; j1++) {
                double w = a[j1] / d[j1 - 1];
                d[j1] -= w * c[j1 - 1];
                rhs[j1] -= w * rhs[j1 - 1];
            }
            V(vz2, j0, m, -1) = rhs[m] / d[m];
            for (int j1 = m - 1; j1 >= 1; j1--)
                V(vz2, j0, j1, -1) = (rhs[j1] - c[j1] * V(vz2, j0, j1 + 1, -1)) / d[j1];
        }
        free(a); free(d); free(c); free(rhs);
    }
    /* fine ghosts vz1(i0,i1,nz1), fine interior y nodes, all fine x cells
     * (update_ghost_vz.cpp:223-249) */
    const int nx1 = r * nx2, ny1 = r * ny2;
#pragma omp parallel for
    for (int i1 = 1; i1 < ny1; i1++) {
        int jl = i1 / r, ju = jl + 1;
        double wl = pw_node_all(i1, jl, r), wu = (ju <= ny2) ? pw_node_all(i1, ju, r) : 0.0;
        for (int i0 = 0; i0 < nx1; i0++) {
            int j0 = i0 / r;
            double s = wl * (V(vz2, j0, jl, 0) + V(vz2, j0, jl, -1));
            if (ju <= ny2) s += wu * (V(vz2, j0, ju, 0) + V(vz2, j0, ju, -1));
            V(vz1, i0, i1, nz1) = -V(vz1, i0, i1, nz1 - 1) + s;
        }
    }
}

/* ------------------------------------------------------------------------- */
/* Ghost sxz (energy-conserving): update_ghost_sxz.cpp:86-297, general ratio */
/* A (9 diagonals, k = 3*(dx+1)+(dy+1)) and B over the interior coarse nodes */
/* j = (1..nx2-1, 1..ny2-1); Jacobi2D with warm start X (zero border) and    */
/* the reference stopping rule ||X_k - X_{k-1}||_2 <= tol                      */
/* (update_ghost_sxz.cpp:231-236, 314-350).                                   */
/* X, Xt: (nx2+1)*(ny2+1), x fastest.  A: 9*(nx2-1)*(ny2-1).  B: (nx2-1)*(ny2-1). */
/* Returns the number of Jacobi sweeps; *out_tol receives the tolerance.      */
/* ------------------------------------------------------------------------- */
static void sxz_assemble(ogrid *g1, ogrid *g2, int r, double *A, double *B)
{
    ofield *vx1 = &g1->f[0], *sxx1 = &g1->f[3], *sxz1 = &g1->f[7], *sxy1 = &g1->f[8];
    ofield *vx2 = &g2->f[0], *sxx2 = &g2->f[3], *sxz2 = &g2->f[7], *sxy2 = &g2->f[8];
    const ofield *b1 = &g1->buoy, *b2 = &g2->buoy;
    const int nx2 = g2->n[0], ny2 = g2->n[1];
    const int nz1 = g1->n[2];
    const double k1x = g1->coeff[0][0], k1y = g1->coeff[1][0], k1z = g1->coeff[2][0];
    const double k2x = g2->coeff[0][0], k2y = g2->coeff[1][0], k2z = g2->coeff[2][0];
    const double rr = (double)r, r2 = rr * rr, r4 = r2 * r2;
    const int n0 = nx2 - 1, n1 = ny2 - 1;

#pragma omp parallel for
    for (int j1 = 1; j1 < ny2; j1++)
        for (int j0 = 1; j0 < nx2; j0++) {
            double a9[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
            double fsum = 0.0;
            for (int i1 = r * j1 - r + 1; i1 <= r * j1 + r - 1; i1++) {
                double wy = pw_node(i1, j1, r, ny2);
                int jy = i1 / r;
                for (int i0 = r * j0 - r + 1; i0 <= r * j0 + r - 1; i0++) {
                    double wx = pw_node(i0, j0, r, nx2);
                    int jx = i0 / r;
                    double w = wx * wy;
                    double bz = V(b1, i0, i1, nz1) * k1z;
                    /* P(sxz2(.,.,0)) at fine node (i0,i1): bilinear, interior coarse nodes */
                    double ps0 = 0.0;
                    for (int ey = 0; ey < 2; ey++)
                        for (int ex = 0; ex < 2; ex++) {
                            int cx = jx + ex, cy = jy + ey;
                            if (cx > nx2 || cy > ny2) continue;
                            double ww = pw_node(i0, cx, r, nx2) * pw_node(i1, cy, r, ny2);
                            if (ww != 0.0) ps0 += ww * V(sxz2, cx, cy, 0);
                        }
                    double pf = V(vx1, i0, i1, nz1)
                              + V(b1, i0, i1, nz1) * (k1x * (V(sxx1, i0, i1, nz1) - V(sxx1, i0 - 1, i1, nz1))
                                                    + k1y * (V(sxy1, i0, i1, nz1) - V(sxy1, i0, i1 - 1, nz1))
                                                    + k1z * (ps0 - 2.0 * V(sxz1, i0, i1, nz1 - 1)));
                    fsum += w * pf;
                    for (int dx = -1; dx <= 1; dx++)
                        for (int dy = -1; dy <= 1; dy++) {
                            double wn = pw_node(i0, j0 + dx, r, nx2) * pw_node(i1, j1 + dy, r, ny2);
                            a9[3 * (dx + 1) + (dy + 1)] += r2 * w * wn * bz;
                        }
                }
            }
            a9[4] += r4 * V(b2, j0, j1, 0) * k2z;
            double pc = V(vx2, j0, j1, 0)
                      + V(b2, j0, j1, 0) * (k2x * (V(sxx2, j0, j1, 0) - V(sxx2, j0 - 1, j1, 0))
                                          + k2y * (V(sxy2, j0, j1, 0) - V(sxy2, j0, j1 - 1, 0))
                                          + k2z * V(sxz2, j0, j1, 0));
            int q = (j1 - 1) * n0 + (j0 - 1);
            for (int k = 0; k < 9; k++) A[(int64_t)k * n0 * n1 + q] = a9[k];
            B[q] = r4 * pc - r2 * fsum;
        }
}

/* Sweeps every solve takes at least (0: the reference rule alone).  The
 * differentiated oracle (adjoint_ad.cpp) sets it so that each solve converges
 * to rounding and its derivative is that of X = A^-1 B, not of a truncated
 * iteration from the warm start. */
int o_jacobi_min_sweeps = 0;

int o_jacobi2d(double *X, const double *A, const double *B, int n0, int n1,
               double tol, double *Xt, int max_iter)
{
    const int ld = n0 + 2;
    const int64_t nn = (int64_t)n0 * n1;
    int it = 0;
    double nrm;
    do {
#pragma omp parallel for
        for (int i1 = 1; i1 <= n1; i1++)
            for (int i0 = 1; i0 <= n0; i0++)
                Xt[i1 * ld + i0] = X[i1 * ld + i0];
#pragma omp parallel for
        for (int i1 = 1; i1 <= n1; i1++)
            for (int i0 = 1; i0 <= n0; i0++) {
                int64_t q = (int64_t)(i1 - 1) * n0 + (i0 - 1);
                X[i1 * ld + i0] = (B[q]
                    - A[0 * nn + q] * Xt[(i1 - 1) * ld + (i0 - 1)]
                    - A[1 * nn + q] * Xt[(i1) * ld + (i0 - 1)]
                    - A[2 * nn + q] * Xt[(i1 + 1) * ld + (i0 - 1)]
                    - A[3 * nn + q] * Xt[(i1 - 1) * ld + (i0)]
                    - A[5 * nn + q] * Xt[(i1 + 1) * ld + (i0)]
                    - A[6 * nn + q] * Xt[(i1 - 1) * ld + (i0 + 1)]
                    - A[7 * nn + q] * Xt[(i1) * ld + (i0 + 1)]
                    - A[8 * nn + q] * Xt[(i1 + 1) * ld + (i0 + 1)]) / A[4 * nn + q];
            }
        double s = 0.0;
#pragma omp parallel for reduction(+ : s)
        for (int i1 = 1; i1 <= n1; i1++)
            for (int i0 = 1; i0 <= n0; i0++) {
                double dlt = X[i1 * ld + i0] - Xt[i1 * ld + i0];
                s += dlt * dlt;
            }
        nrm = sqrt(s);
        it++;
    } while ((nrm > tol || it < o_jacobi_min_sweeps) && (max_iter <= 0 || it < max_iter));
    return it;
}

int o_ghost_sxz_eci(ogrid *g1, ogrid *g2, int r, double *X, double *Xt, double *A, double *B,
                    int max_iter, double *out_tol)
{
    ofield *sxz1 = &g1->f[7], *sxz2 = &g2->f[7];
    const int nx2 = g2->n[0], ny2 = g2->n[1];
    const int nz1 = g1->n[2];
    const int n0 = nx2 - 1, n1 = ny2 - 1, ld = nx2 + 1;

    sxz_assemble(g1, g2, r, A, B);
    double s = 0.0;
    for (int64_t q = 0; q < (int64_t)n0 * n1; q++) s += fabs(B[q]);
    s /= (double)n0 * (double)n1;          /* Array::AvgAbs (array.cpp:172-210) */
    double tol = 1e-5 * s;
    if (tol > 1e-12) tol = 1e-12;           /* FP64 rule (update_ghost_sxz.cpp:235) */
    if (out_tol) *out_tol = tol;
    int it = o_jacobi2d(X, A, B, n0, n1, tol, Xt, max_iter);

    for (int j1 = 1; j1 < ny2; j1++)
        for (int j0 = 1; j0 < nx2; j0++)
            V(sxz2, j0, j1, -1) = X[j1 * ld + j0];
    /* fine ghosts at every interior fine node (update_ghost_sxz.cpp:255-295) */
    const int nx1 = r * nx2, ny1 = r * ny2;
#pragma omp parallel for
    for (int i1 = 1; i1 < ny1; i1++)
        for (int i0 = 1; i0 < nx1; i0++) {
            int jx = i0 / r, jy = i1 / r;
            double acc = 0.0;
            for (int ey = 0; ey < 2; ey++)
                for (int ex = 0; ex < 2; ex++) {
                    int cx = jx + ex, cy = jy + ey;
                    if (cx > nx2 || cy > ny2) continue;
                    double ww = pw_node(i0, cx, r, nx2) * pw_node(i1, cy, r, ny2);
                    if (ww != 0.0) acc += ww * (V(sxz2, cx, cy, -1) + V(sxz2, cx, cy, 0));
                }
            V(sxz1, i0, i1, nz1) = -V(sxz1, i0, i1, nz1 - 1) + acc;
        }
    return it;
}

/* ------------------------------------------------------------------------- */
/* Ghost syz (energy-conserving): update_ghost_syz.cpp:151-240, general ratio */
/* Pointwise closed form per coarse (x,y) cell.                               */
/* ------------------------------------------------------------------------- */
void o_ghost_syz_eci(ogrid *g1, ogrid *g2, int r)
{
    ofield *vy1 = &g1->f[1], *syy1 = &g1->f[4], *syz1 = &g1->f[6], *sxy1 = &g1->f[8];
    ofield *vy2 = &g2->f[1], *syy2 = &g2->f[4], *syz2 = &g2->f[6], *sxy2 = &g2->f[8];
    const ofield *b1 = &g1->buoy, *b2 = &g2->buoy;
    const int nx2 = g2->n[0], ny2 = g2->n[1];
    const int nz1 = g1->n[2];
    const double k1x = g1->coeff[0][0], k1y = g1->coeff[1][0], k1z = g1->coeff[2][0];
    const double k2x = g2->coeff[0][0], k2y = g2->coeff[1][0], k2z = g2->coeff[2][0];
    const double r2 = (double)r * (double)r;

#pragma omp parallel for
    for (int j1 = 0; j1 < ny2; j1++)
        for (int j0 = 0; j0 < nx2; j0++) {
            double c0 = 0.25 * (V(b2, j0, j1, 0) + V(b2, j0 + 1, j1, 0) + V(b2, j0, j1 + 1, 0) + V(b2, j0 + 1, j1 + 1, 0));
            double s0 = V(syz2, j0, j1, 0);
            double num = r2 * (V(vy2, j0, j1, 0)
                               + c0 * (k2x * (V(sxy2, j0 + 1, j1, 0) - V(sxy2, j0, j1, 0))
                                     + k2y * (V(syy2, j0, j1 + 1, 0) - V(syy2, j0, j1, 0))
                                     + k2z * s0));
            double den = r2 * c0 * k2z;
            for (int i1 = r * j1; i1 < r * j1 + r; i1++)
                for (int i0 = r * j0; i0 < r * j0 + r; i0++) {
                    double c = 0.25 * (V(b1, i0, i1, nz1) + V(b1, i0 + 1, i1, nz1) + V(b1, i0, i1 + 1, nz1) + V(b1, i0 + 1, i1 + 1, nz1));
                    num -= V(vy1, i0, i1, nz1)
                         + c * (k1x * (V(sxy1, i0 + 1, i1, nz1) - V(sxy1, i0, i1, nz1))
                              + k1y * (V(syy1, i0, i1 + 1, nz1) - V(syy1, i0, i1, nz1))
                              + k1z * (s0 - 2.0 * V(syz1, i0, i1, nz1 - 1)));
                    den += c * k1z;
                }
            V(syz2, j0, j1, -1) = num / den;
        }
#pragma omp parallel for
    for (int j1 = 0; j1 < ny2; j1++)
        for (int j0 = 0; j0 < nx2; j0++) {
            double t = V(syz2, j0, j1, -1) + V(syz2, j0, j1, 0);
            for (int i1 = r * j1; i1 < r * j1 + r; i1++)
                for (int i0 = r * j0; i0 < r * j0 + r; i0++)
                    V(syz1, i0, i1, nz1) = -V(syz1, i0, i1, nz1 - 1) + t;
        }
}

/* ------------------------------------------------------------------------- */
/* Intuitive interpolation (imode = 0), ratio 2 only: explicit, second-order  */
/* accurate ghosts that do not conserve the discrete energy.                  */
/* update_ghost_vz.cpp:36-123, update_ghost_sxz.cpp:37-84,                    */
/* update_ghost_syz.cpp:23-150.  Each function is written per fine ghost      */
/* point; the terms of every formula are added in the reference's order with  */
/* its constant forms (x/3, x*2/3, 0.375*x ...), so the results are bitwise    */
/* those of the reference's FP64 build.                                       */
/* ------------------------------------------------------------------------- */

/* vz: coarse ghost vz2(j0, j1, -1), j0 in [0,nx2), j1 in [1,ny2): mean of the
 * four fine vz above it (update_ghost_vz.cpp:46-50).  Fine ghost vz1(x, y, nz1)
 * for x in [0,nx1), y in [0,ny1) (y = ny1 is left as it is):
 *   interior x: 1/3 of the fine value below plus x-linear (and y-linear at odd
 *   y) weights of the coarse plane, as fractions (update_ghost_vz.cpp:57-81);
 *   x = 0 and x = nx1-1: one-sided extrapolation in x (:87-110).  The x = nx1-1
 *   formulas index vz2 with the FINE x index nx1-1, which is past the end of
 *   vz2's rows; the reference's row-major layout then reads the element that
 *   many places further on (a later row).  AT() has the same layout, so this
 *   reads the same element.  end_column = 0 leaves x = nx1-1 untouched, as the
 *   revision of update_ghost_vz.cpp:98 that declared a shadowing `int i1`
 *   instead of assigning i0 did (its stray write lands outside the field). */
void o_ghost_vz_ii(ogrid *g1, ogrid *g2, int end_column)
{
    ofield *vz1 = &g1->f[2], *vz2 = &g2->f[2];
    const int nx2 = vz2->end[0] + 1, ny2 = vz2->end[1];
    const int nz1 = vz1->end[2] + 1;
    const int nx1 = 2 * nx2, ny1 = 2 * ny2;

    for (int j1 = 1; j1 < ny2; j1++)
        for (int j0 = 0; j0 < nx2; j0++)
            V(vz2, j0, j1, -1) = 0.25 * (V(vz1, 2 * j0, 2 * j1, nz1 - 2) + V(vz1, 2 * j0 + 1, 2 * j1, nz1 - 2)
                                         + V(vz1, 2 * j0, 2 * j1, nz1 - 1) + V(vz1, 2 * j0 + 1, 2 * j1, nz1 - 1));

#pragma omp parallel for
    for (int y = 0; y < ny1; y++)
        for (int x = 0; x < nx1; x++) {
            const double own = V(vz1, x, y, nz1 - 1);
            const int j1 = y / 2, odd_y = y & 1;
            double v;
            if (x >= 1 && x <= nx1 - 2) {
                const int j0 = (x - 1) / 2, second = (x - 1) & 1;   /* x = 2 j0 + 1 + second */
                /* divisors of c(j0), c(j0+1) on the coarse row j1 (even y), or of
                 * c(j0,j1), c(j0+1,j1), c(j0,j1+1), c(j0+1,j1+1) (odd y) */
                static const double dv[2][2][4] = {{{2, 6, 0, 0}, {6, 2, 0, 0}}, {{4, 12, 4, 12}, {12, 4, 12, 4}}};
                const double *d = dv[odd_y][second];
                v = own / 3 + V(vz2, j0, j1, 0) / d[0] + V(vz2, j0 + 1, j1, 0) / d[1];
                if (odd_y) v = v + V(vz2, j0, j1 + 1, 0) / d[2] + V(vz2, j0 + 1, j1 + 1, 0) / d[3];
            } else {
                if (x == nx1 - 1 && !end_column) continue;
                const int xin = (x == 0) ? 1 : x - 1;   /* x-neighbour one column in */
                const int cx = x;                       /* coarse x index as the reference writes it */
                if (!odd_y)
                    v = own * 2 / 3 - V(vz1, xin, y, nz1 - 1) / 3 + V(vz2, cx, j1, 0) * 2 / 3;
                else   /* the neighbour term reads the even row y-1 (update_ghost_vz.cpp:93,105) */
                    v = own * 2 / 3 - V(vz1, xin, y - 1, nz1 - 1) / 3 + V(vz2, cx, j1, 0) / 3 + V(vz2, cx, j1 + 1, 0) / 3;
            }
            V(vz1, x, y, nz1) = v;
        }
}

/* sxz: coarse ghost sxz2(j0, j1, -1) at the interior coarse nodes = mean of the
 * two fine cells above (update_ghost_sxz.cpp:46-49); fine ghost at every
 * interior fine node (x, y) = 1/3 of the fine value below plus 2/3 of the
 * bilinear coarse interpolation, written per node parity (:55-81). */
void o_ghost_sxz_ii(ogrid *g1, ogrid *g2)
{
    ofield *sxz1 = &g1->f[7], *sxz2 = &g2->f[7];
    const int nx2 = g2->n[0], ny2 = g2->n[1], nz1 = g1->n[2];
    const int nx1 = 2 * nx2, ny1 = 2 * ny2;

    for (int j1 = 1; j1 < ny2; j1++)
        for (int j0 = 1; j0 < nx2; j0++)
            V(sxz2, j0, j1, -1) = 0.5 * (V(sxz1, 2 * j0, 2 * j1, nz1 - 2) + V(sxz1, 2 * j0, 2 * j1, nz1 - 1));

#pragma omp parallel for
    for (int y = 1; y < ny1; y++)
        for (int x = 1; x < nx1; x++) {
            const int j0 = x / 2, j1 = y / 2;
            const double own = V(sxz1, x, y, nz1 - 1);
            double v;
            switch ((x & 1) | ((y & 1) << 1)) {
            case 0: v = own / 3 + V(sxz2, j0, j1, 0) * 2 / 3.0; break;
            case 1: v = own / 3 + V(sxz2, j0, j1, 0) / 3 + V(sxz2, j0 + 1, j1, 0) / 3; break;
            case 2: v = own / 3 + V(sxz2, j0, j1, 0) / 3 + V(sxz2, j0, j1 + 1, 0) / 3; break;
            default:
                v = own / 3 + V(sxz2, j0, j1, 0) / 6 + V(sxz2, j0, j1 + 1, 0) / 6 + V(sxz2, j0 + 1, j1, 0) / 6
                    + V(sxz2, j0 + 1, j1 + 1, 0) / 6;
            }
            V(sxz1, x, y, nz1) = v;
        }
}

/* syz: coarse ghost syz2(j0, j1, -1) at every coarse cell = mean of the eight
 * fine values in the two cell layers above (update_ghost_syz.cpp:33-42).  Fine
 * ghost at every fine cell (x, y):
 *   interior (x in [1,nx1-2], y in [1,ny1-2]): 1/3 of the fine value below plus
 *   the bilinear coarse interpolation scaled by 2/3, weights 9/24 3/24 3/24 1/24
 *   (:49-74);
 *   edges: extrapolation from the fine plane below (:78-134): at the four
 *   corners own - (x-neighbour)/3 - (inward y-neighbour)/3 + 2/3 coarse; along
 *   an edge own/3 + (the other fine cell of the same coarse cell along the
 *   edge)/3 - (inward neighbour)/3 + 2/3 coarse. */
void o_ghost_syz_ii(ogrid *g1, ogrid *g2)
{
    ofield *syz1 = &g1->f[6], *syz2 = &g2->f[6];
    const int nx2 = g2->n[0], ny2 = g2->n[1], nz1 = g1->n[2];
    const int X1 = 2 * nx2 - 1, Y1 = 2 * ny2 - 1;   /* last fine cell */

    for (int j1 = 0; j1 < ny2; j1++)
        for (int j0 = 0; j0 < nx2; j0++) {
            double s = 0.0;
            int first = 1;
            for (int dz = 2; dz >= 1; dz--)
                for (int dy = 0; dy < 2; dy++)
                    for (int dx = 0; dx < 2; dx++) {
                        double t = V(syz1, 2 * j0 + dx, 2 * j1 + dy, nz1 - dz);
                        s = first ? t : s + t;
                        first = 0;
                    }
            V(syz2, j0, j1, -1) = 0.125 * s;
        }

#pragma omp parallel for
    for (int y = 0; y <= Y1; y++)
        for (int x = 0; x <= X1; x++) {
            const double own = V(syz1, x, y, nz1 - 1);
            double v;
            if (x >= 1 && x <= X1 - 1 && y >= 1 && y <= Y1 - 1) {
                const int j0 = (x - 1) / 2, j1 = (y - 1) / 2;
                const int near = ((x - 1) & 1) | (((y - 1) & 1) << 1);   /* coarse corner nearest (x, y) */
                const double c[4] = {V(syz2, j0, j1, 0), V(syz2, j0 + 1, j1, 0), V(syz2, j0, j1 + 1, 0),
                                     V(syz2, j0 + 1, j1 + 1, 0)};
                v = own / 3;
                for (int k = 0; k < 4; k++) {
                    const int far = (k ^ near) == 3, adj = __builtin_popcount(k ^ near) == 1;
                    v = v + (far ? c[k] / 24 : (adj ? 0.125 * c[k] : 0.375 * c[k]));
                }
            } else {
                const double cc = V(syz2, x / 2, y / 2, 0) * 2 / 3;
                if (y == 0 || y == Y1) {
                    const int yin = (y == 0) ? 1 : Y1 - 1;
                    if (x == 0 || x == X1) {
                        const int xin = (x == 0) ? 1 : X1 - 1;
                        v = own - V(syz1, xin, y, nz1 - 1) / 3 - V(syz1, x, yin, nz1 - 1) / 3 + cc;
                    } else {
                        v = own / 3 + V(syz1, x - 1 + 2 * (x % 2), y, nz1 - 1) / 3 - V(syz1, x, yin, nz1 - 1) / 3 + cc;
                    }
                } else {
                    const int xin = (x == 0) ? 1 : X1 - 1;
                    v = own / 3 + V(syz1, x, y - 1 + 2 * (y % 2), nz1 - 1) / 3 - V(syz1, xin, y, nz1 - 1) / 3 + cc;
                }
            }
            V(syz1, x, y, nz1) = v;
        }
}

/* ------------------------------------------------------------------------- */
/* Energy: compute_energy.cpp:34-54 with TriMulFields (field.cpp:482-518).    */
/* dens[3]: density at vx, vy, vz positions; comp[9]: compliance in the       */
/* stiffness order; all R = 0 fields at the matching staggered positions.     */
/* ------------------------------------------------------------------------- */
static double trimul(const ofield *a, const ofield *b, const ofield *c)
{
    double res = 0.0;
#pragma omp parallel for reduction(+ : res)
    for (int i2 = 0; i2 <= a->end[2]; i2++) {
        double m2 = 1.0 - (a->pos[2] ? 0.0 : 0.5 * ((i2 == 0) || (i2 == a->end[2])));
        for (int i1 = 0; i1 <= a->end[1]; i1++) {
            double m1 = 1.0 - (a->pos[1] ? 0.0 : 0.5 * ((i1 == 0) || (i1 == a->end[1])));
            for (int i0 = 0; i0 <= a->end[0]; i0++) {
                double m0 = 1.0 - (a->pos[0] ? 0.0 : 0.5 * ((i0 == 0) || (i0 == a->end[0])));
                res += m2 * m1 * m0 * V(a, i0, i1, i2) * V(b, i0, i1, i2) * V(c, i0, i1, i2);
            }
        }
    }
    return res;
}

double o_energy(ogrid *g, const ofield *vcopy, const ofield *dens, const ofield *comp, const double *h)
{
    double e = 0.0;
    for (int i = 0; i < 3; i++) e += trimul(&dens[i], &g->f[i], &vcopy[i]);
    for (int i = 0; i < 3; i++) e += trimul(&comp[i], &g->f[i + 3], &g->f[i + 3]);
    e += 2.0 * trimul(&comp[3], &g->f[4], &g->f[5]);
    e += 2.0 * trimul(&comp[4], &g->f[3], &g->f[5]);
    e += 2.0 * trimul(&comp[5], &g->f[3], &g->f[4]);
    for (int i = 6; i < 9; i++) e += 2.0 * trimul(&comp[i], &g->f[i], &g->f[i]);
    return e * 0.5 * h[2] * h[1] * h[0];
}

/* ------------------------------------------------------------------------- */
/* Interface residues: compute_res.cpp:4-95 (fine sum - r^2 coarse sum) and   */
/* Field::AvgAbs (field.cpp:210-229).  out[9] in the reference order:         */
/* [res vx-sxz, |vx2|, |sxz2|, res vy-syz, |vy2|, |syz2|, res vz-szz, |vz2|, |szz2|] */
/* which selects the three groups computed: bit 0 vx-sxz, 1 vy-syz, 2 vz-szz. */
/* ------------------------------------------------------------------------- */
double o_avgabs(const ofield *f)
{
    double s = 0.0;
    for (int i2 = 0; i2 <= f->end[2]; i2++)
        for (int i1 = 0; i1 <= f->end[1]; i1++)
            for (int i0 = 0; i0 <= f->end[0]; i0++) s += fabs(V(f, i0, i1, i2));
    s /= (f->end[2] + 1);
    s /= (f->end[1] + 1);
    s /= (f->end[0] + 1);
    return s;
}

void o_residues(ogrid *g1, ogrid *g2, int r, int which, double *out)
{
    const int nx1 = g1->n[0], ny1 = g1->n[1], nz1 = g1->n[2];
    const int nx2 = g2->n[0], ny2 = g2->n[1];
    const double r2 = (double)r * (double)r;
    if (which & 1) {
        double res = 0.0;
        for (int i1 = 1; i1 < ny1; i1++)
            for (int i0 = 1; i0 < nx1; i0++)
                res += V(&g1->f[0], i0, i1, nz1) * (V(&g1->f[7], i0, i1, nz1 - 1) + V(&g1->f[7], i0, i1, nz1));
        for (int i1 = 1; i1 < ny2; i1++)
            for (int i0 = 1; i0 < nx2; i0++)
                res -= r2 * V(&g2->f[0], i0, i1, 0) * (V(&g2->f[7], i0, i1, -1) + V(&g2->f[7], i0, i1, 0));
        out[0] = res; out[1] = o_avgabs(&g2->f[0]); out[2] = o_avgabs(&g2->f[7]);
    }
    if (which & 2) {
        double res = 0.0;
        for (int i1 = 0; i1 < ny1; i1++)
            for (int i0 = 0; i0 < nx1; i0++)
                res += V(&g1->f[1], i0, i1, nz1) * (V(&g1->f[6], i0, i1, nz1 - 1) + V(&g1->f[6], i0, i1, nz1));
        for (int i1 = 0; i1 < ny2; i1++)
            for (int i0 = 0; i0 < nx2; i0++)
                res -= r2 * V(&g2->f[1], i0, i1, 0) * (V(&g2->f[6], i0, i1, -1) + V(&g2->f[6], i0, i1, 0));
        out[3] = res; out[4] = o_avgabs(&g2->f[1]); out[5] = o_avgabs(&g2->f[6]);
    }
    if (which & 4) {
        double res = 0.0;
        for (int i1 = 1; i1 < ny1; i1++)
            for (int i0 = 0; i0 < nx1; i0++)
                res += V(&g1->f[5], i0, i1, nz1) * (V(&g1->f[2], i0, i1, nz1 - 1) + V(&g1->f[2], i0, i1, nz1));
        for (int i1 = 1; i1 < ny2; i1++)
            for (int i0 = 0; i0 < nx2; i0++)
                res -= r2 * V(&g2->f[5], i0, i1, 0) * (V(&g2->f[2], i0, i1, -1) + V(&g2->f[2], i0, i1, 0));
        out[6] = res; out[7] = o_avgabs(&g2->f[2]); out[8] = o_avgabs(&g2->f[5]);
    }
}

/* ------------------------------------------------------------------------- */
/* General anisotropic (21 Cij) stress update.  No reference counterpart: the  */
/* reference implements the orthorhombic form only (update_stress.cpp:17-133). */
/* This is the scheme the CUDA kernel implements; with the 12 off-block       */
/* entries zero it reduces to o_update_stress (shear C44 = c44_ref / 2).      */
/*                                                                           */
/* Voigt stiffness, engineering shear strains.  Storage (R = 0 fields):      */
/*   N  = normal-stress position (1,0,0): slots 0..14 =                      */
/*        C11 C12 C13 C22 C23 C33 C14 C15 C16 C24 C25 C26 C34 C35 C36        */
/*   L4 = syz position (1,1,1): 15 C44, 16 C45, 17 C46                        */
/*   L5 = sxz position (0,0,1): 18 C55, 19 C56                                */
/*   L6 = sxy position (0,1,0): 20 C66                                        */
/* Strain increments e1..e3 at N, e4 at L4, e5 at L5, e6 at L6 (the          */
/* reference's differences times dt/h).  A coupling between positions X and  */
/* Y uses one coefficient per link, taken at one end (N-end for N-L4/L5/L6,   */
/* the L4-end for L4-L5 and L4-L6, the L5-end for L5-L6), and is applied in   */
/* both directions (stress at X gets coeff * average of the strain at Y; the  */
/* stress at Y gets the average over X of coeff * strain), so the discrete   */
/* stiffness operator is symmetric and the energy 1/2 (rho v, v) +           */
/* 1/2 (eps, sigma) is conserved.  Averages run over the 2 or 4 neighbours of */
/* a point and drop neighbours outside the position's extent (a one-sided     */
/* value in that dim), the closure compatible with the trapezoid weights of  */
/* the energy; interface and mirror planes count as outside.  On a free      */
/* surface (top grid, top_bc = 1) szz is held and e3 at the surface is the   */
/* value that keeps its rate zero.                                           */
/* eps (may be NULL): 6 strain accumulators at the stress positions (R = 0),  */
/* incremented by the strains used, for the energy check.                    */
/* ------------------------------------------------------------------------- */
typedef struct {
    int ex[3];          /* extent end per dim */
} oext;

static inline int in_ext(const int e[3], int x, int y, int z)
{
    return x >= 0 && x <= e[0] && y >= 0 && y <= e[1] && z >= 0 && z <= e[2];
}

/* strain increments at existing points (velocities read with their halos) */
static double e1_at(ogrid *g, int x, int y, int z) { return g->coeff[0][0] * (V(&g->f[0], x + 1, y, z) - V(&g->f[0], x, y, z)); }
static double e2_at(ogrid *g, int x, int y, int z) { return g->coeff[1][0] * (V(&g->f[1], x, y, z) - V(&g->f[1], x, y - 1, z)); }
static double e3_at(ogrid *g, int x, int y, int z) { return g->coeff[2][0] * (V(&g->f[2], x, y, z) - V(&g->f[2], x, y, z - 1)); }
static double e4_at(ogrid *g, int x, int y, int z)
{
    return g->coeff[2][0] * (V(&g->f[1], x, y, z + 1) - V(&g->f[1], x, y, z)) + g->coeff[1][0] * (V(&g->f[2], x, y + 1, z) - V(&g->f[2], x, y, z));
}
static double e5_at(ogrid *g, int x, int y, int z)
{
    return g->coeff[2][0] * (V(&g->f[0], x, y, z + 1) - V(&g->f[0], x, y, z)) + g->coeff[0][0] * (V(&g->f[2], x, y, z) - V(&g->f[2], x - 1, y, z));
}
static double e6_at(ogrid *g, int x, int y, int z)
{
    return g->coeff[1][0] * (V(&g->f[0], x, y + 1, z) - V(&g->f[0], x, y, z)) + g->coeff[0][0] * (V(&g->f[1], x, y, z) - V(&g->f[1], x - 1, y, z));
}

/* Average of a quantity q over the neighbours (x+dx_k, y+dy_k, z+dz_k) of a
 * point, two offsets per averaged dim ({a0,a1} in dim d), dropping offsets
 * whose point lies outside the source extent. */
typedef double (*qfun)(void *ctx, int x, int y, int z);

static double avg2d(qfun q, void *ctx, const int ext[3], int x, int y, int z, int d0, int a0, int b0, int d1, int a1, int b1)
{
    double s = 0.0, wsum0 = 0.0;
    int off0[2] = {a0, b0}, off1[2] = {a1, b1};
    /* weights per dim: 1/2 each if both exist, else 1 for the existing one */
    double acc = 0.0;
    int ok0[2], ok1[2];
    for (int i = 0; i < 2; i++) {
        int p[3] = {x, y, z};
        p[d0] += off0[i];
        ok0[i] = (p[d0] >= 0 && p[d0] <= ext[d0]);
        int q2[3] = {x, y, z};
        q2[d1] += off1[i];
        ok1[i] = (q2[d1] >= 0 && q2[d1] <= ext[d1]);
    }
    double w0[2], w1[2];
    for (int i = 0; i < 2; i++) {
        w0[i] = ok0[i] ? ((ok0[0] && ok0[1]) ? 0.5 : 1.0) : 0.0;
        w1[i] = ok1[i] ? ((ok1[0] && ok1[1]) ? 0.5 : 1.0) : 0.0;
    }
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) {
            double w = w0[i] * w1[j];
            if (w == 0.0) continue;
            int p[3] = {x, y, z};
            p[d0] += off0[i];
            p[d1] += off1[j];
            acc += w * q(ctx, p[0], p[1], p[2]);
        }
    (void)s; (void)wsum0;
    return acc;
}

typedef struct {
    ogrid *g;
    const ofield *c21;
    int flag;           /* free surface on this grid */
    double *e3s;        /* condensed e3 at the surface plane (nx * (ny+1)), or NULL */
} g21ctx;

static double C21(const g21ctx *c, int k, int x, int y, int z) { return V(&c->c21[k], x, y, z); }

static double q_e4(void *v, int x, int y, int z) { return e4_at(((g21ctx *)v)->g, x, y, z); }
static double q_e5(void *v, int x, int y, int z) { return e5_at(((g21ctx *)v)->g, x, y, z); }
static double q_e6(void *v, int x, int y, int z) { return e6_at(((g21ctx *)v)->g, x, y, z); }
static double q_Q45(void *v, int x, int y, int z) { g21ctx *c = (g21ctx *)v; return C21(c, 16, x, y, z) * e4_at(c->g, x, y, z); }
static double q_Q46(void *v, int x, int y, int z) { g21ctx *c = (g21ctx *)v; return C21(c, 17, x, y, z) * e4_at(c->g, x, y, z); }
static double q_Q56(void *v, int x, int y, int z) { g21ctx *c = (g21ctx *)v; return C21(c, 19, x, y, z) * e5_at(c->g, x, y, z); }

/* extents of the four positions on grid g */
static void exts(const ogrid *g, int eN[3], int e4[3], int e5[3], int e6[3])
{
    int nx = g->n[0], ny = g->n[1], nz = g->n[2];
    eN[0] = nx - 1; eN[1] = ny; eN[2] = nz;
    e4[0] = nx - 1; e4[1] = ny - 1; e4[2] = nz - 1;
    e5[0] = nx; e5[1] = ny; e5[2] = nz - 1;
    e6[0] = nx; e6[1] = ny - 1; e6[2] = nz;
}

static double Abar4(g21ctx *c, const int e4[3], int x, int y, int z) { return avg2d(q_e4, c, e4, x, y, z, 1, -1, 0, 2, -1, 0); }
static double Abar5(g21ctx *c, const int e5[3], int x, int y, int z) { return avg2d(q_e5, c, e5, x, y, z, 0, 0, 1, 2, -1, 0); }
static double Abar6(g21ctx *c, const int e6[3], int x, int y, int z) { return avg2d(q_e6, c, e6, x, y, z, 0, 0, 1, 1, -1, 0); }

/* e3 used at an N point: native, or condensed on the free surface */
static double e3_used(g21ctx *c, const int e4[3], const int e5[3], const int e6[3], int x, int y, int z)
{
    if (c->flag && z == 0) {
        double num = C21(c, 2, x, y, z) * e1_at(c->g, x, y, z) + C21(c, 4, x, y, z) * e2_at(c->g, x, y, z)
                   + C21(c, 12, x, y, z) * Abar4(c, e4, x, y, z) + C21(c, 13, x, y, z) * Abar5(c, e5, x, y, z)
                   + C21(c, 14, x, y, z) * Abar6(c, e6, x, y, z);
        return -num / C21(c, 5, x, y, z);
    }
    return e3_at(c->g, x, y, z);
}

typedef struct {
    g21ctx *c;
    int e4[3], e5[3], e6[3];
    int j;   /* which P: 4, 5 or 6 */
} pctx;

static double q_P(void *v, int x, int y, int z)
{
    pctx *p = (pctx *)v;
    g21ctx *c = p->c;
    /* rows i = 1..3 of column j: C_ij at N slots (j=4: 6,9,12; j=5: 7,10,13; j=6: 8,11,14) */
    int k0 = 6 + (p->j - 4);
    double e1 = e1_at(c->g, x, y, z), e2 = e2_at(c->g, x, y, z), e3 = e3_used(c, p->e4, p->e5, p->e6, x, y, z);
    return C21(c, k0, x, y, z) * e1 + C21(c, k0 + 3, x, y, z) * e2 + C21(c, k0 + 6, x, y, z) * e3;
}

void o_update_stress21(ogrid *g, const ofield *c21, int top, int bottom, int top_bc, ofield *eps)
{
    (void)bottom;
    ofield *sxx = &g->f[3], *syy = &g->f[4], *szz = &g->f[5], *syz = &g->f[6], *sxz = &g->f[7], *sxy = &g->f[8];
    const int nx = g->n[0], ny = g->n[1], nz = g->n[2];
    const int flag = (top && top_bc) ? 1 : 0;
    int eN[3], e4[3], e5[3], e6[3];
    exts(g, eN, e4, e5, e6);
    g21ctx C = {g, c21, flag, NULL};
    /* all increments from the old velocities, then applied (velocities are not changed here) */
    const int64_t nN = (int64_t)nx * (ny + 1) * (nz + 1);
    double *dN = (double *)calloc(3 * nN, sizeof(double));
    double *eN3 = eps ? (double *)calloc(3 * nN, sizeof(double)) : NULL;
#pragma omp parallel for
    for (int z = 0; z <= nz; z++)
        for (int y = 0; y <= ny; y++)
            for (int x = 0; x < nx; x++) {
                double e1 = e1_at(g, x, y, z), e2 = e2_at(g, x, y, z), e3 = e3_used(&C, e4, e5, e6, x, y, z);
                double a4 = Abar4(&C, e4, x, y, z), a5 = Abar5(&C, e5, x, y, z), a6 = Abar6(&C, e6, x, y, z);
                int64_t q = ((int64_t)z * (ny + 1) + y) * nx + x;
                for (int i = 0; i < 3; i++) {
                    /* row i: C_i1 C_i2 C_i3 then C_i4 C_i5 C_i6 */
                    static const int rowc[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
                    double d = C21(&C, rowc[i][0], x, y, z) * e1 + C21(&C, rowc[i][1], x, y, z) * e2 + C21(&C, rowc[i][2], x, y, z) * e3
                             + C21(&C, 6 + 3 * i, x, y, z) * a4 + C21(&C, 7 + 3 * i, x, y, z) * a5 + C21(&C, 8 + 3 * i, x, y, z) * a6;
                    dN[i * nN + q] = d;
                }
                if (eN3) { eN3[q] = e1; eN3[nN + q] = e2; eN3[2 * nN + q] = e3; }
            }
    const int64_t n4 = (int64_t)nx * ny * nz, n5 = (int64_t)(nx + 1) * (ny + 1) * nz, n6 = (int64_t)(nx + 1) * ny * (nz + 1);
    double *d4 = (double *)calloc(n4, sizeof(double)), *d5 = (double *)calloc(n5, sizeof(double)), *d6 = (double *)calloc(n6, sizeof(double));
#pragma omp parallel for
    for (int z = 0; z < nz; z++)
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++) {
                pctx P = {&C, {e4[0], e4[1], e4[2]}, {e5[0], e5[1], e5[2]}, {e6[0], e6[1], e6[2]}, 4};
                double d = C21(&C, 15, x, y, z) * e4_at(g, x, y, z)
                         + C21(&C, 16, x, y, z) * avg2d(q_e5, &C, e5, x, y, z, 0, 0, 1, 1, 0, 1)
                         + C21(&C, 17, x, y, z) * avg2d(q_e6, &C, e6, x, y, z, 0, 0, 1, 2, 0, 1)
                         + avg2d(q_P, &P, eN, x, y, z, 1, 0, 1, 2, 0, 1);
                d4[((int64_t)z * ny + y) * nx + x] = d;
            }
#pragma omp parallel for
    for (int z = 0; z < nz; z++)
        for (int y = 0; y <= ny; y++)
            for (int x = 0; x <= nx; x++) {
                pctx P = {&C, {e4[0], e4[1], e4[2]}, {e5[0], e5[1], e5[2]}, {e6[0], e6[1], e6[2]}, 5};
                double d = C21(&C, 18, x, y, z) * e5_at(g, x, y, z)
                         + C21(&C, 19, x, y, z) * avg2d(q_e6, &C, e6, x, y, z, 1, -1, 0, 2, 0, 1)
                         + avg2d(q_Q45, &C, e4, x, y, z, 0, -1, 0, 1, -1, 0)
                         + avg2d(q_P, &P, eN, x, y, z, 0, -1, 0, 2, 0, 1);
                d5[((int64_t)z * (ny + 1) + y) * (nx + 1) + x] = d;
            }
#pragma omp parallel for
    for (int z = 0; z <= nz; z++)
        for (int y = 0; y < ny; y++)
            for (int x = 0; x <= nx; x++) {
                pctx P = {&C, {e4[0], e4[1], e4[2]}, {e5[0], e5[1], e5[2]}, {e6[0], e6[1], e6[2]}, 6};
                double d = C21(&C, 20, x, y, z) * e6_at(g, x, y, z)
                         + avg2d(q_Q46, &C, e4, x, y, z, 0, -1, 0, 2, -1, 0)
                         + avg2d(q_Q56, &C, e5, x, y, z, 1, 0, 1, 2, -1, 0)
                         + avg2d(q_P, &P, eN, x, y, z, 0, -1, 0, 1, 0, 1);
                d6[((int64_t)z * ny + y) * (nx + 1) + x] = d;
            }
    /* apply */
    for (int z = 0; z <= nz; z++)
        for (int y = 0; y <= ny; y++)
            for (int x = 0; x < nx; x++) {
                int64_t q = ((int64_t)z * (ny + 1) + y) * nx + x;
                V(sxx, x, y, z) += dN[q];
                V(syy, x, y, z) += dN[nN + q];
                if (!(flag && z == 0)) V(szz, x, y, z) += dN[2 * nN + q];
                if (eps) {
                    V(&eps[0], x, y, z) += eN3[q];
                    V(&eps[1], x, y, z) += eN3[nN + q];
                    V(&eps[2], x, y, z) += eN3[2 * nN + q];
                }
            }
    for (int z = 0; z < nz; z++)
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++) {
                V(syz, x, y, z) += d4[((int64_t)z * ny + y) * nx + x];
                if (eps) V(&eps[3], x, y, z) += e4_at(g, x, y, z);
            }
    for (int z = 0; z < nz; z++)
        for (int y = 0; y <= ny; y++)
            for (int x = 0; x <= nx; x++) {
                V(sxz, x, y, z) += d5[((int64_t)z * (ny + 1) + y) * (nx + 1) + x];
                if (eps) V(&eps[4], x, y, z) += e5_at(g, x, y, z);
            }
    for (int z = 0; z <= nz; z++)
        for (int y = 0; y < ny; y++)
            for (int x = 0; x <= nx; x++) {
                V(sxy, x, y, z) += d6[((int64_t)z * ny + y) * (nx + 1) + x];
                if (eps) V(&eps[5], x, y, z) += e6_at(g, x, y, z);
            }
    /* free-surface odd mirrors of syz, sxz as the reference (update_stress.cpp:260-277) */
    if (flag) {
        for (int y = 0; y < ny; y++)
            for (int x = 0; x < nx; x++) V(syz, x, y, -1) = -V(syz, x, y, 0);
        for (int y = 1; y < ny; y++)
            for (int x = 1; x < nx; x++) V(sxz, x, y, -1) = -V(sxz, x, y, 0);
    }
    free(dN); free(eN3); free(d4); free(d5); free(d6);
}

static void gen21_c3(const ofield *c21, int x, int y, int z, double *c13, double *c23, double *c33)
{
    *c13 = V(&c21[2], x, y, z);
    *c23 = V(&c21[4], x, y, z);
    *c33 = V(&c21[5], x, y, z);
}

static double gen21_szz_extra(ogrid *g, const ofield *c21, int x, int y, int z)
{
    int eN[3], e4[3], e5[3], e6[3];
    exts(g, eN, e4, e5, e6);
    g21ctx C = {g, c21, 0, NULL};
    return V(&c21[12], x, y, z) * Abar4(&C, e4, x, y, z) + V(&c21[13], x, y, z) * Abar5(&C, e5, x, y, z)
         + V(&c21[14], x, y, z) * Abar6(&C, e6, x, y, z);
}
