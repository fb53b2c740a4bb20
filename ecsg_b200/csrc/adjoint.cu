// adjoint.cu -- transposes of the grid operators for misfit gradients.
//
// No reference counterpart.  Every forward operator of the time loop is an
// affine map of the full state (all box entries of the 9 fields, halos and
// ghosts included) whose linear part depends on the medium.  For an operator
// s_out = Op_m(s_in) these kernels apply, given the adjoint lambda of s_out,
//   lambda_in = Op^T lambda_out                  (in place on lambda), and
//   g_m      += d<lambda_out, Op_m(s_in)>/dm     (gradient accumulators),
// reading the forward fields the operator used.  They are written as reverse
// mode of the forward code, term for term, scattering with atomics; the
// operator order is reversed by the caller.
//
// Operators here (one grid each):
//   velocity update (update_vel.cpp:20-69 ranges, radius 1) and its odd halo
//   mirrors, receiver sampling (main.cpp:182-184), and the 21-Cij stress
//   update of stress21.cu including the free-surface condensation and the
//   surface mirrors of syz/sxz.  The interface solves are in interface.cu.
//
// Adjoint state of a grid: lambda of the 9 fields in the grid's box layout;
// gradients: g_b at the nodes (buoyancy) and g_c[21] at the slot positions.
// Work buffers (zero between operators): W[0..5] adjoints of the strain
// increments e1..e6, W[6..8] of the link products Q45, Q46, Q56, W[9..11] of
// P4, P5, P6.
#include "adjoint.cuh"
#include "gen21_device.cuh"

namespace ecsg {

enum { W_E1 = 0, W_E2, W_E3, W_E4, W_E5, W_E6, W_Q45, W_Q46, W_Q56, W_P4, W_P5, W_P6 };

// closure weights of a 2 x 2 neighbourhood (avg4 of gen21_device.cuh)
template <typename T>
__device__ __forceinline__ void weights4(const bool (&a)[2], const bool (&b)[2], T (&w)[2][2])
{
    T wa0, wa1, wb0, wb1;
    w2<T>(a[0], a[1], wa0, wa1);
    w2<T>(b[0], b[1], wb0, wb1);
    w[0][0] = mul_(wa0, wb0); w[0][1] = mul_(wa0, wb1);
    w[1][0] = mul_(wa1, wb0); w[1][1] = mul_(wa1, wb1);
}

// ---------------------------------------------------------------------------
// Velocity update: v += b * (k . D sigma) on the forward ranges.
// lambda_sigma += (b D)^T lambda_v; g_b += lambda_v * (k . D sigma), the vy
// and vz buoyancies being 4-node means (1/4 to each node).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void vel_adj_kernel(GridDev<T> G, AdjDev<T> A, int zt, int bottom)
{
    const Geo &g = G.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int64_t n = (int64_t)nx * ny * (nz + 1);   // x < nx, y < ny cover every updated point
    const int sx = 1, sy = g.px, sz = g.px * g.py;
    const T k0 = G.k[0], k1 = G.k[1], k2 = G.k[2], q = T(0.25);
    const T *b = G.b;
    const T *sxx = G.f[SXX], *syy = G.f[SYY], *szz = G.f[SZZ], *syz = G.f[SYZ], *sxz = G.f[SXZ], *sxy = G.f[SXY];
    T *lsxx = A.l[SXX], *lsyy = A.l[SYY], *lszz = A.l[SZZ], *lsyz = A.l[SYZ], *lsxz = A.l[SXZ], *lsxy = A.l[SXY];
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int ix = (int)(t % nx), iy = (int)((t / nx) % ny), iz = (int)(t / ((int64_t)nx * ny));
        const int p = g.idx(ix, iy, iz);
        const bool zin = iz >= zt && iz <= nz - bottom;
        if (ix >= 1 && iy >= 1 && zin) {   // vx
            const T a = A.l[VX][p];
            if (a != T(0)) {
                const T d = add_(add_(mul_(k0, sub_(sxx[p], sxx[p - sx])), mul_(k1, sub_(sxy[p], sxy[p - sy]))),
                                 mul_(k2, sub_(sxz[p], sxz[p - sz])));
                atom(A.gb + p, mul_(a, d));
                const T u = mul_(a, b[p]);
                atom(lsxx + p, mul_(k0, u)); atom(lsxx + p - sx, -mul_(k0, u));
                atom(lsxy + p, mul_(k1, u)); atom(lsxy + p - sy, -mul_(k1, u));
                atom(lsxz + p, mul_(k2, u)); atom(lsxz + p - sz, -mul_(k2, u));
            }
        }
        if (zin) {   // vy
            const T a = A.l[VY][p];
            if (a != T(0)) {
                const T bb = mul_(q, add_(add_(add_(b[p], b[p + sx]), b[p + sy]), b[p + sy + sx]));
                const T d = add_(add_(mul_(k0, sub_(sxy[p + sx], sxy[p])), mul_(k2, sub_(syz[p], syz[p - sz]))),
                                 mul_(k1, sub_(syy[p + sy], syy[p])));
                const T gq = mul_(q, mul_(a, d));
                atom(A.gb + p, gq); atom(A.gb + p + sx, gq); atom(A.gb + p + sy, gq); atom(A.gb + p + sy + sx, gq);
                const T u = mul_(a, bb);
                atom(lsxy + p + sx, mul_(k0, u)); atom(lsxy + p, -mul_(k0, u));
                atom(lsyz + p, mul_(k2, u)); atom(lsyz + p - sz, -mul_(k2, u));
                atom(lsyy + p + sy, mul_(k1, u)); atom(lsyy + p, -mul_(k1, u));
            }
        }
        if (iy >= 1 && iz <= nz - 1) {   // vz
            const T a = A.l[VZ][p];
            if (a != T(0)) {
                const T bb = mul_(q, add_(add_(add_(b[p], b[p + sz]), b[p + sx]), b[p + sz + sx]));
                const T d = add_(add_(mul_(k0, sub_(sxz[p + sx], sxz[p])), mul_(k2, sub_(szz[p + sz], szz[p]))),
                                 mul_(k1, sub_(syz[p], syz[p - sy])));
                const T gq = mul_(q, mul_(a, d));
                atom(A.gb + p, gq); atom(A.gb + p + sz, gq); atom(A.gb + p + sx, gq); atom(A.gb + p + sz + sx, gq);
                const T u = mul_(a, bb);
                atom(lsxz + p + sx, mul_(k0, u)); atom(lsxz + p, -mul_(k0, u));
                atom(lszz + p + sz, mul_(k2, u)); atom(lszz + p, -mul_(k2, u));
                atom(lsyz + p, mul_(k1, u)); atom(lsyz + p - sy, -mul_(k1, u));
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Velocity mirrors (stencil.cu vel_mirror_kernel): each assignment h = -v[i]
// transposes to lambda[i] -= lambda[h], lambda[h] = 0, phase 1 before phase 0.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void mirror_adj(T *l, int h, int i)
{
    const T v = l[h];
    l[h] = T(0);
    if (v != T(0)) atom(l + i, -v);
}

template <typename T>
__global__ void vel_mirror_adj_kernel(Geo g, T *lvy, T *lvz, int phase, int top_rigid, int bottom, int mirror_fix)
{
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (phase == 0) {
        const int64_t nA = top_rigid ? (int64_t)(ny + 1) * nx : 0;
        const int64_t nB = bottom ? (int64_t)(ny + 1) * nx : 0;
        const int64_t nC = (int64_t)nz * (ny + 1);
        const int64_t nD = (int64_t)(nz + 1) * (ny + 1);
        if (t < nA) { int ix = t % nx, iy = t / nx; mirror_adj(lvz, g.idx(ix, iy, -1), g.idx(ix, iy, 0)); return; }
        t -= nA;
        if (t < nB) { int ix = t % nx, iy = t / nx; mirror_adj(lvz, g.idx(ix, iy, nz), g.idx(ix, iy, nz - 1)); return; }
        t -= nB;
        if (t < nC) { int iy = t % (ny + 1), iz = t / (ny + 1); mirror_adj(lvz, g.idx(-1, iy, iz), g.idx(0, iy, iz)); return; }
        t -= nC;
        if (t < nC) { int iy = t % (ny + 1), iz = t / (ny + 1); mirror_adj(lvz, g.idx(nx, iy, iz), g.idx(nx - 1, iy, iz)); return; }
        t -= nC;
        if (t < nD) { int iy = t % (ny + 1), iz = t / (ny + 1); mirror_adj(lvy, g.idx(-1, iy, iz), g.idx(0, iy, iz)); return; }
        t -= nD;
        if (t < nD) { int iy = t % (ny + 1), iz = t / (ny + 1); mirror_adj(lvy, g.idx(nx, iy, iz), g.idx(nx - 1, iy, iz)); return; }
    } else {
        const int64_t nG = (int64_t)(nz + (mirror_fix ? 1 : 0)) * nx;
        if (t < nG) { int ix = t % nx, iz = t / nx; mirror_adj(lvy, g.idx(ix, -1, iz), g.idx(ix, 0, iz)); return; }
        t -= nG;
        if (t < nG) { int ix = t % nx, iz = t / nx; mirror_adj(lvy, g.idx(ix, ny, iz), g.idx(ix, ny - 1, iz)); return; }
    }
}

// Receiver sampling: lambda_v[rec] += residual (a receiver samples a velocity).
template <typename T>
__global__ void rec_adj_kernel(const RecAdj<T> R)
{
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= R.nrec) return;
    const T v = R.res[i];
    if (v != T(0)) atom(R.lbase[R.grid[i]] + R.off[i], v);
}

// ---------------------------------------------------------------------------
// 21-Cij stress update (stress21.cu), reverse mode in four stages.
//   S1 per point: the sigma adjoints of N, L6, L4, L5 outputs -> gradients of
//      the coefficients that multiply forward values, W[e] of own strains,
//      scattered W[e] / W[Q] / W[P] of the averaged neighbours
//   S2 per point: W[Q], W[P] -> gradients and own W[e]
//   S3 free surface: the condensed e3 -> e1, e2, the averaged e4..e6
//   S4 per point: W[e] -> lambda_v (transpose of the differences)
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T e3u_at(const GridDev<T> &G, const Ext &E, bool surf, int x, int y, int z, int p)
{
    return e3_used(G, E, surf, x, y, z, p, e1_at(G, p), e2_at(G, p));
}

template <typename T>
__global__ void stress21_adj_s1(GridDev<T> G, AdjDev<T> A, int flag)
{
    const Geo &g = G.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const Ext E{nx, ny, nz};
    const int64_t n = (int64_t)(nx + 1) * (ny + 1) * (nz + 1);
    const int sz = g.px * g.py;
    const T *const *c = G.c;
    T *const *W = A.w;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(t % (nx + 1)), y = (int)((t / (nx + 1)) % (ny + 1)), z = (int)(t / ((int64_t)(nx + 1) * (ny + 1)));
        const int p = g.idx(x, y, z);
        bool a_[2], b_[2];
        T w[2][2];
        if (E.n(x, y, z)) {
            const bool surf = flag && z == 0;
            const T a[3] = {A.l[SXX][p], A.l[SYY][p], surf ? T(0) : A.l[SZZ][p]};
            if (a[0] != T(0) || a[1] != T(0) || a[2] != T(0)) {
                const T e[3] = {e1_at(G, p), e2_at(G, p), e3u_at(G, E, surf, x, y, z, p)};
                const T ab[3] = {abar4_g(G, E, x, y, z), abar5_g(G, E, x, y, z), abar6_g(G, E, x, y, z)};
                const int rowc[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
                T le[3] = {T(0), T(0), T(0)}, lab[3] = {T(0), T(0), T(0)};
                for (int i = 0; i < 3; i++) {
                    for (int j = 0; j < 3; j++) {
                        const int s = rowc[i][j];
                        A.gc[s][p] = add_(A.gc[s][p], mul_(a[i], e[j]));
                        le[j] = fma_(a[i], c[s][p], le[j]);
                    }
                    for (int j = 0; j < 3; j++) {
                        const int s = 6 + 3 * i + j;
                        A.gc[s][p] = add_(A.gc[s][p], mul_(a[i], ab[j]));
                        lab[j] = fma_(a[i], c[s][p], lab[j]);
                    }
                }
                W[W_E1][p] = add_(W[W_E1][p], le[0]);
                W[W_E2][p] = add_(W[W_E2][p], le[1]);
                W[W_E3][p] = add_(W[W_E3][p], le[2]);
                // Abar4: L4 (x, y-1+i, z-1+j)
                for (int i = 0; i < 2; i++) { a_[i] = (y - 1 + i) >= 0 && (y - 1 + i) <= ny - 1; b_[i] = (z - 1 + i) >= 0 && (z - 1 + i) <= nz - 1; }
                weights4(a_, b_, w);
                for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++)
                    if (w[i][j] != T(0)) atom(W[W_E4] + g.idx(x, y - 1 + i, z - 1 + j), mul_(w[i][j], lab[0]));
                // Abar5: L5 (x+i, y, z-1+j)
                for (int i = 0; i < 2; i++) { a_[i] = (x + i) <= nx; b_[i] = (z - 1 + i) >= 0 && (z - 1 + i) <= nz - 1; }
                weights4(a_, b_, w);
                for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++)
                    if (w[i][j] != T(0)) atom(W[W_E5] + g.idx(x + i, y, z - 1 + j), mul_(w[i][j], lab[1]));
                // Abar6: L6 (x+i, y-1+j, z)
                for (int i = 0; i < 2; i++) { a_[i] = (x + i) <= nx; b_[i] = (y - 1 + i) >= 0 && (y - 1 + i) <= ny - 1; }
                weights4(a_, b_, w);
                for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++)
                    if (w[i][j] != T(0)) atom(W[W_E6] + g.idx(x + i, y - 1 + j, z), mul_(w[i][j], lab[2]));
            }
        }
        if (E.l6(x, y, z)) {
            const T a = A.l[SXY][p];
            if (a != T(0)) {
                A.gc[20][p] = add_(A.gc[20][p], mul_(a, e6_at(G, p)));
                atom(W[W_E6] + p, mul_(c[20][p], a));
                // Q46 over L4 (x-1+i, y, z-1+j)
                for (int i = 0; i < 2; i++) { a_[i] = (x - 1 + i) >= 0 && (x - 1 + i) <= nx - 1; b_[i] = (z - 1 + i) >= 0 && (z - 1 + i) <= nz - 1; }
                weights4(a_, b_, w);
                for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++)
                    if (w[i][j] != T(0)) atom(W[W_Q46] + g.idx(x - 1 + i, y, z - 1 + j), mul_(w[i][j], a));
                // Q56 over L5 (x, y+i, z-1+j)
                for (int i = 0; i < 2; i++) { a_[i] = (y + i) <= ny; b_[i] = (z - 1 + i) >= 0 && (z - 1 + i) <= nz - 1; }
                weights4(a_, b_, w);
                for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++)
                    if (w[i][j] != T(0)) atom(W[W_Q56] + g.idx(x, y + i, z - 1 + j), mul_(w[i][j], a));
                // P6 over N (x-1+i, y+j, z)
                for (int i = 0; i < 2; i++) { a_[i] = (x - 1 + i) >= 0 && (x - 1 + i) <= nx - 1; b_[i] = (y + i) <= ny; }
                weights4(a_, b_, w);
                for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++)
                    if (w[i][j] != T(0)) atom(W[W_P6] + g.idx(x - 1 + i, y + j, z), mul_(w[i][j], a));
            }
        }
        if (E.l4(x, y, z)) {
            T a = A.l[SYZ][p];
            if (flag && z == 0) {   // surface mirror syz(-1) = -syz(0)
                a = sub_(a, A.l[SYZ][p - sz]);
                A.l[SYZ][p - sz] = T(0);
                A.l[SYZ][p] = a;
            }
            if (a != T(0)) {
                // e5 over L5 (x+i, y+j, z); e6 over L6 (x+i, y, z+j); P4 over N (x, y+i, z+j)
                T v[2][2];
                bool oa[2], ob[2];
                for (int i = 0; i < 2; i++) { oa[i] = (x + i) <= nx; ob[i] = (y + i) <= ny; }
                for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++)
                    v[i][j] = (oa[i] && ob[j]) ? e5_at(G, g.idx(x + i, y + j, z)) : T(0);
                const T t5 = avg4<T>(v, oa, ob);
                weights4(oa, ob, w);
                const T c45 = c[16][p], c46 = c[17][p];
                for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++)
                    if (w[i][j] != T(0)) atom(W[W_E5] + g.idx(x + i, y + j, z), mul_(w[i][j], mul_(c45, a)));
                for (int i = 0; i < 2; i++) { oa[i] = (x + i) <= nx; ob[i] = (z + i) <= nz; }
                for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++)
                    v[i][j] = (oa[i] && ob[j]) ? e6_at(G, g.idx(x + i, y, z + j)) : T(0);
                const T t6 = avg4<T>(v, oa, ob);
                weights4(oa, ob, w);
                for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++)
                    if (w[i][j] != T(0)) atom(W[W_E6] + g.idx(x + i, y, z + j), mul_(w[i][j], mul_(c46, a)));
                for (int i = 0; i < 2; i++) { oa[i] = (y + i) <= ny; ob[i] = (z + i) <= nz; }
                weights4(oa, ob, w);
                for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++)
                    if (w[i][j] != T(0)) atom(W[W_P4] + g.idx(x, y + i, z + j), mul_(w[i][j], a));
                A.gc[15][p] = add_(A.gc[15][p], mul_(a, e4_at(G, p)));
                A.gc[16][p] = add_(A.gc[16][p], mul_(a, t5));
                A.gc[17][p] = add_(A.gc[17][p], mul_(a, t6));
                atom(W[W_E4] + p, mul_(c[15][p], a));
            }
        }
        if (E.l5(x, y, z)) {
            T a = A.l[SXZ][p];
            if (flag && z == 0 && x >= 1 && x <= nx - 1 && y >= 1 && y <= ny - 1) {   // surface mirror of sxz
                a = sub_(a, A.l[SXZ][p - sz]);
                A.l[SXZ][p - sz] = T(0);
                A.l[SXZ][p] = a;
            }
            if (a != T(0)) {
                // e6 over L6 (x, y-1+i, z+j); Q45 over L4 (x-1+i, y-1+j, z); P5 over N (x-1+i, y, z+j)
                T v[2][2];
                bool oa[2], ob[2];
                for (int i = 0; i < 2; i++) { oa[i] = (y - 1 + i) >= 0 && (y - 1 + i) <= ny - 1; ob[i] = (z + i) <= nz; }
                for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++)
                    v[i][j] = (oa[i] && ob[j]) ? e6_at(G, g.idx(x, y - 1 + i, z + j)) : T(0);
                const T t6 = avg4<T>(v, oa, ob);
                weights4(oa, ob, w);
                const T c56 = c[19][p];
                for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++)
                    if (w[i][j] != T(0)) atom(W[W_E6] + g.idx(x, y - 1 + i, z + j), mul_(w[i][j], mul_(c56, a)));
                for (int i = 0; i < 2; i++) { oa[i] = (x - 1 + i) >= 0 && (x - 1 + i) <= nx - 1; ob[i] = (y - 1 + i) >= 0 && (y - 1 + i) <= ny - 1; }
                weights4(oa, ob, w);
                for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++)
                    if (w[i][j] != T(0)) atom(W[W_Q45] + g.idx(x - 1 + i, y - 1 + j, z), mul_(w[i][j], a));
                for (int i = 0; i < 2; i++) { oa[i] = (x - 1 + i) >= 0 && (x - 1 + i) <= nx - 1; ob[i] = (z + i) <= nz; }
                weights4(oa, ob, w);
                for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++)
                    if (w[i][j] != T(0)) atom(W[W_P5] + g.idx(x - 1 + i, y, z + j), mul_(w[i][j], a));
                A.gc[18][p] = add_(A.gc[18][p], mul_(a, e5_at(G, p)));
                A.gc[19][p] = add_(A.gc[19][p], mul_(a, t6));
                atom(W[W_E5] + p, mul_(c[18][p], a));
            }
        }
    }
}

template <typename T>
__global__ void stress21_adj_s2(GridDev<T> G, AdjDev<T> A, int flag)
{
    const Geo &g = G.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const Ext E{nx, ny, nz};
    const int64_t n = (int64_t)(nx + 1) * (ny + 1) * (nz + 1);
    const T *const *c = G.c;
    T *const *W = A.w;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(t % (nx + 1)), y = (int)((t / (nx + 1)) % (ny + 1)), z = (int)(t / ((int64_t)(nx + 1) * (ny + 1)));
        const int p = g.idx(x, y, z);
        if (E.l4(x, y, z)) {
            const T z45 = W[W_Q45][p], z46 = W[W_Q46][p];
            if (z45 != T(0) || z46 != T(0)) {
                const T e4 = e4_at(G, p);
                A.gc[16][p] = add_(A.gc[16][p], mul_(z45, e4));
                A.gc[17][p] = add_(A.gc[17][p], mul_(z46, e4));
                W[W_E4][p] = add_(W[W_E4][p], add_(mul_(c[16][p], z45), mul_(c[17][p], z46)));
                W[W_Q45][p] = T(0);
                W[W_Q46][p] = T(0);
            }
        }
        if (E.l5(x, y, z)) {
            const T z56 = W[W_Q56][p];
            if (z56 != T(0)) {
                A.gc[19][p] = add_(A.gc[19][p], mul_(z56, e5_at(G, p)));
                W[W_E5][p] = add_(W[W_E5][p], mul_(c[19][p], z56));
                W[W_Q56][p] = T(0);
            }
        }
        if (E.n(x, y, z)) {
            const T zp[3] = {W[W_P4][p], W[W_P5][p], W[W_P6][p]};
            if (zp[0] != T(0) || zp[1] != T(0) || zp[2] != T(0)) {
                const bool surf = flag && z == 0;
                const T e[3] = {e1_at(G, p), e2_at(G, p), e3u_at(G, E, surf, x, y, z, p)};
                T le[3] = {T(0), T(0), T(0)};
                for (int k = 0; k < 3; k++)           // P(4+k) = C(1,4+k) e1 + C(2,4+k) e2 + C(3,4+k) e3
                    for (int j = 0; j < 3; j++) {
                        const int s = 6 + 3 * j + k;
                        A.gc[s][p] = add_(A.gc[s][p], mul_(zp[k], e[j]));
                        le[j] = fma_(c[s][p], zp[k], le[j]);
                    }
                W[W_E1][p] = add_(W[W_E1][p], le[0]);
                W[W_E2][p] = add_(W[W_E2][p], le[1]);
                W[W_E3][p] = add_(W[W_E3][p], le[2]);
                W[W_P4][p] = T(0); W[W_P5][p] = T(0); W[W_P6][p] = T(0);
            }
        }
    }
}

// free surface: e3 = -(C13 e1 + C23 e2 + C34 A4 + C35 A5 + C36 A6) / C33 at z = 0
template <typename T>
__global__ void stress21_adj_s3(GridDev<T> G, AdjDev<T> A)
{
    const Geo &g = G.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const Ext E{nx, ny, nz};
    const int n = nx * (ny + 1);
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int x = t % nx, y = t / nx, z = 0;
    const int p = g.idx(x, y, z);
    const T le3 = A.w[W_E3][p];
    if (le3 == T(0)) return;
    A.w[W_E3][p] = T(0);
    const T *const *c = G.c;
    const T c33 = c[5][p];
    const T e1 = e1_at(G, p), e2 = e2_at(G, p), e3 = e3u_at(G, E, true, x, y, z, p);
    const T ab[3] = {abar4_g(G, E, x, y, z), abar5_g(G, E, x, y, z), abar6_g(G, E, x, y, z)};
    const T u = -div_(le3, c33);   // d e3 / d(numerator term) = -1 / C33
    A.w[W_E1][p] = fma_(u, c[2][p], A.w[W_E1][p]);
    A.w[W_E2][p] = fma_(u, c[4][p], A.w[W_E2][p]);
    A.gc[2][p] = fma_(u, e1, A.gc[2][p]);
    A.gc[4][p] = fma_(u, e2, A.gc[4][p]);
    A.gc[5][p] = fma_(u, e3, A.gc[5][p]);   // d e3 / d C33 = -e3 / C33
    for (int k = 0; k < 3; k++) A.gc[12 + k][p] = fma_(u, ab[k], A.gc[12 + k][p]);
    bool a_[2], b_[2];
    T w[2][2];
    const T l4 = mul_(u, c[12][p]), l5 = mul_(u, c[13][p]), l6 = mul_(u, c[14][p]);
    for (int i = 0; i < 2; i++) { a_[i] = (y - 1 + i) >= 0 && (y - 1 + i) <= ny - 1; b_[i] = (z - 1 + i) >= 0 && (z - 1 + i) <= nz - 1; }
    weights4(a_, b_, w);
    for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++)
        if (w[i][j] != T(0)) atom(A.w[W_E4] + g.idx(x, y - 1 + i, z - 1 + j), mul_(w[i][j], l4));
    for (int i = 0; i < 2; i++) { a_[i] = (x + i) <= nx; b_[i] = (z - 1 + i) >= 0 && (z - 1 + i) <= nz - 1; }
    weights4(a_, b_, w);
    for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++)
        if (w[i][j] != T(0)) atom(A.w[W_E5] + g.idx(x + i, y, z - 1 + j), mul_(w[i][j], l5));
    for (int i = 0; i < 2; i++) { a_[i] = (x + i) <= nx; b_[i] = (y - 1 + i) >= 0 && (y - 1 + i) <= ny - 1; }
    weights4(a_, b_, w);
    for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++)
        if (w[i][j] != T(0)) atom(A.w[W_E6] + g.idx(x + i, y - 1 + j, z), mul_(w[i][j], l6));
}

// transpose of the strain differences: W[e] -> lambda_v; the buffers are cleared
template <typename T>
__global__ void stress21_adj_s4(GridDev<T> G, AdjDev<T> A)
{
    const Geo &g = G.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const Ext E{nx, ny, nz};
    const int64_t n = (int64_t)(nx + 1) * (ny + 1) * (nz + 1);
    const int sy = g.px, sz = g.px * g.py;
    const T k0 = G.k[0], k1 = G.k[1], k2 = G.k[2];
    T *lvx = A.l[VX], *lvy = A.l[VY], *lvz = A.l[VZ];
    T *const *W = A.w;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(t % (nx + 1)), y = (int)((t / (nx + 1)) % (ny + 1)), z = (int)(t / ((int64_t)(nx + 1) * (ny + 1)));
        const int p = g.idx(x, y, z);
        if (E.n(x, y, z)) {
            const T w1 = W[W_E1][p], w2_ = W[W_E2][p], w3 = W[W_E3][p];
            if (w1 != T(0)) { const T u = mul_(k0, w1); atom(lvx + p + 1, u); atom(lvx + p, -u); W[W_E1][p] = T(0); }
            if (w2_ != T(0)) { const T u = mul_(k1, w2_); atom(lvy + p, u); atom(lvy + p - sy, -u); W[W_E2][p] = T(0); }
            if (w3 != T(0)) { const T u = mul_(k2, w3); atom(lvz + p, u); atom(lvz + p - sz, -u); W[W_E3][p] = T(0); }
        }
        if (E.l4(x, y, z)) {
            const T w4 = W[W_E4][p];
            if (w4 != T(0)) {
                const T u2 = mul_(k2, w4), u1 = mul_(k1, w4);
                atom(lvy + p + sz, u2); atom(lvy + p, -u2); atom(lvz + p + sy, u1); atom(lvz + p, -u1);
                W[W_E4][p] = T(0);
            }
        }
        if (E.l5(x, y, z)) {
            const T w5 = W[W_E5][p];
            if (w5 != T(0)) {
                const T u2 = mul_(k2, w5), u0 = mul_(k0, w5);
                atom(lvx + p + sz, u2); atom(lvx + p, -u2); atom(lvz + p, u0); atom(lvz + p - 1, -u0);
                W[W_E5][p] = T(0);
            }
        }
        if (E.l6(x, y, z)) {
            const T w6 = W[W_E6][p];
            if (w6 != T(0)) {
                const T u1 = mul_(k1, w6), u0 = mul_(k0, w6);
                atom(lvx + p + sy, u1); atom(lvx + p, -u1); atom(lvy + p, u0); atom(lvy + p - 1, -u0);
                W[W_E6][p] = T(0);
            }
        }
    }
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
static unsigned blocks_for(int64_t n, int sms)
{
    int64_t b = (n + 255) / 256;
    const int64_t cap = (int64_t)sms * 16;
    return (unsigned)(b < 1 ? 1 : (b > cap ? cap : b));
}

template <typename T>
cudaError_t launch_vel_adj(const GridDev<T> &G, const AdjDev<T> &A, int top, int bottom, int top_bc, int mirror_fix,
                           int sms, cudaStream_t st)
{
    const Geo &g = G.g;
    const int top_rigid = (top && top_bc != 1) ? 1 : 0;
    const int64_t n0 = (int64_t)(top_rigid + bottom) * (g.ny + 1) * g.nx + 2LL * g.nz * (g.ny + 1)
                     + 2LL * (g.nz + 1) * (g.ny + 1);
    const int64_t n1 = 2LL * (g.nz + (mirror_fix ? 1 : 0)) * g.nx;
    // reverse order: mirrors (phase 1, then phase 0), then the update
    vel_mirror_adj_kernel<T><<<(unsigned)((n1 + 255) / 256), 256, 0, st>>>(g, A.l[VY], A.l[VZ], 1, top_rigid, bottom, mirror_fix);
    vel_mirror_adj_kernel<T><<<(unsigned)((n0 + 255) / 256), 256, 0, st>>>(g, A.l[VY], A.l[VZ], 0, top_rigid, bottom, mirror_fix);
    const int zt = top_rigid;
    vel_adj_kernel<T><<<blocks_for((int64_t)g.nx * g.ny * (g.nz + 1), sms), 256, 0, st>>>(G, A, zt, bottom);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_stress21_adj(const GridDev<T> &G, const AdjDev<T> &A, int top, int top_bc, int sms, cudaStream_t st)
{
    const Geo &g = G.g;
    const int flag = (top && top_bc) ? 1 : 0;
    const int64_t n = (int64_t)(g.nx + 1) * (g.ny + 1) * (g.nz + 1);
    const unsigned nb = blocks_for(n, sms);
    stress21_adj_s1<T><<<nb, 256, 0, st>>>(G, A, flag);
    stress21_adj_s2<T><<<nb, 256, 0, st>>>(G, A, flag);
    if (flag) stress21_adj_s3<T><<<(g.nx * (g.ny + 1) + 255) / 256, 256, 0, st>>>(G, A);
    stress21_adj_s4<T><<<nb, 256, 0, st>>>(G, A);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_rec_adj(const RecAdj<T> &R, cudaStream_t st)
{
    if (R.nrec <= 0) return cudaSuccess;
    rec_adj_kernel<T><<<(R.nrec + 255) / 256, 256, 0, st>>>(R);
    return cudaGetLastError();
}

#define INST(T)                                                                                              \
    template cudaError_t launch_vel_adj<T>(const GridDev<T> &, const AdjDev<T> &, int, int, int, int, int,      \
                                           cudaStream_t);                                                   \
    template cudaError_t launch_stress21_adj<T>(const GridDev<T> &, const AdjDev<T> &, int, int, int,          \
                                                cudaStream_t);                                              \
    template cudaError_t launch_rec_adj<T>(const RecAdj<T> &, cudaStream_t);
INST(float)
INST(double)
#undef INST

} // namespace ecsg

namespace ecsg {

// Receiver values at full precision (the misfit's samples; sampled as main.cpp:182-184)
template <typename T>
__global__ void rec_sample_kernel(SrcRec S, T *out)
{
    for (int i = threadIdx.x; i < S.nrec; i += blockDim.x) out[i] = ((const T *)S.rec_base[S.rec_grid[i]])[S.rec_off[i]];
}

// residual = sample - observed (in place), loss += 1/2 sum residual^2 (FP64)
template <typename T>
__global__ void residual_kernel(T *rec, const float *obs, int64_t n, double *loss)
{
    __shared__ double red[8];
    double s = 0.0;
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (int64_t)gridDim.x * blockDim.x) {
        const T r = sub_(rec[i], (T)obs[i]);
        rec[i] = r;
        s += 0.5 * (double)r * (double)r;
    }
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = s;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < (int)(blockDim.x >> 5); w++) t += red[w];
        atomicAdd(loss, t);
    }
}

template <typename T>
cudaError_t launch_rec_sample(const SrcRec &S, T *out, cudaStream_t st)
{
    if (S.nrec <= 0) return cudaSuccess;
    rec_sample_kernel<T><<<1, 256, 0, st>>>(S, out);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_residual(T *rec, const float *obs, int64_t n, double *loss, cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    int64_t b = (n + 255) / 256;
    if (b > 1024) b = 1024;
    residual_kernel<T><<<(unsigned)b, 256, 0, st>>>(rec, obs, n, loss);
    return cudaGetLastError();
}

template cudaError_t launch_rec_sample<float>(const SrcRec &, float *, cudaStream_t);
template cudaError_t launch_rec_sample<double>(const SrcRec &, double *, cudaStream_t);
template cudaError_t launch_residual<float>(float *, const float *, int64_t, double *, cudaStream_t);
template cudaError_t launch_residual<double>(double *, const float *, int64_t, double *, cudaStream_t);

} // namespace ecsg
