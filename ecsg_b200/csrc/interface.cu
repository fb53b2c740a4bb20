// interface.cu -- energy-conserving ghost solves at a refinement interface.
//
// Fine grid F (top) and coarse grid C (below) meet at fine z-node nz1 = coarse
// z-node 0, with refinement ratio r in x and y.  Arithmetic is double precision
// whatever the field type (the ghost values are the energy-conservation
// condition).  Operators, for a general ratio r (r = 2 is the reference):
//   P  prolongation coarse -> fine per dim: node dims interpolate linearly from
//      the interior coarse nodes, cell dims copy the coarse cell value;
//   the coarse interface value after an update equals the restriction
//   P^T / r^2 of the fine interface values, and the fine ghost is
//   -(last fine interior value) + P(coarse ghost + coarse first interior value).
// This gives (update_ghost_*.cpp for r = 2):
//   vz : one tridiagonal system along y per coarse x-cell (update_ghost_vz.cpp:124-221)
//        -> assembly (coalesced along x), one CTA per x-cell for parallel
//           cyclic reduction in shared memory, fine-ghost scatter
//   syz: pointwise closed form (update_ghost_syz.cpp:151-240) -> one thread per cell
//   sxz: 9-point system on the interior coarse nodes, warm-started Jacobi with
//        the reference stopping rule ||X_k - X_{k-1}||_2 <= min(1e-12, 1e-5 avg|B|)
//        (update_ghost_sxz.cpp:86-236, 314-350) -> one cooperative persistent
//        kernel: B assembly, Jacobi sweeps with deterministic grid-wide
//        reductions, fine-ghost scatter.  Grid barriers spin with an iteration
//        limit and set a status bit instead of waiting forever; the sweep count
//        is capped and a capped solve sets ST_JACOBI_CAP.
#include "ecsg_device.cuh"
#include "gen21_device.cuh"
#include <cstdio>

namespace ecsg {

__device__ __forceinline__ double pw_node(int i, int j, int r, int n2)
{
    if (j <= 0 || j >= n2) return 0.0;
    int d = i - r * j;
    if (d <= -r || d >= r) return 0.0;
    return 1.0 - (double)abs(d) / (double)r;
}
__device__ __forceinline__ double pw_node_all(int i, int j, int r)
{
    int d = i - r * j;
    if (d <= -r || d >= r) return 0.0;
    return 1.0 - (double)abs(d) / (double)r;
}

template <typename T>
__device__ __forceinline__ void normal_c(const GridDev<T> &G, int medium, int p, double &c13, double &c23, double &c33)
{
    if (medium == MED_ISO5) {
        c33 = (double)G.c[0][p];
        c13 = c23 = (double)G.c[1][p];
    } else if (medium == MED_GEN21) {
        c13 = (double)G.c[2][p];
        c23 = (double)G.c[4][p];
        c33 = (double)G.c[5][p];
    } else {
        c33 = (double)G.c[2][p];
        c23 = (double)G.c[3][p];
        c13 = (double)G.c[4][p];
    }
}

// ---------------------------------------------------------------------------
// vz, in three kernels so that every global access is coalesced along x:
//   1. assemble: thread per unknown (j0 fastest, j1 in [1, ny2-1]) writes the
//      tridiagonal row (lower, diagonal, upper, rhs) to coef[4][j1-1][j0];
//   2. solve: CTA per coarse x-cell j0, parallel cyclic reduction of its
//      system in shared memory, coarse ghost vz2(j0, j1, -1) written back
//      (rounded to the field type, as the fine scatter reads it);
//   3. scatter: thread per fine ghost vz1(i0, i1, nz1), i0 fastest.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void ghost_vz_assemble_kernel(GridDev<T> F, GridDev<T> C, int medium, int r, double *coef)
{
    const int j0 = blockIdx.x * blockDim.x + threadIdx.x;
    const int j1 = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int nx2 = C.g.nx, ny2 = C.g.ny, nz1 = F.g.nz;
    const int m = ny2 - 1;
    if (j0 >= nx2 || j1 > m) return;
    const T *vx1 = F.f[VX], *vy1 = F.f[VY], *szz1 = F.f[SZZ], *vz1 = F.f[VZ];
    const T *vx2 = C.f[VX], *vy2 = C.f[VY], *szz2 = C.f[SZZ], *vz2 = C.f[VZ];
    const double k1x = F.kd[0], k1y = F.kd[1], k1z = F.kd[2];
    const double k2x = C.kd[0], k2y = C.kd[1], k2z = C.kd[2];
    const double rr = (double)r, r3 = rr * rr * rr;
    const int pc = C.g.idx(j0, j1, 0);
    double c13, c23, c33;
    normal_c(C, medium, pc, c13, c23, c33);
    double pred = (double)szz2[pc] + c13 * k2x * ((double)vx2[C.g.idx(j0 + 1, j1, 0)] - (double)vx2[pc])
                + c23 * k2y * ((double)vy2[pc] - (double)vy2[C.g.idx(j0, j1 - 1, 0)])
                + c33 * k2z * (double)vz2[pc];
    if (medium == MED_GEN21) pred += gen21_szz_extra(C, j0, j1, 0);
    double dg = r3 * k2z * c33, lo = 0.0, up = 0.0, fsum = 0.0;
    for (int i0 = r * j0; i0 < r * j0 + r; i0++) {
        for (int i1 = r * (j1 - 1) + 1; i1 <= r * (j1 + 1) - 1; i1++) {
            const double w = pw_node(i1, j1, r, ny2);
            const double wl = pw_node(i1, j1 - 1, r, ny2), wu = pw_node(i1, j1 + 1, r, ny2);
            const int pf = F.g.idx(i0, i1, nz1);
            double f13, f23, f33;
            normal_c(F, medium, pf, f13, f23, f33);
            const double cz = f33 * k1z;
            const int jl = i1 / r, ju = jl + 1;
            double pv0 = pw_node_all(i1, jl, r) * (double)vz2[C.g.idx(j0, jl, 0)];
            if (ju <= ny2) pv0 += pw_node_all(i1, ju, r) * (double)vz2[C.g.idx(j0, ju, 0)];
            double pf_ = (double)szz1[pf] + f13 * k1x * ((double)vx1[pf + 1] - (double)vx1[pf])
                       + f23 * k1y * ((double)vy1[pf] - (double)vy1[pf - F.g.px])
                       + cz * (pv0 - 2.0 * (double)vz1[pf - F.g.px * F.g.py]);
            if (medium == MED_GEN21) pf_ += gen21_szz_extra(F, i0, i1, nz1);
            dg += rr * w * w * cz;
            lo += rr * w * wl * cz;
            up += rr * w * wu * cz;
            fsum += rr * w * pf_;
        }
    }
    const size_t plane = (size_t)m * nx2, q = (size_t)(j1 - 1) * nx2 + j0;
    coef[q] = (j1 == 1) ? 0.0 : lo;          // coupling to a boundary node: not an unknown
    coef[plane + q] = dg;
    coef[2 * plane + q] = (j1 == m) ? 0.0 : up;
    coef[3 * plane + q] = r3 * pred - fsum;
}

template <typename T>
__global__ void ghost_vz_solve_kernel(GridDev<T> C, const double *coef)
{
    extern __shared__ double sm[];
    const int P = blockDim.x;
    const int t = threadIdx.x;
    const int j0 = blockIdx.x;
    const int nx2 = C.g.nx, ny2 = C.g.ny;
    const int m = ny2 - 1;
    double *A = sm, *B = sm + P, *Cc = sm + 2 * P, *D = sm + 3 * P;
    T *vz2 = C.f[VZ];
    const size_t plane = (size_t)m * nx2, q = (size_t)t * nx2 + j0;
    A[t] = t < m ? coef[q] : 0.0;
    B[t] = t < m ? coef[plane + q] : 1.0;
    Cc[t] = t < m ? coef[2 * plane + q] : 0.0;
    D[t] = t < m ? coef[3 * plane + q] : 0.0;
    __syncthreads();
    // parallel cyclic reduction: rows outside [0,m) are identity rows
    for (int s = 1; s < P; s <<= 1) {
        double a = A[t], bb = B[t], c = Cc[t], d = D[t];
        double na = 0.0, nc = 0.0, nb = bb, nd = d;
        if (t - s >= 0) {
            const double k = a / B[t - s];
            na = -A[t - s] * k;
            nb -= Cc[t - s] * k;
            nd -= D[t - s] * k;
        }
        if (t + s < P) {
            const double k = c / B[t + s];
            nc = -Cc[t + s] * k;
            nb -= A[t + s] * k;
            nd -= D[t + s] * k;
        }
        __syncthreads();
        A[t] = na; B[t] = nb; Cc[t] = nc; D[t] = nd;
        __syncthreads();
    }
    if (t < m) vz2[C.g.idx(j0, t + 1, -1)] = (T)(D[t] / B[t]);
}

template <typename T>
__global__ void ghost_vz_scatter_kernel(GridDev<T> F, GridDev<T> C, int r)
{
    const int i0 = blockIdx.x * blockDim.x + threadIdx.x;
    const int i1 = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int ny2 = C.g.ny, nz1 = F.g.nz;
    const int nx1 = r * C.g.nx, ny1 = r * ny2;
    if (i0 >= nx1 || i1 >= ny1) return;
    const T *vz2 = C.f[VZ];
    T *vz1 = F.f[VZ];
    const int j0 = i0 / r, jl = i1 / r, ju = jl + 1;
    const int csz = C.g.px * C.g.py;
    const int pl = C.g.idx(j0, jl, 0);
    double s = pw_node_all(i1, jl, r) * ((double)vz2[pl] + (double)vz2[pl - csz]);
    if (ju <= ny2) {
        const int pu = C.g.idx(j0, ju, 0);
        s += pw_node_all(i1, ju, r) * ((double)vz2[pu] + (double)vz2[pu - csz]);
    }
    const int pf = F.g.idx(i0, i1, nz1);
    vz1[pf] = (T)(-(double)vz1[pf - F.g.px * F.g.py] + s);
}

// ---------------------------------------------------------------------------
// syz: thread per coarse cell (j0, j1).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void ghost_syz_kernel(GridDev<T> F, GridDev<T> C, int r)
{
    const int j0 = blockIdx.x * blockDim.x + threadIdx.x;
    const int j1 = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx2 = C.g.nx, ny2 = C.g.ny, nz1 = F.g.nz;
    if (j0 >= nx2 || j1 >= ny2) return;
    const T *vy1 = F.f[VY], *syy1 = F.f[SYY], *sxy1 = F.f[SXY], *b1 = F.b;
    T *syz1 = F.f[SYZ];
    const T *vy2 = C.f[VY], *syy2 = C.f[SYY], *sxy2 = C.f[SXY], *b2 = C.b;
    T *syz2 = C.f[SYZ];
    const double k1x = F.kd[0], k1y = F.kd[1], k1z = F.kd[2];
    const double k2x = C.kd[0], k2y = C.kd[1], k2z = C.kd[2];
    const double r2 = (double)r * (double)r;
    const int sy1 = F.g.px, sz1 = F.g.px * F.g.py, sy2 = C.g.px;

    const int pc = C.g.idx(j0, j1, 0);
    const double c0 = 0.25 * ((double)b2[pc] + (double)b2[pc + 1] + (double)b2[pc + sy2] + (double)b2[pc + sy2 + 1]);
    const double s0 = (double)syz2[pc];
    double num = r2 * ((double)vy2[pc] + c0 * (k2x * ((double)sxy2[pc + 1] - (double)sxy2[pc])
                                              + k2y * ((double)syy2[pc + sy2] - (double)syy2[pc]) + k2z * s0));
    double den = r2 * c0 * k2z;
    for (int i1 = r * j1; i1 < r * j1 + r; i1++)
        for (int i0 = r * j0; i0 < r * j0 + r; i0++) {
            const int pf = F.g.idx(i0, i1, nz1);
            const double c = 0.25 * ((double)b1[pf] + (double)b1[pf + 1] + (double)b1[pf + sy1] + (double)b1[pf + sy1 + 1]);
            num -= (double)vy1[pf] + c * (k1x * ((double)sxy1[pf + 1] - (double)sxy1[pf])
                                          + k1y * ((double)syy1[pf + sy1] - (double)syy1[pf])
                                          + k1z * (s0 - 2.0 * (double)syz1[pf - sz1]));
            den += c * k1z;
        }
    const T xt = (T)(num / den);
    syz2[pc - C.g.px * C.g.py] = xt;
    const double tsum = (double)xt + s0;
    for (int i1 = r * j1; i1 < r * j1 + r; i1++)
        for (int i0 = r * j0; i0 < r * j0 + r; i0++) {
            const int pf = F.g.idx(i0, i1, nz1);
            syz1[pf] = (T)(-(double)syz1[pf - sz1] + tsum);
        }
}

// ---------------------------------------------------------------------------
// sxz
// ---------------------------------------------------------------------------
// A (time-invariant): 9 diagonals, k = 3*(dx+1)+(dy+1), layout A[k][j1-1][j0-1].
template <typename T>
__global__ void sxz_matrix_kernel(GridDev<T> F, GridDev<T> C, int r, double *A)
{
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    const int nx2 = C.g.nx, ny2 = C.g.ny, nz1 = F.g.nz;
    const int n0 = nx2 - 1, n1 = ny2 - 1;
    if (q >= n0 * n1) return;
    const int j0 = q % n0 + 1, j1 = q / n0 + 1;
    const double rr = (double)r, r2 = rr * rr, r4 = r2 * r2;
    double a9[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0};
    for (int i1 = r * j1 - r + 1; i1 <= r * j1 + r - 1; i1++) {
        const double wy = pw_node(i1, j1, r, ny2);
        for (int i0 = r * j0 - r + 1; i0 <= r * j0 + r - 1; i0++) {
            const double w = pw_node(i0, j0, r, nx2) * wy;
            const double bz = (double)F.b[F.g.idx(i0, i1, nz1)] * F.kd[2];
            for (int dx = -1; dx <= 1; dx++)
                for (int dy = -1; dy <= 1; dy++) {
                    const double wn = pw_node(i0, j0 + dx, r, nx2) * pw_node(i1, j1 + dy, r, ny2);
                    a9[3 * (dx + 1) + (dy + 1)] += r2 * w * wn * bz;
                }
        }
    }
    a9[4] += r4 * (double)C.b[C.g.idx(j0, j1, 0)] * C.kd[2];
    for (int k = 0; k < 9; k++) A[(int64_t)k * n0 * n1 + q] = a9[k];
}

template <typename T>
__device__ double sxz_rhs(const GridDev<T> &F, const GridDev<T> &C, int r, int j0, int j1)
{
    const int nx2 = C.g.nx, ny2 = C.g.ny, nz1 = F.g.nz;
    const T *vx1 = F.f[VX], *sxx1 = F.f[SXX], *sxz1 = F.f[SXZ], *sxy1 = F.f[SXY], *b1 = F.b;
    const T *vx2 = C.f[VX], *sxx2 = C.f[SXX], *sxz2 = C.f[SXZ], *sxy2 = C.f[SXY], *b2 = C.b;
    const double k1x = F.kd[0], k1y = F.kd[1], k1z = F.kd[2];
    const double k2x = C.kd[0], k2y = C.kd[1], k2z = C.kd[2];
    const double rr = (double)r, r2 = rr * rr, r4 = r2 * r2;
    const int sy1 = F.g.px, sz1 = F.g.px * F.g.py, sy2 = C.g.px;
    double fsum = 0.0;
    for (int i1 = r * j1 - r + 1; i1 <= r * j1 + r - 1; i1++) {
        const double wy = pw_node(i1, j1, r, ny2);
        const int jy = i1 / r;
        for (int i0 = r * j0 - r + 1; i0 <= r * j0 + r - 1; i0++) {
            const double w = pw_node(i0, j0, r, nx2) * wy;
            const int jx = i0 / r;
            double ps0 = 0.0;
            for (int ey = 0; ey < 2; ey++)
                for (int ex = 0; ex < 2; ex++) {
                    const int cx = jx + ex, cy = jy + ey;
                    if (cx > nx2 || cy > ny2) continue;
                    const double ww = pw_node(i0, cx, r, nx2) * pw_node(i1, cy, r, ny2);
                    if (ww != 0.0) ps0 += ww * (double)sxz2[C.g.idx(cx, cy, 0)];
                }
            const int pf = F.g.idx(i0, i1, nz1);
            const double pf_ = (double)vx1[pf]
                             + (double)b1[pf] * (k1x * ((double)sxx1[pf] - (double)sxx1[pf - 1])
                                                 + k1y * ((double)sxy1[pf] - (double)sxy1[pf - sy1])
                                                 + k1z * (ps0 - 2.0 * (double)sxz1[pf - sz1]));
            fsum += w * pf_;
        }
    }
    const int pc = C.g.idx(j0, j1, 0);
    const double pc_ = (double)vx2[pc] + (double)b2[pc] * (k2x * ((double)sxx2[pc] - (double)sxx2[pc - 1])
                                                          + k2y * ((double)sxy2[pc] - (double)sxy2[pc - sy2])
                                                          + k2z * (double)sxz2[pc]);
    return r4 * pc_ - r2 * fsum;
}


constexpr long long kSpinLimit = 1LL << 26;   // ~seconds with the nanosleep back-off

__device__ __forceinline__ double block_sum(double v, double *red)
{
    for (int o = 16; o > 0; o >>= 1) v += __shfl_down_sync(0xffffffffu, v, o);
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
    if (l == 0) red[w] = v;
    __syncthreads();
    double s = 0.0;
    if (threadIdx.x == 0)
        for (int i = 0; i < (int)(blockDim.x >> 5); i++) s += red[i];
    __syncthreads();
    return s;   // valid in thread 0
}

// Grid-wide deterministic sum.  Each CTA publishes its partial; the last CTA
// to arrive sums all partials with all its threads (fixed strided split, then
// a fixed tree), publishes the total and releases the others by advancing the
// generation word.  Every CTA returns the same value.  Waiting is bounded: on
// timeout the status bit is set, ok becomes false and the caller stops.
__device__ double grid_sum(double v, const SxzWork &W, double *red, bool &ok)
{
    __threadfence();
    const double bs = block_sum(v, red);   // valid in thread 0
    __shared__ double s_total;
    __shared__ int s_last, s_ok;
    __shared__ unsigned s_gen;
    if (threadIdx.x == 0) {
        s_gen = *(volatile unsigned *)(W.bar + 1);   // generation of this round, read before arriving
        W.partial[blockIdx.x] = bs;
        __threadfence();
        const unsigned prev = atomicAdd(W.bar, 1u);
        s_last = (prev == gridDim.x - 1);
        s_ok = 1;
    }
    __syncthreads();
    if (s_last) {
        __threadfence();
        double t = 0.0;
        for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x) t += __ldcg(W.partial + i);
        const double tot = block_sum(t, red);
        if (threadIdx.x == 0) {
            __stcg(W.total, tot);
            W.bar[0] = 0;
            __threadfence();
            atomicAdd(W.bar + 1, 1u);
            s_total = tot;
        }
    } else if (threadIdx.x == 0) {
        long long spin = 0;
        while (*(volatile unsigned *)(W.bar + 1) == s_gen) {
            if (++spin > kSpinLimit) { atomicOr(W.status, ST_BARRIER_TIMEOUT); s_ok = 0; break; }
            __nanosleep(32);
        }
        __threadfence();
        s_total = __ldcg(W.total);
    }
    __syncthreads();
    ok = s_ok != 0;
    return s_total;
}

template <typename T>
__global__ void __launch_bounds__(256) sxz_solve_kernel(GridDev<T> F, GridDev<T> C, int r, SxzWork W)
{
    __shared__ double red[32];
    const int nx2 = C.g.nx, ny2 = C.g.ny, nz1 = F.g.nz;
    const int n0 = nx2 - 1, n1 = ny2 - 1, ld = nx2 + 1;
    const int nn = n0 * n1;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int gstride = gridDim.x * blockDim.x;
    bool ok = true;

    // B and avg|B| (Array::AvgAbs, array.cpp:172-210)
    double sab = 0.0;
    for (int q = gtid; q < nn; q += gstride) {
        const double bq = sxz_rhs(F, C, r, q % n0 + 1, q / n0 + 1);
        W.B[q] = bq;
        sab += fabs(bq);
    }
    const double sumabs = grid_sum(sab, W, red, ok);
    double tol = 1e-5 * (sumabs / (double)nn);
    if (tol > 1e-12) tol = 1e-12;

    // Jacobi2D (update_ghost_sxz.cpp:314-350), ping-pong instead of copy
    double *Xc = W.X0, *Xn = W.X1;
    int it = 0;
    while (ok) {
        double s = 0.0;
        for (int q = gtid; q < nn; q += gstride) {
            const int i0 = q % n0 + 1, i1 = q / n0 + 1;
            const double *a = W.A + q;
            const double xn = (W.B[q]
                               - a[0 * nn] * __ldcg(Xc + (i1 - 1) * ld + (i0 - 1))
                               - a[1 * nn] * __ldcg(Xc + (i1) * ld + (i0 - 1))
                               - a[2 * nn] * __ldcg(Xc + (i1 + 1) * ld + (i0 - 1))
                               - a[3 * nn] * __ldcg(Xc + (i1 - 1) * ld + (i0))
                               - a[5 * nn] * __ldcg(Xc + (i1 + 1) * ld + (i0))
                               - a[6 * nn] * __ldcg(Xc + (i1 - 1) * ld + (i0 + 1))
                               - a[7 * nn] * __ldcg(Xc + (i1) * ld + (i0 + 1))
                               - a[8 * nn] * __ldcg(Xc + (i1 + 1) * ld + (i0 + 1))) / a[4 * nn];
            const double d = xn - __ldcg(Xc + i1 * ld + i0);
            __stcg(Xn + i1 * ld + i0, xn);
            s += d * d;
        }
        const double tot = grid_sum(s, W, red, ok);
        double *tmp = Xc; Xc = Xn; Xn = tmp;
        it++;
        if (!(sqrt(tot) > tol)) break;
        if (it >= W.max_iter) {
            if (gtid == 0) atomicOr(W.status, ST_JACOBI_CAP);
            break;
        }
    }
    if (gtid == 0) {
        *W.iters = it;
        *W.iters_total += it;
        *W.tol_out = tol;
    }
    // coarse ghost and fine ghosts (update_ghost_sxz.cpp:247-295)
    T *sxz1 = F.f[SXZ];
    T *sxz2 = C.f[SXZ];
    const int csz = C.g.px * C.g.py, fsz = F.g.px * F.g.py;
    for (int q = gtid; q < nn; q += gstride) {
        const int j0 = q % n0 + 1, j1 = q / n0 + 1;
        const double x = __ldcg(Xc + j1 * ld + j0);
        sxz2[C.g.idx(j0, j1, 0) - csz] = (T)x;
        if (Xc != W.X0) W.X0[j1 * ld + j0] = x;
    }
    const int nx1 = r * nx2, ny1 = r * ny2;
    const int nf = (nx1 - 1) * (ny1 - 1);
    for (int q = gtid; q < nf; q += gstride) {
        const int i0 = q % (nx1 - 1) + 1, i1 = q / (nx1 - 1) + 1;
        const int jx = i0 / r, jy = i1 / r;
        double acc = 0.0;
        for (int ey = 0; ey < 2; ey++)
            for (int ex = 0; ex < 2; ex++) {
                const int cx = jx + ex, cy = jy + ey;
                if (cx > nx2 || cy > ny2) continue;
                const double ww = pw_node(i0, cx, r, nx2) * pw_node(i1, cy, r, ny2);
                if (ww != 0.0) {
                    const double xg = (double)(T)__ldcg(Xc + cy * ld + cx);
                    acc += ww * (xg + (double)sxz2[C.g.idx(cx, cy, 0)]);
                }
            }
        const int pf = F.g.idx(i0, i1, nz1);
        sxz1[pf] = (T)(-(double)sxz1[pf - fsz] + acc);
    }
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
template <typename T>
cudaError_t launch_ghost_vz(const GridDev<T> &F, const GridDev<T> &C, int medium, int r, double *coef, cudaStream_t st)
{
    const int m = C.g.ny - 1;
    int P = 32;
    while (P < m) P <<= 1;
    if (P > 1024) return cudaErrorInvalidConfiguration;
    dim3 ba(32, 8), ga((C.g.nx + 31) / 32, (m + 7) / 8);
    ghost_vz_assemble_kernel<T><<<ga, ba, 0, st>>>(F, C, medium, r, coef);
    ghost_vz_solve_kernel<T><<<C.g.nx, P, sizeof(double) * 4 * P, st>>>(C, coef);
    const int nx1 = r * C.g.nx, ny1 = r * C.g.ny;
    dim3 bs(128, 2), gs((nx1 + 127) / 128, (ny1 - 1 + 1) / 2);
    ghost_vz_scatter_kernel<T><<<gs, bs, 0, st>>>(F, C, r);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_ghost_syz(const GridDev<T> &F, const GridDev<T> &C, int r, cudaStream_t st)
{
    dim3 blk(32, 8), grd((C.g.nx + 31) / 32, (C.g.ny + 7) / 8);
    ghost_syz_kernel<T><<<grd, blk, 0, st>>>(F, C, r);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_sxz_matrix(const GridDev<T> &F, const GridDev<T> &C, int r, double *A, cudaStream_t st)
{
    const int nn = (C.g.nx - 1) * (C.g.ny - 1);
    sxz_matrix_kernel<T><<<(nn + 255) / 256, 256, 0, st>>>(F, C, r, A);
    return cudaGetLastError();
}

// Number of co-resident CTAs used by the cooperative sxz solve.
template <typename T>
int sxz_solve_blocks(int nn, int sms)
{
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sxz_solve_kernel<T>, 256, 0) != cudaSuccess || per_sm < 1)
        per_sm = 1;
    int want = (nn + 255) / 256;
    int cap = per_sm * sms;
    if (want > cap) want = cap;
    if (want < 1) want = 1;
    return want;
}

template <typename T>
cudaError_t launch_sxz_solve(const GridDev<T> &F, const GridDev<T> &C, int r, const SxzWork &W, int nblocks,
                             cudaStream_t st)
{
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nblocks);
    cfg.blockDim = dim3(256);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, sxz_solve_kernel<T>, F, C, r, W);
}

#define INST(T)                                                                                         \
    template cudaError_t launch_ghost_vz<T>(const GridDev<T> &, const GridDev<T> &, int, int, double *, cudaStream_t); \
    template cudaError_t launch_ghost_syz<T>(const GridDev<T> &, const GridDev<T> &, int, cudaStream_t);     \
    template cudaError_t launch_sxz_matrix<T>(const GridDev<T> &, const GridDev<T> &, int, double *, cudaStream_t); \
    template int sxz_solve_blocks<T>(int, int);                                                          \
    template cudaError_t launch_sxz_solve<T>(const GridDev<T> &, const GridDev<T> &, int, const SxzWork &, int, cudaStream_t);
INST(float)
INST(double)
#undef INST

} // namespace ecsg
