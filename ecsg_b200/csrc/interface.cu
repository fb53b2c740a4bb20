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
#include "adjoint.cuh"
#include <cstdio>

namespace ecsg {

__device__ __forceinline__ double pw_node(int i, int j, int r, int n2)
{
    if (j <= 0 || j >= n2) return 0.0;
    int d = i - r * j;
    if (d <= -r || d >= r) return 0.0;
    return 1.0 - (double)abs(d) / (double)r;
}
// pw_node for a ratio known at compile time (RR = 2 or 3; 0: the runtime r):
// the weights 1 - |d|/r come from constants the compiler folds with the same
// correctly rounded IEEE arithmetic, so they equal pw_node's bit for bit
// without a division per call
template <int RR>
__device__ __forceinline__ double pw_node_r(int i, int j, int r_, int n2)
{
    const int r = RR ? RR : r_;
    if (j <= 0 || j >= n2) return 0.0;
    const int d = i - r * j;
    if (d <= -r || d >= r) return 0.0;
    const int a = abs(d);
    if (RR == 2) return a == 0 ? 1.0 : 1.0 - 1.0 / 2.0;
    if (RR == 3) return a == 0 ? 1.0 : (a == 1 ? 1.0 - 1.0 / 3.0 : 1.0 - 2.0 / 3.0);
    return 1.0 - (double)a / (double)r;
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

// RR: the refinement ratio when it is known at compile time (2 or 3), so the
// loops over the (2r-1)^2 fine points unroll and their loads overlap; 0: r.
template <typename T, int RR>
__device__ double sxz_rhs(const GridDev<T> &F, const GridDev<T> &C, int r_, int j0, int j1)
{
    const int r = RR ? RR : r_;
    const int nx2 = C.g.nx, ny2 = C.g.ny, nz1 = F.g.nz;
    const T *vx1 = F.f[VX], *sxx1 = F.f[SXX], *sxz1 = F.f[SXZ], *sxy1 = F.f[SXY], *b1 = F.b;
    const T *vx2 = C.f[VX], *sxx2 = C.f[SXX], *sxz2 = C.f[SXZ], *sxy2 = C.f[SXY], *b2 = C.b;
    const double k1x = F.kd[0], k1y = F.kd[1], k1z = F.kd[2];
    const double k2x = C.kd[0], k2y = C.kd[1], k2z = C.kd[2];
    const double rr = (double)r, r2 = rr * rr, r4 = r2 * r2;
    const int sy1 = F.g.px, sz1 = F.g.px * F.g.py, sy2 = C.g.px;
    double fsum = 0.0;
#pragma unroll
    for (int a1 = 0; a1 < 2 * r - 1; a1++) {
        const int i1 = r * j1 - r + 1 + a1;
        const double wy = pw_node_r<RR>(i1, j1, r, ny2);
        const int jy = i1 / r;
#pragma unroll
        for (int a0 = 0; a0 < 2 * r - 1; a0++) {
            const int i0 = r * j0 - r + 1 + a0;
            const double w = pw_node_r<RR>(i0, j0, r, nx2) * wy;
            const int jx = i0 / r;
            double ps0 = 0.0;
            for (int ey = 0; ey < 2; ey++)
                for (int ex = 0; ex < 2; ex++) {
                    const int cx = jx + ex, cy = jy + ey;
                    if (cx > nx2 || cy > ny2) continue;
                    const double ww = pw_node_r<RR>(i0, cx, r, nx2) * pw_node_r<RR>(i1, cy, r, ny2);
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

// Grid-wide deterministic sum.  Each CTA writes its partial into the half of
// W.partial that belongs to this round (rounds alternate between two halves of
// gridDim.x doubles, so a CTA that has already left round k cannot overwrite a
// partial of round k that a slower CTA is still reading: to write into the same
// half again it must pass round k+1, which the slower CTA has not reached),
// then arrives at a barrier: one master thread per CTA releases the CTA's
// writes with a fence and adds to the arrival count; the last to arrive resets
// the count and advances the generation word, the others spin on it.  After
// the barrier every CTA sums all partials in the same fixed order (strided
// split, then a fixed tree), so every CTA gets the same total with no second
// publication round.  Waiting is bounded: on timeout the status bit is set, ok
// becomes false and the caller stops.
// Publish this CTA's partial of round `round` and wait for every CTA (the
// barrier half of grid_sum).  One master thread per CTA releases the CTA's
// writes with a fence and adds to the arrival count; the last to arrive
// resets the count and advances the generation word, on which the others
// wait.  The count and the polled generation sit on separate 128-byte lines.
__device__ void grid_arrive(double v, const SxzWork &W, double *red, bool &ok, int &round)
{
    const double bs = block_sum(v, red);   // valid in thread 0; ends with a CTA barrier
    __shared__ int s_ok;
    double *part = W.partial + (size_t)(round & 1) * gridDim.x;
    round++;
    if (threadIdx.x == 0) {
        unsigned *gen_w = W.bar, *cnt_w = W.bar + 32;
        const unsigned gen = *(volatile unsigned *)gen_w;   // generation of this round, read before arriving
        __stcg(part + blockIdx.x, bs);
        __threadfence();
        int okv = 1;
        if (atomicAdd(cnt_w, 1u) == gridDim.x - 1) {
            *cnt_w = 0;
            __threadfence();
            atomicAdd(gen_w, 1u);
        } else {
            long long spin = 0;
            while (*(volatile unsigned *)gen_w == gen) {
                if (++spin > kSpinLimit) { atomicOr(W.status, ST_BARRIER_TIMEOUT); okv = 0; break; }
                __nanosleep(32);
            }
        }
        __threadfence();
        s_ok = okv;
    }
    __syncthreads();
    ok = s_ok != 0;
}

// This thread's share of the partials of a finished round (fixed strided split)
__device__ __forceinline__ double partial_share(const SxzWork &W, int finished_round)
{
    const double *part = W.partial + (size_t)(finished_round & 1) * gridDim.x;
    double t = 0.0;
    for (unsigned i = threadIdx.x; i < gridDim.x; i += blockDim.x) t += __ldcg(part + i);
    return t;
}

// The total of a share over the CTA (fixed tree), returned to every thread
__device__ __forceinline__ double share_total(double t, double *red)
{
    __shared__ double s_total;
    const double tot = block_sum(t, red);
    if (threadIdx.x == 0) s_total = tot;
    __syncthreads();
    return s_total;
}

__device__ double grid_sum(double v, const SxzWork &W, double *red, bool &ok, int &round)
{
    grid_arrive(v, W, red, ok, round);
    return share_total(partial_share(W, round - 1), red);
}

template <typename T, int RR>
__global__ void __launch_bounds__(256, 4) sxz_solve_kernel(GridDev<T> F, GridDev<T> C, int r, SxzWork W)
{
    __shared__ double red[32];
    const int nx2 = C.g.nx, ny2 = C.g.ny, nz1 = F.g.nz;
    const int n0 = nx2 - 1, n1 = ny2 - 1, ld = nx2 + 1;
    const int nn = n0 * n1;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x;
    const int gstride = gridDim.x * blockDim.x;
    bool ok = true;
    int round = 0;   // grid_sum rounds (alternating halves of W.partial)

    // B and avg|B| (Array::AvgAbs, array.cpp:172-210)
    double sab = 0.0;
    for (int q = gtid; q < nn; q += gstride) {
        const double bq = sxz_rhs<T, RR>(F, C, r, q % n0 + 1, q / n0 + 1);
        W.B[q] = bq;
        sab += fabs(bq);
    }
    const double sumabs = grid_sum(sab, W, red, ok, round);
    double tol = 1e-5 * (sumabs / (double)nn);
    if (tol > 1e-12) tol = 1e-12;

    // Jacobi2D (update_ghost_sxz.cpp:314-350), ping-pong instead of copy
    double *Xc = W.X0, *Xn = W.X1;
    // the row of A and the entry of B of this thread's first unknown stay in
    // registers for the whole solve (further unknowns, on grids with more
    // unknowns than threads, are read from memory)
    double a0[9] = {0, 0, 0, 0, 1, 0, 0, 0, 0}, b0 = 0.0;
    if (gtid < nn) {
#pragma unroll
        for (int k = 0; k < 9; k++) a0[k] = W.A[(size_t)k * nn + gtid];
        b0 = W.B[gtid];
    }
    auto update = [&](const double *Xo, double *Xw, int q, const double (&a)[9], double bq) {
        const int i0 = q % n0 + 1, i1 = q / n0 + 1;
        const double xn = (bq
                           - a[0] * __ldcg(Xo + (i1 - 1) * ld + (i0 - 1))
                           - a[1] * __ldcg(Xo + (i1) * ld + (i0 - 1))
                           - a[2] * __ldcg(Xo + (i1 + 1) * ld + (i0 - 1))
                           - a[3] * __ldcg(Xo + (i1 - 1) * ld + (i0))
                           - a[5] * __ldcg(Xo + (i1 + 1) * ld + (i0))
                           - a[6] * __ldcg(Xo + (i1 - 1) * ld + (i0 + 1))
                           - a[7] * __ldcg(Xo + (i1) * ld + (i0 + 1))
                           - a[8] * __ldcg(Xo + (i1 + 1) * ld + (i0 + 1))) / a[4];
        const double d = xn - __ldcg(Xo + i1 * ld + i0);
        __stcg(Xw + i1 * ld + i0, xn);
        return d * d;
    };
    auto sweep = [&](const double *Xo, double *Xw) {
        double s = 0.0;
        if (gtid < nn) s += update(Xo, Xw, gtid, a0, b0);
        for (int q = gtid + gstride; q < nn; q += gstride) {
            double a[9];
#pragma unroll
            for (int k = 0; k < 9; k++) a[k] = W.A[(size_t)k * nn + q];
            s += update(Xo, Xw, q, a, W.B[q]);
        }
        return s;
    };
    int it = 0;
    while (ok) {
        const double s = sweep(Xc, Xn);
        const double tot = grid_sum(s, W, red, ok, round);
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
    // the same points per thread (q = gtid + k gstride) in batches of NB: every
    // load of a batch before its stores, so the loads of a batch overlap
    constexpr int NB = 4;
    for (int q0 = gtid; q0 < nf; q0 += NB * gstride) {
        double val[NB];
        int pfs[NB];
#pragma unroll
        for (int b = 0; b < NB; b++) {
            const int q = q0 + b * gstride;
            pfs[b] = -1;
            val[b] = 0.0;
            if (q >= nf) continue;
            const int i0 = q % (nx1 - 1) + 1, i1 = q / (nx1 - 1) + 1;
            const int jx = i0 / r, jy = i1 / r;
            double acc = 0.0;
            for (int ey = 0; ey < 2; ey++)
                for (int ex = 0; ex < 2; ex++) {
                    const int cx = jx + ex, cy = jy + ey;
                    if (cx > nx2 || cy > ny2) continue;
                    const double ww = pw_node_r<RR>(i0, cx, r, nx2) * pw_node_r<RR>(i1, cy, r, ny2);
                    if (ww != 0.0) {
                        const double xg = (double)(T)__ldcg(Xc + cy * ld + cx);
                        acc += ww * (xg + (double)sxz2[C.g.idx(cx, cy, 0)]);
                    }
                }
            pfs[b] = F.g.idx(i0, i1, nz1);
            val[b] = -(double)sxz1[pfs[b] - fsz] + acc;
        }
#pragma unroll
        for (int b = 0; b < NB; b++)
            if (pfs[b] >= 0) sxz1[pfs[b]] = (T)val[b];
    }
}

// ---------------------------------------------------------------------------
// Several independent sxz systems in one cooperative launch (the interfaces of
// one step, or one interface of several shots).  System i owns CTAs
// [cta0, cta0 + ncta) and maps its unknowns, its right-hand side and its
// partial sums onto them exactly as its own launch with ncta CTAs would, so
// its result is bitwise that of sxz_solve_kernel.  All CTAs share one grid
// barrier per round; after it every CTA forms the totals of every system in
// the same fixed order and takes the same stopping decisions, so a system
// that has converged (or hit its cap) stops updating while the others go on,
// and every CTA runs the same number of rounds.  The barrier's arrival count
// and generation words are the list's; each system keeps its own partials,
// status, sweep counts and warm start.
// ---------------------------------------------------------------------------
__device__ void grid_arrive_list(double v, double *slot, unsigned *bar, int *status, double *red, bool &ok)
{
    const double bs = block_sum(v, red);   // valid in thread 0; ends with a CTA barrier
    __shared__ int s_ok;
    if (threadIdx.x == 0) {
        unsigned *gen_w = bar, *cnt_w = bar + 32;
        const unsigned gen = *(volatile unsigned *)gen_w;
        __stcg(slot, bs);
        __threadfence();
        int okv = 1;
        if (atomicAdd(cnt_w, 1u) == gridDim.x - 1) {
            *cnt_w = 0;
            __threadfence();
            atomicAdd(gen_w, 1u);
        } else {
            long long spin = 0;
            while (*(volatile unsigned *)gen_w == gen) {
                if (++spin > kSpinLimit) { atomicOr(status, ST_BARRIER_TIMEOUT); okv = 0; break; }
                __nanosleep(32);
            }
        }
        __threadfence();
        s_ok = okv;
    }
    __syncthreads();
    ok = s_ok != 0;
}

// total of one system's partials of a finished round: partial_share's strided
// split over that system's CTAs, then share_total's tree
__device__ __forceinline__ double system_total(const double *part, int ncta, double *red)
{
    double t = 0.0;
    for (int i = threadIdx.x; i < ncta; i += blockDim.x) t += __ldcg(part + i);
    return share_total(t, red);
}

template <typename T, int RR>
__global__ void __launch_bounds__(256, 4) sxz_solve_multi_kernel(const __grid_constant__ SxzSysList<T> L)
{
    __shared__ double red[32];
    __shared__ double s_tol[kMaxSxzSys];
    __shared__ int s_it[kMaxSxzSys], s_act[kMaxSxzSys], s_cap[kMaxSxzSys];
    int me = 0;
    for (int i = 1; i < L.n; i++)
        if ((int)blockIdx.x >= L.s[i].cta0) me = i;
    const SxzSys<T> &S = L.s[me];
    const GridDev<T> &F = S.F, &C = S.C;
    const SxzWork &W = S.W;
    const int r = L.r;
    const int lb = blockIdx.x - S.cta0, ncta = S.ncta;
    const int nx2 = C.g.nx, ny2 = C.g.ny, nz1 = F.g.nz;
    const int n0 = nx2 - 1, n1 = ny2 - 1, ld = nx2 + 1;
    const int nn = n0 * n1;
    const int gtid = lb * blockDim.x + threadIdx.x;
    const int gstride = ncta * blockDim.x;
    bool ok = true;
    int round = 0;
    auto slot = [&](const SxzSys<T> &Y, int rd, int b) { return Y.W.partial + (size_t)(rd & 1) * Y.ncta + b; };

    // B and avg|B| of this CTA's system
    double sab = 0.0;
    for (int q = gtid; q < nn; q += gstride) {
        const double bq = sxz_rhs<T, RR>(F, C, r, q % n0 + 1, q / n0 + 1);
        W.B[q] = bq;
        sab += fabs(bq);
    }
    grid_arrive_list(sab, slot(S, round, lb), L.bar, L.status, red, ok);
    round++;
    for (int i = 0; i < L.n; i++) {
        const SxzSys<T> &Y = L.s[i];
        const double sumabs = system_total(slot(Y, round - 1, 0), Y.ncta, red);
        if (threadIdx.x == 0) {
            const int nni = (Y.C.g.nx - 1) * (Y.C.g.ny - 1);
            double tol = 1e-5 * (sumabs / (double)nni);
            if (tol > 1e-12) tol = 1e-12;
            s_tol[i] = tol;
            s_it[i] = 0;
            s_act[i] = 1;
            s_cap[i] = 0;
        }
    }
    __syncthreads();

    double *Xc = W.X0, *Xn = W.X1;
    double a0[9] = {0, 0, 0, 0, 1, 0, 0, 0, 0}, b0 = 0.0;
    if (gtid < nn) {
#pragma unroll
        for (int k = 0; k < 9; k++) a0[k] = W.A[(size_t)k * nn + gtid];
        b0 = W.B[gtid];
    }
    auto update = [&](const double *Xo, double *Xw, int q, const double (&a)[9], double bq) {
        const int i0 = q % n0 + 1, i1 = q / n0 + 1;
        const double xn = (bq
                           - a[0] * __ldcg(Xo + (i1 - 1) * ld + (i0 - 1))
                           - a[1] * __ldcg(Xo + (i1) * ld + (i0 - 1))
                           - a[2] * __ldcg(Xo + (i1 + 1) * ld + (i0 - 1))
                           - a[3] * __ldcg(Xo + (i1 - 1) * ld + (i0))
                           - a[5] * __ldcg(Xo + (i1 + 1) * ld + (i0))
                           - a[6] * __ldcg(Xo + (i1 - 1) * ld + (i0 + 1))
                           - a[7] * __ldcg(Xo + (i1) * ld + (i0 + 1))
                           - a[8] * __ldcg(Xo + (i1 + 1) * ld + (i0 + 1))) / a[4];
        const double d = xn - __ldcg(Xo + i1 * ld + i0);
        __stcg(Xw + i1 * ld + i0, xn);
        return d * d;
    };
    auto sweep = [&](const double *Xo, double *Xw) {
        double s = 0.0;
        if (gtid < nn) s += update(Xo, Xw, gtid, a0, b0);
        for (int q = gtid + gstride; q < nn; q += gstride) {
            double a[9];
#pragma unroll
            for (int k = 0; k < 9; k++) a[k] = W.A[(size_t)k * nn + q];
            s += update(Xo, Xw, q, a, W.B[q]);
        }
        return s;
    };
    bool any = true;
    while (ok && any) {
        const bool mine = s_act[me] != 0;
        const double s = mine ? sweep(Xc, Xn) : 0.0;
        grid_arrive_list(s, slot(S, round, lb), L.bar, L.status, red, ok);
        round++;
        if (!ok) break;
        for (int i = 0; i < L.n; i++) {
            if (!s_act[i]) continue;   // uniform over the CTA (shared, set by thread 0 below a barrier)
            const SxzSys<T> &Y = L.s[i];
            const double tot = system_total(slot(Y, round - 1, 0), Y.ncta, red);
            if (threadIdx.x == 0) {
                s_it[i]++;
                if (!(sqrt(tot) > s_tol[i])) s_act[i] = 0;
                else if (s_it[i] >= Y.W.max_iter) { s_act[i] = 0; s_cap[i] = 1; }
            }
        }
        __syncthreads();
        if (mine) { double *tmp = Xc; Xc = Xn; Xn = tmp; }
        any = false;
        for (int i = 0; i < L.n; i++) any = any || s_act[i] != 0;
        __syncthreads();   // every thread has read s_act before thread 0 changes it again
    }
    if (gtid == 0) {
        *W.iters = s_it[me];
        *W.iters_total += s_it[me];
        *W.tol_out = s_tol[me];
        if (s_cap[me]) atomicOr(W.status, ST_JACOBI_CAP);
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
    constexpr int NB = 4;
    for (int q0 = gtid; q0 < nf; q0 += NB * gstride) {
        double val[NB];
        int pfs[NB];
#pragma unroll
        for (int b = 0; b < NB; b++) {
            const int q = q0 + b * gstride;
            pfs[b] = -1;
            val[b] = 0.0;
            if (q >= nf) continue;
            const int i0 = q % (nx1 - 1) + 1, i1 = q / (nx1 - 1) + 1;
            const int jx = i0 / r, jy = i1 / r;
            double acc = 0.0;
            for (int ey = 0; ey < 2; ey++)
                for (int ex = 0; ex < 2; ex++) {
                    const int cx = jx + ex, cy = jy + ey;
                    if (cx > nx2 || cy > ny2) continue;
                    const double ww = pw_node_r<RR>(i0, cx, r, nx2) * pw_node_r<RR>(i1, cy, r, ny2);
                    if (ww != 0.0) {
                        const double xg = (double)(T)__ldcg(Xc + cy * ld + cx);
                        acc += ww * (xg + (double)sxz2[C.g.idx(cx, cy, 0)]);
                    }
                }
            pfs[b] = F.g.idx(i0, i1, nz1);
            val[b] = -(double)sxz1[pfs[b] - fsz] + acc;
        }
#pragma unroll
        for (int b = 0; b < NB; b++)
            if (pfs[b] >= 0) sxz1[pfs[b]] = (T)val[b];
    }
}

// ===========================================================================
// Adjoints of the three interface solves (no reference counterpart).  Each
// forward solve overwrites ghost entries with X = A^{-1} rhs(state) and the
// fine ghosts with -(last fine interior) + P(coarse ghost + coarse first
// interior).  Given the adjoint of its output state (in place on the adjoint
// fields of both grids) these kernels
//   1. collect the adjoint of X from the overwritten entries (and zero them),
//      passing the scatter's other reads on;
//   2. solve A^T y = lambda_X (A is symmetric: the vz lines transposed row by
//      row, the sxz 9-point system by bounded Jacobi sweeps);
//   3. add rhs^T y to the adjoint fields and y^T (d rhs/dm - dA/dm X) to the
//      medium gradients (21-Cij slots for vz, node buoyancy for sxz and syz).
// The forward fields hold the solve's output state: the rhs reads no entry the
// solve overwrites, so rhs and X are both available there.  Adjoint path:
// 21-Cij media only (the general form of every medium).
// ===========================================================================

// transpose of the strain increment of kind 4, 5 or 6 at point q (e4_at..e6_at)
template <typename T>
__device__ __forceinline__ void e_adj(const GridDev<T> &G, T *const lv[3], int kind, int q, double a)
{
    const int sy = G.g.px, sz = G.g.px * G.g.py;
    if (kind == 4) {
        const double u2 = G.kd[2] * a, u1 = G.kd[1] * a;
        atom(lv[VY] + q + sz, (T)u2); atom(lv[VY] + q, (T)-u2); atom(lv[VZ] + q + sy, (T)u1); atom(lv[VZ] + q, (T)-u1);
    } else if (kind == 5) {
        const double u2 = G.kd[2] * a, u0 = G.kd[0] * a;
        atom(lv[VX] + q + sz, (T)u2); atom(lv[VX] + q, (T)-u2); atom(lv[VZ] + q, (T)u0); atom(lv[VZ] + q - 1, (T)-u0);
    } else {
        const double u1 = G.kd[1] * a, u0 = G.kd[0] * a;
        atom(lv[VX] + q + sy, (T)u1); atom(lv[VX] + q, (T)-u1); atom(lv[VY] + q, (T)u0); atom(lv[VY] + q - 1, (T)-u0);
    }
}

// transpose of Abar4/5/6 at an N point (gen21_device.cuh abar*_g): a * weight to each neighbour's strain
template <typename T>
__device__ void abar_adj(const GridDev<T> &G, T *const lv[3], int kind, int x, int y, int z, double a)
{
    const Ext E{G.g.nx, G.g.ny, G.g.nz};
    bool o0[2], o1[2];
    int dx[2][2], dy[2][2], dz[2][2];
    for (int i = 0; i < 2; i++) {
        if (kind == 4) { o0[i] = (y - 1 + i) >= 0 && (y - 1 + i) <= E.ny - 1; o1[i] = (z - 1 + i) >= 0 && (z - 1 + i) <= E.nz - 1; }
        else if (kind == 5) { o0[i] = (x + i) >= 0 && (x + i) <= E.nx; o1[i] = (z - 1 + i) >= 0 && (z - 1 + i) <= E.nz - 1; }
        else { o0[i] = (x + i) >= 0 && (x + i) <= E.nx; o1[i] = (y - 1 + i) >= 0 && (y - 1 + i) <= E.ny - 1; }
    }
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) {
            dx[i][j] = kind == 4 ? 0 : i;
            dy[i][j] = kind == 4 ? i - 1 : (kind == 5 ? 0 : j - 1);
            dz[i][j] = kind == 6 ? 0 : j - 1;
        }
    double wa0, wa1, wb0, wb1;
    w2<double>(o0[0], o0[1], wa0, wa1);
    w2<double>(o1[0], o1[1], wb0, wb1);
    const double wa[2] = {wa0, wa1}, wb[2] = {wb0, wb1};
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) {
            const double w = wa[i] * wb[j];
            if (w != 0.0) e_adj(G, lv, kind, G.g.idx(x + dx[i][j], y + dy[i][j], z + dz[i][j]), a * w);
        }
}

// ---- vz -------------------------------------------------------------------
// lambda_X from the coarse ghosts (lx[j1-1][j0], j1 in [1, m]); zero them
template <typename T>
__global__ void vz_adj_collect_coarse(GridDev<T> C, AdjDev<T> AC, double *lx)
{
    const int j0 = blockIdx.x * blockDim.x + threadIdx.x, j1 = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int nx2 = C.g.nx, m = C.g.ny - 1;
    if (j0 >= nx2 || j1 > m) return;
    const int q = C.g.idx(j0, j1, -1);
    lx[(size_t)(j1 - 1) * nx2 + j0] = (double)AC.l[VZ][q];
    AC.l[VZ][q] = T(0);
}

// the fine ghosts vz1(i0, i1, nz1) = -vz1(i0, i1, nz1-1) + sum_j w (vz2(j0, j, 0) + vz2(j0, j, -1))
template <typename T>
__global__ void vz_adj_collect_fine(GridDev<T> F, GridDev<T> C, AdjDev<T> AF, AdjDev<T> AC, int r, double *lx)
{
    const int i0 = blockIdx.x * blockDim.x + threadIdx.x, i1 = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int nx2 = C.g.nx, ny2 = C.g.ny, m = ny2 - 1;
    const int nx1 = r * nx2, ny1 = r * ny2, nz1 = F.g.nz;
    if (i0 >= nx1 || i1 >= ny1) return;
    const int pf = F.g.idx(i0, i1, nz1), fsz = F.g.px * F.g.py;
    const T a = AF.l[VZ][pf];
    if (a == T(0)) return;
    AF.l[VZ][pf] = T(0);
    AF.l[VZ][pf - fsz] = AF.l[VZ][pf - fsz] - a;
    const int j0 = i0 / r, jl = i1 / r;
    for (int j = jl; j <= jl + 1 && j <= ny2; j++) {
        const double w = pw_node_all(i1, j, r);
        if (w == 0.0) continue;
        atom(AC.l[VZ] + C.g.idx(j0, j, 0), (T)(w * (double)a));
        if (j >= 1 && j <= m) atomicAdd(lx + (size_t)(j - 1) * nx2 + j0, w * (double)a);
        else atom(AC.l[VZ] + C.g.idx(j0, j, -1), (T)(w * (double)a));
    }
}

// y = A^{-T} lambda_X per coarse x-cell: the rows of A^T are (up[j-1], dg[j], lo[j+1])
__global__ void vz_adj_solve_kernel(int nx2, int m, const double *coef, const double *lx, double *y)
{
    extern __shared__ double sm[];
    const int P = blockDim.x, t = threadIdx.x, j0 = blockIdx.x;
    double *A = sm, *B = sm + P, *Cc = sm + 2 * P, *D = sm + 3 * P;
    const size_t plane = (size_t)m * nx2;
    auto at = [&](int k, int row) { return coef[k * plane + (size_t)row * nx2 + j0]; };
    A[t] = (t < m && t >= 1) ? at(2, t - 1) : 0.0;      // sub-diagonal of A^T: up of the row above
    B[t] = t < m ? at(1, t) : 1.0;
    Cc[t] = (t + 1 < m) ? at(0, t + 1) : 0.0;           // super-diagonal of A^T: lo of the row below
    D[t] = t < m ? lx[(size_t)t * nx2 + j0] : 0.0;
    __syncthreads();
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
    if (t < m) y[(size_t)t * nx2 + j0] = D[t] / B[t];
}

// rhs^T y and the gradients, coarse rows: rhs = r^3 pred(c) - fsum
template <typename T>
__global__ void vz_adj_coarse(GridDev<T> C, AdjDev<T> AC, int r, const double *y)
{
    const int j0 = blockIdx.x * blockDim.x + threadIdx.x, j1 = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int nx2 = C.g.nx, m = C.g.ny - 1;
    if (j0 >= nx2 || j1 > m) return;
    const double yv = y[(size_t)(j1 - 1) * nx2 + j0];
    if (yv == 0.0) return;
    const double rr = (double)r, r3 = rr * rr * rr, u = r3 * yv;
    const double k2x = C.kd[0], k2y = C.kd[1], k2z = C.kd[2];
    const int pc = C.g.idx(j0, j1, 0), pxp = C.g.idx(j0 + 1, j1, 0), pym = C.g.idx(j0, j1 - 1, 0);
    const double c13 = (double)C.c[2][pc], c23 = (double)C.c[4][pc], c33 = (double)C.c[5][pc];
    const T *vx2 = C.f[VX], *vy2 = C.f[VY], *vz2 = C.f[VZ];
    atom(AC.l[SZZ] + pc, (T)u);
    atom(AC.l[VX] + pxp, (T)(u * c13 * k2x)); atom(AC.l[VX] + pc, (T)(-u * c13 * k2x));
    atom(AC.l[VY] + pc, (T)(u * c23 * k2y)); atom(AC.l[VY] + pym, (T)(-u * c23 * k2y));
    atom(AC.l[VZ] + pc, (T)(u * c33 * k2z));
    const double xg = (double)vz2[C.g.idx(j0, j1, -1)];
    AC.gc[2][pc] = (T)((double)AC.gc[2][pc] + u * k2x * ((double)vx2[pxp] - (double)vx2[pc]));
    AC.gc[4][pc] = (T)((double)AC.gc[4][pc] + u * k2y * ((double)vy2[pc] - (double)vy2[pym]));
    AC.gc[5][pc] = (T)((double)AC.gc[5][pc] + u * k2z * ((double)vz2[pc] - xg));
    const Ext E{C.g.nx, C.g.ny, C.g.nz};
    const double ab[3] = {(double)abar4_g(C, E, j0, j1, 0), (double)abar5_g(C, E, j0, j1, 0), (double)abar6_g(C, E, j0, j1, 0)};
    T *lv[3] = {AC.l[VX], AC.l[VY], AC.l[VZ]};
    for (int k = 0; k < 3; k++) {
        AC.gc[12 + k][pc] = (T)((double)AC.gc[12 + k][pc] + u * ab[k]);
        abar_adj(C, lv, 4 + k, j0, j1, 0, u * (double)C.c[12 + k][pc]);
    }
}

// fine points: beta = sum over rows r w(i1, j1) y(j0, j1) enters as -beta * pf
template <typename T>
__global__ void vz_adj_fine(GridDev<T> F, GridDev<T> C, AdjDev<T> AF, AdjDev<T> AC, int r, const double *y)
{
    const int i0 = blockIdx.x * blockDim.x + threadIdx.x, i1 = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int nx2 = C.g.nx, ny2 = C.g.ny, m = ny2 - 1;
    const int nx1 = r * nx2, ny1 = r * ny2, nz1 = F.g.nz;
    if (i0 >= nx1 || i1 >= ny1) return;
    const int j0 = i0 / r, jl = i1 / r;
    const double rr = (double)r;
    double beta = 0.0, px = 0.0;
    for (int j = jl; j <= jl + 1; j++) {
        if (j < 1 || j > m) continue;
        const double w = pw_node(i1, j, r, ny2);
        beta += rr * w * y[(size_t)(j - 1) * nx2 + j0];
        px += w * (double)C.f[VZ][C.g.idx(j0, j, -1)];
    }
    if (beta == 0.0) return;
    const double k1x = F.kd[0], k1y = F.kd[1], k1z = F.kd[2];
    const int pf = F.g.idx(i0, i1, nz1), fsy = F.g.px, fsz = F.g.px * F.g.py;
    const double f13 = (double)F.c[2][pf], f23 = (double)F.c[4][pf], f33 = (double)F.c[5][pf], cz = f33 * k1z;
    const T *vx1 = F.f[VX], *vy1 = F.f[VY], *vz1 = F.f[VZ], *vz2 = C.f[VZ];
    atom(AF.l[SZZ] + pf, (T)-beta);
    atom(AF.l[VX] + pf + 1, (T)(-beta * f13 * k1x)); atom(AF.l[VX] + pf, (T)(beta * f13 * k1x));
    atom(AF.l[VY] + pf, (T)(-beta * f23 * k1y)); atom(AF.l[VY] + pf - fsy, (T)(beta * f23 * k1y));
    atom(AF.l[VZ] + pf - fsz, (T)(2.0 * beta * cz));
    double pv0 = 0.0;
    for (int j = jl; j <= jl + 1 && j <= ny2; j++) {
        const double w = pw_node_all(i1, j, r);
        if (w == 0.0) continue;
        const int pc = C.g.idx(j0, j, 0);
        pv0 += w * (double)vz2[pc];
        atom(AC.l[VZ] + pc, (T)(-beta * cz * w));
    }
    AF.gc[2][pf] = (T)((double)AF.gc[2][pf] - beta * k1x * ((double)vx1[pf + 1] - (double)vx1[pf]));
    AF.gc[4][pf] = (T)((double)AF.gc[4][pf] - beta * k1y * ((double)vy1[pf] - (double)vy1[pf - fsy]));
    AF.gc[5][pf] = (T)((double)AF.gc[5][pf] - beta * k1z * (pv0 - 2.0 * (double)vz1[pf - fsz] + px));
    const Ext E{F.g.nx, F.g.ny, F.g.nz};
    const double ab[3] = {(double)abar4_g(F, E, i0, i1, nz1), (double)abar5_g(F, E, i0, i1, nz1), (double)abar6_g(F, E, i0, i1, nz1)};
    T *lv[3] = {AF.l[VX], AF.l[VY], AF.l[VZ]};
    for (int k = 0; k < 3; k++) {
        AF.gc[12 + k][pf] = (T)((double)AF.gc[12 + k][pf] - beta * ab[k]);
        abar_adj(F, lv, 4 + k, i0, i1, nz1, -beta * (double)F.c[12 + k][pf]);
    }
}

// ---- syz ------------------------------------------------------------------
// per coarse cell: t = num / den, fine ghosts -syz1(nz1-1) + t + syz2(0)
template <typename T>
__global__ void syz_adj_kernel(GridDev<T> F, GridDev<T> C, AdjDev<T> AF, AdjDev<T> AC, int r)
{
    const int j0 = blockIdx.x * blockDim.x + threadIdx.x, j1 = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx2 = C.g.nx, ny2 = C.g.ny, nz1 = F.g.nz;
    if (j0 >= nx2 || j1 >= ny2) return;
    const int fsy = F.g.px, fsz = F.g.px * F.g.py, csy = C.g.px;
    const int pg = C.g.idx(j0, j1, -1), p0 = C.g.idx(j0, j1, 0);
    double lt = (double)AC.l[SYZ][pg];
    AC.l[SYZ][pg] = T(0);
    double ls0 = 0.0;
    for (int i1 = r * j1; i1 < r * j1 + r; i1++)
        for (int i0 = r * j0; i0 < r * j0 + r; i0++) {
            const int pf = F.g.idx(i0, i1, nz1);
            const T a = AF.l[SYZ][pf];
            if (a == T(0)) continue;
            AF.l[SYZ][pf] = T(0);
            AF.l[SYZ][pf - fsz] = AF.l[SYZ][pf - fsz] - a;
            lt += (double)a;
            ls0 += (double)a;
        }
    const double k1x = F.kd[0], k1y = F.kd[1], k1z = F.kd[2];
    const double k2x = C.kd[0], k2y = C.kd[1], k2z = C.kd[2];
    const double r2 = (double)r * (double)r;
    const T *b1 = F.b, *b2 = C.b;
    const T *vy2 = C.f[VY], *sxy2 = C.f[SXY], *syy2 = C.f[SYY], *syz2 = C.f[SYZ];
    const T *sxy1 = F.f[SXY], *syy1 = F.f[SYY], *syz1 = F.f[SYZ];
    const double c0 = 0.25 * ((double)b2[p0] + (double)b2[p0 + 1] + (double)b2[p0 + csy] + (double)b2[p0 + csy + 1]);
    double den = r2 * c0 * k2z;
    for (int i1 = r * j1; i1 < r * j1 + r; i1++)
        for (int i0 = r * j0; i0 < r * j0 + r; i0++) {
            const int pf = F.g.idx(i0, i1, nz1);
            den += 0.25 * ((double)b1[pf] + (double)b1[pf + 1] + (double)b1[pf + fsy] + (double)b1[pf + fsy + 1]) * k1z;
        }
    const double tg = (double)syz2[pg];   // the forward ghost t
    const double s0 = (double)syz2[p0];
    if (lt != 0.0) {
        const double u = lt / den;
        const double cu = r2 * u;
        atom(AC.l[VY] + p0, (T)cu);
        atom(AC.l[SXY] + p0 + 1, (T)(cu * c0 * k2x)); atom(AC.l[SXY] + p0, (T)(-cu * c0 * k2x));
        atom(AC.l[SYY] + p0 + csy, (T)(cu * c0 * k2y)); atom(AC.l[SYY] + p0, (T)(-cu * c0 * k2y));
        ls0 += cu * c0 * k2z;
        // d t / d c0 = (r^2 (k2x dsxy + k2y dsyy + k2z s0) - t r^2 k2z) / den, c0 = mean of 4 nodes
        const double dc0 = r2 * (k2x * ((double)sxy2[p0 + 1] - (double)sxy2[p0]) + k2y * ((double)syy2[p0 + csy] - (double)syy2[p0])
                                 + k2z * s0) - tg * r2 * k2z;
        const double gq = 0.25 * u * dc0;
        atom(AC.gb + p0, (T)gq); atom(AC.gb + p0 + 1, (T)gq); atom(AC.gb + p0 + csy, (T)gq); atom(AC.gb + p0 + csy + 1, (T)gq);
        for (int i1 = r * j1; i1 < r * j1 + r; i1++)
            for (int i0 = r * j0; i0 < r * j0 + r; i0++) {
                const int pf = F.g.idx(i0, i1, nz1);
                const double c = 0.25 * ((double)b1[pf] + (double)b1[pf + 1] + (double)b1[pf + fsy] + (double)b1[pf + fsy + 1]);
                atom(AF.l[VY] + pf, (T)-u);
                atom(AF.l[SXY] + pf + 1, (T)(-u * c * k1x)); atom(AF.l[SXY] + pf, (T)(u * c * k1x));
                atom(AF.l[SYY] + pf + fsy, (T)(-u * c * k1y)); atom(AF.l[SYY] + pf, (T)(u * c * k1y));
                ls0 -= u * c * k1z;
                atom(AF.l[SYZ] + pf - fsz, (T)(2.0 * u * c * k1z));
                const double dc = -(k1x * ((double)sxy1[pf + 1] - (double)sxy1[pf]) + k1y * ((double)syy1[pf + fsy] - (double)syy1[pf])
                                    + k1z * (s0 - 2.0 * (double)syz1[pf - fsz])) - tg * k1z;
                const double g1 = 0.25 * u * dc;
                atom(AF.gb + pf, (T)g1); atom(AF.gb + pf + 1, (T)g1); atom(AF.gb + pf + fsy, (T)g1); atom(AF.gb + pf + fsy + 1, (T)g1);
            }
    }
    if (ls0 != 0.0) atom(AC.l[SYZ] + p0, (T)ls0);
}

// ---- sxz ------------------------------------------------------------------
// lambda_X at the interior coarse nodes (lx[(j1-1) n0 + j0-1]) from the ghosts
template <typename T>
__global__ void sxz_adj_collect_coarse(GridDev<T> C, AdjDev<T> AC, double *lx)
{
    const int n0 = C.g.nx - 1, n1 = C.g.ny - 1;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n0 * n1) return;
    const int j0 = q % n0 + 1, j1 = q / n0 + 1;
    const int pg = C.g.idx(j0, j1, -1);
    lx[q] = (double)AC.l[SXZ][pg];
    AC.l[SXZ][pg] = T(0);
}

template <typename T>
__global__ void sxz_adj_collect_fine(GridDev<T> F, GridDev<T> C, AdjDev<T> AF, AdjDev<T> AC, int r, double *lx)
{
    const int nx2 = C.g.nx, ny2 = C.g.ny, n0 = nx2 - 1, nz1 = F.g.nz;
    const int nx1 = r * nx2, ny1 = r * ny2;
    const int i0 = blockIdx.x * blockDim.x + threadIdx.x + 1, i1 = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (i0 >= nx1 || i1 >= ny1) return;
    const int pf = F.g.idx(i0, i1, nz1), fsz = F.g.px * F.g.py;
    const T a = AF.l[SXZ][pf];
    if (a == T(0)) return;
    AF.l[SXZ][pf] = T(0);
    AF.l[SXZ][pf - fsz] = AF.l[SXZ][pf - fsz] - a;
    const int jx = i0 / r, jy = i1 / r;
    for (int ey = 0; ey < 2; ey++)
        for (int ex = 0; ex < 2; ex++) {
            const int cx = jx + ex, cy = jy + ey;
            if (cx > nx2 || cy > ny2) continue;
            const double ww = pw_node(i0, cx, r, nx2) * pw_node(i1, cy, r, ny2);
            if (ww == 0.0) continue;
            atom(AC.l[SXZ] + C.g.idx(cx, cy, 0), (T)(ww * (double)a));
            atomicAdd(lx + (size_t)(cy - 1) * n0 + (cx - 1), ww * (double)a);
        }
}

// y = A^{-1} lambda_X (A symmetric) by Jacobi sweeps from the previous y,
// until ||y_k - y_{k-1}||_2 <= 1e-13 sum|lambda_X| or the sweep cap; one
// cooperative kernel with the bounded grid reductions of the forward solve.
__global__ void __launch_bounds__(256) sxz_adj_solve_kernel(int nx2, int ny2, SxzWork W, const double *lx)
{
    __shared__ double red[32];
    const int n0 = nx2 - 1, n1 = ny2 - 1, ld = nx2 + 1, nn = n0 * n1;
    const int gtid = blockIdx.x * blockDim.x + threadIdx.x, gstride = gridDim.x * blockDim.x;
    bool ok = true;
    int round = 0;   // grid_sum rounds (alternating halves of W.partial)
    double sab = 0.0;
    for (int q = gtid; q < nn; q += gstride) sab += fabs(lx[q]);
    const double sum = grid_sum(sab, W, red, ok, round);
    if (!(sum > 0.0)) {   // no adjoint at this interface yet: y = 0
        for (int q = gtid; q < nn; q += gstride) W.X0[(q / n0 + 1) * ld + q % n0 + 1] = 0.0;
        if (gtid == 0) *W.iters = 0;
        return;
    }
    const double tol = 1e-13 * sum;
    double *Xc = W.X0, *Xn = W.X1;
    int it = 0;
    while (ok) {
        double s = 0.0;
        for (int q = gtid; q < nn; q += gstride) {
            const int i0 = q % n0 + 1, i1 = q / n0 + 1;
            const double *a = W.A + q;
            const double xn = (lx[q]
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
        const double tot = grid_sum(s, W, red, ok, round);
        double *tmp = Xc; Xc = Xn; Xn = tmp;
        it++;
        if (!(sqrt(tot) > tol)) break;
        if (it >= W.max_iter) {
            if (gtid == 0) atomicOr(W.status, ST_JACOBI_CAP);
            break;
        }
    }
    if (Xc != W.X0)
        for (int q = gtid; q < nn; q += gstride) {
            const int i0 = q % n0 + 1, i1 = q / n0 + 1;
            W.X0[i1 * ld + i0] = __ldcg(Xc + i1 * ld + i0);
        }
    if (gtid == 0) *W.iters = it;
}

// The adjoint solves of several systems in one cooperative launch, each
// bitwise as sxz_adj_solve_kernel with its ncta CTAs (the same mapping of
// unknowns and partial sums), sharing one barrier per round; every CTA forms
// every system's totals and takes the same stopping decisions, so systems
// that have converged (or have no adjoint yet) idle at the barriers while the
// others sweep.
__global__ void __launch_bounds__(256) sxz_adj_solve_multi_kernel(const __grid_constant__ SxzAdjList L)
{
    __shared__ double red[32];
    __shared__ double s_tol[kMaxSxzSys];
    __shared__ int s_it[kMaxSxzSys], s_act[kMaxSxzSys], s_cap[kMaxSxzSys], s_zero[kMaxSxzSys];
    int me = 0;
    for (int i = 1; i < L.n; i++)
        if ((int)blockIdx.x >= L.s[i].cta0) me = i;
    const SxzAdjSys &S = L.s[me];
    const SxzWork &W = S.W;
    const double *lx = S.lx;
    const int lb = blockIdx.x - S.cta0, ncta = S.ncta;
    const int n0 = S.nx2 - 1, n1 = S.ny2 - 1, ld = S.nx2 + 1, nn = n0 * n1;
    const int gtid = lb * blockDim.x + threadIdx.x, gstride = ncta * blockDim.x;
    bool ok = true;
    int round = 0;
    auto slot = [&](const SxzAdjSys &Y, int rd, int b) { return Y.W.partial + (size_t)(rd & 1) * Y.ncta + b; };
    double sab = 0.0;
    for (int q = gtid; q < nn; q += gstride) sab += fabs(lx[q]);
    grid_arrive_list(sab, slot(S, round, lb), L.bar, L.status, red, ok);
    round++;
    for (int i = 0; i < L.n; i++) {
        const double sum = system_total(slot(L.s[i], round - 1, 0), L.s[i].ncta, red);
        if (threadIdx.x == 0) {
            s_zero[i] = !(sum > 0.0);
            s_tol[i] = 1e-13 * sum;
            s_it[i] = 0;
            s_act[i] = s_zero[i] ? 0 : 1;
            s_cap[i] = 0;
        }
    }
    __syncthreads();
    if (s_zero[me]) {   // no adjoint at this interface yet: y = 0
        for (int q = gtid; q < nn; q += gstride) W.X0[(q / n0 + 1) * ld + q % n0 + 1] = 0.0;
    }
    double *Xc = W.X0, *Xn = W.X1;
    bool any = false;
    for (int i = 0; i < L.n; i++) any = any || s_act[i] != 0;
    while (ok && any) {
        const bool mine = s_act[me] != 0;
        double s = 0.0;
        if (mine)
            for (int q = gtid; q < nn; q += gstride) {
                const int i0 = q % n0 + 1, i1 = q / n0 + 1;
                const double *a = W.A + q;
                const double xn = (lx[q]
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
        grid_arrive_list(s, slot(S, round, lb), L.bar, L.status, red, ok);
        round++;
        if (!ok) break;
        for (int i = 0; i < L.n; i++) {
            if (!s_act[i]) continue;   // uniform over the CTA
            const SxzAdjSys &Y = L.s[i];
            const double tot = system_total(slot(Y, round - 1, 0), Y.ncta, red);
            if (threadIdx.x == 0) {
                s_it[i]++;
                if (!(sqrt(tot) > s_tol[i])) s_act[i] = 0;
                else if (s_it[i] >= Y.W.max_iter) { s_act[i] = 0; s_cap[i] = 1; }
            }
        }
        __syncthreads();
        if (mine) { double *tmp = Xc; Xc = Xn; Xn = tmp; }
        any = false;
        for (int i = 0; i < L.n; i++) any = any || s_act[i] != 0;
        __syncthreads();
    }
    if (Xc != W.X0)
        for (int q = gtid; q < nn; q += gstride) {
            const int i0 = q % n0 + 1, i1 = q / n0 + 1;
            W.X0[i1 * ld + i0] = __ldcg(Xc + i1 * ld + i0);
        }
    if (gtid == 0) {
        *W.iters = s_it[me];
        if (s_cap[me]) atomicOr(W.status, ST_JACOBI_CAP);
    }
}

// rhs^T y (B = r^4 pc - r^2 fsum) and buoyancy gradients, coarse rows
template <typename T>
__global__ void sxz_adj_coarse(GridDev<T> C, AdjDev<T> AC, int r, const double *y)
{
    const int nx2 = C.g.nx, n0 = nx2 - 1, n1 = C.g.ny - 1, ld = nx2 + 1;
    const int q = blockIdx.x * blockDim.x + threadIdx.x;
    if (q >= n0 * n1) return;
    const int j0 = q % n0 + 1, j1 = q / n0 + 1;
    const double yv = y[j1 * ld + j0];
    if (yv == 0.0) return;
    const double rr = (double)r, r4 = rr * rr * rr * rr, u = r4 * yv;
    const double k2x = C.kd[0], k2y = C.kd[1], k2z = C.kd[2];
    const int pc = C.g.idx(j0, j1, 0), sy = C.g.px;
    const double b2 = (double)C.b[pc];
    const T *sxx2 = C.f[SXX], *sxy2 = C.f[SXY], *sxz2 = C.f[SXZ];
    atom(AC.l[VX] + pc, (T)u);
    atom(AC.l[SXX] + pc, (T)(u * b2 * k2x)); atom(AC.l[SXX] + pc - 1, (T)(-u * b2 * k2x));
    atom(AC.l[SXY] + pc, (T)(u * b2 * k2y)); atom(AC.l[SXY] + pc - sy, (T)(-u * b2 * k2y));
    atom(AC.l[SXZ] + pc, (T)(u * b2 * k2z));
    const double xg = (double)sxz2[C.g.idx(j0, j1, -1)];
    const double d = k2x * ((double)sxx2[pc] - (double)sxx2[pc - 1]) + k2y * ((double)sxy2[pc] - (double)sxy2[pc - sy])
                   + k2z * (double)sxz2[pc];
    atom(AC.gb + pc, (T)(u * (d - k2z * xg)));
}

// fine nodes: beta = r^2 (P y)(f) enters as -beta * pf; the fine buoyancy also
// scales A by r^2 w w' b1 k1z
template <typename T>
__global__ void sxz_adj_fine(GridDev<T> F, GridDev<T> C, AdjDev<T> AF, AdjDev<T> AC, int r, const double *y)
{
    const int nx2 = C.g.nx, ny2 = C.g.ny, ld = nx2 + 1, nz1 = F.g.nz;
    const int nx1 = r * nx2, ny1 = r * ny2;
    const int i0 = blockIdx.x * blockDim.x + threadIdx.x + 1, i1 = blockIdx.y * blockDim.y + threadIdx.y + 1;
    if (i0 >= nx1 || i1 >= ny1) return;
    const int jx = i0 / r, jy = i1 / r;
    double py = 0.0, px = 0.0, ps0 = 0.0;
    double wws[2][2];
    for (int ey = 0; ey < 2; ey++)
        for (int ex = 0; ex < 2; ex++) {
            const int cx = jx + ex, cy = jy + ey;
            double ww = 0.0;
            if (cx <= nx2 && cy <= ny2) ww = pw_node(i0, cx, r, nx2) * pw_node(i1, cy, r, ny2);
            wws[ey][ex] = ww;
            if (ww == 0.0) continue;
            py += ww * y[cy * ld + cx];
            px += ww * (double)C.f[SXZ][C.g.idx(cx, cy, -1)];
            ps0 += ww * (double)C.f[SXZ][C.g.idx(cx, cy, 0)];
        }
    const double rr = (double)r, beta = rr * rr * py;
    if (beta == 0.0) return;
    const double k1x = F.kd[0], k1y = F.kd[1], k1z = F.kd[2];
    const int pf = F.g.idx(i0, i1, nz1), fsy = F.g.px, fsz = F.g.px * F.g.py;
    const double b1 = (double)F.b[pf];
    const T *sxx1 = F.f[SXX], *sxy1 = F.f[SXY], *sxz1 = F.f[SXZ];
    atom(AF.l[VX] + pf, (T)-beta);
    atom(AF.l[SXX] + pf, (T)(-beta * b1 * k1x)); atom(AF.l[SXX] + pf - 1, (T)(beta * b1 * k1x));
    atom(AF.l[SXY] + pf, (T)(-beta * b1 * k1y)); atom(AF.l[SXY] + pf - fsy, (T)(beta * b1 * k1y));
    atom(AF.l[SXZ] + pf - fsz, (T)(2.0 * beta * b1 * k1z));
    for (int ey = 0; ey < 2; ey++)
        for (int ex = 0; ex < 2; ex++)
            if (wws[ey][ex] != 0.0) atom(AC.l[SXZ] + C.g.idx(jx + ex, jy + ey, 0), (T)(-beta * b1 * k1z * wws[ey][ex]));
    const double d = k1x * ((double)sxx1[pf] - (double)sxx1[pf - 1]) + k1y * ((double)sxy1[pf] - (double)sxy1[pf - fsy])
                   + k1z * (ps0 - 2.0 * (double)sxz1[pf - fsz]);
    atom(AF.gb + pf, (T)(-beta * (d + k1z * px)));
}

// ---------------------------------------------------------------------------
// Intuitive interpolation (imode 0, ratio 2): explicit ghosts
// (update_ghost_vz.cpp:36-123, update_ghost_sxz.cpp:37-84,
// update_ghost_syz.cpp:23-150).  One thread per fine ghost point of the
// interface plane; the thread at fine (2 j0, 2 j1) also writes the coarse
// ghost of (j0, j1).  Each op reads only fine planes nz1-2, nz1-1 and the
// coarse plane 0 and writes only the ghost planes, so the threads are
// independent.  Every formula adds its terms in the reference's order and
// with the reference's types: with T = float the T-typed terms round in float
// and the terms the reference writes with double literals (0.375 * x,
// x * 2 / 3.0) in double, as in its float build; with T = double all of it is
// double.  The file is compiled without FMA contraction.
// ---------------------------------------------------------------------------

// The element the reference's row-major Field (rows of len0 = extent + 2R)
// reads at (x, y) of a z-plane when x runs past the end of the row: the same
// linear offset, re-split into (x, y).  Identity for x inside the row.
__device__ __forceinline__ void row_major_wrap(int x, int y, int len0, int R, int &xo, int &yo)
{
    const int l = (y + R) * len0 + (x + R);
    yo = l / len0 - R;
    xo = l % len0 - R;
}

// skip_end: leave the fine ghosts of the last x column as they are (the
// revision of update_ghost_vz.cpp that produced the II golden traces)
template <typename T>
__global__ void ghost_vz_ii_kernel(GridDev<T> F, GridDev<T> C, int skip_end)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx2 = C.g.nx, ny2 = C.g.ny, nz1 = F.g.nz;
    const int nx1 = 2 * nx2, ny1 = 2 * ny2;
    if (x >= nx1 || y >= ny1) return;
    T *vz1 = F.f[VZ];
    T *vz2 = C.f[VZ];
    const int sz1 = F.g.px * F.g.py;
    const int pf = F.g.idx(x, y, nz1);
    if (!(x & 1) && !(y & 1) && y > 0) {   // coarse ghost (x/2, y/2, -1), update_ghost_vz.cpp:46-50
        const int q2 = pf - 2 * sz1, q1 = pf - sz1;
        const T s = vz1[q2] + vz1[q2 + 1] + vz1[q1] + vz1[q1 + 1];
        vz2[C.g.idx(x / 2, y / 2, -1)] = (T)(0.25 * (double)s);
    }
    if (skip_end && x == nx1 - 1) return;
    const T own = vz1[pf - sz1];
    const int j1 = y / 2, odd_y = y & 1;
    T v;
    if (x >= 1 && x <= nx1 - 2) {   // update_ghost_vz.cpp:57-81
        const int j0 = (x - 1) / 2, second = (x - 1) & 1;
        const int p0 = C.g.idx(j0, j1, 0);
        const T c00 = vz2[p0], c10 = vz2[p0 + 1];
        if (!odd_y) {
            v = second ? own / (T)3 + c00 / (T)6 + c10 / (T)2 : own / (T)3 + c00 / (T)2 + c10 / (T)6;
        } else {
            const T c01 = vz2[p0 + C.g.px], c11 = vz2[p0 + C.g.px + 1];
            v = second ? own / (T)3 + c00 / (T)12 + c10 / (T)4 + c01 / (T)12 + c11 / (T)4
                       : own / (T)3 + c00 / (T)4 + c10 / (T)12 + c01 / (T)4 + c11 / (T)12;
        }
    } else {   // x = 0 or nx1-1: update_ghost_vz.cpp:87-110
        const int xin = (x == 0) ? 1 : x - 1;
        // the coarse x index is the fine x (nx1-1 at the far column): read where the
        // reference's layout puts it (rows of nx2 + 2R elements for vz)
        int cx0, cy0, cx1, cy1;
        row_major_wrap(x, j1, nx2 + 2 * C.g.R, C.g.R, cx0, cy0);
        row_major_wrap(x, j1 + 1, nx2 + 2 * C.g.R, C.g.R, cx1, cy1);
        const T ca = vz2[C.g.idx(cx0, cy0, 0)];
        if (!odd_y) {
            v = own * (T)2 / (T)3 - vz1[F.g.idx(xin, y, nz1 - 1)] / (T)3 + ca * (T)2 / (T)3;
        } else {
            const T cb = vz2[C.g.idx(cx1, cy1, 0)];
            v = own * (T)2 / (T)3 - vz1[F.g.idx(xin, y - 1, nz1 - 1)] / (T)3 + ca / (T)3 + cb / (T)3;
        }
    }
    vz1[pf] = v;
}

template <typename T>
__global__ void ghost_sxz_ii_kernel(GridDev<T> F, GridDev<T> C)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int y = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int nx2 = C.g.nx, ny2 = C.g.ny, nz1 = F.g.nz;
    if (x >= 2 * nx2 || y >= 2 * ny2) return;
    T *sxz1 = F.f[SXZ];
    T *sxz2 = C.f[SXZ];
    const int sz1 = F.g.px * F.g.py;
    const int pf = F.g.idx(x, y, nz1);
    const int j0 = x / 2, j1 = y / 2;
    const int p0 = C.g.idx(j0, j1, 0), sy2 = C.g.px;
    if (!(x & 1) && !(y & 1))   // update_ghost_sxz.cpp:46-49
        sxz2[p0 - C.g.px * C.g.py] = (T)(0.5 * (double)(sxz1[pf - 2 * sz1] + sxz1[pf - sz1]));
    const T own = sxz1[pf - sz1];
    T v;
    switch ((x & 1) | ((y & 1) << 1)) {   // update_ghost_sxz.cpp:55-81
    case 0: v = (T)((double)(own / (T)3) + (double)(sxz2[p0] * (T)2) / 3.0); break;
    case 1: v = own / (T)3 + sxz2[p0] / (T)3 + sxz2[p0 + 1] / (T)3; break;
    case 2: v = own / (T)3 + sxz2[p0] / (T)3 + sxz2[p0 + sy2] / (T)3; break;
    default:
        v = own / (T)3 + sxz2[p0] / (T)6 + sxz2[p0 + sy2] / (T)6 + sxz2[p0 + 1] / (T)6 + sxz2[p0 + sy2 + 1] / (T)6;
    }
    sxz1[pf] = v;
}

template <typename T>
__global__ void ghost_syz_ii_kernel(GridDev<T> F, GridDev<T> C)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx2 = C.g.nx, ny2 = C.g.ny, nz1 = F.g.nz;
    const int X1 = 2 * nx2 - 1, Y1 = 2 * ny2 - 1;
    if (x > X1 || y > Y1) return;
    T *syz1 = F.f[SYZ];
    T *syz2 = C.f[SYZ];
    const int sy1 = F.g.px, sz1 = F.g.px * F.g.py, sy2 = C.g.px;
    const int pf = F.g.idx(x, y, nz1);
    if (!(x & 1) && !(y & 1)) {   // coarse ghost, update_ghost_syz.cpp:33-42
        const int q2 = pf - 2 * sz1, q1 = pf - sz1;
        const T s = syz1[q2] + syz1[q2 + 1] + syz1[q2 + sy1] + syz1[q2 + sy1 + 1]
                  + syz1[q1] + syz1[q1 + 1] + syz1[q1 + sy1] + syz1[q1 + sy1 + 1];
        syz2[C.g.idx(x / 2, y / 2, -1)] = (T)(0.125 * (double)s);
    }
    const int pb = pf - sz1;   // the fine plane below
    const T own = syz1[pb];
    T v;
    if (x >= 1 && x <= X1 - 1 && y >= 1 && y <= Y1 - 1) {   // update_ghost_syz.cpp:49-74
        const int j0 = (x - 1) / 2, j1 = (y - 1) / 2;
        const int nr = ((x - 1) & 1) | (((y - 1) & 1) << 1);   // coarse corner nearest (x, y)
        const int p0 = C.g.idx(j0, j1, 0);
        const T c[4] = {syz2[p0], syz2[p0 + 1], syz2[p0 + sy2], syz2[p0 + sy2 + 1]};
        // the far corner's term is x/24 (type T) and the near and adjacent ones
        // are 0.375*x and 0.125*x (double); the sum starts in T only when the
        // second term is the far corner's (fine point (2 j0 + 2, 2 j1 + 2))
        double acc = nr == 3 ? (double)(own / (T)3 + c[0] / (T)24)
                             : (double)(own / (T)3) + (nr == 0 ? 0.375 : 0.125) * (double)c[0];
#pragma unroll
        for (int k = 1; k < 4; k++) {
            const int d = k ^ nr;
            acc = acc + (d == 3 ? (double)(c[k] / (T)24) : (d == 0 ? 0.375 * (double)c[k] : 0.125 * (double)c[k]));
        }
        v = (T)acc;
    } else {   // edges, update_ghost_syz.cpp:78-134
        const T cc = syz2[C.g.idx(x / 2, y / 2, 0)] * (T)2 / (T)3;
        if (y == 0 || y == Y1) {
            const int yin = (y == 0) ? 1 : Y1 - 1;
            const T in_y = syz1[F.g.idx(x, yin, nz1 - 1)];
            if (x == 0 || x == X1) {
                const int xin = (x == 0) ? 1 : X1 - 1;
                v = own - syz1[F.g.idx(xin, y, nz1 - 1)] / (T)3 - in_y / (T)3 + cc;
            } else {
                v = own / (T)3 + syz1[F.g.idx(x - 1 + 2 * (x & 1), y, nz1 - 1)] / (T)3 - in_y / (T)3 + cc;
            }
        } else {
            const int xin = (x == 0) ? 1 : X1 - 1;
            v = own / (T)3 + syz1[F.g.idx(x, y - 1 + 2 * (y & 1), nz1 - 1)] / (T)3
              - syz1[F.g.idx(xin, y, nz1 - 1)] / (T)3 + cc;
        }
    }
    syz1[pf] = v;
}

// Transposes of the three imode-0 maps.  Each ghost value is overwritten from
// values of other planes, so its adjoint is read, cleared and spread onto
// those values with the forward weights; the sources are never ghosts, so one
// launch with atomic adds is race free.  The thread layout is the forward's.
template <typename T>
__global__ void ghost_vz_ii_adj_kernel(GridDev<T> F, GridDev<T> C, AdjDev<T> AF, AdjDev<T> AC, int skip_end)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx2 = C.g.nx, ny2 = C.g.ny, nz1 = F.g.nz;
    const int nx1 = 2 * nx2, ny1 = 2 * ny2;
    if (x >= nx1 || y >= ny1) return;
    T *l1 = AF.l[VZ], *l2 = AC.l[VZ];
    const int sz1 = F.g.px * F.g.py;
    const int pf = F.g.idx(x, y, nz1);
    if (!(x & 1) && !(y & 1) && y > 0) {
        const int pg = C.g.idx(x / 2, y / 2, -1);
        const T a = (T)(0.25 * (double)l2[pg]);
        l2[pg] = (T)0;
        const int q2 = pf - 2 * sz1, q1 = pf - sz1;
        atom(l1 + q2, a); atom(l1 + q2 + 1, a); atom(l1 + q1, a); atom(l1 + q1 + 1, a);
    }
    if (skip_end && x == nx1 - 1) return;   // identity there
    const T a = l1[pf];
    l1[pf] = (T)0;
    const int j1 = y / 2, odd_y = y & 1;
    if (x >= 1 && x <= nx1 - 2) {
        const int j0 = (x - 1) / 2, second = (x - 1) & 1;
        const int p0 = C.g.idx(j0, j1, 0);
        atom(l1 + pf - sz1, a / (T)3);
        if (!odd_y) {
            atom(l2 + p0, a / (T)(second ? 6 : 2));
            atom(l2 + p0 + 1, a / (T)(second ? 2 : 6));
        } else {
            const T wn = a / (T)4, wf = a / (T)12;
            atom(l2 + p0, second ? wf : wn);
            atom(l2 + p0 + 1, second ? wn : wf);
            atom(l2 + p0 + C.g.px, second ? wf : wn);
            atom(l2 + p0 + C.g.px + 1, second ? wn : wf);
        }
    } else {
        const int xin = (x == 0) ? 1 : x - 1;
        int cx0, cy0, cx1, cy1;
        row_major_wrap(x, j1, nx2 + 2 * C.g.R, C.g.R, cx0, cy0);
        row_major_wrap(x, j1 + 1, nx2 + 2 * C.g.R, C.g.R, cx1, cy1);
        atom(l1 + pf - sz1, a * (T)2 / (T)3);
        atom(l1 + F.g.idx(xin, odd_y ? y - 1 : y, nz1 - 1), -a / (T)3);
        if (!odd_y) {
            atom(l2 + C.g.idx(cx0, cy0, 0), a * (T)2 / (T)3);
        } else {
            atom(l2 + C.g.idx(cx0, cy0, 0), a / (T)3);
            atom(l2 + C.g.idx(cx1, cy1, 0), a / (T)3);
        }
    }
}

template <typename T>
__global__ void ghost_sxz_ii_adj_kernel(GridDev<T> F, GridDev<T> C, AdjDev<T> AF, AdjDev<T> AC)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x + 1;
    const int y = blockIdx.y * blockDim.y + threadIdx.y + 1;
    const int nx2 = C.g.nx, ny2 = C.g.ny, nz1 = F.g.nz;
    if (x >= 2 * nx2 || y >= 2 * ny2) return;
    T *l1 = AF.l[SXZ], *l2 = AC.l[SXZ];
    const int sz1 = F.g.px * F.g.py;
    const int pf = F.g.idx(x, y, nz1);
    const int p0 = C.g.idx(x / 2, y / 2, 0), sy2 = C.g.px;
    if (!(x & 1) && !(y & 1)) {
        const int pg = p0 - C.g.px * C.g.py;
        const T b = (T)(0.5 * (double)l2[pg]);
        l2[pg] = (T)0;
        atom(l1 + pf - 2 * sz1, b);
        atom(l1 + pf - sz1, b);
    }
    const T a = l1[pf];
    l1[pf] = (T)0;
    atom(l1 + pf - sz1, a / (T)3);
    switch ((x & 1) | ((y & 1) << 1)) {
    case 0: atom(l2 + p0, (T)((double)a * 2.0 / 3.0)); break;
    case 1: atom(l2 + p0, a / (T)3); atom(l2 + p0 + 1, a / (T)3); break;
    case 2: atom(l2 + p0, a / (T)3); atom(l2 + p0 + sy2, a / (T)3); break;
    default: {
        const T w = a / (T)6;
        atom(l2 + p0, w); atom(l2 + p0 + sy2, w); atom(l2 + p0 + 1, w); atom(l2 + p0 + sy2 + 1, w);
    }
    }
}

template <typename T>
__global__ void ghost_syz_ii_adj_kernel(GridDev<T> F, GridDev<T> C, AdjDev<T> AF, AdjDev<T> AC)
{
    const int x = blockIdx.x * blockDim.x + threadIdx.x;
    const int y = blockIdx.y * blockDim.y + threadIdx.y;
    const int nx2 = C.g.nx, ny2 = C.g.ny, nz1 = F.g.nz;
    const int X1 = 2 * nx2 - 1, Y1 = 2 * ny2 - 1;
    if (x > X1 || y > Y1) return;
    T *l1 = AF.l[SYZ], *l2 = AC.l[SYZ];
    const int sy1 = F.g.px, sz1 = F.g.px * F.g.py, sy2 = C.g.px;
    const int pf = F.g.idx(x, y, nz1);
    if (!(x & 1) && !(y & 1)) {
        const int pg = C.g.idx(x / 2, y / 2, -1);
        const T b = (T)(0.125 * (double)l2[pg]);
        l2[pg] = (T)0;
        for (int q = pf - 2 * sz1; q <= pf - sz1; q += sz1) {
            atom(l1 + q, b); atom(l1 + q + 1, b); atom(l1 + q + sy1, b); atom(l1 + q + sy1 + 1, b);
        }
    }
    const T a = l1[pf];
    l1[pf] = (T)0;
    const int pb = pf - sz1;
    if (x >= 1 && x <= X1 - 1 && y >= 1 && y <= Y1 - 1) {
        atom(l1 + pb, a / (T)3);
        const int nr = ((x - 1) & 1) | (((y - 1) & 1) << 1);
        const int p0 = C.g.idx((x - 1) / 2, (y - 1) / 2, 0);
        const int pc[4] = {p0, p0 + 1, p0 + sy2, p0 + sy2 + 1};
#pragma unroll
        for (int k = 0; k < 4; k++) {
            const int d = k ^ nr;
            atom(l2 + pc[k], d == 3 ? a / (T)24 : (d == 0 ? (T)(0.375 * (double)a) : (T)(0.125 * (double)a)));
        }
    } else {
        atom(l2 + C.g.idx(x / 2, y / 2, 0), a * (T)2 / (T)3);
        if (y == 0 || y == Y1) {
            const int yin = (y == 0) ? 1 : Y1 - 1;
            atom(l1 + F.g.idx(x, yin, nz1 - 1), -a / (T)3);
            if (x == 0 || x == X1) {
                atom(l1 + pb, a);
                atom(l1 + F.g.idx((x == 0) ? 1 : X1 - 1, y, nz1 - 1), -a / (T)3);
            } else {
                atom(l1 + pb, a / (T)3);
                atom(l1 + F.g.idx(x - 1 + 2 * (x & 1), y, nz1 - 1), a / (T)3);
            }
        } else {
            atom(l1 + pb, a / (T)3);
            atom(l1 + F.g.idx(x, y - 1 + 2 * (y & 1), nz1 - 1), a / (T)3);
            atom(l1 + F.g.idx((x == 0) ? 1 : X1 - 1, y, nz1 - 1), -a / (T)3);
        }
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

// imode 0 (ratio 2): one launch per op over the fine interface plane;
// op 0 vz, 1 sxz, 2 syz, 3 vz with the last fine x column left as it is
template <typename T>
cudaError_t launch_ghost_ii(int op, const GridDev<T> &F, const GridDev<T> &C, cudaStream_t st)
{
    const int nx1 = 2 * C.g.nx, ny1 = 2 * C.g.ny;
    dim3 b(64, 4);
    switch (op) {
    case 0:
    case 3: ghost_vz_ii_kernel<T><<<dim3((nx1 + 63) / 64, (ny1 + 3) / 4), b, 0, st>>>(F, C, op == 3); break;
    case 1: ghost_sxz_ii_kernel<T><<<dim3((nx1 - 1 + 63) / 64, (ny1 - 1 + 3) / 4), b, 0, st>>>(F, C); break;
    case 2: ghost_syz_ii_kernel<T><<<dim3((nx1 + 63) / 64, (ny1 + 3) / 4), b, 0, st>>>(F, C); break;
    default: return cudaErrorInvalidValue;
    }
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_ghost_ii_adj(int op, const GridDev<T> &F, const GridDev<T> &C, const AdjDev<T> &AF,
                                const AdjDev<T> &AC, cudaStream_t st)
{
    const int nx1 = 2 * C.g.nx, ny1 = 2 * C.g.ny;
    dim3 b(64, 4);
    switch (op) {
    case 0:
    case 3: ghost_vz_ii_adj_kernel<T><<<dim3((nx1 + 63) / 64, (ny1 + 3) / 4), b, 0, st>>>(F, C, AF, AC, op == 3); break;
    case 1: ghost_sxz_ii_adj_kernel<T><<<dim3((nx1 - 1 + 63) / 64, (ny1 - 1 + 3) / 4), b, 0, st>>>(F, C, AF, AC); break;
    case 2: ghost_syz_ii_adj_kernel<T><<<dim3((nx1 + 63) / 64, (ny1 + 3) / 4), b, 0, st>>>(F, C, AF, AC); break;
    default: return cudaErrorInvalidValue;
    }
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
    // the fewest resident CTAs per SM of the three instantiations (any ratio)
    int per_sm = 0, p2 = 0, p3 = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sxz_solve_kernel<T, 0>, 256, 0) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&p2, sxz_solve_kernel<T, 2>, 256, 0) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&p3, sxz_solve_kernel<T, 3>, 256, 0) != cudaSuccess)
        per_sm = 1;
    per_sm = per_sm < p2 ? per_sm : p2;
    per_sm = per_sm < p3 ? per_sm : p3;
    if (per_sm < 1) per_sm = 1;
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
    if (r == 2) return cudaLaunchKernelEx(&cfg, sxz_solve_kernel<T, 2>, F, C, r, W);
    if (r == 3) return cudaLaunchKernelEx(&cfg, sxz_solve_kernel<T, 3>, F, C, r, W);
    return cudaLaunchKernelEx(&cfg, sxz_solve_kernel<T, 0>, F, C, r, W);
}

// CTAs of one multi-system launch that can be co-resident (the fewest per SM
// of the three instantiations)
template <typename T>
int sxz_multi_capacity(int sms)
{
    int p0 = 0, p2 = 0, p3 = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&p0, sxz_solve_multi_kernel<T, 0>, 256, 0) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&p2, sxz_solve_multi_kernel<T, 2>, 256, 0) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&p3, sxz_solve_multi_kernel<T, 3>, 256, 0) != cudaSuccess)
        return 0;
    int per_sm = p0 < p2 ? p0 : p2;
    per_sm = per_sm < p3 ? per_sm : p3;
    return per_sm * sms;
}

// L.s[i].cta0 / ncta set by the caller (consecutive, from 0); the barrier words
// L.bar start at zero and are left at zero count.
template <typename T>
cudaError_t launch_sxz_solve_multi(const SxzSysList<T> &L, cudaStream_t st)
{
    if (L.n < 1 || L.n > kMaxSxzSys) return cudaErrorInvalidValue;
    const int nblocks = L.s[L.n - 1].cta0 + L.s[L.n - 1].ncta;
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
    if (L.r == 2) return cudaLaunchKernelEx(&cfg, sxz_solve_multi_kernel<T, 2>, L);
    if (L.r == 3) return cudaLaunchKernelEx(&cfg, sxz_solve_multi_kernel<T, 3>, L);
    return cudaLaunchKernelEx(&cfg, sxz_solve_multi_kernel<T, 0>, L);
}


template <typename T>
cudaError_t launch_ghost_vz_adj(const GridDev<T> &F, const GridDev<T> &C, const AdjDev<T> &AF, const AdjDev<T> &AC,
                                int r, double *coef, double *lx, double *y, cudaStream_t st)
{
    const int m = C.g.ny - 1, nx2 = C.g.nx;
    int P = 32;
    while (P < m) P <<= 1;
    if (P > 1024) return cudaErrorInvalidConfiguration;
    dim3 ba(32, 8), ga((nx2 + 31) / 32, (m + 7) / 8);
    ghost_vz_assemble_kernel<T><<<ga, ba, 0, st>>>(F, C, MED_GEN21, r, coef);
    vz_adj_collect_coarse<T><<<ga, ba, 0, st>>>(C, AC, lx);
    const int nx1 = r * nx2, ny1 = r * C.g.ny;
    dim3 bf(64, 4), gf((nx1 + 63) / 64, (ny1 - 1 + 3) / 4);
    vz_adj_collect_fine<T><<<gf, bf, 0, st>>>(F, C, AF, AC, r, lx);
    vz_adj_solve_kernel<<<nx2, P, sizeof(double) * 4 * P, st>>>(nx2, m, coef, lx, y);
    vz_adj_coarse<T><<<ga, ba, 0, st>>>(C, AC, r, y);
    vz_adj_fine<T><<<gf, bf, 0, st>>>(F, C, AF, AC, r, y);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_ghost_syz_adj(const GridDev<T> &F, const GridDev<T> &C, const AdjDev<T> &AF, const AdjDev<T> &AC,
                                 int r, cudaStream_t st)
{
    dim3 blk(32, 8), grd((C.g.nx + 31) / 32, (C.g.ny + 7) / 8);
    syz_adj_kernel<T><<<grd, blk, 0, st>>>(F, C, AF, AC, r);
    return cudaGetLastError();
}

// W: the interface's sxz work space (A from sxz_matrix, X0/X1 hold the
// adjoint's warm start y); lx: (nx2-1)(ny2-1) doubles
template <typename T>
cudaError_t launch_ghost_sxz_adj(const GridDev<T> &F, const GridDev<T> &C, const AdjDev<T> &AF, const AdjDev<T> &AC,
                                 int r, const SxzWork &W, int nblocks, double *lx, cudaStream_t st)
{
    const int nx2 = C.g.nx, ny2 = C.g.ny, nn = (nx2 - 1) * (ny2 - 1);
    const int nx1 = r * nx2, ny1 = r * ny2;
    sxz_adj_collect_coarse<T><<<(nn + 255) / 256, 256, 0, st>>>(C, AC, lx);
    dim3 bf(64, 4), gf((nx1 - 1 + 63) / 64, (ny1 - 1 + 3) / 4);
    sxz_adj_collect_fine<T><<<gf, bf, 0, st>>>(F, C, AF, AC, r, lx);
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(nblocks);
    cfg.blockDim = dim3(256);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    cudaError_t e = cudaLaunchKernelEx(&cfg, sxz_adj_solve_kernel, nx2, ny2, W, (const double *)lx);
    if (e != cudaSuccess) return e;
    sxz_adj_coarse<T><<<(nn + 255) / 256, 256, 0, st>>>(C, AC, r, W.X0);
    sxz_adj_fine<T><<<gf, bf, 0, st>>>(F, C, AF, AC, r, W.X0);
    return cudaGetLastError();
}

// The adjoint sxz solve in three parts, for solving several systems in one
// launch: collect lambda_X (and zero the ghosts) ...
template <typename T>
cudaError_t launch_sxz_adj_collect(const GridDev<T> &F, const GridDev<T> &C, const AdjDev<T> &AF, const AdjDev<T> &AC,
                                   int r, double *lx, cudaStream_t st)
{
    const int nx2 = C.g.nx, ny2 = C.g.ny, nn = (nx2 - 1) * (ny2 - 1);
    const int nx1 = r * nx2, ny1 = r * ny2;
    sxz_adj_collect_coarse<T><<<(nn + 255) / 256, 256, 0, st>>>(C, AC, lx);
    dim3 bf(64, 4), gf((nx1 - 1 + 63) / 64, (ny1 - 1 + 3) / 4);
    sxz_adj_collect_fine<T><<<gf, bf, 0, st>>>(F, C, AF, AC, r, lx);
    return cudaGetLastError();
}

// ... solve the systems of a list (cta0 / ncta set by the caller) ...
cudaError_t launch_sxz_adj_solve_multi(const SxzAdjList &L, cudaStream_t st)
{
    if (L.n < 1 || L.n > kMaxSxzSys) return cudaErrorInvalidValue;
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(L.s[L.n - 1].cta0 + L.s[L.n - 1].ncta);
    cfg.blockDim = dim3(256);
    cfg.stream = st;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeCooperative;
    attr[0].val.cooperative = 1;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    return cudaLaunchKernelEx(&cfg, sxz_adj_solve_multi_kernel, L);
}

int sxz_adj_multi_capacity(int sms)
{
    int per_sm = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, sxz_adj_solve_multi_kernel, 256, 0) != cudaSuccess) return 0;
    return per_sm * sms;
}

// ... and add rhs^T y and the buoyancy gradients
template <typename T>
cudaError_t launch_sxz_adj_scatter(const GridDev<T> &F, const GridDev<T> &C, const AdjDev<T> &AF, const AdjDev<T> &AC,
                                   int r, const double *y, cudaStream_t st)
{
    const int nx2 = C.g.nx, ny2 = C.g.ny, nn = (nx2 - 1) * (ny2 - 1);
    const int nx1 = r * nx2, ny1 = r * ny2;
    dim3 bf(64, 4), gf((nx1 - 1 + 63) / 64, (ny1 - 1 + 3) / 4);
    sxz_adj_coarse<T><<<(nn + 255) / 256, 256, 0, st>>>(C, AC, r, y);
    sxz_adj_fine<T><<<gf, bf, 0, st>>>(F, C, AF, AC, r, y);
    return cudaGetLastError();
}

#define INST(T)                                                                                         \
    template cudaError_t launch_ghost_vz_adj<T>(const GridDev<T> &, const GridDev<T> &, const AdjDev<T> &,         \
                                                const AdjDev<T> &, int, double *, double *, double *, cudaStream_t); \
    template cudaError_t launch_ghost_syz_adj<T>(const GridDev<T> &, const GridDev<T> &, const AdjDev<T> &,        \
                                                 const AdjDev<T> &, int, cudaStream_t);                           \
    template cudaError_t launch_ghost_sxz_adj<T>(const GridDev<T> &, const GridDev<T> &, const AdjDev<T> &,        \
                                                 const AdjDev<T> &, int, const SxzWork &, int, double *,        \
                                                 cudaStream_t);                                                   \
    template cudaError_t launch_ghost_vz<T>(const GridDev<T> &, const GridDev<T> &, int, int, double *, cudaStream_t); \
    template cudaError_t launch_ghost_syz<T>(const GridDev<T> &, const GridDev<T> &, int, cudaStream_t);     \
    template cudaError_t launch_ghost_ii<T>(int, const GridDev<T> &, const GridDev<T> &, cudaStream_t);     \
    template cudaError_t launch_ghost_ii_adj<T>(int, const GridDev<T> &, const GridDev<T> &, const AdjDev<T> &,   \
                                                const AdjDev<T> &, cudaStream_t);                               \
    template cudaError_t launch_sxz_matrix<T>(const GridDev<T> &, const GridDev<T> &, int, double *, cudaStream_t); \
    template int sxz_solve_blocks<T>(int, int);                                                          \
    template cudaError_t launch_sxz_solve<T>(const GridDev<T> &, const GridDev<T> &, int, const SxzWork &, int, cudaStream_t); \
    template int sxz_multi_capacity<T>(int);                                                              \
    template cudaError_t launch_sxz_adj_collect<T>(const GridDev<T> &, const GridDev<T> &, const AdjDev<T> &,     \
                                                   const AdjDev<T> &, int, double *, cudaStream_t);            \
    template cudaError_t launch_sxz_adj_scatter<T>(const GridDev<T> &, const GridDev<T> &, const AdjDev<T> &,     \
                                                   const AdjDev<T> &, int, const double *, cudaStream_t);                                                              \
    template cudaError_t launch_sxz_solve_multi<T>(const SxzSysList<T> &, cudaStream_t);
INST(float)
INST(double)
#undef INST

} // namespace ecsg
