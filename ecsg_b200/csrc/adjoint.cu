// adjoint.cu -- transposes of the grid operators for misfit gradients.
//
// No reference counterpart.  Every forward operator of the time loop is an
// affine map of the full state (all box entries of the 9 fields, halos and
// ghosts included) whose linear part depends on the medium.  For an operator
// s_out = Op_m(s_in) these kernels apply, given the adjoint lambda of s_out,
//   lambda_in = Op^T lambda_out                  (in place on lambda), and
//   g_m      += d<lambda_out, Op_m(s_in)>/dm     (gradient accumulators),
// reading the forward fields the operator used.  They are written as reverse
// mode of the forward code, term for term; the operator order is reversed by
// the caller.
//
// Operators here (one grid each):
//   velocity update (update_vel.cpp:20-69 ranges, radius 1) and its odd halo
//   mirrors, receiver sampling (main.cpp:182-184), and the 21-Cij stress
//   update of stress21.cu including the free-surface condensation and the
//   surface mirrors of syz/sxz.  The interface solves are in interface.cu.
//
// Adjoint state of a grid: lambda of the 9 fields in the grid's box layout;
// gradients: g_b at the nodes (buoyancy) and g_c[21] at the slot positions.
// The grid operators are gathers (each adjoint value written by one thread)
// except the buoyancy gradient of the velocity update (the 4-node means of vy
// and vz: atomics) and the free-surface plane.  Multi-shot variants (*_shots)
// run the shots of a point in one thread where the shots add to a common
// gradient, so that gradient and the medium are read once for all of them.
// Work boxes of the stress adjoint: see the stage description below.
#include "adjoint.cuh"
#include "gen21_device.cuh"

namespace ecsg {

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

// The point kernels below run one thread per point on a 3-D launch: 256
// threads cover a 32 x 8 (x, y) tile, blockIdx.z the plane (no index
// division).
__device__ __forceinline__ void tile_xy(int &x, int &y)
{
    x = (int)blockIdx.x * 32 + (int)(threadIdx.x & 31);
    y = (int)blockIdx.y * 8 + (int)(threadIdx.x >> 5);
}
static inline dim3 grid3(int nx, int ny, int nz) { return dim3((unsigned)(nx + 31) / 32, (unsigned)(ny + 7) / 8, (unsigned)nz); }

// A load through the read-only path, for data that no thread of the kernel
// writes: the compiler may then issue it ahead of the kernel's stores (which
// it must otherwise assume could alias it), so the loads of consecutive
// position blocks and shots overlap.
template <typename T>
__device__ __forceinline__ T ro(const T *a, int i)
{
    return __ldg(a + i);
}

// ro() when RO, else an ordinary load (the plain velocity adjoint measured
// faster with ordinary loads, the multi-shot one with read-only loads)
template <bool RO, typename T>
__device__ __forceinline__ T ld_(const T *a, int i)
{
    if constexpr (RO)
        return ro(a, i);
    else
        return a[i];
}

// a point in [2, n - 3] in every dimension: every neighbour range test of the
// velocity and G1 adjoints holds there
__device__ __forceinline__ bool inner_pt(const Geo &g, int x, int y, int z)
{
    return x >= 2 && x <= g.nx - 3 && y >= 2 && y <= g.ny - 3 && z >= 2 && z <= g.nz - 3;
}

// Multi-shot point kernels run the shots of a point in turn in one thread when
// the shots add to a common gradient (G1, the velocity adjoint: the terms are
// summed in registers in shot order and the gradient is read and written
// once), or put the shots of a tile in adjacent CTAs when they do not (G0:
// the medium planes are then shared through L2).

// ---------------------------------------------------------------------------
// Velocity update: v += b * (k . D sigma) on the forward ranges.
// lambda_sigma += (b D)^T lambda_v; g_b += lambda_v * (k . D sigma), the vy
// and vz buoyancies being 4-node means (1/4 to each node).
// ---------------------------------------------------------------------------
// As gathers: the stress adjoints at q collect the transposed differences of
// the velocity points that read them, u = lambda_v * (the buoyancy mean of
// that velocity), zero outside each velocity's update range (the scatter
//   vx: lsxx[p] += k0 u, lsxx[p-1] -= k0 u, lsxy[p] += k1 u, lsxy[p-sy] -= k1 u,
//       lsxz[p] += k2 u, lsxz[p-sz] -= k2 u;
//   vy: lsxy[p+1] += k0 u, lsxy[p] -= k0 u, lsyz[p] += k2 u, lsyz[p-sz] -= k2 u,
//       lsyy[p+sy] += k1 u, lsyy[p] -= k1 u;
//   vz: lsxz[p+1] += k0 u, lsxz[p] -= k0 u, lszz[p+sz] += k2 u, lszz[p] -= k2 u,
//       lsyz[p] += k1 u, lsyz[p-sy] -= k1 u
// read backwards), so no atomics and a fixed order.  The buoyancy-gradient
// terms of the velocity point q are returned in gx (vx, node q) and gy, gz
// (vy, vz: a quarter to each of the four nodes of the mean).  IN: the point
// lies in [2, n - 3] in every dimension, where every range test below holds
// (the same arithmetic without the tests).
template <typename T, bool IN, bool RO>
__device__ __forceinline__ void vel_adj_point(const GridDev<T> &G, const T *const lv[3], const T *const *f, T *const *ls,
                                              int zt, int bottom, int x, int y, int z, T &gx, T &gy, T &gz)
{
    const Geo &g = G.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int sy = g.px, sz = g.px * g.py;
    const T k0 = G.k[0], k1 = G.k[1], k2 = G.k[2], qq = T(0.25);
    const T *b = G.b;
    const int p = g.idx(x, y, z);
    auto zin = [&](int zz) { return zz >= zt && zz <= nz - bottom; };
    auto rx = [&](int xx, int yy, int zz) { return IN || (xx >= 1 && xx <= nx - 1 && yy >= 1 && yy <= ny - 1 && zin(zz)); };
    auto ry = [&](int xx, int yy, int zz) { return IN || (xx >= 0 && xx <= nx - 1 && yy >= 0 && yy <= ny - 1 && zin(zz)); };
    auto rz = [&](int xx, int yy, int zz) {
        return IN || (xx >= 0 && xx <= nx - 1 && yy >= 1 && yy <= ny - 1 && zz >= 0 && zz <= nz - 1);
    };
    auto ux = [&](int xx, int yy, int zz) -> T {
        if (!rx(xx, yy, zz)) return T(0);
        const int i = p + (xx - x) + (yy - y) * sy + (zz - z) * sz;
        return mul_(ld_<RO>(lv[0], i), ld_<RO>(b, i));
    };
    auto uy = [&](int xx, int yy, int zz) -> T {
        if (!ry(xx, yy, zz)) return T(0);
        const int i = p + (xx - x) + (yy - y) * sy + (zz - z) * sz;
        return mul_(ld_<RO>(lv[1], i), mul_(qq, add_(add_(add_(ld_<RO>(b, i), ld_<RO>(b, i + 1)), ld_<RO>(b, i + sy)), ld_<RO>(b, i + sy + 1))));
    };
    auto uz = [&](int xx, int yy, int zz) -> T {
        if (!rz(xx, yy, zz)) return T(0);
        const int i = p + (xx - x) + (yy - y) * sy + (zz - z) * sz;
        return mul_(ld_<RO>(lv[2], i), mul_(qq, add_(add_(add_(ld_<RO>(b, i), ld_<RO>(b, i + sz)), ld_<RO>(b, i + 1)), ld_<RO>(b, i + sz + 1))));
    };
    const T ux0 = ux(x, y, z), uy0 = uy(x, y, z), uz0 = uz(x, y, z);
    const T dsxx = mul_(k0, sub_(ux0, ux(x + 1, y, z)));
    const T dsxy = add_(mul_(k1, sub_(ux0, ux(x, y + 1, z))), mul_(k0, sub_(uy(x - 1, y, z), uy0)));
    const T dsxz = add_(mul_(k2, sub_(ux0, ux(x, y, z + 1))), mul_(k0, sub_(uz(x - 1, y, z), uz0)));
    const T dsyy = mul_(k1, sub_(uy(x, y - 1, z), uy0));
    const T dsyz = add_(mul_(k2, sub_(uy0, uy(x, y, z + 1))), mul_(k1, sub_(uz0, uz(x, y + 1, z))));
    const T dszz = mul_(k2, sub_(uz(x, y, z - 1), uz0));
    // buoyancy-gradient terms of the velocity point p (its own update ranges)
    gx = T(0);
    gy = T(0);
    gz = T(0);
    if (rx(x, y, z)) {
        const T a = ld_<RO>(lv[0], p);
        const T d = add_(add_(mul_(k0, sub_(ld_<RO>(f[SXX], p), ld_<RO>(f[SXX], p - 1))), mul_(k1, sub_(ld_<RO>(f[SXY], p), ld_<RO>(f[SXY], p - sy)))),
                         mul_(k2, sub_(ld_<RO>(f[SXZ], p), ld_<RO>(f[SXZ], p - sz))));
        gx = mul_(a, d);
    }
    if (ry(x, y, z)) {
        const T a = ld_<RO>(lv[1], p);
        const T d = add_(add_(mul_(k0, sub_(ld_<RO>(f[SXY], p + 1), ld_<RO>(f[SXY], p))), mul_(k2, sub_(ld_<RO>(f[SYZ], p), ld_<RO>(f[SYZ], p - sz)))),
                         mul_(k1, sub_(ld_<RO>(f[SYY], p + sy), ld_<RO>(f[SYY], p))));
        gy = mul_(qq, mul_(a, d));
    }
    if (rz(x, y, z)) {
        const T a = ld_<RO>(lv[2], p);
        const T d = add_(add_(mul_(k0, sub_(ld_<RO>(f[SXZ], p + 1), ld_<RO>(f[SXZ], p))), mul_(k2, sub_(ld_<RO>(f[SZZ], p + sz), ld_<RO>(f[SZZ], p)))),
                         mul_(k1, sub_(ld_<RO>(f[SYZ], p), ld_<RO>(f[SYZ], p - sy))));
        gz = mul_(qq, mul_(a, d));
    }
    // every load above before the stores
    if (dsxx != T(0)) ls[SXX][p] = add_(ls[SXX][p], dsxx);
    if (dsxy != T(0)) ls[SXY][p] = add_(ls[SXY][p], dsxy);
    if (dsxz != T(0)) ls[SXZ][p] = add_(ls[SXZ][p], dsxz);
    if (dsyy != T(0)) ls[SYY][p] = add_(ls[SYY][p], dsyy);
    if (dsyz != T(0)) ls[SYZ][p] = add_(ls[SYZ][p], dsyz);
    if (dszz != T(0)) ls[SZZ][p] = add_(ls[SZZ][p], dszz);
}

// the buoyancy-gradient terms of velocity point p into the node gradient
template <typename T>
__device__ __forceinline__ void vel_adj_gb(const Geo &g, T *gb, int p, T gx, T gy, T gz)
{
    const int sy = g.px, sz = g.px * g.py;
    if (gx != T(0)) atom(gb + p, gx);
    if (gy != T(0)) { atom(gb + p, gy); atom(gb + p + 1, gy); atom(gb + p + sy, gy); atom(gb + p + sy + 1, gy); }
    if (gz != T(0)) { atom(gb + p, gz); atom(gb + p + sz, gz); atom(gb + p + 1, gz); atom(gb + p + sz + 1, gz); }
}

// x, y, z in [-1, n]: every stress entry a velocity update reads
// FP32: 5 CTAs per SM (48 registers; 7 % faster than the 54-register
// default, 17 % faster than 6 CTAs at 40)
template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 5 : 1) vel_adj_kernel(GridDev<T> G, AdjDev<T> A, int zt, int bottom)
{
    const Geo &g = G.g;
    int x, y;
    tile_xy(x, y);
    x -= 1;
    y -= 1;
    const int z = (int)blockIdx.z - 1;
    if (x > g.nx || y > g.ny) return;
    const T *lv[3] = {A.l[VX], A.l[VY], A.l[VZ]};
    T gx, gy, gz;
    if (inner_pt(g, x, y, z))
        vel_adj_point<T, true, false>(G, lv, G.f, A.l, zt, bottom, x, y, z, gx, gy, gz);
    else
        vel_adj_point<T, false, false>(G, lv, G.f, A.l, zt, bottom, x, y, z, gx, gy, gz);
    vel_adj_gb(g, A.gb, g.idx(x, y, z), gx, gy, gz);
}

// The velocity adjoint of shots 0 .. ns - 1 (points x, y, z in [-1, n]): a
// thread per point runs each shot's gather in turn and sums the shots'
// buoyancy-gradient terms, in shot order, before one set of atomics.
// FP32: 5 CTAs per SM (48 registers; 5 % faster than 4 at 64)
template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 5 : 2) vel_adj_shots_kernel(GridDev<T> G, T *gb, const __grid_constant__ AdjShots<T> S,
                                                             int zt, int bottom)
{
    const Geo &g = G.g;
    int x, y;
    tile_xy(x, y);
    x -= 1;
    y -= 1;
    const int z = (int)blockIdx.z - 1;
    if (x > g.nx || y > g.ny) return;
    const bool inner = inner_pt(g, x, y, z);
    const int64_t box = S.box;
    T sx = T(0), sy = T(0), sz = T(0);
    for (int s = 0; s < S.ns; s++) {
        T *l = S.l[s];
        const T *fs = S.f[s];
        const T *lv[3] = {l + VX * box, l + VY * box, l + VZ * box};
        const T *f[9];
        T *ls[9];
#pragma unroll
        for (int k = 0; k < 9; k++) {
            f[k] = fs + k * box;
            ls[k] = l + k * box;
        }
        T gx, gy, gz;
        if (inner)
            vel_adj_point<T, true, true>(G, lv, f, ls, zt, bottom, x, y, z, gx, gy, gz);
        else
            vel_adj_point<T, false, true>(G, lv, f, ls, zt, bottom, x, y, z, gx, gy, gz);
        sx = add_(sx, gx);
        sy = add_(sy, gy);
        sz = add_(sz, gz);
    }
    vel_adj_gb(g, gb, g.idx(x, y, z), sx, sy, sz);
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
__device__ __forceinline__ void vel_mirror_adj_body(const Geo &g, T *lvy, T *lvz, int phase, int top_rigid, int bottom,
                                                    int mirror_fix)
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

template <typename T>
__global__ void vel_mirror_adj_kernel(Geo g, T *lvy, T *lvz, int phase, int top_rigid, int bottom, int mirror_fix)
{
    vel_mirror_adj_body(g, lvy, lvz, phase, top_rigid, bottom, mirror_fix);
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
// 21-Cij stress update (stress21.cu), reverse mode as gathers.
// Work boxes: E[0..5] the forward strain increments e1..e6 (e3 condensed on a
// free surface), S[0..2] at N the adjoints of the averages Abar4..6
// (sum_i a_i C_i,4..6), W[0..5] the adjoints of e1..e6.  Every averaging
// relation of the forward (an output point averages a 2 x 2 neighbourhood of
// a source position with its own closure weights) is inverted: a point
// gathers from the output points whose average contains it, with the weight
// that output point gave it.
//   G0 pointwise: E, S, the own-point part of W[N]; the surface mirrors of
//      syz/sxz folded back (lambda at z = -1 added, negated, to z = 0)
//   G1 gathers: the rest of W[N] (link products P4..6 read by L4, L5, L6),
//      W[L4], W[L5], W[L6], and every coefficient gradient
//   G2 free surface: the condensed e3's adjoint to e1, e2, Abar4..6 (atomics
//      on the surface plane only)
//   G3 gathers: W -> lambda_v (transpose of the differences)
// Buffers are read only at positions valid for the grid, so values left by
// other grids (the work boxes are shared) are never seen.
// ---------------------------------------------------------------------------
enum { X_E = 0, X_S = 6, X_W = 9 };

template <typename T>
__device__ __forceinline__ T wgt(bool a0, bool a1, bool b0, bool b1, int i, int j)
{
    T wa0, wa1, wb0, wb1;
    w2<T>(a0, a1, wa0, wa1);
    w2<T>(b0, b1, wb0, wb1);
    return mul_(i ? wa1 : wa0, j ? wb1 : wb0);
}
__device__ __forceinline__ bool in_(int v, int lo, int hi) { return v >= lo && v <= hi; }

template <typename T>
__device__ __forceinline__ void g0_point(const GridDev<T> &G, const AdjDev<T> &A, int flag, const Ext &E, int x, int y, int z)
{
    const Geo &g = G.g;
    const int nx = g.nx, ny = g.ny;
    const int sz = g.px * g.py;
    const T *const *c = G.c;
    T *const *X = A.w;
    const int p = g.idx(x, y, z);
    // all loads and arithmetic of the point first, then its stores (the
    // pointers may alias as far as the compiler knows: a load after a
    // store could not be moved ahead of it and would wait for memory)
    const bool in_n = E.n(x, y, z), in_4 = E.l4(x, y, z), in_5 = E.l5(x, y, z), in_6 = E.l6(x, y, z);
    T en[3] = {}, le[3] = {}, ls[3] = {}, e4 = T(0), e5 = T(0), e6 = T(0);
    if (in_n) {
        const bool surf = flag && z == 0;
        en[0] = e1_at(G, p);
        en[1] = e2_at(G, p);
        en[2] = e3_used(G, E, surf, x, y, z, p, en[0], en[1]);
        const T a[3] = {ro(A.l[SXX], p), ro(A.l[SYY], p), surf ? T(0) : ro(A.l[SZZ], p)};
        const int rowc[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
#pragma unroll
        for (int j = 0; j < 3; j++)
#pragma unroll
            for (int i = 0; i < 3; i++) {
                le[j] = fma_(a[i], c[rowc[i][j]][p], le[j]);
                ls[j] = fma_(a[i], ro(c[6 + 3 * i + j], p), ls[j]);
            }
    }
    // the surface mirrors of syz / sxz folded back: lambda(0) - lambda(-1)
    const bool fold4 = in_4 && flag && z == 0;   // syz(-1) = -syz(0)
    const bool fold5 = in_5 && flag && z == 0 && x >= 1 && x <= nx - 1 && y >= 1 && y <= ny - 1;
    T f4 = T(0), f5 = T(0);
    if (in_4) e4 = e4_at(G, p);
    if (fold4) f4 = sub_(A.l[SYZ][p], A.l[SYZ][p - sz]);
    if (in_5) e5 = e5_at(G, p);
    if (fold5) f5 = sub_(A.l[SXZ][p], A.l[SXZ][p - sz]);
    if (in_6) e6 = e6_at(G, p);
    if (in_n) {
#pragma unroll
        for (int j = 0; j < 3; j++) {
            X[X_E + j][p] = en[j];
            X[X_W + j][p] = le[j];
            X[X_S + j][p] = ls[j];
        }
    }
    if (in_4) X[X_E + 3][p] = e4;
    if (fold4) {
        A.l[SYZ][p] = f4;
        A.l[SYZ][p - sz] = T(0);
    }
    if (in_5) X[X_E + 4][p] = e5;
    if (fold5) {
        A.l[SXZ][p] = f5;
        A.l[SXZ][p - sz] = T(0);
    }
    if (in_6) X[X_E + 5][p] = e6;
}

// FP32: 8 CTAs per SM (32 registers; 21 % faster than 4 CTAs at 64)
template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 8 : 2) stress21_adj_g0(GridDev<T> G, AdjDev<T> A, int flag)
{
    const Geo &g = G.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const Ext E{nx, ny, nz};
    {
        int x, y;
        tile_xy(x, y);
        const int z = blockIdx.z;
        if (x > nx || y > ny) return;
        g0_point(G, A, flag, E, x, y, z);
    }
}

// G1, one shot's share at one point.  Each block (the position kinds N, L4,
// L5, L6) takes the gradient slots of its position in registers (gk, loaded
// and stored by the caller), adds this shot's terms to them and writes the
// shot's strain adjoints W; a caller that holds the slots over several shots
// reads and writes them once for all.
template <typename T, bool IN>
__device__ __forceinline__ void g1_n_shot(const GridDev<T> &G, const AdjDev<T> &A, int flag, const Ext &E, int x, int y,
                                          int z, T (&gk)[15])
{
    const Geo &g = G.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const T *const *c = G.c;
    T *const *X = A.w;
    const T *l4 = A.l[SYZ], *l5 = A.l[SXZ], *l6 = A.l[SXY];
    const int p = g.idx(x, y, z), PY = g.px, PZ = g.px * g.py;
    auto I = [&](int xx, int yy, int zz) { return p + (xx - x) + (yy - y) * PY + (zz - z) * PZ; };
    auto L4 = [&](int xx, int yy, int zz) { return IN || E.l4(xx, yy, zz); };
    auto L5 = [&](int xx, int yy, int zz) { return IN || E.l5(xx, yy, zz); };
    auto L6 = [&](int xx, int yy, int zz) { return IN || E.l6(xx, yy, zz); };
    auto LN = [&](int xx, int yy, int zz) { return IN || E.n(xx, yy, zz); };
    auto inr = [&](int v, int lo, int hi) { return IN || in_(v, lo, hi); };
    auto lq = [&](int v, int hi) { return IN || v <= hi; };
    T v[2][2];
    bool oa[2], ob[2];
    T zp[3] = {T(0), T(0), T(0)};
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) {
            int qx = x, qy = y - i, qz = z - j;   // L4 tp over N (x, y..y+1, z..z+1)
            if (L4(qx, qy, qz))
                zp[0] = fma_(wgt<T>(lq(qy, ny), lq(qy + 1, ny), lq(qz, nz), lq(qz + 1, nz), i, j), ro(l4, I(qx, qy, qz)), zp[0]);
            qx = x + 1 - i; qy = y; qz = z - j;   // L5 tp over N (x-1..x, y, z..z+1)
            if (L5(qx, qy, qz))
                zp[1] = fma_(wgt<T>(inr(qx - 1, 0, nx - 1), inr(qx, 0, nx - 1), lq(qz, nz), lq(qz + 1, nz), i, j),
                             ro(l5, I(qx, qy, qz)), zp[1]);
            qx = x + 1 - i; qy = y - j; qz = z;   // L6 P6 over N (x-1..x, y..y+1, z)
            if (L6(qx, qy, qz))
                zp[2] = fma_(wgt<T>(inr(qx - 1, 0, nx - 1), inr(qx, 0, nx - 1), lq(qy, ny), lq(qy + 1, ny), i, j),
                             ro(l6, I(qx, qy, qz)), zp[2]);
        }
    const T e[3] = {ro(X[X_E + 0], p), ro(X[X_E + 1], p), ro(X[X_E + 2], p)};
    T ab[3];
    for (int i = 0; i < 2; i++) { oa[i] = inr(y - 1 + i, 0, ny - 1); ob[i] = inr(z - 1 + i, 0, nz - 1); }
    for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) v[i][j] = (oa[i] && ob[j]) ? ro(X[X_E + 3], I(x, y - 1 + i, z - 1 + j)) : T(0);
    ab[0] = avg4<T>(v, oa, ob);
    for (int i = 0; i < 2; i++) { oa[i] = lq((x + i), nx); ob[i] = inr(z - 1 + i, 0, nz - 1); }
    for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) v[i][j] = (oa[i] && ob[j]) ? ro(X[X_E + 4], I(x + i, y, z - 1 + j)) : T(0);
    ab[1] = avg4<T>(v, oa, ob);
    for (int i = 0; i < 2; i++) { oa[i] = lq((x + i), nx); ob[i] = inr(y - 1 + i, 0, ny - 1); }
    for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) v[i][j] = (oa[i] && ob[j]) ? ro(X[X_E + 5], I(x + i, y - 1 + j, z)) : T(0);
    ab[2] = avg4<T>(v, oa, ob);
    const bool surf = !IN && flag && z == 0;
    const T a[3] = {ro(A.l[SXX], p), ro(A.l[SYY], p), surf ? T(0) : ro(A.l[SZZ], p)};
    T cs[9];
#pragma unroll
    for (int k = 0; k < 9; k++) cs[k] = ro(c[6 + k], p);
    T le[3] = {X[X_W + 0][p], X[X_W + 1][p], X[X_W + 2][p]};
    const int rowc[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
#pragma unroll
    for (int i = 0; i < 3; i++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            gk[rowc[i][j]] = add_(gk[rowc[i][j]], mul_(a[i], e[j]));
            gk[6 + 3 * i + j] = add_(gk[6 + 3 * i + j], mul_(a[i], ab[j]));
        }
#pragma unroll
    for (int k = 0; k < 3; k++)
#pragma unroll
        for (int j = 0; j < 3; j++) {
            const int s = 6 + 3 * j + k;   // P(4+k) = C(1,4+k) e1 + C(2,4+k) e2 + C(3,4+k) e3
            gk[s] = add_(gk[s], mul_(zp[k], e[j]));
            le[j] = fma_(cs[s - 6], zp[k], le[j]);
        }
    X[X_W + 0][p] = le[0];
    X[X_W + 1][p] = le[1];
    X[X_W + 2][p] = le[2];
}

// L4 q: C44 a4 + C45 Z45 + C46 Z46 + Abar4 adjoints of N; slots 15..17
template <typename T, bool IN>
__device__ __forceinline__ void g1_l4_shot(const GridDev<T> &G, const AdjDev<T> &A, const Ext &E, int x, int y, int z,
                                           T &g15, T &g16, T &g17)
{
    const Geo &g = G.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const T *const *c = G.c;
    T *const *X = A.w;
    const T *l4 = A.l[SYZ], *l5 = A.l[SXZ], *l6 = A.l[SXY];
    const int p = g.idx(x, y, z), PY = g.px, PZ = g.px * g.py;
    auto I = [&](int xx, int yy, int zz) { return p + (xx - x) + (yy - y) * PY + (zz - z) * PZ; };
    auto L4 = [&](int xx, int yy, int zz) { return IN || E.l4(xx, yy, zz); };
    auto L5 = [&](int xx, int yy, int zz) { return IN || E.l5(xx, yy, zz); };
    auto L6 = [&](int xx, int yy, int zz) { return IN || E.l6(xx, yy, zz); };
    auto LN = [&](int xx, int yy, int zz) { return IN || E.n(xx, yy, zz); };
    auto inr = [&](int v, int lo, int hi) { return IN || in_(v, lo, hi); };
    auto lq = [&](int v, int hi) { return IN || v <= hi; };
    T v[2][2];
    bool oa[2], ob[2];
    const T a4 = ro(l4, p), e4 = ro(X[X_E + 3], p);
    T z45 = T(0), z46 = T(0), sn = T(0);
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) {
            int sx = x + 1 - i, sy = y + 1 - j, sz_ = z;   // L5 t45 over L4 (x-1..x, y-1..y, z)
            if (L5(sx, sy, sz_))
                z45 = fma_(wgt<T>(inr(sx - 1, 0, nx - 1), inr(sx, 0, nx - 1), inr(sy - 1, 0, ny - 1), inr(sy, 0, ny - 1), i, j),
                           ro(l5, I(sx, sy, sz_)), z45);
            sx = x + 1 - i; sy = y; sz_ = z + 1 - j;       // L6 t46 over L4 (x-1..x, y, z-1..z)
            if (L6(sx, sy, sz_))
                z46 = fma_(wgt<T>(inr(sx - 1, 0, nx - 1), inr(sx, 0, nx - 1), inr(sz_ - 1, 0, nz - 1), inr(sz_, 0, nz - 1), i, j),
                           ro(l6, I(sx, sy, sz_)), z46);
            sx = x; sy = y + 1 - i; sz_ = z + 1 - j;       // N Abar4 over L4 (x, y-1..y, z-1..z)
            if (LN(sx, sy, sz_))
                sn = fma_(wgt<T>(inr(sy - 1, 0, ny - 1), inr(sy, 0, ny - 1), inr(sz_ - 1, 0, nz - 1), inr(sz_, 0, nz - 1), i, j),
                          ro(X[X_S + 0], I(sx, sy, sz_)), sn);
        }
    // forward averages t5 (e5 over L5 (x..x+1, y..y+1, z)) and t6 (e6 over L6 (x..x+1, y, z..z+1))
    for (int i = 0; i < 2; i++) { oa[i] = lq((x + i), nx); ob[i] = lq((y + i), ny); }
    for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) v[i][j] = (oa[i] && ob[j]) ? ro(X[X_E + 4], I(x + i, y + j, z)) : T(0);
    const T t5 = avg4<T>(v, oa, ob);
    for (int i = 0; i < 2; i++) { oa[i] = lq((x + i), nx); ob[i] = lq((z + i), nz); }
    for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) v[i][j] = (oa[i] && ob[j]) ? ro(X[X_E + 5], I(x + i, y, z + j)) : T(0);
    const T t6 = avg4<T>(v, oa, ob);
    const T c15 = ro(c[15], p), c16 = ro(c[16], p), c17 = ro(c[17], p);
    g15 = add_(g15, mul_(a4, e4));
    g16 = add_(g16, add_(mul_(a4, t5), mul_(z45, e4)));
    g17 = add_(g17, add_(mul_(a4, t6), mul_(z46, e4)));
    X[X_W + 3][p] = add_(fma_(c15, a4, fma_(c16, z45, mul_(c17, z46))), sn);
}

// L5 s: C55 a5 + C56 Z56 + Abar5 adjoints of N + C45 a4 from L4's t5; slots 18, 19
template <typename T, bool IN>
__device__ __forceinline__ void g1_l5_shot(const GridDev<T> &G, const AdjDev<T> &A, const Ext &E, int x, int y, int z,
                                           T &g18, T &g19)
{
    const Geo &g = G.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const T *const *c = G.c;
    T *const *X = A.w;
    const T *l4 = A.l[SYZ], *l5 = A.l[SXZ], *l6 = A.l[SXY];
    const int p = g.idx(x, y, z), PY = g.px, PZ = g.px * g.py;
    auto I = [&](int xx, int yy, int zz) { return p + (xx - x) + (yy - y) * PY + (zz - z) * PZ; };
    auto L4 = [&](int xx, int yy, int zz) { return IN || E.l4(xx, yy, zz); };
    auto L5 = [&](int xx, int yy, int zz) { return IN || E.l5(xx, yy, zz); };
    auto L6 = [&](int xx, int yy, int zz) { return IN || E.l6(xx, yy, zz); };
    auto LN = [&](int xx, int yy, int zz) { return IN || E.n(xx, yy, zz); };
    auto inr = [&](int v, int lo, int hi) { return IN || in_(v, lo, hi); };
    auto lq = [&](int v, int hi) { return IN || v <= hi; };
    T v[2][2];
    bool oa[2], ob[2];
    const T a5 = ro(l5, p), e5 = ro(X[X_E + 4], p);
    T z56 = T(0), sn = T(0), s4 = T(0);
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) {
            int qx = x, qy = y - i, qz = z + 1 - j;      // L6 t56 over L5 (x, y..y+1, z-1..z)
            if (L6(qx, qy, qz))
                z56 = fma_(wgt<T>(lq(qy, ny), lq(qy + 1, ny), inr(qz - 1, 0, nz - 1), inr(qz, 0, nz - 1), i, j), ro(l6, I(qx, qy, qz)), z56);
            qx = x - i; qy = y; qz = z + 1 - j;          // N Abar5 over L5 (x..x+1, y, z-1..z)
            if (LN(qx, qy, qz))
                sn = fma_(wgt<T>(lq(qx, nx), lq(qx + 1, nx), inr(qz - 1, 0, nz - 1), inr(qz, 0, nz - 1), i, j),
                          ro(X[X_S + 1], I(qx, qy, qz)), sn);
            qx = x - i; qy = y - j; qz = z;              // L4 t5 over L5 (x..x+1, y..y+1, z)
            if (L4(qx, qy, qz)) {
                const int q = I(qx, qy, qz);
                s4 = fma_(wgt<T>(lq(qx, nx), lq(qx + 1, nx), lq(qy, ny), lq(qy + 1, ny), i, j), mul_(ro(c[16], q), ro(l4, q)), s4);
            }
        }
    // forward average t6 (e6 over L6 (x, y-1..y, z..z+1))
    for (int i = 0; i < 2; i++) { oa[i] = inr(y - 1 + i, 0, ny - 1); ob[i] = lq((z + i), nz); }
    for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) v[i][j] = (oa[i] && ob[j]) ? ro(X[X_E + 5], I(x, y - 1 + i, z + j)) : T(0);
    const T t6 = avg4<T>(v, oa, ob);
    const T c18 = ro(c[18], p), c19 = ro(c[19], p);
    g18 = add_(g18, mul_(a5, e5));
    g19 = add_(g19, add_(mul_(a5, t6), mul_(z56, e5)));
    X[X_W + 4][p] = add_(add_(fma_(c18, a5, mul_(c19, z56)), sn), s4);
}

// L6 t: C66 a6 + Abar6 adjoints of N + C46 a4 (L4 t6) + C56 a5 (L5 t6); slot 20
template <typename T, bool IN>
__device__ __forceinline__ void g1_l6_shot(const GridDev<T> &G, const AdjDev<T> &A, const Ext &E, int x, int y, int z, T &g20)
{
    const Geo &g = G.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const T *const *c = G.c;
    T *const *X = A.w;
    const T *l4 = A.l[SYZ], *l5 = A.l[SXZ], *l6 = A.l[SXY];
    const int p = g.idx(x, y, z), PY = g.px, PZ = g.px * g.py;
    auto I = [&](int xx, int yy, int zz) { return p + (xx - x) + (yy - y) * PY + (zz - z) * PZ; };
    auto L4 = [&](int xx, int yy, int zz) { return IN || E.l4(xx, yy, zz); };
    auto L5 = [&](int xx, int yy, int zz) { return IN || E.l5(xx, yy, zz); };
    auto L6 = [&](int xx, int yy, int zz) { return IN || E.l6(xx, yy, zz); };
    auto LN = [&](int xx, int yy, int zz) { return IN || E.n(xx, yy, zz); };
    auto inr = [&](int v, int lo, int hi) { return IN || in_(v, lo, hi); };
    auto lq = [&](int v, int hi) { return IN || v <= hi; };
    const T a6 = ro(l6, p);
    T sn = T(0), s4 = T(0), s5 = T(0);
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++) {
            int qx = x - i, qy = y + 1 - j, qz = z;      // N Abar6 over L6 (x..x+1, y-1..y, z)
            if (LN(qx, qy, qz))
                sn = fma_(wgt<T>(lq(qx, nx), lq(qx + 1, nx), inr(qy - 1, 0, ny - 1), inr(qy, 0, ny - 1), i, j),
                          ro(X[X_S + 2], I(qx, qy, qz)), sn);
            qx = x - i; qy = y; qz = z - j;              // L4 t6 over L6 (x..x+1, y, z..z+1)
            if (L4(qx, qy, qz)) {
                const int q = I(qx, qy, qz);
                s4 = fma_(wgt<T>(lq(qx, nx), lq(qx + 1, nx), lq(qz, nz), lq(qz + 1, nz), i, j), mul_(ro(c[17], q), ro(l4, q)), s4);
            }
            qx = x; qy = y + 1 - i; qz = z - j;          // L5 t6 over L6 (x, y-1..y, z..z+1)
            if (L5(qx, qy, qz)) {
                const int q = I(qx, qy, qz);
                s5 = fma_(wgt<T>(inr(qy - 1, 0, ny - 1), inr(qy, 0, ny - 1), lq(qz, nz), lq(qz + 1, nz), i, j),
                          mul_(ro(c[19], q), ro(l5, q)), s5);
            }
        }
    const T e6 = ro(X[X_E + 5], p), c20 = ro(c[20], p);
    g20 = add_(g20, mul_(a6, e6));
    X[X_W + 5][p] = add_(add_(fma_(c20, a6, sn), s4), s5);
}

// One point of G1 for shots 0..ns-1: the gradient slots of each position
// block are read once, take every shot's terms in shot order, and are written
// once.  shot(s, Gs, As) gives shot s's forward-field and adjoint views.
template <typename T, bool IN, typename Shot>
__device__ __forceinline__ void g1_point_k(const GridDev<T> &G, const AdjDev<T> &A0, int flag, const Ext &E, int x, int y,
                                         int z, int ns, Shot shot)
{
    const int p = G.g.idx(x, y, z);
    if (IN || E.n(x, y, z)) {
        T gk[15];
#pragma unroll
        for (int k = 0; k < 15; k++) gk[k] = A0.gc[k][p];
        for (int s = 0; s < ns; s++) {
            GridDev<T> Gs;
            AdjDev<T> As;
            shot(s, Gs, As);
            g1_n_shot<T, IN>(Gs, As, flag, E, x, y, z, gk);
        }
#pragma unroll
        for (int k = 0; k < 15; k++) A0.gc[k][p] = gk[k];
    }
    if (IN || E.l4(x, y, z)) {
        T g15 = A0.gc[15][p], g16 = A0.gc[16][p], g17 = A0.gc[17][p];
        for (int s = 0; s < ns; s++) {
            GridDev<T> Gs;
            AdjDev<T> As;
            shot(s, Gs, As);
            g1_l4_shot<T, IN>(Gs, As, E, x, y, z, g15, g16, g17);
        }
        A0.gc[15][p] = g15;
        A0.gc[16][p] = g16;
        A0.gc[17][p] = g17;
    }
    if (IN || E.l5(x, y, z)) {
        T g18 = A0.gc[18][p], g19 = A0.gc[19][p];
        for (int s = 0; s < ns; s++) {
            GridDev<T> Gs;
            AdjDev<T> As;
            shot(s, Gs, As);
            g1_l5_shot<T, IN>(Gs, As, E, x, y, z, g18, g19);
        }
        A0.gc[18][p] = g18;
        A0.gc[19][p] = g19;
    }
    if (IN || E.l6(x, y, z)) {
        T g20 = A0.gc[20][p];
        for (int s = 0; s < ns; s++) {
            GridDev<T> Gs;
            AdjDev<T> As;
            shot(s, Gs, As);
            g1_l6_shot<T, IN>(Gs, As, E, x, y, z, g20);
        }
        A0.gc[20][p] = g20;
    }
}

template <typename T, typename Shot>
__device__ __forceinline__ void g1_point(const GridDev<T> &G, const AdjDev<T> &A0, int flag, const Ext &E, int x, int y,
                                         int z, int ns, Shot shot)
{
    if (inner_pt(G.g, x, y, z))
        g1_point_k<T, true>(G, A0, flag, E, x, y, z, ns, shot);
    else
        g1_point_k<T, false>(G, A0, flag, E, x, y, z, ns, shot);
}

// FP32: 3 CTAs per SM (80 registers; 7 % faster than 4 CTAs at 64 registers,
// 14 % faster than 2 at 124)
template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 3 : 2) stress21_adj_g1(GridDev<T> G, AdjDev<T> A, int flag)
{
    const Geo &g = G.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const Ext E{nx, ny, nz};
    auto one = [&](int, GridDev<T> &Gs, AdjDev<T> &As) { Gs = G; As = A; };
    {
        int x, y;
        tile_xy(x, y);
        const int z = blockIdx.z;
        if (x > nx || y > ny) return;
        g1_point(G, A, flag, E, x, y, z, 1, one);
    }
}

// Views of shot s: the common medium and gradients with the shot's fields,
// adjoint fields and work boxes.
template <typename T>
__device__ __forceinline__ void shot_views(const GridDev<T> &G, const AdjDev<T> &A0, const AdjShots<T> &S, int s,
                                           GridDev<T> &Gs, AdjDev<T> &As)
{
    Gs = G;
    As = A0;
#pragma unroll
    for (int k = 0; k < 9; k++) {
        Gs.f[k] = S.f[s] + k * S.box;
        As.l[k] = S.l[s] + k * S.box;
    }
#pragma unroll
    for (int k = 0; k < 15; k++) As.w[k] = S.w[s] + k * S.wbox;
}

// G0 of shots 0 .. ns - 1, the shots in turn in one thread per point (the
// coefficients' loads of the next shot hit L1; 8 % faster than putting the
// shots of a tile in side-by-side CTAs)
// FP32: 6 CTAs per SM (40 registers; 11 % faster than 4 at 64)
template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 6 : 2) stress21_adj_g0_shots(GridDev<T> G, AdjDev<T> A0,
                                                                   const __grid_constant__ AdjShots<T> S, int flag)
{
    const Geo &g = G.g;
    const Ext E{g.nx, g.ny, g.nz};
    int x, y;
    tile_xy(x, y);
    const int z = blockIdx.z;
    if (x > g.nx || y > g.ny) return;
    for (int s = 0; s < S.ns; s++) {
        GridDev<T> Gs;
        AdjDev<T> As;
        shot_views(G, A0, S, s, Gs, As);
        g0_point(Gs, As, flag, E, x, y, z);
    }
}

// G1 of shots 0 .. ns - 1: a thread per point runs the shots in turn, the
// point's gradient slots and medium read once for all of them (g1_point).
template <typename T>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? 4 : 2)
    stress21_adj_g1_shots(GridDev<T> G, AdjDev<T> A0, const __grid_constant__ AdjShots<T> S, int flag)
{
    const Geo &g = G.g;
    const Ext E{g.nx, g.ny, g.nz};
    int x, y;
    tile_xy(x, y);
    const int z = blockIdx.z;
    if (x > g.nx || y > g.ny) return;
    auto shot = [&](int s, GridDev<T> &Gs, AdjDev<T> &As) { shot_views(G, A0, S, s, Gs, As); };
    g1_point(G, A0, flag, E, x, y, z, S.ns, shot);
}

// free surface: e3 = -(C13 e1 + C23 e2 + C34 A4 + C35 A5 + C36 A6) / C33 at z = 0
template <typename T>
__global__ void stress21_adj_g2(GridDev<T> G, AdjDev<T> A)
{
    const Geo &g = G.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int n = nx * (ny + 1);
    const int t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= n) return;
    const int x = t % nx, y = t / nx, z = 0;
    const int p = g.idx(x, y, z);
    T *const *X = A.w;
    const T le3 = X[X_W + 2][p];
    if (le3 == T(0)) return;
    X[X_W + 2][p] = T(0);
    const T *const *c = G.c;
    const T c33 = c[5][p];
    const T e1 = X[X_E + 0][p], e2 = X[X_E + 1][p], e3 = X[X_E + 2][p];
    T v[2][2], w[2][2];
    bool oa[2], ob[2];
    T ab[3];
    int bx[3][2][2], by[3][2][2], bz[3][2][2];
    T bw[3][2][2];
    // Abar4: L4 (x, y-1+i, z-1+j); Abar5: L5 (x+i, y, z-1+j); Abar6: L6 (x+i, y-1+j, z)
    for (int k = 0; k < 3; k++) {
        for (int i = 0; i < 2; i++) {
            if (k == 0) { oa[i] = in_(y - 1 + i, 0, ny - 1); ob[i] = in_(z - 1 + i, 0, nz - 1); }
            else if (k == 1) { oa[i] = (x + i) <= nx; ob[i] = in_(z - 1 + i, 0, nz - 1); }
            else { oa[i] = (x + i) <= nx; ob[i] = in_(y - 1 + i, 0, ny - 1); }
        }
        for (int i = 0; i < 2; i++)
            for (int j = 0; j < 2; j++) {
                bx[k][i][j] = k == 0 ? x : x + i;
                by[k][i][j] = k == 0 ? y - 1 + i : (k == 1 ? y : y - 1 + j);
                bz[k][i][j] = k == 2 ? z : z - 1 + j;
                v[i][j] = (oa[i] && ob[j]) ? X[X_E + 3 + k][g.idx(bx[k][i][j], by[k][i][j], bz[k][i][j])] : T(0);
            }
        ab[k] = avg4<T>(v, oa, ob);
        weights4(oa, ob, w);
        for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) bw[k][i][j] = w[i][j];
    }
    const T u = -div_(le3, c33);   // d e3 / d(numerator term) = -1 / C33
    X[X_W + 0][p] = fma_(u, c[2][p], X[X_W + 0][p]);
    X[X_W + 1][p] = fma_(u, c[4][p], X[X_W + 1][p]);
    A.gc[2][p] = fma_(u, e1, A.gc[2][p]);
    A.gc[4][p] = fma_(u, e2, A.gc[4][p]);
    A.gc[5][p] = fma_(u, e3, A.gc[5][p]);   // d e3 / d C33 = -e3 / C33
    for (int k = 0; k < 3; k++) {
        A.gc[12 + k][p] = fma_(u, ab[k], A.gc[12 + k][p]);
        const T lk = mul_(u, c[12 + k][p]);
        for (int i = 0; i < 2; i++)
            for (int j = 0; j < 2; j++)
                if (bw[k][i][j] != T(0)) atom(X[X_W + 3 + k] + g.idx(bx[k][i][j], by[k][i][j], bz[k][i][j]), mul_(bw[k][i][j], lk));
    }
}

// transpose of the strain differences: every velocity entry gathers the W of
// the strains that read it
// G3 at one point: IN: every neighbour range test holds (points in [2, n - 3])
template <typename T, bool IN>
__device__ __forceinline__ void g3_point(const GridDev<T> &G, const AdjDev<T> &A, int x, int y, int z)
{
    const Geo &g = G.g;
    const Ext E{g.nx, g.ny, g.nz};
    const T k0 = G.k[0], k1 = G.k[1], k2 = G.k[2];
    T *const *X = A.w;
    auto I = [&](int xx, int yy, int zz) { return g.idx(xx, yy, zz); };
    auto W = [&](int k, bool ok, int xx, int yy, int zz) -> T { return (IN || ok) ? X[X_W + k][I(xx, yy, zz)] : T(0); };
    const int p = I(x, y, z);
    // vx: e1(N x-1) - e1(N x), e5(L5 z-1) - e5(L5 z), e6(L6 y-1) - e6(L6 y)
    const T gx = add_(add_(mul_(k0, sub_(W(0, E.n(x - 1, y, z), x - 1, y, z), W(0, E.n(x, y, z), x, y, z))),
                           mul_(k2, sub_(W(4, E.l5(x, y, z - 1), x, y, z - 1), W(4, E.l5(x, y, z), x, y, z)))),
                      mul_(k1, sub_(W(5, E.l6(x, y - 1, z), x, y - 1, z), W(5, E.l6(x, y, z), x, y, z))));
    // vy: e2(N y) - e2(N y+1), e4(L4 z-1) - e4(L4 z), e6(L6 x) - e6(L6 x+1)
    const T gy = add_(add_(mul_(k1, sub_(W(1, E.n(x, y, z), x, y, z), W(1, E.n(x, y + 1, z), x, y + 1, z))),
                           mul_(k2, sub_(W(3, E.l4(x, y, z - 1), x, y, z - 1), W(3, E.l4(x, y, z), x, y, z)))),
                      mul_(k0, sub_(W(5, E.l6(x, y, z), x, y, z), W(5, E.l6(x + 1, y, z), x + 1, y, z))));
    // vz: e3(N z) - e3(N z+1), e4(L4 y-1) - e4(L4 y), e5(L5 x) - e5(L5 x+1)
    const T gz = add_(add_(mul_(k2, sub_(W(2, E.n(x, y, z), x, y, z), W(2, E.n(x, y, z + 1), x, y, z + 1))),
                           mul_(k1, sub_(W(3, E.l4(x, y - 1, z), x, y - 1, z), W(3, E.l4(x, y, z), x, y, z)))),
                      mul_(k0, sub_(W(4, E.l5(x, y, z), x, y, z), W(4, E.l5(x + 1, y, z), x + 1, y, z))));
    // the three loads before the first store (they are in the box for every
    // x, y, z in [-1, n])
    const T lx = A.l[VX][p], ly = A.l[VY][p], lz = A.l[VZ][p];
    if (gx != T(0)) A.l[VX][p] = add_(lx, gx);
    if (gy != T(0)) A.l[VY][p] = add_(ly, gy);
    if (gz != T(0)) A.l[VZ][p] = add_(lz, gz);
}

template <typename T>
__device__ __forceinline__ void g3_body(const GridDev<T> &G, const AdjDev<T> &A, int zb)
{
    const Geo &g = G.g;
    int x, y;
    tile_xy(x, y);
    x -= 1;
    y -= 1;
    const int z = zb - 1;
    if (x > g.nx || y > g.ny) return;
    if (inner_pt(g, x, y, z))
        g3_point<T, true>(G, A, x, y, z);
    else
        g3_point<T, false>(G, A, x, y, z);
}

template <typename T>
__global__ void stress21_adj_g3(GridDev<T> G, AdjDev<T> A)
{
    g3_body(G, A, blockIdx.z);
}

// G3 of every shot: blockIdx.z = plane + (nz + 2) * shot
template <typename T>
__global__ void stress21_adj_g3_shots(GridDev<T> G, AdjDev<T> A0, const __grid_constant__ AdjShots<T> S)
{
    const int nzb = G.g.nz + 2;
    GridDev<T> Gs;
    AdjDev<T> As;
    shot_views(G, A0, S, blockIdx.z / nzb, Gs, As);
    g3_body(Gs, As, blockIdx.z % nzb);
}

// velocity mirror transposes of every shot: shot blockIdx.y
template <typename T>
__global__ void vel_mirror_adj_shots_kernel(Geo g, const __grid_constant__ AdjShots<T> S, int phase, int top_rigid,
                                            int bottom, int mirror_fix)
{
    T *l = S.l[blockIdx.y];
    vel_mirror_adj_body(g, l + VY * S.box, l + VZ * S.box, phase, top_rigid, bottom, mirror_fix);
}

// ---------------------------------------------------------------------------
// Launchers
// ---------------------------------------------------------------------------
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
    vel_adj_kernel<T><<<grid3(g.nx + 2, g.ny + 2, g.nz + 2), 256, 0, st>>>(G, A, zt, bottom);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_stress21_adj(const GridDev<T> &G, const AdjDev<T> &A, int top, int top_bc, int sms, cudaStream_t st)
{
    const Geo &g = G.g;
    const int flag = (top && top_bc) ? 1 : 0;
    const dim3 nb = grid3(g.nx + 1, g.ny + 1, g.nz + 1);
    stress21_adj_g0<T><<<nb, 256, 0, st>>>(G, A, flag);
    stress21_adj_g1<T><<<nb, 256, 0, st>>>(G, A, flag);
    if (flag) stress21_adj_g2<T><<<(g.nx * (g.ny + 1) + 255) / 256, 256, 0, st>>>(G, A);
    stress21_adj_g3<T><<<grid3(g.nx + 2, g.ny + 2, g.nz + 2), 256, 0, st>>>(G, A);
    return cudaGetLastError();
}

// The 21-Cij stress adjoint of every shot of one grid: G0 and G1 once for all
// shots, then G2 (free surface) and G3 per shot; A0 holds the common gradients.
template <typename T>
cudaError_t launch_stress21_adj_shots(const GridDev<T> &G, const AdjDev<T> &A0, const AdjShots<T> &S, int top, int top_bc,
                                      int sms, cudaStream_t st)
{
    const Geo &g = G.g;
    const int flag = (top && top_bc) ? 1 : 0;
    stress21_adj_g0_shots<T><<<grid3(g.nx + 1, g.ny + 1, g.nz + 1), 256, 0, st>>>(G, A0, S, flag);
    stress21_adj_g1_shots<T><<<grid3(g.nx + 1, g.ny + 1, g.nz + 1), 256, 0, st>>>(G, A0, S, flag);   // 4 CTAs/SM: 13 % faster than 3
    if (flag)   // the free surface adds to the common gradient without atomics: one shot at a time
        for (int s = 0; s < S.ns; s++) {
            GridDev<T> Gs = G;
            AdjDev<T> As = A0;
            for (int k = 0; k < 9; k++) {
                Gs.f[k] = S.f[s] + k * S.box;
                As.l[k] = S.l[s] + k * S.box;
            }
            for (int k = 0; k < 15; k++) As.w[k] = S.w[s] + k * S.wbox;
            stress21_adj_g2<T><<<(g.nx * (g.ny + 1) + 255) / 256, 256, 0, st>>>(Gs, As);
        }
    stress21_adj_g3_shots<T><<<grid3(g.nx + 2, g.ny + 2, (g.nz + 2) * S.ns), 256, 0, st>>>(G, A0, S);
    return cudaGetLastError();
}

// The velocity adjoint of every shot of one grid: each shot's mirror
// transposes, then the update's transpose for all shots at once.
template <typename T>
cudaError_t launch_vel_adj_shots(const GridDev<T> &G, T *gb, const AdjShots<T> &S, int top, int bottom, int top_bc,
                                 int mirror_fix, int sms, cudaStream_t st)
{
    const Geo &g = G.g;
    const int top_rigid = (top && top_bc != 1) ? 1 : 0;
    const int64_t n0 = (int64_t)(top_rigid + bottom) * (g.ny + 1) * g.nx + 2LL * g.nz * (g.ny + 1)
                     + 2LL * (g.nz + 1) * (g.ny + 1);
    const int64_t n1 = 2LL * (g.nz + (mirror_fix ? 1 : 0)) * g.nx;
    vel_mirror_adj_shots_kernel<T><<<dim3((unsigned)((n1 + 255) / 256), S.ns), 256, 0, st>>>(g, S, 1, top_rigid, bottom,
                                                                                             mirror_fix);
    vel_mirror_adj_shots_kernel<T><<<dim3((unsigned)((n0 + 255) / 256), S.ns), 256, 0, st>>>(g, S, 0, top_rigid, bottom,
                                                                                             mirror_fix);
    vel_adj_shots_kernel<T><<<grid3(g.nx + 2, g.ny + 2, g.nz + 2), 256, 0, st>>>(G, gb, S, top_rigid, bottom);
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
    template cudaError_t launch_rec_adj<T>(const RecAdj<T> &, cudaStream_t);                                  \
    template cudaError_t launch_stress21_adj_shots<T>(const GridDev<T> &, const AdjDev<T> &, const AdjShots<T> &,  \
                                                      int, int, int, cudaStream_t);                              \
    template cudaError_t launch_vel_adj_shots<T>(const GridDev<T> &, T *, const AdjShots<T> &, int, int, int, int,  \
                                                 int, cudaStream_t);
INST(float)
INST(double)
#undef INST

} // namespace ecsg

namespace ecsg {

// Receiver values at full precision (the misfit's samples; sampled as main.cpp:182-184)
template <typename T>
__global__ void rec_sample_kernel(SrcRec S, T *out)
{
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < S.nrec; i += gridDim.x * blockDim.x)
        out[i] = ((const T *)S.rec_base[S.rec_grid[i]])[S.rec_off[i]];
}

// residual = sample - observed (in place); each CTA's share of 1/2 sum
// residual^2 (FP64) into partial[blockIdx.x], summed in CTA order by
// loss_sum_kernel, so the loss is the same on every run
template <typename T>
__global__ void residual_kernel(T *rec, const float *obs, int64_t n, double *partial)
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
        partial[blockIdx.x] = t;
    }
}

__global__ void loss_sum_kernel(const double *partial, int nblocks, double *loss)
{
    double t = 0.0;
    for (int b = 0; b < nblocks; b++) t += partial[b];
    *loss = t;
}

template <typename T>
cudaError_t launch_rec_sample(const SrcRec &S, T *out, cudaStream_t st)
{
    if (S.nrec <= 0) return cudaSuccess;
    const int blocks = (S.nrec + 255) / 256 < 1024 ? (S.nrec + 255) / 256 : 1024;
    rec_sample_kernel<T><<<blocks, 256, 0, st>>>(S, out);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_residual(T *rec, const float *obs, int64_t n, double *loss, double *partial, int max_blocks,
                            cudaStream_t st)
{
    if (n <= 0) return cudaSuccess;
    int64_t b = (n + 255) / 256;
    if (b > max_blocks) b = max_blocks;
    residual_kernel<T><<<(unsigned)b, 256, 0, st>>>(rec, obs, n, partial);
    loss_sum_kernel<<<1, 1, 0, st>>>(partial, (int)b, loss);
    return cudaGetLastError();
}

template cudaError_t launch_rec_sample<float>(const SrcRec &, float *, cudaStream_t);
template cudaError_t launch_rec_sample<double>(const SrcRec &, double *, cudaStream_t);
template cudaError_t launch_residual<float>(float *, const float *, int64_t, double *, double *, int, cudaStream_t);
template cudaError_t launch_residual<double>(double *, const float *, int64_t, double *, double *, int, cudaStream_t);

} // namespace ecsg
