// gen21_device.cuh -- device helpers of the 21-Cij stress update shared by
// stress21.cu and the interface solve (strain increments at the staggered
// positions, closure-weighted neighbour averages, the szz-rate terms beyond
// the orthorhombic ones).  See stress21.cu for the scheme.
#pragma once
#include "ecsg_device.cuh"

namespace ecsg {

// a*b + c: one rounding in FP32 (both FP32 sweeps use the same contractions,
// so they stay bitwise equal to each other); in FP64 the product and the sum
// are rounded separately, the oracle's operation order (the sum is
// commutative, so fma_(a, b, c) == add_(c, mul_(a, b)) bit for bit).
__device__ __forceinline__ float fma_(float a, float b, float c) { return __fmaf_rn(a, b, c); }
__device__ __forceinline__ double fma_(double a, double b, double c) { return add_(mul_(a, b), c); }

struct Ext {
    int nx, ny, nz;
    __device__ __forceinline__ bool n(int x, int y, int z) const { return x >= 0 && x <= nx - 1 && y >= 0 && y <= ny && z >= 0 && z <= nz; }
    __device__ __forceinline__ bool l4(int x, int y, int z) const { return x >= 0 && x <= nx - 1 && y >= 0 && y <= ny - 1 && z >= 0 && z <= nz - 1; }
    __device__ __forceinline__ bool l5(int x, int y, int z) const { return x >= 0 && x <= nx && y >= 0 && y <= ny && z >= 0 && z <= nz - 1; }
    __device__ __forceinline__ bool l6(int x, int y, int z) const { return x >= 0 && x <= nx && y >= 0 && y <= ny - 1 && z >= 0 && z <= nz; }
};

// strain increments at existing points (velocities incl. halos, mirrors, ghosts)
template <typename T>
__device__ __forceinline__ T e1_at(const GridDev<T> &G, int p) { return mul_(G.k[0], sub_(G.f[VX][p + 1], G.f[VX][p])); }
template <typename T>
__device__ __forceinline__ T e2_at(const GridDev<T> &G, int p) { return mul_(G.k[1], sub_(G.f[VY][p], G.f[VY][p - G.g.px])); }
template <typename T>
__device__ __forceinline__ T e3_at(const GridDev<T> &G, int p) { return mul_(G.k[2], sub_(G.f[VZ][p], G.f[VZ][p - G.g.px * G.g.py])); }
template <typename T>
__device__ __forceinline__ T e4_at(const GridDev<T> &G, int p)
{
    const int sy = G.g.px, sz = G.g.px * G.g.py;
    return fma_(G.k[1], sub_(G.f[VZ][p + sy], G.f[VZ][p]), mul_(G.k[2], sub_(G.f[VY][p + sz], G.f[VY][p])));
}
template <typename T>
__device__ __forceinline__ T e5_at(const GridDev<T> &G, int p)
{
    const int sz = G.g.px * G.g.py;
    return fma_(G.k[0], sub_(G.f[VZ][p], G.f[VZ][p - 1]), mul_(G.k[2], sub_(G.f[VX][p + sz], G.f[VX][p])));
}
template <typename T>
__device__ __forceinline__ T e6_at(const GridDev<T> &G, int p)
{
    const int sy = G.g.px;
    return fma_(G.k[0], sub_(G.f[VY][p], G.f[VY][p - 1]), mul_(G.k[1], sub_(G.f[VX][p + sy], G.f[VX][p])));
}

// 1-D closure weights of two neighbours
template <typename T>
__device__ __forceinline__ void w2(bool a, bool b, T &wa, T &wb)
{
    wa = a ? (b ? T(0.5) : T(1)) : T(0);
    wb = b ? (a ? T(0.5) : T(1)) : T(0);
}

// average over (i in {0,1} of dim d0) x (j in {0,1} of dim d1), i outer, in
// the accumulation order of the oracle; v[i][j], ok0[i], ok1[j]
template <typename T>
__device__ __forceinline__ T avg4(const T (&v)[2][2], const bool (&ok0)[2], const bool (&ok1)[2])
{
    T wa0, wa1, wb0, wb1;
    w2<T>(ok0[0], ok0[1], wa0, wa1);
    w2<T>(ok1[0], ok1[1], wb0, wb1);
    const T w0[2] = {wa0, wa1}, w1[2] = {wb0, wb1};
    T acc = T(0);
#pragma unroll
    for (int i = 0; i < 2; i++)
#pragma unroll
        for (int j = 0; j < 2; j++) {
            const T w = mul_(w0[i], w1[j]);
            if (w != T(0)) acc = fma_(w, v[i][j], acc);
        }
    return acc;
}

// Abar4/5/6 at an N point from global memory (used on the free-surface plane
// and by the interface solve): L4 (x, y-1..y, z-1..z), L5 (x..x+1, y, z-1..z),
// L6 (x..x+1, y-1..y, z).
template <typename T>
__device__ T abar4_g(const GridDev<T> &G, const Ext &E, int x, int y, int z)
{
    T v[2][2];
    bool a[2], b[2];
    for (int i = 0; i < 2; i++) {
        a[i] = (y - 1 + i) >= 0 && (y - 1 + i) <= E.ny - 1;
        b[i] = (z - 1 + i) >= 0 && (z - 1 + i) <= E.nz - 1;
    }
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++)
            v[i][j] = (a[i] && b[j]) ? e4_at(G, G.g.idx(x, y - 1 + i, z - 1 + j)) : T(0);
    return avg4<T>(v, a, b);
}
template <typename T>
__device__ T abar5_g(const GridDev<T> &G, const Ext &E, int x, int y, int z)
{
    T v[2][2];
    bool a[2], b[2];
    for (int i = 0; i < 2; i++) {
        a[i] = (x + i) >= 0 && (x + i) <= E.nx;
        b[i] = (z - 1 + i) >= 0 && (z - 1 + i) <= E.nz - 1;
    }
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++)
            v[i][j] = (a[i] && b[j]) ? e5_at(G, G.g.idx(x + i, y, z - 1 + j)) : T(0);
    return avg4<T>(v, a, b);
}
template <typename T>
__device__ T abar6_g(const GridDev<T> &G, const Ext &E, int x, int y, int z)
{
    T v[2][2];
    bool a[2], b[2];
    for (int i = 0; i < 2; i++) {
        a[i] = (x + i) >= 0 && (x + i) <= E.nx;
        b[i] = (y - 1 + i) >= 0 && (y - 1 + i) <= E.ny - 1;
    }
    for (int i = 0; i < 2; i++)
        for (int j = 0; j < 2; j++)
            v[i][j] = (a[i] && b[j]) ? e6_at(G, G.g.idx(x + i, y - 1 + j, z)) : T(0);
    return avg4<T>(v, a, b);
}

// szz-rate terms beyond the orthorhombic ones at an N point (interface solve)
template <typename T>
__device__ __forceinline__ double gen21_szz_extra(const GridDev<T> &G, int x, int y, int z)
{
    const Ext E{G.g.nx, G.g.ny, G.g.nz};
    const int p = G.g.idx(x, y, z);
    return (double)fma_(G.c[14][p], abar6_g(G, E, x, y, z),
                        fma_(G.c[13][p], abar5_g(G, E, x, y, z), mul_(G.c[12][p], abar4_g(G, E, x, y, z))));
}

template <typename T>
__device__ __forceinline__ T e3_used(const GridDev<T> &G, const Ext &E, bool surf, int x, int y, int z, int p, T e1, T e2)
{
    if (!surf) return e3_at(G, p);
    T num = fma_(G.c[14][p], abar6_g(G, E, x, y, z),
                 fma_(G.c[13][p], abar5_g(G, E, x, y, z),
                      fma_(G.c[12][p], abar4_g(G, E, x, y, z), fma_(G.c[4][p], e2, mul_(G.c[2][p], e1)))));
    return -div_(num, G.c[5][p]);
}

} // namespace ecsg
