// stencil_r.cu -- velocity and stress updates of one grid for stencil radius
// R = 2..6: update_vel.cpp:4-249 and update_stress.cpp:4-311 with their radius
// loops, coefficients fd[r]*dt/h from init_del_fdcoeff.cpp:38-85.
//
// The reference adds the R terms of a point one radius at a time (loop order
// z, y, r, x): v += b * (k0[r] D0 + k1[r] D1 + k2[r] D2) for r = 0 .. R-1.
// These kernels keep that order per point (the file is compiled without FMA
// contraction), so the double instantiation is bit-exact with the reference;
// the float one is the single-precision path.  One thread per (x, y) column
// and z-chunk; the +-R neighbours come through L1/L2.
//
// Halo mirrors are listed on the host as faces (one field, one mirrored axis,
// a radius range, the ranges of the other two axes) and run by one kernel per
// phase.  Within a phase every face writes halo points no other face writes,
// and reads points no face of the phase writes.  The velocity mirrors need two
// phases: the vy x-mirrors run over vz's y-extent [0, ny] and so read vy's
// y = ny halo row, which the later y-end mirror rewrites
// (update_vel.cpp:137-165 before :233-246).
#include "ecsg_device.cuh"

#include <vector>

namespace ecsg {

constexpr int kMaxR = 6;

template <typename T>
struct CoefR {
    T k[3][kMaxR];
};

struct MirrorFace {
    int field, axis, base, r0, r1;
    int ds, doff, ss, soff;   // mirrored coordinate: dst = base + ds*r + doff, src = base + ss*r + soff
    int sign;                 // +1 copy (even), -1 negate (odd)
    int lo[2], hi[2];         // the other two axes, lower axis first
};
constexpr int kMaxFaces = 12;
struct MirrorList {
    int n;
    MirrorFace f[kMaxFaces];
};

// ---------------------------------------------------------------------------
// velocity (update_vel.cpp:20-69): vx x,y walls excluded, z in [zt, nz-bottom];
// vy z in [zt, nz-bottom]; vz y walls excluded, z in [0, nz-1]
// ---------------------------------------------------------------------------
template <typename T, int R>
__global__ void __launch_bounds__(256) vel_r_kernel(GridDev<T> G, CoefR<T> K, int zt, int bottom, int zchunk,
                                                    T *vc0, T *vc1, T *vc2)
{
    const Geo &g = G.g;
    const int ix = blockIdx.x * 32 + threadIdx.x;
    const int iy = blockIdx.y * 8 + threadIdx.y;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (ix > nx - 1 || iy > ny) return;
    const int sy = g.px, sz = g.px * g.py;
    T *vx = G.f[VX], *vy = G.f[VY], *vz = G.f[VZ];
    const T *sxx = G.f[SXX], *syy = G.f[SYY], *szz = G.f[SZZ];
    const T *syz = G.f[SYZ], *sxz = G.f[SXZ], *sxy = G.f[SXY], *b = G.b;
    const bool do_vx = ix >= 1 && iy >= 1 && iy <= ny - 1;
    const bool do_vy = iy <= ny - 1;
    const bool do_vz = iy >= 1 && iy <= ny - 1;
    const int z0 = blockIdx.z * zchunk, z1 = min(nz, z0 + zchunk - 1);
    const T q = (T)0.25;
    for (int iz = z0; iz <= z1; iz++) {
        const int p = g.idx(ix, iy, iz);
        if (do_vx && iz >= zt && iz <= nz - bottom) {
            T v = vx[p];
            if (vc0) vc0[p] = v;
            const T bb = b[p];
#pragma unroll
            for (int r = 0; r < R; r++)
                v = v + bb * (K.k[0][r] * (sxx[p + r] - sxx[p - r - 1]) + K.k[1][r] * (sxy[p + r * sy] - sxy[p - (r + 1) * sy])
                              + K.k[2][r] * (sxz[p + r * sz] - sxz[p - (r + 1) * sz]));
            vx[p] = v;
        }
        if (do_vy && iz >= zt && iz <= nz - bottom) {
            T v = vy[p];
            if (vc1) vc1[p] = v;
#pragma unroll
            for (int r = 0; r < R; r++)
                v = v + q * (b[p] + b[p + 1] + b[p + sy] + b[p + sy + 1])
                            * (K.k[0][r] * (sxy[p + r + 1] - sxy[p - r]) + K.k[2][r] * (syz[p + r * sz] - syz[p - (r + 1) * sz])
                               + K.k[1][r] * (syy[p + (r + 1) * sy] - syy[p - r * sy]));
            vy[p] = v;
        }
        if (do_vz && iz <= nz - 1) {
            T v = vz[p];
            if (vc2) vc2[p] = v;
#pragma unroll
            for (int r = 0; r < R; r++)
                v = v + q * (b[p] + b[p + sz] + b[p + 1] + b[p + 1 + sz])
                            * (K.k[0][r] * (sxz[p + r + 1] - sxz[p - r]) + K.k[2][r] * (szz[p + (r + 1) * sz] - szz[p - r * sz])
                               + K.k[1][r] * (syz[p + r * sy] - syz[p - (r + 1) * sy]));
            vz[p] = v;
        }
    }
}

// ---------------------------------------------------------------------------
// stress (update_stress.cpp:36-133): normal stresses with the free-surface
// row (flag) at z = 0, then the three shear stresses
// ---------------------------------------------------------------------------
template <typename T, int MED>
struct StiffR;
template <typename T>
struct StiffR<T, MED_ISO5> {
    __device__ static void normal(const GridDev<T> &G, int p, T &c11, T &c22, T &c33, T &c23, T &c13, T &c12)
    {
        c11 = c22 = c33 = G.c[0][p];
        c23 = c13 = c12 = G.c[1][p];
    }
    __device__ static T shear(const GridDev<T> &G, int k, int p) { return G.c[2 + k][p]; }
};
template <typename T>
struct StiffR<T, MED_ORTHO9> {
    __device__ static void normal(const GridDev<T> &G, int p, T &c11, T &c22, T &c33, T &c23, T &c13, T &c12)
    {
        c11 = G.c[0][p]; c22 = G.c[1][p]; c33 = G.c[2][p];
        c23 = G.c[3][p]; c13 = G.c[4][p]; c12 = G.c[5][p];
    }
    __device__ static T shear(const GridDev<T> &G, int k, int p) { return G.c[6 + k][p]; }
};

template <typename T, int R, int MED>
__global__ void __launch_bounds__(256) stress_r_kernel(GridDev<T> G, CoefR<T> K, int flag, int zchunk)
{
    const Geo &g = G.g;
    const int ix = blockIdx.x * 32 + threadIdx.x;
    const int iy = blockIdx.y * 8 + threadIdx.y;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    if (ix > nx || iy > ny) return;
    const int sy = g.px, sz = g.px * g.py;
    const T *vx = G.f[VX], *vy = G.f[VY], *vz = G.f[VZ];
    T *sxx = G.f[SXX], *syy = G.f[SYY], *szz = G.f[SZZ], *syz = G.f[SYZ], *sxz = G.f[SXZ], *sxy = G.f[SXY];
    const T h = (T)0.5;
    const int z0 = blockIdx.z * zchunk, z1 = min(nz, z0 + zchunk - 1);
    for (int iz = z0; iz <= z1; iz++) {
        const int p = g.idx(ix, iy, iz);
        if (ix <= nx - 1) {   // normal stresses at (1,0,0): x < nx, y <= ny, z <= nz
            T c11, c22, c33, c23, c13, c12;
            StiffR<T, MED>::normal(G, p, c11, c22, c33, c23, c13, c12);
            T a = sxx[p], bq = syy[p];
            if (flag && iz == 0) {
#pragma unroll
                for (int r = 0; r < R; r++) {
                    const T dvx = vx[p + r + 1] - vx[p - r];
                    const T dvy = vy[p + r * sy] - vy[p - (r + 1) * sy];
                    a = a + ((c11 - c13 * c13 / c33) * K.k[0][r] * dvx + (c12 - c13 * c23 / c33) * K.k[1][r] * dvy);
                    bq = bq + ((c12 - c23 * c13 / c33) * K.k[0][r] * dvx + (c22 - c23 * c23 / c33) * K.k[1][r] * dvy);
                }
            } else {
                T c = szz[p];
#pragma unroll
                for (int r = 0; r < R; r++) {
                    const T dvx = vx[p + r + 1] - vx[p - r];
                    const T dvy = vy[p + r * sy] - vy[p - (r + 1) * sy];
                    const T dvz = vz[p + r * sz] - vz[p - (r + 1) * sz];
                    a = a + (c11 * K.k[0][r] * dvx + c12 * K.k[1][r] * dvy + c13 * K.k[2][r] * dvz);
                    bq = bq + (c12 * K.k[0][r] * dvx + c22 * K.k[1][r] * dvy + c23 * K.k[2][r] * dvz);
                    c = c + (c13 * K.k[0][r] * dvx + c23 * K.k[1][r] * dvy + c33 * K.k[2][r] * dvz);
                }
                szz[p] = c;
            }
            sxx[p] = a;
            syy[p] = bq;
        }
        if (ix <= nx - 1 && iy <= ny - 1 && iz <= nz - 1) {   // syz at (1,1,1)
            const T c44 = StiffR<T, MED>::shear(G, 0, p);
            T v = syz[p];
#pragma unroll
            for (int r = 0; r < R; r++)
                v = v + h * c44 * (K.k[2][r] * (vy[p + (r + 1) * sz] - vy[p - r * sz]) + K.k[1][r] * (vz[p + (r + 1) * sy] - vz[p - r * sy]));
            syz[p] = v;
        }
        if (iz <= nz - 1) {   // sxz at (0,0,1)
            const T c55 = StiffR<T, MED>::shear(G, 1, p);
            T v = sxz[p];
#pragma unroll
            for (int r = 0; r < R; r++)
                v = v + h * c55 * (K.k[2][r] * (vx[p + (r + 1) * sz] - vx[p - r * sz]) + K.k[0][r] * (vz[p + r] - vz[p - r - 1]));
            sxz[p] = v;
        }
        if (iy <= ny - 1) {   // sxy at (0,1,0)
            const T c66 = StiffR<T, MED>::shear(G, 2, p);
            T v = sxy[p];
#pragma unroll
            for (int r = 0; r < R; r++)
                v = v + h * c66 * (K.k[1][r] * (vx[p + (r + 1) * sy] - vx[p - r * sy]) + K.k[0][r] * (vy[p + r] - vy[p - r - 1]));
            sxy[p] = v;
        }
    }
}

// ---------------------------------------------------------------------------
// mirrors
// ---------------------------------------------------------------------------
template <typename T>
__global__ void mirror_r_kernel(GridDev<T> G, MirrorList L)
{
    const MirrorFace &f = L.f[blockIdx.y];
    const int nr = f.r1 - f.r0 + 1, n0 = f.hi[0] - f.lo[0] + 1, n1 = f.hi[1] - f.lo[1] + 1;
    if (nr <= 0 || n0 <= 0 || n1 <= 0) return;
    const int o0 = f.axis == 0 ? 1 : 0, o1 = f.axis == 2 ? 1 : 2;
    T *a = G.f[f.field];
    const int64_t total = (int64_t)nr * n0 * n1;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < total; t += (int64_t)gridDim.x * blockDim.x) {
        const int c0 = f.lo[0] + (int)(t % n0);
        const int64_t rest = t / n0;
        const int c1 = f.lo[1] + (int)(rest % n1);
        const int r = f.r0 + (int)(rest / n1);
        int d[3], s[3];
        d[o0] = s[o0] = c0;
        d[o1] = s[o1] = c1;
        d[f.axis] = f.base + f.ds * r + f.doff;
        s[f.axis] = f.base + f.ss * r + f.soff;
        const T v = a[G.g.idx(s[0], s[1], s[2])];
        a[G.g.idx(d[0], d[1], d[2])] = f.sign < 0 ? -v : v;
    }
}

namespace {

// last index of each component per axis (positions of init_del_sim.cpp:14-24)
void ends(const Geo &g, int k, int e[3])
{
    static const int pos[9][3] = {{0, 0, 0}, {1, 1, 0}, {1, 0, 1}, {1, 0, 0}, {1, 0, 0},
                                  {1, 0, 0}, {1, 1, 1}, {0, 0, 1}, {0, 1, 0}};
    const int n[3] = {g.nx, g.ny, g.nz};
    for (int d = 0; d < 3; d++) e[d] = n[d] - pos[k][d];
}

struct Builder {
    MirrorList L{};
    bool ok = true;
    // face of field k mirrored along axis; other axes' ranges [lo, hi] in increasing axis order
    void add(int k, int axis, int base, int r0, int r1, int ds, int doff, int ss, int soff, int sign, int lo0, int hi0,
             int lo1, int hi1)
    {
        if (r1 < r0) return;
        if (L.n >= kMaxFaces) { ok = false; return; }
        MirrorFace &f = L.f[L.n++];
        f.field = k; f.axis = axis; f.base = base; f.r0 = r0; f.r1 = r1;
        f.ds = ds; f.doff = doff; f.ss = ss; f.soff = soff; f.sign = sign;
        f.lo[0] = lo0; f.hi[0] = hi0; f.lo[1] = lo1; f.hi[1] = hi1;
    }
};

template <typename T>
cudaError_t run_faces(const GridDev<T> &G, const MirrorList &L, cudaStream_t st)
{
    if (L.n == 0) return cudaSuccess;
    int64_t most = 0;
    for (int i = 0; i < L.n; i++) {
        const MirrorFace &f = L.f[i];
        const int64_t c = (int64_t)(f.r1 - f.r0 + 1) * (f.hi[0] - f.lo[0] + 1) * (f.hi[1] - f.lo[1] + 1);
        if (c > most) most = c;
    }
    int blocks = (int)((most + 255) / 256);
    if (blocks > 1024) blocks = 1024;
    if (blocks < 1) blocks = 1;
    mirror_r_kernel<T><<<dim3(blocks, L.n), 256, 0, st>>>(G, L);
    return cudaGetLastError();
}

// zchunk for the sweeps: enough CTAs for the 148 SMs
int zchunk_for(const Geo &g)
{
    const int64_t cols = (int64_t)((g.nx + 1 + 31) / 32) * ((g.ny + 1 + 7) / 8);
    int nchunk = (int)((4 * 148 + cols - 1) / cols);
    if (nchunk < 1) nchunk = 1;
    if (nchunk > g.nz + 1) nchunk = g.nz + 1;
    return (g.nz + 1 + nchunk - 1) / nchunk;
}

} // namespace

// Coefficients fd[r]*dt/h per dimension (init_del_fdcoeff.cpp:7-22, 38-85)
bool fd_coefficients(int R, double dt, const double h[3], double k[3][kMaxR])
{
    static const double tab[6][6] = {
        {1.0},
        {9.0 / 8, -1.0 / 24},
        {75.0 / 64, -25.0 / 384, 3.0 / 640},
        {1225.0 / 1024, -245.0 / 3072, 49.0 / 5120, -5.0 / 7168},
        {711.0 / 587, -158.0 / 1761, 296.0 / 21383, -25.0 / 14159, 17.0 / 143243},
        {1225.0 / 1003, -338.0 / 3487, 35.0 / 2006, -127.0 / 42800, 19.0 / 52924, -6.0 / 274627}};
    if (R < 1 || R > kMaxR) return false;
    for (int d = 0; d < 3; d++)
        for (int r = 0; r < kMaxR; r++) k[d][r] = r < R ? tab[R - 1][r] * dt / h[d] : 0.0;
    return true;
}

template <typename T>
static CoefR<T> coef_t(const double k[3][kMaxR])
{
    CoefR<T> K;
    for (int d = 0; d < 3; d++)
        for (int r = 0; r < kMaxR; r++) K.k[d][r] = (T)k[d][r];
    return K;
}

template <typename T>
cudaError_t launch_vel_r(const GridDev<T> &G, const double k[3][kMaxR], int R, int top, int bottom, int top_bc,
                         int mirror_fix, T *const vc[3], cudaStream_t st)
{
    const Geo &g = G.g;
    if (top && top_bc == 1) top = 0;   // free surface: the top plane is updated (update_vel.cpp:17-18)
    const int zc = zchunk_for(g);
    dim3 blk(32, 8), grd((g.nx + 31) / 32, (g.ny + 1 + 7) / 8, (g.nz + 1 + zc - 1) / zc);
    const CoefR<T> K = coef_t<T>(k);
    T *v0 = vc ? vc[0] : nullptr, *v1 = vc ? vc[1] : nullptr, *v2 = vc ? vc[2] : nullptr;
    switch (R) {
    case 2: vel_r_kernel<T, 2><<<grd, blk, 0, st>>>(G, K, top, bottom, zc, v0, v1, v2); break;
    case 3: vel_r_kernel<T, 3><<<grd, blk, 0, st>>>(G, K, top, bottom, zc, v0, v1, v2); break;
    case 4: vel_r_kernel<T, 4><<<grd, blk, 0, st>>>(G, K, top, bottom, zc, v0, v1, v2); break;
    case 5: vel_r_kernel<T, 5><<<grd, blk, 0, st>>>(G, K, top, bottom, zc, v0, v1, v2); break;
    case 6: vel_r_kernel<T, 6><<<grd, blk, 0, st>>>(G, K, top, bottom, zc, v0, v1, v2); break;
    default: return cudaErrorInvalidValue;
    }
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;

    // odd mirrors, update_vel.cpp:73-246 (faces as the reference's loops run them)
    int ex[3], ey[3], ez[3];
    ends(g, VX, ex);
    ends(g, VY, ey);
    ends(g, VZ, ez);
    Builder A, B;
    if (top) {
        A.add(VZ, 2, 0, 1, R - top_bc, -1, 0, 1, -1, -1, 0, ez[0], 0, ez[1]);
        A.add(VX, 2, 0, 1, R - 1, -1, 0, 1, 0, -1, 0, ez[0], 0, ex[1]);
        A.add(VY, 2, 0, 1, R - 1, -1, 0, 1, 0, -1, 0, ez[0], 0, ey[1]);
    }
    if (bottom) {
        A.add(VZ, 2, ez[2], 1, R, 1, 0, -1, 1, -1, 0, ez[0], 0, ez[1]);
        A.add(VX, 2, ex[2], 1, R - 1, 1, 0, -1, 0, -1, 0, ez[0], 0, ex[1]);
        A.add(VY, 2, ey[2], 1, R - 1, 1, 0, -1, 0, -1, 0, ez[0], 0, ey[1]);
    }
    // x start / end: other axes (y, z)
    A.add(VZ, 0, 0, 1, R, -1, 0, 1, -1, -1, 0, ez[1], 0, ez[2]);
    A.add(VX, 0, 0, 1, R - 1, -1, 0, 1, 0, -1, 0, ez[1], 0, ex[2]);
    A.add(VY, 0, 0, 1, R, -1, 0, 1, -1, -1, 0, ez[1], 0, ey[2]);
    A.add(VZ, 0, ez[0], 1, R, 1, 0, -1, 1, -1, 0, ez[1], 0, ez[2]);
    A.add(VX, 0, ex[0], 1, R - 1, 1, 0, -1, 0, -1, 0, ez[1], 0, ex[2]);
    A.add(VY, 0, ey[0], 1, R, 1, 0, -1, 1, -1, 0, ez[1], 0, ey[2]);
    // y start / end: other axes (x, z)
    const int vyz = mirror_fix ? ey[2] : ez[2];
    B.add(VZ, 1, 0, 1, R - 1, -1, 0, 1, 0, -1, 0, ez[0], 0, ez[2]);
    B.add(VX, 1, 0, 1, R - 1, -1, 0, 1, 0, -1, 0, ex[0], 0, ez[2]);
    B.add(VY, 1, 0, 1, R, -1, 0, 1, -1, -1, 0, ey[0], 0, vyz);
    B.add(VZ, 1, ez[1], 1, R - 1, 1, 0, -1, 0, -1, 0, ez[0], 0, ez[2]);
    B.add(VX, 1, ex[1], 1, R - 1, 1, 0, -1, 0, -1, 0, ex[0], 0, ez[2]);
    B.add(VY, 1, ey[1], 1, R, 1, 0, -1, 1, -1, 0, ey[0], 0, vyz);
    if (!A.ok || !B.ok) return cudaErrorInvalidValue;
    if ((e = run_faces(G, A.L, st)) != cudaSuccess) return e;
    return run_faces(G, B.L, st);
}

template <typename T>
cudaError_t launch_stress_r(const GridDev<T> &G, const double k[3][kMaxR], int R, int medium, int top, int bottom,
                            int top_bc, cudaStream_t st)
{
    const Geo &g = G.g;
    const int flag = (top && top_bc) ? 1 : 0;
    const int zc = zchunk_for(g);
    dim3 blk(32, 8), grd((g.nx + 1 + 31) / 32, (g.ny + 1 + 7) / 8, (g.nz + 1 + zc - 1) / zc);
    const CoefR<T> K = coef_t<T>(k);
#define ECSG_STRESS_R(RR)                                                                                   \
    case RR:                                                                                                \
        if (medium == MED_ISO5) stress_r_kernel<T, RR, MED_ISO5><<<grd, blk, 0, st>>>(G, K, flag, zc);       \
        else stress_r_kernel<T, RR, MED_ORTHO9><<<grd, blk, 0, st>>>(G, K, flag, zc);                        \
        break;
    if (medium != MED_ISO5 && medium != MED_ORTHO9) return cudaErrorInvalidValue;
    switch (R) {
        ECSG_STRESS_R(2)
        ECSG_STRESS_R(3)
        ECSG_STRESS_R(4)
        ECSG_STRESS_R(5)
        ECSG_STRESS_R(6)
    default: return cudaErrorInvalidValue;
    }
#undef ECSG_STRESS_R
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) return e;

    // even mirrors, update_stress.cpp:135-309 (all faces independent)
    int en[3], eyz[3], exz[3], exy[3];
    ends(g, SZZ, en);
    ends(g, SYZ, eyz);
    ends(g, SXZ, exz);
    ends(g, SXY, exy);
    Builder A, B;
    // x start / end: other axes (y, z)
    A.add(SXX, 0, 0, 1, R - 1, -1, 0, 1, -1, 1, 0, en[1], 0, en[2]);
    A.add(SXZ, 0, 0, 1, R - 1, -1, 0, 1, 0, 1, 0, exz[1], 0, exz[2]);
    A.add(SXY, 0, 0, 1, R - 1, -1, 0, 1, 0, 1, 0, exy[1], 0, exy[2]);
    A.add(SXX, 0, en[0], 1, R - 1, 1, 0, -1, 1, 1, 0, en[1], 0, en[2]);
    A.add(SXZ, 0, exz[0], 1, R - 1, 1, 0, -1, 0, 1, 0, exz[1], 0, exz[2]);
    A.add(SXY, 0, exy[0], 1, R - 1, 1, 0, -1, 0, 1, 0, exy[1], 0, exy[2]);
    // y start / end: other axes (x, z)
    A.add(SYY, 1, 0, 1, R - 1, -1, 0, 1, 0, 1, 0, en[0], 0, en[2]);
    A.add(SYZ, 1, 0, 1, R - 1, -1, 0, 1, -1, 1, 0, eyz[0], 0, eyz[2]);
    A.add(SXY, 1, 0, 1, R - 1, -1, 0, 1, -1, 1, 0, exy[0], 0, exy[2]);
    A.add(SYY, 1, en[1], 1, R - 1, 1, 0, -1, 0, 1, 0, en[0], 0, en[2]);
    A.add(SYZ, 1, eyz[1], 1, R - 1, 1, 0, -1, 1, 1, 0, eyz[0], 0, eyz[2]);
    A.add(SXY, 1, exy[1], 1, R - 1, 1, 0, -1, 1, 1, 0, exy[0], 0, exy[2]);
    // top / bottom: other axes (x, y)
    if (top) {
        B.add(SZZ, 2, 0, 1, R - 1, -1, 0, 1, 0, 1, 0, en[0], 1, en[1] - 1);
        B.add(SYZ, 2, 0, 1, R - 1 + flag, -1, 0, 1, -1, 1 - 2 * flag, 0, eyz[0], 0, eyz[1]);
        B.add(SXZ, 2, 0, 1, R - 1 + flag, -1, 0, 1, -1, 1 - 2 * flag, 1, exz[0] - 1, 1, exz[1] - 1);
    }
    if (bottom) {
        B.add(SZZ, 2, en[2], 1, R - 1, 1, 0, -1, 0, 1, 0, en[0], 1, en[1] - 1);
        B.add(SYZ, 2, eyz[2], 1, R - 1, 1, 0, -1, 1, 1, 0, eyz[0], 0, eyz[1]);
        B.add(SXZ, 2, exz[2], 1, R - 1, 1, 0, -1, 1, 1, 1, exz[0] - 1, 1, exz[1] - 1);
    }
    if (!A.ok || !B.ok) return cudaErrorInvalidValue;
    if ((e = run_faces(G, A.L, st)) != cudaSuccess) return e;
    return run_faces(G, B.L, st);
}

#define INST(T)                                                                                              \
    template cudaError_t launch_vel_r<T>(const GridDev<T> &, const double[3][kMaxR], int, int, int, int, int,   \
                                         T *const[3], cudaStream_t);                                         \
    template cudaError_t launch_stress_r<T>(const GridDev<T> &, const double[3][kMaxR], int, int, int, int, int, \
                                            cudaStream_t);
INST(float)
INST(double)
#undef INST

} // namespace ecsg
