// stencil.cu -- velocity and stress updates of one uniform sub-grid (radius 1).
//
// Both kernels are HBM-bound sweeps.  A CTA covers a 32 x TY tile of (x,y)
// columns and marches down z; the z-neighbours a cell needs stay in registers
// from the previous plane, the x/y neighbours come from L1 (the tile's own rows)
// or L2 (the one-row halo of the neighbouring tile).  Every compulsory word is
// read from HBM once per sweep.
//
// Arithmetic uses non-contracted rounded operations in the reference's order,
// so the double instantiation reproduces update_vel.cpp / update_stress.cpp bit
// for bit; the float instantiation is the production path.
#include "ecsg_device.cuh"

namespace ecsg {

constexpr int TX = 32;
constexpr int TY = 8;

// ---------------------------------------------------------------------------
// Velocity update, update_vel.cpp:20-69 (radius 1).
//   vx: x,y walls excluded, z in [zt, nz-bottom]
//   vy: z in [zt, nz-bottom]
//   vz: y walls excluded, z in [0, nz-1]
// zt = 1 only on the top grid with a rigid top (update_vel.cpp:17-18).
// When vcopy[0] is non-null the pre-update velocities are written there
// (the energy's v^{n-1/2}, main.cpp:173-176).
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(TX *TY) vel_kernel(GridDev<T> G, int zt, int bottom, int zchunk, T *vc0, T *vc1, T *vc2)
{
    const Geo &g = G.g;
    const int ix = blockIdx.x * TX + threadIdx.x;
    const int iy = blockIdx.y * TY + threadIdx.y;
    if (ix > g.nx || iy > g.ny) return;
    const int z0 = blockIdx.z * zchunk;
    const int z1 = min(g.nz, z0 + zchunk - 1);
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int sx = 1, sy = g.px, sz = g.px * g.py;

    T *__restrict__ vx = G.f[VX];
    T *__restrict__ vy = G.f[VY];
    T *__restrict__ vz = G.f[VZ];
    const T *__restrict__ sxx = G.f[SXX];
    const T *__restrict__ syy = G.f[SYY];
    const T *__restrict__ szz = G.f[SZZ];
    const T *__restrict__ syz = G.f[SYZ];
    const T *__restrict__ sxz = G.f[SXZ];
    const T *__restrict__ sxy = G.f[SXY];
    const T *__restrict__ b = G.b;
    const T k0 = G.k[0], k1 = G.k[1], k2 = G.k[2];
    const T q = T(0.25);

    const bool xin = ix >= 1 && ix <= nx - 1;
    const bool yin = iy >= 1 && iy <= ny - 1;
    const bool xs = ix <= nx - 1;
    const bool ys = iy <= ny - 1;
    const bool do_vx = xin && yin;
    const bool do_vy = xs && ys;
    const bool do_vz = xs && yin;
    if (!(do_vy || do_vz)) return;   // x = nx or y = ny: nothing to update (vx needs both < n too)
    const int zb = nz - bottom;

    int p = g.idx(ix, iy, z0);
    T sxz_m = sxz[p - sz];
    T syz_m = syz[p - sz];
    T szz_c = szz[p];
    T b00 = b[p], b10 = b[p + sx];
    const bool vc = vc0 != nullptr;

    for (int iz = z0; iz <= z1; iz++, p += sz) {
        const T sxz_c = sxz[p];
        const T syz_c = syz[p];
        const T szz_n = szz[p + sz];
        const T b00n = b[p + sz], b10n = b[p + sz + sx];
        const T sxy_c = sxy[p];
        if (do_vx && iz >= zt && iz <= zb) {
            const T d = add_(add_(mul_(k0, sub_(sxx[p], sxx[p - sx])),
                                  mul_(k1, sub_(sxy_c, sxy[p - sy]))),
                             mul_(k2, sub_(sxz_c, sxz_m)));
            const T v = vx[p];
            if (vc) vc0[p] = v;
            vx[p] = add_(v, mul_(b00, d));
        }
        if (do_vy && iz >= zt && iz <= zb) {
            const T bb = mul_(q, add_(add_(add_(b00, b10), b[p + sy]), b[p + sy + sx]));
            const T d = add_(add_(mul_(k0, sub_(sxy[p + sx], sxy_c)),
                                  mul_(k2, sub_(syz_c, syz_m))),
                             mul_(k1, sub_(syy[p + sy], syy[p])));
            const T v = vy[p];
            if (vc) vc1[p] = v;
            vy[p] = add_(v, mul_(bb, d));
        }
        if (do_vz && iz <= nz - 1) {
            const T bb = mul_(q, add_(add_(add_(b00, b00n), b10), b10n));
            const T d = add_(add_(mul_(k0, sub_(sxz[p + sx], sxz_c)),
                                  mul_(k2, sub_(szz_n, szz_c))),
                             mul_(k1, sub_(syz_c, syz[p - sy])));
            const T v = vz[p];
            if (vc) vc2[p] = v;
            vz[p] = add_(v, mul_(bb, d));
        }
        sxz_m = sxz_c;
        syz_m = syz_c;
        szz_c = szz_n;
        b00 = b00n;
        b10 = b10n;
    }
}

// ---------------------------------------------------------------------------
// Odd velocity mirrors into the halos for radius 1 (update_vel.cpp:73-246).
// The reference runs them in sequence; two phases reproduce that order:
//   phase 0: vz top (rigid top only), vz bottom (bottom grid), vz x-start/end,
//            vy x-start/end over vz's y-extent [0, ny] (this reads the y = ny
//            halo of vy before phase 1 rewrites it, as in the reference)
//   phase 1: vy y-start/end over vz's z-extent [0, nz-1], or over vy's own
//            extent [0, nz] when mirror_fix is set (then the updated interface
//            plane of a fine grid gets its wall mirror and the composite
//            energy is conserved exactly)
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void vel_mirror_body(const Geo &g, T *vy, T *vz, int phase, int top_rigid, int bottom,
                                                int mirror_fix)
{
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (phase == 0) {
        const int64_t nA = top_rigid ? (int64_t)(ny + 1) * nx : 0;
        const int64_t nB = bottom ? (int64_t)(ny + 1) * nx : 0;
        const int64_t nC = (int64_t)nz * (ny + 1);
        const int64_t nD = (int64_t)(nz + 1) * (ny + 1);
        if (t < nA) { int ix = t % nx, iy = t / nx; vz[g.idx(ix, iy, -1)] = -vz[g.idx(ix, iy, 0)]; return; }
        t -= nA;
        if (t < nB) { int ix = t % nx, iy = t / nx; vz[g.idx(ix, iy, nz)] = -vz[g.idx(ix, iy, nz - 1)]; return; }
        t -= nB;
        if (t < nC) { int iy = t % (ny + 1), iz = t / (ny + 1); vz[g.idx(-1, iy, iz)] = -vz[g.idx(0, iy, iz)]; return; }
        t -= nC;
        if (t < nC) { int iy = t % (ny + 1), iz = t / (ny + 1); vz[g.idx(nx, iy, iz)] = -vz[g.idx(nx - 1, iy, iz)]; return; }
        t -= nC;
        if (t < nD) { int iy = t % (ny + 1), iz = t / (ny + 1); vy[g.idx(-1, iy, iz)] = -vy[g.idx(0, iy, iz)]; return; }
        t -= nD;
        if (t < nD) { int iy = t % (ny + 1), iz = t / (ny + 1); vy[g.idx(nx, iy, iz)] = -vy[g.idx(nx - 1, iy, iz)]; return; }
    } else {
        const int64_t nG = (int64_t)(nz + (mirror_fix ? 1 : 0)) * nx;
        if (t < nG) { int ix = t % nx, iz = t / nx; vy[g.idx(ix, -1, iz)] = -vy[g.idx(ix, 0, iz)]; return; }
        t -= nG;
        if (t < nG) { int ix = t % nx, iz = t / nx; vy[g.idx(ix, ny, iz)] = -vy[g.idx(ix, ny - 1, iz)]; return; }
    }
}

template <typename T>
__global__ void vel_mirror_kernel(GridDev<T> G, int phase, int top_rigid, int bottom, int mirror_fix)
{
    vel_mirror_body(G.g, G.f[VY], G.f[VZ], phase, top_rigid, bottom, mirror_fix);
}

// the mirrors of several shots of one grid (shot blockIdx.y)
template <typename T>
struct ShotVel {
    T *vy[kMaxShots], *vz[kMaxShots];
};
template <typename T>
__global__ void vel_mirror_shots_kernel(Geo g, const __grid_constant__ ShotVel<T> P, int phase, int top_rigid, int bottom,
                                        int mirror_fix)
{
    vel_mirror_body(g, P.vy[blockIdx.y], P.vz[blockIdx.y], phase, top_rigid, bottom, mirror_fix);
}

// ---------------------------------------------------------------------------
// Stress update, update_stress.cpp:36-133 (radius 1), with the free-surface
// odd mirrors of syz/sxz (update_stress.cpp:260-277) fused: the thread that
// updates the surface value writes its mirror.
//   normal (sxx,syy,szz): x in [0,nx-1], y in [0,ny], z in [flag, nz]; on the
//                         free surface (flag) row z = 0 updates sxx, syy with
//                         the reduced moduli and leaves szz alone
//   syz: x [0,nx-1], y [0,ny-1], z [0,nz-1]
//   sxz: x [0,nx],   y [0,ny],   z [0,nz-1]
//   sxy: x [0,nx],   y [0,ny-1], z [0,nz]
// ---------------------------------------------------------------------------
template <typename T, int MED>
struct Stiff;

template <typename T>
struct Stiff<T, MED_ISO5> {
    T c11, c22, c33, c23, c13, c12;
    __device__ __forceinline__ void load(const GridDev<T> &G, int p)
    {
        c11 = c22 = c33 = ldg(G.c[0] + p);
        c23 = c13 = c12 = ldg(G.c[1] + p);
    }
    __device__ __forceinline__ static T c44(const GridDev<T> &G, int p) { return ldg(G.c[2] + p); }
    __device__ __forceinline__ static T c55(const GridDev<T> &G, int p) { return ldg(G.c[3] + p); }
    __device__ __forceinline__ static T c66(const GridDev<T> &G, int p) { return ldg(G.c[4] + p); }
};

template <typename T>
struct Stiff<T, MED_ORTHO9> {
    T c11, c22, c33, c23, c13, c12;
    __device__ __forceinline__ void load(const GridDev<T> &G, int p)
    {
        c11 = ldg(G.c[0] + p); c22 = ldg(G.c[1] + p); c33 = ldg(G.c[2] + p);
        c23 = ldg(G.c[3] + p); c13 = ldg(G.c[4] + p); c12 = ldg(G.c[5] + p);
    }
    __device__ __forceinline__ static T c44(const GridDev<T> &G, int p) { return ldg(G.c[6] + p); }
    __device__ __forceinline__ static T c55(const GridDev<T> &G, int p) { return ldg(G.c[7] + p); }
    __device__ __forceinline__ static T c66(const GridDev<T> &G, int p) { return ldg(G.c[8] + p); }
};

template <typename T, int MED>
__global__ void __launch_bounds__(TX *TY) stress_kernel(GridDev<T> G, int flag, int zchunk)
{
    const Geo &g = G.g;
    const int i0 = blockIdx.x * TX + threadIdx.x;
    const int i1 = blockIdx.y * TY + threadIdx.y;
    if (i0 > g.nx || i1 > g.ny) return;
    const int z0 = blockIdx.z * zchunk;
    const int z1 = min(g.nz, z0 + zchunk - 1);
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int sx = 1, sy = g.px, sz = g.px * g.py;

    const T *__restrict__ vx = G.f[VX];
    const T *__restrict__ vy = G.f[VY];
    const T *__restrict__ vz = G.f[VZ];
    T *__restrict__ sxx = G.f[SXX];
    T *__restrict__ syy = G.f[SYY];
    T *__restrict__ szz = G.f[SZZ];
    T *__restrict__ syz = G.f[SYZ];
    T *__restrict__ sxz = G.f[SXZ];
    T *__restrict__ sxy = G.f[SXY];
    const T k0 = G.k[0], k1 = G.k[1], k2 = G.k[2];
    const T half = T(0.5);

    const bool do_n = i0 <= nx - 1;
    const bool do_yz = i0 <= nx - 1 && i1 <= ny - 1;
    const bool do_xy = i1 <= ny - 1;
    const bool mir_xz = flag && i0 >= 1 && i0 <= nx - 1 && i1 >= 1 && i1 <= ny - 1;

    int p = g.idx(i0, i1, z0);
    T vz_m = vz[p - sz];
    T vx_c = vx[p];
    T vy_c = vy[p];

    for (int iz = z0; iz <= z1; iz++, p += sz) {
        const T vz_c = vz[p];
        const T vx_n = vx[p + sz];
        const T vy_n = vy[p + sz];
        if (do_n) {
            const T dvx = sub_(vx[p + sx], vx_c);
            const T dvy = sub_(vy_c, vy[p - sy]);
            Stiff<T, MED> C;
            C.load(G, p);
            if (flag && iz == 0) {
                // free surface: szz held, reduced moduli c_ij - c_i3 c_j3 / c33
                const T a11 = sub_(C.c11, div_(mul_(C.c13, C.c13), C.c33));
                const T a12 = sub_(C.c12, div_(mul_(C.c13, C.c23), C.c33));
                const T a21 = sub_(C.c12, div_(mul_(C.c23, C.c13), C.c33));
                const T a22 = sub_(C.c22, div_(mul_(C.c23, C.c23), C.c33));
                sxx[p] = add_(sxx[p], add_(mul_(mul_(a11, k0), dvx), mul_(mul_(a12, k1), dvy)));
                syy[p] = add_(syy[p], add_(mul_(mul_(a21, k0), dvx), mul_(mul_(a22, k1), dvy)));
            } else {
                const T dvz = sub_(vz_c, vz_m);
                sxx[p] = add_(sxx[p], add_(add_(mul_(mul_(C.c11, k0), dvx), mul_(mul_(C.c12, k1), dvy)),
                                           mul_(mul_(C.c13, k2), dvz)));
                syy[p] = add_(syy[p], add_(add_(mul_(mul_(C.c12, k0), dvx), mul_(mul_(C.c22, k1), dvy)),
                                           mul_(mul_(C.c23, k2), dvz)));
                szz[p] = add_(szz[p], add_(add_(mul_(mul_(C.c13, k0), dvx), mul_(mul_(C.c23, k1), dvy)),
                                           mul_(mul_(C.c33, k2), dvz)));
            }
        }
        if (do_yz && iz <= nz - 1) {
            const T s = add_(syz[p], mul_(mul_(half, Stiff<T, MED>::c44(G, p)),
                                          add_(mul_(k2, sub_(vy_n, vy_c)), mul_(k1, sub_(vz[p + sy], vz_c)))));
            syz[p] = s;
            if (flag && iz == 0) syz[p - sz] = -s;
        }
        if (iz <= nz - 1) {
            const T s = add_(sxz[p], mul_(mul_(half, Stiff<T, MED>::c55(G, p)),
                                          add_(mul_(k2, sub_(vx_n, vx_c)), mul_(k0, sub_(vz_c, vz[p - sx])))));
            sxz[p] = s;
            if (mir_xz && iz == 0) sxz[p - sz] = -s;
        }
        if (do_xy) {
            sxy[p] = add_(sxy[p], mul_(mul_(half, Stiff<T, MED>::c66(G, p)),
                                       add_(mul_(k1, sub_(vx[p + sy], vx_c)), mul_(k0, sub_(vy_c, vy[p - sx])))));
        }
        vz_m = vz_c;
        vx_c = vx_n;
        vy_c = vy_n;
    }
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
static int pick_zchunk(const Geo &g, int sms)
{
    const int64_t cols = (int64_t)((g.nx + 1 + TX - 1) / TX) * ((g.ny + 1 + TY - 1) / TY);
    const int64_t want = (int64_t)sms * 8;   // CTAs for a few waves
    int nchunk = (int)((want + cols - 1) / cols);
    if (nchunk < 1) nchunk = 1;
    if (nchunk > g.nz + 1) nchunk = g.nz + 1;
    return (g.nz + 1 + nchunk - 1) / nchunk;
}

template <typename T>
cudaError_t launch_vel(const GridDev<T> &G, int top, int bottom, int top_bc, T *const vcopy[3], int sms, cudaStream_t st)
{
    const Geo &g = G.g;
    const int zt = (top && top_bc != 1) ? 1 : 0;
    const int zc = pick_zchunk(g, sms);
    dim3 blk(TX, TY), grd((g.nx + TX - 1) / TX, (g.ny + TY - 1) / TY, (g.nz + 1 + zc - 1) / zc);
    vel_kernel<T><<<grd, blk, 0, st>>>(G, zt, bottom, zc, vcopy ? vcopy[0] : nullptr, vcopy ? vcopy[1] : nullptr,
                                      vcopy ? vcopy[2] : nullptr);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_vel_mirror(const GridDev<T> &G, int top, int bottom, int top_bc, int mirror_fix, cudaStream_t st)
{
    const Geo &g = G.g;
    const int top_rigid = (top && top_bc != 1) ? 1 : 0;
    const int64_t n0 = (int64_t)(top_rigid + bottom) * (g.ny + 1) * g.nx + 2LL * g.nz * (g.ny + 1)
                     + 2LL * (g.nz + 1) * (g.ny + 1);
    const int64_t n1 = 2LL * (g.nz + (mirror_fix ? 1 : 0)) * g.nx;
    vel_mirror_kernel<T><<<(unsigned)((n0 + 255) / 256), 256, 0, st>>>(G, 0, top_rigid, bottom, mirror_fix);
    vel_mirror_kernel<T><<<(unsigned)((n1 + 255) / 256), 256, 0, st>>>(G, 1, top_rigid, bottom, mirror_fix);
    return cudaGetLastError();
}

// launch_vel_mirror for ns shots of one grid (vy[s], vz[s] the shot's fields)
template <typename T>
cudaError_t launch_vel_mirror_shots(const Geo &g, T *const *vy, T *const *vz, int ns, int top, int bottom, int top_bc,
                                    int mirror_fix, cudaStream_t st)
{
    if (ns < 1 || ns > kMaxShots) return cudaErrorInvalidValue;
    ShotVel<T> P;
    for (int s = 0; s < ns; s++) {
        P.vy[s] = vy[s];
        P.vz[s] = vz[s];
    }
    const int top_rigid = (top && top_bc != 1) ? 1 : 0;
    const int64_t n0 = (int64_t)(top_rigid + bottom) * (g.ny + 1) * g.nx + 2LL * g.nz * (g.ny + 1)
                     + 2LL * (g.nz + 1) * (g.ny + 1);
    const int64_t n1 = 2LL * (g.nz + (mirror_fix ? 1 : 0)) * g.nx;
    vel_mirror_shots_kernel<T><<<dim3((unsigned)((n0 + 255) / 256), ns), 256, 0, st>>>(g, P, 0, top_rigid, bottom, mirror_fix);
    vel_mirror_shots_kernel<T><<<dim3((unsigned)((n1 + 255) / 256), ns), 256, 0, st>>>(g, P, 1, top_rigid, bottom, mirror_fix);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_stress(const GridDev<T> &G, int medium, int top, int top_bc, int sms, cudaStream_t st)
{
    const Geo &g = G.g;
    const int flag = (top && top_bc) ? 1 : 0;
    const int zc = pick_zchunk(g, sms);
    dim3 blk(TX, TY), grd((g.nx + 1 + TX - 1) / TX, (g.ny + 1 + TY - 1) / TY, (g.nz + 1 + zc - 1) / zc);
    if (medium == MED_ISO5)
        stress_kernel<T, MED_ISO5><<<grd, blk, 0, st>>>(G, flag, zc);
    else if (medium == MED_ORTHO9)
        stress_kernel<T, MED_ORTHO9><<<grd, blk, 0, st>>>(G, flag, zc);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

template cudaError_t launch_vel<float>(const GridDev<float> &, int, int, int, float *const[3], int, cudaStream_t);
template cudaError_t launch_vel<double>(const GridDev<double> &, int, int, int, double *const[3], int, cudaStream_t);
template cudaError_t launch_vel_mirror<float>(const GridDev<float> &, int, int, int, int, cudaStream_t);
template cudaError_t launch_vel_mirror<double>(const GridDev<double> &, int, int, int, int, cudaStream_t);
template cudaError_t launch_vel_mirror_shots<float>(const Geo &, float *const *, float *const *, int, int, int, int, int,
                                                    cudaStream_t);
template cudaError_t launch_vel_mirror_shots<double>(const Geo &, double *const *, double *const *, int, int, int, int,
                                                     int, cudaStream_t);
template cudaError_t launch_stress<float>(const GridDev<float> &, int, int, int, int, cudaStream_t);
template cudaError_t launch_stress<double>(const GridDev<double> &, int, int, int, int, cudaStream_t);

} // namespace ecsg
