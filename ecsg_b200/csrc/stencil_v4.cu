// stencil_v4.cu -- float4-vectorised FP32 velocity and stress sweeps (production path).
//
// Same updates, same per-element operation order and therefore the same bits
// as the scalar kernels of stencil.cu, organised for bandwidth:
//   * one lane owns 4 consecutive x cells: every field access is one 16-byte
//     load or store (rows are 128-byte aligned, x = 0 sits at a multiple of 4),
//     so a warp moves 512 contiguous bytes per instruction and four times more
//     bytes are in flight per issued instruction than in the scalar sweep;
//   * x-neighbours come from the adjacent lane by warp shuffle; only the edge
//     lanes of a warp load one scalar from the neighbouring chunk (L1 hit);
//   * a CTA is 8 warps = 8 rows of 128 cells; it marches down z keeping the
//     z-neighbour planes in registers;
//   * cells of a chunk that the update does not cover are stored back
//     unchanged, so each 16-byte chunk is written whole.
// Lanes whose chunk lies past the last cell an update needs (x0 > nx) load
// from chunk 0 of their row (in bounds, values unused) and store nothing.
#include "ecsg_device.cuh"

namespace ecsg {

constexpr int V4_ROWS = 8;
constexpr unsigned FULL = 0xffffffffu;

struct F4 {
    float e[4];
};

__device__ __forceinline__ F4 ldg4(const float *p)
{
    const float4 v = __ldg(reinterpret_cast<const float4 *>(p));
    return {{v.x, v.y, v.z, v.w}};
}
__device__ __forceinline__ F4 ld4(const float *p)
{
    const float4 v = *reinterpret_cast<const float4 *>(p);
    return {{v.x, v.y, v.z, v.w}};
}
__device__ __forceinline__ void st4(float *p, const F4 &a)
{
    *reinterpret_cast<float4 *>(p) = make_float4(a.e[0], a.e[1], a.e[2], a.e[3]);
}
// element x0-1 of a lane's chunk
__device__ __forceinline__ float left_of(const F4 &a, const float *p, int lane)
{
    float l = __shfl_up_sync(FULL, a.e[3], 1);
    if (lane == 0) l = __ldg(p - 1);
    return l;
}
// element x0+4 of a lane's chunk
__device__ __forceinline__ float right_of(const F4 &a, const float *p, int lane)
{
    float r = __shfl_down_sync(FULL, a.e[0], 1);
    if (lane == 31) r = __ldg(p + 4);
    return r;
}

// ---------------------------------------------------------------------------
// Velocity update (update_vel.cpp:20-69), radius 1; ranges as vel_kernel.
// ---------------------------------------------------------------------------
__global__ void __launch_bounds__(32 * V4_ROWS) vel_kernel_v4(GridDev<float> G, int zt, int bottom, int zchunk,
                                                              float *vc0, float *vc1, float *vc2)
{
    const Geo &g = G.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int lane = threadIdx.x;
    const int iy = blockIdx.y * V4_ROWS + threadIdx.y;
    if (iy > ny - 1) return;   // whole warp: vel updates rows [0, ny-1]
    const int x0 = (blockIdx.x * 32 + lane) * 4;
    const bool act = x0 <= nx;
    const int xc = act ? x0 : 0;
    const int z0 = blockIdx.z * zchunk;
    const int z1 = min(nz, z0 + zchunk - 1);
    const int sy = g.px, sz = g.px * g.py;
    float *__restrict__ vx = G.f[VX];
    float *__restrict__ vy = G.f[VY];
    float *__restrict__ vz = G.f[VZ];
    const float *__restrict__ sxx = G.f[SXX];
    const float *__restrict__ syy = G.f[SYY];
    const float *__restrict__ szz = G.f[SZZ];
    const float *__restrict__ syz = G.f[SYZ];
    const float *__restrict__ sxz = G.f[SXZ];
    const float *__restrict__ sxy = G.f[SXY];
    const float *__restrict__ b = G.b;
    const float k0 = G.k[0], k1 = G.k[1], k2 = G.k[2];
    const float q = 0.25f;
    const bool yin = iy >= 1 && iy <= ny - 1;
    const int zb = nz - bottom;
    bool mx_in[4], mx_s[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        mx_in[i] = x0 + i >= 1 && x0 + i <= nx - 1;
        mx_s[i] = x0 + i <= nx - 1;
    }
    const bool vc = vc0 != nullptr;

    int p = g.idx(xc, iy, z0);
    F4 sxz_m = ldg4(sxz + p - sz);
    F4 syz_m = ldg4(syz + p - sz);
    F4 szz_c = ldg4(szz + p);
    F4 b_c = ldg4(b + p);

    for (int iz = z0; iz <= z1; iz++, p += sz) {
        const F4 sxz_c = ldg4(sxz + p);
        const F4 syz_c = ldg4(syz + p);
        const F4 szz_n = ldg4(szz + p + sz);
        const F4 b_n = ldg4(b + p + sz);
        const F4 sxx_c = ldg4(sxx + p);
        const F4 sxy_c = ldg4(sxy + p);
        const F4 sxy_ym = ldg4(sxy + p - sy);
        const F4 syy_c = ldg4(syy + p);
        const F4 syy_yp = ldg4(syy + p + sy);
        const F4 syz_ym = ldg4(syz + p - sy);
        const F4 b_yp = ldg4(b + p + sy);
        F4 vx_c = ld4(vx + p), vy_c = ld4(vy + p), vz_c = ld4(vz + p);
        const float sxx_l = left_of(sxx_c, sxx + p, lane);
        const float sxy_r = right_of(sxy_c, sxy + p, lane);
        const float sxz_r = right_of(sxz_c, sxz + p, lane);
        const float b_r = right_of(b_c, b + p, lane);
        const float bn_r = right_of(b_n, b + p + sz, lane);
        const float byp_r = right_of(b_yp, b + p + sy, lane);
        if (act) {
            if (vc) {
                st4(vc0 + p, vx_c);
                st4(vc1 + p, vy_c);
                st4(vc2 + p, vz_c);
            }
            const bool zvxy = iz >= zt && iz <= zb;
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const float sxx_xm = i == 0 ? sxx_l : sxx_c.e[i > 0 ? i - 1 : 0];
                const float sxy_xp = i == 3 ? sxy_r : sxy_c.e[i < 3 ? i + 1 : 3];
                const float sxz_xp = i == 3 ? sxz_r : sxz_c.e[i < 3 ? i + 1 : 3];
                const float b_xp = i == 3 ? b_r : b_c.e[i < 3 ? i + 1 : 3];
                const float bn_xp = i == 3 ? bn_r : b_n.e[i < 3 ? i + 1 : 3];
                const float byp_xp = i == 3 ? byp_r : b_yp.e[i < 3 ? i + 1 : 3];
                if (mx_in[i] && yin && zvxy) {
                    const float d = add_(add_(mul_(k0, sub_(sxx_c.e[i], sxx_xm)), mul_(k1, sub_(sxy_c.e[i], sxy_ym.e[i]))),
                                         mul_(k2, sub_(sxz_c.e[i], sxz_m.e[i])));
                    vx_c.e[i] = add_(vx_c.e[i], mul_(b_c.e[i], d));
                }
                if (mx_s[i] && zvxy) {
                    const float bb = mul_(q, add_(add_(add_(b_c.e[i], b_xp), b_yp.e[i]), byp_xp));
                    const float d = add_(add_(mul_(k0, sub_(sxy_xp, sxy_c.e[i])), mul_(k2, sub_(syz_c.e[i], syz_m.e[i]))),
                                         mul_(k1, sub_(syy_yp.e[i], syy_c.e[i])));
                    vy_c.e[i] = add_(vy_c.e[i], mul_(bb, d));
                }
                if (mx_s[i] && yin && iz <= nz - 1) {
                    const float bb = mul_(q, add_(add_(add_(b_c.e[i], b_n.e[i]), b_xp), bn_xp));
                    const float d = add_(add_(mul_(k0, sub_(sxz_xp, sxz_c.e[i])), mul_(k2, sub_(szz_n.e[i], szz_c.e[i]))),
                                         mul_(k1, sub_(syz_c.e[i], syz_ym.e[i])));
                    vz_c.e[i] = add_(vz_c.e[i], mul_(bb, d));
                }
            }
            st4(vx + p, vx_c);
            st4(vy + p, vy_c);
            st4(vz + p, vz_c);
        }
        sxz_m = sxz_c;
        syz_m = syz_c;
        szz_c = szz_n;
        b_c = b_n;
    }
}

// ---------------------------------------------------------------------------
// Stress update (update_stress.cpp:36-133), radius 1; ranges as stress_kernel.
// ---------------------------------------------------------------------------
template <int MED>
__device__ __forceinline__ void load_normal(const GridDev<float> &G, int p, F4 &c11, F4 &c22, F4 &c33, F4 &c23, F4 &c13,
                                            F4 &c12)
{
    if (MED == MED_ISO5) {
        c11 = ldg4(G.c[0] + p);
        c22 = c33 = c11;
        c13 = ldg4(G.c[1] + p);
        c23 = c12 = c13;
    } else {
        c11 = ldg4(G.c[0] + p);
        c22 = ldg4(G.c[1] + p);
        c33 = ldg4(G.c[2] + p);
        c23 = ldg4(G.c[3] + p);
        c13 = ldg4(G.c[4] + p);
        c12 = ldg4(G.c[5] + p);
    }
}

template <int MED>
__global__ void __launch_bounds__(32 * V4_ROWS) stress_kernel_v4(GridDev<float> G, int flag, int zchunk)
{
    const Geo &g = G.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int lane = threadIdx.x;
    const int iy = blockIdx.y * V4_ROWS + threadIdx.y;
    if (iy > ny) return;
    const int x0 = (blockIdx.x * 32 + lane) * 4;
    const bool act = x0 <= nx;
    const int xc = act ? x0 : 0;
    const int z0 = blockIdx.z * zchunk;
    const int z1 = min(nz, z0 + zchunk - 1);
    const int sy = g.px, sz = g.px * g.py;
    const float *__restrict__ vx = G.f[VX];
    const float *__restrict__ vy = G.f[VY];
    const float *__restrict__ vz = G.f[VZ];
    float *__restrict__ sxx = G.f[SXX];
    float *__restrict__ syy = G.f[SYY];
    float *__restrict__ szz = G.f[SZZ];
    float *__restrict__ syz = G.f[SYZ];
    float *__restrict__ sxz = G.f[SXZ];
    float *__restrict__ sxy = G.f[SXY];
    const int s44 = MED == MED_ISO5 ? 2 : 6;
    const float k0 = G.k[0], k1 = G.k[1], k2 = G.k[2];
    const float half = 0.5f;
    const bool ys = iy <= ny - 1;
    const bool yin = iy >= 1 && iy <= ny - 1;
    bool mn[4], mxz[4], mm[4];
#pragma unroll
    for (int i = 0; i < 4; i++) {
        mn[i] = x0 + i <= nx - 1;
        mxz[i] = x0 + i <= nx;
        mm[i] = x0 + i >= 1 && x0 + i <= nx - 1;
    }

    int p = g.idx(xc, iy, z0);
    F4 vz_m = ldg4(vz + p - sz);
    F4 vx_c = ldg4(vx + p);
    F4 vy_c = ldg4(vy + p);

    for (int iz = z0; iz <= z1; iz++, p += sz) {
        const F4 vz_c = ldg4(vz + p);
        const F4 vx_n = ldg4(vx + p + sz);
        const F4 vy_n = ldg4(vy + p + sz);
        const F4 vy_ym = ldg4(vy + p - sy);
        const F4 vz_yp = ldg4(vz + p + sy);
        const F4 vx_yp = ldg4(vx + p + sy);
        F4 c11, c22, c33, c23, c13, c12;
        load_normal<MED>(G, p, c11, c22, c33, c23, c13, c12);
        const F4 c44 = ldg4(G.c[s44] + p), c55 = ldg4(G.c[s44 + 1] + p), c66 = ldg4(G.c[s44 + 2] + p);
        F4 s_xx = ld4(sxx + p), s_yy = ld4(syy + p), s_zz = ld4(szz + p);
        F4 s_yz = ld4(syz + p), s_xz = ld4(sxz + p), s_xy = ld4(sxy + p);
        const float vx_r = right_of(vx_c, vx + p, lane);
        const float vy_l = left_of(vy_c, vy + p, lane);
        const float vz_l = left_of(vz_c, vz + p, lane);
        if (act) {
            const bool surf = flag && iz == 0;
#pragma unroll
            for (int i = 0; i < 4; i++) {
                const float vx_xp = i == 3 ? vx_r : vx_c.e[i < 3 ? i + 1 : 3];
                const float vy_xm = i == 0 ? vy_l : vy_c.e[i > 0 ? i - 1 : 0];
                const float vz_xm = i == 0 ? vz_l : vz_c.e[i > 0 ? i - 1 : 0];
                if (mn[i]) {
                    const float dvx = sub_(vx_xp, vx_c.e[i]);
                    const float dvy = sub_(vy_c.e[i], vy_ym.e[i]);
                    if (surf) {
                        const float a11 = sub_(c11.e[i], div_(mul_(c13.e[i], c13.e[i]), c33.e[i]));
                        const float a12 = sub_(c12.e[i], div_(mul_(c13.e[i], c23.e[i]), c33.e[i]));
                        const float a21 = sub_(c12.e[i], div_(mul_(c23.e[i], c13.e[i]), c33.e[i]));
                        const float a22 = sub_(c22.e[i], div_(mul_(c23.e[i], c23.e[i]), c33.e[i]));
                        s_xx.e[i] = add_(s_xx.e[i], add_(mul_(mul_(a11, k0), dvx), mul_(mul_(a12, k1), dvy)));
                        s_yy.e[i] = add_(s_yy.e[i], add_(mul_(mul_(a21, k0), dvx), mul_(mul_(a22, k1), dvy)));
                    } else {
                        const float dvz = sub_(vz_c.e[i], vz_m.e[i]);
                        s_xx.e[i] = add_(s_xx.e[i], add_(add_(mul_(mul_(c11.e[i], k0), dvx), mul_(mul_(c12.e[i], k1), dvy)),
                                                         mul_(mul_(c13.e[i], k2), dvz)));
                        s_yy.e[i] = add_(s_yy.e[i], add_(add_(mul_(mul_(c12.e[i], k0), dvx), mul_(mul_(c22.e[i], k1), dvy)),
                                                         mul_(mul_(c23.e[i], k2), dvz)));
                        s_zz.e[i] = add_(s_zz.e[i], add_(add_(mul_(mul_(c13.e[i], k0), dvx), mul_(mul_(c23.e[i], k1), dvy)),
                                                         mul_(mul_(c33.e[i], k2), dvz)));
                    }
                }
                if (mn[i] && ys && iz <= nz - 1)
                    s_yz.e[i] = add_(s_yz.e[i], mul_(mul_(half, c44.e[i]),
                                                     add_(mul_(k2, sub_(vy_n.e[i], vy_c.e[i])), mul_(k1, sub_(vz_yp.e[i], vz_c.e[i])))));
                if (mxz[i] && iz <= nz - 1)
                    s_xz.e[i] = add_(s_xz.e[i], mul_(mul_(half, c55.e[i]),
                                                     add_(mul_(k2, sub_(vx_n.e[i], vx_c.e[i])), mul_(k0, sub_(vz_c.e[i], vz_xm)))));
                if (mxz[i] && ys)
                    s_xy.e[i] = add_(s_xy.e[i], mul_(mul_(half, c66.e[i]),
                                                     add_(mul_(k1, sub_(vx_yp.e[i], vx_c.e[i])), mul_(k0, sub_(vy_c.e[i], vy_xm)))));
            }
            st4(sxx + p, s_xx);
            st4(syy + p, s_yy);
            st4(szz + p, s_zz);
            st4(syz + p, s_yz);
            st4(sxz + p, s_xz);
            st4(sxy + p, s_xy);
            if (surf) {
                // free-surface odd mirrors (update_stress.cpp:260-277), merged into the halo plane
                F4 myz = ld4(syz + p - sz), mxzv = ld4(sxz + p - sz);
#pragma unroll
                for (int i = 0; i < 4; i++) {
                    if (mn[i] && ys) myz.e[i] = -s_yz.e[i];
                    if (mm[i] && yin) mxzv.e[i] = -s_xz.e[i];
                }
                st4(syz + p - sz, myz);
                st4(sxz + p - sz, mxzv);
            }
        }
        vz_m = vz_c;
        vx_c = vx_n;
        vy_c = vy_n;
    }
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
static int pick_zchunk_v4(int64_t cols, int nz, int sms)
{
    const int64_t want = (int64_t)sms * 6;
    int nchunk = (int)((want + cols - 1) / cols);
    if (nchunk < 1) nchunk = 1;
    if (nchunk > nz + 1) nchunk = nz + 1;
    return (nz + 1 + nchunk - 1) / nchunk;
}

// planes per z-chunk for a requested number of chunks (0: the automatic choice)
static int chunk_planes(int nz, int nchunk)
{
    if (nchunk > nz + 1) nchunk = nz + 1;
    return (nz + 1 + nchunk - 1) / nchunk;
}

cudaError_t launch_vel_v4(const GridDev<float> &G, int top, int bottom, int top_bc, float *const vcopy[3], int sms,
                          cudaStream_t st, int nchunk)
{
    const Geo &g = G.g;
    const int zt = (top && top_bc != 1) ? 1 : 0;
    const int bx = (g.nx + 127) / 128, by = (g.ny + V4_ROWS - 1) / V4_ROWS;
    const int zc = nchunk > 0 ? chunk_planes(g.nz, nchunk) : pick_zchunk_v4((int64_t)bx * by, g.nz, sms);
    dim3 blk(32, V4_ROWS), grd(bx, by, (g.nz + 1 + zc - 1) / zc);
    vel_kernel_v4<<<grd, blk, 0, st>>>(G, zt, bottom, zc, vcopy ? vcopy[0] : nullptr, vcopy ? vcopy[1] : nullptr,
                                       vcopy ? vcopy[2] : nullptr);
    return cudaGetLastError();
}

cudaError_t launch_stress_v4(const GridDev<float> &G, int medium, int top, int top_bc, int sms, cudaStream_t st,
                             int nchunk)
{
    const Geo &g = G.g;
    const int flag = (top && top_bc) ? 1 : 0;
    const int bx = (g.nx + 1 + 127) / 128, by = (g.ny + 1 + V4_ROWS - 1) / V4_ROWS;
    const int zc = nchunk > 0 ? chunk_planes(g.nz, nchunk) : pick_zchunk_v4((int64_t)bx * by, g.nz, sms);
    dim3 blk(32, V4_ROWS), grd(bx, by, (g.nz + 1 + zc - 1) / zc);
    if (medium == MED_ISO5)
        stress_kernel_v4<MED_ISO5><<<grd, blk, 0, st>>>(G, flag, zc);
    else if (medium == MED_ORTHO9)
        stress_kernel_v4<MED_ORTHO9><<<grd, blk, 0, st>>>(G, flag, zc);
    else
        return cudaErrorInvalidValue;
    return cudaGetLastError();
}

} // namespace ecsg
