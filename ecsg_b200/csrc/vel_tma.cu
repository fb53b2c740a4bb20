// vel_tma.cu -- FP32 velocity update with TMA-staged planes (radius 1).
//
// The same update as vel_kernel_v4 (stencil_v4.cu) with the same per-element
// operation order, hence the same bits, organised so that copies, not load
// latency, set the pace (the float4 sweep keeps one plane of loads in flight
// per warp and is latency-bound).  A CTA owns a 64 x 8 tile of (x, y) points
// and marches z.  One producer thread streams, per plane, each stress
// component and the buoyancy as a box with the one-sided halo the update
// reads (update_vel.cpp:20-69):
//   sxx  x-1            sxy  x+1, y-1        sxz  x+1
//   syy  y+1            syz  y-1             szz  -
//   b    x+1, y+1       vx vy vz: the tile (one 4-D copy)
// into a ring of NS plane stages with mbarrier completion (no multicast).  The
// update of plane p reads planes p-1 (sxz, syz), p and p+1 (szz, b), so three
// stages are in use and the others are being filled.  Eight consumer warps
// update two points per thread and store them with coalesced stores.  All
// waits are bounded: on a timeout the CTA sets ST_PIPE_TIMEOUT, stops, and
// drains its own copies before returning.
#include "ecsg_device.cuh"
#include "tma_util.cuh"

#include <cstring>

namespace ecsg {

namespace vtma {
constexpr int TX = 64, TY = 8, NW = 8, NTHREADS = NW * 32 + 32;
constexpr int NS = 5;   // plane stages
// boxes: width, height, x and y of the box origin relative to the tile
struct Box {
    int w, h, ox, oy;
};
constexpr Box B_SXX{TX + 4, TY, -4, 0}, B_SXY{TX + 4, TY + 1, 0, -1}, B_SXZ{TX + 4, TY, 0, 0};
constexpr Box B_SYY{TX, TY + 1, 0, 0}, B_SYZ{TX, TY + 1, 0, -1}, B_SZZ{TX, TY, 0, 0}, B_B{TX + 4, TY + 1, 0, 0};
constexpr Box B_V{TX, TY, 0, 0};
__host__ __device__ constexpr int bytes(const Box &b) { return b.w * b.h * 4; }
__host__ __device__ constexpr int up128(int x) { return (x + 127) / 128 * 128; }
constexpr int O_SXX = 0, O_SXY = O_SXX + up128(bytes(B_SXX)), O_SXZ = O_SXY + up128(bytes(B_SXY));
constexpr int O_SYY = O_SXZ + up128(bytes(B_SXZ)), O_SYZ = O_SYY + up128(bytes(B_SYY));
constexpr int O_SZZ = O_SYZ + up128(bytes(B_SYZ)), O_B = O_SZZ + up128(bytes(B_SZZ));
constexpr int O_V = O_B + up128(bytes(B_B));
constexpr int SLOT = O_V + 3 * bytes(B_V);
static_assert(SLOT % 128 == 0, "stage slots 128-byte aligned");
constexpr int OFF_BAR = NS * SLOT;
constexpr int OFF_FLAG = OFF_BAR + 2 * NS * 8;
constexpr int SMEM = OFF_FLAG + 64;
// bytes of a plane: below the chunk (sxz, syz only), above it (szz, b only), inside (all)
constexpr int TX_LO = bytes(B_SXZ) + bytes(B_SYZ);
constexpr int TX_HI = bytes(B_SZZ) + bytes(B_B);
constexpr int TX_IN = bytes(B_SXX) + bytes(B_SXY) + bytes(B_SXZ) + bytes(B_SYY) + bytes(B_SYZ) + bytes(B_SZZ) +
                      bytes(B_B) + 3 * bytes(B_V);
} // namespace vtma

// The maps of one sweep over NSH shots of one grid that share the medium: the
// buoyancy map is common, the field maps and the velocity outputs per shot.
template <int NSH>
struct VelMaps {
    CUtensorMap b;
    CUtensorMap sxx[NSH], sxy[NSH], sxz[NSH], syy[NSH], syz[NSH], szz[NSH], v[NSH];
    float *vout[NSH][3];   // the shot's vx vy vz
    int ns;
};

__device__ __forceinline__ void vel_consumer_sync() { asm volatile("bar.sync 1, 256;" ::: "memory"); }

// NSH > 1: maps.ns shots of the grid in one launch, the CTAs of one tile
// column adjacent (shot fastest), so the buoyancy planes one of them stages
// are still in L2 for the others.
template <int NSH>
__global__ void __launch_bounds__(vtma::NTHREADS, 2)
    vel_tma_kernel(const __grid_constant__ VelMaps<NSH> maps, GridDev<float> G, int zt, int bottom, int zchunk, float *vc0,
                   float *vc1, float *vc2, int *status)
{
    using namespace vtma;
    extern __shared__ __align__(128) unsigned char sm[];
    const Geo &g = G.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int shot = NSH == 1 ? 0 : (int)(blockIdx.x % (unsigned)maps.ns);
    const int x0 = (NSH == 1 ? (int)blockIdx.x : (int)(blockIdx.x / (unsigned)maps.ns)) * TX, y0 = blockIdx.y * TY;
    const int z0 = blockIdx.z * zchunk, z1 = min(nz, z0 + zchunk - 1);
    const int n = z1 - z0 + 3;   // planes z0-1 .. z1+1
    const unsigned bar0 = smem_u32(sm + OFF_BAR);
    auto full = [&](int s) { return bar0 + 8u * s; };
    auto empty = [&](int s) { return bar0 + 8u * (NS + s); };
    // [0] producer gave up, [1] stages consumed, [3] consumers gave up (written only
    // by consumers before a consumer barrier and read after it)
    volatile int *flags = (volatile int *)(sm + OFF_FLAG);

    if (tid == 0) {
        for (int s = 0; s < NS; s++) { mbar_init(full(s), 1); mbar_init(empty(s), 1); }
        flags[0] = 0; flags[1] = 0; flags[3] = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    int issued = 0;
    if (warp == NW) {
        // ---------------- producer ----------------
        if (lane == 0) {
            const int xa = XOFF + x0, ya = g.R + y0;
            bool ok = true;
            for (int i = 0; i < n && ok; i++) {
                const int s = i % NS, q = z0 - 1 + i;
                if (i >= NS && !mbar_wait(empty(s), ((i / NS) - 1) & 1)) { ok = false; break; }
                const unsigned d = smem_u32(sm + s * SLOT);
                const int zc = g.R + q;
                const bool lo = q < z0, hi = q > z1;
                mbar_expect_tx(full(s), lo ? TX_LO : (hi ? TX_HI : TX_IN));
                if (!hi) {
                    tma_load4(d + O_SXZ, &maps.sxz[shot], xa + B_SXZ.ox, ya + B_SXZ.oy, zc, full(s));
                    tma_load4(d + O_SYZ, &maps.syz[shot], xa + B_SYZ.ox, ya + B_SYZ.oy, zc, full(s));
                }
                if (!lo) {
                    tma_load4(d + O_SZZ, &maps.szz[shot], xa + B_SZZ.ox, ya + B_SZZ.oy, zc, full(s));
                    tma_load4(d + O_B, &maps.b, xa + B_B.ox, ya + B_B.oy, zc, full(s));
                }
                if (!lo && !hi) {
                    tma_load4(d + O_SXX, &maps.sxx[shot], xa + B_SXX.ox, ya + B_SXX.oy, zc, full(s));
                    tma_load4(d + O_SXY, &maps.sxy[shot], xa + B_SXY.ox, ya + B_SXY.oy, zc, full(s));
                    tma_load4(d + O_SYY, &maps.syy[shot], xa + B_SYY.ox, ya + B_SYY.oy, zc, full(s));
                    tma_load4(d + O_V, &maps.v[shot], xa + B_V.ox, ya + B_V.oy, zc, full(s));
                }
                issued = i + 1;
                if (flags[3]) break;
            }
            if (!ok) {
                flags[0] = 1;
                atomicOr(status, ST_PIPE_TIMEOUT);
            }
        }
    } else {
        // ---------------- consumers ----------------
        const int ty = warp, iy = y0 + ty;
        const float k0 = G.k[0], k1 = G.k[1], k2 = G.k[2];
        const float qq = 0.25f;
        float *vxg = maps.vout[shot][0], *vyg = maps.vout[shot][1], *vzg = maps.vout[shot][2];
        const bool vc = vc0 != nullptr;
        const bool yrow = iy <= ny - 1;                  // rows the velocity update touches (vy: 0 .. ny-1)
        const bool yin = iy >= 1 && iy <= ny - 1;        // vx, vz: y walls excluded
        const int zb = nz - bottom;
        auto at = [](const float *box, Box b, int x, int y) { return box[(y - b.oy) * b.w + (x - b.ox)]; };
        int consumed = 0;
        for (int j = 0; j + 2 < n; j++) {
            const int p = z0 + j;
            bool ok = true;
            if (j == 0) ok = mbar_wait(full(0), 0) && mbar_wait(full(1 % NS), 0);
            ok = ok && mbar_wait(full((j + 2) % NS), ((j + 2) / NS) & 1);
            if (!ok) flags[3] = 1;
            vel_consumer_sync();
            if (flags[3]) break;
            consumed = j + 1;
            const unsigned char *Sm = sm + (j % NS) * SLOT;         // plane p-1
            const unsigned char *Sc = sm + ((j + 1) % NS) * SLOT;   // plane p
            const unsigned char *Sp = sm + ((j + 2) % NS) * SLOT;   // plane p+1
            const float *sxx = (const float *)(Sc + O_SXX), *sxy = (const float *)(Sc + O_SXY);
            const float *sxz = (const float *)(Sc + O_SXZ), *syy = (const float *)(Sc + O_SYY);
            const float *syz = (const float *)(Sc + O_SYZ), *szz = (const float *)(Sc + O_SZZ);
            const float *bb = (const float *)(Sc + O_B), *vv = (const float *)(Sc + O_V);
            const float *sxz_m = (const float *)(Sm + O_SXZ), *syz_m = (const float *)(Sm + O_SYZ);
            const float *szz_p = (const float *)(Sp + O_SZZ), *b_p = (const float *)(Sp + O_B);
            const bool zvxy = p >= zt && p <= zb;
            if (yrow) {
#pragma unroll
                for (int h = 0; h < 2; h++) {
                    const int tx = lane + 32 * h, ix = x0 + tx;
                    if (ix > nx) continue;
                    const int gp = g.idx(ix, iy, p);
                    float vxv = vv[0 * TX * TY + ty * TX + tx];
                    float vyv = vv[1 * TX * TY + ty * TX + tx];
                    float vzv = vv[2 * TX * TY + ty * TX + tx];
                    if (vc) {
                        vc0[gp] = vxv;
                        vc1[gp] = vyv;
                        vc2[gp] = vzv;
                    }
                    const bool xs = ix <= nx - 1, xin = ix >= 1 && xs;
                    const float b_c = at(bb, B_B, tx, ty), b_xp = at(bb, B_B, tx + 1, ty);
                    if (xin && yin && zvxy) {
                        const float d = add_(add_(mul_(k0, sub_(at(sxx, B_SXX, tx, ty), at(sxx, B_SXX, tx - 1, ty))),
                                                  mul_(k1, sub_(at(sxy, B_SXY, tx, ty), at(sxy, B_SXY, tx, ty - 1)))),
                                             mul_(k2, sub_(at(sxz, B_SXZ, tx, ty), at(sxz_m, B_SXZ, tx, ty))));
                        vxv = add_(vxv, mul_(b_c, d));
                    }
                    if (xs && zvxy) {
                        const float bq = mul_(qq, add_(add_(add_(b_c, b_xp), at(bb, B_B, tx, ty + 1)), at(bb, B_B, tx + 1, ty + 1)));
                        const float d = add_(add_(mul_(k0, sub_(at(sxy, B_SXY, tx + 1, ty), at(sxy, B_SXY, tx, ty))),
                                                  mul_(k2, sub_(at(syz, B_SYZ, tx, ty), at(syz_m, B_SYZ, tx, ty)))),
                                             mul_(k1, sub_(at(syy, B_SYY, tx, ty + 1), at(syy, B_SYY, tx, ty))));
                        vyv = add_(vyv, mul_(bq, d));
                    }
                    if (xs && yin && p <= nz - 1) {
                        const float bq = mul_(qq, add_(add_(add_(b_c, at(b_p, B_B, tx, ty)), b_xp), at(b_p, B_B, tx + 1, ty)));
                        const float d = add_(add_(mul_(k0, sub_(at(sxz, B_SXZ, tx + 1, ty), at(sxz, B_SXZ, tx, ty))),
                                                  mul_(k2, sub_(at(szz_p, B_SZZ, tx, ty), at(szz, B_SZZ, tx, ty)))),
                                             mul_(k1, sub_(at(syz, B_SYZ, tx, ty), at(syz, B_SYZ, tx, ty - 1))));
                        vzv = add_(vzv, mul_(bq, d));
                    }
                    vxg[gp] = vxv;
                    vyg[gp] = vyv;
                    vzg[gp] = vzv;
                }
            }
            vel_consumer_sync();   // every consumer is done with plane p-1
            if (tid == 0) mbar_arrive(empty(j % NS));
        }
        if (tid == 0) {
            flags[1] = consumed;
            if (flags[3]) atomicOr(status, ST_PIPE_TIMEOUT);
        }
    }
    __syncthreads();
    // drain: copies issued but never consumed (only after a timeout) complete before exit
    if (warp == NW && lane == 0) {
        // stages of planes consumed + 0 and consumed + 1 were waited on by the consumers
        // only if consumed > 0; wait for every issued stage past the last one released
        const int first = flags[1];
        for (int i = first; i < issued; i++) mbar_wait(full(i % NS), (i / NS) & 1);
    }
}

// ---------------------------------------------------------------------------
// Host side
// ---------------------------------------------------------------------------
size_t vel_maps_bytes() { return sizeof(VelMaps<1>); }

// Maps of one grid's velocity sweep; false if the driver entry point is missing
// or an address / pitch is not encodable.
bool vel_encode_maps(void *out, const GridDev<float> &G)
{
    using namespace vtma;
    VelMaps<1> M;
    memset(&M, 0, sizeof M);
    M.ns = 1;
    for (int k = 0; k < 3; k++) M.vout[0][k] = G.f[VX + k];
    const Geo &g = G.g;
    if ((g.px * 4) % 16 != 0) return false;
    // velocities: one allocation at a fixed stride
    for (int k = 1; k < 3; k++)
        if (G.f[k] != G.f[0] + (size_t)k * g.size()) return false;
    bool ok = encode(&M.sxx[0], g, G.f[SXX], 1, B_SXX.w, B_SXX.h) && encode(&M.sxy[0], g, G.f[SXY], 1, B_SXY.w, B_SXY.h) &&
              encode(&M.sxz[0], g, G.f[SXZ], 1, B_SXZ.w, B_SXZ.h) && encode(&M.syy[0], g, G.f[SYY], 1, B_SYY.w, B_SYY.h) &&
              encode(&M.syz[0], g, G.f[SYZ], 1, B_SYZ.w, B_SYZ.h) && encode(&M.szz[0], g, G.f[SZZ], 1, B_SZZ.w, B_SZZ.h) &&
              encode(&M.b, g, G.b, 1, B_B.w, B_B.h) && encode(&M.v[0], g, G.f[VX], 3, B_V.w, B_V.h);
    if (ok) memcpy(out, &M, sizeof M);
    return ok;
}

cudaError_t vel_tma_set_attributes()
{
    cudaError_t e = cudaFuncSetAttribute(vel_tma_kernel<1>, cudaFuncAttributeMaxDynamicSharedMemorySize, vtma::SMEM);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(vel_tma_kernel<kMaxShots>, cudaFuncAttributeMaxDynamicSharedMemorySize, vtma::SMEM);
    return e;
}

cudaError_t launch_vel_tma(const void *maps, const GridDev<float> &G, int top, int bottom, int top_bc,
                           float *const vcopy[3], int *status, int sms, cudaStream_t st, int nchunk_req)
{
    using namespace vtma;
    const Geo &g = G.g;
    const int zt = (top && top_bc != 1) ? 1 : 0;
    const int bx = (g.nx + 1 + TX - 1) / TX, by = (g.ny + TY - 1) / TY;
    const int64_t cols = (int64_t)bx * by;
    // two CTAs per SM: aim for >= 4 waves, chunks of >= 24 planes
    int nchunk = (int)(((int64_t)sms * 8 + cols - 1) / cols);
    if (nchunk < 1) nchunk = 1;
    const int maxc = (g.nz + 1) / 24 > 0 ? (g.nz + 1) / 24 : 1;
    if (nchunk > maxc) nchunk = maxc;
    if (nchunk_req > 0) nchunk = nchunk_req < g.nz + 1 ? nchunk_req : g.nz + 1;   // tuned
    const int zc = (g.nz + 1 + nchunk - 1) / nchunk;
    dim3 grd(bx, by, (g.nz + 1 + zc - 1) / zc);
    vel_tma_kernel<1><<<grd, NTHREADS, SMEM, st>>>(*(const VelMaps<1> *)maps, G, zt, bottom, zc, vcopy ? vcopy[0] : nullptr,
                                                   vcopy ? vcopy[1] : nullptr, vcopy ? vcopy[2] : nullptr, status);
    return cudaGetLastError();
}

// The sweep of ns shots of one grid sharing the medium (no velocity copies):
// maps[s] is shot s's opaque map block (vel_encode_maps); the buoyancy map
// is shot 0's.  Same launch shape as one shot per tile column, the shots'
// CTAs of a column adjacent.
cudaError_t launch_vel_tma_shots(const void *const *maps, int ns, const GridDev<float> &G, int top, int bottom,
                                 int top_bc, int *status, int sms, cudaStream_t st, int nchunk_req)
{
    using namespace vtma;
    if (ns < 1 || ns > kMaxShots) return cudaErrorInvalidValue;
    static thread_local VelMaps<kMaxShots> M;   // host staging of the kernel parameter
    memset(&M, 0, sizeof M);
    M.b = ((const VelMaps<1> *)maps[0])->b;
    M.ns = ns;
    for (int s = 0; s < ns; s++) {
        const VelMaps<1> &Ms = *(const VelMaps<1> *)maps[s];
        M.sxx[s] = Ms.sxx[0];
        M.sxy[s] = Ms.sxy[0];
        M.sxz[s] = Ms.sxz[0];
        M.syy[s] = Ms.syy[0];
        M.syz[s] = Ms.syz[0];
        M.szz[s] = Ms.szz[0];
        M.v[s] = Ms.v[0];
        for (int k = 0; k < 3; k++) M.vout[s][k] = Ms.vout[0][k];
    }
    const Geo &g = G.g;
    const int zt = (top && top_bc != 1) ? 1 : 0;
    const int bx = (g.nx + 1 + TX - 1) / TX, by = (g.ny + TY - 1) / TY;
    const int64_t cols = (int64_t)bx * by * ns;
    int nchunk = (int)(((int64_t)sms * 8 + cols - 1) / cols);
    if (nchunk < 1) nchunk = 1;
    const int maxc = (g.nz + 1) / 24 > 0 ? (g.nz + 1) / 24 : 1;
    if (nchunk > maxc) nchunk = maxc;
    if (nchunk_req > 0) nchunk = nchunk_req < g.nz + 1 ? nchunk_req : g.nz + 1;
    const int zc = (g.nz + 1 + nchunk - 1) / nchunk;
    dim3 grd(bx * ns, by, (g.nz + 1 + zc - 1) / zc);
    vel_tma_kernel<kMaxShots><<<grd, NTHREADS, SMEM, st>>>(M, G, zt, bottom, zc, nullptr, nullptr, nullptr, status);
    return cudaGetLastError();
}

} // namespace ecsg
