// stress21_tma.cu -- FP32 21-Cij stress update with TMA-staged planes.
//
// The same update as stress21.cu (same operation order and contractions, so
// the results are bitwise equal to its FP32 instantiation), organised for
// bandwidth: a CTA owns a 32 x 8 tile of
// (x, y) points and marches z.  One producer thread streams, per plane,
//   * the three velocities as 40 x 10 boxes (tile, one-point halo, the x
//     start rounded down to a 16-byte boundary),
//   * the 12 coefficient slots read around the tile (c6..c14, c16, c17, c19)
//     as 36 x 9 boxes, each with the one-sided halo its products need: slots
//     c6..c14 at x-1 and y+1 (normal products), c16, c17 at x-1 and y-1 (L4
//     links), c19 at x+1 and y+1 (the L5 link),
//   * the other 9 coefficient slots, the 6 stresses and (energy runs) the 3
//     displacement sums (stress21.cu) as 32 x 8 boxes,
// into shared-memory rings with cp.async.bulk.tensor (no multicast),
// completion tracked by mbarriers.  Each group of fields (velocities, the 12
// haloed slots, the 9 other slots, stresses, displacement sums) is one allocation with
// its fields at a fixed stride, so one 4-D tensor map (x, y, z, field) moves
// a whole group or sub-group: 7 copies per plane instead of 36 (small boxes
// from many descriptors kept the copy engine, not HBM, the limit).  Eight consumer warps compute
// every strain / link product of their own point plus one halo row or column
// of one kind per warp (each kind needs a one-sided halo only), exchange them
// through a two-plane ring, and update the stresses.  Velocities stay resident
// for three planes (p-1, p, p+1), coefficients and stresses for one; the
// values the z-staggered outputs (syz, sxz at plane p-1) need from plane p-1
// are carried in registers.  The rings are sized for two CTAs per SM (two
// plane stages, four velocity stages, 112 KB; 96 registers): the second CTA,
// not a deeper ring, hides the copy and dependency latency.  Tiles on the
// domain edges take the same arithmetic with per-thread closure weights.
// All waits are bounded: on a timeout the CTA sets ST_PIPE_TIMEOUT, stops,
// and drains its own copies before returning.
#include "ecsg_device.cuh"
#include "gen21_device.cuh"
#include "tma_util.cuh"

#include <cuda.h>
#include <cstring>
#include <type_traits>

namespace ecsg {

namespace s21t {
constexpr int TX = 32, TY = 8, NT = TX * TY, NTHREADS = NT + 32;
constexpr int BW = 40, BH = 10;              // haloed box: x0-4 .. x0+35, y0-1 .. y0+8
constexpr int HX = 34, HYI = 10, HP = HX * HYI;   // intermediates: x0-1 .. x0+32, y0-1 .. y0+8
constexpr int NQ = 9;
constexpr int NSP = 2, NSV = 4;               // ring depths: plane data, velocities (112 KB in all: 2 CTAs per SM)
constexpr int HBOX = BW * BH * 4;             // 1600 bytes
constexpr int IBOX = TX * TY * 4;             // 1024 bytes
constexpr int CW = 36, CHH = 9, CBOX = CW * CHH * 4;   // one-sided coefficient box: 1296 bytes
constexpr int NCH = 12, NCI = 9;
constexpr int NCA = 9, NCB = 2;               // c6..c14 | c16, c17 | c19
__host__ __device__ constexpr int up128(int b) { return (b + 127) / 128 * 128; }
constexpr int P_CHA = 0, P_CHB = up128(NCA * CBOX), P_CHC = up128(P_CHB + NCB * CBOX);
constexpr int P_CI = up128(P_CHC + CBOX), P_SG = P_CI + NCI * IBOX, P_EP = P_SG + 6 * IBOX;
// low-face boxes of the displacement sums (tiles at x0 = 0 / y0 = 0): x = -4..-1
// beside the tile's 8 rows, and row y = -1 under its 32 columns
constexpr int XFW = 4, XFBOX = XFW * TY * 4, YFBOX = TX * 4;   // 128 bytes each per field
constexpr int P_EX = P_EP + 3 * IBOX, P_EY = P_EX + 3 * XFBOX;
constexpr int PSLOT = P_EY + 3 * YFBOX;       // 35072, a multiple of 128
constexpr int VSLOT = (3 * HBOX + 127) / 128 * 128;   // 4864
static_assert(P_CHB % 128 == 0 && P_CHC % 128 == 0 && P_CI % 128 == 0 && P_SG % 128 == 0 && P_EP % 128 == 0 &&
                  P_EX % 128 == 0 && P_EY % 128 == 0 && PSLOT % 128 == 0, "128-byte aligned boxes");
constexpr int OFF_V = NSP * PSLOT;
constexpr int OFF_IM = OFF_V + NSV * VSLOT;
constexpr int OFF_BAR = OFF_IM + 2 * NQ * HP * 4;   // two-plane ring of intermediates
constexpr int NBAR = 2 * NSP + 2 * NSV;
constexpr int OFF_FLAG = OFF_BAR + NBAR * 8;
constexpr int SMEM = OFF_FLAG + 64;
static_assert(2 * (SMEM + 1024) <= 233472, "two CTAs per SM (228 KB of shared memory, 1 KB reserved per CTA)");
// coefficient slot of each staged box
__host__ __device__ constexpr int ch_slot(int k) { return k < 9 ? 6 + k : (k == 9 ? 16 : (k == 10 ? 17 : 19)); }
__host__ __device__ constexpr int ci_slot(int k) { return k < 6 ? k : (k == 6 ? 15 : (k == 7 ? 18 : 20)); }
} // namespace s21t

// The maps of one sweep over NSH shots of one grid that share the medium:
// the coefficient maps are common, the field maps and output blocks per shot.
template <int NSH>
struct S21Maps {
    CUtensorMap cha;       // c6..c14: boxes x-4 .. x+31, y .. y+8
    CUtensorMap chb;       // c16, c17: boxes x-4 .. x+31, y-1 .. y+7
    CUtensorMap chc;       // c19: box x .. x+35, y .. y+8
    CUtensorMap ci;        // c0..c5, c15, c18, c20: interior boxes
    CUtensorMap v[NSH];    // vx vy vz: haloed boxes
    CUtensorMap sg[NSH];   // sxx syy szz syz sxz sxy: interior boxes
    CUtensorMap ep[NSH];   // displacement sums: interior boxes
    CUtensorMap epx[NSH];  // displacement sums: x = -4..-1 face boxes (tiles at x0 = 0)
    CUtensorMap epy[NSH];  // displacement sums: y = -1 face rows (tiles at y0 = 0)
    float *sg_out[NSH][6]; // the shot's stresses sxx syy szz syz sxz sxy
    float *vin[NSH][3];    // the shot's velocities (read from memory by the free-surface condensation)
    float *u[NSH][3];      // the shot's displacement sums (null: none)
    int ns;
};

// the two closure weights of a neighbour pair (w2 of gen21_device.cuh)
__device__ __forceinline__ void closure_w2(bool a, bool b, float (&w)[2]) { w2<float>(a, b, w[0], w[1]); }

__device__ __forceinline__ void consumer_sync() { asm volatile("bar.sync 1, 256;" ::: "memory"); }

// NSH > 1: maps.ns shots of the grid in one launch, the CTAs of one tile
// column adjacent (shot fastest), so that the coefficient planes one of them
// stages are still in L2 when the others stage them.
template <bool ACC, int NSH>
__global__ void __launch_bounds__(s21t::NTHREADS, 2)
    stress21_tma_kernel(const __grid_constant__ S21Maps<NSH> maps, GridDev<float> G, int flag, int zchunk, int *status)
{
    using namespace s21t;
    extern __shared__ __align__(128) unsigned char sm[];
    const Geo &g = G.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const Ext E{nx, ny, nz};
    const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
    const int shot = NSH == 1 ? 0 : (int)(blockIdx.x % (unsigned)maps.ns);
    const int x0 = (NSH == 1 ? (int)blockIdx.x : (int)(blockIdx.x / (unsigned)maps.ns)) * TX, y0 = blockIdx.y * TY;
    const int z0 = blockIdx.z * zchunk, z1 = min(nz, z0 + zchunk - 1);
    const int qstart = z0 - 1, n = z1 - z0 + 3;   // planes z0-1 .. z1+1
    float *const u0 = maps.u[shot][0], *const u1 = maps.u[shot][1], *const u2 = maps.u[shot][2];
    const int sz = g.px * g.py;
    const unsigned bar0 = smem_u32(sm + OFF_BAR);
    auto fullP = [&](int s) { return bar0 + 8u * s; };
    auto emptyP = [&](int s) { return bar0 + 8u * (NSP + s); };
    auto fullV = [&](int s) { return bar0 + 8u * (2 * NSP + s); };
    auto emptyV = [&](int s) { return bar0 + 8u * (2 * NSP + NSV + s); };
    // [0] producer gave up, [1] P stages consumed, [2] V stages consumed, [3 + (i & 1)]
    // consumers gave up on plane stage i.  A consumer sets it before the stage's
    // first consumer barrier and every consumer reads it right after that barrier;
    // no consumer can reach stage i + 2 (same word) before all have passed the
    // barrier of stage i + 1, so every consumer takes the same branch.
    volatile int *flags = (volatile int *)(sm + OFF_FLAG);
    float *IM = (float *)(sm + OFF_IM);

    if (tid == 0) {
        // a slot is free again once each of the 8 consumer warps has arrived
        for (int s = 0; s < NSP; s++) { mbar_init(fullP(s), 1); mbar_init(emptyP(s), NT / 32); }
        for (int s = 0; s < NSV; s++) { mbar_init(fullV(s), 1); mbar_init(emptyV(s), NT / 32); }
        flags[0] = 0; flags[1] = 0; flags[2] = 0; flags[3] = 0; flags[4] = 0;
        asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    }
    __syncthreads();

    int issuedP = 0, issuedV = 0;
    if (warp == NT / 32) {
        // ---------------- producer ----------------
        if (lane == 0) {
            const int hx0 = XOFF + x0 - 4, hy0 = g.R + y0 - 1, ix0 = XOFF + x0, iy0 = g.R + y0;
            auto issueV = [&](int j) -> bool {
                const int s = j % NSV;
                if (j >= NSV && !mbar_wait(emptyV(s), ((j / NSV) - 1) & 1)) return false;
                const unsigned dst = smem_u32(sm + OFF_V + s * VSLOT);
                mbar_expect_tx(fullV(s), 3 * HBOX);
                const int zc = g.R + qstart - 1 + j;
                tma_load4(dst, &maps.v[shot], hx0, hy0, zc, fullV(s));
                return true;
            };
            auto issueP = [&](int i) -> bool {
                const int s = i % NSP;
                if (i >= NSP && !mbar_wait(emptyP(s), ((i / NSP) - 1) & 1)) return false;
                const int q = qstart + i;
                const bool inner = q >= z0 && q <= z1;
                // displacement sums: interior box on inner planes and on plane -1,
                // face boxes on the inner planes of low-face tiles
                const bool uin = ACC && (inner || q == -1);
                const bool ux = ACC && inner && x0 == 0, uy = ACC && inner && y0 == 0;
                const unsigned dst = smem_u32(sm + s * PSLOT);
                mbar_expect_tx(fullP(s), NCH * CBOX + (inner ? (NCI + 6) * IBOX : 0) + (uin ? 3 * IBOX : 0) +
                                             (ux ? 3 * XFBOX : 0) + (uy ? 3 * YFBOX : 0));
                const int zc = g.R + q;
                tma_load4(dst + P_CHA, &maps.cha, hx0, iy0, zc, fullP(s));
                tma_load4(dst + P_CHB, &maps.chb, hx0, hy0, zc, fullP(s));
                tma_load4(dst + P_CHC, &maps.chc, ix0, iy0, zc, fullP(s));
                if (inner) {
                    tma_load4(dst + P_CI, &maps.ci, ix0, iy0, zc, fullP(s));
                    tma_load4(dst + P_SG, &maps.sg[shot], ix0, iy0, zc, fullP(s));
                }
                if (uin) tma_load4(dst + P_EP, &maps.ep[shot], ix0, iy0, zc, fullP(s));
                if (ux) tma_load4(dst + P_EX, &maps.epx[shot], XOFF - XFW, iy0, zc, fullP(s));
                if (uy) tma_load4(dst + P_EY, &maps.epy[shot], ix0, g.R - 1, zc, fullP(s));
                return true;
            };
            bool ok = true;
            for (int i = 0; i < n && ok; i++) {
                while (ok && issuedV <= i + 2) {
                    ok = issueV(issuedV);
                    if (ok) issuedV++;
                }
                if (ok) {
                    ok = issueP(i);
                    if (ok) issuedP++;
                }
                if (flags[3] || flags[4]) break;
            }
            if (!ok) {
                flags[0] = 1;
                atomicOr(status, ST_PIPE_TIMEOUT);
            }
        }
    } else {
        // ---------------- consumers ----------------
        const int tx = lane, ty = warp;
        const int ox = x0 + tx, oy = y0 + ty;
        const int vb = (ty + 1) * BW + tx + 4, ib = ty * TX + tx, hx = tx + 1, hy = ty + 1;
        const float k0 = G.k[0], k1 = G.k[1], k2 = G.k[2];
        // the free-surface e3 (gen21_device.cuh e3_used) reads the averaged
        // strains around the point from memory: this shot's velocities
        auto e3_surface = [&](int xs, int ys, int ps, int pidx, float a1, float a2) -> float {
            if (NSH == 1) return e3_used(G, E, true, xs, ys, ps, pidx, a1, a2);
            GridDev<float> Gs = G;
            Gs.f[VX] = maps.vin[shot][0];
            Gs.f[VY] = maps.vin[shot][1];
            Gs.f[VZ] = maps.vin[shot][2];
            return e3_used(Gs, E, true, xs, ys, ps, pidx, a1, a2);
        };
        float *sxx = maps.sg_out[shot][0], *syy = maps.sg_out[shot][1], *szz = maps.sg_out[shot][2],
              *syz = maps.sg_out[shot][3], *sxz = maps.sg_out[shot][4], *sxy = maps.sg_out[shot][5];
        // carries from plane pm = p-1 for the syz / sxz outputs
        float c15p = 0.f, c16p = 0.f, c17p = 0.f, c18p = 0.f, c19p = 0.f, s3p = 0.f, s4p = 0.f;
        // the halo job of this warp: kind (0 L4, 1 L5, 2 L6, 3 N) and point
        int hk, hxp, hyp;
        {
            const int w = warp;
            hk = w & 3;
            if (w < 4) {   // rows
                hxp = x0 + lane;
                hyp = (hk == 0 || hk == 2) ? y0 - 1 : y0 + TY;
            } else {       // columns, 9 lanes
                hxp = (hk == 0 || hk == 3) ? x0 - 1 : x0 + TX;
                hyp = (hk == 0 || hk == 2) ? y0 - 1 + lane : y0 + lane;
            }
        }
        const bool hact = warp < 4 || lane < 9;
        const int hvb = (hyp - y0 + 1) * BW + (hxp - x0 + 4), hhb = (hyp - y0 + 1) * HX + (hxp - x0 + 1);
        // coefficient boxes: own point and halo point in each (the halo index is
        // used only with the sub-group that covers this warp's halo kind)
        const int ia = ty * CW + tx + 4, ibb = (ty + 1) * CW + tx + 4, ic = ty * CW + tx;
        const int ha = (hyp - y0) * CW + (hxp - x0) + 4, hb = (hyp - y0 + 1) * CW + (hxp - x0) + 4,
                  hc = (hyp - y0) * CW + (hxp - x0);
        // Tiles whose points and halos all lie strictly inside the grid (x, y in
        // 1 .. n-1): on their planes 1 .. nz-1 every extent test passes and every
        // closure weight is 1/4, so the fast variant drops the tests.
        const bool tile_in = x0 >= 1 && x0 + TX <= nx && y0 >= 1 && y0 + TY <= ny;
        // closure weights of this point's x and y neighbour pairs: xA {x, x+1}
        // (extent 0..nx), xB {x-1, x} (0..nx-1), yA {y-1, y} (0..ny-1), yB {y, y+1} (0..ny)
        float wxA[2], wxB[2], wyA[2], wyB[2];
        closure_w2(ox <= nx, ox + 1 <= nx, wxA);
        closure_w2(ox - 1 >= 0 && ox - 1 <= nx - 1, ox <= nx - 1, wxB);
        closure_w2(oy - 1 >= 0 && oy - 1 <= ny - 1, oy <= ny - 1, wyA);
        closure_w2(oy <= ny, oy + 1 <= ny, wyB);
        const int pbase = g.idx(ox, oy, 0);
        int consumedP = 0, consumedV = 0;
        for (int i = 0; i < n; i++) {
            const int p = qstart + i;
            // ---- wait for plane data p and velocities p-1, p, p+1
            bool ok = true;
            if (i == 0) {
                ok = mbar_wait(fullV(0), 0) && mbar_wait(fullV(1), 0);
            }
            ok = ok && mbar_wait(fullV((i + 2) % NSV), ((i + 2) / NSV) & 1);
            ok = ok && mbar_wait(fullP(i % NSP), (i / NSP) & 1);
            if (!ok) flags[3 + (i & 1)] = 1;
            const unsigned char *PS = sm + (i % NSP) * PSLOT;
            const float *CHA = (const float *)(PS + P_CHA);
            const float *CHB = (const float *)(PS + P_CHB);
            const float *CHC = (const float *)(PS + P_CHC);
            const float *CI = (const float *)(PS + P_CI);
            const float *SG = (const float *)(PS + P_SG);
            const float *EP = (const float *)(PS + P_EP);
            const float *Vm = (const float *)(sm + OFF_V + (i % NSV) * VSLOT);
            const float *Vp = (const float *)(sm + OFF_V + ((i + 1) % NSV) * VSLOT);
            const float *Vn = (const float *)(sm + OFF_V + ((i + 2) % NSV) * VSLOT);
            constexpr int HS = HBOX / 4;   // floats between the haloed boxes of a group
            constexpr int IS = IBOX / 4;
            // two-plane ring: stage i + 1 writes the slot stage i reads as plane
            // p-1, hence the consumer barrier at the end of every stage
            float *IMs = IM + (i & 1) * NQ * HP;
            const float *Rs = IMs;                               // plane p
            const float *Rp = IM + ((i + 1) & 1) * NQ * HP;      // plane p-1
            const bool surf = flag && p == 0;
            const bool inner = p >= z0 && p <= z1;
            const int pm = p - 1;
            const bool outer_pm = pm >= z0 && pm <= z1;
            constexpr int CS = CBOX / 4;   // floats between the coefficient boxes of a sub-group
            // coefficient slot k (0..11 of ch_slot) at this thread's point or at its halo point
            auto cho = [&](int k) { return k < NCA ? CHA[k * CS + ia] : (k < NCA + NCB ? CHB[(k - NCA) * CS + ibb] : CHC[ic]); };
            auto chh = [&](int k) { return k < NCA ? CHA[k * CS + ha] : (k < NCA + NCB ? CHB[(k - NCA) * CS + hb] : CHC[hc]); };

            // closure weights of the z pairs: zA {p-1, p} (extent 0..nz-1) for the
            // outputs at p, zB {pm, pm+1} (extent 0..nz) for the outputs at pm
            float wzA[2], wzB[2];
            closure_w2(p - 1 >= 0 && p - 1 <= nz - 1, p >= 0 && p <= nz - 1, wzA);
            closure_w2(pm <= nz, pm + 1 <= nz, wzB);
            auto body = [&](auto fast_tag) {
                constexpr bool FAST = decltype(fast_tag)::value;
                auto RR = [&](int plane_is_p, int q, int hx_, int hy_) { return (plane_is_p ? Rs : Rp)[q * HP + hy_ * HX + hx_]; };
                // closure-weighted mean of four neighbours: 1/4 each on the fast
                // path, else the per-dimension closure weights w0 (first index of
                // v) and w1 (second).  avg4's order; its skipped zero-weight terms
                // are included here, which leaves the sum bitwise unchanged (the
                // sum starts at +0, so it is never -0, and adding a signed zero to
                // it changes nothing; the neighbours outside an extent hold 0).
                auto av = [&](const float (&v)[2][2], const float (&w0)[2], const float (&w1)[2]) -> float {
                    if (FAST) {
                        const float w = 0.25f;
                        return fma_(w, v[1][1], fma_(w, v[1][0], fma_(w, v[0][1], fma_(w, v[0][0], 0.f))));
                    }
                    float acc = 0.f;
#pragma unroll
                    for (int a = 0; a < 2; a++)
#pragma unroll
                        for (int b = 0; b < 2; b++) acc = fma_(mul_(w0[a], w1[b]), v[a][b], acc);
                    return acc;
                };

                // ---- intermediates of plane p: own point (all kinds), then the halo job
                float e1 = 0.f, e2 = 0.f, e3 = 0.f;
                {
                    float e4 = 0.f, q45 = 0.f, q46 = 0.f, e5 = 0.f, q56 = 0.f, e6 = 0.f, p4 = 0.f, p5 = 0.f, p6 = 0.f;
                    if (FAST || E.l4(ox, oy, p)) {
                        e4 = fma_(k1, sub_(Vp[2 * HS + vb + BW], Vp[2 * HS + vb]), mul_(k2, sub_(Vn[HS + vb], Vp[HS + vb])));
                        q45 = mul_(cho(9), e4);
                        q46 = mul_(cho(10), e4);
                    }
                    if (FAST || E.l5(ox, oy, p)) {
                        e5 = fma_(k0, sub_(Vp[2 * HS + vb], Vp[2 * HS + vb - 1]), mul_(k2, sub_(Vn[vb], Vp[vb])));
                        q56 = mul_(cho(11), e5);
                    }
                    if (FAST || E.l6(ox, oy, p)) e6 = fma_(k0, sub_(Vp[HS + vb], Vp[HS + vb - 1]), mul_(k1, sub_(Vp[vb + BW], Vp[vb])));
                    if (FAST || E.n(ox, oy, p)) {
                        e1 = mul_(k0, sub_(Vp[vb + 1], Vp[vb]));
                        e2 = mul_(k1, sub_(Vp[HS + vb], Vp[HS + vb - BW]));
                        if (!FAST && surf)
                            e3 = e3_surface(ox, oy, p, pbase + p * sz, e1, e2);
                        else
                            e3 = mul_(k2, sub_(Vp[2 * HS + vb], Vm[2 * HS + vb]));
                        p4 = fma_(cho(6), e3, fma_(cho(3), e2, mul_(cho(0), e1)));
                        p5 = fma_(cho(7), e3, fma_(cho(4), e2, mul_(cho(1), e1)));
                        p6 = fma_(cho(8), e3, fma_(cho(5), e2, mul_(cho(2), e1)));
                    }
                    const int hb = hy * HX + hx;
                    IMs[0 * HP + hb] = e4; IMs[1 * HP + hb] = q45; IMs[2 * HP + hb] = q46;
                    IMs[3 * HP + hb] = e5; IMs[4 * HP + hb] = q56; IMs[5 * HP + hb] = e6;
                    IMs[6 * HP + hb] = p4; IMs[7 * HP + hb] = p5; IMs[8 * HP + hb] = p6;
                }
                if (hact) {
                    const int b = hvb, x = hxp, y = hyp;
                    if (hk == 0) {
                        float e4 = 0.f, q45 = 0.f, q46 = 0.f;
                        if (FAST || E.l4(x, y, p)) {
                            e4 = fma_(k1, sub_(Vp[2 * HS + b + BW], Vp[2 * HS + b]), mul_(k2, sub_(Vn[HS + b], Vp[HS + b])));
                            q45 = mul_(chh(9), e4);
                            q46 = mul_(chh(10), e4);
                        }
                        IMs[0 * HP + hhb] = e4; IMs[1 * HP + hhb] = q45; IMs[2 * HP + hhb] = q46;
                    } else if (hk == 1) {
                        float e5 = 0.f, q56 = 0.f;
                        if (FAST || E.l5(x, y, p)) {
                            e5 = fma_(k0, sub_(Vp[2 * HS + b], Vp[2 * HS + b - 1]), mul_(k2, sub_(Vn[b], Vp[b])));
                            q56 = mul_(chh(11), e5);
                        }
                        IMs[3 * HP + hhb] = e5; IMs[4 * HP + hhb] = q56;
                    } else if (hk == 2) {
                        float e6 = 0.f;
                        if (FAST || E.l6(x, y, p)) e6 = fma_(k0, sub_(Vp[HS + b], Vp[HS + b - 1]), mul_(k1, sub_(Vp[b + BW], Vp[b])));
                        IMs[5 * HP + hhb] = e6;
                    } else {
                        float p4 = 0.f, p5 = 0.f, p6 = 0.f;
                        if (FAST || E.n(x, y, p)) {
                            const float f1 = mul_(k0, sub_(Vp[b + 1], Vp[b]));
                            const float f2 = mul_(k1, sub_(Vp[HS + b], Vp[HS + b - BW]));
                            const float f3 = (!FAST && surf) ? e3_surface(x, y, p, g.idx(x, y, p), f1, f2)
                                                             : mul_(k2, sub_(Vp[2 * HS + b], Vm[2 * HS + b]));
                            p4 = fma_(chh(6), f3, fma_(chh(3), f2, mul_(chh(0), f1)));
                            p5 = fma_(chh(7), f3, fma_(chh(4), f2, mul_(chh(1), f1)));
                            p6 = fma_(chh(8), f3, fma_(chh(5), f2, mul_(chh(2), f1)));
                        }
                        IMs[6 * HP + hhb] = p4; IMs[7 * HP + hhb] = p5; IMs[8 * HP + hhb] = p6;
                    }
                }
                consumer_sync();
                if (flags[3 + (i & 1)]) return false;

                // ---- outputs: sigma_N, sigma_6 at plane p; sigma_4, sigma_5 at plane p-1
                if (inner) {
                    const int pp = pbase + p * sz;
                    if (FAST || E.n(ox, oy, p)) {
                        float v[2][2];
                        for (int k = 0; k < 2; k++) for (int j = 0; j < 2; j++) v[k][j] = RR(j, 0, hx, hy - 1 + k);
                        const float a4 = av(v, wyA, wzA);
                        for (int k = 0; k < 2; k++) for (int j = 0; j < 2; j++) v[k][j] = RR(j, 3, hx + k, hy);
                        const float a5 = av(v, wxA, wzA);
                        for (int k = 0; k < 2; k++) for (int j = 0; j < 2; j++) v[k][j] = RR(1, 5, hx + k, hy - 1 + j);
                        const float a6 = av(v, wxA, wyA);
                        const int rowc[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
                        float d[3];
#pragma unroll
                        for (int r = 0; r < 3; r++)
                            d[r] = fma_(cho(2 + 3 * r), a6,
                                        fma_(cho(1 + 3 * r), a5,
                                             fma_(cho(3 * r), a4,
                                                  fma_(CI[rowc[r][2] * IS + ib], e3,
                                                       fma_(CI[rowc[r][1] * IS + ib], e2, mul_(CI[rowc[r][0] * IS + ib], e1))))));
                        sxx[pp] = add_(SG[0 * IS + ib], d[0]);
                        syy[pp] = add_(SG[1 * IS + ib], d[1]);
                        if (FAST || !surf) szz[pp] = add_(SG[2 * IS + ib], d[2]);
                    }
                    if (FAST || E.l6(ox, oy, p)) {
                        float v[2][2];
                        for (int k = 0; k < 2; k++) for (int j = 0; j < 2; j++) v[k][j] = RR(j, 2, hx - 1 + k, hy);
                        const float t46 = av(v, wxB, wzA);
                        for (int k = 0; k < 2; k++) for (int j = 0; j < 2; j++) v[k][j] = RR(j, 4, hx, hy + k);
                        const float t56 = av(v, wyB, wzA);
                        for (int k = 0; k < 2; k++) for (int j = 0; j < 2; j++) v[k][j] = RR(1, 8, hx - 1 + k, hy + j);
                        const float t6 = av(v, wxB, wyB);
                        const float e6 = RR(1, 5, hx, hy);
                        const float dd = add_(add_(fma_(CI[8 * IS + ib], e6, t46), t56), t6);
                        sxy[pp] = add_(SG[5 * IS + ib], dd);
                    }
                }
                if (outer_pm) {
                    const int pp = pbase + pm * sz;
                    if (FAST || E.l4(ox, oy, pm)) {
                        float v[2][2];
                        for (int k = 0; k < 2; k++) for (int j = 0; j < 2; j++) v[k][j] = RR(0, 3, hx + k, hy + j);
                        const float t5 = av(v, wxA, wyB);
                        for (int k = 0; k < 2; k++) for (int j = 0; j < 2; j++) v[k][j] = RR(j, 5, hx + k, hy);
                        const float t6 = av(v, wxA, wzB);
                        for (int k = 0; k < 2; k++) for (int j = 0; j < 2; j++) v[k][j] = RR(j, 6, hx, hy + k);
                        const float tp = av(v, wyB, wzB);
                        const float e4 = RR(0, 0, hx, hy);
                        const float dd = add_(fma_(c17p, t6, fma_(c16p, t5, mul_(c15p, e4))), tp);
                        const float nv = add_(s3p, dd);
                        syz[pp] = nv;
                        if (flag && pm == 0) syz[pp - sz] = -nv;
                    }
                    if (FAST || E.l5(ox, oy, pm)) {
                        float v[2][2];
                        for (int k = 0; k < 2; k++) for (int j = 0; j < 2; j++) v[k][j] = RR(j, 5, hx, hy - 1 + k);
                        const float t6 = av(v, wyA, wzB);
                        for (int k = 0; k < 2; k++) for (int j = 0; j < 2; j++) v[k][j] = RR(0, 1, hx - 1 + k, hy - 1 + j);
                        const float t45 = av(v, wxB, wyA);
                        for (int k = 0; k < 2; k++) for (int j = 0; j < 2; j++) v[k][j] = RR(j, 7, hx - 1 + k, hy);
                        const float tp = av(v, wxB, wzB);
                        const float e5 = RR(0, 3, hx, hy);
                        const float dd = add_(add_(fma_(c19p, t6, mul_(c18p, e5)), t45), tp);
                        const float nv = add_(s4p, dd);
                        sxz[pp] = nv;
                        if (flag && pm == 0 && (FAST || (ox >= 1 && ox <= nx - 1 && oy >= 1 && oy <= ny - 1))) sxz[pp - sz] = -nv;
                    }
                }
                return true;
            };
            // fast planes: interior tile, 1 <= p <= nz-1 (not the free surface,
            // every closure weight 1/4 for the outputs at p and p-1)
            const bool go = (tile_in && p >= 1 && p <= nz - 1) ? body(std::true_type{}) : body(std::false_type{});
            if (!go) break;
            consumedP = i + 1;
            consumedV = i + 3;

            // displacement sums: U += v at this thread's point (x <= nx, y <= ny)
            // of an inner plane and of plane -1 (the grid's first stage), and
            // on inner planes the x = -1 / y = -1 face points beside it
            if (ACC && (inner || p == -1) && ox <= nx && oy <= ny) {
                const int pp = pbase + p * sz;
                u0[pp] = add_(EP[0 * IS + ib], Vp[0 * HS + vb]);
                u1[pp] = add_(EP[1 * IS + ib], Vp[1 * HS + vb]);
                u2[pp] = add_(EP[2 * IS + ib], Vp[2 * HS + vb]);
                if (inner && x0 == 0 && tx == 0) {
                    const float *EX = (const float *)(PS + P_EX);
                    constexpr int XS = XFBOX / 4;
                    u0[pp - 1] = add_(EX[0 * XS + ty * XFW + XFW - 1], Vp[0 * HS + vb - 1]);
                    u1[pp - 1] = add_(EX[1 * XS + ty * XFW + XFW - 1], Vp[1 * HS + vb - 1]);
                    u2[pp - 1] = add_(EX[2 * XS + ty * XFW + XFW - 1], Vp[2 * HS + vb - 1]);
                }
                if (inner && y0 == 0 && ty == 0) {
                    const float *EY = (const float *)(PS + P_EY);
                    constexpr int YS = YFBOX / 4;
                    u0[pp - g.px] = add_(EY[0 * YS + tx], Vp[0 * HS + vb - BW]);
                    u1[pp - g.px] = add_(EY[1 * YS + tx], Vp[1 * HS + vb - BW]);
                    u2[pp - g.px] = add_(EY[2 * YS + tx], Vp[2 * HS + vb - BW]);
                }
            }
            if (inner) {
                c15p = CI[6 * IS + ib]; c18p = CI[7 * IS + ib];
                c16p = cho(9); c17p = cho(10); c19p = cho(11);
                s3p = SG[3 * IS + ib]; s4p = SG[4 * IS + ib];
            }
            // every consumer is done with plane stage i's intermediates and slots
            consumer_sync();
            if (lane == 0) {
                mbar_arrive(emptyP(i % NSP));
                mbar_arrive(emptyV(i % NSV));
            }
        }
        if (tid == 0) {
            flags[1] = consumedP;
            flags[2] = consumedV;
            if (flags[3] || flags[4]) atomicOr(status, ST_PIPE_TIMEOUT);
        }
    }
    __syncthreads();
    // drain: copies issued but never consumed (only after a timeout) complete before exit
    if (warp == NT / 32 && lane == 0) {
        for (int i = flags[1]; i < issuedP; i++) mbar_wait(fullP(i % NSP), (i / NSP) & 1);
        for (int j = flags[2]; j < issuedV; j++) mbar_wait(fullV(j % NSV), (j / NSV) & 1);
    }
}

// ---------------------------------------------------------------------------
// Host side: tensor maps and launch
// ---------------------------------------------------------------------------
// true if ptr(k), k < count, are one field box apart
template <typename F>
static bool strided(const Geo &g, int count, F ptr)
{
    for (int k = 1; k < count; k++)
        if (ptr(k) != ptr(0) + (size_t)k * g.size()) return false;
    return true;
}

// Opaque storage for the maps of one grid (allocated by the caller, s21_maps_bytes()).
size_t s21_maps_bytes() { return sizeof(S21Maps<1>); }

// Fills the maps of one grid; false if the driver entry point is missing, a
// group is not laid out at a fixed stride, or an address / pitch is not
// encodable.
bool s21_encode_maps(void *out, const GridDev<float> &G, float *const disp[3])
{
    using namespace s21t;
    S21Maps<1> M;
    memset(&M, 0, sizeof M);
    M.ns = 1;
    for (int k = 0; k < 6; k++) M.sg_out[0][k] = G.f[SXX + k];
    for (int k = 0; k < 3; k++) M.vin[0][k] = G.f[VX + k];
    for (int k = 0; k < 3; k++) M.u[0][k] = disp ? disp[k] : nullptr;
    const Geo &g = G.g;
    if ((g.px * 4) % 16 != 0 || (XOFF - 4) % 4 != 0) return false;
    bool ok = strided(g, 3, [&](int k) { return (const float *)G.f[k]; }) &&
              strided(g, NCH, [&](int k) { return G.c[ch_slot(k)]; }) &&
              strided(g, NCI, [&](int k) { return G.c[ci_slot(k)]; }) &&
              strided(g, 6, [&](int k) { return (const float *)G.f[SXX + k]; });
    ok = ok && encode(&M.v[0], g, G.f[0], 3, BW, BH) && encode(&M.cha, g, G.c[ch_slot(0)], NCA, CW, CHH) &&
         encode(&M.chb, g, G.c[ch_slot(NCA)], NCB, CW, CHH) && encode(&M.chc, g, G.c[ch_slot(NCA + NCB)], 1, CW, CHH) &&
         encode(&M.ci, g, G.c[ci_slot(0)], NCI, TX, TY) && encode(&M.sg[0], g, G.f[SXX], 6, TX, TY);
    if (ok && disp && disp[0])
        ok = strided(g, 3, [&](int k) { return (const float *)disp[k]; }) && encode(&M.ep[0], g, disp[0], 3, TX, TY) &&
             encode(&M.epx[0], g, disp[0], 3, XFW, TY) && encode(&M.epy[0], g, disp[0], 3, TX, 1);
    if (ok) memcpy(out, &M, sizeof M);
    return ok;
}

// Opt-in to the kernel's shared memory; call outside stream capture.
cudaError_t s21_set_attributes()
{
    cudaError_t e = cudaFuncSetAttribute(stress21_tma_kernel<true, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, s21t::SMEM);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(stress21_tma_kernel<false, 1>, cudaFuncAttributeMaxDynamicSharedMemorySize, s21t::SMEM);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(stress21_tma_kernel<true, kMaxShots>, cudaFuncAttributeMaxDynamicSharedMemorySize, s21t::SMEM);
    if (e == cudaSuccess)
        e = cudaFuncSetAttribute(stress21_tma_kernel<false, kMaxShots>, cudaFuncAttributeMaxDynamicSharedMemorySize, s21t::SMEM);
    return e;
}

cudaError_t launch_stress21_tma(const void *maps, const GridDev<float> &G, int top, int top_bc, float *const disp[3],
                                int *status, int sms, cudaStream_t st, int nchunk_req)
{
    using namespace s21t;
    const Geo &g = G.g;
    const int flag = (top && top_bc) ? 1 : 0;
    const int bx = (g.nx + 1 + TX - 1) / TX, by = (g.ny + 1 + TY - 1) / TY;
    const int64_t cols = (int64_t)bx * by;
    // one CTA per SM: aim for >= 4 waves, chunks of >= 24 planes
    int nchunk = (int)(((int64_t)sms * 4 + cols - 1) / cols);
    if (nchunk < 1) nchunk = 1;
    const int maxc = (g.nz + 1) / 24 > 0 ? (g.nz + 1) / 24 : 1;
    if (nchunk > maxc) nchunk = maxc;
    if (nchunk_req > 0) nchunk = nchunk_req < g.nz + 1 ? nchunk_req : g.nz + 1;   // tuned
    const int zc = (g.nz + 1 + nchunk - 1) / nchunk;
    dim3 grd(bx, by, (g.nz + 1 + zc - 1) / zc);
    const S21Maps<1> &M = *(const S21Maps<1> *)maps;
    if (disp && disp[0]) {
        stress21_tma_kernel<true, 1><<<grd, NTHREADS, SMEM, st>>>(M, G, flag, zc, status);
    } else {
        stress21_tma_kernel<false, 1><<<grd, NTHREADS, SMEM, st>>>(M, G, flag, zc, status);
    }
    return cudaGetLastError();
}

// The sweep of ns shots of one grid sharing the medium (same geometry, same
// coefficients): maps[s] is shot s's opaque map block (s21_encode_maps); the
// coefficient maps are taken from shot 0's.  Same launch shape as one shot
// per tile column, with the shots' CTAs of a column adjacent.
cudaError_t launch_stress21_tma_shots(const void *const *maps, int ns, const GridDev<float> &G, int top, int top_bc,
                                      bool acc, int *status, int sms, cudaStream_t st, int nchunk_req)
{
    using namespace s21t;
    if (ns < 1 || ns > kMaxShots) return cudaErrorInvalidValue;
    static thread_local S21Maps<kMaxShots> M;   // host staging of the kernel parameter (2 KB of maps per shot)
    memset(&M, 0, sizeof M);
    const S21Maps<1> &M0 = *(const S21Maps<1> *)maps[0];
    M.cha = M0.cha;
    M.chb = M0.chb;
    M.chc = M0.chc;
    M.ci = M0.ci;
    M.ns = ns;
    for (int s = 0; s < ns; s++) {
        const S21Maps<1> &Ms = *(const S21Maps<1> *)maps[s];
        M.v[s] = Ms.v[0];
        M.sg[s] = Ms.sg[0];
        M.ep[s] = Ms.ep[0];
        M.epx[s] = Ms.epx[0];
        M.epy[s] = Ms.epy[0];
        for (int k = 0; k < 6; k++) M.sg_out[s][k] = Ms.sg_out[0][k];
        for (int k = 0; k < 3; k++) M.vin[s][k] = Ms.vin[0][k];
        for (int k = 0; k < 3; k++) M.u[s][k] = Ms.u[0][k];
        if (acc && !Ms.u[0][0]) return cudaErrorInvalidValue;
    }
    const Geo &g = G.g;
    const int flag = (top && top_bc) ? 1 : 0;
    const int bx = (g.nx + 1 + TX - 1) / TX, by = (g.ny + 1 + TY - 1) / TY;
    const int64_t cols = (int64_t)bx * by * ns;
    int nchunk = (int)(((int64_t)sms * 4 + cols - 1) / cols);
    if (nchunk < 1) nchunk = 1;
    const int maxc = (g.nz + 1) / 24 > 0 ? (g.nz + 1) / 24 : 1;
    if (nchunk > maxc) nchunk = maxc;
    if (nchunk_req > 0) nchunk = nchunk_req < g.nz + 1 ? nchunk_req : g.nz + 1;
    const int zc = (g.nz + 1 + nchunk - 1) / nchunk;
    dim3 grd(bx * ns, by, (g.nz + 1 + zc - 1) / zc);
    if (acc)
        stress21_tma_kernel<true, kMaxShots><<<grd, NTHREADS, SMEM, st>>>(M, G, flag, zc, status);
    else
        stress21_tma_kernel<false, kMaxShots><<<grd, NTHREADS, SMEM, st>>>(M, G, flag, zc, status);
    return cudaGetLastError();
}

} // namespace ecsg
