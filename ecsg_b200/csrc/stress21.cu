// stress21.cu -- general anisotropic (21 Cij) stress update of one uniform sub-grid.
//
// No reference counterpart: the reference implements the orthorhombic form
// (update_stress.cpp:17-133), which this update reduces to when the 12
// off-block entries vanish.  Voigt stiffness, engineering shear strains.
// Medium slots (all R = 0 position fields in the grid's box):
//   N  (normal-stress position, 1,0,0): 0 C11 1 C12 2 C13 3 C22 4 C23 5 C33
//       6 C14 7 C15 8 C16 9 C24 10 C25 11 C26 12 C34 13 C35 14 C36
//   L4 (syz, 1,1,1): 15 C44 16 C45 17 C46;  L5 (sxz, 0,0,1): 18 C55 19 C56;
//   L6 (sxy, 0,1,0): 20 C66.
// A coupling between two positions uses one coefficient per link, stored at
// one end (N for N-L4/L5/L6, L4 for L4-L5 and L4-L6, L5 for L5-L6), and is
// applied in both directions: the stress at one end gets coefficient x the
// average of the other end's strain, the stress at the other end gets the
// average of coefficient x strain.  The discrete stiffness operator is then
// symmetric and 1/2 (rho v, v') + 1/2 (eps, sigma) is conserved.  Averages
// drop neighbours outside a position's extent (interface and mirror planes
// count as outside), the closure that matches the trapezoid energy weights.
// On a free surface szz is held and e3 takes the value that keeps its rate 0.
//
// Work layout: a CTA owns a TX x TY tile of (x,y) indices and marches z.  Per
// plane it computes, on the tile plus a one-point halo, the strains and link
// products every output needs (e4 Q45 Q46 at L4, e5 Q56 at L5, e6 at L6,
// P4 P5 P6 at N) into a two-plane shared-memory ring, then updates sigma_N and
// sigma_6 of this plane and sigma_4, sigma_5 of the half-plane below.  Every
// velocity and stiffness word comes from HBM once per sweep; the halo points'
// recomputation reads L1/L2.
//
// Optional displacement sums U[3] (the velocities summed over the stress
// updates, at the velocity positions) make the energy computable without
// inverting the stiffness operator: the strains are linear in the
// velocities, so the accumulated strain at every stress position is the
// strain difference of U (gen21_device.cuh), three fields where strain
// accumulators would take six.  Each update adds the velocities it reads on
// U's support: x in [0, nx], y in [0, ny], z in [0, nz] plus the faces
// x = -1, y = -1 and z = -1 that the strain differences reach into.
#include "gen21_device.cuh"

namespace ecsg {

template <typename T>
struct S21 {
    static constexpr int TX = 32;
    static constexpr int TY = sizeof(T) == 4 ? 8 : 4;
    static constexpr int HX = TX + 2, HY = TY + 2, HP = HX * HY;
    static constexpr int NQ = 9;   // e4 Q45 Q46 e5 Q56 e6 P4 P5 P6
};
enum { Q_E4 = 0, Q_Q45, Q_Q46, Q_E5, Q_Q56, Q_E6, Q_P4, Q_P5, Q_P6 };

// U += v on the support of the displacement sums owned by the output point
// (x, y) of plane z: the point itself (x <= nx, y <= ny), its x = -1 / y = -1
// face neighbours when x / y is 0, and the z = -1 point below when lower.
template <typename T>
__device__ __forceinline__ void add_velocities(const GridDev<T> &G, T *u0, T *u1, T *u2, int x, int y, int z, bool lower)
{
    const Geo &g = G.g;
    if (x > g.nx || y > g.ny) return;
    T *const u[3] = {u0, u1, u2};
    const int p = g.idx(x, y, z);
    const int sy = g.px, sz = g.px * g.py;
#pragma unroll
    for (int c = 0; c < 3; c++) {
        const T *v = G.f[VX + c];
        u[c][p] = add_(u[c][p], v[p]);
        if (x == 0) u[c][p - 1] = add_(u[c][p - 1], v[p - 1]);
        if (y == 0) u[c][p - sy] = add_(u[c][p - sy], v[p - sy]);
        if (lower) u[c][p - sz] = add_(u[c][p - sz], v[p - sz]);
    }
}

template <typename T, bool ACC>
__global__ void __launch_bounds__(S21<T>::TX *S21<T>::TY) stress21_kernel(GridDev<T> G, int flag, int zchunk, T *u0, T *u1, T *u2)
{
    using C = S21<T>;
    __shared__ T ring[2][C::NQ][C::HP];
    const Geo &g = G.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const Ext E{nx, ny, nz};
    const int tx = threadIdx.x, ty = threadIdx.y, tid = ty * C::TX + tx, nth = C::TX * C::TY;
    const int x0 = blockIdx.x * C::TX, y0 = blockIdx.y * C::TY;
    const int z0 = blockIdx.z * zchunk;
    const int z1 = min(nz, z0 + zchunk - 1);
    const int sz = g.px * g.py;
    T *sxx = G.f[SXX], *syy = G.f[SYY], *szz = G.f[SZZ], *syz = G.f[SYZ], *sxz = G.f[SXZ], *sxy = G.f[SXY];
    const T *const *c = G.c;
    const int ox = x0 + tx, oy = y0 + ty;   // this thread's output index
    auto R = [&](int slot, int q, int hx, int hy) -> T & { return ring[slot][q][hy * C::HX + hx]; };

    for (int p = z0 - 1; p <= z1 + 1; p++) {
        const int s = p & 1;
        // phase A: L4, L5, L6 intermediates of plane p on the haloed tile
        for (int q = tid; q < C::HP; q += nth) {
            const int hx = q % C::HX, hy = q / C::HX;
            const int x = x0 - 1 + hx, y = y0 - 1 + hy;
            T e4 = T(0), q45 = T(0), q46 = T(0), e5 = T(0), q56 = T(0), e6 = T(0);
            if (E.l4(x, y, p)) {
                const int pp = g.idx(x, y, p);
                e4 = e4_at(G, pp);
                q45 = mul_(c[16][pp], e4);
                q46 = mul_(c[17][pp], e4);
            }
            if (E.l5(x, y, p)) {
                const int pp = g.idx(x, y, p);
                e5 = e5_at(G, pp);
                q56 = mul_(c[19][pp], e5);
            }
            if (E.l6(x, y, p)) e6 = e6_at(G, g.idx(x, y, p));
            R(s, Q_E4, hx, hy) = e4;
            R(s, Q_Q45, hx, hy) = q45;
            R(s, Q_Q46, hx, hy) = q46;
            R(s, Q_E5, hx, hy) = e5;
            R(s, Q_Q56, hx, hy) = q56;
            R(s, Q_E6, hx, hy) = e6;
        }
        // phase B: N link products P4 P5 P6 of plane p
        for (int q = tid; q < C::HP; q += nth) {
            const int hx = q % C::HX, hy = q / C::HX;
            const int x = x0 - 1 + hx, y = y0 - 1 + hy;
            T p4 = T(0), p5 = T(0), p6 = T(0);
            if (E.n(x, y, p)) {
                const int pp = g.idx(x, y, p);
                const T e1 = e1_at(G, pp), e2 = e2_at(G, pp);
                const T e3 = e3_used(G, E, flag && p == 0, x, y, p, pp, e1, e2);
                p4 = fma_(c[12][pp], e3, fma_(c[9][pp], e2, mul_(c[6][pp], e1)));
                p5 = fma_(c[13][pp], e3, fma_(c[10][pp], e2, mul_(c[7][pp], e1)));
                p6 = fma_(c[14][pp], e3, fma_(c[11][pp], e2, mul_(c[8][pp], e1)));
            }
            R(s, Q_P4, hx, hy) = p4;
            R(s, Q_P5, hx, hy) = p5;
            R(s, Q_P6, hx, hy) = p6;
        }
        __syncthreads();
        // phase C: outputs
        const int hx = tx + 1, hy = ty + 1;
        const int sp = (p - 1) & 1;   // slot of plane p-1
        if (p >= z0 && p <= z1) {
            if (E.n(ox, oy, p)) {
                const int pp = g.idx(ox, oy, p);
                const bool surf = flag && p == 0;
                const T e1 = e1_at(G, pp), e2 = e2_at(G, pp);
                const T e3 = e3_used(G, E, surf, ox, oy, p, pp, e1, e2);
                T v[2][2];
                bool a[2], b[2];
                // Abar4: L4 (x, y-1..y, p-1..p)
                for (int i = 0; i < 2; i++) { a[i] = (oy - 1 + i) >= 0 && (oy - 1 + i) <= ny - 1; b[i] = (p - 1 + i) >= 0 && (p - 1 + i) <= nz - 1; }
                for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) v[i][j] = R(j == 0 ? sp : s, Q_E4, hx, hy - 1 + i);
                const T a4 = avg4<T>(v, a, b);
                // Abar5: L5 (x..x+1, y, p-1..p)
                for (int i = 0; i < 2; i++) { a[i] = (ox + i) <= nx; b[i] = (p - 1 + i) >= 0 && (p - 1 + i) <= nz - 1; }
                for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) v[i][j] = R(j == 0 ? sp : s, Q_E5, hx + i, hy);
                const T a5 = avg4<T>(v, a, b);
                // Abar6: L6 (x..x+1, y-1..y, p)
                for (int i = 0; i < 2; i++) { a[i] = (ox + i) <= nx; b[i] = (oy - 1 + i) >= 0 && (oy - 1 + i) <= ny - 1; }
                for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) v[i][j] = R(s, Q_E6, hx + i, hy - 1 + j);
                const T a6 = avg4<T>(v, a, b);
                const int rowc[3][3] = {{0, 1, 2}, {1, 3, 4}, {2, 4, 5}};
                T d[3];
#pragma unroll
                for (int r = 0; r < 3; r++)
                    d[r] = fma_(c[8 + 3 * r][pp], a6,
                                fma_(c[7 + 3 * r][pp], a5,
                                     fma_(c[6 + 3 * r][pp], a4,
                                          fma_(c[rowc[r][2]][pp], e3, fma_(c[rowc[r][1]][pp], e2, mul_(c[rowc[r][0]][pp], e1))))));
                sxx[pp] = add_(sxx[pp], d[0]);
                syy[pp] = add_(syy[pp], d[1]);
                if (!surf) szz[pp] = add_(szz[pp], d[2]);
            }
            if (E.l6(ox, oy, p)) {
                const int pp = g.idx(ox, oy, p);
                T v[2][2];
                bool a[2], b[2];
                // Q46 over L4 (x-1..x, y, p-1..p)
                for (int i = 0; i < 2; i++) { a[i] = (ox - 1 + i) >= 0 && (ox - 1 + i) <= nx - 1; b[i] = (p - 1 + i) >= 0 && (p - 1 + i) <= nz - 1; }
                for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) v[i][j] = R(j == 0 ? sp : s, Q_Q46, hx - 1 + i, hy);
                const T t46 = avg4<T>(v, a, b);
                // Q56 over L5 (x, y..y+1, p-1..p)
                for (int i = 0; i < 2; i++) { a[i] = (oy + i) <= ny; b[i] = (p - 1 + i) >= 0 && (p - 1 + i) <= nz - 1; }
                for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) v[i][j] = R(j == 0 ? sp : s, Q_Q56, hx, hy + i);
                const T t56 = avg4<T>(v, a, b);
                // P6 over N (x-1..x, y..y+1, p)
                for (int i = 0; i < 2; i++) { a[i] = (ox - 1 + i) >= 0 && (ox - 1 + i) <= nx - 1; b[i] = (oy + i) <= ny; }
                for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) v[i][j] = R(s, Q_P6, hx - 1 + i, hy + j);
                const T t6 = avg4<T>(v, a, b);
                const T e6 = R(s, Q_E6, hx, hy);
                const T dd = add_(add_(fma_(c[20][pp], e6, t46), t56), t6);
                sxy[pp] = add_(sxy[pp], dd);
            }
        }
        if (ACC && p >= z0 && p <= z1) add_velocities(G, u0, u1, u2, ox, oy, p, z0 == 0 && p == 0);
        const int pm = p - 1;
        if (pm >= z0 && pm <= z1) {
            if (E.l4(ox, oy, pm)) {
                const int pp = g.idx(ox, oy, pm);
                T v[2][2];
                bool a[2], b[2];
                // e5 over L5 (x..x+1, y..y+1, pm)
                for (int i = 0; i < 2; i++) { a[i] = (ox + i) <= nx; b[i] = (oy + i) <= ny; }
                for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) v[i][j] = R(sp, Q_E5, hx + i, hy + j);
                const T t5 = avg4<T>(v, a, b);
                // e6 over L6 (x..x+1, y, pm..pm+1)
                for (int i = 0; i < 2; i++) { a[i] = (ox + i) <= nx; b[i] = (pm + i) <= nz; }
                for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) v[i][j] = R(j == 0 ? sp : s, Q_E6, hx + i, hy);
                const T t6 = avg4<T>(v, a, b);
                // P4 over N (x, y..y+1, pm..pm+1)
                for (int i = 0; i < 2; i++) { a[i] = (oy + i) <= ny; b[i] = (pm + i) <= nz; }
                for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) v[i][j] = R(j == 0 ? sp : s, Q_P4, hx, hy + i);
                const T tp = avg4<T>(v, a, b);
                const T e4 = R(sp, Q_E4, hx, hy);
                const T dd = add_(fma_(c[17][pp], t6, fma_(c[16][pp], t5, mul_(c[15][pp], e4))), tp);
                const T nv = add_(syz[pp], dd);
                syz[pp] = nv;
                if (flag && pm == 0) syz[pp - sz] = -nv;
            }
            if (E.l5(ox, oy, pm)) {
                const int pp = g.idx(ox, oy, pm);
                T v[2][2];
                bool a[2], b[2];
                // e6 over L6 (x, y-1..y, pm..pm+1)
                for (int i = 0; i < 2; i++) { a[i] = (oy - 1 + i) >= 0 && (oy - 1 + i) <= ny - 1; b[i] = (pm + i) <= nz; }
                for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) v[i][j] = R(j == 0 ? sp : s, Q_E6, hx, hy - 1 + i);
                const T t6 = avg4<T>(v, a, b);
                // Q45 over L4 (x-1..x, y-1..y, pm)
                for (int i = 0; i < 2; i++) { a[i] = (ox - 1 + i) >= 0 && (ox - 1 + i) <= nx - 1; b[i] = (oy - 1 + i) >= 0 && (oy - 1 + i) <= ny - 1; }
                for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) v[i][j] = R(sp, Q_Q45, hx - 1 + i, hy - 1 + j);
                const T t45 = avg4<T>(v, a, b);
                // P5 over N (x-1..x, y, pm..pm+1)
                for (int i = 0; i < 2; i++) { a[i] = (ox - 1 + i) >= 0 && (ox - 1 + i) <= nx - 1; b[i] = (pm + i) <= nz; }
                for (int i = 0; i < 2; i++) for (int j = 0; j < 2; j++) v[i][j] = R(j == 0 ? sp : s, Q_P5, hx - 1 + i, hy);
                const T tp = avg4<T>(v, a, b);
                const T e5 = R(sp, Q_E5, hx, hy);
                const T dd = add_(add_(fma_(c[19][pp], t6, mul_(c[18][pp], e5)), t45), tp);
                const T nv = add_(sxz[pp], dd);
                sxz[pp] = nv;
                if (flag && pm == 0 && ox >= 1 && ox <= nx - 1 && oy >= 1 && oy <= ny - 1) sxz[pp - sz] = -nv;
            }
        }
        __syncthreads();
    }
}

template <typename T>
cudaError_t launch_stress21(const GridDev<T> &G, int top, int top_bc, T *const disp[3], int sms, cudaStream_t st)
{
    using C = S21<T>;
    const Geo &g = G.g;
    const int flag = (top && top_bc) ? 1 : 0;
    const int bx = (g.nx + 1 + C::TX - 1) / C::TX, by = (g.ny + 1 + C::TY - 1) / C::TY;
    const int64_t cols = (int64_t)bx * by;
    int nchunk = (int)(((int64_t)sms * 4 + cols - 1) / cols);
    if (nchunk < 1) nchunk = 1;
    if (nchunk > (g.nz + 1) / 8 + 1) nchunk = (g.nz + 1) / 8 + 1;   // keep >= ~8 planes per CTA (2 recomputed)
    const int zc = (g.nz + 1 + nchunk - 1) / nchunk;
    dim3 blk(C::TX, C::TY), grd(bx, by, (g.nz + 1 + zc - 1) / zc);
    if (disp && disp[0])
        stress21_kernel<T, true><<<grd, blk, 0, st>>>(G, flag, zc, disp[0], disp[1], disp[2]);
    else
        stress21_kernel<T, false><<<grd, blk, 0, st>>>(G, flag, zc, nullptr, nullptr, nullptr);
    return cudaGetLastError();
}

template cudaError_t launch_stress21<float>(const GridDev<float> &, int, int, float *const[3], int, cudaStream_t);
template cudaError_t launch_stress21<double>(const GridDev<double> &, int, int, double *const[3], int, cudaStream_t);

} // namespace ecsg
