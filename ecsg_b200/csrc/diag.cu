// diag.cu -- energy, interface residues, source injection / receiver sampling,
// medium set-up and host-layout conversion kernels.
//
// Reductions are deterministic: each CTA reduces its grid-stride share in a
// fixed tree and writes one partial per term; a single-CTA finalize sums the
// partials in CTA order.  Accumulation is in double precision.
#include "ecsg_device.cuh"
#include "gen21_device.cuh"

#include <type_traits>

namespace ecsg {

constexpr int RED_THREADS = 256;

template <int N>
__device__ __forceinline__ void block_sums(double (&v)[N], double *partial, int nblocks)
{
    __shared__ double red[N][RED_THREADS / 32];
    const int w = threadIdx.x >> 5, l = threadIdx.x & 31;
#pragma unroll
    for (int k = 0; k < N; k++) {
        double x = v[k];
        for (int o = 16; o > 0; o >>= 1) x += __shfl_down_sync(0xffffffffu, x, o);
        if (l == 0) red[k][w] = x;
    }
    __syncthreads();
    if (threadIdx.x < N) {
        double s = 0.0;
        for (int i = 0; i < RED_THREADS / 32; i++) s += red[threadIdx.x][i];
        partial[threadIdx.x * nblocks + blockIdx.x] = s;
    }
}

// ---------------------------------------------------------------------------
// Energy of one grid, compute_energy.cpp:34-54 with TriMulFields
// (field.cpp:482-518).  Densities and compliances are formed on the fly with
// the reference's operation order (InvertParameters, init_del_par_field.cpp:224-283;
// ReshapeField, field.cpp:465-472).  12 term partials per CTA.
// ---------------------------------------------------------------------------
// 21-Cij media: the potential energy 1/2 (eps, sigma) takes the accumulated
// strains as the strain differences of the displacement sums U (stress21.cu),
// evaluated by the stress update's own strain functions on a copy of the grid
// whose velocities are U (GU), e3 condensed on a free surface (flag).
//
// Work is split into tiles of 32 x 8 (x, y) columns by ENERGY_ZC planes; a
// CTA takes tiles blockIdx.x, blockIdx.x + gridDim.x, ... and each thread
// marches z down its column (no per-point index division; neighbours in
// x and y come from the same or an adjacent column, in z from the plane
// before or after, all cached).  The medium kind is a template parameter so
// each kernel holds only its own arithmetic.  The accumulation order is
// fixed by the launch shape, so the result is the same on every run.
constexpr int ENERGY_TX = 32, ENERGY_TY = 8, ENERGY_ZC = 16;

// FP32 fields, 21-Cij medium (the production path): each point's terms in
// FP32 (the precision of the fields they multiply), the point's kinetic and
// potential parts added to two FP64 sums (the finalize of this medium only
// adds the terms up, so the per-term split is not kept).  A thread marches z
// down its column: the values a plane shares with the one before (the
// buoyancy and the displacement sums at p, which the plane before read at
// p + sz, and uz at p - sz) come along in registers, and every other load of
// the point is issued first and unconditionally (the neighbours at n + 1
// and -1 lie in the halo of every box); the terms outside the point's
// position sets are dropped by selects afterwards.  The kinetic terms divide
// by the buoyancy means with __fdividef (within 2 ulp).
struct EnergyCarry {
    float b0, b1, ux0, uy0, uzm;   // b(p), b(p+1), ux(p), uy(p), uz(p - sz)
};

__device__ __forceinline__ void energy_carry_init(const GridDev<float> &G, const GridDev<float> &GU, int p, EnergyCarry &c)
{
    const int sz = G.g.px * G.g.py;
    c.b0 = G.b[p];
    c.b1 = G.b[p + 1];
    c.ux0 = GU.f[VX][p];
    c.uy0 = GU.f[VY][p];
    c.uzm = GU.f[VZ][p - sz];
}

__device__ __forceinline__ void energy_point_f32_gen21(const GridDev<float> &G, const GridDev<float> &GU, const float *vc0,
                                                       const float *vc1, const float *vc2, int flag, int x, int y, int z,
                                                       int p, EnergyCarry &cr, double &kin, double &pot)
{
    const Geo &g = G.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int sy = g.px, sz = g.px * g.py;
    const float *b = G.b;
    const float b000 = cr.b0, b100 = cr.b1, b010 = b[p + sy], b110 = b[p + sy + 1], b001 = b[p + sz], b101 = b[p + sz + 1];
    const float vx = G.f[VX][p], vy = G.f[VY][p], vz = G.f[VZ][p], c0 = vc0[p], c1 = vc1[p], c2 = vc2[p];
    const float sxx = G.f[SXX][p], syy = G.f[SYY][p], szz = G.f[SZZ][p];
    const float syz = G.f[SYZ][p], sxz = G.f[SXZ][p], sxy = G.f[SXY][p];
    const float *ux = GU.f[VX], *uy = GU.f[VY], *uz = GU.f[VZ];
    const float ux0 = cr.ux0, ux1 = ux[p + 1], uxy = ux[p + sy], uxz = ux[p + sz];
    const float uy0 = cr.uy0, uym = uy[p - sy], uyx = uy[p - 1], uyz = uy[p + sz];
    const float uz0 = uz[p], uzm = cr.uzm, uzx = uz[p - 1], uzy = uz[p + sy];
    cr.b0 = b001;
    cr.b1 = b101;
    cr.ux0 = uxz;
    cr.uy0 = uyz;
    cr.uzm = uz0;
    const float k0 = GU.k[0], k1 = GU.k[1], k2 = GU.k[2];
    const float mx = (x == 0 || x == nx) ? 0.5f : 1.0f;
    const float my = (y == 0 || y == ny) ? 0.5f : 1.0f;
    const float mz = (z == 0 || z == nz) ? 0.5f : 1.0f;
    const bool xs = x < nx, ys = y < ny, zs = z < nz;
    // the strain functions of the stress update (e1_at .. e6_at), same operations
    const float e1 = k0 * (ux1 - ux0), e2 = k1 * (uy0 - uym);
    float e3 = k2 * (uz0 - uzm);
    const float e4 = __fmaf_rn(k1, uzy - uz0, k2 * (uyz - uy0));
    const float e5 = __fmaf_rn(k0, uz0 - uzx, k2 * (uxz - ux0));
    const float e6 = __fmaf_rn(k0, uy0 - uyx, k1 * (uxy - ux0));
    float k = __fdividef(mz * my * mx * (vx * c0), b000);
    const float ky = __fdividef(mz * (vy * c1), 0.25f * (b000 + b010 + b100 + b110));
    const float kz = __fdividef(my * (vz * c2), 0.25f * (b000 + b001 + b100 + b101));
    if (xs && ys) k += ky;
    if (xs && zs) k += kz;
    if (flag && z == 0 && xs) e3 = e3_used(GU, Ext{nx, ny, nz}, true, x, y, z, p, e1, e2);
    float e = 0.0f;
    const float w = mz * my;
    const float en = w * (e1 * sxx + e2 * syy + e3 * szz);
    const float e44 = e4 * syz, e55 = my * mx * e5 * sxz, e66 = mz * mx * e6 * sxy;
    if (xs) e += en;
    if (xs && ys && zs) e += e44;
    if (zs) e += e55;
    if (ys) e += e66;
    kin += (double)k;
    pot += (double)e;
}

// The FP32 21-Cij energy: 4 CTAs per SM, one plane per thread at a time (64
// registers, no spills; two planes in flight spilled and measured 4 % slower,
// 5 and 6 CTAs per SM spilled and measured 32 % and 44 % slower).
__global__ void __launch_bounds__(RED_THREADS, 4)
    energy_f32_gen21_kernel(GridDev<float> G, const float *vc0, const float *vc1, const float *vc2, GridDev<float> GU,
                            int flag, double *partial)
{
    const Geo &g = G.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int sz = g.px * g.py;
    const int ntx = (nx + ENERGY_TX) / ENERGY_TX, nty = (ny + ENERGY_TY) / ENERGY_TY;
    const int ntz = (nz + ENERGY_ZC) / ENERGY_ZC;
    const int ntiles = ntx * nty * ntz;
    const int lx = threadIdx.x % ENERGY_TX, ly = threadIdx.x / ENERGY_TX;
    double kin = 0.0, pot = 0.0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int tx = t % ntx, ty = (t / ntx) % nty, tz = t / (ntx * nty);
        const int x = tx * ENERGY_TX + lx, y = ty * ENERGY_TY + ly;
        if (x > nx || y > ny) continue;
        const int z0 = tz * ENERGY_ZC, z1 = min(nz, z0 + ENERGY_ZC - 1);
        int p = g.idx(x, y, z0);
        EnergyCarry cr;
        energy_carry_init(G, GU, p, cr);
        for (int z = z0; z <= z1; z++, p += sz) energy_point_f32_gen21(G, GU, vc0, vc1, vc2, flag, x, y, z, p, cr, kin, pot);
    }
    double acc[12] = {kin, 0.0, 0.0, pot, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0, 0.0};
    block_sums<12>(acc, partial, gridDim.x);
}

template <typename T, int MED>
__device__ __forceinline__ void energy_point(const GridDev<T> &G, const GridDev<T> &GU, const T *vc0, const T *vc1,
                                             const T *vc2, int flag, int x, int y, int z, int p, double (&acc)[12])
{

    const Geo &g = G.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int sy = g.px, sz = g.px * g.py;
    const double mx = (x == 0 || x == nx) ? 0.5 : 1.0;
    const double my = (y == 0 || y == ny) ? 0.5 : 1.0;
    const double mz = (z == 0 || z == nz) ? 0.5 : 1.0;
    const bool xs = x < nx, ys = y < ny, zs = z < nz;
    const double b000 = (double)G.b[p];
    // vx at (0,0,0)
    acc[0] += mz * my * mx * (1.0 / b000) * (double)G.f[VX][p] * (double)vc0[p];
    if (xs && ys) {   // vy at (1,1,0)
        const double b100 = (double)G.b[p + 1], b010 = (double)G.b[p + sy], b110 = (double)G.b[p + sy + 1];
        const double rb = (b000 + b000 + b010 + b010 + b100 + b100 + b110 + b110) / 8;
        acc[1] += mz * (1.0 / rb) * (double)G.f[VY][p] * (double)vc1[p];
    }
    if (xs && zs) {   // vz at (1,0,1)
        const double b001 = (double)G.b[p + sz], b100 = (double)G.b[p + 1], b101 = (double)G.b[p + sz + 1];
        const double rb = (b000 + b001 + b000 + b001 + b100 + b101 + b100 + b101) / 8;
        acc[2] += my * (1.0 / rb) * (double)G.f[VZ][p] * (double)vc2[p];
    }
    if (MED == MED_GEN21) {
        // terms 3..8 in stress order, trapezoid weights per position
        if (xs) {
            const double w = mz * my;
            const T e1 = e1_at(GU, p), e2 = e2_at(GU, p);
            const T e3 = (flag && z == 0) ? e3_used(GU, Ext{nx, ny, nz}, true, x, y, z, p, e1, e2) : e3_at(GU, p);
            acc[3] += w * (double)e1 * (double)G.f[SXX][p];
            acc[4] += w * (double)e2 * (double)G.f[SYY][p];
            acc[5] += w * (double)e3 * (double)G.f[SZZ][p];
        }
        if (xs && ys && zs) acc[6] += (double)e4_at(GU, p) * (double)G.f[SYZ][p];
        if (zs) acc[7] += my * mx * (double)e5_at(GU, p) * (double)G.f[SXZ][p];
        if (ys) acc[8] += mz * mx * (double)e6_at(GU, p) * (double)G.f[SXY][p];
        return;
    }
    if (xs) {         // normal stresses at (1,0,0)
        double k11, k22, k33, k23, k13, k12;
        if (MED == MED_ISO5) {
            const double s11 = (double)G.c[0][p], s13 = (double)G.c[1][p];
            double base = s11 * s13 * s13 * 3 - s13 * s13 * s13 * 2 - s11 * s11 * s11;
            base = 1.0 / base;
            k11 = k22 = k33 = (s13 * s13 - s11 * s11) * base;
            k23 = k13 = k12 = (s13 * s11 - s13 * s13) * base;
        } else {
            const double a = (double)G.c[0][p], e = (double)G.c[1][p], i = (double)G.c[2][p];
            const double f = (double)G.c[3][p], c = (double)G.c[4][p], bb = (double)G.c[5][p];
            // inverse of [[a,bb,c],[bb,e,f],[c,f,i]]
            const double A = e * i - f * f, Bq = -(bb * i - f * c), Cq = bb * f - e * c;
            const double det = a * A + bb * Bq + c * Cq;
            const double id = 1.0 / det;
            k11 = A * id;
            k12 = Bq * id;
            k13 = Cq * id;
            k22 = (a * i - c * c) * id;
            k23 = -(a * f - bb * c) * id;
            k33 = (a * e - bb * bb) * id;
        }
        const double w = mz * my;
        const double sxx = (double)G.f[SXX][p], syy = (double)G.f[SYY][p], szz = (double)G.f[SZZ][p];
        acc[3] += w * k11 * sxx * sxx;
        acc[4] += w * k22 * syy * syy;
        acc[5] += w * k33 * szz * szz;
        acc[6] += w * k23 * syy * szz;
        acc[7] += w * k13 * sxx * szz;
        acc[8] += w * k12 * sxx * syy;
    }
    constexpr int s44 = MED == MED_ISO5 ? 2 : 6;
    if (xs && ys && zs) {   // syz at (1,1,1)
        const double s = (double)G.f[SYZ][p];
        acc[9] += (1.0 / (double)G.c[s44][p]) * s * s;
    }
    if (zs) {               // sxz at (0,0,1)
        const double s = (double)G.f[SXZ][p];
        acc[10] += my * mx * (1.0 / (double)G.c[s44 + 1][p]) * s * s;
    }
    if (ys) {               // sxy at (0,1,0)
        const double s = (double)G.f[SXY][p];
        acc[11] += mz * mx * (1.0 / (double)G.c[s44 + 2][p]) * s * s;
    }
}

template <typename T, int MED>
__global__ void __launch_bounds__(RED_THREADS, 3) energy_kernel(GridDev<T> G, const T *vc0, const T *vc1, const T *vc2,
                                                            GridDev<T> GU, int flag, double *partial)
{
    const Geo &g = G.g;
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int sz = g.px * g.py;
    const int ntx = (nx + ENERGY_TX) / ENERGY_TX, nty = (ny + ENERGY_TY) / ENERGY_TY;
    const int ntz = (nz + ENERGY_ZC) / ENERGY_ZC;
    const int ntiles = ntx * nty * ntz;
    const int lx = threadIdx.x % ENERGY_TX, ly = threadIdx.x / ENERGY_TX;
    double acc[12];
#pragma unroll
    for (int k = 0; k < 12; k++) acc[k] = 0.0;
    for (int t = blockIdx.x; t < ntiles; t += gridDim.x) {
        const int tx = t % ntx, ty = (t / ntx) % nty, tz = t / (ntx * nty);
        const int x = tx * ENERGY_TX + lx, y = ty * ENERGY_TY + ly;
        if (x > nx || y > ny) continue;
        const int z0 = tz * ENERGY_ZC, z1 = min(nz, z0 + ENERGY_ZC - 1);
        int p = g.idx(x, y, z0);
        for (int z = z0; z <= z1; z++, p += sz) energy_point<T, MED>(G, GU, vc0, vc1, vc2, flag, x, y, z, p, acc);
    }
    block_sums<12>(acc, partial, gridDim.x);
}

// Sum term partials in CTA order and combine as compute_energy.cpp:38-52; adds
// the grid's energy into the composite sum over grids (main.cpp:219-223).
// The destination is out[0], or out[*step - 1 - *step0] when the device step
// clock is given (inside a run, after the clock advanced for this step).
__global__ void energy_finalize_kernel(const double *partial, int nblocks, double h0, double h1, double h2,
                                       double *out, const int *step, const int *step0, int first, int *status, int gen21)
{
    __shared__ double term[12];
    if (threadIdx.x < 12) {
        double s = 0.0;
        for (int i = 0; i < nblocks; i++) s += partial[threadIdx.x * nblocks + i];
        term[threadIdx.x] = s;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double res = 0.0;
        // the inverse-stiffness form counts the symmetric cross terms twice
        for (int k = 0; k < 6; k++) res += term[k];
        for (int k = 6; k < 12; k++) res += gen21 ? term[k] : 2 * term[k];
        res *= 0.5 * h2 * h1 * h0;
        double *dst = step ? out + (*step - 1 - *step0) : out;
        const double e = first ? res : *dst + res;
        *dst = e;
        if (!isfinite(e)) atomicOr(status, ST_NONFINITE);
    }
}

// ---------------------------------------------------------------------------
// Interface residues, compute_res.cpp:4-95: fine plane sum - r^2 coarse plane sum.
// group 0: vx with sxz, group 1: vy with syz, group 2: szz with vz.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(RED_THREADS) residue_kernel(GridDev<T> F, GridDev<T> C, int group, double r2,
                                                             double *partial)
{
    // group 0: vx * (sxz + sxz), x,y in [1, n-1]; group 1: vy * (syz + syz), x,y in [0, n-1];
    // group 2: szz * (vz + vz), x in [0, n-1], y in [1, n-1]
    const int a = group == 0 ? VX : (group == 1 ? VY : SZZ);
    const int b2 = group == 0 ? SXZ : (group == 1 ? SYZ : VZ);
    const int x0 = (group == 0) ? 1 : 0, y0 = (group == 1) ? 0 : 1;
    const int nxf = F.g.nx - x0, nyf = F.g.ny - y0;
    const int nxc = C.g.nx - x0, nyc = C.g.ny - y0;
    const int64_t nf = (int64_t)nxf * nyf, nc = (int64_t)nxc * nyc;
    const int nz1 = F.g.nz;
    const int fsz = F.g.px * F.g.py, csz = C.g.px * C.g.py;
    double acc[2] = {0.0, 0.0};
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < nf + nc; t += (int64_t)gridDim.x * blockDim.x) {
        if (t < nf) {
            const int i0 = x0 + (int)(t % nxf), i1 = y0 + (int)(t / nxf);
            const int p = F.g.idx(i0, i1, nz1);
            acc[0] += (double)F.f[a][p] * ((double)F.f[b2][p - fsz] + (double)F.f[b2][p]);
        } else {
            const int64_t u = t - nf;
            const int i0 = x0 + (int)(u % nxc), i1 = y0 + (int)(u / nxc);
            const int p = C.g.idx(i0, i1, 0);
            acc[1] += r2 * (double)C.f[a][p] * ((double)C.f[b2][p - csz] + (double)C.f[b2][p]);
        }
    }
    block_sums<2>(acc, partial, gridDim.x);
}

// Field::AvgAbs over the computational domain of one component (field.cpp:210-229).
template <typename T>
__global__ void __launch_bounds__(RED_THREADS) avgabs_kernel(GridDev<T> G, int comp, int px, int py, int pz, double *partial)
{
    const Geo &g = G.g;
    const int ex = g.nx - px, ey = g.ny - py, ez = g.nz - pz;
    const int64_t n = (int64_t)(ex + 1) * (ey + 1) * (ez + 1);
    double acc[1] = {0.0};
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(t % (ex + 1));
        const int y = (int)((t / (ex + 1)) % (ey + 1));
        const int z = (int)(t / ((int64_t)(ex + 1) * (ey + 1)));
        acc[0] += fabs((double)G.f[comp][g.idx(x, y, z)]);
    }
    block_sums<1>(acc, partial, gridDim.x);
}

// Field::AvgAbs divides by the extents one dim at a time (field.cpp:224-226).
__global__ void avgabs_finalize_kernel(const double *partial, int nblocks, int e2, int e1, int e0, double *out)
{
    if (threadIdx.x == 0) {
        double s = 0.0;
        for (int i = 0; i < nblocks; i++) s += partial[i];
        s /= e2;
        s /= e1;
        s /= e0;
        out[0] = s;
    }
}

__global__ void sum_partials_kernel(const double *partial, int nblocks, int nterms, double *out)
{
    if (threadIdx.x < nterms) {
        double s = 0.0;
        for (int i = 0; i < nblocks; i++) s += partial[threadIdx.x * nblocks + i];
        out[threadIdx.x] = s;
    }
}

// ---------------------------------------------------------------------------
// Receivers and source, main.cpp:182-195: sample the receiver component, then
// add scale*trace[n] (a float product, as the reference's 1000*src_trace[n])
// to the source point while n < nt.  The step clock lives on the device so
// that a captured step replays unchanged; this kernel advances it.
// ---------------------------------------------------------------------------

// receiver samples of the step (mode 1 part of src_rec_kernel), one thread per receiver
template <typename T>
__global__ void rec_trace_kernel(SrcRec S)
{
    const int row = *S.step - *S.step0;
    if (row < 0 || row >= S.trace_cap) return;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < S.nrec; i += gridDim.x * blockDim.x) {
        const T *base = (const T *)S.rec_base[S.rec_grid[i]];
        S.traces[(int64_t)row * S.nrec + i] = (float)base[S.rec_off[i]];
    }
}

template <typename T>
__global__ void src_rec_kernel(SrcRec S)
{
    const int n = *S.step;
    const int row = n - *S.step0;
    if (S.mode & 1)
        for (int i = threadIdx.x; i < S.nrec; i += blockDim.x) {
            const T *base = (const T *)S.rec_base[S.rec_grid[i]];
            if (row >= 0 && row < S.trace_cap) S.traces[(int64_t)row * S.nrec + i] = (float)base[S.rec_off[i]];
        }
    __syncthreads();
    if ((S.mode & 2) && threadIdx.x == 0) {
        if (S.src_base && n >= 0 && n < S.src_nt) {
            T *f = (T *)S.src_base;
            const float amp = S.src_scale * S.src_trace[n];
            f[S.src_off] = f[S.src_off] + (T)amp;
        }
        *S.step = n + 1;
    }
}

// ---------------------------------------------------------------------------
// Set-up and layout conversion
// ---------------------------------------------------------------------------
// Host layout (reference Field, field.cpp:85-149): extents l0 x l1 x l2 with
// halo R, x fastest.  Device layout: the padded box of Geo.
template <typename T, typename S>
__global__ void pack_kernel(T *dst, Geo g, const S *src, int l0, int l1, int l2, int R)
{
    const int64_t n = (int64_t)l0 * l1 * l2;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int i0 = (int)(t % l0), i1 = (int)((t / l0) % l1), i2 = (int)(t / ((int64_t)l0 * l1));
        dst[g.idx(i0 - R, i1 - R, i2 - R)] = (T)src[t];
    }
}

template <typename T>
__global__ void unpack_kernel(double *dst, Geo g, const T *src, int l0, int l1, int l2, int R)
{
    const int64_t n = (int64_t)l0 * l1 * l2;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int i0 = (int)(t % l0), i1 = (int)((t / l0) % l1), i2 = (int)(t / ((int64_t)l0 * l1));
        dst[t] = (double)src[g.idx(i0 - R, i1 - R, i2 - R)];
    }
}

// One movie frame: the computational domain of a field (d0 x d1 x d2, x
// fastest, no halo) as float32, in the order PrintFieldToRSF writes it
// (print.cpp:89-104).  One thread per element, consecutive threads along x.
template <typename T>
__global__ void snapshot_kernel(float *dst, Geo g, const T *src, int d0, int d1, int d2)
{
    const int64_t n = (int64_t)d0 * d1 * d2;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int i0 = (int)(t % d0), i1 = (int)((t / d0) % d1), i2 = (int)(t / ((int64_t)d0 * d1));
        dst[t] = (float)src[g.idx(i0, i1, i2)];
    }
}

// Isotropic medium from node values (init_del_par_field.cpp:99-149):
// s44 = s11 - s13 at nodes, then ReshapeField to the stress positions:
// c11, c13 at (1,0,0); c44 at (1,1,1); c55 at (0,0,1); c66 at (0,1,0).
__device__ __forceinline__ double reshape8(const double *f, int p, int sx, int sy, int sz, int p0, int p1, int p2)
{
    const int ox = p0 * sx, oy = p1 * sy, oz = p2 * sz;
    return (f[p] + f[p + oz] + f[p + oy] + f[p + oy + oz] + f[p + ox] + f[p + ox + oz] + f[p + ox + oy]
            + f[p + ox + oy + oz]) / 8;
}

template <typename T>
__global__ void iso_medium_kernel(Geo g, const double *s11, const double *s13, double *s44, T *c11, T *c13, T *c44,
                                  T *c55, T *c66, int pass)
{
    const int nx = g.nx, ny = g.ny, nz = g.nz;
    const int64_t n = (int64_t)(nx + 1) * (ny + 1) * (nz + 1);
    const int sy = g.px, sz = g.px * g.py;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(t % (nx + 1)), y = (int)((t / (nx + 1)) % (ny + 1)), z = (int)(t / ((int64_t)(nx + 1) * (ny + 1)));
        const int p = g.idx(x, y, z);
        if (pass == 0) {
            s44[p] = s11[p] - s13[p];
        } else {
            if (x < nx) {
                c11[p] = (T)reshape8(s11, p, 1, sy, sz, 1, 0, 0);
                c13[p] = (T)reshape8(s13, p, 1, sy, sz, 1, 0, 0);
            }
            if (x < nx && y < ny && z < nz) c44[p] = (T)reshape8(s44, p, 1, sy, sz, 1, 1, 1);
            if (z < nz) c55[p] = (T)reshape8(s44, p, 1, sy, sz, 0, 0, 1);
            if (y < ny) c66[p] = (T)reshape8(s44, p, 1, sy, sz, 0, 1, 0);
        }
    }
}

// ---------------------------------------------------------------------------
// Host launchers
// ---------------------------------------------------------------------------
template <typename T>
cudaError_t launch_energy(const GridDev<T> &G, int medium, T *const vc[3], T *const disp[3], int flag, double *partial,
                          int nblocks, double h0, double h1, double h2, double *out, const int *step, const int *step0,
                          int first, int *status, cudaStream_t st)
{
    GridDev<T> GU = G;
    for (int k = 0; k < 3; k++) GU.f[VX + k] = disp ? disp[k] : nullptr;
    if (medium == MED_GEN21 && !GU.f[VX]) return cudaErrorInvalidValue;
    // one wave: three CTAs per SM (the kernel's launch bounds), at most nblocks
    // and at most one per tile
    int dev = 0, sms = 0;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
    const Geo &g = G.g;
    const int64_t ntiles = (int64_t)((g.nx + ENERGY_TX) / ENERGY_TX) * ((g.ny + ENERGY_TY) / ENERGY_TY) *
                           ((g.nz + ENERGY_ZC) / ENERGY_ZC);
    int eb = (sms > 0 && 3 * sms < nblocks) ? 3 * sms : nblocks;
    if (ntiles < eb) eb = (int)ntiles;
    bool done = false;
    if constexpr (std::is_same<T, float>::value) {
        if (medium == MED_GEN21) {   // the FP32 production path: its own kernel, 4 CTAs per SM
            int eb4 = (sms > 0 && 4 * sms < nblocks) ? 4 * sms : nblocks;
            if (ntiles < eb4) eb4 = (int)ntiles;
            eb = eb4;
            energy_f32_gen21_kernel<<<eb, RED_THREADS, 0, st>>>(G, vc[0], vc[1], vc[2], GU, flag, partial);
            done = true;
        }
    }
    if (done) {
    } else if (medium == MED_GEN21)
        energy_kernel<T, MED_GEN21><<<eb, RED_THREADS, 0, st>>>(G, vc[0], vc[1], vc[2], GU, flag, partial);
    else if (medium == MED_ISO5)
        energy_kernel<T, MED_ISO5><<<eb, RED_THREADS, 0, st>>>(G, vc[0], vc[1], vc[2], GU, flag, partial);
    else
        energy_kernel<T, MED_ORTHO9><<<eb, RED_THREADS, 0, st>>>(G, vc[0], vc[1], vc[2], GU, flag, partial);
    energy_finalize_kernel<<<1, 32, 0, st>>>(partial, eb, h0, h1, h2, out, step, step0, first, status,
                                             medium == MED_GEN21);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_residue(const GridDev<T> &F, const GridDev<T> &C, int group, double r2, double *partial, int nblocks,
                           double *out2, cudaStream_t st)
{
    residue_kernel<T><<<nblocks, RED_THREADS, 0, st>>>(F, C, group, r2, partial);
    sum_partials_kernel<<<1, 32, 0, st>>>(partial, nblocks, 2, out2);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_avgabs(const GridDev<T> &G, int comp, const int pos[3], double *partial, int nblocks, double *out,
                          cudaStream_t st)
{
    avgabs_kernel<T><<<nblocks, RED_THREADS, 0, st>>>(G, comp, pos[0], pos[1], pos[2], partial);
    avgabs_finalize_kernel<<<1, 32, 0, st>>>(partial, nblocks, G.g.nz + 1 - pos[2], G.g.ny + 1 - pos[1],
                                             G.g.nx + 1 - pos[0], out);
    return cudaGetLastError();
}

// Kernels launched by launch_src_rec for nrec receivers and mode: more than one
// CTA's worth of receivers are sampled by their own multi-CTA launch, the
// injection (after the samples: main.cpp samples before it injects) by a second.
int src_rec_kernels(int nrec, int mode) { return ((mode & 1) && nrec > 256 && (mode & 2)) ? 2 : 1; }

template <typename T>
cudaError_t launch_src_rec(const SrcRec &S, cudaStream_t st)
{
    if ((S.mode & 1) && S.nrec > 256) {
        const int blocks = (S.nrec + 255) / 256 < 1024 ? (S.nrec + 255) / 256 : 1024;
        rec_trace_kernel<T><<<blocks, 256, 0, st>>>(S);
        if (S.mode & 2) {
            SrcRec inj = S;
            inj.mode = 2;
            src_rec_kernel<T><<<1, 32, 0, st>>>(inj);
        }
    } else {
        src_rec_kernel<T><<<1, 256, 0, st>>>(S);
    }
    return cudaGetLastError();
}

template <typename T, typename S>
cudaError_t launch_pack(T *dst, const Geo &g, const S *src, int l0, int l1, int l2, int R, cudaStream_t st)
{
    const int64_t n = (int64_t)l0 * l1 * l2;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 4096) blocks = 4096;
    pack_kernel<T, S><<<blocks, 256, 0, st>>>(dst, g, src, l0, l1, l2, R);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_unpack(double *dst, const Geo &g, const T *src, int l0, int l1, int l2, int R, cudaStream_t st)
{
    const int64_t n = (int64_t)l0 * l1 * l2;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 4096) blocks = 4096;
    unpack_kernel<T><<<blocks, 256, 0, st>>>(dst, g, src, l0, l1, l2, R);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_snapshot(float *dst, const Geo &g, const T *src, int d0, int d1, int d2, cudaStream_t st)
{
    const int64_t n = (int64_t)d0 * d1 * d2;
    int blocks = (int)((n + 255) / 256);
    if (blocks > 8 * 148) blocks = 8 * 148;
    snapshot_kernel<T><<<blocks, 256, 0, st>>>(dst, g, src, d0, d1, d2);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_iso_medium(const Geo &g, const double *s11, const double *s13, double *s44, T *const c[5], cudaStream_t st)
{
    const int64_t n = (int64_t)(g.nx + 1) * (g.ny + 1) * (g.nz + 1);
    int blocks = (int)((n + 255) / 256);
    if (blocks > 4096) blocks = 4096;
    iso_medium_kernel<T><<<blocks, 256, 0, st>>>(g, s11, s13, s44, c[0], c[1], c[2], c[3], c[4], 0);
    iso_medium_kernel<T><<<blocks, 256, 0, st>>>(g, s11, s13, s44, c[0], c[1], c[2], c[3], c[4], 1);
    return cudaGetLastError();
}

#define INST(T)                                                                                               \
    template cudaError_t launch_energy<T>(const GridDev<T> &, int, T *const[3], T *const[3], int, double *, int, \
                                          double, double, double, double *, const int *, const int *, int, int *, \
                                          cudaStream_t);                                                       \
    template cudaError_t launch_residue<T>(const GridDev<T> &, const GridDev<T> &, int, double, double *, int,   \
                                           double *, cudaStream_t);                                            \
    template cudaError_t launch_avgabs<T>(const GridDev<T> &, int, const int[3], double *, int, double *,        \
                                          cudaStream_t);                                                       \
    template cudaError_t launch_src_rec<T>(const SrcRec &, cudaStream_t);                                       \
    template cudaError_t launch_pack<T, float>(T *, const Geo &, const float *, int, int, int, int, cudaStream_t); \
    template cudaError_t launch_pack<T, double>(T *, const Geo &, const double *, int, int, int, int, cudaStream_t); \
    template cudaError_t launch_unpack<T>(double *, const Geo &, const T *, int, int, int, int, cudaStream_t);    \
    template cudaError_t launch_snapshot<T>(float *, const Geo &, const T *, int, int, int, cudaStream_t);      \
    template cudaError_t launch_iso_medium<T>(const Geo &, const double *, const double *, double *, T *const[5], \
                                              cudaStream_t);
INST(float)
INST(double)
#undef INST

} // namespace ecsg
