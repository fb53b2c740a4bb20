// ecsg_device.cuh -- device-side data layout and helpers shared by the ECSG kernels.
//
// HBM layout of one sub-grid.  All field components of a grid share one padded
// box so that every kernel uses the same strides:
//   x in [-R, nx+8]   row pitch px (multiple of 32 elements); element x = 0 of
//                     every row sits XOFF elements into the row, so rows start
//                     on 128-byte boundaries; the right padding of 8 lets the
//                     float4 sweeps read whole 16-byte chunks past x = nx+1
//   y in [-R, ny+R]   py = ny + 1 + 2R rows per plane
//   z in [-R, nz+R]   pz = nz + 1 + 2R planes
// Staggered components use a subset of the box (their extents end at n-1); the
// spare row/plane costs < 1% of memory and keeps the index arithmetic uniform.
// Medium components (buoyancy at nodes, stiffness at the stress positions) use
// the same box and strides.
#pragma once
#include <cstdint>
#include <cuda_runtime.h>

namespace ecsg {

constexpr int XOFF = 32;
constexpr int kMaxGrids = 8;
constexpr int kMaxShots = 16;   // shots advanced in lockstep by one call

struct Geo {
    int nx, ny, nz;   // cells
    int R;            // halo radius
    int px, py, pz;   // pitches (elements)
    int off0;         // linear index of (0,0,0)
    __host__ __device__ __forceinline__ int idx(int x, int y, int z) const
    {
        return off0 + (z * py + y) * px + x;
    }
    __host__ __device__ __forceinline__ int64_t size() const { return (int64_t)px * py * pz; }
};

inline Geo make_geo(int nx, int ny, int nz, int R)
{
    Geo g;
    g.nx = nx; g.ny = ny; g.nz = nz; g.R = R;
    g.px = ((XOFF + nx + 1 + (R > 8 ? R : 8)) + 31) / 32 * 32;
    g.py = ny + 1 + 2 * R;
    g.pz = nz + 1 + 2 * R;
    g.off0 = (R * g.py + R) * g.px + XOFF;
    return g;
}

// Medium kinds.  ISO5: the reference's isotropic layout (c11=c22=c33, c12=c13=c23,
// c44, c55, c66 at their staggered positions; init_del_par_field.cpp:139-149).
// ORTHO9: nine independent fields in the same positions.  GEN21: all 21 Cij.
enum MediumKind { MED_ISO5 = 0, MED_ORTHO9 = 1, MED_GEN21 = 2 };

// Field component order (init_del_sim.cpp:14-24).
enum { VX = 0, VY, VZ, SXX, SYY, SZZ, SYZ, SXZ, SXY };

// Stiffness slots.  ISO5 uses slots 0..4 = c11, c13, c44, c55, c66.
// ORTHO9 uses slots 0..8 = c11 c22 c33 c23 c13 c12 c44 c55 c66 (update_stress.cpp:17-25).
// GEN21 uses slots 0..20 as documented in stress21.cu.
template <typename T>
struct GridDev {
    Geo g;
    T *f[9];
    const T *b;        // buoyancy at nodes
    const T *c[21];    // stiffness fields
    T k[3];            // dt / h_d (radius-1 coefficient, init_del_fdcoeff.cpp:7-22)
    double kd[3];      // same in double (interface solves)
};

// Rounded arithmetic without contraction, so that the double-precision
// instantiation reproduces the reference's rounding sequence operation by
// operation (the stencils are memory-bound; the lost FMA costs nothing).
__device__ __forceinline__ float add_(float a, float b) { return __fadd_rn(a, b); }
__device__ __forceinline__ float sub_(float a, float b) { return __fsub_rn(a, b); }
__device__ __forceinline__ float mul_(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ float div_(float a, float b) { return __fdiv_rn(a, b); }
__device__ __forceinline__ double add_(double a, double b) { return __dadd_rn(a, b); }
__device__ __forceinline__ double sub_(double a, double b) { return __dsub_rn(a, b); }
__device__ __forceinline__ double mul_(double a, double b) { return __dmul_rn(a, b); }
__device__ __forceinline__ double div_(double a, double b) { return __ddiv_rn(a, b); }

template <typename T>
__device__ __forceinline__ T ldg(const T *p) { return __ldg(p); }

// Device status word bits (read back by ecsg_get_status).
enum : int {
    ST_JACOBI_CAP = 1,        // an sxz Jacobi solve stopped at its iteration cap
    ST_BARRIER_TIMEOUT = 2,   // a grid-wide barrier gave up waiting
    ST_NONFINITE = 4,         // a non-finite energy was observed
    ST_PIPE_TIMEOUT = 8,      // a TMA pipeline wait gave up (the CTA stopped early)
};

// Barrier words of one grid-wide solve: [0] generation, [32] arrival count
// (separate 128-byte lines).
constexpr int kBarWords = 64;

// Work space of one sxz interface solve (interface.cu).
struct SxzWork {
    const double *A;          // 9 diagonals, [k][j1-1][j0-1]
    double *B;
    double *X0, *X1;          // (nx2+1)*(ny2+1), zero border; X0 holds the warm start
    double *partial;          // two doubles per CTA of the solve (alternating halves)
    double *total;            // spare word (the total is formed in every CTA)
    unsigned *bar;            // kBarWords words: generation, arrival count (grid_arrive)
    int *status;
    int *iters;               // sweeps of the last solve
    long long *iters_total;   // running sum of sweeps
    double *tol_out;
    int max_iter;
};

// Several sxz systems solved by one cooperative launch (interface.cu,
// sxz_solve_multi_kernel): system i owns CTAs [cta0, cta0 + ncta).
constexpr int kMaxSxzSys = 16;
template <typename T>
struct SxzSys {
    GridDev<T> F, C;
    SxzWork W;       // W.bar is not used: the list's barrier serves all systems
    int cta0, ncta;
};
template <typename T>
struct SxzSysList {
    SxzSys<T> s[kMaxSxzSys];
    int n;
    int r;           // refinement ratio, the same for every system
    unsigned *bar;   // kBarWords barrier words of the launch
    int *status;     // ST_BARRIER_TIMEOUT
};

// Several adjoint sxz systems (A^T y = lambda_X) in one cooperative launch
// (interface.cu, sxz_adj_solve_multi_kernel): system i owns CTAs
// [cta0, cta0 + ncta); W.X0 / W.X1 are its iterates, lx its right-hand side.
struct SxzAdjSys {
    SxzWork W;
    const double *lx;
    int nx2, ny2;
    int cta0, ncta;
};
struct SxzAdjList {
    SxzAdjSys s[kMaxSxzSys];
    int n;
    unsigned *bar;   // kBarWords barrier words of the launch
    int *status;
};

// Receivers and source of one run (diag.cu, src_rec_kernel).
struct SrcRec {
    void *rec_base[kMaxGrids];   // receiver component per grid
    const int *rec_grid;
    const int *rec_off;
    int nrec;
    float *traces;               // [capacity][nrec]
    int trace_cap;
    int *step;                   // device step clock
    const int *step0;            // device: first step of the current run (trace row 0)
    void *src_base;
    int src_off;
    const float *src_trace;
    int src_nt;
    float src_scale;
    int mode;                    // bit 0: sample receivers, bit 1: inject and advance the clock
};

} // namespace ecsg

