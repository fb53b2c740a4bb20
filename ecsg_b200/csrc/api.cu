// api.cu -- the C ABI (include/ecsg_b200.h): device state, set-up, operators
// and the fused time loop.
//
// One ecsg_sim owns one CUDA stream and all device memory of a composite run.
// There is no host fallback: without a usable device every entry point fails.
#include <nvtx3/nvToolsExt.h>
#include <optional>
#include "ecsg_device.cuh"
#include "adjoint.cuh"
#include "../../include/ecsg_b200.h"

#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <string>
#include <type_traits>
#include <vector>

namespace ecsg {
// stencil.cu
template <typename T>
cudaError_t launch_vel(const GridDev<T> &, int, int, int, T *const[3], int, cudaStream_t);
template <typename T>
cudaError_t launch_vel_mirror(const GridDev<T> &, int, int, int, int, cudaStream_t);
template <typename T>
cudaError_t launch_vel_mirror_shots(const Geo &, T *const *, T *const *, int, int, int, int, int, cudaStream_t);
template <typename T>
cudaError_t launch_stress(const GridDev<T> &, int, int, int, int, cudaStream_t);
// stencil_v4.cu (FP32 production sweeps)
cudaError_t launch_vel_v4(const GridDev<float> &, int, int, int, float *const[3], int, cudaStream_t, int);
cudaError_t launch_stress_v4(const GridDev<float> &, int, int, int, int, cudaStream_t, int);
// stress21.cu (21-Cij media)
template <typename T>
cudaError_t launch_stress21(const GridDev<T> &, int, int, T *const[3], int, cudaStream_t);
// stress21_tma.cu (FP32 21-Cij sweeps, TMA-staged)
size_t s21_maps_bytes();
bool s21_encode_maps(void *, const GridDev<float> &, float *const[3]);
cudaError_t s21_set_attributes();
cudaError_t launch_stress21_tma(const void *, const GridDev<float> &, int, int, float *const[3], int *, int, cudaStream_t, int);
cudaError_t launch_stress21_tma_shots(const void *const *, int, const GridDev<float> &, int, int, bool, int *, int,
                                      cudaStream_t, int);
size_t vel_maps_bytes();
bool vel_encode_maps(void *, const GridDev<float> &);
cudaError_t vel_tma_set_attributes();
cudaError_t launch_vel_tma(const void *, const GridDev<float> &, int, int, int, float *const[3], int *, int, cudaStream_t, int);
cudaError_t launch_vel_tma_shots(const void *const *, int, const GridDev<float> &, int, int, int, int *, int, cudaStream_t,
                                 int);
// interface.cu
template <typename T>
cudaError_t launch_ghost_vz(const GridDev<T> &, const GridDev<T> &, int, int, double *, cudaStream_t);
template <typename T>
cudaError_t launch_ghost_syz(const GridDev<T> &, const GridDev<T> &, int, cudaStream_t);
template <typename T>
cudaError_t launch_ghost_ii(int, const GridDev<T> &, const GridDev<T> &, cudaStream_t);
template <typename T>
cudaError_t launch_sxz_matrix(const GridDev<T> &, const GridDev<T> &, int, double *, cudaStream_t);
template <typename T>
int sxz_solve_blocks(int, int);
template <typename T>
cudaError_t launch_sxz_solve(const GridDev<T> &, const GridDev<T> &, int, const SxzWork &, int, cudaStream_t);
template <typename T>
int sxz_multi_capacity(int);
int sxz_adj_multi_capacity(int);
cudaError_t launch_sxz_adj_solve_multi(const SxzAdjList &, cudaStream_t);
template <typename T>
cudaError_t launch_sxz_adj_collect(const GridDev<T> &, const GridDev<T> &, const AdjDev<T> &, const AdjDev<T> &, int,
                                   double *, cudaStream_t);
template <typename T>
cudaError_t launch_sxz_adj_scatter(const GridDev<T> &, const GridDev<T> &, const AdjDev<T> &, const AdjDev<T> &, int,
                                   const double *, cudaStream_t);
template <typename T>
cudaError_t launch_sxz_solve_multi(const SxzSysList<T> &, cudaStream_t);
// diag.cu
template <typename T>
cudaError_t launch_energy(const GridDev<T> &, int, T *const[3], T *const[3], int, double *, int, double, double, double,
                          double *, const int *, const int *, int, int *, cudaStream_t);
template <typename T>
cudaError_t launch_residue(const GridDev<T> &, const GridDev<T> &, int, double, double *, int, double *, cudaStream_t);
template <typename T>
cudaError_t launch_avgabs(const GridDev<T> &, int, const int[3], double *, int, double *, cudaStream_t);
template <typename T>
cudaError_t launch_src_rec(const SrcRec &, cudaStream_t);
int src_rec_kernels(int nrec, int mode);
template <typename T, typename S>
cudaError_t launch_pack(T *, const Geo &, const S *, int, int, int, int, cudaStream_t);
template <typename T>
cudaError_t launch_unpack(double *, const Geo &, const T *, int, int, int, int, cudaStream_t);
template <typename T>
cudaError_t launch_snapshot(float *, const Geo &, const T *, int, int, int, cudaStream_t);
bool fd_coefficients(int R, double dt, const double h[3], double k[3][6]);
template <typename T>
cudaError_t launch_vel_r(const GridDev<T> &, const double[3][6], int, int, int, int, int, T *const[3], cudaStream_t);
template <typename T>
cudaError_t launch_stress_r(const GridDev<T> &, const double[3][6], int, int, int, int, int, cudaStream_t);
template <typename T>
cudaError_t launch_iso_medium(const Geo &, const double *, const double *, double *, T *const[5], cudaStream_t);
// adjoint.cu and the interface adjoints of interface.cu
template <typename T>
cudaError_t launch_vel_adj(const GridDev<T> &, const AdjDev<T> &, int, int, int, int, int, cudaStream_t);
template <typename T>
cudaError_t launch_stress21_adj(const GridDev<T> &, const AdjDev<T> &, int, int, int, cudaStream_t);
template <typename T>
cudaError_t launch_stress21_adj_shots(const GridDev<T> &, const AdjDev<T> &, const AdjShots<T> &, int, int, int, cudaStream_t);
template <typename T>
cudaError_t launch_vel_adj_shots(const GridDev<T> &, T *, const AdjShots<T> &, int, int, int, int, int, cudaStream_t);
template <typename T>
cudaError_t launch_rec_adj(const RecAdj<T> &, cudaStream_t);
template <typename T>
cudaError_t launch_rec_sample(const SrcRec &, T *, cudaStream_t);
template <typename T>
cudaError_t launch_residual(T *, const float *, int64_t, double *, double *, int, cudaStream_t);
template <typename T>
cudaError_t launch_ghost_vz_adj(const GridDev<T> &, const GridDev<T> &, const AdjDev<T> &, const AdjDev<T> &, int,
                                double *, double *, double *, cudaStream_t);
template <typename T>
cudaError_t launch_ghost_syz_adj(const GridDev<T> &, const GridDev<T> &, const AdjDev<T> &, const AdjDev<T> &, int,
                                 cudaStream_t);
template <typename T>
cudaError_t launch_ghost_ii_adj(int, const GridDev<T> &, const GridDev<T> &, const AdjDev<T> &, const AdjDev<T> &,
                                cudaStream_t);
template <typename T>
cudaError_t launch_ghost_sxz_adj(const GridDev<T> &, const GridDev<T> &, const AdjDev<T> &, const AdjDev<T> &, int,
                                 const SxzWork &, int, double *, cudaStream_t);
// medium.cu
template <typename T>
cudaError_t launch_tti_medium(const Geo &, const float *const[5], double, double, double, double *, T *, T *const[21],
                              cudaStream_t);
} // namespace ecsg

using namespace ecsg;

static const int kPos[9][3] = {{0, 0, 0}, {1, 1, 0}, {1, 0, 1}, {1, 0, 0}, {1, 0, 0},
                               {1, 0, 0}, {1, 1, 1}, {0, 0, 1}, {0, 1, 0}};
static const int kStiffPos[9][3] = {{1, 0, 0}, {1, 0, 0}, {1, 0, 0}, {1, 0, 0}, {1, 0, 0},
                                    {1, 0, 0}, {1, 1, 1}, {0, 0, 1}, {0, 1, 0}};
// 21-Cij slots: 0..14 at the normal-stress position, 15..17 syz, 18..19 sxz, 20 sxy
static const int kCij21Pos[21][3] = {{1, 0, 0}, {1, 0, 0}, {1, 0, 0}, {1, 0, 0}, {1, 0, 0}, {1, 0, 0}, {1, 0, 0},
                                     {1, 0, 0}, {1, 0, 0}, {1, 0, 0}, {1, 0, 0}, {1, 0, 0}, {1, 0, 0}, {1, 0, 0},
                                     {1, 0, 0}, {1, 1, 1}, {1, 1, 1}, {1, 1, 1}, {0, 0, 1}, {0, 0, 1}, {0, 1, 0}};

struct Iface {
    int r = 2;
    double *A = nullptr, *B = nullptr, *X0 = nullptr, *X1 = nullptr, *partial = nullptr;
    double *vzc = nullptr;   // vz tridiagonal rows: 4 x (ny2-1) x nx2
    int nblocks = 0;
    bool A_ready = false;
};

struct ecsg_sim {
    int ng = 0, R = 1, imode = 1, top_bc = 0, prec = ECSG_F32, medium = ECSG_MEDIUM_ISO, energy = 0;
    int jacobi_max_iter = 10000, device = 0, sms = 148, mirror_fix = 0, ii_skip_end = 0;
    bool scalar_stencils = false;   // FP32: use the scalar sweeps of stencil.cu (validation)
    double dt = 0;
    size_t tsize = 4;
    Geo geo[kMaxGrids];
    double h[kMaxGrids][3];
    int ztune[kMaxGrids][2] = {};        // z-chunks of the FP32 velocity / stress sweeps (0: automatic; ecsg_autotune)
    const ecsg_sim *share = nullptr;     // medium owner when this instance shares its medium (ecsg_create_shot)
    bool kset[kMaxGrids] = {};           // FD coefficients given by the caller (ecsg_set_coefficients)
    double kover[kMaxGrids][3] = {};
    // Per grid, the 9 fields, the stiffness slots and the displacement sums
    // each live in one allocation (fields of a group at a fixed stride), so
    // that one tensor map can address a whole group.
    void *fblk[kMaxGrids] = {}, *cblk[kMaxGrids] = {}, *dispblk[kMaxGrids] = {};
    void *f[kMaxGrids][9] = {};
    void *b[kMaxGrids] = {};
    void *c[kMaxGrids][21] = {};
    int nc = 5;
    void *vc[kMaxGrids][3] = {};
    void *disp[kMaxGrids][3] = {};  // 21-Cij media with energy: velocities summed over the stress updates (stress21.cu)
    std::vector<unsigned char> s21maps[kMaxGrids];   // TMA tensor maps of the FP32 21-Cij sweep, per grid
    bool s21_ready = false;
    std::vector<unsigned char> velmaps[kMaxGrids];   // TMA tensor maps of the FP32 velocity sweep, per grid
    bool vel_ready = false;
    bool vel_tma = true;             // FP32 velocity sweep: TMA-staged (false: the float4 sweep)
    // Side streams of the coarse grids' sweeps (multi-grid runs): the grids'
    // velocity sweeps are independent of each other, and so are their stress
    // sweeps, so the coarse grids' sweeps run beside the fine grid's and fill
    // the SMs its last wave leaves idle.
    bool side_grids = true;
    // The sxz solves of all interfaces of a step in one cooperative launch
    // (each interface bitwise as in its own launch), when their CTAs fit
    // co-resident (sxz_cap); otherwise one launch per interface.
    bool sxz_fused = true;
    int sxz_cap = 0, sxz_adj_cap = 0;   // co-resident CTAs of the multi-system forward / adjoint solves
    cudaStream_t side[kMaxGrids] = {};
    cudaEvent_t fork_ev = nullptr, join_ev[kMaxGrids] = {};
    // adjoint state (allocated on first use): adjoint fields, gradients, work boxes
    bool adj = false;
    void *lblk[kMaxGrids] = {}, *gbblk[kMaxGrids] = {}, *gcblk[kMaxGrids] = {};
    void *wblk = nullptr;
    size_t wbox = 0;                                  // elements of one work box (the largest grid's box)
    double *adj_lx[kMaxGrids] = {}, *adj_y[kMaxGrids] = {}, *adj_Y0[kMaxGrids] = {}, *adj_Y1[kMaxGrids] = {};
    // misfit-gradient driver: checkpoints, segment states, samples, observations
    char *ckpt = nullptr, *seg = nullptr, *seg2 = nullptr;   // seg2: sub-checkpoints of lockstep shots
    size_t ckpt_cap = 0, seg_cap = 0, seg2_cap = 0;
    void *recT = nullptr;
    size_t recT_cap = 0;
    float *obs = nullptr;
    size_t obs_cap = 0;
    bool medium_set[kMaxGrids] = {};
    Iface itf[kMaxGrids];
    // shared device scalars: [0] status, [1] step clock, [2] last sxz sweeps, [3] first step of the run
    int *ints = nullptr;
    long long *iters_total = nullptr;   // per interface
    double *dscal = nullptr;            // [0] energy, [1] total, [2..] last tol per interface, [16..] residue scratch
    unsigned *bar = nullptr;            // 2 per interface
    double *partial = nullptr;          // reductions
    int red_blocks = 0;
    // source / receivers
    int src_grid = -1, src_off = 0, src_comp = 0, src_nt = 0;
    float src_scale = 1.0f;
    float *src_trace = nullptr;
    int src_cap = 0;
    int nrec = 0, rec_comp = 0;
    int *rec_grid = nullptr, *rec_off = nullptr;
    float *traces = nullptr;
    int trace_cap = 0;
    double *run_energy = nullptr;
    int run_energy_cap = 0;
    double *run_res = nullptr;
    int run_res_cap = 0;
    cudaStream_t st = nullptr;
    cudaEvent_t ev[4] = {nullptr, nullptr, nullptr, nullptr};   // [0,1] run loop, [2,3] user timer
    double last_run_ms = 0;
    long long launches = 0;        // kernels launched by the last ecsg_run (all steps)
    cudaGraphExec_t gx[2] = {nullptr, nullptr};   // cached step graphs: [0] plain, [1] energy step
    long long epoch = 0;           // bumped when anything a captured step refers to changes
    long long gx_epoch[2] = {-1, -1};
    int run_n0 = 0;                // pinned by the async copies at the start of a run
    float *snap = nullptr;         // movie-frame staging (ecsg_get_domain)
    size_t snap_cap = 0;
    long long bytes = 0;
    std::string err;
};

// NVTX range for the duration of a scope (visible in Nsight timelines; no cost
// without a tool attached)
struct NvtxRange {
    explicit NvtxRange(const char *name) { nvtxRangePushA(name); }
    ~NvtxRange() { nvtxRangePop(); }
    NvtxRange(const NvtxRange &) = delete;
    NvtxRange &operator=(const NvtxRange &) = delete;
};

static int fail(ecsg_sim *s, int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (s) s->err = buf;
    return code;
}

#define CK(call)                                                                                   \
    do {                                                                                           \
        cudaError_t e_ = (call);                                                                   \
        if (e_ != cudaSuccess) return fail(s, ECSG_ERR_CUDA, "%s: %s (%s:%d)", #call, cudaGetErrorString(e_), __FILE__, __LINE__); \
    } while (0)

static int dmalloc(ecsg_sim *s, void **p, size_t bytes)
{
    CK(cudaMalloc(p, bytes));
    CK(cudaMemsetAsync(*p, 0, bytes, s->st));
    s->bytes += (long long)bytes;
    return ECSG_OK;
}

template <typename T>
static GridDev<T> dev(const ecsg_sim *s, int g)
{
    GridDev<T> G;
    memset(&G, 0, sizeof G);
    G.g = s->geo[g];
    for (int k = 0; k < 9; k++) G.f[k] = (T *)s->f[g][k];
    G.b = (const T *)s->b[g];
    for (int k = 0; k < s->nc; k++) G.c[k] = (const T *)s->c[g][k];
    for (int d = 0; d < 3; d++) {
        // FD coefficient of radius 1: fd[0]*dt/h with fd[0] = 1 (init_del_fdcoeff.cpp:19)
        const double kd = s->kset[g] ? s->kover[g][d] : 1.0 * s->dt / s->h[g][d];
        G.kd[d] = kd;
        G.k[d] = (T)kd;
    }
    return G;
}

static int field_len(const ecsg_sim *s, int g, int k, int len[3])
{
    const Geo &G = s->geo[g];
    const int n[3] = {G.nx, G.ny, G.nz};
    for (int d = 0; d < 3; d++) len[d] = kPos[k][d] ? n[d] + 2 * s->R : n[d] + 1 + 2 * s->R;
    return 0;
}

// The entry points below take their C linkage from the declarations in
// include/ecsg_b200.h (extern "C").

int ecsg_device_count(void)
{
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess) return 0;
    return n;
}

const char *ecsg_last_error(const ecsg_sim *sim) { return sim ? sim->err.c_str() : "null simulation"; }

long long ecsg_device_bytes(const ecsg_sim *sim) { return sim ? sim->bytes : 0; }

static int create_impl(const ecsg_grid_desc *grids, const ecsg_config *cfg, ecsg_sim **out, const ecsg_sim *share)
{
    if (!grids || !cfg || !out) return ECSG_ERR_INVALID;
    *out = nullptr;
    ecsg_sim *s = new ecsg_sim();
    auto bail = [&](int code) { ecsg_destroy(s); return code; };
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev <= 0) {
        fprintf(stderr, "ecsg_b200: no CUDA device available; this library has no CPU path\n");
        delete s;
        return ECSG_ERR_NO_DEVICE;
    }
    if (cfg->num_grids < 1 || cfg->num_grids > kMaxGrids) { fail(s, ECSG_ERR_INVALID, "num_grids out of range"); return bail(ECSG_ERR_INVALID); }
    if (cfg->radius < 1 || cfg->radius > 6) { fail(s, ECSG_ERR_INVALID, "radius %d: FD coefficients exist for radius 1..6 (init_del_fdcoeff.cpp:38-85)", cfg->radius); return bail(ECSG_ERR_INVALID); }
    if (cfg->radius > 1 && cfg->num_grids > 1) { fail(s, ECSG_ERR_INVALID, "radius %d: the interface conditions are derived for radius 1; composites need radius 1", cfg->radius); return bail(ECSG_ERR_INVALID); }
    if (cfg->radius > 1 && cfg->medium == ECSG_MEDIUM_GEN21) { fail(s, ECSG_ERR_INVALID, "radius %d: the 21-Cij update is radius 1", cfg->radius); return bail(ECSG_ERR_INVALID); }
    if (!(cfg->dt > 0)) { fail(s, ECSG_ERR_INVALID, "dt must be positive"); return bail(ECSG_ERR_INVALID); }
    if (cfg->imode != ECSG_MODE_ECI && cfg->imode != ECSG_MODE_II) { fail(s, ECSG_ERR_INVALID, "imode %d: 0 (intuitive) or 1 (energy-conserving)", cfg->imode); return bail(ECSG_ERR_INVALID); }
    if (cfg->precision != ECSG_F32 && cfg->precision != ECSG_F64) { fail(s, ECSG_ERR_INVALID, "precision"); return bail(ECSG_ERR_INVALID); }
    if (cfg->medium != ECSG_MEDIUM_ISO && cfg->medium != ECSG_MEDIUM_ORTHO9 && cfg->medium != ECSG_MEDIUM_GEN21) { fail(s, ECSG_ERR_INVALID, "medium"); return bail(ECSG_ERR_INVALID); }
    s->ng = cfg->num_grids;
    s->R = cfg->radius;
    s->dt = cfg->dt;
    s->imode = cfg->imode;
    s->top_bc = cfg->top_bc;
    s->prec = cfg->precision;
    s->medium = cfg->medium;
    s->energy = cfg->energy ? 1 : 0;
    s->jacobi_max_iter = cfg->jacobi_max_iter > 0 ? cfg->jacobi_max_iter : 10000;
    s->device = cfg->device;
    s->mirror_fix = cfg->mirror_fix ? 1 : 0;
    s->ii_skip_end = cfg->ii_skip_end_column ? 1 : 0;
    {
        const char *env = getenv("ECSG_SCALAR_STENCILS");
        s->scalar_stencils = env && env[0] == '1';
    }
    {
        const char *env = getenv("ECSG_VEL_TMA");   // "0": the float4 velocity sweep (validation)
        s->vel_tma = !(env && env[0] == '0');
    }
    {
        const char *env = getenv("ECSG_SIDE_GRIDS");   // "0": every sweep on the one stream
        s->side_grids = !(env && env[0] == '0');
    }
    {
        const char *env = getenv("ECSG_SXZ_FUSED");    // "0": one sxz launch per interface
        s->sxz_fused = !(env && env[0] == '0');
    }
    s->tsize = s->prec == ECSG_F32 ? 4 : 8;
    s->nc = s->medium == ECSG_MEDIUM_ISO ? 5 : (s->medium == ECSG_MEDIUM_ORTHO9 ? 9 : 21);
    if (cudaSetDevice(s->device) != cudaSuccess) { fail(s, ECSG_ERR_NO_DEVICE, "cudaSetDevice(%d) failed", s->device); return bail(ECSG_ERR_NO_DEVICE); }
    cudaDeviceProp prop;
    if (cudaGetDeviceProperties(&prop, s->device) != cudaSuccess) return bail(fail(s, ECSG_ERR_CUDA, "cudaGetDeviceProperties"));
    if (prop.major < 10) { fail(s, ECSG_ERR_NO_DEVICE, "device %s is sm_%d%d; this build targets sm_100a", prop.name, prop.major, prop.minor); return bail(ECSG_ERR_NO_DEVICE); }
    s->sms = prop.multiProcessorCount;
    if (cudaStreamCreateWithFlags(&s->st, cudaStreamNonBlocking) != cudaSuccess) return bail(fail(s, ECSG_ERR_CUDA, "stream"));
    for (int e = 0; e < 4; e++)
        if (cudaEventCreate(&s->ev[e]) != cudaSuccess) return bail(fail(s, ECSG_ERR_CUDA, "event"));
    if (s->ng > 1 && s->side_grids) {
        int lo = 0, hi = 0;   // side streams at the lowest priority: the fine grid's CTAs go first
        cudaDeviceGetStreamPriorityRange(&lo, &hi);
        if (cudaEventCreateWithFlags(&s->fork_ev, cudaEventDisableTiming) != cudaSuccess)
            return bail(fail(s, ECSG_ERR_CUDA, "event"));
        for (int g = 1; g < s->ng; g++)
            if (cudaStreamCreateWithPriority(&s->side[g], cudaStreamNonBlocking, lo) != cudaSuccess ||
                cudaEventCreateWithFlags(&s->join_ev[g], cudaEventDisableTiming) != cudaSuccess)
                return bail(fail(s, ECSG_ERR_CUDA, "side stream"));
    }

    for (int g = 0; g < s->ng; g++) {
        for (int d = 0; d < 3; d++) {
            if (grids[g].size[d] < 2 || !(grids[g].step[d] > 0)) { fail(s, ECSG_ERR_INVALID, "grid %d: bad size/step", g); return bail(ECSG_ERR_INVALID); }
            s->h[g][d] = grids[g].step[d];
        }
        s->geo[g] = make_geo(grids[g].size[0], grids[g].size[1], grids[g].size[2], s->R);
        if (s->geo[g].size() >= (int64_t)INT32_MAX) { fail(s, ECSG_ERR_INVALID, "grid %d too large for 32-bit indexing", g); return bail(ECSG_ERR_INVALID); }
    }
    for (int i = 1; i < s->ng; i++) {
        const double rx = s->h[i][0] / s->h[i - 1][0];
        const int r = (int)std::lround(rx);
        if (r < 2 || fabs(rx - r) > 1e-6 * r || fabs(s->h[i][1] / s->h[i - 1][1] - r) > 1e-6 * r) { fail(s, ECSG_ERR_INVALID, "interface %d: x/y refinement ratio must be an integer >= 2", i); return bail(ECSG_ERR_INVALID); }
        if (grids[i - 1].size[0] != r * grids[i].size[0] || grids[i - 1].size[1] != r * grids[i].size[1]) { fail(s, ECSG_ERR_INVALID, "interface %d: fine size must be ratio * coarse size in x and y", i); return bail(ECSG_ERR_INVALID); }
        if (grids[i].size[1] - 1 > 1024) { fail(s, ECSG_ERR_INVALID, "interface %d: coarse ny %d above the 1025 supported by the vz solve", i, grids[i].size[1]); return bail(ECSG_ERR_INVALID); }
        if (cfg->imode == ECSG_MODE_II && r != 2) { fail(s, ECSG_ERR_INVALID, "interface %d: intuitive interpolation (imode 0) is defined for ratio 2 only", i); return bail(ECSG_ERR_INVALID); }
        s->itf[i].r = r;
    }
    int rc;
    // 21-Cij slots in memory order: the 12 read around a tile (c6..c14, c16,
    // c17, c19) first, then the other 9 (c0..c5, c15, c18, c20)
    static const int kGen21Phys[21] = {12, 13, 14, 15, 16, 17, 0, 1, 2, 3, 4, 5, 6, 7, 8, 18, 9, 10, 19, 11, 20};
    for (int g = 0; g < s->ng; g++) {
        const size_t fb = (size_t)s->geo[g].size() * s->tsize;
        if ((rc = dmalloc(s, &s->fblk[g], 9 * fb))) return bail(rc);
        for (int k = 0; k < 9; k++) s->f[g][k] = (char *)s->fblk[g] + k * fb;
        if (share) {   // the medium (and the caller's FD coefficients) of another instance
            s->b[g] = share->b[g];
            for (int k = 0; k < s->nc; k++) s->c[g][k] = share->c[g][k];
            s->medium_set[g] = share->medium_set[g];
            s->kset[g] = share->kset[g];
            for (int d = 0; d < 3; d++) s->kover[g][d] = share->kover[g][d];
        } else {
            if ((rc = dmalloc(s, &s->b[g], fb))) return bail(rc);
            if ((rc = dmalloc(s, &s->cblk[g], s->nc * fb))) return bail(rc);
            for (int k = 0; k < s->nc; k++)
                s->c[g][k] = (char *)s->cblk[g] + (s->medium == ECSG_MEDIUM_GEN21 ? kGen21Phys[k] : k) * fb;
        }
        if (s->energy)
            for (int k = 0; k < 3; k++)
                if ((rc = dmalloc(s, &s->vc[g][k], fb))) return bail(rc);
        if (s->energy && s->medium == ECSG_MEDIUM_GEN21) {
            if ((rc = dmalloc(s, &s->dispblk[g], 3 * fb))) return bail(rc);
            for (int k = 0; k < 3; k++) s->disp[g][k] = (char *)s->dispblk[g] + k * fb;
        }
    }
    s->red_blocks = 4 * s->sms;
    if ((rc = dmalloc(s, (void **)&s->partial, sizeof(double) * 12 * (size_t)s->red_blocks))) return bail(rc);
    if ((rc = dmalloc(s, (void **)&s->ints, sizeof(int) * 4))) return bail(rc);
    if ((rc = dmalloc(s, (void **)&s->iters_total, sizeof(long long) * kMaxGrids))) return bail(rc);
    if ((rc = dmalloc(s, (void **)&s->dscal, sizeof(double) * 64))) return bail(rc);
    if ((rc = dmalloc(s, (void **)&s->bar, sizeof(unsigned) * kBarWords * kMaxGrids))) return bail(rc);
    for (int i = 1; i < s->ng; i++) {
        Iface &I = s->itf[i];
        const Geo &C = s->geo[i];
        const size_t nn = (size_t)(C.nx - 1) * (C.ny - 1);
        const size_t nxy = (size_t)(C.nx + 1) * (C.ny + 1);
        if ((rc = dmalloc(s, (void **)&I.A, sizeof(double) * 9 * nn))) return bail(rc);
        if ((rc = dmalloc(s, (void **)&I.vzc, sizeof(double) * 4 * (size_t)(C.ny - 1) * C.nx))) return bail(rc);
        if ((rc = dmalloc(s, (void **)&I.B, sizeof(double) * nn))) return bail(rc);
        if ((rc = dmalloc(s, (void **)&I.X0, sizeof(double) * nxy))) return bail(rc);
        if ((rc = dmalloc(s, (void **)&I.X1, sizeof(double) * nxy))) return bail(rc);
        I.nblocks = s->prec == ECSG_F32 ? sxz_solve_blocks<float>((int)nn, s->sms) : sxz_solve_blocks<double>((int)nn, s->sms);
        if (i == 1) {
            s->sxz_cap = s->prec == ECSG_F32 ? sxz_multi_capacity<float>(s->sms) : sxz_multi_capacity<double>(s->sms);
            s->sxz_adj_cap = sxz_adj_multi_capacity(s->sms);
        }
        // two halves: the solve's reduction rounds alternate between them
        if ((rc = dmalloc(s, (void **)&I.partial, sizeof(double) * 2 * (size_t)I.nblocks))) return bail(rc);
    }
    if (cudaStreamSynchronize(s->st) != cudaSuccess) return bail(fail(s, ECSG_ERR_CUDA, "initial clear"));
    s->share = share;
    *out = s;
    return ECSG_OK;
}

int ecsg_create(const ecsg_grid_desc *grids, const ecsg_config *cfg, ecsg_sim **out)
{
    return create_impl(grids, cfg, out, nullptr);
}

int ecsg_create_shot(const ecsg_sim *model, ecsg_sim **out)
{
    if (!model || !out) return ECSG_ERR_INVALID;
    for (int g = 0; g < model->ng; g++)
        if (!model->medium_set[g]) return ECSG_ERR_STATE;
    if (model->share) model = model->share;   // shots of a shot share the owner's medium
    std::vector<ecsg_grid_desc> gd(model->ng);
    for (int g = 0; g < model->ng; g++) {
        gd[g].size[0] = model->geo[g].nx;
        gd[g].size[1] = model->geo[g].ny;
        gd[g].size[2] = model->geo[g].nz;
        for (int d = 0; d < 3; d++) gd[g].step[d] = model->h[g][d];
    }
    ecsg_config cfg = {model->ng, model->R, model->dt, model->imode, model->top_bc, model->prec, model->medium,
                       model->energy, model->jacobi_max_iter, model->device, model->mirror_fix,
                       model->ii_skip_end};
    return create_impl(gd.data(), &cfg, out, model);
}

int ecsg_destroy(ecsg_sim *s)
{
    if (!s) return ECSG_OK;
    if (s->st) cudaStreamSynchronize(s->st);
    for (int g = 0; g < kMaxGrids; g++) {
        cudaFree(s->fblk[g]);
        if (!s->share) cudaFree(s->b[g]);
        cudaFree(s->cblk[g]);
        for (int k = 0; k < 3; k++) cudaFree(s->vc[g][k]);
        cudaFree(s->dispblk[g]);
        cudaFree(s->lblk[g]); cudaFree(s->gbblk[g]); cudaFree(s->gcblk[g]);
        cudaFree(s->adj_lx[g]); cudaFree(s->adj_y[g]); cudaFree(s->adj_Y0[g]); cudaFree(s->adj_Y1[g]);
        Iface &I = s->itf[g];
        cudaFree(I.A); cudaFree(I.B); cudaFree(I.X0); cudaFree(I.X1); cudaFree(I.partial); cudaFree(I.vzc);
    }
    cudaFree(s->partial); cudaFree(s->ints); cudaFree(s->iters_total); cudaFree(s->dscal); cudaFree(s->bar);
    cudaFree(s->src_trace); cudaFree(s->rec_grid); cudaFree(s->rec_off); cudaFree(s->traces);
    cudaFree(s->run_energy); cudaFree(s->run_res); cudaFree(s->snap);
    cudaFree(s->wblk); cudaFree(s->ckpt); cudaFree(s->seg); cudaFree(s->seg2); cudaFree(s->recT); cudaFree(s->obs);
    for (int v = 0; v < 2; v++)
        if (s->gx[v]) cudaGraphExecDestroy(s->gx[v]);
    for (int e = 0; e < 4; e++)
        if (s->ev[e]) cudaEventDestroy(s->ev[e]);
    for (int g = 0; g < kMaxGrids; g++) {
        if (s->side[g]) cudaStreamDestroy(s->side[g]);
        if (s->join_ev[g]) cudaEventDestroy(s->join_ev[g]);
    }
    if (s->fork_ev) cudaEventDestroy(s->fork_ev);
    if (s->st) cudaStreamDestroy(s->st);
    delete s;
    return ECSG_OK;
}

// ---------------------------------------------------------------------------
// Media and fields
// ---------------------------------------------------------------------------
template <typename T>
static int set_iso(ecsg_sim *s, int g, const float *buoy, const float *s11, const float *s13)
{
    const Geo &G = s->geo[g];
    const size_t nn = (size_t)(G.nx + 1) * (G.ny + 1) * (G.nz + 1);
    float *stage = nullptr;
    double *d11 = nullptr, *d13 = nullptr, *d44 = nullptr;
    const size_t box = (size_t)G.size() * sizeof(double);
    CK(cudaMalloc(&stage, nn * sizeof(float)));
    CK(cudaMalloc(&d11, box));
    CK(cudaMalloc(&d13, box));
    CK(cudaMalloc(&d44, box));
    CK(cudaMemsetAsync(d11, 0, box, s->st));
    CK(cudaMemsetAsync(d13, 0, box, s->st));
    CK(cudaMemsetAsync(d44, 0, box, s->st));
    CK(cudaMemcpyAsync(stage, buoy, nn * sizeof(float), cudaMemcpyHostToDevice, s->st));
    CK((launch_pack<T, float>((T *)s->b[g], G, stage, G.nx + 1, G.ny + 1, G.nz + 1, 0, s->st)));
    CK(cudaMemcpyAsync(stage, s11, nn * sizeof(float), cudaMemcpyHostToDevice, s->st));
    CK((launch_pack<double, float>(d11, G, stage, G.nx + 1, G.ny + 1, G.nz + 1, 0, s->st)));
    CK(cudaMemcpyAsync(stage, s13, nn * sizeof(float), cudaMemcpyHostToDevice, s->st));
    CK((launch_pack<double, float>(d13, G, stage, G.nx + 1, G.ny + 1, G.nz + 1, 0, s->st)));
    T *c5[5];
    for (int k = 0; k < 5; k++) c5[k] = (T *)s->c[g][k];
    CK(launch_iso_medium<T>(G, d11, d13, d44, c5, s->st));
    CK(cudaStreamSynchronize(s->st));
    cudaFree(stage); cudaFree(d11); cudaFree(d13); cudaFree(d44);
    return ECSG_OK;
}

int ecsg_set_medium_iso(ecsg_sim *s, int g, const float *buoy, const float *s11, const float *s13)
{
    if (s && s->share) return fail(s, ECSG_ERR_STATE, "the medium belongs to another instance (ecsg_create_shot)");
    if (!s || g < 0 || g >= s->ng || !buoy || !s11 || !s13) return fail(s, ECSG_ERR_INVALID, "set_medium_iso: bad arguments");
    if (s->medium != ECSG_MEDIUM_ISO) return fail(s, ECSG_ERR_STATE, "simulation was created for a non-isotropic medium");
    CK(cudaSetDevice(s->device));
    int rc = s->prec == ECSG_F32 ? set_iso<float>(s, g, buoy, s11, s13) : set_iso<double>(s, g, buoy, s11, s13);
    if (rc) return rc;
    s->medium_set[g] = true;
    if (g > 0) s->itf[g].A_ready = false;
    if (g + 1 < s->ng) s->itf[g + 1].A_ready = false;
    return ECSG_OK;
}

template <typename T>
static int set_stiff(ecsg_sim *s, int g, const double *buoy, const double *const *c, int nc, const int (*pos)[3])
{
    const Geo &G = s->geo[g];
    const size_t nn = (size_t)(G.nx + 1) * (G.ny + 1) * (G.nz + 1);
    double *stage = nullptr;
    CK(cudaMalloc(&stage, nn * sizeof(double)));
    CK(cudaMemcpyAsync(stage, buoy, nn * sizeof(double), cudaMemcpyHostToDevice, s->st));
    CK((launch_pack<T, double>((T *)s->b[g], G, stage, G.nx + 1, G.ny + 1, G.nz + 1, 0, s->st)));
    for (int k = 0; k < nc; k++) {
        const int l0 = G.nx + 1 - pos[k][0], l1 = G.ny + 1 - pos[k][1], l2 = G.nz + 1 - pos[k][2];
        CK(cudaMemcpyAsync(stage, c[k], (size_t)l0 * l1 * l2 * sizeof(double), cudaMemcpyHostToDevice, s->st));
        CK((launch_pack<T, double>((T *)s->c[g][k], G, stage, l0, l1, l2, 0, s->st)));
        CK(cudaStreamSynchronize(s->st));
    }
    cudaFree(stage);
    return ECSG_OK;
}

int ecsg_set_medium_ortho9(ecsg_sim *s, int g, const double *buoy, const double *const c[9])
{
    if (s && s->share) return fail(s, ECSG_ERR_STATE, "the medium belongs to another instance (ecsg_create_shot)");
    if (!s || g < 0 || g >= s->ng || !buoy || !c) return fail(s, ECSG_ERR_INVALID, "set_medium_ortho9: bad arguments");
    if (s->medium != ECSG_MEDIUM_ORTHO9) return fail(s, ECSG_ERR_STATE, "simulation was not created for an orthorhombic medium");
    for (int k = 0; k < 9; k++)
        if (!c[k]) return fail(s, ECSG_ERR_INVALID, "set_medium_ortho9: c[%d] is null", k);
    CK(cudaSetDevice(s->device));
    int rc = s->prec == ECSG_F32 ? set_stiff<float>(s, g, buoy, c, 9, kStiffPos) : set_stiff<double>(s, g, buoy, c, 9, kStiffPos);
    if (rc) return rc;
    s->medium_set[g] = true;
    if (g > 0) s->itf[g].A_ready = false;
    if (g + 1 < s->ng) s->itf[g + 1].A_ready = false;
    return ECSG_OK;
}

int ecsg_set_medium_cij21(ecsg_sim *s, int g, const double *buoy, const double *const c[21])
{
    if (s && s->share) return fail(s, ECSG_ERR_STATE, "the medium belongs to another instance (ecsg_create_shot)");
    if (!s || g < 0 || g >= s->ng || !buoy || !c) return fail(s, ECSG_ERR_INVALID, "set_medium_cij21: bad arguments");
    if (s->medium != ECSG_MEDIUM_GEN21) return fail(s, ECSG_ERR_STATE, "simulation was not created for a 21-Cij medium");
    for (int k = 0; k < 21; k++)
        if (!c[k]) return fail(s, ECSG_ERR_INVALID, "set_medium_cij21: c[%d] is null", k);
    CK(cudaSetDevice(s->device));
    int rc = s->prec == ECSG_F32 ? set_stiff<float>(s, g, buoy, c, 21, kCij21Pos) : set_stiff<double>(s, g, buoy, c, 21, kCij21Pos);
    if (rc) return rc;
    s->medium_set[g] = true;
    if (g > 0) s->itf[g].A_ready = false;
    if (g + 1 < s->ng) s->itf[g + 1].A_ready = false;
    return ECSG_OK;
}

template <typename T>
static int set_tti(ecsg_sim *s, int g, const float *const node[5], double eps, double delta, double gamma)
{
    const Geo &G = s->geo[g];
    const size_t nn = (size_t)(G.nx + 1) * (G.ny + 1) * (G.nz + 1);
    const size_t box = (size_t)G.size();
    float *stage = nullptr, *nd[5] = {};
    double *work = nullptr;
    auto release = [&]() {
        cudaFree(stage);
        cudaFree(work);
        for (int k = 0; k < 5; k++) cudaFree(nd[k]);
    };
    cudaError_t e = cudaMalloc(&stage, nn * sizeof(float));
    for (int k = 0; k < 5 && e == cudaSuccess; k++) e = cudaMalloc(&nd[k], box * sizeof(float));
    if (e == cudaSuccess) e = cudaMalloc(&work, box * sizeof(double));
    for (int k = 0; k < 5 && e == cudaSuccess; k++) {
        e = cudaMemcpyAsync(stage, node[k], nn * sizeof(float), cudaMemcpyHostToDevice, s->st);
        if (e == cudaSuccess) e = launch_pack<float, float>(nd[k], G, stage, G.nx + 1, G.ny + 1, G.nz + 1, 0, s->st);
        // the stage buffer is reused by the next component
        if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    }
    T *slot[21];
    for (int k = 0; k < 21; k++) slot[k] = (T *)s->c[g][k];
    if (e == cudaSuccess) e = launch_tti_medium<T>(G, nd, eps, delta, gamma, work, (T *)s->b[g], slot, s->st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(s->st);
    release();
    if (e != cudaSuccess) return fail(s, ECSG_ERR_CUDA, "set_medium_tti: %s", cudaGetErrorString(e));
    return ECSG_OK;
}

int ecsg_set_medium_tti(ecsg_sim *s, int g, const float *vp, const float *vs, const float *rho, const float *dip,
                        const float *azimuth, double epsilon, double delta, double gamma)
{
    if (s && s->share) return fail(s, ECSG_ERR_STATE, "the medium belongs to another instance (ecsg_create_shot)");
    if (!s || g < 0 || g >= s->ng || !vp || !vs || !rho || !dip || !azimuth)
        return fail(s, ECSG_ERR_INVALID, "set_medium_tti: bad arguments");
    if (s->medium != ECSG_MEDIUM_GEN21) return fail(s, ECSG_ERR_STATE, "simulation was not created for a 21-Cij medium");
    if (!(epsilon > -0.5) || !(gamma > -0.5) || !(delta > -0.5))
        return fail(s, ECSG_ERR_INVALID, "set_medium_tti: Thomsen parameters must exceed -1/2");
    CK(cudaSetDevice(s->device));
    const float *node[5] = {vp, vs, rho, dip, azimuth};
    int rc = s->prec == ECSG_F32 ? set_tti<float>(s, g, node, epsilon, delta, gamma)
                                 : set_tti<double>(s, g, node, epsilon, delta, gamma);
    if (rc) return rc;
    s->medium_set[g] = true;
    if (g > 0) s->itf[g].A_ready = false;
    if (g + 1 < s->ng) s->itf[g + 1].A_ready = false;
    return ECSG_OK;
}

long long ecsg_field_elems(const ecsg_sim *s, int g, int k)
{
    if (!s || g < 0 || g >= s->ng || k < 0 || k > 8) return -1;
    int len[3];
    field_len(s, g, k, len);
    return (long long)len[0] * len[1] * len[2];
}

int ecsg_set_field(ecsg_sim *s, int g, int k, const double *src)
{
    if (!s || g < 0 || g >= s->ng || k < 0 || k > 8 || !src) return fail(s, ECSG_ERR_INVALID, "set_field: bad arguments");
    CK(cudaSetDevice(s->device));
    int len[3];
    field_len(s, g, k, len);
    const size_t n = (size_t)len[0] * len[1] * len[2];
    double *stage = nullptr;
    CK(cudaMalloc(&stage, n * sizeof(double)));
    CK(cudaMemcpyAsync(stage, src, n * sizeof(double), cudaMemcpyHostToDevice, s->st));
    if (s->prec == ECSG_F32)
        CK((launch_pack<float, double>((float *)s->f[g][k], s->geo[g], stage, len[0], len[1], len[2], s->R, s->st)));
    else
        CK((launch_pack<double, double>((double *)s->f[g][k], s->geo[g], stage, len[0], len[1], len[2], s->R, s->st)));
    CK(cudaStreamSynchronize(s->st));
    cudaFree(stage);
    return ECSG_OK;
}

int ecsg_get_field(ecsg_sim *s, int g, int k, double *dst)
{
    if (!s || g < 0 || g >= s->ng || k < 0 || k > 8 || !dst) return fail(s, ECSG_ERR_INVALID, "get_field: bad arguments");
    CK(cudaSetDevice(s->device));
    int len[3];
    field_len(s, g, k, len);
    const size_t n = (size_t)len[0] * len[1] * len[2];
    double *stage = nullptr;
    CK(cudaMalloc(&stage, n * sizeof(double)));
    if (s->prec == ECSG_F32)
        CK(launch_unpack<float>(stage, s->geo[g], (const float *)s->f[g][k], len[0], len[1], len[2], s->R, s->st));
    else
        CK(launch_unpack<double>(stage, s->geo[g], (const double *)s->f[g][k], len[0], len[1], len[2], s->R, s->st));
    CK(cudaMemcpyAsync(dst, stage, n * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    cudaFree(stage);
    return ECSG_OK;
}

int ecsg_domain_shape(const ecsg_sim *s, int g, int k, int dims[3])
{
    if (!s || g < 0 || g >= s->ng || k < 0 || k > 8 || !dims) return ECSG_ERR_INVALID;
    const int n[3] = {s->geo[g].nx, s->geo[g].ny, s->geo[g].nz};
    for (int d = 0; d < 3; d++) dims[d] = kPos[k][d] ? n[d] : n[d] + 1;
    return ECSG_OK;
}

int ecsg_get_domain(ecsg_sim *s, int g, int k, float *dst)
{
    int dims[3];
    if (!dst || ecsg_domain_shape(s, g, k, dims) != ECSG_OK) return fail(s, ECSG_ERR_INVALID, "get_domain: bad arguments");
    CK(cudaSetDevice(s->device));
    const size_t n = (size_t)dims[0] * dims[1] * dims[2];
    if (n > s->snap_cap) {
        cudaFree(s->snap);
        s->snap = nullptr;
        s->snap_cap = 0;
        CK(cudaMalloc(&s->snap, n * sizeof(float)));
        s->snap_cap = n;
    }
    if (s->prec == ECSG_F32)
        CK(launch_snapshot<float>(s->snap, s->geo[g], (const float *)s->f[g][k], dims[0], dims[1], dims[2], s->st));
    else
        CK(launch_snapshot<double>(s->snap, s->geo[g], (const double *)s->f[g][k], dims[0], dims[1], dims[2], s->st));
    CK(cudaMemcpyAsync(dst, s->snap, n * sizeof(float), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return ECSG_OK;
}

int ecsg_host_alloc(size_t bytes, void **out)
{
    if (!out) return ECSG_ERR_INVALID;
    *out = nullptr;
    if (cudaHostAlloc(out, bytes ? bytes : 1, cudaHostAllocDefault) != cudaSuccess) {
        *out = nullptr;
        return ECSG_ERR_CUDA;
    }
    return ECSG_OK;
}

int ecsg_host_free(void *p)
{
    if (p && cudaFreeHost(p) != cudaSuccess) return ECSG_ERR_CUDA;
    return ECSG_OK;
}

// ---------------------------------------------------------------------------
// Operators
// ---------------------------------------------------------------------------
static int check_ready(ecsg_sim *s)
{
    for (int g = 0; g < s->ng; g++)
        if (!s->medium_set[g]) return fail(s, ECSG_ERR_STATE, "medium of grid %d not set", g);
    return ECSG_OK;
}

// top / bottom: the grid's boundary roles (update_vel.cpp:4 arguments); -1 takes
// them from the grid's place in the composite (top = grid 0, bottom = last grid)
static int top_of(const ecsg_sim *s, int g, int top) { return top < 0 ? (g == 0) : top; }
static int bottom_of(const ecsg_sim *s, int g, int bottom) { return bottom < 0 ? (g == s->ng - 1) : bottom; }

static bool use_vel_tma(const ecsg_sim *s);
static int stress_prepare(ecsg_sim *s);

template <typename T>
static int vel_kernel_op(ecsg_sim *s, int g, bool with_copy, int top = -1, int bottom = -1)
{
    T *vc[3] = {(T *)s->vc[g][0], (T *)s->vc[g][1], (T *)s->vc[g][2]};
    const int tp = top_of(s, g, top), bt = bottom_of(s, g, bottom);
    if (s->R > 1) {   // radius 2..6: sweep and its halo mirrors (stencil_r.cu)
        double k[3][6];
        fd_coefficients(s->R, s->dt, s->h[g], k);
        CK(launch_vel_r<T>(dev<T>(s, g), k, s->R, tp, bt, s->top_bc, s->mirror_fix, with_copy ? vc : nullptr, s->st));
        return ECSG_OK;
    }
    if constexpr (std::is_same<T, float>::value) {
        if (use_vel_tma(s)) {
            if (int rc = stress_prepare(s)) return rc;
            CK(launch_vel_tma(s->velmaps[g].data(), dev<float>(s, g), tp, bt, s->top_bc, with_copy ? vc : nullptr, s->ints,
                              s->sms, s->st, s->ztune[g][0]));
            return ECSG_OK;
        }
        if (!s->scalar_stencils) {
            CK(launch_vel_v4(dev<float>(s, g), tp, bt, s->top_bc, with_copy ? vc : nullptr, s->sms, s->st, s->ztune[g][0]));
            return ECSG_OK;
        }
    }
    CK(launch_vel<T>(dev<T>(s, g), tp, bt, s->top_bc, with_copy ? vc : nullptr, s->sms, s->st));
    return ECSG_OK;
}

template <typename T>
static int vel_mirror_op(ecsg_sim *s, int g, int top = -1, int bottom = -1)
{
    if (s->R > 1) return ECSG_OK;   // launch_vel_r ran them with the sweep
    CK(launch_vel_mirror<T>(dev<T>(s, g), top_of(s, g, top), bottom_of(s, g, bottom), s->top_bc, s->mirror_fix, s->st));
    return ECSG_OK;
}

template <typename T>
static int vel_op(ecsg_sim *s, int g, bool with_copy, int top = -1, int bottom = -1)
{
    int rc = vel_kernel_op<T>(s, g, with_copy, top, bottom);
    return rc ? rc : vel_mirror_op<T>(s, g, top, bottom);
}

static int med_kind(const ecsg_sim *s)
{
    return s->medium == ECSG_MEDIUM_ISO ? MED_ISO5 : (s->medium == ECSG_MEDIUM_ORTHO9 ? MED_ORTHO9 : MED_GEN21);
}

static bool use_vel_tma(const ecsg_sim *s)
{
    return s->prec == ECSG_F32 && !s->scalar_stencils && s->vel_tma && s->R == 1;
}

static bool use_s21_tma(const ecsg_sim *s)
{
    return s->medium == ECSG_MEDIUM_GEN21 && s->prec == ECSG_F32 && !s->scalar_stencils;
}

// Tensor maps and kernel attributes of the TMA-staged sweeps (velocity, and
// 21-Cij stress); host work only, done once before any capture.
static int stress_prepare(ecsg_sim *s)
{
    if (use_vel_tma(s) && !s->vel_ready) {
        for (int g = 0; g < s->ng; g++) {
            s->velmaps[g].assign(vel_maps_bytes(), 0);
            if (!vel_encode_maps(s->velmaps[g].data(), dev<float>(s, g)))
                return fail(s, ECSG_ERR_CUDA, "grid %d: TMA tensor maps of the velocity sweep could not be encoded", g);
        }
        CK(vel_tma_set_attributes());
        s->vel_ready = true;
    }
    if (!use_s21_tma(s) || s->s21_ready) return ECSG_OK;
    for (int g = 0; g < s->ng; g++) {
        float *disp[3];
        for (int k = 0; k < 3; k++) disp[k] = (float *)s->disp[g][k];
        s->s21maps[g].assign(s21_maps_bytes(), 0);
        if (!s21_encode_maps(s->s21maps[g].data(), dev<float>(s, g), disp))
            return fail(s, ECSG_ERR_CUDA, "grid %d: TMA tensor maps of the 21-Cij sweep could not be encoded", g);
    }
    CK(s21_set_attributes());
    s->s21_ready = true;
    return ECSG_OK;
}

template <typename T>
static int stress_op(ecsg_sim *s, int g, int top = -1, int bottom = -1)
{
    const int med = med_kind(s);
    const int tp = top_of(s, g, top);
    if (s->R > 1) {   // radius 2..6 (stencil_r.cu); its bottom mirrors need the bottom role
        double k[3][6];
        fd_coefficients(s->R, s->dt, s->h[g], k);
        CK(launch_stress_r<T>(dev<T>(s, g), k, s->R, med, tp, bottom_of(s, g, bottom), s->top_bc, s->st));
        return ECSG_OK;
    }
    if (med == MED_GEN21) {
        T *disp[3];
        for (int k = 0; k < 3; k++) disp[k] = (T *)s->disp[g][k];
        if constexpr (std::is_same<T, float>::value) {
            if (use_s21_tma(s)) {
                if (int rc = stress_prepare(s)) return rc;
                CK(launch_stress21_tma(s->s21maps[g].data(), dev<float>(s, g), tp, s->top_bc, disp, s->ints, s->sms, s->st,
                                       s->ztune[g][1]));
                return ECSG_OK;
            }
        }
        CK(launch_stress21<T>(dev<T>(s, g), tp, s->top_bc, disp, s->sms, s->st));
        return ECSG_OK;
    }
    if constexpr (std::is_same<T, float>::value) {
        if (!s->scalar_stencils) {
            CK(launch_stress_v4(dev<float>(s, g), med, tp, s->top_bc, s->sms, s->st, s->ztune[g][1]));
            return ECSG_OK;
        }
    }
    CK(launch_stress<T>(dev<T>(s, g), med, tp, s->top_bc, s->sms, s->st));
    return ECSG_OK;
}

template <typename T>
static int vz_op(ecsg_sim *s, int i)
{
    if (s->imode == ECSG_MODE_II) {
        CK(launch_ghost_ii<T>(s->ii_skip_end ? 3 : 0, dev<T>(s, i - 1), dev<T>(s, i), s->st));
        return ECSG_OK;
    }
    CK(launch_ghost_vz<T>(dev<T>(s, i - 1), dev<T>(s, i), med_kind(s), s->itf[i].r,
                          s->itf[i].vzc, s->st));
    return ECSG_OK;
}

template <typename T>
static int syz_op(ecsg_sim *s, int i)
{
    if (s->imode == ECSG_MODE_II) {
        CK(launch_ghost_ii<T>(2, dev<T>(s, i - 1), dev<T>(s, i), s->st));
        return ECSG_OK;
    }
    CK(launch_ghost_syz<T>(dev<T>(s, i - 1), dev<T>(s, i), s->itf[i].r, s->st));
    return ECSG_OK;
}

template <typename T>
static int sxz_prepare(ecsg_sim *s, int i)
{
    Iface &I = s->itf[i];
    if (s->imode == ECSG_MODE_II) return ECSG_OK;   // explicit: no system to assemble
    if (!I.A_ready) {
        CK(launch_sxz_matrix<T>(dev<T>(s, i - 1), dev<T>(s, i), I.r, I.A, s->st));
        I.A_ready = true;
    }
    return ECSG_OK;
}

static SxzWork sxz_work(ecsg_sim *s, int i)
{
    Iface &I = s->itf[i];
    SxzWork W;
    W.A = I.A;
    W.B = I.B;
    W.X0 = I.X0;
    W.X1 = I.X1;
    W.partial = I.partial;
    W.total = s->dscal + 1;
    W.bar = s->bar + kBarWords * i;
    W.status = s->ints;
    W.iters = s->ints + 2;
    W.iters_total = s->iters_total + i;
    W.tol_out = s->dscal + 2 + i;
    W.max_iter = s->jacobi_max_iter;
    return W;
}

// The sxz solves of every interface: one cooperative launch over all of them
// when there are several of one ratio whose CTAs fit co-resident (barrier
// words: the spare slot 0 of s->bar), else one launch per interface.  The
// interfaces' systems are independent (each reads and writes only the planes
// at its own interface), and each is solved bitwise as in its own launch.
template <typename T>
static int sxz_op(ecsg_sim *s, int i);
static bool sxz_fuses(const ecsg_sim *s)
{
    bool fuse = s->sxz_fused && s->imode != ECSG_MODE_II && s->ng > 2 && s->ng - 1 <= kMaxSxzSys;
    int total = 0;
    for (int i = 1; fuse && i < s->ng; i++) {
        fuse = s->itf[i].r == s->itf[1].r && s->geo[i - 1].nz >= 2;
        total += s->itf[i].nblocks;
    }
    return fuse && total <= s->sxz_cap;
}

template <typename T>
static int sxz_all_op(ecsg_sim *s)
{
    if (!sxz_fuses(s)) {
        for (int i = 1; i < s->ng; i++)
            if (int rc = sxz_op<T>(s, i)) return rc;
        return ECSG_OK;
    }
    SxzSysList<T> L;
    memset(&L, 0, sizeof L);
    L.n = s->ng - 1;
    L.r = s->itf[1].r;
    L.bar = s->bar;
    L.status = s->ints;
    int cta = 0;
    for (int i = 1; i < s->ng; i++) {
        SxzSys<T> &Y = L.s[i - 1];
        Y.F = dev<T>(s, i - 1);
        Y.C = dev<T>(s, i);
        Y.W = sxz_work(s, i);
        Y.cta0 = cta;
        Y.ncta = s->itf[i].nblocks;
        cta += Y.ncta;
    }
    CK(launch_sxz_solve_multi<T>(L, s->st));
    return ECSG_OK;
}

template <typename T>
static int sxz_op(ecsg_sim *s, int i)
{
    if (s->imode == ECSG_MODE_II) {
        CK(launch_ghost_ii<T>(1, dev<T>(s, i - 1), dev<T>(s, i), s->st));
        return ECSG_OK;
    }
    Iface &I = s->itf[i];
    SxzWork W;
    W.A = I.A;
    W.B = I.B;
    W.X0 = I.X0;
    W.X1 = I.X1;
    W.partial = I.partial;
    W.total = s->dscal + 1;
    W.bar = s->bar + kBarWords * i;
    W.status = s->ints;
    W.iters = s->ints + 2;
    W.iters_total = s->iters_total + i;
    W.tol_out = s->dscal + 2 + i;
    W.max_iter = s->jacobi_max_iter;
    CK(launch_sxz_solve<T>(dev<T>(s, i - 1), dev<T>(s, i), I.r, W, I.nblocks, s->st));
    return ECSG_OK;
}

#define DISPATCH(call) (s->prec == ECSG_F32 ? call<float> : call<double>)

int ecsg_update_vel(ecsg_sim *s, int g)
{
    if (!s || g < 0 || g >= s->ng) return fail(s, ECSG_ERR_INVALID, "update_vel: bad grid");
    if (int rc = check_ready(s)) return rc;
    int rc = DISPATCH(vel_op)(s, g, false, -1, -1);
    if (rc) return rc;
    CK(cudaStreamSynchronize(s->st));
    return ECSG_OK;
}

int ecsg_update_vel_ex(ecsg_sim *s, int g, int top, int bottom)
{
    if (!s || g < 0 || g >= s->ng) return fail(s, ECSG_ERR_INVALID, "update_vel_ex: bad grid");
    if (int rc = check_ready(s)) return rc;
    int rc = s->prec == ECSG_F32 ? vel_op<float>(s, g, false, top ? 1 : 0, bottom ? 1 : 0)
                                 : vel_op<double>(s, g, false, top ? 1 : 0, bottom ? 1 : 0);
    if (rc) return rc;
    CK(cudaStreamSynchronize(s->st));
    return ECSG_OK;
}

int ecsg_update_stress_ex(ecsg_sim *s, int g, int top, int bottom)
{
    // bottom matters for radius > 1 only (the bottom mirrors of update_stress.cpp:293-309 are empty at radius 1)
    if (!s || g < 0 || g >= s->ng) return fail(s, ECSG_ERR_INVALID, "update_stress_ex: bad grid");
    if (int rc = check_ready(s)) return rc;
    int rc = s->prec == ECSG_F32 ? stress_op<float>(s, g, top ? 1 : 0, bottom ? 1 : 0)
                                 : stress_op<double>(s, g, top ? 1 : 0, bottom ? 1 : 0);
    if (rc) return rc;
    CK(cudaStreamSynchronize(s->st));
    return ECSG_OK;
}

int ecsg_set_coefficients(ecsg_sim *s, int g, const double k[3])
{
    if (!s || g < 0 || g >= s->ng || !k) return fail(s, ECSG_ERR_INVALID, "set_coefficients: bad arguments");
    if (s->R != 1) return fail(s, ECSG_ERR_INVALID, "set_coefficients: radius-1 coefficients only");
    for (int d = 0; d < 3; d++) {
        if (!(k[d] > 0)) return fail(s, ECSG_ERR_INVALID, "set_coefficients: coefficients must be positive");
        s->kover[g][d] = k[d];
    }
    s->kset[g] = true;
    if (g > 0) s->itf[g].A_ready = false;
    if (g + 1 < s->ng) s->itf[g + 1].A_ready = false;
    s->epoch++;
    return ECSG_OK;
}

int ecsg_update_stress(ecsg_sim *s, int g)
{
    if (!s || g < 0 || g >= s->ng) return fail(s, ECSG_ERR_INVALID, "update_stress: bad grid");
    if (int rc = check_ready(s)) return rc;
    int rc = DISPATCH(stress_op)(s, g, -1, -1);
    if (rc) return rc;
    CK(cudaStreamSynchronize(s->st));
    return ECSG_OK;
}

int ecsg_ghost_vz(ecsg_sim *s, int i)
{
    if (!s || i < 1 || i >= s->ng) return fail(s, ECSG_ERR_INVALID, "ghost_vz: bad interface");
    if (int rc = check_ready(s)) return rc;
    int rc = DISPATCH(vz_op)(s, i);
    if (rc) return rc;
    CK(cudaStreamSynchronize(s->st));
    return ECSG_OK;
}

int ecsg_ghost_syz(ecsg_sim *s, int i)
{
    if (!s || i < 1 || i >= s->ng) return fail(s, ECSG_ERR_INVALID, "ghost_syz: bad interface");
    if (int rc = check_ready(s)) return rc;
    int rc = DISPATCH(syz_op)(s, i);
    if (rc) return rc;
    CK(cudaStreamSynchronize(s->st));
    return ECSG_OK;
}

int ecsg_ghost_sxz(ecsg_sim *s, int i)
{
    if (!s || i < 1 || i >= s->ng) return fail(s, ECSG_ERR_INVALID, "ghost_sxz: bad interface");
    if (int rc = check_ready(s)) return rc;
    int rc = DISPATCH(sxz_prepare)(s, i);
    if (rc) return rc;
    rc = DISPATCH(sxz_op)(s, i);
    if (rc) return rc;
    CK(cudaStreamSynchronize(s->st));
    return ECSG_OK;
}

int ecsg_get_sxz_state(ecsg_sim *s, int i, double *X, int *last_iters, double *last_tol, long long *total_iters)
{
    if (!s || i < 1 || i >= s->ng) return fail(s, ECSG_ERR_INVALID, "get_sxz_state: bad interface");
    CK(cudaSetDevice(s->device));
    const Geo &C = s->geo[i];
    if (X) CK(cudaMemcpyAsync(X, s->itf[i].X0, sizeof(double) * (C.nx + 1) * (C.ny + 1), cudaMemcpyDeviceToHost, s->st));
    int it = 0;
    double tol = 0;
    long long tot = 0;
    CK(cudaMemcpyAsync(&it, s->ints + 2, sizeof(int), cudaMemcpyDeviceToHost, s->st));
    CK(cudaMemcpyAsync(&tol, s->dscal + 2 + i, sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK(cudaMemcpyAsync(&tot, s->iters_total + i, sizeof(long long), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    if (last_iters) *last_iters = it;
    if (last_tol) *last_tol = tol;
    if (total_iters) *total_iters = tot;
    return ECSG_OK;
}

int ecsg_set_sxz_state(ecsg_sim *s, int i, const double *X)
{
    if (!s || i < 1 || i >= s->ng || !X) return fail(s, ECSG_ERR_INVALID, "set_sxz_state: bad arguments");
    CK(cudaSetDevice(s->device));
    const Geo &C = s->geo[i];
    CK(cudaMemcpyAsync(s->itf[i].X0, X, sizeof(double) * (C.nx + 1) * (C.ny + 1), cudaMemcpyHostToDevice, s->st));
    CK(cudaStreamSynchronize(s->st));
    return ECSG_OK;
}

// ---------------------------------------------------------------------------
// Energy and residues
// ---------------------------------------------------------------------------
template <typename T>
static int copy_vel_op(ecsg_sim *s)
{
    for (int g = 0; g < s->ng; g++)
        for (int k = 0; k < 3; k++)
            CK(cudaMemcpyAsync(s->vc[g][k], s->f[g][k], (size_t)s->geo[g].size() * sizeof(T), cudaMemcpyDeviceToDevice, s->st));
    return ECSG_OK;
}

template <typename T>
static int energy_op(ecsg_sim *s, double *out, const int *step, const int *step0)
{
    for (int g = 0; g < s->ng; g++) {
        T *vc[3] = {(T *)s->vc[g][0], (T *)s->vc[g][1], (T *)s->vc[g][2]};
        T *disp[3];
        for (int k = 0; k < 3; k++) disp[k] = (T *)s->disp[g][k];
        const int flag = (top_of(s, g, -1) && s->top_bc) ? 1 : 0;
        CK(launch_energy<T>(dev<T>(s, g), med_kind(s), vc, disp, flag, s->partial,
                            s->red_blocks, s->h[g][0], s->h[g][1], s->h[g][2], out, step, step0, g == 0, s->ints, s->st));
    }
    return ECSG_OK;
}

int ecsg_copy_vel(ecsg_sim *s)
{
    if (!s) return ECSG_ERR_INVALID;
    if (!s->energy) return fail(s, ECSG_ERR_STATE, "copy_vel: simulation created without energy support");
    int rc = DISPATCH(copy_vel_op)(s);
    if (rc) return rc;
    CK(cudaStreamSynchronize(s->st));
    return ECSG_OK;
}

int ecsg_energy(ecsg_sim *s, double *energy)
{
    if (!s || !energy) return ECSG_ERR_INVALID;
    if (!s->energy) return fail(s, ECSG_ERR_STATE, "energy: simulation created without energy support");
    if (int rc = check_ready(s)) return rc;
    int rc = DISPATCH(energy_op)(s, s->dscal, nullptr, nullptr);
    if (rc) return rc;
    CK(cudaMemcpyAsync(energy, s->dscal, sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    return ECSG_OK;
}

// Writes 12 doubles per interface at out: per group [fine sum, r^2 coarse sum, avg|a|, avg|b|].
template <typename T>
static int residue_op(ecsg_sim *s, int i, int which, double *out)
{
    const GridDev<T> F = dev<T>(s, i - 1), C = dev<T>(s, i);
    const double r2 = (double)s->itf[i].r * s->itf[i].r;
    static const int comps[3][2] = {{VX, SXZ}, {VY, SYZ}, {VZ, SZZ}};
    for (int grp = 0; grp < 3; grp++) {
        if (!(which & (1 << grp))) continue;
        CK(launch_residue<T>(F, C, grp, r2, s->partial, s->red_blocks, out + 4 * grp, s->st));
        for (int j = 0; j < 2; j++) {
            const int k = comps[grp][j];
            CK(launch_avgabs<T>(C, k, kPos[k], s->partial, s->red_blocks, out + 4 * grp + 2 + j, s->st));
        }
    }
    return ECSG_OK;
}

int ecsg_residues(ecsg_sim *s, int i, int which, double out[9])
{
    if (!s || i < 1 || i >= s->ng || !out) return fail(s, ECSG_ERR_INVALID, "residues: bad arguments");
    int rc = DISPATCH(residue_op)(s, i, which, s->dscal + 16);
    if (rc) return rc;
    double tmp[12];
    CK(cudaMemcpyAsync(tmp, s->dscal + 16, sizeof tmp, cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    for (int grp = 0; grp < 3; grp++) {
        if (!(which & (1 << grp))) continue;
        out[3 * grp] = tmp[4 * grp] - tmp[4 * grp + 1];
        out[3 * grp + 1] = tmp[4 * grp + 2];
        out[3 * grp + 2] = tmp[4 * grp + 3];
    }
    return ECSG_OK;
}

// ---------------------------------------------------------------------------
// Source, receivers, time loop
// ---------------------------------------------------------------------------
int ecsg_locate(const ecsg_sim *s, const double xyz[3], int loc4[4])
{
    if (!s || !xyz || !loc4) return ECSG_ERR_INVALID;
    int g = 0;
    double z = xyz[2];
    while (z > s->h[g][2] * s->geo[g].nz) {
        z -= s->h[g][2] * s->geo[g].nz;
        g++;
        if (g >= s->ng) return ECSG_ERR_INVALID;
    }
    loc4[0] = g;
    loc4[1] = (int)std::round(xyz[0] / s->h[g][0]);
    loc4[2] = (int)std::round(xyz[1] / s->h[g][1]);
    loc4[3] = (int)std::round(z / s->h[g][2]);
    return ECSG_OK;
}

int ecsg_set_source(ecsg_sim *s, int g, int ix, int iy, int iz, int comp, const float *trace, int nt, float scale)
{
    if (!s) return ECSG_ERR_INVALID;
    if (g < 0 || g >= s->ng || comp < 0 || comp > 8 || nt < 0 || (nt > 0 && !trace)) return fail(s, ECSG_ERR_INVALID, "set_source: bad arguments");
    const Geo &G = s->geo[g];
    if (ix < -s->R || ix > G.nx + s->R || iy < -s->R || iy > G.ny + s->R || iz < -s->R || iz > G.nz + s->R)
        return fail(s, ECSG_ERR_INVALID, "set_source: index outside grid %d", g);
    CK(cudaSetDevice(s->device));
    if (nt > s->src_cap) {
        cudaFree(s->src_trace);
        s->src_trace = nullptr;
        s->src_cap = 0;
        CK(cudaMalloc(&s->src_trace, sizeof(float) * nt));
        s->src_cap = nt;
        s->epoch++;
    }
    if (nt > 0) {
        CK(cudaMemcpyAsync(s->src_trace, trace, sizeof(float) * nt, cudaMemcpyHostToDevice, s->st));
        CK(cudaStreamSynchronize(s->st));
    }
    const int off = G.idx(ix, iy, iz);
    if (g != s->src_grid || off != s->src_off || comp != s->src_comp || nt != s->src_nt || scale != s->src_scale)
        s->epoch++;
    s->src_grid = g;
    s->src_off = off;
    s->src_comp = comp;
    s->src_nt = nt;
    s->src_scale = scale;
    return ECSG_OK;
}

int ecsg_set_receivers(ecsg_sim *s, const int *loc4, int n, int comp)
{
    if (!s || n < 0 || (n > 0 && !loc4) || comp < 0 || comp > 8) return fail(s, ECSG_ERR_INVALID, "set_receivers: bad arguments");
    std::vector<int> gr(n), off(n);
    for (int i = 0; i < n; i++) {
        const int g = loc4[4 * i];
        if (g < 0 || g >= s->ng) return fail(s, ECSG_ERR_INVALID, "receiver %d: bad grid", i);
        const Geo &G = s->geo[g];
        const int x = loc4[4 * i + 1], y = loc4[4 * i + 2], z = loc4[4 * i + 3];
        if (x < -s->R || x > G.nx + s->R || y < -s->R || y > G.ny + s->R || z < -s->R || z > G.nz + s->R)
            return fail(s, ECSG_ERR_INVALID, "receiver %d: index outside grid %d", i, g);
        gr[i] = g;
        off[i] = G.idx(x, y, z);
    }
    CK(cudaSetDevice(s->device));
    cudaFree(s->rec_grid);
    cudaFree(s->rec_off);
    s->rec_grid = s->rec_off = nullptr;
    if (n > 0) {
        CK(cudaMalloc(&s->rec_grid, sizeof(int) * n));
        CK(cudaMalloc(&s->rec_off, sizeof(int) * n));
        CK(cudaMemcpyAsync(s->rec_grid, gr.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s->st));
        CK(cudaMemcpyAsync(s->rec_off, off.data(), sizeof(int) * n, cudaMemcpyHostToDevice, s->st));
        CK(cudaStreamSynchronize(s->st));
    }
    s->nrec = n;
    s->rec_comp = comp;
    s->epoch++;
    return ECSG_OK;
}

static SrcRec make_srcrec(ecsg_sim *s, int mode)
{
    SrcRec S;
    memset(&S, 0, sizeof S);
    for (int g = 0; g < s->ng; g++) S.rec_base[g] = s->f[g][s->rec_comp];
    S.rec_grid = s->rec_grid;
    S.rec_off = s->rec_off;
    S.nrec = s->nrec;
    S.traces = s->traces;
    S.trace_cap = s->trace_cap;
    S.step = s->ints + 1;
    S.step0 = s->ints + 3;
    S.src_base = (s->src_grid >= 0 && s->src_trace) ? s->f[s->src_grid][s->src_comp] : nullptr;
    S.src_off = s->src_off;
    S.src_trace = s->src_trace;
    S.src_nt = s->src_nt;
    S.src_scale = s->src_scale;
    S.mode = mode;
    return S;
}

// One iteration of main.cpp:165-261 (movies excluded).
// op(g) for every grid: grid 0 on the library stream, the coarse grids on
// their side streams (forked from and joined back into the library stream,
// so a graph capture sees parallel branches), or all on the library stream.
template <typename Op>
static int each_grid(ecsg_sim *s, Op op)
{
    int rc;
    if (s->ng == 1 || !s->side[1]) {
        for (int g = 0; g < s->ng; g++)
            if ((rc = op(g))) return rc;
        return ECSG_OK;
    }
    cudaStream_t lib_stream = s->st;
    CK(cudaEventRecord(s->fork_ev, lib_stream));
    for (int g = 1; g < s->ng; g++) CK(cudaStreamWaitEvent(s->side[g], s->fork_ev, 0));
    if ((rc = op(0))) return rc;
    for (int g = 1; g < s->ng; g++) {
        s->st = s->side[g];
        rc = op(g);
        s->st = lib_stream;
        if (rc) return rc;
        CK(cudaEventRecord(s->join_ev[g], s->side[g]));
        CK(cudaStreamWaitEvent(lib_stream, s->join_ev[g], 0));
    }
    return ECSG_OK;
}

// The vz ghost solves of every interface: interface 1 on the library stream,
// the others on side streams, when every middle grid is thick enough (nz >= 8)
// that the planes its two interfaces touch (its top, its bottom) are apart.
// Each interface has its own scratch; these are ordinary (not cooperative)
// launches that wait on nothing.
template <typename T>
static int each_vz_ghost(ecsg_sim *s)
{
    int rc;
    bool side = s->ng > 2 && s->side[1];
    for (int g = 1; g < s->ng - 1 && side; g++)
        if (s->geo[g].nz < 8) side = false;
    if (!side) {
        for (int i = 1; i < s->ng; i++)
            if ((rc = vz_op<T>(s, i))) return rc;
        return ECSG_OK;
    }
    cudaStream_t lib_stream = s->st;
    CK(cudaEventRecord(s->fork_ev, lib_stream));
    for (int i = 2; i < s->ng; i++) CK(cudaStreamWaitEvent(s->side[i], s->fork_ev, 0));
    if ((rc = vz_op<T>(s, 1))) return rc;
    for (int i = 2; i < s->ng; i++) {
        s->st = s->side[i];
        rc = vz_op<T>(s, i);
        s->st = lib_stream;
        if (rc) return rc;
        CK(cudaEventRecord(s->join_ev[i], s->side[i]));
        CK(cudaStreamWaitEvent(lib_stream, s->join_ev[i], 0));
    }
    return ECSG_OK;
}

template <typename T>
static int step_op(ecsg_sim *s, bool energy, double *energy_buf, double *res_row, T *sample_row = nullptr)
{
    int rc;
    if ((rc = each_grid(s, [&](int g) { return vel_op<T>(s, g, energy); }))) return rc;
    if (sample_row) CK(launch_rec_sample<T>(make_srcrec(s, 0), sample_row, s->st));
    if (res_row) {
        CK(launch_src_rec<T>(make_srcrec(s, 1), s->st));
        for (int i = 1; i < s->ng; i++)
            if ((rc = residue_op<T>(s, i, 3, res_row + 12 * (i - 1)))) return rc;
        CK(launch_src_rec<T>(make_srcrec(s, 2), s->st));
    } else {
        CK(launch_src_rec<T>(make_srcrec(s, 3), s->st));
    }
    if ((rc = each_vz_ghost<T>(s))) return rc;
    if (res_row)
        for (int i = 1; i < s->ng; i++)
            if ((rc = residue_op<T>(s, i, 4, res_row + 12 * (i - 1)))) return rc;
    if (energy)
        if ((rc = energy_op<T>(s, energy_buf, s->ints + 1, s->ints + 3))) return rc;
    if ((rc = each_grid(s, [&](int g) { return stress_op<T>(s, g); }))) return rc;
    if ((rc = sxz_all_op<T>(s))) return rc;
    for (int i = 1; i < s->ng; i++)
        if ((rc = syz_op<T>(s, i))) return rc;
    return ECSG_OK;
}

template <typename T>
static int run_op(ecsg_sim *s, int n0, int nsteps, float *traces, double *energy, int energy_every, double *residues,
                  int use_graph)
{
    int rc;
    for (int i = 1; i < s->ng; i++)
        if ((rc = sxz_prepare<T>(s, i))) return rc;
    if ((rc = stress_prepare(s))) return rc;
    if (s->nrec > 0 && s->trace_cap < nsteps) {
        cudaFree(s->traces);
        s->traces = nullptr;
        CK(cudaMalloc(&s->traces, sizeof(float) * (size_t)nsteps * s->nrec));
        s->trace_cap = nsteps;
        s->epoch++;
    }
    if (energy && s->run_energy_cap < nsteps) {
        cudaFree(s->run_energy);
        s->run_energy = nullptr;
        CK(cudaMalloc(&s->run_energy, sizeof(double) * (size_t)nsteps));
        s->run_energy_cap = nsteps;
        s->epoch++;
    }
    const int nres = 12 * (s->ng - 1);
    if (residues && s->run_res_cap < nsteps) {
        cudaFree(s->run_res);
        s->run_res = nullptr;
        CK(cudaMalloc(&s->run_res, sizeof(double) * (size_t)nsteps * nres));
        s->run_res_cap = nsteps;
    }
    if (energy) {
        std::vector<double> nan(nsteps, NAN);
        CK(cudaMemcpyAsync(s->run_energy, nan.data(), sizeof(double) * nsteps, cudaMemcpyHostToDevice, s->st));
    }
    s->run_n0 = n0;
    CK(cudaMemcpyAsync(s->ints + 1, &s->run_n0, sizeof(int), cudaMemcpyHostToDevice, s->st));
    CK(cudaMemcpyAsync(s->ints + 3, &s->run_n0, sizeof(int), cudaMemcpyHostToDevice, s->st));
    const int every = energy_every > 0 ? energy_every : 1;
    bool graphs = use_graph && !residues;
    if (graphs) {
        // one captured step per variant, cached across runs until something it refers to changes
        for (int variant = 0; variant < (energy ? 2 : 1); variant++) {
            if (s->gx[variant] && s->gx_epoch[variant] == s->epoch) continue;
            if (s->gx[variant]) cudaGraphExecDestroy(s->gx[variant]);
            s->gx[variant] = nullptr;
            cudaGraph_t gr = nullptr;
            CK(cudaStreamBeginCapture(s->st, cudaStreamCaptureModeThreadLocal));
            rc = step_op<T>(s, variant == 1, s->run_energy, nullptr);
            cudaError_t e = cudaStreamEndCapture(s->st, &gr);
            if (rc || e != cudaSuccess) {
                if (gr) cudaGraphDestroy(gr);
                cudaGetLastError();
                return rc ? rc : fail(s, ECSG_ERR_CUDA, "graph capture: %s", cudaGetErrorString(e));
            }
            e = cudaGraphInstantiate(&s->gx[variant], gr, 0);
            cudaGraphDestroy(gr);
            if (e != cudaSuccess) {
                s->gx[variant] = nullptr;
                return fail(s, ECSG_ERR_CUDA, "graph instantiate: %s", cudaGetErrorString(e));
            }
            s->gx_epoch[variant] = s->epoch;
        }
    }
    CK(cudaEventRecord(s->ev[0], s->st));
    long long launches = 0;
    // per step: velocity kernel + 2 mirror kernels and the stress kernel per grid,
    // the receiver/source kernel(s), 3 vz + 1 sxz + 1 syz kernels per interface
    // (one sxz kernel for all interfaces when they are fused)
    const int srk = src_rec_kernels(s->nrec, 3);
    const long long per_step = 4LL * s->ng + srk + 5LL * (s->ng - 1) - (sxz_fuses(s) ? s->ng - 2 : 0);
    for (int n = n0; n < n0 + nsteps; n++) {
        const bool e_step = energy && ((n % every) == 0);
        launches += per_step + (e_step ? 2LL * s->ng : 0) + (residues ? (2 - srk) + 18LL * (s->ng - 1) : 0);
        if (graphs) {
            cudaError_t e = cudaGraphLaunch(s->gx[e_step ? 1 : 0], s->st);
            if (e != cudaSuccess) { rc = fail(s, ECSG_ERR_CUDA, "graph launch: %s", cudaGetErrorString(e)); break; }
        } else {
            if ((rc = step_op<T>(s, e_step, s->run_energy, residues ? s->run_res + (size_t)(n - n0) * nres : nullptr)))
                break;
        }
        rc = ECSG_OK;
    }
    CK(cudaEventRecord(s->ev[1], s->st));
    if (rc) return rc;
    s->launches = launches;
    if (traces && s->nrec > 0)
        CK(cudaMemcpyAsync(traces, s->traces, sizeof(float) * (size_t)nsteps * s->nrec, cudaMemcpyDeviceToHost, s->st));
    if (energy)
        CK(cudaMemcpyAsync(energy, s->run_energy, sizeof(double) * nsteps, cudaMemcpyDeviceToHost, s->st));
    std::vector<double> rtmp;
    if (residues) {
        rtmp.resize((size_t)nsteps * nres);
        CK(cudaMemcpyAsync(rtmp.data(), s->run_res, sizeof(double) * rtmp.size(), cudaMemcpyDeviceToHost, s->st));
    }
    CK(cudaStreamSynchronize(s->st));
    float ms = 0;
    CK(cudaEventElapsedTime(&ms, s->ev[0], s->ev[1]));
    s->last_run_ms = ms;
    if (residues) {
        for (int n = 0; n < nsteps; n++)
            for (int i = 0; i < s->ng - 1; i++)
                for (int grp = 0; grp < 3; grp++) {
                    const double *src = &rtmp[(size_t)n * nres + 12 * i + 4 * grp];
                    double *dst = residues + ((size_t)n * (s->ng - 1) + i) * 9 + 3 * grp;
                    dst[0] = src[0] - src[1];
                    dst[1] = src[2];
                    dst[2] = src[3];
                }
    }
    return ECSG_OK;
}

int ecsg_run(ecsg_sim *s, int n0, int nsteps, float *traces, double *energy, int energy_every, double *residues,
             int use_graph)
{
    NvtxRange range("ecsg_run");
    if (!s || nsteps < 0) return fail(s, ECSG_ERR_INVALID, "run: bad arguments");
    if (energy && !s->energy) return fail(s, ECSG_ERR_STATE, "run: energy requested but simulation created without it");
    if (int rc = check_ready(s)) return rc;
    CK(cudaSetDevice(s->device));
    if (nsteps == 0) return ECSG_OK;
    return DISPATCH(run_op)(s, n0, nsteps, traces, energy, energy_every, residues, use_graph);
}

int ecsg_synchronize(ecsg_sim *s)
{
    if (!s) return ECSG_ERR_INVALID;
    CK(cudaStreamSynchronize(s->st));
    return ECSG_OK;
}

int ecsg_get_status(ecsg_sim *s, int *status, int clear)
{
    if (!s || !status) return ECSG_ERR_INVALID;
    CK(cudaMemcpyAsync(status, s->ints, sizeof(int), cudaMemcpyDeviceToHost, s->st));
    if (clear) CK(cudaMemsetAsync(s->ints, 0, sizeof(int), s->st));
    CK(cudaStreamSynchronize(s->st));
    return ECSG_OK;
}

// ---------------------------------------------------------------------------
// Timing (CUDA events on the simulation's stream)
// ---------------------------------------------------------------------------
int ecsg_last_run(ecsg_sim *s, double *device_ms, long long *launches)
{
    if (!s) return ECSG_ERR_INVALID;
    if (device_ms) *device_ms = s->last_run_ms;
    if (launches) *launches = s->launches;
    return ECSG_OK;
}

int ecsg_timer_start(ecsg_sim *s)
{
    if (!s) return ECSG_ERR_INVALID;
    CK(cudaEventRecord(s->ev[2], s->st));
    return ECSG_OK;
}

int ecsg_timer_stop(ecsg_sim *s, double *ms)
{
    if (!s || !ms) return ECSG_ERR_INVALID;
    CK(cudaEventRecord(s->ev[3], s->st));
    CK(cudaEventSynchronize(s->ev[3]));
    float f = 0;
    CK(cudaEventElapsedTime(&f, s->ev[2], s->ev[3]));
    *ms = f;
    return ECSG_OK;
}

template <typename T>
static int time_kernels_op(ecsg_sim *s, int nsteps, double *out)
{
    int rc;
    for (int i = 1; i < s->ng; i++)
        if ((rc = sxz_prepare<T>(s, i))) return rc;
    const int nev = 1 + 6 * kMaxGrids + 1;
    std::vector<cudaEvent_t> ev(2 * nev);
    for (auto &e : ev) CK(cudaEventCreate(&e));
    std::vector<double> acc(7 * kMaxGrids, 0.0);
    CK(cudaMemcpyAsync(s->ints + 3, s->ints + 1, sizeof(int), cudaMemcpyDeviceToDevice, s->st));
    for (int n = 0; n < nsteps; n++) {
        int e = 0;
        auto bracket = [&](int slot, auto fn) -> int {
            CK(cudaEventRecord(ev[2 * e], s->st));
            int r = fn();
            if (r) return r;
            CK(cudaEventRecord(ev[2 * e + 1], s->st));
            CK(cudaEventSynchronize(ev[2 * e + 1]));
            float ms = 0;
            CK(cudaEventElapsedTime(&ms, ev[2 * e], ev[2 * e + 1]));
            acc[slot] += ms;
            e = (e + 1) % nev;
            return ECSG_OK;
        };
        for (int g = 0; g < s->ng; g++) {
            if ((rc = bracket(0 * kMaxGrids + g, [&] { return vel_kernel_op<T>(s, g, false); }))) return rc;
            if ((rc = bracket(1 * kMaxGrids + g, [&] { return vel_mirror_op<T>(s, g); }))) return rc;
        }
        if ((rc = bracket(6 * kMaxGrids, [&] {
                 CK(launch_src_rec<T>(make_srcrec(s, 3), s->st));
                 return (int)ECSG_OK;
             })))
            return rc;
        for (int i = 1; i < s->ng; i++)
            if ((rc = bracket(3 * kMaxGrids + i, [&] { return vz_op<T>(s, i); }))) return rc;
        for (int g = 0; g < s->ng; g++)
            if ((rc = bracket(2 * kMaxGrids + g, [&] { return stress_op<T>(s, g); }))) return rc;
        for (int i = 1; i < s->ng; i++) {
            if ((rc = bracket(4 * kMaxGrids + i, [&] { return sxz_op<T>(s, i); }))) return rc;
            if ((rc = bracket(5 * kMaxGrids + i, [&] { return syz_op<T>(s, i); }))) return rc;
        }
    }
    for (auto &e : ev) cudaEventDestroy(e);
    for (size_t k = 0; k < acc.size(); k++) out[k] = nsteps > 0 ? acc[k] / nsteps : 0.0;
    return ECSG_OK;
}

int ecsg_time_kernels(ecsg_sim *s, int nsteps, double *ms)
{
    if (!s || !ms || nsteps < 1) return fail(s, ECSG_ERR_INVALID, "time_kernels: bad arguments");
    if (int rc = check_ready(s)) return rc;
    CK(cudaSetDevice(s->device));
    return DISPATCH(time_kernels_op)(s, nsteps, ms);
}

// ---------------------------------------------------------------------------
// Adjoint: operator transposes and the misfit gradient (no reference
// counterpart).  21-Cij media only.
// ---------------------------------------------------------------------------
static int adj_alloc(ecsg_sim *s)
{
    if (s->adj) return ECSG_OK;
    int rc;
    size_t maxbox = 0;
    for (int g = 0; g < s->ng; g++) {
        const size_t box = (size_t)s->geo[g].size(), fb = box * s->tsize;
        if (box > maxbox) maxbox = box;
        if ((rc = dmalloc(s, &s->lblk[g], 9 * fb))) return rc;
        if ((rc = dmalloc(s, &s->gbblk[g], fb))) return rc;
        if ((rc = dmalloc(s, &s->gcblk[g], 21 * fb))) return rc;
    }
    s->wbox = maxbox;
    if ((rc = dmalloc(s, &s->wblk, 15 * maxbox * s->tsize))) return rc;
    for (int i = 1; i < s->ng; i++) {
        const Geo &C = s->geo[i];
        const size_t m = (size_t)(C.ny - 1) * C.nx, nn = (size_t)(C.nx - 1) * (C.ny - 1), nxy = (size_t)(C.nx + 1) * (C.ny + 1);
        if ((rc = dmalloc(s, (void **)&s->adj_lx[i], sizeof(double) * (m > nn ? m : nn)))) return rc;
        if ((rc = dmalloc(s, (void **)&s->adj_y[i], sizeof(double) * m))) return rc;
        if ((rc = dmalloc(s, (void **)&s->adj_Y0[i], sizeof(double) * nxy))) return rc;
        if ((rc = dmalloc(s, (void **)&s->adj_Y1[i], sizeof(double) * nxy))) return rc;
    }
    s->adj = true;
    return ECSG_OK;
}

template <typename T>
static AdjDev<T> adj_dev(const ecsg_sim *s, int g)
{
    AdjDev<T> A;
    const size_t box = (size_t)s->geo[g].size();
    for (int k = 0; k < 9; k++) A.l[k] = (T *)s->lblk[g] + k * box;
    A.gb = (T *)s->gbblk[g];
    for (int k = 0; k < 21; k++) A.gc[k] = (T *)s->gcblk[g] + k * box;
    for (int k = 0; k < 15; k++) A.w[k] = (T *)s->wblk + k * s->wbox;
    return A;
}

static int adj_check(ecsg_sim *s)
{
    if (s->R != 1) return fail(s, ECSG_ERR_STATE, "adjoint: radius 1 only");
    if (s->medium != ECSG_MEDIUM_GEN21) return fail(s, ECSG_ERR_STATE, "adjoint: the simulation must use ECSG_MEDIUM_GEN21");
    if (int rc = check_ready(s)) return rc;
    CK(cudaSetDevice(s->device));
    return adj_alloc(s);
}

// zero adjoint fields, gradients and work boxes (and the adjoint sxz warm starts)
static int adj_zero(ecsg_sim *s, bool fields, bool grads)
{
    for (int g = 0; g < s->ng; g++) {
        const size_t fb = (size_t)s->geo[g].size() * s->tsize;
        if (fields) CK(cudaMemsetAsync(s->lblk[g], 0, 9 * fb, s->st));
        if (grads) {
            CK(cudaMemsetAsync(s->gbblk[g], 0, fb, s->st));
            CK(cudaMemsetAsync(s->gcblk[g], 0, 21 * fb, s->st));
        }
    }
    CK(cudaMemsetAsync(s->wblk, 0, 15 * s->wbox * s->tsize, s->st));
    for (int i = 1; i < s->ng; i++) {
        const Geo &C = s->geo[i];
        CK(cudaMemsetAsync(s->adj_Y0[i], 0, sizeof(double) * (C.nx + 1) * (C.ny + 1), s->st));
    }
    return ECSG_OK;
}

template <typename T>
static int adj_op_impl(ecsg_sim *s, int op, int i, const GridDev<T> *Gv)
{
    // Gv: the forward fields of every grid the operator reads (its output state)
    if (s->imode == ECSG_MODE_II && (op == ECSG_ADJ_GHOST_VZ || op == ECSG_ADJ_GHOST_SXZ || op == ECSG_ADJ_GHOST_SYZ)) {
        const int which = op == ECSG_ADJ_GHOST_VZ ? (s->ii_skip_end ? 3 : 0) : (op == ECSG_ADJ_GHOST_SXZ ? 1 : 2);
        CK(launch_ghost_ii_adj<T>(which, Gv[i - 1], Gv[i], adj_dev<T>(s, i - 1), adj_dev<T>(s, i), s->st));
        return ECSG_OK;
    }
    switch (op) {
    case ECSG_ADJ_VEL:
        CK(launch_vel_adj<T>(Gv[i], adj_dev<T>(s, i), i == 0, i == s->ng - 1, s->top_bc, s->mirror_fix, s->sms, s->st));
        break;
    case ECSG_ADJ_STRESS:
        CK(launch_stress21_adj<T>(Gv[i], adj_dev<T>(s, i), i == 0, s->top_bc, s->sms, s->st));
        break;
    case ECSG_ADJ_GHOST_VZ:
        CK(launch_ghost_vz_adj<T>(Gv[i - 1], Gv[i], adj_dev<T>(s, i - 1), adj_dev<T>(s, i), s->itf[i].r, s->itf[i].vzc,
                                  s->adj_lx[i], s->adj_y[i], s->st));
        break;
    case ECSG_ADJ_GHOST_SYZ:
        CK(launch_ghost_syz_adj<T>(Gv[i - 1], Gv[i], adj_dev<T>(s, i - 1), adj_dev<T>(s, i), s->itf[i].r, s->st));
        break;
    case ECSG_ADJ_GHOST_SXZ: {
        if (int rc = sxz_prepare<T>(s, i)) return rc;
        Iface &I = s->itf[i];
        SxzWork W;
        W.A = I.A;
        W.B = I.B;
        W.X0 = s->adj_Y0[i];
        W.X1 = s->adj_Y1[i];
        W.partial = I.partial;
        W.total = s->dscal + 1;
        W.bar = s->bar + kBarWords * i;
        W.status = s->ints;
        W.iters = s->ints + 2;
        W.iters_total = s->iters_total + i;
        W.tol_out = s->dscal + 2 + i;
        W.max_iter = s->jacobi_max_iter;
        CK(launch_ghost_sxz_adj<T>(Gv[i - 1], Gv[i], adj_dev<T>(s, i - 1), adj_dev<T>(s, i), I.r, W, I.nblocks,
                                   s->adj_lx[i], s->st));
        break;
    }
    default:
        return fail(s, ECSG_ERR_INVALID, "adjoint_op: unknown operator %d", op);
    }
    return ECSG_OK;
}

template <typename T>
static int adj_op_current(ecsg_sim *s, int op, int i)
{
    GridDev<T> Gv[kMaxGrids];
    for (int g = 0; g < s->ng; g++) Gv[g] = dev<T>(s, g);
    return adj_op_impl<T>(s, op, i, Gv);
}

int ecsg_adjoint_reset(ecsg_sim *s)
{
    if (!s) return ECSG_ERR_INVALID;
    if (int rc = adj_check(s)) return rc;
    if (int rc = adj_zero(s, true, true)) return rc;
    CK(cudaStreamSynchronize(s->st));
    return ECSG_OK;
}

int ecsg_set_adjoint_field(ecsg_sim *s, int g, int k, const double *src)
{
    if (!s || g < 0 || g >= s->ng || k < 0 || k > 8 || !src) return fail(s, ECSG_ERR_INVALID, "set_adjoint_field: bad arguments");
    if (int rc = adj_check(s)) return rc;
    int len[3];
    field_len(s, g, k, len);
    const size_t n = (size_t)len[0] * len[1] * len[2], box = (size_t)s->geo[g].size();
    double *stage = nullptr;
    CK(cudaMalloc(&stage, n * sizeof(double)));
    CK(cudaMemcpyAsync(stage, src, n * sizeof(double), cudaMemcpyHostToDevice, s->st));
    if (s->prec == ECSG_F32)
        CK((launch_pack<float, double>((float *)s->lblk[g] + k * box, s->geo[g], stage, len[0], len[1], len[2], s->R, s->st)));
    else
        CK((launch_pack<double, double>((double *)s->lblk[g] + k * box, s->geo[g], stage, len[0], len[1], len[2], s->R, s->st)));
    CK(cudaStreamSynchronize(s->st));
    cudaFree(stage);
    return ECSG_OK;
}

static int get_box(ecsg_sim *s, const void *src, const Geo &G, int l0, int l1, int l2, int R, double *dst)
{
    const size_t n = (size_t)l0 * l1 * l2;
    double *stage = nullptr;
    CK(cudaMalloc(&stage, n * sizeof(double)));
    if (s->prec == ECSG_F32)
        CK(launch_unpack<float>(stage, G, (const float *)src, l0, l1, l2, R, s->st));
    else
        CK(launch_unpack<double>(stage, G, (const double *)src, l0, l1, l2, R, s->st));
    CK(cudaMemcpyAsync(dst, stage, n * sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    cudaFree(stage);
    return ECSG_OK;
}

int ecsg_get_adjoint_field(ecsg_sim *s, int g, int k, double *dst)
{
    if (!s || g < 0 || g >= s->ng || k < 0 || k > 8 || !dst) return fail(s, ECSG_ERR_INVALID, "get_adjoint_field: bad arguments");
    if (int rc = adj_check(s)) return rc;
    int len[3];
    field_len(s, g, k, len);
    const size_t box = (size_t)s->geo[g].size();
    return get_box(s, (const char *)s->lblk[g] + k * box * s->tsize, s->geo[g], len[0], len[1], len[2], s->R, dst);
}

int ecsg_get_gradient(ecsg_sim *s, int g, int which, double *dst)
{
    if (!s || g < 0 || g >= s->ng || which < 0 || which > 21 || !dst) return fail(s, ECSG_ERR_INVALID, "get_gradient: bad arguments");
    if (int rc = adj_check(s)) return rc;
    const Geo &G = s->geo[g];
    const size_t box = (size_t)G.size();
    if (which == 0) return get_box(s, s->gbblk[g], G, G.nx + 1, G.ny + 1, G.nz + 1, 0, dst);
    const int k = which - 1;
    return get_box(s, (const char *)s->gcblk[g] + k * box * s->tsize, G, G.nx + 1 - kCij21Pos[k][0],
                   G.ny + 1 - kCij21Pos[k][1], G.nz + 1 - kCij21Pos[k][2], 0, dst);
}

long long ecsg_gradient_elems(const ecsg_sim *s, int g)
{
    if (!s || g < 0 || g >= s->ng) return -1;
    const Geo &G = s->geo[g];
    long long n = (long long)(G.nx + 1) * (G.ny + 1) * (G.nz + 1);
    for (int k = 0; k < 21; k++)
        n += (long long)(G.nx + 1 - kCij21Pos[k][0]) * (G.ny + 1 - kCij21Pos[k][1]) * (G.nz + 1 - kCij21Pos[k][2]);
    return n;
}

// the 22 gradient volumes of grid g, each without halo, x fastest: node
// buoyancy, then the 21 slots at their positions
template <typename T>
static int gradient_move(ecsg_sim *s, int g, double *packed, bool to_packed)
{
    const Geo &G = s->geo[g];
    const size_t box = (size_t)G.size();
    size_t off = 0;
    for (int w = 0; w < 22; w++) {
        T *vol = w == 0 ? (T *)s->gbblk[g] : (T *)s->gcblk[g] + (size_t)(w - 1) * box;
        const int *p = w == 0 ? nullptr : kCij21Pos[w - 1];
        const int l0 = G.nx + 1 - (p ? p[0] : 0), l1 = G.ny + 1 - (p ? p[1] : 0), l2 = G.nz + 1 - (p ? p[2] : 0);
        if (to_packed) CK(launch_unpack<T>(packed + off, G, vol, l0, l1, l2, 0, s->st));
        else CK((launch_pack<T, double>(vol, G, packed + off, l0, l1, l2, 0, s->st)));
        off += (size_t)l0 * l1 * l2;
    }
    return ECSG_OK;
}

int ecsg_pack_gradient(ecsg_sim *s, int g, double *dst)
{
    if (!s || g < 0 || g >= s->ng || !dst) return fail(s, ECSG_ERR_INVALID, "pack_gradient: bad arguments");
    if (int rc = adj_check(s)) return rc;
    return DISPATCH(gradient_move)(s, g, dst, true);
}

int ecsg_unpack_gradient(ecsg_sim *s, int g, const double *src)
{
    if (!s || g < 0 || g >= s->ng || !src) return fail(s, ECSG_ERR_INVALID, "unpack_gradient: bad arguments");
    if (int rc = adj_check(s)) return rc;
    return DISPATCH(gradient_move)(s, g, const_cast<double *>(src), false);
}

void *ecsg_stream(const ecsg_sim *s) { return s ? (void *)s->st : nullptr; }

int ecsg_adjoint_op(ecsg_sim *s, int op, int index)
{
    if (!s) return ECSG_ERR_INVALID;
    const bool grid_op = op == ECSG_ADJ_VEL || op == ECSG_ADJ_STRESS;
    if (grid_op ? (index < 0 || index >= s->ng) : (index < 1 || index >= s->ng))
        return fail(s, ECSG_ERR_INVALID, "adjoint_op: bad grid or interface index");
    if (int rc = adj_check(s)) return rc;
    int rc = s->prec == ECSG_F32 ? adj_op_current<float>(s, op, index) : adj_op_current<double>(s, op, index);
    if (rc) return rc;
    CK(cudaStreamSynchronize(s->st));
    return ECSG_OK;
}

// --- the reverse time loop --------------------------------------------------
static size_t state_bytes(const ecsg_sim *s)
{
    size_t b = 0;
    for (int g = 0; g < s->ng; g++) b += 9 * (size_t)s->geo[g].size() * s->tsize;
    for (int i = 1; i < s->ng; i++) b += sizeof(double) * (size_t)(s->geo[i].nx + 1) * (s->geo[i].ny + 1);
    return b;
}

// fields of every grid and the sxz warm starts (the forward is then recomputed bit for bit)
static int save_state(ecsg_sim *s, char *dst)
{
    for (int g = 0; g < s->ng; g++) {
        const size_t b = 9 * (size_t)s->geo[g].size() * s->tsize;
        CK(cudaMemcpyAsync(dst, s->fblk[g], b, cudaMemcpyDefault, s->st));
        dst += b;
    }
    for (int i = 1; i < s->ng; i++) {
        const size_t b = sizeof(double) * (size_t)(s->geo[i].nx + 1) * (s->geo[i].ny + 1);
        CK(cudaMemcpyAsync(dst, s->itf[i].X0, b, cudaMemcpyDefault, s->st));
        dst += b;
    }
    return ECSG_OK;
}

static int load_state(ecsg_sim *s, const char *src)
{
    for (int g = 0; g < s->ng; g++) {
        const size_t b = 9 * (size_t)s->geo[g].size() * s->tsize;
        CK(cudaMemcpyAsync(s->fblk[g], src, b, cudaMemcpyDefault, s->st));
        src += b;
    }
    for (int i = 1; i < s->ng; i++) {
        const size_t b = sizeof(double) * (size_t)(s->geo[i].nx + 1) * (s->geo[i].ny + 1);
        CK(cudaMemcpyAsync(s->itf[i].X0, src, b, cudaMemcpyDefault, s->st));
        src += b;
    }
    return ECSG_OK;
}

// The whole run state: save_state's part, then the displacement sums of the
// grids that keep them.  buf may be device or host memory.
static size_t run_state_bytes(const ecsg_sim *s)
{
    size_t b = state_bytes(s);
    for (int g = 0; g < s->ng; g++)
        if (s->dispblk[g]) b += 3 * (size_t)s->geo[g].size() * s->tsize;
    return b;
}

static int move_run_state(ecsg_sim *s, char *buf, bool save)
{
    if (int rc = save ? save_state(s, buf) : load_state(s, buf)) return rc;
    char *p = buf + state_bytes(s);
    for (int g = 0; g < s->ng; g++)
        if (s->dispblk[g]) {
            const size_t b = 3 * (size_t)s->geo[g].size() * s->tsize;
            CK(cudaMemcpyAsync(save ? p : s->dispblk[g], save ? s->dispblk[g] : p, b, cudaMemcpyDefault, s->st));
            p += b;
        }
    return ECSG_OK;
}

long long ecsg_state_bytes(const ecsg_sim *s) { return s ? (long long)run_state_bytes(s) : -1; }

int ecsg_save_state(ecsg_sim *s, void *dst)
{
    if (!s || !dst) return fail(s, ECSG_ERR_INVALID, "save_state: bad arguments");
    CK(cudaSetDevice(s->device));
    if (int rc = move_run_state(s, (char *)dst, true)) return rc;
    CK(cudaStreamSynchronize(s->st));
    return ECSG_OK;
}

int ecsg_load_state(ecsg_sim *s, const void *src)
{
    if (!s || !src) return fail(s, ECSG_ERR_INVALID, "load_state: bad arguments");
    CK(cudaSetDevice(s->device));
    if (int rc = move_run_state(s, (char *)src, false)) return rc;
    CK(cudaStreamSynchronize(s->st));
    return ECSG_OK;
}

// the forward fields of grid g as stored in a saved state
template <typename T>
static GridDev<T> dev_state(const ecsg_sim *s, int g, const char *state)
{
    GridDev<T> G = dev<T>(s, g);
    for (int h = 0; h < g; h++) state += 9 * (size_t)s->geo[h].size() * sizeof(T);
    for (int k = 0; k < 9; k++) G.f[k] = (T *)state + k * (size_t)s->geo[g].size();
    return G;
}

static int set_clock(ecsg_sim *s, int n)
{
    s->run_n0 = n;
    CK(cudaMemcpyAsync(s->ints + 1, &s->run_n0, sizeof(int), cudaMemcpyHostToDevice, s->st));
    CK(cudaMemcpyAsync(s->ints + 3, &s->run_n0, sizeof(int), cudaMemcpyHostToDevice, s->st));
    CK(cudaStreamSynchronize(s->st));   // run_n0 is read by the copies above
    return ECSG_OK;
}

template <typename T>
static int misfit_gradient_op(ecsg_sim *s, int nsteps, const float *observed, int k, double *loss)
{
    int rc;
    const size_t sb = state_bytes(s);
    const int ncp = (nsteps + k - 1) / k;
    const size_t nrec = (size_t)s->nrec, nobs = (size_t)nsteps * nrec;
    auto grow = [&](void **p, size_t &cap, size_t want) -> int {
        if (cap >= want) return ECSG_OK;
        cudaFree(*p);
        *p = nullptr;
        cap = 0;
        CK(cudaMalloc(p, want));
        cap = want;
        return ECSG_OK;
    };
    if ((rc = grow((void **)&s->ckpt, s->ckpt_cap, sb * (ncp + 1)))) return rc;   // + the final state
    if ((rc = grow((void **)&s->seg, s->seg_cap, sb * (k + 1)))) return rc;
    if ((rc = grow(&s->recT, s->recT_cap, sizeof(T) * (nobs > 0 ? nobs : 1)))) return rc;
    if ((rc = grow((void **)&s->obs, s->obs_cap, sizeof(float) * (nobs > 0 ? nobs : 1)))) return rc;
    if (nobs) CK(cudaMemcpyAsync(s->obs, observed, sizeof(float) * nobs, cudaMemcpyHostToDevice, s->st));
    for (int i = 1; i < s->ng; i++)
        if ((rc = sxz_prepare<T>(s, i))) return rc;
    if ((rc = stress_prepare(s))) return rc;
    if ((rc = adj_zero(s, true, true))) return rc;
    // forward from rest with checkpoints every k steps
    std::optional<NvtxRange> forward_range;
    forward_range.emplace("misfit forward");
    for (int g = 0; g < s->ng; g++) CK(cudaMemsetAsync(s->fblk[g], 0, 9 * (size_t)s->geo[g].size() * s->tsize, s->st));
    for (int i = 1; i < s->ng; i++)
        CK(cudaMemsetAsync(s->itf[i].X0, 0, sizeof(double) * (s->geo[i].nx + 1) * (s->geo[i].ny + 1), s->st));
    if ((rc = set_clock(s, 0))) return rc;
    T *rec = (T *)s->recT;
    for (int n = 0; n < nsteps; n++) {
        if (n % k == 0 && (rc = save_state(s, s->ckpt + (size_t)(n / k) * sb))) return rc;
        if ((rc = step_op<T>(s, false, nullptr, nullptr, nrec ? rec + (size_t)n * nrec : nullptr))) return rc;
    }
    if ((rc = save_state(s, s->ckpt + (size_t)ncp * sb))) return rc;
    forward_range.reset();
    NvtxRange backward_range("misfit backward");
    CK(cudaMemsetAsync(s->dscal + 8, 0, sizeof(double), s->st));
    CK(launch_residual<T>(rec, s->obs, (int64_t)nobs, s->dscal + 8, s->partial, 12 * s->red_blocks, s->st));
    // backward, segment by segment: recompute the segment's states, then reverse its steps
    GridDev<T> Ga[kMaxGrids], Gb[kMaxGrids];
    RecAdj<T> R;
    memset(&R, 0, sizeof R);
    for (int g = 0; g < s->ng; g++) R.lbase[g] = adj_dev<T>(s, g).l[s->rec_comp];
    R.grid = s->rec_grid;
    R.off = s->rec_off;
    R.nrec = s->nrec;
    for (int c = ncp - 1; c >= 0; c--) {
        const int n0 = c * k, n1 = (n0 + k < nsteps) ? n0 + k : nsteps;
        if ((rc = load_state(s, s->ckpt + (size_t)c * sb))) return rc;
        if ((rc = set_clock(s, n0))) return rc;
        if ((rc = save_state(s, s->seg))) return rc;
        for (int n = n0; n < n1; n++) {
            if ((rc = step_op<T>(s, false, nullptr, nullptr))) return rc;
            if ((rc = save_state(s, s->seg + (size_t)(n - n0 + 1) * sb))) return rc;
        }
        for (int n = n1 - 1; n >= n0; n--) {
            const char *sa = s->seg + (size_t)(n - n0 + 1) * sb, *sbf = s->seg + (size_t)(n - n0) * sb;
            for (int g = 0; g < s->ng; g++) {
                Ga[g] = dev_state<T>(s, g, sa);
                Gb[g] = dev_state<T>(s, g, sbf);
            }
            for (int i = s->ng - 1; i >= 1; i--) {
                if ((rc = adj_op_impl<T>(s, ECSG_ADJ_GHOST_SYZ, i, Ga))) return rc;
                if ((rc = adj_op_impl<T>(s, ECSG_ADJ_GHOST_SXZ, i, Ga))) return rc;
            }
            for (int g = 0; g < s->ng; g++)
                if ((rc = adj_op_impl<T>(s, ECSG_ADJ_STRESS, g, Ga))) return rc;
            for (int i = s->ng - 1; i >= 1; i--)
                if ((rc = adj_op_impl<T>(s, ECSG_ADJ_GHOST_VZ, i, Ga))) return rc;
            if (nrec) {
                R.res = rec + (size_t)n * nrec;
                CK(launch_rec_adj<T>(R, s->st));
            }
            for (int g = s->ng - 1; g >= 0; g--)
                if ((rc = adj_op_impl<T>(s, ECSG_ADJ_VEL, g, Gb))) return rc;
        }
    }
    double l = 0.0;
    CK(cudaMemcpyAsync(&l, s->dscal + 8, sizeof(double), cudaMemcpyDeviceToHost, s->st));
    CK(cudaStreamSynchronize(s->st));
    if (loss) *loss = l;
    // leave the forward fields at the final state, the step clock after the last step
    if ((rc = load_state(s, s->ckpt + (size_t)ncp * sb))) return rc;
    if ((rc = set_clock(s, nsteps))) return rc;
    return ECSG_OK;
}

int ecsg_misfit_gradient(ecsg_sim *s, int nsteps, const float *observed, int ckpt_every, double *loss)
{
    if (!s || nsteps < 1 || ckpt_every < 1 || (s->nrec > 0 && !observed))
        return fail(s, ECSG_ERR_INVALID, "misfit_gradient: bad arguments");
    if (int rc = adj_check(s)) return rc;
    return DISPATCH(misfit_gradient_op)(s, nsteps, observed, ckpt_every, loss);
}

// ---------------------------------------------------------------------------
// Batches of instances (no reference counterpart): independent composites
// (different sizes and media) or shots sharing one medium.
// ---------------------------------------------------------------------------
#include <thread>

template <typename T>
static int batch_run_op(ecsg_sim *const *sims, int n, int n0, int nsteps, float *const *traces, double *ms_out)
{
    int rc;
    ecsg_sim *s0 = sims[0];
    ecsg_sim *s = s0;   // error messages go to the first instance
    for (int b = 0; b < n; b++) {
        ecsg_sim *x = sims[b];
        for (int i = 1; i < x->ng; i++)
            if ((rc = sxz_prepare<T>(x, i))) return rc;
        if ((rc = stress_prepare(x))) return rc;
        if (x->nrec > 0 && x->trace_cap < nsteps) {
            cudaFree(x->traces);
            x->traces = nullptr;
            if (cudaMalloc(&x->traces, sizeof(float) * (size_t)nsteps * x->nrec) != cudaSuccess)
                return fail(s, ECSG_ERR_CUDA, "batch_run: trace buffer of instance %d", b);
            x->trace_cap = nsteps;
            x->epoch++;
        }
        x->run_n0 = n0;
        CK(cudaMemcpyAsync(x->ints + 1, &x->run_n0, sizeof(int), cudaMemcpyHostToDevice, x->st));
        CK(cudaMemcpyAsync(x->ints + 3, &x->run_n0, sizeof(int), cudaMemcpyHostToDevice, x->st));
        CK(cudaStreamSynchronize(x->st));
    }
    // one graph for one step of every instance: fork from a master stream to
    // each instance's stream, join back
    cudaStream_t master;
    CK(cudaStreamCreateWithFlags(&master, cudaStreamNonBlocking));
    std::vector<cudaEvent_t> ev(n + 3);
    for (auto &e : ev) CK(cudaEventCreateWithFlags(&e, cudaEventDefault));
    cudaGraph_t gr = nullptr;
    cudaGraphExec_t gx = nullptr;
    auto cleanup = [&]() {
        if (gx) cudaGraphExecDestroy(gx);
        if (gr) cudaGraphDestroy(gr);
        for (auto &e : ev) cudaEventDestroy(e);
        cudaStreamDestroy(master);
    };
    rc = ECSG_OK;
    if (cudaStreamBeginCapture(master, cudaStreamCaptureModeThreadLocal) != cudaSuccess) {
        cleanup();
        return fail(s, ECSG_ERR_CUDA, "batch_run: capture");
    }
    cudaEventRecord(ev[0], master);
    for (int b = 0; b < n && !rc; b++) {
        ecsg_sim *x = sims[b];
        cudaStreamWaitEvent(x->st, ev[0], 0);
        rc = step_op<T>(x, false, nullptr, nullptr);
        cudaEventRecord(ev[3 + b], x->st);
        cudaStreamWaitEvent(master, ev[3 + b], 0);
    }
    cudaError_t e = cudaStreamEndCapture(master, &gr);
    if (rc || e != cudaSuccess || cudaGraphInstantiate(&gx, gr, 0) != cudaSuccess) {
        cleanup();
        cudaGetLastError();
        return rc ? rc : fail(s, ECSG_ERR_CUDA, "batch_run: graph");
    }
    cudaEventRecord(ev[1], master);
    for (int k = 0; k < nsteps; k++)
        if (cudaGraphLaunch(gx, master) != cudaSuccess) {
            cleanup();
            return fail(s, ECSG_ERR_CUDA, "batch_run: graph launch");
        }
    cudaEventRecord(ev[2], master);
    if (cudaStreamSynchronize(master) != cudaSuccess) {
        cleanup();
        return fail(s, ECSG_ERR_CUDA, "batch_run: %s", cudaGetErrorString(cudaGetLastError()));
    }
    float ms = 0;
    cudaEventElapsedTime(&ms, ev[1], ev[2]);
    if (ms_out) *ms_out = ms;
    cleanup();
    for (int b = 0; b < n; b++) {
        ecsg_sim *x = sims[b];
        x->last_run_ms = ms;
        x->launches = (long long)nsteps * (4LL * x->ng + src_rec_kernels(x->nrec, 3) + 5LL * (x->ng - 1));
        if (traces && traces[b] && x->nrec > 0)
            CK(cudaMemcpy(traces[b], x->traces, sizeof(float) * (size_t)nsteps * x->nrec, cudaMemcpyDeviceToHost));
    }
    return ECSG_OK;
}

static int batch_check(ecsg_sim *const *sims, int n)
{
    if (!sims || n < 1 || !sims[0]) return ECSG_ERR_INVALID;
    for (int b = 0; b < n; b++) {
        if (!sims[b]) return fail(sims[0], ECSG_ERR_INVALID, "batch: instance %d is null", b);
        if (sims[b]->prec != sims[0]->prec || sims[b]->device != sims[0]->device)
            return fail(sims[0], ECSG_ERR_INVALID, "batch: instances need one precision and one device");
        if (int rc = check_ready(sims[b])) return rc;
    }
    if (cudaSetDevice(sims[0]->device) != cudaSuccess) return fail(sims[0], ECSG_ERR_CUDA, "cudaSetDevice");
    return ECSG_OK;
}

int ecsg_batch_run(ecsg_sim *const *sims, int n, int n0, int nsteps, float *const *traces, double *ms)
{
    NvtxRange range("ecsg_batch_run");
    if (int rc = batch_check(sims, n)) return rc;
    if (nsteps < 1) return ECSG_OK;
    return sims[0]->prec == ECSG_F32 ? batch_run_op<float>(sims, n, n0, nsteps, traces, ms)
                                     : batch_run_op<double>(sims, n, n0, nsteps, traces, ms);
}

int ecsg_batch_misfit_gradient(ecsg_sim *const *sims, int n, int nsteps, const float *const *observed, int ckpt_every,
                               double *losses)
{
    if (int rc = batch_check(sims, n)) return rc;
    std::vector<int> rcs(n, ECSG_OK);
    std::vector<std::thread> th;
    // one host thread per instance, each on its own stream: their kernels overlap on the device
    for (int b = 0; b < n; b++)
        th.emplace_back([&, b]() {
            double l = 0.0;
            rcs[b] = ecsg_misfit_gradient(sims[b], nsteps, observed ? observed[b] : nullptr, ckpt_every, &l);
            if (losses) losses[b] = l;
        });
    for (auto &t : th) t.join();
    for (int b = 0; b < n; b++)
        if (rcs[b]) return fail(sims[0], rcs[b], "batch gradient, instance %d: %s", b, sims[b]->err.c_str());
    return ECSG_OK;
}

// dst[i] = sum_b src_b[i], accumulated in double
template <typename T>
__global__ void grad_sum_kernel(T *dst, T *const *src, int n, int64_t count)
{
    for (int64_t i = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (int64_t)gridDim.x * blockDim.x) {
        double acc = 0.0;
        for (int b = 0; b < n; b++) acc += (double)src[b][i];
        dst[i] = (T)acc;
    }
}

int ecsg_sum_gradients(ecsg_sim *dst, ecsg_sim *const *srcs, int n)
{
    if (!dst || !srcs || n < 1) return ECSG_ERR_INVALID;
    ecsg_sim *s = dst;
    if (int rc = adj_check(dst)) return rc;
    for (int b = 0; b < n; b++) {
        if (!srcs[b] || !srcs[b]->adj || srcs[b]->prec != dst->prec || srcs[b]->ng != dst->ng)
            return fail(dst, ECSG_ERR_INVALID, "sum_gradients: instance %d has no gradient of this geometry", b);
        for (int g = 0; g < dst->ng; g++)
            if (srcs[b]->geo[g].size() != dst->geo[g].size()) return fail(dst, ECSG_ERR_INVALID, "sum_gradients: grid sizes differ");
        CK(cudaStreamSynchronize(srcs[b]->st));
    }
    void **dptr = nullptr;
    CK(cudaMalloc(&dptr, sizeof(void *) * n));
    std::vector<void *> hp(n);
    for (int g = 0; g < dst->ng; g++)
        for (int part = 0; part < 2; part++) {
            const int64_t count = (int64_t)dst->geo[g].size() * (part == 0 ? 1 : 21);
            for (int b = 0; b < n; b++) hp[b] = part == 0 ? srcs[b]->gbblk[g] : srcs[b]->gcblk[g];
            CK(cudaMemcpyAsync(dptr, hp.data(), sizeof(void *) * n, cudaMemcpyHostToDevice, dst->st));
            void *out = part == 0 ? dst->gbblk[g] : dst->gcblk[g];
            const unsigned nb = (unsigned)((count + 255) / 256 > 4096 ? 4096 : (count + 255) / 256);
            if (dst->prec == ECSG_F32)
                grad_sum_kernel<float><<<nb, 256, 0, dst->st>>>((float *)out, (float *const *)dptr, n, count);
            else
                grad_sum_kernel<double><<<nb, 256, 0, dst->st>>>((double *)out, (double *const *)dptr, n, count);
            CK(cudaGetLastError());
            CK(cudaStreamSynchronize(dst->st));
        }
    cudaFree(dptr);
    return ECSG_OK;
}

// ---------------------------------------------------------------------------
// Shots in lockstep (no reference counterpart): the misfit gradients of S
// shots that share one medium (instances of one model made by
// ecsg_create_shot), advanced together step by step on one stream.  Every
// phase of a forward or adjoint step runs for all shots before the next
// phase, so that the phases that read the medium (the stress and velocity
// adjoints) or solve interface systems (the sxz solves) do so once for all
// shots; the others run per shot.  Checkpoints: every k steps
// (k = ckpt_every); the states inside a segment are recomputed from its
// checkpoint, directly when the k + 1 states of every shot fit in device
// memory, otherwise through sub-checkpoints every j steps (j ~ sqrt(k)) and
// j + 1 states, for one more forward pass.  The gradient of the sum of the
// shots' misfits is left in sims[0]: the stress and velocity adjoints add
// every shot's terms to sims[0]'s gradient arrays directly (one read-modify-
// write per point for all shots), the interface adjoints add to each shot's
// own arrays, and the shots' arrays are summed in FP64 at the end.
// losses[b] is shot b's misfit.
// ---------------------------------------------------------------------------
static int group_check(ecsg_sim *const *sims, int S)
{
    if (int rc = batch_check(sims, S)) return rc;
    ecsg_sim *m = sims[0];
    const ecsg_sim *model = m->share ? m->share : m;
    for (int b = 0; b < S; b++) {
        ecsg_sim *x = sims[b];
        if (int rc = adj_check(x)) return rc;
        const ecsg_sim *xm = x->share ? x->share : x;
        if (xm != model) return fail(m, ECSG_ERR_INVALID, "shots: instance %d does not share the first instance's medium", b);
        if (x->nrec != m->nrec || x->rec_comp != m->rec_comp)
            return fail(m, ECSG_ERR_INVALID, "shots: instance %d has another receiver count or component", b);
    }
    return ECSG_OK;
}

// Runs f(x, b) for every shot with the shot's library stream set to the group's stream.
template <typename F>
static int each_shot(ecsg_sim *const *sims, int S, F f)
{
    cudaStream_t gs = sims[0]->st;
    for (int b = 0; b < S; b++) {
        ecsg_sim *x = sims[b];
        cudaStream_t own = x->st;
        x->st = gs;
        const int rc = f(x, b);
        x->st = own;
        if (rc) return x == sims[0] ? rc : fail(sims[0], rc, "shot %d: %s", b, x->err.c_str());
    }
    return ECSG_OK;
}

// The sxz solves of every interface of every shot: one cooperative launch over
// as many (shot, interface) systems as fit co-resident, each bitwise as in its
// own launch.
template <typename T>
static int group_sxz_op(ecsg_sim *const *sims, int S)
{
    ecsg_sim *m = sims[0], *s = m;   // s: where CK reports
    if (m->imode == ECSG_MODE_II || !m->sxz_fused)
        return each_shot(sims, S, [&](ecsg_sim *x, int) { return sxz_all_op<T>(x); });
    SxzSysList<T> L;
    memset(&L, 0, sizeof L);
    int cta = 0;
    auto flush = [&]() -> int {
        if (!L.n) return ECSG_OK;
        L.r = m->itf[1].r;
        L.bar = m->bar;
        L.status = m->ints;
        CK(launch_sxz_solve_multi<T>(L, m->st));
        return ECSG_OK;
    };
    for (int b = 0; b < S; b++) {
        ecsg_sim *x = sims[b];
        for (int i = 1; i < x->ng; i++) {
            const int nb = x->itf[i].nblocks;
            if (x->itf[i].r != m->itf[1].r) return fail(m, ECSG_ERR_INVALID, "shots: interfaces of different ratios");
            if (L.n == kMaxSxzSys || cta + nb > m->sxz_cap) {
                if (int rc = flush()) return rc;
                memset(&L, 0, sizeof L);
                cta = 0;
            }
            SxzSys<T> &Y = L.s[L.n++];
            Y.F = dev<T>(x, i - 1);
            Y.C = dev<T>(x, i);
            Y.W = sxz_work(x, i);
            Y.cta0 = cta;
            Y.ncta = nb;
            cta += nb;
        }
    }
    return flush();
}

// One forward step of every shot (the order of main.cpp:165-261 within each
// shot); sample_rows[b]: shot b's receiver samples of this step, or null.
// The FP32 TMA sweeps of every shot of grid g in one launch (the shots' CTAs
// of a tile column adjacent, so the medium planes one stages are L2 hits for
// the others); false where the shots take the per-shot operators.
template <typename T>
static bool group_tma(ecsg_sim *const *sims, int S, bool stress)
{
    if (!std::is_same<T, float>::value || S < 2) return false;
    const char *env = getenv("ECSG_SHOTS_TMA");   // "0": the shots' sweeps launched one shot at a time
    if (env && env[0] == '0') return false;
    for (int b = 0; b < S; b++)
        if (!(stress ? use_s21_tma(sims[b]) : use_vel_tma(sims[b])) || (stress && sims[b]->energy)) return false;
    return true;
}

template <typename T>
static int group_step_op(ecsg_sim *const *sims, int S, T *const *sample_rows)
{
    ecsg_sim *s = sims[0];   // where CK reports
    ecsg_sim *m = s;
    int rc;
    std::vector<const void *> maps(S);
    if (group_tma<T>(sims, S, false)) {
        for (int g = 0; g < m->ng; g++) {
            for (int b = 0; b < S; b++) maps[b] = sims[b]->velmaps[g].data();
            CK(launch_vel_tma_shots(maps.data(), S, dev<float>(m, g), top_of(m, g, -1), bottom_of(m, g, -1), m->top_bc,
                                    m->ints, m->sms, m->st, 0));
            std::vector<T *> vy(S), vz(S);
            for (int b = 0; b < S; b++) {
                vy[b] = (T *)sims[b]->f[g][VY];
                vz[b] = (T *)sims[b]->f[g][VZ];
            }
            CK(launch_vel_mirror_shots<T>(m->geo[g], vy.data(), vz.data(), S, top_of(m, g, -1), bottom_of(m, g, -1),
                                          m->top_bc, m->mirror_fix, m->st));
        }
    } else if ((rc = each_shot(sims, S, [&](ecsg_sim *x, int) {
                    return each_grid(x, [&](int g) { return vel_op<T>(x, g, false); });
                })))
        return rc;
    if ((rc = each_shot(sims, S, [&](ecsg_sim *x, int b) -> int {
             if (sample_rows && sample_rows[b]) CK(launch_rec_sample<T>(make_srcrec(x, 0), sample_rows[b], x->st));
             CK(launch_src_rec<T>(make_srcrec(x, 3), x->st));
             return each_vz_ghost<T>(x);
         })))
        return rc;
    if (group_tma<T>(sims, S, true)) {
        for (int g = 0; g < m->ng; g++) {
            for (int b = 0; b < S; b++) maps[b] = sims[b]->s21maps[g].data();
            CK(launch_stress21_tma_shots(maps.data(), S, dev<float>(m, g), top_of(m, g, -1), m->top_bc, false, m->ints,
                                         m->sms, m->st, 0));
        }
    } else if ((rc = each_shot(sims, S, [&](ecsg_sim *x, int) {
                    return each_grid(x, [&](int g) { return stress_op<T>(x, g); });
                })))
        return rc;
    if ((rc = group_sxz_op<T>(sims, S))) return rc;
    return each_shot(sims, S, [&](ecsg_sim *x, int) -> int {
        for (int i = 1; i < x->ng; i++)
            if (int r2 = syz_op<T>(x, i)) return r2;
        return ECSG_OK;
    });
}

// The shots' views of grid g for the multi-shot adjoint kernels: forward
// fields from each shot's stored state `st[b]`, its adjoint fields and work boxes.
template <typename T>
static AdjShots<T> shot_set(ecsg_sim *const *sims, int S, int g, const char *const *st)
{
    AdjShots<T> A;
    memset(&A, 0, sizeof A);
    A.ns = S;
    A.box = sims[0]->geo[g].size();
    A.wbox = (int64_t)sims[0]->wbox;
    for (int b = 0; b < S; b++) {
        A.f[b] = dev_state<T>(sims[b], g, st[b]).f[0];
        A.l[b] = (T *)sims[b]->lblk[g];
        A.w[b] = (T *)sims[b]->wblk;
    }
    return A;
}

// One adjoint step of every shot: sa[b] / sb[b] are shot b's stored states
// after / before the step.
template <typename T>
static int group_adjoint_step(ecsg_sim *const *sims, int S, const char *const *sa, const char *const *sbf, int n)
{
    ecsg_sim *m = sims[0], *s = m;   // s: where CK reports
    const int ng = m->ng;
    int rc;
    auto states = [&](ecsg_sim *x, int b, const char *const *st, GridDev<T> *Gv) {
        for (int g = 0; g < ng; g++) Gv[g] = dev_state<T>(x, g, st[b]);
    };
    // interfaces from the deepest: per shot the syz adjoint and the collection
    // of the sxz adjoint's right-hand side, the sxz adjoint solves of all shots
    // in shared cooperative launches, then per shot their scatter
    for (int i = ng - 1; i >= 1; i--) {
        if ((rc = each_shot(sims, S, [&](ecsg_sim *x, int b) -> int {
                 GridDev<T> Ga[kMaxGrids];
                 states(x, b, sa, Ga);
                 if (int r2 = adj_op_impl<T>(x, ECSG_ADJ_GHOST_SYZ, i, Ga)) return r2;
                 if (x->imode == ECSG_MODE_II) return adj_op_impl<T>(x, ECSG_ADJ_GHOST_SXZ, i, Ga);
                 CK(launch_sxz_adj_collect<T>(Ga[i - 1], Ga[i], adj_dev<T>(x, i - 1), adj_dev<T>(x, i), x->itf[i].r,
                                              x->adj_lx[i], x->st));
                 return ECSG_OK;
             })))
            return rc;
        if (m->imode == ECSG_MODE_II) continue;
        SxzAdjList L;
        memset(&L, 0, sizeof L);
        int cta = 0;
        auto flush = [&]() -> int {
            if (!L.n) return ECSG_OK;
            L.bar = m->bar;
            L.status = m->ints;
            CK(launch_sxz_adj_solve_multi(L, m->st));
            memset(&L, 0, sizeof L);
            cta = 0;
            return ECSG_OK;
        };
        for (int b = 0; b < S; b++) {
            ecsg_sim *x = sims[b];
            const int nb = x->itf[i].nblocks;
            if (L.n == kMaxSxzSys || cta + nb > m->sxz_adj_cap)
                if ((rc = flush())) return rc;
            SxzAdjSys &Y = L.s[L.n++];
            Y.W = sxz_work(x, i);
            Y.W.X0 = x->adj_Y0[i];
            Y.W.X1 = x->adj_Y1[i];
            Y.lx = x->adj_lx[i];
            Y.nx2 = x->geo[i].nx;
            Y.ny2 = x->geo[i].ny;
            Y.cta0 = cta;
            Y.ncta = nb;
            cta += nb;
        }
        if ((rc = flush())) return rc;
        if ((rc = each_shot(sims, S, [&](ecsg_sim *x, int b) -> int {
                 GridDev<T> Ga[kMaxGrids];
                 states(x, b, sa, Ga);
                 CK(launch_sxz_adj_scatter<T>(Ga[i - 1], Ga[i], adj_dev<T>(x, i - 1), adj_dev<T>(x, i), x->itf[i].r,
                                              x->adj_Y0[i], x->st));
                 return ECSG_OK;
             })))
            return rc;
    }
    for (int g = 0; g < ng; g++)
        CK(launch_stress21_adj_shots<T>(dev<T>(m, g), adj_dev<T>(m, g), shot_set<T>(sims, S, g, sa), g == 0, m->top_bc,
                                        m->sms, m->st));
    if ((rc = each_shot(sims, S, [&](ecsg_sim *x, int b) -> int {
             GridDev<T> Ga[kMaxGrids];
             states(x, b, sa, Ga);
             for (int i = ng - 1; i >= 1; i--)
                 if (int r2 = adj_op_impl<T>(x, ECSG_ADJ_GHOST_VZ, i, Ga)) return r2;
             if (x->nrec) {
                 RecAdj<T> R;
                 memset(&R, 0, sizeof R);
                 for (int g = 0; g < ng; g++) R.lbase[g] = adj_dev<T>(x, g).l[x->rec_comp];
                 R.grid = x->rec_grid;
                 R.off = x->rec_off;
                 R.nrec = x->nrec;
                 R.res = (T *)x->recT + (size_t)n * x->nrec;
                 CK(launch_rec_adj<T>(R, x->st));
             }
             return ECSG_OK;
         })))
        return rc;
    for (int g = ng - 1; g >= 0; g--)
        CK(launch_vel_adj_shots<T>(dev<T>(m, g), (T *)m->gbblk[g], shot_set<T>(sims, S, g, sbf), g == 0, g == ng - 1,
                                   m->top_bc, m->mirror_fix, m->sms, m->st));
    return ECSG_OK;
}

template <typename T>
static int group_gradient_op(ecsg_sim *const *sims, int S, int nsteps, const float *const *observed, int k_req,
                             int sub_every, double *losses)
{
    int rc;
    ecsg_sim *m = sims[0], *s = m;   // s: where CK reports
    cudaStream_t gs = m->st;
    const size_t sb = state_bytes(m);
    // Memory plan, per shot: checkpoints every k steps (ncp + 1 states) and
    // one segment of k + 1 states.  When the requested interval does not fit,
    // a shorter one that does is taken first (the same single recomputation
    // of each segment, only more checkpoints); only when none fits is the
    // segment split again by sub-checkpoints every j steps (two levels, one
    // more forward pass of each segment).
    size_t margin = (size_t)1 << 30;
    size_t have = 0;
    {
        size_t free_b = 0, total_b = 0;
        CK(cudaMemGetInfo(&free_b, &total_b));
        have = free_b;
        for (int b = 0; b < S; b++) have += sims[b]->ckpt_cap + sims[b]->seg_cap + sims[b]->seg2_cap;
        // ECSG_SHOTS_MEMORY: the bytes the plan may give checkpoints and
        // segments, no margin (to exercise the plans on small cases)
        if (const char *env = getenv("ECSG_SHOTS_MEMORY")) {
            const size_t cap = (size_t)strtoull(env, nullptr, 10);
            if (cap > 0 && cap < have) have = cap;
            margin = 0;
        }
    }
    auto states = [&](int kk, int jj) {   // per shot, checkpoint interval kk, sub-checkpoints every jj
        const size_t ncp_ = (size_t)(nsteps + kk - 1) / kk;
        return (ncp_ + 1) + (size_t)(jj + 1) + (jj < kk ? (size_t)((kk + jj - 1) / jj) : 0);
    };
    auto fits_n = [&](int n, int kk, int jj) { return (size_t)n * sb * states(kk, jj) + margin <= have; };
    auto fits = [&](int kk, int jj) { return fits_n(S, kk, jj); };
    auto one_level = [&](int n) {   // the longest interval <= k_req at which n shots fit one level (0: none)
        int kk = k_req;
        while (kk >= 1 && !fits_n(n, kk, kk)) kk--;
        return kk;
    };
    auto release = [&](ecsg_sim *x) {
        cudaFree(x->ckpt);
        cudaFree(x->seg);
        cudaFree(x->seg2);
        x->ckpt = x->seg = x->seg2 = nullptr;
        x->ckpt_cap = x->seg_cap = x->seg2_cap = 0;
    };
    int k = k_req, j = k_req;
    if (sub_every > 0 && sub_every < k) {
        j = sub_every;
    } else if (!fits(k, k)) {
        const int kk = one_level(S);
        if (kk >= 1) {
            k = j = kk;
        } else {
            // groups of fewer shots that fit one level run in turn (each group
            // shares the medium; a two-level plan would cost one more forward
            // pass of every segment); their gradients are summed at the end
            int S1 = S;
            while (S1 > 1 && one_level(S1) < 1) S1 = (S1 + 1) / 2;
            if (S1 < S && one_level(S1) >= 1) {
                CK(cudaStreamSynchronize(gs));
                std::vector<ecsg_sim *> heads;
                for (int b0 = 0; b0 < S; b0 += S1) {
                    const int n = S - b0 < S1 ? S - b0 : S1;
                    for (int b = 0; b < S; b++) release(sims[b]);
                    if ((rc = group_gradient_op<T>(sims + b0, n, nsteps, observed ? observed + b0 : nullptr, k_req, 0,
                                                   losses ? losses + b0 : nullptr)))
                        return rc;
                    heads.push_back(sims[b0]);
                }
                for (int b = 0; b < S; b++) release(sims[b]);
                return heads.size() > 1 ? ecsg_sum_gradients(m, heads.data(), (int)heads.size()) : ECSG_OK;
            }
            j = 1;
            while ((size_t)j * j < (size_t)k) j++;
        }
    }
    if (!fits(k, j)) return fail(m, ECSG_ERR_CUDA, "shots: %d shots do not fit in device memory", S);
    const int ncp = (nsteps + k - 1) / k;
    const size_t nrec = (size_t)m->nrec, nobs = (size_t)nsteps * nrec;
    auto grow = [&](ecsg_sim *x, void **p, size_t &cap, size_t want) -> int {
        if (cap >= want) return ECSG_OK;
        cudaFree(*p);
        *p = nullptr;
        cap = 0;
        if (cudaMalloc(p, want) != cudaSuccess) {
            cudaGetLastError();
            return fail(m, ECSG_ERR_CUDA, "shots: %zu bytes of checkpoint memory for shot %p", want, (void *)x);
        }
        cap = want;
        return ECSG_OK;
    };
    // checkpoints and observations first, then the segment buffers (k + 1
    // states, or j + 1 and the sub-checkpoints); a shot whose buffers must
    // grow releases its old segment buffers first, as the plan counted them
    for (int b = 0; b < S; b++) {
        ecsg_sim *x = sims[b];
        if (x->ckpt_cap < sb * (ncp + 1) || x->seg_cap < sb * (j + 1)) {
            cudaFree(x->seg);
            cudaFree(x->seg2);
            x->seg = x->seg2 = nullptr;
            x->seg_cap = x->seg2_cap = 0;
        }
        if ((rc = grow(x, (void **)&x->ckpt, x->ckpt_cap, sb * (ncp + 1)))) return rc;
        if ((rc = grow(x, &x->recT, x->recT_cap, sizeof(T) * (nobs > 0 ? nobs : 1)))) return rc;
        if ((rc = grow(x, (void **)&x->obs, x->obs_cap, sizeof(float) * (nobs > 0 ? nobs : 1)))) return rc;
        if (nobs) CK(cudaMemcpyAsync(x->obs, observed[b], sizeof(float) * nobs, cudaMemcpyHostToDevice, gs));
    }
    const int nsub = (k + j - 1) / j;
    for (int b = 0; b < S; b++) {
        ecsg_sim *x = sims[b];
        if ((rc = grow(x, (void **)&x->seg, x->seg_cap, sb * (j + 1)))) return rc;
        if (j < k && (rc = grow(x, (void **)&x->seg2, x->seg2_cap, sb * nsub))) return rc;
    }
    if ((rc = each_shot(sims, S, [&](ecsg_sim *x, int) -> int {
             for (int i = 1; i < x->ng; i++)
                 if (int r2 = sxz_prepare<T>(x, i)) return r2;
             if (int r2 = stress_prepare(x)) return r2;
             return adj_zero(x, true, true);
         })))
        return rc;
    auto set_clocks = [&](int n) -> int {
        for (int b = 0; b < S; b++) {
            ecsg_sim *x = sims[b];
            x->run_n0 = n;
            CK(cudaMemcpyAsync(x->ints + 1, &x->run_n0, sizeof(int), cudaMemcpyHostToDevice, gs));
            CK(cudaMemcpyAsync(x->ints + 3, &x->run_n0, sizeof(int), cudaMemcpyHostToDevice, gs));
        }
        CK(cudaStreamSynchronize(gs));   // run_n0 is read by the copies above
        return ECSG_OK;
    };
    auto save_all = [&](char *ecsg_sim::*buf, size_t idx) {
        return each_shot(sims, S, [&](ecsg_sim *x, int) { return save_state(x, x->*buf + idx * sb); });
    };
    auto load_all = [&](char *ecsg_sim::*buf, size_t idx) {
        return each_shot(sims, S, [&](ecsg_sim *x, int) { return load_state(x, x->*buf + idx * sb); });
    };
    std::vector<T *> rows(S);
    // forward from rest with checkpoints every k steps
    {
        NvtxRange range("shots forward");
        for (int b = 0; b < S; b++) {
            ecsg_sim *x = sims[b];
            for (int g = 0; g < x->ng; g++) CK(cudaMemsetAsync(x->fblk[g], 0, 9 * (size_t)x->geo[g].size() * x->tsize, gs));
            for (int i = 1; i < x->ng; i++)
                CK(cudaMemsetAsync(x->itf[i].X0, 0, sizeof(double) * (x->geo[i].nx + 1) * (x->geo[i].ny + 1), gs));
        }
        if ((rc = set_clocks(0))) return rc;
        for (int n = 0; n < nsteps; n++) {
            if (n % k == 0 && (rc = save_all(&ecsg_sim::ckpt, n / k))) return rc;
            for (int b = 0; b < S; b++) rows[b] = nrec ? (T *)sims[b]->recT + (size_t)n * nrec : nullptr;
            if ((rc = group_step_op<T>(sims, S, rows.data()))) return rc;
        }
        if ((rc = save_all(&ecsg_sim::ckpt, ncp))) return rc;
    }
    NvtxRange range("shots backward");
    for (int b = 0; b < S; b++) {
        ecsg_sim *x = sims[b];
        CK(cudaMemsetAsync(x->dscal + 8, 0, sizeof(double), gs));
        CK(launch_residual<T>((T *)x->recT, x->obs, (int64_t)nobs, x->dscal + 8, x->partial, 12 * x->red_blocks, gs));
    }
    std::vector<const char *> sa(S), sbf(S);
    for (int c = ncp - 1; c >= 0; c--) {
        const int n0 = c * k, n1 = (n0 + k < nsteps) ? n0 + k : nsteps;
        if (j < k) {   // sub-checkpoints of this segment, up to the start of its last sub-segment
            if ((rc = load_all(&ecsg_sim::ckpt, c))) return rc;
            if ((rc = set_clocks(n0))) return rc;
            const int last = n0 + ((n1 - n0 - 1) / j) * j;
            for (int n = n0; n <= last; n++) {
                if ((n - n0) % j == 0 && (rc = save_all(&ecsg_sim::seg2, (n - n0) / j))) return rc;
                if (n < last && (rc = group_step_op<T>(sims, S, nullptr))) return rc;
            }
        }
        for (int d = (n1 - n0 - 1) / j; d >= 0; d--) {
            const int m0 = n0 + d * j, m1 = (m0 + j < n1) ? m0 + j : n1;
            if ((rc = j < k ? load_all(&ecsg_sim::seg2, d) : load_all(&ecsg_sim::ckpt, c))) return rc;
            if ((rc = set_clocks(m0))) return rc;
            if ((rc = save_all(&ecsg_sim::seg, 0))) return rc;
            for (int n = m0; n < m1; n++) {
                if ((rc = group_step_op<T>(sims, S, nullptr))) return rc;
                if ((rc = save_all(&ecsg_sim::seg, n - m0 + 1))) return rc;
            }
            for (int n = m1 - 1; n >= m0; n--) {
                for (int b = 0; b < S; b++) {
                    sa[b] = sims[b]->seg + (size_t)(n - m0 + 1) * sb;
                    sbf[b] = sims[b]->seg + (size_t)(n - m0) * sb;
                }
                if ((rc = group_adjoint_step<T>(sims, S, sa.data(), sbf.data(), n))) return rc;
            }
        }
    }
    // losses, then the shots' shares of the gradient summed (FP64) into sims[0]
    std::vector<double> l(S, 0.0);
    for (int b = 0; b < S; b++) CK(cudaMemcpyAsync(&l[b], sims[b]->dscal + 8, sizeof(double), cudaMemcpyDeviceToHost, gs));
    CK(cudaStreamSynchronize(gs));
    if (losses)
        for (int b = 0; b < S; b++) losses[b] = l[b];
    if (S > 1 && (rc = ecsg_sum_gradients(m, sims, S))) return rc;
    // leave every shot at its final forward state, the step clock after the last step
    if ((rc = load_all(&ecsg_sim::ckpt, ncp))) return rc;
    return set_clocks(nsteps);
}

int ecsg_shots_misfit_gradient(ecsg_sim *const *sims, int n, int nsteps, const float *const *observed, int ckpt_every,
                               int sub_every, double *losses)
{
    NvtxRange range("ecsg_shots_misfit_gradient");
    if (!sims || !sims[0]) return ECSG_ERR_INVALID;
    if (n < 1 || n > kMaxShots || nsteps < 1 || ckpt_every < 1)
        return fail(sims[0], ECSG_ERR_INVALID, "shots_misfit_gradient: bad arguments (1 <= n <= %d shots)", kMaxShots);
    if (int rc = group_check(sims, n)) return rc;
    if (sims[0]->nrec > 0 && !observed) return fail(sims[0], ECSG_ERR_INVALID, "shots_misfit_gradient: observed data missing");
    for (int b = 0; b < n && sims[0]->nrec > 0; b++)
        if (!observed[b]) return fail(sims[0], ECSG_ERR_INVALID, "shots_misfit_gradient: observed data of shot %d missing", b);
    return sims[0]->prec == ECSG_F32 ? group_gradient_op<float>(sims, n, nsteps, observed, ckpt_every, sub_every, losses)
                                     : group_gradient_op<double>(sims, n, nsteps, observed, ckpt_every, sub_every, losses);
}

// ---------------------------------------------------------------------------
// Autotuner: z-chunks of the FP32 velocity and stress sweeps per grid
// ---------------------------------------------------------------------------
int ecsg_autotune(ecsg_sim *s, int reps)
{
    NvtxRange range("ecsg_autotune");
    if (!s) return ECSG_ERR_INVALID;
    if (int rc = check_ready(s)) return rc;
    CK(cudaSetDevice(s->device));
    if (s->prec != ECSG_F32 || s->scalar_stencils) return ECSG_OK;   // only the FP32 sweeps take a chunk count
    if (reps < 1) reps = 3;
    int rc;
    if ((rc = stress_prepare(s))) return rc;
    // the trial sweeps change the fields (and displacement sums): keep and restore them
    char *save = nullptr;
    CK(cudaMalloc(&save, run_state_bytes(s) + 1));
    if ((rc = move_run_state(s, save, true))) { cudaFree(save); return rc; }
    cudaEvent_t e0, e1;
    CK(cudaEventCreate(&e0));
    CK(cudaEventCreate(&e1));
    const int cand[] = {0, 1, 2, 3, 4, 6, 8, 12, 16, 24};
    for (int g = 0; g < s->ng; g++)
        for (int kind = 0; kind < 2; kind++) {
            float best = 1e30f;
            int best_c = 0;
            for (int c : cand) {
                if (c > s->geo[g].nz + 1) continue;
                s->ztune[g][kind] = c;
                float t = 1e30f;
                for (int r = 0; r <= reps; r++) {   // the first repetition warms up
                    CK(cudaEventRecord(e0, s->st));
                    rc = kind == 0 ? vel_kernel_op<float>(s, g, false) : stress_op<float>(s, g);
                    if (rc) { cudaFree(save); return rc; }
                    CK(cudaEventRecord(e1, s->st));
                    CK(cudaEventSynchronize(e1));
                    float ms = 0;
                    CK(cudaEventElapsedTime(&ms, e0, e1));
                    if (r > 0 && ms < t) t = ms;
                }
                if (t < best * 0.99f) { best = t; best_c = c; }
            }
            s->ztune[g][kind] = best_c;
        }
    cudaEventDestroy(e0);
    cudaEventDestroy(e1);
    rc = move_run_state(s, save, false);
    CK(cudaStreamSynchronize(s->st));
    cudaFree(save);
    s->epoch++;   // the cached step graphs hold the old launch shapes
    return rc;
}

int ecsg_get_tuning(const ecsg_sim *s, int g, int chunks[2])
{
    if (!s || g < 0 || g >= s->ng || !chunks) return ECSG_ERR_INVALID;
    chunks[0] = s->ztune[g][0];
    chunks[1] = s->ztune[g][1];
    return ECSG_OK;
}
