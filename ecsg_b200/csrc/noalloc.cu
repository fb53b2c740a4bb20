// noalloc.cu -- the sxz interface solve for callers that cannot allocate device memory.
//
// Some hosts of this solver may not call cudaMalloc: a caller whose device
// memory is owned by another framework's allocator, or one running under a
// fixed memory budget where every byte was reserved up front, can hand over the
// fields it already holds but cannot let the library allocate work space.
// ecsg_ghost_sxz_noalloc serves them.  Its work space (the 9-diagonal matrix,
// the right-hand side, the second Jacobi iterate, the CTA partial sums and the
// grid-barrier words) lives in one file-scope device array of fixed size, so
// every GPU that loads the library holds those bytes until the process exits.
//
// The address of the array is taken once per device with cudaGetSymbolAddress
// (host code only sees a host-side stand-in under the array's name; that
// stand-in must never be handed to a kernel).  The first call on a device does
// this set-up, so that first call should come before any stream capture.
//
// Calls share the array and it keeps the last call's contents.  Each call
// clears the parts that must start at zero (the second iterate, whose border
// must be zero, and the barrier and per-call status words) before it launches;
// the matrix and right-hand side are rebuilt every call.  Calls that overlap on
// the GPU (from two streams, or two host threads) race on the array.
//
// A call that does not wait (iters == NULL) cannot return the solve's outcome.
// So every call also ORs its per-call status bits into a sticky word of the
// array, which no call clears; ecsg_ghost_sxz_noalloc_status reads it (and
// clears it on request) once the caller's stream has drained.
#include "ecsg_device.cuh"
#include "../../include/ecsg_b200.h"

#include <climits>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <mutex>

namespace ecsg {
template <typename T>
cudaError_t launch_sxz_matrix(const GridDev<T> &, const GridDev<T> &, int, double *, cudaStream_t);
template <typename T>
int sxz_solve_blocks(int, int);
template <typename T>
cudaError_t launch_sxz_solve(const GridDev<T> &, const GridDev<T> &, int, const SxzWork &, int, cudaStream_t);
} // namespace ecsg

using namespace ecsg;

namespace {
// Limits: (nx2-1)*(ny2-1) interior coarse nodes and (nx2+1)*(ny2+1) nodes.
constexpr size_t kMaxUnknowns = ECSG_NOALLOC_MAX_UNKNOWNS;
constexpr size_t kMaxNodes = ECSG_NOALLOC_MAX_NODES;
constexpr size_t kMaxBlocks = 4096;
// Carving of the array (bytes, each region 256-byte aligned).
constexpr size_t align256(size_t b) { return (b + 255) / 256 * 256; }
constexpr size_t kOffA = 0;
constexpr size_t kOffB = kOffA + align256(9 * kMaxUnknowns * sizeof(double));
constexpr size_t kOffX1 = kOffB + align256(kMaxUnknowns * sizeof(double));
constexpr size_t kOffPartial = kOffX1 + align256(kMaxNodes * sizeof(double));
constexpr size_t kOffWords = kOffPartial + align256(kMaxBlocks * sizeof(double));
// words: double total, double tol, long long iters_total, (spare), int status, int iters
constexpr size_t kWordsBytes = 64;
constexpr size_t kOffBar = kOffWords + align256(kWordsBytes);   // grid-barrier words
constexpr size_t kBarBytes = kBarWords * sizeof(unsigned);
// sticky status: the OR of every call's status bits since the last clear
constexpr size_t kOffSticky = kOffBar + align256(kBarBytes);
constexpr size_t kScratchBytes = kOffSticky + 256;
static_assert(kScratchBytes < (16u << 20), "scratch must stay modest");

constexpr int kMaxDevices = 64;
} // namespace

static __device__ __align__(256) unsigned char g_sxz_scratch[kScratchBytes];

// One thread: sticky |= this call's status (device code names the array itself).
__global__ void latch_status_kernel()
{
    int *sticky = (int *)(g_sxz_scratch + kOffSticky);
    const int st = *(const int *)(g_sxz_scratch + kOffWords + 32);
    if (st) *sticky |= st;
}

static void *scratch_address(int device, cudaError_t *err)
{
    static std::mutex mu;
    static void *addr[kMaxDevices] = {};
    std::lock_guard<std::mutex> lock(mu);
    *err = cudaSuccess;
    if (!addr[device]) {
        void *p = nullptr;
        *err = cudaGetSymbolAddress(&p, g_sxz_scratch);
        if (*err != cudaSuccess) return nullptr;
        addr[device] = p;
    }
    return addr[device];
}

static int report(char *errbuf, size_t errlen, int code, const char *msg)
{
    if (errbuf && errlen) snprintf(errbuf, errlen, "%s", msg);
    fprintf(stderr, "ecsg_ghost_sxz_noalloc: %s\n", msg);
    return code;
}

// The layout of a view must hold every element the kernels may index: x, y, z
// in [-radius, size + radius] inside the box the pitches span, with 32-bit
// indices (the kernels' index type).  Returns why not, or NULL.
static const char *check_view(const ecsg_grid_view *v)
{
    const long long R = v->radius;
    for (int d = 0; d < 3; d++) {
        if (v->size[d] < 1 || !(v->step[d] > 0)) return "grid view: size must be >= 1 and step > 0";
        if ((long long)v->pitch[d] < v->size[d] + 1 + 2 * R) return "grid view: pitch[d] must be >= size[d] + 1 + 2 * radius";
    }
    for (int k = 0; k < 9; k++)
        if (!v->field[k]) return "grid view: null field pointer";
    if (!v->buoy) return "grid view: null buoyancy pointer";
    const long long px = v->pitch[0], py = v->pitch[1], pz = v->pitch[2];
    const long long lo = v->origin - R * (px * py + px + 1);
    const long long hi = v->origin + ((v->size[2] + R) * py + v->size[1] + R) * px + v->size[0] + R;
    if (lo < 0 || hi >= px * py * pz) return "grid view: origin puts the halo outside the box of the pitches";
    if (px * py * pz > (long long)INT_MAX) return "grid view: box larger than 32-bit indexing";
    return nullptr;
}

template <typename T>
static GridDev<T> view_dev(const ecsg_grid_view *v, double dt)
{
    GridDev<T> G;
    memset(&G, 0, sizeof G);
    G.g.nx = v->size[0];
    G.g.ny = v->size[1];
    G.g.nz = v->size[2];
    G.g.R = v->radius;
    G.g.px = v->pitch[0];
    G.g.py = v->pitch[1];
    G.g.pz = v->pitch[2];
    G.g.off0 = (int)v->origin;
    for (int k = 0; k < 9; k++) G.f[k] = (T *)v->field[k];
    G.b = (const T *)v->buoy;
    for (int d = 0; d < 3; d++) {
        G.kd[d] = 1.0 * dt / v->step[d];
        G.k[d] = (T)G.kd[d];
    }
    return G;
}

template <typename T>
static int solve(const ecsg_grid_view *fine, const ecsg_grid_view *coarse, int r, double dt, double *X, int max_iter,
                 cudaStream_t st, int *iters, char *errbuf, size_t errlen)
{
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) return report(errbuf, errlen, ECSG_ERR_NO_DEVICE, "no current CUDA device");
    unsigned char *base = (unsigned char *)scratch_address(dev, &e);
    if (!base) return report(errbuf, errlen, ECSG_ERR_CUDA, cudaGetErrorString(e));
    int sms = 0;
    if (cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || sms <= 0)
        return report(errbuf, errlen, ECSG_ERR_CUDA, "cannot query the SM count");
    const int nn = (coarse->size[0] - 1) * (coarse->size[1] - 1);
    const int nblocks = sxz_solve_blocks<T>(nn, sms);
    if (2 * (size_t)nblocks > kMaxBlocks)   // two halves of partial sums (alternating reduction rounds)
        return report(errbuf, errlen, ECSG_ERR_INVALID, "too many SMs for the static partial sums");
    const size_t nodes = (size_t)(coarse->size[0] + 1) * (coarse->size[1] + 1);
    // zero the second iterate (its border must be zero) and the barrier/status words
    if ((e = cudaMemsetAsync(base + kOffX1, 0, nodes * sizeof(double), st)) != cudaSuccess ||
        (e = cudaMemsetAsync(base + kOffWords, 0, kOffBar - kOffWords + kBarBytes, st)) != cudaSuccess)
        return report(errbuf, errlen, ECSG_ERR_CUDA, cudaGetErrorString(e));
    const GridDev<T> F = view_dev<T>(fine, dt), C = view_dev<T>(coarse, dt);
    double *A = (double *)(base + kOffA);
    if ((e = launch_sxz_matrix<T>(F, C, r, A, st)) != cudaSuccess) return report(errbuf, errlen, ECSG_ERR_CUDA, cudaGetErrorString(e));
    unsigned char *w = base + kOffWords;
    SxzWork W;
    W.A = A;
    W.B = (double *)(base + kOffB);
    W.X0 = X;
    W.X1 = (double *)(base + kOffX1);
    W.partial = (double *)(base + kOffPartial);
    W.total = (double *)(w + 0);
    W.tol_out = (double *)(w + 8);
    W.iters_total = (long long *)(w + 16);
    W.bar = (unsigned *)(base + kOffBar);
    W.status = (int *)(w + 32);
    W.iters = (int *)(w + 36);
    W.max_iter = max_iter > 0 ? max_iter : 10000;
    if ((e = launch_sxz_solve<T>(F, C, r, W, nblocks, st)) != cudaSuccess) return report(errbuf, errlen, ECSG_ERR_CUDA, cudaGetErrorString(e));
    latch_status_kernel<<<1, 1, 0, st>>>();
    if ((e = cudaGetLastError()) != cudaSuccess) return report(errbuf, errlen, ECSG_ERR_CUDA, cudaGetErrorString(e));
    if (iters) {
        int hv[2] = {0, 0};
        if ((e = cudaMemcpyAsync(hv, W.status, sizeof hv, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
            (e = cudaStreamSynchronize(st)) != cudaSuccess)
            return report(errbuf, errlen, ECSG_ERR_CUDA, cudaGetErrorString(e));
        *iters = hv[1];
        if (hv[0] & ST_BARRIER_TIMEOUT) return report(errbuf, errlen, ECSG_ERR_CUDA, "grid barrier timed out");
        if (hv[0] & ST_JACOBI_CAP) return ECSG_ERR_NOT_CONVERGED;
    }
    return ECSG_OK;
}

int ecsg_ghost_sxz_noalloc(const ecsg_grid_view *fine, const ecsg_grid_view *coarse, double dt, int precision,
                           double *X, int max_iter, void *stream, int *iters, char *errbuf, size_t errlen)
{
    if (!fine || !coarse || !X || !(dt > 0)) return report(errbuf, errlen, ECSG_ERR_INVALID, "null argument or dt <= 0");
    if (precision != ECSG_F32 && precision != ECSG_F64) return report(errbuf, errlen, ECSG_ERR_INVALID, "precision");
    if (fine->radius != 1 || coarse->radius != 1) return report(errbuf, errlen, ECSG_ERR_INVALID, "radius must be 1");
    for (const ecsg_grid_view *v : {fine, coarse})
        if (const char *why = check_view(v)) return report(errbuf, errlen, ECSG_ERR_INVALID, why);
    // the same ratio rules as ecsg_create: an integer >= 2, equal in x and y
    const double rx = coarse->step[0] / fine->step[0];
    const int r = (int)std::lround(rx);
    if (r < 2 || fabs(rx - r) > 1e-6 * r || fabs(coarse->step[1] / fine->step[1] - r) > 1e-6 * r)
        return report(errbuf, errlen, ECSG_ERR_INVALID, "x/y refinement ratio must be an integer >= 2");
    if (fine->size[0] != r * coarse->size[0] || fine->size[1] != r * coarse->size[1])
        return report(errbuf, errlen, ECSG_ERR_INVALID, "fine size must be ratio * coarse size in x and y");
    const size_t nn = (size_t)(coarse->size[0] - 1) * (coarse->size[1] - 1);
    const size_t nodes = (size_t)(coarse->size[0] + 1) * (coarse->size[1] + 1);
    if (coarse->size[0] < 2 || coarse->size[1] < 2 || nn > kMaxUnknowns || nodes > kMaxNodes) {
        char msg[200];
        snprintf(msg, sizeof msg,
                 "coarse interface %dx%d cells exceeds the static work space (at most %zu interior nodes and %zu "
                 "nodes, e.g. 362x362 cells); use ecsg_ghost_sxz on an ecsg_sim instead",
                 coarse->size[0], coarse->size[1], kMaxUnknowns, kMaxNodes);
        return report(errbuf, errlen, ECSG_ERR_INVALID, msg);
    }
    cudaStream_t st = (cudaStream_t)stream;
    return precision == ECSG_F32 ? solve<float>(fine, coarse, r, dt, X, max_iter, st, iters, errbuf, errlen)
                                 : solve<double>(fine, coarse, r, dt, X, max_iter, st, iters, errbuf, errlen);
}

int ecsg_ghost_sxz_noalloc_status(void *stream, int *status, int clear)
{
    if (!status) return report(nullptr, 0, ECSG_ERR_INVALID, "status: null pointer");
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess || dev < 0 || dev >= kMaxDevices) return report(nullptr, 0, ECSG_ERR_NO_DEVICE, "no current CUDA device");
    unsigned char *base = (unsigned char *)scratch_address(dev, &e);
    if (!base) return report(nullptr, 0, ECSG_ERR_CUDA, cudaGetErrorString(e));
    cudaStream_t st = (cudaStream_t)stream;
    int v = 0;
    if ((e = cudaMemcpyAsync(&v, base + kOffSticky, sizeof v, cudaMemcpyDeviceToHost, st)) != cudaSuccess ||
        (clear && (e = cudaMemsetAsync(base + kOffSticky, 0, sizeof(int), st)) != cudaSuccess) ||
        (e = cudaStreamSynchronize(st)) != cudaSuccess)
        return report(nullptr, 0, ECSG_ERR_CUDA, cudaGetErrorString(e));
    *status = v;
    return ECSG_OK;
}
