// medium.cu -- tilted transversely isotropic (TTI) media built on the device.
//
// No reference counterpart: the reference reads isotropic node media only
// (init_del_par_field.cpp:99-149).  Input per node: vp, vs, rho, the tilt
// (dip) of the symmetry axis from vertical and its azimuth from x (radians),
// plus Thomsen's epsilon, delta, gamma for the whole grid.  In the frame of
// the symmetry axis (Thomsen 1986):
//   C33 = rho vp^2, C44 = C55 = rho vs^2, C11 = C22 = C33 (1 + 2 eps),
//   C66 = C44 (1 + 2 gamma), C12 = C11 - 2 C66,
//   C13 = C23 = sqrt((C33 - C44)(C33 (1 + 2 delta) - C44)) - C44.
// The tensor is rotated by a = Rz(azimuth) Ry(dip) (symmetry axis
// (sin dip cos az, sin dip sin az, cos dip)) with the Bond stress matrix:
// C' = M C M^T, M_IJ = a_ik a_jk for J = (k,k), a_ik a_jl + a_il a_jk for
// J = (k,l), k != l, with Voigt pairs 1:(1,1) 2:(2,2) 3:(3,3) 4:(2,3) 5:(3,1)
// 6:(1,2) (Auld, Acoustic Fields and Waves in Solids, ch. 3).
// Node values are then averaged to the slot positions with the 2/4/8-point
// means of the reference's ReshapeField (field.cpp:428-476).
#include "ecsg_device.cuh"

namespace ecsg {

__constant__ int kVoigt[6][2] = {{0, 0}, {1, 1}, {2, 2}, {1, 2}, {2, 0}, {0, 1}};

__device__ __forceinline__ double bond(const double a[3][3], int I, int J)
{
    const int i = kVoigt[I][0], j = kVoigt[I][1], k = kVoigt[J][0], l = kVoigt[J][1];
    return J < 3 ? a[i][k] * a[j][k] : a[i][k] * a[j][l] + a[i][l] * a[j][k];
}

// rotated stiffness entry (I, J), 0-based Voigt indices
__device__ double tti_cij(int I, int J, double vp, double vs, double rho, double dip, double azi, double eps,
                          double delta, double gamma)
{
    const double c33 = rho * vp * vp, c44 = rho * vs * vs;
    const double c11 = c33 * (1.0 + 2.0 * eps), c66 = c44 * (1.0 + 2.0 * gamma);
    const double c12 = c11 - 2.0 * c66;
    const double c13 = sqrt((c33 - c44) * (c33 * (1.0 + 2.0 * delta) - c44)) - c44;
    const double C[6][6] = {{c11, c12, c13, 0, 0, 0}, {c12, c11, c13, 0, 0, 0}, {c13, c13, c33, 0, 0, 0},
                            {0, 0, 0, c44, 0, 0},     {0, 0, 0, 0, c44, 0},     {0, 0, 0, 0, 0, c66}};
    double sd, cd, sa, ca;
    sincos(dip, &sd, &cd);
    sincos(azi, &sa, &ca);
    const double a[3][3] = {{ca * cd, -sa, ca * sd}, {sa * cd, ca, sa * sd}, {-sd, 0.0, cd}};
    double mi[6], mj[6];
#pragma unroll
    for (int K = 0; K < 6; K++) {
        mi[K] = bond(a, I, K);
        mj[K] = bond(a, J, K);
    }
    double s = 0.0;
#pragma unroll
    for (int K = 0; K < 6; K++)
#pragma unroll
        for (int L = 0; L < 6; L++)
            if (C[K][L] != 0.0) s += mi[K] * C[K][L] * mj[L];
    return s;
}

// One rotated entry at every node of the grid, node values in the box layout.
__global__ void tti_node_kernel(Geo g, const float *vp, const float *vs, const float *rho, const float *dip,
                                const float *azi, double eps, double delta, double gamma, int I, int J, double *out)
{
    const int64_t n = (int64_t)(g.nx + 1) * (g.ny + 1) * (g.nz + 1);
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(t % (g.nx + 1)), y = (int)((t / (g.nx + 1)) % (g.ny + 1)), z = (int)(t / ((int64_t)(g.nx + 1) * (g.ny + 1)));
        const int p = g.idx(x, y, z);
        out[p] = tti_cij(I, J, vp[p], vs[p], rho[p], dip[p], azi[p], eps, delta, gamma);
    }
}

template <typename T>
__global__ void node_buoy_kernel(Geo g, const float *rho, T *b)
{
    const int64_t n = (int64_t)(g.nx + 1) * (g.ny + 1) * (g.nz + 1);
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(t % (g.nx + 1)), y = (int)((t / (g.nx + 1)) % (g.ny + 1)), z = (int)(t / ((int64_t)(g.nx + 1) * (g.ny + 1)));
        const int p = g.idx(x, y, z);
        b[p] = (T)(1.0 / (double)rho[p]);
    }
}

// 2/4/8-point mean of node values at a staggered position (ReshapeField order)
template <typename T>
__global__ void stagger_kernel(Geo g, const double *f, int p0, int p1, int p2, T *dst)
{
    const int l0 = g.nx + 1 - p0, l1 = g.ny + 1 - p1, l2 = g.nz + 1 - p2;
    const int64_t n = (int64_t)l0 * l1 * l2;
    const int ox = p0, oy = p1 * g.px, oz = p2 * g.px * g.py;
    for (int64_t t = (int64_t)blockIdx.x * blockDim.x + threadIdx.x; t < n; t += (int64_t)gridDim.x * blockDim.x) {
        const int x = (int)(t % l0), y = (int)((t / l0) % l1), z = (int)(t / ((int64_t)l0 * l1));
        const int p = g.idx(x, y, z);
        dst[p] = (T)((f[p] + f[p + oz] + f[p + oy] + f[p + oy + oz] + f[p + ox] + f[p + ox + oz] + f[p + ox + oy]
                      + f[p + ox + oy + oz]) / 8);
    }
}

static int grid_blocks(int64_t n)
{
    int64_t b = (n + 255) / 256;
    return (int)(b > 8192 ? 8192 : b);
}

// node: vp, vs, rho, dip, azimuth in the box layout (float); work: one double box.
// slot[k] of the 21-Cij layout (Voigt pair and position of each slot below).
template <typename T>
cudaError_t launch_tti_medium(const Geo &g, const float *const node[5], double eps, double delta, double gamma,
                              double *work, T *buoy, T *const slot[21], cudaStream_t st)
{
    static const int pair[21][2] = {{0, 0}, {0, 1}, {0, 2}, {1, 1}, {1, 2}, {2, 2}, {0, 3}, {0, 4}, {0, 5}, {1, 3}, {1, 4},
                                    {1, 5}, {2, 3}, {2, 4}, {2, 5}, {3, 3}, {3, 4}, {3, 5}, {4, 4}, {4, 5}, {5, 5}};
    static const int pos[21][3] = {{1, 0, 0}, {1, 0, 0}, {1, 0, 0}, {1, 0, 0}, {1, 0, 0}, {1, 0, 0}, {1, 0, 0},
                                   {1, 0, 0}, {1, 0, 0}, {1, 0, 0}, {1, 0, 0}, {1, 0, 0}, {1, 0, 0}, {1, 0, 0},
                                   {1, 0, 0}, {1, 1, 1}, {1, 1, 1}, {1, 1, 1}, {0, 0, 1}, {0, 0, 1}, {0, 1, 0}};
    const int64_t nn = (int64_t)(g.nx + 1) * (g.ny + 1) * (g.nz + 1);
    node_buoy_kernel<T><<<grid_blocks(nn), 256, 0, st>>>(g, node[2], buoy);
    for (int k = 0; k < 21; k++) {
        tti_node_kernel<<<grid_blocks(nn), 256, 0, st>>>(g, node[0], node[1], node[2], node[3], node[4], eps, delta,
                                                        gamma, pair[k][0], pair[k][1], work);
        stagger_kernel<T><<<grid_blocks(nn), 256, 0, st>>>(g, work, pos[k][0], pos[k][1], pos[k][2], slot[k]);
    }
    return cudaGetLastError();
}

template cudaError_t launch_tti_medium<float>(const Geo &, const float *const[5], double, double, double, double *,
                                              float *, float *const[21], cudaStream_t);
template cudaError_t launch_tti_medium<double>(const Geo &, const float *const[5], double, double, double, double *,
                                               double *, double *const[21], cudaStream_t);

} // namespace ecsg
