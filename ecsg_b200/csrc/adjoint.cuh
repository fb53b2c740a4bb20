// adjoint.cuh -- adjoint state shared by adjoint.cu (grid operators),
// interface.cu (interface solves) and api.cu (the reverse time loop).
#pragma once
#include "ecsg_device.cuh"

namespace ecsg {

template <typename T>
struct AdjDev {
    T *l[9];     // adjoint of the 9 fields, the grid's box layout
    T *gb;       // gradient w.r.t. the node buoyancy
    T *gc[21];   // gradient w.r.t. the 21 stiffness slots
    T *w[15];    // work boxes of the stress adjoint (strains, average adjoints, strain adjoints)
};

// Shots of one grid advanced together (shots sharing one medium): per shot
// the block of the 9 forward fields the operator reads (field k at
// f[s] + k * box), the block of its 9 adjoint fields (l[s] + k * box) and its
// 15 work boxes (w[s] + k * wbox).  The medium and the gradient arrays are
// the shots' common ones.
template <typename T>
struct AdjShots {
    int ns;
    T *f[kMaxShots];
    T *l[kMaxShots];
    T *w[kMaxShots];
    int64_t box, wbox;
};

// Receiver adjoint sources of one step: lambda_{comp}[grid][off] += res[i].
template <typename T>
struct RecAdj {
    T *lbase[kMaxGrids];
    const int *grid;
    const int *off;
    const T *res;
    int nrec;
};

__device__ __forceinline__ void atom(float *p, float v) { atomicAdd(p, v); }
__device__ __forceinline__ void atom(double *p, double v) { atomicAdd(p, v); }

} // namespace ecsg
