// tma_util.cuh -- mbarrier and TMA helpers shared by the TMA-staged sweeps
// (stress21_tma.cu, vel_tma.cu), and the host encoder of their 4-D maps.
#pragma once
#include "ecsg_device.cuh"

#include <cuda.h>

namespace ecsg {

constexpr long long kWaitLimit = 1LL << 24;   // polls of an mbarrier before giving up

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned a, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(a), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(unsigned a, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(a), "r"(bytes) : "memory");
}
__device__ __forceinline__ void mbar_arrive(unsigned a)
{
    asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(a) : "memory");
}
__device__ __forceinline__ bool mbar_test(unsigned a, unsigned parity)
{
    unsigned ok;
    asm volatile("{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}"
                 : "=r"(ok)
                 : "r"(a), "r"(parity)
                 : "memory");
    return ok != 0;
}
// bounded wait; false after kWaitLimit polls
__device__ __forceinline__ bool mbar_wait(unsigned a, unsigned parity)
{
    for (long long i = 0; i < kWaitLimit; i++) {
        if (mbar_test(a, parity)) return true;
        if (i > 64) __nanosleep(64);
    }
    return false;
}
// one box of every field of a group: coordinates (x, y, z, first field)
__device__ __forceinline__ void tma_load4(unsigned dst, const CUtensorMap *map, int x, int y, int z, unsigned bar)
{
    asm volatile("cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes [%0], [%1, {%2, %3, %4, %5}], [%6];"
                 ::"r"(dst), "l"((unsigned long long)map), "r"(x), "r"(y), "r"(z), "r"(0), "r"(bar)
                 : "memory");
}

// ---------------------------------------------------------------------------
// Host: 4-D tensor maps (x, y, z, field) over fields of one grid box
// ---------------------------------------------------------------------------
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                  const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                  CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

inline EncodeTiledFn encode_fn()
{
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPointByVersion("cuTensorMapEncodeTiled", &p, 12000, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = (EncodeTiledFn)p;
    }
    return fn;
}

// 4-D map over `count` fields of one group: base = the group's first field,
// the others at a stride of one field box.
inline bool encode(CUtensorMap *m, const Geo &g, const void *base, int count, int bw, int bh)
{
    EncodeTiledFn fn = encode_fn();
    if (!fn || !base) return false;
    const cuuint64_t dims[4] = {(cuuint64_t)g.px, (cuuint64_t)g.py, (cuuint64_t)g.pz, (cuuint64_t)count};
    const cuuint64_t strides[3] = {(cuuint64_t)g.px * 4, (cuuint64_t)g.px * g.py * 4, (cuuint64_t)g.size() * 4};
    const cuuint32_t box[4] = {(cuuint32_t)bw, (cuuint32_t)bh, 1, (cuuint32_t)count};
    const cuuint32_t es[4] = {1, 1, 1, 1};
    return fn(m, CU_TENSOR_MAP_DATA_TYPE_FLOAT32, 4, const_cast<void *>(base), dims, strides, box, es,
              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}


} // namespace ecsg
