// Tensor-memory-accelerator plumbing shared by the tiled kernels: mbarrier
// operations with bounded waits, the 3-D bulk tensor load into shared memory,
// the tensor-map encoder (through the driver entry point, no link against
// libcuda) and the one-time opening of a kernel's dynamic shared memory.
// Every copy here targets this GPU's own memory and none uses cluster
// multicast.
#pragma once
#include <cuda.h>
#include <cudaTypedefs.h>

#include <utility>

#include "hevi_common.cuh"

namespace hevi {
namespace tma {

constexpr long long WAIT_CYCLES = 4000000000LL; // ~2 s: bound of every mbarrier wait

__device__ __forceinline__ unsigned smem_u32(const void *p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, unsigned count)
{
    asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, unsigned bytes)
{
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes)
                 : "memory");
}
// one test of the phase with the given parity; true once it has completed
__device__ __forceinline__ bool mbar_try(uint64_t *bar, unsigned parity)
{
    unsigned done;
    asm volatile("{\n\t.reg .pred p;\n\t"
                 "mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n\t"
                 "selp.u32 %0, 1, 0, p;\n\t}"
                 : "=r"(done)
                 : "r"(smem_u32(bar)), "r"(parity)
                 : "memory");
    return done != 0;
}
// bounded wait: gives up after about WAIT_CYCLES clocks
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, unsigned parity)
{
    const long long t0 = clock64();
    while (!mbar_try(bar, parity))
        if (clock64() - t0 > WAIT_CYCLES) return false;
    return true;
}
__device__ __forceinline__ void tma_load_3d(void *dst, const CUtensorMap *map, int x, int y, int z, uint64_t *bar)
{
    asm volatile("cp.async.bulk.tensor.3d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
                 " [%0], [%1, {%2, %3, %4}], [%5];" ::"r"(smem_u32(dst)),
                 "l"(reinterpret_cast<uint64_t>(map)), "r"(x), "r"(y), "r"(z), "r"(smem_u32(bar))
                 : "memory");
}
// orders this thread's earlier generic-proxy accesses of shared memory before
// a following bulk copy into it
__device__ __forceinline__ void fence_proxy_async() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

static inline PFN_cuTensorMapEncodeTiled_v12000 encode_fn()
{
    static PFN_cuTensorMapEncodeTiled_v12000 fn = nullptr;
    static bool tried = false;
    if (!tried) {
        tried = true;
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q{};
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<PFN_cuTensorMapEncodeTiled_v12000>(p);
    }
    return fn;
}

// FP64 or FP32 (KA, IA, JA) tensor with a box of bk x bw x bh elements; false
// unless the base address and the strides are multiples of 16 bytes
template <typename T>
static bool encode(CUtensorMap *m, const T *base, const Grid &g, int bk, int bw, int bh)
{
    auto fn = encode_fn();
    const size_t sk = (size_t)g.KA * sizeof(T), sj = (size_t)g.KA * g.IA * sizeof(T);
    if (!fn || ((uintptr_t)base & 15u) || (sk & 15u) || (sj & 15u) || ((size_t)bk * sizeof(T)) % 16u) return false;
    const cuuint64_t dims[3] = {(cuuint64_t)g.KA, (cuuint64_t)g.IA, (cuuint64_t)g.JA};
    const cuuint64_t strides[2] = {(cuuint64_t)sk, (cuuint64_t)sj};
    const cuuint32_t box[3] = {(cuuint32_t)bk, (cuuint32_t)bw, (cuuint32_t)bh};
    const cuuint32_t estr[3] = {1, 1, 1};
    const CUtensorMapDataType dt = sizeof(T) == 8 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT64 : CU_TENSOR_MAP_DATA_TYPE_FLOAT32;
    return fn(m, dt, 3, const_cast<T *>(base), dims, strides, box, estr, CU_TENSOR_MAP_INTERLEAVE_NONE,
              CU_TENSOR_MAP_SWIZZLE_NONE, CU_TENSOR_MAP_L2_PROMOTION_L2_256B,
              CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) == CUDA_SUCCESS;
}

// opens the dynamic shared memory of a kernel instantiation, once per device
template <class K>
cudaError_t open_smem(K kern, size_t bytes)
{
    static std::pair<const void *, int> done[64];
    static int ndone = 0;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    for (int q = 0; q < ndone; ++q)
        if (done[q].first == (const void *)kern && done[q].second == dev) return cudaSuccess;
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    if (e == cudaSuccess && ndone < 64) done[ndone++] = {(const void *)kern, dev};
    return e;
}

}  // namespace tma
}  // namespace hevi
