/*
 * Stand-in for the names warpcore takes from the hpc_helpers project, which
 * is not vendored with the reference and cannot be fetched offline.  Written
 * from the names the reference headers use (macros, helpers::lambda_kernel,
 * global_thread_id, atomicAggInc, available_gpu_memory, device ffs and the
 * unsigned long atomics).  Used only to compile the reference for golden
 * vectors and for the reference GPU timing; it is copied into oracle/_ref/.
 */
#ifndef WC_REF_CUDA_HELPERS_STANDIN
#define WC_REF_CUDA_HELPERS_STANDIN

#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <cuda_runtime.h>
#include <cooperative_groups.h>

#define HOSTQUALIFIER __host__
#define DEVICEQUALIFIER __device__
#define HOSTDEVICEQUALIFIER __host__ __device__
#define INLINEQUALIFIER inline
#define GLOBALQUALIFIER __global__
#ifndef MAXBLOCKSIZE
#define MAXBLOCKSIZE 1024
#endif
#define SDIV(x, y) (((x) + (y) - 1) / (y))
#define H2D (cudaMemcpyHostToDevice)
#define D2H (cudaMemcpyDeviceToHost)
#define D2D (cudaMemcpyDeviceToDevice)
#define CUERR                                                                  \
    {                                                                          \
        cudaError_t e_ = cudaGetLastError();                                   \
        if (e_ != cudaSuccess) {                                               \
            std::fprintf(stderr, "CUDA error: %s (%s:%d)\n",                   \
                         cudaGetErrorString(e_), __FILE__, __LINE__);          \
            std::exit(1);                                                      \
        }                                                                      \
    }

namespace helpers {

template <class F>
__global__ void lambda_kernel(F f) { f(); }

__device__ __forceinline__ std::uint64_t global_thread_id()
{
    return std::uint64_t(blockDim.x) * std::uint64_t(blockIdx.x) + threadIdx.x;
}

/* warp-aggregated increment: one atomicAdd per set of converged lanes */
template <class T>
__device__ __forceinline__ T atomicAggInc(T *ctr)
{
    namespace cg = cooperative_groups;
    auto g = cg::coalesced_threads();
    T base = 0;
    if (g.thread_rank() == 0)
        base = atomicAdd((unsigned long long *)ctr, (unsigned long long)g.size());
    return g.shfl(base, 0) + g.thread_rank();
}

inline std::size_t available_gpu_memory()
{
    std::size_t free_b = 0, total_b = 0;
    cudaMemGetInfo(&free_b, &total_b);
    return free_b;
}

} // namespace helpers

__device__ __forceinline__ int ffs(unsigned int x) { return __ffs(int(x)); }

__device__ __forceinline__ unsigned long atomicCAS(unsigned long *a,
                                                   unsigned long c,
                                                   unsigned long v)
{
    return (unsigned long)atomicCAS((unsigned long long *)a,
                                    (unsigned long long)c,
                                    (unsigned long long)v);
}
__device__ __forceinline__ unsigned long atomicAdd(unsigned long *a,
                                                   unsigned long v)
{
    return (unsigned long)atomicAdd((unsigned long long *)a,
                                    (unsigned long long)v);
}
__device__ __forceinline__ unsigned long atomicExch(unsigned long *a,
                                                    unsigned long v)
{
    return (unsigned long)atomicExch((unsigned long long *)a,
                                     (unsigned long long)v);
}
__device__ __forceinline__ unsigned long atomicOr(unsigned long *a,
                                                  unsigned long v)
{
    return (unsigned long)atomicOr((unsigned long long *)a,
                                   (unsigned long long)v);
}

#endif
