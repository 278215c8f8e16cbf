/*
 * wc_noalloc.cu -- wc_slots_size_noalloc: counts the occupied slots of a slot
 * array without allocating any device memory.
 *
 * Who needs it: a caller that holds a table's slot array but did not create
 * the table through this library, so it has no handle and none of the small
 * device scratch a handle carries, and that may not allocate device memory
 * itself.  Examples: a process that received the table's memory from another
 * process through CUDA IPC, or a plugin whose host framework owns every device
 * allocation through its own pool and refuses direct cudaMalloc calls.
 *
 * How: the count is computed in two kernels.  The first writes one partial
 * count per chunk of kChunkSlots slots into a scratch array that is compiled
 * into this library (a file-scope __device__ array, so every GPU that loads
 * the library holds it until the process exits); the second sums the
 * partials into the caller's output.  Every partial that the second kernel
 * reads was written by the first kernel of the same call, so nothing has to
 * be cleared between calls.  All calls share the one array: calls whose
 * kernels overlap on the GPU (two streams, or two host threads) race on it
 * and must be serialised by the caller.
 *
 * Every call resolves the array's device address with cudaGetSymbolAddress
 * in the current device's context (the first call on a device also loads the
 * module there); make the first call on each device before any stream
 * capture.
 */
#include <warpcore_b200.h>

#include "wc_internal.h"

#include <string>

using namespace warpcore::b200;

namespace {

constexpr uint64_t kChunkSlots = 1ull << 18;
constexpr uint64_t kMaxChunks = WC_NOALLOC_MAX_SLOTS / kChunkSlots; /* 65536 */

/* 512 KiB of partial counts, one per chunk */
static __device__ __align__(256) unsigned long long g_noalloc_partials[kMaxChunks];

int noalloc_fail(int code, const std::string &msg)
{
    set_last_error(msg.c_str());
    return code;
}

/* count of chunk blockIdx.x: slots [c * kChunkSlots, min(+kChunkSlots, cap)) */
template <class L>
__global__ void __launch_bounds__(256) count_chunk_kernel(const void *slots, uint64_t capacity,
                                                          uint64_t empty, uint64_t tomb,
                                                          unsigned long long *partials)
{
    using K = typename L::key_t;
    constexpr int SB = L::kSlotBytes;
    constexpr int SPV = 16 / SB; /* slots per 16-byte vector */
    const uint64_t first = uint64_t(blockIdx.x) * kChunkSlots;
    const uint64_t last = first + kChunkSlots < capacity ? first + kChunkSlots : capacity;
    const unsigned char *base = reinterpret_cast<const unsigned char *>(slots) + first * SB;
    const uint64_t nvec = (last - first) / SPV;
    unsigned long long c = 0;
    for (uint64_t v = threadIdx.x; v < nvec; v += blockDim.x) {
        const LaneWords lw = load_lane<16>(base + v * 16);
#pragma unroll
        for (int s = 0; s < SPV; ++s) {
            const K k = slot_key<L>(lw, s);
            c += (k != K(empty) && k != K(tomb));
        }
    }
    const uint64_t rem = (last - first) % SPV;
    if (threadIdx.x < rem) {
        const K k = *reinterpret_cast<const K *>(base + (nvec * SPV + threadIdx.x) * SB);
        c += (k != K(empty) && k != K(tomb));
    }
    c = __reduce_add_sync(kFull, unsigned(c));
    __shared__ unsigned long long sm[8];
    if ((threadIdx.x & 31) == 0) sm[threadIdx.x >> 5] = c;
    __syncthreads();
    if (threadIdx.x == 0) {
        unsigned long long s = 0;
        for (int w = 0; w < int(blockDim.x >> 5); ++w) s += sm[w];
        partials[blockIdx.x] = s;
    }
}

__global__ void __launch_bounds__(256) sum_partials_kernel(const unsigned long long *partials,
                                                           uint64_t n, unsigned long long *out)
{
    unsigned long long s = 0;
    for (uint64_t i = threadIdx.x; i < n; i += blockDim.x) s += partials[i];
    __shared__ unsigned long long sm[256];
    sm[threadIdx.x] = s;
    __syncthreads();
    for (int w = 128; w > 0; w >>= 1) {
        if (int(threadIdx.x) < w) sm[threadIdx.x] += sm[threadIdx.x + w];
        __syncthreads();
    }
    if (threadIdx.x == 0) *out = sm[0];
}

/* Device address of the scratch array in the current device's context.  It
 * is looked up on every call (a lookup allocates nothing): a cached address
 * would go stale when the context it came from is destroyed and the module
 * is loaded again, e.g. after cudaDeviceReset. */
int scratch_address(unsigned long long **out)
{
    void *p = nullptr;
    const cudaError_t e = cudaGetSymbolAddress(&p, g_noalloc_partials);
    if (e != cudaSuccess || p == nullptr)
        return noalloc_fail(WC_ERR_CUDA,
                            std::string("cudaGetSymbolAddress: ") + cudaGetErrorString(e));
    *out = reinterpret_cast<unsigned long long *>(p);
    return WC_OK;
}

template <class L>
int launch_count(const void *slots, uint64_t capacity, uint64_t empty, uint64_t tomb,
                 cudaStream_t s, unsigned long long *partials, unsigned long long *out)
{
    const uint64_t nchunks = (capacity + kChunkSlots - 1) / kChunkSlots;
    if (nchunks)
        count_chunk_kernel<L><<<unsigned(nchunks), 256, 0, s>>>(slots, capacity, empty, tomb,
                                                               partials);
    sum_partials_kernel<<<1, 256, 0, s>>>(partials, nchunks, out);
    note_launches(nchunks ? 2u : 1u);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess)
        return noalloc_fail(WC_ERR_CUDA, std::string("kernel launch: ") + cudaGetErrorString(e));
    return WC_OK;
}

} // namespace

extern "C" int wc_slots_size_noalloc(const void *slots, uint64_t capacity, uint32_t key_bytes,
                                     uint32_t value_bytes, uint64_t empty_key,
                                     uint64_t tombstone_key, wc_stream_t stream,
                                     uint64_t *size_out)
{
    if (!size_out) return noalloc_fail(WC_ERR_INVALID_ARGUMENT, "size_out is NULL");
    if (key_bytes != 4 && key_bytes != 8)
        return noalloc_fail(WC_ERR_UNSUPPORTED, "key_bytes must be 4 or 8");
    if (value_bytes != 0 && value_bytes != key_bytes)
        return noalloc_fail(WC_ERR_UNSUPPORTED, "value_bytes must be 0 or equal key_bytes");
    if (capacity > WC_NOALLOC_MAX_SLOTS)
        return noalloc_fail(WC_ERR_INVALID_ARGUMENT,
                            "capacity " + std::to_string(capacity) +
                                " exceeds the no-alloc scratch limit of 2^34 slots");
    if (capacity && (!slots || (reinterpret_cast<uintptr_t>(slots) & 15)))
        return noalloc_fail(WC_ERR_INVALID_ARGUMENT, "slots must be a 16-byte aligned device pointer");
    unsigned long long *partials = nullptr;
    int rc = scratch_address(&partials);
    if (rc) return rc;
    const uint64_t km = key_bytes == 4 ? 0xffffffffull : ~0ull;
    const uint64_t e = empty_key & km, t = tombstone_key & km;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    unsigned long long *out = reinterpret_cast<unsigned long long *>(size_out);
    if (value_bytes == 0)
        return key_bytes == 4 ? launch_count<LayoutSet32>(slots, capacity, e, t, s, partials, out)
                              : launch_count<LayoutSet64>(slots, capacity, e, t, s, partials, out);
    return key_bytes == 4 ? launch_count<LayoutKV32>(slots, capacity, e, t, s, partials, out)
                          : launch_count<LayoutKV64>(slots, capacity, e, t, s, partials, out);
}
