/*
 * wc_partition.cu -- routes keys to the rank that owns them, for tables
 * sharded over several GPUs (the reference is single-GPU; this is the
 * exchange step of the sharded form).
 *
 * owner(key) = (hi32(fmix64(key ^ salt)) * parts) >> 32: a multiply-shift
 * range reduction of a mix that is independent of the probing hashers, so
 * every shard sees a uniform sample of the key space.  The keys (and values)
 * are grouped by owner with a counting sort: a count pass, an exclusive
 * scan, and a scatter pass; within an owner the order is unspecified, and
 * perm_out[j] names the input position of output j so that answers can be
 * put back.  Atomics are aggregated per warp over lanes with equal owners.
 * Every output position is checked against n; a key that fails the check
 * (possible only if the keys change between the count and scatter passes)
 * is dropped and counted in the error word, so the call cannot write out of
 * bounds.
 *
 * A sharded Bloom filter routes by its own block instead: shard s holds the
 * blocks b with b * parts / num_blocks == s (wc_bloom_partition), so that a
 * key's bits all live on one shard.  The kernels take the owner as a
 * functor and are otherwise the same.
 */
#include <warpcore_b200.h>

#include "wc_internal.h"

namespace warpcore {
namespace b200 {

__host__ __device__ __forceinline__ uint32_t partition_owner(uint64_t key, uint64_t salt,
                                                             uint32_t parts)
{
    const uint64_t h = fmix64(key ^ salt);
    return uint32_t(((h >> 32) * uint64_t(parts)) >> 32);
}

struct SaltOwner {
    uint64_t salt;
    uint32_t parts;
    template <class K>
    __device__ __forceinline__ uint32_t operator()(K key) const
    {
        return partition_owner(uint64_t(key), salt, parts);
    }
};

/* the shard holding the key's block of a filter of num_blocks blocks: the
 * block index as the Bloom kernels compute it, then a range split */
struct BlockOwner {
    uint64_t seed, num_blocks, magic;
    uint32_t hasher, parts;
    template <class K>
    __device__ __forceinline__ uint32_t operator()(K key) const
    {
        const uint64_t blk = fast_mod(hash_key<K>(hasher, K(key + seed)), num_blocks, magic);
        return uint32_t(blk * parts / num_blocks);
    }
};

/* Both passes walk tiles of kTile = 256 x kKeysPerThread keys; a thread
 * holds key j of its tile at t0 + j * 256 + threadIdx.x, so every load and
 * every store of one j is coalesced, and each thread has kKeysPerThread
 * independent loads in flight. */
constexpr int kPartThreads = 256;
constexpr int kKeysPerThread = 8;
constexpr uint64_t kTile = uint64_t(kPartThreads) * kKeysPerThread;

/* warp-aggregated shared-memory increment of hist[owner] by the lanes that
 * share `owner`; returns this lane's rank among them, offset by the old
 * count.  owner >= parts (inactive lanes) takes no part. */
__device__ __forceinline__ unsigned tile_rank(unsigned int *hist, uint32_t owner, uint32_t parts)
{
    const int lane = threadIdx.x & 31;
    const unsigned peers = __match_any_sync(kFull, owner);
    const int leader = __ffs(peers) - 1;
    unsigned base = 0;
    if (owner < parts && lane == leader) base = atomicAdd(&hist[owner], unsigned(__popc(peers)));
    base = __shfl_sync(kFull, base, leader);
    return base + unsigned(__popc(peers & ((1u << lane) - 1u)));
}

template <class K, class Owner>
__global__ void __launch_bounds__(kPartThreads) partition_count_kernel(const K *keys, uint64_t n,
                                                                       uint32_t parts, Owner owner_of,
                                                                       unsigned long long *counts)
{
    /* The owner is held in a range-checked local and the increments are
     * aggregated per warp.  Written instead as one atomicAdd on
     * hist[partition_owner(...)], this kernel counted every key in hist[0]
     * on sm_100a (CUDA 12.9); the GPU test with one repeated key whose owner
     * is not 0 guards against that. */
    __shared__ unsigned int hist[WC_PARTITION_MAX_PARTS];
    for (uint32_t p = threadIdx.x; p < parts; p += blockDim.x) hist[p] = 0;
    __syncthreads();
    const uint64_t ntiles = (n + kTile - 1) / kTile;
    for (uint64_t tb = blockIdx.x; tb < ntiles; tb += gridDim.x) {
        const uint64_t t0 = tb * kTile;
        K k[kKeysPerThread];
#pragma unroll
        for (int j = 0; j < kKeysPerThread; ++j) {
            const uint64_t i = t0 + uint64_t(j) * kPartThreads + threadIdx.x;
            k[j] = i < n ? keys[i] : K(0);
        }
#pragma unroll
        for (int j = 0; j < kKeysPerThread; ++j) {
            const uint64_t i = t0 + uint64_t(j) * kPartThreads + threadIdx.x;
            const uint32_t owner = i < n ? owner_of(k[j]) : 0xFFFFFFFFu;
            tile_rank(hist, owner, parts);
        }
    }
    __syncthreads();
    for (uint32_t p = threadIdx.x; p < parts; p += blockDim.x)
        if (hist[p]) atomicAdd(&counts[p], (unsigned long long)hist[p]);
}

__global__ void partition_scan_kernel(const unsigned long long *counts, uint32_t parts,
                                      unsigned long long *offsets, unsigned long long *cursors,
                                      unsigned long long *dropped)
{
    /* parts <= 1024: one thread does the exclusive scan */
    if (threadIdx.x == 0) {
        unsigned long long s = 0;
        for (uint32_t p = 0; p < parts; ++p) {
            offsets[p] = s;
            s += counts[p];
        }
    }
    for (uint32_t p = threadIdx.x; p < parts; p += blockDim.x) cursors[p] = 0;
    if (threadIdx.x == 0) *dropped = 0;
}

/* A tile ranks its keys per owner in shared memory, then claims one range
 * per owner with a single global atomicAdd on that owner's cursor; the
 * keys of one owner in a tile land in consecutive positions. */
template <class K, class V, class Owner>
__global__ void __launch_bounds__(kPartThreads) partition_scatter_kernel(
    const K *keys, const V *values, uint64_t n, uint32_t parts, Owner owner_of,
    const unsigned long long *offsets, unsigned long long *cursors, K *keys_out, V *values_out,
    unsigned long long *perm_out, unsigned long long *dropped)
{
    __shared__ unsigned int tile_cnt[WC_PARTITION_MAX_PARTS];
    __shared__ unsigned long long tile_base[WC_PARTITION_MAX_PARTS];
    const uint64_t ntiles = (n + kTile - 1) / kTile;
    for (uint64_t tb = blockIdx.x; tb < ntiles; tb += gridDim.x) {
        for (uint32_t p = threadIdx.x; p < parts; p += blockDim.x) tile_cnt[p] = 0;
        __syncthreads();
        const uint64_t t0 = tb * kTile;
        K k[kKeysPerThread];
        uint32_t own[kKeysPerThread];
        unsigned rank[kKeysPerThread];
#pragma unroll
        for (int j = 0; j < kKeysPerThread; ++j) {
            const uint64_t i = t0 + uint64_t(j) * kPartThreads + threadIdx.x;
            k[j] = i < n ? keys[i] : K(0);
        }
#pragma unroll
        for (int j = 0; j < kKeysPerThread; ++j) {
            const uint64_t i = t0 + uint64_t(j) * kPartThreads + threadIdx.x;
            own[j] = i < n ? owner_of(k[j]) : 0xFFFFFFFFu;
            rank[j] = tile_rank(tile_cnt, own[j], parts);
        }
        __syncthreads();
        for (uint32_t p = threadIdx.x; p < parts; p += blockDim.x) {
            const unsigned c = tile_cnt[p];
            tile_base[p] = c ? atomicAdd(&cursors[p], (unsigned long long)c) : 0ull;
        }
        __syncthreads();
#pragma unroll
        for (int j = 0; j < kKeysPerThread; ++j) {
            const uint64_t i = t0 + uint64_t(j) * kPartThreads + threadIdx.x;
            if (own[j] < parts) {
                const uint64_t pos = offsets[own[j]] + tile_base[own[j]] + rank[j];
                if (pos < n) {
                    keys_out[pos] = k[j];
                    if (values) values_out[pos] = values[i];
                    perm_out[pos] = i;
                } else {
                    atomicAdd(dropped, 1ull);
                }
            }
        }
        __syncthreads(); /* tile_cnt / tile_base are reused by the next tile */
    }
}

/* the inverse step of a sharded retrieve: answer j (in owner order) goes
 * back to input position perm[j]; its value only on a hit (status 0), as
 * the reference's retrieve writes hits only, or always without statuses
 * (a Bloom filter's flags) */
template <class V>
__global__ void __launch_bounds__(256) partition_restore_kernel(
    const V *values, const uint32_t *status, const unsigned long long *perm, uint64_t n,
    V *values_out, uint32_t *status_out)
{
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t j = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; j < n; j += stride) {
        const unsigned long long p = perm[j];
        if (p >= n) continue; /* not a permutation of [0, n): nothing to write */
        const uint32_t st = status ? status[j] : 0u;
        if (st == 0) values_out[p] = values[j];
        if (status_out) status_out[p] = st;
    }
}

/* count, scan and scatter passes for one key width and owner function */
template <class K, class Owner>
int partition_launch(const void *keys, const void *values, uint64_t n, uint32_t num_parts,
                     Owner owner_of, void *keys_out, void *values_out, uint64_t *perm_out,
                     uint64_t *counts_out, uint64_t *scratch, cudaStream_t s)
{
    auto *counts = reinterpret_cast<unsigned long long *>(counts_out);
    auto *offsets = reinterpret_cast<unsigned long long *>(scratch);
    auto *cursors = offsets + num_parts;
    auto *dropped = cursors + num_parts;
    cudaError_t e = cudaMemsetAsync(counts, 0, sizeof(unsigned long long) * num_parts, s);
    if (e != cudaSuccess) return host_cuda_fail(e, "cudaMemsetAsync");
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
    const uint64_t need = (n + kTile - 1) / kTile; /* one block per tile, up to 4 per SM */
    const unsigned grid = unsigned(need < uint64_t(sms) * 4 ? (need ? need : 1) : uint64_t(sms) * 4);
    partition_count_kernel<K, Owner><<<grid, kPartThreads, 0, s>>>(
        reinterpret_cast<const K *>(keys), n, num_parts, owner_of, counts);
    if ((e = cudaGetLastError()) != cudaSuccess) return host_cuda_fail(e, "partition_count_kernel");
    partition_scan_kernel<<<1, 256, 0, s>>>(counts, num_parts, offsets, cursors, dropped);
    if ((e = cudaGetLastError()) != cudaSuccess) return host_cuda_fail(e, "partition_scan_kernel");
    partition_scatter_kernel<K, K, Owner><<<grid, kPartThreads, 0, s>>>(
        reinterpret_cast<const K *>(keys), reinterpret_cast<const K *>(values), n, num_parts,
        owner_of, offsets, cursors, reinterpret_cast<K *>(keys_out), reinterpret_cast<K *>(values_out),
        reinterpret_cast<unsigned long long *>(perm_out), dropped);
    if ((e = cudaGetLastError()) != cudaSuccess) return host_cuda_fail(e, "partition_scatter_kernel");
    note_launches(3);
    return WC_OK;
}

int partition_check(uint32_t key_bytes, uint32_t num_parts, const void *keys, const void *values,
                    uint64_t n, void *keys_out, void *values_out, uint64_t *perm_out,
                    uint64_t *counts_out, uint64_t *scratch)
{
    if (key_bytes != 4 && key_bytes != 8) return host_fail(WC_ERR_UNSUPPORTED, "key_bytes must be 4 or 8");
    if (num_parts == 0 || num_parts > WC_PARTITION_MAX_PARTS)
        return host_fail(WC_ERR_INVALID_ARGUMENT, "num_parts must be 1 .. WC_PARTITION_MAX_PARTS");
    if (!counts_out || !scratch || (n && (!keys || !keys_out || !perm_out || (values && !values_out))))
        return host_fail(WC_ERR_INVALID_ARGUMENT, "NULL buffer");
    return WC_OK;
}

} // namespace b200
} // namespace warpcore

using namespace warpcore::b200;

extern "C" int wc_partition(const void *keys, const void *values, uint64_t n, uint32_t key_bytes,
                            uint32_t value_bytes, uint32_t num_parts, uint64_t salt,
                            void *keys_out, void *values_out, uint64_t *perm_out,
                            uint64_t *counts_out, uint64_t *scratch, wc_stream_t stream)
{
    int rc = partition_check(key_bytes, num_parts, keys, values, n, keys_out, values_out, perm_out,
                             counts_out, scratch);
    if (rc) return rc;
    if (values && value_bytes != key_bytes)
        return host_fail(WC_ERR_UNSUPPORTED, "value_bytes must equal key_bytes");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const SaltOwner own{salt, num_parts};
    if (key_bytes == 4)
        return partition_launch<uint32_t>(keys, values, n, num_parts, own, keys_out, values_out,
                                          perm_out, counts_out, scratch, s);
    return partition_launch<unsigned long long>(keys, values, n, num_parts, own, keys_out,
                                                values_out, perm_out, counts_out, scratch, s);
}

int warpcore::b200::partition_by_bloom_block(const void *keys, uint64_t n, uint32_t key_bytes,
                                             uint32_t num_parts, uint64_t seed, uint32_t hasher,
                                             uint64_t num_blocks, void *keys_out,
                                             uint64_t *perm_out, uint64_t *counts_out,
                                             uint64_t *scratch, wc_stream_t stream)
{
    int rc = partition_check(key_bytes, num_parts, keys, nullptr, n, keys_out, nullptr, perm_out,
                             counts_out, scratch);
    if (rc) return rc;
    if (num_blocks == 0 || num_blocks > (~0ull) / WC_PARTITION_MAX_PARTS)
        return host_fail(WC_ERR_INVALID_ARGUMENT, "num_blocks out of range");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const BlockOwner own{seed, num_blocks, barrett_magic(num_blocks), hasher, num_parts};
    if (key_bytes == 4)
        return partition_launch<uint32_t>(keys, nullptr, n, num_parts, own, keys_out, nullptr,
                                          perm_out, counts_out, scratch, s);
    return partition_launch<unsigned long long>(keys, nullptr, n, num_parts, own, keys_out,
                                                nullptr, perm_out, counts_out, scratch, s);
}

extern "C" int wc_partition_restore(const void *values, const uint32_t *status,
                                    const uint64_t *perm, uint64_t n, uint32_t value_bytes,
                                    void *values_out, uint32_t *status_out, wc_stream_t stream)
{
    if (n == 0) return WC_OK;
    if (value_bytes != 1 && value_bytes != 4 && value_bytes != 8) {
        set_last_error("value_bytes must be 1, 4 or 8");
        return WC_ERR_UNSUPPORTED;
    }
    if (!values || !perm || !values_out) {
        set_last_error("NULL buffer");
        return WC_ERR_INVALID_ARGUMENT;
    }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, 0);
    const uint64_t need = (n + 255) / 256;
    const unsigned grid = unsigned(need < uint64_t(sms) * 8 ? need : uint64_t(sms) * 8);
    const auto *pp = reinterpret_cast<const unsigned long long *>(perm);
    if (value_bytes == 1)
        partition_restore_kernel<uint8_t><<<grid, 256, 0, s>>>(
            reinterpret_cast<const uint8_t *>(values), status, pp, n,
            reinterpret_cast<uint8_t *>(values_out), status_out);
    else if (value_bytes == 4)
        partition_restore_kernel<uint32_t><<<grid, 256, 0, s>>>(
            reinterpret_cast<const uint32_t *>(values), status, pp, n,
            reinterpret_cast<uint32_t *>(values_out), status_out);
    else
        partition_restore_kernel<unsigned long long><<<grid, 256, 0, s>>>(
            reinterpret_cast<const unsigned long long *>(values), status, pp, n,
            reinterpret_cast<unsigned long long *>(values_out), status_out);
    const cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) {
        set_last_error(cudaGetErrorString(e));
        return WC_ERR_CUDA;
    }
    note_launches(1);
    return WC_OK;
}
