/*
 * wc_gen.cu -- on-device input generators (the reference's
 * random_distributions.cuh:50-326: uniform, unique and Zipf), as
 * counter-based kernels: element i depends only on (seed, i), so every
 * kernel is one coalesced, grid-stride pass and the result does not depend
 * on the launch shape.  The reference draws from kiss_rng (an absent,
 * unpinned dependency); these use splitmix64, whose i-th output is a mix of
 * seed + (i + 1) * golden ratio, and MurmurHash3's fmix, a bijection.
 *
 * - uniform: splitmix64 output i (its low 4 bytes for 32-bit elements).
 * - unique: fmix of (j + seed * golden) over the key width, j = i with the
 *   two indices skipped whose image is a sentinel.  The reference rejects
 *   Bloom-filter positives instead (random_distributions.cuh:144-194); a
 *   bijection needs no filter and no second draw.
 * - zipf: the rejection sampler of random_distributions.cuh:285-310, each
 *   output drawing from its own splitmix64 stream; 1-based ranks, or
 *   in[rank - 1] when an input array is given.
 */
#include <warpcore_b200.h>

#include "wc_internal.h"

#include <cmath>

using namespace warpcore::b200;

namespace {

constexpr int kBlock = 256;
constexpr uint64_t kGolden = 0x9e3779b97f4a7c15ull;

__host__ __device__ __forceinline__ uint64_t splitmix_mix(uint64_t z)
{
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

/* splitmix64 output i of a stream seeded with `seed` */
__host__ __device__ __forceinline__ uint64_t splitmix_at(uint64_t seed, uint64_t i)
{
    return splitmix_mix(seed + (i + 1) * kGolden);
}

template <class T>
__global__ void __launch_bounds__(kBlock) gen_uniform_kernel(T *out, uint64_t n, uint64_t seed)
{
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        out[i] = T(splitmix_at(seed, i));
}

/* skip[0] <= skip[1]: the indices whose key would be a sentinel */
template <class T>
__global__ void __launch_bounds__(kBlock) gen_unique_kernel(T *out, uint64_t n, uint64_t offset,
                                                             uint64_t skip0, uint64_t skip1)
{
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        uint64_t j = i;
        if (j >= skip0) ++j;
        if (j >= skip1) ++j;
        if constexpr (sizeof(T) == 4)
            out[i] = T(fmix32(uint32_t(j + offset)));
        else
            out[i] = T(fmix64(j + offset));
    }
}

/* u01 from the top 53 bits */
__device__ __forceinline__ double gen_u01(uint64_t x)
{
    return double(x >> 11) * (1.0 / 9007199254740992.0);
}

template <class T>
__global__ void __launch_bounds__(kBlock) gen_zipf_kernel(const T *in, uint64_t n_in, T *out,
                                                           uint64_t n_out, double s, double t,
                                                           uint64_t seed)
{
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n_out; i += stride) {
        /* output i's own stream: splitmix64 seeded with a mix of (seed, i) */
        const uint64_t st = splitmix_mix(seed ^ (i * kGolden + 0x632be59bd9b4e019ull));
        uint64_t draw = 0, k = 1;
        for (;;) {
            const double p = gen_u01(splitmix_at(st, draw++));
            const double pt = p * t;
            const double inv_b = pt <= 1.0 ? pt : pow(pt * (1.0 - s) + s, 1.0 / (1.0 - s));
            k = uint64_t(inv_b + 1.0);
            const double y = gen_u01(splitmix_at(st, draw++));
            const double b = k <= 1 ? 1.0 / t : pow(inv_b, -s) / t;
            const double rat = pow(double(k), -s) / (b * t);
            if (y < rat || draw >= 1u << 20) break; /* bounded: acceptance is about 1/2 per draw */
        }
        if (k > n_in) k = n_in;
        if (k < 1) k = 1;
        out[i] = in ? in[k - 1] : T(k);
    }
}

int gen_fail(int code, const char *msg) { return host_fail(code, msg); }

#define GEN_CUDA(call)                                                         \
    do {                                                                       \
        cudaError_t e_ = (call);                                               \
        if (e_ != cudaSuccess) return host_cuda_fail(e_, #call);               \
    } while (0)

/* inverse of x * c modulo 2^64 (c odd), by Newton's iteration */
uint64_t inv_mul64(uint64_t c)
{
    uint64_t x = c; /* correct to 3 bits */
    for (int i = 0; i < 5; ++i) x *= 2 - c * x;
    return x;
}

/* inverse of x ^= x >> r on w-bit words */
uint64_t unxorshift(uint64_t y, int r, int w)
{
    const uint64_t mask = w == 64 ? ~0ull : ((1ull << w) - 1);
    uint64_t x = y;
    for (int s = r; s < w; s += r) x = y ^ (x >> r);
    return x & mask;
}

/* preimage of `key` under MurmurHash3's fmix32 / fmix64 (both bijections) */
uint64_t fmix_inverse(uint64_t key, int bits)
{
    if (bits == 32) {
        uint64_t x = key & 0xffffffffull;
        x = unxorshift(x, 16, 32);
        x = (x * (inv_mul64(0xc2b2ae35ull) & 0xffffffffull)) & 0xffffffffull;
        x = unxorshift(x, 13, 32);
        x = (x * (inv_mul64(0x85ebca6bull) & 0xffffffffull)) & 0xffffffffull;
        return unxorshift(x, 16, 32);
    }
    uint64_t x = key;
    x = unxorshift(x, 33, 64);
    x *= inv_mul64(0xc4ceb9fe1a85ec53ull);
    x = unxorshift(x, 33, 64);
    x *= inv_mul64(0xff51afd7ed558ccdull);
    return unxorshift(x, 33, 64);
}

unsigned grid_of(const void *k, uint64_t n) { return host_grid(k, kBlock, n, kBlock); }

} // namespace

extern "C" {

int wc_gen_uniform(void *out, uint64_t n, uint32_t bytes, uint64_t seed, wc_stream_t stream)
{
    if (bytes != 4 && bytes != 8) return gen_fail(WC_ERR_UNSUPPORTED, "bytes must be 4 or 8");
    if (n == 0) return WC_OK;
    if (!out) return gen_fail(WC_ERR_INVALID_ARGUMENT, "out is NULL");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (bytes == 4) {
        const void *k = reinterpret_cast<const void *>(gen_uniform_kernel<uint32_t>);
        gen_uniform_kernel<uint32_t><<<grid_of(k, n), kBlock, 0, s>>>(static_cast<uint32_t *>(out), n, seed);
    } else {
        const void *k = reinterpret_cast<const void *>(gen_uniform_kernel<unsigned long long>);
        gen_uniform_kernel<unsigned long long><<<grid_of(k, n), kBlock, 0, s>>>(
            static_cast<unsigned long long *>(out), n, seed);
    }
    GEN_CUDA(cudaGetLastError());
    note_launches(1);
    return WC_OK;
}

int wc_gen_unique(void *out, uint64_t n, uint32_t key_bytes, uint64_t seed, wc_stream_t stream)
{
    if (key_bytes != 4 && key_bytes != 8) return gen_fail(WC_ERR_UNSUPPORTED, "key_bytes must be 4 or 8");
    if (key_bytes == 4 && n > 0xfffffffeull)
        return gen_fail(WC_ERR_INVALID_ARGUMENT, "at most 2^32 - 2 distinct 32-bit keys");
    if (n == 0) return WC_OK;
    if (!out) return gen_fail(WC_ERR_INVALID_ARGUMENT, "out is NULL");
    const int bits = key_bytes * 8;
    const uint64_t mask = bits == 32 ? 0xffffffffull : ~0ull;
    const uint64_t offset = (seed * kGolden) & mask;
    /* the sequence index of each sentinel's preimage */
    uint64_t s0 = (fmix_inverse(0, bits) - offset) & mask;
    uint64_t s1 = (fmix_inverse(mask, bits) - offset) & mask;
    if (s0 > s1) {
        const uint64_t x = s0;
        s0 = s1;
        s1 = x;
    }
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (key_bytes == 4) {
        const void *k = reinterpret_cast<const void *>(gen_unique_kernel<uint32_t>);
        gen_unique_kernel<uint32_t><<<grid_of(k, n), kBlock, 0, s>>>(static_cast<uint32_t *>(out), n,
                                                                     offset, s0, s1);
    } else {
        const void *k = reinterpret_cast<const void *>(gen_unique_kernel<unsigned long long>);
        gen_unique_kernel<unsigned long long><<<grid_of(k, n), kBlock, 0, s>>>(
            static_cast<unsigned long long *>(out), n, offset, s0, s1);
    }
    GEN_CUDA(cudaGetLastError());
    note_launches(1);
    return WC_OK;
}

int wc_gen_zipf(const void *in, uint64_t n_in, void *out, uint64_t n_out, uint32_t bytes,
                double s, uint64_t seed, wc_stream_t stream)
{
    if (bytes != 4 && bytes != 8) return gen_fail(WC_ERR_UNSUPPORTED, "bytes must be 4 or 8");
    if (n_in == 0) return gen_fail(WC_ERR_INVALID_ARGUMENT, "n_in must be at least 1");
    if (!(s > 0.0) || s == 1.0 || std::isnan(s))
        return gen_fail(WC_ERR_INVALID_ARGUMENT, "the skew must be positive and not 1");
    if (n_out == 0) return WC_OK;
    if (!out) return gen_fail(WC_ERR_INVALID_ARGUMENT, "out is NULL");
    const double t = (std::pow(double(n_in), 1.0 - s) - s) / (1.0 - s);
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    if (bytes == 4) {
        const void *k = reinterpret_cast<const void *>(gen_zipf_kernel<uint32_t>);
        gen_zipf_kernel<uint32_t><<<grid_of(k, n_out), kBlock, 0, st>>>(
            static_cast<const uint32_t *>(in), n_in, static_cast<uint32_t *>(out), n_out, s, t, seed);
    } else {
        const void *k = reinterpret_cast<const void *>(gen_zipf_kernel<unsigned long long>);
        gen_zipf_kernel<unsigned long long><<<grid_of(k, n_out), kBlock, 0, st>>>(
            static_cast<const unsigned long long *>(in), n_in, static_cast<unsigned long long *>(out),
            n_out, s, t, seed);
    }
    GEN_CUDA(cudaGetLastError());
    note_launches(1);
    return WC_OK;
}

} // extern "C"
