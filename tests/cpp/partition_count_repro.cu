// Minimal reproduction of a miscount seen in the partition count kernel
// (warpcore_b200/csrc/wc_partition.cu).  Two shared-memory histograms of the
// same keys over `parts` owners, owner = ((hi32(fmix64(key ^ salt))) * parts)
// >> 32, which is always below parts (every index is in bounds):
//   count_direct: atomicAdd(&hist[partition_owner(key, salt, parts)], 1u);
//   count_local:  the owner held in a local, range-checked, then the add.
// Both are well-defined C++.  Built with nvcc 12.9 for sm_100a at -O3,
// count_direct counted every key in bin 0 on B200, count_local counted
// right; the library uses the local form.  The program prints one line per
// case and exits 0; tests/test_partition_repro_gpu.py builds and runs it and
// requires the local form to be right everywhere.
#include <cstdio>
#include <cstdint>
#include <vector>
#include <cuda_runtime.h>
__host__ __device__ __forceinline__ uint64_t fmix64(uint64_t k) {
    k ^= k >> 33; k *= 0xff51afd7ed558ccdull; k ^= k >> 33; k *= 0xc4ceb9fe1a85ec53ull; k ^= k >> 33; return k;
}
__host__ __device__ __forceinline__ uint32_t partition_owner(uint64_t key, uint64_t salt, uint32_t parts) {
    const uint64_t h = fmix64(key ^ salt);
    return uint32_t(((h >> 32) * uint64_t(parts)) >> 32);
}
constexpr int kMax = 1024;
template <class K>
__global__ void count_direct(const K *keys, uint64_t n, uint32_t parts, uint64_t salt, unsigned long long *counts) {
    __shared__ unsigned int hist[kMax];
    for (uint32_t p = threadIdx.x; p < parts; p += blockDim.x) hist[p] = 0;
    __syncthreads();
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride)
        atomicAdd(&hist[partition_owner(uint64_t(keys[i]), salt, parts)], 1u);
    __syncthreads();
    for (uint32_t p = threadIdx.x; p < parts; p += blockDim.x)
        if (hist[p]) atomicAdd(&counts[p], (unsigned long long)hist[p]);
}
template <class K>
__global__ void count_local(const K *keys, uint64_t n, uint32_t parts, uint64_t salt, unsigned long long *counts) {
    __shared__ unsigned int hist[kMax];
    for (uint32_t p = threadIdx.x; p < parts; p += blockDim.x) hist[p] = 0;
    __syncthreads();
    const uint64_t stride = uint64_t(gridDim.x) * blockDim.x;
    for (uint64_t i = uint64_t(blockIdx.x) * blockDim.x + threadIdx.x; i < n; i += stride) {
        const uint32_t owner = partition_owner(uint64_t(keys[i]), salt, parts);
        if (owner < parts) atomicAdd(&hist[owner], 1u);
    }
    __syncthreads();
    for (uint32_t p = threadIdx.x; p < parts; p += blockDim.x)
        if (hist[p]) atomicAdd(&counts[p], (unsigned long long)hist[p]);
}
template <class K>
int run(uint32_t parts, bool repeated) {
    const uint64_t n = 100000, salt = 0x1234567;
    std::vector<K> h(n);
    for (uint64_t i = 0; i < n; ++i) h[i] = K(repeated ? 0xdeadbeef12345ull : fmix64(i + 99));
    std::vector<unsigned long long> ref(parts, 0);
    for (uint64_t i = 0; i < n; ++i) ref[partition_owner(uint64_t(h[i]), salt, parts)]++;
    K *d; unsigned long long *c1, *c2;
    cudaMalloc(&d, n * sizeof(K)); cudaMalloc(&c1, parts * 8); cudaMalloc(&c2, parts * 8);
    cudaMemcpy(d, h.data(), n * sizeof(K), cudaMemcpyHostToDevice);
    cudaMemset(c1, 0, parts * 8); cudaMemset(c2, 0, parts * 8);
    count_direct<K><<<64, 256>>>(d, n, parts, salt, c1);
    count_local<K><<<64, 256>>>(d, n, parts, salt, c2);
    std::vector<unsigned long long> g1(parts), g2(parts);
    cudaMemcpy(g1.data(), c1, parts * 8, cudaMemcpyDeviceToHost);
    cudaMemcpy(g2.data(), c2, parts * 8, cudaMemcpyDeviceToHost);
    cudaFree(d); cudaFree(c1); cudaFree(c2);
    int bad1 = 0, bad2 = 0;
    for (uint32_t p = 0; p < parts; ++p) { bad1 += g1[p] != ref[p]; bad2 += g2[p] != ref[p]; }
    printf("{\"key_bytes\": %zu, \"parts\": %u, \"repeated\": %d, \"direct_bad_bins\": %d, \"local_bad_bins\": %d, \"bin0_direct\": %llu, \"bin0_ref\": %llu}\n",
           sizeof(K), parts, int(repeated), bad1, bad2, g1[0], ref[0]);
    return bad1 + bad2;
}
int main() {
    int bad = 0;
    for (uint32_t parts : {2u, 3u, 7u, 64u, 1024u})
        for (bool rep : {false, true}) { bad += run<uint64_t>(parts, rep); bad += run<uint32_t>(parts, rep); }
    cudaError_t e = cudaDeviceSynchronize();
    printf("rc %d bad %d\n", int(e), bad);
    return int(e);
}
