/*
 * wc_internal.h -- kernel registry shared by the translation units of
 * libwarpcore_b200.so (not a public header).
 */
#ifndef WC_INTERNAL_H
#define WC_INTERNAL_H

#include <warpcore_b200.h>

#include "wc_bloom.cuh"
#include "wc_batch.cuh"
#include "wc_fp_kernels.cuh"
#include "wc_lane_kernels.cuh"
#include "wc_mv.cuh"

namespace warpcore {
namespace b200 {

enum : int {
    kLayoutKV32 = 0,
    kLayoutKV64 = 1,
    kLayoutSet32 = 2,
    kLayoutSet64 = 3,
    kLayoutK32V64 = 4,
    kLayoutK64V32 = 5
};

using TableKernel = void (*)(TableOpArgs);
using BloomKernel = void (*)(BloomArgs);
using CountKernel = void (*)(const void *, uint64_t, uint64_t, uint64_t, unsigned long long *);
using DumpKernel = void (*)(const void *, uint64_t, uint64_t, uint64_t, void *, void *,
                            unsigned long long *);

/* kernel for (window width W, op); nullptr if the combination is not built */
TableKernel table_kernel_kv32(int W, int op, bool fingerprints);
TableKernel table_kernel_kv64(int W, int op, bool fingerprints);
TableKernel table_kernel_set32(int W, int op, bool fingerprints);
TableKernel table_kernel_set64(int W, int op, bool fingerprints);
TableKernel table_kernel_k32v64(int W, int op, bool fingerprints);
TableKernel table_kernel_k64v32(int W, int op, bool fingerprints);
/* the one-key-per-lane window kernel of (W, op), nullptr if not built */
TableKernel lane_kernel_kv32(int W, int op);
TableKernel lane_kernel_kv64(int W, int op);
TableKernel lane_kernel_set32(int W, int op);
TableKernel lane_kernel_set64(int W, int op);
TableKernel lane_kernel_k32v64(int W, int op);
TableKernel lane_kernel_k64v32(int W, int op);

/* struct-of-arrays single-value tables (wc_tables_soa.cu): the window
 * kernel of (key width, value width, W, op) for insert, retrieve and erase,
 * nullptr otherwise; and the dump of (key array, value array) */
TableKernel table_kernel_soa(uint32_t key_bytes, uint32_t value_bytes, int W, int op);
using SoaDumpKernel = void (*)(const void *, const void *, uint64_t, uint64_t, uint64_t, void *,
                               void *, unsigned long long *);
SoaDumpKernel soa_dump_kernel_ptr(uint32_t key_bytes, uint32_t value_bytes);

CountKernel count_kernel(int layout);
using RebuildKernel = void (*)(const void *, uint64_t, uint64_t, uint64_t, unsigned char *);
RebuildKernel fp_rebuild_kernel_ptr(int layout);
DumpKernel dump_kernel_ptr(int layout);

/* the Bloom kernel of a configuration; multi_pass selects the variant built
 * for region passes, *lane_kernel (if not null) tells whether the kernel is
 * the one-key-per-lane kernel, the only one that honours region bounds */
BloomKernel bloom_kernel_ptr(int key_bytes, int slot_bytes, int cg, bool insert, bool multi_pass,
                             bool *lane_kernel);

/* random-access region of the multi-pass kernels for inserts or queries
 * (bytes; wc_region_bytes) */
uint64_t region_bytes(bool insert);

/* multi-table batch kernel for a slot layout (KV32 / KV64) and window width;
 * inline_desc selects the variant taking BatchInlineArgs */
const void *batch_kernel_ptr(int layout, int W, bool inline_desc);

/* MultiValueHashTable kernels of a layout (KV32 / KV64) and window width;
 * null pointers if not built */
struct MvKernels {
    const void *insert = nullptr, *count = nullptr, *values = nullptr, *unique = nullptr;
};
MvKernels mv_kernels(int layout, int W);
MvKernels mv_kernels_mixed(int layout, int W); /* u32/u64 and u64/u32 */
struct MvScanKernels {
    const void *tile_sums, *tile_offsets, *apply, *dry_status;
};
MvScanKernels mv_scan_kernels();

/* message returned by wc_last_error() on the calling thread */
void set_last_error(const char *msg);

/* host helpers of wc_capi.cu for the other translation units: set the
 * error message and return `code`; map a CUDA error to a WC_ERR code;
 * launch geometry (at most one wave of resident blocks); the capacity rule */
int host_fail(int code, const char *msg);
int host_cuda_fail(cudaError_t e, const char *what);
unsigned host_grid(const void *kernel, int block, uint64_t items, uint64_t per_block);
uint64_t host_valid_capacity(uint64_t min_capacity, uint64_t cg);
/* the multi-value tables' shared host steps: per-key counts (in end) to
 * begin / end offsets, a host-side Status join, a dry run's statuses, one
 * device counter read back */
int host_offsets_scan(void **scratch, uint64_t *scratch_bytes, uint64_t *begin, uint64_t *end,
                      uint64_t n, cudaStream_t s);
int host_join_status(uint32_t *status, uint32_t bits, cudaStream_t s);
int host_dry_run_status(void *status_out, uint64_t n, int handler, uint32_t ignore, cudaStream_t s);
int host_read_counter(const unsigned long long *d, cudaStream_t s, uint64_t *out);

/* wc_partition's passes with the owner of a key = the shard holding its
 * block of a Bloom filter of num_blocks blocks (wc_partition.cu) */
int partition_by_bloom_block(const void *keys, uint64_t n, uint32_t key_bytes, uint32_t num_parts,
                             uint64_t seed, uint32_t hasher, uint64_t num_blocks, void *keys_out,
                             uint64_t *perm_out, uint64_t *counts_out, uint64_t *scratch,
                             wc_stream_t stream);

/* kernels this library launched (wc_launch_count) */
void note_launches(uint32_t n);

/* bytes [off, off + len) of the memory image of an empty single-value
 * table placed by wc_svht_create_on */
int host_svht_empty_image(const wc_table_config *cfg, uint64_t min_capacity, unsigned char *dst,
                          uint64_t off, uint64_t len);

/* the device view, slot layout and window width of an initialized
 * single-value table, and the windows a probing length allows */
int host_svht_view(const wc_table *t, TableView *view, int *layout, uint32_t *cg,
                   uint64_t probing_length, uint64_t *max_windows_out);

} // namespace b200
} // namespace warpcore

#endif
