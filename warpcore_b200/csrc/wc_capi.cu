/*
 * wc_capi.cu -- host side of the C ABI declared in include/warpcore_b200.h.
 *
 * Owns the device allocations of each table / filter (the reference's
 * constructors allocate with cudaMalloc and the destructors free,
 * single_value_hash_table.cuh:112-169, storage.cuh:454-516), checks arguments,
 * picks the kernel for (slot layout, window width, operation) and sizes the
 * grid as a whole number of waves: SM count x resident blocks per SM.
 */
#include <warpcore_b200.h>

#include "wc_internal.h"

#include <atomic>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <dlfcn.h>
#include <mutex>
#include <string>
#include <unordered_map>
#include <vector>

#include "wc_primes.inc"

using namespace warpcore::b200;

namespace {

thread_local std::string g_last_error;

int fail(int code, const char *fmt, ...) __attribute__((format(printf, 2, 3)));
int fail(int code, const char *fmt, ...)
{
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    std::vsnprintf(buf, sizeof(buf), fmt, ap);
    va_end(ap);
    g_last_error = buf;
    return code;
}

int cuda_fail(cudaError_t e, const char *what)
{
    return fail(e == cudaErrorMemoryAllocation ? WC_ERR_OUT_OF_MEMORY : WC_ERR_CUDA,
                "%s: %s", what, cudaGetErrorString(e));
}

#define WC_CUDA(call)                                                          \
    do {                                                                       \
        cudaError_t e_ = (call);                                               \
        if (e_ != cudaSuccess) return cuda_fail(e_, #call);                    \
    } while (0)

/* ---- capacity rule (base.cuh:27-34) over the generated prime table ---- */

const uint64_t *prime_table()
{
    static uint64_t *table = nullptr;
    static std::once_flag once;
    std::call_once(once, [] {
        table = new uint64_t[kNumPrimes];
        uint64_t p = kPrimeStep + kPrimeGaps[0];
        table[0] = p;
        for (uint64_t i = 1; i < kNumPrimes; ++i) {
            p += kPrimeStep + kPrimeGaps[i];
            table[i] = p;
        }
    });
    return table;
}

uint64_t valid_capacity(uint64_t min_capacity, uint64_t cg)
{
    const uint64_t *pt = prime_table();
    const uint64_t x = (min_capacity + cg - 1) / cg;
    uint64_t lo = 0, hi = kNumPrimes;
    while (lo < hi) {
        const uint64_t mid = (lo + hi) / 2;
        if (pt[mid] < x) lo = mid + 1;
        else hi = mid;
    }
    return lo == kNumPrimes ? 0 : pt[lo] * cg;
}

bool valid_cg(uint32_t cg)
{
    return cg == 1 || cg == 2 || cg == 4 || cg == 8 || cg == 16 || cg == 32;
}

/* ---- launch geometry ---- */

struct DeviceProps {
    int sms = 148;
    int l2_bytes = 0;
    int persist_max = 0; /* cudaDevAttrMaxPersistingL2CacheSize */
    int window_max = 0;  /* cudaDevAttrMaxAccessPolicyWindowSize */
};

const DeviceProps &device_props()
{
    static std::mutex mu;
    static std::unordered_map<int, DeviceProps> cache;
    int dev = 0;
    cudaGetDevice(&dev);
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache.find(dev);
    if (it != cache.end()) return it->second;
    DeviceProps p;
    cudaDeviceGetAttribute(&p.sms, cudaDevAttrMultiProcessorCount, dev);
    cudaDeviceGetAttribute(&p.l2_bytes, cudaDevAttrL2CacheSize, dev);
    cudaDeviceGetAttribute(&p.persist_max, cudaDevAttrMaxPersistingL2CacheSize, dev);
    cudaDeviceGetAttribute(&p.window_max, cudaDevAttrMaxAccessPolicyWindowSize, dev);
    cudaGetLastError(); /* an attribute this device lacks reads as 0 */
    return cache.emplace(dev, p).first->second;
}

/* ---- L2 persistence for tables that fit in L2 ----
 * A table (or filter) whose slot array fits the device's persisting-L2
 * maximum gets an access-policy window over that array on each of its own
 * launches (a launch attribute, so the caller's streams are untouched):
 * its lines are kept as persisting and the streamed keys and outputs cannot
 * evict them.  The set-aside is this process's context limit
 * cudaLimitPersistingL2CacheSize, made once per device when the first
 * eligible table is created; it ends with the context. */
std::atomic<int> g_l2_mode{1};

/* Fingerprints (one byte per slot, b200_core.cuh) pay off where probing
 * reads DRAM: slot arrays larger than L2.  WC_FINGERPRINTS_AUTO gives them
 * to those tables only; ALWAYS / NEVER override for tables created later. */
std::atomic<int> g_fp_mode{-1}; /* -1: not yet read from the environment */

/* Operations (bit kOp*) that run the fingerprint-first kernel on tables
 * with fingerprints; the others run the whole-window kernel, which keeps
 * the fingerprints up to date.  Bit 4 makes the fingerprint kernel load a
 * claim's slot before its compare-and-swap.  Measured on B200 with u64
 * pairs at load 0.9, 2^27 keys: retrieve 13.0 -> 20.5 G/s on fingerprints;
 * the window insert slows down on a fingerprint table (9.1 G/s, its
 * fingerprint byte writes miss L2) more than the fingerprint insert does
 * (11.7 G/s), so every operation reads fingerprints first. */
std::atomic<uint32_t> g_fp_ops{0xFu};

/* Operations (bit kOp*) whose whole-window probing runs the one-key-per-lane
 * kernel (wc_lane_kernels.cuh) where a window is at most 128 bytes; the
 * others run table_op_kernel.  Counting inserts always run table_op_kernel. */
std::atomic<uint32_t> g_lane_ops{0xDu};

/* Random-access regions of the multi-pass kernels, for inserts and for
 * queries (bytes; 0 = one pass).  Random 64-byte reads on B200 measured
 * 64 G/s over 256 MiB, 19 G/s over 320 MiB and 13.5 G/s over 512 MiB, so a
 * pass works on at most 256 MiB.  Smaller regions cost another pass over
 * the keys each: on the 2^32-bit filter with 2^28 keys, regions of 64 /
 * 128 / 256 MiB ran inserts at 11.0 / 14.9 / 17.0 G keys/s and queries at
 * 11.8 / 17.0 / 21.2. */
std::atomic<uint64_t> g_region_bytes[2] = {{256ull << 20}, {256ull << 20}};

} // namespace

uint64_t warpcore::b200::region_bytes(bool insert)
{
    return g_region_bytes[insert ? 0 : 1].load(std::memory_order_relaxed);
}

namespace {

int fp_mode()
{
    int m = g_fp_mode.load(std::memory_order_relaxed);
    if (m < 0) {
        /* WARPCORE_B200_FINGERPRINTS = auto | always | never */
        const char *e = std::getenv("WARPCORE_B200_FINGERPRINTS");
        int want = WC_FINGERPRINTS_AUTO;
        if (e && std::strcmp(e, "always") == 0) want = WC_FINGERPRINTS_ALWAYS;
        if (e && std::strcmp(e, "never") == 0) want = WC_FINGERPRINTS_NEVER;
        int expect = -1;
        g_fp_mode.compare_exchange_strong(expect, want);
        m = g_fp_mode.load(std::memory_order_relaxed);
    }
    return m;
}

bool want_fingerprints(uint64_t slot_bytes_total)
{
    const int m = fp_mode();
    if (m == WC_FINGERPRINTS_ALWAYS) return true;
    if (m == WC_FINGERPRINTS_NEVER) return false;
    return slot_bytes_total > uint64_t(device_props().l2_bytes);
}

size_t l2_setaside(int dev)
{
    static std::mutex mu;
    static std::unordered_map<int, size_t> done;
    std::lock_guard<std::mutex> lock(mu);
    auto it = done.find(dev);
    if (it != done.end()) return it->second;
    const DeviceProps &p = device_props();
    size_t want = size_t(p.persist_max);
    const size_t cap = size_t(p.l2_bytes) / 4 * 3;
    if (want > cap) want = cap;
    size_t got = 0;
    if (want && cudaDeviceSetLimit(cudaLimitPersistingL2CacheSize, want) == cudaSuccess)
        cudaDeviceGetLimit(&got, cudaLimitPersistingL2CacheSize);
    cudaGetLastError();
    done.emplace(dev, got);
    return got;
}

/* window over [base, base + bytes) if the array fits; 0 bytes = none */
struct L2Window {
    void *base = nullptr;
    uint64_t bytes = 0;
    float hit_ratio = 0.f;
    int device = -1;
};

/* Bytes of the live windows per device.  A new array gets a window only
 * while all windows together fit the set-aside: with many resident tables
 * (more than L2 holds), the first ones to fit keep their lines and the
 * others run as plain launches, instead of all of them evicting each
 * other's persisting lines and shrinking L2 for everything else. */
std::mutex g_l2_mu;
std::unordered_map<int, uint64_t> g_l2_committed;

L2Window l2_window_for(void *base, uint64_t bytes)
{
    L2Window w;
    if (!g_l2_mode.load(std::memory_order_relaxed) || !base || !bytes) return w;
    const DeviceProps &p = device_props();
    if (p.persist_max <= 0 || p.window_max <= 0) return w;
    if (bytes > uint64_t(p.persist_max) || bytes > uint64_t(p.window_max)) return w;
    int dev = 0;
    cudaGetDevice(&dev);
    const size_t setaside = l2_setaside(dev);
    if (!setaside || bytes > setaside) return w;
    std::lock_guard<std::mutex> lock(g_l2_mu);
    uint64_t &used = g_l2_committed[dev];
    if (used + bytes > setaside) return w;
    used += bytes;
    w.base = base;
    w.bytes = bytes;
    w.hit_ratio = 1.f;
    w.device = dev;
    return w;
}

/* gives the window's bytes back and returns its lines to normal */
void l2_window_release(L2Window &w)
{
    if (!w.bytes) return;
    {
        std::lock_guard<std::mutex> lock(g_l2_mu);
        uint64_t &used = g_l2_committed[w.device];
        used = used >= w.bytes ? used - w.bytes : 0;
    }
    cudaCtxResetPersistingL2Cache();
    w = L2Window();
}

cudaError_t launch_in_window(const void *kfn, unsigned grid, unsigned block, void **args,
                             cudaStream_t s, const L2Window &w)
{
    if (!w.bytes || !g_l2_mode.load(std::memory_order_relaxed)) {
        const cudaError_t e = cudaLaunchKernel(kfn, dim3(grid), dim3(block), args, 0, s);
        if (e == cudaSuccess) note_launches(1);
        return e;
    }
    cudaLaunchConfig_t cfg = {};
    cfg.gridDim = dim3(grid);
    cfg.blockDim = dim3(block);
    cfg.dynamicSmemBytes = 0;
    cfg.stream = s;
    cudaLaunchAttribute attr[1];
    attr[0].id = cudaLaunchAttributeAccessPolicyWindow;
    attr[0].val.accessPolicyWindow.base_ptr = w.base;
    attr[0].val.accessPolicyWindow.num_bytes = size_t(w.bytes);
    attr[0].val.accessPolicyWindow.hitRatio = w.hit_ratio;
    attr[0].val.accessPolicyWindow.hitProp = cudaAccessPropertyPersisting;
    attr[0].val.accessPolicyWindow.missProp = cudaAccessPropertyStreaming;
    cfg.attrs = attr;
    cfg.numAttrs = 1;
    const cudaError_t e = cudaLaunchKernelExC(&cfg, kfn, args);
    if (e == cudaSuccess) note_launches(1);
    return e;
}

int blocks_per_sm(const void *kernel, int block)
{
    static std::mutex mu;
    static std::unordered_map<const void *, int> cache[6];
    const int slot = block >= 256 ? 0 : block >= 128 ? 1 : block >= 64 ? 2 : block >= 32 ? 3 : 4;
    std::lock_guard<std::mutex> lock(mu);
    auto it = cache[slot].find(kernel);
    if (it != cache[slot].end()) return it->second;
    int n = 0;
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, kernel, block, 0) != cudaSuccess || n < 1) {
        cudaGetLastError();
        n = 1;
    }
    cache[slot].emplace(kernel, n);
    return n;
}

/* ---- launch tuning table (filled by the autotuner through wc_tune_set) ----
 * keyed on key width, operation, load-factor bucket and batch-size bucket;
 * an empty entry means the default geometry (256 threads, occupancy limit) */
struct TuneEntry {
    uint32_t block = 0, blocks_per_sm = 0;
};
constexpr int kTuneOps = 4, kTuneLoads = WC_TUNE_LOAD_BUCKETS, kTuneSizes = WC_TUNE_SIZE_BUCKETS;
TuneEntry g_tune[2][kTuneOps][kTuneLoads][kTuneSizes];
std::mutex g_tune_mu;

int tune_size_bucket(uint64_t n)
{
    int lg = 0;
    while ((1ull << (lg + 1)) <= n && lg < 62) ++lg;
    int b = (lg - 6) / 2;
    return b < 0 ? 0 : (b >= kTuneSizes ? kTuneSizes - 1 : b);
}

int tune_load_bucket(double lf)
{
    return lf < 0.5 ? 0 : lf < 0.7 ? 1 : lf < 0.85 ? 2 : 3;
}

TuneEntry tune_lookup(uint32_t key_bytes, int op, double lf, uint64_t n)
{
    std::lock_guard<std::mutex> lock(g_tune_mu);
    return g_tune[key_bytes == 8][op & 3][tune_load_bucket(lf)][tune_size_bucket(n)];
}

/* grid for `items` work items of which one block handles `per_block` per
 * pass; at most one full wave of resident blocks (grid-stride beyond) */
unsigned grid_for(const void *kernel, int block, uint64_t items, uint64_t per_block)
{
    const uint64_t wave = uint64_t(device_props().sms) * blocks_per_sm(kernel, block);
    uint64_t need = (items + per_block - 1) / per_block;
    if (need < 1) need = 1;
    return unsigned(need < wave ? need : wave);
}

constexpr int kBlock = 256;

} // namespace

void warpcore::b200::set_last_error(const char *msg) { g_last_error = msg; }

int warpcore::b200::host_fail(int code, const char *msg)
{
    g_last_error = msg;
    return code;
}

int warpcore::b200::host_cuda_fail(cudaError_t e, const char *what) { return cuda_fail(e, what); }

unsigned warpcore::b200::host_grid(const void *kernel, int block, uint64_t items,
                                   uint64_t per_block)
{
    return grid_for(kernel, block, items, per_block);
}

uint64_t warpcore::b200::host_valid_capacity(uint64_t min_capacity, uint64_t cg)
{
    return valid_capacity(min_capacity, cg);
}

/* counts in end -> end = inclusive prefix sums, begin = exclusive ones (the
 * reference's cub::DeviceScan::InclusiveSum step): tile sums, tile offsets,
 * apply.  The tile-sum buffer grows on demand. */
int warpcore::b200::host_offsets_scan(void **scratch, uint64_t *scratch_bytes, uint64_t *begin,
                                      uint64_t *end, uint64_t n, cudaStream_t s)
{
    const MvScanKernels k = mv_scan_kernels();
    const uint64_t ntiles = (n + kScanTile - 1) / kScanTile;
    const uint64_t need = ntiles * sizeof(unsigned long long);
    if (need > *scratch_bytes) {
        WC_CUDA(cudaStreamSynchronize(s));
        if (*scratch) cudaFree(*scratch);
        *scratch = nullptr;
        *scratch_bytes = 0;
        WC_CUDA(cudaMalloc(scratch, need));
        *scratch_bytes = need;
    }
    auto *e = reinterpret_cast<unsigned long long *>(end);
    auto *b = reinterpret_cast<unsigned long long *>(begin);
    auto *ts = reinterpret_cast<unsigned long long *>(*scratch);
    uint64_t nn = n, nt = ntiles;
    void *a1[] = {&e, &nn, &ts};
    WC_CUDA(cudaLaunchKernel(k.tile_sums, dim3(unsigned(ntiles)), dim3(kScanThreads), a1, 0, s));
    void *a2[] = {&ts, &nt};
    WC_CUDA(cudaLaunchKernel(k.tile_offsets, dim3(1), dim3(kScanThreads), a2, 0, s));
    /* end == begin + 1: the scan writes end only, begin[0] is zero */
    int write_begin = e == b + 1 ? 0 : 1;
    if (!write_begin) WC_CUDA(cudaMemsetAsync(b, 0, sizeof(unsigned long long), s));
    void *a3[] = {&e, &b, &nn, &ts, &write_begin};
    WC_CUDA(cudaLaunchKernel(k.apply, dim3(unsigned(ntiles)), dim3(kScanThreads), a3, 0, s));
    note_launches(3);
    return WC_OK;
}

/* join bits into a device Status word from the host (synchronises) */
int warpcore::b200::host_join_status(uint32_t *status, uint32_t bits, cudaStream_t s)
{
    uint32_t cur = 0;
    WC_CUDA(cudaMemcpyAsync(&cur, status, sizeof(cur), cudaMemcpyDeviceToHost, s));
    WC_CUDA(cudaStreamSynchronize(s));
    cur |= bits;
    WC_CUDA(cudaMemcpyAsync(status, &cur, sizeof(cur), cudaMemcpyHostToDevice, s));
    WC_CUDA(cudaStreamSynchronize(s));
    return WC_OK;
}

/* a dry run's per-key statuses: dry_run for every key */
int warpcore::b200::host_dry_run_status(void *status_out, uint64_t n, int handler,
                                        uint32_t ignore, cudaStream_t s)
{
    if (!status_out || handler == WC_HANDLER_NOTHING || n == 0) return WC_OK;
    const MvScanKernels k = mv_scan_kernels();
    uint64_t nn = n;
    int h = handler;
    uint32_t mask = (~ignore) ^ 0xFFFu;
    void *args[] = {&status_out, &nn, &h, &mask};
    WC_CUDA(cudaLaunchKernel(k.dry_status, dim3(grid_for(k.dry_status, kBlock, n, kBlock)),
                             dim3(kBlock), args, 0, s));
    note_launches(1);
    return WC_OK;
}

/* one device counter read back (synchronises) */
int warpcore::b200::host_read_counter(const unsigned long long *d, cudaStream_t s, uint64_t *out)
{
    unsigned long long h = 0;
    WC_CUDA(cudaMemcpyAsync(&h, d, sizeof(h), cudaMemcpyDeviceToHost, s));
    WC_CUDA(cudaStreamSynchronize(s));
    *out = h;
    return WC_OK;
}

static std::atomic<unsigned long long> g_launches{0};
void warpcore::b200::note_launches(uint32_t n) { g_launches.fetch_add(n, std::memory_order_relaxed); }

/* ------------------------------------------------------------------ */
/* handles                                                              */
/* ------------------------------------------------------------------ */

struct wc_table {
    int kind = 0; /* 0 single-value, 1 hash set, 2 counting */
    wc_table_config cfg{};
    int layout = 0;
    uint32_t slot_bytes = 0;
    uint64_t capacity = 0;
    uint64_t num_buckets = 0;
    uint64_t seed = 0;
    uint64_t max_count = 0;
    bool initialized = false;
    void *slots = nullptr;
    uint32_t *status = nullptr;            /* device Status word */
    unsigned long long *counter = nullptr; /* device scratch counter */
    unsigned long long *live = nullptr;    /* device: kLiveStripes valid-key counters */
    bool owns_memory = true;               /* false: placed on caller memory */
    int device = 0;
    uint64_t keys_inserted = 0; /* since init: an upper bound of size(), for tuning */
    L2Window l2;                /* access-policy window over the slots, if they fit */
    unsigned char *fps = nullptr; /* one fingerprint byte per slot, or NULL */
    /* multi-value tables */
    uint64_t max_values = ~0ull;
    unsigned long long *num_keys = nullptr; /* device: keys holding at least one value */
    void *scratch = nullptr;                /* device: scan tile sums, grown on demand */
    uint64_t scratch_bytes = 0;
    /* single-value tables stored as a struct of arrays: slots holds the
     * keys (probed as a hash set's slots), values one value per slot */
    bool soa = false;
    void *values = nullptr;
};

struct wc_bloom {
    wc_bloom_config cfg{};
    uint64_t num_bits = 0, num_slots = 0, num_blocks = 0, k = 0, seed = 0;
    uint64_t block_base = 0, local_blocks = 0; /* the blocks this filter holds */
    void *words = nullptr;
    int device = 0;
    L2Window l2;
};

namespace {

uint64_t key_mask(uint32_t key_bytes)
{
    return key_bytes == 4 ? 0xffffffffull : ~0ull;
}

/* a table's small device block: Status word at 0, scratch counter at 128,
 * multi-value key count at 192, the striped valid-key counters at 256 */
constexpr uint64_t kLiveBytes = uint64_t(kLiveStripes) * kLiveStride * 8;
constexpr uint64_t kAuxBytes = 256 + kLiveBytes;

TableView view_of(const wc_table *t)
{
    TableView v;
    v.slots = t->slots;
    v.status = t->status;
    v.fps = t->fps;
    /* multi-value tables count values per key and have no live counter */
    v.live = t->kind == 3 ? nullptr : t->live;
    v.num_buckets = t->num_buckets;
    v.seed = t->seed;
    v.empty_key = t->cfg.empty_key;
    v.tombstone_key = t->cfg.tombstone_key;
    v.max_count = t->max_count;
    v.magic_nb = barrett_magic(t->num_buckets);
    v.magic_nb1 = barrett_magic(t->num_buckets > 1 ? t->num_buckets - 1 : 1);
    v.probing = t->cfg.probing;
    v.hasher1 = t->cfg.hasher1;
    v.hasher2 = t->cfg.hasher2;
    v.cg_size = t->cfg.cg_size;
    v.values = t->values;
    return v;
}

int check_config(const wc_table_config *cfg, int kind)
{
    if (!cfg) return fail(WC_ERR_INVALID_ARGUMENT, "config is NULL");
    if (cfg->key_bytes != 4 && cfg->key_bytes != 8)
        return fail(WC_ERR_UNSUPPORTED, "key_bytes must be 4 or 8");
    /* tables with values take 4- or 8-byte values with either key width */
    if (kind != 1 && cfg->value_bytes != 4 && cfg->value_bytes != 8)
        return fail(WC_ERR_UNSUPPORTED, "value_bytes must be 4 or 8 (got %u)", cfg->value_bytes);
    if (!valid_cg(cfg->cg_size))
        return fail(WC_ERR_INVALID_ARGUMENT, "cg_size must be 1, 2, 4, 8, 16 or 32");
    if (cfg->probing > WC_PROBING_QUADRATIC)
        return fail(WC_ERR_INVALID_ARGUMENT, "unknown probing scheme %u", cfg->probing);
    if (cfg->hasher1 > WC_HASH_IDENTITY64 || cfg->hasher2 > WC_HASH_IDENTITY64)
        return fail(WC_ERR_INVALID_ARGUMENT, "unknown hasher");
    const uint64_t km = key_mask(cfg->key_bytes);
    if ((cfg->empty_key & km) == (cfg->tombstone_key & km))
        return fail(WC_ERR_INVALID_ARGUMENT, "empty key and tombstone key must differ");
    return WC_OK;
}

int fill_slots(wc_table *t, cudaStream_t stream)
{
    /* 16 bytes of empty slots: key = empty, payload = 0 */
    const uint64_t e = t->cfg.empty_key & key_mask(t->cfg.key_bytes);
    uint32_t w[4];
    switch (t->layout) {
    case kLayoutKV32: w[0] = uint32_t(e); w[1] = 0; w[2] = uint32_t(e); w[3] = 0; break;
    case kLayoutKV64:
    case kLayoutK32V64: /* e < 2^32 there: the key's upper half is 0 */
    case kLayoutK64V32: w[0] = uint32_t(e); w[1] = uint32_t(e >> 32); w[2] = 0; w[3] = 0; break;
    case kLayoutSet32: w[0] = w[1] = w[2] = w[3] = uint32_t(e); break;
    default: w[0] = uint32_t(e); w[1] = uint32_t(e >> 32); w[2] = w[0]; w[3] = w[1]; break;
    }
    const uint4 pattern = make_uint4(w[0], w[1], w[2], w[3]);
    const uint64_t n_u32 = t->capacity * t->slot_bytes / 4;
    const void *kfn = reinterpret_cast<const void *>(fill_kernel<0>);
    const unsigned grid = grid_for(kfn, kBlock, n_u32 / 4, kBlock);
    uint32_t *p = reinterpret_cast<uint32_t *>(t->slots);
    uint64_t n = n_u32;
    uint4 pat = pattern;
    void *args[] = {&p, &n, &pat};
    WC_CUDA(launch_in_window(kfn, grid, kBlock, args, stream, t->l2));
    return WC_OK;
}

/* Memory of a table placed on caller-provided device memory: the slots at
 * offset 0, the small device block (Status word, counters) at the next
 * 256-byte boundary, then the fingerprints if the policy gives them. */
struct TablePlacement {
    uint64_t slot_bytes, fp_bytes, aux_off, fp_off, total;
};

TablePlacement placement(uint64_t cap, uint32_t slot_bytes, bool fingerprints)
{
    TablePlacement p;
    p.slot_bytes = cap * slot_bytes;
    p.fp_bytes = fingerprints ? cap : 0;
    p.aux_off = (p.slot_bytes + 255) & ~uint64_t(255);
    p.fp_off = p.aux_off + ((kAuxBytes + 255) & ~uint64_t(255));
    p.total = p.fp_off + p.fp_bytes;
    return p;
}

int table_create(int kind, const wc_table_config *cfg, uint64_t min_capacity, uint64_t seed,
                 uint64_t max_count, int no_init, wc_table **out, void *memory = nullptr,
                 uint64_t memory_bytes = 0, cudaStream_t stream = nullptr, bool soa = false)
{
    if (!out) return fail(WC_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    int rc = check_config(cfg, kind);
    if (rc) return rc;
    const uint64_t cap = valid_capacity(min_capacity, cfg->cg_size);
    if (cap == 0)
        return fail(WC_ERR_INVALID_ARGUMENT,
                    "min_capacity %llu exceeds the largest table capacity",
                    (unsigned long long)min_capacity);
    auto *t = new wc_table();
    t->kind = kind;
    t->cfg = *cfg;
    if (kind == 1) t->cfg.value_bytes = 0;
    t->cfg.empty_key &= key_mask(cfg->key_bytes);
    t->cfg.tombstone_key &= key_mask(cfg->key_bytes);
    if (kind == 1) {
        t->layout = cfg->key_bytes == 4 ? kLayoutSet32 : kLayoutSet64;
        t->slot_bytes = cfg->key_bytes;
    } else if (cfg->value_bytes == cfg->key_bytes) {
        t->layout = cfg->key_bytes == 4 ? kLayoutKV32 : kLayoutKV64;
        t->slot_bytes = 2 * cfg->key_bytes;
    } else {
        t->layout = cfg->key_bytes == 4 ? kLayoutK32V64 : kLayoutK64V32;
        t->slot_bytes = 16;
    }
    if (soa) {
        /* the key array is a hash set's slot array */
        t->soa = true;
        t->layout = cfg->key_bytes == 4 ? kLayoutSet32 : kLayoutSet64;
        t->slot_bytes = cfg->key_bytes;
    }
    t->capacity = cap;
    t->num_buckets = cap / cfg->cg_size;
    t->seed = seed & key_mask(cfg->key_bytes);
    const uint64_t vmax = cfg->value_bytes == 4 ? 0xffffffffull : ~0ull;
    t->max_count = kind == 2 ? (max_count < vmax ? max_count : vmax) : ~0ull;
    cudaGetDevice(&t->device);

    const uint64_t bytes = cap * t->slot_bytes;
    const uint64_t fp_bytes = (kind != 3 && !soa && want_fingerprints(bytes)) ? cap : 0;
    const uint64_t value_bytes = soa ? cap * cfg->value_bytes : 0;
    if (memory) {
        /* caller-provided memory: carve the slots, the device block and the
         * fingerprints out of it; the table does not free it */
        const TablePlacement pl = placement(cap, t->slot_bytes, fp_bytes != 0);
        if (memory_bytes < pl.total || (reinterpret_cast<uintptr_t>(memory) & 255)) {
            delete t;
            return fail(WC_ERR_INVALID_ARGUMENT,
                        "memory must be 256-byte aligned and hold %llu bytes",
                        (unsigned long long)pl.total);
        }
        unsigned char *base = reinterpret_cast<unsigned char *>(memory);
        t->owns_memory = false;
        t->slots = base;
        t->status = reinterpret_cast<uint32_t *>(base + pl.aux_off);
        t->counter = reinterpret_cast<unsigned long long *>(base + pl.aux_off + 128);
        t->num_keys = reinterpret_cast<unsigned long long *>(base + pl.aux_off + 192);
        t->live = reinterpret_cast<unsigned long long *>(base + pl.aux_off + 256);
        t->fps = fp_bytes ? base + pl.fp_off : nullptr;
        if (no_init == 2) {
            /* the memory holds a table image of this configuration */
            t->initialized = true;
        } else {
            cudaError_t e = cudaMemsetAsync(t->status, 0, kAuxBytes, stream);
            if (e == cudaSuccess) e = cudaStreamSynchronize(stream);
            if (e != cudaSuccess) {
                delete t;
                return cuda_fail(e, "cudaMemsetAsync");
            }
            if (!no_init) {
                rc = wc_table_init(t, t->seed, reinterpret_cast<wc_stream_t>(stream));
                if (rc) {
                    delete t;
                    return rc;
                }
            }
        }
        *out = t;
        return WC_OK;
    }
    /* the reference checks free memory before allocating (storage.cuh:464-473) */
    size_t free_b = 0, total_b = 0;
    if (cudaMemGetInfo(&free_b, &total_b) != cudaSuccess) {
        delete t;
        return cuda_fail(cudaGetLastError(), "cudaMemGetInfo");
    }
    if (bytes + fp_bytes + value_bytes + 4096 > free_b) {
        delete t;
        return fail(WC_ERR_OUT_OF_MEMORY, "table needs %llu bytes, %llu free",
                    (unsigned long long)(bytes + fp_bytes + value_bytes), (unsigned long long)free_b);
    }
    cudaError_t e = cudaMalloc(&t->slots, bytes);
    if (e == cudaSuccess && fp_bytes) e = cudaMalloc(&t->fps, fp_bytes);
    if (e == cudaSuccess && value_bytes) e = cudaMalloc(&t->values, value_bytes);
    if (e == cudaSuccess) {
        void *aux = nullptr;
        e = cudaMalloc(&aux, kAuxBytes);
        if (e == cudaSuccess) {
            t->status = reinterpret_cast<uint32_t *>(aux);
            t->counter = reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(aux) + 128);
            t->num_keys = reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(aux) + 192);
            t->live = reinterpret_cast<unsigned long long *>(reinterpret_cast<char *>(aux) + 256);
        }
    }
    if (e != cudaSuccess) {
        if (t->slots) cudaFree(t->slots);
        if (t->fps) cudaFree(t->fps);
        if (t->values) cudaFree(t->values);
        delete t;
        return cuda_fail(e, "cudaMalloc");
    }
    e = cudaMemset(t->status, 0, kAuxBytes);
    if (e != cudaSuccess) {
        wc_table_destroy(t);
        return cuda_fail(e, "cudaMemset");
    }
    t->l2 = l2_window_for(t->slots, bytes);
    if (!no_init) {
        rc = wc_table_init(t, t->seed, nullptr);
        if (rc) {
            wc_table_destroy(t);
            return rc;
        }
    }
    *out = t;
    return WC_OK;
}

int check_table(const wc_table *t, int kind_mask)
{
    if (!t) return fail(WC_ERR_INVALID_ARGUMENT, "table is NULL");
    if (!((1 << t->kind) & kind_mask))
        return fail(WC_ERR_INVALID_ARGUMENT, "operation does not apply to this table kind");
    if (!t->initialized) return fail(WC_ERR_NOT_INITIALIZED, "table is not initialized");
    return WC_OK;
}

/* The one-key-per-lane window kernel reads a window with one 32-byte load
 * per sector.  On a table that L2 holds, that beats groups of lanes per
 * window and their ballots (B200, CUDA events: u32 pairs, 16 MB table:
 * retrieve 60.2 vs 38.0 G keys/s, insert 21.1 vs 18.0; u64 pairs, 48 MB:
 * retrieve 29.5 vs 16.8, insert 13.2 vs 14.8).  On a table in DRAM its
 * sector requests cost more than one request per window (u64 pairs,
 * 2.4 GB: insert 5.9 vs 14.5), so larger tables keep the group kernel.
 * Inserts take the lane kernel for windows of at most 64 bytes. */
TableKernel pick_lane_kernel(const wc_table *t, int op)
{
    if (!((g_lane_ops.load(std::memory_order_relaxed) >> op) & 1u)) return nullptr;
    if (t->capacity * t->slot_bytes > uint64_t(device_props().l2_bytes)) return nullptr;
    if (op == kOpInsert && uint64_t(t->cfg.cg_size) * t->slot_bytes > 64) return nullptr;
    const int W = int(t->cfg.cg_size);
    switch (t->layout) {
    case kLayoutKV32: return lane_kernel_kv32(W, op);
    case kLayoutKV64: return lane_kernel_kv64(W, op);
    case kLayoutSet32: return lane_kernel_set32(W, op);
    case kLayoutK32V64: return lane_kernel_k32v64(W, op);
    case kLayoutK64V32: return lane_kernel_k64v32(W, op);
    default: return lane_kernel_set64(W, op);
    }
}

TableKernel pick_window_kernel(const wc_table *t, int op)
{
    if (t->soa) return table_kernel_soa(t->cfg.key_bytes, t->cfg.value_bytes, int(t->cfg.cg_size), op);
    if (TableKernel k = pick_lane_kernel(t, op)) return k;
    const int W = int(t->cfg.cg_size);
    switch (t->layout) {
    case kLayoutKV32: return table_kernel_kv32(W, op, false);
    case kLayoutKV64: return table_kernel_kv64(W, op, false);
    case kLayoutSet32: return table_kernel_set32(W, op, false);
    case kLayoutK32V64: return table_kernel_k32v64(W, op, false);
    case kLayoutK64V32: return table_kernel_k64v32(W, op, false);
    default: return table_kernel_set64(W, op, false);
    }
}

TableKernel pick_table_kernel(const wc_table *t, int op)
{
    const int W = int(t->cfg.cg_size);
    const bool fp = t->fps != nullptr && ((g_fp_ops.load(std::memory_order_relaxed) >> op) & 1u);
    if (!fp) return pick_window_kernel(t, op);
    switch (t->layout) {
    case kLayoutKV32: return table_kernel_kv32(W, op, fp);
    case kLayoutKV64: return table_kernel_kv64(W, op, fp);
    case kLayoutSet32: return table_kernel_set32(W, op, fp);
    case kLayoutK32V64: return table_kernel_k32v64(W, op, fp);
    case kLayoutK64V32: return table_kernel_k64v32(W, op, fp);
    default: return table_kernel_set64(W, op, fp);
    }
}

int table_op(wc_table *t, int op, const void *keys, const void *values, void *out,
             uint64_t n, wc_stream_t stream, uint64_t probing_length, void *status_out,
             int handler, uint32_t ignore)
{
    if (handler < WC_HANDLER_NOTHING || handler > WC_HANDLER_BOOLEAN)
        return fail(WC_ERR_INVALID_ARGUMENT, "unknown status handler %d", handler);
    if (n == 0) return WC_OK;
    if (!keys) return fail(WC_ERR_INVALID_ARGUMENT, "keys_in is NULL");
    if (op == kOpInsert && t->kind == 0 && !values)
        return fail(WC_ERR_INVALID_ARGUMENT, "values_in is NULL");
    if (op == kOpRetrieve && !out) return fail(WC_ERR_INVALID_ARGUMENT, "output is NULL");
    /* A large insert into a table whose fingerprints exceed half of L2 runs
     * the whole-window kernel without fingerprint writes and then rebuilds
     * all fingerprints in one streaming pass (see fp_rebuild_kernel). */
    const bool rebuild = t->fps && (op == kOpInsert || op == kOpCount) &&
                         n * 8 > t->capacity &&
                         t->capacity > uint64_t(device_props().l2_bytes) / 2 &&
                         (g_fp_ops.load(std::memory_order_relaxed) & 0x20u) == 0;
    TableKernel k = rebuild ? pick_window_kernel(t, op) : pick_table_kernel(t, op);
    if (!k) return fail(WC_ERR_UNSUPPORTED, "no kernel for this configuration");
    TableOpArgs a;
    a.t = view_of(t);
    if (rebuild) a.t.fps = nullptr; /* the window kernel writes no fingerprints */
    a.keys = keys;
    a.values = values;
    a.out = out;
    a.status_out = handler == WC_HANDLER_NOTHING ? nullptr : status_out;
    a.n = n;
    a.max_windows = max_windows(probing_length, t->cfg.cg_size, t->num_buckets);
    a.bool_mask = (~ignore) ^ 0xFFFu; /* ~Status(Ignore), status.cuh:142-146 */
    a.handler = handler;
    a.is_set = t->kind == 1;
    a.flags = (g_fp_ops.load(std::memory_order_relaxed) & 0x10u) ? kFlagPreloadClaim : 0u;
    /* launch geometry: the tuned entry for this key width, operation, load
     * and batch size, else 256 threads and the occupancy limit */
    const double lf = t->capacity ? double(t->keys_inserted) / double(t->capacity) : 0.0;
    const TuneEntry te = tune_lookup(t->cfg.key_bytes, op, lf > 1.0 ? 1.0 : lf, n);
    const int block = te.block ? int(te.block) : kBlock;
    const void *kfn = reinterpret_cast<const void *>(k);
    const int occ = blocks_per_sm(kfn, block);
    const uint64_t bps = te.blocks_per_sm && int(te.blocks_per_sm) < occ ? te.blocks_per_sm : uint64_t(occ);
    const uint64_t wave = uint64_t(device_props().sms) * bps;
    uint64_t need = (n + block - 1) / block;
    const unsigned grid = unsigned(need < wave ? need : (wave ? wave : 1));
    void *args[] = {&a};
    WC_CUDA(launch_in_window(kfn, grid, unsigned(block), args,
                             reinterpret_cast<cudaStream_t>(stream), t->l2));
    if (rebuild) {
        const RebuildKernel rk = fp_rebuild_kernel_ptr(t->layout);
        const void *rfn = reinterpret_cast<const void *>(rk);
        const unsigned rgrid = grid_for(rfn, kBlock, t->capacity * t->slot_bytes / 64 + 1, kBlock);
        const void *sl = t->slots;
        uint64_t cap = t->capacity, em = t->cfg.empty_key, tb = t->cfg.tombstone_key;
        unsigned char *fp = t->fps;
        void *rargs[] = {&sl, &cap, &em, &tb, &fp};
        WC_CUDA(cudaLaunchKernel(rfn, dim3(rgrid), dim3(kBlock), rargs, 0,
                                 reinterpret_cast<cudaStream_t>(stream)));
        note_launches(1);
    }
    if (op == kOpInsert || op == kOpCount) t->keys_inserted += n;
    return WC_OK;
}

} // namespace

/* Bytes [off, off + len) of the memory image of an empty single-value
 * table placed on caller memory (wc_svht_create_on's layout): empty slots
 * (the empty key, payload 0), then zeros (padding, the Status word and
 * counters, empty fingerprints).  Copying this image in and adopting it
 * (no_init 2) equals wc_svht_create_on with no_init 0 without a kernel. */
int warpcore::b200::host_svht_empty_image(const wc_table_config *cfg, uint64_t min_capacity,
                                          unsigned char *dst, uint64_t off, uint64_t len)
{
    int rc = check_config(cfg, 0);
    if (rc) return rc;
    const uint64_t cap = valid_capacity(min_capacity, cfg->cg_size);
    const uint32_t sb = cfg->value_bytes == cfg->key_bytes ? 2 * cfg->key_bytes : 16;
    const uint64_t slot_total = cap * sb;
    const uint64_t e = cfg->empty_key & key_mask(cfg->key_bytes);
    unsigned char pat[16] = {0};
    std::memcpy(pat, &e, cfg->key_bytes); /* key first, payload (and padding) zero */
    const uint64_t in_slots = off < slot_total ? (slot_total - off < len ? slot_total - off : len) : 0;
    /* the slot pattern from the first slot boundary on, doubled by copies */
    uint64_t head = (sb - off % sb) % sb;
    if (head > in_slots) head = in_slots;
    for (uint64_t i = 0; i < head; ++i) dst[i] = pat[(off + i) % sb];
    uint64_t filled = 0;
    unsigned char *body = dst + head;
    const uint64_t body_len = in_slots - head;
    if (body_len) {
        const uint64_t first = body_len < sb ? body_len : sb;
        std::memcpy(body, pat, first);
        filled = first;
        while (filled < body_len) {
            const uint64_t n = filled < body_len - filled ? filled : body_len - filled;
            std::memcpy(body + filled, body, n);
            filled += n;
        }
    }
    if (len > in_slots) std::memset(dst + in_slots, 0, len - in_slots);
    return WC_OK;
}

int warpcore::b200::host_svht_view(const wc_table *t, TableView *view, int *layout, uint32_t *cg,
                                   uint64_t probing_length, uint64_t *max_windows_out)
{
    if (!t) return fail(WC_ERR_INVALID_ARGUMENT, "table is NULL");
    if (t->kind != 0) return fail(WC_ERR_INVALID_ARGUMENT, "not a single-value table");
    if (!t->initialized) return fail(WC_ERR_NOT_INITIALIZED, "table is not initialized");
    *view = view_of(t);
    *layout = t->layout;
    *cg = t->cfg.cg_size;
    *max_windows_out = max_windows(probing_length, t->cfg.cg_size, t->num_buckets);
    return WC_OK;
}

/* ------------------------------------------------------------------ */
/* C ABI                                                                 */
/* ------------------------------------------------------------------ */

extern "C" {

const char *wc_last_error(void) { return g_last_error.c_str(); }

const char *wc_version(void) { return "warpcore-b200 0.1 (sm_100a)"; }

void wc_svht_default_config(wc_table_config *cfg, uint32_t key_bytes, uint32_t value_bytes)
{
    if (!cfg) return;
    cfg->key_bytes = key_bytes;
    cfg->value_bytes = value_bytes;
    cfg->empty_key = 0;
    cfg->tombstone_key = key_mask(key_bytes);
    cfg->probing = WC_PROBING_DOUBLE;
    cfg->hasher1 = WC_HASH_MURMUR;
    cfg->hasher2 = WC_HASH_MURMUR;
    cfg->cg_size = 8;
}

void wc_hashset_default_config(wc_table_config *cfg, uint32_t key_bytes)
{
    wc_svht_default_config(cfg, key_bytes, 0);
    if (cfg) cfg->cg_size = 16;
}

void wc_counting_default_config(wc_table_config *cfg, uint32_t key_bytes, uint32_t value_bytes)
{
    wc_svht_default_config(cfg, key_bytes, value_bytes);
    if (cfg) cfg->cg_size = 4;
}

uint64_t wc_valid_capacity(uint64_t min_capacity, uint64_t cg_size)
{
    if (!valid_cg(uint32_t(cg_size))) return 0;
    return valid_capacity(min_capacity, cg_size);
}

int wc_svht_create(const wc_table_config *cfg, uint64_t min_capacity, uint64_t seed, int no_init,
                   wc_table **out)
{
    return table_create(0, cfg, min_capacity, seed, 0, no_init, out);
}

int wc_svht_memory_bytes(const wc_table_config *cfg, uint64_t min_capacity, uint64_t *bytes_out)
{
    if (!bytes_out) return fail(WC_ERR_INVALID_ARGUMENT, "bytes_out is NULL");
    *bytes_out = 0;
    int rc = check_config(cfg, 0);
    if (rc) return rc;
    const uint64_t cap = valid_capacity(min_capacity, cfg->cg_size);
    if (cap == 0) return fail(WC_ERR_INVALID_ARGUMENT, "min_capacity exceeds the largest table capacity");
    const uint32_t sb = cfg->value_bytes == cfg->key_bytes ? 2 * cfg->key_bytes : 16;
    *bytes_out = placement(cap, sb, want_fingerprints(cap * sb)).total;
    return WC_OK;
}

int wc_svht_create_on(const wc_table_config *cfg, uint64_t min_capacity, uint64_t seed,
                      int no_init, void *memory, uint64_t memory_bytes, wc_stream_t stream,
                      wc_table **out)
{
    if (!memory) return fail(WC_ERR_INVALID_ARGUMENT, "memory is NULL");
    if (no_init < 0 || no_init > 2) return fail(WC_ERR_INVALID_ARGUMENT, "no_init must be 0, 1 or 2");
    return table_create(0, cfg, min_capacity, seed, 0, no_init, out, memory, memory_bytes,
                        reinterpret_cast<cudaStream_t>(stream));
}

int wc_svht_create_soa(const wc_table_config *cfg, uint64_t min_capacity, uint64_t seed,
                       int no_init, wc_table **out)
{
    return table_create(0, cfg, min_capacity, seed, 0, no_init, out, nullptr, 0, nullptr, true);
}

int wc_hashset_create(const wc_table_config *cfg, uint64_t min_capacity, uint64_t seed,
                      wc_table **out)
{
    return table_create(1, cfg, min_capacity, seed, 0, 0, out);
}

int wc_counting_create(const wc_table_config *cfg, uint64_t min_capacity, uint64_t seed,
                       uint64_t max_count, int no_init, wc_table **out)
{
    return table_create(2, cfg, min_capacity, seed, max_count, no_init, out);
}

int wc_table_destroy(wc_table *t)
{
    if (!t) return WC_OK;
    if (!t->owns_memory) {
        delete t;
        return WC_OK;
    }
    if (t->slots) cudaFree(t->slots);
    if (t->fps) cudaFree(t->fps);
    if (t->values) cudaFree(t->values);
    if (t->status) cudaFree(t->status);
    if (t->scratch) cudaFree(t->scratch);
    l2_window_release(t->l2);
    delete t;
    return WC_OK;
}

int wc_table_init(wc_table *t, uint64_t seed, wc_stream_t stream)
{
    if (!t) return fail(WC_ERR_INVALID_ARGUMENT, "table is NULL");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    t->initialized = false;
    t->keys_inserted = 0;
    t->seed = seed & key_mask(t->cfg.key_bytes);
    int rc = fill_slots(t, s);
    if (rc) return rc;
    if (t->fps) WC_CUDA(cudaMemsetAsync(t->fps, kFpEmpty, t->capacity, s));
    if (t->values) WC_CUDA(cudaMemsetAsync(t->values, 0, t->capacity * t->cfg.value_bytes, s));
    WC_CUDA(cudaMemsetAsync(t->status, 0, sizeof(uint32_t), s));
    WC_CUDA(cudaMemsetAsync(t->live, 0, kLiveBytes, s));
    if (t->kind == 3) WC_CUDA(cudaMemsetAsync(t->num_keys, 0, sizeof(unsigned long long), s));
    WC_CUDA(cudaStreamSynchronize(s));
    t->initialized = true;
    return WC_OK;
}

int wc_svht_insert(wc_table *t, const void *keys_in, const void *values_in, uint64_t num_in,
                   wc_stream_t stream, uint64_t probing_length, void *status_out,
                   int status_handler, uint32_t ignore)
{
    int rc = check_table(t, 1 << 0);
    if (rc) return rc;
    return table_op(t, kOpInsert, keys_in, values_in, nullptr, num_in, stream, probing_length,
                    status_out, status_handler, ignore);
}

int wc_svht_retrieve(wc_table *t, const void *keys_in, uint64_t num_in, void *values_out,
                     wc_stream_t stream, uint64_t probing_length, void *status_out,
                     int status_handler, uint32_t ignore)
{
    int rc = check_table(t, 1 << 0);
    if (rc) return rc;
    return table_op(t, kOpRetrieve, keys_in, nullptr, values_out, num_in, stream,
                    probing_length, status_out, status_handler, ignore);
}

int wc_svht_erase(wc_table *t, const void *keys_in, uint64_t num_in, wc_stream_t stream,
                  uint64_t probing_length, void *status_out, int status_handler, uint32_t ignore)
{
    int rc = check_table(t, 1 << 0);
    if (rc) return rc;
    return table_op(t, kOpErase, keys_in, nullptr, nullptr, num_in, stream, probing_length,
                    status_out, status_handler, ignore);
}

int wc_hashset_insert(wc_table *t, const void *keys_in, uint64_t num_in, wc_stream_t stream,
                      uint64_t probing_length, void *status_out, int status_handler,
                      uint32_t ignore)
{
    int rc = check_table(t, 1 << 1);
    if (rc) return rc;
    return table_op(t, kOpInsert, keys_in, nullptr, nullptr, num_in, stream, probing_length,
                    status_out, status_handler, ignore);
}

int wc_hashset_retrieve(wc_table *t, const void *keys_in, uint64_t num_in, uint8_t *flags_out,
                        wc_stream_t stream, uint64_t probing_length, void *status_out,
                        int status_handler, uint32_t ignore)
{
    int rc = check_table(t, 1 << 1);
    if (rc) return rc;
    return table_op(t, kOpRetrieve, keys_in, nullptr, flags_out, num_in, stream,
                    probing_length, status_out, status_handler, ignore);
}

int wc_hashset_erase(wc_table *t, const void *keys_in, uint64_t num_in, wc_stream_t stream,
                     uint64_t probing_length, void *status_out, int status_handler,
                     uint32_t ignore)
{
    int rc = check_table(t, 1 << 1);
    if (rc) return rc;
    return table_op(t, kOpErase, keys_in, nullptr, nullptr, num_in, stream, probing_length,
                    status_out, status_handler, ignore);
}

int wc_counting_insert(wc_table *t, const void *keys_in, uint64_t num_in, wc_stream_t stream,
                       uint64_t probing_length, void *status_out, int status_handler,
                       uint32_t ignore)
{
    int rc = check_table(t, 1 << 2);
    if (rc) return rc;
    return table_op(t, kOpCount, keys_in, nullptr, nullptr, num_in, stream, probing_length,
                    status_out, status_handler, ignore);
}

int wc_counting_retrieve(wc_table *t, const void *keys_in, uint64_t num_in, void *values_out,
                         wc_stream_t stream, uint64_t probing_length, void *status_out,
                         int status_handler, uint32_t ignore)
{
    int rc = check_table(t, 1 << 2);
    if (rc) return rc;
    return table_op(t, kOpRetrieve, keys_in, nullptr, values_out, num_in, stream,
                    probing_length, status_out, status_handler, ignore);
}

int wc_counting_erase(wc_table *t, const void *keys_in, uint64_t num_in, wc_stream_t stream,
                      uint64_t probing_length, void *status_out, int status_handler,
                      uint32_t ignore)
{
    int rc = check_table(t, 1 << 2);
    if (rc) return rc;
    return table_op(t, kOpErase, keys_in, nullptr, nullptr, num_in, stream, probing_length,
                    status_out, status_handler, ignore);
}

int wc_table_size(wc_table *t, wc_stream_t stream, uint64_t *size_out)
{
    if (!size_out) return fail(WC_ERR_INVALID_ARGUMENT, "size_out is NULL");
    *size_out = 0;
    int rc = check_table(t, 0xF); /* every table kind */
    if (rc) return rc;
    if (t->kind == 3) return wc_table_size_scan(t, stream, size_out);
    /* the sum of the valid-key counters that claims and erases maintain */
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    unsigned long long h[kLiveStripes * kLiveStride];
    WC_CUDA(cudaMemcpyAsync(h, t->live, kLiveBytes, cudaMemcpyDeviceToHost, s));
    WC_CUDA(cudaStreamSynchronize(s));
    unsigned long long sum = 0;
    for (int i = 0; i < kLiveStripes; ++i) sum += h[i * kLiveStride];
    *size_out = sum;
    return WC_OK;
}

int wc_table_size_scan(wc_table *t, wc_stream_t stream, uint64_t *size_out)
{
    if (!size_out) return fail(WC_ERR_INVALID_ARGUMENT, "size_out is NULL");
    *size_out = 0;
    int rc = check_table(t, 0xF); /* every table kind */
    if (rc) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    CountKernel k = count_kernel(t->layout);
    WC_CUDA(cudaMemsetAsync(t->counter, 0, sizeof(unsigned long long), s));
    const uint64_t nvec = t->capacity * t->slot_bytes / 16;
    const unsigned grid = grid_for(reinterpret_cast<const void *>(k), kBlock, nvec, kBlock * 4);
    k<<<grid, kBlock, 0, s>>>(t->slots, t->capacity, t->cfg.empty_key, t->cfg.tombstone_key,
                              t->counter);
    note_launches(1);
    WC_CUDA(cudaGetLastError());
    unsigned long long h = 0;
    WC_CUDA(cudaMemcpyAsync(&h, t->counter, sizeof(h), cudaMemcpyDeviceToHost, s));
    WC_CUDA(cudaStreamSynchronize(s));
    *size_out = h;
    return WC_OK;
}

int wc_table_retrieve_all(wc_table *t, void *keys_out, void *values_out, uint64_t *num_out,
                          wc_stream_t stream)
{
    if (!num_out || !keys_out) return fail(WC_ERR_INVALID_ARGUMENT, "NULL output");
    *num_out = 0;
    int rc = check_table(t, 0xF); /* every table kind: all (key, value) pairs */
    if (rc) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    WC_CUDA(cudaMemsetAsync(t->counter, 0, sizeof(unsigned long long), s));
    if (t->soa) {
        const SoaDumpKernel k = soa_dump_kernel_ptr(t->cfg.key_bytes, t->cfg.value_bytes);
        const unsigned grid = grid_for(reinterpret_cast<const void *>(k), kBlock, t->capacity, kBlock);
        k<<<grid, kBlock, 0, s>>>(t->slots, t->values, t->capacity, t->cfg.empty_key,
                                  t->cfg.tombstone_key, keys_out, values_out, t->counter);
    } else {
        DumpKernel k = dump_kernel_ptr(t->layout);
        const unsigned grid = grid_for(reinterpret_cast<const void *>(k), kBlock, t->capacity, kBlock);
        k<<<grid, kBlock, 0, s>>>(t->slots, t->capacity, t->cfg.empty_key, t->cfg.tombstone_key,
                                  keys_out, t->kind == 1 ? nullptr : values_out, t->counter);
    }
    note_launches(1);
    WC_CUDA(cudaGetLastError());
    unsigned long long h = 0;
    WC_CUDA(cudaMemcpyAsync(&h, t->counter, sizeof(h), cudaMemcpyDeviceToHost, s));
    WC_CUDA(cudaStreamSynchronize(s));
    *num_out = h;
    return WC_OK;
}

int wc_table_peek_status(wc_table *t, wc_stream_t stream, uint32_t *out)
{
    if (!t || !out) return fail(WC_ERR_INVALID_ARGUMENT, "NULL argument");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    uint32_t h = 0;
    WC_CUDA(cudaMemcpyAsync(&h, t->status, sizeof(h), cudaMemcpyDeviceToHost, s));
    WC_CUDA(cudaStreamSynchronize(s));
    *out = t->initialized ? h : (h | WC_STATUS_NOT_INITIALIZED);
    return WC_OK;
}

int wc_table_pop_status(wc_table *t, wc_stream_t stream, uint32_t *out)
{
    int rc = wc_table_peek_status(t, stream, out);
    if (rc) return rc;
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    WC_CUDA(cudaMemsetAsync(t->status, 0, sizeof(uint32_t), s));
    WC_CUDA(cudaStreamSynchronize(s));
    return WC_OK;
}

int wc_table_get_info(const wc_table *t, wc_table_info *info)
{
    if (!t || !info) return fail(WC_ERR_INVALID_ARGUMENT, "NULL argument");
    info->kind = uint32_t(t->kind);
    info->key_bytes = t->cfg.key_bytes;
    info->value_bytes = t->cfg.value_bytes;
    info->slot_bytes = t->slot_bytes;
    info->cg_size = t->cfg.cg_size;
    info->probing = t->cfg.probing;
    info->hasher1 = t->cfg.hasher1;
    info->hasher2 = t->cfg.hasher2;
    info->capacity = t->capacity;
    info->num_buckets = t->num_buckets;
    info->seed = t->seed;
    info->empty_key = t->cfg.empty_key;
    info->tombstone_key = t->cfg.tombstone_key;
    info->max_count = t->max_count;
    info->bytes_total = t->capacity * t->slot_bytes + kAuxBytes + (t->fps ? t->capacity : 0) +
                        (t->soa ? t->capacity * t->cfg.value_bytes : 0);
    info->slots = t->slots;
    info->status = t->status;
    info->is_initialized = t->initialized ? 1 : 0;
    info->fingerprints = t->fps;
    info->num_keys = t->kind == 3 ? t->num_keys : nullptr;
    info->max_values_per_key = t->max_values;
    info->live = t->kind == 3 ? nullptr : t->live;
    info->values = t->values;
    return WC_OK;
}

/* ---- MultiValueHashTable (multi_value_hash_table.cuh) ---- */

int wc_mvht_create(const wc_table_config *cfg, uint64_t min_capacity, uint64_t seed,
                   uint64_t max_values_per_key, int no_init, wc_table **out)
{
    if (max_values_per_key == 0)
        return fail(WC_ERR_INVALID_ARGUMENT, "max_values_per_key must be at least 1");
    int rc = table_create(3, cfg, min_capacity, seed, 0, 1, out);
    if (rc) return rc;
    (*out)->max_values = max_values_per_key;
    if (!no_init) {
        rc = wc_table_init(*out, (*out)->seed, nullptr);
        if (rc) {
            wc_table_destroy(*out);
            *out = nullptr;
            return rc;
        }
    }
    return WC_OK;
}

namespace {

MvArgs mv_args(wc_table *t, const void *keys, uint64_t n, uint64_t probing_length, bool find,
               void *status_out, int handler, uint32_t ignore)
{
    MvArgs a{};
    a.t = view_of(t);
    a.keys = keys;
    a.n = n;
    /* for_each caps the probing length at the capacity (:623) */
    const uint64_t pl = find && probing_length > t->capacity ? t->capacity : probing_length;
    a.max_windows = max_windows(pl, t->cfg.cg_size, t->num_buckets);
    a.max_values = t->max_values;
    a.status_out = handler == WC_HANDLER_NOTHING ? nullptr : status_out;
    a.handler = handler;
    a.bool_mask = (~ignore) ^ 0xFFFu;
    return a;
}

int mv_launch(const void *k, wc_table *t, uint64_t items, MvArgs &a, cudaStream_t s)
{
    void *args[] = {&a};
    const unsigned grid = grid_for(k, kBlock, items, kBlock);
    WC_CUDA(cudaLaunchKernel(k, dim3(grid), dim3(kBlock), args, 0, s));
    note_launches(1);
    return WC_OK;
}

/* per-key counts (and their sum, read back to the host) */
int mv_count(wc_table *t, const void *keys, uint64_t n, uint64_t *counts_dev, uint64_t *total,
             cudaStream_t s, uint64_t probing_length, void *status_out, int handler,
             uint32_t ignore)
{
    const MvKernels k = mv_kernels(t->layout, int(t->cfg.cg_size));
    if (!k.count) return fail(WC_ERR_UNSUPPORTED, "no kernel for this configuration");
    WC_CUDA(cudaMemsetAsync(t->counter, 0, sizeof(unsigned long long), s));
    MvArgs a = mv_args(t, keys, n, probing_length, true, status_out, handler, ignore);
    a.counts_out = reinterpret_cast<unsigned long long *>(counts_dev);
    a.total = t->counter;
    int rc = mv_launch(k.count, t, n, a, s);
    if (rc) return rc;
    unsigned long long h = 0;
    WC_CUDA(cudaMemcpyAsync(&h, t->counter, sizeof(h), cudaMemcpyDeviceToHost, s));
    WC_CUDA(cudaStreamSynchronize(s));
    *total = h;
    return WC_OK;
}

/* counts in end -> end = inclusive prefix sums, begin = exclusive ones */
int mv_scan(wc_table *t, uint64_t *begin, uint64_t *end, uint64_t n, cudaStream_t s)
{
    return host_offsets_scan(&t->scratch, &t->scratch_bytes, begin, end, n, s);
}

int mv_join(wc_table *t, uint32_t bits, cudaStream_t s)
{
    return host_join_status(t->status, bits, s);
}

} // namespace

int wc_mvht_insert(wc_table *t, const void *keys_in, const void *values_in, uint64_t num_in,
                   wc_stream_t stream, uint64_t probing_length, void *status_out,
                   int status_handler, uint32_t ignore)
{
    int rc = check_table(t, 1 << 3);
    if (rc) return rc;
    if (num_in == 0) return WC_OK;
    if (!keys_in || !values_in) return fail(WC_ERR_INVALID_ARGUMENT, "keys_in / values_in is NULL");
    const MvKernels k = mv_kernels(t->layout, int(t->cfg.cg_size));
    if (!k.insert) return fail(WC_ERR_UNSUPPORTED, "no kernel for this configuration");
    MvArgs a = mv_args(t, keys_in, num_in, probing_length, false, status_out, status_handler,
                       ignore);
    a.values = values_in;
    a.num_keys = t->num_keys;
    return mv_launch(k.insert, t, num_in, a, reinterpret_cast<cudaStream_t>(stream));
}

int wc_mvht_num_values(wc_table *t, const void *keys_in, uint64_t num_in, uint64_t *num_out,
                       uint64_t *num_per_key_out, wc_stream_t stream, uint64_t probing_length,
                       void *status_out, int status_handler, uint32_t ignore)
{
    int rc = check_table(t, 1 << 3);
    if (rc) return rc;
    if (!num_out) return fail(WC_ERR_INVALID_ARGUMENT, "num_out is NULL");
    *num_out = 0;
    if (num_in == 0) return WC_OK;
    if (!keys_in) return fail(WC_ERR_INVALID_ARGUMENT, "keys_in is NULL");
    return mv_count(t, keys_in, num_in, num_per_key_out, num_out,
                    reinterpret_cast<cudaStream_t>(stream), probing_length, status_out,
                    status_handler, ignore);
}

int wc_mvht_retrieve(wc_table *t, const void *keys_in, uint64_t num_in,
                     uint64_t *begin_offsets_out, uint64_t *end_offsets_out, void *values_out,
                     uint64_t *num_out, wc_stream_t stream, uint64_t probing_length,
                     void *status_out, int status_handler, uint32_t ignore)
{
    int rc = check_table(t, 1 << 3);
    if (rc) return rc;
    if (!num_out) return fail(WC_ERR_INVALID_ARGUMENT, "num_out is NULL");
    *num_out = 0;
    if (num_in == 0) return WC_OK;
    if (!keys_in || !end_offsets_out || (values_out && !begin_offsets_out))
        return fail(WC_ERR_INVALID_ARGUMENT, "NULL buffer");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    /* pass 1: counts per key into end_offsets, and each key's status (the
     * values pass reads values only) */
    rc = mv_count(t, keys_in, num_in, end_offsets_out, num_out, s, probing_length,
                  values_out ? status_out : nullptr,
                  values_out ? status_handler : WC_HANDLER_NOTHING, ignore);
    if (rc) return rc;
    if (!values_out) {
        /* dry run: per-key counts, status dry_run for every key */
        rc = host_dry_run_status(status_out, num_in, status_handler, ignore, s);
        if (rc) return rc;
        return mv_join(t, kStDryRun, s);
    }
    /* pass 2: offsets; pass 3: values, each key at its begin offset */
    rc = mv_scan(t, begin_offsets_out, end_offsets_out, num_in, s);
    if (rc) return rc;
    const MvKernels k = mv_kernels(t->layout, int(t->cfg.cg_size));
    MvArgs a = mv_args(t, keys_in, num_in, probing_length, true, status_out, status_handler,
                       ignore);
    a.values_out = values_out;
    a.begin = reinterpret_cast<const unsigned long long *>(begin_offsets_out);
    a.end = reinterpret_cast<const unsigned long long *>(end_offsets_out);
    return mv_launch(k.values, t, num_in, a, s);
}

int wc_mvht_retrieve_all_keys(wc_table *t, void *keys_out, uint64_t *num_out, wc_stream_t stream)
{
    int rc = check_table(t, 1 << 3);
    if (rc) return rc;
    if (!num_out) return fail(WC_ERR_INVALID_ARGUMENT, "num_out is NULL");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    if (!keys_out) {
        rc = wc_mvht_num_keys(t, stream, num_out);
        if (rc) return rc;
        return mv_join(t, kStDryRun, s);
    }
    const MvKernels k = mv_kernels(t->layout, int(t->cfg.cg_size));
    if (!k.unique) return fail(WC_ERR_UNSUPPORTED, "no kernel for this configuration");
    WC_CUDA(cudaMemsetAsync(t->counter, 0, sizeof(unsigned long long), s));
    TableView v = view_of(t);
    uint64_t cap = t->capacity;
    unsigned long long *cnt = t->counter;
    void *args[] = {&v, &cap, &keys_out, &cnt};
    WC_CUDA(cudaLaunchKernel(k.unique, dim3(grid_for(k.unique, kBlock, cap, kBlock)), dim3(kBlock),
                             args, 0, s));
    note_launches(1);
    unsigned long long h = 0;
    WC_CUDA(cudaMemcpyAsync(&h, t->counter, sizeof(h), cudaMemcpyDeviceToHost, s));
    WC_CUDA(cudaStreamSynchronize(s));
    *num_out = h;
    return WC_OK;
}

int wc_mvht_num_keys(wc_table *t, wc_stream_t stream, uint64_t *out)
{
    int rc = check_table(t, 1 << 3);
    if (rc) return rc;
    if (!out) return fail(WC_ERR_INVALID_ARGUMENT, "out is NULL");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    unsigned long long h = 0;
    WC_CUDA(cudaMemcpyAsync(&h, t->num_keys, sizeof(h), cudaMemcpyDeviceToHost, s));
    WC_CUDA(cudaStreamSynchronize(s));
    *out = h;
    return WC_OK;
}

int wc_launch_count(uint64_t *out)
{
    if (!out) return fail(WC_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = g_launches.load(std::memory_order_relaxed);
    return WC_OK;
}

int wc_fingerprint_ops(uint32_t op_mask, uint32_t *previous)
{
    const uint32_t prev = g_fp_ops.exchange(op_mask & 0x3Fu);
    if (previous) *previous = prev;
    return WC_OK;
}

int wc_lane_ops(uint32_t op_mask, uint32_t *previous)
{
    const uint32_t prev = g_lane_ops.exchange(op_mask & 0xDu);
    if (previous) *previous = prev;
    return WC_OK;
}

int wc_fingerprint_policy(int mode, int *previous)
{
    if (mode != WC_FINGERPRINTS_AUTO && mode != WC_FINGERPRINTS_ALWAYS &&
        mode != WC_FINGERPRINTS_NEVER)
        return fail(WC_ERR_INVALID_ARGUMENT, "unknown fingerprint policy %d", mode);
    const int prev = fp_mode();
    g_fp_mode.store(mode);
    if (previous) *previous = prev;
    return WC_OK;
}

int wc_region_bytes(int op, uint64_t bytes, uint64_t *previous)
{
    if (op != WC_REGION_INSERT && op != WC_REGION_QUERY)
        return fail(WC_ERR_INVALID_ARGUMENT, "unknown region operation %d", op);
    if (bytes && (bytes < (1ull << 20) || bytes > (1ull << 40)))
        return fail(WC_ERR_INVALID_ARGUMENT, "region must be 0 (one pass) or 1 MiB .. 1 TiB");
    const uint64_t prev = g_region_bytes[op == WC_REGION_INSERT ? 0 : 1].exchange(bytes);
    if (previous) *previous = prev;
    return WC_OK;
}

/* ---- launch tuning ---- */

int wc_l2_persistence(int enable, int *previous)
{
    const int prev = g_l2_mode.exchange(enable ? 1 : 0);
    if (previous) *previous = prev;
    return WC_OK;
}

int wc_table_l2_window(const wc_table *t, uint64_t *bytes_out, float *hit_ratio_out)
{
    if (!t || !bytes_out) return fail(WC_ERR_INVALID_ARGUMENT, "NULL argument");
    const bool on = g_l2_mode.load() != 0;
    *bytes_out = on ? t->l2.bytes : 0;
    if (hit_ratio_out) *hit_ratio_out = on ? t->l2.hit_ratio : 0.f;
    return WC_OK;
}

int wc_tune_set(uint32_t key_bytes, int op, uint32_t load_bucket, uint32_t size_bucket,
                uint32_t block_threads, uint32_t blocks_per_sm_)
{
    if ((key_bytes != 4 && key_bytes != 8) || op < 0 || op > 3 || load_bucket >= uint32_t(kTuneLoads) ||
        size_bucket >= uint32_t(kTuneSizes))
        return fail(WC_ERR_INVALID_ARGUMENT, "tuning key out of range");
    if (block_threads && (block_threads % 32 || block_threads > 256))
        return fail(WC_ERR_INVALID_ARGUMENT, "block_threads must be a multiple of 32, at most 256");
    std::lock_guard<std::mutex> lock(g_tune_mu);
    g_tune[key_bytes == 8][op][load_bucket][size_bucket] = TuneEntry{block_threads, blocks_per_sm_};
    return WC_OK;
}

/* Reads the "entries" array of a tuning file written by
 * warpcore_b200.autotune: [[key_bytes, op, load_bucket, size_bucket,
 * block_threads, blocks_per_sm], ...].  Only that array is parsed: numbers
 * in brackets after the "entries" key, six per entry. */
int wc_tune_load(const char *path, uint64_t *loaded)
{
    std::string file;
    if (path) {
        file = path;
    } else if (const char *env = std::getenv("WARPCORE_B200_TUNING")) {
        file = env;
    } else {
        /* tuning_b200.json next to this library */
        Dl_info info;
        if (!dladdr(reinterpret_cast<void *>(&wc_tune_load), &info) || !info.dli_fname)
            return fail(WC_ERR_INVALID_ARGUMENT, "cannot locate the library");
        file = info.dli_fname;
        const size_t slash = file.rfind('/');
        file = (slash == std::string::npos ? std::string(".") : file.substr(0, slash)) +
               "/tuning_b200.json";
    }
    if (loaded) *loaded = 0;
    if (file == "none") return WC_OK;
    FILE *f = std::fopen(file.c_str(), "rb");
    if (!f) return fail(WC_ERR_INVALID_ARGUMENT, "cannot open tuning file %s", file.c_str());
    std::string text;
    char buf[65536];
    size_t got;
    while ((got = std::fread(buf, 1, sizeof buf, f)) > 0) text.append(buf, got);
    std::fclose(f);
    size_t pos = text.find("\"entries\"");
    if (pos == std::string::npos) return fail(WC_ERR_INVALID_ARGUMENT, "no entries in %s", file.c_str());
    pos = text.find('[', pos);
    if (pos == std::string::npos) return fail(WC_ERR_INVALID_ARGUMENT, "malformed %s", file.c_str());
    ++pos; /* inside the outer array */
    uint64_t n = 0;
    for (;;) {
        while (pos < text.size() && (text[pos] == ' ' || text[pos] == '\n' || text[pos] == '\r' ||
                                     text[pos] == '\t' || text[pos] == ','))
            ++pos;
        if (pos >= text.size()) return fail(WC_ERR_INVALID_ARGUMENT, "malformed %s", file.c_str());
        if (text[pos] == ']') break;
        if (text[pos] != '[') return fail(WC_ERR_INVALID_ARGUMENT, "malformed %s", file.c_str());
        ++pos;
        unsigned long long v[6];
        for (int i = 0; i < 6; ++i) {
            while (pos < text.size() && (text[pos] == ' ' || text[pos] == ',' || text[pos] == '\n'))
                ++pos;
            char *end = nullptr;
            v[i] = std::strtoull(text.c_str() + pos, &end, 10);
            if (end == text.c_str() + pos)
                return fail(WC_ERR_INVALID_ARGUMENT, "malformed entry in %s", file.c_str());
            pos = size_t(end - text.c_str());
        }
        pos = text.find(']', pos);
        if (pos == std::string::npos) return fail(WC_ERR_INVALID_ARGUMENT, "malformed %s", file.c_str());
        ++pos;
        const int rc = wc_tune_set(uint32_t(v[0]), int(v[1]), uint32_t(v[2]), uint32_t(v[3]),
                                   uint32_t(v[4]), uint32_t(v[5]));
        if (rc) return rc;
        ++n;
    }
    if (loaded) *loaded = n;
    return WC_OK;
}

int wc_tune_reset(void)
{
    std::lock_guard<std::mutex> lock(g_tune_mu);
    for (auto &a : g_tune)
        for (auto &b : a)
            for (auto &c : b)
                for (auto &e : c) e = TuneEntry{};
    return WC_OK;
}

/* ---- Bloom filter ---- */

/* shape of the whole filter, and the blocks [lo, hi) that this object holds
 * (shard s of S holds the blocks b with b * S / num_blocks == s) */
static int bloom_new(const wc_bloom_config *cfg, uint64_t num_bits, uint64_t k, uint64_t seed,
                     uint32_t shard, uint32_t num_shards, wc_bloom **out)
{
    if (!out || !cfg) return fail(WC_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    if (cfg->key_bytes != 4 && cfg->key_bytes != 8)
        return fail(WC_ERR_UNSUPPORTED, "key_bytes must be 4 or 8");
    if (cfg->slot_bytes != 4 && cfg->slot_bytes != 8)
        return fail(WC_ERR_UNSUPPORTED, "slot_bytes must be 4 or 8");
    if (!valid_cg(cfg->cg_size)) return fail(WC_ERR_INVALID_ARGUMENT, "bad cg_size");
    if (cfg->hasher > WC_HASH_IDENTITY64) return fail(WC_ERR_INVALID_ARGUMENT, "unknown hasher");
    if (num_bits == 0) return fail(WC_ERR_INVALID_ARGUMENT, "num_bits must be positive");
    if (num_shards == 0 || shard >= num_shards)
        return fail(WC_ERR_INVALID_ARGUMENT, "shard %u of %u", shard, num_shards);
    const uint64_t slot_bits = uint64_t(cfg->slot_bytes) * 8;
    const uint64_t num_slots = (num_bits + slot_bits - 1) / slot_bits;
    if (num_shards > 1) {
        if (cfg->cg_size * cfg->slot_bytes > 128)
            return fail(WC_ERR_UNSUPPORTED, "sharded filters take blocks of at most 128 bytes");
        if (num_slots % cfg->cg_size)
            return fail(WC_ERR_UNSUPPORTED,
                        "sharded filters take whole blocks (num_bits a multiple of the block bits)");
    }
    auto *b = new wc_bloom();
    b->cfg = *cfg;
    b->num_bits = num_bits;
    b->num_slots = num_slots;
    b->num_blocks = (num_slots + cfg->cg_size - 1) / cfg->cg_size;
    b->k = k;
    b->seed = seed & key_mask(cfg->key_bytes);
    const uint64_t nb = b->num_blocks, S = num_shards;
    b->block_base = (uint64_t(shard) * nb + S - 1) / S;
    b->local_blocks = ((uint64_t(shard) + 1) * nb + S - 1) / S - b->block_base;
    cudaGetDevice(&b->device);
    /* padded to whole blocks so that full-block vector loads stay inside */
    const uint64_t bytes =
        (b->local_blocks ? b->local_blocks : 1) * cfg->cg_size * cfg->slot_bytes;
    cudaError_t e = cudaMalloc(&b->words, bytes);
    if (e != cudaSuccess) {
        delete b;
        return cuda_fail(e, "cudaMalloc");
    }
    b->l2 = l2_window_for(b->words, bytes);
    int rc = wc_bloom_init(b, b->seed, nullptr);
    if (rc) {
        wc_bloom_destroy(b);
        return rc;
    }
    *out = b;
    return WC_OK;
}

int wc_bloom_create(const wc_bloom_config *cfg, uint64_t num_bits, uint64_t k, uint64_t seed,
                    wc_bloom **out)
{
    return bloom_new(cfg, num_bits, k, seed, 0, 1, out);
}

int wc_bloom_create_shard(const wc_bloom_config *cfg, uint64_t num_bits, uint64_t k,
                          uint64_t seed, uint32_t shard, uint32_t num_shards, wc_bloom **out)
{
    return bloom_new(cfg, num_bits, k, seed, shard, num_shards, out);
}

int wc_bloom_partition(const wc_bloom *b, const void *keys, uint64_t n, uint32_t num_parts,
                       void *keys_out, uint64_t *perm_out, uint64_t *counts_out,
                       uint64_t *scratch, wc_stream_t stream)
{
    if (!b) return fail(WC_ERR_INVALID_ARGUMENT, "filter is NULL");
    return partition_by_bloom_block(keys, n, b->cfg.key_bytes, num_parts, b->seed, b->cfg.hasher,
                                    b->num_blocks, keys_out, perm_out, counts_out, scratch, stream);
}

int wc_bloom_destroy(wc_bloom *b)
{
    if (!b) return WC_OK;
    if (b->words) cudaFree(b->words);
    l2_window_release(b->l2);
    delete b;
    return WC_OK;
}

int wc_bloom_init(wc_bloom *b, uint64_t seed, wc_stream_t stream)
{
    if (!b) return fail(WC_ERR_INVALID_ARGUMENT, "filter is NULL");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    b->seed = seed & key_mask(b->cfg.key_bytes);
    const uint64_t bytes = b->local_blocks * b->cfg.cg_size * b->cfg.slot_bytes;
    WC_CUDA(cudaMemsetAsync(b->words, 0, bytes, s));
    WC_CUDA(cudaStreamSynchronize(s));
    return WC_OK;
}

static int bloom_op(wc_bloom *b, const void *keys, uint64_t n, uint8_t *flags, wc_stream_t stream,
                    bool insert)
{
    if (!b) return fail(WC_ERR_INVALID_ARGUMENT, "filter is NULL");
    if (n == 0) return WC_OK;
    if (!keys) return fail(WC_ERR_INVALID_ARGUMENT, "keys_in is NULL");
    if (!insert && !flags) return fail(WC_ERR_INVALID_ARGUMENT, "flags_out is NULL");
    /* a filter whose words outgrow one random-access region runs in region
     * passes (bloom_lane_kernel): pass r serves the keys of blocks
     * [r * local_blocks / R, (r + 1) * local_blocks / R) */
    const uint64_t block_bytes = uint64_t(b->cfg.cg_size) * b->cfg.slot_bytes;
    const uint64_t fbytes = b->local_blocks * block_bytes;
    const uint64_t rb = region_bytes(insert);
    uint64_t passes = rb ? (fbytes + rb - 1) / rb : 1;
    if (passes < 1) passes = 1;
    /* the region kernel keeps a block's offset in its region in 32 bits */
    const uint64_t min_passes = (b->local_blocks >> 31) + 1;
    if (passes > 1 && passes < min_passes) passes = min_passes;
    bool lane = false;
    BloomKernel k = bloom_kernel_ptr(int(b->cfg.key_bytes), int(b->cfg.slot_bytes),
                                     int(b->cfg.cg_size), insert, passes > 1, &lane);
    if (!k) return fail(WC_ERR_UNSUPPORTED, "no kernel for this configuration");
    if (!lane) passes = 1;
    BloomArgs a;
    a.words = b->words;
    a.keys = keys;
    a.flags_out = flags;
    a.n = n;
    a.num_slots = b->num_slots;
    a.num_blocks = b->num_blocks;
    a.magic_blocks = barrett_magic(b->num_blocks);
    a.k = b->k;
    a.seed = b->seed;
    a.hasher = b->cfg.hasher;
    a.block_base = b->block_base;
    a.local_blocks = b->local_blocks;
    const unsigned grid = grid_for(reinterpret_cast<const void *>(k), kBlock, n, kBlock);
    void *args[] = {&a};
    for (uint64_t r = 0; r < passes; ++r) {
        a.region_lo = r * b->local_blocks / passes;
        a.region_hi = (r + 1) * b->local_blocks / passes; /* local_blocks for the last */
        WC_CUDA(launch_in_window(reinterpret_cast<const void *>(k), grid, kBlock, args,
                                 reinterpret_cast<cudaStream_t>(stream), b->l2));
    }
    return WC_OK;
}

int wc_bloom_insert(wc_bloom *b, const void *keys_in, uint64_t num_in, wc_stream_t stream)
{
    return bloom_op(b, keys_in, num_in, nullptr, stream, true);
}

int wc_bloom_retrieve(wc_bloom *b, const void *keys_in, uint64_t num_in, uint8_t *flags_out,
                      wc_stream_t stream)
{
    return bloom_op(b, keys_in, num_in, flags_out, stream, false);
}

int wc_bloom_get_info(const wc_bloom *b, wc_bloom_info *info)
{
    if (!b || !info) return fail(WC_ERR_INVALID_ARGUMENT, "NULL argument");
    info->key_bytes = b->cfg.key_bytes;
    info->slot_bytes = b->cfg.slot_bytes;
    info->cg_size = b->cfg.cg_size;
    info->hasher = b->cfg.hasher;
    info->num_bits = b->num_bits;
    info->num_slots = b->num_slots;
    info->num_blocks = b->num_blocks;
    info->block_base = b->block_base;
    info->local_blocks = b->local_blocks;
    info->k = b->k;
    info->seed = b->seed;
    info->words = b->words;
    return WC_OK;
}

/* the reference's analytic estimate, bloom_filter.cuh:342-408, in the same
 * double arithmetic (it overflows to NaN for very large filters, as the
 * reference does) */
int wc_bloom_fpr(const wc_bloom *b, uint64_t n, double *out)
{
    if (!b || !out) return fail(WC_ERR_INVALID_ARGUMENT, "NULL argument");
    const uint64_t block_bits = uint64_t(b->cfg.slot_bytes) * 8 * b->cfg.cg_size;
    const uint64_t nblocks_int = b->num_bits / block_bits;
    if (nblocks_int == 0) return fail(WC_ERR_INVALID_ARGUMENT, "filter smaller than one block");
    const double bl = double(nblocks_int);
    double res = 0.0;
    const uint64_t upper = 5 * n / nblocks_int;
    const uint64_t m = uint64_t(double(b->num_bits) / bl);
    for (uint64_t i = 0; i < upper; ++i) {
        double binom = 1.0;
        for (uint64_t j = n - i + 1; j <= n; ++j) binom *= double(j);
        for (uint64_t j = 1; j <= i; ++j) binom /= double(j);
        binom *= std::pow(1.0 / bl, double(i)) * std::pow(1.0 - 1.0 / bl, double(n - i));
        const double base = std::pow(1.0 - std::pow(1.0 - 1.0 / double(m), double(i * b->k)),
                                     double(b->k));
        res += binom * base;
    }
    *out = res;
    return WC_OK;
}

} // extern "C"

/* ------------------------------------------------------------------ */
/* Bulk operations on host buffers, pipelined through device staging     */
/* ------------------------------------------------------------------ */

struct wc_host_pipe {
    int device = 0;
    uint64_t chunk = 0;             /* keys per chunk */
    uint32_t depth = 0;             /* staging slots */
    char *stage = nullptr;          /* depth x (chunk x 8 keys | chunk x 8 values/outputs) */
    cudaStream_t h2d = nullptr, d2h = nullptr;
    std::vector<cudaEvent_t> in_done, kern_done, slot_free;
    cudaEvent_t call_start = nullptr; /* the caller's stream at entry */
    std::vector<char> used;
    uint32_t next = 0;
};

namespace {

int host_pipe_destroy(wc_host_pipe *p);

} // namespace

extern "C" int wc_host_pipe_create(uint64_t chunk_keys, uint32_t depth, wc_host_pipe **out)
{
    if (!out) return fail(WC_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    if (chunk_keys == 0) chunk_keys = uint64_t(1) << 22;
    if (depth == 0) depth = 3;
    if (depth > 64) return fail(WC_ERR_INVALID_ARGUMENT, "depth must be 1 .. 64");
    if (chunk_keys > (uint64_t(1) << 30)) return fail(WC_ERR_INVALID_ARGUMENT, "chunk_keys > 2^30");
    auto *p = new wc_host_pipe();
    cudaGetDevice(&p->device);
    p->chunk = chunk_keys;
    p->depth = depth;
    cudaError_t e = cudaMalloc(&p->stage, size_t(depth) * chunk_keys * 16);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->h2d, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->d2h, cudaStreamNonBlocking);
    p->in_done.assign(depth, nullptr);
    p->kern_done.assign(depth, nullptr);
    p->slot_free.assign(depth, nullptr);
    p->used.assign(depth, 0);
    if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->call_start, cudaEventDisableTiming);
    for (uint32_t i = 0; i < depth && e == cudaSuccess; ++i) {
        e = cudaEventCreateWithFlags(&p->in_done[i], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->kern_done[i], cudaEventDisableTiming);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&p->slot_free[i], cudaEventDisableTiming);
    }
    if (e != cudaSuccess) {
        host_pipe_destroy(p);
        return cuda_fail(e, "wc_host_pipe_create");
    }
    *out = p;
    return WC_OK;
}

extern "C" int wc_host_pipe_destroy(wc_host_pipe *p)
{
    return host_pipe_destroy(p);
}

namespace {

int host_pipe_destroy(wc_host_pipe *p)
{
    if (!p) return WC_OK;
    if (p->h2d) cudaStreamSynchronize(p->h2d);
    if (p->d2h) cudaStreamSynchronize(p->d2h);
    for (uint32_t i = 0; i < p->depth; ++i) {
        if (p->slot_free[i]) cudaEventSynchronize(p->slot_free[i]);
        if (p->in_done[i]) cudaEventDestroy(p->in_done[i]);
        if (p->kern_done[i]) cudaEventDestroy(p->kern_done[i]);
        if (p->slot_free[i]) cudaEventDestroy(p->slot_free[i]);
    }
    if (p->call_start) cudaEventDestroy(p->call_start);
    if (p->h2d) cudaStreamDestroy(p->h2d);
    if (p->d2h) cudaStreamDestroy(p->d2h);
    if (p->stage) cudaFree(p->stage);
    delete p;
    return WC_OK;
}

uint32_t out_bytes_of(const wc_table *t)
{
    return t->kind == 1 ? 1u : t->cfg.value_bytes;
}

int host_op(wc_host_pipe *p, wc_table *t, bool insert, const void *h_keys, const void *h_values,
            void *h_out, const void *miss_fill, uint64_t n, wc_stream_t stream,
            uint64_t probing_length)
{
    if (!p) return fail(WC_ERR_INVALID_ARGUMENT, "pipe is NULL");
    int rc = check_table(t, 0x7);
    if (rc) return rc;
    if (n == 0) return WC_OK;
    if (!h_keys) return fail(WC_ERR_INVALID_ARGUMENT, "keys_in is NULL");
    if (insert && t->kind == 0 && !h_values) return fail(WC_ERR_INVALID_ARGUMENT, "values_in is NULL");
    if (!insert && !h_out) return fail(WC_ERR_INVALID_ARGUMENT, "output is NULL");
    cudaStream_t s = reinterpret_cast<cudaStream_t>(stream);
    const uint32_t kb = t->cfg.key_bytes;
    const uint32_t vb = t->cfg.value_bytes;
    const uint32_t ob = out_bytes_of(t);
    /* sets write a flag for every key; single-value and counting tables
     * write hits only, so a miss keeps the output's earlier content: copied
     * in with the keys, or `miss_fill` */
    const bool hits_only = !insert && t->kind != 1;
    const int op = insert ? (t->kind == 2 ? kOpCount : kOpInsert) : kOpRetrieve;
    const char *hk = static_cast<const char *>(h_keys);
    const char *hv = static_cast<const char *>(h_values);
    char *ho = static_cast<char *>(h_out);
    std::vector<char> touched(p->depth, 0);
    /* stream order: no copy of this call starts before the caller's
     * earlier work on `stream` (which may have written the host inputs) */
    WC_CUDA(cudaEventRecord(p->call_start, s));
    WC_CUDA(cudaStreamWaitEvent(p->h2d, p->call_start, 0));
    for (uint64_t off = 0; off < n; off += p->chunk) {
        const uint64_t m = n - off < p->chunk ? n - off : p->chunk;
        const uint32_t slot = p->next;
        p->next = (p->next + 1) % p->depth;
        char *dk = p->stage + size_t(slot) * p->chunk * 16;
        char *dv = dk + p->chunk * 8;
        if (p->used[slot]) WC_CUDA(cudaStreamWaitEvent(p->h2d, p->slot_free[slot], 0));
        WC_CUDA(cudaMemcpyAsync(dk, hk + off * kb, m * kb, cudaMemcpyHostToDevice, p->h2d));
        if (insert && t->kind == 0)
            WC_CUDA(cudaMemcpyAsync(dv, hv + off * vb, m * vb, cudaMemcpyHostToDevice, p->h2d));
        if (hits_only && !miss_fill)
            WC_CUDA(cudaMemcpyAsync(dv, ho + off * ob, m * ob, cudaMemcpyHostToDevice, p->h2d));
        WC_CUDA(cudaEventRecord(p->in_done[slot], p->h2d));
        WC_CUDA(cudaStreamWaitEvent(s, p->in_done[slot], 0));
        if (hits_only && miss_fill) {
            uint32_t w[4];
            if (ob == 4) {
                std::memcpy(&w[0], miss_fill, 4);
                w[1] = w[2] = w[3] = w[0];
            } else {
                std::memcpy(&w[0], miss_fill, 8);
                w[2] = w[0];
                w[3] = w[1];
            }
            uint32_t *fp = reinterpret_cast<uint32_t *>(dv);
            uint64_t fn = m * ob / 4;
            uint4 pat = make_uint4(w[0], w[1], w[2], w[3]);
            void *fargs[] = {&fp, &fn, &pat};
            const void *fk = reinterpret_cast<const void *>(fill_kernel<0>);
            WC_CUDA(cudaLaunchKernel(fk, dim3(grid_for(fk, kBlock, fn / 4, kBlock)), dim3(kBlock),
                                     fargs, 0, s));
            note_launches(1);
        }
        rc = table_op(t, op, dk, insert ? dv : nullptr, insert ? nullptr : dv, m, stream,
                      probing_length, nullptr, WC_HANDLER_NOTHING, 0);
        if (rc) return rc;
        if (insert) {
            WC_CUDA(cudaEventRecord(p->slot_free[slot], s));
        } else {
            WC_CUDA(cudaEventRecord(p->kern_done[slot], s));
            WC_CUDA(cudaStreamWaitEvent(p->d2h, p->kern_done[slot], 0));
            WC_CUDA(cudaMemcpyAsync(ho + off * ob, dv, m * ob, cudaMemcpyDeviceToHost, p->d2h));
            WC_CUDA(cudaEventRecord(p->slot_free[slot], p->d2h));
        }
        p->used[slot] = 1;
        touched[slot] = 1;
    }
    /* the caller's stream passes this call only when every copy-out is done */
    if (!insert)
        for (uint32_t i = 0; i < p->depth; ++i)
            if (touched[i]) WC_CUDA(cudaStreamWaitEvent(s, p->slot_free[i], 0));
    return WC_OK;
}

} // namespace

extern "C" {

int wc_table_insert_host(wc_host_pipe *p, wc_table *t, const void *h_keys, const void *h_values,
                         uint64_t num_in, wc_stream_t stream, uint64_t probing_length)
{
    return host_op(p, t, true, h_keys, h_values, nullptr, nullptr, num_in, stream, probing_length);
}

int wc_table_retrieve_host(wc_host_pipe *p, wc_table *t, const void *h_keys, uint64_t num_in,
                           void *h_out, const void *miss_fill, wc_stream_t stream,
                           uint64_t probing_length)
{
    return host_op(p, t, false, h_keys, nullptr, h_out, miss_fill, num_in, stream, probing_length);
}

} // extern "C"

/* ------------------------------------------------------------------ */
/* batches (wc_batch.cuh)                                                */
/* ------------------------------------------------------------------ */

struct wc_batch {
    uint32_t max_requests = 0;
    uint32_t depth = 0;
    uint32_t next = 0;
    struct Slot {
        BatchDesc *host = nullptr; /* pinned */
        BatchDesc *dev = nullptr;
        cudaEvent_t done = nullptr;
        bool used = false;
        /* one instantiated graph per (kernel, grid) seen on this slot */
        const void *kernel = nullptr;
        unsigned grid = 0;
        cudaGraph_t graph = nullptr;
        cudaGraphExec_t exec = nullptr;
        cudaGraphNode_t copy_node = nullptr, kernel_node = nullptr;
        BatchInlineArgs *inline_args = nullptr; /* host copy of small-batch parameters */
    };
    std::vector<Slot> slots;
};

namespace {

void release_graph(wc_batch::Slot &s)
{
    if (s.exec) cudaGraphExecDestroy(s.exec);
    if (s.graph) cudaGraphDestroy(s.graph);
    s.exec = nullptr;
    s.graph = nullptr;
    s.kernel = nullptr;
}

/* graph of one staging slot: [descriptor copy ->] batch kernel */
int build_graph(wc_batch::Slot &s, const void *kernel, unsigned grid, void *args, size_t bytes)
{
    release_graph(s);
    WC_CUDA(cudaGraphCreate(&s.graph, 0));
    const bool with_copy = bytes != 0;
    if (with_copy)
        WC_CUDA(cudaGraphAddMemcpyNode1D(&s.copy_node, s.graph, nullptr, 0, s.dev, s.host, bytes,
                                         cudaMemcpyHostToDevice));
    else
        s.copy_node = nullptr;
    cudaKernelNodeParams kp{};
    void *kargs[] = {args};
    kp.func = const_cast<void *>(kernel);
    kp.gridDim = dim3(grid);
    kp.blockDim = dim3(kBlock);
    kp.sharedMemBytes = 0;
    kp.kernelParams = kargs;
    WC_CUDA(cudaGraphAddKernelNode(&s.kernel_node, s.graph, with_copy ? &s.copy_node : nullptr,
                                   with_copy ? 1 : 0, &kp));
    WC_CUDA(cudaGraphInstantiate(&s.exec, s.graph, 0));
    s.kernel = kernel;
    s.grid = grid;
    return WC_OK;
}

} // namespace

extern "C" {

int wc_batch_create(uint32_t max_requests, uint32_t depth, wc_batch **out)
{
    if (!out || max_requests == 0) return fail(WC_ERR_INVALID_ARGUMENT, "bad batch arguments");
    *out = nullptr;
    if (depth == 0) depth = 2;
    auto *b = new wc_batch();
    b->max_requests = max_requests;
    b->depth = depth;
    b->slots.resize(depth);
    for (auto &s : b->slots) {
        cudaError_t e = cudaMallocHost(&s.host, sizeof(BatchDesc) * max_requests);
        if (e == cudaSuccess) e = cudaMalloc(&s.dev, sizeof(BatchDesc) * max_requests);
        if (e == cudaSuccess) e = cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming);
        if (e == cudaSuccess) s.inline_args = new BatchInlineArgs();
        if (e != cudaSuccess) {
            wc_batch_destroy(b);
            return cuda_fail(e, "wc_batch_create");
        }
    }
    *out = b;
    return WC_OK;
}

int wc_batch_destroy(wc_batch *b)
{
    if (!b) return WC_OK;
    for (auto &s : b->slots) {
        if (s.done) cudaEventSynchronize(s.done);
        release_graph(s);
        if (s.done) cudaEventDestroy(s.done);
        if (s.host) cudaFreeHost(s.host);
        if (s.dev) cudaFree(s.dev);
        delete s.inline_args;
    }
    delete b;
    return WC_OK;
}

int wc_batch_run(wc_batch *b, const wc_batch_request *reqs, uint32_t num_requests,
                 wc_stream_t stream, uint64_t probing_length, uint32_t blocks_per_sm_req)
{
    if (!b) return fail(WC_ERR_INVALID_ARGUMENT, "batch is NULL");
    if (num_requests == 0) return WC_OK;
    if (!reqs) return fail(WC_ERR_INVALID_ARGUMENT, "requests are NULL");
    if (num_requests > b->max_requests)
        return fail(WC_ERR_INVALID_ARGUMENT, "%u requests exceed the batch capacity %u",
                    num_requests, b->max_requests);
    const wc_table *t0 = reqs[0].table;
    if (!t0) return fail(WC_ERR_INVALID_ARGUMENT, "request 0 has no table");
    const int layout = t0->layout;
    const uint32_t W = t0->cfg.cg_size;
    const bool inl = num_requests <= uint32_t(kBatchInline);
    const void *kfn = batch_kernel_ptr(layout, int(W), inl);
    if (!kfn) return fail(WC_ERR_UNSUPPORTED, "batches serve u32/u32 and u64/u64 single-value tables");

    wc_batch::Slot &s = b->slots[b->next];
    b->next = (b->next + 1) % b->depth;
    if (s.used) WC_CUDA(cudaEventSynchronize(s.done)); /* staging slot still in flight */

    BatchInlineArgs *ia = s.inline_args;
    BatchDesc *descs = inl ? ia->desc : s.host;
    uint64_t total = 0;
    for (uint32_t r = 0; r < num_requests; ++r) {
        const wc_batch_request &q = reqs[r];
        const wc_table *t = q.table;
        if (!t || t->kind != 0 || t->layout != layout || t->cfg.cg_size != W)
            return fail(WC_ERR_INVALID_ARGUMENT,
                        "request %u: every table of a batch must be a single-value table "
                        "of the same layout and cg_size",
                        r);
        if (!t->initialized) return fail(WC_ERR_NOT_INITIALIZED, "request %u: table not initialized", r);
        if (q.op != WC_OP_INSERT && q.op != WC_OP_RETRIEVE)
            return fail(WC_ERR_INVALID_ARGUMENT, "request %u: op must be insert or retrieve", r);
        if (q.num && (!q.keys || (q.op == WC_OP_INSERT && !q.values) ||
                      (q.op == WC_OP_RETRIEVE && !q.values_out)))
            return fail(WC_ERR_INVALID_ARGUMENT, "request %u: missing buffer", r);
        BatchDesc &d = descs[r];
        d.t = view_of(t);
        d.keys = q.keys;
        d.values = q.values;
        d.out = q.values_out;
        d.status_out = q.status_handler == WC_HANDLER_NOTHING ? nullptr : q.status_out;
        d.begin = total;
        d.n = q.num;
        d.max_windows = max_windows(probing_length, W, t->num_buckets);
        d.bool_mask = (~q.ignore) ^ 0xFFFu;
        d.op = q.op == WC_OP_INSERT ? kOpInsert : kOpRetrieve;
        d.handler = q.status_handler;
        d.pad = 0;
        total += q.num;
    }
    if (total == 0) return WC_OK;

    const uint64_t wave = uint64_t(device_props().sms) *
                          (blocks_per_sm_req ? blocks_per_sm_req : uint32_t(blocks_per_sm(kfn, kBlock)));
    const uint64_t need = (total + kBlock - 1) / kBlock;
    const unsigned grid = unsigned(need < wave ? need : wave);

    BatchArgs args;
    args.desc = s.dev;
    args.nreq = num_requests;
    args.total = total;
    ia->nreq = num_requests;
    ia->total = total;
    void *argp = inl ? static_cast<void *>(ia) : static_cast<void *>(&args);
    const size_t bytes = inl ? 0 : sizeof(BatchDesc) * num_requests;
    if (s.kernel != kfn || !s.exec) {
        /* a graph per staging slot and kernel; grid, argument values and
         * copy size are updated in place on later runs */
        const int rc = build_graph(s, kfn, grid, argp, bytes);
        if (rc) return rc;
    } else {
        if (!inl)
            WC_CUDA(cudaGraphExecMemcpyNodeSetParams1D(s.exec, s.copy_node, s.dev, s.host, bytes,
                                                       cudaMemcpyHostToDevice));
        cudaKernelNodeParams kp{};
        void *kargs[] = {argp};
        kp.func = const_cast<void *>(kfn);
        kp.gridDim = dim3(grid);
        kp.blockDim = dim3(kBlock);
        kp.sharedMemBytes = 0;
        kp.kernelParams = kargs;
        WC_CUDA(cudaGraphExecKernelNodeSetParams(s.exec, s.kernel_node, &kp));
    }
    cudaStream_t st = reinterpret_cast<cudaStream_t>(stream);
    WC_CUDA(cudaGraphLaunch(s.exec, st));
    note_launches(1); /* the graph's one kernel (beside its descriptor copy) */
    WC_CUDA(cudaEventRecord(s.done, st));
    s.used = true;
    return WC_OK;
}

} // extern "C"
