/*
 * wc_pserve.cu -- persistent serving kernel.
 *
 * One kernel stays resident for the life of a server and takes requests
 * (insert or retrieve of a batch of keys on a resident single-value table)
 * from a ring in mapped host memory, so that a request costs no kernel
 * launch:
 *
 *   host      writes the request into ring slot seq % kPsRing and publishes
 *             it by a release store of `tail`;
 *   dispatcher (warp 0 of block 0) polls `tail` (system-scope acquire),
 *             copies each new request into device memory, cuts it into
 *             chunks of chunk_keys keys and appends the chunks to a chunk
 *             ring in device memory (release store of chunk_tail);
 *   workers   (every other warp) take tickets in order from chunk_head; a
 *             ticket names one chunk, which the warp probes with the warp-
 *             batched loop of table_op_kernel (group_range, wc_kernels.cuh),
 *             then counts the request's remaining chunks down; the warp that
 *             finishes a request's last chunk writes its completion time
 *             (%globaltimer) and sequence number to mapped host memory.
 *
 * Requests that are in flight together must commute: the host submits a
 * request only when no request of the other kind on the same table is in
 * flight (wc_serve_run does this), so every table sees its requests in
 * arrival order.
 *
 * Every wait is bounded.  The dispatcher ends the kernel after
 * idle_timeout_us without a new request (or on the host's stop flag); a
 * worker waiting for its ticket's chunk leaves once the dispatcher has
 * stopped and no chunk is left for it, or after the idle limit plus a
 * margin.  A kernel that ended on the idle limit reports WC_ERR_TIMEOUT
 * when the host stops the server, and the context stays usable.
 */
#include <warpcore_b200.h>

#include "wc_internal.h"

#include <chrono>
#include <cstring>
#include <new>
#include <thread>
#include <unordered_map>
#include <vector>

namespace warpcore {
namespace b200 {

constexpr uint32_t kPsRing = 4096;              /* request slots */
constexpr uint64_t kPsChunkRing = 1ull << 20;   /* chunk slots */
constexpr uint64_t kPsBeginBits = 40;           /* chunk entry: slot << 40 | first key */
constexpr uint32_t kPsErrTimeout = 1, kPsErrChunkRing = 2, kPsErrWorkerTimeout = 4;

struct PsRequest {
    TableView t;
    const void *keys;
    const void *values;
    void *out;
    uint64_t n;
    uint64_t max_windows;
    uint64_t seq;
    int op;
    uint32_t chunk; /* keys per chunk, set by the dispatcher */
};

static_assert(sizeof(PsRequest) % 8 == 0, "requests are copied in 8-byte words");

/* mapped host memory: written by the host (tail, stop, ring) or by the
 * kernel (start_ns, error, done_*) */
struct PsHost {
    uint64_t tail;
    uint32_t stop;
    uint32_t pad0;
    uint64_t start_ns;
    uint32_t error;
    uint32_t pad1;
    uint64_t pad2[4];
    PsRequest ring[kPsRing];
    uint64_t done_seq[kPsRing]; /* seq + 1 once complete */
    uint64_t done_ns[kPsRing];  /* %globaltimer at completion */
};

/* device memory */
struct PsDev {
    unsigned long long chunk_tail; /* chunks published */
    unsigned long long chunk_head; /* tickets handed out */
    uint32_t stop;
    uint32_t error;
    unsigned long long remaining[kPsRing];
    PsRequest req[kPsRing];
    unsigned long long chunk[kPsChunkRing];
};

__device__ __forceinline__ uint64_t global_ns()
{
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}

__device__ __forceinline__ uint64_t ld_acquire_sys(const uint64_t *p)
{
    uint64_t v;
    asm volatile("ld.acquire.sys.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ uint32_t ld_volatile_u32(const uint32_t *p)
{
    return *reinterpret_cast<const volatile uint32_t *>(p);
}

__device__ __forceinline__ unsigned long long ld_acquire_gpu(const unsigned long long *p)
{
    unsigned long long v;
    asm volatile("ld.acquire.gpu.global.u64 %0, [%1];" : "=l"(v) : "l"(p) : "memory");
    return v;
}

__device__ __forceinline__ void st_release_gpu(unsigned long long *p, unsigned long long v)
{
    asm volatile("st.release.gpu.global.u64 [%0], %1;" ::"l"(p), "l"(v) : "memory");
}

__device__ __forceinline__ void ps_fail(PsHost *h, PsDev *d, uint32_t bits)
{
    atomicOr(&d->error, bits);
    atomicOr(&h->error, bits);
    __threadfence_system();
    atomicExch(&d->stop, 1u);
}

/* warp 0 of block 0.  Each round reads the host's tail once and takes up
 * to 32 new requests: their descriptors are copied by all lanes at once
 * (one round trip to host memory for the batch), lane j sizes request j's
 * chunks, a warp prefix sum places them in the chunk ring, and one release
 * store of chunk_tail publishes them all.  Chunk sizes follow the load:
 * while fewer than a quarter of the worker warps' worth of chunks wait
 * unclaimed, a request gets chunks of n / (worker warps) keys (at least 32,
 * a multiple of 32, at most chunk_keys), so that one large request spreads
 * over all resident warps; once chunks queue up, requests get chunks of
 * chunk_keys keys, which cost fewer claims per key.  (Measured on the
 * served mix at 1M requests/s: chunks spread over all warps at every load
 * gave 12.6 Gops/s, over half of them 17.7.) */
__device__ void ps_dispatch(PsHost *h, PsDev *d, uint64_t chunk_keys, uint64_t idle_ns)
{
    const int lane = threadIdx.x & 31;
    const unsigned lanemask_lt = (1u << lane) - 1u;
    const uint64_t workers = uint64_t(gridDim.x) * (blockDim.x >> 5) - 1;
    uint64_t seen = 0;
    unsigned long long ctail = 0;
    if (lane == 0) {
        const uint64_t now = global_ns();
        *reinterpret_cast<volatile uint64_t *>(&h->start_ns) = now ? now : 1;
        __threadfence_system();
    }
    uint64_t last = global_ns();
    for (;;) {
        uint64_t tail = 0;
        uint32_t stop = 0;
        if (lane == 0) {
            tail = ld_acquire_sys(&h->tail);
            stop = ld_volatile_u32(&h->stop);
        }
        tail = __shfl_sync(kFull, tail, 0);
        stop = __shfl_sync(kFull, stop, 0);
        if (seen < tail) {
            const int k = int(tail - seen < 32 ? tail - seen : 32);
            /* copy k descriptors into device memory, 8 bytes per lane */
            constexpr int kWords = int(sizeof(PsRequest) / 8);
            for (int w = lane; w < k * kWords; w += 32) {
                const uint32_t slot = uint32_t((seen + uint64_t(w / kWords)) % kPsRing);
                const uint64_t *src = reinterpret_cast<const uint64_t *>(&h->ring[slot]);
                uint64_t *dst = reinterpret_cast<uint64_t *>(&d->req[slot]);
                dst[w % kWords] = *reinterpret_cast<const volatile uint64_t *>(src + w % kWords);
            }
            __syncwarp();
            /* chunks published and not yet claimed */
            unsigned long long head = 0;
            if (lane == 0) head = ld_acquire_gpu(&d->chunk_head);
            head = __shfl_sync(kFull, head, 0);
            const unsigned long long backlog = ctail > head ? ctail - head : 0;
            const bool busy = backlog * 4 >= workers;
            /* lane j: request seen + j */
            const uint32_t slot = uint32_t((seen + uint64_t(lane)) % kPsRing);
            unsigned long long nch = 0;
            uint64_t chunk = 32;
            if (lane < k) {
                const uint64_t n = d->req[slot].n;
                chunk = busy ? chunk_keys : (n / (workers ? workers : 1) + 31) & ~uint64_t(31);
                if (chunk < 32) chunk = 32;
                if (chunk > chunk_keys) chunk = chunk_keys;
                nch = (n + chunk - 1) / chunk;
                d->req[slot].chunk = uint32_t(chunk);
            }
            /* inclusive prefix sum of the chunk counts */
            unsigned long long incl = nch;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const unsigned long long v = __shfl_up_sync(kFull, incl, o);
                if (lane >= o) incl += v;
            }
            const unsigned long long total = __shfl_sync(kFull, incl, 31);
            const unsigned long long first = ctail + incl - nch;
            /* room in the chunk ring: entries that a worker may not have
             * read yet; tickets are handed out in order and every warp
             * holds at most one, so entries below chunk_head - workers are
             * read */
            if (total) {
                const uint64_t t_wait = global_ns();
                bool room = false;
                for (;;) {
                    unsigned long long used = 0;
                    if (lane == 0) {
                        const unsigned long long h2 = ld_acquire_gpu(&d->chunk_head);
                        const unsigned long long read = h2 > workers ? h2 - workers : 0;
                        used = ctail - (read < ctail ? read : ctail);
                    }
                    used = __shfl_sync(kFull, used, 0);
                    if (used + total <= kPsChunkRing) {
                        room = true;
                        break;
                    }
                    if (global_ns() - t_wait > idle_ns) break;
                    __nanosleep(1000);
                }
                if (!room) {
                    if (lane == 0) ps_fail(h, d, kPsErrChunkRing);
                    return;
                }
            }
            if (lane < k) {
                if (nch == 0) {
                    /* an empty request is complete at once */
                    *reinterpret_cast<volatile uint64_t *>(&h->done_ns[slot]) = global_ns();
                    __threadfence_system();
                    *reinterpret_cast<volatile uint64_t *>(&h->done_seq[slot]) = d->req[slot].seq + 1;
                } else {
                    d->remaining[slot] = nch;
                }
            }
            /* chunk entries, request by request, all lanes writing */
            for (int j = 0; j < k; ++j) {
                const unsigned long long nj = __shfl_sync(kFull, nch, j);
                const unsigned long long fj = __shfl_sync(kFull, first, j);
                const uint64_t cj = __shfl_sync(kFull, chunk, j);
                const uint32_t sj = __shfl_sync(kFull, slot, j);
                for (unsigned long long c = lane; c < nj; c += 32)
                    d->chunk[(fj + c) % kPsChunkRing] = (uint64_t(sj) << kPsBeginBits) | (c * cj);
            }
            (void)lanemask_lt;
            __threadfence();
            __syncwarp();
            ctail += total;
            if (lane == 0 && total) st_release_gpu(&d->chunk_tail, ctail);
            seen += uint64_t(k);
            last = global_ns();
            continue;
        }
        if (stop) {
            if (lane == 0) atomicExch(&d->stop, 1u);
            return;
        }
        if (global_ns() - last > idle_ns) {
            if (lane == 0) ps_fail(h, d, kPsErrTimeout);
            return;
        }
        /* (each poll is a round trip to host memory; no sleep between) */
    }
}

template <class L, int W>
__global__ void __launch_bounds__(256, 2) pserve_kernel(PsHost *h, PsDev *d, uint64_t chunk_keys,
                                                        uint64_t idle_ns)
{
    using K = typename L::key_t;
    using V = typename L::val_t;
    __shared__ uint64_t sh_bucket[8][32];
    __shared__ K sh_key[8][32];
    __shared__ uint32_t sh_off[8][32];
    const int lane = threadIdx.x & 31;
    const int wib = threadIdx.x >> 5;
    if (blockIdx.x == 0 && wib == 0) {
        ps_dispatch(h, d, chunk_keys, idle_ns);
        return;
    }
    /* a worker waits at most this long for its ticket's chunk */
    const uint64_t worker_limit = idle_ns + 200000000ull;
    for (;;) {
        unsigned long long ticket = 0;
        if (lane == 0) ticket = atomicAdd(&d->chunk_head, 1ull);
        ticket = __shfl_sync(kFull, ticket, 0);
        const uint64_t t_wait = global_ns();
        bool got = false;
        for (;;) {
            int state = 0; /* 1 chunk ready, 2 leave */
            if (lane == 0) {
                if (ticket < ld_acquire_gpu(&d->chunk_tail)) state = 1;
                else if (ld_volatile_u32(&d->stop)) state = 2;
                else if (global_ns() - t_wait > worker_limit) {
                    ps_fail(h, d, kPsErrWorkerTimeout);
                    state = 2;
                }
            }
            state = __shfl_sync(kFull, state, 0);
            if (state == 1) {
                got = true;
                break;
            }
            if (state == 2) break;
            __nanosleep(256);
        }
        if (!got) return;
        const unsigned long long e = d->chunk[ticket % kPsChunkRing];
        const uint32_t slot = uint32_t(e >> kPsBeginBits);
        const uint64_t begin = e & ((1ull << kPsBeginBits) - 1);
        const PsRequest &r = d->req[slot];
        TableOpArgs a;
        a.t = r.t;
        a.keys = r.keys;
        a.values = r.values;
        a.out = r.out;
        a.status_out = nullptr;
        a.n = r.n;
        a.max_windows = r.max_windows;
        a.bool_mask = 0;
        a.handler = kHandlerNothing;
        a.is_set = 0;
        a.flags = 0;
        const uint64_t end = begin + r.chunk < r.n ? begin + r.chunk : r.n;
        uint32_t join = 0;
        int live_delta = 0;
        if (r.op == kOpInsert)
            group_range<L, W, kOpInsert>(a, begin, end, sh_bucket[wib], sh_key[wib], sh_off[wib],
                                         nullptr, nullptr, false, join, live_delta);
        else
            group_range<L, W, kOpRetrieve>(a, begin, end, sh_bucket[wib], sh_key[wib], sh_off[wib],
                                           nullptr, nullptr, false, join, live_delta);
        const uint32_t wjoin = __reduce_or_sync(kFull, join);
        const int wlive = int(__reduce_add_sync(kFull, unsigned(live_delta)));
        if (lane == 0) {
            join_status(a.t.status, wjoin);
            live_add(a.t, wlive);
            __threadfence();
            if (atomicAdd(&d->remaining[slot], ~0ull) == 1ull) { /* minus one */
                /* last chunk of the request: every chunk's writes were
                 * fenced before its count-down */
                __threadfence_system();
                *reinterpret_cast<volatile uint64_t *>(&h->done_ns[slot]) = global_ns();
                __threadfence_system();
                *reinterpret_cast<volatile uint64_t *>(&h->done_seq[slot]) = r.seq + 1;
            }
        }
        __syncwarp();
    }
}

template <class L>
static const void *pick_pserve(int W)
{
    switch (W) {
    case 1: return reinterpret_cast<const void *>(pserve_kernel<L, 1>);
    case 2: return reinterpret_cast<const void *>(pserve_kernel<L, 2>);
    case 4: return reinterpret_cast<const void *>(pserve_kernel<L, 4>);
    case 8: return reinterpret_cast<const void *>(pserve_kernel<L, 8>);
    case 16: return reinterpret_cast<const void *>(pserve_kernel<L, 16>);
    case 32: return reinterpret_cast<const void *>(pserve_kernel<L, 32>);
    default: return nullptr;
    }
}

} // namespace b200
} // namespace warpcore

using namespace warpcore::b200;

struct wc_pserver {
    wc_pserver_options opt{};
    int layout = 0;
    int device = 0;
    PsHost *host = nullptr;     /* mapped pinned memory */
    PsHost *host_dev = nullptr; /* its device address */
    PsDev *dev = nullptr;
    cudaStream_t stream = nullptr;
    uint64_t next_seq = 0;
    std::vector<uint8_t> busy; /* slot holds a request not yet seen complete */
    /* completion stamps of requests whose slot was reused before they were
     * polled */
    std::unordered_map<uint64_t, uint64_t> retired_ns;
    std::chrono::steady_clock::time_point t_host0;
    double start_host_us = -1; /* host time (from t_host0) the kernel was seen running */
    uint64_t start_ns = 0;
    bool running = false;
};

namespace {

int ps_fail_host(int code, const char *msg)
{
    set_last_error(msg);
    return code;
}

double host_us(const wc_pserver *s)
{
    return std::chrono::duration<double, std::micro>(std::chrono::steady_clock::now() - s->t_host0)
        .count();
}

void ps_free(wc_pserver *s)
{
    if (s->host) cudaFreeHost(s->host);
    if (s->dev) cudaFree(s->dev);
    delete s;
}

} // namespace

extern "C" int wc_pserver_start(const wc_pserver_options *opt, wc_stream_t stream,
                                wc_pserver **out)
{
    if (!opt || !out) return ps_fail_host(WC_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = nullptr;
    if (opt->key_bytes != 4 && opt->key_bytes != 8)
        return ps_fail_host(WC_ERR_UNSUPPORTED, "key_bytes must be 4 or 8");
    const int layout = opt->key_bytes == 4 ? kLayoutKV32 : kLayoutKV64;
    const void *kfn = layout == kLayoutKV32 ? pick_pserve<LayoutKV32>(int(opt->cg_size))
                                            : pick_pserve<LayoutKV64>(int(opt->cg_size));
    if (!kfn) return ps_fail_host(WC_ERR_INVALID_ARGUMENT, "cg_size must be 1, 2, 4, 8, 16 or 32");
    auto *s = new (std::nothrow) wc_pserver();
    if (!s) return ps_fail_host(WC_ERR_OUT_OF_MEMORY, "host allocation");
    s->opt = *opt;
    if (!s->opt.chunk_keys) s->opt.chunk_keys = 1024;
    if (!s->opt.idle_timeout_us) s->opt.idle_timeout_us = 2000000;
    if (!s->opt.blocks_per_sm) s->opt.blocks_per_sm = 2;
    if (s->opt.chunk_keys >= (1ull << kPsBeginBits)) {
        ps_free(s);
        return ps_fail_host(WC_ERR_INVALID_ARGUMENT, "chunk_keys too large");
    }
    s->layout = layout;
    s->stream = reinterpret_cast<cudaStream_t>(stream);
    s->busy.assign(kPsRing, 0);
    cudaGetDevice(&s->device);
    cudaError_t e = cudaHostAlloc(reinterpret_cast<void **>(&s->host), sizeof(PsHost),
                                  cudaHostAllocMapped);
    if (e == cudaSuccess) {
        std::memset(s->host, 0, sizeof(PsHost));
        e = cudaHostGetDevicePointer(reinterpret_cast<void **>(&s->host_dev), s->host, 0);
    }
    if (e == cudaSuccess) e = cudaMalloc(reinterpret_cast<void **>(&s->dev), sizeof(PsDev));
    if (e == cudaSuccess) e = cudaMemsetAsync(s->dev, 0, sizeof(PsDev), s->stream);
    if (e != cudaSuccess) {
        ps_free(s);
        return host_cuda_fail(e, "persistent server allocation");
    }
    int occ = 0;
    cudaOccupancyMaxActiveBlocksPerMultiprocessor(&occ, kfn, 256, 0);
    int sms = 148;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, s->device);
    const int bps = int(s->opt.blocks_per_sm) < occ ? int(s->opt.blocks_per_sm) : occ;
    if (bps < 1) {
        ps_free(s);
        return ps_fail_host(WC_ERR_CUDA, "persistent kernel does not fit on an SM");
    }
    PsHost *hd = s->host_dev;
    PsDev *dd = s->dev;
    uint64_t ck = s->opt.chunk_keys, idle_ns = s->opt.idle_timeout_us * 1000ull;
    void *args[] = {&hd, &dd, &ck, &idle_ns};
    s->t_host0 = std::chrono::steady_clock::now();
    e = cudaLaunchKernel(kfn, dim3(unsigned(sms * bps)), dim3(256), args, 0, s->stream);
    if (e != cudaSuccess) {
        ps_free(s);
        return host_cuda_fail(e, "persistent kernel launch");
    }
    note_launches(1);
    s->running = true;
    /* wait (bounded) until the dispatcher runs; its start time maps
     * %globaltimer onto the host clock */
    const double limit = double(s->opt.idle_timeout_us) + 5e6;
    while (*reinterpret_cast<volatile uint64_t *>(&s->host->start_ns) == 0) {
        if (host_us(s) > limit || cudaStreamQuery(s->stream) != cudaErrorNotReady) {
            wc_pserver_stop(s);
            return ps_fail_host(WC_ERR_CUDA, "persistent kernel did not start");
        }
        std::this_thread::yield();
    }
    s->start_host_us = host_us(s);
    s->start_ns = *reinterpret_cast<volatile uint64_t *>(&s->host->start_ns);
    *out = s;
    return WC_OK;
}

extern "C" int wc_pserver_submit(wc_pserver *s, wc_table *t, int op, const void *keys,
                                 const void *values, void *values_out, uint64_t num,
                                 uint64_t *ticket_out)
{
    if (!s || !ticket_out) return ps_fail_host(WC_ERR_INVALID_ARGUMENT, "NULL argument");
    if (op != WC_OP_INSERT && op != WC_OP_RETRIEVE)
        return ps_fail_host(WC_ERR_INVALID_ARGUMENT, "op must be WC_OP_INSERT or WC_OP_RETRIEVE");
    if (num && (!keys || (op == WC_OP_INSERT ? !values : !values_out)))
        return ps_fail_host(WC_ERR_INVALID_ARGUMENT, "NULL buffer");
    PsRequest r{};
    int layout = 0;
    uint32_t cg = 0;
    int rc = host_svht_view(t, &r.t, &layout, &cg, s->opt.probing_length, &r.max_windows);
    if (rc) return rc;
    if (layout != s->layout || cg != s->opt.cg_size)
        return ps_fail_host(WC_ERR_INVALID_ARGUMENT,
                            "table's key width or cg_size differs from the server's");
    const uint64_t seq = s->next_seq;
    const uint32_t slot = uint32_t(seq % kPsRing);
    /* the slot's previous request must be complete (bounded wait) */
    if (s->busy[slot]) {
        const double t0 = host_us(s);
        while (*reinterpret_cast<volatile uint64_t *>(&s->host->done_seq[slot]) != seq - kPsRing + 1) {
            if (*reinterpret_cast<volatile uint32_t *>(&s->host->error) ||
                host_us(s) - t0 > double(s->opt.idle_timeout_us) + 1e6)
                return ps_fail_host(WC_ERR_CUDA, "request ring full and the kernel is not draining it");
            std::this_thread::yield();
        }
        s->retired_ns[seq - kPsRing] = *reinterpret_cast<volatile uint64_t *>(&s->host->done_ns[slot]);
    }
    r.keys = keys;
    r.values = values;
    r.out = values_out;
    r.n = num;
    r.seq = seq;
    r.op = op == WC_OP_INSERT ? kOpInsert : kOpRetrieve;
    s->host->ring[slot] = r;
    s->busy[slot] = 1;
    s->next_seq = seq + 1;
    /* publish: the slot's contents before the tail (release) */
    __atomic_store_n(&s->host->tail, seq + 1, __ATOMIC_RELEASE);
    *ticket_out = seq;
    return WC_OK;
}

extern "C" int wc_pserver_poll(wc_pserver *s, uint64_t ticket, int *done, double *complete_us)
{
    if (!s || !done) return ps_fail_host(WC_ERR_INVALID_ARGUMENT, "NULL argument");
    if (ticket >= s->next_seq) return ps_fail_host(WC_ERR_INVALID_ARGUMENT, "unknown ticket");
    *done = 0;
    if (s->next_seq - ticket > kPsRing) {
        /* its slot was reused, so it completed */
        *done = 1;
        auto it = s->retired_ns.find(ticket);
        if (it != s->retired_ns.end()) {
            if (complete_us) *complete_us = s->start_host_us + double(it->second - s->start_ns) * 1e-3;
            s->retired_ns.erase(it);
        } else if (complete_us) {
            *complete_us = -1;
        }
        return WC_OK;
    }
    const uint32_t slot = uint32_t(ticket % kPsRing);
    const uint64_t ds = __atomic_load_n(&s->host->done_seq[slot], __ATOMIC_ACQUIRE);
    if (ds == ticket + 1) {
        *done = 1;
        if (complete_us) {
            const uint64_t ns = *reinterpret_cast<volatile uint64_t *>(&s->host->done_ns[slot]);
            *complete_us = s->start_host_us + double(ns - s->start_ns) * 1e-3;
        }
    }
    return WC_OK;
}

extern "C" int wc_pserver_now_us(const wc_pserver *s, double *now_us)
{
    if (!s || !now_us) return ps_fail_host(WC_ERR_INVALID_ARGUMENT, "NULL argument");
    *now_us = host_us(s);
    return WC_OK;
}

extern "C" int wc_pserver_stop(wc_pserver *s)
{
    if (!s) return WC_OK;
    int rc = WC_OK;
    if (s->running) {
        __atomic_store_n(&s->host->stop, 1u, __ATOMIC_RELEASE);
        const cudaError_t e = cudaStreamSynchronize(s->stream);
        if (e != cudaSuccess) rc = host_cuda_fail(e, "persistent kernel");
        const uint32_t err = *reinterpret_cast<volatile uint32_t *>(&s->host->error);
        if (rc == WC_OK && err) {
            rc = WC_ERR_TIMEOUT;
            set_last_error((err & kPsErrTimeout) ? "persistent kernel ended: no request within its idle limit"
                           : (err & kPsErrChunkRing) ? "persistent kernel ended: chunk ring full"
                                                     : "persistent kernel ended: a worker's wait ran out");
        }
    }
    ps_free(s);
    return rc;
}
