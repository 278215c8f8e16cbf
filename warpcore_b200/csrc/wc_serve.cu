/*
 * wc_serve.cu -- real-time serving loop over resident tables.
 *
 * Replays a stream of timestamped requests (arrival times relative to the
 * start of the run) against tables that are already resident on the device,
 * in one of two forms:
 *
 *   WC_SERVE_PLAIN    every request is its own kernel launch, issued when it
 *                     arrives; requests of one table stay on one stream (of
 *                     `streams`), so each table sees its requests in order.
 *   WC_SERVE_BATCHED  continuous batching: whenever fewer than `depth`
 *                     batches are on the GPU, every request that has arrived
 *                     and may run now is packed into one wc_batch_run launch
 *                     (a batch of one request runs as that request's kernel).
 *                     Batches go round-robin onto `streams` streams; a batch
 *                     waits (stream event wait) for the earlier batches of its
 *                     tables that run on other streams.
 *                     A request may join a batch when no earlier request of
 *                     its table is still waiting and the batch holds no
 *                     request of the other kind on that table, so every
 *                     table sees its requests in arrival order.  Requests that
 *                     arrive while a batch runs are admitted to the next one.
 *
 * Completion times come from CUDA events (one per request, or one per
 * batch), measured from an event recorded at the start of the run.
 */
#include <warpcore_b200.h>

#include "wc_internal.h"

#include <chrono>
#include <algorithm>
#include <cstring>
#include <deque>
#include <thread>
#include <vector>

namespace {

using Clock = std::chrono::steady_clock;

int serve_fail(int code, const char *msg)
{
    warpcore::b200::set_last_error(msg);
    return code;
}

#define SERVE_CUDA(call)                                                       \
    do {                                                                       \
        cudaError_t e_ = (call);                                               \
        if (e_ != cudaSuccess) return serve_fail(WC_ERR_CUDA, cudaGetErrorString(e_)); \
    } while (0)

double since(Clock::time_point t0)
{
    return std::chrono::duration<double, std::micro>(Clock::now() - t0).count();
}

} // namespace

/* ------------------------------------------------------------------ */
/* Table pool: admission against a device-memory budget                 */
/* ------------------------------------------------------------------ */

struct PoolTable {
    wc_table_config cfg{};
    uint64_t min_capacity = 0, seed = 0, bytes = 0;
    wc_table *t = nullptr;  /* resident handle, or NULL */
    void *mem = nullptr;    /* its device memory (from the pool's memory pool) */
    std::vector<unsigned char> host; /* copy of the memory, once swapped out */
    bool saved = false;     /* host holds the table's contents */
    uint64_t last_use = 0;  /* admission clock */
};

struct wc_table_pool {
    uint64_t budget = 0;
    uint64_t resident_bytes = 0;
    uint64_t buffer_bytes = 0; /* request buffers in flight, charged to the budget */
    uint64_t clock = 0;
    std::vector<PoolTable> tables;
    cudaMemPool_t mempool = nullptr;
    cudaStream_t stream = nullptr;
    /* pinned bounce buffer for table copies, allocated with the pool: a
     * page-locked allocation synchronises the device, so none may happen
     * while a persistent server runs */
    unsigned char *bounce = nullptr;
    uint64_t bounce_bytes = 0;
    wc_table_pool_stats stats{};
};

namespace {

int pool_fail(int code, const char *msg)
{
    warpcore::b200::set_last_error(msg);
    return code;
}

/* copy a resident table to host memory (through the pinned bounce buffer)
 * and release its device memory */
int pool_evict(wc_table_pool *p, PoolTable &e)
{
    e.host.resize(e.bytes);
    for (uint64_t off = 0; off < e.bytes; off += p->bounce_bytes) {
        const uint64_t n = e.bytes - off < p->bounce_bytes ? e.bytes - off : p->bounce_bytes;
        SERVE_CUDA(cudaMemcpyAsync(p->bounce, reinterpret_cast<unsigned char *>(e.mem) + off, n,
                                   cudaMemcpyDeviceToHost, p->stream));
        SERVE_CUDA(cudaStreamSynchronize(p->stream));
        std::memcpy(e.host.data() + off, p->bounce, n);
    }
    wc_table_destroy(e.t);
    e.t = nullptr;
    SERVE_CUDA(cudaFreeAsync(e.mem, p->stream));
    SERVE_CUDA(cudaStreamSynchronize(p->stream));
    e.mem = nullptr;
    e.saved = true;
    p->resident_bytes -= e.bytes;
    ++p->stats.evictions;
    return WC_OK;
}

/* Place a table in device memory: its host copy, or the image of an empty
 * table, goes in through the bounce buffer by the copy engine and the table
 * adopts it.  No kernel runs: a persistent server may hold the SMs' registers,
 * so a kernel on another stream (an init) could wait for it to end. */
int pool_admit(wc_table_pool *p, PoolTable &e)
{
    SERVE_CUDA(cudaMallocFromPoolAsync(&e.mem, e.bytes, p->mempool, p->stream));
    const wc_stream_t ws = reinterpret_cast<wc_stream_t>(p->stream);
    for (uint64_t off = 0; off < e.bytes; off += p->bounce_bytes) {
        const uint64_t n = e.bytes - off < p->bounce_bytes ? e.bytes - off : p->bounce_bytes;
        if (e.saved) {
            std::memcpy(p->bounce, e.host.data() + off, n);
        } else {
            const int r0 = warpcore::b200::host_svht_empty_image(&e.cfg, e.min_capacity, p->bounce,
                                                                 off, n);
            if (r0) return r0;
        }
        SERVE_CUDA(cudaMemcpyAsync(reinterpret_cast<unsigned char *>(e.mem) + off, p->bounce, n,
                                   cudaMemcpyHostToDevice, p->stream));
        SERVE_CUDA(cudaStreamSynchronize(p->stream));
    }
    const int rc = wc_svht_create_on(&e.cfg, e.min_capacity, e.seed, 2, e.mem, e.bytes, ws, &e.t);
    if (rc) {
        cudaFreeAsync(e.mem, p->stream);
        cudaStreamSynchronize(p->stream);
        e.mem = nullptr;
        return rc;
    }
    p->resident_bytes += e.bytes;
    if (e.saved) ++p->stats.restores;
    ++p->stats.admissions;
    if (p->resident_bytes + p->buffer_bytes > p->stats.peak_bytes)
        p->stats.peak_bytes = p->resident_bytes + p->buffer_bytes;
    return WC_OK;
}

/* Make table `id` resident with `extra` more bytes of request buffers
 * charged, evicting the least recently used tables that `busy` says have
 * nothing in flight.  Returns 1 if it is resident and charged, 0 if the
 * budget cannot take it now (the caller retries after completions). */
int pool_acquire(wc_table_pool *p, uint64_t id, uint64_t extra,
                 const std::vector<uint32_t> &busy, int *rc)
{
    PoolTable &e = p->tables[id];
    const uint64_t need = (e.t ? 0 : e.bytes) + extra;
    while (p->resident_bytes + p->buffer_bytes + need > p->budget) {
        uint64_t victim = ~0ull, oldest = ~0ull;
        for (uint64_t j = 0; j < p->tables.size(); ++j) {
            const PoolTable &c = p->tables[j];
            if (j != id && c.t && busy[j] == 0 && c.last_use < oldest) {
                oldest = c.last_use;
                victim = j;
            }
        }
        if (victim == ~0ull) return 0;
        *rc = pool_evict(p, p->tables[victim]);
        if (*rc) return 0;
    }
    if (!e.t) {
        *rc = pool_admit(p, e);
        if (*rc) return 0;
    }
    e.last_use = ++p->clock;
    p->buffer_bytes += extra;
    if (p->resident_bytes + p->buffer_bytes > p->stats.peak_bytes)
        p->stats.peak_bytes = p->resident_bytes + p->buffer_bytes;
    return 1;
}

} // namespace

extern "C" int wc_table_pool_create(uint64_t budget_bytes, wc_table_pool **out)
{
    if (!out) return pool_fail(WC_ERR_INVALID_ARGUMENT, "out is NULL");
    *out = nullptr;
    auto *p = new wc_table_pool();
    p->budget = budget_bytes;
    int dev = 0;
    cudaGetDevice(&dev);
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaError_t e = cudaMemPoolCreate(&p->mempool, &props);
    if (e == cudaSuccess) {
        /* keep freed memory in the pool for the next admission */
        uint64_t keep = budget_bytes;
        e = cudaMemPoolSetAttribute(p->mempool, cudaMemPoolAttrReleaseThreshold, &keep);
    }
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&p->stream, cudaStreamNonBlocking);
    p->bounce_bytes = 16ull << 20;
    if (e == cudaSuccess)
        e = cudaHostAlloc(reinterpret_cast<void **>(&p->bounce), p->bounce_bytes, cudaHostAllocDefault);
    if (e != cudaSuccess) {
        if (p->stream) cudaStreamDestroy(p->stream);
        if (p->mempool) cudaMemPoolDestroy(p->mempool);
        delete p;
        return pool_fail(WC_ERR_CUDA, cudaGetErrorString(e));
    }
    *out = p;
    return WC_OK;
}

extern "C" int wc_table_pool_add(wc_table_pool *p, const wc_table_config *cfg,
                                 uint64_t min_capacity, uint64_t seed, uint64_t *id_out)
{
    if (!p || !cfg || !id_out) return pool_fail(WC_ERR_INVALID_ARGUMENT, "NULL argument");
    PoolTable e;
    e.cfg = *cfg;
    e.min_capacity = min_capacity;
    e.seed = seed;
    int rc = wc_svht_memory_bytes(cfg, min_capacity, &e.bytes);
    if (rc) return rc;
    e.bytes = (e.bytes + 255) & ~uint64_t(255);
    if (e.bytes > p->budget) return pool_fail(WC_ERR_OUT_OF_MEMORY, "table larger than the pool's budget");
    *id_out = p->tables.size();
    p->tables.push_back(e);
    return WC_OK;
}

extern "C" int wc_table_pool_table(wc_table_pool *p, uint64_t id, wc_table **out)
{
    if (!p || !out || id >= p->tables.size()) return pool_fail(WC_ERR_INVALID_ARGUMENT, "bad table id");
    std::vector<uint32_t> idle(p->tables.size(), 0);
    int rc = WC_OK;
    if (!pool_acquire(p, id, 0, idle, &rc))
        return rc ? rc : pool_fail(WC_ERR_OUT_OF_MEMORY, "budget cannot take the table");
    *out = p->tables[id].t;
    return WC_OK;
}

extern "C" int wc_table_pool_get_stats(const wc_table_pool *p, wc_table_pool_stats *out)
{
    if (!p || !out) return pool_fail(WC_ERR_INVALID_ARGUMENT, "NULL argument");
    *out = p->stats;
    out->resident_bytes = p->resident_bytes;
    uint64_t n = 0;
    for (const auto &e : p->tables) n += e.t != nullptr;
    out->resident_tables = n;
    return WC_OK;
}

extern "C" int wc_table_pool_destroy(wc_table_pool *p)
{
    if (!p) return WC_OK;
    for (auto &e : p->tables) {
        if (e.t) wc_table_destroy(e.t);
        if (e.mem) cudaFreeAsync(e.mem, p->stream);
    }
    cudaStreamSynchronize(p->stream);
    cudaFreeHost(p->bounce);
    cudaStreamDestroy(p->stream);
    cudaMemPoolDestroy(p->mempool);
    delete p;
    return WC_OK;
}

namespace {

/* WC_SERVE_PERSISTENT: one resident kernel (wc_pserve.cu); the host
 * submits each request when it arrives, unless a request of the other kind
 * on its table is in flight or an earlier request of its table waits, and
 * polls completions in mapped host memory.  With a table pool, a request
 * is submitted only once its table is resident and the budget holds its
 * buffers too; otherwise it waits (with the later requests of its table)
 * and is retried whenever a request completes. */
int serve_persistent(const wc_serve_request *reqs, uint64_t num_requests,
                     const wc_serve_options *opt, double *issue_us, double *complete_us,
                     wc_serve_stats *stats)
{
    wc_table_pool *pool = opt->pool;
    uint64_t max_table = 0;
    for (uint64_t i = 0; i < num_requests; ++i) {
        max_table = reqs[i].table_id > max_table ? reqs[i].table_id : max_table;
        if (pool && reqs[i].table_id >= pool->tables.size())
            return serve_fail(WC_ERR_INVALID_ARGUMENT, "table_id not in the pool");
    }
    wc_table_config cfg0{};
    if (pool) {
        cfg0 = pool->tables[reqs[0].table_id].cfg;
    } else {
        wc_table_info inf{};
        const int r0 = wc_table_get_info(reqs[0].table, &inf);
        if (r0) return r0;
        cfg0.key_bytes = inf.key_bytes;
        cfg0.value_bytes = inf.value_bytes;
        cfg0.cg_size = inf.cg_size;
    }
    const uint64_t pair_bytes = uint64_t(cfg0.key_bytes) + cfg0.value_bytes;
    cudaStream_t stream = nullptr;
    SERVE_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    SERVE_CUDA(cudaDeviceSynchronize());
    wc_pserver_options po{};
    po.key_bytes = cfg0.key_bytes;
    po.cg_size = cfg0.cg_size;
    po.blocks_per_sm = opt->blocks_per_sm;
    po.chunk_keys = opt->max_batch_keys;
    po.probing_length = opt->probing_length;
    wc_pserver *srv = nullptr;
    int rc = wc_pserver_start(&po, reinterpret_cast<wc_stream_t>(stream), &srv);
    if (rc) {
        cudaStreamDestroy(stream);
        return rc;
    }
    /* per table: kind of the requests in flight (1 insert, 2 retrieve),
     * their number, the requests waiting in arrival order, and what holds
     * the table in the pool (in flight + waiting) */
    std::vector<uint8_t> kind(max_table + 1, 0);
    std::vector<uint32_t> count(max_table + 1, 0);
    std::vector<uint32_t> hold(pool ? pool->tables.size() : max_table + 1, 0);
    std::vector<std::deque<uint64_t>> waiting(max_table + 1);
    std::vector<uint8_t> on_budget_list(max_table + 1, 0);
    std::deque<uint64_t> budget_list; /* tables whose front request waits for budget */
    std::vector<uint64_t> ticket(num_requests, 0);
    std::vector<uint64_t> inflight;
    inflight.reserve(4096);
    double t0 = 0;
    wc_pserver_now_us(srv, &t0);
    auto now = [&]() {
        double u = 0;
        wc_pserver_now_us(srv, &u);
        return u - t0;
    };
    /* submit request id if its table and buffers fit; *blocked = true if
     * the budget cannot take them now */
    auto submit = [&](uint64_t id, bool *blocked) -> int {
        const wc_serve_request &q = reqs[id];
        wc_table *tbl = q.table;
        *blocked = false;
        if (pool) {
            int prc = WC_OK;
            if (!pool_acquire(pool, q.table_id, q.num * pair_bytes, hold, &prc)) {
                if (prc) return prc;
                *blocked = true;
                return WC_OK;
            }
            tbl = pool->tables[q.table_id].t;
        }
        if (issue_us) issue_us[id] = now();
        const int r2 = wc_pserver_submit(srv, tbl, q.op, q.keys, q.values, q.values_out, q.num,
                                         &ticket[id]);
        if (r2) return r2;
        kind[q.table_id] = q.op == WC_OP_INSERT ? 1 : 2;
        ++count[q.table_id];
        ++hold[q.table_id];
        inflight.push_back(id);
        return WC_OK;
    };
    /* submit the waiting requests of table tb that may run now */
    auto release = [&](uint64_t tb) -> int {
        while (!waiting[tb].empty()) {
            const uint64_t w = waiting[tb].front();
            const uint8_t k = reqs[w].op == WC_OP_INSERT ? 1 : 2;
            if (count[tb] != 0 && kind[tb] != k) return WC_OK;
            bool blocked = false;
            const int r3 = submit(w, &blocked);
            if (r3) return r3;
            if (blocked) {
                if (!on_budget_list[tb]) {
                    on_budget_list[tb] = 1;
                    budget_list.push_back(tb);
                }
                return WC_OK;
            }
            waiting[tb].pop_front();
            --hold[tb]; /* counted again by submit as in flight */
        }
        return WC_OK;
    };
    uint64_t next = 0, done = 0;
    uint64_t spins = 0;
    while (done < num_requests && rc == WC_OK) {
        /* the kernel must still run while requests are outstanding: it ends
         * on its own only on a bounded wait that ran out */
        if ((++spins & 1023) == 0 && cudaStreamQuery(stream) != cudaErrorNotReady) {
            rc = serve_fail(WC_ERR_TIMEOUT, "persistent kernel ended with requests outstanding");
            break;
        }
        const double t = now();
        bool idle = true;
        while (next < num_requests && reqs[next].arrival_us <= t && rc == WC_OK) {
            const uint64_t id = next++;
            const uint64_t tb = reqs[id].table_id;
            const uint8_t k = reqs[id].op == WC_OP_INSERT ? 1 : 2;
            bool blocked = false;
            if (waiting[tb].empty() && (count[tb] == 0 || kind[tb] == k)) rc = submit(id, &blocked);
            else blocked = true;
            if (blocked && rc == WC_OK) {
                waiting[tb].push_back(id);
                ++hold[tb];
                if (pool && count[tb] == 0 && !on_budget_list[tb]) {
                    /* it waits for budget, not for the other kind */
                    on_budget_list[tb] = 1;
                    budget_list.push_back(tb);
                    ++pool->stats.waits;
                }
            }
            idle = false;
        }
        bool completed = false;
        for (size_t j = 0; j < inflight.size() && rc == WC_OK;) {
            const uint64_t id = inflight[j];
            int fin = 0;
            double cu = 0;
            rc = wc_pserver_poll(srv, ticket[id], &fin, &cu);
            if (rc || !fin) {
                ++j;
                continue;
            }
            complete_us[id] = cu - t0;
            ++done;
            idle = false;
            completed = true;
            inflight[j] = inflight.back();
            inflight.pop_back();
            const uint64_t tb = reqs[id].table_id;
            --hold[tb];
            if (pool) pool->buffer_bytes -= reqs[id].num * pair_bytes;
            if (--count[tb] == 0) {
                kind[tb] = 0;
                rc = release(tb);
            }
        }
        if ((completed || inflight.empty()) && pool && rc == WC_OK && !budget_list.empty()) {
            /* budget freed up: retry the tables waiting for it, in order */
            const size_t n = budget_list.size();
            for (size_t j = 0; j < n && rc == WC_OK; ++j) {
                const uint64_t tb = budget_list.front();
                budget_list.pop_front();
                on_budget_list[tb] = 0;
                rc = release(tb);
            }
        }
        if (idle && inflight.empty() && next < num_requests) {
            const double wait = reqs[next].arrival_us - now();
            if (wait > 50) std::this_thread::sleep_for(std::chrono::microseconds(int64_t(wait - 40)));
        }
        if (inflight.empty() && next >= num_requests && done < num_requests && !budget_list.empty() &&
            rc == WC_OK) {
            /* nothing in flight and requests still wait: the budget is too
             * small for them even with every other table evicted */
            rc = serve_fail(WC_ERR_OUT_OF_MEMORY, "a request does not fit the pool's budget");
        }
    }
    const int rs = wc_pserver_stop(srv);
    if (rc == WC_OK) rc = rs;
    cudaStreamDestroy(stream);
    if (stats) {
        stats->launches = 1;
        stats->batches = num_requests;
        stats->max_keys_in_batch = po.chunk_keys ? po.chunk_keys : 1024;
        stats->gpu_batch_us = 0;
        stats->host_launch_us = 0;
        stats->host_wall_us = now();
    }
    return rc;
}

} // namespace

extern "C" int wc_serve_run(const wc_serve_request *reqs, uint64_t num_requests,
                            const wc_serve_options *opt, double *issue_us, double *complete_us,
                            wc_serve_stats *stats)
{
    if (!reqs || !opt || !complete_us) return serve_fail(WC_ERR_INVALID_ARGUMENT, "NULL argument");
    if (num_requests == 0) return WC_OK;
    for (uint64_t i = 1; i < num_requests; ++i)
        if (reqs[i].arrival_us < reqs[i - 1].arrival_us)
            return serve_fail(WC_ERR_INVALID_ARGUMENT, "requests must be sorted by arrival");

    if (opt->mode == WC_SERVE_PERSISTENT)
        return serve_persistent(reqs, num_requests, opt, issue_us, complete_us, stats);
    const int nstreams = opt->streams ? int(opt->streams) : 4;
    std::vector<cudaStream_t> streams(nstreams);
    for (auto &s : streams) SERVE_CUDA(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    cudaEvent_t start;
    SERVE_CUDA(cudaEventCreate(&start));

    /* one event per request (plain) or per batch (batched) */
    const uint64_t nevents = num_requests;
    std::vector<cudaEvent_t> ev(nevents);
    for (auto &e : ev) SERVE_CUDA(cudaEventCreate(&e));
    /* batched form: an event before each batch too, for the GPU time of a batch */
    std::vector<cudaEvent_t> pre(opt->mode == WC_SERVE_BATCHED ? nevents : 0);
    for (auto &e : pre) SERVE_CUDA(cudaEventCreate(&e));
    double host_launch_us = 0;
    std::vector<int64_t> event_of(num_requests, -1);

    wc_batch *batch = nullptr;
    const uint32_t max_req = opt->max_batch_requests ? opt->max_batch_requests : 4096;
    const uint32_t depth = opt->depth ? opt->depth : 2;
    if (opt->mode == WC_SERVE_BATCHED) {
        /* staging slots for every batch that can be in flight */
        const int rc = wc_batch_create(max_req, depth * uint32_t(nstreams), &batch);
        if (rc) return rc;
    }

    SERVE_CUDA(cudaDeviceSynchronize());
    SERVE_CUDA(cudaEventRecord(start, streams[0]));
    SERVE_CUDA(cudaEventSynchronize(start));
    const Clock::time_point t0 = Clock::now();

    uint64_t launches = 0, batches = 0, max_keys_in_batch = 0;
    int rc = WC_OK;
    if (opt->mode == WC_SERVE_PLAIN) {
        for (uint64_t i = 0; i < num_requests && rc == WC_OK; ++i) {
            const wc_serve_request &q = reqs[i];
            while (since(t0) < q.arrival_us) { /* wait for the arrival */
            }
            if (issue_us) issue_us[i] = since(t0);
            cudaStream_t s = streams[q.table_id % uint64_t(nstreams)];
            wc_stream_t ws = reinterpret_cast<wc_stream_t>(s);
            if (q.op == WC_OP_INSERT)
                rc = wc_svht_insert(q.table, q.keys, q.values, q.num, ws, opt->probing_length,
                                    nullptr, WC_HANDLER_NOTHING, 0);
            else
                rc = wc_svht_retrieve(q.table, q.keys, q.num, q.values_out, ws,
                                      opt->probing_length, nullptr, WC_HANDLER_NOTHING, 0);
            if (rc == WC_OK && cudaEventRecord(ev[i], s) != cudaSuccess) rc = WC_ERR_CUDA;
            event_of[i] = int64_t(i);
            ++launches;
        }
    } else {
        std::deque<uint64_t> ready;
        uint64_t next_arrival = 0;
        std::deque<std::pair<int64_t, uint64_t>> inflight; /* (event, batch id) */
        std::vector<wc_batch_request> br;
        br.reserve(max_req);
        std::vector<uint64_t> members;
        /* per-table state during the formation of one batch */
        std::vector<uint8_t> kind_in_batch;  /* 0 none, 1 insert, 2 retrieve */
        std::vector<uint8_t> blocked;
        std::vector<uint32_t> touched;
        uint64_t max_table = 0;
        for (uint64_t i = 0; i < num_requests; ++i)
            max_table = reqs[i].table_id > max_table ? reqs[i].table_id : max_table;
        kind_in_batch.assign(max_table + 1, 0);
        blocked.assign(max_table + 1, 0);
        /* last batch that touched each table, and the stream of every batch:
         * a batch waits for the previous batches of its tables that run on
         * other streams, so each table still sees its requests in order */
        std::vector<int64_t> last_batch_of(max_table + 1, -1);
        std::vector<int> stream_of_batch;
        std::vector<int64_t> waits;
        uint64_t done = 0, issued = 0;
        int64_t next_event = 0;
        int next_stream = 0;
        while (done < num_requests && rc == WC_OK) {
            const double now = since(t0);
            while (next_arrival < num_requests && reqs[next_arrival].arrival_us <= now)
                ready.push_back(next_arrival++);
            for (auto it = inflight.begin(); it != inflight.end();) {
                if (cudaEventQuery(ev[it->first]) == cudaSuccess) {
                    done += it->second;
                    it = inflight.erase(it);
                } else {
                    ++it;
                }
            }
            if (inflight.size() >= depth * uint64_t(nstreams) || ready.empty()) {
                if (ready.empty() && inflight.empty() && next_arrival < num_requests) {
                    const double wait = reqs[next_arrival].arrival_us - since(t0);
                    if (wait > 50) std::this_thread::sleep_for(std::chrono::microseconds(int64_t(wait - 40)));
                }
                continue;
            }
            /* form one batch from the ready requests, in arrival order */
            br.clear();
            members.clear();
            uint64_t keys = 0;
            std::deque<uint64_t> rest;
            for (uint64_t id : ready) {
                const wc_serve_request &q = reqs[id];
                const uint8_t kind = q.op == WC_OP_INSERT ? 1 : 2;
                const uint64_t tb = q.table_id;
                bool take = br.size() < max_req && !blocked[tb] &&
                            (kind_in_batch[tb] == 0 || kind_in_batch[tb] == kind) &&
                            (br.empty() || opt->max_batch_keys == 0 || keys + q.num <= opt->max_batch_keys);
                if (take) {
                    if (kind_in_batch[tb] == 0) touched.push_back(uint32_t(tb));
                    kind_in_batch[tb] = kind;
                    wc_batch_request r{};
                    r.table = q.table;
                    r.op = q.op;
                    r.status_handler = WC_HANDLER_NOTHING;
                    r.keys = q.keys;
                    r.values = q.values;
                    r.values_out = q.values_out;
                    r.num = q.num;
                    br.push_back(r);
                    members.push_back(id);
                    keys += q.num;
                } else {
                    /* later requests of this table wait too (arrival order) */
                    if (!blocked[tb]) touched.push_back(uint32_t(tb));
                    blocked[tb] = 1;
                    rest.push_back(id);
                }
            }
            for (uint32_t tb : touched) {
                kind_in_batch[tb] = 0;
                blocked[tb] = 0;
            }
            touched.clear();
            ready.swap(rest);
            const double issue = since(t0);
            for (uint64_t id : members)
                if (issue_us) issue_us[id] = issue;
            const int64_t e = next_event++;
            const int si = next_stream;
            next_stream = (next_stream + 1) % nstreams;
            cudaStream_t bs = streams[si];
            waits.clear();
            for (uint64_t id : members) {
                const int64_t prev = last_batch_of[reqs[id].table_id];
                if (prev >= 0 && stream_of_batch[prev] != si) waits.push_back(prev);
                last_batch_of[reqs[id].table_id] = e;
            }
            std::sort(waits.begin(), waits.end());
            waits.erase(std::unique(waits.begin(), waits.end()), waits.end());
            for (int64_t w : waits)
                if (cudaStreamWaitEvent(bs, ev[w], 0) != cudaSuccess) rc = WC_ERR_CUDA;
            stream_of_batch.push_back(si);
            if (rc == WC_OK && cudaEventRecord(pre[e], bs) != cudaSuccess) rc = WC_ERR_CUDA;
            if (rc) break;
            const wc_stream_t ws = reinterpret_cast<wc_stream_t>(bs);
            if (br.size() == 1) {
                /* a batch of one is cheapest as the request's own kernel */
                const wc_batch_request &q = br[0];
                rc = q.op == WC_OP_INSERT
                         ? wc_svht_insert(q.table, q.keys, q.values, q.num, ws, opt->probing_length,
                                          nullptr, WC_HANDLER_NOTHING, 0)
                         : wc_svht_retrieve(q.table, q.keys, q.num, q.values_out, ws,
                                            opt->probing_length, nullptr, WC_HANDLER_NOTHING, 0);
            } else {
                rc = wc_batch_run(batch, br.data(), uint32_t(br.size()), ws, opt->probing_length,
                                  opt->blocks_per_sm);
            }
            host_launch_us += since(t0) - issue;
            if (rc) break;
            if (cudaEventRecord(ev[e], bs) != cudaSuccess) {
                rc = WC_ERR_CUDA;
                break;
            }
            for (uint64_t id : members) event_of[id] = e;
            inflight.emplace_back(e, uint64_t(members.size()));
            issued += members.size();
            ++batches;
            ++launches;
            max_keys_in_batch = keys > max_keys_in_batch ? keys : max_keys_in_batch;
        }
        (void)issued;
    }
    cudaError_t e = cudaDeviceSynchronize();
    if (rc == WC_OK && e != cudaSuccess) rc = serve_fail(WC_ERR_CUDA, cudaGetErrorString(e));
    if (rc == WC_OK) {
        for (uint64_t i = 0; i < num_requests; ++i) {
            float ms = 0;
            if (event_of[i] < 0 || cudaEventElapsedTime(&ms, start, ev[event_of[i]]) != cudaSuccess) {
                rc = serve_fail(WC_ERR_CUDA, "missing completion event");
                break;
            }
            complete_us[i] = double(ms) * 1e3;
        }
    }
    double gpu_us = 0;
    if (rc == WC_OK && opt->mode == WC_SERVE_BATCHED) {
        for (uint64_t b = 0; b < batches; ++b) {
            float ms = 0;
            if (cudaEventElapsedTime(&ms, pre[b], ev[b]) == cudaSuccess) gpu_us += double(ms) * 1e3;
        }
    }
    if (stats) {
        stats->gpu_batch_us = gpu_us;
        stats->host_launch_us = host_launch_us;
        stats->launches = launches;
        stats->batches = batches;
        stats->max_keys_in_batch = max_keys_in_batch;
        stats->host_wall_us = since(t0);
    }
    if (batch) wc_batch_destroy(batch);
    for (auto &ee : ev) cudaEventDestroy(ee);
    for (auto &ee : pre) cudaEventDestroy(ee);
    cudaEventDestroy(start);
    for (auto &s : streams) cudaStreamDestroy(s);
    return rc;
}
