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

/* WC_SERVE_PERSISTENT: one resident kernel (wc_pserve.cu); the host
 * submits each request when it arrives, unless a request of the other kind
 * on its table is in flight or an earlier request of its table waits, and
 * polls completions in mapped host memory. */
int serve_persistent(const wc_serve_request *reqs, uint64_t num_requests,
                     const wc_serve_options *opt, double *issue_us, double *complete_us,
                     wc_serve_stats *stats)
{
    uint64_t max_table = 0;
    for (uint64_t i = 0; i < num_requests; ++i)
        max_table = reqs[i].table_id > max_table ? reqs[i].table_id : max_table;
    wc_table_info inf{};
    int rc = wc_table_get_info(reqs[0].table, &inf);
    if (rc) return rc;
    cudaStream_t stream = nullptr;
    SERVE_CUDA(cudaStreamCreateWithFlags(&stream, cudaStreamNonBlocking));
    SERVE_CUDA(cudaDeviceSynchronize());
    wc_pserver_options po{};
    po.key_bytes = inf.key_bytes;
    po.cg_size = inf.cg_size;
    po.blocks_per_sm = opt->blocks_per_sm;
    po.chunk_keys = opt->max_batch_keys;
    po.probing_length = opt->probing_length;
    wc_pserver *srv = nullptr;
    rc = wc_pserver_start(&po, reinterpret_cast<wc_stream_t>(stream), &srv);
    if (rc) {
        cudaStreamDestroy(stream);
        return rc;
    }
    /* per table: kind of the requests in flight (1 insert, 2 retrieve),
     * their number, and the requests waiting behind them in arrival order */
    std::vector<uint8_t> kind(max_table + 1, 0);
    std::vector<uint32_t> count(max_table + 1, 0);
    std::vector<std::deque<uint64_t>> waiting(max_table + 1);
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
    auto submit = [&](uint64_t id) -> int {
        const wc_serve_request &q = reqs[id];
        if (issue_us) issue_us[id] = now();
        const int r2 = wc_pserver_submit(srv, q.table, q.op, q.keys, q.values, q.values_out, q.num,
                                         &ticket[id]);
        if (r2) return r2;
        kind[q.table_id] = q.op == WC_OP_INSERT ? 1 : 2;
        ++count[q.table_id];
        inflight.push_back(id);
        return WC_OK;
    };
    uint64_t next = 0, done = 0;
    while (done < num_requests && rc == WC_OK) {
        const double t = now();
        bool idle = true;
        while (next < num_requests && reqs[next].arrival_us <= t && rc == WC_OK) {
            const uint64_t id = next++;
            const uint64_t tb = reqs[id].table_id;
            const uint8_t k = reqs[id].op == WC_OP_INSERT ? 1 : 2;
            if (waiting[tb].empty() && (count[tb] == 0 || kind[tb] == k)) rc = submit(id);
            else waiting[tb].push_back(id);
            idle = false;
        }
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
            inflight[j] = inflight.back();
            inflight.pop_back();
            const uint64_t tb = reqs[id].table_id;
            if (--count[tb] == 0) {
                kind[tb] = 0;
                /* release the waiting requests of this table that commute */
                while (!waiting[tb].empty() && rc == WC_OK) {
                    const uint64_t w = waiting[tb].front();
                    const uint8_t k = reqs[w].op == WC_OP_INSERT ? 1 : 2;
                    if (count[tb] != 0 && kind[tb] != k) break;
                    waiting[tb].pop_front();
                    rc = submit(w);
                }
            }
        }
        if (idle && inflight.empty() && next < num_requests) {
            const double wait = reqs[next].arrival_us - now();
            if (wait > 50) std::this_thread::sleep_for(std::chrono::microseconds(int64_t(wait - 40)));
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
