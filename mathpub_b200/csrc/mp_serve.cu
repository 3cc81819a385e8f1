// mp_serve.cu -- request serving with continuous batching (include/mathpub_gpu.h, serving).
//
// A server owns K workers.  Each worker is a handle of its own (stream, scratch buffers)
// that uses the server's resident sieving-prime table and presieve patterns, built once at
// open for every height the server accepts.  Requests wait in one FIFO.  A worker takes
// the next request when an in-flight slot is free and the request's device-memory estimate
// fits in what is left of the device's free memory, read with cudaMemGetInfo at admission
// time (and of the option's cap), so requests that arrive while others are on the GPU are
// admitted as soon as slots and memory free up.
//   range request      runs the batched sieve on the worker's stream, at most `chunk`
//                      integers at a time: a longer range goes back to the end of the queue
//                      after each chunk (processor sharing), so that the short requests
//                      behind it are not held up for its whole length.  The chunks' results
//                      join exactly: counts add, and every gap belongs to the chunk of the
//                      prime that starts it (each chunk sees the primes past its end);
//                      K workers overlap on the device;
//   primality request  a worker that picks one takes every primality request waiting at
//                      that moment (up to a candidate cap) and runs them as ONE persistent
//                      batched BPSW launch over all their lists (continuous batching).
// Results are those of the same request run alone: the kernels are the same and every
// request has its own outputs; only scheduling differs.
#include "mp_common.cuh"
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <deque>
#include <thread>
#include <unordered_map>

struct ServeReq {
    u64 id = 0;
    u32 kind = 0;                    // 1 range, 2 primality
    u64 lo = 0, hi = 0;
    u64 next = 0;                    // range: the first integer not yet sieved
    u64 chunk = 0;                   // range: integers per turn
    std::vector<u64> cand;
    u8 *out_bits = nullptr;
    u64 mem = 0;
    bool done = false;
    mp_serve_result res;
};

struct mp_server {
    mp_handle *main = nullptr;
    std::vector<mp_handle *> workers;
    std::vector<std::thread> threads;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<ServeReq *> pending;
    std::unordered_map<u64, ServeReq *> reqs;
    u64 next_id = 1;
    bool closing = false;
    u64 budget = 0, mem_used = 0;    // budget: the cap from the options (or half the free HBM at open)
    std::atomic<u64> free_hbm{0};    // device free memory, last read (outside the lock)
    std::atomic<double> free_at{0};  // when it was read (seconds)
    std::atomic<int> reading{0};     // a worker is reading it now
    u64 reserve = 256ull << 20;      // free HBM never handed out
    u32 max_inflight = 256, inflight = 0;
    u64 prime_limit = 0;
    u64 chunk = 1ull << 32;          // least integers of a range request per turn
    u64 bpsw_cap = 1ull << 22;       // candidates per merged primality launch
};

static double now_s()
{
    return std::chrono::duration<double>(std::chrono::steady_clock::now().time_since_epoch()).count();
}

// device memory a request occupies while it runs (scratch of its launch)
static u64 range_mem(u64 lo, u64 hi)
{
    const u64 bits = (hi + MP_TAIL - (lo & ~1ull)) / 2;
    const u64 tiles = (bits >> 20) + 1;
    const u64 wave = std::min<u64>(tiles, 1184);
    return tiles * 64 + wave * (1ull << 20) + (1ull << 20);
}

static u64 bpsw_mem(u64 count) { return count * 8 + count / 8 + 4096; }

// the next chunk of a range request, joined into its result; true when the range is done
static bool run_range(mp_handle *w, ServeReq *r)
{
    const u64 chunk = r->chunk;
    mp_sieve_opts o;
    memset(&o, 0, sizeof o);
    o.mode = MP_MODE_BATCHED;
    mp_range_stats st;
    memset(&st, 0, sizeof st);
    const u64 a = r->next, b = r->hi - a > chunk ? a + chunk : r->hi;
    const int rc = mp_sieve_range(w, a, b, &o, &st, nullptr, nullptr, nullptr);
    if (rc != MP_OK) { r->res.status = rc; return true; }
    r->res.pi += st.pi;
    r->res.twins += st.twins;
    if (st.max_gap > r->res.max_gap) { r->res.max_gap = st.max_gap; r->res.gap_start = st.gap_start; }
    r->next = b;
    return b >= r->hi;
}

static void run_bpsw(mp_handle *w, std::vector<ServeReq *> &batch)
{
    std::vector<const uint64_t *> lists;
    std::vector<uint32_t> lens;
    std::vector<uint8_t *> outs;
    for (ServeReq *r : batch) {
        lists.push_back(r->cand.data());
        lens.push_back((uint32_t)r->cand.size());
        outs.push_back(r->out_bits);
    }
    const int rc = mp_bpsw_batches(w, lists.data(), lens.data(), (uint32_t)batch.size(), outs.data());
    for (ServeReq *r : batch) r->res.status = rc;
}

// the device's free memory, read again with cudaMemGetInfo when the last reading is over
// 20 ms old, by one worker at a time and never under the server's lock: the driver call can
// wait behind other threads' copies, and under the lock that wait would hold up every worker
// and every submission
static void refresh_free(mp_server *s)
{
    if (now_s() - s->free_at.load(std::memory_order_relaxed) < 0.020) return;
    int idle = 0;
    if (!s->reading.compare_exchange_strong(idle, 1)) return;
    size_t fr = 0, tot = 0;
    if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) s->free_hbm.store(fr, std::memory_order_relaxed);
    s->free_at.store(now_s(), std::memory_order_relaxed);
    s->reading.store(0);
}

// the bytes of in-flight requests the server may hold now: the option's cap, and no more than
// the device's free memory at the last reading less a reserve.  The workers' scratch was
// allocated at open, so the reading also tracks what other processes on the device take.
static u64 admit_limit(const mp_server *s)
{
    const u64 fr = s->free_hbm.load(std::memory_order_relaxed);
    const u64 by_free = fr > s->reserve ? fr - s->reserve : 0;
    return std::min(s->budget, by_free);
}

static void worker_loop(mp_server *s, mp_handle *w)
{
    cudaSetDevice(w->device);
    for (;;) {
        std::vector<ServeReq *> take;
        refresh_free(s);
        {
            std::unique_lock<std::mutex> lk(s->mu);
            for (;;) {
                if (s->closing && s->pending.empty()) return;
                bool by_mem = false;
                if (!s->pending.empty() && s->inflight < s->max_inflight) {
                    ServeReq *head = s->pending.front();
                    // admission by free device memory; the head always fits when nothing else
                    // holds memory (a single request larger than the limit still runs, alone)
                    if (s->mem_used + head->mem <= admit_limit(s) || s->mem_used == 0) break;
                    by_mem = true;
                }
                if (by_mem) {
                    // held back by memory: read it again (outside the lock) and look again soon
                    lk.unlock();
                    refresh_free(s);
                    lk.lock();
                    s->cv_work.wait_for(lk, std::chrono::milliseconds(2));
                } else {
                    s->cv_work.wait_for(lk, std::chrono::milliseconds(50));
                }
            }
            ServeReq *head = s->pending.front();
            if (head->kind == 1) {
                s->pending.pop_front();
                take.push_back(head);
            } else {
                // merge every waiting primality request (in arrival order) into one launch
                u64 cand = 0;
                for (auto it = s->pending.begin(); it != s->pending.end();) {
                    ServeReq *r = *it;
                    if (r->kind == 2 && (take.empty() || (cand + r->cand.size() <= s->bpsw_cap &&
                                                         s->mem_used + r->mem <= admit_limit(s) &&
                                                         s->inflight + take.size() < s->max_inflight))) {
                        cand += r->cand.size();
                        take.push_back(r);
                        s->mem_used += r->mem;
                        it = s->pending.erase(it);
                    } else ++it;
                }
                for (ServeReq *r : take) s->mem_used -= r->mem;   // re-added below, once
            }
            for (ServeReq *r : take) s->mem_used += r->mem;
            s->inflight += (u32)take.size();
        }
        bool finished = true;
        if (take[0]->kind == 1) finished = run_range(w, take[0]);
        else run_bpsw(w, take);
        {
            std::lock_guard<std::mutex> lk(s->mu);
            const double t = now_s();
            for (ServeReq *r : take) {
                s->mem_used -= r->mem;
                if (!finished) { s->pending.push_back(r); continue; }   // its next turn
                r->res.done_s = t;
                r->done = true;
            }
            s->inflight -= (u32)take.size();
        }
        s->cv_done.notify_all();
        s->cv_work.notify_all();
    }
}

extern "C" {

int mp_serve_open(mp_handle *h, const mp_serve_opts *opts, mp_server **out)
{
    if (!h || !out) return MP_EINVAL;
    *out = nullptr;
    mp_serve_opts o;
    memset(&o, 0, sizeof o);
    if (opts) o = *opts;
    std::lock_guard<std::recursive_mutex> lk(h->mu);
    MP_CUDA(h, cudaSetDevice(h->device));
    const u64 limit = o.prime_limit ? o.prime_limit : (1ull << 30);
    // the resident table covers every height whose square root is below the limit
    MP_TRY(mp_tables_ensure(h, limit > 0xffffffffull ? 0xffffffffull : limit));
    mp_server *s = new mp_server();
    s->main = h;
    s->prime_limit = h->tab->limit;
    size_t fr = 0, tot = 0;
    MP_CUDA(h, cudaMemGetInfo(&fr, &tot));
    s->budget = o.mem_budget ? o.mem_budget : (u64)fr / 2;
    s->max_inflight = o.max_inflight ? o.max_inflight : 256;
    s->chunk = o.chunk ? o.chunk : (1ull << 32);
    const u32 k = o.streams ? o.streams : 4;
    for (u32 i = 0; i < k; i++) {
        mp_handle *w = nullptr;
        int rc = mp_init(h->device, &w);
        if (rc != MP_OK) {
            mp_serve_close(s);
            return mp_set_error(h, rc, "serving worker %u could not be created", i);
        }
        w->tab = h->tab;
        w->shared_tables = true;
        w->pat = h->pat;
        w->pat_ready = true;
        w->no_graphs = true;
        w->tune = h->tune;
        s->workers.push_back(w);
    }
    // Size every worker's scratch for its largest turn now: a buffer that grows later frees
    // the old one, and cudaFree synchronises the whole device, which stalls every worker.
    // The largest turn is the longest chunk at the top height the table serves; the largest
    // primality launch is one merged batch.
    {
        const u64 pl = std::min<u64>(s->prime_limit, 0xffffffffull);
        const u64 top = std::min<u64>(MP_HI_MAX, pl * pl - MP_TAIL);
        const u64 len = std::min<u64>(std::max<u64>(s->chunk, 64 * h->tab->count_le(pl)), top / 2);
        std::vector<u64> zeros(s->bpsw_cap, 0);
        const uint64_t *lists[1] = {zeros.data()};
        const uint32_t lens[1] = {(uint32_t)zeros.size()};
        std::vector<u8> bits(zeros.size() / 8 + 8);
        uint8_t *outs[1] = {bits.data()};
        mp_sieve_opts wo;
        memset(&wo, 0, sizeof wo);
        for (mp_handle *w : s->workers) {
            mp_range_stats st;
            int rc = mp_sieve_range(w, top - len, top, &wo, &st, nullptr, nullptr, nullptr);
            if (rc == MP_OK) rc = mp_bpsw_batches(w, lists, lens, 1, outs);
            if (rc != MP_OK) {
                const int e = mp_set_error(h, rc, "serving worker warm-up failed: %s", w->err);
                mp_serve_close(s);
                return e;
            }
        }
    }
    // the first reading of free memory, with every worker's scratch in place
    if (cudaMemGetInfo(&fr, &tot) == cudaSuccess) s->free_hbm.store(fr);
    s->free_at.store(now_s());
    for (mp_handle *w : s->workers) s->threads.emplace_back(worker_loop, s, w);
    h->servers_open++;
    *out = s;
    return MP_OK;
}

static int submit(mp_server *s, ServeReq *r, uint64_t *req_id)
{
    r->res.submit_s = now_s();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->closing) { delete r; return MP_EINVAL; }
        r->id = s->next_id++;
        s->reqs[r->id] = r;
        s->pending.push_back(r);
    }
    if (req_id) *req_id = r->id;
    s->cv_work.notify_one();
    return MP_OK;
}

int mp_serve_submit_range(mp_server *s, uint64_t lo, uint64_t hi, uint64_t *req_id)
{
    if (!s || hi <= lo || hi > MP_HI_MAX) return MP_EINVAL;
    if (mp_isqrt64(hi + MP_TAIL - 1) > s->prime_limit) return MP_ERANGE;
    ServeReq *r = new ServeReq();
    memset(&r->res, 0, sizeof r->res);
    r->kind = 1;
    r->lo = lo;
    r->hi = hi;
    r->next = lo;
    // every turn sets up the large sieving primes of the range again (about the work of 15
    // integers each), so a turn covers at least 64 integers per sieving prime up to sqrt(hi)
    const u64 np = s->main->tab->count_le(mp_isqrt64(hi + MP_TAIL - 1));
    r->chunk = std::max<u64>(s->chunk, 64 * np);
    r->mem = range_mem(lo, hi - lo > r->chunk ? lo + r->chunk : hi);   // one chunk in flight
    r->res.kind = 1;
    return submit(s, r, req_id);
}

int mp_serve_submit_bpsw(mp_server *s, const uint64_t *n, uint32_t count, uint8_t *verdict_bits, uint64_t *req_id)
{
    if (!s || (count && (!n || !verdict_bits)) || count > (1u << 24)) return MP_EINVAL;
    ServeReq *r = new ServeReq();
    memset(&r->res, 0, sizeof r->res);
    r->kind = 2;
    r->cand.assign(n, n + count);
    r->out_bits = verdict_bits;
    r->mem = bpsw_mem(count);
    r->res.kind = 2;
    r->res.count = count;
    if (!count) {
        // nothing to test: done at once
        std::lock_guard<std::mutex> lk(s->mu);
        r->id = s->next_id++;
        r->done = true;
        r->res.submit_s = r->res.done_s = now_s();
        s->reqs[r->id] = r;
        if (req_id) *req_id = r->id;
        return MP_OK;
    }
    return submit(s, r, req_id);
}

int mp_serve_poll(mp_server *s, uint64_t req_id, mp_serve_result *res, int wait_ms)
{
    if (!s || !res) return MP_EINVAL;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->reqs.find(req_id);
    if (it == s->reqs.end()) return MP_EINVAL;
    ServeReq *r = it->second;
    if (!r->done && wait_ms > 0)
        s->cv_done.wait_for(lk, std::chrono::milliseconds(wait_ms), [&] { return r->done; });
    if (!r->done) return MP_EAGAIN;
    *res = r->res;
    s->reqs.erase(it);
    delete r;
    return MP_OK;
}

int mp_serve_close(mp_server *s)
{
    if (!s) return MP_EINVAL;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->closing = true;
    }
    s->cv_work.notify_all();
    for (auto &t : s->threads) t.join();
    for (mp_handle *w : s->workers) mp_free(w);
    for (auto &kv : s->reqs) delete kv.second;
    if (s->main && !s->threads.empty()) {
        std::lock_guard<std::recursive_mutex> lk(s->main->mu);
        s->main->servers_open--;
    }
    delete s;
    return MP_OK;
}

}  // extern "C"
