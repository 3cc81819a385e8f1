// mp_primesieve.cu -- the primesieve C API of include/primesieve.h on the B200 sieve, so
// that the Mathpub tools, which call primesieve in 37 source files, link against libmathpub
// unmodified and take their primes from the GPU.
//
// The reference tools' call pattern (e.g. A000230/a000230.c:40-57, A158939/a158939.c:706-770,
// A001220/wieferich.c:1138-1205): one iterator per worker thread, jump_to(lo, hi) then
// next_prime (or the buffer primes[0..size) after generate_next_primes) until the primes pass
// hi.  Here every buffer refill sieves a chunk of the number line on the GPU (count, then
// emit the primes in order) and copies the primes to a pinned host buffer.  Chunks start at
// the stop hint's length (at least 2^20 integers, more than any prime gap below 2^64) and
// double while the iterator keeps going, up to about 2^23 primes per refill.
//
// One handle per process owns the resident table of sieving primes and the presieve patterns;
// every iterator and bulk call borrows a worker (a handle with its own stream and scratch, and
// a pinned host buffer) from a pool, and the workers read the shared table.  A call that needs a larger table grows it
// under an exclusive lock while no worker is sieving.  There is no CPU fallback: without a GPU
// the iterator reports is_error and the bulk calls return their error values.
#include "mp_common.cuh"
#include "../../include/primesieve.h"
#include <algorithm>
#include <math.h>
#include <shared_mutex>
#include <stdlib.h>

namespace {

std::mutex g_mu;                     // the process handle and the worker pool
std::shared_mutex g_tab;             // shared: sieving with the table; exclusive: growing it
mp_handle *g_main = nullptr;
int g_main_err = MP_OK;
struct Worker {
    mp_handle *h = nullptr;
    u64 *buf = nullptr;              // pinned host buffer of primes
    u64 cap = 0;
};
std::vector<Worker *> g_pool;
int g_threads = 0, g_sieve_kib = 32;

const u64 kMaxStop = MP_HI_MAX - 1;  // the largest stop of a range [start, stop]

// the process handle with a first table and the patterns; nullptr when no GPU is usable
mp_handle *process_handle()
{
    std::lock_guard<std::mutex> lk(g_mu);
    if (g_main || g_main_err != MP_OK) return g_main;
    const char *d = getenv("MATHPUB_DEVICE");
    mp_handle *h = nullptr;
    int rc = mp_init(d ? atoi(d) : 0, &h);
    if (rc == MP_OK) {
        std::lock_guard<std::recursive_mutex> hl(h->mu);
        rc = cudaSetDevice(h->device) == cudaSuccess ? mp_tables_ensure(h, 1u << 22) : MP_ECUDA;
    }
    if (rc != MP_OK) {
        if (h) mp_free(h);
        g_main_err = rc;
        return nullptr;
    }
    g_main = h;
    return g_main;
}

Worker *take_worker()
{
    mp_handle *m = process_handle();
    if (!m) return nullptr;
    {
        std::lock_guard<std::mutex> lk(g_mu);
        if (!g_pool.empty()) {
            Worker *w = g_pool.back();
            g_pool.pop_back();
            return w;
        }
    }
    mp_handle *h = nullptr;
    if (mp_init(m->device, &h) != MP_OK) return nullptr;
    h->tab = m->tab;                 // the shared table: never rebuilt through a worker
    h->shared_tables = true;
    h->pat = m->pat;
    h->pat_ready = true;
    h->no_graphs = true;             // the table may be reallocated between calls
    h->tune = m->tune;
    Worker *w = new (std::nothrow) Worker();
    if (!w) { mp_free(h); return nullptr; }
    w->h = h;
    return w;
}

void give_worker(Worker *w)
{
    if (!w) return;
    std::lock_guard<std::mutex> lk(g_mu);
    g_pool.push_back(w);
}

// the worker's pinned buffer holds at least n primes
bool reserve(Worker *w, u64 n)
{
    if (n <= w->cap) return true;
    const u64 c = std::max<u64>(n, 2 * w->cap);
    if (w->buf) cudaFreeHost(w->buf);
    w->buf = nullptr;
    w->cap = 0;
    if (cudaMallocHost(&w->buf, (size_t)c * 8) != cudaSuccess) { w->buf = nullptr; return false; }
    w->cap = c;
    return true;
}

// the shared table must reach sqrt(hi + tail - 1)
int ensure_table(u64 hi)
{
    const u64 need = mp_isqrt64(hi + MP_TAIL - 1);
    {
        std::shared_lock<std::shared_mutex> lk(g_tab);
        if (g_main->tab->limit >= need) return MP_OK;
    }
    std::unique_lock<std::shared_mutex> lk(g_tab);
    std::lock_guard<std::recursive_mutex> hl(g_main->mu);
    if (cudaSetDevice(g_main->device) != cudaSuccess) return MP_ECUDA;
    return mp_tables_ensure(g_main, need);
}

// primes in [lo, hi) (hi <= MP_HI_MAX) into a device buffer of worker w; *n = their number
int sieve_primes(mp_handle *w, u64 lo, u64 hi, u64 *n)
{
    *n = 0;
    if (hi <= lo) return MP_OK;
    MP_TRY(ensure_table(hi));
    std::shared_lock<std::shared_mutex> lk(g_tab);
    std::lock_guard<std::recursive_mutex> hl(w->mu);
    MP_CUDA(w, cudaSetDevice(w->device));
    u64 c = 0, c2 = 0;
    MP_TRY(mp_sieve_emit_primes(w, lo, hi, nullptr, 0, &c, w->stream));
    if (!c) return MP_OK;
    MP_CUDA(w, w->ferm_p.ensure((size_t)c * 8));
    MP_TRY(mp_sieve_emit_primes(w, lo, hi, w->ferm_p.as<u64>(), c, &c2, w->stream));
    *n = c;
    return MP_OK;
}

// copy the first n primes of the worker's device buffer to host memory
int copy_primes(mp_handle *w, u64 *dst, u64 n)
{
    if (!n) return MP_OK;
    MP_CUDA(w, cudaMemcpyAsync(dst, w->ferm_p.p, (size_t)n * 8, cudaMemcpyDeviceToHost, w->stream));
    MP_CUDA(w, cudaStreamSynchronize(w->stream));
    return MP_OK;
}

// at most about 2^23 primes per chunk: the prime density near x is 1 / ln x
u64 max_chunk(u64 x)
{
    const double len = 8388608.0 * log((double)std::max<u64>(x, 64));
    return (u64)std::min(len, 1073741824.0);
}

struct IterState {
    Worker *w = nullptr;             // borrowed at the first refill, returned by free_iterator
    u64 lo = 0, hi = 0;              // the integers [lo, hi) the buffer covers
    bool fresh = true;               // no buffer since the last jump_to
    u64 chunk = 0;                   // length of the last chunk
    u64 err = PRIMESIEVE_ERROR;      // the one-value buffers for errors and "no prime below"
    u64 zero = 0;
};

IterState *state_of(primesieve_iterator *it)
{
    if (!it->memory) it->memory = new (std::nothrow) IterState();
    return (IterState *)it->memory;
}

u64 g_err_value = PRIMESIEVE_ERROR;

void set_error(primesieve_iterator *it, IterState *s)
{
    it->is_error = 1;
    it->primes = s ? &s->err : &g_err_value;
    it->size = 1;
    it->i = 0;
}

// fill the buffer with the primes of [lo, hi); false on an error
bool fill(primesieve_iterator *it, IterState *s, u64 lo, u64 hi, u64 *n)
{
    if (!s->w) s->w = take_worker();
    if (!s->w) return false;
    if (sieve_primes(s->w->h, lo, hi, n) != MP_OK) return false;
    if (!reserve(s->w, *n)) return false;
    if (copy_primes(s->w->h, s->w->buf, *n) != MP_OK) return false;
    it->primes = s->w->buf;
    s->lo = lo;
    s->hi = hi;
    s->fresh = false;
    return true;
}

u64 next_chunk(primesieve_iterator *it, IterState *s, u64 from, bool up)
{
    u64 len;
    if (s->fresh) {
        // the stop hint bounds the first chunk (downwards a hint of 0 means none)
        const u64 hint = up ? (it->stop_hint > from ? it->stop_hint - from : 0)
                            : (it->stop_hint && from > it->stop_hint ? from - it->stop_hint : 0);
        len = hint > ~0ull - (1u << 12) ? hint : hint + (1u << 12);
    } else len = 2 * s->chunk;
    len = std::max<u64>(len, 1u << 20);
    len = std::min<u64>(len, max_chunk(from));
    s->chunk = len;
    return len;
}

// the primes of a range as an array of the requested element type (malloc'd)
void *convert(const u64 *p, u64 n, int type)
{
    size_t es;
    u64 maxv;
    switch (type) {
    case SHORT_PRIMES: case INT16_PRIMES: es = 2; maxv = 0x7fff; break;
    case USHORT_PRIMES: case UINT16_PRIMES: es = 2; maxv = 0xffff; break;
    case INT_PRIMES: case INT32_PRIMES: es = 4; maxv = 0x7fffffff; break;
    case UINT_PRIMES: case UINT32_PRIMES: es = 4; maxv = 0xffffffff; break;
    case LONG_PRIMES: es = sizeof(long); maxv = sizeof(long) == 8 ? 0x7fffffffffffffffull : 0x7fffffff; break;
    case ULONG_PRIMES: es = sizeof(unsigned long); maxv = sizeof(long) == 8 ? ~0ull : 0xffffffff; break;
    case LONGLONG_PRIMES: case INT64_PRIMES: es = 8; maxv = 0x7fffffffffffffffull; break;
    case ULONGLONG_PRIMES: case UINT64_PRIMES: es = 8; maxv = ~0ull; break;
    default: return nullptr;
    }
    if (n && p[n - 1] > maxv) return nullptr;
    char *out = (char *)malloc(std::max<size_t>(1, (size_t)n * es));
    if (!out) return nullptr;
    for (u64 i = 0; i < n; i++) {
        if (es == 2) ((u16 *)out)[i] = (u16)p[i];
        else if (es == 4) ((u32 *)out)[i] = (u32)p[i];
        else ((u64 *)out)[i] = p[i];
    }
    return out;
}

// range statistics on a borrowed worker
int range_stats(u64 lo, u64 hi, mp_range_stats *st)
{
    Worker *w = take_worker();
    if (!w) return MP_ECUDA;
    int rc = ensure_table(hi);
    if (rc == MP_OK) {
        std::shared_lock<std::shared_mutex> lk(g_tab);
        mp_sieve_opts o;
        memset(&o, 0, sizeof o);
        rc = mp_sieve_range(w->h, lo, hi, &o, st, nullptr, nullptr, nullptr);
    }
    give_worker(w);
    return rc;
}

}  // namespace

extern "C" {

void primesieve_init(primesieve_iterator *it)
{
    if (!it) return;
    memset(it, 0, sizeof *it);
    it->stop_hint = kMaxStop;
    IterState *s = state_of(it);
    if (s) it->primes = &s->zero;
    else set_error(it, nullptr);
}

void primesieve_free_iterator(primesieve_iterator *it)
{
    if (!it) return;
    IterState *s = (IterState *)it->memory;
    if (s) {
        give_worker(s->w);
        delete s;
    }
    it->memory = nullptr;
    it->primes = nullptr;
    it->size = it->i = 0;
}

void primesieve_jump_to(primesieve_iterator *it, uint64_t start, uint64_t stop_hint)
{
    if (!it) return;
    IterState *s = state_of(it);
    it->start = start;
    it->stop_hint = stop_hint;
    it->i = it->size = 0;
    it->is_error = 0;
    if (!s) { set_error(it, nullptr); return; }
    it->primes = &s->zero;
    s->fresh = true;
    s->chunk = 0;
    s->lo = s->hi = start;
}

void primesieve_clear(primesieve_iterator *it) { primesieve_jump_to(it, 0, kMaxStop); }

void primesieve_generate_next_primes(primesieve_iterator *it)
{
    IterState *s = state_of(it);
    if (!s) { set_error(it, nullptr); return; }
    u64 lo = s->fresh ? it->start : s->hi;
    for (;;) {
        if (lo > kMaxStop) { set_error(it, s); return; }
        const u64 len = next_chunk(it, s, lo, true);
        const u64 hi = std::min<u64>(lo + len, kMaxStop + 1);
        u64 n = 0;
        if (!fill(it, s, lo, hi, &n)) { set_error(it, s); return; }
        if (n) {
            it->size = n;
            it->i = 0;
            it->is_error = 0;
            return;
        }
        lo = hi;                     // no prime in the chunk (only at the very top): go on
    }
}

void primesieve_generate_prev_primes(primesieve_iterator *it)
{
    IterState *s = state_of(it);
    if (!s) { set_error(it, nullptr); return; }
    // after jump_to the previous prime may be start itself
    u64 hi = s->fresh ? (it->start >= kMaxStop ? kMaxStop + 1 : it->start + 1) : s->lo;
    for (;;) {
        if (hi <= 2) {               // nothing below: primesieve returns 0
            it->primes = &s->zero;
            it->size = 1;
            it->i = 0;
            s->lo = s->hi = 0;
            s->fresh = false;
            return;
        }
        const u64 len = next_chunk(it, s, hi, false);
        const u64 lo = hi > len ? hi - len : 0;
        u64 n = 0;
        if (!fill(it, s, lo, hi, &n)) { set_error(it, s); return; }
        if (n) {
            it->size = n;
            it->i = n - 1;
            it->is_error = 0;
            return;
        }
        hi = lo;
    }
}

void *primesieve_generate_primes(uint64_t start, uint64_t stop, size_t *size, int type)
{
    if (size) *size = 0;
    if (stop > kMaxStop || !size) return nullptr;
    if (start > stop) return convert(nullptr, 0, type);
    Worker *w = take_worker();
    if (!w) return nullptr;
    u64 n = 0;
    void *out = nullptr;
    if (sieve_primes(w->h, start, stop + 1, &n) == MP_OK) {
        std::vector<u64> p(n);
        if (copy_primes(w->h, p.data(), n) == MP_OK) {
            out = convert(p.data(), n, type);
            if (out) *size = (size_t)n;
        }
    }
    give_worker(w);
    return out;
}

void *primesieve_generate_n_primes(uint64_t n, uint64_t start, int type)
{
    std::vector<u64> all;
    all.reserve((size_t)std::min<u64>(n, 1ull << 26));
    primesieve_iterator it;
    primesieve_init(&it);
    primesieve_jump_to(&it, start, kMaxStop);
    bool ok = true;
    while (all.size() < n) {
        primesieve_generate_next_primes(&it);
        if (it.is_error) { ok = false; break; }
        const u64 take = std::min<u64>(it.size, n - all.size());
        all.insert(all.end(), it.primes, it.primes + take);
    }
    primesieve_free_iterator(&it);
    return ok ? convert(all.data(), all.size(), type) : nullptr;
}

void primesieve_free(void *primes) { free(primes); }

uint64_t primesieve_count_primes(uint64_t start, uint64_t stop)
{
    if (stop > kMaxStop) return PRIMESIEVE_ERROR;
    if (start > stop) return 0;
    mp_range_stats st;
    return range_stats(start, stop + 1, &st) == MP_OK ? st.pi : PRIMESIEVE_ERROR;
}

uint64_t primesieve_count_twins(uint64_t start, uint64_t stop)
{
    if (stop > kMaxStop) return PRIMESIEVE_ERROR;
    if (stop < 2 || start > stop - 2) return 0;
    // pairs (p, p + 2) with start <= p and p + 2 <= stop: first members p in [start, stop - 1)
    mp_range_stats st;
    return range_stats(start, stop - 1, &st) == MP_OK ? st.twins : PRIMESIEVE_ERROR;
}

uint64_t primesieve_get_max_stop(void) { return kMaxStop; }
void primesieve_set_num_threads(int num_threads) { g_threads = num_threads; }
int primesieve_get_num_threads(void) { return g_threads; }
void primesieve_set_sieve_size(int sieve_size) { g_sieve_kib = sieve_size; }
int primesieve_get_sieve_size(void) { return g_sieve_kib; }
const char *primesieve_version(void) { return PRIMESIEVE_VERSION; }

}  // extern "C"
