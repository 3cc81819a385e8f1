// mp_common.cuh -- shared internals of libmathpub (B200, sm_100a): integer helpers used by
// every kernel, the handle, device buffers and the error plumbing of the C ABI.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/mathpub_gpu.h"

typedef uint8_t u8;
typedef uint16_t u16;
typedef uint32_t u32;
typedef uint64_t u64;
typedef int32_t i32;
typedef int64_t i64;

#define MP_GOLD 0x9E3779B97F4A7C15ULL
#define MP_FNV_OFFSET 0xcbf29ce484222325ULL
#define MP_FNV_PRIME 0x100000001b3ULL
#define MP_NONE (~0ULL)

// Integers sieved past hi so that the prime after the last in-range prime, and the members
// of 6-tuples that start below hi, are known.  The largest prime gap below 2^64 is 1550,
// far below this.
#define MP_TAIL ((u64)1 << 16)
#define MP_HI_MAX (~0ULL - ((u64)1 << 18) + 1)

// ---------------------------------------------------------------------------------------
// host + device integer helpers
// ---------------------------------------------------------------------------------------

// splitmix64 finaliser with the golden-ratio increment (the reference's mix64,
// A350826/a350826.c:425-431)
__host__ __device__ __forceinline__ u64 mp_mix64(u64 z)
{
    z += MP_GOLD;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

// x mod q for x < 2^64, 3 <= q < 2^32, with m = floor((2^64 - 1) / q): the quotient estimate
// umulhi(x, m) is at most 2 below floor(x / q), so two conditional subtractions finish.
__device__ __forceinline__ u32 mp_mod_barrett(u64 x, u32 q, u64 m)
{
    const u64 qh = __umul64hi(x, m);
    u64 r = x - qh * (u64)q;
    if (r >= q) r -= q;
    if (r >= q) r -= q;
    return (u32)r;
}

// index j >= 0 of the first odd multiple x0 + 2j of q that is >= x0 and >= q^2, for odd x0
// and odd prime q; r = x0 mod q.  Returns min(j, cap).
__device__ __forceinline__ u64 mp_first_odd_multiple(u64 x0, u32 q, u32 r, u64 cap)
{
    u64 j;
    if (r == 0) j = 0;
    else {
        const u32 d = q - r;                       // x0 + d = 0 mod q
        j = (d & 1) ? (((u64)d + q) >> 1) : (u64)(d >> 1);   // 64-bit: q may exceed 2^31
    }
    const u64 qq = (u64)q * q;
    if (qq > x0) {
        const u64 jq = (qq - x0) >> 1;             // q^2 = x0 + 2 jq, same class mod q
        j = jq;
    }
    return j < cap ? j : cap;
}

// Wheel of 30 over the odd-only map.  The odd multiples q k of a sieving prime q lie q bits
// apart.  Those with 3 | k or 5 | k are multiples of 3 or 5, which the presieve patterns mark
// in every tile, so a prime q >= 7 marks only the q k with k coprime to 30: 8 of every 15.
// After k = R[w] (mod 30), R = 1, 7, 11, 13, 17, 19, 23, 29, the next such multiple lies
// D[w] q bits on, D = 3, 2, 1, 2, 1, 2, 3, 1 (the 2-bit fields of MP_W30_STEP); one turn of
// the wheel is 15 q bits.
#define MP_W30_STEP 0x799Bu
#define MP_W30_STEP2 0x799B799Bu        // two copies, so rotations by 2 w keep the sequence
// for odd k mod 30 = 2h + 1: the index w of the first R[w] >= 2h + 1 (3-bit fields) and the
// distance to it in q bits (2-bit fields)
#define MP_W30_IDX 0x1ffdac8d2248ull
#define MP_W30_ADV 0x6104118u

// j: bit of an odd multiple q k of the sieving prime q >= 7 (bit j <-> x0 + 2 j), xm = x0 mod
// 30.  Returns the bit of the first multiple q k' >= q k with k' coprime to 30 and sets *w to
// the index of k' mod 30 in R.  k mod 30 = (x0 + 2 j) q^-1 mod 30, and q^-1 = q^3 mod 30
// because every unit mod 30 has an order dividing 4.
__device__ __forceinline__ u64 mp_w30_first(u32 j, u32 xm, u32 q, u32 *w)
{
    const u32 c = q % 30u;
    const u32 inv = (c * c % 30u) * c % 30u;
    const u32 t = (xm + 2u * (j % 15u)) % 30u;
    const u32 h = (t * inv % 30u) >> 1;
    *w = (u32)(MP_W30_IDX >> (3u * h)) & 7u;
    return (u64)j + (u64)q * ((MP_W30_ADV >> (2u * h)) & 3u);
}

// the step fields from residue index w on: the next step is s & 3, then s = rotr(s, 2)
__device__ __forceinline__ u32 mp_w30_steps(u32 w)
{
    return __funnelshift_r(MP_W30_STEP2, MP_W30_STEP2, 2u * w);
}

// sum of the first n (<= 8) step fields of s: the distance in q bits from the residue s starts
// at to the n-th one after it
__device__ __forceinline__ u32 mp_w30_span(u32 s, u32 n)
{
    const u32 x = s & ((1u << (2u * n)) - 1u);
    return __popc(x & 0x55555555u) + 2u * __popc(x & 0xAAAAAAAAu);
}

// ---------------------------------------------------------------------------------------
// handle
// ---------------------------------------------------------------------------------------

// grow-only device buffer; every reallocation bumps *gen (the handle's buffer generation),
// which invalidates CUDA graphs captured with the old pointers
struct DevBuf {
    void *p = nullptr;
    size_t bytes = 0;
    u64 *gen = nullptr;
    cudaError_t ensure(size_t need)
    {
        if (need <= bytes && p) return cudaSuccess;
        if (p) { cudaFree(p); p = nullptr; bytes = 0; }
        if (gen) (*gen)++;
        size_t b = need < 256 ? 256 : need;
        cudaError_t e = cudaMalloc(&p, b);
        if (e == cudaSuccess) bytes = b;
        return e;
    }
    void release()
    {
        if (p) { cudaFree(p); if (gen) (*gen)++; }
        p = nullptr;
        bytes = 0;
    }
    template <class T> T *as() const { return (T *)p; }
};

// presieve patterns: odd numbers 2j+1 divisible by a small prime, as a bit string over j
// with period = the product of the pattern's primes
#define MP_NPAT 5
struct PatternSet {
    u32 period[MP_NPAT];
    u64 words[MP_NPAT];              // u32 words stored per pattern
    u32 *d_words[MP_NPAT];
};

// odd sieving primes 3 <= q <= limit with Barrett constants, resident on the device; a host
// copy of the primes answers the index queries that pick the prime tiers of a launch
struct PrimeTable {
    u64 limit = 0;
    u64 n = 0;
    DevBuf q;                        // u32[n]
    DevBuf magic;                    // u64[n] floor((2^64-1)/q)
    std::vector<u32> host;
    std::vector<double> inv_prefix;  // inv_prefix[i] = sum of 1/q over the first i primes
    u64 count_le(u64 x) const;       // number of table primes <= x
};

struct Autotune {
    int sieve_tile_log2 = 0;         // 0 = not tuned
    int sieve_threads = 0;
    int fermat_variant = 0;
    int bpsw_variant = 0;            // warps per CTA x candidates per chunk of the batched BPSW kernel
    int scatter_staged = 1;          // 1: the staged (sorted) bucket scatter, 0: the binned one
    int bucket_div = 1;              // primes above tile bits / bucket_div (1, 2 or 4) go to the bucket scatter
    int no_pipeline = 0;             // 1: batched sieve calls as a host loop of wave launches
    u64 tuned_at = 0;
};

struct GraphCache;
struct ChainDev;                     // the constellation sieve's plan and buffers (mp_chain.cu)

// per-kernel timing for measurement: when enabled, each launch of a timed kernel category is
// bracketed by CUDA events on its own stream; mp_profile_read sums them
enum { PROF_SCATTER, PROF_TILE, PROF_FOLD, PROF_HASH, PROF_BPSW_BATCHED, PROF_BPSW_PLAIN, PROF_FERMAT,
       PROF_FERMAT_STATS, PROF_PIPELINE, PROF_NCAT };
struct ProfEv {
    int cat;
    cudaEvent_t a, b;
};

struct mp_handle {
    int device = 0;
    int sm_count = 0;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    std::recursive_mutex mu;
    char err[512] = {0};
    double last_ms = 0;

    PrimeTable boot;                 // odd primes < 2^16 (bootstraps the big table)
    PrimeTable table;                // odd primes up to table.limit
    PrimeTable *tab = &table;        // the table in use: a serving worker uses its server's
    bool shared_tables = false;      // tab and pat belong to another handle (never rebuilt here)
    PatternSet pat;
    bool pat_ready = false;
    bool no_graphs = false;          // run batched sieve calls directly (no capture / replay)
    int servers_open = 0;            // servers sharing this handle's table (it may not be rebuilt)

    // scratch
    DevBuf tilesum, blockacc, rec, reccnt, queue, errflag, scratch_bitmap, bpsw_n, bpsw_bits, bpsw_list,
        ferm_p, ferm_q, ferm_part, stats_out, small_out, tstate, gap_acc;
    // CTA bounds of the bucket scatter, one buffer per (first prime, end prime, CTAs): a
    // captured graph reads the buffer it was captured with, so a buffer's contents are never
    // rewritten; the least recently used one is freed (which invalidates the graphs) when a
    // new key needs room
    struct ScatBounds {
        u64 key[3] = {~0ull, ~0ull, ~0ull};
        u32 nblk = 0;
        u64 stamp = 0;
        DevBuf buf;
    };
    static const int NSCAT = 8;
    ScatBounds scat[NSCAT];
    const ScatBounds *scat_cur = nullptr;   // the bounds of the sieve call in progress
    u64 scat_clock = 0;
    std::vector<u32> scat_host;
    u32 *h_err = nullptr;            // pinned mirror of errflag

    Autotune tune;
    GraphCache *graphs = nullptr;
    ChainDev *chain = nullptr;

    u64 buf_gen = 0;                 // bumped by every scratch reallocation
    u64 tune_gen = 0;                // bumped by every change of the tuned sieve plan
    bool prof_on = false;
    std::vector<ProfEv> prof;
    std::vector<cudaEvent_t> prof_pool;
    u64 bpsw_work[4] = {0, 0, 0, 0};
};

// bracket one launch with events when profiling is on (never inside a stream capture)
struct ProfScope {
    mp_handle *h;
    cudaStream_t st;
    int cat;
    cudaEvent_t a = nullptr, b = nullptr;
    ProfScope(mp_handle *h_, int cat_, cudaStream_t st_) : h(h_), st(st_), cat(cat_)
    {
        if (!h->prof_on) return;
        a = take();
        b = take();
        if (a && b) cudaEventRecord(a, st);
    }
    ~ProfScope()
    {
        if (!h->prof_on || !a || !b) return;
        cudaEventRecord(b, st);
        h->prof.push_back({cat, a, b});
    }
    cudaEvent_t take()
    {
        cudaEvent_t e = nullptr;
        if (!h->prof_pool.empty()) { e = h->prof_pool.back(); h->prof_pool.pop_back(); }
        else if (cudaEventCreate(&e) != cudaSuccess) e = nullptr;
        return e;
    }
};

int mp_set_error(mp_handle *h, int code, const char *fmt, ...);

#define MP_CUDA(h, call)                                                                      \
    do {                                                                                      \
        cudaError_t e_ = (call);                                                              \
        if (e_ != cudaSuccess)                                                                \
            return mp_set_error((h), e_ == cudaErrorMemoryAllocation ? MP_ENOMEM : MP_ECUDA,  \
                                "%s failed: %s (%s:%d)", #call, cudaGetErrorString(e_),      \
                                __FILE__, __LINE__);                                          \
    } while (0)

#define MP_TRY(expr)                                                                          \
    do {                                                                                      \
        int r_ = (expr);                                                                      \
        if (r_ != MP_OK) return r_;                                                           \
    } while (0)

static inline cudaStream_t mp_stream_of(mp_handle *h, void *s)
{
    return s ? (cudaStream_t)s : h->stream;
}

static inline u64 mp_isqrt64(u64 n)
{
    u64 r = 0, bit = 1ULL << 62;
    while (bit > n) bit >>= 2;
    while (bit) {
        if (n >= r + bit) { n -= r + bit; r = (r >> 1) + bit; }
        else r >>= 1;
        bit >>= 2;
    }
    return r;
}

// ---- cross-file internal entry points (implemented in the .cu files) ----
int mp_tables_ensure(mp_handle *h, u64 limit);                       // mp_sieve.cu
int mp_patterns_ensure(mp_handle *h);                                // mp_sieve.cu
int mp_sieve_run(mp_handle *h, u64 lo, u64 hi, const mp_sieve_opts *o, mp_range_stats *d_out,
                 mp_block_stats *d_blocks, u64 *d_hash, u64 *d_bitmap, cudaStream_t st);
int mp_sieve_emit_primes(mp_handle *h, u64 lo, u64 hi, u64 *d_primes, u64 cap, u64 *count,
                         cudaStream_t st);                           // synchronises
int mp_sieve_errors(mp_handle *h, cudaStream_t st);                  // synchronises; reads the error flag
int mp_bpsw_run(mp_handle *h, const u64 *d_n, const u64 *offs, const u32 *lens, u32 nlists,
                u32 *d_bits, u32 mode, cudaStream_t st);             // mp_bpsw.cu
const char *mp_bpsw_variant_name(int v);
int mp_fermat_run(mp_handle *h, const u64 *d_p, u64 count, u64 *d_q, cudaStream_t st,
                  int variant, u64 *d_partials);                     // mp_fermat.cu
int mp_fermat_reduce(mp_handle *h, const u64 *d_p, const u64 *d_q, u64 count,
                     mp_wief_stats *d_stats, cudaStream_t st);
void mp_graphs_free(mp_handle *h);                                   // mp_api.cu
void mp_chain_free(mp_handle *h);                                    // mp_chain.cu
