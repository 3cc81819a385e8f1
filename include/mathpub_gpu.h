/*
 * mathpub_gpu.h -- C ABI of the B200 (sm_100a) engine for the integer hot path that the
 * Mathpub OEIS searches share: the segmented odd-only sieve with its prime-count, twin,
 * gap and 6-tuple scans; the 64-bit Montgomery BPSW test; and the Fermat quotient
 * 2^(p-1) mod p^2.
 *
 * Conventions (all entry points):
 *   - plain C types and pointers only; every call returns an int status (MP_OK = 0, or a
 *     negative MP_E* code) and never calls exit();
 *   - mp_last_error() gives a message for the last failing call on a handle;
 *   - a handle owns one CUDA stream, the device-resident sieving-prime tables and scratch
 *     buffers; calls on one handle are serialised internally, so several host threads may
 *     share a handle; separate handles run independently;
 *   - "host" entry points take caller-owned host buffers and copy in and out themselves;
 *     the *_dev variants take device pointers and a cudaStream_t passed as void* (NULL =
 *     the handle's stream) and return without synchronising.
 *
 * Reference interfaces replaced (paths inside the Mathpub project):
 *   mp_bpsw_u64 / mp_bpsw_batches   bool bpsw(u128)          A350826/a350826.c:965
 *                                    (with sprp2_64 :618, slprp64 :766, test_batch64 :1392)
 *   mp_sieve_range                   the segment sieve + scans of process_class
 *                                    A350826/a350826.c:1522, tw_run A007508/a007508.c:368,
 *                                    scan_interval A228768/a228768.c:372, the gap walk of
 *                                    A000230/a000230.c:38-60, and the primesieve calls
 *                                    (primesieve_jump_to / next_prime / count_twins) that
 *                                    e.g. A001220/wieferich.c:1138-1141 makes
 *   mp_fermat_q_base2                u64 fermat_quotient(u64 p, int j, u128 *res)
 *                                    A001220/wieferich.c:939
 *   mp_wieferich_range               scan_chunk + process_batch + finish_lanes
 *                                    A001220/wieferich.c:1129, :1086, :1051
 *   the int-status / caller-owned-buffer style follows the reference's own C/CUDA split,
 *   gapchain/gapsieve_cuda.h:1-70.
 */
#ifndef MATHPUB_GPU_H
#define MATHPUB_GPU_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ---- status codes ---- */
#define MP_OK         0
#define MP_EINVAL    -1   /* bad argument (range, size, null pointer)            */
#define MP_ENOMEM    -2   /* device or host allocation failed                     */
#define MP_ECUDA     -3   /* CUDA runtime error                                   */
#define MP_ETIMEOUT  -4   /* a bounded device wait gave up (error flag set)       */
#define MP_EOVERFLOW -5   /* a device buffer bound was exceeded (retry failed)    */
#define MP_ERANGE    -6   /* outside the supported range (e.g. hi > 2^64 - 2^18)  */
#define MP_EAGAIN    -7   /* serving: result not ready yet                        */
#define MP_EBUSY     -8   /* serving: queue full / not enough free device memory  */

typedef struct mp_handle mp_handle;

/* ---- handle ---- */
int mp_init(int device, mp_handle **out);
int mp_free(mp_handle *h);
const char *mp_last_error(const mp_handle *h);
int mp_version(void);                       /* 100 * major + minor */
/* last device time of the main kernels of the previous call, in milliseconds (CUDA events
   on the handle's stream around the launches; 0 if not timed) */
double mp_last_kernel_ms(const mp_handle *h);

/* ---- sieve ----
 * Odd-only bitmap: base = lo & ~1, bit i <-> the odd number base + 2i + 1, bit = 1 for a
 * prime; in-range bits i < (hi - base) / 2.  Outputs:
 *   pi        number of primes p in [lo, hi) (2 included when lo <= 2 < hi)
 *   twins     number of p in [lo, hi) with p + 2 prime
 *   max_gap   max over primes p in [lo, hi) of nextprime(p) - p (the next prime may lie
 *             beyond hi), gap_start = the smallest p attaining it; 0, 0 without primes
 *   tuple6    number of p in [lo, hi) with p + {0, 4, 6, 10, 12, 16} all prime (members may
 *             lie beyond hi); tuple6_cks = sum of mix64(p) mod 2^64 (splitmix64 finaliser,
 *             A350826/a350826.c:425-438), the reference's order-free checksum
 *   first_prime / last_prime   first and last prime in [lo, hi) (0 if none)
 * Blocks: block b = [lo + b 2^block_log2, lo + (b+1) 2^block_log2) intersected with
 * [lo, hi), nblocks = ceil((hi - lo) / 2^block_log2), with the same fields per block.
 * Hashes: FNV-1a-64 per hash segment of 2^hash_log2 integers = 2^(hash_log2 - 1) bits,
 * over ceil(len/8) bytes (bit j of byte k = bit 8k + j of the segment), nseg =
 * ceil(nbits / 2^(hash_log2 - 1)).
 * Bitmap: ceil(nbits / 64) little-endian u64 words, bits beyond the range zero.
 * Limits: lo < hi <= 2^64 - 2^18.
 */
typedef struct {
    uint64_t pi, twins, max_gap, gap_start, tuple6, tuple6_cks, first_prime, last_prime;
} mp_range_stats;

typedef mp_range_stats mp_block_stats;

/* MP_MODE_BATCHED: the range in waves of tiles; per wave a bucket scatter for the large
 *   primes, then a tile launch in which each CTA sieves a contiguous run of tiles and carries
 *   the state of its sparse primes from tile to tile; the whole call is captured once as a
 *   CUDA graph and replayed.  With the binned scatter (mp_tune_set) and no
 *   MP_TUNE_NO_PIPELINE, one persistent launch runs every wave's scatter and tile work from a
 *   device queue instead.
 * MP_MODE_PLAIN: the reference's per-segment launch loop on a full grid: one launch per group
 *   of SM-count 32 KiB segments, one segment per CTA, every segment set up from scratch,
 *   each group with its own bucket scatter; no graph. */
#define MP_MODE_BATCHED 0
#define MP_MODE_PLAIN   1

typedef struct {
    uint32_t mode;          /* MP_MODE_BATCHED (default) or MP_MODE_PLAIN */
    uint32_t tile_log2;     /* bits per tile: 0 = autotuned, else 18, 19 or 20 */
    uint32_t block_log2;    /* per-block stats width (integers); 0 = none; else >= tile_log2+1 */
    uint32_t hash_log2;     /* hash segment width (integers); 0 = no hashes; else 4..40 */
    uint32_t threads;       /* threads per CTA: 0 = autotuned, else 256, 512 or 1024 */
    uint32_t reserved[3];
} mp_sieve_opts;

/* number of blocks / hash segments / bitmap words that mp_sieve_range fills for [lo, hi) */
uint64_t mp_sieve_nblocks(uint64_t lo, uint64_t hi, uint32_t block_log2);
uint64_t mp_sieve_nhashes(uint64_t lo, uint64_t hi, uint32_t hash_log2);
uint64_t mp_sieve_nwords(uint64_t lo, uint64_t hi);

int mp_sieve_range(mp_handle *h, uint64_t lo, uint64_t hi, const mp_sieve_opts *opts,
                   mp_range_stats *out, mp_block_stats *blocks /* nullable */,
                   uint64_t *seg_hash /* nullable */, uint64_t *bitmap /* nullable */);

/* same with device output buffers (each nullable except d_out) on `stream` (NULL = the
   handle's stream); returns once the work is queued */
int mp_sieve_range_dev(mp_handle *h, uint64_t lo, uint64_t hi, const mp_sieve_opts *opts,
                       mp_range_stats *d_out, mp_block_stats *d_blocks, uint64_t *d_hash,
                       uint64_t *d_bitmap, void *stream);

/* all primes in [lo, hi) in increasing order into a host array of cap entries; *count =
   the number of primes (only min(count, cap) are written) */
int mp_primes_range(mp_handle *h, uint64_t lo, uint64_t hi, uint64_t *primes, size_t cap,
                    size_t *count);

/* ---- gap statistics: consumers of the per-prime gap stream ----
 * For the primes p in [lo, hi), with the primes after p = q_1 < q_2 < ... and gaps
 * g_1 = q_1 - p, g_i = q_i - q_(i-1):
 *   gap_hist[g / 2]   primes whose gap g_1 is the even g (gap_hist[0] holds the gap 1 of
 *                     p = 2); the power sums T_k = sum of count(g) g^k of A252768 come from it
 *                     (A252768/README.md:386-425: the chunk totals of its ordered hand-off)
 *   run_hist[L]       primes with L(p) = L, L(p) = the largest n with g_1 < g_2 < ... < g_n
 *                     (A158939/a158939.c:17-30; L >= 1; run_hist[0] stays 0)
 *   run_first[L]      the smallest such prime, 0 if none (A158939's a(L))
 *   unsettled         primes whose run goes on past the look-ahead of 2^16 integers after hi
 *                     (not counted in run_hist; none below 2^64 is known)
 * Replaces the per-prime walks of A158939/a158939.c:720-770 (its chunk scan) and the gap
 * histogram of A252768/a252768.c (its chunk totals).  hi <= 2^64 - 2^18 - 2^17. */
#define MP_GAP_BINS 1024
#define MP_RUN_MAX 64
#define MP_CHAIN_MAX 32
typedef struct {
    uint64_t gap_hist[MP_GAP_BINS];
    uint64_t run_hist[MP_RUN_MAX];
    uint64_t run_first[MP_RUN_MAX];
    uint64_t unsettled;
    /* chain_hist[L]: primes p in [lo, hi) that head a chain of exactly L consecutive primes
       with gaps 2, 4, 6, ..., 2(L - 1) (A016045; the members are p + m(m + 1), m < L); the
       last bin holds L >= MP_CHAIN_MAX - 1 */
    uint64_t chain_hist[MP_CHAIN_MAX];
} mp_gap_stats;

int mp_gap_stats_range(mp_handle *h, uint64_t lo, uint64_t hi, mp_gap_stats *out);

/* the heads p in [lo, hi) of chains of at least min_len (>= 2) primes with gaps 2, 4, 6, ...,
 * in increasing order, with their lengths (capped at MP_CHAIN_MAX - 1), into caller arrays of
 * cap entries; *count = the number of heads (only min(count, cap) are written).  Replaces the
 * chain walk of gapchain/gapchain_ps.c:336-366 (its default --gaps inc) over the same range. */
int mp_gap_chains(mp_handle *h, uint64_t lo, uint64_t hi, uint32_t min_len, uint64_t *heads, uint32_t *lens,
                  size_t cap, size_t *count);

/* chains by the constellation sieve, which enumerates no primes: residue classes of a wheel,
 * rotated bit patterns of the primes up to 199 over every member, base-2 strong tests of the
 * survivors' members, then exact verification on the GPU (BPSW on the members and on the odd
 * numbers between them).  The method of gapchain/gapsieve.c (gapchain/README_SIEVE.md).
 *   shape MP_CHAIN_INC: gaps 2, 4, 6, ... (A016045); the same heads and lengths as
 *                       mp_gap_chains(lo, hi, k) (2 <= k < MP_CHAIN_MAX; k < 4 is enumerated)
 *   shape MP_CHAIN_DEC: gaps ..., 6, 4, 2 (A263049; 4 <= k < MP_CHAIN_MAX).  A chain is found
 *                       by its k-prime pattern p, p + 2(k-1), ..., which ends it, and is
 *                       reported from its first prime with its full length, as the reference's
 *                       gapchain_ps.c:365-395 and gapsieve.c:888-916 do; p (the key) lies in
 *                       [lo, hi), the first prime may lie below lo
 * heads[] ascending, lens[] capped at MP_CHAIN_MAX - 1; *count = the number of chains. */
#define MP_CHAIN_INC 0u
#define MP_CHAIN_DEC 1u
#define MP_CHAIN_SIEVE_HI_MAX (0xffffffffffffffffull - 4095ull)   /* 2^64 - 2^12 */
int mp_chain_sieve(mp_handle *h, uint64_t lo, uint64_t hi, uint32_t k, uint32_t shape, uint64_t *heads,
                   uint32_t *lens, size_t cap, size_t *count);

/* the first chain of at least k primes (4 <= k < MP_CHAIN_MAX) whose key lies in [lo, hi), as
 * gapsieve --first finds it (gapchain/gapsieve.c:1202-1230, the hit ranked by key): the range is
 * sieved in ascending runs and the call returns after the first run that holds a chain.  The
 * key is the head for MP_CHAIN_INC and, for MP_CHAIN_DEC, the start of the k-prime pattern that
 * ends the chain (what A263049 records); *head is the chain's first prime, *len its length
 * (capped at MP_CHAIN_MAX - 1); *len = 0 when [lo, hi) holds none. */
int mp_chain_first(mp_handle *h, uint64_t lo, uint64_t hi, uint32_t k, uint32_t shape, uint64_t *key,
                   uint64_t *head, uint32_t *len);

/* the same two calls for ranges above 2^64, as the reference's gapsieve searches them: lo, hi,
 * the heads and the keys are 128-bit numbers given as (low word, high word) pairs, and
 * hi <= 3.3e24 (MP_CHAIN128_HI_MAX_W1 2^64 + MP_CHAIN128_HI_MAX_W0), below which Miller-Rabin
 * with the 13 prime bases 2..41 proves primality (Sorenson and Webster 2015; the bound of
 * gapchain/gapsieve.c, PSI13).  Members below 2^64 are certified by BPSW, the others by those
 * 13 bases; heads[2 i], heads[2 i + 1] hold chain i.  k >= 4 for both shapes. */
#define MP_CHAIN128_HI_MAX_W1 178893ull
#define MP_CHAIN128_HI_MAX_W0 6612421877182758912ull
int mp_chain_sieve128(mp_handle *h, const uint64_t lo[2], const uint64_t hi[2], uint32_t k, uint32_t shape,
                      uint64_t *heads, uint32_t *lens, size_t cap, size_t *count);
int mp_chain_first128(mp_handle *h, const uint64_t lo[2], const uint64_t hi[2], uint32_t k, uint32_t shape,
                      uint64_t key[2], uint64_t head[2], uint32_t *len);

/* a prime constellation by the same sieve: *count = the number of p in [lo, hi) with p + offs[i]
 * prime for every i (members may lie beyond hi), *cks = the sum of mix64(p) mod 2^64 over them.
 * offs[0] = 0 < offs[1] < ... < offs[k-1] <= MP_TUPLE_MAXOFF, all even, 2 <= k <= MP_TUPLE_MAXK,
 * hi <= MP_CHAIN_SIEVE_HI_MAX.  With offs = {0, 4, 6, 10, 12, 16} it counts the prime sextuplets
 * of A350826 as that program's class sieve does (process_class A350826/a350826.c:1522, the
 * count and checksum of found :1364-1379): the same count and checksum as mp_sieve_range's
 * tuple6 and tuple6_cks, from a search that sieves the admissible classes only. */
#define MP_TUPLE_MAXK 64
#define MP_TUPLE_MAXOFF 2048
int mp_tuple_count(mp_handle *h, uint64_t lo, uint64_t hi, const uint32_t *offs, uint32_t k, uint64_t *count,
                   uint64_t *cks);
/* the same for ranges above 2^64 (lo, hi as (low word, high word) pairs, hi <= 3.3e24, members
 * above 2^64 certified by the 13 prime bases 2..41); the checksum term of p is the reference's
 * hashp(p) = mix64(lo64(p) ^ hi64(p) * GOLD) (A350826/a350826.c:434-438), mix64(p) below 2^64 */
int mp_tuple_count128(mp_handle *h, const uint64_t lo[2], const uint64_t hi[2], const uint32_t *offs, uint32_t k,
                      uint64_t *count, uint64_t *cks);

/* ---- BPSW ----
 * verdict bit i (bit i & 7 of byte i >> 3) = 1 iff n[i] is prime.  For n < 2^64 this is
 * BPSW (base-2 strong test + strong Lucas test with Selfridge's parameters) after trial
 * division; there is no BPSW pseudoprime below 2^64, so the verdict is exact.
 */
int mp_bpsw_u64(mp_handle *h, const uint64_t *n, size_t count, uint8_t *verdict_bits);

/* many candidate lists of uneven length in one batched call: out[i] receives
   ceil(lens[i] / 8) bytes of verdict bits for lists[i] */
int mp_bpsw_batches(mp_handle *h, const uint64_t *const *lists, const uint32_t *lens,
                    uint32_t nlists, uint8_t *const *out);

/* device form: candidates laid out as nlists lists, list i at d_n + offs[i] (offs[i] a
   multiple of 32, host array offs[0..nlists]), verdict words (u32, bit i & 31 of word
   i >> 5) at d_bits + offs[i] / 32; mode MP_MODE_BATCHED (one persistent launch over
   every list for trial division and the base-2 test, then two launches for the Lucas test
   on the base-2 passers) or MP_MODE_PLAIN (one launch per list) */
int mp_bpsw_lists_dev(mp_handle *h, const uint64_t *d_n, const uint64_t *offs,
                      const uint32_t *lens, uint32_t nlists, uint32_t *d_bits, uint32_t mode,
                      void *stream);

/* ---- Fermat quotient, base 2 ----
 * q = (2^(p-1) mod p^2 - 1) / p for odd primes 3 <= p < 2^63 (A001220/wieferich.c:939);
 * for p = 2 or an even p the entry is 0.  A result that fails Fermat's little theorem
 * (q >= p: a wrong residue) is returned as UINT64_MAX and counted as an error.
 */
int mp_fermat_q_base2(mp_handle *h, const uint64_t *p, size_t count, uint64_t *q_out);
int mp_fermat_q_base2_dev(mp_handle *h, const uint64_t *d_p, size_t count, uint64_t *d_q,
                          void *stream);

/* every prime p in [lo, hi), hi <= 2^63, found by the GPU sieve; per p >= 3: q as above,
 *   primes        number of primes in [lo, hi) (2 included)
 *   tests         number of quotients computed (p >= 3)
 *   near          number of p with 1000 |A| < p, A = the symmetric residue of q
 *                 (A001220/wieferich.c:1068)
 *   flt           number of results failing q < p (0 unless the device is faulty)
 *   cks           sum of mix64(q ^ (p * 0x9E3779B97F4A7C15)) mod 2^64 (the reference's
 *                 checksum, A001220/wieferich.c:1064)
 *   ordered_hash  H <- H * 0x100000001b3 + mix64(p ^ mix64(q)) (mod 2^64) in p order
 *   hits          the Wieferich primes (q = 0): the smallest min(nhits, 16) of the nhits found,
 *                 in increasing order; the other slots are 0 */
typedef struct {
    uint64_t primes, tests, near, flt, cks, ordered_hash, nhits;
    uint64_t hits[16];
} mp_wief_stats;

int mp_wieferich_range(mp_handle *h, uint64_t lo, uint64_t hi, mp_wief_stats *out);

/* The statistics that mp_wieferich_range reports, for device arrays of primes d_p[0..count)
 * and their quotients d_q (as mp_fermat_q_base2_dev writes them), into d_stats in device
 * memory (`primes` there = count), queued on `stream` (NULL = the legacy default stream).
 * For callers that cannot allocate device memory -- a framework whose allocator owns the
 * whole device, or a loop where a cudaMalloc, which may synchronise, is not allowed -- it
 * allocates nothing and takes no handle.  Its scratch is a fixed array of about 400 KB inside
 * the library that every device holds until exit and that all calls on a device share:
 * calls that overlap on the GPU race.  count above MP_NOALLOC_MAX_COUNT is refused with
 * MP_EINVAL.  The first call on a device looks up the array's device address; make that
 * call before any stream capture.  The address is kept for the life of the process, so a
 * device reset (cudaDeviceReset) between calls is not supported.  A CUDA error already
 * pending in the calling thread is left for the caller and the call returns MP_ECUDA
 * without running; an error from this call's own launches is cleared and returned as
 * MP_ECUDA.  This entry point has no counterpart in the reference. */
#define MP_NOALLOC_MAX_COUNT (1u << 24)
int mp_wieferich_stats_noalloc(const uint64_t *d_p, const uint64_t *d_q, uint64_t count,
                               mp_wief_stats *d_stats, void *stream);

/* ---- autotuner ----
 * Times the sieve tile geometry (tile bits x threads) on a short range at height `lo`
 * and the Fermat kernel variants, and keeps the fastest per handle.  Called implicitly
 * (on a small range) by the first call that needs it; call it explicitly to tune for a
 * given height.  *report receives a short text summary (nullable, cap bytes). */
int mp_autotune(mp_handle *h, uint64_t lo, char *report, size_t cap);

/* Sets one of the autotuner's choices on the handle, as mp_autotune would (so that callers
 * and tests can pin each one):
 *   MP_TUNE_TILE_LOG2      sieve tile bits (0 = default, 18, 19, 20)
 *   MP_TUNE_THREADS        sieve threads per CTA (0 = default, 256, 512, 1024)
 *   MP_TUNE_SCATTER_STAGED 1: the staged bucket scatter, 0: the binned one
 *   MP_TUNE_BUCKET_DIV     primes above tile bits / value (1, 2 or 4) go to the buckets
 *   MP_TUNE_NO_PIPELINE    1: batched sieve calls as a host loop of wave launches, 0: one
 *                          persistent pipeline launch (with the binned scatter only; the
 *                          staged scatter always runs the wave loop)
 *   MP_TUNE_BPSW_VARIANT   0..3: warps x candidates per chunk of the batched BPSW kernel
 *   MP_TUNE_FERMAT_ILP2    1: two primes per thread in the Fermat kernel
 * Returns MP_EINVAL for an unknown knob or a value out of range.  No reference counterpart
 * (the reference picks its wheel and chunk by a cost model, A350826/a350826.c:1976-2015). */
#define MP_TUNE_TILE_LOG2 1
#define MP_TUNE_THREADS 2
#define MP_TUNE_SCATTER_STAGED 3
#define MP_TUNE_BUCKET_DIV 4
#define MP_TUNE_NO_PIPELINE 5
#define MP_TUNE_BPSW_VARIANT 6
#define MP_TUNE_FERMAT_ILP2 7
int mp_tune_set(mp_handle *h, int knob, int value);

/* ---- measurement ----
 * mp_profile_enable(h, 1) brackets every launch of the timed kernels with CUDA events on the
 * stream it runs on (batched sieve calls then run directly instead of replaying a captured
 * graph); mp_profile_read fills, for the categories "scatter, tile, fold, hash, bpsw_batched,
 * bpsw_plain, fermat, fermat_stats, pipeline" in that order (the first ncat of them), the
 * launch counts and summed device milliseconds since the previous read.  "pipeline" is the
 * persistent launch that runs a batched sieve call's scatter and tile work together.
 * mp_probe_peaks measures device-wide rates (operations per second): shared-memory atomicOr
 * with the lanes of a warp on distinct banks and on random words, 32-bit integer
 * multiply-adds, and global atomicOr on random words of a 64 MB buffer (the L2 atomic rate).
 * These are the roofline denominators of the sieve and the Montgomery kernels.
 */
int mp_profile_enable(mp_handle *h, int on);
int mp_profile_read(mp_handle *h, uint64_t *launches, double *ms, int ncat);
int mp_probe_peaks(mp_handle *h, double *smem_atomic_conflict_free, double *smem_atomic_random,
                   double *imad32, double *l2_atomic_random);

/* ---- serving (continuous batching) ----
 * Requests of two kinds: range queries [lo, hi) -> pi, max gap (+ start), twins; and
 * primality batches of up to 65536 candidates -> verdict bits.  Requests are admitted
 * while device memory (a budget) and in-flight slots allow; admitted work is cut into
 * tiles and candidate slices that share the device with other requests' work.  A long
 * range runs a chunk at a time and goes back to the end of the queue between chunks, so
 * short requests are not held up behind it.  Every worker's scratch is sized at open for
 * its largest turn, so that no buffer grows (and no cudaFree synchronises the device) while
 * requests run.  Each result is identical to the same request run alone.
 */
typedef struct mp_server mp_server;

typedef struct {
    uint64_t mem_budget;    /* bytes of device memory for in-flight requests (0 = auto) */
    uint32_t max_inflight;  /* requests admitted at once (0 = 256) */
    uint32_t streams;       /* device streams that overlap batches (0 = 4) */
    uint64_t prime_limit;   /* resident sieving primes up to this bound (0 = 2^30: heights to ~1.15e18) */
    uint64_t chunk;         /* a range request runs at least this many integers at a time (and at
                               least 64 per sieving prime up to its sqrt(hi)), then yields to the
                               queue (processor sharing); 0 = 2^32 */
} mp_serve_opts;

typedef struct {
    uint32_t kind;          /* 1 = range, 2 = primality */
    int32_t status;         /* MP_OK or an error code */
    uint64_t pi, max_gap, gap_start, twins;     /* range results */
    uint32_t count;         /* primality: number of candidates */
    double submit_s, done_s;                    /* host clock (seconds) at submit / completion */
} mp_serve_result;

int mp_serve_open(mp_handle *h, const mp_serve_opts *opts, mp_server **out);
int mp_serve_submit_range(mp_server *s, uint64_t lo, uint64_t hi, uint64_t *req_id);
/* the candidates are copied at submit; verdict bits go to `verdict_bits` (caller-owned,
   ceil(count/8) bytes, valid once poll reports the request done) */
int mp_serve_submit_bpsw(mp_server *s, const uint64_t *n, uint32_t count,
                         uint8_t *verdict_bits, uint64_t *req_id);
/* MP_OK and *res filled when done (the request is then retired), MP_EAGAIN if pending;
   waits up to wait_ms milliseconds */
int mp_serve_poll(mp_server *s, uint64_t req_id, mp_serve_result *res, int wait_ms);
int mp_serve_close(mp_server *s);

#ifdef __cplusplus
}
#endif
#endif
