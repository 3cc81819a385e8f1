/*
 * primesieve.h -- drop-in for the primesieve C API (kimwalisch/primesieve, pinned >= 11 by the
 * Mathpub tools), backed by the B200 sieve of libmathpub.  A tool that includes this header
 * and links -lmathpub instead of -lprimesieve gets its primes from the GPU.
 *
 * Provided: the calls the Mathpub tools make (the iterator, bulk generation, counting and
 * the settings).  The list, with the reference call sites each one replaces:
 *   primesieve_init / free_iterator / jump_to / next_prime / prev_prime
 *       e.g. A000230/a000230.c:40-57, A001220/wieferich.c:1138-1205, gapchain/gapchain_ps.c:323
 *   primesieve_generate_next_primes   A158939/a158939.c:712,767, A053686/a053686.c:954,971,
 *                                     A003630/a003630.c:455 (the buffer primes[0..size) is read directly)
 *   primesieve_generate_primes / primesieve_free
 *                                     A158939/a158939.c:1299, A053686/a053686.c:1634, A137723/a137723.c:601
 *   primesieve_generate_n_primes      A128344/a128344.c:325
 *   primesieve_count_primes           A053686/a053686.c:1591
 *   primesieve_count_twins            A007508/a007508.c:592
 *   primesieve_get_max_stop           A252768/a252768.c:1462, A158939/a158939.c:1081
 *   primesieve_set_num_threads        A007508/a007508.c:785
 *   primesieve_set_sieve_size         A158939/a158939.c:856
 *
 * Semantics (as the tools rely on them):
 *   - after primesieve_jump_to(it, start, stop_hint), primesieve_next_prime() returns the first
 *     prime >= start and primesieve_prev_prime() the last prime <= start;
 *   - primesieve_generate_next_primes() fills it->primes[0..it->size) with the next primes in
 *     increasing order and sets it->i = 0; primesieve_generate_prev_primes() fills it with the
 *     primes below the buffer in increasing order and sets it->i = it->size - 1;
 *   - on an error (no GPU, a range beyond primesieve_get_max_stop()) it->is_error is set and
 *     the buffer holds the single value PRIMESIEVE_ERROR; primesieve_prev_prime() returns 0
 *     below 2, as primesieve does.
 * The buffer is refilled a chunk of the number line at a time on the GPU (up to several million
 * primes per refill, where primesieve takes about a thousand); stop_hint bounds the first
 * chunk.  Iterators are per thread, as in primesieve; all iterators of a process share one
 * resident table of sieving primes per device.  The device is MATHPUB_DEVICE (default 0).
 * There is no CPU fallback.
 */
#ifndef MATHPUB_PRIMESIEVE_H
#define MATHPUB_PRIMESIEVE_H

#include <stddef.h>
#include <stdint.h>

#define PRIMESIEVE_VERSION "12.0-mathpub-b200"
#define PRIMESIEVE_ERROR ((uint64_t)~(uint64_t)0)

#ifdef __cplusplus
extern "C" {
#endif

/* element types for primesieve_generate_primes / primesieve_generate_n_primes */
enum { SHORT_PRIMES, USHORT_PRIMES, INT_PRIMES, UINT_PRIMES, LONG_PRIMES, ULONG_PRIMES, LONGLONG_PRIMES,
       ULONGLONG_PRIMES, INT16_PRIMES, UINT16_PRIMES, INT32_PRIMES, UINT32_PRIMES, INT64_PRIMES, UINT64_PRIMES };

typedef struct {
    size_t i;            /* index of the current prime in primes[] */
    size_t size;         /* primes in the buffer */
    uint64_t start;      /* the start of the last jump_to */
    uint64_t stop_hint;  /* the stop hint of the last jump_to */
    uint64_t *primes;    /* the buffer */
    void *memory;        /* the iterator's state (owned by the library) */
    int is_error;
} primesieve_iterator;

void primesieve_init(primesieve_iterator *it);
void primesieve_free_iterator(primesieve_iterator *it);
void primesieve_clear(primesieve_iterator *it);
void primesieve_jump_to(primesieve_iterator *it, uint64_t start, uint64_t stop_hint);
void primesieve_generate_next_primes(primesieve_iterator *it);
void primesieve_generate_prev_primes(primesieve_iterator *it);

static inline uint64_t primesieve_next_prime(primesieve_iterator *it)
{
    it->i++;
    if (it->i >= it->size) primesieve_generate_next_primes(it);
    return it->primes[it->i];
}

static inline uint64_t primesieve_prev_prime(primesieve_iterator *it)
{
    if (it->i == 0) primesieve_generate_prev_primes(it);
    else it->i--;
    return it->primes[it->i];
}

/* primes in [start, stop] as an array of `type` (free with primesieve_free); NULL and
   *size = 0 on an error */
void *primesieve_generate_primes(uint64_t start, uint64_t stop, size_t *size, int type);
/* the first n primes >= start */
void *primesieve_generate_n_primes(uint64_t n, uint64_t start, int type);
void primesieve_free(void *primes);

/* primes, and twin pairs (p, p + 2) with both members, in [start, stop]; PRIMESIEVE_ERROR on an
   error */
uint64_t primesieve_count_primes(uint64_t start, uint64_t stop);
uint64_t primesieve_count_twins(uint64_t start, uint64_t stop);

uint64_t primesieve_get_max_stop(void);
/* accepted for compatibility; the GPU sieve picks its own geometry */
void primesieve_set_num_threads(int num_threads);
int primesieve_get_num_threads(void);
void primesieve_set_sieve_size(int sieve_size);
int primesieve_get_sieve_size(void);
const char *primesieve_version(void);

#ifdef __cplusplus
}
#endif

#endif
