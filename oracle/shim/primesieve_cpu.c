/*
 * primesieve_cpu.c -- the CPU stand-in declared in shim/primesieve.h (test infrastructure;
 * only the reference-tool checker under oracle/_ref links it).  Primes come from the
 * oracle's odd-only segmented sieve.
 */
#include <stdlib.h>
#include <string.h>
#include "primesieve.h"

size_t or_primes_range(uint64_t lo, uint64_t hi, uint64_t *out, size_t cap, int threads);

#define CHUNK ((uint64_t)1 << 22)   /* integers buffered per refill */

void primesieve_init(primesieve_iterator *it) { memset(it, 0, sizeof *it); }

void primesieve_free_iterator(primesieve_iterator *it) { free(it->primes); free(it->pbuf); memset(it, 0, sizeof *it); }

void primesieve_jump_to(primesieve_iterator *it, uint64_t start, uint64_t stop_hint)
{
    it->i = it->size = 0;
    it->next_lo = start;
    it->stop_hint = stop_hint;
    it->pi = 0;
    it->prev_hi = start + 1;          /* prev_prime starts with the last prime <= start */
}

static void refill(primesieve_iterator *it)
{
    it->i = it->size = 0;
    while (it->size == 0) {
        const uint64_t lo = it->next_lo;
        if (lo >= PRIMESIEVE_ERROR - CHUNK) { it->primes = realloc(it->primes, 8); it->primes[0] = PRIMESIEVE_ERROR; it->size = 1; return; }
        const uint64_t hi = lo + CHUNK;
        const size_t cap = CHUNK / 2 + 8;
        if (it->cap < cap) { it->primes = realloc(it->primes, cap * 8); it->cap = cap; }
        it->size = or_primes_range(lo, hi, it->primes, cap, 1);
        it->next_lo = hi;
    }
}

uint64_t primesieve_prev_prime(primesieve_iterator *it)
{
    while (it->pi == 0) {
        if (it->prev_hi <= 2) return 0;
        const uint64_t hi = it->prev_hi, lo = hi > CHUNK ? hi - CHUNK : 0;
        const size_t cap = (size_t)((hi - lo) / 2 + 8);
        if (it->pcap < cap) { it->pbuf = realloc(it->pbuf, cap * 8); it->pcap = cap; }
        it->pi = or_primes_range(lo, hi, it->pbuf, cap, 1);
        it->prev_hi = lo;
    }
    return it->pbuf[--it->pi];
}

void primesieve_generate_next_primes(primesieve_iterator *it)
{
    refill(it);
    it->is_error = it->size == 1 && it->primes[0] == PRIMESIEVE_ERROR;
}

uint64_t primesieve_next_prime(primesieve_iterator *it)
{
    if (it->i >= it->size) refill(it);
    return it->primes[it->i++];
}

void *primesieve_generate_primes(uint64_t start, uint64_t stop, size_t *size, int type)
{
    /* stop is inclusive in primesieve */
    const uint64_t hi = stop + 1;
    size_t cap = hi > start ? (size_t)((hi - start) / 2 + 8) : 8;
    uint64_t *p = malloc(cap * 8);
    size_t n = hi > start ? or_primes_range(start, hi, p, cap, 1) : 0;
    *size = n;
    if (type == UINT32_PRIMES || type == INT32_PRIMES || type == UINT_PRIMES || type == INT_PRIMES) {
        uint32_t *q = malloc(n * 4 + 4);
        for (size_t i = 0; i < n; i++) q[i] = (uint32_t)p[i];
        free(p);
        return q;
    }
    return p;
}

void primesieve_free(void *primes) { free(primes); }

uint64_t primesieve_count_primes(uint64_t start, uint64_t stop)
{
    size_t n;
    void *p = primesieve_generate_primes(start, stop, &n, UINT64_PRIMES);
    free(p);
    return n;
}

uint64_t primesieve_count_twins(uint64_t start, uint64_t stop)
{
    size_t n;
    uint64_t *p = primesieve_generate_primes(start, stop, &n, UINT64_PRIMES), c = 0;
    for (size_t i = 0; i + 1 < n; i++) c += p[i + 1] - p[i] == 2;
    free(p);
    return c;
}

uint64_t primesieve_get_max_stop(void) { return PRIMESIEVE_ERROR - 1; }
void primesieve_set_num_threads(int num_threads) { (void)num_threads; }
void primesieve_set_sieve_size(int sieve_size) { (void)sieve_size; }
