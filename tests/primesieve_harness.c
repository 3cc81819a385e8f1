/*
 * primesieve_harness.c -- drives the primesieve drop-in (include/primesieve.h, libmathpub.so)
 * the way the Mathpub tools do and prints one JSON line per operation, for
 * tests/test_primesieve.py to compare with the oracle.  Sums are mod 2^64: s1 = sum of p,
 * s2 = sum of i * p over the i-th value (0-based), so that order errors show.
 *
 *   next  START HINT N        N primes from next_prime after jump_to(START, HINT)
 *   prev  START N             up to N primes from prev_prime after jump_to(START, 0),
 *                             stopping at the 0 that means "no prime below"
 *   buffer LO HI              generate_next_primes until the buffer passes HI (primes < HI)
 *   mixed START               next x3, prev x5, next x10 after jump_to(START, START + 1000)
 *   gen   START STOP TYPE     generate_primes (TYPE 64 or 32)
 *   genn  N START             generate_n_primes, 64-bit
 *   count START STOP          count_primes and count_twins
 *   top                       get_max_stop, and an iterator jumped past it
 */
#include <inttypes.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "primesieve.h"

static uint64_t num(const char *s) { return strtoull(s, NULL, 0); }

static void emit(const char *op, uint64_t n, uint64_t first, uint64_t last, uint64_t s1, uint64_t s2, int err)
{
    printf("{\"op\": \"%s\", \"n\": %" PRIu64 ", \"first\": %" PRIu64 ", \"last\": %" PRIu64 ", \"s1\": %" PRIu64
           ", \"s2\": %" PRIu64 ", \"err\": %d}\n", op, n, first, last, s1, s2, err);
}

int main(int argc, char **argv)
{
    if (argc < 2) return 2;
    const char *op = argv[1];
    uint64_t n = 0, first = 0, last = 0, s1 = 0, s2 = 0;
    int err = 0;
    primesieve_iterator it;
    primesieve_init(&it);
    if (!strcmp(op, "next") && argc == 5) {
        primesieve_jump_to(&it, num(argv[2]), num(argv[3]));
        const uint64_t want = num(argv[4]);
        for (; n < want; n++) {
            const uint64_t p = primesieve_next_prime(&it);
            if (it.is_error) { err = 1; last = p; break; }
            if (!n) first = p;
            last = p; s1 += p; s2 += n * p;
        }
    } else if (!strcmp(op, "prev") && argc == 4) {
        primesieve_jump_to(&it, num(argv[2]), 0);
        const uint64_t want = num(argv[3]);
        for (; n < want; n++) {
            const uint64_t p = primesieve_prev_prime(&it);
            if (it.is_error) { err = 1; break; }
            if (!n) first = p;
            last = p; s1 += p; s2 += n * p;
            if (!p) { n++; break; }
        }
    } else if (!strcmp(op, "buffer") && argc == 4) {
        const uint64_t lo = num(argv[2]), hi = num(argv[3]);
        primesieve_jump_to(&it, lo, hi);
        int done = 0;
        while (!done) {
            primesieve_generate_next_primes(&it);
            if (it.is_error || it.size == 0) { err = 1; break; }
            for (size_t i = 0; i < it.size; i++) {
                const uint64_t p = it.primes[i];
                if (p >= hi) { done = 1; break; }
                if (!n) first = p;
                last = p; s1 += p; s2 += n * p; n++;
            }
        }
    } else if (!strcmp(op, "mixed") && argc == 3) {
        const uint64_t start = num(argv[2]);
        primesieve_jump_to(&it, start, start + 1000);
        const int steps[3] = {3, -5, 10};
        for (int k = 0; k < 3; k++) {
            const int c = steps[k] > 0 ? steps[k] : -steps[k];
            for (int j = 0; j < c; j++) {
                const uint64_t p = steps[k] > 0 ? primesieve_next_prime(&it) : primesieve_prev_prime(&it);
                if (it.is_error) err = 1;
                if (!n) first = p;
                last = p; s1 += p; s2 += n * p; n++;
            }
        }
    } else if (!strcmp(op, "gen") && argc == 5) {
        size_t sz = 0;
        const int bits = atoi(argv[4]);
        void *v = primesieve_generate_primes(num(argv[2]), num(argv[3]), &sz, bits == 32 ? UINT32_PRIMES : UINT64_PRIMES);
        if (!v) err = 1;
        for (size_t i = 0; v && i < sz; i++) {
            const uint64_t p = bits == 32 ? ((uint32_t *)v)[i] : ((uint64_t *)v)[i];
            if (!n) first = p;
            last = p; s1 += p; s2 += n * p; n++;
        }
        primesieve_free(v);
    } else if (!strcmp(op, "genn") && argc == 4) {
        const uint64_t want = num(argv[2]);
        uint64_t *v = (uint64_t *)primesieve_generate_n_primes(want, num(argv[3]), UINT64_PRIMES);
        if (!v) err = 1;
        for (uint64_t i = 0; v && i < want; i++) {
            const uint64_t p = v[i];
            if (!n) first = p;
            last = p; s1 += p; s2 += n * p; n++;
        }
        primesieve_free(v);
    } else if (!strcmp(op, "count") && argc == 4) {
        const uint64_t a = num(argv[2]), b = num(argv[3]);
        n = primesieve_count_primes(a, b);
        s1 = primesieve_count_twins(a, b);
        err = n == PRIMESIEVE_ERROR || s1 == PRIMESIEVE_ERROR;
    } else if (!strcmp(op, "top") && argc == 2) {
        first = primesieve_get_max_stop();
        primesieve_jump_to(&it, first + 1, ~(uint64_t)0);
        last = primesieve_next_prime(&it);
        err = it.is_error;
    } else {
        primesieve_free_iterator(&it);
        return 2;
    }
    primesieve_free_iterator(&it);
    emit(op, n, first, last, s1, s2, err);
    return 0;
}
