/*
 * primesieve.h -- minimal CPU stand-in for the primesieve C API (kimwalisch/primesieve,
 * pinned >= 11 by the Mathpub tools), used ONLY to compile the reference's own tools
 * (A001220/wieferich.c) as a checker under oracle/_ref.  Test infrastructure: the primes
 * come from the oracle's odd-only sieve (mp_oracle.c).  Only the calls those tools make
 * are provided; the iterator fields are this stand-in's own.
 */
#ifndef MATHPUB_ORACLE_PRIMESIEVE_H
#define MATHPUB_ORACLE_PRIMESIEVE_H
#include <stdint.h>
#include <stddef.h>

#define PRIMESIEVE_ERROR ((uint64_t)~0ULL)
enum { SHORT_PRIMES, USHORT_PRIMES, INT_PRIMES, UINT_PRIMES, LONG_PRIMES, ULONG_PRIMES,
       LONGLONG_PRIMES, ULONGLONG_PRIMES, INT16_PRIMES, UINT16_PRIMES, INT32_PRIMES,
       UINT32_PRIMES, INT64_PRIMES, UINT64_PRIMES };

typedef struct {
    size_t i, size;        /* next index into primes[], number of buffered primes */
    uint64_t next_lo;      /* first number not yet covered by the buffer */
    uint64_t stop_hint;
    uint64_t *primes;
    size_t cap;
    int is_error;
    uint64_t *pbuf;        /* backward buffer of prev_prime: pbuf[0..pi) are still to come */
    size_t pi, pcap;
    uint64_t prev_hi;      /* the primes below it are not buffered yet */
} primesieve_iterator;

void primesieve_init(primesieve_iterator *it);
void primesieve_free_iterator(primesieve_iterator *it);
void primesieve_jump_to(primesieve_iterator *it, uint64_t start, uint64_t stop_hint);
uint64_t primesieve_next_prime(primesieve_iterator *it);
void primesieve_generate_next_primes(primesieve_iterator *it);   /* primes[0..size), i = 0 */
uint64_t primesieve_prev_prime(primesieve_iterator *it);         /* 0 below 2 */
void *primesieve_generate_primes(uint64_t start, uint64_t stop, size_t *size, int type);
void primesieve_free(void *primes);
uint64_t primesieve_count_primes(uint64_t start, uint64_t stop);
uint64_t primesieve_count_twins(uint64_t start, uint64_t stop);
uint64_t primesieve_get_max_stop(void);
void primesieve_set_num_threads(int num_threads);
void primesieve_set_sieve_size(int sieve_size);
#endif
