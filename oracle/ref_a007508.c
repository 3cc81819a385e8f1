/*
 * ref_a007508.c -- builds the reference's own A007508/a007508.c twin-class sieve into
 * oracle/_ref/libref_a007508.so, as a checker of twin counts and as the reference's own CPU
 * sieve for the timed baseline.
 *
 * TEST INFRASTRUCTURE ONLY.  The reference source is included from the reference tree at
 * build time (see oracle/Makefile); nothing of it is copied into this repository.  Its
 * sieving primes come from the CPU stand-in for primesieve in shim/ (the oracle's sieve),
 * since primesieve itself is not vendored.
 */
#define main mathpub_ref_a007508_main
#include "A007508/a007508.c"
#undef main

static pthread_once_t ref_tw_once = PTHREAD_ONCE_INIT;

/* the table set-up the reference's main runs before any count (A007508/a007508.c:782-785) */
static void ref_tw_init(void)
{
    wheel_init();
    presieve_init();
    presieve2_init();
    primesieve_set_num_threads(1);
}

typedef struct { uint64_t K0, K1, seg_k, count; } rtw_job;

static void *ref_tw_part(void *arg)
{
    rtw_job *j = (rtw_job *)arg;
    j->count = count_twins_twin(j->K0, j->K1, j->seg_k);
    return NULL;
}

/* Twin pairs (p, p + 2) with p = 30k + r, r in {11, 17, 29}, K0 <= k < K1: the reference's
 * twin kernel (count_twins_twin, A007508/a007508.c:514) with its default segment of 2^22
 * k-units, the k-range split evenly over `threads` workers.  For lo and hi multiples of 30
 * (K0 = lo / 30, K1 = hi / 30) this is the number of twin pairs with lo <= p < hi, lo > 5. */
uint64_t ref_twins_k(uint64_t K0, uint64_t K1, int threads)
{
    pthread_once(&ref_tw_once, ref_tw_init);
    if (K1 <= K0) return 0;
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t th[256];
    rtw_job jb[256];
    const uint64_t per = (K1 - K0 + (uint64_t)threads - 1) / (uint64_t)threads;
    int k = 0;
    for (uint64_t a = K0; a < K1 && k < threads; a += per, k++) {
        jb[k].K0 = a;
        jb[k].K1 = a + per < K1 ? a + per : K1;
        jb[k].seg_k = 1ULL << 22;
        jb[k].count = 0;
        pthread_create(&th[k], NULL, ref_tw_part, &jb[k]);
    }
    uint64_t total = 0;
    for (int i = 0; i < k; i++) {
        pthread_join(th[i], NULL);
        total += jb[i].count;
    }
    return total;
}
