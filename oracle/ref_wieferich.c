/*
 * ref_wieferich.c -- builds the reference's own A001220/wieferich.c (Fermat quotients
 * mod p^2) into oracle/_ref/libref_wieferich.so as a checker and CPU baseline, against the
 * CPU primesieve stand-in in oracle/shim.
 *
 * TEST INFRASTRUCTURE ONLY.  The reference source is included from the reference tree at
 * build time (see oracle/Makefile); nothing of it is copied into this repository.
 */
#define main mathpub_ref_wieferich_main
#include "A001220/wieferich.c"
#undef main

static void ref_bases2(void)
{
    static bool done = false;
    if (!done) { const u32 b = 2; bases_setup(&b, 1); done = true; }
}

/* q_p(2) through the reference's production kernel (fermat_quotient, :939) */
u64 ref_fermat_q2(u64 p, u64 *res_lo, u64 *res_hi)
{
    ref_bases2();
    u128 r;
    const u64 q = fermat_quotient(p, 0, &r);
    if (res_lo) *res_lo = (u64)r;
    if (res_hi) *res_hi = (u64)(r >> 64);
    return q;
}

/* quotients for a list of odd primes, LANES per group through run_group (:914), split over
   threads: the reference's fast path for one base */
typedef struct { const u64 *p; u64 *q; size_t a, b; } rf_job;

static void *ref_fermat_part(void *arg)
{
    rf_job *j = (rf_job *)arg;
    pctx_t ctx[LANES];
    lane_t L[LANES];
    u128 r[LANES];
    for (size_t i = j->a; i < j->b; i += LANES) {
        int nl = 0;
        for (; nl < LANES && i + (size_t)nl < j->b; nl++) {
            pctx_init(&ctx[nl], j->p[i + nl]);
            L[nl].c = &ctx[nl]; L[nl].pw = B.pw[0]; L[nl].e = j->p[i + nl] - 1; L[nl].j = 0;
        }
        for (int g = nl; g < LANES; g++) L[g] = L[nl - 1];
        run_group(L, B.w[0], r);
        for (int g = 0; g < nl; g++) j->q[i + g] = ((u64)r[g] - 1) * ctx[g].pinv;
    }
    return NULL;
}

void ref_fermat_batch(const u64 *p, size_t count, u64 *q, int threads)
{
    ref_bases2();
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t th[256];
    rf_job jb[256];
    size_t per = (count + (size_t)threads - 1) / (size_t)threads;
    int k = 0;
    for (size_t a = 0; a < count && k < threads; a += per, k++) {
        jb[k].p = p; jb[k].q = q; jb[k].a = a; jb[k].b = a + per < count ? a + per : count;
        pthread_create(&th[k], NULL, ref_fermat_part, &jb[k]);
    }
    for (int i = 0; i < k; i++) pthread_join(th[i], NULL);
}

/* the reference scan of [lo, hi) for base 2 (run_scan, :1382): prime count and checksum,
   as one line of its chunk log would report them */
int ref_wieferich_scan(u64 lo, u64 hi, int threads, u64 *primes, u64 *cks, u64 *flt)
{
    ref_bases2();
    g_print = false;
    const u64 span = hi - lo;
    u64 k = (u64)threads * 8;
    while (k > 1 && span % k) k--;
    run_scan(lo, hi, span / k, threads, NULL, 60, true);
    *primes = S.primes;
    *cks = S.cks[0];
    *flt = S.flt;
    return 0;
}
