/*
 * ref_a350826.c -- builds the reference's own A350826/a350826.c (BPSW and the sextuplet
 * counter) into oracle/_ref/libref_a350826.so as a checker and CPU baseline.
 *
 * TEST INFRASTRUCTURE ONLY.  The reference source is included from the reference tree
 * at build time (see oracle/Makefile); nothing of it is copied into this repository.
 * Each wrapper calls the reference's static functions unchanged.
 */
#define main mathpub_ref_a350826_main
#include "A350826/a350826.c"
#undef main

/* the reference's own verdict for any n < 2^64, with the small-factor handling that its
   callers do before bpsw() (cmd_check, A350826/a350826.c:2287; bpsw needs odd n > 41
   without a factor <= 41) */
int ref_bpsw(u64 n)
{
    static const u32 sp[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41};
    if (n < 2) return 0;
    for (int i = 0; i < 13; i++) {
        if (n == sp[i]) return 1;
        if (n % sp[i] == 0) return 0;
    }
    if (n < 43 * 43) return 1;
    return bpsw((u128)n);
}

int ref_sprp2_64(u64 n) { return sprp2_64(n); }
int ref_slprp64(u64 n) { return slprp64(n); }
int ref_is_prime(u64 n) { return is_prime_ref((u128)n); }
u64 ref_mix64(u64 z) { return mix64(z); }

/* verdict bits (bit i&7 of byte i>>3) for n[a..b), the reference's fast path: small
   factors, then four base-2 tests in lock step (sprp2_64x4, :651) and strong Lucas
   (slprp64, :766) on the passers, as test_batch64 (:1392) runs them */
typedef struct { const u64 *n; u8 *bits; size_t a, b; } rb_job;

static void *ref_bpsw_part(void *arg)
{
    rb_job *j = (rb_job *)arg;
    static const u32 sp[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41};
    u64 pend[4];
    size_t pidx[4];
    int np = 0;
    for (size_t i = j->a; i < j->b; i++) j->bits[i >> 3] &= (u8)~(1u << (i & 7));
    for (size_t i = j->a; i < j->b; i++) {
        const u64 n = j->n[i];
        int v = -1;
        if (n < 2) v = 0;
        else {
            for (int k = 0; k < 13; k++) {
                if (n == sp[k]) { v = 1; break; }
                if (n % sp[k] == 0) { v = 0; break; }
            }
            if (v < 0 && n < 43 * 43) v = 1;
        }
        if (v >= 0) { if (v) j->bits[i >> 3] |= (u8)(1u << (i & 7)); continue; }
        pend[np] = n; pidx[np] = i; np++;
        if (np == 4 || i + 1 == j->b) {
            bool r[4] = {false, false, false, false};
            if (np == 4) sprp2_64x4(pend, r);
            else for (int l = 0; l < np; l++) r[l] = sprp2_64(pend[l]);
            for (int l = 0; l < np; l++)
                if (r[l] && slprp64(pend[l])) j->bits[pidx[l] >> 3] |= (u8)(1u << (pidx[l] & 7));
            np = 0;
        }
    }
    if (np) {
        for (int l = 0; l < np; l++)
            if (sprp2_64(pend[l]) && slprp64(pend[l])) j->bits[pidx[l] >> 3] |= (u8)(1u << (pidx[l] & 7));
    }
    return NULL;
}

void ref_bpsw_batch(const u64 *n, size_t count, u8 *bits, int threads)
{
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    pthread_t th[256];
    rb_job jb[256];
    size_t per = (count + (size_t)threads - 1) / (size_t)threads;
    per = (per + 7) & ~(size_t)7;
    int k = 0;
    for (size_t a = 0; a < count && k < threads; a += per, k++) {
        jb[k].n = n; jb[k].bits = bits; jb[k].a = a; jb[k].b = a + per < count ? a + per : count;
        pthread_create(&th[k], NULL, ref_bpsw_part, &jb[k]);
    }
    for (int i = 0; i < k; i++) pthread_join(th[i], NULL);
}

/* the reference sextuplet counter on [lo, hi) with its production defaults (automatic
   wheel, B = 2^16, S = 2^18, pattern bound 256), as its selftest runs it (run_quiet,
   :2550); returns 1 if no candidate was rejected by the Lucas test */
int ref_count_sext(u64 lo, u64 hi, int threads, u64 *count, u64 *cks)
{
    g_print = false;
    return run_quiet((u128)lo, (u128)hi, 0, 1u << 16, 0, 256, 0, 0, threads, count, cks) ? 1 : 0;
}
