/*
 * mp_workload.c -- seeded synthetic inputs for the measured workloads (libmpwork.so).
 *
 * Not part of the compute path: it produces the candidate lists that the tests, the
 * smoke check and bench.py feed to libmathpub, identically on every machine.  The random
 * numbers are splitmix64 (the reference's mix64, A350826/a350826.c:425) stepped by the
 * golden-ratio constant from a seed.
 *
 * BPSW batch (2^26 odd u64 candidates, 4096 lists):
 *   60%  uniform odd in [2^40, 2^64)
 *   30%  p*q, p and q uniform from the primes in [2^31 - 2^21, 2^31 + 2^21)
 *    5%  (k+1)(2k+1), k uniform from the k in [2^30, 2^30 + 2^24) with k+1, 2k+1 prime
 *    5%  (6k+1)(12k+1)(18k+1), k uniform from all k >= 1 with the three factors prime and
 *        the product below 2^64 (Chernick's Carmichael numbers)
 *   list lengths: L = 2^e + r with e uniform in 8..17 and r uniform in [0, 2^e) (piecewise
 *   log-uniform in [2^8, 2^18)), then rescaled to sum exactly to the candidate count:
 *   L' = floor(L * count / sum), and the remainder is spread +1 over the first lists.
 * Pool membership is decided by an exact sieve of each window (plain C, below).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef uint64_t u64;
typedef uint32_t u32;
typedef unsigned __int128 u128;

#define GOLD 0x9E3779B97F4A7C15ULL

static u64 mix(u64 z)
{
    z += GOLD;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

typedef struct { u64 s; } rng_t;
static u64 rnext(rng_t *r) { return mix(r->s += GOLD); }

/* byte flags: f[i] = 1 iff lo + i is prime, for lo >= 2 (segmented by small primes) */
static unsigned char *prime_flags(u64 lo, u64 n)
{
    unsigned char *f = malloc(n);
    memset(f, 1, n);
    u64 hi = lo + n;
    u64 lim = 1;
    while ((lim + 1) * (lim + 1) <= hi) lim++;
    unsigned char *s = calloc(lim + 1, 1);
    for (u64 q = 2; q <= lim; q++) {
        if (s[q]) continue;
        for (u64 m = q * q; m <= lim; m += q) s[m] = 1;
        u64 st = (lo + q - 1) / q * q;
        if (st < q * q) st = q * q;
        for (u64 m = st; m < hi; m += q) f[m - lo] = 0;
    }
    free(s);
    for (u64 i = 0; i < n && lo + i < 2; i++) f[i] = 0;
    return f;
}

int mpw_bpsw_batch(u64 seed, u64 count, u32 nlists, u64 *cands, u32 *lens)
{
    rng_t r = {seed};
    /* pool A: primes near 2^31 */
    const u64 alo = (1ULL << 31) - (1ULL << 21), an = 1ULL << 22;
    unsigned char *fa = prime_flags(alo, an);
    u64 *A = malloc(an / 2 * sizeof *A), na = 0;
    for (u64 i = 0; i < an; i++) if (fa[i]) A[na++] = alo + i;
    free(fa);
    /* pool B: k with k+1 and 2k+1 prime */
    const u64 k0 = 1ULL << 30, kn = 1ULL << 24;
    unsigned char *f1 = prime_flags(k0 + 1, kn), *f2 = prime_flags(2 * k0 + 1, 2 * kn);
    u64 *Bk = malloc(kn / 8 * sizeof *Bk + 8), nb = 0;
    for (u64 i = 0; i < kn; i++) if (f1[i] && f2[2 * i] && nb < kn / 8) Bk[nb++] = k0 + i;
    free(f1); free(f2);
    /* pool C: Chernick k */
    u64 kmax = 1;
    while ((u128)(6 * (kmax + 1) + 1) * (12 * (kmax + 1) + 1) * (18 * (kmax + 1) + 1) < ((u128)1 << 64)) kmax++;
    unsigned char *fc = prime_flags(2, 18 * kmax + 2);
    u64 *Ck = malloc((kmax + 1) * sizeof *Ck), nc = 0;
    for (u64 k = 1; k <= kmax; k++)
        if (fc[6 * k + 1 - 2] && fc[12 * k + 1 - 2] && fc[18 * k + 1 - 2]) Ck[nc++] = k;
    free(fc);
    if (!na || !nb || !nc) { free(A); free(Bk); free(Ck); return -1; }
    for (u64 i = 0; i < count; i++) {
        const u64 u = rnext(&r) % 100;
        u64 n;
        if (u < 60) n = ((1ULL << 40) + rnext(&r) % (0ULL - (1ULL << 40))) | 1;
        else if (u < 90) n = A[rnext(&r) % na] * A[rnext(&r) % na];
        else if (u < 95) { const u64 k = Bk[rnext(&r) % nb]; n = (k + 1) * (2 * k + 1); }
        else { const u64 k = Ck[rnext(&r) % nc]; n = (6 * k + 1) * (12 * k + 1) * (18 * k + 1); }
        cands[i] = n;
    }
    free(A); free(Bk); free(Ck);
    if (nlists) {
        u64 sum = 0;
        for (u32 i = 0; i < nlists; i++) {
            const u64 e = 8 + rnext(&r) % 10;
            lens[i] = (u32)((1ULL << e) + rnext(&r) % (1ULL << e));
            sum += lens[i];
        }
        u64 tot = 0;
        for (u32 i = 0; i < nlists; i++) { lens[i] = (u32)((u128)lens[i] * count / sum); tot += lens[i]; }
        for (u32 i = 0; tot < count; i = (i + 1) % nlists, tot++) lens[i]++;
    }
    return 0;
}

/* n uniform odd numbers in [lo, hi) (for small parity cases) */
void mpw_uniform_odd(u64 seed, u64 lo, u64 hi, u64 count, u64 *out)
{
    rng_t r = {seed};
    for (u64 i = 0; i < count; i++) out[i] = (lo + rnext(&r) % (hi - lo)) | 1;
}
