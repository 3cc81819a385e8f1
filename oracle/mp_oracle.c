/*
 * mp_oracle.c -- CPU restatement of the Mathpub integer hot path.
 *
 * TEST INFRASTRUCTURE ONLY.  This library is the checker for the CUDA engine in
 * mathpub_b200/: only tests/, the smoke check in __graft_entry__.py and the CPU-baseline
 * leg of bench.py load it, and only to compute the expected answer or a CPU timing.  The
 * product library (libmathpub.so) never links, loads or calls anything in oracle/.
 *
 * What is restated, and from where (paths inside the Mathpub project):
 *   mix64 / hashp ..................... A350826/a350826.c:425-438
 *   inv64, mmul64, madd/msub/mhalf .... A350826/a350826.c:565-604
 *   sprp2_64 .......................... A350826/a350826.c:618-638
 *   jacobi, selfridge, slprp64 ........ A350826/a350826.c:693-799 (is_square uses an exact
 *                                       integer square root instead of sqrtl + fix-up)
 *   bpsw (n < 2^64) ................... A350826/a350826.c:965-969 with the small-factor
 *                                       handling of its callers (cmd_check, :2287)
 *   mr_ref / is_prime_ref ............. A350826/a350826.c:504-541
 *   odd-only segmented sieve .......... A228768/a228768.c:301-318 (base primes) and
 *                                       :372-415 (scan_interval: first odd multiple,
 *                                       start at q^2, step 2q)
 *   gap attribution ................... A000230/a000230.c:12-16,38-60 (a gap belongs to the
 *                                       prime that starts it; the next prime may lie
 *                                       beyond the range end)
 *   twin pairs ........................ A007508/a007508.c:1-10 (p and p+2 prime, counted
 *                                       by p)
 *   6-tuples {0,4,6,10,12,16} ......... A350826/a350826.c:22-31, counted by initial member p
 *                                       with checksum sum of hashp(p) (:1364-1379)
 *   Fermat quotient mod p^2 ........... A001220/wieferich.c:546-645 (pctx_init, msqr, redc)
 *                                       and :1051-1075 (finish_lanes: q = (r-1) p^-1 mod
 *                                       2^64, FLT check q < p, cks += mix64(q ^ p*GOLD),
 *                                       symmetric residue A); 2^128 mod N is computed with an
 *                                       exact 128-bit remainder, never a double estimate.
 *
 * Definitions that the reference does not fix (the CUDA engine follows the same ones):
 *   - odd-only bitmap: base = lo & ~1; bit i <-> base + 2i + 1; in-range bits are
 *     i < (hi - base) / 2; bit value 1 = prime.
 *   - per-segment hash: FNV-1a-64 over the bytes of the bitmap of a segment of 2^h
 *     integers (2^(h-1) bits), byte k holding bits 8k..8k+7 (bit j of byte k = bit 8k+j),
 *     ceil(len/8) bytes for a segment of len bits, bits at or beyond the range end zero.
 *   - blocks: block b = [lo + b 2^k, lo + (b+1) 2^k) intersected with [lo, hi).
 *   - max gap: max over primes p in the range (or block) of nextprime(p) - p; the next
 *     prime may lie beyond hi; ties go to the smallest p.  No prime: gap 0, start 0.
 *   - Wieferich ordered hash: H <- H * 0x100000001b3 + mix64(p ^ mix64(q)) (mod 2^64) over
 *     the primes p >= 3 in increasing order.
 */
#define _GNU_SOURCE
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

typedef uint8_t u8;
typedef uint32_t u32;
typedef uint64_t u64;
typedef int64_t i64;
typedef unsigned __int128 u128;

#define GOLD 0x9E3779B97F4A7C15ULL
#define FNV_OFFSET 0xcbf29ce484222325ULL
#define FNV_PRIME 0x100000001b3ULL

/* ------------------------------------------------------------------ */
/* hashing                                                              */
/* ------------------------------------------------------------------ */

/* splitmix64 step (A350826/a350826.c:425-431). */
u64 or_mix64(u64 z)
{
    z += GOLD;
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ULL;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBULL;
    return z ^ (z >> 31);
}

/* FNV-1a-64 over n bytes. */
u64 or_fnv1a64(const u8 *b, size_t n)
{
    u64 h = FNV_OFFSET;
    for (size_t i = 0; i < n; i++) { h ^= b[i]; h *= FNV_PRIME; }
    return h;
}

/* ------------------------------------------------------------------ */
/* reference primality (A350826/a350826.c:466-541)                      */
/* ------------------------------------------------------------------ */

static u64 mulmod64(u64 a, u64 b, u64 n) { return (u64)(((u128)a * b) % n); }

static u64 powmod64(u64 a, u64 e, u64 n)
{
    u64 r = 1 % n;
    a %= n;
    while (e) {
        if (e & 1) r = mulmod64(r, a, n);
        a = mulmod64(a, a, n);
        e >>= 1;
    }
    return r;
}

/* strong probable-prime test of odd n > a to base a (A350826/a350826.c:504-517) */
static int mr_ref(u64 n, u64 a)
{
    u64 d = n - 1;
    int s = 0;
    while (!(d & 1)) { d >>= 1; s++; }
    u64 x = powmod64(a, d, n);
    if (x == 1 || x == n - 1) return 1;
    for (int i = 1; i < s; i++) {
        x = mulmod64(x, x, n);
        if (x == n - 1) return 1;
        if (x == 1) return 0;
    }
    return 0;
}

/* deterministic primality for all n < 2^64: trial division by the primes <= 41, then
   strong tests to the 13 prime bases 2..41 (A350826/a350826.c:529-541) */
int or_is_prime_ref(u64 n)
{
    static const u32 sp[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41};
    if (n < 2) return 0;
    for (int i = 0; i < 13; i++) {
        if (n == sp[i]) return 1;
        if (n % sp[i] == 0) return 0;
    }
    if (n < 43 * 43) return 1;
    for (int i = 0; i < 13; i++) if (!mr_ref(n, sp[i])) return 0;
    return 1;
}

/* ------------------------------------------------------------------ */
/* 64-bit Montgomery BPSW (A350826/a350826.c:565-799)                   */
/* ------------------------------------------------------------------ */

static inline u64 inv64(u64 n)
{
    u64 x = n;
    for (int i = 0; i < 5; i++) x *= 2 - n * x;
    return x;
}

static inline u64 mmul64(u64 a, u64 b, u64 n, u64 ni)
{
    u128 t = (u128)a * b;
    u64 m = (u64)t * ni;
    u64 mh = (u64)(((u128)m * n) >> 64);
    u64 th = (u64)(t >> 64);
    u64 r = th - mh;
    return th < mh ? r + n : r;
}

static inline u64 madd64(u64 a, u64 b, u64 n) { u64 s = a + b; return (s < a || s >= n) ? s - n : s; }
static inline u64 msub64(u64 a, u64 b, u64 n) { return a >= b ? a - b : a - b + n; }
static inline u64 mhalf64(u64 a, u64 n) { return (a & 1) ? (a >> 1) + (n >> 1) + 1 : a >> 1; }

/* base-2 strong probable-prime test, odd n > 2 (A350826/a350826.c:618-638) */
int or_sprp2(u64 n)
{
    const u64 ni = inv64(n);
    const u64 one = (u64)(-n) % n, mone = n - one;
    u64 d = n - 1;
    const int s = __builtin_ctzll(d);
    d >>= s;
    int b = 63 - __builtin_clzll(d);
    u64 x = madd64(one, one, n);
    while (b-- > 0) {
        x = mmul64(x, x, n, ni);
        if ((d >> b) & 1) x = madd64(x, x, n);
    }
    if (x == one || x == mone) return 1;
    for (int i = 1; i < s; i++) {
        x = mmul64(x, x, n, ni);
        if (x == mone) return 1;
        if (x == one) return 0;
    }
    return 0;
}

/* Jacobi symbol (a/n), odd n >= 1 (A350826/a350826.c:693-713) */
static int jacobi(i64 a, u64 n)
{
    int t = 1;
    u64 x;
    if (a < 0) {
        x = (u64)(-(a + 1)) + 1;
        if ((n & 3) == 3) t = -t;
    } else x = (u64)a;
    x %= n;
    while (x) {
        while (!(x & 1)) {
            x >>= 1;
            unsigned r = (unsigned)(n & 7);
            if (r == 3 || r == 5) t = -t;
        }
        u64 tmp = x; x = n; n = tmp;
        if ((x & 3) == 3 && (n & 3) == 3) t = -t;
        x %= n;
    }
    return n == 1 ? t : 0;
}

/* exact integer square root floor(sqrt(n)) (digit by digit, no floating point) */
static u64 isqrt64(u64 n)
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

static int is_square(u64 n) { u64 r = isqrt64(n); return r * r == n; }

/* Selfridge method A (A350826/a350826.c:739-751) */
static int selfridge(u64 n, i64 *Dout)
{
    if (is_square(n)) return 0;
    i64 D = 5;
    for (;;) {
        int j = jacobi(D, n);
        if (j == -1) break;
        if (j == 0 && (u64)(D < 0 ? -D : D) != n) return 0;
        D = D > 0 ? -(D + 2) : -(D - 2);
    }
    *Dout = D;
    return 1;
}

/* strong Lucas probable-prime test, Selfridge parameters (A350826/a350826.c:766-799) */
int or_slprp(u64 n)
{
    i64 D;
    if (!selfridge(n, &D)) return 0;
    const i64 Q = (1 - D) / 4;
    const u64 ni = inv64(n), one = (u64)(-n) % n;
#define TOM64(v) ((u64)(((u128)(v) * one) % n))
    const u64 Qm = TOM64(Q >= 0 ? (u64)Q % n : n - (u64)(-Q) % n);
    const u64 Dm = TOM64(D >= 0 ? (u64)D % n : n - (u64)(-D) % n);
#undef TOM64
    u64 d = n + 1;
    const int s = __builtin_ctzll(d);
    d >>= s;
    u64 U = one, V = one, Qk = Qm;
    for (int b = 62 - __builtin_clzll(d); b >= 0; b--) {
        U = mmul64(U, V, n, ni);
        V = msub64(mmul64(V, V, n, ni), madd64(Qk, Qk, n), n);
        Qk = mmul64(Qk, Qk, n, ni);
        if ((d >> b) & 1) {
            const u64 U2 = madd64(U, V, n);
            const u64 V2 = madd64(mmul64(Dm, U, n, ni), V, n);
            U = mhalf64(U2, n);
            V = mhalf64(V2, n);
            Qk = mmul64(Qk, Qm, n, ni);
        }
    }
    if (U == 0 || V == 0) return 1;
    for (int r = 1; r < s; r++) {
        V = msub64(mmul64(V, V, n, ni), madd64(Qk, Qk, n), n);
        if (V == 0) return 1;
        Qk = mmul64(Qk, Qk, n, ni);
    }
    return 0;
}

/* verdict for any n < 2^64: trial division by the primes <= 41 (settles n < 43^2), then
   BPSW = base-2 strong test and strong Lucas test (A350826/a350826.c:965-969) */
int or_bpsw(u64 n)
{
    static const u32 sp[] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41};
    if (n < 2) return 0;
    for (int i = 0; i < 13; i++) {
        if (n == sp[i]) return 1;
        if (n % sp[i] == 0) return 0;
    }
    if (n < 43 * 43) return 1;
    return or_sprp2(n) && or_slprp(n);
}

/* ------------------------------------------------------------------ */
/* thread helper                                                        */
/* ------------------------------------------------------------------ */

typedef struct {
    void (*fn)(void *ctx, size_t a, size_t b);
    void *ctx;
    size_t a, b;
} job_t;

static void *job_run(void *arg)
{
    job_t *j = (job_t *)arg;
    j->fn(j->ctx, j->a, j->b);
    return NULL;
}

/* run fn(ctx, a, b) over [0, n) split into `threads` contiguous parts; boundaries are
   multiples of `align` (so byte-packed outputs are never shared between threads). */
static void parallel_for(size_t n, int threads, size_t align, void (*fn)(void *, size_t, size_t), void *ctx)
{
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    if (threads == 1 || n < 2 * align) { fn(ctx, 0, n); return; }
    pthread_t th[256];
    job_t jb[256];
    size_t per = (n + (size_t)threads - 1) / (size_t)threads;
    per = (per + align - 1) / align * align;
    int k = 0;
    for (size_t a = 0; a < n && k < threads; a += per, k++) {
        jb[k].fn = fn; jb[k].ctx = ctx; jb[k].a = a; jb[k].b = a + per < n ? a + per : n;
        if (pthread_create(&th[k], NULL, job_run, &jb[k]) != 0) { fn(ctx, jb[k].a, jb[k].b); th[k] = 0; }
    }
    for (int i = 0; i < k; i++) if (th[i]) pthread_join(th[i], NULL);
}

/* ---- batched BPSW: verdict bit i (bit i&7 of byte i>>3) for each n[i] ---- */
typedef struct { const u64 *n; u8 *bits; } bpsw_ctx;

static void bpsw_part(void *c, size_t a, size_t b)
{
    bpsw_ctx *x = (bpsw_ctx *)c;
    for (size_t i = a; i < b; i += 8) {
        u8 v = 0;
        for (size_t k = 0; k < 8 && i + k < b; k++) v |= (u8)(or_bpsw(x->n[i + k]) << k);
        x->bits[i >> 3] = v;
    }
}

void or_bpsw_batch(const u64 *n, size_t count, u8 *bits, int threads)
{
    bpsw_ctx c = {n, bits};
    parallel_for(count, threads, 8, bpsw_part, &c);
}

/* ------------------------------------------------------------------ */
/* Fermat quotient 2^(p-1) mod p^2 (A001220/wieferich.c:546-645)        */
/* ------------------------------------------------------------------ */

typedef struct { u128 N, one; u64 p, pinv, ninv; } fctx_t;

static void fctx_init(fctx_t *c, u64 p)
{
    u64 x = (3 * p) ^ 2;                                 /* correct to 5 bits for odd p */
    for (int i = 0; i < 4; i++) x *= 2 - p * x;           /* 10, 20, 40, 80 bits */
    c->p = p;
    c->pinv = x;
    c->N = (u128)p * p;
    c->ninv = 0 - x * x;                                  /* -N^-1 mod 2^64 */
    c->one = ((u128)0 - c->N) % c->N;                     /* 2^128 mod N, exact */
}

/* Montgomery product a b / 2^128 mod N for a, b < N < 2^126 */
static u128 fmul(u128 a, u128 b, const fctx_t *c)
{
    const u64 a0 = (u64)a, a1 = (u64)(a >> 64), b0 = (u64)b, b1 = (u64)(b >> 64);
    const u64 n0 = (u64)c->N, n1 = (u64)(c->N >> 64);
    const u128 p00 = (u128)a0 * b0, p01 = (u128)a0 * b1, p10 = (u128)a1 * b0, p11 = (u128)a1 * b1;
    const u64 t0 = (u64)p00;
    const u128 mid = (p00 >> 64) + (u64)p01 + (u64)p10;
    u64 t1 = (u64)mid;
    const u128 hi = (mid >> 64) + (p01 >> 64) + (p10 >> 64) + p11;
    u64 t2 = (u64)hi, t3 = (u64)(hi >> 64);
    u64 m = t0 * c->ninv;
    u128 s = (u128)m * n0 + t0;
    s = (u128)m * n1 + t1 + (u64)(s >> 64);
    t1 = (u64)s;
    s = (u128)t2 + (u64)(s >> 64);
    t2 = (u64)s;
    t3 += (u64)(s >> 64);
    m = t1 * c->ninv;
    s = (u128)m * n0 + t1;
    s = (u128)m * n1 + t2 + (u64)(s >> 64);
    const u64 r0 = (u64)s;
    s = (u128)t3 + (u64)(s >> 64);
    const u128 r = ((u128)(u64)s << 64) | r0;
    return r >= c->N ? r - c->N : r;
}

static inline u128 fdbl(u128 x, const fctx_t *c) { u128 y = x << 1; return y >= c->N ? y - c->N : y; }

/* leave Montgomery form: x / 2^128 mod N */
static u128 fredc(u128 x, const fctx_t *c) { return fmul(x, 1, c); }

/* q = (2^(p-1) mod p^2 - 1) / p mod 2^64 for odd p, 3 <= p < 2^63; *res = the residue */
u64 or_fermat_q2(u64 p, u64 *res_lo, u64 *res_hi)
{
    fctx_t c;
    fctx_init(&c, p);
    const u64 e = p - 1;
    int b = 63 - __builtin_clzll(e);
    u128 x = fdbl(c.one, &c);                             /* top bit of e: 2 */
    while (b-- > 0) {
        x = fmul(x, x, &c);
        if ((e >> b) & 1) x = fdbl(x, &c);
    }
    const u128 r = fredc(x, &c);
    if (res_lo) *res_lo = (u64)r;
    if (res_hi) *res_hi = (u64)(r >> 64);
    return ((u64)r - 1) * c.pinv;
}

typedef struct { const u64 *p; u64 *q; } ferm_ctx;

static void ferm_part(void *c, size_t a, size_t b)
{
    ferm_ctx *x = (ferm_ctx *)c;
    for (size_t i = a; i < b; i++) x->q[i] = x->p[i] >= 3 ? or_fermat_q2(x->p[i], NULL, NULL) : 0;
}

void or_fermat_batch(const u64 *p, size_t count, u64 *q, int threads)
{
    ferm_ctx c = {p, q};
    parallel_for(count, threads, 1, ferm_part, &c);
}

/* ------------------------------------------------------------------ */
/* odd-only segmented sieve (A228768/a228768.c:301-318, 372-415)        */
/* ------------------------------------------------------------------ */

/* odd primes 3 <= q <= lim, segmented so that lim may reach 2^32 */
u32 *or_odd_primes_upto(u64 lim, size_t *count)
{
    *count = 0;
    if (lim < 3) return (u32 *)malloc(4);
    if (lim > 0xFFFFFFFFULL) lim = 0xFFFFFFFFULL;
    /* primes up to sqrt(lim) <= 65536 by a plain odd sieve */
    const u32 sl = (u32)isqrt64(lim);
    u8 *c = (u8 *)calloc(sl / 2 + 2, 1);
    u32 small[6600];
    size_t ns = 0;
    for (u32 i = 1; 2 * i + 1 <= sl; i++) {
        if (c[i]) continue;
        const u32 q = 2 * i + 1;
        small[ns++] = q;
        for (u64 j = (u64)q * q; j <= sl; j += 2 * q) c[j / 2] = 1;
    }
    free(c);
    size_t cap = 1024, n = 0;
    u32 *out = (u32 *)malloc(cap * sizeof *out);
    const u64 W = 1 << 20;                                /* odd numbers per window */
    u8 *f = (u8 *)malloc(W);
    for (u64 o0 = 3; o0 <= lim; o0 += 2 * W) {            /* window: odd o0 .. o0 + 2(W-1) */
        u64 cnt = W;
        if (o0 + 2 * (cnt - 1) > lim) cnt = (lim - o0) / 2 + 1;
        memset(f, 0, cnt);
        const u64 w1 = o0 + 2 * cnt;
        for (size_t k = 0; k < ns; k++) {
            const u64 q = small[k];
            if (q * q >= w1) break;
            u64 s = (o0 + q - 1) / q * q;
            if (!(s & 1)) s += q;
            if (s < q * q) s = q * q;
            for (u64 m = s; m < w1; m += 2 * q) f[(m - o0) >> 1] = 1;
        }
        for (u64 i = 0; i < cnt; i++) {
            if (f[i]) continue;
            if (n == cap) { cap *= 2; out = (u32 *)realloc(out, cap * sizeof *out); }
            out[n++] = (u32)(o0 + 2 * i);
        }
    }
    free(f);
    *count = n;
    return out;
}

void or_free(void *p) { free(p); }

typedef struct {
    u64 base, nbits;      /* bits [0, nbits) of the odd-only map: bit i <-> base + 2i + 1 */
    const u32 *pr;
    size_t np;
    u64 *words;           /* output: 1 = prime */
} sv_ctx;

/* sieve bits [a, b) (a, b multiples of 64 except b = nbits) */
static void sieve_part(void *cp, size_t a, size_t b)
{
    sv_ctx *x = (sv_ctx *)cp;
    const u64 base = x->base;
    const u64 WB = 1 << 20;                               /* bits per window */
    u64 *next = (u64 *)malloc((x->np ? x->np : 1) * sizeof *next);
    /* bit index of the first odd multiple >= the first number of the part, at least q^2;
       kept as an offset from x0 so that nothing overflows near 2^64 */
    const u64 x0 = base + 2 * (u64)a + 1;
    size_t np = 0;
    const u64 xend = base + 2 * (u64)b + 1;
    for (size_t k = 0; k < x->np; k++) {
        const u64 q = x->pr[k];
        if ((u128)q * q >= xend) break;
        const u64 r = x0 % q;
        u64 d = r ? q - r : 0;                            /* x0 + d is a multiple of q */
        if (d & 1) d += q;                                /* ... and odd */
        u64 j = a + d / 2;
        if (q * q > x0) j = a + (q * q - x0) / 2;
        next[k] = j;
        np = k + 1;
    }
    for (u64 w0 = a; w0 < b; w0 += WB) {
        const u64 w1 = w0 + WB < b ? w0 + WB : b;
        /* set window bits to 1 */
        for (u64 i = w0; i < w1; ) {
            if ((i & 63) == 0 && i + 64 <= w1) { x->words[i >> 6] = ~0ULL; i += 64; }
            else { x->words[i >> 6] |= 1ULL << (i & 63); i++; }
        }
        for (size_t k = 0; k < np; k++) {
            const u64 q = x->pr[k];
            u64 j = next[k];
            for (; j < w1; j += q) x->words[j >> 6] &= ~(1ULL << (j & 63));
            next[k] = j;
        }
    }
    free(next);
}

/* odd-only prime bitmap of the bits [0, nbits) for base (even); words must hold
   ceil(nbits/64) u64; bits >= nbits in the last word are cleared */
int or_sieve_bits(u64 base, u64 nbits, u64 *words, int threads)
{
    if (base & 1) return -1;
    const u64 top = base + 2 * nbits;                     /* largest number < top */
    size_t np;
    u32 *pr = or_odd_primes_upto(isqrt64(top) + 1, &np);
    const size_t nw = (size_t)((nbits + 63) >> 6);
    memset(words, 0, nw * 8);
    sv_ctx c = {base, nbits, pr, np, words};
    parallel_for((size_t)nbits, threads, 64, sieve_part, &c);
    if (base == 0 && nbits) words[0] &= ~1ULL;            /* 1 is not prime */
    free(pr);
    return 0;
}

/* ------------------------------------------------------------------ */
/* range statistics from the bitmap                                     */
/* ------------------------------------------------------------------ */

typedef struct {
    u64 pi, twins, max_gap, gap_start, tuple6, tuple6_cks, first_prime, last_prime;
} or_stats_t;

static inline int getbit(const u64 *w, u64 i) { return (int)((w[i >> 6] >> (i & 63)) & 1); }

/* first set bit at index >= i and < n, or n if there is none */
static u64 next_bit(const u64 *w, u64 i, u64 n)
{
    while (i < n) {
        u64 x = w[i >> 6] >> (i & 63);
        if (x) { u64 j = i + (u64)__builtin_ctzll(x); return j < n ? j : n; }
        i = (i | 63) + 1;
    }
    return n;
}

static void stats_add_gap(or_stats_t *s, u64 p, u64 g)
{
    if (g > s->max_gap) { s->max_gap = g; s->gap_start = p; }
}

/*
 * or_sieve_range: the full definition of the range outputs.
 *   lo < hi <= 2^64 - 2^17; tail = extra integers sieved past hi (>= 16) to find the
 *   prime after the last one in range and the members of 6-tuples that cross hi.
 *   block_log2 (0 = no blocks): block width 2^block_log2 integers, nblocks =
 *   ceil((hi - lo) / 2^k); blocks[] holds nblocks entries.
 *   hash_log2 (0 = no hashes, else >= 4): hashes[] holds ceil(nbits / 2^(h-1)) values.
 *   bitmap (nullable): ceil(nbits/64) words of the in-range bitmap.
 *   Returns 0, or -1 for bad arguments, -2 if no prime follows the last prime of the
 *   range within the tail.
 */
int or_sieve_range(u64 lo, u64 hi, u64 tail, int block_log2, int hash_log2, or_stats_t *out,
                   or_stats_t *blocks, u64 *hashes, u64 *bitmap, int threads)
{
    if (hi <= lo || tail < 16 || hi > 0xFFFFFFFFFFFFFFFFULL - 2 * tail) return -1;
    if (hash_log2 && hash_log2 < 4) return -1;
    const u64 base = lo & ~1ULL;
    const u64 nbits = (hi - base) >> 1;
    const u64 nbx = (hi + tail - base) >> 1;
    u64 *w = (u64 *)malloc(((nbx + 63) >> 6) * 8 + 8);
    if (!w) return -3;
    or_sieve_bits(base, nbx, w, threads);
    memset(out, 0, sizeof *out);
    const u64 nblk = block_log2 ? ((hi - lo - 1) >> block_log2) + 1 : 0;
    if (blocks) memset(blocks, 0, nblk * sizeof *blocks);
    const int has2 = lo <= 2 && 2 < hi;
    if (has2) {
        out->pi = 1; out->max_gap = 1; out->gap_start = 2; out->first_prime = 2; out->last_prime = 2;
        if (blocks) { or_stats_t *B = &blocks[(2 - lo) >> block_log2]; B->pi = 1; B->max_gap = 1; B->gap_start = 2; B->first_prime = B->last_prime = 2; }
    }
    int status = 0;
    /* walk the in-range primes in order */
    for (u64 wi = 0; wi < ((nbits + 63) >> 6); wi++) {
        u64 x = w[wi];
        if ((wi << 6) + 64 > nbits) x &= (nbits & 63) ? ((1ULL << (nbits & 63)) - 1) : ~0ULL;
        while (x) {
            const u64 i = (wi << 6) + (u64)__builtin_ctzll(x);
            x &= x - 1;
            const u64 p = base + 2 * i + 1;
            or_stats_t *B = blocks ? &blocks[(p - lo) >> block_log2] : NULL;
            out->pi++;
            if (!out->first_prime) out->first_prime = p;
            out->last_prime = p;
            if (B) { B->pi++; if (!B->first_prime) B->first_prime = p; B->last_prime = p; }
            if (getbit(w, i + 1)) { out->twins++; if (B) B->twins++; }
            if (getbit(w, i + 2) && getbit(w, i + 3) && getbit(w, i + 5) && getbit(w, i + 6) && getbit(w, i + 8)) {
                const u64 h = or_mix64(p);
                out->tuple6++; out->tuple6_cks += h;
                if (B) { B->tuple6++; B->tuple6_cks += h; }
            }
            /* the gap belongs to p: find the next prime (may be beyond hi) */
            const u64 j = next_bit(w, i + 1, nbx);
            if (j >= nbx) { status = -2; continue; }
            const u64 g = 2 * (j - i);
            stats_add_gap(out, p, g);
            if (B) stats_add_gap(B, p, g);
        }
    }
    if (hashes && hash_log2) {
        const u64 sb = 1ULL << (hash_log2 - 1);           /* bits per hash segment */
        const u64 ns = (nbits + sb - 1) / sb;
        for (u64 s = 0; s < ns; s++) {
            const u64 b0 = s * sb, len = (b0 + sb < nbits ? sb : nbits - b0);
            u64 h = FNV_OFFSET;
            for (u64 k = 0; k < (len + 7) / 8; k++) {
                const u64 bit = b0 + 8 * k;                   /* multiple of 8 */
                u8 byte = (u8)(w[bit >> 6] >> (bit & 63));
                const u64 rem = len - 8 * k;
                if (rem < 8) byte &= (u8)((1u << rem) - 1);
                h ^= byte; h *= FNV_PRIME;
            }
            hashes[s] = h;
        }
    }
    if (bitmap) {
        const size_t nw = (size_t)((nbits + 63) >> 6);
        memcpy(bitmap, w, nw * 8);
        if (nbits & 63) bitmap[nw - 1] &= (1ULL << (nbits & 63)) - 1;
    }
    free(w);
    return status;
}

/* all primes in [lo, hi) into out (cap entries); returns the number of primes (which may
   exceed cap: then only the first cap are stored) */
size_t or_primes_range(u64 lo, u64 hi, u64 *out, size_t cap, int threads)
{
    if (hi <= lo) return 0;
    size_t n = 0;
    if (lo <= 2 && 2 < hi) { if (n < cap) out[n] = 2; n++; }
    const u64 base = lo & ~1ULL, nbits = (hi - base) >> 1;
    u64 *w = (u64 *)malloc(((nbits + 63) >> 6) * 8 + 8);
    or_sieve_bits(base, nbits, w, threads);
    for (u64 wi = 0; wi < ((nbits + 63) >> 6); wi++) {
        u64 x = w[wi];
        while (x) {
            const u64 i = (wi << 6) + (u64)__builtin_ctzll(x);
            x &= x - 1;
            if (n < cap) out[n] = base + 2 * i + 1;
            n++;
        }
    }
    free(w);
    return n;
}

/* ------------------------------------------------------------------ */
/* Wieferich base-2 range (A001220/wieferich.c:1051-1075, 1129-1177)    */
/* ------------------------------------------------------------------ */

typedef struct {
    u64 primes, tests, near, flt, cks, ordered_hash, nhits;
    u64 hits[16];
} or_wief_t;

typedef struct { const u64 *p; size_t n; u64 *q; } wq_ctx;

int or_wieferich_range(u64 lo, u64 hi, or_wief_t *out, int threads)
{
    memset(out, 0, sizeof *out);
    if (hi <= lo || hi > (1ULL << 63)) return -1;
    const u64 span = hi - lo;
    size_t cap = (size_t)(span / 2 + 16);
    if (cap > ((size_t)1 << 31)) return -1;
    u64 *p = (u64 *)malloc(cap * 8), *q;
    size_t n = or_primes_range(lo, hi, p, cap, threads);
    q = (u64 *)malloc((n ? n : 1) * 8);
    or_fermat_batch(p, n, q, threads);
    out->primes = n;
    for (size_t i = 0; i < n; i++) {
        if (p[i] == 2) continue;
        out->tests++;
        if (q[i] >= p[i]) { out->flt++; continue; }
        out->cks += or_mix64(q[i] ^ (p[i] * GOLD));
        const u64 A = q[i] <= p[i] / 2 ? q[i] : p[i] - q[i];
        if ((u128)A * 1000 < p[i]) out->near++;
        if (q[i] == 0) { if (out->nhits < 16) out->hits[out->nhits] = p[i]; out->nhits++; }
        out->ordered_hash = out->ordered_hash * FNV_PRIME + or_mix64(p[i] ^ or_mix64(q[i]));
    }
    free(p); free(q);
    return 0;
}
