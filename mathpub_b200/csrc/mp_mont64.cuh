// mp_mont64.cuh -- arithmetic modulo an odd 64-bit n, and the BPSW primality test built on it,
// for B200 (sm_100a).  Used by the BPSW kernels (mp_bpsw.cu) and the constellation sieve
// (mp_chain.cu).
//
// What is computed follows the reference (paths inside the Mathpub project): the base-2 strong
// probable-prime test (sprp2_64, A350826/a350826.c:618), the strong Lucas test with Selfridge's
// parameters (slprp64 :766, D from selfridge :739) and their conjunction (bpsw :965).  Both
// give exact primality below 2^64, so the verdicts are the reference's.  How it is computed is
// this file's own design, from the published mathematics:
//
//  * A residue is two 32-bit limbs; each product is one PTX block of 32-bit multiply-add carry
//    chains, with the subtracting reduction of the 128-bit product t (R = 2^64): m = t n^-1 mod
//    2^64, then (t - m n) / R = t_hi - hi(m n), exact since the low halves agree, plus n when it
//    borrows.  In and out in [0, n), for any odd n, and its input may be up to n R, which lets
//    the doubling below fold into the product for n < 2^63.
//  * Base-2 exponentiation, left to right, in two size classes (warps run one class at a time):
//    n < 2^63, one product x (x 2^b) per bit (below 2 n^2 < n R); n >= 2^63, a square, then a
//    doubling by a funnel shift of the residue by the exponent bit b and one conditional
//    subtraction (no select between two residues).  (A word-by-word adding reduction with lazy
//    residues in [0, 2n) for n < 2^62, a square then a doubling per bit, measured 2.5% slower on
//    the whole batched BPSW than the folded product.)
//  * Lucas sequences (P = 1, Q = (1 - D)/4) run as the ladder (V_k, V_k+1, Q^k) with
//        V_2k = V_k^2 - 2 Q^k,   V_2k+1 = V_k V_k+1 - P Q^k,
//    the same four products for either exponent bit (the bit only selects operands), so the
//    lanes of a warp never diverge on the exponent.  U_d = 0 (mod n) is read off as
//    2 V_d+1 = P V_d (mod n): D U_k = 2 V_k+1 - P V_k, and gcd(D, n) = 1 when (D/n) = -1.
//  * The Jacobi symbol is the binary (shift and subtract) algorithm after one reduction n mod
//    |D|; the perfect-square check (a square has no D with (D/n) = -1) runs only after 24 values
//    of D have failed.
#pragma once
#include "mp_common.cuh"

// n^-1 mod 2^64 for odd n.  n n = 1 (mod 8), so n is its own inverse to 3 bits; each Newton
// step x (2 - n x) doubles the correct bits: 6, 12, 24, 48, 96.
__host__ __device__ __forceinline__ u64 inv64(u64 n)
{
    u64 x = n;
    x *= 2 - n * x;
    x *= 2 - n * x;
    x *= 2 - n * x;
    x *= 2 - n * x;
    x *= 2 - n * x;
    return x;
}

// the modulus with what the products need: n^-1 mod 2^64 and R mod n
struct Mod64 {
    u64 n;
    u64 ni;        // n^-1 mod 2^64 (the subtracting reduction)
    u64 one;       // R mod n, the residue of 1
};

// ---- products: t = a b (128 bits), then the reduction, result t / 2^64 ----

// the subtracting reduction of t3:t2:t1:t0 (< n R): m = (t1:t0) n^-1 mod 2^64 (i1:i0), then
// (t3:t2) - hi64(m n) + (n if it borrows).  The words of m n below 2^64 equal t1:t0, so only
// their carries into word 2 are formed.
#define MM_REDUCE_SUB                                    \
    "mul.lo.u32     m0, t0, i0;\n\t"                     \
    "mul.hi.u32     m1, t0, i0;\n\t"                     \
    "mad.lo.u32     m1, t0, i1, m1;\n\t"                 \
    "mad.lo.u32     m1, t1, i0, m1;\n\t"                 \
    "mul.hi.u32     v1, m0, n0;\n\t"                     \
    "mad.lo.cc.u32  v1, m0, n1, v1;\n\t"                 \
    "madc.hi.u32    v2, m0, n1, 0;\n\t"                  \
    "mad.lo.cc.u32  v1, m1, n0, v1;\n\t"                 \
    "madc.hi.cc.u32 v2, m1, n0, v2;\n\t"                 \
    "addc.u32       v3, 0, 0;\n\t"                       \
    "mad.lo.cc.u32  v2, m1, n1, v2;\n\t"                 \
    "madc.hi.u32    v3, m1, n1, v3;\n\t"                 \
    "sub.cc.u32     t2, t2, v2;\n\t"                     \
    "subc.cc.u32    t3, t3, v3;\n\t"                     \
    "subc.u32       bw, 0, 0;\n\t"                       \
    "and.b32        k0, n0, bw;\n\t"                     \
    "and.b32        k1, n1, bw;\n\t"                     \
    "add.cc.u32     t2, t2, k0;\n\t"                     \
    "addc.u32       t3, t3, k1;\n\t"

#define MS_REGS ".reg .u32 a0, a1, b0, b1, n0, n1, i0, i1, t0, t1, t2, t3, m0, m1, v1, v2, v3, bw, k0, k1;\n\t"

// a b / R mod n by the subtracting reduction: a, b < n (or a b < n R), result in [0, n)
__device__ __forceinline__ u64 ms_mul(u64 a, u64 b, const Mod64 &M)
{
    u64 r;
    asm("{\n\t" MS_REGS
        "mov.b64 {a0, a1}, %1;\n\t"
        "mov.b64 {b0, b1}, %2;\n\t"
        "mov.b64 {n0, n1}, %3;\n\t"
        "mov.b64 {i0, i1}, %4;\n\t"
        "mul.lo.u32     t0, a0, b0;\n\t"
        "mul.hi.u32     t1, a0, b0;\n\t"
        "mul.lo.u32     t2, a1, b1;\n\t"
        "mul.hi.u32     t3, a1, b1;\n\t"
        "mad.lo.cc.u32  t1, a0, b1, t1;\n\t"
        "madc.hi.cc.u32 t2, a0, b1, t2;\n\t"
        "addc.u32       t3, t3, 0;\n\t"
        "mad.lo.cc.u32  t1, a1, b0, t1;\n\t"
        "madc.hi.cc.u32 t2, a1, b0, t2;\n\t"
        "addc.u32       t3, t3, 0;\n\t"
        MM_REDUCE_SUB
        "mov.b64 %0, {t2, t3};\n\t}"
        : "=l"(r) : "l"(a), "l"(b), "l"(M.n), "l"(M.ni));
    return r;
}

// a^2 / R mod n by the subtracting reduction, a in [0, n)
__device__ __forceinline__ u64 ms_sqr(u64 a, const Mod64 &M)
{
    u64 r;
    asm("{\n\t" MS_REGS
        "mov.b64 {a0, a1}, %1;\n\t"
        "mov.b64 {n0, n1}, %2;\n\t"
        "mov.b64 {i0, i1}, %3;\n\t"
        "mul.lo.u32     t0, a0, a0;\n\t"
        "mul.hi.u32     t1, a0, a0;\n\t"
        "mul.lo.u32     t2, a1, a1;\n\t"
        "mul.hi.u32     t3, a1, a1;\n\t"
        "mad.lo.cc.u32  t1, a0, a1, t1;\n\t"
        "madc.hi.cc.u32 t2, a0, a1, t2;\n\t"
        "addc.u32       t3, t3, 0;\n\t"
        "mad.lo.cc.u32  t1, a0, a1, t1;\n\t"
        "madc.hi.cc.u32 t2, a0, a1, t2;\n\t"
        "addc.u32       t3, t3, 0;\n\t"
        MM_REDUCE_SUB
        "mov.b64 %0, {t2, t3};\n\t}"
        : "=l"(r) : "l"(a), "l"(M.n), "l"(M.ni));
    return r;
}

// x 2^b mod n for b in {0, 1} and x in [0, n): a funnel shift by b (the bit shifted out of 64
// is kept), then one conditional subtraction; result in [0, n)
__device__ __forceinline__ u64 mm_dbl(u64 x, u32 b, const Mod64 &M)
{
    u64 r;
        asm("{\n\t.reg .u32 x0, x1, n0, n1, y0, y1, c, d0, d1, bw;\n\t.reg .pred p;\n\t"
            "mov.b64 {x0, x1}, %1;\n\t"
            "mov.b64 {n0, n1}, %2;\n\t"
            "shl.b32         y0, x0, %3;\n\t"
            "shf.l.clamp.b32 y1, x0, x1, %3;\n\t"
            "shr.b32         c, x1, 31;\n\t"
            "and.b32         c, c, %3;\n\t"
            "sub.cc.u32      d0, y0, n0;\n\t"
            "subc.cc.u32     d1, y1, n1;\n\t"
            "subc.u32        bw, c, 0;\n\t"
            "setp.ne.u32     p, bw, 0;\n\t"
            "selp.u32        y0, y0, d0, p;\n\t"
            "selp.u32        y1, y1, d1, p;\n\t"
            "mov.b64 %0, {y0, y1};\n\t}"
            : "=l"(r) : "l"(x), "l"(M.n), "r"(b));
    return r;
}

// (a + b) mod n and (a - b) mod n for a, b in [0, n)
__device__ __forceinline__ u64 mm_add(u64 a, u64 b, u64 n)
{
    const u64 s = a + b;
    const u64 t = s - n;
    // a + b >= n exactly when the sum wrapped past 2^64 or the difference did not borrow
    return (s < a || s >= n) ? t : s;
}
__device__ __forceinline__ u64 mm_sub(u64 a, u64 b, u64 n)
{
    const u64 d = a - b;
    return a < b ? d + n : d;
}

// the modulus set-up: n^-1 mod 2^64 and R mod n.  R mod n = 2^64 mod n is reached from
// 2^(bitlen(n) - 1) < n by doublings, which are exact.
__device__ __forceinline__ Mod64 mm_setup(u64 n)
{
    Mod64 M;
    M.n = n;
    M.ni = inv64(n);
    const int top = 63 - __clzll((long long)n);
    u64 x = 1ull << top;
    for (int i = top; i < 64; i++) x = mm_dbl(x, 1u, M);
    M.one = x;
    return M;
}

// Montgomery residue of a small signed integer v (|v| < n): |v| R by double-and-add of R mod n
// over the bits of |v|, then negated
__device__ __forceinline__ u64 mm_from_small(i32 v, const Mod64 &M)
{
    const u32 a = v < 0 ? (u32)(-v) : (u32)v;
    u64 r = 0;
    for (int i = 31 - __clz(a | 1u); i >= 0; i--) {
        r = mm_dbl(r, 1u, M);
        if ((a >> i) & 1u) r = mm_add(r, M.one, M.n);
    }
    return (v < 0 && r) ? M.n - r : r;
}

// ---- base-2 strong probable-prime test ----

// size classes of the base-2 ladder: below 2^63 (the doubling folded into the product), 2^63
// and above (a square, then the doubling)
#define SP_FOLD 1
#define SP_WIDE 2

__device__ __forceinline__ int spsp2_class(u64 n) { return n < (1ull << 63) ? SP_FOLD : SP_WIDE; }

// n - 1 = d 2^s with d odd: 2^d (mod n) by the left-to-right ladder, then the strong
// condition 2^d = 1, or 2^(d 2^r) = -1 for some 0 <= r < s.  Odd n > 2 in size class CLS.
template <int CLS>
__device__ __forceinline__ bool spsp2(const Mod64 &M)
{
    const u64 n = M.n;
    const int s = __ffsll((long long)(n - 1)) - 1;
    const u64 d = (n - 1) >> s;
    const int L = 63 - __clzll((long long)d);               // d's top bit: the ladder starts at 2
    u64 x = mm_dbl(M.one, 1u, M);
    for (int i = L - 1; i >= 0; i--) {
        const u32 bit = (u32)(d >> i) & 1u;
        if (CLS == SP_FOLD) {
            x = ms_mul(x, x << bit, M);                     // x (x 2^bit) / R < 2 n^2 / R < n
        } else {
            x = ms_sqr(x, M);
            x = mm_dbl(x, bit, M);
        }
    }
    const u64 mone = n - M.one;                             // the residue of -1
    bool pass = x == M.one || x == mone;
    for (int r = 1; r < s && !pass; r++) {
        if (x == M.one) break;                              // 1 before -1: not a strong probable prime
        x = ms_sqr(x, M);
        pass = x == mone;
    }
    return pass;
}

// the test for any odd n > 2, in its size class
__device__ __forceinline__ bool spsp2_u64(u64 n)
{
    const Mod64 M = mm_setup(n);
    const int c = spsp2_class(n);
    return c == SP_FOLD ? spsp2<SP_FOLD>(M) : spsp2<SP_WIDE>(M);
}

// ---- strong Lucas test ----

// Jacobi symbol (a/m) for odd m > 0 and 0 <= a < m: strip factors 2 of a (each flips the sign
// when m = 3, 5 mod 8), swap by reciprocity when a < m (flip when a = m = 3 mod 4), subtract
__device__ __forceinline__ int jacobi32(u32 a, u32 m)
{
    int t = 1;
    while (a) {
        const int z = __ffs((int)a) - 1;
        a >>= z;
        if ((z & 1) && ((m & 7u) == 3u || (m & 7u) == 5u)) t = -t;
        if (a < m) {
            const u32 x = a;
            a = m;
            m = x;
            if (a & m & 2u) t = -t;
        }
        a -= m;
    }
    return m == 1 ? t : 0;
}

// (D/n) for odd n > |D|, D odd: (-1/n) for the sign, then reciprocity (|D|/n) = +-(n mod |D| / |D|)
__device__ __forceinline__ int jacobi_dn(i32 D, u64 n)
{
    const u32 a = D < 0 ? (u32)(-D) : (u32)D;
    int t = 1;
    if (D < 0 && (n & 3) == 3) t = -t;
    if ((a & 3u) == 3u && (n & 3) == 3) t = -t;
    return t * jacobi32((u32)(n % a), a);
}

// exact test for a perfect square: residue filters mod 64 and 63, then the integer root by
// bits from the top
__device__ __forceinline__ bool is_square64(u64 n)
{
    if (!((0x0202021202030213ull >> (n & 63)) & 1)) return false;
    if (!((0x0402483012450293ull >> (n % 63)) & 1)) return false;
    u64 r = 0;
    for (int b = 31; b >= 0; b--) {
        const u64 c = r | (1ull << b);
        if (c * c <= n) r = c;
    }
    return r * r == n;
}

// Selfridge's method A: the first D of 5, -7, 9, -11, 13, ... with (D/n) = -1.  Returns 0 when
// n is shown composite on the way: some |D| < n shares a factor with n, or n is a perfect
// square (no D exists then).  Odd n, larger than the |D| reached.
__device__ __forceinline__ i32 selfridge_d(u64 n)
{
    for (int k = 0; k < 2048; k++) {
        const i32 a = 5 + 2 * k;
        const i32 D = (k & 1) ? -a : a;
        const int j = jacobi_dn(D, n);
        if (j < 0) return D;
        if (j == 0 && (u64)a != n) return 0;
        if (k == 23 && is_square64(n)) return 0;
    }
    return 0;
}

// strong Lucas probable prime with P = 1, Q = (1 - D)/4 (D = 1 mod 4 here, so Q is exact):
// n + 1 = d 2^s, d odd; U_d = 0, or V_(d 2^r) = 0 for some 0 <= r < s.  Odd n > 2, n < 2^64 - 1.
__device__ __forceinline__ bool lucas_strong(const Mod64 &M, i32 D)
{
    const u64 n = M.n;
    const i32 Q = (1 - D) / 4;
    const u64 q1 = mm_from_small(Q, M);
    const int s = __ffsll((long long)(n + 1)) - 1;
    const u64 d = (n + 1) >> s;
    // k = 1 (d's top bit): V_1 = P = 1, V_2 = P^2 - 2Q, Q^1
    u64 vk = M.one;
    u64 vk1 = mm_sub(M.one, mm_add(q1, q1, n), n);
    u64 qk = q1;
    for (int i = 62 - __clzll((long long)d); i >= 0; i--) {
        const bool b = (d >> i) & 1;
        const u64 w = mm_sub(ms_mul(vk, vk1, M), qk, n);               // V_2k+1
        const u64 qb = ms_mul(qk, b ? q1 : M.one, M);                  // Q^(k+b)
        const u64 sq = ms_sqr(b ? vk1 : vk, M);
        const u64 v2 = mm_sub(sq, mm_add(qb, qb, n), n);               // V_2(k+b)
        qk = ms_mul(qk, qb, M);                                        // Q^(2k+b)
        vk = b ? w : v2;
        vk1 = b ? v2 : w;
    }
    if (vk == 0 || mm_add(vk1, vk1, n) == vk) return true;             // V_d = 0 or U_d = 0
    for (int r = 1; r < s; r++) {
        vk = mm_sub(ms_sqr(vk, M), mm_add(qk, qk, n), n);               // V_(d 2^r)
        if (vk == 0) return true;
        qk = ms_sqr(qk, M);
    }
    return false;
}

// the same test for D = 5 (P = 1, Q = -1), the D of about half of all candidates: Q^k = (-1)^k is
// a sign, so a ladder step takes the two V products only.  From (V_k, V_k+1) with Q^k = sg:
// V_2k+1 = V_k V_k+1 - sg, V_2k = V_k^2 - 2 sg, V_2k+2 = V_k+1^2 + 2 sg (Q^(k+1) = -sg); k's
// parity after the step is the exponent bit.  Then Q^d = -1 (d odd), so V_2d = V_d^2 + 2 and
// V_(d 2^r) = V^2 - 2 for r >= 2.
__device__ __forceinline__ bool lucas_strong_d5(const Mod64 &M)
{
    const u64 n = M.n;
    const int s = __ffsll((long long)(n + 1)) - 1;
    const u64 d = (n + 1) >> s;
    const u64 one = M.one, two = mm_add(one, one, n);
    // k = 1: V_1 = 1, V_2 = 1 + 2 = 3, Q^1 = -1
    u64 vk = one, vk1 = mm_add(two, one, n);
    bool neg = true;                                                   // Q^k = -1
    for (int i = 62 - __clzll((long long)d); i >= 0; i--) {
        const bool b = (d >> i) & 1;
        const u64 p = ms_mul(vk, vk1, M);
        const u64 w = neg ? mm_add(p, one, n) : mm_sub(p, one, n);     // V_2k+1
        const u64 sq = ms_sqr(b ? vk1 : vk, M);
        // V_2k = sq - 2 sg; V_2k+2 = sq + 2 sg: subtract 2 exactly when (sg = +1) != b
        const bool sub2 = (!neg) != b;
        const u64 v2 = sub2 ? mm_sub(sq, two, n) : mm_add(sq, two, n);
        vk = b ? w : v2;
        vk1 = b ? v2 : w;
        neg = b;
    }
    if (vk == 0 || mm_add(vk1, vk1, n) == vk) return true;             // V_d = 0 or U_d = 0
    for (int r = 1; r < s; r++) {
        const u64 sq = ms_sqr(vk, M);
        vk = r == 1 ? mm_add(sq, two, n) : mm_sub(sq, two, n);         // V_(d 2^r)
        if (vk == 0) return true;
    }
    return false;
}

// the Lucas half of BPSW for an odd n > 2 that passed the base-2 test
__device__ __forceinline__ bool lucas_u64(u64 n)
{
    if (n == ~0ull) return false;                                      // 3 | 2^64 - 1
    const i32 D = selfridge_d(n);
    if (!D) return false;
    return lucas_strong(mm_setup(n), D);
}

// primality of an odd n > 2 with no small factor to look for first: the base-2 strong test and
// the strong Lucas test (BPSW; exact below 2^64)
__device__ __forceinline__ bool bpsw_odd(u64 n)
{
    if (n == ~0ull) return false;
    const Mod64 M = mm_setup(n);
    const int c = spsp2_class(n);
    const bool p2 = c == SP_FOLD ? spsp2<SP_FOLD>(M) : spsp2<SP_WIDE>(M);
    if (!p2) return false;
    const i32 D = selfridge_d(n);
    return D && lucas_strong(M, D);
}
