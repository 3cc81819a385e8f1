// mp_mont64.cuh -- 64-bit Montgomery arithmetic (R = 2^64) and the two halves of BPSW: the
// base-2 strong probable-prime test and the strong Lucas test with Selfridge's parameters.
// Shared by the BPSW kernels (mp_bpsw.cu) and the constellation sieve (mp_chain.cu).
//
// Reference (paths inside the Mathpub project): inv64/mmul64/madd64/msub64/mhalf64
// A350826/a350826.c:565-604, sprp2_64 :618-638, jacobi :693, selfridge :739, slprp64
// :766-799.  R mod n is found by doubling (exact; no floating-point estimate).
#pragma once
#include "mp_common.cuh"

// ---- 64-bit Montgomery arithmetic, R = 2^64 ----

__device__ __forceinline__ u64 m_mul(u64 a, u64 b, u64 n, u64 ni)
{
    const u64 tl = a * b, th = __umul64hi(a, b);
    const u64 m = tl * ni;
    const u64 mh = __umul64hi(m, n);
    const u64 r = th - mh;
    return th < mh ? r + n : r;
}
__device__ __forceinline__ u64 m_add(u64 a, u64 b, u64 n) { const u64 s = a + b; return (s < a || s >= n) ? s - n : s; }
__device__ __forceinline__ u64 m_sub(u64 a, u64 b, u64 n) { return a >= b ? a - b : a - b + n; }
__device__ __forceinline__ u64 m_half(u64 a, u64 n) { return (a & 1) ? (a >> 1) + (n >> 1) + 1 : a >> 1; }

// n^-1 mod 2^64 for odd n: (3n) xor 2 is correct to 5 bits; four Newton steps give 80
__device__ __forceinline__ u64 m_inv(u64 n)
{
    u64 x = (3 * n) ^ 2;
    x *= 2 - n * x;
    x *= 2 - n * x;
    x *= 2 - n * x;
    x *= 2 - n * x;
    return x;
}

// 2^64 mod n for odd n > 1, by doubling 2^b (b = top bit of n, so 2^b < n) 64 - b times
__device__ __forceinline__ u64 m_one(u64 n)
{
    const int b = 63 - __clzll((long long)n);
    u64 x = 1ull << b;
    for (int i = b; i < 64; i++) x = m_add(x, x, n);
    return x;
}

// Montgomery form of a small signed integer v (|v| < n) by double-and-add of `one`
__device__ __forceinline__ u64 m_small(i32 v, u64 one, u64 n)
{
    u32 a = v < 0 ? (u32)(-v) : (u32)v;
    u64 r = 0;
    for (int i = 31 - __clz((int)(a | 1)); i >= 0; i--) {
        r = m_add(r, r, n);
        if ((a >> i) & 1) r = m_add(r, one, n);
    }
    if (v < 0 && r) r = n - r;
    return r;
}

// ---- base-2 strong probable-prime test (odd n > 2) ----
__device__ __forceinline__ bool sprp2_dev(u64 n, u64 ni, u64 one)
{
    const u64 mone = n - one;
    u64 d = n - 1;
    const int s = __ffsll((long long)d) - 1;
    d >>= s;
    const int top = 63 - __clzll((long long)d);
    u64 x = m_add(one, one, n);                  // 2, for the top bit of d
    for (int i = top - 1; i >= 0; i--) {
        x = m_mul(x, x, n, ni);
        const u64 y = m_add(x, x, n);
        x = ((d >> i) & 1) ? y : x;
    }
    if (x == one || x == mone) return true;
    for (int i = 1; i < s; i++) {
        x = m_mul(x, x, n, ni);
        if (x == mone) return true;
        if (x == one) return false;
    }
    return false;
}

// ---- strong Lucas test ----

// Jacobi symbol (D/n) for odd D with |D| < n, odd n
__device__ __forceinline__ int jacobi_small(i32 D, u64 n)
{
    int t = 1;
    u32 a;
    if (D < 0) {
        a = (u32)(-D);
        if ((n & 3) == 3) t = -t;             // (-1/n)
    } else a = (u32)D;
    if ((a & 3) == 3 && (n & 3) == 3) t = -t; // reciprocity (a/n) = +-(n/a), a odd
    u32 x = (u32)(n % a), m = a;
    while (x) {
        while (!(x & 1)) {
            x >>= 1;
            const u32 r = m & 7;
            if (r == 3 || r == 5) t = -t;
        }
        const u32 tmp = x; x = m; m = tmp;
        if ((x & 3) == 3 && (m & 3) == 3) t = -t;
        x %= m;
    }
    return m == 1 ? t : 0;
}

__device__ __forceinline__ u64 isqrt_dev(u64 n)
{
    u64 r = 0, bit = 1ull << 62;
    while (bit > n) bit >>= 2;
    while (bit) {
        if (n >= r + bit) { n -= r + bit; r = (r >> 1) + bit; }
        else r >>= 1;
        bit >>= 2;
    }
    return r;
}

__device__ __forceinline__ bool is_square_dev(u64 n)
{
    // squares mod 64 are 0, 1, 4, 9, 16, 17, 25, 33, 36, 41, 49, 57
    const u64 sq64 = (1ull << 0) | (1ull << 1) | (1ull << 4) | (1ull << 9) | (1ull << 16) | (1ull << 17) |
                     (1ull << 25) | (1ull << 33) | (1ull << 36) | (1ull << 41) | (1ull << 49) | (1ull << 57);
    if (!((sq64 >> (n & 63)) & 1)) return false;
    const u64 r = isqrt_dev(n);
    return r * r == n;
}

// Selfridge method A: first D in 5, -7, 9, -11, ... with (D/n) = -1.  The search is bounded;
// for n < 2^64 that is not a square a suitable D has |D| far below the bound.
__device__ __forceinline__ bool selfridge_dev(u64 n, i32 *Dout)
{
    if (is_square_dev(n)) return false;
    i32 D = 5;
    for (int it = 0; it < 4096; it++) {
        const int j = jacobi_small(D, n);
        if (j == -1) { *Dout = D; return true; }
        if (j == 0 && (u64)(D < 0 ? -D : D) != n) return false;
        D = D > 0 ? -(D + 2) : -(D - 2);
    }
    return false;
}

__device__ __forceinline__ bool slprp_dev(u64 n, u64 ni, u64 one)
{
    i32 D;
    if (!selfridge_dev(n, &D)) return false;
    const i32 Q = (1 - D) / 4;
    const u64 Qm = m_small(Q, one, n), Dm = m_small(D, one, n);
    u64 d = n + 1;                               // n < 2^64 - 1 here (2^64 - 1 has factor 3)
    const int s = __ffsll((long long)d) - 1;
    d >>= s;
    u64 U = one, V = one, Qk = Qm;
    for (int b = 62 - __clzll((long long)d); b >= 0; b--) {
        U = m_mul(U, V, n, ni);
        V = m_sub(m_mul(V, V, n, ni), m_add(Qk, Qk, n), n);
        Qk = m_mul(Qk, Qk, n, ni);
        if ((d >> b) & 1) {
            const u64 U2 = m_add(U, V, n);
            const u64 V2 = m_add(m_mul(Dm, U, n, ni), V, n);
            U = m_half(U2, n);
            V = m_half(V2, n);
            Qk = m_mul(Qk, Qm, n, ni);
        }
    }
    if (U == 0 || V == 0) return true;
    for (int r = 1; r < s; r++) {
        V = m_sub(m_mul(V, V, n, ni), m_add(Qk, Qk, n), n);
        if (V == 0) return true;
        Qk = m_mul(Qk, Qk, n, ni);
    }
    return false;
}

// primality of an odd n > 2 without small factors to look for first: the base-2 strong test
// and the strong Lucas test (BPSW; exact for n < 2^64)
__device__ __forceinline__ bool bpsw_odd(u64 n)
{
    const u64 ni = m_inv(n), one = m_one(n);
    return sprp2_dev(n, ni, one) && slprp_dev(n, ni, one);
}
