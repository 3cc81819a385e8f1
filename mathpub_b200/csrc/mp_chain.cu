// mp_chain.cu -- the constellation sieve for chains of consecutive primes with gaps 2, 4, 6, ...
// (A016045) and with gaps ..., 6, 4, 2 (A263049), without enumerating primes.  The method is
// the one gapchain/README_SIEVE.md describes for gapchain/gapsieve.c:
//
//   wheel     the residues of p modulo the primes 2..q_w that leave every member coprime to
//             them, combined by CRT into the admissible classes mod W; a segment of 2^17 W
//             integers from `base` holds, in class j, p = base + s0 + kW, s0 = (res_j - base)
//             mod W, k < 2^17
//   patterns  for each sieve prime q above the wheel, member o of p is divisible by q exactly
//             when k + r = -W^-1 o (mod q), r = W^-1 (base + s0) mod q.  The forbidden
//             residues of a group of primes (period P = their product) make one bit pattern,
//             which a class reads from the rotation R = CRT(r) mod P, so 2^17 values of k cost
//             a few 64-bit window reads and ANDs per word (gapsieve.c:1136-1180)
//   screen    every member of every survivor by the base-2 strong test (a composite verdict
//             is a proof): one member at a time over the whole list with compaction between
//             rounds, then the remaining members per candidate
//   verify    members prime (exact: BPSW below 2^64, Miller-Rabin with the 13 prime bases 2..41
//             above, to 3.3e24), the odd numbers between them composite, the chain extended
//             (forwards for gaps 2, 4, ...; backwards for ..., 4, 2, whose pattern ends every
//             chain it is part of)
//
// Front ends sharing the kernels:
//   cu_*              the C ABI of gapchain/gapsieve_cuda.h (include/gapsieve_cuda.h), so the
//                     reference's host program gapchain/gapsieve_cuda_host.c runs unmodified
//                     on these kernels; its host builds the tables and proves the survivors,
//                     up to its ceiling 3.3e24 (two-word Montgomery arithmetic above 2^64)
//   mp_chain_sieve    every chain with its key in a range, in order, like mp_gap_chains; the
//                     tables built here and the verification on the GPU (and its 128-bit form)
//   mp_chain_first    the first chain of a range, as gapsieve --first (and its 128-bit form)
//   mp_tuple_count    count and checksum of a prime constellation (A350826's sextuplets)
#include "mp_mont64.cuh"
#include <algorithm>
#include <numeric>
#include "../../include/gapsieve_cuda.h"

#define CS_K 131072u                          // values of k per class and segment
#define CS_THREADS 256u
#define CS_MAXG 64                            // pattern groups
#define CS_SIEVE_LO 1024u                     // mp_chain_sieve: heads below this are checked one by one
#define CS_PMAX_LIMIT 509u                    // pattern primes stay below CS_SIEVE_LO
#define CS_PERIOD_MAX (1u << 24)
#define CS_MAXLEN (MP_CHAIN_MAX - 1)
#define CS_NCNT (CU_MAXK + 2)                 // counters per shape: raw, after each round, final

typedef unsigned __int128 u128t;
typedef unsigned long long ull;

// ---- two-word Montgomery arithmetic (R = 2^128) for odd n < 2^127 ----

struct w2 { u64 lo, hi; };

__device__ __forceinline__ bool w2_ge(w2 a, w2 b) { return a.hi != b.hi ? a.hi > b.hi : a.lo >= b.lo; }
__device__ __forceinline__ bool w2_eq(w2 a, w2 b) { return a.hi == b.hi && a.lo == b.lo; }
__device__ __forceinline__ w2 w2_sub(w2 a, w2 b) { return w2{a.lo - b.lo, a.hi - b.hi - (a.lo < b.lo)}; }
// a + b mod n for a, b < n < 2^127 (the sum fits in 128 bits)
__device__ __forceinline__ w2 w2_madd(w2 a, w2 b, w2 n)
{
    w2 s;
    s.lo = a.lo + b.lo;
    s.hi = a.hi + b.hi + (s.lo < a.lo);
    return w2_ge(s, n) ? w2_sub(s, n) : s;
}
// CIOS product a b 2^-128 mod n for a, b < n; ni = -n^-1 mod 2^64.  After each word of b the
// running sum is below 2n, so three words hold it and one subtraction finishes.
__device__ __forceinline__ w2 w2_mmul(w2 a, w2 b, w2 n, u64 ni)
{
    u64 t0, t1, t2, m;
    u128t p;
    p = (u128t)a.lo * b.lo;                       t0 = (u64)p;
    p = (u128t)a.hi * b.lo + (u64)(p >> 64);      t1 = (u64)p; t2 = (u64)(p >> 64);
    m = t0 * ni;
    p = (u128t)m * n.lo + t0;
    p = (u128t)m * n.hi + t1 + (u64)(p >> 64);    t0 = (u64)p;
    p = (u128t)t2 + (u64)(p >> 64);               t1 = (u64)p; t2 = (u64)(p >> 64);
    p = (u128t)a.lo * b.hi + t0;                  t0 = (u64)p;
    p = (u128t)a.hi * b.hi + t1 + (u64)(p >> 64); t1 = (u64)p; t2 += (u64)(p >> 64);
    m = t0 * ni;
    p = (u128t)m * n.lo + t0;
    p = (u128t)m * n.hi + t1 + (u64)(p >> 64);    t0 = (u64)p;
    p = (u128t)t2 + (u64)(p >> 64);               t1 = (u64)p; t2 = (u64)(p >> 64);
    const w2 r{t0, t1};
    return (t2 || w2_ge(r, n)) ? w2_sub(r, n) : r;
}

// the base-2 strong probable-prime test, odd 3 <= n < 2^127
__device__ bool sprp2_w2(w2 n)
{
    const u64 ni = 0 - inv64(n.lo);
    // 1 in Montgomery form, 2^128 mod n, by doubling 2^b (b = the top bit of n, so 2^b < n)
    const int b = n.hi ? 127 - __clzll((long long)n.hi) : 63 - __clzll((long long)n.lo);
    w2 one = b >= 64 ? w2{0, 1ull << (b - 64)} : w2{1ull << b, 0};
    for (int i = b; i < 128; i++) one = w2_madd(one, one, n);
    w2 d = w2_sub(n, w2{1, 0});
    int s = 0;
    if (!d.lo) { s = 64; d.lo = d.hi; d.hi = 0; }
    const int z = __ffsll((long long)d.lo) - 1;
    if (z) { d.lo = (d.lo >> z) | (d.hi << (64 - z)); d.hi >>= z; }
    s += z;
    const w2 mone = w2_sub(n, one);
    w2 x = w2_madd(one, one, n);              // 2, for the top bit of d
    const int top = d.hi ? 127 - __clzll((long long)d.hi) : 63 - __clzll((long long)d.lo);
    for (int i = top - 1; i >= 0; i--) {
        x = w2_mmul(x, x, n, ni);
        const u64 bit = i >= 64 ? (d.hi >> (i - 64)) & 1 : (d.lo >> i) & 1;
        if (bit) x = w2_madd(x, x, n);
    }
    if (w2_eq(x, one) || w2_eq(x, mone)) return true;
    for (int i = 1; i < s; i++) {
        x = w2_mmul(x, x, n, ni);
        if (w2_eq(x, mone)) return true;
        if (w2_eq(x, one)) return false;
    }
    return false;
}

// the base-2 strong test of the member base + off + o (128-bit sum, odd, >= 3)
__device__ __forceinline__ bool member_sprp2(u64 base_lo, u64 base_hi, u64 off, u32 o)
{
    u64 lo = base_lo + off;
    u64 hi = base_hi + (lo < off);
    const u64 l2 = lo + o;
    hi += l2 < lo;
    lo = l2;
    if (!hi) return spsp2_u64(lo);
    return sprp2_w2(w2{lo, hi});
}

// exact primality for any u64: trial division below 2^20, BPSW above (no pseudoprime below 2^64)
// after trial division by the primes 3..61, which settles most of the odd numbers between the
// members of a chain (those were never sieved) without an exponentiation
__device__ bool is_prime_exact(u64 x)
{
    if (x < 4) return x >= 2;
    if (!(x & 1)) return false;
    if (x < (1u << 20)) {
        const u32 y = (u32)x;
        for (u32 d = 3; d * d <= y; d += 2)
            if (y % d == 0) return false;
        return true;
    }
    if (x % 3 == 0 || x % 5 == 0 || x % 7 == 0 || x % 11 == 0 || x % 13 == 0 || x % 17 == 0 || x % 19 == 0 ||
        x % 23 == 0 || x % 29 == 0 || x % 31 == 0 || x % 37 == 0 || x % 41 == 0 || x % 43 == 0 || x % 47 == 0 ||
        x % 53 == 0 || x % 59 == 0 || x % 61 == 0)
        return false;
    return bpsw_odd(x);
}

// the strong probable-prime test to base a (2 <= a < n) for odd n >= 2^64 below 2^127, with
// one = R mod n and r2 = R^2 mod n (R = 2^128), n - 1 = d 2^s
__device__ bool mr_w2(w2 n, u64 ni, w2 one, w2 r2, w2 d, int s, u32 a)
{
    const w2 am = w2_mmul(w2{a, 0}, r2, n, ni);         // a R mod n
    const w2 mone = w2_sub(n, one);
    w2 x = am;                                          // for the top bit of d
    const int top = d.hi ? 127 - __clzll((long long)d.hi) : 63 - __clzll((long long)d.lo);
    for (int i = top - 1; i >= 0; i--) {
        x = w2_mmul(x, x, n, ni);
        const u64 bit = i >= 64 ? (d.hi >> (i - 64)) & 1 : (d.lo >> i) & 1;
        if (bit) x = w2_mmul(x, am, n, ni);
    }
    if (w2_eq(x, one) || w2_eq(x, mone)) return true;
    for (int i = 1; i < s; i++) {
        x = w2_mmul(x, x, n, ni);
        if (w2_eq(x, mone)) return true;
        if (w2_eq(x, one)) return false;
    }
    return false;
}

// exact primality below 3.317e24: BPSW below 2^64; above, Miller-Rabin with the 13 prime bases
// 2..41, which no composite below 3,317,044,064,679,887,385,961,981 passes (Sorenson and
// Webster, 2015), after trial division by the primes to 41
__device__ bool is_prime_w2(w2 n)
{
    if (!n.hi) return is_prime_exact(n.lo);
    if (!(n.lo & 1)) return false;
    const u32 B[13] = {2, 3, 5, 7, 11, 13, 17, 19, 23, 29, 31, 37, 41};
    // n mod q from the two words: (hi 2^64 + lo) mod q, 2^64 mod q by (2^64 - 1) mod q + 1
    for (int i = 1; i < 13; i++) {
        const u64 q = B[i], t = (~0ull % q + 1) % q;
        if (((n.hi % q) * t + n.lo % q) % q == 0) return false;
    }
    const u64 ni = 0 - inv64(n.lo);
    const int b = 127 - __clzll((long long)n.hi);
    w2 one = w2{0, 1ull << (b - 64)};
    for (int i = b; i < 128; i++) one = w2_madd(one, one, n);
    w2 r2 = one;
    for (int i = 0; i < 128; i++) r2 = w2_madd(r2, r2, n);
    w2 d = w2_sub(n, w2{1, 0});
    int s = 0;
    if (!d.lo) { s = 64; d.lo = d.hi; d.hi = 0; }
    const int z = __ffsll((long long)d.lo) - 1;
    if (z) { d.lo = (d.lo >> z) | (d.hi << (64 - z)); d.hi >>= z; }
    s += z;
    for (int i = 0; i < 13; i++)
        if (!mr_w2(n, ni, one, r2, d, s, B[i])) return false;
    return true;
}

__device__ __forceinline__ w2 w2_addu(w2 a, u64 b) { const u64 lo = a.lo + b; return w2{lo, a.hi + (lo < b)}; }
__device__ __forceinline__ w2 w2_subu(w2 a, u64 b) { return w2{a.lo - b, a.hi - (a.lo < b)}; }

// ---- the kernels ----

struct CsTables {                             // shared by both shapes and every unit
    const u32 *ginfo;                         // per group: P, first sieve prime, primes, word offset
    const u32 *q, *qinv, *crt;                // per sieve prime: q, W^-1 mod q, CRT coefficient mod P
    u32 ngroups, nps;
};
struct CsShape {
    const u64 *pat;                           // the groups' patterns back to back
    const u32 *res;                           // admissible residues mod W
    const u32 *offs;                          // member offsets
    u32 A, k;
};
struct CsUnit {
    u64 base_lo, base_hi;                     // segment 0 starts here
    u64 lim;                                  // the largest candidate offset in range
    u64 segsize;                              // CS_K W
    u32 W, bmodW, nseg;
    u32 j0, nj;                               // classes j0 .. j0 + nj - 1
    const u32 *bq;                            // [segment][sieve prime]: the segment's base mod q
};

// ANDs one group's rotated pattern into a thread's CS_CPT 128-bit chunks.  Chunk c of the class
// bitmap (bits 128c .. 128c + 127) comes from pattern bits abit + 128c ...: the aligned 16-byte
// chunks a + c and a + c + 1 (a = abit / 128) joined by four 32-bit funnel shifts; Q =
// (abit mod 128) / 32 picks the words, s = abit mod 32 the shift.  A chunk with no live bit
// left loads nothing: at long chains most are dead after the first few groups, which is what
// keeps the L2 traffic down.
template <int Q>
__device__ __forceinline__ void cs_and_group(u32 (&acc)[4][4], const uint4 *__restrict__ pc, u32 s)
{
#pragma unroll
    for (u32 i = 0; i < 4; i++)
        if (acc[i][0] | acc[i][1] | acc[i][2] | acc[i][3]) {
            const uint4 X = __ldg(pc + CS_THREADS * i), Y = __ldg(pc + CS_THREADS * i + 1);
            const u32 x[8] = {X.x, X.y, X.z, X.w, Y.x, Y.y, Y.z, Y.w};
#pragma unroll
            for (int w = 0; w < 4; w++) acc[i][w] &= __funnelshift_r(x[w + Q], x[w + Q + 1], s);
        }
}

// one CTA per CS_CPB classes of one segment: AND the rotated patterns over each class's 2^17
// values of k and append the survivors' offsets from the unit's base.  The rotations of all
// the CTA's classes and groups are taken in parallel before one barrier.
#define CS_CPB 8u                             // classes per CTA
#define CS_CPT (CS_K / 128 / CS_THREADS)      // 128-bit chunks per thread and class
static_assert(CS_CPT == 4, "cs_and_group takes 4 chunks per thread");
__global__ void __launch_bounds__(CS_THREADS) cs_sieve_kernel(CsTables T, CsShape S, CsUnit U, u64 *list, u64 cap,
                                                              ull *count)
{
    __shared__ u32 s_chunk[CS_CPB][CS_MAXG];  // first 16-byte chunk of the window
    __shared__ u32 s_bit[CS_CPB][CS_MAXG];    // bit offset of the window in that chunk
    __shared__ u32 s_s0[CS_CPB];
    const u32 nblk = (U.nj + CS_CPB - 1) / CS_CPB;
    const u32 jb = blockIdx.x % nblk, g = blockIdx.x / nblk;
    const u32 *bq = U.bq + (size_t)g * T.nps;
    for (u32 x = threadIdx.x; x < CS_CPB * T.ngroups; x += CS_THREADS) {
        const u32 c = x / T.ngroups, gi = x - c * T.ngroups, jj = jb * CS_CPB + c;
        if (jj >= U.nj) continue;
        const u32 r = S.res[U.j0 + jj];
        const u32 s0 = r >= U.bmodW ? r - U.bmodW : r + U.W - U.bmodW;
        if (gi == 0) s_s0[c] = s0;
        const u32 P = T.ginfo[4 * gi], first = T.ginfo[4 * gi + 1], n = T.ginfo[4 * gi + 2];
        u64 R = 0;
        for (u32 i = first; i < first + n; i++) {
            const u32 q = T.q[i];
            u32 t = bq[i] + s0 % q;
            if (t >= q) t -= q;
            R += (u64)((u64)T.qinv[i] * t % q) * T.crt[i];
        }
        const u64 abit = 64ull * T.ginfo[4 * gi + 3] + R % P;
        s_chunk[c][gi] = (u32)(abit >> 7);
        s_bit[c][gi] = (u32)(abit & 127);
    }
    __syncthreads();
    const uint4 *pat = (const uint4 *)S.pat;
    const u32 lane = threadIdx.x & 31;
    for (u32 c = 0; c < CS_CPB; c++) {
        if (jb * CS_CPB + c >= U.nj) break;                             // uniform
        u32 acc[4][4];
#pragma unroll
        for (u32 i = 0; i < 4; i++)
#pragma unroll
            for (u32 w = 0; w < 4; w++) acc[i][w] = ~0u;
        for (u32 gi = 0; gi < T.ngroups; gi++) {
            const uint4 *pc = pat + s_chunk[c][gi] + threadIdx.x;
            const u32 bit = s_bit[c][gi], s = bit & 31;
            switch (bit >> 5) {                                         // uniform
            case 0: cs_and_group<0>(acc, pc, s); break;
            case 1: cs_and_group<1>(acc, pc, s); break;
            case 2: cs_and_group<2>(acc, pc, s); break;
            default: cs_and_group<3>(acc, pc, s); break;
            }
        }
        // word w of chunk i holds k = 32 (4 (thread + 256 i) + w) + b
        const u64 off0 = (u64)g * U.segsize + s_s0[c];
        if (off0 + (u64)(CS_K - 1) * U.W > U.lim) {                     // the unit's end: offsets <= lim only
#pragma unroll
            for (u32 i = 0; i < 4; i++)
#pragma unroll
                for (u32 w = 0; w < 4; w++) {
                    const u64 o0 = off0 + 32ull * (4 * (threadIdx.x + CS_THREADS * i) + w) * U.W;
                    const u64 room = o0 > U.lim ? 0 : (U.lim - o0) / U.W + 1;
                    if (room < 32) acc[i][w] &= (1u << room) - 1;
                }
        }
        u32 nb = 0;
#pragma unroll
        for (u32 i = 0; i < 4; i++)
#pragma unroll
            for (u32 w = 0; w < 4; w++) nb += __popc(acc[i][w]);
        if (!__ballot_sync(0xffffffffu, nb)) continue;                  // warp-uniform
        u32 incl = nb;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const u32 v = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= (u32)d) incl += v;
        }
        const u32 tot = __shfl_sync(0xffffffffu, incl, 31);
        ull bpos = 0;
        if (lane == 31) bpos = atomicAdd(count, (ull)tot);
        bpos = __shfl_sync(0xffffffffu, bpos, 31);
        u64 pos = bpos + incl - nb;
        if (!nb) continue;
#pragma unroll
        for (u32 i = 0; i < 4; i++)
#pragma unroll
            for (u32 w = 0; w < 4; w++) {
                u32 m = acc[i][w];
                const u64 o0 = off0 + 32ull * (4 * (threadIdx.x + CS_THREADS * i) + w) * U.W;
                while (m) {
                    const u32 b = __ffs(m) - 1;
                    m &= m - 1;
                    if (pos < cap) list[pos] = o0 + (u64)b * U.W;
                    pos++;
                }
            }
    }
}

// warp-aggregated append (every lane of the warp takes part)
__device__ __forceinline__ void cs_append(bool keep, u64 v, u64 *out, ull *nout)
{
    const u32 lane = threadIdx.x & 31;
    const u32 bal = __ballot_sync(0xffffffffu, keep);
    if (!bal) return;
    ull base = 0;
    if (lane == 0) base = atomicAdd(nout, (ull)__popc(bal));
    base = __shfl_sync(0xffffffffu, base, 0);
    if (keep) out[base + __popc(bal & ((1u << lane) - 1))] = v;
}

// member m over the whole list: keep the offsets whose member passes the base-2 test
__global__ void __launch_bounds__(256) cs_screen_member(const u64 *__restrict__ in, const ull *nin, u64 cap, u64 *out,
                                                        ull *nout, u64 base_lo, u64 base_hi, const u32 *offs, u32 m)
{
    const u64 n = min((u64)*nin, cap);
    const u32 o = offs[m];
    for (u64 i0 = (u64)blockIdx.x * blockDim.x; i0 < n; i0 += (u64)gridDim.x * blockDim.x) {
        const u64 i = i0 + threadIdx.x;
        const u64 off = i < n ? in[i] : 0;
        const bool keep = i < n && member_sprp2(base_lo, base_hi, off, o);
        cs_append(keep, off, out, nout);
    }
}

// members m0 .. k - 1 per candidate, stopping at the first composite
__global__ void __launch_bounds__(256) cs_screen_tail(const u64 *__restrict__ in, const ull *nin, u64 cap, u64 *out,
                                                      ull *nout, u64 base_lo, u64 base_hi, const u32 *offs, u32 m0,
                                                      u32 k)
{
    const u64 n = min((u64)*nin, cap);
    for (u64 i0 = (u64)blockIdx.x * blockDim.x; i0 < n; i0 += (u64)gridDim.x * blockDim.x) {
        const u64 i = i0 + threadIdx.x;
        const u64 off = i < n ? in[i] : 0;
        bool keep = i < n;
        for (u32 m = m0; m < k && keep; m++) keep = member_sprp2(base_lo, base_hi, off, offs[m]);
        cs_append(keep, off, out, nout);
    }
}

// mp_chain_sieve's exact check of the screen's survivors p = base + off (128-bit): shape 0
// (gaps 2, 4, ...): members p + m(m + 1) prime and the odd numbers between them composite,
// extended forwards; shape 1 (..., 4, 2): the k-member pattern p + m(2k - 1 - m) exact, then
// extended backwards while the gap before the first prime is 2 len.  Chains of CS_MAXLEN primes
// are not extended further.  Heads are written as (low, high) word pairs.
__global__ void __launch_bounds__(128) cs_verify_kernel(const u64 *__restrict__ in, const ull *nin, u64 cap,
                                                        u64 base_lo, u64 base_hi, u32 k, u32 shape, u64 *heads,
                                                        u32 *lens, ull *nres)
{
    const u64 n = min((u64)*nin, cap);
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        const w2 p = w2_addu(w2{base_lo, base_hi}, in[i]);
        w2 head = p;
        u32 len = 0;
        if (shape == 0) {
            for (u32 m = 0; m < CS_MAXLEN; m++) {
                const w2 x = w2_addu(p, (u64)m * (m + 1));
                if (!is_prime_w2(x)) break;
                bool clear = true;
                for (u32 t = 1; m && t < m && clear; t++) clear = !is_prime_w2(w2_subu(x, 2 * (u64)t));
                if (!clear) break;
                len = m + 1;
            }
            if (len < k) len = 0;
        } else {
            bool ok = true;
            for (u32 m = 0; m < k && ok; m++) {
                const w2 x = w2_addu(p, (u64)m * (2 * k - 1 - m));
                ok = is_prime_w2(x);
                for (u32 t = 1; ok && m + 1 < k && t < k - 1 - m; t++) ok = !is_prime_w2(w2_addu(x, 2 * (u64)t));
            }
            if (ok) {
                len = k;
                while (len < CS_MAXLEN) {
                    const u64 gap = 2 * (u64)len;
                    if (!head.hi && head.lo < gap + 3) break;
                    const w2 prev = w2_subu(head, gap);
                    bool step = is_prime_w2(prev);
                    for (u32 t = 1; step && t < len; t++) step = !is_prime_w2(w2_addu(prev, 2 * (u64)t));
                    if (!step) break;
                    head = prev;
                    len++;
                }
            }
        }
        if (len) {
            const ull j = atomicAdd(nres, 1ull);
            if (j < cap) { heads[2 * j] = head.lo; heads[2 * j + 1] = head.hi; lens[j] = len; }
        }
    }
}

// the same check when every value of the unit lies below 2^64 - 2^12: one-word arithmetic (and
// half the registers of the two-word form), heads written as (head, 0) pairs
__global__ void __launch_bounds__(128) cs_verify64_kernel(const u64 *__restrict__ in, const ull *nin, u64 cap, u64 base,
                                                          u32 k, u32 shape, u64 *heads, u32 *lens, ull *nres)
{
    const u64 n = min((u64)*nin, cap);
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        const u64 p = base + in[i];
        u64 head = p;
        u32 len = 0;
        if (shape == 0) {
            for (u32 m = 0; m < CS_MAXLEN; m++) {
                const u64 x = p + (u64)m * (m + 1);
                if (!is_prime_exact(x)) break;
                bool clear = true;
                for (u64 y = x - 2 * (u64)m + 2; m && y < x && clear; y += 2) clear = !is_prime_exact(y);
                if (!clear) break;
                len = m + 1;
            }
            if (len < k) len = 0;
        } else {
            bool ok = true;
            for (u32 m = 0; m < k && ok; m++) {
                const u64 x = p + (u64)m * (2 * k - 1 - m);
                ok = is_prime_exact(x);
                for (u64 y = x + 2; ok && m + 1 < k && y < x + 2 * (u64)(k - 1 - m); y += 2) ok = !is_prime_exact(y);
            }
            if (ok) {
                len = k;
                while (len < CS_MAXLEN) {
                    const u64 gap = 2 * (u64)len;
                    if (head < gap + 3) break;
                    const u64 prev = head - gap;
                    bool step = is_prime_exact(prev);
                    for (u64 y = prev + 2; step && y < head; y += 2) step = !is_prime_exact(y);
                    if (!step) break;
                    head = prev;
                    len++;
                }
            }
        }
        if (len) {
            const ull j = atomicAdd(nres, 1ull);
            if (j < cap) { heads[2 * j] = head; heads[2 * j + 1] = 0; lens[j] = len; }
        }
    }
}

// all the kernels of one unit of one shape, queued on st.  The survivors end in lists[*fin];
// counters: cnt[0] the sieve's, cnt[r + 1] after screening round r, cnt[*fcnt] the final one.
struct CsLists {
    u64 *list[2];
    u64 cap;
    ull *cnt;                                  // CS_NCNT counters
};
static void cs_queue_unit(const CsTables &T, const CsShape &S, const CsUnit &U, const CsLists &L, u32 split,
                          int sm_count, cudaStream_t st, int *fin, u32 *fcnt)
{
    const u32 rounds = std::min(split, S.k);
    cudaMemsetAsync(L.cnt, 0, (size_t)(rounds + 2) * sizeof(ull), st);
    cs_sieve_kernel<<<(U.nj + CS_CPB - 1) / CS_CPB * U.nseg, CS_THREADS, 0, st>>>(T, S, U, L.list[0], L.cap, L.cnt);
    const unsigned grid = (unsigned)sm_count * 8;
    int cur = 0;
    for (u32 r = 0; r < rounds; r++, cur ^= 1)
        cs_screen_member<<<grid, 256, 0, st>>>(L.list[cur], L.cnt + r, L.cap, L.list[cur ^ 1], L.cnt + r + 1,
                                               U.base_lo, U.base_hi, S.offs, r);
    if (rounds < S.k) {
        cs_screen_tail<<<grid, 256, 0, st>>>(L.list[cur], L.cnt + rounds, L.cap, L.list[cur ^ 1],
                                             L.cnt + rounds + 1, U.base_lo, U.base_hi, S.offs, rounds, S.k);
        cur ^= 1;
        *fcnt = rounds + 1;
    } else {
        *fcnt = rounds;
    }
    *fin = cur;
}

// ---- host tables (the reference host builds the same ones for the cu_* path) ----

namespace {

u64 inv_mod(u64 a, u64 m)                      // a^-1 mod m, gcd(a, m) = 1
{
    i64 t = 0, nt = 1, r = (i64)m, nr = (i64)(a % m);
    while (nr) {
        const i64 q = r / nr;
        i64 x = t - q * nt; t = nt; nt = x;
        x = r - q * nr; r = nr; nr = x;
    }
    return (u64)(t < 0 ? t + (i64)m : t);
}

bool is_small_prime(u32 q)
{
    if (q < 2) return false;
    for (u32 d = 2; d * d <= q; d++)
        if (q % d == 0) return false;
    return true;
}

struct CsPlan {
    u32 k = 0;
    u64 W = 1;
    std::vector<u32> res, offs, ginfo, q, qinv, crt;
    std::vector<u64> pat;
    double survive = 1;                         // the fraction of k values the patterns keep
};

// member offsets of a chain of k primes: gaps 2, 4, ... (shape 0) or ..., 4, 2 (shape 1)
std::vector<u32> chain_offsets(u32 k, u32 shape)
{
    std::vector<u32> o(k);
    for (u32 m = 0; m < k; m++) o[m] = shape == 0 ? m * (m + 1) : m * (2 * k - 1 - m);
    return o;
}

// for the member offsets offs: the wheel (grown while W <= 3e7 and the classes number at most
// 24,000), the pattern groups of the primes above it up to pattern_pmax (periods up to 2^24) and
// their patterns.  False when some prime leaves no admissible residue: then no p at or above
// CS_SIEVE_LO has all its members prime.
// the largest pattern prime for patterns of k members: the screen's work falls with the
// survivors, each further prime q removing about k/q of them, while every group costs a window
// read per live word; short patterns leave many survivors and gain from deeper patterns
u32 pattern_pmax(u32 k)
{
    return (k >= 6 && k < 12) ? CS_PMAX_LIMIT : 199u;
}

bool make_plan(const std::vector<u32> &offs, CsPlan &P)
{
    const u32 pmax = pattern_pmax((u32)offs.size());
    static_assert(CS_PMAX_LIMIT < CS_SIEVE_LO, "members above CS_SIEVE_LO exceed every pattern prime");
    P.k = (u32)offs.size();
    P.offs = offs;
    std::vector<u64> cls{0};
    u64 W = 1;
    u32 q = 2;
    for (; q <= pmax; q++) {
        if (!is_small_prime(q)) continue;
        std::vector<u32> adm;
        for (u32 r = 0; r < q; r++) {
            bool ok = true;
            for (u32 o : P.offs) ok = ok && (r + o) % q != 0;
            if (ok) adm.push_back(r);
        }
        if (adm.empty()) return false;
        if (q > 2 && (W * q > 30000000ull || cls.size() * adm.size() > 24000)) break;
        std::vector<u64> nc;                    // CRT: x = c (mod W), x = r (mod q)
        const u64 Wi = inv_mod(W % q, q);
        for (u64 c : cls)
            for (u32 r : adm) nc.push_back(c + W * (((r + q - c % q) % q) * Wi % q));
        cls.swap(nc);
        W *= q;
    }
    std::sort(cls.begin(), cls.end());
    P.W = W;
    P.res.assign(cls.begin(), cls.end());
    // groups of the next primes up to pmax
    std::vector<std::vector<u32>> groups;
    std::vector<u32> cur;
    u64 per = 1;
    for (; q <= pmax; q++) {
        if (!is_small_prime(q)) continue;
        if (per * q > CS_PERIOD_MAX) { groups.push_back(cur); cur.clear(); per = 1; }
        cur.push_back(q);
        per *= q;
    }
    if (!cur.empty()) groups.push_back(cur);
    if (groups.size() > CS_MAXG) return false;
    for (const auto &G : groups) {
        u64 Pg = 1;
        for (u32 qq : G) Pg *= qq;
        const u32 first = (u32)P.q.size();
        std::vector<u8> ok(Pg, 1);
        for (u32 qq : G) {
            const u64 Wi = inv_mod(W % qq, qq);
            std::vector<u8> bad(qq, 0);
            u32 nbad = 0;
            for (u32 o : P.offs) {
                const u64 f = (qq - o % qq) % qq * Wi % qq;          // k + r = -W^-1 o (mod q)
                if (bad[f]) continue;
                bad[f] = 1;
                nbad++;
                for (u64 y = f; y < Pg; y += qq) ok[y] = 0;
            }
            if (nbad == qq) return false;
            P.survive *= 1.0 - (double)nbad / qq;
            const u64 M = Pg / qq;
            P.q.push_back(qq);
            P.qinv.push_back((u32)Wi);
            P.crt.push_back((u32)(M * inv_mod(M % qq, qq) % Pg));
        }
        // the period, then its first CS_K + 128 bits again, so that no window read wraps
        const u64 nbits = Pg + CS_K + 128, nw = (nbits + 63) / 64;
        const u64 w0 = P.pat.size();
        P.ginfo.insert(P.ginfo.end(), {(u32)Pg, first, (u32)G.size(), (u32)w0});
        P.pat.resize(w0 + nw, 0);
        for (u64 y = 0, yy = 0; y < nbits; y++, yy = yy + 1 == Pg ? 0 : yy + 1)
            if (ok[yy]) P.pat[w0 + (y >> 6)] |= 1ull << (y & 63);
    }
    return true;
}

// LSD radix sort of (head, len) pairs by head (128-bit), skipping the digits where all heads agree
void sort_chains(std::vector<u128t> &H, std::vector<u32> &L)
{
    const size_t n = H.size();
    if (n < 2) return;
    std::vector<u128t> h2(n);
    std::vector<u32> l2(n);
    u128t top = 0;
    for (const u128t &v : H) top |= v;
    for (int sh = 0; sh < 128 && (top >> sh); sh += 11) {
        std::vector<size_t> cnt(2048, 0);
        for (const u128t &v : H) cnt[(size_t)(v >> sh) & 2047]++;
        if (*std::max_element(cnt.begin(), cnt.end()) == n) continue;
        size_t pos = 0;
        for (size_t &c : cnt) { const size_t t = c; c = pos; pos += t; }
        for (size_t i = 0; i < n; i++) {
            const size_t d = cnt[(size_t)(H[i] >> sh) & 2047]++;
            h2[d] = H[i];
            l2[d] = L[i];
        }
        H.swap(h2);
        L.swap(l2);
    }
}

template <class T> cudaError_t upload(DevBuf &b, const std::vector<T> &v)
{
    cudaError_t e = b.ensure(std::max<size_t>(v.size(), 1) * sizeof(T));
    if (e == cudaSuccess && !v.empty()) e = cudaMemcpy(b.p, v.data(), v.size() * sizeof(T), cudaMemcpyHostToDevice);
    return e;
}

}  // namespace

// exact check of the screen's survivors for mp_tuple_count: every member prime; count and sum
// of mix64(p) into the two counters
__global__ void __launch_bounds__(128) cs_tuple_kernel(const u64 *__restrict__ in, const ull *nin, u64 cap, u64 base,
                                                       const u32 *__restrict__ offs, u32 k, ull *acc)
{
    const u64 n = min((u64)*nin, cap);
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        const u64 p = base + in[i];
        bool ok = true;
        for (u32 m = 0; m < k && ok; m++) ok = is_prime_exact(p + offs[m]);
        if (ok) {
            atomicAdd(acc, 1ull);
            atomicAdd(acc + 1, (ull)mp_mix64(p));
        }
    }
}

// the same above 2^64: every member prime (13-base Miller-Rabin above 2^64), and the reference's
// checksum term hashp(p) = mix64(lo64(p) xor hi64(p) GOLD) (A350826/a350826.c:434-438), which is
// mix64(p) below 2^64
__global__ void __launch_bounds__(128) cs_tuple128_kernel(const u64 *__restrict__ in, const ull *nin, u64 cap,
                                                          u64 base_lo, u64 base_hi, const u32 *__restrict__ offs,
                                                          u32 k, ull *acc)
{
    const u64 n = min((u64)*nin, cap);
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        const w2 p = w2_addu(w2{base_lo, base_hi}, in[i]);
        bool ok = true;
        for (u32 m = 0; m < k && ok; m++) ok = is_prime_w2(w2_addu(p, offs[m]));
        if (ok) {
            atomicAdd(acc, 1ull);
            atomicAdd(acc + 1, (ull)mp_mix64(p.lo ^ (p.hi * MP_GOLD)));
        }
    }
}

// ---- mp_chain_sieve, mp_chain_first and mp_tuple_count: one plan and buffers per handle ----

#define CS_MODE_TUPLE 2u                       // modes 0 and 1 are the chain shapes

struct ChainDev {
    u32 mode = 0, k = 0;
    std::vector<u32> key;                      // the member offsets the plan was built for
    bool ok = false;                           // false: no admissible p at or above CS_SIEVE_LO
    CsPlan plan;
    // the last chain list when the caller's arrays were too small, for the call that follows
    // with room for all of it (count first, then fill) so that the range is not sieved twice
    bool kept = false;
    u128t kept_lo = 0, kept_hi = 0;
    std::vector<u128t> kept_h;
    std::vector<u32> kept_l;
    DevBuf ginfo, q, qinv, crt, pat, res, offs, bq, l0, l1, cnt, rh, rl;
    void release()
    {
        for (DevBuf *b : {&ginfo, &q, &qinv, &crt, &pat, &res, &offs, &bq, &l0, &l1, &cnt, &rh, &rl}) b->release();
    }
};
// counters in D.cnt: CS_NCNT for the unit's lists, then the chain count, then the tuple count
// and checksum
#define CS_CNT_RES CS_NCNT
#define CS_CNT_TUPLE (CS_NCNT + 1)

void mp_chain_free(mp_handle *h)
{
    if (!h->chain) return;
    h->chain->release();
    delete h->chain;
    h->chain = nullptr;
}

// the handle's plan for (mode, offs), built and uploaded when it differs from the last one
static int cs_prepare(mp_handle *h, u32 mode, const std::vector<u32> &offs)
{
    if (h->chain && h->chain->mode == mode && h->chain->key == offs) return MP_OK;
    mp_chain_free(h);
    h->chain = new ChainDev();
    ChainDev &D = *h->chain;
    D.mode = mode;
    D.k = (u32)offs.size();
    D.key = offs;
    D.ok = make_plan(offs, D.plan);
    const CsPlan &P = D.plan;
    if (D.ok) {
        MP_CUDA(h, upload(D.ginfo, P.ginfo));
        MP_CUDA(h, upload(D.q, P.q));
        MP_CUDA(h, upload(D.qinv, P.qinv));
        MP_CUDA(h, upload(D.crt, P.crt));
        MP_CUDA(h, upload(D.pat, P.pat));
        MP_CUDA(h, upload(D.res, P.res));
    }
    MP_CUDA(h, upload(D.offs, P.offs));
    MP_CUDA(h, D.cnt.ensure((CS_NCNT + 3) * sizeof(ull)));
    return MP_OK;
}

// every candidate of [lo, hi) (128-bit): the odd p below CS_SIEVE_LO (where a member may be a
// sieve prime) as one list, then the sieve's units.  collect(list, count on the device,
// capacity, base, expected survivors) checks each list exactly; done() is asked after the
// strip and after every run of segments (all its classes): true ends the range there
// (candidates come in ascending runs, so an earlier run holds smaller p).
template <class Collect, class Done>
static int cs_sieve_range(mp_handle *h, ChainDev &D, u128t lo, u128t hi, cudaStream_t st, Collect &&collect,
                          Done &&done)
{
    const CsPlan &P = D.plan;
    if (lo < CS_SIEVE_LO) {
        std::vector<u64> strip;
        const u64 e = hi < CS_SIEVE_LO ? (u64)hi : CS_SIEVE_LO;
        for (u64 p = std::max<u64>((u64)lo, 3) | 1; p < e; p += 2) strip.push_back(p);
        if (!strip.empty()) {
            MP_CUDA(h, upload(D.l0, strip));
            const ull n = strip.size();
            MP_CUDA(h, cudaMemcpy(D.cnt.p, &n, sizeof n, cudaMemcpyHostToDevice));
            MP_TRY(collect(D.l0.as<u64>(), D.cnt.as<ull>(), n, (u128t)0, n));
        }
    }
    if (done()) return MP_OK;
    const u128t slo = lo > CS_SIEVE_LO ? lo : (u128t)CS_SIEVE_LO;
    if (!D.ok || slo >= hi) return MP_OK;
    const u64 W = P.W, segsize = (u64)CS_K * W;
    const u32 A = (u32)P.res.size(), nps = (u32)P.q.size();
    const u64 nseg_all = (u64)((hi - slo + segsize - 1) / segsize);
    // units: runs of segments (or, for dense patterns, runs of classes of one segment) sized
    // for about 2^24 expected sieve survivors
    const double per_class = (double)CS_K * P.survive, target = 16777216.0;
    u32 useg = 1, ucls = A;
    if (per_class * A <= target) useg = (u32)std::min<double>(256.0, std::floor(target / (per_class * A)));
    else ucls = (u32)std::max<double>(1.0, std::floor(target / per_class));
    u64 ucap = (u64)(1.25 * per_class * ucls * useg) + 65536;
    const CsTables T{D.ginfo.as<u32>(), D.q.as<u32>(), D.qinv.as<u32>(), D.crt.as<u32>(), (u32)(P.ginfo.size() / 4),
                     nps};
    const CsShape S{D.pat.as<u64>(), D.res.as<u32>(), D.offs.as<u32>(), A, D.k};
    std::vector<u32> bq((size_t)useg * nps);
    MP_CUDA(h, D.bq.ensure(bq.size() * 4));
    for (u64 s = 0; s < nseg_all; s += useg) {
        const u32 ns = (u32)std::min<u64>(useg, nseg_all - s);
        const u128t base = slo + (u128t)s * segsize;
        for (u32 g = 0; g < ns; g++)
            for (u32 i = 0; i < nps; i++) bq[(size_t)g * nps + i] = (u32)((base + (u128t)g * segsize) % P.q[i]);
        MP_CUDA(h, cudaMemcpyAsync(D.bq.p, bq.data(), (size_t)ns * nps * 4, cudaMemcpyHostToDevice, st));
        const u128t room = hi - 1 - base;
        const u64 lim = room > (u128t)~0ull ? ~0ull : (u64)room;
        for (u32 j0 = 0; j0 < A; j0 += ucls) {
            const CsUnit U{(u64)base, (u64)(base >> 64), lim, segsize, (u32)W, (u32)(base % W), ns, j0,
                           std::min(ucls, A - j0), D.bq.as<u32>()};
            for (;;) {
                MP_CUDA(h, D.l0.ensure(ucap * 8));
                MP_CUDA(h, D.l1.ensure(ucap * 8));
                const CsLists Ls{{D.l0.as<u64>(), D.l1.as<u64>()}, ucap, D.cnt.as<ull>()};
                int fin = 0;
                u32 fcnt = 0;
                cs_queue_unit(T, S, U, Ls, 3, h->sm_count, st, &fin, &fcnt);
                MP_CUDA(h, cudaGetLastError());
                ull raw = 0;
                MP_CUDA(h, cudaMemcpyAsync(&raw, D.cnt.p, sizeof raw, cudaMemcpyDeviceToHost, st));
                MP_CUDA(h, cudaStreamSynchronize(st));
                if (raw > ucap) { ucap = raw + raw / 4 + 65536; continue; }       // lists overflowed: again
                MP_TRY(collect(Ls.list[fin], D.cnt.as<ull>() + fcnt, ucap, base, raw / 8 + 1));
                break;
            }
        }
        if (done()) return MP_OK;
    }
    return MP_OK;
}

static bool cs_never() { return false; }

// verify a survivor list (offsets from base, count on the device) and append the chains
static int cs_collect(mp_handle *h, ChainDev &D, const u64 *list, const ull *nin, u64 cap, u128t base, u64 expect,
                      std::vector<u128t> &H, std::vector<u32> &L, cudaStream_t st)
{
    ull *nres = D.cnt.as<ull>() + CS_CNT_RES;
    MP_CUDA(h, D.rh.ensure(cap * 16));
    MP_CUDA(h, D.rl.ensure(cap * 4));
    MP_CUDA(h, cudaMemsetAsync(nres, 0, sizeof(ull), st));
    const u64 grid = std::max<u64>(1, std::min<u64>((expect + 127) / 128, (u64)h->sm_count * 16));
    // one-word arithmetic when every candidate, member and interloper of the list stays below
    // 2^64 - 2^12: a unit spans at most 256 segments of 2^17 W < 2^17 3e7 integers (below 2^50),
    // and members and extensions lie within 2^11 of their candidate
    if (base < ((u128t)1 << 64) - ((u128t)1 << 51))
        cs_verify64_kernel<<<(unsigned)grid, 128, 0, st>>>(list, nin, cap, (u64)base, D.k, D.mode, D.rh.as<u64>(),
                                                           D.rl.as<u32>(), nres);
    else
        cs_verify_kernel<<<(unsigned)grid, 128, 0, st>>>(list, nin, cap, (u64)base, (u64)(base >> 64), D.k, D.mode,
                                                         D.rh.as<u64>(), D.rl.as<u32>(), nres);
    MP_CUDA(h, cudaGetLastError());
    ull nr = 0;
    MP_CUDA(h, cudaMemcpyAsync(&nr, nres, sizeof nr, cudaMemcpyDeviceToHost, st));
    MP_CUDA(h, cudaStreamSynchronize(st));
    if (nr > cap) return mp_set_error(h, MP_EOVERFLOW, "chain sieve: more chains than survivors");
    if (nr) {
        std::vector<u64> w(2 * nr);
        const size_t o = H.size();
        L.resize(o + nr);
        MP_CUDA(h, cudaMemcpyAsync(w.data(), D.rh.p, nr * 16, cudaMemcpyDeviceToHost, st));
        MP_CUDA(h, cudaMemcpyAsync(L.data() + o, D.rl.p, nr * 4, cudaMemcpyDeviceToHost, st));
        MP_CUDA(h, cudaStreamSynchronize(st));
        H.resize(o + nr);
        for (size_t i = 0; i < nr; i++) H[o + i] = (u128t)w[2 * i + 1] << 64 | w[2 * i];
    }
    return MP_OK;
}

static const u128t CS_HI128_MAX = (u128t)MP_CHAIN128_HI_MAX_W1 << 64 | MP_CHAIN128_HI_MAX_W0;

// the chains with keys in [lo, hi), sorted by head; *H and *L receive them (the kept list when
// the previous call asked for the same range with too little room)
static int cs_chains(mp_handle *h, u128t lo, u128t hi, u32 k, u32 shape, std::vector<u128t> &H, std::vector<u32> &L)
{
    cudaStream_t st = h->stream;
    MP_TRY(cs_prepare(h, shape, chain_offsets(k, shape)));
    ChainDev &D = *h->chain;
    if (D.kept && D.kept_lo == lo && D.kept_hi == hi) {
        H.swap(D.kept_h);
        L.swap(D.kept_l);
        D.kept = false;
        return MP_OK;
    }
    D.kept = false;
    MP_TRY(cs_sieve_range(
        h, D, lo, hi, st,
        [&](const u64 *list, const ull *nin, u64 cap_, u128t base, u64 expect) {
            return cs_collect(h, D, list, nin, cap_, base, expect, H, L, st);
        },
        cs_never));
    sort_chains(H, L);
    return MP_OK;
}

// keep what did not fit for the next call with the same range
static void cs_keep(mp_handle *h, u128t lo, u128t hi, size_t cap, std::vector<u128t> &H, std::vector<u32> &L)
{
    if (cap >= H.size()) return;
    ChainDev &D = *h->chain;
    D.kept = true;
    D.kept_lo = lo;
    D.kept_hi = hi;
    D.kept_h.swap(H);
    D.kept_l.swap(L);
}

extern "C" int mp_chain_sieve(mp_handle *h, uint64_t lo, uint64_t hi, uint32_t k, uint32_t shape, uint64_t *heads,
                              uint32_t *lens, size_t cap, size_t *count)
{
    if (!h || !count || (cap && (!heads || !lens))) return MP_EINVAL;
    *count = 0;
    if (shape > 1) return mp_set_error(h, MP_EINVAL, "shape must be MP_CHAIN_INC or MP_CHAIN_DEC");
    if (k < (shape ? 4u : 2u) || k > CS_MAXLEN)
        return mp_set_error(h, MP_EINVAL, "k must be in %u..%d", shape ? 4u : 2u, CS_MAXLEN);
    if (hi > MP_CHAIN_SIEVE_HI_MAX) return mp_set_error(h, MP_ERANGE, "hi must be <= 2^64 - 2^12");
    if (hi <= lo) return MP_OK;
    if (shape == 0 && k < 4) return mp_gap_chains(h, lo, hi, k, heads, lens, cap, count);   // dense: enumerate
    std::lock_guard<std::recursive_mutex> lk(h->mu);
    MP_CUDA(h, cudaSetDevice(h->device));
    std::vector<u128t> H;
    std::vector<u32> L;
    MP_TRY(cs_chains(h, lo, hi, k, shape, H, L));
    const size_t m = std::min(cap, H.size());
    for (size_t i = 0; i < m; i++) { heads[i] = (u64)H[i]; lens[i] = L[i]; }
    *count = H.size();
    cs_keep(h, lo, hi, cap, H, L);
    return MP_OK;
}

extern "C" int mp_chain_sieve128(mp_handle *h, const uint64_t lo[2], const uint64_t hi[2], uint32_t k, uint32_t shape,
                                 uint64_t *heads, uint32_t *lens, size_t cap, size_t *count)
{
    if (!h || !lo || !hi || !count || (cap && (!heads || !lens))) return MP_EINVAL;
    *count = 0;
    if (shape > 1) return mp_set_error(h, MP_EINVAL, "shape must be MP_CHAIN_INC or MP_CHAIN_DEC");
    if (k < 4 || k > CS_MAXLEN) return mp_set_error(h, MP_EINVAL, "k must be in 4..%d", CS_MAXLEN);
    const u128t L0 = (u128t)lo[1] << 64 | lo[0], H0 = (u128t)hi[1] << 64 | hi[0];
    if (H0 > CS_HI128_MAX) return mp_set_error(h, MP_ERANGE, "hi must be <= 3.3e24");
    if (H0 <= L0) return MP_OK;
    std::lock_guard<std::recursive_mutex> lk(h->mu);
    MP_CUDA(h, cudaSetDevice(h->device));
    std::vector<u128t> H;
    std::vector<u32> L;
    MP_TRY(cs_chains(h, L0, H0, k, shape, H, L));
    const size_t m = std::min(cap, H.size());
    for (size_t i = 0; i < m; i++) { heads[2 * i] = (u64)H[i]; heads[2 * i + 1] = (u64)(H[i] >> 64); lens[i] = L[i]; }
    *count = H.size();
    cs_keep(h, L0, H0, cap, H, L);
    return MP_OK;
}

// the first chain: runs in ascending order, stopping after the first run that holds one; the
// smallest key wins (the head for gaps 2, 4, ...; for ..., 4, 2 the start of the k-prime
// pattern that ends the chain, member len - k of it)
static int cs_first(mp_handle *h, u128t lo, u128t hi, u32 k, u32 shape, u128t *key, u128t *head, u32 *len)
{
    cudaStream_t st = h->stream;
    MP_TRY(cs_prepare(h, shape, chain_offsets(k, shape)));
    ChainDev &D = *h->chain;
    D.kept = false;
    std::vector<u128t> H;
    std::vector<u32> L;
    MP_TRY(cs_sieve_range(
        h, D, lo, hi, st,
        [&](const u64 *list, const ull *nin, u64 cap_, u128t base, u64 expect) {
            return cs_collect(h, D, list, nin, cap_, base, expect, H, L, st);
        },
        [&]() { return !H.empty(); }));
    for (size_t i = 0; i < H.size(); i++) {
        const u64 j = L[i] - k;
        const u128t kk = shape == 0 ? H[i] : H[i] + (u128t)(j * (2 * (u64)L[i] - 1 - j));
        if (!*len || kk < *key) { *key = kk; *head = H[i]; *len = L[i]; }
    }
    return MP_OK;
}

extern "C" int mp_chain_first(mp_handle *h, uint64_t lo, uint64_t hi, uint32_t k, uint32_t shape, uint64_t *key,
                              uint64_t *head, uint32_t *len)
{
    if (!h || !key || !head || !len) return MP_EINVAL;
    *key = *head = 0;
    *len = 0;
    if (shape > 1) return mp_set_error(h, MP_EINVAL, "shape must be MP_CHAIN_INC or MP_CHAIN_DEC");
    if (k < 4 || k > CS_MAXLEN) return mp_set_error(h, MP_EINVAL, "k must be in 4..%d", CS_MAXLEN);
    if (hi > MP_CHAIN_SIEVE_HI_MAX) return mp_set_error(h, MP_ERANGE, "hi must be <= 2^64 - 2^12");
    if (hi <= lo) return MP_OK;
    std::lock_guard<std::recursive_mutex> lk(h->mu);
    MP_CUDA(h, cudaSetDevice(h->device));
    u128t K = 0, Hd = 0;
    MP_TRY(cs_first(h, lo, hi, k, shape, &K, &Hd, len));
    *key = (u64)K;
    *head = (u64)Hd;
    return MP_OK;
}

extern "C" int mp_chain_first128(mp_handle *h, const uint64_t lo[2], const uint64_t hi[2], uint32_t k, uint32_t shape,
                                 uint64_t key[2], uint64_t head[2], uint32_t *len)
{
    if (!h || !lo || !hi || !key || !head || !len) return MP_EINVAL;
    key[0] = key[1] = head[0] = head[1] = 0;
    *len = 0;
    if (shape > 1) return mp_set_error(h, MP_EINVAL, "shape must be MP_CHAIN_INC or MP_CHAIN_DEC");
    if (k < 4 || k > CS_MAXLEN) return mp_set_error(h, MP_EINVAL, "k must be in 4..%d", CS_MAXLEN);
    const u128t L0 = (u128t)lo[1] << 64 | lo[0], H0 = (u128t)hi[1] << 64 | hi[0];
    if (H0 > CS_HI128_MAX) return mp_set_error(h, MP_ERANGE, "hi must be <= 3.3e24");
    if (H0 <= L0) return MP_OK;
    std::lock_guard<std::recursive_mutex> lk(h->mu);
    MP_CUDA(h, cudaSetDevice(h->device));
    u128t K = 0, Hd = 0;
    MP_TRY(cs_first(h, L0, H0, k, shape, &K, &Hd, len));
    key[0] = (u64)K; key[1] = (u64)(K >> 64);
    head[0] = (u64)Hd; head[1] = (u64)(Hd >> 64);
    return MP_OK;
}

static int cs_tuple_check(mp_handle *h, const uint32_t *offs, uint32_t k)
{
    if (k < 2 || k > MP_TUPLE_MAXK) return mp_set_error(h, MP_EINVAL, "k must be in 2..%d", MP_TUPLE_MAXK);
    if (offs[0] != 0) return mp_set_error(h, MP_EINVAL, "offs[0] must be 0");
    for (u32 i = 1; i < k; i++)
        if (offs[i] <= offs[i - 1] || (offs[i] & 1) || offs[i] > MP_TUPLE_MAXOFF)
            return mp_set_error(h, MP_EINVAL, "offsets must be even and increasing, at most %d", MP_TUPLE_MAXOFF);
    return MP_OK;
}

static int cs_tuples(mp_handle *h, u128t lo, u128t hi, const uint32_t *offs, uint32_t k, uint64_t *count,
                     uint64_t *cks)
{
    cudaStream_t st = h->stream;
    MP_TRY(cs_prepare(h, CS_MODE_TUPLE, std::vector<u32>(offs, offs + k)));
    ChainDev &D = *h->chain;
    ull *acc = D.cnt.as<ull>() + CS_CNT_TUPLE;
    MP_CUDA(h, cudaMemsetAsync(acc, 0, 2 * sizeof(ull), st));
    MP_TRY(cs_sieve_range(
        h, D, lo, hi, st,
        [&](const u64 *list, const ull *nin, u64 cap_, u128t base, u64 expect) {
            const u64 grid = std::max<u64>(1, std::min<u64>((expect + 127) / 128, (u64)h->sm_count * 16));
            if (base < ((u128t)1 << 64) - ((u128t)1 << 51))          // every member below 2^64 - 2^12
                cs_tuple_kernel<<<(unsigned)grid, 128, 0, st>>>(list, nin, cap_, (u64)base, D.offs.as<u32>(), D.k,
                                                                acc);
            else
                cs_tuple128_kernel<<<(unsigned)grid, 128, 0, st>>>(list, nin, cap_, (u64)base, (u64)(base >> 64),
                                                                   D.offs.as<u32>(), D.k, acc);
            return cudaGetLastError() == cudaSuccess ? MP_OK : mp_set_error(h, MP_ECUDA, "tuple kernel launch failed");
        },
        cs_never));
    ull r[2] = {0, 0};
    MP_CUDA(h, cudaMemcpyAsync(r, acc, sizeof r, cudaMemcpyDeviceToHost, st));
    MP_CUDA(h, cudaStreamSynchronize(st));
    *count = r[0];
    *cks = r[1];
    return MP_OK;
}

extern "C" int mp_tuple_count(mp_handle *h, uint64_t lo, uint64_t hi, const uint32_t *offs, uint32_t k,
                              uint64_t *count, uint64_t *cks)
{
    if (!h || !offs || !count || !cks) return MP_EINVAL;
    *count = 0;
    *cks = 0;
    MP_TRY(cs_tuple_check(h, offs, k));
    if (hi > MP_CHAIN_SIEVE_HI_MAX) return mp_set_error(h, MP_ERANGE, "hi must be <= 2^64 - 2^12");
    if (hi <= lo) return MP_OK;
    std::lock_guard<std::recursive_mutex> lk(h->mu);
    MP_CUDA(h, cudaSetDevice(h->device));
    return cs_tuples(h, lo, hi, offs, k, count, cks);
}

extern "C" int mp_tuple_count128(mp_handle *h, const uint64_t lo[2], const uint64_t hi[2], const uint32_t *offs,
                                 uint32_t k, uint64_t *count, uint64_t *cks)
{
    if (!h || !lo || !hi || !offs || !count || !cks) return MP_EINVAL;
    *count = 0;
    *cks = 0;
    MP_TRY(cs_tuple_check(h, offs, k));
    const u128t L0 = (u128t)lo[1] << 64 | lo[0], H0 = (u128t)hi[1] << 64 | hi[0];
    if (H0 > CS_HI128_MAX) return mp_set_error(h, MP_ERANGE, "hi must be <= 3.3e24");
    if (H0 <= L0) return MP_OK;
    std::lock_guard<std::recursive_mutex> lk(h->mu);
    MP_CUDA(h, cudaSetDevice(h->device));
    return cs_tuples(h, L0, H0, offs, k, count, cks);
}

// ---- the cu_* interface of gapchain/gapsieve_cuda.h ----

namespace {

struct CuSlot {
    bool set = false, did[2] = {false, false};
    u32 unit = 0, cap = 0;
    DevBuf bq, list[2][2], cnt;
    u32 *h_bq = nullptr;                       // pinned staging, unit x nps
    ull *h_cnt = nullptr;                      // pinned: raw and final count per shape
    cudaEvent_t ev = nullptr;
    int fin[2] = {0, 0};
    std::vector<u64> host[2];
};

struct CuState {
    std::mutex mu;
    bool init = false;
    int sm = 0;
    cudaStream_t st = nullptr, cp = nullptr;   // the units' stream, the list copies' stream
    DevBuf ginfo, q, qinv, crt;
    u32 ngroups = 0, nps = 0;
    struct Shape {
        DevBuf pat, res, offs;
        u32 A = 0, k = 0;
        bool on = false;
    } sh[2];
    CuSlot slot[CU_MAXSLOT];
};

CuState &cu()
{
    static CuState s;
    return s;
}

int cu_lists(CuSlot &X, u32 cap)
{
    CuState &C = cu();
    for (int d = 0; d < 2; d++)
        for (int b = 0; b < 2; b++) {
            X.list[d][b].release();
            if (C.sh[d].on && X.list[d][b].ensure((size_t)cap * 8) != cudaSuccess) return -1;
        }
    X.cap = cap;
    return 0;
}

}  // namespace

extern "C" int cu_init(char *name, size_t n)
{
    CuState &C = cu();
    std::lock_guard<std::mutex> lk(C.mu);
    int nd = 0;
    if (cudaGetDeviceCount(&nd) != cudaSuccess || nd < 1) return -1;
    int dev = 0;
    cudaDeviceProp pr;
    if (cudaGetDevice(&dev) != cudaSuccess || cudaGetDeviceProperties(&pr, dev) != cudaSuccess) return -1;
    if (name && n) snprintf(name, n, "%s", pr.name);
    if (!C.init) {
        if (cudaStreamCreateWithFlags(&C.st, cudaStreamNonBlocking) != cudaSuccess) return -1;
        if (cudaStreamCreateWithFlags(&C.cp, cudaStreamNonBlocking) != cudaSuccess) return -1;
        C.sm = pr.multiProcessorCount;
        C.init = true;
    }
    return 0;
}

extern "C" int cu_tables(uint32_t ngroups, const uint32_t *ginfo, uint32_t nps, const uint32_t *q,
                         const uint32_t *qinv, const uint32_t *crt)
{
    CuState &C = cu();
    std::lock_guard<std::mutex> lk(C.mu);
    if (!C.init || !ngroups || ngroups > CS_MAXG || !nps || !ginfo || !q || !qinv || !crt) return -1;
    const std::vector<u32> gi(ginfo, ginfo + 4 * (size_t)ngroups), qq(q, q + nps), qi(qinv, qinv + nps),
        cr(crt, crt + nps);
    if (upload(C.ginfo, gi) || upload(C.q, qq) || upload(C.qinv, qi) || upload(C.crt, cr)) return -1;
    C.ngroups = ngroups;
    C.nps = nps;
    return 0;
}

extern "C" int cu_shape(int d, const uint32_t *pat, size_t npat, const uint32_t *res, uint32_t A,
                        const uint32_t *offs, uint32_t k)
{
    CuState &C = cu();
    std::lock_guard<std::mutex> lk(C.mu);
    if (!C.init || d < 0 || d > 1 || !pat || !npat || (npat & 1) || !res || !A || !offs || !k || k > CU_MAXK) return -1;
    auto &S = C.sh[d];
    const std::vector<u32> pv(pat, pat + npat), rv(res, res + A), ov(offs, offs + k);
    if (upload(S.pat, pv) || upload(S.res, rv) || upload(S.offs, ov)) return -1;
    S.A = A;
    S.k = k;
    S.on = true;
    return 0;
}

extern "C" int cu_slot(int slot, uint32_t unit, uint32_t cap)
{
    CuState &C = cu();
    std::lock_guard<std::mutex> lk(C.mu);
    if (!C.init || slot < 0 || slot >= CU_MAXSLOT || !unit || !cap || !C.nps) return -1;
    CuSlot &X = C.slot[slot];
    if (X.bq.ensure((size_t)unit * C.nps * 4) != cudaSuccess) return -1;
    if (X.cnt.ensure(2 * CS_NCNT * sizeof(ull)) != cudaSuccess) return -1;
    if (X.h_bq) { cudaFreeHost(X.h_bq); X.h_bq = nullptr; }
    if (!X.h_cnt && cudaMallocHost(&X.h_cnt, 4 * sizeof(ull)) != cudaSuccess) { X.h_cnt = nullptr; return -1; }
    if (cudaMallocHost(&X.h_bq, (size_t)unit * C.nps * 4) != cudaSuccess) { X.h_bq = nullptr; return -1; }
    if (!X.ev && cudaEventCreateWithFlags(&X.ev, cudaEventDisableTiming) != cudaSuccess) return -1;
    X.unit = unit;
    if (cu_lists(X, cap)) return -1;
    X.set = true;
    return 0;
}

extern "C" int cu_grow(int slot, uint32_t cap)
{
    CuState &C = cu();
    std::lock_guard<std::mutex> lk(C.mu);
    if (slot < 0 || slot >= CU_MAXSLOT || !C.slot[slot].set || !cap) return -1;
    return cu_lists(C.slot[slot], cap);
}

extern "C" int cu_submit(int slot, const uint32_t *bq, uint32_t nseg, uint32_t nps, const struct cu_params *p[2],
                         int split)
{
    CuState &C = cu();
    std::lock_guard<std::mutex> lk(C.mu);
    if (slot < 0 || slot >= CU_MAXSLOT || !bq || !p) return -1;
    CuSlot &X = C.slot[slot];
    if (!X.set || !nseg || nseg > X.unit || nps != C.nps) return -1;
    for (int d = 0; d < 2; d++) {
        const cu_params *q = p[d];
        if (!q) continue;
        const auto &S = C.sh[d];
        if (!S.on || q->k != S.k || q->A != S.A || q->nps != C.nps || q->ngroups != C.ngroups || q->nseg != nseg ||
            q->segsize != (u64)CS_K * q->W || q->bmodW >= q->W || q->cap > X.cap)
            return -1;
    }
    memcpy(X.h_bq, bq, (size_t)nseg * nps * 4);
    if (cudaMemcpyAsync(X.bq.p, X.h_bq, (size_t)nseg * nps * 4, cudaMemcpyHostToDevice, C.st) != cudaSuccess) return -1;
    const CsTables T{C.ginfo.as<u32>(), C.q.as<u32>(), C.qinv.as<u32>(), C.crt.as<u32>(), C.ngroups, C.nps};
    for (int d = 0; d < 2; d++) {
        X.did[d] = p[d] != nullptr;
        if (!p[d]) continue;
        const cu_params &q = *p[d];
        const auto &S0 = C.sh[d];
        const CsShape S{S0.pat.as<u64>(), S0.res.as<u32>(), S0.offs.as<u32>(), S0.A, S0.k};
        const CsUnit U{q.base_lo, q.base_hi, q.lim, q.segsize, q.W, q.bmodW, nseg, 0, S0.A, X.bq.as<u32>()};
        const CsLists L{{X.list[d][0].as<u64>(), X.list[d][1].as<u64>()}, X.cap, X.cnt.as<ull>() + d * CS_NCNT};
        u32 fcnt = 0;
        cs_queue_unit(T, S, U, L, split < 0 ? 0u : (u32)split, C.sm, C.st, &X.fin[d], &fcnt);
        cudaMemcpyAsync(X.h_cnt + 2 * d, L.cnt, sizeof(ull), cudaMemcpyDeviceToHost, C.st);
        cudaMemcpyAsync(X.h_cnt + 2 * d + 1, L.cnt + fcnt, sizeof(ull), cudaMemcpyDeviceToHost, C.st);
    }
    if (cudaEventRecord(X.ev, C.st) != cudaSuccess) return -1;
    return cudaPeekAtLastError() == cudaSuccess ? 0 : -1;
}

extern "C" int cu_wait(int slot, uint32_t stat[2], uint32_t nfin[2])
{
    CuState &C = cu();
    if (slot < 0 || slot >= CU_MAXSLOT || !C.slot[slot].set || !stat || !nfin) return -1;
    CuSlot &X = C.slot[slot];
    if (cudaEventSynchronize(X.ev) != cudaSuccess) return -1;
    std::lock_guard<std::mutex> lk(C.mu);
    for (int d = 0; d < 2; d++) {
        if (!X.did[d]) continue;
        const ull raw = X.h_cnt[2 * d], fin = X.h_cnt[2 * d + 1];
        stat[d] = (u32)std::min<ull>(raw, 0xffffffffull);
        nfin[d] = (u32)std::min<ull>(fin, X.cap);
    }
    return cudaGetLastError() == cudaSuccess ? 0 : -1;
}

extern "C" const uint64_t *cu_list(int slot, int d, uint32_t n)
{
    CuState &C = cu();
    std::lock_guard<std::mutex> lk(C.mu);
    if (slot < 0 || slot >= CU_MAXSLOT || d < 0 || d > 1) return nullptr;
    CuSlot &X = C.slot[slot];
    if (!X.set || !X.did[d] || n > X.cap) return nullptr;
    X.host[d].resize(std::max<u32>(n, 1));
    if (n && (cudaMemcpyAsync(X.host[d].data(), X.list[d][X.fin[d]].p, (size_t)n * 8, cudaMemcpyDeviceToHost, C.cp) !=
                  cudaSuccess ||
              cudaStreamSynchronize(C.cp) != cudaSuccess))
        return nullptr;
    return X.host[d].data();
}

__global__ void cu_sprp_kernel(const u64 *__restrict__ n, size_t count, u8 *ok)
{
    for (size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x; i < count; i += (size_t)gridDim.x * blockDim.x) {
        const u64 lo = n[2 * i], hi = n[2 * i + 1];
        bool r;
        if (!hi && lo < 3) r = lo == 2;
        else if (!(lo & 1)) r = false;
        else r = member_sprp2(lo, hi, 0, 0);
        ok[i] = r;
    }
}

extern "C" int cu_sprp_batch(const uint64_t *n, size_t count, uint8_t *ok)
{
    if (!count) return 0;
    if (!n || !ok) return -1;
    for (size_t i = 0; i < count; i++)
        if (n[2 * i + 1] >> 63) return -1;     // n >= 2^127
    CuState &C = cu();
    if (!C.init && cu_init(nullptr, 0)) return -1;
    DevBuf dn, dk;
    if (dn.ensure(count * 16) != cudaSuccess || dk.ensure(count) != cudaSuccess) return -1;
    int rc = 0;
    if (cudaMemcpyAsync(dn.p, n, count * 16, cudaMemcpyHostToDevice, C.cp) != cudaSuccess) rc = -1;
    if (!rc) {
        const unsigned grid = (unsigned)std::max<size_t>(1, std::min<size_t>((count + 255) / 256, (size_t)C.sm * 8));
        cu_sprp_kernel<<<grid, 256, 0, C.cp>>>(dn.as<u64>(), count, dk.as<u8>());
        if (cudaMemcpyAsync(ok, dk.p, count, cudaMemcpyDeviceToHost, C.cp) != cudaSuccess ||
            cudaStreamSynchronize(C.cp) != cudaSuccess)
            rc = -1;
    }
    dn.release();
    dk.release();
    return rc;
}
