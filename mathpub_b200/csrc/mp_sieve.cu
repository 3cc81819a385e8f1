// mp_sieve.cu -- the segmented odd-only sieve of Eratosthenes for B200 (sm_100a) and its
// scans: prime counts, twin pairs, 6-tuples {0,4,6,10,12,16}, maximal gaps, per-block
// statistics, per-segment FNV-1a hashes, the prime bitmap and prime lists.
//
// Reference behaviour (paths inside the Mathpub project): the odd-only layout and the
// start of marking at max(q^2, first odd multiple) follow scan_interval in
// A228768/a228768.c:372-415; small primes applied as periodic patterns follow
// pattern_setup/presieve in A350826/a350826.c:1192-1271; large primes filed by the segment
// of their next hit follow the bucket sieve of A007508/a007508.c:282-338,447-480; the gap
// belongs to the prime that starts it (A000230/a000230.c:12-16); twins and 6-tuples are
// counted by their first member (A007508/a007508.c:1-10, A350826/a350826.c:22-31) with the
// tuple checksum sum of mix64(p) (A350826/a350826.c:1364-1379).
//
// Layout on the device: bit i of the odd-only map stands for base + 2i + 1 (base = lo & ~1).
// The map is cut into tiles of 2^TLOG bits (TLOG = 18..20) that live in shared memory, each
// with a halo of 1024 bits sieved twice so that twins and 6-tuples that start in a tile are
// decided inside it.  Sieving primes are split into tiers by size:
//   3..89          five product patterns (periods 4849845, 765049, 4391633, 17120443,
//                  42600829 bits) ORed into the tile with 128-bit vector loads;
//   97..2047       one warp per prime, lanes on consecutive multiples, shared atomics;
//   2048..2^TLOG   one thread per prime, shared atomics;
//   > 2^TLOG       bucket records: a scatter kernel files the hit offsets of each prime
//                  for a wave of tiles; the tile kernel ORs them in.
// A tile summary (count, twins, tuples, checksum, first/last prime, widest internal gap)
// goes to HBM; a one-CTA fold kernel joins the summaries in order into block and range
// results, attributing every gap to the prime that starts it.
#include "mp_common.cuh"
#include <algorithm>
#include <math.h>
#include <stdarg.h>

#define HALO_WORDS 32u
#define HALO_BITS (HALO_WORDS * 32u)
// tier bounds: the warp tier takes 97 <= q < QWARP, the dense thread tier QWARP <= q < QDENSE
// (never above T / 32), the sparse thread tier the rest up to the bucket threshold.  Measured
// at config 2 (2^20-bit tiles): QWARP 4096 and QDENSE 8192 (T / 128) 5.95 ms of tile kernel,
// 2048 and T / 32 6.05 ms, 8192 and T / 32 6.10 ms, 2048 and T / 16 6.14 ms
#define QWARP 4096u
#define QDENSE 8192u
#define PAT_MAXQ 89u
#define MAX_TLOG 20

static const u32 kPatPrimes[MP_NPAT][7] = {
    {3, 5, 7, 11, 13, 17, 19}, {23, 29, 31, 37, 0}, {41, 43, 47, 53, 0}, {59, 61, 67, 71, 0}, {73, 79, 83, 89, 0}};
__constant__ u32 c_pat_primes[MP_NPAT][7] = {
    {3, 5, 7, 11, 13, 17, 19}, {23, 29, 31, 37, 0}, {41, 43, 47, 53, 0}, {59, 61, 67, 71, 0}, {73, 79, 83, 89, 0}};

struct TileSum {
    u64 first, last;   // first / last prime bit in the tile (bits < nbx); MP_NONE if none
    u64 lastin;        // last prime bit below limit; MP_NONE if none
    u64 mgs;           // bit of the prime starting the widest internal gap; MP_NONE if none
    u64 cks;           // sum of mix64(p) over the 6-tuple starts p (bits < limit)
    u32 mg;            // widest internal gap in bits (pairs whose first prime is in range)
    u32 count;         // primes with bit < limit
    u32 twins, tuples;
};

struct SieveGeom {
    u64 base, limit, nbx;   // base even; bits [0, limit) in range; bits [0, nbx) sieved
    u32 tlog, ntiles;
};

struct TileArgs {
    SieveGeom g;
    u32 t0, nt;                          // tiles [t0, t0 + nt) of this launch
    const u32 *q;
    const u64 *magic;
    u32 iw0, iw1, itd, it1;              // warp tier [iw0, iw1), thread tier [iw1, itd) dense, [itd, it1) sparse
    const u32 *pat[MP_NPAT];
    u32 period[MP_NPAT];
    const u32 *rec;                      // bucket records of tiles [t0, t0 + nt) (nullable)
    u32 *reccnt;
    u32 reccap;
    TileSum *sums;                       // by global tile index
    u32 *bitmap32;                       // nullable
    const u64 *emit_off;                 // emit mode: per-tile offset of its first prime
    u64 *emit64;
    u32 *emit32;
    u32 *tstate;                         // per CTA: next multiple of each sparse thread-tier prime
};

// the per-launch (or per-item) part of a wave: its first tile and tile count, and its bucket
// records and their counts; passed by value so that the argument structs stay in the
// kernel's parameter space
struct Wave {
    u32 t0, wt;
    u32 *rec, *cnt;
};

// state of a sparse thread-tier prime between the tiles of a CTA's run: (next bit relative to
// the next tile) << 3 | wheel index, or W30_NOSTATE (set it up from x0 again)
#define W30_NOSTATE 0xffffffffu
#define W30_FAR (1u << 28)

// ---------------------------------------------------------------------------------------
// ordered combine of tile / thread summaries
// ---------------------------------------------------------------------------------------

struct Part {
    u64 first, last, lastin, mgs, cks;
    u32 mg, count, twins, tuples;
};

__device__ __forceinline__ void part_init(Part &p)
{
    p.first = p.last = p.lastin = p.mgs = MP_NONE;
    p.cks = 0;
    p.mg = p.count = p.twins = p.tuples = 0;
}

// L followed by R (R's bits all above L's); gaps compare strictly so the earliest start wins
__device__ __forceinline__ Part part_join(const Part &L, const Part &R, u64 limit)
{
    Part o;
    o.count = L.count + R.count;
    o.twins = L.twins + R.twins;
    o.tuples = L.tuples + R.tuples;
    o.cks = L.cks + R.cks;
    o.mg = L.mg;
    o.mgs = L.mgs;
    if (L.first == MP_NONE) {
        o.first = R.first; o.last = R.last; o.lastin = R.lastin; o.mg = R.mg; o.mgs = R.mgs;
        return o;
    }
    o.first = L.first;
    if (R.first == MP_NONE) { o.last = L.last; o.lastin = L.lastin; return o; }
    o.last = R.last;
    o.lastin = R.lastin != MP_NONE ? R.lastin : L.lastin;
    if (L.last < limit) {
        const u32 g = (u32)(R.first - L.last);
        if (g > o.mg) { o.mg = g; o.mgs = L.last; }
    }
    if (R.mg > o.mg) { o.mg = R.mg; o.mgs = R.mgs; }
    return o;
}

__device__ __forceinline__ Part part_shfl_down(const Part &p, int d)
{
    Part o;
    o.first = __shfl_down_sync(0xffffffffu, p.first, d);
    o.last = __shfl_down_sync(0xffffffffu, p.last, d);
    o.lastin = __shfl_down_sync(0xffffffffu, p.lastin, d);
    o.mgs = __shfl_down_sync(0xffffffffu, p.mgs, d);
    o.cks = __shfl_down_sync(0xffffffffu, p.cks, d);
    o.mg = __shfl_down_sync(0xffffffffu, p.mg, d);
    o.count = __shfl_down_sync(0xffffffffu, p.count, d);
    o.twins = __shfl_down_sync(0xffffffffu, p.twins, d);
    o.tuples = __shfl_down_sync(0xffffffffu, p.tuples, d);
    return o;
}

// in-order reduction over the lanes of a warp; lane 0 holds the result
__device__ __forceinline__ Part part_warp_reduce(Part p, u64 limit)
{
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        Part r = part_shfl_down(p, d);
        if ((lane & (2 * d - 1)) == 0) p = part_join(p, r, limit);
    }
    return p;
}

// ---------------------------------------------------------------------------------------
// tile kernel
// ---------------------------------------------------------------------------------------

__device__ __forceinline__ u32 bits_mask(u64 start, u64 bound)
{
    // bits start .. start+31 below bound
    if (start >= bound) return 0;
    const u64 n = bound - start;
    return n >= 32 ? 0xffffffffu : ((1u << n) - 1);
}

// a 16-byte bucket-record load: streaming through L1 in a kernel of its own, through L2 only
// inside the pipeline kernel
__device__ __forceinline__ uint4 rec_ld(const uint4 *p, bool l2_only) { return l2_only ? __ldcg(p) : __ldcs(p); }

template <int TLOG>
__device__ __forceinline__ void presieve(u32 *sm, const TileArgs &a, const u32 *s_off)
{
    constexpr u32 NW = (1u << TLOG) / 32 + HALO_WORDS;
    const u32 tid = threadIdx.x, nth = blockDim.x;
    for (u32 w4 = tid * 4; w4 < NW; w4 += nth * 4) {
        u32 o0 = 0, o1 = 0, o2 = 0, o3 = 0;
        uint4 LO[MP_NPAT], HI[MP_NPAT];
#pragma unroll
        for (int p = 0; p < MP_NPAT; p++) {          // all loads first: ten in flight per thread
            const u32 a4 = ((s_off[p] >> 5) + w4) & ~3u;
            LO[p] = __ldg((const uint4 *)(a.pat[p] + a4));
            HI[p] = __ldg((const uint4 *)(a.pat[p] + a4 + 4));
        }
#pragma unroll
        for (int p = 0; p < MP_NPAT; p++) {
            const u32 bit = s_off[p] + w4 * 32;
            const u32 s = bit >> 5, sh = bit & 31;
            const uint4 lo = LO[p], hi = HI[p];
            u32 v0, v1, v2, v3, v4;
            switch (s & 3) {          // uniform across the CTA for a given tile and pattern
            case 0: v0 = lo.x; v1 = lo.y; v2 = lo.z; v3 = lo.w; v4 = hi.x; break;
            case 1: v0 = lo.y; v1 = lo.z; v2 = lo.w; v3 = hi.x; v4 = hi.y; break;
            case 2: v0 = lo.z; v1 = lo.w; v2 = hi.x; v3 = hi.y; v4 = hi.z; break;
            default: v0 = lo.w; v1 = hi.x; v2 = hi.y; v3 = hi.z; v4 = hi.w; break;
            }
            o0 |= __funnelshift_r(v0, v1, sh);
            o1 |= __funnelshift_r(v1, v2, sh);
            o2 |= __funnelshift_r(v2, v3, sh);
            o3 |= __funnelshift_r(v3, v4, sh);
        }
        *(uint4 *)&sm[w4] = make_uint4(o0, o1, o2, o3);
    }
}

// Tiles [rb, re) of wave W (relative to W.t0), in order, by the whole CTA, with the tile in
// shared memory `sm` (TW + HALO_WORDS words) and the carried state of the sparse thread-tier
// primes in `tst`.  EMIT = 0: statistics (+ optional bitmap); EMIT = 1: write the in-range
// primes.  PIPE: the tile runs inside the pipeline kernel, whose bucket records were written
// by other CTAs of the same launch: they are read through L2 (not L1, which may hold the
// lines of an earlier wave), and each tile's record count is reset once it is consumed, so
// that the ring slot is clean for the wave after next.
template <int TLOG, int EMIT, bool PIPE>
__device__ __forceinline__ void tile_run(const TileArgs &a, const Wave W, u32 rb, u32 re, u32 *tst, u32 *sm)
{
    constexpr u32 T = 1u << TLOG;
    constexpr u32 TW = T / 32;
    constexpr u32 NB = T + HALO_BITS;          // bits held in shared memory
    __shared__ u32 s_off[MP_NPAT];
    __shared__ Part s_part[32];
    __shared__ u32 s_cnt[32];

    const u32 tid = threadIdx.x, nth = blockDim.x, lane = tid & 31, warp = tid >> 5, nwarps = nth >> 5;
    const u64 base = a.g.base, limit = a.g.limit, nbx = a.g.nbx;

    for (u32 rel = rb; rel < re; rel++) {
        const bool fresh = rel == rb;                             // no carried state yet
        const bool keep = rel + 1 < re;                           // the next tile follows here
        const u32 t = W.t0 + rel;
        const u64 G = (u64)t << TLOG;           // first bit of the tile
        const u64 x0 = base + 2 * G + 1;        // the odd number of that bit
        if (tid < MP_NPAT) s_off[tid] = (u32)((base / 2 + G) % a.period[tid]);
        __syncthreads();

        // 1. small primes: patterns
        presieve<TLOG>(sm, a, s_off);
        __syncthreads();
        if (x0 <= PAT_MAXQ && tid == 0) {
            // the pattern primes themselves are prime; 1 is not
            for (int p = 0; p < MP_NPAT; p++)
                for (int k = 0; k < 7 && c_pat_primes[p][k]; k++) {
                    const u64 q = c_pat_primes[p][k];
                    if (q >= x0 && ((q - x0) >> 1) < NB) {
                        const u32 j = (u32)((q - x0) >> 1);
                        atomicAnd(&sm[j >> 5], ~(1u << (j & 31)));
                    }
                }
            if (x0 == 1) atomicOr(&sm[0], 1u);
        }

        // multiples q k with k coprime to 30 only (wheel of 30; the patterns hold 3 and 5)
        const u32 xm = (u32)(x0 % 30u);
        // 2. warp tier.  Warp w takes the primes w, w + nwarps, w + 2 nwarps, ... of the tier
        //    (equal shares of the marks), 32 at a time: lane i sets up prime i of the batch
        //    (first multiple and wheel index), then the warp marks the batch one prime after the
        //    other, lane l walking residue (l & 7) of the wheel in turn (l >> 3), four turns
        //    (60 q bits) per step.
        for (u32 kb = a.iw0 + warp; kb < a.iw1; kb += 32 * nwarps) {
            const u32 k = kb + nwarps * lane;
            u32 q = 0, jw = NB, w = 0;                         // jw >= NB: nothing to mark
            if (k < a.iw1) {
                q = __ldg(a.q + k);
                const u32 r = mp_mod_barrett(x0, q, __ldg(a.magic + k));
                const u64 j64 = mp_first_odd_multiple(x0, q, r, NB);
                if (j64 < NB) jw = (u32)mp_w30_first((u32)j64, xm, q, &w);
            }
            const u32 n = min(32u, (a.iw1 - kb + nwarps - 1) / nwarps);
            for (u32 i = 0; i < n; i++) {
                const u32 qi = __shfl_sync(0xffffffffu, q, i), ji = __shfl_sync(0xffffffffu, jw, i);
                const u32 wi = __shfl_sync(0xffffffffu, w, i);
                if (ji >= NB) continue;
                const u32 j0 = ji + qi * (mp_w30_span(mp_w30_steps(wi), lane & 7) + 15u * (lane >> 3));
                const u32 d = 60u * qi;
                u32 j = j0;
                for (; j + d < NB; j += 2 * d) {
                    atomicOr(&sm[j >> 5], __funnelshift_l(0u, 1u, j));
                    atomicOr(&sm[(j + d) >> 5], __funnelshift_l(0u, 1u, j + d));
                }
                if (j < NB) atomicOr(&sm[j >> 5], __funnelshift_l(0u, 1u, j));
            }
        }
        // 3. thread tier, one thread per prime.  Dense primes (q < QDENSE) have several
        //    multiples per residue of the wheel in a tile: set up from x0 in every tile and
        //    walked as 8 progressions of stride 15 q.
        for (u32 k = a.iw1 + tid; k < a.itd; k += nth) {
            const u32 q = __ldg(a.q + k);
            const u32 r = mp_mod_barrett(x0, q, __ldg(a.magic + k));
            const u64 j64 = mp_first_odd_multiple(x0, q, r, NB);
            if (j64 >= NB) continue;
            u32 w;
            u32 j = (u32)mp_w30_first((u32)j64, xm, q, &w);
            u32 s = mp_w30_steps(w);
            const u32 turn = 15u * q;
#pragma unroll
            for (int i = 0; i < 8; i++) {
                u32 jj = j;
                for (; jj + turn < NB; jj += 2 * turn) {
                    atomicOr(&sm[jj >> 5], __funnelshift_l(0u, 1u, jj));
                    atomicOr(&sm[(jj + turn) >> 5], __funnelshift_l(0u, 1u, jj + turn));
                }
                if (jj < NB) atomicOr(&sm[jj >> 5], __funnelshift_l(0u, 1u, jj));
                j += q * (s & 3u);
                s >>= 2;
            }
        }
        //    Sparse primes (QDENSE <= q <= T) have a few multiples per tile: one walk through
        //    the residues, with the next multiple carried to the CTA's next tile, so that the
        //    modular set-up runs once per run of tiles.  Eight primes per thread are loaded
        //    ahead.
        for (u32 k = a.itd + tid; k < a.it1; k += 8 * nth) {
            u32 qv[8], sv[8];
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const u32 kk = k + u * nth;
                qv[u] = kk < a.it1 ? __ldg(a.q + kk) : 0u;
                sv[u] = (kk < a.it1 && !fresh) ? tst[kk - a.itd] : W30_NOSTATE;
            }
#pragma unroll
            for (int u = 0; u < 8; u++) {
                const u32 q = qv[u];
                if (!q) continue;
                const u32 kk = k + u * nth;
                u32 j, w;
                if (sv[u] == W30_NOSTATE) {
                    const u32 r = mp_mod_barrett(x0, q, __ldg(a.magic + kk));
                    const u64 j64 = mp_first_odd_multiple(x0, q, r, W30_FAR);
                    if (j64 >= W30_FAR) {                      // q^2 far beyond this tile
                        if (keep) tst[kk - a.itd] = W30_NOSTATE;
                        continue;
                    }
                    j = (u32)mp_w30_first((u32)j64, xm, q, &w);
                } else {
                    j = sv[u] >> 3;
                    w = sv[u] & 7u;
                }
                u32 s = mp_w30_steps(w), n = 0;
                for (; j < T; j += q * (s & 3u), s = __funnelshift_r(s, s, 2), n++)
                    atomicOr(&sm[j >> 5], __funnelshift_l(0u, 1u, j));
                if (keep) tst[kk - a.itd] = ((j - T) << 3) | ((w + n) & 7u);
                for (; j < NB; j += q * (s & 3u), s = __funnelshift_r(s, s, 2))     // halo bits
                    atomicOr(&sm[j >> 5], __funnelshift_l(0u, 1u, j));
            }
        }
        // 4. large primes: bucket records of this tile.  Records and bitmap words are read or
        //    written once, with streaming cache hints, so that the prime table and the carried
        //    state of the sparse primes stay in L2.
        if (W.rec) {
            u32 n = PIPE ? __ldcg(W.cnt + rel) : __ldg(W.cnt + rel);
            if (n > a.reccap) n = a.reccap;
            const u32 *R = W.rec + (u64)rel * a.reccap;       // reccap is a multiple of 4
            const uint4 *R4 = (const uint4 *)R;
            const u32 n4 = n >> 2;
            u32 i = tid;
            for (; i + 3 * nth < n4; i += 4 * nth) {             // 16 records in flight per thread
                const uint4 r0 = rec_ld(R4 + i, PIPE), r1 = rec_ld(R4 + i + nth, PIPE);
                const uint4 r2 = rec_ld(R4 + i + 2 * nth, PIPE), r3 = rec_ld(R4 + i + 3 * nth, PIPE);
                const u32 js[16] = {r0.x, r0.y, r0.z, r0.w, r1.x, r1.y, r1.z, r1.w,
                                    r2.x, r2.y, r2.z, r2.w, r3.x, r3.y, r3.z, r3.w};
#pragma unroll
                for (int k = 0; k < 16; k++) atomicOr(&sm[js[k] >> 5], 1u << (js[k] & 31));
            }
            for (; i < n4; i += nth) {
                const uint4 r0 = rec_ld(R4 + i, PIPE);
                atomicOr(&sm[r0.x >> 5], __funnelshift_l(0u, 1u, r0.x));
                atomicOr(&sm[r0.y >> 5], __funnelshift_l(0u, 1u, r0.y));
                atomicOr(&sm[r0.z >> 5], __funnelshift_l(0u, 1u, r0.z));
                atomicOr(&sm[r0.w >> 5], __funnelshift_l(0u, 1u, r0.w));
            }
            for (u32 k = (n4 << 2) + tid; k < n; k += nth) {
                const u32 j = PIPE ? __ldcg(R + k) : __ldcs(R + k);
                atomicOr(&sm[j >> 5], __funnelshift_l(0u, 1u, j));
            }
        }
        __syncthreads();
        if (PIPE && W.rec && tid == 0) W.cnt[rel] = 0;            // every thread has read it

        // 5. scans
        if (!EMIT) {
            // Warp w scans words [w * wpw, (w + 1) * wpw) in rows of 128 words; in a row, lane l
            // holds words 4l .. 4l + 3 (one 16-byte load, no bank conflicts).  Positions are
            // bits relative to the tile.  The prime before a lane's first prime is the last
            // prime of an earlier lane of the row (a max-scan) or of an earlier row (carry).
            const u32 wpw = TW / nwarps;
            const u32 wbase = warp * wpw;
            const u32 NONE32 = 0xffffffffu;
            u32 cnt = 0, tw = 0, tu = 0;
            u64 cks = 0;
            u32 first = NONE32, last = NONE32, lastin = NONE32, bg = 0, bs = NONE32, carry = NONE32;
            const u64 lim_rel = limit > G ? limit - G : 0;         // bits of the tile below limit
            const u64 nbx_rel = nbx > G ? nbx - G : 0;
            u32 thr = 0;                                             // the warp's widest gap so far
            for (u32 r = 0; r < wpw; r += 128) {
                const u32 w = wbase + r + 4 * lane;
                const uint4 v = *(const uint4 *)&sm[w];
                u32 p[5];
                p[0] = ~v.x; p[1] = ~v.y; p[2] = ~v.z; p[3] = ~v.w;
                u32 nx = __shfl_down_sync(0xffffffffu, p[0], 1);
                if (lane == 31) nx = ~sm[w + 4];
                p[4] = nx;
                const u32 b0 = w * 32;
                if ((u64)b0 + 160 > nbx_rel) {
#pragma unroll
                    for (int k = 0; k < 5; k++) p[k] &= bits_mask((u64)b0 + 32 * k, nbx_rel);
                }
                u32 lm[4] = {~0u, ~0u, ~0u, ~0u};
                if ((u64)b0 + 128 > lim_rel) {
#pragma unroll
                    for (int k = 0; k < 4; k++) lm[k] = bits_mask((u64)b0 + 32 * k, lim_rel);
                }
                u32 lf = NONE32, ll = NONE32;
#pragma unroll
                for (int k = 0; k < 4; k++) {
                    const u32 pk = p[k], pin = pk & lm[k];
                    cnt += __popc(pin);
                    tw += __popc(pin & __funnelshift_r(pk, p[k + 1], 1));
                    u32 tup = pin & __funnelshift_r(pk, p[k + 1], 2) & __funnelshift_r(pk, p[k + 1], 3) &
                              __funnelshift_r(pk, p[k + 1], 5) & __funnelshift_r(pk, p[k + 1], 6) &
                              __funnelshift_r(pk, p[k + 1], 8);
                    if (tup) {
                        tu += __popc(tup);
                        while (tup) {
                            const u32 b = __ffs(tup) - 1;
                            tup &= tup - 1;
                            cks += mp_mix64(base + 2 * (G + b0 + 32 * k + b) + 1);
                        }
                    }
                    if (pin) lastin = b0 + 32 * k + 31 - __clz(pin);
                }
                // gaps inside the lane's 128 bits.  While the warp's widest gap is below 32
                // bits every prime is walked.  From 32 bits on, a gap inside one 32-bit word
                // can neither beat nor tie it, so only the gaps from the last prime of a word
                // to the first prime of a later one are taken (thr is the same in every lane).
                if (thr < 32) {
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        u32 y = p[k];
                        while (y) {
                            const u32 pos = b0 + 32 * k + __ffs(y) - 1;
                            y &= y - 1;
                            if (ll == NONE32) lf = pos;
                            else if ((u64)ll < lim_rel) {
                                const u32 g = pos - ll;
                                if (g > bg || (g == bg && ll < bs)) { bg = g; bs = ll; }
                            }
                            ll = pos;
                        }
                    }
                } else {
#pragma unroll
                    for (int k = 0; k < 4; k++) {
                        const u32 pk = p[k];
                        if (pk) {
                            const u32 f = b0 + 32 * k + __ffs(pk) - 1;
                            if (ll == NONE32) lf = f;
                            else if ((u64)ll < lim_rel) {
                                const u32 g = f - ll;
                                if (g > bg || (g == bg && ll < bs)) { bg = g; bs = ll; }
                            }
                            ll = b0 + 32 * k + 31 - __clz(pk);
                        }
                    }
                }
                // last prime before this lane's first: inclusive max-scan of (last + 1)
                u32 sc = ll == NONE32 ? 0u : ll + 1;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const u32 u = __shfl_up_sync(0xffffffffu, sc, d);
                    if (lane >= (u32)d && u > sc) sc = u;
                }
                u32 ex = __shfl_up_sync(0xffffffffu, sc, 1);
                if (lane == 0) ex = 0;
                const u32 prev = ex ? ex - 1 : carry;
                if (lf != NONE32 && prev != NONE32 && (u64)prev < lim_rel) {
                    const u32 g = lf - prev;
                    if (g > bg || (g == bg && prev < bs)) { bg = g; bs = prev; }
                }
                const u32 rowlast = __shfl_sync(0xffffffffu, sc, 31);
                if (rowlast) carry = rowlast - 1;
                thr = bg;
#pragma unroll
                for (int d = 16; d >= 1; d >>= 1) thr = max(thr, __shfl_xor_sync(0xffffffffu, thr, d));
                if (first == NONE32 && lf != NONE32) first = lf;
                if (ll != NONE32) last = ll;
            }
            // warp reduction (sums, min first, max last / lastin, widest gap with the smallest
            // start), then the warps join in order
#pragma unroll
            for (int d = 16; d >= 1; d >>= 1) {
                cnt += __shfl_xor_sync(0xffffffffu, cnt, d);
                tw += __shfl_xor_sync(0xffffffffu, tw, d);
                tu += __shfl_xor_sync(0xffffffffu, tu, d);
                cks += __shfl_xor_sync(0xffffffffu, cks, d);
                first = min(first, __shfl_xor_sync(0xffffffffu, first, d));
                const u32 ol = __shfl_xor_sync(0xffffffffu, last, d);
                last = (last == NONE32) ? ol : (ol == NONE32 ? last : max(last, ol));
                const u32 oi = __shfl_xor_sync(0xffffffffu, lastin, d);
                lastin = (lastin == NONE32) ? oi : (oi == NONE32 ? lastin : max(lastin, oi));
                const u32 og = __shfl_xor_sync(0xffffffffu, bg, d), os = __shfl_xor_sync(0xffffffffu, bs, d);
                if (og > bg || (og == bg && os < bs)) { bg = og; bs = os; }
            }
            if (lane == 0) {
                Part P;
                P.count = cnt; P.twins = tw; P.tuples = tu; P.cks = cks;
                P.first = first == NONE32 ? MP_NONE : G + first;
                P.last = last == NONE32 ? MP_NONE : G + last;
                P.lastin = lastin == NONE32 ? MP_NONE : G + lastin;
                P.mg = bs == NONE32 ? 0 : bg;
                P.mgs = bs == NONE32 ? MP_NONE : G + bs;
                s_part[warp] = P;
            }
            __syncthreads();
            if (warp == 0) {
                Part Q;
                if (lane < nwarps) Q = s_part[lane];
                else part_init(Q);
                Q = part_warp_reduce(Q, limit);
                if (lane == 0) {
                    TileSum S;
                    S.first = Q.first; S.last = Q.last; S.lastin = Q.lastin; S.mgs = Q.mgs; S.cks = Q.cks;
                    S.mg = Q.mg; S.count = Q.count; S.twins = Q.twins; S.tuples = Q.tuples;
                    a.sums[t] = S;
                }
            }
            if (a.bitmap32) {
                // in-range prime words, up to the next multiple of 64 bits
                const u64 lim64 = (limit + 63) & ~63ull;
                for (u32 w = tid; w < TW; w += nth) {
                    const u64 bit0 = G + 32ull * w;
                    if (bit0 >= lim64) break;
                    __stcs(a.bitmap32 + (G >> 5) + w, ~sm[w] & bits_mask(bit0, limit));
                }
            }
        } else {
            // emit: in-range primes in order; thread `tid` owns words [w0, w0 + wpt); per-thread
            // counts, then a CTA-wide scan
            const u32 wpt = TW / nth;
            const u32 w0 = tid * wpt;
            u32 c = 0;
            for (u32 w = w0; w < w0 + wpt; w++) c += __popc(~sm[w] & bits_mask(G + 32ull * w, limit));
            u32 incl = c;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const u32 v = __shfl_up_sync(0xffffffffu, incl, d);
                if (lane >= (u32)d) incl += v;
            }
            if (lane == 31) s_cnt[warp] = incl;
            __syncthreads();
            if (warp == 0) {
                u32 v = lane < nwarps ? s_cnt[lane] : 0, iv = v;
#pragma unroll
                for (int d = 1; d < 32; d <<= 1) {
                    const u32 u = __shfl_up_sync(0xffffffffu, iv, d);
                    if (lane >= (u32)d) iv += u;
                }
                if (lane < nwarps) s_cnt[lane] = iv - v;   // exclusive warp offsets
            }
            __syncthreads();
            u64 pos = a.emit_off[t] + s_cnt[warp] + (incl - c);
            for (u32 w = w0; w < w0 + wpt; w++) {
                const u64 bit0 = G + 32ull * w;
                u32 y = ~sm[w] & bits_mask(bit0, limit);
                while (y) {
                    const u32 b = __ffs(y) - 1;
                    y &= y - 1;
                    const u64 p = base + 2 * (bit0 + b) + 1;
                    if (a.emit64) a.emit64[pos] = p;
                    else a.emit32[pos] = (u32)p;
                    pos++;
                }
            }
        }
        __syncthreads();
    }
}

// CTA b sieves the contiguous run of tiles [b per, (b + 1) per) of the launch, so that the
// sparse thread-tier primes carry their next multiple from one tile to the next
template <int TLOG, int EMIT>
__global__ void __launch_bounds__(1024) tile_kernel(TileArgs a)
{
    extern __shared__ __align__(16) u32 sm[];  // TW + HALO_WORDS words
    const u32 per = (a.nt + gridDim.x - 1) / gridDim.x;
    const u32 rb = blockIdx.x * per;
    const u32 re = min(rb + per, a.nt);
    const Wave W = {a.t0, a.nt, (u32 *)a.rec, a.reccnt};
    if (rb < re) tile_run<TLOG, EMIT, false>(a, W, rb, re, a.tstate + (u64)blockIdx.x * (a.it1 - a.itd), sm);
}

// ---------------------------------------------------------------------------------------
// bucket scatter for primes > 2^TLOG
// ---------------------------------------------------------------------------------------

struct ScatterArgs {
    u64 base;
    u32 tlog, t0, wt;                // wave = tiles [t0, t0 + wt)
    u64 nbx;
    const u32 *q;
    const u64 *magic;
    const u32 *bounds;               // CTA b takes primes [bounds[b], bounds[b + 1])
    u32 *rec;                        // [wt][cap]
    u32 *cnt;                        // [wt], zeroed before the launch
    u32 cap;
    u32 *err;
};

// Every hit j of a large prime q in the wave (plus the first HALO_BITS bits after it) is a
// record (tile, offset) of its own tile, and also (tile - 1, offset + 2^TLOG) when it lies in
// the first HALO_BITS bits of a tile, because the previous tile sieves those bits as its halo.
// The staged scatter's hits are the multiples q k with k coprime to 210 (the wheel of 210, below:
// 48 progressions of stride 105 q, walked eight at a time); the binned scatter's are those with k
// coprime to 30 (the wheel of 30: 8 progressions of stride 15 q).
//
// One pass, staged in shared memory: each persistent CTA owns a run of primes of equal sum
// of 1/q (equal expected hits); every thread walks one prime at a time, one turn of the wheel
// (8 hits) per round, and appends the records to the CTA's stage with one shared atomic per
// warp.  When the stage is nearly full the CTA sorts it by tile (counting sort), reserves one
// run per tile in the bucket with one global atomic, and writes the runs out, so that the
// record stores of a warp are coalesced.  Halo copies (one hit in 1024) go to the bucket
// directly.  Measured on B200 at 1e15 (2^34 integers): stage 8192 with three CTAs per SM
// 4.36 ms, 12288 with two 4.58 ms, 24576 with one 6.4 ms (5.0 ms with 1024 threads).

#ifndef SC_THREADS
#define SC_THREADS 512
#endif
#ifndef SC_STAGE
#define SC_STAGE 8192                     // staged records per CTA (two buffers of them)
#endif
#ifndef SC_CTAS_PER_SM
#define SC_CTAS_PER_SM 3                  // 48 warps per SM: the walk is latency-bound
#endif
#define SC_OFF_BITS 21                    // staged record: tile << 21 | offset (offset < 2^21)

// set up prime k: the 8 progression starts (ascending, below j + 15 q) relative to the wave;
// returns false when the prime has no hit in the wave
__device__ __forceinline__ bool scatter_setup(const ScatterArgs &a, u32 k, u64 x0, u32 xm, u32 span, u32 *jj,
                                              u32 &turn)
{
    const u32 q = __ldg(a.q + k);
    const u32 r = mp_mod_barrett(x0, q, __ldg(a.magic + k));
    const u64 j64 = mp_first_odd_multiple(x0, q, r, span);
    if (j64 >= span) return false;
    u32 w;
    u64 j = mp_w30_first((u32)j64, xm, q, &w);
    u32 s = mp_w30_steps(w);
    // span < 2^31: a stride of 2^31 or more leaves one hit per progression at most, so the
    // stride is clamped there and the positions stay below 2^32
    const u64 turn64 = 15ull * q;
    turn = turn64 >= (1ull << 31) ? (1u << 31) : (u32)turn64;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        jj[i] = j < span ? (u32)j : span;
        j += (u64)q * (s & 3u);
        s >>= 2;
    }
    return jj[0] < span;
}

// The staged scatter walks the wheel of 210: a bucket prime q marks only the q k with k coprime
// to 210, the multiples of 7 among the wheel-30 hits being marked by the presieve patterns
// already (1/7 of the records fewer).  The 48 residues of k mod 210 (all odd) give 48
// progressions of stride 105 q bits; a thread walks them eight at a time, as six groups.
// c_w210_off[t] = (R[t mod 48] + 210 (t div 48) - 1) / 2 for the residues R in increasing
// order, so the progression m places from residue index w lies q (off[w + m] - off[w]) bits on;
// for an odd k mod 210, c_w210_nidx / c_w210_ndist give the index of the first residue at or
// above it and the distance to it in q bits; c_w210_inv[q mod 210] = q^-1 mod 210.
__constant__ u8 c_w210_off[96] = {
    0, 5, 6, 8, 9, 11, 14, 15, 18, 20, 21, 23, 26, 29, 30, 33, 35, 36, 39, 41, 44, 48, 50, 51,
    53, 54, 56, 60, 63, 65, 68, 69, 71, 74, 75, 78, 81, 83, 84, 86, 89, 90, 93, 95, 96, 98, 99, 104,
    105, 110, 111, 113, 114, 116, 119, 120, 123, 125, 126, 128, 131, 134, 135, 138, 140, 141, 144, 146, 149, 153, 155, 156,
    158, 159, 161, 165, 168, 170, 173, 174, 176, 179, 180, 183, 186, 188, 189, 191, 194, 195, 198, 200, 201, 203, 204, 209,
};
__constant__ u8 c_w210_nidx[210] = {
    0, 0, 0, 1, 0, 1, 0, 1, 0, 1, 0, 1, 0, 2, 0, 3, 0, 3, 0, 4, 0, 5, 0, 5,
    0, 6, 0, 6, 0, 6, 0, 7, 0, 8, 0, 8, 0, 8, 0, 9, 0, 9, 0, 10, 0, 11, 0, 11,
    0, 12, 0, 12, 0, 12, 0, 13, 0, 13, 0, 13, 0, 14, 0, 15, 0, 15, 0, 15, 0, 16, 0, 16,
    0, 17, 0, 18, 0, 18, 0, 18, 0, 19, 0, 19, 0, 20, 0, 20, 0, 20, 0, 21, 0, 21, 0, 21,
    0, 21, 0, 22, 0, 22, 0, 23, 0, 24, 0, 24, 0, 25, 0, 26, 0, 26, 0, 27, 0, 27, 0, 27,
    0, 27, 0, 28, 0, 28, 0, 28, 0, 29, 0, 29, 0, 30, 0, 30, 0, 30, 0, 31, 0, 32, 0, 32,
    0, 33, 0, 33, 0, 33, 0, 34, 0, 35, 0, 35, 0, 35, 0, 36, 0, 36, 0, 36, 0, 37, 0, 37,
    0, 38, 0, 39, 0, 39, 0, 40, 0, 40, 0, 40, 0, 41, 0, 42, 0, 42, 0, 42, 0, 43, 0, 43,
    0, 44, 0, 45, 0, 45, 0, 46, 0, 47, 0, 47, 0, 47, 0, 47, 0, 47,
};
__constant__ u8 c_w210_ndist[210] = {
    0, 0, 0, 4, 0, 3, 0, 2, 0, 1, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 1, 0, 0,
    0, 2, 0, 1, 0, 0, 0, 0, 0, 2, 0, 1, 0, 0, 0, 1, 0, 0, 0, 0, 0, 1, 0, 0,
    0, 2, 0, 1, 0, 0, 0, 2, 0, 1, 0, 0, 0, 0, 0, 2, 0, 1, 0, 0, 0, 1, 0, 0,
    0, 0, 0, 2, 0, 1, 0, 0, 0, 1, 0, 0, 0, 2, 0, 1, 0, 0, 0, 3, 0, 2, 0, 1,
    0, 0, 0, 1, 0, 0, 0, 0, 0, 1, 0, 0, 0, 0, 0, 1, 0, 0, 0, 3, 0, 2, 0, 1,
    0, 0, 0, 2, 0, 1, 0, 0, 0, 1, 0, 0, 0, 2, 0, 1, 0, 0, 0, 0, 0, 1, 0, 0,
    0, 2, 0, 1, 0, 0, 0, 0, 0, 2, 0, 1, 0, 0, 0, 2, 0, 1, 0, 0, 0, 1, 0, 0,
    0, 0, 0, 1, 0, 0, 0, 2, 0, 1, 0, 0, 0, 0, 0, 2, 0, 1, 0, 0, 0, 1, 0, 0,
    0, 0, 0, 1, 0, 0, 0, 0, 0, 4, 0, 3, 0, 2, 0, 1, 0, 0,
};
__constant__ u8 c_w210_inv[210] = {
    0, 1, 0, 0, 0, 0, 0, 0, 0, 0, 0, 191, 0, 97, 0, 0, 0, 173, 0, 199, 0, 0, 0, 137,
    0, 0, 0, 0, 0, 29, 0, 61, 0, 0, 0, 0, 0, 193, 0, 0, 0, 41, 0, 127, 0, 0, 0, 143,
    0, 0, 0, 0, 0, 107, 0, 0, 0, 0, 0, 89, 0, 31, 0, 0, 0, 0, 0, 163, 0, 0, 0, 71,
    0, 187, 0, 0, 0, 0, 0, 109, 0, 0, 0, 167, 0, 0, 0, 0, 0, 59, 0, 0, 0, 0, 0, 0,
    0, 13, 0, 0, 0, 131, 0, 157, 0, 0, 0, 53, 0, 79, 0, 0, 0, 197, 0, 0, 0, 0, 0, 0,
    0, 151, 0, 0, 0, 0, 0, 43, 0, 0, 0, 101, 0, 0, 0, 0, 0, 23, 0, 139, 0, 0, 0, 47,
    0, 0, 0, 0, 0, 179, 0, 121, 0, 0, 0, 0, 0, 103, 0, 0, 0, 0, 0, 67, 0, 0, 0, 83,
    0, 169, 0, 0, 0, 17, 0, 0, 0, 0, 0, 149, 0, 181, 0, 0, 0, 0, 0, 73, 0, 0, 0, 11,
    0, 37, 0, 0, 0, 113, 0, 19, 0, 0, 0, 0, 0, 0, 0, 0, 0, 209,
};

struct W210 {                                    // the tables, staged in shared memory per CTA
    u8 off[96], nidx[210], ndist[210], inv[210];
};

__device__ __forceinline__ void w210_load(W210 &t)
{
    for (u32 i = threadIdx.x; i < 210; i += blockDim.x) {
        if (i < 96) t.off[i] = c_w210_off[i];
        t.nidx[i] = c_w210_nidx[i];
        t.ndist[i] = c_w210_ndist[i];
        t.inv[i] = c_w210_inv[i];
    }
}

// prime k over the wave: the bit jf of its first hit (a multiple q k' >= max(x0, q^2) with k'
// coprime to 210) and the residue index w of k'; false when the wave has none.  xm = x0 mod 210
__device__ __forceinline__ bool w210_prime(const ScatterArgs &a, const W210 &t, u32 k, u64 x0, u32 xm, u32 span,
                                           u32 &q, u32 &jf, u32 &w)
{
    q = __ldg(a.q + k);
    const u32 r = mp_mod_barrett(x0, q, __ldg(a.magic + k));
    const u64 j64 = mp_first_odd_multiple(x0, q, r, span);
    if (j64 >= span) return false;
    const u32 km = (xm + 2u * (u32)(j64 % 105u)) % 210u * t.inv[q % 210u] % 210u;   // k mod 210
    w = t.nidx[km];
    const u64 j = j64 + (u64)q * t.ndist[km];
    if (j >= span) return false;
    jf = (u32)j;
    return true;
}

// group g (0..5) of the prime: the starts of its eight progressions, ascending, below the
// first one + 105 q (or span when past the wave's end); false when the group has no hit
__device__ __forceinline__ bool w210_group(const W210 &t, u32 q, u32 jf, u32 w, u32 g, u32 span, u32 *jj)
{
    const u32 b = t.off[w];
#pragma unroll
    for (int i = 0; i < 8; i++) {
        const u64 j = jf + (u64)q * (u32)(t.off[w + 8 * g + i] - b);
        jj[i] = j < span ? (u32)j : span;
    }
    return jj[0] < span;
}

// sort the staged records by tile and write them to their buckets (all threads)
__device__ __forceinline__ void scatter_flush(const ScatterArgs &a, u32 *stage, u32 *sorted, u32 *hist, u32 *gb,
                                           u32 *s_fill, u32 *s_wsum)
{
    const u32 tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, wt = a.wt;
    __syncthreads();
    const u32 n = *s_fill;
    // exclusive scan of the tile counts; thread t owns tiles [t per, (t + 1) per)
    const u32 per = (wt + SC_THREADS - 1) / SC_THREADS;
    const u32 t0 = tid * per;
    u32 sum = 0;
    for (u32 t = t0; t < t0 + per && t < wt; t++) sum += hist[t];
    u32 incl = sum;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const u32 v = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= (u32)d) incl += v;
    }
    if (lane == 31) s_wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const u32 v = lane < SC_THREADS / 32 ? s_wsum[lane] : 0u;
        u32 iv = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const u32 u = __shfl_up_sync(0xffffffffu, iv, d);
            if (lane >= (u32)d) iv += u;
        }
        if (lane < SC_THREADS / 32) s_wsum[lane] = iv - v;
    }
    __syncthreads();
    // reserve each tile's run in its bucket; hist becomes the placement cursor and gb the
    // bucket slot of sorted index 0 of that run (mod 2^32)
    u32 start = s_wsum[warp] + incl - sum;
    for (u32 t = t0; t < t0 + per && t < wt; t++) {
        const u32 c = hist[t];
        if (c) {
            const u32 g = atomicAdd(a.cnt + t, c);
            if (g + c > a.cap) atomicOr(a.err, 2u);
            gb[t] = g - start;
        }
        hist[t] = start;
        start += c;
    }
    __syncthreads();
    for (u32 i = tid; i < n; i += SC_THREADS) {
        const u32 r = stage[i];
        sorted[atomicAdd(&hist[r >> SC_OFF_BITS], 1u)] = r;
    }
    __syncthreads();
    // the runs of one tile are consecutive in sorted order and in the bucket
    for (u32 i = tid; i < n; i += SC_THREADS) {
        const u32 r = sorted[i], tl = r >> SC_OFF_BITS, slot = gb[tl] + i;
        if (slot < a.cap) __stcs(a.rec + (u64)tl * a.cap + slot, r & ((1u << SC_OFF_BITS) - 1u));
    }
    __syncthreads();
    for (u32 t = tid; t < wt; t += SC_THREADS) hist[t] = 0;
    if (tid == 0) *s_fill = 0;
    __syncthreads();
}

__global__ void __launch_bounds__(SC_THREADS, SC_CTAS_PER_SM) scatter_kernel(ScatterArgs a)
{
    extern __shared__ __align__(16) u32 ssm[];
    u32 *stage = ssm, *sorted = ssm + SC_STAGE, *hist = ssm + 2 * SC_STAGE, *gb = hist + a.wt;
    __shared__ u32 s_fill;
    __shared__ u32 s_wsum[SC_THREADS / 32];
    __shared__ W210 s_w210;
    const u32 tid = threadIdx.x, lane = tid & 31, wt = a.wt, tlog = a.tlog, tmask = (1u << tlog) - 1;
    for (u32 i = tid; i < wt; i += SC_THREADS) hist[i] = 0;
    if (tid == 0) s_fill = 0;
    w210_load(s_w210);
    const u64 wstart = (u64)a.t0 << tlog;
    u64 wend = (u64)(a.t0 + wt) << tlog;
    if (wend > a.nbx) wend = a.nbx;
    u64 wend_halo = wend + HALO_BITS;
    if (wend_halo > a.nbx) wend_halo = a.nbx;
    const u64 x0 = a.base + 2 * wstart + 1;
    const u32 xm = (u32)(x0 % 210u);
    const u32 span = (u32)(wend_halo - wstart);          // < 2^31 (checked by the planner)
    const u32 k1 = __ldg(a.bounds + blockIdx.x + 1);
    u32 k = __ldg(a.bounds + blockIdx.x) + tid;
    // the thread's prime q, its first hit jf and residue index w, and the group g of its eight
    // progressions being walked (5: no group left)
    u32 jj[8], turn = 0, q = 0, jf = 0, w = 0, g = 5;
    bool have = false;
    __syncthreads();
    for (;;) {
        while (!have) {
            if (g < 5) {
                // the next group; groups start further on one after the other, so a group with no
                // hit ends the prime
                have = w210_group(s_w210, q, jf, w, ++g, span, jj);
                if (!have) g = 5;
            } else if (k < k1) {
                if (w210_prime(a, s_w210, k, x0, xm, span, q, jf, w)) {
                    // span < 2^31: a stride of 2^31 or more leaves one hit per progression at
                    // most, so it is clamped there and the positions stay below 2^32
                    const u64 turn64 = 105ull * q;
                    turn = turn64 >= (1ull << 31) ? (1u << 31) : (u32)turn64;
                    g = 0;
                    have = w210_group(s_w210, q, jf, w, 0, span, jj);
                    if (!have) g = 5;
                }
                k += SC_THREADS;
            } else {
                break;
            }
        }
        if (!__syncthreads_or(have)) break;                // the last round's appends are done
        // every thread takes the fill before any thread appends again, so the flush decision
        // (and the barriers inside the flush) is the same in every thread
        const u32 fill = s_fill;
        __syncthreads();
        if (fill > SC_STAGE - 8 * SC_THREADS)
            scatter_flush(a, stage, sorted, hist, gb, &s_fill, s_wsum);
        // one turn of the wheel: up to 8 records
        u32 rec[8], nmine = 0;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            const bool v = have && jj[i] < span;
            const u32 tl = jj[i] >> tlog, off = jj[i] & tmask;
            const bool own = v && tl < wt;
            rec[i] = own ? (tl << SC_OFF_BITS) | off : 0xffffffffu;
            nmine += own;
            if (v && off < HALO_BITS && tl >= 1 && tl - 1 < wt) {     // halo copy for tile tl - 1
                const u32 slot = atomicAdd(a.cnt + tl - 1, 1u);
                if (slot < a.cap) __stcs(a.rec + (u64)(tl - 1) * a.cap + slot, off + (1u << tlog));
                else atomicOr(a.err, 2u);
            }
            jj[i] = v ? jj[i] + turn : span;
        }
        have = have && jj[0] < span;
        // warp-aggregated append to the stage
        u32 incl = nmine;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const u32 u = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= (u32)d) incl += u;
        }
        u32 base = 0;
        if (lane == 31) base = atomicAdd(&s_fill, incl);
        base = __shfl_sync(0xffffffffu, base, 31);
        u32 pos = base + incl - nmine;
#pragma unroll
        for (int i = 0; i < 8; i++) {
            if (rec[i] != 0xffffffffu) {
                stage[pos++] = rec[i];
                atomicAdd(&hist[rec[i] >> SC_OFF_BITS], 1u);
            }
        }
    }
    scatter_flush(a, stage, sorted, hist, gb, &s_fill, s_wsum);
}

// The binned form of the same scatter: one CTA of SB_THREADS threads per SM, whose shared
// memory holds a bin of `binc` records per tile of the wave.  A record goes straight into its
// tile's bin (one shared atomic for the slot), so no sort is needed: every SB_FLUSH_ROUNDS
// rounds (the same round in every thread, so the decision is uniform) each warp writes whole
// bins of its tiles as coalesced runs, with one global atomic per tile to reserve the run in
// the bucket.  A record that finds its bin full goes to an overflow list, and past that
// straight to its bucket with a global atomic of its own; results are exact either way.
// Measured on B200 at 1e15 (2^34 integers) it is about 6x slower than the staged form: in a
// round the CTA's threads walk primes of about the same size from the start of the wave, so
// their hits crowd into the same few dozen tiles, whose bins overflow at once and send most
// records down the overflow path.  The staged form sorts whatever arrives and is the default.
#define SB_THREADS 1024
#define SB_OVF 1024
#define SB_FLUSH_ROUNDS 4

__device__ __forceinline__ void sb_direct(const ScatterArgs &a, const Wave &W, u32 tl, u32 off)
{
    const u32 slot = atomicAdd(W.cnt + tl, 1u);
    if (slot < a.cap) __stcs(W.rec + (u64)tl * a.cap + slot, off);
    else atomicOr(a.err, 2u);
}

__device__ __forceinline__ void sb_flush(const ScatterArgs &a, const Wave &W, const u32 *bin, u32 *cnt, const u32 *ovf,
                                         u32 *s_novf, u32 binc)
{
    const u32 tid = threadIdx.x, lane = tid & 31, warp = tid >> 5, nwarps = blockDim.x >> 5, wt = W.wt;
    // warp w: tiles w * 32 + l for its lanes l, then every 32 * nwarps; lane l reserves the
    // run of tile l of the group, then the warp writes the group's runs one after the other
    for (u32 t0 = warp * 32; t0 < wt; t0 += 32 * nwarps) {
        const u32 t = t0 + lane;
        const u32 n = t < wt ? min(cnt[t], binc) : 0u;
        u32 g = 0;
        if (n) {
            g = atomicAdd(W.cnt + t, n);
            if (g + n > a.cap) atomicOr(a.err, 2u);
        }
        u32 m = __ballot_sync(0xffffffffu, n != 0);
        while (m) {
            const u32 l = __ffs(m) - 1;
            m &= m - 1;
            const u32 nl = __shfl_sync(0xffffffffu, n, l), gl = __shfl_sync(0xffffffffu, g, l);
            const u32 *b = bin + (t0 + l) * binc;
            u32 *dst = W.rec + (u64)(t0 + l) * a.cap;
            for (u32 i = lane; i < nl; i += 32)
                if (gl + i < a.cap) __stcs(dst + gl + i, b[i]);
        }
    }
    const u32 no = min(*s_novf, (u32)SB_OVF);
    for (u32 i = tid; i < no; i += blockDim.x)
        sb_direct(a, W, ovf[i] >> SC_OFF_BITS, ovf[i] & ((1u << SC_OFF_BITS) - 1u));
    __syncthreads();
    for (u32 t = tid; t < wt; t += blockDim.x) cnt[t] = 0;
    if (tid == 0) *s_novf = 0;
    __syncthreads();
}

// the large primes [k_begin, k_end) of the table over wave W, by the whole CTA, with the bins
// in shared memory `ssm` (W.wt * binc + W.wt + SB_OVF words)
__device__ __forceinline__ void scatter_binned_run(const ScatterArgs &a, const Wave W, u32 k_begin, u32 k_end, u32 binc,
                                                   u32 *ssm)
{
    const u32 wt = W.wt;
    u32 *bin = ssm, *cnt = ssm + wt * binc, *ovf = cnt + wt;
    __shared__ u32 s_novf;
    const u32 tid = threadIdx.x, nth = blockDim.x, tlog = a.tlog, tmask = (1u << tlog) - 1;
    for (u32 i = tid; i < wt; i += nth) cnt[i] = 0;
    if (tid == 0) s_novf = 0;
    const u64 wstart = (u64)W.t0 << tlog;
    u64 wend = (u64)(W.t0 + wt) << tlog;
    if (wend > a.nbx) wend = a.nbx;
    u64 wend_halo = wend + HALO_BITS;
    if (wend_halo > a.nbx) wend_halo = a.nbx;
    const u64 x0 = a.base + 2 * wstart + 1;
    const u32 xm = (u32)(x0 % 30u);
    const u32 span = (u32)(wend_halo - wstart);          // < 2^31 (checked by the planner)
    u32 k = k_begin + tid;
    u32 jj[8], turn = 0;
    bool have = false;
    __syncthreads();
    for (u32 round = 1;; round++) {
        while (!have && k < k_end) {
            have = scatter_setup(a, k, x0, xm, span, jj, turn);
            k += nth;
        }
        if (have) {
            // one turn of the wheel: up to 8 records, each into its tile's bin
#pragma unroll
            for (int i = 0; i < 8; i++) {
                const u32 j = jj[i];
                if (j < span) {
                    const u32 tl = j >> tlog, off = j & tmask;
                    if (tl < wt) {
                        const u32 slot = atomicAdd(&cnt[tl], 1u);
                        if (slot < binc) bin[tl * binc + slot] = off;
                        else {
                            const u32 o = atomicAdd(&s_novf, 1u);
                            if (o < SB_OVF) ovf[o] = (tl << SC_OFF_BITS) | off;
                            else sb_direct(a, W, tl, off);
                        }
                    }
                    if (off < HALO_BITS && tl >= 1 && tl - 1 < wt) sb_direct(a, W, tl - 1, off + (1u << tlog));
                    jj[i] = j + turn;
                }
            }
            have = jj[0] < span;
        }
        // every append of the round is done; the loop goes on while any thread holds a prime
        // or still has primes to set up (a large prime often ends within one turn, so `have`
        // alone would end the loop with primes left)
        const int more = __syncthreads_or(have || k < k_end);
        if (!more) break;
        if (round % SB_FLUSH_ROUNDS == 0) sb_flush(a, W, bin, cnt, ovf, &s_novf, binc);
    }
    sb_flush(a, W, bin, cnt, ovf, &s_novf, binc);
}

__global__ void __launch_bounds__(SB_THREADS, 1) scatter_binned_kernel(ScatterArgs a, u32 binc)
{
    extern __shared__ __align__(16) u32 ssm[];
    const Wave W = {a.t0, a.wt, a.rec, a.cnt};
    scatter_binned_run(a, W, __ldg(a.bounds + blockIdx.x), __ldg(a.bounds + blockIdx.x + 1), binc, ssm);
}

// ---------------------------------------------------------------------------------------
// the pipeline: every wave of a range in one persistent launch
//
// Work items, numbered in the order the device queue hands them out:
//   S(0) ... S(1) T(0) ... S(2) T(1) ... S(W-1) T(W-2) ... T(W-1)
// S(w, r) is the binned scatter of the large primes [bounds[r], bounds[r+1]) over wave w;
// T(w, r) sieves tiles [r run, (r+1) run) of wave w.  The records of wave w live in ring slot
// w & 1.  T(w, .) waits until every S(w, .) has finished; S(w, .) for w >= 2 waits until
// every T(w-2, .) has finished with the slot (each tile item resets the record counts it has
// consumed, so the slot is clean).  A CTA only ever waits for items that the queue handed out
// before its own, to CTAs that are running them, so the waits always end; each is still
// bounded, and on running out it sets bit 8 of the error flag (the call then fails).
// Scatter items of the next wave run beside the tile items of this one on other SMs, and no
// kernel boundary separates the waves.
// ---------------------------------------------------------------------------------------

struct PipeArgs {
    TileArgs ta;                 // geometry, tiers, patterns and outputs
    ScatterArgs sa;              // scatter parameters
    u32 nwaves, wt, ntiles;      // waves of wt tiles, the last one holding the rest of ntiles
    u32 nscat, run, binc;        // scatter items per wave, tiles per tile item, records per bin
    u32 *rec[2], *cnt[2];        // the record ring
    u32 *ctl;                    // [0] next item, [1 + w] S(w) done, [1 + nwaves + w] T(w) done
    u32 spin_limit;              // polls of a wait before it gives up
};

__device__ __forceinline__ u32 pipe_wave_tiles(const PipeArgs &p, u32 w)
{
    return w + 1 < p.nwaves ? p.wt : p.ntiles - w * p.wt;
}
__device__ __forceinline__ u32 pipe_titems(const PipeArgs &p, u32 w) { return (pipe_wave_tiles(p, w) + p.run - 1) / p.run; }

__device__ __forceinline__ u32 pipe_total(const PipeArgs &p)
{
    const u32 tf = (p.wt + p.run - 1) / p.run;
    return p.nscat + (p.nwaves - 1) * (p.nscat + tf) + pipe_titems(p, p.nwaves - 1);
}

// item i -> kind (0 scatter, 1 tiles), wave, index within the wave's items of that kind
__device__ __forceinline__ void pipe_decode(const PipeArgs &p, u32 i, u32 &kind, u32 &w, u32 &r)
{
    if (i < p.nscat) { kind = 0; w = 0; r = i; return; }
    const u32 tf = (p.wt + p.run - 1) / p.run, B = p.nscat + tf, j = i - p.nscat, b = j / B;
    if (b < p.nwaves - 1) {
        const u32 q = j - b * B;
        if (q < p.nscat) { kind = 0; w = b + 1; r = q; }
        else { kind = 1; w = b; r = q - p.nscat; }
    } else {
        kind = 1; w = p.nwaves - 1; r = j - (p.nwaves - 1) * B;
    }
}

// thread 0 polls *flag until it reaches need (bounded), then the CTA goes on together
__device__ __forceinline__ void pipe_wait(const PipeArgs &p, const u32 *flag, u32 need)
{
    if (threadIdx.x == 0) {
        u32 polls = 0;
        while (*(volatile const u32 *)flag < need) {
            if (++polls > p.spin_limit) { atomicOr(p.sa.err, 8u); break; }
            __nanosleep(256);
        }
        __threadfence();
    }
    __syncthreads();
}

// every thread's writes of the item are made visible, then thread 0 counts the item done
__device__ __forceinline__ void pipe_signal(u32 *flag)
{
    __threadfence();
    __syncthreads();
    if (threadIdx.x == 0) atomicAdd(flag, 1u);
}

template <int TLOG>
__global__ void __launch_bounds__(1024, 1) sieve_pipeline_kernel(PipeArgs p)
{
    extern __shared__ __align__(16) u32 dyn[];
    __shared__ u32 s_item;
    const u32 total = pipe_total(p);
    u32 *const sdone = p.ctl + 1, *const tdone = p.ctl + 1 + p.nwaves;
    u32 *const tst = p.ta.tstate + (u64)blockIdx.x * (p.ta.it1 - p.ta.itd);
    for (;;) {
        if (threadIdx.x == 0) s_item = atomicAdd(p.ctl, 1u);
        __syncthreads();
        const u32 it = s_item;
        __syncthreads();                                   // s_item is read before it is reused
        if (it >= total) break;
        u32 kind, w, r;
        pipe_decode(p, it, kind, w, r);
        const Wave W = {w * p.wt, pipe_wave_tiles(p, w), p.rec[w & 1], p.cnt[w & 1]};
        if (kind == 0) {
            if (w >= 2) pipe_wait(p, tdone + (w - 2), pipe_titems(p, w - 2));
            scatter_binned_run(p.sa, W, __ldg(p.sa.bounds + r), __ldg(p.sa.bounds + r + 1), p.binc, dyn);
            pipe_signal(sdone + w);
        } else {
            pipe_wait(p, sdone + w, p.nscat);
            const u32 rb = r * p.run, re = min(rb + p.run, W.wt);
            tile_run<TLOG, 0, true>(p.ta, W, rb, re, tst, dyn);
            pipe_signal(tdone + w);
        }
    }
}

// ---------------------------------------------------------------------------------------
// fold: tile summaries -> block and range results
// ---------------------------------------------------------------------------------------

struct FoldArgs {
    u64 base, limit, lo, hi;
    const TileSum *sums;
    u32 ntiles, tpb;                 // tiles per block
    u32 nblocks, nblocks_ext;        // blocks in range / over all tiles
    Part *acc;                       // scratch [nblocks_ext]
    mp_range_stats *out;
    mp_block_stats *blocks;          // nullable
    u32 *err;
    int has2;
};

__device__ __forceinline__ Part tile_part(const TileSum &S)
{
    Part p;
    p.first = S.first; p.last = S.last; p.lastin = S.lastin; p.mgs = S.mgs; p.cks = S.cks;
    p.mg = S.mg; p.count = S.count; p.twins = S.twins; p.tuples = S.tuples;
    return p;
}

__device__ __forceinline__ void stats_from_part(mp_range_stats &o, const Part &p, u64 base, u64 limit, u64 nprimes_u64)
{
    o.pi = nprimes_u64;
    o.twins = p.twins;
    o.tuple6 = p.tuples;
    o.tuple6_cks = p.cks;
    o.max_gap = p.mgs == MP_NONE ? 0 : 2ull * p.mg;
    o.gap_start = p.mgs == MP_NONE ? 0 : base + 2 * p.mgs + 1;
    o.first_prime = (p.first == MP_NONE || p.first >= limit) ? 0 : base + 2 * p.first + 1;
    o.last_prime = p.lastin == MP_NONE ? 0 : base + 2 * p.lastin + 1;
}

struct RangeAcc {
    u64 n, tw, tu, cks, first, lastin, mgs;
    u32 mg;
};

__device__ __forceinline__ void racc_init(RangeAcc &r)
{
    r.n = r.tw = r.tu = r.cks = 0;
    r.first = r.lastin = r.mgs = MP_NONE;
    r.mg = 0;
}

// append block part B (bits above everything in r)
__device__ __forceinline__ void racc_add(RangeAcc &r, const Part &B)
{
    r.n += B.count; r.tw += B.twins; r.tu += B.tuples; r.cks += B.cks;
    if (r.first == MP_NONE) r.first = B.first;
    if (B.lastin != MP_NONE) r.lastin = B.lastin;
    if (B.mgs != MP_NONE && (r.mgs == MP_NONE || B.mg > r.mg)) { r.mg = B.mg; r.mgs = B.mgs; }
}

__device__ __forceinline__ void racc_join(RangeAcc &r, const RangeAcc &B)
{
    r.n += B.n; r.tw += B.tw; r.tu += B.tu; r.cks += B.cks;
    if (r.first == MP_NONE) r.first = B.first;
    if (B.lastin != MP_NONE) r.lastin = B.lastin;
    if (B.mgs != MP_NONE && (r.mgs == MP_NONE || B.mg > r.mg)) { r.mg = B.mg; r.mgs = B.mgs; }
}

// 64-bit totals: block parts carry u32 counts (a block is at most 2^31 bits); the range
// total is summed in 64 bits
__global__ void __launch_bounds__(512) fold_kernel(FoldArgs a)
{
    const u32 tid = threadIdx.x, nth = blockDim.x;
    // 1. blocks (over all tiles, including the tail)
    for (u32 b = tid; b < a.nblocks_ext; b += nth) {
        Part P;
        part_init(P);
        const u32 t0 = b * a.tpb;
        u32 t1 = t0 + a.tpb;
        if (t1 > a.ntiles) t1 = a.ntiles;
        for (u32 t = t0; t < t1; t++) P = part_join(P, tile_part(a.sums[t]), a.limit);
        a.acc[b] = P;
    }
    __syncthreads();
    // 2. trailing gap of each in-range block: from its last prime to the first prime of a
    //    later block
    for (u32 b = tid; b < a.nblocks; b += nth) {
        Part P = a.acc[b];
        if (P.last != MP_NONE && P.last < a.limit) {
            u64 nf = MP_NONE;
            for (u32 c = b + 1; c < a.nblocks_ext; c++) {
                const u64 f = a.acc[c].first;
                if (f != MP_NONE) { nf = f; break; }
            }
            if (nf == MP_NONE) atomicOr(a.err, 4u);
            else {
                const u32 g = (u32)(nf - P.last);
                if (g > P.mg) { a.acc[b].mg = g; a.acc[b].mgs = P.last; }
            }
        }
    }
    __syncthreads();
    // 3. block outputs (prime 2 joins the block that holds it)
    if (a.blocks) {
        for (u32 b = tid; b < a.nblocks; b += nth) {
            const Part P = a.acc[b];
            mp_range_stats o;
            stats_from_part(o, P, a.base, a.limit, P.count);
            if (a.has2 && b == 0) {
                o.pi += 1;
                o.first_prime = 2;
                if (P.lastin == MP_NONE) o.last_prime = 2;
                if (o.max_gap <= 1) { o.max_gap = 1; o.gap_start = 2; }
            }
            a.blocks[b] = o;
        }
    }
    // 4. range: in-order join of the in-range blocks, whose parts already hold their
    //    trailing gaps (each thread a contiguous run of blocks, then thread 0 in order)
    __shared__ RangeAcc s_r[512];
    {
        const u32 per = (a.nblocks + nth - 1) / nth;
        RangeAcc R;
        racc_init(R);
        for (u32 b = tid * per; b < (tid + 1) * per && b < a.nblocks; b++) racc_add(R, a.acc[b]);
        s_r[tid] = R;
    }
    __syncthreads();
    if (tid == 0) {
        RangeAcc R;
        racc_init(R);
        for (u32 i = 0; i < nth; i++) racc_join(R, s_r[i]);
        mp_range_stats o;
        o.pi = R.n;
        o.twins = R.tw;
        o.tuple6 = R.tu;
        o.tuple6_cks = R.cks;
        o.max_gap = R.mgs == MP_NONE ? 0 : 2ull * R.mg;
        o.gap_start = R.mgs == MP_NONE ? 0 : a.base + 2 * R.mgs + 1;
        o.first_prime = (R.first == MP_NONE || R.first >= a.limit) ? 0 : a.base + 2 * R.first + 1;
        o.last_prime = R.lastin == MP_NONE ? 0 : a.base + 2 * R.lastin + 1;
        if (a.has2) {
            o.pi += 1;
            o.first_prime = 2;
            if (R.lastin == MP_NONE) o.last_prime = 2;
            if (o.max_gap <= 1) { o.max_gap = 1; o.gap_start = 2; }
        }
        *a.out = o;
    }
}

// ---------------------------------------------------------------------------------------
// FNV-1a-64 per hash segment of the bitmap.  The hash is a serial chain over the segment's
// bytes, so each thread hashes one segment; one warp per CTA spreads the segments over every
// SM.  Each thread keeps HASH_AHEAD 16-byte loads (256 bytes) in flight ahead of its chain,
// which otherwise waits on every load.
// ---------------------------------------------------------------------------------------

#define HASH_AHEAD 16

__device__ __forceinline__ void fnv_word(u64 &h, u32 w)
{
#pragma unroll
    for (int j = 0; j < 4; j++) { h ^= (w >> (8 * j)) & 0xffu; h *= MP_FNV_PRIME; }
}

__device__ __forceinline__ void fnv_16(u64 &h, const uint4 v)
{
    fnv_word(h, v.x); fnv_word(h, v.y); fnv_word(h, v.z); fnv_word(h, v.w);
}

__global__ void __launch_bounds__(32) hash_kernel(const u32 *__restrict__ bm, u64 nbits, u64 seg_bits, u64 nseg,
                                                  u64 *out)
{
    const u64 s = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (s >= nseg) return;
    const u64 b0 = s * seg_bits;
    const u64 len = b0 + seg_bits <= nbits ? seg_bits : nbits - b0;
    const u64 nbytes = (len + 7) >> 3;
    const u8 *p = (const u8 *)bm + (b0 >> 3);       // seg_bits is a multiple of 8
    u64 h = MP_FNV_OFFSET;
    u64 k = 0;
    // bytes up to a 16-byte boundary (all but the last byte of the segment are whole)
    for (; k + 1 < nbytes && (((uintptr_t)(p + k)) & 15); k++) { h ^= p[k]; h *= MP_FNV_PRIME; }
    // whole blocks of HASH_AHEAD 16-byte words: the loads of block b + 1 are issued while
    // block b is hashed
    const u64 nblk = nbytes > k + 1 ? (nbytes - k - 1) / (16 * HASH_AHEAD) : 0;
    if (nblk) {
        const uint4 *v = (const uint4 *)(p + k);
        uint4 buf[HASH_AHEAD];
#pragma unroll
        for (int i = 0; i < HASH_AHEAD; i++) buf[i] = __ldcs(v + i);
        for (u64 b = 0; b < nblk; b++) {
            const uint4 *nx = v + (b + 1) * HASH_AHEAD;
            const bool more = b + 1 < nblk;
#pragma unroll
            for (int i = 0; i < HASH_AHEAD; i++) {
                const uint4 x = buf[i];
                if (more) buf[i] = __ldcs(nx + i);
                fnv_16(h, x);
            }
        }
        k += nblk * 16 * HASH_AHEAD;
    }
    // the rest in 16-byte words while one byte more remains, then bytes; the last byte keeps
    // only the bits of the segment
    for (; k + 16 < nbytes; k += 16) fnv_16(h, __ldcs((const uint4 *)(p + k)));
    for (; k < nbytes; k++) {
        u8 c = p[k];
        const u64 rem = len - 8 * k;
        if (rem < 8) c &= (u8)((1u << rem) - 1);
        h ^= c; h *= MP_FNV_PRIME;
    }
    out[s] = h;
}

// exclusive prefix of tile counts -> emit offsets; total to *total (one CTA)
__global__ void __launch_bounds__(1024) tile_scan_kernel(const TileSum *sums, u32 ntiles, u64 *off, u64 *total)
{
    __shared__ u64 s[1024];
    const u32 tid = threadIdx.x, nth = blockDim.x;
    const u32 per = (ntiles + nth - 1) / nth;
    u64 c = 0;
    for (u32 t = tid * per; t < (tid + 1) * per && t < ntiles; t++) c += sums[t].count;
    s[tid] = c;
    __syncthreads();
    if (tid == 0) {
        u64 acc = 0;
        for (u32 i = 0; i < nth; i++) { const u64 v = s[i]; s[i] = acc; acc += v; }
        *total = acc;
    }
    __syncthreads();
    u64 acc = s[tid];
    for (u32 t = tid * per; t < (tid + 1) * per && t < ntiles; t++) { off[t] = acc; acc += sums[t].count; }
}

// ---------------------------------------------------------------------------------------
// tables: bootstrap primes, big table, Barrett constants, patterns
// ---------------------------------------------------------------------------------------

// odd primes below 2^16, in one CTA: sieve of Eratosthenes over the odd numbers, then an
// ordered compaction
__global__ void __launch_bounds__(1024) boot_primes_kernel(u32 *out, u32 *count)
{
    __shared__ u8 comp[32768];      // odd j: 2j + 1 < 65536
    __shared__ u32 s_cnt[1024];
    const u32 tid = threadIdx.x, nth = blockDim.x;
    for (u32 j = tid; j < 32768; j += nth) comp[j] = 0;
    __syncthreads();
    comp[0] = 1;   // 1
    for (u32 q = 3; q * q < 65536; q += 2) {
        __syncthreads();
        if (comp[q >> 1]) continue;             // uniform: every thread reads the same byte
        for (u32 m = q * q + 2 * q * tid; m < 65536; m += 2 * q * nth) comp[m >> 1] = 1;
    }
    __syncthreads();
    const u32 per = 32768 / nth;
    u32 c = 0;
    for (u32 j = tid * per; j < (tid + 1) * per; j++) c += !comp[j];
    s_cnt[tid] = c;
    __syncthreads();
    if (tid == 0) {
        u32 acc = 0;
        for (u32 i = 0; i < nth; i++) { const u32 v = s_cnt[i]; s_cnt[i] = acc; acc += v; }
        *count = acc;
    }
    __syncthreads();
    u32 pos = s_cnt[tid];
    for (u32 j = tid * per; j < (tid + 1) * per; j++)
        if (!comp[j]) out[pos++] = 2 * j + 1;
}

__global__ void magic_kernel(const u32 *q, u64 n, u64 *magic)
{
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x)
        magic[i] = ~0ull / q[i];
}

// pattern p: bit j set iff 2j + 1 is divisible by one of the pattern's primes
__global__ void pattern_kernel(u32 *w, u64 nwords, u32 q0, u32 q1, u32 q2, u32 q3, u32 q4, u32 q5, u32 q6)
{
    const u32 qs[7] = {q0, q1, q2, q3, q4, q5, q6};
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < nwords; i += (u64)gridDim.x * blockDim.x) {
        u32 v = 0;
        for (u32 b = 0; b < 32; b++) {
            const u64 x = 2 * (32 * i + b) + 1;
            for (int k = 0; k < 7; k++)
                if (qs[k] && x % qs[k] == 0) { v |= 1u << b; break; }
        }
        w[i] = v;
    }
}

u64 PrimeTable::count_le(u64 x) const
{
    return (u64)(std::upper_bound(host.begin(), host.end(), (u32)(x > 0xffffffffull ? 0xffffffffull : x)) - host.begin());
}

int mp_patterns_ensure(mp_handle *h)
{
    if (h->pat_ready) return MP_OK;
    const u64 slack_bits = (1ull << MAX_TLOG) + HALO_BITS + 8 * 32 + 256;
    for (int p = 0; p < MP_NPAT; p++) {
        u64 per = 1;
        for (int k = 0; k < 7 && kPatPrimes[p][k]; k++) per *= kPatPrimes[p][k];
        h->pat.period[p] = (u32)per;
        const u64 words = (per + slack_bits) / 32 + 16;
        h->pat.words[p] = words;
        MP_CUDA(h, cudaMalloc(&h->pat.d_words[p], words * 4));
        const u32 *Q = kPatPrimes[p];
        pattern_kernel<<<1024, 256, 0, h->stream>>>(h->pat.d_words[p], words, Q[0], Q[1], Q[2], Q[3], Q[4], Q[5], Q[6]);
        MP_CUDA(h, cudaGetLastError());
    }
    MP_CUDA(h, cudaStreamSynchronize(h->stream));
    h->pat_ready = true;
    return MP_OK;
}

// ---------------------------------------------------------------------------------------
// host driver
// ---------------------------------------------------------------------------------------

struct Tiers { u32 iw0, iw1, itd, it1, iend; };

// qbucket: the primes above it go to the bucket scatter (the tile size, or a half or quarter
// of it when the autotuner finds that moving the sparsest thread-tier primes to buckets pays)
static Tiers tiers_for(const PrimeTable &tb, u32 tlog, u64 top, u64 qbucket)
{
    Tiers r;
    const u64 sq = mp_isqrt64(top - 1) + 1;
    r.iend = (u32)tb.count_le(sq);
    r.iw0 = (u32)std::min<u64>(tb.count_le(PAT_MAXQ), r.iend);
    r.iw1 = (u32)std::min<u64>(tb.count_le(QWARP - 1), r.iend);
    r.it1 = (u32)std::min<u64>(tb.count_le(qbucket), r.iend);
    r.itd = std::max(r.iw1, (u32)std::min<u64>(tb.count_le(std::min<u64>(QDENSE, (1ull << tlog) / 32) - 1), r.it1));
    return r;
}

// the tile kernel's dynamic shared memory, with its limit raised once per device
template <int TLOG, int EMIT>
static cudaError_t tile_smem(size_t *smem)
{
    *smem = ((1u << TLOG) / 32 + HALO_WORDS) * 4;
    static bool attr_set[16] = {false};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 16) return cudaErrorInvalidDevice;
    if (!attr_set[dev]) {
        e = cudaFuncSetAttribute(tile_kernel<TLOG, EMIT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)*smem);
        if (e != cudaSuccess) return e;
        attr_set[dev] = true;
    }
    return cudaSuccess;
}

template <int TLOG, int EMIT>
static cudaError_t launch_tile(const TileArgs &a, int grid, int nth, cudaStream_t st)
{
    size_t smem = 0;
    const cudaError_t e = tile_smem<TLOG, EMIT>(&smem);
    if (e != cudaSuccess) return e;
    tile_kernel<TLOG, EMIT><<<grid, nth, smem, st>>>(a);
    return cudaGetLastError();
}

// resident tile-kernel CTAs per SM at this geometry, from the occupancy calculation (shared
// memory, threads and registers: at 64 registers a thread, 2048 threads of a 2^19-bit tile do
// not fit on one SM although their shared memory does)
template <int TLOG, int EMIT>
static cudaError_t tile_occupancy(int nth, int *per_sm)
{
    size_t smem = 0;
    const cudaError_t e = tile_smem<TLOG, EMIT>(&smem);
    if (e != cudaSuccess) return e;
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, tile_kernel<TLOG, EMIT>, nth, smem);
}

static cudaError_t launch_tile_any(const TileArgs &a, int grid, int nth, int emit, cudaStream_t st)
{
    switch (a.g.tlog * 2 + emit) {
    case 36: return launch_tile<18, 0>(a, grid, nth, st);
    case 37: return launch_tile<18, 1>(a, grid, nth, st);
    case 38: return launch_tile<19, 0>(a, grid, nth, st);
    case 39: return launch_tile<19, 1>(a, grid, nth, st);
    case 40: return launch_tile<20, 0>(a, grid, nth, st);
    case 41: return launch_tile<20, 1>(a, grid, nth, st);
    default: return cudaErrorInvalidValue;
    }
}

// resident CTAs per SM for the tile kernel at this geometry (at least 1)
static int tile_ctas_per_sm(u32 tlog, int nth, int emit)
{
    int r = 0;
    cudaError_t e;
    switch (tlog * 2 + (emit ? 1 : 0)) {
    case 36: e = tile_occupancy<18, 0>(nth, &r); break;
    case 37: e = tile_occupancy<18, 1>(nth, &r); break;
    case 38: e = tile_occupancy<19, 0>(nth, &r); break;
    case 39: e = tile_occupancy<19, 1>(nth, &r); break;
    case 40: e = tile_occupancy<20, 0>(nth, &r); break;
    default: e = tile_occupancy<20, 1>(nth, &r); break;
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        r = 1;
    }
    return r < 1 ? 1 : r;
}

// expected bucket records per tile for the large primes (Mertens' theorem: the sum of 1/q
// over primes in (a, b] is about ln(ln b / ln a); the wheel of 30 keeps 8 of every 15 odd
// multiples), with a margin
static u32 bucket_cap(u32 tlog, u64 qlo, u64 qmax)
{
    const double T = (double)(1u << tlog) + HALO_BITS;
    const double a = (double)qlo;
    double s = qmax > (u64)a ? log(log((double)qmax) / log(a)) * (8.0 / 15.0) : 0.0;
    double e = T * s * 1.06 + 8.0 * sqrt(T * s + 1.0) + 4096.0;
    if (e > 4.0e9) e = 4.0e9;
    return ((u32)e + 3) & ~3u;
}

struct SievePlan {
    SieveGeom g;
    Tiers ti;
    int nth;
    bool large;
    u32 wt, cap, nwaves;
};

static int plan_sieve(mp_handle *h, const PrimeTable &tb, u64 lo, u64 hi, u32 tlog, int nth, SievePlan &P)
{
    P.g.base = lo & ~1ull;
    P.g.limit = (hi - P.g.base) >> 1;
    const u64 top = hi + MP_TAIL;
    P.g.nbx = (top - P.g.base) >> 1;
    P.g.tlog = tlog;
    const u64 ntiles = (P.g.nbx + (1ull << tlog) - 1) >> tlog;
    if (ntiles >= (1ull << 31)) return mp_set_error(h, MP_ERANGE, "range too long (%llu tiles)", (unsigned long long)ntiles);
    P.g.ntiles = (u32)ntiles;
    const u32 bdiv = h->tune.bucket_div == 2 || h->tune.bucket_div == 4 ? (u32)h->tune.bucket_div : 1u;
    const u64 qbucket = (1ull << tlog) / bdiv;
    P.ti = tiers_for(tb, tlog, top, qbucket);
    if (tb.limit < mp_isqrt64(top - 1)) return mp_set_error(h, MP_EINVAL, "prime table too small");
    P.nth = nth;
    P.large = P.ti.iend > P.ti.it1;
    if (P.large) {
        const u64 qmax = tb.host[P.ti.iend - 1];
        P.cap = bucket_cap(tlog, qbucket, qmax);
        // wave: enough tiles to keep every SM busy for several tiles (8 per SM), within
        // 2 GB of records
        u64 wt = 8ull * (u64)h->sm_count;
        const u64 wmem = (2048ull << 20) / ((u64)P.cap * 4);
        if (wt > wmem) wt = wmem;
        if (wt < 1) wt = 1;
        if (wt > P.g.ntiles) wt = P.g.ntiles;
        if (wt > 2048) wt = 2048;                  // the scatter's staged records keep 11 bits of tile
        while (wt > 1 && (wt << tlog) + HALO_BITS >= (1ull << 31)) wt /= 2;   // 32-bit wave positions
        P.wt = (u32)wt;
        P.nwaves = (P.g.ntiles + P.wt - 1) / P.wt;
    } else {
        P.cap = 0; P.wt = P.g.ntiles; P.nwaves = 1;
    }
    return MP_OK;
}

static void fill_tile_args(mp_handle *h, const PrimeTable &tb, const SievePlan &P, TileArgs &a)
{
    memset(&a, 0, sizeof a);
    a.g = P.g;
    a.q = tb.q.as<u32>();
    a.magic = tb.magic.as<u64>();
    a.iw0 = P.ti.iw0; a.iw1 = P.ti.iw1; a.itd = P.ti.itd; a.it1 = P.ti.it1;
    for (int p = 0; p < MP_NPAT; p++) { a.pat[p] = h->pat.d_words[p]; a.period[p] = h->pat.period[p]; }
}

static cudaError_t launch_scatter(const ScatterArgs &s, u32 nblk, cudaStream_t st)
{
    const size_t smem = ((size_t)2 * SC_STAGE + 2 * s.wt) * 4;
    static bool attr_set[16] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 16) return cudaErrorInvalidDevice;
    if (!attr_set[dev]) {
        // the largest wave (2048 tiles)
        cudaError_t e = cudaFuncSetAttribute(scatter_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                             (int)(((size_t)2 * SC_STAGE + 2 * 2048) * 4));
        if (e != cudaSuccess) return e;
        attr_set[dev] = true;
    }
    scatter_kernel<<<nblk, SC_THREADS, smem, st>>>(s);
    return cudaGetLastError();
}

// records per tile bin of the binned scatter for a wave of wt tiles in `smem_max` bytes of
// shared memory; 0 when the bins would be too small to be worth it
static u32 binned_capacity(u32 wt, int smem_max)
{
    const long long room = (long long)smem_max - 4ll * (wt + SB_OVF) - 256;
    if (room <= 0) return 0;
    u64 c = (u64)room / (4ull * wt);
    if (c > 96) c = 96;
    return c >= 8 ? (u32)c : 0u;
}

static cudaError_t launch_scatter_binned(const ScatterArgs &s, u32 nblk, u32 binc, int smem_max, cudaStream_t st)
{
    const size_t smem = ((size_t)s.wt * binc + s.wt + SB_OVF) * 4;
    static bool attr_set[16] = {false};
    int dev = 0;
    cudaGetDevice(&dev);
    if (dev < 0 || dev >= 16) return cudaErrorInvalidDevice;
    if (!attr_set[dev]) {
        cudaError_t e = cudaFuncSetAttribute(scatter_binned_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
        if (e != cudaSuccess) return e;
        attr_set[dev] = true;
    }
    scatter_binned_kernel<<<nblk, SB_THREADS, smem, st>>>(s, binc);
    return cudaGetLastError();
}

// CTA boundaries for the scatter kernel: contiguous runs of the large primes [i0, i1) of equal
// work, where a prime's work is its expected hits in a wave (proportional to 1/q) plus its
// set-up, worth about 8 hits in a wave of 2^30 bits; per_sm persistent CTAs per SM.  Built on
// the host from the table's prefix sums of 1/q and uploaded once per (i0, i1, CTAs) into a
// buffer of its own (never inside a capture: a capture finds the bounds of its direct run).
// Sets h->scat_cur.
static int scatter_bounds(mp_handle *h, const PrimeTable &tb, u32 i0, u32 i1, u32 per_sm, cudaStream_t st)
{
    const u32 want = (u32)std::max<u64>(1, std::min<u64>((u64)h->sm_count * per_sm, i1 - i0));
    mp_handle::ScatBounds *slot = &h->scat[0];
    for (auto &e : h->scat) {
        if (e.key[0] == i0 && e.key[1] == i1 && e.key[2] == want && e.nblk) {
            e.stamp = ++h->scat_clock;
            h->scat_cur = &e;
            return MP_OK;
        }
        if (e.stamp < slot->stamp) slot = &e;
    }
    if (tb.inv_prefix.size() < (size_t)i1 + 1) return mp_set_error(h, MP_EINVAL, "prime table has no prefix sums");
    const double c = 8.0 / ((double)(1u << 30) * 8.0 / 15.0);      // set-up, in units of 1/q
    auto W = [&](u32 i) { return tb.inv_prefix[i] + c * i; };
    std::vector<u32> &b = h->scat_host;
    b.clear();
    b.push_back(i0);
    const double w0 = W(i0), w1 = W(i1);
    for (u32 n = 1; n < want; n++) {
        const double target = w0 + (w1 - w0) * n / want;
        u32 lo = b.back() + 1, hi = i1;                               // first i with W(i) >= target
        while (lo < hi) {
            const u32 mid = lo + (hi - lo) / 2;
            if (W(mid) < target) lo = mid + 1; else hi = mid;
        }
        if (lo >= i1) break;
        b.push_back(lo);
    }
    b.push_back(i1);
    // the evicted buffer may be in a cached graph: free it (that invalidates the graphs) and
    // allocate the new one
    slot->nblk = 0;
    slot->key[0] = slot->key[1] = slot->key[2] = ~0ull;
    slot->buf.release();
    MP_CUDA(h, slot->buf.ensure(b.size() * 4));
    MP_CUDA(h, cudaMemcpyAsync(slot->buf.p, b.data(), b.size() * 4, cudaMemcpyHostToDevice, st));
    MP_CUDA(h, cudaStreamSynchronize(st));
    slot->key[0] = i0; slot->key[1] = i1; slot->key[2] = want;
    slot->nblk = (u32)b.size() - 1;
    slot->stamp = ++h->scat_clock;
    h->scat_cur = slot;
    return MP_OK;
}

template <int TLOG>
static cudaError_t launch_pipeline(const PipeArgs &p, int grid, int nth, size_t smem, cudaStream_t st)
{
    sieve_pipeline_kernel<TLOG><<<grid, nth, smem, st>>>(p);
    return cudaGetLastError();
}

// resident CTAs per SM at `smem` bytes of dynamic shared memory, after raising the kernel's
// limit on dynamic shared memory to `smem_max` (the occupancy calculation honours that limit,
// so it is set first)
template <int TLOG>
static cudaError_t pipeline_ctas_per_sm(int nth, size_t smem, int smem_max, int *per_sm)
{
    static int attr_set[16] = {0};
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= 16) return cudaErrorInvalidDevice;
    if (attr_set[dev] != smem_max) {
        e = cudaFuncSetAttribute(sieve_pipeline_kernel<TLOG>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_max);
        if (e != cudaSuccess) return e;
        attr_set[dev] = smem_max;
    }
    return cudaOccupancyMaxActiveBlocksPerMultiprocessor(per_sm, sieve_pipeline_kernel<TLOG>, nth, smem);
}

// the pipeline kernel's static shared memory (its tile scans and scatter counters)
template <int TLOG>
static cudaError_t pipeline_static_smem(size_t *bytes)
{
    cudaFuncAttributes fa;
    const cudaError_t e = cudaFuncGetAttributes(&fa, sieve_pipeline_kernel<TLOG>);
    if (e == cudaSuccess) *bytes = fa.sharedSizeBytes;
    return e;
}

// the batched form in one persistent launch (sieve_pipeline_kernel): every wave's scatter and
// tile items from one device queue, the records in a ring of two wave slots
static int run_pipeline(mp_handle *h, const PrimeTable &tb, const SievePlan &P, TileArgs a, int smem_max,
                        int grid_pers, cudaStream_t st)
{
    const int nth = P.nth;
    const u32 tlog = P.g.tlog, nw = P.nwaves;
    // the dynamic shared memory left beside the kernel's static shared memory bounds the bins
    size_t stat = 0;
    MP_CUDA(h, tlog == 18 ? pipeline_static_smem<18>(&stat) : tlog == 19 ? pipeline_static_smem<19>(&stat)
                                                                         : pipeline_static_smem<20>(&stat));
    smem_max = smem_max + 1024 - (int)stat - 256;
    const u32 binc = binned_capacity(P.wt, smem_max);
    if (!binc) return mp_set_error(h, MP_EINVAL, "the pipeline's scatter bins do not fit in shared memory");
    const size_t tile_smem = ((1u << tlog) / 32 + HALO_WORDS) * 4;
    const size_t scat_smem = ((size_t)P.wt * binc + P.wt + SB_OVF) * 4;
    const size_t smem = std::max(tile_smem, scat_smem);
    int per_sm = 0;
    cudaError_t e = tlog == 18 ? pipeline_ctas_per_sm<18>(nth, smem, smem_max, &per_sm)
                  : tlog == 19 ? pipeline_ctas_per_sm<19>(nth, smem, smem_max, &per_sm)
                               : pipeline_ctas_per_sm<20>(nth, smem, smem_max, &per_sm);
    MP_CUDA(h, e);
    if (per_sm < 1) return mp_set_error(h, MP_EINVAL, "the pipeline kernel does not fit on an SM");
    const int grid = h->sm_count * per_sm;
    // carried state: one slot per sparse prime per CTA of whichever launch is larger
    MP_CUDA(h, h->tstate.ensure((size_t)std::max(grid, grid_pers) * (P.ti.it1 - P.ti.itd) * 4 + 64));
    a.tstate = h->tstate.as<u32>();
    MP_CUDA(h, h->rec.ensure((size_t)2 * P.wt * P.cap * 4));
    MP_CUDA(h, h->reccnt.ensure(((size_t)2 * P.wt + 1 + 2 * (size_t)nw) * 4 + 64));
    u32 *cnt0 = h->reccnt.as<u32>();
    MP_CUDA(h, cudaMemsetAsync(cnt0, 0, ((size_t)2 * P.wt + 1 + 2 * (size_t)nw) * 4, st));
    PipeArgs p;
    memset(&p, 0, sizeof p);
    p.ta = a;
    p.ta.reccap = P.cap;
    ScatterArgs &s = p.sa;
    s.base = P.g.base; s.tlog = tlog; s.nbx = P.g.nbx;
    s.q = tb.q.as<u32>(); s.magic = tb.magic.as<u64>();
    s.bounds = h->scat_cur->buf.as<u32>();
    s.cap = P.cap; s.err = h->errflag.as<u32>();
    p.nwaves = nw; p.wt = P.wt; p.ntiles = P.g.ntiles;
    p.nscat = h->scat_cur->nblk;
    p.run = std::max<u32>(1, P.wt / (u32)grid);
    p.binc = binc;
    p.rec[0] = h->rec.as<u32>();
    p.rec[1] = p.rec[0] + (size_t)P.wt * P.cap;
    p.cnt[0] = cnt0;
    p.cnt[1] = cnt0 + P.wt;
    p.ctl = cnt0 + 2 * P.wt;
    p.spin_limit = 1u << 23;
    ProfScope ps(h, PROF_PIPELINE, st);
    e = tlog == 18 ? launch_pipeline<18>(p, grid, nth, smem, st)
      : tlog == 19 ? launch_pipeline<19>(p, grid, nth, smem, st)
                   : launch_pipeline<20>(p, grid, nth, smem, st);
    MP_CUDA(h, e);
    return MP_OK;
}

// mode: 0 batched (waves of tile launches, each CTA a contiguous run of tiles), 1 plain (the
// reference's per-segment launch loop on a full grid: one launch per group of sm_count
// segments, one segment per CTA, each set up from scratch, with its own bucket scatter)
static int run_tiles(mp_handle *h, const PrimeTable &tb, const SievePlan &P, TileArgs a, int mode, int emit,
                     cudaStream_t st)
{
    const int nth = P.nth;
    const u32 plain_w = (u32)std::max(1, h->sm_count);
    const u32 nlaunch = mode == 1 ? (P.g.ntiles + plain_w - 1) / plain_w : P.nwaves;
    const int grid_pers = h->sm_count * tile_ctas_per_sm(P.g.tlog, nth, emit);
    // carried state of the sparse thread-tier primes: one slot per prime per CTA (written and
    // read by the tile kernel only; nothing needs clearing)
    MP_CUDA(h, h->tstate.ensure((size_t)grid_pers * (P.ti.it1 - P.ti.itd) * 4 + 64));
    a.tstate = h->tstate.as<u32>();
    u32 *errp = h->errflag.as<u32>();
    const u32 wmax = mode == 1 ? std::min(plain_w, P.g.ntiles) : P.wt;
    if (P.large) {
        MP_CUDA(h, h->rec.ensure((size_t)wmax * P.cap * 4));
        MP_CUDA(h, h->reccnt.ensure((size_t)wmax * 4 * 2));
    }
    // the binned scatter (one CTA per SM) unless the wave's bins would not fit or the handle
    // asks for the staged form
    int smem_max = 0;
    MP_CUDA(h, cudaDeviceGetAttribute(&smem_max, cudaDevAttrMaxSharedMemoryPerBlockOptin, h->device));
    smem_max -= 1024;                                   // the kernel's static shared memory and slack
    const u32 binc = P.large && h->tune.scatter_staged == 0 ? binned_capacity(wmax, smem_max) : 0u;
    if (P.large) MP_TRY(scatter_bounds(h, tb, P.ti.it1, P.ti.iend, binc ? 1u : (u32)SC_CTAS_PER_SM, st));
    if (mode == 0 && !emit && binc && !h->tune.no_pipeline) return run_pipeline(h, tb, P, a, smem_max, grid_pers, st);
    for (u32 L = 0; L < nlaunch; L++) {
        const u32 t0 = L * wmax;
        const u32 nt = std::min(wmax, P.g.ntiles - t0);
        if (P.large) {
            ScatterArgs s;
            s.base = P.g.base; s.tlog = P.g.tlog; s.t0 = t0; s.wt = nt; s.nbx = P.g.nbx;
            s.q = tb.q.as<u32>(); s.magic = tb.magic.as<u64>();
            s.bounds = h->scat_cur->buf.as<u32>();
            s.rec = h->rec.as<u32>(); s.cnt = h->reccnt.as<u32>(); s.cap = P.cap; s.err = errp;
            MP_CUDA(h, cudaMemsetAsync(s.cnt, 0, (size_t)nt * 4, st));
            const u32 nblk = h->scat_cur->nblk;
            {
                ProfScope ps(h, PROF_SCATTER, st);
                if (binc) MP_CUDA(h, launch_scatter_binned(s, nblk, binc, smem_max, st));
                else MP_CUDA(h, launch_scatter(s, nblk, st));
            }
            a.rec = s.rec; a.reccnt = s.cnt; a.reccap = P.cap;
        }
        a.t0 = t0; a.nt = nt;
        const int grid = mode == 1 ? (int)nt : (int)std::min<u64>((u64)grid_pers, nt);
        ProfScope ps(h, PROF_TILE, st);
        MP_CUDA(h, launch_tile_any(a, grid, nth, emit, st));
    }
    return MP_OK;
}

static int check_errflag(mp_handle *h, cudaStream_t st)
{
    MP_CUDA(h, cudaMemcpyAsync(h->h_err, h->errflag.p, 4, cudaMemcpyDeviceToHost, st));
    MP_CUDA(h, cudaStreamSynchronize(st));
    const u32 e = *h->h_err;
    if (e) {
        MP_CUDA(h, cudaMemsetAsync(h->errflag.p, 0, 4, st));
        if (e & 2) return mp_set_error(h, MP_EOVERFLOW, "bucket records exceeded their capacity");
        if (e & 4) return mp_set_error(h, MP_ERANGE, "no prime follows the last prime of the range within the tail");
        if (e & 8) return mp_set_error(h, MP_ETIMEOUT, "a wait of the sieve pipeline ran out (its results are not valid)");
        return mp_set_error(h, MP_ETIMEOUT, "device error flag 0x%x", e);
    }
    return MP_OK;
}

int mp_tables_ensure(mp_handle *h, u64 limit)
{
    MP_TRY(mp_patterns_ensure(h));
    if (limit <= h->tab->limit) return MP_OK;
    if (h->shared_tables || h->servers_open)
        return mp_set_error(h, MP_ERANGE, "needs sieving primes up to %llu, above the resident table (%llu) that "
                            "an open server shares", (unsigned long long)limit, (unsigned long long)h->tab->limit);
    cudaStream_t st = h->stream;
    if (!h->boot.n) {
        MP_CUDA(h, h->boot.q.ensure(6600 * 4));
        MP_CUDA(h, h->boot.magic.ensure(6600 * 8));
        MP_CUDA(h, h->small_out.ensure(64));
        boot_primes_kernel<<<1, 1024, 0, st>>>(h->boot.q.as<u32>(), h->small_out.as<u32>());
        MP_CUDA(h, cudaGetLastError());
        u32 n = 0;
        MP_CUDA(h, cudaMemcpyAsync(&n, h->small_out.p, 4, cudaMemcpyDeviceToHost, st));
        MP_CUDA(h, cudaStreamSynchronize(st));
        h->boot.n = n;
        h->boot.limit = 65536;   // every prime <= 65536 (65536 itself is not prime)
        magic_kernel<<<64, 256, 0, st>>>(h->boot.q.as<u32>(), n, h->boot.magic.as<u64>());
        MP_CUDA(h, cudaGetLastError());
        h->boot.host.resize(n);
        MP_CUDA(h, cudaMemcpyAsync(h->boot.host.data(), h->boot.q.p, (size_t)n * 4, cudaMemcpyDeviceToHost, st));
        MP_CUDA(h, cudaStreamSynchronize(st));
    }
    u64 L = std::max<u64>(limit, std::max<u64>(1ull << 22, 2 * h->table.limit));
    if (L > 0xffffffffull) L = 0xffffffffull;
    if (limit > L) return mp_set_error(h, MP_ERANGE, "sieving primes above 2^32 are not supported");
    // sieve [3, L] with the bootstrap primes and emit the odd primes as u32
    SievePlan P;
    const u64 lo = 3, hi = L + 1;
    MP_TRY(plan_sieve(h, h->boot, lo, hi, 20, 1024, P));
    // the tail is not needed for a prime list, but plan_sieve adds it; primes beyond hi are
    // not emitted (limit bits)
    MP_CUDA(h, h->tilesum.ensure((size_t)P.g.ntiles * sizeof(TileSum)));
    MP_CUDA(h, h->blockacc.ensure((size_t)P.g.ntiles * 8 + 16));
    TileArgs a;
    fill_tile_args(h, h->boot, P, a);
    a.sums = h->tilesum.as<TileSum>();
    MP_TRY(run_tiles(h, h->boot, P, a, 0, 0, st));
    u64 *off = h->blockacc.as<u64>();
    tile_scan_kernel<<<1, 1024, 0, st>>>(a.sums, P.g.ntiles, off, off + P.g.ntiles);
    MP_CUDA(h, cudaGetLastError());
    u64 total = 0;
    MP_CUDA(h, cudaMemcpyAsync(&total, off + P.g.ntiles, 8, cudaMemcpyDeviceToHost, st));
    MP_CUDA(h, cudaStreamSynchronize(st));
    h->table.q.release();
    h->table.magic.release();
    h->table.n = 0;
    h->table.limit = 0;
    MP_CUDA(h, h->table.q.ensure((size_t)total * 4 + 64));
    MP_CUDA(h, h->table.magic.ensure((size_t)total * 8 + 64));
    a.emit_off = off;
    a.emit32 = h->table.q.as<u32>();
    a.emit64 = nullptr;
    MP_TRY(run_tiles(h, h->boot, P, a, 0, 1, st));
    magic_kernel<<<1024, 256, 0, st>>>(h->table.q.as<u32>(), total, h->table.magic.as<u64>());
    MP_CUDA(h, cudaGetLastError());
    h->table.host.resize(total);
    MP_CUDA(h, cudaMemcpyAsync(h->table.host.data(), h->table.q.p, (size_t)total * 4, cudaMemcpyDeviceToHost, st));
    MP_CUDA(h, cudaStreamSynchronize(st));
    h->table.inv_prefix.resize(total + 1);
    h->table.inv_prefix[0] = 0.0;
    for (u64 i = 0; i < total; i++) h->table.inv_prefix[i + 1] = h->table.inv_prefix[i] + 1.0 / h->table.host[i];
    // the prime indices changed meaning: drop every scatter bound (and with them the graphs)
    for (auto &e : h->scat) {
        e.buf.release();
        e.nblk = 0;
        e.key[0] = e.key[1] = e.key[2] = ~0ull;
    }
    h->scat_cur = nullptr;
    MP_TRY(check_errflag(h, st));
    h->table.n = total;
    h->table.limit = L;
    return MP_OK;
}

static int pick_geometry(mp_handle *h, const mp_sieve_opts *o, u32 &tlog, int &nth)
{
    tlog = o && o->tile_log2 ? o->tile_log2 : (h->tune.sieve_tile_log2 ? (u32)h->tune.sieve_tile_log2 : 20);
    nth = o && o->threads ? (int)o->threads : (h->tune.sieve_threads ? h->tune.sieve_threads : 1024);
    if (tlog < 18 || tlog > 20) return mp_set_error(h, MP_EINVAL, "tile_log2 must be 18, 19 or 20");
    if (nth != 256 && nth != 512 && nth != 1024) return mp_set_error(h, MP_EINVAL, "threads must be 256, 512 or 1024");
    return MP_OK;
}

int mp_sieve_run(mp_handle *h, u64 lo, u64 hi, const mp_sieve_opts *o, mp_range_stats *d_out,
                 mp_block_stats *d_blocks, u64 *d_hash, u64 *d_bitmap, cudaStream_t st)
{
    if (hi <= lo) return mp_set_error(h, MP_EINVAL, "need lo < hi");
    if (hi > MP_HI_MAX) return mp_set_error(h, MP_ERANGE, "hi must be <= 2^64 - 2^18");
    if (!d_out) return mp_set_error(h, MP_EINVAL, "null output");
    const u32 mode = o ? o->mode : MP_MODE_BATCHED;
    if (mode > 1) return mp_set_error(h, MP_EINVAL, "bad mode");
    u32 tlog;
    int nth;
    MP_TRY(pick_geometry(h, o, tlog, nth));
    if (mode == MP_MODE_PLAIN && !(o && o->tile_log2)) tlog = 18;   // the reference's 32 KiB segment
    const u32 block_log2 = o ? o->block_log2 : 0, hash_log2 = o ? o->hash_log2 : 0;
    if (block_log2 && (block_log2 < tlog + 1 || block_log2 > 32))
        return mp_set_error(h, MP_EINVAL, "block_log2 must be 0 or in [tile_log2 + 1, 32]");
    if (hash_log2 && (hash_log2 < 4 || hash_log2 > 40)) return mp_set_error(h, MP_EINVAL, "hash_log2 must be 0 or 4..40");
    if (d_blocks && !block_log2) return mp_set_error(h, MP_EINVAL, "blocks requested without block_log2");
    const u64 top = hi + MP_TAIL;
    MP_TRY(mp_tables_ensure(h, mp_isqrt64(top - 1)));
    SievePlan P;
    MP_TRY(plan_sieve(h, *h->tab, lo, hi, tlog, nth, P));
    MP_CUDA(h, h->tilesum.ensure((size_t)P.g.ntiles * sizeof(TileSum)));
    // bitmap: the caller's, or scratch when only hashes are wanted
    const u64 nwords64 = (P.g.limit + 63) >> 6;
    u32 *bm = (u32 *)d_bitmap;
    if (!bm && hash_log2) {
        MP_CUDA(h, h->scratch_bitmap.ensure((size_t)nwords64 * 8 + 64));
        bm = h->scratch_bitmap.as<u32>();
    }
    TileArgs a;
    fill_tile_args(h, *h->tab, P, a);
    a.sums = h->tilesum.as<TileSum>();
    a.bitmap32 = bm;
    MP_TRY(run_tiles(h, *h->tab, P, a, (int)mode, 0, st));
    // fold
    u32 tpb;
    u64 nblocks;
    if (block_log2) {
        tpb = 1u << (block_log2 - 1 - tlog);
        nblocks = ((hi - lo - 1) >> block_log2) + 1;
    } else {
        tpb = 8;
        while ((P.g.ntiles + tpb - 1) / tpb > 65536) tpb *= 2;
        const u64 bb = (u64)tpb << tlog;
        nblocks = (P.g.limit + bb - 1) / bb;
        if (nblocks == 0) nblocks = 1;
    }
    const u64 nbe = (P.g.ntiles + tpb - 1) / tpb;
    if (nbe > (1ull << 26)) return mp_set_error(h, MP_ERANGE, "too many blocks");
    MP_CUDA(h, h->blockacc.ensure((size_t)nbe * sizeof(Part)));
    FoldArgs f;
    f.base = P.g.base; f.limit = P.g.limit; f.lo = lo; f.hi = hi;
    f.sums = a.sums; f.ntiles = P.g.ntiles; f.tpb = tpb;
    f.nblocks = (u32)std::min<u64>(nblocks, nbe); f.nblocks_ext = (u32)nbe;
    f.acc = h->blockacc.as<Part>();
    f.out = d_out; f.blocks = d_blocks; f.err = h->errflag.as<u32>();
    f.has2 = lo <= 2 && 2 < hi;
    {
        ProfScope ps(h, PROF_FOLD, st);
        fold_kernel<<<1, 512, 0, st>>>(f);
    }
    MP_CUDA(h, cudaGetLastError());
    if (hash_log2) {
        const u64 sb = 1ull << (hash_log2 - 1);
        const u64 ns = (P.g.limit + sb - 1) / sb;
        ProfScope ps(h, PROF_HASH, st);
        hash_kernel<<<(unsigned)((ns + 31) / 32), 32, 0, st>>>(bm, P.g.limit, sb, ns, d_hash);
        MP_CUDA(h, cudaGetLastError());
    }
    return MP_OK;
}

int mp_sieve_errors(mp_handle *h, cudaStream_t st) { return check_errflag(h, st); }

// all primes in [lo, hi) to d_primes (cap entries); *count = number of primes; synchronises
int mp_sieve_emit_primes(mp_handle *h, u64 lo, u64 hi, u64 *d_primes, u64 cap, u64 *count, cudaStream_t st)
{
    if (hi <= lo) { *count = 0; return MP_OK; }
    if (hi > MP_HI_MAX) return mp_set_error(h, MP_ERANGE, "hi must be <= 2^64 - 2^18");
    u32 tlog;
    int nth;
    MP_TRY(pick_geometry(h, nullptr, tlog, nth));
    const u64 top = hi + MP_TAIL;
    MP_TRY(mp_tables_ensure(h, mp_isqrt64(top - 1)));
    SievePlan P;
    MP_TRY(plan_sieve(h, *h->tab, lo, hi, tlog, nth, P));
    MP_CUDA(h, h->tilesum.ensure((size_t)P.g.ntiles * sizeof(TileSum)));
    MP_CUDA(h, h->blockacc.ensure((size_t)P.g.ntiles * 8 + 16));
    TileArgs a;
    fill_tile_args(h, *h->tab, P, a);
    a.sums = h->tilesum.as<TileSum>();
    MP_TRY(run_tiles(h, *h->tab, P, a, 0, 0, st));
    u64 *off = h->blockacc.as<u64>();
    tile_scan_kernel<<<1, 1024, 0, st>>>(a.sums, P.g.ntiles, off, off + P.g.ntiles);
    MP_CUDA(h, cudaGetLastError());
    u64 total = 0;
    MP_CUDA(h, cudaMemcpyAsync(&total, off + P.g.ntiles, 8, cudaMemcpyDeviceToHost, st));
    MP_CUDA(h, cudaStreamSynchronize(st));
    const u64 odd_total = total;
    const int has2 = lo <= 2 && 2 < hi;
    *count = odd_total + has2;
    if (*count > cap || *count == 0) return MP_OK;   // caller re-sizes
    u64 *dst = d_primes;
    if (has2) {
        const u64 two = 2;
        MP_CUDA(h, cudaMemcpyAsync(d_primes, &two, 8, cudaMemcpyHostToDevice, st));
        dst = d_primes + 1;
    }
    a.emit_off = off;
    a.emit64 = dst;
    a.emit32 = nullptr;
    MP_TRY(run_tiles(h, *h->tab, P, a, 0, 1, st));
    MP_CUDA(h, cudaStreamSynchronize(st));
    return check_errflag(h, st);
}
