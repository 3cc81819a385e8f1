// mp_fermat.cu -- Fermat quotients q_p(2) = (2^(p-1) mod p^2 - 1) / p on B200 (sm_100a).
//
// Reference (paths inside the Mathpub project): pctx_init / msqr / redc
// A001220/wieferich.c:546-645 (Montgomery arithmetic mod N = p^2 with R = 2^128, p^-1 by
// Newton from (3p) xor 2), fermat_quotient :939 (q = (r - 1) p^-1 mod 2^64), finish_lanes
// :1051-1075 (Fermat's little theorem check q < p, checksum mix64(q ^ p * GOLD), symmetric
// residue A).
//
// The device form keeps the same mathematics with a different number layout: N = p^2 is
// held in K 32-bit limbs (K = 3, R = 2^96, for p < 2^47; K = 4, R = 2^128, for p < 2^63),
// multiplied with the CIOS Montgomery product on 32x32->64 integer multiply-adds.  The form
// of 1 (R mod N) is found by doubling 2^(bitlen(N)-1) up to R, exactly; the reference's
// double-precision quotient estimates are not used.  The exponent p - 1 is processed left
// to right: square, then double when the bit is 1 (base 2 needs no multiplier table).  Where
// 8N < R (p < 2^46 with three limbs, p < 2^62 with four) the two are one product,
// x (x 2^bit) / R, the doubling being a funnel shift of one operand.
#include "mp_common.cuh"

// t[0..K] += a[0..K-1] * b: the low halves of the products in one carry chain, then the high
// halves one word up in a second; each chain is one asm block, so that nothing between its
// instructions can touch the carry flag.  The multiply-adds run on the multiply pipe.  The
// callers keep t below 2^(32 (K + 1)), so nothing carries out of t[K] (see mmul_lazy).
template <int K>
__device__ __forceinline__ void mac_row(u32 (&t)[K + 1], const u32 (&a)[K], u32 b);

template <>
__device__ __forceinline__ void mac_row<3>(u32 (&t)[4], const u32 (&a)[3], u32 b)
{
    asm("mad.lo.cc.u32  %0, %4, %7, %0;\n\t"
        "madc.lo.cc.u32 %1, %5, %7, %1;\n\t"
        "madc.lo.cc.u32 %2, %6, %7, %2;\n\t"
        "addc.u32       %3, %3, 0;\n\t"
        "mad.hi.cc.u32  %1, %4, %7, %1;\n\t"
        "madc.hi.cc.u32 %2, %5, %7, %2;\n\t"
        "madc.hi.u32    %3, %6, %7, %3;"
        : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(b));
}

template <>
__device__ __forceinline__ void mac_row<4>(u32 (&t)[5], const u32 (&a)[4], u32 b)
{
    asm("mad.lo.cc.u32  %0, %5, %9, %0;\n\t"
        "madc.lo.cc.u32 %1, %6, %9, %1;\n\t"
        "madc.lo.cc.u32 %2, %7, %9, %2;\n\t"
        "madc.lo.cc.u32 %3, %8, %9, %3;\n\t"
        "addc.u32       %4, %4, 0;\n\t"
        "mad.hi.cc.u32  %1, %5, %9, %1;\n\t"
        "madc.hi.cc.u32 %2, %6, %9, %2;\n\t"
        "madc.hi.cc.u32 %3, %7, %9, %3;\n\t"
        "madc.hi.u32    %4, %8, %9, %4;"
        : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b));
}

// t - n with the borrow out in one chain: returns 0 when t >= n, all ones otherwise
template <int K>
__device__ __forceinline__ u32 sub_n(u32 (&d)[K], const u32 (&t)[K], const u32 (&n)[K]);

template <>
__device__ __forceinline__ u32 sub_n<3>(u32 (&d)[3], const u32 (&t)[3], const u32 (&n)[3])
{
    u32 bw;
    asm("sub.cc.u32  %0, %4, %7;\n\t"
        "subc.cc.u32 %1, %5, %8;\n\t"
        "subc.cc.u32 %2, %6, %9;\n\t"
        "subc.u32    %3, 0, 0;"
        : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(bw)
        : "r"(t[0]), "r"(t[1]), "r"(t[2]), "r"(n[0]), "r"(n[1]), "r"(n[2]));
    return bw;
}

template <>
__device__ __forceinline__ u32 sub_n<4>(u32 (&d)[4], const u32 (&t)[4], const u32 (&n)[4])
{
    u32 bw;
    asm("sub.cc.u32  %0, %5, %9;\n\t"
        "subc.cc.u32 %1, %6, %10;\n\t"
        "subc.cc.u32 %2, %7, %11;\n\t"
        "subc.cc.u32 %3, %8, %12;\n\t"
        "subc.u32    %4, 0, 0;"
        : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(bw)
        : "r"(t[0]), "r"(t[1]), "r"(t[2]), "r"(t[3]), "r"(n[0]), "r"(n[1]), "r"(n[2]), "r"(n[3]));
    return bw;
}

template <int K>
__device__ __forceinline__ void cond_sub(u32 (&t)[K], u32 top, const u32 (&n)[K])
{
    // t (with carry word `top`) < 2N: subtract N once if t >= N
    u32 d[K];
    const u32 bw = sub_n<K>(d, t, n);
    const bool ge = top || !bw;
#pragma unroll
    for (int j = 0; j < K; j++) t[j] = ge ? d[j] : t[j];
}

// r = a * b / R mod N, CIOS with 32-bit limbs: per word b[i], t += a b[i], then t += m N with
// m = t[0] (-N^-1) mod 2^32, which clears t[0], and t shifts down a word.  With a, b < 2N and
// 4N < R the result (ab + mN) / R is below N (4N / R + 1) < 2N, so values stay in [0, 2N)
// without a subtraction (lazy reduction); only the value that leaves the loop is reduced.
// Bounds: before a row pair t < 3N (K words), after it t < 3N (1 + 2^32) < 2^(32 (K + 1)).
template <int K>
__device__ __forceinline__ void mmul_lazy(u32 (&r)[K], const u32 (&a)[K], const u32 (&b)[K], const u32 (&n)[K],
                                          u32 np)
{
    u32 t[K + 1];
#pragma unroll
    for (int j = 0; j < K + 1; j++) t[j] = 0;
#pragma unroll
    for (int i = 0; i < K; i++) {
        mac_row<K>(t, a, b[i]);
        const u32 m = t[0] * np;
        mac_row<K>(t, n, m);
#pragma unroll
        for (int j = 0; j < K; j++) t[j] = t[j + 1];
        t[K] = 0;
    }
#pragma unroll
    for (int j = 0; j < K; j++) r[j] = t[j];
}

// the same, reduced to [0, N) (for a product below 2N)
template <int K>
__device__ __forceinline__ void mmul(u32 (&r)[K], const u32 (&a)[K], const u32 (&b)[K], const u32 (&n)[K], u32 np)
{
    mmul_lazy<K>(r, a, b, n, np);
    cond_sub<K>(r, 0u, n);
}

// x = 2x, reduced below m (x < m, 2m <= R): m = N keeps [0, N), m = 2N keeps [0, 2N)
template <int K>
__device__ __forceinline__ void mdbl(u32 (&x)[K], const u32 (&n)[K])
{
    u32 y[K];
    y[0] = x[0] << 1;
#pragma unroll
    for (int j = 1; j < K; j++) y[j] = (x[j] << 1) | (x[j - 1] >> 31);
    cond_sub<K>(y, 0u, n);
#pragma unroll
    for (int j = 0; j < K; j++) x[j] = y[j];
}

struct FermOut { u64 q; bool ok; };

// q_p(2) for odd p >= 3 (p < 2^47 for K = 3, p < 2^63 for K = 4)
template <int K>
__device__ __forceinline__ FermOut fermat_one(u64 p)
{
    u64 pinv = (3 * p) ^ 2;
    pinv *= 2 - p * pinv;
    pinv *= 2 - p * pinv;
    pinv *= 2 - p * pinv;
    pinv *= 2 - p * pinv;
    const u32 np = 0u - (u32)(pinv * pinv);            // -N^-1 mod 2^32
    const u64 N0 = p * p, N1 = __umul64hi(p, p);
    u32 n[K];
    n[0] = (u32)N0; n[1] = (u32)(N0 >> 32); n[2] = (u32)N1;
    if (K == 4) n[K - 1] = (u32)(N1 >> 32);
    // one = R mod N: start at 2^(top bit of N), double up to 2^(32K)
    const int topbit = N1 ? 64 + 63 - __clzll((long long)N1) : 63 - __clzll((long long)N0);
    u32 x[K];
#pragma unroll
    for (int j = 0; j < K; j++) x[j] = (topbit >> 5) == j ? (1u << (topbit & 31)) : 0u;
    for (int i = topbit; i < 32 * K; i++) mdbl<K>(x, n);
    // left-to-right binary exponentiation of 2 to e = p - 1 on representatives in [0, 2N)
    // (lazy reduction; 4N < R for both limb counts); leading zero bits keep x = 1
    u32 n2[K];
    n2[0] = n[0] << 1;
#pragma unroll
    for (int j = 1; j < K; j++) n2[j] = (n[j] << 1) | (n[j - 1] >> 31);
    const u64 e = p - 1;
    if (p < (K == 3 ? (1ull << 46) : (1ull << 62))) {
        // 8N < R: the doubling for a 1 bit goes into the product.  x (x 2^bit) / R with
        // x < 2N and x 2^bit < 4N (a funnel shift, no subtraction) is below
        // (8N^2 + R N) / R < 2N, so the square-and-double of one bit is one product
        for (int b = 63 - __clzll((long long)e); b >= 0; b--) {
            const u32 bit = (u32)(e >> b) & 1u;
            u32 y[K];
            y[0] = x[0] << bit;
#pragma unroll
            for (int j = 1; j < K; j++) y[j] = __funnelshift_l(x[j - 1], x[j], bit);
            mmul_lazy<K>(x, x, y, n, np);
        }
    } else {
        for (int b = 63 - __clzll((long long)e); b >= 0; b--) {
            mmul_lazy<K>(x, x, x, n, np);
            u32 y[K];
#pragma unroll
            for (int j = 0; j < K; j++) y[j] = x[j];
            mdbl<K>(y, n2);
            const bool bit = (e >> b) & 1;
#pragma unroll
            for (int j = 0; j < K; j++) x[j] = bit ? y[j] : x[j];
        }
    }
    // leave Montgomery form: multiply by 1; with x < 2N the product (x + mN) / R is at most N,
    // and mmul's subtraction brings it to [0, N)
    u32 one[K];
#pragma unroll
    for (int j = 0; j < K; j++) one[j] = j == 0 ? 1u : 0u;
    mmul<K>(x, x, one, n, np);
    const u64 r = (u64)x[0] | ((u64)x[1] << 32);
    FermOut o;
    o.q = (r - 1) * pinv;
    o.ok = o.q < p;
    return o;
}

// one prime per thread (ILP = 1) or two interleaved primes per thread (ILP = 2)
template <int K, int ILP>
__global__ void __launch_bounds__(256) fermat_kernel(const u64 *__restrict__ P, u64 count, u64 *__restrict__ Q)
{
    const u64 stride = (u64)gridDim.x * blockDim.x * ILP;
    for (u64 i = ((u64)blockIdx.x * blockDim.x + threadIdx.x) * ILP; i < count; i += stride) {
        if (ILP == 1) {
            const u64 p = __ldg(P + i);
            u64 q = 0;
            if (p >= 3 && (p & 1)) { const FermOut o = fermat_one<K>(p); q = o.ok ? o.q : ~0ull; }
            Q[i] = q;
        } else {
            const u64 p0 = __ldg(P + i), p1 = i + 1 < count ? __ldg(P + i + 1) : 3;
            const bool v0 = p0 >= 3 && (p0 & 1), v1 = p1 >= 3 && (p1 & 1);
            const FermOut o0 = fermat_one<K>(v0 ? p0 : 3), o1 = fermat_one<K>(v1 ? p1 : 3);
            Q[i] = v0 ? (o0.ok ? o0.q : ~0ull) : 0;
            if (i + 1 < count) Q[i + 1] = v1 ? (o1.ok ? o1.q : ~0ull) : 0;
        }
    }
}

// ---- statistics: checksum, near count, FLT errors, hits, ordered hash ----

struct FermPart {
    u64 h, len;          // ordered hash over the segment and its number of terms
    u64 cks, near, flt, tests;
};

__device__ __forceinline__ u64 pow_u64(u64 b, u64 e)
{
    u64 r = 1;
    while (e) { if (e & 1) r *= b; b *= b; e >>= 1; }
    return r;
}

__device__ __forceinline__ void fp_join(FermPart &L, const FermPart &R)
{
    L.h = L.h * pow_u64(MP_FNV_PRIME, R.len) + R.h;
    L.len += R.len;
    L.cks += R.cks; L.near += R.near; L.flt += R.flt; L.tests += R.tests;
}

#define FS_THREADS 256
#define FS_PER 8                                           // consecutive entries per thread
#define FS_TILE (FS_THREADS * FS_PER)                      // entries per CTA

// one CTA per FS_TILE entries: the tile's primes and quotients are staged in shared memory
// with coalesced loads, each thread folds its FS_PER consecutive entries in order (the ordered
// hash by Horner's rule), then the threads join in order
__global__ void __launch_bounds__(FS_THREADS) fermat_stats_kernel(const u64 *__restrict__ P, const u64 *__restrict__ Q,
                                                                  u64 count, FermPart *parts, u64 *hits, u64 *nhits)
{
    __shared__ FermPart s_w[FS_THREADS / 32];
    // entry k at k + k / FS_PER: a thread's FS_PER entries are 9 words apart from the next
    // thread's, which keeps the reads nearly free of bank conflicts
    __shared__ u64 sp[FS_TILE + FS_TILE / FS_PER], sq[FS_TILE + FS_TILE / FS_PER];
    const u64 t0 = (u64)blockIdx.x * FS_TILE;
    for (u32 k = threadIdx.x; k < FS_TILE; k += FS_THREADS) {
        const bool in = t0 + k < count;
        sp[k + k / FS_PER] = in ? __ldcs(P + t0 + k) : 0;
        sq[k + k / FS_PER] = in ? __ldcs(Q + t0 + k) : 0;
    }
    __syncthreads();
    FermPart f = {0, 0, 0, 0, 0, 0};
#pragma unroll
    for (int u = 0; u < FS_PER; u++) {
        const u64 p = sp[threadIdx.x * (FS_PER + 1) + u], q = sq[threadIdx.x * (FS_PER + 1) + u];
        if (p < 3) continue;                               // 2 is not tested (and padding)
        f.tests++;
        if (q >= p) { f.flt++; continue; }
        f.cks += mp_mix64(q ^ (p * MP_GOLD));
        const u64 A = q <= p / 2 ? q : p - q;
        f.near += A <= (p - 1) / 1000;                     // 1000 A < p
        f.h = f.h * MP_FNV_PRIME + mp_mix64(p ^ mp_mix64(q));
        f.len++;
        if (q == 0) {
            // keep the 16 smallest hits, sorted, whatever the order the threads arrive in:
            // slot j keeps the smaller of its value and the incoming one and passes the larger
            // on, so slot j ends with the (j+1)-th smallest value that ever reached it
            atomicAdd((unsigned long long *)nhits, 1ull);
            u64 v = p;
            for (int j = 0; j < 16 && v != ~0ull; j++) {
                const u64 old = atomicMin((unsigned long long *)(hits + j), (unsigned long long)v);
                v = old > v ? old : v;
            }
        }
    }
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        FermPart r;
        r.h = __shfl_down_sync(0xffffffffu, f.h, d);
        r.len = __shfl_down_sync(0xffffffffu, f.len, d);
        r.cks = __shfl_down_sync(0xffffffffu, f.cks, d);
        r.near = __shfl_down_sync(0xffffffffu, f.near, d);
        r.flt = __shfl_down_sync(0xffffffffu, f.flt, d);
        r.tests = __shfl_down_sync(0xffffffffu, f.tests, d);
        if ((lane & (2 * d - 1)) == 0 && lane + d < 32) fp_join(f, r);
    }
    if (lane == 0) s_w[warp] = f;
    __syncthreads();
    if (threadIdx.x == 0) {
        FermPart b = s_w[0];
        for (int w = 1; w < FS_THREADS / 32; w++) fp_join(b, s_w[w]);
        parts[blockIdx.x] = b;
    }
}

__global__ void __launch_bounds__(1024) fermat_final_kernel(const FermPart *parts, u64 nparts, const u64 *nhits,
                                                            const u64 *hits, mp_wief_stats *out)
{
    __shared__ FermPart s[1024];
    const u32 tid = threadIdx.x, nth = blockDim.x;
    const u64 per = (nparts + nth - 1) / nth;
    FermPart f = {0, 0, 0, 0, 0, 0};
    for (u64 b = tid * per; b < (tid + 1) * per && b < nparts; b++) fp_join(f, parts[b]);
    s[tid] = f;
    __syncthreads();
    if (tid == 0) {
        FermPart g = s[0];
        for (u32 i = 1; i < nth; i++) fp_join(g, s[i]);
        out->tests = g.tests;
        out->near = g.near;
        out->flt = g.flt;
        out->cks = g.cks;
        out->ordered_hash = g.h;
        out->nhits = *nhits;
        for (int k = 0; k < 16; k++) out->hits[k] = (u64)k < *nhits ? hits[k] : 0;
    }
}

// ---- host side ----

int mp_fermat_run(mp_handle *h, const u64 *d_p, u64 count, u64 *d_q, cudaStream_t st, int variant, u64 *)
{
    if (!count) return MP_OK;
    // variant: bit 0 = limbs (0: K=3, 1: K=4); bit 1 = two primes per thread
    const int k4 = variant & 1, ilp2 = (variant >> 1) & 1;
    const u64 work = ilp2 ? (count + 1) / 2 : count;
    u64 grid = (work + 255) / 256;
    const u64 gmax = (u64)h->sm_count * 64;
    if (grid > gmax) grid = gmax;
    ProfScope ps(h, PROF_FERMAT, st);
    if (!k4 && !ilp2) fermat_kernel<3, 1><<<(unsigned)grid, 256, 0, st>>>(d_p, count, d_q);
    else if (!k4 && ilp2) fermat_kernel<3, 2><<<(unsigned)grid, 256, 0, st>>>(d_p, count, d_q);
    else if (k4 && !ilp2) fermat_kernel<4, 1><<<(unsigned)grid, 256, 0, st>>>(d_p, count, d_q);
    else fermat_kernel<4, 2><<<(unsigned)grid, 256, 0, st>>>(d_p, count, d_q);
    MP_CUDA(h, cudaGetLastError());
    return MP_OK;
}

int mp_fermat_reduce(mp_handle *h, const u64 *d_p, const u64 *d_q, u64 count, mp_wief_stats *d_stats, cudaStream_t st)
{
    const u64 nb = count ? (count + FS_TILE - 1) / FS_TILE : 1;
    MP_CUDA(h, h->ferm_part.ensure((size_t)nb * sizeof(FermPart) + 256));
    FermPart *parts = h->ferm_part.as<FermPart>();
    u64 *hits = (u64 *)((char *)h->ferm_part.p + nb * sizeof(FermPart));
    u64 *nhits = hits + 16;
    MP_CUDA(h, cudaMemsetAsync(hits, 0xff, 16 * 8, st));        // empty slots hold 2^64 - 1
    MP_CUDA(h, cudaMemsetAsync(nhits, 0, 8, st));
    if (count) {
        ProfScope ps(h, PROF_FERMAT_STATS, st);
        fermat_stats_kernel<<<(unsigned)nb, FS_THREADS, 0, st>>>(d_p, d_q, count, parts, hits, nhits);
        MP_CUDA(h, cudaGetLastError());
    } else {
        MP_CUDA(h, cudaMemsetAsync(parts, 0, sizeof(FermPart), st));
    }
    fermat_final_kernel<<<1, 1024, 0, st>>>(parts, nb, nhits, hits, d_stats);
    MP_CUDA(h, cudaGetLastError());
    return MP_OK;
}

// ---------------------------------------------------------------------------------------
// mp_wieferich_stats_noalloc: the statistics of mp_wieferich_range for caller-supplied device
// arrays of primes and quotients, for callers that must not allocate device memory -- code
// that runs under a memory manager or pool that owns the whole device, inside a framework
// whose allocator may not be bypassed, or in a latency-critical loop where a cudaMalloc
// (which can synchronise the device) is not allowed.  It uses no handle (a handle allocates
// its tables and buffers) and no allocation of any kind: its scratch lives in the file-scope
// array below, which every GPU that loads this library keeps until the process exits.
// ---------------------------------------------------------------------------------------

#define NOALLOC_PARTS (MP_NOALLOC_MAX_COUNT / FS_TILE)    // one partial per stats CTA
static_assert(MP_NOALLOC_MAX_COUNT % FS_TILE == 0, "the scratch limit must be whole stats tiles");
static_assert((u64)NOALLOC_PARTS * FS_TILE >= MP_NOALLOC_MAX_COUNT, "one partial per CTA of the largest call");

struct NoallocScratch {
    FermPart parts[NOALLOC_PARTS];                          // 384 KB
    u64 hits[16];
    u64 nhits;
};

static __device__ __align__(256) NoallocScratch g_noalloc_scratch;

// The host sees g_noalloc_scratch only as a stand-in symbol: its device address is looked up
// once per device with cudaGetSymbolAddress (with that device current) and kept here.  A
// device reset between calls would move the array; that is not supported.
static std::mutex g_noalloc_mu;
static void *g_noalloc_ptr[64] = {nullptr};

// the hit list and its count carry over from the previous call: empty slots hold 2^64 - 1
__global__ void noalloc_clear_kernel(NoallocScratch *s)
{
    if (threadIdx.x < 16) s->hits[threadIdx.x] = ~0ull;
    if (threadIdx.x == 0) s->nhits = 0;
}

__global__ void noalloc_count_kernel(mp_wief_stats *out, u64 count) { out->primes = count; }

extern "C" int mp_wieferich_stats_noalloc(const uint64_t *d_p, const uint64_t *d_q, uint64_t count,
                                           mp_wief_stats *d_stats, void *stream)
{
    if (!d_stats || (count && (!d_p || !d_q))) return MP_EINVAL;
    if (count > MP_NOALLOC_MAX_COUNT) return MP_EINVAL;    // beyond the fixed scratch
    // an error already pending in this thread belongs to the caller: leave it for the caller
    // to read, and run nothing
    if (cudaPeekAtLastError() != cudaSuccess) return MP_ECUDA;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= 64) return MP_ECUDA;
    NoallocScratch *s = nullptr;
    {
        std::lock_guard<std::mutex> lk(g_noalloc_mu);
        if (!g_noalloc_ptr[dev]) {
            void *p = nullptr;
            if (cudaGetSymbolAddress(&p, g_noalloc_scratch) != cudaSuccess || !p) {
                cudaGetLastError();                          // this call's own failure
                return MP_ECUDA;
            }
            g_noalloc_ptr[dev] = p;
        }
        s = (NoallocScratch *)g_noalloc_ptr[dev];
    }
    cudaStream_t st = (cudaStream_t)stream;
    // every launch is checked; a failure here is this call's own, so it is cleared
#define NOALLOC_CHECK()                                                                       \
    do {                                                                                      \
        if (cudaPeekAtLastError() != cudaSuccess) { cudaGetLastError(); return MP_ECUDA; }   \
    } while (0)
    noalloc_clear_kernel<<<1, 32, 0, st>>>(s);
    NOALLOC_CHECK();
    const u64 nb = count ? (count + FS_TILE - 1) / FS_TILE : 0;
    if (count) {
        fermat_stats_kernel<<<(unsigned)nb, FS_THREADS, 0, st>>>(d_p, d_q, count, s->parts, s->hits, &s->nhits);
        NOALLOC_CHECK();
    } else if (cudaMemsetAsync(s->parts, 0, sizeof(FermPart), st) != cudaSuccess) {
        cudaGetLastError();
        return MP_ECUDA;                                     // no input: one empty partial
    }
    fermat_final_kernel<<<1, 1024, 0, st>>>(s->parts, nb ? nb : 1, &s->nhits, s->hits, d_stats);
    NOALLOC_CHECK();
    noalloc_count_kernel<<<1, 1, 0, st>>>(d_stats, count);
    NOALLOC_CHECK();
#undef NOALLOC_CHECK
    return MP_OK;
}
