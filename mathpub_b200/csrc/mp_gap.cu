// mp_gap.cu -- statistics of the prime-gap stream (include/mathpub_gpu.h, gap statistics):
// the histogram of the gaps that follow the primes of a range, from which A252768's power
// sums come, and the run lengths of A158939 (L(p) = the number of strictly increasing gaps
// that follow p, A158939/a158939.c:17-30) with the smallest prime of each length.
//
// The range is sieved a chunk at a time (2^34 integers) into the odd-only bitmap, with a
// look-ahead of 2^16 integers past the chunk, and gap_kernel reads the bitmap: each CTA takes
// 2^16 bits plus 2^15 bits of look-ahead, compacts the prime positions into shared memory in
// order, and every thread takes primes of the segment, reads the gap to the next prime and
// walks on while the gaps increase (L(p) depends only on the gaps after p, the fact (F1) of
// A158939/a158939.c:32-35, so segments need nothing from each other).  The same walk gives
// the chains of gapchain_ps (gapchain/gapchain_ps.c:336-366): from a head p the gaps 2, 4,
// 6, ..., that is 1, 2, 3, ... bits of the odd-only map.  Counts go to shared histograms
// and then to the device accumulator with one atomic per bin; chain heads of at least the
// requested length go to a device list.
#include "mp_common.cuh"
#include <algorithm>

#define GAP_SEG_BITS 65536u                 // bits of the odd-only map per CTA
#define GAP_LOOK_BITS 32768u                // look-ahead: 2^16 integers
#define GAP_WORDS ((GAP_SEG_BITS + GAP_LOOK_BITS) / 32)
#define GAP_MAXP 20480u                     // primes per CTA window; the densest window, the odd
                                            // numbers below 196608, holds 17,700
#define GAP_THREADS 512
#define GAP_CHUNK ((u64)1 << 34)            // integers sieved per pass
#define GAP_LOOK ((u64)1 << 16)

struct ChainOut {
    u32 min_len;                            // list heads with at least this many primes (0: none)
    u64 cap;
    u64 *heads;
    u32 *lens;
    unsigned long long *n;
};

__global__ void __launch_bounds__(GAP_THREADS) gap_kernel(const u32 *__restrict__ bm, u64 nbits_in, u64 nbits_all,
                                                          u64 base, mp_gap_stats *acc, u32 *err, ChainOut co)
{
    extern __shared__ __align__(16) u32 gsm[];
    u32 *w = gsm;                           // GAP_WORDS words of the map
    u32 *P = gsm + GAP_WORDS;               // GAP_MAXP prime positions (bits from the segment start)
    __shared__ u32 hist[MP_GAP_BINS], rh[MP_RUN_MAX], rf[MP_RUN_MAX], ch[MP_CHAIN_MAX], s_wsum[GAP_THREADS / 32];
    __shared__ u32 s_uns;
    const u32 tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const u64 seg0 = (u64)blockIdx.x * GAP_SEG_BITS;
    for (u32 i = tid; i < GAP_WORDS; i += GAP_THREADS) {       // zero at and past the sieved bits
        const u64 b = seg0 + 32ull * i;
        u32 v = 0;
        if (b < nbits_all) {
            v = __ldg(bm + (b >> 5));
            if (b + 32 > nbits_all) v &= (1u << (u32)(nbits_all - b)) - 1u;
        }
        w[i] = v;
    }
    for (u32 i = tid; i < MP_GAP_BINS; i += GAP_THREADS) hist[i] = 0;
    if (tid < MP_RUN_MAX) { rh[tid] = 0; rf[tid] = 0xffffffffu; }
    if (tid < MP_CHAIN_MAX) ch[tid] = 0;
    if (tid == 0) s_uns = 0;
    __syncthreads();
    // compaction in order: thread t owns words [t wpt, (t + 1) wpt)
    constexpr u32 wpt = GAP_WORDS / GAP_THREADS;
    u32 c = 0;
#pragma unroll
    for (u32 k = 0; k < wpt; k++) c += __popc(w[tid * wpt + k]);
    u32 incl = c;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const u32 v = __shfl_up_sync(0xffffffffu, incl, d);
        if (lane >= (u32)d) incl += v;
    }
    if (lane == 31) s_wsum[warp] = incl;
    __syncthreads();
    if (warp == 0) {
        const u32 v = lane < GAP_THREADS / 32 ? s_wsum[lane] : 0u;
        u32 iv = v;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const u32 u = __shfl_up_sync(0xffffffffu, iv, d);
            if (lane >= (u32)d) iv += u;
        }
        if (lane < GAP_THREADS / 32) s_wsum[lane] = iv;         // inclusive warp totals
    }
    __syncthreads();
    const u32 total = s_wsum[GAP_THREADS / 32 - 1];
    u32 pos = (warp ? s_wsum[warp - 1] : 0u) + incl - c;
#pragma unroll
    for (u32 k = 0; k < wpt; k++) {
        u32 y = w[tid * wpt + k];
        while (y) {
            const u32 b = __ffs(y) - 1;
            y &= y - 1;
            if (pos < GAP_MAXP) P[pos] = (tid * wpt + k) * 32 + b;
            pos++;
        }
    }
    if (tid == 0 && total > GAP_MAXP) atomicOr(err, 8u);
    __syncthreads();
    const u32 n = total < GAP_MAXP ? total : GAP_MAXP;
    // the primes of this segment in [lo, hi): gap to the next prime, then the run
    for (u32 i = tid; i < n; i += GAP_THREADS) {
        const u32 p = P[i];
        if (p >= GAP_SEG_BITS || seg0 + p >= nbits_in) continue;
        if (i + 1 >= n) { atomicAdd(&s_uns, 1u); continue; }
        const u32 g1 = P[i + 1] - p;                            // the gap / 2 (every gap < 2048)
        atomicAdd(&hist[g1 < MP_GAP_BINS ? g1 : MP_GAP_BINS - 1], 1u);
        // chain: the m-th gap after p is 2m integers = m bits
        u32 cl = 1, jc = i;
        while (jc + 1 < n && P[jc + 1] - P[jc] == cl) { cl++; jc++; }
        if (jc + 1 >= n) atomicAdd(&s_uns, 1u);                 // still a chain at the window end
        else {
            atomicAdd(&ch[cl < MP_CHAIN_MAX ? cl : MP_CHAIN_MAX - 1], 1u);
            if (co.min_len && cl >= co.min_len) {
                const unsigned long long k = atomicAdd(co.n, 1ull);
                if (k < co.cap) {
                    co.heads[k] = base + 2 * (seg0 + p) + 1;
                    co.lens[k] = cl < MP_CHAIN_MAX ? cl : MP_CHAIN_MAX - 1;
                }
            }
        }
        u32 L = 1, j = i + 1, gp = g1;
        bool ended = false;
        while (j + 1 < n) {
            const u32 g = P[j + 1] - P[j];
            if (g <= gp) { ended = true; break; }
            L++;
            gp = g;
            j++;
        }
        if (!ended) { atomicAdd(&s_uns, 1u); continue; }
        const u32 l = L < MP_RUN_MAX ? L : MP_RUN_MAX - 1;
        atomicAdd(&rh[l], 1u);
        atomicMin(&rf[l], p);
    }
    __syncthreads();
    for (u32 i = tid; i < MP_GAP_BINS; i += GAP_THREADS)
        if (hist[i]) atomicAdd((unsigned long long *)&acc->gap_hist[i], (unsigned long long)hist[i]);
    if (tid < MP_RUN_MAX && rh[tid]) {
        atomicAdd((unsigned long long *)&acc->run_hist[tid], (unsigned long long)rh[tid]);
        atomicMin((unsigned long long *)&acc->run_first[tid], (unsigned long long)(base + 2 * (seg0 + rf[tid]) + 1));
    }
    if (tid < MP_CHAIN_MAX && ch[tid]) atomicAdd((unsigned long long *)&acc->chain_hist[tid], (unsigned long long)ch[tid]);
    if (tid == 0 && s_uns) atomicAdd((unsigned long long *)&acc->unsettled, (unsigned long long)s_uns);
}

// sieve [lo, hi) a chunk at a time and run gap_kernel over it; the accumulator and the chain
// list stay on the device (the caller copies them)
static int gap_run(mp_handle *h, u64 lo, u64 hi, mp_gap_stats *acc, ChainOut co, cudaStream_t st)
{
    const size_t smem = (size_t)(GAP_WORDS + GAP_MAXP) * 4;
    MP_CUDA(h, cudaFuncSetAttribute(gap_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem));
    MP_CUDA(h, cudaMemsetAsync(acc, 0, sizeof(mp_gap_stats), st));
    MP_CUDA(h, cudaMemsetAsync(acc->run_first, 0xff, sizeof acc->run_first, st));
    MP_CUDA(h, h->small_out.ensure(256));
    mp_sieve_opts o;
    memset(&o, 0, sizeof o);
    o.mode = MP_MODE_BATCHED;
    for (u64 c = lo; c < hi;) {
        const u64 c1 = hi - c > GAP_CHUNK ? c + GAP_CHUNK : hi;
        const u64 ext = c1 + GAP_LOOK;
        const u64 base = c & ~1ull;
        const u64 nbits_all = (ext - base) >> 1, nbits_in = (c1 - base) >> 1;
        MP_CUDA(h, h->scratch_bitmap.ensure((size_t)((nbits_all + 63) >> 6) * 8 + 64));
        MP_TRY(mp_sieve_run(h, c, ext, &o, h->small_out.as<mp_range_stats>(), nullptr, nullptr,
                            h->scratch_bitmap.as<u64>(), st));
        const u64 nseg = (nbits_in + GAP_SEG_BITS - 1) / GAP_SEG_BITS;
        if (nseg) {
            gap_kernel<<<(unsigned)nseg, GAP_THREADS, smem, st>>>(h->scratch_bitmap.as<u32>(), nbits_in, nbits_all, base,
                                                                  acc, h->errflag.as<u32>(), co);
            MP_CUDA(h, cudaGetLastError());
        }
        c = c1;
    }
    return MP_OK;
}

// the prime 2 is outside the odd-only map: its gap is 1; 1 < 2 (3 -> 5) >= 2 (5 -> 7) gives
// L(2) = 2; and no chain starts with the gap 1
static void add_two(mp_gap_stats *out, u64 lo, u64 hi)
{
    if (lo <= 2 && 2 < hi) {
        out->gap_hist[0]++;
        out->run_hist[2]++;
        if (out->run_first[2] > 2) out->run_first[2] = 2;
        out->chain_hist[1]++;
    }
    for (int l = 0; l < MP_RUN_MAX; l++)
        if (out->run_first[l] == ~0ull) out->run_first[l] = 0;
}

extern "C" int mp_gap_stats_range(mp_handle *h, uint64_t lo, uint64_t hi, mp_gap_stats *out)
{
    if (!h || !out) return MP_EINVAL;
    memset(out, 0, sizeof *out);
    if (hi <= lo) return MP_OK;
    std::lock_guard<std::recursive_mutex> lk(h->mu);
    if (hi > MP_HI_MAX - 2 * GAP_LOOK) return mp_set_error(h, MP_ERANGE, "hi must be <= 2^64 - 2^18 - 2^17");
    MP_CUDA(h, cudaSetDevice(h->device));
    cudaStream_t st = h->stream;
    MP_CUDA(h, h->gap_acc.ensure(sizeof(mp_gap_stats) + 64));
    mp_gap_stats *acc = h->gap_acc.as<mp_gap_stats>();
    ChainOut co;
    memset(&co, 0, sizeof co);
    MP_TRY(gap_run(h, lo, hi, acc, co, st));
    MP_CUDA(h, cudaMemcpyAsync(out, acc, sizeof *out, cudaMemcpyDeviceToHost, st));
    MP_TRY(mp_sieve_errors(h, st));                      // synchronises
    add_two(out, lo, hi);
    return MP_OK;
}

extern "C" int mp_gap_chains(mp_handle *h, uint64_t lo, uint64_t hi, uint32_t min_len, uint64_t *heads, uint32_t *lens,
                             size_t cap, size_t *count)
{
    if (!h || !count || (cap && (!heads || !lens))) return MP_EINVAL;
    *count = 0;
    if (min_len < 2) return mp_set_error(h, MP_EINVAL, "min_len must be at least 2");
    if (hi <= lo) return MP_OK;
    std::lock_guard<std::recursive_mutex> lk(h->mu);
    if (hi > MP_HI_MAX - 2 * GAP_LOOK) return mp_set_error(h, MP_ERANGE, "hi must be <= 2^64 - 2^18 - 2^17");
    MP_CUDA(h, cudaSetDevice(h->device));
    cudaStream_t st = h->stream;
    MP_CUDA(h, h->gap_acc.ensure(sizeof(mp_gap_stats) + 64));
    mp_gap_stats *acc = h->gap_acc.as<mp_gap_stats>();
    // the list: cap entries (at least one, so that the device pointers are valid)
    const u64 dcap = cap ? cap : 1;
    MP_CUDA(h, h->ferm_p.ensure((size_t)dcap * 12 + 64));
    ChainOut co;
    co.min_len = min_len;
    co.cap = cap;
    co.heads = h->ferm_p.as<u64>();
    co.lens = (u32 *)(co.heads + dcap);
    co.n = (unsigned long long *)((char *)h->gap_acc.p + sizeof(mp_gap_stats));
    MP_CUDA(h, cudaMemsetAsync(co.n, 0, 8, st));
    MP_TRY(gap_run(h, lo, hi, acc, co, st));
    u64 n = 0;
    MP_CUDA(h, cudaMemcpyAsync(&n, co.n, 8, cudaMemcpyDeviceToHost, st));
    MP_TRY(mp_sieve_errors(h, st));                      // synchronises
    const u64 m = n < cap ? n : cap;
    std::vector<u64> hd(m);
    std::vector<u32> ln(m);
    if (m) {
        MP_CUDA(h, cudaMemcpyAsync(hd.data(), co.heads, m * 8, cudaMemcpyDeviceToHost, st));
        MP_CUDA(h, cudaMemcpyAsync(ln.data(), co.lens, m * 4, cudaMemcpyDeviceToHost, st));
        MP_CUDA(h, cudaStreamSynchronize(st));
    }
    // the device appends in arbitrary order: sort by head (only when the list is complete is
    // the order of a partial list meaningful, so a partial list is sorted as found)
    std::vector<u64> ord(m);
    for (u64 i = 0; i < m; i++) ord[i] = i;
    std::sort(ord.begin(), ord.end(), [&](u64 x, u64 y) { return hd[x] < hd[y]; });
    for (u64 i = 0; i < m; i++) { heads[i] = hd[ord[i]]; lens[i] = ln[ord[i]]; }
    *count = (size_t)n;
    return MP_OK;
}
