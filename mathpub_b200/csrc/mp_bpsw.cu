// mp_bpsw.cu -- 64-bit BPSW primality test for B200 (sm_100a): batches of candidate lists.
//
// Reference (paths inside the Mathpub project): bpsw A350826/a350826.c:965 (the base-2 strong
// test sprp2_64 :618 and the strong Lucas test slprp64 :766 with Selfridge's D :739), after
// the trivial small-factor handling of is_prime_ref :529; the breadth-first batching of
// test_batch64 :1392.  The arithmetic and the two tests are in mp_mont64.cuh.  Trial division
// by the odd primes up to 127 uses the multiplicative-inverse test (q | r iff r q^-1 mod 2^32
// <= (2^32 - 1) / q, for odd q) on n's remainders modulo six products of them, all 30 primes
// for every candidate, with no early exit.  The
// verdict is primality for every n < 2^64 (BPSW has no pseudoprime below 2^64).
//
// Two launch structures:
//   plain    one launch per candidate list, one thread per candidate, all phases inline;
//   batched  one persistent launch over every list: warps pop chunks of candidates from a
//            device work queue, trial-divide them, and file the survivors in two size classes
//            (below 2^63 and above; mp_mont64.cuh runs a different ladder step for each).
//            Each class runs the base-2 test in batches of 32 that are uniform in kind and
//            nearly so in exponent length, the passers are compacted with warp
//            ballots and appended to the launch's Lucas list, and the warp writes the chunk's
//            verdict words.  Warps never wait for one another.  Two more launches then run
//            the Lucas test over the whole list, one passer per thread: Selfridge's search
//            files the passers by D (D = 5 apart), and the ladders set the bits of the primes,
//            those with D = 5 in a two-product step.  (Run inside each chunk, the few dozen
//            passers of a chunk left most lanes idle through the Lucas ladder, and the Lucas
//            phase took half of the time for 4% of the candidates.)  The warps per CTA and
//            candidates per chunk are picked by the autotuner.
#include "mp_mont64.cuh"

#define TD_N 30            // odd primes 3..127
#define TD_NG 6            // in six groups whose products are below 2^32

__constant__ u32 c_tdg_prod[TD_NG];      // the groups' products
__constant__ u64 c_tdg_magic[TD_NG];     // floor((2^64 - 1) / product), for the Barrett remainder
__constant__ u32 c_td_inv32[TD_N];       // p^-1 mod 2^32
__constant__ u32 c_td_lim32[TD_N];       // floor((2^32 - 1) / p)
__constant__ u64 c_small_prime_mask[2];   // bit n set iff n < 128 is prime

// ---- trial division ----
// 1 = prime, 0 = composite, -1 = undecided (odd, no factor <= 127, n >= 131^2).  Per group one
// 64-bit Barrett remainder r = n mod (product of the group), then for each prime p of the group
// p | r iff r p^-1 mod 2^32 <= (2^32 - 1) / p: one 32-bit multiply and one compare a prime,
// instead of a 64-bit product and a 64-bit compare
__device__ __forceinline__ int td_verdict(u64 n)
{
    if (n < 128) return (int)((c_small_prime_mask[n >> 6] >> (n & 63)) & 1);
    bool f = !(n & 1);
    const int gsize[TD_NG] = {8, 5, 5, 5, 4, 3};   // 3..23, 29..43, 47..67, 71..89, 97..107, 109..127
    int k = 0;
#pragma unroll
    for (int g = 0; g < TD_NG; g++) {
        const u32 r = mp_mod_barrett(n, c_tdg_prod[g], c_tdg_magic[g]);
#pragma unroll
        for (int j = 0; j < gsize[g]; j++, k++) f |= r * c_td_inv32[k] <= c_td_lim32[k];
    }
    if (f) return 0;
    return n < 131ull * 131ull ? 1 : -1;
}

__device__ __forceinline__ bool bpsw_full(u64 n)
{
    const int v = td_verdict(n);
    if (v >= 0) return v != 0;
    return bpsw_odd(n);
}

// ---- plain form: one thread per candidate of one list ----
__global__ void __launch_bounds__(256) bpsw_plain_kernel(const u64 *__restrict__ n, u32 len, u32 *__restrict__ bits)
{
    const u32 i = blockIdx.x * blockDim.x + threadIdx.x;
    bool v = false;
    if (i < len) v = bpsw_full(__ldg(n + i));
    const u32 b = __ballot_sync(0xffffffffu, v);
    if ((threadIdx.x & 31) == 0 && i < len) bits[i >> 5] = b;
}

// ---- batched form: persistent warps over chunks of the concatenated lists ----
// a work-queue chunk is BPSW_WCHUNK candidates per warp, BPSW_WARPS warps per CTA; the
// autotuner picks among the instantiated pairs (bpsw_batched_launch)

template <int BPSW_WARPS, int BPSW_WCHUNK>
__global__ void __launch_bounds__(BPSW_WARPS * 32) bpsw_batched_kernel(const u64 *__restrict__ n, u64 total,
                                                                       u32 *__restrict__ bits, u32 *queue,
                                                                       u32 *__restrict__ lucas_list)
{
    __shared__ u16 s_idx[BPSW_WARPS][BPSW_WCHUNK];   // survivors below 2^63
    __shared__ u16 s_pas[BPSW_WARPS][BPSW_WCHUNK];   // base-2 passers
    __shared__ u32 s_bits[BPSW_WARPS][BPSW_WCHUNK / 32];
    const u32 lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const u32 lt = (1u << lane) - 1;
    u16 *idx = s_idx[warp], *pas = s_pas[warp];
    u32 *wb = s_bits[warp];
    const u64 nchunks = (total + BPSW_WCHUNK - 1) / BPSW_WCHUNK;
    for (;;) {
        u32 c = 0;
        if (lane == 0) c = atomicAdd(queue, 1u);
        c = __shfl_sync(0xffffffffu, c, 0);
        if (c >= nchunks) break;
        const u64 c0 = (u64)c * BPSW_WCHUNK;
        const u32 len = (u32)(total - c0 < BPSW_WCHUNK ? total - c0 : BPSW_WCHUNK);
        const u64 *nc = n + c0;
        // 1. trial division: verdict words of the decided candidates; survivors filed by size
        //    class: below 2^63 in idx, 2^63 and above in pas (free until the base-2 passers are
        //    collected)
        u32 nm = 0, nw = 0;
        for (u32 base = 0; base < len; base += 32) {
            const u32 i = base + lane;
            const u64 x = i < len ? __ldg(nc + i) : 0;
            const int v = i < len ? td_verdict(x) : 0;
            const u32 pm = __ballot_sync(0xffffffffu, v == 1);
            const int c = spsp2_class(x);
            const bool cm = v < 0 && c == SP_FOLD, cw = v < 0 && c == SP_WIDE;
            const u32 mm = __ballot_sync(0xffffffffu, cm), mw = __ballot_sync(0xffffffffu, cw);
            if (lane == 0) wb[base >> 5] = pm;
            if (cm) idx[nm + __popc(mm & lt)] = (u16)i;
            if (cw) pas[nw + __popc(mw & lt)] = (u16)i;
            nm += __popc(mm);
            nw += __popc(mw);
        }
        __syncwarp();
        // 2. base-2 strong test, one class after the other; the passers are compacted to the
        //    front of pas.  The widest class goes first: it is read from pas, and a batch's
        //    passers are written only after every lane has read its entry (np <= base)
        u32 np = 0;
        for (u32 base = 0; base < nw; base += 32) {
            const u32 k = base + lane;
            const u32 i = k < nw ? pas[k] : 0;
            const bool pass = k < nw && spsp2<SP_WIDE>(mm_setup(__ldg(nc + i)));
            const u32 m = __ballot_sync(0xffffffffu, pass);
            if (pass) pas[np + __popc(m & lt)] = (u16)i;
            np += __popc(m);
            __syncwarp();
        }
        for (u32 base = 0; base < nm; base += 32) {
            const u32 k = base + lane;
            const u32 i = k < nm ? idx[k] : 0;
            const bool pass = k < nm && spsp2<SP_FOLD>(mm_setup(__ldg(nc + i)));
            const u32 m = __ballot_sync(0xffffffffu, pass);
            if (pass) pas[np + __popc(m & lt)] = (u16)i;
            np += __popc(m);
        }
        __syncwarp();
        // 3. the base-2 passers go to the launch's Lucas list (queue[1] counts it), which
        //    bpsw_lucas_kernel works through in full warps once every chunk is done: a chunk
        //    has a few dozen passers, too few to keep a warp's lanes busy through the Lucas
        //    ladder, and their Selfridge searches differ in length
        u32 g = 0;
        if (lane == 0 && np) g = atomicAdd(queue + 1, np);
        g = __shfl_sync(0xffffffffu, g, 0);
        for (u32 k = lane; k < np; k += 32) lucas_list[g + k] = (u32)(c0 + pas[k]);
        __syncwarp();
        const u32 nwords = (len + 31) / 32;
        for (u32 w = lane; w < nwords; w += 32) bits[(c0 >> 5) + w] = wb[w];
        __syncwarp();
    }
}

// The strong Lucas test on the list of base-2 passers of a batched launch (indices into n,
// count at *count), one candidate per thread, in two launches.  Selfridge's search for D, whose
// length differs from candidate to candidate (a few Jacobi symbols, each after a 64-bit
// remainder), files each candidate: D = 5 (about half of them: n = 2 or 3 mod 5) in one list,
// any other D with its value in another; D = 0 (shown composite by the search) in neither.
// Then the Lucas ladders run with the warps' lanes together, the D = 5 list first with its
// two-product step (Q = -1), and a prime's verdict bit is set in its word.  Lists: l5 indices
// (count ctr[0]); lo indices and dl their D (count ctr[1]).
__global__ void __launch_bounds__(256) bpsw_selfridge_kernel(const u64 *__restrict__ n, const u32 *__restrict__ list,
                                                             const u32 *count, u32 *__restrict__ l5,
                                                             u32 *__restrict__ lo, i32 *__restrict__ dl, u32 *ctr)
{
    const u32 cnt = *count, lane = threadIdx.x & 31, lt = (1u << lane) - 1;
    // warp-uniform trip count, so that every lane takes part in the ballots
    for (u32 b0 = blockIdx.x * blockDim.x + (threadIdx.x & ~31u); b0 < cnt; b0 += gridDim.x * blockDim.x) {
        const u32 i = b0 + lane;
        u32 idx = 0;
        i32 D = 0;
        if (i < cnt) {
            idx = list[i];
            const u64 x = __ldg(n + idx);
            D = x == ~0ull ? 0 : selfridge_d(x);                         // 3 | 2^64 - 1
        }
        const u32 m5 = __ballot_sync(0xffffffffu, D == 5), mo = __ballot_sync(0xffffffffu, D != 0 && D != 5);
        u32 g5 = 0, go = 0;
        if (lane == 0) {
            if (m5) g5 = atomicAdd(ctr, (u32)__popc(m5));
            if (mo) go = atomicAdd(ctr + 1, (u32)__popc(mo));
        }
        g5 = __shfl_sync(0xffffffffu, g5, 0);
        go = __shfl_sync(0xffffffffu, go, 0);
        if (D == 5) l5[g5 + __popc(m5 & lt)] = idx;
        else if (D) {
            const u32 k = go + __popc(mo & lt);
            lo[k] = idx;
            dl[k] = D;
        }
    }
}

__global__ void __launch_bounds__(256) bpsw_lucas_kernel(const u64 *__restrict__ n, const u32 *__restrict__ l5,
                                                         const u32 *__restrict__ lo, const i32 *__restrict__ dl,
                                                         const u32 *ctr, u32 *bits)
{
    const u32 c5 = ctr[0], cnt = c5 + ctr[1];
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < cnt; i += gridDim.x * blockDim.x) {
        const bool f = i < c5;
        const u32 idx = f ? l5[i] : lo[i - c5];
        const Mod64 M = mm_setup(__ldg(n + idx));
        if (f ? lucas_strong_d5(M) : lucas_strong(M, dl[i - c5])) atomicOr(bits + (idx >> 5), 1u << (idx & 31));
    }
}

// ---- host side ----

static bool g_bpsw_consts[16] = {false};

static int bpsw_consts(mp_handle *h)
{
    if (h->device >= 0 && h->device < 16 && g_bpsw_consts[h->device]) return MP_OK;
    static const u32 tdp[TD_N] = {3,  5,  7,  11, 13, 17, 19, 23, 29, 31, 37, 41,  43,  47,  53,
                                  59, 61, 67, 71, 73, 79, 83, 89, 97, 101, 103, 107, 109, 113, 127};
    static const int gsize[TD_NG] = {8, 5, 5, 5, 4, 3};
    u32 inv[TD_N], lim[TD_N], prod[TD_NG];
    u64 magic[TD_NG], mask[2] = {0, 0};
    for (int k = 0; k < TD_N; k++) {
        const u32 q = tdp[k];
        inv[k] = (u32)inv64(q);              // q^-1 mod 2^64, so also mod 2^32
        lim[k] = 0xffffffffu / q;
    }
    for (int g = 0, k = 0; g < TD_NG; g++) {
        u64 pr = 1;
        for (int j = 0; j < gsize[g]; j++, k++) pr *= tdp[k];
        if (pr >> 32) return mp_set_error(h, MP_EINVAL, "trial-division group product above 2^32");
        prod[g] = (u32)pr;
        magic[g] = ~0ull / pr;
    }
    for (u32 v = 2; v < 128; v++) {
        bool p = true;
        for (u32 d = 2; d * d <= v; d++) if (v % d == 0) { p = false; break; }
        if (p) mask[v >> 6] |= 1ull << (v & 63);
    }
    MP_CUDA(h, cudaMemcpyToSymbol(c_td_inv32, inv, sizeof inv));
    MP_CUDA(h, cudaMemcpyToSymbol(c_td_lim32, lim, sizeof lim));
    MP_CUDA(h, cudaMemcpyToSymbol(c_tdg_prod, prod, sizeof prod));
    MP_CUDA(h, cudaMemcpyToSymbol(c_tdg_magic, magic, sizeof magic));
    MP_CUDA(h, cudaMemcpyToSymbol(c_small_prime_mask, mask, sizeof mask));
    if (h->device >= 0 && h->device < 16) g_bpsw_consts[h->device] = true;
    return MP_OK;
}

// one persistent launch: as many CTAs as fit on the device, no more than the chunks need;
// then the Lucas launch over the passers it listed
template <int WARPS, int CHUNK>
static cudaError_t bpsw_batched_launch(mp_handle *h, const u64 *d_n, u64 total, u32 *d_bits, u32 *d_list,
                                       u64 lcap, cudaStream_t st)
{
    int per_sm = 0;
    cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bpsw_batched_kernel<WARPS, CHUNK>,
                                                                  WARPS * 32, 0);
    if (e != cudaSuccess) return e;
    if (per_sm < 1) per_sm = 1;
    u64 grid = (u64)h->sm_count * per_sm;
    const u64 nchunks = (total + CHUNK - 1) / CHUNK;
    const u64 need = (nchunks + WARPS - 1) / WARPS;
    if (grid > need) grid = need;
    u32 *queue = h->queue.as<u32>();
    bpsw_batched_kernel<WARPS, CHUNK><<<(unsigned)grid, WARPS * 32, 0, st>>>(d_n, total, d_bits, queue, d_list);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    int lper = 0;
    e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&lper, bpsw_lucas_kernel, 256, 0);
    if (e != cudaSuccess) return e;
    if (lper < 1) lper = 1;
    u64 lgrid = (u64)h->sm_count * lper;
    const u64 lneed = (total + 255) / 256;
    if (lgrid > lneed) lgrid = lneed;
    u32 *l5 = d_list + lcap, *lo = d_list + 2 * lcap;
    i32 *dl = (i32 *)(d_list + 3 * lcap);
    bpsw_selfridge_kernel<<<(unsigned)lgrid, 256, 0, st>>>(d_n, d_list, queue + 1, l5, lo, dl, queue + 2);
    bpsw_lucas_kernel<<<(unsigned)lgrid, 256, 0, st>>>(d_n, l5, lo, dl, queue + 2, d_bits);
    return cudaGetLastError();
}

// lists at d_n + offs[i] (offs multiples of 32, host array of nlists + 1 entries), verdict
// words at d_bits + offs[i] / 32
int mp_bpsw_run(mp_handle *h, const u64 *d_n, const u64 *offs, const u32 *lens, u32 nlists, u32 *d_bits,
                u32 mode, cudaStream_t st)
{
    MP_TRY(bpsw_consts(h));
    if (mode == MP_MODE_PLAIN) {
        for (u32 i = 0; i < nlists; i++) {
            if (!lens[i]) continue;
            if (offs[i] & 31) return mp_set_error(h, MP_EINVAL, "list offsets must be multiples of 32");
            ProfScope ps(h, PROF_BPSW_PLAIN, st);
            bpsw_plain_kernel<<<(lens[i] + 255) / 256, 256, 0, st>>>(d_n + offs[i], lens[i], d_bits + offs[i] / 32);
            MP_CUDA(h, cudaGetLastError());
        }
        return MP_OK;
    }
    const u64 total = offs[nlists];
    if (!total) return MP_OK;
    // slices of at most 2^31 candidates, so that the Lucas list holds 32-bit indices
    const u64 slice = 1ull << 31;
    MP_CUDA(h, h->queue.ensure(64));
    const u64 lcap = std::min(total, slice);
    MP_CUDA(h, h->bpsw_list.ensure((size_t)lcap * 16));         // passers; D = 5 ones; others; their D
    ProfScope ps(h, PROF_BPSW_BATCHED, st);
    for (u64 b = 0; b < total; b += slice) {
        const u64 t = std::min(slice, total - b);
        const u64 *dn = d_n + b;
        u32 *db = d_bits + b / 32, *dl = h->bpsw_list.as<u32>();
        MP_CUDA(h, cudaMemsetAsync(h->queue.p, 0, 16, st));
        switch (h->tune.bpsw_variant) {
        case 1: MP_CUDA(h, (bpsw_batched_launch<4, 1024>(h, dn, t, db, dl, lcap, st))); break;
        case 2: MP_CUDA(h, (bpsw_batched_launch<8, 512>(h, dn, t, db, dl, lcap, st))); break;
        case 3: MP_CUDA(h, (bpsw_batched_launch<16, 512>(h, dn, t, db, dl, lcap, st))); break;
        default: MP_CUDA(h, (bpsw_batched_launch<8, 1024>(h, dn, t, db, dl, lcap, st))); break;
        }
    }
    return MP_OK;
}

const char *mp_bpsw_variant_name(int v)
{
    static const char *names[4] = {"8 warps x 1024 candidates", "4 warps x 1024 candidates",
                                   "8 warps x 512 candidates", "16 warps x 512 candidates"};
    return names[v & 3];
}
