// mp_bpsw.cu -- 64-bit Montgomery BPSW primality test for B200 (sm_100a).
//
// Reference (paths inside the Mathpub project): inv64/mmul64/madd64/msub64/mhalf64
// A350826/a350826.c:565-604, sprp2_64 :618-638, jacobi :693, selfridge :739, slprp64
// :766-799, bpsw :965-969, and the breadth-first batching of test_batch64 :1392.
//
// Differences in method, not in results:
//   - R mod n (the Montgomery form of 1) is computed by doubling 2^(bitlen(n)-1) up to 2^64
//     (exact; no division and no floating-point estimate), and the forms of Q and D by
//     double-and-add of that one;
//   - trial division by the odd primes up to 127 uses the multiplicative-inverse test
//     (q | n iff n * q^-1 mod 2^64 <= (2^64 - 1) / q, for odd q) before any exponentiation;
//   - perfect squares are rejected with an exact integer square root.
// The verdict is primality for every n < 2^64 (BPSW has no pseudoprime below 2^64).
//
// Two launch structures:
//   plain    one launch per candidate list, one thread per candidate, all phases inline;
//   batched  one persistent launch over every list: warps pop chunks of 1024 candidates from
//            a device work queue, trial-divide, compact the survivors with warp ballots, run
//            the base-2 test on them, compact the passers, run the Lucas test, and write the
//            verdict words.  Compaction keeps the lanes on uniform work; warps never wait for
//            one another.
#include "mp_mont64.cuh"

#define TD_N 30            // odd primes 3..127

__constant__ u64 c_td_inv[TD_N];
__constant__ u64 c_td_lim[TD_N];
__constant__ u64 c_small_prime_mask[2];   // bit n set iff n < 128 is prime

// ---- trial division ----
// 1 = prime, 0 = composite, -1 = undecided (odd, no factor <= 127, n >= 131^2)
__device__ __forceinline__ int td_verdict(u64 n)
{
    if (n < 128) return (int)((c_small_prime_mask[n >> 6] >> (n & 63)) & 1);
    if (!(n & 1)) return 0;
#pragma unroll
    for (int k = 0; k < TD_N; k++)
        if (n * c_td_inv[k] <= c_td_lim[k]) return 0;
    if (n < 131ull * 131ull) return 1;
    return -1;
}

__device__ __forceinline__ bool bpsw_full(u64 n)
{
    const int v = td_verdict(n);
    if (v >= 0) return v != 0;
    const u64 ni = m_inv(n), one = m_one(n);
    return sprp2_dev(n, ni, one) && slprp_dev(n, ni, one);
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
// Each warp pops chunks of BPSW_WCHUNK candidates from the device work queue and runs the
// three phases on them with ballot compaction in between, so its lanes stay on uniform work;
// warps never wait for each other (no CTA barrier).
#define BPSW_WCHUNK 1024
#define BPSW_WARPS 8

__global__ void __launch_bounds__(BPSW_WARPS * 32) bpsw_batched_kernel(const u64 *__restrict__ n, u64 total,
                                                                       u32 *__restrict__ bits, u32 *queue)
{
    __shared__ u16 s_idx[BPSW_WARPS][BPSW_WCHUNK];
    __shared__ u32 s_bits[BPSW_WARPS][BPSW_WCHUNK / 32];
    const u32 lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const u32 lt = (1u << lane) - 1;
    u16 *idx = s_idx[warp];
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
        // 1. trial division; verdict words for the decided candidates, survivors compacted
        u32 ns = 0;
        for (u32 base = 0; base < len; base += 32) {
            const u32 i = base + lane;
            const u64 x = i < len ? __ldg(nc + i) : 0;
            const int v = i < len ? td_verdict(x) : 0;
            const u32 pm = __ballot_sync(0xffffffffu, v == 1);
            const u32 um = __ballot_sync(0xffffffffu, v < 0);
            if (lane == 0) wb[base >> 5] = pm;
            if (v < 0) idx[ns + __popc(um & lt)] = (u16)i;
            ns += __popc(um);
        }
        __syncwarp();
        // 2. base-2 strong test on the survivors; passers compacted to the front of idx
        u32 nl = 0;
        for (u32 base = 0; base < ns; base += 32) {
            const u32 k = base + lane;
            const bool act = k < ns;
            const u32 i = act ? idx[k] : 0;
            bool pass = false;
            if (act) {
                const u64 x = __ldg(nc + i);
                pass = sprp2_dev(x, m_inv(x), m_one(x));
            }
            const u32 m = __ballot_sync(0xffffffffu, pass);   // every lane has read idx[k]
            if (pass) idx[nl + __popc(m & lt)] = (u16)i;
            nl += __popc(m);
            __syncwarp();
        }
        // 3. strong Lucas test on the base-2 passers
        for (u32 base = 0; base < nl; base += 32) {
            const u32 k = base + lane;
            if (k < nl) {
                const u32 i = idx[k];
                const u64 x = __ldg(nc + i);
                if (slprp_dev(x, m_inv(x), m_one(x))) atomicOr(&wb[i >> 5], 1u << (i & 31));
            }
        }
        __syncwarp();
        const u32 nw = (len + 31) / 32;
        for (u32 w = lane; w < nw; w += 32) bits[(c0 >> 5) + w] = wb[w];
        __syncwarp();
    }
}

// ---- host side ----

static bool g_bpsw_consts[16] = {false};

static int bpsw_consts(mp_handle *h)
{
    if (h->device >= 0 && h->device < 16 && g_bpsw_consts[h->device]) return MP_OK;
    static const u32 tdp[TD_N] = {3,  5,  7,  11, 13, 17, 19, 23, 29, 31, 37, 41,  43,  47,  53,
                                  59, 61, 67, 71, 73, 79, 83, 89, 97, 101, 103, 107, 109, 113, 127};
    u64 inv[TD_N], lim[TD_N], mask[2] = {0, 0};
    for (int k = 0; k < TD_N; k++) {
        const u64 q = tdp[k];
        u64 x = (3 * q) ^ 2;
        for (int i = 0; i < 4; i++) x *= 2 - q * x;
        inv[k] = x;
        lim[k] = ~0ull / q;
    }
    for (u32 v = 2; v < 128; v++) {
        bool p = true;
        for (u32 d = 2; d * d <= v; d++) if (v % d == 0) { p = false; break; }
        if (p) mask[v >> 6] |= 1ull << (v & 63);
    }
    MP_CUDA(h, cudaMemcpyToSymbol(c_td_inv, inv, sizeof inv));
    MP_CUDA(h, cudaMemcpyToSymbol(c_td_lim, lim, sizeof lim));
    MP_CUDA(h, cudaMemcpyToSymbol(c_small_prime_mask, mask, sizeof mask));
    if (h->device >= 0 && h->device < 16) g_bpsw_consts[h->device] = true;
    return MP_OK;
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
    MP_CUDA(h, h->queue.ensure(64));
    MP_CUDA(h, cudaMemsetAsync(h->queue.p, 0, 4, st));
    int per_sm = 0;
    MP_CUDA(h, cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, bpsw_batched_kernel, BPSW_WARPS * 32, 0));
    if (per_sm < 1) per_sm = 1;
    u64 grid = (u64)h->sm_count * per_sm;
    const u64 nchunks = (total + BPSW_WCHUNK - 1) / BPSW_WCHUNK;
    const u64 need = (nchunks + BPSW_WARPS - 1) / BPSW_WARPS;
    if (grid > need) grid = need;
    ProfScope ps(h, PROF_BPSW_BATCHED, st);
    bpsw_batched_kernel<<<(unsigned)grid, BPSW_WARPS * 32, 0, st>>>(d_n, total, d_bits, h->queue.as<u32>());
    MP_CUDA(h, cudaGetLastError());
    return MP_OK;
}
