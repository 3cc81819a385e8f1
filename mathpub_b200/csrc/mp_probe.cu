// mp_probe.cu -- measurement utilities: per-kernel timing (mp_profile_*) and microbenchmarks
// of the on-chip rates that bound the kernels here (shared-memory atomics for the sieve,
// 32-bit integer multiply-add for the Montgomery kernels).  These give the roofline
// denominators that a copy-bandwidth or GEMM peak does not.
#include "mp_common.cuh"

// shared-memory atomicOr throughput: 1024 threads, 32768 words; `conflict_free` puts the 32
// lanes of a warp on 32 different banks, otherwise every (thread, iteration) takes an
// independent hashed word, so that the lanes of a warp meet the bank conflicts of uniformly
// random addresses (about 3.5 wavefronts per warp instruction)
__device__ __forceinline__ u32 probe_hash(u32 x)
{
    x ^= x >> 16; x *= 0x7feb352du; x ^= x >> 15; x *= 0x846ca68bu; x ^= x >> 16;
    return x;
}

template <bool CONFLICT_FREE>
__global__ void __launch_bounds__(1024, 1) smem_atomic_probe(u32 iters, u32 *sink)
{
    extern __shared__ u32 sm[];
    const u32 tid = threadIdx.x;
    for (u32 i = tid; i < 32768; i += blockDim.x) sm[i] = 0;
    __syncthreads();
    const u32 seed = (blockIdx.x << 10 | tid) * 0x9E3779B9u;
    for (u32 i = 0; i < iters; i++) {
        u32 idx;
        if (CONFLICT_FREE) idx = (i * 1024u + tid) & 32767u;
        else idx = probe_hash(seed + i) & 32767u;
        atomicOr(&sm[idx], 1u << (i & 31));
    }
    __syncthreads();
    if (tid == 0) atomicAdd(sink, sm[blockIdx.x & 32767]);
}

// 32-bit integer multiply-add throughput: 8 independent chains per thread
__global__ void __launch_bounds__(1024) imad_probe(u32 iters, u32 a, u32 *sink)
{
    u32 x0 = threadIdx.x, x1 = x0 + 1, x2 = x0 + 2, x3 = x0 + 3, x4 = x0 + 4, x5 = x0 + 5, x6 = x0 + 6, x7 = x0 + 7;
    const u32 c = blockIdx.x | 1;
    for (u32 i = 0; i < iters; i++) {
        x0 = x0 * a + c; x1 = x1 * a + c; x2 = x2 * a + c; x3 = x3 * a + c;
        x4 = x4 * a + c; x5 = x5 * a + c; x6 = x6 * a + c; x7 = x7 * a + c;
    }
    const u32 s = x0 ^ x1 ^ x2 ^ x3 ^ x4 ^ x5 ^ x6 ^ x7;
    if (s == 0x12345678u) atomicAdd(sink, 1u);
}

// global atomicOr (no return value) on random words of a buffer of `words` u32 (a power of 2);
// with a buffer well inside the L2 this is the L2 atomic rate
__global__ void __launch_bounds__(256) l2_atomic_probe(u32 *buf, u32 mask, u32 iters)
{
    u32 x = (blockIdx.x * blockDim.x + threadIdx.x) * 2654435761u + 12345u;
    for (u32 i = 0; i < iters; i++) {
        x = x * 1664525u + 1013904223u;
        atomicOr(buf + ((x >> 3) & mask), 1u << (x & 31));
    }
}

extern "C" {

int mp_profile_enable(mp_handle *h, int on)
{
    if (!h) return MP_EINVAL;
    std::lock_guard<std::recursive_mutex> lk(h->mu);
    h->prof_on = on != 0;
    return MP_OK;
}

// per category: launches and summed milliseconds since the last read; names in order
// "scatter tile fold hash bpsw_batched bpsw_plain fermat fermat_stats pipeline"
int mp_profile_read(mp_handle *h, uint64_t *launches, double *ms, int ncat)
{
    if (!h || !launches || !ms) return MP_EINVAL;
    std::lock_guard<std::recursive_mutex> lk(h->mu);
    MP_CUDA(h, cudaSetDevice(h->device));
    for (int c = 0; c < ncat; c++) { launches[c] = 0; ms[c] = 0; }
    for (auto &e : h->prof) {
        MP_CUDA(h, cudaEventSynchronize(e.b));
        float t = 0;
        MP_CUDA(h, cudaEventElapsedTime(&t, e.a, e.b));
        if (e.cat < ncat) { launches[e.cat]++; ms[e.cat] += t; }
        h->prof_pool.push_back(e.a);
        h->prof_pool.push_back(e.b);
    }
    h->prof.clear();
    return MP_OK;
}

// rates in operations per second over the whole device: shared atomicOr with lanes on
// distinct banks, shared atomicOr on random addresses, 32-bit integer multiply-adds
int mp_probe_peaks(mp_handle *h, double *smem_atomic_cf, double *smem_atomic_rand, double *imad, double *l2_atomic)
{
    if (!h) return MP_EINVAL;
    std::lock_guard<std::recursive_mutex> lk(h->mu);
    MP_CUDA(h, cudaSetDevice(h->device));
    cudaStream_t st = h->stream;
    MP_CUDA(h, h->small_out.ensure(4096));
    u32 *sink = h->small_out.as<u32>();
    const int smem = 32768 * 4;
    MP_CUDA(h, cudaFuncSetAttribute(smem_atomic_probe<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    MP_CUDA(h, cudaFuncSetAttribute(smem_atomic_probe<false>, cudaFuncAttributeMaxDynamicSharedMemorySize, smem));
    const u32 it = 1u << 16;
    float ms = 0;
    double r[3];
    for (int k = 0; k < 3; k++) {
        float best = 0;
        for (int rep = 0; rep < 4; rep++) {       // the first pass warms up; best of the others
            MP_CUDA(h, cudaEventRecord(h->ev0, st));
            if (k == 0) smem_atomic_probe<true><<<h->sm_count, 1024, smem, st>>>(it, sink);
            else if (k == 1) smem_atomic_probe<false><<<h->sm_count, 1024, smem, st>>>(it, sink);
            else imad_probe<<<h->sm_count * 2, 1024, 0, st>>>(it, 0x9E3779B1u, sink);
            MP_CUDA(h, cudaGetLastError());
            MP_CUDA(h, cudaEventRecord(h->ev1, st));
            MP_CUDA(h, cudaEventSynchronize(h->ev1));
            MP_CUDA(h, cudaEventElapsedTime(&ms, h->ev0, h->ev1));
            if (rep == 1 || (rep > 1 && ms < best)) best = ms;
        }
        ms = best;
        const double ops = k < 2 ? (double)h->sm_count * 1024.0 * it : (double)h->sm_count * 2 * 1024.0 * it * 8;
        r[k] = ops / (ms * 1e-3);
    }
    // L2 atomics: 2^24 words (64 MB) of scratch
    if (l2_atomic) {
        const u32 words = 1u << 24, iters = 1u << 10;
        MP_CUDA(h, h->scratch_bitmap.ensure((size_t)words * 4));
        MP_CUDA(h, cudaMemsetAsync(h->scratch_bitmap.p, 0, (size_t)words * 4, st));
        const int grid = h->sm_count * 8;
        for (int rep = 0; rep < 2; rep++) {
            MP_CUDA(h, cudaEventRecord(h->ev0, st));
            l2_atomic_probe<<<grid, 256, 0, st>>>(h->scratch_bitmap.as<u32>(), words - 1, iters);
            MP_CUDA(h, cudaGetLastError());
            MP_CUDA(h, cudaEventRecord(h->ev1, st));
            MP_CUDA(h, cudaEventSynchronize(h->ev1));
            MP_CUDA(h, cudaEventElapsedTime(&ms, h->ev0, h->ev1));
        }
        *l2_atomic = (double)grid * 256.0 * iters / (ms * 1e-3);
    }
    if (smem_atomic_cf) *smem_atomic_cf = r[0];
    if (smem_atomic_rand) *smem_atomic_rand = r[1];
    if (imad) *imad = r[2];
    return MP_OK;
}

}  // extern "C"
