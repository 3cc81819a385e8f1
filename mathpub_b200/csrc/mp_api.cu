// mp_api.cu -- the extern "C" entry points of libmathpub (see include/mathpub_gpu.h): handles,
// errors, host-buffer wrappers around the device kernels, CUDA-graph replay of repeated
// batched sieve calls, and the autotuner.
#include "mp_common.cuh"
#include <algorithm>
#include <chrono>
#include <stdarg.h>

int mp_set_error(mp_handle *h, int code, const char *fmt, ...)
{
    if (h) {
        va_list ap;
        va_start(ap, fmt);
        vsnprintf(h->err, sizeof h->err, fmt, ap);
        va_end(ap);
    }
    return code;
}

// ---------------------------------------------------------------------------------------
// graph cache: one captured graph per distinct batched sieve call signature (last 8 kept)
// ---------------------------------------------------------------------------------------

struct GraphKey {
    u64 lo, hi;
    mp_sieve_opts o;
    void *out, *blocks, *hash, *bitmap;
    cudaStream_t st;
    u64 tune_gen;                    // the tuned plan (tile, threads, scatter form, threshold) it ran with
    bool operator==(const GraphKey &k) const
    {
        return lo == k.lo && hi == k.hi && !memcmp(&o, &k.o, sizeof o) && out == k.out && blocks == k.blocks &&
               hash == k.hash && bitmap == k.bitmap && st == k.st && tune_gen == k.tune_gen;
    }
};

struct GraphEntry {
    GraphKey key;
    cudaGraphExec_t exec = nullptr;
    u64 stamp = 0;
    u64 gen = 0;                     // buffer generation the graph's pointers belong to
};

struct GraphCache {
    GraphEntry e[8];
    u64 clock = 0;
};

void mp_graphs_free(mp_handle *h)
{
    if (!h->graphs) return;
    for (auto &g : h->graphs->e)
        if (g.exec) cudaGraphExecDestroy(g.exec);
    delete h->graphs;
    h->graphs = nullptr;
}


extern "C" {

int mp_version(void) { return 100; }

int mp_init(int device, mp_handle **out)
{
    if (!out) return MP_EINVAL;
    *out = nullptr;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0) return MP_ECUDA;
    if (device < 0 || device >= ndev) return MP_EINVAL;
    mp_handle *h = new (std::nothrow) mp_handle();
    if (!h) return MP_ENOMEM;
    h->device = device;
    cudaError_t e = cudaSetDevice(device);
    if (e == cudaSuccess) e = cudaDeviceGetAttribute(&h->sm_count, cudaDevAttrMultiProcessorCount, device);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&h->stream, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaEventCreate(&h->ev0);
    if (e == cudaSuccess) e = cudaEventCreate(&h->ev1);
    if (e == cudaSuccess) e = cudaMallocHost(&h->h_err, 64);
    if (e == cudaSuccess) e = h->errflag.ensure(64);
    if (e == cudaSuccess) e = cudaMemset(h->errflag.p, 0, 64);
    if (e != cudaSuccess) {
        delete h;
        return MP_ECUDA;
    }
    h->graphs = new GraphCache();
    DevBuf *bufs[] = {&h->tilesum, &h->blockacc, &h->rec, &h->reccnt, &h->queue, &h->errflag, &h->scratch_bitmap,
                      &h->bpsw_n, &h->bpsw_bits, &h->bpsw_list, &h->ferm_p, &h->ferm_q, &h->ferm_part, &h->stats_out, &h->small_out,
                      &h->boot.q, &h->boot.magic, &h->table.q, &h->table.magic, &h->tstate, &h->gap_acc};
    for (DevBuf *b : bufs) b->gen = &h->buf_gen;
    for (auto &e : h->scat) e.buf.gen = &h->buf_gen;
    *out = h;
    return MP_OK;
}

int mp_free(mp_handle *h)
{
    if (!h) return MP_EINVAL;
    cudaSetDevice(h->device);
    if (h->stream) cudaStreamSynchronize(h->stream);
    mp_graphs_free(h);
    mp_chain_free(h);
    DevBuf *bufs[] = {&h->tilesum, &h->blockacc, &h->rec, &h->reccnt, &h->queue, &h->errflag, &h->scratch_bitmap,
                      &h->bpsw_n, &h->bpsw_bits, &h->bpsw_list, &h->ferm_p, &h->ferm_q, &h->ferm_part, &h->stats_out, &h->small_out,
                      &h->boot.q, &h->boot.magic, &h->table.q, &h->table.magic, &h->tstate, &h->gap_acc};
    for (DevBuf *b : bufs) b->release();
    for (auto &e : h->scat) e.buf.release();
    for (int p = 0; p < MP_NPAT; p++)
        if (!h->shared_tables && h->pat_ready && h->pat.d_words[p]) cudaFree(h->pat.d_words[p]);
    if (h->h_err) cudaFreeHost(h->h_err);
    if (h->ev0) cudaEventDestroy(h->ev0);
    if (h->ev1) cudaEventDestroy(h->ev1);
    if (h->stream) cudaStreamDestroy(h->stream);
    delete h;
    return MP_OK;
}

const char *mp_last_error(const mp_handle *h) { return h ? h->err : "null handle"; }

double mp_last_kernel_ms(const mp_handle *h) { return h ? h->last_ms : 0.0; }

uint64_t mp_sieve_nblocks(uint64_t lo, uint64_t hi, uint32_t block_log2)
{
    if (hi <= lo || !block_log2 || block_log2 > 63) return 0;
    return ((hi - lo - 1) >> block_log2) + 1;
}

uint64_t mp_sieve_nhashes(uint64_t lo, uint64_t hi, uint32_t hash_log2)
{
    if (hi <= lo || hash_log2 < 4 || hash_log2 > 40) return 0;
    const u64 nbits = (hi - (lo & ~1ull)) >> 1, sb = 1ull << (hash_log2 - 1);
    return (nbits + sb - 1) / sb;
}

uint64_t mp_sieve_nwords(uint64_t lo, uint64_t hi)
{
    if (hi <= lo) return 0;
    return (((hi - (lo & ~1ull)) >> 1) + 63) >> 6;
}

// ---- sieve ----

int mp_sieve_range_dev(mp_handle *h, uint64_t lo, uint64_t hi, const mp_sieve_opts *opts, mp_range_stats *d_out,
                       mp_block_stats *d_blocks, uint64_t *d_hash, uint64_t *d_bitmap, void *stream)
{
    if (!h) return MP_EINVAL;
    std::lock_guard<std::recursive_mutex> lk(h->mu);
    MP_CUDA(h, cudaSetDevice(h->device));
    cudaStream_t st = mp_stream_of(h, stream);
    mp_sieve_opts o;
    memset(&o, 0, sizeof o);
    if (opts) o = *opts;
    if (o.hash_log2 && !d_hash) return mp_set_error(h, MP_EINVAL, "hash_log2 set but no hash buffer");
    if (o.mode == MP_MODE_PLAIN || h->prof_on || h->no_graphs)
        return mp_sieve_run(h, lo, hi, &o, d_out, d_blocks, d_hash, d_bitmap, st);
    // batched: replay a captured graph of an identical earlier call.  The tables are built
    // before capture (they synchronise), so the graph holds kernel launches and memsets only.
    if (hi > lo && hi <= MP_HI_MAX) MP_TRY(mp_tables_ensure(h, mp_isqrt64(hi + MP_TAIL - 1)));
    GraphKey key;
    memset(&key, 0, sizeof key);
    key.lo = lo; key.hi = hi; key.o = o; key.out = d_out; key.blocks = d_blocks; key.hash = d_hash;
    key.bitmap = d_bitmap; key.st = st; key.tune_gen = h->tune_gen;
    GraphCache *gc = h->graphs;
    for (auto &g : gc->e)
        if (g.exec && g.key == key && g.gen == h->buf_gen) {
            g.stamp = ++gc->clock;
            MP_CUDA(h, cudaGraphLaunch(g.exec, st));
            return MP_OK;
        }
    // first call with this signature: run it directly (sizes buffers), then capture for reuse
    MP_TRY(mp_sieve_run(h, lo, hi, &o, d_out, d_blocks, d_hash, d_bitmap, st));
    cudaStreamCaptureStatus cs;
    MP_CUDA(h, cudaStreamIsCapturing(st, &cs));
    if (cs != cudaStreamCaptureStatusNone) return MP_OK;   // the caller is capturing
    cudaGraph_t graph = nullptr;
    const u64 gen0 = h->buf_gen;
    MP_CUDA(h, cudaStreamBeginCapture(st, cudaStreamCaptureModeThreadLocal));
    const int r = mp_sieve_run(h, lo, hi, &o, d_out, d_blocks, d_hash, d_bitmap, st);
    const cudaError_t ce = cudaStreamEndCapture(st, &graph);
    if (r != MP_OK || ce != cudaSuccess || !graph || h->buf_gen != gen0) {
        if (graph) cudaGraphDestroy(graph);
        cudaGetLastError();
        return MP_OK;   // the direct run above already produced the results
    }
    // the direct run already produced the results; keep the graph for the next call
    GraphEntry *slot = &gc->e[0];
    for (auto &g : gc->e) {
        if (!g.exec) { slot = &g; break; }
        if (g.stamp < slot->stamp) slot = &g;
    }
    if (slot->exec) cudaGraphExecDestroy(slot->exec);
    slot->exec = nullptr;
    cudaGraphExec_t exec = nullptr;
    const cudaError_t ie = cudaGraphInstantiate(&exec, graph, 0);
    cudaGraphDestroy(graph);
    if (ie == cudaSuccess) {
        slot->exec = exec;
        slot->key = key;
        slot->stamp = ++gc->clock;
        slot->gen = gen0;
    } else cudaGetLastError();
    return MP_OK;
}

int mp_sieve_range(mp_handle *h, uint64_t lo, uint64_t hi, const mp_sieve_opts *opts, mp_range_stats *out,
                   mp_block_stats *blocks, uint64_t *seg_hash, uint64_t *bitmap)
{
    if (!h || !out) return MP_EINVAL;
    std::lock_guard<std::recursive_mutex> lk(h->mu);
    MP_CUDA(h, cudaSetDevice(h->device));
    mp_sieve_opts o;
    memset(&o, 0, sizeof o);
    if (opts) o = *opts;
    if (hi <= lo) return mp_set_error(h, MP_EINVAL, "need lo < hi");
    if (blocks && !o.block_log2) return mp_set_error(h, MP_EINVAL, "blocks requested without block_log2");
    if (!seg_hash) o.hash_log2 = 0;
    const u64 nb = blocks ? mp_sieve_nblocks(lo, hi, o.block_log2) : 0;
    const u64 nh = o.hash_log2 ? mp_sieve_nhashes(lo, hi, o.hash_log2) : 0;
    if (!nh) o.hash_log2 = 0;
    const u64 nw = bitmap ? mp_sieve_nwords(lo, hi) : 0;
    // one device allocation for all outputs
    const size_t off_b = 256, off_h = off_b + ((nb * sizeof(mp_block_stats) + 255) & ~255ull),
                 off_w = off_h + ((nh * 8 + 255) & ~255ull), total = off_w + nw * 8 + 256;
    MP_CUDA(h, h->stats_out.ensure(total));
    char *d = h->stats_out.as<char>();
    cudaStream_t st = h->stream;
    MP_CUDA(h, cudaEventRecord(h->ev0, st));
    MP_TRY(mp_sieve_range_dev(h, lo, hi, &o, (mp_range_stats *)d, blocks ? (mp_block_stats *)(d + off_b) : nullptr,
                              nh ? (u64 *)(d + off_h) : nullptr, nw ? (u64 *)(d + off_w) : nullptr, st));
    MP_CUDA(h, cudaEventRecord(h->ev1, st));
    MP_CUDA(h, cudaMemcpyAsync(out, d, sizeof *out, cudaMemcpyDeviceToHost, st));
    if (nb) MP_CUDA(h, cudaMemcpyAsync(blocks, d + off_b, nb * sizeof(mp_block_stats), cudaMemcpyDeviceToHost, st));
    if (nh) MP_CUDA(h, cudaMemcpyAsync(seg_hash, d + off_h, nh * 8, cudaMemcpyDeviceToHost, st));
    if (nw) MP_CUDA(h, cudaMemcpyAsync(bitmap, d + off_w, nw * 8, cudaMemcpyDeviceToHost, st));
    MP_CUDA(h, cudaStreamSynchronize(st));
    float ms = 0;
    if (cudaEventElapsedTime(&ms, h->ev0, h->ev1) == cudaSuccess) h->last_ms = ms;
    return mp_sieve_errors(h, st);
}

int mp_primes_range(mp_handle *h, uint64_t lo, uint64_t hi, uint64_t *primes, size_t cap, size_t *count)
{
    if (!h || !count) return MP_EINVAL;
    std::lock_guard<std::recursive_mutex> lk(h->mu);
    MP_CUDA(h, cudaSetDevice(h->device));
    *count = 0;
    if (hi <= lo) return MP_OK;
    cudaStream_t st = h->stream;
    u64 n = 0;
    // count first (cap 0), then emit into a device buffer of the exact size
    MP_TRY(mp_sieve_emit_primes(h, lo, hi, nullptr, 0, &n, st));
    *count = (size_t)n;
    if (!n) return MP_OK;
    MP_CUDA(h, h->ferm_p.ensure((size_t)n * 8));
    u64 n2 = 0;
    MP_TRY(mp_sieve_emit_primes(h, lo, hi, h->ferm_p.as<u64>(), n, &n2, st));
    const size_t m = std::min<size_t>(cap, (size_t)n);
    if (m && primes) MP_CUDA(h, cudaMemcpyAsync(primes, h->ferm_p.p, m * 8, cudaMemcpyDeviceToHost, st));
    MP_CUDA(h, cudaStreamSynchronize(st));
    return MP_OK;
}

// ---- BPSW ----

int mp_bpsw_lists_dev(mp_handle *h, const uint64_t *d_n, const uint64_t *offs, const uint32_t *lens, uint32_t nlists,
                      uint32_t *d_bits, uint32_t mode, void *stream)
{
    if (!h || (!d_n && nlists) || !offs || !lens) return MP_EINVAL;
    std::lock_guard<std::recursive_mutex> lk(h->mu);
    MP_CUDA(h, cudaSetDevice(h->device));
    for (u32 i = 0; i < nlists; i++)
        if ((offs[i] & 31) || offs[i] + lens[i] > offs[i + 1]) return mp_set_error(h, MP_EINVAL, "bad list layout");
    return mp_bpsw_run(h, d_n, offs, lens, nlists, d_bits, mode, mp_stream_of(h, stream));
}

int mp_bpsw_batches(mp_handle *h, const uint64_t *const *lists, const uint32_t *lens, uint32_t nlists,
                    uint8_t *const *out)
{
    if (!h || (nlists && (!lists || !lens || !out))) return MP_EINVAL;
    std::lock_guard<std::recursive_mutex> lk(h->mu);
    MP_CUDA(h, cudaSetDevice(h->device));
    std::vector<u64> offs(nlists + 1);
    u64 tot = 0;
    for (u32 i = 0; i < nlists; i++) { offs[i] = tot; tot += (lens[i] + 31ull) & ~31ull; }
    offs[nlists] = tot;
    if (!tot) return MP_OK;
    cudaStream_t st = h->stream;
    MP_CUDA(h, h->bpsw_n.ensure((size_t)tot * 8));
    MP_CUDA(h, h->bpsw_bits.ensure((size_t)tot / 8 + 64));
    u64 *dn = h->bpsw_n.as<u64>();
    // padding entries (never read back) are zero
    MP_CUDA(h, cudaMemsetAsync(dn, 0, (size_t)tot * 8, st));
    for (u32 i = 0; i < nlists; i++)
        if (lens[i]) MP_CUDA(h, cudaMemcpyAsync(dn + offs[i], lists[i], (size_t)lens[i] * 8, cudaMemcpyHostToDevice, st));
    MP_CUDA(h, cudaEventRecord(h->ev0, st));
    MP_TRY(mp_bpsw_run(h, dn, offs.data(), lens, nlists, h->bpsw_bits.as<u32>(), MP_MODE_BATCHED, st));
    MP_CUDA(h, cudaEventRecord(h->ev1, st));
    std::vector<u32> words((size_t)(tot / 32));
    MP_CUDA(h, cudaMemcpyAsync(words.data(), h->bpsw_bits.p, (size_t)tot / 8, cudaMemcpyDeviceToHost, st));
    MP_CUDA(h, cudaStreamSynchronize(st));
    float ms = 0;
    if (cudaEventElapsedTime(&ms, h->ev0, h->ev1) == cudaSuccess) h->last_ms = ms;
    for (u32 i = 0; i < nlists; i++)
        if (lens[i]) memcpy(out[i], (const u8 *)(words.data() + offs[i] / 32), (lens[i] + 7) / 8);
    return MP_OK;
}

int mp_bpsw_u64(mp_handle *h, const uint64_t *n, size_t count, uint8_t *verdict_bits)
{
    if (!h) return MP_EINVAL;
    if (!count) return MP_OK;
    if (!n || !verdict_bits) return MP_EINVAL;
    if (count > 0xffffffffull) return mp_set_error(h, MP_EINVAL, "count must be below 2^32");
    const uint64_t *lists[1] = {n};
    const uint32_t lens[1] = {(uint32_t)count};
    uint8_t *outs[1] = {verdict_bits};
    return mp_bpsw_batches(h, lists, lens, 1, outs);
}

// ---- Fermat ----

int mp_fermat_q_base2_dev(mp_handle *h, const uint64_t *d_p, size_t count, uint64_t *d_q, void *stream)
{
    if (!h) return MP_EINVAL;
    std::lock_guard<std::recursive_mutex> lk(h->mu);
    MP_CUDA(h, cudaSetDevice(h->device));
    // 4 limbs: valid for every p < 2^63
    const int variant = 1 | (h->tune.fermat_variant & 2);
    return mp_fermat_run(h, d_p, count, d_q, mp_stream_of(h, stream), variant, nullptr);
}

int mp_fermat_q_base2(mp_handle *h, const uint64_t *p, size_t count, uint64_t *q_out)
{
    if (!h) return MP_EINVAL;
    if (!count) return MP_OK;
    if (!p || !q_out) return MP_EINVAL;
    std::lock_guard<std::recursive_mutex> lk(h->mu);
    MP_CUDA(h, cudaSetDevice(h->device));
    u64 pmax = 0;
    for (size_t i = 0; i < count; i++) {
        if (p[i] >> 63) return mp_set_error(h, MP_ERANGE, "p must be below 2^63");
        pmax = std::max<u64>(pmax, p[i]);
    }
    cudaStream_t st = h->stream;
    MP_CUDA(h, h->ferm_p.ensure(count * 8));
    MP_CUDA(h, h->ferm_q.ensure(count * 8));
    MP_CUDA(h, cudaMemcpyAsync(h->ferm_p.p, p, count * 8, cudaMemcpyHostToDevice, st));
    const int variant = (pmax >> 47 ? 1 : 0) | (h->tune.fermat_variant & 2);
    MP_CUDA(h, cudaEventRecord(h->ev0, st));
    MP_TRY(mp_fermat_run(h, h->ferm_p.as<u64>(), count, h->ferm_q.as<u64>(), st, variant, nullptr));
    MP_CUDA(h, cudaEventRecord(h->ev1, st));
    MP_CUDA(h, cudaMemcpyAsync(q_out, h->ferm_q.p, count * 8, cudaMemcpyDeviceToHost, st));
    MP_CUDA(h, cudaStreamSynchronize(st));
    float ms = 0;
    if (cudaEventElapsedTime(&ms, h->ev0, h->ev1) == cudaSuccess) h->last_ms = ms;
    return MP_OK;
}

int mp_wieferich_range(mp_handle *h, uint64_t lo, uint64_t hi, mp_wief_stats *out)
{
    if (!h || !out) return MP_EINVAL;
    std::lock_guard<std::recursive_mutex> lk(h->mu);
    MP_CUDA(h, cudaSetDevice(h->device));
    memset(out, 0, sizeof *out);
    if (hi <= lo) return MP_OK;
    if (hi > (1ull << 63)) return mp_set_error(h, MP_ERANGE, "hi must be <= 2^63");
    cudaStream_t st = h->stream;
    u64 n = 0;
    MP_TRY(mp_sieve_emit_primes(h, lo, hi, nullptr, 0, &n, st));
    MP_CUDA(h, h->ferm_p.ensure((size_t)n * 8 + 8));
    MP_CUDA(h, h->ferm_q.ensure((size_t)n * 8 + 8));
    MP_CUDA(h, h->stats_out.ensure(sizeof(mp_wief_stats) + 256));
    u64 n2 = 0;
    MP_TRY(mp_sieve_emit_primes(h, lo, hi, h->ferm_p.as<u64>(), n, &n2, st));
    const int variant = ((hi - 1) >> 47 ? 1 : 0) | (h->tune.fermat_variant & 2);
    mp_wief_stats *ds = h->stats_out.as<mp_wief_stats>();
    MP_CUDA(h, cudaEventRecord(h->ev0, st));
    MP_TRY(mp_fermat_run(h, h->ferm_p.as<u64>(), n, h->ferm_q.as<u64>(), st, variant, nullptr));
    MP_TRY(mp_fermat_reduce(h, h->ferm_p.as<u64>(), h->ferm_q.as<u64>(), n, ds, st));
    MP_CUDA(h, cudaEventRecord(h->ev1, st));
    MP_CUDA(h, cudaMemcpyAsync(out, ds, sizeof *out, cudaMemcpyDeviceToHost, st));
    MP_CUDA(h, cudaStreamSynchronize(st));
    float ms = 0;
    if (cudaEventElapsedTime(&ms, h->ev0, h->ev1) == cudaSuccess) h->last_ms = ms;
    out->primes = n;
    return MP_OK;
}

}  // extern "C"
