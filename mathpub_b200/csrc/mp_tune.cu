// mp_tune.cu -- the measured autotuner: times the sieve tile geometry (bits per tile x
// threads per CTA), the bucket scatter's form, the bucket threshold, the batched form
// (persistent pipeline or wave loop), the Fermat kernel variants (limbs fixed by p, one or two
// primes per thread) and the batched BPSW kernel's warps per CTA x candidates per queue chunk
// on the device with CUDA events, and keeps the fastest per handle.  The reference
// chooses its wheel and chunk by a fitted cost model (auto_wheel / auto_chunk,
// A350826/a350826.c:1976-2015); here the candidates are timed instead.
#include "mp_common.cuh"
#include <algorithm>

static int time_sieve(mp_handle *h, u64 lo, u64 hi, u32 tlog, u32 nth, mp_range_stats *d_out, float *ms)
{
    mp_sieve_opts o;
    memset(&o, 0, sizeof o);
    o.mode = MP_MODE_BATCHED;
    o.tile_log2 = tlog;
    o.threads = nth;
    cudaStream_t st = h->stream;
    MP_TRY(mp_sieve_run(h, lo, hi, &o, d_out, nullptr, nullptr, nullptr, st));   // warm-up
    MP_CUDA(h, cudaEventRecord(h->ev0, st));
    for (int r = 0; r < 3; r++) MP_TRY(mp_sieve_run(h, lo, hi, &o, d_out, nullptr, nullptr, nullptr, st));
    MP_CUDA(h, cudaEventRecord(h->ev1, st));
    MP_CUDA(h, cudaEventSynchronize(h->ev1));
    MP_CUDA(h, cudaEventElapsedTime(ms, h->ev0, h->ev1));
    return MP_OK;
}

extern "C" int mp_autotune(mp_handle *h, uint64_t lo, char *report, size_t cap)
{
    if (!h) return MP_EINVAL;
    std::lock_guard<std::recursive_mutex> lk(h->mu);
    MP_CUDA(h, cudaSetDevice(h->device));
    std::string rep;
    char line[160];
    // sieve: a range of 2^34 integers at height lo (several waves, as in long scans); a choice
    // replaces the default only when it is more than 2% faster, so that timing noise between
    // near-equal forms does not decide
    const u64 span = 1ull << 34;
    const float margin = 1.02f;
    if (lo > MP_HI_MAX - span) lo = MP_HI_MAX - span;
    MP_CUDA(h, h->small_out.ensure(4096));
    mp_range_stats *d_out = (mp_range_stats *)h->small_out.p;
    float best = 1e30f, dflt = 1e30f;
    u32 bt = 20, bn = 1024;
    static const u32 tl[3] = {18, 19, 20}, th[3] = {256, 512, 1024};
    for (u32 a : tl)
        for (u32 b : th) {
            float ms = 0;
            const int r = time_sieve(h, lo, lo + span, a, b, d_out, &ms);
            if (r != MP_OK) return r;
            snprintf(line, sizeof line, "sieve tile 2^%u x %u threads: %.3f ms / 2^34\n", a, b, ms / 3);
            rep += line;
            if (ms < best) { best = ms; bt = a; bn = b; }
            if (a == 20 && b == 1024) dflt = ms;
        }
    if (dflt <= best * margin) { bt = 20; bn = 1024; }
    h->tune.sieve_tile_log2 = (int)bt;
    h->tune.sieve_threads = (int)bn;
    h->tune.tuned_at = lo;
    h->tune_gen++;
    // one knob at a time at that geometry, on the same range, the first value the default:
    //   the bucket scatter's form: staged (three CTAs per SM, a sorted stage) or binned (one
    //   CTA per SM, a bin per tile);
    //   the bucket threshold: primes above the tile size, half of it or a quarter of it go to
    //   the scatter (fewer visits of sparse primes per tile against more bucket records);
    //   the batched form as one persistent pipeline launch or as a host loop of wave launches
    struct Knob { const char *name; int *field; int vals[3]; int nv; const char *labels[3]; };
    Knob knobs[3] = {
        {"scatter", &h->tune.scatter_staged, {1, 0, 0}, 2, {"staged", "binned", ""}},
        {"bucket threshold", &h->tune.bucket_div, {1, 2, 4}, 3, {"tile", "tile/2", "tile/4"}},
        {"batched form", &h->tune.no_pipeline, {0, 1, 0}, 2, {"pipeline", "wave loop", ""}},
    };
    for (Knob &k : knobs) {
        // the pipeline runs with the binned scatter only: with the staged one the knob changes nothing
        if (k.field == &h->tune.no_pipeline && h->tune.scatter_staged) continue;
        float kb = 1e30f, k0 = 1e30f;
        int kv = k.vals[0];
        for (int i = 0; i < k.nv; i++) {
            *k.field = k.vals[i];
            float ms = 0;
            const int r = time_sieve(h, lo, lo + span, bt, bn, d_out, &ms);
            if (r != MP_OK) { *k.field = k.vals[0]; h->tune_gen++; return r; }
            snprintf(line, sizeof line, "%s %s: %.3f ms / 2^34\n", k.name, k.labels[i], ms / 3);
            rep += line;
            if (ms < kb) { kb = ms; kv = k.vals[i]; }
            if (i == 0) k0 = ms;
        }
        *k.field = k0 <= kb * margin ? k.vals[0] : kv;
    }
    h->tune_gen++;
    snprintf(line, sizeof line, "sieve choice: tile 2^%u, %u threads, %s scatter, bucket threshold tile/%d, %s\n", bt,
             bn, h->tune.scatter_staged ? "staged" : "binned", h->tune.bucket_div,
             (h->tune.no_pipeline || h->tune.scatter_staged) ? "wave loop" : "pipeline");
    rep += line;
    // Fermat: 2^20 primes near max(lo, 1e12), one vs two per thread
    u64 plo = std::max<u64>(lo, 1000000000000ull);
    if (plo > (1ull << 62)) plo = 1ull << 40;
    u64 n = 0;
    MP_TRY(mp_sieve_emit_primes(h, plo, plo + (1ull << 26), nullptr, 0, &n, h->stream));
    MP_CUDA(h, h->ferm_p.ensure((size_t)n * 8 + 8));
    MP_CUDA(h, h->ferm_q.ensure((size_t)n * 8 + 8));
    u64 n2 = 0;
    MP_TRY(mp_sieve_emit_primes(h, plo, plo + (1ull << 26), h->ferm_p.as<u64>(), n, &n2, h->stream));
    const int k4 = (plo + (1ull << 26)) >> 47 ? 1 : 0;
    float fb = 1e30f;
    int fv = 0;
    for (int ilp = 0; ilp < 2; ilp++) {
        const int v = k4 | (ilp << 1);
        MP_TRY(mp_fermat_run(h, h->ferm_p.as<u64>(), n, h->ferm_q.as<u64>(), h->stream, v, nullptr));
        MP_CUDA(h, cudaEventRecord(h->ev0, h->stream));
        for (int r = 0; r < 3; r++) MP_TRY(mp_fermat_run(h, h->ferm_p.as<u64>(), n, h->ferm_q.as<u64>(), h->stream, v, nullptr));
        MP_CUDA(h, cudaEventRecord(h->ev1, h->stream));
        MP_CUDA(h, cudaEventSynchronize(h->ev1));
        float ms = 0;
        MP_CUDA(h, cudaEventElapsedTime(&ms, h->ev0, h->ev1));
        snprintf(line, sizeof line, "fermat %s limbs, %d prime(s)/thread: %.3f ms for %llu primes\n", k4 ? "4" : "3",
                 ilp + 1, ms / 3, (unsigned long long)n);
        rep += line;
        if (ms < fb) { fb = ms; fv = v; }
    }
    h->tune.fermat_variant = fv & 2;
    snprintf(line, sizeof line, "fermat choice: %d prime(s)/thread\n", (fv & 2) ? 2 : 1);
    rep += line;
    // batched BPSW: 2^23 seeded odd candidates (three in four in [2^62, 2^64), the rest in
    // [2^40, 2^62)), one list, each warps x chunk pair the kernel is built for.  Enough chunks
    // for several per warp: with fewer CTAs than SMs the launch's tail would decide
    {
        const u64 cnt = 1ull << 23;
        std::vector<u64> cand(cnt);
        u64 z = 0x5eed5eedull;
        for (u64 i = 0; i < cnt; i++) {
            z += MP_GOLD;
            u64 x = mp_mix64(z);
            x = (i & 3) ? (x | (1ull << 62)) : ((x >> 24) | (1ull << 40));
            cand[i] = x | 1;
        }
        MP_CUDA(h, h->bpsw_n.ensure(cnt * 8));
        MP_CUDA(h, h->bpsw_bits.ensure(cnt / 8 + 64));
        MP_CUDA(h, cudaMemcpyAsync(h->bpsw_n.p, cand.data(), cnt * 8, cudaMemcpyHostToDevice, h->stream));
        const u64 offs[2] = {0, cnt};
        const u32 lens[1] = {(u32)cnt};
        float bb = 1e30f;
        int bv = 0;
        for (int v = 0; v < 4; v++) {
            h->tune.bpsw_variant = v;
            MP_TRY(mp_bpsw_run(h, h->bpsw_n.as<u64>(), offs, lens, 1, h->bpsw_bits.as<u32>(), MP_MODE_BATCHED, h->stream));
            MP_CUDA(h, cudaEventRecord(h->ev0, h->stream));
            for (int r = 0; r < 3; r++)
                MP_TRY(mp_bpsw_run(h, h->bpsw_n.as<u64>(), offs, lens, 1, h->bpsw_bits.as<u32>(), MP_MODE_BATCHED,
                                   h->stream));
            MP_CUDA(h, cudaEventRecord(h->ev1, h->stream));
            MP_CUDA(h, cudaEventSynchronize(h->ev1));
            float ms = 0;
            MP_CUDA(h, cudaEventElapsedTime(&ms, h->ev0, h->ev1));
            snprintf(line, sizeof line, "bpsw %s: %.3f ms for 2^23 candidates\n", mp_bpsw_variant_name(v), ms / 3);
            rep += line;
            if (ms < bb) { bb = ms; bv = v; }
        }
        h->tune.bpsw_variant = bv;
        snprintf(line, sizeof line, "bpsw choice: %s\n", mp_bpsw_variant_name(bv));
        rep += line;
    }
    if (report && cap) {
        strncpy(report, rep.c_str(), cap - 1);
        report[cap - 1] = 0;
    }
    return MP_OK;
}

extern "C" int mp_tune_set(mp_handle *h, int knob, int value)
{
    if (!h) return MP_EINVAL;
    std::lock_guard<std::recursive_mutex> lk(h->mu);
    switch (knob) {
    case MP_TUNE_TILE_LOG2:
        if (value != 0 && (value < 18 || value > 20)) return MP_EINVAL;
        h->tune.sieve_tile_log2 = value;
        break;
    case MP_TUNE_THREADS:
        if (value != 0 && value != 256 && value != 512 && value != 1024) return MP_EINVAL;
        h->tune.sieve_threads = value;
        break;
    case MP_TUNE_SCATTER_STAGED:
        if (value != 0 && value != 1) return MP_EINVAL;
        h->tune.scatter_staged = value;
        break;
    case MP_TUNE_BUCKET_DIV:
        if (value != 1 && value != 2 && value != 4) return MP_EINVAL;
        h->tune.bucket_div = value;
        break;
    case MP_TUNE_NO_PIPELINE:
        if (value != 0 && value != 1) return MP_EINVAL;
        h->tune.no_pipeline = value;
        break;
    case MP_TUNE_BPSW_VARIANT:
        if (value < 0 || value > 3) return MP_EINVAL;
        h->tune.bpsw_variant = value;
        break;
    case MP_TUNE_FERMAT_ILP2:
        if (value != 0 && value != 1) return MP_EINVAL;
        h->tune.fermat_variant = value ? 2 : 0;
        break;
    default:
        return MP_EINVAL;
    }
    h->tune_gen++;
    return MP_OK;
}
