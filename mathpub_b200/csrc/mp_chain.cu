// mp_chain.cu -- the constellation sieve for chains of consecutive primes with gaps 2, 4, 6,
// ... (A016045): the heads p whose members p + m(m + 1), m < k, are all prime with nothing
// prime in between.  It finds what mp_gap_chains finds by enumeration without enumerating
// primes; the method is the one gapchain/README_SIEVE.md describes for gapchain/gapsieve.c.
//
//   wheel     the residues of p modulo the primes 2..q_w that leave every member coprime to
//             them, combined by CRT into the classes s0 of p mod W (W = 2 3 5 ... q_w, grown
//             while W <= 3e7 and the classes number at most 24,000); p = b + s0 + k W
//   patterns  for the primes q above the wheel up to 199: member m is divisible by q exactly
//             when (k + t + s0 W^-1) mod q = -m(m + 1) W^-1 mod q, t = b / W.  The forbidden
//             residues of each group of primes (periods multiplied up to 2^24) are one bit
//             pattern; a class reads it from the rotation (t + C) mod P, C = CRT(s0 W^-1), so
//             2^17 values of k cost a few 64-bit window reads and ANDs per word
//   screen    the survivors' members in order with the base-2 strong test; a composite
//             verdict is exact
//   verify    every member certified by BPSW (exact below 2^64), every odd number between
//             consecutive members composite, and the chain extended past k
// Heads below 2^24 (where a member could be a sieving prime) come from mp_gap_chains.
#include "mp_mont64.cuh"
#include <algorithm>
#include <numeric>

#define CH_K 131072u                          // k values per class and segment
#define CH_WORDS (CH_K / 64)
#define CH_PMAX 199u                          // pattern primes up to this
#define CH_PERIOD_MAX (1u << 24)
#define CH_LOW ((u64)1 << 24)                 // heads below this come from the enumeration
#define CH_MAXG 24

struct ChainSieveArgs {
    u64 b0;                                    // segment 0 starts at b0 (a multiple of W)
    u64 W;
    u32 nclass, ngroup, seg0, nseg;           // segments [seg0, seg0 + nseg)
    u64 lo, hi;                               // heads in [lo, hi)
    const u32 *s0;                            // [nclass]
    const u32 *C;                             // [nclass][ngroup]
    const u64 *pat[CH_MAXG];                  // group patterns
    u32 period[CH_MAXG];
    u32 tmod[CH_MAXG];                        // (b0 / W + seg0 * CH_K) mod period
    u64 *cand;
    u64 cap;
    unsigned long long *ncand;
};

// one CTA per (class, segment): AND the rotated group patterns over the segment's 2^17 values
// of k and append the survivors' p
__global__ void __launch_bounds__(256) chain_sieve_kernel(ChainSieveArgs a)
{
    const u32 c = blockIdx.x % a.nclass, s = blockIdx.x / a.nclass;
    const u64 base = a.b0 + (u64)(a.seg0 + s) * CH_K * a.W + a.s0[c];
    const u32 lane = threadIdx.x & 31;
    for (u32 w = threadIdx.x; w < CH_WORDS; w += blockDim.x) {
        u64 acc = ~0ull;
        for (u32 g = 0; g < a.ngroup; g++) {
            const u32 P = a.period[g];
            // rotation of this class and segment, then the word's first bit
            u64 y = (u64)a.tmod[g] + (u64)s * (CH_K % P) + a.C[(u64)c * a.ngroup + g];
            y %= P;
            y += 64ull * w;
            const u64 *pw = a.pat[g] + (y >> 6);
            const u32 sh = (u32)(y & 63);
            const u64 lo64 = __ldg(pw), hi64 = __ldg(pw + 1);
            acc &= sh ? (lo64 >> sh) | (hi64 << (64 - sh)) : lo64;
        }
        // heads in [lo, hi) only (a word's 64 values span 63 W)
        const u64 p0 = base + 64ull * w * a.W;
        if (p0 < a.lo || p0 + 63 * a.W >= a.hi) {
            u64 bits = acc;
            while (bits) {
                const u32 b = __ffsll((long long)bits) - 1;
                bits &= bits - 1;
                const u64 p = p0 + (u64)b * a.W;
                if (p < a.lo || p >= a.hi) acc &= ~(1ull << b);
            }
        }
        const u32 nb = __popcll(acc);
        // warp-aggregated append (every thread takes CH_WORDS / blockDim.x words: all lanes here)
        u32 incl = nb;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const u32 v = __shfl_up_sync(0xffffffffu, incl, d);
            if (lane >= (u32)d) incl += v;
        }
        const u32 tot = __shfl_sync(0xffffffffu, incl, 31);
        unsigned long long bpos = 0;
        if (lane == 31 && tot) bpos = atomicAdd(a.ncand, (unsigned long long)tot);
        bpos = __shfl_sync(0xffffffffu, bpos, 31);
        u64 pos = bpos + incl - nb;
        while (acc) {
            const u32 b = __ffsll((long long)acc) - 1;
            acc &= acc - 1;
            if (pos < a.cap) a.cand[pos] = p0 + (u64)b * a.W;
            pos++;
        }
    }
}

// the base-2 strong test on every member, in order; survivors go to the passer list
__global__ void __launch_bounds__(256) chain_screen_kernel(const u64 *__restrict__ cand, u64 n, u32 k, u64 *pass,
                                                           u64 cap, unsigned long long *npass)
{
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        const u64 p = cand[i];
        bool ok = true;
        for (u32 m = 0; m < k && ok; m++) {
            const u64 x = p + (u64)m * (m + 1);
            ok = sprp2_dev(x, m_inv(x), m_one(x));
        }
        if (ok) {
            const unsigned long long j = atomicAdd(npass, 1ull);
            if (j < cap) pass[j] = p;
        }
    }
}

// certify, check the interlopers, extend; chains of at least k primes go to the result list
__global__ void __launch_bounds__(128) chain_verify_kernel(const u64 *__restrict__ pass, u64 n, u32 k, u64 *heads,
                                                           u32 *lens, u64 cap, unsigned long long *nres)
{
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        const u64 p = pass[i];
        u32 len = 0;
        // member m is p + m(m + 1); between members m and m + 1 lie the odd numbers
        // p + m(m + 1) + 2, ..., p + m(m + 1) + 2m
        for (u32 m = 0; m < MP_CHAIN_MAX - 1; m++) {
            const u64 x = p + (u64)m * (m + 1);
            if (!bpsw_odd(x)) break;
            if (m) {
                bool clear = true;
                const u64 prev = p + (u64)(m - 1) * m;
                for (u64 y = prev + 2; y < x && clear; y += 2) clear = !bpsw_odd(y);
                if (!clear) break;
            }
            len = m + 1;
        }
        if (len >= k) {
            const unsigned long long j = atomicAdd(nres, 1ull);
            if (j < cap) { heads[j] = p; lens[j] = len; }
        }
    }
}

// ---- host: wheel, patterns, rounds ----

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

struct ChainPlan {
    u32 k = 0;
    u64 W = 1;
    std::vector<u32> s0;                        // classes of p mod W
    std::vector<std::vector<u32>> gq;           // pattern groups
    std::vector<u32> period;
    std::vector<u32> C;                         // [class][group]
    std::vector<std::vector<u64>> pat;          // host copies of the patterns
    double survive = 1;                         // expected fraction of k surviving the patterns
};

// false when some small prime leaves no admissible residue: no chain of length k has a head
// at or above CH_LOW
bool make_plan(u32 k, ChainPlan &P)
{
    P.k = k;
    std::vector<u64> offs(k);
    for (u32 m = 0; m < k; m++) offs[m] = (u64)m * (m + 1);
    std::vector<u64> cls{0};
    u64 W = 1;
    u32 q = 2;
    for (; q <= CH_PMAX; q++) {
        if (!is_small_prime(q)) continue;
        std::vector<u32> adm;
        for (u32 r = 0; r < q; r++) {
            bool ok = true;
            for (u64 o : offs) ok = ok && (r + o) % q != 0;
            if (ok) adm.push_back(r);
        }
        if (adm.empty()) return false;
        if (q > 2 && (W * q > 30000000ull || cls.size() * adm.size() > 24000)) break;
        // CRT: x = c (mod W), x = r (mod q)
        std::vector<u64> nc;
        const u64 Wi = inv_mod(W % q, q);
        for (u64 c : cls)
            for (u32 r : adm) {
                const u64 t = ((r + q - c % q) % q) * Wi % q;
                nc.push_back(c + W * t);
            }
        cls.swap(nc);
        W *= q;
    }
    std::sort(cls.begin(), cls.end());
    P.W = W;
    P.s0.assign(cls.begin(), cls.end());
    // pattern groups from the first prime above the wheel up to CH_PMAX
    std::vector<u32> gq;
    u64 per = 1;
    for (; q <= CH_PMAX; q++) {
        if (!is_small_prime(q)) continue;
        if (per * q > CH_PERIOD_MAX) { P.gq.push_back(gq); gq.clear(); per = 1; }
        gq.push_back(q);
        per *= q;
    }
    if (!gq.empty()) P.gq.push_back(gq);
    const u32 G = (u32)P.gq.size();
    P.period.resize(G);
    P.pat.resize(G);
    for (u32 g = 0; g < G; g++) {
        u64 Pg = 1;
        for (u32 qq : P.gq[g]) Pg *= qq;
        P.period[g] = (u32)Pg;
        // forbidden residues per prime, -m(m + 1) W^-1 mod q: strike their classes over one period
        std::vector<u8> ok(Pg, 1);
        for (u32 qq : P.gq[g]) {
            std::vector<char> bad(qq, 0);
            const u64 Wi = inv_mod(W % qq, qq);
            u32 nbad = 0;
            for (u64 o : offs) {
                const u64 f = (qq - (o % qq)) % qq * Wi % qq;
                if (bad[f]) continue;
                bad[f] = 1;
                nbad++;
                for (u64 y = f; y < Pg; y += qq) ok[y] = 0;
            }
            P.survive *= 1.0 - (double)nbad / qq;
        }
        // the period, then the first CH_K + 128 bits again, so that no window read wraps
        const u64 nbits = Pg + CH_K + 128;
        std::vector<u64> bits((nbits + 63) / 64 + 1, 0);
        for (u64 y = 0, yy = 0; y < nbits; y++, yy = yy + 1 == Pg ? 0 : yy + 1)
            if (ok[yy]) bits[y >> 6] |= 1ull << (y & 63);
        P.pat[g].swap(bits);
    }
    // per class and group: C = CRT over the group's primes of s0 W^-1 mod q
    P.C.resize(P.s0.size() * G);
    for (size_t c = 0; c < P.s0.size(); c++)
        for (u32 g = 0; g < G; g++) {
            u64 x = 0, M = 1;
            for (u32 qq : P.gq[g]) {
                const u64 r = (u64)P.s0[c] % qq * inv_mod(W % qq, qq) % qq;
                const u64 t = ((r + qq - x % qq) % qq) * inv_mod(M % qq, qq) % qq;
                x += M * t;
                M *= qq;
            }
            P.C[c * G + g] = (u32)x;
        }
    return true;
}

}  // namespace

struct ChainDev {
    u32 k = 0;
    ChainPlan plan;
    std::vector<DevBuf> pat;
    DevBuf s0, C, cand, pass, res, cnt;
    void release()
    {
        for (DevBuf &b : pat) b.release();
        for (DevBuf *b : {&s0, &C, &cand, &pass, &res, &cnt}) b->release();
    }
};

void mp_chain_free(mp_handle *h)
{
    if (!h->chain) return;
    h->chain->release();
    delete h->chain;
    h->chain = nullptr;
}

static int chain_round(mp_handle *h, ChainDev &D, u64 lo, u64 hi, u64 b0, u32 seg0, u32 nseg, std::vector<u64> &heads,
                       std::vector<u32> &lens, cudaStream_t st)
{
    const ChainPlan &P = D.plan;
    const u32 nclass = (u32)P.s0.size(), G = (u32)P.period.size();
    const double expect = (double)nclass * nseg * CH_K * P.survive;
    const u64 cap = (u64)(2.0 * expect) + (1u << 20);
    MP_CUDA(h, D.cand.ensure((size_t)cap * 8));
    MP_CUDA(h, D.cnt.ensure(64));
    unsigned long long *cnt = D.cnt.as<unsigned long long>();
    MP_CUDA(h, cudaMemsetAsync(cnt, 0, 64, st));
    ChainSieveArgs a;
    memset(&a, 0, sizeof a);
    a.b0 = b0; a.W = P.W; a.nclass = nclass; a.ngroup = G; a.seg0 = seg0; a.nseg = nseg; a.lo = lo; a.hi = hi;
    a.s0 = D.s0.as<u32>(); a.C = D.C.as<u32>();
    for (u32 g = 0; g < G; g++) {
        a.pat[g] = D.pat[g].as<u64>();
        a.period[g] = P.period[g];
        const u64 t0 = b0 / P.W + (u64)seg0 * CH_K;
        a.tmod[g] = (u32)(t0 % P.period[g]);
    }
    a.cand = D.cand.as<u64>(); a.cap = cap; a.ncand = cnt;
    chain_sieve_kernel<<<nclass * nseg, 256, 0, st>>>(a);
    MP_CUDA(h, cudaGetLastError());
    u64 nc = 0;
    MP_CUDA(h, cudaMemcpyAsync(&nc, cnt, 8, cudaMemcpyDeviceToHost, st));
    MP_CUDA(h, cudaStreamSynchronize(st));
    if (nc > cap) {                                  // more survivors than room: split the round
        if (nseg == 1) return mp_set_error(h, MP_EOVERFLOW, "chain sieve: survivors exceed the candidate buffer");
        MP_TRY(chain_round(h, D, lo, hi, b0, seg0, nseg / 2, heads, lens, st));
        return chain_round(h, D, lo, hi, b0, seg0 + nseg / 2, nseg - nseg / 2, heads, lens, st);
    }
    if (!nc) return MP_OK;
    const u64 pcap = nc / 16 + 4096;
    MP_CUDA(h, D.pass.ensure((size_t)pcap * 8));
    u64 grid = std::min<u64>((nc + 255) / 256, (u64)h->sm_count * 64);
    chain_screen_kernel<<<(unsigned)grid, 256, 0, st>>>(D.cand.as<u64>(), nc, P.k, D.pass.as<u64>(), pcap, cnt + 1);
    MP_CUDA(h, cudaGetLastError());
    u64 np = 0;
    MP_CUDA(h, cudaMemcpyAsync(&np, cnt + 1, 8, cudaMemcpyDeviceToHost, st));
    MP_CUDA(h, cudaStreamSynchronize(st));
    if (np > pcap) return mp_set_error(h, MP_EOVERFLOW, "chain sieve: screen passers exceed their buffer");
    if (!np) return MP_OK;
    MP_CUDA(h, D.res.ensure((size_t)np * 12 + 64));
    u64 *rh = D.res.as<u64>();
    u32 *rl = (u32 *)(rh + np);
    grid = std::min<u64>((np + 127) / 128, (u64)h->sm_count * 16);
    chain_verify_kernel<<<(unsigned)grid, 128, 0, st>>>(D.pass.as<u64>(), np, P.k, rh, rl, np, cnt + 2);
    MP_CUDA(h, cudaGetLastError());
    u64 nr = 0;
    MP_CUDA(h, cudaMemcpyAsync(&nr, cnt + 2, 8, cudaMemcpyDeviceToHost, st));
    MP_CUDA(h, cudaStreamSynchronize(st));
    if (nr) {
        const size_t o = heads.size();
        heads.resize(o + nr);
        lens.resize(o + nr);
        MP_CUDA(h, cudaMemcpyAsync(heads.data() + o, rh, nr * 8, cudaMemcpyDeviceToHost, st));
        MP_CUDA(h, cudaMemcpyAsync(lens.data() + o, rl, nr * 4, cudaMemcpyDeviceToHost, st));
        MP_CUDA(h, cudaStreamSynchronize(st));
    }
    return MP_OK;
}

extern "C" int mp_chain_sieve(mp_handle *h, uint64_t lo, uint64_t hi, uint32_t k, uint64_t *heads, uint32_t *lens,
                              size_t cap, size_t *count)
{
    if (!h || !count || (cap && (!heads || !lens))) return MP_EINVAL;
    *count = 0;
    if (k < 4 || k >= MP_CHAIN_MAX) return mp_set_error(h, MP_EINVAL, "k must be in 4..%d", MP_CHAIN_MAX - 1);
    if (hi > (1ull << 63)) return mp_set_error(h, MP_ERANGE, "hi must be <= 2^63");
    if (hi <= lo) return MP_OK;
    std::lock_guard<std::recursive_mutex> lk(h->mu);
    MP_CUDA(h, cudaSetDevice(h->device));
    cudaStream_t st = h->stream;
    std::vector<u64> H;
    std::vector<u32> L;
    // heads below CH_LOW by enumeration
    if (lo < CH_LOW) {
        const u64 e = std::min<u64>(hi, CH_LOW);
        size_t n = 0;
        MP_TRY(mp_gap_chains(h, lo, e, k, nullptr, nullptr, 0, &n));
        H.resize(n);
        L.resize(n);
        if (n) MP_TRY(mp_gap_chains(h, lo, e, k, H.data(), L.data(), n, &n));
    }
    const u64 slo = std::max<u64>(lo, CH_LOW);
    if (slo < hi) {
        if (!h->chain || h->chain->k != k) {
            mp_chain_free(h);
            h->chain = new ChainDev();
            ChainDev &D = *h->chain;
            D.k = k;
            if (make_plan(k, D.plan)) {
                const ChainPlan &P = D.plan;
                D.pat.resize(P.pat.size());
                for (size_t g = 0; g < P.pat.size(); g++) {
                    MP_CUDA(h, D.pat[g].ensure(P.pat[g].size() * 8));
                    MP_CUDA(h, cudaMemcpy(D.pat[g].p, P.pat[g].data(), P.pat[g].size() * 8, cudaMemcpyHostToDevice));
                }
                MP_CUDA(h, D.s0.ensure(P.s0.size() * 4));
                MP_CUDA(h, cudaMemcpy(D.s0.p, P.s0.data(), P.s0.size() * 4, cudaMemcpyHostToDevice));
                MP_CUDA(h, D.C.ensure(P.C.size() * 4));
                MP_CUDA(h, cudaMemcpy(D.C.p, P.C.data(), P.C.size() * 4, cudaMemcpyHostToDevice));
            } else D.plan.s0.clear();             // no chain of length k above CH_LOW
        }
        ChainDev &D = *h->chain;
        if (!D.plan.s0.empty()) {
            if (D.plan.period.size() > CH_MAXG) return mp_set_error(h, MP_EINVAL, "too many pattern groups");
            const u64 W = D.plan.W, span = (u64)CH_K * W;
            const u64 b0 = slo / W * W;
            const u64 nseg = (hi - b0 + span - 1) / span;
            // rounds of segments sized for about 2^24 expected survivors
            const double per = (double)D.plan.s0.size() * CH_K * D.plan.survive;
            const u32 step = (u32)std::max<double>(1.0, std::min<double>(4096.0, 16777216.0 / per));
            for (u64 s = 0; s < nseg; s += step)
                MP_TRY(chain_round(h, D, slo, hi, b0, (u32)s, (u32)std::min<u64>(step, nseg - s), H, L, st));
        }
    }
    std::vector<size_t> ord(H.size());
    std::iota(ord.begin(), ord.end(), 0);
    std::sort(ord.begin(), ord.end(), [&](size_t x, size_t y) { return H[x] < H[y]; });
    const size_t m = std::min(cap, H.size());
    for (size_t i = 0; i < m; i++) { heads[i] = H[ord[i]]; lens[i] = L[ord[i]]; }
    *count = H.size();
    return MP_OK;
}
