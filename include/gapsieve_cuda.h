/*
 * gapsieve_cuda.h -- the GPU constellation-sieve interface of the reference's gapsieve
 * (gapchain/gapsieve_cuda.h:1-70), implemented by libmathpub on sm_100a.  The reference's own
 * host program, gapchain/gapsieve_cuda_host.c (which includes gapchain/gapsieve.c), compiles
 * against this interface unchanged and links against libmathpub instead of its own kernels.
 *
 * The host computes every table: the wheel's admissible residues, the sieve primes with
 * W^-1 mod q and their CRT coefficients within each pattern group, the groups' bit patterns,
 * and for every segment of a unit its base mod each sieve prime.  The GPU sieves every class
 * of every segment of a unit (segments of 2^17 W integers), screens every member of every
 * survivor with the base-2 strong test, and returns the survivors' offsets from the unit's
 * base; the host proves them.  The struct layout and the call signatures must stay those of
 * the reference header, since the host program is compiled from the reference's sources.
 */
#ifndef GAPSIEVE_CUDA_H
#define GAPSIEVE_CUDA_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define CU_MAXSLOT 8            /* units in flight */
#define CU_MAXK 1024            /* member offsets per shape */

/* one unit of one shape (gapchain/gapsieve_cuda_host.c:169-176 fills it) */
struct cu_params {
    uint64_t base_lo, base_hi;  /* the unit's first segment starts at base (128-bit) */
    uint64_t lim;               /* candidates have offsets 0 .. lim from base */
    uint64_t segsize;           /* 2^17 W */
    uint32_t W, bmodW, A, ngroups, nps, k;
    uint32_t cap;               /* entries in each candidate list */
    uint32_t nseg;              /* segments in the unit */
    uint32_t dense;             /* a tuning hint of the reference kernels; unused here */
};

/* select the GPU and write its name; 0 on success */
int cu_init(char *name, size_t n);

/* the shared tables: per group (P, index of its first sieve prime, its primes, 64-bit word
   offset of its pattern), per sieve prime q, W^-1 mod q and its CRT coefficient mod P */
int cu_tables(uint32_t ngroups, const uint32_t *ginfo, uint32_t nps, const uint32_t *q, const uint32_t *qinv,
              const uint32_t *crt);

/* shape d (0: gaps 2, 4, ...; 1: ..., 4, 2): its patterns (npat 32-bit words, 64-bit words
   in little-endian halves), A admissible residues mod W, k member offsets */
int cu_shape(int d, const uint32_t *pat, size_t npat, const uint32_t *res, uint32_t A, const uint32_t *offs,
             uint32_t k);

/* device buffers for one slot: units of up to `unit` segments, lists of cap entries */
int cu_slot(int slot, uint32_t unit, uint32_t cap);

/* the slot's lists again, with cap entries */
int cu_grow(int slot, uint32_t cap);

/* queue a unit (asynchronous; units run in submission order): bq[g * nps + i] = segment g's
   base mod sieve prime i; p[d] NULL for a shape the unit does not need; `split` rounds screen
   one member each over the whole list before one kernel tests the rest per candidate */
int cu_submit(int slot, const uint32_t *bq, uint32_t nseg, uint32_t nps, const struct cu_params *p[2], int split);

/* wait for the slot's unit: 0 done, -1 failed; stat[d] = the sieve's survivors (more than cap:
   the lists overflowed and the unit must be redone), nfin[d] = the screen's survivors */
int cu_wait(int slot, uint32_t stat[2], uint32_t nfin[2]);

/* after cu_wait: shape d's n survivors, offsets from the unit's base, in no particular order */
const uint64_t *cu_list(int slot, int d, uint32_t n);

/* the base-2 strong probable-prime verdict of count numbers given as (lo, hi) 64-bit pairs,
   n < 2^127; ok[i] = 1 or 0 (2 counts as prime, other even n and n < 2 as not) */
int cu_sprp_batch(const uint64_t *n, size_t count, uint8_t *ok);

#ifdef __cplusplus
}
#endif

#endif
