/*
 * CPU restatement of the seeded index sampler (TEST INFRASTRUCTURE ONLY).
 *
 * The reference draws sample(1:NN, r, replace=false) and sorts it
 * (codes/GPU_implementation/seed/compres_single_block_spheres_for_sweep2.jl:492-495) with an
 * unseeded global RNG, so its index sets cannot be reproduced. The B200 library instead
 * draws them from Philox4x32-10 (Salmon, Moraes, Dror, Shaw, "Parallel random numbers: as
 * easy as 1, 2, 3", SC'11) with Floyd's algorithm for r distinct values out of D
 * (Bentley & Floyd, CACM 1987). This file restates that definition so tests can check the
 * device sampler bit for bit:
 *
 *   word(i)  = Philox4x32-10(counter = {i, block, round, stream}, key = {seed_lo, seed_hi})[0]
 *   for j = D-r .. D-1 (i = j-(D-r)):  t = (word(i) * (j+1)) >> 32
 *                                      take t, or j if t was already taken
 *   output   = taken values in increasing order (0-based)
 *
 * Streams: 0 = sampled rows I, 1 = sampled columns J, 2 = extra estimator rows drawn from
 * the rows not in I, 3 = extra estimator columns drawn from the columns not in J (the k-th
 * smallest unsampled index is returned for a draw of k).
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

static void philox_round(uint32_t c[4], const uint32_t k[2])
{
    const uint64_t p0 = (uint64_t)0xD2511F53u * c[0];
    const uint64_t p1 = (uint64_t)0xCD9E8D57u * c[2];
    const uint32_t hi0 = (uint32_t)(p0 >> 32), lo0 = (uint32_t)p0;
    const uint32_t hi1 = (uint32_t)(p1 >> 32), lo1 = (uint32_t)p1;
    const uint32_t n0 = hi1 ^ c[1] ^ k[0];
    const uint32_t n2 = hi0 ^ c[3] ^ k[1];
    c[0] = n0;
    c[1] = lo1;
    c[2] = n2;
    c[3] = lo0;
}

/* all four output words of Philox4x32-10 for an explicit counter and key */
void oracle_philox4(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4])
{
    uint32_t c[4] = {ctr[0], ctr[1], ctr[2], ctr[3]};
    uint32_t k[2] = {key[0], key[1]};
    for (int r = 0; r < 10; ++r) {
        philox_round(c, k);
        k[0] += 0x9E3779B9u;
        k[1] += 0xBB67AE85u;
    }
    for (int i = 0; i < 4; ++i) out[i] = c[i];
}

uint32_t oracle_philox_word(uint32_t i, uint32_t block, uint32_t round, uint32_t stream,
                            uint64_t seed)
{
    uint32_t c[4] = {i, block, round, stream};
    uint32_t k[2] = {(uint32_t)seed, (uint32_t)(seed >> 32)};
    for (int r = 0; r < 10; ++r) {
        philox_round(c, k);
        k[0] += 0x9E3779B9u;
        k[1] += 0xBB67AE85u;
    }
    return c[0];
}

/* r distinct sorted values from [0, D); returns 0 or -1 if r > D. */
int oracle_sample(int *out, int r, int D, uint32_t block, uint32_t round, uint32_t stream,
                  uint64_t seed)
{
    if (r < 0 || r > D) return -1;
    unsigned char *taken = (unsigned char *)calloc((size_t)D + 1, 1);
    if (!taken) return -1;
    for (int j = D - r, i = 0; j < D; ++j, ++i) {
        const uint32_t w = oracle_philox_word((uint32_t)i, block, round, stream, seed);
        const uint32_t t = (uint32_t)(((uint64_t)w * (uint64_t)(j + 1)) >> 32);
        if (taken[t]) taken[j] = 1; else taken[t] = 1;
    }
    int n = 0;
    for (int v = 0; v < D; ++v)
        if (taken[v]) out[n++] = v;
    free(taken);
    return 0;
}

/* p extra indices drawn from the complement of the sorted set I (size r) in [0, m); stream 2
   for extra rows, 3 for extra columns. */
int oracle_sample_extra(int *out, int p, const int *I, int r, int m, uint32_t block,
                        uint32_t round, uint32_t stream, uint64_t seed)
{
    const int free_rows = m - r;
    if (p > free_rows) p = free_rows;
    if (p <= 0) return 0;
    int *pick = (int *)malloc(sizeof(int) * (size_t)p);
    if (!pick) return -1;
    oracle_sample(pick, p, free_rows, block, round, stream, seed);
    /* map the k-th free row to its index */
    int k = 0, ii = 0, n = 0;
    for (int v = 0; v < m && n < p; ++v) {
        if (ii < r && I[ii] == v) { ++ii; continue; }
        if (k == pick[n]) out[n++] = v;
        ++k;
    }
    free(pick);
    return p;
}
