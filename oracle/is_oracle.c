/*
 * is_oracle.c -- CPU oracle for the NPB IS path.
 *
 * TEST INFRASTRUCTURE ONLY.  This file is the oracle of the tests, never the
 * product: only tests/, __graft_entry__.smoke() and the cpu_baseline legs of
 * bench.py may load liboracle.so.  libcgb.so neither links nor calls anything
 * here.
 *
 * It restates, in plain C, the IS benchmark of the GMAP/NPB-GPU reference
 * (paths relative to that project, CUDA/IS/is.cu):
 *   - create_seq          :508-566  key i = (int)(MAX_KEY/4 * (r1+r2+r3+r4)),
 *                         r the LCG's draws 4i+1 .. 4i+4 (seed 314159265,
 *                         multiplier 5^13; randlc of c_randdp.cpp:84-114)
 *   - rank, per iteration :725-1000 key[it] = it, key[it+10] = MAX_KEY - it;
 *                         the five test keys read; the keys' counts by
 *                         value, then their running sum; each test key's
 *                         rank (count of smaller keys) checked against the
 *                         class's table with its per-class offsets
 *                         (rank_gpu_kernel_7)
 *   - main                :335-505  one untimed rank(1), then rank(1..10)
 *   - full_verify         :567-700  counting sort by the last running sums,
 *                         then the count of out-of-order neighbours
 *   - class table (TOTAL_KEYS_LOG_2, MAX_KEY_LOG_2: :86-140) and the test
 *     index / rank arrays (:157-190)
 * Verification passes when the partial checks and the full check add up to
 * 5 x 10 + 1 (:474).  Keys are 32-bit (every class's values are below
 * 2^27); counts and ranks 64-bit.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

double orc_randlc(double *x, double a); /* cg_oracle.c */

#define IS_ITER 10
#define IS_TESTS 5

/* The keys of a 2^total_log2-key, 2^max_log2-value instance (is.cu:508-566). */
int orc_is_keys(int total_log2, int max_log2, int32_t *keys)
{
    const int64_t n = (int64_t)1 << total_log2;
    const double k = (double)((int64_t)1 << max_log2) / 4.0;
    double s = 314159265.0;
    const double a = 1220703125.0;
    for (int64_t i = 0; i < n; i++) {
        double x = orc_randlc(&s, a);
        x += orc_randlc(&s, a);
        x += orc_randlc(&s, a);
        x += orc_randlc(&s, a);
        keys[i] = (int32_t)(k * x);
    }
    return 0;
}

/* The expected rank offset of test key i at iteration `it` for a class
 * (rank_gpu_kernel_7's table): +1 or -1 times the returned shift. */
static int64_t expected_rank(char cls, int i, int64_t base, int64_t it)
{
    switch (cls) {
    case 'S': return i <= 2 ? base + it : base - it;
    case 'W': return i < 2 ? base + (it - 2) : base - it;
    case 'A': return i <= 2 ? base + (it - 1) : base - (it - 1);
    case 'B': return (i == 1 || i == 2 || i == 4) ? base + it : base - it;
    case 'C': return i <= 2 ? base + it : base - it;
    default: return i < 2 ? base + it : base - it; /* 'D' */
    }
}

/* The benchmark: keys generated, one untimed rank(1), rank(1..10) with the
 * partial checks, the full check.  Returns the passed count (51 verifies);
 * counts_out (nullable, 2^max_log2 entries) receives the last running sums
 * (keys <= v). */
int64_t orc_is_run(char cls, int total_log2, int max_log2, const int64_t *test_index,
                   const int64_t *test_rank, int64_t *counts_out)
{
    const int64_t n = (int64_t)1 << total_log2, maxk = (int64_t)1 << max_log2;
    int32_t *keys = malloc(sizeof(int32_t) * n), *sorted = malloc(sizeof(int32_t) * n);
    int64_t *cnt = malloc(sizeof(int64_t) * maxk);
    if (!keys || !sorted || !cnt) {
        free(keys);
        free(sorted);
        free(cnt);
        return -1;
    }
    orc_is_keys(total_log2, max_log2, keys);
    int64_t passed = 0;
    for (int pass = 0; pass <= IS_ITER; pass++) {
        const int64_t it = pass == 0 ? 1 : pass; /* pass 0: the untimed rank(1) */
        if (pass == 1) passed = 0;
        keys[it] = (int32_t)it;
        keys[it + IS_ITER] = (int32_t)(maxk - it);
        int64_t probe[IS_TESTS];
        for (int i = 0; i < IS_TESTS; i++) probe[i] = keys[test_index[i]];
        memset(cnt, 0, sizeof(int64_t) * maxk);
        for (int64_t j = 0; j < n; j++) cnt[keys[j]]++;
        for (int64_t v = 1; v < maxk; v++) cnt[v] += cnt[v - 1];
        for (int i = 0; i < IS_TESTS; i++) {
            const int64_t key = probe[i];
            if (0 < key && key <= n - 1 && cnt[key - 1] == expected_rank(cls, i, test_rank[i], it))
                passed++;
        }
    }
    /* full_verify: place each key by the running sums, then count the
     * out-of-order neighbours */
    if (counts_out) memcpy(counts_out, cnt, sizeof(int64_t) * maxk);
    for (int64_t j = 0; j < n; j++) sorted[--cnt[keys[j]]] = keys[j];
    int64_t bad = 0;
    for (int64_t j = 1; j < n; j++) bad += sorted[j - 1] > sorted[j];
    if (bad == 0) passed++;
    free(keys);
    free(sorted);
    free(cnt);
    return passed;
}
