/*
 * ps4_oracle.h -- CPU restatement of the reference census engine (exhaustive/s4.c).
 *
 * TEST INFRASTRUCTURE ONLY.  This is the checker the parity tests, smoke() and the
 * cpu_baseline leg of bench.py compare the CUDA path against.  The product library
 * (libps4.so) never links, loads or calls it.
 *
 * Parity pin: the restatement reproduces the reference's golden vectors
 * (sorted-output sha256 and every TOTAL counter at S<1e7 and S<1e9, the singleton-S
 * logs exhaustive/logs/boundary_*.err, the known five-sets of exhaustive/test_verify.py)
 * -- see tests/test_oracle.py.
 */
#ifndef PS4_ORACLE_H
#define PS4_ORACLE_H
#include <stdint.h>
#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

/* Counters of one search, same meaning as the reference's stats_t (exhaustive/s4.c:80-91). */
typedef struct {
    uint64_t S_done, pairs, S_ge3, triples, sets4, sets5, sets6, multi, ext_cand, ext_sqrt;
    uint64_t hist5[100];
    uint64_t max_reps, max_divisors, max_extensions;
} orc_stats;

enum {
    ORC_NOEXT  = 1,   /* --noext  (s4.c:242)            */
    ORC_VERIFY = 2,   /* --verify (s4.c:229-233)        */
    ORC_TEST6  = 4    /* --test-sixset drill (s4.c:255) */
};

/* Search every S in [lo, hi).  Result lines are appended to the file `out_path`
 * (the 6-set alert lines too; the oracle writes no SIXSET_FOUND.txt).
 * chunk_log2 is the reference's chunk width; results never depend on it.
 * dump4: emit the first `dump4` 4-sets as "4:" lines (0 = none).
 * cap_*: capacity caps (reference defaults 512 / 16384 / 64).
 * Returns 0 on success, 2 on a capacity failure with the reference's FATAL text in err. */
int orc_search(uint64_t lo, uint64_t hi, unsigned chunk_log2, long dump4, int flags,
               unsigned cap_reps, unsigned cap_divs, unsigned cap_ext,
               const char *out_path, orc_stats *st, char *err, size_t errlen);

/* floor(sqrt(n)) for n < 2^128 given as (hi, lo) 64-bit halves; exact. */
uint64_t orc_isqrt128(uint64_t hi, uint64_t lo);
int orc_is_square128(uint64_t hi, uint64_t lo);

/* Triple extension (the batched "extend this triple" query, for which the reference
 * has no function; this restates the reference's extension step, s4.c:160-207, for a
 * three-element set).  For distinct positive a,b,c with a+b, a+c, b+c all square, find
 * every d with 0 < d <= dmax, d not in {a,b,c}, and d+a, d+b, d+c all square.
 * Writes up to `cap` values ascending into out; returns the total count (may exceed cap),
 * or -1 if (a,b,c) is not a valid triple. */
long orc_extend_triple(uint64_t a, uint64_t b, uint64_t c, uint64_t dmax, uint64_t *out, long cap);

#ifdef __cplusplus
}
#endif
#endif
