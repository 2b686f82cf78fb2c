/*
 * ps4_oracle_main.c -- command-line wrapper of the CPU restatement (test infrastructure).
 *
 *   ps4_oracle S_lo S_hi [--dump4 N] [--noext] [--verify] [--test-sixset] [--chunk L]
 *
 * Result lines go to stdout; TOTAL / histogram / CAPACITY lines to stderr in the
 * reference's format (exhaustive/s4.c:498-506), one region, no wall time.
 */
#include "ps4_oracle.h"

#include <stdio.h>
#include <stdlib.h>
#include <string.h>

int main(int argc, char **argv) {
    unsigned long long lo = 1, hi = 10000000ULL;
    long dump4 = 0; int flags = 0, pos = 0; unsigned chunk = 20;
    for (int i = 1; i < argc; i++) {
        if (!strcmp(argv[i], "--noext")) flags |= ORC_NOEXT;
        else if (!strcmp(argv[i], "--verify")) flags |= ORC_VERIFY;
        else if (!strcmp(argv[i], "--test-sixset")) flags |= ORC_TEST6;
        else if (!strcmp(argv[i], "--dump4") && i + 1 < argc) dump4 = atol(argv[++i]);
        else if (!strcmp(argv[i], "--chunk") && i + 1 < argc) chunk = (unsigned)atoi(argv[++i]);
        else if (++pos == 1) lo = strtoull(argv[i], 0, 10);
        else if (pos == 2) hi = strtoull(argv[i], 0, 10);
    }
    fflush(stdout);
    orc_stats st; char err[256];
    int rc = orc_search(lo, hi, chunk, dump4, flags, 0, 0, 0, "/dev/stdout", &st, err, sizeof err);
    if (rc) { fprintf(stderr, "%s\n", err); return rc; }
    fprintf(stderr, "TOTAL: S_done=%llu pairs=%llu S_ge3=%llu triples=%llu 4-sets=%llu 5-sets=%llu 6-sets=%llu "
            "multi-ext-4sets=%llu ext_cand=%llu ext_sqrt=%llu\n",
            (unsigned long long)st.S_done, (unsigned long long)st.pairs, (unsigned long long)st.S_ge3,
            (unsigned long long)st.triples, (unsigned long long)st.sets4, (unsigned long long)st.sets5,
            (unsigned long long)st.sets6, (unsigned long long)st.multi, (unsigned long long)st.ext_cand,
            (unsigned long long)st.ext_sqrt);
    fprintf(stderr, "5-sets by log2(largest element):");
    for (int i = 0; i < 100; i++) if (st.hist5[i]) fprintf(stderr, " %d:%llu", i, (unsigned long long)st.hist5[i]);
    fprintf(stderr, "\nCAPACITY: reps=%llu/512 divisors=%llu/16384 extensions=%llu/64\n",
            (unsigned long long)st.max_reps, (unsigned long long)st.max_divisors, (unsigned long long)st.max_extensions);
    return 0;
}
