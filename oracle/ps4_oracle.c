/*
 * ps4_oracle.c -- CPU restatement of the reference census engine exhaustive/s4.c.
 *
 * TEST INFRASTRUCTURE ONLY (see ps4_oracle.h).  Single-threaded and written for
 * clarity: it follows the reference's algorithm step by step so that every counter
 * and every output line agrees with it, and it is deliberately independent of the
 * CUDA path's restructured enumeration (closed-form triple ranges, halved divisor
 * walk, residue folding), so that a mismatch between the two points at a bug.
 * Each function cites the reference lines it restates.
 */
#define _GNU_SOURCE
#include "ps4_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;
typedef uint64_t u64;
typedef int64_t i64;
typedef uint32_t u32;

/* ------------------------------------------------------------------ exact roots */

/* floor(sqrt(n)), n < 2^64.  Estimate from libm, then exact integer correction
 * (restates s4.c:95-100, including the clamp that keeps (r+1)^2 in range). */
static u64 orc_isqrt64(u64 n) {
    u64 r = (u64)sqrt((double)n);
    if (r > 0xFFFFFFFFull) r = 0xFFFFFFFFull;
    while (r * r > n) r--;
    while (r < 0xFFFFFFFFull && (r + 1) * (r + 1) <= n) r++;
    return r;
}

/* floor(sqrt(n)), n < 2^128 (restates s4.c:101-107). */
static u64 orc_isqrt_u128(u128 n) {
    if (n >> 64 == 0) return orc_isqrt64((u64)n);
    u64 r = (u64)sqrtl((long double)n);
    while ((u128)r * r > n) r--;
    while ((u128)(r + 1) * (r + 1) <= n) r++;
    return r;
}

static int orc_is_sq(u128 n) {             /* s4.c:108 */
    u64 r = orc_isqrt_u128(n);
    return (u128)r * r == n;
}

uint64_t orc_isqrt128(uint64_t hi, uint64_t lo) { return orc_isqrt_u128(((u128)hi << 64) | lo); }
int orc_is_square128(uint64_t hi, uint64_t lo) { return orc_is_sq(((u128)hi << 64) | lo); }

/* ------------------------------------------------------------------ tables */

/* Tables over m < n (s4.c:436-447): smallest prime factor, cofactor m/spf(m), divisor
 * count, and the quadratic-residue flags mod 64, 63, 65.  Built here with a linear
 * sieve and the multiplicative divisor-count recurrence instead of the reference's
 * trial sieve and O(n log n) divisor sieve; the contents are identical. */
typedef struct {
    u64 n;
    u32 *spf, *quot;
    uint16_t *ndiv;
    unsigned char qr64[64], qr63[63], qr65[65];
} orc_tables;

static int tables_build(orc_tables *t, u64 n) {
    memset(t, 0, sizeof *t);
    t->n = n;
    t->spf = calloc(n, sizeof(u32));
    t->quot = calloc(n, sizeof(u32));
    t->ndiv = calloc(n, sizeof(uint16_t));
    unsigned char *expo = calloc(n, 1);
    u32 *rest = calloc(n, sizeof(u32));
    u32 *primes = malloc(sizeof(u32) * (n / 2 + 16));
    if (!t->spf || !t->quot || !t->ndiv || !expo || !rest || !primes) return -1;
    u64 np = 0;
    for (u64 m = 2; m < n; m++) {
        if (t->spf[m] == 0) { t->spf[m] = (u32)m; primes[np++] = (u32)m; }
        for (u64 j = 0; j < np && primes[j] <= t->spf[m] && m * primes[j] < n; j++)
            t->spf[m * primes[j]] = primes[j];
    }
    if (n > 0) { t->spf[0] = 0; t->quot[0] = 0; }
    if (n > 1) { t->spf[1] = 1; t->quot[1] = 1; t->ndiv[1] = 1; rest[1] = 1; }
    for (u64 m = 2; m < n; m++) {
        u32 p = t->spf[m], c = (u32)(m / p);
        t->quot[m] = c;
        if (c > 1 && t->spf[c] == p) { expo[m] = (unsigned char)(expo[c] + 1); rest[m] = rest[c]; }
        else { expo[m] = 1; rest[m] = c; }
        t->ndiv[m] = (uint16_t)(t->ndiv[rest[m]] * (expo[m] + 1));
    }
    free(expo); free(rest); free(primes);
    for (int i = 0; i < 64; i++) t->qr64[(i * i) & 63] = 1;
    for (int i = 0; i < 63; i++) t->qr63[(i * i) % 63] = 1;
    for (int i = 0; i < 65; i++) t->qr65[(i * i) % 65] = 1;
    return 0;
}

static void tables_free(orc_tables *t) { free(t->spf); free(t->quot); free(t->ndiv); }

/* ------------------------------------------------------------------ output */

typedef struct {
    FILE *out;
    orc_stats *st;
    const orc_tables *tb;
    long dump4, dumped;
    int flags, test6_fired, failed;
    unsigned cap_reps, cap_divs, cap_ext;
    char *err; size_t errlen;
} orc_run;

static void fail(orc_run *r, const char *msg) {
    if (!r->failed) snprintf(r->err, r->errlen, "FATAL: %s; this interval is NOT certified complete", msg);
    r->failed = 1;
}

static void put_u128(FILE *f, u128 v) {          /* decimal, as s4.c:110-114 */
    char tmp[48]; int i = 0;
    if (v == 0) { fputc('0', f); return; }
    while (v) { tmp[i++] = (char)('0' + (int)(v % 10)); v /= 10; }
    while (i) fputc(tmp[--i], f);
}

/* all pairwise sums square and members distinct (s4.c:209-212) */
static int set_ok(const u128 *x, int n) {
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++)
            if (x[i] == x[j] || !orc_is_sq(x[i] + x[j])) return 0;
    return 1;
}

/* "tag [members, largest first] S=..." plus the verify marker (s4.c:214-220) */
static void put_set(FILE *f, const char *tag, u128 *x, int n, u64 S) {
    for (int i = 1; i < n; i++) {                      /* insertion sort, descending */
        u128 key = x[i]; int j = i - 1;
        while (j >= 0 && x[j] < key) { x[j + 1] = x[j]; j--; }
        x[j + 1] = key;
    }
    fprintf(f, "%s [", tag);
    for (int i = 0; i < n; i++) { put_u128(f, x[i]); if (i < n - 1) fputc(',', f); }
    fprintf(f, "] S=%llu%s\n", (unsigned long long)S, set_ok(x, n) ? "" : "  *** VERIFY FAILED ***");
}

/* ------------------------------------------------------------------ extension */

typedef struct { u64 p[24]; int e[24]; int n; } orc_fact;

/* merge the prime factorisation of m into f, new primes appended in the order the
 * smallest-prime-factor walk meets them (s4.c:141-147) */
static void fact_merge(const orc_tables *tb, orc_fact *f, u64 m) {
    while (m > 1) {
        u64 pr = tb->spf[m]; int e = 0;
        while (m > 1 && tb->spf[m] == pr) { m = tb->quot[m]; e++; }
        int i = 0;
        while (i < f->n && f->p[i] != pr) i++;
        if (i == f->n) { f->p[f->n] = pr; f->e[f->n] = 0; f->n++; }
        f->e[i] += e;
    }
}

/* divisors in mixed-radix order, first prime fastest (s4.c:149-156); -1 past cap */
static long divisors_mixed_radix(const orc_fact *f, u64 *out, long cap) {
    long n = 1; out[0] = 1;
    for (int i = 0; i < f->n; i++) {
        long block = n; u64 pk = 1;
        for (int e = 1; e <= f->e[i]; e++) {
            pk *= f->p[i];
            for (long j = 0; j < block; j++) { if (n >= cap) return -1; out[n++] = out[j] * pk; }
        }
    }
    return n;
}

/* every e extending the 4-set v (roots rt) -- restates extend4, s4.c:160-207 */
static int extend_quad(orc_run *r, const u64 v[4], u32 rt[4][4], u128 *ext, u64 *divs) {
    static const int pairs[6][3] = {{0,1,2},{2,3,0},{0,2,1},{1,3,0},{0,3,1},{1,2,0}};
    const orc_tables *tb = r->tb;
    u64 best = ~0ull; int bi = 0, bj = 1, bk = 2;
    for (int t = 0; t < 6; t++) {                   /* cheapest difference, first wins ties */
        int i = pairs[t][0], j = pairs[t][1], k = pairs[t][2];
        if (v[i] < v[j]) { int s = i; i = j; j = s; }
        u64 ra = rt[i][k], rb = rt[j][k];
        u64 est = (u64)tb->ndiv[ra - rb] * tb->ndiv[ra + rb];
        if (est < best) { best = est; bi = i; bj = j; bk = k; }
    }
    u64 A = v[bi];
    orc_fact fa; fa.n = 0;
    fact_merge(tb, &fa, (u64)rt[bi][bk] - rt[bj][bk]);
    fact_merge(tb, &fa, (u64)rt[bi][bk] + rt[bj][bk]);
    long nd = divisors_mixed_radix(&fa, divs, r->cap_divs);
    if (nd < 0) { fail(r, "divisor capacity exceeded"); return 0; }
    if ((u64)nd > r->st->max_divisors) r->st->max_divisors = (u64)nd;
    int o[2], no = 0;
    for (int t = 0; t < 4; t++) if (t != bi && t != bj) o[no++] = t;
    u64 C1 = v[o[0]], C2 = v[o[1]];
    i64 d1 = (i64)C1 - (i64)A, d2 = (i64)C2 - (i64)A;
    /* residues of e+C = u^2 + d modulo 64, 63, 65 */
    u64 r1[3], r2[3];
    const i64 mods[3] = {64, 63, 65};
    for (int m = 0; m < 3; m++) { r1[m] = (u64)(((d1 % mods[m]) + mods[m]) % mods[m]); r2[m] = (u64)(((d2 % mods[m]) + mods[m]) % mods[m]); }
    int ne = 0;
    for (long t = 0; t < nd; t++) {
        u64 f = divs[t], g = divs[nd - 1 - t];        /* complementary in mixed-radix order */
        if (f >= g || ((f ^ g) & 1)) continue;
        u64 u = (f + g) >> 1;
        r->st->ext_cand++;
        u64 w = u & 63;
        if (!tb->qr64[(w * w + r1[0]) & 63] || !tb->qr64[(w * w + r2[0]) & 63]) continue;
        w = u % 63;
        if (!tb->qr63[(w * w + r1[1]) % 63] || !tb->qr63[(w * w + r2[1]) % 63]) continue;
        w = u % 65;
        if (!tb->qr65[(w * w + r1[2]) % 65] || !tb->qr65[(w * w + r2[2]) % 65]) continue;
        u128 usq = (u128)u * u;
        if (usq <= A) continue;
        u128 e = usq - A;
        if (e == v[0] || e == v[1] || e == v[2] || e == v[3]) continue;
        r->st->ext_sqrt++;
        if (!orc_is_sq(e + C1) || !orc_is_sq(e + C2)) continue;
        if ((unsigned)ne >= r->cap_ext) { fail(r, "extension capacity exceeded"); return ne; }
        ext[ne++] = e;
    }
    if ((u64)ne > r->st->max_extensions) r->st->max_extensions = (u64)ne;
    return ne;
}

/* one 4-set: verify, dump, extend, report (restates handle_4set, s4.c:225-278) */
static void on_quad(orc_run *r, u64 S, i64 a, i64 b, i64 c, i64 d,
                    u32 r_ab, u32 r_ac, u32 r_ad, u32 r_bc, u32 r_bd, u32 r_cd,
                    u128 *ext, u64 *divs) {
    u64 v[4] = {(u64)a, (u64)b, (u64)c, (u64)d};
    u32 rt[4][4] = {{0, r_ab, r_ac, r_ad}, {r_ab, 0, r_bc, r_bd}, {r_ac, r_bc, 0, r_cd}, {r_ad, r_bd, r_cd, 0}};
    if (r->flags & ORC_VERIFY) {
        for (int i = 0; i < 4; i++)
            for (int j = i + 1; j < 4; j++)
                if ((u64)rt[i][j] * rt[i][j] != v[i] + v[j] || v[i] == v[j]) {
                    fprintf(r->out, "BAD 4-set S=%llu [%lld,%lld,%lld,%lld]\n", (unsigned long long)S,
                            (long long)a, (long long)b, (long long)c, (long long)d);
                    fail(r, "quadruple verification failed");
                    return;
                }
    }
    r->st->sets4++;
    if (r->dump4 && r->dumped < r->dump4) {
        r->dumped++;
        fprintf(r->out, "4: [%lld,%lld,%lld,%lld] S=%llu\n", (long long)a, (long long)b, (long long)c,
                (long long)d, (unsigned long long)S);
    }
    if (r->flags & ORC_NOEXT) return;
    int ne = extend_quad(r, v, rt, ext, divs);
    if (r->failed || ne == 0) return;
    u64 vmax = v[0];
    for (int i = 1; i < 4; i++) if (v[i] > vmax) vmax = v[i];
    if (ne >= 2) {
        r->st->multi++;
        fprintf(r->out, "M: [%llu,%llu,%llu,%llu] ext=[", (unsigned long long)v[0], (unsigned long long)v[1],
                (unsigned long long)v[2], (unsigned long long)v[3]);
        for (int t = 0; t < ne; t++) { put_u128(r->out, ext[t]); if (t < ne - 1) fputc(',', r->out); }
        fprintf(r->out, "] S=%llu\n", (unsigned long long)S);
        if ((r->flags & ORC_TEST6) && !r->test6_fired) {
            r->test6_fired = 1;
            u128 x[6] = {v[0], v[1], v[2], v[3], ext[0], ext[1]};
            put_set(r->out, "TEST-6SET (NOT A SOLUTION, --test-sixset drill):", x, 6, S);
        }
    }
    for (int t = 0; t < ne; t++) {
        if (ext[t] <= vmax) continue;
        r->st->sets5++;
        int lg = 0; u128 e = ext[t];
        while (e > 1) { e >>= 1; lg++; }
        r->st->hist5[lg > 99 ? 99 : lg]++;
        u128 x[5] = {v[0], v[1], v[2], v[3], ext[t]};
        put_set(r->out, "5:", x, 5, S);
    }
    for (int t = 0; t < ne; t++)
        for (int s = t + 1; s < ne; s++)
            if (orc_is_sq(ext[t] + ext[s])) {
                r->st->sets6++;
                u128 x[6] = {v[0], v[1], v[2], v[3], ext[t], ext[s]};
                put_set(r->out, "!!!!!!!! FOUND 6-SET:", x, 6, S);
            }
}

/* ------------------------------------------------------------------ chunks */

/* every S in [S0,S1): bucket the representations S = p^2+q^2 (1<=p<=q) by S with a
 * counting sort, then build every 4-set from each triple of representations
 * (restates process_chunk, s4.c:280-341).  Each chunk starts its q cursors afresh. */
static void do_chunk(orc_run *r, u64 S0, u64 S1, uint16_t *cnt, u32 *off, u32 **pv, u64 *pvcap,
                     u64 *pl, u64 *ql, u64 *P, u64 *Q, u128 *ext, u64 *divs) {
    u64 n = S1 - S0;
    u64 pmax = orc_isqrt64((S1 - 1) / 2);
    memset(cnt, 0, n * sizeof *cnt);
    /* first q >= p with p^2+q^2 >= S0 */
#define FIRST_Q(p) ({ u64 _q = (p); if (S0 > 2 * (p) * (p)) { _q = orc_isqrt64(S0 - (p) * (p)); if (_q * _q < S0 - (p) * (p)) _q++; } _q; })
    for (u64 p = 1; p <= pmax; p++)
        for (u64 q = FIRST_Q(p), s = p * p + q * q; s < S1; s += 2 * q + 1, q++) cnt[s - S0]++;
    u64 total = 0;
    for (u64 i = 0; i < n; i++) { off[i] = (u32)total; total += cnt[i]; }
    r->st->pairs += total;
    if (total > *pvcap) { *pvcap = total + total / 4 + 1024; *pv = realloc(*pv, *pvcap * sizeof(u32)); }
    for (u64 p = 1; p <= pmax; p++)
        for (u64 q = FIRST_Q(p), s = p * p + q * q; s < S1; s += 2 * q + 1, q++) (*pv)[off[s - S0]++] = (u32)p;
#undef FIRST_Q
    for (u64 i = 0; i < n && !r->failed; i++) {
        unsigned k = cnt[i];
        r->st->S_done++;
        if (k > r->st->max_reps) r->st->max_reps = k;
        u64 S = S0 + i;
        if (k < 3 || (S & 3) == 2) continue;           /* 4-subsets of 5-/6-sets never have S = 2 mod 4 */
        r->st->S_ge3++;
        if (k > r->cap_reps) { fail(r, "representation capacity exceeded"); return; }
        u64 start = off[i] - k;                        /* off[i] now points past S's bucket */
        for (unsigned t = 0; t < k; t++) {
            pl[t] = (*pv)[start + t]; P[t] = pl[t] * pl[t]; Q[t] = S - P[t]; ql[t] = orc_isqrt64(Q[t]);
        }
        int Sodd = (int)(S & 1);
        for (unsigned x = 0; x < k; x++)
            for (unsigned y = x + 1; y < k; y++)
                for (unsigned z = y + 1; z < k; z++) {
                    r->st->triples++;
                    int par = (int)((pl[x] + pl[y] + pl[z]) & 1);
                    for (int cls = 0; cls < 2; cls++) {
                        /* class 0 pairs (Q_x,Q_y,Q_z), class 1 (Q_x,Q_y,P_z); S=2p^2 makes them coincide */
                        if (cls == 0 ? par != 0 : (par != Sodd || Q[z] == P[z])) continue;
                        i64 x1 = (i64)Q[x], x2 = (i64)Q[y], x3 = (i64)(cls == 0 ? Q[z] : P[z]), SS = (i64)S;
                        i64 a = (x1 + x2 + x3 - SS) / 2, b = (x1 - x2 - x3 + SS) / 2;
                        i64 c = (-x1 + x2 - x3 + SS) / 2, d = (-x1 - x2 + x3 + SS) / 2;
                        if (a <= 0 || b <= 0 || c <= 0 || d <= 0) continue;
                        u32 r_ad = (u32)(cls == 0 ? ql[z] : pl[z]);
                        u32 r_bc = (u32)(cls == 0 ? pl[z] : ql[z]);
                        on_quad(r, S, a, b, c, d, (u32)ql[x], (u32)ql[y], r_ad, r_bc, (u32)pl[y], (u32)pl[x], ext, divs);
                        if (r->failed) return;
                    }
                }
    }
}

int orc_search(uint64_t lo, uint64_t hi, unsigned chunk_log2, long dump4, int flags,
               unsigned cap_reps, unsigned cap_divs, unsigned cap_ext,
               const char *out_path, orc_stats *st, char *err, size_t errlen) {
    if (lo < 1) lo = 1;
    memset(st, 0, sizeof *st);
    if (err && errlen) err[0] = 0;
    if (hi <= lo) return 0;
    if (chunk_log2 == 0 || chunk_log2 > 30) chunk_log2 = 20;
    FILE *out = fopen(out_path, "a");
    if (!out) { if (err) snprintf(err, errlen, "cannot open %s", out_path); return 1; }
    orc_tables tb;
    if (tables_build(&tb, 2 * orc_isqrt64(hi) + 64) != 0) { fclose(out); return 1; }
    orc_run r = {out, st, &tb, dump4, 0, flags, 0, 0,
                 cap_reps ? cap_reps : 512, cap_divs ? cap_divs : 16384, cap_ext ? cap_ext : 64, err, errlen};
    u64 W = 1ull << chunk_log2;
    uint16_t *cnt = malloc(W * sizeof *cnt);
    u32 *off = malloc((W + 1) * sizeof *off);
    u64 pvcap = W / 2 + 4096;
    u32 *pv = malloc(pvcap * sizeof *pv);
    unsigned kc = r.cap_reps;
    u64 *pl = malloc(kc * sizeof(u64)), *ql = malloc(kc * sizeof(u64)), *P = malloc(kc * sizeof(u64)), *Q = malloc(kc * sizeof(u64));
    u128 *ext = malloc((r.cap_ext + 1) * sizeof(u128));
    u64 *divs = malloc((u64)r.cap_divs * sizeof(u64));
    for (u64 S0 = lo; S0 < hi && !r.failed; S0 += W) {
        u64 S1 = S0 + W < hi ? S0 + W : hi;
        do_chunk(&r, S0, S1, cnt, off, &pv, &pvcap, pl, ql, P, Q, ext, divs);
    }
    free(cnt); free(off); free(pv); free(pl); free(ql); free(P); free(Q); free(ext); free(divs);
    tables_free(&tb);
    fclose(out);
    return r.failed ? 2 : 0;
}

/* ------------------------------------------------------------------ triple extension */

static void factor_trial(orc_fact *f, u64 m) {        /* fresh primes appended ascending */
    for (u64 p = 2; p * p <= m; p++) {
        if (m % p) continue;
        int e = 0;
        while (m % p == 0) { m /= p; e++; }
        int i = 0;
        while (i < f->n && f->p[i] != p) i++;
        if (i == f->n) { f->p[f->n] = p; f->e[f->n] = 0; f->n++; }
        f->e[i] += e;
    }
    if (m > 1) {
        int i = 0;
        while (i < f->n && f->p[i] != m) i++;
        if (i == f->n) { f->p[f->n] = m; f->e[f->n] = 0; f->n++; }
        f->e[i] += 1;
    }
}

static int cmp_u64(const void *x, const void *y) {
    u64 a = *(const u64 *)x, b = *(const u64 *)y;
    return a < b ? -1 : a > b;
}

long orc_extend_triple(uint64_t a, uint64_t b, uint64_t c, uint64_t dmax, uint64_t *out, long cap) {
    u64 m[3] = {a, b, c};
    qsort(m, 3, sizeof m[0], cmp_u64);
    if (m[0] == 0 || m[0] == m[1] || m[1] == m[2]) return -1;
    if (!orc_is_sq((u128)m[0] + m[1]) || !orc_is_sq((u128)m[0] + m[2]) || !orc_is_sq((u128)m[1] + m[2])) return -1;
    /* D = m2 - m1 = (r02 - r12)... use A = m[2] > B = m[1] with third member C = m[0]:
       e + A = u^2, e + B = w^2  =>  (u - w)(u + w) = A - B = r(A+C)^2 - r(B+C)^2 */
    u64 A = m[2], B = m[1], C = m[0];
    u64 rA = orc_isqrt_u128((u128)A + C), rB = orc_isqrt_u128((u128)B + C);
    orc_fact fa; fa.n = 0;
    factor_trial(&fa, rA - rB);
    factor_trial(&fa, rA + rB);
    long nd = 1;
    for (int i = 0; i < fa.n; i++) nd *= fa.e[i] + 1;
    u64 *divs = malloc(sizeof(u64) * (size_t)nd);
    divisors_mixed_radix(&fa, divs, nd);
    u64 umax = orc_isqrt_u128((u128)dmax + A);
    long cnt = 0;
    for (long t = 0; t < nd; t++) {
        u64 f = divs[t], g = divs[nd - 1 - t];
        if (f >= g || ((f ^ g) & 1)) continue;
        u64 u = (f + g) >> 1;
        if (u > umax) continue;
        u128 usq = (u128)u * u;
        if (usq <= A) continue;
        u128 e = usq - A;                               /* e + B = ((g - f)/2)^2 by construction */
        if (e > dmax || e == A || e == B || e == C) continue;
        if (!orc_is_sq(e + C)) continue;
        if (cnt < cap) out[cnt] = (u64)e;
        cnt++;
    }
    free(divs);
    if (cnt <= cap) qsort(out, (size_t)cnt, sizeof out[0], cmp_u64);
    return cnt;
}
