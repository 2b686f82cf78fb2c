/*
 * s4gpu.c -- drop-in replacement of the reference's census process `s4` (exhaustive/s4.c)
 * that runs the search on a B200 through libps4.
 *
 *   s4gpu S_lo S_hi [threads=auto] [log2 chunk=20] [--out FILE] [--ckpt FILE] [--resume]
 *                                  [--noext] [--verify] [--dump4 N] [--test-sixset]
 *
 * Same argv grammar (s4.c:414-431), result lines (s4.c:24-27), stderr header / thread /
 * TOTAL / histogram / CAPACITY lines (s4.c:459-506), `s4ckpt v1` checkpoint (s4.c:367-412)
 * and exit codes (0 ok, 1 usage/IO/checkpoint mismatch, 2 FATAL capacity or verify).
 * "threads" keeps its meaning as the number of equal S regions the interval is split into
 * (s4.c:452-456), so checkpoints stay interchangeable with the reference's; the regions are
 * searched on the GPU one batch of whole chunks at a time.  Capacity caps can be lowered
 * for failure-injection tests through the environment variables S4_MAX_REPS / S4_MAX_DIVS /
 * S4_MAX_EXT (the reference's compile-time macros of the same names, s4.c:45-54).
 *
 * SIGTERM / SIGINT (a block controller's deadline, run_exhaustive.py:221-224) stop the run at
 * the next batch boundary: the checkpoint is written with the positions reached (no DONE),
 * the results are flushed, and the signal is raised again with its default action, so the
 * exit status is the reference's (killed by that signal) and a --resume continues without
 * repeating or losing a line.  No kernel is cut off mid-launch.
 */
#define _GNU_SOURCE
#include <signal.h>
#include <stdint.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>
#include <time.h>
#include <unistd.h>

#include "../../include/ps4.h"

typedef uint64_t u64;

static u64 S_lo = 1, S_hi = 10000000ULL;
static int nthreads = 0;
static u64 W = 1ull << 20;
static int opt_noext = 0, opt_verify = 0, opt_resume = 0, opt_test6 = 0, test6_fired = 0;
static long opt_dump4 = 0;
static const char *opt_out = NULL, *opt_ckpt = NULL;
static FILE *out_fp = NULL;
static unsigned cap_reps = 512, cap_divs = 16384, cap_ext = 64;

typedef struct {
    ps4_stats s;        /* cumulative counters (restored from a checkpoint on resume) */
    u64 region_lo, region_hi, next_S0;
    u64 hist_run[100];  /* this run only */
    double secs;
    long dumped;
} region_t;

static double now_sec(void) {
    struct timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return ts.tv_sec + ts.tv_nsec * 1e-9;
}

static void fatal_exit(const char *msg) {              /* msg already carries "FATAL: ..." */
    fprintf(stderr, "%s\n", msg);
    fflush(stderr);
    exit(2);
}

static void write_out(const char *s, size_t n) {
    if (n && (fwrite(s, 1, n, out_fp) != n || fflush(out_fp) != 0))
        fatal_exit("FATAL: result output failed; this interval is NOT certified complete");
}

/* a 6-set, or the drill: at once + fsync to the results, SIXSET_FOUND.txt and stderr (s4.c:129-137) */
static void durable_alert(const char *line) {
    FILE *f = fopen("SIXSET_FOUND.txt", "a");
    if (f) { fputs(line, f); fflush(f); fsync(fileno(f)); fclose(f); }
    fputs(line, out_fp); fflush(out_fp); fsync(fileno(out_fp));
    fputs(line, stderr); fflush(stderr);
}

/* ---------- checkpoint, format s4ckpt v1 (s4.c:367-412) ---------- */
static void write_ckpt(region_t *rg, int done_all) {
    if (!opt_ckpt) return;
    fflush(out_fp);
    fsync(fileno(out_fp));
    char tmp[4200];
    snprintf(tmp, sizeof tmp, "%s.tmp", opt_ckpt);
    FILE *f = fopen(tmp, "w");
    if (!f) { perror("checkpoint open"); return; }
    fprintf(f, "s4ckpt v1\n%llu %llu %d %llu\n", (unsigned long long)S_lo, (unsigned long long)S_hi, nthreads,
            (unsigned long long)W);
    for (int t = 0; t < nthreads; t++) {
        const ps4_stats *s = &rg[t].s;
        fprintf(f, "%d %llu %llu %llu %llu %llu %llu %llu %llu %llu %llu %llu %llu\n", t,
                (unsigned long long)rg[t].next_S0, (unsigned long long)rg[t].region_hi,
                (unsigned long long)s->S_done, (unsigned long long)s->pairs, (unsigned long long)s->S_ge3,
                (unsigned long long)s->triples, (unsigned long long)s->sets4, (unsigned long long)s->sets5,
                (unsigned long long)s->sets6, (unsigned long long)s->multi, (unsigned long long)s->ext_cand,
                (unsigned long long)s->ext_sqrt);
    }
    if (done_all) fprintf(f, "DONE\n");
    fflush(f);
    fsync(fileno(f));
    fclose(f);
    if (rename(tmp, opt_ckpt) != 0) perror("checkpoint rename");
}

static int ckpt_thread_count(void) {
    FILE *f = fopen(opt_ckpt, "r");
    if (!f) return -1;
    char hdr[64];
    unsigned long long a, b, d;
    int c = -1;
    if (!fgets(hdr, sizeof hdr, f) || fscanf(f, "%llu %llu %d %llu", &a, &b, &c, &d) != 4) c = -1;
    fclose(f);
    return c;
}

/* 0 = no checkpoint, 1 = positions restored, 2 = range already complete */
static int read_ckpt(region_t *rg) {
    FILE *f = fopen(opt_ckpt, "r");
    if (!f) return 0;
    char hdr[64];
    if (!fgets(hdr, sizeof hdr, f) || strncmp(hdr, "s4ckpt v1", 9)) {
        fprintf(stderr, "checkpoint %s: bad header\n", opt_ckpt);
        exit(1);
    }
    unsigned long long a, b, d;
    int c;
    if (fscanf(f, "%llu %llu %d %llu\n", &a, &b, &c, &d) != 4 || a != S_lo || b != S_hi || c != nthreads || d != W) {
        fprintf(stderr, "checkpoint %s was written for S_lo=%llu S_hi=%llu threads=%d chunk=%llu; current parameters differ\n",
                opt_ckpt, a, b, c, d);
        exit(1);
    }
    for (int t = 0; t < nthreads; t++) {
        int id;
        unsigned long long ns, rh, v[10];
        if (fscanf(f, "%d %llu %llu %llu %llu %llu %llu %llu %llu %llu %llu %llu %llu\n", &id, &ns, &rh, &v[0], &v[1],
                   &v[2], &v[3], &v[4], &v[5], &v[6], &v[7], &v[8], &v[9]) != 13 ||
            id != t || rh != rg[t].region_hi) {
            fprintf(stderr, "checkpoint %s: bad line for thread %d\n", opt_ckpt, t);
            exit(1);
        }
        rg[t].region_lo = ns > rg[t].region_hi ? rg[t].region_hi : ns;
        ps4_stats *s = &rg[t].s;
        s->S_done = v[0]; s->pairs = v[1]; s->S_ge3 = v[2]; s->triples = v[3]; s->sets4 = v[4];
        s->sets5 = v[5]; s->sets6 = v[6]; s->multi = v[7]; s->ext_cand = v[8]; s->ext_sqrt = v[9];
    }
    char tail[16];
    int done = (fgets(tail, sizeof tail, f) != NULL && !strncmp(tail, "DONE", 4));
    fclose(f);
    return done ? 2 : 1;
}

/* ---------- result buffers ---------- */
typedef struct {
    ps4_results r;
    char *text; size_t text_cap, text_len;
} batch_out;

static void text_append(batch_out *b, const char *s, size_t n) {
    if (b->text_len + n + 1 > b->text_cap) {
        b->text_cap = (b->text_len + n + 1) * 2 + 65536;
        b->text = realloc(b->text, b->text_cap);
        if (!b->text) { perror("realloc"); exit(1); }
    }
    memcpy(b->text + b->text_len, s, n);
    b->text_len += n;
}

static void ensure(void **p, uint64_t *cap, uint64_t need, size_t elem) {
    if (need <= *cap) return;
    *cap = need + need / 2 + 1024;
    *p = realloc(*p, *cap * elem);
    if (!*p) { perror("realloc"); exit(1); }
}

static int cmp_key(u64 S1, const uint32_t *o1, u64 S2, const uint32_t *o2) {
    if (S1 != S2) return S1 < S2 ? -1 : 1;
    for (int i = 0; i < 4; i++)
        if (o1[i] != o2[i]) return o1[i] < o2[i] ? -1 : 1;
    return 0;
}

typedef struct { u64 S; uint32_t order[4]; uint64_t idx; } qkey;
static int cmp_qkey(const void *x, const void *y) {
    const qkey *a = x, *b = y;
    return cmp_key(a->S, a->order, b->S, b->order);
}

/* one batch [lo,hi) of region rg: search, then write its lines in the reference's order */
static void run_batch(ps4_ctx *ctx, region_t *rg, u64 lo, u64 hi, batch_out *b) {
    for (;;) {
        b->r.n_hits = b->r.n_exts = b->r.n_sixes = b->r.n_quads = 0;
        int want_dump = opt_dump4 && rg->dumped < opt_dump4;
        uint64_t qcap_saved = b->r.quads_cap;
        if (!want_dump) b->r.quads_cap = 0;
        ps4_stats add;
        memset(&add, 0, sizeof add);
        int rc = ps4_search_range(ctx, lo, hi, &add, &b->r);
        if (!want_dump) b->r.quads_cap = qcap_saved;
        if (rc == PS4_ERR_OUTPUT_FULL) {
            ensure((void **)&b->r.hits, &b->r.hits_cap, b->r.n_hits, sizeof(ps4_hit));
            ensure((void **)&b->r.exts, &b->r.exts_cap, b->r.n_exts, sizeof(ps4_ext));
            ensure((void **)&b->r.sixes, &b->r.sixes_cap, b->r.n_sixes, sizeof(ps4_six));
            if (want_dump) ensure((void **)&b->r.quads, &b->r.quads_cap, b->r.n_quads, sizeof(ps4_quad));
            continue;
        }
        if (rc == PS4_ERR_VERIFY) {
            char line[512];
            snprintf(line, sizeof line, "%s\n", ps4_last_error(ctx));
            write_out(line, strlen(line));
            fatal_exit("FATAL: quadruple verification failed; this interval is NOT certified complete");
        }
        if (rc >= PS4_ERR_CAP_REPS && rc <= PS4_ERR_CAP_EXT) fatal_exit(ps4_last_error(ctx));
        if (rc != PS4_OK) {
            fprintf(stderr, "s4gpu: %s\n", ps4_last_error(ctx));
            exit(1);
        }
        /* counters */
        uint64_t *dst = &rg->s.S_done;
        const uint64_t *src = &add.S_done;
        for (int i = 0; i < 10; i++) dst[i] += src[i];
        for (int i = 0; i < 100; i++) { rg->s.hist5[i] += add.hist5[i]; rg->hist_run[i] += add.hist5[i]; }
        if (add.max_reps > rg->s.max_reps) rg->s.max_reps = add.max_reps;
        if (add.max_divisors > rg->s.max_divisors) rg->s.max_divisors = add.max_divisors;
        if (add.max_extensions > rg->s.max_extensions) rg->s.max_extensions = add.max_extensions;
        break;
    }
    /* lines: 4-set dumps and hits merged in the reference's processing order */
    b->text_len = 0;
    qkey *qs = NULL;
    uint64_t nq = 0;
    if (opt_dump4 && rg->dumped < opt_dump4 && b->r.n_quads) {
        qs = malloc(b->r.n_quads * sizeof *qs);
        for (uint64_t i = 0; i < b->r.n_quads; i++) {
            u64 v[4];
            ps4_quad_values(&b->r.quads[i], &qs[i].S, v, qs[i].order);
            qs[i].idx = i;
        }
        qsort(qs, b->r.n_quads, sizeof *qs, cmp_qkey);
        nq = b->r.n_quads;
        if ((long)nq > opt_dump4 - rg->dumped) nq = (uint64_t)(opt_dump4 - rg->dumped);
        rg->dumped += (long)nq;
    }
    char line[8192];
    uint64_t qi = 0;
    for (uint64_t h = 0; h <= b->r.n_hits; h++) {
        const ps4_hit *hit = h < b->r.n_hits ? &b->r.hits[h] : NULL;
        while (qi < nq && (!hit || cmp_key(qs[qi].S, qs[qi].order, hit->S, hit->order) <= 0)) {
            long n = ps4_format_quad(&b->r.quads[qs[qi].idx], line, sizeof line);
            if (n > 0) text_append(b, line, (size_t)n);
            qi++;
        }
        if (!hit) break;
        long n = ps4_format_hit(hit, b->r.exts, line, sizeof line);
        if (hit->n_ext >= 2) {                            /* the M line comes first */
            const char *nl = memchr(line, '\n', (size_t)(n > 0 ? n : 0));
            size_t mlen = nl ? (size_t)(nl - line) + 1 : 0;
            text_append(b, line, mlen);
            if (opt_test6 && !test6_fired) {
                test6_fired = 1;
                char dl[2048];
                if (ps4_format_drill(hit, b->r.exts, dl, sizeof dl) > 0) durable_alert(dl);
            }
            if (n > 0 && (size_t)n > mlen) text_append(b, line + mlen, (size_t)n - mlen);
        } else if (n > 0) {
            text_append(b, line, (size_t)n);
        }
        for (uint64_t s = 0; s < b->r.n_sixes; s++)
            if (b->r.sixes[s].hit == h && ps4_format_six(hit, b->r.exts, &b->r.sixes[s], line, sizeof line) > 0)
                durable_alert(line);
    }
    free(qs);
    write_out(b->text, b->text_len);
}

static volatile sig_atomic_t stop_signal = 0;
static void on_stop_signal(int sig) { stop_signal = sig; }

static unsigned env_cap(const char *name, unsigned dflt) {
    const char *s = getenv(name);
    return s && *s ? (unsigned)strtoul(s, NULL, 10) : dflt;
}

int main(int argc, char **argv) {
    int pos = 0;
    for (int i = 1; i < argc; i++) {                  /* s4.c:416-426 */
        if (!strcmp(argv[i], "--noext")) opt_noext = 1;
        else if (!strcmp(argv[i], "--verify")) opt_verify = 1;
        else if (!strcmp(argv[i], "--resume")) opt_resume = 1;
        else if (!strcmp(argv[i], "--test-sixset")) opt_test6 = 1;
        else if (!strcmp(argv[i], "--dump4") && i + 1 < argc) opt_dump4 = atol(argv[++i]);
        else if (!strcmp(argv[i], "--out") && i + 1 < argc) opt_out = argv[++i];
        else if (!strcmp(argv[i], "--ckpt") && i + 1 < argc) opt_ckpt = argv[++i];
        else {
            pos++;
            if (pos == 1) S_lo = strtoull(argv[i], 0, 10);
            else if (pos == 2) S_hi = strtoull(argv[i], 0, 10);
            else if (pos == 3) nthreads = atoi(argv[i]);
            else if (pos == 4) W = 1ull << atoi(argv[i]);
        }
    }
    if (S_lo < 1) S_lo = 1;
    if (nthreads <= 0) {
        long n = sysconf(_SC_NPROCESSORS_ONLN);
        nthreads = n > 0 ? (int)n : 1;
        if (opt_ckpt && opt_resume) { int c = ckpt_thread_count(); if (c > 0) nthreads = c; }
    }
    if (opt_ckpt && !opt_resume && access(opt_ckpt, F_OK) == 0) {
        fprintf(stderr, "checkpoint %s exists: add --resume to continue it, or delete it to start over\n", opt_ckpt);
        return 1;
    }
    if (opt_out) {
        out_fp = fopen(opt_out, "a");
        if (!out_fp) { perror(opt_out); return 1; }
    } else out_fp = stdout;
    cap_reps = env_cap("S4_MAX_REPS", 512);
    cap_divs = env_cap("S4_MAX_DIVS", 16384);
    cap_ext = env_cap("S4_MAX_EXT", 64);

    region_t *rg = calloc((size_t)nthreads, sizeof *rg);
    u64 total = S_hi > S_lo ? S_hi - S_lo : 0;
    for (int t = 0; t < nthreads; t++) {              /* s4.c:452-456 */
        rg[t].region_lo = S_lo + (u64)((unsigned __int128)total * t / nthreads);
        rg[t].region_hi = S_lo + (u64)((unsigned __int128)total * (t + 1) / nthreads);
    }
    int rs = (opt_ckpt && opt_resume) ? read_ckpt(rg) : 0;
    if (rs == 2) {
        fprintf(stderr, "checkpoint %s marks S in [%llu, %llu) as complete; nothing to do\n", opt_ckpt,
                (unsigned long long)S_lo, (unsigned long long)S_hi);
        return 0;
    }
    struct sigaction sa;
    memset(&sa, 0, sizeof sa);
    sa.sa_handler = on_stop_signal;
    sigemptyset(&sa.sa_mask);
    sa.sa_flags = SA_RESTART;
    sigaction(SIGTERM, &sa, NULL);
    sigaction(SIGINT, &sa, NULL);
    ps4_config cfg;
    memset(&cfg, 0, sizeof cfg);
    cfg.device = 0;
    cfg.s_hi_max = S_hi > 2 ? S_hi : 2;
    cfg.cap_reps = cap_reps; cfg.cap_divs = cap_divs; cfg.cap_ext = cap_ext;
    cfg.flags = (opt_noext ? PS4_F_NOEXT : 0) | (opt_verify ? PS4_F_VERIFY : 0) | (opt_dump4 ? PS4_F_DUMP4 : 0);
    const char *kern = getenv("PS4_KERNEL");
    cfg.kernel = (kern && !strcmp(kern, "plain")) ? PS4_KERNEL_PLAIN : PS4_KERNEL_BATCHED;
    ps4_ctx *ctx = NULL;
    if (ps4_create(&cfg, &ctx) != PS4_OK) {
        fprintf(stderr, "s4gpu: %s\n", ctx ? ps4_last_error(ctx) : "cannot create context");
        return 1;
    }
    fprintf(stderr, "s4: S in [%llu, %llu), %d threads, chunk %llu, ext=%s%s%s\n", (unsigned long long)S_lo,
            (unsigned long long)S_hi, nthreads, (unsigned long long)W, opt_noext ? "off" : "on",
            opt_ckpt ? ", checkpointing" : "", rs == 1 ? ", RESUMED from checkpoint" : "");
    u64 total_chunks = 0, done_chunks = 0;
    for (int t = 0; t < nthreads; t++) {
        total_chunks += (rg[t].region_hi - rg[t].region_lo + W - 1) / W;
        if (rs == 1)
            fprintf(stderr, "  thread %2d resumes at S=%llu (region end %llu)\n", t, (unsigned long long)rg[t].region_lo,
                    (unsigned long long)rg[t].region_hi);
        rg[t].next_S0 = rg[t].region_lo;
    }
    batch_out bo;
    memset(&bo, 0, sizeof bo);
    if (opt_dump4) ensure((void **)&bo.r.quads, &bo.r.quads_cap, 1u << 16, sizeof(ps4_quad));
    double t0 = now_sec(), last_ckpt = -1e9;
    int last_report = 0;
    u64 chunks_per_batch = 1;
    for (int t = 0; t < nthreads && !stop_signal; t++) {
        double rt0 = now_sec();
        for (u64 S0 = rg[t].region_lo; S0 < rg[t].region_hi && !stop_signal;) {
            u64 span = chunks_per_batch * W;
            u64 S1 = rg[t].region_hi - S0 > span ? S0 + span : rg[t].region_hi;
            double b0 = now_sec();
            run_batch(ctx, &rg[t], S0, S1, &bo);
            double bt = now_sec() - b0;
            done_chunks += (S1 - S0 + W - 1) / W;
            rg[t].next_S0 = S1;
            S0 = S1;
            if (bt < 0.25 && chunks_per_batch < (1ull << 20)) chunks_per_batch *= 2;
            else if (bt > 2.0 && chunks_per_batch > 1) chunks_per_batch /= 2;
            double el = now_sec() - t0;
            if (el - last_ckpt >= 5.0) { last_ckpt = el; write_ckpt(rg, 0); }
            int slot = (int)el / 30;
            if (slot != last_report && slot > 0) {
                last_report = slot;
                u64 s4 = 0, s5 = 0, s6 = 0;
                for (int k = 0; k < nthreads; k++) { s4 += rg[k].s.sets4; s5 += rg[k].s.sets5; s6 += rg[k].s.sets6; }
                fprintf(stderr, "[%.0fs] chunks %llu/%llu  4-sets %llu  5-sets %llu  6-sets %llu\n", el,
                        (unsigned long long)done_chunks, (unsigned long long)total_chunks, (unsigned long long)s4,
                        (unsigned long long)s5, (unsigned long long)s6);
                fflush(stderr);
            }
        }
        rg[t].secs = now_sec() - rt0;
    }
    if (stop_signal) {
        const int sig = stop_signal;
        write_ckpt(rg, 0);
        fprintf(stderr, "s4gpu: stopped by signal %d at a batch boundary%s\n", sig,
                opt_ckpt ? "; the checkpoint holds the positions reached" : "");
        fflush(stderr);
        ps4_destroy(ctx);
        if (out_fp != stdout) fclose(out_fp); else fflush(stdout);
        signal(sig, SIG_DFL);
        raise(sig);
        return 128 + sig;
    }
    double el = now_sec() - t0;
    write_ckpt(rg, 1);
    ps4_stats tot;
    memset(&tot, 0, sizeof tot);
    u64 hist_run[100] = {0};
    for (int t = 0; t < nthreads; t++) {              /* s4.c:489-497 */
        uint64_t *dst = &tot.S_done;
        const uint64_t *src = &rg[t].s.S_done;
        for (int i = 0; i < 10; i++) dst[i] += src[i];
        if (rg[t].s.max_reps > tot.max_reps) tot.max_reps = rg[t].s.max_reps;
        if (rg[t].s.max_divisors > tot.max_divisors) tot.max_divisors = rg[t].s.max_divisors;
        if (rg[t].s.max_extensions > tot.max_extensions) tot.max_extensions = rg[t].s.max_extensions;
        for (int i = 0; i < 100; i++) hist_run[i] += rg[t].hist_run[i];
        fprintf(stderr, "  thread %2d: S [%llu,%llu) 4-sets %llu 5-sets %llu  %.1fs\n", t,
                (unsigned long long)rg[t].region_lo, (unsigned long long)rg[t].region_hi,
                (unsigned long long)rg[t].s.sets4, (unsigned long long)rg[t].s.sets5, rg[t].secs);
    }
    fprintf(stderr,
            "TOTAL: S_done=%llu pairs=%llu S_ge3=%llu triples=%llu 4-sets=%llu 5-sets=%llu 6-sets=%llu "
            "multi-ext-4sets=%llu ext_cand=%llu ext_sqrt=%llu  wall=%.1fs%s\n",
            (unsigned long long)tot.S_done, (unsigned long long)tot.pairs, (unsigned long long)tot.S_ge3,
            (unsigned long long)tot.triples, (unsigned long long)tot.sets4, (unsigned long long)tot.sets5,
            (unsigned long long)tot.sets6, (unsigned long long)tot.multi, (unsigned long long)tot.ext_cand,
            (unsigned long long)tot.ext_sqrt, el,
            rs == 1 ? " (counters cumulative over resumed runs; wall time of this run only)" : "");
    fprintf(stderr, "5-sets by log2(largest element)%s:", rs == 1 ? " (this run only)" : "");
    for (int i = 0; i < 100; i++)
        if (hist_run[i]) fprintf(stderr, " %d:%llu", i, (unsigned long long)hist_run[i]);
    fprintf(stderr, "\n");
    fprintf(stderr, "CAPACITY: reps=%llu/%u divisors=%llu/%u extensions=%llu/%u%s\n", (unsigned long long)tot.max_reps,
            cap_reps, (unsigned long long)tot.max_divisors, cap_divs, (unsigned long long)tot.max_extensions, cap_ext,
            rs == 1 ? " (maxima this resumed invocation only)" : "");
    ps4_destroy(ctx);
    if (out_fp != stdout) fclose(out_fp);
    return 0;
}
