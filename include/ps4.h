/*
 * ps4.h -- C-ABI of libps4.so, the B200 (sm_100a) search for sets of positive integers
 * whose pairwise sums are all perfect squares.
 *
 * The reference exposes this path as a process (exhaustive/s4.c), not a library: its
 * in-process seam is process_chunk(S0,S1,&work,&stats) (exhaustive/s4.c:280) feeding
 * handle_4set (exhaustive/s4.c:225).  Each entry point below names the reference code it
 * replaces.  Plain pointers and sizes only; every function returns 0 or a PS4_ERR_* code,
 * with the message in ps4_last_error().  One host thread per context.
 *
 * Output records are raw (numbers, not text); ps4_format_* turn them into the reference's
 * exact result lines (exhaustive/s4.c:24-27,110-137,209-220,237-277).
 */
#ifndef PS4_H
#define PS4_H
#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define PS4_ABI_VERSION 1

/* ---- status codes ---- */
enum {
    PS4_OK = 0,
    PS4_ERR_ARG = 1,          /* bad argument (message says which)                                  */
    PS4_ERR_CUDA = 3,         /* CUDA runtime failure, or no usable sm_100 device                   */
    PS4_ERR_CAP_REPS = 10,    /* "representation capacity exceeded"  (s4.c:321)                    */
    PS4_ERR_CAP_DIVS = 11,    /* "divisor capacity exceeded"         (s4.c:176)                    */
    PS4_ERR_CAP_EXT = 12,     /* "extension capacity exceeded"       (s4.c:201)                    */
    PS4_ERR_VERIFY = 13,      /* "quadruple verification failed"     (s4.c:232, --verify only)     */
    PS4_ERR_CAP_INTERNAL = 14,/* ps4_search_range_noalloc only: a tile's fixed shared-memory list
                                 overflowed (message names it); the interval is not certified       */
    PS4_ERR_OUTPUT_FULL = 20, /* a caller buffer in ps4_results is too small; n_* hold the needed sizes */
    PS4_ERR_TIMEOUT = 21      /* a device-side bounded wait gave up (persistent kernels, serving)   */
};

/* ---- flags (ps4_config.flags) ---- */
enum {
    PS4_F_NOEXT = 1,   /* count 4-sets only, no extension step            (s4 --noext, s4.c:242)  */
    PS4_F_VERIFY = 2,  /* re-check the six roots of every 4-set on device (s4 --verify, s4.c:229) */
    PS4_F_DUMP4 = 4    /* return every 4-set as a ps4_quad record         (s4 --dump4, s4.c:237)  */
};

/* ---- kernel choice (ps4_config.kernel) ---- */
enum {
    PS4_KERNEL_BATCHED = 0, /* per batch of S: persistent tile kernel queues every 4-set, then the
                               extension engine pools their divisor pairs warp-wide (default)        */
    PS4_KERNEL_PLAIN = 1,   /* one CTA per tile, one thread per S, inline extension (baseline)       */
    PS4_KERNEL_FUSED = 2,   /* one persistent kernel: tiles, staging and per-lane extension fused    */
    PS4_KERNEL_PERSIST = 3  /* one launch per call over every subrange: CTAs switch between writing
                               tiles' 4-sets into a device ring and running the extension engine on
                               the ring; falls back to PS4_KERNEL_BATCHED when one of its bounded
                               waits gives up                                                          */
};

typedef struct ps4_ctx ps4_ctx;

typedef struct {
    int device;            /* CUDA device ordinal                                                   */
    uint64_t s_hi_max;     /* largest S_hi to be searched; sizes the factor tables (<= 2^44)         */
    uint32_t cap_reps;     /* representation cap per S        (S4_MAX_REPS, default 512,   s4.c:46)  */
    uint32_t cap_divs;     /* divisor cap per difference      (S4_MAX_DIVS, default 16384, s4.c:52)  */
    uint32_t cap_ext;      /* extension cap per 4-set         (S4_MAX_EXT,  default 64,    s4.c:49)  */
    uint32_t flags;        /* PS4_F_*                                                               */
    uint32_t kernel;       /* PS4_KERNEL_*                                                          */
    uint32_t log2_tile;    /* S values per tile = 2^log2_tile (12..14); 0 = autotuned/default        */
    uint32_t ctas_per_sm;  /* resident CTAs per SM for the persistent kernel; 0 = default            */
    void *stream;          /* cudaStream_t to launch on; NULL = a stream owned by the context        */
    uint32_t use_graph;    /* PS4_GRAPH_*: run a call's launch sequence as one captured CUDA graph   */
    uint32_t time_kernels; /* 1: time every launch with events (ps4_last_kernel_split); no graphs     */
} ps4_config;

enum {
    PS4_GRAPH_AUTO = 0,    /* graph for batched calls of two or more batches (default)               */
    PS4_GRAPH_ALWAYS = 1,
    PS4_GRAPH_NEVER = 2
};

/* Counters, identical in meaning to the reference's stats_t (exhaustive/s4.c:80-91). */
typedef struct {
    uint64_t S_done, pairs, S_ge3, triples, sets4, sets5, sets6, multi, ext_cand, ext_sqrt;
    uint64_t hist5[100];
    uint64_t max_reps, max_divisors, max_extensions;
} ps4_stats;

/* A 4-set with at least one extension (what handle_4set prints about, s4.c:243-277). */
typedef struct {
    uint64_t S;
    uint64_t v[4];        /* a,b,c,d in the reference's formula order (s4.c:333)                      */
    uint32_t n_ext;       /* extensions, stored at exts[first_ext .. first_ext+n_ext) in the         */
    uint32_t first_ext;   /*   reference's divisor order (s4.c:185-204)                              */
    uint32_t flags;       /* PS4_HIT_*                                                               */
    uint32_t item;        /* index of the query (subrange or triple) this hit belongs to              */
    uint32_t order[4];    /* sort key reproducing the reference's emission order: px, py, pz, class   */
} ps4_hit;

enum { PS4_HIT_MULTI = 1,        /* >= 2 extensions: an "M:" line                    */
       PS4_HIT_DRILL_OK = 2 };   /* {v, ext0, ext1} passes verify_set (drill line)   */

typedef struct {
    uint64_t lo, hi;      /* the extension e = hi*2^64 + lo                                          */
    uint32_t key;         /* divisor index of the pair that produced e (reference order)             */
    uint32_t flags;       /* PS4_EXT_*                                                               */
} ps4_ext;

enum { PS4_EXT_FIVE = 1,         /* e > max(v): a "5:" line                         */
       PS4_EXT_FIVE_OK = 2 };    /* that 5-set passes verify_set                    */

typedef struct {            /* a 6-set {v, ext t, ext s} (s4.c:270-276)                      */
    uint32_t hit, t, s, flags;   /* flags bit 0: passes verify_set                            */
} ps4_six;

typedef struct {            /* one 4-set for --dump4: the six pair roots, formula order         */
    uint32_t r_ab, r_ac, r_ad, r_bc, r_bd, r_cd;
} ps4_quad;

/* Caller-owned host output buffers.  On return n_* hold the record counts; if any
 * count exceeds its *_cap the call returns PS4_ERR_OUTPUT_FULL, nothing is written
 * past the caps, and the call can be repeated with larger buffers. */
typedef struct {
    ps4_hit *hits;   uint64_t hits_cap;   uint64_t n_hits;
    ps4_ext *exts;   uint64_t exts_cap;   uint64_t n_exts;
    ps4_six *sixes;  uint64_t sixes_cap;  uint64_t n_sixes;
    ps4_quad *quads; uint64_t quads_cap;  uint64_t n_quads;
} ps4_results;

/* ---- lifetime ---- */

/* Build the factor / divisor-count tables for S < cfg->s_hi_max on the device and
 * allocate the working buffers.  (Replaces the table set-up of s4.c:436-447.) */
int ps4_create(const ps4_config *cfg, ps4_ctx **out);
void ps4_destroy(ps4_ctx *ctx);
const char *ps4_last_error(const ps4_ctx *ctx);
int ps4_abi_version(void);

/* ---- the search ----
 *
 * Every S in [lo, hi): enumerate all 4-sets with sum S, extend each by divisor pairs,
 * report every 4-set with >= 1 extension, and add the reference's counters into *stats
 * (+=).  Replaces the worker loop over process_chunk (exhaustive/s4.c:344-364 calling
 * :280-341, :225-278, :160-207).  Results are independent of how [lo,hi) is split into
 * calls.  Host buffers; the call returns when results are in them. */
int ps4_search_range(ps4_ctx *ctx, uint64_t lo, uint64_t hi, ps4_stats *stats, ps4_results *res);

/* Many independent subranges [lo[i], hi[i]) in ONE persistent launch (the block controller's
 * sequence of s4 invocations, run_exhaustive.py:200-238, done as one device batch).  stats
 * points at n_items ps4_stats (+=); every hit carries its item index.  Subranges may overlap;
 * each is searched in full. */
int ps4_search_batch(ps4_ctx *ctx, const uint64_t *lo, const uint64_t *hi, uint32_t n_items,
                     ps4_stats *stats, ps4_results *res);

/* The same search split in two: enqueue on the context's stream and return at once (no
 * result copies), then wait, check and collect.  Lets a caller overlap host work with the
 * device search, or time the device work alone with events on the stream.  At most one
 * search may be enqueued per context.  (Same reference code as ps4_search_range.) */
int ps4_search_enqueue(ps4_ctx *ctx, uint64_t lo, uint64_t hi);
int ps4_search_finish(ps4_ctx *ctx, ps4_stats *stats, ps4_results *res);

/* Bytes copied host->device and device->host by the last search call (inputs and results). */
void ps4_last_transfer_bytes(const ps4_ctx *ctx, uint64_t *h2d, uint64_t *d2h);

/* ps4_search_range without any device allocation.  No counterpart in the reference (its
 * CPU engine allocates on the host freely); this serves callers that cannot call cudaMalloc
 * at search time -- code that owns a fixed device-memory budget or its own pool and must not
 * grow it, or a serving loop that cannot afford cudaMalloc/cudaFree, which block the host
 * and (cudaFree) synchronise the device.
 *
 * Same inputs and outputs as ps4_search_range: S in [lo, hi) and the context's factor
 * tables (built by ps4_create, read only here) in, counters (+=) and host result records
 * out, with the records in device order (not sorted).  The only other device memory it
 * uses is one static array in the library of 65.5 MB (62.5 MiB) -- 4-set staging for 148
 * CTAs plus fixed result buffers of 65536 hits, 131072 extensions and 256 6-sets -- which
 * every GPU that loads the library holds until the process exits.  It rejects, with
 * PS4_ERR_ARG and a message, contexts made with PS4_F_DUMP4 or cap_reps > 512, ranges past
 * the context's s_hi_max and ranges of 2^43 S or more.  The first call on each device
 * looks up the array's device address (cudaGetSymbolAddress), so make that first call before
 * any stream capture; the address is kept per device and looked up again when the device's
 * primary context has changed (after cudaDeviceReset) or a call failed.  Every call on a device
 * shares the array and overwrites it: calls whose work overlaps on the GPU (other threads,
 * other streams) race and must be serialised by the caller.  Synchronous on the context's
 * stream.
 *
 * Errors besides the regular search's: more records than the fixed buffers hold give
 * PS4_ERR_OUTPUT_FULL with n_* set to the counts the search produced (at least one above its
 * PS4_NOALLOC_MAX_* limit; nothing is copied; search a shorter range).  A tile whose lists
 * outgrow their fixed shared-memory sizes gives PS4_ERR_CAP_INTERNAL: a capacity failure that a
 * shorter range does not avoid, reported like the reference's FATAL lines (interval not
 * certified complete). */
#define PS4_NOALLOC_MAX_HITS 65536u
#define PS4_NOALLOC_MAX_EXTS 131072u
#define PS4_NOALLOC_MAX_SIXES 256u
int ps4_search_range_noalloc(ps4_ctx *ctx, uint64_t lo, uint64_t hi, ps4_stats *stats, ps4_results *res);

/* ---- one range on several devices ----
 *
 * Cut [lo, hi) into n contiguous shards of about equal search cost, for n devices (one
 * process or context each) searching one range.  Every result line and counter of the search
 * is a function of S alone (exhaustive/s4.c:313-341), so the shards' result lines concatenate
 * in shard order into the whole range's canonical order, and their counters add (the three
 * CAPACITY maxima take the maximum).  Replaces the reference's equal-width split of [S_lo,
 * S_hi) into thread regions (exhaustive/s4.c:452-456): the search's cost per S grows with S,
 * so equal widths leave the top shard the slowest.  The cost model is a density proportional
 * to S^0.16, fitted to this library's measured rates (5.5e-11 s per S averaged over [1,1e10),
 * 1.2e-10 s per S near 5e11); shard i is [bounds[i], bounds[i+1]) with bounds[0] = max(lo, 1),
 * bounds[n] = hi, and inner bounds on multiples of 2^14 S (one tile).  Host only (no device).
 * bounds holds n + 1 values; n >= 1. */
int ps4_plan_shards(uint64_t lo, uint64_t hi, uint32_t n, uint64_t *bounds);

/* ---- exact-root self-check ----
 *
 * Runs the device's exact integer square roots -- the routines every square test and tile
 * scan of the search uses, restating isqrt64 / isqrt128 / is_sq128 (exhaustive/s4.c:95-108) --
 * on n[i] = hi[i]*2^64 + lo[i], so that they can be checked against exact host arithmetic
 * at their edges.  roots[4i..4i+3] = floor(sqrt(n)) (128-bit), floor(sqrt(lo)), ceil(sqrt(lo)),
 * and floor(sqrt(lo)) by the tile scan's single-precision estimate (lo < 2^46, else 0);
 * flags[i] bit 0: n is a square (exact test), bit 1: n is a square by the search's fast test,
 * evaluated only for n < 2^100, its precondition (else 0).  Allocates and frees its own device
 * buffers on `device`; synchronous. */
int ps4_check_roots(int device, const uint64_t *lo, const uint64_t *hi, uint32_t n, uint64_t *roots,
                    uint32_t *flags);

/* Self-check of the bounded waits of PS4_KERNEL_PERSIST: one device thread waits, as a consuming
 * warp does, for a ring position that nothing publishes.  The wait gives up after its time limit
 * (2 s) and records the timeout instead of spinning on; the call returns PS4_ERR_TIMEOUT when that
 * happened as designed (PS4_OK would mean the wait ended otherwise) and *waited_ns the time it
 * waited.  No counterpart in the reference (its threads never wait on one another).  Allocates
 * and frees its own small device buffers on `device`; synchronous. */
int ps4_check_ring_wait(int device, uint64_t *waited_ns);

/* ---- triple extension ----
 *
 * For each triple {a, b, c} of distinct positive integers whose three pairwise sums are
 * squares, every d with 0 < d <= dmax, d not in the triple, and d+a, d+b, d+c all squares.
 * The reference runs this step only inside its search, on 4-sets: extend4 (exhaustive/s4.c:
 * 160-207) with the same divisor-pair construction -- e + A = u^2, e + B = w^2 gives
 * (u - w)(u + w) = A - B, enumerated through the factorisation of A - B = r_AC^2 - r_BC^2
 * -- and its pair choice by estimated divisor count (s4.c:163-171). */
typedef struct {
    uint64_t d;           /* the extension                                                        */
    uint32_t item;        /* index of the triple in the call's input                              */
    uint32_t reserved;    /* 0                                                                    */
} ps4_tri_ext;

typedef struct {
    uint64_t triples;     /* triples searched (valid ones)                                        */
    uint64_t invalid;     /* inputs that are not a square-sum triple of distinct positive integers */
    uint64_t ext_cand;    /* same-parity complementary divisor pairs f < g enumerated (ext_cand)  */
    uint64_t ext_sqrt;    /* exact square tests of d + C after the residue filters                */
    uint64_t exts;        /* extensions found                                                     */
} ps4_tri_stats;

/* abc holds 3*n members (triple i = abc[3i..3i+2], any order); state (n bytes, may be NULL)
 * receives 0 for a searched triple and 1 for an input that is not a square-sum triple of
 * distinct positive integers (no records; the oracle returns -1 for those).  Members must
 * stay below 2^44 and their pairwise-sum roots inside the context's factor tables (largest
 * member <= s_hi_max / 2 is always enough), dmax <= 2^62; otherwise PS4_ERR_ARG.  Records
 * are sorted by (item, d); stats (+=, may be NULL).  More records than out_cap give
 * PS4_ERR_OUTPUT_FULL with *n_out the needed count.  Synchronous on the context's stream. */
int ps4_extend_triples(ps4_ctx *ctx, const uint64_t *abc, uint32_t n, uint64_t dmax, uint8_t *state,
                       ps4_tri_ext *out, uint64_t out_cap, uint64_t *n_out, ps4_tri_stats *stats);

/* ---- serving: continuous batching of subrange and triple queries ----
 *
 * The reference serves its search as one s4 process per block from a Python controller
 * (run_exhaustive.py:200-238, one subprocess per block, results parsed from stdout) and has
 * no triple query.  A server replaces that loop in-process: queries are submitted as they
 * arrive, admitted while a device slot and room in a fixed device-memory budget are free, and
 * run in steps -- each step one launch of the search kernels over chunks of every admitted
 * subrange (shortest remaining first, the oldest always included) plus one triple-extension
 * launch over every admitted triple query -- so queries that arrive while others run join
 * the next step and share its kernels.  Counters and result records of each query accumulate
 * on the device in its slot; a finished query's results are copied to the host once.  Each
 * query's results are the ones ps4_search_range / ps4_extend_triples give for it alone.
 * One host thread per server; the context's tables are shared read-only. */
typedef struct ps4_server ps4_server;

typedef struct {
    uint64_t hbm_budget;        /* device bytes for the server: step buffers + per-query arena (0 = 8 GiB) */
    uint32_t max_slots;         /* queries resident on the device at once (0 = 1024)                      */
    uint32_t max_step_items;    /* subrange chunks per step (0 = 4096)                                    */
    uint64_t step_S;            /* S values per step over all chunks (0 = 2^27)                           */
    uint32_t max_step_triples;  /* triple queries per step (0 = 65536)                                    */
    uint32_t hits_floor;        /* result-buffer quota of a subrange query: hits_floor + hits_per_1e6_S    */
    uint32_t hits_per_1e6_S;    /*   hits per million S, extensions twice that (0, 0 = 256, 40); a query   */
    uint32_t reserved;          /*   that outgrows its quota is re-admitted with larger buffers and re-run */
} ps4_serve_config;

enum { PS4_Q_RANGE = 0, PS4_Q_TRIPLE = 1 };

typedef struct {              /* one finished query, reported by ps4_serve_progress                     */
    uint64_t tag;             /* the caller's tag given at submit                                       */
    int32_t status;           /* PS4_OK or the error the same query alone would give                    */
    uint32_t kind;            /* PS4_Q_*                                                                */
    uint64_t n_records;       /* hits (subrange) or extensions (triple)                                 */
    double t_submit, t_admit, t_done;   /* host monotonic clock (CLOCK_MONOTONIC), seconds              */
    uint32_t steps;           /* steps that carried work of this query                                  */
    uint32_t reruns;          /* re-runs after its device result buffers overflowed                     */
    char message[160];        /* error text when status != PS4_OK                                       */
} ps4_serve_done;

typedef struct {
    uint64_t submitted, waiting, active, finished, steps, step_reruns;
    uint64_t arena_bytes, arena_used, arena_peak;   /* per-query state and result buffers           */
    uint64_t device_bytes;                          /* everything the server holds on the device     */
    double gpu_ms;                                  /* summed device time of the steps' kernels      */
} ps4_serve_info;

/* Create a server on a context (made without PS4_F_DUMP4).  Allocates its whole budget. */
int ps4_serve_create(ps4_ctx *ctx, const ps4_serve_config *cfg, ps4_server **out);
void ps4_serve_destroy(ps4_server *srv);
const char *ps4_serve_last_error(const ps4_server *srv);
/* Queue a query; returns at once.  Tags must be unique among queries not yet taken. */
int ps4_serve_submit_range(ps4_server *srv, uint64_t tag, uint64_t lo, uint64_t hi);
int ps4_serve_submit_triple(ps4_server *srv, uint64_t tag, const uint64_t abc[3], uint64_t dmax);
/* Drive the server: collect finished steps, admit waiting queries, launch the next steps.
 * Waits up to wait_us for a query to finish; reports up to cap finished queries. */
int ps4_serve_progress(ps4_server *srv, uint32_t wait_us, ps4_serve_done *done, uint32_t cap, uint32_t *n_done);
/* Results of a finished query, in the layout and order of the single-query calls; the query
 * is forgotten afterwards (PS4_ERR_OUTPUT_FULL keeps it, with the needed counts set). */
int ps4_serve_take_range(ps4_server *srv, uint64_t tag, ps4_stats *stats, ps4_results *res);
int ps4_serve_take_triple(ps4_server *srv, uint64_t tag, uint8_t *state, ps4_tri_ext *out, uint64_t out_cap,
                          uint64_t *n_out, ps4_tri_stats *stats);
void ps4_serve_get_info(const ps4_server *srv, ps4_serve_info *info);

/* ---- autotuning of the batched search ----
 *
 * Launch shape of the two-kernel pipeline: S per tile, resident tile-kernel CTAs per SM,
 * resident engine CTAs per SM, and the largest job queue (entries, a power of two; one batch
 * of the search fills at most 90 % of it).  No counterpart in the reference (its engine has
 * fixed compile-time sizes, s4.c:46-52). */
typedef struct {
    uint32_t log2_tile;       /* 12 .. 14                                                            */
    uint32_t gen_ctas;        /* 1 .. 2: tile-kernel threads per SM in units of 512 (512-thread CTAs  */
                              /* on 2^14-S tiles, 256-thread ones on smaller tiles)                 */
    uint32_t ext_ctas;        /* 1 .. 3                                                              */
    uint32_t log2_jobs;       /* 20 .. 29                                                            */
    double rate;              /* S/s the tuner measured for this shape (0 if set by hand)            */
} ps4_tuning;

/* Time candidate shapes on a sample of the given workload (a slice of each of up to 8 items
 * spread over its S span, about 2e8 S in all) and keep the fastest on the context; *best
 * (may be NULL) receives it.  Runs for roughly budget_s seconds (0 = 2).  Results of later
 * calls do not depend on the shape. */
int ps4_autotune(ps4_ctx *ctx, const uint64_t *lo, const uint64_t *hi, uint32_t n_items, double budget_s,
                 ps4_tuning *best);
int ps4_set_tuning(ps4_ctx *ctx, const ps4_tuning *t);
void ps4_get_tuning(const ps4_ctx *ctx, ps4_tuning *t);
/* CUDA-graph use of the context so far: graphs captured, graph replays. */
void ps4_graph_counts(const ps4_ctx *ctx, uint64_t *captures, uint64_t *replays);

/* Device time (ms, CUDA events on the launch stream) of the kernels of the last search call. */
double ps4_last_kernel_ms(const ps4_ctx *ctx);
/* Device time (ms) of the last search call split by kernel: the tile kernel (4-set generation)
 * and the extension engine, summed over the call's batches.  Needs time_kernels = 1. */
void ps4_last_kernel_split(const ps4_ctx *ctx, double *gen_ms, double *ext_ms);
/* Number of kernel launches made by the last search call. */
uint64_t ps4_last_launches(const ps4_ctx *ctx);

/* ---- text output, byte-identical to the reference ----
 *
 * Write the buffered result lines of `hit` -- the "M:" line, then the "5:" lines in
 * extension order -- into buf, NUL-terminated (s4.c:247-269, format_set s4.c:214-220).
 * Returns the length, or -1 if cap is too small.  `exts` is the results' ext array. */
long ps4_format_hit(const ps4_hit *hit, const ps4_ext *exts, char *buf, size_t cap);
/* ps4_format_hit's lines of hits[0..n) concatenated into buf (NUL-terminated), and the query
 * item of each line into line_items (may be NULL; at most n + the hits' extension count lines).
 * Returns the length, or -(length needed + 1) when cap is too small (then nothing past the
 * last complete hit is written and line_items stops there too); *n_lines gets the line count. */
long ps4_format_hits(const ps4_hit *hits, uint64_t n, const ps4_ext *exts, char *buf, size_t cap,
                     uint32_t *line_items, uint64_t *n_lines);
/* The "!!!!!!!! FOUND 6-SET:" alert line of a 6-set record (s4.c:270-276).  Returns length or -1. */
long ps4_format_six(const ps4_hit *hit, const ps4_ext *exts, const ps4_six *six, char *buf, size_t cap);
/* The --test-sixset drill line for an M hit (s4.c:255-260).  Returns length or -1. */
long ps4_format_drill(const ps4_hit *hit, const ps4_ext *exts, char *buf, size_t cap);
/* A "4:" dump line (s4.c:239).  Returns length or -1. */
long ps4_format_quad(const ps4_quad *q, char *buf, size_t cap);
/* S, v[4] and the reference's emission-order key of a dump record. */
void ps4_quad_values(const ps4_quad *q, uint64_t *S, uint64_t v[4], uint32_t order[4]);

#ifdef __cplusplus
}
#endif
#endif
