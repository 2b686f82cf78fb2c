// ps4_api.cu -- host side of the C-ABI (include/ps4.h): context, device tables, launches,
// automatic re-runs on internal capacity limits, and result collection.
//
// Replaces the driver part of exhaustive/s4.c: table set-up (s4.c:436-447), the per-thread
// chunk loop (s4.c:344-364) and the counter totals (s4.c:488-495).  One host thread per
// context; every search call is synchronous on the context's stream.

#include <cuda_runtime.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <ctime>
#include <string>
#include <vector>

#include "ps4_internal.h"

using namespace ps4;

struct PendingSearch {
    std::vector<Item> items;
    bool dump = false;
    bool active = false;
    uint64_t tiles = 0;
};

struct ps4_ctx {
    ps4_config cfg;
    cudaStream_t stream = nullptr;
    bool own_stream = false;
    int num_sms = 0;
    uint64_t tab_n = 0;
    uint64_t *d_spfq = nullptr;
    uint16_t *d_ndiv = nullptr;
    uint4 *d_fac3 = nullptr;
    // working buffers (grown on demand)
    Item *d_items = nullptr; uint32_t items_cap = 0;
    unsigned long long *d_counters = nullptr; uint32_t counters_items = 0;
    ps4_hit *d_hits = nullptr; uint32_t hits_cap = 0;
    ps4_ext *d_exts = nullptr; uint32_t exts_cap = 0;
    ps4_six *d_sixes = nullptr; uint32_t sixes_cap = 0;
    ps4_quad *d_quads = nullptr; uint64_t quads_cap = 0;
    uint32_t *d_scratch = nullptr; size_t scratch_words = 0;
    Status *d_status = nullptr;
    Status *h_status = nullptr;          // pinned
    cudaEvent_t ev0 = nullptr, ev1 = nullptr;
    double last_ms = 0.0;
    uint64_t last_launches = 0;
    unsigned tile_log2 = 13;             // current tile size (may shrink on E_TILE)
    PendingSearch pend;
    uint64_t *d_raw = nullptr;           // per tile-kernel CTA: SUPER_K tile lists of RAW_PER_TILE
    uint64_t raw_words = 0;
    uint32_t *d_jobs = nullptr;          // 4-set job queue of the two-kernel pipeline (jobs_cap 24-byte records)
    uint64_t jobs_cap = 1ull << 20;          // grows with the calls, up to jobs_cap_max
    uint64_t d_jobs_words = 0;
    uint32_t batch_div = 1;              // narrows the batches after a queue overflow
    bool fused_fallback = false;         // this call re-runs on the fused kernel (engine list overflow)
    bool persist_fallback = false;       // this call re-runs on the two-kernel pipeline (a persistent-kernel
                                         //   wait gave up, or a tile outgrew the 2^13-S tile lists)
    uint32_t *d_seq = nullptr;           // the persistent kernel's ring: slot states (ring_cap u32); its
    uint64_t seq_cap = 0;                //   4-sets use d_jobs with ring_cap entries
    uint64_t ring_cap = 1ull << 26;
    uint64_t h2d_bytes = 0, d2h_bytes = 0;
    // tuning (ps4_autotune / ps4_set_tuning)
    uint32_t gen_ctas = 2, ext_ctas = 3;     // per SM: tile-kernel threads in units of 512 / engine CTAs
    uint64_t jobs_cap_max = 1ull << 29;      // largest job queue (entries; 2^29 = 12.9 GB): fewer,
                                             //   longer batches, fewer launch tails
    double tuned_rate = 0.0;
    // pinned staging of the segments, and the kept CUDA graph of a multi-batch call
    Item *h_segs = nullptr; uint64_t h_segs_cap = 0;
    // pinned landing buffers of the result records (copied back at full speed, then ordered into the
    // caller's buffers)
    ps4_hit *h_hits = nullptr; uint64_t h_hits_cap = 0;
    ps4_ext *h_exts = nullptr; uint64_t h_exts_cap = 0;
    ps4_six *h_sixes = nullptr; uint64_t h_sixes_cap = 0;
    cudaGraphExec_t graph_exec = nullptr;
    std::string graph_key;
    uint64_t graph_launches = 0, graph_captures = 0, graph_replays = 0;
    // per-launch timing (cfg.time_kernels): event pairs around each tile / engine launch
    std::vector<cudaEvent_t> kev;
    size_t kev_used = 0;
    double gen_ms = 0.0, ext_ms = 0.0;
    // triple extension (grown on demand)
    uint64_t *d_tri_in = nullptr; uint64_t tri_in_cap = 0;
    uint8_t *d_tri_state = nullptr; uint64_t tri_state_cap = 0;
    ps4_tri_ext *d_tri_out = nullptr; uint64_t tri_out_cap = 0;
    unsigned long long *d_tri_cnt = nullptr; uint64_t tri_cnt_cap = 0;   // n_out, n_cand, n_sqrt
    std::string err;
};

static int set_err(ps4_ctx *c, int code, const char *fmt, ...) {
    char buf[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(buf, sizeof buf, fmt, ap);
    va_end(ap);
    if (c) c->err = buf;
    return code;
}

#define CUDA_TRY(ctx, call)                                                                          \
    do {                                                                                             \
        cudaError_t _e = (call);                                                                     \
        if (_e != cudaSuccess)                                                                       \
            return set_err(ctx, PS4_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(_e));      \
    } while (0)

template <class T>
static int grow(ps4_ctx *c, T *&ptr, uint64_t &cap, uint64_t need) {
    if (need <= cap && ptr) return 0;
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
    if (need == 0) return 0;
    CUDA_TRY(c, cudaMalloc((void **)&ptr, need * sizeof(T)));
    cap = need;
    return 0;
}
template <class T>
static int grow32(ps4_ctx *c, T *&ptr, uint32_t &cap, uint64_t need) {
    uint64_t cap64 = cap;
    int rc = grow(c, ptr, cap64, need);
    cap = (uint32_t)cap64;
    return rc;
}

// a pinned host buffer of at least `need` elements (grown by half again, kept between calls)
template <class T>
static int grow_pinned(ps4_ctx *c, T *&ptr, uint64_t &cap, uint64_t need) {
    if (need <= cap && ptr) return 0;
    if (ptr) cudaFreeHost(ptr);
    ptr = nullptr;
    cap = 0;
    const uint64_t n = std::max<uint64_t>(need + need / 2, 1024);
    CUDA_TRY(c, cudaMallocHost((void **)&ptr, n * sizeof(T)));
    cap = n;
    return 0;
}

static uint64_t isqrt_host(uint64_t n) {
    uint64_t r = (uint64_t)std::sqrt((double)n);
    while (r * r > n) r--;
    while ((r + 1) * (r + 1) <= n) r++;
    return r;
}

extern "C" int ps4_abi_version(void) { return PS4_ABI_VERSION; }

extern "C" const char *ps4_last_error(const ps4_ctx *ctx) { return ctx ? ctx->err.c_str() : "null context"; }

extern "C" double ps4_last_kernel_ms(const ps4_ctx *ctx) { return ctx ? ctx->last_ms : 0.0; }

extern "C" uint64_t ps4_last_launches(const ps4_ctx *ctx) { return ctx ? ctx->last_launches : 0; }

extern "C" void ps4_destroy(ps4_ctx *c) {
    if (!c) return;
    cudaFree(c->d_spfq); cudaFree(c->d_ndiv); cudaFree(c->d_items); cudaFree(c->d_counters);
    cudaFree(c->d_hits); cudaFree(c->d_exts); cudaFree(c->d_sixes); cudaFree(c->d_quads);
    cudaFree(c->d_scratch); cudaFree(c->d_status); cudaFree(c->d_jobs); cudaFree(c->d_raw); cudaFree(c->d_seq);
    cudaFree(c->d_fac3);
    cudaFree(c->d_tri_in); cudaFree(c->d_tri_state); cudaFree(c->d_tri_out); cudaFree(c->d_tri_cnt);
    if (c->h_status) cudaFreeHost(c->h_status);
    if (c->h_segs) cudaFreeHost(c->h_segs);
    if (c->h_hits) cudaFreeHost(c->h_hits);
    if (c->h_exts) cudaFreeHost(c->h_exts);
    if (c->h_sixes) cudaFreeHost(c->h_sixes);
    if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
    for (cudaEvent_t e : c->kev) cudaEventDestroy(e);
    if (c->ev0) cudaEventDestroy(c->ev0);
    if (c->ev1) cudaEventDestroy(c->ev1);
    if (c->own_stream && c->stream) cudaStreamDestroy(c->stream);
    delete c;
}

static const uint64_t S_LIMIT = 1ull << 44;   // roots < 2^22: 4-set staging packs 10 bits above them

extern "C" int ps4_create(const ps4_config *cfg, ps4_ctx **out) {
    if (!cfg || !out) return PS4_ERR_ARG;
    *out = nullptr;
    ps4_ctx *c = new ps4_ctx();
    c->cfg = *cfg;
    if (c->cfg.cap_reps == 0) c->cfg.cap_reps = 512;
    if (c->cfg.cap_divs == 0) c->cfg.cap_divs = 16384;
    if (c->cfg.cap_ext == 0) c->cfg.cap_ext = 64;
    if (c->cfg.s_hi_max < 2) c->cfg.s_hi_max = 2;
    if (c->cfg.s_hi_max > S_LIMIT) {
        int rc = set_err(c, PS4_ERR_ARG, "s_hi_max %llu exceeds the supported bound 2^44",
                         (unsigned long long)c->cfg.s_hi_max);
        *out = c;
        return rc;
    }
    // default tiles: 2^13 S for the two-kernel pipeline (four 256-thread tile CTAs per SM), 2^14
    // for the one-kernel designs, whose CTAs keep 512 threads
    if (c->cfg.kernel != PS4_KERNEL_BATCHED) c->tile_log2 = 14;
    if (c->cfg.log2_tile) c->tile_log2 = std::min(14u, std::max(12u, c->cfg.log2_tile));
    *out = c;
    int ndev = 0;
    if (cudaGetDeviceCount(&ndev) != cudaSuccess || ndev == 0)
        return set_err(c, PS4_ERR_CUDA, "no CUDA device available (libps4 has no CPU path)");
    CUDA_TRY(c, cudaSetDevice(cfg->device));
    cudaDeviceProp prop;
    CUDA_TRY(c, cudaGetDeviceProperties(&prop, cfg->device));
    if (prop.major != 10)
        return set_err(c, PS4_ERR_CUDA, "device %d is sm_%d%d; libps4 is built for sm_100a only", cfg->device,
                       prop.major, prop.minor);
    c->num_sms = prop.multiProcessorCount;
    if (cfg->stream) {
        c->stream = (cudaStream_t)cfg->stream;
    } else {
        CUDA_TRY(c, cudaStreamCreateWithFlags(&c->stream, cudaStreamNonBlocking));
        c->own_stream = true;
    }
    CUDA_TRY(c, cudaEventCreate(&c->ev0));
    CUDA_TRY(c, cudaEventCreate(&c->ev1));
    c->tab_n = 2 * isqrt_host(c->cfg.s_hi_max) + 64;      // s4.c:440
    CUDA_TRY(c, cudaMalloc((void **)&c->d_spfq, c->tab_n * sizeof(uint64_t)));
    CUDA_TRY(c, cudaMalloc((void **)&c->d_ndiv, c->tab_n * sizeof(uint16_t)));
    CUDA_TRY(c, cudaMalloc((void **)&c->d_status, sizeof(Status)));
    CUDA_TRY(c, cudaMallocHost((void **)&c->h_status, sizeof(Status)));
    CUDA_TRY(c, (cudaError_t)launch_tables(c->d_spfq, c->d_ndiv, c->tab_n, c->stream));
    CUDA_TRY(c, cudaMalloc((void **)&c->d_fac3, c->tab_n * sizeof(uint4)));
    CUDA_TRY(c, (cudaError_t)launch_fac3(c->d_fac3, c->tab_n, c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    return PS4_OK;
}

namespace ps4 {
void stats_add(ps4_stats *s, const unsigned long long *k) {
    uint64_t *add = &s->S_done;          // S_done .. ext_sqrt are contiguous
    for (int i = 0; i < 10; i++) add[i] += k[i];
    for (int i = 0; i < 100; i++) s->hist5[i] += k[K_HIST5 + i];
    s->max_reps = std::max<uint64_t>(s->max_reps, k[K_MAX_REPS]);
    s->max_divisors = std::max<uint64_t>(s->max_divisors, k[K_MAX_DIVS]);
    s->max_extensions = std::max<uint64_t>(s->max_extensions, k[K_MAX_EXT]);
}

const char *fatal_text(unsigned code) {
    switch (code) {
        case E_CAP_REPS: return "representation capacity exceeded";
        case E_CAP_DIVS: return "divisor capacity exceeded";
        case E_CAP_EXT: return "extension capacity exceeded";
        case E_VERIFY: return "quadruple verification failed";
        default: return "internal capacity exceeded";
    }
}

// 4-sets per S grow slowly with S (0.13 below 1e10, 0.29 near 2e12); a batch of the
// two-kernel pipeline is sized so that this bound, with margin, fills at most 90 % of the queue.
double jobs_per_S_bound(uint64_t S_hi) {
    const double dec = S_hi > 1000000000ull ? std::log10((double)S_hi / 1e9) : 0.0;
    return 0.25 + 0.05 * dec;
}

// Hits in a deterministic order -- item, S, then the reference's emission order (px, py, pz,
// class) -- with each hit's extensions moved behind it and 6-set records re-pointed and sorted.
// Writes the ordered hits and extensions to out_hits / out_exts (nh and the extensions' count
// entries, not overlapping the inputs); sorts sixes in place.
void canonical_order_into(const ps4_hit *hits, uint64_t nh, const ps4_ext *exts, ps4_six *sixes, uint64_t ns,
                          ps4_hit *out_hits, ps4_ext *out_exts) {
    struct Key {                       // the sort key next to the index: one contiguous array to sort
        uint64_t S;
        uint32_t item, o[4], idx;
    };
    std::vector<Key> key(nh);
    for (uint64_t i = 0; i < nh; i++) {
        const ps4_hit &h = hits[i];
        key[i] = Key{h.S, h.item, {h.order[0], h.order[1], h.order[2], h.order[3]}, (uint32_t)i};
    }
    std::sort(key.begin(), key.end(), [](const Key &x, const Key &y) {
        if (x.item != y.item) return x.item < y.item;
        if (x.S != y.S) return x.S < y.S;
        for (int i = 0; i < 4; i++)
            if (x.o[i] != y.o[i]) return x.o[i] < y.o[i];
        return false;
    });
    std::vector<uint32_t> newpos(ns ? nh : 0);
    uint32_t ne = 0;
    for (uint64_t i = 0; i < nh; i++) {
        ps4_hit h = hits[key[i].idx];
        if (ns) newpos[key[i].idx] = (uint32_t)i;
        if (h.n_ext) memcpy(out_exts + ne, exts + h.first_ext, h.n_ext * sizeof(ps4_ext));
        h.first_ext = ne;
        ne += h.n_ext;
        out_hits[i] = h;
    }
    for (uint64_t s = 0; s < ns; s++) sixes[s].hit = newpos[sixes[s].hit];
    std::sort(sixes, sixes + ns, [](const ps4_six &x, const ps4_six &y) {
        if (x.hit != y.hit) return x.hit < y.hit;
        if (x.t != y.t) return x.t < y.t;
        return x.s < y.s;
    });
}

void canonical_order(std::vector<ps4_hit> &hits, std::vector<ps4_ext> &exts, std::vector<ps4_six> &sixes) {
    std::vector<ps4_hit> h2(hits.size());
    std::vector<ps4_ext> e2(exts.size());
    canonical_order_into(hits.data(), hits.size(), exts.data(), sixes.data(), sixes.size(), h2.data(), e2.data());
    hits.swap(h2);
    exts.swap(e2);
}
}  // namespace ps4

// ---- one search = enqueue (host prep + launch, no wait) + finish (wait, check, collect) ----

// Cut a call's items into batches for the two-kernel pipeline: each batch holds at most
// ~90 % of the job queue in expected 4-sets (jobs_per_S_bound).  Within a batch the segments
// are ordered by estimated cost per tile, ascending; the tile kernels claim tiles from the
// last one down (tile_bounds), so the costliest tiles -- the highest S, whose representation
// and 4-set counts are largest -- start first and narrow partial tiles fill the tail.
static void plan_batches(ps4_ctx *c, const std::vector<Item> &items, unsigned TL, std::vector<Item> &segs,
                         std::vector<size_t> &batch_start, std::vector<uint64_t> &batch_tiles) {
    const uint32_t n_items = (uint32_t)items.size();
    size_t i = 0;
    uint64_t pos = n_items ? items[0].lo : 0;
    while (i < n_items) {
        const size_t b0 = segs.size();
        double budget = 0.9 * (double)c->jobs_cap / (double)c->batch_div;
        while (i < n_items && budget > 0) {
            const Item &it = items[i];
            if (pos < it.lo) pos = it.lo;
            const double dens = jobs_per_S_bound(it.hi);
            uint64_t room = (uint64_t)(budget / dens);
            room = std::max<uint64_t>(room >> TL, 1) << TL;          // whole tiles
            const uint64_t end = it.hi - pos > room ? pos + room : it.hi;
            if (end > pos) {
                Item sg;
                sg.lo = pos; sg.hi = end; sg.id = it.id; sg.pad = 0; sg.tile_base = 0;
                segs.push_back(sg);
            }
            budget -= dens * (double)(end - pos);
            pos = end;
            if (pos >= it.hi) { i++; if (i < n_items) pos = items[i].lo; }
        }
        if (segs.size() == b0) continue;
        std::stable_sort(segs.begin() + b0, segs.end(), [](const Item &x, const Item &y) {
            if (x.hi != y.hi) return x.hi < y.hi;               // cost density grows with S
            return x.hi - x.lo < y.hi - y.lo;
        });
        uint64_t tiles = 0;
        for (size_t k = b0; k < segs.size(); k++) {
            segs[k].tile_base = tiles;
            tiles += (segs[k].hi - segs[k].lo + (1ull << TL) - 1) >> TL;
        }
        batch_start.push_back(b0);
        batch_tiles.push_back(tiles);
    }
}

template <class T>
static void key_add(std::string &k, const T &v) {
    k.append(reinterpret_cast<const char *>(&v), sizeof v);
}

static int enqueue_items(ps4_ctx *c) {
    PendingSearch &p = c->pend;
    const uint32_t n_items = (uint32_t)p.items.size();
    int kernel = c->fused_fallback ? (int)PS4_KERNEL_FUSED : (int)c->cfg.kernel;
    if (kernel == PS4_KERNEL_PERSIST && c->persist_fallback) kernel = PS4_KERNEL_BATCHED;
    const bool persist = kernel == PS4_KERNEL_PERSIST;
    const unsigned TL = persist ? 13u : c->tile_log2;      // the persistent kernel's tiles are 2^13 S
    if (kernel == PS4_KERNEL_BATCHED) {          // queue: the call's expected 4-sets, 2^20 .. jobs_cap_max
        double need = 0;
        for (uint32_t i = 0; i < n_items; i++)
            need += jobs_per_S_bound(p.items[i].hi) * (double)(p.items[i].hi - p.items[i].lo);
        while (c->jobs_cap < c->jobs_cap_max && (double)c->jobs_cap * 0.9 < need) c->jobs_cap <<= 1;
    }
    std::vector<Item> segs;                      // all batches' segments, batch after batch
    std::vector<size_t> batch_start;             // segs index where each batch begins
    std::vector<uint64_t> batch_tiles;
    if (kernel == PS4_KERNEL_BATCHED) {
        plan_batches(c, p.items, TL, segs, batch_start, batch_tiles);
    } else if (persist) {
        // every item in one launch, ordered by estimated cost per tile (the tiles are taken from
        // the last one down, so the costliest start first and narrow ones fill the tail)
        segs = p.items;
        std::stable_sort(segs.begin(), segs.end(), [](const Item &x, const Item &y) {
            if (x.hi != y.hi) return x.hi < y.hi;
            return x.hi - x.lo < y.hi - y.lo;
        });
        uint64_t tiles = 0;
        for (auto &sg : segs) {
            sg.tile_base = tiles;
            tiles += (sg.hi - sg.lo + (1ull << TL) - 1) >> TL;
        }
        batch_start.push_back(0);
        batch_tiles.push_back(tiles);
    } else {
        uint64_t tiles = 0;
        for (uint32_t i = 0; i < n_items; i++) {
            Item sg = p.items[i];
            sg.tile_base = tiles;
            tiles += (sg.hi - sg.lo + (1ull << TL) - 1) >> TL;
            segs.push_back(sg);
        }
        batch_start.push_back(0);
        batch_tiles.push_back(tiles);
    }
    uint64_t tiles_total = 0;
    for (uint64_t t : batch_tiles) {
        if (t >= (1ull << 31))
            return set_err(c, PS4_ERR_ARG, "range too large for one call (%llu tiles); split it", (unsigned long long)t);
        tiles_total += t;
    }
    p.tiles = tiles_total;

    // every allocation before any launch (a captured call may allocate nothing)
    if (grow32(c, c->d_items, c->items_cap, std::max<size_t>(segs.size(), 1))) return PS4_ERR_CUDA;
    if (c->h_segs_cap < segs.size() || !c->h_segs) {
        if (c->h_segs) cudaFreeHost(c->h_segs);
        c->h_segs = nullptr;
        c->h_segs_cap = std::max<uint64_t>(segs.size(), 1024);
        CUDA_TRY(c, cudaMallocHost((void **)&c->h_segs, c->h_segs_cap * sizeof(Item)));
    }
    if (kernel == PS4_KERNEL_BATCHED && c->d_jobs_words < 6 * c->jobs_cap)
        if (grow(c, c->d_jobs, c->d_jobs_words, 6 * c->jobs_cap)) return PS4_ERR_CUDA;
    if (kernel == PS4_KERNEL_BATCHED &&
        c->raw_words < (uint64_t)c->num_sms * c->gen_ctas * SUPER_K * RAW_PER_TILE)
        if (grow(c, c->d_raw, c->raw_words, (uint64_t)c->num_sms * 2 * SUPER_K * RAW_PER_TILE)) return PS4_ERR_CUDA;
    const int g_persist = c->num_sms * persist_ctas_per_sm();
    const uint32_t raw_cap_persist = RAW_PER_TILE / 2;           // 2^13-S tiles: half the representations
    if (persist) {
        if (c->d_jobs_words < 6 * c->ring_cap && grow(c, c->d_jobs, c->d_jobs_words, 6 * c->ring_cap))
            return PS4_ERR_CUDA;
        if (grow(c, c->d_seq, c->seq_cap, c->ring_cap)) return PS4_ERR_CUDA;
        if (c->raw_words < (uint64_t)g_persist * SUPER_K * raw_cap_persist &&
            grow(c, c->d_raw, c->raw_words, (uint64_t)g_persist * SUPER_K * raw_cap_persist))
            return PS4_ERR_CUDA;
    }
    const uint32_t stage_cap = stage_cap_for(TL, c->cfg.cap_reps);
    int grid = c->num_sms * (c->cfg.ctas_per_sm ? (int)c->cfg.ctas_per_sm : 1);
    if ((uint64_t)grid > tiles_total) grid = (int)std::max<uint64_t>(tiles_total, 1);
    if (kernel == PS4_KERNEL_FUSED) {
        uint64_t cap = c->scratch_words;
        if (grow(c, c->d_scratch, cap, (uint64_t)grid * 6 * stage_cap)) return PS4_ERR_CUDA;
        c->scratch_words = cap;
    }

    SearchArgs a;
    memset(&a, 0, sizeof a);
    a.log2_tile = TL;
    a.spfq = c->d_spfq; a.ndiv = c->d_ndiv; a.tab_n = c->tab_n; a.fac3 = c->d_fac3;
    a.counters = c->d_counters;
    a.hits = c->d_hits; a.hits_cap = c->hits_cap;
    a.exts = c->d_exts; a.exts_cap = c->exts_cap;
    a.sixes = c->d_sixes; a.sixes_cap = c->sixes_cap;
    a.quads = p.dump ? c->d_quads : nullptr; a.quads_cap = p.dump ? c->quads_cap : 0;
    a.status = c->d_status;
    a.cap_reps = c->cfg.cap_reps; a.cap_divs = c->cfg.cap_divs; a.cap_ext = c->cfg.cap_ext;
    a.flags = c->cfg.flags & (p.dump ? ~0u : ~(uint32_t)PS4_F_DUMP4);
    a.jobs = c->d_jobs;
    a.jobs_cap = c->jobs_cap;
    if (kernel == PS4_KERNEL_BATCHED) { a.raw = c->d_raw; a.raw_cap = raw_cap_for(TL); }
    if (persist) {
        a.jobs_cap = c->ring_cap;
        a.seq = c->d_seq;
        a.ring_mask = c->ring_cap - 1;
        a.ring_fast = 2ull * (uint64_t)g_persist * PBS;          // > every warp claiming 32 at once
        a.ring_high = 32ull * (uint64_t)g_persist * PBS;         // ~1 ms of engine work at full rate
        a.ring_low = 4ull * (uint64_t)g_persist * PBS;
        a.raw = c->d_raw;
        a.raw_cap = raw_cap_persist;
    }
    const bool ext = !(c->cfg.flags & PS4_F_NOEXT);
    // gen_ctas counts 512 threads per SM: one or two 512-thread CTAs on 2^14-S tiles, twice as
    // many 256-thread ones on smaller tiles
    const int g_gen = c->num_sms * (int)c->gen_ctas * (gen_threads(14) / gen_threads(TL)), g_ext = c->num_sms * (int)c->ext_ctas;

    // A call of several batches runs as one CUDA graph holding its whole launch sequence; the
    // graph is kept and replayed while the next call is the same (items, sizes, buffers).
    const bool graph = !c->cfg.time_kernels &&
                       (c->cfg.use_graph == PS4_GRAPH_ALWAYS ||
                        (c->cfg.use_graph == PS4_GRAPH_AUTO &&
                         ((kernel == PS4_KERNEL_BATCHED && batch_start.size() >= 2) || persist)));
    const bool timed = c->cfg.time_kernels && kernel == PS4_KERNEL_BATCHED;
    c->kev_used = 0;
    if (timed) {                                  // 4 events per batch: gen start/end, ext start/end
        while (c->kev.size() < 4 * batch_start.size()) {
            cudaEvent_t e;
            CUDA_TRY(c, cudaEventCreate(&e));
            c->kev.push_back(e);
        }
    }
    std::string key;
    if (graph) {
        key.append(reinterpret_cast<const char *>(segs.data()), segs.size() * sizeof(Item));
        for (size_t b : batch_start) key_add(key, b);
        key_add(key, a);
        key_add(key, kernel); key_add(key, n_items); key_add(key, grid); key_add(key, g_gen); key_add(key, g_ext);
        key_add(key, stage_cap); key_add(key, c->d_scratch); key_add(key, c->h_segs); key_add(key, c->d_items);
        key_add(key, c->stream);
    }
    if (!segs.empty()) memcpy(c->h_segs, segs.data(), segs.size() * sizeof(Item));
    c->h2d_bytes += segs.size() * sizeof(Item);
    CUDA_TRY(c, cudaEventRecord(c->ev0, c->stream));
    if (graph && c->graph_exec && key == c->graph_key) {
        CUDA_TRY(c, cudaGraphLaunch(c->graph_exec, c->stream));
        c->last_launches += c->graph_launches;
        c->graph_replays++;
    } else {
        if (graph) CUDA_TRY(c, cudaStreamBeginCapture(c->stream, cudaStreamCaptureModeRelaxed));
        const uint64_t launches0 = c->last_launches;
        int rc = PS4_OK;
        cudaError_t e = cudaSuccess;
        if (!segs.empty())
            e = cudaMemcpyAsync(c->d_items, c->h_segs, segs.size() * sizeof(Item), cudaMemcpyHostToDevice, c->stream);
        if (e == cudaSuccess)
            e = cudaMemsetAsync(c->d_counters, 0, (size_t)n_items * K_SLOTS * sizeof(unsigned long long), c->stream);
        if (e == cudaSuccess) e = cudaMemsetAsync(c->d_status, 0, sizeof(Status), c->stream);
        if (e == cudaSuccess && kernel == PS4_KERNEL_BATCHED) {
            for (size_t b = 0; b < batch_start.size() && e == cudaSuccess; b++) {
                const size_t s0 = batch_start[b], s1 = b + 1 < batch_start.size() ? batch_start[b + 1] : segs.size();
                a.items = c->d_items + s0;
                a.n_items = (uint32_t)(s1 - s0);
                a.n_tiles = batch_tiles[b];
                const int g = (int)std::min<uint64_t>((uint64_t)g_gen, std::max<uint64_t>(a.n_tiles, 1));
                // n_jobs, tile_next, ext_next: the per-batch tail of the status block
                e = cudaMemsetAsync(&c->d_status->n_jobs, 0, 2 * sizeof(unsigned long long), c->stream);
                if (timed && e == cudaSuccess) e = cudaEventRecord(c->kev[4 * b], c->stream);
                if (e == cudaSuccess) e = (cudaError_t)launch_gen(a, g, c->stream);
                if (timed && e == cudaSuccess) e = cudaEventRecord(c->kev[4 * b + 1], c->stream);
                c->last_launches++;
                if (e == cudaSuccess && ext) {
                    if (timed) e = cudaEventRecord(c->kev[4 * b + 2], c->stream);
                    if (e == cudaSuccess) e = (cudaError_t)launch_ext(a, g_ext, c->stream);
                    if (timed && e == cudaSuccess) e = cudaEventRecord(c->kev[4 * b + 3], c->stream);
                    c->last_launches++;
                }
                if (timed) c->kev_used = 4 * (b + 1);
            }
        } else if (e == cudaSuccess && persist && tiles_total > 0) {
            a.items = c->d_items; a.n_items = (uint32_t)segs.size(); a.n_tiles = tiles_total;
            e = (cudaError_t)launch_ring_init(c->d_seq, c->ring_cap, c->stream);
            if (e == cudaSuccess) e = (cudaError_t)launch_persist(a, g_persist, c->stream);
            c->last_launches += 2;
        } else if (e == cudaSuccess && tiles_total > 0) {
            a.items = c->d_items; a.n_items = (uint32_t)segs.size(); a.n_tiles = tiles_total;
            a.scratch = c->d_scratch; a.stage_cap = stage_cap;
            // launch_search's selector: PS4_KERNEL_BATCHED there is the fused persistent kernel
            e = (cudaError_t)launch_search(a, kernel == PS4_KERNEL_PLAIN ? PS4_KERNEL_PLAIN : PS4_KERNEL_BATCHED, grid,
                                           c->stream);
            c->last_launches++;
        }
        if (graph) {
            cudaGraph_t g = nullptr;
            const cudaError_t e2 = cudaStreamEndCapture(c->stream, &g);
            if (e == cudaSuccess) e = e2;
            if (e == cudaSuccess) {
                if (c->graph_exec) cudaGraphExecDestroy(c->graph_exec);
                c->graph_exec = nullptr;
                c->graph_key.clear();
                e = cudaGraphInstantiate(&c->graph_exec, g, 0);
            }
            if (g) cudaGraphDestroy(g);
            if (e == cudaSuccess) e = cudaGraphLaunch(c->graph_exec, c->stream);
            if (e == cudaSuccess) {
                c->graph_key.swap(key);
                c->graph_launches = c->last_launches - launches0;
                c->graph_captures++;
            }
        }
        if (e != cudaSuccess) rc = set_err(c, PS4_ERR_CUDA, "search launch failed: %s", cudaGetErrorString(e));
        if (rc) return rc;
    }
    CUDA_TRY(c, cudaEventRecord(c->ev1, c->stream));
    CUDA_TRY(c, cudaMemcpyAsync(c->h_status, c->d_status, sizeof(Status), cudaMemcpyDeviceToHost, c->stream));
    return PS4_OK;
}

static int begin_items(ps4_ctx *c, const uint64_t *lo, const uint64_t *hi, uint32_t n_items, bool want_dump,
                       uint64_t dump_cap) {
    if (c->pend.active) return set_err(c, PS4_ERR_ARG, "a search is already enqueued on this context");
    PendingSearch &p = c->pend;
    p.items.assign(n_items, Item{});
    c->fused_fallback = false;
    c->persist_fallback = false;
    c->last_launches = 0;
    c->last_ms = 0.0;
    c->h2d_bytes = c->d2h_bytes = 0;
    for (uint32_t i = 0; i < n_items; i++) {
        uint64_t a = std::max<uint64_t>(lo[i], 1), b = hi[i];
        if (b > c->cfg.s_hi_max)
            return set_err(c, PS4_ERR_ARG, "S_hi %llu exceeds the context's s_hi_max %llu", (unsigned long long)b,
                           (unsigned long long)c->cfg.s_hi_max);
        if (b < a) b = a;
        p.items[i].lo = a;
        p.items[i].hi = b;
        p.items[i].id = i;
    }
    if (grow32(c, c->d_items, c->items_cap, n_items)) return PS4_ERR_CUDA;
    if (grow32(c, c->d_counters, c->counters_items, (uint64_t)n_items * K_SLOTS)) return PS4_ERR_CUDA;
    p.dump = (c->cfg.flags & PS4_F_DUMP4) && want_dump && dump_cap > 0;
    if (p.dump && grow(c, c->d_quads, c->quads_cap, dump_cap)) return PS4_ERR_CUDA;
    // result buffers sized up front from the call's width (4-sets with an extension stay below
    // 1.5e-5 per S on every checked range), so a long call is not repeated to grow them
    double width = 0;
    for (uint32_t i = 0; i < n_items; i++) width += (double)(p.items[i].hi - p.items[i].lo);
    const uint64_t hits_est = std::min<uint64_t>(1024 + (uint64_t)(2e-5 * width), 1ull << 30);
    if (grow32(c, c->d_hits, c->hits_cap, std::max<uint64_t>({(uint64_t)c->hits_cap, 1u << 16, hits_est})))
        return PS4_ERR_CUDA;
    if (grow32(c, c->d_exts, c->exts_cap, std::max<uint64_t>({(uint64_t)c->exts_cap, 1u << 17, 2 * hits_est})))
        return PS4_ERR_CUDA;
    if (grow32(c, c->d_sixes, c->sixes_cap, std::max<uint32_t>(c->sixes_cap, 1024))) return PS4_ERR_CUDA;
    int rc = enqueue_items(c);
    if (rc == PS4_OK) p.active = true;
    return rc;
}

// Wait for the enqueued search, re-run it on internal capacity limits, then copy the results
// into the caller's buffers and add the counters (stats: one per item, +=).
static int finish_items(ps4_ctx *c, ps4_stats *stats, ps4_results *res) {
    PendingSearch &p = c->pend;
    if (!p.active) return set_err(c, PS4_ERR_ARG, "no search enqueued on this context");
    p.active = false;
    const uint32_t n_items = (uint32_t)p.items.size();
    for (int attempt = 0; attempt < 16; attempt++) {
        if (attempt > 0) {
            int rc = enqueue_items(c);
            if (rc) return rc;
        }
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
        c->d2h_bytes += sizeof(Status);
        if (p.tiles > 0) {
            float ms = 0.f;
            cudaEventElapsedTime(&ms, c->ev0, c->ev1);
            c->last_ms = ms;                     // the attempt whose results are kept
            c->gen_ms = c->ext_ms = 0.0;
            const bool ext = !(c->cfg.flags & PS4_F_NOEXT);
            for (size_t i = 0; i + 3 < c->kev_used; i += 4) {
                float g = 0.f, x = 0.f;
                cudaEventElapsedTime(&g, c->kev[i], c->kev[i + 1]);
                if (ext) cudaEventElapsedTime(&x, c->kev[i + 2], c->kev[i + 3]);
                c->gen_ms += g;
                c->ext_ms += x;
            }
        }
        const Status &st = *c->h_status;
        const unsigned code = (unsigned)(st.err & 0xFF);
        const unsigned long long errS = st.err >> 8;
        if (code == E_QUEUE) {                   // a batch outgrew the job queue: narrower batches
            if (c->batch_div < (1u << 16)) { c->batch_div *= 2; continue; }
            return set_err(c, PS4_ERR_CUDA, "job queue overflow persists near S=%llu", errS);
        }
        if ((code == E_TIMEOUT || code == E_TILE) && c->cfg.kernel == PS4_KERNEL_PERSIST && !c->persist_fallback &&
            !c->fused_fallback) {
            c->persist_fallback = true;          // the two-kernel pipeline: no waits, smaller tiles on E_TILE
            continue;
        }
        if (code == E_TIMEOUT)
            return set_err(c, PS4_ERR_TIMEOUT, "a bounded device wait gave up (wait %llu); the call did not complete",
                           errS);
        if (code == E_EXTLIST && (c->cfg.kernel == PS4_KERNEL_BATCHED || c->cfg.kernel == PS4_KERNEL_PERSIST) &&
            !c->fused_fallback) {
            c->fused_fallback = true;            // more extensions in one engine round than its list holds: fused kernel
            continue;
        }
        if (code == E_TILE || code == E_EXTLIST) {
            if (c->tile_log2 > 12) { c->tile_log2--; continue; }
            static const char *list_name[5] = {"?", "selected-S list", "representation list", "4-set staging",
                                               "extension list"};
            return set_err(c, PS4_ERR_CAP_REPS,
                           "FATAL: tile capacity exceeded near S=%llu (%s: %llu > %llu); this interval is NOT "
                           "certified complete", errS, list_name[st.diag[0] < 5 ? st.diag[0] : 0], st.diag[1],
                           st.diag[2]);
        }
        if (code != 0) {
            if (code == E_VERIFY)
                return set_err(c, PS4_ERR_VERIFY, "BAD 4-set S=%llu [%lld,%lld,%lld,%lld]", st.verify_bad[0],
                               (long long)st.verify_bad[1], (long long)st.verify_bad[2], (long long)st.verify_bad[3],
                               (long long)st.verify_bad[4]);
            return set_err(c, (int)code, "FATAL: %s; this interval is NOT certified complete", fatal_text(code));
        }
        bool regrow = false;
        if (st.n_hits > c->hits_cap) {
            if (grow32(c, c->d_hits, c->hits_cap, (uint64_t)st.n_hits * 3 / 2 + 1024)) return PS4_ERR_CUDA;
            regrow = true;
        }
        if (st.n_exts > c->exts_cap) {
            if (grow32(c, c->d_exts, c->exts_cap, (uint64_t)st.n_exts * 3 / 2 + 1024)) return PS4_ERR_CUDA;
            regrow = true;
        }
        if (st.n_sixes > c->sixes_cap) {
            if (grow32(c, c->d_sixes, c->sixes_cap, (uint64_t)st.n_sixes * 3 / 2 + 64)) return PS4_ERR_CUDA;
            regrow = true;
        }
        if (regrow) continue;
        if (res) {
            res->n_quads = p.dump ? st.n_quads : 0;
            if (p.dump && st.n_quads > res->quads_cap) {
                res->n_hits = st.n_hits; res->n_exts = st.n_exts; res->n_sixes = st.n_sixes;
                p.active = true;                 // results stay on the device: finish may be called again
                return set_err(c, PS4_ERR_OUTPUT_FULL, "dump4 buffer holds %llu 4-sets, %llu needed",
                               (unsigned long long)res->quads_cap, st.n_quads);
            }
        }
        std::vector<unsigned long long> k((size_t)n_items * K_SLOTS);
        CUDA_TRY(c, cudaMemcpyAsync(k.data(), c->d_counters, k.size() * sizeof(unsigned long long),
                                    cudaMemcpyDeviceToHost, c->stream));
        const bool fits = res && st.n_hits <= res->hits_cap && st.n_exts <= res->exts_cap &&
                          st.n_sixes <= res->sixes_cap;
        if (fits) {                              // the records land in pinned buffers, then go in order to res
            if (grow_pinned(c, c->h_hits, c->h_hits_cap, st.n_hits) ||
                grow_pinned(c, c->h_exts, c->h_exts_cap, st.n_exts) ||
                grow_pinned(c, c->h_sixes, c->h_sixes_cap, st.n_sixes))
                return PS4_ERR_CUDA;
            if (st.n_hits)
                CUDA_TRY(c, cudaMemcpyAsync(c->h_hits, c->d_hits, st.n_hits * sizeof(ps4_hit), cudaMemcpyDeviceToHost,
                                            c->stream));
            if (st.n_exts)
                CUDA_TRY(c, cudaMemcpyAsync(c->h_exts, c->d_exts, st.n_exts * sizeof(ps4_ext), cudaMemcpyDeviceToHost,
                                            c->stream));
            if (st.n_sixes)
                CUDA_TRY(c, cudaMemcpyAsync(c->h_sixes, c->d_sixes, st.n_sixes * sizeof(ps4_six),
                                            cudaMemcpyDeviceToHost, c->stream));
        }
        if (res && p.dump && st.n_quads)
            CUDA_TRY(c, cudaMemcpyAsync(res->quads, c->d_quads, st.n_quads * sizeof(ps4_quad), cudaMemcpyDeviceToHost,
                                        c->stream));
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
        c->d2h_bytes += k.size() * sizeof(unsigned long long) +
                        (fits ? st.n_hits * sizeof(ps4_hit) + st.n_exts * sizeof(ps4_ext) +
                                    st.n_sixes * sizeof(ps4_six)
                              : 0) +
                        ((res && p.dump) ? st.n_quads * sizeof(ps4_quad) : 0);
        if (res) {
            res->n_hits = st.n_hits;
            res->n_exts = st.n_exts;
            res->n_sixes = st.n_sixes;
            if (!fits) {
                p.active = true;                 // results stay on the device: finish may be called again
                return set_err(c, PS4_ERR_OUTPUT_FULL, "result buffers too small: need hits=%llu exts=%llu sixes=%llu",
                               (unsigned long long)res->n_hits, (unsigned long long)res->n_exts,
                               (unsigned long long)res->n_sixes);
            }
            canonical_order_into(c->h_hits, st.n_hits, c->h_exts, c->h_sixes, st.n_sixes, res->hits, res->exts);
            if (st.n_sixes) memcpy(res->sixes, c->h_sixes, st.n_sixes * sizeof(ps4_six));
        }
        if (stats)
            for (uint32_t i = 0; i < n_items; i++) stats_add(&stats[i], &k[(size_t)i * K_SLOTS]);
        return PS4_OK;
    }
    return set_err(c, PS4_ERR_CUDA, "search did not converge after repeated re-runs");
}

extern "C" int ps4_search_range(ps4_ctx *c, uint64_t lo, uint64_t hi, ps4_stats *stats, ps4_results *res) {
    if (!c) return PS4_ERR_ARG;
    int rc = begin_items(c, &lo, &hi, 1, res != nullptr, res ? res->quads_cap : 0);
    if (rc == PS4_OK) rc = finish_items(c, stats, res);
    c->pend.active = false;              // a synchronous call is repeated whole after any error
    return rc;
}

extern "C" int ps4_search_batch(ps4_ctx *c, const uint64_t *lo, const uint64_t *hi, uint32_t n_items, ps4_stats *stats,
                                ps4_results *res) {
    if (!c) return PS4_ERR_ARG;
    if (!lo || !hi || n_items == 0) return set_err(c, PS4_ERR_ARG, "ps4_search_batch: empty batch");
    int rc = begin_items(c, lo, hi, n_items, res != nullptr, res ? res->quads_cap : 0);
    if (rc == PS4_OK) rc = finish_items(c, stats, res);
    c->pend.active = false;
    return rc;
}

extern "C" int ps4_search_enqueue(ps4_ctx *c, uint64_t lo, uint64_t hi) {
    if (!c) return PS4_ERR_ARG;
    int rc = begin_items(c, &lo, &hi, 1, false, 0);
    if (rc) c->pend.active = false;
    return rc;
}

extern "C" int ps4_search_finish(ps4_ctx *c, ps4_stats *stats, ps4_results *res) {
    if (!c) return PS4_ERR_ARG;
    return finish_items(c, stats, res);
}

extern "C" void ps4_last_transfer_bytes(const ps4_ctx *c, uint64_t *h2d, uint64_t *d2h) {
    if (h2d) *h2d = c ? c->h2d_bytes : 0;
    if (d2h) *d2h = c ? c->d2h_bytes : 0;
}

// ---- one range on several devices ----

extern "C" int ps4_plan_shards(uint64_t lo, uint64_t hi, uint32_t n, uint64_t *bounds) {
    if (n == 0 || !bounds) return PS4_ERR_ARG;
    lo = std::max<uint64_t>(lo, 1);
    hi = std::max(hi, lo);
    // cumulative cost C(S) = S^(1+beta): density ~ S^beta, beta fitted to the measured rates
    const double beta = 0.16, g = 1.0 + beta;
    const double c0 = std::pow((double)lo, g), c1 = std::pow((double)hi, g);
    const uint64_t tile = 1ull << 14;
    bounds[0] = lo;
    for (uint32_t i = 1; i < n; i++) {
        const double x = std::pow(c0 + (c1 - c0) * (double)i / (double)n, 1.0 / g);
        uint64_t b = x <= (double)lo ? lo : x >= (double)hi ? hi : (uint64_t)x;
        b = (b + tile / 2) / tile * tile;                   // nearest tile boundary
        b = std::min(hi, std::max(b, bounds[i - 1]));
        bounds[i] = b;
    }
    bounds[n] = hi;
    return PS4_OK;
}

// ---- self-check of the persistent kernel's bounded wait ----

extern "C" int ps4_check_ring_wait(int device, uint64_t *waited_ns) {
    if (waited_ns) *waited_ns = 0;
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess) return PS4_ERR_CUDA;
    Status *d_st = nullptr;
    uint32_t *d_seq = nullptr;
    unsigned long long *d_out = nullptr;
    cudaError_t e = cudaMalloc((void **)&d_st, sizeof(Status));
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_seq, sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_out, 2 * sizeof(unsigned long long));
    if (e == cudaSuccess) e = cudaMemset(d_st, 0, sizeof(Status));
    if (e == cudaSuccess) e = cudaMemset(d_seq, 0, sizeof(uint32_t));     // position 0 never published
    int rc = PS4_ERR_CUDA;
    if (e == cudaSuccess) {
        SearchArgs a;
        memset(&a, 0, sizeof a);
        a.status = d_st;
        a.seq = d_seq;
        a.ring_mask = 0;
        a.jobs_cap = 1;
        a.n_tiles = 1;                                  // a tile still to come: the wait cannot end early
        e = (cudaError_t)launch_ring_wait_probe(a, d_out, nullptr);
        unsigned long long out[2] = {0, 0};
        Status st;
        if (e == cudaSuccess) e = cudaMemcpy(out, d_out, sizeof out, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) e = cudaMemcpy(&st, d_st, sizeof st, cudaMemcpyDeviceToHost);
        if (e == cudaSuccess) {
            if (waited_ns) *waited_ns = out[1];
            rc = (out[0] == 0 && (st.err & 0xFF) == E_TIMEOUT && (st.err >> 8) == 1) ? PS4_ERR_TIMEOUT : PS4_OK;
        }
    }
    cudaFree(d_st);
    cudaFree(d_seq);
    cudaFree(d_out);
    if (prev != device) cudaSetDevice(prev);
    return rc;
}

// ---- tuning ----

extern "C" int ps4_set_tuning(ps4_ctx *c, const ps4_tuning *t) {
    if (!c || !t) return PS4_ERR_ARG;
    if (t->log2_tile < 12 || t->log2_tile > 14 || t->gen_ctas < 1 || t->gen_ctas > 2 || t->ext_ctas < 1 ||
        t->ext_ctas > 3 || t->log2_jobs < 20 || t->log2_jobs > 29)
        return set_err(c, PS4_ERR_ARG, "tuning out of range (log2_tile 12..14, gen_ctas 1..2, ext_ctas 1..3, "
                                       "log2_jobs 20..29)");
    c->tile_log2 = t->log2_tile;
    c->gen_ctas = t->gen_ctas;
    c->ext_ctas = t->ext_ctas;
    c->jobs_cap_max = 1ull << t->log2_jobs;
    if (c->jobs_cap > c->jobs_cap_max) c->jobs_cap = c->jobs_cap_max;
    c->tuned_rate = t->rate;
    return PS4_OK;
}

extern "C" void ps4_get_tuning(const ps4_ctx *c, ps4_tuning *t) {
    if (!c || !t) return;
    t->log2_tile = c->tile_log2;
    t->gen_ctas = c->gen_ctas;
    t->ext_ctas = c->ext_ctas;
    uint32_t lj = 0;
    while ((1ull << lj) < c->jobs_cap_max) lj++;
    t->log2_jobs = lj;
    t->rate = c->tuned_rate;
}

extern "C" void ps4_last_kernel_split(const ps4_ctx *c, double *gen_ms, double *ext_ms) {
    if (gen_ms) *gen_ms = c ? c->gen_ms : 0.0;
    if (ext_ms) *ext_ms = c ? c->ext_ms : 0.0;
}

extern "C" void ps4_graph_counts(const ps4_ctx *c, uint64_t *captures, uint64_t *replays) {
    if (captures) *captures = c ? c->graph_captures : 0;
    if (replays) *replays = c ? c->graph_replays : 0;
}

// The tuner's sample: a slice of up to 8 items chosen at even quantiles of their start, each
// slice centred in its item, about 2e8 S in all -- enough for every candidate shape to fill
// the device several times over while the whole tuning stays within a few seconds.
extern "C" int ps4_autotune(ps4_ctx *c, const uint64_t *lo, const uint64_t *hi, uint32_t n_items, double budget_s,
                            ps4_tuning *best) {
    if (!c) return PS4_ERR_ARG;
    if (!lo || !hi || n_items == 0) return set_err(c, PS4_ERR_ARG, "ps4_autotune: empty workload");
    if (c->cfg.kernel != PS4_KERNEL_BATCHED) return set_err(c, PS4_ERR_ARG, "ps4_autotune tunes the batched kernels");
    if (c->pend.active) return set_err(c, PS4_ERR_ARG, "a search is enqueued on this context");
    if (budget_s <= 0) budget_s = 2.0;
    std::vector<uint32_t> idx(n_items);
    for (uint32_t i = 0; i < n_items; i++) idx[i] = i;
    std::sort(idx.begin(), idx.end(), [&](uint32_t x, uint32_t y) { return lo[x] < lo[y]; });
    const uint32_t k = std::min<uint32_t>(n_items, 8);
    const uint64_t per = (uint64_t)(2e8 / k);
    std::vector<uint64_t> slo, shi;
    for (uint32_t j = 0; j < k; j++) {
        const uint32_t i = idx[(uint64_t)j * n_items / k + (n_items / k) / 2];
        const uint64_t a = std::max<uint64_t>(lo[i], 1), b = std::max(hi[i], a);
        const uint64_t w = std::min<uint64_t>(b - a, per);
        const uint64_t s0 = a + ((b - a) - w) / 2;
        if (w) { slo.push_back(s0); shi.push_back(s0 + w); }
    }
    if (slo.empty()) return set_err(c, PS4_ERR_ARG, "ps4_autotune: workload has no S");
    uint64_t sample_S = 0;
    for (size_t j = 0; j < slo.size(); j++) sample_S += shi[j] - slo[j];
    std::vector<ps4_stats> st(slo.size());
    ps4_tuning cur;
    ps4_get_tuning(c, &cur);
    const ps4_tuning start = cur;
    ps4_tuning top = cur;
    top.rate = 0.0;
    struct timespec w0, w1;
    clock_gettime(CLOCK_MONOTONIC, &w0);
    for (uint32_t tl : {14u, 13u, 12u})
        for (uint32_t gc : {2u, 1u})
            for (uint32_t ec : {3u, 2u}) {
                clock_gettime(CLOCK_MONOTONIC, &w1);
                const double el = (double)(w1.tv_sec - w0.tv_sec) + 1e-9 * (double)(w1.tv_nsec - w0.tv_nsec);
                if (el > budget_s && top.rate > 0) break;
                ps4_tuning t = cur;
                t.log2_tile = tl; t.gen_ctas = gc; t.ext_ctas = ec; t.rate = 0;
                int rc = ps4_set_tuning(c, &t);
                double ms = 1e300;
                for (int rep = 0; rep < 2 && rc == PS4_OK; rep++) {
                    rc = begin_items(c, slo.data(), shi.data(), (uint32_t)slo.size(), false, 0);
                    if (rc == PS4_OK) rc = finish_items(c, st.data(), nullptr);
                    c->pend.active = false;
                    if (rc == PS4_OK && rep == 1) ms = c->last_ms;
                }
                if (rc != PS4_OK) {
                    ps4_set_tuning(c, &start);
                    return rc;
                }
                const double rate = (double)sample_S / (ms * 1e-3);
                if (rate > top.rate) { top = t; top.rate = rate; }
            }
    ps4_set_tuning(c, &top);
    if (best) *best = top;
    return PS4_OK;
}

// ---- triple extension ----

extern "C" int ps4_extend_triples(ps4_ctx *c, const uint64_t *abc, uint32_t n, uint64_t dmax, uint8_t *state,
                                  ps4_tri_ext *out, uint64_t out_cap, uint64_t *n_out, ps4_tri_stats *stats) {
    if (!c) return PS4_ERR_ARG;
    if (c->pend.active) return set_err(c, PS4_ERR_ARG, "a search is enqueued on this context");
    if (n_out) *n_out = 0;
    c->last_launches = 0;
    c->last_ms = 0.0;
    c->h2d_bytes = c->d2h_bytes = 0;
    if (n == 0) return PS4_OK;
    if (!abc) return set_err(c, PS4_ERR_ARG, "ps4_extend_triples: no input");
    if (dmax > (1ull << 62)) return set_err(c, PS4_ERR_ARG, "dmax %llu exceeds 2^62", (unsigned long long)dmax);
    if (grow(c, c->d_tri_in, c->tri_in_cap, 3 * (uint64_t)n)) return PS4_ERR_CUDA;
    if (grow(c, c->d_tri_state, c->tri_state_cap, n)) return PS4_ERR_CUDA;
    if (grow(c, c->d_tri_cnt, c->tri_cnt_cap, 3)) return PS4_ERR_CUDA;
    if (grow(c, c->d_tri_out, c->tri_out_cap, std::max<uint64_t>(c->tri_out_cap, std::max<uint64_t>(out_cap, 1u << 16))))
        return PS4_ERR_CUDA;
    CUDA_TRY(c, cudaMemcpyAsync(c->d_tri_in, abc, 3 * (size_t)n * sizeof(uint64_t), cudaMemcpyHostToDevice, c->stream));
    c->h2d_bytes += 3 * (uint64_t)n * sizeof(uint64_t);
    unsigned long long cnt[3];
    for (int attempt = 0; attempt < 2; attempt++) {
        CUDA_TRY(c, cudaMemsetAsync(c->d_tri_cnt, 0, 3 * sizeof(unsigned long long), c->stream));
        TriArgs t;
        t.abc = c->d_tri_in; t.n = n; t.dmax = dmax;
        t.spfq = c->d_spfq; t.ndiv = c->d_ndiv; t.tab_n = c->tab_n;
        t.state = c->d_tri_state;
        t.out = c->d_tri_out; t.out_cap = c->tri_out_cap;
        t.n_out = c->d_tri_cnt; t.n_cand = c->d_tri_cnt + 1; t.n_sqrt = c->d_tri_cnt + 2;
        t.item_base = 0;
        t.cand_per = t.sqrt_per = nullptr;
        CUDA_TRY(c, cudaEventRecord(c->ev0, c->stream));
        CUDA_TRY(c, (cudaError_t)launch_triples(t, c->stream));
        CUDA_TRY(c, cudaEventRecord(c->ev1, c->stream));
        c->last_launches++;
        CUDA_TRY(c, cudaMemcpyAsync(cnt, c->d_tri_cnt, sizeof cnt, cudaMemcpyDeviceToHost, c->stream));
        CUDA_TRY(c, cudaStreamSynchronize(c->stream));
        c->d2h_bytes += sizeof cnt;
        float ms = 0.f;
        cudaEventElapsedTime(&ms, c->ev0, c->ev1);
        c->last_ms = ms;
        if (cnt[0] <= c->tri_out_cap) break;
        // more records than the device buffer holds: grow it and run again (results do not
        // depend on the buffer)
        if (grow(c, c->d_tri_out, c->tri_out_cap, cnt[0] * 3 / 2 + 1024)) return PS4_ERR_CUDA;
    }
    std::vector<uint8_t> st(n);
    CUDA_TRY(c, cudaMemcpyAsync(st.data(), c->d_tri_state, n, cudaMemcpyDeviceToHost, c->stream));
    std::vector<ps4_tri_ext> recs(cnt[0]);
    if (cnt[0])
        CUDA_TRY(c, cudaMemcpyAsync(recs.data(), c->d_tri_out, cnt[0] * sizeof(ps4_tri_ext), cudaMemcpyDeviceToHost,
                                    c->stream));
    CUDA_TRY(c, cudaStreamSynchronize(c->stream));
    c->d2h_bytes += n + cnt[0] * sizeof(ps4_tri_ext);
    uint64_t n_invalid = 0;
    for (uint32_t i = 0; i < n; i++) {
        if (st[i] == TRI_RANGE)
            return set_err(c, PS4_ERR_ARG,
                           "triple %u (%llu, %llu, %llu) is beyond the context's factor tables (s_hi_max %llu)", i,
                           (unsigned long long)abc[3 * i], (unsigned long long)abc[3 * i + 1],
                           (unsigned long long)abc[3 * i + 2], (unsigned long long)c->cfg.s_hi_max);
        n_invalid += st[i] == TRI_INVALID;
    }
    if (state) memcpy(state, st.data(), n);
    std::sort(recs.begin(), recs.end(), [](const ps4_tri_ext &x, const ps4_tri_ext &y) {
        return x.item != y.item ? x.item < y.item : x.d < y.d;
    });
    if (n_out) *n_out = cnt[0];
    if (cnt[0] > out_cap)
        return set_err(c, PS4_ERR_OUTPUT_FULL, "triple output holds %llu records, %llu needed",
                       (unsigned long long)out_cap, cnt[0]);
    if (cnt[0]) memcpy(out, recs.data(), cnt[0] * sizeof(ps4_tri_ext));
    if (stats) {
        stats->triples += n - n_invalid;
        stats->invalid += n_invalid;
        stats->ext_cand += cnt[1];
        stats->ext_sqrt += cnt[2];
        stats->exts += cnt[0];
    }
    return PS4_OK;
}

// ---- read-only view of a context for the allocation-free entry point (ps4_kernels.cu) ----
namespace ps4 {
int ctx_view(ps4_ctx *c, CtxView *v) {
    if (!c || !c->d_spfq) return PS4_ERR_ARG;
    v->spfq = c->d_spfq; v->ndiv = c->d_ndiv; v->fac3 = c->d_fac3; v->tab_n = c->tab_n; v->s_hi_max = c->cfg.s_hi_max;
    v->cap_reps = c->cfg.cap_reps; v->cap_divs = c->cfg.cap_divs; v->cap_ext = c->cfg.cap_ext;
    v->flags = c->cfg.flags; v->device = c->cfg.device; v->num_sms = c->num_sms; v->stream = c->stream;
    return PS4_OK;
}
int ctx_fail(ps4_ctx *c, int code, const char *msg) { return set_err(c, code, "%s", msg); }
}  // namespace ps4
