// ps4_serve.cu -- the serving loop behind ps4_serve_* (include/ps4.h): continuous batching of
// subrange queries and triple-extension queries on one device.
//
// The reference serves its search by launching one s4 process per block from a Python
// controller (run_exhaustive.py:200-238) and parsing each process's stdout; nothing of that
// loop is kept.  Here:
//
//  * a query is admitted when a device slot is free and the per-query arena (a fixed part of
//    the server's device-memory budget, allocated once) can hold its counters and result
//    buffers; admission is FIFO.
//  * a step is one launch of the search kernels (tile kernel + extension engine) over chunks
//    of the admitted subranges -- the oldest query first, then shortest remaining first,
//    within a budget of S values and job-queue entries -- plus one triple-extension launch,
//    on a second stream, over every admitted triple query.  Queries admitted while a step
//    runs join the next one.  Two step buffer sets alternate, so one step is always queued
//    behind the running one.
//  * after a step, small kernels on a third stream fold its per-chunk counters into the
//    queries' slot counters and append its records to their slot buffers; a query whose last
//    work has been folded is copied to the host once, its slot and arena space freed.
//  * internal capacity events (job queue, engine list, tile lists, step result buffers) re-run
//    the step with adjusted sizes before anything is folded, so results never depend on them.
//    A query whose slot buffers overflow is re-admitted with larger ones and run again.

#include <cuda_runtime.h>
#include <time.h>

#include <algorithm>
#include <cmath>
#include <cstdarg>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <string>
#include <unordered_map>
#include <vector>

#include "ps4_internal.h"

using namespace ps4;

namespace {

typedef unsigned long long ull;

// ---------------------------------------------------------------- device side

// One query's device-resident state: counters as the single-query calls keep them per item
// (K_* slots), triple counters, and its result buffers in the arena.
struct SlotDev {
    ull k[K_SLOTS];
    ull tri_cand, tri_sqrt;
    unsigned n_hits, n_exts, n_sixes, n_tri;
    unsigned cap_hits, cap_exts, cap_sixes, cap_tri;
    ps4_hit *hits;
    ps4_ext *exts;
    ps4_six *sixes;
    ps4_tri_ext *tri;
};

__global__ void k_init_slot(SlotDev *slots, uint32_t s, uint32_t ch, uint32_t ce, uint32_t cs, uint32_t ct,
                            ps4_hit *h, ps4_ext *e, ps4_six *x, ps4_tri_ext *t) {
    SlotDev &d = slots[s];
    for (int j = threadIdx.x; j < K_SLOTS; j += blockDim.x) d.k[j] = 0;
    if (threadIdx.x == 0) {
        d.tri_cand = d.tri_sqrt = 0;
        d.n_hits = d.n_exts = d.n_sixes = d.n_tri = 0;
        d.cap_hits = ch; d.cap_exts = ce; d.cap_sixes = cs; d.cap_tri = ct;
        d.hits = h; d.exts = e; d.sixes = x; d.tri = t;
    }
}

// block i, thread j: counter j of chunk i into its query's slot (maxima by max, the rest by add)
__global__ void k_merge_counters(SlotDev *slots, const uint32_t *item_slot, const ull *k) {
    const uint32_t i = blockIdx.x;
    const int j = threadIdx.x;
    const ull v = k[(size_t)i * K_SLOTS + j];
    if (v == 0) return;
    ull *dst = &slots[item_slot[i]].k[j];
    if (j >= K_MAX_REPS && j <= K_MAX_EXT) atomicMax(dst, v);
    else atomicAdd(dst, v);
}

__global__ void k_scatter_hits(SlotDev *slots, const uint32_t *item_slot, const ps4_hit *hits, const ps4_ext *exts,
                               uint32_t n, uint32_t *remap) {
    for (uint32_t h = blockIdx.x * blockDim.x + threadIdx.x; h < n; h += gridDim.x * blockDim.x) {
        ps4_hit x = hits[h];
        SlotDev &d = slots[item_slot[x.item]];
        const unsigned pos = atomicAdd(&d.n_hits, 1u), epos = atomicAdd(&d.n_exts, x.n_ext);
        remap[h] = pos;
        if (pos < d.cap_hits && (uint64_t)epos + x.n_ext <= d.cap_exts) {
            for (uint32_t t = 0; t < x.n_ext; t++) d.exts[epos + t] = exts[x.first_ext + t];
            x.first_ext = epos;
            x.item = 0;
            d.hits[pos] = x;
        }
    }
}

__global__ void k_scatter_sixes(SlotDev *slots, const uint32_t *item_slot, const ps4_hit *hits, const ps4_six *six,
                                uint32_t n, const uint32_t *remap) {
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        ps4_six x = six[i];
        SlotDev &d = slots[item_slot[hits[x.hit].item]];
        const unsigned pos = atomicAdd(&d.n_sixes, 1u);
        if (pos < d.cap_sixes) {
            x.hit = remap[x.hit];
            d.sixes[pos] = x;
        }
    }
}

__global__ void k_scatter_tri(SlotDev *slots, const uint32_t *tri_slot, const ps4_tri_ext *out, uint32_t n_out,
                              const ull *cand_per, const ull *sqrt_per, uint32_t n_tri) {
    const uint32_t n = n_out > n_tri ? n_out : n_tri;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        if (i < n_out) {
            ps4_tri_ext x = out[i];
            SlotDev &d = slots[tri_slot[x.item]];
            const unsigned pos = atomicAdd(&d.n_tri, 1u);
            if (pos < d.cap_tri) {
                x.item = 0;
                d.tri[pos] = x;
            }
        }
        if (i < n_tri) {
            SlotDev &d = slots[tri_slot[i]];
            if (cand_per[i]) atomicAdd(&d.tri_cand, cand_per[i]);
            if (sqrt_per[i]) atomicAdd(&d.tri_sqrt, sqrt_per[i]);
        }
    }
}

// ---------------------------------------------------------------- host side

double now_s() {
    timespec ts;
    clock_gettime(CLOCK_MONOTONIC, &ts);
    return (double)ts.tv_sec + 1e-9 * (double)ts.tv_nsec;
}

struct Range {
    uint64_t lo, hi;
};

struct Query {
    uint64_t tag = 0;
    uint32_t kind = PS4_Q_RANGE;
    uint64_t lo = 0, hi = 0;
    uint64_t abc[3] = {0, 0, 0};
    uint64_t dmax = 0;
    uint64_t seq = 0;                  // admission order
    std::deque<Range> pending;         // S ranges not yet in a successful step
    bool tri_pending = false;
    int slot = -1;
    uint64_t arena_off = 0, arena_bytes = 0;
    uint32_t cap_hits = 0, cap_exts = 0, cap_sixes = 0, cap_tri = 0;
    uint32_t inflight = 0;             // steps in flight carrying its work
    uint32_t steps = 0, reruns = 0;
    bool failed = false, finished = false;
    int status = PS4_OK;
    std::string msg;
    double t_submit = 0, t_admit = 0, t_done = 0;
    uint8_t tri_state = 0;
    // results on the host once finished
    ps4_stats stats;
    ps4_tri_stats tstats;
    std::vector<ps4_hit> hits;
    std::vector<ps4_ext> exts;
    std::vector<ps4_six> sixes;
    std::vector<ps4_tri_ext> tri;
};

// First-fit allocator over the arena (offsets in bytes, 256-byte granules), coalescing on free.
struct Arena {
    uint64_t size = 0, used = 0, peak = 0;
    std::map<uint64_t, uint64_t> free_;
    void reset(uint64_t n) {
        size = n; used = peak = 0;
        free_.clear();
        if (n) free_[0] = n;
    }
    static uint64_t round(uint64_t n) { return (n + 255) & ~255ull; }
    bool alloc(uint64_t n, uint64_t &off) {
        n = round(n);
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            off = it->first;
            const uint64_t rest = it->second - n;
            free_.erase(it);
            if (rest) free_[off + n] = rest;
            used += n;
            peak = std::max(peak, used);
            return true;
        }
        return false;
    }
    void release(uint64_t off, uint64_t n) {
        n = round(n);
        used -= n;
        auto it = free_.emplace(off, n).first;
        auto nx = std::next(it);
        if (nx != free_.end() && it->first + it->second == nx->first) {
            it->second += nx->second;
            free_.erase(nx);
        }
        if (it != free_.begin()) {
            auto pv = std::prev(it);
            if (pv->first + pv->second == it->first) {
                pv->second += it->second;
                free_.erase(it);
            }
        }
    }
};

struct Chunk {
    uint32_t q;
    uint64_t lo, hi;
};

enum { BUF_FREE = 0, BUF_KERNELS = 1, BUF_POST = 2 };

struct StepBuf {
    int state = BUF_FREE;
    bool fused = false;
    unsigned tile_log2 = 13;
    std::vector<Chunk> chunks;
    std::vector<uint32_t> tris;           // triple queries of the step
    std::vector<uint32_t> queries;        // distinct queries of the step
    std::vector<uint32_t> completing;     // queries to finish once the step's folding is done
    // device
    Item *d_items = nullptr;
    uint32_t *d_item_slot = nullptr;
    ull *d_counters = nullptr;
    Status *d_status = nullptr;
    ps4_hit *d_hits = nullptr; uint64_t hits_cap = 0;
    ps4_ext *d_exts = nullptr; uint64_t exts_cap = 0;
    ps4_six *d_sixes = nullptr; uint64_t sixes_cap = 0;
    uint32_t *d_remap = nullptr; uint64_t remap_cap = 0;
    uint64_t *d_abc = nullptr;
    uint32_t *d_tri_slot = nullptr;
    uint8_t *d_tri_state = nullptr;
    ps4_tri_ext *d_tri_out = nullptr; uint64_t tri_out_cap = 0;
    ull *d_tri_cnt = nullptr;             // n_out, n_cand, n_sqrt
    ull *d_cand_per = nullptr, *d_sqrt_per = nullptr;
    // pinned host staging
    Item *h_items = nullptr;
    uint32_t *h_item_slot = nullptr;
    uint64_t *h_abc = nullptr;
    uint32_t *h_tri_slot = nullptr;
    uint8_t *h_tri_state = nullptr;
    Status *h_status = nullptr;
    ull *h_tri_cnt = nullptr;
    cudaEvent_t ev_start = nullptr, ev_kern = nullptr, ev_post = nullptr, ev_fork = nullptr, ev_join = nullptr;
};

const uint32_t RANGE_SIXES = 16;
const uint32_t TRI_RECS = 64;

}  // namespace

struct ps4_server {
    ps4_ctx *ctx = nullptr;
    CtxView v;
    ps4_serve_config cfg;
    cudaStream_t s_main = nullptr, s_tri = nullptr, s_post = nullptr, s_copy = nullptr;
    uint32_t *d_jobs = nullptr;
    uint64_t jobs_cap = 0;
    uint64_t *d_raw = nullptr;               // per tile-kernel CTA representation lists
    uint32_t *d_scratch = nullptr;
    uint64_t scratch_words = 0;
    SlotDev *d_slots = nullptr;
    unsigned char *d_arena = nullptr;
    Arena arena;
    StepBuf buf[2];
    int next_buf = 0;
    std::vector<std::unique_ptr<Query>> qs;
    std::vector<uint32_t> free_ids;
    std::unordered_map<uint64_t, uint32_t> by_tag;
    std::deque<uint32_t> waiting;
    std::vector<uint32_t> active;
    std::vector<int> free_slots;
    std::deque<uint32_t> unreported;
    unsigned tile_log2 = 13;
    uint32_t batch_div = 1;
    bool fused_next = false;
    uint64_t seq = 0;
    uint64_t n_submitted = 0, n_finished = 0, n_steps = 0, n_step_reruns = 0;
    uint64_t device_bytes = 0;
    double gpu_ms = 0;
    std::string err;
};

namespace {

int srv_err(ps4_server *s, int code, const char *fmt, ...) {
    char b[512];
    va_list ap;
    va_start(ap, fmt);
    vsnprintf(b, sizeof b, fmt, ap);
    va_end(ap);
    if (s) s->err = b;
    return code;
}

#define SRV_CUDA(s, call)                                                                               \
    do {                                                                                                \
        cudaError_t _e = (call);                                                                        \
        if (_e != cudaSuccess) return srv_err(s, PS4_ERR_CUDA, "%s failed: %s", #call, cudaGetErrorString(_e)); \
    } while (0)

template <class T>
int dev_alloc(ps4_server *s, T *&p, uint64_t n) {
    if (p) { cudaFree(p); p = nullptr; }
    if (n == 0) return PS4_OK;
    SRV_CUDA(s, cudaMalloc((void **)&p, n * sizeof(T)));
    s->device_bytes += n * sizeof(T);
    return PS4_OK;
}

template <class T>
int host_alloc(ps4_server *s, T *&p, uint64_t n) {
    SRV_CUDA(s, cudaMallocHost((void **)&p, std::max<uint64_t>(n, 1) * sizeof(T)));
    return PS4_OK;
}

template <class T>
int grow_dev(ps4_server *s, T *&p, uint64_t &cap, uint64_t need) {
    if (need <= cap && p) return PS4_OK;
    if (p) s->device_bytes -= cap * sizeof(T);
    cap = 0;
    if (dev_alloc(s, p, need)) return PS4_ERR_CUDA;
    cap = need;
    return PS4_OK;
}

Query &Q(ps4_server *s, uint32_t id) { return *s->qs[id]; }

// Result-buffer quota of a subrange query: 4-sets with an extension run below 1.5e-5 per S on
// every checked range (5.4e-6 over [1,1e10), 7e-7 near 2e12); 4e-5 per S plus a floor covers
// them with margin.  An overflow re-runs the query with larger buffers.
void range_quota(ps4_server *s, Query &q, uint64_t min_hits, uint64_t min_exts, uint64_t min_sixes) {
    const uint64_t w = q.hi - q.lo;
    uint64_t h = s->cfg.hits_floor + (uint64_t)std::ceil(1e-6 * s->cfg.hits_per_1e6_S * (double)w);
    h = std::max(h, min_hits);
    uint64_t e = std::max<uint64_t>(2 * h, min_exts);
    const uint64_t cap_limit = s->arena.size / 4 / (sizeof(ps4_hit) + 2 * sizeof(ps4_ext));
    h = std::min(h, std::max(cap_limit, min_hits));
    e = std::min(e, std::max(2 * cap_limit, min_exts));
    h = std::max<uint64_t>(h, 1);
    e = std::max<uint64_t>(e, 2);
    q.cap_hits = (uint32_t)std::min<uint64_t>(h, 0xFFFFFFF0u);
    q.cap_exts = (uint32_t)std::min<uint64_t>(e, 0xFFFFFFF0u);
    q.cap_sixes = (uint32_t)std::max<uint64_t>(RANGE_SIXES, min_sixes);
    q.cap_tri = 0;
}

uint64_t quota_bytes(const Query &q) {
    return Arena::round((uint64_t)q.cap_hits * sizeof(ps4_hit)) + Arena::round((uint64_t)q.cap_exts * sizeof(ps4_ext)) +
           Arena::round((uint64_t)q.cap_sixes * sizeof(ps4_six)) + Arena::round((uint64_t)q.cap_tri * sizeof(ps4_tri_ext));
}

void finish_query(ps4_server *s, uint32_t id, double t) {
    Query &q = Q(s, id);
    q.finished = true;
    q.t_done = t;
    if (q.slot >= 0) {
        s->free_slots.push_back(q.slot);
        q.slot = -1;
    }
    if (q.arena_bytes) {
        s->arena.release(q.arena_off, q.arena_bytes);
        q.arena_bytes = 0;
    }
    s->active.erase(std::remove(s->active.begin(), s->active.end(), id), s->active.end());
    s->unreported.push_back(id);
    s->n_finished++;
}

void fail_query(ps4_server *s, uint32_t id, int code, const std::string &msg) {
    Query &q = Q(s, id);
    if (q.failed) return;
    q.failed = true;
    q.status = code;
    q.msg = msg;
    q.pending.clear();
    q.tri_pending = false;
}

// Admit waiting queries in FIFO order while a slot and arena room are free.
int admit(ps4_server *s) {
    while (!s->waiting.empty()) {
        const uint32_t id = s->waiting.front();
        Query &q = Q(s, id);
        const bool empty = q.kind == PS4_Q_RANGE && q.lo >= q.hi;
        if (empty) {                                          // nothing to search: zero counters
            s->waiting.pop_front();
            q.t_admit = now_s();
            memset(&q.stats, 0, sizeof q.stats);
            s->active.push_back(id);
            finish_query(s, id, q.t_admit);
            continue;
        }
        const uint64_t bytes = quota_bytes(q);
        if (bytes > s->arena.size) {
            s->waiting.pop_front();
            q.t_admit = now_s();
            s->active.push_back(id);
            fail_query(s, id, PS4_ERR_OUTPUT_FULL, "results of this query exceed the server's arena; search it alone");
            finish_query(s, id, q.t_admit);
            continue;
        }
        if (s->free_slots.empty()) break;
        uint64_t off = 0;
        if (!s->arena.alloc(bytes, off)) break;
        s->waiting.pop_front();
        q.slot = s->free_slots.back();
        s->free_slots.pop_back();
        q.arena_off = off;
        q.arena_bytes = bytes;
        q.seq = s->seq++;
        q.t_admit = now_s();
        unsigned char *base = s->d_arena + off;
        ps4_hit *h = (ps4_hit *)base;
        base += Arena::round((uint64_t)q.cap_hits * sizeof(ps4_hit));
        ps4_ext *e = (ps4_ext *)base;
        base += Arena::round((uint64_t)q.cap_exts * sizeof(ps4_ext));
        ps4_six *x = (ps4_six *)base;
        base += Arena::round((uint64_t)q.cap_sixes * sizeof(ps4_six));
        ps4_tri_ext *t = (ps4_tri_ext *)base;
        k_init_slot<<<1, 128, 0, s->s_main>>>(s->d_slots, (uint32_t)q.slot, q.cap_hits, q.cap_exts, q.cap_sixes,
                                              q.cap_tri, h, e, x, t);
        SRV_CUDA(s, cudaGetLastError());
        if (q.kind == PS4_Q_RANGE) {
            q.pending.clear();
            q.pending.push_back(Range{q.lo, q.hi});
        } else {
            q.tri_pending = true;
        }
        s->active.push_back(id);
    }
    return PS4_OK;
}

bool has_work(ps4_server *s) {
    for (uint32_t id : s->active) {
        const Query &q = Q(s, id);
        if (!q.failed && (!q.pending.empty() || q.tri_pending)) return true;
    }
    return false;
}

// Choose the step's chunks and triples.
void plan_step(ps4_server *s, StepBuf &b) {
    b.chunks.clear();
    b.tris.clear();
    b.queries.clear();
    b.completing.clear();
    b.tile_log2 = s->tile_log2;
    b.fused = s->fused_next;
    s->fused_next = false;
    std::vector<uint32_t> cand;
    for (uint32_t id : s->active) {
        const Query &q = Q(s, id);
        if (q.kind == PS4_Q_RANGE && !q.failed && !q.pending.empty()) cand.push_back(id);
    }
    if (!cand.empty()) {
        auto oldest = std::min_element(cand.begin(), cand.end(),
                                       [&](uint32_t a, uint32_t c) { return Q(s, a).seq < Q(s, c).seq; });
        std::iter_swap(cand.begin(), oldest);
        auto remaining = [&](uint32_t id) {
            uint64_t r = 0;
            for (const Range &x : Q(s, id).pending) r += x.hi - x.lo;
            return r;
        };
        std::vector<std::pair<uint64_t, uint32_t>> rest;
        for (size_t i = 1; i < cand.size(); i++) rest.push_back({remaining(cand[i]), cand[i]});
        std::sort(rest.begin(), rest.end());
        for (size_t i = 1; i < cand.size(); i++) cand[i] = rest[i - 1].second;
    }
    const uint64_t tile = 1ull << b.tile_log2;
    double jobs_left = 0.9 * (double)s->jobs_cap / (double)s->batch_div;
    uint64_t S_left = std::max<uint64_t>(s->cfg.step_S / s->batch_div, tile);
    for (uint32_t id : cand) {
        Query &q = Q(s, id);
        bool used = false;
        while (!q.pending.empty() && S_left > 0 && jobs_left > 0 && b.chunks.size() < s->cfg.max_step_items) {
            Range &r = q.pending.front();
            const double dens = jobs_per_S_bound(r.hi);
            uint64_t take = std::min<uint64_t>(r.hi - r.lo, S_left);
            take = std::min<uint64_t>(take, (uint64_t)(jobs_left / dens));
            if (take == 0) break;
            b.chunks.push_back(Chunk{id, r.lo, r.lo + take});
            r.lo += take;
            if (r.lo == r.hi) q.pending.pop_front();
            S_left -= std::min<uint64_t>(S_left, std::max<uint64_t>(take, tile));
            jobs_left -= dens * (double)take;
            used = true;
        }
        if (used) b.queries.push_back(id);
        if (S_left == 0 || jobs_left <= 0 || b.chunks.size() >= s->cfg.max_step_items) break;
    }
    for (uint32_t id : s->active) {
        Query &q = Q(s, id);
        if (b.tris.size() >= s->cfg.max_step_triples) break;
        if (q.kind == PS4_Q_TRIPLE && !q.failed && q.tri_pending) {
            q.tri_pending = false;
            b.tris.push_back(id);
            b.queries.push_back(id);
        }
    }
    for (uint32_t id : b.queries) {
        Q(s, id).inflight++;
        Q(s, id).steps++;
    }
}

int launch_step(ps4_server *s, StepBuf &b) {
    const uint32_t n_items = (uint32_t)b.chunks.size(), n_tri = (uint32_t)b.tris.size();
    const unsigned TL = b.tile_log2;
    uint64_t tiles = 0;
    for (uint32_t i = 0; i < n_items; i++) {
        const Chunk &c = b.chunks[i];
        Item it;
        it.lo = c.lo; it.hi = c.hi; it.tile_base = tiles; it.id = i; it.pad = 0;
        tiles += (c.hi - c.lo + (1ull << TL) - 1) >> TL;
        b.h_items[i] = it;
        b.h_item_slot[i] = (uint32_t)Q(s, c.q).slot;
    }
    for (uint32_t i = 0; i < n_tri; i++) {
        const Query &q = Q(s, b.tris[i]);
        b.h_abc[3 * i] = q.abc[0]; b.h_abc[3 * i + 1] = q.abc[1]; b.h_abc[3 * i + 2] = q.abc[2];
        b.h_tri_slot[i] = (uint32_t)q.slot;
    }
    cudaStream_t st = s->s_main;
    if (n_items) {
        SRV_CUDA(s, cudaMemcpyAsync(b.d_items, b.h_items, n_items * sizeof(Item), cudaMemcpyHostToDevice, st));
        SRV_CUDA(s, cudaMemcpyAsync(b.d_item_slot, b.h_item_slot, n_items * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
        SRV_CUDA(s, cudaMemsetAsync(b.d_counters, 0, (size_t)n_items * K_SLOTS * sizeof(ull), st));
    }
    if (n_tri) {
        SRV_CUDA(s, cudaMemcpyAsync(b.d_abc, b.h_abc, 3 * (size_t)n_tri * sizeof(uint64_t), cudaMemcpyHostToDevice, st));
        SRV_CUDA(s, cudaMemcpyAsync(b.d_tri_slot, b.h_tri_slot, n_tri * sizeof(uint32_t), cudaMemcpyHostToDevice, st));
    }
    SRV_CUDA(s, cudaMemsetAsync(b.d_status, 0, sizeof(Status), st));
    SRV_CUDA(s, cudaMemsetAsync(b.d_tri_cnt, 0, 3 * sizeof(ull), st));
    SRV_CUDA(s, cudaEventRecord(b.ev_start, st));
    if (n_tri) {                          // the triple kernel runs beside the search kernels
        SRV_CUDA(s, cudaEventRecord(b.ev_fork, st));
        SRV_CUDA(s, cudaStreamWaitEvent(s->s_tri, b.ev_fork, 0));
        TriArgs t;
        memset(&t, 0, sizeof t);
        t.abc = b.d_abc; t.n = n_tri; t.dmax = 0;
        t.spfq = s->v.spfq; t.ndiv = s->v.ndiv; t.tab_n = s->v.tab_n;
        t.state = b.d_tri_state;
        t.out = b.d_tri_out; t.out_cap = b.tri_out_cap;
        t.n_out = b.d_tri_cnt; t.n_cand = b.d_tri_cnt + 1; t.n_sqrt = b.d_tri_cnt + 2;
        t.item_base = 0;
        t.cand_per = b.d_cand_per; t.sqrt_per = b.d_sqrt_per;
        // one dmax per launch: runs of equal bound (the serving stream uses one)
        uint32_t i0 = 0;
        while (i0 < n_tri) {
            const uint64_t dm = Q(s, b.tris[i0]).dmax;
            uint32_t i1 = i0 + 1;
            while (i1 < n_tri && Q(s, b.tris[i1]).dmax == dm) i1++;
            TriArgs u = t;
            u.abc = b.d_abc + 3 * (uint64_t)i0;
            u.n = i1 - i0;
            u.dmax = dm;
            u.state = b.d_tri_state + i0;
            u.item_base = i0;
            u.cand_per = b.d_cand_per + i0;
            u.sqrt_per = b.d_sqrt_per + i0;
            SRV_CUDA(s, (cudaError_t)launch_triples(u, s->s_tri));
            i0 = i1;
        }
        SRV_CUDA(s, cudaEventRecord(b.ev_join, s->s_tri));
    }
    if (n_items) {
        SearchArgs a;
        memset(&a, 0, sizeof a);
        a.items = b.d_items; a.n_items = n_items; a.n_tiles = tiles; a.log2_tile = TL;
        a.spfq = s->v.spfq; a.ndiv = s->v.ndiv; a.fac3 = s->v.fac3; a.tab_n = s->v.tab_n;
        a.counters = b.d_counters;
        a.hits = b.d_hits; a.hits_cap = (uint32_t)b.hits_cap;
        a.exts = b.d_exts; a.exts_cap = (uint32_t)b.exts_cap;
        a.sixes = b.d_sixes; a.sixes_cap = (uint32_t)b.sixes_cap;
        a.status = b.d_status;
        a.cap_reps = s->v.cap_reps; a.cap_divs = s->v.cap_divs; a.cap_ext = s->v.cap_ext;
        a.flags = s->v.flags & ~(uint32_t)PS4_F_DUMP4;
        a.jobs = s->d_jobs; a.jobs_cap = s->jobs_cap;
        if (!b.fused) {
            a.raw = s->d_raw; a.raw_cap = raw_cap_for(TL);
            const int g = (int)std::min<uint64_t>((uint64_t)gen_grid(s->v.num_sms, TL), std::max<uint64_t>(tiles, 1));
            SRV_CUDA(s, (cudaError_t)launch_gen(a, g, st));
            if (!(s->v.flags & PS4_F_NOEXT)) SRV_CUDA(s, (cudaError_t)launch_ext(a, ext_grid(s->v.num_sms), st));
        } else {
            const uint32_t stage_cap = stage_cap_for(TL, s->v.cap_reps);
            const int grid = (int)std::min<uint64_t>((uint64_t)s->v.num_sms, std::max<uint64_t>(tiles, 1));
            if (grow_dev(s, s->d_scratch, s->scratch_words, (uint64_t)grid * 6 * stage_cap)) return PS4_ERR_CUDA;
            a.scratch = s->d_scratch; a.stage_cap = stage_cap;
            SRV_CUDA(s, (cudaError_t)launch_search(a, PS4_KERNEL_BATCHED, grid, st));
        }
    }
    if (n_tri) SRV_CUDA(s, cudaStreamWaitEvent(st, b.ev_join, 0));
    SRV_CUDA(s, cudaEventRecord(b.ev_kern, st));
    SRV_CUDA(s, cudaMemcpyAsync(b.h_status, b.d_status, sizeof(Status), cudaMemcpyDeviceToHost, st));
    SRV_CUDA(s, cudaMemcpyAsync(b.h_tri_cnt, b.d_tri_cnt, 3 * sizeof(ull), cudaMemcpyDeviceToHost, st));
    if (n_tri) SRV_CUDA(s, cudaMemcpyAsync(b.h_tri_state, b.d_tri_state, n_tri, cudaMemcpyDeviceToHost, st));
    // the host reads the copies once ev_post (recorded behind them) has completed
    SRV_CUDA(s, cudaEventRecord(b.ev_post, st));
    b.state = BUF_KERNELS;
    s->n_steps++;
    return PS4_OK;
}

// Return a step's work to its queries (nothing of it was folded).
void requeue(ps4_server *s, StepBuf &b) {
    for (size_t i = b.chunks.size(); i-- > 0;) {
        Query &q = Q(s, b.chunks[i].q);
        if (q.failed) continue;
        // merge with the front range when adjacent, otherwise put back in front
        if (!q.pending.empty() && q.pending.front().lo == b.chunks[i].hi) q.pending.front().lo = b.chunks[i].lo;
        else q.pending.push_front(Range{b.chunks[i].lo, b.chunks[i].hi});
    }
    for (uint32_t id : b.tris)
        if (!Q(s, id).failed) Q(s, id).tri_pending = true;
}

// The step's kernels and status copies are done: check it, then fold it (post stream) or re-run it.
int check_step(ps4_server *s, StepBuf &b) {
    const Status &st = *b.h_status;
    float ms = 0.f;
    if (cudaEventElapsedTime(&ms, b.ev_start, b.ev_kern) == cudaSuccess) s->gpu_ms += ms;
    const unsigned code = (unsigned)(st.err & 0xFF);
    const unsigned long long errS = st.err >> 8;
    bool rerun = false;
    auto chunk_of = [&](uint64_t S) -> int {
        for (size_t i = 0; i < b.chunks.size(); i++)
            if (b.chunks[i].lo <= S && S < b.chunks[i].hi) return (int)i;
        return -1;
    };
    if (code == E_QUEUE) {
        if (s->batch_div < (1u << 16)) s->batch_div *= 2;
        rerun = true;
    } else if (code == E_EXTLIST && !b.fused) {
        s->fused_next = true;
        rerun = true;
    } else if (code == E_TILE || code == E_EXTLIST) {
        if (s->tile_log2 > 12) {
            s->tile_log2--;
            s->fused_next = b.fused;
        } else {
            const int c = chunk_of(errS);
            char m[256];
            snprintf(m, sizeof m, "FATAL: tile capacity exceeded near S=%llu; this interval is NOT certified complete",
                     errS);
            if (c >= 0) fail_query(s, b.chunks[c].q, PS4_ERR_CAP_REPS, m);
            else return srv_err(s, PS4_ERR_CUDA, "%s", m);
        }
        rerun = true;
    } else if (code != 0) {
        const int c = chunk_of(errS);
        char m[256];
        if (code == E_VERIFY)
            snprintf(m, sizeof m, "BAD 4-set S=%llu [%lld,%lld,%lld,%lld]", st.verify_bad[0], (long long)st.verify_bad[1],
                     (long long)st.verify_bad[2], (long long)st.verify_bad[3], (long long)st.verify_bad[4]);
        else
            snprintf(m, sizeof m, "FATAL: %s; this interval is NOT certified complete", fatal_text(code));
        if (c < 0) return srv_err(s, PS4_ERR_CUDA, "step error outside its chunks: %s", m);
        fail_query(s, b.chunks[c].q, (int)code, m);
        rerun = true;
    }
    if (!rerun) {
        if (st.n_hits > b.hits_cap || st.n_exts > b.exts_cap || st.n_sixes > b.sixes_cap ||
            b.h_tri_cnt[0] > b.tri_out_cap) {
            if (st.n_hits > b.hits_cap && grow_dev(s, b.d_hits, b.hits_cap, (uint64_t)st.n_hits * 3 / 2 + 1024))
                return PS4_ERR_CUDA;
            if (st.n_hits > b.remap_cap && grow_dev(s, b.d_remap, b.remap_cap, b.hits_cap)) return PS4_ERR_CUDA;
            if (st.n_exts > b.exts_cap && grow_dev(s, b.d_exts, b.exts_cap, (uint64_t)st.n_exts * 3 / 2 + 1024))
                return PS4_ERR_CUDA;
            if (st.n_sixes > b.sixes_cap && grow_dev(s, b.d_sixes, b.sixes_cap, (uint64_t)st.n_sixes * 3 / 2 + 64))
                return PS4_ERR_CUDA;
            if (b.h_tri_cnt[0] > b.tri_out_cap &&
                grow_dev(s, b.d_tri_out, b.tri_out_cap, (uint64_t)b.h_tri_cnt[0] * 3 / 2 + 1024))
                return PS4_ERR_CUDA;
            rerun = true;
        }
    }
    if (!rerun) {
        for (size_t i = 0; i < b.tris.size(); i++) {
            Query &q = Q(s, b.tris[i]);
            q.tri_state = b.h_tri_state[i];
            if (q.tri_state == TRI_RANGE) {
                char m[256];
                snprintf(m, sizeof m, "triple 0 (%llu, %llu, %llu) is beyond the context's factor tables (s_hi_max %llu)",
                         (unsigned long long)q.abc[0], (unsigned long long)q.abc[1], (unsigned long long)q.abc[2],
                         (unsigned long long)s->v.s_hi_max);
                fail_query(s, b.tris[i], PS4_ERR_ARG, m);
            }
        }
        // fold the step into the slots on the post stream, beside the next step's kernels
        cudaStream_t ps = s->s_post;
        SRV_CUDA(s, cudaStreamWaitEvent(ps, b.ev_kern, 0));
        const uint32_t n_items = (uint32_t)b.chunks.size(), n_tri = (uint32_t)b.tris.size();
        if (n_items) {
            k_merge_counters<<<n_items, K_SLOTS, 0, ps>>>(s->d_slots, b.d_item_slot, b.d_counters);
            SRV_CUDA(s, cudaGetLastError());
        }
        if (st.n_hits) {
            const uint32_t g = std::min<uint32_t>((st.n_hits + 255) / 256, 1024);
            k_scatter_hits<<<g, 256, 0, ps>>>(s->d_slots, b.d_item_slot, b.d_hits, b.d_exts, st.n_hits, b.d_remap);
            SRV_CUDA(s, cudaGetLastError());
        }
        if (st.n_sixes) {
            k_scatter_sixes<<<1, 64, 0, ps>>>(s->d_slots, b.d_item_slot, b.d_hits, b.d_sixes, st.n_sixes, b.d_remap);
            SRV_CUDA(s, cudaGetLastError());
        }
        if (n_tri) {
            const uint32_t n = std::max<uint32_t>((uint32_t)b.h_tri_cnt[0], n_tri);
            const uint32_t g = std::min<uint32_t>((n + 255) / 256, 1024);
            k_scatter_tri<<<g, 256, 0, ps>>>(s->d_slots, b.d_tri_slot, b.d_tri_out, (uint32_t)b.h_tri_cnt[0],
                                             b.d_cand_per, b.d_sqrt_per, n_tri);
            SRV_CUDA(s, cudaGetLastError());
        }
    } else {
        requeue(s, b);
        s->n_step_reruns++;
        SRV_CUDA(s, cudaStreamWaitEvent(s->s_post, b.ev_kern, 0));
    }
    for (uint32_t id : b.queries) {
        Query &q = Q(s, id);
        q.inflight--;
        if (q.inflight == 0 && (q.failed || (q.pending.empty() && !q.tri_pending))) b.completing.push_back(id);
    }
    // queries finish once this and every earlier fold on the post stream is done
    SRV_CUDA(s, cudaEventRecord(b.ev_post, s->s_post));
    b.state = BUF_POST;
    return PS4_OK;
}

// The step's folding is done: copy finished queries to the host, free their slots.
int complete_step(ps4_server *s, StepBuf &b) {
    const double t = now_s();
    std::vector<uint32_t> ok;
    for (uint32_t id : b.completing) {
        Query &q = Q(s, id);
        if (q.failed) finish_query(s, id, t);
        else ok.push_back(id);
    }
    b.completing.clear();
    b.state = BUF_FREE;
    if (ok.empty()) return PS4_OK;
    std::vector<SlotDev> hdr(ok.size());
    for (size_t i = 0; i < ok.size(); i++)
        SRV_CUDA(s, cudaMemcpyAsync(&hdr[i], s->d_slots + Q(s, ok[i]).slot, sizeof(SlotDev), cudaMemcpyDeviceToHost,
                                    s->s_copy));
    SRV_CUDA(s, cudaStreamSynchronize(s->s_copy));
    std::vector<uint32_t> fetch;
    for (size_t i = 0; i < ok.size(); i++) {
        Query &q = Q(s, ok[i]);
        const SlotDev &h = hdr[i];
        if (h.n_hits > h.cap_hits || h.n_exts > h.cap_exts || h.n_sixes > h.cap_sixes || h.n_tri > h.cap_tri) {
            // the query's slot buffers overflowed: re-admit it first in line with larger ones
            const uint32_t id = ok[i];
            s->free_slots.push_back(q.slot);
            q.slot = -1;
            s->arena.release(q.arena_off, q.arena_bytes);
            q.arena_bytes = 0;
            s->active.erase(std::remove(s->active.begin(), s->active.end(), id), s->active.end());
            if (q.kind == PS4_Q_RANGE) range_quota(s, q, (uint64_t)h.n_hits * 3 / 2 + 64, (uint64_t)h.n_exts * 3 / 2 + 128,
                                                   (uint64_t)h.n_sixes * 2 + 16);
            else q.cap_tri = std::max<uint32_t>(q.cap_tri, h.n_tri * 2);
            q.reruns++;
            s->waiting.push_front(id);
            continue;
        }
        q.hits.resize(h.n_hits);
        q.exts.resize(h.n_exts);
        q.sixes.resize(h.n_sixes);
        q.tri.resize(h.n_tri);
        if (h.n_hits)
            SRV_CUDA(s, cudaMemcpyAsync(q.hits.data(), h.hits, h.n_hits * sizeof(ps4_hit), cudaMemcpyDeviceToHost, s->s_copy));
        if (h.n_exts)
            SRV_CUDA(s, cudaMemcpyAsync(q.exts.data(), h.exts, h.n_exts * sizeof(ps4_ext), cudaMemcpyDeviceToHost, s->s_copy));
        if (h.n_sixes)
            SRV_CUDA(s, cudaMemcpyAsync(q.sixes.data(), h.sixes, h.n_sixes * sizeof(ps4_six), cudaMemcpyDeviceToHost,
                                        s->s_copy));
        if (h.n_tri)
            SRV_CUDA(s, cudaMemcpyAsync(q.tri.data(), h.tri, h.n_tri * sizeof(ps4_tri_ext), cudaMemcpyDeviceToHost,
                                        s->s_copy));
        memset(&q.stats, 0, sizeof q.stats);
        stats_add(&q.stats, h.k);
        memset(&q.tstats, 0, sizeof q.tstats);
        if (q.kind == PS4_Q_TRIPLE) {
            q.tstats.triples = q.tri_state == TRI_OK;
            q.tstats.invalid = q.tri_state == TRI_INVALID;
            q.tstats.ext_cand = h.tri_cand;
            q.tstats.ext_sqrt = h.tri_sqrt;
            q.tstats.exts = h.n_tri;
        }
        fetch.push_back(ok[i]);
    }
    SRV_CUDA(s, cudaStreamSynchronize(s->s_copy));
    const double t2 = now_s();
    for (uint32_t id : fetch) {
        Query &q = Q(s, id);
        if (q.kind == PS4_Q_RANGE) canonical_order(q.hits, q.exts, q.sixes);
        else std::sort(q.tri.begin(), q.tri.end(), [](const ps4_tri_ext &x, const ps4_tri_ext &y) { return x.d < y.d; });
        finish_query(s, id, t2);
    }
    return PS4_OK;
}

int pump(ps4_server *s) {
    for (int i = 0; i < 2; i++) {
        StepBuf &b = s->buf[i];
        if (b.state == BUF_KERNELS) {
            // ev_post, recorded behind the status copies, doubles as "kernels and copies done"
            cudaError_t e = cudaEventQuery(b.ev_post);
            if (e == cudaErrorNotReady) continue;
            if (e != cudaSuccess) return srv_err(s, PS4_ERR_CUDA, "step failed: %s", cudaGetErrorString(e));
            int rc = check_step(s, b);
            if (rc) return rc;
        }
    }
    for (int i = 0; i < 2; i++) {
        StepBuf &b = s->buf[i];
        if (b.state == BUF_POST) {
            cudaError_t e = cudaEventQuery(b.ev_post);
            if (e == cudaErrorNotReady) continue;
            if (e != cudaSuccess) return srv_err(s, PS4_ERR_CUDA, "step fold failed: %s", cudaGetErrorString(e));
            int rc = complete_step(s, b);
            if (rc) return rc;
        }
    }
    int rc = admit(s);
    if (rc) return rc;
    for (int k = 0; k < 2; k++) {
        StepBuf &b = s->buf[s->next_buf];
        if (b.state != BUF_FREE || !has_work(s)) break;
        plan_step(s, b);
        if (b.chunks.empty() && b.tris.empty()) break;
        rc = launch_step(s, b);
        if (rc) return rc;
        s->next_buf ^= 1;
    }
    return PS4_OK;
}

int init_buf(ps4_server *s, StepBuf &b) {
    const uint32_t ni = s->cfg.max_step_items, nt = s->cfg.max_step_triples;
    if (dev_alloc(s, b.d_items, ni) || dev_alloc(s, b.d_item_slot, ni) || dev_alloc(s, b.d_counters, (uint64_t)ni * K_SLOTS) ||
        dev_alloc(s, b.d_status, 1) || dev_alloc(s, b.d_abc, 3 * (uint64_t)nt) || dev_alloc(s, b.d_tri_slot, nt) ||
        dev_alloc(s, b.d_tri_state, nt) || dev_alloc(s, b.d_tri_cnt, 3) || dev_alloc(s, b.d_cand_per, nt) ||
        dev_alloc(s, b.d_sqrt_per, nt))
        return PS4_ERR_CUDA;
    const uint64_t hits0 = 4096 + (uint64_t)(4e-5 * (double)s->cfg.step_S);
    if (grow_dev(s, b.d_hits, b.hits_cap, hits0) || grow_dev(s, b.d_remap, b.remap_cap, hits0) ||
        grow_dev(s, b.d_exts, b.exts_cap, 2 * hits0) || grow_dev(s, b.d_sixes, b.sixes_cap, 1024) ||
        grow_dev(s, b.d_tri_out, b.tri_out_cap, std::max<uint64_t>(4096, nt)))
        return PS4_ERR_CUDA;
    if (host_alloc(s, b.h_items, ni) || host_alloc(s, b.h_item_slot, ni) || host_alloc(s, b.h_abc, 3 * (uint64_t)nt) ||
        host_alloc(s, b.h_tri_slot, nt) || host_alloc(s, b.h_tri_state, nt) || host_alloc(s, b.h_status, 1) ||
        host_alloc(s, b.h_tri_cnt, 3))
        return PS4_ERR_CUDA;
    SRV_CUDA(s, cudaEventCreate(&b.ev_start));
    SRV_CUDA(s, cudaEventCreate(&b.ev_kern));
    SRV_CUDA(s, cudaEventCreateWithFlags(&b.ev_post, cudaEventDisableTiming));
    SRV_CUDA(s, cudaEventCreateWithFlags(&b.ev_fork, cudaEventDisableTiming));
    SRV_CUDA(s, cudaEventCreateWithFlags(&b.ev_join, cudaEventDisableTiming));
    return PS4_OK;
}

void free_buf(StepBuf &b) {
    cudaFree(b.d_items); cudaFree(b.d_item_slot); cudaFree(b.d_counters); cudaFree(b.d_status);
    cudaFree(b.d_hits); cudaFree(b.d_exts); cudaFree(b.d_sixes); cudaFree(b.d_remap);
    cudaFree(b.d_abc); cudaFree(b.d_tri_slot); cudaFree(b.d_tri_state); cudaFree(b.d_tri_out);
    cudaFree(b.d_tri_cnt); cudaFree(b.d_cand_per); cudaFree(b.d_sqrt_per);
    cudaFreeHost(b.h_items); cudaFreeHost(b.h_item_slot); cudaFreeHost(b.h_abc); cudaFreeHost(b.h_tri_slot);
    cudaFreeHost(b.h_tri_state); cudaFreeHost(b.h_status); cudaFreeHost(b.h_tri_cnt);
    for (cudaEvent_t e : {b.ev_start, b.ev_kern, b.ev_post, b.ev_fork, b.ev_join})
        if (e) cudaEventDestroy(e);
}

uint32_t new_query(ps4_server *s) {
    uint32_t id;
    if (!s->free_ids.empty()) {
        id = s->free_ids.back();
        s->free_ids.pop_back();
        s->qs[id].reset(new Query());
    } else {
        id = (uint32_t)s->qs.size();
        s->qs.emplace_back(new Query());
    }
    return id;
}

void forget(ps4_server *s, uint64_t tag) {
    auto it = s->by_tag.find(tag);
    if (it == s->by_tag.end()) return;
    s->qs[it->second].reset();
    s->free_ids.push_back(it->second);
    s->by_tag.erase(it);
}

}  // namespace

// ---------------------------------------------------------------- C-ABI

extern "C" int ps4_serve_create(ps4_ctx *ctx, const ps4_serve_config *cfg, ps4_server **out) {
    if (!out) return PS4_ERR_ARG;
    *out = nullptr;
    ps4_server *s = new ps4_server();
    *out = s;
    if (!ctx || ctx_view(ctx, &s->v) != PS4_OK) return srv_err(s, PS4_ERR_ARG, "ps4_serve_create: no usable context");
    if (s->v.flags & PS4_F_DUMP4) return srv_err(s, PS4_ERR_ARG, "serving does not support PS4_F_DUMP4 contexts");
    s->ctx = ctx;
    ps4_serve_config c;
    memset(&c, 0, sizeof c);
    if (cfg) c = *cfg;
    if (!c.hbm_budget) c.hbm_budget = 8ull << 30;
    if (!c.max_slots) c.max_slots = 1024;
    if (!c.max_step_items) c.max_step_items = 4096;
    if (!c.step_S) c.step_S = 1ull << 27;
    if (!c.max_step_triples) c.max_step_triples = 65536;
    if (!c.hits_floor && !c.hits_per_1e6_S) { c.hits_floor = 256; c.hits_per_1e6_S = 40; }
    c.step_S = std::max<uint64_t>(c.step_S, 1ull << 14);
    s->cfg = c;
    SRV_CUDA(s, cudaSetDevice(s->v.device));
    SRV_CUDA(s, cudaStreamCreateWithFlags(&s->s_main, cudaStreamNonBlocking));
    SRV_CUDA(s, cudaStreamCreateWithFlags(&s->s_tri, cudaStreamNonBlocking));
    SRV_CUDA(s, cudaStreamCreateWithFlags(&s->s_post, cudaStreamNonBlocking));
    SRV_CUDA(s, cudaStreamCreateWithFlags(&s->s_copy, cudaStreamNonBlocking));
    // job queue for one step at the densest S the context allows
    const double need = jobs_per_S_bound(s->v.s_hi_max) * (double)c.step_S / 0.9;
    s->jobs_cap = 1ull << 20;
    while (s->jobs_cap < (1ull << 27) && (double)s->jobs_cap < need) s->jobs_cap <<= 1;
    if (dev_alloc(s, s->d_jobs, 6 * s->jobs_cap)) return PS4_ERR_CUDA;
    // lists for the tile kernel's full residency at any tile size (the same bytes at every size)
    if (dev_alloc(s, s->d_raw, (uint64_t)gen_grid(s->v.num_sms, 14) * SUPER_K * RAW_PER_TILE)) return PS4_ERR_CUDA;
    if (dev_alloc(s, s->d_slots, c.max_slots)) return PS4_ERR_CUDA;
    for (int i = 0; i < 2; i++)
        if (init_buf(s, s->buf[i])) return PS4_ERR_CUDA;
    if (s->device_bytes + (16ull << 20) > c.hbm_budget)
        return srv_err(s, PS4_ERR_ARG, "hbm_budget %llu leaves no arena: step buffers take %llu bytes",
                       (unsigned long long)c.hbm_budget, (unsigned long long)s->device_bytes);
    const uint64_t arena = (c.hbm_budget - s->device_bytes) & ~255ull;
    if (dev_alloc(s, s->d_arena, arena)) return PS4_ERR_CUDA;
    s->arena.reset(arena);
    for (int i = (int)c.max_slots - 1; i >= 0; i--) s->free_slots.push_back(i);
    SRV_CUDA(s, cudaDeviceSynchronize());
    return PS4_OK;
}

extern "C" void ps4_serve_destroy(ps4_server *s) {
    if (!s) return;
    if (s->s_main) {
        cudaStreamSynchronize(s->s_main);
        cudaStreamSynchronize(s->s_tri);
        cudaStreamSynchronize(s->s_post);
        cudaStreamSynchronize(s->s_copy);
    }
    for (int i = 0; i < 2; i++) free_buf(s->buf[i]);
    cudaFree(s->d_jobs); cudaFree(s->d_raw); cudaFree(s->d_scratch); cudaFree(s->d_slots); cudaFree(s->d_arena);
    for (cudaStream_t st : {s->s_main, s->s_tri, s->s_post, s->s_copy})
        if (st) cudaStreamDestroy(st);
    delete s;
}

extern "C" const char *ps4_serve_last_error(const ps4_server *s) { return s ? s->err.c_str() : "null server"; }

static int submit(ps4_server *s, Query &&proto) {
    if (s->by_tag.count(proto.tag)) return srv_err(s, PS4_ERR_ARG, "tag %llu is already in use", (unsigned long long)proto.tag);
    const uint32_t id = new_query(s);
    Query &q = *s->qs[id];
    q = std::move(proto);
    q.t_submit = now_s();
    s->by_tag[q.tag] = id;
    s->waiting.push_back(id);
    s->n_submitted++;
    return PS4_OK;
}

extern "C" int ps4_serve_submit_range(ps4_server *s, uint64_t tag, uint64_t lo, uint64_t hi) {
    if (!s || !s->ctx) return PS4_ERR_ARG;
    if (hi > s->v.s_hi_max)
        return srv_err(s, PS4_ERR_ARG, "S_hi %llu exceeds the context's s_hi_max %llu", (unsigned long long)hi,
                       (unsigned long long)s->v.s_hi_max);
    Query q;
    q.tag = tag;
    q.kind = PS4_Q_RANGE;
    q.lo = std::max<uint64_t>(lo, 1);
    q.hi = std::max<uint64_t>(hi, q.lo);
    if (q.hi - q.lo >= (1ull << 43)) return srv_err(s, PS4_ERR_ARG, "range too large for one query; split it");
    range_quota(s, q, 0, 0, 0);
    return submit(s, std::move(q));
}

extern "C" int ps4_serve_submit_triple(ps4_server *s, uint64_t tag, const uint64_t abc[3], uint64_t dmax) {
    if (!s || !s->ctx || !abc) return PS4_ERR_ARG;
    if (dmax > (1ull << 62)) return srv_err(s, PS4_ERR_ARG, "dmax %llu exceeds 2^62", (unsigned long long)dmax);
    Query q;
    q.tag = tag;
    q.kind = PS4_Q_TRIPLE;
    q.abc[0] = abc[0]; q.abc[1] = abc[1]; q.abc[2] = abc[2];
    q.dmax = dmax;
    q.cap_tri = TRI_RECS;
    return submit(s, std::move(q));
}

extern "C" int ps4_serve_progress(ps4_server *s, uint32_t wait_us, ps4_serve_done *done, uint32_t cap, uint32_t *n_done) {
    if (!s || !s->ctx) return PS4_ERR_ARG;
    if (n_done) *n_done = 0;
    const double t_end = now_s() + 1e-6 * (double)wait_us;
    for (;;) {
        int rc = pump(s);
        if (rc) return rc;
        uint32_t n = 0;
        while (!s->unreported.empty() && n < cap && done) {
            const Query &q = Q(s, s->unreported.front());
            s->unreported.pop_front();
            ps4_serve_done &d = done[n++];
            memset(&d, 0, sizeof d);
            d.tag = q.tag;
            d.status = q.status;
            d.kind = q.kind;
            d.n_records = q.kind == PS4_Q_RANGE ? q.hits.size() : q.tri.size();
            d.t_submit = q.t_submit; d.t_admit = q.t_admit; d.t_done = q.t_done;
            d.steps = q.steps;
            d.reruns = q.reruns;
            snprintf(d.message, sizeof d.message, "%s", q.msg.c_str());
        }
        if (n_done) *n_done = n;
        const bool busy = s->buf[0].state != BUF_FREE || s->buf[1].state != BUF_FREE;
        if (n > 0 || !busy || now_s() >= t_end) return PS4_OK;
        struct timespec ts = {0, 20000};
        nanosleep(&ts, nullptr);
    }
}

static Query *finished_query(ps4_server *s, uint64_t tag, uint32_t kind) {
    auto it = s->by_tag.find(tag);
    if (it == s->by_tag.end()) { srv_err(s, PS4_ERR_ARG, "unknown tag %llu", (unsigned long long)tag); return nullptr; }
    Query &q = *s->qs[it->second];
    if (!q.finished) { srv_err(s, PS4_ERR_ARG, "query %llu has not finished", (unsigned long long)tag); return nullptr; }
    if (q.kind != kind) { srv_err(s, PS4_ERR_ARG, "query %llu is of the other kind", (unsigned long long)tag); return nullptr; }
    return &q;
}

extern "C" int ps4_serve_take_range(ps4_server *s, uint64_t tag, ps4_stats *stats, ps4_results *res) {
    if (!s) return PS4_ERR_ARG;
    Query *q = finished_query(s, tag, PS4_Q_RANGE);
    if (!q) return PS4_ERR_ARG;
    if (q->failed) {
        const int code = q->status;
        srv_err(s, code, "%s", q->msg.c_str());
        forget(s, tag);
        return code;
    }
    if (res) {
        res->n_hits = q->hits.size(); res->n_exts = q->exts.size(); res->n_sixes = q->sixes.size(); res->n_quads = 0;
        if (res->n_hits > res->hits_cap || res->n_exts > res->exts_cap || res->n_sixes > res->sixes_cap)
            return srv_err(s, PS4_ERR_OUTPUT_FULL, "result buffers too small: need hits=%llu exts=%llu sixes=%llu",
                           (unsigned long long)res->n_hits, (unsigned long long)res->n_exts,
                           (unsigned long long)res->n_sixes);
        if (!q->hits.empty()) memcpy(res->hits, q->hits.data(), q->hits.size() * sizeof(ps4_hit));
        if (!q->exts.empty()) memcpy(res->exts, q->exts.data(), q->exts.size() * sizeof(ps4_ext));
        if (!q->sixes.empty()) memcpy(res->sixes, q->sixes.data(), q->sixes.size() * sizeof(ps4_six));
    }
    if (stats) {
        uint64_t *dst = &stats->S_done;
        const uint64_t *src = &q->stats.S_done;
        for (int i = 0; i < 10; i++) dst[i] += src[i];
        for (int i = 0; i < 100; i++) stats->hist5[i] += q->stats.hist5[i];
        stats->max_reps = std::max(stats->max_reps, q->stats.max_reps);
        stats->max_divisors = std::max(stats->max_divisors, q->stats.max_divisors);
        stats->max_extensions = std::max(stats->max_extensions, q->stats.max_extensions);
    }
    forget(s, tag);
    return PS4_OK;
}

extern "C" int ps4_serve_take_triple(ps4_server *s, uint64_t tag, uint8_t *state, ps4_tri_ext *out, uint64_t out_cap,
                                     uint64_t *n_out, ps4_tri_stats *stats) {
    if (!s) return PS4_ERR_ARG;
    Query *q = finished_query(s, tag, PS4_Q_TRIPLE);
    if (!q) return PS4_ERR_ARG;
    if (q->failed) {
        const int code = q->status;
        srv_err(s, code, "%s", q->msg.c_str());
        forget(s, tag);
        return code;
    }
    if (n_out) *n_out = q->tri.size();
    if (q->tri.size() > out_cap)
        return srv_err(s, PS4_ERR_OUTPUT_FULL, "triple output holds %llu records, %llu needed",
                       (unsigned long long)out_cap, (unsigned long long)q->tri.size());
    if (!q->tri.empty()) memcpy(out, q->tri.data(), q->tri.size() * sizeof(ps4_tri_ext));
    if (state) *state = q->tri_state;
    if (stats) {
        stats->triples += q->tstats.triples;
        stats->invalid += q->tstats.invalid;
        stats->ext_cand += q->tstats.ext_cand;
        stats->ext_sqrt += q->tstats.ext_sqrt;
        stats->exts += q->tstats.exts;
    }
    forget(s, tag);
    return PS4_OK;
}

extern "C" void ps4_serve_get_info(const ps4_server *s, ps4_serve_info *info) {
    if (!info) return;
    memset(info, 0, sizeof *info);
    if (!s) return;
    info->submitted = s->n_submitted;
    info->waiting = s->waiting.size();
    info->active = s->active.size();
    info->finished = s->n_finished;
    info->steps = s->n_steps;
    info->step_reruns = s->n_step_reruns;
    info->arena_bytes = s->arena.size;
    info->arena_used = s->arena.used;
    info->arena_peak = s->arena.peak;
    info->device_bytes = s->device_bytes;
    info->gpu_ms = s->gpu_ms;
}
