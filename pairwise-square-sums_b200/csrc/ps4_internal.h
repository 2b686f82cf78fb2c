// ps4_internal.h -- layouts shared by the device kernels (ps4_kernels.cu) and the host
// orchestration behind the C-ABI (ps4_api.cu).  Not part of the public interface.
#pragma once
#include <stdint.h>

#include <vector>

#include "../../include/ps4.h"

namespace ps4 {

// ---- per-item counter block (u64 slots), one block per query item -------------------
// Slots 0..9 are the reference's additive counters in stats_t order (s4.c:81), 10..12
// the capacity high-water marks (s4.c:90), 16..115 the 5-set log2 histogram (s4.c:82).
enum {
    K_S_DONE = 0, K_PAIRS, K_S_GE3, K_TRIPLES, K_SETS4, K_SETS5, K_SETS6, K_MULTI, K_EXT_CAND, K_EXT_SQRT,
    K_MAX_REPS = 10, K_MAX_DIVS = 11, K_MAX_EXT = 12,
    K_HIST5 = 16,
    K_SLOTS = 128
};

// ---- device error word: code in bits 0..7, the S where it happened in bits 8..63 -----
enum {
    E_NONE = 0,
    E_CAP_REPS = PS4_ERR_CAP_REPS,
    E_CAP_DIVS = PS4_ERR_CAP_DIVS,
    E_CAP_EXT = PS4_ERR_CAP_EXT,
    E_VERIFY = PS4_ERR_VERIFY,
    E_TILE = 100,      // a tile outgrew its shared-memory lists: re-run with smaller tiles
    E_EXTLIST = 101,   // more extensions than a tile's (fused kernel) or an engine round's list holds
    E_QUEUE = 102,     // the 4-set job queue of a batch overflowed: re-run with narrower batches
    E_TIMEOUT = PS4_ERR_TIMEOUT   // a bounded wait of the persistent kernel gave up (code | where << 8)
};

// One query segment: every S in [lo, hi) of query item `id`.  Tiles of the segment are
// numbered from tile_base.
struct Item {
    uint64_t lo, hi;
    uint64_t tile_base;   // prefix sum of tile counts over the segments before this one
    uint32_t id;          // the query item the segment belongs to (counters, hit records)
    uint32_t pad;
};

// Status block copied back after every launch.
struct Status {
    unsigned long long err;        // first error (code | S << 8)
    unsigned long long verify_bad[5];  // --verify failure: S, a, b, c, d
    unsigned int n_hits, n_exts, n_sixes, pad0;
    unsigned long long n_quads;
    unsigned long long diag[4];    // first internal-capacity event: which list, size, limit, S
    // per batch of the two-kernel pipeline (cleared before every batch)
    unsigned long long n_jobs;     // 4-sets queued by gen_jobs
    unsigned int tile_next;        // tile work counter of the tile kernels (tiles handed out)
    unsigned int ext_next;         // extend_jobs work counter (queued 4-sets handed out)
    // the persistent kernel's 4-set ring (positions count up from 0 over a call; slot = pos & mask)
    unsigned long long q_tail;     // positions reserved by producing CTAs
    unsigned long long q_head;     // positions claimed by consuming warps
    unsigned long long q_freed;    // positions whose 4-set is finished and whose slot is free again
    unsigned long long q_produced; // tiles whose 4-sets are all written
    unsigned long long q_pub;      // 4-sets written and published (any order): what claims may count on
};

// Arguments of one search launch (passed by value).
struct SearchArgs {
    const Item *items;
    uint32_t n_items;
    uint64_t n_tiles;
    unsigned log2_tile;
    const uint64_t *spfq;      // spf | quot << 32, m < tab_n
    const uint16_t *ndiv;      // divisor counts, m < tab_n
    uint64_t tab_n;
    const uint4 *fac3;         // odd m: up to three odd primes (p | e << 24, ascending) and the cofactor
    unsigned long long *counters;   // [n_items][K_SLOTS]
    ps4_hit *hits;   uint32_t hits_cap;
    ps4_ext *exts;   uint32_t exts_cap;
    ps4_six *sixes;  uint32_t sixes_cap;
    ps4_quad *quads; unsigned long long quads_cap;
    uint32_t *scratch;         // per-CTA 4-set staging (batched kernel): 6 * stage_cap u32 per CTA
    uint32_t stage_cap;        // 4-sets the staging of one CTA holds
    Status *status;
    uint32_t cap_reps, cap_divs, cap_ext;
    uint32_t flags;            // PS4_F_*
    uint32_t *jobs;            // 4-set job queue between gen_jobs and extend_jobs: jobs_cap 24-byte records
    uint64_t jobs_cap;
    uint64_t *raw;             // optional (gen_jobs): per CTA, SUPER_K lists of one tile's representations,
    uint32_t raw_cap;          //   raw_cap entries each, in one equal slice per warp
    // persistent kernel: jobs is a ring of jobs_cap (a power of two) slots; seq[slot] tells its state
    // for position pos = slot + lap * jobs_cap: pos = free for pos, pos + 1 = 4-set of pos written
    uint32_t *seq;
    uint64_t ring_mask;        // jobs_cap - 1
    uint64_t ring_fast;        // claims may take positions without a compare-and-swap while this many
                               //   reserved positions are unclaimed (> every warp's claim at once)
    uint64_t ring_high;        // a CTA turns to the engine when this many 4-sets are queued ...
    uint64_t ring_low;         //   and its warps stop claiming below this many while tiles are left
};
// the persistent kernel's threads per CTA, and the time any of its waits may take before it gives up
constexpr int PBS = 256;
constexpr unsigned long long WAIT_NS = 2000000000ull;
// representations a 2^14-S tile's list holds: (pi/8) * 2^14 = 6434 expected, 8192 with margin;
// a 2^TL-S tile's list holds raw_cap_for(TL), in proportion
constexpr uint32_t RAW_PER_TILE = 8192;
constexpr uint32_t raw_cap_for(unsigned TL) { return RAW_PER_TILE >> (14 - TL); }
// tiles a tile-kernel CTA claims at once and scans as one range: the scan of a tile costs
// ~0.29 sqrt(S) steps whatever its width, so one scan of SUPER_K adjacent tiles, recorded into
// their lists, divides that cost by SUPER_K (lists: 592 CTAs x 16 x 32 KB = 310 MB; 16 tiles of
// 2^13 S instead of 8: tile kernel -8 % at S = 5e11, per 5e8-S step).  With these tiles the group
// scan pays at every S: per [1,1e10) step of the tile kernel 195.4 ms with groups from S = 5e9 up,
// 161.0 from 1e9, 159.7 everywhere.
constexpr uint32_t SUPER_K = 16;
// threads of a tile-kernel CTA: 512 on 2^14-S tiles (two CTAs per SM), 256 on smaller ones (four
// per SM).  At 2^13 S and four CTAs a barrier waits for 8 warps, not 16, and while one CTA waits
// at it the other three issue: per [1,1e10) step of the tile kernel 219.2 -> 195.2 ms.
constexpr int gen_threads(unsigned TL) { return TL >= 14 ? 512 : 256; }

// Arguments of one triple-extension launch (ps4_triples.cu).
struct TriArgs {
    const uint64_t *abc;       // 3 members per triple, any order
    uint64_t n;                // triples
    uint64_t dmax;             // extensions d <= dmax
    const uint64_t *spfq;
    const uint16_t *ndiv;
    uint64_t tab_n;
    uint8_t *state;            // per triple: TRI_OK / TRI_INVALID / TRI_RANGE
    ps4_tri_ext *out;
    uint64_t out_cap;
    unsigned long long *n_out;     // records found (may exceed out_cap: nothing written past it)
    unsigned long long *n_cand;    // same-parity complementary divisor pairs of the chosen differences
    unsigned long long *n_sqrt;    // exact square tests of d + C
    uint32_t item_base;            // added to the triple index in the records
    unsigned long long *cand_per;  // optional (may be null): ext_cand of each triple
    unsigned long long *sqrt_per;  // optional (may be null): ext_sqrt of each triple
};
enum { TRI_OK = 0, TRI_INVALID = 1, TRI_RANGE = 2 };

// Host helpers shared by the single-query calls and the server (ps4_api.cu).
void stats_add(ps4_stats *s, const unsigned long long *k);      // fold one counter block into stats (+=)
const char *fatal_text(unsigned code);                            // the reference's FATAL message text
double jobs_per_S_bound(uint64_t S_hi);                           // 4-set job queue entries per S, bound
void canonical_order(std::vector<ps4_hit> &hits, std::vector<ps4_ext> &exts, std::vector<ps4_six> &sixes);
void canonical_order_into(const ps4_hit *hits, uint64_t nh, const ps4_ext *exts, ps4_six *sixes, uint64_t ns,
                          ps4_hit *out_hits, ps4_ext *out_exts);

// Read-only view of a context (ps4_api.cu), for the allocation-free entry point and the server.
struct CtxView {
    const uint64_t *spfq;
    const uint16_t *ndiv;
    const uint4 *fac3;
    uint64_t tab_n, s_hi_max;
    uint32_t cap_reps, cap_divs, cap_ext, flags;
    int device, num_sms;
    void *stream;
};
int ctx_view(ps4_ctx *c, CtxView *v);
int ctx_fail(ps4_ctx *c, int code, const char *msg);

// Launchers (ps4_kernels.cu).  Return a cudaError_t value.
int launch_tables(uint64_t *spfq, uint16_t *ndiv, uint64_t tab_n, void *stream);
int launch_fac3(uint4 *fac3, uint64_t tab_n, void *stream);
// two-kernel pipeline (ps4_extend.cu): 4-set generation into the job queue, then extension
int launch_gen(const SearchArgs &a, int grid, void *stream);
int launch_ext(const SearchArgs &a, int grid, void *stream);
// the persistent kernel (ps4_extend.cu): tiles of 2^13 S, ring of a.jobs_cap slots
int launch_persist(const SearchArgs &a, int grid, void *stream);
int launch_ring_init(uint32_t *seq, uint64_t n, void *stream);
int launch_ring_wait_probe(const SearchArgs &a, unsigned long long *out, void *stream);
int persist_ctas_per_sm();
int gen_grid(int num_sms, unsigned TL);      // the tile kernel's full residency for 2^TL-S tiles
int ext_grid(int num_sms);
int launch_search(const SearchArgs &a, int kernel, int grid, void *stream);
int launch_triples(const TriArgs &t, void *stream);
size_t search_smem_bytes(int kernel, unsigned log2_tile);
int search_block_threads();
uint32_t stage_cap_for(unsigned log2_tile, uint32_t cap_reps);

}  // namespace ps4
