// ps4_extend.cu -- the batched search as two persistent kernels per batch of S:
//
//   gen_jobs<TL,NT>  tiles of 2^TL S in shared memory (P1-P4 of ps4_device.cuh), then every
//                 4-set of the tile (P5: closed-form z ranges per representation pair) is
//                 written to a global job queue: a count pass, one block scan, one atomic
//                 reservation per tile, a write pass.                         (s4.c:280-341)
//   extend_jobs   the extension engine.  Each lane of a warp holds one queued 4-set; it picks
//                 the difference to extend by and factors it.  In rounds, the warp places the
//                 factored odd-divisor lists of as many of its 4-sets as fit in its shared
//                 buffer, pools the candidates of those 4-sets -- the complementary divisor
//                 pairs (f,g), f<g, of equal parity, each visited once -- and splits them into
//                 32 equal contiguous runs, one per lane, so every lane does the same work
//                 whatever the divisor counts; lanes whose 4-set is done take the next one from
//                 the queue before the next round.  Residue filters mod 64/63/65 are bit tests
//                 against per-4-set masks indexed by u's residue; the candidates that pass (the
//                 reference's ext_sqrt) go through a warp queue and are square-tested 32 at a
//                 time.                                                        (s4.c:160-207)
//
// Every counter and every reported line is identical to the reference's.

#include <cuda_runtime.h>
#include <stdint.h>

#include "ps4_device.cuh"

namespace ps4 {

// ================================================================== job records

// A queued 4-set: its six pair roots (< 2^22), one 24-byte record per 4-set (three 8-byte
// stores and loads; six u32 arrays took 2.2 % more tile-kernel and 1.2 % more engine time per
// [1,1e10) step).  The query item id (< 2^20) rides in the spare top bits of r_ac (bits 0..9
// of the id) and r_ad (bits 10..19).  The queue of cap records is 6 * cap u32.
__device__ __forceinline__ void put_job(uint32_t *jobs, uint64_t j, const uint32_t r[6], uint32_t item) {
    uint2 *p = (uint2 *)(jobs + 6 * j);               // 8-byte aligned: 24 * j
    p[0] = make_uint2(r[0], r[1] | ((item & 1023u) << 22));
    p[1] = make_uint2(r[2] | (((item >> 10) & 1023u) << 22), r[3]);
    p[2] = make_uint2(r[4], r[5]);
}

// COH: the queue is a ring whose slots are rewritten while the kernel runs, so its words are read
// through L2 (coherent), not the read-only path that may hold a slot's previous 4-set.
template <bool COH = false>
__device__ __forceinline__ void get_job(const uint32_t *jobs, uint64_t j, uint32_t r[6], uint32_t &item) {
    const uint2 *p = (const uint2 *)(jobs + 6 * j);
    const uint2 x = COH ? __ldcg(p) : __ldg(p), y = COH ? __ldcg(p + 1) : __ldg(p + 1),
                z = COH ? __ldcg(p + 2) : __ldg(p + 2);
    const uint32_t w1 = x.y, w2 = y.x;
    r[0] = x.x;
    r[1] = w1 & 0x3FFFFFu;
    r[2] = w2 & 0x3FFFFFu;
    r[3] = y.y;
    r[4] = z.x;
    r[5] = z.y;
    item = (w1 >> 22) | ((w2 >> 22) << 10);
}

// ================================================================== the persistent kernel's ring
//
// Producing CTAs reserve positions (q_tail), wait until each position's slot is free of its
// previous lap, write the 4-set, and publish it: seq[slot] = pos + 1 after a fence.  Consuming
// warps claim positions below q_tail (q_head), wait until each is published, and after the 4-set
// is extended and reported free its slot: seq[slot] = pos + ring size.  Every wait is bounded in
// time (WAIT_NS); a wait that gives up sets the error word to E_TIMEOUT (with which wait in the S
// field: 1 published, 2 slot free, 3 ring room, 4 idle) and the kernel ends, the host re-running
// the call on the two-kernel pipeline.

__device__ __forceinline__ uint64_t gtimer() {
    uint64_t t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    return t;
}
__device__ __forceinline__ uint32_t ld_vol(const uint32_t *p) { return *(const volatile uint32_t *)p; }
__device__ __forceinline__ ull ld_vol(const ull *p) { return *(const volatile ull *)p; }

// Tracks one wait's elapsed time: true once it has lasted WAIT_NS (and records the timeout).
struct WaitClock {
    uint64_t t0 = 0;
    __device__ __forceinline__ bool expired(const SearchArgs &a, unsigned which) {
        const uint64_t t = gtimer();
        if (!t0) { t0 = t; return false; }
        if (t - t0 <= WAIT_NS) return false;
        raise_error(a.status, E_TIMEOUT, which);
        return true;
    }
};

// A producer's slot: wait until it is free for position pos.  False if the call stopped.
__device__ __noinline__ bool ring_wait_free(const SearchArgs &a, uint64_t pos) {
    const uint32_t *f = a.seq + (pos & a.ring_mask);
    WaitClock wc;
    for (uint32_t k = 0;; k++) {
        if (ld_vol(f) == (uint32_t)pos) return true;
        if ((k & 15) == 15 && (ld_vol(&a.status->err) != 0ull || wc.expired(a, 2))) return false;
        __nanosleep(64);
    }
}

// A consumer's claimed position: wait until its 4-set is published.  False if the call stopped,
// or if the position will never be written (every tile is produced and the position lies past
// the last reserved one: a claim that overtook the reservations, see ring_claim).
__device__ __noinline__ bool ring_wait_ready(const SearchArgs &a, uint64_t pos) {
    const uint32_t *f = a.seq + (pos & a.ring_mask);
    WaitClock wc;
    for (uint32_t k = 0;; k++) {
        if (ld_vol(f) == (uint32_t)(pos + 1)) {
            __threadfence();                       // the 4-set's words after its flag
            return true;
        }
        if ((k & 15) == 15) {
            if (ld_vol(&a.status->err) != 0ull) return false;
            if (ld_vol(&a.status->q_produced) >= a.n_tiles && pos >= ld_vol(&a.status->q_tail)) return false;
            if (wc.expired(a, 1)) return false;
        }
        __nanosleep(32);
    }
}

__device__ __forceinline__ void ring_release(const SearchArgs &a, uint64_t pos) {
    __threadfence();                               // every read of the slot before it is handed back
    *(volatile uint32_t *)&a.seq[pos & a.ring_mask] = (uint32_t)(pos + a.ring_mask + 1);
}

// Claim up to n positions below q_tail (one lane of a warp).  The thresholds count published
// 4-sets (q_pub), so that claims rarely land on positions still being written.  While tiles are
// left, fewer than ring_low published 4-sets are left for later (the warp stops consuming, its
// CTA turns to tiles).  While at least ring_fast published positions are unclaimed, an add cannot
// overtake the reservations (every warp of the grid claiming at once takes fewer), so it is
// used; closer to q_tail a compare-and-swap claims only what is reserved.  *got receives the count, the first
// position is returned.
__device__ __forceinline__ uint64_t ring_claim(const SearchArgs &a, uint32_t n, uint32_t *got) {
    ull *head = &a.status->q_head;
    ull h = ld_vol(head);
    const ull t = ld_vol(&a.status->q_tail);
    const long long pub = (long long)(ld_vol(&a.status->q_pub) - h);   // published and unclaimed (about)
    *got = 0;
    if ((long long)(t - h) <= 0) return 0;
    if (pub < (long long)a.ring_low && ld_vol(&a.status->tile_next) < a.n_tiles) return 0;
    if (pub >= (long long)a.ring_fast) {
        *got = n;
        return atomicAdd(head, (ull)n);
    }
    for (int k = 0; k < 16; k++) {
        const ull tt = ld_vol(&a.status->q_tail);
        if ((long long)(tt - h) <= 0) break;
        const ull take = tt - h < n ? tt - h : n;
        const ull prev = atomicCAS(head, h, h + take);
        if (prev == h) {
            *got = (uint32_t)take;
            return h;
        }
        h = prev;
    }
    return 0;
}

// ================================================================== gen_jobs

// The 4-sets of representation pair gidx of the tile (P5), pair given as list s and (x, y).
// Counts them; with WRITE also builds, checks, dumps and (when `store`) queues them at out, ...
template <bool WRITE, bool RING = false>
__device__ __forceinline__ uint32_t pair_quads(const SearchArgs &a, uint32_t st, uint32_t k, uint64_t S,
                                               uint32_t x, uint32_t y, const uint32_t *rep_p,
                                               const uint32_t *rep_q, uint32_t item, uint64_t out, bool store) {
    const uint32_t px = rep_p[st + x], py = rep_p[st + y];
    const uint64_t Px = (uint64_t)px * px, Py = (uint64_t)py * py;
    const uint32_t pxy = (px + py) & 1;
    const uint32_t Sodd = (uint32_t)(S & 1);
    uint32_t n = 0;
    for (int cls = 0; cls < 2; cls++) {
        // class 0: z upward while P_z < P_x + P_y;  class 1: z downward while P_z > S - P_x - P_y
        const uint32_t want = cls == 0 ? 0u : Sodd;
        for (uint32_t z = cls == 0 ? y + 1 : k - 1; z > y && z < k; z = cls == 0 ? z + 1 : z - 1) {
            const uint32_t pz = rep_p[st + z];
            const uint64_t Pz = (uint64_t)pz * pz;
            if (cls == 0 ? Pz >= Px + Py : Pz <= S - Px - Py) break;
            if (((pxy + pz) & 1) != want) continue;
            const uint32_t qz = rep_q[st + z];
            if (cls == 1 && qz == pz) continue;
            if (WRITE) {
                uint32_t r[6];
                r[0] = rep_q[st + x]; r[1] = rep_q[st + y]; r[4] = py; r[5] = px;
                r[2] = cls == 0 ? qz : pz;
                r[3] = cls == 0 ? pz : qz;
                if (a.flags & PS4_F_VERIFY) {
                    uint64_t v[4], Sq;
                    quad_values(r, v, Sq);
                    if (!quad_roots_ok(v, r)) record_verify_failure(a, S, v);
                }
                if (a.flags & PS4_F_DUMP4) dump_quad(a, r);
                if (store) {
                    if (!RING) {
                        put_job(a.jobs, out + n, r, item);
                    } else if (ring_wait_free(a, out + n)) {
                        put_job(a.jobs, (out + n) & a.ring_mask, r, item);
                    }
                }
            }
            n++;
        }
    }
    return n;
}

// A lane's share of P5: the pairs g = gw + lane, gw + lane + 32, ... below ge of its warp's
// contiguous block.  Neighbouring lanes take neighbouring pairs (mostly the same S), and each
// lane finds its pair's S by one binary search, then by stepping forward.
template <bool WRITE, bool RING = false>
__device__ __forceinline__ uint32_t lane_pairs(const SearchArgs &a, uint32_t gw, uint32_t ge, int lane, uint32_t nI,
                                               const uint16_t *is_off, const uint16_t *is_k,
                                               const uint16_t *is_start, const uint32_t *is_pbase,
                                               const uint32_t *rep_p, const uint32_t *rep_q, uint64_t S0,
                                               uint32_t item, uint64_t out, bool store) {
    uint32_t g = gw + (uint32_t)lane;
    if (g >= ge) return 0;
    uint32_t lo = 0, hi = nI;
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (is_pbase[mid] <= g) lo = mid; else hi = mid;
    }
    uint32_t n = 0;
    for (; g < ge; g += 32) {
        while (lo + 1 < nI && is_pbase[lo + 1] <= g) lo++;
        uint32_t x, y;
        decode_pair(g - is_pbase[lo], x, y);
        n += pair_quads<WRITE, RING>(a, is_start[lo], is_k[lo], S0 + is_off[lo], x, y, rep_p, rep_q, item, out + n,
                                     store);
    }
    return n;
}

// One claimed group of tiles, the last-but-c0 SUPER_K tiles of the launch (tiles are taken from
// the last one down, costliest first): per segment of the group one scan for all its tiles (when
// `lists` is given), then per tile P1-P4, the count pass, one reservation for the tile's
// 4-sets, the write pass.  NT threads.  RING: the 4-sets go to the persistent kernel's ring and
// each lane publishes its contiguous run after a fence.  Returns the number of tiles.
template <int TL, int NT, bool RING>
__device__ uint32_t produce_group(const SearchArgs &a, TileShared &ts, unsigned char *smem, uint64_t c0,
                                  uint64_t *lists, uint32_t *raw_n, uint32_t slice, unsigned long long &s_base,
                                  int &s_store) {
    using L = TileLayout<TL>;
    constexpr int NW = NT / 32;
    const int tid = threadIdx.x;
    const bool noext = (a.flags & PS4_F_NOEXT) != 0;
    const bool need_write_pass = !noext || (a.flags & (PS4_F_DUMP4 | PS4_F_VERIFY));
    const uint64_t cn = min((uint64_t)SUPER_K, a.n_tiles - c0);
    uint64_t ti = a.n_tiles - c0 - cn;
    const uint64_t ti_end = a.n_tiles - c0;
    while (ti < ti_end) {
        // a group: the claimed tiles of one segment, one scan for all of them
        uint32_t lo = 0, hi = a.n_items;
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (a.items[mid].tile_base <= ti) lo = mid; else hi = mid;
        }
        const Item it = a.items[lo];
        const uint64_t seg_tiles = (it.hi - it.lo + (1ull << TL) - 1) >> TL;
        const uint64_t g_end = min(ti_end, it.tile_base + seg_tiles);
        const uint32_t ng = (uint32_t)(g_end - ti);
        const uint64_t SA = it.lo + ((ti - it.tile_base) << TL);
        const uint64_t SB = min(it.hi, SA + ((uint64_t)ng << TL));
        const uint32_t item = it.id;
        const bool grouped = lists != nullptr;
        if (grouped) {
            if (tid < SUPER_K * NW) raw_n[tid] = 0;
            __syncthreads();
            scan_group<NT>(SA, SB, TL, lists, a.raw_cap, raw_n, slice);
            __syncthreads();
        }
        for (uint32_t j = 0; j < ng; j++) {
            tile_reset(ts);
            __syncthreads();
            const uint64_t S0 = SA + ((uint64_t)j << TL);
            const uint32_t n = (uint32_t)min((uint64_t)L::W, SB - S0);
            bool use_list = grouped;
            for (int w = 0; w < NW; w++) use_list = use_list && raw_n[j * NW + w] <= slice;
            if (!tile_reps<TL, NT>(a, ts, smem, S0, n, use_list ? lists + (size_t)j * a.raw_cap : nullptr,
                                   &raw_n[j * NW], slice)) { __syncthreads(); continue; }
            const uint16_t *is_off = (const uint16_t *)(smem + L::OFF_IS_OFF);
            const uint16_t *is_k = (const uint16_t *)(smem + L::OFF_IS_K);
            const uint16_t *is_start = (const uint16_t *)(smem + L::OFF_IS_START);
            const uint32_t *is_pbase = (const uint32_t *)(smem + L::OFF_IS_PBASE);
            const uint32_t *rep_p = (const uint32_t *)(smem + L::OFF_REP_P);
            const uint32_t *rep_q = (const uint32_t *)(smem + L::OFF_REP_Q);
            const uint32_t nI = ts.n_is, nPairs = ts.n_pairs;
            // count pass, one reservation for the tile, write pass in the same order
            // each warp a contiguous block of pairs (whole multiples of 32)
            const int lane = tid & 31, wid = tid >> 5;
            const uint32_t blk = ((nPairs + NW * 32 - 1) / (NW * 32)) * 32;
            const uint32_t gw = (uint32_t)wid * blk, ge = min(nPairs, gw + blk);
            uint32_t mine = lane_pairs<false>(a, gw, ge, lane, nI, is_off, is_k, is_start, is_pbase, rep_p, rep_q, S0,
                                              item, 0, false);
            uint32_t off, d1, d2, tot[3];
            block_scan3<NT>(mine, 0u, 0u, off, d1, d2, tot, ts.wsum);
            if (tid == 0) {
                ts.cnt[K_SETS4] += tot[0];
                s_base = 0;
                s_store = 0;
                if (!noext && tot[0]) {
                    if (RING) {
                        // room: the ring holds the reserved-but-unfinished 4-sets plus this tile's
                        WaitClock wc;
                        bool ok = true;
                        while (ld_vol(&a.status->q_tail) + tot[0] - ld_vol(&a.status->q_freed) > a.jobs_cap) {
                            if (ld_vol(&a.status->err) != 0ull || wc.expired(a, 3)) { ok = false; break; }
                            __nanosleep(256);
                        }
                        if (ok) {
                            s_base = atomicAdd(&a.status->q_tail, (ull)tot[0]);
                            s_store = 1;
                        }
                    } else {
                        s_base = atomicAdd(&a.status->n_jobs, (ull)tot[0]);
                        if (s_base + tot[0] <= a.jobs_cap) s_store = 1;
                        else raise_capacity(a.status, E_QUEUE, 5, s_base + tot[0], a.jobs_cap, S0);
                    }
                }
            }
            __syncthreads();
            if (need_write_pass) {
                const bool store = s_store != 0;
                lane_pairs<true, RING>(a, gw, ge, lane, nI, is_off, is_k, is_start, is_pbase, rep_p, rep_q, S0, item,
                                       s_base + off, store);
                if (RING && store && mine) {       // publish this lane's run [s_base+off, +mine)
                    __threadfence();
                    for (uint32_t i = 0; i < mine; i++) {
                        const uint64_t pos = s_base + off + i;
                        *(volatile uint32_t *)&a.seq[pos & a.ring_mask] = (uint32_t)(pos + 1);
                    }
                }
            }
            __syncthreads();
            if (RING && tid == 0 && s_store && tot[0]) atomicAdd(&a.status->q_pub, (ull)tot[0]);
            tile_flush_counters(a, ts, item);
            __syncthreads();
        }
        ti = g_end;
    }
    return (uint32_t)cn;
}

template <int TL, int NT>
__global__ void __launch_bounds__(NT, BS / NT * 2) gen_jobs(const SearchArgs a) {
    using L = TileLayout<TL>;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ TileShared ts;
    __shared__ unsigned long long s_base;
    __shared__ int s_store;
    __shared__ unsigned long long s_claim;
    const int tid = threadIdx.x;
    uint64_t *lists = a.raw ? a.raw + (size_t)blockIdx.x * SUPER_K * a.raw_cap : nullptr;
    // per tile of a group and warp: representations appended to the tile's list; in the tile
    // layout's extension-list area, which this kernel does not use otherwise
    uint32_t *raw_n = (uint32_t *)(smem + L::OFF_ELIST);
    const uint32_t slice = a.raw ? a.raw_cap / (NT / 32) : 0;
    for (;;) {
        // claim SUPER_K tiles; tiles are taken from the last one down (costliest first)
        if (tid == 0) {
            s_claim = atomicAdd(&a.status->tile_next, SUPER_K);
            ts.skip = *(volatile ull *)&a.status->err != 0ull;
        }
        __syncthreads();
        const uint64_t c0 = s_claim;
        const bool stop = c0 >= a.n_tiles || ts.skip;
        __syncthreads();                                                 // s_claim read by all
        if (stop) break;                                                 // block-uniform
        produce_group<TL, NT, false>(a, ts, smem, c0, lists, raw_n, slice, s_base, s_store);
    }
}

// ================================================================== extend_jobs

constexpr int EBS = 256;                 // threads per CTA
constexpr int EWARPS = EBS / 32;
constexpr int DCAP = 416;                // divisor-list entries per warp (u64)
constexpr int QCAP = 64;                 // square-test queue per warp
constexpr int EXCAP = 8;                 // extensions per warp and round
constexpr int FSLOT = 16;                // prime slots per lane: m1's primes from 0, m2's from 8

// The odd part D_odd of a difference is kept factored: its odd primes are split into a low
// group (the first primes of the reference's order) and a high group, with divisor lists
// lo[0..L) and hi[0..H) in mixed-radix order.  The odd divisor with mixed-radix index
// t = l + L*h is lo[l]*hi[h], and its complement (index ndo-1-t) is lo[L-1-l]*hi[H-1-h]:
// L+H entries instead of ndo = L*H.
struct __align__(16) EJob {              // one lane's 4-set, read by every lane in phase B
    uint64_t m64, m63, m65;              // bit s: u^2 + (C - A) is a residue for both C (mod 64/63/65)
    uint32_t rA0, rA1;                   // rA0..rA2: the roots sqrt(A + v) of the three other members
    uint32_t uA, rAA, rA2, ncand;        // u <= uA: e <= 0; rAA = sqrt(2A) if integral, else 0;
                                         //   e = u^2 - A is a member of the 4-set iff u is one of
                                         //   rAA, rA0, rA1, rA2
    uint16_t base, L, H;                 // lo list at dbuf[base..base+L), hi list right after it
    uint8_t E2, flags;                   // flags: 1 = D even
    uint64_t A;                          // extend by D = A - B
    uint64_t C1, C2;                     // the other two members (square tests)
};

struct WarpArea {
    uint64_t dbuf[DCAP];
    EJob job[32];
    uint32_t cstart[33];
    uint32_t qidx[QCAP];                 // candidate: l | h << 12 | d2 << 24
    uint64_t qu[QCAP];
    uint8_t qj[QCAP];
    ExtEntry ext[EXCAP];
    uint32_t fp[FSLOT][32];              // each lane's primes of D with their exponents (p | e << 24),
                                         //   lane-minor (no bank conflicts)
    uint32_t jsq[32];                    // ext_sqrt of each lane's 4-set in this round
    uint32_t jid[32];                    // queue index of each lane's 4-set
    uint32_t n_ext;
};

static_assert(EWARPS * sizeof(WarpArea) + 1024 <= 228 * 1024 / 3, "three engine CTAs per SM");

// Residue masks indexed by u's residue: bit w of q_m[a] is set iff w^2 + a is a square mod m.
// A 4-set's mask for its two remaining members C1, C2 is q_m[(C1-A) mod m] & q_m[(C2-A) mod m],
// so the filters of e + C = u^2 + (C - A) (s4.c:192-194) become one bit test per modulus on
// u mod m.  Mod 65 has 65 residues, but 64 = -1 and 1 have the same square, so bit 64 equals
// bit 1 and residue 64 is looked up as 1.
struct UResTabs {
    uint64_t q64[64], q63[63], q65[65];
};
constexpr bool is_qr_mod(int m, int r) {
    return r < 64 ? ((qr_bits(m) >> r) & 1) != 0 : true;          // r = 64 (m = 65) is 8^2
}
constexpr UResTabs make_ures() {
    UResTabs t{};
    for (int a = 0; a < 64; a++) {
        uint64_t x = 0;
        for (int w = 0; w < 64; w++) if (is_qr_mod(64, (w * w + a) % 64)) x |= 1ull << w;
        t.q64[a] = x;
    }
    for (int a = 0; a < 63; a++) {
        uint64_t x = 0;
        for (int w = 0; w < 63; w++) if (is_qr_mod(63, (w * w + a) % 63)) x |= 1ull << w;
        t.q63[a] = x;
    }
    for (int a = 0; a < 65; a++) {
        uint64_t x = 0;
        for (int w = 0; w < 64; w++) if (is_qr_mod(65, (w * w + a) % 65)) x |= 1ull << w;
        t.q65[a] = x;
    }
    return t;
}
__device__ const UResTabs UQ = make_ures();

// (d mod 63, d mod 65) for |d| < 2^48, by folding 24-bit halves (2^24 = 1 mod 63 and mod 65)
__device__ __forceinline__ void res6365(int64_t d, uint32_t &r63, uint32_t &r65) {
    const uint64_t x = d < 0 ? (uint64_t)(-d) : (uint64_t)d;
    const uint32_t r = (uint32_t)(x >> 24) + (uint32_t)(x & 0xFFFFFFu);
    r63 = r % 63u;
    r65 = r % 65u;
    if (d < 0) { r63 = r63 ? 63u - r63 : 0u; r65 = r65 ? 65u - r65 : 0u; }
}

// One lane's counters for the item of the 4-set it is working on, added to that item's
// counter block whenever the item changes (queries of a batch are separate items).
struct LaneCounters {
    uint32_t item = 0xFFFFFFFFu;
    ull cand = 0, sqrt_ = 0;
    uint32_t mdiv = 0;
    __device__ __forceinline__ void flush(const SearchArgs &a) {
        if (item != 0xFFFFFFFFu) {
            ull *k = a.counters + (size_t)item * K_SLOTS;
            if (cand) atomicAdd(&k[K_EXT_CAND], cand);
            if (sqrt_) atomicAdd(&k[K_EXT_SQRT], sqrt_);
            if (mdiv) atomicMax(&k[K_MAX_DIVS], (ull)mdiv);
        }
        cand = 0; sqrt_ = 0; mdiv = 0;
    }
    __device__ __forceinline__ void use(const SearchArgs &a, uint32_t it) {
        if (it != item) { flush(a); item = it; }
    }
};

// Report the extensions of one warp round: group them per 4-set, emit hit / ext / six
// records and the counters sets5 / multi / sets6 / hist5 / max_extensions (s4.c:243-277).
template <bool COH>
static __device__ void report_warp_exts(const SearchArgs &a, ExtEntry *el, uint32_t n) {
    for (uint32_t x = 1; x < n; x++) {
        ExtEntry k = el[x];
        uint32_t y = x;
        while (y > 0 && (el[y - 1].qid > k.qid || (el[y - 1].qid == k.qid && el[y - 1].key > k.key))) {
            el[y] = el[y - 1];
            y--;
        }
        el[y] = k;
    }
    for (uint32_t g0 = 0; g0 < n;) {
        uint32_t g1 = g0 + 1;
        while (g1 < n && el[g1].qid == el[g0].qid) g1++;
        const uint32_t ne = g1 - g0;
        uint32_t roots[6], item;                              // the 4-set and its item, from the queue
        get_job<COH>(a.jobs, el[g0].qid, roots, item);
        ull *cnt = a.counters + (size_t)item * K_SLOTS;
        uint64_t v[4], S;
        quad_values(roots, v, S);
        if (ne > a.cap_ext) { raise_error(a.status, E_CAP_EXT, S); g0 = g1; continue; }
        atomicMax(&cnt[K_MAX_EXT], (ull)ne);
        uint64_t vmax = v[0];
        for (int i = 1; i < 4; i++) vmax = v[i] > vmax ? v[i] : vmax;
        bool prints = ne >= 2;
        for (uint32_t t = 0; t < ne; t++) prints |= (el[g0 + t].hi != 0 || el[g0 + t].lo > vmax);
        uint32_t hslot = 0, eslot = 0;
        if (prints) {
            hslot = atomicAdd(&a.status->n_hits, 1u);
            eslot = atomicAdd(&a.status->n_exts, ne);
        }
        uint32_t hflags = 0;
        if (ne >= 2) {
            hflags |= PS4_HIT_MULTI;
            atomicAdd(&cnt[K_MULTI], 1ull);
            u128 x[6] = {v[0], v[1], v[2], v[3], ((u128)el[g0].hi << 64) | el[g0].lo,
                         ((u128)el[g0 + 1].hi << 64) | el[g0 + 1].lo};
            if (verify_set(x, 6)) hflags |= PS4_HIT_DRILL_OK;
        }
        for (uint32_t t = 0; t < ne; t++) {
            const u128 e = ((u128)el[g0 + t].hi << 64) | el[g0 + t].lo;
            uint32_t ef = 0;
            if (e > vmax) {
                ef |= PS4_EXT_FIVE;
                atomicAdd(&cnt[K_SETS5], 1ull);
                int lg = 0;
                for (u128 z = e; z > 1; z >>= 1) lg++;
                atomicAdd(&cnt[K_HIST5 + (lg > 99 ? 99 : lg)], 1ull);
                u128 x[5] = {v[0], v[1], v[2], v[3], e};
                if (verify_set(x, 5)) ef |= PS4_EXT_FIVE_OK;
            }
            if (prints && eslot + t < a.exts_cap) {
                ps4_ext rec;
                rec.lo = el[g0 + t].lo; rec.hi = el[g0 + t].hi; rec.key = el[g0 + t].key; rec.flags = ef;
                a.exts[eslot + t] = rec;
            }
        }
        for (uint32_t t = 0; t < ne; t++)
            for (uint32_t s = t + 1; s < ne; s++) {
                const u128 et = ((u128)el[g0 + t].hi << 64) | el[g0 + t].lo;
                const u128 es = ((u128)el[g0 + s].hi << 64) | el[g0 + s].lo;
                if (!is_square_exact(et + es)) continue;
                atomicAdd(&cnt[K_SETS6], 1ull);
                u128 x[6] = {v[0], v[1], v[2], v[3], et, es};
                const uint32_t sslot = atomicAdd(&a.status->n_sixes, 1u);
                if (sslot < a.sixes_cap) {
                    ps4_six rec;
                    rec.hit = hslot; rec.t = t; rec.s = s; rec.flags = verify_set(x, 6) ? 1u : 0u;
                    a.sixes[sslot] = rec;
                }
            }
        if (prints && hslot < a.hits_cap) {
            ps4_hit h;
            h.S = S;
            for (int i = 0; i < 4; i++) h.v[i] = v[i];
            h.n_ext = ne; h.first_ext = eslot; h.flags = hflags; h.item = item;
            h.order[0] = roots[5]; h.order[1] = roots[4];
            h.order[2] = roots[2] < roots[3] ? roots[2] : roots[3];
            h.order[3] = roots[2] < roots[3] ? 1u : 0u;
            a.hits[hslot] = h;
        }
        g0 = g1;
    }
}

// Phase A state of one lane: its 4-set, the difference to extend by and its factorisation.
struct LaneJob {
    uint32_t r[6], item;
    uint64_t v[4], S, A, C1, C2;
    int bi, bj, bk;
    int np;                              // distinct primes, in w->fp[0..np)[lane]
    bool has2;
    int E2, j0, js;                      // odd primes are pr[j0..np); the high group starts at js
    uint32_t ndo, nd, ncand, L, H;
};

// Factor D = m1*m2 (m1 = ra-rb, m2 = ra+rb, both < 2^23, of equal parity).  The power of two
// comes from counting trailing zeros; each odd part's first three primes come in one 16-byte
// load (fac3), and the rare cofactor left over is walked through spfq (one table load per
// distinct prime), both walks interleaved so that their dependent loads overlap.  Without fac3
// (null) every prime is walked through spfq.  m1's primes are stored from slot 0, m2's from
// slot 8 (each has at most 7 distinct odd primes), then m2's are merged into m1's list --
// primes in first-seen order, as s4.c:141-147.  A new prime is written to a slot below every
// unread slot of m2, so the merge is in place.
__device__ __forceinline__ int factor_pair(const uint64_t *spfq, const uint4 *fac3, uint32_t m1, uint32_t m2,
                                           uint32_t (*fp)[32], int lane) {
    int na = 0, nb = 0;
    if (m1 > 1 && !(m1 & 1)) {                      // both even
        const uint32_t z1 = (uint32_t)__ffs((int)m1) - 1, z2 = (uint32_t)__ffs((int)m2) - 1;
        fp[0][lane] = 2u | ((z1 + z2) << 24);
        na = 1;
        m1 >>= z1;
        m2 >>= z2;
    }
    if (fac3) {
        const uint4 fa = m1 > 1 ? __ldg(&fac3[m1]) : make_uint4(0, 0, 0, 1);
        const uint4 fb = m2 > 1 ? __ldg(&fac3[m2]) : make_uint4(0, 0, 0, 1);
        if (fa.x) fp[na++][lane] = fa.x;
        if (fa.y) fp[na++][lane] = fa.y;
        if (fa.z) fp[na++][lane] = fa.z;
        if (fb.x) fp[8 + nb++][lane] = fb.x;
        if (fb.y) fp[8 + nb++][lane] = fb.y;
        if (fb.z) fp[8 + nb++][lane] = fb.z;
        m1 = fa.w;
        m2 = fb.w;
    }
    uint64_t sa = m1 > 1 ? __ldg(&spfq[m1]) : 0, sb = m2 > 1 ? __ldg(&spfq[m2]) : 0;
    while (m1 > 1 || m2 > 1) {
        if (m1 > 1) {
            fp[na][lane] = (uint32_t)sa;                   // p | e << 24, as the table stores it
            na++;
            m1 = spf_cof(sa);
            if (m1 > 1) sa = __ldg(&spfq[m1]);
        }
        if (m2 > 1) {
            fp[8 + nb][lane] = (uint32_t)sb;
            nb++;
            m2 = spf_cof(sb);
            if (m2 > 1) sb = __ldg(&spfq[m2]);
        }
    }
    int np = na;
    for (int j = 0; j < nb; j++) {
        const uint32_t x = fp[8 + j][lane], p = x & 0xFFFFFFu;
        int i = 0;
        while (i < na && (fp[i][lane] & 0xFFFFFFu) != p) i++;
        if (i < na) fp[i][lane] += x & 0xFF000000u;
        else { fp[np][lane] = x; np++; }
    }
    return np;
}

template <bool COH>
__device__ __forceinline__ bool job_setup(const SearchArgs &a, uint64_t j, LaneJob &J, uint32_t (*fp)[32],
                                          int lane) {
    get_job<COH>(a.jobs, j, J.r, J.item);
    quad_values(J.r, J.v, J.S);
    uint32_t best;
    choose_pair(J.v, J.r, a.ndiv, J.bi, J.bj, J.bk, best);
    const uint32_t ra = pick6(J.r, pair_slot(J.bi, J.bk)), rb = pick6(J.r, pair_slot(J.bj, J.bk));
    J.A = pick4(J.v, J.bi);
    int o1 = -1, o2 = -1;
#pragma unroll
    for (int t = 0; t < 4; t++)
        if (t != J.bi && t != J.bj) { if (o1 < 0) o1 = t; else o2 = t; }
    J.C1 = pick4(J.v, o1);
    J.C2 = pick4(J.v, o2);
    J.np = factor_pair(a.spfq, a.fac3, ra - rb, ra + rb, fp, lane);
    // D even => both factors even => 2 is the first prime and 4 | D
    J.has2 = J.np > 0 && (fp[0][lane] & 0xFFFFFFu) == 2;
    J.E2 = J.has2 ? fp[0][lane] >> 24 : 0;
    J.j0 = J.has2 ? 1 : 0;
    uint32_t ndo = 1;
    for (int q = J.j0; q < J.np; q++) ndo *= (fp[q][lane] >> 24) + 1;
    J.ndo = ndo;
    // low group: the leading odd primes while their radix product stays <= sqrt(ndo)
    uint32_t L = 1, js = J.j0;
    while (js < J.np && L * ((fp[js][lane] >> 24) + 1) * L * ((fp[js][lane] >> 24) + 1) <= ndo)
        L *= (fp[js++][lane] >> 24) + 1;
    J.js = js;
    J.L = L;
    J.H = ndo / L;
    const uint64_t nd = (uint64_t)ndo * (uint64_t)(J.E2 + 1);
    J.nd = (uint32_t)nd;
    // same-parity complementary pairs with f < g: the reference's ext_cand (s4.c:191)
    J.ncand = J.has2 ? (uint32_t)(((uint64_t)(J.E2 - 1) * ndo) >> 1) : (uint32_t)(nd >> 1);
    if (nd > a.cap_divs) { raise_error(a.status, E_CAP_DIVS, J.S); return false; }
    return true;
}

// The n divisors of prod pr[q]^ex[q], q in [q0, q1), in mixed-radix order (first prime
// fastest), in one flat loop: prime q's block repeats the list so far ex[q] times, each copy
// times p_q, so d[j] = d[j - cur] * p_q with cur the list length before q.
__device__ __forceinline__ void gen_list(uint64_t *d, const uint32_t (*fp)[32], int lane,
                                         int q0, uint32_t n) {
    d[0] = 1;
    if (n <= 1) return;
    int q = q0;
    uint32_t x = fp[q][lane];
    uint32_t p = x & 0xFFFFFFu, cur = 1, end = (x >> 24) + 1;
    for (uint32_t j = 1; j < n; j++) {
        if (j == end) {
            cur = end;
            x = fp[++q][lane];
            p = x & 0xFFFFFFu;
            end = cur * ((x >> 24) + 1);
        }
        d[j] = d[j - cur] * p;
    }
}

// A 4-set whose factored divisor lists exceed the warp buffer: the per-lane divisor walk.
static __device__ __noinline__ void extend_big(const SearchArgs &a, const LaneJob &J, uint32_t qid, ull &cand,
                                               ull &sq, ExtEntry *el, uint32_t *el_n) {
    uint32_t md = 0;
    extend_quad(a, J.r, J.v, J.S, J.bi, J.bj, J.bk, qid, cand, sq, md, el, el_n, EXCAP);
}

// Square tests of queue entries [first, first+count), one per lane (s4.c:199-203); a hit
// gets its order key, the reference's mixed-radix index of the smaller divisor.
__device__ __forceinline__ void process_queue(const SearchArgs &a, WarpArea *w, uint32_t first, uint32_t count,
                                              int lane) {
    if ((uint32_t)lane < count) {
        const uint32_t idx = first + lane;
        const uint64_t u = w->qu[idx];
        const uint32_t jl = w->qj[idx];
        const EJob &J = w->job[jl];
        const u128 e = (u128)u * u - J.A;
        // is_square_fast needs n < 2^100: u = (f+g)/2 <= (D+1)/2 < 2^44 and C < S < 2^44, so
        // e + C < u^2 + C < 2^89
        if (is_square_fast(e + J.C1) && is_square_fast(e + J.C2)) {
            const uint32_t c = w->qidx[idx], l = c & 0xFFFu, h = (c >> 12) & 0xFFFu, d2 = c >> 24;
            const uint64_t fo = w->dbuf[J.base + l] * w->dbuf[J.base + J.L + h];
            const uint64_t go = w->dbuf[J.base + J.L - 1 - l] * w->dbuf[J.base + J.L + J.H - 1 - h];
            const uint32_t to = l + J.L * h;
            const uint32_t t = (J.flags & 1) ? d2 + (J.E2 + 1u) * to : to;
            const uint32_t nd = (uint32_t)J.L * J.H * ((J.flags & 1) ? J.E2 + 1u : 1u);
            const uint32_t key = (fo << d2) < (go << (J.E2 - d2)) ? t : nd - 1 - t;
            const uint32_t slot = atomicAdd(&w->n_ext, 1u);
            if (slot < EXCAP) {
                ExtEntry &x = w->ext[slot];
                x.qid = w->jid[jl];
                x.key = key;
                x.lo = (uint64_t)e;
                x.hi = (uint64_t)(e >> 64);
            } else {
                raise_capacity(a.status, E_EXTLIST, 4, slot + 1, EXCAP, 0);
            }
        }
    }
}

// The engine loop of one warp.  Linear (RING false): the batch's queue [0, njobs), filled before
// the launch; the loop ends when it is drained.  RING: the persistent kernel's ring; positions are
// claimed below q_tail and waited for until published, each finished 4-set's slot is handed back
// after the round's report, and the loop ends when a claim finds the ring empty and no lane holds
// a 4-set.  Returns whether the warp took any 4-set.
template <bool RING>
__device__ __forceinline__ bool engine_loop(const SearchArgs &a, WarpArea *w, int lane, uint64_t njobs) {
    const unsigned FULL = 0xffffffffu;
    if (lane == 0) w->n_ext = 0;
    w->jsq[lane] = 0;
    __syncwarp();
    LaneCounters cnt;
    LaneJob J;
    bool pending = false, old = false, drained = false, rel = false, took = false;
    uint32_t myjob = 0;
    uint64_t mypos = 0;

    // Rolling rounds: before each round every lane without a 4-set takes the next one from the
    // queue (phase A), so every round runs with a full warp of 4-sets; a lane whose divisor
    // lists did not fit keeps its 4-set and goes first in the next round's placement.
    for (;;) {
        if (!drained) {
            const bool need = !pending;
            const unsigned m = __ballot_sync(FULL, need);
            uint64_t base = 0;
            uint32_t got = 0;
            int stop = 0;
            if (RING) {
                if (lane == 0) {
                    if (m) base = ring_claim(a, (uint32_t)__popc(m), &got);
                    stop = *(volatile ull *)&a.status->err != 0ull;
                }
                base = __shfl_sync(FULL, base, 0);
            } else {
                uint32_t b32 = 0;                  // the batch queue's counter is 32-bit
                if (lane == 0) {
                    if (m) b32 = atomicAdd(&a.status->ext_next, (uint32_t)__popc(m));
                    stop = *(volatile ull *)&a.status->err != 0ull;
                }
                base = __shfl_sync(FULL, b32, 0);
            }
            stop = __shfl_sync(FULL, stop, 0);
            if (stop) break;                                             // warp-uniform
            if (RING) {
                got = __shfl_sync(FULL, got, 0);
                if (got < (uint32_t)__popc(m)) drained = true;           // the ring is empty for now
            } else if (base + __popc(m) >= njobs) {
                drained = true;                                          // warp-uniform
            }
            if (need) {
                const uint32_t rank = __popc(m & ((1u << lane) - 1u));
                const uint64_t jidx = base + rank;
                bool have = RING ? rank < got : jidx < njobs;
                if (RING && have) {
                    have = ring_wait_ready(a, jidx);
                    mypos = jidx;
                }
                if (have) {
                    myjob = (uint32_t)(RING ? (jidx & a.ring_mask) : jidx);
                    old = false;
                    took = true;
                    // ---- phase A: one 4-set per lane
                    pending = job_setup<RING>(a, myjob, J, w->fp, lane);
                    const bool big = pending && J.L + J.H > (uint32_t)DCAP;
                    if (pending) {
                        cnt.use(a, J.item);
                        if (J.nd > cnt.mdiv) cnt.mdiv = J.nd;
                        if (!big) cnt.cand += J.ncand;
                    }
                    if (big) {               // extremely rare: its factored lists exceed the buffer
                        extend_big(a, J, myjob, cnt.cand, cnt.sqrt_, w->ext, &w->n_ext);
                        pending = false;
                    }
                    if (RING && !pending) rel = true;                  // done in phase A: freed after the report
                }
            }
        }
        const bool round = __any_sync(FULL, pending);
        if (round) {
            // place the factored divisor lists of as many pending lanes as fit: lanes left over
            // from the last round first, then the new ones, each in lane order
            const uint32_t want = pending ? J.L + J.H : 0;
            uint32_t io = old ? want : 0, in = old ? 0 : want;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t yo = __shfl_up_sync(FULL, io, o), yn = __shfl_up_sync(FULL, in, o);
                if (lane >= o) { io += yo; in += yn; }
            }
            const uint32_t tot_old = __shfl_sync(FULL, io, 31);           // every lane takes part
            const uint32_t incl = old ? io : tot_old + in;
            const uint32_t base = incl - want;
            const bool fits = pending && incl <= (uint32_t)DCAP;
            if (fits) w->jid[lane] = myjob;
            if (fits) {
                gen_list(w->dbuf + base, w->fp, lane, J.j0, J.L);               // lo: L entries
                gen_list(w->dbuf + base + J.L, w->fp, lane, J.js, J.H);         // hi: H entries
                EJob &E = w->job[lane];
                E.A = J.A; E.C1 = J.C1; E.C2 = J.C2;
                const int64_t dd1 = (int64_t)J.C1 - (int64_t)J.A, dd2 = (int64_t)J.C2 - (int64_t)J.A;
                uint32_t a63, a65, b63, b65;
                res6365(dd1, a63, a65);
                res6365(dd2, b63, b65);
                E.m64 = UQ.q64[(uint32_t)dd1 & 63u] & UQ.q64[(uint32_t)dd2 & 63u];
                E.m63 = UQ.q63[a63] & UQ.q63[b63];
                E.m65 = UQ.q65[a65] & UQ.q65[b65];
                E.uA = isqrt_lt2p46(J.A);                        // < 2^22 (A < 2^44)
                const uint32_t r2A = isqrt_lt2p46(2 * J.A);      // < 2^23
                E.rAA = (uint64_t)r2A * r2A == 2 * J.A ? r2A : 0u;
                // the three roots through A, r[pair_slot(bi, x)]^2 = A + v_x (the member test takes
                // them as a set): slots 0,1,2 through index 0; 0,3,4 through 1; 1,3,5 through 2;
                // 2,4,5 through 3
                const int bi = J.bi;
                E.rA0 = bi <= 1 ? J.r[0] : (bi == 2 ? J.r[1] : J.r[2]);
                E.rA1 = bi == 0 ? J.r[1] : (bi == 3 ? J.r[4] : J.r[3]);
                E.rA2 = bi == 0 ? J.r[2] : (bi == 1 ? J.r[4] : J.r[5]);
                E.ncand = J.ncand;
                E.base = (uint16_t)base; E.L = (uint16_t)J.L; E.H = (uint16_t)J.H;
                E.E2 = (uint8_t)J.E2;
                E.flags = (uint8_t)(J.has2 ? 1 : 0);
            }
            // ---- phase B: the pooled candidates, 32 equal contiguous runs
            const uint32_t nc = fits ? J.ncand : 0;
            const unsigned nonempty = __ballot_sync(FULL, nc != 0);          // jobs with candidates
            uint32_t ci = nc;
#pragma unroll
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t y = __shfl_up_sync(FULL, ci, o);
                if (lane >= o) ci += y;
            }
            w->cstart[lane] = ci - nc;
            const uint32_t C = __shfl_sync(FULL, ci, 31);
            if (lane == 31) w->cstart[32] = C;
            __syncwarp();
            const uint32_t g0 = (uint32_t)(((uint64_t)lane * C) >> 5);
            const uint32_t g1 = (uint32_t)(((uint64_t)(lane + 1) * C) >> 5);
            const uint32_t iters = (C + 31) >> 5;
            uint32_t jl = 0;
            {
                uint32_t lo = 0, hi = 32;                 // last job with cstart <= g0
                while (hi - lo > 1) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (w->cstart[mid] <= g0) lo = mid; else hi = mid;
                }
                jl = lo;
            }
            // the current job of this lane's run, in registers
            uint64_t m64 = 0, m63 = 0, m65 = 0, hv = 0, hc = 0;
            uint32_t uA = 0, rAA = 0, rA0 = 0, rA1 = 0, rA2 = 0;
            uint32_t ncand = 0, jb = 0, L = 1, H = 1, E2 = 0, flg = 0, R = 1, dlo = 0, dhi = 0;
            uint32_t cc = 0, l = 0, h = 0, d2 = 0;
            // hv/hc are reloaded only for a new row h or a new job: the loads of the lanes that keep
            // their row are predicated off, so fewer divisor-buffer wavefronts (engine -1.8 % per
            // [1,1e10) step; the same for the lo values, which change every candidate of odd D, +3 %)
            bool hre = true;
            // job fields in four vector loads; entering a job at its first candidate needs no division
            auto load_job = [&](uint32_t j) {
                const ulonglong2 x0 = *(const ulonglong2 *)&w->job[j].m64;
                const ulonglong2 x1 = *(const ulonglong2 *)&w->job[j].m65;    // m65, rA0 | rA1 << 32
                const uint4 y = *(const uint4 *)&w->job[j].uA;
                const uint2 z = *(const uint2 *)&w->job[j].base;
                m64 = x0.x; m63 = x0.y; m65 = x1.x;
                rA0 = (uint32_t)x1.y; rA1 = (uint32_t)(x1.y >> 32);
                uA = y.x; rAA = y.y; rA2 = y.z; ncand = y.w;
                jb = z.x & 0xFFFFu; L = z.x >> 16; H = z.y & 0xFFFFu; E2 = (z.y >> 16) & 0xFFu; flg = z.y >> 24;
                R = (flg & 1) ? E2 - 1 : 1;
                dlo = flg & 1; dhi = (flg & 1) ? E2 - 1 : 0;      // 2-exponents of f: [1, E2-1] or {0}
                cc = 0; l = 0; h = 0; d2 = (flg & 1) ? 1u : 0u;
            };
            if (g0 < g1) {
                load_job(jl);
                const uint32_t cidx = g0 - w->cstart[jl];
                const uint32_t to = (flg & 1) ? cidx / R : cidx;
                d2 = (flg & 1) ? 1 + cidx % R : 0;
                h = to / L;
                l = to - h * L;
                cc = cidx;
            }
            uint32_t qn = 0, sq_run = 0;
            for (uint32_t it = 0; it < iters; it++) {
                bool pass = false;
                uint64_t u = 0;
                uint32_t cidx = 0, jcur = jl;              // the job of THIS candidate
                if (it < g1 - g0) {
                    if (hre) {
                        hv = w->dbuf[jb + L + h];
                        hc = w->dbuf[jb + L + H - 1 - h];
                    }
                    // f = 2^d2 * lo[l]*hi[h], g = 2^(E2-d2) * lo[L-1-l]*hi[H-1-h]: complementary divisors
                    const uint64_t fo = w->dbuf[jb + l] * hv, go = w->dbuf[jb + L - 1 - l] * hc;
                    u = ((fo << d2) + (go << (E2 - d2))) >> 1;
                    // e + C = u^2 + (C - A): residues mod 64, 63, 65 for both C (s4.c:192-194), as
                    // bits of the 4-set's u-indexed masks
                    const uint32_t w64 = (uint32_t)u & 63u;
                    const uint32_t rr = (uint32_t)(u >> 24) + ((uint32_t)u & 0xFFFFFFu);   // 2^24 = 1 mod 63, 65
                    const uint32_t w63 = rr % 63u, w65r = rr % 65u;
                    const uint32_t w65 = w65r == 64u ? 1u : w65r;     // 64^2 = 1^2 mod 65: same bit
                    // e = u^2 - A in v (s4.c:197) iff u^2 = A + v_i: u is one of the 4-set's roots
                    // through A (all below 2^23, so u's low word decides once u < 2^32)
                    const uint32_t ul = (uint32_t)u;
                    const bool member = (u >> 32) == 0 && (ul == rA0 || ul == rA1 || ul == rA2 || ul == rAA);
                    pass = ((m64 >> w64) & (m63 >> w63) & (m65 >> w65) & 1u) && u > uA && !member;
                    if (pass) { sq_run++; cidx = l | (h << 12) | (d2 << 24); }
                    // next candidate of this lane's run
                    {                                          // (l, h, d2) advance, branch-free
                        d2++;
                        const uint32_t wd = d2 > dhi ? 1u : 0u;
                        d2 = wd ? dlo : d2;
                        l += wd;
                        const uint32_t wl = l == L ? 1u : 0u;
                        l = wl ? 0u : l;
                        h += wl;
                        hre = wl != 0;
                    }
                    if (++cc == ncand && it + 1 < g1 - g0) {
                        if (sq_run) atomicAdd(&w->jsq[jl], sq_run);
                        sq_run = 0;
                        jl = min((uint32_t)__ffs(nonempty & (0xFFFFFFFEu << jl)) - 1u, 31u);
                        load_job(jl);
                        hre = true;
                    }
                }
                const unsigned m = __ballot_sync(FULL, pass);
                if (pass) {
                    const uint32_t pos = qn + __popc(m & ((1u << lane) - 1u));
                    w->qu[pos] = u;
                    w->qidx[pos] = cidx;
                    w->qj[pos] = (uint8_t)jcur;
                }
                qn += __popc(m);
                __syncwarp();
                if (qn >= 32) {
                    process_queue(a, w, qn - 32, 32, lane);
                    qn -= 32;
                    __syncwarp();
                }
            }
            if (sq_run) atomicAdd(&w->jsq[jl], sq_run);
            if (qn) process_queue(a, w, 0, qn, lane);
            __syncwarp();
            if (fits) {                        // this lane's 4-set is done: its ext_sqrt into its item
                cnt.use(a, J.item);
                cnt.sqrt_ += w->jsq[lane];
                w->jsq[lane] = 0;
                if (RING) rel = true;
            }
            pending = pending && !fits;
            old = pending;
        }
        __syncwarp();
        if (lane == 0 && w->n_ext) {          // this round's extensions (and any from the per-lane path)
            report_warp_exts<RING>(a, w->ext, min(w->n_ext, (uint32_t)EXCAP));
            w->n_ext = 0;
        }
        __syncwarp();
        if (RING) {                            // the round's finished 4-sets hand their slots back
            const unsigned rm = __ballot_sync(FULL, rel);
            if (rel) ring_release(a, mypos);
            rel = false;
            if (lane == 0 && rm) atomicAdd(&a.status->q_freed, (ull)__popc(rm));
        }
        if (!round && drained) break;          // warp-uniform
    }
    cnt.flush(a);
    return RING ? __any_sync(FULL, took) : false;
}

__global__ void __launch_bounds__(EBS, 3) extend_jobs(const SearchArgs a) {
    extern __shared__ __align__(16) unsigned char esmem[];
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    WarpArea *w = (WarpArea *)(esmem + (size_t)wid * sizeof(WarpArea));
    const uint64_t njobs = min(*(volatile ull *)&a.status->n_jobs, (ull)a.jobs_cap);
    engine_loop<false>(a, w, lane, njobs);
}

// ================================================================== the persistent kernel

// One launch for a whole call.  Every CTA (PBS threads, three per SM) loops over two roles:
// producing -- claim the next group of SUPER_K tiles of 2^13 S (highest cost first), run P1-P5
// and write the 4-sets into the ring -- or consuming -- its warps run the extension engine on
// 4-sets claimed from the ring.  A CTA consumes while at least CONSUME_AT 4-sets are queued,
// produces while tiles are left and the ring is less than half full, and ends when every tile is
// produced and every 4-set claimed.  The roles switch with hysteresis: a CTA turns to the engine
// when ring_high 4-sets are queued, and its warps keep claiming until fewer than ring_low are
// left (while tiles remain), so that every warp has 4-sets to pool, claims take the add path,
// and role changes are rare next to the work between them.  A call of any number of subranges is
// one launch.  The tile layout and the engine's warp areas share the CTA's shared memory (one
// role at a time).
constexpr int PTL = 13;
constexpr int PWARPS = PBS / 32;
// the tile state of the producing role sits in the dynamic area too, after the tile layout and
// the group's list counters, so that the kernel's static shared memory stays a few words and three
// CTAs (each with the 1 KB the hardware reserves per block) fit in the SM's 228 KB
constexpr size_t P_TS_OFF = (TileLayout<PTL>::OFF_ELIST + SUPER_K * PWARPS * sizeof(uint32_t) + 15) & ~(size_t)15;
static_assert(P_TS_OFF + sizeof(TileShared) <= PWARPS * sizeof(WarpArea),
              "the tile layout and tile state fit in the engine's warp areas");
static_assert(PWARPS * sizeof(WarpArea) + 1024 + 128 <= 228 * 1024 / 3, "three persistent CTAs per SM");

__global__ void __launch_bounds__(PBS, 3) search_persist(const SearchArgs a) {
    using L = TileLayout<PTL>;
    extern __shared__ __align__(16) unsigned char smem[];
    TileShared &ts = *reinterpret_cast<TileShared *>(smem + P_TS_OFF);
    __shared__ unsigned long long s_base, s_idle0;
    __shared__ unsigned int s_claim;
    __shared__ int s_store, s_role, s_busy;
    const int tid = threadIdx.x, lane = tid & 31, wid = tid >> 5;
    uint64_t *lists = a.raw ? a.raw + (size_t)blockIdx.x * SUPER_K * a.raw_cap : nullptr;
    uint32_t *raw_n = (uint32_t *)(smem + L::OFF_ELIST);
    const uint32_t slice = a.raw ? a.raw_cap / PWARPS : 0;
    if (tid == 0) s_idle0 = 0;
    for (;;) {
        if (tid == 0) {
            int role = 2;                                    // 0 end, 1 produce, 2 consume
            if (ld_vol(&a.status->err) != 0ull) {
                role = 0;
            } else {
                const ull tail = ld_vol(&a.status->q_tail), head = ld_vol(&a.status->q_head);
                const ull freed = ld_vol(&a.status->q_freed), pub = ld_vol(&a.status->q_pub);
                const uint32_t tn = ld_vol(&a.status->tile_next);
                const long long queued = (long long)(tail - head);
                if ((long long)(pub - head) >= (long long)a.ring_high || (tn >= a.n_tiles && queued > 0)) {
                    role = 2;
                } else if (tn < a.n_tiles && tail - freed < (a.jobs_cap >> 1)) {
                    const uint32_t c = atomicAdd(&a.status->tile_next, SUPER_K);
                    if (c < a.n_tiles) {
                        role = 1;
                        s_claim = c;
                    }
                } else if (tn >= a.n_tiles && ld_vol(&a.status->q_produced) >= a.n_tiles && queued <= 0) {
                    role = 0;
                }
            }
            s_role = role;
            s_busy = 0;
        }
        __syncthreads();
        const int role = s_role;
        if (role == 0) break;                                // block-uniform
        if (role == 1) {
            const uint32_t cn = produce_group<PTL, PBS, true>(a, ts, smem, s_claim, lists, raw_n, slice, s_base, s_store);
            if (tid == 0) {
                __threadfence();
                atomicAdd(&a.status->q_produced, (ull)cn);
                s_idle0 = 0;
            }
        } else {
            WarpArea *w = (WarpArea *)(smem + (size_t)wid * sizeof(WarpArea));
            if (engine_loop<true>(a, w, lane, 0) && lane == 0) s_busy = 1;
            __syncthreads();
            if (tid == 0) {
                if (s_busy) {
                    s_idle0 = 0;
                } else {                                     // nothing to take: wait a little, bounded
                    const uint64_t t = gtimer();
                    if (!s_idle0) s_idle0 = t;
                    else if (t - s_idle0 > 2 * WAIT_NS) raise_error(a.status, E_TIMEOUT, 4);
                    __nanosleep(1000);
                }
            }
        }
        __syncthreads();
    }
}

// One consumer wait on position 0 of a one-slot ring that nothing publishes, with tiles still
// unproduced: the wait must give up after WAIT_NS and record E_TIMEOUT (ps4_check_ring_wait).
__global__ void ring_wait_probe(const SearchArgs a, unsigned long long *out) {
    const uint64_t t0 = gtimer();
    out[0] = ring_wait_ready(a, 0) ? 1ull : 0ull;
    out[1] = gtimer() - t0;
}

// seq[i] = i: every slot free for its first lap
__global__ void ring_init(uint32_t *seq, uint64_t n) {
    for (uint64_t i = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        seq[i] = (uint32_t)i;
}

// ================================================================== launchers

int gen_grid(int num_sms, unsigned TL) { return num_sms * (BS / gen_threads(TL)) * 2; }
int ext_grid(int num_sms) { return num_sms * 3; }

template <int TL>
static int launch_gen_tl(const SearchArgs &a, int grid, cudaStream_t s) {
    // the tile layout up to its extension-list area, then the group's list counters there
    constexpr int NT = gen_threads(TL);
    const size_t smem = TileLayout<TL>::OFF_ELIST + SUPER_K * (NT / 32) * sizeof(uint32_t);
    cudaFuncSetAttribute(gen_jobs<TL, NT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    gen_jobs<TL, NT><<<grid, NT, smem, s>>>(a);
    return (int)cudaGetLastError();
}

int launch_gen(const SearchArgs &a, int grid, void *stream) {
    cudaStream_t s = (cudaStream_t)stream;
    switch (a.log2_tile) {
        case 12: return launch_gen_tl<12>(a, grid, s);
        case 13: return launch_gen_tl<13>(a, grid, s);
        default: return launch_gen_tl<14>(a, grid, s);
    }
}

// resident CTAs per SM of the persistent kernel (three by design; fewer if the device says so, so
// that no CTA of the grid waits for another to exit)
int persist_ctas_per_sm() {
    int n = 0;
    if (cudaFuncSetAttribute(search_persist, cudaFuncAttributeMaxDynamicSharedMemorySize,
                             (int)(PWARPS * sizeof(WarpArea))) != cudaSuccess ||
        cudaOccupancyMaxActiveBlocksPerMultiprocessor(&n, search_persist, PBS, PWARPS * sizeof(WarpArea)) !=
            cudaSuccess)
        n = 1;
    return n < 1 ? 1 : (n > 3 ? 3 : n);
}

int launch_persist(const SearchArgs &a, int grid, void *stream) {
    const size_t smem = PWARPS * sizeof(WarpArea);
    cudaFuncSetAttribute(search_persist, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    search_persist<<<grid, PBS, smem, (cudaStream_t)stream>>>(a);
    return (int)cudaGetLastError();
}

int launch_ring_wait_probe(const SearchArgs &a, unsigned long long *out, void *stream) {
    ring_wait_probe<<<1, 1, 0, (cudaStream_t)stream>>>(a, out);
    return (int)cudaGetLastError();
}

int launch_ring_init(uint32_t *seq, uint64_t n, void *stream) {
    ring_init<<<1184, 256, 0, (cudaStream_t)stream>>>(seq, n);
    return (int)cudaGetLastError();
}

int launch_ext(const SearchArgs &a, int grid, void *stream) {
    const size_t smem = EWARPS * sizeof(WarpArea);
    cudaFuncSetAttribute(extend_jobs, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    extend_jobs<<<grid, EBS, smem, (cudaStream_t)stream>>>(a);
    return (int)cudaGetLastError();
}

}  // namespace ps4
