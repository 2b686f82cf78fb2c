// ps4_kernels.cu -- sm_100a kernels of the square-sum set search.
//
// The reference engine (exhaustive/s4.c) walks S in chunks on CPU threads.  Here a tile
// of 2^TL consecutive S values is owned by one CTA and lives in shared memory:
//
//   P1  count     every representation S = p^2+q^2 (1<=p<=q) with S in the tile, q-major
//                 scan, packed 16-bit shared-memory counters            (s4.c:284-298)
//   P2  scan      block scan -> list of S with >= 3 representations and S != 2 mod 4,
//                 closed-form triple counts, capacity checks             (s4.c:299-321)
//   P3  fill      second scan writes (p,q) of those S into shared lists  (s4.c:306-310)
//   P4  sort      each list ascending in p (the reference's bucket order)
//   P5  4-sets    batched: every rep pair (x,y) scans only the z ranges that give positive
//                 4-sets (class A: P_z < P_x+P_y, class B: P_z > S-P_x-P_y); each 4-set
//                 picks its extension difference and is staged, binned by divisor cost
//                 plain:   one thread per S runs all triples and extends inline (s4.c:311-341)
//   P6  extend    batched: warps take staged 4-sets most-expensive bin first; each lane
//                 walks half of the divisor pairs of its difference with an odometer and
//                 exact modular inverses; residue filters; exact 128-bit square tests
//                 (s4.c:160-207)
//   P7  report    group the tile's extensions per 4-set; M / 5 / 6-set records, verify
//                 flags, counters (s4.c:243-277)
//
// All arithmetic is exact integer arithmetic.  Floating point only produces square-root
// estimates that are then corrected (isqrt*) or checked by an exact integer square
// (is_square_fast).  No tensor cores: nothing here is a contraction.

#include <cuda_runtime.h>
#include <stdint.h>
#include <stdio.h>
#include <string.h>

#include <algorithm>

#include "ps4_internal.h"

namespace ps4 {

typedef unsigned long long ull;
typedef unsigned __int128 u128;

constexpr int BS = 512;         // threads per CTA
constexpr int NWARP = BS / 32;
constexpr int NBIN = 16;        // divisor-cost bins of the extension phase
constexpr int MAXP = 16;        // distinct primes of a difference D < 2^64 (15 suffice)

// ------------------------------------------------------------------ exact roots

// floor(sqrt(n)) for n < 2^64: libm-style estimate, then exact integer correction.
__device__ __forceinline__ uint64_t isqrt64(uint64_t n) {
    uint64_t r = (uint64_t)sqrt((double)n);
    if (r > 0xFFFFFFFFull) r = 0xFFFFFFFFull;
    while (r * r > n) r--;
    while (r < 0xFFFFFFFFull && (r + 1) * (r + 1) <= n) r++;
    return r;
}

__device__ __forceinline__ uint64_t ceil_sqrt64(uint64_t n) {
    uint64_t r = isqrt64(n);
    return r * r < n ? r + 1 : r;
}

__device__ __forceinline__ double u128_to_double(u128 n) {
    return (double)(uint64_t)(n >> 64) * 18446744073709551616.0 + (double)(uint64_t)n;
}

// floor(sqrt(n)) for n < 2^126, exact.
__device__ __forceinline__ uint64_t isqrt128(u128 n) {
    if ((n >> 64) == 0) return isqrt64((uint64_t)n);
    uint64_t r = (uint64_t)sqrt(u128_to_double(n));
    while ((u128)r * r > n) r--;
    while ((u128)(r + 1) * (r + 1) <= n) r++;
    return r;
}

__device__ __forceinline__ bool is_square_exact(u128 n) {
    uint64_t r = isqrt128(n);
    return (u128)r * r == n;
}

// Exact square test for n < 2^100.  If n = s^2 then s < 2^50; the double conversion and
// the correctly rounded sqrt leave an error below s*2^-52 < 1/4, so rounding to nearest
// returns s exactly and the integer check r*r == n succeeds.  If n is not a square no
// integer r satisfies r*r == n.  Hence the result is exact.
__device__ __forceinline__ bool is_square_fast(u128 n) {
    uint64_t r = __double2ull_rn(sqrt(u128_to_double(n)));
    return (u128)r * r == n;
}

// ------------------------------------------------------------------ residues

__host__ __device__ constexpr uint64_t qr_bits(int m) {
    uint64_t x = 0;
    for (int i = 0; i < m; i++) {
        int r = (i * i) % m;
        if (r < 64) x |= 1ull << r;
    }
    return x;
}
constexpr uint64_t QR64 = qr_bits(64);
constexpr uint64_t QR63 = qr_bits(63);
constexpr uint64_t QR65 = qr_bits(65);   // residues 0..63; residue 64 = 8^2 is a square too

__device__ __forceinline__ bool qr65(uint32_t r) { return r == 64 ? true : ((QR65 >> r) & 1); }

// inverse of odd q modulo 2^64 (Newton: each step doubles the correct low bits)
__device__ __forceinline__ uint64_t inv64(uint64_t q) {
    uint32_t q32 = (uint32_t)q, x = q32;          // q*q == 1 mod 8: 3 bits
    x *= 2u - q32 * x;                             // 6
    x *= 2u - q32 * x;                             // 12
    x *= 2u - q32 * x;                             // 24
    x *= 2u - q32 * x;                             // 32
    uint64_t y = x;
    y *= 2ull - q * y;                             // 64
    return y;
}

// ------------------------------------------------------------------ 4-set helpers

// roots: r[0..5] = r_ab, r_ac, r_ad, r_bc, r_bd, r_cd; v = a,b,c,d (formula order)
__device__ __forceinline__ int pair_slot(int i, int j) {
    int lo = i < j ? i : j, hi = i < j ? j : i;
    return lo == 0 ? hi - 1 : (lo == 1 ? hi + 1 : 5);
}

__device__ __forceinline__ uint32_t pick6(const uint32_t r[6], int s) {
    uint32_t x = r[0];
    x = s == 1 ? r[1] : x; x = s == 2 ? r[2] : x; x = s == 3 ? r[3] : x;
    x = s == 4 ? r[4] : x; x = s == 5 ? r[5] : x;
    return x;
}

__device__ __forceinline__ uint64_t pick4(const uint64_t v[4], int s) {
    uint64_t x = v[0];
    x = s == 1 ? v[1] : x; x = s == 2 ? v[2] : x; x = s == 3 ? v[3] : x;
    return x;
}

__device__ __forceinline__ void quad_values(const uint32_t r[6], uint64_t v[4], uint64_t &S) {
    uint64_t ab = (uint64_t)r[0] * r[0], ac = (uint64_t)r[1] * r[1], ad = (uint64_t)r[2] * r[2];
    uint64_t bc = (uint64_t)r[3] * r[3], cd = (uint64_t)r[5] * r[5];
    uint64_t a = (ab + ac - bc) >> 1;
    v[0] = a; v[1] = ab - a; v[2] = ac - a; v[3] = ad - a;
    S = ab + cd;
}

// The difference to extend by: the pair (i,j), v_i > v_j, whose D = v_i - v_j =
// (r_ik - r_jk)(r_ik + r_jk) has the fewest estimated divisors d(r_ik-r_jk)*d(r_ik+r_jk);
// candidate order and strict '<' tie-break as s4.c:163-171.
__device__ __forceinline__ void choose_pair(const uint64_t v[4], const uint32_t r[6], const uint16_t *ndiv,
                                            int &bi, int &bj, int &bk, uint32_t &best) {
    const int P[6][3] = {{0, 1, 2}, {2, 3, 0}, {0, 2, 1}, {1, 3, 0}, {0, 3, 1}, {1, 2, 0}};
    best = 0xFFFFFFFFu; bi = 0; bj = 1; bk = 2;
#pragma unroll
    for (int t = 0; t < 6; t++) {
        const int i = P[t][0], j = P[t][1], k = P[t][2];
        const bool sw = v[i] < v[j];
        const uint32_t rik = r[pair_slot(i, k)], rjk = r[pair_slot(j, k)];
        const uint32_t ra = sw ? rjk : rik, rb = sw ? rik : rjk;
        const uint32_t est = (uint32_t)__ldg(&ndiv[ra - rb]) * (uint32_t)__ldg(&ndiv[ra + rb]);
        if (est < best) { best = est; bi = sw ? j : i; bj = sw ? i : j; bk = k; }
    }
}

// Merge the factorisation of m into (pr, ex, np), primes in first-seen order of the
// smallest-prime-factor walk (s4.c:141-147).
__device__ __forceinline__ void factor_merge(const uint64_t *spfq, uint32_t m, uint32_t *pr, uint8_t *ex, int &np) {
    while (m > 1) {
        uint64_t sq = __ldg(&spfq[m]);
        const uint32_t p = (uint32_t)sq;
        int e = 0;
        for (;;) {
            m = (uint32_t)(sq >> 32);
            e++;
            if (m <= 1) break;
            sq = __ldg(&spfq[m]);
            if ((uint32_t)sq != p) break;
        }
        int i = 0;
        while (i < np && pr[i] != p) i++;
        if (i == np) { pr[np] = p; ex[np] = 0; np++; }
        ex[i] = (uint8_t)(ex[i] + e);
    }
}

struct ExtEntry {            // one extension found in a tile (48 bytes)
    uint32_t qid, key;
    uint32_t r[6];
    uint64_t lo, hi;
};

__device__ __forceinline__ void raise_error(Status *st, unsigned code, uint64_t S) {
    atomicCAS(&st->err, 0ull, (ull)code | ((ull)S << 8));
}

// internal list overflow: record which list (1 = selected S, 2 = their representations,
// 3 = staged 4-sets, 4 = tile extensions), its size and limit, then raise the re-run code
__device__ __forceinline__ void raise_capacity(Status *st, unsigned code, unsigned which, uint64_t size,
                                               uint64_t limit, uint64_t S) {
    if (atomicCAS(&st->err, 0ull, (ull)code | ((ull)S << 8)) == 0ull) {
        st->diag[0] = which; st->diag[1] = size; st->diag[2] = limit; st->diag[3] = S;
    }
}

// Extend one 4-set (v, roots r) by every e: e+v_i square for all i.  Restates extend4
// (s4.c:160-207) with the same difference choice (bi,bj,bk), the same counters and the
// same order key (the reference's mixed-radix divisor index of the smaller divisor),
// but walks each complementary divisor pair once instead of twice and counts ext_cand
// in closed form.
__device__ void extend_quad(const SearchArgs &a, const uint32_t r[6], const uint64_t v[4], uint64_t S,
                            int bi, int bj, int bk, uint32_t qid,
                            ull &n_cand, ull &n_sqrt, uint32_t &max_divs,
                            ExtEntry *elist, uint32_t *elist_n, uint32_t elist_cap) {
    const uint32_t ra = pick6(r, pair_slot(bi, bk)), rb = pick6(r, pair_slot(bj, bk));
    const uint64_t A = pick4(v, bi);
    int o1 = -1, o2 = -1;
#pragma unroll
    for (int t = 0; t < 4; t++)
        if (t != bi && t != bj) { if (o1 < 0) o1 = t; else o2 = t; }
    const uint64_t C1 = pick4(v, o1), C2 = pick4(v, o2);

    uint32_t pr[MAXP];
    uint8_t ex[MAXP];
    int np = 0;
    factor_merge(a.spfq, ra - rb, pr, ex, np);
    factor_merge(a.spfq, ra + rb, pr, ex, np);

    // D even => both factors even => 2 is the first prime and 4 | D
    const bool has2 = np > 0 && pr[0] == 2;
    const int E2 = has2 ? ex[0] : 0;
    const int j0 = has2 ? 1 : 0;
    uint64_t qinv[MAXP], qpow[MAXP], qipow[MAXP];
    uint64_t ndo = 1, Dodd = 1;
    for (int j = j0; j < np; j++) {
        const uint64_t q = pr[j], qi = inv64(q);
        uint64_t pw = 1, ipw = 1;
        for (int e = 0; e < ex[j]; e++) { pw *= q; ipw *= qi; }
        qinv[j] = qi; qpow[j] = pw; qipow[j] = ipw;
        ndo *= (uint64_t)ex[j] + 1;
        Dodd *= pw;
    }
    const uint64_t nd = ndo * (uint64_t)(E2 + 1);
    if (nd > a.cap_divs) { raise_error(a.status, E_CAP_DIVS, S); return; }
    if ((uint32_t)nd > max_divs) max_divs = (uint32_t)nd;
    // same-parity complementary pairs with f < g  (the reference's ext_cand, s4.c:191)
    n_cand += has2 ? ((uint64_t)(E2 - 1) * ndo) >> 1 : nd >> 1;

    const int64_t d1 = (int64_t)C1 - (int64_t)A, d2 = (int64_t)C2 - (int64_t)A;
    const uint32_t a64 = (uint32_t)(((d1 % 64) + 64) % 64), b64 = (uint32_t)(((d2 % 64) + 64) % 64);
    const uint32_t a63 = (uint32_t)(((d1 % 63) + 63) % 63), b63 = (uint32_t)(((d2 % 63) + 63) % 63);
    const uint32_t a65 = (uint32_t)(((d1 % 65) + 65) % 65), b65 = (uint32_t)(((d2 % 65) + 65) % 65);

    uint8_t dig[MAXP];
    for (int j = 0; j < MAXP; j++) dig[j] = 0;
    uint64_t fo = 1, go = Dodd, todd = 0;
    const int dlo = has2 ? 1 : 0, dhi = has2 ? E2 - 1 : 0;
    while (2 * todd + 1 <= ndo) {                      // todd <= its complement ndo-1-todd
        const bool mid = (2 * todd + 1 == ndo);
        for (int d2 = dlo; d2 <= dhi; d2++) {
            if (mid && 2 * d2 >= E2) break;            // self-complementary half already seen
            const uint64_t ft = fo << d2, gt = go << (E2 - d2);
            const uint64_t t = has2 ? (uint64_t)d2 + (uint64_t)(E2 + 1) * todd : todd;
            uint64_t f, g;
            uint32_t key;
            if (ft < gt) { f = ft; g = gt; key = (uint32_t)t; }
            else { f = gt; g = ft; key = (uint32_t)(nd - 1 - t); }
            const uint64_t u = (f + g) >> 1;
            // residue filters of e + C = u^2 + (C - A)  (s4.c:192-194)
            uint32_t w = (uint32_t)(u & 63), w2 = w * w;
            if (!((QR64 >> ((w2 + a64) & 63)) & 1) || !((QR64 >> ((w2 + b64) & 63)) & 1)) continue;
            w = (uint32_t)(u % 63); w2 = w * w;
            if (!((QR63 >> ((w2 + a63) % 63)) & 1) || !((QR63 >> ((w2 + b63) % 63)) & 1)) continue;
            w = (uint32_t)(u % 65); w2 = w * w;
            if (!qr65((w2 + a65) % 65) || !qr65((w2 + b65) % 65)) continue;
            const u128 usq = (u128)u * u;
            if (usq <= A) continue;
            const u128 e = usq - A;
            if (e == v[0] || e == v[1] || e == v[2] || e == v[3]) continue;
            n_sqrt++;
            if (!is_square_fast(e + C1) || !is_square_fast(e + C2)) continue;
            const uint32_t slot = atomicAdd(elist_n, 1u);
            if (slot < elist_cap) {
                ExtEntry &x = elist[slot];
                x.qid = qid; x.key = key;
#pragma unroll
                for (int i = 0; i < 6; i++) x.r[i] = r[i];
                x.lo = (uint64_t)e; x.hi = (uint64_t)(e >> 64);
            } else {
                raise_capacity(a.status, E_EXTLIST, 4, slot + 1, elist_cap, S);
            }
        }
        todd++;
        for (int j = j0; j < np; j++) {                // odometer over the odd primes
            if (dig[j] < ex[j]) { dig[j]++; fo *= pr[j]; go *= qinv[j]; break; }
            dig[j] = 0; fo *= qipow[j]; go *= qpow[j];
        }
    }
}

// ------------------------------------------------------------------ block helpers

// exclusive block scan of three u32 values; returns totals in tot[3]
__device__ __forceinline__ void block_scan3(uint32_t x0, uint32_t x1, uint32_t x2, uint32_t &e0, uint32_t &e1,
                                            uint32_t &e2, uint32_t tot[3], uint32_t *wsum /* 3*NWARP */) {
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t i0 = x0, i1 = x1, i2 = x2;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y0 = __shfl_up_sync(0xffffffffu, i0, o), y1 = __shfl_up_sync(0xffffffffu, i1, o),
                 y2 = __shfl_up_sync(0xffffffffu, i2, o);
        if (lane >= o) { i0 += y0; i1 += y1; i2 += y2; }
    }
    if (lane == 31) { wsum[wid] = i0; wsum[NWARP + wid] = i1; wsum[2 * NWARP + wid] = i2; }
    __syncthreads();
    if (wid == 0) {
        uint32_t s0 = lane < NWARP ? wsum[lane] : 0, s1 = lane < NWARP ? wsum[NWARP + lane] : 0,
                 s2 = lane < NWARP ? wsum[2 * NWARP + lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y0 = __shfl_up_sync(0xffffffffu, s0, o), y1 = __shfl_up_sync(0xffffffffu, s1, o),
                     y2 = __shfl_up_sync(0xffffffffu, s2, o);
            if (lane >= o) { s0 += y0; s1 += y1; s2 += y2; }
        }
        if (lane < NWARP) { wsum[lane] = s0; wsum[NWARP + lane] = s1; wsum[2 * NWARP + lane] = s2; }
    }
    __syncthreads();
    const uint32_t b0 = wid ? wsum[wid - 1] : 0, b1 = wid ? wsum[NWARP + wid - 1] : 0,
                   b2 = wid ? wsum[2 * NWARP + wid - 1] : 0;
    e0 = b0 + i0 - x0; e1 = b1 + i1 - x1; e2 = b2 + i2 - x2;
    tot[0] = wsum[NWARP - 1]; tot[1] = wsum[2 * NWARP - 1]; tot[2] = wsum[3 * NWARP - 1];
    __syncthreads();
}

__device__ __forceinline__ ull warp_sum(ull x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x += __shfl_xor_sync(0xffffffffu, x, o);
    return x;
}
__device__ __forceinline__ uint32_t warp_max(uint32_t x) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) x = max(x, __shfl_xor_sync(0xffffffffu, x, o));
    return x;
}

// ------------------------------------------------------------------ tile state

struct TileShared {
    ull cnt[16];               // per-tile counters (K_* slots 0..12)
    uint32_t wsum[3 * NWARP];
    uint32_t n_is, n_rep, n_pairs, n_quads;
    uint32_t n_staged, flushed;    // 4-sets staged for extension / already extended in this tile
    uint32_t elist_n, work;
    uint32_t binhist[NBIN], binstart[NBIN];
    uint32_t skip;             // tile abandoned (error)
    uint64_t tile;
};

template <int TL>
struct TileLayout {
    static constexpr uint32_t W = 1u << TL;
    static constexpr uint32_t IS_CAP = W / 8;
    static constexpr uint32_t REP_CAP = (W * 3) / 8;
    static constexpr size_t OFF_CNT = 0;                                   // W/2 u32
    static constexpr size_t OFF_IS_OFF = OFF_CNT + 2 * (size_t)W;          // IS_CAP u16
    static constexpr size_t OFF_IS_K = OFF_IS_OFF + 2 * (size_t)IS_CAP;
    static constexpr size_t OFF_IS_START = OFF_IS_K + 2 * (size_t)IS_CAP;
    static constexpr size_t OFF_IS_PBASE = OFF_IS_START + 2 * (size_t)IS_CAP;   // IS_CAP+1 u32 (pad to 8)
    static constexpr size_t OFF_REP_P = (OFF_IS_PBASE + 4 * ((size_t)IS_CAP + 2) + 15) & ~(size_t)15;
    static constexpr size_t OFF_REP_Q = OFF_REP_P + 4 * (size_t)REP_CAP;
    static constexpr uint32_t ELIST_CAP = 256;                              // extensions per tile
    static constexpr size_t OFF_ELIST = OFF_REP_Q + 4 * (size_t)REP_CAP;
    static constexpr size_t BYTES = OFF_ELIST + ELIST_CAP * sizeof(ExtEntry);
    static constexpr uint32_t FLUSH_AT = W / 2;                             // staged 4-sets that trigger P6
};

// locate a tile: tiles are handed out highest-S first (longest work first)
__device__ __forceinline__ void tile_bounds(const SearchArgs &a, uint64_t tile, unsigned TLv, uint32_t &item,
                                            uint64_t &S0, uint32_t &n) {
    const uint64_t ti = a.n_tiles - 1 - tile;
    uint32_t lo = 0, hi = a.n_items;                   // last item with tile_base <= ti
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a.items[mid].tile_base <= ti) lo = mid; else hi = mid;
    }
    item = lo;
    const Item it = a.items[lo];
    S0 = it.lo + ((ti - it.tile_base) << TLv);
    const uint64_t S1 = S0 + (1ull << TLv) < it.hi ? S0 + (1ull << TLv) : it.hi;
    n = (uint32_t)(S1 - S0);
}

// P1 / P3: scan every representation S = p^2 + q^2, 1 <= p <= q, S in [S0, S0+n).
// q-major: q runs over [ceil(sqrt(S0/2)), isqrt(S1-2)], p from ceil(sqrt(S0-q^2)).
template <bool FILL>
__device__ __forceinline__ uint32_t scan_reps(uint64_t S0, uint32_t n, uint32_t *cnt32, uint32_t *rep_p,
                                              uint32_t *rep_q) {
    const uint64_t S1 = S0 + n;
    uint64_t qmin = ceil_sqrt64((S0 + 1) >> 1);
    if (qmin < 1) qmin = 1;
    const uint64_t qmax = S1 >= 2 ? isqrt64(S1 - 2) : 0;
    uint32_t found = 0;
    for (uint64_t q = qmin + threadIdx.x; q <= qmax; q += BS) {
        const uint64_t q2 = q * q;
        uint64_t p = 1;
        if (S0 > q2 + 1) p = ceil_sqrt64(S0 - q2);
        for (uint64_t s = p * p + q2; p <= q && s < S1; s += 2 * p + 1, p++) {
            const uint32_t i = (uint32_t)(s - S0), w = i >> 1, sh = (i & 1) * 16;
            if (!FILL) {
                atomicAdd(&cnt32[w], 1u << sh);
                found++;
            } else {
                const uint32_t cur = (((volatile uint32_t *)cnt32)[w] >> sh) & 0xFFFFu;
                if (cur == 0xFFFFu) continue;          // S not selected
                const uint32_t pos = (atomicAdd(&cnt32[w], 1u << sh) >> sh) & 0xFFFFu;
                rep_p[pos] = (uint32_t)p;
                rep_q[pos] = (uint32_t)q;
            }
        }
    }
    return found;
}

// P1-P4 for one tile.  Returns false if the tile was abandoned (error raised).
template <int TL>
__device__ bool tile_reps(const SearchArgs &a, TileShared &ts, unsigned char *smem, uint64_t S0, uint32_t n) {
    using L = TileLayout<TL>;
    uint32_t *cnt32 = (uint32_t *)(smem + L::OFF_CNT);
    uint16_t *is_off = (uint16_t *)(smem + L::OFF_IS_OFF);
    uint16_t *is_k = (uint16_t *)(smem + L::OFF_IS_K);
    uint16_t *is_start = (uint16_t *)(smem + L::OFF_IS_START);
    uint32_t *is_pbase = (uint32_t *)(smem + L::OFF_IS_PBASE);
    uint32_t *rep_p = (uint32_t *)(smem + L::OFF_REP_P);
    uint32_t *rep_q = (uint32_t *)(smem + L::OFF_REP_Q);
    const int tid = threadIdx.x;

    for (uint32_t i = tid; i < L::W / 2; i += BS) cnt32[i] = 0;
    __syncthreads();
    // P1: count
    const uint32_t found = scan_reps<false>(S0, n, cnt32, rep_p, rep_q);
    ull f = warp_sum((ull)found);
    if ((tid & 31) == 0 && f) atomicAdd(&ts.cnt[K_PAIRS], f);
    __syncthreads();

    // P2: select S with >= 3 representations and S != 2 (mod 4)
    constexpr uint32_t SEG = L::W / BS;               // even: a thread owns whole counter words
    const uint32_t i0 = tid * SEG;
    uint32_t nI = 0, nR = 0, nP = 0, kmax = 0;
    ull trip = 0;
    bool over = false;
    for (uint32_t i = i0; i < i0 + SEG && i < n; i++) {
        const uint32_t k = (cnt32[i >> 1] >> ((i & 1) * 16)) & 0xFFFFu;
        kmax = max(kmax, k);
        if (k >= 3 && ((S0 + i) & 3) != 2) {
            nI++; nR += k; nP += k * (k - 1) / 2;
            trip += (ull)k * (k - 1) * (k - 2) / 6;
            if (k > a.cap_reps) over = true;
        }
    }
    if (over) raise_error(a.status, E_CAP_REPS, S0);
    uint32_t bI, bR, bP, tot[3];
    block_scan3(nI, nR, nP, bI, bR, bP, tot, ts.wsum);
    {
        const ull tw = warp_sum(trip);
        const uint32_t km = warp_max(kmax);
        if ((tid & 31) == 0) {
            if (tw) atomicAdd(&ts.cnt[K_TRIPLES], tw);
            atomicMax(&ts.cnt[K_MAX_REPS], (ull)km);
        }
    }
    if (tot[0] > L::IS_CAP || tot[1] > L::REP_CAP) {
        if (tid == 0) {
            if (tot[0] > L::IS_CAP) raise_capacity(a.status, E_TILE, 1, tot[0], L::IS_CAP, S0);
            else raise_capacity(a.status, E_TILE, 2, tot[1], L::REP_CAP, S0);
        }
        return false;
    }
    if (tid == 0) {
        ts.n_is = tot[0]; ts.n_rep = tot[1]; ts.n_pairs = tot[2];
        ts.cnt[K_S_DONE] += n;
        ts.cnt[K_S_GE3] += tot[0];
        is_pbase[tot[0]] = tot[2];
    }
    for (uint32_t i = i0; i < i0 + SEG; i += 2) {
        uint32_t word = 0;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const uint32_t ii = i + h;
            uint32_t val = 0xFFFFu;
            if (ii < n) {
                const uint32_t k = (cnt32[ii >> 1] >> (h * 16)) & 0xFFFFu;
                if (k >= 3 && ((S0 + ii) & 3) != 2) {
                    is_off[bI] = (uint16_t)ii; is_k[bI] = (uint16_t)k; is_start[bI] = (uint16_t)bR;
                    is_pbase[bI] = bP;
                    val = bR;
                    bI++; bR += k; bP += k * (k - 1) / 2;
                }
            }
            word |= val << (h * 16);
        }
        cnt32[i >> 1] = word;
    }
    __syncthreads();
    // P3: fill
    scan_reps<true>(S0, n, cnt32, rep_p, rep_q);
    __syncthreads();
    // P4: each list ascending in p
    for (uint32_t s = tid; s < ts.n_is; s += BS) {
        const uint32_t st = is_start[s], k = is_k[s];
        for (uint32_t x = st + 1; x < st + k; x++) {
            const uint32_t kp = rep_p[x], kq = rep_q[x];
            uint32_t y = x;
            while (y > st && rep_p[y - 1] > kp) { rep_p[y] = rep_p[y - 1]; rep_q[y] = rep_q[y - 1]; y--; }
            rep_p[y] = kp; rep_q[y] = kq;
        }
    }
    __syncthreads();
    return true;
}

// verify the six roots of a 4-set (s4.c:229-233)
__device__ __forceinline__ bool quad_roots_ok(const uint64_t v[4], const uint32_t r[6]) {
    const int I[6] = {0, 0, 0, 1, 1, 2}, J[6] = {1, 2, 3, 2, 3, 3};
#pragma unroll
    for (int t = 0; t < 6; t++) {
        if ((uint64_t)r[t] * r[t] != v[I[t]] + v[J[t]] || v[I[t]] == v[J[t]]) return false;
    }
    return true;
}

__device__ __forceinline__ void record_verify_failure(const SearchArgs &a, uint64_t S, const uint64_t v[4]) {
    if (atomicCAS(&a.status->err, 0ull, (ull)E_VERIFY | ((ull)S << 8)) == 0ull) {
        a.status->verify_bad[0] = S;
        for (int i = 0; i < 4; i++) a.status->verify_bad[1 + i] = v[i];
    }
}

__device__ __forceinline__ void dump_quad(const SearchArgs &a, const uint32_t r[6]) {
    const ull slot = atomicAdd(&a.status->n_quads, 1ull);
    if (slot < a.quads_cap) {
        ps4_quad q;
        q.r_ab = r[0]; q.r_ac = r[1]; q.r_ad = r[2]; q.r_bc = r[3]; q.r_bd = r[4]; q.r_cd = r[5];
        a.quads[slot] = q;
    }
}

// all pairwise sums square, members distinct (s4.c:209-212)
__device__ bool verify_set(const u128 *x, int n) {
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++)
            if (x[i] == x[j] || !is_square_exact(x[i] + x[j])) return false;
    return true;
}

// P7: turn the tile's extension list into hit / ext / six records (s4.c:243-277).
// Runs on one thread; tiles hold a handful of extensions at most.
__device__ void tile_report(const SearchArgs &a, TileShared &ts, ExtEntry *el, uint32_t n_el, uint32_t item) {
    for (uint32_t x = 1; x < n_el; x++) {             // sort by (qid, key)
        ExtEntry k = el[x];
        uint32_t y = x;
        while (y > 0 && (el[y - 1].qid > k.qid || (el[y - 1].qid == k.qid && el[y - 1].key > k.key))) {
            el[y] = el[y - 1];
            y--;
        }
        el[y] = k;
    }
    ull *cnt = a.counters + (size_t)item * K_SLOTS;
    for (uint32_t g0 = 0; g0 < n_el;) {
        uint32_t g1 = g0 + 1;
        while (g1 < n_el && el[g1].qid == el[g0].qid) g1++;
        const uint32_t ne = g1 - g0;
        uint64_t v[4], S;
        quad_values(el[g0].r, v, S);
        if (ne > a.cap_ext) { raise_error(a.status, E_CAP_EXT, S); g0 = g1; continue; }
        if (ne > ts.cnt[K_MAX_EXT]) ts.cnt[K_MAX_EXT] = ne;
        uint64_t vmax = v[0];
        for (int i = 1; i < 4; i++) vmax = v[i] > vmax ? v[i] : vmax;
        bool prints = ne >= 2;                          // an "M:" line, or a "5:" line below
        for (uint32_t t = 0; t < ne; t++) prints |= (el[g0 + t].hi != 0 || el[g0 + t].lo > vmax);
        if (!prints) { g0 = g1; continue; }             // a lone extension below max(v): no output
        const uint32_t hslot = atomicAdd(&a.status->n_hits, 1u);
        const uint32_t eslot = atomicAdd(&a.status->n_exts, ne);
        uint32_t hflags = 0;
        if (ne >= 2) {
            hflags |= PS4_HIT_MULTI;
            ts.cnt[K_MULTI]++;
            u128 x[6] = {v[0], v[1], v[2], v[3], ((u128)el[g0].hi << 64) | el[g0].lo,
                         ((u128)el[g0 + 1].hi << 64) | el[g0 + 1].lo};
            if (verify_set(x, 6)) hflags |= PS4_HIT_DRILL_OK;
        }
        for (uint32_t t = 0; t < ne; t++) {
            const u128 e = ((u128)el[g0 + t].hi << 64) | el[g0 + t].lo;
            uint32_t ef = 0;
            if (e > vmax) {
                ef |= PS4_EXT_FIVE;
                ts.cnt[K_SETS5]++;
                int lg = 0;
                for (u128 z = e; z > 1; z >>= 1) lg++;
                atomicAdd(&cnt[K_HIST5 + (lg > 99 ? 99 : lg)], 1ull);
                u128 x[5] = {v[0], v[1], v[2], v[3], e};
                if (verify_set(x, 5)) ef |= PS4_EXT_FIVE_OK;
            }
            if (eslot + t < a.exts_cap) {
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
                ts.cnt[K_SETS6]++;
                u128 x[6] = {v[0], v[1], v[2], v[3], et, es};
                const uint32_t sslot = atomicAdd(&a.status->n_sixes, 1u);
                if (sslot < a.sixes_cap) {
                    ps4_six rec;
                    rec.hit = hslot; rec.t = t; rec.s = s; rec.flags = verify_set(x, 6) ? 1u : 0u;
                    a.sixes[sslot] = rec;
                }
            }
        if (hslot < a.hits_cap) {
            ps4_hit h;
            h.S = S;
            for (int i = 0; i < 4; i++) h.v[i] = v[i];
            h.n_ext = ne; h.first_ext = eslot; h.flags = hflags; h.item = item;
            const uint32_t *r = el[g0].r;
            h.order[0] = r[5]; h.order[1] = r[4];
            h.order[2] = r[2] < r[3] ? r[2] : r[3];
            h.order[3] = r[2] < r[3] ? 1u : 0u;
            a.hits[hslot] = h;
        }
        g0 = g1;
    }
}

__device__ __forceinline__ void tile_flush_counters(const SearchArgs &a, TileShared &ts, uint32_t item) {
    if (threadIdx.x != 0) return;
    ull *cnt = a.counters + (size_t)item * K_SLOTS;
    for (int k = 0; k < 10; k++)
        if (ts.cnt[k]) atomicAdd(&cnt[k], ts.cnt[k]);
    for (int k = K_MAX_REPS; k <= K_MAX_EXT; k++)
        if (ts.cnt[k]) atomicMax(&cnt[k], ts.cnt[k]);
}

__device__ __forceinline__ void tile_reset(TileShared &ts) {
    if (threadIdx.x < 16) ts.cnt[threadIdx.x] = 0;
    if (threadIdx.x < NBIN) ts.binhist[threadIdx.x] = 0;
    if (threadIdx.x == 0) {
        ts.n_quads = 0; ts.n_staged = 0; ts.flushed = 0; ts.elist_n = 0; ts.work = 0; ts.skip = 0;
    }
}

__device__ __forceinline__ void block_add_ext_counters(TileShared &ts, ull c, ull s, uint32_t md) {
    c = warp_sum(c); s = warp_sum(s); md = warp_max(md);
    if ((threadIdx.x & 31) == 0) {
        if (c) atomicAdd(&ts.cnt[K_EXT_CAND], c);
        if (s) atomicAdd(&ts.cnt[K_EXT_SQRT], s);
        if (md) atomicMax(&ts.cnt[K_MAX_DIVS], (ull)md);
    }
}

// decode pair index j -> (x < y) with j = y(y-1)/2 + x
__device__ __forceinline__ void decode_pair(uint32_t j, uint32_t &x, uint32_t &y) {
    uint32_t yy = (uint32_t)((1.0f + sqrtf(1.0f + 8.0f * (float)j)) * 0.5f);
    while (yy * (yy - 1) / 2 > j) yy--;
    while ((yy + 1) * yy / 2 <= j) yy++;
    y = yy;
    x = j - yy * (yy - 1) / 2;
}

// ================================================================== batched kernel

// P5.5 + P6 over the staged 4-sets [0, staged): in chunks of up to W, order each chunk by
// divisor-cost bin (most expensive first, so the longest walks start first), then warps pull
// 32 staged 4-sets at a time and each lane extends one.
template <int TL>
__device__ void extend_staged(const SearchArgs &a, TileShared &ts, const uint32_t *scr, uint16_t *perm, ExtEntry *el,
                              uint32_t staged, uint32_t qid_base, ull &c_cand, ull &c_sqrt, uint32_t &c_mdiv) {
    using L = TileLayout<TL>;
    const int tid = threadIdx.x, lane = tid & 31;
    const uint32_t cap = a.stage_cap;
    for (uint32_t c0 = 0; c0 < staged; c0 += L::W) {
        const uint32_t c1 = min(c0 + L::W, staged), nc = c1 - c0;
        if (tid < NBIN) ts.binhist[tid] = 0;
        if (tid == 0) ts.work = 0;
        __syncthreads();
        for (uint32_t i = c0 + tid; i < c1; i += BS) atomicAdd(&ts.binhist[(scr[i] >> 22) & 15u], 1u);
        __syncthreads();
        if (tid == 0) {
            uint32_t s = 0;
            for (int b = NBIN - 1; b >= 0; b--) { ts.binstart[b] = s; s += ts.binhist[b]; }
        }
        __syncthreads();
        for (uint32_t i = c0 + tid; i < c1; i += BS)
            perm[atomicAdd(&ts.binstart[(scr[i] >> 22) & 15u], 1u)] = (uint16_t)(i - c0);
        __syncthreads();
        for (;;) {
            uint32_t base = 0;
            if (lane == 0) base = atomicAdd(&ts.work, 32u);
            base = __shfl_sync(0xffffffffu, base, 0);
            if (base >= nc) break;
            const uint32_t pos = base + lane;
            if (pos < nc) {
                const uint32_t qi = c0 + perm[pos];
                const uint32_t w0 = scr[qi];
                uint32_t r[6];
                r[0] = w0 & 0x3FFFFFu;
                r[1] = scr[1 * cap + qi]; r[2] = scr[2 * cap + qi]; r[3] = scr[3 * cap + qi];
                r[4] = scr[4 * cap + qi]; r[5] = scr[5 * cap + qi];
                uint64_t v[4], S;
                quad_values(r, v, S);
                extend_quad(a, r, v, S, (w0 >> 26) & 3, (w0 >> 28) & 3, (w0 >> 30) & 3, qid_base + qi, c_cand,
                            c_sqrt, c_mdiv, el, &ts.elist_n, L::ELIST_CAP);
            }
        }
        __syncthreads();
    }
}

template <int TL>
__global__ void __launch_bounds__(BS, 1) search_batched(const SearchArgs a) {
    using L = TileLayout<TL>;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ TileShared ts;
    const uint32_t cap = a.stage_cap;
    uint32_t *scr = a.scratch + (size_t)blockIdx.x * 6 * cap;
    const int tid = threadIdx.x;
    ExtEntry *el = (ExtEntry *)(smem + L::OFF_ELIST);
    uint16_t *perm = (uint16_t *)(smem + L::OFF_CNT);           // the counters are dead after P3

    for (;;) {
        tile_reset(ts);
        if (tid == 0) {
            ts.tile = atomicAdd((unsigned int *)&a.status->tile_next, 1u);
            ts.skip = *(volatile ull *)&a.status->err != 0ull;   // any error ends the launch
        }
        __syncthreads();
        const uint64_t tile = ts.tile;
        if (tile >= a.n_tiles || ts.skip) break;                 // block-uniform
        uint32_t item, n;
        uint64_t S0;
        tile_bounds(a, tile, TL, item, S0, n);
        if (!tile_reps<TL>(a, ts, smem, S0, n)) { __syncthreads(); continue; }

        const uint16_t *is_off = (const uint16_t *)(smem + L::OFF_IS_OFF);
        const uint16_t *is_k = (const uint16_t *)(smem + L::OFF_IS_K);
        const uint16_t *is_start = (const uint16_t *)(smem + L::OFF_IS_START);
        const uint32_t *is_pbase = (const uint32_t *)(smem + L::OFF_IS_PBASE);
        const uint32_t *rep_p = (const uint32_t *)(smem + L::OFF_REP_P);
        const uint32_t *rep_q = (const uint32_t *)(smem + L::OFF_REP_Q);
        const uint32_t nI = ts.n_is, nPairs = ts.n_pairs;
        ull c_cand = 0, c_sqrt = 0;
        uint32_t c_mdiv = 0;

        // P5 in waves of one representation pair (x,y) per thread; only the z that give positive
        // members are visited.  A wave stages at most BS * 2(k-2) 4-sets, so the staging holds any
        // wave on top of FLUSH_AT; whenever FLUSH_AT is passed (and after the last wave) the staged
        // 4-sets are extended (P5.5/P6) and the staging restarts.
        for (uint32_t wave = 0; wave < nPairs; wave += BS) {
            const uint32_t gidx = wave + tid;
            if (gidx < nPairs) {
                uint32_t lo = 0, hi = nI;
                while (hi - lo > 1) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (is_pbase[mid] <= gidx) lo = mid; else hi = mid;
                }
                const uint32_t st = is_start[lo], k = is_k[lo];
                const uint64_t S = S0 + is_off[lo];
                uint32_t x, y;
                decode_pair(gidx - is_pbase[lo], x, y);
                const uint32_t px = rep_p[st + x], qx = rep_q[st + x], py = rep_p[st + y], qy = rep_q[st + y];
                const uint64_t Px = (uint64_t)px * px, Py = (uint64_t)py * py;
                const uint32_t pxy = (px + py) & 1;
                const uint32_t Sodd = (uint32_t)(S & 1);
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
                        uint32_t r[6];
                        r[0] = qx; r[1] = qy; r[4] = py; r[5] = px;
                        r[2] = cls == 0 ? qz : pz;
                        r[3] = cls == 0 ? pz : qz;
                        uint64_t v[4], Sq;
                        quad_values(r, v, Sq);
                        if ((a.flags & PS4_F_VERIFY) && !quad_roots_ok(v, r)) { record_verify_failure(a, S, v); continue; }
                        if (a.flags & PS4_F_DUMP4) dump_quad(a, r);
                        atomicAdd(&ts.n_quads, 1u);
                        if (a.flags & PS4_F_NOEXT) continue;
                        const uint32_t si = atomicAdd(&ts.n_staged, 1u);
                        if (si >= cap) { raise_capacity(a.status, E_TILE, 3, si + 1, cap, S0); continue; }
                        int bi, bj, bk;
                        uint32_t best;
                        choose_pair(v, r, a.ndiv, bi, bj, bk, best);
                        const uint32_t bin = min(31 - __clz(best | 1), NBIN - 1);
                        scr[0 * cap + si] = r[0] | (bin << 22) | ((uint32_t)bi << 26) | ((uint32_t)bj << 28) |
                                            ((uint32_t)bk << 30);
                        scr[1 * cap + si] = r[1];
                        scr[2 * cap + si] = r[2];
                        scr[3 * cap + si] = r[3];
                        scr[4 * cap + si] = r[4];
                        scr[5 * cap + si] = r[5];
                    }
                }
            }
            __syncthreads();
            const uint32_t staged = min(ts.n_staged, cap);
            if (staged > 0 && (staged >= L::FLUSH_AT || wave + BS >= nPairs)) {      // block-uniform
                extend_staged<TL>(a, ts, scr, perm, el, staged, ts.flushed, c_cand, c_sqrt, c_mdiv);
                if (tid == 0) { ts.flushed += staged; ts.n_staged = 0; }
                __syncthreads();
            }
        }
        block_add_ext_counters(ts, c_cand, c_sqrt, c_mdiv);
        __syncthreads();
        // P7
        if (tid == 0) {
            ts.cnt[K_SETS4] += ts.n_quads;
            if (ts.elist_n) tile_report(a, ts, el, min(ts.elist_n, L::ELIST_CAP), item);
        }
        __syncthreads();
        tile_flush_counters(a, ts, item);
        __syncthreads();
    }
}

// ================================================================== plain kernel

// One CTA per tile, one thread per selected S: every triple of representations, both
// classes, positivity tested per triple, each 4-set extended on the spot by the same
// thread -- the straightforward GPU transcription of process_chunk/handle_4set.
template <int TL>
__global__ void __launch_bounds__(BS, 1) search_plain(const SearchArgs a) {
    using L = TileLayout<TL>;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ TileShared ts;
    __shared__ ExtEntry el[64];
    const int tid = threadIdx.x;
    tile_reset(ts);
    __syncthreads();
    uint32_t item, n;
    uint64_t S0;
    tile_bounds(a, blockIdx.x, TL, item, S0, n);
    if (!tile_reps<TL>(a, ts, smem, S0, n)) return;
    const uint16_t *is_off = (const uint16_t *)(smem + L::OFF_IS_OFF);
    const uint16_t *is_k = (const uint16_t *)(smem + L::OFF_IS_K);
    const uint16_t *is_start = (const uint16_t *)(smem + L::OFF_IS_START);
    const uint32_t *rep_p = (const uint32_t *)(smem + L::OFF_REP_P);
    const uint32_t *rep_q = (const uint32_t *)(smem + L::OFF_REP_Q);
    ull c_cand = 0, c_sqrt = 0, c_quads = 0;
    uint32_t c_mdiv = 0;
    for (uint32_t s = tid; s < ts.n_is; s += BS) {
        const uint32_t st = is_start[s], k = is_k[s];
        const uint64_t S = S0 + is_off[s];
        const int Sodd = (int)(S & 1);
        for (uint32_t x = 0; x < k; x++)
            for (uint32_t y = x + 1; y < k; y++)
                for (uint32_t z = y + 1; z < k; z++) {
                    const uint64_t pxl = rep_p[st + x], pyl = rep_p[st + y], pzl = rep_p[st + z];
                    const uint64_t Px = pxl * pxl, Py = pyl * pyl, Pz = pzl * pzl;
                    const int par = (int)((pxl + pyl + pzl) & 1);
                    for (int cls = 0; cls < 2; cls++) {
                        if (cls == 0 ? par != 0 : (par != Sodd || S - Pz == Pz)) continue;
                        const int64_t x1 = (int64_t)(S - Px), x2 = (int64_t)(S - Py),
                                      x3 = (int64_t)(cls == 0 ? S - Pz : Pz), SS = (int64_t)S;
                        const int64_t aa = (x1 + x2 + x3 - SS) / 2, bb = (x1 - x2 - x3 + SS) / 2,
                                      cc = (-x1 + x2 - x3 + SS) / 2, dd = (-x1 - x2 + x3 + SS) / 2;
                        if (aa <= 0 || bb <= 0 || cc <= 0 || dd <= 0) continue;
                        uint32_t r[6];
                        r[0] = rep_q[st + x]; r[1] = rep_q[st + y]; r[4] = (uint32_t)pyl; r[5] = (uint32_t)pxl;
                        r[2] = cls == 0 ? rep_q[st + z] : (uint32_t)pzl;
                        r[3] = cls == 0 ? (uint32_t)pzl : rep_q[st + z];
                        const uint64_t v[4] = {(uint64_t)aa, (uint64_t)bb, (uint64_t)cc, (uint64_t)dd};
                        if ((a.flags & PS4_F_VERIFY) && !quad_roots_ok(v, r)) { record_verify_failure(a, S, v); continue; }
                        c_quads++;
                        if (a.flags & PS4_F_DUMP4) dump_quad(a, r);
                        if (a.flags & PS4_F_NOEXT) continue;
                        int bi, bj, bk;
                        uint32_t best;
                        choose_pair(v, r, a.ndiv, bi, bj, bk, best);
                        const uint32_t qid = atomicAdd(&ts.n_quads, 1u);
                        extend_quad(a, r, v, S, bi, bj, bk, qid, c_cand, c_sqrt, c_mdiv, el, &ts.elist_n, 64);
                    }
                }
    }
    block_add_ext_counters(ts, c_cand, c_sqrt, c_mdiv);
    c_quads = warp_sum(c_quads);
    if ((tid & 31) == 0 && c_quads) atomicAdd(&ts.cnt[K_SETS4], c_quads);
    __syncthreads();
    if (tid == 0 && ts.elist_n) tile_report(a, ts, el, min(ts.elist_n, 64u), item);
    __syncthreads();
    tile_flush_counters(a, ts, item);
}

// ================================================================== tables

// spf[m] | (m / spf[m]) << 32 and the divisor count of m, for m < n, by trial division
// (s4.c:439-447 builds the same tables with sieves; spf[0]=0, spf[1]=1, quot[1]=1).
__global__ void build_tables(uint64_t *spfq, uint16_t *ndiv, uint64_t n) {
    for (uint64_t m = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; m < n; m += (uint64_t)gridDim.x * blockDim.x) {
        if (m < 2) {
            spfq[m] = m | (m << 32);
            ndiv[m] = (uint16_t)m;
            continue;
        }
        uint32_t x = (uint32_t)m, sp = 0, nd = 1;
        for (uint32_t d = 2; d * d <= x; d += (d == 2 ? 1 : 2)) {
            if (x % d) continue;
            if (!sp) sp = d;
            uint32_t e = 0;
            while (x % d == 0) { x /= d; e++; }
            nd *= e + 1;
        }
        if (x > 1) { if (!sp) sp = x; nd *= 2; }
        spfq[m] = (uint64_t)sp | ((uint64_t)((uint32_t)m / sp) << 32);
        ndiv[m] = (uint16_t)nd;
    }
}

// ================================================================== launchers

int search_block_threads() { return BS; }

// staging per CTA: FLUSH_AT plus the most one P5 wave can stage, BS pairs x 2(k-2) 4-sets each
uint32_t stage_cap_for(unsigned log2_tile, uint32_t cap_reps) {
    const uint32_t k = cap_reps > 2 ? cap_reps : 3;
    return (1u << log2_tile) / 2 + (uint32_t)BS * 2u * (k - 2u);
}

size_t search_smem_bytes(int kernel, unsigned log2_tile) {
    (void)kernel;
    switch (log2_tile) {
        case 12: return TileLayout<12>::BYTES;
        case 13: return TileLayout<13>::BYTES;
        default: return TileLayout<14>::BYTES;
    }
}

template <int TL>
static int launch_tl(const SearchArgs &a, int kernel, int grid, cudaStream_t s) {
    const size_t smem = TileLayout<TL>::BYTES;
    if (kernel == PS4_KERNEL_PLAIN) {
        cudaFuncSetAttribute(search_plain<TL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        search_plain<TL><<<(unsigned)a.n_tiles, BS, smem, s>>>(a);
    } else {
        cudaFuncSetAttribute(search_batched<TL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        search_batched<TL><<<grid, BS, smem, s>>>(a);
    }
    return (int)cudaGetLastError();
}

int launch_search(const SearchArgs &a, int kernel, int grid, void *stream) {
    cudaStream_t s = (cudaStream_t)stream;
    switch (a.log2_tile) {
        case 12: return launch_tl<12>(a, kernel, grid, s);
        case 13: return launch_tl<13>(a, kernel, grid, s);
        default: return launch_tl<14>(a, kernel, grid, s);
    }
}

int launch_tables(uint64_t *spfq, uint16_t *ndiv, uint64_t tab_n, void *stream) {
    build_tables<<<1184, 256, 0, (cudaStream_t)stream>>>(spfq, ndiv, tab_n);
    return (int)cudaGetLastError();
}

}  // namespace ps4

// ================================================================== allocation-free variant
//
// ps4_search_range_noalloc (include/ps4.h) runs a variant of the batched kernel whose only
// device memory beyond the context's read-only factor tables is one file-scope array,
// ps4_noalloc_scratch below: the per-CTA 4-set staging plus small fixed result buffers.

namespace ps4 {
namespace noalloc {
constexpr int TL = 12;                        // S values per tile: 4096
constexpr uint32_t CTAS = 148;                // at most one CTA per SM of a B200
constexpr uint32_t STAGE = 16384;             // staged 4-sets per CTA
constexpr uint32_t HITS = 65536, EXTS = 131072, SIXES = 256;
constexpr size_t al(size_t x) { return (x + 255) & ~(size_t)255; }
constexpr size_t OFF_STAGE = 0;
constexpr size_t OFF_STATUS = al(OFF_STAGE + (size_t)CTAS * 6 * STAGE * sizeof(uint32_t));
constexpr size_t OFF_COUNTERS = al(OFF_STATUS + sizeof(Status));
constexpr size_t OFF_ITEM = al(OFF_COUNTERS + K_SLOTS * sizeof(unsigned long long));
constexpr size_t OFF_HITS = al(OFF_ITEM + sizeof(Item));
constexpr size_t OFF_EXTS = al(OFF_HITS + (size_t)HITS * sizeof(ps4_hit));
constexpr size_t OFF_SIXES = al(OFF_EXTS + (size_t)EXTS * sizeof(ps4_ext));
constexpr size_t BYTES = al(OFF_SIXES + (size_t)SIXES * sizeof(ps4_six));   // 65.5 MB (62.5 MiB)
}  // namespace noalloc

// The batched kernel with a fixed staging of STAGE 4-sets per CTA: the width of each P5 wave
// (representation pairs emitted before the staging is checked) is set per tile from its
// largest representation count k, so that one wave stages at most 2(k-2) 4-sets per pair
// on top of FLUSH_AT and can never overflow the staging.  Otherwise as search_batched.
template <int TL>
__global__ void __launch_bounds__(BS, 1) search_batched_fixed(const SearchArgs a) {
    using L = TileLayout<TL>;
    extern __shared__ __align__(16) unsigned char smem[];
    __shared__ TileShared ts;
    const uint32_t cap = a.stage_cap;
    uint32_t *scr = a.scratch + (size_t)blockIdx.x * 6 * cap;
    const int tid = threadIdx.x;
    ExtEntry *el = (ExtEntry *)(smem + L::OFF_ELIST);
    uint16_t *perm = (uint16_t *)(smem + L::OFF_CNT);

    for (;;) {
        tile_reset(ts);
        if (tid == 0) {
            ts.tile = atomicAdd((unsigned int *)&a.status->tile_next, 1u);
            ts.skip = *(volatile ull *)&a.status->err != 0ull;
        }
        __syncthreads();
        const uint64_t tile = ts.tile;
        if (tile >= a.n_tiles || ts.skip) break;
        uint32_t item, n;
        uint64_t S0;
        tile_bounds(a, tile, TL, item, S0, n);
        if (!tile_reps<TL>(a, ts, smem, S0, n)) { __syncthreads(); continue; }

        const uint16_t *is_off = (const uint16_t *)(smem + L::OFF_IS_OFF);
        const uint16_t *is_k = (const uint16_t *)(smem + L::OFF_IS_K);
        const uint16_t *is_start = (const uint16_t *)(smem + L::OFF_IS_START);
        const uint32_t *is_pbase = (const uint32_t *)(smem + L::OFF_IS_PBASE);
        const uint32_t *rep_p = (const uint32_t *)(smem + L::OFF_REP_P);
        const uint32_t *rep_q = (const uint32_t *)(smem + L::OFF_REP_Q);
        const uint32_t nI = ts.n_is, nPairs = ts.n_pairs;
        const uint32_t kmax = (uint32_t)ts.cnt[K_MAX_REPS];
        const uint32_t per_pair = 2u * (kmax > 2 ? kmax - 2 : 1);
        const uint32_t wave_w = max(1u, min((uint32_t)BS, (cap - L::FLUSH_AT) / per_pair));
        ull c_cand = 0, c_sqrt = 0;
        uint32_t c_mdiv = 0;

        for (uint32_t wave = 0; wave < nPairs; wave += wave_w) {
            const uint32_t gidx = wave + tid;
            if (tid < wave_w && gidx < nPairs) {
                uint32_t lo = 0, hi = nI;
                while (hi - lo > 1) {
                    const uint32_t mid = (lo + hi) >> 1;
                    if (is_pbase[mid] <= gidx) lo = mid; else hi = mid;
                }
                const uint32_t st = is_start[lo], k = is_k[lo];
                const uint64_t S = S0 + is_off[lo];
                uint32_t x, y;
                decode_pair(gidx - is_pbase[lo], x, y);
                const uint32_t px = rep_p[st + x], qx = rep_q[st + x], py = rep_p[st + y], qy = rep_q[st + y];
                const uint64_t Px = (uint64_t)px * px, Py = (uint64_t)py * py;
                const uint32_t pxy = (px + py) & 1;
                const uint32_t Sodd = (uint32_t)(S & 1);
                for (int cls = 0; cls < 2; cls++) {
                    const uint32_t want = cls == 0 ? 0u : Sodd;
                    for (uint32_t z = cls == 0 ? y + 1 : k - 1; z > y && z < k; z = cls == 0 ? z + 1 : z - 1) {
                        const uint32_t pz = rep_p[st + z];
                        const uint64_t Pz = (uint64_t)pz * pz;
                        if (cls == 0 ? Pz >= Px + Py : Pz <= S - Px - Py) break;
                        if (((pxy + pz) & 1) != want) continue;
                        const uint32_t qz = rep_q[st + z];
                        if (cls == 1 && qz == pz) continue;
                        uint32_t r[6];
                        r[0] = qx; r[1] = qy; r[4] = py; r[5] = px;
                        r[2] = cls == 0 ? qz : pz;
                        r[3] = cls == 0 ? pz : qz;
                        uint64_t v[4], Sq;
                        quad_values(r, v, Sq);
                        if ((a.flags & PS4_F_VERIFY) && !quad_roots_ok(v, r)) { record_verify_failure(a, S, v); continue; }
                        atomicAdd(&ts.n_quads, 1u);
                        if (a.flags & PS4_F_NOEXT) continue;
                        const uint32_t si = atomicAdd(&ts.n_staged, 1u);
                        if (si >= cap) { raise_capacity(a.status, E_TILE, 3, si + 1, cap, S0); continue; }
                        int bi, bj, bk;
                        uint32_t best;
                        choose_pair(v, r, a.ndiv, bi, bj, bk, best);
                        const uint32_t bin = min(31 - __clz(best | 1), NBIN - 1);
                        scr[0 * cap + si] = r[0] | (bin << 22) | ((uint32_t)bi << 26) | ((uint32_t)bj << 28) |
                                            ((uint32_t)bk << 30);
                        scr[1 * cap + si] = r[1];
                        scr[2 * cap + si] = r[2];
                        scr[3 * cap + si] = r[3];
                        scr[4 * cap + si] = r[4];
                        scr[5 * cap + si] = r[5];
                    }
                }
            }
            __syncthreads();
            const uint32_t staged = min(ts.n_staged, cap);
            if (staged > 0 && (staged >= L::FLUSH_AT || wave + wave_w >= nPairs)) {
                extend_staged<TL>(a, ts, scr, perm, el, staged, ts.flushed, c_cand, c_sqrt, c_mdiv);
                if (tid == 0) { ts.flushed += staged; ts.n_staged = 0; }
                __syncthreads();
            }
        }
        block_add_ext_counters(ts, c_cand, c_sqrt, c_mdiv);
        __syncthreads();
        if (tid == 0) {
            ts.cnt[K_SETS4] += ts.n_quads;
            if (ts.elist_n) tile_report(a, ts, el, min(ts.elist_n, L::ELIST_CAP), item);
        }
        __syncthreads();
        tile_flush_counters(a, ts, item);
        __syncthreads();
    }
}
}  // namespace ps4

// The whole device memory of ps4_search_range_noalloc beyond the caller's context: loaded
// with the library's device code on every GPU that runs it, held until the process exits.
static __device__ __align__(256) unsigned char ps4_noalloc_scratch[ps4::noalloc::BYTES];

extern "C" int ps4_search_range_noalloc(ps4_ctx *ctx, uint64_t lo, uint64_t hi, ps4_stats *stats, ps4_results *res) {
    using namespace ps4;
    namespace na = ps4::noalloc;
    CtxView v;
    if (ctx_view(ctx, &v) != PS4_OK) return PS4_ERR_ARG;
    if (!stats || !res) return ctx_fail(ctx, PS4_ERR_ARG, "ps4_search_range_noalloc: stats and res are required");
    if (v.flags & PS4_F_DUMP4)
        return ctx_fail(ctx, PS4_ERR_ARG, "ps4_search_range_noalloc: --dump4 output has no fixed bound; use ps4_search_range");
    if (v.cap_reps > 512)
        return ctx_fail(ctx, PS4_ERR_ARG, "ps4_search_range_noalloc: its fixed 4-set staging supports cap_reps <= 512");
    if (lo < 1) lo = 1;
    if (hi < lo) hi = lo;
    if (hi > v.s_hi_max)
        return ctx_fail(ctx, PS4_ERR_ARG, "ps4_search_range_noalloc: S_hi exceeds the context's s_hi_max");
    const uint64_t n_tiles = (hi - lo + (1ull << na::TL) - 1) >> na::TL;
    if (n_tiles >= (1ull << 31))
        return ctx_fail(ctx, PS4_ERR_ARG, "ps4_search_range_noalloc: range too large for one call; split it");
    res->n_hits = res->n_exts = res->n_sixes = res->n_quads = 0;
    if (n_tiles == 0) return PS4_OK;

    // Once per device, with that device current: the device address of the static array.
    // (The host-side name ps4_noalloc_scratch is only a stand-in and must not reach a kernel.)
    static void *base_of[64];
    if (v.device < 0 || v.device >= 64) return ctx_fail(ctx, PS4_ERR_ARG, "device ordinal out of range");
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess) return ctx_fail(ctx, PS4_ERR_CUDA, "cudaGetDevice failed");
    if (prev != v.device && cudaSetDevice(v.device) != cudaSuccess)
        return ctx_fail(ctx, PS4_ERR_CUDA, "cudaSetDevice failed");
    int rc = PS4_OK;
    char msg[256];
    do {
        if (!base_of[v.device]) {
            void *p = nullptr;
            cudaError_t e = cudaGetSymbolAddress(&p, ps4_noalloc_scratch);
            if (e != cudaSuccess) {
                snprintf(msg, sizeof msg, "cudaGetSymbolAddress(ps4_noalloc_scratch) failed: %s", cudaGetErrorString(e));
                rc = ctx_fail(ctx, PS4_ERR_CUDA, msg);
                break;
            }
            base_of[v.device] = p;
        }
        unsigned char *base = (unsigned char *)base_of[v.device];
        Status *d_status = (Status *)(base + na::OFF_STATUS);
        unsigned long long *d_counters = (unsigned long long *)(base + na::OFF_COUNTERS);
        Item *d_item = (Item *)(base + na::OFF_ITEM);
        cudaStream_t s = (cudaStream_t)v.stream;
        Item it;
        it.lo = lo; it.hi = hi; it.tile_base = 0;
        SearchArgs a;
        memset(&a, 0, sizeof a);
        a.items = d_item; a.n_items = 1; a.n_tiles = n_tiles; a.log2_tile = na::TL;
        a.spfq = v.spfq; a.ndiv = v.ndiv; a.tab_n = v.tab_n;
        a.counters = d_counters;
        a.hits = (ps4_hit *)(base + na::OFF_HITS); a.hits_cap = na::HITS;
        a.exts = (ps4_ext *)(base + na::OFF_EXTS); a.exts_cap = na::EXTS;
        a.sixes = (ps4_six *)(base + na::OFF_SIXES); a.sixes_cap = na::SIXES;
        a.scratch = (uint32_t *)(base + na::OFF_STAGE); a.stage_cap = na::STAGE;
        a.status = d_status;
        a.cap_reps = v.cap_reps; a.cap_divs = v.cap_divs; a.cap_ext = v.cap_ext;
        a.flags = v.flags & ~(uint32_t)PS4_F_DUMP4;
        const unsigned grid = (unsigned)std::min<uint64_t>(std::min<uint64_t>(na::CTAS, (uint64_t)v.num_sms), n_tiles);
        const size_t smem = TileLayout<na::TL>::BYTES;
        // what must start at zero: the status (error word, record counts, tile counter) and the counters
        cudaError_t e = cudaMemcpyAsync(d_item, &it, sizeof it, cudaMemcpyHostToDevice, s);
        if (e == cudaSuccess) e = cudaMemsetAsync(d_status, 0, sizeof(Status), s);
        if (e == cudaSuccess) e = cudaMemsetAsync(d_counters, 0, K_SLOTS * sizeof(unsigned long long), s);
        if (e == cudaSuccess)
            e = cudaFuncSetAttribute(search_batched_fixed<na::TL>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
        if (e == cudaSuccess) {
            search_batched_fixed<na::TL><<<grid, BS, smem, s>>>(a);
            e = cudaGetLastError();
        }
        Status st;
        if (e == cudaSuccess) e = cudaMemcpyAsync(&st, d_status, sizeof st, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            snprintf(msg, sizeof msg, "ps4_search_range_noalloc: %s", cudaGetErrorString(e));
            rc = ctx_fail(ctx, PS4_ERR_CUDA, msg);
            break;
        }
        const unsigned code = (unsigned)(st.err & 0xFF);
        if (code == E_CAP_REPS || code == E_CAP_DIVS || code == E_CAP_EXT) {
            const char *what = code == E_CAP_REPS ? "representation" : code == E_CAP_DIVS ? "divisor" : "extension";
            snprintf(msg, sizeof msg, "FATAL: %s capacity exceeded; this interval is NOT certified complete", what);
            rc = ctx_fail(ctx, (int)code, msg);
            break;
        }
        if (code == E_VERIFY) {
            snprintf(msg, sizeof msg, "BAD 4-set S=%llu [%lld,%lld,%lld,%lld]", st.verify_bad[0],
                     (long long)st.verify_bad[1], (long long)st.verify_bad[2], (long long)st.verify_bad[3],
                     (long long)st.verify_bad[4]);
            rc = ctx_fail(ctx, PS4_ERR_VERIFY, msg);
            break;
        }
        if (code != 0) {
            snprintf(msg, sizeof msg, "ps4_search_range_noalloc: a tile near S=%llu outgrew the fixed shared-memory "
                     "lists; search it with ps4_search_range", st.err >> 8);
            rc = ctx_fail(ctx, PS4_ERR_CAP_REPS, msg);
            break;
        }
        if (st.n_hits > na::HITS || st.n_exts > na::EXTS || st.n_sixes > na::SIXES) {
            snprintf(msg, sizeof msg, "ps4_search_range_noalloc: %u result records exceed the fixed buffers "
                     "(%u hits); search a shorter range", st.n_hits, na::HITS);
            rc = ctx_fail(ctx, PS4_ERR_OUTPUT_FULL, msg);
            break;
        }
        res->n_hits = st.n_hits; res->n_exts = st.n_exts; res->n_sixes = st.n_sixes;
        if (res->n_hits > res->hits_cap || res->n_exts > res->exts_cap || res->n_sixes > res->sixes_cap) {
            rc = ctx_fail(ctx, PS4_ERR_OUTPUT_FULL, "ps4_search_range_noalloc: result buffers too small; n_* hold the sizes");
            break;
        }
        unsigned long long k[K_SLOTS];
        e = cudaMemcpyAsync(k, d_counters, sizeof k, cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess && st.n_hits)
            e = cudaMemcpyAsync(res->hits, a.hits, st.n_hits * sizeof(ps4_hit), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess && st.n_exts)
            e = cudaMemcpyAsync(res->exts, a.exts, st.n_exts * sizeof(ps4_ext), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess && st.n_sixes)
            e = cudaMemcpyAsync(res->sixes, a.sixes, st.n_sixes * sizeof(ps4_six), cudaMemcpyDeviceToHost, s);
        if (e == cudaSuccess) e = cudaStreamSynchronize(s);
        if (e != cudaSuccess) {
            snprintf(msg, sizeof msg, "ps4_search_range_noalloc: %s", cudaGetErrorString(e));
            rc = ctx_fail(ctx, PS4_ERR_CUDA, msg);
            break;
        }
        uint64_t *add = &stats->S_done;
        for (int i = 0; i < 10; i++) add[i] += k[i];
        for (int i = 0; i < 100; i++) stats->hist5[i] += k[K_HIST5 + i];
        stats->max_reps = std::max<uint64_t>(stats->max_reps, k[K_MAX_REPS]);
        stats->max_divisors = std::max<uint64_t>(stats->max_divisors, k[K_MAX_DIVS]);
        stats->max_extensions = std::max<uint64_t>(stats->max_extensions, k[K_MAX_EXT]);
    } while (0);
    if (prev != v.device) cudaSetDevice(prev);
    return rc;
}
