// ps4_device.cuh -- device building blocks shared by the sm_100a kernels of the search:
// exact integer roots, residue masks, 4-set helpers, the factor walk, the per-lane divisor
// odometer (extend_quad), the tile phases P1-P4 (tile_reps) and the report step P7.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>

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

// floor(sqrt(n)) for any n < 2^128, exact.  The double estimate is within a few units of the
// root; the increment loop stops at 2^64-1, whose successor's square no longer fits.
__device__ __forceinline__ uint64_t isqrt128(u128 n) {
    if ((n >> 64) == 0) return isqrt64((uint64_t)n);
    const double x = sqrt(u128_to_double(n));
    uint64_t r = x >= 18446744073709551615.0 ? ~0ull : (uint64_t)x;
    while ((u128)r * r > n) r--;
    while (r != ~0ull && (u128)(r + 1) * (r + 1) <= n) r++;
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

// Factor table entry of m >= 2 (build_tables): its smallest prime p (bits 0..23), the exponent
// of p in m (bits 24..31) and the cofactor m / p^e (bits 32..63), so a walk takes one
// dependent load per distinct prime.
__device__ __forceinline__ uint32_t spf_p(uint64_t t) { return (uint32_t)t & 0xFFFFFFu; }
__device__ __forceinline__ uint32_t spf_e(uint64_t t) { return ((uint32_t)t >> 24) & 0xFFu; }
__device__ __forceinline__ uint32_t spf_cof(uint64_t t) { return (uint32_t)(t >> 32); }

// Merge the factorisation of m into (pr, ex, np), primes in first-seen order of the
// smallest-prime-factor walk (s4.c:141-147): ascending within m.  The power of two is
// taken by counting trailing zeros.
__device__ __forceinline__ void factor_merge(const uint64_t *spfq, uint32_t m, uint32_t *pr, uint8_t *ex, int &np) {
    auto merge = [&](uint32_t p, uint32_t e) {
        int i = 0;
        while (i < np && pr[i] != p) i++;
        if (i == np) { pr[np] = p; ex[np] = 0; np++; }
        ex[i] = (uint8_t)(ex[i] + e);
    };
    if (m > 1 && !(m & 1)) {
        const uint32_t z = (uint32_t)__ffs((int)m) - 1;
        merge(2, z);
        m >>= z;
    }
    while (m > 1) {
        const uint64_t t = __ldg(&spfq[m]);
        merge(spf_p(t), spf_e(t));
        m = spf_cof(t);
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
__device__ inline void extend_quad(const SearchArgs &a, const uint32_t r[6], const uint64_t v[4], uint64_t S,
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
            // e + C < u^2 + S < 2^89 (u <= (D+1)/2 < 2^44): inside is_square_fast's n < 2^100
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

// exclusive block scan of three u32 values over NT threads; returns totals in tot[3]
template <int NT = BS>
__device__ __forceinline__ void block_scan3(uint32_t x0, uint32_t x1, uint32_t x2, uint32_t &e0, uint32_t &e1,
                                            uint32_t &e2, uint32_t tot[3], uint32_t *wsum /* 3*NWARP; 3*NT/32 used */) {
    constexpr int NW = NT / 32;
    const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
    uint32_t i0 = x0, i1 = x1, i2 = x2;
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        uint32_t y0 = __shfl_up_sync(0xffffffffu, i0, o), y1 = __shfl_up_sync(0xffffffffu, i1, o),
                 y2 = __shfl_up_sync(0xffffffffu, i2, o);
        if (lane >= o) { i0 += y0; i1 += y1; i2 += y2; }
    }
    if (lane == 31) { wsum[wid] = i0; wsum[NW + wid] = i1; wsum[2 * NW + wid] = i2; }
    __syncthreads();
    if (wid == 0) {
        uint32_t s0 = lane < NW ? wsum[lane] : 0, s1 = lane < NW ? wsum[NW + lane] : 0,
                 s2 = lane < NW ? wsum[2 * NW + lane] : 0;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            uint32_t y0 = __shfl_up_sync(0xffffffffu, s0, o), y1 = __shfl_up_sync(0xffffffffu, s1, o),
                     y2 = __shfl_up_sync(0xffffffffu, s2, o);
            if (lane >= o) { s0 += y0; s1 += y1; s2 += y2; }
        }
        if (lane < NW) { wsum[lane] = s0; wsum[NW + lane] = s1; wsum[2 * NW + lane] = s2; }
    }
    __syncthreads();
    const uint32_t b0 = wid ? wsum[wid - 1] : 0, b1 = wid ? wsum[NW + wid - 1] : 0,
                   b2 = wid ? wsum[2 * NW + wid - 1] : 0;
    e0 = b0 + i0 - x0; e1 = b1 + i1 - x1; e2 = b2 + i2 - x2;
    tot[0] = wsum[NW - 1]; tot[1] = wsum[2 * NW - 1]; tot[2] = wsum[3 * NW - 1];
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

// locate a tile: tiles are handed out highest-S first (longest work first); `item` is the
// query item of the segment holding the tile
__device__ __forceinline__ void tile_bounds(const SearchArgs &a, uint64_t tile, unsigned TLv, uint32_t &item,
                                            uint64_t &S0, uint32_t &n) {
    const uint64_t ti = a.n_tiles - 1 - tile;
    uint32_t lo = 0, hi = a.n_items;                   // last item with tile_base <= ti
    while (hi - lo > 1) {
        const uint32_t mid = (lo + hi) >> 1;
        if (a.items[mid].tile_base <= ti) lo = mid; else hi = mid;
    }
    const Item it = a.items[lo];
    item = it.id;
    S0 = it.lo + ((ti - it.tile_base) << TLv);
    const uint64_t S1 = S0 + (1ull << TLv) < it.hi ? S0 + (1ull << TLv) : it.hi;
    n = (uint32_t)(S1 - S0);
}

// floor(sqrt(x)) for x < 2^46: a float estimate is within one unit of the root (the root is
// < 2^23 and float carries 24 bits), then exact integer correction (products < 2^47).
__device__ __forceinline__ uint32_t isqrt_lt2p46(uint64_t x) {
    uint32_t r = (uint32_t)sqrtf((float)x);
    while ((uint64_t)r * r > x) r--;
    while ((uint64_t)(r + 1) * (r + 1) <= x) r++;
    return r;
}

// P1 / P3: scan every representation S = p^2 + q^2, 1 <= p <= q, S in [S0, S0+n).
// q-major: q runs over [ceil(sqrt(S0/2)), isqrt(S1-2)] (strided over the threads), p from
// ceil(sqrt(S0-q^2)) by a float estimate with exact integer correction (S < 2^44).
template <bool FILL, int NT = BS>
__device__ __forceinline__ uint32_t scan_reps(uint64_t S0, uint32_t n, uint32_t *cnt32, uint32_t *rep_p,
                                              uint32_t *rep_q) {
    const uint64_t S1 = S0 + n;
    uint32_t qmin = (uint32_t)ceil_sqrt64((S0 + 1) >> 1);
    if (qmin < 1) qmin = 1;
    const uint32_t qmax = S1 >= 2 ? (uint32_t)isqrt64(S1 - 2) : 0;
    uint32_t found = 0;
    for (uint32_t q = qmin + threadIdx.x; q <= qmax; q += NT) {
        const uint64_t q2 = (uint64_t)q * q;
        uint32_t p = 1;
        if (S0 > q2 + 1) {
            const uint64_t m = S0 - q2;                // p = ceil(sqrt(m))
            const uint32_t r = isqrt_lt2p46(m);
            p = r + ((uint64_t)r * r < m ? 1u : 0u);
        }
        for (uint64_t s = (uint64_t)p * p + q2; p <= q && s < S1; s += 2 * p + 1, p++) {
            const uint32_t i = (uint32_t)(s - S0), w = i >> 1, sh = (i & 1) * 16;
            if (!FILL) {
                atomicAdd(&cnt32[w], 1u << sh);
                found++;
            } else {
                const uint32_t cur = (((volatile uint32_t *)cnt32)[w] >> sh) & 0xFFFFu;
                if (cur == 0xFFFFu) continue;          // S not selected
                const uint32_t pos = (atomicAdd(&cnt32[w], 1u << sh) >> sh) & 0xFFFFu;
                rep_p[pos] = p;
                rep_q[pos] = q;
            }
        }
    }
    return found;
}

// The scan of scan_reps over a group of up to SUPER_K adjacent tiles [SS0, SS1) of one
// segment, done once: every representation goes to its tile's list (offset in the tile | p << 14 |
// q << 36; p <= q < 2^22, offset < 2^14), in the slice of the warp that found it (one shared
// atomic per representation).  Slice counts above `slice` mean the list overflowed; that tile
// then scans for itself.  NT threads, NT/32 warp slices per tile.
template <int NT = BS>
__device__ __forceinline__ void scan_group(uint64_t SS0, uint64_t SS1, unsigned TLv, uint64_t *lists,
                                           uint32_t list_cap, uint32_t *raw_n, uint32_t slice) {
    uint32_t qmin = (uint32_t)ceil_sqrt64((SS0 + 1) >> 1);
    if (qmin < 1) qmin = 1;
    const uint32_t qmax = SS1 >= 2 ? (uint32_t)isqrt64(SS1 - 2) : 0;
    const int wid = threadIdx.x >> 5;
    const uint32_t wmask = (1u << TLv) - 1u;
    for (uint32_t q = qmin + threadIdx.x; q <= qmax; q += NT) {
        const uint64_t q2 = (uint64_t)q * q;
        uint32_t p = 1;
        if (SS0 > q2 + 1) {
            const uint64_t m = SS0 - q2;
            const uint32_t r = isqrt_lt2p46(m);
            p = r + ((uint64_t)r * r < m ? 1u : 0u);
        }
        for (uint64_t s = (uint64_t)p * p + q2; p <= q && s < SS1; s += 2 * p + 1, p++) {
            const uint32_t i = (uint32_t)(s - SS0), j = i >> TLv;
            const uint32_t pos = atomicAdd(&raw_n[j * (NT / 32) + wid], 1u);
            if (pos < slice)
                lists[(size_t)j * list_cap + (size_t)wid * slice + pos] =
                    (uint64_t)(i & wmask) | ((uint64_t)p << 14) | ((uint64_t)q << 36);
        }
    }
}

// P1-P4 for one tile.  Returns false if the tile was abandoned (error raised).  With `list` (the
// tile's representations from scan_group, list_n[w] entries in warp slice w of `slice`) P1 and
// P3 read the list; without, they scan.
template <int TL, int NT = BS>
__device__ bool tile_reps(const SearchArgs &a, TileShared &ts, unsigned char *smem, uint64_t S0, uint32_t n,
                          const uint64_t *list = nullptr, const uint32_t *list_n = nullptr, uint32_t slice = 0) {
    using L = TileLayout<TL>;
    uint32_t *cnt32 = (uint32_t *)(smem + L::OFF_CNT);
    uint16_t *is_off = (uint16_t *)(smem + L::OFF_IS_OFF);
    uint16_t *is_k = (uint16_t *)(smem + L::OFF_IS_K);
    uint16_t *is_start = (uint16_t *)(smem + L::OFF_IS_START);
    uint32_t *is_pbase = (uint32_t *)(smem + L::OFF_IS_PBASE);
    uint32_t *rep_p = (uint32_t *)(smem + L::OFF_REP_P);
    uint32_t *rep_q = (uint32_t *)(smem + L::OFF_REP_Q);
    const int tid = threadIdx.x;

    for (uint32_t i = tid; i < L::W / 2; i += NT) cnt32[i] = 0;
    __syncthreads();
    // P1: count, from the list or by scanning
    uint32_t found = 0;
    if (list) {
        for (int w = 0; w < NT / 32; w++) {
            const uint32_t cw = list_n[w];
            for (uint32_t o = tid; o < cw; o += NT) {
                const uint32_t i = (uint32_t)list[(size_t)w * slice + o] & 0x3FFFu;
                atomicAdd(&cnt32[i >> 1], 1u << ((i & 1) * 16));
                found++;
            }
        }
    } else {
        found = scan_reps<false, NT>(S0, n, cnt32, rep_p, rep_q);
    }
    ull f = warp_sum((ull)found);
    if ((tid & 31) == 0 && f) atomicAdd(&ts.cnt[K_PAIRS], f);
    __syncthreads();

    // P2: select S with >= 3 representations and S != 2 (mod 4).  A thread owns SEG consecutive
    // S, i.e. WT counter words, and visits them from a lane-dependent rotation so that the lanes
    // of a warp touch 32 different banks (in plain order they would all hit the same two)
    constexpr uint32_t SEG = L::W / NT;
    constexpr uint32_t WT = SEG / 2;
    static_assert(WT >= 1 && WT <= 32 && (WT & (WT - 1)) == 0, "counter words per thread: a power of two");
    const uint32_t i0 = tid * SEG, w0 = tid * WT;
    const uint32_t rot = (((uint32_t)tid & 31u) * WT / 32u) & (WT - 1);
    uint32_t nI = 0, nR = 0, nP = 0, kmax = 0;
    ull trip = 0;
    bool over = false;
    for (uint32_t it = 0; it < WT; it++) {
        const uint32_t wi = (it + rot) & (WT - 1);
        const uint32_t word = cnt32[w0 + wi];
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const uint32_t i = i0 + 2 * wi + h;
            const uint32_t k = (word >> (h * 16)) & 0xFFFFu;
            if (i >= n) continue;
            kmax = max(kmax, k);
            if (k >= 3 && ((S0 + i) & 3) != 2) {
                nI++; nR += k; nP += k * (k - 1) / 2;
                trip += (ull)k * (k - 1) * (k - 2) / 6;
                if (k > a.cap_reps) over = true;
            }
        }
    }
    if (over) raise_error(a.status, E_CAP_REPS, S0);
    uint32_t bI, bR, bP, tot[3];
    block_scan3<NT>(nI, nR, nP, bI, bR, bP, tot, ts.wsum);
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
    for (uint32_t it = 0; it < WT; it++) {
        const uint32_t wi = (it + rot) & (WT - 1);
        const uint32_t i = i0 + 2 * wi, cw = cnt32[w0 + wi];
        uint32_t word = 0;
#pragma unroll
        for (int h = 0; h < 2; h++) {
            const uint32_t ii = i + h;
            uint32_t val = 0xFFFFu;
            if (ii < n) {
                const uint32_t k = (cw >> (h * 16)) & 0xFFFFu;
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
    // P3: fill, from the list or by scanning again
    if (list) {
        for (int w = 0; w < NT / 32; w++) {
            const uint32_t cw = list_n[w];
            for (uint32_t o = tid; o < cw; o += NT) {
                const uint64_t e = list[(size_t)w * slice + o];
                const uint32_t i = (uint32_t)e & 0x3FFFu, wd = i >> 1, sh = (i & 1) * 16;
                const uint32_t cur = (((volatile uint32_t *)cnt32)[wd] >> sh) & 0xFFFFu;
                if (cur == 0xFFFFu) continue;          // S not selected
                const uint32_t pos = (atomicAdd(&cnt32[wd], 1u << sh) >> sh) & 0xFFFFu;
                rep_p[pos] = (uint32_t)(e >> 14) & 0x3FFFFFu;
                rep_q[pos] = (uint32_t)(e >> 36);
            }
        }
    } else {
        scan_reps<true, NT>(S0, n, cnt32, rep_p, rep_q);
    }
    __syncthreads();
    // P4: each list ascending in p
    for (uint32_t s = tid; s < ts.n_is; s += NT) {
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
__device__ inline bool verify_set(const u128 *x, int n) {
    for (int i = 0; i < n; i++)
        for (int j = i + 1; j < n; j++)
            if (x[i] == x[j] || !is_square_exact(x[i] + x[j])) return false;
    return true;
}

// P7: turn the tile's extension list into hit / ext / six records (s4.c:243-277).
// Runs on one thread; tiles hold a handful of extensions at most.
__device__ inline void tile_report(const SearchArgs &a, TileShared &ts, ExtEntry *el, uint32_t n_el, uint32_t item) {
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

}  // namespace ps4
