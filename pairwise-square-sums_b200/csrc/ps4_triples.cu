// ps4_triples.cu -- batched triple extension: for each square-sum triple {a,b,c}, every d with
// 0 < d <= dmax, d not in the triple, and d+a, d+b, d+c all squares.
//
// The reference has no function for this query; it is its extension step (exhaustive/s4.c:160-207)
// applied to three members instead of four: with A > B two members and C the third,
// e + A = u^2 and e + B = w^2 give (u-w)(u+w) = A - B = D, and D = r_AC^2 - r_BC^2 =
// (r_AC - r_BC)(r_AC + r_BC) factors through the smallest-prime-factor table.  Every pair of
// complementary divisors f, g of equal parity gives u = (f+g)/2 and e = u^2 - A; e + B is then
// a square by construction and e + C is tested exactly.  The pair of members to extend by is
// the one with the fewest estimated divisors, as s4.c:163-171 chooses it.
//
// One warp per triple: every lane factors D (the same few table loads, broadcast), then the
// lanes split the flattened (odd divisor, power of two) index space of the half enumeration
// into 32 contiguous runs, each started by a mixed-radix decode and walked by the odometer.

#include <cuda_runtime.h>
#include <stdint.h>

#include "ps4_device.cuh"

namespace ps4 {

constexpr int TBS = 256;   // threads per CTA of the triple kernel

__global__ void __launch_bounds__(TBS) extend_triples_kernel(const TriArgs t) {
    const int lane = threadIdx.x & 31;
    const uint64_t nwarps = ((uint64_t)gridDim.x * TBS) >> 5;
    ull cand = 0, nsqrt = 0;
    for (uint64_t i = ((uint64_t)blockIdx.x * TBS + threadIdx.x) >> 5; i < t.n; i += nwarps) {
        uint64_t m[3] = {t.abc[3 * i], t.abc[3 * i + 1], t.abc[3 * i + 2]};
        if (m[0] > m[1]) { const uint64_t s = m[0]; m[0] = m[1]; m[1] = s; }
        if (m[1] > m[2]) { const uint64_t s = m[1]; m[1] = m[2]; m[2] = s; }
        if (m[0] > m[1]) { const uint64_t s = m[0]; m[0] = m[1]; m[1] = s; }
        // m[0] < m[1] < m[2] from here on, or the triple is rejected
        int st = TRI_OK;
        uint64_t r01 = 0, r02 = 0, r12 = 0;
        if (m[0] == 0 || m[0] == m[1] || m[1] == m[2]) {
            st = TRI_INVALID;
        } else if (m[2] >= (1ull << 44)) {
            st = TRI_RANGE;
        } else {
            r01 = isqrt64(m[0] + m[1]); r02 = isqrt64(m[0] + m[2]); r12 = isqrt64(m[1] + m[2]);
            if (r01 * r01 != m[0] + m[1] || r02 * r02 != m[0] + m[2] || r12 * r12 != m[1] + m[2]) st = TRI_INVALID;
            else if (r12 + r02 >= t.tab_n) st = TRI_RANGE;
        }
        if (lane == 0) {
            t.state[i] = (uint8_t)st;
            if (st != TRI_OK && t.cand_per) { t.cand_per[i] = 0; t.sqrt_per[i] = 0; }
        }
        if (st != TRI_OK) continue;

        // the three differences A - B with third member C; roots ra = r_AC > rb = r_BC
        const uint64_t cA[3] = {m[2], m[2], m[1]}, cB[3] = {m[1], m[0], m[0]}, cC[3] = {m[0], m[1], m[2]};
        const uint32_t cra[3] = {(uint32_t)r02, (uint32_t)r12, (uint32_t)r12};
        const uint32_t crb[3] = {(uint32_t)r01, (uint32_t)r01, (uint32_t)r02};
        int best = 0;
        uint32_t best_est = 0xFFFFFFFFu;
#pragma unroll
        for (int k = 0; k < 3; k++) {
            const uint32_t est = (uint32_t)__ldg(&t.ndiv[cra[k] - crb[k]]) * __ldg(&t.ndiv[cra[k] + crb[k]]);
            if (est < best_est) { best_est = est; best = k; }
        }
        const uint64_t A = best == 0 ? cA[0] : best == 1 ? cA[1] : cA[2];
        const uint64_t B = best == 0 ? cB[0] : best == 1 ? cB[1] : cB[2];
        const uint64_t C = best == 0 ? cC[0] : best == 1 ? cC[1] : cC[2];
        const uint32_t ra = best == 0 ? cra[0] : best == 1 ? cra[1] : cra[2];
        const uint32_t rb = best == 0 ? crb[0] : best == 1 ? crb[1] : crb[2];
        const uint64_t uA = isqrt64(A);                           // u <= uA: e <= 0
        const uint64_t umax = isqrt64(t.dmax + A);                // u > umax: e > dmax  (dmax + A < 2^63)

        uint32_t pr[MAXP];
        uint8_t ex[MAXP];
        int np = 0;
        factor_merge(t.spfq, ra - rb, pr, ex, np);
        factor_merge(t.spfq, ra + rb, pr, ex, np);
        const bool has2 = np > 0 && pr[0] == 2;                 // D even => both factors even, 4 | D
        const int E2 = has2 ? ex[0] : 0, j0 = has2 ? 1 : 0;
        uint64_t qinv[MAXP];
        uint64_t ndo = 1, Dodd = 1;
        for (int j = j0; j < np; j++) {
            qinv[j] = inv64(pr[j]);
            for (int e = 0; e < ex[j]; e++) Dodd *= pr[j];
            ndo *= (uint64_t)ex[j] + 1;
        }
        // same-parity complementary pairs f < g, the reference's ext_cand (s4.c:191)
        const ull tcand = has2 ? ((uint64_t)(E2 - 1) * ndo) >> 1 : ndo >> 1;
        if (lane == 0) cand += tcand;

        const int64_t dC = (int64_t)C - (int64_t)A;            // e + C = u^2 + (C - A)
        const uint32_t a64 = (uint32_t)dC & 63u;
        const uint32_t a63 = (uint32_t)(((dC % 63) + 63) % 63), a65 = (uint32_t)(((dC % 65) + 65) % 65);

        // flattened index x = todd * W2 + (d2 - dlo) over odd-divisor indices todd <= their
        // complement and 2-exponents d2 of f (both factors even: 1..E2-1)
        const int dlo = has2 ? 1 : 0, dhi = has2 ? E2 - 1 : 0;
        const uint64_t W2 = (uint64_t)(dhi - dlo + 1);
        const uint64_t total = ((ndo + 1) >> 1) * W2;
        const uint64_t run = (total + 31) >> 5;
        const uint64_t x0 = (uint64_t)lane * run, x1 = min(total, x0 + run);
        const ull sqrt0 = nsqrt;
        if (x0 < x1) {
            uint64_t todd = x0 / W2;
            int d2 = dlo + (int)(x0 - todd * W2);
            uint8_t dig[MAXP];
            uint64_t fo = 1, go = Dodd;
            {
                uint64_t x = todd;
                for (int j = j0; j < np; j++) {                       // mixed radix, first prime fastest
                    const uint64_t rdx = (uint64_t)ex[j] + 1, q = x / rdx;
                    dig[j] = (uint8_t)(x - q * rdx);
                    x = q;
                    for (int e = 0; e < dig[j]; e++) { fo *= pr[j]; go *= qinv[j]; }
                }
            }
            for (uint64_t x = x0; x < x1; x++) {
                const bool mid = (2 * todd + 1 == ndo);              // self-complementary odd part
                if (!(mid && 2 * d2 >= E2)) {
                    const uint64_t f = fo << d2, g = go << (E2 - d2);
                    const uint64_t u = (f + g) >> 1;
                    if (u > uA && u <= umax) {
                        const uint32_t w64 = (uint32_t)u & 63u, w63 = (uint32_t)(u % 63), w65 = (uint32_t)(u % 65);
                        if (((QR64 >> ((w64 * w64 + a64) & 63u)) & 1) && ((QR63 >> ((w63 * w63 + a63) % 63u)) & 1) &&
                            qr65((w65 * w65 + a65) % 65u)) {
                            const uint64_t e = u * u - A;             // 0 < e <= dmax
                            if (e != A && e != B && e != C) {
                                nsqrt++;
                                // e <= dmax <= 2^62 and C < 2^44: e + C < 2^63, inside
                                // is_square_fast's n < 2^100
                                if (is_square_fast((u128)(e + C))) {
                                    const unsigned long long slot = atomicAdd(t.n_out, 1ull);
                                    if (slot < t.out_cap) {
                                        ps4_tri_ext rec;
                                        rec.d = e; rec.item = t.item_base + (uint32_t)i; rec.reserved = 0;
                                        t.out[slot] = rec;
                                    }
                                }
                            }
                        }
                    }
                }
                if (++d2 > dhi) {
                    d2 = dlo;
                    todd++;
                    for (int j = j0; j < np; j++) {                   // odometer over the odd primes
                        if (dig[j] < ex[j]) { dig[j]++; fo *= pr[j]; go *= qinv[j]; break; }
                        for (int e = 0; e < dig[j]; e++) { fo *= qinv[j]; go *= pr[j]; }
                        dig[j] = 0;
                    }
                }
            }
        }
        if (t.cand_per) {                                         // per-triple counters (serving)
            const ull ts = warp_sum(nsqrt - sqrt0);
            if (lane == 0) { t.cand_per[i] = tcand; t.sqrt_per[i] = ts; }
        }
    }
    cand = warp_sum(cand);
    nsqrt = warp_sum(nsqrt);
    if (lane == 0) {
        if (cand) atomicAdd(t.n_cand, cand);
        if (nsqrt) atomicAdd(t.n_sqrt, nsqrt);
    }
}

int launch_triples(const TriArgs &t, void *stream) {
    if (t.n == 0) return 0;
    const uint64_t want = (t.n + (TBS / 32) - 1) / (TBS / 32);
    const int grid = (int)(want < 8192 ? want : 8192);
    extend_triples_kernel<<<grid, TBS, 0, (cudaStream_t)stream>>>(t);
    return (int)cudaGetLastError();
}

}  // namespace ps4
