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
#include <mutex>

#include "ps4_internal.h"

#include "ps4_device.cuh"

namespace ps4 {

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
            spfq[m] = 0;
            ndiv[m] = (uint16_t)m;
            continue;
        }
        // entry: smallest prime p | its exponent e << 24 | cofactor m / p^e << 32
        uint32_t x = (uint32_t)m, sp = 0, se = 0, nd = 1;
        for (uint32_t d = 2; d * d <= x; d += (d == 2 ? 1 : 2)) {
            if (x % d) continue;
            uint32_t e = 0;
            while (x % d == 0) { x /= d; e++; }
            if (!sp) { sp = d; se = e; }
            nd *= e + 1;
        }
        if (x > 1) { if (!sp) { sp = x; se = 1; } nd *= 2; }
        uint32_t cof = (uint32_t)m;
        for (uint32_t e = 0; e < se; e++) cof /= sp;
        spfq[m] = (uint64_t)sp | ((uint64_t)se << 24) | ((uint64_t)cof << 32);
        ndiv[m] = (uint16_t)nd;
    }
}

// ================================================================== exact-root self-check

// The search's exact roots on n = hi*2^64 + lo, one thread per value (ps4_check_roots):
// out[4i..4i+3] = isqrt128(n), isqrt64(lo), ceil_sqrt64(lo), isqrt_lt2p46(lo) (the last only
// for lo < 2^46, else 0); flags[i] bit 0 = is_square_exact(n), bit 1 = is_square_fast(n) (only
// for n < 2^100, its precondition; else 0).
__global__ void check_roots(const uint64_t *lo, const uint64_t *hi, uint32_t n, uint64_t *out, uint32_t *flags) {
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const u128 x = ((u128)hi[i] << 64) | lo[i];
    out[4 * (size_t)i + 0] = isqrt128(x);
    out[4 * (size_t)i + 1] = isqrt64(lo[i]);
    out[4 * (size_t)i + 2] = ceil_sqrt64(lo[i]);
    out[4 * (size_t)i + 3] = lo[i] < (1ull << 46) ? isqrt_lt2p46(lo[i]) : 0ull;
    uint32_t f = is_square_exact(x) ? 1u : 0u;
    if ((x >> 100) == 0 && is_square_fast(x)) f |= 2u;
    flags[i] = f;
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

// For odd m (the engine looks up odd parts only): its first three odd primes in ascending order,
// each as p | e << 24, zero where m has fewer, and the cofactor m / (their powers), 1 when none
// is left -- so the engine's factor walk of a difference takes one load for most m and continues
// through spfq from the cofactor otherwise.  The prime order is the smallest-prime walk's
// (s4.c:141-147).  Trial division, one thread per m.
__global__ void build_fac3(uint4 *fac3, uint64_t n) {
    for (uint64_t m = blockIdx.x * (uint64_t)blockDim.x + threadIdx.x; m < n; m += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t w[3] = {0, 0, 0}, k = 0, x = (uint32_t)m;
        if (m >= 2) {
            while (!(x & 1)) x >>= 1;
            for (uint32_t d = 3; d * d <= x && k < 3; d += 2) {
                if (x % d) continue;
                uint32_t e = 0;
                while (x % d == 0) { x /= d; e++; }
                w[k++] = d | (e << 24);
            }
            if (x > 1 && k < 3) { w[k++] = x | (1u << 24); x = 1; }
        }
        fac3[m] = make_uint4(w[0], w[1], w[2], m >= 2 ? x : 1u);
    }
}

int launch_fac3(uint4 *fac3, uint64_t tab_n, void *stream) {
    build_fac3<<<1184, 256, 0, (cudaStream_t)stream>>>(fac3, tab_n);
    return (int)cudaGetLastError();
}

int launch_tables(uint64_t *spfq, uint16_t *ndiv, uint64_t tab_n, void *stream) {
    build_tables<<<1184, 256, 0, (cudaStream_t)stream>>>(spfq, ndiv, tab_n);
    return (int)cudaGetLastError();
}

}  // namespace ps4

// Self-check of the device's exact roots (no context: device buffers of its own, synchronous).
extern "C" int ps4_check_roots(int device, const uint64_t *lo, const uint64_t *hi, uint32_t n, uint64_t *roots,
                               uint32_t *flags) {
    if (n == 0) return PS4_OK;
    if (!lo || !hi || !roots || !flags) return PS4_ERR_ARG;
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess) return PS4_ERR_CUDA;
    uint64_t *d_in = nullptr, *d_out = nullptr;
    uint32_t *d_flags = nullptr;
    cudaError_t e = cudaMalloc((void **)&d_in, 2 * (size_t)n * sizeof(uint64_t));
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_out, 4 * (size_t)n * sizeof(uint64_t));
    if (e == cudaSuccess) e = cudaMalloc((void **)&d_flags, (size_t)n * sizeof(uint32_t));
    if (e == cudaSuccess) e = cudaMemcpy(d_in, lo, (size_t)n * sizeof(uint64_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) e = cudaMemcpy(d_in + n, hi, (size_t)n * sizeof(uint64_t), cudaMemcpyHostToDevice);
    if (e == cudaSuccess) {
        ps4::check_roots<<<(n + 255) / 256, 256>>>(d_in, d_in + n, n, d_out, d_flags);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaMemcpy(roots, d_out, 4 * (size_t)n * sizeof(uint64_t), cudaMemcpyDeviceToHost);
    if (e == cudaSuccess) e = cudaMemcpy(flags, d_flags, (size_t)n * sizeof(uint32_t), cudaMemcpyDeviceToHost);
    cudaFree(d_in);
    cudaFree(d_out);
    cudaFree(d_flags);
    if (prev != device) cudaSetDevice(prev);
    return e == cudaSuccess ? PS4_OK : PS4_ERR_CUDA;
}

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
constexpr uint32_t HITS = PS4_NOALLOC_MAX_HITS, EXTS = PS4_NOALLOC_MAX_EXTS, SIXES = PS4_NOALLOC_MAX_SIXES;
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

namespace {
// The device address of ps4_noalloc_scratch on each device, with the primary context it was
// looked up in.  Host code only ever holds the array's host-side stand-in; a kernel must be
// given the address looked up here.  Guarded by a mutex: two host threads may make their
// first calls on a device at the same time.
struct NoallocBase {
    void *cu_ctx = nullptr;
    void *base = nullptr;
};
std::mutex noalloc_mu;
NoallocBase noalloc_base[64];

// The calling thread's current CUDA context (the device's primary context once the runtime
// has set the device up), through the driver entry point the runtime hands out: nullptr if
// it cannot be had, in which case the cached address is trusted as it is.
void *current_cu_ctx() {
    typedef int (*get_ctx_t)(void **);
    static const get_ctx_t fn = []() -> get_ctx_t {
        void *f = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuCtxGetCurrent", &f, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess)
            f = nullptr;
        return (get_ctx_t)f;
    }();
    void *ctx = nullptr;
    if (fn && fn(&ctx) != 0) ctx = nullptr;
    return ctx;
}

// The array's address on `device` (current): looked up once per device and primary context.
cudaError_t noalloc_base_of(int device, void **out) {
    std::lock_guard<std::mutex> lock(noalloc_mu);
    NoallocBase &nb = noalloc_base[device];
    void *ctx = current_cu_ctx();
    if (!nb.base || (ctx && ctx != nb.cu_ctx)) {
        void *p = nullptr;
        const cudaError_t e = cudaGetSymbolAddress(&p, ps4_noalloc_scratch);
        if (e != cudaSuccess) return e;
        nb.base = p;
        nb.cu_ctx = ctx ? ctx : current_cu_ctx();
    }
    *out = nb.base;
    return cudaSuccess;
}

// After a failed call the next one looks the address up again.
void noalloc_forget(int device) {
    std::lock_guard<std::mutex> lock(noalloc_mu);
    noalloc_base[device] = NoallocBase();
}
}  // namespace

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
    if (v.device < 0 || v.device >= 64) return ctx_fail(ctx, PS4_ERR_ARG, "device ordinal out of range");

    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess) return ctx_fail(ctx, PS4_ERR_CUDA, "cudaGetDevice failed");
    if (prev != v.device && cudaSetDevice(v.device) != cudaSuccess)
        return ctx_fail(ctx, PS4_ERR_CUDA, "cudaSetDevice failed");
    int rc = PS4_OK;
    bool cuda_failed = false;
    char msg[320];
    do {
        // once per device (and primary context), with that device current: the device address
        // of the static array -- the host-side name ps4_noalloc_scratch must not reach a kernel
        void *basep = nullptr;
        cudaError_t e = noalloc_base_of(v.device, &basep);
        if (e != cudaSuccess) {
            snprintf(msg, sizeof msg, "cudaGetSymbolAddress(ps4_noalloc_scratch) failed: %s", cudaGetErrorString(e));
            rc = ctx_fail(ctx, PS4_ERR_CUDA, msg);
            cuda_failed = true;
            break;
        }
        unsigned char *base = (unsigned char *)basep;
        Status *d_status = (Status *)(base + na::OFF_STATUS);
        unsigned long long *d_counters = (unsigned long long *)(base + na::OFF_COUNTERS);
        Item *d_item = (Item *)(base + na::OFF_ITEM);
        cudaStream_t s = (cudaStream_t)v.stream;
        Item it;
        it.lo = lo; it.hi = hi; it.tile_base = 0; it.id = 0; it.pad = 0;
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
        e = cudaMemcpyAsync(d_item, &it, sizeof it, cudaMemcpyHostToDevice, s);
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
            cuda_failed = true;
            break;
        }
        const unsigned code = (unsigned)(st.err & 0xFF);
        const unsigned long long errS = st.err >> 8;
        if (code == E_CAP_REPS || code == E_CAP_DIVS || code == E_CAP_EXT) {
            snprintf(msg, sizeof msg, "FATAL: %s; this interval is NOT certified complete", fatal_text(code));
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
            // a tile's fixed shared-memory list (selected S, representations, 4-set staging or
            // extension list) overflowed: the tile's size is fixed here, so a shorter range meets
            // the same tile again
            static const char *list_name[5] = {"?", "selected-S list", "representation list", "4-set staging",
                                               "extension list"};
            snprintf(msg, sizeof msg,
                     "FATAL: internal capacity exceeded near S=%llu (%s: %llu > %llu); this interval is NOT "
                     "certified complete", errS, list_name[st.diag[0] < 5 ? st.diag[0] : 0], st.diag[1], st.diag[2]);
            rc = ctx_fail(ctx, PS4_ERR_CAP_INTERNAL, msg);
            break;
        }
        res->n_hits = st.n_hits; res->n_exts = st.n_exts; res->n_sixes = st.n_sixes;
        if (st.n_hits > na::HITS || st.n_exts > na::EXTS || st.n_sixes > na::SIXES) {
            snprintf(msg, sizeof msg,
                     "ps4_search_range_noalloc: the fixed result buffers overflowed (%s%s%s): hits %u of %u, "
                     "extensions %u of %u, 6-sets %u of %u; nothing was copied, search a shorter range",
                     st.n_hits > na::HITS ? "hits " : "", st.n_exts > na::EXTS ? "extensions " : "",
                     st.n_sixes > na::SIXES ? "6-sets" : "", st.n_hits, na::HITS, st.n_exts, na::EXTS, st.n_sixes,
                     na::SIXES);
            rc = ctx_fail(ctx, PS4_ERR_OUTPUT_FULL, msg);
            break;
        }
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
            cuda_failed = true;
            break;
        }
        stats_add(stats, k);
    } while (0);
    if (cuda_failed) noalloc_forget(v.device);
    if (prev != v.device) cudaSetDevice(prev);
    return rc;
}
