// Brute-force kNN (euclidean / squared euclidean, fp32 data) with a bf16
// tensor-core candidate pass and an exact fp32 re-score.
//
// Ranking value of train row j for query q: v'_j = |x_j|^2 - 2 x_j.q (the
// squared distance minus the query's own |q|^2).  The tcgen05 pass computes
// v'_tc from three bf16 products (x = xh + xl, -2q = qh + ql:
// xh.qh + xh.ql + xl.qh) accumulated in fp32 in TMEM, plus the fp32 |x_j|^2.
// A rigorous bound |v'_tc - v'_plain| <= eps_q (v'_plain: the plain path's
// fp32 squared distance, in the reference's accumulation order, minus |q|^2)
// gives the certificate: every row of the plain top-k has
// v'_tc <= v'_tc(k) + 2 eps_q, where v'_tc(k) is the k-th smallest v'_tc.
//
// Every query keeps a threshold theta_q >= v'_tc(k) + 2 eps_q, shared by all
// CTAs through global memory (atomicMin of order-preserving bits).  The
// epilogue appends every (v'_tc, j) with v'_tc < theta_q to the query's list;
// at every window boundary of the list, a warp merges a complete window into
// the query's smallest listed values and lowers theta_q to their k-th
// + 2 eps_q -- k distinct listed rows, so never below the global k-th:
// theta_q stays a valid bound while it tightens.  theta_q starts from an
// exact pre-pass over slices of the first training rows (the k-th smallest
// plain distance within any slice bounds the global one).  The finalize kernel re-scores the listed rows
// with v'_tc < theta_q exactly (the plain kernel's formula and order) and
// keeps the k best by (distance, index): the plain path's neighbours.
#include "b200_common.cuh"
#include "b200_kernels.hpp"
#include "tc_common.cuh"
#include <cuda_bf16.h>
#include <cmath>

namespace b200 {

using namespace tc;

namespace {

constexpr int TK_BM = 128;         // train rows per tile (UMMA M, TMEM lanes)
constexpr int TK_BN = 256;         // queries per tile (UMMA N, TMEM columns), at most
constexpr int TK_KB = 64;          // bf16 elements per 128-byte K block
constexpr int TK_THREADS = 320;    // TMA warp, MMA warp, 8 epilogue warps
constexpr int TK_PRE_SLICE = 2048; // unit of the threshold pre-pass's row count
constexpr int TK_BEST = 256;       // smallest listed values kept per query (>= k)
constexpr int TK_WIN = 128;        // list entries merged into them per refresh
constexpr int TK_CHUNK_TILES = 64; // train tiles per work item
constexpr int TK_FIN_MAX = 8192;   // candidates re-scored per query (more: fallback)
// values below threshold held per lane before reserving list slots (the
// 256-query tile keeps 4: its shared memory is needed for the stages)
__host__ __device__ constexpr int tk_stash(int bn) { return bn >= 256 ? 4 : 8; }
static_assert(TK_CHUNK_TILES <= 64 && TK_BN <= 256, "stash entry bit fields");

struct KnnTcArgs {
    int nx, nq, k, nkb, stages, n_qtiles, n_xtiles, n_items, cap;
    int kk_last; // K steps of 16 in the last K block (the rest are zero columns)
    const float *xnorm;   // nx: fp32 |x_j|^2
    const float *margin;  // n_qtiles * BN: 2 eps_q (nudged up)
    unsigned *theta;      // n_qtiles * BN: threshold, order-preserving bits
    int *cnt;             // n_qtiles * BN: entries appended
    int2 *list;           // nq * cap: (value bits, train row)
    float *best;          // n_qtiles * BN * TK_BEST: smallest listed values so far
    int *lock;            // n_qtiles * BN: refresh of `best` in progress
    int *err;
};

struct __align__(16) TkShared {
    uint64_t full[8], empty[8], tfull[2], tempty[2], bfull, bempty;
    uint32_t tmem_base;
    int abort_flag;
};

__device__ __forceinline__ unsigned ord_bits(float f) {
    const unsigned b = __float_as_uint(f);
    return (b & 0x80000000u) ? ~b : (b | 0x80000000u);
}
__device__ __forceinline__ float ord_float(unsigned o) {
    return __uint_as_float((o & 0x80000000u) ? (o & 0x7fffffffu) : ~o);
}
__device__ __forceinline__ float nudge_up(float t) {
    return t + fabsf(t) * 9.5367431640625e-7f + 1e-30f;
}
__device__ __forceinline__ void tk_raise(int *abort_flag, int *err, int code) {
    *((volatile int *)abort_flag) = 1;
    atomicExch(err, code);
}

// v[u] for a runtime u without dynamic register indexing (selects).
__device__ __forceinline__ float pick32(const float (&v)[32], int u) {
    float r = v[0];
#pragma unroll
    for (int i = 1; i < 32; ++i) r = (u == i) ? v[i] : r;
    return r;
}

// Ascending bitonic sort of 512 floats held 16 per lane (element i = 16 lane + e).
__device__ __forceinline__ void warp_sort512(float (&a)[16]) {
    const int lane = threadIdx.x & 31;
#pragma unroll
    for (int size = 2; size <= 512; size <<= 1) {
#pragma unroll
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            if (stride >= 16) {
                const int lx = stride >> 4;
#pragma unroll
                for (int e = 0; e < 16; ++e) {
                    const float o = __shfl_xor_sync(0xffffffffu, a[e], lx);
                    const int i = lane * 16 + e;
                    const bool asc = (i & size) == 0, lower = (i & stride) == 0;
                    a[e] = (asc == lower) ? fminf(a[e], o) : fmaxf(a[e], o);
                }
            } else {
#pragma unroll
                for (int e = 0; e < 16; ++e) {
                    if ((e & stride) == 0) {
                        const int j = e ^ stride;
                        const int i = lane * 16 + e;
                        const bool asc = (i & size) == 0;
                        const float lo = fminf(a[e], a[j]), hi = fmaxf(a[e], a[j]);
                        a[e] = asc ? lo : hi;
                        a[j] = asc ? hi : lo;
                    }
                }
            }
        }
    }
}

// The ranking value of a train row: squared euclidean |x|^2 - 2 x.q (xs =
// |x|^2), or cosine -2 x.q / |x| with q normalised (xs = 1 / |x|), which is
// 2 (cosine distance - 1).
template <bool COS> __device__ __forceinline__ float tk_val(float v, float xs) {
    return COS ? __fmul_rn(v, xs) : __fadd_rn(v, xs);
}

// BN: queries per tile (UMMA N, TMEM columns per accumulator): 64, 128 or
// 256, the smallest that holds a small batch (less tensor work per train tile).
template <int BN, bool COS>
__global__ void __launch_bounds__(TK_THREADS, 1)
knn_tc_kernel(const __grid_constant__ CUtensorMap tmAh, const __grid_constant__ CUtensorMap tmAl,
              const __grid_constant__ CUtensorMap tmBh, const __grid_constant__ CUtensorMap tmBl,
              KnnTcArgs a) {
    extern __shared__ __align__(1024) unsigned char tk_raw[];
    unsigned char *base = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(tk_raw) + 1023) & ~uintptr_t(1023));
    const int S = a.stages, nkb = a.nkb;
    constexpr uint32_t kB = BN * 128u; // one K block of the query tile
    constexpr uint32_t kA = TK_BM * 128u; // one K block of a train tile (16 KB)
    unsigned char *Bh = base;
    unsigned char *Bl = Bh + (size_t)nkb * kB;
    unsigned char *As = Bl + (size_t)nkb * kB; // S stages of (Ah, Al) for one K block
    float *th_w = reinterpret_cast<float *>(As + (size_t)S * 2 * kA); // 8 warps x BN
    int *col_w = reinterpret_cast<int *>(th_w + 8 * BN);                // 8 warps x BN
    constexpr int STASH = tk_stash(BN);
    int2 *stash_w = reinterpret_cast<int2 *>(col_w + 8 * BN); // 8 warps x 32 lanes x STASH
    TkShared *sh = reinterpret_cast<TkShared *>(stash_w + 8 * 32 * STASH);

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&sh->full[s], 1);
            mbar_init(&sh->empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&sh->tfull[b], 1);
            mbar_init(&sh->tempty[b], 4 * 32);
        }
        mbar_init(&sh->bfull, 1);
        mbar_init(&sh->bempty, 1);
        sh->abort_flag = 0;
        fence_barrier_init();
    }
    for (int i = threadIdx.x; i < 8 * BN; i += blockDim.x) col_w[i] = 0;
    if (warp == 1) {
        tmem_alloc(&sh->tmem_base, 2u * BN);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = sh->tmem_base;

    if (warp == 0) {
        // ---------------------------------------------------- TMA producer --
        if (lane == 0) {
            prefetch_tmap(&tmAh);
            prefetch_tmap(&tmBh);
            int us = 0, ii = 0;
            bool ok = true;
            for (int item = blockIdx.x; ok && item < a.n_items; item += gridDim.x, ++ii) {
                const int xc = item / a.n_qtiles, qt = item % a.n_qtiles;
                if (ii > 0 && !mbar_wait(&sh->bempty, (uint32_t)((ii - 1) & 1))) {
                    tk_raise(&sh->abort_flag, a.err, 11);
                    break;
                }
                mbar_arrive_expect_tx(&sh->bfull, (uint32_t)(2 * nkb) * kB);
                for (int kb = 0; kb < nkb; ++kb) {
                    tma_load_2d(&tmBh, &sh->bfull, Bh + (size_t)kb * kB, kb * TK_KB, qt * BN);
                    tma_load_2d(&tmBl, &sh->bfull, Bl + (size_t)kb * kB, kb * TK_KB, qt * BN);
                }
                const int x0 = xc * TK_CHUNK_TILES, x1 = min(a.n_xtiles, x0 + TK_CHUNK_TILES);
                for (int xt = x0; ok && xt < x1; ++xt) {
                    for (int kb = 0; kb < nkb; ++kb, ++us) {
                        const int s = us % S;
                        if (!mbar_wait(&sh->empty[s], (uint32_t)(((us / S) & 1) ^ 1))) {
                            tk_raise(&sh->abort_flag, a.err, 12);
                            ok = false;
                            break;
                        }
                        if (*((volatile int *)&sh->abort_flag)) {
                            ok = false;
                            break;
                        }
                        unsigned char *st = As + (size_t)s * 2 * kA;
                        mbar_arrive_expect_tx(&sh->full[s], 2 * kA);
                        tma_load_2d(&tmAh, &sh->full[s], st, kb * TK_KB, xt * TK_BM);
                        tma_load_2d(&tmAl, &sh->full[s], st + kA, kb * TK_KB, xt * TK_BM);
                    }
                }
            }
            // every issued stage must have landed before exit
            for (int u = (us > S ? us - S : 0); u < us; ++u)
                mbar_wait(&sh->full[u % S], (uint32_t)((u / S) & 1));
        }
    } else if (warp == 1) {
        // ---------------------------------------------------- MMA issuer ----
        if (lane == 0) {
            const uint32_t idesc = idesc_bf16_f32(TK_BM, BN);
            int us = 0, tc = 0, ii = 0;
            bool ok = true;
            for (int item = blockIdx.x; ok && item < a.n_items; item += gridDim.x, ++ii) {
                const int xc = item / a.n_qtiles;
                if (!mbar_wait(&sh->bfull, (uint32_t)(ii & 1))) {
                    tk_raise(&sh->abort_flag, a.err, 13);
                    break;
                }
                const int x0 = xc * TK_CHUNK_TILES, x1 = min(a.n_xtiles, x0 + TK_CHUNK_TILES);
                for (int xt = x0; ok && xt < x1; ++xt, ++tc) {
                    const int b = tc & 1;
                    if (!mbar_wait(&sh->tempty[b], (uint32_t)(((tc >> 1) & 1) ^ 1))) {
                        tk_raise(&sh->abort_flag, a.err, 14);
                        ok = false;
                        break;
                    }
                    const uint32_t tacc = tbase + (uint32_t)(b * BN);
                    uint32_t acc = 0;
                    for (int kb = 0; kb < nkb; ++kb, ++us) {
                        const int s = us % S;
                        if (!mbar_wait(&sh->full[s], (uint32_t)((us / S) & 1))) {
                            tk_raise(&sh->abort_flag, a.err, 15);
                            ok = false;
                            break;
                        }
                        if (*((volatile int *)&sh->abort_flag)) {
                            ok = false;
                            break;
                        }
                        tc_fence_after();
                        const uint32_t ah = smem_u32(As + (size_t)s * 2 * kA);
                        const uint32_t al = ah + kA;
                        const uint32_t bh = smem_u32(Bh + (size_t)kb * kB);
                        const uint32_t bl = smem_u32(Bl + (size_t)kb * kB);
                        const int nkk = kb == nkb - 1 ? a.kk_last : TK_KB / 16;
#pragma unroll
                        for (int kk = 0; kk < TK_KB / 16; ++kk) {
                            if (kk >= nkk) break;
                            mma_f16_ss(tacc, desc_k_sw128(ah + kk * 32), desc_k_sw128(bh + kk * 32),
                                       idesc, acc);
                            acc = 1;
                            mma_f16_ss(tacc, desc_k_sw128(ah + kk * 32), desc_k_sw128(bl + kk * 32),
                                       idesc, 1);
                            mma_f16_ss(tacc, desc_k_sw128(al + kk * 32), desc_k_sw128(bh + kk * 32),
                                       idesc, 1);
                        }
                        mma_commit(&sh->empty[s]);
                    }
                    if (!ok) break;
                    mma_commit(&sh->tfull[b]);
                }
                mma_commit(&sh->bempty);
            }
            // the accumulators of the last tiles must be complete before the
            // TMEM is released
            for (int u = (tc > 2 ? tc - 2 : 0); u < tc; ++u)
                mbar_wait(&sh->tfull[u & 1], (uint32_t)((u >> 1) & 1));
        }
    } else {
        // ---------------------------------------------------- epilogue ------
        const int e = warp - 2;
        const int g = e >> 2;     // accumulator buffer / tile parity
        const int q = warp & 3;   // TMEM lane quarter
        float *thw = th_w + e * BN;
        int *colcnt = col_w + e * BN;                          // zero between flushes
        // stash entry: (column | tile offset in the work item << 8 | rank << 14,
        // value bits); the rank is assigned when list slots are reserved
        int2 *stash = stash_w + (size_t)(e * 32 + lane) * STASH;
        int ns = 0;
        const float inf = __int_as_float(0x7f800000);
        // Reserve list slots for the stashed values (one global atomic per
        // query column, all columns at once), write them, and merge the list
        // windows they complete into the queries' best values (threshold
        // refresh).  Warp-cooperative, once a lane's stash is full or the
        // work item (query tile qt_, train tiles from x0_) ends: the global
        // round trips are paid once per many tiles.
        auto flush = [&](int qt_, int x0_) {
            if (!__any_sync(0xffffffffu, ns > 0)) return;
            for (int i = 0; i < ns; ++i) {
                const int col = stash[i].x & 0xFF;
                const int rank = atomicAdd(&colcnt[col], 1);
                stash[i].x = (stash[i].x & 0x3FFF) | (rank << 14);
            }
            __syncwarp();
            int nn[BN / 32], bb[BN / 32];
#pragma unroll
            for (int j = 0; j < BN / 32; ++j) {
                const int col = j * 32 + lane;
                nn[j] = colcnt[col];
                bb[j] = nn[j] > 0 ? atomicAdd(&a.cnt[qt_ * BN + col], nn[j]) : 0;
            }
#pragma unroll
            for (int j = 0; j < BN / 32; ++j) colcnt[j * 32 + lane] = bb[j];
            __syncwarp();
            for (int i = 0; i < ns; ++i) {
                const int x = stash[i].x;
                const int col = x & 0xFF, rank = x >> 14;
                const int row_ = (x0_ + ((x >> 8) & 0x3F)) * TK_BM + q * 32 + lane;
                const int pos = colcnt[col] + rank;
                if (pos < a.cap)
                    a.list[(size_t)(qt_ * BN + col) * a.cap + pos] = make_int2(stash[i].y, row_);
            }
            ns = 0;
            __syncwarp();
#pragma unroll
            for (int j = 0; j < BN / 32; ++j) colcnt[j * 32 + lane] = 0;
#pragma unroll
            for (int j = 0; j < BN / 32; ++j) {
                // Crossing a window boundary: merge the window before the one
                // just completed (its entries have been written by now; one
                // still in flight reads as +inf) into the query's smallest
                // listed values, and lower theta to their k-th + 2 eps.  They
                // are distinct listed rows, so their k-th is never below the
                // global k-th.  One warp at a time per query (a refresh that
                // finds another in progress is skipped: a later one catches up).
                const int w_mine = ((bb[j] + nn[j]) / TK_WIN) * TK_WIN;
                const bool cross = nn[j] > 0 && w_mine > bb[j] && w_mine >= 2 * TK_WIN &&
                                   w_mine <= a.cap;
                unsigned todo = __ballot_sync(0xffffffffu, cross);
                while (todo) {
                    const int src = __ffs(todo) - 1;
                    todo &= todo - 1;
                    const int col = j * 32 + src;
                    const int gq = qt_ * BN + col;
                    const int w_end = __shfl_sync(0xffffffffu, w_mine, src);
                    __threadfence();
                    // a short, bounded wait for the lock (its holder never
                    // waits, so it is released within a refresh time)
                    int got = 0;
                    if (lane == 0)
                        for (int t = 0; t < 256 && !got; ++t)
                            got = atomicCAS(&a.lock[gq], 0, 1) == 0;
                    got = __shfl_sync(0xffffffffu, got, 0);
                    if (got) {
                        __threadfence();
                        float *bq = a.best + (size_t)gq * TK_BEST;
                        const int2 *lw = a.list + (size_t)gq * a.cap + (w_end - 2 * TK_WIN);
                        float s16[16];
#pragma unroll
                        for (int t = 0; t < 8; ++t) s16[t] = __ldcg(&bq[lane * 8 + t]);
#pragma unroll
                        for (int t = 0; t < 4; ++t)
                            s16[8 + t] = __int_as_float(__ldcg(&lw[lane * 4 + t].x));
#pragma unroll
                        for (int t = 12; t < 16; ++t) s16[t] = __int_as_float(0x7f800000);
                        warp_sort512(s16);
                        if (lane < TK_BEST / 16) {
#pragma unroll
                            for (int t = 0; t < 16; ++t) __stcg(&bq[lane * 16 + t], s16[t]);
                        }
                        float kth = 0.f;
#pragma unroll
                        for (int t = 0; t < 16; ++t)
                            if (t == (a.k - 1) % 16) kth = s16[t];
                        kth = __shfl_sync(0xffffffffu, kth, (a.k - 1) / 16);
                        const float thn = nudge_up(kth + a.margin[gq]);
                        if (thn < thw[col] && lane == 0) {
                            atomicMin(&a.theta[gq], ord_bits(thn));
                            thw[col] = thn;
                        }
                        __threadfence();
                        __syncwarp();
                        if (lane == 0) atomicExch(&a.lock[gq], 0);
                    }
                    __syncwarp();
                }
            }
        };
        int tc = 0;
        bool ok = true;
        for (int item = blockIdx.x; ok && item < a.n_items; item += gridDim.x) {
            const int xc = item / a.n_qtiles, qt = item % a.n_qtiles;
            const int x0 = xc * TK_CHUNK_TILES, x1 = min(a.n_xtiles, x0 + TK_CHUNK_TILES);
            for (int xt = x0; xt < x1; ++xt, ++tc) {
                if ((tc & 1) != g) continue;
                const int b = g;
                const int row = xt * TK_BM + q * 32 + lane;
                // rows past the end never pass (+inf, or NaN for cosine)
                const float xn = row < a.nx ? a.xnorm[row] : (COS ? __int_as_float(0x7fc00000) : inf);
                unsigned tb[BN / 32];
#pragma unroll
                for (int u = 0; u < BN / 32; ++u) tb[u] = a.theta[qt * BN + u * 32 + lane];
                bool w = mbar_wait(&sh->tfull[b], (uint32_t)((tc >> 1) & 1));
                if (!w) tk_raise(&sh->abort_flag, a.err, 16);
                w = w && !*((volatile int *)&sh->abort_flag);
                if (!__all_sync(0xffffffffu, w)) {
                    ok = false;
                    break;
                }
#pragma unroll
                for (int u = 0; u < BN / 32; ++u) thw[u * 32 + lane] = ord_float(tb[u]);
                __syncwarp();
                tc_fence_after();
                const uint32_t trow = tbase + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * BN);
                // pass over the tile: values below their query's threshold
                // go to this lane's stash (column, tile, value)
                for (int c = 0; c < BN / 32; ++c) {
                    float v[32];
                    tmem_ld32(trow + (uint32_t)(c * 32), v);
                    float m = inf;
#pragma unroll
                    for (int u = 0; u < 32; ++u)
                        m = fminf(m, tk_val<COS>(v[u], xn) - thw[c * 32 + u]);
                    if (!__any_sync(0xffffffffu, m < 0.f)) continue;
                    unsigned bits = 0;
#pragma unroll
                    for (int u = 0; u < 32; ++u)
                        bits |= (tk_val<COS>(v[u], xn) < thw[c * 32 + u] ? 1u : 0u) << u;
                    while (__any_sync(0xffffffffu, bits != 0)) {
                        while (bits && ns < STASH) {
                            const int u = __ffs(bits) - 1;
                            bits &= bits - 1;
                            stash[ns++] = make_int2((c * 32 + u) | ((xt - x0) << 8),
                                                    __float_as_int(tk_val<COS>(pick32(v, u), xn)));
                        }
                        // some lane's stash is full: reserve and write now
                        if (__any_sync(0xffffffffu, bits != 0)) flush(qt, x0);
                    }
                }
                tc_fence_before();
                mbar_arrive(&sh->tempty[b]);
            }
            if (!ok) break;
            flush(qt, x0);
        }
    }
    tc_fence_before();
    __syncthreads();
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tbase, 2u * BN);
    }
}

// -2q split into bf16 hi / lo (rows nq..nq_pad-1 zero), the query norms |q|
// and the margins 2 eps_q; thresholds +inf (padded queries -inf), counts 0.
// Cosine (qnorm: the plain path's query norms): -2 q / |q| instead, and the
// margin 2 e1 for every query.
__global__ void knn_tc_prep_queries(const float *Q, int ld, int nq, int d, int nq_pad, int ldo,
                                    __nv_bfloat16 *Qh, __nv_bfloat16 *Ql, float e1, float e2,
                                    const float *xmax, float *margin, unsigned *theta, int *cnt,
                                    float *qsq, const float *qnorm) {
    const int qi = blockIdx.x * (blockDim.x >> 5) + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (qi >= nq_pad) return;
    const float qinv = (qnorm && qi < nq) ? __frcp_rn(qnorm[qi]) : 1.f;
    float s = 0.f;
    for (int f = lane; f < ldo; f += 32) {
        const float x = (qi < nq && f < d) ? Q[(size_t)qi * ld + f] : 0.f;
        s = __fmaf_rn(x, x, s);
        const float y = qnorm ? -2.f * __fmul_rn(x, qinv) : -2.f * x;
        const __nv_bfloat16 h = __float2bfloat16_rn(y);
        Qh[(size_t)qi * ldo + f] = h;
        Ql[(size_t)qi * ldo + f] = __float2bfloat16_rn(y - __bfloat162float(h));
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) s += __shfl_xor_sync(0xffffffffu, s, off);
    if (lane == 0) {
        const float qn = sqrtf(s) * 1.0001f;
        const float xm = qnorm ? 0.f : *xmax;
        const float eps = qnorm ? e1 : e1 * xm * qn + e2 * (xm * xm + qn * qn);
        margin[qi] = nudge_up(2.f * eps);
        theta[qi] = qi < nq ? ord_bits(__int_as_float(0x7f800000)) : ord_bits(-__int_as_float(0x7f800000));
        cnt[qi] = 0;
        qsq[qi] = s;
    }
}

__global__ void knn_tc_fill_best(float *best, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) best[i] = __int_as_float(0x7f800000);
}

__global__ void knn_tc_fill_list(int2 *list, size_t n) {
    const size_t i = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) list[i] = make_int2(0x7f800000, 0x7fffffff);
}

// The plain path's squared euclidean distance of one pair, in its exact
// accumulation order: per group of 4 dims, dims 4t, 4t+1 into g1 and
// 4t+2, 4t+3 into g2 (fma of the rounded difference), g1 += g2 at the end of
// every kc-block and of the last full group; remaining dims into g1.
__device__ __forceinline__ float sqeuc_ref(const float *x, const float *q, int d, int kc) {
    const int d4 = d & ~3;
    float g1 = 0.f, g2 = 0.f;
    for (int kg = 0; kg < d4; kg += 4) {
        const float t0 = __fsub_rn(q[kg], x[kg]), t1 = __fsub_rn(q[kg + 1], x[kg + 1]);
        const float t2 = __fsub_rn(q[kg + 2], x[kg + 2]), t3 = __fsub_rn(q[kg + 3], x[kg + 3]);
        g1 = __fmaf_rn(t0, t0, g1);
        g1 = __fmaf_rn(t1, t1, g1);
        g2 = __fmaf_rn(t2, t2, g2);
        g2 = __fmaf_rn(t3, t3, g2);
        if (((kg + 4) % kc) == 0 || (kg + 4) == d4) {
            g1 = __fadd_rn(g1, g2);
            g2 = 0.f;
        }
    }
    for (int f = d4; f < d; ++f) {
        const float t = __fsub_rn(q[f], x[f]);
        g1 = __fmaf_rn(t, t, g1);
    }
    return g1;
}

// One block per query: the listed rows with v'_tc < theta_q, their exact
// distances, sorted by (distance, index); the first k are written (sqrt for
// euclidean).  A query whose list overflowed, or with more than TK_FIN_MAX
// survivors, is flagged for the plain path (*n_fallback).
// The plain path's cosine distance 1 - g / (|x| |q|), g one sequential fma
// chain over the features, the norms the plain path's.
__device__ __forceinline__ float cos_ref(const float *x, const float *q, int d, float xn,
                                         float qn) {
    float g = 0.f;
    for (int f = 0; f < d; ++f) g = __fmaf_rn(x[f], q[f], g);
    return __fsub_rn(1.f, __fdiv_rn(g, __fmul_rn(xn, qn)));
}

// ---------------------------------------------------- threshold pre-pass --
// theta_q starts from the k-th smallest plain key p over the first rows of
// the training set: theta_q = p - |q|^2 + 4 eps_q >= v'_tc(k) + 2 eps_q (k
// rows with plain value <= p have v'_tc <= p - |q|^2 + eps_q; the fp32 |q|^2
// is within eps_q of |q|^2).  Cosine: p is a plain cosine distance and
// theta_q = 2 (p - 1) + 4 eps.  The rows are cut into slices of TK_PRE_SLICE;
// block (slice, query) computes the keys of its slice and keeps their k
// smallest, and one block per query takes the k-th smallest of those.

constexpr int TK_PRE_WARPS = 16;

// The k-th smallest (1-based) of n keys in shared memory, by a radix select
// on four 8-bit digits, most significant first.  Block-wide (every thread
// gets the result); n >= k >= 1.
__device__ unsigned block_kth(const unsigned *keys, int n, int k, int *hist, int *sel) {
    unsigned prefix = 0, mask = 0;
    int kk = k; // rank of the wanted key among those matching prefix
    for (int shift = 24; shift >= 0; shift -= 8) {
        for (int b = threadIdx.x; b < 256; b += blockDim.x) hist[b] = 0;
        __syncthreads();
        for (int i = threadIdx.x; i < n; i += blockDim.x) {
            const unsigned u = keys[i];
            if ((u & mask) == prefix) atomicAdd(&hist[(u >> shift) & 255u], 1);
        }
        __syncthreads();
        if (threadIdx.x < 32) {
            const int lane = threadIdx.x;
            int c[8], sum = 0;
#pragma unroll
            for (int j = 0; j < 8; ++j) {
                c[j] = hist[lane * 8 + j];
                sum += c[j];
            }
            int inc = sum;
#pragma unroll
            for (int off = 1; off < 32; off <<= 1) {
                const int t = __shfl_up_sync(0xffffffffu, inc, off);
                if (lane >= off) inc += t;
            }
            const int exc = inc - sum;
            if (exc < kk && kk <= inc) { // this lane's 8 digits hold the kk-th key
                int run = exc, b = 7;
                for (int j = 0; j < 8; ++j) {
                    if (run + c[j] >= kk) {
                        b = j;
                        break;
                    }
                    run += c[j];
                }
                sel[0] = lane * 8 + b;
                sel[1] = kk - run;
            }
        }
        __syncthreads();
        prefix |= (unsigned)sel[0] << shift;
        mask |= 0xFFu << shift;
        kk = sel[1];
    }
    return prefix;
}

// Keys (order-preserving bits) of rows r0 .. r0+n-1 against the query qv in
// shared memory: each warp stages 32 rows x 32 columns at a time with
// coalesced loads, and each lane accumulates one row in the plain path's
// order (sqeuc_ref; cos_ref for cosine), carried across the column slabs.
__device__ void block_keys(const float *X, int ld, int d, int kc, int r0, int n, const float *qv,
                           unsigned *keys, float *stage, const float *xnp, float qn) {
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    float *t = stage + warp * 32 * 33;
    const int d4 = d & ~3;
    for (int rb = warp * 32; rb < n; rb += TK_PRE_WARPS * 32) {
        const int nr = min(32, n - rb);
        float g1 = 0.f, g2 = 0.f;
        for (int c0 = 0; c0 < d; c0 += 32) {
            const int cw = min(32, d - c0);
            __syncwarp();
            for (int r = 0; r < nr; ++r)
                if (lane < cw) t[r * 33 + lane] = X[(size_t)(r0 + rb + r) * ld + c0 + lane];
            __syncwarp();
            if (lane < nr) {
                const float *x = t + lane * 33 - c0; // x[f] for f in [c0, c0 + cw)
                if (xnp) {
                    for (int f = c0; f < c0 + cw; ++f) g1 = __fmaf_rn(x[f], qv[f], g1);
                } else {
                    int kg = c0;
                    for (; kg < c0 + cw && kg < d4; kg += 4) {
                        const float t0 = __fsub_rn(qv[kg], x[kg]), t1 = __fsub_rn(qv[kg + 1], x[kg + 1]);
                        const float t2 = __fsub_rn(qv[kg + 2], x[kg + 2]);
                        const float t3 = __fsub_rn(qv[kg + 3], x[kg + 3]);
                        g1 = __fmaf_rn(t0, t0, g1);
                        g1 = __fmaf_rn(t1, t1, g1);
                        g2 = __fmaf_rn(t2, t2, g2);
                        g2 = __fmaf_rn(t3, t3, g2);
                        if (((kg + 4) % kc) == 0 || (kg + 4) == d4) {
                            g1 = __fadd_rn(g1, g2);
                            g2 = 0.f;
                        }
                    }
                    for (int f = max(kg, d4); f < c0 + cw; ++f) {
                        const float u = __fsub_rn(qv[f], x[f]);
                        g1 = __fmaf_rn(u, u, g1);
                    }
                }
            }
        }
        if (lane < nr) {
            const int i = rb + lane;
            const float v = xnp ? __fsub_rn(1.f, __fdiv_rn(g1, __fmul_rn(xnp[r0 + i], qn))) : g1;
            keys[i] = ord_bits(v);
        }
    }
}

__device__ __forceinline__ unsigned pre_theta_bits(unsigned kth, float qsq, float margin,
                                                   bool cosm) {
    const float pk = ord_float(kth);
    const float t = cosm ? nudge_up(2.f * (pk - 1.f) + 2.f * margin)
                         : nudge_up(pk - qsq + 2.f * margin);
    return t == t ? ord_bits(t) : ord_bits(__int_as_float(0x7f800000));
}

// Block (slice, query).  slices == 1: theta_q directly from the slice's k-th
// key.  Otherwise the slice's k smallest keys (padded with +inf when the
// slice holds fewer than k rows) go to out[(q * slices + slice) * k ...].
__global__ void __launch_bounds__(TK_PRE_WARPS * 32)
knn_tc_pre_slice(const float *X, const float *Q, int ld, int d, int kc, int nx, int nq, int k,
                 int slices, const float *qsq, const float *margin, unsigned *theta,
                 unsigned *out, const float *xnp, const float *qnp) {
    __shared__ int hist[256];
    __shared__ int sel[2];
    __shared__ int nlt;
    extern __shared__ __align__(16) unsigned pre_sm[];
    unsigned *keys = pre_sm;                                        // TK_PRE_SLICE
    float *stage = reinterpret_cast<float *>(keys + TK_PRE_SLICE);  // warps x 32 x 33
    float *qv = stage + TK_PRE_WARPS * 32 * 33;                     // d
    const int sl = blockIdx.x, qi = blockIdx.y;
    const int r0 = sl * TK_PRE_SLICE;
    const int n = max(0, min(TK_PRE_SLICE, nx - r0));
    for (int f = threadIdx.x; f < d; f += blockDim.x) qv[f] = Q[(size_t)qi * ld + f];
    if (threadIdx.x == 0) nlt = 0;
    __syncthreads();
    block_keys(X, ld, d, kc, r0, n, qv, keys, stage, xnp, xnp ? qnp[qi] : 1.f);
    __syncthreads();
    if (slices == 1) {
        if (n < k) return;
        const unsigned kth = block_kth(keys, n, k, hist, sel);
        if (threadIdx.x == 0) theta[qi] = pre_theta_bits(kth, qsq[qi], margin[qi], xnp != nullptr);
        return;
    }
    unsigned *o = out + ((size_t)qi * slices + sl) * k;
    if (n <= k) {
        for (int i = threadIdx.x; i < k; i += blockDim.x)
            o[i] = i < n ? keys[i] : ord_bits(__int_as_float(0x7f800000));
        return;
    }
    const unsigned kth = block_kth(keys, n, k, hist, sel);
    for (int i = threadIdx.x; i < n; i += blockDim.x)
        if (keys[i] < kth) o[atomicAdd(&nlt, 1)] = keys[i];
    __syncthreads();
    for (int i = nlt + threadIdx.x; i < k; i += blockDim.x) o[i] = kth; // ties at the k-th
}

// One block per query: theta_q from the k-th smallest of the slices' keys.
__global__ void __launch_bounds__(256)
knn_tc_pre_merge(const unsigned *in, int slices, int k, int nq, const float *qsq,
                 const float *margin, unsigned *theta, int cosm) {
    __shared__ int hist[256];
    __shared__ int sel[2];
    extern __shared__ __align__(16) unsigned merge_sm[]; // slices * k
    const int qi = blockIdx.x;
    const int n = slices * k;
    for (int i = threadIdx.x; i < n; i += blockDim.x) merge_sm[i] = in[(size_t)qi * n + i];
    __syncthreads();
    const unsigned kth = block_kth(merge_sm, n, k, hist, sel);
    if (threadIdx.x == 0) theta[qi] = pre_theta_bits(kth, qsq[qi], margin[qi], cosm != 0);
}

__global__ void __launch_bounds__(256)
knn_tc_finalize(const float *X, const float *Q, int ld, int d, int kc, int k, int cap,
                const unsigned *theta, const int *cnt, const int2 *list, int take_sqrt,
                float *out_key, int *out_idx, int *fallback, int *n_fallback,
                const float *xnp, const float *qnp) {
    __shared__ int scount;
    extern __shared__ __align__(16) float fin_smem[];
    float *skey = fin_smem;                                  // TK_FIN_MAX
    int *sidx = reinterpret_cast<int *>(skey + TK_FIN_MAX);  // TK_FIN_MAX
    float *qs = reinterpret_cast<float *>(sidx + TK_FIN_MAX); // d
    const int qi = blockIdx.x;
    const int n = cnt[qi];
    const float th = ord_float(theta[qi]);
    if (threadIdx.x == 0) scount = 0;
    for (int f = threadIdx.x; f < d; f += blockDim.x) qs[f] = Q[(size_t)qi * ld + f];
    __syncthreads();
    // fallback reasons counted at n_fallback[2..4]: list overflow, more
    // survivors than the re-score holds, fewer survivors than k
    if (n > cap) {
        if (threadIdx.x == 0) {
            fallback[qi] = 1;
            atomicAdd(n_fallback, 1);
            atomicAdd(n_fallback + 2, 1);
        }
        return;
    }
    for (int e = threadIdx.x; e < n; e += blockDim.x) {
        const int2 ev = list[(size_t)qi * cap + e];
        if (__int_as_float(ev.x) < th) {
            const int p = atomicAdd(&scount, 1);
            if (p < TK_FIN_MAX) sidx[p] = ev.y;
        }
    }
    __syncthreads();
    const int m = scount;
    if (m > TK_FIN_MAX || m < k) {
        if (threadIdx.x == 0) {
            fallback[qi] = 1;
            atomicAdd(n_fallback, 1);
            atomicAdd(n_fallback + (m > TK_FIN_MAX ? 3 : 4), 1);
        }
        return;
    }
    int np2 = 1;
    while (np2 < m) np2 <<= 1;
    for (int e = threadIdx.x; e < np2; e += blockDim.x) {
        if (e < m) {
            skey[e] = xnp ? cos_ref(X + (size_t)sidx[e] * ld, qs, d, xnp[sidx[e]], qnp[qi])
                          : sqeuc_ref(X + (size_t)sidx[e] * ld, qs, d, kc);
        } else {
            skey[e] = __int_as_float(0x7f800000);
            sidx[e] = 0x7fffffff;
        }
    }
    __syncthreads();
    // bitonic sort of (key, index) pairs, ascending
    for (int size = 2; size <= np2; size <<= 1) {
        for (int stride = size >> 1; stride > 0; stride >>= 1) {
            for (int i = threadIdx.x; i < np2; i += blockDim.x) {
                const int j = i ^ stride;
                if (j > i) {
                    const bool asc = (i & size) == 0;
                    const float ki = skey[i], kj = skey[j];
                    const int ii = sidx[i], ij = sidx[j];
                    const bool gt = key_less(kj, ij, ki, ii); // (i) > (j)
                    if (gt == asc) {
                        skey[i] = kj;
                        skey[j] = ki;
                        sidx[i] = ij;
                        sidx[j] = ii;
                    }
                }
            }
            __syncthreads();
        }
    }
    for (int r = threadIdx.x; r < k; r += blockDim.x) {
        const float kv = skey[r];
        out_key[(size_t)qi * k + r] = take_sqrt ? __fsqrt_rn(kv) : kv;
        out_idx[(size_t)qi * k + r] = sidx[r];
    }
}

__global__ void max_value_kernel(const float *v, int n, float *out) {
    float m = 0.f;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x)
        m = fmaxf(m, v[i]);
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) m = fmaxf(m, __shfl_xor_sync(0xffffffffu, m, off));
    if ((threadIdx.x & 31) == 0) atomicMax(reinterpret_cast<int *>(out), __float_as_int(m));
}
__global__ void sqrt_inplace_kernel(float *v) { *v = sqrtf(*v) * 1.0001f; }

size_t tk_smem_bytes(int nkb, int stages, int bn = TK_BN) {
    return 1024 + (size_t)nkb * 2 * bn * 128 + (size_t)stages * 2 * TK_BM * 128 +
           (size_t)8 * bn * 4 * 2 + (size_t)8 * 32 * tk_stash(bn) * 8 + sizeof(TkShared) + 64;
}

} // namespace

int knn_tc_supported(int nx, int d, int k) {
    if (k < 1 || k > 256 || nx < k || d < 1) return 0;
    const int nkb = (d + TK_KB - 1) / TK_KB;
    return tk_smem_bytes(nkb, 2) <= 225 * 1024 ? 1 : 0;
}

size_t knn_tc_list_cap() { return 16384; }

__global__ void recip_kernel(const float *v, int n, float *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < n) out[i] = __frcp_rn(v[i]);
}
cudaError_t launch_recip(const float *v, int n, float *out, cudaStream_t s) {
    if (n <= 0) return cudaSuccess;
    recip_kernel<<<(n + 255) / 256, 256, 0, s>>>(v, n, out);
    return cudaGetLastError();
}

cudaError_t launch_knn_tc_train_prep(const float *X, int ld, int nx, int d, void *Xh, void *Xl,
                                     int ldbf, float *xnorm2, float *xmax, cudaStream_t s) {
    cudaError_t e = launch_split_bf16(X, ld, nx, d, Xh, Xl, ldbf, s);
    if (e != cudaSuccess) return e;
    e = launch_row_sqnorms<float>(X, ld, nx, d, xnorm2, s);
    if (e != cudaSuccess) return e;
    e = cudaMemsetAsync(xmax, 0, sizeof(float), s);
    if (e != cudaSuccess) return e;
    max_value_kernel<<<148 * 4, 256, 0, s>>>(xnorm2, nx, xmax);
    sqrt_inplace_kernel<<<1, 1, 0, s>>>(xmax);
    return cudaGetLastError();
}

cudaError_t launch_knn_tc(const float *X, const void *Xh, const void *Xl, const float *xnorm2,
                          const float *xmax, int nx, int ld, int ldbf, int d, const float *Q,
                          int nq, int k, int kc, int take_sqrt, void *qbuf, void *list,
                          int *fallback, int *n_fallback, int *err, float *out_key,
                          int *out_idx, cudaStream_t s, const KnnTcCosine *cosine) {
    // ldbf: the bf16 rows' length (d rounded up to 8, at least 64); the MMA
    // runs nkb K blocks of 64, the last with only the 16-column steps that
    // hold data (the tensor maps zero-fill the columns past ldbf)
    const int nkb = (ldbf + TK_KB - 1) / TK_KB;
    const int kk_last = (d - (nkb - 1) * TK_KB + 15) / 16;
    // query tile width: small batches use a narrower MMA (the train rows are
    // read once either way; the tensor work and the epilogue scale with it)
    const int bn = nq <= 64 ? 64 : nq <= 128 ? 128 : TK_BN;
    const int n_qtiles = (nq + bn - 1) / bn, nq_pad = n_qtiles * bn;
    const int n_xtiles = (nx + TK_BM - 1) / TK_BM;
    const int n_xchunks = (n_xtiles + TK_CHUNK_TILES - 1) / TK_CHUNK_TILES;
    const int cap = (int)knn_tc_list_cap();
    // query-side buffers carved from qbuf with the region sizes of
    // knn_tc_query_bytes / knn_tc_counts (256-query padding, 64-column K
    // blocks), whatever the tile width
    const size_t nq_alloc = (size_t)((nq + TK_BN - 1) / TK_BN) * TK_BN;
    const size_t qrow = (size_t)nkb * TK_KB;
    unsigned char *p = static_cast<unsigned char *>(qbuf);
    __nv_bfloat16 *Qh = reinterpret_cast<__nv_bfloat16 *>(p);
    __nv_bfloat16 *Ql = Qh + nq_alloc * qrow;
    float *margin = reinterpret_cast<float *>(Ql + nq_alloc * qrow);
    unsigned *theta = reinterpret_cast<unsigned *>(margin + nq_alloc);
    int *cnt = reinterpret_cast<int *>(theta + nq_alloc);
    float *qsq = reinterpret_cast<float *>(cnt + nq_alloc);
    int *lock = reinterpret_cast<int *>(qsq + nq_alloc);
    float *best = reinterpret_cast<float *>(lock + nq_alloc);
    // |v'_tc - v'_plain| <= e1 |x||q| + e2 (|x|^2 + |q|^2)  (u = 2^-24):
    //   bf16 hi/lo split of x and of -2q, dropped lo.lo term: 3.1 2^-16 |x||2q|
    //   fp32 accumulation of K_total = 3 Kp products in the tensor core
    //   (allowing truncation): 2 K_total u |x||2q|
    //   fp32 |x|^2 (Kp-term fma chain) and the final add: (Kp + 2) u |x|^2, u |2xq|
    //   the plain path's direct-difference sum: (d + 4) u (|x| + |q|)^2
    const double u = std::ldexp(1.0, -24);
    const double kp = (double)nkb * TK_KB, ktot = 3.0 * kp;
    const double e1 = 1.1 * (3.1 * std::ldexp(1.0, -16) * 2.0 + 2.0 * ktot * u * 2.0 + 2.0 * u +
                             (d + 4.0) * u * 2.0);
    const double e2 = 1.1 * ((kp + 2.0) * u + (d + 4.0) * u * 2.0 + 2.0 * u);
    // cosine, r = -2 x.q / (|x| |q|) = 2 (distance - 1), |x|, |q| the plain
    // path's norms: bf16 hi/lo split and fp32 accumulation as above on unit-
    // scale products, the scalings by 1/|q| and 1/|x| (4 u), and twice the
    // plain distance's own error (d fma terms, the product, division and
    // subtraction: (d + 6) u)
    const double ec = 1.1 * (2.0 * (3.1 * std::ldexp(1.0, -16) + 2.0 * ktot * u + 4.0 * u) +
                             2.0 * (d + 6.0) * u);
    const bool cosm = cosine != nullptr;
    {
        const int wpb = 8;
        knn_tc_prep_queries<<<(nq_pad + wpb - 1) / wpb, wpb * 32, 0, s>>>(
            Q, ld, nq, d, nq_pad, ldbf, Qh, Ql, (float)(cosm ? ec : e1), (float)e2, xmax, margin,
            theta, cnt, qsq, cosm ? cosine->qnorm : nullptr);
        // exact pre-pass over the first rows (slices of TK_PRE_SLICE): at
        // least two blocks per SM in all, enough rows that the starting
        // threshold alone would keep about 4,096 candidates per query over
        // the whole set, at most 64 slices and about eight blocks per SM
        {
            const long long want_rows = (long long)nx * k / 4096;
            int slices = std::max(296 / std::max(1, nq),
                                  (int)std::min<long long>(64, (want_rows + TK_PRE_SLICE - 1) /
                                                                   TK_PRE_SLICE));
            slices = std::min(slices, std::max(1, 1184 / std::max(1, nq)));
            slices = std::max(1, std::min(std::min(slices, 64), (nx + TK_PRE_SLICE - 1) / TK_PRE_SLICE));
            const size_t psm = (size_t)TK_PRE_SLICE * 4 + (size_t)TK_PRE_WARPS * 32 * 33 * 4 +
                               (size_t)d * sizeof(float);
            cudaError_t e = ensure_smem_limit(reinterpret_cast<const void *>(knn_tc_pre_slice), psm);
            if (e != cudaSuccess) return e;
            // the slices' keys sit in the candidate list buffer (nq * cap
            // entries of 8 bytes; slices * k <= 16,384 keys of 4), which is
            // refilled below
            unsigned *keys = static_cast<unsigned *>(list);
            knn_tc_pre_slice<<<dim3(slices, nq), TK_PRE_WARPS * 32, psm, s>>>(
                X, Q, ld, d, kc, nx, nq, k, slices, qsq, margin, theta, keys,
                cosm ? cosine->xnorm : nullptr, cosm ? cosine->qnorm : nullptr);
            if (slices > 1) {
                const size_t msm = (size_t)slices * k * sizeof(unsigned);
                e = ensure_smem_limit(reinterpret_cast<const void *>(knn_tc_pre_merge), msm);
                if (e != cudaSuccess) return e;
                knn_tc_pre_merge<<<nq, 256, msm, s>>>(keys, slices, k, nq, qsq, margin, theta,
                                                      cosm ? 1 : 0);
            }
        }
        const size_t nl = (size_t)nq * cap;
        knn_tc_fill_list<<<(unsigned)((nl + 255) / 256), 256, 0, s>>>(static_cast<int2 *>(list), nl);
        const size_t nb = (size_t)nq_pad * TK_BEST;
        knn_tc_fill_best<<<(unsigned)((nb + 255) / 256), 256, 0, s>>>(best, nb);
        cudaError_t e = cudaMemsetAsync(lock, 0, (size_t)nq_pad * sizeof(int), s);
        if (e == cudaSuccess) e = cudaMemsetAsync(fallback, 0, (size_t)nq * sizeof(int), s);
        if (e == cudaSuccess) e = cudaMemsetAsync(n_fallback, 0, sizeof(int), s);
        if (e == cudaSuccess) e = cudaMemsetAsync(n_fallback + 2, 0, 3 * sizeof(int), s);
        if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), s);
        if (e != cudaSuccess) return e;
    }
    CUtensorMap mah, mal, mbh, mbl;
    if (!make_map_bf16_rows(&mah, Xh, nx, ldbf, TK_BM) ||
        !make_map_bf16_rows(&mal, Xl, nx, ldbf, TK_BM) ||
        !make_map_bf16_rows(&mbh, Qh, nq_pad, ldbf, bn) ||
        !make_map_bf16_rows(&mbl, Ql, nq_pad, ldbf, bn))
        return cudaErrorInvalidValue;
    int stages = 8;
    while (stages > 2 && tk_smem_bytes(nkb, stages, bn) > 225 * 1024) --stages;
    const size_t smem = tk_smem_bytes(nkb, stages, bn);
    auto kern = cosm ? (bn == 64 ? knn_tc_kernel<64, true> : bn == 128 ? knn_tc_kernel<128, true>
                                                                       : knn_tc_kernel<TK_BN, true>)
                     : (bn == 64 ? knn_tc_kernel<64, false> : bn == 128 ? knn_tc_kernel<128, false>
                                                                        : knn_tc_kernel<TK_BN, false>);
    cudaError_t e = ensure_smem_limit(reinterpret_cast<const void *>(kern), smem);
    if (e != cudaSuccess) return e;
    KnnTcArgs a;
    a.nx = nx;
    a.nq = nq;
    a.k = k;
    a.nkb = nkb;
    a.kk_last = kk_last;
    a.stages = stages;
    a.n_qtiles = n_qtiles;
    a.n_xtiles = n_xtiles;
    a.n_items = n_qtiles * n_xchunks;
    a.cap = cap;
    a.xnorm = cosm ? cosine->xinv : xnorm2;
    a.margin = margin;
    a.theta = theta;
    a.cnt = cnt;
    a.list = static_cast<int2 *>(list);
    a.best = best;
    a.lock = lock;
    a.err = err;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    // one block per work item (64 train tiles): blocks end often, so the
    // kernels of a higher-priority stream get SMs within one item's time
    (void)nsm;
    const int grid = a.n_items;
    kern<<<grid, TK_THREADS, smem, s>>>(mah, mal, mbh, mbl, a);
    e = cudaGetLastError();
    if (e != cudaSuccess) return e;
    const size_t fsm = (size_t)TK_FIN_MAX * 8 + (size_t)d * sizeof(float);
    e = ensure_smem_limit(reinterpret_cast<const void *>(knn_tc_finalize), fsm);
    if (e != cudaSuccess) return e;
    knn_tc_finalize<<<nq, 256, fsm, s>>>(
        X, Q, ld, d, kc, k, cap, theta, cnt, static_cast<const int2 *>(list),
        cosm ? 0 : take_sqrt, out_key, out_idx, fallback, n_fallback,
        cosm ? cosine->xnorm : nullptr, cosm ? cosine->qnorm : nullptr);
    return cudaGetLastError();
}

__global__ void rows_gather_kernel(const float *src, int ld, const int *idx, int m, float *dst) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)m * ld) return;
    const int i = (int)(e / ld), c = (int)(e % ld);
    dst[e] = src[(size_t)idx[i] * ld + c];
}
__global__ void results_scatter_kernel(const float *key, const int *ind, const int *idx, int m,
                                       int k, float *out_key, int *out_idx) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)m * k) return;
    const int i = (int)(e / k), r = (int)(e % k);
    out_key[(size_t)idx[i] * k + r] = key[e];
    out_idx[(size_t)idx[i] * k + r] = ind[e];
}

cudaError_t launch_rows_gather(const float *src, int ld, const int *idx, int m, float *dst,
                               cudaStream_t s) {
    const size_t n = (size_t)m * ld;
    if (n == 0) return cudaSuccess;
    rows_gather_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(src, ld, idx, m, dst);
    return cudaGetLastError();
}
cudaError_t launch_results_scatter(const float *key, const int *ind, const int *idx, int m, int k,
                                   float *out_key, int *out_idx, cudaStream_t s) {
    const size_t n = (size_t)m * k;
    if (n == 0) return cudaSuccess;
    results_scatter_kernel<<<(unsigned)((n + 255) / 256), 256, 0, s>>>(key, ind, idx, m, k,
                                                                        out_key, out_idx);
    return cudaGetLastError();
}

int *knn_tc_counts(void *qbuf, int nq, int d) {
    const int nkb = (d + TK_KB - 1) / TK_KB;
    const size_t nq_pad = (size_t)((nq + TK_BN - 1) / TK_BN) * TK_BN;
    unsigned char *p = static_cast<unsigned char *>(qbuf) + nq_pad * nkb * TK_KB * 2 * 2;
    return reinterpret_cast<int *>(p + nq_pad * 8);
}

size_t knn_tc_query_bytes(int nq, int d) {
    const int nkb = (d + TK_KB - 1) / TK_KB;
    const size_t nq_pad = (size_t)((nq + TK_BN - 1) / TK_BN) * TK_BN;
    return nq_pad * nkb * TK_KB * 2 * 2 + nq_pad * 20 + nq_pad * TK_BEST * 4 + 256;
}

} // namespace b200
