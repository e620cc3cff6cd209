// SIMT (CUDA-core) distance engine for sm_100a: the plain FP32/FP64 path.
//
// Every pair value is accumulated in exactly the order of the AOCL-DA packed
// micro-kernels, so squared-euclidean / manhattan / dot values are bit-identical
// to the reference CPU results:
//   * squared euclidean (metrics_kernels.hpp:419-496): dims are consumed in
//     groups of four, dims 4t,4t+1 chained into accumulator g1 and dims
//     4t+2,4t+3 into g2; at the end of every KC slice (and after the last full
//     group) g1 += g2, g2 = 0; the d%4 remainder dims are chained into g1.
//     KC is the reference's slice length (partitioning_infrastructure.hpp:45-59).
//   * manhattan / cosine-dot / minkowski: one sequential chain over the dims.
// The order is fixed per pair and independent of tiling, so results do not
// depend on batch composition or tile position.
//
// Tiling (B200-native): 256 threads, a BM x BN tile of pairs, each thread a
// TM x TN register micro-tile; operands staged through double-buffered shared
// memory in BK-dim slabs with 16-byte vector loads.
#include "b200_common.cuh"
#include <cuda/atomic>
#include "b200_kernels.hpp"
#include "simt_engine.cuh"
#include <map>
#include <mutex>

namespace b200 {

// 16-byte vector of T
template <typename T> struct Vec16Of;
template <> struct Vec16Of<float> { using V = float4; };
template <> struct Vec16Of<double> { using V = double2; };
// Raises (never lowers) a kernel's dynamic shared-memory limit on the current
// device.  The limit belongs to the function and device for the whole
// process, so callers on several threads that need different sizes must not
// lower it under one another; a larger limit does not change a launch that
// asks for less.
cudaError_t ensure_smem_limit(const void *func, size_t smem) {
    static std::mutex mu;
    static std::map<std::pair<const void *, int>, size_t> done;
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    std::lock_guard<std::mutex> g(mu);
    size_t &have = done[{func, dev}];
    if (have >= smem) return cudaSuccess;
    e = cudaFuncSetAttribute(func, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e == cudaSuccess) have = smem;
    return e;
}
} // namespace b200

namespace b200 {

// Post-operation of one accumulated pair value (reference post-ops:
// cosine_distance.cpp:66-88, minkowski_distance.cpp:67-77,
// euclidean_gemm_distance.cpp:108-135, nearest_neighbors.cpp:662-665).
template <typename T>
B200_DEV T post_value(int post, T g, T xn, T yn, T invp) {
    switch (post) {
    case POST_SQRT: return sqrt_rn(g);
    case POST_COSINE: return sub_rn(T(1), div_rn(g, mul_rn(xn, yn)));
    case POST_GEMM_SQ: return fma_rn(T(-2), g, add_rn(xn, yn));
    case POST_GEMM_SQRT: return sqrt_rn(fma_rn(T(-2), g, add_rn(xn, yn)));
    case POST_GEMM_SQ_CLAMP: {
        T v = fma_rn(T(-2), g, add_rn(xn, yn));
        return v < T(0) ? T(0) : v;
    }
    case POST_POW: return pow_(g, invp);
    case POST_NEG: return -g;
    default: return g;
    }
}

// ------------------------------------------------------------ pairwise ----
template <typename T, int ACC>
__global__ void __launch_bounds__(256)
pairwise_kernel(const T *X, int m, const T *Y, int n, int ld, int d, const T *xn, const T *yn,
                int post, int kc, T p, T invp, int x_is_y, int out_rowmajor, T *D, T thr,
                int *hits, int nch) {
    using C = SimtCfg<T>;
    constexpr int TM = C::TM, TN = C::TN, BK = C::BK, BM = 16 * TM, BN = 16 * TN;
    __shared__ __align__(16) Stage<T, BM, BN, BK> st[2];
    const int tid = threadIdx.x;
    const int i0 = blockIdx.y * BM, j0 = blockIdx.x * BN;
    Acc<T, TM, TN> acc;
    compute_tile<T, ACC, TM, TN, BM, BN, BK>(st, X, ld, m, i0, Y, ld, n, j0, d, kc, p, acc, tid);
    const int tm = tid / 16, tn = tid % 16;
    // row-major D with n a multiple of 4: a thread's four consecutive columns
    // go out as 16-byte stores (D from cudaMalloc, rows of n elements)
    const bool vec_out = out_rowmajor && (n & 3) == 0 &&
                         (reinterpret_cast<uintptr_t>(D) & 15) == 0;
    int hit[TM];
#pragma unroll
    for (int i = 0; i < TM; ++i) {
        hit[i] = 0;
        const int gi = i0 + tm * 4 + i;
        if (gi >= m) continue;
        const T xv = xn ? xn[gi] : T(0);
#pragma unroll
        for (int g = 0; g < TN / 4; ++g) {
            const int gj0 = j0 + g * 64 + tn * 4;
            T v[4];
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                const int gj = gj0 + u;
                const T yv = (yn && gj < n) ? yn[gj] : T(0);
                v[u] = post_value<T>(post, acc.g1[i][g * 4 + u], xv, yv, invp);
                if (x_is_y && gi == gj && (post == POST_COSINE || post == POST_GEMM_SQ ||
                                           post == POST_GEMM_SQRT))
                    v[u] = T(0);
                if (gj < n) hit[i] += v[u] <= thr ? 1 : 0;
            }
            if (vec_out && gj0 + 3 < n) {
                using V = typename Vec16Of<T>::V;
                constexpr int W = 16 / (int)sizeof(T);
#pragma unroll
                for (int u = 0; u < 4; u += W)
                    *reinterpret_cast<V *>(D + (size_t)gi * n + gj0 + u) =
                        *reinterpret_cast<const V *>(&v[u]);
            } else {
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    const int gj = gj0 + u;
                    if (gj >= n) continue;
                    if (out_rowmajor)
                        D[(size_t)gi * n + gj] = v[u];
                    else
                        D[(size_t)gj * m + gi] = v[u];
                }
            }
        }
    }
    if (!hits) return;
    // the tile's hits per row: the 16 lanes of a row group (one half-warp)
    // sum theirs, lane tn = 0 adds them to the row's chunk (a tile lies in
    // one chunk: RADIUS_CHUNK is a multiple of BN)
    static_assert(RADIUS_CHUNK % BN == 0, "tiles within one radius chunk");
#pragma unroll
    for (int i = 0; i < TM; ++i) {
        int c = hit[i];
#pragma unroll
        for (int off = 8; off > 0; off >>= 1) c += __shfl_xor_sync(0xffffffffu, c, off);
        const int gi = i0 + tm * 4 + i;
        if (tn == 0 && gi < m && c > 0) atomicAdd(&hits[(size_t)gi * nch + j0 / RADIUS_CHUNK], c);
    }
}

template <typename T>
cudaError_t launch_pairwise(const T *X, int ldx, int m, const T *Y, int ldy, int n, int d,
                            const T *xn, const T *yn, const PairwiseArgs &a, T *D,
                            cudaStream_t s) {
    using C = SimtCfg<T>;
    constexpr int BM = 16 * C::TM, BN = 16 * C::TN;
    if (ldx != ldy) return cudaErrorInvalidValue;
    dim3 grid((n + BN - 1) / BN, (m + BM - 1) / BM);
    const T p = T(a.p);
    const T invp = T(1.0 / (double)p);
    if (a.hits && !a.out_rowmajor) return cudaErrorInvalidValue;
    const T thr = T(a.thr);
    const int nch = radius_chunks(n);
    switch (a.acc) {
    case ACC_SQEUC:
        pairwise_kernel<T, ACC_SQEUC><<<grid, 256, 0, s>>>(X, m, Y, n, ldx, d, xn, yn, a.post,
                                                           a.kc, p, invp, a.x_is_y,
                                                           a.out_rowmajor, D, thr, a.hits, nch);
        break;
    case ACC_DOT:
        pairwise_kernel<T, ACC_DOT><<<grid, 256, 0, s>>>(X, m, Y, n, ldx, d, xn, yn, a.post, a.kc,
                                                         p, invp, a.x_is_y, a.out_rowmajor, D,
                                                         thr, a.hits, nch);
        break;
    case ACC_MANHATTAN:
        pairwise_kernel<T, ACC_MANHATTAN><<<grid, 256, 0, s>>>(X, m, Y, n, ldx, d, xn, yn,
                                                               a.post, a.kc, p, invp, a.x_is_y,
                                                               a.out_rowmajor, D, thr, a.hits,
                                                               nch);
        break;
    default:
        pairwise_kernel<T, ACC_MINKOWSKI><<<grid, 256, 0, s>>>(X, m, Y, n, ldx, d, xn, yn,
                                                               a.post, a.kc, p, invp, a.x_is_y,
                                                               a.out_rowmajor, D, thr, a.hits,
                                                               nch);
        break;
    }
    return cudaGetLastError();
}

// ------------------------------------------------------------ kNN fused ---
// Per-query running top-k lists in shared memory, a survivor buffer per
// query, and a warp-cooperative rank merge.
template <typename T, int BM, int KCAP, int BUF> struct TopkSmem {
    T list_key[BM][KCAP];
    int list_idx[BM][KCAP];
    T buf_key[BM][BUF];
    int buf_idx[BM][BUF];
    T thresh[BM];
    int list_n[BM];
    int buf_n[BM];
    int any;
};

template <typename T, int KCAP, int BUF>
B200_DEV void merge_query(T *lk, int *li, int &ln, T *bk, int *bi, int &bn, T &thr, int k,
                          int lane) {
    const int nl = ln, nb = bn;
    const int total = nl + nb;
    constexpr int MAXE = (KCAP + BUF + 31) / 32;
    T ek[MAXE];
    int ei[MAXE], er[MAXE];
#pragma unroll
    for (int r = 0; r < MAXE; ++r) {
        const int e = lane + 32 * r;
        er[r] = 0x7fffffff;
        if (e < total) {
            T key;
            int idx;
            int rank;
            if (e < nl) {
                key = lk[e];
                idx = li[e];
                int c = 0;
                for (int t = 0; t < nb; ++t) c += key_less(bk[t], bi[t], key, idx) ? 1 : 0;
                rank = e + c;
            } else {
                const int eb = e - nl;
                key = bk[eb];
                idx = bi[eb];
                int lo = 0, hi = nl; // lower bound in the sorted list
                while (lo < hi) {
                    int mid = (lo + hi) >> 1;
                    if (key_less(lk[mid], li[mid], key, idx)) lo = mid + 1;
                    else hi = mid;
                }
                int c = 0;
                for (int t = 0; t < nb; ++t) c += key_less(bk[t], bi[t], key, idx) ? 1 : 0;
                rank = lo + c;
            }
            ek[r] = key;
            ei[r] = idx;
            er[r] = rank;
        }
    }
    __syncwarp();
#pragma unroll
    for (int r = 0; r < MAXE; ++r) {
        if (er[r] < k) {
            lk[er[r]] = ek[r];
            li[er[r]] = ei[r];
        }
    }
    __syncwarp();
    const int newn = total < k ? total : k;
    if (lane == 0) {
        ln = newn;
        bn = 0;
        thr = (newn == k) ? lk[k - 1] : Lim<T>::inf();
    }
    __syncwarp();
}

template <typename T, int ACC, int KCAP>
__global__ void __launch_bounds__(256)
knn_chunk_kernel(const T *Q, int nq, const T *X, int nx, int ld, int d, const T *qn,
                 const T *xn, int post, int kc, T p, T invp, int k, int chunk_rows,
                 int n_chunks, T *part_key, int *part_idx) {
    using C = SimtCfg<T>;
    constexpr int TM = C::TM, TN = C::TN, BK = C::BK, BM = 16 * TM, BN = 16 * TN;
    constexpr int BUF = BN;
    using TS = TopkSmem<T, BM, KCAP, BUF>;
    extern __shared__ __align__(16) unsigned char smem_raw[];
    auto *st = reinterpret_cast<Stage<T, BM, BN, BK> *>(smem_raw);
    TS &ts = *reinterpret_cast<TS *>(smem_raw + 2 * sizeof(Stage<T, BM, BN, BK>));

    const int tid = threadIdx.x, lane = tid & 31, warp = tid >> 5;
    const int q0 = blockIdx.x * BM;
    const int c = blockIdx.y;
    const int x_begin = c * chunk_rows;
    const int x_end = min(nx, x_begin + chunk_rows);
    const int tm = tid / 16, tn = tid % 16;

    for (int q = tid; q < BM; q += 256) {
        ts.list_n[q] = 0;
        ts.buf_n[q] = 0;
        ts.thresh[q] = Lim<T>::inf();
    }
    if (tid == 0) ts.any = 0;
    __syncthreads();

    T qv[TM];
#pragma unroll
    for (int i = 0; i < TM; ++i) {
        const int gq = q0 + tm * 4 + i;
        qv[i] = (qn && gq < nq) ? qn[gq] : T(0);
    }

    Acc<T, TM, TN> acc;
    for (int x0 = x_begin; x0 < x_end; x0 += BN) {
        compute_tile<T, ACC, TM, TN, BM, BN, BK>(st, Q, ld, nq, q0, X, ld, x_end, x0, d, kc, p,
                                                 acc, tid);
        // filter against the per-query thresholds
        bool any = false;
#pragma unroll
        for (int i = 0; i < TM; ++i) {
            const int ql = tm * 4 + i;
            if (q0 + ql >= nq) continue;
            const T thr = ts.thresh[ql];
            const bool open = ts.list_n[ql] < k; // list not full: accept every finite key
#pragma unroll
            for (int j = 0; j < TN; ++j) {
                const int gx = x0 + (j / 4) * 64 + tn * 4 + (j % 4);
                if (gx >= x_end) continue;
                const T xv = xn ? xn[gx] : T(0);
                const T key = post_value<T>(post, acc.g1[i][j], qv[i], xv, invp);
                // Within one chunk rows arrive in ascending index order, so a
                // strict '<' against the k-th key is the (key, index) order.
                if (key == key && (open || key < thr)) {
                    const int pos = atomicAdd(&ts.buf_n[ql], 1);
                    ts.buf_key[ql][pos] = key;
                    ts.buf_idx[ql][pos] = gx;
                    any = true;
                }
            }
        }
        if (any) ts.any = 1;
        __syncthreads();
        if (ts.any) {
            for (int ql = warp; ql < BM; ql += 8) {
                if (ts.buf_n[ql] > 0)
                    merge_query<T, KCAP, BUF>(ts.list_key[ql], ts.list_idx[ql], ts.list_n[ql],
                                              ts.buf_key[ql], ts.buf_idx[ql], ts.buf_n[ql],
                                              ts.thresh[ql], k, lane);
            }
            __syncthreads();
            if (tid == 0) ts.any = 0;
        }
    }
    __syncthreads();
    // write the chunk list (padded with (+inf, INT_MAX))
    for (int ql = warp; ql < BM; ql += 8) {
        const int gq = q0 + ql;
        if (gq >= nq) continue;
        const size_t base = ((size_t)gq * n_chunks + c) * k;
        const int ln = ts.list_n[ql];
        for (int r = lane; r < k; r += 32) {
            if (r < ln) {
                part_key[base + r] = ts.list_key[ql][r];
                part_idx[base + r] = ts.list_idx[ql][r];
            } else {
                part_key[base + r] = Lim<T>::inf();
                part_idx[base + r] = 0x7fffffff;
            }
        }
    }
}

template <typename T, int ACC, int KCAP>
static cudaError_t launch_knn_chunks_t(const T *Q, int nq, const T *X, int nx, int ld, int d,
                                       const T *qn, const T *xn, const KnnArgs &a, T *pk,
                                       int *pi, cudaStream_t s) {
    using C = SimtCfg<T>;
    constexpr int BM = 16 * C::TM, BN = 16 * C::TN, BK = C::BK;
    const size_t smem = 2 * sizeof(Stage<T, BM, BN, BK>) + sizeof(TopkSmem<T, BM, KCAP, BN>);
    auto kern = knn_chunk_kernel<T, ACC, KCAP>;
    cudaError_t e = ensure_smem_limit(reinterpret_cast<const void *>(kern), smem);
    if (e != cudaSuccess) return e;
    dim3 grid((nq + BM - 1) / BM, a.n_chunks);
    const T p = T(a.p);
    const T invp = T(1.0 / (double)p);
    kern<<<grid, 256, smem, s>>>(Q, nq, X, nx, ld, d, qn, xn, a.post, a.kc, p, invp, a.k,
                                 a.chunk_rows, a.n_chunks, pk, pi);
    return cudaGetLastError();
}

template <typename T, int KCAP>
static cudaError_t dispatch_acc(const T *Q, int nq, const T *X, int nx, int ld, int d,
                                const T *qn, const T *xn, const KnnArgs &a, T *pk, int *pi,
                                cudaStream_t s) {
    switch (a.acc) {
    case ACC_SQEUC: return launch_knn_chunks_t<T, ACC_SQEUC, KCAP>(Q, nq, X, nx, ld, d, qn, xn, a, pk, pi, s);
    case ACC_DOT: return launch_knn_chunks_t<T, ACC_DOT, KCAP>(Q, nq, X, nx, ld, d, qn, xn, a, pk, pi, s);
    case ACC_MANHATTAN: return launch_knn_chunks_t<T, ACC_MANHATTAN, KCAP>(Q, nq, X, nx, ld, d, qn, xn, a, pk, pi, s);
    default: return launch_knn_chunks_t<T, ACC_MINKOWSKI, KCAP>(Q, nq, X, nx, ld, d, qn, xn, a, pk, pi, s);
    }
}

int knn_tile_rows_train(bool fp64) { return fp64 ? 16 * SimtCfg<double>::TN : 16 * SimtCfg<float>::TN; }
int knn_max_k(bool fp64) { return fp64 ? 128 : 256; }

template <typename T>
cudaError_t launch_knn_chunks(const T *Q, int ldq, int nq, const T *X, int ldx, int nx, int d,
                              const T *qn, const T *xn, const KnnArgs &a, T *part_key,
                              int *part_idx, int *err_flag, cudaStream_t s) {
    (void)err_flag;
    if (ldq != ldx) return cudaErrorInvalidValue;
    if (a.k <= 32) return dispatch_acc<T, 32>(Q, nq, X, nx, ldx, d, qn, xn, a, part_key, part_idx, s);
    if (a.k <= 128) return dispatch_acc<T, 128>(Q, nq, X, nx, ldx, d, qn, xn, a, part_key, part_idx, s);
    if constexpr (sizeof(T) == 4) {
        if (a.k <= 256) return dispatch_acc<T, 256>(Q, nq, X, nx, ldx, d, qn, xn, a, part_key, part_idx, s);
    }
    return cudaErrorInvalidValue;
}

// ------------------------------------------------------------ kNN merge ---
// One warp per query: every element's final rank is its position in its own
// chunk list plus the number of smaller elements in every other list
// (binary search); elements with rank < k are written.
template <typename T>
__global__ void knn_merge_kernel(const T *pk, const int *pi, int nq, int nc, int k, int tf,
                                 int out_colmajor, T *ok, int *oi) {
    const int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (warp >= nq) return;
    const size_t base = (size_t)warp * nc * k;
    const int total = nc * k;
    for (int e = lane; e < total; e += 32) {
        const int c = e / k, r = e % k;
        const T key = pk[base + e];
        const int idx = pi[base + e];
        int rank = r;
        for (int c2 = 0; c2 < nc && rank < k; ++c2) {
            if (c2 == c) continue;
            const T *lk = pk + base + (size_t)c2 * k;
            const int *li = pi + base + (size_t)c2 * k;
            int lo = 0, hi = k;
            while (lo < hi) {
                int mid = (lo + hi) >> 1;
                if (key_less(lk[mid], li[mid], key, idx)) lo = mid + 1;
                else hi = mid;
            }
            rank += lo;
        }
        if (rank < k && idx != 0x7fffffff) {
            T v = key;
            if (tf == 1) v = sqrt_rn(v);
            else if (tf == 2) v = -v;
            const size_t o = out_colmajor ? ((size_t)rank * nq + warp) : ((size_t)warp * k + rank);
            ok[o] = v;
            oi[o] = idx;
        }
    }
}

template <typename T>
cudaError_t launch_knn_merge(const T *part_key, const int *part_idx, int nq, int n_chunks, int k,
                             int out_transform, T *out_key, int *out_idx, cudaStream_t s) {
    // out_transform: low bits = 0 none / 1 sqrt / 2 negate; bit 4 = column-major output
    const int tf = out_transform & 3;
    const int colmaj = (out_transform >> 4) & 1;
    const int threads = 256;
    const int blocks = (nq * 32 + threads - 1) / threads;
    knn_merge_kernel<T><<<blocks, threads, 0, s>>>(part_key, part_idx, nq, n_chunks, k, tf,
                                                   colmaj, out_key, out_idx);
    return cudaGetLastError();
}

// ------------------------------------------------------------ row norms ---
// Squared norms as one sequential fma chain per row.  A block of 256 threads
// takes 32 rows: 64-feature slabs of them are staged in shared memory with
// coalesced loads (rows padded to 65 words), then 32 threads carry the chains.
template <typename T>
__global__ void __launch_bounds__(256) row_sqnorms_kernel(const T *X, int ld, int rows, int d,
                                                          T *out) {
    __shared__ T slab[32][65];
    const int r0 = blockIdx.x * 32;
    const int nr = min(32, rows - r0);
    T s = T(0);
    for (int f0 = 0; f0 < d; f0 += 64) {
        const int nf = min(64, d - f0);
        __syncthreads();
        for (int e = threadIdx.x; e < 32 * 64; e += 256) {
            const int i = e >> 6, f = e & 63;
            if (i < nr && f < nf) slab[i][f] = X[(size_t)(r0 + i) * ld + f0 + f];
        }
        __syncthreads();
        if ((int)threadIdx.x < nr)
            for (int f = 0; f < nf; ++f)
                s = fma_rn(slab[threadIdx.x][f], slab[threadIdx.x][f], s);
    }
    if ((int)threadIdx.x < nr) out[r0 + threadIdx.x] = s;
}
template <typename T>
__global__ void row_norms_eps1_kernel(const T *X, int ld, int rows, int d, T eps, T *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= rows) return;
    const T *x = X + (size_t)i * ld;
    double s = 0.0;
    for (int j = 0; j < d; ++j) s = fma((double)x[j], (double)x[j], s);
    T nv = T(sqrt(s));
    out[i] = (nv <= eps) ? T(1) : nv;
}
template <typename T>
cudaError_t launch_row_sqnorms(const T *X, int ld, int rows, int d, T *out, cudaStream_t s) {
    if (rows <= 0) return cudaSuccess;
    row_sqnorms_kernel<T><<<(rows + 31) / 32, 256, 0, s>>>(X, ld, rows, d, out);
    return cudaGetLastError();
}
template <typename T>
cudaError_t launch_row_norms_eps1(const T *X, int ld, int rows, int d, T *out, cudaStream_t s) {
    const T eps = sizeof(T) == 4 ? T(FLT_EPSILON) : T(DBL_EPSILON);
    row_norms_eps1_kernel<T><<<(rows + 255) / 256, 256, 0, s>>>(X, ld, rows, d, eps, out);
    return cudaGetLastError();
}

// --------------------------------------------------------------- ingest ---
template <typename T>
__global__ void colmajor_to_rowmajor_kernel(const T *src, int rows, int cols, T *dst, int ldo) {
    __shared__ T tile[32][33];
    const int c0 = blockIdx.x * 32, r0 = blockIdx.y * 32;
    for (int y = threadIdx.y; y < 32; y += 8) {
        const int c = c0 + y, r = r0 + threadIdx.x;
        tile[y][threadIdx.x] = (c < cols && r < rows) ? src[(size_t)c * rows + r] : T(0);
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += 8) {
        const int r = r0 + y, c = c0 + threadIdx.x;
        if (r < rows && c < ldo) dst[(size_t)r * ldo + c] = (c < cols) ? tile[threadIdx.x][y] : T(0);
    }
}
template <typename T>
__global__ void rowmajor_to_colmajor_kernel(const T *src, int rows, int cols, int ldi, T *dst,
                                            long ldc) {
    __shared__ T tile[32][33];
    const int r0 = blockIdx.x * 32, c0 = blockIdx.y * 32;
    for (int y = threadIdx.y; y < 32; y += 8) {
        const int r = r0 + y, c = c0 + threadIdx.x;
        tile[y][threadIdx.x] = (r < rows && c < cols) ? src[(size_t)r * ldi + c] : T(0);
    }
    __syncthreads();
    for (int y = threadIdx.y; y < 32; y += 8) {
        const int c = c0 + y, r = r0 + threadIdx.x;
        if (r < rows && c < cols) dst[(size_t)c * ldc + r] = tile[threadIdx.x][y];
    }
}
template <typename T>
cudaError_t launch_colmajor_to_rowmajor(const T *src, int rows, int cols, T *dst, int ldo,
                                        cudaStream_t s) {
    dim3 grid((ldo + 31) / 32, (rows + 31) / 32), block(32, 8);
    colmajor_to_rowmajor_kernel<T><<<grid, block, 0, s>>>(src, rows, cols, dst, ldo);
    return cudaGetLastError();
}
template <typename T>
cudaError_t launch_rowmajor_to_colmajor(const T *src, int rows, int cols, int ldi, T *dst,
                                        long ldc, cudaStream_t s) {
    dim3 grid((rows + 31) / 32, (cols + 31) / 32), block(32, 8);
    rowmajor_to_colmajor_kernel<T><<<grid, block, 0, s>>>(src, rows, cols, ldi, dst, ldc);
    return cudaGetLastError();
}

// ------------------------------------------------------- instantiations ---
#define B200_INST(T)                                                                          \
    template cudaError_t launch_pairwise<T>(const T *, int, int, const T *, int, int, int,     \
                                            const T *, const T *, const PairwiseArgs &, T *,   \
                                            cudaStream_t);                                     \
    template cudaError_t launch_knn_chunks<T>(const T *, int, int, const T *, int, int, int,   \
                                              const T *, const T *, const KnnArgs &, T *,      \
                                              int *, int *, cudaStream_t);                     \
    template cudaError_t launch_knn_merge<T>(const T *, const int *, int, int, int, int, T *,  \
                                             int *, cudaStream_t);                             \
    template cudaError_t launch_row_sqnorms<T>(const T *, int, int, int, T *, cudaStream_t);   \
    template cudaError_t launch_row_norms_eps1<T>(const T *, int, int, int, T *, cudaStream_t);\
    template cudaError_t launch_colmajor_to_rowmajor<T>(const T *, int, int, T *, int,         \
                                                        cudaStream_t);                         \
    template cudaError_t launch_rowmajor_to_colmajor<T>(const T *, int, int, int, T *, long,   \
                                                        cudaStream_t);
B200_INST(float)
B200_INST(double)

// ------------------------------------------------------ radius search ---
// nearest_neighbors.cpp:2070-2247 keeps, per query, the training rows with
// D <= (squared) radius.  The distance kernel counts the hits of every (row,
// 16,384-column chunk) piece; the pieces' output offsets come from a chained
// scan; one block per piece compacts it in index order (exclusive scans
// over tiles of columns), so each row's hits come out in index order.
template <typename T>
__global__ void radius_emit_kernel(const T *D, int n, size_t ld, T thr, int chunk,
                                   const long long *start, int *idx, T *val) {
    const T *row = D + (size_t)blockIdx.y * ld;
    __shared__ int ws[33];
    long long base = start[(size_t)blockIdx.y * gridDim.x + blockIdx.x];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int j1 = min(n, (int)(blockIdx.x + 1) * chunk);
    for (int j0 = (int)blockIdx.x * chunk; j0 < j1; j0 += blockDim.x) {
        const int j = j0 + threadIdx.x;
        const T v = j < j1 ? row[j] : T(0);
        const int f = (j < j1 && v <= thr) ? 1 : 0;
        const unsigned b = __ballot_sync(0xffffffffu, f);
        const int inw = __popc(b & ((1u << lane) - 1u));
        if (lane == 0) ws[w] = __popc(b);
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            for (int q = 0; q < nw; ++q) {
                const int c = ws[q];
                ws[q] = t;
                t += c;
            }
            ws[32] = t;
        }
        __syncthreads();
        if (f) {
            const long long pos = base + ws[w] + inw;
            idx[pos] = j;
            val[pos] = v;
        }
        base += ws[32];
        __syncthreads();
    }
}
// radius_emit_kernel with W consecutive elements per thread (one 16-byte
// load; rows and chunk bounds multiples of W): the thread's hits in index
// order, a warp scan of the per-thread counts, then the warps in order.
template <typename T>
__global__ void radius_emit_vec_kernel(const T *D, int n, size_t ld, T thr, int chunk,
                                       const long long *start, int *idx, T *val) {
    constexpr int W = 16 / (int)sizeof(T);
    using V = typename Vec16Of<T>::V;
    const T *row = D + (size_t)blockIdx.y * ld;
    __shared__ int ws[33];
    long long base = start[(size_t)blockIdx.y * gridDim.x + blockIdx.x];
    const int lane = threadIdx.x & 31, w = threadIdx.x >> 5, nw = blockDim.x >> 5;
    const int j1 = min(n, (int)(blockIdx.x + 1) * chunk);
    for (int j0 = (int)blockIdx.x * chunk; j0 < j1; j0 += (int)blockDim.x * W) {
        const int j = j0 + (int)threadIdx.x * W;
        T v[W];
        if (j < j1) {
            const V t = *reinterpret_cast<const V *>(row + j);
            const T *tp = reinterpret_cast<const T *>(&t);
#pragma unroll
            for (int u = 0; u < W; ++u) v[u] = tp[u];
        }
        int c = 0;
        unsigned fm = 0;
#pragma unroll
        for (int u = 0; u < W; ++u)
            if (j < j1 && v[u] <= thr) {
                fm |= 1u << u;
                ++c;
            }
        int x = c;
#pragma unroll
        for (int o = 1; o < 32; o <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, o);
            if (lane >= o) x += y;
        }
        if (lane == 31) ws[w] = x;
        __syncthreads();
        if (threadIdx.x == 0) {
            int t = 0;
            for (int q = 0; q < nw; ++q) {
                const int cq = ws[q];
                ws[q] = t;
                t += cq;
            }
            ws[32] = t;
        }
        __syncthreads();
        long long pos = base + ws[w] + (x - c);
#pragma unroll
        for (int u = 0; u < W; ++u)
            if (fm & (1u << u)) {
                idx[pos] = j + u;
                val[pos] = v[u];
                ++pos;
            }
        base += ws[32];
        __syncthreads();
    }
}
int radius_chunks(int n) { return (n + RADIUS_CHUNK - 1) / RADIUS_CHUNK; }
// Output offsets of the (row, chunk) pieces from their hit counts (made by
// the distance kernel): a chained scan in (row, chunk) order over groups of
// 32 pieces, one warp per group.  Each warp takes the next logical group from
// a ticket (so every group before it has a warp running or done), scans its
// 32 counts with shuffles and publishes the group's count; lane 0 then looks
// back over the groups before it -- a group's word holds 2 flag bits (1: its
// count, 2: its inclusive prefix) and a 62-bit value -- adding counts until
// it meets a prefix, and publishes the group's inclusive prefix.  The
// look-back waits on global memory for a predecessor that has not published
// yet; every wait is bounded (`limit` polls), after which the warp sets
// err[0] = 1 and leaves its own prefix unpublished (its successors then time
// out as well: the call fails with a status, the device stays usable).
// start[piece] = the exclusive prefix, total[0] = all hits.  skip_first
// (testing): group 0 publishes nothing.
__global__ void __launch_bounds__(32)
radius_scan_groups_kernel(const int *hits, int pieces, int groups, unsigned *ticket,
                          unsigned long long *state, long long *start, long long *total,
                          int *err, unsigned limit, int skip_first) {
    const int lane = threadIdx.x;
    int id = 0;
    if (lane == 0) id = (int)atomicAdd(ticket, 1u);
    id = __shfl_sync(0xffffffffu, id, 0);
    if (id >= groups) return;
    const int p = id * 32 + lane;
    const int c = p < pieces ? hits[p] : 0;
    int x = c; // inclusive scan of the group's counts
#pragma unroll
    for (int o = 1; o < 32; o <<= 1) {
        const int y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    const long long gsum = (long long)__shfl_sync(0xffffffffu, x, 31);
    constexpr unsigned long long AGG = 1ull << 62, PRE = 2ull << 62, VAL = (1ull << 62) - 1;
    long long excl = 0;
    int failed = 0;
    if (lane == 0) {
        cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> me(state[id]);
        if (id == 0) {
            if (!skip_first) me.store(PRE | (unsigned long long)gsum, cuda::memory_order_release);
        } else {
            me.store(AGG | (unsigned long long)gsum, cuda::memory_order_release);
            unsigned polls = 0;
            for (int j = id - 1; j >= 0;) {
                cuda::atomic_ref<unsigned long long, cuda::thread_scope_device> pj(state[j]);
                const unsigned long long v = pj.load(cuda::memory_order_acquire);
                const unsigned long long flag = v & ~VAL;
                if (flag == 0) {
                    if (++polls > limit) {
                        failed = 1;
                        break;
                    }
                    __nanosleep(64);
                    continue;
                }
                excl += (long long)(v & VAL);
                if (flag == PRE) break;
                --j;
            }
            if (failed) atomicExch(err, 1);
            else me.store(PRE | (unsigned long long)(excl + gsum), cuda::memory_order_release);
        }
    }
    failed = __shfl_sync(0xffffffffu, failed, 0);
    excl = __shfl_sync(0xffffffffu, excl, 0);
    if (failed) return;
    if (p < pieces) start[p] = excl + x - c;
    if (p == pieces - 1) *total = excl + x;
}

template <typename T>
cudaError_t launch_radius_count_scan(const T *D, int rows, int n, size_t ld, T thr, void *work,
                                     long long *start, long long *total, int *err, int test_wait,
                                     cudaStream_t s, const int *hits) {
    (void)D, (void)ld, (void)thr;
    if (rows <= 0 || n <= 0) return cudaSuccess;
    if (!hits) return cudaErrorInvalidValue;
    const int nch = radius_chunks(n);
    const int pieces = rows * nch;
    const int groups = (pieces + 31) / 32;
    unsigned *ticket = static_cast<unsigned *>(work);
    unsigned long long *state = reinterpret_cast<unsigned long long *>(static_cast<char *>(work) + 256);
    cudaError_t e = cudaMemsetAsync(work, 0, 256 + (size_t)groups * 8, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(err, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
    // about a second of polling; the test mode's wait runs out in microseconds
    const unsigned limit = test_wait ? 2000u : (1u << 24);
    radius_scan_groups_kernel<<<groups, 32, 0, s>>>(hits, pieces, groups, ticket, state, start,
                                                    total, err, limit, test_wait);
    return cudaGetLastError();
}
size_t radius_scan_work_bytes(int rows, int n) { return 256 + (size_t)rows * radius_chunks(n) * 8; }
template cudaError_t launch_radius_count_scan<float>(const float *, int, int, size_t, float,
                                                     void *, long long *, long long *, int *, int,
                                                     cudaStream_t, const int *);
template cudaError_t launch_radius_count_scan<double>(const double *, int, int, size_t, double,
                                                      void *, long long *, long long *, int *,
                                                      int, cudaStream_t, const int *);

template <typename T>
cudaError_t launch_radius_emit(const T *D, int rows, int n, size_t ld, T thr,
                               const long long *start, int *idx, T *val, cudaStream_t s) {
    if (rows <= 0 || n <= 0) return cudaSuccess;
    const dim3 grid(radius_chunks(n), rows);
    constexpr int W = 16 / (int)sizeof(T);
    if (n % W == 0 && ld % W == 0 && (reinterpret_cast<uintptr_t>(D) & 15) == 0)
        radius_emit_vec_kernel<T><<<grid, 256, 0, s>>>(D, n, ld, thr, RADIUS_CHUNK, start, idx,
                                                       val);
    else
        radius_emit_kernel<T><<<grid, 256, 0, s>>>(D, n, ld, thr, RADIUS_CHUNK, start, idx, val);
    return cudaGetLastError();
}
template cudaError_t launch_radius_emit<float>(const float *, int, int, size_t, float,
                                               const long long *, int *, float *, cudaStream_t);
template cudaError_t launch_radius_emit<double>(const double *, int, int, size_t, double,
                                                const long long *, int *, double *, cudaStream_t);

} // namespace b200
