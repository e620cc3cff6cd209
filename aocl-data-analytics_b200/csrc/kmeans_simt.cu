// k-means (Lloyd) kernels for sm_100a: SIMT assignment with fused argmin,
// deterministic counting-sort centroid update in fp64, k-means++ helpers.
//
// Reference algorithm (AOCL-DA):
//   assignment  kmeans_lloyd.hpp:189-198 (W = -2 C A^T, then argmin_j W_ij + |c_j|^2
//               in kmeans_kernels.cpp:209-234; strict '<', so ties keep the lower j)
//   update      kmeans_lloyd.hpp:275-361 (sum of member rows), :364-405 (divide by
//               max(count,1): an empty cluster becomes the zero vector)
//   shift       kmeans.cpp:1334-1355, convergence kmeans.cpp:1359-1397
//   inertia     kmeans.cpp:1061-1124
//   k-means++   kmeans.cpp:1491-1664
// Here sums, shift and inertia are accumulated in fp64 in a fixed order, so
// every result is run-to-run deterministic and independent of scheduling.
#include "b200_common.cuh"
#include <algorithm>
#include "b200_kernels.hpp"
#include "simt_engine.cuh"
#include "kmeans_fx.cuh"

namespace b200 {

static constexpr int SORT_ROWS = 1024; // rows per counting-sort block

int kmeans_assign_block_rows() { return SORT_ROWS; }
int kmeans_max_clusters_fused() { return 1 << 20; }

// ------------------------------------------------------------- assign ----
// CTA = BM rows x all clusters (cluster tiles of BN), thread tile TM x TN.
template <typename T>
__global__ void __launch_bounds__(256)
kmeans_assign_kernel(const T *X, int n, int ld, int d, const T *C, int k, const T *cnorm,
                     int *labels, const int *labels_prev, int *flags) {
    using Cf = SimtCfg<T>;
    constexpr int TM = Cf::TM, TN = Cf::TN, BK = Cf::BK, BM = 16 * TM, BN = 16 * TN;
    __shared__ __align__(16) Stage<T, BM, BN, BK> st[2];
    __shared__ int changed;
    const int tid = threadIdx.x, tm = tid / 16, tn = tid % 16;
    const int i0 = blockIdx.x * BM;
    if (tid == 0) changed = 0;

    T best[TM];
    int bidx[TM];
#pragma unroll
    for (int i = 0; i < TM; ++i) {
        best[i] = Lim<T>::inf();
        bidx[i] = 0x7fffffff;
    }
    Acc<T, TM, TN> acc;
    for (int j0 = 0; j0 < k; j0 += BN) {
        compute_tile<T, ACC_DOT, TM, TN, BM, BN, BK>(st, X, ld, n, i0, C, ld, k, j0, d, 256,
                                                     T(0), acc, tid);
#pragma unroll
        for (int j = 0; j < TN; ++j) {
            const int gj = j0 + (j / 4) * 64 + tn * 4 + (j % 4);
            if (gj >= k) continue;
            const T cn = cnorm[gj];
#pragma unroll
            for (int i = 0; i < TM; ++i) {
                // |c|^2 - 2 x.c: -2 s is exact, so this is the reference's
                // fl(fl(-2 s) + |c|^2).
                const T v = fma_rn(T(-2), acc.g1[i][j], cn);
                if (key_less(v, gj, best[i], bidx[i])) {
                    best[i] = v;
                    bidx[i] = gj;
                }
            }
        }
    }
    // reduce across the 16 lanes that share these rows (lanes tn = 0..15)
#pragma unroll
    for (int i = 0; i < TM; ++i) {
#pragma unroll
        for (int off = 8; off >= 1; off >>= 1) {
            const T ov = __shfl_xor_sync(0xffffffffu, best[i], off);
            const int oi = __shfl_xor_sync(0xffffffffu, bidx[i], off);
            if (key_less(ov, oi, best[i], bidx[i])) {
                best[i] = ov;
                bidx[i] = oi;
            }
        }
    }
    if (tn == 0) {
        int ch = 0;
#pragma unroll
        for (int i = 0; i < TM; ++i) {
            const int gi = i0 + tm * 4 + i;
            if (gi < n) {
                // NaN distances never win: fall back to cluster 0 as the
                // reference's scalar kernel does (label initialised to 0).
                const int lbl = (bidx[i] == 0x7fffffff) ? 0 : bidx[i];
                // read before the write: labels may be labels_prev (in place)
                if (labels_prev && labels_prev[gi] != lbl) ch = 1;
                labels[gi] = lbl;
            }
        }
        if (ch) changed = 1;
    }
    __syncthreads();
    if (tid == 0 && changed && flags) atomicOr(&flags[0], 1);
}

template <typename T>
cudaError_t launch_kmeans_assign(const T *X, int ldx, int n, int d, const T *C, int ldc, int k,
                                 const T *cnorm, int *labels, const int *labels_prev,
                                 int *block_counts, int *flags, cudaStream_t s) {
    (void)block_counts;
    if (ldx != ldc) return cudaErrorInvalidValue;
    using Cf = SimtCfg<T>;
    constexpr int BM = 16 * Cf::TM;
    kmeans_assign_kernel<T><<<(n + BM - 1) / BM, 256, 0, s>>>(X, n, ldx, d, C, k, cnorm, labels,
                                                              labels_prev, flags);
    return cudaGetLastError();
}

// ------------------------------------------------------- counting sort ---
// (1) per SORT_ROWS block histogram of labels.
__global__ void label_hist_kernel(const int *labels, int n, int k, int *block_counts) {
    extern __shared__ int h[];
    for (int j = threadIdx.x; j < k; j += blockDim.x) h[j] = 0;
    __syncthreads();
    const int r0 = blockIdx.x * SORT_ROWS;
    const int r1 = min(n, r0 + SORT_ROWS);
    for (int i = r0 + threadIdx.x; i < r1; i += blockDim.x) atomicAdd(&h[labels[i]], 1);
    __syncthreads();
    for (int j = threadIdx.x; j < k; j += blockDim.x)
        block_counts[(size_t)blockIdx.x * k + j] = h[j];
}
// (2) one warp per cluster: exclusive scan of its block counts (in place).
__global__ void block_scan_kernel(int *block_counts, int nblocks, int k, int *counts) {
    const int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    if (j >= k) return;
    int carry = 0;
    for (int b0 = 0; b0 < nblocks; b0 += 32) {
        const int b = b0 + lane;
        const int v = (b < nblocks) ? block_counts[(size_t)b * k + j] : 0;
        int x = v;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const int y = __shfl_up_sync(0xffffffffu, x, off);
            if (lane >= off) x += y;
        }
        if (b < nblocks) block_counts[(size_t)b * k + j] = carry + x - v;
        carry += __shfl_sync(0xffffffffu, x, 31);
    }
    if (lane == 0) counts[j] = carry;
}
// (3) single CTA: cluster offsets and per-cluster segment-chunk starts.
__global__ void cluster_offsets_kernel(const int *counts, int k, int seg_rows, int *offsets,
                                       int *seg_chunk_start, int *flags) {
    __shared__ int s_off[1024], s_seg[1024];
    int carry_off = 0, carry_seg = 0;
    for (int j0 = 0; j0 < k; j0 += 1024) {
        const int j = j0 + threadIdx.x;
        const int c = (j < k) ? counts[j] : 0;
        const int sc = (c + seg_rows - 1) / seg_rows;
        s_off[threadIdx.x] = c;
        s_seg[threadIdx.x] = sc;
        __syncthreads();
        // Hillis-Steele inclusive scan over 1024 entries
        for (int off = 1; off < 1024; off <<= 1) {
            int a = 0, b = 0;
            if ((int)threadIdx.x >= off) {
                a = s_off[threadIdx.x - off];
                b = s_seg[threadIdx.x - off];
            }
            __syncthreads();
            s_off[threadIdx.x] += a;
            s_seg[threadIdx.x] += b;
            __syncthreads();
        }
        if (j < k) {
            offsets[j] = carry_off + s_off[threadIdx.x] - c;
            seg_chunk_start[j] = carry_seg + s_seg[threadIdx.x] - sc;
        }
        const int tot_off = s_off[1023], tot_seg = s_seg[1023];
        __syncthreads();
        carry_off += tot_off;
        carry_seg += tot_seg;
    }
    if (threadIdx.x == 0) {
        offsets[k] = carry_off;
        seg_chunk_start[k] = carry_seg;
    }
    // empty-cluster count
    __shared__ int s_empty;
    if (threadIdx.x == 0) s_empty = 0;
    __syncthreads();
    for (int j = threadIdx.x; j < k; j += blockDim.x)
        if (counts[j] == 0) atomicAdd(&s_empty, 1);
    __syncthreads();
    if (threadIdx.x == 0 && flags) flags[1] = s_empty;
}
// (4) one warp per SORT_ROWS block: stable scatter of row ids.
__global__ void label_scatter_kernel(const int *labels, int n, int k, const int *block_offsets,
                                     const int *offsets, int *sorted_rows) {
    extern __shared__ int ctr[];
    const int b = blockIdx.x;
    const int lane = threadIdx.x;
    for (int j = lane; j < k; j += 32) ctr[j] = offsets[j] + block_offsets[(size_t)b * k + j];
    __syncwarp();
    const int r0 = b * SORT_ROWS;
    const int r1 = min(n, r0 + SORT_ROWS);
    for (int base = r0; base < r1; base += 32) {
        const int i = base + lane;
        const bool valid = i < r1;
        const unsigned active = __ballot_sync(0xffffffffu, valid);
        if (valid) {
            const int lbl = labels[i];
            const unsigned peers = __match_any_sync(active, lbl);
            const unsigned lt = (1u << lane) - 1u;
            const int pos = ctr[lbl] + __popc(peers & lt);
            sorted_rows[pos] = i;
            __syncwarp(active);
            if ((__ffs(peers) - 1) == lane) ctr[lbl] += __popc(peers);
        }
        __syncwarp();
    }
}

cudaError_t launch_kmeans_sort(const int *labels, int n, int k, const int *block_counts_in,
                               int *counts, int *offsets, int *seg_chunk_start, int seg_rows,
                               int *sorted_rows, int *flags, cudaStream_t s) {
    int *block_counts = const_cast<int *>(block_counts_in);
    const int nblocks = (n + SORT_ROWS - 1) / SORT_ROWS;
    const size_t hs = (size_t)k * sizeof(int);
    label_hist_kernel<<<nblocks, 256, hs, s>>>(labels, n, k, block_counts);
    block_scan_kernel<<<(k * 32 + 255) / 256, 256, 0, s>>>(block_counts, nblocks, k, counts);
    cluster_offsets_kernel<<<1, 1024, 0, s>>>(counts, k, seg_rows, offsets, seg_chunk_start,
                                              flags);
    label_scatter_kernel<<<nblocks, 32, hs, s>>>(labels, n, k, block_counts, offsets,
                                                 sorted_rows);
    return cudaGetLastError();
}

// ------------------------------------------------------------- update ----
// One warp per (cluster, chunk of seg_rows sorted rows): fp64 sums in row order.
template <typename T>
__global__ void seg_sum_kernel(const T *X, int ld, int d, int k, const int *sorted_rows,
                               const int *offsets, const int *seg_chunk_start, int seg_rows,
                               double *chunk_sums) {
    const int w = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
    const int lane = threadIdx.x & 31;
    const int total = seg_chunk_start[k];
    if (w >= total) return;
    // cluster of chunk w: last j with seg_chunk_start[j] <= w
    int lo = 0, hi = k - 1;
    while (lo < hi) {
        const int mid = (lo + hi + 1) >> 1;
        if (seg_chunk_start[mid] <= w) lo = mid;
        else hi = mid - 1;
    }
    const int j = lo;
    const int r_begin = offsets[j] + (w - seg_chunk_start[j]) * seg_rows;
    const int r_end = min(offsets[j + 1], r_begin + seg_rows);
    double *out = chunk_sums + (size_t)w * ld;
    for (int d0 = 0; d0 < d; d0 += 128) {
        double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
        const int c0 = d0 + lane, c1 = c0 + 32, c2 = c0 + 64, c3 = c0 + 96;
        for (int r = r_begin; r < r_end; ++r) {
            const T *x = X + (size_t)sorted_rows[r] * ld;
            if (c0 < d) a0 += (double)x[c0];
            if (c1 < d) a1 += (double)x[c1];
            if (c2 < d) a2 += (double)x[c2];
            if (c3 < d) a3 += (double)x[c3];
        }
        if (c0 < d) out[c0] = a0;
        if (c1 < d) out[c1] = a1;
        if (c2 < d) out[c2] = a2;
        if (c3 < d) out[c3] = a3;
    }
}
// One thread per (cluster, feature): combine the cluster's chunks in order,
// divide, and emit per-block fp64 partials of |C_prev|^2 and |C_prev-C_new|^2.
template <typename T>
__global__ void centre_finalize_kernel(int k, int d, int ld, const int *counts,
                                       const int *seg_chunk_start, const double *chunk_sums,
                                       const T *C_prev, T *C_new, double *block_partials) {
    __shared__ double s0[256], s1[256];
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    double pn = 0.0, ps = 0.0;
    if (e < k * d) {
        const int j = e / d, f = e % d;
        double sum = 0.0;
        for (int c = seg_chunk_start[j]; c < seg_chunk_start[j + 1]; ++c)
            sum += chunk_sums[(size_t)c * ld + f];
        const int cnt = counts[j];
        const T cn = T(sum / (double)(cnt > 0 ? cnt : 1));
        const size_t o = (size_t)j * ld + f;
        const T cp = C_prev[o];
        C_new[o] = cn;
        pn = (double)cp * (double)cp;
        const double df = (double)cp - (double)cn;
        ps = df * df;
    }
    s0[threadIdx.x] = pn;
    s1[threadIdx.x] = ps;
    __syncthreads();
    for (int off = 128; off > 0; off >>= 1) {
        if ((int)threadIdx.x < off) {
            s0[threadIdx.x] += s0[threadIdx.x + off];
            s1[threadIdx.x] += s1[threadIdx.x + off];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        block_partials[2 * blockIdx.x] = s0[0];
        block_partials[2 * blockIdx.x + 1] = s1[0];
    }
}
// Single warp: sum per-block partials in block order (deterministic).
__global__ void sum_partials_kernel(const double *partials, int nblocks, int stride,
                                    int nvals, double *out) {
    const int lane = threadIdx.x;
    for (int v = 0; v < nvals; ++v) {
        double a = 0.0;
        for (int b = lane; b < nblocks; b += 32) a += partials[(size_t)b * stride + v];
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) a += __shfl_down_sync(0xffffffffu, a, off);
        if (lane == 0) out[v] = a;
    }
}

template <typename T>
cudaError_t launch_kmeans_update(const T *X, int ldx, int n, int d, int k,
                                 const int *sorted_rows, const int *offsets,
                                 const int *seg_chunk_start, int seg_rows, double *chunk_sums,
                                 const int *counts, const T *C_prev, T *C_new, int ldc,
                                 double *scalars, int *flags, cudaStream_t s) {
    (void)flags;
    (void)n;
    if (ldx != ldc) return cudaErrorInvalidValue;
    // chunk count upper bound: n / seg_rows + k
    const int max_chunks = n / seg_rows + k + 1;
    seg_sum_kernel<T><<<(max_chunks * 32 + 255) / 256, 256, 0, s>>>(
        X, ldx, d, k, sorted_rows, offsets, seg_chunk_start, seg_rows, chunk_sums);
    const int e = k * d;
    const int nb = (e + 255) / 256;
    // block partials live after the scalars block (scalars[8...])
    double *partials = scalars + 8;
    centre_finalize_kernel<T><<<nb, 256, 0, s>>>(k, d, ldc, counts, seg_chunk_start, chunk_sums,
                                                 C_prev, C_new, partials);
    sum_partials_kernel<<<1, 32, 0, s>>>(partials, nb, 2, 2, scalars);
    return cudaGetLastError();
}

// ------------------------------------------------------- centre norms ----
template <typename T>
cudaError_t launch_centre_norms(const T *C, int ldc, int k, int d, T *out, cudaStream_t s) {
    return launch_row_sqnorms<T>(C, ldc, k, d, out, s);
}

// ------------------------------------------------------------ inertia ----
template <typename T>
__global__ void inertia_kernel(const T *X, int ld, int n, int d, const T *C, const int *labels,
                               double *block_partials) {
    __shared__ double sh[8];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double acc = 0.0;
    // one warp per row (rows strided by the grid), lanes over features
    const int gw = blockIdx.x * 8 + warp;
    const int nw = gridDim.x * 8;
    for (int i = gw; i < n; i += nw) {
        const T *x = X + (size_t)i * ld;
        const T *c = C + (size_t)labels[i] * ld;
        double r = 0.0;
        for (int f = lane; f < d; f += 32) {
            const double t = (double)x[f] - (double)c[f];
            r += t * t;
        }
        acc += r;
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if (lane == 0) sh[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += sh[w];
        block_partials[blockIdx.x] = t;
    }
}
template <typename T>
cudaError_t launch_kmeans_inertia(const T *X, int ldx, int n, int d, const T *C, int ldc,
                                  const int *labels, double *block_partials, double *out,
                                  cudaStream_t s) {
    if (ldx != ldc) return cudaErrorInvalidValue;
    const int nb = 148 * 8;
    inertia_kernel<T><<<nb, 256, 0, s>>>(X, ldx, n, d, C, labels, block_partials);
    sum_partials_kernel<<<1, 32, 0, s>>>(block_partials, nb, 1, 1, out);
    return cudaGetLastError();
}

// ------------------------------------------------------------ k-means++ --
// D[c*n + i] = fl(-2 x_i.x_c + fl(|x_i|^2 + |x_c|^2)) -- the GEMM form of
// euclidean_gemm_distance with precomputed norms (kmeans.cpp:1491-1521); the
// dot product is one fma chain over the features in order.  One thread per
// row: the row is read once per group of KPP_G candidates with 16-byte loads
// (rows start on 16-byte boundaries), the candidates' rows broadcast from
// shared memory (or read through L1 when they do not fit).
static constexpr int KPP_G = 8;
template <typename T> struct Vec16;
template <> struct Vec16<float> {
    using V = float4;
    static constexpr int W = 4;
    static __device__ __forceinline__ void get(const float *p, float (&o)[4]) {
        const float4 v = *reinterpret_cast<const float4 *>(p);
        o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
    }
};
template <> struct Vec16<double> {
    static constexpr int W = 2;
    static __device__ __forceinline__ void get(const double *p, double (&o)[2]) {
        const double2 v = *reinterpret_cast<const double2 *>(p);
        o[0] = v.x; o[1] = v.y;
    }
};
template <typename T>
__global__ void __launch_bounds__(256) kpp_dist_kernel(const T *X, int ld, int n, int d,
                                                       const T *xnorm, const int *cand, int t,
                                                       T *D, int use_smem, const T *xinv,
                                                       int cosine) {
    extern __shared__ __align__(16) unsigned char sm[];
    T *cs = reinterpret_cast<T *>(sm);
    if (use_smem) {
        for (int e = threadIdx.x; e < t * d; e += blockDim.x) {
            const int c = e / d, f = e % d;
            cs[e] = X[(size_t)cand[c] * ld + f];
        }
        __syncthreads();
    }
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    constexpr int W = Vec16<T>::W;
    const T *x = X + (size_t)i * ld;
    const T xn = xnorm[i];
    for (int c0 = 0; c0 < t; c0 += KPP_G) {
        T s[KPP_G];
        const T *y[KPP_G];
#pragma unroll
        for (int g = 0; g < KPP_G; ++g) {
            const int c = min(c0 + g, t - 1);
            s[g] = T(0);
            y[g] = use_smem ? cs + (size_t)c * d : X + (size_t)cand[c] * ld;
        }
        int f = 0;
        for (; f + W <= d; f += W) {
            T xv[W];
            Vec16<T>::get(x + f, xv);
#pragma unroll
            for (int u = 0; u < W; ++u)
#pragma unroll
                for (int g = 0; g < KPP_G; ++g) s[g] = fma_rn(xv[u], y[g][f + u], s[g]);
        }
        for (; f < d; ++f) {
            const T xf = x[f];
#pragma unroll
            for (int g = 0; g < KPP_G; ++g) s[g] = fma_rn(xf, y[g][f], s[g]);
        }
#pragma unroll
        for (int g = 0; g < KPP_G; ++g)
            if (c0 + g < t) {
                const int cg = cand[c0 + g];
                D[(size_t)(c0 + g) * n + i] =
                    cosine ? cos_dist_kpp(s[g], xinv, i, cg)
                           : fma_rn(T(-2), s[g], add_rn(xn, xnorm[cg]));
            }
    }
}
template <typename T>
cudaError_t launch_kpp_dist(const T *X, int ldx, int n, int d, const T *xnorm, const int *cand,
                            int t, T *D, cudaStream_t s, const T *xinv, int cosine) {
    if (ldx % 4 != 0 || (reinterpret_cast<uintptr_t>(X) & 15) != 0) return cudaErrorInvalidValue;
    const size_t want = (size_t)t * d * sizeof(T);
    const int use_smem = want <= 48 * 1024 ? 1 : 0;
    kpp_dist_kernel<T><<<(n + 255) / 256, 256, use_smem ? want : 0, s>>>(X, ldx, n, d, xnorm,
                                                                        cand, t, D, use_smem,
                                                                        xinv, cosine);
    return cudaGetLastError();
}
template <typename T>
__global__ void kpp_cost_kernel(const T *w, const T *D, int n, int t, double *block_partials) {
    __shared__ double sh[256];
    for (int c = 0; c < t; ++c) {
        double a = 0.0;
        for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
            T v = D[(size_t)c * n + i];
            T wi = w[i];
            T m = v < wi ? v : wi;
            if (!(m > T(0))) m = T(0);
            a += (double)m;
        }
        sh[threadIdx.x] = a;
        __syncthreads();
        for (int off = 128; off > 0; off >>= 1) {
            if ((int)threadIdx.x < off) sh[threadIdx.x] += sh[threadIdx.x + off];
            __syncthreads();
        }
        if (threadIdx.x == 0) block_partials[(size_t)blockIdx.x * t + c] = sh[0];
        __syncthreads();
    }
}
template <typename T>
cudaError_t launch_kpp_cost(const T *w, const T *D, int n, int t, double *block_partials,
                            double *cost, cudaStream_t s) {
    const int nb = 148 * 4;
    kpp_cost_kernel<T><<<nb, 256, 0, s>>>(w, D, n, t, block_partials);
    sum_partials_kernel<<<1, 32, 0, s>>>(block_partials, nb, t, t, cost);
    return cudaGetLastError();
}
template <typename T>
__global__ void kpp_update_kernel(T *w, const T *Dc, int n, int chosen) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    T v = Dc[i], wi = w[i];
    T m = v < wi ? v : wi;
    if (!(m > T(0))) m = T(0);
    w[i] = (i == chosen) ? T(0) : m;
}
template <typename T>
cudaError_t launch_kpp_update(T *w, const T *Dc, int n, int chosen, cudaStream_t s) {
    kpp_update_kernel<T><<<(n + 255) / 256, 256, 0, s>>>(w, Dc, n, chosen);
    return cudaGetLastError();
}

#define B200_KM_INST(T)                                                                        \
    template cudaError_t launch_kmeans_assign<T>(const T *, int, int, int, const T *, int, int, \
                                                 const T *, int *, const int *, int *, int *,   \
                                                 cudaStream_t);                                 \
    template cudaError_t launch_kmeans_update<T>(const T *, int, int, int, int, const int *,    \
                                                 const int *, const int *, int, double *,       \
                                                 const int *, const T *, T *, int, double *,    \
                                                 int *, cudaStream_t);                          \
    template cudaError_t launch_centre_norms<T>(const T *, int, int, int, T *, cudaStream_t);   \
    template cudaError_t launch_kmeans_inertia<T>(const T *, int, int, int, const T *, int,     \
                                                  const int *, double *, double *,              \
                                                  cudaStream_t);                                \
    template cudaError_t launch_kpp_dist<T>(const T *, int, int, int, const T *, const int *,   \
                                            int, T *, cudaStream_t, const T *, int);            \
    template cudaError_t launch_kpp_cost<T>(const T *, const T *, int, int, double *, double *, \
                                            cudaStream_t);                                      \
    template cudaError_t launch_kpp_update<T>(T *, const T *, int, int, cudaStream_t);
B200_KM_INST(float)
B200_KM_INST(double)

// ------------------------------------------- spherical (cosine) k-means ---
// Inverse norms of the rows (kmeans.cpp:681-703: safe_inv of the row norm)
// and the normalised rows Xs = x_i inv_i that the centroid update sums
// (kmeans_lloyd.hpp:279-300), one element per thread.
template <typename T>
__global__ void sph_data_kernel(const T *X, int ld, int n, int d, const T *sqnorm, T *inv, T *Xs) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)n * ld) return;
    const int i = (int)(e / ld), f = (int)(e - (size_t)i * ld);
    const T sq = sqnorm[i];
    const T r = sq > T(0) ? div_rn(T(1), sqrt_rn(sq)) : T(0);
    if (f == 0) inv[i] = r;
    if (Xs) Xs[e] = f < d ? mul_rn(X[e], r) : T(0);
}
template <typename T>
cudaError_t launch_sph_data(const T *X, int ld, int n, int d, const T *sqnorm, T *inv, T *Xs,
                            cudaStream_t s) {
    const size_t tot = (size_t)n * ld;
    if (tot == 0) return cudaSuccess;
    sph_data_kernel<T><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(X, ld, n, d, sqnorm, inv, Xs);
    return cudaGetLastError();
}

// Centres to unit length (kmeans_lloyd.hpp:373-405, normalize_rows_inplace of
// da_utils.cpp:807-853; a zero row keeps the factor 1): one warp per centre;
// lane 0 sums the squares in feature order in fp64, every lane scales its
// features by 1 / sqrt of that sum.  With C_prev, per-block fp64 partials of
// |c_prev|^2 and |c_prev - c|^2 (fixed reduction order).
template <typename T>
__global__ void __launch_bounds__(256)
sph_centres_kernel(const T *C_prev, T *C, int k, int d, int ld, double *block_partials) {
    __shared__ double sh[2][8];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int j = blockIdx.x * 8 + warp;
    double pn = 0.0, ps = 0.0;
    if (j < k) {
        T *c = C + (size_t)j * ld;
        double sq = 0.0;
        if (lane == 0)
            for (int f = 0; f < d; ++f) {
                const double v = (double)c[f];
                sq = __fma_rn(v, v, sq);
            }
        sq = __shfl_sync(0xffffffffu, sq, 0);
        const double r = sq > 0.0 ? __ddiv_rn(1.0, __dsqrt_rn(sq)) : 1.0;
        for (int f = lane; f < d; f += 32) {
            const T v = (T)__dmul_rn((double)c[f], r);
            c[f] = v;
            if (C_prev) {
                const double cp = (double)C_prev[(size_t)j * ld + f];
                pn += cp * cp;
                const double df = cp - (double)v;
                ps += df * df;
            }
        }
    }
    if (!C_prev) return;
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) {
        pn += __shfl_down_sync(0xffffffffu, pn, off);
        ps += __shfl_down_sync(0xffffffffu, ps, off);
    }
    if (lane == 0) {
        sh[0][warp] = pn;
        sh[1][warp] = ps;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0, b = 0.0;
        for (int w = 0; w < 8; ++w) {
            a += sh[0][w];
            b += sh[1][w];
        }
        block_partials[2 * blockIdx.x] = a;
        block_partials[2 * blockIdx.x + 1] = b;
    }
}
template <typename T>
cudaError_t launch_sph_centres(const T *C_prev, T *C, int k, int d, int ld, double *block_partials,
                               double *scalars, cudaStream_t s) {
    const int nb = (k + 7) / 8;
    sph_centres_kernel<T><<<nb, 256, 0, s>>>(C_prev, C, k, d, ld, block_partials);
    if (C_prev) sum_partials_kernel<<<1, 32, 0, s>>>(block_partials, nb, 2, 2, scalars);
    return cudaGetLastError();
}

// Spherical inertia (kmeans.cpp:1065-1098): per row 1 - cos with the dot as
// one fma chain over the features in T, one thread per row, fp64 sum in a
// fixed order.
template <typename T>
__global__ void __launch_bounds__(256)
sph_inertia_kernel(const T *X, int ld, int n, int d, const T *C, const int *labels, const T *inv,
                   double *block_partials) {
    __shared__ double sh[8];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double acc = 0.0;
    for (int i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) {
        const T *x = X + (size_t)i * ld;
        const T *c = C + (size_t)labels[i] * ld;
        T dot = T(0);
        for (int f = 0; f < d; ++f) dot = fma_rn(x[f], c[f], dot);
        const T cs = inv ? mul_rn(dot, inv[i]) : dot;
        acc += (double)sub_rn(T(1), cs);
    }
#pragma unroll
    for (int off = 16; off > 0; off >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, off);
    if (lane == 0) sh[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += sh[w];
        block_partials[blockIdx.x] = t;
    }
}
template <typename T>
cudaError_t launch_sph_inertia(const T *X, int ld, int n, int d, const T *C, const int *labels,
                               const T *inv, double *block_partials, double *out, cudaStream_t s) {
    const int nb = 148 * 8;
    sph_inertia_kernel<T><<<nb, 256, 0, s>>>(X, ld, n, d, C, labels, inv, block_partials);
    sum_partials_kernel<<<1, 32, 0, s>>>(block_partials, nb, 1, 1, out);
    return cudaGetLastError();
}

// Cosine transform (kmeans.cpp:821-858 with dot_to_cosine_distance_*):
// D holds -dot; D = 1 - clamp(dot inv_i) with inv_i = safe_inv_sqrt(|x_i|^2).
template <typename T>
__global__ void sph_transform_kernel(T *D, int m, int k, int rowmajor, const T *sqnorm) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (e >= (size_t)m * k) return;
    const int i = rowmajor ? (int)(e / k) : (int)(e % m);
    T r = T(1);
    if (sqnorm) {
        const T sq = sqnorm[i];
        r = sq > T(0) ? div_rn(T(1), sqrt_rn(sq)) : T(0);
    }
    T cs = mul_rn(-D[e], r);
    cs = cs < T(1) ? cs : T(1);
    cs = T(-1) < cs ? cs : T(-1);
    D[e] = sub_rn(T(1), cs);
}
template <typename T>
cudaError_t launch_sph_transform(T *D, int m, int k, bool rowmajor, const T *sqnorm,
                                 cudaStream_t s) {
    const size_t tot = (size_t)m * k;
    if (tot == 0) return cudaSuccess;
    sph_transform_kernel<T><<<(unsigned)((tot + 255) / 256), 256, 0, s>>>(D, m, k, rowmajor ? 1 : 0,
                                                                         sqnorm);
    return cudaGetLastError();
}

#define B200_SPH_INST(T)                                                                       \
    template cudaError_t launch_sph_data<T>(const T *, int, int, int, const T *, T *, T *,      \
                                            cudaStream_t);                                      \
    template cudaError_t launch_sph_centres<T>(const T *, T *, int, int, int, double *, double *,\
                                               cudaStream_t);                                   \
    template cudaError_t launch_sph_inertia<T>(const T *, int, int, int, const T *, const int *,\
                                               const T *, double *, double *, cudaStream_t);    \
    template cudaError_t launch_sph_transform<T>(T *, int, int, bool, const T *, cudaStream_t);
B200_SPH_INST(float)
B200_SPH_INST(double)


// ------------------------------------------- fixed-point update (fp32 X) ---
// Centroid sums as exact 64-bit integer sums of fixed-point features: feature
// f of a row becomes q = round(x * 2^s_f), with s_f chosen once per data set
// so that n * max_i |x_if| * 2^s_f < 2^62 and max_i |x_if| * 2^s_f < 2^44.  Integer addition is associative,
// so the sums (and the centres) do not depend on the order in which rows are
// added: one streaming pass over X with shared-memory accumulators, no sort.
// The rounding error per term is at most 2^-(s_f+1) = max_i |x_if| 2^-(E+1)
// with E = min(62 - L, 44) (n <= 2^L): for n >= 2^18 that is 2^-(63-L) of the
// column maximum, below the error of an fp64 running sum over the same rows.
namespace {
constexpr int FX_SMEM_LIMIT = 200 * 1024;
constexpr int FX_THREADS = 1024;
constexpr int FX_ROWS = 8;     // rows in flight per warp (1 or 2 features per lane)
constexpr int FX_ROWS_V4 = 6;  // rows in flight per sub-warp (4 features per lane)
constexpr int FX_BATCH = 8192; // rows sorted by label per pass of a CTA
static_assert(FX_BATCH / (FX_THREADS / 32) + 1 <= 511, "run sums must fit in int32");
} // namespace

size_t fx_update_smem(int k, int d) {
    return (size_t)k * d * 8 + (size_t)FX_BATCH * 4 + (size_t)(2 * k + 2) * 4 + (size_t)d * 4;
}
int fx_update_supported(int k, int d) { return fx_update_smem(k, d) <= FX_SMEM_LIMIT ? 1 : 0; }

__global__ void col_absmax_kernel(const float *X, int ld, int n, int d, unsigned *colmax,
                                  int *nonfinite) {
    extern __shared__ unsigned cm[];
    for (int f = threadIdx.x; f < d; f += blockDim.x) cm[f] = 0u;
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    int bad = 0;
    for (int r = blockIdx.x * nw + warp; r < n; r += gridDim.x * nw) {
        const float *x = X + (size_t)r * ld;
        for (int f = lane; f < d; f += 32) {
            const unsigned b = __float_as_uint(x[f]) & 0x7fffffffu;
            if (b >= 0x7f800000u) bad = 1;
            else atomicMax(&cm[f], b);
        }
    }
    if (bad) *nonfinite = 1;
    __syncthreads();
    for (int f = threadIdx.x; f < d; f += blockDim.x) atomicMax(&colmax[f], cm[f]);
}

cudaError_t launch_col_absmax(const float *X, int ld, int n, int d, unsigned *colmax,
                              int *nonfinite, cudaStream_t s) {
    cudaError_t e = cudaMemsetAsync(colmax, 0, (size_t)d * sizeof(unsigned), s);
    if (e == cudaSuccess) e = cudaMemsetAsync(nonfinite, 0, sizeof(int), s);
    if (e != cudaSuccess) return e;
    const int blocks = max(1, min(148 * 4, (n + 31) / 32));
    col_absmax_kernel<<<blocks, 256, (size_t)d * sizeof(unsigned), s>>>(X, ld, n, d, colmax,
                                                                         nonfinite);
    return cudaGetLastError();
}

// One CTA per SM over a contiguous range of rows, in batches of FX_BATCH:
// the batch's rows are bucketed by label in shared memory (counting sort; the
// order inside a bucket does not matter, the sums are integers), then each
// warp walks an equal share of the bucketed list, keeping the running sums of
// the current cluster in registers and adding them to the CTA's shared
// accumulators only when the cluster changes.  Lanes hold VW consecutive
// features (one vector load per row); with VW = 4 and d <= 128 a row takes
// `sub_w` lanes (the next power of two >= d / 4) and the warp's 32 / sub_w
// sub-warps walk separate parts of its share, so one warp instruction serves
// several rows.  The CTA's sums and counts are finally added (integer
// reductions, order-free) into the global accumulators gsum / gcnt.
template <int VW>
__global__ void __launch_bounds__(FX_THREADS, 1)
fx_update_kernel(const float *X, int ld, int n, int d, int k, const int *labels,
                 const float *scale, unsigned long long *gsum, int *gcnt, int sub_w,
                 const int *gate, int gate_max) {
    // skipped when the gate word is at most gate_max (the graph loop's
    // delta update kept the sums up to date: fx_rescore_delta_kernel)
    if (gate && *gate <= gate_max) return;
    extern __shared__ __align__(16) unsigned char fx_smem[];
    unsigned long long *acc = reinterpret_cast<unsigned long long *>(fx_smem);
    int *list = reinterpret_cast<int *>(acc + (size_t)k * d); // FX_BATCH row ids
    int *off = list + FX_BATCH;                                  // k + 1 bucket starts
    int *cur = off + k + 1;                                      // k + 1 cursors / counts
    float *sc = reinterpret_cast<float *>(cur + k + 1);
    const int kd = k * d;
    for (int e = threadIdx.x; e < kd; e += blockDim.x) acc[e] = 0ull;
    for (int f = threadIdx.x; f < d; f += blockDim.x) sc[f] = scale[f];
    const long long per = ((long long)n + gridDim.x - 1) / gridDim.x;
    const int r0 = (int)min((long long)n, per * blockIdx.x);
    const int r1 = (int)min((long long)n, per * (blockIdx.x + 1));
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    const int W = VW == 4 ? sub_w : 32;
    const int R = 32 / W, sub = lane / W, sl = lane - sub * W;
    for (int b0 = r0; b0 < r1; b0 += FX_BATCH) {
        const int nb = min(FX_BATCH, r1 - b0);
        for (int j = threadIdx.x; j <= k; j += blockDim.x) cur[j] = 0;
        __syncthreads();
        for (int i = threadIdx.x; i < nb; i += blockDim.x) atomicAdd(&cur[labels[b0 + i]], 1);
        __syncthreads();
        if (warp == 0) { // exclusive scan of the counts -> bucket starts
            int carry = 0;
            for (int j0 = 0; j0 < k; j0 += 32) {
                const int j = j0 + lane;
                const int c = j < k ? cur[j] : 0;
                if (c > 0) atomicAdd(&gcnt[j], c);
                int x = c;
#pragma unroll
                for (int o = 1; o < 32; o <<= 1) {
                    const int y = __shfl_up_sync(0xffffffffu, x, o);
                    if (lane >= o) x += y;
                }
                if (j < k) off[j] = carry + x - c;
                carry += __shfl_sync(0xffffffffu, x, 31);
            }
            if (lane == 0) off[k] = carry;
        }
        __syncthreads();
        for (int j = threadIdx.x; j < k; j += blockDim.x) cur[j] = off[j];
        __syncthreads();
        for (int i = threadIdx.x; i < nb; i += blockDim.x)
            list[atomicAdd(&cur[labels[b0 + i]], 1)] = b0 + i;
        __syncthreads();
        // this sub-warp's part of the warp's share of the bucketed list
        const int w0 = (int)((long long)nb * warp / nw), w1 = (int)((long long)nb * (warp + 1) / nw);
        const int p0 = w0 + (int)((long long)(w1 - w0) * sub / R);
        const int p1 = w0 + (int)((long long)(w1 - w0) * (sub + 1) / R);
        if (p0 < p1) {
            int j0 = 0; // bucket holding position p0: last j with off[j] <= p0
            {
                int lo = 0, hi = k - 1;
                while (lo < hi) {
                    const int mid = (lo + hi + 1) >> 1;
                    if (off[mid] <= p0) lo = mid;
                    else hi = mid - 1;
                }
                j0 = lo;
            }
            for (int fb = 0; fb < d; fb += VW * W) {
                const int f = fb + VW * sl;
                float sv[VW], sv22[VW];
#pragma unroll
                for (int v = 0; v < VW; ++v) {
                    sv[v] = f + v < d ? sc[f + v] : 0.f;
                    sv22[v] = sv[v] * 2.384185791015625e-07f;
                }
                int j = j0;
                int jend = off[j + 1];
                FxRunV<VW> run;
                run.reset();
                constexpr int NR = VW == 4 ? FX_ROWS_V4 : FX_ROWS;
                for (int p = p0; p < p1; p += NR) {
                    float xv[NR][VW];
#pragma unroll
                    for (int u = 0; u < NR; ++u) {
#pragma unroll
                        for (int v = 0; v < VW; ++v) xv[u][v] = 0.f;
                        if (p + u < p1 && f < d) {
                            const float *xr = X + (size_t)list[p + u] * ld + f;
                            if (VW == 4) {
                                const float4 t = *reinterpret_cast<const float4 *>(xr);
                                xv[u][0] = t.x, xv[u][1] = t.y, xv[u][VW > 2 ? 2 : 0] = t.z,
                                xv[u][VW > 3 ? 3 : 0] = t.w;
                            } else if (VW == 2) {
                                const float2 t = *reinterpret_cast<const float2 *>(xr);
                                xv[u][0] = t.x, xv[u][VW > 1 ? 1 : 0] = t.y;
                            } else {
                                xv[u][0] = *xr;
                            }
                        }
                    }
#pragma unroll
                    for (int u = 0; u < NR; ++u) {
                        if (p + u < p1) {
                            while (p + u >= jend) { // next non-empty bucket
                                fx_flush_v<VW>(acc, d, j, f, run);
                                ++j;
                                jend = off[j + 1];
                            }
#pragma unroll
                            for (int v = 0; v < VW; ++v)
                                fx_acc(xv[u][v], sv22[v], sv[v], run.h[v], run.l[v]);
                            ++run.n;
                        }
                    }
                }
                fx_flush_v<VW>(acc, d, j, f, run);
            }
        }
        __syncthreads();
    }
    for (int e = threadIdx.x; e < kd; e += blockDim.x)
        if (acc[e]) atomicAdd(&gsum[e], acc[e]);
}

// Vector width and sub-warp width of the update for X's layout.
static void fx_shape(const float *X, int ld, int d, int &vw, int &sub_w) {
    const uintptr_t a = reinterpret_cast<uintptr_t>(X);
    sub_w = 32;
    if (d % 4 == 0 && ld % 4 == 0 && (a & 15) == 0 && d <= 128) {
        vw = 4;
        sub_w = 1;
        while (sub_w * 4 < d) sub_w <<= 1;
    } else if (d % 2 == 0 && ld % 2 == 0 && (a & 7) == 0) {
        vw = 2;
    } else {
        vw = 1;
    }
}

static void fx_launch(const float *X, int ld, int n, int d, int k, const int *labels,
                      const float *scale, unsigned long long *sums, int *counts, int nsm,
                      size_t smem, cudaStream_t s, const int *gate = nullptr, int gate_max = 0) {
    int vw = 1, sub_w = 32;
    fx_shape(X, ld, d, vw, sub_w);
    if (vw == 4)
        fx_update_kernel<4><<<nsm, FX_THREADS, smem, s>>>(X, ld, n, d, k, labels, scale, sums,
                                                          counts, sub_w, gate, gate_max);
    else if (vw == 2)
        fx_update_kernel<2><<<nsm, FX_THREADS, smem, s>>>(X, ld, n, d, k, labels, scale, sums,
                                                          counts, sub_w, gate, gate_max);
    else
        fx_update_kernel<1><<<nsm, FX_THREADS, smem, s>>>(X, ld, n, d, k, labels, scale, sums,
                                                          counts, sub_w, gate, gate_max);
}


// The graph loop's exact re-score and delta update in one launch.  Every
// block reads the final counts of the tensor-core pass first: with the
// changed certified rows plus the listed (uncertified) rows within `cap` the
// sums are brought up to date here -- a listed row whose exact label differs
// from its previous one moves its fixed-point features at once, the changed
// certified rows from the change list -- else the sums and counts are
// cleared and *recount = 1 asks the recount that follows.  Listed rows: one
// lane per row over warp tasks of 32 rows dealt to the blocks first, the
// candidates' dot products as the plain path's fma chains (features in
// order), v = fl(-2 s + |c|^2), ties to the lower cluster; a row with no
// candidate list scans every cluster with the whole warp.  Xr: the rows the
// labels are computed from; Xu: the rows the sums hold (the same here).
template <bool VEC>
__global__ void __launch_bounds__(256)
fx_rescore_delta_kernel(const float *Xr, const float *Xu, int ld, int d, const float *C, int k,
                        const float *cnorm, AmbList amb, int *labels, int *flags,
                        const float *scale, const int *count, int cap, const int *rows,
                        const int *olds, const int *news, unsigned long long *sum, int *cnt,
                        int *recount) {
    const int lane = threadIdx.x & 31, wib = threadIdx.x >> 5, nwb = blockDim.x >> 5;
    const int na = *amb.count;
    const int c = *count;
    const bool delta = (long long)c + na <= (long long)cap;
    if (blockIdx.x == 0 && threadIdx.x == 0) *recount = delta ? 0 : 1;
    if (!delta) {
        const int kd = k * d;
        for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < kd; e += gridDim.x * blockDim.x)
            sum[e] = 0ull;
        for (int j = blockIdx.x * blockDim.x + threadIdx.x; j < k; j += gridDim.x * blockDim.x)
            cnt[j] = 0;
    }
    const int nwarps = gridDim.x * nwb;
    const int gw = wib * gridDim.x + blockIdx.x;
    const float inf = __int_as_float(0x7f800000);
    int changed = 0;
    for (int e0 = gw * 32; e0 < na; e0 += nwarps * 32) {
        const int e = e0 + lane;
        const bool in = e < na;
        const int nc = in ? amb.ncand[e] : -1;
        const int r = in ? amb.rows[e] : 0;
        int cand_raw[KM_AMB_MAXC];
#pragma unroll
        for (int q = 0; q < KM_AMB_MAXC; ++q)
            cand_raw[q] = in ? amb.cand[(size_t)e * KM_AMB_MAXC + q] : 0;
        const int old_l = in ? labels[r] : -1;
        int lbl = old_l;
        if (nc > 0) {
            int cj[KM_AMB_MAXC];
            const float *cp[KM_AMB_MAXC];
            float sd[KM_AMB_MAXC];
#pragma unroll
            for (int q = 0; q < KM_AMB_MAXC; ++q) {
                cj[q] = q < nc ? cand_raw[q] : cand_raw[0];
                cp[q] = C + (size_t)cj[q] * ld;
                sd[q] = 0.f;
            }
            const float *xr = Xr + (size_t)r * ld;
            if (VEC) {
#pragma unroll 4
                for (int f = 0; f < d; f += 4) {
                    const float4 xv = *reinterpret_cast<const float4 *>(xr + f);
#pragma unroll
                    for (int q = 0; q < KM_AMB_MAXC; ++q) {
                        const float4 cv = *reinterpret_cast<const float4 *>(cp[q] + f);
                        sd[q] = __fmaf_rn(xv.x, cv.x, sd[q]);
                        sd[q] = __fmaf_rn(xv.y, cv.y, sd[q]);
                        sd[q] = __fmaf_rn(xv.z, cv.z, sd[q]);
                        sd[q] = __fmaf_rn(xv.w, cv.w, sd[q]);
                    }
                }
            } else {
                for (int f = 0; f < d; ++f) {
                    const float xf = xr[f];
#pragma unroll
                    for (int q = 0; q < KM_AMB_MAXC; ++q) sd[q] = __fmaf_rn(xf, cp[q][f], sd[q]);
                }
            }
            float best = inf;
            int bi = 0x7fffffff;
#pragma unroll
            for (int q = 0; q < KM_AMB_MAXC; ++q) {
                if (q < nc) {
                    const float v = __fmaf_rn(-2.f, sd[q], cnorm[cj[q]]);
                    if (key_less(v, cj[q], best, bi)) {
                        best = v;
                        bi = cj[q];
                    }
                }
            }
            lbl = (bi == 0x7fffffff) ? cj[0] : bi;
        }
        unsigned full = __ballot_sync(0xffffffffu, nc == 0);
        while (full) {
            const int src = __ffs(full) - 1;
            full &= full - 1;
            const float *xr = Xr + (size_t)__shfl_sync(0xffffffffu, r, src) * ld;
            float best = inf;
            int bi = 0x7fffffff;
            for (int j0 = lane; j0 < k; j0 += 128) {
                const float *cc[4];
                float sd[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
                for (int t = 0; t < 4; ++t) cc[t] = C + (size_t)min(j0 + 32 * t, k - 1) * ld;
                for (int f = 0; f < d; ++f) {
                    const float xf = xr[f];
#pragma unroll
                    for (int t = 0; t < 4; ++t) sd[t] = __fmaf_rn(xf, cc[t][f], sd[t]);
                }
#pragma unroll
                for (int t = 0; t < 4; ++t) {
                    const int j = j0 + 32 * t;
                    if (j < k) {
                        const float v = __fmaf_rn(-2.f, sd[t], cnorm[j]);
                        if (key_less(v, j, best, bi)) {
                            best = v;
                            bi = j;
                        }
                    }
                }
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) {
                const float ov = __shfl_xor_sync(0xffffffffu, best, off);
                const int oi = __shfl_xor_sync(0xffffffffu, bi, off);
                if (key_less(ov, oi, best, bi)) {
                    best = ov;
                    bi = oi;
                }
            }
            if (lane == src) lbl = (bi == 0x7fffffff) ? 0 : bi;
        }
        if (in) labels[r] = lbl;
        const bool ch = in && lbl != old_l;
        if (ch) changed = 1;
        // the changed rows' features move from the old cluster to the new
        unsigned mv = __ballot_sync(0xffffffffu, ch && delta);
        while (mv) {
            const int src = __ffs(mv) - 1;
            mv &= mv - 1;
            const int rs = __shfl_sync(0xffffffffu, r, src);
            const int jo = __shfl_sync(0xffffffffu, old_l, src);
            const int jn = __shfl_sync(0xffffffffu, lbl, src);
            const float *x = Xu + (size_t)rs * ld;
            for (int f = lane; f < d; f += 32) {
                const long long q = __double2ll_rn((double)x[f] * (double)scale[f]);
                atomicAdd(&sum[(size_t)jn * d + f], (unsigned long long)q);
                atomicAdd(&sum[(size_t)jo * d + f], (unsigned long long)(-q));
            }
            if (lane == 0) {
                atomicAdd(&cnt[jn], 1);
                atomicSub(&cnt[jo], 1);
            }
        }
    }
    if (__any_sync(0xffffffffu, changed) && lane == 0) atomicOr(&flags[0], 1);
    if (!delta) return;
    // the changed certified rows: one warp per row moves its fixed-point
    // features q = round-to-nearest-even(x * 2^s_f), the values fx_acc adds
    for (int e = gw; e < c; e += nwarps) {
        const int r = rows[e], jo = olds[e], jn = news[e];
        const float *x = Xu + (size_t)r * ld;
        for (int f = lane; f < d; f += 32) {
            const long long q = __double2ll_rn((double)x[f] * (double)scale[f]);
            atomicAdd(&sum[(size_t)jn * d + f], (unsigned long long)q);
            atomicAdd(&sum[(size_t)jo * d + f], (unsigned long long)(-q));
        }
        if (lane == 0) {
            atomicAdd(&cnt[jn], 1);
            atomicSub(&cnt[jo], 1);
        }
    }
}

// One thread per (cluster, feature): the mean from the global sums, and fp64
// block partials of |C_prev|^2 and |C_prev - C_new|^2; the last block to
// finish sums the block partials in block order (deterministic) into
// scalars[0..1] and re-arms the ticket.  The other accumulator pair
// (nsum / ncnt, used by the next update) is cleared here when given.
// Counts are int (one device's accumulators) or int64 (the sum over the
// shards of a data set split across processes).
//
// With `ls` (the Lloyd loop run as a CUDA graph), the last block also makes
// the convergence test of the host loop for iteration ls->it -- no label
// changed after iteration 1, or |C_prev - C_new| < tol |C_prev| -- and ends
// the graph's WHILE node (cond) when it passes or max_iter is reached.
template <typename CT>
__global__ void __launch_bounds__(256)
fx_finalize_kernel(int k, int d, int ld, const unsigned long long *gsum, const CT *gcnt,
                   unsigned long long *nsum, int *ncnt, const double *inv_scale,
                   const float *C_prev, float *C_new, int *counts, double *block_partials,
                   double *scalars, int *flags, unsigned *ticket, LloydLoopState *ls,
                   unsigned long long cond, int *rearm0 = nullptr, int *rearm1 = nullptr) {
    __shared__ double s0[256], s1[256];
    __shared__ bool last;
    const int kd = k * d;
    const int e = blockIdx.x * blockDim.x + threadIdx.x;
    double pn = 0.0, ps = 0.0;
    if (e < kd) {
        const int j = e / d, f = e - j * d;
        const long long S = (long long)gsum[e];
        const long long c = (long long)gcnt[j];
        if (nsum) nsum[e] = 0ull;
        if (ncnt && f == 0) ncnt[j] = 0;
        const double mean = ((double)S * inv_scale[f]) / (double)(c > 0 ? c : 1);
        const float cn = (float)mean;
        const size_t o = (size_t)j * ld + f;
        const float cp = C_prev[o];
        C_new[o] = cn;
        pn = (double)cp * (double)cp;
        const double df = (double)cp - (double)cn;
        ps = df * df;
        if (f == 0) {
            if (counts) counts[j] = (int)c;
            if (c == 0 && flags) atomicAdd(&flags[1], 1);
        }
    }
    s0[threadIdx.x] = pn;
    s1[threadIdx.x] = ps;
    __syncthreads();
    for (int off = 128; off > 0; off >>= 1) {
        if ((int)threadIdx.x < off) {
            s0[threadIdx.x] += s0[threadIdx.x + off];
            s1[threadIdx.x] += s1[threadIdx.x + off];
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        block_partials[2 * blockIdx.x] = s0[0];
        block_partials[2 * blockIdx.x + 1] = s1[0];
        __threadfence();
        last = atomicAdd(ticket, 1u) == gridDim.x - 1;
    }
    __syncthreads();
    if (last && threadIdx.x < 32) {
        __threadfence();
        const int lane = threadIdx.x;
        double sv[2];
        for (int v = 0; v < 2; ++v) {
            double a = 0.0;
            for (int b = lane; b < (int)gridDim.x; b += 32)
                a += __ldcg(&block_partials[2 * b + v]);
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) a += __shfl_down_sync(0xffffffffu, a, off);
            if (lane == 0) scalars[v] = a;
            sv[v] = a;
        }
        if (lane == 0) *ticket = 0u;
        if (ls && lane == 0) {
            const int it = ls->it;
            int conv = 0;
            if (it > 1 && *((volatile int *)flags) == 0) conv = 2;
            if (conv == 0 && sqrt(sv[1]) < ls->tol * sqrt(sv[0])) conv = 1;
            const int next = it + 1;
            const bool stop = conv > 0 || next >= ls->max_iter;
            ls->conv = conv;
            ls->n_iter = conv > 0 ? it : next;
            ls->it = next;
            if (stop) cudaGraphSetConditional(cond, 0);
            // the next iteration's counters start at zero: the label-change and
            // empty-cluster flags (read above), the relabel list count and its
            // full-scan count (rearm0[0], rearm0[2]; rearm0[1] is the sticky
            // error word), the changed-row count (rearm1[0])
            flags[0] = 0;
            flags[1] = 0;
            if (rearm0) {
                rearm0[0] = 0;
                rearm0[2] = 0;
            }
            if (rearm1) rearm1[0] = 0;
        }
    }
}

static cudaError_t fx_smem_limit(size_t smem) {
    cudaError_t e = ensure_smem_limit(reinterpret_cast<const void *>(fx_update_kernel<4>), smem);
    if (e == cudaSuccess)
        e = ensure_smem_limit(reinterpret_cast<const void *>(fx_update_kernel<2>), smem);
    if (e == cudaSuccess)
        e = ensure_smem_limit(reinterpret_cast<const void *>(fx_update_kernel<1>), smem);
    return e;
}

cudaError_t launch_kmeans_update_fx(const float *X, int ld, int n, int d, int k,
                                    const int *labels, const float *scale,
                                    const double *inv_scale, void *accum, int parity,
                                    const float *C_prev, float *C_new, int *counts,
                                    double *block_partials, double *scalars, int *flags,
                                    unsigned *ticket, cudaStream_t s) {
    const size_t smem = fx_update_smem(k, d);
    if (smem > (size_t)FX_SMEM_LIMIT) return cudaErrorInvalidValue;
    cudaError_t e = fx_smem_limit(smem);
    if (e != cudaSuccess) return e;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const size_t kd = (size_t)k * d;
    unsigned long long *sum[2] = {static_cast<unsigned long long *>(accum),
                                  static_cast<unsigned long long *>(accum) + kd};
    int *cnt[2] = {reinterpret_cast<int *>(sum[1] + kd),
                   reinterpret_cast<int *>(sum[1] + kd) + k};
    const int p = parity & 1;
    fx_launch(X, ld, n, d, k, labels, scale, sum[p], cnt[p], nsm, smem, s);
    const int nb = (int)((kd + 255) / 256);
    fx_finalize_kernel<int><<<nb, 256, 0, s>>>(k, d, ld, sum[p], cnt[p], sum[1 - p], cnt[1 - p],
                                               inv_scale, C_prev, C_new, counts, block_partials,
                                               scalars, flags, ticket, nullptr, 0ull);
    return cudaGetLastError();
}

cudaError_t launch_kmeans_update_fx_loop(const float *X, int ld, int n, int d, int k,
                                         int *labels, const float *scale,
                                         const double *inv_scale, void *accum, float *C,
                                         int *counts, double *block_partials, double *scalars,
                                         int *flags, unsigned *ticket, LloydLoopState *ls,
                                         unsigned long long cond, const ChangeList &chg,
                                         int *rearm, const float *cnorm, const AmbList &amb,
                                         int *recount, cudaStream_t s) {
    const size_t smem = fx_update_smem(k, d);
    if (smem > (size_t)FX_SMEM_LIMIT || !chg.count || !amb.count || !recount)
        return cudaErrorInvalidValue;
    cudaError_t e = fx_smem_limit(smem);
    if (e != cudaSuccess) return e;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    const size_t kd = (size_t)k * d;
    unsigned long long *sum = static_cast<unsigned long long *>(accum);
    int *cnt = reinterpret_cast<int *>(sum + 2 * kd);
    // the listed rows' exact labels with a short change list's delta update,
    // or with the clearing of the sums for the recount that follows
    const bool vec = (d % 4 == 0) && (ld % 4 == 0) &&
                     ((reinterpret_cast<uintptr_t>(X) | reinterpret_cast<uintptr_t>(C)) & 15) == 0;
    if (vec)
        fx_rescore_delta_kernel<true><<<nsm * 4, 256, 0, s>>>(
            X, X, ld, d, C, k, cnorm, amb, labels, flags, scale, chg.count, chg.cap, chg.rows,
            chg.olds, chg.news, sum, cnt, recount);
    else
        fx_rescore_delta_kernel<false><<<nsm * 4, 256, 0, s>>>(
            X, X, ld, d, C, k, cnorm, amb, labels, flags, scale, chg.count, chg.cap, chg.rows,
            chg.olds, chg.news, sum, cnt, recount);
    fx_launch(X, ld, n, d, k, labels, scale, sum, cnt, nsm, smem, s, recount, 0);
    const int nb = (int)((kd + 255) / 256);
    // in place: each element's old value is read by the thread that writes it;
    // the last block re-arms the iteration's counters
    fx_finalize_kernel<int><<<nb, 256, 0, s>>>(k, d, ld, sum, cnt, nullptr, nullptr, inv_scale,
                                               C, C, counts, block_partials, scalars, flags,
                                               ticket, ls, cond, rearm, chg.count);
    return cudaGetLastError();
}

// acc[k*d + j] = counts[j]; acc[k*d + k] = the label-change flag.
__global__ void fx_pack_counts_kernel(int k, int kd, const int *counts, const int *changed,
                                      long long *acc) {
    const int j = blockIdx.x * blockDim.x + threadIdx.x;
    if (j < k) acc[kd + j] = (long long)counts[j];
    if (j == k) acc[kd + k] = changed ? (long long)(*changed != 0) : 0ll;
}

cudaError_t launch_kmeans_sums_fx(const float *X, int ld, int n, int d, int k, const int *labels,
                                  const float *scale, long long *acc, int *counts,
                                  const int *changed, cudaStream_t s) {
    unsigned long long *sums = reinterpret_cast<unsigned long long *>(acc);
    const size_t smem = fx_update_smem(k, d);
    if (smem > (size_t)FX_SMEM_LIMIT) return cudaErrorInvalidValue;
    int dev = 0, nsm = 148;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    cudaError_t e = fx_smem_limit(smem);
    if (e == cudaSuccess) e = cudaMemsetAsync(sums, 0, (size_t)k * d * 8, s);
    if (e == cudaSuccess) e = cudaMemsetAsync(counts, 0, (size_t)k * 4, s);
    if (e != cudaSuccess) return e;
    fx_launch(X, ld, n, d, k, labels, scale, sums, counts, nsm, smem, s);
    fx_pack_counts_kernel<<<(k + 1 + 255) / 256, 256, 0, s>>>(k, k * d, counts, changed, acc);
    return cudaGetLastError();
}

cudaError_t launch_kmeans_finalize_shards(int k, int d, int ld, const long long *acc,
                                          const double *inv_scale, const float *C_prev,
                                          float *C_new, double *block_partials, double *scalars,
                                          int *flags, unsigned *ticket, cudaStream_t s) {
    const size_t kd = (size_t)k * d;
    const int nb = (int)((kd + 255) / 256);
    fx_finalize_kernel<long long><<<nb, 256, 0, s>>>(
        k, d, ld, reinterpret_cast<const unsigned long long *>(acc), acc + kd, nullptr, nullptr,
        inv_scale, C_prev, C_new, nullptr, block_partials, scalars, flags, ticket, nullptr, 0ull);
    return cudaGetLastError();
}

size_t fx_accum_bytes(int k, int d) { return (size_t)2 * k * d * 8 + (size_t)2 * k * 4; }

} // namespace b200
