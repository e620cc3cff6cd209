// IVF-flat inverted-list scan (approximate_neighbors.cpp:971-1191): for every
// query, the GEMM-form squared distances |q|^2 + |v|^2 - 2 q.v (or, for the
// inner-product and cosine indexes, -q.v) to the vectors of its n_probe
// probed lists, and the k smallest of them.
//
// One CTA per query.  The probed lists are contiguous row ranges of the
// list-ordered index (rows padded to a multiple of 4 elements, so every row
// starts on a 16-byte boundary); a batch of 256 candidates is scored by groups
// of four lanes (16-byte loads, two shuffles per dot product), then the
// candidates below the current k-th key are merged into the shared-memory
// top-k by rank counting.  Keys are (distance, global index) pairs compared
// lexicographically, so the result is exact and deterministic: the k smallest
// distances over the probed lists, equal distances in index order.
#include "b200_common.cuh"
#include "b200_kernels.hpp"

namespace b200 {

namespace {

constexpr int IVF_THREADS = 256;
constexpr int IVF_GROUP = 4;          // lanes per candidate row
constexpr int IVF_BATCH = 256;        // candidates per merge step (== threads)
constexpr int IVF_NOID = 0x7fffffff;  // empty top-k slot

template <typename T> struct V16;
template <> struct V16<float> {
    using V = float4;
    static constexpr int N = 4;
    static B200_DEV float dot(const float4 &a, const float4 &b, float acc) {
        acc = fmaf(a.x, b.x, acc);
        acc = fmaf(a.y, b.y, acc);
        acc = fmaf(a.z, b.z, acc);
        return fmaf(a.w, b.w, acc);
    }
};
template <> struct V16<double> {
    using V = double2;
    static constexpr int N = 2;
    static B200_DEV double dot(const double2 &a, const double2 &b, double acc) {
        acc = fma(a.x, b.x, acc);
        return fma(a.y, b.y, acc);
    }
};

template <typename T>
__global__ void __launch_bounds__(IVF_THREADS)
ivf_scan_kernel(const T *__restrict__ Q, const T *__restrict__ qn, int ld, int nq,
                const int *__restrict__ probe, int n_probe, const long long *__restrict__ loff,
                const T *__restrict__ X, const T *__restrict__ xn, const int *__restrict__ gid,
                int k, int out, T *__restrict__ out_d, int *__restrict__ out_i) {
    using V = typename V16<T>::V;
    extern __shared__ __align__(16) unsigned char ivf_smem[];
    T *Ld = reinterpret_cast<T *>(ivf_smem); // current top-k, ascending
    T *Nd = Ld + k;                          // merge output
    T *Bd = Nd + k;                          // batch distances
    T *Sd = Bd + IVF_BATCH;                  // survivors
    int *Li = reinterpret_cast<int *>(Sd + IVF_BATCH);
    int *Ni = Li + k;
    int *Bi = Ni + k;
    int *Si = Bi + IVF_BATCH;
    __shared__ int s_ns;
    const int tid = threadIdx.x;
    const int g = tid / IVF_GROUP, lane = tid % IVF_GROUP;
    const int nvec = ld / V16<T>::N;
    const T inf = Lim<T>::inf();

    for (int q = blockIdx.x; q < nq; q += gridDim.x) {
        for (int r = tid; r < k; r += IVF_THREADS) {
            Ld[r] = inf;
            Li[r] = IVF_NOID;
        }
        const V *qv = reinterpret_cast<const V *>(Q + (size_t)q * ld);
        const T qq = qn[q];
        __syncthreads();
        for (int p = 0; p < n_probe; ++p) {
            const int list = probe[(size_t)q * n_probe + p];
            const long long beg = loff[list], end = loff[list + 1];
            for (long long b0 = beg; b0 < end; b0 += IVF_BATCH) {
                const int nb = (int)((end - b0) < IVF_BATCH ? (end - b0) : IVF_BATCH);
                // every thread runs the same number of iterations: the group
                // shuffles below always have the whole warp
                for (int c = g; c < IVF_BATCH; c += IVF_THREADS / IVF_GROUP) {
                    T acc = T(0);
                    const bool valid = c < nb;
                    if (valid) {
                        const V *row = reinterpret_cast<const V *>(X + (size_t)(b0 + c) * ld);
                        for (int j = lane; j < nvec; j += IVF_GROUP)
                            acc = V16<T>::dot(__ldg(qv + j), __ldg(row + j), acc);
                    }
                    acc += __shfl_xor_sync(0xffffffffu, acc, 1);
                    acc += __shfl_xor_sync(0xffffffffu, acc, 2);
                    if (lane == 0) {
                        if (valid) {
                            Bd[c] = out >= IVF_OUT_IP ? -acc
                                                      : add_rn(add_rn(qq, xn[b0 + c]), T(-2) * acc);
                            Bi[c] = gid[b0 + c];
                        } else {
                            Bd[c] = inf;
                            Bi[c] = IVF_NOID;
                        }
                    }
                }
                if (tid == 0) s_ns = 0;
                __syncthreads();
                // survivors: keys below the current k-th key
                {
                    const T td = Ld[k - 1];
                    const int ti = Li[k - 1];
                    const T d = Bd[tid];
                    const int i = Bi[tid];
                    if (i != IVF_NOID && key_less(d, i, td, ti)) {
                        const int slot = atomicAdd(&s_ns, 1);
                        Sd[slot] = d;
                        Si[slot] = i;
                    }
                }
                __syncthreads();
                const int ns = s_ns;
                if (ns > 0) {
                    // merged position = own rank + the other list's count below
                    if (tid < ns) {
                        const T d = Sd[tid];
                        const int i = Si[tid];
                        int r = 0;
                        for (int j = 0; j < ns; ++j) r += key_less(Sd[j], Si[j], d, i) ? 1 : 0;
                        int lo = 0, hi = k;
                        while (lo < hi) {
                            const int mid = (lo + hi) >> 1;
                            if (key_less(Ld[mid], Li[mid], d, i)) lo = mid + 1;
                            else hi = mid;
                        }
                        r += lo;
                        if (r < k) {
                            Nd[r] = d;
                            Ni[r] = i;
                        }
                    }
                    for (int e = tid; e < k; e += IVF_THREADS) {
                        const T d = Ld[e];
                        const int i = Li[e];
                        int r = e;
                        for (int j = 0; j < ns; ++j) r += key_less(Sd[j], Si[j], d, i) ? 1 : 0;
                        if (r < k) {
                            Nd[r] = d;
                            Ni[r] = i;
                        }
                    }
                    __syncthreads();
                    for (int e = tid; e < k; e += IVF_THREADS) {
                        Ld[e] = Nd[e];
                        Li[e] = Ni[e];
                    }
                }
                __syncthreads();
            }
        }
        // empty slots: index -1, key +inf; euclidean: the square root of
        // non-negative values; inner product: -key; cosine: 1 + key
        // (approximate_neighbors.cpp:1287-1312)
        for (int r = tid; r < k; r += IVF_THREADS) {
            const int i = Li[r];
            T d = i == IVF_NOID ? inf : Ld[r];
            if (out == IVF_OUT_SQRT && d >= T(0)) d = sqrt_rn(d);
            else if (out == IVF_OUT_IP) d = -d;
            else if (out == IVF_OUT_COS) d = add_rn(T(1), d);
            out_d[(size_t)q * k + r] = d;
            out_i[(size_t)q * k + r] = i == IVF_NOID ? -1 : i;
        }
        __syncthreads();
    }
}

} // namespace

size_t ivf_scan_smem(int k, bool fp64) {
    const size_t e = (fp64 ? sizeof(double) : sizeof(float)) + sizeof(int);
    return (2 * (size_t)k + 2 * IVF_BATCH) * e;
}

template <typename T>
cudaError_t launch_ivf_scan(const T *Q, const T *qn, int ld, int nq, const int *probe,
                            int n_probe, const long long *loff, const T *X, const T *xn,
                            const int *gid, int k, int out, T *out_d, int *out_i,
                            cudaStream_t s) {
    if (nq <= 0) return cudaSuccess;
    if (ld % 4 != 0 || k < 1) return cudaErrorInvalidValue;
    const size_t smem = ivf_scan_smem(k, sizeof(T) == 8);
    cudaError_t e = ensure_smem_limit((const void *)ivf_scan_kernel<T>, smem);
    if (e != cudaSuccess) return e;
    const int grid = nq < 148 * 64 ? nq : 148 * 64;
    ivf_scan_kernel<T><<<grid, IVF_THREADS, smem, s>>>(Q, qn, ld, nq, probe, n_probe, loff, X,
                                                        xn, gid, k, out, out_d, out_i);
    return cudaGetLastError();
}

template cudaError_t launch_ivf_scan<float>(const float *, const float *, int, int, const int *,
                                            int, const long long *, const float *, const float *,
                                            const int *, int, int, float *, int *, cudaStream_t);
template cudaError_t launch_ivf_scan<double>(const double *, const double *, int, int,
                                             const int *, int, const long long *,
                                             const double *, const double *, const int *, int,
                                             int, double *, int *, cudaStream_t);

} // namespace b200
