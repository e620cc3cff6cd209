// k-means++ initialisation on the device (clustering/kmeans/kmeans.cpp:
// 1524-1664) with the reference's random draws.
//
// The reference picks every candidate centre with std::discrete_distribution
// over the current minimum squared distances w: one canonical double u in
// [0, 1) per draw, then the first index i whose cumulative probability
// cp_i >= u, where cp is the sequential double prefix sum of w_j / S and S
// the sequential double sum of w (cp of the last index set to 1).  The host
// draws the u values from the same engine in the same order; the device
// maps them to indices:
//   * kpp_draw_kernel: block sums of w (2,048 weights a block, written by
//     the kernel that last changed w), their prefix, the block holding u S
//     and the index within it -- a parallel prefix whose value P'_i / S'
//     differs from the sequential cp_i by at most
//     bound = 1.2 (2 n + 2 nb + 4200) 2^-53 (first-order rounding of the two
//     sequential sums, the divisions and the parallel sums).  The index is
//     certified when u - P'_{i-1} / S' and P'_i / S' - u both exceed the
//     bound; then the sequential search returns the same index.
//   * kpp_exact_kernel: the draws that are not certified (about one per
//     k-means++ run on a million rows) are redone with the sequential sums
//     themselves, in the reference's order of operations.
// The candidates' distances are the kpp_dist kernel; their costs are the
// reference's serial sums in the working precision, reproduced exactly by
// kpp_serial_cost_kernel (at a million fp32 rows the rounding of those sums
// decides between candidates whose costs are that close, so an fp64 sum
// would choose differently); kpp_select_update_kernel picks the candidate
// with the smallest finite cost (repeats skipped, first strictly smaller wins), writes it to
// `chosen`, lowers w to the minimum with its distances, zeroes its own
// weight and writes the block sums of the new w.  No host round trip per
// centre.
#include "b200_common.cuh"

namespace b200 {

static constexpr int KPP_THREADS = 256;
static constexpr int KPP_PER_THREAD = 8;
static constexpr int KPP_BLOCK = KPP_THREADS * KPP_PER_THREAD;
static constexpr int KPP_EXACT_TILE = 4096;

__device__ __forceinline__ bool finite_(float v) { return isfinite(v); }
__device__ __forceinline__ bool finite_(double v) { return isfinite(v); }

// Block-wide exclusive prefix sum of one double per thread (fixed order);
// `total` receives the block's sum.  sh: KPP_THREADS / 32 + 1 doubles.
__device__ double block_exclusive_scan(double v, double *sh, double &total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    double x = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const double y = __shfl_up_sync(0xffffffffu, x, off);
        if (lane >= off) x += y;
    }
    double ex = __shfl_up_sync(0xffffffffu, x, 1);
    if (lane == 0) ex = 0.0;
    __syncthreads();
    if (lane == 31) sh[warp] = x;
    __syncthreads();
    if (threadIdx.x == 0) {
        double a = 0.0;
        for (int w = 0; w < KPP_THREADS / 32; ++w) {
            const double t = sh[w];
            sh[w] = a;
            a += t;
        }
        sh[KPP_THREADS / 32] = a;
    }
    __syncthreads();
    total = sh[KPP_THREADS / 32];
    return sh[warp] + ex;
}

// w_i = 0 where negative or not finite, and at the first centre; block sums
// of w; flag[0] = 1 when some weight is positive (kmeans.cpp:1571-1590).
template <typename T>
__global__ void __launch_bounds__(KPP_THREADS)
kpp_clamp_kernel(T *w, int n, int first, double *bs, int *flag) {
    __shared__ double sh[KPP_THREADS / 32 + 1];
    const size_t base = (size_t)blockIdx.x * KPP_BLOCK + (size_t)threadIdx.x * KPP_PER_THREAD;
    double s = 0.0;
    bool pos = false;
#pragma unroll
    for (int j = 0; j < KPP_PER_THREAD; ++j) {
        const size_t i = base + j;
        if (i < (size_t)n) {
            T v = w[i];
            if (!finite_(v) || v < T(0) || (int)i == first) v = T(0);
            w[i] = v;
            pos = pos || v > T(0);
            s += (double)v;
        }
    }
    double tot;
    block_exclusive_scan(s, sh, tot);
    if (threadIdx.x == 0) bs[blockIdx.x] = tot;
    if (__syncthreads_or(pos) && threadIdx.x == 0) atomicOr(flag, 1);
}

// One block per draw t: the index that std::discrete_distribution gives for
// u = U[t] over the weights w, certified against the bound (unc[t] = 0), or
// an approximate index with unc[t] = 1 for the exact kernel to redo.
template <typename T>
__global__ void __launch_bounds__(KPP_THREADS)
kpp_draw_kernel(const T *w, int n, const double *bs, int nb, const double *U, double bound,
                int force_exact, int *cand, int *unc) {
    __shared__ double sh[KPP_THREADS / 32 + 1];
    __shared__ double s_prev;
    __shared__ int s_block, s_idx;
    __shared__ double s_pi, s_pim1;
    const int t = blockIdx.x;
    const double u = U[t];
    // S: the sum of the block sums (strided per thread, then the scan's total)
    double part = 0.0;
    for (int j = threadIdx.x; j < nb; j += KPP_THREADS) part += bs[j];
    double S;
    block_exclusive_scan(part, sh, S);
    const double target = u * S;
    // the first block whose cumulative sum reaches u S (chunked scan)
    if (threadIdx.x == 0) {
        s_block = 0x7fffffff;
        s_prev = 0.0;
    }
    __syncthreads();
    double carry = 0.0;
    for (int c0 = 0; c0 < nb; c0 += KPP_THREADS) {
        const int j = c0 + (int)threadIdx.x;
        const double v = j < nb ? bs[j] : 0.0;
        double tot;
        const double ex = carry + block_exclusive_scan(v, sh, tot);
        const double in = ex + v;
        // several blocks can qualify only within rounding of u S (then the
        // draw is not certified); the first one is taken
        if (j < nb && in >= target && ex < target) atomicMin(&s_block, j);
        carry += tot;
        __syncthreads();
        if (j == s_block) s_prev = ex;
        __syncthreads();
        if (s_block != 0x7fffffff) break;
    }
    int b = s_block;
    double prev = s_prev;
    const bool found_block = b != 0x7fffffff;
    if (!found_block) {
        b = nb - 1;
        prev = carry - bs[nb - 1];
    }
    // prefix within block b, in index order
    const size_t base = (size_t)b * KPP_BLOCK + (size_t)threadIdx.x * KPP_PER_THREAD;
    T v[KPP_PER_THREAD];
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < KPP_PER_THREAD; ++j) {
        const size_t i = base + j;
        v[j] = i < (size_t)n ? w[i] : T(0);
        s += (double)v[j];
    }
    double tot;
    const double ex = block_exclusive_scan(s, sh, tot);
    if (threadIdx.x == 0) s_idx = 0x7fffffff;
    __syncthreads();
    double run = prev + ex;
    int mine = 0x7fffffff;
    double pi = 0.0, pim1 = 0.0;
#pragma unroll
    for (int j = 0; j < KPP_PER_THREAD; ++j) {
        const size_t i = base + j;
        const double before = run;
        run += (double)v[j];
        if (mine == 0x7fffffff && i < (size_t)n && run >= target) {
            mine = (int)i;
            pi = run;
            pim1 = before;
        }
    }
    if (mine != 0x7fffffff) atomicMin(&s_idx, mine);
    __syncthreads();
    if (mine != 0x7fffffff && mine == s_idx) {
        s_pi = pi;
        s_pim1 = pim1;
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        int idx = s_idx;
        bool certified = found_block && idx != 0x7fffffff && S > 0.0 && isfinite(S);
        if (idx == 0x7fffffff) idx = n - 1;
        if (certified) {
            const double hi = s_pi / S - u;
            const double lo = u - s_pim1 / S;
            certified = hi > bound && lo > bound;
        }
        cand[t] = idx;
        unc[t] = (certified && !force_exact) ? 0 : 1;
    }
}

// The uncertified draws with the reference's sequential arithmetic: S =
// sum w (double, index order, from 0), p_i = w_i / S, cp_i = cp_{i-1} + p_i,
// cp_{n-1} = 1, the first i with cp_i >= u.  One block; thread 0 carries the
// sequential sums over tiles that all threads stage in shared memory.
// count[0] accumulates the number of redone draws.
template <typename T>
__global__ void __launch_bounds__(KPP_THREADS)
kpp_exact_kernel(const T *w, int n, const double *U, int nt, int *cand, const int *unc,
                 int *count) {
    __shared__ double tile[KPP_EXACT_TILE];
    __shared__ double s_sum;
    __shared__ int s_any;
    if (threadIdx.x == 0) {
        int a = 0;
        for (int t = 0; t < nt; ++t) a += unc[t] ? 1 : 0;
        s_any = a;
        if (a) atomicAdd(count, a);
    }
    __syncthreads();
    if (!s_any) return;
    // S, sequentially
    double S = 0.0;
    for (int t0 = 0; t0 < n; t0 += KPP_EXACT_TILE) {
        const int m = min(KPP_EXACT_TILE, n - t0);
        for (int j = threadIdx.x; j < m; j += KPP_THREADS) tile[j] = (double)w[t0 + j];
        __syncthreads();
        if (threadIdx.x == 0)
            for (int j = 0; j < m; ++j) S = __dadd_rn(S, tile[j]);
        __syncthreads();
    }
    if (threadIdx.x == 0) s_sum = S;
    __syncthreads();
    S = s_sum;
    for (int t = 0; t < nt; ++t) {
        if (!unc[t]) continue;
        const double u = U[t];
        __shared__ int s_done, s_res;
        if (threadIdx.x == 0) {
            s_done = 0;
            s_res = n - 1;
        }
        __syncthreads();
        double cp = 0.0;
        for (int t0 = 0; t0 < n; t0 += KPP_EXACT_TILE) {
            const int m = min(KPP_EXACT_TILE, n - t0);
            for (int j = threadIdx.x; j < m; j += KPP_THREADS)
                tile[j] = __ddiv_rn((double)w[t0 + j], S);
            __syncthreads();
            if (threadIdx.x == 0) {
                for (int j = 0; j < m; ++j) {
                    cp = __dadd_rn(cp, tile[j]);
                    if (t0 + j == n - 1) cp = 1.0;
                    if (cp >= u) {
                        s_res = t0 + j;
                        s_done = 1;
                        break;
                    }
                }
            }
            __syncthreads();
            if (s_done) break;
        }
        if (threadIdx.x == 0) cand[t] = s_res;
        __syncthreads();
    }
}

// ------------------------------------------------ serial cost sums ------
// The reference's candidate cost (kmeans.cpp:1624-1636) is the serial sum,
// in the working precision T and index order from 0, of m_i = max(0,
// min(w_i, d_i)).  It is reproduced exactly, not approximated: while the
// running sum s stays inside one binade [2^E, 2^(E+1)) every addition
// rounds to the grid g = 2^(E - MANT) (s itself lies on it), so
// fl(s + m_i) = s + RN_g(m_i) and a whole run of additions is one integer
// sum of the independently rounded terms q_i = RN_g(m_i).  A chunk of 4,096
// terms is added that way when no term is a tie (m_i / g exactly half-way,
// where ties-to-even depends on the running sum's last bit) and the sum stays
// below 2^(E+1); otherwise the terms before the first such term are added
// as integers, that term is added serially in T (fl(s + m_p)), and the walk
// goes on after it with the new binade.  One block per candidate; the
// result is the T value the reference computes, stored as a double.
template <typename T> struct FpTraits;
template <> struct FpTraits<float> {
    static constexpr int MANT = 23, EMIN = -126;
    static __device__ __forceinline__ int exponent(float s) {
        return (int)((__float_as_uint(s) >> 23) & 0xFF) - 127;
    }
};
template <> struct FpTraits<double> {
    static constexpr int MANT = 52, EMIN = -1022;
    static __device__ __forceinline__ int exponent(double s) {
        return (int)((__double_as_longlong(s) >> 52) & 0x7FF) - 1023;
    }
};

static constexpr int SC_THREADS = 512;
static constexpr int SC_PER = 8;
static constexpr int SC_CHUNK = SC_THREADS * SC_PER;
static constexpr unsigned long long SC_SAT = 1ull << 62;

__device__ __forceinline__ unsigned long long sat_add(unsigned long long a, unsigned long long b) {
    const unsigned long long r = a + b; // a, b <= 2^62: no wrap
    return r > SC_SAT ? SC_SAT : r;
}

// the reference's works5 element: std::max(0, std::min(w, d))
template <typename T> __device__ __forceinline__ T kpp_term(T wv, T dv) {
    const T mn = (dv < wv) ? dv : wv;
    return (T(0) < mn) ? mn : T(0);
}

template <typename T>
__global__ void __launch_bounds__(SC_THREADS)
kpp_serial_cost_kernel(const T *w, const T *D, int n, double *cost) {
    using F = FpTraits<T>;
    __shared__ unsigned long long s_wsum[SC_THREADS / 32];
    __shared__ int s_wflag[SC_THREADS / 32];
    __shared__ int s_p;
    __shared__ T s_sum;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const T *Dt = D + (size_t)blockIdx.x * n;
    T s = T(0);
    long long pos = 0;
    T m[SC_PER], mn[SC_PER];
    // terms [at + 8 tid, at + 8 tid + 8) of the walk (0 past the end)
    auto load = [&](T (&dst)[SC_PER], long long at) {
#pragma unroll
        for (int e = 0; e < SC_PER; ++e) {
            const long long i = at + (long long)threadIdx.x * SC_PER + e;
            dst[e] = i < n ? kpp_term(w[i], Dt[i]) : T(0);
        }
    };
    load(m, 0);
    while (pos < n && isfinite(s)) {
        load(mn, pos + SC_CHUNK); // the next chunk, in flight while this one is summed
        if (s == T(0)) {
            // 0 + m = m exactly: the first nonzero term starts the sum
            int mine = 0x7fffffff;
#pragma unroll
            for (int e = SC_PER - 1; e >= 0; --e)
                if (m[e] != T(0)) mine = (int)threadIdx.x * SC_PER + e;
            __syncthreads();
            if (threadIdx.x == 0) s_p = 0x7fffffff;
            __syncthreads();
            if (mine != 0x7fffffff) atomicMin(&s_p, mine);
            __syncthreads();
            const int p = s_p;
            if (p == 0x7fffffff) {
                pos += SC_CHUNK;
#pragma unroll
                for (int e = 0; e < SC_PER; ++e) m[e] = mn[e];
                continue;
            }
            if ((int)threadIdx.x == p / SC_PER) {
#pragma unroll
                for (int e = 0; e < SC_PER; ++e)
                    if (e == p % SC_PER) s_sum = m[e];
            }
            __syncthreads();
            s = s_sum;
            pos += p + 1;
            load(m, pos);
            continue;
        }
        // the grid of the current binade, in units of g = 2^-sh
        const int ex = F::exponent(s);
        const bool sub = ex < F::EMIN;
        const int E = sub ? F::EMIN : ex;
        const int sh = F::MANT - E;
        const unsigned long long limit = sub ? (1ull << F::MANT) : (2ull << F::MANT);
        const unsigned long long s_int = (unsigned long long)ldexp((double)s, sh);
        unsigned long long q[SC_PER];
        unsigned long long tsum = 0;
        int tie = 0;
#pragma unroll
        for (int e = 0; e < SC_PER; ++e) {
            const double x = ldexp((double)m[e], sh);
            unsigned long long qe = SC_SAT; // leaves the binade by itself
            if (x < (double)limit) {
                const double fl = floor(x), fr = x - fl;
                qe = (unsigned long long)fl + (fr > 0.5 ? 1ull : 0ull);
                if (fr == 0.5) {
                    tie = 1;
                    qe = SC_SAT; // ties-to-even needs the running sum: serial
                }
            }
            q[e] = qe;
            tsum = sat_add(tsum, qe);
        }
        // block total (saturating) and tie flag
        unsigned long long incl = tsum;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const unsigned long long y = __shfl_up_sync(0xffffffffu, incl, off);
            if (lane >= off) incl = sat_add(incl, y);
        }
        unsigned long long exw = __shfl_up_sync(0xffffffffu, incl, 1);
        if (lane == 0) exw = 0;
        const int wt = __any_sync(0xffffffffu, tie);
        __syncthreads();
        if (lane == 31) {
            s_wsum[warp] = incl;
            s_wflag[warp] = wt;
        }
        __syncthreads();
        unsigned long long Q = 0, before = 0;
        int anytie = 0;
        for (int v = 0; v < SC_THREADS / 32; ++v) {
            if (v == warp) before = Q;
            Q = sat_add(Q, s_wsum[v]);
            anytie |= s_wflag[v];
        }
        if (!anytie && s_int + Q < limit) {
            s = (T)ldexp((double)(s_int + Q), -sh);
            pos += SC_CHUNK;
#pragma unroll
            for (int e = 0; e < SC_PER; ++e) m[e] = mn[e];
            continue;
        }
        // the first term that ties or leaves the binade
        unsigned long long run = sat_add(before, exw);
        int mine = 0x7fffffff;
        unsigned long long run_at = 0;
#pragma unroll
        for (int e = 0; e < SC_PER; ++e) {
            const unsigned long long nxt = sat_add(run, q[e]);
            if (mine == 0x7fffffff && (q[e] == SC_SAT || s_int + nxt >= limit)) {
                mine = (int)threadIdx.x * SC_PER + e;
                run_at = run;
            }
            run = nxt;
        }
        if (threadIdx.x == 0) s_p = 0x7fffffff;
        __syncthreads();
        if (mine != 0x7fffffff) atomicMin(&s_p, mine);
        __syncthreads();
        const int p = s_p;
        if (mine == p) {
            // the terms before p on the grid, then term p serially in T
            T mp = T(0);
#pragma unroll
            for (int e = 0; e < SC_PER; ++e)
                if (e == p % SC_PER) mp = m[e];
            const T sp = (T)ldexp((double)(s_int + run_at), -sh);
            s_sum = add_rn(sp, mp);
        }
        __syncthreads();
        s = s_sum;
        pos += p + 1;
        load(m, pos);
    }
    if (threadIdx.x == 0) cost[blockIdx.x] = (double)s;
}

template <typename T>
cudaError_t launch_kpp_serial_cost(const T *w, const T *D, int n, int nt, double *cost,
                                   cudaStream_t s) {
    kpp_serial_cost_kernel<T><<<nt, SC_THREADS, 0, s>>>(w, D, n, cost);
    return cudaGetLastError();
}

// Choose the candidate (kmeans.cpp:1614-1646): repeats skipped, the first
// finite cost strictly below the best so far; none: index 0.  Every block
// makes the same choice; block 0 records it.  Then w_i = max(0, min(w_i,
// D_best,i)), the chosen row's weight 0, and the block sums of the new w.
template <typename T>
__global__ void __launch_bounds__(KPP_THREADS)
kpp_select_update_kernel(T *w, const T *D, int n, const double *cost, const int *cand, int nt,
                         int *chosen, int c, double *bs) {
    __shared__ double sh[KPP_THREADS / 32 + 1];
    __shared__ int s_best_t, s_best;
    if (threadIdx.x == 0) {
        int bt = -1, best = 0;
        double bc = __longlong_as_double(0x7ff0000000000000ULL);
        for (int t = 0; t < nt; ++t) {
            bool rep = false;
            for (int q = 0; q < t; ++q) rep = rep || cand[q] == cand[t];
            if (rep) continue;
            const double ct = cost[t];
            if (isfinite(ct) && ct < bc) {
                bc = ct;
                bt = t;
                best = cand[t];
            }
        }
        s_best_t = bt;
        s_best = best;
        if (blockIdx.x == 0) chosen[c] = best;
    }
    __syncthreads();
    const int bt = s_best_t, best = s_best;
    const T *Dc = bt >= 0 ? D + (size_t)bt * n : nullptr;
    const size_t base = (size_t)blockIdx.x * KPP_BLOCK + (size_t)threadIdx.x * KPP_PER_THREAD;
    double s = 0.0;
#pragma unroll
    for (int j = 0; j < KPP_PER_THREAD; ++j) {
        const size_t i = base + j;
        if (i < (size_t)n) {
            T v = w[i];
            if (Dc) {
                const T dv = Dc[i];
                T m = dv < v ? dv : v;
                if (!(m > T(0))) m = T(0);
                v = m;
            }
            if ((int)i == best) v = T(0);
            w[i] = v;
            s += (double)v;
        }
    }
    double tot;
    block_exclusive_scan(s, sh, tot);
    if (threadIdx.x == 0) bs[blockIdx.x] = tot;
}

int kpp_num_blocks(int n) { return (n + KPP_BLOCK - 1) / KPP_BLOCK; }

double kpp_draw_bound(int n) {
    const double nb = (double)kpp_num_blocks(n);
    return 1.2 * (2.0 * n + 2.0 * nb + 4200.0) * 0x1p-53;
}

template <typename T>
cudaError_t launch_kpp_clamp(T *w, int n, int first, double *bs, int *flag, cudaStream_t s) {
    kpp_clamp_kernel<T><<<kpp_num_blocks(n), KPP_THREADS, 0, s>>>(w, n, first, bs, flag);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_kpp_draw(const T *w, int n, const double *bs, const double *U, int nt,
                            int force_exact, int *cand, int *unc, int *exact_count,
                            cudaStream_t s) {
    const int nb = kpp_num_blocks(n);
    kpp_draw_kernel<T><<<nt, KPP_THREADS, 0, s>>>(w, n, bs, nb, U, kpp_draw_bound(n), force_exact,
                                                  cand, unc);
    kpp_exact_kernel<T><<<1, KPP_THREADS, 0, s>>>(w, n, U, nt, cand, unc, exact_count);
    return cudaGetLastError();
}

template <typename T>
cudaError_t launch_kpp_select_update(T *w, const T *D, int n, const double *cost,
                                     const int *cand, int nt, int *chosen, int c, double *bs,
                                     cudaStream_t s) {
    kpp_select_update_kernel<T><<<kpp_num_blocks(n), KPP_THREADS, 0, s>>>(w, D, n, cost, cand, nt,
                                                                          chosen, c, bs);
    return cudaGetLastError();
}

#define B200_KPP_INST(T)                                                                       \
    template cudaError_t launch_kpp_clamp<T>(T *, int, int, double *, int *, cudaStream_t);     \
    template cudaError_t launch_kpp_draw<T>(const T *, int, const double *, const double *,     \
                                            int, int, int *, int *, int *, cudaStream_t);       \
    template cudaError_t launch_kpp_select_update<T>(T *, const T *, int, const double *,       \
                                                     const int *, int, int *, int, double *,    \
                                                     cudaStream_t);                             \
    template cudaError_t launch_kpp_serial_cost<T>(const T *, const T *, int, int, double *,    \
                                                   cudaStream_t);
B200_KPP_INST(float)
B200_KPP_INST(double)

} // namespace b200
