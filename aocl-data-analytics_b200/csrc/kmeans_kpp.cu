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
// cp_{n-1} = 1, the first i with !(cp_i < u) (std::lower_bound).  One block; thread 0 carries the
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
                    // std::lower_bound's test !(cp < u): with all weights
                    // zero (S = 0) every cp is NaN and the first index wins
                    if (!(cp < u)) {
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
// min(w_i, d_i)).  It is reproduced exactly, not approximated.  While the
// running sum s stays inside one binade [2^E, 2^(E+1)) every addition rounds
// to the grid g = 2^(E - MANT) (s itself lies on it), so fl(s + m_i) =
// s + RN_g(m_i) and a run of additions is one integer sum of the
// independently rounded terms q_i = RN_g(m_i) -- unless a term is a tie
// (m_i / g exactly half-way: ties-to-even then depends on the running sum's
// last bit) or the sum leaves the binade; such a term is added serially in T.
// Three passes per candidate set:
//   * kpp_dist_csum_kernel: the candidates' distances and, per 256-row
//     chunk, the fp64 sum of its terms;
//   * kpp_chunk_q_kernel: the fp64 prefix of the chunk sums predicts the
//     binade E_j of the serial sum at each chunk; the chunk's integer total
//     Q_j on that binade's grid (flagged when a term ties);
//   * kpp_walk_kernel, one block per candidate: walks the chunk records; a
//     chunk is added as s += Q_j g when the running sum is in binade E_j, the
//     chunk has no tie and the sum stays in the binade -- else the chunk is
//     summed exactly term by term (integer runs, serial steps at the first
//     tie or binade crossing).  The prediction only chooses the fast path;
//     every fast step is checked, so the result is the reference's T value
//     whatever the fp64 prefix says.
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

static constexpr int CK = 256;           // terms per chunk
static constexpr int WALK_THREADS = 256;
static constexpr int WALK_PER = 4; // chunk records per thread per pass
static constexpr int NO_BINADE = -100000; // chunk record: sum it exactly
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

// The grid of the binade of s > 0: raw exponent (subnormals: EMIN - 1),
// sh = -log2(g), the binade's end in grid units, s in grid units.
template <typename T> struct Binade {
    int ex, sh;
    unsigned long long limit, s_int;
    __device__ __forceinline__ void set(T s) {
        using F = FpTraits<T>;
        ex = F::exponent(s);
        const bool sub = ex < F::EMIN;
        sh = F::MANT - (sub ? F::EMIN : ex);
        limit = sub ? (1ull << F::MANT) : (2ull << F::MANT);
        s_int = (unsigned long long)ldexp((double)s, sh);
    }
    // q = RN_g(m) for a non-tie; SC_SAT for a tie or a term that leaves the
    // binade by itself.  t = 2 m / g is exact (power-of-two scaling in
    // double, in two factors so that neither overflows); RN(t / 2) of a
    // non-tie = (floor(t) + 1) / 2; a tie is t an odd integer.
    __device__ __forceinline__ unsigned long long q(T m) const {
        const int e2 = sh + 1, ea = min(e2, 1000), eb = e2 - ea;
        const double sa = __longlong_as_double((long long)(ea + 1023) << 52);
        const double sb = __longlong_as_double((long long)(eb + 1023) << 52);
        const double tt = ((double)m * sa) * sb;
        if (!(tt < 2.0 * (double)limit)) return SC_SAT;
        const unsigned long long ti = __double2ull_rz(tt);
        if ((ti & 1ull) && tt == __ull2double_rn(ti)) return SC_SAT;
        return (ti + 1ull) >> 1;
    }
    // q for a term staying inside the binade by itself: RN_g(m) for a
    // non-tie; for a tie (m / g = k + 1/2) k, with *tie set (its rounding
    // depends on the running sum's parity); SC_SAT for a term that leaves
    // the binade by itself
    __device__ __forceinline__ unsigned long long qt(T m, bool &tie) const {
        const int e2 = sh + 1, ea = min(e2, 1000), eb = e2 - ea;
        const double sa = __longlong_as_double((long long)(ea + 1023) << 52);
        const double sb = __longlong_as_double((long long)(eb + 1023) << 52);
        const double tt = ((double)m * sa) * sb;
        tie = false;
        if (!(tt < 2.0 * (double)limit)) return SC_SAT;
        const unsigned long long ti = __double2ull_rz(tt);
        if ((ti & 1ull) && tt == __ull2double_rn(ti)) {
            tie = true;
            return ti >> 1;
        }
        return (ti + 1ull) >> 1;
    }
    // m stays inside the binade by itself (so SC_SAT from q() means a tie)
    __device__ __forceinline__ bool q_in_range(T m) const {
        const int e2 = sh + 1, ea = min(e2, 1000), eb = e2 - ea;
        const double sa = __longlong_as_double((long long)(ea + 1023) << 52);
        const double sb = __longlong_as_double((long long)(eb + 1023) << 52);
        return ((double)m * sa) * sb < 2.0 * (double)limit;
    }
    __device__ __forceinline__ T value(unsigned long long units) const {
        return (T)ldexp((double)units, -sh);
    }
};

// A run of additions on one grid as a function of the running sum's parity
// (its last bit in grid units) at the run's start: q0 / q1 the run's total
// for start parity 0 / 1, o bit p the parity at its end for start parity p.
// A non-tie term q: (q, q, parity flips with q's last bit).  A tie term
// m / g = k + 1/2 rounds to the even neighbour: k + ((R + k) & 1) for a
// running sum R, after which the sum is even.  Runs compose associatively,
// so a scan over them gives the running sum before every term.
struct Pf {
    unsigned long long q0, q1;
    int o;
};
__device__ __forceinline__ Pf pf_id() { return Pf{0ull, 0ull, 2}; }
__device__ __forceinline__ Pf pf_term(unsigned long long q, bool tie) {
    if (!tie) {
        const int b = (int)(q & 1ull);
        return Pf{q, q, b | ((1 ^ b) << 1)};
    }
    return Pf{q + (q & 1ull), q + ((q + 1ull) & 1ull), 0};
}
__device__ __forceinline__ unsigned long long pf_q(const Pf &f, int p) { return p ? f.q1 : f.q0; }
__device__ __forceinline__ int pf_o(const Pf &f, int p) { return (f.o >> p) & 1; }
// a, then b
__device__ __forceinline__ Pf pf_cat(const Pf &a, const Pf &b) {
    const int a0 = a.o & 1, a1 = (a.o >> 1) & 1;
    return Pf{sat_add(a.q0, pf_q(b, a0)), sat_add(a.q1, pf_q(b, a1)),
              pf_o(b, a0) | (pf_o(b, a1) << 1)};
}
__device__ __forceinline__ Pf pf_shfl_up(const Pf &v, int off) {
    return Pf{__shfl_up_sync(0xffffffffu, v.q0, off), __shfl_up_sync(0xffffffffu, v.q1, off),
              __shfl_up_sync(0xffffffffu, v.o, off)};
}

// Scan of one run per thread over a block of NT threads in thread order:
// the composition of the runs before this thread's (`excl`) and of all
// (`total`).  shm: 2 * (NT / 32) + 1 entries.
template <int NT>
__device__ void block_scan_pf(const Pf &v, Pf *shm, Pf &excl, Pf &total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    constexpr int NW = NT / 32;
    Pf x = v;
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const Pf y = pf_shfl_up(x, off);
        if (lane >= off) x = pf_cat(y, x);
    }
    Pf xe = pf_shfl_up(x, 1);
    if (lane == 0) xe = pf_id();
    __syncthreads();
    if (lane == 31) shm[warp] = x;
    __syncthreads();
    if (warp == 0) {
        Pf y = lane < NW ? shm[lane] : pf_id();
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const Pf z = pf_shfl_up(y, off);
            if (lane >= off) y = pf_cat(z, y);
        }
        Pf ye = pf_shfl_up(y, 1);
        if (lane == 0) ye = pf_id();
        if (lane < NW) shm[NW + lane] = ye;
        if (lane == NW - 1) shm[2 * NW] = y;
    }
    __syncthreads();
    total = shm[2 * NW];
    excl = pf_cat(shm[NW + warp], xe);
}

// Distances of a 256-row chunk to the candidates (one thread per row), with
// the chunk's fp64 sum of the cost terms per candidate.  A thread holds 64
// (fp32) or 32 (fp64) features of its row in registers at a time -- 16
// independent 16-byte loads in flight -- and runs eight candidates' fma
// chains over them (features in order), the candidates' values broadcast
// from shared memory (SMEM) or read through L1.
template <typename T> struct SegTraits;
template <> struct SegTraits<float> {
    static constexpr int SEG = 64; // features per register segment
    using V = float4;
    static constexpr int W = 4;
    static __device__ __forceinline__ void split(const float4 &v, float (&o)[4]) {
        o[0] = v.x; o[1] = v.y; o[2] = v.z; o[3] = v.w;
    }
};
template <> struct SegTraits<double> {
    static constexpr int SEG = 32;
    using V = double2;
    static constexpr int W = 2;
    static __device__ __forceinline__ void split(const double2 &v, double (&o)[2]) {
        o[0] = v.x; o[1] = v.y;
    }
};

template <typename T, bool SMEM>
__global__ void __launch_bounds__(CK, 2)
kpp_dist_csum_kernel(const T *X, int ld, int n, int d, const T *xnorm, const int *cand, int t,
                     const T *w, T *D, double *csum, int nchunks, const T *xinv, int cosine) {
    using S = SegTraits<T>;
    constexpr int NV = S::SEG / S::W;
    extern __shared__ __align__(16) unsigned char sm[];
    __shared__ double red[CK / 32][8];
    T *cs = reinterpret_cast<T *>(sm); // [t][dp] when SMEM
    const int dp = (d + S::W - 1) / S::W * S::W;
    if (SMEM) {
        for (int e = threadIdx.x; e < t * dp; e += CK) {
            const int c = e / dp, f = e % dp;
            cs[e] = f < d ? X[(size_t)cand[c] * ld + f] : T(0);
        }
        __syncthreads();
    }
    const int i = blockIdx.x * CK + threadIdx.x;
    const bool valid = i < n;
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const T *x = X + (size_t)(valid ? i : 0) * ld;
    const T xn = valid ? xnorm[i] : T(0);
    const T wi = valid ? w[i] : T(0);
    for (int c0 = 0; c0 < t; c0 += 8) {
        T s[8];
#pragma unroll
        for (int g = 0; g < 8; ++g) s[g] = T(0);
        int cg[8];
#pragma unroll
        for (int g = 0; g < 8; ++g) cg[g] = min(c0 + g, t - 1);
        if (valid) {
            for (int f0 = 0; f0 < d; f0 += S::SEG) {
                typename S::V xv[NV];
#pragma unroll
                for (int v = 0; v < NV; ++v)
                    if (f0 + v * S::W < d) // rows are padded to 16 bytes
                        xv[v] = *reinterpret_cast<const typename S::V *>(x + f0 + v * S::W);
#pragma unroll
                for (int v = 0; v < NV; ++v) {
                    const int fb = f0 + v * S::W;
                    if (fb >= d) break;
                    T xe[S::W];
                    S::split(xv[v], xe);
#pragma unroll
                    for (int g = 0; g < 8; ++g) {
                        T ce[S::W];
                        if (SMEM) {
                            S::split(*reinterpret_cast<const typename S::V *>(cs + (size_t)cg[g] * dp + fb), ce);
                        } else {
                            const T *yr = X + (size_t)cand[cg[g]] * ld + fb;
                            S::split(*reinterpret_cast<const typename S::V *>(yr), ce);
                        }
#pragma unroll
                        for (int u = 0; u < S::W; ++u)
                            if (fb + u < d) s[g] = fma_rn(xe[u], ce[u], s[g]);
                    }
                }
            }
        }
        double part[8];
#pragma unroll
        for (int g = 0; g < 8; ++g) {
            part[g] = 0.0;
            if (valid && c0 + g < t) {
                const int cc = cand[c0 + g];
                const T dv = cosine ? cos_dist_kpp(s[g], xinv, i, cc)
                                    : fma_rn(T(-2), s[g], add_rn(xn, xnorm[cc]));
                D[(size_t)(c0 + g) * n + i] = dv;
                part[g] = (double)kpp_term(wi, dv);
            }
#pragma unroll
            for (int off = 16; off > 0; off >>= 1) part[g] += __shfl_xor_sync(0xffffffffu, part[g], off);
        }
        __syncthreads();
        if (lane == 0)
#pragma unroll
            for (int g = 0; g < 8; ++g) red[warp][g] = part[g];
        __syncthreads();
        if (threadIdx.x < 8 && c0 + (int)threadIdx.x < t) {
            double a = 0.0;
            for (int v = 0; v < CK / 32; ++v) a += red[v][threadIdx.x];
            csum[(size_t)(c0 + threadIdx.x) * nchunks + blockIdx.x] = a;
        }
    }
}

// Exclusive fp64 prefix of the chunk sums of candidate blockIdx.x.
__global__ void __launch_bounds__(1024) kpp_chunk_prefix_kernel(const double *csum, int nchunks,
                                                                double *P) {
    __shared__ double shd[33];
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const double *cs = csum + (size_t)blockIdx.x * nchunks;
    double *Pt = P + (size_t)blockIdx.x * nchunks;
    double carry = 0.0;
    for (int c0 = 0; c0 < nchunks; c0 += 1024) {
        const int j = c0 + threadIdx.x;
        const double v = j < nchunks ? cs[j] : 0.0;
        double x = v;
#pragma unroll
        for (int off = 1; off < 32; off <<= 1) {
            const double y = __shfl_up_sync(0xffffffffu, x, off);
            if (lane >= off) x += y;
        }
        __syncthreads();
        if (lane == 31) shd[warp] = x;
        __syncthreads();
        if (threadIdx.x == 0) {
            double a = 0.0;
            for (int q = 0; q < 32; ++q) {
                const double tq = shd[q];
                shd[q] = a;
                a += tq;
            }
            shd[32] = a;
        }
        __syncthreads();
        if (j < nchunks) Pt[j] = carry + shd[warp] + (x - v);
        carry += shd[32];
    }
}

// Chunk records of candidate blockIdx.y, one warp per chunk: the binade the
// fp64 prefix predicts for the serial sum at the chunk (raw exponent of
// (T)P_j, or NO_BINADE when P_j is 0 or not finite) and the chunk's run on
// that binade's grid as a parity function (saturating totals).
template <typename T>
__global__ void __launch_bounds__(256)
kpp_chunk_q_kernel(const T *w, const T *D, int n, int nchunks, const double *P,
                   unsigned long long *Q0, unsigned long long *Q1, int *Or, int *Er) {
    const int t = blockIdx.y;
    const int j = blockIdx.x * 8 + (threadIdx.x >> 5);
    const int lane = threadIdx.x & 31;
    if (j >= nchunks) return;
    const size_t r = (size_t)t * nchunks + j;
    const double Pj = P[r];
    const T Ts = (T)Pj;
    if (!(Pj > 0.0) || !isfinite(Ts) || Ts == T(0)) {
        if (lane == 0) {
            Q0[r] = Q1[r] = 0;
            Or[r] = 2;
            Er[r] = NO_BINADE;
        }
        return;
    }
    Binade<T> b;
    b.set(Ts);
    const T *Dt = D + (size_t)t * n;
    // each lane composes 8 consecutive terms, then the lanes' runs in lane
    // order (a tree over neighbouring blocks of lanes)
    Pf acc = pf_id();
#pragma unroll
    for (int u = 0; u < CK / 32; ++u) {
        const int i = j * CK + lane * (CK / 32) + u;
        if (i < n) {
            bool tie;
            const unsigned long long q = b.qt(kpp_term(w[i], Dt[i]), tie);
            acc = pf_cat(acc, pf_term(q, tie));
        }
    }
#pragma unroll
    for (int off = 1; off < 32; off <<= 1) {
        const Pf y = Pf{__shfl_down_sync(0xffffffffu, acc.q0, off),
                        __shfl_down_sync(0xffffffffu, acc.q1, off),
                        __shfl_down_sync(0xffffffffu, acc.o, off)};
        if ((lane & (2 * off - 1)) == 0) acc = pf_cat(acc, y);
    }
    if (lane == 0) {
        Q0[r] = acc.q0;
        Q1[r] = acc.q1;
        Or[r] = acc.o;
        Er[r] = b.ex;
    }
}

// The serial sum of candidate blockIdx.x over the chunk records (see above).
template <typename T>
__global__ void __launch_bounds__(WALK_THREADS)
kpp_walk_kernel(const T *w, const T *D, int n, int nchunks, const unsigned long long *Q0,
                const unsigned long long *Q1, const int *Or, const int *Er, double *cost) {
    __shared__ Pf shm[2 * (WALK_THREADS / 32) + 1];
    __shared__ int s_f;
    __shared__ T s_val;
    const int t = blockIdx.x;
    const T *Dt = D + (size_t)t * n;
    const size_t ro = (size_t)t * nchunks;
    T s = T(0);
    int j = 0;
    while (j < nchunks && isfinite(s)) {
        Binade<T> b;
        b.ex = NO_BINADE - 1;
        b.sh = 0;
        b.limit = 0;
        b.s_int = 0;
        if (s != T(0)) b.set(s);
        const int p0 = (int)(b.s_int & 1ull);
        // WALK_PER consecutive records per thread
        const int r0 = j + (int)threadIdx.x * WALK_PER;
        Pf rv[WALK_PER];
        bool okv[WALK_PER];
        Pf loc = pf_id();
#pragma unroll
        for (int u = 0; u < WALK_PER; ++u) {
            const int r = r0 + u;
            const bool valid = r < nchunks;
            rv[u] = valid ? Pf{Q0[ro + r], Q1[ro + r], Or[ro + r]} : pf_id();
            okv[u] = !valid || Er[ro + r] == b.ex;
            loc = pf_cat(loc, rv[u]);
        }
        Pf excl, total;
        block_scan_pf<WALK_THREADS>(loc, shm, excl, total);
        int mine = 0x7fffffff;
        unsigned long long R = b.s_int + pf_q(excl, p0), R_at = 0; // running sum, grid units
        int par = pf_o(excl, p0);
#pragma unroll
        for (int u = 0; u < WALK_PER; ++u) {
            const unsigned long long q = pf_q(rv[u], par);
            if (mine == 0x7fffffff && r0 + u < nchunks && (!okv[u] || R + q >= b.limit)) {
                mine = (int)threadIdx.x * WALK_PER + u;
                R_at = R;
            }
            R = sat_add(R, q);
            par = pf_o(rv[u], par);
        }
        if (threadIdx.x == 0) s_f = 0x7fffffff;
        __syncthreads();
        if (mine != 0x7fffffff) atomicMin(&s_f, mine);
        __syncthreads();
        const int f = s_f;
        if (f == 0x7fffffff) {
            s = b.value(b.s_int + pf_q(total, p0));
            j += WALK_THREADS * WALK_PER;
            continue;
        }
        // the records before f on the grid
        if (mine == f) s_val = (f == 0) ? s : b.value(R_at);
        __syncthreads();
        s = s_val;
        __syncthreads();
        // chunk j + f, term by term: ties by their parity rule, a serial
        // step only where the sum leaves the binade (or a term does by itself)
        const int c = j + f;
        int pos = c * CK;
        const int end = min(n, pos + CK);
        const int i = pos + (int)threadIdx.x;
        const T mi = ((int)threadIdx.x < CK && i < end) ? kpp_term(w[i], Dt[i]) : T(0);
        while (pos < end && isfinite(s)) {
            const bool in = (int)threadIdx.x < CK && i >= pos && i < end;
            const T m = in ? mi : T(0);
            if (s == T(0)) {
                // 0 + m = m exactly: the first nonzero term starts the sum
                if (threadIdx.x == 0) s_f = 0x7fffffff;
                __syncthreads();
                if (in && m != T(0)) atomicMin(&s_f, i);
                __syncthreads();
                const int p = s_f;
                if (p == 0x7fffffff) {
                    pos = end;
                    break;
                }
                if (i == p) s_val = m;
                __syncthreads();
                s = s_val;
                pos = p + 1;
                __syncthreads();
                continue;
            }
            Binade<T> bb;
            bb.set(s);
            const int pp = (int)(bb.s_int & 1ull);
            bool tie = false;
            const unsigned long long qv = in ? bb.qt(m, tie) : 0ull;
            const Pf e = in ? pf_term(qv, tie) : pf_id();
            Pf ex, tot;
            block_scan_pf<WALK_THREADS>(e, shm, ex, tot);
            const unsigned long long Rb = bb.s_int + pf_q(ex, pp);
            const bool bad = in && (qv == SC_SAT || Rb + pf_q(e, pf_o(ex, pp)) >= bb.limit);
            if (threadIdx.x == 0) s_f = 0x7fffffff;
            __syncthreads();
            if (bad) atomicMin(&s_f, i);
            __syncthreads();
            const int p = s_f;
            if (p == 0x7fffffff) {
                s = bb.value(bb.s_int + pf_q(tot, pp));
                pos = end;
                break;
            }
            // the terms before p on the grid, then term p serially in T
            if (i == p) s_val = add_rn(bb.value(Rb), m);
            __syncthreads();
            s = s_val;
            pos = p + 1;
            __syncthreads();
        }
        j = c + 1;
    }
    if (threadIdx.x == 0) cost[t] = (double)s;
}

int kpp_num_chunks(int n) { return (n + CK - 1) / CK; }

template <typename T>
cudaError_t launch_kpp_dist_cost(const T *X, int ldx, int n, int d, const T *xnorm,
                                 const int *cand, int t, const T *w, T *D, double *cost,
                                 void *work, cudaStream_t s, const T *xinv, int cosine) {
    if (ldx % 4 != 0 || (reinterpret_cast<uintptr_t>(X) & 15) != 0) return cudaErrorInvalidValue;
    const int nch = kpp_num_chunks(n);
    double *csum = static_cast<double *>(work);
    double *P = csum + (size_t)t * nch;
    unsigned long long *Q0 = reinterpret_cast<unsigned long long *>(P + (size_t)t * nch);
    unsigned long long *Q1 = Q0 + (size_t)t * nch;
    int *Or = reinterpret_cast<int *>(Q1 + (size_t)t * nch);
    int *Er = Or + (size_t)t * nch;
    // candidates' rows padded to 16 bytes, in shared memory when they fit
    const int W = 16 / (int)sizeof(T);
    const size_t want = (size_t)t * ((d + W - 1) / W * W) * sizeof(T);
    if (want <= 96 * 1024) {
        cudaError_t e = ensure_smem_limit(
            reinterpret_cast<const void *>(kpp_dist_csum_kernel<T, true>), want);
        if (e != cudaSuccess) return e;
        kpp_dist_csum_kernel<T, true><<<nch, CK, want, s>>>(X, ldx, n, d, xnorm, cand, t, w, D,
                                                            csum, nch, xinv, cosine);
    } else {
        kpp_dist_csum_kernel<T, false><<<nch, CK, 0, s>>>(X, ldx, n, d, xnorm, cand, t, w, D, csum,
                                                          nch, xinv, cosine);
    }
    kpp_chunk_prefix_kernel<<<t, 1024, 0, s>>>(csum, nch, P);
    kpp_chunk_q_kernel<T><<<dim3((nch + 7) / 8, t), 256, 0, s>>>(w, D, n, nch, P, Q0, Q1, Or,
                                                                  Er);
    kpp_walk_kernel<T><<<t, WALK_THREADS, 0, s>>>(w, D, n, nch, Q0, Q1, Or, Er, cost);
    return cudaGetLastError();
}

size_t kpp_cost_work_bytes(int n, int t) {
    return (size_t)kpp_num_chunks(n) * t * (8 + 8 + 8 + 8 + 4 + 4) + 256;
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
    template cudaError_t launch_kpp_dist_cost<T>(const T *, int, int, int, const T *,           \
                                                 const int *, int, const T *, T *, double *,     \
                                                 void *, cudaStream_t, const T *, int);
B200_KPP_INST(float)
B200_KPP_INST(double)

} // namespace b200
