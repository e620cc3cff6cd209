// Fixed-point centroid sums shared by the k-means update kernels: exact
// 64-bit integer sums of q = round(x * 2^s_f), so that any order of the
// additions gives the same sums.
#pragma once
#include <cuda_runtime.h>

namespace b200 {

// acc += q (64-bit, in shared memory) as two 32-bit atomics: the low word's
// atomic returns its old value, from which this addition's carry into the
// high word is exact whatever the interleaving of the other threads' adds.
__device__ __forceinline__ void fx_add(unsigned long long *acc, long long q) {
    unsigned *w = reinterpret_cast<unsigned *>(acc);
    const unsigned l = (unsigned)q, h = (unsigned)((unsigned long long)q >> 32);
    const unsigned o = atomicAdd(w, l);
    atomicAdd(w + 1, h + (o + l < o ? 1u : 0u));
}

// Add a run's register sums into the shared accumulators (two 32-bit
// atomics with an exact carry; other warps may flush into the same cluster).
// Run sums of q = round(x * 2^s) split as q = hi * 2^22 + lo, both parts
// accumulated as raw float bits of hi + 1.5 * 2^23 and lo + 1.5 * 2^23 in
// wrapping 32-bit registers (four FMA-pipe operations and two integer adds
// per value):
//   t  = fma(x, 2^(s-22), 1.5 * 2^23)   = 1.5 * 2^23 + round(x 2^(s-22))
//   nh = fma(t, -2^22, 1.5 * 2^45)      = -hi * 2^22               (exact)
//   yl = fma(x, 2^s, nh)                = x 2^s - hi * 2^22        (exact, |yl| <= 2^21)
//   lo = yl + 1.5 * 2^23                 (rounds yl to an integer)
// With |x 2^s| < 2^44 and at most 511 rows per run, the unbiased sums fit in
// int32 (|sum hi| < 2^31, |sum lo| < 2^30).
struct FxRun {
    unsigned h0 = 0, l0 = 0, h1 = 0, l1 = 0;
    unsigned n = 0;
};
__device__ __forceinline__ void fx_acc(float x, float s22, float s, unsigned &h, unsigned &l) {
    const float t = __fmaf_rn(x, s22, 12582912.f);
    const float nh = __fmaf_rn(t, -4194304.f, 52776558133248.f);
    const float yl = __fmaf_rn(x, s, nh);
    h += __float_as_uint(t);
    l += __float_as_uint(__fadd_rn(yl, 12582912.f));
}
__device__ __forceinline__ long long fx_run_sum(unsigned h, unsigned l, unsigned n) {
    const int hs = (int)(h - n * 0x4B400000u), ls = (int)(l - n * 0x4B400000u);
    return ((long long)hs << 22) + ls;
}
__device__ __forceinline__ void fx_flush(unsigned long long *acc, int d, int j, int f,
                                         FxRun &run, bool two) {
    if (run.n) {
        if (f < d) fx_add(acc + (size_t)j * d + f, fx_run_sum(run.h0, run.l0, run.n));
        if (two && f + 1 < d) fx_add(acc + (size_t)j * d + f + 1, fx_run_sum(run.h1, run.l1, run.n));
    }
    run = FxRun();
}

// The same run sums for VW consecutive features of one lane.
template <int VW> struct FxRunV {
    unsigned h[VW], l[VW];
    unsigned n;
    __device__ __forceinline__ void reset() {
#pragma unroll
        for (int v = 0; v < VW; ++v) h[v] = l[v] = 0u;
        n = 0u;
    }
};
template <int VW>
__device__ __forceinline__ void fx_flush_v(unsigned long long *acc, int d, int j, int f,
                                           FxRunV<VW> &run) {
    if (run.n) {
#pragma unroll
        for (int v = 0; v < VW; ++v)
            if (f + v < d)
                fx_add(acc + (size_t)j * d + f + v, fx_run_sum(run.h[v], run.l[v], run.n));
    }
    run.reset();
}

} // namespace b200
