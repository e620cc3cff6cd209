// Batched k-means (Lloyd): many independent fp32 data sets of different n, d
// and k fitted together.  Every Lloyd iteration of every instance is one pass
// of four launches over (instance, tile) work tables -- centre norms, the
// assignment, the fixed-point update and the finalisation with the
// instance's own convergence test -- so the whole fit is captured once in a
// CUDA graph and replayed without host round trips.  Converged instances
// skip their work items.
//
// Each instance follows exactly the single-data-set path with precision mode
// "plain", n_init = 1 and supplied initial centres (kmeans.cpp:996-1058 as
// restated in kmeans.cpp here): the same assignment formula and order, the
// same order-independent fixed-point centroid sums and scales, the same
// shift reduction and convergence test, the same final relabelling; so its
// labels, centres and iteration count equal that path's.
#include "b200_common.cuh"
#include "b200_kernels.hpp"
#include "device_alloc.hpp"
#include "kmeans_fx.cuh"
#include "simt_engine.cuh"
#include "../../include/aoclda_b200_ext.h"
#include <algorithm>
#include <cmath>
#include <cstring>
#include <vector>

namespace b200 {

namespace {

constexpr int KB_BATCH = 8192;  // rows bucketed per update item
constexpr int KB_UPD_THREADS = 512;

struct KbInst {
    int n, d, ld, k, L;
    long long xo, co, lo, no, ao, so; // offsets into the packed buffers
    // state, updated on the device
    int it, done, conv, n_iter, relabel, changed;
    int fc, fl; // buffers of the final centres and of the final labels
    double normc2, shift2;
};
struct KbItem {
    int inst, r0;
};

// Per-feature absolute maxima -> fixed-point scales (the single-data-set rule:
// s_f = min(62 - L, 44) - E_f with max|x_f| < 2^E_f, clamped to [-126, 127]).
__global__ void kb_scales(const float *X, KbInst *inst, float *scale, double *inv, int *bad) {
    KbInst &I = inst[blockIdx.x];
    extern __shared__ unsigned cm[];
    for (int f = threadIdx.x; f < I.d; f += blockDim.x) cm[f] = 0u;
    __syncthreads();
    const float *x = X + I.xo;
    for (long long e = threadIdx.x; e < (long long)I.n * I.d; e += blockDim.x) {
        const int r = (int)(e / I.d), f = (int)(e - (long long)r * I.d);
        const unsigned b = __float_as_uint(x[(size_t)r * I.ld + f]) & 0x7fffffffu;
        if (b >= 0x7f800000u) atomicOr(bad, 1);
        else atomicMax(&cm[f], b);
    }
    __syncthreads();
    for (int f = threadIdx.x; f < I.d; f += blockDim.x) {
        const unsigned m = cm[f];
        int E = 0;
        if (m != 0u) frexpf(__uint_as_float(m), &E); // m < 2^E
        int sf = min(62 - I.L, 44) - E;
        sf = max(-126, min(127, sf));
        scale[I.so + f] = __uint_as_float((unsigned)(sf + 127) << 23);
        inv[I.so + f] = ldexp(1.0, -sf);
    }
}

// Iteration start: |c_j|^2 of the previous centres (one fma chain per centre,
// as the single path) and cleared accumulators.
__global__ void kb_begin(KbInst *inst, const float *Cb0, const float *Cb1, float *cnorm,
                         unsigned long long *acc, int *cnt) {
    KbInst &I = inst[blockIdx.x];
    if (I.done) return;
    const float *C = ((I.it & 1) ? Cb1 : Cb0) + I.co;
    for (int j = threadIdx.x; j < I.k; j += blockDim.x) {
        const float *c = C + (size_t)j * I.ld;
        float s = 0.f;
        for (int f = 0; f < I.d; ++f) s = __fmaf_rn(c[f], c[f], s);
        cnorm[I.no + j] = s;
        cnt[I.no + j] = 0;
    }
    for (int e = threadIdx.x; e < I.k * I.d; e += blockDim.x) acc[I.ao + e] = 0ull;
    if (threadIdx.x == 0) I.changed = 0;
}

// |c_j|^2 of the final centres of the instances flagged for relabelling.
__global__ void kb_final_norms(KbInst *inst, const float *Cb0, const float *Cb1, float *cnorm) {
    KbInst &I = inst[blockIdx.x];
    if (!I.relabel) return;
    const float *C = (I.fc ? Cb1 : Cb0) + I.co;
    for (int j = threadIdx.x; j < I.k; j += blockDim.x) {
        const float *c = C + (size_t)j * I.ld;
        float s = 0.f;
        for (int f = 0; f < I.d; ++f) s = __fmaf_rn(c[f], c[f], s);
        cnorm[I.no + j] = s;
    }
}

// Assignment of a 64-row tile of one instance (the single path's SIMT tile:
// x.c as one fma chain over the features, v = fma(-2, x.c, |c|^2), ties to
// the lower index).  relabel_pass: only instances flagged for the final
// relabelling, against their final centres, into their final label buffer.
__global__ void __launch_bounds__(256)
kb_assign(const float *X, KbInst *inst, const KbItem *items, const float *Cb0, const float *Cb1,
          const float *cnorm, int *Lb0, int *Lb1, int relabel_pass) {
    using Cf = SimtCfg<float>;
    constexpr int TM = Cf::TM, TN = Cf::TN, BK = Cf::BK, BM = 16 * TM, BN = 16 * TN;
    __shared__ __align__(16) Stage<float, BM, BN, BK> st[2];
    __shared__ int changed;
    const KbItem it = items[blockIdx.x];
    KbInst &I = inst[it.inst];
    if (relabel_pass ? !I.relabel : I.done) return;
    // relabel: against the final centres Cb[fc], into the final buffer Lb[fl]
    const int cb = relabel_pass ? I.fc : (I.it & 1);
    const float *C = (cb ? Cb1 : Cb0) + I.co;
    const int lb = relabel_pass ? I.fl : (I.it & 1);
    int *L = (lb ? Lb1 : Lb0) + I.lo;
    const int *Lp = relabel_pass ? nullptr : ((lb ? Lb0 : Lb1) + I.lo);
    const float *Xi = X + I.xo;
    const int n = I.n, k = I.k, d = I.d, ld = I.ld, i0 = it.r0;
    const int tid = threadIdx.x, tm = tid / 16, tn = tid % 16;
    if (tid == 0) changed = 0;
    float best[TM];
    int bidx[TM];
#pragma unroll
    for (int i = 0; i < TM; ++i) {
        best[i] = Lim<float>::inf();
        bidx[i] = 0x7fffffff;
    }
    Acc<float, TM, TN> acc;
    for (int j0 = 0; j0 < k; j0 += BN) {
        compute_tile<float, ACC_DOT, TM, TN, BM, BN, BK>(st, Xi, ld, n, i0, C, ld, k, j0, d, 256,
                                                         0.f, acc, tid);
#pragma unroll
        for (int j = 0; j < TN; ++j) {
            const int gj = j0 + (j / 4) * 64 + tn * 4 + (j % 4);
            if (gj >= k) continue;
            const float cn = cnorm[I.no + gj];
#pragma unroll
            for (int i = 0; i < TM; ++i) {
                const float v = fma_rn(-2.f, acc.g1[i][j], cn);
                if (key_less(v, gj, best[i], bidx[i])) {
                    best[i] = v;
                    bidx[i] = gj;
                }
            }
        }
    }
#pragma unroll
    for (int i = 0; i < TM; ++i) {
#pragma unroll
        for (int off = 8; off >= 1; off >>= 1) {
            const float ov = __shfl_xor_sync(0xffffffffu, best[i], off);
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
                const int lbl = (bidx[i] == 0x7fffffff) ? 0 : bidx[i];
                L[gi] = lbl;
                if (Lp && Lp[gi] != lbl) ch = 1;
            }
        }
        if (ch) changed = 1;
    }
    __syncthreads();
    if (tid == 0 && changed) atomicOr(&I.changed, 1);
}

// Fixed-point sums of one batch of one instance's rows (bucketed by label in
// shared memory, run sums in registers), added into the instance's int64
// accumulators; the cluster counts likewise.
__global__ void __launch_bounds__(KB_UPD_THREADS)
kb_update(const float *X, KbInst *inst, const KbItem *items, const int *Lb0, const int *Lb1,
          const float *scale, unsigned long long *gacc, int *gcnt) {
    extern __shared__ __align__(16) unsigned char kb_smem[];
    const KbItem itm = items[blockIdx.x];
    KbInst &I = inst[itm.inst];
    if (I.done) return;
    const int k = I.k, d = I.d, ld = I.ld;
    const int *labels = ((I.it & 1) ? Lb1 : Lb0) + I.lo;
    const float *Xi = X + I.xo;
    const int kd = k * d;
    unsigned long long *acc = reinterpret_cast<unsigned long long *>(kb_smem);
    int *list = reinterpret_cast<int *>(acc + kd);
    int *off = list + KB_BATCH;
    int *cur = off + k + 1;
    float *sc = reinterpret_cast<float *>(cur + k + 1);
    for (int e = threadIdx.x; e < kd; e += blockDim.x) acc[e] = 0ull;
    for (int f = threadIdx.x; f < d; f += blockDim.x) sc[f] = scale[I.so + f];
    for (int j = threadIdx.x; j <= k; j += blockDim.x) cur[j] = 0;
    const int b0 = itm.r0, nb = min(KB_BATCH, I.n - b0);
    __syncthreads();
    for (int i = threadIdx.x; i < nb; i += blockDim.x) atomicAdd(&cur[labels[b0 + i]], 1);
    __syncthreads();
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31, nw = blockDim.x >> 5;
    if (warp == 0) {
        int carry = 0;
        for (int j0 = 0; j0 < k; j0 += 32) {
            const int j = j0 + lane;
            const int c = j < k ? cur[j] : 0;
            if (c > 0) atomicAdd(&gcnt[I.no + j], c);
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
    for (int i = threadIdx.x; i < nb; i += blockDim.x) list[atomicAdd(&cur[labels[b0 + i]], 1)] = b0 + i;
    __syncthreads();
    const int p0 = (int)((long long)nb * warp / nw), p1 = (int)((long long)nb * (warp + 1) / nw);
    if (p0 < p1) {
        int j0 = 0;
        {
            int lo = 0, hi = k - 1;
            while (lo < hi) {
                const int mid = (lo + hi + 1) >> 1;
                if (off[mid] <= p0) lo = mid;
                else hi = mid - 1;
            }
            j0 = lo;
        }
        for (int fb = 0; fb < d; fb += 32) {
            const int f = fb + lane;
            const float s0 = f < d ? sc[f] : 0.f;
            const float s0_22 = s0 * 2.384185791015625e-07f;
            int j = j0;
            int jend = off[j + 1];
            FxRun run;
            for (int p = p0; p < p1; ++p) {
                const float xv = f < d ? Xi[(size_t)list[p] * ld + f] : 0.f;
                while (p >= jend) {
                    fx_flush(acc, d, j, f, run, false);
                    ++j;
                    jend = off[j + 1];
                }
                fx_acc(xv, s0_22, s0, run.h0, run.l0);
                ++run.n;
            }
            fx_flush(acc, d, j, f, run, false);
        }
    }
    __syncthreads();
    for (int e = threadIdx.x; e < kd; e += blockDim.x)
        if (acc[e]) atomicAdd(&gacc[I.ao + e], acc[e]);
}

// New centres, the shift sums (the single path's reduction: 256-element
// blocks, tree within a block, blocks lane-strided then shuffled), the
// convergence test and the state update; one CTA per instance.
__global__ void __launch_bounds__(256)
kb_finalize(KbInst *inst, float *Cb0, float *Cb1, const unsigned long long *gacc, const int *gcnt,
            const double *inv, int max_iter, double tol, double *scratch) {
    KbInst &I = inst[blockIdx.x];
    if (I.done) return;
    __shared__ double s0[256], s1[256];
    const float *Cp = ((I.it & 1) ? Cb1 : Cb0) + I.co;
    float *Cn = ((I.it & 1) ? Cb0 : Cb1) + I.co;
    const int k = I.k, d = I.d, kd = k * d;
    const int nblk = (kd + 255) / 256;
    double *bp = scratch + (size_t)blockIdx.x * 2 * ((8192 + 255) / 256);
    for (int blk = 0; blk < nblk; ++blk) {
        const int e = blk * 256 + threadIdx.x;
        double pn = 0.0, ps = 0.0;
        if (e < kd) {
            const int j = e / d, f = e - j * d;
            const long long S = (long long)gacc[I.ao + e];
            const int c = gcnt[I.no + j];
            const float cn = (float)(((double)S * inv[I.so + f]) / (double)(c > 0 ? c : 1));
            const float cp = Cp[(size_t)j * I.ld + f];
            Cn[(size_t)j * I.ld + f] = cn;
            pn = (double)cp * (double)cp;
            const double df = (double)cp - (double)cn;
            ps = df * df;
        }
        s0[threadIdx.x] = pn;
        s1[threadIdx.x] = ps;
        __syncthreads();
        for (int o = 128; o > 0; o >>= 1) {
            if ((int)threadIdx.x < o) {
                s0[threadIdx.x] += s0[threadIdx.x + o];
                s1[threadIdx.x] += s1[threadIdx.x + o];
            }
            __syncthreads();
        }
        if (threadIdx.x == 0) {
            bp[2 * blk] = s0[0];
            bp[2 * blk + 1] = s1[0];
        }
        __syncthreads();
    }
    if (threadIdx.x < 32) {
        const int lane = threadIdx.x;
        double v2[2];
        for (int v = 0; v < 2; ++v) {
            double a = 0.0;
            for (int b = lane; b < nblk; b += 32) a += bp[2 * b + v];
#pragma unroll
            for (int o = 16; o > 0; o >>= 1) a += __shfl_down_sync(0xffffffffu, a, o);
            v2[v] = a;
        }
        if (lane == 0) {
            I.normc2 = v2[0];
            I.shift2 = v2[1];
            int conv = 0;
            if (I.it > 1 && I.changed == 0) conv = 2;
            if (conv == 0 && sqrt(v2[1]) < tol * sqrt(v2[0])) conv = 1;
            // final centres: this iteration's new ones; final labels: this
            // iteration's, or the relabelling's (into the other buffer)
            if (conv > 0) {
                I.done = 1;
                I.conv = conv;
                I.n_iter = I.it;
                I.relabel = conv == 1 ? 1 : 0;
                I.fc = (I.it + 1) & 1;
                I.fl = conv == 1 ? ((I.it + 1) & 1) : (I.it & 1);
            } else if (I.it + 1 == max_iter) {
                I.done = 1;
                I.conv = 0;
                I.n_iter = max_iter;
                I.relabel = 1;
                I.fc = (I.it + 1) & 1;
                I.fl = (I.it + 1) & 1;
            }
            I.it += 1;
        }
    }
}

// Inertia sum_i |x_i - c_{label_i}|^2 in fp64 (one CTA per instance, rows
// over warps, fixed reduction order).
__global__ void kb_inertia(const float *X, KbInst *inst, const float *Cb0, const float *Cb1,
                           const int *Lb0, const int *Lb1, double *out) {
    KbInst &I = inst[blockIdx.x];
    __shared__ double sh[8];
    const float *C = (I.fc ? Cb1 : Cb0) + I.co;
    const int *L = (I.fl ? Lb1 : Lb0) + I.lo;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    double acc = 0.0;
    for (int i = warp; i < I.n; i += 8) {
        const float *x = X + I.xo + (size_t)i * I.ld;
        const float *c = C + (size_t)L[i] * I.ld;
        double r = 0.0;
        for (int f = lane; f < I.d; f += 32) {
            const double t = (double)x[f] - (double)c[f];
            r += t * t;
        }
        acc += r;
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) sh[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += sh[w];
        out[blockIdx.x] = t;
    }
}

template <typename V> struct DBuf {
    V *p = nullptr;
    ~DBuf() {
        if (p) cudaFree(p);
    }
    cudaError_t alloc(size_t n) {
        return device_alloc(reinterpret_cast<void **>(&p), std::max<size_t>(n, 1) * sizeof(V));
    }
};

} // namespace

} // namespace b200

using namespace b200;

extern "C" da_status da_b200_kmeans_batched_s(da_int n_inst, const da_int *n_samples,
                                              const da_int *n_features, const da_int *n_clusters,
                                              const float *const *A, const da_int *lda,
                                              const float *const *C_init, da_int max_iter,
                                              double tol, float *const *C_out,
                                              da_int *const *labels_out, da_int *n_iter,
                                              double *inertia, da_int *converged, void *stream) {
    if (sizeof(da_int) != sizeof(int)) return da_status_not_implemented;
    if (n_inst < 1) return da_status_invalid_array_dimension;
    if (!n_samples || !n_features || !n_clusters || !A || !lda || !C_init || !C_out ||
        !labels_out || !n_iter || !inertia || !converged)
        return da_status_invalid_pointer;
    if (max_iter < 1 || !(tol >= 0.0)) return da_status_invalid_input;
    int dev_count = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) {
        cudaGetLastError();
        return da_status_arch_not_supported;
    }
    // layout of the packed device buffers
    std::vector<KbInst> hi(n_inst);
    std::vector<KbItem> assign_items, update_items;
    long long xo = 0, co = 0, lo = 0, no = 0, ao = 0, so = 0;
    size_t max_smem_kd = 0;
    for (da_int i = 0; i < n_inst; ++i) {
        const da_int n = n_samples[i], d = n_features[i], k = n_clusters[i];
        if (n < 1 || d < 1 || k < 1 || k > n) return da_status_invalid_array_dimension;
        if ((long long)k * d > 8192) return da_status_invalid_array_dimension;
        if (!A[i] || !C_init[i] || !C_out[i] || !labels_out[i]) return da_status_invalid_pointer;
        if (lda[i] < d) return da_status_invalid_leading_dimension;
        KbInst &I = hi[i];
        std::memset(&I, 0, sizeof(I));
        I.n = (int)n;
        I.d = (int)d;
        I.ld = pad4((int)d);
        I.k = (int)k;
        int L = 0;
        while ((1LL << L) < (long long)n) ++L;
        I.L = L;
        I.xo = xo;
        I.co = co;
        I.lo = lo;
        I.no = no;
        I.ao = ao;
        I.so = so;
        xo += (long long)n * I.ld;
        co += (long long)k * I.ld;
        lo += n;
        no += k;
        ao += (long long)k * d;
        so += d;
        max_smem_kd = std::max(max_smem_kd, (size_t)k * d);
        for (int r = 0; r < n; r += 64) assign_items.push_back({(int)i, r});
        for (int r = 0; r < n; r += KB_BATCH) update_items.push_back({(int)i, r});
    }
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DBuf<float> X, Cb0, Cb1, cn, sc;
    DBuf<int> Lb0, Lb1, cnt, bad;
    DBuf<unsigned long long> acc;
    DBuf<double> inv, scratch, inert;
    DBuf<KbInst> inst;
    DBuf<KbItem> aitems, uitems;
    cudaError_t e = cudaSuccess;
    auto ok = [&](cudaError_t r) {
        if (e == cudaSuccess) e = r;
        return e == cudaSuccess;
    };
    ok(X.alloc(xo));
    ok(Cb0.alloc(co));
    ok(Cb1.alloc(co));
    ok(cn.alloc(no));
    ok(sc.alloc(so));
    ok(Lb0.alloc(lo));
    ok(Lb1.alloc(lo));
    ok(cnt.alloc(no));
    ok(bad.alloc(1));
    ok(acc.alloc(ao));
    ok(inv.alloc(so));
    ok(scratch.alloc((size_t)n_inst * 2 * 32));
    ok(inert.alloc(n_inst));
    ok(inst.alloc(n_inst));
    ok(aitems.alloc(assign_items.size()));
    ok(uitems.alloc(update_items.size()));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return da_status_memory_error;
    }
    // upload: rows padded to ld by the copy engine, initial centres into Cb0
    {
        ok(cudaMemsetAsync(X.p, 0, xo * sizeof(float), s));
        ok(cudaMemsetAsync(Cb0.p, 0, co * sizeof(float), s));
        for (da_int i = 0; i < n_inst && e == cudaSuccess; ++i) {
            const KbInst &I = hi[i];
            ok(cudaMemcpy2DAsync(X.p + I.xo, (size_t)I.ld * 4, A[i], (size_t)lda[i] * 4,
                                 (size_t)I.d * 4, I.n, cudaMemcpyHostToDevice, s));
            ok(cudaMemcpy2DAsync(Cb0.p + I.co, (size_t)I.ld * 4, C_init[i], (size_t)I.d * 4,
                                 (size_t)I.d * 4, I.k, cudaMemcpyHostToDevice, s));
        }
        ok(cudaMemsetAsync(Cb1.p, 0, co * sizeof(float), s));
        ok(cudaMemsetAsync(Lb0.p, 0, lo * sizeof(int), s));
        ok(cudaMemsetAsync(Lb1.p, 0, lo * sizeof(int), s));
        ok(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
        ok(cudaMemcpyAsync(inst.p, hi.data(), hi.size() * sizeof(KbInst), cudaMemcpyHostToDevice, s));
        ok(cudaMemcpyAsync(aitems.p, assign_items.data(), assign_items.size() * sizeof(KbItem),
                           cudaMemcpyHostToDevice, s));
        ok(cudaMemcpyAsync(uitems.p, update_items.data(), update_items.size() * sizeof(KbItem),
                           cudaMemcpyHostToDevice, s));
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        return da_status_internal_error;
    }
    int max_d = 0;
    for (const KbInst &I : hi) max_d = std::max(max_d, I.d);
    kb_scales<<<n_inst, 256, (size_t)max_d * sizeof(unsigned), s>>>(X.p, inst.p, sc.p, inv.p, bad.p);
    int h_bad = 0;
    ok(cudaMemcpyAsync(&h_bad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    ok(cudaStreamSynchronize(s));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return da_status_internal_error;
    }
    if (h_bad) return da_status_invalid_input; // inf / NaN in the data
    int max_k = 0;
    for (const KbInst &I : hi) max_k = std::max(max_k, I.k);
    const size_t usmem = max_smem_kd * 8 + (size_t)KB_BATCH * 4 + (size_t)2 * (max_k + 1) * 4 +
                         (size_t)max_d * 4 + 16;
    ok(ensure_smem_limit(reinterpret_cast<const void *>(kb_update), usmem));
    // The whole fit as one CUDA graph: max_iter iterations of four launches
    // (finished instances skip their work), the final relabelling and the
    // inertia; replayed once.
    cudaStream_t cs = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ok(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    if (e == cudaSuccess && ok(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal))) {
        for (da_int it = 0; it < max_iter; ++it) {
            kb_begin<<<n_inst, 128, 0, cs>>>(inst.p, Cb0.p, Cb1.p, cn.p, acc.p, cnt.p);
            kb_assign<<<(unsigned)assign_items.size(), 256, 0, cs>>>(
                X.p, inst.p, aitems.p, Cb0.p, Cb1.p, cn.p, Lb0.p, Lb1.p, 0);
            kb_update<<<(unsigned)update_items.size(), KB_UPD_THREADS, usmem, cs>>>(
                X.p, inst.p, uitems.p, Lb0.p, Lb1.p, sc.p, acc.p, cnt.p);
            kb_finalize<<<n_inst, 256, 0, cs>>>(inst.p, Cb0.p, Cb1.p, acc.p, cnt.p, inv.p,
                                                (int)max_iter, tol, scratch.p);
        }
        kb_final_norms<<<n_inst, 128, 0, cs>>>(inst.p, Cb0.p, Cb1.p, cn.p);
        kb_assign<<<(unsigned)assign_items.size(), 256, 0, cs>>>(X.p, inst.p, aitems.p, Cb0.p,
                                                                  Cb1.p, cn.p, Lb0.p, Lb1.p, 1);
        kb_inertia<<<n_inst, 256, 0, cs>>>(X.p, inst.p, Cb0.p, Cb1.p, Lb0.p, Lb1.p, inert.p);
        const cudaError_t ce = cudaStreamEndCapture(cs, &graph);
        ok(cudaGetLastError());
        ok(ce);
        if (e == cudaSuccess) ok(cudaGraphInstantiate(&exec, graph, 0));
    }
    // order the graph after the uploads on the caller's stream
    cudaEvent_t ev = nullptr;
    ok(cudaEventCreateWithFlags(&ev, cudaEventDisableTiming));
    ok(cudaEventRecord(ev, s));
    ok(cudaStreamWaitEvent(cs, ev, 0));
    if (e == cudaSuccess) ok(cudaGraphLaunch(exec, cs));
    ok(cudaStreamSynchronize(cs));
    // results
    std::vector<KbInst> fin(n_inst);
    std::vector<double> hin(n_inst);
    ok(cudaMemcpy(fin.data(), inst.p, fin.size() * sizeof(KbInst), cudaMemcpyDeviceToHost));
    ok(cudaMemcpy(hin.data(), inert.p, hin.size() * sizeof(double), cudaMemcpyDeviceToHost));
    for (da_int i = 0; i < n_inst && e == cudaSuccess; ++i) {
        const KbInst &I = fin[i];
        ok(cudaMemcpy2DAsync(C_out[i], (size_t)I.d * 4, (I.fc ? Cb1.p : Cb0.p) + I.co,
                             (size_t)I.ld * 4, (size_t)I.d * 4, I.k, cudaMemcpyDeviceToHost, cs));
        ok(cudaMemcpyAsync(labels_out[i], (I.fl ? Lb1.p : Lb0.p) + I.lo, (size_t)I.n * sizeof(int),
                           cudaMemcpyDeviceToHost, cs));
        n_iter[i] = I.n_iter;
        inertia[i] = hin[i];
        converged[i] = I.conv;
    }
    ok(cudaStreamSynchronize(cs));
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    if (ev) cudaEventDestroy(ev);
    if (cs) cudaStreamDestroy(cs);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return da_status_internal_error;
    }
    return da_status_success;
}
