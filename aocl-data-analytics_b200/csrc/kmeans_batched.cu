// Batched k-means (Lloyd): many independent fp32 data sets of different n, d
// and k fitted together on one device.
//
// Work is cut into (instance, tile) items.  Every Lloyd iteration is
//   kb_begin     the previous centres' norms, cleared change counters;
//   kb_assign    persistent blocks that pull tiles of 256 rows off a work
//                queue (one atomic counter per tile shape): the tile's rows
//                and its instance's centres are staged in shared memory, each
//                thread assigns one row from registers, and rows whose label
//                changed are appended to their instance's change list;
//   kb_delta     persistent blocks that pull chunks of the change lists and
//                move each changed row's fixed-point values from its old
//                cluster's sums to its new one's (exact 64-bit integers, so
//                the sums equal a full recount whatever the order);
//   kb_finalize  new centres, the shift reduction and the convergence test,
//                one block per instance;
// and the whole fit (all iterations, the final relabelling, the inertia) is
// one CUDA graph replayed without host round trips.  Converged instances
// skip their items.  The assignment kernel comes in tile shapes -- the row
// width it holds in registers (16, 32, 64, 128 or any wider) times the
// centres it scores at once (2, 4 or 8) -- and the shape for each (width,
// k range) is picked by timing the candidates on the first data sets that
// need it (kept for the process: an autotuner).
//
// Each instance follows exactly the single-data-set path with precision mode
// "plain", n_init = 1 and supplied initial centres (kmeans.cpp:996-1058 as
// restated in kmeans.cpp here): the same assignment formula and order (x.c
// one fma chain over the features, v = fma(-2, x.c, |c|^2), ties to the
// lower index), the same fixed-point centroid sums and scales, the same
// shift reduction and convergence test, the same final relabelling; so its
// labels, centres and iteration count equal that path's.
#include "b200_common.cuh"
#include "b200_kernels.hpp"
#include "device_alloc.hpp"
#include "kmeans_fx.cuh"
#include "../../include/aoclda_b200_ext.h"
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

namespace b200 {

namespace {

constexpr int KB_T = 256;          // threads of an assignment block
constexpr int KB_ROWS = 128;       // rows per assignment tile
constexpr int KB_SCAN_ROWS = 4096; // rows per item of the column-maxima and inertia passes
constexpr int KB_CH = 2048;        // change-list entries per update item
constexpr int KB_NW = 5;           // row widths of the assignment: 16, 32, 64, 128, wider
constexpr int KB_NK = 4;           // k ranges: <= 16, <= 32, <= 64, more
constexpr int KB_NG = 3;           // centres per thread in the register tile: 2, 4, 8

struct KbInst {
    int n, d, ld, k, L;
    int it, done, conv, n_iter, relabel, fc, nchg;
    int s0, sn; // the instance's items of the scan passes
    long long xo, co, lo, no, ao, so;
    double normc2, shift2;
};
struct KbItem {
    int inst, r0;
};

__host__ __device__ constexpr int kb_width(int wi) { return wi < 4 ? (16 << wi) : 0; }
// sub-tiles of KB_ROWS rows in one assignment tile: narrow rows take more
// rows per tile (the same staged bytes, fewer queue trips per row)
__host__ __device__ constexpr int kb_subtiles(int w) { return w == 0 || w >= 128 ? 1 : w == 64 ? 2 : 4; }

// 16-byte asynchronous copy global -> shared (src_bytes 16, or 0 to write
// zeros without reading), so that a thread has many loads in flight.
__device__ __forceinline__ void kb_cp16(void *smem, const void *gmem, int src_bytes) {
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;" ::"r"(
                     static_cast<unsigned>(__cvta_generic_to_shared(smem))),
                 "l"(gmem), "r"(src_bytes)
                 : "memory");
}
__device__ __forceinline__ void kb_cp_wait() {
    asm volatile("cp.async.commit_group;\n\tcp.async.wait_group 0;" ::: "memory");
}

// ------------------------------------------------------- fixed-point scales --
// Per-feature max |x| (as bits) of one scan item, into the instance's maxima;
// inf / NaN raise *bad.
__global__ void __launch_bounds__(256)
kb_colmax(const float *X, const KbInst *inst, const KbItem *items, unsigned *colmax, int *bad) {
    extern __shared__ unsigned cm[];
    const KbItem it = items[blockIdx.x];
    const KbInst &I = inst[it.inst];
    const int d = I.d;
    for (int f = threadIdx.x; f < d; f += blockDim.x) cm[f] = 0u;
    __syncthreads();
    int tpr = 32; // threads per row, a power of two
    while (tpr > 1 && tpr / 2 >= d) tpr >>= 1;
    const int sub = threadIdx.x % tpr, rstep = blockDim.x / tpr;
    const int nr = min(KB_SCAN_ROWS, I.n - it.r0);
    const float *x = X + I.xo + (size_t)it.r0 * I.ld;
    unsigned m[4] = {0u, 0u, 0u, 0u};
    int badl = 0;
    for (int r = threadIdx.x / tpr; r < nr; r += rstep) {
        const float *xr = x + (size_t)r * I.ld;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
            const int f = sub + c * tpr;
            if (f < d) {
                const unsigned b = __float_as_uint(xr[f]) & 0x7fffffffu;
                if (b >= 0x7f800000u) badl = 1;
                else m[c] = max(m[c], b);
            }
        }
        for (int f = sub + 4 * tpr; f < d; f += tpr) {
            const unsigned b = __float_as_uint(xr[f]) & 0x7fffffffu;
            if (b >= 0x7f800000u) badl = 1;
            else atomicMax(&cm[f], b);
        }
    }
#pragma unroll
    for (int c = 0; c < 4; ++c)
        if (sub + c * tpr < d) atomicMax(&cm[sub + c * tpr], m[c]);
    if (badl) atomicOr(bad, 1);
    __syncthreads();
    for (int f = threadIdx.x; f < d; f += blockDim.x) atomicMax(&colmax[I.so + f], cm[f]);
}

// Scales from the maxima (the single-data-set rule: s_f = min(62 - L, 44) -
// E_f with max|x_f| < 2^E_f, clamped to [-126, 127]).
__global__ void kb_scales(const KbInst *inst, const unsigned *colmax, float *scale, double *inv) {
    const KbInst &I = inst[blockIdx.x];
    for (int f = threadIdx.x; f < I.d; f += blockDim.x) {
        const unsigned m = colmax[I.so + f];
        int E = 0;
        if (m != 0u) frexpf(__uint_as_float(m), &E); // m < 2^E
        int sf = min(62 - I.L, 44) - E;
        sf = max(-126, min(127, sf));
        scale[I.so + f] = __uint_as_float((unsigned)(sf + 127) << 23);
        inv[I.so + f] = ldexp(1.0, -sf);
    }
}

// ---------------------------------------------------------- iteration start --
// |c_j|^2 of the previous centres (one fma chain per centre, as the single
// path) and a cleared change counter; block 0 re-arms the work queues.
__global__ void kb_begin(KbInst *inst, const float *Cb0, const float *Cb1, float *cnorm,
                         int *queues, int n_queues) {
    if (blockIdx.x == 0)
        for (int q = threadIdx.x; q < n_queues; q += blockDim.x) queues[q] = 0;
    KbInst &I = inst[blockIdx.x];
    if (I.done) return;
    const float *C = ((I.it & 1) ? Cb1 : Cb0) + I.co;
    for (int j = threadIdx.x; j < I.k; j += blockDim.x) {
        const float *c = C + (size_t)j * I.ld;
        float s = 0.f;
        for (int f = 0; f < I.d; ++f) s = __fmaf_rn(c[f], c[f], s);
        cnorm[I.no + j] = s;
    }
    if (threadIdx.x == 0) I.nchg = 0;
}

// |c_j|^2 of the final centres of the instances flagged for relabelling.
__global__ void kb_final_norms(const KbInst *inst, const float *Cb0, const float *Cb1,
                               float *cnorm) {
    const KbInst &I = inst[blockIdx.x];
    if (!I.relabel) return;
    const float *C = (I.fc ? Cb1 : Cb0) + I.co;
    for (int j = threadIdx.x; j < I.k; j += blockDim.x) {
        const float *c = C + (size_t)j * I.ld;
        float s = 0.f;
        for (int f = 0; f < I.d; ++f) s = __fmaf_rn(c[f], c[f], s);
        cnorm[I.no + j] = s;
    }
}

// --------------------------------------------------------------- assignment --
// Persistent: blocks take tiles of KB_ROWS rows of one instance off the
// queue.  W > 0 (rows of at most W features, zero-padded to W: the padded
// terms come after the real ones in every chain and add exact zeros): the
// tile's rows and the instance's centres are staged in shared memory and
// thread (rg, cg) of 32 x 8 scores rows rg + 32 i (i < 4) against centres
// cb + cg + 8 j (j < TC) of each block of 8 TC centres, a 4 x TC register
// tile fed by 16-byte shared-memory reads (4 + TC reads per 16 TC fmas); the
// 8 threads of a row group then reduce their best centres with shuffles.
// W == 0 (wider rows): one thread per row, rows read from global memory.
// mode 0: a Lloyd iteration (labels, change list); 1: the final relabelling
// of the flagged instances against their final centres; 2: a timing run of
// the autotuner (labels only, every instance, previous centres).
template <int W, int TC>
__global__ void __launch_bounds__(KB_T)
kb_assign(const float *X, KbInst *inst, const KbItem *items, int n_items, int *queue,
          const float *Cb0, const float *Cb1, const float *cnorm, int *lab, int2 *chg, int mode,
          int kmax) {
    extern __shared__ __align__(16) float kb_sm[];
    constexpr int WS = W + 4;          // staged row stride: conflict-free 16-byte reads
    constexpr int CB = 8 * TC;         // centres per block of the register tile
    constexpr int RT = kb_subtiles(W); // sub-tiles of KB_ROWS rows per tile
    __shared__ int s_item;
    const int tid = threadIdx.x, lane = tid & 31;
    const int rg = tid >> 3, cg = tid & 7;
    for (;;) {
        __syncthreads(); // the previous tile's shared data are used up
        if (tid == 0) s_item = atomicAdd(queue, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= n_items) break;
        const KbItem it = items[item];
        KbInst &I = inst[it.inst];
        if (mode == 1 ? !I.relabel : (mode == 0 && I.done)) continue;
        const int cb_ = mode == 1 ? I.fc : (I.it & 1);
        const float *C = (cb_ ? Cb1 : Cb0) + I.co;
        const int k = I.k, d = I.d, ld = I.ld, r0 = it.r0;
        const int nr = min(KB_ROWS * RT, I.n - r0);
        const float *Xi = X + I.xo + (size_t)r0 * ld;
        // the current labels of this thread's rows (thread cg == 0 of each
        // row group: rows st * KB_ROWS + rg + 32 i), loaded before the work
        int old[RT][4];
#pragma unroll
        for (int st = 0; st < RT; ++st)
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int r = st * KB_ROWS + rg + 32 * i;
                old[st][i] = (mode == 0 && cg == 0 && r < nr) ? lab[I.lo + r0 + r] : 0;
            }
        // labels of sub-tile st; changed rows join the instance's change list
        // (at most one counter atomic per warp and sub-tile)
        auto emit = [&](int st, const int (&lbl)[4]) {
            const int sr = st * KB_ROWS;
            unsigned m[4];
            int tot = 0;
#pragma unroll
            for (int i = 0; i < 4; ++i) {
                const int r = sr + rg + 32 * i;
                const bool mine = cg == 0 && r < nr;
                const bool ch = mine && (mode != 0 || old[st][i] != lbl[i]);
                if (ch) lab[I.lo + r0 + r] = lbl[i];
                m[i] = mode == 0 ? __ballot_sync(0xffffffffu, ch) : 0u;
                tot += __popc(m[i]);
            }
            if (mode == 0 && tot > 0) {
                int base = 0;
                if (lane == 0) base = atomicAdd(&I.nchg, tot);
                base = __shfl_sync(0xffffffffu, base, 0);
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    const int r = sr + rg + 32 * i;
                    if ((m[i] >> lane) & 1u)
                        chg[I.lo + base + __popc(m[i] & ((1u << lane) - 1u))] =
                            make_int2(r0 + r, (old[st][i] + 1) | (lbl[i] << 16));
                    base += __popc(m[i]);
                }
            }
        };
        if constexpr (W > 0) {
            float *xs = kb_sm;                   // RT * KB_ROWS x WS
            float *cs = xs + RT * KB_ROWS * WS;  // kpad x WS
            float *cns = cs + (size_t)kmax * WS; // kpad
            const int kpad = (k + CB - 1) / CB * CB;
            // centres and rows, 16 bytes per copy (rows are ld = d rounded up
            // to 4 floats long, zero beyond d; zeros written past ld and for
            // the padding centres and rows)
            constexpr int W4 = W / 4;
            for (int e = tid; e < kpad * W4; e += KB_T) {
                const int j = e / W4, f = (e % W4) * 4;
                const bool in = j < k && f < ld;
                kb_cp16(&cs[j * WS + f], C + (in ? (size_t)j * ld + f : 0), in ? 16 : 0);
            }
            for (int e = tid; e < RT * KB_ROWS * W4; e += KB_T) {
                const int r = e / W4, f = (e % W4) * 4;
                const bool in = r < nr && f < ld;
                kb_cp16(&xs[r * WS + f], Xi + (in ? (size_t)r * ld + f : 0), in ? 16 : 0);
            }
            for (int j = tid; j < kpad; j += KB_T) cns[j] = j < k ? cnorm[I.no + j] : 0.f;
            kb_cp_wait();
            __syncthreads();
#pragma unroll
            for (int st = 0; st < RT; ++st) {
                const int sr = st * KB_ROWS;
                if (sr >= nr) break;
                const float *xt = xs + sr * WS;
                float best[4];
                int bi[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) {
                    best[i] = Lim<float>::inf();
                    bi[i] = 0x7fffffff;
                }
                for (int cb = 0; cb < k; cb += CB) {
                    float acc[4][TC];
#pragma unroll
                    for (int i = 0; i < 4; ++i)
#pragma unroll
                        for (int j = 0; j < TC; ++j) acc[i][j] = 0.f;
#pragma unroll 4
                    for (int q = 0; q < W; q += 4) {
                        float4 xv[4], cv[TC];
#pragma unroll
                        for (int i = 0; i < 4; ++i)
                            xv[i] = *reinterpret_cast<const float4 *>(&xt[(rg + 32 * i) * WS + q]);
#pragma unroll
                        for (int j = 0; j < TC; ++j)
                            cv[j] =
                                *reinterpret_cast<const float4 *>(&cs[(cb + cg + 8 * j) * WS + q]);
#pragma unroll
                        for (int i = 0; i < 4; ++i)
#pragma unroll
                            for (int j = 0; j < TC; ++j) {
                                acc[i][j] = fma_rn(xv[i].x, cv[j].x, acc[i][j]);
                                acc[i][j] = fma_rn(xv[i].y, cv[j].y, acc[i][j]);
                                acc[i][j] = fma_rn(xv[i].z, cv[j].z, acc[i][j]);
                                acc[i][j] = fma_rn(xv[i].w, cv[j].w, acc[i][j]);
                            }
                    }
#pragma unroll
                    for (int j = 0; j < TC; ++j) {
                        const int c = cb + cg + 8 * j;
                        if (c < k) {
                            const float cn = cns[c];
#pragma unroll
                            for (int i = 0; i < 4; ++i) {
                                const float v = fma_rn(-2.f, acc[i][j], cn);
                                if (key_less(v, c, best[i], bi[i])) {
                                    best[i] = v;
                                    bi[i] = c;
                                }
                            }
                        }
                    }
                }
                // the row group's 8 threads: best of their centres
                int lbl[4];
#pragma unroll
                for (int i = 0; i < 4; ++i) {
#pragma unroll
                    for (int off = 1; off < 8; off <<= 1) {
                        const float ov = __shfl_xor_sync(0xffffffffu, best[i], off);
                        const int oi = __shfl_xor_sync(0xffffffffu, bi[i], off);
                        if (key_less(ov, oi, best[i], bi[i])) {
                            best[i] = ov;
                            bi[i] = oi;
                        }
                    }
                    lbl[i] = bi[i] == 0x7fffffff ? 0 : bi[i];
                }
                emit(st, lbl);
            }
        } else {
            float *cs = kb_sm;                  // k x d
            float *cns = cs + (size_t)kmax * d; // k
            for (int e = tid; e < k * d; e += KB_T) {
                const int j = e / d, f = e - j * d;
                cs[e] = C[(size_t)j * ld + f];
            }
            for (int j = tid; j < k; j += KB_T) cns[j] = cnorm[I.no + j];
            __syncthreads();
            // thread (rg, cg == 0) takes rows rg + 32 i, like the tiled path
            int lbl[4] = {0, 0, 0, 0};
            if (cg == 0) {
#pragma unroll 1
                for (int i = 0; i < 4; ++i) {
                    const int r = rg + 32 * i;
                    if (r >= nr) continue;
                    const float *xr = Xi + (size_t)r * ld;
                    float best = Lim<float>::inf();
                    int bi = 0x7fffffff;
                    for (int j = 0; j < k; ++j) {
                        float a = 0.f;
                        for (int f = 0; f < d; ++f) a = fma_rn(xr[f], cs[j * d + f], a);
                        const float v = fma_rn(-2.f, a, cns[j]);
                        if (key_less(v, j, best, bi)) {
                            best = v;
                            bi = j;
                        }
                    }
                    lbl[i] = bi == 0x7fffffff ? 0 : bi;
                }
            }
            emit(0, lbl);
        }
    }
}

// ------------------------------------------------------------------- update --
// Persistent: blocks take chunks of KB_CH entries of one instance's change
// list (row, old label + 1, new label); every changed row's fixed-point
// values q = round(x * 2^s_f) leave its old cluster's sums (none in the first
// iteration, where every row is listed) and join its new one's, first in
// shared memory, then added to the instance's 64-bit sums.
__global__ void __launch_bounds__(256)
kb_delta(const float *X, const KbInst *inst, const KbItem *items, int n_items, int *queue,
         const int2 *chg, const float *scale, unsigned long long *gacc, int *gcnt, int kdmax,
         int kmax) {
    extern __shared__ __align__(16) unsigned long long dsm[];
    unsigned long long *acc = dsm;                          // kdmax
    int *cnt = reinterpret_cast<int *>(acc + kdmax);        // kmax
    float *sc = reinterpret_cast<float *>(cnt + kmax);      // d
    __shared__ int s_item;
    const int tid = threadIdx.x;
    for (;;) {
        __syncthreads();
        if (tid == 0) s_item = atomicAdd(queue, 1);
        __syncthreads();
        const int item = s_item;
        if (item >= n_items) break;
        const KbItem it = items[item];
        const KbInst &I = inst[it.inst];
        if (I.done) continue;
        const int nc = *((volatile const int *)&I.nchg);
        if (it.r0 >= nc) continue;
        const int c1 = min(nc, it.r0 + KB_CH);
        const int k = I.k, d = I.d, kd = k * d;
        for (int e = tid; e < kd; e += blockDim.x) acc[e] = 0ull;
        for (int j = tid; j < k; j += blockDim.x) cnt[j] = 0;
        for (int f = tid; f < d; f += blockDim.x) sc[f] = scale[I.so + f];
        __syncthreads();
        int tpe = 32; // lanes per entry, a power of two
        while (tpe > 1 && tpe / 2 >= d) tpe >>= 1;
        const int sub = tid % tpe;
        for (int e = it.r0 + tid / tpe; e < c1; e += blockDim.x / tpe) {
            const int2 ce = chg[I.lo + e];
            const int jo = (ce.y & 0xFFFF) - 1, jn = ce.y >> 16;
            const float *x = X + I.xo + (size_t)ce.x * I.ld;
            for (int f = sub; f < d; f += tpe) {
                const long long q = __double2ll_rn((double)x[f] * (double)sc[f]);
                atomicAdd(&acc[jn * d + f], (unsigned long long)q);
                if (jo >= 0) atomicAdd(&acc[jo * d + f], (unsigned long long)(-q));
            }
            if (sub == 0) {
                atomicAdd(&cnt[jn], 1);
                if (jo >= 0) atomicSub(&cnt[jo], 1);
            }
        }
        __syncthreads();
        for (int e = tid; e < kd; e += blockDim.x)
            if (acc[e]) atomicAdd(&gacc[I.ao + e], acc[e]);
        for (int j = tid; j < k; j += blockDim.x)
            if (cnt[j]) atomicAdd(&gcnt[I.no + j], cnt[j]);
    }
}

// New centres, the shift sums (the single path's reduction: 256-element
// blocks, tree within a block, blocks lane-strided then shuffled), the
// convergence test and the state update; one CTA per instance.  The sums
// carry over to the next iteration (the update moves only changed rows).
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
            if (I.it > 1 && I.nchg == 0) conv = 2;
            if (conv == 0 && sqrt(v2[1]) < tol * sqrt(v2[0])) conv = 1;
            // final centres: this iteration's new ones; final labels: this
            // iteration's, or the relabelling's
            if (conv > 0) {
                I.done = 1;
                I.conv = conv;
                I.n_iter = I.it;
                I.relabel = conv == 1 ? 1 : 0;
                I.fc = (I.it + 1) & 1;
            } else if (I.it + 1 == max_iter) {
                I.done = 1;
                I.conv = 0;
                I.n_iter = max_iter;
                I.relabel = 1;
                I.fc = (I.it + 1) & 1;
            }
            I.it += 1;
        }
    }
}

// Inertia sum_i |x_i - c_{label_i}|^2 in fp64: one partial per scan item
// (rows over 8 warps, features over lanes, fixed reduction order), summed
// per instance in item order.
__global__ void __launch_bounds__(256)
kb_inertia_part(const float *X, const KbInst *inst, const KbItem *items, const float *Cb0,
                const float *Cb1, const int *lab, double *part) {
    const KbItem it = items[blockIdx.x];
    const KbInst &I = inst[it.inst];
    __shared__ double sh[8];
    const float *C = (I.fc ? Cb1 : Cb0) + I.co;
    const int *L = lab + I.lo;
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int r1 = min(I.n, it.r0 + KB_SCAN_ROWS);
    double acc = 0.0;
    for (int i = it.r0 + warp; i < r1; i += 8) {
        const float *x = X + I.xo + (size_t)i * I.ld;
        const float *c = C + (size_t)L[i] * I.ld;
        for (int f = lane; f < I.d; f += 32) {
            const double t = (double)x[f] - (double)c[f];
            acc += t * t;
        }
    }
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) acc += __shfl_down_sync(0xffffffffu, acc, o);
    if (lane == 0) sh[warp] = acc;
    __syncthreads();
    if (threadIdx.x == 0) {
        double t = 0.0;
        for (int w = 0; w < 8; ++w) t += sh[w];
        part[blockIdx.x] = t;
    }
}
__global__ void kb_inertia_sum(const KbInst *inst, int n_inst, const double *part, double *out) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n_inst) return;
    const KbInst &I = inst[i];
    double t = 0.0;
    for (int s = 0; s < I.sn; ++s) t += part[I.s0 + s];
    out[i] = t;
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

// ------------------------------------------------------ kernel shapes, tuner --
typedef void (*AssignFn)(const float *, KbInst *, const KbItem *, int, int *, const float *,
                         const float *, const float *, int *, int2 *, int, int);

template <int W> AssignFn assign_for_g(int gi) {
    return gi == 0 ? kb_assign<W, 2> : gi == 1 ? kb_assign<W, 4> : kb_assign<W, 8>;
}
AssignFn assign_fn(int wi, int gi) {
    switch (wi) {
    case 0: return assign_for_g<16>(gi);
    case 1: return assign_for_g<32>(gi);
    case 2: return assign_for_g<64>(gi);
    case 3: return assign_for_g<128>(gi);
    default: return assign_for_g<0>(gi);
    }
}
// kmax: the group's largest k rounded up to a whole block of 64 centres
// (the largest register tile)
size_t assign_smem(int wi, int kmax, int dmax) {
    const int w = kb_width(wi);
    return w > 0 ? (size_t)kb_subtiles(w) * KB_ROWS * (w + 4) * 4 + (size_t)kmax * (w + 4) * 4 +
                       (size_t)kmax * 4
                 : (size_t)kmax * dmax * 4 + (size_t)kmax * 4;
}
int width_index(int d) {
    for (int wi = 0; wi < 4; ++wi)
        if (d <= kb_width(wi)) return wi;
    return 4;
}
int k_index(int k) { return k <= 16 ? 0 : k <= 32 ? 1 : k <= 64 ? 2 : 3; }

int resident_blocks(const void *fn, int threads, size_t smem) {
    int dev = 0, nsm = 148, per = 1;
    cudaGetDevice(&dev);
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
    if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per, fn, threads, smem) != cudaSuccess ||
        per < 1) {
        cudaGetLastError();
        per = 1;
    }
    return nsm * per;
}

// The tuner's choices: (device, row width, k range) -> centres scored at once.
std::mutex g_tune_mu;
std::map<std::tuple<int, int, int>, int> g_tune;

thread_local double g_last_ms[3] = {0.0, 0.0, 0.0};

} // namespace

} // namespace b200

using namespace b200;

extern "C" da_status da_b200_kmeans_batched_timing(double *upload_ms, double *fit_ms,
                                                   double *download_ms) {
    if (!upload_ms || !fit_ms || !download_ms) return da_status_invalid_pointer;
    *upload_ms = g_last_ms[0];
    *fit_ms = g_last_ms[1];
    *download_ms = g_last_ms[2];
    return da_status_success;
}

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
    int dev_count = 0, dev = 0;
    if (cudaGetDeviceCount(&dev_count) != cudaSuccess || dev_count == 0) {
        cudaGetLastError();
        return da_status_arch_not_supported;
    }
    cudaGetDevice(&dev);
    // layout of the packed device buffers and the work tables
    constexpr int NGRP = KB_NW * KB_NK; // assignment groups (row width, k range)
    std::vector<KbInst> hi(n_inst);
    std::vector<KbItem> scan_items, delta_items;
    std::vector<std::vector<KbItem>> grp_items(NGRP);
    std::vector<int> grp_kmax(NGRP, 0), grp_dmax(NGRP, 0);
    long long xo = 0, co = 0, lo = 0, no = 0, ao = 0, so = 0;
    int max_d = 0, max_k = 0, max_kd = 0;
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
        max_d = std::max(max_d, (int)d);
        max_k = std::max(max_k, (int)k);
        max_kd = std::max(max_kd, (int)(k * d));
        const int g = width_index((int)d) * KB_NK + k_index((int)k);
        grp_kmax[g] = std::max(grp_kmax[g], (int)k);
        grp_dmax[g] = std::max(grp_dmax[g], (int)d);
        const int rows = KB_ROWS * kb_subtiles(kb_width(g / KB_NK));
        for (int r = 0; r < n; r += rows) grp_items[g].push_back({(int)i, r});
        I.s0 = (int)scan_items.size();
        for (int r = 0; r < n; r += KB_SCAN_ROWS) scan_items.push_back({(int)i, r});
        I.sn = (int)scan_items.size() - I.s0;
        for (int r = 0; r < n; r += KB_CH) delta_items.push_back({(int)i, r});
    }
    // assignment items of all groups in one table, each group a slice
    std::vector<KbItem> assign_items;
    std::vector<int> grp_first(NGRP, 0);
    for (int g = 0; g < NGRP; ++g) {
        grp_first[g] = (int)assign_items.size();
        assign_items.insert(assign_items.end(), grp_items[g].begin(), grp_items[g].end());
    }
    const int n_queues = NGRP + 2; // assignment groups, update, spare
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    DBuf<float> X, Cb0, Cb1, cn, sc;
    DBuf<int> lab, cnt, bad, queues;
    DBuf<int2> chg;
    DBuf<unsigned> colmax;
    DBuf<unsigned long long> acc;
    DBuf<double> inv, scratch, part, inert;
    DBuf<KbInst> inst;
    DBuf<KbItem> aitems, ditems, sitems;
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
    ok(lab.alloc(lo));
    ok(chg.alloc(lo));
    ok(cnt.alloc(no));
    ok(bad.alloc(1));
    ok(queues.alloc(n_queues));
    ok(colmax.alloc(so));
    ok(acc.alloc(ao));
    ok(inv.alloc(so));
    ok(scratch.alloc((size_t)n_inst * 2 * 32));
    ok(part.alloc(scan_items.size()));
    ok(inert.alloc(n_inst));
    ok(inst.alloc(n_inst));
    ok(aitems.alloc(assign_items.size()));
    ok(ditems.alloc(delta_items.size()));
    ok(sitems.alloc(scan_items.size()));
    if (e != cudaSuccess) {
        cudaGetLastError();
        return da_status_memory_error;
    }
    cudaEvent_t ev[6] = {};
    for (auto &x : ev) ok(cudaEventCreate(&x));
    ok(cudaEventRecord(ev[0], s));
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
        ok(cudaMemcpyAsync(inst.p, hi.data(), hi.size() * sizeof(KbInst), cudaMemcpyHostToDevice, s));
        ok(cudaMemcpyAsync(aitems.p, assign_items.data(), assign_items.size() * sizeof(KbItem),
                           cudaMemcpyHostToDevice, s));
        ok(cudaMemcpyAsync(ditems.p, delta_items.data(), delta_items.size() * sizeof(KbItem),
                           cudaMemcpyHostToDevice, s));
        ok(cudaMemcpyAsync(sitems.p, scan_items.data(), scan_items.size() * sizeof(KbItem),
                           cudaMemcpyHostToDevice, s));
    }
    ok(cudaEventRecord(ev[1], s));
    // state: no labels yet (every row is a change in the first iteration),
    // empty sums and counts
    ok(cudaMemsetAsync(Cb1.p, 0, co * sizeof(float), s));
    ok(cudaMemsetAsync(lab.p, 0xFF, lo * sizeof(int), s));
    ok(cudaMemsetAsync(acc.p, 0, ao * sizeof(unsigned long long), s));
    ok(cudaMemsetAsync(cnt.p, 0, no * sizeof(int), s));
    ok(cudaMemsetAsync(bad.p, 0, sizeof(int), s));
    ok(cudaMemsetAsync(colmax.p, 0, so * sizeof(unsigned), s));
    if (e != cudaSuccess) {
        cudaGetLastError();
        for (auto &x : ev)
            if (x) cudaEventDestroy(x);
        return da_status_internal_error;
    }
    kb_colmax<<<(unsigned)scan_items.size(), 256, (size_t)max_d * sizeof(unsigned), s>>>(
        X.p, inst.p, sitems.p, colmax.p, bad.p);
    kb_scales<<<n_inst, 128, 0, s>>>(inst.p, colmax.p, sc.p, inv.p);
    int h_bad = 0;
    ok(cudaGetLastError());
    ok(cudaMemcpyAsync(&h_bad, bad.p, sizeof(int), cudaMemcpyDeviceToHost, s));
    ok(cudaStreamSynchronize(s));
    auto cleanup_events = [&] {
        for (auto &x : ev)
            if (x) cudaEventDestroy(x);
    };
    if (e != cudaSuccess) {
        cudaGetLastError();
        cleanup_events();
        return da_status_internal_error;
    }
    if (h_bad) {
        cleanup_events();
        return da_status_invalid_input; // inf / NaN in the data
    }
    // kernel shapes: shared memory limits, resident blocks, the tuner's picks
    struct Launch {
        AssignFn fn;
        size_t smem;
        int grid, first, count, kmax, q;
    };
    std::vector<Launch> launches;
    for (int g = 0; g < NGRP; ++g)
        if (g / KB_NK < 4) grp_kmax[g] = (grp_kmax[g] + 63) / 64 * 64;
    for (int g = 0; g < NGRP && e == cudaSuccess; ++g) {
        if (grp_items[g].empty()) continue;
        const int wi = g / KB_NK, ki = g % KB_NK;
        const size_t smem = assign_smem(wi, grp_kmax[g], grp_dmax[g]);
        for (int gi = 0; gi < KB_NG; ++gi)
            ok(ensure_smem_limit(reinterpret_cast<const void *>(assign_fn(wi, gi)), smem));
        int pick = -1;
        {
            std::lock_guard<std::mutex> lk(g_tune_mu);
            auto f = g_tune.find(std::make_tuple(dev, wi, ki));
            if (f != g_tune.end()) pick = f->second;
        }
        if (pick < 0 && e == cudaSuccess) {
            // time every shape on (up to) the first 2,048 tiles of the group,
            // labels into the label buffer (reset below), twice each
            const int cnt_items = std::min<int>((int)grp_items[g].size(), 2048);
            float best_ms = 0.f;
            for (int gi = 0; gi < KB_NG && e == cudaSuccess; ++gi) {
                AssignFn fn = assign_fn(wi, gi);
                const int grid = std::min(cnt_items, resident_blocks(
                                                         reinterpret_cast<const void *>(fn), KB_T, smem));
                float ms = 0.f;
                for (int rep = 0; rep < 2 && e == cudaSuccess; ++rep) {
                    ok(cudaMemsetAsync(queues.p + NGRP + 1, 0, sizeof(int), s));
                    ok(cudaEventRecord(ev[4], s));
                    fn<<<grid, KB_T, smem, s>>>(X.p, inst.p, aitems.p + grp_first[g], cnt_items,
                                                queues.p + NGRP + 1, Cb0.p, Cb1.p, cn.p, lab.p,
                                                chg.p, 2, grp_kmax[g]);
                    ok(cudaGetLastError());
                    ok(cudaEventRecord(ev[5], s));
                    ok(cudaEventSynchronize(ev[5]));
                    if (e == cudaSuccess) ok(cudaEventElapsedTime(&ms, ev[4], ev[5]));
                }
                if (e == cudaSuccess && (pick < 0 || ms < best_ms)) {
                    pick = gi;
                    best_ms = ms;
                }
            }
            if (e == cudaSuccess) {
                std::lock_guard<std::mutex> lk(g_tune_mu);
                g_tune[std::make_tuple(dev, wi, ki)] = pick;
            }
        }
        if (e != cudaSuccess) break;
        AssignFn fn = assign_fn(wi, pick);
        const int n_it = (int)grp_items[g].size();
        const int grid = std::min(n_it, resident_blocks(reinterpret_cast<const void *>(fn), KB_T, smem));
        launches.push_back({fn, smem, grid, grp_first[g], n_it, grp_kmax[g], g});
    }
    // the tuner's runs wrote labels: back to "none"
    ok(cudaMemsetAsync(lab.p, 0xFF, lo * sizeof(int), s));
    const size_t dsmem = (size_t)max_kd * 8 + (size_t)max_k * 4 + (size_t)max_d * 4 + 16;
    ok(ensure_smem_limit(reinterpret_cast<const void *>(kb_delta), dsmem));
    const int dgrid = std::min<int>((int)delta_items.size(),
                                    resident_blocks(reinterpret_cast<const void *>(kb_delta), 256, dsmem));
    // The whole fit as one CUDA graph: max_iter iterations (finished
    // instances skip their work), the final relabelling and the inertia;
    // replayed once.
    // The assignment launches (one per tile shape) are parallel branches of
    // the graph: their persistent blocks share the device.
    cudaStream_t cs = nullptr;
    cudaGraph_t graph = nullptr;
    cudaGraphExec_t exec = nullptr;
    ok(cudaStreamCreateWithFlags(&cs, cudaStreamNonBlocking));
    std::vector<cudaStream_t> bs(launches.size(), nullptr);
    std::vector<cudaEvent_t> be(launches.size() + 1, nullptr);
    for (auto &x : bs) ok(cudaStreamCreateWithFlags(&x, cudaStreamNonBlocking));
    for (auto &x : be) ok(cudaEventCreateWithFlags(&x, cudaEventDisableTiming));
    auto assign_all = [&](int mode) {
        cudaEventRecord(be.back(), cs);
        for (size_t b = 0; b < launches.size(); ++b) {
            const Launch &l = launches[b];
            cudaStreamWaitEvent(bs[b], be.back(), 0);
            l.fn<<<l.grid, KB_T, l.smem, bs[b]>>>(X.p, inst.p, aitems.p + l.first, l.count,
                                                   queues.p + l.q, Cb0.p, Cb1.p, cn.p, lab.p,
                                                   chg.p, mode, l.kmax);
            cudaEventRecord(be[b], bs[b]);
            cudaStreamWaitEvent(cs, be[b], 0);
        }
    };
    if (e == cudaSuccess && ok(cudaStreamBeginCapture(cs, cudaStreamCaptureModeThreadLocal))) {
        for (da_int it = 0; it < max_iter; ++it) {
            kb_begin<<<n_inst, 128, 0, cs>>>(inst.p, Cb0.p, Cb1.p, cn.p, queues.p, n_queues);
            assign_all(0);
            kb_delta<<<dgrid, 256, dsmem, cs>>>(X.p, inst.p, ditems.p, (int)delta_items.size(),
                                                queues.p + NGRP, chg.p, sc.p, acc.p, cnt.p,
                                                max_kd, max_k);
            kb_finalize<<<n_inst, 256, 0, cs>>>(inst.p, Cb0.p, Cb1.p, acc.p, cnt.p, inv.p,
                                                (int)max_iter, tol, scratch.p);
        }
        kb_final_norms<<<n_inst, 128, 0, cs>>>(inst.p, Cb0.p, Cb1.p, cn.p);
        cudaMemsetAsync(queues.p, 0, n_queues * sizeof(int), cs);
        assign_all(1);
        kb_inertia_part<<<(unsigned)scan_items.size(), 256, 0, cs>>>(X.p, inst.p, sitems.p, Cb0.p,
                                                                      Cb1.p, lab.p, part.p);
        kb_inertia_sum<<<(n_inst + 127) / 128, 128, 0, cs>>>(inst.p, n_inst, part.p, inert.p);
        const cudaError_t ce = cudaStreamEndCapture(cs, &graph);
        ok(cudaGetLastError());
        ok(ce);
        if (e == cudaSuccess) ok(cudaGraphInstantiate(&exec, graph, 0));
    }
    // order the graph after the uploads on the caller's stream
    ok(cudaEventRecord(ev[4], s));
    ok(cudaStreamWaitEvent(cs, ev[4], 0));
    ok(cudaEventRecord(ev[2], cs));
    if (e == cudaSuccess) ok(cudaGraphLaunch(exec, cs));
    ok(cudaEventRecord(ev[3], cs));
    ok(cudaStreamSynchronize(cs));
    // results
    std::vector<KbInst> fin(n_inst);
    std::vector<double> hin(n_inst);
    ok(cudaMemcpy(fin.data(), inst.p, fin.size() * sizeof(KbInst), cudaMemcpyDeviceToHost));
    ok(cudaMemcpy(hin.data(), inert.p, hin.size() * sizeof(double), cudaMemcpyDeviceToHost));
    ok(cudaEventRecord(ev[4], cs));
    for (da_int i = 0; i < n_inst && e == cudaSuccess; ++i) {
        const KbInst &I = fin[i];
        ok(cudaMemcpy2DAsync(C_out[i], (size_t)I.d * 4, (I.fc ? Cb1.p : Cb0.p) + I.co,
                             (size_t)I.ld * 4, (size_t)I.d * 4, I.k, cudaMemcpyDeviceToHost, cs));
        ok(cudaMemcpyAsync(labels_out[i], lab.p + I.lo, (size_t)I.n * sizeof(int),
                           cudaMemcpyDeviceToHost, cs));
        n_iter[i] = I.n_iter;
        inertia[i] = hin[i];
        converged[i] = I.conv;
    }
    ok(cudaEventRecord(ev[5], cs));
    ok(cudaStreamSynchronize(cs));
    if (e == cudaSuccess) {
        float a = 0.f, b = 0.f, c = 0.f;
        cudaEventElapsedTime(&a, ev[0], ev[1]);
        cudaEventElapsedTime(&b, ev[2], ev[3]);
        cudaEventElapsedTime(&c, ev[4], ev[5]);
        g_last_ms[0] = a;
        g_last_ms[1] = b;
        g_last_ms[2] = c;
    }
    if (exec) cudaGraphExecDestroy(exec);
    if (graph) cudaGraphDestroy(graph);
    cleanup_events();
    for (auto &x : be)
        if (x) cudaEventDestroy(x);
    for (auto &x : bs)
        if (x) cudaStreamDestroy(x);
    if (cs) cudaStreamDestroy(cs);
    if (e != cudaSuccess) {
        cudaGetLastError();
        return da_status_internal_error;
    }
    return da_status_success;
}
