// Tensor-core (tcgen05) k-means assignment for sm_100a.
//
// S = X_bf16 * C_bf16^T is accumulated in fp32 in TMEM (128 rows per tile,
// N = all clusters, <= 256), fed by 128-byte-swizzled TMA tiles.  The epilogue
// forms v_j = |c_j|^2 - 2 s_j and keeps, per row, the smallest and the
// second-smallest v.  The label of the plain fp32 path is certified when the
// gap exceeds twice a rigorous bound on |v_bf16 - v_fp32|:
//   eps_i = 2 delta |x_i| cmax + 2^-23 (cmax^2 + 2 |x_i| cmax),
//   delta = 2^-7 (1 + 2^-7) + K 2^-21
// (bf16 rounding of both operands: |x~c~ - xc| <= 2^-7 |xc|; fp32 accumulation
// of the tensor core and of the plain path: K 2^-23 each; two fma roundings).
// Rows whose gap is not certified are appended to a list and relabelled by
// the exact fp32 kernel, so every label equals the plain path's label.
//
// Warp roles (320 threads): warp 0 TMA producer, warp 1 TMEM owner + MMA
// issuer, warps 2-9 two epilogue warpgroups (each owns one TMEM buffer and
// every other tile).
// Accumulators are double-buffered in TMEM so MMA of tile t+1 overlaps the
// epilogue of tile t.
#include "b200_common.cuh"
#include "b200_kernels.hpp"
#include "tc_common.cuh"
#include <cuda_bf16.h>

namespace b200 {

using namespace tc;

static constexpr int TC_BM = 128;       // rows per tile (UMMA M)
static constexpr int TC_KB = 64;        // bf16 elements per 128-byte K block
static constexpr int TC_THREADS = 320;  // 10 warps
static constexpr int TC_MAXC = 4;       // candidates kept per uncertified row

struct TcAssignArgs {
    int n, k, npad, nkb, stages, bufcols;
    const float *cnorm;  // k   (fp32, plain formula)
    const float *xnorm;  // n   (fp32 |x_i|)
    const float *cmax;   // 1   (max_j |c_j|)
    int *labels;
    const int *labels_prev;
    int *flags;          // [0] labels changed
    int *amb_rows;       // rows to relabel exactly
    int *amb_cand;       // TC_MAXC candidate clusters per listed row
    int *amb_ncand;      // number of candidates (0: scan every cluster)
    int *amb_count;
    int *err;            // set on a timed-out wait
    float delta;
};

struct __align__(16) TcShared {
    uint64_t full[8], empty[8], tfull[2], tempty[2], bfull;
    uint32_t tmem_base;
    int abort_flag;
    int changed;
};

__device__ __forceinline__ void raise(int *abort_flag, int *err, int code) {
    *((volatile int *)abort_flag) = 1;
    atomicExch(err, code);
}

__global__ void __launch_bounds__(TC_THREADS, 1)
kmeans_assign_tc_kernel(const __grid_constant__ CUtensorMap tmX,
                        const __grid_constant__ CUtensorMap tmC, TcAssignArgs a) {
    extern __shared__ __align__(1024) unsigned char smem_raw[];
    // 1024-byte alignment for the swizzled operand tiles
    unsigned char *base = reinterpret_cast<unsigned char *>(
        (reinterpret_cast<uintptr_t>(smem_raw) + 1023) & ~uintptr_t(1023));
    const int S = a.stages, nkb = a.nkb;
    const uint32_t b_bytes = (uint32_t)a.npad * 128u;       // one K block of C
    const uint32_t a_bytes = (uint32_t)TC_BM * 128u;        // one K block of a tile
    unsigned char *Bs = base;
    unsigned char *As = Bs + (size_t)nkb * b_bytes;
    TcShared *sh = reinterpret_cast<TcShared *>(As + (size_t)S * nkb * a_bytes);
    float *cn_s = reinterpret_cast<float *>(sh + 1);      // npad32 entries, +inf pad
    const int npad32 = (a.npad + 31) & ~31;
    int *cand_s = reinterpret_cast<int *>(cn_s + npad32); // [TC_THREADS][TC_MAXC]

    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const int ntiles = (a.n + TC_BM - 1) / TC_BM;

    if (threadIdx.x == 0) {
        for (int s = 0; s < S; ++s) {
            mbar_init(&sh->full[s], 1);
            mbar_init(&sh->empty[s], 1);
        }
        for (int b = 0; b < 2; ++b) {
            mbar_init(&sh->tfull[b], 1);
            mbar_init(&sh->tempty[b], 128);
        }
        mbar_init(&sh->bfull, 1);
        sh->abort_flag = 0;
        sh->changed = 0;
        fence_barrier_init();
    }
    for (int j = threadIdx.x; j < npad32; j += blockDim.x)
        cn_s[j] = j < a.k ? a.cnorm[j] : __int_as_float(0x7f800000);
    if (warp == 1) {
        tmem_alloc(&sh->tmem_base, 2u * a.bufcols);
        tmem_relinquish();
    }
    tc_fence_before();
    __syncthreads();
    tc_fence_after();
    const uint32_t tbase = sh->tmem_base;

    if (warp == 0) {
        // ------------------------------------------------ TMA producer ----
        if (lane == 0) {
            prefetch_tmap(&tmX);
            prefetch_tmap(&tmC);
            mbar_arrive_expect_tx(&sh->bfull, (uint32_t)nkb * b_bytes);
            for (int kb = 0; kb < nkb; ++kb)
                tma_load_2d(&tmC, &sh->bfull, Bs + (size_t)kb * b_bytes, kb * TC_KB, 0);
            int it = 0;
            for (int t = blockIdx.x; t < ntiles; t += gridDim.x, ++it) {
                const int s = it % S;
                const uint32_t ph = (uint32_t)((it / S) & 1);
                if (!mbar_wait(&sh->empty[s], ph ^ 1u)) {
                    raise(&sh->abort_flag, a.err, 1);
                    break;
                }
                if (*((volatile int *)&sh->abort_flag)) break;
                mbar_arrive_expect_tx(&sh->full[s], (uint32_t)nkb * a_bytes);
                for (int kb = 0; kb < nkb; ++kb)
                    tma_load_2d(&tmX, &sh->full[s], As + ((size_t)s * nkb + kb) * a_bytes,
                                kb * TC_KB, t * TC_BM);
            }
            // drain: every issued stage must have landed before exit
            const int issued = it;
            for (int u = (issued > S ? issued - S : 0); u < issued; ++u) {
                const int s = u % S;
                mbar_wait(&sh->full[s], (uint32_t)((u / S) & 1));
            }
        }
    } else if (warp == 1) {
        // ------------------------------------------------ MMA issuer ------
        if (lane == 0) {
            const uint32_t idesc = idesc_bf16_f32(TC_BM, a.npad);
            bool ok = mbar_wait(&sh->bfull, 0);
            if (!ok) raise(&sh->abort_flag, a.err, 2);
            int it = 0;
            for (int t = blockIdx.x; ok && t < ntiles; t += gridDim.x, ++it) {
                const int s = it % S, b = it & 1;
                if (!mbar_wait(&sh->tempty[b], (uint32_t)(((it >> 1) & 1) ^ 1))) {
                    raise(&sh->abort_flag, a.err, 3);
                    break;
                }
                if (!mbar_wait(&sh->full[s], (uint32_t)((it / S) & 1))) {
                    raise(&sh->abort_flag, a.err, 4);
                    break;
                }
                if (*((volatile int *)&sh->abort_flag)) break;
                tc_fence_after();
                const uint32_t tacc = tbase + (uint32_t)(b * a.bufcols);
                for (int kb = 0; kb < nkb; ++kb) {
                    const uint32_t abase = smem_u32(As + ((size_t)s * nkb + kb) * a_bytes);
                    const uint32_t bbase = smem_u32(Bs + (size_t)kb * b_bytes);
#pragma unroll
                    for (int kk = 0; kk < TC_KB / 16; ++kk)
                        mma_f16_ss(tacc, desc_k_sw128(abase + kk * 32), desc_k_sw128(bbase + kk * 32),
                                   idesc, (kb | kk) != 0);
                }
                mma_commit(&sh->empty[s]);
                mma_commit(&sh->tfull[b]);
            }
            // the accumulators of the last tiles must be complete before the
            // TMEM is released (returns at once when they were consumed)
            for (int u = (it > 2 ? it - 2 : 0); u < it; ++u)
                mbar_wait(&sh->tfull[u & 1], (uint32_t)((u >> 1) & 1));
        }
    } else {
        // ------------------------------------------------ epilogue --------
        // Group g (warps 2-5 / 6-9) owns TMEM buffer g and the local tiles
        // it = g, g+2, ...; each thread owns one row (its TMEM lane) and scans
        // all clusters.  The groups never wait on each other.
        const int g = (warp - 2) / 4;
        const int q = warp & 3;            // TMEM lane quarter of this warp
        const int row_in_tile = q * 32 + lane;
        const int nchunks = (a.npad + 31) / 32;
        const float cmax = *a.cmax;
        int changed = 0;
        int it = g;
        for (int t = blockIdx.x + g * gridDim.x; t < ntiles; t += 2 * gridDim.x, it += 2) {
            const int b = g;
            if (!mbar_wait(&sh->tfull[b], (uint32_t)((it >> 1) & 1))) {
                raise(&sh->abort_flag, a.err, 5);
                break;
            }
            if (*((volatile int *)&sh->abort_flag)) break;
            tc_fence_after();
            const uint32_t trow = tbase + ((uint32_t)(q * 32) << 16) + (uint32_t)(b * a.bufcols);
            const int r = t * TC_BM + row_in_tile;
            const float xn = r < a.n ? a.xnorm[r] : 0.f;
            // pass 1: smallest v_j = |c_j|^2 - 2 s_j (tree minimum per 32 columns)
            float b1 = __int_as_float(0x7f800000);
            for (int c = 0; c < nchunks; ++c) {
                float v[32];
                tmem_ld32(trow + (uint32_t)(c * 32), v);
                const float4 *cn4 = reinterpret_cast<const float4 *>(cn_s + c * 32);
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const float4 cc = cn4[u];
                    v[4 * u + 0] = __fmaf_rn(-2.f, v[4 * u + 0], cc.x);
                    v[4 * u + 1] = __fmaf_rn(-2.f, v[4 * u + 1], cc.y);
                    v[4 * u + 2] = __fmaf_rn(-2.f, v[4 * u + 2], cc.z);
                    v[4 * u + 3] = __fmaf_rn(-2.f, v[4 * u + 3], cc.w);
                }
#pragma unroll
                for (int w = 16; w >= 1; w >>= 1)
#pragma unroll
                    for (int u = 0; u < w; ++u) v[u] = fminf(v[u], v[u + w]);
                b1 = fminf(b1, v[0]);
            }
            // pass 2: every cluster within 2 eps of the minimum is a candidate
            const float eps = 1.01f * (2.f * a.delta * xn * cmax +
                                       1.1920929e-7f * (cmax * cmax + 2.f * xn * cmax));
            const float tau = b1 + 2.f * eps;
            int cnt = 0;
            int *my = cand_s + threadIdx.x * TC_MAXC;
            for (int c = 0; c < nchunks; ++c) {
                float v[32];
                tmem_ld32(trow + (uint32_t)(c * 32), v);
                const float4 *cn4 = reinterpret_cast<const float4 *>(cn_s + c * 32);
#pragma unroll
                for (int u = 0; u < 8; ++u) {
                    const float4 cc = cn4[u];
                    const float w4[4] = {__fmaf_rn(-2.f, v[4 * u + 0], cc.x),
                                         __fmaf_rn(-2.f, v[4 * u + 1], cc.y),
                                         __fmaf_rn(-2.f, v[4 * u + 2], cc.z),
                                         __fmaf_rn(-2.f, v[4 * u + 3], cc.w)};
#pragma unroll
                    for (int e = 0; e < 4; ++e) {
                        const int j = c * 32 + 4 * u + e;
                        if (w4[e] <= tau && j < a.k) { // padded columns are never candidates
                            if (cnt < TC_MAXC) my[cnt] = j;
                            ++cnt;
                        }
                    }
                }
            }
            tc_fence_before();
            mbar_arrive(&sh->tempty[b]);
            const bool valid = r < a.n;
            if (valid && cnt == 1) {
                // a single candidate: the fp32 label is certified
                const int lbl = my[0];
                a.labels[r] = lbl;
                if (a.labels_prev && a.labels_prev[r] != lbl) changed = 1;
            }
            // near-ties (or NaN): appended, one atomic per warp, for the exact
            // fp32 re-score of their candidates
            const bool amb = valid && cnt != 1;
            const unsigned mask = __ballot_sync(0xffffffffu, amb);
            if (mask) {
                int base0 = 0;
                if (lane == 0) base0 = atomicAdd(a.amb_count, __popc(mask));
                base0 = __shfl_sync(0xffffffffu, base0, 0);
                if (amb) {
                    const int pos = base0 + __popc(mask & ((1u << lane) - 1u));
                    a.amb_rows[pos] = r;
                    const int nc = (cnt >= 2 && cnt <= TC_MAXC) ? cnt : 0;
                    a.amb_ncand[pos] = nc;
                    for (int e = 0; e < nc; ++e) a.amb_cand[pos * TC_MAXC + e] = my[e];
                }
            }
        }
        if (changed) sh->changed = 1;
    }
    tc_fence_before();
    __syncthreads();
    if (threadIdx.x == 0 && sh->changed && a.flags) atomicOr(&a.flags[0], 1);
    if (warp == 1) {
        tc_fence_after();
        tmem_dealloc(tbase, 2u * a.bufcols);
    }
}

// Exact fp32 relabelling of the uncertified rows: the plain path's formula
// fl(|c|^2 - 2 x.c) with the dot product as one fma chain over the features,
// evaluated for the listed candidates (every cluster when the list
// overflowed); ties -> lower index.  Each warp stages the centres and 32
// listed rows in shared memory (coalesced loads, rows padded to d+1 floats so
// the per-lane sequential dot products are bank-conflict free); one lane per
// listed row.
__global__ void __launch_bounds__(256)
kmeans_rescore_kernel(const float *X, int ld, int d, const float *C, int k,
                      const float *cnorm, const int *amb_rows, const int *amb_cand,
                      const int *amb_ncand, const int *amb_count, int *labels,
                      const int *labels_prev, int *flags, int c_in_smem) {
    extern __shared__ float rs_smem[];
    const int dp = d + 1;
    float *cs = rs_smem;                                            // k x dp (optional)
    float *xs = rs_smem + (c_in_smem ? (size_t)k * dp : 0) + (threadIdx.x >> 5) * 32 * dp;
    const int lane = threadIdx.x & 31;
    const int cnt = *amb_count;
    if (c_in_smem) {
        for (int e = threadIdx.x; e < k * d; e += blockDim.x) {
            const int j = e / d, f = e % d;
            cs[j * dp + f] = C[(size_t)j * ld + f];
        }
        __syncthreads();
    }
    int changed = 0;
    const int warps_total = (gridDim.x * blockDim.x) >> 5;
    for (int e0 = ((blockIdx.x * blockDim.x + threadIdx.x) >> 5) * 32; e0 < cnt;
         e0 += warps_total * 32) {
        const int ne = min(32, cnt - e0);
        // coalesced staging of the (up to) 32 listed rows
        for (int i = 0; i < ne; ++i) {
            const float *x = X + (size_t)amb_rows[e0 + i] * ld;
            for (int f = lane; f < d; f += 32) xs[i * dp + f] = x[f];
        }
        __syncwarp();
        if (lane < ne) {
            const int e = e0 + lane;
            const int r = amb_rows[e];
            const float *x = xs + lane * dp;
            const int nc = amb_ncand[e];
            float best = __int_as_float(0x7f800000);
            int bi = 0x7fffffff;
            const int m = nc > 0 ? nc : k;
            for (int u = 0; u < m; ++u) {
                const int j = nc > 0 ? amb_cand[e * TC_MAXC + u] : u;
                float sdot = 0.f;
                if (c_in_smem) {
                    const float *c = cs + j * dp;
                    for (int f = 0; f < d; ++f) sdot = __fmaf_rn(x[f], c[f], sdot);
                } else {
                    const float *c = C + (size_t)j * ld;
                    for (int f = 0; f < d; ++f) sdot = __fmaf_rn(x[f], c[f], sdot);
                }
                const float v = __fmaf_rn(-2.f, sdot, cnorm[j]);
                if (key_less(v, j, best, bi)) {
                    best = v;
                    bi = j;
                }
            }
            const int lbl = (bi == 0x7fffffff) ? 0 : bi;
            labels[r] = lbl;
            if (labels_prev && labels_prev[r] != lbl) changed = 1;
        }
        __syncwarp();
    }
    if (changed && flags) atomicOr(&flags[0], 1);
}

// fp32 (row-major, ld) -> bf16 (row-major, ldo = nkb*64), zero padded.
__global__ void to_bf16_kernel(const float *X, int ld, int rows, int d, __nv_bfloat16 *Y, int ldo) {
    const size_t e = (size_t)blockIdx.x * blockDim.x + threadIdx.x;
    const size_t total = (size_t)rows * ldo;
    if (e >= total) return;
    const int r = (int)(e / ldo), c = (int)(e % ldo);
    Y[e] = __float2bfloat16_rn((c < d) ? X[(size_t)r * ld + c] : 0.f);
}
// |x_i| (fp32 sqrt of the fma-chain squared norm) and, optionally, the max.
__global__ void row_norm_max_kernel(const float *X, int ld, int rows, int d, float *out,
                                    float *maxv) {
    const int i = blockIdx.x * blockDim.x + threadIdx.x;
    float v = 0.f;
    if (i < rows) {
        const float *x = X + (size_t)i * ld;
        float s = 0.f;
        for (int j = 0; j < d; ++j) s = __fmaf_rn(x[j], x[j], s);
        v = __fsqrt_rn(s);
        out[i] = v;
    }
    if (maxv) {
#pragma unroll
        for (int off = 16; off > 0; off >>= 1) v = fmaxf(v, __shfl_xor_sync(0xffffffffu, v, off));
        if ((threadIdx.x & 31) == 0) atomicMax(reinterpret_cast<int *>(maxv), __float_as_int(v));
    }
}

// ------------------------------------------------------------- host side --
typedef CUresult (*EncodeTiledFn)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *,
                                  const cuuint64_t *, const cuuint64_t *, const cuuint32_t *,
                                  const cuuint32_t *, CUtensorMapInterleave, CUtensorMapSwizzle,
                                  CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn get_encode() {
    static EncodeTiledFn fn = nullptr;
    if (!fn) {
        void *p = nullptr;
        cudaDriverEntryPointQueryResult q;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) ==
                cudaSuccess &&
            q == cudaDriverEntryPointSuccess)
            fn = reinterpret_cast<EncodeTiledFn>(p);
    }
    return fn;
}

// 2-D bf16 tensor map over a row-major [rows x cols] matrix, box {64, box_rows},
// 128-byte swizzle, zero fill out of bounds.
static bool make_map_bf16(CUtensorMap *m, const void *ptr, int rows, int cols, int box_rows) {
    EncodeTiledFn enc = get_encode();
    if (!enc) return false;
    cuuint64_t dims[2] = {(cuuint64_t)cols, (cuuint64_t)rows};
    cuuint64_t strides[1] = {(cuuint64_t)cols * 2};
    cuuint32_t box[2] = {(cuuint32_t)TC_KB, (cuuint32_t)box_rows};
    cuuint32_t estr[2] = {1, 1};
    return enc(m, CU_TENSOR_MAP_DATA_TYPE_BFLOAT16, 2, const_cast<void *>(ptr), dims, strides, box,
               estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_128B,
               CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE) ==
           CUDA_SUCCESS;
}

int tc_assign_supported(int k, int d) {
    if (k < 1 || k > 256) return 0;
    const int nkb = (d + TC_KB - 1) / TC_KB;
    const int npad = (k + 15) & ~15;
    const size_t need = (size_t)nkb * npad * 128 + 2 * (size_t)nkb * TC_BM * 128 + 4096;
    return need <= 200 * 1024 ? 1 : 0;
}

cudaError_t launch_to_bf16(const float *X, int ld, int rows, int d, void *Y, int ldo,
                           cudaStream_t s) {
    const size_t total = (size_t)rows * ldo;
    to_bf16_kernel<<<(unsigned)((total + 255) / 256), 256, 0, s>>>(
        X, ld, rows, d, reinterpret_cast<__nv_bfloat16 *>(Y), ldo);
    return cudaGetLastError();
}

cudaError_t launch_row_norm_max(const float *X, int ld, int rows, int d, float *out, float *maxv,
                                cudaStream_t s) {
    if (maxv) {
        cudaError_t e = cudaMemsetAsync(maxv, 0, sizeof(float), s);
        if (e != cudaSuccess) return e;
    }
    row_norm_max_kernel<<<(rows + 255) / 256, 256, 0, s>>>(X, ld, rows, d, out, maxv);
    return cudaGetLastError();
}

cudaError_t launch_kmeans_assign_tc(const void *Xbf, int n, int ldbf, const void *Cbf, int k,
                                    const float *cnorm, const float *xnorm, const float *cmax,
                                    int *labels, const int *labels_prev, int *flags,
                                    int *amb_rows, int *amb_cand, int *amb_ncand, int *amb_count,
                                    int *err, cudaStream_t s) {
    const int nkb = ldbf / TC_KB;
    const int npad = (k + 15) & ~15;
    CUtensorMap mx, mc;
    if (!make_map_bf16(&mx, Xbf, n, ldbf, TC_BM) || !make_map_bf16(&mc, Cbf, npad, ldbf, npad))
        return cudaErrorInvalidValue;
    const size_t b_bytes = (size_t)nkb * npad * 128;
    const size_t a_stage = (size_t)nkb * TC_BM * 128;
    int stages = (int)((150 * 1024 - b_bytes) / a_stage);
    stages = stages < 2 ? 2 : (stages > 6 ? 6 : stages);
    const size_t smem = 1024 + b_bytes + stages * a_stage + sizeof(TcShared) +
                        (size_t)((npad + 31) & ~31) * 4 + TC_THREADS * TC_MAXC * 4 + 64;
    int bufcols = 32;
    while (bufcols < npad) bufcols <<= 1;
    TcAssignArgs a;
    a.n = n;
    a.k = k;
    a.npad = npad;
    a.nkb = nkb;
    a.stages = stages;
    a.bufcols = bufcols;
    a.cnorm = cnorm;
    a.xnorm = xnorm;
    a.cmax = cmax;
    a.labels = labels;
    a.labels_prev = labels_prev;
    a.flags = flags;
    a.amb_rows = amb_rows;
    a.amb_cand = amb_cand;
    a.amb_ncand = amb_ncand;
    a.amb_count = amb_count;
    a.err = err;
    a.delta = 0.0078125f * (1.f + 0.0078125f) + (float)(nkb * TC_KB) * 4.76837158e-7f;
    cudaError_t e = cudaFuncSetAttribute(kmeans_assign_tc_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int ntiles = (n + TC_BM - 1) / TC_BM;
    int nsm = 148;
    cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, 0);
    const int grid = ntiles < nsm ? ntiles : nsm;
    kmeans_assign_tc_kernel<<<grid, TC_THREADS, smem, s>>>(mx, mc, a);
    return cudaGetLastError();
}

cudaError_t launch_kmeans_rescore(const float *X, int ld, int d, const float *C, int k,
                                  const float *cnorm, const int *amb_rows, const int *amb_cand,
                                  const int *amb_ncand, const int *amb_count, int max_rows,
                                  int *labels, const int *labels_prev, int *flags,
                                  cudaStream_t s) {
    if (max_rows <= 0) return cudaSuccess;
    const size_t xs_bytes = (size_t)8 * 32 * (d + 1) * 4;
    const size_t cs_bytes = (size_t)k * (d + 1) * 4;
    const int c_in_smem = (cs_bytes + xs_bytes <= 200 * 1024) ? 1 : 0;
    const size_t smem = xs_bytes + (c_in_smem ? cs_bytes : 0);
    if (smem > 220 * 1024) return cudaErrorInvalidValue;
    cudaError_t e = cudaFuncSetAttribute(kmeans_rescore_kernel,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return e;
    const int blocks = min(148 * 2, (max_rows + 255) / 256);
    kmeans_rescore_kernel<<<blocks, 256, smem, s>>>(X, ld, d, C, k, cnorm, amb_rows, amb_cand,
                                                    amb_ncand, amb_count, labels, labels_prev,
                                                    flags, c_in_smem);
    return cudaGetLastError();
}

} // namespace b200

namespace b200 {
// The epilogue reads |c_j|^2 as float4 right after the barrier block.
static_assert(sizeof(TcShared) % 16 == 0, "TcShared must keep the cnorm array 16-byte aligned");
} // namespace b200
