// Shared SIMT tile engine (CUDA cores) used by the distance, kNN and k-means
// kernels.  See dist_simt.cu for the accumulation-order contract.
#pragma once
#include "b200_common.cuh"

namespace b200 {

template <typename T> struct SimtCfg;
template <> struct SimtCfg<float> {
    static constexpr int TM = 4, TN = 8, BK = 16;
};
template <> struct SimtCfg<double> {
    static constexpr int TM = 4, TN = 4, BK = 16;
};

// Vector of 4 elements (16 B for fp32, 32 B for fp64).
template <typename T> struct V4 {
    T v[4];
};
template <typename T> B200_DEV V4<T> ld4_global(const T *p) {
    V4<T> r;
    if constexpr (sizeof(T) == 4) {
        float4 x = __ldg(reinterpret_cast<const float4 *>(p));
        r.v[0] = x.x; r.v[1] = x.y; r.v[2] = x.z; r.v[3] = x.w;
    } else {
        double2 x = __ldg(reinterpret_cast<const double2 *>(p));
        double2 y = __ldg(reinterpret_cast<const double2 *>(p) + 1);
        r.v[0] = x.x; r.v[1] = x.y; r.v[2] = y.x; r.v[3] = y.y;
    }
    return r;
}
template <typename T> B200_DEV V4<T> ld4_shared(const T *p) {
    V4<T> r;
    if constexpr (sizeof(T) == 4) {
        float4 x = *reinterpret_cast<const float4 *>(p);
        r.v[0] = x.x; r.v[1] = x.y; r.v[2] = x.z; r.v[3] = x.w;
    } else {
        double2 x = *reinterpret_cast<const double2 *>(p);
        double2 y = *(reinterpret_cast<const double2 *>(p) + 1);
        r.v[0] = x.x; r.v[1] = x.y; r.v[2] = y.x; r.v[3] = y.y;
    }
    return r;
}

// Shared-memory operand staging for one BK-dim slab.
template <typename T, int BM, int BN, int BK> struct Stage {
    T a[BK][BM + 4];
    T b[BK][BN + 4];
};

// Register prefetch of one slab of a (rows x BK) block of a row-major matrix.
template <typename T, int ROWS, int BK> struct SlabRegs {
    static constexpr int NV = ROWS * (BK / 4) / 256; // 4-vectors per thread
    V4<T> v[NV];
    B200_DEV void load(const T *M, int ld, int row0, int nrows, int k0, int tid) {
#pragma unroll
        for (int u = 0; u < NV; ++u) {
            int e = tid + u * 256;
            int r = e / (BK / 4);
            int kq = (e % (BK / 4)) * 4;
            int gr = row0 + r, gk = k0 + kq;
            if (gr < nrows && gk < ld) {
                v[u] = ld4_global(M + (size_t)gr * ld + gk);
            } else {
                v[u].v[0] = v[u].v[1] = v[u].v[2] = v[u].v[3] = T(0);
            }
        }
    }
    template <int S>
    B200_DEV void store(T (*dst)[S], int tid) const {
#pragma unroll
        for (int u = 0; u < NV; ++u) {
            int e = tid + u * 256;
            int r = e / (BK / 4);
            int kq = (e % (BK / 4)) * 4;
#pragma unroll
            for (int w = 0; w < 4; ++w) dst[kq + w][r] = v[u].v[w];
        }
    }
};

// Per-thread accumulator state.
template <typename T, int TM, int TN> struct Acc {
    T g1[TM][TN];
    T g2[TM][TN];
    B200_DEV void zero() {
#pragma unroll
        for (int i = 0; i < TM; ++i)
#pragma unroll
            for (int j = 0; j < TN; ++j) g1[i][j] = g2[i][j] = T(0);
    }
};

// Consume one shared-memory slab (dims k0 .. k0+BK-1) into the accumulators,
// following the reference's per-element order for the metric family.
template <typename T, int ACC, int TM, int TN, int BM, int BN, int BK>
B200_DEV void consume_slab(const Stage<T, BM, BN, BK> &st, int k0, int d, int d4, int kc,
                           T p, Acc<T, TM, TN> &acc, int tm, int tn) {
    constexpr int NG = TN / 4; // column groups of 4 at stride 64
#pragma unroll
    for (int grp = 0; grp < BK / 4; ++grp) {
        const int kg = k0 + 4 * grp;
        if (ACC == ACC_SQEUC) {
            if (kg + 4 <= d4) {
                V4<T> a[4], b[4][NG];
#pragma unroll
                for (int u = 0; u < 4; ++u) {
                    a[u] = ld4_shared(&st.a[4 * grp + u][tm * 4]);
#pragma unroll
                    for (int g = 0; g < NG; ++g)
                        b[u][g] = ld4_shared(&st.b[4 * grp + u][g * 64 + tn * 4]);
                }
#pragma unroll
                for (int i = 0; i < TM; ++i)
#pragma unroll
                    for (int j = 0; j < TN; ++j) {
                        const int g = j / 4, jj = j % 4;
                        T t0 = sub_rn(a[0].v[i], b[0][g].v[jj]);
                        T t1 = sub_rn(a[1].v[i], b[1][g].v[jj]);
                        T t2 = sub_rn(a[2].v[i], b[2][g].v[jj]);
                        T t3 = sub_rn(a[3].v[i], b[3][g].v[jj]);
                        acc.g1[i][j] = fma_rn(t0, t0, acc.g1[i][j]);
                        acc.g1[i][j] = fma_rn(t1, t1, acc.g1[i][j]);
                        acc.g2[i][j] = fma_rn(t2, t2, acc.g2[i][j]);
                        acc.g2[i][j] = fma_rn(t3, t3, acc.g2[i][j]);
                    }
                if (((kg + 4) % kc) == 0 || (kg + 4) == d4) {
#pragma unroll
                    for (int i = 0; i < TM; ++i)
#pragma unroll
                        for (int j = 0; j < TN; ++j) {
                            acc.g1[i][j] = add_rn(acc.g1[i][j], acc.g2[i][j]);
                            acc.g2[i][j] = T(0);
                        }
                }
            } else if (kg == d4 && kg < d) {
                // d % 4 remainder: sequential into g1 (2-way then 1-way in the
                // reference; both chain into the same accumulator in order).
                for (int u = 0; u < d - d4; ++u) {
                    V4<T> a = ld4_shared(&st.a[4 * grp + u][tm * 4]);
                    V4<T> b[NG];
#pragma unroll
                    for (int g = 0; g < NG; ++g)
                        b[g] = ld4_shared(&st.b[4 * grp + u][g * 64 + tn * 4]);
#pragma unroll
                    for (int i = 0; i < TM; ++i)
#pragma unroll
                        for (int j = 0; j < TN; ++j) {
                            T t = sub_rn(a.v[i], b[j / 4].v[j % 4]);
                            acc.g1[i][j] = fma_rn(t, t, acc.g1[i][j]);
                        }
                }
            }
        } else {
            const int nu = (kg + 4 <= d) ? 4 : (kg < d ? d - kg : 0);
            if (nu == 0) continue;
#pragma unroll
            for (int u = 0; u < 4; ++u) {
                if (u >= nu) break;
                V4<T> a = ld4_shared(&st.a[4 * grp + u][tm * 4]);
                V4<T> b[NG];
#pragma unroll
                for (int g = 0; g < NG; ++g)
                    b[g] = ld4_shared(&st.b[4 * grp + u][g * 64 + tn * 4]);
#pragma unroll
                for (int i = 0; i < TM; ++i)
#pragma unroll
                    for (int j = 0; j < TN; ++j) {
                        const T av = a.v[i], bv = b[j / 4].v[j % 4];
                        if (ACC == ACC_DOT) {
                            acc.g1[i][j] = fma_rn(av, bv, acc.g1[i][j]);
                        } else if (ACC == ACC_MANHATTAN) {
                            acc.g1[i][j] = add_rn(acc.g1[i][j], abs_(sub_rn(av, bv)));
                        } else {
                            acc.g1[i][j] = add_rn(acc.g1[i][j], pow_(abs_(sub_rn(av, bv)), p));
                        }
                    }
            }
        }
    }
}

// Full d-loop for one BM x BN tile: A rows (a_row0..) of A, B rows of B.
template <typename T, int ACC, int TM, int TN, int BM, int BN, int BK>
B200_DEV void compute_tile(Stage<T, BM, BN, BK> *st, const T *A, int lda, int na, int a_row0,
                           const T *B, int ldb, int nb, int b_row0, int d, int kc, T p,
                           Acc<T, TM, TN> &acc, int tid) {
    const int tm = tid / 16, tn = tid % 16;
    const int d4 = d & ~3;
    const int ld = lda; // both operands padded to the same width (pad4(d))
    (void)ldb;
    SlabRegs<T, BM, BK> ra;
    SlabRegs<T, BN, BK> rb;
    acc.zero();
    const int nslab = (d + BK - 1) / BK;
    ra.load(A, ld, a_row0, na, 0, tid);
    rb.load(B, ld, b_row0, nb, 0, tid);
    __syncthreads(); // previous users of st are done
    ra.store(st[0].a, tid);
    rb.store(st[0].b, tid);
    __syncthreads();
    for (int s = 0; s < nslab; ++s) {
        const int cur = s & 1;
        if (s + 1 < nslab) {
            ra.load(A, ld, a_row0, na, (s + 1) * BK, tid);
            rb.load(B, ld, b_row0, nb, (s + 1) * BK, tid);
        }
        consume_slab<T, ACC, TM, TN, BM, BN, BK>(st[cur], s * BK, d, d4, kc, p, acc, tm, tn);
        if (s + 1 < nslab) {
            ra.store(st[cur ^ 1].a, tid);
            rb.store(st[cur ^ 1].b, tid);
        }
        __syncthreads();
    }
}


} // namespace b200
