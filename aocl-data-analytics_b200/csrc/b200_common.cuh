// Common device-side helpers for the B200 distance / kNN / k-means kernels.
#pragma once
#include <cuda_runtime.h>
#include <stdint.h>
#include <math.h>
#include <float.h>
#include "b200_kernels.hpp"

#define B200_DEV __device__ __forceinline__

namespace b200 {

template <typename T> struct Lim;
template <> struct Lim<float> {
    static B200_DEV float inf() { return __int_as_float(0x7f800000); }
};
template <> struct Lim<double> {
    static B200_DEV double inf() { return __longlong_as_double(0x7ff0000000000000ULL); }
};

// Explicitly rounded arithmetic so that nvcc never contracts or reorders the
// operations whose rounding must match the reference CPU kernels.
B200_DEV float sub_rn(float a, float b) { return __fsub_rn(a, b); }
B200_DEV double sub_rn(double a, double b) { return __dsub_rn(a, b); }
B200_DEV float add_rn(float a, float b) { return __fadd_rn(a, b); }
B200_DEV double add_rn(double a, double b) { return __dadd_rn(a, b); }
B200_DEV float mul_rn(float a, float b) { return __fmul_rn(a, b); }
B200_DEV double mul_rn(double a, double b) { return __dmul_rn(a, b); }
B200_DEV float fma_rn(float a, float b, float c) { return __fmaf_rn(a, b, c); }
B200_DEV double fma_rn(double a, double b, double c) { return __fma_rn(a, b, c); }
B200_DEV float div_rn(float a, float b) { return __fdiv_rn(a, b); }
B200_DEV double div_rn(double a, double b) { return __ddiv_rn(a, b); }
B200_DEV float sqrt_rn(float a) { return __fsqrt_rn(a); }
B200_DEV double sqrt_rn(double a) { return __dsqrt_rn(a); }
B200_DEV float abs_(float a) { return fabsf(a); }
B200_DEV double abs_(double a) { return fabs(a); }

// Spherical k-means++ distance of row i to data row c (kmeans.cpp:1491-1510):
// max(0, 1 - cos) with cos = fl(fl(dot inv_i) inv_c) for normalised data
// (inv: inverse row norms), else cos = dot.  A NaN gives 0, as std::max(0, v).
template <typename T> B200_DEV T cos_dist_kpp(T dot, const T *inv, int i, int c) {
    const T cs = inv ? mul_rn(mul_rn(dot, inv[i]), inv[c]) : dot;
    const T v = sub_rn(T(1), cs);
    return T(0) < v ? v : T(0);
}
B200_DEV float pow_(float a, float p) { return powf(a, p); }
B200_DEV double pow_(double a, double p) { return pow(a, p); }

// Lexicographic (distance, index) order: ties go to the lower index.
template <typename T> B200_DEV bool key_less(T da, int ia, T db, int ib) {
    return (da < db) || (da == db && ia < ib);
}

} // namespace b200
