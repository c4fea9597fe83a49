// Forward-mode dual numbers for the adjoint kernels: a value and its
// derivatives with respect to N seeded inputs, FP64. Comparisons act on the
// value, so min/max and every branch take the active piece and differentiate
// it (the HLL wave-speed switches are handled piecewise).
#pragma once
#include <cuda_runtime.h>

namespace rb200 {

// the real-number overloads stay visible next to the dual ones below
using ::fabs;
using ::isfinite;
using ::sqrt;

template <int N> struct Dual {
    double v;
    double d[N];
    __device__ __forceinline__ Dual() {}
    __device__ __forceinline__ Dual(double x) : v(x) {
#pragma unroll
        for (int i = 0; i < N; ++i) d[i] = 0;
    }
    // the seeded input i of value x
    __device__ __forceinline__ static Dual seed(double x, int i) {
        Dual r(x);
        if (i >= 0 && i < N) r.d[i] = 1;
        return r;
    }
};

template <int N> __device__ __forceinline__ Dual<N> operator+(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v + b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator-(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v - b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator-(const Dual<N>& a) {
    Dual<N> r;
    r.v = -a.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator*(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    r.v = a.v * b.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> operator/(const Dual<N>& a, const Dual<N>& b) {
    Dual<N> r;
    const double inv = 1 / b.v;
    r.v = a.v * inv;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * inv;
    return r;
}
template <int N> __device__ __forceinline__ Dual<N>& operator+=(Dual<N>& a, const Dual<N>& b) { return a = a + b; }
template <int N> __device__ __forceinline__ Dual<N>& operator-=(Dual<N>& a, const Dual<N>& b) { return a = a - b; }
template <int N> __device__ __forceinline__ Dual<N>& operator*=(Dual<N>& a, const Dual<N>& b) { return a = a * b; }
template <int N> __device__ __forceinline__ bool operator<(const Dual<N>& a, const Dual<N>& b) { return a.v < b.v; }
template <int N> __device__ __forceinline__ bool operator>(const Dual<N>& a, const Dual<N>& b) { return a.v > b.v; }
template <int N> __device__ __forceinline__ bool operator<=(const Dual<N>& a, const Dual<N>& b) { return a.v <= b.v; }
template <int N> __device__ __forceinline__ bool operator>=(const Dual<N>& a, const Dual<N>& b) { return a.v >= b.v; }
template <int N> __device__ __forceinline__ bool operator==(const Dual<N>& a, const Dual<N>& b) { return a.v == b.v; }
template <int N> __device__ __forceinline__ bool operator!=(const Dual<N>& a, const Dual<N>& b) { return a.v != b.v; }
template <int N> __device__ __forceinline__ bool isfinite(const Dual<N>& a) { return ::isfinite(a.v); }
template <int N> __device__ __forceinline__ Dual<N> sqrt(const Dual<N>& a) {
    Dual<N> r;
    r.v = ::sqrt(a.v);
    const double s = .5 / r.v;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * s;
    return r;
}
template <int N> __device__ __forceinline__ Dual<N> fabs(const Dual<N>& a) { return a.v < 0 ? -a : a; }

// Value of a real or dual number.
__device__ __forceinline__ double valueOf(double x) { return x; }
__device__ __forceinline__ float valueOf(float x) { return x; }
template <int N> __device__ __forceinline__ double valueOf(const Dual<N>& x) { return x.v; }

}  // namespace rb200
