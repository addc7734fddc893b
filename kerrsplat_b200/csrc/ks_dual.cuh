// ks_dual.cuh -- forward-mode dual numbers for the adjoint kernels.
//
// Dual<T, N> carries a value and N partials in scalar type T (double on the FP64 path, float on
// the mixed path). The transport functions are templates in their scalar type, so instantiating
// them with a Dual gives the derivatives the reference takes with ForwardDiff duals in its dual
// sweep (src/Splats/dual_gradient.jl:1-19, src/Transfer/transport.jl:221-245): seven partials
// through the step operator and seven through a splat's fluid rows. Branches compare values only,
// as ForwardDiff does.
#pragma once
#include <type_traits>

namespace ks {

template <class T, int N>
struct Dual {
    T v;
    T d[N];
    __host__ __device__ Dual() {}
    __host__ __device__ Dual(T x) : v(x) {
#pragma unroll
        for (int i = 0; i < N; ++i) d[i] = T(0);
    }
    template <class U, class = typename std::enable_if<std::is_arithmetic<U>::value && !std::is_same<U, T>::value>::type>
    __host__ __device__ Dual(U x) : v(T(x)) {
#pragma unroll
        for (int i = 0; i < N; ++i) d[i] = T(0);
    }
    // value x seeded in partial k with unit derivative
    __host__ __device__ static Dual seed(T x, int k) {
        Dual r(x);
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = (i == k) ? T(1) : T(0);
        return r;
    }
    __host__ __device__ Dual& operator+=(const Dual& b) { v += b.v;
#pragma unroll
        for (int i = 0; i < N; ++i) d[i] += b.d[i];
        return *this; }
    __host__ __device__ Dual& operator-=(const Dual& b) { v -= b.v;
#pragma unroll
        for (int i = 0; i < N; ++i) d[i] -= b.d[i];
        return *this; }
    __host__ __device__ Dual& operator*=(const Dual& b) { *this = *this * b; return *this; }
    __host__ __device__ Dual& operator/=(const Dual& b) { *this = *this / b; return *this; }

    friend __host__ __device__ Dual operator+(const Dual& a, const Dual& b) { Dual r; r.v = a.v + b.v;
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = a.d[i] + b.d[i];
        return r; }
    friend __host__ __device__ Dual operator-(const Dual& a, const Dual& b) { Dual r; r.v = a.v - b.v;
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = a.d[i] - b.d[i];
        return r; }
    friend __host__ __device__ Dual operator-(const Dual& a) { Dual r; r.v = -a.v;
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = -a.d[i];
        return r; }
    friend __host__ __device__ Dual operator*(const Dual& a, const Dual& b) { Dual r; r.v = a.v * b.v;
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b.v + a.v * b.d[i];
        return r; }
    friend __host__ __device__ Dual operator/(const Dual& a, const Dual& b) { Dual r; const T ib = T(1) / b.v; r.v = a.v * ib;
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = (a.d[i] - r.v * b.d[i]) * ib;
        return r; }
    // with the scalar type
    friend __host__ __device__ Dual operator+(const Dual& a, T b) { Dual r = a; r.v += b; return r; }
    friend __host__ __device__ Dual operator+(T a, const Dual& b) { Dual r = b; r.v += a; return r; }
    friend __host__ __device__ Dual operator-(const Dual& a, T b) { Dual r = a; r.v -= b; return r; }
    friend __host__ __device__ Dual operator-(T a, const Dual& b) { Dual r = -b; r.v += a; return r; }
    friend __host__ __device__ Dual operator*(const Dual& a, T b) { Dual r; r.v = a.v * b;
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = a.d[i] * b;
        return r; }
    friend __host__ __device__ Dual operator*(T a, const Dual& b) { return b * a; }
    friend __host__ __device__ Dual operator/(const Dual& a, T b) { return a * (T(1) / b); }
    friend __host__ __device__ Dual operator/(T a, const Dual& b) { Dual r; const T ib = T(1) / b.v; r.v = a * ib; const T f = -r.v * ib;
#pragma unroll
        for (int i = 0; i < N; ++i) r.d[i] = b.d[i] * f;
        return r; }
    // comparisons by value
    friend __host__ __device__ bool operator<(const Dual& a, const Dual& b) { return a.v < b.v; }
    friend __host__ __device__ bool operator>(const Dual& a, const Dual& b) { return a.v > b.v; }
    friend __host__ __device__ bool operator<=(const Dual& a, const Dual& b) { return a.v <= b.v; }
    friend __host__ __device__ bool operator>=(const Dual& a, const Dual& b) { return a.v >= b.v; }
    friend __host__ __device__ bool operator==(const Dual& a, const Dual& b) { return a.v == b.v; }
    friend __host__ __device__ bool operator!=(const Dual& a, const Dual& b) { return a.v != b.v; }
    friend __host__ __device__ bool operator<(const Dual& a, T b) { return a.v < b; }
    friend __host__ __device__ bool operator>(const Dual& a, T b) { return a.v > b; }
    friend __host__ __device__ bool operator<=(const Dual& a, T b) { return a.v <= b; }
    friend __host__ __device__ bool operator>=(const Dual& a, T b) { return a.v >= b; }
    friend __host__ __device__ bool operator==(const Dual& a, T b) { return a.v == b; }
    friend __host__ __device__ bool operator!=(const Dual& a, T b) { return a.v != b; }
    friend __host__ __device__ bool operator<(T a, const Dual& b) { return a < b.v; }
    friend __host__ __device__ bool operator>(T a, const Dual& b) { return a > b.v; }
};

// the scalar type of a (possibly dual) type
template <class T> struct ScalarOf { using type = T; };
template <class T, int N> struct ScalarOf<Dual<T, N>> { using type = T; };
template <class T> using scalar_t = typename ScalarOf<T>::type;
template <class T> constexpr bool is_f32 = std::is_same<scalar_t<T>, float>::value;
template <class T> __device__ __forceinline__ scalar_t<T> value_of(const T& x) { return x; }
template <class T, int N> __device__ __forceinline__ T value_of(const Dual<T, N>& x) { return x.v; }

}  // namespace ks

// The math functions of a dual live in the global namespace beside the CUDA float/double overloads:
// declared inside namespace ks they would hide those overloads from the code of that namespace.
// chain rule: f(x) with f'(x) = df
template <class T, int N>
__device__ __forceinline__ ks::Dual<T, N> dchain(const ks::Dual<T, N>& x, T f, T df) {
    ks::Dual<T, N> r;
    r.v = f;
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = x.d[i] * df;
    return r;
}

// sqrt with a zero derivative at 0 (a clamped argument: sqrt(fmax(x, 0)), R_F's sqrt(0) of a constant)
template <class T, int N> __device__ __forceinline__ ks::Dual<T, N> sqrt(const ks::Dual<T, N>& x) {
    const T s = sqrt(x.v);
    return dchain(x, s, s > T(0) ? T(0.5) / s : T(0));
}
template <class T, int N> __device__ __forceinline__ ks::Dual<T, N> exp(const ks::Dual<T, N>& x) { T e = exp(x.v); return dchain(x, e, e); }
template <class T, int N> __device__ __forceinline__ ks::Dual<T, N> expm1(const ks::Dual<T, N>& x) { return dchain(x, expm1(x.v), exp(x.v)); }
template <class T, int N> __device__ __forceinline__ ks::Dual<T, N> log(const ks::Dual<T, N>& x) { return dchain(x, log(x.v), T(1) / x.v); }
template <class T, int N> __device__ __forceinline__ ks::Dual<T, N> sin(const ks::Dual<T, N>& x) { T s, c; sincos(x.v, &s, &c); return dchain(x, s, c); }
template <class T, int N> __device__ __forceinline__ ks::Dual<T, N> cos(const ks::Dual<T, N>& x) { T s, c; sincos(x.v, &s, &c); return dchain(x, c, -s); }
template <class T, int N> __device__ __forceinline__ ks::Dual<T, N> sinh(const ks::Dual<T, N>& x) { return dchain(x, sinh(x.v), cosh(x.v)); }
template <class T, int N> __device__ __forceinline__ ks::Dual<T, N> cosh(const ks::Dual<T, N>& x) { return dchain(x, cosh(x.v), sinh(x.v)); }
template <class T, int N> __device__ __forceinline__ ks::Dual<T, N> tanh(const ks::Dual<T, N>& x) { T t = tanh(x.v); return dchain(x, t, T(1) - t * t); }
template <class T, int N> __device__ __forceinline__ ks::Dual<T, N> fabs(const ks::Dual<T, N>& x) { return x.v < T(0) ? -x : x; }
template <class T, int N> __device__ __forceinline__ ks::Dual<T, N> fmin(const ks::Dual<T, N>& a, const ks::Dual<T, N>& b) { return b.v < a.v ? b : a; }
template <class T, int N> __device__ __forceinline__ ks::Dual<T, N> fmax(const ks::Dual<T, N>& a, const ks::Dual<T, N>& b) { return b.v > a.v ? b : a; }
template <class T, int N> __device__ __forceinline__ ks::Dual<T, N> fma(const ks::Dual<T, N>& a, const ks::Dual<T, N>& b, const ks::Dual<T, N>& c) { return a * b + c; }
template <class T, int N> __device__ __forceinline__ bool isfinite(const ks::Dual<T, N>& x) { return isfinite(x.v); }
template <class T, int N>
__device__ __forceinline__ ks::Dual<T, N> atan2(const ks::Dual<T, N>& y, const ks::Dual<T, N>& x) {
    ks::Dual<T, N> r;
    r.v = atan2(y.v, x.v);
    const T den = x.v * x.v + y.v * y.v;
    const T fx = den > T(0) ? -y.v / den : T(0), fy = den > T(0) ? x.v / den : T(0);
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = fy * y.d[i] + fx * x.d[i];
    return r;
}
// asin with a zero derivative where the argument reaches +-1 (a clamped argument)
template <class T, int N> __device__ __forceinline__ ks::Dual<T, N> asin(const ks::Dual<T, N>& x) {
    const T s = T(1) - x.v * x.v;
    return dchain(x, asin(x.v), s > T(0) ? T(1) / sqrt(s) : T(0));
}
// acos with a zero derivative where the argument reaches +-1 (safe_acos, step.jl:157-172)
template <class T, int N> __device__ __forceinline__ ks::Dual<T, N> acos(const ks::Dual<T, N>& x) {
    const T s = T(1) - x.v * x.v;
    return dchain(x, acos(x.v), s > T(0) ? -T(1) / sqrt(s) : T(0));
}
template <class T, int N> __device__ __forceinline__ ks::Dual<T, N> atan(const ks::Dual<T, N>& x) { return dchain(x, atan(x.v), T(1) / (T(1) + x.v * x.v)); }
template <class T, int N> __device__ __forceinline__ ks::Dual<T, N> cbrt(const ks::Dual<T, N>& x) {
    const T c = cbrt(x.v);
    return dchain(x, c, c != T(0) ? T(1) / (T(3) * c * c) : T(0));
}
template <class T, int N> __device__ __forceinline__ ks::Dual<T, N> hypot(const ks::Dual<T, N>& x, const ks::Dual<T, N>& y) { return sqrt(x * x + y * y); }
template <class T, int N> __device__ __forceinline__ ks::Dual<T, N> copysign(const ks::Dual<T, N>& x, const ks::Dual<T, N>& y) {
    return (signbit(x.v) != signbit(y.v)) ? -x : x;
}
// piecewise constant: the value's floor, no partials
template <class T, int N> __device__ __forceinline__ ks::Dual<T, N> floor(const ks::Dual<T, N>& x) { return ks::Dual<T, N>(floor(x.v)); }

// x^y; the log term only when the exponent carries partials (a constant exponent at x <= 0 stays finite)
template <class T, int N>
__device__ __forceinline__ ks::Dual<T, N> pow(const ks::Dual<T, N>& x, const ks::Dual<T, N>& y) {
    ks::Dual<T, N> r;
    r.v = pow(x.v, y.v);
    bool ydep = false;
#pragma unroll
    for (int i = 0; i < N; ++i) ydep = ydep || (y.d[i] != T(0));
    const T dx = x.v != T(0) ? y.v * r.v / x.v : (y.v == T(1) ? T(1) : T(0));
    const T dy = ydep ? r.v * log(x.v) : T(0);
#pragma unroll
    for (int i = 0; i < N; ++i) r.d[i] = dx * x.d[i] + (ydep ? dy * y.d[i] : T(0));
    return r;
}

namespace ks {


// acos of a cosine that may round past +-1: the value at the clamped argument, and the derivative
// -1/sqrt(1 - x^2) at the clamped value, zero on the boundary (safe_acos, src/Transfer/step.jl:157-172)
template <class T>
__device__ __forceinline__ T safe_acos(T x) { return acos(fmin(T(1), fmax(T(-1), x))); }
template <class T, int N>
__device__ __forceinline__ Dual<T, N> safe_acos(const Dual<T, N>& x) {
    const T v = fmin(T(1), fmax(T(-1), x.v));
    const T s = T(1) - v * v;
    return dchain(x, acos(v), s > T(0) ? -T(1) / sqrt(s) : T(0));
}

}  // namespace ks
