// ks_elliptic.cuh -- FP64 elliptic-function building blocks for the per-ray constants and the anchor
// table (device and host): Carlson's R_F (Carlson 1995, duplication algorithm), F(phi | m) with
// quasi-periodic unfolding, K(m), and the Jacobi amplitude am(u | m) by the AGM scale
// (DLMF 22.20(ii)). The reference takes these from JacobiElliptic.jl 0.3.10 (CarlsonAlg.am,
// K; src/Geodesics/jacobi.jl:21-25, quadrature.jl:94) and from Krang's closed forms.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#include "ks_dual.cuh"

#ifndef KS_HD
#define KS_HD __host__ __device__ __forceinline__
#endif

namespace ks {

constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double kEps = 2.220446049250313e-16;

// The building blocks are templates in the scalar type: double for the FP64 geodesics, a dual number
// for the spacetime derivatives (iterations and branches compare values).
template <class T> KS_HD double val(const T& x) { return value_of(x); }
KS_HD double val(double x) { return x; }

template <class T>
KS_HD T rf(T x, T y, T z) {
    T A0 = (x + y + z) / 3.0;
    T Q = 3.7982022430228585e+02 /* (3 eps / 2)^(-1/6) */ *
          fmax(fabs(A0 - x), fmax(fabs(A0 - y), fabs(A0 - z)));
    T xn = x, yn = y, zn = z, An = A0;
    double f = 1.0;
    for (int it = 0; it < 60 && f * val(Q) >= fabs(val(An)); ++it) {
        T sx = sqrt(xn), sy = sqrt(yn), sz = sqrt(zn);
        T lam = sx * sy + sx * sz + sy * sz;
        xn = (xn + lam) * 0.25; yn = (yn + lam) * 0.25; zn = (zn + lam) * 0.25;
        An = (An + lam) * 0.25; f *= 0.25;
    }
    T X = (A0 - x) * f / An, Y = (A0 - y) * f / An, Z = -X - Y;
    T E2 = X * Y - Z * Z, E3 = X * Y * Z;
    return (1.0 - E2 / 10.0 + E3 / 14.0 + E2 * E2 / 24.0 - 3.0 * E2 * E3 / 44.0) / sqrt(An);
}

template <class T>
KS_HD T ellip_k(T m) { return rf(T(0.0), T(1.0) - m, T(1.0)); }

template <class T>
KS_HD T ellip_f(T phi, T m) {
    double j = nearbyint(val(phi) / kPi);
    T pr = phi - j * kPi;
    T s = sin(pr), c = cos(pr);
    T F = s * rf(c * c, T(1.0) - m * s * s, T(1.0));
    if (j != 0.0) F += 2.0 * j * ellip_k(m);
    return F;
}

template <class T>
KS_HD T jacobi_am(T u, T m) {
    if (val(m) == 0.0) return u;
    T a[12], c[12];
    a[0] = T(1.0); c[0] = sqrt(m);
    T b = sqrt(T(1.0) - m);
    int n = 0;
    while (n < 11 && fabs(val(c[n])) > kEps * val(a[n])) {
        a[n + 1] = 0.5 * (a[n] + b);
        c[n + 1] = c[n] * c[n] / (4.0 * a[n + 1]);
        b = sqrt(a[n] * b);
        ++n;
    }
    T phi = (a[n] * u) * ldexp(1.0, n);
    for (int i = n; i > 0; --i) phi = 0.5 * (phi + asin(c[i] * sin(phi) / a[i]));
    return phi;
}

template <class T>
struct JS { T sn, cn, dn; };

template <class T>
KS_HD JS<T> jstate(T u, T mu) {
    T ph = jacobi_am(u, mu);
    T s = sin(ph), c = cos(ph);
    return {s, c, sqrt(fma(-mu, s * s, T(1.0)))};
}

template <class T>
KS_HD JS<T> jstep_constants(T delta, T mu) {
    JS<T> x = jstate(fabs(delta), mu);
    return {copysign(x.sn, delta), x.cn, x.dn};
}

// The addition theorems (fifteen multiplications, one division), any precision.
template <class T>
KS_HD JS<T> jstep(const JS<T>& x, const JS<T>& d, T mu) {
    T den = T(1) - mu * (x.sn * x.sn) * (d.sn * d.sn);
    T sn = x.sn * d.cn * d.dn + d.sn * x.cn * x.dn;
    T cn = x.cn * d.cn - x.sn * x.dn * d.sn * d.dn;
    T dn = x.dn * d.dn - mu * x.sn * x.cn * d.sn * d.cn;
    if constexpr (!is_f32<T>) {
        return {sn / den, cn / den, dn / den};
    } else {
        T inv = T(1) / den;   // one reciprocal in FP32
        return {sn * inv, cn * inv, dn * inv};
    }
}

}  // namespace ks
