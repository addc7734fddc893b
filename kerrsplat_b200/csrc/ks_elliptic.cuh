// ks_elliptic.cuh -- FP64 elliptic-function building blocks for the per-ray constants and the anchor
// table (device and host): Carlson's R_F (Carlson 1995, duplication algorithm), F(phi | m) with
// quasi-periodic unfolding, K(m), and the Jacobi amplitude am(u | m) by the AGM scale
// (DLMF 22.20(ii)). The reference takes these from JacobiElliptic.jl 0.3.10 (CarlsonAlg.am,
// K; src/Geodesics/jacobi.jl:21-25, quadrature.jl:94) and from Krang's closed forms.
#pragma once
#include <cuda_runtime.h>
#include <math.h>

#ifndef KS_HD
#define KS_HD __host__ __device__ __forceinline__
#endif

namespace ks {

constexpr double kPi = 3.141592653589793238462643383279502884;
constexpr double kEps = 2.220446049250313e-16;

KS_HD double rf(double x, double y, double z) {
    double A0 = (x + y + z) / 3.0;
    double Q = 3.7982022430228585e+02 /* (3 eps / 2)^(-1/6) */ *
               fmax(fabs(A0 - x), fmax(fabs(A0 - y), fabs(A0 - z)));
    double xn = x, yn = y, zn = z, An = A0, f = 1.0;
    for (int it = 0; it < 60 && f * Q >= fabs(An); ++it) {
        double sx = sqrt(xn), sy = sqrt(yn), sz = sqrt(zn);
        double lam = sx * sy + sx * sz + sy * sz;
        xn = (xn + lam) * 0.25; yn = (yn + lam) * 0.25; zn = (zn + lam) * 0.25;
        An = (An + lam) * 0.25; f *= 0.25;
    }
    double X = (A0 - x) * f / An, Y = (A0 - y) * f / An, Z = -X - Y;
    double E2 = X * Y - Z * Z, E3 = X * Y * Z;
    return (1.0 - E2 / 10.0 + E3 / 14.0 + E2 * E2 / 24.0 - 3.0 * E2 * E3 / 44.0) / sqrt(An);
}

KS_HD double ellip_k(double m) { return rf(0.0, 1.0 - m, 1.0); }

KS_HD double ellip_f(double phi, double m) {
    double j = nearbyint(phi / kPi);
    double pr = phi - j * kPi;
    double s = sin(pr), c = cos(pr);
    double F = s * rf(c * c, 1.0 - m * s * s, 1.0);
    if (j != 0.0) F += 2.0 * j * ellip_k(m);
    return F;
}

KS_HD double jacobi_am(double u, double m) {
    if (m == 0.0) return u;
    double a[12], c[12];
    a[0] = 1.0; c[0] = sqrt(m);
    double b = sqrt(1.0 - m);
    int n = 0;
    while (n < 11 && fabs(c[n]) > kEps * a[n]) {
        a[n + 1] = 0.5 * (a[n] + b);
        c[n + 1] = c[n] * c[n] / (4.0 * a[n + 1]);
        b = sqrt(a[n] * b);
        ++n;
    }
    double phi = ldexp(a[n] * u, n);
    for (int i = n; i > 0; --i) phi = 0.5 * (phi + asin(c[i] * sin(phi) / a[i]));
    return phi;
}

template <class T>
struct JS { T sn, cn, dn; };

KS_HD JS<double> jstate(double u, double mu) {
    double ph = jacobi_am(u, mu);
    double s = sin(ph), c = cos(ph);
    return {s, c, sqrt(fma(-mu, s * s, 1.0))};
}

KS_HD JS<double> jstep_constants(double delta, double mu) {
    JS<double> x = jstate(fabs(delta), mu);
    return {copysign(x.sn, delta), x.cn, x.dn};
}

// The addition theorems (fifteen multiplications, one division), any precision.
template <class T>
KS_HD JS<T> jstep(const JS<T>& x, const JS<T>& d, T mu) {
    T den = T(1) - mu * (x.sn * x.sn) * (d.sn * d.sn);
    T sn = x.sn * d.cn * d.dn + d.sn * x.cn * x.dn;
    T cn = x.cn * d.cn - x.sn * x.dn * d.sn * d.dn;
    T dn = x.dn * d.dn - mu * x.sn * x.cn * d.sn * d.cn;
    if constexpr (sizeof(T) == 8) {
        return {sn / den, cn / den, dn / den};
    } else {
        T inv = T(1) / den;   // one reciprocal in FP32
        return {sn * inv, cn * inv, dn * inv};
    }
}

}  // namespace ks
