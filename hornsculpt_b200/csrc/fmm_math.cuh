// Spherical-wave expansions of the fast-multipole form: special functions,
// rotation and coaxial translation coefficients, as host+device functions.
//
// Conventions (exp(+i w t) phasor, outgoing wave exp(-i k r)):
//   G(x, y) = exp(-i k |x - y|) / (4 pi |x - y|)
//           = -i k sum_{n,m} h_n(k|x - c|) Y_n^m(x - c) conj(j_n(k|y - c|) Y_n^m(y - c)),  |x - c| > |y - c|,
// h_n = j_n - i y_n (spherical Hankel of the second kind), Y_n^m orthonormal
// with the Condon-Shortley phase, Y_n^m = Theta_n^|m|(cos t) exp(i m phi),
// Theta_n^-m = (-1)^m Theta_n^m. A multipole of centre c is the coefficient
// vector M with field -i k sum M_nm h_n Y_n^m; a local expansion L has field
// -i k sum L_nm j_n Y_n^m. Coefficient (n, m) sits at n*n + n + m.
//
// Translations are rotation -> coaxial translation -> rotation back (the
// point-and-shoot scheme of the reference's LF transfers,
// cuda/wideband_rotation.cu:19-99 and cuda/wideband_axial.cu:10-90). The
// coaxial coefficients come from the addition theorem through Gaunt
// coefficients,
//   (E|F)^m_{n' n}(t z) = 4 pi sum_l i^(n - n' - l) f_l(k t) Y_l^0(z) G(n m; l 0; n' m),
// f = h for multipole-to-local and j for multipole-to-multipole and
// local-to-local; rotations use Wigner small-d matrices.
#pragma once

#include "pair_rules.cuh"

#include <cmath>
#include <cstdint>

namespace hsb {

constexpr int kFmmMaxOrder = 60;
constexpr double kFmmPi = 3.141592653589793;

HS_HD int coefIndex(int n, int m) { return n * n + n + m; }
HS_HD int triIndex(int n, int m) { return n * (n + 1) / 2 + m; }  // Theta_n^m, 0 <= m <= n
// Offset of the Wigner block of degree n: sum_{j < n} (2j + 1)^2.
HS_HD size_t wignerOffset(int n) { return size_t(n) * (4 * size_t(n) * n - 1) / 3; }

// Theta_n^m(x), m <= n <= P, for one m (s = sqrt(1 - x^2)); th indexed by triIndex.
HS_HD void thetaColumn(int m, int P, double x, double s, double *th) {
    if (m > P)
        return;
    double v = 0.28209479177387814;  // 1 / sqrt(4 pi)
    for (int i = 1; i <= m; ++i)
        v *= -sqrt((2.0 * i + 1) / (2.0 * i)) * s;
    th[triIndex(m, m)] = v;
    if (m + 1 > P)
        return;
    double a2 = v, a1 = sqrt(2.0 * m + 3) * x * v;
    th[triIndex(m + 1, m)] = a1;
    for (int n = m + 2; n <= P; ++n) {
        const double a = sqrt((4.0 * n * n - 1) / double(n * n - m * m));
        const double b = sqrt(((n - 1.0) * (n - 1) - double(m) * m) / (4.0 * (n - 1) * (n - 1) - 1));
        const double v2 = a * (x * a1 - b * a2);
        th[triIndex(n, m)] = v2;
        a2 = a1;
        a1 = v2;
    }
}

// Spherical Bessel j_n(x), n = 0..P, x >= 0: upward recurrence while n < x,
// downward continued-fraction ratios beyond (both stable where used).
HS_HD void besselJ(int P, double x, double *j) {
    if (!(x > 1e-300)) {
        j[0] = 1;
        for (int n = 1; n <= P; ++n)
            j[n] = 0;
        return;
    }
    const double sx = sin(x), cx = cos(x);
    j[0] = sx / x;
    int up = 0;
    if (P >= 1 && x > 1.0) {
        j[1] = sx / (x * x) - cx / x;
        up = 1;
        while (up < P && up + 1 < x) {
            j[up + 1] = (2 * up + 1) / x * j[up] - j[up - 1];
            ++up;
        }
    }
    if (up >= P)
        return;
    const int L = P + 24 + int(x);
    double rho = 0;
    for (int n = L; n > up; --n) {
        rho = x / (2 * n + 1 - x * rho);
        if (n <= P)
            j[n] = rho;  // j_n / j_(n-1), turned into values below
    }
    for (int n = up + 1; n <= P; ++n)
        j[n] *= j[n - 1];
}

// Spherical Neumann y_n(x), n = 0..P, x > 0 (upward recurrence, stable).
HS_HD void besselY(int P, double x, double *y) {
    const double sx = sin(x), cx = cos(x);
    y[0] = -cx / x;
    if (P >= 1)
        y[1] = -cx / (x * x) - sx / x;
    for (int n = 1; n < P; ++n)
        y[n + 1] = (2 * n + 1) / x * y[n] - y[n - 1];
}

// Jacobi polynomial P_k^(a,b)(x) by the three-term recurrence in k.
HS_HD double jacobiP(int k, double a, double b, double x) {
    if (k == 0)
        return 1.0;
    double p0 = 1.0, p1 = (a + 1) + (a + b + 2) * (x - 1) / 2;
    for (int n = 2; n <= k; ++n) {
        const double c = 2.0 * n + a + b;
        const double a1 = 2.0 * n * (n + a + b) * (c - 2);
        const double a2 = (c - 1) * (c * (c - 2) * x + a * a - b * b);
        const double a3 = 2.0 * (n + a - 1) * (n + b - 1) * c;
        const double p2 = (a2 * p1 - a3 * p0) / a1;
        p0 = p1;
        p1 = p2;
    }
    return p1;
}

// log of the binomial coefficient C(n, k).
HS_HD double logChoose(double n, double k) { return lgamma(n + 1) - lgamma(k + 1) - lgamma(n - k + 1); }

// Wigner small-d d^j_{mp, m}(beta) through its Jacobi-polynomial form (the
// standard closed form, valid for all index orders via the minimal k).
HS_HD double wignerSmallD(int j, int mp, int m, double cosb, double sinHalf, double cosHalf) {
    int k = j + m < j - m ? j + m : j - m;
    k = j + mp < k ? j + mp : k;
    k = j - mp < k ? j - mp : k;
    int a, lambda;
    if (k == j + m) {
        a = mp - m;
        lambda = mp - m;
    } else if (k == j - m) {
        a = m - mp;
        lambda = 0;
    } else if (k == j + mp) {
        a = m - mp;
        lambda = 0;
    } else {
        a = mp - m;
        lambda = mp - m;
    }
    const int b = 2 * j - 2 * k - a;
    const double scale = exp(0.5 * (logChoose(2 * j - k, k + a) - logChoose(k + b, b)));
    const double sign = (lambda & 1) ? -1.0 : 1.0;
    return sign * scale * pow(sinHalf, a) * pow(cosHalf, b) * jacobiP(k, a, b, cosb);
}

}  // namespace hsb
