// Correctly rounded sin/cos and hypot in double-double arithmetic, for code
// whose decisions must be reproduced bit for bit on the host and the device.
//
// The interaction planner compares error estimates of adaptive quadrature
// patches; a one-ulp difference in one sample can reorder leaves whose errors
// tie and so change the plan. glibc rounds sin, cos and hypot correctly on
// the arguments the planner meets (checked against these functions on the
// host), while the device's library functions carry up to two ulp of error.
// These versions evaluate each function to about 2^-90 relative error and
// round once, so they return the correctly rounded value except when the true
// value lies within 2^-90 of a rounding midpoint.
//
// Method (published): Cody-Waite reduction by pi/2 with a four-part constant
// in double-double, Tang's table method (sin and cos of j*pi/128 in
// double-double, j = 0..34) and short Taylor series for the remainder
// |t| <= pi/256; hypot as the square root of the exactly formed sum of squares
// with one Newton correction. The constants are the successive 53-bit chunks
// of pi/2 and pi/128 and the table values, computed to 90 digits with a
// decimal Machin series and Taylor sums.
//
// Every product that must be exact goes through fma(); all other operations
// are single IEEE operations, so the code must be compiled without
// floating-point contraction (nvcc -fmad=false; g++ defaults on x86-64).
#pragma once

#include "pair_rules.cuh"

namespace hsb {
namespace cr {

struct DD {
    double hi, lo;
};

HS_HD DD twoSum(double a, double b) {
    const double s = a + b, bb = s - a;
    return {s, (a - (s - bb)) + (b - bb)};
}
HS_HD DD fastTwoSum(double a, double b) {  // |a| >= |b|
    const double s = a + b;
    return {s, b - (s - a)};
}
HS_HD DD twoProd(double a, double b) {
    const double p = a * b;
    return {p, fma(a, b, -p)};
}
HS_HD DD add(DD x, DD y) {
    DD s = twoSum(x.hi, y.hi);
    const DD t = twoSum(x.lo, y.lo);
    s.lo += t.hi;
    s = fastTwoSum(s.hi, s.lo);
    s.lo += t.lo;
    return fastTwoSum(s.hi, s.lo);
}
HS_HD DD neg(DD x) { return {-x.hi, -x.lo}; }
HS_HD DD mul(DD x, DD y) {
    DD p = twoProd(x.hi, y.hi);
    p.lo += x.hi * y.lo + x.lo * y.hi;
    return fastTwoSum(p.hi, p.lo);
}
HS_HD DD mulD(DD x, double y) {
    DD p = twoProd(x.hi, y);
    p.lo += x.lo * y;
    return fastTwoSum(p.hi, p.lo);
}

#define HS_CR_SINCOS_TABLE \
    0x0.0p+0, 0x0.0p+0, 0x1.0000000000000p+0, 0x0.0p+0,  \
    0x1.92155f7a3667ep-6, -0x1.b1d63091a0130p-64, 0x1.ffd886084cd0dp-1, -0x1.1354d4556e4cbp-55,  \
    0x1.91f65f10dd814p-5, -0x1.912bd0d569a90p-61, 0x1.ff621e3796d7ep-1, -0x1.c57bc2e24aa15p-57,  \
    0x1.2d52092ce19f6p-4, -0x1.9a088a8bf6b2cp-59, 0x1.fe9cdad01883ap-1, 0x1.521ecd0c67e35p-57,  \
    0x1.917a6bc29b42cp-4, -0x1.e2718d26ed688p-60, 0x1.fd88da3d12526p-1, -0x1.87df6378811c7p-55,  \
    0x1.f564e56a9730ep-4, 0x1.a2704729ae56dp-59, 0x1.fc26470e19fd3p-1, 0x1.1ec8668ecaceep-55,  \
    0x1.2c8106e8e613ap-3, 0x1.13000a89a11e0p-58, 0x1.fa7557f08a517p-1, -0x1.7a0a8ca13571fp-55,  \
    0x1.5e214448b3fc6p-3, 0x1.531ff779ddac6p-57, 0x1.f8764fa714ba9p-1, 0x1.ab256778ffcb6p-56,  \
    0x1.8f8b83c69a60bp-3, -0x1.26d19b9ff8d82p-57, 0x1.f6297cff75cb0p-1, 0x1.562172a361fd3p-56,  \
    0x1.c0b826a7e4f63p-3, -0x1.af1439e521935p-62, 0x1.f38f3ac64e589p-1, -0x1.d7bafb51f72e6p-56,  \
    0x1.f19f97b215f1bp-3, -0x1.42deef11da2c4p-57, 0x1.f0a7efb9230d7p-1, 0x1.52c7adc6b4989p-56,  \
    0x1.111d262b1f677p-2, 0x1.824c20ab7aa9ap-56, 0x1.ed740e7684963p-1, 0x1.e82c791f59cc2p-56,  \
    0x1.294062ed59f06p-2, -0x1.5d28da2c4612dp-56, 0x1.e9f4156c62ddap-1, 0x1.760b1e2e3f81ep-55,  \
    0x1.4135c94176601p-2, 0x1.0c97c4afa2518p-56, 0x1.e6288ec48e112p-1, -0x1.16b56f2847754p-57,  \
    0x1.58f9a75ab1fddp-2, -0x1.efdc0d58cf620p-62, 0x1.e212104f686e5p-1, -0x1.014c76c126527p-55,  \
    0x1.7088530fa459fp-2, -0x1.44b19e0864c5dp-56, 0x1.ddb13b6ccc23cp-1, 0x1.83c37c6107db3p-55,  \
    0x1.87de2a6aea963p-2, -0x1.72cedd3d5a610p-57, 0x1.d906bcf328d46p-1, 0x1.457e610231ac2p-56,  \
    0x1.9ef7943a8ed8ap-2, 0x1.6da81290bdbabp-57, 0x1.d4134d14dc93ap-1, -0x1.4ef5295d25af2p-55,  \
    0x1.b5d1009e15cc0p-2, 0x1.5b362cb974183p-57, 0x1.ced7af43cc773p-1, -0x1.e7b6bb5ab58aep-58,  \
    0x1.cc66e9931c45ep-2, 0x1.6850e59c37f8fp-58, 0x1.c954b213411f5p-1, -0x1.2fb761e946603p-58,  \
    0x1.e2b5d3806f63bp-2, 0x1.e0d891d3c6841p-58, 0x1.c38b2f180bdb1p-1, -0x1.6e0b1757c8d07p-56,  \
    0x1.f8ba4dbf89abap-2, -0x1.2ec1fc1b776b8p-60, 0x1.bd7c0ac6f952ap-1, -0x1.825a732ac700ap-55,  \
    0x1.073879922ffeep-1, -0x1.a5a014347406cp-55, 0x1.b728345196e3ep-1, -0x1.bc69f324e6d61p-55,  \
    0x1.11eb3541b4b23p-1, -0x1.ef23b69abe4f1p-55, 0x1.b090a58150200p-1, -0x1.926da300ffccep-55,  \
    0x1.1c73b39ae68c8p-1, 0x1.b25dd267f6600p-55, 0x1.a9b66290ea1a3p-1, 0x1.9f630e8b6dac8p-60,  \
    0x1.26d054cdd12dfp-1, -0x1.5da743ef3770cp-55, 0x1.a29a7a0462782p-1, -0x1.128bb015df175p-56,  \
    0x1.30ff7fce17035p-1, -0x1.efcc626f74a6fp-57, 0x1.9b3e047f38741p-1, -0x1.30ee286712474p-55,  \
    0x1.3affa292050b9p-1, 0x1.e3e25e3954964p-56, 0x1.93a22499263fbp-1, 0x1.3d419a920df0bp-55,  \
    0x1.44cf325091dd6p-1, 0x1.8076a2cfdc6b3p-57, 0x1.8bc806b151741p-1, -0x1.2c5e12ed1336dp-55,  \
    0x1.4e6cabbe3e5e9p-1, 0x1.3c293edceb327p-57, 0x1.83b0e0bff976ep-1, -0x1.6f420f8ea3475p-56,  \
    0x1.57d69348ceca0p-1, -0x1.75720992bfbb2p-55, 0x1.7b5df226aafafp-1, -0x1.0f537acdf0ad7p-56,  \
    0x1.610b7551d2cdfp-1, -0x1.251b352ff2a37p-56, 0x1.72d0837efff96p-1, 0x1.0d4ef0f1d915cp-55,  \
    0x1.6a09e667f3bcdp-1, -0x1.bdd3413b26456p-55, 0x1.6a09e667f3bcdp-1, -0x1.bdd3413b26456p-55,  \
    0x1.72d0837efff96p-1, 0x1.0d4ef0f1d915cp-55, 0x1.610b7551d2cdfp-1, -0x1.251b352ff2a37p-56,  \
    0x1.7b5df226aafafp-1, -0x1.0f537acdf0ad7p-56, 0x1.57d69348ceca0p-1, -0x1.75720992bfbb2p-55

#if defined(__CUDACC__)
static __device__ const double kSinCosTableDevice[35 * 4] = {HS_CR_SINCOS_TABLE};
#endif
static const double kSinCosTableHost[35 * 4] = {HS_CR_SINCOS_TABLE};
#undef HS_CR_SINCOS_TABLE

HS_HD const double *sinCosTable() {
#if defined(__CUDA_ARCH__)
    return kSinCosTableDevice;
#else
    return kSinCosTableHost;
#endif
}

// sin and cos of x, each correctly rounded (see the file comment). Valid for
// |x| < 2^24; returns false (and leaves the outputs untouched) beyond that or
// for a non-finite x.
HS_HD bool sinCos(double x, double *sinOut, double *cosOut) {
    if (x == 0) {
        *sinOut = x;
        *cosOut = 1;
        return true;
    }
    if (!(fabs(x) < 16777216.0))
        return false;
    // pi/2 = P0 + P1 + P2 + P3
    const double P0 = 0x1.921fb54442d18p+0, P1 = 0x1.1a62633145c07p-54, P2 = -0x1.f1976b7ed8fbcp-110,
                 P3 = 0x1.4cf98e804177dp-164;
    const double n = rint(x * 0x1.45f306dc9c883p-1);  // nearest multiple of pi/2 (off by one is harmless)
    DD p = twoProd(n, P0);
    DD r{x - p.hi, 0};  // exact: x and n*P0 agree in sign and lie within a factor two (Sterbenz), or n = 0
    r = add(r, DD{-p.lo, 0});
    r = add(r, neg(twoProd(n, P1)));
    r = add(r, neg(twoProd(n, P2)));
    r = add(r, DD{-(n * P3), 0});
    // r = a + t with a = j pi/128, |t| <= pi/256
    const double Q0 = 0x1.921fb54442d18p-6, Q1 = 0x1.1a62633145c07p-60, Q2 = -0x1.f1976b7ed8fbcp-116;
    const double j = rint(r.hi * 0x1.45f306dc9c883p+5);
    DD t = add(r, neg(twoProd(j, Q0)));
    t = add(t, neg(twoProd(j, Q1)));
    t = add(t, DD{-(j * Q2), 0});
    const DD u = mul(t, t);
    // sin t = t + t u (-1/6 + u (1/120 + u R(u)))
    const double uh = u.hi;
    const double rs = -1.0 / 5040 + uh * (1.0 / 362880 + uh * (-1.0 / 39916800 + uh * (1.0 / 6227020800.0)));
    DD ps = add(DD{0x1.1111111111111p-7, 0x1.1111111111111p-63}, DD{uh * rs, 0});
    ps = add(DD{-0x1.5555555555555p-3, -0x1.5555555555555p-57}, mul(u, ps));
    const DD st = add(t, mul(t, mul(u, ps)));
    // cos t = 1 + u (-1/2 + u (1/24 + u Rc(u)))
    const double rc =
        -1.0 / 720 + uh * (1.0 / 40320 + uh * (-1.0 / 3628800 + uh * (1.0 / 479001600 + uh * (-1.0 / 87178291200.0))));
    DD pc = add(DD{0x1.5555555555555p-5, 0x1.5555555555555p-59}, DD{uh * rc, 0});
    pc = add(DD{-0.5, 0}, mul(u, pc));
    const DD ct = add(DD{1, 0}, mul(u, pc));
    // sin and cos of a from the table (odd / even in j)
    const int ja = int(fabs(j));
    const double *row = sinCosTable() + 4 * (ja < 34 ? ja : 34);
    const double sg = j < 0 ? -1.0 : 1.0;
    const DD sa{sg * row[0], sg * row[1]}, ca{row[2], row[3]};
    const DD sr = add(mul(sa, ct), mul(ca, st));
    const DD cr = add(mul(ca, ct), neg(mul(sa, st)));
    // quadrant
    const long long q = (long long)n & 3;
    double s, c;
    if (q == 0) {
        s = sr.hi;
        c = cr.hi;
    } else if (q == 1) {
        s = cr.hi;
        c = -sr.hi;
    } else if (q == 2) {
        s = -sr.hi;
        c = -cr.hi;
    } else {
        s = -cr.hi;
        c = sr.hi;
    }
    *sinOut = s;
    *cosOut = c;
    return true;
}

// sqrt(a^2 + b^2), correctly rounded for finite arguments whose squares
// neither overflow nor underflow (|a|, |b| in [2^-480, 2^480], or zero);
// outside that range it returns the plain formula's value.
HS_HD double hypot(double a, double b) {
    a = fabs(a);
    b = fabs(b);
    if (a < b) {
        const double tmp = a;
        a = b;
        b = tmp;
    }
    if (b == 0 || !(a <= 0x1p480) || a < 0x1p-480 || (b < 0x1p-480))
        return b == 0 ? a : sqrt(a * a + b * b);
    const DD s = add(twoProd(a, a), twoProd(b, b));
    const double y = sqrt(s.hi);
    const DD yy = twoProd(y, y);
    const double d = ((s.hi - yy.hi) - yy.lo) + s.lo;  // s - y^2; s.hi - yy.hi is exact
    return y + d / (2 * y);
}

}  // namespace cr
}  // namespace hsb
