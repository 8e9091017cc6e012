// Double-precision sine for the actuation phase, evaluated identically on
// every device: Cody & Waite (1980) reduction x = k*(pi/2) + r with a
// three-part pi/2 (33 + 33 bits + remainder, exact products for |k| < 2^20),
// then the Taylor series of sin or cos on |r| <= pi/4 by Horner's rule with
// fused multiply-adds.  Constants: (-1)^k/(2k+1)!, (-1)^k/(2k)! and the pi/2
// split, each the correctly rounded double of the exact value (pi from
// Machin's formula).  Every operation is an explicit round-to-nearest
// intrinsic, so the result does not depend on compiler contraction.
#pragma once

namespace mb {

__device__ __forceinline__ double sin_cw(double x) {
    constexpr double kTwoOverPi = 0.6366197723675814;
    constexpr double kPio2_1 = 1.5707963267341256;
    constexpr double kPio2_2 = 6.077100506303966e-11;
    constexpr double kPio2_3 = 2.0222662487959506e-21;
    const double k = rint(__dmul_rn(x, kTwoOverPi));
    double r = __fma_rn(-k, kPio2_1, x);
    r = __fma_rn(-k, kPio2_2, r);
    r = __fma_rn(-k, kPio2_3, r);
    const long long q = (long long)k & 3;
    const double r2 = __dmul_rn(r, r);
    double p;
    if (q == 0 || q == 2) {
        p = -8.22063524662433e-18;
        p = __fma_rn(p, r2, 2.8114572543455206e-15);
        p = __fma_rn(p, r2, -7.647163731819816e-13);
        p = __fma_rn(p, r2, 1.6059043836821613e-10);
        p = __fma_rn(p, r2, -2.505210838544172e-08);
        p = __fma_rn(p, r2, 2.7557319223985893e-06);
        p = __fma_rn(p, r2, -0.0001984126984126984);
        p = __fma_rn(p, r2, 0.008333333333333333);
        p = __fma_rn(p, r2, -0.16666666666666666);
        p = __fma_rn(p, r2, 1.0);
        p = __dmul_rn(p, r);
    } else {
        p = 4.110317623312165e-19;
        p = __fma_rn(p, r2, -1.5619206968586225e-16);
        p = __fma_rn(p, r2, 4.779477332387385e-14);
        p = __fma_rn(p, r2, -1.1470745597729725e-11);
        p = __fma_rn(p, r2, 2.08767569878681e-09);
        p = __fma_rn(p, r2, -2.755731922398589e-07);
        p = __fma_rn(p, r2, 2.48015873015873e-05);
        p = __fma_rn(p, r2, -0.001388888888888889);
        p = __fma_rn(p, r2, 0.041666666666666664);
        p = __fma_rn(p, r2, -0.5);
        p = __fma_rn(p, r2, 1.0);
    }
    return (q >= 2) ? -p : p;
}

}  // namespace mb
