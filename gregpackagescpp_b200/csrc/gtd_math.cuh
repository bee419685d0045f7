// Device arithmetic shared by the FP64 force kernels.
#pragma once

#include <cuda_runtime.h>

namespace gtd {

// r2^(-3/2) in FP64 for r2 > 0 (the factor of G m_j (x_j - x_i) in cumulative_acc,
// gregsys.hpp:352-357, which divides by |r|^3).
//
// A hardware seed y ~ r2^(-1/2) (PTX rsqrt.approx.ftz.f64, one MUFU operation) is corrected with
// the binomial series of the exact factor: with e = 1 - r2 y^2 (|e| ~ the seed's relative error),
//     r2^(-3/2) = y^3 (1 - e)^(-3/2) = y^3 (1 + 3/2 e + 15/8 e^2 + 35/16 e^3 + ...),
// truncated after e^2.  e is formed with one FMA, so its absolute error is one rounding of 1;
// the dropped 35/16 e^3 term is below 2^-60 for a seed accurate to 2^-21.  Six FP64 operations
// and one MUFU.  r2 = 0 gives inf or NaN: callers whose rows may hold the self pair select it away.
__device__ __forceinline__ double rsqrt_seed_f64(double x) {
    double y;
    asm("rsqrt.approx.ftz.f64 %0, %1;" : "=d"(y) : "d"(x));
    return y;
}

__device__ __forceinline__ double inv_r3(double r2) {
    const double y = rsqrt_seed_f64(r2);
    const double y2 = y * y;
    const double e = fma(-r2, y2, 1.0);
    const double p = fma(1.875, e, 1.5);
    const double c = fma(e, p, 1.0);
    return (y2 * y) * c;
}

// r2^(-1/2) from the same seed: y (1 - e)^(-1/2) = y (1 + 1/2 e + 3/8 e^2 + ...), truncated after e^2.
__device__ __forceinline__ double inv_r(double r2) {
    const double y = rsqrt_seed_f64(r2);
    const double e = fma(-r2, y * y, 1.0);
    return y * fma(e, fma(0.375, e, 0.5), 1.0);
}

}  // namespace gtd
