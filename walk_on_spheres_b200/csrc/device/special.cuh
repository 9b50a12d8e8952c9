// Special functions of the screened-Poisson and Helmholtz weights.
//
// The reference evaluates e^-x I0(x) and e^x K0(x) with libstdc++'s
// std::cyl_bessel_i / std::cyl_bessel_k below x = 50 and with the Hankel
// asymptotic series above (include/wos/bessel.hpp:16-87).  There is no
// libstdc++ special-function code on the device, so:
//   I0(x)      power series sum (x^2/4)^k / (k!)^2 (all terms positive);
//   K0(x<=2)   series -(ln(x/2)+gamma) I0(x) + sum (x^2/4)^k/(k!)^2 H_k;
//   e^x K0(x)  for 2 < x < 50 from K0(x) = int_0^inf exp(-x cosh t) dt with
//              s = sinh(t/2), s = w/sqrt(2x):
//                e^x K0(x) = sqrt(2/x) int_0^inf e^{-w^2} (1 + w^2/(2x))^{-1/2} dw,
//              an even integrand analytic for |Im w| < sqrt(2x), so the
//              trapezoidal rule with step 1/4 converges to double precision
//              with 27 nodes;
//   x >= 50    the Hankel series with the reference's truncation rule.
// The same code (double) is the C oracle's (oracle/wos_oracle.c); both agree
// with libstdc++ to a few ulps.  J0 / Y0 are the reference's own truncated
// series (include/wos/fastmath.hpp:15-50), restated exactly.
#pragma once
#include <cmath>

namespace wosb {

template <typename T>
struct Limits;
template <>
struct Limits<double> {
    __device__ static constexpr double eps() { return 2.220446049250313e-16; }
    __device__ static constexpr double tiny_rel() { return 1e-17; }
};
template <>
struct Limits<float> {
    __device__ static constexpr float eps() { return 1.1920929e-07f; }
    __device__ static constexpr float tiny_rel() { return 3e-8f; }
};

constexpr double kPi = 3.14159265358979323846;

template <typename T>
__device__ __forceinline__ T hankel_sum(T x, bool alternating) {
    T sum = T(1), term = T(1), prev = T(INFINITY);
    for (int k = 1; k <= 24; ++k) {
        const T odd = static_cast<T>(2 * k - 1);
        T f = odd * odd / (T(8) * x * static_cast<T>(k));
        if (alternating) f = -f;
        term *= f;
        const T mag = fabs(term);
        if (mag > prev) break;
        sum += term;
        if (mag <= Limits<T>::eps() * fabs(sum)) break;
        prev = mag;
    }
    return sum;
}

template <typename T>
__device__ __forceinline__ T i0_series(T x) {
    const T q = T(0.25) * x * x;
    T term = T(1), sum = T(1);
    for (int k = 1; k < 500; ++k) {
        term *= q / (static_cast<T>(k) * static_cast<T>(k));
        sum += term;
        if (term <= Limits<T>::tiny_rel() * sum) break;
    }
    return sum;
}

template <typename T>
__device__ __forceinline__ T k0_scaled_integral(T x) {
    const T h = T(0.25);
    const T inv2x = T(1) / (T(2) * x);
    T sum = T(0.5);
    for (int k = 1; k <= 27; ++k) {
        const T w = h * static_cast<T>(k);
        sum += exp(-w * w) / sqrt(T(1) + w * w * inv2x);
    }
    return sqrt(T(2) / x) * h * sum;
}

template <typename T>
__device__ __forceinline__ T k0_series(T x) {
    const T gamma = T(0.57721566490153286061);
    const T q = T(0.25) * x * x;
    T term = T(1), h = T(0), sum = T(0);
    for (int k = 1; k < 60; ++k) {
        term *= q / (static_cast<T>(k) * static_cast<T>(k));
        h += T(1) / static_cast<T>(k);
        sum += term * h;
        if (term * h <= T(1e-18) * fabs(sum)) break;
    }
    return -(log(T(0.5) * x) + gamma) * i0_series(x) + sum;
}

template <typename T>
__device__ __forceinline__ T i0_scaled(T x) {
    x = fabs(x);
    if (x < T(50)) return exp(-x) * i0_series(x);
    return hankel_sum(x, false) / sqrt(T(2) * T(kPi) * x);
}

template <typename T>
__device__ __forceinline__ T k0_scaled(T x) {
    if (x < T(0)) return T(NAN);
    if (x == T(0)) return T(INFINITY);
    if (x < T(50)) {
        if (x <= T(2)) return exp(x) * k0_series(x);
        return k0_scaled_integral(x);
    }
    return sqrt(T(kPi) / (T(2) * x)) * hankel_sum(x, true);
}

template <typename T>
__device__ __forceinline__ T log_i0(T x) {
    x = fabs(x);
    return x + log(i0_scaled(x));
}

template <typename T>
__device__ __forceinline__ T log_k0(T x) {
    if (x < T(0)) return T(NAN);
    if (x == T(0)) return T(INFINITY);
    return -x + log(k0_scaled(x));
}

// FP32 walks (FAST_FP32): the polynomial approximations of Abramowitz &
// Stegun, Handbook of Mathematical Functions, 9.8.1, 9.8.2, 9.8.5 and 9.8.6,
// whose absolute errors on the scaled forms (I0(x) for x < 3.75,
// sqrt(x) e^-x I0(x) above; K0(x) + ln(x/2) I0(x) for x <= 2, sqrt(x) e^x K0(x)
// above) are below 1.9e-7.  That is FP32 resolution; the series and the
// quadrature above would cost dozens of iterations per call for nothing.
__device__ __forceinline__ float as_i0_small(float x) {  // 9.8.1, |x| < 3.75
    const float t = x * (1.0f / 3.75f);
    const float u = t * t;
    return 1.0f +
           u * (3.5156229f +
                u * (3.0899424f +
                     u * (1.2067492f + u * (0.2659732f + u * (0.0360768f + u * 0.0045813f)))));
}

template <>
__device__ __forceinline__ float log_i0<float>(float x) {
    x = fabsf(x);
    if (x < 3.75f) return logf(as_i0_small(x));
    const float u = 3.75f / x;  // 9.8.2
    const float q =
        0.39894228f +
        u * (0.01328592f +
             u * (0.00225319f +
                  u * (-0.00157565f +
                       u * (0.00916281f +
                            u * (-0.02057706f +
                                 u * (0.02635537f + u * (-0.01647633f + u * 0.00392377f)))))));
    return x - 0.5f * logf(x) + logf(q);
}

template <>
__device__ __forceinline__ float log_k0<float>(float x) {
    if (x < 0.0f) return NAN;
    if (x == 0.0f) return INFINITY;
    if (x <= 2.0f) {  // 9.8.5
        const float y = 0.25f * x * x;
        const float k =
            -logf(0.5f * x) * as_i0_small(x) +
            (-0.57721566f +
             y * (0.42278420f +
                  y * (0.23069756f +
                       y * (0.03488590f + y * (0.00262698f + y * (0.00010750f + y * 0.0000074f))))));
        return logf(k);
    }
    const float u = 2.0f / x;  // 9.8.6
    const float q =
        1.25331414f +
        u * (-0.07832358f +
             u * (0.02189568f +
                  u * (-0.01062446f + u * (0.00587872f + u * (-0.00251540f + u * 0.00053208f)))));
    return -x - 0.5f * logf(x) + logf(q);
}

// include/wos/fastmath.hpp:15-28 (series truncated at a 1e-8 term)
template <typename T>
__device__ __forceinline__ T bessel_j0(T x) {
    const T hx = T(0.25) * x * x;
    T term = T(1), sum = T(1);
    for (int k = 1; k < 200; ++k) {
        term *= hx / static_cast<T>(k * k);
        if (term < T(1e-8)) return sum;
        sum += (k % 2 == 0 ? term : -term);
    }
    return sum;
}

}  // namespace wosb
