/* Inverse error function for the reference oracle build.
 *
 * The reference only calls boost::math::erf_inv(long double) to turn the
 * storage P threshold into a t threshold (src/Utility.cpp:244-250).  This
 * is written from the definition: Newton's method on erf(x) - z = 0 in long
 * double, with derivative 2/sqrt(pi) * exp(-x^2), started from the
 * Winitzki (2008) closed-form approximation and iterated to convergence. */
#ifndef OA_REF_BOOST_ERF_HPP
#define OA_REF_BOOST_ERF_HPP
#include <cmath>
namespace boost { namespace math {
inline long double erf_inv(long double z)
{
    if (z <= -1.0L) return -HUGE_VALL;
    if (z >= 1.0L) return HUGE_VALL;
    if (z == 0.0L) return 0.0L;
    const long double a = 0.147L;
    const long double pi = 3.141592653589793238462643383279502884L;
    long double ln = std::log(1.0L - z * z);
    long double t1 = 2.0L / (pi * a) + ln / 2.0L;
    long double x = std::sqrt(std::sqrt(t1 * t1 - ln / a) - t1);
    if (z < 0) x = -x;
    const long double c = 2.0L / std::sqrt(pi);
    for (int it = 0; it < 100; ++it) {
        long double f = std::erf(x) - z;
        long double step = f / (c * std::exp(-x * x));
        x -= step;
        if (std::fabs(step) <= 1e-19L * (1.0L + std::fabs(x))) break;
    }
    return x;
}
inline double erf_inv(double z) { return (double)erf_inv((long double)z); }
inline float erf_inv(float z) { return (float)erf_inv((long double)z); }
}}
#endif
