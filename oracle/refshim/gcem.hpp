// Stand-in for the gcem header the reference fetches at configure time (not
// vendored, no network here).  The reference reaches gcem through its
// `constexpr_math` alias (include/math/math/ConstexprMath.h:47-53) for exp,
// pow and sin, and calls gcem::floor/abs in its fast-sine helper.  Each
// function forwards to the GCC math builtin, which GCC folds in constant
// expressions and lowers to libm at run time, so both uses keep working.
#pragma once
namespace gcem {
template <typename T>
constexpr T abs(T x) { return x < T(0) ? -x : x; }
template <typename T>
constexpr T floor(T x) { return static_cast<T>(__builtin_floor(static_cast<double>(x))); }
constexpr double exp(double x) { return __builtin_exp(x); }
constexpr double sin(double x) { return __builtin_sin(x); }
constexpr double cos(double x) { return __builtin_cos(x); }
constexpr double sqrt(double x) { return __builtin_sqrt(x); }
constexpr double log(double x) { return __builtin_log(x); }
template <typename A, typename B>
constexpr double pow(A x, B y) { return __builtin_pow(static_cast<double>(x), static_cast<double>(y)); }
}  // namespace gcem
