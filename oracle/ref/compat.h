/*
 * compat.h -- force-included when compiling the reference's sources for the
 * test oracle.  Modern libstdc++ has no operator*(int, std::complex<double>),
 * which lib/lattice_util.cpp:2173 and :2288 use; this supplies it with the
 * meaning the old compilers gave it (promote the int to double).
 */
#ifndef QKX_REF_COMPAT_H
#define QKX_REF_COMPAT_H
#include <complex>
inline std::complex<double> operator*(int a, const std::complex<double>& b) {
  return static_cast<double>(a) * b;
}
inline std::complex<double> operator*(const std::complex<double>& b, int a) {
  return static_cast<double>(a) * b;
}
#endif
