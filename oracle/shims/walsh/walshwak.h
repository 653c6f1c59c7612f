// Project-written stand-in for FXT's walsh_wak (Walsh transform in
// Walsh-Kronecker, i.e. natural Sylvester-Hadamard, order; unnormalised,
// in place), the only FXT routine the reference calls
// (transform.hpp:111,128; tests.cpp:656-658).  FXT is not installed in this
// image.  Test infrastructure for the CPU oracle/baseline only.
#ifndef CMM_SHIM_WALSHWAK_H
#define CMM_SHIM_WALSHWAK_H

template <typename Type>
inline void walsh_wak(Type* f, unsigned long ldn) {
  const unsigned long n = 1UL << ldn;
  for (unsigned long len = 1; len < n; len <<= 1)
    for (unsigned long s = 0; s < n; s += 2 * len)
      for (unsigned long k = s; k < s + len; ++k) {
        const Type u = f[k], v = f[k + len];
        f[k] = u + v;
        f[k + len] = u - v;
      }
}

#endif  // CMM_SHIM_WALSHWAK_H
