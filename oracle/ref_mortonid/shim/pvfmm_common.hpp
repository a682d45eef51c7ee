// Minimal stand-in for the reference's include/pvfmm_common.hpp, enough to
// compile the reference's src/mortonid.cpp and include/mortonid.{hpp,txx}
// from their own sources.  The real header pulls in the SCTL submodule,
// which is absent; mortonid only needs PVFMM_MAX_DEPTH and sctl::pow.
#ifndef _PVFMM_COMMON_HPP_
#define _PVFMM_COMMON_HPP_
#include <cassert>
#include <cstdint>
#define PVFMM_MAX_DEPTH 30
namespace sctl {
template <long N, class T>
constexpr T pow(const T& x) {
  return N <= 0 ? T(1) : x * pow<(N > 0 ? N - 1 : 0), T>(x);
}
}  // namespace sctl
#endif
