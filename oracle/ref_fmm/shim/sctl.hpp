// Stand-in for the part of SCTL (https://github.com/dmalhotra/SCTL, the
// reference's un-vendored submodule; no commit is pinned in the reference
// tree) that the reference's particle-FMM path calls.  Test infrastructure:
// it lets the reference's own sources build here to pin the oracle and to
// time the reference on the host CPU.  Each piece restates the published
// behaviour the reference relies on:
//   - scalar math (fabs, pow, sqrt, sin, cos, log, const_pi, machine_eps);
//   - Vec<T, N>: an N-lane SIMD value with loads, stores, arithmetic, FMA,
//     comparisons into masks (GCC vector extensions);
//   - approx_rsqrt<digits>(x, mask): 1/sqrt(x) to at least `digits` decimal
//     digits where mask is set, 0 elsewhere: a hardware estimate refined by
//     Newton-Raphson steps y <- y (3 - x y^2) / 2, each doubling the bits;
//   - ScratchBuf<T>: a temporary aligned buffer;
//   - mat::gemm / mat::svd: the BLAS dgemm / LAPACK dgesvd calling
//     conventions (column-major), forwarded to the OpenBLAS that scipy
//     bundles; mat::pinv: the truncated pseudo-inverse V S+ U^T with the
//     singular values below eps * max S dropped;
//   - Matrix<T>: a row-major matrix with pinv (one call site, the periodic
//     corner correction).
#ifndef PVFMM_REF_SCTL_SHIM_HPP
#define PVFMM_REF_SCTL_SHIM_HPP

#include <immintrin.h>

#include <algorithm>
#include <cassert>
#include <functional>
#include <iostream>
#include <map>
#include <set>
#include <sstream>
#include <string>
#include <cmath>
#include <cstdint>
#include <cstdlib>
#include <cstring>
#include <limits>
#include <type_traits>
#include <vector>

extern "C" {
void scipy_dgemm_(const char*, const char*, const int*, const int*, const int*, const double*, const double*,
                  const int*, const double*, const int*, const double*, double*, const int*);
void scipy_sgemm_(const char*, const char*, const int*, const int*, const int*, const float*, const float*,
                  const int*, const float*, const int*, const float*, float*, const int*);
void scipy_dgesvd_(const char*, const char*, const int*, const int*, double*, const int*, double*, double*,
                   const int*, double*, const int*, double*, const int*, int*);
void scipy_sgesvd_(const char*, const char*, const int*, const int*, float*, const int*, float*, float*, const int*,
                   float*, const int*, float*, const int*, int*);
}

namespace sctl {

typedef long Long;
typedef int Integer;

template <class T>
inline T* Ptr2Itr(T* p, Long) {
  return p;
}
template <class T>
inline const T* Ptr2Itr(const T* p, Long) {
  return p;
}

template <class T>
constexpr T const_pi() {
  return (T)3.141592653589793238462643383279502884L;
}
template <class T>
inline T machine_eps() {
  return std::numeric_limits<T>::epsilon();
}

template <class T>
inline T fabs(const T a) {
  return a < 0 ? -a : a;
}
template <class T>
inline T sqrt(const T a) {
  return std::sqrt(a);
}
template <class T>
inline T sin(const T a) {
  return std::sin(a);
}
template <class T>
inline T cos(const T a) {
  return std::cos(a);
}
template <class T>
inline T log(const T a) {
  return std::log(a);
}
template <class T>
inline T exp(const T a) {
  return std::exp(a);
}

// b^e; integer bases and exponents by repeated multiplication (exact).
template <class Real, class ExpType>
inline Real pow(const Real b, const ExpType e) {
  if constexpr (std::is_integral<Real>::value && std::is_integral<ExpType>::value) {
    Real r = 1;
    for (ExpType i = 0; i < e; ++i) r *= b;
    return r;
  } else {
    return std::pow(b, (Real)e);
  }
}
// b^e with e known at compile time.
template <Long e, class ValueType>
constexpr ValueType pow(const ValueType b) {
  return e <= 0 ? ValueType(1) : b * pow<(e > 0 ? e - 1 : 0), ValueType>(b);
}

template <class T>
struct TypeTraits {
  static constexpr Integer SigBits = std::numeric_limits<T>::digits;
};

#if defined(__AVX512F__)
constexpr Integer kAlignBytes = 64;
#elif defined(__AVX__)
constexpr Integer kAlignBytes = 32;
#else
constexpr Integer kAlignBytes = 16;
#endif

template <class T>
constexpr Integer DefaultVecLen() {
  return kAlignBytes / (Integer)sizeof(T);
}

template <class T, Long N>
class Vec;

template <class T, Long N>
struct Mask {
  using IT = typename std::conditional<sizeof(T) == 8, int64_t, int32_t>::type;
  typedef IT VI __attribute__((vector_size(N * sizeof(T))));
  VI m;
};

template <class T, Long N>
class Vec {
 public:
  typedef T VT __attribute__((vector_size(N * sizeof(T))));
  typedef T ScalarType;
  typedef Mask<T, N> MaskType;
  static constexpr Integer Size() { return N; }

  Vec() = default;
  Vec(const T a) {
    for (Long i = 0; i < N; ++i) v[i] = a;
  }
  static Vec Zero() { return Vec((T)0); }
  static Vec Load1(const T* p) { return Vec(*p); }
  static Vec Load(const T* p) {
    Vec r;
    std::memcpy(&r.v, p, sizeof(VT));
    return r;
  }
  static Vec LoadAligned(const T* p) {
    Vec r;
    r.v = *reinterpret_cast<const VT*>(__builtin_assume_aligned(p, sizeof(VT)));
    return r;
  }
  void Store(T* p) const { std::memcpy(p, &v, sizeof(VT)); }
  void StoreAligned(T* p) const { *reinterpret_cast<VT*>(__builtin_assume_aligned(p, sizeof(VT))) = v; }
  T operator[](Integer i) const { return v[i]; }
  void insert(Integer i, T x) { v[i] = x; }

  friend Vec operator+(Vec a, const Vec& b) {
    a.v += b.v;
    return a;
  }
  friend Vec operator-(Vec a, const Vec& b) {
    a.v -= b.v;
    return a;
  }
  friend Vec operator*(Vec a, const Vec& b) {
    a.v *= b.v;
    return a;
  }
  friend Vec operator/(Vec a, const Vec& b) {
    a.v /= b.v;
    return a;
  }
  friend Vec operator-(Vec a) {
    a.v = -a.v;
    return a;
  }
  Vec& operator+=(const Vec& b) {
    v += b.v;
    return *this;
  }
  Vec& operator-=(const Vec& b) {
    v -= b.v;
    return *this;
  }
  Vec& operator*=(const Vec& b) {
    v *= b.v;
    return *this;
  }
  Vec& operator/=(const Vec& b) {
    v /= b.v;
    return *this;
  }
  friend Vec FMA(const Vec& a, const Vec& b, const Vec& c) {
    Vec r;
#if defined(__FMA__)
    for (Long i = 0; i < N; ++i) r.v[i] = std::fma(a.v[i], b.v[i], c.v[i]);
#else
    r.v = a.v * b.v + c.v;
#endif
    return r;
  }
  friend MaskType operator>(const Vec& a, const Vec& b) {
    MaskType m;
    m.m = a.v > b.v;
    return m;
  }
  friend MaskType operator<(const Vec& a, const Vec& b) {
    MaskType m;
    m.m = a.v < b.v;
    return m;
  }
  // mask ? a : 0
  friend Vec and_mask(const Vec& a, const MaskType& m) {
    Vec r;
    for (Long i = 0; i < N; ++i) r.v[i] = m.m[i] ? a.v[i] : (T)0;
    return r;
  }
  friend void sincos(Vec& s, Vec& c, const Vec& x) {
    for (Long i = 0; i < N; ++i) {
      s.v[i] = std::sin(x.v[i]);
      c.v[i] = std::cos(x.v[i]);
    }
  }

  VT v;
};

// Newton steps needed to reach `digits` decimal digits from an estimate with
// `bits0` correct bits (each step doubles the correct bits).
constexpr int rsqrt_newton_steps(int digits, int bits0) {
  int bits = bits0, n = 0;
  while (bits < (int)(digits * 3.3219280948873623) + 1 && n < 4) {
    bits *= 2;
    ++n;
  }
  return n;
}

template <int digits, class T, Long N>
inline Vec<T, N> approx_rsqrt(const Vec<T, N>& x, const Mask<T, N>& m) {
  Vec<T, N> y;
  int bits0 = 11;
#if defined(__AVX512F__)
  if constexpr (sizeof(T) == 8 && N == 8) {
    y.v = (typename Vec<T, N>::VT)_mm512_rsqrt14_pd((__m512d)x.v);
    bits0 = 14;
  } else if constexpr (sizeof(T) == 4 && N == 16) {
    y.v = (typename Vec<T, N>::VT)_mm512_rsqrt14_ps((__m512)x.v);
    bits0 = 14;
  } else
#endif
#if defined(__AVX__)
      if constexpr (sizeof(T) == 8 && N == 4) {
    y.v = (typename Vec<T, N>::VT)_mm256_cvtps_pd(_mm_rsqrt_ps(_mm256_cvtpd_ps((__m256d)x.v)));
  } else if constexpr (sizeof(T) == 4 && N == 8) {
    y.v = (typename Vec<T, N>::VT)_mm256_rsqrt_ps((__m256)x.v);
  } else
#endif
  {
    for (Long i = 0; i < N; ++i) y.v[i] = (T)(1.0f / std::sqrt((float)x.v[i]));
  }
  constexpr int steps8 = rsqrt_newton_steps(digits, 11);
  const int steps = bits0 >= 14 ? rsqrt_newton_steps(digits, 14) : steps8;
  const Vec<T, N> half_x = x * Vec<T, N>((T)0.5), three_half((T)1.5);
  for (int s = 0; s < steps; ++s) y = y * (three_half - half_x * y * y);
  return and_mask(y, m);
}

template <class T>
class ScratchBuf {
 public:
  explicit ScratchBuf(Long n) : n_(n) {
    p_ = static_cast<T*>(std::aligned_alloc(64, ((size_t)std::max<Long>(n, 1) * sizeof(T) + 63) / 64 * 64));
  }
  ~ScratchBuf() { std::free(p_); }
  ScratchBuf(const ScratchBuf&) = delete;
  ScratchBuf& operator=(const ScratchBuf&) = delete;
  T& operator[](Long i) { return p_[i]; }
  const T& operator[](Long i) const { return p_[i]; }
  T* begin() { return p_; }
  Long Dim() const { return n_; }

 private:
  T* p_;
  Long n_;
};

namespace mat {

inline void gemm(char ta, char tb, int M, int N, int K, double alpha, const double* A, int lda, const double* B,
                 int ldb, double beta, double* C, int ldc) {
  if (M <= 0 || N <= 0) return;
  scipy_dgemm_(&ta, &tb, &M, &N, &K, &alpha, A, &lda, B, &ldb, &beta, C, &ldc);
}
inline void gemm(char ta, char tb, int M, int N, int K, float alpha, const float* A, int lda, const float* B,
                 int ldb, float beta, float* C, int ldc) {
  if (M <= 0 || N <= 0) return;
  scipy_sgemm_(&ta, &tb, &M, &N, &K, &alpha, A, &lda, B, &ldb, &beta, C, &ldc);
}

inline void svd(char* ju, char* jvt, int* M, int* N, double* A, int* lda, double* S, double* U, int* ldu, double* VT,
                int* ldvt, double* work, int* lwork, int* info) {
  scipy_dgesvd_(ju, jvt, M, N, A, lda, S, U, ldu, VT, ldvt, work, lwork, info);
}
inline void svd(char* ju, char* jvt, int* M, int* N, float* A, int* lda, float* S, float* U, int* ldu, float* VT,
                int* ldvt, float* work, int* lwork, int* info) {
  scipy_sgesvd_(ju, jvt, M, N, A, lda, S, U, ldu, VT, ldvt, work, lwork, info);
}

// M (n1 x n2, row-major) -> M_ (n2 x n1, row-major) = V S+ U^T, singular
// values below eps * max S dropped.
template <class T>
void pinv(const T* M, int n1, int n2, T eps, T* M_) {
  if (n1 <= 0 || n2 <= 0) return;
  // column-major view: A (n2 x n1) = M^T; A = U S VT  =>  M = VT^T S U^T
  const int m = n2, n = n1, k = std::min(m, n);
  std::vector<T> A(M, M + (size_t)n1 * n2), S(k), U((size_t)m * k), VT((size_t)k * n);
  char job = 'S';
  int lda = m, ldu = m, ldvt = k, info = 0, lwork = -1;
  T wq = 0;
  svd(&job, &job, const_cast<int*>(&m), const_cast<int*>(&n), A.data(), &lda, S.data(), U.data(), &ldu, VT.data(),
      &ldvt, &wq, &lwork, &info);
  lwork = (int)wq + 1;
  std::vector<T> work(lwork);
  svd(&job, &job, const_cast<int*>(&m), const_cast<int*>(&n), A.data(), &lda, S.data(), U.data(), &ldu, VT.data(),
      &ldvt, work.data(), &lwork, &info);
  const T cut = (k > 0 ? S[0] : 0) * eps;
  for (int i = 0; i < k; ++i) S[i] = (S[i] > cut && S[i] > 0) ? 1 / S[i] : 0;
  // pinv(M) = pinv(A^T) = (V S+ U^T)^T = U S+ VT (n2 x n1), stored row-major
  for (int r = 0; r < n2; ++r)
    for (int c = 0; c < n1; ++c) {
      T s = 0;
      for (int j = 0; j < k; ++j) s += VT[(size_t)c * k + j] * S[j] * U[(size_t)j * m + r];
      M_[(size_t)r * n1 + c] = s;
    }
}

}  // namespace mat

template <class T>
class Matrix {
 public:
  Matrix() = default;
  Matrix(Long d0, Long d1) : d0_(d0), d1_(d1), a_((size_t)d0 * d1) {}
  Long Dim(int i) const { return i == 0 ? d0_ : d1_; }
  T* operator[](Long i) { return a_.data() + (size_t)i * d1_; }
  const T* operator[](Long i) const { return a_.data() + (size_t)i * d1_; }
  // pseudo-inverse; eps < 0 selects sqrt(machine epsilon)
  Matrix pinv(T eps = -1) const {
    if (eps < 0) eps = std::sqrt(machine_eps<T>());
    Matrix r(d1_, d0_);
    mat::pinv(a_.data(), (int)d0_, (int)d1_, eps, r.a_.data());
    return r;
  }

 private:
  Long d0_ = 0, d1_ = 0;
  std::vector<T> a_;
};

}  // namespace sctl

#endif
