// Device-side building blocks of libpvfmm_b200: Morton keys, kernel
// functions, error handling and the per-context device buffers.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <stdexcept>
#include <string>
#include <vector>

namespace pvfmm_b200 {

#define PVFMM_CUDA_CHECK(expr)                                                                  \
  do {                                                                                          \
    cudaError_t err__ = (expr);                                                                 \
    if (err__ != cudaSuccess)                                                                   \
      throw std::runtime_error(std::string("CUDA error: ") + cudaGetErrorString(err__) + " at " \
                               + __FILE__ + ":" + std::to_string(__LINE__));                    \
  } while (0)

constexpr int kMaxDepth = 30;          // PVFMM_MAX_DEPTH (include/pvfmm_common.hpp:29)
constexpr double kRad0 = 1.05;         // PVFMM_RAD0
constexpr double kRad1 = 2.95;         // PVFMM_RAD1
constexpr uint32_t kTwo30 = 1u << 30;

// ---------------------------------------------------------------------------
// Morton keys.  The order of (hi, lo) equals MortonId::operator<
// (reference include/mortonid.txx:107-118): the most significant differing
// coordinate bit decides, z before y before x at equal bits; equal
// coordinates order by depth.  hi holds coordinate bits 29..9 interleaved
// (63 bits), lo holds bits 8..0 interleaved (27 bits) << 5 | depth.
// ---------------------------------------------------------------------------
struct MKey {
  unsigned long long hi;
  unsigned int lo;
  unsigned int pad;
};

__host__ __device__ inline bool key_less(const MKey& a, const MKey& b) {
  return a.hi < b.hi || (a.hi == b.hi && a.lo < b.lo);
}
__host__ __device__ inline bool key_eq(const MKey& a, const MKey& b) { return a.hi == b.hi && a.lo == b.lo; }

__host__ __device__ inline unsigned long long spread3(unsigned int v) {  // 21 bits -> every 3rd bit
  unsigned long long x = v & 0x1fffffu;
  x = (x | (x << 32)) & 0x1f00000000ffffULL;
  x = (x | (x << 16)) & 0x1f0000ff0000ffULL;
  x = (x | (x << 8)) & 0x100f00f00f00f00fULL;
  x = (x | (x << 4)) & 0x10c30c30c30c30c3ULL;
  x = (x | (x << 2)) & 0x1249249249249249ULL;
  return x;
}
__host__ __device__ inline unsigned int compact3(unsigned long long x) {
  x &= 0x1249249249249249ULL;
  x = (x | (x >> 2)) & 0x10c30c30c30c30c3ULL;
  x = (x | (x >> 4)) & 0x100f00f00f00f00fULL;
  x = (x | (x >> 8)) & 0x1f0000ff0000ffULL;
  x = (x | (x >> 16)) & 0x1f00000000ffffULL;
  x = (x | (x >> 32)) & 0x1fffffULL;
  return (unsigned int)x;
}

__host__ __device__ inline MKey make_key(unsigned int X, unsigned int Y, unsigned int Z, unsigned int depth) {
  MKey k;
  k.hi = spread3(X >> 9) | (spread3(Y >> 9) << 1) | (spread3(Z >> 9) << 2);
  const unsigned long long l = spread3(X & 511u) | (spread3(Y & 511u) << 1) | (spread3(Z & 511u) << 2);
  k.lo = (unsigned int)((l << 5) | depth);
  k.pad = 0;
  return k;
}

__host__ __device__ inline void decode_key(const MKey& k, unsigned int& X, unsigned int& Y, unsigned int& Z,
                                           unsigned int& depth) {
  const unsigned long long l = k.lo >> 5;
  X = (compact3(k.hi) << 9) | compact3(l);
  Y = (compact3(k.hi >> 1) << 9) | compact3(l >> 1);
  Z = (compact3(k.hi >> 2) << 9) | compact3(l >> 2);
  depth = k.lo & 31u;
}

// Key larger than every point in node (X,Y,Z,d) and smaller than every key
// after the node's subtree.
__host__ __device__ inline MKey node_end_key(unsigned int X, unsigned int Y, unsigned int Z, unsigned int d) {
  const unsigned int w = kTwo30 >> d;
  return make_key(X + w - 1, Y + w - 1, Z + w - 1, 31);
}

// First index i in sorted [0,n) with !(a[i] < k).
__device__ inline long lower_bound_key(const MKey* a, long n, const MKey& k) {
  long lo = 0, hi = n;
  while (lo < hi) {
    const long mid = (lo + hi) >> 1;
    if (key_less(a[mid], k)) lo = mid + 1;
    else hi = mid;
  }
  return lo;
}

// ---------------------------------------------------------------------------
// Reciprocal square root with the kernels' r == 0 mask (kernel.txx:1283).
// FP64: FP32 hardware estimate refined by two Newton-Raphson steps
// y <- y (3/2 - r2 y^2 / 2) in FP64 (from a 2^-22 estimate two steps reach
// full double accuracy); r2 below the FP32 normal range takes the FP64
// library rsqrt.  FP32: hardware estimate + one Newton step.
// ---------------------------------------------------------------------------
__device__ __forceinline__ double rsqrt_nr(double r2) {
  if (r2 < 1e-30) return r2 > 0 ? rsqrt(r2) : 0.0;
  double y = (double)rsqrtf((float)r2);
  const double h = 0.5 * r2;
  y = y * (1.5 - h * y * y);
  y = y * (1.5 - h * y * y);
  return y;
}
// FP32: one hardware reciprocal square root (rsqrt.approx.ftz, relative
// error about 2^-22) refined by one Newton-Raphson step for f(y) = 1/y^2 - x,
// y <- y (3 - x y^2) / 2; 0 for r2 == 0 (and for r2 below the FP32 normal
// range, which flushes to zero).  Without the step the potential is as
// accurate, but the approximation's error is not sign-balanced and builds up
// in gradients, whose near-field terms largely cancel (1e-5 instead of 1e-6
// relative on position derivatives at 1M points).
__device__ __forceinline__ float rsqrt_nr(float r2) {
  float y0;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y0) : "f"(r2));
  const float y = y0 * (1.5f - 0.5f * r2 * y0 * y0);
  return r2 > 0.f ? y : 0.f;
}
// FP64 with one Newton step from the FP32 seed (relative error ~1e-13), for
// r2 in the FP32 normal range; used where the pair distance is bounded away
// from zero (equivalent-surface sources).
__device__ __forceinline__ double rsqrt_nr1(double r2) {
  float y0;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(y0) : "f"((float)r2));
  const double y = (double)y0;
  return y * (1.5 - 0.5 * r2 * y * y);
}

// ---------------------------------------------------------------------------
// Kernel functions (reference include/kernel.txx:1276-1364), unscaled: the
// 1/(4 pi) or 1/(8 pi) factor is applied once to the summed result, as
// GenericKernel::Eval does after each source block (kernel.txx:1243-1246).
// KS: number of source components, KT: number of target components.
// ---------------------------------------------------------------------------
enum KerType {
  kKerLaplace = 0,
  kKerLaplaceGrad = 1,
  kKerStokes = 2,
  kKerLaplacePG = 3,
  kKerStokesPress = 4,  // stokes_press_, kernel.txx:1366-1378
  kKerStokesGrad = 5,   // stokes_grad_, kernel.txx:1404-1432
  kKerBiotSavart = 6,   // biot_savart_, kernel.txx:1492-1506
  // double-layer kernels: KS = k0 + 3 source values per point (density and
  // normal, read in the order the reference's uKerEval reads them)
  kKerLaplaceDbl = 7,   // laplace_dbl_poten_, kernel.txx:1299-1311
  kKerStokesDbl = 8     // stokes_sym_dip_, kernel.txx:1437-1456
};

template <int Ker>
struct KerDims;
template <>
struct KerDims<kKerLaplace> { static constexpr int KS = 1, KT = 1; };
template <>
struct KerDims<kKerLaplaceGrad> { static constexpr int KS = 1, KT = 3; };
template <>
struct KerDims<kKerStokes> { static constexpr int KS = 3, KT = 3; };
template <>
struct KerDims<kKerLaplacePG> { static constexpr int KS = 1, KT = 4; };
template <>
struct KerDims<kKerStokesPress> { static constexpr int KS = 3, KT = 1; };
template <>
struct KerDims<kKerStokesGrad> { static constexpr int KS = 3, KT = 9; };
template <>
struct KerDims<kKerBiotSavart> { static constexpr int KS = 3, KT = 3; };
template <>
struct KerDims<kKerLaplaceDbl> { static constexpr int KS = 4, KT = 1; };
template <>
struct KerDims<kKerStokesDbl> { static constexpr int KS = 6, KT = 3; };

// Adds K(r) f to u (r = target - source).
// Surface1 = true: the source is an equivalent-surface point at a distance
// bounded away from zero, and FP64 needs only one Newton step.
template <int Ker, class Real, bool Surface1 = false>
__device__ __forceinline__ void ker_eval(Real rx, Real ry, Real rz, const Real* f, Real* u) {
  const Real r2 = rx * rx + ry * ry + rz * rz;
  Real rinv;
  if constexpr (Surface1 && sizeof(Real) == 8) rinv = rsqrt_nr1(r2);
  else rinv = rsqrt_nr(r2);
  if constexpr (Ker == kKerLaplace) {
    u[0] += rinv * f[0];
  } else if constexpr (Ker == kKerLaplaceGrad) {
    const Real fr3 = rinv * rinv * rinv * f[0];
    u[0] += rx * fr3;
    u[1] += ry * fr3;
    u[2] += rz * fr3;
  } else if constexpr (Ker == kKerLaplacePG) {
    const Real fr = rinv * f[0];
    const Real fr3 = rinv * rinv * fr;
    u[0] += fr;
    u[1] += rx * fr3;
    u[2] += ry * fr3;
    u[3] += rz * fr3;
  } else if constexpr (Ker == kKerStokesPress) {  // (r . f) / r^3
    const Real rinv3 = rinv * rinv * rinv;
    u[0] += (rx * f[0] + ry * f[1] + rz * f[2]) * rinv3;
  } else if constexpr (Ker == kKerStokesGrad) {
    // u[3i+j] += (delta_ij (r.f) + r_j f_i - f_j r_i - 3 (r.f) r_i r_j / r^2) / r^3
    const Real rinv2 = rinv * rinv, rinv3 = rinv2 * rinv;
    const Real ip = f[0] * rx + f[1] * ry + f[2] * rz;
    const Real r[3] = {rx, ry, rz};
    const Real c3 = (Real)3 * ip * rinv2;
#pragma unroll
    for (int i = 0; i < 3; ++i)
#pragma unroll
      for (int j = 0; j < 3; ++j) {
        Real v = r[j] * f[i] - f[j] * r[i] - c3 * r[i] * r[j];
        if (i == j) v += ip;
        u[3 * i + j] += v * rinv3;
      }
  } else if constexpr (Ker == kKerBiotSavart) {  // (f x r) / r^3
    const Real rinv3 = rinv * rinv * rinv;
    u[0] += rinv3 * (f[1] * rz - f[2] * ry);
    u[1] += rinv3 * (f[2] * rx - f[0] * rz);
    u[2] += rinv3 * (f[0] * ry - f[1] * rx);
  } else if constexpr (Ker == kKerLaplaceDbl) {  // (r . f[0:3]) f[3] / r^3
    const Real rinv3 = rinv * rinv * rinv;
    u[0] += (rx * f[0] + ry * f[1] + rz * f[2]) * rinv3 * f[3];
  } else if constexpr (Ker == kKerStokesDbl) {
    // f = v[0:3], n = v[3:6]; n.f is formed as v0 v3 + v1 v1 + v2 v2, as the
    // reference forms it; u += r (n.f - 3 (r.n)(r.f) / r^2) / r^3
    const Real rinv2 = rinv * rinv, rinv3 = rinv2 * rinv;
    const Real rdf = f[0] * rx + f[1] * ry + f[2] * rz;
    const Real rdn = f[3] * rx + f[4] * ry + f[5] * rz;
    const Real ndf = f[0] * f[3] + f[1] * f[1] + f[2] * f[2];
    const Real common = (ndf - (Real)3 * rdn * rdf * rinv2) * rinv3;
    u[0] += rx * common;
    u[1] += ry * common;
    u[2] += rz * common;
  } else {  // Stokes velocity
    const Real rinv2 = rinv * rinv;
    const Real ip = (f[0] * rx + f[1] * ry + f[2] * rz) * rinv2;
    u[0] += rinv * (f[0] + rx * ip);
    u[1] += rinv * (f[1] + ry * ip);
    u[2] += rinv * (f[2] + rz * ip);
  }
}

// 1/(8 pi) for Stokes velocity and velocity gradient, -1/(8 pi) for the
// Stokes double layer, 1/(4 pi) otherwise (the kernels' ScaleFactor,
// kernel.txx:1278, 1301, 1353, 1368, 1407, 1436, 1494).
__host__ __device__ constexpr double ker_scale(int ker) {
  return (ker == kKerStokes || ker == kKerStokesGrad) ? 1.0 / (8 * 3.14159265358979323846)
         : ker == kKerStokesDbl                       ? -1.0 / (8 * 3.14159265358979323846)
                                                      : 1.0 / (4 * 3.14159265358979323846);
}

// ---------------------------------------------------------------------------
// Reusable device buffer: grows, never shrinks, freed with the context.
// ---------------------------------------------------------------------------
struct DevBuf {
  void* ptr = nullptr;
  size_t cap = 0;
  void* ensure(size_t bytes) {
    if (bytes == 0) bytes = 16;
    if (bytes > cap) {
      if (ptr) PVFMM_CUDA_CHECK(cudaFree(ptr));
      ptr = nullptr;
      cap = 0;
      const cudaError_t e = cudaMalloc(&ptr, bytes);
      if (e != cudaSuccess) {
        cudaGetLastError();
        size_t fr = 0, tot = 0;
        cudaMemGetInfo(&fr, &tot);
        throw std::runtime_error("device allocation of " + std::to_string(bytes >> 20) + " MiB failed (" +
                                 cudaGetErrorString(e) + "; " + std::to_string(fr >> 20) + " MiB free of " +
                                 std::to_string(tot >> 20) + ")");
      }
      cap = bytes;
    }
    return ptr;
  }
  template <class T>
  T* as(size_t n) {
    return static_cast<T*>(ensure(n * sizeof(T)));
  }
  template <class T>
  T* get() const {
    return static_cast<T*>(ptr);
  }
  void release() {
    if (ptr) cudaFree(ptr);
    ptr = nullptr;
    cap = 0;
  }
};

inline unsigned int ceil_div(long a, long b) { return (unsigned int)((a + b - 1) / b); }

// FP64 tensor cores: D (8x8) += A (8x4, row) * B (4x8, col).  Lane l = 4g + t
// holds a = A[g][t], b = B[t][g], d = (D[g][2t], D[g][2t+1]).
__device__ __forceinline__ void dmma(double (&d)[2], double a, double b) {
  asm volatile("mma.sync.aligned.m8n8k4.row.col.f64.f64.f64.f64 {%0,%1}, {%2}, {%3}, {%0,%1};\n"
               : "+d"(d[0]), "+d"(d[1])
               : "d"(a), "d"(b));
}

}  // namespace pvfmm_b200
