// FMM evaluation on the device (FMM_Tree::RunFMM, reference
// include/fmm_tree.txx:237-738, evaluation halves of include/fmm_pts.txx).
//
// Data layout in HBM:
//   points     sorted by Morton key; FP64 SoA coordinates relative to the
//              centre of the point's leaf; FP64 densities [n_src][k0]
//   UE, DC     FP64 per node, [n_nodes][ns*ke]: upward equivalent densities
//              and downward check potentials (the reference's upward_equiv
//              and dnward_equiv, fmm_pts.txx:1306-1480)
//   spectra    per V-list parent, [parent][freq][child*ke+comp] complex, in
//              the working precision Real
// Precision forms:
//   plain  Real = double everywhere.
//   mixed  Real = float for the two dominant stages, the V-list (DFTs and
//          Hadamard products) and the near field (U list P2P, W list, D2T
//          target evaluation); FP32 tile sums are promoted to FP64 per
//          tile.  The check->equivalent chain (S2U and X check potentials,
//          the pseudo-inverse GEMMs, U2U, D2D) stays FP64: the SVD
//          pseudo-inverse amplifies check-potential errors by up to 1/(4 eps
//          max S), so FP32 check potentials would need the FP32 cutoff,
//          which alone costs ~8e-7 relative error at m=8.
// Stages:
//   S2U   check-surface evaluation + 2 FP64 tensor-core products (pinv
//         factors, fmm_pts.txx:4390-4426), the second one writing the leaves'
//         rows of UE (translate.cu)
//   U2U   one product per level over the contiguous child blocks, written to
//         the parents' rows (fmm_pts.txx:2017-2271)
//   V     pruned DFT of the 8 children, Hadamard with the 26 parent offsets,
//         pruned inverse DFT onto the children's check surfaces (fmm_pts.txx:2689-3759)
//   X     check-surface evaluation (fmm_pts.txx:4444-4736)
//   D2D   one product per level from the parents' rows into the contiguous
//         child blocks (fmm_pts.txx:3762-3790)
//   D2T   2 products (pinv factors, leaves' rows gathered and scaled by
//         2^-depth in the first), then with W and U one fused near-field
//         kernel per target leaf (fmm_pts.txx:4246-4426, 4746-5022, 5032-5418).
#include <algorithm>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <functional>

#include "fmm_context.cuh"

namespace pvfmm_b200 {
namespace {

constexpr int kNT = 128;  // threads per block of the point/surface kernels

template <class Real>
struct Cplx {
  Real re, im;
};

__device__ __forceinline__ void node_geom(const MKey& k, double& cx, double& cy, double& cz, double& half, int& depth) {
  unsigned int X, Y, Z, d;
  decode_key(k, X, Y, Z, d);
  const double h = 1.0 / (double)(1u << d);
  half = 0.5 * h;
  cx = X * (1.0 / kTwo30) + half;
  cy = Y * (1.0 / kTwo30) + half;
  cz = Z * (1.0 / kTwo30) + half;
  depth = (int)d;
}

// Periodic boundaries: moves a source node's centre by the unit-cube image
// shift of its list entry (code (sx+1) + 3(sy+1) + 9(sz+1)).
__device__ __forceinline__ void image_shift(unsigned char code, double& cx, double& cy, double& cz) {
  cx += (double)(code % 3) - 1.0;
  cy += (double)((code / 3) % 3) - 1.0;
  cz += (double)(code / 9) - 1.0;
}

// ---------------------------------------------------------------------------
// Source tiles in shared memory and the per-thread evaluation loop.
// ---------------------------------------------------------------------------
template <class Real, int KS>
struct Tile {
  Real x[kNT], y[kNT], z[kNT], f[KS][kNT];
  // FP32 tiles carry the rounding remainder of each coordinate, so that the
  // difference target - source is as accurate as FP32 rounding of the
  // difference itself (close pairs dominate the gradient kernels).
  Real xl[sizeof(Real) == 4 ? kNT : 1], yl[sizeof(Real) == 4 ? kNT : 1], zl[sizeof(Real) == 4 ? kNT : 1];
};

// Target coordinate as (hi, lo) in Real.
template <class Real>
struct Pt {
  Real x, y, z, xl, yl, zl;
};
template <class Real>
__device__ __forceinline__ Pt<Real> make_pt(double x, double y, double z) {
  Pt<Real> p;
  p.x = (Real)x;
  p.y = (Real)y;
  p.z = (Real)z;
  p.xl = (Real)(x - (double)p.x);
  p.yl = (Real)(y - (double)p.y);
  p.zl = (Real)(z - (double)p.z);
  return p;
}

template <class Real, int KS>
__device__ __forceinline__ void tile_store(Tile<Real, KS>& tl, int i, double x, double y, double z) {
  tl.x[i] = (Real)x;
  tl.y[i] = (Real)y;
  tl.z[i] = (Real)z;
  if constexpr (sizeof(Real) == 4) {
    tl.xl[i] = (Real)(x - (double)tl.x[i]);
    tl.yl[i] = (Real)(y - (double)tl.y[i]);
    tl.zl[i] = (Real)(z - (double)tl.z[i]);
  }
}

template <class Real, int KS>
__device__ __forceinline__ void tile_diff(const Tile<Real, KS>& tl, int j, const Pt<Real>& p, Real& rx, Real& ry,
                                          Real& rz) {
  if constexpr (sizeof(Real) == 4) {
    rx = (p.x - tl.x[j]) + (p.xl - tl.xl[j]);
    ry = (p.y - tl.y[j]) + (p.yl - tl.yl[j]);
    rz = (p.z - tl.z[j]) + (p.zl - tl.zl[j]);
  } else {
    rx = p.x - tl.x[j];
    ry = p.y - tl.y[j];
    rz = p.z - tl.z[j];
  }
}

// Sums sources j = j0, j0+js, ... < n of the tile into acc (FP64).  Two
// independent partial sums in Real give ILP; the tile sum is promoted to
// FP64, so FP32 rounding never accumulates over more than one tile.
template <class Real, int Ker, bool Surface1 = false>
__device__ __forceinline__ void tile_sum(const Tile<Real, KerDims<Ker>::KS>& tl, int n, int j0, int js,
                                         const Pt<Real>& p, double* acc) {
  constexpr int KS = KerDims<Ker>::KS, KT = KerDims<Ker>::KT;
  Real u0[KT], u1[KT];
#pragma unroll
  for (int k = 0; k < KT; ++k) u0[k] = u1[k] = 0;
  int j = j0;
  for (; j + js < n; j += 2 * js) {
    Real f0[KS], f1[KS];
#pragma unroll
    for (int i = 0; i < KS; ++i) {
      f0[i] = tl.f[i][j];
      f1[i] = tl.f[i][j + js];
    }
    Real rx, ry, rz;
    tile_diff(tl, j, p, rx, ry, rz);
    ker_eval<Ker, Real, Surface1>(rx, ry, rz, f0, u0);
    tile_diff(tl, j + js, p, rx, ry, rz);
    ker_eval<Ker, Real, Surface1>(rx, ry, rz, f1, u1);
  }
  if (j < n) {
    Real f0[KS];
#pragma unroll
    for (int i = 0; i < KS; ++i) f0[i] = tl.f[i][j];
    Real rx, ry, rz;
    tile_diff(tl, j, p, rx, ry, rz);
    ker_eval<Ker, Real, Surface1>(rx, ry, rz, f0, u0);
  }
#pragma unroll
  for (int k = 0; k < KT; ++k) acc[k] += (double)u0[k] + (double)u1[k];
}

// Work split of a block over a chunk of nc targets: thread t evaluates target
// t % nc against the sources j == t / nc (mod G) of every tile.
struct Split {
  int nc, G, ti, g;
  bool active;
  __device__ explicit Split(int n_targets) {
    nc = max(1, min(kNT, n_targets));
    G = min(8, kNT / nc);
    ti = threadIdx.x % nc;
    g = threadIdx.x / nc;
    active = g < G && ti < n_targets;
  }
};

// Sources = sorted points [lo,hi) of a leaf whose centre is at offset (ox,oy,oz).
template <class Real, int Ker, bool Surface1 = false>
__device__ void point_sources(Tile<Real, KerDims<Ker>::KS>& tl, const double* __restrict__ sx,
                              const double* __restrict__ sy, const double* __restrict__ sz,
                              const double* __restrict__ den, int lo, int hi, double ox, double oy, double oz,
                              const Split& sp, const Pt<Real>& pt, double* acc) {
  constexpr int KS = KerDims<Ker>::KS;
  for (int p0 = lo; p0 < hi; p0 += kNT) {
    const int n = min(kNT, hi - p0);
    __syncthreads();
    if (threadIdx.x < n) {
      const int p = p0 + threadIdx.x;
      tile_store(tl, threadIdx.x, sx[p] + ox, sy[p] + oy, sz[p] + oz);
#pragma unroll
      for (int i = 0; i < KS; ++i) tl.f[i][threadIdx.x] = (Real)den[(long)p * KS + i];
    }
    __syncthreads();
    if (sp.active) tile_sum<Real, Ker, Surface1>(tl, n, sp.g, sp.G, pt, acc);
  }
}

// Adds the G partial sums of each target (deterministic order) and stores.
template <int KT>
__device__ void reduce_store(double (*red)[KT], const Split& sp, const double* acc, double scale, double* out,
                             bool accumulate) {
  __syncthreads();
  if (sp.active)
#pragma unroll
    for (int k = 0; k < KT; ++k) red[threadIdx.x][k] = acc[k];
  __syncthreads();
  if (sp.active && sp.g == 0) {
    double s[KT];
#pragma unroll
    for (int k = 0; k < KT; ++k) s[k] = red[sp.ti][k];
    for (int g = 1; g < sp.G; ++g)
#pragma unroll
      for (int k = 0; k < KT; ++k) s[k] += red[g * sp.nc + sp.ti][k];
#pragma unroll
    for (int k = 0; k < KT; ++k) {
      if (accumulate) out[sp.ti * KT + k] += s[k] * scale;
      else out[sp.ti * KT + k] = s[k] * scale;
    }
  }
}

// ---------------------------------------------------------------------------
// Near field of one target leaf: D2T (own downward equivalent surface), W
// (upward equivalent surfaces of the W list) and U (points of the P2P list),
// fused.  One block per target leaf.
//
// The sources of all list entries are packed back to back into tiles of
// kTile records in shared memory (leaves hold a few dozen points, so one tile
// spans many entries), double-buffered so that one barrier per tile suffices.
// A record is one source point relative to the target leaf's centre plus its
// KS densities, stored as 16-byte chunks, chunk-major.  FP32 records also
// carry each coordinate's rounding remainder (hi + lo), so target - source
// keeps FP32 relative accuracy for close pairs.  Every thread evaluates two
// targets per loaded record; when a leaf has fewer than 2*kNF targets the
// source records are split among G groups of threads and the G partial sums
// are added in a fixed order.
// ---------------------------------------------------------------------------
constexpr int kNF = 128;        // threads per near-field block
#ifndef PVFMM_NEAR_MIN_BLOCKS_F32
#define PVFMM_NEAR_MIN_BLOCKS_F32 5  // resident blocks per SM the register budget is sized for
#endif
#ifndef PVFMM_NEAR_MIN_BLOCKS_F32_K1
#define PVFMM_NEAR_MIN_BLOCKS_F32_K1 6  // the same for one source density (Laplace kernels)
#endif
#ifndef PVFMM_NEAR_MIN_BLOCKS_F64
#define PVFMM_NEAR_MIN_BLOCKS_F64 5
#endif
#ifndef PVFMM_NEAR_TILE_MULT
#define PVFMM_NEAR_TILE_MULT 2
#endif
#ifndef PVFMM_NEAR_UNROLL
#define PVFMM_NEAR_UNROLL 1
#endif
#ifndef PVFMM_NEAR_GMAX
#define PVFMM_NEAR_GMAX 16  // most thread groups splitting the source records of a small leaf
#endif

constexpr int kNearUnroll = PVFMM_NEAR_UNROLL;      // unroll of the record loop
constexpr int kTile = PVFMM_NEAR_TILE_MULT * kNF;  // source records per tile
#ifndef PVFMM_NEAR_TILE_MULT_K1
#define PVFMM_NEAR_TILE_MULT_K1 2
#endif
// records per tile of the near-field kernel for Real, Ker (the FP32 kernels
// with one source density have the smallest records)
template <class Real, int Ker>
constexpr int near_tile() {
  return sizeof(Real) == 4 && KerDims<Ker>::KS == 1 ? PVFMM_NEAR_TILE_MULT_K1 * kNF : kTile;
}

template <class Real>
struct Vec16 {
  using type = double2;
};
template <>
struct Vec16<float> {
  using type = float4;
};

template <class Real, int KS>
struct Rec {
  static constexpr bool kLo = sizeof(Real) == 4;
  static constexpr int NV = (kLo ? 6 : 3) + KS;
  static constexpr int PER = 16 / (int)sizeof(Real);
  static constexpr int NC = (NV + PER - 1) / PER;
  static constexpr int NVP = NC * PER;
  // value slots: x y z f0 | xl yl zl f1 f2 (FP32);  x y z f0 f1 f2 (FP64)
  __host__ __device__ static constexpr int F(int i) { return kLo ? (i == 0 ? 3 : 6 + i) : 3 + i; }
};

template <class Real, int KS, int TS = kTile>
__device__ __forceinline__ void rec_store(typename Vec16<Real>::type* tile, int j, double x, double y, double z,
                                          const Real* f) {
  using R = Rec<Real, KS>;
  Real v[R::NVP];
#pragma unroll
  for (int i = 0; i < R::NVP; ++i) v[i] = 0;
  v[0] = (Real)x;
  v[1] = (Real)y;
  v[2] = (Real)z;
  if constexpr (R::kLo) {
    v[4] = (Real)(x - (double)v[0]);
    v[5] = (Real)(y - (double)v[1]);
    v[6] = (Real)(z - (double)v[2]);
  }
#pragma unroll
  for (int i = 0; i < KS; ++i) v[R::F(i)] = f[i];
#pragma unroll
  for (int c = 0; c < R::NC; ++c) {
    typename Vec16<Real>::type w;
    memcpy(&w, &v[c * R::PER], 16);
    tile[c * TS + j] = w;
  }
}

// Adds the records j = j0, j0+js, ... < n to two targets (FP64 accumulators;
// FP32 sums never run over more than one tile).
template <class Real, int Ker, bool Surface1 = false, int TS = kTile>
__device__ __forceinline__ void rec_sum2(const typename Vec16<Real>::type* tile, int n, int j0, int js,
                                         const Pt<Real>& pa, const Pt<Real>& pb, double (&acc)[2][KerDims<Ker>::KT]) {
  constexpr int KS = KerDims<Ker>::KS, KT = KerDims<Ker>::KT;
  using R = Rec<Real, KS>;
  // FP32 partial sums run over 16 records at most before going to FP64
  const int step = sizeof(Real) == 4 ? 16 * js : n;
  for (int jb = j0; jb < n; jb += step) {
  const int jend = sizeof(Real) == 4 ? min(n, jb + step) : n;
  Real ua[KT], ub[KT];
#pragma unroll
  for (int k = 0; k < KT; ++k) ua[k] = ub[k] = 0;
#pragma unroll kNearUnroll
  for (int j = jb; j < jend; j += js) {
    Real v[R::NVP];
#pragma unroll
    for (int c = 0; c < R::NC; ++c) {
      const typename Vec16<Real>::type w = tile[c * TS + j];
      memcpy(&v[c * R::PER], &w, 16);
    }
    Real f[KS];
#pragma unroll
    for (int i = 0; i < KS; ++i) f[i] = v[R::F(i)];
    Real rx, ry, rz;
    if constexpr (R::kLo) {
      rx = (pa.x - v[0]) + (pa.xl - v[4]);
      ry = (pa.y - v[1]) + (pa.yl - v[5]);
      rz = (pa.z - v[2]) + (pa.zl - v[6]);
    } else {
      rx = pa.x - v[0];
      ry = pa.y - v[1];
      rz = pa.z - v[2];
    }
    ker_eval<Ker, Real, Surface1>(rx, ry, rz, f, ua);
    if constexpr (R::kLo) {
      rx = (pb.x - v[0]) + (pb.xl - v[4]);
      ry = (pb.y - v[1]) + (pb.yl - v[5]);
      rz = (pb.z - v[2]) + (pb.zl - v[6]);
    } else {
      rx = pb.x - v[0];
      ry = pb.y - v[1];
      rz = pb.z - v[2];
    }
    ker_eval<Ker, Real, Surface1>(rx, ry, rz, f, ub);
  }
#pragma unroll
  for (int k = 0; k < KT; ++k) {
    acc[0][k] += (double)ua[k];
    acc[1][k] += (double)ub[k];
  }
  }
}

// ---------------------------------------------------------------------------
// Packed FP32 pairs (add/sub/mul/fma .f32x2 of sm_100): the mixed form's near
// field evaluates a source record against its thread's two targets in the two
// halves of 64-bit registers, one instruction per operation for both targets
// (the same round-to-nearest FP32 operations as two scalar evaluations).
// ---------------------------------------------------------------------------
typedef unsigned long long f2_t;
__device__ __forceinline__ f2_t f2_pack(float lo, float hi) {
  f2_t r;
  asm("mov.b64 %0, {%1, %2};" : "=l"(r) : "f"(lo), "f"(hi));
  return r;
}
__device__ __forceinline__ void f2_unpack(f2_t v, float& lo, float& hi) {
  asm("mov.b64 {%0, %1}, %2;" : "=f"(lo), "=f"(hi) : "l"(v));
}
__device__ __forceinline__ f2_t f2_add(f2_t a, f2_t b) {
  f2_t d;
  asm("add.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2_t f2_sub(f2_t a, f2_t b) {
  f2_t d;
  asm("sub.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2_t f2_mul(f2_t a, f2_t b) {
  f2_t d;
  asm("mul.rn.f32x2 %0, %1, %2;" : "=l"(d) : "l"(a), "l"(b));
  return d;
}
__device__ __forceinline__ f2_t f2_fma(f2_t a, f2_t b, f2_t c) {
  f2_t d;
  asm("fma.rn.f32x2 %0, %1, %2, %3;" : "=l"(d) : "l"(a), "l"(b), "l"(c));
  return d;
}

// Kernels with a packed form (the others evaluate the two targets in turn).
template <int Ker>
constexpr bool kHasPacked = Ker == kKerLaplace || Ker == kKerLaplaceGrad || Ker == kKerLaplacePG || Ker == kKerStokes;

// ker_eval<Ker, float> for two targets at once: r = target - source per half,
// f the source densities (the same in both halves).  1/r: one hardware
// reciprocal square root per half (0 for r2 == 0) and one packed
// Newton-Raphson step y <- y (3/2 - r2 y^2 / 2), as rsqrt_nr(float).
template <int Ker>
__device__ __forceinline__ void ker_eval_x2(f2_t rx, f2_t ry, f2_t rz, const f2_t* f, f2_t* u) {
  const f2_t r2 = f2_fma(rz, rz, f2_fma(ry, ry, f2_mul(rx, rx)));
  float a, b;
  f2_unpack(r2, a, b);
  float ya, yb;
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(ya) : "f"(a));
  asm("rsqrt.approx.ftz.f32 %0, %1;" : "=f"(yb) : "f"(b));
  ya = a > 0.f ? ya : 0.f;
  yb = b > 0.f ? yb : 0.f;
  f2_t y = f2_pack(ya, yb);
  const f2_t half = f2_pack(0.5f, 0.5f), three_half = f2_pack(1.5f, 1.5f);
  y = f2_mul(y, f2_sub(three_half, f2_mul(f2_mul(half, r2), f2_mul(y, y))));
  if constexpr (Ker == kKerLaplace) {
    u[0] = f2_fma(y, f[0], u[0]);
  } else if constexpr (Ker == kKerLaplaceGrad) {
    const f2_t fr3 = f2_mul(f2_mul(y, y), f2_mul(y, f[0]));
    u[0] = f2_fma(rx, fr3, u[0]);
    u[1] = f2_fma(ry, fr3, u[1]);
    u[2] = f2_fma(rz, fr3, u[2]);
  } else if constexpr (Ker == kKerLaplacePG) {
    const f2_t fr = f2_mul(y, f[0]);
    const f2_t fr3 = f2_mul(f2_mul(y, y), fr);
    u[0] = f2_add(u[0], fr);
    u[1] = f2_fma(rx, fr3, u[1]);
    u[2] = f2_fma(ry, fr3, u[2]);
    u[3] = f2_fma(rz, fr3, u[3]);
  } else {  // Stokes velocity: u += (f + r (f.r) / r^2) / r
    const f2_t ip = f2_mul(f2_fma(f[2], rz, f2_fma(f[1], ry, f2_mul(f[0], rx))), f2_mul(y, y));
    u[0] = f2_fma(y, f2_fma(rx, ip, f[0]), u[0]);
    u[1] = f2_fma(y, f2_fma(ry, ip, f[1]), u[1]);
    u[2] = f2_fma(y, f2_fma(rz, ip, f[2]), u[2]);
  }
}

// rec_sum2 for FP32 records with the packed pair evaluation.
template <int Ker, int TS = kTile>
__device__ __forceinline__ void rec_sum2_x2(const float4* tile, int n, int j0, int js, const Pt<float>& pa,
                                            const Pt<float>& pb, double (&acc)[2][KerDims<Ker>::KT]) {
  constexpr int KS = KerDims<Ker>::KS, KT = KerDims<Ker>::KT;
  using R = Rec<float, KS>;
  const f2_t px = f2_pack(pa.x, pb.x), py = f2_pack(pa.y, pb.y), pz = f2_pack(pa.z, pb.z);
  const f2_t pxl = f2_pack(pa.xl, pb.xl), pyl = f2_pack(pa.yl, pb.yl), pzl = f2_pack(pa.zl, pb.zl);
  // FP32 partial sums run over 16 records at most before going to FP64
  const int step = 16 * js;
  for (int jb = j0; jb < n; jb += step) {
    const int jend = min(n, jb + step);
    f2_t u[KT];
#pragma unroll
    for (int k = 0; k < KT; ++k) u[k] = 0ull;  // (0.f, 0.f)
#pragma unroll kNearUnroll
    for (int j = jb; j < jend; j += js) {
      float v[R::NVP];
#pragma unroll
      for (int c = 0; c < R::NC; ++c) {
        const float4 w = tile[c * TS + j];
        memcpy(&v[c * R::PER], &w, 16);
      }
      f2_t f[KS];
#pragma unroll
      for (int i = 0; i < KS; ++i) f[i] = f2_pack(v[R::F(i)], v[R::F(i)]);
      const f2_t rx = f2_add(f2_sub(px, f2_pack(v[0], v[0])), f2_sub(pxl, f2_pack(v[4], v[4])));
      const f2_t ry = f2_add(f2_sub(py, f2_pack(v[1], v[1])), f2_sub(pyl, f2_pack(v[5], v[5])));
      const f2_t rz = f2_add(f2_sub(pz, f2_pack(v[2], v[2])), f2_sub(pzl, f2_pack(v[6], v[6])));
      ker_eval_x2<Ker>(rx, ry, rz, f, u);
    }
#pragma unroll
    for (int k = 0; k < KT; ++k) {
      float a, b;
      f2_unpack(u[k], a, b);
      acc[0][k] += (double)a;
      acc[1][k] += (double)b;
    }
  }
}

// One list entry of a target leaf as a segment of the packed source stream:
// the points of a leaf (kind 0, `node` = first point), the upward equivalent
// surface of a node (kind 1, `node` = node index) or the leaf's own downward
// equivalent surface (kind 2, `node` = row of the D2T densities).  The offset
// between node centres is a small multiple of a power of two, exact in FP32.
struct NearSeg {
  float ox, oy, oz;
  int node;
  int kind_depth;  // kind | depth << 4
};
constexpr int kSegCap = 128;  // list entries per batch

// kDbl: the double-layer pass, P2P sources only (surface values in `den`),
// added to pot.  with_p2p = 0: no P2P sources (no single-layer densities;
// the W and D2T entries still come from the expansions).
template <class Real, int Ker, bool kDbl = false>
__global__ void __launch_bounds__(kNF, sizeof(Real) == 8       ? PVFMM_NEAR_MIN_BLOCKS_F64
                                       : KerDims<Ker>::KS == 1 ? PVFMM_NEAR_MIN_BLOCKS_F32_K1
                                                               : PVFMM_NEAR_MIN_BLOCKS_F32)
    near_field_kernel(const int* __restrict__ tleaf, const MKey* __restrict__ keys, const int* __restrict__ tlo,
                      const int* __restrict__ thi, const int* __restrict__ slo, const int* __restrict__ shi,
                      const int* __restrict__ p_off, const int* __restrict__ p_list, const int* __restrict__ w_off,
                      const int* __restrict__ w_list, const unsigned char* __restrict__ p_img,
                      const unsigned char* __restrict__ w_img, const double* __restrict__ tx,
                      const double* __restrict__ ty, const double* __restrict__ tz, const double* __restrict__ sx,
                      const double* __restrict__ sy, const double* __restrict__ sz, const double* __restrict__ den,
                      const double* __restrict__ ue, const double* __restrict__ de, const double* __restrict__ usurf,
                      int ns, double scale, int with_p2p, double* __restrict__ pot) {
  constexpr int KS = KerDims<Ker>::KS, KT = KerDims<Ker>::KT;
  constexpr bool kF32 = sizeof(Real) == 4;
  constexpr bool kPacked = kF32 && kHasPacked<Ker>;
  constexpr int TPT = 2;  // targets per thread
  constexpr int TILE = near_tile<Real, Ker>();  // source records per tile
  constexpr int RPT = TILE / kNF;                 // records each thread fetches per tile
  using V = typename Vec16<Real>::type;
  __shared__ V tiles[2][Rec<Real, KS>::NC * TILE];
  // the FP64 D2T records of the mixed form come first and reuse the tiles
  // (a barrier separates their last read from the first tile store), and so
  // do the partial sums of the final fixed-order reduction
  static_assert(Rec<double, KS>::NC * 16 <= 2 * Rec<Real, KS>::NC * (int)sizeof(V), "D2T records fit the tiles");
  double2* tile64 = reinterpret_cast<double2*>(&tiles[0][0]);
  static_assert(sizeof(tiles) >= sizeof(double) * kNF * TPT * KT, "reduction buffer larger than the tiles");
  double(*red)[TPT][KT] = reinterpret_cast<double(*)[TPT][KT]>(&tiles[0][0]);
  __shared__ NearSeg seg[kSegCap];
  __shared__ int start[kSegCap + 1];
  const int b = blockIdx.x;
  const int T = tleaf[b];
  double cx, cy, cz, half;
  int dT;
  node_geom(keys[T], cx, cy, cz, half, dT);
  const int t0 = tlo[T], nt = thi[T] - t0;
  const int dim = ns * KS;
  const int wb = kDbl ? 0 : w_off[T], nW = kDbl ? 0 : w_off[T + 1] - wb;
  const int pbeg = p_off[T], nP = with_p2p ? p_off[T + 1] - pbeg : 0;
  const int nD = (!kDbl && de && !kF32) ? 1 : 0;  // plain form: D2T is a segment of the stream
  const int n_ent = nD + nW + nP;
  int buf = 0;
  for (int c0 = 0; c0 < nt; c0 += TPT * kNF) {
    // thread (ti, g): targets ti + q nc (q < TPT) of the chunk, source records
    // g, g + G, ... of every tile
    const int m = min(TPT * kNF, nt - c0);
    const int nc = (m + TPT - 1) / TPT;
    const int G = min(PVFMM_NEAR_GMAX, kNF / nc);
    const int ti = threadIdx.x % nc, g = threadIdx.x / nc;
    const bool active = g < G;
    int tq[TPT];
    Pt<Real> pt[TPT];
#pragma unroll
    for (int q = 0; q < TPT; ++q) {
      tq[q] = t0 + c0 + (ti + q * nc < m ? ti + q * nc : ti);  // a missing target repeats the first
      pt[q] = make_pt<Real>(tx[tq[q]], ty[tq[q]], tz[tq[q]]);
    }
    double acc[TPT][KT];
#pragma unroll
    for (int q = 0; q < TPT; ++q)
#pragma unroll
      for (int k = 0; k < KT; ++k) acc[q][k] = 0;
    // D2T of the mixed form: the downward equivalent densities come from the
    // FP64-cutoff pseudo-inverse, whose large cancelling components only FP64
    // sums resolve, so they are evaluated from FP64 records.
    if constexpr (kF32 && !kDbl) {
      if (de) {
        const double hr = half * kRad1;
        const double* dens = de + (long)b * dim;
        for (int k0 = 0; k0 < ns; k0 += TILE) {
          const int n = min(TILE, ns - k0);
          __syncthreads();
          for (int i = threadIdx.x; i < n; i += kNF) {
            const int k = k0 + i;
            double f[KS];
#pragma unroll
            for (int c = 0; c < KS; ++c) f[c] = dens[k * KS + c];
            rec_store<double, KS, TILE>(tile64, i, hr * usurf[k * 3 + 0], hr * usurf[k * 3 + 1],
                                        hr * usurf[k * 3 + 2], f);
          }
          __syncthreads();
          if (active)
#pragma unroll
            for (int h = 0; h < TPT / 2; ++h) {
              const Pt<double> pa64 = make_pt<double>(tx[tq[2 * h]], ty[tq[2 * h]], tz[tq[2 * h]]);
              const Pt<double> pb64 = make_pt<double>(tx[tq[2 * h + 1]], ty[tq[2 * h + 1]], tz[tq[2 * h + 1]]);
              rec_sum2<double, Ker, true, TILE>(tile64, n, g, G, pa64, pb64,
                                          *reinterpret_cast<double(*)[2][KT]>(&acc[2 * h][0]));
            }
        }
      }
    }
    for (int e0 = 0; e0 < n_ent; e0 += kSegCap) {
      const int ne = min(kSegCap, n_ent - e0);
      __syncthreads();  // the previous batch (or chunk) is done with seg, start and the tiles
      for (int i = threadIdx.x; i < ne; i += kNF) {
        const int e = e0 + i;
        NearSeg sg;
        int cnt;
        if (e < nD) {
          sg = {0.f, 0.f, 0.f, b, 2 | (dT << 4)};
          cnt = ns;
        } else {
          const bool is_w = e < nD + nW;
          const int q = is_w ? wb + e - nD : pbeg + e - nD - nW;
          const int S = is_w ? w_list[q] : p_list[q];
          double sxc, syc, szc, sh;
          int dS;
          node_geom(keys[S], sxc, syc, szc, sh, dS);
          if (p_img) image_shift(is_w ? w_img[q] : p_img[q], sxc, syc, szc);
          sg.ox = (float)(sxc - cx);
          sg.oy = (float)(syc - cy);
          sg.oz = (float)(szc - cz);
          if (is_w) {
            sg.node = S;
            sg.kind_depth = 1 | (dS << 4);
            cnt = ns;
          } else {
            sg.node = slo[S];
            sg.kind_depth = 0;
            cnt = shi[S] - slo[S];
          }
        }
        seg[i] = sg;
        start[i] = cnt;
      }
      __syncthreads();
      if (threadIdx.x < 32) {  // exclusive scan of the counts (4 entries per lane)
        const int lane = threadIdx.x;
        int v[4], sum = 0;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int idx = lane * 4 + q;
          v[q] = idx < ne ? start[idx] : 0;
          sum += v[q];
        }
        int inc = sum;
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
          const int y = __shfl_up_sync(0xffffffffu, inc, d);
          if (lane >= d) inc += y;
        }
        int ex = inc - sum;
#pragma unroll
        for (int q = 0; q < 4; ++q) {
          const int idx = lane * 4 + q;
          if (idx < ne) start[idx] = ex;
          ex += v[q];
        }
        if (lane == 31) start[ne] = inc;
      }
      __syncthreads();
      const int total = start[ne];
      const int ntile = (total + TILE - 1) / TILE;
      // records j = threadIdx.x + u * kNF of a tile, fetched one tile ahead
      double rx_[RPT], ry_[RPT], rz_[RPT], rf_[RPT][KS];
      auto fetch = [&](int t) {
#pragma unroll
        for (int u = 0; u < RPT; ++u) {
          const int r = t * TILE + threadIdx.x + u * kNF;
          if (r >= total) continue;
          int lo = 0, hi = ne;  // largest s with start[s] <= r
          while (hi - lo > 1) {
            const int mid = (lo + hi) >> 1;
            if (start[mid] <= r) lo = mid;
            else hi = mid;
          }
          const NearSeg sg = seg[lo];
          const int i = r - start[lo];
          const int kind = sg.kind_depth & 15;
          if (kind == 0) {
            const int p = sg.node + i;
            rx_[u] = sx[p] + (double)sg.ox;
            ry_[u] = sy[p] + (double)sg.oy;
            rz_[u] = sz[p] + (double)sg.oz;
#pragma unroll
            for (int c = 0; c < KS; ++c) rf_[u][c] = den[(long)p * KS + c];
          } else {
            const double hr = ldexp(kind == 1 ? kRad0 : kRad1, -((sg.kind_depth >> 4) + 1));
            const double* dens = (kind == 1 ? ue : de) + (long)sg.node * dim;
            rx_[u] = (double)sg.ox + hr * usurf[i * 3 + 0];
            ry_[u] = (double)sg.oy + hr * usurf[i * 3 + 1];
            rz_[u] = (double)sg.oz + hr * usurf[i * 3 + 2];
#pragma unroll
            for (int c = 0; c < KS; ++c) rf_[u][c] = dens[i * KS + c];
          }
        }
      };
      if (ntile > 0) fetch(0);
      for (int t = 0; t < ntile; ++t) {
        const int n = min(TILE, total - t * TILE);
#pragma unroll
        for (int u = 0; u < RPT; ++u) {
          const int j = threadIdx.x + u * kNF;
          if (j < n) {
            Real f[KS];
#pragma unroll
            for (int c = 0; c < KS; ++c) f[c] = (Real)rf_[u][c];
            rec_store<Real, KS, TILE>(tiles[buf], j, rx_[u], ry_[u], rz_[u], f);
          }
        }
        if (t + 1 < ntile) fetch(t + 1);
        __syncthreads();  // tiles[buf] complete; tiles[buf^1] no longer read (its readers passed this barrier)
        if (active) {
          if constexpr (kPacked) rec_sum2_x2<Ker, TILE>(tiles[buf], n, g, G, pt[0], pt[1], acc);
          else rec_sum2<Real, Ker, false, TILE>(tiles[buf], n, g, G, pt[0], pt[1], acc);
        }
        buf ^= 1;
      }
    }
    // fixed-order sum of the G partial sums of each target (in the tiles'
    // memory: every thread is done reading them past this barrier)
    __syncthreads();
    if (active)
#pragma unroll
      for (int q = 0; q < TPT; ++q)
#pragma unroll
        for (int k = 0; k < KT; ++k) red[threadIdx.x][q][k] = acc[q][k];
    __syncthreads();
    if (active && g == 0) {
#pragma unroll
      for (int q = 0; q < TPT; ++q) {
        if (ti + q * nc >= m) break;
        double sum[KT];
#pragma unroll
        for (int k = 0; k < KT; ++k) sum[k] = red[ti][q][k];
        for (int gg = 1; gg < G; ++gg)
#pragma unroll
          for (int k = 0; k < KT; ++k) sum[k] += red[gg * nc + ti][q][k];
        const long o = (long)(t0 + c0 + ti + q * nc) * KT;
#pragma unroll
        for (int k = 0; k < KT; ++k) pot[o + k] = kDbl ? pot[o + k] + sum[k] * scale : sum[k] * scale;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// Sources -> check surface of a node, FP64.  mode 0 (S2U, fmm_pts.txx:
// 2275-2637): node = sleaf[b], sources = its own points, output row b of
// `out` scaled by scale*2^-depth (level factor of the check->equivalent
// operator).  mode 1 (X, fmm_pts.txx:4444-4736): node = xtrg[b], sources =
// the X list, added to DC[node].
// ---------------------------------------------------------------------------
// mode 2: as mode 0, added to the row (the double-layer pass after the single
// layer's).
// Surface1 (mode 0 only): the check surface lies at least 1.2 half-widths
// from every point of the leaf, so FP64 needs one Newton step (mixed form).
template <int Ker, bool Surface1 = false>
__global__ void __launch_bounds__(kNT) surface_check_kernel(
    int mode, const int* __restrict__ nodes, const MKey* __restrict__ keys, const int* __restrict__ slo,
    const int* __restrict__ shi, const int* __restrict__ x_off, const int* __restrict__ x_list,
    const unsigned char* __restrict__ x_img, const double* __restrict__ sx, const double* __restrict__ sy,
    const double* __restrict__ sz,
    const double* __restrict__ den, const double* __restrict__ usurf, int ns, double rad, double scale, int deg,
    double* __restrict__ out) {
  constexpr int KT = KerDims<Ker>::KT;
  __shared__ Tile<double, KerDims<Ker>::KS> tl;
  __shared__ double red[kNT][KT];
  const int b = blockIdx.x;
  const int T = nodes[b];
  double cx, cy, cz, half;
  int dT;
  node_geom(keys[T], cx, cy, cz, half, dT);
  const double hr = half * rad;
  const int dim = ns * KT;
  double* o = mode != 1 ? out + (long)b * dim : out + (long)T * dim;
  const double oscale = mode != 1 ? scale * ldexp(1.0, -deg * dT) : scale;
  // a leaf's own sources (mode 0, 2) that fit one tile are staged once for
  // every chunk of check points; a chunk of kNT points (one group) then writes
  // its sums directly, with no block barrier
  const int lo0 = slo[T], n0 = shi[T] - lo0;
  if (mode != 1 && n0 <= kNT) {
    if (threadIdx.x < n0) {
      const int p = lo0 + threadIdx.x;
      tile_store(tl, threadIdx.x, sx[p], sy[p], sz[p]);
#pragma unroll
      for (int i = 0; i < KerDims<Ker>::KS; ++i) tl.f[i][threadIdx.x] = den[(long)p * KerDims<Ker>::KS + i];
    }
    __syncthreads();
    for (int c0 = 0; c0 < ns; c0 += kNT) {
      const Split sp(ns - c0);
      const int k = c0 + sp.ti;
      double px = 0, py = 0, pz = 0;
      if (sp.active) {
        px = hr * usurf[k * 3 + 0];
        py = hr * usurf[k * 3 + 1];
        pz = hr * usurf[k * 3 + 2];
      }
      const Pt<double> pt = make_pt<double>(px, py, pz);
      double acc[KT];
#pragma unroll
      for (int c = 0; c < KT; ++c) acc[c] = 0;
      if (sp.active) tile_sum<double, Ker, Surface1>(tl, n0, sp.g, sp.G, pt, acc);
      if (sp.G == 1) {
        if (sp.active)
#pragma unroll
          for (int c = 0; c < KT; ++c) {
            double* dst = o + (c0 + sp.ti) * KT + c;
            *dst = mode == 2 ? *dst + acc[c] * oscale : acc[c] * oscale;
          }
      } else {
        reduce_store<KT>(red, sp, acc, oscale, o + c0 * KT, mode != 0);
      }
    }
    return;
  }
  for (int c0 = 0; c0 < ns; c0 += kNT) {
    const Split sp(ns - c0);
    const int k = c0 + sp.ti;
    double px = 0, py = 0, pz = 0;
    if (sp.active) {
      px = hr * usurf[k * 3 + 0];
      py = hr * usurf[k * 3 + 1];
      pz = hr * usurf[k * 3 + 2];
    }
    const Pt<double> pt = make_pt<double>(px, py, pz);
    double acc[KT];
#pragma unroll
    for (int c = 0; c < KT; ++c) acc[c] = 0;
    if (mode != 1) {
      point_sources<double, Ker, Surface1>(tl, sx, sy, sz, den, slo[T], shi[T], 0, 0, 0, sp, pt, acc);
    } else {
      for (int q = x_off[T]; q < x_off[T + 1]; ++q) {
        const int S = x_list[q];
        double sxc, syc, szc, sh;
        int dS;
        node_geom(keys[S], sxc, syc, szc, sh, dS);
        if (x_img) image_shift(x_img[q], sxc, syc, szc);
        point_sources<double, Ker>(tl, sx, sy, sz, den, slo[S], shi[S], sxc - cx, syc - cy, szc - cz, sp, pt, acc);
      }
    }
    reduce_store<KT>(red, sp, acc, oscale, o + c0 * KT, mode != 0);
  }
}

// ---------------------------------------------------------------------------
// V-list: pruned separable DFTs over the (2m)^3 grid (FFT_UpEquiv /
// FFT_Check2Equiv, fmm_pts.txx:2689-2858) and the Hadamard products
// (VListHadamard, fmm_pts.txx:3249-3344).  Only the m^3 corner holding the
// upward equivalent surface enters the forward transform and only the m^3
// corner holding the check surface is produced by the inverse.  The grid
// size is a compile-time constant.  A block handles G grids (child x
// component) of one parent.
// ---------------------------------------------------------------------------
template <class Real, int M>
struct FftSizes {
  static constexpr int N1 = 2 * M, NH = M + 1, M3 = M * M * M, N3H = N1 * N1 * NH;
  // forward: grid g [M3] real, a1 [M*M][NH] complex, a2 [M][N1][NH] complex
  // (+4 complex of padding per grid, so that the z-lines of 4 neighbouring
  // grids fall into different banks)
  static constexpr int A2S = M * N1 * NH + 4;
  static constexpr size_t up_grid_bytes = sizeof(Real) * (M3 + 2 * (M * M * NH + A2S));
  // inverse: b1 [M][N1][NH] (+4 padding), b2 [M][M][NH] complex, o [M3] real
  static constexpr int B1S = M * N1 * NH + 4;
  static constexpr size_t dn_grid_bytes = sizeof(Real) * (2 * (B1S + M * M * NH) + M3);
  static constexpr size_t tw_bytes = sizeof(Real) * 2 * N1;
  static constexpr int threads(int G) { return ((8 * NH * G + 31) / 32) * 32; }  // one thread per line of the widest stage
};

// Each stage of the separable DFTs: one thread per input line; it loads the
// line into registers once and writes every output along that axis
// (twiddle index (k * x) mod N1 known at compile time, read as a broadcast).
// Output layout: FP64 with ke == 1 writes the spectra piece-major,
// spec[f][child][q] (16 bytes per child), so that the scalar Hadamard's
// gathers over Morton-adjacent parents coalesce; otherwise rows
// spec[q][f][child*ke+comp] (the tensor-core Hadamard reads a 64-byte FP32
// row with four lanes).
template <class Real, int M>
__global__ void __launch_bounds__(288) fft_up_kernel(int ke, int G, int ngroups, const int* __restrict__ vsrc,
                                                      const int* __restrict__ child0, const double* __restrict__ ue,
                                                      const int* __restrict__ fft_map, int ns, long n_q, int kz0,
                                                      int nkz, Cplx<Real>* __restrict__ spec) {
  using F = FftSizes<Real, M>;
  constexpr int N1 = F::N1, NH = F::NH, M3 = F::M3, N3H = F::N3H, A2S = F::A2S;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Real* twr = reinterpret_cast<Real*>(smem_raw);
  Real* twi = twr + N1;
  Real* g = twi + N1;                                          // G * M3
  Cplx<Real>* a1 = reinterpret_cast<Cplx<Real>*>(g + G * M3);  // G * M*M*NH
  Cplx<Real>* a2 = a1 + G * M * M * NH;                        // G * A2S
  const int q = blockIdx.x / ngroups;
  const int gb = (blockIdx.x % ngroups) * G;
  const int ngrid = 8 * ke;
  const int gn = min(G, ngrid - gb);
  const int P = vsrc[q];
  const int c0 = child0[P];
  const int dim = ns * ke;
  for (int j = threadIdx.x; j < N1; j += blockDim.x) {
    double sn, cs;
    sincospi(-2.0 * j / N1, &sn, &cs);
    twr[j] = (Real)cs;
    twi[j] = (Real)sn;
  }
  for (int i = threadIdx.x; i < gn * M3; i += blockDim.x) g[i] = 0;
  __syncthreads();
  for (int i = threadIdx.x; i < gn * ns; i += blockDim.x) {
    const int gi = i / ns, k = i % ns;
    const int gg = gb + gi, c = gg / ke, comp = gg % ke;
    const int idx = fft_map[k];  // x + N1*y + N1*N1*z, all < M
    const int x = idx % N1, y = (idx / N1) % N1, z = idx / (N1 * N1);
    g[gi * M3 + x + M * (y + M * z)] = (Real)ue[(long)(c0 + c) * dim + k * ke + comp];
  }
  __syncthreads();
  // x -> kx (real input): line = (gi, z, y)
  for (int r = threadIdx.x; r < gn * M * M; r += blockDim.x) {
    const Real* row = g + r * M;
    Real v[M];
#pragma unroll
    for (int x = 0; x < M; ++x) v[x] = row[x];
#pragma unroll
    for (int kx = 0; kx < NH; ++kx) {
      Real re = 0, im = 0;
#pragma unroll
      for (int x = 0; x < M; ++x) {
        const int w = (kx * x) % N1;
        re += v[x] * twr[w];
        im += v[x] * twi[w];
      }
      a1[r * NH + kx] = {re, im};
    }
  }
  __syncthreads();
  // y -> ky: line = (gi, z, kx), kx fastest
  for (int i = threadIdx.x; i < gn * M * NH; i += blockDim.x) {
    const int kx = i % NH, zg = i / NH;  // zg = gi*M + z
    const int gi = zg / M, z = zg % M;
    const Cplx<Real>* col = a1 + (zg * M) * NH + kx;
    Cplx<Real> v[M];
#pragma unroll
    for (int y = 0; y < M; ++y) v[y] = col[y * NH];
    Cplx<Real>* dst = a2 + gi * A2S + (z * N1) * NH + kx;
#pragma unroll
    for (int ky = 0; ky < N1; ++ky) {
      Real re = 0, im = 0;
#pragma unroll
      for (int y = 0; y < M; ++y) {
        const int w = (ky * y) % N1;
        re += v[y].re * twr[w] - v[y].im * twi[w];
        im += v[y].re * twi[w] + v[y].im * twr[w];
      }
      dst[ky * NH] = {re, im};
    }
  }
  __syncthreads();
  // z -> kz: line = (gi, ky, kx), gi fastest; spectrum index f = kx + NH*(ky + N1*kz);
  // only the slab kz in [kz0, kz0+nkz) is written, at f - N1*NH*kz0
  Cplx<Real>* out = spec + (long)q * (N1 * NH * nkz) * ngrid;
  for (int i = threadIdx.x; i < gn * N1 * NH; i += blockDim.x) {
    const int gi = i % gn, l = i / gn;  // l = ky*NH + kx
    const Cplx<Real>* col = a2 + gi * A2S + l;
    Cplx<Real> v[M];
#pragma unroll
    for (int z = 0; z < M; ++z) v[z] = col[z * N1 * NH];
#pragma unroll
    for (int kz = 0; kz < N1; ++kz) {
      if (kz < kz0 || kz >= kz0 + nkz) continue;
      Real re = 0, im = 0;
#pragma unroll
      for (int z = 0; z < M; ++z) {
        const int w = (kz * z) % N1;
        re += v[z].re * twr[w] - v[z].im * twi[w];
        im += v[z].re * twi[w] + v[z].im * twr[w];
      }
      const int f = l + N1 * NH * (kz - kz0);
      if (sizeof(Real) == 8 && ke == 1) spec[((long)f * 8 + gb + gi) * n_q + q] = {re, im};
      else out[(long)f * ngrid + gb + gi] = {re, im};
    }
  }
}

template <class Real, int M>
__global__ void __launch_bounds__(288) ifft_dn_kernel(int ke, int G, int ngroups, const int* __restrict__ vtrg,
                                                       const int* __restrict__ child0, const MKey* __restrict__ keys,
                                                       const Cplx<Real>* __restrict__ spec,
                                                       const int* __restrict__ ifft_map, int ns, int deg, int kz0,
                                                       int nkz, double* __restrict__ dc) {
  using F = FftSizes<Real, M>;
  constexpr int N1 = F::N1, NH = F::NH, M3 = F::M3, N3H = F::N3H;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Real* twr = reinterpret_cast<Real*>(smem_raw);
  Real* twi = twr + N1;
  constexpr int B1S = F::B1S;
  Cplx<Real>* b1 = reinterpret_cast<Cplx<Real>*>(twi + N1);  // G * B1S
  Cplx<Real>* b2 = b1 + G * B1S;                             // G * M*M*NH
  Real* o = reinterpret_cast<Real*>(b2 + G * M * M * NH);    // G * M3
  const int vt = blockIdx.x / ngroups;
  const int gb = (blockIdx.x % ngroups) * G;
  const int ngrid = 8 * ke;
  const int gn = min(G, ngrid - gb);
  const int P = vtrg[vt];
  const int c0 = child0[P];
  unsigned int X, Y, Z, dP;
  decode_key(keys[P], X, Y, Z, dP);
  const double lscale = ldexp(1.0, deg * ((int)dP + 1));  // 2^(trg_scal * level of the children)
  const int dim = ns * ke;
  for (int j = threadIdx.x; j < N1; j += blockDim.x) {
    double sn, cs;
    sincospi(2.0 * j / N1, &sn, &cs);  // inverse twiddles
    twr[j] = (Real)cs;
    twi[j] = (Real)sn;
  }
  __syncthreads();
  const Cplx<Real>* in = spec + (long)vt * (N1 * NH * nkz) * ngrid + gb;
  // kz -> z in [M, 2M): line = (gi, ky, kx) read straight from the spectrum
  // row of the parent (gi fastest: neighbouring threads read neighbouring
  // children of one frequency).  With a slab of kz the transform of the
  // slab's frequencies alone is added into dc (the transform is linear).
  for (int i = threadIdx.x; i < gn * N1 * NH; i += blockDim.x) {
    const int gi = i % gn, l = i / gn;  // l = ky*NH + kx
    Cplx<Real> v[N1];
#pragma unroll
    for (int kz = 0; kz < N1; ++kz)
      v[kz] = (kz >= kz0 && kz < kz0 + nkz) ? in[(long)(l + N1 * NH * (kz - kz0)) * ngrid + gi] : Cplx<Real>{0, 0};
#pragma unroll
    for (int zp = 0; zp < M; ++zp) {
      Real re = 0, im = 0;
#pragma unroll
      for (int kz = 0; kz < N1; ++kz) {
        const int w = (kz * (M + zp)) % N1;
        re += v[kz].re * twr[w] - v[kz].im * twi[w];
        im += v[kz].re * twi[w] + v[kz].im * twr[w];
      }
      b1[gi * B1S + zp * N1 * NH + l] = {re, im};
    }
  }
  __syncthreads();
  // ky -> y in [M, 2M): line = (gi, zp, kx), kx fastest
  for (int i = threadIdx.x; i < gn * M * NH; i += blockDim.x) {
    const int kx = i % NH, zg = i / NH;  // zg = gi*M + zp
    const Cplx<Real>* col = b1 + (zg / M) * B1S + ((zg % M) * N1) * NH + kx;
    Cplx<Real> v[N1];
#pragma unroll
    for (int ky = 0; ky < N1; ++ky) v[ky] = col[ky * NH];
#pragma unroll
    for (int yp = 0; yp < M; ++yp) {
      Real re = 0, im = 0;
#pragma unroll
      for (int ky = 0; ky < N1; ++ky) {
        const int w = (ky * (M + yp)) % N1;
        re += v[ky].re * twr[w] - v[ky].im * twi[w];
        im += v[ky].re * twi[w] + v[ky].im * twr[w];
      }
      b2[(zg * M + yp) * NH + kx] = {re, im};
    }
  }
  __syncthreads();
  // kx -> x in [M, 2M), c2r: line = (gi, zp, yp)
  for (int r = threadIdx.x; r < gn * M * M; r += blockDim.x) {
    const Cplx<Real>* row = b2 + r * NH;
    Cplx<Real> v[NH];
#pragma unroll
    for (int kx = 0; kx < NH; ++kx) v[kx] = row[kx];
#pragma unroll
    for (int xp = 0; xp < M; ++xp) {
      Real acc = 0;
#pragma unroll
      for (int kx = 0; kx < NH; ++kx) {
        const int w = (kx * (M + xp)) % N1;
        const Real t = v[kx].re * twr[w] - v[kx].im * twi[w];
        acc += (kx == 0 || 2 * kx == N1) ? t : (Real)2 * t;
      }
      o[r * M + xp] = acc;
    }
  }
  __syncthreads();
  for (int i = threadIdx.x; i < gn * ns; i += blockDim.x) {
    const int gi = i / ns, k = i % ns;
    const int gg = gb + gi, c = gg / ke, comp = gg % ke;
    const int idx = ifft_map[k];
    const int x = idx % N1 - M, y = (idx / N1) % N1 - M, z = idx / (N1 * N1) - M;
    dc[(long)(c0 + c) * dim + k * ke + comp] += (double)o[gi * M3 + x + M * (y + M * z)] * lscale;
  }
}

// 16-byte asynchronous global->shared copy; src_bytes = 0 zero-fills.
__device__ __forceinline__ void cp_async16(void* smem, const void* gmem, int src_bytes) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(src_bytes));
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_async_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}

// Hadamard products (VListHadamard, fmm_pts.txx:3249-3344) for vector
// expansions, organised as a register-tiled SIMT product per frequency f:
//   OUT[P][j1][c] += sum_{offset o, source child j2, i} M[f][o][j1][j2][i][c] * IN[Q_o(P)][f][j2][i]
// (KI equivalent-density components i, KO check-potential components c).  A
// block owns 128 target parents at one frequency and KOC output components
// (blockIdx.z picks the group); a thread owns one parent.  The offset blocks
// of frequency f sit in shared memory (chunks of OC offsets), read by every
// thread at the same address (broadcast).  The neighbour spectra of offset
// o+1 are copied asynchronously into a second shared buffer while offset o is
// computed; a thread only reads the rows it copied itself, so waiting on its
// own copy group is enough.  Missing neighbours are zero-filled and skipped.
template <class Real, int KI, int KO, int KOC, int OC>
__global__ void __launch_bounds__(128) hadamard_kernel(int n3h, long n_vtrg, long vt_stride, const int* __restrict__ vtab,
                                                       const Cplx<Real>* __restrict__ spec_in,
                                                       const Cplx<Real>* __restrict__ vop,
                                                       Cplx<Real>* __restrict__ spec_out) {
  constexpr int NGI = 8 * KI, NGO = 8 * KOC;
  constexpr int BLK = 64 * KI * KO;                               // complex entries per offset
  constexpr int ROW = NGI * sizeof(Cplx<Real>) / 16;              // 16-byte chunks per input row
  constexpr int STRIDE = NGI + 16 / (int)sizeof(Cplx<Real>);      // padded row (complex), breaks bank aliasing
  constexpr int NT = 128;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  Cplx<Real>* Ms = reinterpret_cast<Cplx<Real>*>(smem_raw);       // OC * BLK
  Cplx<Real>* xb = Ms + OC * BLK;                                 // 2 * NT * STRIDE
  const int f = blockIdx.y;
  const int c0 = blockIdx.z * KOC;
  const long p = (long)blockIdx.x * NT + threadIdx.x;
  Real ar[NGO], ai[NGO];
#pragma unroll
  for (int j = 0; j < NGO; ++j) ar[j] = ai[j] = 0;
  auto issue = [&](int o, int buf) {
    const int q = (o < 26 && p < n_vtrg) ? __ldg(vtab + (long)o * vt_stride + p) : -1;
    const Cplx<Real>* src = spec_in + ((long)(q < 0 ? 0 : q) * n3h + f) * NGI;
    Cplx<Real>* dst = xb + ((long)buf * NT + threadIdx.x) * STRIDE;
#pragma unroll
    for (int c = 0; c < ROW; ++c)
      cp_async16(reinterpret_cast<unsigned char*>(dst) + 16 * c, reinterpret_cast<const unsigned char*>(src) + 16 * c,
                 q >= 0 ? 16 : 0);
    cp_async_commit();
    return q;
  };
  int qc = issue(0, 0), qn = -1;
  for (int oc = 0; oc < 26; oc += OC) {
    const int no = min(OC, 26 - oc);
    __syncthreads();
    const Cplx<Real>* src = vop + ((long)f * 26 + oc) * BLK;
    for (int i = threadIdx.x; i < no * BLK; i += NT) Ms[i] = src[i];
    __syncthreads();
    for (int oo = 0; oo < no; ++oo) {
      const int o = oc + oo;
      qn = issue(o + 1, (o + 1) & 1);   // empty group past the last offset
      cp_async_wait<1>();               // this thread's row of offset o has landed
      const Cplx<Real>* Mo = Ms + oo * BLK;
      if (qc >= 0) {
        const Cplx<Real>* xr = xb + ((long)(o & 1) * NT + threadIdx.x) * STRIDE;
#pragma unroll
        for (int j2 = 0; j2 < 8; ++j2) {
          Cplx<Real> x[KI];
#pragma unroll
          for (int i = 0; i < KI; ++i) x[i] = xr[j2 * KI + i];
#pragma unroll
          for (int j1 = 0; j1 < 8; ++j1)
#pragma unroll
            for (int i = 0; i < KI; ++i)
#pragma unroll
              for (int c = 0; c < KOC; ++c) {
                const Cplx<Real> a = Mo[((j1 * 8 + j2) * KI + i) * KO + c0 + c];
                ar[j1 * KOC + c] += a.re * x[i].re - a.im * x[i].im;
                ai[j1 * KOC + c] += a.re * x[i].im + a.im * x[i].re;
              }
        }
      }
      qc = qn;
    }
  }
  cp_async_wait<0>();
  if (p < n_vtrg) {
    Cplx<Real>* out = spec_out + (p * n3h + f) * (8 * KO);
#pragma unroll
    for (int j1 = 0; j1 < 8; ++j1)
#pragma unroll
      for (int c = 0; c < KOC; ++c) out[j1 * KO + c0 + c] = {ar[j1 * KOC + c], ai[j1 * KOC + c]};
  }
}

// Hadamard products for scalar expansions (ke = 1), register form.  Same
// product as hadamard_kernel,
//   OUT[P][j1] += sum_{offset o, source child j2} M[f][o][j1][j2] * IN[Q_o(P)][f][j2],
// but each thread gathers the neighbour spectra of its PB target parents
// straight from global memory (L2) into registers, one offset ahead of the one
// it multiplies, so shared memory holds only the 26 operator blocks of the
// block's frequency (read as 16-byte broadcasts).  The input spectra are
// piece-major (IN[f][piece][Q]): the neighbours Q_o(P) of the Morton-ordered
// parents of a warp are mostly adjacent, so each 16-byte gather of a warp
// coalesces.  Offsets that none of the thread's parents has are skipped.
template <class Real, int PB>
__global__ void __launch_bounds__(128, 4) hadamard_rd_kernel(int n3h, long n_vtrg, long vt_stride, long n_vsrc,
                                                             const int* __restrict__ vtab,
                                                             const unsigned* __restrict__ vmask,
                                                          const Cplx<Real>* __restrict__ spec_in,
                                                          const Cplx<Real>* __restrict__ vop,
                                                          Cplx<Real>* __restrict__ spec_out) {
  constexpr int NT = 128;
  constexpr int BLK = 64;                                       // 8 x 8 complex per offset
  using V = typename Vec16<Real>::type;                         // 16 bytes
  constexpr int CPV = 16 / (int)sizeof(Cplx<Real>);             // complex values per vector (2 or 1)
  constexpr int NV = 8 / CPV;                                   // vectors per spectrum row
  __shared__ V Ms[26 * BLK / CPV];
  const int f = blockIdx.y;
  const long pbase = (long)blockIdx.x * NT * PB + threadIdx.x;
  {
    const V* src = reinterpret_cast<const V*>(vop + (long)f * 26 * BLK);
    for (int i = threadIdx.x; i < 26 * BLK / CPV; i += NT) Ms[i] = __ldg(src + i);
  }
  long prow[PB];
  bool pin[PB];
#pragma unroll
  for (int k = 0; k < PB; ++k) {
    prow[k] = pbase + (long)k * NT;
    pin[k] = prow[k] < n_vtrg;
  }
  Real ar[PB][8], ai[PB][8];
#pragma unroll
  for (int k = 0; k < PB; ++k)
#pragma unroll
    for (int j = 0; j < 8; ++j) ar[k][j] = ai[k][j] = 0;
  V xc[PB][NV], xn[PB][NV];
  unsigned mc = 0, mn = 0;  // bit k: parent k has offset o
  auto load = [&](int o, V (&x)[PB][NV], unsigned& mask) {
    mask = 0;
#pragma unroll
    for (int k = 0; k < PB; ++k) {
      const int q = pin[k] ? __ldg(vtab + (long)o * vt_stride + prow[k]) : -1;
      if (q >= 0) {
        mask |= 1u << k;
        const V* r = reinterpret_cast<const V*>(spec_in) + (long)f * NV * n_vsrc + q;
#pragma unroll
        for (int v = 0; v < NV; ++v) x[k][v] = __ldg(r + (long)v * n_vsrc);
      } else {
#pragma unroll
        for (int v = 0; v < NV; ++v) memset(&x[k][v], 0, 16);
      }
    }
  };
  auto compute = [&](int o, const V (&x)[PB][NV], unsigned mask) {
    if (!mask) return;
    const V* Mo = Ms + o * (BLK / CPV);
#pragma unroll
    for (int jv = 0; jv < NV; ++jv) {  // source children j2 = jv*CPV .. jv*CPV+CPV-1
      Real xr[PB][CPV], xi[PB][CPV];
#pragma unroll
      for (int k = 0; k < PB; ++k) {
        Real t[2 * CPV];
        memcpy(t, &x[k][jv], 16);
#pragma unroll
        for (int c = 0; c < CPV; ++c) {
          xr[k][c] = t[2 * c];
          xi[k][c] = t[2 * c + 1];
        }
      }
#pragma unroll
      for (int j1 = 0; j1 < 8; ++j1) {
        Real m[2 * CPV];
        const V mv = Mo[(j1 * 8) / CPV + jv];
        memcpy(m, &mv, 16);
#pragma unroll
        for (int c = 0; c < CPV; ++c)
#pragma unroll
          for (int k = 0; k < PB; ++k) {
            ar[k][j1] += m[2 * c] * xr[k][c] - m[2 * c + 1] * xi[k][c];
            ai[k][j1] += m[2 * c] * xi[k][c] + m[2 * c + 1] * xr[k][c];
          }
      }
    }
  };
  __syncthreads();  // Ms staged
  // the offsets occupied for any parent of the warp, in increasing order (the
  // targets are ordered by occupied-offset pattern, so the others are
  // common); two register sets in turn: the gathers of the next offset are in
  // flight while one is multiplied
  unsigned pm = 0;
#pragma unroll
  for (int k = 0; k < PB; ++k) pm |= pin[k] ? __ldg(vmask + prow[k]) : 0u;
  unsigned rem = __reduce_or_sync(0xffffffffu, pm);
  const int nlive = __popc(rem);
  auto take = [&]() {
    const int o = __ffs(rem) - 1;
    rem &= rem - 1;
    return o;
  };
  int oc = nlive > 0 ? take() : 0;
  if (nlive > 0) load(oc, xc, mc);
#pragma unroll 1
  for (int i = 0; i < nlive; i += 2) {
    const int on = i + 1 < nlive ? take() : -1;
    if (on >= 0) load(on, xn, mn);
    compute(oc, xc, mc);
    const int onn = i + 2 < nlive ? take() : -1;
    if (onn >= 0) load(onn, xc, mc);
    if (on >= 0) compute(on, xn, mn);
    oc = onn;
  }
#pragma unroll
  for (int k = 0; k < PB; ++k) {
    if (!pin[k]) continue;
    V* out = reinterpret_cast<V*>(spec_out + (prow[k] * n3h + f) * 8);
#pragma unroll
    for (int v = 0; v < NV; ++v) {
      Real t[2 * CPV];
#pragma unroll
      for (int c = 0; c < CPV; ++c) {
        t[2 * c] = ar[k][v * CPV + c];
        t[2 * c + 1] = ai[k][v * CPV + c];
      }
      V w;
      memcpy(&w, t, 16);
      out[v] = w;
    }
  }
}

// ---------------------------------------------------------------------------
// Hadamard products of the mixed form (ke = 1) on the tensor cores:
// mma.sync m16n8k8 TF32 with FP32 accumulation, each product split into
// three (a_hi b_hi + a_hi b_lo + a_lo b_hi, hi = the value rounded to TF32,
// lo = the remainder rounded to TF32), which carries the products to ~2^-22
// relative (an emulation of the whole FMM with this split changes the result
// by ~1e-8 relative).
//
// Per frequency f the product is a real GEMM over parent rows:
//   OUT[P][(j1, re|im)] += sum_o sum_(j2, re|im) IN[Q_o(P)][(j2, re|im)] * B_o[(j2, re|im)][(j1, re|im)]
// with B_o the real form of the complex 8x8 block M[f][o].  A warp owns MT
// tiles of 16 target parents.  The A fragments come straight from the input
// spectrum rows in L2: lane (g, t) loads the 16-byte piece t (children 2t and
// 2t+1, re and im) of rows g and g+8 (four lanes read one 64-byte row), which
// is exactly its fragment once the K order is chosen as k-step s, column
// c -> float 4t + 2s (+1 for c = t + 4).  The B fragments of every (f, o, lane) are precomputed on the
// host in that order, hi and lo, and staged per block in shared memory.
// ---------------------------------------------------------------------------
__device__ __forceinline__ void mma_tf32_16x8x8(float (&d)[4], const unsigned (&a)[4], unsigned b0, unsigned b1) {
  asm volatile(
      "mma.sync.aligned.m16n8k8.row.col.f32.tf32.tf32.f32 {%0,%1,%2,%3}, {%4,%5,%6,%7}, {%8,%9}, "
      "{%0,%1,%2,%3};\n"
      : "+f"(d[0]), "+f"(d[1]), "+f"(d[2]), "+f"(d[3])
      : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(b0), "r"(b1));
}

// hi = x rounded to TF32 (cvt.rna), lo = (x - hi) rounded to TF32: hi + lo
// carries x to ~2^-23 relative.  (Passing unrounded FP32 values leaves the
// conversion to the MMA's truncation, up to 2^-20 relative per product,
// which showed as ~1e-6 in the FMM result.)
__device__ __forceinline__ void tf32_split(float x, unsigned& hi, unsigned& lo) {
  unsigned h, l;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
  const float r = x - __uint_as_float(h);
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(l) : "f"(r));
  hi = h;
  lo = l;
}

constexpr int kTcWarps = 8;  // warps per block of the tensor-core Hadamard
#ifndef PVFMM_TC_MIN_BLOCKS
#define PVFMM_TC_MIN_BLOCKS 2
#endif
#ifndef PVFMM_TC_CHUNKS
#define PVFMM_TC_CHUNKS 8  // target-parent chunks per block (operator fragments staged once)
#endif

template <int MT>
__global__ void __launch_bounds__(32 * kTcWarps, PVFMM_TC_MIN_BLOCKS) hadamard_tc_kernel(int n3h, long n_vtrg, long vt_stride, long n_vsrc,
                                                                       int chunks,
                                                                       const int* __restrict__ vtab,
                                                                       const unsigned* __restrict__ vmask,
                                                                       const float4* __restrict__ spec_in,
                                                                       const float4* __restrict__ bfrag,
                                                                       float2* __restrict__ spec_out) {
  extern __shared__ float4 Bs[];  // [26 offsets][4 blocks (s, nt)][32 lanes]: (b0 hi, b1 hi, b0 lo, b1 lo)
  constexpr int NP = kTcWarps * 16 * MT;  // target parents of a chunk
  int* qs = reinterpret_cast<int*>(Bs + 26 * 4 * 32);  // [26][NP] source parent of each (offset, parent)
  unsigned* ms = reinterpret_cast<unsigned*>(qs + 26 * NP);  // [NP] occupied-offset pattern of each parent
  const int f = blockIdx.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  {
    const float4* src = bfrag + (long)f * 26 * 4 * 32;
    for (int i = threadIdx.x; i < 26 * 4 * 32; i += 32 * kTcWarps) Bs[i] = __ldg(src + i);
  }
  // the block's operator fragments stay staged over `chunks` chunks of NP
  // target parents (the condition below is uniform across the block)
  for (int c = 0; c < chunks; ++c) {
    const long pb = ((long)blockIdx.x * chunks + c) * NP;
    if (pb >= n_vtrg) break;
    if (c > 0) __syncthreads();  // every warp is done with the previous chunk's qs
    for (int i = threadIdx.x; i < 26 * NP; i += 32 * kTcWarps) {
      const int o = i / NP;
      const long p = pb + i % NP;
      qs[i] = p < n_vtrg ? __ldg(vtab + (long)o * vt_stride + p) : -1;
    }
    for (int i = threadIdx.x; i < NP; i += 32 * kTcWarps) ms[i] = pb + i < n_vtrg ? __ldg(vmask + pb + i) : 0u;
    __syncthreads();
    const int w0 = warp * 16 * MT;  // first parent of the warp within the chunk
    const long p0 = pb + w0;
    const float4* in_f = spec_in + (long)f * 4 + t;  // row q: in_f[q * n3h * 4]
    float acc[MT][2][4];
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
      for (int nt = 0; nt < 2; ++nt)
#pragma unroll
        for (int i = 0; i < 4; ++i) acc[mt][nt][i] = 0.f;
    float4 xa[MT][2], xb[MT][2], xc[MT][2];
    // offsets without a source parent for any of the warp's parents are
    // neither loaded nor multiplied (their products are zero); the targets
    // are ordered by occupied-offset pattern, so such offsets are common
    unsigned live = 0;
    for (int k = lane; k < 16 * MT; k += 32) live |= ms[w0 + k];
    live = __reduce_or_sync(0xffffffffu, live);
    auto load = [&](int o, float4 (&x)[MT][2]) {
#pragma unroll
      for (int mt = 0; mt < MT; ++mt)
#pragma unroll
        for (int h = 0; h < 2; ++h) {
          const int q = qs[o * NP + w0 + mt * 16 + g + 8 * h];
          x[mt][h] = q >= 0 ? __ldg(in_f + (long)q * n3h * 4) : make_float4(0.f, 0.f, 0.f, 0.f);
        }
    };
    auto compute = [&](int o, const float4 (&x)[MT][2]) {
      float4 bq[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) bq[i] = Bs[(o * 4 + i) * 32 + lane];  // consecutive lanes: conflict-free
#pragma unroll
      for (int mt = 0; mt < MT; ++mt) {
        unsigned ah[2][4], al[2][4];
        tf32_split(x[mt][0].x, ah[0][0], al[0][0]);
        tf32_split(x[mt][1].x, ah[0][1], al[0][1]);
        tf32_split(x[mt][0].y, ah[0][2], al[0][2]);
        tf32_split(x[mt][1].y, ah[0][3], al[0][3]);
        tf32_split(x[mt][0].z, ah[1][0], al[1][0]);
        tf32_split(x[mt][1].z, ah[1][1], al[1][1]);
        tf32_split(x[mt][0].w, ah[1][2], al[1][2]);
        tf32_split(x[mt][1].w, ah[1][3], al[1][3]);
        // this offset's products accumulate in a fresh fragment and join the
        // running sum with rounded FP32 adds: the tensor cores' own FP32
        // accumulation is not round-to-nearest and, carried over all 26
        // offsets, left a bias of ~2e-6 in the far-field potential
        float d[2][4];
#pragma unroll
        for (int nt = 0; nt < 2; ++nt)
#pragma unroll
          for (int i = 0; i < 4; ++i) d[nt][i] = 0.f;
#pragma unroll
        for (int s = 0; s < 2; ++s)
#pragma unroll
          for (int nt = 0; nt < 2; ++nt) {
            const float4 b = bq[s * 2 + nt];
            const unsigned bh0 = __float_as_uint(b.x), bh1 = __float_as_uint(b.y);
            const unsigned bl0 = __float_as_uint(b.z), bl1 = __float_as_uint(b.w);
            mma_tf32_16x8x8(d[nt], al[s], bh0, bh1);
            mma_tf32_16x8x8(d[nt], ah[s], bl0, bl1);
            mma_tf32_16x8x8(d[nt], ah[s], bh0, bh1);
          }
#pragma unroll
        for (int nt = 0; nt < 2; ++nt)
#pragma unroll
          for (int i = 0; i < 4; ++i) acc[mt][nt][i] += d[nt][i];
      }
    };
    // The warp's occupied offsets in increasing order, one set bit at a
    // time; three register sets in turn: the gathers of the next two offsets
    // are in flight while one offset is multiplied.
    unsigned rem = live;
    const int nlive = __popc(live);
    auto take = [&]() {
      const int o = __ffs(rem) - 1;
      rem &= rem - 1;
      return o;
    };
    int oa = 0, ob = 0, oc = 0;
    if (nlive > 0) {
      oa = take();
      load(oa, xa);
    }
    if (nlive > 1) {
      ob = take();
      load(ob, xb);
    }
#pragma unroll 1
    for (int i = 0; i < nlive; i += 3) {
      if (i + 2 < nlive) {
        oc = take();
        load(oc, xc);
      }
      compute(oa, xa);
      if (i + 3 < nlive) {
        oa = take();
        load(oa, xa);
      }
      if (i + 1 < nlive) compute(ob, xb);
      if (i + 4 < nlive) {
        ob = take();
        load(ob, xb);
      }
      if (i + 2 < nlive) compute(oc, xc);
    }
    // C fragment: (row g, cols 2t, 2t+1) and (row g+8, same cols); column
    // n = nt*8 + 2t (+1) is child j1 = 4nt + t, re (im).
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
      for (int h = 0; h < 2; ++h) {
        const long p = p0 + mt * 16 + g + 8 * h;
        if (p >= n_vtrg) continue;
        float2* out = spec_out + (p * n3h + f) * 8;
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) out[4 * nt + t] = make_float2(acc[mt][nt][2 * h], acc[mt][nt][2 * h + 1]);
      }
  }
}

// ---------------------------------------------------------------------------
// Hadamard products of the mixed form for 3-component expansions (Stokes
// velocity, pressure and velocity gradient, Biot-Savart) on the tensor cores,
// with the same TF32 3-term split as hadamard_tc_kernel.  Per frequency f and
// group z of KOC output components:
//   OUT[P][(j1, c, re|im)] += sum_o sum_(j2, i, re|im) IN[Q_o(P)][(j2, i, re|im)] B_o[..][(j1, c, re|im)]
// a real GEMM with K = 48 (8 children x 3 components x re|im, 6 k-steps) and
// N = 16 KOC (2 KOC n-tiles), B_o the real form of the complex block
// M[f][o][(j1, c)][(j2, i)].  A warp owns 16 target parents (rows); lane
// (g, t) loads the 16-byte pieces u = 0..2 at float 16u + 4t of the 48-float
// input rows g and g+8, which are its A fragments for k-steps 2u and 2u+1
// when the K order is chosen as k-step 2u+v, column c -> float
// 16u + 4(c % 4) + 2v + c / 4.  The B fragments of an offset (18 KB for
// KOC = 3) are too many to stage for all 26 offsets, so the block streams
// them, PVFMM_TC3_OPB offsets at a time, into a double buffer in shared
// memory (cp.async, one barrier per group; two offsets per group measured
// 3% faster than one at 2M Stokes points), shared by its 8 warps; offsets that no parent of
// the block has are skipped, those that no parent of a warp has are skipped
// by that warp.  Each pair of k-steps accumulates in a fresh fragment that
// joins the running sum with a rounded FP32 add (see hadamard_tc_kernel).
// ---------------------------------------------------------------------------
constexpr int kTc3Warps = 8;
#ifndef PVFMM_TC3_OPB
#define PVFMM_TC3_OPB 2  // offsets whose B fragments are staged per barrier
#endif
constexpr int kTc3Opb = PVFMM_TC3_OPB;

template <int KOC>
__global__ void __launch_bounds__(32 * kTc3Warps, 2)
    hadamard_tc3_kernel(int n3h, long n_vtrg, long vt_stride, int ko, const int* __restrict__ vtab,
                        const unsigned* __restrict__ vmask, const float4* __restrict__ spec_in,
                        const float4* __restrict__ bfrag, float2* __restrict__ spec_out) {
  constexpr int NNT = 2 * KOC;        // n-tiles of the group
  constexpr int NB = 6 * NNT;         // (k-step, n-tile) fragment blocks per offset
  constexpr int NP = kTc3Warps * 16;  // target parents of the block
  constexpr int OPB = kTc3Opb;
  extern __shared__ float4 Bs[];      // [2][OPB][NB][32 lanes]: (b0 hi, b1 hi, b0 lo, b1 lo)
  int* qs = reinterpret_cast<int*>(Bs + 2 * OPB * NB * 32);  // [26][NP] source parent of each (offset, parent)
  unsigned* wl = reinterpret_cast<unsigned*>(qs + 26 * NP);  // [kTc3Warps] occupied offsets of each warp
  const int f = blockIdx.y, z = blockIdx.z, ngroups = gridDim.z;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const long pb = (long)blockIdx.x * NP;
  for (int i = threadIdx.x; i < 26 * NP; i += 32 * kTc3Warps) {
    const int o = i / NP;
    const long p = pb + i % NP;
    qs[i] = p < n_vtrg ? __ldg(vtab + (long)o * vt_stride + p) : -1;
  }
  {
    const long p = pb + warp * 16 + (lane & 15);
    unsigned m = (lane < 16 && p < n_vtrg) ? __ldg(vmask + p) : 0u;
    m = __reduce_or_sync(0xffffffffu, m);
    if (lane == 0) wl[warp] = m;
  }
  __syncthreads();
  unsigned blive = 0;
#pragma unroll
  for (int w = 0; w < kTc3Warps; ++w) blive |= wl[w];
  const unsigned wlive = wl[warp];
  const float4* bsrc = bfrag + ((long)f * 26 * ngroups + z) * NB * 32;  // + o * ngroups * NB * 32
  // the next (up to) OPB block-live offsets of srem into buffer buf
  unsigned srem = blive;
  auto stage_group = [&](int buf) {
#pragma unroll
    for (int j = 0; j < OPB; ++j) {
      if (!srem) break;
      const int o = __ffs(srem) - 1;
      srem &= srem - 1;
      const float4* src = bsrc + (long)o * ngroups * NB * 32;
      float4* dst = Bs + (buf * OPB + j) * NB * 32;
      for (int i = threadIdx.x; i < NB * 32; i += 32 * kTc3Warps) cp_async16(dst + i, src + i, 16);
    }
  };
  const int w0 = warp * 16;
  auto load = [&](int o, float4 (&x)[3][2]) {
#pragma unroll
    for (int h = 0; h < 2; ++h) {
      const int q = qs[o * NP + w0 + g + 8 * h];
      const float4* row = spec_in + ((long)(q < 0 ? 0 : q) * n3h + f) * 12 + t;
#pragma unroll
      for (int u = 0; u < 3; ++u) x[u][h] = q >= 0 ? __ldg(row + 4 * u) : make_float4(0.f, 0.f, 0.f, 0.f);
    }
  };
  float acc[NNT][4];
#pragma unroll
  for (int nt = 0; nt < NNT; ++nt)
#pragma unroll
    for (int i = 0; i < 4; ++i) acc[nt][i] = 0.f;
  float4 xn[3][2];
  unsigned rem = blive;
  int oc = rem ? __ffs(rem) - 1 : 0;
  if (rem) {
    stage_group(0);
    if (wlive >> oc & 1u) load(oc, xn);
  }
  cp_async_commit();
#pragma unroll 1
  for (int k = 0; rem; ++k) {
    rem &= rem - 1;
    const int on = rem ? __ffs(rem) - 1 : -1;
    const int grp = k / OPB, slot = k % OPB;
    if (slot == 0) {
      cp_async_wait<0>();  // this thread's copies of the group's offsets have landed
      __syncthreads();     // everyone's have; every warp is done with the other buffer
      stage_group((grp + 1) & 1);
      cp_async_commit();
    }
    if (wlive >> oc & 1u) {
      unsigned ah[6][4], al[6][4];
#pragma unroll
      for (int u = 0; u < 3; ++u) {
        tf32_split(xn[u][0].x, ah[2 * u][0], al[2 * u][0]);
        tf32_split(xn[u][1].x, ah[2 * u][1], al[2 * u][1]);
        tf32_split(xn[u][0].y, ah[2 * u][2], al[2 * u][2]);
        tf32_split(xn[u][1].y, ah[2 * u][3], al[2 * u][3]);
        tf32_split(xn[u][0].z, ah[2 * u + 1][0], al[2 * u + 1][0]);
        tf32_split(xn[u][1].z, ah[2 * u + 1][1], al[2 * u + 1][1]);
        tf32_split(xn[u][0].w, ah[2 * u + 1][2], al[2 * u + 1][2]);
        tf32_split(xn[u][1].w, ah[2 * u + 1][3], al[2 * u + 1][3]);
      }
      if (on >= 0 && (wlive >> on & 1u)) load(on, xn);  // the next offset's rows, in flight meanwhile
      const float4* bq = Bs + ((grp & 1) * OPB + slot) * NB * 32 + lane;
#pragma unroll
      for (int nt = 0; nt < NNT; ++nt)
#pragma unroll
        for (int u = 0; u < 3; ++u) {
          float d[4] = {0.f, 0.f, 0.f, 0.f};
#pragma unroll
          for (int v = 0; v < 2; ++v) {
            const int sk = 2 * u + v;
            const float4 b = bq[(sk * NNT + nt) * 32];
            const unsigned bh0 = __float_as_uint(b.x), bh1 = __float_as_uint(b.y);
            const unsigned bl0 = __float_as_uint(b.z), bl1 = __float_as_uint(b.w);
            mma_tf32_16x8x8(d, al[sk], bh0, bh1);
            mma_tf32_16x8x8(d, ah[sk], bl0, bl1);
            mma_tf32_16x8x8(d, ah[sk], bh0, bh1);
          }
#pragma unroll
          for (int i = 0; i < 4; ++i) acc[nt][i] += d[i];
        }
    } else if (on >= 0 && (wlive >> on & 1u)) {
      load(on, xn);
    }
    oc = on;
  }
  cp_async_wait<0>();
  // C fragment: (row g, cols 2t, 2t+1) and (row g+8, same cols); columns
  // nt*8 + 2t (+1) are the re (im) part of output element e = 4nt + t =
  // j1 * KOC + c of the group.
#pragma unroll
  for (int h = 0; h < 2; ++h) {
    const long p = pb + w0 + g + 8 * h;
    if (p >= n_vtrg) continue;
    float2* out = spec_out + (p * n3h + f) * (8 * ko) + z * KOC;
#pragma unroll
    for (int nt = 0; nt < NNT; ++nt) {
      const int e = 4 * nt + t;
      out[(e / KOC) * ko + e % KOC] = make_float2(acc[nt][2 * h], acc[nt][2 * h + 1]);
    }
  }
}

template <int KOC>
void launch_hadamard_tc3(Context& ctx, int n3h, long f_base, int ko, const Cplx<float>* sin_, Cplx<float>* sout,
                         long p0, long np) {
  DevTree& T = ctx.tree;
  constexpr int NB = 12 * KOC, NP = kTc3Warps * 16;
  const int ngroups = ko / KOC;
  const size_t sm = (size_t)2 * kTc3Opb * NB * 32 * sizeof(float4) + (size_t)26 * NP * sizeof(int) +
                    kTc3Warps * sizeof(int);
  PVFMM_CUDA_CHECK(cudaFuncSetAttribute(hadamard_tc3_kernel<KOC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  dim3 grid(ceil_div(np, (long)NP), n3h, ngroups);
  ++ctx.n_launch;
  hadamard_tc3_kernel<KOC><<<grid, 32 * kTc3Warps, sm, ctx.stream>>>(
      n3h, np, T.n_vtrg, ko, T.vtab.get<int>() + p0, T.vmask.get<unsigned>() + p0,
      reinterpret_cast<const float4*>(sin_), ctx.dops.vop_frag.get<float4>() + f_base * 26 * ngroups * NB * 32,
      reinterpret_cast<float2*>(sout));
}

// ---------------------------------------------------------------------------
// Hadamard products of the plain form for 3-component expansions on the FP64
// tensor cores (mma.sync m8n8k4 .f64).  The same real GEMM per frequency f and
// output group z as hadamard_tc3_kernel, K = 48 in 12 k-steps of 4, N = 16 KOC
// in 2 KOC n-tiles of 8, in FP64 with no split.  A warp owns 8 target parents
// (rows); lane (g, t) holds row g, and with the K order k-step s, column
// c -> double 12c + s its A values for all 12 k-steps are the contiguous
// doubles 12t .. 12t+11 of the row (6 16-byte loads).  The B fragments of an
// offset (18 KB for KOC = 3) are streamed offset by offset into a double
// buffer in shared memory (cp.async, one barrier per offset) shared by the
// block's 8 warps; offsets no parent of the block has are skipped, those no
// parent of a warp has are skipped by that warp.
// ---------------------------------------------------------------------------
constexpr int kDmWarps = 8;

template <int KOC>
__global__ void __launch_bounds__(32 * kDmWarps, 2)
    hadamard_dmma3_kernel(int n3h, long n_vtrg, long vt_stride, int ko, const int* __restrict__ vtab,
                          const unsigned* __restrict__ vmask, const double2* __restrict__ spec_in,
                          const double* __restrict__ bfrag, double2* __restrict__ spec_out) {
  constexpr int NNT = 2 * KOC;       // n-tiles of the group
  constexpr int NB = 12 * NNT;       // (k-step, n-tile) fragment blocks per offset
  constexpr int NP = kDmWarps * 8;   // target parents of the block
  extern __shared__ double Bd[];     // [2][NB][32 lanes]
  int* qs = reinterpret_cast<int*>(Bd + 2 * NB * 32);  // [26][NP]
  unsigned* wl = reinterpret_cast<unsigned*>(qs + 26 * NP);  // [kDmWarps]
  const int f = blockIdx.y, z = blockIdx.z, ngroups = gridDim.z;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  const long pb = (long)blockIdx.x * NP;
  for (int i = threadIdx.x; i < 26 * NP; i += 32 * kDmWarps) {
    const int o = i / NP;
    const long p = pb + i % NP;
    qs[i] = p < n_vtrg ? __ldg(vtab + (long)o * vt_stride + p) : -1;
  }
  {
    const long p = pb + warp * 8 + (lane & 7);
    unsigned m = (lane < 8 && p < n_vtrg) ? __ldg(vmask + p) : 0u;
    m = __reduce_or_sync(0xffffffffu, m);
    if (lane == 0) wl[warp] = m;
  }
  __syncthreads();
  unsigned blive = 0;
#pragma unroll
  for (int w = 0; w < kDmWarps; ++w) blive |= wl[w];
  const unsigned wlive = wl[warp];
  const double* bsrc = bfrag + ((long)f * 26 * ngroups + z) * NB * 32;
  auto stage = [&](int o, int buf) {
    const double2* src = reinterpret_cast<const double2*>(bsrc + (long)o * ngroups * NB * 32);
    double2* dst = reinterpret_cast<double2*>(Bd + buf * NB * 32);
    for (int i = threadIdx.x; i < NB * 16; i += 32 * kDmWarps) cp_async16(dst + i, src + i, 16);
  };
  const int w0 = warp * 8;
  auto load = [&](int o, double2 (&x)[6]) {
    const int q = qs[o * NP + w0 + g];
    const double2* row = spec_in + ((long)(q < 0 ? 0 : q) * n3h + f) * 24 + 6 * t;
#pragma unroll
    for (int u = 0; u < 6; ++u) x[u] = q >= 0 ? __ldg(row + u) : make_double2(0.0, 0.0);
  };
  double acc[NNT][2];
#pragma unroll
  for (int nt = 0; nt < NNT; ++nt) acc[nt][0] = acc[nt][1] = 0.0;
  double2 xc[6], xn[6];
  unsigned rem = blive;
  int oc = rem ? __ffs(rem) - 1 : 0;
  if (rem) {
    stage(oc, 0);
    if (wlive >> oc & 1u) load(oc, xn);
  }
  cp_async_commit();
#pragma unroll 1
  for (int k = 0; rem; ++k) {
    rem &= rem - 1;
    const int on = rem ? __ffs(rem) - 1 : -1;
    cp_async_wait<0>();  // this thread's copies of offset oc have landed
    __syncthreads();     // everyone's have; every warp is done with the other buffer
    if (on >= 0) stage(on, (k + 1) & 1);
    cp_async_commit();
    if (wlive >> oc & 1u) {
#pragma unroll
      for (int u = 0; u < 6; ++u) xc[u] = xn[u];
      if (on >= 0 && (wlive >> on & 1u)) load(on, xn);  // the next offset's row, in flight meanwhile
      const double* bq = Bd + (k & 1) * NB * 32 + lane;
#pragma unroll
      for (int sk = 0; sk < 12; ++sk) {
        const double a = sk & 1 ? xc[sk >> 1].y : xc[sk >> 1].x;
#pragma unroll
        for (int nt = 0; nt < NNT; ++nt) dmma(acc[nt], a, bq[(sk * NNT + nt) * 32]);
      }
    } else if (on >= 0 && (wlive >> on & 1u)) {
      load(on, xn);
    }
    oc = on;
  }
  cp_async_wait<0>();
  // C fragment: (row g, cols 2t, 2t+1): the re and im part of output element
  // e = 4 nt + t = j1 * KOC + c of the group
  const long p = pb + w0 + g;
  if (p < n_vtrg) {
    double2* out = spec_out + (p * n3h + f) * (8 * ko) + z * KOC;
#pragma unroll
    for (int nt = 0; nt < NNT; ++nt) {
      const int e = 4 * nt + t;
      out[(e / KOC) * ko + e % KOC] = make_double2(acc[nt][0], acc[nt][1]);
    }
  }
}

// ---------------------------------------------------------------------------
// Hadamard products of the plain form for scalar expansions (ke = 1) on the
// FP64 tensor cores: per frequency the real GEMM OUT[P][(j1, re|im)] +=
// sum_o IN[Q_o(P)][(j2, re|im)] B_o[..][..] with K = N = 16 (4 k-steps, 2
// n-tiles of mma.sync m8n8k4 .f64).  A warp owns MT tiles of 8 target parents;
// with the K order k-step s, column t -> child 2t + s/2, re|im = s % 2, lane
// (g, t) needs children 2t and 2t+1 of row g: two 16-byte pieces of the
// piece-major input spectra (IN[f][child][Q], so the gathers of Morton-close
// parents coalesce), gathered from L2 two offsets ahead.  A block stages its
// frequency's B fragments (26 offsets, 53 KB) once and walks `chunks` chunks
// of target parents; each warp walks only the offsets occupied for one of its
// parents.
// ---------------------------------------------------------------------------
constexpr int kDm1Warps = 8;

template <int MT>
__global__ void __launch_bounds__(32 * kDm1Warps, 2)
    hadamard_dmma1_kernel(int n3h, long n_vtrg, long vt_stride, long n_vsrc, int chunks, const int* __restrict__ vtab,
                          const unsigned* __restrict__ vmask, const double2* __restrict__ spec_in,
                          const double* __restrict__ bfrag, double2* __restrict__ spec_out) {
  extern __shared__ double Bs1[];  // [26 offsets][8 blocks (s, nt)][32 lanes]
  constexpr int NP = kDm1Warps * 8 * MT;  // target parents of a chunk
  int* qs = reinterpret_cast<int*>(Bs1 + 26 * 8 * 32);  // [26][NP]
  unsigned* ms = reinterpret_cast<unsigned*>(qs + 26 * NP);  // [NP]
  const int f = blockIdx.y;
  const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
  const int g = lane >> 2, t = lane & 3;
  {
    const double2* src = reinterpret_cast<const double2*>(bfrag + (long)f * 26 * 8 * 32);
    double2* dst = reinterpret_cast<double2*>(Bs1);
    for (int i = threadIdx.x; i < 26 * 8 * 16; i += 32 * kDm1Warps) dst[i] = __ldg(src + i);
  }
  const double2* in0 = spec_in + ((long)f * 8 + 2 * t) * n_vsrc;  // child 2t; child 2t+1 at + n_vsrc
  for (int c = 0; c < chunks; ++c) {
    const long pb = ((long)blockIdx.x * chunks + c) * NP;
    if (pb >= n_vtrg) break;
    if (c > 0) __syncthreads();  // every warp is done with the previous chunk's qs
    for (int i = threadIdx.x; i < 26 * NP; i += 32 * kDm1Warps) {
      const int o = i / NP;
      const long p = pb + i % NP;
      qs[i] = p < n_vtrg ? __ldg(vtab + (long)o * vt_stride + p) : -1;
    }
    for (int i = threadIdx.x; i < NP; i += 32 * kDm1Warps) ms[i] = pb + i < n_vtrg ? __ldg(vmask + pb + i) : 0u;
    __syncthreads();
    const int w0 = warp * 8 * MT;
    double acc[MT][2][2];
#pragma unroll
    for (int mt = 0; mt < MT; ++mt)
#pragma unroll
      for (int nt = 0; nt < 2; ++nt) acc[mt][nt][0] = acc[mt][nt][1] = 0.0;
    unsigned live = 0;
    for (int k = lane; k < 8 * MT; k += 32) live |= ms[w0 + k];
    live = __reduce_or_sync(0xffffffffu, live);
    double2 xa[MT][2], xb[MT][2], xc[MT][2];
    auto load = [&](int o, double2 (&x)[MT][2]) {
#pragma unroll
      for (int mt = 0; mt < MT; ++mt) {
        const int q = qs[o * NP + w0 + mt * 8 + g];
        x[mt][0] = q >= 0 ? __ldg(in0 + q) : make_double2(0.0, 0.0);
        x[mt][1] = q >= 0 ? __ldg(in0 + n_vsrc + q) : make_double2(0.0, 0.0);
      }
    };
    auto compute = [&](int o, const double2 (&x)[MT][2]) {
      double b[4][2];
#pragma unroll
      for (int sk = 0; sk < 4; ++sk)
#pragma unroll
        for (int nt = 0; nt < 2; ++nt) b[sk][nt] = Bs1[((o * 4 + sk) * 2 + nt) * 32 + lane];
#pragma unroll
      for (int mt = 0; mt < MT; ++mt) {
        const double a[4] = {x[mt][0].x, x[mt][0].y, x[mt][1].x, x[mt][1].y};
#pragma unroll
        for (int sk = 0; sk < 4; ++sk)
#pragma unroll
          for (int nt = 0; nt < 2; ++nt) dmma(acc[mt][nt], a[sk], b[sk][nt]);
      }
    };
    unsigned rem = live;
    const int nlive = __popc(live);
    auto take = [&]() {
      const int o = __ffs(rem) - 1;
      rem &= rem - 1;
      return o;
    };
    int oa = 0, ob = 0, oc = 0;
    if (nlive > 0) {
      oa = take();
      load(oa, xa);
    }
    if (nlive > 1) {
      ob = take();
      load(ob, xb);
    }
#pragma unroll 1
    for (int i = 0; i < nlive; i += 3) {
      if (i + 2 < nlive) {
        oc = take();
        load(oc, xc);
      }
      compute(oa, xa);
      if (i + 3 < nlive) {
        oa = take();
        load(oa, xa);
      }
      if (i + 1 < nlive) compute(ob, xb);
      if (i + 4 < nlive) {
        ob = take();
        load(ob, xb);
      }
      if (i + 2 < nlive) compute(oc, xc);
    }
    // C fragment: (row g, cols 2t, 2t+1) of n-tile nt = the re and im part of
    // child j1 = 4 nt + t
#pragma unroll
    for (int mt = 0; mt < MT; ++mt) {
      const long p = pb + w0 + mt * 8 + g;
      if (p >= n_vtrg) continue;
      double2* out = spec_out + (p * n3h + f) * 8;
#pragma unroll
      for (int nt = 0; nt < 2; ++nt) out[4 * nt + t] = make_double2(acc[mt][nt][0], acc[mt][nt][1]);
    }
  }
}

void launch_hadamard_dmma1(Context& ctx, int n3h, long f_base, const Cplx<double>* sin_, Cplx<double>* sout, long p0,
                           long np) {
  DevTree& T = ctx.tree;
  constexpr int MT = 2;
  const size_t sm = (size_t)26 * 8 * 32 * sizeof(double) + (size_t)27 * kDm1Warps * 8 * MT * sizeof(int);
  PVFMM_CUDA_CHECK(
      cudaFuncSetAttribute(hadamard_dmma1_kernel<MT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  const int chunks = 8;
  dim3 grid(ceil_div(np, (long)8 * MT * kDm1Warps * chunks), n3h);
  ++ctx.n_launch;
  hadamard_dmma1_kernel<MT><<<grid, 32 * kDm1Warps, sm, ctx.stream>>>(
      n3h, np, T.n_vtrg, T.n_vsrc, chunks, T.vtab.get<int>() + p0, T.vmask.get<unsigned>() + p0,
      reinterpret_cast<const double2*>(sin_), ctx.dops.vop_frag.get<double>() + f_base * 26 * 8 * 32,
      reinterpret_cast<double2*>(sout));
}

template <int KOC>
void launch_hadamard_dmma3(Context& ctx, int n3h, long f_base, int ko, const Cplx<double>* sin_, Cplx<double>* sout,
                           long p0, long np) {
  DevTree& T = ctx.tree;
  constexpr int NB = 24 * KOC, NP = kDmWarps * 8;
  const int ngroups = ko / KOC;
  const size_t sm = (size_t)2 * NB * 32 * sizeof(double) + (size_t)26 * NP * sizeof(int) + kDmWarps * sizeof(int);
  PVFMM_CUDA_CHECK(
      cudaFuncSetAttribute(hadamard_dmma3_kernel<KOC>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  dim3 grid(ceil_div(np, (long)NP), n3h, ngroups);
  ++ctx.n_launch;
  hadamard_dmma3_kernel<KOC><<<grid, 32 * kDmWarps, sm, ctx.stream>>>(
      n3h, np, T.n_vtrg, ko, T.vtab.get<int>() + p0, T.vmask.get<unsigned>() + p0,
      reinterpret_cast<const double2*>(sin_), ctx.dops.vop_frag.get<double>() + f_base * 26 * ngroups * NB * 32,
      reinterpret_cast<double2*>(sout));
}

// Target parents [p0, p0 + np) of the V-list; sout holds their rows.
void launch_hadamard_tc(Context& ctx, int n3h, long f_base, const Cplx<float>* sin_, Cplx<float>* sout, long p0,
                        long np) {
  DevTree& T = ctx.tree;
  constexpr int MT = 2;
  const size_t sm = (size_t)26 * 4 * 32 * sizeof(float4) + (size_t)27 * kTcWarps * 16 * MT * sizeof(int);
  PVFMM_CUDA_CHECK(cudaFuncSetAttribute(hadamard_tc_kernel<MT>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  const int chunks = PVFMM_TC_CHUNKS;
  dim3 grid(ceil_div(np, (long)16 * MT * kTcWarps * chunks), n3h);
  ++ctx.n_launch;
  hadamard_tc_kernel<MT><<<grid, 32 * kTcWarps, sm, ctx.stream>>>(
      n3h, np, T.n_vtrg, T.n_vsrc, chunks, T.vtab.get<int>() + p0, T.vmask.get<unsigned>() + p0,
      reinterpret_cast<const float4*>(sin_),
      ctx.dops.vop_frag.get<float4>() + f_base * 26 * 4 * 32, reinterpret_cast<float2*>(sout));
}

template <class Real, int PB>
void launch_hadamard_rd(Context& ctx, int n3h, long f_base, const Cplx<Real>* sin_, Cplx<Real>* sout, long p0,
                        long np) {
  DevTree& T = ctx.tree;
  dim3 grid(ceil_div(np, 128 * PB), n3h);
  ++ctx.n_launch;
  hadamard_rd_kernel<Real, PB><<<grid, 128, 0, ctx.stream>>>(n3h, np, T.n_vtrg, T.n_vsrc, T.vtab.get<int>() + p0,
                                                             T.vmask.get<unsigned>() + p0, sin_,
                                                             ctx.dops.vop.get<Cplx<Real>>() + f_base * 26 * 64, sout);
}

// Target parents per thread (register tile) of the FP64 scalar Hadamard.
#ifndef PVFMM_HAD_PB_F64
#define PVFMM_HAD_PB_F64 1
#endif

template <class Real, int KI, int KO, int OC>
size_t hadamard_smem() {
  constexpr int STRIDE = 8 * KI + 16 / (int)sizeof(Cplx<Real>);
  return sizeof(Cplx<Real>) * ((size_t)OC * 64 * KI * KO + 2 * 128 * STRIDE);
}

template <class Real, int KI, int KO, int KOC, int OC>
void launch_hadamard(Context& ctx, int n3h, long f_base, const Cplx<Real>* sin_, Cplx<Real>* sout, long p0,
                     long np) {
  static_assert(KO % KOC == 0, "output components in whole groups");
  DevTree& T = ctx.tree;
  const size_t sm = hadamard_smem<Real, KI, KO, OC>();
  PVFMM_CUDA_CHECK(cudaFuncSetAttribute(hadamard_kernel<Real, KI, KO, KOC, OC>,
                                        cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm));
  dim3 grid(ceil_div(np, 128), n3h, KO / KOC);
  ++ctx.n_launch;
  hadamard_kernel<Real, KI, KO, KOC, OC><<<grid, 128, sm, ctx.stream>>>(
      n3h, np, T.n_vtrg, T.vtab.get<int>() + p0, sin_, ctx.dops.vop.get<Cplx<Real>>() + f_base * 26 * 64 * KI * KO,
      sout);
}

// ---------------------------------------------------------------------------
// Small helpers.
// ---------------------------------------------------------------------------
// Per-component scales of the C interface's rescale (at most 9 components):
// scale_x^src_scal of the densities, scale_x * scale_x^src_scal and 1 of the
// double-layer values, scale_x^trg_scal of the outputs.
struct OutScales {
  double v[9];
};

// Densities (k values per point) in sorted order, each scaled in the input
// precision as the reference scales them (pvfmm-wrapper.cpp:591-599).
template <class Tin>
__global__ void sort_densities(const Tin* __restrict__ in, const int* __restrict__ perm, long n, int k,
                               OutScales sc, double* __restrict__ out) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long p = perm[i];
  for (int j = 0; j < k; ++j) out[i * k + j] = (double)((Tin)in[p * k + j] * (Tin)sc.v[j]);
}

// Periodic lattice sum: subtracts from every target value the volume
// potential of the mean source density, taken as the sum of the root's
// upward equivalent density per component (the reference's PostProcessing,
// fmm_pts.txx:5741-5771, with laplace_vol_poten -|x|^2/6 and
// stokes_vol_poten -(|x|^2 - x_l^2)/4 of kernel.txx:1289-1295, 1456-1467) at
// the target's unit-cube position x.  kin = k1 = 1 (Laplace potential) or 3
// (Stokes velocity).  Every block forms the sums itself (ns*kin values).
__global__ void __launch_bounds__(256) periodic_mean_correction(
    long n_trg, const int* __restrict__ trg_leaf, const MKey* __restrict__ keys, const double* __restrict__ tx,
    const double* __restrict__ ty, const double* __restrict__ tz, const double* __restrict__ ue_root, int ns, int kin,
    int k1, double* __restrict__ pot) {
  __shared__ double part[256][3];
  __shared__ double avg[3];
  double a[3] = {0, 0, 0};
  for (int i = threadIdx.x; i < ns; i += blockDim.x)
    for (int k = 0; k < kin && k < 3; ++k) a[k] += ue_root[(long)i * kin + k];
  for (int k = 0; k < 3; ++k) part[threadIdx.x][k] = a[k];
  __syncthreads();
  if (threadIdx.x < 3) {
    double v = 0;
    for (int j = 0; j < (int)blockDim.x; ++j) v += part[j][threadIdx.x];
    avg[threadIdx.x] = v;
  }
  __syncthreads();
  for (long t = blockIdx.x * (long)blockDim.x + threadIdx.x; t < n_trg; t += (long)gridDim.x * blockDim.x) {
    double cx, cy, cz, half;
    int d;
    node_geom(keys[trg_leaf[t]], cx, cy, cz, half, d);
    const double x = tx[t] + cx, y = ty[t] + cy, z = tz[t] + cz;
    if (k1 == 1) {
      pot[t] += avg[0] * (x * x + y * y + z * z) / 6;
    } else {
      pot[t * 3 + 0] += avg[0] * (y * y + z * z) / 4;
      pot[t * 3 + 1] += avg[1] * (x * x + z * z) / 4;
      pot[t * 3 + 2] += avg[2] * (x * x + y * y) / 4;
    }
  }
}

template <class Tout>
__global__ void unsort_values(const double* __restrict__ pot, const int* __restrict__ perm, long n, int k1,
                              OutScales sc, Tout* __restrict__ out) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long p = perm[i];
  for (int k = 0; k < k1; ++k) out[p * k1 + k] = (Tout)((Tout)pot[i * k1 + k] * (Tout)sc.v[k]);
}

template <class Real>
void upload_vec(DevBuf& b, const std::vector<double>& v, cudaStream_t s) {
  std::vector<Real> tmp(v.begin(), v.end());
  Real* d = b.as<Real>(tmp.size());
  PVFMM_CUDA_CHECK(cudaMemcpyAsync(d, tmp.data(), tmp.size() * sizeof(Real), cudaMemcpyHostToDevice, s));
  PVFMM_CUDA_CHECK(cudaStreamSynchronize(s));
}

// Largest divisor G of ngrid with fixed + G*per_grid <= budget and at most
// 288 threads (the DFT kernels' launch bound) for threads(G) (at least 1).
template <class F>
int grids_per_block(size_t per_grid, size_t fixed, int ngrid, size_t budget) {
  int best = 1;
  for (int G = 1; G <= ngrid; ++G)
    if (ngrid % G == 0 && fixed + G * per_grid <= budget && F::threads(G) <= 288) best = G;
  return best;
}

// V-list: forward DFTs of every source parent, then the Hadamard products
// and inverse DFTs of the target parents in chunks of `chunk` parents (the
// output spectra of one chunk at a time; one chunk when device memory
// allows).  With several chunks, stage 4 ends after the first chunk's
// products and stage 5 covers the rest.
// Kernel of the mixed form's scalar Hadamard: the warp-level MMA kernel
// gathering from L2 (hadamard_tc_kernel), or with PVFMM_B200_HADAMARD=tcgen05
// the tcgen05 kernel with TMEM accumulators over tiles of Morton-consecutive
// targets (hadamard_tc.cu).
bool use_tc5(const Context&) {
  const char* e = std::getenv("PVFMM_B200_HADAMARD");
  return e && std::strcmp(e, "tcgen05") == 0;
}
// Hadamard of 3-component expansions: tensor cores (hadamard_tc3_kernel in
// the mixed form, hadamard_dmma3_kernel in the plain form), or with
// PVFMM_B200_HADAMARD3=simt the SIMT kernel (hadamard_kernel).
bool use_simt3() {
  const char* e = std::getenv("PVFMM_B200_HADAMARD3");
  return e && std::strcmp(e, "simt") == 0;
}
// Plain-form Hadamard of scalar expansions: FP64 tensor cores
// (hadamard_dmma1_kernel), or with PVFMM_B200_HADAMARD=simt the FP64 SIMT
// kernel (hadamard_rd_kernel).
bool use_simt1() {
  const char* e = std::getenv("PVFMM_B200_HADAMARD");
  return e && std::strcmp(e, "simt") == 0;
}

template <class Real, int M>
void vlist_fft_t(Context& ctx, const double* ue, double* dc, Cplx<Real>* sin_, Cplx<Real>* sout, int kin, int kout,
                 long chunk, int nslab, const std::function<void(int)>& ev) {
  DevTree& T = ctx.tree;
  auto s = ctx.stream;
  using F = FftSizes<Real, M>;
  const int ngrid_up = 8 * kin, ngrid_dn = 8 * kout;
  const int Gu = grids_per_block<F>(F::up_grid_bytes, F::tw_bytes, ngrid_up, 64 * 1024);
  const size_t sm_up = F::tw_bytes + Gu * F::up_grid_bytes;
  PVFMM_CUDA_CHECK(cudaFuncSetAttribute(fft_up_kernel<Real, M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_up));
  const int Gd = grids_per_block<F>(F::dn_grid_bytes, F::tw_bytes, ngrid_dn, 80 * 1024);
  const size_t sm_dn = F::tw_bytes + Gd * F::dn_grid_bytes;
  PVFMM_CUDA_CHECK(
      cudaFuncSetAttribute(ifft_dn_kernel<Real, M>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_dn));
  // slabs of kz (the slowest frequency index): each slab's forward DFT rows,
  // products and inverse DFT contribution in turn (nslab = 1: all at once)
  for (int sl = 0; sl < nslab; ++sl) {
    const int kz0 = F::N1 * sl / nslab, nkz = F::N1 * (sl + 1) / nslab - kz0;
    const int n3h = F::N1 * F::NH * nkz;           // the slab's frequencies
    const long f_base = (long)F::N1 * F::NH * kz0;  // its first frequency
    ++ctx.n_launch;
    fft_up_kernel<Real, M><<<T.n_vsrc * (ngrid_up / Gu), F::threads(Gu), sm_up, s>>>(
        kin, Gu, ngrid_up / Gu, T.vsrc.get<int>(), T.child0.get<int>(), ue, ctx.dops.fft_map.get<int>(), ctx.ns,
        T.n_vsrc, kz0, nkz, sin_);
    if (sl == 0) ev(4);
    for (long p0 = 0; p0 < T.n_vtrg; p0 += chunk) {
      const long np = std::min(chunk, T.n_vtrg - p0);
      if (kin == 1 && kout == 1) {
        if constexpr (sizeof(Real) == 8) {
          if (use_simt1()) launch_hadamard_rd<Real, PVFMM_HAD_PB_F64>(ctx, n3h, f_base, sin_, sout, p0, np);
          else launch_hadamard_dmma1(ctx, n3h, f_base, sin_, sout, p0, np);
        }
        else if (use_tc5(ctx)) launch_hadamard_tc5(ctx, n3h, f_base, sin_, sout, p0, np);
        else launch_hadamard_tc(ctx, n3h, f_base, sin_, sout, p0, np);
      } else if (!use_simt3()) {  // 3-component expansions: tensor cores (TF32 x3 or FP64)
        if constexpr (sizeof(Real) == 4) {
          if (kout == 1) launch_hadamard_tc3<1>(ctx, n3h, f_base, 1, sin_, sout, p0, np);
          else launch_hadamard_tc3<3>(ctx, n3h, f_base, kout, sin_, sout, p0, np);
        } else {
          if (kout == 1) launch_hadamard_dmma3<1>(ctx, n3h, f_base, 1, sin_, sout, p0, np);
          else launch_hadamard_dmma3<3>(ctx, n3h, f_base, kout, sin_, sout, p0, np);
        }
      } else if (kout == 3) {  // Stokes velocity, Biot-Savart
        launch_hadamard<Real, 3, 3, 3, 4>(ctx, n3h, f_base, sin_, sout, p0, np);
      } else if (kout == 1) {  // Stokes pressure
        launch_hadamard<Real, 3, 1, 1, 4>(ctx, n3h, f_base, sin_, sout, p0, np);
      } else {  // Stokes velocity gradient: 9 outputs in 3 groups of 3
        launch_hadamard<Real, 3, 9, 3, 2>(ctx, n3h, f_base, sin_, sout, p0, np);
      }
      if (p0 == 0 && sl == 0) ev(5);
      ++ctx.n_launch;
      ifft_dn_kernel<Real, M><<<np * (ngrid_dn / Gd), F::threads(Gd), sm_dn, s>>>(
          kout, Gd, ngrid_dn / Gd, T.vtrg.get<int>() + p0, T.child0.get<int>(), T.key.get<MKey>(), sout,
          ctx.dops.ifft_map.get<int>(), ctx.ns, ctx.ki.deg, kz0, nkz, dc);
    }
  }
}

// V-list of equivalent densities with kin components onto check potentials
// with kout components.
template <class Real>
void vlist(Context& ctx, const double* ue, double* dc, int kin, int kout, const std::function<void(int)>& ev) {
  DevTree& T = ctx.tree;
  const int m = ctx.m, n1 = 2 * m, n3h_all = 4 * m * m * (m + 1);
  // input spectra of all source parents for a slab of kz: the whole spectrum
  // (one slab) when it takes at most 45% of the free device memory (counting
  // this buffer's current allocation), else the fewest slabs that do
  const size_t in_all = (size_t)T.n_vsrc * n3h_all * 8 * kin * sizeof(Cplx<Real>);
  int nslab = 1;
  if (in_all > ctx.spec_in.cap) {
    size_t free_b = 0, total_b = 0;
    PVFMM_CUDA_CHECK(cudaMemGetInfo(&free_b, &total_b));
    const double avail = 0.45 * (double)(free_b + ctx.spec_in.cap + ctx.spec_out.cap);
    while (nslab < n1 && (double)in_all / nslab > avail) ++nslab;
  }
  // PVFMM_B200_VLIST_SLABS sets the slab count (to exercise the slab path)
  if (const char* e = std::getenv("PVFMM_B200_VLIST_SLABS")) {
    const int v = std::atoi(e);
    if (v > 0) nslab = std::min(v, n1);
  }
  const int n3h = n1 * (m + 1) * ((n1 + nslab - 1) / nslab);  // frequencies of the largest slab
  Cplx<Real>* sin_ = ctx.spec_in.as<Cplx<Real>>((size_t)T.n_vsrc * n3h * 8 * kin);
  // output spectra: all target parents at once when they fit in 90% of the
  // free device memory (counting this buffer's current allocation), else
  // chunks of that size
  const size_t row = (size_t)n3h * 8 * kout * sizeof(Cplx<Real>);
  long chunk = T.n_vtrg;
  if ((size_t)T.n_vtrg * row > ctx.spec_out.cap) {  // query the device only when the buffer must grow
    size_t free_b = 0, total_b = 0;
    PVFMM_CUDA_CHECK(cudaMemGetInfo(&free_b, &total_b));
    const double avail = 0.9 * (double)(free_b + ctx.spec_out.cap);
    if ((double)T.n_vtrg * row > avail) chunk = std::max(256L, (long)(avail / row));
  }
  // PVFMM_B200_VLIST_CHUNK caps the chunk (to exercise the chunked path)
  if (const char* e = std::getenv("PVFMM_B200_VLIST_CHUNK")) {
    const long c = std::atol(e);
    if (c > 0) chunk = std::min(chunk, c);
  }
  // the tcgen05 Hadamard walks tiles of Morton-consecutive targets, which stay
  // inside windows of 2048 positions: its chunks are whole windows
  if (sizeof(Real) == 4 && kin == 1 && kout == 1 && use_tc5(ctx) && chunk < T.n_vtrg)
    chunk = std::max(2048L, chunk / 2048 * 2048);
  Cplx<Real>* sout = ctx.spec_out.as<Cplx<Real>>((size_t)std::min(chunk, T.n_vtrg) * n3h * 8 * kout);
  switch (m) {
    case 2: vlist_fft_t<Real, 2>(ctx, ue, dc, sin_, sout, kin, kout, chunk, nslab, ev); break;
    case 4: vlist_fft_t<Real, 4>(ctx, ue, dc, sin_, sout, kin, kout, chunk, nslab, ev); break;
    case 6: vlist_fft_t<Real, 6>(ctx, ue, dc, sin_, sout, kin, kout, chunk, nslab, ev); break;
    case 8: vlist_fft_t<Real, 8>(ctx, ue, dc, sin_, sout, kin, kout, chunk, nslab, ev); break;
    case 10: vlist_fft_t<Real, 10>(ctx, ue, dc, sin_, sout, kin, kout, chunk, nslab, ev); break;
    case 12: vlist_fft_t<Real, 12>(ctx, ue, dc, sin_, sout, kin, kout, chunk, nslab, ev); break;
    case 14: vlist_fft_t<Real, 14>(ctx, ue, dc, sin_, sout, kin, kout, chunk, nslab, ev); break;
    case 16: vlist_fft_t<Real, 16>(ctx, ue, dc, sin_, sout, kin, kout, chunk, nslab, ev); break;
    default: throw std::runtime_error("unsupported multipole order");
  }
}

template <class Real, int KerS2T, int KerExp>
void evaluate_impl(Context& ctx, const void* den_in, const void* dl_in, bool den_float, void* out, bool out_float) {
  DevTree& T = ctx.tree;
  // double-layer kernels of the source -> check and source -> target
  // sub-kernels (Laplace potential: laplace_dbl_poten; Stokes velocity:
  // stokes_sym_dip; kernel.txx:1334-1340, 1470-1473)
  constexpr int KerDblExp = KerExp == kKerLaplace ? kKerLaplaceDbl : KerExp == kKerStokes ? kKerStokesDbl : -1;
  constexpr int KerDblS2T = KerS2T == kKerLaplace ? kKerLaplaceDbl : KerS2T == kKerStokes ? kKerStokesDbl : -1;
  const bool has_sl = den_in != nullptr, has_dl = dl_in != nullptr;
  if (has_dl && (KerDblExp < 0 || KerDblS2T < 0))
    throw std::runtime_error("this kernel has no double-layer kernel (dl_den must be NULL)");
  if (T.src_counted && T.layers != ((int)has_sl | (int)has_dl << 1))
    throw std::runtime_error("setup=0 requires the same densities (sl_den, dl_den) passed or NULL as at setup");
  auto s = ctx.stream;
  // expansion dims: equivalent densities din = ns*kin, check potentials
  // dout = ns*kout (kin = kout for Laplace and Stokes velocity); the
  // pseudo-inverse factors pass through r = min(din, dout) values
  const int ns = ctx.ns, kin = KerDims<KerExp>::KS, kout = KerDims<KerExp>::KT;
  const int din = ns * kin, dout = ns * kout, deg = ctx.ki.deg;
  // inner widths of the upward and downward check -> equivalent products
  // (the kept singular directions, padded to even)
  const int ru = ctx.ru, rd = ctx.rd;
  const int k0 = ctx.ki.k0, k1 = ctx.ki.k1;
  const long N = T.n_nodes;
  const MKey* keys = T.key.get<MKey>();
  // periodic boundaries: image codes of the list entries (null: free space)
  const unsigned char* pimg = ctx.periodic ? T.p_img.get<unsigned char>() : nullptr;
  const unsigned char* wimg = ctx.periodic ? T.w_img.get<unsigned char>() : nullptr;
  const unsigned char* ximg = ctx.periodic ? T.x_img.get<unsigned char>() : nullptr;
  const std::function<void(int)> ev = [&](int i) {
    if (ctx.events_ready) PVFMM_CUDA_CHECK(cudaEventRecord(ctx.ev[i], s));
  };
  ev(0);
  if (ctx.den_pending) {  // densities uploaded on the side stream during the tree build
    PVFMM_CUDA_CHECK(cudaStreamWaitEvent(s, ctx.den_ev, 0));
    ctx.den_pending = false;
  }
  // densities (sorted, scaled by scale_x^src_scal: pvfmm-wrapper.cpp:522-541, 591-595)
  double* den = ctx.den.as<double>(std::max(T.n_src, 1L) * k0);
  // double-layer values (sorted, scaled by surf_scal: scale_x * scale_x^src_scal
  // for the k0 densities, 1 for the normal; pvfmm-wrapper.cpp:528-535, 596-599)
  double* surf = has_dl ? ctx.surf.as<double>(std::max(T.n_src, 1L) * (k0 + 3)) : nullptr;
  OutScales ss, sf, ts;
  for (int j = 0; j < 9; ++j) {
    ss.v[j] = den_float ? (double)std::pow((float)T.scale_x, (float)ctx.ki.src_scal[j % 3])
                        : std::pow(T.scale_x, ctx.ki.src_scal[j % 3]);
    ts.v[j] = out_float ? (double)std::pow((float)T.scale_x, (float)ctx.ki.trg_scal[j])
                        : std::pow(T.scale_x, ctx.ki.trg_scal[j]);
  }
  for (int j = 0; j < 9; ++j)
    sf.v[j] = j >= k0 ? 1.0 : den_float ? (double)((float)T.scale_x * (float)ss.v[j]) : T.scale_x * ss.v[j];
  auto sort_vals = [&](const void* in, int k, const OutScales& sc, double* o) {
    ++ctx.n_launch;
    if (den_float)
      sort_densities<float><<<ceil_div(T.n_src, 256), 256, 0, s>>>((const float*)in, T.src_perm.get<int>(), T.n_src,
                                                                   k, sc, o);
    else
      sort_densities<double><<<ceil_div(T.n_src, 256), 256, 0, s>>>((const double*)in, T.src_perm.get<int>(),
                                                                    T.n_src, k, sc, o);
  };
  if (T.src_counted && has_sl) sort_vals(den_in, k0, ss, den);
  if (T.src_counted && has_dl) sort_vals(dl_in, k0 + 3, sf, surf);
  double* ue = ctx.ue.as<double>((size_t)N * din);
  double* dc = ctx.dc.as<double>((size_t)N * dout);
  PVFMM_CUDA_CHECK(cudaMemsetAsync(ue, 0, (size_t)N * din * sizeof(double), s));
  PVFMM_CUDA_CHECK(cudaMemsetAsync(dc, 0, (size_t)N * dout * sizeof(double), s));
  // mixed form, Stokes kernel: the FP32 stages (V-list input, W list) read
  // the upward equivalent densities projected onto the directions above the
  // FP32 cutoff (ue32 = ue U_k U_k^T); the FP64 stages keep ue.  (2M-point
  // m=10 Stokes error 3.3e-4 without, 2.8e-5 with; no change for Laplace.)
  // The leaves' rows come from the first r32 columns of the S2U
  // intermediate, the internal nodes' from ue after U2U; leaves without
  // sources keep zero rows.
  const bool proj32 = sizeof(Real) == 4 && kin == 3 && T.src_counted && N > 0 && ctx.r32 > 0;
  double* ue32 = nullptr;
  if (proj32) {
    ue32 = ctx.ue_c.as<double>((size_t)N * din);
    PVFMM_CUDA_CHECK(cudaMemsetAsync(ue32, 0, (size_t)N * din * sizeof(double), s));
  }
  const double* usurf = ctx.dops.usurf.get<double>();
  const double* sx = T.sx.get<double>();
  const double* sy = T.sy.get<double>();
  const double* sz = T.sz.get<double>();
  const int* slo = T.src_lo.get<int>();
  const int* shi = T.src_hi.get<int>();
  const double kscale_exp = ker_scale(KerExp);
  ev(1);
  // ---- S2U
  if (T.src_counted && T.n_sleaf > 0) {
    double* uc = ctx.uc_c.as<double>((size_t)T.n_sleaf * dout);
    double* t1 = ctx.tmp_c.as<double>((size_t)T.n_sleaf * ru);
    ++ctx.n_launch;
    // full FP64 rsqrt here in both forms: the check potentials feed the
    // FP64-cutoff pseudo-inverse, which amplifies their rounding into
    // near-null components of the equivalent densities; the mixed form's FP32
    // V-list does not cancel those (one Newton step here raised the 4M-point
    // potential error from 3e-7 to 2.5e-6)
    if (has_sl)
      surface_check_kernel<KerExp, false><<<T.n_sleaf, kNT, 0, s>>>(
          0, T.sleaf.get<int>(), keys, slo, shi, nullptr, nullptr, nullptr, sx, sy, sz, den, usurf, ns, kRad1, kscale_exp, deg,
          uc);
    if constexpr (KerDblExp >= 0) {
      if (has_dl) {
        ++ctx.n_launch;
        surface_check_kernel<KerDblExp, false><<<T.n_sleaf, kNT, 0, s>>>(
            has_sl ? 2 : 0, T.sleaf.get<int>(), keys, slo, shi, nullptr, nullptr, nullptr, sx, sy, sz, surf, usurf, ns, kRad1,
            ker_scale(KerDblExp), deg, uc);
      }
    }
    // equivalent densities (uc UC2UE0) UC2UE1 straight into the leaves' rows of UE
    ++ctx.n_launch;
    translate_gemm(s, T.n_sleaf, ru, dout, uc, dout, nullptr, ctx.dops.uc2ue0.get<double>(), ru, t1, ru, nullptr,
                   nullptr, false);
    if (!proj32) {
      ++ctx.n_launch;
      translate_gemm(s, T.n_sleaf, din, ru, t1, ru, nullptr, ctx.dops.uc2ue1.get<double>(), din, ue, din,
                     T.sleaf.get<int>(), nullptr, false);
    } else {
      // the first r32 directions give the leaves' projected rows, ue U_k U_k^T
      // = (t1 columns 0..r32) (UC2UE1 rows 0..r32); ue adds the other
      // directions to a copy of them (both arrays are zero outside the
      // leaves' rows here)
      const int r32 = ctx.r32;
      ++ctx.n_launch;
      translate_gemm(s, T.n_sleaf, din, r32, t1, ru, nullptr, ctx.dops.uc2ue1.get<double>(), din, ue32, din,
                     T.sleaf.get<int>(), nullptr, false);
      PVFMM_CUDA_CHECK(cudaMemcpyAsync(ue, ue32, (size_t)N * din * sizeof(double), cudaMemcpyDeviceToDevice, s));
      if (ru > r32) {
        ++ctx.n_launch;
        translate_gemm(s, T.n_sleaf, din, ru - r32, t1 + r32, ru, nullptr,
                       ctx.dops.uc2ue1.get<double>() + (size_t)r32 * din, din, ue, din, T.sleaf.get<int>(), nullptr,
                       true);
      }
    }
  }
  ev(2);
  // ---- U2U, bottom-up
  if (T.src_counted) {
    for (int d = T.depth - 1; d >= 0; --d) {
      const long ni = T.n_internal[d];
      if (ni == 0) continue;
      // the 8 children of the level's k-th internal node are the k-th block
      // of 8 rows of the next level: one row of 8*din values per parent.  The
      // long K (8 children) is split per child, so that the coarse levels
      // with few parents still fill the GPU; the 8 pieces are added in order.
      ctx.n_launch += 2;
      double* part = ctx.tmp_c.as<double>((size_t)8 * ni * din);
      translate_gemm(s, ni, din, 8 * din, ue + (size_t)T.level_off[d + 1] * din, 8 * din, nullptr,
                     ctx.dops.u2u.get<double>(), din, ue, din, T.int_idx.get<int>() + T.int_off[d], nullptr, false, 8,
                     part);
    }
  }
  // the internal nodes' projected rows: (ue U_k) U_k^T through a compact
  // n_internal x r32 intermediate
  if (proj32) {
    long nint = 0;
    for (int d = 0; d < T.depth; ++d) nint += T.n_internal[d];
    if (nint > 0) {
      const int r32 = ctx.r32;
      double* tp = ctx.tmp_c.as<double>((size_t)nint * r32);
      ctx.n_launch += 2;
      translate_gemm(s, nint, r32, din, ue, din, T.int_idx.get<int>(), ctx.dops.ue_basis.get<double>(), r32, tp, r32,
                     nullptr, nullptr, false);
      translate_gemm(s, nint, din, r32, tp, r32, nullptr, ctx.dops.uc2ue1.get<double>(), din, ue32, din,
                     T.int_idx.get<int>(), nullptr, false);
    }
  }
  if (!proj32) ue32 = ue;
  // periodic boundaries (PeriodicBC, fmm_pts.txx:2642-2676): the root's
  // downward check potential of the images beyond its 3x3x3 block
  if (ctx.periodic && T.src_counted && N > 0) {
    ++ctx.n_launch;
    translate_gemm(s, 1, dout, din, ue, din, nullptr, ctx.dops.bc.get<double>(), dout, dc, dout, nullptr, nullptr,
                   true);
  }
  ev(3);
  // ---- V-list
  if (T.src_counted && T.n_vtrg > 0 && T.n_vsrc > 0) {
    vlist<Real>(ctx, ue32, dc, kin, kout, ev);
  } else {
    ev(4);
    ev(5);
  }
  if (ctx.tc5_err) {  // the tensor-core Hadamard's error word, checked by the caller after synchronising
    PVFMM_CUDA_CHECK(cudaMemcpyAsync(ctx.tc5_err_host, ctx.tc5_err, sizeof(int), cudaMemcpyDeviceToHost, s));
    ctx.tc5_err = nullptr;
  }
  ev(6);
  // ---- X-list
  if (T.src_counted && T.n_xtrg > 0) {
    ++ctx.n_launch;
    if (has_sl)
      surface_check_kernel<KerExp><<<T.n_xtrg, kNT, 0, s>>>(1, T.xtrg.get<int>(), keys, slo, shi, T.x_off.get<int>(),
                                                             T.x_list.get<int>(), ximg, sx, sy, sz, den, usurf, ns, kRad0,
                                                             kscale_exp, deg, dc);
    if constexpr (KerDblExp >= 0) {
      if (has_dl) {
        ++ctx.n_launch;
        surface_check_kernel<KerDblExp><<<T.n_xtrg, kNT, 0, s>>>(
            1, T.xtrg.get<int>(), keys, slo, shi, T.x_off.get<int>(), T.x_list.get<int>(), ximg, sx, sy, sz, surf, usurf,
            ns, kRad0, ker_scale(KerDblExp), deg, dc);
      }
    }
  }
  ev(7);
  // ---- D2D, top-down
  for (int d = 0; d < T.depth; ++d) {
    const long ni = T.n_internal[d];
    if (ni == 0) continue;
    if (ctx.d2d_factored) {  // (parents' dc DC2DE0) over the kept directions, then DC2DE1 M_pe2c
      double* tp = ctx.tmp_c.as<double>((size_t)ni * rd);
      ctx.n_launch += 2;
      translate_gemm(s, ni, rd, dout, dc, dout, T.int_idx.get<int>() + T.int_off[d], ctx.dops.dc2de0.get<double>(),
                     rd, tp, rd, nullptr, nullptr, false);
      translate_gemm(s, ni, 8 * dout, rd, tp, rd, nullptr, ctx.dops.d2d_f2.get<double>(), 8 * dout,
                     dc + (size_t)T.level_off[d + 1] * dout, 8 * dout, nullptr, nullptr, true);
    } else {
      ++ctx.n_launch;
      translate_gemm(s, ni, 8 * dout, dout, dc, dout, T.int_idx.get<int>() + T.int_off[d],
                     ctx.dops.d2d.get<double>(), 8 * dout, dc + (size_t)T.level_off[d + 1] * dout, 8 * dout, nullptr,
                     nullptr, true);
    }
  }
  ev(8);
  // ---- D2T equivalent densities, then the fused near field
  double* pot = ctx.pot.as<double>(std::max(T.n_trg, 1L) * k1);
  if (T.n_tleaf > 0) {
    double* de = ctx.de_c.as<double>((size_t)T.n_tleaf * din);
    double* t1 = ctx.uc_c.as<double>((size_t)T.n_tleaf * rd);
    // (2^(-deg depth) DC[leaf] DC2DE0) DC2DE1, the check potentials gathered
    // from the leaves' rows of DC
    ctx.n_launch += 2;
    translate_gemm(s, T.n_tleaf, rd, dout, dc, dout, T.tleaf.get<int>(), ctx.dops.dc2de0.get<double>(), rd, t1, rd,
                   nullptr, keys, false, 1, nullptr, deg);
    translate_gemm(s, T.n_tleaf, din, rd, t1, rd, nullptr, ctx.dops.dc2de1.get<double>(), din, de, din, nullptr,
                   nullptr, false);
    ev(12);
    ++ctx.n_launch;
    near_field_kernel<Real, KerS2T><<<T.n_tleaf, kNF, 0, s>>>(
        T.tleaf.get<int>(), keys, T.trg_lo.get<int>(), T.trg_hi.get<int>(), slo, shi, T.p_off.get<int>(),
        T.p_list.get<int>(), T.w_off.get<int>(), T.w_list.get<int>(), pimg, wimg, T.tx.get<double>(),
        T.ty.get<double>(), T.tz.get<double>(), sx, sy, sz, den, ue32, T.src_counted ? de : nullptr, usurf, ns,
        ker_scale(KerS2T), has_sl ? 1 : 0, pot);
    if constexpr (KerDblS2T >= 0) {
      if (has_dl) {  // the double layer's P2P sources, added
        ++ctx.n_launch;
        near_field_kernel<Real, KerDblS2T, true><<<T.n_tleaf, kNF, 0, s>>>(
            T.tleaf.get<int>(), keys, T.trg_lo.get<int>(), T.trg_hi.get<int>(), slo, shi, T.p_off.get<int>(),
            T.p_list.get<int>(), T.w_off.get<int>(), T.w_list.get<int>(), pimg, wimg, T.tx.get<double>(),
            T.ty.get<double>(), T.tz.get<double>(), sx, sy, sz, surf, nullptr, nullptr, usurf, ns,
            ker_scale(KerDblS2T), 1, pot);
      }
    }
  } else {
    ev(12);
  }
  // periodic lattice sum of a kernel with a volume potential: the potential
  // of the mean density is taken out (PostProcessing, fmm_pts.txx:5741-5771)
  if (ctx.periodic && ctx.periodic_axes == 7 && ctx.bc_lattice && T.src_counted && T.n_trg > 0 &&
      (ctx.kernel == kLaplacePot || ctx.kernel == kStokesVel)) {
    ++ctx.n_launch;
    periodic_mean_correction<<<592, 256, 0, s>>>(T.n_trg, T.trg_leaf.get<int>(), keys, T.tx.get<double>(),
                                                 T.ty.get<double>(), T.tz.get<double>(), ue, ns, kin, k1, pot);
  }
  ev(9);
  // ---- output in input order, scaled by scale_x^trg_scal
  ++ctx.n_launch;
  if (out_float)
    unsort_values<float><<<ceil_div(T.n_trg, 256), 256, 0, s>>>(pot, T.trg_perm.get<int>(), T.n_trg, k1, ts,
                                                                (float*)out);
  else
    unsort_values<double><<<ceil_div(T.n_trg, 256), 256, 0, s>>>(pot, T.trg_perm.get<int>(), T.n_trg, k1, ts,
                                                                 (double*)out);
  ev(10);
  PVFMM_CUDA_CHECK(cudaGetLastError());
}

}  // namespace

// B fragments of hadamard_tc_kernel: for frequency f, offset o, lane (g, t)
// and block (k-step s, n-tile nt): b0 = B[(j2, re)][(j1, pout)],
// b1 = B[(j2, im)][(j1, pout)] with j2 = 2t + s, j1 = 4 nt + g/2,
// pout = g % 2, where the real form of the complex block M = M[f][o][j1][j2]
// is B[(j2,re)][(j1,re)] = Re M, B[(j2,im)][(j1,re)] = -Im M,
// B[(j2,re)][(j1,im)] = Im M, B[(j2,im)][(j1,im)] = Re M.  Each value is
// stored as [f][o][block (s, nt)][lane] float4 = (b0 hi, b1 hi, b0 lo, b1 lo),
// hi = the value rounded to TF32, lo = the remainder rounded to TF32 (round
// half away from zero, as cvt.rna), so that a warp's loads of one block are
// consecutive.
static float tf32_rna(float x) {
  unsigned u;
  std::memcpy(&u, &x, 4);
  if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & 0xffffe000u;
  float r;
  std::memcpy(&r, &u, 4);
  return r;
}

static void upload_vop_fragments(Context& ctx) {
  const HostOperators& h = ctx.hops;
  const int m = ctx.m, n3h = 4 * m * m * (m + 1);
  std::vector<float> fr((size_t)n3h * 26 * 4 * 32 * 4);
  auto split = [](float x, float& hi, float& lo) {
    hi = tf32_rna(x);
    lo = tf32_rna(x - hi);
  };
  for (int f = 0; f < n3h; ++f)
    for (int o = 0; o < 26; ++o)
      for (int lane = 0; lane < 32; ++lane) {
        const int g = lane >> 2, t = lane & 3;
        for (int s = 0; s < 2; ++s)
          for (int nt = 0; nt < 2; ++nt) {
            const int j2 = 2 * t + s, j1 = 4 * nt + (g >> 1), pout = g & 1;
            const size_t src = ((((size_t)f * 26 + o) * 8 + j1) * 8 + j2) * 2;
            const float mr = (float)h.vop[src], mi = (float)h.vop[src + 1];
            const float b0 = pout == 0 ? mr : mi;   // from (j2, re)
            const float b1 = pout == 0 ? -mi : mr;  // from (j2, im)
            float* d = &fr[((((size_t)f * 26 + o) * 4 + s * 2 + nt) * 32 + lane) * 4];
            split(b0, d[0], d[2]);
            split(b1, d[1], d[3]);
          }
      }
  float* dev = ctx.dops.vop_frag.as<float>(fr.size());
  PVFMM_CUDA_CHECK(cudaMemcpyAsync(dev, fr.data(), fr.size() * sizeof(float), cudaMemcpyHostToDevice, ctx.stream));
  PVFMM_CUDA_CHECK(cudaStreamSynchronize(ctx.stream));
}

// B fragments of hadamard_tc3_kernel: for frequency f, offset o, output group
// z (KOC components), block (k-step s = 2u + v, n-tile nt) and lane (g, t):
// b0 = B[(e_in, re)][(e_out, re|im)], b1 = B[(e_in, im)][(e_out, re|im)] with
// input element e_in = 8u + 2t + v = j2 * 3 + i, output element
// e_out = 4 nt + g / 2 = j1 * KOC + c (component z KOC + c), re|im = g % 2;
// stored as [f][o][z][block][lane] float4 = (b0 hi, b1 hi, b0 lo, b1 lo).
// Built on the device from the FP32 operator blocks vop[f][o][j1][j2][i][c].
__global__ void vop3_fragments_kernel(long n, int ko, int koc, const float2* __restrict__ vop,
                                      float4* __restrict__ frag) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const int nnt = 2 * koc, nb = 6 * nnt, ngroups = ko / koc;
  const int lane = (int)(idx % 32);
  const int blk = (int)(idx / 32 % nb);
  const long fo = idx / 32 / nb / ngroups;  // f * 26 + o
  const int z = (int)(idx / 32 / nb % ngroups);
  const int sk = blk / nnt, nt = blk % nnt;
  const int g = lane >> 2, t = lane & 3, u = sk >> 1, v = sk & 1;
  const int e_in = 8 * u + 2 * t + v, e_out = 4 * nt + g / 2, pout = g & 1;
  const int j2 = e_in / 3, i = e_in % 3, j1 = e_out / koc, c = z * koc + e_out % koc;
  const float2 mv = vop[((fo * 8 + j1) * 8 + j2) * 3 * ko + i * ko + c];
  const float b0 = pout == 0 ? mv.x : mv.y;   // from (e_in, re)
  const float b1 = pout == 0 ? -mv.y : mv.x;  // from (e_in, im)
  unsigned h0, l0, h1, l1;
  tf32_split(b0, h0, l0);
  tf32_split(b1, h1, l1);
  frag[idx] = make_float4(__uint_as_float(h0), __uint_as_float(h1), __uint_as_float(l0), __uint_as_float(l1));
}

// B fragments of hadamard_dmma3_kernel: for frequency f, offset o, output
// group z, block (k-step s, n-tile nt) and lane (g, t): b = B[k][n] with
// k = double 12t + s of the input row (element e_in = k / 2 = j2 * 3 + i,
// re|im = k % 2) and n = 8 nt + g (element e_out = n / 2 = j1 * KOC + c,
// re|im = g % 2); stored as [f][o][z][block][lane] doubles.  Built on the
// device from the FP64 operator blocks.
__global__ void vop_dmma3_fragments_kernel(long n, int ko, int koc, const double2* __restrict__ vop,
                                           double* __restrict__ frag) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const int nnt = 2 * koc, nb = 12 * nnt, ngroups = ko / koc;
  const int lane = (int)(idx % 32);
  const int blk = (int)(idx / 32 % nb);
  const int z = (int)(idx / 32 / nb % ngroups);
  const long fo = idx / 32 / nb / ngroups;  // f * 26 + o
  const int sk = blk / nnt, nt = blk % nnt;
  const int g = lane >> 2, t = lane & 3;
  const int k = 12 * t + sk, e_in = k / 2, pin = k % 2;
  const int e_out = 4 * nt + g / 2, pout = g & 1;
  const int j2 = e_in / 3, i = e_in % 3, j1 = e_out / koc, c = z * koc + e_out % koc;
  const double2 mv = vop[((fo * 8 + j1) * 8 + j2) * 3 * ko + i * ko + c];
  // real form of the complex product: [re; im] of the input times
  // [[Re, Im], [-Im, Re]] gives [re; im] of the output
  frag[idx] = pin == 0 ? (pout == 0 ? mv.x : mv.y) : (pout == 0 ? -mv.y : mv.x);
}

// B fragments of hadamard_dmma1_kernel: for frequency f, offset o, block
// (k-step s, n-tile nt) and lane (g, t): b = B[k][n] with k = (child
// 2t + s/2, re|im s % 2) and n = 8 nt + g (child 4 nt + g/2, re|im g % 2);
// stored as [f][o][s][nt][lane] doubles.
__global__ void vop_dmma1_fragments_kernel(long n, const double2* __restrict__ vop, double* __restrict__ frag) {
  const long idx = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (idx >= n) return;
  const int lane = (int)(idx % 32), nt = (int)(idx / 32 % 2), sk = (int)(idx / 64 % 4);
  const long fo = idx / 256;  // f * 26 + o
  const int g = lane >> 2, t = lane & 3;
  const int j2 = 2 * t + (sk >> 1), pin = sk & 1, j1 = 4 * nt + g / 2, pout = g & 1;
  const double2 mv = vop[(fo * 8 + j1) * 8 + j2];
  frag[idx] = pin == 0 ? (pout == 0 ? mv.x : mv.y) : (pout == 0 ? -mv.y : mv.x);
}

static void upload_vop_dmma1_fragments(Context& ctx) {
  const int m = ctx.m, n3h = 4 * m * m * (m + 1);
  const long n = (long)n3h * 26 * 8 * 32;
  double* dev = ctx.dops.vop_frag.as<double>(n);
  ++ctx.n_launch;
  vop_dmma1_fragments_kernel<<<ceil_div(n, 256L), 256, 0, ctx.stream>>>(n, ctx.dops.vop.get<double2>(), dev);
  PVFMM_CUDA_CHECK(cudaGetLastError());
  PVFMM_CUDA_CHECK(cudaStreamSynchronize(ctx.stream));
}

static void upload_vop_dmma3_fragments(Context& ctx) {
  const HostOperators& h = ctx.hops;
  const int m = ctx.m, n3h = 4 * m * m * (m + 1);
  const int ko = h.kout, koc = ko == 1 ? 1 : 3;
  const long n = (long)n3h * 26 * (ko / koc) * (24 * koc) * 32;
  double* dev = ctx.dops.vop_frag.as<double>(n);
  ++ctx.n_launch;
  vop_dmma3_fragments_kernel<<<ceil_div(n, 256L), 256, 0, ctx.stream>>>(n, ko, koc, ctx.dops.vop.get<double2>(),
                                                                         dev);
  PVFMM_CUDA_CHECK(cudaGetLastError());
  PVFMM_CUDA_CHECK(cudaStreamSynchronize(ctx.stream));
}

static void upload_vop3_fragments(Context& ctx) {
  const HostOperators& h = ctx.hops;
  const int m = ctx.m, n3h = 4 * m * m * (m + 1);
  const int ko = h.kout, koc = ko == 1 ? 1 : 3;
  const long n = (long)n3h * 26 * (ko / koc) * (12 * koc) * 32;
  float4* dev = ctx.dops.vop_frag.as<float4>(n);
  ++ctx.n_launch;
  vop3_fragments_kernel<<<ceil_div(n, 256L), 256, 0, ctx.stream>>>(n, ko, koc, ctx.dops.vop.get<float2>(), dev);
  PVFMM_CUDA_CHECK(cudaGetLastError());
  PVFMM_CUDA_CHECK(cudaStreamSynchronize(ctx.stream));
}

// Check -> equivalent factors C2E0 (rows x r) and C2E1 (r x cols) without the
// directions the cutoff dropped: a zero column of C2E0 multiplies its row of
// C2E1 by zero, so the product is unchanged when both are left out.  The
// directions listed in `first` come first (padded to an even count with a
// zero direction, *n_first), then the other kept ones; the inner width *rc is
// padded to even as well (the translation products take 16-byte rows).
void compact_factors(const std::vector<double>& c0, const std::vector<double>& c1, int rows, int r, int cols,
                     const std::vector<int>& first, std::vector<double>& o0, std::vector<double>& o1, int* rc,
                     int* n_first, std::vector<int>* order_out = nullptr) {
  std::vector<int> order(first);
  if (order.size() & 1) order.push_back(-1);
  *n_first = (int)order.size();
  std::vector<char> taken(r, 0);
  for (int j : first) taken[j] = 1;
  for (int j = 0; j < r; ++j) {
    if (taken[j]) continue;
    bool kept = false;
    for (int i = 0; i < rows && !kept; ++i) kept = c0[(size_t)i * r + j] != 0.0;
    if (kept) order.push_back(j);
  }
  if (order.size() & 1) order.push_back(-1);
  if (order.empty()) order.assign(2, -1);
  const int n = (int)order.size();
  *rc = n;
  o0.assign((size_t)rows * n, 0.0);
  o1.assign((size_t)n * cols, 0.0);
  for (int k = 0; k < n; ++k) {
    const int j = order[k];
    if (j < 0) continue;
    for (int i = 0; i < rows; ++i) o0[(size_t)i * n + k] = c0[(size_t)i * r + j];
    std::copy(c1.begin() + (size_t)j * cols, c1.begin() + (size_t)(j + 1) * cols, o1.begin() + (size_t)k * cols);
  }
  if (order_out) *order_out = std::move(order);
}

void upload_operators(Context& ctx) {
  const HostOperators& h = ctx.hops;
  auto s = ctx.stream;
  {
    const int din = h.ns * h.kin, dout = h.ns * h.kout, rk = std::min(din, dout);
    const bool proj32 = ctx.precision == 1 && ctx.ki.ke == 3;
    std::vector<double> a0, a1, b0, b1;
    int nf = 0;
    compact_factors(h.uc2ue0, h.uc2ue1, dout, rk, din, proj32 ? h.ue32_dirs : std::vector<int>(), a0, a1, &ctx.ru,
                    &ctx.r32);
    std::vector<int> dorder;
    compact_factors(h.dc2de0, h.dc2de1, dout, rk, din, std::vector<int>(), b0, b1, &ctx.rd, &nf, &dorder);
    upload_vec<double>(ctx.dops.uc2ue0, a0, s);
    upload_vec<double>(ctx.dops.uc2ue1, a1, s);
    upload_vec<double>(ctx.dops.dc2de0, b0, s);
    upload_vec<double>(ctx.dops.dc2de1, b1, s);
    // D2D = DC2DE0 (DC2DE1 M_pe2c): through the rd kept downward directions
    // the two products take 2 rd dout (1 + 8) flops per parent against
    // 16 dout^2 for the formed operator (mixed Stokes form: rd = 520 of
    // 1464); taken when that saves a quarter of the flops, since the split
    // adds a launch and an intermediate per level
    ctx.d2d_factored = !h.d2d_f2.empty() && 3L * ctx.rd < 2L * dout;
    if (ctx.d2d_factored) {
      std::vector<double> f2((size_t)ctx.rd * 8 * dout, 0.0);
      for (int k = 0; k < ctx.rd; ++k)
        if (dorder[k] >= 0)
          std::copy(h.d2d_f2.begin() + (size_t)dorder[k] * 8 * dout,
                    h.d2d_f2.begin() + (size_t)(dorder[k] + 1) * 8 * dout, f2.begin() + (size_t)k * 8 * dout);
      upload_vec<double>(ctx.dops.d2d_f2, f2, s);
    }
    if (proj32) {
      // U_k (din x r32): the transpose of the first r32 rows of the compacted
      // UC2UE1, so that ue U_k U_k^T is the projection onto those directions
      std::vector<double> ub((size_t)din * std::max(ctx.r32, 1), 0.0);
      for (int k = 0; k < ctx.r32; ++k)
        for (int a = 0; a < din; ++a) ub[(size_t)a * ctx.r32 + k] = a1[(size_t)k * din + a];
      upload_vec<double>(ctx.dops.ue_basis, ub, s);
    }
    PVFMM_CUDA_CHECK(cudaStreamSynchronize(s));  // the host vectors go out of scope
  }
  upload_vec<double>(ctx.dops.u2u, h.u2u, s);
  upload_vec<double>(ctx.dops.d2d, h.d2d, s);
  upload_vec<double>(ctx.dops.usurf, h.usurf, s);
  if (ctx.precision == 0) upload_vec<double>(ctx.dops.vop, h.vop, s);
  else upload_vec<float>(ctx.dops.vop, h.vop, s);
  if (ctx.precision == 1 && ctx.ki.ke == 1) {
    upload_vop_fragments(ctx);
    std::vector<float> lay;
    hadamard_tc5_operator_layout(h.vop, 4 * ctx.m * ctx.m * (ctx.m + 1), lay);
    float* dev = ctx.dops.vop_tc5.as<float>(lay.size());
    PVFMM_CUDA_CHECK(cudaMemcpyAsync(dev, lay.data(), lay.size() * sizeof(float), cudaMemcpyHostToDevice, s));
    PVFMM_CUDA_CHECK(cudaStreamSynchronize(s));
    if (!ctx.tc5_err_host) PVFMM_CUDA_CHECK(cudaMallocHost((void**)&ctx.tc5_err_host, sizeof(int)));
    *ctx.tc5_err_host = 0;
  }
  int* fm = ctx.dops.fft_map.as<int>(h.fft_map.size());
  int* im = ctx.dops.ifft_map.as<int>(h.ifft_map.size());
  PVFMM_CUDA_CHECK(cudaMemcpyAsync(fm, h.fft_map.data(), h.fft_map.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  PVFMM_CUDA_CHECK(cudaMemcpyAsync(im, h.ifft_map.data(), h.ifft_map.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  PVFMM_CUDA_CHECK(cudaStreamSynchronize(s));
  if (ctx.precision == 1 && ctx.ki.ke == 3) upload_vop3_fragments(ctx);  // from the uploaded FP32 vop
  if (ctx.precision == 0 && ctx.ki.ke == 3) upload_vop_dmma3_fragments(ctx);  // from the uploaded FP64 vop
  if (ctx.precision == 0 && ctx.ki.ke == 1) upload_vop_dmma1_fragments(ctx);
}

void evaluate(Context& ctx, const void* den_in, const void* dl_in, bool den_float, void* out, bool out_float) {
  const bool f32 = ctx.precision == 1;
  switch (ctx.kernel) {
    case kLaplacePot:
      if (f32) evaluate_impl<float, kKerLaplace, kKerLaplace>(ctx, den_in, dl_in, den_float, out, out_float);
      else evaluate_impl<double, kKerLaplace, kKerLaplace>(ctx, den_in, dl_in, den_float, out, out_float);
      break;
    case kLaplaceGrad:
      if (f32) evaluate_impl<float, kKerLaplaceGrad, kKerLaplace>(ctx, den_in, dl_in, den_float, out, out_float);
      else evaluate_impl<double, kKerLaplaceGrad, kKerLaplace>(ctx, den_in, dl_in, den_float, out, out_float);
      break;
    case kLaplacePotGrad:
      if (f32) evaluate_impl<float, kKerLaplacePG, kKerLaplace>(ctx, den_in, dl_in, den_float, out, out_float);
      else evaluate_impl<double, kKerLaplacePG, kKerLaplace>(ctx, den_in, dl_in, den_float, out, out_float);
      break;
    case kStokesVel:
      if (f32) evaluate_impl<float, kKerStokes, kKerStokes>(ctx, den_in, dl_in, den_float, out, out_float);
      else evaluate_impl<double, kKerStokes, kKerStokes>(ctx, den_in, dl_in, den_float, out, out_float);
      break;
    // the kernels that expand themselves (kernel.txx:894-901)
    case kStokesPress:
      if (f32) evaluate_impl<float, kKerStokesPress, kKerStokesPress>(ctx, den_in, dl_in, den_float, out, out_float);
      else evaluate_impl<double, kKerStokesPress, kKerStokesPress>(ctx, den_in, dl_in, den_float, out, out_float);
      break;
    case kStokesVelGrad:
      if (f32) evaluate_impl<float, kKerStokesGrad, kKerStokesGrad>(ctx, den_in, dl_in, den_float, out, out_float);
      else evaluate_impl<double, kKerStokesGrad, kKerStokesGrad>(ctx, den_in, dl_in, den_float, out, out_float);
      break;
    case kBiotSavart:
      if (f32) evaluate_impl<float, kKerBiotSavart, kKerBiotSavart>(ctx, den_in, dl_in, den_float, out, out_float);
      else evaluate_impl<double, kKerBiotSavart, kKerBiotSavart>(ctx, den_in, dl_in, den_float, out, out_float);
      break;
    default:
      throw std::runtime_error("unsupported kernel");
  }
}

}  // namespace pvfmm_b200
