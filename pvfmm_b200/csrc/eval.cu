// FMM evaluation on the device (FMM_Tree::RunFMM, reference
// include/fmm_tree.txx:237-738, FMM_Pts eval halves in include/fmm_pts.txx).
//
// Data layout in HBM (Real = double for the plain form, float for the mixed form):
//   points     sorted by Morton key, SoA coordinates relative to the centre of
//              the point's leaf, densities [n_src][k0], values [n_trg][k1]
//   UE, DC     per node, [n_nodes][ns*ke]: upward equivalent densities and
//              downward check potentials (the reference's upward_equiv and
//              dnward_equiv, fmm_pts.txx:1306-1480)
//   spectra    per V-list parent, [parent][freq][child*ke+comp] complex
// Stages:
//   S2U   surface evaluation to the upward check surface + 2 GEMMs (pinv factors)
//   U2U   one GEMM per level over the contiguous child blocks
//   V     pruned DFT of the 8 children, Hadamard with the 26 parent offsets,
//         pruned inverse DFT onto the children's check surfaces
//   X     surface evaluation to the downward check surface
//   D2D   one GEMM per level into the contiguous child blocks
//   D2T   2 GEMMs (pinv factors), then together with W and U one fused
//         near-field kernel per target leaf.
#include <cublas_v2.h>

#include <cmath>
#include <cstring>

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

// ---------------------------------------------------------------------------
// Source tiles in shared memory.
// ---------------------------------------------------------------------------
template <class Real, int KS>
struct Tile {
  Real x[kNT], y[kNT], z[kNT], f[KS][kNT];
};

template <class Real, int Ker>
__device__ __forceinline__ void accumulate_tile(const Tile<Real, KerDims<Ker>::KS>& tl, int n, Real px, Real py,
                                                Real pz, Acc<Real>* acc) {
  constexpr int KS = KerDims<Ker>::KS;
#pragma unroll 4
  for (int j = 0; j < n; ++j) {
    Real f[KS];
#pragma unroll
    for (int i = 0; i < KS; ++i) f[i] = tl.f[i][j];
    ker_eval<Ker, Real>(px - tl.x[j], py - tl.y[j], pz - tl.z[j], f, acc);
  }
}

// Sources on a cube surface: centre offset (ox,oy,oz), points off + hr*u_k.
template <class Real, int Ker>
__device__ void surface_sources(Tile<Real, KerDims<Ker>::KS>& tl, const Real* __restrict__ usurf, int ns, Real ox,
                                Real oy, Real oz, Real hr, const Real* __restrict__ dens, bool active, Real px, Real py,
                                Real pz, Acc<Real>* acc) {
  constexpr int KS = KerDims<Ker>::KS;
  for (int k0 = 0; k0 < ns; k0 += kNT) {
    const int n = min(kNT, ns - k0);
    __syncthreads();
    if (threadIdx.x < n) {
      const int k = k0 + threadIdx.x;
      tl.x[threadIdx.x] = ox + hr * usurf[k * 3 + 0];
      tl.y[threadIdx.x] = oy + hr * usurf[k * 3 + 1];
      tl.z[threadIdx.x] = oz + hr * usurf[k * 3 + 2];
#pragma unroll
      for (int i = 0; i < KS; ++i) tl.f[i][threadIdx.x] = dens[k * KS + i];
    }
    __syncthreads();
    if (active) accumulate_tile<Real, Ker>(tl, n, px, py, pz, acc);
  }
}

// Sources = sorted points [lo,hi) of a leaf whose centre is at offset (ox,oy,oz).
template <class Real, int Ker>
__device__ void point_sources(Tile<Real, KerDims<Ker>::KS>& tl, const Real* __restrict__ sx, const Real* __restrict__ sy,
                              const Real* __restrict__ sz, const Real* __restrict__ den, int lo, int hi, Real ox, Real oy,
                              Real oz, bool active, Real px, Real py, Real pz, Acc<Real>* acc) {
  constexpr int KS = KerDims<Ker>::KS;
  for (int p0 = lo; p0 < hi; p0 += kNT) {
    const int n = min(kNT, hi - p0);
    __syncthreads();
    if (threadIdx.x < n) {
      const int p = p0 + threadIdx.x;
      tl.x[threadIdx.x] = sx[p] + ox;
      tl.y[threadIdx.x] = sy[p] + oy;
      tl.z[threadIdx.x] = sz[p] + oz;
#pragma unroll
      for (int i = 0; i < KS; ++i) tl.f[i][threadIdx.x] = den[(long)p * KS + i];
    }
    __syncthreads();
    if (active) accumulate_tile<Real, Ker>(tl, n, px, py, pz, acc);
  }
}

// ---------------------------------------------------------------------------
// Near field of one target leaf: D2T (own downward equivalent surface), W
// (upward equivalent surfaces) and U (points), fused (fmm_pts.txx:4246-4426,
// 4746-5022, 5032-5418).  One block per target leaf.
// ---------------------------------------------------------------------------
template <class Real, int Ker>
__global__ void __launch_bounds__(kNT) near_field_kernel(
    const int* __restrict__ tleaf, const MKey* __restrict__ keys, const int* __restrict__ tlo, const int* __restrict__ thi,
    const int* __restrict__ slo, const int* __restrict__ shi, const int* __restrict__ p_off, const int* __restrict__ p_list,
    const int* __restrict__ w_off, const int* __restrict__ w_list, const Real* __restrict__ tx, const Real* __restrict__ ty,
    const Real* __restrict__ tz, const Real* __restrict__ sx, const Real* __restrict__ sy, const Real* __restrict__ sz,
    const Real* __restrict__ den, const Real* __restrict__ ue, const Real* __restrict__ de, const Real* __restrict__ usurf,
    int ns, Real scale, Real* __restrict__ pot) {
  constexpr int KS = KerDims<Ker>::KS, KT = KerDims<Ker>::KT;
  __shared__ Tile<Real, KS> tl;
  const int b = blockIdx.x;
  const int T = tleaf[b];
  double cx, cy, cz, half;
  int dT;
  node_geom(keys[T], cx, cy, cz, half, dT);
  const int t0 = tlo[T], nt = thi[T] - t0;
  const int dim = ns * KS;
  for (int c0 = 0; c0 < nt; c0 += kNT) {
    const int t = c0 + threadIdx.x;
    const bool active = t < nt;
    Real px = 0, py = 0, pz = 0;
    if (active) {
      px = tx[t0 + t];
      py = ty[t0 + t];
      pz = tz[t0 + t];
    }
    Acc<Real> acc[KT];
#pragma unroll
    for (int k = 0; k < KT; ++k) acc[k].init();
    // D2T: downward equivalent surface of T (radius RAD1)
    if (de) surface_sources<Real, Ker>(tl, usurf, ns, 0, 0, 0, (Real)(half * kRad1), de + (long)b * dim, active, px, py, pz, acc);
    // W: upward equivalent surfaces (radius RAD0) of the W-list nodes
    for (int w = w_off[T]; w < w_off[T + 1]; ++w) {
      const int S = w_list[w];
      double sxc, syc, szc, sh;
      int dS;
      node_geom(keys[S], sxc, syc, szc, sh, dS);
      surface_sources<Real, Ker>(tl, usurf, ns, (Real)(sxc - cx), (Real)(syc - cy), (Real)(szc - cz), (Real)(sh * kRad0),
                                 ue + (long)S * dim, active, px, py, pz, acc);
    }
    // U: point-to-point from the P2P list
    for (int q = p_off[T]; q < p_off[T + 1]; ++q) {
      const int S = p_list[q];
      double sxc, syc, szc, sh;
      int dS;
      node_geom(keys[S], sxc, syc, szc, sh, dS);
      point_sources<Real, Ker>(tl, sx, sy, sz, den, slo[S], shi[S], (Real)(sxc - cx), (Real)(syc - cy), (Real)(szc - cz),
                               active, px, py, pz, acc);
    }
    if (active)
#pragma unroll
      for (int k = 0; k < KT; ++k) pot[(long)(t0 + t) * KT + k] = acc[k].get() * scale;
  }
}

// ---------------------------------------------------------------------------
// Sources -> check surface of a node.  mode 0 (S2U, fmm_pts.txx:2275-2637):
// node = sleaf[b], sources = its own points, output row b of `out` scaled by
// scale*2^-depth (the level factor of the check->equivalent operator).
// mode 1 (X, fmm_pts.txx:4444-4736): node = xtrg[b], sources = the X list,
// added to DC[node].
// ---------------------------------------------------------------------------
template <class Real, int Ker>
__global__ void __launch_bounds__(kNT) surface_check_kernel(
    int mode, const int* __restrict__ nodes, const MKey* __restrict__ keys, const int* __restrict__ slo,
    const int* __restrict__ shi, const int* __restrict__ x_off, const int* __restrict__ x_list, const Real* __restrict__ sx,
    const Real* __restrict__ sy, const Real* __restrict__ sz, const Real* __restrict__ den, const Real* __restrict__ usurf,
    int ns, Real rad, Real scale, Real* __restrict__ out) {
  constexpr int KS = KerDims<Ker>::KS, KT = KerDims<Ker>::KT;
  __shared__ Tile<Real, KS> tl;
  const int b = blockIdx.x;
  const int T = nodes[b];
  double cx, cy, cz, half;
  int dT;
  node_geom(keys[T], cx, cy, cz, half, dT);
  const Real hr = (Real)(half * rad);
  const int dim = ns * KT;
  Real* o = mode == 0 ? out + (long)b * dim : out + (long)T * dim;
  const Real oscale = mode == 0 ? (Real)((double)scale * ldexp(1.0, -dT)) : scale;
  for (int c0 = 0; c0 < ns; c0 += kNT) {
    const int k = c0 + threadIdx.x;
    const bool active = k < ns;
    Real px = 0, py = 0, pz = 0;
    if (active) {
      px = hr * usurf[k * 3 + 0];
      py = hr * usurf[k * 3 + 1];
      pz = hr * usurf[k * 3 + 2];
    }
    Acc<Real> acc[KT];
#pragma unroll
    for (int c = 0; c < KT; ++c) acc[c].init();
    if (mode == 0) {
      point_sources<Real, Ker>(tl, sx, sy, sz, den, slo[T], shi[T], 0, 0, 0, active, px, py, pz, acc);
    } else {
      for (int q = x_off[T]; q < x_off[T + 1]; ++q) {
        const int S = x_list[q];
        double sxc, syc, szc, sh;
        int dS;
        node_geom(keys[S], sxc, syc, szc, sh, dS);
        point_sources<Real, Ker>(tl, sx, sy, sz, den, slo[S], shi[S], (Real)(sxc - cx), (Real)(syc - cy),
                                 (Real)(szc - cz), active, px, py, pz, acc);
      }
    }
    if (active) {
      if (mode == 0) {
#pragma unroll
        for (int c = 0; c < KT; ++c) o[k * KT + c] = acc[c].get() * oscale;
      } else {
#pragma unroll
        for (int c = 0; c < KT; ++c) o[k * KT + c] += acc[c].get() * oscale;
      }
    }
  }
}

// ---------------------------------------------------------------------------
// V-list: pruned separable DFTs over the (2m)^3 grid (FFT_UpEquiv /
// FFT_Check2Equiv, fmm_pts.txx:2689-2858) and the Hadamard products
// (VListHadamard, fmm_pts.txx:3249-3344).  Only the m^3 corner that holds
// the upward equivalent surface is transformed forward, and only the m^3
// corner that holds the check surface is produced by the inverse.
// ---------------------------------------------------------------------------
struct FftDims {
  int m, n1, nh, n3h, ns, ke, G;
};

template <class Real>
__global__ void fft_up_kernel(FftDims fd, const int* __restrict__ vsrc, const int* __restrict__ child0,
                              const Real* __restrict__ ue, const int* __restrict__ fft_map, Cplx<Real>* __restrict__ spec) {
  extern __shared__ unsigned char smem_raw[];
  Real* sm = reinterpret_cast<Real*>(smem_raw);
  const int m = fd.m, n1 = fd.n1, nh = fd.nh, ns = fd.ns, ke = fd.ke, G = fd.G;
  const int m3 = m * m * m;
  const int ngrid = 8 * ke;
  Real* twr = sm;
  Real* twi = twr + n1;
  Real* g = twi + n1;                          // G * m3
  Cplx<Real>* a1 = reinterpret_cast<Cplx<Real>*>(g + G * m3);  // G * m*m*nh
  Cplx<Real>* a2 = a1 + G * m * m * nh;        // G * m*n1*nh
  const int q = blockIdx.x;
  const int P = vsrc[q];
  const int c0 = child0[P];
  const int dim = ns * ke;
  for (int j = threadIdx.x; j < n1; j += blockDim.x) {
    double s, c;
    sincospi(-2.0 * j / n1, &s, &c);
    twr[j] = (Real)c;
    twi[j] = (Real)s;
  }
  Cplx<Real>* out = spec + (long)q * fd.n3h * ngrid;
  for (int gb = 0; gb < ngrid; gb += G) {
    const int gn = min(G, ngrid - gb);
    __syncthreads();
    for (int i = threadIdx.x; i < gn * m3; i += blockDim.x) g[i] = 0;
    __syncthreads();
    for (int i = threadIdx.x; i < gn * ns; i += blockDim.x) {
      const int gi = i / ns, k = i % ns;
      const int gg = gb + gi, c = gg / ke, comp = gg % ke;
      const int idx = fft_map[k];  // x + n1*y + n1*n1*z, all < m
      const int x = idx % n1, y = (idx / n1) % n1, z = idx / (n1 * n1);
      g[gi * m3 + x + m * (y + m * z)] = ue[(long)(c0 + c) * dim + k * ke + comp];
    }
    __syncthreads();
    // x -> kx (real input)
    for (int i = threadIdx.x; i < gn * m * m * nh; i += blockDim.x) {
      const int kx = i % nh, y = (i / nh) % m, z = (i / (nh * m)) % m, gi = i / (nh * m * m);
      const Real* row = g + gi * m3 + m * (y + m * z);
      Real re = 0, im = 0;
      for (int x = 0; x < m; ++x) {
        const int w = (kx * x) % n1;
        re += row[x] * twr[w];
        im += row[x] * twi[w];
      }
      a1[i] = {re, im};
    }
    __syncthreads();
    // y -> ky
    for (int i = threadIdx.x; i < gn * m * n1 * nh; i += blockDim.x) {
      const int kx = i % nh, ky = (i / nh) % n1, z = (i / (nh * n1)) % m, gi = i / (nh * n1 * m);
      const Cplx<Real>* col = a1 + ((gi * m + z) * m) * nh + kx;
      Real re = 0, im = 0;
      for (int y = 0; y < m; ++y) {
        const int w = (ky * y) % n1;
        const Cplx<Real> v = col[y * nh];
        re += v.re * twr[w] - v.im * twi[w];
        im += v.re * twi[w] + v.im * twr[w];
      }
      a2[i] = {re, im};
    }
    __syncthreads();
    // z -> kz, written as spec[q][f][grid]
    for (int i = threadIdx.x; i < gn * fd.n3h; i += blockDim.x) {
      const int gi = i % gn, f = i / gn;
      const int kx = f % nh, ky = (f / nh) % n1, kz = f / (nh * n1);
      const Cplx<Real>* col = a2 + ((gi * m) * n1 + ky) * nh + kx;
      Real re = 0, im = 0;
      for (int z = 0; z < m; ++z) {
        const int w = (kz * z) % n1;
        const Cplx<Real> v = col[z * n1 * nh];
        re += v.re * twr[w] - v.im * twi[w];
        im += v.re * twi[w] + v.im * twr[w];
      }
      out[(long)f * ngrid + gb + gi] = {re, im};
    }
  }
}

// One thread per (target parent, frequency); the 26 parent offsets are walked
// in the same order by every thread, so the operator loads are uniform.
template <class Real, int KE>
__global__ void __launch_bounds__(128) hadamard_kernel(int n3h, long n_vtrg, const int* __restrict__ vtab,
                                                       const Cplx<Real>* __restrict__ spec_in,
                                                       const Cplx<Real>* __restrict__ vop,
                                                       Cplx<Real>* __restrict__ spec_out) {
  constexpr int NG = 8 * KE;
  const long vt = blockIdx.x * (long)blockDim.x + threadIdx.x;
  const int f = blockIdx.y;
  if (vt >= n_vtrg) return;
  Real ar[NG], ai[NG];
#pragma unroll
  for (int j = 0; j < NG; ++j) ar[j] = ai[j] = 0;
  for (int o = 0; o < 26; ++o) {
    const int q = vtab[vt * 26 + o];
    if (q < 0) continue;
    const Cplx<Real>* in = spec_in + ((long)q * n3h + f) * NG;
    const Cplx<Real>* M = vop + ((long)f * 26 + o) * 64 * KE * KE;
#pragma unroll
    for (int j2 = 0; j2 < 8; ++j2) {
      Cplx<Real> x[KE];
#pragma unroll
      for (int i = 0; i < KE; ++i) x[i] = in[j2 * KE + i];
#pragma unroll
      for (int j1 = 0; j1 < 8; ++j1)
#pragma unroll
        for (int i = 0; i < KE; ++i)
#pragma unroll
          for (int k = 0; k < KE; ++k) {
            const Cplx<Real> a = M[((j1 * 8 + j2) * KE + i) * KE + k];
            ar[j1 * KE + k] += a.re * x[i].re - a.im * x[i].im;
            ai[j1 * KE + k] += a.re * x[i].im + a.im * x[i].re;
          }
    }
  }
  Cplx<Real>* out = spec_out + ((long)vt * n3h + f) * NG;
#pragma unroll
  for (int j = 0; j < NG; ++j) out[j] = {ar[j], ai[j]};
}

template <class Real>
__global__ void ifft_dn_kernel(FftDims fd, const int* __restrict__ vtrg, const int* __restrict__ child0,
                               const MKey* __restrict__ keys, const Cplx<Real>* __restrict__ spec,
                               const int* __restrict__ ifft_map, Real* __restrict__ dc) {
  extern __shared__ unsigned char smem_raw[];
  Real* sm = reinterpret_cast<Real*>(smem_raw);
  const int m = fd.m, n1 = fd.n1, nh = fd.nh, ns = fd.ns, ke = fd.ke, G = fd.G, n3h = fd.n3h;
  const int m3 = m * m * m;
  const int ngrid = 8 * ke;
  Real* twr = sm;
  Real* twi = twr + n1;
  Cplx<Real>* S = reinterpret_cast<Cplx<Real>*>(twi + n1);  // G * n3h
  Cplx<Real>* b1 = S + G * n3h;                             // G * m*n1*nh
  Cplx<Real>* b2 = b1 + G * m * n1 * nh;                    // G * m*m*nh
  Real* o = reinterpret_cast<Real*>(b2 + G * m * m * nh);   // G * m3
  const int vt = blockIdx.x;
  const int P = vtrg[vt];
  const int c0 = child0[P];
  unsigned int X, Y, Z, dP;
  decode_key(keys[P], X, Y, Z, dP);
  const Real lscale = (Real)ldexp(1.0, (int)dP + 1);  // trg_scal * level of the children
  const int dim = ns * ke;
  for (int j = threadIdx.x; j < n1; j += blockDim.x) {
    double s, c;
    sincospi(2.0 * j / n1, &s, &c);  // inverse twiddles
    twr[j] = (Real)c;
    twi[j] = (Real)s;
  }
  const Cplx<Real>* in = spec + (long)vt * n3h * ngrid;
  for (int gb = 0; gb < ngrid; gb += G) {
    const int gn = min(G, ngrid - gb);
    __syncthreads();
    for (int i = threadIdx.x; i < gn * n3h; i += blockDim.x) {
      const int gi = i % gn, f = i / gn;
      S[gi * n3h + f] = in[(long)f * ngrid + gb + gi];
    }
    __syncthreads();
    // kz -> z in [m, 2m)
    for (int i = threadIdx.x; i < gn * m * n1 * nh; i += blockDim.x) {
      const int kx = i % nh, ky = (i / nh) % n1, zp = (i / (nh * n1)) % m, gi = i / (nh * n1 * m);
      const int z = m + zp;
      const Cplx<Real>* col = S + gi * n3h + ky * nh + kx;
      Real re = 0, im = 0;
      for (int kz = 0; kz < n1; ++kz) {
        const int w = (kz * z) % n1;
        const Cplx<Real> v = col[kz * n1 * nh];
        re += v.re * twr[w] - v.im * twi[w];
        im += v.re * twi[w] + v.im * twr[w];
      }
      b1[i] = {re, im};
    }
    __syncthreads();
    // ky -> y in [m, 2m)
    for (int i = threadIdx.x; i < gn * m * m * nh; i += blockDim.x) {
      const int kx = i % nh, yp = (i / nh) % m, zp = (i / (nh * m)) % m, gi = i / (nh * m * m);
      const int y = m + yp;
      const Cplx<Real>* col = b1 + ((gi * m + zp) * n1) * nh + kx;
      Real re = 0, im = 0;
      for (int ky = 0; ky < n1; ++ky) {
        const int w = (ky * y) % n1;
        const Cplx<Real> v = col[ky * nh];
        re += v.re * twr[w] - v.im * twi[w];
        im += v.re * twi[w] + v.im * twr[w];
      }
      b2[i] = {re, im};
    }
    __syncthreads();
    // kx -> x in [m, 2m), real output (Hermitian weights, c2r)
    for (int i = threadIdx.x; i < gn * m3; i += blockDim.x) {
      const int xp = i % m, yp = (i / m) % m, zp = (i / (m * m)) % m, gi = i / m3;
      const int x = m + xp;
      const Cplx<Real>* row = b2 + ((gi * m + zp) * m + yp) * nh;
      Real acc = 0;
      for (int kx = 0; kx < nh; ++kx) {
        const int w = (kx * x) % n1;
        const Cplx<Real> v = row[kx];
        const Real t = v.re * twr[w] - v.im * twi[w];
        acc += (kx == 0 || 2 * kx == n1) ? t : (Real)2 * t;
      }
      o[i] = acc;
    }
    __syncthreads();
    for (int i = threadIdx.x; i < gn * ns; i += blockDim.x) {
      const int gi = i / ns, k = i % ns;
      const int gg = gb + gi, c = gg / ke, comp = gg % ke;
      const int idx = ifft_map[k];
      const int x = idx % n1 - m, y = (idx / n1) % n1 - m, z = idx / (n1 * n1) - m;
      dc[(long)(c0 + c) * dim + k * ke + comp] += o[gi * m3 + x + m * (y + m * z)] * lscale;
    }
  }
}

// ---------------------------------------------------------------------------
// Small helpers.
// ---------------------------------------------------------------------------
template <class Real>
__global__ void scatter_rows(const Real* __restrict__ src, const int* __restrict__ rows, long n, int dim,
                             Real* __restrict__ dst) {
  const long i = blockIdx.x;
  if (i >= n) return;
  const long r = rows[i];
  for (int j = threadIdx.x; j < dim; j += blockDim.x) dst[r * dim + j] = src[i * dim + j];
}

// dst[i] = src[rows[i]] * 2^(-depth(rows[i])) if scale_level else src[rows[i]].
template <class Real>
__global__ void gather_rows(const Real* __restrict__ src, const int* __restrict__ rows, long n, int dim,
                            const MKey* __restrict__ keys, int scale_level, Real* __restrict__ dst) {
  const long i = blockIdx.x;
  if (i >= n) return;
  const long r = rows[i];
  Real s = 1;
  if (scale_level) s = (Real)ldexp(1.0, -(int)(keys[r].lo & 31u));
  for (int j = threadIdx.x; j < dim; j += blockDim.x) dst[i * dim + j] = src[r * dim + j] * s;
}

template <class Tin, class Real>
__global__ void sort_densities(const Tin* __restrict__ in, const int* __restrict__ perm, long n, int k0,
                               double s0, double s1, double s2, Real* __restrict__ out) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long p = perm[i];
  const double sc[3] = {s0, s1, s2};
  for (int j = 0; j < k0; ++j) out[i * k0 + j] = (Real)((Tin)in[p * k0 + j] * (Tin)sc[j]);
}

template <class Real, class Tout>
__global__ void unsort_values(const Real* __restrict__ pot, const int* __restrict__ perm, long n, int k1, double s0,
                              double s1, double s2, double s3, Tout* __restrict__ out) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long p = perm[i];
  const double sc[4] = {s0, s1, s2, s3};
  for (int k = 0; k < k1; ++k) out[p * k1 + k] = (Tout)((Tout)pot[i * k1 + k] * (Tout)sc[k]);
}

template <class Real>
struct Blas;
template <>
struct Blas<double> {
  static void gemm(cublasHandle_t h, int M, int N, int K, const double* A, int lda, const double* B, int ldb, double* C,
                   int ldc, double beta) {
    const double one = 1.0;
    // Row-major C(MxN) = A(MxK) B(KxN)  <=>  column-major C^T = B^T A^T.
    if (cublasDgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, N, M, K, &one, B, ldb, A, lda, &beta, C, ldc) != CUBLAS_STATUS_SUCCESS)
      throw std::runtime_error("cublasDgemm failed");
  }
};
template <>
struct Blas<float> {
  static void gemm(cublasHandle_t h, int M, int N, int K, const float* A, int lda, const float* B, int ldb, float* C,
                   int ldc, float beta) {
    const float one = 1.0f;
    if (cublasSgemm(h, CUBLAS_OP_N, CUBLAS_OP_N, N, M, K, &one, B, ldb, A, lda, &beta, C, ldc) != CUBLAS_STATUS_SUCCESS)
      throw std::runtime_error("cublasSgemm failed");
  }
};

template <class Real>
void upload_vec(DevBuf& b, const std::vector<double>& v, cudaStream_t s) {
  std::vector<Real> tmp(v.begin(), v.end());
  Real* d = b.as<Real>(tmp.size());
  PVFMM_CUDA_CHECK(cudaMemcpyAsync(d, tmp.data(), tmp.size() * sizeof(Real), cudaMemcpyHostToDevice, s));
  PVFMM_CUDA_CHECK(cudaStreamSynchronize(s));
}

int fft_batch(size_t per_grid_bytes, size_t fixed_bytes, int ngrid) {
  const size_t budget = 200 * 1024;
  int G = (int)((budget - fixed_bytes) / per_grid_bytes);
  return std::max(1, std::min(G, ngrid));
}

template <class Real, int KerS2T, int KerExp>
void evaluate_impl(Context& ctx, const void* den_in, bool den_float, void* out, bool out_float) {
  DevTree& T = ctx.tree;
  auto s = ctx.stream;
  const int ns = ctx.ns, ke = ctx.ki.ke, dim = ns * ke;
  const int k0 = ctx.ki.k0, k1 = ctx.ki.k1;
  const long N = T.n_nodes;
  const MKey* keys = T.key.get<MKey>();
  auto ev = [&](int i) {
    if (ctx.events_ready) PVFMM_CUDA_CHECK(cudaEventRecord(ctx.ev[i], s));
  };
  ev(0);
  // densities (sorted, scaled by scale_x^src_scal: pvfmm-wrapper.cpp:522-541, 591-595)
  Real* den = ctx.den.as<Real>(std::max(T.n_src, 1L) * k0);
  double ss[3], ts[4];
  for (int j = 0; j < 3; ++j) ss[j] = den_float ? (double)std::pow((float)T.scale_x, (float)ctx.ki.src_scal[j])
                                                : std::pow(T.scale_x, ctx.ki.src_scal[j]);
  for (int j = 0; j < 4; ++j) ts[j] = out_float ? (double)std::pow((float)T.scale_x, (float)ctx.ki.trg_scal[j])
                                                : std::pow(T.scale_x, ctx.ki.trg_scal[j]);
  if (T.src_counted) {
    if (den_float)
      sort_densities<float, Real><<<ceil_div(T.n_src, 256), 256, 0, s>>>((const float*)den_in, T.src_perm.get<int>(),
                                                                          T.n_src, k0, ss[0], ss[1], ss[2], den);
    else
      sort_densities<double, Real><<<ceil_div(T.n_src, 256), 256, 0, s>>>((const double*)den_in, T.src_perm.get<int>(),
                                                                           T.n_src, k0, ss[0], ss[1], ss[2], den);
  }
  Real* ue = ctx.ue.as<Real>((size_t)N * dim);
  Real* dc = ctx.dc.as<Real>((size_t)N * dim);
  PVFMM_CUDA_CHECK(cudaMemsetAsync(ue, 0, (size_t)N * dim * sizeof(Real), s));
  PVFMM_CUDA_CHECK(cudaMemsetAsync(dc, 0, (size_t)N * dim * sizeof(Real), s));
  const Real* usurf = ctx.dops.usurf.get<Real>();
  const Real* sx = T.sx.get<Real>();
  const Real* sy = T.sy.get<Real>();
  const Real* sz = T.sz.get<Real>();
  const int* slo = T.src_lo.get<int>();
  const int* shi = T.src_hi.get<int>();
  if (cublasSetStream(ctx.cublas, s) != CUBLAS_STATUS_SUCCESS) throw std::runtime_error("cublasSetStream failed");
  const Real kscale_exp = (Real)ker_scale(KerExp);
  ev(1);
  // ---- S2U
  if (T.src_counted && T.n_sleaf > 0) {
    Real* uc = ctx.uc_c.as<Real>((size_t)T.n_sleaf * dim);
    Real* t1 = ctx.tmp_c.as<Real>((size_t)T.n_sleaf * dim);
    surface_check_kernel<Real, KerExp><<<T.n_sleaf, kNT, 0, s>>>(0, T.sleaf.get<int>(), keys, slo, shi, nullptr, nullptr,
                                                                  sx, sy, sz, den, usurf, ns, (Real)kRad1, kscale_exp, uc);
    Blas<Real>::gemm(ctx.cublas, (int)T.n_sleaf, dim, dim, uc, dim, ctx.dops.uc2ue0.get<Real>(), dim, t1, dim, 0);
    Blas<Real>::gemm(ctx.cublas, (int)T.n_sleaf, dim, dim, t1, dim, ctx.dops.uc2ue1.get<Real>(), dim, uc, dim, 0);
    scatter_rows<Real><<<T.n_sleaf, 128, 0, s>>>(uc, T.sleaf.get<int>(), T.n_sleaf, dim, ue);
  }
  ev(2);
  // ---- U2U, bottom-up
  if (T.src_counted) {
    for (int d = T.depth - 1; d >= 0; --d) {
      const long ni = T.n_internal[d];
      if (ni == 0) continue;
      Real* c = ctx.tmp_c.as<Real>((size_t)ni * dim);
      Blas<Real>::gemm(ctx.cublas, (int)ni, dim, 8 * dim, ue + (size_t)T.level_off[d + 1] * dim, 8 * dim,
                       ctx.dops.u2u.get<Real>(), dim, c, dim, 0);
      scatter_rows<Real><<<ni, 128, 0, s>>>(c, T.int_idx.get<int>() + T.int_off[d], ni, dim, ue);
    }
  }
  ev(3);
  // ---- V-list
  const int m = ctx.m, n1 = 2 * m, nh = m + 1, n3h = n1 * n1 * nh;
  const int ngrid = 8 * ke;
  const bool vlist = T.src_counted && T.n_vtrg > 0 && T.n_vsrc > 0;
  if (vlist) {
    Cplx<Real>* sin_ = ctx.spec_in.as<Cplx<Real>>((size_t)T.n_vsrc * n3h * ngrid);
    Cplx<Real>* sout = ctx.spec_out.as<Cplx<Real>>((size_t)T.n_vtrg * n3h * ngrid);
    FftDims fd{m, n1, nh, n3h, ns, ke, 1};
    const size_t per_up = sizeof(Real) * (m * m * m + 2 * m * m * nh + 2 * m * n1 * nh);
    fd.G = fft_batch(per_up, sizeof(Real) * 2 * n1, ngrid);
    const size_t sm_up = sizeof(Real) * 2 * n1 + per_up * fd.G;
    PVFMM_CUDA_CHECK(cudaFuncSetAttribute(fft_up_kernel<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_up));
    fft_up_kernel<Real><<<T.n_vsrc, 256, sm_up, s>>>(fd, T.vsrc.get<int>(), T.child0.get<int>(), ue,
                                                     ctx.dops.fft_map.get<int>(), sin_);
    ev(4);
    dim3 grid(ceil_div(T.n_vtrg, 128), n3h);
    hadamard_kernel<Real, (KerExp == kKerStokes ? 3 : 1)><<<grid, 128, 0, s>>>(
        n3h, T.n_vtrg, T.vtab.get<int>(), sin_, ctx.dops.vop.get<Cplx<Real>>(), sout);
    ev(5);
    FftDims fi = fd;
    const size_t per_dn = sizeof(Real) * (2 * n3h + 2 * m * n1 * nh + 2 * m * m * nh + m * m * m);
    fi.G = fft_batch(per_dn, sizeof(Real) * 2 * n1, ngrid);
    const size_t sm_dn = sizeof(Real) * 2 * n1 + per_dn * fi.G;
    PVFMM_CUDA_CHECK(cudaFuncSetAttribute(ifft_dn_kernel<Real>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)sm_dn));
    ifft_dn_kernel<Real><<<T.n_vtrg, 256, sm_dn, s>>>(fi, T.vtrg.get<int>(), T.child0.get<int>(), keys, sout,
                                                      ctx.dops.ifft_map.get<int>(), dc);
  } else {
    ev(4);
    ev(5);
  }
  ev(6);
  // ---- X-list
  if (T.src_counted && T.n_xtrg > 0)
    surface_check_kernel<Real, KerExp><<<T.n_xtrg, kNT, 0, s>>>(1, T.xtrg.get<int>(), keys, slo, shi, T.x_off.get<int>(),
                                                                 T.x_list.get<int>(), sx, sy, sz, den, usurf, ns,
                                                                 (Real)kRad0, kscale_exp, dc);
  ev(7);
  // ---- D2D, top-down
  for (int d = 0; d < T.depth; ++d) {
    const long ni = T.n_internal[d];
    if (ni == 0) continue;
    Real* g = ctx.tmp_c.as<Real>((size_t)ni * dim);
    gather_rows<Real><<<ni, 128, 0, s>>>(dc, T.int_idx.get<int>() + T.int_off[d], ni, dim, keys, 0, g);
    Blas<Real>::gemm(ctx.cublas, (int)ni, 8 * dim, dim, g, dim, ctx.dops.d2d.get<Real>(), 8 * dim,
                     dc + (size_t)T.level_off[d + 1] * dim, 8 * dim, 1);
  }
  ev(8);
  // ---- D2T equivalent densities
  Real* de = nullptr;
  if (T.n_tleaf > 0) {
    Real* g = ctx.tmp_c.as<Real>((size_t)T.n_tleaf * dim);
    de = ctx.de_c.as<Real>((size_t)T.n_tleaf * dim);
    Real* t1 = ctx.uc_c.as<Real>((size_t)T.n_tleaf * dim);
    gather_rows<Real><<<T.n_tleaf, 128, 0, s>>>(dc, T.tleaf.get<int>(), T.n_tleaf, dim, keys, 1, g);
    Blas<Real>::gemm(ctx.cublas, (int)T.n_tleaf, dim, dim, g, dim, ctx.dops.dc2de0.get<Real>(), dim, t1, dim, 0);
    Blas<Real>::gemm(ctx.cublas, (int)T.n_tleaf, dim, dim, t1, dim, ctx.dops.dc2de1.get<Real>(), dim, de, dim, 0);
    // ---- fused near field: D2T + W + U
    Real* pot = ctx.pot.as<Real>(std::max(T.n_trg, 1L) * k1);
    near_field_kernel<Real, KerS2T><<<T.n_tleaf, kNT, 0, s>>>(
        T.tleaf.get<int>(), keys, T.trg_lo.get<int>(), T.trg_hi.get<int>(), slo, shi, T.p_off.get<int>(),
        T.p_list.get<int>(), T.w_off.get<int>(), T.w_list.get<int>(), T.tx.get<Real>(), T.ty.get<Real>(),
        T.tz.get<Real>(), sx, sy, sz, den, ue, T.src_counted ? de : nullptr, usurf, ns, (Real)ker_scale(KerS2T), pot);
  }
  ev(9);
  // ---- output in input order, scaled by scale_x^trg_scal
  {
    const Real* pot = ctx.pot.get<Real>();
    if (out_float)
      unsort_values<Real, float><<<ceil_div(T.n_trg, 256), 256, 0, s>>>(pot, T.trg_perm.get<int>(), T.n_trg, k1, ts[0],
                                                                         ts[1], ts[2], ts[3], (float*)out);
    else
      unsort_values<Real, double><<<ceil_div(T.n_trg, 256), 256, 0, s>>>(pot, T.trg_perm.get<int>(), T.n_trg, k1,
                                                                          ts[0], ts[1], ts[2], ts[3], (double*)out);
  }
  ev(10);
  PVFMM_CUDA_CHECK(cudaGetLastError());
}

}  // namespace

void upload_operators(Context& ctx) {
  const HostOperators& h = ctx.hops;
  auto s = ctx.stream;
  if (ctx.precision == 0) {
    upload_vec<double>(ctx.dops.uc2ue0, h.uc2ue0, s);
    upload_vec<double>(ctx.dops.uc2ue1, h.uc2ue1, s);
    upload_vec<double>(ctx.dops.dc2de0, h.dc2de0, s);
    upload_vec<double>(ctx.dops.dc2de1, h.dc2de1, s);
    upload_vec<double>(ctx.dops.u2u, h.u2u, s);
    upload_vec<double>(ctx.dops.d2d, h.d2d, s);
    upload_vec<double>(ctx.dops.vop, h.vop, s);
    upload_vec<double>(ctx.dops.usurf, h.usurf, s);
  } else {
    upload_vec<float>(ctx.dops.uc2ue0, h.uc2ue0, s);
    upload_vec<float>(ctx.dops.uc2ue1, h.uc2ue1, s);
    upload_vec<float>(ctx.dops.dc2de0, h.dc2de0, s);
    upload_vec<float>(ctx.dops.dc2de1, h.dc2de1, s);
    upload_vec<float>(ctx.dops.u2u, h.u2u, s);
    upload_vec<float>(ctx.dops.d2d, h.d2d, s);
    upload_vec<float>(ctx.dops.vop, h.vop, s);
    upload_vec<float>(ctx.dops.usurf, h.usurf, s);
  }
  int* fm = ctx.dops.fft_map.as<int>(h.fft_map.size());
  int* im = ctx.dops.ifft_map.as<int>(h.ifft_map.size());
  PVFMM_CUDA_CHECK(cudaMemcpyAsync(fm, h.fft_map.data(), h.fft_map.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  PVFMM_CUDA_CHECK(cudaMemcpyAsync(im, h.ifft_map.data(), h.ifft_map.size() * sizeof(int), cudaMemcpyHostToDevice, s));
  PVFMM_CUDA_CHECK(cudaStreamSynchronize(s));
}

void evaluate(Context& ctx, const void* den_in, bool den_float, void* out, bool out_float) {
  const bool f32 = ctx.precision == 1;
  switch (ctx.kernel) {
    case kLaplacePot:
      if (f32) evaluate_impl<float, kKerLaplace, kKerLaplace>(ctx, den_in, den_float, out, out_float);
      else evaluate_impl<double, kKerLaplace, kKerLaplace>(ctx, den_in, den_float, out, out_float);
      break;
    case kLaplaceGrad:
      if (f32) evaluate_impl<float, kKerLaplaceGrad, kKerLaplace>(ctx, den_in, den_float, out, out_float);
      else evaluate_impl<double, kKerLaplaceGrad, kKerLaplace>(ctx, den_in, den_float, out, out_float);
      break;
    case kLaplacePotGrad:
      if (f32) evaluate_impl<float, kKerLaplacePG, kKerLaplace>(ctx, den_in, den_float, out, out_float);
      else evaluate_impl<double, kKerLaplacePG, kKerLaplace>(ctx, den_in, den_float, out, out_float);
      break;
    case kStokesVel:
      if (f32) evaluate_impl<float, kKerStokes, kKerStokes>(ctx, den_in, den_float, out, out_float);
      else evaluate_impl<double, kKerStokes, kKerStokes>(ctx, den_in, den_float, out, out_float);
      break;
    default:
      throw std::runtime_error("unsupported kernel");
  }
}

}  // namespace pvfmm_b200

namespace pvfmm_b200 {
void evaluate_adjoint(Context& ctx, const void* trg_den, bool in_float, void* src_out, bool out_float) {
  (void)ctx; (void)trg_den; (void)in_float; (void)src_out; (void)out_float;
  throw std::runtime_error("adjoint evaluation is not available in this build");
}
}  // namespace pvfmm_b200
