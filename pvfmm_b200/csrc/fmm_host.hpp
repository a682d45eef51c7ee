// Host-side declarations shared by the precompute, the tree/evaluation driver
// and the C interface of libpvfmm_b200.
#pragma once

#include <cstdint>
#include <string>
#include <vector>

namespace pvfmm_b200 {

// Kernel ids follow the PVFMMKernel enum (reference include/pvfmm.h:21-28),
// plus 6 = Laplace potential+gradient.
enum KernelId {
  kLaplacePot = 0,
  kLaplaceGrad = 1,
  kStokesPress = 2,
  kStokesVel = 3,
  kStokesVelGrad = 4,
  kBiotSavart = 5,
  kLaplacePotGrad = 6
};

// Expansion kernels (the k_s2m/k_m2m/k_m2l/k_l2l sub-kernels of
// include/kernel.txx:1333-1344, 1475-1479).
// Stokes pressure, Stokes velocity gradient and Biot-Savart have no separate
// expansion kernels and expand themselves (kernel.txx:894-901, 1480-1511).
enum ExpKernel { kExpLaplace = 0, kExpStokes = 1, kExpStokesPress = 2, kExpStokesGrad = 3, kExpBiotSavart = 4 };

// Source and target dims of an expansion kernel (equivalent densities carry
// kin components, check potentials kout).
void exp_kernel_dims(int exp_kernel, int* kin, int* kout);

struct KernelInfo {
  int id;
  const char* name;        // reference ker_name (kernel.txx:1334, 1341, 1476)
  int k0, k1;              // source / target dims of the s2t kernel
  int exp_kernel;          // ExpKernel of the expansions
  int ke;                  // dims of the expansion kernel (ke x ke)
  double src_scal[3];      // scale exponents of the s2t kernel (kernel.txx:64-196)
  double trg_scal[9];
  int flops;               // per-pair flop count convention (kernel.txx:1277,1317,1352)
  int deg;                 // degree of the expansion kernel, K(x/2) = 2^deg K(x): check -> equivalent
                           // operators of level l are 2^(-deg l) times the level-0 ones
};

// Kernels the CUDA evaluation implements (every PVFMMKernel value, plus the
// Laplace potential+gradient).
bool kernel_info(int id, KernelInfo* out);
// Same as kernel_info (kept for the host precompute's callers).
bool kernel_info_host(int id, KernelInfo* out);

// Level-0 operators of one kernel and multipole order.  All FP64, row-major,
// row-vector convention (out_row = in_row * M), as in fmm_pts.txx:453-764.
struct HostOperators {
  int kernel = -1, m = 0, ns = 0, ke = 1, n1 = 0, n3 = 0, n3h = 0;
  // expansion dims: equivalent densities ns*kin, check potentials ns*kout
  // (kin = kout = ke for the kernels the CUDA path evaluates)
  int kin = 1, kout = 1;
  bool mixed = false;
  std::vector<double> usurf;            // ns x 3 unit cube-surface points u in [-1,1]^3
  // check -> equivalent factors, r = min(ns*kin, ns*kout):
  // C2E0 (ns*kout) x r, C2E1 r x (ns*kin)
  std::vector<double> uc2ue0, uc2ue1;
  // (ns*kin) x (ns*kin): orthogonal projector onto the upward equivalent
  // directions whose singular value (equivalent -> check) is above the FP32
  // cutoff 4*eps32*max; the mixed form applies it to the upward equivalent
  // densities before its FP32 stages
  std::vector<double> ue_proj;
  std::vector<int> ue32_dirs;           // the singular directions j (rows of UC2UE1) spanning ue_proj
  std::vector<double> dc2de0, dc2de1;
  std::vector<double> u2u;              // (8*ns*kin) x (ns*kin), row block c = child octant c
  std::vector<double> d2d;              // (ns*kout) x (8*ns*kout), column block c = child octant c
  std::vector<double> d2d_f2;           // r x (8*ns*kout): D2D = DC2DE0 * d2d_f2 (DC2DE1 * M_pe2c per block)
  std::vector<double> vop;              // complex (re,im): [n3h][26][8][8][kin][kout]
  std::vector<int> fft_map, ifft_map;   // ns grid indices (x + n1*y + n1*n1*z)
};

// Builds the operators.  `mixed` selects the pseudo-inverse cutoff of the
// mixed form: singular values below 4*eps32*max are dropped (the cutoff the
// reference's float build uses), otherwise 4*eps64*max (fmm_pts.txx:496-504).
// down_eps32: FP32 cutoff for the downward check -> equivalent factors only
// (and so for D2D), the mixed form's downward chain.
void build_operators(int kernel, int m, bool mixed, HostOperators& ops, bool down_eps32 = false);

// Periodic boundary operator (BoundaryType Periodic, fmm_pts.txx:790-1232):
// (ns*kin) x (ns*kout), root upward equivalent density -> root downward check
// potential of the periodic images outside the root's 3x3x3 block.  lattice
// false: the images of the 5x5x5 block (the reference built with
// PVFMM_EXTENDED_BC, its CMake default), any kernel; lattice true: the full
// lattice sum (the option off), for the kernels lattice_bc_supported()
// accepts (Laplace potential and gradient, Stokes velocity); throws otherwise.
bool lattice_bc_supported(int kernel);
// axes: the periodic axes (bit 0 x, bit 1 y, bit 2 z; 1 = PX, 3 = PXY,
// 7 = PXYZ == Periodic).
std::vector<double> build_bc_operator(int kernel, int m, bool lattice, int axes = 7);

// One-sided Jacobi SVD of a rows x cols row-major matrix (rows >= cols):
// A = U diag(S) V^T with U rows x cols (column j scaled to unit length, or
// zero when S_j == 0), V cols x cols.  Public for the CPU tests.
void jacobi_svd(int rows, int cols, const double* A, std::vector<double>& U, std::vector<double>& S,
                std::vector<double>& V);

// FP64 kernel matrix, BuildMatrix layout (kernel.txx:1059-1135):
// M[i*k0+j][t*k1+k] = K_jk(trg_t - src_i), r == 0 gives 0.
void exp_kernel_matrix(int exp_kernel, const double* src, int n_src, const double* trg, int n_trg,
                       double* M);

// Unit surface of PVFMM's surface() (fmm_pts.txx:54-97) as u in [-1,1]^3.
std::vector<double> unit_surface(int m);

void set_last_error(const std::string& msg);
const char* get_last_error();

}  // namespace pvfmm_b200
