// Per-context state of libpvfmm_b200: operators on the device, the octree of
// the last setup, interaction lists and evaluation buffers.
#pragma once

#include <array>
#include <vector>

#include "fmm_device.cuh"
#include "fmm_host.hpp"

namespace pvfmm_b200 {

// Octree of the last setup=1 call, all on the device except the level table.
// Nodes are stored level by level; each level is in Morton order and the 8
// children of an internal node are consecutive in the next level.
struct DevTree {
  long n_nodes = 0;
  int depth = 0;                      // deepest level
  std::vector<long> level_off;        // level d occupies [level_off[d], level_off[d+1])
  std::vector<long> n_internal;       // internal nodes per level
  DevBuf key;                         // MKey per node
  DevBuf leaf;                        // uint8 per node
  DevBuf parent, child0;              // int per node (-1 if none)
  DevBuf src_lo, src_hi, trg_lo, trg_hi;   // int per node: ranges into the sorted points
  DevBuf colleague;                   // int[27] per node
  DevBuf int_idx;                     // internal node ids, level by level (offsets int_off)
  std::vector<long> int_off;
  // point data (sorted)
  long n_src = 0, n_trg = 0;
  // point sets the source positions stand for: 1 per density passed
  // (sl_den single layer, dl_den double layer), 0 when neither is; each
  // counts in the refinement and in pt_cnt[0] (fmm_node.txx:81-92,
  // fmm_pts.txx:1332-1333)
  int src_weight = 1;
  bool src_counted = true;            // src_weight > 0
  int layers = 1;                     // densities passed at setup: 1 single layer, 2 double layer, 3 both
  DevBuf src_perm, trg_perm;          // int: sorted index -> input index
  DevBuf src_key, trg_key;            // MKey (sorted)
  DevBuf src_leaf, trg_leaf;          // int: leaf node id of each sorted point
  DevBuf sx, sy, sz, tx, ty, tz;      // Real coordinates relative to the point's leaf centre
  // compact node lists
  long n_sleaf = 0, n_tleaf = 0, n_vsrc = 0, n_vtrg = 0, n_xtrg = 0;
  DevBuf sleaf, tleaf;                // leaves with sources / targets
  DevBuf vsrc, vtrg;                  // non-leaf nodes: spectra sources / targets
  DevBuf node2vsrc;                   // int per node (-1)
  DevBuf vtab;                        // int[26] per vtrg: vsrc index per colleague offset (-1)
  DevBuf vmask;                       // unsigned per vtrg: bit o set when vtab[o] >= 0 (vtrg sorted by it)
  DevBuf vmorton;                     // int per vtrg: position of the target of each Morton rank
  // tiles of 128 Morton-consecutive V-list targets (tcgen05 Hadamard): the
  // sorted union of their source parents and each (target, offset)'s index
  // into it; built on first use after a tree build
  DevBuf vunion, vucount, vlocal;
  bool vtiles_valid = false;
  DevBuf xtrg;                        // target nodes with X-list entries
  DevBuf x_off, x_list;               // CSR over xtrg
  DevBuf p_off, p_list;               // CSR over tleaf: P2P source leaves
  DevBuf w_off, w_list;               // CSR over tleaf: W source nodes
  // periodic boundaries: the image code of each p / x / w list entry
  // ((sx+1) + 3(sy+1) + 9(sz+1), the unit-cube shift that places the source)
  DevBuf p_img, x_img, w_img;
  long n_p2p = 0, n_x = 0, n_w = 0;   // list sizes
  double scale_x = 1, shift_x[3] = {0, 0, 0};
  bool valid = false;
};

// Device copies of the operators in the working precision.
struct DevOps {
  DevBuf uc2ue0, uc2ue1, dc2de0, dc2de1, u2u, d2d, vop;
  DevBuf vop_frag;  // mixed form: Hadamard operators as TF32 hi/lo MMA fragments
  DevBuf vop_tc5;   // mixed form, ke = 1: Hadamard operators in the tcgen05 shared-memory layout
  DevBuf ue_basis;  // mixed Stokes form: din x r32, the upward directions above the FP32 cutoff
  DevBuf bc;        // periodic boundaries: din x dout, root upward equivalent -> root downward check
  DevBuf d2d_f2;    // rd x (8 dout): D2D through the kept downward directions (when rd is small)
  DevBuf usurf;     // ns x 3 (Real)
  DevBuf fft_map, ifft_map;
};

struct Context {
  int kernel = 0;
  KernelInfo ki{};
  int m = 0, ns = 0, max_pts = 0;
  int precision = 0;      // 0 plain FP64, 1 mixed FP32
  bool float_api = false; // created by the F entry points
  bool unit_box = false;  // coordinates used as given in [0,1)^3, tree points = targets
  // source points carry one layer each (the C++ interface's separate single-
  // and double-layer point sets, passed concatenated with zero values for the
  // other layer): a source counts once in the tree whatever densities are passed
  bool layer_points = false;
  HostOperators hops;
  DevOps dops;
  // inner widths of the uploaded check -> equivalent factors: the directions
  // the cutoff kept, padded to even (upward ru, downward rd); the first r32
  // upward ones span the mixed Stokes form's projection (0 otherwise)
  int ru = 0, rd = 0, r32 = 0;
  bool d2d_factored = false;  // D2D as (dc DC2DE0) d2d_f2 over rd directions
  // periodic boundaries (box_size > 0): points scaled by 1 / box_size and
  // wrapped into the unit cube; bc_lattice selects the lattice-sum operator,
  // bc_user an operator added to the 5x5x5-image one (empty: none)
  bool periodic = false;
  int periodic_axes = 7;  // bit 0 x, bit 1 y, bit 2 z: 7 = PXYZ (the C interface), 1 = PX, 3 = PXY
  double box_size = 0;
  int bc_lattice = 0;
  std::vector<double> bc_user;
  DevTree tree;
  cudaStream_t stream = nullptr;
  int device = 0;
  // evaluation buffers
  DevBuf den;             // sorted densities (Real, n_src x k0)
  DevBuf surf;            // sorted double-layer values (FP64, n_src x (k0 + 3))
  DevBuf ue_c;            // mixed form: projected upward equivalent densities
  DevBuf pot;             // sorted target values (Real, n_trg x k1)
  DevBuf ue, dc;          // per node (Real)
  DevBuf uc_c, tmp_c, de_c;  // compact GEMM buffers
  DevBuf spec_in, spec_out;  // V-list spectra
  DevBuf scratch;         // sort / scan temporaries
  DevBuf scratch2;
  DevBuf io_src, io_trg, io_den, io_val;  // staging for host-pointer calls
  DevBuf io_dl;
  DevBuf stat;            // small status / reduction buffer
  DevBuf t[24];           // temporaries of the tree build, reused across calls
  std::vector<DevBuf> lvlR, lvlS;  // per-level internal-node keys (refined / balanced)
  long n_launch = 0;      // own kernels launched since context creation
  std::vector<float> stage_ms;
  std::array<cudaEvent_t, 13> ev{};
  bool events_ready = false;
  // pinned host staging
  void* pinned = nullptr;
  size_t pinned_cap = 0;
  int* chk = nullptr;  // pinned slots for counts read back at the end of a tree build
  int* tc5_err = nullptr;  // device error word of the running evaluation's tcgen05 Hadamard (nullptr: none)
  DevBuf tc5_err_buf;
  int* tc5_err_host = nullptr;  // pinned copy of it, read after the evaluation synchronises
  // host-pointer evaluations upload the densities on a side stream while the
  // tree is built; the evaluation waits for den_ev when den_pending
  cudaStream_t side = nullptr;
  cudaEvent_t den_ev = nullptr;
  bool den_pending = false;
};

// tree.cu
void build_tree(Context& ctx, const void* src_pos, long n_src, const void* trg_pos, long n_trg, bool pos_float,
                int src_weight, bool trg_alias);
// eval.cu
// den_in: single-layer densities (n_src x k0) or NULL; dl_in: double-layer
// values (n_src x (k0 + 3)) or NULL; both in the input order and precision
void evaluate(Context& ctx, const void* den_in, const void* dl_in, bool den_float, void* out, bool out_float);
void upload_operators(Context& ctx);
// hadamard_tc.cu: mixed-form V-list Hadamard of target parents [p0, p0+np)
// on tcgen05 (rows of sout relative to p0) over n3h frequencies starting at
// frequency f_base of the operators, and its operator layout
void launch_hadamard_tc5(Context& ctx, int n3h, long f_base, const void* sin_, void* sout, long p0, long np);
void hadamard_tc5_operator_layout(const std::vector<double>& vop, int n3h, std::vector<float>& out);
// translate.cu: C[crow(i)] (+)= 2^(-deg depth(key[arow(i)])) A[arow(i)] B on the FP64
// tensor cores (rows gathered / scattered through the index lists when given);
// with ksplit > 1 the K range is cut into ksplit equal pieces summed in
// `partial` (ksplit * M * N doubles) and added in a fixed order
void translate_gemm(cudaStream_t s, long M, int N, int K, const double* A, long lda, const int* arows,
                    const double* B, long ldb, double* C, long ldc, const int* crows, const MKey* scale_keys,
                    bool accumulate, int ksplit = 1, double* partial = nullptr, int deg = 1);

}  // namespace pvfmm_b200
