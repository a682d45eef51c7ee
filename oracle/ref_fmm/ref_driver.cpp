// Test-infrastructure driver around the reference's own C interface
// (src/pvfmm-wrapper.cpp, compiled here from the reference's sources over the
// stand-ins in shim/).  It adds read-only access to the reference's octree
// and interaction lists after an evaluation, so that the oracle's tree, lists
// and FMM values can be pinned to the reference's, and a stage-time hook for
// the CPU baseline.  Nothing of the product library links this.
#include "pvfmm-wrapper.cpp"

#include <omp.h>

#include <chrono>
#include <cstdint>
#include <cstring>
#include <iostream>
#include <sstream>

extern "C" void scipy_openblas_set_num_threads(int);

namespace {
typedef pvfmm::FMM_Node<pvfmm::MPI_Node<double> > RefNode;

// The reference calls BLAS from inside its OpenMP loops (one GEMM per block
// per thread), so the BLAS library itself runs single-threaded.
__attribute__((constructor)) void single_threaded_blas() { scipy_openblas_set_num_threads(1); }

// (X, Y, Z, depth) of a node's Morton id, X in units of 2^-30.
void node_key(RefNode* n, int64_t* out) {
  double c[3];
  n->GetMortonId().GetCoord(c);
  for (int k = 0; k < 3; ++k) out[k] = (int64_t)(c[k] * (double)(1u << 30) + 0.5);
  out[3] = n->Depth();
}

std::vector<RefNode*> nodes_of(const void* ctx_) {
  PVFMMContext<double>* ctx = (PVFMMContext<double>*)ctx_;
  std::vector<RefNode*> out;
  std::vector<RefNode*>& all = ctx->tree->GetNodeList();
  for (RefNode* n : all)
    if (!n->IsGhost()) out.push_back(n);
  return out;
}
}  // namespace

extern "C" {

// Nodes of the last tree, one record of 10 int64 per node in the tree's node
// order: X, Y, Z, depth, leaf, #sources, #targets (points held by the leaf;
// a source position counts once whether it carries single-layer values,
// double-layer values or both), pt_cnt[0], pt_cnt[1], 0.  Returns the node
// count; writes at most cap records.
long ref_tree_nodes(const void* ctx, int64_t* out, long cap) {
  std::vector<RefNode*> nodes = nodes_of(ctx);
  for (long i = 0; i < (long)nodes.size() && i < cap; ++i) {
    RefNode* n = nodes[i];
    int64_t* r = out + 10 * i;
    node_key(n, r);
    r[4] = n->IsLeaf() ? 1 : 0;
    r[5] = (int64_t)(std::max(n->src_coord.Dim(), n->surf_coord.Dim()) / 3);
    r[6] = (int64_t)(n->trg_coord.Dim() / 3);
    r[7] = (int64_t)n->pt_cnt[0];
    r[8] = (int64_t)n->pt_cnt[1];
    r[9] = 0;
  }
  return (long)nodes.size();
}

// Interaction-list entries of the last tree, one record of 6 int64 per
// non-empty slot: owner node index (tree node order), list type (the
// reference's Mat_Type: U0 8, U1 9, U2 10, W 12, X 13, V1 14), slot, member
// node index, 0, 0.  Returns the record count; writes at most cap records.
long ref_tree_lists(const void* ctx, int64_t* out, long cap) {
  std::vector<RefNode*> nodes = nodes_of(ctx);
  std::map<RefNode*, long> index;
  for (long i = 0; i < (long)nodes.size(); ++i) index[nodes[i]] = i;
  const int types[] = {pvfmm::U0_Type, pvfmm::U1_Type, pvfmm::U2_Type, pvfmm::W_Type, pvfmm::X_Type, pvfmm::V1_Type};
  long cnt = 0;
  for (long i = 0; i < (long)nodes.size(); ++i)
    for (int t : types) {
      pvfmm::Vector<RefNode*>& L = nodes[i]->interac_list[t];
      for (size_t s = 0; s < L.Dim(); ++s) {
        if (!L[s]) continue;
        auto it = index.find(L[s]);
        if (cnt < cap) {
          int64_t* r = out + 6 * cnt;
          r[0] = i;
          r[1] = t;
          r[2] = (int64_t)s;
          r[3] = it == index.end() ? -1 : it->second;
          r[4] = r[5] = 0;
        }
        ++cnt;
      }
    }
  return cnt;
}

// The reference's integral of a kernel's expansion (m2l) kernel over the
// box [0, r]^3 at target s with a constant unit density (cheb_integ of degree
// 0, include/cheb_utils.txx:1037), the input of its periodic-boundary
// precompute: out[j + k*k0] as cheb_integ returns it.  Returns the number of
// values, or -1 for an unknown kernel.
int ref_cheb_integ0(int kernel, const double* s, double r, double* out) {
  const pvfmm::Kernel<double>* ker = nullptr;
  if (kernel == PVFMMLaplacePotential) ker = &pvfmm::LaplaceKernel<double>::potential();
  if (kernel == PVFMMLaplaceGradient) ker = &pvfmm::LaplaceKernel<double>::gradient();
  if (kernel == PVFMMStokesVelocity) ker = &pvfmm::StokesKernel<double>::velocity();
  if (!ker) return -1;
  ker->Initialize(false);
  double sc[3] = {s[0], s[1], s[2]};
  std::vector<double> v = pvfmm::cheb_integ<double>(0, sc, r, *ker->k_m2l);
  std::memcpy(out, v.data(), sizeof(double) * v.size());
  return (int)v.size();
}

// Sets the number of OpenMP threads the reference uses (0 leaves the
// current setting) and returns the count in effect.
int ref_set_threads(int n) {
  if (n > 0) omp_set_num_threads(n);
  return omp_get_max_threads();
}

// Enables the reference's profiler (pvfmm::Profile, the per-stage tags of
// fmm_tree.txx / fmm_pts.txx) for the following evaluations, with a cleared
// log, or turns it off (keeping the log).
void ref_profile_enable(int on) {
  if (on) pvfmm::Profile::reset();
  pvfmm::Profile::Enable(on != 0);
}

// The profiler's table (pvfmm::Profile::print: one line per tag, indented by
// nesting, then t_min t_avg t_max ... in seconds; printing consumes the log).
// With buf == NULL the table is formed and kept, and its length returned;
// a following call with a buffer copies the kept table (at most cap - 1
// bytes, NUL-terminated).
long ref_profile_report(char* buf, long cap) {
  static std::string table;
  if (!buf) {
    std::stringstream ss;
    std::streambuf* old = std::cout.rdbuf(ss.rdbuf());
    pvfmm::Profile::print();
    std::cout.rdbuf(old);
    table = ss.str();
    return (long)table.size();
  }
  if (cap > 0) {
    const long n = std::min<long>(cap - 1, (long)table.size());
    std::memcpy(buf, table.data(), n);
    buf[n] = 0;
  }
  return (long)table.size();
}

// The reference's C++ particle interface (include/pvfmm.txx:216-328): a tree
// over single-layer points (n_sl, may be 0) and a separate double-layer point
// set (n_dl, may be 0; k0 + 3 values per point) with the targets as the
// tree's point set, coordinates in [0,1)^3 used as given, FreeSpace;
// PtFMM_Evaluate writes n_trg * k1 values to out.  Returns 0, or 1 for an
// unknown kernel.
int ref_ptfmm_eval_bc(int kernel, int m, int max_pts, int periodic, long n_sl, const double* sl_coord,
                      const double* sl_den, long n_dl, const double* dl_coord, const double* dl_den, long n_trg,
                      const double* trg_coord, double* out);
int ref_ptfmm_eval(int kernel, int m, int max_pts, long n_sl, const double* sl_coord, const double* sl_den,
                   long n_dl, const double* dl_coord, const double* dl_den, long n_trg, const double* trg_coord,
                   double* out) {
  return ref_ptfmm_eval_bc(kernel, m, max_pts, 0, n_sl, sl_coord, sl_den, n_dl, dl_coord, dl_den, n_trg, trg_coord,
                           out);
}

// The same with the boundary type: `periodic` is the BoundaryType value
// (0 FreeSpace, 1 PX, 2 PXY, 3 PXYZ == Periodic).
int ref_ptfmm_eval_bc(int kernel, int m, int max_pts, int periodic, long n_sl, const double* sl_coord,
                      const double* sl_den, long n_dl, const double* dl_coord, const double* dl_den, long n_trg,
                      const double* trg_coord, double* out) {
  const pvfmm::Kernel<double>* ker = nullptr;
  if (kernel == PVFMMLaplacePotential) ker = &pvfmm::LaplaceKernel<double>::potential();
  if (kernel == PVFMMLaplaceGradient) ker = &pvfmm::LaplaceKernel<double>::gradient();
  if (kernel == PVFMMStokesVelocity) ker = &pvfmm::StokesKernel<double>::velocity();
  if (!ker) return 1;
  const int k0 = ker->ker_dim[0], k1 = ker->ker_dim[1];
  std::vector<double> sc(sl_coord, sl_coord + 3 * n_sl), sv(sl_den, sl_den + k0 * n_sl);
  std::vector<double> dc(dl_coord, dl_coord + 3 * n_dl), dv(dl_den, dl_den + (k0 + 3) * n_dl);
  std::vector<double> tc(trg_coord, trg_coord + 3 * n_trg);
  pvfmm::PtFMM<double> matrices;
  matrices.Initialize(m, MPI_COMM_WORLD, ker);
  if (periodic < 0 || periodic > 3) return 1;
  auto* tree = pvfmm::PtFMM_CreateTree(sc, sv, dc, dv, tc, MPI_COMM_WORLD, max_pts, (pvfmm::BoundaryType)periodic);
  tree->SetupFMM(&matrices);
  std::vector<double> val;
  pvfmm::PtFMM_Evaluate(tree, val, n_trg);
  std::memcpy(out, val.data(), sizeof(double) * std::min<size_t>(val.size(), (size_t)n_trg * k1));
  delete tree;
  return 0;
}

}  // extern "C"
