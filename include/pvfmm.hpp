// pvfmm.hpp -- C++ particle-FMM interface of libpvfmm_b200 (header only).
//
// Mirrors the particle half of the reference C++ interface
// (dmalhotra/pvfmm include/pvfmm.hpp:199-318, include/pvfmm.txx:216-328,
// include/kernel.hpp:27-136) on top of the C interface in pvfmm.h, so code
// written against the reference keeps its shape:
//
//   const pvfmm::Kernel<double>& ker = pvfmm::LaplaceKernel<double>::gradient();
//   pvfmm::PtFMM<double> matrices;
//   matrices.Initialize(m, comm, &ker);
//   auto* tree = pvfmm::PtFMM_CreateTree(src_coord, src_value, trg_coord, comm, max_pts, pvfmm::FreeSpace);
//   tree->SetupFMM(&matrices);
//   std::vector<double> trg_value;
//   pvfmm::PtFMM_Evaluate(tree, trg_value, n_trg);
//   tree->ClearFMMData();
//   pvfmm::PtFMM_Evaluate(tree, trg_value, n_trg, &new_src_value);
//   delete tree;
//
// As in the reference C++ interface (unlike PVFMMEval), coordinates must lie
// in [0,1)^3 and are used as given: no bounding-box rescale and no seed grid
// (the tree's point set is the targets, include/pvfmm.txx:229-240).
// Double-layer sources have their own point set (surf_coord, k0 + 3 values
// per point) for the kernels with a double-layer kernel (LaplaceKernel<T>::
// potential(), StokesKernel<T>::velocity()).
// Differences: single rank; free space only.
// Real = float runs the mixed-precision form.
#ifndef PVFMM_B200_PVFMM_HPP_
#define PVFMM_B200_PVFMM_HPP_

#include <algorithm>
#include <stdexcept>
#include <string>
#include <type_traits>
#include <vector>

#include "pvfmm.h"

namespace pvfmm {

// Boundary types with the reference's values (include/mpi_tree.hpp:23-30):
// free space, or periodic along x (PX), x and y (PXY) or all axes (PXYZ ==
// Periodic).
enum BoundaryType { FreeSpace = 0, PX, PXY, PXYZ, Periodic = PXYZ };

// Kernel object (reference include/kernel.hpp:27-106).  ker_poten is the
// direct evaluation k_out += sum_s K(trg - src) v_src (include/kernel.hpp:40-41),
// run on the GPU through PVFMMKernelEvalD.
template <class T>
struct Kernel {
  typedef void (*Ker_t)(T* r_src, int src_cnt, T* v_src, int dof, T* r_trg, int trg_cnt, T* k_out, void* mem_mgr);
  int dim = 3;
  int ker_dim[2] = {0, 0};
  std::string ker_name;
  PVFMMKernel id = PVFMMLaplacePotential;
  Ker_t ker_poten = nullptr;

  // M[i*k0+j][t*k1+k] = K_jk(trg_t - src_i) (include/kernel.txx:1059-1135),
  // built one unit density at a time.
  void BuildMatrix(T* r_src, int src_cnt, T* r_trg, int trg_cnt, T* k_out) const {
    const size_t row_len = (size_t)trg_cnt * ker_dim[1];
    std::vector<T> row(row_len);
    for (int s = 0; s < src_cnt; ++s)
      for (int j = 0; j < ker_dim[0]; ++j) {
        std::fill(row.begin(), row.end(), (T)0);
        T f[3] = {0, 0, 0};
        f[j] = 1;
        ker_poten(r_src + 3 * s, 1, f, 1, r_trg, trg_cnt, row.data(), nullptr);
        std::copy(row.begin(), row.end(), k_out + ((size_t)s * ker_dim[0] + j) * row_len);
      }
  }
};

namespace detail {
template <class T>
void ker_poten_gpu(PVFMMKernel id, int k0, int k1, T* r_src, int src_cnt, T* v_src, T* r_trg, int trg_cnt, T* k_out) {
  std::vector<double> s(r_src, r_src + 3 * (size_t)src_cnt), v(v_src, v_src + (size_t)k0 * src_cnt),
      t(r_trg, r_trg + 3 * (size_t)trg_cnt), o(k_out, k_out + (size_t)k1 * trg_cnt);
  if (PVFMMKernelEvalD(id, s.data(), v.data(), src_cnt, t.data(), o.data(), trg_cnt) != 0)
    throw std::runtime_error(PVFMMGetLastError());
  for (size_t i = 0; i < o.size(); ++i) k_out[i] = (T)o[i];
}
template <class T, PVFMMKernel ID, int K0, int K1>
void ker_fn(T* r_src, int src_cnt, T* v_src, int dof, T* r_trg, int trg_cnt, T* k_out, void*) {
  if (dof != 1) throw std::runtime_error("ker_poten: dof must be 1");  // as include/kernel.txx:1141
  ker_poten_gpu<T>(ID, K0, K1, r_src, src_cnt, v_src, r_trg, trg_cnt, k_out);
}
template <class T, PVFMMKernel ID, int K0, int K1>
const Kernel<T>& make_kernel(const char* name) {
  static const Kernel<T> k = [&] {
    Kernel<T> r;
    r.ker_dim[0] = K0;
    r.ker_dim[1] = K1;
    r.ker_name = name;
    r.id = ID;
    r.ker_poten = &ker_fn<T, ID, K0, K1>;
    return r;
  }();
  return k;
}
}  // namespace detail

// Kernel families (reference include/kernel.hpp:160-180, kernel.txx:1333-1479).
template <class T>
struct LaplaceKernel {
  static const Kernel<T>& potential() { return detail::make_kernel<T, PVFMMLaplacePotential, 1, 1>("laplace"); }
  static const Kernel<T>& gradient() { return detail::make_kernel<T, PVFMMLaplaceGradient, 1, 3>("laplace_grad"); }
  // extension: potential and -grad in one pass
  static const Kernel<T>& potgrad() { return detail::make_kernel<T, PVFMMLaplacePotGrad, 1, 4>("laplace_potgrad"); }
};
template <class T>
struct StokesKernel {
  static const Kernel<T>& velocity() { return detail::make_kernel<T, PVFMMStokesVelocity, 3, 3>("stokes_vel"); }
};

// Translation operators of one kernel and order (reference FMM_Pts::Initialize,
// include/fmm_pts.txx:223-331).  The operators are built when a tree is set up.
template <class Real>
class PtFMM {
 public:
  void Initialize(int mult_order, const MPI_Comm& comm, const Kernel<Real>* kernel) {
    (void)comm;
    if (!kernel) throw std::runtime_error("PtFMM::Initialize: null kernel");
    m_ = mult_order;
    kernel_ = kernel;
  }
  int MultipoleOrder() const { return m_; }
  const Kernel<Real>* kernel() const { return kernel_; }

 private:
  int m_ = 0;
  const Kernel<Real>* kernel_ = nullptr;
};

// Octree plus its evaluation state (reference FMM_Tree, include/fmm_tree.hpp).
template <class Real>
class PtFMM_Tree {
 public:
  PtFMM_Tree(const std::vector<Real>& src_coord, const std::vector<Real>& src_value,
             const std::vector<Real>& trg_coord, int max_pts, BoundaryType bndry = FreeSpace)
      : src_(src_coord), den_(src_value), trg_(trg_coord), max_pts_(max_pts), bndry_(bndry) {}
  // with a separate double-layer point set (surf_coord, k0 + 3 values per point)
  PtFMM_Tree(const std::vector<Real>& src_coord, const std::vector<Real>& src_value,
             const std::vector<Real>& surf_coord, const std::vector<Real>& surf_value,
             const std::vector<Real>& trg_coord, int max_pts, BoundaryType bndry = FreeSpace)
      : src_(src_coord), den_(src_value), surf_(surf_coord), dl_(surf_value), trg_(trg_coord), max_pts_(max_pts),
        bndry_(bndry) {}
  ~PtFMM_Tree() { release(); }
  PtFMM_Tree(const PtFMM_Tree&) = delete;
  PtFMM_Tree& operator=(const PtFMM_Tree&) = delete;

  // Creates the GPU context for the kernel and order of `mat` (reference
  // FMM_Tree::SetupFMM, include/fmm_tree.txx:72-183); the octree is built by
  // the next evaluation.
  void SetupFMM(PtFMM<Real>* mat) {
    release();
    const Kernel<Real>* k = mat->kernel();
    if (!k) throw std::runtime_error("SetupFMM: PtFMM not initialized");
    k0_ = k->ker_dim[0];
    k1_ = k->ker_dim[1];
    const int precision = std::is_same<Real, float>::value ? PVFMMPrecisionMixed : PVFMMPrecisionPlain;
    // periodic: period 1, the unit cube itself (the coordinates are used as
    // given), along x (PX), x and y (PXY) or all axes (PXYZ == Periodic)
    ctx_ = PVFMMCreateContextExD(bndry_ != FreeSpace ? 1.0 : -1.0, max_pts_, mat->MultipoleOrder(), k->id, precision);
    if (!ctx_) throw std::runtime_error(PVFMMGetLastError());
    if (bndry_ == PX || bndry_ == PXY) {
      if (PVFMMSetPeriodicAxes(ctx_, bndry_ == PX ? 1 : 3) != 0) throw std::runtime_error(PVFMMGetLastError());
    }
    if (PVFMMSetUnitBox(ctx_, 1) != 0) throw std::runtime_error(PVFMMGetLastError());
    // both point sets count in the tree (include/fmm_node.txx:81-92): they are
    // passed concatenated, each point with its own layer's values
    if (!surf_.empty() && PVFMMSetLayerPoints(ctx_, 1) != 0) throw std::runtime_error(PVFMMGetLastError());
    needs_setup_ = true;
  }
  // Clears expansions between evaluations (reference FMM_Tree::ClearFMMData);
  // every evaluation here starts from cleared expansions.
  void ClearFMMData() {}

  void evaluate(std::vector<Real>& trg_val, const std::vector<Real>* sl_density,
                const std::vector<Real>* dl_density = nullptr) {
    if (!ctx_) throw std::runtime_error("PtFMM_Evaluate: call SetupFMM first");
    if (sl_density) den_ = *sl_density;
    if (dl_density) dl_ = *dl_density;
    const long n_sl = (long)src_.size() / 3, n_dl = (long)surf_.size() / 3, nt = (long)trg_.size() / 3;
    const long ns = n_sl + n_dl;
    std::vector<double> s(src_.begin(), src_.end()), t(trg_.begin(), trg_.end());
    s.insert(s.end(), surf_.begin(), surf_.end());
    std::vector<double> d, dl;
    if (n_dl == 0) {
      d.assign(den_.begin(), den_.end());
    } else {  // single-layer points then double-layer points, zeros for the other layer
      if (den_.size() != (size_t)(n_sl * k0_) || dl_.size() != (size_t)(n_dl * (k0_ + 3)))
        throw std::runtime_error("PtFMM_Evaluate: density sizes do not match the point sets");
      d.assign((size_t)ns * k0_, 0.0);
      std::copy(den_.begin(), den_.end(), d.begin());
      dl.assign((size_t)ns * (k0_ + 3), 0.0);
      std::copy(dl_.begin(), dl_.end(), dl.begin() + (size_t)n_sl * (k0_ + 3));
    }
    std::vector<double> out((size_t)nt * k1_);
    PVFMMEvalD(s.data(), d.empty() ? nullptr : d.data(), dl.empty() ? nullptr : dl.data(), ns, t.data(),
               out.data(), nt, ctx_, needs_setup_ ? 1 : 0);
    const std::string err = PVFMMGetLastError();
    if (!err.empty()) throw std::runtime_error(err);
    needs_setup_ = false;
    trg_val.assign(out.begin(), out.end());
  }

 private:
  void release() {
    if (ctx_) PVFMMDestroyContextD(&ctx_);
  }
  std::vector<Real> src_, den_, surf_, dl_, trg_;
  int max_pts_;
  BoundaryType bndry_ = FreeSpace;
  int k0_ = 1, k1_ = 1;
  void* ctx_ = nullptr;
  bool needs_setup_ = true;
};

template <class Real>
PtFMM_Tree<Real>* PtFMM_CreateTree(const std::vector<Real>& sl_coord, const std::vector<Real>& sl_density,
                                   const std::vector<Real>& dl_coord, const std::vector<Real>& dl_density,
                                   const std::vector<Real>& trg_coord, MPI_Comm comm, int max_pts = 100,
                                   BoundaryType bndry = FreeSpace, int init_depth = 0) {
  (void)comm;
  (void)init_depth;
  if (bndry != FreeSpace && bndry != PX && bndry != PXY && bndry != PXYZ)
    throw std::runtime_error("PtFMM_CreateTree: unknown boundary type");
  return new PtFMM_Tree<Real>(sl_coord, sl_density, dl_coord, dl_density, trg_coord, max_pts, bndry);
}

template <class Real>
PtFMM_Tree<Real>* PtFMM_CreateTree(const std::vector<Real>& sl_coord, const std::vector<Real>& sl_density,
                                   const std::vector<Real>& trg_coord, MPI_Comm comm, int max_pts = 100,
                                   BoundaryType bndry = FreeSpace, int init_depth = 0) {
  const std::vector<Real> none;
  return PtFMM_CreateTree(sl_coord, sl_density, none, none, trg_coord, comm, max_pts, bndry, init_depth);
}

// Reference include/pvfmm.txx:257-328: optional new densities, evaluate,
// values in input order.  loc_size is accepted for signature compatibility.
template <class Real>
void PtFMM_Evaluate(const PtFMM_Tree<Real>* tree, std::vector<Real>& trg_val, size_t loc_size = 0,
                    const std::vector<Real>* sl_density = nullptr, const std::vector<Real>* dl_density = nullptr) {
  (void)loc_size;
  const_cast<PtFMM_Tree<Real>*>(tree)->evaluate(trg_val, sl_density, dl_density);
}

}  // namespace pvfmm

#endif  // PVFMM_B200_PVFMM_HPP_
