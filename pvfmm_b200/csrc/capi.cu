// C interface of libpvfmm_b200 (declared in include/pvfmm.h).
//
// Mirrors the particle half of the reference C interface
// (src/pvfmm-wrapper.cpp:367-928): a context owns the operators, the device
// buffers and the tree of the last setup; PVFMMEval* copies host arrays to
// the device, runs the GPU pipeline and copies the values back.
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <limits>
#include <memory>
#include <mutex>
#include <string>

#include "../../include/pvfmm.h"
#include "fmm_context.cuh"

using namespace pvfmm_b200;

namespace {

constexpr unsigned int kMagic = 0x50564642u;  // "PVFB"

struct Handle {
  unsigned int magic = kMagic;
  Context ctx;
  void* adjoint = nullptr;  // companion context with sources and targets exchanged
};

Handle* as_handle(const void* p) {
  Handle* h = (Handle*)p;
  if (!h || h->magic != kMagic) throw std::runtime_error("invalid PVFMM context pointer");
  return h;
}

// A bounded wait of the tensor-core V-list Hadamard that ran out (its error
// word, copied to pinned memory at the end of the evaluation) fails the call
// that observes it once the context's stream is synchronised.
void check_tc5_error(Context& c) {
  if (c.tc5_err_host && *(volatile int*)c.tc5_err_host != 0) {
    const int e = *c.tc5_err_host;
    *c.tc5_err_host = 0;
    throw std::runtime_error("V-list tensor-core Hadamard: a bounded wait ran out (error word " + std::to_string(e) +
                             "); the results of that evaluation are invalid");
  }
}

void destroy_context(Context& c) {
  cudaSetDevice(c.device);
  if (c.stream) cudaStreamSynchronize(c.stream);
  DevBuf* bufs[] = {&c.dops.uc2ue0, &c.dops.uc2ue1, &c.dops.dc2de0, &c.dops.dc2de1, &c.dops.u2u,
                    &c.dops.d2d, &c.dops.vop, &c.dops.vop_frag, &c.dops.vop_tc5, &c.tc5_err_buf,
                    &c.dops.ue_basis, &c.ue_c, &c.dops.usurf, &c.dops.fft_map, &c.dops.ifft_map, &c.den,
                    &c.surf, &c.pot, &c.ue, &c.dc, &c.uc_c, &c.tmp_c, &c.de_c, &c.spec_in, &c.spec_out,
                    &c.scratch, &c.scratch2, &c.io_src, &c.io_trg, &c.io_den, &c.io_dl, &c.io_val, &c.stat};
  for (DevBuf* b : bufs) b->release();
  for (auto& b : c.t) b.release();
  for (auto& b : c.lvlR) b.release();
  for (auto& b : c.lvlS) b.release();
  DevTree& T = c.tree;
  DevBuf* tb[] = {&T.key, &T.leaf, &T.parent, &T.child0, &T.src_lo, &T.src_hi, &T.trg_lo, &T.trg_hi, &T.colleague,
                  &T.int_idx, &T.src_perm, &T.trg_perm, &T.src_key, &T.trg_key, &T.src_leaf, &T.trg_leaf, &T.sx,
                  &T.sy, &T.sz, &T.tx, &T.ty, &T.tz, &T.sleaf, &T.tleaf, &T.vsrc, &T.vtrg, &T.node2vsrc, &T.vtab, &T.vmask, &T.vmorton, &T.vunion, &T.vucount, &T.vlocal,
                  &T.xtrg, &T.x_off, &T.x_list, &T.p_off, &T.p_list, &T.w_off, &T.w_list, &T.p_img, &T.x_img,
                  &T.w_img, &c.dops.bc, &c.dops.d2d_f2};
  for (DevBuf* b : tb) b->release();
  if (c.events_ready)
    for (auto& e : c.ev) cudaEventDestroy(e);
  if (c.stream) cudaStreamDestroy(c.stream);
  if (c.pinned) cudaFreeHost(c.pinned);
  if (c.chk) cudaFreeHost(c.chk);
  if (c.tc5_err_host) cudaFreeHost(c.tc5_err_host);
  if (c.side) cudaStreamSynchronize(c.side);
  if (c.den_ev) cudaEventDestroy(c.den_ev);
  if (c.side) cudaStreamDestroy(c.side);
}

// Periodic boundary operator of the context (BC_Type, fmm_pts.txx:790-1232)
// in device memory: the 5x5x5-image form plus the user's operator, or the
// lattice sum.
void upload_bc(Context& c) {
  std::vector<double> M = build_bc_operator(c.kernel, c.m, c.bc_lattice != 0, c.periodic_axes);
  if (!c.bc_user.empty())
    for (size_t i = 0; i < M.size(); ++i) M[i] += c.bc_user[i];
  double* d = c.dops.bc.as<double>(M.size());
  PVFMM_CUDA_CHECK(cudaMemcpyAsync(d, M.data(), M.size() * sizeof(double), cudaMemcpyHostToDevice, c.stream));
  PVFMM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
}

void* create_context(double box_size, int n, int m, int kernel, int precision, bool float_api) {
  try {
    if (n < 1) throw std::runtime_error("max points per leaf must be positive");
    KernelInfo ki;
    if (!kernel_info(kernel, &ki)) throw std::runtime_error("unsupported PVFMMKernel value " + std::to_string(kernel));
    if (precision != 0 && precision != 1) throw std::runtime_error("unknown precision form");
    std::unique_ptr<Handle> h(new Handle);
    Context& c = h->ctx;
    c.kernel = kernel;
    c.ki = ki;
    c.m = m;
    c.ns = 6 * (m - 1) * (m - 1) + 2;
    c.max_pts = n;
    c.precision = precision;
    c.float_api = float_api;
    // Both forms use the FP64-cutoff operators: the mixed form keeps the
    // check->equivalent chain in FP64 (see eval.cu).
    // Mixed form of the Stokes kernel: FP32 cutoff in the downward
    // check -> equivalent factors.  The downward pseudo-inverse amplifies the
    // FP32 rounding of the V-list output for targets outside the downward
    // check surface (leaf corners); with the FP64 cutoff the 2M-point m=10
    // Stokes error was 2.8e-5, with the FP32 cutoff 3.7e-7.  The Laplace
    // kernels keep the FP64 cutoff (the FP32 one raised their error).
    build_operators(kernel, m, false, c.hops, precision == 1 && ki.ke == 3);
    PVFMM_CUDA_CHECK(cudaGetDevice(&c.device));
    PVFMM_CUDA_CHECK(cudaStreamCreateWithFlags(&c.stream, cudaStreamNonBlocking));
    for (auto& e : c.ev) PVFMM_CUDA_CHECK(cudaEventCreate(&e));
    c.events_ready = true;
    upload_operators(c);
    // box_size > 0: periodic boundaries (pvfmm-wrapper.cpp:397-404), with the
    // boundary operator of the reference's default build
    if (box_size > 0) {
      c.periodic = true;
      c.box_size = box_size;
      upload_bc(c);
    }
    set_last_error("");
    return h.release();
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return nullptr;
  }
}

template <class T>
int eval_device(const void* ctx_, const T* src, const T* den, const T* dl, long n_src, const T* trg, T* val,
                long n_trg, int setup, void* stream) {
  try {
    Handle* h = as_handle(ctx_);
    Context& c = h->ctx;
    PVFMM_CUDA_CHECK(cudaSetDevice(c.device));
    const bool is_f = std::is_same<T, float>::value;
    // NULL: the legacy default stream (the call then returns on completion)
    cudaStream_t user = stream ? (cudaStream_t)stream : cudaStreamLegacy;
    if (user != c.stream) {
      // order the context stream after the caller's stream
      PVFMM_CUDA_CHECK(cudaEventRecord(c.ev[11], user));
      PVFMM_CUDA_CHECK(cudaStreamWaitEvent(c.stream, c.ev[11], 0));
    }
    check_tc5_error(c);  // a wait of the previous (asynchronous) evaluation that ran out
    if (dl && c.kernel != PVFMMLaplacePotential && c.kernel != PVFMMStokesVelocity)
      throw std::runtime_error("double-layer densities (dl_den) need the LaplacePotential or StokesVelocity kernel");
    if (n_trg <= 0) return 0;
    if (n_src <= 0) {
      PVFMM_CUDA_CHECK(cudaMemsetAsync(val, 0, (size_t)n_trg * c.ki.k1 * sizeof(T), c.stream));
      PVFMM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
      return 0;
    }
    const bool alias = (src == trg) && (n_src == n_trg);
    if (setup || !c.tree.valid) {
      PVFMM_CUDA_CHECK(cudaEventRecord(c.ev[11], c.stream));
      const int w = c.layer_points ? ((den || dl) ? 1 : 0) : (den != nullptr) + (dl != nullptr);
      build_tree(c, src, n_src, trg, n_trg, is_f, w, alias);
      c.tree.layers = (den ? 1 : 0) | (dl ? 2 : 0);
    } else if (c.tree.n_src != n_src || c.tree.n_trg != n_trg) {
      throw std::runtime_error("setup=0 requires the point counts of the last setup");
    } else {
      PVFMM_CUDA_CHECK(cudaEventRecord(c.ev[11], c.stream));
    }
    evaluate(c, den, dl, is_f, val, is_f);
    if (stream && user != c.stream) {
      PVFMM_CUDA_CHECK(cudaEventRecord(c.ev[10], c.stream));
      PVFMM_CUDA_CHECK(cudaStreamWaitEvent(user, c.ev[10], 0));
    } else {
      PVFMM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
      check_tc5_error(c);
    }
    set_last_error("");
    return 0;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return 1;
  }
}

template <class T>
void eval_host(const T* src_pos, const T* sl_den, const T* dl_den, long n_src, const T* trg_pos, T* trg_val, long n_trg,
               const void* ctx_, int setup) {
  int k1 = 1;
  try {
    Handle* h = as_handle(ctx_);
    Context& c = h->ctx;
    k1 = c.ki.k1;
    PVFMM_CUDA_CHECK(cudaSetDevice(c.device));
    if (n_trg <= 0) return;
    const bool alias = (src_pos == trg_pos) && (n_src == n_trg);
    T* d_src = c.io_src.as<T>(std::max(n_src, 1L) * 3);
    T* d_den = sl_den ? c.io_den.as<T>(std::max(n_src, 1L) * c.ki.k0) : nullptr;
    T* d_dl = dl_den ? c.io_dl.as<T>(std::max(n_src, 1L) * (c.ki.k0 + 3)) : nullptr;
    T* d_trg = alias ? d_src : c.io_trg.as<T>(n_trg * 3);
    T* d_val = c.io_val.as<T>(n_trg * c.ki.k1);
    if (n_src > 0) PVFMM_CUDA_CHECK(cudaMemcpyAsync(d_src, src_pos, n_src * 3 * sizeof(T), cudaMemcpyHostToDevice, c.stream));
    if (!alias) PVFMM_CUDA_CHECK(cudaMemcpyAsync(d_trg, trg_pos, n_trg * 3 * sizeof(T), cudaMemcpyHostToDevice, c.stream));
    if (n_src > 0 && (sl_den || dl_den)) {
      // the densities are first read after the tree build: upload them on a
      // side stream meanwhile (overlaps when they are pinned host memory)
      if (!c.side) {
        PVFMM_CUDA_CHECK(cudaStreamCreateWithFlags(&c.side, cudaStreamNonBlocking));
        PVFMM_CUDA_CHECK(cudaEventCreateWithFlags(&c.den_ev, cudaEventDisableTiming));
      }
      if (sl_den)
        PVFMM_CUDA_CHECK(cudaMemcpyAsync(d_den, sl_den, n_src * c.ki.k0 * sizeof(T), cudaMemcpyHostToDevice, c.side));
      if (dl_den)
        PVFMM_CUDA_CHECK(
            cudaMemcpyAsync(d_dl, dl_den, n_src * (c.ki.k0 + 3) * sizeof(T), cudaMemcpyHostToDevice, c.side));
      PVFMM_CUDA_CHECK(cudaEventRecord(c.den_ev, c.side));
      c.den_pending = true;
    }
    if (eval_device<T>(ctx_, d_src, d_den, d_dl, n_src, d_trg, d_val, n_trg, setup, c.stream) != 0)
      throw std::runtime_error(get_last_error());
    PVFMM_CUDA_CHECK(cudaMemcpyAsync(trg_val, d_val, n_trg * c.ki.k1 * sizeof(T), cudaMemcpyDeviceToHost, c.stream));
    PVFMM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    check_tc5_error(c);
    set_last_error("");
  } catch (const std::exception& e) {
    const std::string msg = e.what();
    if (trg_val)
      for (long i = 0; i < n_trg * (long)k1; ++i) trg_val[i] = std::numeric_limits<T>::quiet_NaN();
    set_last_error(msg);
  }
}

void destroy(void** ctx) {
  if (!ctx || !ctx[0]) return;
  try {
    Handle* h = as_handle(ctx[0]);
    if (h->adjoint) destroy(&h->adjoint);
    destroy_context(h->ctx);
    h->magic = 0;
    delete h;
  } catch (const std::exception& e) {
    set_last_error(e.what());
  }
  ctx[0] = nullptr;
}

// src_val = the context's kernel with sources and targets exchanged:
// src_val[j*k1+k] = sum_i K_k(src_j - trg_i) trg_den_i.  When the two point
// sets are the same array the context's own tree serves (setup=0 reuses the
// tree of the forward evaluation); otherwise a companion context with the same
// kernel, order, leaf size, precision and tree rule holds the exchanged tree.
template <class T>
int eval_adjoint(const void* ctx, const T* src, long n_src, const T* trg, const T* trg_den, long n_trg, T* src_val,
                 int setup, void* stream) {
  try {
    Handle* h = as_handle(ctx);
    Context& c = h->ctx;
    // the lattice form takes the mean density's potential out at the targets,
    // which the role exchange does not transpose
    if (c.periodic && c.bc_lattice)
      throw std::runtime_error("the adjoint evaluation needs free space or the 5x5x5-image periodic form");
    if (src == trg && n_src == n_trg)
      return eval_device<T>(ctx, trg, trg_den, nullptr, n_trg, src, src_val, n_src, setup, stream);
    if (!h->adjoint) {
      h->adjoint = create_context(c.periodic ? c.box_size : -1.0, c.max_pts, c.m, c.kernel, c.precision,
                                  c.float_api);
      if (!h->adjoint) throw std::runtime_error(std::string("companion context: ") + get_last_error());
      Context& a = as_handle(h->adjoint)->ctx;
      a.unit_box = c.unit_box;
      if (c.periodic && (!c.bc_user.empty() || c.periodic_axes != 7)) {  // symmetric in the roles
        a.bc_user = c.bc_user;
        a.periodic_axes = c.periodic_axes;
        upload_bc(a);
      }
      setup = 1;
    }
    return eval_device<T>(h->adjoint, trg, trg_den, nullptr, n_trg, src, src_val, n_src, setup, stream);
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return 1;
  }
}

template <class T>
long copy_dev(const DevBuf& b, long count, void* out, long n, cudaStream_t s) {
  if (out && n > 0 && count > 0) {
    PVFMM_CUDA_CHECK(cudaMemcpyAsync(out, b.ptr, std::min(count, n) * sizeof(T), cudaMemcpyDeviceToHost, s));
    PVFMM_CUDA_CHECK(cudaStreamSynchronize(s));
  }
  return count;
}

}  // namespace

extern "C" {

void* PVFMMCreateContextD(double box_size, int n, int m, enum PVFMMKernel kernel, MPI_Comm comm) {
  (void)comm;
  return create_context(box_size, n, m, (int)kernel, PVFMMPrecisionPlain, false);
}
void* PVFMMCreateContextF(float box_size, int n, int m, enum PVFMMKernel kernel, MPI_Comm comm) {
  (void)comm;
  return create_context(box_size, n, m, (int)kernel, PVFMMPrecisionMixed, true);
}
void* PVFMMCreateContextDWorld(double box_size, int n, int m, enum PVFMMKernel kernel) {
  return create_context(box_size, n, m, (int)kernel, PVFMMPrecisionPlain, false);
}
void* PVFMMCreateContextFWorld(float box_size, int n, int m, enum PVFMMKernel kernel) {
  return create_context(box_size, n, m, (int)kernel, PVFMMPrecisionMixed, true);
}
void* PVFMMCreateContextExD(double box_size, int n, int m, enum PVFMMKernel kernel, int precision) {
  return create_context(box_size, n, m, (int)kernel, precision, false);
}

int PVFMMSetPeriodicAxes(void* ctx, int axes) {
  try {
    Context& c = as_handle(ctx)->ctx;
    PVFMM_CUDA_CHECK(cudaSetDevice(c.device));
    if (!c.periodic) throw std::runtime_error("the context has free-space boundaries (box_size <= 0)");
    if (axes != 1 && axes != 3 && axes != 7) throw std::runtime_error("periodic axes must be 1 (x), 3 (xy) or 7 (xyz)");
    PVFMM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    const int old = c.periodic_axes;
    c.periodic_axes = axes;
    try {
      upload_bc(c);
    } catch (...) {
      c.periodic_axes = old;
      throw;
    }
    if (axes != old) c.tree.valid = false;  // the tree's balance and lists depend on the axes
    Handle* h = as_handle(ctx);
    if (h->adjoint) destroy(&h->adjoint);
    set_last_error("");
    return 0;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return -1;
  }
}

int PVFMMSetPeriodicBC(void* ctx, int lattice, const double* m2c) {
  try {
    Context& c = as_handle(ctx)->ctx;
    PVFMM_CUDA_CHECK(cudaSetDevice(c.device));
    if (!c.periodic) throw std::runtime_error("the context has free-space boundaries (box_size <= 0)");
    if (lattice != 0 && lattice != 1) throw std::runtime_error("lattice must be 0 or 1");
    if (lattice && m2c) throw std::runtime_error("a user operator adds to the 5x5x5-image form only (lattice 0)");
    if (lattice && !lattice_bc_supported(c.kernel))
      throw std::runtime_error("the periodic lattice sum needs the LaplacePotential, LaplaceGradient or "
                               "StokesVelocity kernel");
    PVFMM_CUDA_CHECK(cudaStreamSynchronize(c.stream));  // no evaluation reads the operator while it changes
    const int kin = c.hops.kin, kout = c.hops.kout;
    std::vector<double> user;
    if (m2c) user.assign(m2c, m2c + (size_t)c.ns * kin * c.ns * kout);
    const int old_lattice = c.bc_lattice;
    std::vector<double> old_user = c.bc_user;
    c.bc_lattice = lattice;
    c.bc_user = std::move(user);
    try {
      upload_bc(c);
    } catch (...) {
      c.bc_lattice = old_lattice;
      c.bc_user = std::move(old_user);
      throw;
    }
    Handle* h = as_handle(ctx);
    if (h->adjoint) destroy(&h->adjoint);  // rebuilt with the new operator on its next use
    set_last_error("");
    return 0;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return -1;
  }
}

void PVFMMEvalD(const double* src_pos, const double* sl_den, const double* dl_den, long n_src, const double* trg_pos,
                double* trg_val, long n_trg, const void* ctx, int setup) {
  eval_host<double>(src_pos, sl_den, dl_den, n_src, trg_pos, trg_val, n_trg, ctx, setup);
}
void PVFMMEvalF(const float* src_pos, const float* sl_den, const float* dl_den, long n_src, const float* trg_pos,
                float* trg_val, long n_trg, const void* ctx, int setup) {
  eval_host<float>(src_pos, sl_den, dl_den, n_src, trg_pos, trg_val, n_trg, ctx, setup);
}

int PVFMMEvalLayersDeviceD(const void* ctx, const double* src_pos, const double* sl_den, const double* dl_den,
                           long n_src, const double* trg_pos, double* trg_val, long n_trg, int setup, void* stream) {
  return eval_device<double>(ctx, src_pos, sl_den, dl_den, n_src, trg_pos, trg_val, n_trg, setup, stream);
}
int PVFMMEvalLayersDeviceF(const void* ctx, const float* src_pos, const float* sl_den, const float* dl_den,
                           long n_src, const float* trg_pos, float* trg_val, long n_trg, int setup, void* stream) {
  return eval_device<float>(ctx, src_pos, sl_den, dl_den, n_src, trg_pos, trg_val, n_trg, setup, stream);
}
int PVFMMEvalDeviceD(const void* ctx, const double* src_pos, const double* sl_den, long n_src, const double* trg_pos,
                     double* trg_val, long n_trg, int setup, void* stream) {
  return eval_device<double>(ctx, src_pos, sl_den, nullptr, n_src, trg_pos, trg_val, n_trg, setup, stream);
}
int PVFMMEvalDeviceF(const void* ctx, const float* src_pos, const float* sl_den, long n_src, const float* trg_pos,
                     float* trg_val, long n_trg, int setup, void* stream) {
  return eval_device<float>(ctx, src_pos, sl_den, nullptr, n_src, trg_pos, trg_val, n_trg, setup, stream);
}

int PVFMMEvalAdjointDeviceD(const void* ctx, const double* src_pos, long n_src, const double* trg_pos,
                            const double* trg_den, long n_trg, double* src_val, int setup, void* stream) {
  return eval_adjoint<double>(ctx, src_pos, n_src, trg_pos, trg_den, n_trg, src_val, setup, stream);
}
int PVFMMEvalAdjointDeviceF(const void* ctx, const float* src_pos, long n_src, const float* trg_pos,
                            const float* trg_den, long n_trg, float* src_val, int setup, void* stream) {
  return eval_adjoint<float>(ctx, src_pos, n_src, trg_pos, trg_den, n_trg, src_val, setup, stream);
}

int PVFMMSetLayerPoints(void* ctx, int on) {
  try {
    Handle* h = as_handle(ctx);
    h->ctx.layer_points = on != 0;
    h->ctx.tree.valid = false;
    set_last_error("");
    return 0;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return 1;
  }
}

int PVFMMSetUnitBox(void* ctx, int on) {
  try {
    Handle* h = as_handle(ctx);
    h->ctx.unit_box = on != 0;
    h->ctx.tree.valid = false;
    set_last_error("");
    return 0;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return 1;
  }
}

void PVFMMDestroyContextD(void** ctx) { destroy(ctx); }
void PVFMMDestroyContextF(void** ctx) { destroy(ctx); }

// Fortran bindings (reference src/pvfmm-wrapper.cpp:831-875): every argument
// by reference, the communicator as a Fortran handle (single rank here).
void pvfmmcreatecontextd_(void** ctx, double* box_size, int32_t* n, int32_t* m, int32_t* kernel, int32_t* fcomm) {
  (void)fcomm;
  *ctx = PVFMMCreateContextD(*box_size, *n, *m, (enum PVFMMKernel) * kernel, MPI_COMM_WORLD);
}
void pvfmmcreatecontextf_(void** ctx, float* box_size, int32_t* n, int32_t* m, int32_t* kernel, int32_t* fcomm) {
  (void)fcomm;
  *ctx = PVFMMCreateContextF(*box_size, *n, *m, (enum PVFMMKernel) * kernel, MPI_COMM_WORLD);
}
void pvfmmevald_(const double* src_pos, const double* sl_den, int64_t* n_src, const double* trg_pos, double* trg_val,
                 int64_t* n_trg, void** ctx, int32_t* setup) {
  PVFMMEvalD(src_pos, sl_den, nullptr, (long)*n_src, trg_pos, trg_val, (long)*n_trg, *ctx, *setup);
}
void pvfmmevalf_(const float* src_pos, const float* sl_den, int64_t* n_src, const float* trg_pos, float* trg_val,
                 int64_t* n_trg, void** ctx, int32_t* setup) {
  PVFMMEvalF(src_pos, sl_den, nullptr, (long)*n_src, trg_pos, trg_val, (long)*n_trg, *ctx, *setup);
}
void pvfmmdestroycontextd_(void** ctx) { PVFMMDestroyContextD(ctx); }
void pvfmmdestroycontextf_(void** ctx) { PVFMMDestroyContextF(ctx); }

const char* PVFMMGetLastError(void) { return get_last_error(); }

long PVFMMGetLaunchCount(const void* ctx) {
  try {
    return as_handle(ctx)->ctx.n_launch;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return -1;
  }
}

int PVFMMGetStageTimes(const void* ctx, double* ms, int n) {
  try {
    Handle* h = as_handle(ctx);
    Context& c = h->ctx;
    PVFMM_CUDA_CHECK(cudaSetDevice(c.device));
    PVFMM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    float t[12] = {0};
    auto el = [&](int a, int b) {
      float x = 0;
      if (cudaEventElapsedTime(&x, c.ev[a], c.ev[b]) != cudaSuccess) x = 0;
      return x;
    };
    t[0] = el(11, 0);
    t[1] = el(1, 2);
    t[2] = el(2, 3);
    t[3] = el(3, 4);
    t[4] = el(4, 5);
    t[5] = el(5, 6);
    t[6] = el(6, 7);
    t[7] = el(7, 8);
    t[8] = el(8, 9);
    t[9] = el(11, 10);
    t[10] = el(12, 9);
    t[11] = el(8, 12);
    const int k = std::min(n, 12);
    for (int i = 0; i < k; ++i) ms[i] = t[i];
    return k;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return 0;
  }
}

long PVFMMGetTreeData(const void* ctx, int what, void* out, long n) {
  try {
    Handle* h = as_handle(ctx);
    Context& c = h->ctx;
    DevTree& T = c.tree;
    PVFMM_CUDA_CHECK(cudaSetDevice(c.device));
    PVFMM_CUDA_CHECK(cudaStreamSynchronize(c.stream));
    if (!T.valid) throw std::runtime_error("no tree: call an evaluation with setup=1 first");
    const long N = T.n_nodes;
    const int dim = c.ns * c.ki.ke;
    auto s = c.stream;
    switch (what) {
      case 0:
        if (out && n > 0) *(long long*)out = N;
        return 1;
      case 1:
        if (out && n > 0) *(long long*)out = T.depth;
        return 1;
      case 2: {
        std::vector<MKey> k(N);
        PVFMM_CUDA_CHECK(cudaMemcpy(k.data(), T.key.ptr, N * sizeof(MKey), cudaMemcpyDeviceToHost));
        if (out)
          for (long i = 0; i < N && 4 * i + 3 < n; ++i) {
            unsigned int X, Y, Z, d;
            decode_key(k[i], X, Y, Z, d);
            long long* o = (long long*)out + 4 * i;
            o[0] = X;
            o[1] = Y;
            o[2] = Z;
            o[3] = d;
          }
        return 4 * N;
      }
      case 3: {
        std::vector<unsigned char> l(N);
        PVFMM_CUDA_CHECK(cudaMemcpy(l.data(), T.leaf.ptr, N, cudaMemcpyDeviceToHost));
        if (out)
          for (long i = 0; i < N && i < n; ++i) ((long long*)out)[i] = l[i];
        return N;
      }
      case 4:
      case 5: {
        std::vector<int> lo(N), hi(N);
        PVFMM_CUDA_CHECK(cudaMemcpy(lo.data(), (what == 4 ? T.src_lo : T.trg_lo).ptr, N * sizeof(int), cudaMemcpyDeviceToHost));
        PVFMM_CUDA_CHECK(cudaMemcpy(hi.data(), (what == 4 ? T.src_hi : T.trg_hi).ptr, N * sizeof(int), cudaMemcpyDeviceToHost));
        if (out)
          for (long i = 0; i < N && 2 * i + 1 < n; ++i) {
            ((long long*)out)[2 * i] = lo[i];
            ((long long*)out)[2 * i + 1] = hi[i];
          }
        return 2 * N;
      }
      case 6: {
        std::vector<int> p(N);
        PVFMM_CUDA_CHECK(cudaMemcpy(p.data(), T.parent.ptr, N * sizeof(int), cudaMemcpyDeviceToHost));
        if (out)
          for (long i = 0; i < N && i < n; ++i) ((long long*)out)[i] = p[i];
        return N;
      }
      case 7:
      case 8: {
        const long cnt = N * dim;
        if (!out) return cnt;
        const DevBuf& b = what == 7 ? c.ue : c.dc;
        const long k = std::min(cnt, n);
        if (c.precision == 0) {
          PVFMM_CUDA_CHECK(cudaMemcpy(out, b.ptr, k * sizeof(double), cudaMemcpyDeviceToHost));
        } else {
          std::vector<float> f(k);
          PVFMM_CUDA_CHECK(cudaMemcpy(f.data(), b.ptr, k * sizeof(float), cudaMemcpyDeviceToHost));
          for (long i = 0; i < k; ++i) ((double*)out)[i] = f[i];
        }
        return cnt;
      }
      case 9:
      case 10: {
        const long cnt = what == 9 ? T.n_src : T.n_trg;
        std::vector<int> p(cnt);
        PVFMM_CUDA_CHECK(cudaMemcpy(p.data(), (what == 9 ? T.src_perm : T.trg_perm).ptr, cnt * sizeof(int), cudaMemcpyDeviceToHost));
        if (out)
          for (long i = 0; i < cnt && i < n; ++i) ((long long*)out)[i] = p[i];
        return cnt;
      }
      case 11: {
        // [n_nodes, depth, n_sleaf, n_tleaf, n_vsrc, n_vtrg, n_xtrg, p2p list entries, x entries,
        //  w entries, p2p pairs, x pairs (sources x check points), w pairs (surface x targets),
        //  d2t pairs, s2u pairs, n_leaves, n_src, n_trg, V-list parent pairs]
        std::vector<int> slo(N), shi(N), tlo(N), thi(N), po(N + 1), xo(N + 1), wo(N + 1);
        std::vector<unsigned char> lf(N);
        PVFMM_CUDA_CHECK(cudaMemcpy(slo.data(), T.src_lo.ptr, N * sizeof(int), cudaMemcpyDeviceToHost));
        PVFMM_CUDA_CHECK(cudaMemcpy(shi.data(), T.src_hi.ptr, N * sizeof(int), cudaMemcpyDeviceToHost));
        PVFMM_CUDA_CHECK(cudaMemcpy(tlo.data(), T.trg_lo.ptr, N * sizeof(int), cudaMemcpyDeviceToHost));
        PVFMM_CUDA_CHECK(cudaMemcpy(thi.data(), T.trg_hi.ptr, N * sizeof(int), cudaMemcpyDeviceToHost));
        PVFMM_CUDA_CHECK(cudaMemcpy(po.data(), T.p_off.ptr, (N + 1) * sizeof(int), cudaMemcpyDeviceToHost));
        PVFMM_CUDA_CHECK(cudaMemcpy(xo.data(), T.x_off.ptr, (N + 1) * sizeof(int), cudaMemcpyDeviceToHost));
        PVFMM_CUDA_CHECK(cudaMemcpy(wo.data(), T.w_off.ptr, (N + 1) * sizeof(int), cudaMemcpyDeviceToHost));
        PVFMM_CUDA_CHECK(cudaMemcpy(lf.data(), T.leaf.ptr, N, cudaMemcpyDeviceToHost));
        std::vector<int> pl(std::max(T.n_p2p, 1L)), xl(std::max(T.n_x, 1L));
        if (T.n_p2p) PVFMM_CUDA_CHECK(cudaMemcpy(pl.data(), T.p_list.ptr, T.n_p2p * sizeof(int), cudaMemcpyDeviceToHost));
        if (T.n_x) PVFMM_CUDA_CHECK(cudaMemcpy(xl.data(), T.x_list.ptr, T.n_x * sizeof(int), cudaMemcpyDeviceToHost));
        double p2p = 0, xp = 0, wp = 0, d2t = 0, s2u = 0, nleaf = 0;
        for (long t = 0; t < N; ++t) {
          const double nt = thi[t] - tlo[t];
          nleaf += lf[t];
          for (int q = po[t]; q < po[t + 1]; ++q) p2p += nt * (shi[pl[q]] - slo[pl[q]]);
          for (int q = xo[t]; q < xo[t + 1]; ++q) xp += (double)c.ns * (shi[xl[q]] - slo[xl[q]]);
          wp += nt * (double)c.ns * (wo[t + 1] - wo[t]);
          if (lf[t] && nt > 0) d2t += nt * c.ns;
          if (lf[t]) s2u += (double)c.ns * (shi[t] - slo[t]);
        }
        // V-list (target parent, offset) pairs with a source parent
        double vpairs = 0;
        if (T.n_vtrg > 0) {
          std::vector<int> vt((size_t)T.n_vtrg * 26);
          PVFMM_CUDA_CHECK(cudaMemcpy(vt.data(), T.vtab.ptr, vt.size() * sizeof(int), cudaMemcpyDeviceToHost));
          for (int q : vt) vpairs += q >= 0;
        }
        const double v[19] = {(double)N, (double)T.depth, (double)T.n_sleaf, (double)T.n_tleaf, (double)T.n_vsrc,
                              (double)T.n_vtrg, (double)T.n_xtrg, (double)T.n_p2p, (double)T.n_x, (double)T.n_w,
                              p2p, xp, wp, d2t, s2u, nleaf, (double)T.n_src, (double)T.n_trg, vpairs};
        if (out)
          for (long i = 0; i < 19 && i < n; ++i) ((double*)out)[i] = v[i];
        return 19;
      }
      default:
        throw std::runtime_error("unknown tree data selector");
    }
    (void)s;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return -1;
  }
}

long PVFMMPrecompOperator(enum PVFMMKernel kernel, int m, int precision, int which, double* out, long n) {
  static std::mutex mu;
  static HostOperators ops;
  static std::vector<double> bc;
  static int bc_kernel = -1, bc_m = 0, bc_which = 0;
  std::lock_guard<std::mutex> lock(mu);
  try {
    if (which == 9 || which == 10) {  // periodic boundary operator: 5x5x5 images / lattice sum
      if (bc_kernel != (int)kernel || bc_m != m || bc_which != which) {
        bc_kernel = -1;
        bc = build_bc_operator((int)kernel, m, which == 10);
        bc_kernel = (int)kernel;
        bc_m = m;
        bc_which = which;
      }
      if (out && n > 0) std::memcpy(out, bc.data(), sizeof(double) * std::min<long>(n, (long)bc.size()));
      return (long)bc.size();
    }
    if (ops.kernel != (int)kernel || ops.m != m || ops.mixed != (precision == 1))
      build_operators((int)kernel, m, precision == 1, ops);
    const std::vector<double>* v = nullptr;
    switch (which) {
      case 0: v = &ops.uc2ue0; break;
      case 1: v = &ops.uc2ue1; break;
      case 2: v = &ops.dc2de0; break;
      case 3: v = &ops.dc2de1; break;
      case 4: v = &ops.u2u; break;
      case 5: v = &ops.d2d; break;
      case 6: v = &ops.usurf; break;
      case 7: v = &ops.vop; break;
      case 8: v = &ops.ue_proj; break;
      default: throw std::runtime_error("unknown operator selector");
    }
    if (out && n > 0) std::memcpy(out, v->data(), sizeof(double) * std::min<long>(n, (long)v->size()));
    return (long)v->size();
  } catch (const std::exception& e) {
    ops.kernel = -1;
    set_last_error(e.what());
    return -1;
  }
}

}  // extern "C"
