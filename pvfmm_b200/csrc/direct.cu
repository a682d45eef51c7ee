// Direct kernel evaluation on the device: the GPU counterpart of the
// reference's Kernel<T>::ker_poten (include/kernel.hpp:40-41,
// GenericKernel::Eval in include/kernel.txx:1137-1265): k_out += sum over
// all sources of K(trg - src) den, r == 0 excluded.
//
// Work split: targets in tiles of 128 (one thread each), sources in S chunks,
// one block per (target tile, source chunk).  Each block writes FP64 partial
// sums to scratch[chunk][target][k]; a second kernel adds the S partials of
// every target in chunk order (deterministic) into k_out.  S is chosen so
// that there are about four blocks per SM.
#include <cuda_runtime.h>

#include <algorithm>
#include <mutex>
#include <stdexcept>
#include <string>

#include "../../include/pvfmm.h"
#include "fmm_device.cuh"
#include "fmm_host.hpp"

namespace pvfmm_b200 {
namespace {

constexpr int kDT = 128;

template <int Ker>
__global__ void __launch_bounds__(kDT) direct_partial_kernel(const double* __restrict__ src,
                                                             const double* __restrict__ den, long n_src,
                                                             const double* __restrict__ trg, long n_trg, int n_chunks,
                                                             double* __restrict__ partial) {
  constexpr int KS = KerDims<Ker>::KS, KT = KerDims<Ker>::KT;
  __shared__ double sx[kDT], sy[kDT], sz[kDT], sf[KS][kDT];
  const long t = (long)blockIdx.x * kDT + threadIdx.x;
  const int chunk = blockIdx.y;
  const long per = (n_src + n_chunks - 1) / n_chunks;
  const long lo = chunk * per, hi = min(n_src, lo + per);
  double px = 0, py = 0, pz = 0;
  if (t < n_trg) {
    px = trg[t * 3 + 0];
    py = trg[t * 3 + 1];
    pz = trg[t * 3 + 2];
  }
  double u[KT];
#pragma unroll
  for (int k = 0; k < KT; ++k) u[k] = 0;
  for (long s0 = lo; s0 < hi; s0 += kDT) {
    const int n = (int)min((long)kDT, hi - s0);
    __syncthreads();
    if (threadIdx.x < n) {
      const long s = s0 + threadIdx.x;
      sx[threadIdx.x] = src[s * 3 + 0];
      sy[threadIdx.x] = src[s * 3 + 1];
      sz[threadIdx.x] = src[s * 3 + 2];
#pragma unroll
      for (int i = 0; i < KS; ++i) sf[i][threadIdx.x] = den[s * KS + i];
    }
    __syncthreads();
    if (t < n_trg)
      for (int j = 0; j < n; ++j) {
        double f[KS];
#pragma unroll
        for (int i = 0; i < KS; ++i) f[i] = sf[i][j];
        ker_eval<Ker, double>(px - sx[j], py - sy[j], pz - sz[j], f, u);
      }
  }
  if (t < n_trg)
#pragma unroll
    for (int k = 0; k < KT; ++k) partial[((long)chunk * n_trg + t) * KT + k] = u[k];
}

template <int KT>
__global__ void direct_reduce_kernel(const double* __restrict__ partial, long n_trg, int n_chunks, double scale,
                                     double* __restrict__ out) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n_trg * KT) return;
  double s = 0;
  for (int c = 0; c < n_chunks; ++c) s += partial[(long)c * n_trg * KT + i];
  out[i] += s * scale;
}

int ker_type(int kernel) {
  switch (kernel) {
    case kLaplacePot: return kKerLaplace;
    case kLaplaceGrad: return kKerLaplaceGrad;
    case kStokesVel: return kKerStokes;
    case kLaplacePotGrad: return kKerLaplacePG;
    case kStokesPress: return kKerStokesPress;
    case kStokesVelGrad: return kKerStokesGrad;
    case kBiotSavart: return kKerBiotSavart;
    default: throw std::runtime_error("unsupported PVFMMKernel value " + std::to_string(kernel));
  }
}

int sm_count() {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return 148;
  return n;
}

// Number of source chunks: about 4 blocks per SM, at most one chunk per 512
// sources, at most `cap` partial rows.
int choose_chunks(long n_src, long n_trg, long cap_chunks) {
  const long tiles = (n_trg + kDT - 1) / kDT;
  long S = std::max(1L, (4L * sm_count() + tiles - 1) / tiles);
  S = std::min(S, std::max(1L, n_src / 512));
  S = std::min(S, cap_chunks);
  return (int)std::max(1L, S);
}

}  // namespace

template <int Ker>
void direct_eval_t(const double* src, const double* den, long n_src, const double* trg, double* out, long n_trg,
                   int n_chunks, double* partial, cudaStream_t s) {
  constexpr int KT = KerDims<Ker>::KT;
  dim3 grid((unsigned)((n_trg + kDT - 1) / kDT), (unsigned)n_chunks);
  const unsigned rb = (unsigned)((n_trg * KT + 255) / 256);
  direct_partial_kernel<Ker><<<grid, kDT, 0, s>>>(src, den, n_src, trg, n_trg, n_chunks, partial);
  direct_reduce_kernel<KT><<<rb, 256, 0, s>>>(partial, n_trg, n_chunks, ker_scale(Ker), out);
}

// Launches the two kernels with `partial` holding n_chunks * n_trg * KT doubles.
void direct_eval(int kernel, const double* src, const double* den, long n_src, const double* trg, double* out, long n_trg,
                 int n_chunks, double* partial, cudaStream_t s) {
  switch (ker_type(kernel)) {
    case kKerLaplace: direct_eval_t<kKerLaplace>(src, den, n_src, trg, out, n_trg, n_chunks, partial, s); break;
    case kKerLaplaceGrad: direct_eval_t<kKerLaplaceGrad>(src, den, n_src, trg, out, n_trg, n_chunks, partial, s); break;
    case kKerStokes: direct_eval_t<kKerStokes>(src, den, n_src, trg, out, n_trg, n_chunks, partial, s); break;
    case kKerStokesPress: direct_eval_t<kKerStokesPress>(src, den, n_src, trg, out, n_trg, n_chunks, partial, s); break;
    case kKerStokesGrad: direct_eval_t<kKerStokesGrad>(src, den, n_src, trg, out, n_trg, n_chunks, partial, s); break;
    case kKerBiotSavart: direct_eval_t<kKerBiotSavart>(src, den, n_src, trg, out, n_trg, n_chunks, partial, s); break;
    default: direct_eval_t<kKerLaplacePG>(src, den, n_src, trg, out, n_trg, n_chunks, partial, s); break;
  }
  PVFMM_CUDA_CHECK(cudaGetLastError());
}

int direct_chunks(long n_src, long n_trg, long cap_chunks) { return choose_chunks(n_src, n_trg, cap_chunks); }

}  // namespace pvfmm_b200

using namespace pvfmm_b200;

extern "C" int PVFMMKernelEvalDeviceD(enum PVFMMKernel kernel, const double* src_pos, const double* den, long n_src,
                                      const double* trg_pos, double* trg_val, long n_trg, void* stream) {
  try {
    KernelInfo ki;
    if (!kernel_info((int)kernel, &ki)) throw std::runtime_error("unsupported PVFMMKernel value");
    if (n_trg <= 0 || n_src <= 0) {
      set_last_error("");
      return 0;
    }
    cudaStream_t s = (cudaStream_t)stream;
    const int S = choose_chunks(n_src, n_trg, 1L << 20);
    double* partial = nullptr;
    PVFMM_CUDA_CHECK(cudaMallocAsync((void**)&partial, (size_t)S * n_trg * ki.k1 * sizeof(double), s));
    direct_eval((int)kernel, src_pos, den, n_src, trg_pos, trg_val, n_trg, S, partial, s);
    PVFMM_CUDA_CHECK(cudaFreeAsync(partial, s));
    set_last_error("");
    return 0;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return 1;
  }
}

// Host-pointer form (the calling convention of Kernel<T>::ker_poten): copies
// the arrays to the current device, runs the same two kernels on a private
// stream and copies the accumulated values back.
extern "C" int PVFMMKernelEvalD(enum PVFMMKernel kernel, const double* src_pos, const double* den, long n_src,
                                const double* trg_pos, double* trg_val, long n_trg) {
  cudaStream_t s = nullptr;
  double* buf = nullptr;
  try {
    KernelInfo ki;
    if (!kernel_info((int)kernel, &ki)) throw std::runtime_error("unsupported PVFMMKernel value");
    if (n_trg <= 0 || n_src <= 0) {
      set_last_error("");
      return 0;
    }
    PVFMM_CUDA_CHECK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking));
    const int S = choose_chunks(n_src, n_trg, 1L << 20);
    const size_t n_s3 = (size_t)n_src * 3, n_sd = (size_t)n_src * ki.k0, n_t3 = (size_t)n_trg * 3,
                 n_tv = (size_t)n_trg * ki.k1, n_p = (size_t)S * n_trg * ki.k1;
    PVFMM_CUDA_CHECK(cudaMallocAsync((void**)&buf, (n_s3 + n_sd + n_t3 + n_tv + n_p) * sizeof(double), s));
    double *d_src = buf, *d_den = d_src + n_s3, *d_trg = d_den + n_sd, *d_val = d_trg + n_t3, *d_part = d_val + n_tv;
    PVFMM_CUDA_CHECK(cudaMemcpyAsync(d_src, src_pos, n_s3 * sizeof(double), cudaMemcpyHostToDevice, s));
    PVFMM_CUDA_CHECK(cudaMemcpyAsync(d_den, den, n_sd * sizeof(double), cudaMemcpyHostToDevice, s));
    PVFMM_CUDA_CHECK(cudaMemcpyAsync(d_trg, trg_pos, n_t3 * sizeof(double), cudaMemcpyHostToDevice, s));
    PVFMM_CUDA_CHECK(cudaMemcpyAsync(d_val, trg_val, n_tv * sizeof(double), cudaMemcpyHostToDevice, s));
    direct_eval((int)kernel, d_src, d_den, n_src, d_trg, d_val, n_trg, S, d_part, s);
    PVFMM_CUDA_CHECK(cudaMemcpyAsync(trg_val, d_val, n_tv * sizeof(double), cudaMemcpyDeviceToHost, s));
    PVFMM_CUDA_CHECK(cudaFreeAsync(buf, s));
    buf = nullptr;
    PVFMM_CUDA_CHECK(cudaStreamSynchronize(s));
    PVFMM_CUDA_CHECK(cudaStreamDestroy(s));
    set_last_error("");
    return 0;
  } catch (const std::exception& e) {
    if (s) {
      if (buf) cudaFreeAsync(buf, s);
      cudaStreamSynchronize(s);
      cudaStreamDestroy(s);
    }
    set_last_error(e.what());
    return 1;
  }
}

// ---------------------------------------------------------------------------
// Allocation-free variant of the direct evaluation.
//
// Some callers cannot allocate device memory at the point where they need a
// direct sum: code that runs inside a host framework which owns the whole
// device memory pool (a cudaMalloc there would go around its allocator or
// fail once the pool has reserved the memory), and latency-critical loops
// that must not pay for an allocation, which can synchronize the device.
// For them the partial sums live in a fixed array in this library's device
// image: 1 Mi doubles (8 MiB), held by every GPU that loads the library until
// the process exits.
//
// The array's host-side name is only a stand-in for the symbol, not a device
// address, so the first call on each device looks up the real address with
// cudaGetSymbolAddress (with that device current) and caches it for the life
// of the process; make that first call before any stream capture.  The cached
// address belongs to the device's primary context: after cudaDeviceReset it is
// stale, and this entry point must not be called again in that process.  Every call shares the array and
// leaves its partial sums in it; nothing in it needs to start at zero, because
// each call writes every entry it later reads.  Calls whose work overlaps on
// the GPU (concurrent streams, or other host threads) race on the array and
// must be serialised by the caller.
// ---------------------------------------------------------------------------
namespace {
constexpr long kNoAllocScratchDoubles = 1L << 20;
__device__ __align__(256) double g_noalloc_scratch[kNoAllocScratchDoubles];
std::mutex g_noalloc_mutex;
double* g_noalloc_addr[128] = {nullptr};

double* noalloc_scratch_address() {
  int dev = 0;
  PVFMM_CUDA_CHECK(cudaGetDevice(&dev));
  if (dev < 0 || dev >= 128) throw std::runtime_error("device index out of range for the fixed scratch table");
  std::lock_guard<std::mutex> lock(g_noalloc_mutex);
  if (!g_noalloc_addr[dev]) {
    void* p = nullptr;
    const cudaError_t err = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (err != cudaSuccess)
      throw std::runtime_error(std::string("cudaGetSymbolAddress of the fixed scratch failed: ") + cudaGetErrorString(err));
    g_noalloc_addr[dev] = (double*)p;
  }
  return g_noalloc_addr[dev];
}
}  // namespace

extern "C" int PVFMMKernelEvalDeviceNoAllocD(enum PVFMMKernel kernel, const double* src_pos, const double* den,
                                             long n_src, const double* trg_pos, double* trg_val, long n_trg,
                                             void* stream) {
  try {
    KernelInfo ki;
    if (!kernel_info((int)kernel, &ki)) throw std::runtime_error("unsupported PVFMMKernel value");
    if (n_trg <= 0 || n_src <= 0) {
      set_last_error("");
      return 0;
    }
    const long rows = n_trg * ki.k1;
    if (rows > kNoAllocScratchDoubles)
      throw std::runtime_error("n_trg * k1 = " + std::to_string(rows) + " exceeds the fixed scratch of " +
                               std::to_string(kNoAllocScratchDoubles) +
                               " doubles of the allocation-free entry point; split the targets");
    double* scratch = noalloc_scratch_address();
    const int S = choose_chunks(n_src, n_trg, kNoAllocScratchDoubles / rows);
    direct_eval((int)kernel, src_pos, den, n_src, trg_pos, trg_val, n_trg, S, scratch, (cudaStream_t)stream);
    set_last_error("");
    return 0;
  } catch (const std::exception& e) {
    set_last_error(e.what());
    return 1;
  }
}
