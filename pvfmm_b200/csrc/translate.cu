// FP64 translation products of the FMM on the FP64 tensor cores
// (mma.sync m8n8k4 .f64, the only FP64 MMA of sm_100): the check ->
// equivalent pseudo-inverse products of S2U and D2T, U2U and D2D
// (reference: the per-interaction-block GEMMs of FMM_Pts::EvalList,
// include/fmm_pts.txx:2017-2271, and the surface GEMMs of EvalListPts,
// :4246-4302 and :4390-4426).
//
// Every translation here has the same shape: a tall matrix of node rows
// (one row = the ns*ke values of one node's surface) times one small operator
// shared by all rows,
//   C[crow(i)][:] (+)= s(i) * A[arow(i)][:] * B,
// where the rows of A may be gathered through an index list (the nodes of a
// level, the target leaves), the rows of C may be scattered through one, and
// s(i) is 1 or the level factor 2^-depth of the node.  B (at most
// 8*ns*ke x ns*ke) stays in L2 across the whole launch; the rows of A are
// read once per column tile.
//
// Tiling: a block computes a 128 x 64 tile of C with 8 warps (4 x 2), each
// warp a 32 x 32 tile = 4 x 4 MMA tiles of 8 x 8, FP64 accumulators in
// registers (each A and B fragment feeds four MMAs).
// K advances in steps of 16; the A and B tiles of the next step are copied
// into shared memory with 16-byte cp.async while the current step runs.
// Row lengths are even (ns = 6(m-1)^2+2), so every row of A, B and C starts
// on a 16-byte boundary.
#include <algorithm>

#include "fmm_context.cuh"

namespace pvfmm_b200 {
namespace {

constexpr int kBM = 128, kBN = 64, kBK = 16;
constexpr int kAStride = kBK + 4;  // doubles per A row in shared memory
constexpr int kBStride = kBN + 4;  // doubles per B row in shared memory (B fragment loads conflict-free)
constexpr int kThreadsG = 256;
constexpr int kSmemG = (int)sizeof(double) * (2 * kBM * kAStride + 2 * kBK * kBStride) + (int)sizeof(long) * kBM;

__device__ __forceinline__ void cp16(void* smem, const void* gmem, bool valid) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(s), "l"(gmem), "r"(valid ? 16 : 0));
}
__device__ __forceinline__ void cp_commit() { asm volatile("cp.async.commit_group;\n" ::); }
template <int N>
__device__ __forceinline__ void cp_wait() {
  asm volatile("cp.async.wait_group %0;\n" ::"n"(N));
}


struct RowMap {
  const int* rows;  // nullptr: identity
  __device__ __forceinline__ long operator()(long i) const { return rows ? (long)rows[i] : i; }
};

__global__ void __launch_bounds__(kThreadsG, 2)
    translate_gemm_kernel(int M, int N, int K, const double* __restrict__ A, long lda, const int* __restrict__ arows,
                          const double* __restrict__ B, long ldb, double* __restrict__ C, long ldc,
                          const int* __restrict__ crows, const MKey* __restrict__ keys, int deg, int accumulate,
                          long m_base, int kchunk, double* __restrict__ partial) {
  extern __shared__ __align__(16) double tsm[];
  double(*As)[kBM * kAStride] = reinterpret_cast<double(*)[kBM * kAStride]>(tsm);
  double(*Bs)[kBK * kBStride] = reinterpret_cast<double(*)[kBK * kBStride]>(tsm + 2 * kBM * kAStride);
  long* arow_s = reinterpret_cast<long*>(tsm + 2 * kBM * kAStride + 2 * kBK * kBStride);
  const int tid = threadIdx.x, warp = tid >> 5, lane = tid & 31;
  const int g = lane >> 2, t = lane & 3;
  const int wm = warp >> 1, wn = warp & 1;  // warp tile (32 rows) x (32 cols)
  const long m0 = m_base + (long)blockIdx.y * kBM;
  const int n0 = blockIdx.x * kBN;
  const RowMap amap{arows};
  // split K: this block sums k in [kbeg, kend) (the whole of K without a split)
  const int kbeg = blockIdx.z * kchunk, kend = min(K, kbeg + kchunk);
  if (tid < kBM) arow_s[tid] = m0 + tid < M ? amap(m0 + tid) : -1;
  __syncthreads();
  // copy plan: A tile 128 rows x 16 doubles = 1024 chunks of 16 B, 4 per
  // thread; B tile 16 rows x 64 doubles = 512 chunks, 2 per thread
  auto issue = [&](int k0, int buf) {
#pragma unroll
    for (int u = 0; u < 4; ++u) {
      const int c = tid + u * kThreadsG;
      const int r = c >> 3, kc = (c & 7) * 2;  // row, first double of the chunk
      const long ar = arow_s[r];
      const bool v = ar >= 0 && k0 + kc < kend;
      const double* src = v ? A + ar * lda + k0 + kc : A;
      cp16(&As[buf][r * kAStride + kc], src, v);
    }
#pragma unroll
    for (int u = 0; u < 2; ++u) {
      const int c = tid + u * kThreadsG;
      const int r = c >> 5, nc = (c & 31) * 2;
      const bool v = k0 + r < kend && n0 + nc < N;
      const double* src = v ? B + (long)(k0 + r) * ldb + n0 + nc : B;
      cp16(&Bs[buf][r * kBStride + nc], src, v);
    }
    cp_commit();
  };
  double acc[4][4][2];
#pragma unroll
  for (int i = 0; i < 4; ++i)
#pragma unroll
    for (int j = 0; j < 4; ++j) acc[i][j][0] = acc[i][j][1] = 0.0;
  const int nk = (kend - kbeg + kBK - 1) / kBK;
  issue(kbeg, 0);
  for (int ks = 0; ks < nk; ++ks) {
    const int buf = ks & 1;
    if (ks + 1 < nk) {
      issue(kbeg + (ks + 1) * kBK, buf ^ 1);
      cp_wait<1>();
    } else {
      cp_wait<0>();
    }
    __syncthreads();
    const double* as = As[buf] + (wm * 32) * kAStride;
    const double* bs = Bs[buf] + wn * 32;
#pragma unroll
    for (int kk = 0; kk < kBK; kk += 4) {
      double a[4], b[4];
#pragma unroll
      for (int i = 0; i < 4; ++i) a[i] = as[(i * 8 + g) * kAStride + kk + t];
#pragma unroll
      for (int j = 0; j < 4; ++j) b[j] = bs[(kk + t) * kBStride + j * 8 + g];
#pragma unroll
      for (int i = 0; i < 4; ++i)
#pragma unroll
        for (int j = 0; j < 4; ++j) dmma(acc[i][j], a[i], b[j]);
    }
    __syncthreads();  // buffer buf is refilled by the next step's issue
  }
  // epilogue: rows g (+8i), columns 2t, 2t+1 of each 8x8 tile
#pragma unroll
  for (int i = 0; i < 4; ++i) {
    const long mi = m0 + wm * 32 + i * 8 + g;
    if (mi >= M) continue;
    if (partial) {  // split K: plain partial sums, reduced by translate_reduce
      double* prow = partial + ((long)blockIdx.z * M + mi) * N;
#pragma unroll
      for (int j = 0; j < 4; ++j) {
        const int n = n0 + wn * 32 + j * 8 + 2 * t;
        if (n < N) *reinterpret_cast<double2*>(prow + n) = make_double2(acc[i][j][0], acc[i][j][1]);
      }
      continue;
    }
    double s = 1.0;
    if (keys) s = ldexp(1.0, -deg * (int)(keys[arow_s[mi - m0]].lo & 31u));
    const long cr = crows ? (long)crows[mi] : mi;
    double* crow = C + cr * ldc;
#pragma unroll
    for (int j = 0; j < 4; ++j) {
      const int n = n0 + wn * 32 + j * 8 + 2 * t;
      if (n >= N) continue;  // N is even: n < N implies n + 1 < N
      double2 v = make_double2(acc[i][j][0] * s, acc[i][j][1] * s);
      double2* p = reinterpret_cast<double2*>(crow + n);
      if (accumulate) {
        const double2 o = *p;
        v.x += o.x;
        v.y += o.y;
      }
      *p = v;
    }
  }
}

// C[crow(i)][n] (+)= s(i) * sum_z partial[z][i][n], the K pieces added in order.
__global__ void translate_reduce(long M, int N, int ksplit, const double* __restrict__ partial,
                                 const int* __restrict__ arows, const int* __restrict__ crows,
                                 const MKey* __restrict__ keys, int deg, int accumulate, double* __restrict__ C,
                                 long ldc) {
  const long e = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (e >= M * N) return;
  const long i = e / N;
  const int n = (int)(e % N);
  double v = 0;
  for (int z = 0; z < ksplit; ++z) v += partial[((long)z * M + i) * N + n];
  if (keys) v *= ldexp(1.0, -deg * (int)(keys[arows ? arows[i] : i].lo & 31u));
  double* c = C + (crows ? (long)crows[i] : i) * ldc + n;
  *c = accumulate ? *c + v : v;
}

}  // namespace

void translate_gemm(cudaStream_t s, long M, int N, int K, const double* A, long lda, const int* arows,
                    const double* B, long ldb, double* C, long ldc, const int* crows, const MKey* scale_keys,
                    bool accumulate, int ksplit, double* partial, int deg) {
  if (M <= 0 || N <= 0) return;
  if (ksplit < 1 || (ksplit > 1 && (!partial || K % ksplit != 0 || (K / ksplit) % 2 != 0)))
    throw std::runtime_error("translate_gemm: bad K split");
  if ((N & 1) || (K & 1) || (lda & 1) || (ldb & 1) || (ldc & 1))
    throw std::runtime_error("translate_gemm: row lengths must be even (16-byte rows)");
  if (M >= (1L << 31)) throw std::runtime_error("translate_gemm: too many rows");
  PVFMM_CUDA_CHECK(cudaFuncSetAttribute(translate_gemm_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, kSmemG));
  // the column tiles of one row tile are consecutive blocks (they share the
  // A rows in L2); row tiles in launches of at most 65535
  const long tiles = (M + kBM - 1) / kBM;
  for (long t0 = 0; t0 < tiles; t0 += 65535) {
    dim3 grid((unsigned)((N + kBN - 1) / kBN), (unsigned)std::min(65535L, tiles - t0), (unsigned)ksplit);
    translate_gemm_kernel<<<grid, kThreadsG, kSmemG, s>>>((int)M, N, K, A, lda, arows, B, ldb, C, ldc, crows, scale_keys,
                                                      deg, accumulate ? 1 : 0, t0 * kBM, K / ksplit,
                                                      ksplit > 1 ? partial : nullptr);
    PVFMM_CUDA_CHECK(cudaGetLastError());
  }
  if (ksplit > 1) {
    translate_reduce<<<(unsigned)((M * N + 255) / 256), 256, 0, s>>>(M, N, ksplit, partial, arows, crows, scale_keys,
                                                                     deg, accumulate ? 1 : 0, C, ldc);
    PVFMM_CUDA_CHECK(cudaGetLastError());
  }
}

}  // namespace pvfmm_b200

// Self-check of the FP64 translation product on random data (internal entry
// point used by the GPU tests; no counterpart in the reference): computes
// C[crow(i)] (+)= s(i) A[arow(i)] B on device copies of the host arrays (K
// split into `ksplit` pieces when > 1) and copies C back.  arows / crows /
// depth may be NULL.  Returns 0 on success.
extern "C" int PVFMMB200TranslateGemmCheck(long M, int N, int K, const double* A, long a_rows, const int* arows,
                                           const double* B, double* C, long c_rows, const int* crows,
                                           const int* depth_of_arow_target, int accumulate, int ksplit) {
  using namespace pvfmm_b200;
  void* buf = nullptr;
  try {
    const size_t nA = (size_t)a_rows * K, nB = (size_t)K * N, nC = (size_t)c_rows * N;
    const size_t nP = ksplit > 1 ? (size_t)ksplit * M * N : 0;
    const size_t bytes = (nA + nB + nC + nP) * 8 + (size_t)M * 4 * 2 + (size_t)a_rows * sizeof(MKey) + 256;
    PVFMM_CUDA_CHECK(cudaMalloc(&buf, bytes));
    double* dA = (double*)buf;
    double* dB = dA + nA;
    double* dC = dB + nB;
    double* dP = dC + nC;
    int* dar = (int*)(dP + nP);
    int* dcr = dar + M;
    MKey* dk = (MKey*)(((uintptr_t)(dcr + M) + 15) & ~(uintptr_t)15);
    PVFMM_CUDA_CHECK(cudaMemcpy(dA, A, nA * 8, cudaMemcpyHostToDevice));
    PVFMM_CUDA_CHECK(cudaMemcpy(dB, B, nB * 8, cudaMemcpyHostToDevice));
    PVFMM_CUDA_CHECK(cudaMemcpy(dC, C, nC * 8, cudaMemcpyHostToDevice));
    if (arows) PVFMM_CUDA_CHECK(cudaMemcpy(dar, arows, M * 4, cudaMemcpyHostToDevice));
    if (crows) PVFMM_CUDA_CHECK(cudaMemcpy(dcr, crows, M * 4, cudaMemcpyHostToDevice));
    if (depth_of_arow_target) {
      std::vector<MKey> k(a_rows);
      for (long i = 0; i < a_rows; ++i) k[i] = make_key(0, 0, 0, (unsigned)depth_of_arow_target[i]);
      PVFMM_CUDA_CHECK(cudaMemcpy(dk, k.data(), a_rows * sizeof(MKey), cudaMemcpyHostToDevice));
    }
    translate_gemm(nullptr, M, N, K, dA, K, arows ? dar : nullptr, dB, N, dC, N, crows ? dcr : nullptr,
                   depth_of_arow_target ? dk : nullptr, accumulate != 0, ksplit, dP);
    PVFMM_CUDA_CHECK(cudaMemcpy(C, dC, nC * 8, cudaMemcpyDeviceToHost));
    cudaFree(buf);
    set_last_error("");
    return 0;
  } catch (const std::exception& e) {
    if (buf) cudaFree(buf);
    set_last_error(e.what());
    return 1;
  }
}
