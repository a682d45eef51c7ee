// V-list Hadamard products of the mixed form (ke = 1) on the 5th-generation
// tensor cores: tcgen05.mma kind::tf32 with TMEM accumulators (reference:
// VListHadamard / matmult_8x8x2, include/fmm_pts.txx:3249-3344, 2860-3247).
//
// Per frequency f the V-list translation is, for every target parent P,
//   OUT[P][f] = sum over occupied offsets o of  IN[Q_o(P)][f] * B_o(f),
// a 16-float spectrum row (8 children, re/im interleaved) times the 16 x 16
// real form of the 8 x 8 complex operator block of offset o.  A CTA owns one
// frequency and runs four independent pipelines (warpgroups), each walking
// tiles of 128 target parents (M = 128 rows, one TMEM lane per parent):
//   - the 26 operator blocks of the frequency, each as TF32 hi and lo parts
//     in the canonical K-major no-swizzle layout, arrive once by a bulk
//     asynchronous copy (cp.async.bulk, 53 KB) and stay in shared memory for
//     all four pipelines;
//   - for each offset occupied by some parent of the tile, every thread
//     stages its parent's neighbour row (64 B, from L2) with cp.async four
//     offsets ahead, then splits each value into TF32 hi + lo (both rounded
//     to nearest) and stores them into an A stage in TMEM (tcgen05.st); once
//     the four warps of the pipeline have arrived on an mbarrier, one thread
//     issues 6 MMAs (2 K-steps x {lo*hi, hi*lo, hi*hi}) into a fresh
//     16-column TMEM accumulator and commits them to another mbarrier;
//   - while the tensor cores work on offset j, the threads drain offset j-1's
//     accumulator (tcgen05.ld) into their running FP32 sums with rounded FP32
//     adds.  A fresh accumulator per offset keeps the tensor cores' own
//     accumulation to 6 products (carried over all offsets, its rounding
//     biased the far-field potential by ~2e-6).
// TMEM per pipeline: 2 A stages (hi 16 + lo 16 columns each) + 2 accumulators
// of 16 columns (96 of 128 columns; 512 per CTA).  Every wait is bounded: a
// wait that runs out sets the error word, and the host reports it.
#include <cstring>

#include "fmm_context.cuh"

namespace pvfmm_b200 {
namespace {

constexpr int kTcThreads = 128;          // one thread per row (TMEM lane) of the tile
constexpr int kTcTile = 128;             // target parents per tile
constexpr int kOpBlockBytes = 512;       // one K-step (16 N x 8 K TF32) of one part of one offset
constexpr int kOpBytes = 26 * 2 * 2 * kOpBlockBytes;  // [offset][hi, lo][K-step] = 53,248 B
constexpr unsigned kTmemCols = 128;
constexpr unsigned long long kWaitLimitNs = 2000000000ull;  // bounded waits: 2 s

__device__ __forceinline__ unsigned smem_u32(const void* p) { return (unsigned)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(unsigned long long* bar, unsigned count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;\n" ::"r"(smem_u32(bar)), "r"(count));
}
__device__ __forceinline__ bool mbar_try_wait(unsigned long long* bar, unsigned parity) {
  unsigned ok;
  asm volatile(
      "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
      : "=r"(ok)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return ok != 0;
}
// Waits for the completion of the phase with the given parity.  A wait that
// runs out sets the error word and returns false; the kernel then carries on
// without the result (the host reports the error), so every thread still
// reaches every barrier and the TMEM is freed.
__device__ __forceinline__ bool mbar_wait(unsigned long long* bar, unsigned parity, int* err, int code) {
  unsigned long long t0;
  asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t0));
  for (;;) {
    if (mbar_try_wait(bar, parity)) return true;
    if (*(volatile int*)err != 0) return false;  // an earlier wait already ran out: do not wait again
    unsigned long long t;
    asm volatile("mov.u64 %0, %%globaltimer;" : "=l"(t));
    if (t - t0 > kWaitLimitNs) break;
  }
  atomicOr(err, code);
  return false;
}

__device__ __forceinline__ void tc_fence_before() { asm volatile("tcgen05.fence::before_thread_sync;\n" ::: "memory"); }
__device__ __forceinline__ void tc_fence_after() { asm volatile("tcgen05.fence::after_thread_sync;\n" ::: "memory"); }

// D[tmem d] (+)= A[tmem a] * B[smem desc b], kind::tf32, M = 128, N = 16, K = 8.
__device__ __forceinline__ void mma_tf32(unsigned d, unsigned a, unsigned long long b_desc, unsigned idesc,
                                         bool accumulate) {
  asm volatile(
      "{\n .reg .pred p;\n setp.ne.b32 p, %4, 0;\n"
      " tcgen05.mma.cta_group::1.kind::tf32 [%0], [%1], %2, %3, p;\n}\n" ::"r"(d),
      "r"(a), "l"(b_desc), "r"(idesc), "r"(accumulate ? 1 : 0));
}
__device__ __forceinline__ void mma_commit(unsigned long long* bar) {
  asm volatile("tcgen05.commit.cta_group::1.mbarrier::arrive::one.shared::cluster.b64 [%0];\n" ::"r"(smem_u32(bar))
               : "memory");
}

// Instruction descriptor of kind::tf32: D FP32 (bits 4-5 = 1), A and B TF32
// (bits 7-9, 10-12 = 2), both K-major, N >> 3 at bits 17-22, M >> 4 at 24-28.
constexpr unsigned kIdesc = (1u << 4) | (2u << 7) | (2u << 10) | ((16u >> 3) << 17) | ((128u >> 4) << 24);

// Shared-memory matrix descriptor, canonical K-major layout without swizzle:
// core matrices of 8 rows x 16 B (128 contiguous bytes); LBO = byte step
// between core matrices along K, SBO = along N; version 1 (bit 46).
__device__ __forceinline__ unsigned long long smem_desc(unsigned addr, unsigned lbo, unsigned sbo) {
  return (unsigned long long)((addr >> 4) & 0x3fff) | ((unsigned long long)((lbo >> 4) & 0x3fff) << 16) |
         ((unsigned long long)((sbo >> 4) & 0x3fff) << 32) | (1ull << 46);
}

__device__ __forceinline__ void tmem_st16(unsigned taddr, const unsigned (&v)[16]) {
  asm volatile(
      "tcgen05.st.sync.aligned.32x32b.x16.b32 [%0], {%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15,%16};\n" ::"r"(
          taddr),
      "r"(v[0]), "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]),
      "r"(v[10]), "r"(v[11]), "r"(v[12]), "r"(v[13]), "r"(v[14]), "r"(v[15])
      : "memory");
}
__device__ __forceinline__ void tmem_ld16(unsigned taddr, float (&v)[16]) {
  unsigned r[16];
  asm volatile(
      "tcgen05.ld.sync.aligned.32x32b.x16.b32 {%0,%1,%2,%3,%4,%5,%6,%7,%8,%9,%10,%11,%12,%13,%14,%15}, [%16];\n"
      : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]),
        "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(r[12]), "=r"(r[13]), "=r"(r[14]), "=r"(r[15])
      : "r"(taddr)
      : "memory");
#pragma unroll
  for (int i = 0; i < 16; ++i) v[i] = __uint_as_float(r[i]);
}
__device__ __forceinline__ void tmem_wait_st() { asm volatile("tcgen05.wait::st.sync.aligned;\n" ::: "memory"); }
__device__ __forceinline__ void tmem_wait_ld() { asm volatile("tcgen05.wait::ld.sync.aligned;\n" ::: "memory"); }

__device__ __forceinline__ unsigned tf32_rna(float x) {
  unsigned h;
  asm("cvt.rna.tf32.f32 %0, %1;" : "=r"(h) : "f"(x));
  return h;
}

// Error word codes (bit set per failing wait kind).
constexpr int kErrOperators = 1, kErrMma = 2;

constexpr int kGroups = 4;                      // tile pipelines (warpgroups) per CTA
constexpr int kRowBytes = 64;                   // one spectrum row: 8 children x complex FP32
constexpr int kUnionEntries = kTcTile * 26;     // (target, offset) pairs of a tile
constexpr int kUnionCap = 512;                  // union rows a pipeline stages in shared memory
constexpr int kLocalStride = 32;                // offsets per target in the local-index table (26 used)
constexpr int kUnionBytes = kUnionCap * kRowBytes;
constexpr int kLocalBytes = kTcTile * kLocalStride * 2;
constexpr int kGroupBytes = kUnionBytes + kLocalBytes;
constexpr size_t kSmemBytes = (size_t)kOpBytes + (size_t)kGroups * kGroupBytes + 256;
constexpr unsigned short kNoSource = 0xffff;

__device__ __forceinline__ void cp16(unsigned smem, const void* gmem, bool valid) {
  asm volatile("cp.async.cg.shared.global [%0], [%1], 16, %2;\n" ::"r"(smem), "l"(gmem), "r"(valid ? 16 : 0)
               : "memory");
}

// Source unions of the tiles of 128 Morton-consecutive V-list targets (one
// block per tile): the (target, offset) pairs of the tile are sorted by source
// parent (bitonic sort of 4096 keys in shared memory), the distinct sources
// form the tile's union (sorted), and each pair gets the index of its source
// in the union (kNoSource where the target has no source at that offset).
// The tiles of a Morton window share most of their neighbours: at 300k
// Gaussian points a tile's 3,328 pairs reference ~270 distinct sources.
__global__ void __launch_bounds__(512) vlist_tile_unions(long n_vtrg, long vt_stride, const int* __restrict__ vtab,
                                                         const int* __restrict__ vmorton, int* __restrict__ vunion,
                                                         int* __restrict__ vucount, unsigned short* __restrict__ vlocal) {
  constexpr int NE = 4096, NT = 512;
  __shared__ unsigned long long e[NE];  // source << 32 | pair index; ~0 = no source
  __shared__ int wsum[NT / 32];
  const int tid = threadIdx.x;
  const long tile = blockIdx.x;
  unsigned short* loc = vlocal + tile * kTcTile * kLocalStride;
  for (int i = tid; i < kTcTile * kLocalStride; i += NT) loc[i] = kNoSource;
  for (int i = tid; i < NE; i += NT) {
    unsigned long long v = ~0ull;
    if (i < kUnionEntries) {
      const int r = i / 26, o = i % 26;
      const long k = tile * kTcTile + r;
      const int q = k < n_vtrg ? vtab[(long)o * vt_stride + vmorton[k]] : -1;
      if (q >= 0) v = (unsigned long long)(unsigned)q << 32 | (unsigned)i;
    }
    e[i] = v;
  }
  __syncthreads();
  for (int k = 2; k <= NE; k <<= 1)
    for (int j = k >> 1; j > 0; j >>= 1) {
      for (int i = tid; i < NE; i += NT) {
        const int l = i ^ j;
        if (l > i) {
          const unsigned long long a = e[i], b = e[l];
          const bool up = (i & k) == 0;
          if ((a > b) == up) {
            e[i] = b;
            e[l] = a;
          }
        }
      }
      __syncthreads();
    }
  // thread t owns entries [8t, 8t+8): distinct-source flags, then a block scan
  constexpr int PER = NE / NT;
  int cnt = 0;
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    const int i = tid * PER + u;
    const unsigned long long v = e[i];
    if (v != ~0ull && (i == 0 || (e[i - 1] >> 32) != (v >> 32))) ++cnt;
  }
  const int lane = tid & 31, w = tid >> 5;
  int inc = cnt;
#pragma unroll
  for (int d = 1; d < 32; d <<= 1) {
    const int y = __shfl_up_sync(0xffffffffu, inc, d);
    if (lane >= d) inc += y;
  }
  if (lane == 31) wsum[w] = inc;
  __syncthreads();
  int before = 0;
  for (int x = 0; x < w; ++x) before += wsum[x];
  int pos = before + inc - cnt - 1;  // index of the last distinct source before this thread's entries
  int* un = vunion + tile * kUnionEntries;
#pragma unroll
  for (int u = 0; u < PER; ++u) {
    const int i = tid * PER + u;
    const unsigned long long v = e[i];
    if (v == ~0ull) continue;
    if (i == 0 || (e[i - 1] >> 32) != (v >> 32)) {
      ++pos;
      un[pos] = (int)(v >> 32);
    }
    const int pair = (int)(v & 0xffffffffu), r = pair / 26, o = pair % 26;
    loc[r * kLocalStride + o] = (unsigned short)pos;
  }
  if (tid == NT - 1) {
    int total = 0;
    for (int x = 0; x < NT / 32; ++x) total += wsum[x];
    vucount[tile] = total;
  }
}

// One CTA per SM: four independent tile pipelines (warpgroups of 128 threads,
// one TMEM lane per target) share the frequency's operator blocks.  A tile is
// 128 Morton-consecutive targets; at its start the pipeline stages the rows
// of the tile's source union at this frequency (up to kUnionCap rows; the
// chunks of row u at slot c ^ ((u >> 1) & 3), against bank conflicts) and the
// tile's local-index table, so that each (target, offset) row is then read
// from shared memory.
__global__ void __launch_bounds__(kGroups * kTcThreads, 1)
    hadamard_tc5_kernel(int n3h, long p0, long np, long vt_stride, int tiles_per_cta, const int* __restrict__ vmorton,
                        const unsigned* __restrict__ vmask, const int* __restrict__ vunion,
                        const int* __restrict__ vucount, const unsigned short* __restrict__ vlocal,
                        const float4* __restrict__ spec_in, const unsigned char* __restrict__ ops,
                        float4* __restrict__ spec_out, int* __restrict__ err) {
  extern __shared__ __align__(1024) unsigned char smem[];
  unsigned char* Bs = smem;                                          // kOpBytes
  unsigned char* gsm = smem + kOpBytes;                              // [group]: union rows, local indices
  // mbarriers: [0] operators arrived; per group g at 1 + 4g: [+0, +1] MMAs of
  // A stage 0/1 done, [+2, +3] A stage 0/1 written by the group's four warps
  unsigned long long* bars = reinterpret_cast<unsigned long long*>(smem + kOpBytes + (size_t)kGroups * kGroupBytes);
  unsigned* tmem_slot = reinterpret_cast<unsigned*>(bars + 1 + 4 * kGroups);
  unsigned* live_s = tmem_slot + 1;                                  // [kGroups]
  const int tid = threadIdx.x, warp = tid >> 5;
  const int grp = tid / kTcThreads, gt = tid % kTcThreads, gwarp = gt >> 5;
  const int f = blockIdx.y;
  unsigned long long* gbar = bars + 1 + 4 * grp;

  if (tid == 0) {
    mbar_init(&bars[0], 1);
    for (int g = 0; g < kGroups; ++g) {
      mbar_init(&bars[1 + 4 * g + 0], 1);
      mbar_init(&bars[1 + 4 * g + 1], 1);
      mbar_init(&bars[1 + 4 * g + 2], kTcThreads / 32);
      mbar_init(&bars[1 + 4 * g + 3], kTcThreads / 32);
    }
    asm volatile("fence.mbarrier_init.release.cluster;\n" ::: "memory");
  }
  if (warp == 0) {
    asm volatile("tcgen05.alloc.cta_group::1.sync.aligned.shared::cta.b32 [%0], %1;\n" ::"r"(smem_u32(tmem_slot)),
                 "r"(kTmemCols * kGroups)
                 : "memory");
    asm volatile("tcgen05.relinquish_alloc_permit.cta_group::1.sync.aligned;\n" ::: "memory");
  }
  __syncthreads();
  tc_fence_after();
  // this group's TMEM: columns [0,32) A stage 0 (hi 0-15, lo 16-31), [32,64)
  // A stage 1, [64,80) accumulator 0, [80,96) accumulator 1; the group's four
  // warps cover lanes 0-127
  const unsigned tmem = *tmem_slot + kTmemCols * grp;
  const unsigned lane_base = (unsigned)(gwarp * 32) << 16;

  // the frequency's operator blocks: one bulk copy, completion on bars[0]
  if (tid == 0) {
    asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;\n" ::"r"(smem_u32(&bars[0])),
                 "r"((unsigned)kOpBytes)
                 : "memory");
    asm volatile(
        "cp.async.bulk.shared::cluster.global.mbarrier::complete_tx::bytes [%0], [%1], %2, [%3];\n" ::"r"(smem_u32(Bs)),
        "l"(ops + (size_t)f * kOpBytes), "r"((unsigned)kOpBytes), "r"(smem_u32(&bars[0]))
        : "memory");
  }
  mbar_wait(&bars[0], 0, err, kErrOperators);
  const unsigned b_base = smem_u32(Bs);
  const unsigned union_base = smem_u32(gsm) + (unsigned)(grp * kGroupBytes);
  const unsigned local_base = union_base + kUnionBytes;
  const long n_tiles = (np + kTcTile - 1) / kTcTile;

  unsigned jglob = 0;  // offsets processed by this group (mbarrier phase bookkeeping)
  for (int tl = grp; tl < tiles_per_cta; tl += kGroups) {
    const long tile = (long)blockIdx.x * tiles_per_cta + tl;  // within the chunk
    if (tile >= n_tiles) break;                                // uniform across the group
    const long tg = p0 / kTcTile + tile;                       // tile of the whole V-list
    const long k = p0 + tile * kTcTile + gt;                   // this thread's Morton rank
    const bool in = k < p0 + np;
    const long p = in ? (long)__ldg(vmorton + k) : 0;          // its position (output row p - p0)
    // every thread of the group is done with the previous tile's shared rows
    asm volatile("bar.sync %0, %1;\n" ::"r"(1 + grp), "r"(kTcThreads) : "memory");
    if (gt == 0) live_s[grp] = 0;
    // stage the tile's union rows (at this frequency) and local-index table
    const int nu = __ldg(vucount + tg);
    const int ns_ = min(nu, kUnionCap);
    const int* un = vunion + tg * kUnionEntries;
    for (int u = gt; u < ns_; u += kTcThreads) {
      const float4* src = spec_in + ((long)__ldg(un + u) * n3h + f) * 4;
      const unsigned dst = union_base + (unsigned)(u * kRowBytes);
      const int sw = (u >> 1) & 3;
#pragma unroll
      for (int c = 0; c < 4; ++c) cp16(dst + 16u * (unsigned)(c ^ sw), src + c, true);
    }
    {
      const unsigned char* lsrc = reinterpret_cast<const unsigned char*>(vlocal + tg * kTcTile * kLocalStride);
#pragma unroll
      for (int c = 0; c < kLocalBytes / 16 / kTcThreads; ++c) {
        const int chunk = gt + c * kTcThreads;
        cp16(local_base + 16u * (unsigned)chunk, lsrc + 16 * chunk, true);
      }
    }
    asm volatile("cp.async.commit_group;\n" ::: "memory");
    asm volatile("bar.sync %0, %1;\n" ::"r"(1 + grp), "r"(kTcThreads) : "memory");
    const unsigned mine = in ? __ldg(vmask + p) : 0u;
    const unsigned wl = __reduce_or_sync(0xffffffffu, mine);
    if ((gt & 31) == 0 && wl) atomicOr(&live_s[grp], wl);
    asm volatile("cp.async.wait_group 0;\n" ::: "memory");
    asm volatile("bar.sync %0, %1;\n" ::"r"(1 + grp), "r"(kTcThreads) : "memory");
    unsigned rem = live_s[grp];
    const int nlive = __popc(rem);
    float sum[16];
#pragma unroll
    for (int i = 0; i < 16; ++i) sum[i] = 0.f;
    auto drain = [&](unsigned j) {  // adds offset j's accumulator into sum
      const unsigned s = j & 1u;
      mbar_wait(&gbar[s], (j >> 1) & 1u, err, kErrMma);
      __syncwarp();
      tc_fence_after();
      float d[16];
      tmem_ld16(tmem + lane_base + 64u + 16u * s, d);
      tmem_wait_ld();
#pragma unroll
      for (int k2 = 0; k2 < 16; ++k2) sum[k2] = __fadd_rn(sum[k2], d[k2]);
    };
    for (int i = 0; i < nlive; ++i) {
      const int o = __ffs(rem) - 1;
      rem &= rem - 1;
      const unsigned j = jglob + (unsigned)i;
      // this target's neighbour row at offset o: from the staged union, from
      // L2 past the staged rows, zeros without a source
      unsigned short u;
      asm volatile("ld.shared.u16 %0, [%1];\n" : "=h"(u) : "r"(local_base + 2u * (unsigned)(gt * kLocalStride + o)));
      float v[16];
      if (u == kNoSource) {
#pragma unroll
        for (int e2 = 0; e2 < 16; ++e2) v[e2] = 0.f;
      } else if (u < kUnionCap) {
        const unsigned src = union_base + (unsigned)(u * kRowBytes);
        const int sw = (u >> 1) & 3;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          float4 w;
          asm volatile("ld.shared.v4.f32 {%0,%1,%2,%3}, [%4];\n"
                       : "=f"(w.x), "=f"(w.y), "=f"(w.z), "=f"(w.w)
                       : "r"(src + 16u * (unsigned)(c ^ sw))
                       : "memory");
          v[4 * c] = w.x;
          v[4 * c + 1] = w.y;
          v[4 * c + 2] = w.z;
          v[4 * c + 3] = w.w;
        }
      } else {
        const float4* r = spec_in + ((long)__ldg(un + u) * n3h + f) * 4;
#pragma unroll
        for (int c = 0; c < 4; ++c) {
          const float4 w = __ldg(r + c);
          v[4 * c] = w.x;
          v[4 * c + 1] = w.y;
          v[4 * c + 2] = w.z;
          v[4 * c + 3] = w.w;
        }
      }
      // TF32 hi / lo parts of the 16 values (K order = memory order)
      unsigned hi[16], lo[16];
#pragma unroll
      for (int e2 = 0; e2 < 16; ++e2) {
        const unsigned h = tf32_rna(v[e2]);
        hi[e2] = h;
        lo[e2] = tf32_rna(v[e2] - __uint_as_float(h));
      }
      // A stage j&1 was last read by the MMAs of offset j-2, complete since
      // offset j-1 was drained (commits complete in order)
      const unsigned a_col = 32u * (j & 1u);
      __syncwarp();
      tmem_st16(tmem + lane_base + a_col, hi);
      tmem_st16(tmem + lane_base + a_col + 16u, lo);
      tmem_wait_st();
      tc_fence_before();
      __syncwarp();
      // one arrival per warp; only the group's MMA-issuing thread waits for
      // all four
      if ((gt & 31) == 0)
        asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];\n" ::"r"(smem_u32(&gbar[2 + (j & 1u)])) : "memory");
      if (gt == 0) {
        mbar_wait(&gbar[2 + (j & 1u)], (j >> 1) & 1u, err, kErrMma);
        tc_fence_after();
        const unsigned d_col = tmem + 64u + 16u * (j & 1u);
        const unsigned a_hi = tmem + a_col, a_lo = tmem + a_col + 16u;
        const unsigned ob = b_base + (unsigned)o * (4 * kOpBlockBytes);
#pragma unroll
        for (int ks = 0; ks < 2; ++ks) {
          const unsigned long long bh = smem_desc(ob + (0 * 2 + ks) * kOpBlockBytes, 128, 256);
          const unsigned long long bl = smem_desc(ob + (1 * 2 + ks) * kOpBlockBytes, 128, 256);
          mma_tf32(d_col, a_lo + 8u * ks, bh, kIdesc, ks > 0);
          mma_tf32(d_col, a_hi + 8u * ks, bl, kIdesc, true);
          mma_tf32(d_col, a_hi + 8u * ks, bh, kIdesc, true);
        }
        mma_commit(&gbar[j & 1u]);
      }
      if (i > 0) drain(j - 1);
    }
    if (nlive > 0) drain(jglob + (unsigned)nlive - 1);
    jglob += (unsigned)nlive;
    if (in) {
      float4* out = spec_out + ((p - p0) * n3h + f) * 4;
#pragma unroll
      for (int c = 0; c < 4; ++c) out[c] = make_float4(sum[4 * c], sum[4 * c + 1], sum[4 * c + 2], sum[4 * c + 3]);
    }
  }
  tc_fence_before();
  __syncthreads();
  if (warp == 0) {
    tc_fence_after();
    asm volatile("tcgen05.dealloc.cta_group::1.sync.aligned.b32 %0, %1;\n" ::"r"(*tmem_slot),
                 "r"(kTmemCols * kGroups)
                 : "memory");
  }
}

}  // namespace

// Operator blocks in the layout hadamard_tc5_kernel stages: per frequency f
// and offset o, [hi, lo][K-step ks][512 B]; a 512-B block holds the 16 (N) x
// 8 (K) TF32 values B[k = 8 ks + kk][n] as core matrices of 8 rows (n) x 4
// values (k): core (n / 8, kk / 4) at byte (2 (n / 8) + kk / 4) * 128, row
// n % 8 at +16 (n % 8), value kk % 4 at +4 (kk % 4).  B is the real form of the
// complex block M = M[f][o][j1][j2] (k = 2 j2 + (0 re | 1 im), n = 2 j1 + (0
// re | 1 im)): B[re][re] = B[im][im] = Re M, B[im][re] = -Im M, B[re][im] = Im M.
// hi = value rounded to TF32 (to nearest, ties away), lo = the remainder
// rounded likewise.
void hadamard_tc5_operator_layout(const std::vector<double>& vop, int n3h, std::vector<float>& out) {
  out.assign((size_t)n3h * kOpBytes / 4, 0.f);
  auto rna = [](float x) {
    unsigned u;
    std::memcpy(&u, &x, 4);
    if ((u & 0x7f800000u) != 0x7f800000u) u = (u + 0x1000u) & 0xffffe000u;
    float r;
    std::memcpy(&r, &u, 4);
    return r;
  };
  for (int f = 0; f < n3h; ++f)
    for (int o = 0; o < 26; ++o)
      for (int k = 0; k < 16; ++k)
        for (int n = 0; n < 16; ++n) {
          const int j2 = k >> 1, ci = k & 1, j1 = n >> 1, co = n & 1;
          const size_t src = ((((size_t)f * 26 + o) * 8 + j1) * 8 + j2) * 2;
          const float mr = (float)vop[src], mi = (float)vop[src + 1];
          const float b = ci == co ? mr : (ci == 1 ? -mi : mi);
          const float h = rna(b), l = rna(b - h);
          const int ks = k >> 3, kk = k & 7;
          const size_t within = (size_t)(2 * (n >> 3) + (kk >> 2)) * 128 + (n & 7) * 16 + (kk & 3) * 4;
          for (int part = 0; part < 2; ++part) {
            const size_t byte = (size_t)f * kOpBytes + (size_t)o * 4 * kOpBlockBytes +
                                (size_t)(part * 2 + ks) * kOpBlockBytes + within;
            out[byte / 4] = part == 0 ? h : l;
          }
        }
}

// The tiles' source unions and local indices, once per tree.
void ensure_tile_unions(Context& ctx) {
  DevTree& T = ctx.tree;
  if (T.vtiles_valid) return;
  const long all_tiles = (T.n_vtrg + kTcTile - 1) / kTcTile;
  int* un = T.vunion.as<int>((size_t)all_tiles * kUnionEntries);
  int* uc = T.vucount.as<int>(all_tiles);
  unsigned short* lc = T.vlocal.as<unsigned short>((size_t)all_tiles * kTcTile * kLocalStride);
  ++ctx.n_launch;
  vlist_tile_unions<<<(unsigned)all_tiles, 512, 0, ctx.stream>>>(T.n_vtrg, T.n_vtrg, T.vtab.get<int>(),
                                                                 T.vmorton.get<int>(), un, uc, lc);
  PVFMM_CUDA_CHECK(cudaGetLastError());
  T.vtiles_valid = true;
}

// Morton ranks and pattern positions agree on windows of 2048 targets, so a
// chunk must consist of whole windows (or run to the end).
void check_window_chunk(const Context& ctx, long p0, long np) {
  if (p0 % 2048 != 0 || (p0 + np != ctx.tree.n_vtrg && np % 2048 != 0))
    throw std::runtime_error("V-list Hadamard: chunk of target parents not made of whole Morton windows");
}

void launch_hadamard_tc5(Context& ctx, int n3h, long f_base, const void* sin_, void* sout, long p0, long np) {
  DevTree& T = ctx.tree;
  check_window_chunk(ctx, p0, np);
  ensure_tile_unions(ctx);
  PVFMM_CUDA_CHECK(
      cudaFuncSetAttribute(hadamard_tc5_kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)kSmemBytes));
  const int tiles = 32;  // tiles of 128 targets per CTA (operators staged once)
  const long n_tiles = (np + kTcTile - 1) / kTcTile;
  dim3 grid((unsigned)((n_tiles + tiles - 1) / tiles), (unsigned)n3h);
  int* err = ctx.tc5_err_buf.as<int>(1);
  if (!ctx.tc5_err) PVFMM_CUDA_CHECK(cudaMemsetAsync(err, 0, sizeof(int), ctx.stream));  // once per evaluation
  ++ctx.n_launch;
  hadamard_tc5_kernel<<<grid, kGroups * kTcThreads, kSmemBytes, ctx.stream>>>(
      n3h, p0, np, T.n_vtrg, tiles, T.vmorton.get<int>(), T.vmask.get<unsigned>(), T.vunion.get<int>(),
      T.vucount.get<int>(), T.vlocal.get<unsigned short>(), reinterpret_cast<const float4*>(sin_),
      ctx.dops.vop_tc5.get<unsigned char>() + f_base * kOpBytes, reinterpret_cast<float4*>(sout), err);
  PVFMM_CUDA_CHECK(cudaGetLastError());
  ctx.tc5_err = err;
}

}  // namespace pvfmm_b200
