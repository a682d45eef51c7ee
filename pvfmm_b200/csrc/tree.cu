// GPU octree construction for the particle FMM.
//
// Reproduces, on the device, the tree PVFMM builds on one rank:
//   * bounding-box map into [0,1)^3        src/pvfmm-wrapper.cpp:458-590
//   * Morton ids + stable sort              include/mortonid.txx:25-53,107-118,
//                                           include/parUtils.txx:527 (ties keep input order)
//   * refinement: a leaf splits while depth < MAX_DEPTH-1 and either the
//     context's seed grid (pvfmm-wrapper.cpp:416-432) or src+trg counts exceed
//     max_pts                               include/fmm_node.txx:63-98, mpi_tree.txx:403-492
//   * 2:1 balance as the closure of the internal-node set under
//     X -> parent(NbrList(X))              include/mpi_tree.txx:745-943
//   * colleagues                            include/mpi_tree.txx:1136-1256
//   * U/V/W/X lists with the Nsrf rule      include/interac_list.txx:98-279,
//                                           include/fmm_pts.txx:4629, 4929, 5295, 5325
// Each level is a Morton-sorted array; children of an internal node are the
// 8 consecutive nodes of the next level.
#include <cub/cub.cuh>

#include <algorithm>
#include <cmath>

#include "fmm_context.cuh"

namespace pvfmm_b200 {
namespace {

constexpr int kThreads = 256;

// ------------------------------------------------------------------ bbox
template <class T>
__global__ void bbox_partial(const T* __restrict__ pos, long n, double* __restrict__ part) {
  __shared__ double smin[3][kThreads], smax[3][kThreads];
  double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
  for (long i = blockIdx.x * (long)blockDim.x + threadIdx.x; i < n; i += (long)gridDim.x * blockDim.x)
    for (int d = 0; d < 3; ++d) {
      const double v = (double)pos[i * 3 + d];
      mn[d] = fmin(mn[d], v);
      mx[d] = fmax(mx[d], v);
    }
  for (int d = 0; d < 3; ++d) {
    smin[d][threadIdx.x] = mn[d];
    smax[d][threadIdx.x] = mx[d];
  }
  __syncthreads();
  for (int s = blockDim.x / 2; s > 0; s >>= 1) {
    if (threadIdx.x < s)
      for (int d = 0; d < 3; ++d) {
        smin[d][threadIdx.x] = fmin(smin[d][threadIdx.x], smin[d][threadIdx.x + s]);
        smax[d][threadIdx.x] = fmax(smax[d][threadIdx.x], smax[d][threadIdx.x + s]);
      }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int d = 0; d < 3; ++d) {
      part[blockIdx.x * 6 + d] = smin[d][0];
      part[blockIdx.x * 6 + 3 + d] = smax[d][0];
    }
}

__global__ void bbox_final(const double* __restrict__ part, int nb, double* __restrict__ out) {
  __shared__ double smin[3][kThreads], smax[3][kThreads];
  double mn[3] = {1e300, 1e300, 1e300}, mx[3] = {-1e300, -1e300, -1e300};
  for (int b = threadIdx.x; b < nb; b += blockDim.x)
    for (int d = 0; d < 3; ++d) {
      mn[d] = fmin(mn[d], part[b * 6 + d]);
      mx[d] = fmax(mx[d], part[b * 6 + 3 + d]);
    }
  for (int d = 0; d < 3; ++d) {
    smin[d][threadIdx.x] = mn[d];
    smax[d][threadIdx.x] = mx[d];
  }
  __syncthreads();
  for (int st = blockDim.x / 2; st > 0; st >>= 1) {
    if (threadIdx.x < st)
      for (int d = 0; d < 3; ++d) {
        smin[d][threadIdx.x] = fmin(smin[d][threadIdx.x], smin[d][threadIdx.x + st]);
        smax[d][threadIdx.x] = fmax(smax[d][threadIdx.x], smax[d][threadIdx.x + st]);
      }
    __syncthreads();
  }
  if (threadIdx.x == 0)
    for (int d = 0; d < 3; ++d) {
      out[d] = smin[d][0];
      out[3 + d] = smax[d][0];
    }
}

// ------------------------------------------------------------------ keys
// c = pos*scale + shift in the input precision, without fused multiply-add
// (pvfmm-wrapper.cpp:582-586), wrapped into [0,1); Morton coordinate
// floor(c*2^30) (mortonid.txx:39-53).  The reference wraps by adding or
// subtracting 1 until c lies in [0,1); every step but the last is exact, so
// c - floor(c) (one rounding, then 1 -> 0) is the same value and takes no
// loop for coordinates far outside a periodic box.
template <class T>
__device__ __forceinline__ T map_coord(T x, T s, T sh);
template <>
__device__ __forceinline__ double map_coord<double>(double x, double s, double sh) {
  double c = __dadd_rn(__dmul_rn(x, s), sh);
  if (!(c >= 0.0 && c < 1.0) && c == c) {
    c = __dadd_rn(c, -floor(c));
    if (c >= 1.0) c = __dadd_rn(c, -1.0);
  }
  return c;
}
template <>
__device__ __forceinline__ float map_coord<float>(float x, float s, float sh) {
  float c = __fadd_rn(__fmul_rn(x, s), sh);
  if (!(c >= 0.f && c < 1.f) && c == c) {
    c = __fadd_rn(c, -floorf(c));
    if (c >= 1.f) c = __fadd_rn(c, -1.f);
  }
  return c;
}

template <class T>
__global__ void map_and_key(const T* __restrict__ pos, long n, T scale, T sh0, T sh1, T sh2,
                            double* __restrict__ mapped, unsigned long long* __restrict__ hi,
                            unsigned int* __restrict__ lo, int* __restrict__ idx) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const T sh[3] = {sh0, sh1, sh2};
  unsigned int q[3];
  for (int d = 0; d < 3; ++d) {
    const T c = map_coord<T>(pos[i * 3 + d], scale, sh[d]);
    mapped[i * 3 + d] = (double)c;
    q[d] = (unsigned int)floor((double)c * (double)kTwo30);
  }
  const MKey k = make_key(q[0], q[1], q[2], kMaxDepth);
  hi[i] = k.hi;
  lo[i] = k.lo;
  idx[i] = (int)i;
}

__global__ void gather_u64(const unsigned long long* __restrict__ in, const int* __restrict__ perm, long n,
                           unsigned long long* __restrict__ out) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[perm[i]];
}

__global__ void assemble_keys(const unsigned long long* __restrict__ hi, const unsigned int* __restrict__ lo_unsorted,
                              const int* __restrict__ perm, long n, MKey* __restrict__ keys) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  MKey k;
  k.hi = hi[i];
  k.lo = lo_unsorted[perm[i]];
  k.pad = 0;
  keys[i] = k;
}

// ------------------------------------------------------------------ refine
// sw: point sets the source positions stand for (1 per density passed)
__global__ void refine_level(const MKey* __restrict__ cur, long n_cur, int d, const MKey* __restrict__ sk, long n_s,
                             int sw, const MKey* __restrict__ tk, long n_t, const MKey* __restrict__ gk, long n_g,
                             long max_pts, int max_depth, int* __restrict__ split) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n_cur) return;
  unsigned int X, Y, Z, dd;
  decode_key(cur[i], X, Y, Z, dd);
  int s = 0;
  if (d < max_depth - 1) {
    const MKey b = cur[i], e = node_end_key(X, Y, Z, d);
    const long g = lower_bound_key(gk, n_g, e) - lower_bound_key(gk, n_g, b);
    long c = 0;
    if (sk) c += sw * (lower_bound_key(sk, n_s, e) - lower_bound_key(sk, n_s, b));
    c += lower_bound_key(tk, n_t, e) - lower_bound_key(tk, n_t, b);
    s = (g > max_pts || c > max_pts) ? 1 : 0;
  }
  split[i] = s;
}

__global__ void make_children(const MKey* __restrict__ cur, const int* __restrict__ flag, const int* __restrict__ offs,
                              long n_cur, int d, MKey* __restrict__ next, MKey* __restrict__ internal_out) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n_cur || !flag[i]) return;
  const long k = offs[i];
  if (internal_out) internal_out[k] = cur[i];
  if (next) {
    unsigned int X, Y, Z, dd;
    decode_key(cur[i], X, Y, Z, dd);
    const unsigned int w = kTwo30 >> (d + 1);
    for (int c = 0; c < 8; ++c)
      next[k * 8 + c] = make_key(X + ((c & 1) ? w : 0), Y + ((c & 2) ? w : 0), Z + ((c & 4) ? w : 0), d + 1);
  }
}

// ------------------------------------------------------------------ balance
// For internal node X at level d: parents (level d-1) of its 3^3 neighbours
// clipped to the unit box; per axis these are parent(x) and the parent on the
// side of x within its parent.  Invalid candidates get the sentinel key.
// periodic: the mask of periodic axes (bit 0 x, bit 1 y, bit 2 z; 0 = free space)
__global__ void nbr_parents(const MKey* __restrict__ S, long n, int d, int periodic, MKey* __restrict__ out) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned int q[3], dd;
  decode_key(S[i], q[0], q[1], q[2], dd);
  const unsigned int w = kTwo30 >> d;
  const unsigned int pmask = ~((kTwo30 >> (d - 1)) - 1u);
  long cand[3][2];
  for (int a = 0; a < 3; ++a) {
    const long p0 = (long)(q[a] & pmask);
    cand[a][0] = p0;
    // the neighbour parent across the near face; outside the unit cube it
    // wraps around for periodic boundaries (NbrList, mortonid.cpp:15-55)
    long c = (q[a] & w) ? p0 + 2L * w : p0 - 2L * w;
    if (c < 0 || c >= (long)kTwo30) c = ((periodic >> a) & 1) ? (c + (long)kTwo30) % (long)kTwo30 : -1;
    cand[a][1] = c;
  }
  for (int c = 0; c < 8; ++c) {
    const long x = cand[0][c & 1], y = cand[1][(c >> 1) & 1], z = cand[2][(c >> 2) & 1];
    out[i * 8 + c] = (x < 0 || y < 0 || z < 0) ? MKey{~0ULL, ~0u, 0}
                                               : make_key((unsigned int)x, (unsigned int)y, (unsigned int)z, d - 1);
  }
}

__global__ void split_keys(const MKey* __restrict__ k, long n, unsigned long long* __restrict__ hi,
                           unsigned int* __restrict__ lo, int* __restrict__ idx) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  hi[i] = k[i].hi;
  lo[i] = k[i].lo;
  idx[i] = (int)i;
}

__global__ void unique_flags(const unsigned long long* __restrict__ hi, const unsigned int* __restrict__ lo, long n,
                             int* __restrict__ flag) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const bool sentinel = hi[i] == ~0ULL && lo[i] == ~0u;
  const bool first = i == 0 || hi[i] != hi[i - 1] || lo[i] != lo[i - 1];
  flag[i] = (first && !sentinel) ? 1 : 0;
}

__global__ void compact_keys(const unsigned long long* __restrict__ hi, const unsigned int* __restrict__ lo,
                             const int* __restrict__ flag, const int* __restrict__ offs, long n, MKey* __restrict__ out) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n || !flag[i]) return;
  MKey k;
  k.hi = hi[i];
  k.lo = lo[i];
  k.pad = 0;
  out[offs[i]] = k;
}

// ------------------------------------------------------------------ final tree
__global__ void children_of(const MKey* __restrict__ S, long n, int d, MKey* __restrict__ out) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned int X, Y, Z, dd;
  decode_key(S[i], X, Y, Z, dd);
  const unsigned int w = kTwo30 >> (d + 1);
  for (int c = 0; c < 8; ++c)
    out[i * 8 + c] = make_key(X + ((c & 1) ? w : 0), Y + ((c & 2) ? w : 0), Z + ((c & 4) ? w : 0), d + 1);
}

__global__ void member_flags(const MKey* __restrict__ keys, long n, const MKey* __restrict__ S, long nS,
                             int* __restrict__ internal) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  int f = 0;
  if (nS > 0) {
    const long p = lower_bound_key(S, nS, keys[i]);
    f = (p < nS && key_eq(S[p], keys[i])) ? 1 : 0;
  }
  internal[i] = f;
}

// Links of one level.  `cap` is the level's internal-node count known on the
// host (the size of the next level / 8 and of this level's int_idx segment);
// the scan's own total is checked against it only after the build's final
// synchronisation, so a rank k >= cap is skipped here instead of written out
// of bounds (the host check then reports the mismatch).
__global__ void level_links(const int* __restrict__ internal, const int* __restrict__ offs, long n, long base,
                            long next_base, long int_base, long cap, unsigned char* __restrict__ leaf,
                            int* __restrict__ child0, int* __restrict__ parent, int* __restrict__ int_idx) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long g = base + i;
  if (internal[i] && offs[i] < cap) {
    const long k = offs[i];
    leaf[g] = 0;
    child0[g] = (int)(next_base + 8 * k);
    int_idx[int_base + k] = (int)g;
    for (int c = 0; c < 8; ++c) parent[next_base + 8 * k + c] = (int)g;
  } else {
    leaf[g] = 1;
    child0[g] = -1;
  }
}

__global__ void node_ranges(const MKey* __restrict__ keys, long n, const MKey* __restrict__ sk, long n_s,
                            const MKey* __restrict__ tk, long n_t, int* __restrict__ slo, int* __restrict__ shi,
                            int* __restrict__ tlo, int* __restrict__ thi) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  unsigned int X, Y, Z, d;
  decode_key(keys[i], X, Y, Z, d);
  const MKey e = node_end_key(X, Y, Z, d);
  if (sk) {
    slo[i] = (int)lower_bound_key(sk, n_s, keys[i]);
    shi[i] = (int)lower_bound_key(sk, n_s, e);
  } else {
    slo[i] = shi[i] = 0;
  }
  tlo[i] = (int)lower_bound_key(tk, n_t, keys[i]);
  thi[i] = (int)lower_bound_key(tk, n_t, e);
}

// Colleague index ((z+1)*3+(y+1))*3+(x+1) (mpi_tree.txx:1143-1145).
// Colleagues (the 27 same-level cells around a node, itself included; slot
// ci = (dx+1) + 3(dy+1) + 9(dz+1)), from the parent's colleagues: the cell at
// offset d from octant c of parent P is octant (c + d) mod 2 of P's colleague
// at offset floor((c + d) / 2), which exists at this level iff that colleague
// is internal (every internal node has all 8 children in the level arrays).
// Same result as searching the level's sorted keys (interac_list.txx:98-130).
// Periodic boundaries: every colleague of the root along the periodic axes
// (mask `periodic`: bit 0 x, bit 1 y, bit 2 z) is the root itself (one image
// per slot, mpi_tree.txx:1142-1168), and the rule above then wraps the
// colleagues of every level around the unit cube along those axes.
__global__ void colleagues_kernel(long base, long n_level, const int* __restrict__ parent,
                                  const int* __restrict__ child0, int periodic, int* __restrict__ coll) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n_level) return;
  const long v = base + i;
  if (v == 0) {
    for (int ci = 0; ci < 27; ++ci) {
      const int dx = ci % 3 - 1, dy = (ci / 3) % 3 - 1, dz = ci / 9 - 1;
      const bool img = periodic && (dx == 0 || (periodic & 1)) && (dy == 0 || (periodic & 2)) &&
                       (dz == 0 || (periodic & 4));
      coll[ci] = (ci == 13 || img) ? 0 : -1;
    }
    return;
  }
  const int P = parent[v];
  const int oc = (int)(v - child0[P]);
  const int ox = oc & 1, oy = (oc >> 1) & 1, oz = (oc >> 2) & 1;
  for (int ci = 0; ci < 27; ++ci) {
    const int cx = ox + ci % 3 - 1, cy = oy + (ci / 3) % 3 - 1, cz = oz + ci / 9 - 1;  // in [-1, 2]
    const int pci = ((cx >> 1) + 1) + 3 * ((cy >> 1) + 1) + 9 * ((cz >> 1) + 1);
    const int pc = coll[(long)P * 27 + pci];
    int r = -1;
    if (pc >= 0) {
      const int c0 = child0[pc];
      if (c0 >= 0) r = c0 + ((cx & 1) | ((cy & 1) << 1) | ((cz & 1) << 2));
    }
    coll[v * 27 + ci] = r;
  }
}

// Point -> leaf map and coordinates relative to the leaf centre.
template <class Real>
__global__ void localize(const int* __restrict__ leaves, long n_leaves, const MKey* __restrict__ keys,
                         const int* __restrict__ lo, const int* __restrict__ hi, const double* __restrict__ coord,
                         Real* __restrict__ x, Real* __restrict__ y, Real* __restrict__ z, int* __restrict__ pt_leaf) {
  const long li = blockIdx.x;
  if (li >= n_leaves) return;
  const int node = leaves[li];
  if (node < 0) return;  // slot left unfilled by a count mismatch (reported by the host)
  unsigned int X, Y, Z, d;
  decode_key(keys[node], X, Y, Z, d);
  const double h = 1.0 / (double)(1u << d);
  const double c[3] = {X * (1.0 / kTwo30) + 0.5 * h, Y * (1.0 / kTwo30) + 0.5 * h, Z * (1.0 / kTwo30) + 0.5 * h};
  for (int p = lo[node] + threadIdx.x; p < hi[node]; p += blockDim.x) {
    x[p] = (Real)(coord[p * 3 + 0] - c[0]);
    y[p] = (Real)(coord[p * 3 + 1] - c[1]);
    z[p] = (Real)(coord[p * 3 + 2] - c[2]);
    pt_leaf[p] = node;
  }
}

__global__ void gather_coords(const double* __restrict__ in, const int* __restrict__ perm, long n,
                              double* __restrict__ out) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const long p = perm[i];
  out[i * 3 + 0] = in[p * 3 + 0];
  out[i * 3 + 1] = in[p * 3 + 1];
  out[i * 3 + 2] = in[p * 3 + 2];
}

// ------------------------------------------------------------------ lists
// Image of colleague c at slot ci of node v (periodic boundaries): the
// shift, in units of the unit cube, that moves c to the slot's position next
// to v, coded (sx+1) + 3(sy+1) + 9(sz+1) with s in {-1, 0, 1}; 13 = none.
// The reference stores the same shifts as coord_shift per interaction
// (fmm_pts.txx:2490-2500, 4646-4656, 4932-4942).
__device__ __forceinline__ unsigned char image_code(const MKey* keys, long v, int ci, long c) {
  unsigned int X[3], Y[3], dv, dc;
  decode_key(keys[v], X[0], X[1], X[2], dv);
  decode_key(keys[c], Y[0], Y[1], Y[2], dc);
  const long w = (long)(kTwo30 >> dv);
  const int off[3] = {ci % 3 - 1, (ci / 3) % 3 - 1, ci / 9 - 1};
  int code = 0, mul = 1;
  for (int a = 0; a < 3; ++a) {
    const long e = (long)X[a] + off[a] * w - (long)Y[a];  // a multiple of 2^30
    const int sh = e < 0 ? -1 : (e > 0 ? 1 : 0);
    code += (sh + 1) * mul;
    mul *= 3;
  }
  return (unsigned char)code;
}

// One pass per target node (n_trg > 0); `mode` 0 counts, 1 fills.
// Relative coordinates follow InteracList::BuildList (interac_list.txx:98-279).
// With image arrays (periodic boundaries) every entry also gets the image
// code of its source (U1 / U2 / W: of the node's colleague; U0 / X: of the
// parent's colleague).
__global__ void build_lists(long n_nodes, const unsigned char* __restrict__ leaf, const int* __restrict__ parent,
                            const int* __restrict__ child0, const int* __restrict__ coll, const int* __restrict__ slo,
                            const int* __restrict__ shi, const int* __restrict__ tlo, const int* __restrict__ thi,
                            long nsrf, int sw, int mode, int* __restrict__ p_cnt, int* __restrict__ x_cnt,
                            int* __restrict__ w_cnt,
                            int* __restrict__ v_cnt, const int* __restrict__ p_off, const int* __restrict__ x_off,
                            const int* __restrict__ w_off, int* __restrict__ p_list, int* __restrict__ x_list,
                            int* __restrict__ w_list, const MKey* __restrict__ keys, unsigned char* __restrict__ p_img,
                            unsigned char* __restrict__ x_img, unsigned char* __restrict__ w_img) {
  const long t = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (t >= n_nodes) return;
  const int nt = thi[t] - tlo[t];
  int np = 0, nx = 0, nw = 0, nv = 0;
  if (nt > 0) {
    const bool tleaf = leaf[t];
    const bool img = mode && p_img;
    int* pl = mode ? p_list + p_off[t] : nullptr;
    int* xl = mode ? x_list + x_off[t] : nullptr;
    int* wl = mode ? w_list + w_off[t] : nullptr;
    unsigned char* pi = img ? p_img + p_off[t] : nullptr;
    unsigned char* xi = img ? x_img + x_off[t] : nullptr;
    unsigned char* wi = img ? w_img + w_off[t] : nullptr;
    unsigned char code = 13;
#define ADD(list, cnt, v)      \
  do {                         \
    if (mode) {                \
      list[cnt] = (v);         \
      if (img) list##_img_[cnt] = code; \
    }                          \
    ++cnt;                     \
  } while (0)
    unsigned char* pl_img_ = pi;
    unsigned char* xl_img_ = xi;
    unsigned char* wl_img_ = wi;
    if (tleaf) {
      for (int ci = 0; ci < 27; ++ci) {
        const int c = coll[t * 27 + ci];
        if (c < 0) continue;
        if (img) code = image_code(keys, t, ci, c);
        if (leaf[c]) {
          if (shi[c] > slo[c]) ADD(pl, np, c);  // U1
        } else {
          for (int j = 0; j < 8; ++j) {
            const int ch = child0[c] + j;
            const int rx = (ci % 3) * 4 - 4 + ((j & 1) ? 2 : 0) - 1;
            const int ry = ((ci / 3) % 3) * 4 - 4 + ((j & 2) ? 2 : 0) - 1;
            const int rz = (ci / 9) * 4 - 4 + ((j & 4) ? 2 : 0) - 1;
            const int ns_ch = shi[ch] - slo[ch];
            if (ns_ch <= 0) continue;
            if (max(abs(rx), max(abs(ry), abs(rz))) <= 3) {
              ADD(pl, np, ch);  // U2
            } else if (leaf[ch] && (long)ns_ch * sw <= nsrf) {  // pt_cnt[0] counts each layer
              ADD(pl, np, ch);  // W handled as P2P (fmm_pts.txx:5325)
            } else {
              ADD(wl, nw, ch);  // W (fmm_pts.txx:4929)
            }
          }
        }
      }
    }
    const int p = parent[t];
    if (p >= 0) {
      int p2n = 0;
      {
        const int c0 = child0[p];
        p2n = (int)(t - c0);
      }
      for (int ci = 0; ci < 27; ++ci) {
        const int c = coll[(long)p * 27 + ci];
        if (c < 0 || !leaf[c]) continue;
        if (shi[c] <= slo[c]) continue;
        if (img) code = image_code(keys, p, ci, c);
        const int rx = (ci % 3) * 4 - 4 - ((p2n & 1) ? 2 : 0) + 1;
        const int ry = ((ci / 3) % 3) * 4 - 4 - ((p2n & 2) ? 2 : 0) + 1;
        const int rz = (ci / 9) * 4 - 4 - ((p2n & 4) ? 2 : 0) + 1;
        if (max(abs(rx), max(abs(ry), abs(rz))) <= 3) {
          if (tleaf) ADD(pl, np, c);  // U0
        } else if (tleaf && nt <= nsrf) {
          ADD(pl, np, c);  // X handled as P2P (fmm_pts.txx:5295)
        } else {
          ADD(xl, nx, c);  // X (fmm_pts.txx:4629)
        }
      }
    }
    if (!tleaf) {
      for (int ci = 0; ci < 27; ++ci) {
        if (ci == 13) continue;
        const int c = coll[t * 27 + ci];
        if (c >= 0 && !leaf[c] && shi[c] > slo[c]) ++nv;
      }
    }
#undef ADD
  }
  if (!mode) {
    p_cnt[t] = np;
    x_cnt[t] = nx;
    w_cnt[t] = nw;
    v_cnt[t] = nv;
  }
}

// V-list targets are ordered by their pattern of occupied offsets within
// windows of kVsortWindow consecutive (Morton-ordered) targets: bit o of the
// pattern is set when the target has a source parent at colleague offset o
// (the offsets of fill_vtab).  key[i] = window << 26 | pattern.
#ifndef PVFMM_VSORT_WINDOW
#define PVFMM_VSORT_WINDOW 2048
#endif
constexpr long kVsortWindow = PVFMM_VSORT_WINDOW;
__global__ void vlist_keys(const int* __restrict__ vtrg, long n_vtrg, const int* __restrict__ coll,
                           const int* __restrict__ node2vsrc, unsigned long long* __restrict__ key) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n_vtrg) return;
  const long t = vtrg[i];
  unsigned m = 0;
  for (int ci = 0, o = 0; ci < 27; ++ci) {
    if (ci == 13) continue;
    const int c = coll[t * 27 + ci];
    if (c >= 0 && node2vsrc[c] >= 0) m |= 1u << o;
    ++o;
  }
  key[i] = (unsigned long long)(i / kVsortWindow) << 26 | m;
}
// Pattern order from the sorted Morton ranks: position p takes the node of
// rank rank_sorted[p]; vmorton[rank] = p.
__global__ void vlist_reorder(const int* __restrict__ vtrg_morton, const int* __restrict__ rank_sorted, long n,
                              int* __restrict__ vtrg_sorted, int* __restrict__ vmorton) {
  const long p = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (p >= n) return;
  const int r = rank_sorted[p];
  vtrg_sorted[p] = vtrg_morton[r];
  vmorton[r] = (int)p;
}

__global__ void vlist_patterns(const unsigned long long* __restrict__ key, long n, unsigned* __restrict__ mask) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) mask[i] = (unsigned)(key[i] & ((1u << 26) - 1));
}

__global__ void fill_vtab(const int* __restrict__ vtrg, long n_vtrg, const int* __restrict__ coll,
                          const int* __restrict__ node2vsrc, int* __restrict__ vtab) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n_vtrg) return;
  const long t = vtrg[i];
  for (int ci = 0, o = 0; ci < 27; ++ci) {
    if (ci == 13) continue;
    const int c = coll[t * 27 + ci];
    vtab[(long)o * n_vtrg + i] = (c >= 0) ? node2vsrc[c] : -1;  // offset-major: coalesced per offset
    ++o;
  }
}

template <class Pred>
__global__ void flag_nodes(long n, Pred pred, int* __restrict__ flag) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) flag[i] = pred(i) ? 1 : 0;
}

// out[offs[i]] = i for flagged i; ranks >= cap (the capacity of out) are
// skipped, so a count that disagrees with the host's expectation (checked
// after the build's final synchronisation) never writes out of bounds.
__global__ void compact_index(const int* __restrict__ flag, const int* __restrict__ offs, long n, long cap,
                              int* __restrict__ out, int* __restrict__ map) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const bool f = flag[i] && offs[i] < cap;
  if (f) out[offs[i]] = (int)i;
  if (map) map[i] = f ? offs[i] : -1;
}

__global__ void gather_u32(const unsigned int* __restrict__ in, const int* __restrict__ perm, long n,
                           unsigned int* __restrict__ out) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) out[i] = in[perm[i]];
}

__global__ void iota_kernel(int* __restrict__ a, long n) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) a[i] = (int)i;
}

// Pinned host slots of a tree build (ctx.chk): the deferred counts, two
// slots for the totals read back at once, and 12 doubles of bounding boxes.
constexpr int kChkLists = 40, kChkLeaves = 48, kChkScan = 60, kChkSlots = 64;
constexpr size_t kChkBytes = kChkSlots * sizeof(int) + 12 * sizeof(double);
inline double* chk_bbox(Context& ctx) { return reinterpret_cast<double*>(ctx.chk + kChkSlots); }

// Exclusive prefix sum of n ints; returns the total (synchronous read through
// pinned slots).
long exclusive_scan(Context& ctx, const int* in, int* out, long n) {
  if (n <= 0) return 0;
  size_t bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, (int)n, ctx.stream);
  void* tmp = ctx.scratch2.ensure(bytes);
  cub::DeviceScan::ExclusiveSum(tmp, bytes, in, out, (int)n, ctx.stream);
  int* h = ctx.chk + kChkScan;
  PVFMM_CUDA_CHECK(cudaMemcpyAsync(&h[0], out + n - 1, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
  PVFMM_CUDA_CHECK(cudaMemcpyAsync(&h[1], in + n - 1, sizeof(int), cudaMemcpyDeviceToHost, ctx.stream));
  PVFMM_CUDA_CHECK(cudaStreamSynchronize(ctx.stream));
  return (long)h[0] + h[1];
}

// Pinned count slots of a tree build: [0, kMaxDepth] internal nodes per level,
// then the compacted list sizes and the leaf count.
static_assert(kMaxDepth < kChkLists, "per-level slots overlap the list slots");

// Exclusive prefix sum of n ints without reading the total back; the total
// (out[n-1] + in[n-1]) is copied into the pinned slot *slot (valid after the
// stream's next synchronisation) and, with `close`, also stored as out[n].
__global__ void scan_total(const int* __restrict__ in, int* __restrict__ out, long n, int* __restrict__ slot,
                           bool close) {
  const int t = out[n - 1] + in[n - 1];
  *slot = t;
  if (close) out[n] = t;
}

void exclusive_scan_deferred(Context& ctx, const int* in, int* out, long n, int* slot, bool close = false) {
  if (n <= 0) {
    *slot = 0;
    return;
  }
  size_t bytes = 0;
  cub::DeviceScan::ExclusiveSum(nullptr, bytes, in, out, (int)n, ctx.stream);
  void* tmp = ctx.scratch2.ensure(bytes);
  cub::DeviceScan::ExclusiveSum(tmp, bytes, in, out, (int)n, ctx.stream);
  ++ctx.n_launch;
  scan_total<<<1, 1, 0, ctx.stream>>>(in, out, n, slot, close);
}

// Stable sort of 96-bit keys (hi, lo): by lo, then stably by hi.  On return
// perm[i] is the input position of the i-th smallest key and hs/ls hold the
// sorted halves.  Uses temporaries t[base..base+2].
void sort_hilo(Context& ctx, long n, const unsigned long long* hi, const unsigned int* lo, unsigned long long* hs,
               unsigned int* ls, int* perm, int base) {
  auto& s = ctx.stream;
  int* idx = ctx.t[base].as<int>(n);
  int* p1 = ctx.t[base + 1].as<int>(n);
  unsigned long long* hg = ctx.t[base + 2].as<unsigned long long>(n);
  ++ctx.n_launch;
  iota_kernel<<<ceil_div(n, kThreads), kThreads, 0, s>>>(idx, n);
  size_t b1 = 0, b2 = 0;
  cub::DeviceRadixSort::SortPairs(nullptr, b1, lo, ls, idx, p1, (int)n, 0, 32, s);
  cub::DeviceRadixSort::SortPairs(nullptr, b2, hg, hs, p1, perm, (int)n, 0, 64, s);
  void* tmp = ctx.scratch.ensure(std::max(b1, b2));
  cub::DeviceRadixSort::SortPairs(tmp, b1, lo, ls, idx, p1, (int)n, 0, 32, s);
  ++ctx.n_launch;
  gather_u64<<<ceil_div(n, kThreads), kThreads, 0, s>>>(hi, p1, n, hg);
  cub::DeviceRadixSort::SortPairs(tmp, b2, hg, hs, p1, perm, (int)n, 0, 64, s);
  ++ctx.n_launch;
  gather_u32<<<ceil_div(n, kThreads), kThreads, 0, s>>>(lo, perm, n, ls);
}

__global__ void unique_flags_hi(const unsigned long long* __restrict__ hi, long n, int* __restrict__ flag) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  flag[i] = (hi[i] != ~0ULL && (i == 0 || hi[i] != hi[i - 1])) ? 1 : 0;
}

__global__ void compact_keys_hi(const unsigned long long* __restrict__ hi, const int* __restrict__ flag,
                                const int* __restrict__ offs, long n, unsigned int lo, MKey* __restrict__ out) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i >= n || !flag[i]) return;
  MKey k;
  k.hi = hi[i];
  k.lo = lo;
  k.pad = 0;
  out[offs[i]] = k;
}

__global__ void key_hi(const MKey* __restrict__ k, long n, unsigned long long* __restrict__ hi) {
  const long i = blockIdx.x * (long)blockDim.x + threadIdx.x;
  if (i < n) hi[i] = k[i].hi;
}

// Sorts node keys of one depth and removes duplicates and sentinels; returns
// the count.  A node of depth L <= 21 has zero coordinate bits below 30 - L,
// so its key is hi (top 3L bits of the 63-bit interleave) with lo = L: one
// keys-only radix sort over those bits (and bit 63, which only the sentinels
// set) orders them.  Deeper levels use the full 96-bit sort.
long sort_unique(Context& ctx, const MKey* in, long n, DevBuf& out, int depth) {
  auto& s = ctx.stream;
  if (n == 0) return 0;
  if (depth <= 21) {
    unsigned long long* h = ctx.t[10].as<unsigned long long>(n);
    unsigned long long* hs = ctx.t[13].as<unsigned long long>(n);
    ++ctx.n_launch;
    key_hi<<<ceil_div(n, kThreads), kThreads, 0, s>>>(in, n, h);
    const int begin_bit = 3 * (21 - depth);
    size_t bytes = 0;
    cub::DeviceRadixSort::SortKeys(nullptr, bytes, h, hs, (int)n, begin_bit, 64, s);
    void* tmp = ctx.scratch.ensure(bytes);
    cub::DeviceRadixSort::SortKeys(tmp, bytes, h, hs, (int)n, begin_bit, 64, s);
    int* fl = ctx.t[19].as<int>(n);
    int* of = ctx.t[20].as<int>(n);
    ++ctx.n_launch;
    unique_flags_hi<<<ceil_div(n, kThreads), kThreads, 0, s>>>(hs, n, fl);
    const long cnt = exclusive_scan(ctx, fl, of, n);
    MKey* o = out.as<MKey>(std::max(cnt, 1L));
    ++ctx.n_launch;
    compact_keys_hi<<<ceil_div(n, kThreads), kThreads, 0, s>>>(hs, fl, of, n, (unsigned int)depth, o);
    return cnt;
  }
  unsigned long long* h = ctx.t[10].as<unsigned long long>(n);
  unsigned int* l = ctx.t[11].as<unsigned int>(n);
  int* ix = ctx.t[12].as<int>(n);
  ++ctx.n_launch;
  split_keys<<<ceil_div(n, kThreads), kThreads, 0, s>>>(in, n, h, l, ix);
  unsigned long long* hs = ctx.t[13].as<unsigned long long>(n);
  unsigned int* ls = ctx.t[14].as<unsigned int>(n);
  int* perm = ctx.t[15].as<int>(n);
  sort_hilo(ctx, n, h, l, hs, ls, perm, 16);
  int* fl = ctx.t[19].as<int>(n);
  int* of = ctx.t[20].as<int>(n);
  ++ctx.n_launch;
  unique_flags<<<ceil_div(n, kThreads), kThreads, 0, s>>>(hs, ls, n, fl);
  const long cnt = exclusive_scan(ctx, fl, of, n);
  MKey* o = out.as<MKey>(std::max(cnt, 1L));
  ++ctx.n_launch;
  compact_keys<<<ceil_div(n, kThreads), kThreads, 0, s>>>(hs, ls, fl, of, n, o);
  return cnt;
}

// Sorts mapped points: perm (sorted -> input), sorted keys, sorted coords.
void sort_point_set(Context& ctx, long n, const unsigned long long* hi, const unsigned int* lo, const double* mapped,
                    DevBuf& perm_out, DevBuf& keys_out, DevBuf& coord_out) {
  auto& s = ctx.stream;
  unsigned long long* hs = ctx.t[5].as<unsigned long long>(n);
  unsigned int* ls = ctx.t[6].as<unsigned int>(n);
  int* perm = perm_out.as<int>(n);
  sort_hilo(ctx, n, hi, lo, hs, ls, perm, 16);
  MKey* keys = keys_out.as<MKey>(n);
  ++ctx.n_launch;
  assemble_keys<<<ceil_div(n, kThreads), kThreads, 0, s>>>(hs, lo, perm, n, keys);
  double* c = coord_out.as<double>(n * 3);
  ++ctx.n_launch;
  gather_coords<<<ceil_div(n, kThreads), kThreads, 0, s>>>(mapped, perm, n, c);
}

// Reference bounding-box rule (pvfmm-wrapper.cpp:469-520) in precision Real.
template <class Real>
void bbox_scale_shift(const double* bs, const double* bt, double& scale_out, double* shift_out) {
  const Real eps = std::numeric_limits<Real>::epsilon() * (Real)64;
  auto one = [&](const double* b, Real& sc, Real* sh) {
    const double* mn = b;
    const double* mx = b + 3;
    sc = (Real)1 / (Real)(mx[0] - mn[0] + 2 * (double)eps);
    for (int k = 0; k < 3; ++k) sc = std::min(sc, (Real)(1.0 / (mx[k] - mn[k] + 2 * (double)eps)));
    if (sc * (Real)0 != (Real)0) sc = (Real)1;
    for (int k = 0; k < 3; ++k) sh[k] = (Real)(-mn[k]) * sc + eps;
  };
  Real s0, x0[3], s1, x1[3];
  one(bs, s0, x0);
  one(bt, s1, x1);
  Real c0[3], c1[3];
  for (int k = 0; k < 3; ++k) {
    c0[k] = (Real)(0.5 - (double)x0[k]) / s0;
    c1[k] = (Real)(0.5 - (double)x1[k]) / s1;
  }
  Real sc = 0;
  for (int k = 0; k < 3; ++k) sc = std::max(sc, (Real)std::fabs(c0[k] - c1[k]));
  sc = (Real)1 / (sc + (Real)1 / s0 + (Real)1 / s1);
  scale_out = (double)sc;
  for (int k = 0; k < 3; ++k) shift_out[k] = (double)((Real)0.5 - (c0[k] + c1[k]) * sc / (Real)2);
}

template <class T>
void point_bbox(Context& ctx, const T* pos, long n, double* host6) {
  const int nb = (int)std::min<long>(1024, std::max<long>(1, ceil_div(n, kThreads)));
  double* part = ctx.t[0].as<double>((size_t)nb * 6 + 6);
  ++ctx.n_launch;
  bbox_partial<T><<<nb, kThreads, 0, ctx.stream>>>(pos, n, part);
  ++ctx.n_launch;
  bbox_final<<<1, kThreads, 0, ctx.stream>>>(part, nb, part + (size_t)nb * 6);
  // host6: pinned; the caller synchronises
  PVFMM_CUDA_CHECK(cudaMemcpyAsync(host6, part + (size_t)nb * 6, 6 * sizeof(double), cudaMemcpyDeviceToHost, ctx.stream));
}

template <class T>
void map_points(Context& ctx, const T* pos, long n, double scale, const double* shift, DevBuf& mapped,
                DevBuf& hi, DevBuf& lo) {
  double* mp = mapped.as<double>(n * 3);
  unsigned long long* h = hi.as<unsigned long long>(n);
  unsigned int* l = lo.as<unsigned int>(n);
  int* idx = ctx.t[4].as<int>(n);
  ++ctx.n_launch;
  map_and_key<T><<<ceil_div(n, kThreads), kThreads, 0, ctx.stream>>>(pos, n, (T)scale, (T)shift[0], (T)shift[1],
                                                                      (T)shift[2], mp, h, l, idx);
}

}  // namespace

// Seed grid of the context's initial tree (pvfmm-wrapper.cpp:416-432), as
// sorted Morton keys, in the precision of the context.
static std::vector<MKey> seed_grid_keys(int max_pts, bool real_float) {
  std::vector<MKey> keys;
  long NN;
  if (real_float) NN = (long)std::ceil(std::pow((float)max_pts, 1.0 / 3.0));
  else NN = (long)std::ceil(std::pow((double)max_pts, 1.0 / 3.0));
  keys.reserve(NN * NN * NN);
  for (long i = 0; i < NN * NN * NN; ++i) {
    unsigned int q[3];
    const long comp[3] = {i % NN, (i / NN) % NN, (i / (NN * NN)) % NN};
    for (int d = 0; d < 3; ++d) {
      if (real_float) {
        const float c = (float)((float)comp[d] + 0.5f) / (float)NN;
        q[d] = (unsigned int)std::floor((double)c * (double)kTwo30);
      } else {
        const double c = ((double)comp[d] + 0.5) / (double)NN;
        q[d] = (unsigned int)std::floor(c * (double)kTwo30);
      }
    }
    keys.push_back(make_key(q[0], q[1], q[2], kMaxDepth));
  }
  std::sort(keys.begin(), keys.end(), [](const MKey& a, const MKey& b) { return key_less(a, b); });
  return keys;
}

void build_tree(Context& ctx, const void* src_pos, long n_src, const void* trg_pos, long n_trg, bool pos_float,
                int src_weight, bool trg_alias) {
  if (n_src < 1 || n_trg < 1) throw std::runtime_error("build_tree needs at least one source and one target");
  if (!ctx.chk) PVFMM_CUDA_CHECK(cudaMallocHost((void**)&ctx.chk, kChkBytes));
  DevTree& T = ctx.tree;
  auto& s = ctx.stream;
  T.valid = false;
  T.n_src = n_src;
  T.n_trg = n_trg;
  T.src_weight = n_src > 0 ? src_weight : 0;
  T.src_counted = T.src_weight > 0;
  // 1. bounding box and map (both boxes read back with one synchronisation)
  double* bs = chk_bbox(ctx);
  double* bt = bs + 6;
  if (pos_float) {
    point_bbox<float>(ctx, (const float*)src_pos, n_src, bs);
    if (!trg_alias) point_bbox<float>(ctx, (const float*)trg_pos, n_trg, bt);
  } else {
    point_bbox<double>(ctx, (const double*)src_pos, n_src, bs);
    if (!trg_alias) point_bbox<double>(ctx, (const double*)trg_pos, n_trg, bt);
  }
  PVFMM_CUDA_CHECK(cudaStreamSynchronize(ctx.stream));
  if (trg_alias) std::copy(bs, bs + 6, bt);
  if (!ctx.unit_box && !ctx.periodic) {
    if (pos_float) bbox_scale_shift<float>(bs, bt, T.scale_x, T.shift_x);
    else bbox_scale_shift<double>(bs, bt, T.scale_x, T.shift_x);
  }
  if (ctx.periodic) {
    // periodic boundaries (pvfmm-wrapper.cpp:512-517): scale 1 / box_size in
    // the interface precision, no shift; the mapping wraps into [0,1)
    T.scale_x = pos_float ? (double)(1.0f / (float)ctx.box_size) : 1.0 / ctx.box_size;
    T.shift_x[0] = T.shift_x[1] = T.shift_x[2] = 0.0;
  } else if (ctx.unit_box) {
    // C++ interface (include/pvfmm.txx:216-244): coordinates are used as
    // given, so they must lie in the unit cube.
    for (const double* b : {bs, bt})
      for (int k = 0; k < 3; ++k)
        if (!(b[k] >= 0.0) || !(b[3 + k] < 1.0))
          throw std::runtime_error("coordinates must lie in [0,1)^3 for a unit-box tree");
    T.scale_x = 1.0;
    T.shift_x[0] = T.shift_x[1] = T.shift_x[2] = 0.0;
  }
  DevBuf& src_mapped = ctx.t[1];
  DevBuf& trg_mapped = ctx.t[2];
  DevBuf& hi = ctx.t[7];
  DevBuf& lo = ctx.t[8];
  DevBuf& coords_s = ctx.t[21];
  DevBuf& coords_t = ctx.t[22];
  // 2. sources
  if (pos_float) map_points<float>(ctx, (const float*)src_pos, n_src, T.scale_x, T.shift_x, src_mapped, hi, lo);
  else map_points<double>(ctx, (const double*)src_pos, n_src, T.scale_x, T.shift_x, src_mapped, hi, lo);
  sort_point_set(ctx, n_src, hi.get<unsigned long long>(), lo.get<unsigned int>(), src_mapped.get<double>(),
                 T.src_perm, T.src_key, coords_s);
  // 3. targets
  if (trg_alias) {
    PVFMM_CUDA_CHECK(cudaMemcpyAsync(T.trg_perm.as<int>(n_src), T.src_perm.get<int>(), n_src * sizeof(int),
                                     cudaMemcpyDeviceToDevice, s));
    PVFMM_CUDA_CHECK(cudaMemcpyAsync(T.trg_key.as<MKey>(n_src), T.src_key.get<MKey>(), n_src * sizeof(MKey),
                                     cudaMemcpyDeviceToDevice, s));
    PVFMM_CUDA_CHECK(cudaMemcpyAsync(coords_t.as<double>(n_src * 3), coords_s.get<double>(), n_src * 3 * sizeof(double),
                                     cudaMemcpyDeviceToDevice, s));
  } else {
    if (pos_float) map_points<float>(ctx, (const float*)trg_pos, n_trg, T.scale_x, T.shift_x, trg_mapped, hi, lo);
    else map_points<double>(ctx, (const double*)trg_pos, n_trg, T.scale_x, T.shift_x, trg_mapped, hi, lo);
    sort_point_set(ctx, n_trg, hi.get<unsigned long long>(), lo.get<unsigned int>(), trg_mapped.get<double>(),
                   T.trg_perm, T.trg_key, coords_t);
  }
  // 4. the tree's point set: the seed grid of the C interface, or the
  //    targets for a unit-box tree (pt_coord = trg_coord, pvfmm.txx:238)
  const MKey* sk = T.src_counted ? T.src_key.get<MKey>() : nullptr;
  const MKey* tk = T.trg_key.get<MKey>();
  std::vector<MKey> gk;
  const MKey* d_gk = tk;
  long n_gk = n_trg;
  if (!ctx.unit_box) {
    gk = seed_grid_keys(ctx.max_pts, pos_float);
    MKey* g = ctx.t[9].as<MKey>(gk.size());
    PVFMM_CUDA_CHECK(cudaMemcpyAsync(g, gk.data(), gk.size() * sizeof(MKey), cudaMemcpyHostToDevice, s));
    d_gk = g;
    n_gk = (long)gk.size();
  }
  // 5. refinement, level by level
  std::vector<long> nR;
  {
    // two persistent level buffers (no allocation in steady state)
    DevBuf* cur_b = &ctx.t[16];
    DevBuf* next_b = &ctx.t[17];
    MKey root = make_key(0, 0, 0, 0);
    PVFMM_CUDA_CHECK(cudaMemcpyAsync(cur_b->as<MKey>(1), &root, sizeof(MKey), cudaMemcpyHostToDevice, s));
    long n_cur = 1;
    int d = 0;
    while (n_cur > 0) {
      int* split = ctx.t[3].as<int>(n_cur);
      int* offs = ctx.t[23].as<int>(n_cur);
      ++ctx.n_launch;
      refine_level<<<ceil_div(n_cur, kThreads), kThreads, 0, s>>>(cur_b->get<MKey>(), n_cur, d, sk, T.n_src,
                                                                   T.src_weight, tk, T.n_trg, d_gk, n_gk,
                                                                   ctx.max_pts, kMaxDepth, split);
      const long n_split = exclusive_scan(ctx, split, offs, n_cur);
      if (n_split == 0) break;
      if ((long)ctx.lvlR.size() <= d) ctx.lvlR.resize(d + 1);
      MKey* R = ctx.lvlR[d].as<MKey>(n_split);
      MKey* next = next_b->as<MKey>(n_split * 8);
      ++ctx.n_launch;
      make_children<<<ceil_div(n_cur, kThreads), kThreads, 0, s>>>(cur_b->get<MKey>(), split, offs, n_cur, d, next, R);
      nR.push_back(n_split);
      std::swap(cur_b, next_b);
      n_cur = n_split * 8;
      ++d;
    }
  }
  const int dint = (int)nR.size() - 1;  // deepest level with internal nodes (-1: root is a leaf)
  // 6. 2:1 balance closure
  std::vector<long> nS(std::max(dint + 1, 0), 0);
  if ((long)ctx.lvlS.size() < dint + 1) ctx.lvlS.resize(dint + 1);
  if (dint >= 0) {
    PVFMM_CUDA_CHECK(cudaMemcpyAsync(ctx.lvlS[dint].as<MKey>(nR[dint]), ctx.lvlR[dint].get<MKey>(),
                                     nR[dint] * sizeof(MKey), cudaMemcpyDeviceToDevice, s));
    nS[dint] = nR[dint];
    for (int d = dint; d >= 1; --d) {
      const long nc = nR[d - 1] + 8 * nS[d];
      MKey* cand = ctx.t[9].as<MKey>(nc);
      PVFMM_CUDA_CHECK(cudaMemcpyAsync(cand, ctx.lvlR[d - 1].get<MKey>(), nR[d - 1] * sizeof(MKey),
                                       cudaMemcpyDeviceToDevice, s));
      ++ctx.n_launch;
      nbr_parents<<<ceil_div(nS[d], kThreads), kThreads, 0, s>>>(ctx.lvlS[d].get<MKey>(), nS[d], d,
                                                                 ctx.periodic ? ctx.periodic_axes : 0,
                                                                 cand + nR[d - 1]);
      nS[d - 1] = sort_unique(ctx, cand, nc, ctx.lvlS[d - 1], d - 1);
    }
  }
  // 7. final node arrays
  const int D = dint + 1;  // deepest level
  T.depth = D;
  T.level_off.assign(D + 2, 0);
  T.n_internal.assign(D + 1, 0);
  T.level_off[0] = 0;
  T.level_off[1] = 1;
  for (int d = 1; d <= D; ++d) T.level_off[d + 1] = T.level_off[d] + 8 * nS[d - 1];
  const long N = T.level_off[D + 1];
  T.n_nodes = N;
  MKey* keys = T.key.as<MKey>(N);
  unsigned char* leaf = T.leaf.as<unsigned char>(N);
  int* parent = T.parent.as<int>(N);
  int* child0 = T.child0.as<int>(N);
  long n_int_total = 0;
  for (int d = 0; d < D; ++d) n_int_total += nS[d];
  int* int_idx = T.int_idx.as<int>(std::max(n_int_total, 1L));
  T.int_off.assign(D + 1, 0);
  {
    MKey root = make_key(0, 0, 0, 0);
    PVFMM_CUDA_CHECK(cudaMemcpyAsync(keys, &root, sizeof(MKey), cudaMemcpyHostToDevice, s));
    const int minus1 = -1;
    PVFMM_CUDA_CHECK(cudaMemcpyAsync(parent, &minus1, sizeof(int), cudaMemcpyHostToDevice, s));
  }
  long int_base = 0;
  for (int d = 0; d <= D; ++d) {
    const long base = T.level_off[d], nl = T.level_off[d + 1] - base;
    if (d > 0) ++ctx.n_launch;
    if (d > 0) children_of<<<ceil_div(nS[d - 1], kThreads), kThreads, 0, s>>>(ctx.lvlS[d - 1].get<MKey>(), nS[d - 1],
                                                                              d - 1, keys + base);
    int* internal = ctx.t[3].as<int>(nl);
    int* offs = ctx.t[23].as<int>(nl);
    const long nSd = d < D ? nS[d] : 0;
    ++ctx.n_launch;
    member_flags<<<ceil_div(nl, kThreads), kThreads, 0, s>>>(keys + base, nl, d < D ? ctx.lvlS[d].get<MKey>() : nullptr,
                                                             nSd, internal);
    // the count is known (nSd); the scan's total is checked after the build's
    // final synchronisation instead of waiting for it here
    exclusive_scan_deferred(ctx, internal, offs, nl, ctx.chk + d);
    const long nint = nSd;
    T.n_internal[d] = nint;
    T.int_off[d] = int_base;
    ++ctx.n_launch;
    level_links<<<ceil_div(nl, kThreads), kThreads, 0, s>>>(internal, offs, nl, base, T.level_off[d + 1], int_base,
                                                            nSd, leaf, child0, parent, int_idx);
    int_base += nint;
  }
  // 8. point ranges and colleagues
  int* slo = T.src_lo.as<int>(N);
  int* shi = T.src_hi.as<int>(N);
  int* tlo = T.trg_lo.as<int>(N);
  int* thi = T.trg_hi.as<int>(N);
  ++ctx.n_launch;
  node_ranges<<<ceil_div(N, kThreads), kThreads, 0, s>>>(keys, N, sk, T.n_src, tk, T.n_trg, slo, shi, tlo, thi);
  int* coll = T.colleague.as<int>(N * 27);
  for (int d = 0; d <= D; ++d) {
    const long base = T.level_off[d], nl = T.level_off[d + 1] - base;
    ++ctx.n_launch;
    colleagues_kernel<<<ceil_div(nl, kThreads), kThreads, 0, s>>>(base, nl, parent, child0,
                                                                   ctx.periodic ? ctx.periodic_axes : 0, coll);
  }
  // 9. compact node lists.  The compacted lists are sized for all N nodes so
  //    that the eight counts are read back together at one synchronisation.
  {
    int* flag = ctx.t[3].as<int>(N);
    int* offs = ctx.t[23].as<int>(N);
    int* cnt = ctx.chk + kChkLists;  // sleaf tleaf vsrc p2p x w xtrg vtrg
    auto compact = [&](auto pred, DevBuf& out, int* map, int* slot) {
      ++ctx.n_launch;
      flag_nodes<<<ceil_div(N, kThreads), kThreads, 0, s>>>(N, pred, flag);
      exclusive_scan_deferred(ctx, flag, offs, N, slot);
      int* o = out.as<int>(N);
      ++ctx.n_launch;
      compact_index<<<ceil_div(N, kThreads), kThreads, 0, s>>>(flag, offs, N, N, o, map);
    };
    compact([=] __device__(long i) { return leaf[i] && shi[i] > slo[i]; }, T.sleaf, nullptr, cnt + 0);
    compact([=] __device__(long i) { return leaf[i] && thi[i] > tlo[i]; }, T.tleaf, nullptr, cnt + 1);
    int* n2v = T.node2vsrc.as<int>(N);
    compact([=] __device__(long i) { return !leaf[i] && shi[i] > slo[i]; }, T.vsrc, n2v, cnt + 2);
    // lists: count
    int* pc = ctx.t[4].as<int>(N);
    int* xc = ctx.t[5].as<int>(N);
    int* wc = ctx.t[6].as<int>(N);
    int* vc = ctx.t[0].as<int>(N);
    const long nsrf = ctx.ns;
    ++ctx.n_launch;
    build_lists<<<ceil_div(N, 128), 128, 0, s>>>(N, leaf, parent, child0, coll, slo, shi, tlo, thi, nsrf,
                                                 T.src_weight, 0, pc, xc, wc, vc, nullptr, nullptr, nullptr, nullptr,
                                                 nullptr, nullptr, keys, nullptr, nullptr, nullptr);
    int* po = T.p_off.as<int>(N + 1);
    int* xo = T.x_off.as<int>(N + 1);
    int* wo = T.w_off.as<int>(N + 1);
    exclusive_scan_deferred(ctx, pc, po, N, cnt + 3, true);
    exclusive_scan_deferred(ctx, xc, xo, N, cnt + 4, true);
    exclusive_scan_deferred(ctx, wc, wo, N, cnt + 5, true);
    compact([=] __device__(long i) { return xc[i] > 0; }, T.xtrg, nullptr, cnt + 6);
    compact([=] __device__(long i) { return vc[i] > 0; }, T.vtrg, nullptr, cnt + 7);
    PVFMM_CUDA_CHECK(cudaStreamSynchronize(s));
    T.n_sleaf = cnt[0];
    T.n_tleaf = cnt[1];
    T.n_vsrc = cnt[2];
    T.n_p2p = cnt[3];
    T.n_x = cnt[4];
    T.n_w = cnt[5];
    T.n_xtrg = cnt[6];
    T.n_vtrg = cnt[7];
    int* pl = T.p_list.as<int>(std::max(T.n_p2p, 1L));
    int* xl = T.x_list.as<int>(std::max(T.n_x, 1L));
    int* wl = T.w_list.as<int>(std::max(T.n_w, 1L));
    unsigned char* pim = ctx.periodic ? T.p_img.as<unsigned char>(std::max(T.n_p2p, 1L)) : nullptr;
    unsigned char* xim = ctx.periodic ? T.x_img.as<unsigned char>(std::max(T.n_x, 1L)) : nullptr;
    unsigned char* wim = ctx.periodic ? T.w_img.as<unsigned char>(std::max(T.n_w, 1L)) : nullptr;
    ++ctx.n_launch;
    build_lists<<<ceil_div(N, 128), 128, 0, s>>>(N, leaf, parent, child0, coll, slo, shi, tlo, thi, nsrf,
                                                 T.src_weight, 1, nullptr, nullptr, nullptr, nullptr, po, xo, wo, pl,
                                                 xl, wl, keys, pim, xim, wim);
    int* vt = T.vtab.as<int>(std::max(T.n_vtrg, 1L) * 26);
    unsigned* vm = T.vmask.as<unsigned>(std::max(T.n_vtrg, 1L));
    if (T.n_vtrg > 0) {
      // V-list targets ordered by their pattern of occupied offsets within
      // windows of Morton order (stable: Morton order within a pattern), so
      // that the Hadamard kernels can skip the offsets that are empty for all
      // the parents of a tile while a block's parents stay close in space.
      // Every target is computed independently: the order changes no value.
      // The sort carries each target's Morton rank: vmorton[rank] is the
      // target's position in the pattern order (ranks and positions stay
      // within the same window, so windows of Morton order are contiguous
      // ranges of positions too).
      unsigned long long* key = ctx.t[10].as<unsigned long long>(T.n_vtrg);
      unsigned long long* keys_sorted = ctx.t[13].as<unsigned long long>(T.n_vtrg);
      int* vs = ctx.t[11].as<int>(T.n_vtrg);
      int* rank_in = ctx.t[12].as<int>(T.n_vtrg);
      int* rank_sorted = ctx.t[14].as<int>(T.n_vtrg);
      ++ctx.n_launch;
      vlist_keys<<<ceil_div(T.n_vtrg, kThreads), kThreads, 0, s>>>(T.vtrg.get<int>(), T.n_vtrg, coll, n2v, key);
      ++ctx.n_launch;
      iota_kernel<<<ceil_div(T.n_vtrg, kThreads), kThreads, 0, s>>>(rank_in, T.n_vtrg);
      int end_bit = 27;
      while (end_bit < 64 && ((T.n_vtrg - 1) / kVsortWindow) >> (end_bit - 26)) ++end_bit;
      size_t bytes = 0;
      cub::DeviceRadixSort::SortPairs(nullptr, bytes, key, keys_sorted, rank_in, rank_sorted, (int)T.n_vtrg, 0,
                                      end_bit, s);
      void* tmp = ctx.scratch.ensure(bytes);
      cub::DeviceRadixSort::SortPairs(tmp, bytes, key, keys_sorted, rank_in, rank_sorted, (int)T.n_vtrg, 0, end_bit,
                                      s);
      int* vmorton = T.vmorton.as<int>(T.n_vtrg);
      ++ctx.n_launch;
      vlist_reorder<<<ceil_div(T.n_vtrg, kThreads), kThreads, 0, s>>>(T.vtrg.get<int>(), rank_sorted, T.n_vtrg, vs,
                                                                      vmorton);
      PVFMM_CUDA_CHECK(cudaMemcpyAsync(T.vtrg.get<int>(), vs, T.n_vtrg * sizeof(int), cudaMemcpyDeviceToDevice, s));
      T.vtiles_valid = false;
      ++ctx.n_launch;
      vlist_patterns<<<ceil_div(T.n_vtrg, kThreads), kThreads, 0, s>>>(keys_sorted, T.n_vtrg, vm);
      ++ctx.n_launch;
      fill_vtab<<<ceil_div(T.n_vtrg, kThreads), kThreads, 0, s>>>(T.vtrg.get<int>(), T.n_vtrg, coll, n2v, vt);
    }
  }
  // 10. point -> leaf and local coordinates
  {
    const long n_leaves_all = N - n_int_total;
    int* flag = ctx.t[3].as<int>(N);
    int* offs = ctx.t[23].as<int>(N);
    ++ctx.n_launch;
    flag_nodes<<<ceil_div(N, kThreads), kThreads, 0, s>>>(N, [=] __device__(long i) { return leaf[i] != 0; }, flag);
    // the leaf count is known; the scan's total is checked at the end
    exclusive_scan_deferred(ctx, flag, offs, N, ctx.chk + kChkLeaves);
    const long nl = n_leaves_all;
    int* leaves = ctx.t[0].as<int>(std::max(nl, 1L));
    // -1 marks a slot that no leaf filled (a count mismatch, reported below)
    PVFMM_CUDA_CHECK(cudaMemsetAsync(leaves, 0xff, std::max(nl, 1L) * sizeof(int), s));
    ++ctx.n_launch;
    compact_index<<<ceil_div(N, kThreads), kThreads, 0, s>>>(flag, offs, N, nl, leaves, nullptr);
    double* sx = T.sx.as<double>(std::max(T.n_src, 1L));
    double* sy = T.sy.as<double>(std::max(T.n_src, 1L));
    double* sz = T.sz.as<double>(std::max(T.n_src, 1L));
    double* tx = T.tx.as<double>(std::max(T.n_trg, 1L));
    double* ty = T.ty.as<double>(std::max(T.n_trg, 1L));
    double* tz = T.tz.as<double>(std::max(T.n_trg, 1L));
    int* sl = T.src_leaf.as<int>(std::max(T.n_src, 1L));
    int* tl = T.trg_leaf.as<int>(std::max(T.n_trg, 1L));
    if (nl > 0) {
      // source coordinates are localized even when sl_den is NULL (unused then)
      ++ctx.n_launch;
      localize<double><<<nl, 128, 0, s>>>(leaves, nl, keys, slo, shi, coords_s.get<double>(), sx, sy, sz, sl);
      ++ctx.n_launch;
      localize<double><<<nl, 128, 0, s>>>(leaves, nl, keys, tlo, thi, coords_t.get<double>(), tx, ty, tz, tl);
    }
  }
  PVFMM_CUDA_CHECK(cudaStreamSynchronize(s));
  PVFMM_CUDA_CHECK(cudaGetLastError());
  for (int d = 0; d <= D; ++d)
    if (ctx.chk[d] != (int)T.n_internal[d]) throw std::runtime_error("octree build: balanced internal set is not closed");
  if (ctx.chk[kChkLeaves] != (int)(N - n_int_total)) throw std::runtime_error("octree build: leaf count mismatch");
  T.valid = true;
}

}  // namespace pvfmm_b200

// Self-check of the bounded writes of the tree build's deferred count check
// (internal entry point, used by the GPU tests; no counterpart in the
// reference).  Runs compact_index and level_links with `n` flagged entries
// against capacities of `cap` < n, in buffers followed by a guard band, and
// checks that the ranks below cap are written and nothing at or beyond it.
// Returns 0 when the bounds hold, 1 otherwise (message in PVFMMGetLastError).
extern "C" int PVFMMB200CheckBoundedWrites(long n, long cap) {
  using namespace pvfmm_b200;
  constexpr long kGuard = 64;
  int* buf = nullptr;
  unsigned char* lf = nullptr;
  try {
    if (n <= 0 || cap < 0 || cap > n || n > (1L << 24)) throw std::runtime_error("bad sizes");
    // flag[n] = 1, offs[n] = iota, out[cap + guard], child0/parent/int_idx sized for cap internal nodes
    const long n_out = cap + kGuard, n_par = 8 * cap + kGuard;
    const long total = 2 * n + n_out + n + n_par + n_out;
    PVFMM_CUDA_CHECK(cudaMalloc((void**)&buf, total * sizeof(int)));
    PVFMM_CUDA_CHECK(cudaMalloc((void**)&lf, n));
    int* flag = buf;
    int* offs = flag + n;
    int* out = offs + n;
    int* child0 = out + n_out;
    int* parent = child0 + n;
    int* int_idx = parent + n_par;
    std::vector<int> h(total, -7);
    for (long i = 0; i < n; ++i) {
      h[i] = 1;
      h[n + i] = (int)i;
    }
    PVFMM_CUDA_CHECK(cudaMemcpy(buf, h.data(), total * sizeof(int), cudaMemcpyHostToDevice));
    compact_index<<<ceil_div(n, kThreads), kThreads>>>(flag, offs, n, cap, out, nullptr);
    // one level of n nodes at base 0, its children at next_base = n
    level_links<<<ceil_div(n, kThreads), kThreads>>>(flag, offs, n, 0, 0, 0, cap, lf, child0, parent, int_idx);
    PVFMM_CUDA_CHECK(cudaGetLastError());
    PVFMM_CUDA_CHECK(cudaMemcpy(h.data(), buf, total * sizeof(int), cudaMemcpyDeviceToHost));
    cudaFree(buf);
    cudaFree(lf);
    buf = nullptr;
    lf = nullptr;
    const int* ho = h.data() + 2 * n;
    const int* hp = ho + n_out + n;
    const int* hi = hp + n_par;
    for (long k = 0; k < n_out; ++k) {
      const int want = k < cap ? (int)k : -7;
      if (ho[k] != want) throw std::runtime_error("compact_index wrote rank " + std::to_string(k) + " wrongly");
      if (hi[k] != want) throw std::runtime_error("level_links wrote int_idx rank " + std::to_string(k) + " wrongly");
    }
    for (long k = 0; k < n_par; ++k) {
      const int want = k < 8 * cap ? (int)(k / 8) : -7;
      if (hp[k] != want) throw std::runtime_error("level_links wrote parent slot " + std::to_string(k) + " wrongly");
    }
    set_last_error("");
    return 0;
  } catch (const std::exception& e) {
    if (buf) cudaFree(buf);
    if (lf) cudaFree(lf);
    set_last_error(e.what());
    return 1;
  }
}
