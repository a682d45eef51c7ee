// C wrapper around the reference's pvfmm::MortonId (compiled from the
// reference sources by build.sh), used only to generate golden vectors that
// pin the oracle's Morton order.
#include <mortonid.hpp>

#include <algorithm>
#include <cstdint>
#include <numeric>
#include <vector>

using pvfmm::MortonId;

static MortonId from_ints(int64_t x, int64_t y, int64_t z, int d) {
  const double s = 1.0 / (double)(1u << 30);
  return MortonId((double)x * s, (double)y * s, (double)z * s, (uint8_t)d);
}

static void to_ints(MortonId m, int64_t* out) {
  double c[3];
  m.GetCoord(c);
  for (int k = 0; k < 3; ++k) out[k] = (int64_t)(c[k] * (double)(1u << 30));
  out[3] = m.GetDepth();
}

extern "C" {
// Morton coordinates of points: MortonId(coord) at depth 30.
void ref_point_ids(const double* c, long n, int64_t* out) {
  for (long i = 0; i < n; ++i) to_ints(MortonId(&c[i * 3]), &out[i * 4]);
}
// Stable sort by MortonId::operator<; order[i] = input index of the i-th id.
void ref_sort(const int64_t* ids, long n, int64_t* order) {
  std::vector<MortonId> m(n);
  for (long i = 0; i < n; ++i) m[i] = from_ints(ids[i * 4], ids[i * 4 + 1], ids[i * 4 + 2], (int)ids[i * 4 + 3]);
  std::vector<int64_t> idx(n);
  std::iota(idx.begin(), idx.end(), 0);
  std::stable_sort(idx.begin(), idx.end(), [&](int64_t a, int64_t b) { return m[a] < m[b]; });
  std::copy(idx.begin(), idx.end(), order);
}
// Children of each id (8 per id, 4 ints each).
void ref_children(const int64_t* ids, long n, int64_t* out) {
  for (long i = 0; i < n; ++i) {
    std::vector<MortonId> ch = from_ints(ids[i * 4], ids[i * 4 + 1], ids[i * 4 + 2], (int)ids[i * 4 + 3]).Children();
    for (int c = 0; c < 8; ++c) to_ints(ch[c], &out[(i * 8 + c) * 4]);
  }
}
// NbrList at the id's own depth, non-periodic: 27 slots, depth -1 = absent.
void ref_nbrs(const int64_t* ids, long n, int64_t* out) {
  for (long i = 0; i < n; ++i) {
    MortonId m = from_ints(ids[i * 4], ids[i * 4 + 1], ids[i * 4 + 2], (int)ids[i * 4 + 3]);
    std::vector<MortonId> nb;
    m.NbrList(nb, (uint8_t)ids[i * 4 + 3], 0);
    for (int k = 0; k < 27; ++k) out[(i * 27 + k) * 4 + 3] = -1;
    for (size_t k = 0; k < nb.size(); ++k) to_ints(nb[k], &out[(i * 27 + k) * 4]);
  }
}
}
