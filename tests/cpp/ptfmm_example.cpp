// Exercises include/pvfmm.hpp the way the reference's C++ examples use
// include/pvfmm.hpp (examples/src/example1.cpp:59-112): kernel object,
// PtFMM::Initialize, PtFMM_CreateTree, SetupFMM, PtFMM_Evaluate, a second
// evaluation with new densities after ClearFMMData, ker_poten and BuildMatrix.
// With n_dl > 0 the tree also holds a separate double-layer point set
// (PtFMM_CreateTree with surf_coord / surf_value, k0 + 3 values per point),
// and the second evaluation passes new values for both layers.  With a
// trailing "periodic", "px" or "pxy" the tree has that BoundaryType.  Writes inputs and
// outputs as raw doubles for the Python test to compare against the oracle.
//
// usage: ptfmm_example <out.bin> <kernel id> <m> <max_pts> <n_src> <n_trg> <seed> <real: d|f> [n_dl [periodic|px|pxy]]
#include <cmath>
#include <cstdint>
#include <cstdio>
#include <cstdlib>
#include <string>
#include <vector>

#include "pvfmm.hpp"

namespace {

struct Rng {  // splitmix64
  uint64_t s;
  double uniform() {
    uint64_t z = (s += 0x9E3779B97F4A7C15ull);
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    z ^= z >> 31;
    return (double)(z >> 11) * (1.0 / 9007199254740992.0);
  }
};

template <class Real>
const pvfmm::Kernel<Real>& kernel_of(int id) {
  switch (id) {
    case 0: return pvfmm::LaplaceKernel<Real>::potential();
    case 1: return pvfmm::LaplaceKernel<Real>::gradient();
    case 3: return pvfmm::StokesKernel<Real>::velocity();
    default: return pvfmm::LaplaceKernel<Real>::potgrad();
  }
}

template <class Real>
void put(std::vector<double>& out, const std::vector<Real>& v) {
  out.push_back((double)v.size());
  out.insert(out.end(), v.begin(), v.end());
}

template <class Real>
int run(const char* path, int kid, int m, int max_pts, long ns, long nt, uint64_t seed, long n_dl,
        pvfmm::BoundaryType bndry) {
  Rng rng{seed};
  const pvfmm::Kernel<Real>& ker = kernel_of<Real>(kid);
  const int k0 = ker.ker_dim[0], k1 = ker.ker_dim[1];
  std::vector<Real> src(3 * ns), den(k0 * ns), trg(3 * nt), den2(k0 * ns);
  for (auto& x : src) x = (Real)rng.uniform();
  for (auto& x : trg) x = (Real)rng.uniform();
  for (auto& x : den) x = (Real)(2 * rng.uniform() - 1);
  for (auto& x : den2) x = (Real)(2 * rng.uniform() - 1);
  std::vector<Real> dl(3 * n_dl), dd((k0 + 3) * n_dl), dd2((k0 + 3) * n_dl);
  for (auto& x : dl) x = (Real)rng.uniform();
  for (auto& x : dd) x = (Real)(2 * rng.uniform() - 1);
  for (auto& x : dd2) x = (Real)(2 * rng.uniform() - 1);

  MPI_Comm comm = MPI_COMM_WORLD;
  pvfmm::PtFMM<Real> matrices;
  matrices.Initialize(m, comm, &ker);
  pvfmm::PtFMM_Tree<Real>* tree =
      n_dl > 0 ? pvfmm::PtFMM_CreateTree(src, den, dl, dd, trg, comm, max_pts, bndry)
               : pvfmm::PtFMM_CreateTree(src, den, trg, comm, max_pts, bndry);
  tree->SetupFMM(&matrices);
  std::vector<Real> val1, val2;
  pvfmm::PtFMM_Evaluate(tree, val1, nt);
  tree->ClearFMMData();
  pvfmm::PtFMM_Evaluate(tree, val2, nt, &den2, n_dl > 0 ? &dd2 : nullptr);
  delete tree;

  // ker_poten accumulates: evaluate the first 64 targets twice over 200 sources
  const int ds = (int)std::min<long>(ns, 200), dt = (int)std::min<long>(nt, 64);
  std::vector<Real> kp((size_t)dt * k1, (Real)0);
  ker.ker_poten(src.data(), ds, den.data(), 1, trg.data(), dt, kp.data(), nullptr);
  ker.ker_poten(src.data(), ds, den.data(), 1, trg.data(), dt, kp.data(), nullptr);
  std::vector<Real> mat((size_t)3 * k0 * dt * k1);
  ker.BuildMatrix(src.data(), 3, trg.data(), dt, mat.data());

  std::vector<double> out;
  out.push_back((double)k0);
  out.push_back((double)k1);
  put(out, src);
  put(out, den);
  put(out, den2);
  put(out, trg);
  put(out, val1);
  put(out, val2);
  put(out, kp);
  put(out, mat);
  put(out, dl);
  put(out, dd);
  put(out, dd2);
  FILE* f = std::fopen(path, "wb");
  if (!f) return 2;
  std::fwrite(out.data(), sizeof(double), out.size(), f);
  std::fclose(f);
  return 0;
}

}  // namespace

int main(int argc, char** argv) {
  if (argc < 9 || argc > 11) {
    std::fprintf(stderr, "usage: %s out kernel m max_pts n_src n_trg seed d|f [n_dl [periodic|px|pxy]]\n", argv[0]);
    return 1;
  }
  try {
    const int kid = std::atoi(argv[2]), m = std::atoi(argv[3]), mp = std::atoi(argv[4]);
    const long ns = std::atol(argv[5]), nt = std::atol(argv[6]);
    const uint64_t seed = std::strtoull(argv[7], nullptr, 10);
    const long n_dl = argc >= 10 ? std::atol(argv[9]) : 0;
    const std::string bc = argc == 11 ? argv[10] : "";
    const pvfmm::BoundaryType bndry = bc == "periodic" ? pvfmm::Periodic
                                      : bc == "px"     ? pvfmm::PX
                                      : bc == "pxy"    ? pvfmm::PXY
                                                       : pvfmm::FreeSpace;
    if (std::string(argv[8]) == "f") return run<float>(argv[1], kid, m, mp, ns, nt, seed, n_dl, bndry);
    return run<double>(argv[1], kid, m, mp, ns, nt, seed, n_dl, bndry);
  } catch (const std::exception& e) {
    std::fprintf(stderr, "error: %s\n", e.what());
    return 3;
  }
}
