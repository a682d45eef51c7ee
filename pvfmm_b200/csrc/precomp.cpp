// Host FP64 precompute of the translation operators.
//
// Follows FMM_Pts::Precomp (reference include/fmm_pts.txx:453-764):
//   UC2UE0/1, DC2DE0/1  pseudo-inverse factors of the equivalent->check kernel
//                       matrices, by SVD with the 4*eps*max(S) cutoff (:478-581)
//   U2U, D2D            child<->parent translations (:582-643), one per octant
//   V / V1              kernel on the (2m)^3 convolution grid, r2c DFT, and the
//                       8x8 child blocks per parent offset divided by n3 (:671-764)
// Scale invariance (all expansion kernels here are homogeneous of degree -1
// with uniform exponents src=0, trg=1) makes the level-0 operators valid on
// every level; the level factors are applied at evaluation time.
#include <algorithm>
#include <cmath>
#include <complex>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <fstream>
#include <iterator>
#include <stdexcept>
#include <string>
#include <unistd.h>

#include "fmm_host.hpp"

namespace pvfmm_b200 {

namespace {
constexpr double kRad0 = 1.05;  // PVFMM_RAD0 (include/pvfmm_common.hpp:33)
constexpr double kRad1 = 2.95;  // PVFMM_RAD1 (include/pvfmm_common.hpp:34)
constexpr double kPi = 3.14159265358979323846;

thread_local std::string g_last_error;

// Row-major dense product C = A(r x k) * B(k x c).  Blocks of 8 rows x 256
// columns share each row segment of B from cache; every C[i][j] is still the
// sum over l in increasing order.
std::vector<double> matmul(const std::vector<double>& A, const std::vector<double>& B, int r, int k, int c) {
  constexpr int kRows = 8, kCols = 256;
  std::vector<double> C((size_t)r * c, 0.0);
  const int nrb = (r + kRows - 1) / kRows, ncb = (c + kCols - 1) / kCols;
#pragma omp parallel for schedule(static)
  for (int blk = 0; blk < nrb * ncb; ++blk) {
    const int i0 = (blk / ncb) * kRows, i1 = std::min(r, i0 + kRows);
    const int j0 = (blk % ncb) * kCols, j1 = std::min(c, j0 + kCols);
    for (int l = 0; l < k; ++l) {
      const double* bl = &B[(size_t)l * c];
      for (int i = i0; i < i1; ++i) {
        const double a = A[(size_t)i * k + l];
        if (a == 0.0) continue;
        double* ci = &C[(size_t)i * c];
        for (int j = j0; j < j1; ++j) ci[j] += a * bl[j];
      }
    }
  }
  return C;
}

// Points center + half*rad*u for the unit surface u.
std::vector<double> place_surface(const std::vector<double>& u, const double* center, double half, double rad) {
  std::vector<double> p(u.size());
  for (size_t i = 0; i < u.size() / 3; ++i)
    for (int d = 0; d < 3; ++d) p[i * 3 + d] = center[d] + half * rad * u[i * 3 + d];
  return p;
}

// Pseudo-inverse factors (fmm_pts.txx:478-537): for M (rows x cols) = U S V^T
// with r = min(rows, cols) singular values, C2E0 = V S^+ (cols x r) and
// C2E1 = U^T (r x rows).  With U_out / S_out the SVD's U (rows x r) and S are
// handed back as well.  A matrix with fewer rows than columns is decomposed
// through its transpose.
void pinv_factors(const std::vector<double>& M, int rows, int cols, double eps, std::vector<double>& c2e0,
                  std::vector<double>& c2e1, std::vector<double>* U_out = nullptr,
                  std::vector<double>* S_out = nullptr) {
  std::vector<double> U, S, V;
  if (rows >= cols) {
    jacobi_svd(rows, cols, M.data(), U, S, V);  // U rows x cols, V cols x cols
  } else {
    std::vector<double> Mt((size_t)cols * rows);
    for (int i = 0; i < rows; ++i)
      for (int j = 0; j < cols; ++j) Mt[(size_t)j * rows + i] = M[(size_t)i * cols + j];
    jacobi_svd(cols, rows, Mt.data(), V, S, U);  // M^T = V S U^T: V cols x rows, U rows x rows
  }
  const int r = std::min(rows, cols);
  double smax = 0;
  for (double s : S) smax = std::max(smax, std::fabs(s));
  const double cut = eps * smax * 4;
  c2e0.assign((size_t)cols * r, 0.0);
  for (int i = 0; i < cols; ++i)
    for (int j = 0; j < r; ++j) c2e0[(size_t)i * r + j] = (S[j] > cut) ? V[(size_t)i * r + j] / S[j] : 0.0;
  c2e1.assign((size_t)r * rows, 0.0);
  for (int j = 0; j < r; ++j)
    for (int i = 0; i < rows; ++i) c2e1[(size_t)j * rows + i] = U[(size_t)i * r + j];
  if (U_out) *U_out = std::move(U);
  if (S_out) *S_out = std::move(S);
}

// Pseudo-inverse factors with the FP64 cutoff and the singular values they
// were formed with (S_j = 0 for dropped directions).
struct PinvFactors {
  std::vector<double> c2e0, c2e1, S;
};

// c2e0 (n x r) with the columns whose singular value is not above
// 4*eps*max zeroed: the factor pinv_factors forms with cutoff eps (eps >= the
// FP64 cutoff the columns were kept with), entry for entry.
std::vector<double> with_cutoff(const PinvFactors& f, int n, int r, double eps) {
  double smax = 0;
  for (double v : f.S) smax = std::max(smax, std::fabs(v));
  const double cut = eps * smax * 4;
  std::vector<double> c = f.c2e0;
  for (int j = 0; j < r; ++j)
    if (!(f.S[j] > cut))
      for (int i = 0; i < n; ++i) c[(size_t)i * r + j] = 0.0;
  return c;
}

// ---------------------------------------------------------------------------
// Operator cache in the reference's precompute-file layout (Save2File and
// LoadFile, include/precomp_mat.txx:213-345; file name
// include/fmm_pts.txx:246-276): int sizeof(real) (8), int scale_invar (1),
// then for each of the 16 matrix types in Mat_Type order
// (include/precomp_mat.hpp:20-39) an int count n followed by n matrices, each
// int rows, int cols and rows*cols reals, row-major.  This library writes the
// pseudo-inverse factors UC2UE0, UC2UE1, DC2DE0, DC2DE1 (FP64 cutoff, the
// expensive SVD part of the precompute) as entry 0 of types 0-3 and leaves the
// other types empty, which a reference build fills itself; it reads entry 0
// of types 0-3 of any file in this layout and skips all other entries.  The
// cache is used only when the environment variable PVFMM_DIR names its
// directory (the reference's fallback location); without it no file is read
// or written.
// ---------------------------------------------------------------------------
constexpr int kMatTypes = 16;  // Type_Count

std::string cache_path(const KernelInfo& ki, int m) {
  const char* dir = std::getenv("PVFMM_DIR");
  if (!dir || !*dir) return "";
  return std::string(dir) + "/Precomp_" + ki.name + "_m" + std::to_string(m) + ".data";
}

// Reads the factors of f[0] (upward) and f[1] (downward); false when the file
// does not exist, an exception when it exists but is not a usable cache.
bool load_factors(const std::string& path, int din, int dout, PinvFactors (&f)[2]) {
  const int r = std::min(din, dout);
  std::ifstream in(path, std::ios::binary);
  if (!in) return false;
  std::vector<char> buf((std::istreambuf_iterator<char>(in)), std::istreambuf_iterator<char>());
  size_t pos = 0;
  auto bad = [&](const std::string& why) { return std::runtime_error("operator cache " + path + ": " + why); };
  auto get_int = [&]() {
    if (pos + sizeof(int) > buf.size()) throw bad("truncated");
    int v;
    std::memcpy(&v, buf.data() + pos, sizeof(int));
    pos += sizeof(int);
    return v;
  };
  if (get_int() != (int)sizeof(double)) throw bad("not an FP64 operator file");
  if (get_int() != 1) throw bad("operators of a kernel that is not scale-invariant");
  std::vector<double> mats[4];
  for (int t = 0; t < kMatTypes; ++t) {
    const int n = get_int();
    if (n < 0) throw bad("negative matrix count");
    for (int j = 0; j < n; ++j) {
      const int n1 = get_int(), n2 = get_int();
      if (n1 < 0 || n2 < 0) throw bad("negative matrix size");
      const size_t left = (buf.size() - pos) / sizeof(double);
      if (n1 > 0 && (size_t)n2 > left / (size_t)n1) throw bad("truncated");
      const size_t bytes = (size_t)n1 * n2 * sizeof(double);
      if (t < 4 && j == 0) {
        // C2E0 (types 0, 2): (ns*kout) x r; C2E1 (types 1, 3): r x (ns*kin)
        const int e1 = (t & 1) ? r : dout, e2 = (t & 1) ? din : r;
        if (n1 != e1 || n2 != e2)
          throw bad("matrix type " + std::to_string(t) + " is " + std::to_string(n1) + " x " + std::to_string(n2) +
                    ", expected " + std::to_string(e1) + " x " + std::to_string(e2));
        mats[t].resize((size_t)n1 * n2);
        std::memcpy(mats[t].data(), buf.data() + pos, bytes);
      }
      pos += bytes;
    }
  }
  for (int t = 0; t < 4; ++t)
    if (mats[t].empty()) throw bad("lacks matrix type " + std::to_string(t));
  for (int k = 0; k < 2; ++k) {
    f[k].c2e0 = std::move(mats[2 * k]);
    f[k].c2e1 = std::move(mats[2 * k + 1]);
    // C2E0 = V S^+ with orthonormal V: column j has length 1 / S_j (0 when dropped)
    f[k].S.assign(r, 0.0);
    for (int j = 0; j < r; ++j) {
      double n2 = 0;
      for (int i = 0; i < dout; ++i) n2 += f[k].c2e0[(size_t)i * r + j] * f[k].c2e0[(size_t)i * r + j];
      f[k].S[j] = n2 > 0 ? 1.0 / std::sqrt(n2) : 0.0;
    }
  }
  return true;
}

// Writes the factors (through a temporary file renamed into place, so that a
// concurrent reader never sees a partial file).  A directory that cannot be
// written is skipped silently, as the reference does.
void save_factors(const std::string& path, int din, int dout, const PinvFactors (&f)[2]) {
  const int r = std::min(din, dout);
  const std::string tmp = path + ".tmp" + std::to_string((long)getpid());
  FILE* fp = std::fopen(tmp.c_str(), "wb");
  if (!fp) return;
  bool ok = true;
  auto put_int = [&](int v) { ok = ok && std::fwrite(&v, sizeof(int), 1, fp) == 1; };
  put_int((int)sizeof(double));
  put_int(1);
  for (int t = 0; t < kMatTypes; ++t) {
    if (t >= 4) {
      put_int(0);
      continue;
    }
    const std::vector<double>& M = (t & 1) ? f[t / 2].c2e1 : f[t / 2].c2e0;
    put_int(1);
    put_int((t & 1) ? r : dout);
    put_int((t & 1) ? din : r);
    ok = ok && std::fwrite(M.data(), sizeof(double), M.size(), fp) == M.size();
  }
  ok = (std::fclose(fp) == 0) && ok;
  if (!ok || std::rename(tmp.c_str(), path.c_str()) != 0) std::remove(tmp.c_str());
}

// 1D complex DFT of length n along a strided line, sign -1 (forward).
void dft_line(std::complex<double>* x, int n, int stride, const std::vector<std::complex<double>>& w,
              std::vector<std::complex<double>>& tmp) {
  for (int k = 0; k < n; ++k) {
    std::complex<double> s = 0;
    for (int j = 0; j < n; ++j) s += x[(size_t)j * stride] * w[(size_t)(k * j) % n];
    tmp[k] = s;
  }
  for (int k = 0; k < n; ++k) x[(size_t)k * stride] = tmp[k];
}
}  // namespace

void set_last_error(const std::string& msg) { g_last_error = msg; }
const char* get_last_error() { return g_last_error.c_str(); }

bool kernel_info(int id, KernelInfo* out) {
  // scale exponents of the C interface's rescale (src_scal / trg_scal, found by
  // Kernel::Initialize, kernel.txx:64-196): a kernel of degree d, K(x/2) =
  // 2^d K(x), has src_scal 0 and trg_scal d per component
  KernelInfo k{};
  switch (id) {
    case kLaplacePot:
      k = {id, "laplace", 1, 1, kExpLaplace, 1, {0, 0, 0}, {1, 0, 0, 0}, 9, 1};
      break;
    case kLaplaceGrad:
      k = {id, "laplace_grad", 1, 3, kExpLaplace, 1, {0, 0, 0}, {2, 2, 2, 0}, 16, 1};
      break;
    case kStokesVel:
      k = {id, "stokes_vel", 3, 3, kExpStokes, 3, {0, 0, 0}, {1, 1, 1, 0}, 29, 1};
      break;
    case kLaplacePotGrad:
      k = {id, "laplace_potgrad", 1, 4, kExpLaplace, 1, {0, 0, 0}, {1, 2, 2, 2}, 18, 1};
      break;
    // Stokes pressure, Stokes velocity gradient and Biot-Savart expand
    // themselves (no separate expansion kernels, kernel.txx:894-901), with
    // kin = 3 equivalent-density and kout = k1 check-potential components
    case kStokesPress:  // StokesKernel<T>::pressure(), kernel.txx:1480-1483
      k = {id, "stokes_press", 3, 1, kExpStokesPress, 3, {0, 0, 0}, {2, 0, 0, 0}, 16, 2};
      break;
    case kStokesVelGrad:  // StokesKernel<T>::vel_grad(), kernel.txx:1488-1491
      k = {id, "stokes_grad", 3, 9, kExpStokesGrad, 3, {0, 0, 0}, {2, 2, 2, 2, 2, 2, 2, 2, 2}, 94, 2};
      break;
    case kBiotSavart:  // BiotSavartKernel<T>::potential(), kernel.txx:1508-1511
      k = {id, "biot_savart", 3, 3, kExpBiotSavart, 3, {0, 0, 0}, {2, 2, 2, 0}, 24, 2};
      break;
    default:
      return false;
  }
  if (out) *out = k;
  return true;
}

bool kernel_info_host(int id, KernelInfo* out) { return kernel_info(id, out); }

void exp_kernel_dims(int exp_kernel, int* kin, int* kout) {
  switch (exp_kernel) {
    case kExpLaplace: *kin = 1; *kout = 1; break;
    case kExpStokesPress: *kin = 3; *kout = 1; break;
    case kExpStokesGrad: *kin = 3; *kout = 9; break;
    default: *kin = 3; *kout = 3; break;  // Stokes velocity, Biot-Savart
  }
}

std::vector<double> unit_surface(int p) {
  // Same point order as surface() (fmm_pts.txx:54-97), unscaled.
  const int n = 6 * (p - 1) * (p - 1) + 2;
  std::vector<double> c((size_t)n * 3);
  c[0] = c[1] = c[2] = -1.0;
  int cnt = 1;
  for (int i = 0; i < p - 1; ++i)
    for (int j = 0; j < p - 1; ++j, ++cnt) {
      c[cnt * 3 + 0] = -1;
      c[cnt * 3 + 1] = (2.0 * (i + 1) - p + 1) / (p - 1);
      c[cnt * 3 + 2] = (2.0 * j - p + 1) / (p - 1);
    }
  for (int i = 0; i < p - 1; ++i)
    for (int j = 0; j < p - 1; ++j, ++cnt) {
      c[cnt * 3 + 0] = (2.0 * i - p + 1) / (p - 1);
      c[cnt * 3 + 1] = -1;
      c[cnt * 3 + 2] = (2.0 * (j + 1) - p + 1) / (p - 1);
    }
  for (int i = 0; i < p - 1; ++i)
    for (int j = 0; j < p - 1; ++j, ++cnt) {
      c[cnt * 3 + 0] = (2.0 * (i + 1) - p + 1) / (p - 1);
      c[cnt * 3 + 1] = (2.0 * j - p + 1) / (p - 1);
      c[cnt * 3 + 2] = -1;
    }
  for (int i = 0; i < (n / 2) * 3; ++i) c[(size_t)cnt * 3 + i] = -c[i];
  return c;
}

void exp_kernel_matrix(int exp_kernel, const double* src, int n_src, const double* trg, int n_trg, double* M) {
  if (exp_kernel == kExpLaplace) {
    const double s = 1.0 / (4 * kPi);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n_src; ++i)
      for (int t = 0; t < n_trg; ++t) {
        const double dx = trg[t * 3] - src[i * 3], dy = trg[t * 3 + 1] - src[i * 3 + 1],
                     dz = trg[t * 3 + 2] - src[i * 3 + 2];
        const double r2 = dx * dx + dy * dy + dz * dz;
        M[(size_t)i * n_trg + t] = r2 > 0 ? s / std::sqrt(r2) : 0.0;
      }
  } else if (exp_kernel == kExpStokes) {
    const double s = 1.0 / (8 * kPi);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n_src; ++i)
      for (int t = 0; t < n_trg; ++t) {
        const double r[3] = {trg[t * 3] - src[i * 3], trg[t * 3 + 1] - src[i * 3 + 1], trg[t * 3 + 2] - src[i * 3 + 2]};
        const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
        const double rinv = r2 > 0 ? 1.0 / std::sqrt(r2) : 0.0;
        const double rinv3 = rinv * rinv * rinv;
        for (int j = 0; j < 3; ++j)
          for (int k = 0; k < 3; ++k)
            M[((size_t)i * 3 + j) * n_trg * 3 + (size_t)t * 3 + k] =
                s * ((j == k ? rinv : 0.0) + r[j] * r[k] * rinv3);
      }
  } else {
    // Stokes pressure (kernel.txx:1366-1378), Stokes velocity gradient
    // (:1404-1432) and Biot-Savart (:1492-1505), source component j
    int kin, kout;
    exp_kernel_dims(exp_kernel, &kin, &kout);
#pragma omp parallel for schedule(static)
    for (int i = 0; i < n_src; ++i)
      for (int t = 0; t < n_trg; ++t) {
        const double r[3] = {trg[t * 3] - src[i * 3], trg[t * 3 + 1] - src[i * 3 + 1], trg[t * 3 + 2] - src[i * 3 + 2]};
        const double r2 = r[0] * r[0] + r[1] * r[1] + r[2] * r[2];
        const double rinv = r2 > 0 ? 1.0 / std::sqrt(r2) : 0.0;
        const double rinv2 = rinv * rinv, rinv3 = rinv2 * rinv;
        for (int j = 0; j < 3; ++j) {
          double* row = &M[((size_t)i * kin + j) * n_trg * kout + (size_t)t * kout];
          if (exp_kernel == kExpStokesPress) {
            row[0] = r[j] * rinv3 / (4 * kPi);  // (r . f) / r^3
          } else if (exp_kernel == kExpStokesGrad) {
            // u[3a+b] = (r_b f_a - f_b r_a + (r . f)(delta_ab - 3 r_a r_b / r^2)) / r^3
            for (int a = 0; a < 3; ++a)
              for (int b = 0; b < 3; ++b) {
                double v = r[j] * ((a == b ? 1.0 : 0.0) - 3 * r[a] * r[b] * rinv2);
                if (j == a) v += r[b];
                if (j == b) v -= r[a];
                row[3 * a + b] = v * rinv3 / (8 * kPi);
              }
          } else {  // (f x r) / r^3: u_k = e_kjl f_j r_l
            const int k1 = (j + 1) % 3, k2 = (j + 2) % 3;
            row[j] = 0.0;
            row[k2] = r[k1] * rinv3 / (4 * kPi);   // e_{k2 j k1} = +1
            row[k1] = -r[k2] * rinv3 / (4 * kPi);  // e_{k1 j k2} = -1
          }
        }
      }
  }
}

void jacobi_svd(int rows, int cols, const double* A, std::vector<double>& U, std::vector<double>& S,
                std::vector<double>& V) {
  if (rows < cols) throw std::runtime_error("jacobi_svd: rows < cols");
  const int n = cols;
  const int np = n + (n & 1);  // padded to even for the round-robin pairing
  // Column-major working copies: W[j] = column j of A*V, Vc[j] = column j of V.
  std::vector<double> W((size_t)np * rows, 0.0), Vc((size_t)np * n, 0.0);
  for (int j = 0; j < n; ++j) {
    for (int i = 0; i < rows; ++i) W[(size_t)j * rows + i] = A[(size_t)i * cols + j];
    Vc[(size_t)j * n + j] = 1.0;
  }
  std::vector<int> order(np);
  for (int i = 0; i < np; ++i) order[i] = i;
  const double tol = 1e-15;
  for (int sweep = 0; sweep < 80; ++sweep) {
    long rotations = 0;
    for (int round = 0; round < np - 1; ++round) {
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : rotations)
      for (int k = 0; k < np / 2; ++k) {
        int p = order[k], q = order[np - 1 - k];
        if (p >= n || q >= n) continue;
        if (p > q) std::swap(p, q);
        double* wp = &W[(size_t)p * rows];
        double* wq = &W[(size_t)q * rows];
        double a = 0, b = 0, g = 0;
        for (int i = 0; i < rows; ++i) {
          a += wp[i] * wp[i];
          b += wq[i] * wq[i];
          g += wp[i] * wq[i];
        }
        if (a == 0 || b == 0 || std::fabs(g) <= tol * std::sqrt(a * b)) continue;
        const double zeta = (b - a) / (2 * g);
        const double t = (zeta >= 0 ? 1.0 : -1.0) / (std::fabs(zeta) + std::sqrt(1 + zeta * zeta));
        const double c = 1 / std::sqrt(1 + t * t), s = c * t;
        for (int i = 0; i < rows; ++i) {
          const double x = wp[i], y = wq[i];
          wp[i] = c * x - s * y;
          wq[i] = s * x + c * y;
        }
        double* vp = &Vc[(size_t)p * n];
        double* vq = &Vc[(size_t)q * n];
        for (int i = 0; i < n; ++i) {
          const double x = vp[i], y = vq[i];
          vp[i] = c * x - s * y;
          vq[i] = s * x + c * y;
        }
        ++rotations;
      }
      // rotate all but the first entry
      const int last = order[np - 1];
      for (int i = np - 1; i > 1; --i) order[i] = order[i - 1];
      order[1] = last;
    }
    if (rotations == 0) break;
  }
  S.assign(n, 0.0);
  U.assign((size_t)rows * n, 0.0);
  V.assign((size_t)n * n, 0.0);
  for (int j = 0; j < n; ++j) {
    double nrm = 0;
    for (int i = 0; i < rows; ++i) nrm += W[(size_t)j * rows + i] * W[(size_t)j * rows + i];
    nrm = std::sqrt(nrm);
    S[j] = nrm;
    for (int i = 0; i < rows; ++i) U[(size_t)i * n + j] = nrm > 0 ? W[(size_t)j * rows + i] / nrm : 0.0;
    for (int i = 0; i < n; ++i) V[(size_t)i * n + j] = Vc[(size_t)j * n + i];
  }
}

void build_operators(int kernel, int m, bool mixed, HostOperators& ops, bool down_eps32) {
  KernelInfo ki;
  if (!kernel_info_host(kernel, &ki)) throw std::runtime_error("unsupported kernel");
  if (m < 2 || m > 16 || (m & 1)) throw std::runtime_error("multipole order must be even and in [2,16]");
  const int ke = ki.ke;
  int kin, kout;
  exp_kernel_dims(ki.exp_kernel, &kin, &kout);
  const int ns = 6 * (m - 1) * (m - 1) + 2;
  // equivalent densities din = ns*kin, check potentials dout = ns*kout, r
  // singular values per check -> equivalent factor
  const int din = ns * kin, dout = ns * kout, rk = std::min(din, dout);
  ops.kernel = kernel;
  ops.m = m;
  ops.ns = ns;
  ops.ke = ke;
  ops.kin = kin;
  ops.kout = kout;
  ops.mixed = mixed;
  ops.n1 = 2 * m;
  ops.n3 = ops.n1 * ops.n1 * ops.n1;
  ops.n3h = ops.n1 * ops.n1 * (ops.n1 / 2 + 1);
  ops.usurf = unit_surface(m);
  const double eps = mixed ? std::ldexp(1.0, -23) : std::ldexp(1.0, -52);
  const double zero[3] = {0, 0, 0};

  // Pseudo-inverse factors with the FP64 cutoff, from the operator cache or
  // from the SVDs: f[0] UC2UE0/1, upward equivalent (RAD0) -> upward check
  // (RAD1), level 0 (:478-537); f[1] DC2DE0/1, downward equivalent (RAD1) ->
  // downward check (RAD0) (:538-581).  A larger cutoff drops further columns.
  const double eps64 = std::ldexp(1.0, -52), eps32 = std::ldexp(1.0, -23);
  PinvFactors f[2];
  const std::string cache = cache_path(ki, m);
  if (cache.empty() || !load_factors(cache, din, dout, f)) {
    for (int k = 0; k < 2; ++k) {
      auto eq = place_surface(ops.usurf, zero, 0.5, k == 0 ? kRad0 : kRad1);
      auto ck = place_surface(ops.usurf, zero, 0.5, k == 0 ? kRad1 : kRad0);
      std::vector<double> M((size_t)din * dout);
      exp_kernel_matrix(ki.exp_kernel, eq.data(), ns, ck.data(), ns, M.data());
      pinv_factors(M, din, dout, eps64, f[k].c2e0, f[k].c2e1, nullptr, &f[k].S);
    }
    if (!cache.empty()) save_factors(cache, din, dout, f);
  }
  ops.uc2ue0 = with_cutoff(f[0], dout, rk, eps);
  ops.uc2ue1 = f[0].c2e1;
  ops.dc2de0 = with_cutoff(f[1], dout, rk, down_eps32 ? eps32 : eps);
  ops.dc2de1 = f[1].c2e1;
  // ue = (uc V S+) U^T lies in the span of U's columns (U^T = UC2UE1); its
  // components along singular values below 4*eps32*max are amplified FP64
  // rounding of the check potentials, cancelling in exact arithmetic but not
  // in FP32.  P = U_k U_k^T over the columns above that cutoff.
  {
    const std::vector<double>& Ut = f[0].c2e1;  // Ut[j][a] = U[a][j], r x din
    double smax = 0;
    for (double v : f[0].S) smax = std::max(smax, std::fabs(v));
    const double cut32 = 4.0 * eps32 * smax;
    ops.ue_proj.assign((size_t)din * din, 0.0);
    ops.ue32_dirs.clear();
    for (int j = 0; j < rk; ++j) {
      if (!(f[0].S[j] > cut32)) continue;
      ops.ue32_dirs.push_back(j);
      for (int a = 0; a < din; ++a) {
        const double ua = Ut[(size_t)j * din + a];
        double* row = &ops.ue_proj[(size_t)a * din];
        for (int b = 0; b < din; ++b) row[b] += ua * Ut[(size_t)j * din + b];
      }
    }
  }
  // U2U (:582-606): (M_ce2c * UC2UE0) * UC2UE1, child c of a level-0 parent.
  ops.u2u.assign((size_t)8 * din * din, 0.0);
  ops.d2d.assign((size_t)dout * 8 * dout, 0.0);
  ops.d2d_f2.assign((size_t)rk * 8 * dout, 0.0);
  for (int c = 0; c < 8; ++c) {
    const double cc[3] = {((c & 1) ? 0.25 : -0.25), ((c & 2) ? 0.25 : -0.25), ((c & 4) ? 0.25 : -0.25)};
    {
      auto ce = place_surface(ops.usurf, cc, 0.25, kRad0);
      auto pc = place_surface(ops.usurf, zero, 0.5, kRad1);
      std::vector<double> M((size_t)din * dout);
      exp_kernel_matrix(ki.exp_kernel, ce.data(), ns, pc.data(), ns, M.data());
      auto T = matmul(matmul(M, ops.uc2ue0, din, dout, rk), ops.uc2ue1, din, rk, din);
      std::memcpy(&ops.u2u[(size_t)c * din * din], T.data(), sizeof(double) * din * din);
    }
    // D2D (:607-643): DC2DE0 * (DC2DE1 * M_pe2c), parent level 0 -> child c.
    {
      auto pe = place_surface(ops.usurf, zero, 0.5, kRad1);
      auto cc2 = place_surface(ops.usurf, cc, 0.25, kRad0);
      std::vector<double> M((size_t)din * dout);
      exp_kernel_matrix(ki.exp_kernel, pe.data(), ns, cc2.data(), ns, M.data());
      auto F = matmul(ops.dc2de1, M, rk, din, dout);
      auto T = matmul(ops.dc2de0, F, dout, rk, dout);
      for (int r = 0; r < dout; ++r)
        std::memcpy(&ops.d2d[(size_t)r * 8 * dout + (size_t)c * dout], &T[(size_t)r * dout], sizeof(double) * dout);
      for (int r = 0; r < rk; ++r)
        std::memcpy(&ops.d2d_f2[(size_t)r * 8 * dout + (size_t)c * dout], &F[(size_t)r * dout],
                    sizeof(double) * dout);
    }
  }
  // FFT maps (:2703-2712, :2790-2797): lattice index s = (u+1)(m-1)/2.
  ops.fft_map.resize(ns);
  ops.ifft_map.resize(ns);
  const int n1 = ops.n1;
  for (int i = 0; i < ns; ++i) {
    int s[3];
    for (int d = 0; d < 3; ++d) s[d] = (int)std::lround((ops.usurf[i * 3 + d] + 1.0) * (m - 1) * 0.5);
    ops.fft_map[i] = (m - 1 - s[0]) + (m - 1 - s[1]) * n1 + (m - 1 - s[2]) * n1 * n1;
    ops.ifft_map[i] = (2 * m - 1 - s[0]) + (2 * m - 1 - s[1]) * n1 + (2 * m - 1 - s[2]) * n1 * n1;
  }
  // V operators (:671-718): for source-minus-target child offset rel (child
  // units, box 1), kernel from the conv grid (i-m)*RAD0/(m-1)+rel to the
  // origin, then a 3D r2c DFT with x the halved axis.
  const int n3 = ops.n3, nh = n1 / 2 + 1, n3h = ops.n3h, kk = kin * kout;
  std::vector<std::complex<double>> w(n1);
  for (int j = 0; j < n1; ++j) w[j] = std::polar(1.0, -2 * kPi * j / n1);
  std::vector<std::vector<std::complex<double>>> vhat(343);  // index (i+3)+7(j+3)+49(k+3)
#pragma omp parallel for schedule(dynamic)
  for (int idx = 0; idx < 343; ++idx) {
    const int ri = idx % 7 - 3, rj = (idx / 7) % 7 - 3, rk = idx / 49 - 3;
    if (std::max(std::abs(ri), std::max(std::abs(rj), std::abs(rk))) <= 1) continue;
    std::vector<double> grid((size_t)n3 * 3);
    for (int k = 0; k < n1; ++k)
      for (int j = 0; j < n1; ++j)
        for (int i = 0; i < n1; ++i) {
          const size_t g = (size_t)i + (size_t)n1 * j + (size_t)n1 * n1 * k;
          grid[g * 3 + 0] = (i - m) * kRad0 / (m - 1) + ri;
          grid[g * 3 + 1] = (j - m) * kRad0 / (m - 1) + rj;
          grid[g * 3 + 2] = (k - m) * kRad0 / (m - 1) + rk;
        }
    std::vector<double> P((size_t)n3 * kk);
    exp_kernel_matrix(ki.exp_kernel, grid.data(), n3, zero, 1, P.data());  // P[g*kin+i][k]
    std::vector<std::complex<double>> out((size_t)n3h * kk);
    std::vector<std::complex<double>> cube((size_t)n3), tmp(n1);
    for (int comp = 0; comp < kk; ++comp) {
      for (int g = 0; g < n3; ++g) cube[g] = P[(size_t)g * kk + comp];
      for (int k = 0; k < n1; ++k)
        for (int j = 0; j < n1; ++j) dft_line(&cube[(size_t)n1 * j + (size_t)n1 * n1 * k], n1, 1, w, tmp);
      for (int k = 0; k < n1; ++k)
        for (int i = 0; i < nh; ++i) dft_line(&cube[(size_t)i + (size_t)n1 * n1 * k], n1, n1, w, tmp);
      for (int j = 0; j < n1; ++j)
        for (int i = 0; i < nh; ++i) dft_line(&cube[(size_t)i + (size_t)n1 * j], n1, n1 * n1, w, tmp);
      for (int k = 0; k < n1; ++k)
        for (int j = 0; j < n1; ++j)
          for (int i = 0; i < nh; ++i)
            out[(((size_t)k * n1 + j) * nh + i) * kk + comp] = cube[(size_t)i + (size_t)n1 * j + (size_t)n1 * n1 * k];
    }
    vhat[idx] = std::move(out);
  }
  // Hadamard operators (V1, :719-764): parent offset o (colleague index ci,
  // ci != 13), target child j1, source child j2: rel = 2*po - bits(j1) + bits(j2);
  // adjacent children give zero blocks.  Divided by n3 (inverse DFT scale).
  ops.vop.assign((size_t)n3h * 26 * 64 * kk * 2, 0.0);
  for (int ci = 0, o = 0; ci < 27; ++ci) {
    if (ci == 13) continue;
    const int po[3] = {ci % 3 - 1, (ci / 3) % 3 - 1, ci / 9 - 1};
    for (int j1 = 0; j1 < 8; ++j1)
      for (int j2 = 0; j2 < 8; ++j2) {
        int rel[3];
        for (int d = 0; d < 3; ++d) rel[d] = 2 * po[d] - ((j1 >> d) & 1) + ((j2 >> d) & 1);
        if (std::max(std::abs(rel[0]), std::max(std::abs(rel[1]), std::abs(rel[2]))) <= 1) continue;
        const auto& vh = vhat[(rel[0] + 3) + 7 * (rel[1] + 3) + 49 * (rel[2] + 3)];
        for (int f = 0; f < n3h; ++f)
          for (int c = 0; c < kk; ++c) {
            const size_t dst = ((((size_t)f * 26 + o) * 64 + j1 * 8 + j2) * kk + c) * 2;
            ops.vop[dst + 0] = vh[(size_t)f * kk + c].real() / n3;
            ops.vop[dst + 1] = vh[(size_t)f * kk + c].imag() / n3;
          }
      }
    ++o;
  }
}

// ---------------------------------------------------------------------------
// Periodic boundary operator (the reference's BC_Type precompute for
// BoundaryType Periodic == PXYZ, include/fmm_pts.txx:790-1232): the linear
// map from the root's upward equivalent density to the downward check
// potential of the periodic images outside the root's 3x3x3 block.  Two
// forms, as the reference's build option PVFMM_EXTENDED_BC selects: the
// images of the 5x5x5 block only (option on, the reference's CMake default;
// a user operator may be added to it), or the lattice sum over all images
// (option off: 45 levels of coarsened images, zero-average projections, the
// far field of the unit volume potential and the corner correction; all
// products at order m+2 and brought back to order m at the end).
// ---------------------------------------------------------------------------
namespace {

// Gauss-Legendre nodes and weights on [0, 1] (Newton iteration on P_n from
// the Chebyshev-like initial guesses cos(pi (i + 3/4) / (n + 1/2))).
void gauss_legendre01(int n, std::vector<double>& x, std::vector<double>& w) {
  x.assign(n, 0.0);
  w.assign(n, 0.0);
  for (int i = 0; i < n; ++i) {
    double z = std::cos(kPi * (i + 0.75) / (n + 0.5)), dp = 1;
    for (int it = 0; it < 100; ++it) {
      double p0 = 1, p1 = z;
      for (int k = 2; k <= n; ++k) {
        const double p2 = ((2 * k - 1) * z * p1 - (k - 1) * p0) / k;
        p0 = p1;
        p1 = p2;
      }
      dp = n * (z * p1 - p0) / (z * z - 1);
      const double dz = p1 / dp;
      z -= dz;
      if (std::fabs(dz) < 1e-16) break;
    }
    x[i] = 0.5 * (1 - z);
    w[i] = 1.0 / ((1 - z * z) * dp * dp);  // 2 / ((1 - z^2) P_n'^2) on [-1, 1], halved
  }
}

// Integral of the expansion kernel (homogeneous of degree -1) over the box
// [lo, lo + side]^3 at target x, out[k*ke + l] for source component k and
// target component l: the box is the signed union of the six pyramids with
// apex x over its faces, and along each pyramid's rays the degree -1 kernel
// integrates in closed form, leaving (h_F / 2) int_F K(x - z) dA_z with h_F
// the signed distance from x to face F (outward normal).  The faces are
// smooth integrands for targets off their planes: composite Gauss-Legendre,
// panels of side <= 1/2 with 16 x 16 nodes.  (The reference evaluates these
// integrals with its Chebyshev quadrature, cheb_integ, include/cheb_utils.txx:1037.)
void box_integral(int exp_kernel, int ke, const double* x, double lo, double side, double* out) {
  static thread_local std::vector<double> gx, gw;
  if (gx.empty()) gauss_legendre01(16, gx, gw);
  const int G = (int)gx.size();
  const int P = std::max(1, (int)std::ceil(side / 0.5 - 1e-12));
  const double ps = side / P;
  std::vector<double> nodes, wts, K;
  for (int i = 0; i < ke * ke; ++i) out[i] = 0;
  for (int f = 0; f < 6; ++f) {
    const int a = f >> 1;               // normal axis
    const double plane = lo + ((f & 1) ? side : 0.0);
    const double h = (f & 1) ? plane - x[a] : x[a] - plane;  // outward normal distance from x
    if (h == 0.0) continue;
    const int b = (a + 1) % 3, c = (a + 2) % 3;
    nodes.clear();
    wts.clear();
    for (int pb = 0; pb < P; ++pb)
      for (int pc = 0; pc < P; ++pc)
        for (int ib = 0; ib < G; ++ib)
          for (int ic = 0; ic < G; ++ic) {
            double z[3];
            z[a] = plane;
            z[b] = lo + (pb + gx[ib]) * ps;
            z[c] = lo + (pc + gx[ic]) * ps;
            nodes.insert(nodes.end(), z, z + 3);
            wts.push_back(gw[ib] * gw[ic] * ps * ps);
          }
    const int n = (int)wts.size();
    K.resize((size_t)n * ke * ke);
    exp_kernel_matrix(exp_kernel, nodes.data(), n, x, 1, K.data());  // [i*ke + k][l]
    for (int i = 0; i < n; ++i)
      for (int k = 0; k < ke; ++k)
        for (int l = 0; l < ke; ++l) out[k * ke + l] += 0.5 * h * wts[i] * K[((size_t)i * ke + k) * ke + l];
  }
}

// Surface of order p around the box with lower corner c at depth `depth`
// (side 2^-depth) scaled by rad about its centre (u_equiv_surf and its
// siblings, include/fmm_pts.txx:54-160).
std::vector<double> box_surface(const std::vector<double>& u, const double* c, int depth, double rad) {
  const double r = 0.5 * std::ldexp(1.0, -depth);
  const double ctr[3] = {c[0] + r, c[1] + r, c[2] + r};
  return place_surface(u, ctr, r, rad);
}

std::vector<double> kmat(int exp_kernel, int ke, const std::vector<double>& src, const std::vector<double>& trg) {
  const int ns = (int)src.size() / 3, nt = (int)trg.size() / 3;
  std::vector<double> M((size_t)ns * ke * nt * ke);
  exp_kernel_matrix(exp_kernel, src.data(), ns, trg.data(), nt, M.data());
  return M;
}

// The reference's volume potential of a unit density (vol_poten, kernel.txx:
// 1289-1295 Laplace, :1456-1467 Stokes) at n points: out[k][i*ke + l].
void vol_poten(int exp_kernel, const double* p, int n, double* out) {
  const int ke = exp_kernel == kExpStokes ? 3 : 1;
  for (int i = 0; i < n * ke * ke; ++i) out[i] = 0;
  for (int i = 0; i < n; ++i) {
    const double x = p[3 * i], y = p[3 * i + 1], z = p[3 * i + 2];
    if (ke == 1) {
      out[i] = -(x * x + y * y + z * z) / 6;
    } else {
      const double r2[3] = {y * y + z * z, x * x + z * z, x * x + y * y};
      for (int k = 0; k < 3; ++k) out[(size_t)k * n * 3 + i * 3 + k] = -r2[k] / 4;
    }
  }
}

}  // namespace

std::vector<double> lattice_bc(const KernelInfo& ki, int m, int axes);

// An image offset is taken when every axis it moves along is periodic
// (axes: bit 0 x, bit 1 y, bit 2 z; BoundaryType PX 1, PXY 3, PXYZ 7).
bool image_axes_ok(int axes, int x0, int x1, int x2) {
  return (x0 == 0 || (axes & 1)) && (x1 == 0 || (axes & 2)) && (x2 == 0 || (axes & 4));
}

bool lattice_bc_supported(int kernel) { return kernel == kLaplacePot || kernel == kLaplaceGrad || kernel == kStokesVel; }

std::vector<double> build_bc_operator(int kernel, int m, bool lattice, int axes) {
  KernelInfo ki;
  if (!kernel_info_host(kernel, &ki)) throw std::runtime_error("periodic boundaries: unknown kernel");
  if (axes != 1 && axes != 3 && axes != 7) throw std::runtime_error("periodic axes must be x, xy or xyz");
  if (!lattice) {
    // the reference's default build (PVFMM_EXTENDED_BC, :1189-1232): the
    // images in [-2, 2]^3 outside [-1, 1]^3 (along the periodic axes) at
    // order m, nothing beyond them
    int kin, kout;
    exp_kernel_dims(ki.exp_kernel, &kin, &kout);
    const std::vector<double> u = unit_surface(m);
    const int ns = (int)u.size() / 3;
    const double zero[3] = {0, 0, 0};
    const std::vector<double> dk = box_surface(u, zero, 0, kRad0);
    std::vector<double> M((size_t)ns * kin * ns * kout, 0.0), T(M.size());
    for (int x0 = -2; x0 <= 2; ++x0)
      for (int x1 = -2; x1 <= 2; ++x1)
        for (int x2 = -2; x2 <= 2; ++x2) {
          if (std::abs(x0) <= 1 && std::abs(x1) <= 1 && std::abs(x2) <= 1) continue;
          if (!image_axes_ok(axes, x0, x1, x2)) continue;
          const double c[3] = {(double)x0, (double)x1, (double)x2};
          const std::vector<double> src = box_surface(u, c, 0, kRad0);
          exp_kernel_matrix(ki.exp_kernel, src.data(), ns, dk.data(), ns, T.data());
          for (size_t i = 0; i < M.size(); ++i) M[i] += T[i];
        }
    return M;
  }
  if (!lattice_bc_supported(kernel)) throw std::runtime_error("periodic lattice sum: kernel not supported");
  // operator file (with PVFMM_DIR, beside the pseudo-inverse factors): int
  // rows, int cols, rows*cols FP64 values; the order m+2 SVDs of the lattice
  // sum take minutes for Stokes at m >= 10
  const std::string base = cache_path(ki, m);
  const std::string path = base.empty() ? ""
                                         : base.substr(0, base.size() - 5) + "_lattice_bc" +
                                               (axes == 1 ? "_px" : axes == 3 ? "_pxy" : "") + ".data";
  {
    const int n = 6 * (m - 1) * (m - 1) + 2, dim = n * ki.ke;
    std::ifstream in(path, std::ios::binary);
    if (!path.empty() && in) {
      int rc[2] = {0, 0};
      std::vector<double> M((size_t)dim * dim);
      in.read(reinterpret_cast<char*>(rc), sizeof(rc));
      if (!in || rc[0] != dim || rc[1] != dim) throw std::runtime_error("operator file " + path + ": wrong sizes");
      in.read(reinterpret_cast<char*>(M.data()), (std::streamsize)(M.size() * sizeof(double)));
      if (!in) throw std::runtime_error("operator file " + path + ": truncated");
      return M;
    }
  }
  std::vector<double> M = lattice_bc(ki, m, axes);
  if (!path.empty()) {  // written through a temporary file renamed into place; an unwritable directory is skipped
    const std::string tmp = path + ".tmp" + std::to_string((long)getpid());
    if (FILE* fp = std::fopen(tmp.c_str(), "wb")) {
      const int dim = (int)std::lround(std::sqrt((double)M.size()));
      const int rc[2] = {dim, dim};
      bool ok = std::fwrite(rc, sizeof(int), 2, fp) == 2 &&
                std::fwrite(M.data(), sizeof(double), M.size(), fp) == M.size();
      ok = (std::fclose(fp) == 0) && ok;
      if (!ok || std::rename(tmp.c_str(), path.c_str()) != 0) std::remove(tmp.c_str());
    }
  }
  return M;
}

// The lattice sum itself (the reference built without PVFMM_EXTENDED_BC).
std::vector<double> lattice_bc(const KernelInfo& ki, int m, int axes) {
  const int ex = ki.exp_kernel, ke = ki.ke;
  const int kernel = ki.id;
  // the reference attaches the volume potential to the Laplace potential and
  // Stokes velocity kernels only (the gradient kernel's expansion kernel has
  // none), and uses it for PXYZ only
  const bool has_vol = (kernel == kLaplacePot || kernel == kStokesVel) && axes == 7;
  const int m1 = m + 2;  // mult_upsample = 2
  const std::vector<double> u1 = unit_surface(m1), u0 = unit_surface(m);
  const int ns1 = (int)u1.size() / 3, ns0 = (int)u0.size() / 3;
  const int n1 = ns1 * ke, n0 = ns0 * ke;
  const double eps = std::ldexp(1.0, -52);
  const double zero[3] = {0, 0, 0}, mone[3] = {-1, -1, -1}, mhalf[3] = {-0.5, -0.5, -0.5};
  // pseudo-inverse factors at order m1, depth 0 (side 1); depth -1 (side 2)
  // follows from homogeneity: the kernel matrices scale by 2^-deg, their
  // pseudo-inverses by 2^deg
  std::vector<double> uc0, uc1, dc0, dc1;
  pinv_factors(kmat(ex, ke, box_surface(u1, zero, 0, kRad0), box_surface(u1, zero, 0, kRad1)), n1, n1, eps, uc0, uc1);
  pinv_factors(kmat(ex, ke, box_surface(u1, zero, 0, kRad1), box_surface(u1, zero, 0, kRad0)), n1, n1, eps, dc0, dc1);
  const double up = std::ldexp(1.0, ki.deg);
  std::vector<double> uc0m(uc0), dc0m(dc0);
  for (double& v : uc0m) v *= up;
  for (double& v : dc0m) v *= up;
  auto add = [](std::vector<double>& a, const std::vector<double>& b) {
    for (size_t i = 0; i < a.size(); ++i) a[i] += b[i];
  };
  // zero-average projections (:859-911): Pe removes from an equivalent
  // density the multiple of a unit volume source (row-normalised), Pc the
  // mean of each check-potential component
  std::vector<double> Pe((size_t)n1 * n1, 0.0), Pc((size_t)n1 * n1, 0.0);
  {
    const std::vector<double> uc = box_surface(u1, zero, 0, kRad1);
    std::vector<double> s2c((size_t)ke * n1);
    std::vector<double> I(ke * ke);
    for (int i = 0; i < ns1; ++i) {
      box_integral(ex, ke, &uc[3 * i], 0.0, 1.0, I.data());
      for (int j = 0; j < ke; ++j)
        for (int k = 0; k < ke; ++k) s2c[(size_t)j * n1 + i * ke + k] = I[k * ke + j];
    }
    std::vector<double> s2e = matmul(matmul(s2c, uc0, ke, n1, n1), uc1, ke, n1, n1);
    for (int j = 0; j < ke; ++j) {
      double s = 0;
      for (int c = 0; c < n1; ++c) s += s2e[(size_t)j * n1 + c];
      for (int c = 0; c < n1; ++c) s2e[(size_t)j * n1 + c] /= s;
    }
    for (int r = 0; r < n1; ++r) {
      Pe[(size_t)r * n1 + r] += 1;
      Pc[(size_t)r * n1 + r] += 1;
      for (int c = 0; c < n1; ++c) Pe[(size_t)r * n1 + c] -= s2e[(size_t)(r % ke) * n1 + c];
    }
    for (int i = 0; i < ns1; ++i)
      for (int j = 0; j < ns1; ++j)
        for (int k = 0; k < ke; ++k) Pc[((size_t)i * ke + k) * n1 + j * ke + k] -= 1.0 / ns1;
  }
  // M2M: the 8 children (side 1) of a side-2 parent, each with the same
  // equivalent density, to the parent's equivalent density
  std::vector<double> M2M((size_t)n1 * n1, 0.0);
  {
    const std::vector<double> ck = box_surface(u1, mone, -1, kRad1);
    for (int c = 0; c < 8; ++c) {
      if (!image_axes_ok(axes, c & 1, (c >> 1) & 1, (c >> 2) & 1)) continue;
      const double sb[3] = {-1.0 + (c & 1), -1.0 + ((c >> 1) & 1), -1.0 + ((c >> 2) & 1)};
      add(M2M, kmat(ex, ke, box_surface(u1, sb, 0, kRad0), ck));
    }
    M2M = matmul(matmul(M2M, uc0m, n1, n1, n1), uc1, n1, n1, n1);
  }
  // L2L: parent (side 2) downward check -> child (side 1) downward check
  std::vector<double> L2L =
      matmul(dc0m, matmul(dc1, kmat(ex, ke, box_surface(u1, mone, -1, kRad1), box_surface(u1, mone, 0, kRad0)), n1,
                          n1, n1),
             n1, n1, n1);
  // M2L: the images at offsets in [-2, 3]^3 outside [-1, 1]^3 to the root's
  // downward check surface
  std::vector<double> M2L((size_t)n1 * n1, 0.0);
  {
    const std::vector<double> dk = box_surface(u1, zero, 0, kRad0);
    for (int k0 = -2; k0 < 4; ++k0)
      for (int k1 = -2; k1 < 4; ++k1)
        for (int k2 = -2; k2 < 4; ++k2) {
          if (std::abs(k0) <= 1 && std::abs(k1) <= 1 && std::abs(k2) <= 1) continue;
          if (!image_axes_ok(axes, k0, k1, k2)) continue;
          const double sb[3] = {(double)k0, (double)k1, (double)k2};
          add(M2L, kmat(ex, ke, box_surface(u1, sb, 0, kRad0), dk));
        }
  }
  M2M = matmul(matmul(Pe, M2M, n1, n1, n1), Pe, n1, n1, n1);
  L2L = matmul(matmul(Pc, L2L, n1, n1, n1), Pc, n1, n1, n1);
  M2L = matmul(matmul(Pe, M2L, n1, n1, n1), Pc, n1, n1, n1);
  // lattice levels (PVFMM_BC_LEVELS = 45): M = M2L + M2M (Pr M Pc) L2L, the
  // level scalings Pr = 2^-src_scal = 1 and Pc = 2^-trg_scal = 2^-deg of the
  // degree -deg expansion kernel
  std::vector<double> M = M2L;
  const double pc = std::ldexp(1.0, -ki.deg);
  for (int level = 1; level < 45; ++level) {
    std::vector<double> T = matmul(matmul(M2M, M, n1, n1, n1), L2L, n1, n1, n1);
    for (size_t i = 0; i < M.size(); ++i) M[i] = M2L[i] + pc * T[i];
  }
  // far field of the unit volume potential (:1001-1034): the analytic
  // potential minus the 3x3x3 block's integral, on the check surface of the
  // block's centre box
  if (has_vol) {
    const double c1[3] = {1, 1, 1};
    const std::vector<double> dc = box_surface(u1, c1, 0, kRad0);
    std::vector<double> far((size_t)ke * n1);
    vol_poten(ex, dc.data(), ns1, far.data());
    std::vector<double> I(ke * ke);
    for (int i = 0; i < ns1; ++i) {
      box_integral(ex, ke, &dc[3 * i], 0.0, 3.0, I.data());
      for (int j = 0; j < ke; ++j)
        for (int k = 0; k < ke; ++k) far[(size_t)j * n1 + i * ke + k] -= I[k * ke + j];
    }
    for (int i = 0; i < ns1; ++i)
      for (int k = 0; k < ke; ++k)
        for (int j = 0; j < n1; ++j) M[((size_t)i * ke + k) * n1 + j] += far[(size_t)k * n1 + j];
  }
  // corner correction (:1036-1161): the constant and linear parts of the
  // potential, fitted to its values at the root's 8 corners (the far images
  // through M, the 3x3x3 block's images through the upward equivalent
  // surface), are removed on the check surface
  {
    double corner[24];
    for (int i = 0; i < 8; ++i) {
      corner[3 * i] = i & 1;
      corner[3 * i + 1] = (i >> 1) & 1;
      corner[3 * i + 2] = (i >> 2) & 1;
    }
    const std::vector<double> ue = box_surface(u1, zero, 0, kRad0), de = box_surface(u1, zero, 0, kRad1),
                              dk = box_surface(u1, zero, 0, kRad0);
    const std::vector<double> cp(corner, corner + 24);
    std::vector<double> cv =
        matmul(matmul(M, dc0, n1, n1, n1), matmul(dc1, kmat(ex, ke, de, cp), n1, n1, 8 * ke), n1, n1, 8 * ke);
    for (int k = 0; k < 8; ++k)
      for (int j0 = -1; j0 <= 1; ++j0)
        for (int j1 = -1; j1 <= 1; ++j1)
          for (int j2 = -1; j2 <= 1; ++j2) {
            if (!image_axes_ok(axes, j0, j1, j2)) continue;
            const std::vector<double> pt = {corner[3 * k] - j0, corner[3 * k + 1] - j1, corner[3 * k + 2] - j2};
            if (std::fabs(pt[0] - 0.5) < 1 && std::fabs(pt[1] - 0.5) < 1 && std::fabs(pt[2] - 0.5) < 1) continue;
            const std::vector<double> E = kmat(ex, ke, ue, pt);  // n1 x ke
            for (int i = 0; i < n1; ++i)
              for (int l = 0; l < ke; ++l) cv[(size_t)i * 8 * ke + k * ke + l] += E[(size_t)i * ke + l];
          }
    if (has_vol) {
      std::vector<double> va((size_t)ke * 8 * ke);
      vol_poten(ex, corner, 8, va.data());
      for (int j = 0; j < ns1; ++j)
        for (int k = 0; k < ke; ++k)
          for (int i = 0; i < 8 * ke; ++i) cv[((size_t)j * ke + k) * 8 * ke + i] -= va[(size_t)k * 8 * ke + i];
    }
    // coefficients of a + bx + cy + dz + exy + fxz + gyz + hxyz through the
    // inverse of the corners' Vandermonde matrix (nonsingular); the constant
    // term and the linear terms of the periodic axes are enabled (PXYZ: a,
    // b, c, d; PXY: a, b, c; PX: a, b)
    const double en[4] = {1.0, 1.0, (axes & 2) ? 1.0 : 0.0, (axes & 4) ? 1.0 : 0.0};
    std::vector<double> V(64), Vi;
    for (int i = 0; i < 8; ++i) {
      const double x = corner[3 * i], y = corner[3 * i + 1], z = corner[3 * i + 2];
      const double row[8] = {1, x, y, z, x * y, x * z, y * z, x * y * z};
      for (int r = 0; r < 8; ++r) V[r * 8 + i] = row[r];
    }
    {
      std::vector<double> c0, c1;
      pinv_factors(V, 8, 8, eps, c0, c1);
      Vi = matmul(c0, c1, 8, 8, 8);  // V^+ (8 x 8)
    }
    for (int i = 0; i < n1; ++i)
      for (int l = 0; l < ke; ++l) {
        // values of equivalent entry i, check component l at the 8 corners
        double coef[4] = {0, 0, 0, 0};
        for (int q = 0; q < 4; ++q)
          for (int k = 0; k < 8; ++k) coef[q] += cv[(size_t)i * 8 * ke + k * ke + l] * Vi[k * 8 + q];
        for (int p = 0; p < ns1; ++p)
          M[(size_t)i * n1 + p * ke + l] -= en[0] * coef[0] + en[1] * coef[1] * dk[3 * p] +
                                            en[2] * coef[2] * dk[3 * p + 1] + en[3] * coef[3] * dk[3 * p + 2];
      }
  }
  // back to order m (:1164-1188): order-m equivalent -> order-m1 equivalent,
  // order-m1 downward equivalent -> order-m check
  std::vector<double> up_m =
      matmul(matmul(kmat(ex, ke, box_surface(u0, mhalf, 0, kRad0), box_surface(u1, mhalf, 0, kRad1)), uc0, n0, n1,
                    n1),
             uc1, n0, n1, n1);
  std::vector<double> dn_m =
      matmul(dc0, matmul(dc1, kmat(ex, ke, box_surface(u1, mhalf, 0, kRad1), box_surface(u0, mhalf, 0, kRad0)), n1,
                         n1, n0),
             n1, n1, n0);
  return matmul(matmul(up_m, M, n0, n1, n1), dn_m, n0, n1, n0);
}

}  // namespace pvfmm_b200
