// Host (FP64) generation of the geometry-dependent operators of the plan.
//
//  - Basis order: degree ascending, then alpha_x, then alpha_y (upstream
//    include/cdfmm/multi_index.hpp:62-71).
//  - M2M child->parent shift A(d)[alpha][eta] = d^(alpha-eta)/(alpha-eta)!,
//    d = c_parent - c_child; L2L parent->child B(d)[beta][eta] =
//    d^(eta-beta)/(eta-beta)!, d = c_child - c_parent (upstream docs/math.md
//    "Static geometry-dependent linear maps"; src/static_operators.cpp:257-298).
//    Both depend on (level, child parity class) only: 8 classes per level
//    (src/uniform_fmm.cpp:457-500).
//  - Normalised M2L matrix T^(t)[beta][alpha] = D^{alpha+beta} G(t) for the
//    integer translation t = (target - source) box coordinates
//    (src/static_operators.cpp:159-184, src/uniform_fmm.cpp:502-625); the level
//    scalings D_M = w^-|alpha|, D_L = w^-(|beta|+1) with w = 2^-level in
//    normalised units are exact powers of two applied in the kernels.
//  - D^gamma G is produced by the Cartesian recurrence for the Taylor
//    coefficients of 1/|R| (our own method; upstream uses Taylor-jet
//    arithmetic, src/taylor_jet.cpp:68-148); both give the same derivatives,
//    which the tests check against the reference's matrices.
#include <unistd.h>

#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <stdexcept>
#include <string>
#include <vector>

#include "fmm_internal.hpp"

namespace cdfmm_b200 {

namespace {

struct BasisTable {
  int p;
  std::vector<int> ax, ay, az;
  explicit BasisTable(int order) : p(order) {
    for (int d = 0; d <= order; ++d)
      for (int a = 0; a <= d; ++a)
        for (int b = 0; a + b <= d; ++b) {
          ax.push_back(a);
          ay.push_back(b);
          az.push_back(d - a - b);
        }
  }
  int size() const { return static_cast<int>(ax.size()); }
  static int rank(int a, int b, int c) {
    const int d = a + b + c;
    return d * (d + 1) * (d + 2) / 6 + a * (d + 1) - a * (a - 1) / 2 + b;
  }
};

long double ld_factorial(int k) {
  long double v = 1.0L;
  for (int i = 2; i <= k; ++i) v *= i;
  return v;
}

double monomial_over_factorial(const double d[3], int a, int b, int c) {
  return std::pow(d[0], a) * std::pow(d[1], b) * std::pow(d[2], c) /
         static_cast<double>(ld_factorial(a) * ld_factorial(b) * ld_factorial(c));
}

} // namespace

std::vector<double> laplace_derivatives(int order, const double R[3]) {
  const BasisTable B(order);
  const int m = B.size();
  std::vector<long double> a(static_cast<std::size_t>(m), 0.0L);
  const long double x = R[0], y = R[1], z = R[2];
  const long double r2 = x * x + y * y + z * z;
  if (r2 == 0.0L) throw std::invalid_argument("laplace_derivatives: R must be nonzero");
  a[0] = 1.0L / std::sqrt(r2);
  for (int i = 1; i < m; ++i) {
    const int gx = B.ax[i], gy = B.ay[i], gz = B.az[i];
    const int g = gx + gy + gz;
    long double s1 = 0.0L, s2 = 0.0L;
    if (gx >= 1) s1 += x * a[BasisTable::rank(gx - 1, gy, gz)];
    if (gy >= 1) s1 += y * a[BasisTable::rank(gx, gy - 1, gz)];
    if (gz >= 1) s1 += z * a[BasisTable::rank(gx, gy, gz - 1)];
    if (gx >= 2) s2 += a[BasisTable::rank(gx - 2, gy, gz)];
    if (gy >= 2) s2 += a[BasisTable::rank(gx, gy - 2, gz)];
    if (gz >= 2) s2 += a[BasisTable::rank(gx, gy, gz - 2)];
    a[i] = -((2 * g - 1) * s1 + (g - 1) * s2) / (g * r2);
  }
  const long double inv4pi = 1.0L / (4.0L * 3.141592653589793238462643383279502884L);
  std::vector<double> out(static_cast<std::size_t>(m));
  for (int i = 0; i < m; ++i)
    out[i] = static_cast<double>(a[i] * ld_factorial(B.ax[i]) * ld_factorial(B.ay[i]) *
                                 ld_factorial(B.az[i]) * inv4pi);
  return out;
}

HostOperators build_host_operators(int p, int depth, int m2l_ld_multiple) {
  HostOperators ops;
  const BasisTable B(p);
  ops.p = p;
  ops.n = B.size();
  ops.depth = depth;
  ops.ax = B.ax;
  ops.ay = B.ay;
  ops.az = B.az;
  const int n = ops.n;

  // Pair lists.  M2M: out alpha <- sum_{g <= alpha} c_g * in(alpha - g).
  // L2L: out beta <- sum_{|beta + g| <= p} c_g * in(beta + g).
  ops.m2m_off.assign(static_cast<std::size_t>(n) + 1, 0);
  ops.l2l_off.assign(static_cast<std::size_t>(n) + 1, 0);
  for (int a = 0; a < n; ++a) {
    for (int g = 0; g < n; ++g) {
      if (B.ax[g] <= B.ax[a] && B.ay[g] <= B.ay[a] && B.az[g] <= B.az[a]) {
        ops.m2m_pair_g.push_back(g);
        ops.m2m_pair_in.push_back(
            BasisTable::rank(B.ax[a] - B.ax[g], B.ay[a] - B.ay[g], B.az[a] - B.az[g]));
      }
      const int sx = B.ax[a] + B.ax[g], sy = B.ay[a] + B.ay[g], sz = B.az[a] + B.az[g];
      if (sx + sy + sz <= p) {
        ops.l2l_pair_g.push_back(g);
        ops.l2l_pair_in.push_back(BasisTable::rank(sx, sy, sz));
      }
    }
    ops.m2m_off[a + 1] = static_cast<int>(ops.m2m_pair_g.size());
    ops.l2l_off[a + 1] = static_cast<int>(ops.l2l_pair_g.size());
  }

  // Shift coefficients per (level, child class) in normalised units: the
  // child half width at level l is 2^-(l+1) (root width 1); child offset from
  // its parent is +-half width per axis by the class bits (x=1, y=2, z=4).
  ops.m2m_coef.assign(static_cast<std::size_t>(depth + 1) * 8 * n, 0.0F);
  ops.l2l_coef.assign(static_cast<std::size_t>(depth + 1) * 8 * n, 0.0F);
  for (int level = 1; level <= depth; ++level) {
    const double h = std::ldexp(1.0, -(level + 1));
    for (int c = 0; c < 8; ++c) {
      const double off[3] = {(c & 1) ? h : -h, (c & 2) ? h : -h, (c & 4) ? h : -h};
      const double to_parent[3] = {-off[0], -off[1], -off[2]};
      for (int g = 0; g < n; ++g) {
        const std::size_t at = (static_cast<std::size_t>(level) * 8 + c) * n + g;
        ops.m2m_coef[at] = static_cast<float>(monomial_over_factorial(to_parent, B.ax[g], B.ay[g], B.az[g]));
        ops.l2l_coef[at] = static_cast<float>(monomial_over_factorial(off, B.ax[g], B.ay[g], B.az[g]));
      }
    }
  }

  // Normalised M2L matrices for the 7^3 stencil (near slots left zero).
  ops.m2l_ld = round_up(n, m2l_ld_multiple);
  if (depth >= 2) {
    ops.m2l_T64 = m2l_matrices(p);
    ops.m2l_T = m2l_matrices_fp32(p, ops.m2l_ld, ops.m2l_T64);
  }
  return ops;
}

namespace {

std::mutex g_operator_mutex;
std::map<int, std::shared_ptr<const std::vector<double>>> g_m2l64;
std::map<std::pair<int, int>, std::shared_ptr<const std::vector<float>>> g_m2l32;

constexpr char kCacheMagic[8] = {'C', 'D', 'F', 'M', 'M', 'M', '2', 'L'};
constexpr uint32_t kCacheVersion = 1;

struct CacheHeader {
  char magic[8];
  uint32_t version;
  int32_t order;
  int32_t n;
  uint32_t reserved;
  uint64_t checksum; // FNV-1a 64 of the matrix bytes
};

uint64_t fnv1a(const void *data, std::size_t bytes) {
  const unsigned char *b = static_cast<const unsigned char *>(data);
  uint64_t h = 1469598103934665603ULL;
  for (std::size_t i = 0; i < bytes; ++i) {
    h ^= b[i];
    h *= 1099511628211ULL;
  }
  return h;
}

std::string cache_file(int p) {
  const char *dir = std::getenv("CDFMM_B200_OPERATOR_CACHE");
  if (dir == nullptr || *dir == '\0') return std::string();
  return std::string(dir) + "/m2l_p" + std::to_string(p) + ".bin";
}

bool read_cache(const std::string &path, int p, int n, std::vector<double> &out) {
  std::FILE *f = std::fopen(path.c_str(), "rb");
  if (f == nullptr) return false;
  CacheHeader h{};
  const std::size_t count = static_cast<std::size_t>(343) * n * n;
  out.assign(count, 0.0);
  bool ok = std::fread(&h, sizeof h, 1, f) == 1 && std::memcmp(h.magic, kCacheMagic, 8) == 0 &&
            h.version == kCacheVersion && h.order == p && h.n == n &&
            std::fread(out.data(), sizeof(double), count, f) == count;
  if (ok) {
    char extra;
    ok = std::fread(&extra, 1, 1, f) == 0 && fnv1a(out.data(), count * sizeof(double)) == h.checksum;
  }
  std::fclose(f);
  if (!ok) out.clear();
  return ok;
}

// Writes the file under a temporary name and renames it into place, so a
// reader never sees a partial file; failures leave no file and are ignored.
void write_cache(const std::string &path, int p, int n, const std::vector<double> &T) {
  const std::string tmp = path + ".tmp." + std::to_string(static_cast<long>(getpid()));
  std::FILE *f = std::fopen(tmp.c_str(), "wb");
  if (f == nullptr) return;
  CacheHeader h{};
  std::memcpy(h.magic, kCacheMagic, 8);
  h.version = kCacheVersion;
  h.order = p;
  h.n = n;
  h.checksum = fnv1a(T.data(), T.size() * sizeof(double));
  const bool ok = std::fwrite(&h, sizeof h, 1, f) == 1 && std::fwrite(T.data(), sizeof(double), T.size(), f) == T.size();
  const bool closed = std::fclose(f) == 0;
  if (!ok || !closed || std::rename(tmp.c_str(), path.c_str()) != 0) std::remove(tmp.c_str());
}

std::vector<double> compute_m2l_matrices(int p) {
  const BasisTable B(p);
  const int n = B.size();
  std::vector<double> T64(static_cast<std::size_t>(343) * n * n, 0.0);
  for (int tx = -3; tx <= 3; ++tx)
    for (int ty = -3; ty <= 3; ++ty)
      for (int tz = -3; tz <= 3; ++tz) {
        if (std::abs(tx) <= 1 && std::abs(ty) <= 1 && std::abs(tz) <= 1) continue;
        const double R[3] = {static_cast<double>(tx), static_cast<double>(ty), static_cast<double>(tz)};
        const std::vector<double> deriv = laplace_derivatives(2 * p, R);
        const int slot = (tx + 3) * 49 + (ty + 3) * 7 + (tz + 3);
        double *T = T64.data() + static_cast<std::size_t>(slot) * n * n;
        for (int a = 0; a < n; ++a)
          for (int b = 0; b < n; ++b)
            T[static_cast<std::size_t>(a) * n + b] =
                deriv[BasisTable::rank(B.ax[a] + B.ax[b], B.ay[a] + B.ay[b], B.az[a] + B.az[b])];
      }
  return T64;
}

} // namespace

std::shared_ptr<const std::vector<double>> m2l_matrices(int p, OperatorSource *source) {
  std::lock_guard<std::mutex> lock(g_operator_mutex);
  auto it = g_m2l64.find(p);
  if (it != g_m2l64.end()) {
    if (source) *source = OperatorSource::Process;
    return it->second;
  }
  const int n = BasisTable(p).size();
  const std::string path = cache_file(p);
  auto T = std::make_shared<std::vector<double>>();
  if (!path.empty() && read_cache(path, p, n, *T)) {
    if (source) *source = OperatorSource::Disk;
  } else {
    *T = compute_m2l_matrices(p);
    if (!path.empty()) write_cache(path, p, n, *T);
    if (source) *source = OperatorSource::Computed;
  }
  g_m2l64[p] = T;
  return T;
}

// FP32 copy of the matrices with rows padded to `ld` (zero padding).
std::shared_ptr<const std::vector<float>> m2l_matrices_fp32(int p, int ld,
                                                            const std::shared_ptr<const std::vector<double>> &T64) {
  std::lock_guard<std::mutex> lock(g_operator_mutex);
  auto it = g_m2l32.find({p, ld});
  if (it != g_m2l32.end()) return it->second;
  const int n = BasisTable(p).size();
  auto T = std::make_shared<std::vector<float>>(static_cast<std::size_t>(343) * n * ld, 0.0F);
  for (std::size_t sa = 0; sa < static_cast<std::size_t>(343) * n; ++sa)
    for (int b = 0; b < n; ++b) (*T)[sa * ld + b] = static_cast<float>((*T64)[sa * n + b]);
  g_m2l32[{p, ld}] = T;
  return T;
}

} // namespace cdfmm_b200
