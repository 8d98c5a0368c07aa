// tables.cpp -- see tables.h.
#include "tables.h"

#include <cmath>
#include <mutex>

namespace rodv {

namespace {

constexpr double kJacStep = 0.0001;
constexpr double kJacTol = 8.0;
const int kJacSize = (int)(kJacTol / kJacStep) + 1;

template <class T>
int fast_round(T v) {
  return v > T(0) ? (int)(v + T(0.5)) : (int)(v - T(0.5));
}

// log10(10^a + 10^b) by the Jacobian table, evaluated in precision T
// (context.h:66-82).
template <class T>
T log10_sum(T small, T big, const std::vector<T>& jac) {
  if (small > big) std::swap(small, big);
  if (std::isinf(small) || std::isinf(big)) return big;
  const T diff = big - small;
  if (diff >= T(kJacTol)) return big;
  return big + jac[fast_round<T>(diff * T(1.0 / kJacStep))];
}

template <class T>
std::vector<T> match_to_match(const std::vector<T>& jac) {
  std::vector<T> mm(kMmTableSize);
  const double inv_ln10 = 1.0 / std::log(10.0);
  for (int hi = 0, off = 0; hi < 128; off += ++hi) {
    for (int lo = 0; lo <= hi; ++lo) {
      const T s = log10_sum<T>(T(-0.1 * hi), T(-0.1 * lo), jac);
      const double l = std::log1p(-std::fmin(1.0, std::pow(10.0, (double)s))) * inv_ln10;
      mm[off + lo] = T(std::pow(10.0, l));
    }
  }
  return mm;
}

HostPriorTables build() {
  HostPriorTables t;
  std::vector<double> jac_d(kJacSize);
  std::vector<float> jac_f(kJacSize);
  for (int k = 0; k < kJacSize; ++k) {
    jac_d[k] = std::log10(1.0 + std::pow(10.0, -(double)k * kJacStep));
    jac_f[k] = (float)jac_d[k];
  }
  t.mm_d = match_to_match<double>(jac_d);
  t.mm_f = match_to_match<float>(jac_f);
  t.ph2pr_d.resize(128);
  t.ph2pr_f.resize(128);
  for (int q = 0; q < 128; ++q) {
    t.ph2pr_d[q] = std::pow(10.0, -(double)q / 10.0);
    t.ph2pr_f[q] = std::pow(10.f, -(float)q / 10.f);
  }
  return t;
}

}  // namespace

const HostPriorTables& host_prior_tables() {
  static std::once_flag once;
  static HostPriorTables tables;
  std::call_once(once, [] { tables = build(); });
  return tables;
}

}  // namespace rodv
