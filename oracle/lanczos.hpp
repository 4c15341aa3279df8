// ORACLE — test infrastructure only.
// Largest eigenvalue of a symmetric positive semi-definite operator by plain
// Lanczos (no re-orthogonalisation; ghost copies do not move the extreme Ritz
// value) with a Sturm-bisection solve of the tridiagonal matrix.  This stands
// in for the Spectra Arnoldi call the reference uses to size the time step
// (Discretization.hpp:7103-7118, tolerance 2e-2), which cannot be reproduced
// without Spectra; parity runs pin the step with `SET step`.
#pragma once
#include <cmath>
#include <cstdint>
#include <functional>
#include <vector>

namespace orc {

inline double tridiag_max_eig(const std::vector<double>& a, const std::vector<double>& b) {
  // a: diagonal (m), b: off-diagonal (m-1).  Bisection on the Sturm count.
  const size_t m = a.size();
  double lo = a[0], hi = a[0];
  for (size_t i = 0; i < m; i++) {
    double r = (i > 0 ? std::fabs(b[i - 1]) : 0) + (i + 1 < m ? std::fabs(b[i]) : 0);
    lo = std::fmin(lo, a[i] - r);
    hi = std::fmax(hi, a[i] + r);
  }
  auto count_below = [&](double x) {
    int c = 0;
    double d = 1;
    for (size_t i = 0; i < m; i++) {
      d = a[i] - x - (i > 0 ? b[i - 1] * b[i - 1] / d : 0);
      if (d == 0) d = 1e-300;
      if (d < 0) c++;
    }
    return c;
  };
  for (int it = 0; it < 200; it++) {
    double mid = 0.5 * (lo + hi);
    if (count_below(mid) >= (int)m) hi = mid;
    else lo = mid;
    if (hi - lo <= 1e-15 * std::fabs(hi)) break;
  }
  return hi;
}

inline double lanczos_max(size_t n, const std::function<void(const double*, double*)>& apply, int max_iter = 300,
                          double tol = 1e-9) {
  std::vector<double> v(n), w(n), vprev(n, 0.0);
  uint64_t s = 0x9E3779B97F4A7C15ull;  // fixed seed: deterministic estimate
  double nrm = 0;
  for (size_t i = 0; i < n; i++) {
    s ^= s << 13; s ^= s >> 7; s ^= s << 17;
    v[i] = (double)(s >> 11) / 9007199254740992.0 - 0.5;
    nrm += v[i] * v[i];
  }
  nrm = std::sqrt(nrm);
  for (auto& x : v) x /= nrm;
  std::vector<double> al, be;
  double beta = 0, last = 0;
  for (int j = 0; j < max_iter && (size_t)j < n; j++) {
    apply(v.data(), w.data());
    double alpha = 0;
    for (size_t i = 0; i < n; i++) alpha += w[i] * v[i];
    for (size_t i = 0; i < n; i++) w[i] -= alpha * v[i] + beta * vprev[i];
    al.push_back(alpha);
    double nb = 0;
    for (size_t i = 0; i < n; i++) nb += w[i] * w[i];
    nb = std::sqrt(nb);
    if (j % 10 == 9 || nb == 0) {
      double cur = tridiag_max_eig(al, be);
      if (nb == 0 || std::fabs(cur - last) <= tol * std::fabs(cur)) return cur;
      last = cur;
    }
    be.push_back(nb);
    beta = nb;
    vprev.swap(v);
    for (size_t i = 0; i < n; i++) v[i] = w[i] / nb;
  }
  be.resize(al.size() - 1);
  return tridiag_max_eig(al, be);
}

}  // namespace orc
