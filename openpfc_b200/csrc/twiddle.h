// twiddle.h -- host-side FP64 twiddle tables shared by the library's entry points.
#pragma once
#include <cmath>
#include <vector>

namespace opfc {

// cos/sin(2 pi k / n) with octant reduction so that quarter turns are exact.
inline void unit_root_host(long k, long n, double *c, double *s) {
  const double pi = 3.14159265358979323846264338327950288;
  k %= n;
  if (k < 0) k += n;
  if (n % 8 == 0) {
    const long oct = (8 * k) / n;
    const long rem = k - oct * (n / 8);
    const double a = 2.0 * pi * (double)rem / (double)n;
    const double ca = std::cos(a), sa = std::sin(a);
    const double r2 = 0.70710678118654752440084436210484903928;
    double cc, ss;
    switch (oct) {
      case 0: cc = ca; ss = sa; break;
      case 1: cc = r2 * (ca - sa); ss = r2 * (ca + sa); break;
      case 2: cc = -sa; ss = ca; break;
      case 3: cc = -r2 * (ca + sa); ss = r2 * (ca - sa); break;
      case 4: cc = -ca; ss = -sa; break;
      case 5: cc = -r2 * (ca - sa); ss = -r2 * (ca + sa); break;
      case 6: cc = sa; ss = -ca; break;
      default: cc = r2 * (ca + sa); ss = -r2 * (ca - sa); break;
    }
    *c = cc;
    *s = ss;
    return;
  }
  if (4 * k == n) { *c = 0; *s = 1; return; }
  if (2 * k == n) { *c = -1; *s = 0; return; }
  if (4 * k == 3 * n) { *c = 0; *s = -1; return; }
  const double a = 2.0 * pi * (double)k / (double)n;
  *c = std::cos(a);
  *s = std::sin(a);
}

// tw[k] = exp(-2 pi i k / n), k = 0..n-1, interleaved (re, im), FP64.
inline std::vector<double> twiddle_table(int n) {
  std::vector<double> d(2 * (size_t)n);
  for (int k = 0; k < n; ++k) {
    double c, s;
    unit_root_host(k, n, &c, &s);
    d[2 * k] = c;
    d[2 * k + 1] = -s;
  }
  return d;
}

}  // namespace opfc
