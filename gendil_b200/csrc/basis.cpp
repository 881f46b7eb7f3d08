#include "basis.h"

#include <algorithm>
#include <cmath>
#include <utility>

namespace dgop {

namespace {

// P_n(x) and P_{n-1}(x) by the three-term recurrence.
void legendre(int n, long double x, long double& pn, long double& pnm1) {
  long double a = 1.0L, b = x;
  if (n == 0) {
    pn = 1.0L;
    pnm1 = 0.0L;
    return;
  }
  for (int k = 2; k <= n; ++k) {
    const long double c = ((2 * k - 1) * x * b - (k - 1) * a) / k;
    a = b;
    b = c;
  }
  pn = b;
  pnm1 = a;
}

// P_n'(x) for |x| < 1 from (x^2 - 1) P_n' = n (x P_n - P_{n-1}).
long double legendre_deriv(int n, long double x, long double pn, long double pnm1) {
  return n * (x * pn - pnm1) / (x * x - 1.0L);
}

}  // namespace

bool gauss_points(int kind, int n, double* x, double* w) {
  if (n < 1 || n > 8) return false;
  if (n == 1) {
    x[0] = 0.5;
    w[0] = 1.0;
    return true;
  }
  const long double pi = 3.141592653589793238462643383279502884L;
  std::pair<long double, long double> pw[8];
  if (kind == 1) {
    for (int i = 0; i < n; ++i) {
      long double r = std::cos(pi * (i + 0.75L) / (n + 0.5L));
      for (int it = 0; it < 64; ++it) {
        long double p, q;
        legendre(n, r, p, q);
        const long double step = p / legendre_deriv(n, r, p, q);
        r -= step;
        if (std::fabs(step) < 1e-30L) break;
      }
      long double p, q;
      legendre(n, r, p, q);
      const long double dp = legendre_deriv(n, r, p, q);
      pw[i] = {r, 2.0L / ((1.0L - r * r) * dp * dp)};
    }
  } else {
    const int m = n - 1;
    pw[0].first = -1.0L;
    pw[n - 1].first = 1.0L;
    for (int i = 1; i < n - 1; ++i) {
      long double r = -std::cos(pi * i / m);
      for (int it = 0; it < 64; ++it) {
        long double p, q;
        legendre(m, r, p, q);
        const long double d1 = legendre_deriv(m, r, p, q);
        const long double d2 = (2.0L * r * d1 - m * (m + 1.0L) * p) / (1.0L - r * r);
        const long double step = d1 / d2;
        r -= step;
        if (std::fabs(step) < 1e-30L) break;
      }
      pw[i].first = r;
    }
    for (int i = 0; i < n; ++i) {
      long double p, q;
      legendre(m, pw[i].first, p, q);
      pw[i].second = 2.0L / ((long double)n * m * p * p);
    }
  }
  std::sort(pw, pw + n, [](const auto& a, const auto& b) { return a.first < b.first; });
  for (int i = 0; i < n; ++i) {
    x[i] = (double)(0.5L * (pw[i].first + 1.0L));
    w[i] = (double)(0.5L * pw[i].second);
  }
  if (kind == 0) {
    x[0] = 0.0;
    x[n - 1] = 1.0;
  }
  return true;
}

double lagrange_value(const double* nodes, int n, int j, double x) {
  double num = 1.0, den = 1.0;
  for (int i = 0; i < n; ++i) {
    if (i == j) continue;
    num *= (x - nodes[i]);
    den *= (nodes[j] - nodes[i]);
  }
  return num / den;
}

double lagrange_grad(const double* nodes, int n, int j, double x) {
  double sum = 0.0;
  for (int i = 0; i < n; ++i) {
    if (i == j) continue;
    double num = 1.0, den = nodes[j] - nodes[i];
    for (int k = 0; k < n; ++k) {
      if (k == i || k == j) continue;
      num *= (x - nodes[k]);
      den *= (nodes[j] - nodes[k]);
    }
    sum += num / den;
  }
  return sum;
}

}  // namespace dgop
