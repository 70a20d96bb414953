#include "host_fft.h"

#include <cmath>

namespace cuvhs {
namespace {

int smallest_factor(int n) {
  for (int p : {4, 2, 3, 5, 7})
    if (n % p == 0) return p;
  for (int p = 11; (long long)p * p <= n; p += 2)
    if (n % p == 0) return p;
  return n;
}

// out[0..n) = DFT of in[0], in[stride], ... ; roots[t] = e^{sign 2 pi i t / N0}, step = N0 / n.
void rec(const cd* in, int stride, cd* out, int n, const std::vector<cd>& roots, int step) {
  if (n == 1) {
    out[0] = in[0];
    return;
  }
  int p = smallest_factor(n);
  int m = n / p;
  for (int r = 0; r < p; r++) rec(in + (size_t)r * stride, stride * p, out + (size_t)r * m, m, roots, step * p);
  std::vector<cd> tmp(p);
  const int N0 = (int)roots.size();
  for (int k = 0; k < m; k++) {
    for (int q = 0; q < p; q++) {
      cd acc = 0.0;
      const int kk = k + m * q;
      for (int r = 0; r < p; r++) {
        long long e = ((long long)r * kk) % n;
        acc += out[(size_t)r * m + k] * roots[(size_t)((e * step) % N0)];
      }
      tmp[q] = acc;
    }
    for (int q = 0; q < p; q++) out[(size_t)q * m + k] = tmp[q];
  }
}

}  // namespace

std::vector<cd> host_dft(const std::vector<cd>& x, int sign) {
  const int n = (int)x.size();
  std::vector<cd> roots(n), out(n);
  for (int t = 0; t < n; t++) {
    double a = (double)sign * 2.0 * M_PI * (double)t / (double)n;
    roots[t] = cd(std::cos(a), std::sin(a));
  }
  if (n > 0) rec(x.data(), 1, out.data(), n, roots, 1);
  return out;
}

}  // namespace cuvhs
