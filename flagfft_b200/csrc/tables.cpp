#include "tables.hpp"

#include <stdexcept>

namespace ffb {

static const long double kPiL = 3.141592653589793238462643383279502884L;

cld unit_root(int64_t m, int64_t n, int sign) {
  m %= n;
  if (m < 0) m += n;
  // exact values at the quarter points; elsewhere reduce to the first octant
  if ((4 * m) % n == 0) {
    int q = (int)((4 * m) / n);
    static const long double c[4] = {1, 0, -1, 0}, s[4] = {0, 1, 0, -1};
    return cld(c[q], sign * s[q]);
  }
  long double a = 2.0L * kPiL * (long double)m / (long double)n;
  return cld(cosl(a), sign * sinl(a));
}

cld chirp_value(int64_t k, int64_t n, int sign) {
  int64_t red = (int64_t)(((__int128)k * k) % (2 * n));
  long double a = kPiL * (long double)red / (long double)n;
  return cld(cosl(a), sign * sinl(a));
}

static void fft_rec(cld *x, int64_t n, int64_t stride, cld *out, int sign, std::vector<cld> &scratch);

static int64_t smallest_factor(int64_t n) {
  for (int64_t d = 2; d * d <= n; ++d)
    if (n % d == 0) return d;
  return n;
}

// Bluestein in long double for a length with a large prime factor.
static void bluestein_ld(std::vector<cld> &x, int sign) {
  const int64_t n = (int64_t)x.size();
  int64_t m = 1;
  while (m < 2 * n - 1) m <<= 1;
  std::vector<cld> a(m), b(m);
  for (int64_t k = 0; k < n; ++k) {
    cld c = chirp_value(k, n, sign);
    a[k] = x[k] * c;
    b[k] = std::conj(c);
    if (k) b[m - k] = std::conj(c);
  }
  host_fft(a, -1);
  host_fft(b, -1);
  for (int64_t k = 0; k < m; ++k) a[k] *= b[k];
  host_fft(a, +1);
  for (int64_t k = 0; k < n; ++k) x[k] = a[k] / (long double)m * chirp_value(k, n, sign);
}

static void fft_rec(cld *x, int64_t n, int64_t stride, cld *out, int sign, std::vector<cld> &scratch) {
  if (n == 1) {
    out[0] = x[0];
    return;
  }
  int64_t r = smallest_factor(n);
  int64_t m = n / r;
  // decimation in time: out[k + m q] = sum_j W_n^{jk} W_r^{jq} Y_j[k]
  for (int64_t j = 0; j < r; ++j) fft_rec(x + j * stride, m, stride * r, out + j * m, sign, scratch);
  std::vector<cld> t((size_t)r), y((size_t)r);
  std::vector<cld> wr((size_t)r);
  for (int64_t q = 0; q < r; ++q) wr[(size_t)q] = unit_root(q, r, sign);
  std::vector<cld> res((size_t)n);
  for (int64_t k = 0; k < m; ++k) {
    for (int64_t j = 0; j < r; ++j) t[(size_t)j] = out[j * m + k] * unit_root(j * k, n, sign);
    for (int64_t q = 0; q < r; ++q) {
      cld acc = 0;
      for (int64_t j = 0; j < r; ++j) acc += t[(size_t)j] * wr[(size_t)((j * q) % r)];
      res[(size_t)(k + m * q)] = acc;
    }
  }
  for (int64_t i = 0; i < n; ++i) out[i] = res[(size_t)i];
}

void host_fft(std::vector<cld> &x, int sign) {
  const int64_t n = (int64_t)x.size();
  if (n <= 1) return;
  // largest prime factor decides between mixed radix and Bluestein
  int64_t t = n, big = 1;
  for (int64_t d = 2; d * d <= t; ++d)
    while (t % d == 0) {
      big = d;
      t /= d;
    }
  if (t > 1) big = std::max(big, t);
  if (big > 64) {
    bluestein_ld(x, sign);
    return;
  }
  std::vector<cld> out((size_t)n), scratch;
  fft_rec(x.data(), n, 1, out.data(), sign, scratch);
  x.swap(out);
}

int64_t dif_position(int64_t k, const std::vector<int> &r) {
  int64_t L = 1;
  for (int v : r) L *= v;
  int64_t p = 0, rem = k, span = L;
  for (size_t s = 0; s < r.size(); ++s) {
    int64_t d = rem % r[s];
    rem /= r[s];
    span /= r[s];
    p += d * span;
  }
  return p;
}

}  // namespace ffb
