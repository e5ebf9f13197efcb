#include "tables.hpp"

#include <stdexcept>

namespace ffb {

static const long double kPiL = 3.141592653589793238462643383279502884L;

cld unit_root(int64_t m, int64_t n, int sign) {
  m %= n;
  if (m < 0) m += n;
  // exact values at the quarter points
  if ((4 * m) % n == 0) {
    int q = (int)((4 * m) / n);
    static const long double c[4] = {1, 0, -1, 0}, s[4] = {0, 1, 0, -1};
    return cld(c[q], sign * s[q]);
  }
  long double sn, cs;
  sincosl(2.0L * kPiL * (long double)m / (long double)n, &sn, &cs);
  return cld(cs, sign * sn);
}

cld chirp_value(int64_t k, int64_t n, int sign) {
  int64_t red = (int64_t)(((__int128)k * k) % (2 * n));
  long double sn, cs;
  sincosl(kPiL * (long double)red / (long double)n, &sn, &cs);
  return cld(cs, sign * sn);
}

// Plain complex product (std::complex's operator* takes the slow path that
// handles infinities and NaNs, which these finite tables never hold).
template <typename R>
static inline std::complex<R> mul(const std::complex<R> &a, const std::complex<R> &b) {
  return std::complex<R>(a.real() * b.real() - a.imag() * b.imag(), a.real() * b.imag() + a.imag() * b.real());
}

static int64_t smallest_factor(int64_t n) {
  if (n % 4 == 0) return 4;
  for (int64_t d = 2; d * d <= n; ++d)
    if (n % d == 0) return d;
  return n;
}

// Mixed-radix decimation in time over the top-level length N's root table
// w[e] = W_N^e: a sub-transform of length n at stride `stride` reads its roots
// as w[e * N / n].  out[k + m q] = sum_j W_n^{jk} W_r^{jq} Y_j[k], r <= 64;
// scr is scratch aligned with out.
template <typename R>
static void fft_rec(const std::complex<R> *x, int64_t n, int64_t stride, std::complex<R> *out, std::complex<R> *scr,
                    const std::vector<std::complex<R>> &w, int64_t N) {
  using C = std::complex<R>;
  if (n == 1) {
    out[0] = x[0];
    return;
  }
  const int64_t r = smallest_factor(n), m = n / r, step = N / n, rstep = N / r;
  for (int64_t j = 0; j < r; ++j) fft_rec(x + j * stride, m, stride * r, out + j * m, scr + j * m, w, N);
  C t[64], wr[64];
  for (int64_t q = 0; q < r; ++q) wr[q] = w[(size_t)(q * rstep)];
  for (int64_t k = 0; k < m; ++k) {
    for (int64_t j = 0; j < r; ++j) t[j] = mul(out[j * m + k], w[(size_t)(j * k * step)]);
    for (int64_t q = 0; q < r; ++q) {
      C acc = t[0];
      for (int64_t j = 1, e = q; j < r; ++j, e = (e + q) % r) acc += mul(t[j], wr[e]);
      scr[k + m * q] = acc;
    }
  }
  for (int64_t i = 0; i < n; ++i) out[i] = scr[i];
}

// Bluestein in long double for a length with a prime factor above 64.
static void bluestein_ld(std::vector<cld> &x, int sign) {
  const int64_t n = (int64_t)x.size();
  int64_t m = 1;
  while (m < 2 * n - 1) m <<= 1;
  std::vector<cld> a(m), b(m);
  for (int64_t k = 0; k < n; ++k) {
    cld c = chirp_value(k, n, sign);
    a[k] = mul(x[k], c);
    b[k] = std::conj(c);
    if (k) b[m - k] = std::conj(c);
  }
  host_fft(a, -1);
  host_fft(b, -1);
  for (int64_t k = 0; k < m; ++k) a[k] = mul(a[k], b[k]);
  host_fft(a, +1);
  for (int64_t k = 0; k < n; ++k) x[k] = mul(a[k] / (long double)m, chirp_value(k, n, sign));
}

// Above this length the mixed-radix recursion runs in double (its results
// are rounded to at most double precision anyway; the recursion's error
// stays a few ulp times log n).
constexpr int64_t kLongDoubleMaxN = 4096;

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
  if (n <= kLongDoubleMaxN) {
    std::vector<cld> w((size_t)n), out((size_t)n), scr((size_t)n);
    for (int64_t e = 0; e < n; ++e) w[(size_t)e] = unit_root(e, n, sign);
    fft_rec(x.data(), n, 1, out.data(), scr.data(), w, n);
    x.swap(out);
    return;
  }
  using cd = std::complex<double>;
  std::vector<cd> xd((size_t)n), w((size_t)n), out((size_t)n), scr((size_t)n);
  const double two_pi = 6.283185307179586476925286766559;
  for (int64_t e = 0; e < n; ++e) {
    const double a = two_pi * (double)e / (double)n;
    w[(size_t)e] = cd(std::cos(a), sign * std::sin(a));
    xd[(size_t)e] = cd((double)x[(size_t)e].real(), (double)x[(size_t)e].imag());
  }
  fft_rec(xd.data(), n, 1, out.data(), scr.data(), w, n);
  for (int64_t e = 0; e < n; ++e) x[(size_t)e] = cld(out[(size_t)e].real(), out[(size_t)e].imag());
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
