// Plan-time tables, computed on the host in long double and rounded once to
// the working precision.  The reference builds the same tables in double on
// the host (src/codegen/tables.cpp); the Bluestein/Rader kernel spectra it
// computes on the device in working precision (src/exec/raw_nodes.cpp:140-151)
// are computed here in long double instead.
#pragma once

#include <complex>
#include <cstdint>
#include <vector>

namespace ffb {

using cld = std::complex<long double>;

// exp(sign * 2*pi*i * m / n) with m reduced exactly mod n.
cld unit_root(int64_t m, int64_t n, int sign);

// exp(sign * i*pi * (k^2 mod 2n) / n): Bluestein chirp with the square reduced
// in exact integers (src/codegen/tables.cpp:149-216).
cld chirp_value(int64_t k, int64_t n, int sign);

// In-place DFT of arbitrary length, long double, sign -1 forward / +1 inverse
// (unnormalized).  Mixed radix for small prime factors, Bluestein otherwise.
void host_fft(std::vector<cld> &x, int sign);

// DIF output position of natural index k for radices r[0..S-1]:
// k = sum d_s * (r0..r(s-1))  ->  p = sum d_s * L / (r0..rs).
int64_t dif_position(int64_t k, const std::vector<int> &radices);

}  // namespace ffb
