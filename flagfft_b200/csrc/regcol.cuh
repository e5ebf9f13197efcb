// One transform of the register column pass (regcol.cu): a single codelet
// in registers, one thread per transform.  Shared with the batch kernel.
#pragma once

#include "kernels.cuh"

namespace ffb {

template <typename T, int R, bool INV>
FFB_HD void regcol_transform(const TileArgs<T> &a, long long by, long long g) {
  const cpx<T> *in = reinterpret_cast<const cpx<T> *>(a.in) + by * a.ib + g * a.ig;
  cpx<T> *out = reinterpret_cast<cpx<T> *>(a.out) + by * a.ob + g * a.og;
  cpx<T> v[R];
  if (a.chirp_mode == 1) {
#pragma unroll
    for (int i = 0; i < R; ++i) {
      const long long j = (long long)i * a.cj_e + g * a.cj_g;
      v[i] = j < a.n ? cmul(ldg_c(in + i * a.ii), ldg_c(a.chirp + j)) : mk((T)0, (T)0);
    }
  } else {
#pragma unroll
    for (int i = 0; i < R; ++i) v[i] = ldg_c(in + i * a.ii);
  }
  dft_fixed<R, INV, T>(v);
  if (a.chirp_mode == 2) {
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const long long j = (long long)k * a.cj_e + g * a.cj_g;
      if (j < a.n) out[k * a.ok] = cmul(v[k], ldg_c(a.chirp + j));
    }
  } else if (a.post_twiddle) {
    // output k of transform g times W_N^{g k} = hi[m / split] * lo[m % split]
#pragma unroll
    for (int k = 0; k < R; ++k) {
      const uint32_t m = (uint32_t)(g * k);
      const uint32_t hi = fdiv(m, a.ptw_div);
      cpx<T> t = cmul(ldg_c(a.ptw_hi + hi), ldg_c(a.ptw_lo + (m - hi * a.ptw_div.d)));
      if constexpr (INV) t.y = -t.y;
      out[k * a.ok] = cmul(v[k], t);
    }
  } else {
#pragma unroll
    for (int k = 0; k < R; ++k) out[k * a.ok] = v[k];
  }
}

}  // namespace ffb
