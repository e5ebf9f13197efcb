// On-chip FFT passes for sm_100a.
//
// One kernel template covers every pass that keeps whole transforms in shared
// memory: contiguous rows (1-D batches, 2-D rows), strided column tiles (2-D
// columns, four-step column and row passes), the fused Bluestein and Rader
// chains, and the fused real-to-complex / complex-to-real packing.  Each CTA
// holds W transforms; every element crosses HBM once on the way in and once on
// the way out.
//
// The body (tile_body) is written once against an execution policy: DevX runs
// it as a CUDA thread block; HostX runs the identical code sequentially on the
// CPU with one "thread" and no-op barriers (built only with
// FFB_HOST_EMULATION, for host-side checks of the index arithmetic; never part
// of libflagfft.so).  Sequential execution is exact because every phase's
// iterations touch disjoint shared-memory positions.
#pragma once

#include "kernels.cuh"

#include <algorithm>
#include <cstring>
#include <vector>

namespace ffb {
namespace tile {

template <typename T>
FFB_HD cpx<T> ld_cpx(const void *base, long long idx) {
  return ldg_c(reinterpret_cast<const cpx<T> *>(base) + idx);
}
template <typename T>
FFB_HD T ld_real(const void *base, long long idx) {
  return ldg_v(reinterpret_cast<const T *>(base) + idx);
}
template <typename T>
FFB_HD void st_cpx(void *base, long long idx, cpx<T> v) {
  reinterpret_cast<cpx<T> *>(base)[idx] = v;
}
template <typename T>
FFB_HD void st_real(void *base, long long idx, T v) {
  reinterpret_cast<T *>(base)[idx] = v;
}

// CUDA thread block.
struct DevX {
  int tpt;
  FFB_HD int tid() const {
#ifdef __CUDA_ARCH__
    return threadIdx.x;
#else
    return 0;
#endif
  }
  FFB_HD int nthreads() const {
#ifdef __CUDA_ARCH__
    return blockDim.x;
#else
    return 1;
#endif
  }
  FFB_HD void sync() const {
#ifdef __CUDA_ARCH__
    __syncthreads();
#endif
  }
  int wfast;
  // Runs f(slot, tid-in-slot, threads-per-slot) for this thread's transform.
  // Column tiles put consecutive transforms on consecutive threads.
  // f has one call site (its barriers must be the same instructions for
  // every thread of a warp).
  template <class F>
  FFB_HD void per_slot(int W, F f) const {
    const int t = tid();
    const int slot = wfast ? t % W : t / tpt;
    f(slot, wfast ? t / W : t - slot * tpt, tpt);
  }
};

// Sequential host execution of one block.
struct HostX {
  FFB_HD int tid() const { return 0; }
  FFB_HD int nthreads() const { return 1; }
  FFB_HD void sync() const {}
  template <class F>
  FFB_HD void per_slot(int W, F f) const {
    for (int s = 0; s < W; ++s) f(s, 0, 1);
  }
};

// A value with the offset it goes to.
template <typename T>
struct ElemAt {
  cpx<T> v;
  int at;
};

// Splits a flat element counter e over (transform w, element i) of a CTA tile.
FFB_HD void split_elem(int e, int W, int Lx, int wfast, const FastDiv &wdiv, const FastDiv &ldiv, int &w, int &i) {
  if (wfast) {
    i = (int)fdiv((uint32_t)e, wdiv);
    w = e - i * W;
  } else {
    w = (int)fdiv((uint32_t)e, ldiv);
    i = e - w * Lx;
  }
}

template <typename T, int KIND, int IO, class X>
FFB_HD void tile_body(const TileArgs<T> &a, long long bx, long long by, cpx<T> *sm, const X &x) {
  constexpr int G = Swz<T>::G;
  const int L = a.core.L;                // core (buffer) length
  const int Lp = Swz<T>::padded(L) + G;  // + a spare group: Rader's x0 / X0 slots
  const int W = a.W;
  const long long b = by;
  const long long g0 = bx * W;
  constexpr bool real_in = IO == 1 || IO == 3 || IO == 5;
  constexpr bool real_out = IO == 2 || IO == 4 || IO == 6;
  const void *in = reinterpret_cast<const unsigned char *>(a.in) +
                   b * a.ib * (long long)(real_in ? sizeof(T) : sizeof(cpx<T>));
  void *out = reinterpret_cast<unsigned char *>(a.out) + b * a.ob * (long long)(real_out ? sizeof(T) : sizeof(cpx<T>));
  const int n = a.n;
  const int half_n = n / 2;  // real transforms: n reals, half_n + 1 bins
  const int t0 = x.tid(), nt = x.nthreads();

  // Logical input element i of the core's transform g.
  auto core_input = [&](long long g, int i) FFB_INL -> cpx<T> {
    const long long base = g * a.ig;
    if constexpr (IO == 0 || IO == 6) {
      return ld_cpx<T>(in, base + (long long)i * a.ii);
    } else if constexpr (IO == 1 || IO == 5) {  // z_i = x_2i + i x_2i+1: adjacent reals at i*ii
      T re = ld_real<T>(in, base + (long long)i * a.ii);
      T im = ld_real<T>(in, base + (long long)i * a.ii + 1);
      return mk(re, im);
    } else if constexpr (IO == 3) {  // real x_i, imaginary part 0
      return mk(ld_real<T>(in, base + (long long)i * a.ii), (T)0);
    } else if constexpr (IO == 2) {
      // Z_i = (X_i + conj X_{L-i}) + i (X_i - conj X_{L-i}) W_n^{-i};  Im X_0, Im X_L dropped
      cpx<T> xk = ld_cpx<T>(in, base + (long long)i * a.ii);
      cpx<T> xm = ld_cpx<T>(in, base + (long long)(half_n - i) * a.ii);
      if (i == 0) {
        xk.y = (T)0;
        xm.y = (T)0;
      }
      cpx<T> s = mk(xk.x + xm.x, xk.y - xm.y);
      cpx<T> d = mk(xk.x - xm.x, xk.y + xm.y);
      cpx<T> w = ldg_c(a.rtw + i);
      cpx<T> dw = mk(d.x * w.x + d.y * w.y, d.y * w.x - d.x * w.y);  // d * conj(w)
      return mk(s.x - dw.y, s.y + dw.x);                           // s + i dw
    } else {  // IO == 4: Hermitian expansion of the half spectrum to n points
      const bool mirror = i > half_n;
      cpx<T> v = ld_cpx<T>(in, base + (long long)(mirror ? n - i : i) * a.ii);
      if (mirror) v.y = -v.y;
      if (i == 0 || ((n & 1) == 0 && i == half_n)) v.y = (T)0;
      return v;
    }
  };

  // ---------------------------------------------------------------- load
  {
    const int total = W * L;
    const int nl = (IO == 1 || IO == 2) ? half_n : n;  // Bluestein logical length
    auto produce = [&](int e) FFB_INL -> cpx<T> {
      int w, i;
      split_elem(e, W, L, a.wfast, a.wdiv, a.ldiv, w, i);
      const long long g = g0 + w;
      cpx<T> v = mk((T)0, (T)0);
      if constexpr (KIND == 0) {
        if (a.chirp_mode == 1) {
          const long long j = (long long)i * a.cj_e + g * a.cj_g;
          if (g < a.G && j < n) v = cmul(core_input(g, i), ldg_c(a.chirp + j));
        } else if (g < a.G) {
          v = core_input(g, i);
        }
      } else if constexpr (KIND == 3) {
        if (g < a.G) v = core_input(g, i);
      } else if constexpr (KIND == 1) {
        if (g < a.G && i < nl) v = cmul(core_input(g, i), ldg_c(a.chirp + i));
      } else {  // Rader: a[q] = x[g^-q], q < L = p - 1
        if (g < a.G) v = core_input(g, ldg_v(a.perm_in + i));
      }
      return v;
    };
    auto consume = [&](int e, cpx<T> v) FFB_INL {
      int w, i;
      split_elem(e, W, L, a.wfast, a.wdiv, a.ldiv, w, i);
      if constexpr (KIND == 0) {
        sm[w * Lp + Swz<T>::phys(dit_position(i, a.core))] = v;
      } else {
        sm[w * Lp + Swz<T>::phys(i)] = v;
      }
    };
    chunked_loop<8, cpx<T>>(t0, nt, total, produce, consume);
    if constexpr (KIND == 2) {
      for (int w = t0; w < W; w += nt) {
        const long long g = g0 + w;
        sm[w * Lp + Lp - G] = (g < a.G) ? core_input(g, 0) : mk((T)0, (T)0);  // x0
      }
    }
  }
  x.sync();

  // ---------------------------------------------------------------- core
  auto sync = [&]() FFB_INL { x.sync(); };
  x.per_slot(W, [&](int slot, int tid, int tpt) FFB_INL {
    cpx<T> *buf = sm + slot * Lp;
    if constexpr (KIND == 0) {
      run_dit<T>(buf, a.core, tid, tpt, a.tw, a.inv != 0, sync);
    } else {
      run_dif<T>(buf, a.core, tid, tpt, a.tw, false, sync);
      const cpx<T> *kern = a.kern;
      if constexpr (KIND == 3) kern += (g0 + slot < a.G ? g0 + slot : 0) * a.kern_stride;
      for (int p = tid; p < L; p += tpt) {
        cpx<T> v = buf[Swz<T>::phys(p)];
        if constexpr (KIND == 2) {
          if (p == 0) buf[Lp - G + 1] = v + buf[Lp - G];  // X0 = x0 + sum_q a[q]
        }
        buf[Swz<T>::phys(p)] = cmul(v, ldg_c(kern + p));
      }
      sync();
      run_dit<T>(buf, a.core2, tid, tpt, a.tw2, true, sync);
    }
  });

  // Four-step column passes multiply output k of transform g by W_N^{g k}
  // (forward sign; conjugated for the inverse), g*k < N < 2^31.
  auto post_twiddle = [&](cpx<T> v, long long g, int k) FFB_INL -> cpx<T> {
    if (!a.post_twiddle) return v;
    const uint32_t m = (uint32_t)(g * (long long)k);
    const uint32_t hi = fdiv(m, a.ptw_div);
    const uint32_t lo = m - hi * a.ptw_div.d;
    cpx<T> t = cmul(ldg_c(a.ptw_hi + hi), ldg_c(a.ptw_lo + lo));
    if (a.inv) t.y = -t.y;
    return cmul(v, t);
  };

  // Natural-order output element k of the core's transform in slot w.
  auto out_elem = [&](int w, int k) FFB_INL -> cpx<T> {
    const cpx<T> *bw = sm + w * Lp;
    if constexpr (KIND == 0 || KIND == 3) {
      return bw[Swz<T>::phys(k)];
    } else if constexpr (KIND == 1) {
      return cmul(bw[Swz<T>::phys(k)], ldg_c(a.chirp + k));
    } else {
      if (k == 0) return bw[Lp - G + 1];
      const int q = ldg_v(a.perm_in + L + k);  // log_g(k)
      return bw[Lp - G] + bw[Swz<T>::phys(q)];
    }
  };

  // ---------------------------------------------------------------- store
  // output mapping: consecutive threads take consecutive transforms when a
  // transform's outputs are strided (ok > og), else consecutive elements
  const int ofast = a.ok > a.og ? 1 : 0;
  if constexpr (IO == 0) {
    if constexpr (KIND == 2) {
      // X[g^q] = x0 + conv[q] (scatter by q keeps the reads conflict-free);  X[0] = x0 + sum
      const int total = W * L;
      for (int e = t0; e < total; e += nt) {
        int w, q;
        split_elem(e, W, L, ofast, a.wdiv, a.ldiv, w, q);
        const long long g = g0 + w;
        if (g < a.G) {
          const cpx<T> *bw = sm + w * Lp;
          const int k = ldg_v(a.perm_out + q);
          st_cpx<T>(out, g * a.og + (long long)k * a.ok, post_twiddle(bw[Lp - G] + bw[Swz<T>::phys(q)], g, k));
        }
      }
      for (int w = t0; w < W; w += nt) {
        const long long g = g0 + w;
        if (g < a.G) st_cpx<T>(out, g * a.og, sm[w * Lp + Lp - G + 1]);
      }
    } else {
      const int nout = KIND == 1 ? n : L;
      const int total = W * nout;
      auto produce = [&](int e) FFB_INL -> cpx<T> {
        int w, k;
        split_elem(e, W, nout, ofast, a.wdiv, KIND == 1 ? a.ndiv : a.ldiv, w, k);
        const long long g = g0 + w;
        const long long gc = g < a.G ? g : a.G - 1;
        cpx<T> v = out_elem(w, k);
        if constexpr (KIND == 0) {
          if (a.chirp_mode == 2) {  // Bluestein output: y_j = conv_j * chirp_j, j < n
            const long long j = (long long)k * a.cj_e + gc * a.cj_g;
            return j < n ? cmul(v, ldg_c(a.chirp + j)) : v;
          }
        }
        return post_twiddle(v, gc, k);
      };
      auto consume = [&](int e, cpx<T> v) FFB_INL {
        int w, k;
        split_elem(e, W, nout, ofast, a.wdiv, KIND == 1 ? a.ndiv : a.ldiv, w, k);
        const long long g = g0 + w;
        if (g >= a.G) return;
        if constexpr (KIND == 0) {
          if (a.chirp_mode == 2 && (long long)k * a.cj_e + g * a.cj_g >= n) return;
        }
        st_cpx<T>(out, g * a.og + (long long)k * a.ok, v);
      };
      chunked_loop<8, cpx<T>>(t0, nt, total, produce, consume);
    }
  } else if constexpr (IO == 1) {
    // X_k = E_k + W_n^k O_k,  E = (Z_k + conj Z_{L-k})/2,  O = -i (Z_k - conj Z_{L-k})/2
    const int nbins = half_n + 1;
    const int total = W * nbins;
    for (int e = t0; e < total; e += nt) {
      int w, k;
      if (ofast) {
        k = e / W;
        w = e - k * W;
      } else {
        w = e / nbins;
        k = e - w * nbins;
      }
      const long long g = g0 + w;
      if (g >= a.G) continue;
      cpx<T> zk = out_elem(w, k == half_n ? 0 : k);
      cpx<T> zm = out_elem(w, k == 0 ? 0 : half_n - k);
      cpx<T> ev = mk((zk.x + zm.x) * (T)0.5, (zk.y - zm.y) * (T)0.5);
      cpx<T> od = mk((zk.y + zm.y) * (T)0.5, (zm.x - zk.x) * (T)0.5);
      st_cpx<T>(out, g * a.og + (long long)k * a.ok, ev + cmul(ldg_c(a.rtw + k), od));
    }
  } else if constexpr (IO == 2 || IO == 6) {
    // x_2j = Re z_j, x_2j+1 = Im z_j: adjacent reals at j*ok
    const int cnt = IO == 2 ? half_n : L;
    const int total = W * cnt;
    for (int e = t0; e < total; e += nt) {
      int w, j;
      split_elem(e, W, cnt, ofast, a.wdiv, IO == 2 ? a.hdiv : a.ldiv, w, j);
      const long long g = g0 + w;
      if (g >= a.G) continue;
      cpx<T> z = out_elem(w, j);
      st_real<T>(out, g * a.og + (long long)j * a.ok, z.x);
      st_real<T>(out, g * a.og + (long long)j * a.ok + 1, z.y);
    }
  } else if constexpr (IO == 5) {
    const int total = W * L;
    for (int e = t0; e < total; e += nt) {
      int w, k;
      split_elem(e, W, L, ofast, a.wdiv, a.ldiv, w, k);
      const long long g = g0 + w;
      if (g < a.G) st_cpx<T>(out, g * a.og + (long long)k * a.ok, post_twiddle(out_elem(w, k), g, k));
    }
  } else if constexpr (IO == 3) {
    const int nbins = half_n + 1;
    const int total = W * nbins;
    for (int e = t0; e < total; e += nt) {
      int w, k;
      if (ofast) {
        k = e / W;
        w = e - k * W;
      } else {
        w = e / nbins;
        k = e - w * nbins;
      }
      const long long g = g0 + w;
      if (g < a.G) st_cpx<T>(out, g * a.og + (long long)k * a.ok, out_elem(w, k));
    }
  } else {  // IO == 4
    const int total = W * n;
    for (int e = t0; e < total; e += nt) {
      int w, k;
      split_elem(e, W, n, ofast, a.wdiv, a.ndiv, w, k);
      const long long g = g0 + w;
      if (g < a.G) st_real<T>(out, g * a.og + (long long)k * a.ok, out_elem(w, k).x);
    }
  }
}

// Stockham ping-pong pass for C2C tiles.  A coalesced load phase fills
// buffer 0 of every slot (natural order, chirp / permutation / zero padding
// applied); all stages run shared -> shared (one code path per radix, warm in the
// instruction cache after the first stage); a coalesced store phase writes
// the result (unchirp / scatter / four-step twiddle applied).
// Slot layout: two buffers of pp_size(L) and three spare elements (Rader x0,
// X0, and one so the slot stride is odd: consecutive slots then fall in
// different banks).  Offsets inside a CTA's tile are 32-bit.
template <typename T>
FFB_HD int pp_slot_len(int L) {
  return 2 * pp_size(L) + 3;
}

// INV: direction of a Dit core (KIND 0); convolutions (KIND 1-3) run their
// forward core and inverse core2 whatever INV is.  Stages: the stage runner
// (GenericStages, or FixedStagesRunner for a compile-time radix sequence
// that core and core2 both have).
template <typename T, int KIND, bool INV, class X, class Stages = GenericStages<T>>
FFB_HD void tile_body_pp(const TileArgs<T> &a, long long bx, long long by, cpx<T> *sm, const X &x,
                         const Stages &stages = Stages{}) {
  const int L = a.core.L;
  const int Lq = pp_size(L);
  const int slot_len = pp_slot_len<T>(L);
  const int W = a.W;
  const long long g0 = bx * W;
  // CTA base pointers; transform w of the tile is at w * ig, element i at i * ii
  const cpx<T> *in = reinterpret_cast<const cpx<T> *>(a.in) + by * a.ib + g0 * a.ig;
  cpx<T> *out = reinterpret_cast<cpx<T> *>(a.out) + by * a.ob + g0 * a.og;
  const int ig = (int)a.ig, ii = (int)a.ii, og = (int)a.og, ok = (int)a.ok;
  const int wlive = (int)((a.G - g0) < W ? (a.G - g0) : W);  // live transforms in this tile
  const int n = a.n;
  const int t0 = x.tid(), nt = x.nthreads();
  constexpr int U = sizeof(T) == 4 ? 16 : 8;

  // ---- load
  {
    const int total = W * L;
    // produce: the element's value and its shared-memory position
    auto produce = [&](int e) FFB_INL -> ElemAt<T> {
      int w, i;
      split_elem(e, W, L, a.wfast, a.wdiv, a.ldiv, w, i);
      const int wc = w < wlive ? w : wlive - 1;
      const cpx<T> *xin = in + wc * ig;
      const int at = w * slot_len + pp_pos(i);
      if constexpr (KIND == 0) {
        if (a.chirp_mode == 1) {
          const long long j = (long long)i * a.cj_e + (g0 + wc) * a.cj_g;
          return {j < n ? cmul(ldg_c(xin + i * ii), ldg_c(a.chirp + j)) : mk((T)0, (T)0), at};
        }
        return {ldg_c(xin + i * ii), at};
      } else if constexpr (KIND == 1) {
        return {i < n ? cmul(ldg_c(xin + i * ii), ldg_c(a.chirp + i)) : mk((T)0, (T)0), at};
      } else if constexpr (KIND == 2) {
        return {ldg_c(xin + ldg_v(a.perm_in + i) * ii), at};
      } else {
        return {ldg_c(xin + i * ii), at};
      }
    };
    auto consume = [&](int, ElemAt<T> p) FFB_INL { sm[p.at] = p.v; };
    chunked_loop<U, ElemAt<T>>(t0, nt, total, produce, consume);
    if constexpr (KIND == 2) {
      for (int w = t0; w < W; w += nt) {
        const int wc = w < wlive ? w : wlive - 1;
        sm[w * slot_len + 2 * Lq] = ldg_c(in + wc * ig);  // x0
      }
    }
  }
  x.sync();

  // ---- stages
  auto sync = [&]() FFB_INL { x.sync(); };
  {
    x.per_slot(W, [&](int slot, int tid, int tpt) FFB_INL {
      cpx<T> *const b0 = sm + slot * slot_len, *const b1 = b0 + Lq;
      const int S = a.core.nst;
      stages.template run<KIND == 0 && INV>(a.core, b0, b1, tid, tpt, a.tw, sync);
      if constexpr (KIND != 0) {
        // kernel product on the forward result (natural order), then the inverse
        const int wc = slot < wlive ? slot : wlive - 1;
        const cpx<T> *kern = a.kern;
        if constexpr (KIND == 3) kern += (g0 + wc) * a.kern_stride;
        cpx<T> *const r = (S & 1) ? b1 : b0;
        for (int p = tid; p < L; p += tpt) {
          cpx<T> v = r[pp_pos(p)];
          if constexpr (KIND == 2) {
            if (p == 0) b0[2 * Lq + 1] = v + b0[2 * Lq];  // X0 = x0 + sum_q a[q]
          }
          r[pp_pos(p)] = cmul(v, ldg_c(kern + p));
        }
        sync();
        stages.template run<true>(a.core2, r, (S & 1) ? b0 : b1, tid, tpt, a.tw2, sync);
      }
    });
  }

  // ---- store
  const int S_total = a.core.nst + (KIND == 0 ? 0 : a.core2.nst);
  const int res_off = (S_total & 1) ? Lq : 0;
  auto post_twiddle = [&](cpx<T> v, long long g, int k) FFB_INL -> cpx<T> {
    if (!a.post_twiddle) return v;
    const uint32_t m = (uint32_t)(g * (long long)k);
    const uint32_t hi = fdiv(m, a.ptw_div);
    const uint32_t lo = m - hi * a.ptw_div.d;
    cpx<T> t = cmul(ldg_c(a.ptw_hi + hi), ldg_c(a.ptw_lo + lo));
    if (a.inv) t.y = -t.y;
    return cmul(v, t);
  };
  const int nout = KIND == 1 ? n : L;
  const int total = W * nout;
  // output mapping: consecutive threads take consecutive transforms when a
  // transform's outputs are strided (ok > og), else consecutive elements, so
  // both the loads and the stores of a column tile are coalesced
  const int ofast = a.ok > a.og ? 1 : 0;
  // produce: the output value and its offset from `out`, or -1 when the
  // element is not written (a dead transform of the last tile, or a
  // chirp-on-store position past n)
  auto produce = [&](int e) FFB_INL -> ElemAt<T> {
    int w, k;
    split_elem(e, W, nout, ofast, a.wdiv, KIND == 1 ? a.ndiv : a.ldiv, w, k);
    const int wc = w < wlive ? w : wlive - 1;
    const int at = w < wlive ? w * og + k * ok : -1;
    const cpx<T> *bw = sm + w * slot_len;
    cpx<T> v = bw[res_off + pp_pos(k)];
    if constexpr (KIND == 0) {
      if (a.chirp_mode == 2) {
        const long long j = (long long)k * a.cj_e + (g0 + wc) * a.cj_g;
        return j < n ? ElemAt<T>{cmul(v, ldg_c(a.chirp + j)), at} : ElemAt<T>{v, -1};
      }
      return {post_twiddle(v, g0 + wc, k), at};
    } else if constexpr (KIND == 1) {
      return {post_twiddle(cmul(v, ldg_c(a.chirp + k)), g0 + wc, k), at};
    } else if constexpr (KIND == 2) {
      const int ko = ldg_v(a.perm_out + k);  // frequency index of output k
      return {post_twiddle(bw[2 * Lq] + v, g0 + wc, ko), w < wlive ? w * og + ko * ok : -1};
    } else {
      return {post_twiddle(v, g0 + wc, k), at};
    }
  };
  auto consume = [&](int, ElemAt<T> p) FFB_INL {
    if (p.at >= 0) out[p.at] = p.v;
  };
  chunked_loop<U, ElemAt<T>>(t0, nt, total, produce, consume);
  if constexpr (KIND == 2) {
    for (int w = t0; w < wlive; w += nt) out[w * og] = sm[w * slot_len + 2 * Lq + 1];
  }
}

template <typename T>
struct TileBounds {
  // float kernels run up to 512 threads (128 registers); double up to 256 (255)
  static constexpr int kMaxThreads = sizeof(T) == 4 ? 512 : 256;
};

template <typename T, int KIND, int IO>
__global__ void __launch_bounds__(TileBounds<T>::kMaxThreads) k_tile(const __grid_constant__ TileArgs<T> a) {
  pdl_entry();
  extern __shared__ __align__(16) unsigned char smraw[];
  DevX x{a.tpt, a.wfast};
  tile_body<T, KIND, IO>(a, (long long)blockIdx.x, (long long)blockIdx.y, reinterpret_cast<cpx<T> *>(smraw), x);
}

template <typename T, int KIND, bool INV>
__global__ void __launch_bounds__(TileBounds<T>::kMaxThreads) k_tile_pp(const __grid_constant__ TileArgs<T> a) {
  pdl_entry();
  extern __shared__ __align__(16) unsigned char smraw[];
  DevX x{a.tpt, a.wfast};
  tile_body_pp<T, KIND, INV>(a, (long long)blockIdx.x, (long long)blockIdx.y, reinterpret_cast<cpx<T> *>(smraw), x);
}

template <typename T, int KIND, bool INV, int L, int... Rs>
__global__ void __launch_bounds__(TileBounds<T>::kMaxThreads) k_tile_pp_fixed(const __grid_constant__ TileArgs<T> a) {
  pdl_entry();
  extern __shared__ __align__(16) unsigned char smraw[];
  DevX x{a.tpt, a.wfast};
  tile_body_pp<T, KIND, INV>(a, (long long)blockIdx.x, (long long)blockIdx.y, reinterpret_cast<cpx<T> *>(smraw), x,
                             FixedStagesRunner<T, L, Rs...>{});
}

// True when `c` is exactly the radix sequence Rs... of length L.
template <int L, int... Rs>
FFB_HD bool core_is(const Core &c) {
  constexpr int n = sizeof...(Rs);
  const int r[n] = {Rs...};
  if (c.L != L || c.nst != n) return false;
  for (int s = 0; s < n; ++s)
    if (c.radix[s] != r[s]) return false;
  return true;
}

#ifndef FFB_HOST_EMULATION
template <typename T, int KIND, bool INV, int L, int... Rs>
cudaError_t launch_pp_fixed(const TileArgs<T> &a, size_t smem, cudaStream_t s) {
  {
    cudaError_t e = set_smem_limit_once<k_tile_pp_fixed<T, KIND, INV, L, Rs...>>(232448);
    if (e != cudaSuccess) return e;
  }
  dim3 grid((unsigned)((a.G + a.W - 1) / a.W), (unsigned)a.nbatch, 1);
  dim3 block((unsigned)(a.W * a.tpt), 1, 1);
  return launch_pdl(k_tile_pp_fixed<T, KIND, INV, L, Rs...>, grid, block, smem, s, a);
}
#else
template <typename T, int KIND, bool INV, int L, int... Rs>
cudaError_t launch_pp_fixed(const TileArgs<T> &a, size_t smem, cudaStream_t) {
  std::vector<unsigned char> buf(smem + 64);
  cpx<T> *sm = reinterpret_cast<cpx<T> *>(buf.data());
  const long long tiles = (a.G + a.W - 1) / a.W;
  HostX x;
  for (long long by = 0; by < a.nbatch; ++by)
    for (long long bx = 0; bx < tiles; ++bx) {
      std::memset(buf.data(), 0xff, buf.size());
      tile_body_pp<T, KIND, INV>(a, bx, by, sm, x, FixedStagesRunner<T, L, Rs...>{});
    }
  return cudaSuccess;
}
#endif

// Launches the fixed-sequence kernel matching the pass's core (and core2 for
// convolutions); cudaErrorNotSupported when none matches.
template <typename T, int KIND, bool INV>
cudaError_t launch_pp_fixed_any(const TileArgs<T> &a, size_t smem, cudaStream_t s) {
#define FFB_TRY(L, ...)                                                                              \
  if (core_is<L, __VA_ARGS__>(a.core) && (KIND == 0 || core_is<L, __VA_ARGS__>(a.core2)))           \
    return launch_pp_fixed<T, KIND, INV, L, __VA_ARGS__>(a, smem, s);
  FFB_FIXED_SEQUENCES(FFB_TRY)
#undef FFB_TRY
  return cudaErrorNotSupported;
}

#ifndef FFB_HOST_EMULATION
template <typename T, int KIND, int IO>
cudaError_t launch_one(const TileArgs<T> &a, size_t smem, cudaStream_t s) {
  {
    cudaError_t e = set_smem_limit_once<k_tile<T, KIND, IO>>(232448);
    if (e != cudaSuccess) return e;
  }
  dim3 grid((unsigned)((a.G + a.W - 1) / a.W), (unsigned)a.nbatch, 1);
  dim3 block((unsigned)(a.W * a.tpt), 1, 1);
  return launch_pdl(k_tile<T, KIND, IO>, grid, block, smem, s, a);
}
template <typename T, int KIND, bool INV>
cudaError_t launch_pp(const TileArgs<T> &a, size_t smem, cudaStream_t s) {
  {
    cudaError_t e = set_smem_limit_once<k_tile_pp<T, KIND, INV>>(232448);
    if (e != cudaSuccess) return e;
  }
  dim3 grid((unsigned)((a.G + a.W - 1) / a.W), (unsigned)a.nbatch, 1);
  dim3 block((unsigned)(a.W * a.tpt), 1, 1);
  return launch_pdl(k_tile_pp<T, KIND, INV>, grid, block, smem, s, a);
}
#else
template <typename T, int KIND, bool INV>
cudaError_t launch_pp(const TileArgs<T> &a, size_t smem, cudaStream_t) {
  std::vector<unsigned char> buf(smem + 64);
  cpx<T> *sm = reinterpret_cast<cpx<T> *>(buf.data());
  const long long tiles = (a.G + a.W - 1) / a.W;
  HostX x;
  for (long long by = 0; by < a.nbatch; ++by)
    for (long long bx = 0; bx < tiles; ++bx) {
      std::memset(buf.data(), 0xff, buf.size());
      tile_body_pp<T, KIND, INV>(a, bx, by, sm, x);
    }
  return cudaSuccess;
}

template <typename T, int KIND, int IO>
cudaError_t launch_one(const TileArgs<T> &a, size_t smem, cudaStream_t) {
  std::vector<unsigned char> buf(smem + 64);
  cpx<T> *sm = reinterpret_cast<cpx<T> *>(buf.data());
  const long long tiles = (a.G + a.W - 1) / a.W;
  HostX x;
  for (long long by = 0; by < a.nbatch; ++by)
    for (long long bx = 0; bx < tiles; ++bx) {
      std::memset(buf.data(), 0xff, buf.size());  // poison: unwritten positions show up as NaN
      tile_body<T, KIND, IO>(a, bx, by, sm, x);
    }
  return cudaSuccess;
}
#endif

// Launches every IO variant of core kind K (one translation unit per
// (precision, kind) keeps the compile parallel).
template <typename T, int K>
cudaError_t launch_group(const TileArgs<T> &a, int io, size_t smem, cudaStream_t s) {
  switch (io) {
    case 0: return launch_one<T, K, 0>(a, smem, s);
    case 1: return launch_one<T, K, 1>(a, smem, s);
    case 2: return launch_one<T, K, 2>(a, smem, s);
    case 3: return launch_one<T, K, 3>(a, smem, s);
    case 4: return launch_one<T, K, 4>(a, smem, s);
    default: break;
  }
  return cudaErrorInvalidValue;
}

}  // namespace tile
}  // namespace ffb
