// Row passes with the whole shape fixed at compile time.
//
// A Stockham pass whose transforms are contiguous rows (element i of
// transform g at g * ig + i, output k at g * og + k) and whose core is one of
// the compile-time radix sequences runs here, with the threads per transform
// (TPT) a constant too.  Against the general ping-pong tile body this
//   * reads the first Stockham stage's butterfly inputs straight from global
//     memory (butterfly j of the first stage takes elements j + r * L/R0, so
//     consecutive threads read consecutive addresses), skipping the load
//     phase's shared-memory round trip and barrier;
//   * writes the last stage's outputs straight to global memory (the last
//     stage's butterfly j writes elements j + q * L/R_last, coalesced the
//     same way), skipping the store phase;
//   * in a convolution, multiplies the forward transform's last-stage outputs
//     by the kernel spectrum in registers before they reach shared memory;
//   * keeps one shared-memory buffer per row instead of a ping-pong pair (a
//     stage's values wait in registers across a barrier between its reads
//     and writes), so twice the rows fit on an SM;
//   * has every loop bound and shared-memory offset compile-time, so a
//     thread's R reads and R writes of a stage are one address each plus
//     constant offsets.
// A length-L transform with S stages thus makes S - 1 shared-memory round
// trips (2S - 1 for a convolution) instead of S + 1 (2S + 2).
#pragma once

#include "tile_impl.cuh"

namespace ffb {
namespace rows {

// Compile-time radix sequence: radix, span (product of the earlier radices)
// and twiddle-block offset of stage s, laid out as the host builds a Dit
// core's per-stage table (stage s block: R_s - 1 rows of span_s entries).
template <int... Rs>
struct Seq {
  static constexpr int n = sizeof...(Rs);
  static FFB_HD constexpr int r(int s) {
    constexpr int a[] = {Rs...};
    return a[s];
  }
  static FFB_HD constexpr int span(int s) {
    int p = 1;
    for (int i = 0; i < s; ++i) p *= r(i);
    return p;
  }
  static FFB_HD constexpr int twoff(int s) {
    int o = 0;
    for (int i = 0; i < s; ++i) o += (r(i) - 1) * span(i);
    return o;
  }
  static FFB_HD constexpr int rmax() {
    int m = 0;
    for (int i = 0; i < n; ++i) m = r(i) > m ? r(i) : m;
    return m;
  }
};

// Threads per transform of a length-L core whose largest radix is rmax: one
// butterfly of the largest radix per thread, rounded up to a power of two
// below 32 and to a multiple of 32 above (the executor's rule).
FFB_HD constexpr int tpt_of(int L, int rmax) {
  const int t = (L + rmax - 1) / rmax;
  if (t <= 32) {
    int p = 1;
    while (p < t) p <<= 1;
    return p;
  }
  return (t + 31) / 32 * 32;
}

// Threads per row of a row kernel: tpt_of, at most the precision's CTA
// limit (L = 16384 runs 512 threads, two radix-16 butterflies each).
template <typename T, int L, int... Rs>
FFB_HD constexpr int rows_tpt() {
  return tpt_of(L, Seq<Rs...>::rmax()) < tile::TileBounds<T>::kMaxThreads ? tpt_of(L, Seq<Rs...>::rmax())
                                                                           : tile::TileBounds<T>::kMaxThreads;
}

// The wide form of a sequence with a radix that is not a power of two: one
// butterfly of its smallest radix of at least 5 per thread, so that no such
// stage takes a second round (1701 = 9 9 7 3: 243 -> 256 threads instead of
// 189 -> 192, whose radix-7 stage runs two rounds).  Equal to rows_tpt for
// powers of two.  The executor takes it for small batches (exec.cpp
// wide_tpt).
template <int... Rs>
FFB_HD constexpr int thread_radix() {
  constexpr bool pow2 = (((Rs & (Rs - 1)) == 0) && ...);
  int m = Seq<Rs...>::rmax();
  if (!pow2) ((Rs >= 5 && Rs < m ? (void)(m = Rs) : (void)0), ...);
  return m;
}
template <typename T, int L, int... Rs>
FFB_HD constexpr int rows_tpt_wide() {
  return tpt_of(L, thread_radix<Rs...>()) < tile::TileBounds<T>::kMaxThreads ? tpt_of(L, thread_radix<Rs...>())
                                                                             : tile::TileBounds<T>::kMaxThreads;
}

// Thread policy: DevT runs a phase's body once as this CUDA thread; HostT
// (host emulation of the index arithmetic) runs it for every thread in turn.
struct DevT {
  template <class F>
  FFB_HD void each(int, F &&f) const {
#ifdef __CUDA_ARCH__
    f((int)threadIdx.x);
#else
    (void)f;
#endif
  }
  FFB_HD void sync() const {
#ifdef __CUDA_ARCH__
    __syncthreads();
#endif
  }
  // A barrier-separated pipeline of per-thread steps: first() starts it,
  // step() crosses a barrier and maps this thread's state to the next,
  // last() crosses a barrier and consumes it.
  template <class F>
  FFB_HD auto first(int, F &&f) const {
#ifdef __CUDA_ARCH__
    return f((int)threadIdx.x);
#else
    return f(0);
#endif
  }
  template <class F, class S>
  FFB_HD auto step(int, F &&f, const S &st) const {
#ifdef __CUDA_ARCH__
    __syncthreads();
    return f((int)threadIdx.x, st);
#else
    return f(0, st);
#endif
  }
  template <class F, class S>
  FFB_HD void last(int, F &&f, const S &st) const {
#ifdef __CUDA_ARCH__
    __syncthreads();
    f((int)threadIdx.x, st);
#else
    (void)f;
    (void)st;
#endif
  }
  // rd's result stays in this thread's registers across the barrier
  template <class FR, class FW>
  FFB_HD void each2(int, FR &&rd, FW &&wr) const {
#ifdef __CUDA_ARCH__
    const auto st = rd((int)threadIdx.x);
    __syncthreads();
    wr((int)threadIdx.x, st);
#else
    (void)rd;
    (void)wr;
#endif
  }
};
struct HostT {
  template <class F>
  FFB_HD void each(int nthr, F &&f) const {
    for (int t = 0; t < nthr; ++t) f(t);
  }
  FFB_HD void sync() const {}
  // the pipeline with one state per thread, every step over all threads
  template <class F>
  FFB_HD auto first(int nthr, F &&f) const {
    std::vector<decltype(f(0))> out;
#ifndef __CUDA_ARCH__
    out.reserve((size_t)nthr);
    for (int t = 0; t < nthr; ++t) out.push_back(f(t));
#endif
    return out;
  }
  template <class F, class S>
  FFB_HD auto step(int nthr, F &&f, const std::vector<S> &st) const {
    std::vector<decltype(f(0, st[0]))> out;
#ifndef __CUDA_ARCH__
    out.reserve((size_t)nthr);
    for (int t = 0; t < nthr; ++t) out.push_back(f(t, st[(size_t)t]));
#endif
    return out;
  }
  template <class F, class S>
  FFB_HD void last(int nthr, F &&f, const std::vector<S> &st) const {
#ifndef __CUDA_ARCH__
    for (int t = 0; t < nthr; ++t) f(t, st[(size_t)t]);
#endif
  }
  template <class FR, class FW>
  FFB_HD void each2(int nthr, FR &&rd, FW &&wr) const {
#ifndef __CUDA_ARCH__
    std::vector<decltype(rd(0))> st;
    st.reserve((size_t)nthr);
    for (int t = 0; t < nthr; ++t) st.push_back(rd(t));
    for (int t = 0; t < nthr; ++t) wr(t, st[(size_t)t]);
#else
    (void)nthr;
    (void)rd;
    (void)wr;
#endif
  }
};

// Streaming read of a row element: not kept in L1, which then holds the
// twiddle, chirp and kernel tables the stages re-read.
FFB_HD cpx<float> ld_stream(const cpx<float> *p) {
#ifdef __CUDA_ARCH__
  float x, y;
  asm("ld.global.nc.L1::no_allocate.v2.f32 {%0, %1}, [%2];" : "=f"(x), "=f"(y) : "l"(p));
  return mk(x, y);
#else
  return *p;
#endif
}
FFB_HD cpx<double> ld_stream(const cpx<double> *p) {
#ifdef __CUDA_ARCH__
  double x, y;
  asm("ld.global.nc.L1::no_allocate.v2.f64 {%0, %1}, [%2];" : "=d"(x), "=d"(y) : "l"(p));
  return mk(x, y);
#else
  return *p;
#endif
}

// Ping-pong buffer access: get reads elements j + r * S (r < R), put writes
// elements base + q * S.
template <typename T>
struct SmemIO {
  cpx<T> *b;
  template <int S, int R>
  FFB_HD void get(int j, cpx<T> (&x)[R]) const {
    if constexpr (S % 16 == 0) {
      const cpx<T> *p = b + pp_pos(j);
#pragma unroll
      for (int r = 0; r < R; ++r) x[r] = p[r * (S + S / 16)];
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) x[r] = b[pp_pos(j + r * S)];
    }
  }
  template <int S, int R>
  FFB_HD void put(int base, const cpx<T> (&x)[R]) const {
    if constexpr (S % 16 == 0) {
      cpx<T> *p = b + pp_pos(base);
#pragma unroll
      for (int q = 0; q < R; ++q) p[q * (S + S / 16)] = x[q];
    } else if constexpr (S == 1 && 16 % R == 0) {
      cpx<T> *p = b + pp_pos(base);  // base is a multiple of R: R positions inside one 16-block
#pragma unroll
      for (int q = 0; q < R; ++q) p[q] = x[q];
    } else {
#pragma unroll
      for (int q = 0; q < R; ++q) b[pp_pos(base + q * S)] = x[q];
    }
  }
};

// Last forward stage of a convolution: output k (natural order) times the
// kernel spectrum entry k, into the ping-pong buffer.
template <typename T>
struct SmemKernIO {
  cpx<T> *b;
  const cpx<T> *kern;
  template <int S, int R>
  FFB_HD void put(int base, const cpx<T> (&x)[R]) const {
    cpx<T> y[R];
#pragma unroll
    for (int q = 0; q < R; ++q) y[q] = cmul(x[q], ldg_c(kern + base + q * S));
    SmemIO<T>{b}.template put<S, R>(base, y);
  }
};

// Four-step post-twiddle W_N^{g k} (conjugated for the inverse) from the two
// split tables, m = g * k < N.
template <typename T>
FFB_HD cpx<T> post_twiddle(const TileArgs<T> &a, cpx<T> v, long long g, int k) {
  const uint32_t m = (uint32_t)(g * (long long)k);
  const uint32_t hi = fdiv(m, a.ptw_div);
  const uint32_t lo = m - hi * a.ptw_div.d;
  cpx<T> t = cmul(ldg_c(a.ptw_hi + hi), ldg_c(a.ptw_lo + lo));
  if (a.inv) t.y = -t.y;
  return cmul(v, t);
}

// First stage's reader: element i of the row in global memory, with the
// pass kind's load-side factor (KIND 1: chirp, zero past n; KIND 0 with
// chirp_mode 1: chirp at j = i * cj_e + g * cj_g, zero past n).
template <typename T, int KIND>
struct GlobalIn {
  const TileArgs<T> *a;
  const cpx<T> *row;
  long long g;
  template <int S, int R>
  FFB_HD void get(int j, cpx<T> (&x)[R]) const {
    if constexpr (KIND == 1) {
      const int n = a->n;
#pragma unroll
      for (int r = 0; r < R; ++r) {
        const int i = j + r * S;
        x[r] = i < n ? cmul(ld_stream(row + i), ldg_c(a->chirp + i)) : mk((T)0, (T)0);
      }
    } else if constexpr (KIND == 0) {
      if (a->chirp_mode == 1) {
        const long long n = a->n;
#pragma unroll
        for (int r = 0; r < R; ++r) {
          const int i = j + r * S;
          const long long c = (long long)i * a->cj_e + g * a->cj_g;
          x[r] = c < n ? cmul(ld_stream(row + i), ldg_c(a->chirp + c)) : mk((T)0, (T)0);
        }
      } else {
#pragma unroll
        for (int r = 0; r < R; ++r) x[r] = ld_stream(row + j + r * S);
      }
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) x[r] = ld_stream(row + j + r * S);
    }
  }
};

// Last stage's writer: output k of the row to global memory, with the pass
// kind's store-side factor (KIND 1: chirp, only k < n; KIND 0 with
// chirp_mode 2: chirp at j = k * cj_e + g * cj_g, only j < n; otherwise the
// optional four-step post-twiddle).  Nothing is written for a dead row.
template <typename T, int KIND>
struct GlobalOut {
  const TileArgs<T> *a;
  cpx<T> *row;
  long long g;
  bool live;
  template <int S, int R>
  FFB_HD void put(int base, const cpx<T> (&x)[R]) const {
    if (!live) return;
    const bool ptw = a->post_twiddle != 0;
    if constexpr (KIND == 1) {
      const int n = a->n;
#pragma unroll
      for (int q = 0; q < R; ++q) {
        const int k = base + q * S;
        if (k < n) {
          cpx<T> v = cmul(x[q], ldg_c(a->chirp + k));
          row[k] = ptw ? post_twiddle(*a, v, g, k) : v;
        }
      }
    } else {
      if (KIND == 0 && a->chirp_mode == 2) {
        const long long n = a->n;
#pragma unroll
        for (int q = 0; q < R; ++q) {
          const int k = base + q * S;
          const long long c = (long long)k * a->cj_e + g * a->cj_g;
          if (c < n) row[k] = cmul(x[q], ldg_c(a->chirp + c));
        }
      } else if (ptw) {
#pragma unroll
        for (int q = 0; q < R; ++q) row[base + q * S] = post_twiddle(*a, x[q], g, base + q * S);
      } else {
#pragma unroll
        for (int q = 0; q < R; ++q) row[base + q * S] = x[q];
      }
    }
  }
};

// Stockham stage with span Ns and radix R of a length-L transform for the
// butterflies of one thread (j = t, t + TPT, ... < L/R): inputs j + r L/R
// from rd, twiddles W_{Ns R}^{r (j mod Ns)} from the stage block, outputs
// (j - j mod Ns) R + j mod Ns + q Ns to wr.  stage_read does the reads and
// the arithmetic, stage_write the writes, so a stage may read and write the
// same buffer with a barrier between.
template <typename T, int L, int TPT, int R>
struct StageRegs {
  static constexpr int V = (L / R + TPT - 1) / TPT;
  cpx<T> x[V][R];
};

// 16 bytes from shared memory (a 16-byte aligned address) into w[0..3].
FFB_HD void lds_f4(const void *p, float (&w)[4]) {
#ifdef __CUDA_ARCH__
  asm volatile("ld.shared.v4.f32 {%0, %1, %2, %3}, [%4];"
               : "=f"(w[0]), "=f"(w[1]), "=f"(w[2]), "=f"(w[3])
               : "r"((uint32_t)__cvta_generic_to_shared(p)));
#else
  const float *f = static_cast<const float *>(p);
  for (int i = 0; i < 4; ++i) w[i] = f[i];
#endif
}

// Where the stage twiddles are: TW_GLOBAL the host's block (R - 1 rows of Ns
// entries) in global memory; TW_SHARED the same block in shared memory;
// TW_PAIRS (single precision, shared memory) rows r, r + 1 interleaved, so
// one 16-byte load brings W^{r k} and W^{(r+1) k}: entry (m, k) of the
// block holds rows 2m + 1 and 2m + 2 (the second one unused past R - 1).
enum : int { TW_GLOBAL = 0, TW_SHARED = 1, TW_PAIRS = 2 };

template <typename T, bool INV, int L, int TPT, int Ns, int R, int TWS = TW_GLOBAL, class Rd>
FFB_HD StageRegs<T, L, TPT, R> stage_read(int t, const cpx<T> *__restrict__ blk, const Rd &rd) {
  static_assert(TWS != TW_PAIRS || sizeof(T) == 4, "twiddle pairs are single precision");
  constexpr int nb = L / R;
  StageRegs<T, L, TPT, R> st;
#pragma unroll
  for (int v = 0; v < st.V; ++v) {
    const int j = t + v * TPT;
    if (nb % TPT == 0 || j < nb) {
      const int k = Ns == 1 ? 0 : j % Ns;
      rd.template get<nb, R>(j, st.x[v]);
      if constexpr (Ns > 1 && TWS == TW_PAIRS) {
        const cpx<T> *row = blk + 2 * k;
#pragma unroll
        for (int r = 1; r < R; r += 2) {
          float w[4];
          lds_f4(row + (r - 1) * Ns, w);
          st.x[v][r] = cmul(st.x[v][r], mk((T)w[0], (T)w[1]));
          if (r + 1 < R) st.x[v][r + 1] = cmul(st.x[v][r + 1], mk((T)w[2], (T)w[3]));
        }
      } else if constexpr (Ns > 1) {
        const cpx<T> *row = blk + k;
#pragma unroll
        for (int r = 1; r < R; ++r)
          st.x[v][r] = cmul(st.x[v][r], TWS == TW_SHARED ? row[(r - 1) * Ns] : ldg_c(row + (r - 1) * Ns));
      }
      dft_fixed<R, INV, T>(st.x[v]);
    }
  }
  return st;
}

template <typename T, int L, int TPT, int Ns, int R, class Wr>
FFB_HD void stage_write(int t, const StageRegs<T, L, TPT, R> &st, const Wr &wr) {
  constexpr int nb = L / R;
#pragma unroll
  for (int v = 0; v < st.V; ++v) {
    const int j = t + v * TPT;
    if (nb % TPT == 0 || j < nb) {
      const int k = Ns == 1 ? 0 : j % Ns;
      wr.template put<Ns, R>((j - k) * R + k, st.x[v]);
    }
  }
}

// Shared memory of one row: one padded buffer (positions pp_pos) plus a
// spare element so the slot stride is odd.
template <int L>
FFB_HD constexpr int slot_len() {
  return pp_size(L) + 1;
}

// Stages S.. of sequence Q on the row's buffer.  A stage that reads and
// writes the buffer has a barrier between its reads and its writes (the
// values wait in registers), which halves the shared memory a ping-pong pair
// of buffers would take: more CTAs per SM, measured 1.1-1.4x faster on B200.
// Stage 0 reads through first(w, buf) (shared memory when FS), the last
// stage writes through last(w, buf) (shared memory when LS).  A barrier
// separates consecutive stages; none follows the last.
template <typename T, bool INV, int L, int TPT, bool FS, bool LS, class Q, int S, class X, class First,
          class Last>
FFB_HD void run_chain(const X &x, int nthr, const cpx<T> *__restrict__ tw, cpx<T> *sm, const First &first,
                      const Last &last) {
  if constexpr (S < Q::n) {
    constexpr int R = Q::r(S), Ns = Q::span(S), TwOff = Q::twoff(S);
    constexpr int slot = slot_len<L>();
    constexpr bool is_first = S == 0, is_last = S == Q::n - 1;
    auto rd = [&](int tid) FFB_INL {
      const int w = tid / TPT, t = tid - w * TPT;
      if constexpr (is_first) {
        return stage_read<T, INV, L, TPT, Ns, R>(t, tw + TwOff, first(w, sm + w * slot));
      } else {
        return stage_read<T, INV, L, TPT, Ns, R>(t, tw + TwOff, SmemIO<T>{sm + w * slot});
      }
    };
    auto wr = [&](int tid, const StageRegs<T, L, TPT, R> &st) FFB_INL {
      const int w = tid / TPT, t = tid - w * TPT;
      if constexpr (is_last) {
        stage_write<T, L, TPT, Ns, R>(t, st, last(w, sm + w * slot));
      } else {
        stage_write<T, L, TPT, Ns, R>(t, st, SmemIO<T>{sm + w * slot});
      }
    };
    constexpr bool reads_smem = !is_first || FS, writes_smem = !is_last || LS;
    if constexpr (reads_smem && writes_smem) {
      x.each2(nthr, rd, wr);
    } else {
      x.each(nthr, [&](int tid) FFB_INL { wr(tid, rd(tid)); });
    }
    if constexpr (S + 1 < Q::n) {
      x.sync();
      run_chain<T, INV, L, TPT, FS, LS, Q, S + 1>(x, nthr, tw, sm, first, last);
    }
  }
}

// One CTA tile of W rows (W = blockDim / TPT): KIND 0 a Dit transform in
// direction INV, KIND 1 the fused Bluestein chain, KIND 3 a convolution row
// (forward core, kernel product, inverse core2).
template <typename T, int KIND, bool INV, int L, int TPT, class X, int... Rs>
FFB_HD void rows_body(const TileArgs<T> &a, long long bx, long long by, cpx<T> *sm, const X &x) {
  using Q = Seq<Rs...>;
  const int W = a.W;
  const int nthr = W * TPT;
  const long long g0 = bx * W;
  const int wlive = (int)((a.G - g0) < W ? (a.G - g0) : W);
  const cpx<T> *in = reinterpret_cast<const cpx<T> *>(a.in) + by * a.ib + g0 * a.ig;
  cpx<T> *out = reinterpret_cast<cpx<T> *>(a.out) + by * a.ob + g0 * a.og;
  const TileArgs<T> *ap = &a;
  // dead rows of the last tile compute on the last live row's data and store nothing
  auto first = [&](int w, cpx<T> *) FFB_INL {
    const int wc = w < wlive ? w : wlive - 1;
    return GlobalIn<T, KIND>{ap, in + wc * a.ig, g0 + wc};
  };
  auto last = [&](int w, cpx<T> *) FFB_INL {
    return GlobalOut<T, KIND>{ap, out + w * a.og, g0 + w, w < wlive};
  };
  if constexpr (KIND == 0) {
    run_chain<T, INV, L, TPT, false, false, Q, 0>(x, nthr, a.tw, sm, first, last);
  } else {
    auto kern_last = [&](int w, cpx<T> *buf) FFB_INL {
      const cpx<T> *kern = a.kern;
      if constexpr (KIND == 3) {
        const int wc = w < wlive ? w : wlive - 1;
        kern += (g0 + wc) * a.kern_stride;
      }
      return SmemKernIO<T>{buf, kern};
    };
    auto smem_first = [&](int, cpx<T> *buf) FFB_INL { return SmemIO<T>{buf}; };
    run_chain<T, false, L, TPT, false, true, Q, 0>(x, nthr, a.tw, sm, first, kern_last);
    x.sync();
    run_chain<T, true, L, TPT, true, false, Q, 0>(x, nthr, a.tw2, sm, smem_first, last);
  }
}

template <typename T, int KIND, bool INV, int MB, int L, int TPT, int... Rs>
__global__ void __launch_bounds__(tile::TileBounds<T>::kMaxThreads, MB) k_rows(const __grid_constant__ TileArgs<T> a) {
  pdl_entry();
  extern __shared__ __align__(16) unsigned char smraw[];
  rows_body<T, KIND, INV, L, TPT, DevT, Rs...>(a, (long long)blockIdx.x, (long long)blockIdx.y,
                                               reinterpret_cast<cpx<T> *>(smraw), DevT{});
}

// True when the pass can run as rows of this sequence with TPT threads a
// row: contiguous rows on both sides, the executor's threads per transform,
// and (convolutions) the same sequence for the inverse core.
template <typename T, int KIND, int L, int TPT, int... Rs>
FFB_HD bool rows_fit(const TileArgs<T> &a) {
  return a.pp && !a.wfast && a.ii == 1 && a.ok == 1 && a.tpt == TPT &&
         a.W * TPT <= tile::TileBounds<T>::kMaxThreads && tile::core_is<L, Rs...>(a.core) &&
         (KIND == 0 || tile::core_is<L, Rs...>(a.core2));
}

// Shared memory of a row-kernel launch.
template <typename T, int L>
size_t rows_smem(const TileArgs<T> &a) {
  return (size_t)a.W * slot_len<L>() * sizeof(cpx<T>);
}

#ifndef FFB_HOST_EMULATION
template <typename T, int KIND, bool INV, int MB, int L, int TPT, int... Rs>
cudaError_t launch_rows_mb(const TileArgs<T> &a, cudaStream_t s) {
  {
    cudaError_t e = set_smem_limit_once<k_rows<T, KIND, INV, MB, L, TPT, Rs...>>(232448);
    if (e != cudaSuccess) return e;
  }
  dim3 grid((unsigned)((a.G + a.W - 1) / a.W), (unsigned)a.nbatch, 1);
  dim3 block((unsigned)(a.W * TPT), 1, 1);
  return launch_pdl(k_rows<T, KIND, INV, MB, L, TPT, Rs...>, grid, block, rows_smem<T, L>(a), s, a);
}
// Double-precision transforms of up to 4096 points are compiled for two
// CTAs per SM (at most 128 registers, no spills): without the bound the
// compiler took 146-208 registers and left one 256-thread CTA per SM
// (Z2Z 4096 x 8192: 274 us against 200 us with it).  The convolution kernels
// ran slower with it, and 8192 points would spill.
template <typename T, int KIND, int L>
constexpr int rows_min_blocks() {
  return sizeof(T) == 8 && KIND == 0 && L <= 4096 ? 2 : 1;
}
template <typename T, int KIND, bool INV, int L, int TPT, int... Rs>
cudaError_t launch_rows(const TileArgs<T> &a, cudaStream_t s) {
  return launch_rows_mb<T, KIND, INV, rows_min_blocks<T, KIND, L>(), L, TPT, Rs...>(a, s);
}
#else
template <typename T, int KIND, bool INV, int L, int TPT, int... Rs>
cudaError_t launch_rows(const TileArgs<T> &a, cudaStream_t) {
  std::vector<unsigned char> buf(rows_smem<T, L>(a) + 64);
  cpx<T> *sm = reinterpret_cast<cpx<T> *>(buf.data());
  const long long tiles = (a.G + a.W - 1) / a.W;
  for (long long by = 0; by < a.nbatch; ++by)
    for (long long bx = 0; bx < tiles; ++bx) {
      std::memset(buf.data(), 0xff, buf.size());
      rows_body<T, KIND, INV, L, TPT, HostT, Rs...>(a, bx, by, sm, HostT{});
    }
  return cudaSuccess;
}
#endif

// Shared memory of the row kernel that runs the pass, or 0 when the pass is
// not rows of a compile-time sequence.
template <typename T, int KIND>
size_t rows_smem_any(const TileArgs<T> &a) {
#define FFB_ROWS_SMEM(L, ...)                                                                 \
  if (rows_fit<T, KIND, L, rows_tpt<T, L, __VA_ARGS__>(), __VA_ARGS__>(a) ||                 \
      rows_fit<T, KIND, L, rows_tpt_wide<T, L, __VA_ARGS__>(), __VA_ARGS__>(a))              \
    return rows_smem<T, L>(a);
  FFB_FIXED_SEQUENCES(FFB_ROWS_SMEM)
#undef FFB_ROWS_SMEM
  return 0;
}

// Launches the row kernel of the pass's sequence; cudaErrorNotSupported when
// the pass is not rows of a compile-time sequence.
template <typename T, int KIND, bool INV>
cudaError_t launch_rows_any(const TileArgs<T> &a, size_t, cudaStream_t s) {
#define FFB_TRY_ROWS(L, ...)                                                                              \
  if (rows_fit<T, KIND, L, rows_tpt<T, L, __VA_ARGS__>(), __VA_ARGS__>(a))                                \
    return launch_rows<T, KIND, INV, L, rows_tpt<T, L, __VA_ARGS__>(), __VA_ARGS__>(a, s);                \
  if constexpr (rows_tpt_wide<T, L, __VA_ARGS__>() != rows_tpt<T, L, __VA_ARGS__>()) {                    \
    if (rows_fit<T, KIND, L, rows_tpt_wide<T, L, __VA_ARGS__>(), __VA_ARGS__>(a))                         \
      return launch_rows<T, KIND, INV, L, rows_tpt_wide<T, L, __VA_ARGS__>(), __VA_ARGS__>(a, s);         \
  }
  FFB_FIXED_SEQUENCES(FFB_TRY_ROWS)
#undef FFB_TRY_ROWS
  return cudaErrorNotSupported;
}

}  // namespace rows
}  // namespace ffb
