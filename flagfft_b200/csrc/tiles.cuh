// Tile passes of the compile-time radix sequences for strided layouts.
//
// A pass whose transforms are columns (element i of transform g at
// g * ig + i * ii with ii > ig, or outputs at k * ok > og) is coalesced only
// when one CTA holds W consecutive transforms, so that a warp reads or writes
// W-element segments of each row.  The general tile body keeps two ping-pong
// buffers per transform, which leaves room for W = 3 transforms of 4096
// points (24-byte segments).  Here each transform keeps one padded buffer,
// the stages hold their values in registers across a barrier between reads
// and writes (as the row kernels do), and the W transforms are processed as
// NG groups of NR (NR x TPT threads): twice the transforms per CTA.
//   load:   global -> shared, consecutive threads on consecutive transforms
//           when the input is strided, else on consecutive elements;
//   stages: one pipeline over the groups (two barriers per stage, a thread
//           holds one group's values at a time);
//   store:  shared -> global, mapped by the output layout the same way, with
//           the optional chirp or four-step post-twiddle.
#pragma once

#include "rows.cuh"

namespace ffb {
namespace tiles {

using rows::Seq;
using rows::SmemIO;
using rows::slot_len;

// Threads, rows per group and groups of the tile kernel of a length-L
// sequence: NT = NR * TPT threads, NR rows per group (at most 8, within the
// precision's thread limit), NG groups (2..4) so that W = NR * NG reaches the
// transforms a 128-byte row segment holds (16 single, 8 double precision)
// where shared memory allows.  A small W keeps several CTAs per SM, whose
// global loads overlap.
template <typename T, int L, int... Rs>
struct Shape {
  static constexpr int TPT = rows::rows_tpt<T, L, Rs...>();
  static constexpr int nr_max = tile::TileBounds<T>::kMaxThreads / TPT;
  static constexpr int NR = nr_max < 8 ? nr_max : 8;
  static constexpr int NT = NR * TPT;
  static constexpr int slot = slot_len<L>();
  static constexpr int fit = (int)(232448 / ((size_t)NR * slot * sizeof(cpx<T>)));
  static constexpr int target = sizeof(T) == 4 ? 16 : 8;
  static constexpr int want = (target + NR - 1) / NR < 2 ? 2 : (target + NR - 1) / NR;
  static constexpr int cap = fit < 4 ? fit : 4;
  static constexpr int NG = want < cap ? want : cap;
  static constexpr int W = NR * NG;
  // CTAs per SM that shared memory allows (at most 8): the register budget
  // the kernel is compiled for
  static constexpr size_t smem = (size_t)W * slot * sizeof(cpx<T>);
  static constexpr int per_sm = smem ? (int)(232448 / (smem + 1024)) : 1;
  static constexpr int min_blocks = per_sm < 1 ? 1 : per_sm > 8 ? 8 : per_sm;
};

template <typename T, bool INV, int L, class Q, class Sh, int S>
struct Stage {
  static constexpr int R = Q::r(S), Ns = Q::span(S), TwOff = Q::twoff(S);
  using Regs = rows::StageRegs<T, L, Sh::TPT, R>;
  static FFB_HD Regs read(const cpx<T> *tw, cpx<T> *sm, int grp, int tid) {
    const int w = grp * Sh::NR + tid / Sh::TPT, t = tid % Sh::TPT;
    return rows::stage_read<T, INV, L, Sh::TPT, Ns, R>(t, tw + TwOff, SmemIO<T>{sm + w * Sh::slot});
  }
  static FFB_HD void write(cpx<T> *sm, int grp, int tid, const Regs &st) {
    const int w = grp * Sh::NR + tid / Sh::TPT, t = tid % Sh::TPT;
    rows::stage_write<T, L, Sh::TPT, Ns, R>(t, st, SmemIO<T>{sm + w * Sh::slot});
  }
};

// Step K of the pipeline reads group K % NG of stage K / NG; between two
// barriers a thread writes what it read in the previous step, then reads.
// With NG >= 2 a write and the read after it touch different groups, and a
// group's reads follow its previous writes by at least one barrier.
#pragma nv_exec_check_disable
template <typename T, bool INV, int L, class Q, class Sh, int K, class X, class St>
FFB_HD void pipe(const X &x, const cpx<T> *tw, cpx<T> *sm, const St &st) {
  static_assert(Sh::NG >= 2, "the pipeline needs two groups or more");
  constexpr int P = K - 1;
  using Prev = Stage<T, INV, L, Q, Sh, P / Sh::NG>;
  if constexpr (K == Sh::NG * Q::n) {
    x.last(Sh::NT, [&](int tid, const typename Prev::Regs &s) FFB_INL { Prev::write(sm, P % Sh::NG, tid, s); }, st);
  } else {
    using Cur = Stage<T, INV, L, Q, Sh, K / Sh::NG>;
    auto nxt = x.step(
        Sh::NT,
        [&](int tid, const typename Prev::Regs &s) FFB_INL {
          Prev::write(sm, P % Sh::NG, tid, s);
          return Cur::read(tw, sm, K % Sh::NG, tid);
        },
        st);
    pipe<T, INV, L, Q, Sh, K + 1>(x, tw, sm, nxt);
  }
}

// One tile (W transforms from g0 = bx * W, batch by) of a Dit pass in
// direction INV.
#pragma nv_exec_check_disable
template <typename T, bool INV, int L, class X, int... Rs>
FFB_HD void tile_body(const TileArgs<T> &a, long long bx, long long by, cpx<T> *sm, const X &x) {
  using Q = Seq<Rs...>;
  using Sh = Shape<T, L, Rs...>;
  constexpr int W = Sh::W, NT = Sh::NT, total = W * L;
  constexpr int U = sizeof(T) == 4 ? 8 : 4;  // global accesses in flight per thread
  const long long g0 = bx * W;
  const int wlive = (int)((a.G - g0) < W ? (a.G - g0) : W);
  const cpx<T> *in = reinterpret_cast<const cpx<T> *>(a.in) + by * a.ib + g0 * a.ig;
  cpx<T> *out = reinterpret_cast<cpx<T> *>(a.out) + by * a.ob + g0 * a.og;
  const long long n = a.n;

  // load: element e of the tile -> (transform w, element i).  A strided input
  // whose tile width divides the thread count keeps one transform per thread
  // (w = tid % W) and steps its element by NT / W: one pointer increment per
  // load.
  const bool in_fast = a.ii > a.ig;
  bool loaded = false;
  if constexpr (NT % W == 0) {
    if (in_fast && a.chirp_mode == 0) {
      x.each(NT, [&](int tid) FFB_INL {
        constexpr int IS = NT / W, M = (L + IS - 1) / IS;
        const int w = tid % W, i0 = tid / W;
        const int wc = w < wlive ? w : wlive - 1;
        const cpx<T> *src = in + wc * a.ig + (long long)i0 * a.ii;
        const long long step = (long long)IS * a.ii;
        cpx<T> *dst = sm + w * Sh::slot;
#pragma unroll 1
        for (int m0 = 0; m0 < M; m0 += U) {
          cpx<T> v[U];
#pragma unroll
          for (int u = 0; u < U; ++u)
            if (m0 + u < M && (L % IS == 0 || i0 + (m0 + u) * IS < L)) v[u] = rows::ld_stream(src + (m0 + u) * step);
#pragma unroll
          for (int u = 0; u < U; ++u)
            if (m0 + u < M && (L % IS == 0 || i0 + (m0 + u) * IS < L)) dst[pp_pos(i0 + (m0 + u) * IS)] = v[u];
        }
      });
      loaded = true;
    }
  }
  if (!loaded) x.each(NT, [&](int tid) FFB_INL {
#pragma unroll 1
    for (int c = tid; c < total; c += U * NT) {
      cpx<T> v[U];
      int at[U];
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int e = c + u * NT;
        at[u] = -1;
        if (e < total) {
          const int w = in_fast ? e % W : e / L, i = in_fast ? e / W : e % L;
          const int wc = w < wlive ? w : wlive - 1;
          const cpx<T> *src = in + wc * a.ig + (long long)i * a.ii;
          if (a.chirp_mode == 1) {
            const long long j = (long long)i * a.cj_e + (g0 + wc) * a.cj_g;
            v[u] = j < n ? cmul(rows::ld_stream(src), ldg_c(a.chirp + j)) : mk((T)0, (T)0);
          } else {
            v[u] = rows::ld_stream(src);
          }
          at[u] = w * Sh::slot + pp_pos(i);
        }
      }
#pragma unroll
      for (int u = 0; u < U; ++u)
        if (at[u] >= 0) sm[at[u]] = v[u];
    }
  });
  x.sync();

  // stages
  {
    using First = Stage<T, INV, L, Q, Sh, 0>;
    auto st = x.first(NT, [&](int tid) FFB_INL { return First::read(a.tw, sm, 0, tid); });
    pipe<T, INV, L, Q, Sh, 1>(x, a.tw, sm, st);
  }
  x.sync();

  // store: element e of the tile -> (transform w, output k); a strided output
  // keeps one transform per thread as the load does
  const bool out_fast = a.ok > a.og;
  if constexpr (NT % W == 0) {
    if (out_fast && a.chirp_mode == 0) {
      x.each(NT, [&](int tid) FFB_INL {
        constexpr int IS = NT / W, M = (L + IS - 1) / IS;
        const int w = tid % W, k0 = tid / W;
        if (w >= wlive) return;
        const long long g = g0 + w;
        cpx<T> *dst = out + w * a.og + (long long)k0 * a.ok;
        const long long step = (long long)IS * a.ok;
        const cpx<T> *src = sm + w * Sh::slot;
        const bool ptw = a.post_twiddle != 0;
#pragma unroll 4
        for (int m = 0; m < M; ++m) {
          const int k = k0 + m * IS;
          if (L % IS != 0 && k >= L) break;
          const cpx<T> v = src[pp_pos(k)];
          dst[m * step] = ptw ? rows::post_twiddle(a, v, g, k) : v;
        }
      });
      return;
    }
  }
  x.each(NT, [&](int tid) FFB_INL {
#pragma unroll 1
    for (int c = tid; c < total; c += U * NT) {
#pragma unroll
      for (int u = 0; u < U; ++u) {
        const int e = c + u * NT;
        if (e >= total) continue;
        const int w = out_fast ? e % W : e / L, k = out_fast ? e / W : e % L;
        if (w >= wlive) continue;
        const long long g = g0 + w;
        cpx<T> v = sm[w * Sh::slot + pp_pos(k)];
        cpx<T> *dst = out + w * a.og + (long long)k * a.ok;
        if (a.chirp_mode == 2) {
          const long long j = (long long)k * a.cj_e + g * a.cj_g;
          if (j < n) *dst = cmul(v, ldg_c(a.chirp + j));
        } else if (a.post_twiddle) {
          *dst = rows::post_twiddle(a, v, g, k);
        } else {
          *dst = v;
        }
      }
    }
  });
}

template <typename T, bool INV, int L, int... Rs>
__global__ void __launch_bounds__(Shape<T, L, Rs...>::NT, Shape<T, L, Rs...>::min_blocks) k_tiles(const __grid_constant__ TileArgs<T> a) {
  pdl_entry();
  extern __shared__ __align__(16) unsigned char smraw[];
  tile_body<T, INV, L, rows::DevT, Rs...>(a, (long long)blockIdx.x, (long long)blockIdx.y,
                                          reinterpret_cast<cpx<T> *>(smraw), rows::DevT{});
}

template <typename T, int L, int... Rs>
constexpr size_t smem_of() {
  return (size_t)Shape<T, L, Rs...>::W * slot_len<L>() * sizeof(cpx<T>);
}

#ifndef FFB_HOST_EMULATION
template <typename T, bool INV, int L, int... Rs>
cudaError_t launch(const TileArgs<T> &a, cudaStream_t s) {
  {
    cudaError_t e = set_smem_limit_once<k_tiles<T, INV, L, Rs...>>((int)smem_of<T, L, Rs...>());
    if (e != cudaSuccess) return e;
  }
  using Sh = Shape<T, L, Rs...>;
  dim3 grid((unsigned)((a.G + Sh::W - 1) / Sh::W), (unsigned)a.nbatch, 1);
  return launch_pdl(k_tiles<T, INV, L, Rs...>, grid, dim3(Sh::NT), smem_of<T, L, Rs...>(), s, a);
}
#else
template <typename T, bool INV, int L, int... Rs>
cudaError_t launch(const TileArgs<T> &a, cudaStream_t) {
  using Sh = Shape<T, L, Rs...>;
  std::vector<unsigned char> buf(smem_of<T, L, Rs...>() + 64);
  cpx<T> *sm = reinterpret_cast<cpx<T> *>(buf.data());
  const long long tiles = (a.G + Sh::W - 1) / Sh::W;
  for (long long by = 0; by < a.nbatch; ++by)
    for (long long bx = 0; bx < tiles; ++bx) {
      std::memset(buf.data(), 0xff, buf.size());
      tile_body<T, INV, L, rows::HostT, Rs...>(a, bx, by, sm, rows::HostT{});
    }
  return cudaSuccess;
}
#endif

}  // namespace tiles
}  // namespace ffb
