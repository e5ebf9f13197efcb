// Column passes of long compile-time sequences (1024, 2048, 4096 points)
// with TMA-staged tiles.
//
// A strided pass over transforms of L points (element i of transform g at
// g + i * ii: a column of a row-major matrix) is coalesced only when a CTA
// moves several adjacent columns at once, and at L = 4096 the columns one CTA
// can hold (a padded buffer per transform) fill its shared memory: the plain
// tile kernel then loads, transforms and stores one tile after the other with
// nothing to overlap.  Here a persistent CTA walks a sequence of column groups
// (GC adjacent transforms) and keeps two raw landing buffers beside one padded
// working buffer:
//   * the TMA unit loads group i + 1 into one raw buffer while the threads
//     transform group i (the load is issued right after group i's first
//     stage, once the store that last read that buffer has drained);
//   * stage 0 reads group i's raw tile (dense, the layout the copy left) and
//     writes the padded working buffer; the middle stages run in place there
//     (values held in registers across a barrier); the last stage writes the
//     output tile into the raw buffer in the output's dense layout, with the
//     optional four-step post-twiddle;
//   * one thread stores the tile with a TMA store and moves on.
// A tile layout is "columns" ([i][c]: the transforms adjacent in memory, a
// copy moves 256-row boxes of GC columns) or "rows" ([c][i]: each transform's
// elements contiguous, one copy moves GC whole rows).  A stage that touches a
// column-layout tile maps consecutive threads to consecutive transforms, so a
// warp's shared-memory accesses are contiguous.
#pragma once

#include "rows.cuh"
#include "tma.cuh"

namespace ffb {
namespace tcols {

using rows::Seq;
using rows::slot_len;
using rows::SmemIO;

template <typename T, int L, int... Rs>
struct Shape {
  static constexpr int TPT = rows::rows_tpt<T, L, Rs...>();
  static constexpr int NT = tile::TileBounds<T>::kMaxThreads;  // threads per CTA
  static constexpr int GC = NT / TPT;                          // transforms per group
  static constexpr int slot = slot_len<L>();
  static constexpr int RB = L < 256 ? L : 256;  // rows per column-layout box
  static constexpr size_t raw_elems = (size_t)GC * L;
  static constexpr size_t raw_bytes = raw_elems * sizeof(cpx<T>);
  static constexpr size_t head = 1024;  // two mbarriers, padded so the raw tiles start 1 KB-aligned
  static constexpr size_t smem = head + 2 * raw_bytes + (size_t)GC * slot * sizeof(cpx<T>);
  static_assert(NT % TPT == 0 && GC >= 1, "threads per CTA must be a multiple of the threads per transform");
  static_assert((2 * GC * sizeof(T)) % 16 == 0, "a column box row must be a multiple of 16 bytes");
  static_assert(L % 128 == 0, "row tiles move 128-element chunks");
};

// Kernel arguments: the pass, its two tensor maps (device build) and views.
template <typename T>
struct alignas(64) Args {
#ifndef FFB_HOST_EMULATION
  CUtensorMap in_map;
  CUtensorMap out_map;
#endif
  tma::View in_view, out_view;
  TileArgs<T> a;
  long long groups_per_batch;  // ceil(G / GC)
  long long total_groups;      // groups_per_batch * nbatch
  int in_rows, out_rows;       // tile layouts (1 rows, 0 columns)
};

// Dense raw tiles: columns [i][c] and rows [c][i].
template <typename T, int GC>
struct RawCols {
  cpx<T> *b;
  int c;
  template <int S, int R>
  FFB_HD void get(int j, cpx<T> (&x)[R]) const {
#pragma unroll
    for (int r = 0; r < R; ++r) x[r] = b[(j + r * S) * GC + c];
  }
  template <int S, int R>
  FFB_HD void put(int base, const cpx<T> (&x)[R]) const {
#pragma unroll
    for (int q = 0; q < R; ++q) b[(base + q * S) * GC + c] = x[q];
  }
};
template <typename T>
struct RawRows {
  cpx<T> *b;  // this transform's row
  template <int S, int R>
  FFB_HD void get(int j, cpx<T> (&x)[R]) const {
#pragma unroll
    for (int r = 0; r < R; ++r) x[r] = b[j + r * S];
  }
  template <int S, int R>
  FFB_HD void put(int base, const cpx<T> (&x)[R]) const {
#pragma unroll
    for (int q = 0; q < R; ++q) b[base + q * S] = x[q];
  }
};

// Last-stage writer: the optional four-step post-twiddle W_N^{g k} of a live
// transform g, then the raw tile.
template <typename T, class W>
struct TwiddledOut {
  const TileArgs<T> *a;
  W w;
  long long g;
  bool tw;
  template <int S, int R>
  FFB_HD void put(int base, const cpx<T> (&x)[R]) const {
    if (tw) {
      cpx<T> y[R];
#pragma unroll
      for (int q = 0; q < R; ++q) y[q] = rows::post_twiddle(*a, x[q], g, base + q * S);
      w.template put<S, R>(base, y);
    } else {
      w.template put<S, R>(base, x);
    }
  }
};

// Stages S..SE-1 of sequence Q on group g0's tile: stage 0 reads the raw tile
// and writes the working buffers, the middle stages run in place on the
// working buffers (reads, barrier, writes), the last stage writes the raw
// tile.  A barrier separates consecutive stages; none follows stage SE-1.
template <typename T, bool INV, int L, class Sh, class Q, int S, int SE, bool IN_ROWS, bool OUT_ROWS, class X>
FFB_HD void run_stages(const X &x, const TileArgs<T> &a, cpx<T> *raw, cpx<T> *work, long long g0) {
  static_assert(Q::n >= 2, "the raw tile is read by the first stage and written by the last");
  constexpr int R = Q::r(S), Ns = Q::span(S), TwOff = Q::twoff(S);
  constexpr int GC = Sh::GC, TPT = Sh::TPT, NT = Sh::NT;
  constexpr bool first = S == 0, last = S == Q::n - 1;
  constexpr bool cfast = (first && !IN_ROWS) || (last && !OUT_ROWS);
  using Regs = rows::StageRegs<T, L, TPT, R>;
  auto rd = [&](int tid) FFB_INL {
    const int c = cfast ? tid % GC : tid / TPT, t = cfast ? tid / GC : tid % TPT;
    if constexpr (first) {
      if constexpr (IN_ROWS)
        return rows::stage_read<T, INV, L, TPT, Ns, R>(t, a.tw + TwOff, RawRows<T>{raw + c * L});
      else
        return rows::stage_read<T, INV, L, TPT, Ns, R>(t, a.tw + TwOff, RawCols<T, GC>{raw, c});
    } else {
      return rows::stage_read<T, INV, L, TPT, Ns, R>(t, a.tw + TwOff, SmemIO<T>{work + c * Sh::slot});
    }
  };
  auto wr = [&](int tid, const Regs &st) FFB_INL {
    const int c = cfast ? tid % GC : tid / TPT, t = cfast ? tid / GC : tid % TPT;
    if constexpr (last) {
      const long long g = g0 + c;
      const bool tw = a.post_twiddle != 0 && g < a.G;  // dead columns: no table reads past the pass
      if constexpr (OUT_ROWS)
        rows::stage_write<T, L, TPT, Ns, R>(t, st, TwiddledOut<T, RawRows<T>>{&a, RawRows<T>{raw + c * L}, g, tw});
      else
        rows::stage_write<T, L, TPT, Ns, R>(t, st, TwiddledOut<T, RawCols<T, GC>>{&a, RawCols<T, GC>{raw, c}, g, tw});
    } else {
      rows::stage_write<T, L, TPT, Ns, R>(t, st, SmemIO<T>{work + c * Sh::slot});
    }
  };
  if constexpr (first || last) {
    // reads and writes touch different buffers
    x.each(NT, [&](int tid) FFB_INL { wr(tid, rd(tid)); });
  } else {
    x.each2(NT, rd, wr);
  }
  if constexpr (S + 1 < SE) {
    x.sync();
    run_stages<T, INV, L, Sh, Q, S + 1, SE, IN_ROWS, OUT_ROWS>(x, a, raw, work, g0);
  }
}

// Coordinates of group q: outer batch b, first transform g0.
struct Group {
  long long b, g0;
};
template <int GC>
FFB_HD Group group_of(long long q, long long per_batch) {
  return {q / per_batch, (q % per_batch) * GC};
}

#ifndef FFB_HOST_EMULATION

template <typename T, int L, int GC, int RB>
__device__ __forceinline__ void issue_load(const Args<T> &p, const CUtensorMap *map, long long q, cpx<T> *raw,
                                           uint64_t *bar) {
  const Group gr = group_of<GC>(q, p.groups_per_batch);
  tma::mbar_expect_tx(bar, (uint32_t)(GC * L * sizeof(cpx<T>)));
  if (p.in_rows) {
    tma::load_4d(raw, map, 0, 0, (int)gr.g0, (int)gr.b, bar);
  } else {
#pragma unroll 1
    for (int k = 0; k < L / RB; ++k) tma::load_4d(raw + k * RB * GC, map, (int)(2 * gr.g0), k * RB, (int)gr.b, 0, bar);
  }
}

template <typename T, int L, int GC, int RB>
__device__ __forceinline__ void issue_store(const Args<T> &p, const CUtensorMap *map, long long q, const cpx<T> *raw) {
  const Group gr = group_of<GC>(q, p.groups_per_batch);
  if (p.out_rows) {
    tma::store_4d(map, 0, 0, (int)gr.g0, (int)gr.b, raw);
  } else {
#pragma unroll 1
    for (int k = 0; k < L / RB; ++k) tma::store_4d(map, (int)(2 * gr.g0), k * RB, (int)gr.b, 0, raw + k * RB * GC);
  }
  tma::commit();
}

// Device counter of waits that gave up (copies that never landed).
static __device__ int g_tcols_wait_failures;

template <typename T, bool INV, int L, bool IN_ROWS, bool OUT_ROWS, int... Rs>
__global__ void __launch_bounds__(Shape<T, L, Rs...>::NT, 1) k_tcols(const __grid_constant__ Args<T> p) {
  using Sh = Shape<T, L, Rs...>;
  using Q = Seq<Rs...>;
  extern __shared__ __align__(1024) unsigned char smraw[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(smraw);
  cpx<T> *raw0 = reinterpret_cast<cpx<T> *>(smraw + Sh::head);
  cpx<T> *raw1 = raw0 + Sh::raw_elems;
  cpx<T> *work = raw1 + Sh::raw_elems;
  const int tid = (int)threadIdx.x;
  if (tid == 0) {
    tma::mbar_init(&bar[0], 1);
    tma::mbar_init(&bar[1], 1);
    tma::fence_mbar_init();
  }
  __syncthreads();
  long long q = blockIdx.x;
  if (tid == 0 && q < p.total_groups) issue_load<T, L, Sh::GC, Sh::RB>(p, &p.in_map, q, raw0, &bar[0]);
  const rows::DevT x{};
  int failed_slot = -1;
  uint32_t failed_parity = 0;
  for (int i = 0; q < p.total_groups; ++i, q += gridDim.x) {
    const int s = i & 1;
    cpx<T> *raw = s ? raw1 : raw0;
    const uint32_t parity = (uint32_t)((i >> 1) & 1);
    const bool ok = tma::mbar_wait(&bar[s], parity);
    if (__syncthreads_or(!ok)) {
      failed_slot = s;
      failed_parity = parity;
      break;
    }
    const Group gr = group_of<Sh::GC>(q, p.groups_per_batch);
    // stage 0 (raw tile -> working buffers); then, while the other stages
    // run, the next group's load into the other raw buffer
    run_stages<T, INV, L, Sh, Q, 0, 1, IN_ROWS, OUT_ROWS>(x, p.a, raw, work, gr.g0);
    __syncthreads();
    if (tid == 0) {
      const long long qn = q + gridDim.x;
      if (qn < p.total_groups) {
        tma::wait_read<0>();  // the store that last read that buffer has drained
        issue_load<T, L, Sh::GC, Sh::RB>(p, &p.in_map, qn, s ? raw0 : raw1, &bar[s ^ 1]);
      }
    }
    run_stages<T, INV, L, Sh, Q, 1, Q::n, IN_ROWS, OUT_ROWS>(x, p.a, raw, work, gr.g0);
    tma::fence_async_smem();
    __syncthreads();
    if (tid == 0) issue_store<T, L, Sh::GC, Sh::RB>(p, &p.out_map, q, raw);
  }
  if (tid == 0) {
    tma::wait_all<0>();
    if (failed_slot >= 0) {
      atomicAdd(&g_tcols_wait_failures, 1);
      tma::mbar_wait(&bar[failed_slot], failed_parity);  // bounded: the copy that did not land
    }
  }
}

#endif  // !FFB_HOST_EMULATION

}  // namespace tcols
}  // namespace ffb
