// Column passes of long compile-time sequences (1024, 2048, 4096 points)
// with TMA-staged tiles.
//
// A strided pass over transforms of L points (element i of transform g at
// g + i * ii: a column of a row-major matrix) is coalesced only when a CTA
// moves several adjacent columns at once, and at L = 4096 the columns one CTA
// can hold fill most of its shared memory: a kernel that loads, transforms and
// stores one tile after the other has nothing to overlap.  Here a persistent
// CTA walks a sequence of column groups (GC adjacent transforms) through a
// ring of three tile buffers:
//   * a producer warp keeps the next two groups' loads in flight (TMA tensor
//     copies completing on an mbarrier per buffer), stores each finished
//     group with a TMA store, and refills the buffer once the store has read
//     it out;
//   * the compute warps transform a group in place in its buffer: stage 0
//     reads the tile in the layout the copy left, every stage holds its
//     values in registers across a barrier and writes them back, the middle
//     stages in a swizzled layout (element i of transform c at
//     c * (L + PAD) + (i ^ ((i >> 4) & 15)): the radix-16 Stockham strides
//     then fall on distinct banks, and PAD spreads the transforms one
//     wavefront touches over the banks, so a tile needs no second buffer),
//     and the last stage writes the output layout, with the optional
//     four-step post-twiddle.
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

// Transforms per group: as many as the precision's thread limit allows,
// rounded down to an even count in single precision (a column box row must
// be a multiple of 16 bytes).
template <typename T>
constexpr int tcols_gc(int tpt) {
  const int g = tile::TileBounds<T>::kMaxThreads / tpt;
  return sizeof(T) == 4 ? g / 2 * 2 : g;
}

template <typename T, int L, int... Rs>
struct Shape {
  static constexpr int TPT = rows::rows_tpt<T, L, Rs...>();
  static constexpr int GC = tcols_gc<T>(TPT);  // transforms per group
  static constexpr int NT = GC * TPT;          // compute threads per CTA
  static constexpr int RB = L < 256 ? L : 256;  // rows per column-layout box
  static constexpr int NBUF = 3;                // tile buffers in the ring
  // working layout: transform c at c * (L + PAD), so that the GC transforms
  // of one shared-memory wavefront (128 bytes) start on distinct banks
  static constexpr int PAD = (int)(128 / sizeof(cpx<T>)) / GC;
  static constexpr size_t raw_elems = (size_t)GC * L + (size_t)(GC - 1) * PAD;  // one tile, working layout included
  // ring slots start 1 KB apart: a TMA copy's shared-memory address must be
  // 128-byte aligned, and the working layout's padding makes a tile a little
  // longer than GC * L elements
  static constexpr size_t buf_bytes = (raw_elems * sizeof(cpx<T>) + 1023) / 1024 * 1024;
  static constexpr size_t buf_elems = buf_bytes / sizeof(cpx<T>);
  static constexpr size_t head = 1024;  // mbarriers, padded so the tiles start 1 KB-aligned
  static constexpr size_t smem = head + NBUF * buf_bytes;
  static_assert(buf_bytes % 1024 == 0 && head % 1024 == 0, "ring slots must stay 1 KB-aligned");
  static_assert(GC >= 1 && NT % 32 == 0, "a group needs one or more transforms and whole warps");
  static_assert((2 * GC * sizeof(T)) % 16 == 0, "a column box row must be a multiple of 16 bytes");
  static_assert(L % 128 == 0, "row tiles move 128-element chunks");
  static_assert(smem <= 232448, "the tile ring must fit one CTA's shared memory");
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

// A transform's working layout: element i at i ^ ((i >> 4) & 15) (a
// permutation inside each 16-element block).
FFB_HD constexpr int swz(int i) { return i ^ ((i >> 4) & 15); }
template <typename T>
struct SwzIO {
  cpx<T> *b;  // this transform's L elements
  template <int S, int R>
  FFB_HD void get(int j, cpx<T> (&x)[R]) const {
#pragma unroll
    for (int r = 0; r < R; ++r) x[r] = b[swz(j + r * S)];
  }
  template <int S, int R>
  FFB_HD void put(int base, const cpx<T> (&x)[R]) const {
#pragma unroll
    for (int q = 0; q < R; ++q) b[swz(base + q * S)] = x[q];
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

// Stages S.. of sequence Q on group g0's tile, in place: stage 0 reads the
// tile in the input's layout, the last writes it in the output's layout, the
// ones between use the swizzled working layout.  Every stage reads, crosses a
// barrier (its values wait in registers) and writes; a barrier separates
// consecutive stages and none follows the last.
template <typename T, bool INV, int L, class Sh, class Q, int S, bool IN_ROWS, bool OUT_ROWS, class X>
FFB_HD void run_stages(const X &x, const TileArgs<T> &a, cpx<T> *raw, long long g0) {
  static_assert(Q::n >= 2, "the tile is read by the first stage and written by the last");
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
      return rows::stage_read<T, INV, L, TPT, Ns, R>(t, a.tw + TwOff, SwzIO<T>{raw + c * (L + Sh::PAD)});
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
      rows::stage_write<T, L, TPT, Ns, R>(t, st, SwzIO<T>{raw + c * (L + Sh::PAD)});
    }
  };
  x.each2(NT, rd, wr);
  if constexpr (!last) {
    x.sync();
    run_stages<T, INV, L, Sh, Q, S + 1, IN_ROWS, OUT_ROWS>(x, a, raw, g0);
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

// The compute threads (warps 0 .. NT/32 - 1) synchronise among themselves on
// named barrier 1, so the producer warp never holds them up.
struct ComputeThreads {
  int nt;
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
    asm volatile("bar.sync 1, %0;" ::"r"(nt) : "memory");
#endif
  }
  template <class FR, class FW>
  FFB_HD void each2(int, FR &&rd, FW &&wr) const {
#ifdef __CUDA_ARCH__
    const auto st = rd((int)threadIdx.x);
    sync();
    wr((int)threadIdx.x, st);
#else
    (void)rd;
    (void)wr;
#endif
  }
  // barrier 1 with an OR over the compute threads' predicates
  __device__ __forceinline__ bool sync_or(bool v) const {
    uint32_t r;
    asm volatile(
        "{\n"
        "  .reg .pred p, q;\n"
        "  setp.ne.u32 p, %1, 0;\n"
        "  barrier.cta.red.or.pred q, 1, %2, p;\n"
        "  selp.u32 %0, 1, 0, q;\n"
        "}\n"
        : "=r"(r)
        : "r"((uint32_t)v), "r"(nt)
        : "memory");
    return r != 0;
  }
};

// One CTA per SM, NT compute threads plus one producer warp.
//   producer (lane 0 of the last warp): loads the first NBUF groups into the
//     ring (full[s] counts each load's bytes); for every group, once the
//     compute warps report it written (ready[s]) it stores the tile, waits
//     for the store to read the buffer out, and loads the group NBUF ahead
//     into it;
//   compute warps: wait full[s], run the stages in place, report ready[s].
// Every wait is bounded; a wait that gives up is counted in
// g_tcols_wait_failures and ends the loop on both sides (the compute
// threads decide together, so none is left at a barrier).
template <typename T, bool INV, int L, bool IN_ROWS, bool OUT_ROWS, int... Rs>
__global__ void __launch_bounds__(Shape<T, L, Rs...>::NT + 32, 1) k_tcols(const __grid_constant__ Args<T> p) {
  pdl_entry();
  using Sh = Shape<T, L, Rs...>;
  using Q = Seq<Rs...>;
  constexpr int NW = Sh::NT / 32, NB = Sh::NBUF;
  extern __shared__ __align__(1024) unsigned char smraw[];
  uint64_t *full = reinterpret_cast<uint64_t *>(smraw);  // [NB]
  uint64_t *ready = full + NB;                           // [NB]
  cpx<T> *ring = reinterpret_cast<cpx<T> *>(smraw + Sh::head);
  const int tid = (int)threadIdx.x;
  if (tid == 0) {
    for (int k = 0; k < NB; ++k) {
      tma::mbar_init(&full[k], 1);
      tma::mbar_init(&ready[k], NW);
    }
    tma::fence_mbar_init();
  }
  __syncthreads();
  const long long q0 = blockIdx.x, step = gridDim.x;
  if (tid >= Sh::NT) {
    // ---- producer warp
    if (tid != Sh::NT) return;
    bool failed = false;
    for (int k = 0; k < NB; ++k)
      if (q0 + k * step < p.total_groups)
        issue_load<T, L, Sh::GC, Sh::RB>(p, &p.in_map, q0 + k * step, ring + k * Sh::buf_elems, &full[k]);
    int i = 0;
    for (long long q = q0; q < p.total_groups; q += step, ++i) {
      const int s = i % NB;
      cpx<T> *buf = ring + s * Sh::buf_elems;
      if (!tma::mbar_wait(&ready[s], (uint32_t)((i / NB) & 1))) {
        failed = true;
        break;
      }
      issue_store<T, L, Sh::GC, Sh::RB>(p, &p.out_map, q, buf);
      const long long qn = q + NB * step;
      if (qn < p.total_groups) {
        tma::wait_read<0>();  // the store has read the buffer out
        issue_load<T, L, Sh::GC, Sh::RB>(p, &p.in_map, qn, buf, &full[s]);
      }
    }
    tma::wait_all<0>();
    if (failed) {
      atomicAdd(&g_tcols_wait_failures, 1);
      // loads still in flight land before the CTA ends (bounded)
      for (int k = 0; k < NB; ++k) {
        const int j = i + k;
        if (q0 + (long long)j * step < p.total_groups) tma::mbar_wait(&full[j % NB], (uint32_t)((j / NB) & 1));
      }
    }
    return;
  }
  // ---- compute warps
  const ComputeThreads x{Sh::NT};
  int i = 0;
  for (long long q = q0; q < p.total_groups; q += step, ++i) {
    const int s = i % NB;
    const bool ok = tma::mbar_wait(&full[s], (uint32_t)((i / NB) & 1));
    if (x.sync_or(!ok)) {  // all compute threads agree
      if (tid == 0) atomicAdd(&g_tcols_wait_failures, 1);
      break;
    }
    const Group gr = group_of<Sh::GC>(q, p.groups_per_batch);
    run_stages<T, INV, L, Sh, Q, 0, IN_ROWS, OUT_ROWS>(x, p.a, ring + s * Sh::buf_elems, gr.g0);
    tma::fence_async_smem();  // the tile's writes, before the producer's TMA store reads it
    __syncwarp();
    if ((tid & 31) == 0) tma::mbar_arrive(&ready[s]);
  }
}

#endif  // !FFB_HOST_EMULATION

}  // namespace tcols
}  // namespace ffb
