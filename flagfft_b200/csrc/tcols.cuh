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

// Shared-memory twiddle table of sequence Q: stage s > 0 block at
// tw_off_of(s), of (R_s - 1) * span_s entries, or 2 * ceil((R_s - 1) / 2) *
// span_s as pairs (stage 0 reads none).
template <class Q, bool PAIRS>
FFB_HD constexpr int tw_off_of(int s) {
  int o = 0;
  for (int i = 1; i < s; ++i) o += (PAIRS ? 2 * (Q::r(i) / 2) : Q::r(i) - 1) * Q::span(i);
  return o;
}
template <bool PAIRS, int... Rs>
FFB_HD constexpr int tw_table_elems() {
  return tw_off_of<Seq<Rs...>, PAIRS>(Seq<Rs...>::n);
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
  // ring slots start on 128-byte boundaries (a TMA copy's shared-memory
  // address must be 128-byte aligned, and the working layout's padding makes
  // a tile a little longer than GC * L elements)
  static constexpr size_t buf_bytes = (raw_elems * sizeof(cpx<T>) + 127) / 128 * 128;
  static constexpr size_t buf_elems = buf_bytes / sizeof(cpx<T>);
  static constexpr size_t head = 128;  // mbarriers; the ring starts 128-byte aligned
  // the sequence's twiddle blocks (stages 1.., stage 0 has none), copied
  // into shared memory after the ring where they fit: read once per stage
  // element, from global memory they miss the L1 the ring leaves.  Single
  // precision keeps them as pairs (rows::TW_PAIRS), double as the host's block.
  static constexpr int tw_elems = tw_table_elems<sizeof(T) == 4, Rs...>();
  static constexpr size_t tw_bytes = ((size_t)tw_elems * sizeof(cpx<T>) + 127) / 128 * 128;
  static constexpr bool tw_fits = head + NBUF * buf_bytes + tw_bytes <= 232448;
  static constexpr int TWS = !tw_fits ? rows::TW_GLOBAL : sizeof(T) == 4 ? rows::TW_PAIRS : rows::TW_SHARED;
  static constexpr size_t tw_at = head + NBUF * buf_bytes;
  static constexpr size_t smem = head + NBUF * buf_bytes + (tw_fits ? tw_bytes : 0);
  static_assert(buf_bytes % 128 == 0 && head % 128 == 0, "ring slots must stay 128-byte aligned");
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

// W_N^m (conjugated for the inverse) from the two split tables, m < N.
template <typename T>
FFB_HD cpx<T> split_root(const TileArgs<T> &a, uint32_t m) {
  const uint32_t hi = fdiv(m, a.ptw_div);
  cpx<T> t = cmul(ldg_c(a.ptw_hi + hi), ldg_c(a.ptw_lo + (m - hi * a.ptw_div.d)));
  if (a.inv) t.y = -t.y;
  return t;
}

// Last-stage writer: the optional four-step post-twiddle W_N^{g k} of a live
// transform g, then the raw tile.  Outputs k = base + q S of one butterfly
// take W^{g base} W^{g q S}: the first factor once per butterfly, the second
// the same in every thread of a transform (one cached line per warp) --
// instead of two scattered table reads per output.
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
      const cpx<T> t0 = split_root(*a, (uint32_t)(g * base));
      y[0] = cmul(x[0], t0);
#pragma unroll
      for (int q = 1; q < R; ++q) y[q] = cmul(x[q], cmul(t0, split_root(*a, (uint32_t)(g * (long long)(q * S)))));
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
// tw: the host's twiddle block in global memory (TWS = rows::TW_GLOBAL) or
// the shared-memory table (tw_table_off layout).
template <typename T, bool INV, int L, class Sh, class Q, int S, bool IN_ROWS, bool OUT_ROWS, int TWS, class X>
FFB_HD void run_stages(const X &x, const TileArgs<T> &a, const cpx<T> *tw, cpx<T> *raw, long long g0) {
  static_assert(Q::n >= 2, "the tile is read by the first stage and written by the last");
  constexpr int R = Q::r(S), Ns = Q::span(S);
  constexpr int TwOff = TWS == rows::TW_GLOBAL ? Q::twoff(S) : tw_off_of<Q, TWS == rows::TW_PAIRS>(S);
  constexpr int GC = Sh::GC, TPT = Sh::TPT, NT = Sh::NT;
  constexpr bool first = S == 0, last = S == Q::n - 1;
  constexpr bool cfast = (first && !IN_ROWS) || (last && !OUT_ROWS);
  using Regs = rows::StageRegs<T, L, TPT, R>;
  auto rd = [&](int tid) FFB_INL {
    const int c = cfast ? tid % GC : tid / TPT, t = cfast ? tid / GC : tid % TPT;
    if constexpr (first) {
      if constexpr (IN_ROWS)
        return rows::stage_read<T, INV, L, TPT, Ns, R, TWS>(t, tw + TwOff, RawRows<T>{raw + c * L});
      else
        return rows::stage_read<T, INV, L, TPT, Ns, R, TWS>(t, tw + TwOff, RawCols<T, GC>{raw, c});
    } else {
      return rows::stage_read<T, INV, L, TPT, Ns, R, TWS>(t, tw + TwOff, SwzIO<T>{raw + c * (L + Sh::PAD)});
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
    run_stages<T, INV, L, Sh, Q, S + 1, IN_ROWS, OUT_ROWS, TWS>(x, a, tw, raw, g0);
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

// The shared-memory twiddle table (layout Sh::TWS) from the host's block.
template <typename T, class Sh, class Q>
FFB_HD void fill_twiddles(cpx<T> *tws, const cpx<T> *g, int tid) {
  if constexpr (Sh::TWS == rows::TW_SHARED) {
    for (int e = tid; e < Sh::tw_elems; e += Sh::NT) tws[e] = ldg_c(g + (Q::r(0) - 1) + e);
  } else if constexpr (Sh::TWS == rows::TW_PAIRS) {
#pragma unroll
    for (int st = 1; st < Q::n; ++st) {  // (unrolled: the radices fold to constants)
      const int R = Q::r(st), Ns = Q::span(st), pairs = R / 2;
      cpx<T> *blk = tws + tw_off_of<Q, true>(st);
      const cpx<T> *src = g + Q::twoff(st);
      for (int e = tid; e < 2 * pairs * Ns; e += Sh::NT) {
        const int h = e & 1, mk_ = e >> 1, m = mk_ / Ns, k = mk_ - m * Ns, r = 2 * m + h + 1;
        blk[e] = r <= R - 1 ? ldg_c(src + (r - 1) * Ns + k) : mk((T)1, (T)0);
      }
    }
  }
}

#ifndef FFB_HOST_EMULATION

// Copies of one group: one box each way (a row tile: GC rows of L; a column
// tile: GC columns of L as [L / RB][RB][GC]), issued by one thread.  A
// load's bytes complete on `bar`; a store is one bulk group.
template <typename T, int L, int GC, int RB>
__device__ __forceinline__ void issue_load(const Args<T> &p, const CUtensorMap *map, long long q, cpx<T> *raw,
                                           uint64_t *bar) {
  const Group gr = group_of<GC>(q, p.groups_per_batch);
  tma::mbar_expect_tx(bar, (uint32_t)(GC * L * sizeof(cpx<T>)));
  if (p.in_rows)
    tma::load_4d(raw, map, 0, 0, (int)gr.g0, (int)gr.b, bar);
  else
    tma::load_4d(raw, map, (int)(2 * gr.g0), 0, 0, (int)gr.b, bar);
}

template <typename T, int L, int GC, int RB>
__device__ __forceinline__ void issue_store(const Args<T> &p, const CUtensorMap *map, long long q, const cpx<T> *raw) {
  const Group gr = group_of<GC>(q, p.groups_per_batch);
  if (p.out_rows)
    tma::store_4d(map, 0, 0, (int)gr.g0, (int)gr.b, raw);
  else
    tma::store_4d(map, (int)(2 * gr.g0), 0, 0, (int)gr.b, raw);
  tma::commit();
}

// Device counter of waits that gave up (copies that never landed).
static __device__ int g_tcols_wait_failures;

// The CTA's threads synchronise on named barrier 1 (the whole CTA).
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
  // barrier 1 with an OR over the threads' predicates
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

// One CTA per SM, NT threads, all of them transforming; thread 0 also issues
// every copy, one TMA instruction per group and direction (a separate
// producer warp would make 17 warps, five on one scheduler, and cap the
// registers at 96: the radix-16 stages spilled).  Group i lives in ring slot
// i % 3.  At the start of group i (after the barrier that ends group i - 1,
// whose writes every thread fenced for the async proxy) thread 0 stores
// group i - 1, waits until its store of group i - 2 has read its slot out --
// issued a group of compute earlier, so in practice no wait -- and loads
// group i + 1 into that slot: a load has a group of compute to land.
// (Loading group i + 2 late in group i instead, once the store of group
// i - 1 has drained, measured 8-26% slower on the 2^24-point real
// transforms: thread 0's wait for that store held every warp at the next
// barrier.)  full[s] counts a load's bytes.  Every wait is bounded; a wait
// that gives up is counted in g_tcols_wait_failures, the threads leave the
// loop together and thread 0 lets the load in flight land before the CTA
// ends.
template <typename T, bool INV, int L, bool IN_ROWS, bool OUT_ROWS, int... Rs>
__global__ void __launch_bounds__(Shape<T, L, Rs...>::NT, 1) k_tcols(const __grid_constant__ Args<T> p) {
  pdl_entry();
  using Sh = Shape<T, L, Rs...>;
  using Q = Seq<Rs...>;
  constexpr int NB = Sh::NBUF;
  static_assert(NB == 3, "the copy schedule is written for three slots");
  extern __shared__ __align__(1024) unsigned char smraw[];
  uint64_t *full = reinterpret_cast<uint64_t *>(smraw);  // [NB]
  cpx<T> *ring = reinterpret_cast<cpx<T> *>(smraw + Sh::head);
  const int tid = (int)threadIdx.x;
  const bool issuer = tid == 0;
  const long long q0 = blockIdx.x, step = gridDim.x;
  auto group = [&](long long i) { return q0 + i * step; };
  auto slot = [&](long long i) { return ring + (i % NB) * Sh::buf_elems; };
  if (tid == 0) {
    for (int k = 0; k < NB; ++k) tma::mbar_init(&full[k], 1);
    tma::fence_mbar_init();
  }
  __syncwarp();
  if (issuer && group(0) < p.total_groups) issue_load<T, L, Sh::GC, Sh::RB>(p, &p.in_map, group(0), slot(0), &full[0]);
  const ComputeThreads x{Sh::NT};
  const cpx<T> *tw = p.a.tw;
  if constexpr (Sh::TWS != rows::TW_GLOBAL) {
    cpx<T> *tws = reinterpret_cast<cpx<T> *>(smraw + Sh::tw_at);
    fill_twiddles<T, Sh, Q>(tws, p.a.tw, tid);
    tw = tws;
  }
  __syncthreads();  // barriers initialised, twiddles in place
  long long i = 0;
  bool failed = false;
  for (; group(i) < p.total_groups; ++i) {
    const bool ok = tma::mbar_wait(&full[i % NB], (uint32_t)((i / NB) & 1));
    if (x.sync_or(!ok)) {  // every thread agrees; group i - 1 is written
      failed = true;
      break;
    }
    if (issuer) {
      if (i > 0) issue_store<T, L, Sh::GC, Sh::RB>(p, &p.out_map, group(i - 1), slot(i - 1));
      if (group(i + 1) < p.total_groups) {
        tma::wait_read<1>();  // the store of group i - 2 has read slot (i + 1) % 3 out
        issue_load<T, L, Sh::GC, Sh::RB>(p, &p.in_map, group(i + 1), slot(i + 1), &full[(i + 1) % NB]);
      }
    }
    const Group gr = group_of<Sh::GC>(group(i), p.groups_per_batch);
    run_stages<T, INV, L, Sh, Q, 0, IN_ROWS, OUT_ROWS, Sh::TWS>(x, p.a, tw, slot(i), gr.g0);
    tma::fence_async_smem();  // this thread's writes, before thread 0's TMA store reads them
  }
  x.sync();  // the last group is written (or the threads left together)
  if (issuer) {
    if (!failed && i > 0) issue_store<T, L, Sh::GC, Sh::RB>(p, &p.out_map, group(i - 1), slot(i - 1));
    tma::wait_all<0>();
    if (failed) {
      atomicAdd(&g_tcols_wait_failures, 1);
      // the load in flight (group i) lands before the CTA ends (bounded)
      tma::mbar_wait(&full[i % NB], (uint32_t)((i / NB) & 1));
    }
  }
}

#endif  // !FFB_HOST_EMULATION

}  // namespace tcols
}  // namespace ffb
