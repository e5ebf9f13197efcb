// One-pass Bluestein over a four-step convolution held in one CTA.
//
// For a length-n Bluestein whose convolution length M = N1 x L2 does not fit
// one ping-pong row but whose N1 rows of L2 points fit shared memory as one
// padded buffer each (f32: L2 = 2048, N1 <= 13 is 174-227 KB), one CTA runs
// the whole chain of one transform:
//   1. columns: a_j = x_j c_j (j = j1 L2 + j2 < n, else 0), the N1-point DFT
//      over j1 in registers, times W_M^{k1 j2}, into row k1 of shared memory;
//   2. rows: the L2-point Stockham FFT of every row (compile-time sequence),
//      times the kernel spectrum B[k1 + N1 k2] / M in registers, then the
//      inverse FFT;
//   3. columns: times W_M^{-k1 j2}, the inverse N1-point DFT over k1, times
//      the chirp, y_j for j < n straight to global memory.
// Every element crosses HBM once each way, against five transits of the
// M-point workspace for the three-pass chain (src/exec/raw_nodes.cpp:153-204
// runs the same chain as separate launches).  Row stages hold their values in
// registers across a barrier between reads and writes; the rows are done in
// two groups so that only half of the convolution is in registers at a time
// (row_pipe).
#pragma once

#include <atomic>

#include "rows.cuh"

namespace ffb {
namespace blue4 {

using rows::Seq;
using rows::SmemIO;
using rows::SmemKernIO;
using rows::slot_len;
using rows::tpt_of;

// W_M^m (forward sign) from the pass's two split four-step tables, m < M.
template <typename T>
FFB_HD cpx<T> split_twiddle(const TileArgs<T> &a, uint32_t m) {
  const uint32_t hi = fdiv(m, a.ptw_div);
  return cmul(ldg_c(a.ptw_hi + hi), ldg_c(a.ptw_lo + (m - hi * a.ptw_div.d)));
}

// Shape of the kernel for N1 rows of sequence Rs...: TPT threads per row,
// rows processed in two groups of NR, NT threads in all.
template <int N1, int L2, int... Rs>
struct Shape {
  static constexpr int TPT = tpt_of(L2, Seq<Rs...>::rmax());
  static constexpr int NR = (N1 + 1) / 2;
  static constexpr int NG = (N1 + NR - 1) / NR;
  static constexpr int NT = NR * TPT;
  static constexpr int slot = slot_len<L2>();
};

// The row convolution as one pipeline of 2 x nst stages (nst forward, then
// nst inverse; the last forward stage multiplies by the kernel spectrum row)
// over two groups of rows.  Step k reads group k % 2 of stage k / 2; between
// two barriers a thread writes what it read in the previous step and reads
// the next group:  R(0,0) | W(0,0) R(0,1) | W(0,1) R(1,0) | ... | W(last,1).
// A write and the read after it touch different row groups, and every read
// of a group follows a barrier after that group's previous writes, so a
// stage costs two barriers and a thread holds one group's values at a time.
template <typename T, int N1, int L2, class Q, class Sh, int S>
struct RowStage {
  static constexpr int nst = Q::n;
  static constexpr bool inv = S >= nst;
  static constexpr int qs = inv ? S - nst : S;
  static constexpr int R = Q::r(qs), Ns = Q::span(qs), TwOff = Q::twoff(qs);
  using Regs = rows::StageRegs<T, L2, Sh::TPT, R>;

  static FFB_HD Regs read(const TileArgs<T> &a, cpx<T> *sm, int grp, int tid) {
    const int wr_ = grp * Sh::NR + tid / Sh::TPT, t = tid % Sh::TPT;
    const int w = wr_ < N1 ? wr_ : N1 - 1;  // threads past the last row read a live row, write nothing
    return rows::stage_read<T, inv, L2, Sh::TPT, Ns, R>(t, (inv ? a.tw2 : a.tw) + TwOff, SmemIO<T>{sm + w * Sh::slot});
  }
  static FFB_HD void write(const TileArgs<T> &a, cpx<T> *sm, const cpx<T> *kern, int grp, int tid, const Regs &st) {
    const int w = grp * Sh::NR + tid / Sh::TPT, t = tid % Sh::TPT;
    if (w >= N1) return;
    if constexpr (S == nst - 1) {
      rows::stage_write<T, L2, Sh::TPT, Ns, R>(t, st, SmemKernIO<T>{sm + w * Sh::slot, kern + w * a.kern_stride});
    } else {
      rows::stage_write<T, L2, Sh::TPT, Ns, R>(t, st, SmemIO<T>{sm + w * Sh::slot});
    }
  }
};

// (host emulation instantiates it with per-thread state vectors).  kern: the
// kernel spectrum row of the first row in sm.
#pragma nv_exec_check_disable
template <typename T, int N1, int L2, class Q, class Sh, int K, class X, class St>
FFB_HD void row_pipe(const X &x, const TileArgs<T> &a, cpx<T> *sm, const cpx<T> *kern, const St &st) {
  static_assert(Sh::NG == 2, "the pipeline runs two row groups");
  constexpr int P = K - 1;  // the step whose reads st holds
  using Prev = RowStage<T, N1, L2, Q, Sh, P / 2>;
  if constexpr (K == 4 * Q::n) {
    x.last(Sh::NT, [&](int tid, const typename Prev::Regs &s) FFB_INL { Prev::write(a, sm, kern, P % 2, tid, s); }, st);
  } else {
    using Cur = RowStage<T, N1, L2, Q, Sh, K / 2>;
    auto nxt = x.step(
        Sh::NT,
        [&](int tid, const typename Prev::Regs &s) FFB_INL {
          Prev::write(a, sm, kern, P % 2, tid, s);
          return Cur::read(a, sm, K % 2, tid);
        },
        st);
    row_pipe<T, N1, L2, Q, Sh, K + 1>(x, a, sm, kern, nxt);
  }
}

// w[k1] = W_M^{k1 j2} for 1 <= k1 < N1: W^{j2} and W^{2 j2} from the split
// tables, the others as products (w[2m] = w[m]^2, w[k] = w[p] w[k - p] with
// p the highest power of two below k), at most three products deep.  Against
// a table pair for every k1 this cut C2C 10007 x 1024 from 176.9 to 162.1 us
// and 8009 x 1024 from 142.0 to 125.6 us on B200; the relative error stays
// within that of the same chain evaluated in single precision by the
// reference's algorithm (2.6e-7 against 2.9e-7 at N = 10007).
template <typename T, int N1>
FFB_HD void col_twiddles(const TileArgs<T> &a, int j2, cpx<T> (&w)[N1]) {
  w[1] = split_twiddle(a, (uint32_t)j2);
  if constexpr (N1 > 2) w[2] = split_twiddle(a, (uint32_t)(2 * j2));
#pragma unroll
  for (int k = 3; k < N1; ++k) {
    int p = 1;
    while (2 * p <= k) p *= 2;
    w[k] = p == k ? cmul(w[k / 2], w[k / 2]) : cmul(w[p], w[k - p]);
  }
}

// Column j2 of the forward column phase: a_j = x_j c_j for j = j1 L2 + j2
// (0 past n), the N1-point DFT over j1, times W_M^{k1 j2}.
template <typename T, int N1, int L2>
FFB_HD void col_forward(const TileArgs<T> &a, const cpx<T> *in, int j2, cpx<T> (&v)[N1]) {
  const int n = a.n;
#pragma unroll
  for (int j1 = 0; j1 < N1; ++j1) {
    const int i = j1 * L2 + j2;
    v[j1] = i < n ? cmul(rows::ld_stream(in + i), ldg_c(a.chirp + i)) : mk((T)0, (T)0);
  }
  dft_fixed<N1, false, T>(v);
  if (j2) {
    cpx<T> w[N1];
    col_twiddles<T, N1>(a, j2, w);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1) v[k1] = cmul(v[k1], w[k1]);
  }
}

// Column j2 of the inverse column phase from the convolution rows' values
// v[k1]: times W_M^{-k1 j2}, the inverse N1-point DFT over k1, times the
// chirp, y_j for j = j1 L2 + j2 < n.
template <typename T, int N1, int L2>
FFB_HD void col_inverse(const TileArgs<T> &a, cpx<T> *out, int j2, cpx<T> (&v)[N1]) {
  const int n = a.n;
  if (j2) {
    cpx<T> w[N1];
    col_twiddles<T, N1>(a, j2, w);
#pragma unroll
    for (int k1 = 1; k1 < N1; ++k1) v[k1] = cmul(v[k1], conjg(w[k1]));
  }
  dft_fixed<N1, true, T>(v);
#pragma unroll
  for (int j1 = 0; j1 < N1; ++j1) {
    const int i = j1 * L2 + j2;
    if (i < n) out[i] = cmul(v[j1], ldg_c(a.chirp + i));
  }
}

// One transform (batch index by) of the one-pass chain.  TileArgs: core /
// core2 the row sequence with tables tw / tw2, kern the N1 x L2 kernel
// spectrum rows (kern_stride = L2), chirp the n-point chirp, ptw_* the split
// W_M tables, n the logical length, ib / ob the transform distances.
#pragma nv_exec_check_disable
template <typename T, int N1, int L2, class X, int... Rs>
FFB_HD void blue4_body(const TileArgs<T> &a, long long by, cpx<T> *sm, const X &x) {
  using Q = Seq<Rs...>;
  using Sh = Shape<N1, L2, Rs...>;
  const cpx<T> *in = reinterpret_cast<const cpx<T> *>(a.in) + by * a.ib;
  cpx<T> *out = reinterpret_cast<cpx<T> *>(a.out) + by * a.ob;

  // 1. chirp, column DFT over j1, W_M^{k1 j2}, into row k1
  x.each(Sh::NT, [&](int tid) FFB_INL {
#pragma unroll 1
    for (int j2 = tid; j2 < L2; j2 += Sh::NT) {
      cpx<T> v[N1];
      col_forward<T, N1, L2>(a, in, j2, v);
      const int p = pp_pos(j2);
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) sm[k1 * Sh::slot + p] = v[k1];
    }
  });
  x.sync();

  // 2. row FFTs, kernel product, inverse row FFTs
  {
    using First = RowStage<T, N1, L2, Q, Sh, 0>;
    auto st = x.first(Sh::NT, [&](int tid) FFB_INL { return First::read(a, sm, 0, tid); });
    row_pipe<T, N1, L2, Q, Sh, 1>(x, a, sm, a.kern, st);
  }
  x.sync();

  // 3. W_M^{-k1 j2}, inverse column DFT over k1, chirp, y_j for j < n
  x.each(Sh::NT, [&](int tid) FFB_INL {
#pragma unroll 1
    for (int j2 = tid; j2 < L2; j2 += Sh::NT) {
      cpx<T> v[N1];
      const int p = pp_pos(j2);
#pragma unroll
      for (int k1 = 0; k1 < N1; ++k1) v[k1] = sm[k1 * Sh::slot + p];
      col_inverse<T, N1, L2>(a, out, j2, v);
    }
  });
}

// ---------------------------------------------------------------------------
// Pair form: one transform on a cluster of two CTAs.  Rank c holds rows
// [c NL, c NL + NL) of the N1 x L2 convolution (NL = N1 / 2) in its shared
// memory and owns columns [c L2 / 2, c L2 / 2 + L2 / 2): its column phases
// compute all N1 rows of its own columns and write (forward) or read
// (inverse) the peer's half through distributed shared memory; the row phase
// is the single-CTA pipeline over the NL local rows.  It makes double
// precision one pass (10 x 2048 rows are 348 KB, two CTAs' worth of shared
// memory); three cluster barriers per transform order the exchanges.  The
// planner takes it only on request: a pair CTA runs 12 warps, and on B200 it
// measured slower than one CTA (single precision) and than the three-pass
// chain (double precision) at N = 10007.
// ---------------------------------------------------------------------------

// The peer CTA's rows: st / ld of element i (padded position) through
// st/ld.shared::cluster at the peer's mapped address; in host emulation a
// plain pointer to the other emulated CTA's buffer.
template <typename T>
struct PeerRows {
  uintptr_t base;
  FFB_HD void st(int i, const cpx<T> &v) const {
#ifdef __CUDA_ARCH__
    const uint32_t adr = (uint32_t)base + (uint32_t)i * (uint32_t)sizeof(cpx<T>);
    if constexpr (sizeof(T) == 4) {
      asm volatile("st.shared::cluster.v2.f32 [%0], {%1, %2};" ::"r"(adr), "f"(v.x), "f"(v.y) : "memory");
    } else {
      asm volatile("st.shared::cluster.v2.f64 [%0], {%1, %2};" ::"r"(adr), "d"(v.x), "d"(v.y) : "memory");
    }
#else
    reinterpret_cast<cpx<T> *>(base)[i] = v;
#endif
  }
  FFB_HD cpx<T> ld(int i) const {
#ifdef __CUDA_ARCH__
    const uint32_t adr = (uint32_t)base + (uint32_t)i * (uint32_t)sizeof(cpx<T>);
    T x, y;
    if constexpr (sizeof(T) == 4) {
      asm volatile("ld.shared::cluster.v2.f32 {%0, %1}, [%2];" : "=f"(x), "=f"(y) : "r"(adr) : "memory");
    } else {
      asm volatile("ld.shared::cluster.v2.f64 {%0, %1}, [%2];" : "=d"(x), "=d"(y) : "r"(adr) : "memory");
    }
    return mk(x, y);
#else
    return reinterpret_cast<const cpx<T> *>(base)[i];
#endif
  }
};

template <int N1, int L2, int... Rs>
using PairShape = Shape<N1 / 2, L2, Rs...>;

// 1. rank c's columns: chirp, column DFT, twiddle; rows k1 < NL to rank 0,
// the rest to rank 1 (values chosen by select, so both stores are fixed).
#pragma nv_exec_check_disable
template <typename T, int N1, int L2, class X, int... Rs>
FFB_HD void pair_cols_in(const TileArgs<T> &a, long long by, int c, cpx<T> *own, const PeerRows<T> &peer,
                         const X &x) {
  using Sh = PairShape<N1, L2, Rs...>;
  constexpr int NL = N1 / 2, H = L2 / 2;
  const cpx<T> *in = reinterpret_cast<const cpx<T> *>(a.in) + by * a.ib;
  x.each(Sh::NT, [&](int tid) FFB_INL {
#pragma unroll 1
    for (int j2 = c * H + tid; j2 < c * H + H; j2 += Sh::NT) {
      cpx<T> v[N1];
      col_forward<T, N1, L2>(a, in, j2, v);
      const int p = pp_pos(j2);
#pragma unroll
      for (int r = 0; r < NL; ++r) {
        own[r * Sh::slot + p] = c ? v[NL + r] : v[r];
        peer.st(r * Sh::slot + p, c ? v[r] : v[NL + r]);
      }
    }
  });
}

// 2. the NL local rows: FFT, kernel product (rows c NL.. of the spectrum), IFFT.
#pragma nv_exec_check_disable
template <typename T, int N1, int L2, class X, int... Rs>
FFB_HD void pair_rows(const TileArgs<T> &a, int c, cpx<T> *own, const X &x) {
  using Q = Seq<Rs...>;
  using Sh = PairShape<N1, L2, Rs...>;
  constexpr int NL = N1 / 2;
  using First = RowStage<T, NL, L2, Q, Sh, 0>;
  auto st = x.first(Sh::NT, [&](int tid) FFB_INL { return First::read(a, own, 0, tid); });
  row_pipe<T, NL, L2, Q, Sh, 1>(x, a, own, a.kern + (long long)c * NL * a.kern_stride, st);
}

// 3. rank c's columns: all N1 rows (half from the peer), inverse column phase.
#pragma nv_exec_check_disable
template <typename T, int N1, int L2, class X, int... Rs>
FFB_HD void pair_cols_out(const TileArgs<T> &a, long long by, int c, const cpx<T> *own, const PeerRows<T> &peer,
                          const X &x) {
  using Sh = PairShape<N1, L2, Rs...>;
  constexpr int NL = N1 / 2, H = L2 / 2;
  cpx<T> *out = reinterpret_cast<cpx<T> *>(a.out) + by * a.ob;
  x.each(Sh::NT, [&](int tid) FFB_INL {
#pragma unroll 1
    for (int j2 = c * H + tid; j2 < c * H + H; j2 += Sh::NT) {
      cpx<T> v[N1];
      const int p = pp_pos(j2);
#pragma unroll
      for (int r = 0; r < NL; ++r) {
        const cpx<T> o = own[r * Sh::slot + p], q = peer.ld(r * Sh::slot + p);
        v[r] = c ? q : o;
        v[NL + r] = c ? o : q;
      }
      col_inverse<T, N1, L2>(a, out, j2, v);
    }
  });
}

// The input of transform nx into L2 (one bulk prefetch of its 16-byte
// aligned interior) while the CTA computes the current one.
template <typename T>
__device__ __forceinline__ void prefetch_input(const TileArgs<T> &a, long long nx) {
  const char *row = reinterpret_cast<const char *>(reinterpret_cast<const cpx<T> *>(a.in) + nx * a.ib);
  const uintptr_t b0 = (reinterpret_cast<uintptr_t>(row) + 15) & ~(uintptr_t)15;
  const uintptr_t b1 = (reinterpret_cast<uintptr_t>(row) + (size_t)a.n * sizeof(cpx<T>)) & ~(uintptr_t)15;
  if (b1 > b0) asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(b0), "r"((uint32_t)(b1 - b0)) : "memory");
}

template <typename T, int N1, int L2, int... Rs>
__global__ void __launch_bounds__(Shape<N1, L2, Rs...>::NT) k_blue4(const __grid_constant__ TileArgs<T> a) {
  pdl_entry();
  extern __shared__ __align__(16) unsigned char smraw[];
  for (long long by = blockIdx.x; by < a.nbatch; by += gridDim.x) {
    const long long nx = by + gridDim.x;
    if (threadIdx.x == 0 && nx < a.nbatch) prefetch_input(a, nx);
    blue4_body<T, N1, L2, rows::DevT, Rs...>(a, by, reinterpret_cast<cpx<T> *>(smraw), rows::DevT{});
    __syncthreads();  // the next transform's first phase rewrites the rows
  }
}

// All threads of both CTAs of the cluster; shared::cluster writes before it
// are visible to reads after it (release / acquire at cluster scope).
__device__ __forceinline__ void cluster_barrier() {
  asm volatile("barrier.cluster.arrive.release.aligned;\n\tbarrier.cluster.wait.acquire.aligned;" ::: "memory");
}

// CTAs per SM the pair kernel is compiled for: single precision's halves
// (87 KB at 10 x 2048) leave room for two.
template <typename T>
constexpr int pair_min_blocks() {
  return sizeof(T) == 4 ? 2 : 1;
}

// Persistent pairs: cluster p (CTAs 2p, 2p + 1) walks transforms p, p + P, ...
// Both ranks take the same transforms, so their barriers match; the first
// barrier makes sure the peer has started before its shared memory is
// written, the last of each transform that it has finished reading ours.
template <typename T, int N1, int L2, int... Rs>
__global__ void __cluster_dims__(2, 1, 1) __launch_bounds__(PairShape<N1, L2, Rs...>::NT, pair_min_blocks<T>())
    k_blue4_pair(const __grid_constant__ TileArgs<T> a) {
  pdl_entry();
  extern __shared__ __align__(16) unsigned char smraw[];
  cpx<T> *own = reinterpret_cast<cpx<T> *>(smraw);
  uint32_t c, peer_adr;
  asm volatile("mov.u32 %0, %%cluster_ctarank;" : "=r"(c));
  asm volatile("mapa.shared::cluster.u32 %0, %1, %2;"
               : "=r"(peer_adr)
               : "r"((uint32_t)__cvta_generic_to_shared(own)), "r"(c ^ 1u));
  const PeerRows<T> peer{(uintptr_t)peer_adr};
  const long long npairs = gridDim.x / 2;
  cluster_barrier();
  for (long long by = blockIdx.x / 2; by < a.nbatch; by += npairs) {
    const long long nx = by + npairs;
    if (c == 0 && threadIdx.x == 0 && nx < a.nbatch) prefetch_input(a, nx);
    pair_cols_in<T, N1, L2, rows::DevT, Rs...>(a, by, (int)c, own, peer, rows::DevT{});
    cluster_barrier();
    pair_rows<T, N1, L2, rows::DevT, Rs...>(a, (int)c, own, rows::DevT{});
    cluster_barrier();
    pair_cols_out<T, N1, L2, rows::DevT, Rs...>(a, by, (int)c, own, peer, rows::DevT{});
    cluster_barrier();
  }
}

template <typename T, int N1, int L2>
constexpr size_t smem_of() {
  return (size_t)N1 * slot_len<L2>() * sizeof(cpx<T>);
}

#ifndef FFB_HOST_EMULATION
template <typename T, int N1, int L2, int... Rs>
cudaError_t launch(const TileArgs<T> &a, cudaStream_t s) {
  {
    cudaError_t e = set_smem_limit_once<k_blue4<T, N1, L2, Rs...>>((int)smem_of<T, N1, L2>());
    if (e != cudaSuccess) return e;
  }
  int dev = 0, sms = 148;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  const long long grid = std::min<long long>(a.nbatch, sms);
  return launch_pdl(k_blue4<T, N1, L2, Rs...>, dim3((unsigned)grid), dim3(Shape<N1, L2, Rs...>::NT), smem_of<T, N1, L2>(), s, a);
}

// Pairs resident at once on the current device (cudaOccupancyMaxActiveClusters
// for this kernel and its shared memory), looked up once per device.
template <typename T, int N1, int L2, int... Rs>
cudaError_t resident_pairs(int *pairs) {
  static std::atomic<int> cached[64];
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev >= 0 && dev < 64 && (*pairs = cached[dev].load(std::memory_order_relaxed)) > 0) return cudaSuccess;
  cudaLaunchConfig_t cfg = {};
  int sms = 148;
  cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  cfg.gridDim = dim3((unsigned)(2 * sms));
  cfg.blockDim = dim3(PairShape<N1, L2, Rs...>::NT);
  cfg.dynamicSmemBytes = smem_of<T, N1 / 2, L2>();
  int n = 0;
  e = cudaOccupancyMaxActiveClusters(&n, k_blue4_pair<T, N1, L2, Rs...>, &cfg);
  if (e != cudaSuccess) return e;
  if (n <= 0) return cudaErrorInvalidConfiguration;
  if (dev >= 0 && dev < 64) cached[dev].store(n, std::memory_order_relaxed);
  *pairs = n;
  return cudaSuccess;
}

template <typename T, int N1, int L2, int... Rs>
cudaError_t launch_pair(const TileArgs<T> &a, cudaStream_t s) {
  static_assert(N1 % 2 == 0, "the pair splits the rows in halves");
  {
    cudaError_t e = set_smem_limit_once<k_blue4_pair<T, N1, L2, Rs...>>((int)smem_of<T, N1 / 2, L2>());
    if (e != cudaSuccess) return e;
  }
  int pairs = 0;
  cudaError_t e = resident_pairs<T, N1, L2, Rs...>(&pairs);
  if (e != cudaSuccess) return e;
  const long long np = std::min<long long>(a.nbatch, pairs);
  return launch_pdl(k_blue4_pair<T, N1, L2, Rs...>, dim3((unsigned)(2 * np)), dim3(PairShape<N1, L2, Rs...>::NT),
                    smem_of<T, N1 / 2, L2>(), s, a);
}
#else
template <typename T, int N1, int L2, int... Rs>
cudaError_t launch(const TileArgs<T> &a, cudaStream_t) {
  std::vector<unsigned char> buf(smem_of<T, N1, L2>() + 64);
  cpx<T> *sm = reinterpret_cast<cpx<T> *>(buf.data());
  for (long long by = 0; by < a.nbatch; ++by) {
    std::memset(buf.data(), 0xff, buf.size());
    blue4_body<T, N1, L2, rows::HostT, Rs...>(a, by, sm, rows::HostT{});
  }
  return cudaSuccess;
}

// The pair's two CTAs emulated phase by phase (each phase of rank 0, then
// of rank 1, between the cluster barriers).
template <typename T, int N1, int L2, int... Rs>
cudaError_t launch_pair(const TileArgs<T> &a, cudaStream_t) {
  const size_t bytes = smem_of<T, N1 / 2, L2>() + 64;
  std::vector<unsigned char> b0(bytes), b1(bytes);
  cpx<T> *sm[2] = {reinterpret_cast<cpx<T> *>(b0.data()), reinterpret_cast<cpx<T> *>(b1.data())};
  for (long long by = 0; by < a.nbatch; ++by) {
    std::memset(b0.data(), 0xff, bytes);
    std::memset(b1.data(), 0xff, bytes);
    for (int c = 0; c < 2; ++c)
      pair_cols_in<T, N1, L2, rows::HostT, Rs...>(a, by, c, sm[c], PeerRows<T>{(uintptr_t)sm[c ^ 1]}, rows::HostT{});
    for (int c = 0; c < 2; ++c) pair_rows<T, N1, L2, rows::HostT, Rs...>(a, c, sm[c], rows::HostT{});
    for (int c = 0; c < 2; ++c)
      pair_cols_out<T, N1, L2, rows::HostT, Rs...>(a, by, c, sm[c], PeerRows<T>{(uintptr_t)sm[c ^ 1]}, rows::HostT{});
  }
  return cudaSuccess;
}
#endif

}  // namespace blue4
}  // namespace ffb
