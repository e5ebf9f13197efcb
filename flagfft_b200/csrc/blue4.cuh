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
  static FFB_HD void write(const TileArgs<T> &a, cpx<T> *sm, int grp, int tid, const Regs &st) {
    const int w = grp * Sh::NR + tid / Sh::TPT, t = tid % Sh::TPT;
    if (w >= N1) return;
    if constexpr (S == nst - 1) {
      rows::stage_write<T, L2, Sh::TPT, Ns, R>(t, st, SmemKernIO<T>{sm + w * Sh::slot, a.kern + w * a.kern_stride});
    } else {
      rows::stage_write<T, L2, Sh::TPT, Ns, R>(t, st, SmemIO<T>{sm + w * Sh::slot});
    }
  }
};

// (host emulation instantiates it with per-thread state vectors)
#pragma nv_exec_check_disable
template <typename T, int N1, int L2, class Q, class Sh, int K, class X, class St>
FFB_HD void row_pipe(const X &x, const TileArgs<T> &a, cpx<T> *sm, const St &st) {
  static_assert(Sh::NG == 2, "the pipeline runs two row groups");
  constexpr int P = K - 1;  // the step whose reads st holds
  using Prev = RowStage<T, N1, L2, Q, Sh, P / 2>;
  if constexpr (K == 4 * Q::n) {
    x.last(Sh::NT, [&](int tid, const typename Prev::Regs &s) FFB_INL { Prev::write(a, sm, P % 2, tid, s); }, st);
  } else {
    using Cur = RowStage<T, N1, L2, Q, Sh, K / 2>;
    auto nxt = x.step(
        Sh::NT,
        [&](int tid, const typename Prev::Regs &s) FFB_INL {
          Prev::write(a, sm, P % 2, tid, s);
          return Cur::read(a, sm, K % 2, tid);
        },
        st);
    row_pipe<T, N1, L2, Q, Sh, K + 1>(x, a, sm, nxt);
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
  const int n = a.n;
  const cpx<T> *in = reinterpret_cast<const cpx<T> *>(a.in) + by * a.ib;
  cpx<T> *out = reinterpret_cast<cpx<T> *>(a.out) + by * a.ob;

  // 1. chirp, column DFT over j1, W_M^{k1 j2}, into row k1
  x.each(Sh::NT, [&](int tid) FFB_INL {
#pragma unroll 1
    for (int j2 = tid; j2 < L2; j2 += Sh::NT) {
      cpx<T> v[N1];
#pragma unroll
      for (int j1 = 0; j1 < N1; ++j1) {
        const int i = j1 * L2 + j2;
        v[j1] = i < n ? cmul(rows::ld_stream(in + i), ldg_c(a.chirp + i)) : mk((T)0, (T)0);
      }
      dft_fixed<N1, false, T>(v);
      if (j2) {
#pragma unroll
        for (int k1 = 1; k1 < N1; ++k1) v[k1] = cmul(v[k1], split_twiddle(a, (uint32_t)(k1 * j2)));
      }
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
    row_pipe<T, N1, L2, Q, Sh, 1>(x, a, sm, st);
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
      if (j2) {
#pragma unroll
        for (int k1 = 1; k1 < N1; ++k1) v[k1] = cmul(v[k1], conjg(split_twiddle(a, (uint32_t)(k1 * j2))));
      }
      dft_fixed<N1, true, T>(v);
#pragma unroll
      for (int j1 = 0; j1 < N1; ++j1) {
        const int i = j1 * L2 + j2;
        if (i < n) out[i] = cmul(v[j1], ldg_c(a.chirp + i));
      }
    }
  });
}

template <typename T, int N1, int L2, int... Rs>
__global__ void __launch_bounds__(Shape<N1, L2, Rs...>::NT) k_blue4(const __grid_constant__ TileArgs<T> a) {
  pdl_entry();
  extern __shared__ __align__(16) unsigned char smraw[];
  for (long long by = blockIdx.x; by < a.nbatch; by += gridDim.x) {
    const long long nx = by + gridDim.x;
    if (threadIdx.x == 0 && nx < a.nbatch) {
      // the next transform's input into L2 while this one computes
      const char *row = reinterpret_cast<const char *>(reinterpret_cast<const cpx<T> *>(a.in) + nx * a.ib);
      const uintptr_t b0 = (reinterpret_cast<uintptr_t>(row) + 15) & ~(uintptr_t)15;
      const uintptr_t b1 = (reinterpret_cast<uintptr_t>(row) + (size_t)a.n * sizeof(cpx<T>)) & ~(uintptr_t)15;
      if (b1 > b0)
        asm volatile("cp.async.bulk.prefetch.L2.global [%0], %1;" ::"l"(b0), "r"((uint32_t)(b1 - b0)) : "memory");
    }
    blue4_body<T, N1, L2, rows::DevT, Rs...>(a, by, reinterpret_cast<cpx<T> *>(smraw), rows::DevT{});
    __syncthreads();  // the next transform's first phase rewrites the rows
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
#endif

}  // namespace blue4
}  // namespace ffb
