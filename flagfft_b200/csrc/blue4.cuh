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
// two groups so that only half of the convolution is in registers at a time.
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
// rows processed in groups of NR (two groups), NT threads in all.
template <int N1, int L2, int... Rs>
struct Shape {
  static constexpr int TPT = tpt_of(L2, Seq<Rs...>::rmax());
  static constexpr int NR = (N1 + 1) / 2;
  static constexpr int NG = (N1 + NR - 1) / NR;
  static constexpr int NT = NR * TPT;
  static constexpr int slot = slot_len<L2>();
};

// Stage S.. of the row FFTs of all N1 rows in direction INV; KERN: the last
// stage multiplies by the kernel spectrum row before its writes.
template <typename T, bool INV, bool KERN, int N1, int L2, class Q, int S, class Sh, class X>
FFB_HD void row_chain(const X &x, const cpx<T> *__restrict__ tw, cpx<T> *sm, const cpx<T> *kern,
                      long long kstride) {
  if constexpr (S < Q::n) {
    constexpr int R = Q::r(S), Ns = Q::span(S), TwOff = Q::twoff(S);
    constexpr bool last = S == Q::n - 1;
#pragma unroll 1
    for (int grp = 0; grp < Sh::NG; ++grp) {
      auto rd = [&](int tid) FFB_INL {
        const int wr_ = grp * Sh::NR + tid / Sh::TPT, t = tid % Sh::TPT;
        const int w = wr_ < N1 ? wr_ : N1 - 1;  // threads past the last row read a live row, write nothing
        return rows::stage_read<T, INV, L2, Sh::TPT, Ns, R>(t, tw + TwOff, SmemIO<T>{sm + w * Sh::slot});
      };
      auto wr = [&](int tid, const rows::StageRegs<T, L2, Sh::TPT, R> &st) FFB_INL {
        const int w = grp * Sh::NR + tid / Sh::TPT, t = tid % Sh::TPT;
        if (w >= N1) return;
        if constexpr (KERN && last) {
          rows::stage_write<T, L2, Sh::TPT, Ns, R>(t, st, SmemKernIO<T>{sm + w * Sh::slot, kern + w * kstride});
        } else {
          rows::stage_write<T, L2, Sh::TPT, Ns, R>(t, st, SmemIO<T>{sm + w * Sh::slot});
        }
      };
      // reads of this group, barrier, writes of this group (the next group's
      // reads touch other rows, so they follow without a barrier)
      x.each2(Sh::NT, rd, wr);
    }
    x.sync();
    row_chain<T, INV, KERN, N1, L2, Q, S + 1, Sh>(x, tw, sm, kern, kstride);
  }
}

// One transform (batch index by) of the one-pass chain.  TileArgs: core /
// core2 the row sequence with tables tw / tw2, kern the N1 x L2 kernel
// spectrum rows (kern_stride = L2), chirp the n-point chirp, ptw_* the split
// W_M tables, n the logical length, ib / ob the transform distances.
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
  row_chain<T, false, true, N1, L2, Q, 0, Sh>(x, a.tw, sm, a.kern, a.kern_stride);
  row_chain<T, true, false, N1, L2, Q, 0, Sh>(x, a.tw2, sm, nullptr, 0);

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
  extern __shared__ __align__(16) unsigned char smraw[];
  blue4_body<T, N1, L2, rows::DevT, Rs...>(a, (long long)blockIdx.x, reinterpret_cast<cpx<T> *>(smraw), rows::DevT{});
}

template <typename T, int N1, int L2>
constexpr size_t smem_of() {
  return (size_t)N1 * slot_len<L2>() * sizeof(cpx<T>);
}

#ifndef FFB_HOST_EMULATION
template <typename T, int N1, int L2, int... Rs>
cudaError_t launch(const TileArgs<T> &a, cudaStream_t s) {
  static bool configured = false;
  if (!configured) {
    cudaError_t e = cudaFuncSetAttribute(k_blue4<T, N1, L2, Rs...>, cudaFuncAttributeMaxDynamicSharedMemorySize,
                                         (int)smem_of<T, N1, L2>());
    if (e != cudaSuccess) return e;
    configured = true;
  }
  k_blue4<T, N1, L2, Rs...><<<dim3((unsigned)a.nbatch), dim3(Shape<N1, L2, Rs...>::NT), smem_of<T, N1, L2>(), s>>>(a);
  return cudaGetLastError();
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
