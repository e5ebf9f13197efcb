// Host-visible kernel interface of the on-chip FFT passes (kernels.cu).
#pragma once

#include <cuda_runtime.h>

#include <cstdint>

#include "engine.cuh"

namespace ffb {

// What one CTA-resident transform computes.
enum class CoreKind : int {
  Dit = 0,        // plain C2C: digit-reversed load, DIT stages, natural store
  Bluestein = 1,  // chirp * x zero-padded -> DIF fwd -> x kernel -> DIT inv -> x chirp
  Rader = 2,      // permuted load -> DIF fwd -> x kernel -> DIT inv -> permuted store + x0
  Conv = 3,       // DIF fwd -> x kernel (per transform: kern + g * kern_stride) -> DIT inv
};

// How the pass reads its input and writes its output.
enum class IoKind : int {
  C2C = 0,  // complex in, complex out
  R2C = 1,  // real in (n = 2L reals packed as L complex), half spectrum out (L+1 bins)
  C2R = 2,  // half spectrum in (L+1 bins), real out (2L reals)
  R2CFull = 3,  // real in, complex core of length n (imag 0), first n/2+1 bins out
  C2RFull = 4,  // half spectrum in, Hermitian-expanded core of length n, real part out
  PackC2C = 5,    // real pairs in (z_i = in[i*ii] + i in[i*ii + 1]), complex out
  C2CUnpack = 6,  // complex in, real pairs out (out[k*ok] = Re z_k, out[k*ok + 1] = Im z_k)
};

// One pass = nbatch x G independent transforms, W of them per CTA.
// Transform g of outer batch b reads element i at  in + b*ib + g*ig + i*ii
// and writes element k at                          out + b*ob + g*og + k*ok
// (units: elements of the pass's input / output type).
// The compile-time radix sequences with their own kernels: radix-16 chains
// of the power-of-two lengths 128..16384 (one smaller radix last), 1536 =
// 16 * 16 * 6, and the mixed-radix 1701 = 9 * 9 * 7 * 3.  The executor runs a length that has one
// on it (and prefers such lengths for convolutions).
#define FFB_FIXED_SEQUENCES(X)        \
  X(1701, 9, 9, 7, 3)                 \
  X(128, 16, 8)                       \
  X(256, 16, 16)                      \
  X(512, 16, 16, 2)                   \
  X(1024, 16, 16, 4)                  \
  X(1536, 16, 16, 6)                  \
  X(2048, 16, 16, 8)                  \
  X(4096, 16, 16, 16)                 \
  X(8192, 16, 16, 16, 2)              \
  X(16384, 16, 16, 16, 4)

// Shapes (N1 rows of an L2-point compile-time sequence) of the one-pass
// four-step Bluestein kernel (blue4.cuh), single precision: the N1 padded
// rows fit one CTA's shared memory.
#define FFB_BLUE4_SHAPES(X)                                                                              \
  X(8, 2048, 16, 16, 8) X(9, 2048, 16, 16, 8) X(10, 2048, 16, 16, 8) X(11, 2048, 16, 16, 8)              \
  X(12, 2048, 16, 16, 8) X(13, 2048, 16, 16, 8) X(13, 1024, 16, 16, 4) X(15, 1024, 16, 16, 4)            \
  X(16, 1024, 16, 16, 4)

// Shapes of the pair form (blue4.cuh k_blue4_pair): N1 even, N1 / 2 padded
// rows per CTA (double precision: 139-209 KB).
#define FFB_BLUE4_PAIR_SHAPES(X) X(8, 2048, 16, 16, 8) X(10, 2048, 16, 16, 8) X(12, 2048, 16, 16, 8)

inline bool blue4_pair_shape(int n1, int L2) {
#define FFB_B4P_HAS(N1, L2_, ...) \
  if (n1 == (N1) && L2 == (L2_)) return true;
  FFB_BLUE4_PAIR_SHAPES(FFB_B4P_HAS)
#undef FFB_B4P_HAS
  return false;
}

inline bool blue4_shape(int n1, int L2) {
#define FFB_B4_HAS(N1, L2_, ...) \
  if (n1 == (N1) && L2 == (L2_)) return true;
  FFB_BLUE4_SHAPES(FFB_B4_HAS)
#undef FFB_B4_HAS
  return false;
}

template <typename T>
struct TileArgs {
  const void *in;
  void *out;
  long long nbatch;
  long long ib, ig, ii;
  long long ob, og, ok;
  int G;
  int W;
  int tpt;    // threads per transform
  int wfast;  // 1: consecutive threads take consecutive transforms (strided tiles)
  int inv;    // direction of a Dit core
  int n;      // logical length: Bluestein n, Rader p, real-transform n; else core.L
  Core core;   // Dit stages, or the forward DIF stages of a convolution
  Core core2;  // inverse DIT stages of a convolution (radices reversed)
  const cpx<T> *tw;     // per-stage twiddle blocks of core (Core::twoff)
  const cpx<T> *tw2;    // per-stage twiddle blocks of core2
  const cpx<T> *chirp;  // Bluestein chirp, n entries (direction folded in)
  const cpx<T> *kern;   // convolution kernel spectrum / L, in DIF position order
  const int *perm_in;   // Rader: q -> g^-q mod p
  const int *perm_out;  // Rader: q -> g^q mod p
  const cpx<T> *rtw;    // real-transform twiddles W_n^k, k <= n/2 (IoKind R2C / C2R)
  // optional post-twiddle of a four-step column pass: output k of transform g
  // is multiplied by W_N^{g*k} = hi[m / split] * lo[m % split], m = g*k < N
  int post_twiddle;
  const cpx<T> *ptw_lo;
  const cpx<T> *ptw_hi;
  FastDiv ptw_div;
  FastDiv ldiv;  // / core.L
  FastDiv wdiv;  // / W
  FastDiv ndiv;  // / n
  FastDiv hdiv;  // / (n / 2)
  // Bluestein chirp on a Dit core's load (chirp_mode 1) or store (2): element
  // e of transform g is logical index j = e*cj_e + g*cj_g, live while j < n.
  int chirp_mode;
  long long cj_e, cj_g;
  // Conv cores: transform g multiplies by kern + g * kern_stride.
  long long kern_stride;
  // 1: Stockham ping-pong path (C2C passes whose two buffers fit; convolution
  // kernels then in natural order).  0: in-place DIT/DIF path.
  int pp;
  // 1: register column pass -- one thread per transform, the whole transform
  // one codelet in registers, no shared memory (Dit core with one stage,
  // C2C, transforms contiguous in memory on both sides: ig == og == 1).
  int regcol;
  // > 0: one-pass four-step Bluestein (blue4.cuh) with this many columns
  // (rows of the core's sequence); one CTA per transform, or with blue_pair
  // a cluster of two CTAs holding half of the rows each.
  int blue_cols;
  int blue_pair;
  // 1: strided tile kernel of a compile-time sequence (tiles.cuh): W is its
  // fixed tile width, one shared buffer per transform.
  int tiles;
  // 1: a ping-pong pass only a row kernel can run (its one buffer per row
  // fits shared memory, two do not); never a general ping-pong tile.
  int rows_only;
  // 1: a strided pass of a TMA column sequence (tcols.cuh) runs on the
  // persistent TMA kernel when its buffers meet the copy rules (else on the
  // configuration above); its threads and shared memory per CTA.
  int tcols;
  int tc_threads;
  int tc_smem;
};

// Shared memory the general ping-pong tile body needs for a pass's W
// transforms (two buffers and three spare elements per transform).
template <typename T>
inline size_t pp_tile_smem(const TileArgs<T> &a) {
  return (size_t)a.W * (2 * (size_t)pp_size(a.core.L) + 3) * sizeof(cpx<T>);
}

// Real-transform pre/post processing between the passes of a multi-pass
// R2C / C2R (L = n/2 complex points per transform, rtw[k] = W_n^k, k <= L):
//   post: X_k = (Z_k + conj Z_{L-k})/2 - i W_n^k (Z_k - conj Z_{L-k})/2, k = 0..L
//         (in place allowed: z and x may alias with zdist == xdist)
//   pre:  Z_k = (X_k + conj X_{L-k}) + i W_n^-k (X_k - conj X_{L-k}), k < L,
//         Im X_0 and Im X_L ignored
// Elementwise conversions around a full-length complex transform of a real
// signal (any n, batch rows):
//   mode 0 widen:  z[k] = x[k] + 0i, k < n           (x real, row dist xd; z complex, zd)
//   mode 1 half:   y[k] = z[k], k <= n/2             (complex -> complex)
//   mode 2 expand: z[k] = X[k] (k <= n/2), conj X[n-k] (k > n/2), Im X[0] and, for
//                  even n, Im X[n/2] taken as 0       (complex half -> complex full)
//   mode 3 real:   y[k] = Re z[k], k < n            (complex -> real)
template <typename T>
cudaError_t launch_real_convert(int mode, const void *src, void *dst, long long batch, long long sdist,
                                long long ddist, long long n, cudaStream_t stream);

// Four-step twiddle W_N^m from two split tables (m < N): W_N^m =
// hi[m / split] * lo[m % split], conjugated for the inverse.
template <typename T>
struct SplitTw {
  const cpx<T> *lo = nullptr;
  const cpx<T> *hi = nullptr;
  FastDiv split{};
  bool inv = false;
};

// Batched out-of-place transpose of complex matrices: in (batch, R, C)
// row-major -> out (batch, C, R), matrix b of the input at b * sdist and of
// the output at b * ddist (0: R * C), through 32 x 32 shared-memory tiles
// (both sides coalesced); with tw.lo, element (r, c) is multiplied by
// W_N^{r c} on the way.  Used by the lowerings that exchange axes between
// passes (2-D transforms with an axis too long for one CTA, the plan tree's
// four-step over a multi-pass child).
template <typename T>
cudaError_t launch_transpose(const cpx<T> *in, cpx<T> *out, long long batch, long long R, long long C,
                             cudaStream_t stream, long long sdist = 0, long long ddist = 0,
                             const SplitTw<T> &tw = SplitTw<T>{});

// The elementwise steps of a Rader chain over a multi-pass length-m
// (m = p - 1) transform (src/exec/raw_nodes.cpp:252-305): rows of p inputs
// x (distance xdist), the working rows w of m elements (distance m) and,
// after them, x_0 and A_0 per row (ws + batch * m: 2 * batch elements):
//   mode 0 prepare:   w[q] = x[perm_in[q]], x0 saved;
//   mode 1 pointwise: A_0 = w[0] saved; w[q] = conj(w[q] * kern[q])
//                     (kern = FFT_m(b) / m);
//   mode 2 finalize:  y[perm_out[q]] = x_0 + conj(w[q]); y[0] = x_0 + A_0
//                     (rows of p outputs, distance ydist).
template <typename T>
cudaError_t launch_rader_step(int mode, const cpx<T> *x, cpx<T> *ws, cpx<T> *y, long long batch, long long p,
                              long long xdist, long long ydist, const int *perm, const cpx<T> *kern,
                              cudaStream_t stream);

// Real-transform twiddles W_n^k, k <= n/2, as two short tables:
// W_n^k = hi[k / split] * lo[k % split] (lo: split entries, hi: n/2/split + 1),
// so a long transform's twiddles stay cache resident instead of streaming an
// n/2-entry table beside the data.
template <typename T>
struct RealTw {
  const cpx<T> *lo;
  const cpx<T> *hi;
  FastDiv split;
};
template <typename T>
FFB_HD cpx<T> real_tw(const RealTw<T> &t, uint32_t k) {
  const uint32_t q = fdiv(k, t.split);
  return cmul(ldg_c(t.hi + q), ldg_c(t.lo + (k - q * t.split.d)));
}

template <typename T>
cudaError_t launch_real_post(const cpx<T> *z, cpx<T> *x, long long batch, long long zdist, long long xdist, int L,
                             const RealTw<T> &rtw, cudaStream_t stream);
template <typename T>
cudaError_t launch_real_pre(const cpx<T> *x, cpx<T> *z, long long batch, long long xdist, long long zdist, int L,
                            const RealTw<T> &rtw, cudaStream_t stream);

template <typename T>
cudaError_t launch_tile(const TileArgs<T> &a, CoreKind kind, IoKind io, size_t smem_bytes, cudaStream_t stream);
// Dynamic shared memory the launch of a tile pass uses (the row kernels of
// the compile-time sequences take less than the pass's general figure).
template <typename T>
size_t tile_smem(const TileArgs<T> &a, CoreKind kind, IoKind io, size_t smem_bytes);

// Strided tile kernels of the compile-time sequences (TileArgs::tiles);
// defined in k_f32_tiles.cu / k_f64_tiles.cu.  tiles_shape gives the tile
// width, threads and shared memory for a sequence length (false: none).
template <typename T>
cudaError_t launch_tiles(const TileArgs<T> &a, cudaStream_t stream);
template <typename T>
bool tiles_shape(int L, int *W, int *threads, size_t *smem);

// TMA column passes (TileArgs::tcols); defined in k_f32_tcols.cu /
// k_f64_tcols.cu.  launch_tcols returns cudaErrorNotSupported when the
// pass's buffers break the copy rules; tcols_eligible says at plan time
// whether a pass of length L with these strides can take it (threads and
// shared memory per CTA); tcols_wait_failures counts the kernel's bounded
// waits that gave up on this device (-1: unreadable).
template <typename T>
cudaError_t launch_tcols(const TileArgs<T> &a, cudaStream_t stream);
template <typename T>
bool tcols_eligible(int L, long long nbatch, long long G, long long ib, long long ig, long long ii, long long ob,
                    long long og, long long ok, int *threads, size_t *smem);
template <typename T>
long long tcols_wait_failures();

// One-pass four-step Bluestein (TileArgs::blue_cols, blue_pair); defined in
// k_f32_blue4.cu and k_f64_blue4.cu.
template <typename T>
cudaError_t launch_blue4(const TileArgs<T> &a, cudaStream_t stream);
// Its dynamic shared memory and threads per CTA (pair: per CTA of the pair).
size_t blue4_smem(int n1, int L2, size_t elem_bytes, bool pair);
int blue4_threads(int n1, int L2, bool pair);

// Register column pass (TileArgs::regcol); defined in regcol.cu.
template <typename T>
cudaError_t launch_regcol(const TileArgs<T> &a, cudaStream_t stream);
// Codelet lengths the register column pass has kernels for.
inline bool regcol_supports(int L) {
  switch (L) {
    case 2: case 3: case 4: case 5: case 6: case 7: case 8: case 9: case 10:
    case 11: case 12: case 13: case 15: case 16: case 17: case 19:
      return true;
    default:
      return false;
  }
}

// Shared memory one transform of the pass occupies (bytes).
template <typename T>
inline size_t tile_smem_per_transform(int core_len) {
  return (size_t)Swz<T>::padded(core_len) * sizeof(cpx<T>);
}

}  // namespace ffb
