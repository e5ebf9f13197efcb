// On-chip FFT engine for sm_100a: complex arithmetic, radix codelets, in-place
// mixed-radix decimation stages over a shared-memory buffer.
//
// Design (B200-first, not a port of the reference's Triton leaf):
//  * One transform of length L lives in one CTA's shared memory (up to 227 KB:
//    29056 complex64 / 14528 complex128 points).  Stages run in place; each
//    butterfly reads and writes the same R positions, so a stage needs no
//    second buffer and a thread holds one butterfly of a large radix, or a
//    group of up to 16 values of a small one, in registers at a time -- any L
//    that fits in shared memory runs at any thread count.
//  * DIT stages consume a digit-reversed buffer and leave natural order; DIF
//    stages consume natural order and leave it digit-reversed.  A DIF pass with
//    radices (R0..Rk) followed by a DIT pass with the radices reversed needs no
//    reordering in between: Bluestein and Rader convolutions multiply in that
//    permuted order with a pre-permuted kernel spectrum.
//  * Shared-memory positions are XOR-swizzled inside aligned 16-element
//    (complex64) / 8-element (complex128) groups so the stride-R accesses of
//    the early stages and the digit-reversed loads spread over the banks.
//  * Twiddles come from per-stage tables built on the host in extended
//    precision and rounded once (the reference also builds its stage twiddles
//    in double and casts, src/codegen/tables.cpp:39-69); the inverse direction
//    conjugates.
//  * Codelets are the forward DFT; the inverse is conj(DFT(conj x)), the same
//    convention the reference's codelets use (python/flagfft_codegen/kernels.py:493-512).
#pragma once

#include <cstdint>
#include <cuda_runtime.h>

#include "device_once.hpp"

// Every engine function is host+device: the host build runs the same code
// sequentially (one "thread", barriers as no-ops) to check index arithmetic
// without a GPU.
#define FFB_HD __host__ __device__ __forceinline__
// Lambdas in kernel bodies: always inlined, so shared-memory pointers keep
// their address space and no call frame appears.
#define FFB_INL __attribute__((always_inline))

namespace ffb {

#include "roots.inc"

// Programmatic dependent launch.  Every kernel starts with pdl_entry(): it
// lets the next kernel on the stream begin launching once all of this grid's
// CTAs run (launch_dependents), then waits for the previous kernel's
// completion and memory (wait) before it touches global memory.  Launched
// with the attribute, a kernel's CTAs thus take their SM slots while the
// previous kernel drains; launched without it, both instructions are no-ops.
FFB_HD void pdl_entry() {
#ifdef __CUDA_ARCH__
  asm volatile("griddepcontrol.launch_dependents;" ::: "memory");
  asm volatile("griddepcontrol.wait;" ::: "memory");
#endif
}

#ifndef FFB_HOST_EMULATION
// Whether launches from this thread carry the programmatic-serialization
// attribute: on unless FLAGFFT_PDL=0 (read once) or the thread turned it off
// (PdlOff).  Threads that feed several streams at once (the request server)
// turn it off: a dependent grid's CTAs take SM slots as soon as the previous
// grid's CTAs all run, and on a busy GPU those slots are what the other
// streams' kernels are waiting for.
bool pdl_enabled();
struct PdlOff {
  PdlOff();
  ~PdlOff();
  bool prev;
};

// Launches a kernel (one that begins with pdl_entry) with programmatic
// dependent launch on stream s (a plain launch when pdl_enabled() is false).
template <typename... KArgs, typename... Args>
inline cudaError_t launch_pdl(void (*kernel)(KArgs...), dim3 grid, dim3 block, size_t smem, cudaStream_t s,
                              Args &&...args) {
  cudaLaunchConfig_t cfg{};
  cfg.gridDim = grid;
  cfg.blockDim = block;
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute attr[1];
  attr[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  attr[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = attr;
  cfg.numAttrs = pdl_enabled() ? 1 : 0;
  return cudaLaunchKernelEx(&cfg, kernel, static_cast<KArgs>(args)...);
}

// Raises Kernel's dynamic shared-memory limit to `bytes` on the current
// device, once per device (the attribute belongs to the device).  One flag
// set per kernel instantiation: Kernel is a template argument, so kernels of
// the same signature keep separate flags.
template <auto Kernel>
inline cudaError_t set_smem_limit_once(int bytes) {
  static DeviceOnce once;
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (once.done(dev)) return cudaSuccess;
  e = cudaFuncSetAttribute(Kernel, cudaFuncAttributeMaxDynamicSharedMemorySize, bytes);
  if (e == cudaSuccess) once.mark(dev);
  return e;
}
#endif

template <typename T>
struct alignas(2 * sizeof(T)) cpx {
  T x, y;
};

template <typename T>
FFB_HD cpx<T> mk(T x, T y) {
  cpx<T> r;
  r.x = x;
  r.y = y;
  return r;
}
template <typename T>
FFB_HD cpx<T> operator+(cpx<T> a, cpx<T> b) { return mk(a.x + b.x, a.y + b.y); }
template <typename T>
FFB_HD cpx<T> operator-(cpx<T> a, cpx<T> b) { return mk(a.x - b.x, a.y - b.y); }
template <typename T>
FFB_HD cpx<T> cmul(cpx<T> a, cpx<T> b) {
  return mk(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
template <typename T>
FFB_HD cpx<T> cscale(cpx<T> a, T s) { return mk(a.x * s, a.y * s); }
template <typename T>
FFB_HD cpx<T> conjg(cpx<T> a) { return mk(a.x, -a.y); }
// multiply by -i
template <typename T>
FFB_HD cpx<T> mul_mi(cpx<T> a) { return mk(a.y, -a.x); }

// ---------------------------------------------------------------------------
// Division by a runtime divisor d (1 <= d < 2^31) for dividends n < 2^31
// (Granlund-Montgomery): l = ceil(log2 d), m = floor(2^32 (2^l - d) / d) + 1,
// n / d == (umulhi(n, m) + n) >> l.  n < 2^31 keeps the sum below 2^32.
// ---------------------------------------------------------------------------
struct FastDiv {
  uint32_t d, m, s;
};

inline FastDiv make_fastdiv(uint32_t d) {
  FastDiv f;
  f.d = d;
  uint32_t l = 0;
  while ((1ull << l) < d) ++l;
  f.s = l;
  f.m = (uint32_t)(((1ull << 32) * ((1ull << l) - d)) / d + 1);
  return f;
}

FFB_HD uint32_t fdiv(uint32_t n, const FastDiv &f) {
#ifdef __CUDA_ARCH__
  return (__umulhi(n, f.m) + n) >> f.s;
#else
  return (uint32_t)((((uint64_t)n * f.m >> 32) + n) >> f.s);
#endif
}

// ---------------------------------------------------------------------------
// Codelets: forward DFT of R values held in registers, natural order in/out.
// ---------------------------------------------------------------------------

// Multiply by the compile-time root W_R^m = exp(-2*pi*i*m/R), skipping the
// trivial ones.
template <int R, typename T>
FFB_HD cpx<T> twiddle_const(cpx<T> a, int m) {
  m %= R;
  if (m == 0) return a;
  if (2 * m == R) return mk(-a.x, -a.y);
  if (4 * m == R) return mul_mi(a);
  if (4 * m == 3 * R) return mk(-a.y, a.x);
  const T c = (T)RootTable<R>::c(m);
  const T s = (T)RootTable<R>::s(m);
  // exp(-i theta) = c - i s;  45-degree multiples need two multiplies
  if (RootTable<R>::c(m) == RootTable<R>::s(m)) return mk(c * (a.x + a.y), c * (a.y - a.x));
  if (RootTable<R>::c(m) == -RootTable<R>::s(m)) return mk(c * (a.x - a.y), c * (a.y + a.x));
  return mk(a.x * c + a.y * s, a.y * c - a.x * s);
}

template <int R, typename T>
struct Dft;

template <typename T>
struct Dft<1, T> {
  static FFB_HD void run(cpx<T> *) {}
};

template <typename T>
struct Dft<2, T> {
  static FFB_HD void run(cpx<T> *v) {
    cpx<T> a = v[0], b = v[1];
    v[0] = a + b;
    v[1] = a - b;
  }
};

template <typename T>
struct Dft<3, T> {
  static FFB_HD void run(cpx<T> *v) {
    const T c = (T)-0.5, s = (T)0.86602540378443864676;
    cpx<T> t1 = v[1] + v[2], t2 = v[1] - v[2];
    cpx<T> y0 = v[0] + t1;
    cpx<T> m1 = mk(v[0].x + c * t1.x, v[0].y + c * t1.y);
    // -i * s * t2
    cpx<T> m2 = mk(s * t2.y, -s * t2.x);
    v[0] = y0;
    v[1] = m1 + m2;
    v[2] = m1 - m2;
  }
};

template <typename T>
struct Dft<4, T> {
  static FFB_HD void run(cpx<T> *v) {
    cpx<T> a = v[0] + v[2], b = v[0] - v[2];
    cpx<T> c = v[1] + v[3], d = mul_mi(v[1] - v[3]);
    v[0] = a + c;
    v[2] = a - c;
    v[1] = b + d;
    v[3] = b - d;
  }
};

// Odd prime P: pair n with P-n.  y_k = x0 + sum_n a_n cos(2 pi n k/P)
//                                  - i sum_n b_n sin(2 pi n k/P),
// a_n = x_n + x_{P-n}, b_n = x_n - x_{P-n}; y_{P-k} flips the sine term.
template <int P, typename T>
struct DftPrime {
  static FFB_HD void run(cpx<T> *v) {
    constexpr int H = (P - 1) / 2;
    cpx<T> a[H], b[H];
#pragma unroll
    for (int n = 1; n <= H; ++n) {
      a[n - 1] = v[n] + v[P - n];
      b[n - 1] = v[n] - v[P - n];
    }
    const cpx<T> x0 = v[0];
    cpx<T> sum = x0;
#pragma unroll
    for (int n = 0; n < H; ++n) sum = sum + a[n];
    v[0] = sum;
#pragma unroll
    for (int k = 1; k <= H; ++k) {
      cpx<T> A = x0, B = mk((T)0, (T)0);
#pragma unroll
      for (int n = 1; n <= H; ++n) {
        const int m = (n * k) % P;
        const T c = (T)RootTable<P>::c(m);
        const T s = (T)RootTable<P>::s(m);
        A.x += a[n - 1].x * c;
        A.y += a[n - 1].y * c;
        B.x += b[n - 1].x * s;
        B.y += b[n - 1].y * s;
      }
      // -i*B = (B.y, -B.x)
      v[k] = mk(A.x + B.y, A.y - B.x);
      v[P - k] = mk(A.x - B.y, A.y + B.x);
    }
  }
};

template <typename T> struct Dft<5, T> : DftPrime<5, T> {};
template <typename T> struct Dft<7, T> : DftPrime<7, T> {};
template <typename T> struct Dft<11, T> : DftPrime<11, T> {};
template <typename T> struct Dft<13, T> : DftPrime<13, T> {};
template <typename T> struct Dft<17, T> : DftPrime<17, T> {};
template <typename T> struct Dft<19, T> : DftPrime<19, T> {};

// Composite R = R1 * R2 (Cooley-Tukey inside the codelet):
// X[k1 + R1 k2] = sum_n2 W_R2^{n2 k2} W_R^{n2 k1} sum_n1 x[R2 n1 + n2] W_R1^{n1 k1}
template <int R1, int R2, typename T>
struct DftSplit {
  static FFB_HD void run(cpx<T> *v) {
    constexpr int R = R1 * R2;
    cpx<T> u[R];
#pragma unroll
    for (int n2 = 0; n2 < R2; ++n2) {
      cpx<T> t[R1];
#pragma unroll
      for (int n1 = 0; n1 < R1; ++n1) t[n1] = v[R2 * n1 + n2];
      Dft<R1, T>::run(t);
#pragma unroll
      for (int k1 = 0; k1 < R1; ++k1) u[n2 * R1 + k1] = twiddle_const<R, T>(t[k1], n2 * k1);
    }
#pragma unroll
    for (int k1 = 0; k1 < R1; ++k1) {
      cpx<T> t[R2];
#pragma unroll
      for (int n2 = 0; n2 < R2; ++n2) t[n2] = u[n2 * R1 + k1];
      Dft<R2, T>::run(t);
#pragma unroll
      for (int k2 = 0; k2 < R2; ++k2) v[k1 + R1 * k2] = t[k2];
    }
  }
};

template <typename T> struct Dft<6, T> : DftSplit<2, 3, T> {};
template <typename T> struct Dft<8, T> : DftSplit<2, 4, T> {};
template <typename T> struct Dft<9, T> : DftSplit<3, 3, T> {};
template <typename T> struct Dft<10, T> : DftSplit<2, 5, T> {};
template <typename T> struct Dft<12, T> : DftSplit<4, 3, T> {};
template <typename T> struct Dft<15, T> : DftSplit<3, 5, T> {};
template <typename T> struct Dft<16, T> : DftSplit<4, 4, T> {};

template <int R, typename T>
FFB_HD void dft_dir(cpx<T> *v, bool inv) {
  if (inv) {
#pragma unroll
    for (int r = 0; r < R; ++r) v[r].y = -v[r].y;
  }
  Dft<R, T>::run(v);
  if (inv) {
#pragma unroll
    for (int r = 0; r < R; ++r) v[r].y = -v[r].y;
  }
}

// ---------------------------------------------------------------------------
// Shared-memory layout
// ---------------------------------------------------------------------------

// Swizzle inside aligned groups of G = 128 bytes / sizeof(cpx<T>) elements.
template <typename T>
struct Swz {
  static constexpr int G = 128 / (2 * (int)sizeof(T));  // 16 (c64) or 8 (c128)
  static constexpr int B = G == 16 ? 4 : 3;
  static FFB_HD int phys(int p) { return p ^ (((p >> B) ^ (p >> (2 * B))) & (G - 1)); }
  static FFB_HD int padded(int L) { return (L + G - 1) / G * G; }
};

constexpr int kMaxStages = 16;

// One on-chip transform of length L as a sequence of radix stages.
//   DIT stage s:  span[s] = R0*...*R(s-1)       (sub-transform length before it)
//   DIF stage s:  span[s] = L / (R0*...*R(s-1)) (sub-length it splits)
//   twoff[s] is the offset of stage s's twiddle block in the core's table:
//   R(s)-1 rows of `inner` entries (inner = span[s] for DIT and Stockham
//   stages, span[s]/R(s) for DIF); entry j of row r-1 is W_{inner R}^{r j},
//   conjugated in a table built for the inverse direction.  Neighbouring
//   butterflies read neighbouring entries of each row (one coalesced load per
//   row across a warp), and no twiddle needs a sign change at run time.
//   sdiv[s] divides the butterfly index by the inner block length
//   (DIT: span[s]; DIF: span[s]/R(s)).
//   rdiv[s] divides by R(s) (digit reversal).
struct Core {
  int L;
  int nst;
  int radix[kMaxStages];
  int span[kMaxStages];
  int twoff[kMaxStages];
  FastDiv sdiv[kMaxStages];
  FastDiv rdiv[kMaxStages];
};

// Position of input element i for a DIT pass over `c` (digit reversal):
// i = sum_s d_s * L/(R0..Rs)  ->  p = sum_s d_s * (R0..R(s-1)).
FFB_HD int dit_position(int i, const Core &c) {
  int p = 0;
  int rem = i;
  for (int s = c.nst - 1; s >= 0; --s) {
    int q = (int)fdiv((uint32_t)rem, c.rdiv[s]);
    int d = rem - q * c.radix[s];
    rem = q;
    p += d * c.span[s];
  }
  return p;
}

FFB_HD cpx<float> ldg_c(const cpx<float> *p) {
#ifdef __CUDA_ARCH__
  float2 v = __ldg(reinterpret_cast<const float2 *>(p));
  return mk(v.x, v.y);
#else
  return *p;
#endif
}
FFB_HD cpx<double> ldg_c(const cpx<double> *p) {
#ifdef __CUDA_ARCH__
  double2 v = __ldg(reinterpret_cast<const double2 *>(p));
  return mk(v.x, v.y);
#else
  return *p;
#endif
}
template <typename V>
FFB_HD V ldg_v(const V *p) {
#ifdef __CUDA_ARCH__
  return __ldg(p);
#else
  return *p;
#endif
}

// w[r-1] = blk[(r-1) * inner + j], r = 1..R-1: the R-1 twiddles of column j
// of a stage block.
template <int R, typename T>
FFB_HD void load_tw_col(const cpx<T> *__restrict__ blk, int inner, int j, cpx<T> *w) {
  const cpx<T> *p = blk + j;
#pragma unroll
  for (int r = 1; r < R; ++r) w[r - 1] = ldg_c(p + (r - 1) * inner);
}

// Codelet in a compile-time direction: the inverse is conj(DFT(conj x)); the
// conjugations fold into the codelet's additions.
template <int R, bool INV, typename T>
FFB_HD void dft_fixed(cpx<T> *v) {
  if constexpr (INV) {
#pragma unroll
    for (int r = 0; r < R; ++r) v[r].y = -v[r].y;
  }
  Dft<R, T>::run(v);
  if constexpr (INV) {
#pragma unroll
    for (int r = 0; r < R; ++r) v[r].y = -v[r].y;
  }
}

// In-place DIT stage s: combine R sub-transforms of length Ls.  The first
// stage (Ls == 1) has only unit twiddles and skips them.
template <int R, typename T>
FFB_HD void dit_stage_r(cpx<T> *buf, const Core &c, int s, int tid, int nthr,
                                            const cpx<T> *__restrict__ tw, bool inv) {
  const int Ls = c.span[s];
  const cpx<T> *blk = tw + c.twoff[s];
  const FastDiv sd = c.sdiv[s];
  const int nb = c.L / R;
  for (int u = tid; u < nb; u += nthr) {
    const int b = (int)fdiv((uint32_t)u, sd);
    const int j = u - b * Ls;
    const int base = b * Ls * R + j;
    cpx<T> v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = buf[Swz<T>::phys(base + r * Ls)];
    if (Ls > 1) {
      cpx<T> w[R - 1];
      load_tw_col<R, T>(blk, Ls, j, w);
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], w[r - 1]);
    }
    dft_dir<R, T>(v, inv);
#pragma unroll
    for (int q = 0; q < R; ++q) buf[Swz<T>::phys(base + q * Ls)] = v[q];
  }
}

// In-place DIF stage s: split sub-transforms of length Ms into R interleaved
// parts; outputs are multiplied by W_Ms^{q j} after the butterfly (none in
// the last stage, Ms == R).
template <int R, typename T>
FFB_HD void dif_stage_r(cpx<T> *buf, const Core &c, int s, int tid, int nthr,
                                            const cpx<T> *__restrict__ tw, bool inv) {
  const int Ms = c.span[s];
  const int stride = Ms / R;
  const cpx<T> *blk = tw + c.twoff[s];
  const FastDiv sd = c.sdiv[s];
  const int nb = c.L / R;
  for (int u = tid; u < nb; u += nthr) {
    const int b = (int)fdiv((uint32_t)u, sd);
    const int j = u - b * stride;
    const int base = b * Ms + j;
    cpx<T> v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = buf[Swz<T>::phys(base + r * stride)];
    dft_dir<R, T>(v, inv);
    if (stride > 1) {
      cpx<T> w[R - 1];
      load_tw_col<R, T>(blk, stride, j, w);
#pragma unroll
      for (int q = 1; q < R; ++q) v[q] = cmul(v[q], w[q - 1]);
    }
#pragma unroll
    for (int q = 0; q < R; ++q) buf[Swz<T>::phys(base + q * stride)] = v[q];
  }
}

#define FFB_RADIX_SWITCH(R_, CALL)                                     \
  switch (R_) {                                                        \
    case 2: CALL(2); break;                                            \
    case 3: CALL(3); break;                                            \
    case 4: CALL(4); break;                                            \
    case 5: CALL(5); break;                                            \
    case 6: CALL(6); break;                                            \
    case 7: CALL(7); break;                                            \
    case 8: CALL(8); break;                                            \
    case 9: CALL(9); break;                                            \
    case 10: CALL(10); break;                                          \
    case 11: CALL(11); break;                                          \
    case 12: CALL(12); break;                                          \
    case 13: CALL(13); break;                                          \
    case 15: CALL(15); break;                                          \
    case 16: CALL(16); break;                                          \
    case 17: CALL(17); break;                                          \
    case 19: CALL(19); break;                                          \
    default: break;                                                    \
  }

// All DIT stages (digit-reversed in, natural out).  Every thread of the
// group calls this; `sync` is the barrier that covers the group's threads.
template <typename T, typename Sync>
FFB_HD void run_dit(cpx<T> *buf, const Core &c, int tid, int nthr,
                                        const cpx<T> *__restrict__ tw, bool inv, Sync sync) {
  for (int s = 0; s < c.nst; ++s) {
#define FFB_DIT_CALL(R) dit_stage_r<R, T>(buf, c, s, tid, nthr, tw, inv)
    FFB_RADIX_SWITCH(c.radix[s], FFB_DIT_CALL)
#undef FFB_DIT_CALL
    sync();
  }
}

// All DIF stages (natural in, digit-reversed out).
template <typename T, typename Sync>
FFB_HD void run_dif(cpx<T> *buf, const Core &c, int tid, int nthr,
                                        const cpx<T> *__restrict__ tw, bool inv, Sync sync) {
  for (int s = 0; s < c.nst; ++s) {
#define FFB_DIF_CALL(R) dif_stage_r<R, T>(buf, c, s, tid, nthr, tw, inv)
    FFB_RADIX_SWITCH(c.radix[s], FFB_DIF_CALL)
#undef FFB_DIF_CALL
    sync();
  }
}

// ---------------------------------------------------------------------------
// Stockham autosort (out of place, natural order in and out).
//
// Stage s with radix R and Ns = R0*...*R(s-1): butterfly j (< L/R) reads
// elements j + r*L/R, multiplies input r by W_{Ns R}^{r (j mod Ns)}, and writes
// output q to (j - j mod Ns)*R + j mod Ns + q*Ns.  Stages ping-pong between two
// shared-memory buffers; reads are unit-stride across a warp.  Uses the DIT
// core's fields (span = Ns, twiddle block at twoff, sdiv = / Ns).
// ---------------------------------------------------------------------------

// Shared-memory position of element p in a ping-pong buffer: one pad element
// per 16 spreads the stride-R writes of the early stages over the banks.
FFB_HD constexpr int pp_pos(int p) { return p + (p >> 4); }
FFB_HD constexpr int pp_size(int L) { return ((L + (L >> 4) + 1) + 1) & ~1; }

template <int R, bool INV, typename T, class Src, class Dst>
FFB_HD void stockham_stage_r(const Core &c, int s, int tid, int nthr, const cpx<T> *__restrict__ tw,
                             const Src &src, const Dst &dst) {
  const int Ns = c.span[s], nb = c.L / R;
  const cpx<T> *blk = tw + c.twoff[s];
  const FastDiv sd = c.sdiv[s];
  for (int j = tid; j < nb; j += nthr) {
    const int g = (int)fdiv((uint32_t)j, sd);
    const int k = j - g * Ns;
    cpx<T> v[R];
#pragma unroll
    for (int r = 0; r < R; ++r) v[r] = src(j + r * nb);
    if (Ns > 1) {
      cpx<T> w[R - 1];
      load_tw_col<R, T>(blk, Ns, k, w);
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], w[r - 1]);
    }
    dft_fixed<R, INV, T>(v);
    const int base = g * Ns * R + k;
#pragma unroll
    for (int q = 0; q < R; ++q) dst(base + q * Ns, v[q]);
  }
}

// Shared-memory reader / writer of a ping-pong buffer.
template <typename T>
struct PPRead {
  const cpx<T> *b;
  FFB_HD cpx<T> operator()(int p) const { return b[pp_pos(p)]; }
};
template <typename T>
struct PPWrite {
  cpx<T> *b;
  FFB_HD void operator()(int p, cpx<T> v) const { b[pp_pos(p)] = v; }
};

// Flat loop over e = t0, t0 + nt, ... < total, U iterations at a time: the U
// values are all produced (their global loads issued back to back) before
// any is consumed, so a thread keeps U loads in flight instead of one.
template <int U, class V, class Produce, class Consume>
FFB_HD void chunked_loop(int t0, int nt, int total, Produce &&produce, Consume &&consume) {
  int base = t0;
  // whole chunks: no per-element bounds test
#pragma unroll 1
  for (; base + (U - 1) * nt < total; base += U * nt) {
    V v[U];
#pragma unroll
    for (int u = 0; u < U; ++u) v[u] = produce(base + u * nt);
#pragma unroll
    for (int u = 0; u < U; ++u) consume(base + u * nt, v[u]);
  }
  // the rest, one element at a time
#pragma unroll 1
  for (; base < total; base += nt) consume(base, produce(base));
}

// All stages of `c` shared -> shared in direction INV: stage s reads buffer
// (s even ? src : oth) and writes the other; every stage ends with a barrier.
// The result is in `src` when nst is even, in `oth` when odd.
template <typename T, bool INV, class Sync>
FFB_HD void run_stockham_smem(const Core &c, cpx<T> *src, cpx<T> *oth, int tid, int nthr,
                              const cpx<T> *__restrict__ tw, Sync sync) {
  for (int s = 0; s < c.nst; ++s) {
    const PPRead<T> rd{(s & 1) ? oth : src};
    const PPWrite<T> w{(s & 1) ? src : oth};
#define FFB_SS(R) stockham_stage_r<R, INV, T>(c, s, tid, nthr, tw, rd, w)
    FFB_RADIX_SWITCH(c.radix[s], FFB_SS)
#undef FFB_SS
    sync();
  }
}

// Stage runner of a ping-pong pass: the runtime radix sequence of a Core.
template <typename T>
struct GenericStages {
  template <bool INV, class Sync>
  FFB_HD void run(const Core &c, cpx<T> *src, cpx<T> *oth, int tid, int nthr, const cpx<T> *__restrict__ tw,
                  Sync sync) const {
    run_stockham_smem<T, INV>(c, src, oth, tid, nthr, tw, sync);
  }
};

// ---------------------------------------------------------------------------
// Stockham stages with the radix sequence fixed at compile time (radix-16
// chains of power-of-two lengths).  With L, Ns and R constants, j mod Ns is a
// mask, the twiddle rows sit at constant strides, and the padded positions
// p + p/16 of a butterfly's R reads (and R writes) are one base plus constant
// offsets whenever the stride between them is a multiple of 16 (or the
// butterfly's outputs are R consecutive positions inside one 16-block): two
// address computations per butterfly instead of 2R.
// ---------------------------------------------------------------------------
template <typename T, bool INV, int L, int Ns, int R>
FFB_HD void fixed_stage(const cpx<T> *src, cpx<T> *dst, int tid, int nthr, const cpx<T> *__restrict__ tw) {
  constexpr int nb = L / R;
  for (int j = tid; j < nb; j += nthr) {
    const int k = Ns == 1 ? 0 : j % Ns;
    cpx<T> v[R];
    if constexpr (nb % 16 == 0) {
      const cpx<T> *rp = src + pp_pos(j);
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = rp[r * (nb + nb / 16)];
    } else {
#pragma unroll
      for (int r = 0; r < R; ++r) v[r] = src[pp_pos(j + r * nb)];
    }
    if constexpr (Ns > 1) {
      const cpx<T> *row = tw + k;  // row r-1 of the stage block at (r-1) * Ns
#pragma unroll
      for (int r = 1; r < R; ++r) v[r] = cmul(v[r], ldg_c(row + (r - 1) * Ns));
    }
    dft_fixed<R, INV, T>(v);
    const int base = (j - k) * R + k;
    if constexpr (Ns % 16 == 0) {
      cpx<T> *wp = dst + pp_pos(base);
#pragma unroll
      for (int q = 0; q < R; ++q) wp[q * (Ns + Ns / 16)] = v[q];
    } else if constexpr (Ns == 1 && 16 % R == 0) {
      cpx<T> *wp = dst + pp_pos(base);  // R consecutive positions inside one 16-block
#pragma unroll
      for (int q = 0; q < R; ++q) wp[q] = v[q];
    } else {
#pragma unroll
      for (int q = 0; q < R; ++q) dst[pp_pos(base + q * Ns)] = v[q];
    }
  }
}

// Stages Ns, Ns*R0, ... of a length-L transform: stage reads `src`, writes
// `oth`, then the two swap; `twoff` is the stage's block in the core's table.
template <typename T, bool INV, int L, int Ns, int TwOff, int... Rs>
struct FixedStages {
  template <class Sync>
  static FFB_HD void run(cpx<T> *, cpx<T> *, int, int, const cpx<T> *__restrict__, Sync) {}
};
template <typename T, bool INV, int L, int Ns, int TwOff, int R, int... Rest>
struct FixedStages<T, INV, L, Ns, TwOff, R, Rest...> {
  template <class Sync>
  static FFB_HD void run(cpx<T> *src, cpx<T> *oth, int tid, int nthr, const cpx<T> *__restrict__ tw, Sync sync) {
    fixed_stage<T, INV, L, Ns, R>(src, oth, tid, nthr, tw + TwOff);
    sync();
    FixedStages<T, INV, L, Ns * R, TwOff + (R - 1) * Ns, Rest...>::run(oth, src, tid, nthr, tw, sync);
  }
};

// Stage runner for one compile-time radix sequence (the Core it runs must
// have exactly these radices).
template <typename T, int L, int... Rs>
struct FixedStagesRunner {
  template <bool INV, class Sync>
  FFB_HD void run(const Core &, cpx<T> *src, cpx<T> *oth, int tid, int nthr, const cpx<T> *__restrict__ tw,
                  Sync sync) const {
    FixedStages<T, INV, L, 1, 0, Rs...>::run(src, oth, tid, nthr, tw, sync);
  }
};

}  // namespace ffb
