// Precision mode (prototype for its ship-or-not decision): the radix-16
// Stockham stages of a 256- or 4096-point complex transform as dense 16-point
// DFT-matrix products on the tcgen05 tensor cores, with split-bf16 operands
// and fp32 accumulation in tensor memory.
//
// One CTA holds 256 butterflies per stage (a 4096-point transform, or sixteen
// 256-point ones), one per thread.  Per stage a thread gathers its 16 inputs,
// applies the stage twiddles in fp32, splits each value into bf16 terms and
// writes its row of A; one thread issues the MMAs of two M = 128 tiles
// (N = 32: the real and imaginary parts of the 16 outputs) and commits them
// to an mbarrier; every warp then loads its 32 rows back from tensor memory
// (thread t receives row t: its own 16 outputs) and writes them where the
// next stage reads them.
//
// The 16-point DFT y = x F is the real product [Re y, Im y] = [Re x, Im x] W
// with W = [[Re F, Im F], [-Im F, Re F]] (32 x 32).  Split-bf16 keeps ~8
// bits per term:
//   3 terms: x = xh + xl, W = Wh + Wl: A = [xh xh xl], B = [Wh; Wl; Wh]
//            (the three products of the two-term split, K = 96);
//   6 terms: x = xh + xm + xl, W = Wh + Wm + Wl: A = [xh xh xh xm xm xl],
//            B = [Wh; Wm; Wl; Wh; Wm; Wh] (every product down to 2^-24, K = 192).
// W and its terms are built on the host in double; twiddles in long double.
#include <cuda_bf16.h>
#include <cuda_runtime.h>

#include <cmath>
#include <cstring>
#include <map>
#include <mutex>
#include <tuple>
#include <vector>

#include "../../include/flagfft_b200.h"
#include "exec.hpp"
#include "tc.cuh"

namespace ffb {
namespace pm {

constexpr int kRows = 256;  // butterflies per CTA and stage (two M = 128 tiles)

template <int TERMS>
struct Layout {
  static constexpr int K = 32 * TERMS;
  static constexpr int SBO = (K / 8) * 128;  // bytes between 8-row groups
  static constexpr int LBO = 128;            // bytes between 8-element k groups
  static constexpr int A_TILE = 16 * SBO;    // 128 rows
  static constexpr int A_BYTES = 2 * A_TILE;
  static constexpr int B_BYTES = 4 * SBO;  // 32 rows (N)
};

// Byte offset of (row, k) in a K-major no-swizzle operand.
__host__ __device__ constexpr int op_offset(int row, int k, int sbo) {
  return (row / 8) * sbo + (k / 8) * 128 + (row % 8) * 16 + 2 * (k % 8);
}

// Dynamic shared memory: header, A, B, the transforms' data buffers -- and,
// past them if need be, enough slack that the tensor core's reads of B would
// stay inside this CTA's allocation even with the two descriptor strides
// read the other way round (a guard; the layout follows the descriptor as
// documented).
template <int S, int TERMS>
constexpr size_t smem_bytes() {
  constexpr int L = 1 << (4 * S);
  constexpr int T = kRows / (L / 16);
  using Ly = Layout<TERMS>;
  constexpr size_t used = 1024 + Ly::A_BYTES + Ly::B_BYTES + (size_t)T * pp_size(L) * sizeof(cpx<float>);
  constexpr size_t guard = 1024 + Ly::A_BYTES + 4 * 128 + (size_t)(Ly::K / 8) * Ly::SBO;
  return used > guard ? used : guard;
}

struct Args {
  const cpx<float> *in;
  cpx<float> *out;
  long long batch;
  const unsigned char *btile;  // B operand bytes, already in the shared-memory layout
  const cpx<float> *tw;        // stage twiddles: stage 1 block (15 x 16), then stage 2 (15 x 256)
};

#ifndef FFB_HOST_EMULATION

static __device__ int g_pm_wait_failures;

__device__ __forceinline__ uint32_t pack2(__nv_bfloat16 a, __nv_bfloat16 b) {
  return (uint32_t)__bfloat16_as_ushort(a) | ((uint32_t)__bfloat16_as_ushort(b) << 16);
}

// Writes the A row of one butterfly: for every term, 16 real parts then 16
// imaginary parts of the term's split component.
template <int TERMS>
__device__ __forceinline__ void write_a_row(unsigned char *a_row, const cpx<float> (&v)[16]) {
  __nv_bfloat16 h[32], m[32], l[32];
#pragma unroll
  for (int q = 0; q < 32; ++q) {
    const float x = q < 16 ? v[q].x : v[q - 16].y;
    h[q] = __float2bfloat16_rn(x);
    const float r1 = x - __bfloat162float(h[q]);
    m[q] = __float2bfloat16_rn(r1);
    const float r2 = r1 - __bfloat162float(m[q]);
    l[q] = __float2bfloat16_rn(TERMS == 3 ? r1 : r2);
  }
  // component per term: 3 terms h h l; 6 terms h h h m m l
  constexpr int comp3[3] = {0, 0, 2}, comp6[6] = {0, 0, 0, 1, 1, 2};
#pragma unroll
  for (int t = 0; t < TERMS; ++t) {
    const int c = TERMS == 3 ? comp3[t] : comp6[t];
    const __nv_bfloat16 *src = c == 0 ? h : c == 1 ? m : l;
#pragma unroll
    for (int g = 0; g < 4; ++g) {
      uint4 w;
      w.x = pack2(src[8 * g + 0], src[8 * g + 1]);
      w.y = pack2(src[8 * g + 2], src[8 * g + 3]);
      w.z = pack2(src[8 * g + 4], src[8 * g + 5]);
      w.w = pack2(src[8 * g + 6], src[8 * g + 7]);
      *reinterpret_cast<uint4 *>(a_row + (4 * t + g) * 128) = w;  // k group 4t + g
    }
  }
}

template <int S, int TERMS>
__global__ void __launch_bounds__(kRows, 1) k_pm(const __grid_constant__ Args p) {
  pdl_entry();
  constexpr int L = 1 << (4 * S), NB = L / 16, T = kRows / NB;
  using Ly = Layout<TERMS>;
  constexpr uint32_t idesc = tc::idesc_bf16_f32(128, 32);
  extern __shared__ __align__(1024) unsigned char sm[];
  uint64_t *bar = reinterpret_cast<uint64_t *>(sm);
  uint32_t *tmem_slot = reinterpret_cast<uint32_t *>(sm + 8);
  unsigned char *A = sm + 1024;
  unsigned char *B = A + Ly::A_BYTES;
  cpx<float> *data = reinterpret_cast<cpx<float> *>(B + Ly::B_BYTES);
  const int tid = (int)threadIdx.x, warp = tid >> 5;
  const long long t0 = (long long)blockIdx.x * T;
  const int tloc = tid / NB, j = tid % NB;
  const long long tr = t0 + tloc;
  const bool live = tr < p.batch;
  for (int i = tid; i < Ly::B_BYTES / 16; i += kRows)
    reinterpret_cast<uint4 *>(B)[i] = reinterpret_cast<const uint4 *>(p.btile)[i];
  if (tid == 0) {
    tma::mbar_init(bar, 1);
    tma::fence_mbar_init();
  }
  if (warp == 0) tc::tmem_alloc(tmem_slot, 64);
  tma::fence_async_smem();
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  const uint32_t tmem = *tmem_slot;
  cpx<float> *buf = data + tloc * pp_size(L);
  const cpx<float> *src = p.in + (live ? tr : t0) * L;
  // this thread's A row: tile tid / 128, row tid % 128
  unsigned char *a_row = A + (tid / 128) * Ly::A_TILE + op_offset(tid % 128, 0, Ly::SBO);
  bool failed = false;  // the same in every thread: set from the barrier's OR
  int stage = 0;
#pragma unroll 1
  for (int Ns = 1; Ns < L; Ns *= 16, ++stage) {
    const bool last = Ns * 16 == L;
    cpx<float> v[16];
#pragma unroll
    for (int r = 0; r < 16; ++r) v[r] = Ns == 1 ? src[j + r * NB] : buf[pp_pos(j + r * NB)];
    if (Ns > 1) {
      const int k = j % Ns;
      const cpx<float> *tw = p.tw + (Ns == 16 ? 0 : 15 * 16) + k;
#pragma unroll
      for (int r = 1; r < 16; ++r) v[r] = cmul(v[r], ldg_c(tw + (r - 1) * Ns));
    }
    write_a_row<TERMS>(a_row, v);
    tma::fence_async_smem();  // A rows (generic writes) before the tensor core reads them
    tc::fence_before_sync();
    __syncthreads();
    if (tid == 0) {
      tc::fence_after_sync();
      const uint32_t a0 = tma::smem_u32(A), b0 = tma::smem_u32(B);
#pragma unroll
      for (int tile = 0; tile < 2; ++tile)
#pragma unroll
        for (int kk = 0; kk < Ly::K / 16; ++kk)
          tc::mma_bf16(tmem + 32 * tile, tc::smem_desc(a0 + tile * Ly::A_TILE + kk * 256, Ly::LBO, Ly::SBO),
                       tc::smem_desc(b0 + kk * 256, Ly::LBO, Ly::SBO), idesc, kk > 0 ? 1u : 0u);
      tc::commit(bar);
    }
    const bool ok = tma::mbar_wait(bar, (uint32_t)(stage & 1));
    if (__syncthreads_or(!ok)) {
      failed = true;
      break;
    }
    tc::fence_after_sync();
    uint32_t r32[32];
    tc::ld_32x32(tmem + ((uint32_t)(32 * (warp % 4)) << 16) + 32u * (uint32_t)(warp / 4), r32);
    tc::wait_ld();
    const int base = (j - j % Ns) * 16 + j % Ns;
#pragma unroll
    for (int q = 0; q < 16; ++q) {
      const cpx<float> y = mk(__uint_as_float(r32[q]), __uint_as_float(r32[16 + q]));
      if (last) {
        if (live) p.out[tr * L + base + q * Ns] = y;
      } else {
        buf[pp_pos(base + q * Ns)] = y;
      }
    }
    tc::fence_before_sync();
    __syncthreads();
  }
  if (failed) {
    if (tid == 0) {
      atomicAdd(&g_pm_wait_failures, 1);
      tma::mbar_wait(bar, (uint32_t)(stage & 1));  // bounded: the MMAs still in flight
    }
    __syncthreads();
  }
  tc::fence_after_sync();
  if (warp == 0) tc::tmem_dealloc(tmem, 64);
}

#endif  // !FFB_HOST_EMULATION

// ---- host tables

uint16_t bf16_bits(double d) {
  const float f = (float)d;
  uint32_t u;
  std::memcpy(&u, &f, 4);
  u += 0x7FFFu + ((u >> 16) & 1u);  // round to nearest even
  return (uint16_t)(u >> 16);
}
double bf16_value(uint16_t b) {
  const uint32_t u = (uint32_t)b << 16;
  float f;
  std::memcpy(&f, &u, 4);
  return f;
}

// B operand bytes (N = 32 rows, K = 32 * terms, K-major) for the forward (or
// inverse) 16-point DFT matrix.
std::vector<unsigned char> b_tile(int terms, bool inverse) {
  const int K = 32 * terms, sbo = (K / 8) * 128;
  std::vector<unsigned char> out((size_t)4 * sbo, 0);
  const long double pi = 3.14159265358979323846264338327950288L;
  for (int n = 0; n < 32; ++n)
    for (int kk = 0; kk < 32; ++kk) {
      // W[kk][n]: kk < 16 multiplies Re x_kk, kk >= 16 Im x_(kk-16); n < 16 gives Re y_n, n >= 16 Im y_(n-16)
      const int jj = kk % 16, qq = n % 16;
      const long double ang = (inverse ? 2 : -2) * pi * (long double)((jj * qq) % 16) / 16.0L;
      const double fr = (double)cosl(ang), fi = (double)sinl(ang);
      const double w = kk < 16 ? (n < 16 ? fr : fi) : (n < 16 ? -fi : fr);
      const uint16_t h = bf16_bits(w);
      const uint16_t m = bf16_bits(w - bf16_value(h));
      const uint16_t l = bf16_bits(w - bf16_value(h) - bf16_value(m));
      // component per term: 3 terms h l h; 6 terms h m l h m h
      static const int comp3[3] = {0, 2, 0}, comp6[6] = {0, 1, 2, 0, 1, 0};
      for (int t = 0; t < terms; ++t) {
        const int c = terms == 3 ? comp3[t] : comp6[t];
        // 3 terms: the low component is the whole remainder w - h
        const uint16_t v = c == 0 ? h : c == 1 ? m : (terms == 3 ? bf16_bits(w - bf16_value(h)) : l);
        std::memcpy(&out[(size_t)op_offset(n, 32 * t + kk, sbo)], &v, 2);
      }
    }
  return out;
}

// Stage twiddles: stage 1 (span 16) then stage 2 (span 256), entry
// (r - 1) * span + k = W_{16 span}^{r k}, conjugated for the inverse.
std::vector<cpx<float>> twiddles(bool inverse) {
  std::vector<cpx<float>> t;
  const long double pi = 3.14159265358979323846264338327950288L;
  for (int span : {16, 256})
    for (int r = 1; r < 16; ++r)
      for (int k = 0; k < span; ++k) {
        const long long e = ((long long)r * k) % (16 * span);
        const long double a = (inverse ? 2 : -2) * pi * (long double)e / (long double)(16 * span);
        t.push_back(mk((float)cosl(a), (float)sinl(a)));
      }
  return t;
}

struct Tables {
  DevPtr b, tw;
};

const Tables &tables(int terms, bool inverse) {
  static std::mutex mu;
  static std::map<std::tuple<int, int, bool>, Tables> cache;
  int dev = 0;
  cudaGetDevice(&dev);
  std::lock_guard<std::mutex> lock(mu);
  auto key = std::make_tuple(dev, terms, inverse);
  auto it = cache.find(key);
  if (it != cache.end()) return it->second;
  Tables t;
  const auto b = b_tile(terms, inverse);
  const auto w = twiddles(inverse);
  t.b = upload(b.data(), b.size());
  t.tw = upload(w.data(), w.size() * sizeof(cpx<float>));
  return cache.emplace(key, t).first->second;
}

#ifndef FFB_HOST_EMULATION
template <int S, int TERMS>
cudaError_t launch(const Args &a, cudaStream_t s) {
  constexpr int L = 1 << (4 * S), T = kRows / (L / 16);
  cudaError_t e = set_smem_limit_once<k_pm<S, TERMS>>((int)smem_bytes<S, TERMS>());
  if (e != cudaSuccess) return e;
  const unsigned grid = (unsigned)((a.batch + T - 1) / T);
  return launch_pdl(k_pm<S, TERMS>, dim3(grid), dim3(kRows), smem_bytes<S, TERMS>(), s, a);
}
#endif

}  // namespace pm
}  // namespace ffb

using namespace ffb;

extern "C" flagfftResult flagfftB200PrecisionC2C(const flagfftComplex *idata, flagfftComplex *odata, int n, int batch,
                                                int direction, int terms, flagfftStream_t stream) {
  if (idata == nullptr || odata == nullptr || batch <= 0 || batch > (1 << 26)) return FLAGFFT_INVALID_VALUE;
  if (direction != FLAGFFT_FORWARD && direction != FLAGFFT_INVERSE) return FLAGFFT_INVALID_VALUE;
  if ((n != 256 && n != 4096) || (terms != 3 && terms != 6)) return FLAGFFT_NOT_SUPPORTED;
#ifdef FFB_HOST_EMULATION
  (void)stream;
  return FLAGFFT_NOT_SUPPORTED;
#else
  try {
    const pm::Tables &t = pm::tables(terms, direction == FLAGFFT_INVERSE);
    pm::Args a{reinterpret_cast<const cpx<float> *>(idata), reinterpret_cast<cpx<float> *>(odata), batch,
               reinterpret_cast<const unsigned char *>(t.b->ptr), reinterpret_cast<const cpx<float> *>(t.tw->ptr)};
    cudaStream_t s = static_cast<cudaStream_t>(stream);
    cudaError_t e = n == 256 ? (terms == 3 ? pm::launch<2, 3>(a, s) : pm::launch<2, 6>(a, s))
                             : (terms == 3 ? pm::launch<3, 3>(a, s) : pm::launch<3, 6>(a, s));
    return e == cudaSuccess ? FLAGFFT_SUCCESS : FLAGFFT_EXEC_FAILED;
  } catch (const std::bad_alloc &) {
    return FLAGFFT_ALLOC_FAILED;
  } catch (const std::exception &) {
    return FLAGFFT_EXEC_FAILED;
  }
#endif
}

extern "C" flagfftResult flagfftB200PrecisionWaitFailures(long long *count) {
  if (count == nullptr) return FLAGFFT_INVALID_VALUE;
#ifndef FFB_HOST_EMULATION
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, pm::g_pm_wait_failures, sizeof(int)) != cudaSuccess) return FLAGFFT_INVALID_DEVICE;
  *count = v;
#else
  *count = 0;
#endif
  return FLAGFFT_SUCCESS;
}
