// flagfftB200ExecC2CNoAlloc: a batched power-of-two C2C transform whose
// four-step workspace and tables live in fixed device arrays of this library,
// for callers that cannot allocate device memory (see include/flagfft_b200.h).
//
// The transform runs the same two tile passes a four-step plan uses (column
// FFTs of length n1 with the W_n^{j2 k1} twiddle fused into their store, then
// row FFTs of length n2), through launch_tile, with every pointer taken from
// the static arrays below instead of plan-owned allocations.
#include <cuda_runtime.h>

#include <cmath>
#include <cstdio>
#include <mutex>

#include "../../include/flagfft_b200.h"
#include "kernels.cuh"

namespace ffb {
namespace {

// Workspace: up to 2^22 complex64 elements (32 MiB) of batch * n.
constexpr long long kNoAllocMaxElems = 1ll << 22;
// Per-stage twiddle blocks of the radix-16 cores of every power of two
// 2..4096, one table per direction (the length-2^l core's blocks, 2^l - 1
// entries, at offset 2^l - l - 1; 8178 entries in all).
constexpr int kRootLen = 4096;
constexpr int kStageTableLen = 8192;
// Four-step twiddle W_n^m = hi[m >> 12] * lo[m & 4095] for n <= 2^24.
constexpr int kSplitBits = 12;
constexpr int kSplit = 1 << kSplitBits;

static __device__ __align__(256) cpx<float> g_scratch[kNoAllocMaxElems];
static __device__ __align__(256) cpx<float> g_roots[2 * kStageTableLen];  // forward, inverse
static __device__ __align__(256) cpx<float> g_ptw_lo[kSplit];
static __device__ __align__(256) cpx<float> g_ptw_hi[kSplit];

struct DeviceState {
  bool ready = false;
  cpx<float> *scratch = nullptr, *roots = nullptr, *lo = nullptr, *hi = nullptr;
};
constexpr int kMaxDevices = 64;
DeviceState g_state[kMaxDevices];
std::mutex g_mutex;

// exp(-2 pi i m / n), computed in double and rounded once.
__global__ void k_fill_roots(cpx<float> *dst, int count, long long n, long long step) {
  for (int m = blockIdx.x * blockDim.x + threadIdx.x; m < count; m += gridDim.x * blockDim.x) {
    const long long e = ((long long)m * step) % n;
    double s, c;
    sincospi(-2.0 * (double)e / (double)n, &s, &c);
    dst[m] = mk((float)c, (float)s);
  }
}

// Offset of the length-2^l core's stage blocks in one direction's table.
__host__ __device__ inline int stage_table_offset(int l) { return (1 << l) - l - 1; }

// Fills one direction's stage blocks of pow2_core(2^l), l = 1..12: entry k of
// row r - 1 of stage s is W_{span R}^{r k} (conjugated when inverse), span =
// 16^s, R = 16 or the smaller last radix.
__global__ void k_fill_stage_tables(cpx<float> *dst, int inverse) {
  for (int l = 1; l <= 12; ++l) {
    const int L = 1 << l;
    cpx<float> *t = dst + stage_table_offset(l);
    for (int e = blockIdx.x * blockDim.x + threadIdx.x; e < L - 1; e += gridDim.x * blockDim.x) {
      int span = 1, rem = L, off = 0;
      while (rem > 1) {
        const int R = rem >= 16 ? 16 : rem;
        if (e < off + (R - 1) * span) {
          const int r = 1 + (e - off) / span, k = (e - off) % span;
          double sn, cs;
          sincospi((inverse ? 2.0 : -2.0) * (double)(r * k) / (double)(span * R), &sn, &cs);
          t[e] = mk((float)cs, (float)sn);
          break;
        }
        off += (R - 1) * span;
        span *= R;
        rem /= R;
      }
    }
  }
}

// Device addresses of the static arrays for the current device; filled once
// per device (the first call on a device does this set-up).
cudaError_t device_state(DeviceState **out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  if (dev < 0 || dev >= kMaxDevices) return cudaErrorInvalidDevice;
  std::lock_guard<std::mutex> lock(g_mutex);
  DeviceState &st = g_state[dev];
  if (!st.ready) {
    if ((e = cudaGetSymbolAddress(reinterpret_cast<void **>(&st.scratch), g_scratch)) != cudaSuccess) return e;
    if ((e = cudaGetSymbolAddress(reinterpret_cast<void **>(&st.roots), g_roots)) != cudaSuccess) return e;
    if ((e = cudaGetSymbolAddress(reinterpret_cast<void **>(&st.lo), g_ptw_lo)) != cudaSuccess) return e;
    if ((e = cudaGetSymbolAddress(reinterpret_cast<void **>(&st.hi), g_ptw_hi)) != cudaSuccess) return e;
    k_fill_stage_tables<<<16, 256>>>(st.roots, 0);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    k_fill_stage_tables<<<16, 256>>>(st.roots + kStageTableLen, 1);
    if ((e = cudaGetLastError()) != cudaSuccess) return e;
    if ((e = cudaDeviceSynchronize()) != cudaSuccess) return e;
    st.ready = true;
  }
  *out = &st;
  return cudaSuccess;
}

Core pow2_core(int L) {
  // radix-16 stages, one smaller power-of-two stage for the remainder
  Core c{};
  c.L = L;
  int rem = L, span = 1, s = 0, off = 0;
  while (rem > 1) {
    const int r = rem >= 16 ? 16 : rem;
    c.radix[s] = r;
    c.span[s] = span;
    c.twoff[s] = off;
    off += (r - 1) * span;
    c.sdiv[s] = make_fastdiv((uint32_t)span);
    c.rdiv[s] = make_fastdiv((uint32_t)r);
    span *= r;
    rem /= r;
    ++s;
  }
  c.nst = s;
  return c;
}

TileArgs<float> pass_args(int L, int G, long long nbatch, long long ib, long long ig, long long ii, long long ob,
                          long long og, long long ok, bool inverse, const cpx<float> *roots, size_t *smem) {
  TileArgs<float> a{};
  a.nbatch = nbatch;
  a.ib = ib;
  a.ig = ig;
  a.ii = ii;
  a.ob = ob;
  a.og = og;
  a.ok = ok;
  a.G = G;
  a.inv = inverse ? 1 : 0;
  a.n = L;
  a.core = pow2_core(L);
  int l = 0;
  while ((1 << l) < L) ++l;
  a.tw = roots + (inverse ? kStageTableLen : 0) + stage_table_offset(l);
  a.pp = 1;
  a.wfast = ii > ig ? 1 : 0;
  const int rmax = L >= 16 ? 16 : L;
  int tpt = (L + rmax - 1) / rmax;
  tpt = tpt <= 32 ? tpt : (tpt + 31) / 32 * 32;
  const size_t per = (2 * (size_t)pp_size(L) + 3) * sizeof(cpx<float>);
  int W = a.wfast ? 8 : (256 / tpt > 1 ? 256 / tpt : 1);
  if (W > G) W = G;
  while (W > 1 && per * W > 110 * 1024) --W;
  if (W * tpt > 512) tpt = 512 / W;
  a.W = W;
  a.tpt = tpt;
  a.ldiv = make_fastdiv((uint32_t)L);
  a.wdiv = make_fastdiv((uint32_t)W);
  a.ndiv = make_fastdiv((uint32_t)L);
  a.hdiv = make_fastdiv((uint32_t)(L / 2 > 0 ? L / 2 : 1));
  *smem = per * (size_t)W;
  return a;
}

}  // namespace
}  // namespace ffb

using namespace ffb;

extern "C" flagfftResult flagfftB200ExecC2CNoAlloc(const flagfftComplex *idata, flagfftComplex *odata, int n,
                                                   int batch, int direction, flagfftStream_t stream) {
  if (idata == nullptr || odata == nullptr || batch <= 0) return FLAGFFT_INVALID_VALUE;
  if (direction != FLAGFFT_FORWARD && direction != FLAGFFT_INVERSE) return FLAGFFT_INVALID_VALUE;
  if (n < 2 * kRootLen || (long long)n > kNoAllocMaxElems || (n & (n - 1)) != 0) {
    std::fprintf(stderr, "[flagfft] ExecC2CNoAlloc: n=%d must be a power of two in [8192, 2^22]\n", n);
    return FLAGFFT_INVALID_SIZE;
  }
  if ((long long)n * batch > kNoAllocMaxElems || batch > 65535) {
    std::fprintf(stderr,
                 "[flagfft] ExecC2CNoAlloc: batch*n=%lld exceeds the fixed workspace of %lld elements\n",
                 (long long)n * batch, kNoAllocMaxElems);
    return FLAGFFT_INVALID_SIZE;
  }
  DeviceState *st = nullptr;
  if (device_state(&st) != cudaSuccess) {
    cudaGetLastError();
    return FLAGFFT_INVALID_DEVICE;
  }
  // n = n1 * n2 with n1 = 2^floor(log2 n / 2), n2 = n / n1; both <= 4096
  int lg = 0;
  while ((1 << lg) < n) ++lg;
  const int n1 = 1 << (lg / 2), n2 = n / n1;
  const bool inverse = direction == FLAGFFT_INVERSE;
  cudaStream_t s = static_cast<cudaStream_t>(stream);

  // this call's four-step twiddle tables: lo[m] = W_n^m, hi[m] = W_n^{m * 4096}
  const int nhi = (n + kSplit - 1) / kSplit;
  k_fill_roots<<<16, 256, 0, s>>>(st->lo, kSplit, n, 1);
  k_fill_roots<<<16, 256, 0, s>>>(st->hi, nhi, n, kSplit);

  size_t smem_a = 0, smem_b = 0;
  // pass A: columns j2 (stride n2) of length n1, x W_n^{j2 k1}, rows Y[j2][k1] in the workspace
  TileArgs<float> a = pass_args(n1, n2, batch, n, 1, n2, n, n1, 1, inverse, st->roots, &smem_a);
  a.in = idata;
  a.out = st->scratch;
  a.post_twiddle = 1;
  a.ptw_lo = st->lo;
  a.ptw_hi = st->hi;
  a.ptw_div = make_fastdiv((uint32_t)kSplit);
  // pass B: for each k1, length n2 over Y[j2][k1] -> X[k1 + n1 k2]
  TileArgs<float> b = pass_args(n2, n1, batch, n, 1, n1, n, 1, n1, inverse, st->roots, &smem_b);
  b.in = st->scratch;
  b.out = odata;
  cudaError_t e = launch_tile<float>(a, CoreKind::Dit, IoKind::C2C, smem_a, s);
  if (e == cudaSuccess) e = launch_tile<float>(b, CoreKind::Dit, IoKind::C2C, smem_b, s);
  if (e != cudaSuccess) {
    std::fprintf(stderr, "[flagfft] ExecC2CNoAlloc failed: %s\n", cudaGetErrorString(e));
    return FLAGFFT_EXEC_FAILED;
  }
  return FLAGFFT_SUCCESS;
}
