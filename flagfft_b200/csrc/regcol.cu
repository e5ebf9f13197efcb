// Register column pass: one thread per transform for single-codelet lengths
// (L <= 19) whose transforms sit side by side in memory (input and output
// transform distance 1, elements strided) -- the column passes of the
// three-pass Bluestein chain.  A warp's load or store of element i touches 32
// consecutive transforms, so every access is a full coalesced line; the
// transform itself is one codelet in registers, so the pass needs no shared
// memory and no barrier, and as many threads as the register file allows stay
// resident to keep loads in flight.  Chirp-on-load (chirp_mode 1),
// chirp-on-store (chirp_mode 2) and the four-step post-twiddle follow the tile
// passes' definitions (kernels.cuh).
#include "regcol.cuh"

namespace ffb {
namespace {

constexpr int kRegcolThreads = 128;

template <typename T, int R, bool INV>
__global__ void __launch_bounds__(kRegcolThreads) k_regcol(const __grid_constant__ TileArgs<T> a) {
  pdl_entry();
  const long long g = (long long)blockIdx.x * kRegcolThreads + threadIdx.x;
  if (g < a.G) regcol_transform<T, R, INV>(a, (long long)blockIdx.y, g);
}

template <typename T, int R, bool INV>
cudaError_t launch_dir(const TileArgs<T> &a, cudaStream_t s) {
#ifndef FFB_HOST_EMULATION
  dim3 grid((unsigned)((a.G + kRegcolThreads - 1) / kRegcolThreads), (unsigned)a.nbatch, 1);
  return launch_pdl(k_regcol<T, R, INV>, grid, dim3(kRegcolThreads), 0, s, a);
#else
  (void)s;
  for (long long by = 0; by < a.nbatch; ++by)
    for (long long g = 0; g < a.G; ++g) regcol_transform<T, R, INV>(a, by, g);
  return cudaSuccess;
#endif
}

template <typename T, int R>
cudaError_t launch_r(const TileArgs<T> &a, cudaStream_t s) {
  return a.inv ? launch_dir<T, R, true>(a, s) : launch_dir<T, R, false>(a, s);
}

}  // namespace

template <typename T>
cudaError_t launch_regcol(const TileArgs<T> &a, cudaStream_t s) {
  if (a.core.nst != 1 || a.core.radix[0] != a.core.L) return cudaErrorInvalidValue;
#define FFB_REGCOL(R) return launch_r<T, R>(a, s)
  FFB_RADIX_SWITCH(a.core.L, FFB_REGCOL)
#undef FFB_REGCOL
  return cudaErrorInvalidValue;
}

template cudaError_t launch_regcol<float>(const TileArgs<float> &, cudaStream_t);
template cudaError_t launch_regcol<double>(const TileArgs<double> &, cudaStream_t);

}  // namespace ffb
