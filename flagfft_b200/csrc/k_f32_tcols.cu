// Instantiates the TMA column passes (tcols.cuh) in float precision.
#include "tcols_impl.cuh"

namespace ffb {

template <>
cudaError_t launch_tcols<float>(const TileArgs<float> &a, cudaStream_t s) {
  return tcols::launch_any<float>(a, s);
}

template <>
bool tcols_eligible<float>(int L, long long nbatch, long long G, long long ib, long long ig, long long ii, long long ob,
                          long long og, long long ok, int *threads, size_t *smem) {
  return tcols::eligible<float>(L, nbatch, G, ib, ig, ii, ob, og, ok, threads, smem);
}

template <>
long long tcols_wait_failures<float>() {
#ifndef FFB_HOST_EMULATION
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, tcols::g_tcols_wait_failures, sizeof(int)) != cudaSuccess) return -1;
  return v;
#else
  return 0;
#endif
}

}  // namespace ffb
