// Instantiates the TMA column passes (tcols.cuh) in double precision.
#include "tcols_impl.cuh"

namespace ffb {

template <>
cudaError_t launch_tcols<double>(const TileArgs<double> &a, cudaStream_t s) {
  return tcols::launch_any<double>(a, s);
}

template <>
bool tcols_eligible<double>(int L, long long nbatch, long long G, long long ib, long long ig, long long ii, long long ob,
                          long long og, long long ok, int *threads, size_t *smem) {
  return tcols::eligible<double>(L, nbatch, G, ib, ig, ii, ob, og, ok, threads, smem);
}

template <>
long long tcols_wait_failures<double>() {
#ifndef FFB_HOST_EMULATION
  int v = 0;
  if (cudaMemcpyFromSymbol(&v, tcols::g_tcols_wait_failures, sizeof(int)) != cudaSuccess) return -1;
  return v;
#else
  return 0;
#endif
}

}  // namespace ffb
