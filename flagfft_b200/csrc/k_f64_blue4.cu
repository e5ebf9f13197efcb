// Instantiates the one-pass four-step Bluestein kernels (double precision:
// the pair form only, since N1 rows of 2048 double-complex points exceed one
// CTA's shared memory).
#include "blue4.cuh"

namespace ffb {

template <>
cudaError_t launch_blue4<double>(const TileArgs<double> &a, cudaStream_t s) {
#define FFB_B4P_LAUNCH(N1, L2, ...)                                                                                  \
  if (a.blue_pair && a.blue_cols == (N1) && tile::core_is<L2, __VA_ARGS__>(a.core) &&                              \
      tile::core_is<L2, __VA_ARGS__>(a.core2))                                                                     \
    return blue4::launch_pair<double, N1, L2, __VA_ARGS__>(a, s);
  FFB_BLUE4_PAIR_SHAPES(FFB_B4P_LAUNCH)
#undef FFB_B4P_LAUNCH
  return cudaErrorNotSupported;
}

}  // namespace ffb
