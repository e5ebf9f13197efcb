// Instantiates the strided tile kernels of the compile-time sequences
// (float); sequences whose tiles would hold fewer than two groups have none.
#include "tiles.cuh"

namespace ffb {

template <>
cudaError_t launch_tiles<float>(const TileArgs<float> &a, cudaStream_t s) {
#define FFB_TILES_LAUNCH(L, ...)                                                        \
  if (tile::core_is<L, __VA_ARGS__>(a.core)) {                                          \
    if constexpr (tiles::Shape<float, L, __VA_ARGS__>::NG >= 2)                           \
      return a.inv ? tiles::launch<float, true, L, __VA_ARGS__>(a, s)                     \
                   : tiles::launch<float, false, L, __VA_ARGS__>(a, s);                   \
    return cudaErrorNotSupported;                                                      \
  }
  FFB_FIXED_SEQUENCES(FFB_TILES_LAUNCH)
#undef FFB_TILES_LAUNCH
  return cudaErrorNotSupported;
}

template <>
bool tiles_shape<float>(int L, int *W, int *threads, size_t *smem) {
#define FFB_TILES_SHAPE(L_, ...)                                        \
  if (L == (L_)) {                                                      \
    using Sh = tiles::Shape<float, L_, __VA_ARGS__>;                      \
    if (Sh::NG < 2) return false;                                      \
    *W = Sh::W;                                                        \
    *threads = Sh::NT;                                                 \
    *smem = tiles::smem_of<float, L_, __VA_ARGS__>();                     \
    return true;                                                       \
  }
  FFB_FIXED_SEQUENCES(FFB_TILES_SHAPE)
#undef FFB_TILES_SHAPE
  return false;
}

}  // namespace ffb
