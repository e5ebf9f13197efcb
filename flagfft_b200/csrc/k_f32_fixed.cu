// Instantiates the ping-pong kernels with compile-time radix sequences
// (float, Dit cores).
#include "tile_impl.cuh"

namespace ffb {
namespace tile {
template cudaError_t launch_pp_fixed_any<float, 0, false>(const TileArgs<float> &, size_t, cudaStream_t);
template cudaError_t launch_pp_fixed_any<float, 0, true>(const TileArgs<float> &, size_t, cudaStream_t);
}  // namespace tile
}  // namespace ffb
