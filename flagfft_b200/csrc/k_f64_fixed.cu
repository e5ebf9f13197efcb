// Instantiates the ping-pong kernels with compile-time radix sequences
// (double, Dit cores).
#include "tile_impl.cuh"

namespace ffb {
namespace tile {
template cudaError_t launch_pp_fixed_any<double, 0, false>(const TileArgs<double> &, size_t, cudaStream_t);
template cudaError_t launch_pp_fixed_any<double, 0, true>(const TileArgs<double> &, size_t, cudaStream_t);
}  // namespace tile
}  // namespace ffb
