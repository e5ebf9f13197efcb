// Instantiates one group of on-chip FFT pass kernels (float); split from
// kernels.cu so the kernel variants compile in parallel.
#include "tile_impl.cuh"

namespace ffb {
namespace tile {
template cudaError_t launch_group<float, 2>(const TileArgs<float> &, int, size_t, cudaStream_t);
template cudaError_t launch_one<float, 3, 0>(const TileArgs<float> &, size_t, cudaStream_t);
}  // namespace tile
}  // namespace ffb
