// Instantiates one group of on-chip FFT pass kernels (float); split from
// kernels.cu so the kernel variants compile in parallel.
#include "tile_impl.cuh"

namespace ffb {
namespace tile {
template cudaError_t launch_pp<float, 0, false>(const TileArgs<float> &, size_t, cudaStream_t);
template cudaError_t launch_pp<float, 0, true>(const TileArgs<float> &, size_t, cudaStream_t);
template cudaError_t launch_pp<float, 1, false>(const TileArgs<float> &, size_t, cudaStream_t);
}  // namespace tile
}  // namespace ffb
