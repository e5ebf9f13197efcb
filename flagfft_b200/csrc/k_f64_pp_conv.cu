// Instantiates one group of on-chip FFT pass kernels (double); split from
// kernels.cu so the kernel variants compile in parallel.
#include "tile_impl.cuh"

namespace ffb {
namespace tile {
template cudaError_t launch_pp<double, 2, false>(const TileArgs<double> &, size_t, cudaStream_t);
template cudaError_t launch_pp<double, 3, false>(const TileArgs<double> &, size_t, cudaStream_t);
}  // namespace tile
}  // namespace ffb
