// Instantiates the row kernels with compile-time radix sequences (float, fused
// Bluestein and convolution-row passes).
#include "rows.cuh"

namespace ffb {
namespace rows {
template cudaError_t launch_rows_any<float, 1, false>(const TileArgs<float> &, size_t, cudaStream_t);
template cudaError_t launch_rows_any<float, 3, false>(const TileArgs<float> &, size_t, cudaStream_t);
}  // namespace rows
}  // namespace ffb
