// Instantiates the row kernels with compile-time radix sequences (double, fused
// Bluestein and convolution-row passes).
#include "rows.cuh"

namespace ffb {
namespace rows {
template cudaError_t launch_rows_any<double, 1, false>(const TileArgs<double> &, size_t, cudaStream_t);
template cudaError_t launch_rows_any<double, 3, false>(const TileArgs<double> &, size_t, cudaStream_t);
}  // namespace rows
}  // namespace ffb
