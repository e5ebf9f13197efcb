// Instantiates the row kernels with compile-time radix sequences (float, plain
// transforms in both directions).
#include "rows.cuh"

namespace ffb {
namespace rows {
template cudaError_t launch_rows_any<float, 0, false>(const TileArgs<float> &, size_t, cudaStream_t);
template cudaError_t launch_rows_any<float, 0, true>(const TileArgs<float> &, size_t, cudaStream_t);
}  // namespace rows
}  // namespace ffb
