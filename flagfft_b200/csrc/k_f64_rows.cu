// Instantiates the row kernels with compile-time radix sequences (double, plain
// transforms in both directions).
#include "rows.cuh"

namespace ffb {
namespace rows {
template cudaError_t launch_rows_any<double, 0, false>(const TileArgs<double> &, size_t, cudaStream_t);
template cudaError_t launch_rows_any<double, 0, true>(const TileArgs<double> &, size_t, cudaStream_t);
}  // namespace rows
}  // namespace ffb
