// Instantiates the persistent batch kernel (double).
#include "batch_impl.cuh"

namespace ffb {
template cudaError_t launch_batch<double>(const TileArgs<double> *, const int *, const BatchItem *, int, int *, int, size_t,
                                        int, cudaStream_t);
template int batch_resident_ctas<double>(int, size_t);
}  // namespace ffb
