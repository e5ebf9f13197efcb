// Instantiates the persistent batch kernel (float).
#include "batch_impl.cuh"

namespace ffb {
template cudaError_t launch_batch<float>(const TileArgs<float> *, const int *, const BatchItem *, int, int *, int, size_t,
                                        int, cudaStream_t);
template int batch_resident_ctas<float>(int, size_t);
}  // namespace ffb
