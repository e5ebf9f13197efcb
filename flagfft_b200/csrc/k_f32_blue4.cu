// Instantiates the one-pass four-step Bluestein kernels (single precision).
#include "blue4.cuh"

namespace ffb {

template <>
cudaError_t launch_blue4<float>(const TileArgs<float> &a, cudaStream_t s) {
#define FFB_B4_LAUNCH(N1, L2, ...)                                                                                   \
  if (!a.blue_pair && a.blue_cols == (N1) && tile::core_is<L2, __VA_ARGS__>(a.core) &&                             \
      tile::core_is<L2, __VA_ARGS__>(a.core2))                                                                     \
    return blue4::launch<float, N1, L2, __VA_ARGS__>(a, s);
  FFB_BLUE4_SHAPES(FFB_B4_LAUNCH)
#undef FFB_B4_LAUNCH
#define FFB_B4P_LAUNCH(N1, L2, ...)                                                                                  \
  if (a.blue_pair && a.blue_cols == (N1) && tile::core_is<L2, __VA_ARGS__>(a.core) &&                              \
      tile::core_is<L2, __VA_ARGS__>(a.core2))                                                                     \
    return blue4::launch_pair<float, N1, L2, __VA_ARGS__>(a, s);
  FFB_BLUE4_PAIR_SHAPES(FFB_B4P_LAUNCH)
#undef FFB_B4P_LAUNCH
  return cudaErrorNotSupported;
}

int blue4_threads(int n1, int L2, bool pair) {
#define FFB_B4_NT(N1, L2_, ...) \
  if (!pair && n1 == (N1) && L2 == (L2_)) return blue4::Shape<N1, L2_, __VA_ARGS__>::NT;
  FFB_BLUE4_SHAPES(FFB_B4_NT)
#undef FFB_B4_NT
#define FFB_B4P_NT(N1, L2_, ...) \
  if (pair && n1 == (N1) && L2 == (L2_)) return blue4::PairShape<N1, L2_, __VA_ARGS__>::NT;
  FFB_BLUE4_PAIR_SHAPES(FFB_B4P_NT)
#undef FFB_B4P_NT
  return 0;
}

size_t blue4_smem(int n1, int L2, size_t elem_bytes, bool pair) {
  // rows::slot_len<L2>() per row; a pair's CTA holds half of the rows
  return (size_t)(pair ? n1 / 2 : n1) * (size_t)(pp_size(L2) + 1) * elem_bytes;
}

}  // namespace ffb
