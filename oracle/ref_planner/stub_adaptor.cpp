// Test infrastructure only: the two device queries the reference planner needs,
// answered without a GPU so its unmodified sources link on the host.
// The reference declares both in src/adaptor/adaptor.h; its CUDA backend
// answers them from the driver (src/adaptor/backend/cuda/adaptor.cpp).
#include <cstdint>
#include <cstdlib>
#include <string>

namespace flagfft::adaptor {

std::string backend_name() { return "cuda"; }

// B200 opt-in dynamic shared memory per block (cudaDevAttrMaxSharedMemoryPerBlockOptin);
// FFO_SMEM overrides it so other devices' plans can be reproduced.
int64_t max_dynamic_smem_bytes(int) {
  const char *v = std::getenv("FFO_SMEM");
  return v ? std::atoll(v) : 232448;
}

}  // namespace flagfft::adaptor
