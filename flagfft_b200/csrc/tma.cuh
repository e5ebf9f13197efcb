// Tensor-memory-accelerator (TMA) copies and mbarriers for sm_100a, in
// hand-written inline PTX.
//
// Only plain tiled copies are used: every load fills this CTA's shared memory
// from this GPU's global memory (no .multicast::cluster), every store writes
// a shared-memory tile back.  A tensor map describes a 4-D view of global
// memory in units of the real scalar (float or double; a complex element is
// two scalars), so a copy's innermost coordinate is always an even scalar
// index: for complex64 tiles its byte offset is a multiple of 16 whenever the
// complex column index is even, which the tile shapes guarantee (the host
// checks every map before it encodes one).
//
// Waits are bounded: mbar_wait gives up after about a second of device clock
// and returns false, so a copy that never lands turns into an error status
// instead of a hung GPU.
#pragma once

#include <cstdint>

#include "engine.cuh"

#ifndef FFB_HOST_EMULATION
#include <cuda.h>
#endif

namespace ffb {
namespace tma {

// A 4-D tiled view of global memory in scalar units (dims[0] innermost),
// with the box one copy moves.  The device build also carries the encoded
// CUtensorMap; the host-emulation build copies boxes by hand from these
// numbers, so the same index arithmetic runs on the CPU.
struct View {
  void *base = nullptr;
  unsigned long long dims[4] = {1, 1, 1, 1};
  unsigned long long strides[3] = {0, 0, 0};  // bytes of dims 1..3
  unsigned box[4] = {1, 1, 1, 1};
  int scalar_bytes = 4;
};

#ifndef FFB_HOST_EMULATION

__device__ __forceinline__ uint32_t smem_u32(const void *p) { return (uint32_t)__cvta_generic_to_shared(p); }

__device__ __forceinline__ void mbar_init(uint64_t *bar, uint32_t count) {
  asm volatile("mbarrier.init.shared::cta.b64 [%0], %1;" ::"r"(smem_u32(bar)), "r"(count) : "memory");
}

// Makes initialised mbarriers visible to the asynchronous (TMA) proxy.
__device__ __forceinline__ void fence_mbar_init() { asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory"); }

// Orders this thread's ordinary shared-memory writes before later TMA reads
// of the same memory (a TMA store of a tile the threads just wrote).
__device__ __forceinline__ void fence_async_smem() { asm volatile("fence.proxy.async.shared::cta;" ::: "memory"); }

// One arrival that also expects `bytes` of TMA transactions on the barrier.
__device__ __forceinline__ void mbar_expect_tx(uint64_t *bar, uint32_t bytes) {
  asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(smem_u32(bar)), "r"(bytes) : "memory");
}

// One plain arrival (release: this thread's earlier shared-memory writes are
// visible to the thread that sees the phase complete).
__device__ __forceinline__ void mbar_arrive(uint64_t *bar) {
  asm volatile("mbarrier.arrive.shared::cta.b64 _, [%0];" ::"r"(smem_u32(bar)) : "memory");
}

__device__ __forceinline__ bool mbar_try_wait(uint64_t *bar, uint32_t parity) {
  uint32_t done;
  asm volatile(
      "{\n"
      "  .reg .pred p;\n"
      "  mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n"
      "  selp.u32 %0, 1, 0, p;\n"
      "}\n"
      : "=r"(done)
      : "r"(smem_u32(bar)), "r"(parity)
      : "memory");
  return done != 0;
}

// Waits for the barrier's phase `parity` to complete; false after about
// 2^31 device clocks (~1 s at 1.9 GHz) without completion.
__device__ __forceinline__ bool mbar_wait(uint64_t *bar, uint32_t parity) {
  if (mbar_try_wait(bar, parity)) return true;
  const long long t0 = clock64();
  while (!mbar_try_wait(bar, parity)) {
    if (clock64() - t0 > (1ll << 31)) return false;
  }
  return true;
}

// Tiled 4-D load of one box into shared memory; its bytes complete on `bar`.
__device__ __forceinline__ void load_4d(void *dst, const CUtensorMap *map, int c0, int c1, int c2, int c3,
                                        uint64_t *bar) {
  asm volatile(
      "cp.async.bulk.tensor.4d.shared::cluster.global.tile.mbarrier::complete_tx::bytes"
      " [%0], [%1, {%2, %3, %4, %5}], [%6];" ::"r"(smem_u32(dst)),
      "l"(reinterpret_cast<uint64_t>(map)), "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(bar))
      : "memory");
}

// Tiled 4-D store of one box from shared memory (bulk async group).
__device__ __forceinline__ void store_4d(const CUtensorMap *map, int c0, int c1, int c2, int c3, const void *src) {
  asm volatile(
      "cp.async.bulk.tensor.4d.global.shared::cta.tile.bulk_group"
      " [%0, {%1, %2, %3, %4}], [%5];" ::"l"(reinterpret_cast<uint64_t>(map)),
      "r"(c0), "r"(c1), "r"(c2), "r"(c3), "r"(smem_u32(src))
      : "memory");
}

__device__ __forceinline__ void commit() { asm volatile("cp.async.bulk.commit_group;" ::: "memory"); }

// Waits until at most N committed store groups still read shared memory.
template <int N>
__device__ __forceinline__ void wait_read() {
  asm volatile("cp.async.bulk.wait_group.read %0;" ::"n"(N) : "memory");
}

// Waits until at most N committed store groups are still in flight.
template <int N>
__device__ __forceinline__ void wait_all() {
  asm volatile("cp.async.bulk.wait_group %0;" ::"n"(N) : "memory");
}

#endif  // !FFB_HOST_EMULATION

// Host emulation of one box copy between a View and a dense shared-memory
// box (box[0] innermost), zero-filling reads outside the view and dropping
// writes outside it, as the hardware does.
// A copy the hardware would refuse (shared-memory address not 128-byte
// aligned, global base not 16-byte aligned, or an innermost coordinate whose
// byte offset is not a multiple of 16) moves nothing, so the caller's result
// comes out wrong instead of silently right.
inline void emulate_box(const View &v, int c0, int c1, int c2, int c3, void *smem, bool load) {
  const size_t sb = (size_t)v.scalar_bytes;
  unsigned char *s = static_cast<unsigned char *>(smem);
  if ((reinterpret_cast<uintptr_t>(smem) & 127) != 0 || (reinterpret_cast<uintptr_t>(v.base) & 15) != 0 ||
      (((long long)c0 * (long long)sb) & 15) != 0)
    return;
  for (unsigned i3 = 0; i3 < v.box[3]; ++i3)
    for (unsigned i2 = 0; i2 < v.box[2]; ++i2)
      for (unsigned i1 = 0; i1 < v.box[1]; ++i1)
        for (unsigned i0 = 0; i0 < v.box[0]; ++i0) {
          const long long x0 = (long long)c0 + i0, x1 = (long long)c1 + i1, x2 = (long long)c2 + i2,
                          x3 = (long long)c3 + i3;
          unsigned char *sp = s + ((((size_t)i3 * v.box[2] + i2) * v.box[1] + i1) * v.box[0] + i0) * sb;
          const bool in = x0 >= 0 && x1 >= 0 && x2 >= 0 && x3 >= 0 && (unsigned long long)x0 < v.dims[0] &&
                          (unsigned long long)x1 < v.dims[1] && (unsigned long long)x2 < v.dims[2] &&
                          (unsigned long long)x3 < v.dims[3];
          unsigned char *gp = static_cast<unsigned char *>(v.base) + (size_t)x0 * sb + (size_t)x1 * v.strides[0] +
                              (size_t)x2 * v.strides[1] + (size_t)x3 * v.strides[2];
          if (load) {
            for (size_t b = 0; b < sb; ++b) sp[b] = in ? gp[b] : 0;
          } else if (in) {
            for (size_t b = 0; b < sb; ++b) gp[b] = sp[b];
          }
        }
}

}  // namespace tma
}  // namespace ffb
