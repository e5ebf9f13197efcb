// Persistent batch kernel: one launch runs a queue of work items drawn from
// many plans of different lengths (the passes of one phase of a batch
// program).  Each CTA takes the next item from a device counter, runs it with
// the same tile bodies as the per-plan kernels, and loops until the queue is
// empty, so lengths of very different cost share the GPU without a launch per
// length.  An item is (index of its pass's TileArgs, tile index):
//   ping-pong passes (kinds 0-3 = Dit, Bluestein, Rader, Conv): tile =
//     by * ceil(G / W) + bx, the CTA tile of the per-plan launch;
//   register-column passes (kind 8): tile = by * ceil(G / blockDim) + chunk,
//     blockDim consecutive transforms, one per thread.
// The CTA is as wide as the widest item of the launch; a narrower ping-pong
// item leaves the extra threads idle through its stages (they still meet
// every barrier).
#pragma once

#include "kernels.cuh"
#include "regcol.cuh"
#include "tile_impl.cuh"

namespace ffb {

enum BatchKind : int {
  kBatchPpDit = 0,
  kBatchPpBluestein = 1,
  kBatchPpRader = 2,
  kBatchPpConv = 3,
  kBatchR2C = 4,  // an on-chip Dit core with the real pack / Hermitian post on its load / store (in-place tile)
  kBatchC2R = 5,  // the same with the Hermitian pre / unpack
  kBatchRegcol = 8
};

struct BatchItem {
  int args;
  int tile;
};

// Dynamic shared memory a batch launch reserves ahead of the items' tiles.
constexpr size_t kBatchSmemHeader = 16;

namespace batch {

// CUDA thread block wider than the item's W * tpt threads.
struct DevXWide {
  int tpt, wfast, W;
  FFB_HD int tid() const {
#ifdef __CUDA_ARCH__
    return threadIdx.x;
#else
    return 0;
#endif
  }
  FFB_HD int nthreads() const {
#ifdef __CUDA_ARCH__
    return blockDim.x;
#else
    return 1;
#endif
  }
  FFB_HD void sync() const {
#ifdef __CUDA_ARCH__
    __syncthreads();
#endif
  }
  // Threads past the item's W * tpt run the stage loops with a first index
  // beyond every loop bound: no work, same barriers.  f has one call site:
  // its barriers are aligned (bar.sync), so every thread of a warp must reach
  // them through the same instructions, idle or not.
  template <class F>
  FFB_HD void per_slot(int Wn, F f) const {
    const int t = tid();
    int slot = 0, sub = 1 << 29;
    if (t < Wn * tpt) {
      slot = wfast ? t % Wn : t / tpt;
      sub = wfast ? t / Wn : t - slot * tpt;
    }
    f(slot, sub, tpt);
  }
};

template <typename T, bool INV>
FFB_HD void regcol_one(const TileArgs<T> &a, long long by, long long g) {
#define FFB_RC(R) regcol_transform<T, R, INV>(a, by, g)
  FFB_RADIX_SWITCH(a.core.L, FFB_RC)
#undef FFB_RC
}

// Runs item `tile` of a pass of kind `kind` with execution policy x.  The
// direction of a Dit core or a register column is the pass's own (a.inv):
// the passes of one phase need not share it (the column passes of a
// three-pass Bluestein run forward, then inverse).
template <typename T, class X>
FFB_HD void run_item(const TileArgs<T> &a, int kind, int tile, cpx<T> *sm, const X &x) {
  if (kind == kBatchRegcol) {
    const int width = x.nthreads();
    const int chunks = (a.G + width - 1) / width;
    const int by = tile / chunks;
    const long long g = (long long)(tile - by * chunks) * width + x.tid();
    if (g < a.G) {
      if (a.inv)
        regcol_one<T, true>(a, by, g);
      else
        regcol_one<T, false>(a, by, g);
    }
    return;
  }
  const int tiles = (a.G + a.W - 1) / a.W;
  const int by = tile / tiles, bx = tile - by * tiles;
  if (kind == kBatchR2C) {
    tile::tile_body<T, 0, (int)IoKind::R2C>(a, bx, by, sm, x);
  } else if (kind == kBatchC2R) {
    tile::tile_body<T, 0, (int)IoKind::C2R>(a, bx, by, sm, x);
  } else if (kind == kBatchPpDit) {
    if (a.inv)
      tile::tile_body_pp<T, 0, true>(a, bx, by, sm, x);
    else
      tile::tile_body_pp<T, 0, false>(a, bx, by, sm, x);
  } else if (kind == kBatchPpBluestein) {
    tile::tile_body_pp<T, 1, false>(a, bx, by, sm, x);
  } else if (kind == kBatchPpRader) {
    tile::tile_body_pp<T, 2, false>(a, bx, by, sm, x);
  } else {
    tile::tile_body_pp<T, 3, false>(a, bx, by, sm, x);
  }
}

template <typename T>
__global__ void __launch_bounds__(tile::TileBounds<T>::kMaxThreads)
    k_batch(const TileArgs<T> *__restrict__ args, const int *__restrict__ kinds, const BatchItem *__restrict__ items,
            int nitems, int *__restrict__ next) {
  pdl_entry();
  // the queue slot lives in the first 16 bytes of dynamic shared memory (a
  // static __shared__ variable would lower the dynamic limit below 227 KB)
  extern __shared__ __align__(16) unsigned char smraw[];
  int *const cur = reinterpret_cast<int *>(smraw);
  cpx<T> *sm = reinterpret_cast<cpx<T> *>(smraw + kBatchSmemHeader);
  for (;;) {
    if (threadIdx.x == 0) *cur = atomicAdd(next, 1);
    __syncthreads();
    const int it = *cur;  // every thread reads it before the barrier that ends the item
    if (it >= nitems) return;
    const BatchItem w = items[it];
    const TileArgs<T> &a = args[w.args];
    const DevXWide x{a.tpt, a.wfast, a.W};
    run_item<T>(a, kinds[w.args], w.tile, sm, x);
    __syncthreads();  // shared memory is reused by the next item
  }
}

}  // namespace batch

// Shared-memory classes of the persistent launches of a phase: items are
// grouped by the shared memory their tiles need, so small items get many CTAs
// per SM instead of the one a 227 KB item allows; the classes of a phase run
// concurrently on their own streams.  Class 4 holds register-column items.
constexpr int kBatchClasses = 5;
// Passes wider than kBatchWidth threads, or with tiles above 113 KB, share
// class 3 (one 512-thread CTA per SM); the others run kBatchWidth-thread CTAs,
// two or more per SM.
constexpr int kBatchWidth = 256;
inline int batch_class(size_t smem, int threads, bool regcol) {
  if (regcol) return 4;
  const size_t s = smem + kBatchSmemHeader;
  if (threads > kBatchWidth) return 3;
  return s <= 32 * 1024 ? 0 : s <= 76 * 1024 ? 1 : s <= 113 * 1024 ? 2 : 3;
}

// Launch of one phase: `ctas` persistent CTAs of `threads` threads with
// `smem` bytes of dynamic shared memory for the items' tiles (the launch adds
// kBatchSmemHeader) over `nitems` items; *next must be 0.
// Host-emulation builds run the items in order on the CPU from the same
// arrays (host memory there).
template <typename T>
cudaError_t launch_batch(const TileArgs<T> *args, const int *kinds, const BatchItem *items, int nitems, int *next,
                         int threads, size_t smem, int ctas, cudaStream_t s);

// Persistent CTAs the device holds at once for a launch shape (0 on error).
template <typename T>
int batch_resident_ctas(int threads, size_t smem);

}  // namespace ffb
