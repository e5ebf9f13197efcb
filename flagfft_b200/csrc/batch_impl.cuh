// Definitions of the batch launchers, instantiated per precision in
// k_f32_batch.cu / k_f64_batch.cu.
#pragma once

#include <map>
#include <mutex>
#include <tuple>

#include "batch.cuh"

namespace ffb {

#ifndef FFB_HOST_EMULATION
template <typename T>
static cudaError_t batch_configure() {
  return set_smem_limit_once<batch::k_batch<T>>(232448);
}

template <typename T>
cudaError_t launch_batch(const TileArgs<T> *args, const int *kinds, const BatchItem *items, int nitems, int *next,
                         int threads, size_t smem, int ctas, cudaStream_t s) {
  cudaError_t e = batch_configure<T>();
  if (e != cudaSuccess) return e;
  // a persistent grid fills every SM: launched with programmatic dependence
  // its CTAs would take their slots as soon as the previous grid runs, so it
  // launches plainly (its pdl_entry instructions are then no-ops)
  PdlOff off;
  return launch_pdl(batch::k_batch<T>, dim3(ctas), dim3(threads), smem + kBatchSmemHeader, s, args, kinds, items,
                    nitems, next);
}

template <typename T>
int batch_resident_ctas(int threads, size_t smem) {
  if (batch_configure<T>() != cudaSuccess) return 0;
  // the occupancy query costs microseconds and a server asks it for every
  // launch of every tick: remember the answer per (device, threads, smem)
  static std::mutex mu;
  static std::map<std::tuple<int, int, size_t>, int> memo;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  const auto key = std::make_tuple(dev, threads, smem);
  {
    std::lock_guard<std::mutex> lock(mu);
    auto it = memo.find(key);
    if (it != memo.end()) return it->second;
  }
  int per_sm = 0, sms = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, batch::k_batch<T>, threads, smem + kBatchSmemHeader) !=
          cudaSuccess ||
      cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) {
    cudaGetLastError();
    return 0;
  }
  std::lock_guard<std::mutex> lock(mu);
  memo[key] = per_sm * sms;
  return per_sm * sms;
}
#else
// Sequential host run: the ping-pong bodies with one "thread" per slot
// (HostX), every transform of a register-column chunk in turn.
template <typename T>
cudaError_t launch_batch(const TileArgs<T> *args, const int *kinds, const BatchItem *items, int nitems, int *next,
                         int threads, size_t smem, int, cudaStream_t) {
  std::vector<unsigned char> buf(smem + 64);
  cpx<T> *sm = reinterpret_cast<cpx<T> *>(buf.data());
  for (int i = *next; i < nitems; ++i) {
    const BatchItem w = items[i];
    const TileArgs<T> &a = args[w.args];
    if (kinds[w.args] == kBatchRegcol) {
      const int chunks = (a.G + threads - 1) / threads;
      const int by = w.tile / chunks;
      for (int t = 0; t < threads; ++t) {
        const long long g = (long long)(w.tile - by * chunks) * threads + t;
        if (g >= a.G) break;
        if (a.inv)
          batch::regcol_one<T, true>(a, by, g);
        else
          batch::regcol_one<T, false>(a, by, g);
      }
    } else {
      std::memset(buf.data(), 0xff, buf.size());
      batch::run_item<T>(a, kinds[w.args], w.tile, sm, tile::HostX{});
    }
  }
  *next = nitems;
  return cudaSuccess;
}

template <typename T>
int batch_resident_ctas(int, size_t) {
  return 1;
}
#endif

}  // namespace ffb
