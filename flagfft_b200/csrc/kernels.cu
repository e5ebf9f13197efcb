// Dispatch of the on-chip FFT passes (the kernel bodies are in tile_impl.cuh,
// instantiated per precision and core kind in k_*.cu) and the elementwise
// real-transform pre/post kernels.
#include <algorithm>
#include <cstring>

#include "kernels.cuh"
#include "rows.cuh"

namespace ffb {

namespace tile {
// defined in k_*.cu
template <typename T, int K>
cudaError_t launch_group(const TileArgs<T> &a, int io, size_t smem, cudaStream_t s);
template <typename T, int K, bool INV>
cudaError_t launch_pp(const TileArgs<T> &a, size_t smem, cudaStream_t s);
template <typename T, int KIND, bool INV>
cudaError_t launch_pp_fixed_any(const TileArgs<T> &a, size_t smem, cudaStream_t s);
template <typename T, int KIND, int IO>
cudaError_t launch_one(const TileArgs<T> &a, size_t smem, cudaStream_t s);
}  // namespace tile

namespace rows {
// defined in k_*_rows*.cu
template <typename T, int KIND, bool INV>
cudaError_t launch_rows_any(const TileArgs<T> &a, size_t smem, cudaStream_t s);
}  // namespace rows

namespace {

// Pair (k, L-k), k = 0..L/2, of the Hermitian post-processing: from both Z
// values, both X values (k = 0: X_0 and X_L from Z_0).
template <typename T>
FFB_HD void real_post_vals(cpx<T> zk, cpx<T> zm, int L, int k, const RealTw<T> &rtw, cpx<T> &xk, cpx<T> &xm) {
  auto post = [&](cpx<T> a, cpx<T> b, int kk) {
    cpx<T> ev = mk((a.x + b.x) * (T)0.5, (a.y - b.y) * (T)0.5);
    cpx<T> od = mk((a.y + b.y) * (T)0.5, (b.x - a.x) * (T)0.5);
    return ev + cmul(real_tw(rtw, (uint32_t)kk), od);
  };
  xk = post(zk, zm, k);
  xm = post(zm, zk, L - k);
}
// One thread per pair: reads both Z values, writes both X values, so z and
// x may alias.
template <typename T>
FFB_HD void real_post_pair(const cpx<T> *z, cpx<T> *x, int L, int k, const RealTw<T> &rtw) {
  const int m = L - k;
  cpx<T> xk, xm;
  real_post_vals<T>(z[k], z[k == 0 ? 0 : m], L, k, rtw, xk, xm);
  x[k] = xk;
  if (m != k) x[m] = xm;
}

// Pair (k, L-k) of the Hermitian pre-processing: Z_k and Z_{L-k} from X_k
// and X_{L-k} (Z_0 from X_0 and X_L; Im X_0 and Im X_L ignored).
template <typename T>
FFB_HD void real_pre_vals(cpx<T> xk, cpx<T> xm, int L, int k, const RealTw<T> &rtw, cpx<T> &zk, cpx<T> &zm) {
  auto pre = [&](cpx<T> a, cpx<T> b, int kk) {  // a = X_kk, b = X_{L-kk}
    const cpx<T> s = mk(a.x + b.x, a.y - b.y);
    const cpx<T> d = mk(a.x - b.x, a.y + b.y);
    const cpx<T> w = real_tw(rtw, (uint32_t)kk);
    const cpx<T> dw = mk(d.x * w.x + d.y * w.y, d.y * w.x - d.x * w.y);
    return mk(s.x - dw.y, s.y + dw.x);
  };
  if (k == 0) {
    xk.y = (T)0;
    xm.y = (T)0;
  }
  zk = pre(xk, xm, k);
  zm = pre(xm, xk, L - k);
}
template <typename T>
FFB_HD void real_pre_pair(const cpx<T> *x, cpx<T> *z, int L, int k, const RealTw<T> &rtw) {
  const int m = L - k;
  cpx<T> zk, zm;
  real_pre_vals<T>(x[k], x[m], L, k, rtw, zk, zm);
  z[k] = zk;
  if (m != k && m < L) z[m] = zm;
}

#ifndef FFB_HOST_EMULATION

constexpr int kRealThreads = 256, kRealUnroll = 4;

// U pairs per thread, k = k0 + u * stride: every load of the U pairs issued
// before the first store (bytes in flight), pairs of one thread disjoint
// from every other thread's, so the passes may run in place.
template <typename T>
__global__ void __launch_bounds__(kRealThreads) k_real_post(const cpx<T> *z, cpx<T> *x, long long zdist,
                                                            long long xdist, int L, const RealTw<T> rtw) {
  pdl_entry();
  const long long b = blockIdx.y;
  z += b * zdist;
  x += b * xdist;
  const int stride = gridDim.x * blockDim.x, half = L / 2;
  for (int k0 = blockIdx.x * blockDim.x + threadIdx.x; k0 <= half; k0 += kRealUnroll * stride) {
    cpx<T> a[kRealUnroll], c[kRealUnroll];
#pragma unroll
    for (int u = 0; u < kRealUnroll; ++u) {
      const int k = k0 + u * stride;
      if (k <= half) {
        a[u] = z[k];
        c[u] = z[k == 0 ? 0 : L - k];
      }
    }
#pragma unroll
    for (int u = 0; u < kRealUnroll; ++u) {
      const int k = k0 + u * stride;
      if (k <= half) {
        cpx<T> xk, xm;
        real_post_vals<T>(a[u], c[u], L, k, rtw, xk, xm);
        x[k] = xk;
        if (L - k != k) x[L - k] = xm;
      }
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(kRealThreads) k_real_pre(const cpx<T> *x, cpx<T> *z, long long xdist,
                                                           long long zdist, int L, const RealTw<T> rtw) {
  pdl_entry();
  const long long b = blockIdx.y;
  x += b * xdist;
  z += b * zdist;
  const int stride = gridDim.x * blockDim.x, half = L / 2;
  for (int k0 = blockIdx.x * blockDim.x + threadIdx.x; k0 <= half; k0 += kRealUnroll * stride) {
    cpx<T> a[kRealUnroll], c[kRealUnroll];
#pragma unroll
    for (int u = 0; u < kRealUnroll; ++u) {
      const int k = k0 + u * stride;
      if (k <= half) {
        a[u] = x[k];
        c[u] = x[L - k];
      }
    }
#pragma unroll
    for (int u = 0; u < kRealUnroll; ++u) {
      const int k = k0 + u * stride;
      if (k <= half) {
        cpx<T> zk, zm;
        real_pre_vals<T>(a[u], c[u], L, k, rtw, zk, zm);
        z[k] = zk;
        if (L - k != k && L - k < L) z[L - k] = zm;
      }
    }
  }
}

#endif  // !FFB_HOST_EMULATION

template <typename T>
__global__ void __launch_bounds__(256) k_transpose(const cpx<T> *in, cpx<T> *out, long long R, long long C,
                                                   long long sdist, long long ddist, const SplitTw<T> tw) {
  pdl_entry();
  __shared__ cpx<T> tile[32][33];
  const long long b = blockIdx.z;
  const long long r0 = (long long)blockIdx.y * 32, c0 = (long long)blockIdx.x * 32;
  in += b * sdist;
  out += b * ddist;
#pragma unroll
  for (int i = threadIdx.y; i < 32; i += 8) {
    const long long r = r0 + i, c = c0 + threadIdx.x;
    if (r < R && c < C) {
      cpx<T> v = in[r * C + c];
      if (tw.lo) {
        const uint32_t m = (uint32_t)(r * c), hi = fdiv(m, tw.split);
        cpx<T> w = cmul(ldg_c(tw.hi + hi), ldg_c(tw.lo + (m - hi * tw.split.d)));
        if (tw.inv) w.y = -w.y;
        v = cmul(v, w);
      }
      tile[i][threadIdx.x] = v;
    }
  }
  __syncthreads();
#pragma unroll
  for (int i = threadIdx.y; i < 32; i += 8) {
    const long long c = c0 + i, r = r0 + threadIdx.x;
    if (r < R && c < C) out[c * R + r] = tile[threadIdx.x][i];
  }
}

// One Rader chain step for element q of row b (see launch_rader_step).
template <typename T>
FFB_HD void rader_step_one(int mode, const cpx<T> *x, cpx<T> *ws, cpx<T> *y, long long batch, long long p,
                           long long xdist, long long ydist, const int *perm, const cpx<T> *kern, long long b,
                           long long q) {
  const long long m = p - 1;
  cpx<T> *w = ws + b * m;
  cpx<T> *x0 = ws + batch * m + b, *a0 = ws + batch * m + batch + b;
  if (mode == 0) {
    w[q] = x[b * xdist + perm[q]];
    if (q == 0) *x0 = x[b * xdist];
  } else if (mode == 1) {
    const cpx<T> v = w[q];
    if (q == 0) *a0 = v;
    const cpx<T> t = cmul(v, ldg_c(kern + q));
    w[q] = mk(t.x, -t.y);
  } else {
    const cpx<T> base = *x0, v = w[q];
    y[b * ydist + perm[q]] = mk(base.x + v.x, base.y - v.y);
    if (q == 0) y[b * ydist] = base + *a0;
  }
}

#ifndef FFB_HOST_EMULATION
template <typename T>
__global__ void __launch_bounds__(256) k_rader_step(int mode, const cpx<T> *x, cpx<T> *ws, cpx<T> *y,
                                                    long long batch, long long p, long long xdist, long long ydist,
                                                    const int *perm, const cpx<T> *kern) {
  pdl_entry();
  const long long b = blockIdx.y;
  for (long long q = (long long)blockIdx.x * blockDim.x + threadIdx.x; q < p - 1; q += (long long)gridDim.x * blockDim.x)
    rader_step_one<T>(mode, x, ws, y, batch, p, xdist, ydist, perm, kern, b, q);
}
#endif

}  // namespace

template <typename T>
cudaError_t launch_transpose(const cpx<T> *in, cpx<T> *out, long long batch, long long R, long long C,
                             cudaStream_t s, long long sdist, long long ddist, const SplitTw<T> &tw) {
  if (batch <= 0 || R <= 0 || C <= 0) return cudaSuccess;
  if ((R + 31) / 32 > 65535 || batch > 65535) return cudaErrorInvalidValue;
  if (sdist == 0) sdist = R * C;
  if (ddist == 0) ddist = R * C;
#ifndef FFB_HOST_EMULATION
  return launch_pdl(k_transpose<T>, dim3((unsigned)((C + 31) / 32), (unsigned)((R + 31) / 32), (unsigned)batch),
                    dim3(32, 8), 0, s, in, out, R, C, sdist, ddist, tw);
#else
  (void)s;
  for (long long b = 0; b < batch; ++b)
    for (long long r = 0; r < R; ++r)
      for (long long c = 0; c < C; ++c) {
        cpx<T> v = in[b * sdist + r * C + c];
        if (tw.lo) {
          const uint32_t m = (uint32_t)(r * c), hi = fdiv(m, tw.split);
          cpx<T> w = cmul(tw.hi[hi], tw.lo[m - hi * tw.split.d]);
          if (tw.inv) w.y = -w.y;
          v = cmul(v, w);
        }
        out[b * ddist + c * R + r] = v;
      }
  return cudaSuccess;
#endif
}

template <typename T>
cudaError_t launch_rader_step(int mode, const cpx<T> *x, cpx<T> *ws, cpx<T> *y, long long batch, long long p,
                              long long xdist, long long ydist, const int *perm, const cpx<T> *kern,
                              cudaStream_t s) {
  if (batch <= 0 || p < 3) return cudaSuccess;
  if (batch > 65535) return cudaErrorInvalidValue;
#ifndef FFB_HOST_EMULATION
  const unsigned blocks = (unsigned)std::min<long long>((p - 1 + 255) / 256, 4096);
  return launch_pdl(k_rader_step<T>, dim3(blocks, (unsigned)batch), dim3(256), 0, s, mode, x, ws, y, batch, p, xdist,
                    ydist, perm, kern);
#else
  (void)s;
  for (long long b = 0; b < batch; ++b)
    for (long long q = 0; q < p - 1; ++q) rader_step_one<T>(mode, x, ws, y, batch, p, xdist, ydist, perm, kern, b, q);
  return cudaSuccess;
#endif
}

template cudaError_t launch_rader_step<float>(int, const cpx<float> *, cpx<float> *, cpx<float> *, long long,
                                              long long, long long, long long, const int *, const cpx<float> *,
                                              cudaStream_t);
template cudaError_t launch_rader_step<double>(int, const cpx<double> *, cpx<double> *, cpx<double> *, long long,
                                               long long, long long, long long, const int *, const cpx<double> *,
                                               cudaStream_t);

template cudaError_t launch_transpose<float>(const cpx<float> *, cpx<float> *, long long, long long, long long,
                                             cudaStream_t, long long, long long, const SplitTw<float> &);
template cudaError_t launch_transpose<double>(const cpx<double> *, cpx<double> *, long long, long long, long long,
                                              cudaStream_t, long long, long long, const SplitTw<double> &);

template <typename T>
cudaError_t launch_real_post(const cpx<T> *z, cpx<T> *x, long long batch, long long zdist, long long xdist, int L,
                             const RealTw<T> &rtw, cudaStream_t s) {
#ifndef FFB_HOST_EMULATION
  const int per = kRealThreads * kRealUnroll;
  const int blocks = (int)std::min<long long>((L / 2 + per) / per, 2048);
  return launch_pdl(k_real_post<T>, dim3(blocks, (unsigned)batch), dim3(kRealThreads), 0, s, z, x, zdist, xdist, L,
                    rtw);
#else
  for (long long b = 0; b < batch; ++b)
    for (int k = 0; k <= L / 2; ++k) real_post_pair<T>(z + b * zdist, x + b * xdist, L, k, rtw);
  return cudaSuccess;
#endif
}

template <typename T>
cudaError_t launch_real_pre(const cpx<T> *x, cpx<T> *z, long long batch, long long xdist, long long zdist, int L,
                            const RealTw<T> &rtw, cudaStream_t s) {
#ifndef FFB_HOST_EMULATION
  const int per = kRealThreads * kRealUnroll;
  const int blocks = (int)std::min<long long>((L / 2 + per) / per, 2048);
  return launch_pdl(k_real_pre<T>, dim3(blocks, (unsigned)batch), dim3(kRealThreads), 0, s, x, z, xdist, zdist, L,
                    rtw);
#else
  for (long long b = 0; b < batch; ++b)
    for (int k = 0; k <= L / 2; ++k) real_pre_pair<T>(x + b * xdist, z + b * zdist, L, k, rtw);
  return cudaSuccess;
#endif
}

namespace {
template <typename T>
FFB_HD void real_convert_one(int mode, const void *src, void *dst, long long sdist, long long ddist, long long n,
                             long long b, long long k) {
  if (mode == 0) {
    const T *x = reinterpret_cast<const T *>(src) + b * sdist;
    reinterpret_cast<cpx<T> *>(dst)[b * ddist + k] = mk(x[k], (T)0);
  } else if (mode == 1) {
    reinterpret_cast<cpx<T> *>(dst)[b * ddist + k] = reinterpret_cast<const cpx<T> *>(src)[b * sdist + k];
  } else if (mode == 2) {
    const cpx<T> *X = reinterpret_cast<const cpx<T> *>(src) + b * sdist;
    cpx<T> v = k <= n / 2 ? X[k] : conjg(X[n - k]);
    if (k == 0 || (n % 2 == 0 && k == n / 2)) v.y = (T)0;
    reinterpret_cast<cpx<T> *>(dst)[b * ddist + k] = v;
  } else {
    reinterpret_cast<T *>(dst)[b * ddist + k] = reinterpret_cast<const cpx<T> *>(src)[b * sdist + k].x;
  }
}

template <typename T>
__global__ void k_real_convert(int mode, const void *src, void *dst, long long batch, long long sdist,
                               long long ddist, long long n, long long count) {
  pdl_entry();
  const long long b = blockIdx.y;
  for (long long k = (long long)blockIdx.x * blockDim.x + threadIdx.x; k < count; k += (long long)gridDim.x * blockDim.x)
    real_convert_one<T>(mode, src, dst, sdist, ddist, n, b, k);
}
}  // namespace

template <typename T>
cudaError_t launch_real_convert(int mode, const void *src, void *dst, long long batch, long long sdist,
                                long long ddist, long long n, cudaStream_t s) {
  const long long count = mode == 1 ? n / 2 + 1 : n;
#ifndef FFB_HOST_EMULATION
  const int threads = 256;
  const int blocks = (int)std::min<long long>((count + threads - 1) / threads, 2048);
  return launch_pdl(k_real_convert<T>, dim3(blocks, (unsigned)batch), dim3(threads), 0, s, mode, src, dst, batch, sdist,
                    ddist, n, count);
#else
  (void)s;
  for (long long b = 0; b < batch; ++b)
    for (long long k = 0; k < count; ++k) real_convert_one<T>(mode, src, dst, sdist, ddist, n, b, k);
  return cudaSuccess;
#endif
}

template cudaError_t launch_real_convert<float>(int, const void *, void *, long long, long long, long long, long long,
                                                cudaStream_t);
template cudaError_t launch_real_convert<double>(int, const void *, void *, long long, long long, long long, long long,
                                                 cudaStream_t);

template cudaError_t launch_real_post<float>(const cpx<float> *, cpx<float> *, long long, long long, long long, int,
                                             const RealTw<float> &, cudaStream_t);
template cudaError_t launch_real_post<double>(const cpx<double> *, cpx<double> *, long long, long long, long long,
                                              int, const RealTw<double> &, cudaStream_t);
template cudaError_t launch_real_pre<float>(const cpx<float> *, cpx<float> *, long long, long long, long long, int,
                                            const RealTw<float> &, cudaStream_t);
template cudaError_t launch_real_pre<double>(const cpx<double> *, cpx<double> *, long long, long long, long long,
                                             int, const RealTw<double> &, cudaStream_t);

template <typename T>
cudaError_t launch_tile(const TileArgs<T> &a, CoreKind kind, IoKind io, size_t smem, cudaStream_t s) {
  const int k = (int)kind, o = (int)io;
  if (a.regcol) return launch_regcol<T>(a, s);
  if (a.blue_cols) return launch_blue4<T>(a, s);
  if (a.tcols) {
    const cudaError_t e = launch_tcols<T>(a, s);
    if (e != cudaErrorNotSupported) return e;  // else: buffers off the copy rules, the tile kernels below
  }
  if (a.tiles) return launch_tiles<T>(a, s);
  if (a.pp && o == 0) {
    // compile-time radix sequences first: contiguous rows, then any layout
    // (cudaErrorNotSupported: no kernel for this pass)
    if (k == 0 || k == 1 || k == 3) {
      const cudaError_t e = k == 0 ? (a.inv ? rows::launch_rows_any<T, 0, true>(a, smem, s)
                                            : rows::launch_rows_any<T, 0, false>(a, smem, s))
                            : k == 1 ? rows::launch_rows_any<T, 1, false>(a, smem, s)
                                     : rows::launch_rows_any<T, 3, false>(a, smem, s);
      if (e != cudaErrorNotSupported) return e;
    }
    if (a.rows_only) return cudaErrorInvalidConfiguration;  // no general tile fits its shared memory
    if (k == 0 || k == 1 || k == 3) {
      const cudaError_t e = k == 0 ? (a.inv ? tile::launch_pp_fixed_any<T, 0, true>(a, smem, s)
                                            : tile::launch_pp_fixed_any<T, 0, false>(a, smem, s))
                            : k == 1 ? tile::launch_pp_fixed_any<T, 1, false>(a, smem, s)
                                     : tile::launch_pp_fixed_any<T, 3, false>(a, smem, s);
      if (e != cudaErrorNotSupported) return e;
    }
    switch (k) {
      case 0: return a.inv ? tile::launch_pp<T, 0, true>(a, smem, s) : tile::launch_pp<T, 0, false>(a, smem, s);
      case 1: return tile::launch_pp<T, 1, false>(a, smem, s);
      case 2: return tile::launch_pp<T, 2, false>(a, smem, s);
      case 3: return tile::launch_pp<T, 3, false>(a, smem, s);
      default: return cudaErrorInvalidValue;
    }
  }
  if (k == 3 && o == 0) return tile::launch_one<T, 3, 0>(a, smem, s);
  if (k == 0 && (o == 5 || o == 6)) return o == 5 ? tile::launch_one<T, 0, 5>(a, smem, s) : tile::launch_one<T, 0, 6>(a, smem, s);
  if (k == 0) return tile::launch_group<T, 0>(a, o, smem, s);
  if (k == 1) return tile::launch_group<T, 1>(a, o, smem, s);
  if (k == 2) return tile::launch_group<T, 2>(a, o, smem, s);
  return cudaErrorInvalidValue;
}

template <typename T>
size_t tile_smem(const TileArgs<T> &a, CoreKind kind, IoKind io, size_t smem) {
  const int k = (int)kind;
  if (a.regcol) return 0;
  if (a.blue_cols) return blue4_smem(a.blue_cols, a.core.L, sizeof(cpx<T>), a.blue_pair != 0);
  if (a.tiles) return smem;
  if (a.pp && io == IoKind::C2C && (k == 0 || k == 1 || k == 3)) {
    const size_t r = k == 0 ? rows::rows_smem_any<T, 0>(a) : k == 1 ? rows::rows_smem_any<T, 1>(a)
                                                                     : rows::rows_smem_any<T, 3>(a);
    if (r) return r;
  }
  return smem;
}

template size_t tile_smem<float>(const TileArgs<float> &, CoreKind, IoKind, size_t);
template size_t tile_smem<double>(const TileArgs<double> &, CoreKind, IoKind, size_t);
template cudaError_t launch_tile<float>(const TileArgs<float> &, CoreKind, IoKind, size_t, cudaStream_t);
template cudaError_t launch_tile<double>(const TileArgs<double> &, CoreKind, IoKind, size_t, cudaStream_t);

}  // namespace ffb
