// Host side of the TMA column passes (tcols.cuh): tile views, tensor-map
// encoding and launch, instantiated per precision in k_f32_tcols.cu /
// k_f64_tcols.cu.  The host-emulation build runs the same group loop on the
// CPU with the copies done by hand (tma::emulate_box).
#pragma once

#include <cmath>
#include <mutex>
#include <vector>

#include "tcols.cuh"

namespace ffb {
namespace tcols {

// Sequences with a TMA column kernel.
#define FFB_TCOLS_SEQUENCES(X) \
  X(1024, 16, 16, 4)           \
  X(1536, 16, 16, 6)           \
  X(2048, 16, 16, 8)           \
  X(4096, 16, 16, 16)

// Tile views of one side of a pass: "rows" when a transform's elements are
// contiguous (stride 1), "columns" when the transforms are adjacent (stride
// 1 between transforms).  False when neither, or when a stride or the base
// breaks TMA's 16-byte rules.
template <typename T, int L, int GC, int RB>
bool make_view(const void *base, long long nbatch, long long G, long long b_stride, long long g_stride,
               long long e_stride, tma::View *v, int *is_rows) {
  const unsigned long long es = sizeof(cpx<T>);
  *v = tma::View{};
  v->base = const_cast<void *>(base);
  v->scalar_bytes = (int)sizeof(T);
  if (reinterpret_cast<uintptr_t>(base) % 16 != 0) return false;
  if (G <= 0 || nbatch <= 0 || 2 * G >= (1ll << 31) || nbatch >= (1ll << 31)) return false;
  if (e_stride == 1 && g_stride >= L) {
    *is_rows = 1;
    v->dims[0] = 256;  // 128 complex elements, in scalars
    v->dims[1] = L / 128;
    v->dims[2] = (unsigned long long)G;
    v->dims[3] = (unsigned long long)nbatch;
    v->strides[0] = 128 * es;
    v->strides[1] = (unsigned long long)g_stride * es;
    v->strides[2] = nbatch > 1 ? (unsigned long long)b_stride * es : v->strides[1] * v->dims[2];
    v->box[0] = 256;
    v->box[1] = L / 128;
    v->box[2] = GC;
    v->box[3] = 1;
  } else if (g_stride == 1 && e_stride >= G) {
    // element i = i_hi * RB + i_lo: the whole GC x L tile is one box
    // (boxes are at most 256 per dimension), laid out [i_hi][i_lo][c]
    *is_rows = 0;
    v->dims[0] = 2 * (unsigned long long)G;
    v->dims[1] = RB;
    v->dims[2] = L / RB;
    v->dims[3] = (unsigned long long)nbatch;
    v->strides[0] = (unsigned long long)e_stride * es;
    v->strides[1] = v->strides[0] * RB;
    v->strides[2] = nbatch > 1 ? (unsigned long long)b_stride * es : v->strides[1] * (L / RB);
    v->box[0] = 2 * GC;
    v->box[1] = RB;
    v->box[2] = L / RB;
    v->box[3] = 1;
  } else {
    return false;
  }
  for (int i = 0; i < 3; ++i)
    if (v->strides[i] % 16 != 0 || v->strides[i] >= (1ull << 40) || v->strides[i] == 0) return false;
  return true;
}

template <typename T, int L, int GC, int RB>
bool make_views(const TileArgs<T> &a, Args<T> *p) {
  int in_rows = 0, out_rows = 0;
  if (!make_view<T, L, GC, RB>(a.in, a.nbatch, a.G, a.ib, a.ig, a.ii, &p->in_view, &in_rows)) return false;
  if (!make_view<T, L, GC, RB>(a.out, a.nbatch, a.G, a.ob, a.og, a.ok, &p->out_view, &out_rows)) return false;
  if (in_rows && out_rows) return false;  // a row pass: the row kernels take it
  p->in_rows = in_rows;
  p->out_rows = out_rows;
  p->a = a;
  p->groups_per_batch = (a.G + GC - 1) / GC;
  p->total_groups = p->groups_per_batch * a.nbatch;
  return true;
}

#ifndef FFB_HOST_EMULATION

using EncodeTiled = CUresult (*)(CUtensorMap *, CUtensorMapDataType, cuuint32_t, void *, const cuuint64_t *,
                                 const cuuint64_t *, const cuuint32_t *, const cuuint32_t *, CUtensorMapInterleave,
                                 CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

// cuTensorMapEncodeTiled through the runtime's driver entry point (the
// library does not link libcuda directly).
inline EncodeTiled encode_fn() {
  static EncodeTiled fn = nullptr;
  static std::once_flag once;
  std::call_once(once, []() {
    void *p = nullptr;
    cudaDriverEntryPointQueryResult q{};
    if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) == cudaSuccess &&
        q == cudaDriverEntryPointSuccess)
      fn = reinterpret_cast<EncodeTiled>(p);
  });
  return fn;
}

template <typename T>
bool encode(const tma::View &v, CUtensorMap *map) {
  EncodeTiled fn = encode_fn();
  if (!fn) return false;
  const cuuint32_t estr[4] = {1, 1, 1, 1};
  const CUresult r = fn(map, sizeof(T) == 4 ? CU_TENSOR_MAP_DATA_TYPE_FLOAT32 : CU_TENSOR_MAP_DATA_TYPE_FLOAT64, 4,
                        v.base, reinterpret_cast<const cuuint64_t *>(v.dims),
                        reinterpret_cast<const cuuint64_t *>(v.strides), reinterpret_cast<const cuuint32_t *>(v.box),
                        estr, CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                        CU_TENSOR_MAP_L2_PROMOTION_L2_256B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
  return r == CUDA_SUCCESS;
}

inline int sm_count() {
  int dev = 0, n = 0;
  if (cudaGetDevice(&dev) != cudaSuccess || cudaDeviceGetAttribute(&n, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess)
    return 148;
  return n > 0 ? n : 148;
}

template <typename T, bool INV, int L, int... Rs>
cudaError_t launch_seq(const TileArgs<T> &a, cudaStream_t s) {
  using Sh = Shape<T, L, Rs...>;
  Args<T> p{};
  if (!make_views<T, L, Sh::GC, Sh::RB>(a, &p)) return cudaErrorNotSupported;
  if (!encode<T>(p.in_view, &p.in_map) || !encode<T>(p.out_view, &p.out_map)) return cudaErrorNotSupported;
  const long long ctas = std::min<long long>(p.total_groups, sm_count());
  cudaError_t e;
#define FFB_TCOLS_GO(IR, OR)                                                             \
  {                                                                                      \
    auto k = k_tcols<T, INV, L, IR, OR, Rs...>;                                          \
    if ((e = set_smem_limit_once<k_tcols<T, INV, L, IR, OR, Rs...>>((int)Sh::smem)) != cudaSuccess) return e; \
    if ((e = launch_pdl(k, dim3((unsigned)ctas), dim3(Sh::NT), Sh::smem, s, p)) != cudaSuccess) return e; \
  }
  if (p.in_rows)
    FFB_TCOLS_GO(true, false)
  else if (p.out_rows)
    FFB_TCOLS_GO(false, true)
  else
    FFB_TCOLS_GO(false, false)
#undef FFB_TCOLS_GO
  return cudaGetLastError();
}

#else  // FFB_HOST_EMULATION

template <typename T, bool INV, int L, bool IR, bool OR, int... Rs>
void emulate(const Args<T> &p) {
  using Sh = Shape<T, L, Rs...>;
  using Q = Seq<Rs...>;
  // the shared-memory image of the kernel: a 1 KB head, then NBUF ring
  // slots, the group q in slot q % NBUF
  std::vector<unsigned char> image(Sh::smem + 1024);
  unsigned char *base = image.data() + (1024 - (reinterpret_cast<uintptr_t>(image.data()) & 1023));
  cpx<T> *const ring = reinterpret_cast<cpx<T> *>(base + Sh::head);
  const cpx<T> *tw = p.a.tw;
  if constexpr (Sh::TWS != rows::TW_GLOBAL) {  // the kernel's shared-memory table, filled as its threads do
    cpx<T> *tws = reinterpret_cast<cpx<T> *>(base + Sh::tw_at);
    for (int t = 0; t < Sh::NT; ++t) fill_twiddles<T, Sh, Q>(tws, p.a.tw, t);
    tw = tws;
  }
  for (long long q = 0; q < p.total_groups; ++q) {
    const Group gr = group_of<Sh::GC>(q, p.groups_per_batch);
    cpx<T> *const raw = ring + (size_t)(q % Sh::NBUF) * Sh::buf_elems;
    std::fill(raw, raw + Sh::raw_elems, mk((T)NAN, (T)NAN));
    if (IR)
      tma::emulate_box(p.in_view, 0, 0, (int)gr.g0, (int)gr.b, raw, true);
    else
      tma::emulate_box(p.in_view, (int)(2 * gr.g0), 0, 0, (int)gr.b, raw, true);
    run_stages<T, INV, L, Sh, Q, 0, IR, OR, Sh::TWS>(rows::HostT{}, p.a, tw, raw, gr.g0);
    if (OR)
      tma::emulate_box(p.out_view, 0, 0, (int)gr.g0, (int)gr.b, raw, false);
    else
      tma::emulate_box(p.out_view, (int)(2 * gr.g0), 0, 0, (int)gr.b, raw, false);
  }
}

template <typename T, bool INV, int L, int... Rs>
cudaError_t launch_seq(const TileArgs<T> &a, cudaStream_t) {
  using Sh = Shape<T, L, Rs...>;
  Args<T> p{};
  if (!make_views<T, L, Sh::GC, Sh::RB>(a, &p)) return cudaErrorNotSupported;
  if (p.in_rows)
    emulate<T, INV, L, true, false, Rs...>(p);
  else if (p.out_rows)
    emulate<T, INV, L, false, true, Rs...>(p);
  else
    emulate<T, INV, L, false, false, Rs...>(p);
  return cudaSuccess;
}

#endif

// Launch for a pass whose core is one of the TMA column sequences;
// cudaErrorNotSupported when the pass or its buffers do not fit the views
// (the caller then runs the plain tile kernels).
template <typename T>
cudaError_t launch_any(const TileArgs<T> &a, cudaStream_t s) {
  if (a.chirp_mode != 0 || a.nbatch <= 0) return cudaErrorNotSupported;
#define FFB_TCOLS_TRY(L, ...)                                                                                   \
  if (tile::core_is<L, __VA_ARGS__>(a.core))                                                                  \
    return a.inv ? launch_seq<T, true, L, __VA_ARGS__>(a, s) : launch_seq<T, false, L, __VA_ARGS__>(a, s);
  FFB_TCOLS_SEQUENCES(FFB_TCOLS_TRY)
#undef FFB_TCOLS_TRY
  return cudaErrorNotSupported;
}

// Whether a pass of length L with these strides can take the TMA column
// kernel (buffer addresses are checked at launch).
template <typename T>
bool eligible(int L, long long nbatch, long long G, long long ib, long long ig, long long ii, long long ob,
              long long og, long long ok, int *threads, size_t *smem) {
#define FFB_TCOLS_ELIG(L_, ...)                                                                          \
  if (L == (L_)) {                                                                                     \
    using Sh = Shape<T, L_, __VA_ARGS__>;                                                               \
    tma::View v;                                                                                       \
    int ir = 0, orr = 0;                                                                               \
    alignas(16) static const unsigned char probe[16] = {};                                            \
    if (G < Sh::GC) return false;                                                                      \
    if (!make_view<T, L_, Sh::GC, Sh::RB>(probe, nbatch, G, ib, ig, ii, &v, &ir)) return false;         \
    if (!make_view<T, L_, Sh::GC, Sh::RB>(probe, nbatch, G, ob, og, ok, &v, &orr)) return false;        \
    if (ir && orr) return false;                                                                       \
    *threads = Sh::NT;                                                                                 \
    *smem = Sh::smem;                                                                                  \
    return true;                                                                                       \
  }
  FFB_TCOLS_SEQUENCES(FFB_TCOLS_ELIG)
#undef FFB_TCOLS_ELIG
  return false;
}

}  // namespace tcols
}  // namespace ffb
