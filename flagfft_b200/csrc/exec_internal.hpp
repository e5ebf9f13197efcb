// Pass types of a lowered program, shared by the executor (exec.cpp) and
// the request server (serve.cpp).
#pragma once

#include <memory>
#include <sstream>
#include <string>

#include "exec.hpp"

namespace ffb {

inline const char *buf_name(Buf b) {
  switch (b) {
    case Buf::In: return "in";
    case Buf::Out: return "out";
    case Buf::Scratch0: return "ws0";
    case Buf::Scratch1: return "ws1";
  }
  return "?";
}

inline const char *kind_name(CoreKind k) {
  switch (k) {
    case CoreKind::Dit: return "stockham-dit";
    case CoreKind::Bluestein: return "bluestein-fused";
    case CoreKind::Rader: return "rader-fused";
    case CoreKind::Conv: return "convolution-rows";
  }
  return "?";
}

inline const char *io_name(IoKind k) {
  switch (k) {
    case IoKind::C2C: return "c2c";
    case IoKind::R2C: return "r2c-halfpack";
    case IoKind::C2R: return "c2r-halfpack";
    case IoKind::R2CFull: return "r2c-full";
    case IoKind::C2RFull: return "c2r-full";
    case IoKind::PackC2C: return "real-pairs-in";
    case IoKind::C2CUnpack: return "real-pairs-out";
  }
  return "?";
}

template <typename T>
struct TilePass final : PassBase {
  TileArgs<T> a{};
  CoreKind kind = CoreKind::Dit;
  IoKind io = IoKind::C2C;
  size_t smem = 0;
  Buf src = Buf::In, dst = Buf::Out;
  std::string note;

  static void *pick(Buf b, const void *in, void *out, void *s0, void *s1) {
    switch (b) {
      case Buf::In: return const_cast<void *>(in);
      case Buf::Out: return out;
      case Buf::Scratch0: return s0;
      case Buf::Scratch1: return s1;
    }
    return nullptr;
  }

  cudaError_t run(const void *in, void *out, void *s0, void *s1, cudaStream_t st) const override {
    TileArgs<T> b = a;
    b.in = pick(src, in, out, s0, s1);
    b.out = pick(dst, in, out, s0, s1);
    return launch_tile<T>(b, kind, io, smem, st);
  }

  std::string describe() const override {
    std::ostringstream o;
    o << (a.regcol ? "register-columns" : a.blue_pair ? "bluestein-four-step-pair" : a.blue_cols ? "bluestein-four-step" : kind_name(kind)) << "/" << io_name(io)
      << " "
      << (sizeof(T) == 4 ? "f32" : "f64") << " L=" << a.core.L
      << " radices=[";
    for (int s = 0; s < a.core.nst; ++s) o << (s ? "," : "") << a.core.radix[s];
    o << "] n=" << a.n << " transforms=" << a.nbatch << "x" << a.G << " per_cta=" << a.W
      << " threads=" << (a.blue_cols ? blue4_threads(a.blue_cols, a.core.L, a.blue_pair != 0) : a.tiles ? a.tpt : a.W * a.tpt)
      << (a.tiles ? " tiles" : "") << " smem=" << tile_smem<T>(a, kind, io, smem) << " " << buf_name(src) << "->"
      << buf_name(dst);
    if (a.tcols) o << " tma-columns(threads=" << a.tc_threads << " smem=" << a.tc_smem << ")";
    if (a.post_twiddle) o << " +twiddle";
    if (!note.empty()) o << " (" << note << ")";
    return o.str();
  }
};

// Elementwise real-transform post (Z -> half spectrum) or pre (half spectrum
// -> Z) processing between the passes of a multi-pass R2C / C2R.
template <typename T>
struct RealPass final : PassBase {
  bool post;
  Buf src, dst;
  long long batch, sdist, ddist;
  int L;
  RealTw<T> rtw;
  RealPass(bool post_, Buf s, Buf d, long long b, long long sd, long long dd, int64_t L_, const RealTw<T> &r)
      : post(post_), src(s), dst(d), batch(b), sdist(sd), ddist(dd), L((int)L_), rtw(r) {}
  cudaError_t run(const void *in, void *out, void *s0, void *s1, cudaStream_t st) const override {
    auto *sp = reinterpret_cast<const cpx<T> *>(TilePass<T>::pick(src, in, out, s0, s1));
    auto *dp = reinterpret_cast<cpx<T> *>(TilePass<T>::pick(dst, in, out, s0, s1));
    return post ? launch_real_post<T>(sp, dp, batch, sdist, ddist, L, rtw, st)
                : launch_real_pre<T>(sp, dp, batch, sdist, ddist, L, rtw, st);
  }
  std::shared_ptr<PassBase> rebatched(long long from, long long to) const override {
    auto q = std::make_shared<RealPass<T>>(*this);
    q->batch = batch / from * to;
    return q;
  }
  std::string describe() const override {
    std::ostringstream o;
    o << (post ? "real-post" : "real-pre") << " " << (sizeof(T) == 4 ? "f32" : "f64") << " L=" << L
      << " transforms=" << batch << " " << buf_name(src) << "->" << buf_name(dst);
    return o.str();
  }
};

// Axis exchange between passes: (batch, R, C) -> (batch, C, R), matrix b at
// b * sdist / b * ddist (0: R * C), with the optional four-step twiddle
// W_N^{r c} (tw.lo set).
template <typename T>
struct TransposePass final : PassBase {
  Buf src, dst;
  long long batch, R, C, sdist = 0, ddist = 0;
  SplitTw<T> tw{};
  TransposePass(Buf s, Buf d, long long b, long long r, long long c) : src(s), dst(d), batch(b), R(r), C(c) {}
  cudaError_t run(const void *in, void *out, void *s0, void *s1, cudaStream_t st) const override {
    return launch_transpose<T>(reinterpret_cast<const cpx<T> *>(TilePass<T>::pick(src, in, out, s0, s1)),
                               reinterpret_cast<cpx<T> *>(TilePass<T>::pick(dst, in, out, s0, s1)), batch, R, C, st,
                               sdist, ddist, tw);
  }
  std::shared_ptr<PassBase> rebatched(long long from, long long to) const override {
    auto q = std::make_shared<TransposePass<T>>(*this);
    q->batch = batch / from * to;
    return q;
  }
  std::string describe() const override {
    std::ostringstream o;
    o << "transpose " << (sizeof(T) == 4 ? "f32" : "f64") << " " << R << "x" << C << " transforms=" << batch << " "
      << buf_name(src) << "->" << buf_name(dst) << (tw.lo ? " +twiddle" : "");
    return o.str();
  }
};

// One elementwise step of a multi-pass Rader chain (launch_rader_step); the
// working rows and the saved x_0 / A_0 live in `ws`.
template <typename T>
struct RaderStepPass final : PassBase {
  int mode;
  Buf src, ws, dst;
  long long batch, p, xdist, ydist;
  const int *perm;
  const cpx<T> *kern;
  RaderStepPass(int m, Buf s, Buf w, Buf d, long long b, long long p_, long long xd, long long yd, const int *pm,
                const cpx<T> *k)
      : mode(m), src(s), ws(w), dst(d), batch(b), p(p_), xdist(xd), ydist(yd), perm(pm), kern(k) {}
  cudaError_t run(const void *in, void *out, void *s0, void *s1, cudaStream_t st) const override {
    return launch_rader_step<T>(mode, reinterpret_cast<const cpx<T> *>(TilePass<T>::pick(src, in, out, s0, s1)),
                                reinterpret_cast<cpx<T> *>(TilePass<T>::pick(ws, in, out, s0, s1)),
                                reinterpret_cast<cpx<T> *>(TilePass<T>::pick(dst, in, out, s0, s1)), batch, p, xdist,
                                ydist, perm, kern, st);
  }
  std::shared_ptr<PassBase> rebatched(long long from, long long to) const override {
    auto q = std::make_shared<RaderStepPass<T>>(*this);
    q->batch = batch / from * to;
    return q;
  }
  std::string describe() const override {
    static const char *names[3] = {"rader-gather", "rader-kernel-product", "rader-scatter"};
    std::ostringstream o;
    o << names[mode] << " " << (sizeof(T) == 4 ? "f32" : "f64") << " p=" << p << " transforms=" << batch << " "
      << buf_name(mode == 0 ? src : ws) << "->" << buf_name(mode == 2 ? dst : ws);
    return o.str();
  }
};

// Elementwise widen / take / expand around a full complex transform of a
// real signal (launch_real_convert).
template <typename T>
struct ConvertPass final : PassBase {
  int mode;
  Buf src, dst;
  long long batch, sdist, ddist, n;
  ConvertPass(int m, Buf s, Buf d, long long b, long long sd, long long dd, long long n_)
      : mode(m), src(s), dst(d), batch(b), sdist(sd), ddist(dd), n(n_) {}
  cudaError_t run(const void *in, void *out, void *s0, void *s1, cudaStream_t st) const override {
    return launch_real_convert<T>(mode, TilePass<T>::pick(src, in, out, s0, s1),
                                  TilePass<T>::pick(dst, in, out, s0, s1), batch, sdist, ddist, n, st);
  }
  std::shared_ptr<PassBase> rebatched(long long from, long long to) const override {
    auto q = std::make_shared<ConvertPass<T>>(*this);
    q->batch = batch / from * to;
    return q;
  }
  std::string describe() const override {
    static const char *names[4] = {"real-widen", "half-take", "hermitian-expand", "real-take"};
    std::ostringstream o;
    o << names[mode & 3] << " " << (sizeof(T) == 4 ? "f32" : "f64") << " n=" << n << " transforms=" << batch << " "
      << buf_name(src) << "->" << buf_name(dst);
    return o.str();
  }
};

}  // namespace ffb
