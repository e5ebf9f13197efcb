/*
 * ORACLE -- test infrastructure only.  Nothing in the product (the flagfft_b200
 * package, libflagfft.so, bench.py's timed arm) links, imports or calls this
 * file; tests/, __graft_entry__.smoke() and bench.py's cpu_baseline leg use it
 * as the checker.
 *
 * A CPU restatement, in plain C, of the FFT algorithms the reference FlagFFT
 * runs on its Exec path (flagfftExec* -> CompiledRaw*Node::execute), driven by
 * the same plan trees its planner builds.  Built twice from ffo_impl.h:
 *   *_d  FP64 arithmetic and tables -- the oracle proper;
 *   *_f  float arithmetic with tables rounded from double as the reference's
 *        src/codegen/tables.cpp does -- an estimate of the reference's own
 *        FP32 output, used for "no worse than the reference" comparisons.
 * Plus ffo_naive_dft: an O(n^2) long-double DFT used to pin the FP64 path.
 *
 * Plan encoding (int64 preorder, mirrors the node shapes of
 * src/utils/include/flagfft/plan.hpp:14-98):
 *   leaf       [0, n, nfactors, f0, f1, ...]
 *   four_step  [1, n, n1, n2, <row n1>, <col n2>]
 *   bluestein  [2, n, m, <child m>]
 *   rader      [3, p, g, <child p-1>]
 *   direct     [4, n]
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <unistd.h>

#define FFO_PI 3.14159265358979323846264338327950288
#define FFO_PI_L 3.14159265358979323846264338327950288L

enum { FFO_LEAF = 0, FFO_FOUR_STEP = 1, FFO_BLUESTEIN = 2, FFO_RADER = 3, FFO_DIRECT = 4 };

typedef struct ffo_node {
  int kind;
  int64_t length;
  int64_t factors[64];
  int nfactors;
  int64_t n1, n2, m, root;
  struct ffo_node *a, *b;
  /* Bluestein / Rader: FFT of the kernel sequence for the sign `kern_sign`,
   * computed once per call before the rows run (ffo_impl.h prepare) */
  void *kern;
  int kern_sign;
} ffo_node;

static void ffo_free(ffo_node *nd) {
  if (!nd) return;
  ffo_free(nd->a);
  ffo_free(nd->b);
  free(nd->kern);
  free(nd);
}

static ffo_node *ffo_parse(const int64_t *code, int64_t *pos) {
  ffo_node *nd = (ffo_node *)calloc(1, sizeof(ffo_node));
  nd->kind = (int)code[(*pos)++];
  nd->length = code[(*pos)++];
  switch (nd->kind) {
    case FFO_LEAF: {
      nd->nfactors = (int)code[(*pos)++];
      int64_t prod = 1;
      for (int i = 0; i < nd->nfactors; ++i) {
        nd->factors[i] = code[(*pos)++];
        prod *= nd->factors[i];
        if (nd->factors[i] > 64) {
          ffo_free(nd);
          return NULL;
        }
      }
      if (prod != nd->length || nd->nfactors < 1) {
        ffo_free(nd);
        return NULL;
      }
      break;
    }
    case FFO_FOUR_STEP:
      nd->n1 = code[(*pos)++];
      nd->n2 = code[(*pos)++];
      nd->a = ffo_parse(code, pos);
      nd->b = ffo_parse(code, pos);
      if (!nd->a || !nd->b || nd->n1 * nd->n2 != nd->length) {
        ffo_free(nd);
        return NULL;
      }
      break;
    case FFO_BLUESTEIN:
      nd->m = code[(*pos)++];
      nd->a = ffo_parse(code, pos);
      if (!nd->a || nd->a->length != nd->m || nd->m < 2 * nd->length - 1) {
        ffo_free(nd);
        return NULL;
      }
      break;
    case FFO_RADER:
      nd->root = code[(*pos)++];
      nd->a = ffo_parse(code, pos);
      if (!nd->a || nd->a->length != nd->length - 1) {
        ffo_free(nd);
        return NULL;
      }
      break;
    case FFO_DIRECT:
      break;
    default:
      ffo_free(nd);
      return NULL;
  }
  return nd;
}

/* Parallel loop over [0, count) on the host's cores (pthreads): threads take
 * indices from a shared counter.  `ffo_in_worker` marks the worker threads so
 * a loop reached from inside one runs serially.  FFO_THREADS caps the threads. */
static __thread int ffo_in_worker;

typedef struct {
  void (*body)(void *ctx, int64_t i);
  void *ctx;
  int64_t count;
  int64_t next;
} ffo_loop;

static void *ffo_loop_worker(void *arg) {
  ffo_loop *lp = (ffo_loop *)arg;
  ffo_in_worker = 1;
  for (;;) {
    int64_t i = __atomic_fetch_add(&lp->next, 1, __ATOMIC_RELAXED);
    if (i >= lp->count) break;
    lp->body(lp->ctx, i);
  }
  return NULL;
}

static int ffo_threads(void) {
  const char *e = getenv("FFO_THREADS");
  long t = e ? strtol(e, NULL, 10) : sysconf(_SC_NPROCESSORS_ONLN);
  if (t < 1) t = 1;
  if (t > 256) t = 256;
  return (int)t;
}

static void ffo_parallel_for(int64_t count, void (*body)(void *, int64_t), void *ctx) {
  int nt = ffo_in_worker ? 1 : ffo_threads();
  if (nt > count) nt = (int)count;
  if (nt <= 1) {
    for (int64_t i = 0; i < count; ++i) body(ctx, i);
    return;
  }
  ffo_loop lp = {body, ctx, count, 0};
  pthread_t th[256];
  int started = 0;
  for (int t = 0; t < nt - 1; ++t)
    if (pthread_create(&th[started], NULL, ffo_loop_worker, &lp) == 0) ++started;
  ffo_loop_worker(&lp);
  ffo_in_worker = 0;
  for (int t = 0; t < started; ++t) pthread_join(th[t], NULL);
}

/* Cache of cos/sin(2*pi*m/n), m < n, for n up to 2^20 (computed in double,
 * the precision the reference builds its tables in).  Rows run on several
 * OpenMP threads: a slot is claimed under a lock and published by storing its
 * length after its table (release), which readers load with acquire. */
#define FFO_ROOT_SLOTS 1024
#define FFO_ROOT_CACHE(NAME, T, COS, SIN, PI)                                                          \
  static int64_t NAME##_n[FFO_ROOT_SLOTS];                                                             \
  static T *NAME##_tab[FFO_ROOT_SLOTS];                                                                \
  static pthread_mutex_t NAME##_lock = PTHREAD_MUTEX_INITIALIZER;                                      \
  static const T *NAME(int64_t n) {                                                                    \
    if (n <= 0 || n > (1 << 20)) return NULL;                                                          \
    uint64_t h = ((uint64_t)n * 0x9e3779b97f4a7c15ULL) >> 54;                                          \
    for (int pass = 0; pass < 2; ++pass) {                                                             \
      if (pass == 1) pthread_mutex_lock(&NAME##_lock);                                                 \
      for (int probe = 0; probe < FFO_ROOT_SLOTS; ++probe) {                                           \
        int slot = (int)((h + (uint64_t)probe) % FFO_ROOT_SLOTS);                                      \
        int64_t have = __atomic_load_n(&NAME##_n[slot], __ATOMIC_ACQUIRE);                             \
        if (have == n) {                                                                               \
          if (pass == 1) pthread_mutex_unlock(&NAME##_lock);                                           \
          return NAME##_tab[slot];                                                                     \
        }                                                                                              \
        if (have == 0) {                                                                               \
          if (pass == 0) break; /* not cached: claim a slot under the lock */                          \
          T *t = (T *)malloc(sizeof(T) * 2 * (size_t)n);                                               \
          for (int64_t m = 0; m < n; ++m) {                                                            \
            T a = 2 * (PI) * (T)m / (T)n;                                                              \
            t[2 * m] = COS(a);                                                                         \
            t[2 * m + 1] = SIN(a);                                                                     \
          }                                                                                            \
          NAME##_tab[slot] = t;                                                                        \
          __atomic_store_n(&NAME##_n[slot], n, __ATOMIC_RELEASE);                                      \
          pthread_mutex_unlock(&NAME##_lock);                                                          \
          return t;                                                                                    \
        }                                                                                              \
      }                                                                                                \
    }                                                                                                  \
    pthread_mutex_unlock(&NAME##_lock);                                                                \
    return NULL;                                                                                       \
  }

FFO_ROOT_CACHE(ffo_unit_roots, double, cos, sin, FFO_PI)
FFO_ROOT_CACHE(ffo_unit_roots_l, long double, cosl, sinl, FFO_PI_L)

#define TREAL double
#define TROOTS ffo_unit_roots
#define TCOS cos
#define TSIN sin
#define TPI FFO_PI
#define REAL double
#define SFX(name) name##_d
#include "ffo_impl.h"
#undef REAL
#undef SFX

#define REAL float
#define SFX(name) name##_f
#include "ffo_impl.h"
#undef REAL
#undef SFX
#undef TREAL
#undef TROOTS
#undef TCOS
#undef TSIN
#undef TPI

/* Long double: the same algorithms with tables, angles and arithmetic in
 * long double -- a truth about 2^11 times more precise than FP64, used to
 * measure the error of the FP64 restatement itself (an estimate of the
 * reference's own FP64 Exec error). */
#define TREAL long double
#define TROOTS ffo_unit_roots_l
#define TCOS cosl
#define TSIN sinl
#define TPI FFO_PI_L
#define REAL long double
#define SFX(name) name##_l
#include "ffo_impl.h"
#undef REAL
#undef SFX
#undef TREAL
#undef TROOTS
#undef TCOS
#undef TSIN
#undef TPI

/* O(n^2) DFT accumulated in long double with the phase index j*k reduced
 * exactly mod n: the independent pin for the FP64 restatement. */
int ffo_naive_dft(const double *in, double *out, int64_t n, int direction) {
  const long double pi = 3.14159265358979323846264338327950288L;
  for (int64_t k = 0; k < n; ++k) {
    long double re = 0, im = 0;
    for (int64_t j = 0; j < n; ++j) {
      int64_t m = (int64_t)(((__int128)j * k) % n);
      long double a = (direction > 0 ? 2.0L : -2.0L) * pi * (long double)m / (long double)n;
      long double c = cosl(a), s = sinl(a);
      re += (long double)in[2 * j] * c - (long double)in[2 * j + 1] * s;
      im += (long double)in[2 * j] * s + (long double)in[2 * j + 1] * c;
    }
    out[2 * k] = (double)re;
    out[2 * k + 1] = (double)im;
  }
  return 0;
}
