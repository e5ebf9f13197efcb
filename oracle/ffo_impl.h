/*
 * Test infrastructure (the oracle) -- never linked into the product library.
 *
 * Precision-generic body of the CPU restatement of the reference FFT
 * algorithms.  ffo.c includes this file twice: once with REAL=double (the
 * FP64 oracle every parity test checks against) and once with REAL=float
 * (the same algorithm, with the reference's float tables and float
 * arithmetic, used to estimate the error the reference's own FP32 Exec
 * output carries).
 *
 * Required macros: REAL, SFX(name) (appends the precision suffix), and the
 * precision tables and angles are built in: TREAL (the table type), TROOTS(n)
 * (the cached table of n-th roots of unity in TREAL, or NULL), TCOS / TSIN
 * and TPI.  The FP64 and float builds take their tables in double, as the
 * reference builds its tables; the long-double build (a more precise truth
 * used to measure the FP64 restatement's own error) in long double.
 */

typedef struct {
  REAL re, im;
} SFX(cpx);

static SFX(cpx) SFX(cmul)(SFX(cpx) a, SFX(cpx) b) {
  SFX(cpx) r;
  r.re = a.re * b.re - a.im * b.im;
  r.im = a.im * b.re + a.re * b.im;
  return r;
}

static SFX(cpx) SFX(cadd)(SFX(cpx) a, SFX(cpx) b) {
  SFX(cpx) r;
  r.re = a.re + b.re;
  r.im = a.im + b.im;
  return r;
}

static SFX(cpx) SFX(conj)(SFX(cpx) a) {
  a.im = -a.im;
  return a;
}

/* exp(sign * 2*pi*i * num / den) computed in double with the integer product
 * reduced exactly, then rounded to REAL -- the reference builds every table in
 * double and casts (src/codegen/tables.cpp:39-69, 116-147). */
static SFX(cpx) SFX(root)(int64_t num, int64_t den, int sign) {
  int64_t m = num % den;
  if (m < 0) m += den;
  const TREAL *tab = TROOTS(den);
  SFX(cpx) r;
  if (tab) {
    r.re = (REAL)tab[2 * m];
    r.im = (REAL)(sign > 0 ? tab[2 * m + 1] : -tab[2 * m + 1]);
  } else {
    TREAL a = (TREAL)sign * 2 * TPI * (TREAL)m / (TREAL)den;
    r.re = (REAL)TCOS(a);
    r.im = (REAL)TSIN(a);
  }
  return r;
}

/* Radix-R butterfly: y[q] = sum_j t[j] * W_R^{sign*j*q}.  The reference's
 * straight-line codelets (python/flagfft_codegen/codelet/radix*.py) compute
 * the same forward DFT; the inverse is conj(forward(conj x))
 * (python/flagfft_codegen/kernels.py:493-512), which equals the +sign DFT. */
static void SFX(dft_small)(const SFX(cpx) *t, SFX(cpx) *y, int64_t R, int sign) {
  for (int64_t q = 0; q < R; ++q) {
    SFX(cpx) acc = t[0];
    for (int64_t j = 1; j < R; ++j) acc = SFX(cadd)(acc, SFX(cmul)(t[j], SFX(root)(j * q, R, sign)));
    y[q] = acc;
  }
}

/* Mixed-radix decimation-in-time leaf (python/flagfft_codegen/kernels.py:515-831):
 * stage 0 is a radix-f[0] DFT over the most significant time digit (digit-
 * reversed load, kernels.py:519-547); stage s multiplies by
 * W_{L_s*f[s]}^{k'*j} (L_s = f[0]*...*f[s-1], k' the frequency prefix; the
 * twiddle of src/codegen/tables.cpp:39-69) and applies the radix-f[s]
 * butterfly; the output is in natural order (kernels.py:550-581).
 * Written as the equivalent recursion: the last stage combines f[S-1]
 * decimated sub-transforms x[j + f[S-1]*m]. */
static void SFX(dit)(const SFX(cpx) *x, int64_t n, int64_t stride, const int64_t *f, int nf, SFX(cpx) *out,
                     int sign) {
  if (nf == 1) {
    SFX(cpx) t[64];
    for (int64_t j = 0; j < n; ++j) t[j] = x[j * stride];
    SFX(dft_small)(t, out, n, sign);
    return;
  }
  int64_t R = f[nf - 1];
  int64_t M = n / R;
  SFX(cpx) *sub = (SFX(cpx) *)malloc(sizeof(SFX(cpx)) * (size_t)n);
  for (int64_t j = 0; j < R; ++j) SFX(dit)(x + j * stride, M, stride * R, f, nf - 1, sub + j * M, sign);
  SFX(cpx) t[64], y[64];
  for (int64_t k = 0; k < M; ++k) {
    for (int64_t j = 0; j < R; ++j) {
      t[j] = sub[j * M + k];
      if (j != 0 && k != 0) t[j] = SFX(cmul)(t[j], SFX(root)(j * k, n, sign));
    }
    SFX(dft_small)(t, y, R, sign);
    for (int64_t q = 0; q < R; ++q) out[k + M * q] = y[q];
  }
  free(sub);
}

static void SFX(exec_node)(const ffo_node *nd, const SFX(cpx) *in, SFX(cpx) *out, int sign);

/* Direct DFT node (reference: DirectDFTPlanNode, src/plan/nodes.cpp). */
static void SFX(direct)(int64_t n, const SFX(cpx) *in, SFX(cpx) *out, int sign) {
  for (int64_t k = 0; k < n; ++k) {
    SFX(cpx) acc = {0, 0};
    for (int64_t j = 0; j < n; ++j) acc = SFX(cadd)(acc, SFX(cmul)(in[j], SFX(root)(j * k, n, sign)));
    out[k] = acc;
  }
}

/* Fused four-step (src/exec/raw_nodes.cpp:84-104; row/col IO modes
 * python/flagfft_codegen/kernels.py:710-742,796-815): Y[j2][k1] =
 * DFT_n1 over j1 of x[j1*n2 + j2]; Y *= W_N^{j2*k1} (the N-entry table of
 * src/codegen/tables.cpp:116-147); X[k1 + n1*k2] = DFT_n2 over j2. */
typedef struct {
  const ffo_node *nd;
  const SFX(cpx) *in;
  SFX(cpx) *out, *y;
  int sign;
} SFX(fs_ctx);

/* column j2: Y[j2][k1] = DFT_n1 over j1 of x[j1*n2 + j2], times W_N^{j2*k1} */
static void SFX(fs_column)(void *vc, int64_t j2) {
  const SFX(fs_ctx) *c = (const SFX(fs_ctx) *)vc;
  const ffo_node *nd = c->nd;
  int64_t n1 = nd->n1, n2 = nd->n2, n = nd->length;
  SFX(cpx) *col = (SFX(cpx) *)malloc(sizeof(SFX(cpx)) * 2 * (size_t)n1);
  SFX(cpx) *res = col + n1;
  for (int64_t j1 = 0; j1 < n1; ++j1) col[j1] = c->in[j1 * n2 + j2];
  SFX(exec_node)(nd->a, col, res, c->sign);
  for (int64_t k1 = 0; k1 < n1; ++k1) c->y[j2 * n1 + k1] = SFX(cmul)(res[k1], SFX(root)(j2 * k1, n, c->sign));
  free(col);
}

/* row k1: X[k1 + n1*k2] = DFT_n2 over j2 of Y[j2][k1] */
static void SFX(fs_row)(void *vc, int64_t k1) {
  const SFX(fs_ctx) *c = (const SFX(fs_ctx) *)vc;
  const ffo_node *nd = c->nd;
  int64_t n1 = nd->n1, n2 = nd->n2;
  SFX(cpx) *col = (SFX(cpx) *)malloc(sizeof(SFX(cpx)) * 2 * (size_t)n2);
  SFX(cpx) *res = col + n2;
  for (int64_t j2 = 0; j2 < n2; ++j2) col[j2] = c->y[j2 * n1 + k1];
  SFX(exec_node)(nd->b, col, res, c->sign);
  for (int64_t k2 = 0; k2 < n2; ++k2) c->out[k1 + n1 * k2] = res[k2];
  free(col);
}

/* A long transform reached outside a worker thread spreads its (independent)
 * columns and rows over the host threads. */
static void SFX(four_step)(const ffo_node *nd, const SFX(cpx) *in, SFX(cpx) *out, int sign) {
  int64_t n = nd->length;
  SFX(fs_ctx) c = {nd, in, out, (SFX(cpx) *)malloc(sizeof(SFX(cpx)) * (size_t)n), sign};
  if (n >= (1 << 15)) {
    ffo_parallel_for(nd->n2, SFX(fs_column), &c);
    ffo_parallel_for(nd->n1, SFX(fs_row), &c);
  } else {
    for (int64_t j2 = 0; j2 < nd->n2; ++j2) SFX(fs_column)(&c, j2);
    for (int64_t k1 = 0; k1 < nd->n1; ++k1) SFX(fs_row)(&c, k1);
  }
  free(c.y);
}

/* exp(sign * i*pi * (k^2 mod 2n) / n): the chirp of
 * src/codegen/tables.cpp:149-216 (k^2 reduced mod 2n before the angle). */
static SFX(cpx) SFX(chirp)(int64_t k, int64_t n, double sign) {
  int64_t red = (int64_t)(((__int128)k * k) % (2 * n));
  TREAL a = (TREAL)sign * TPI * (TREAL)red / (TREAL)n;
  SFX(cpx) r;
  r.re = (REAL)TCOS(a);
  r.im = (REAL)TSIN(a);
  return r;
}

/* B = FFT_m(b), b[k] = chirp(k) with the conjugate sign, mirrored at m - k
 * (the reference's lazily built b_fft_buf, src/exec/raw_nodes.cpp:140-151):
 * the node's cached copy when prepare() made one for this sign. */
static SFX(cpx) *SFX(bluestein_kernel)(const ffo_node *nd, int sign) {
  if (nd->kern && nd->kern_sign == sign) return (SFX(cpx) *)nd->kern;
  int64_t n = nd->length, m = nd->m;
  double csign = sign > 0 ? 1.0 : -1.0;
  SFX(cpx) *b = (SFX(cpx) *)calloc((size_t)m, sizeof(SFX(cpx)));
  SFX(cpx) *bf = (SFX(cpx) *)malloc(sizeof(SFX(cpx)) * (size_t)m);
  for (int64_t k = 0; k < n; ++k) {
    SFX(cpx) v = SFX(chirp)(k, n, -csign);
    b[k] = v;
    if (k) b[m - k] = v;
  }
  SFX(exec_node)(nd->a, b, bf, -1);
  free(b);
  return bf;
}

/* Bluestein chain (src/exec/raw_nodes.cpp:140-204, kernels
 * python/flagfft_codegen/jit_source.py:125-228): chirp c[k] =
 * exp(-+ i*pi*k^2/n) (+ for the inverse), b[k] = conj-sign chirp mirrored at
 * m-k, B = FFT_m(b) with the forward child; a = x*c zero-padded to m;
 * P = conj(FFT(a) * B); y[k] = conj(FFT(P))[k] / m * c[k]. */
static void SFX(bluestein)(const ffo_node *nd, const SFX(cpx) *in, SFX(cpx) *out, int sign) {
  int64_t n = nd->length, m = nd->m;
  double csign = sign > 0 ? 1.0 : -1.0;
  SFX(cpx) *bf = SFX(bluestein_kernel)(nd, sign);
  SFX(cpx) *a = (SFX(cpx) *)calloc((size_t)m, sizeof(SFX(cpx)));
  SFX(cpx) *af = (SFX(cpx) *)malloc(sizeof(SFX(cpx)) * (size_t)m);
  for (int64_t k = 0; k < n; ++k) a[k] = SFX(cmul)(in[k], SFX(chirp)(k, n, csign));
  SFX(exec_node)(nd->a, a, af, -1);
  for (int64_t k = 0; k < m; ++k) a[k] = SFX(conj)(SFX(cmul)(af[k], bf[k]));
  SFX(exec_node)(nd->a, a, af, -1);
  for (int64_t k = 0; k < n; ++k) {
    SFX(cpx) c;
    c.re = af[k].re / (REAL)m;
    c.im = -af[k].im / (REAL)m;
    out[k] = SFX(cmul)(c, SFX(chirp)(k, n, csign));
  }
  if (bf != (SFX(cpx) *)nd->kern) free(bf);
  free(a);
  free(af);
}

/* FFT_m of b[q] = W_p^{sign g^q} (src/codegen/tables.cpp:218-258): the
 * node's cached copy when prepare() made one for this sign. */
static SFX(cpx) *SFX(rader_kernel)(const ffo_node *nd, int sign) {
  if (nd->kern && nd->kern_sign == sign) return (SFX(cpx) *)nd->kern;
  int64_t p = nd->length, m = p - 1, g = nd->root;
  SFX(cpx) *b = (SFX(cpx) *)malloc(sizeof(SFX(cpx)) * (size_t)m);
  SFX(cpx) *bf = (SFX(cpx) *)malloc(sizeof(SFX(cpx)) * (size_t)m);
  int64_t v = 1;
  for (int64_t q = 0; q < m; ++q) {
    b[q] = SFX(root)(v, p, sign);
    v = (v * g) % p;
  }
  SFX(exec_node)(nd->a, b, bf, -1);
  free(b);
  return bf;
}

/* Rader chain (src/exec/raw_nodes.cpp:240-305, kernels
 * python/flagfft_codegen/jit_source.py:270-388, tables
 * src/plan/rader_utils.cpp:55-90 and src/codegen/tables.cpp:218-258):
 * idx[q] = g^q mod p; a[q] = x[idx[(m-q) mod m]]; b[q] = W_p^{sign*idx[q]};
 * P = conj(FFT(a) * FFT(b)); X[idx[q]] = x[0] + conj(FFT(P))[q] / m;
 * X[0] = sum x. */
static void SFX(rader)(const ffo_node *nd, const SFX(cpx) *in, SFX(cpx) *out, int sign) {
  int64_t p = nd->length, m = p - 1, g = nd->root;
  int64_t *idx = (int64_t *)malloc(sizeof(int64_t) * (size_t)m);
  int64_t v = 1;
  for (int64_t q = 0; q < m; ++q) {
    idx[q] = v;
    v = (v * g) % p;
  }
  SFX(cpx) *bf = SFX(rader_kernel)(nd, sign);
  SFX(cpx) *a = (SFX(cpx) *)malloc(sizeof(SFX(cpx)) * (size_t)m);
  SFX(cpx) *af = (SFX(cpx) *)malloc(sizeof(SFX(cpx)) * (size_t)m);
  for (int64_t q = 0; q < m; ++q) a[q] = in[idx[q == 0 ? 0 : m - q]];
  SFX(exec_node)(nd->a, a, af, -1);
  for (int64_t q = 0; q < m; ++q) a[q] = SFX(conj)(SFX(cmul)(af[q], bf[q]));
  SFX(exec_node)(nd->a, a, af, -1);
  SFX(cpx) s = {0, 0};
  for (int64_t k = 0; k < p; ++k) s = SFX(cadd)(s, in[k]);
  for (int64_t q = 0; q < m; ++q) {
    SFX(cpx) c;
    c.re = in[0].re + af[q].re / (REAL)m;
    c.im = in[0].im - af[q].im / (REAL)m;
    out[idx[q]] = c;
  }
  out[0] = s;
  free(idx);
  if (bf != (SFX(cpx) *)nd->kern) free(bf);
  free(a);
  free(af);
}

static void SFX(exec_node)(const ffo_node *nd, const SFX(cpx) *in, SFX(cpx) *out, int sign) {
  switch (nd->kind) {
    case FFO_LEAF:
      SFX(dit)(in, nd->length, 1, nd->factors, nd->nfactors, out, sign);
      break;
    case FFO_FOUR_STEP:
      SFX(four_step)(nd, in, out, sign);
      break;
    case FFO_BLUESTEIN:
      SFX(bluestein)(nd, in, out, sign);
      break;
    case FFO_RADER:
      SFX(rader)(nd, in, out, sign);
      break;
    default:
      SFX(direct)(nd->length, in, out, sign);
      break;
  }
}

/* Builds, before the rows run, every Bluestein / Rader kernel spectrum the
 * tree needs for a transform of this sign (the children of a convolution
 * always run forward; a four-step's children take its sign).  The rows then
 * share them read-only. */
static void SFX(prepare)(ffo_node *nd, int sign) {
  if (!nd) return;
  if (nd->kind == FFO_FOUR_STEP) {
    SFX(prepare)(nd->a, sign);
    SFX(prepare)(nd->b, sign);
  } else if (nd->kind == FFO_BLUESTEIN || nd->kind == FFO_RADER) {
    SFX(prepare)(nd->a, -1);
    if (nd->kern && nd->kern_sign != sign) {
      free(nd->kern);
      nd->kern = NULL;
    }
    if (!nd->kern) {
      nd->kern = nd->kind == FFO_BLUESTEIN ? SFX(bluestein_kernel)(nd, sign) : SFX(rader_kernel)(nd, sign);
      nd->kern_sign = sign;
    }
  }
}

/* Rows of a batch run on the host threads; a long row runs alone and its
 * four-step spreads its columns over them instead. */
typedef struct {
  const ffo_node *nd;
  const REAL *in;
  REAL *out;
  int64_t idist, odist;
  int sign, mode; /* mode 0 C2C, 1 R2C, 2 C2R */
} SFX(rows_ctx);

static void SFX(one_row)(void *vc, int64_t b) {
  const SFX(rows_ctx) *c = (const SFX(rows_ctx) *)vc;
  int64_t n = c->nd->length, half = n / 2 + 1;
  SFX(cpx) *x = (SFX(cpx) *)malloc(sizeof(SFX(cpx)) * 2 * (size_t)n);
  SFX(cpx) *y = x + n;
  if (c->mode == 0) {
    memcpy(x, c->in + 2 * b * c->idist, sizeof(SFX(cpx)) * (size_t)n);
    SFX(exec_node)(c->nd, x, y, c->sign);
    memcpy(c->out + 2 * b * c->odist, y, sizeof(SFX(cpx)) * (size_t)n);
  } else if (c->mode == 1) {
    for (int64_t k = 0; k < n; ++k) {
      x[k].re = c->in[b * c->idist + k];
      x[k].im = 0;
    }
    SFX(exec_node)(c->nd, x, y, -1);
    memcpy(c->out + 2 * b * c->odist, y, sizeof(SFX(cpx)) * (size_t)half);
  } else {
    const REAL *row = c->in + 2 * b * c->idist;
    for (int64_t k = 0; k < n; ++k) {
      int64_t src = k < half ? k : n - k;
      x[k].re = row[2 * src];
      x[k].im = k < half ? row[2 * src + 1] : -row[2 * src + 1];
      if (k == 0 || (n % 2 == 0 && k == n / 2)) x[k].im = 0;
    }
    SFX(exec_node)(c->nd, x, y, 1);
    for (int64_t k = 0; k < n; ++k) c->out[b * c->odist + k] = y[k].re;
  }
  free(x);
}

static void SFX(run_rows)(const SFX(rows_ctx) *c, int64_t batch) {
  if (batch > 1 && c->nd->length < (1 << 16))
    ffo_parallel_for(batch, SFX(one_row), (void *)c);
  else
    for (int64_t b = 0; b < batch; ++b) SFX(one_row)((void *)c, b);
}

/* Batched C2C with element distances idist/odist (contiguous rows). */
int SFX(ffo_c2c)(const int64_t *code, const REAL *in, REAL *out, int64_t batch, int64_t idist, int64_t odist,
                 int direction) {
  int64_t pos = 0;
  ffo_node *nd = ffo_parse(code, &pos);
  if (!nd) return -1;
  int sign = direction > 0 ? 1 : -1;
  SFX(prepare)(nd, sign);
  SFX(rows_ctx) c = {nd, in, out, idist, odist, sign, 0};
  SFX(run_rows)(&c, batch);
  ffo_free(nd);
  return 0;
}

/* R2C: expand to complex, full forward C2C, keep bins 0..n/2
 * (src/exec/raw_nodes.cpp:419-456; python/flagfft_codegen/kernels.py:1098-1156). */
int SFX(ffo_r2c)(const int64_t *code, const REAL *in, REAL *out, int64_t batch, int64_t idist, int64_t odist) {
  int64_t pos = 0;
  ffo_node *nd = ffo_parse(code, &pos);
  if (!nd) return -1;
  SFX(prepare)(nd, -1);
  SFX(rows_ctx) c = {nd, in, out, idist, odist, -1, 1};
  SFX(run_rows)(&c, batch);
  ffo_free(nd);
  return 0;
}

/* C2R: Hermitian expansion with Im(DC) and, for even n, Im(Nyquist) forced to
 * zero, inverse C2C, real part (src/exec/raw_nodes.cpp:480-519;
 * python/flagfft_codegen/kernels.py:1159-1221). */
int SFX(ffo_c2r)(const int64_t *code, const REAL *in, REAL *out, int64_t batch, int64_t idist, int64_t odist) {
  int64_t pos = 0;
  ffo_node *nd = ffo_parse(code, &pos);
  if (!nd) return -1;
  SFX(prepare)(nd, 1);
  SFX(rows_ctx) c = {nd, in, out, idist, odist, 1, 2};
  SFX(run_rows)(&c, batch);
  ffo_free(nd);
  return 0;
}

/* 2-D RTRT (src/exec/raw_nodes.cpp:549-852): C2C = row FFT along n1 then
 * column FFT along n0; R2C = row R2C along n1, column C2C along n0 over the
 * n1/2+1 kept columns; C2R = column inverse C2C first, then row C2R.
 * kind: 0 C2C, 1 R2C, 2 C2R.  row_code/col_code are the n1 and n0 plans. */
typedef struct {
  const ffo_node *row, *col;
  const REAL *src;
  REAL *dst;
  SFX(cpx) *grid;
  int64_t n0, n1, h1;
  int sign, csign, kind;
} SFX(grid_ctx);

/* first half of a 2-D transform, row r of the grid: C2C row FFT, or R2C
 * (expand, forward FFT, keep the half spectrum) */
static void SFX(grid_row_in)(void *vc, int64_t r) {
  const SFX(grid_ctx) *c = (const SFX(grid_ctx) *)vc;
  int64_t n1 = c->n1;
  SFX(cpx) *t = (SFX(cpx) *)malloc(sizeof(SFX(cpx)) * 2 * (size_t)n1);
  SFX(cpx) *u = t + n1;
  if (c->kind == 0) {
    SFX(exec_node)(c->row, (const SFX(cpx) *)c->src + r * n1, c->grid + r * n1, c->sign);
  } else {
    for (int64_t k = 0; k < n1; ++k) {
      t[k].re = c->src[r * n1 + k];
      t[k].im = 0;
    }
    SFX(exec_node)(c->row, t, u, -1);
    memcpy(c->grid + r * n1, u, sizeof(SFX(cpx)) * (size_t)c->h1);
  }
  free(t);
}

/* column cc of the grid */
static void SFX(grid_col)(void *vc, int64_t cc) {
  const SFX(grid_ctx) *c = (const SFX(grid_ctx) *)vc;
  int64_t n0 = c->n0, n1 = c->n1;
  SFX(cpx) *t = (SFX(cpx) *)malloc(sizeof(SFX(cpx)) * 2 * (size_t)n0);
  SFX(cpx) *u = t + n0;
  for (int64_t r = 0; r < n0; ++r) t[r] = c->grid[r * n1 + cc];
  SFX(exec_node)(c->col, t, u, c->csign);
  for (int64_t r = 0; r < n0; ++r) c->grid[r * n1 + cc] = u[r];
  free(t);
}

/* last half of a 2-D C2R, row r: Hermitian expansion, inverse FFT, real part */
static void SFX(grid_row_out)(void *vc, int64_t r) {
  const SFX(grid_ctx) *c = (const SFX(grid_ctx) *)vc;
  int64_t n1 = c->n1, h1 = c->h1;
  SFX(cpx) *t = (SFX(cpx) *)malloc(sizeof(SFX(cpx)) * 2 * (size_t)n1);
  SFX(cpx) *u = t + n1;
  for (int64_t k = 0; k < n1; ++k) {
    int64_t s = k < h1 ? k : n1 - k;
    t[k] = c->grid[r * n1 + s];
    if (k >= h1) t[k].im = -t[k].im;
    if (k == 0 || (n1 % 2 == 0 && k == n1 / 2)) t[k].im = 0;
  }
  SFX(exec_node)(c->row, t, u, 1);
  for (int64_t k = 0; k < n1; ++k) c->dst[r * n1 + k] = u[k].re;
  free(t);
}

/* 2-D RTRT (src/exec/raw_nodes.cpp:549-852): C2C = row FFT along n1 then
 * column FFT along n0; R2C = row R2C along n1, column C2C along n0 over the
 * n1/2+1 kept columns; C2R = column inverse C2C first, then row C2R.
 * kind: 0 C2C, 1 R2C, 2 C2R.  row_code/col_code are the n1 and n0 plans.
 * The rows, then the columns, run on the host threads. */
int SFX(ffo_2d)(int kind, const int64_t *row_code, const int64_t *col_code, int64_t n0, int64_t n1,
                const REAL *in, REAL *out, int64_t batch, int direction) {
  int64_t p0 = 0, p1 = 0;
  ffo_node *row = ffo_parse(row_code, &p0);
  ffo_node *col = ffo_parse(col_code, &p1);
  if (!row || !col) return -1;
  int sign = direction > 0 ? 1 : -1;
  int64_t h1 = n1 / 2 + 1;
  int64_t ncols = kind == 0 ? n1 : h1;
  int csign = kind == 1 ? -1 : (kind == 2 ? 1 : sign);
  SFX(prepare)(row, kind == 0 ? sign : (kind == 1 ? -1 : 1));
  SFX(prepare)(col, csign);
  SFX(cpx) *grid = (SFX(cpx) *)malloc(sizeof(SFX(cpx)) * (size_t)(n0 * n1));
  for (int64_t b = 0; b < batch; ++b) {
    SFX(grid_ctx) c = {row, col, NULL, NULL, grid, n0, n1, h1, sign, csign, kind};
    if (kind == 0) {
      c.src = in + 2 * b * n0 * n1;
      ffo_parallel_for(n0, SFX(grid_row_in), &c);
    } else if (kind == 1) {
      c.src = in + b * n0 * n1;
      ffo_parallel_for(n0, SFX(grid_row_in), &c);
    } else {
      const SFX(cpx) *src = (const SFX(cpx) *)in + b * n0 * h1;
      for (int64_t r = 0; r < n0; ++r) memcpy(grid + r * n1, src + r * h1, sizeof(SFX(cpx)) * (size_t)h1);
    }
    ffo_parallel_for(ncols, SFX(grid_col), &c);
    if (kind == 0) {
      memcpy((SFX(cpx) *)out + b * n0 * n1, grid, sizeof(SFX(cpx)) * (size_t)(n0 * n1));
    } else if (kind == 1) {
      SFX(cpx) *dst = (SFX(cpx) *)out + b * n0 * h1;
      for (int64_t r = 0; r < n0; ++r) memcpy(dst + r * h1, grid + r * n1, sizeof(SFX(cpx)) * (size_t)h1);
    } else {
      c.dst = out + b * n0 * n1;
      ffo_parallel_for(n0, SFX(grid_row_out), &c);
    }
  }
  free(grid);
  ffo_free(row);
  ffo_free(col);
  return 0;
}
