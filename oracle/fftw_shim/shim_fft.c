/*
 * shim_fft.c -- FP64 FFT engine behind the oracle's fftw3.h shim.
 *
 * TEST INFRASTRUCTURE ONLY (see fftw3.h).  It exists because FFTW3 is not
 * installed here and the reference cc/grid/fft_grid.cc calls it.
 *
 * Methods, all written from the textbook descriptions:
 *   - 1-D complex DFT: iterative mixed-radix Stockham autosort (radix 4, 2,
 *     3, 5 butterflies plus a generic O(p^2) butterfly for other primes up to
 *     31), as in Govindaraju et al., "High performance discrete Fourier
 *     transforms on graphics processors" (SC'08), applied on the CPU.
 *   - Lengths with a prime factor > 31: Bluestein's chirp-z algorithm with a
 *     power-of-two convolution.
 *   - Real-to-complex of even length n: one complex DFT of length n/2 on the
 *     even/odd packed sequence followed by the standard split step; odd n uses
 *     a full-length complex DFT.  Complex-to-real is the exact inverse.
 *   - Multi-dimensional transforms: r2c along the last dimension, then
 *     complex DFTs along the remaining dimensions (c2r in reverse order),
 *     processing blocks of adjacent columns for cache locality.
 * Twiddle factors are generated with exact integer argument reduction, so the
 * error is O(eps log n) like any Cooley-Tukey FFT.  Plans are immutable once
 * created; every execute call allocates its own scratch, so concurrent
 * new-array execution from several threads (the reference's FFTSLAB mode) is
 * safe.
 */
#include "fftw3.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

typedef struct {
  double re, im;
} cpx;

static inline cpx cmul(cpx a, cpx b) {
  cpx r;
  r.re = a.re * b.re - a.im * b.im;
  r.im = a.re * b.im + a.im * b.re;
  return r;
}

static inline cpx cadd(cpx a, cpx b) {
  cpx r = {a.re + b.re, a.im + b.im};
  return r;
}

static inline cpx csub(cpx a, cpx b) {
  cpx r = {a.re - b.re, a.im - b.im};
  return r;
}

static inline cpx cconj(cpx a) {
  cpx r = {a.re, -a.im};
  return r;
}

/* exp(sign * 2 pi i * num / den) with num reduced modulo den first. */
static cpx unit_root(int sign, long long num, long long den) {
  long long q = num % den;
  if (q < 0) q += den;
  double ang = 2.0 * M_PI * (double)q / (double)den;
  cpx r = {cos(ang), sign * sin(ang)};
  return r;
}

#define MAX_STAGES 48
#define MAX_GENERIC_RADIX 31
#define BLOCK 16

typedef struct fft1d {
  int n;
  int sign;
  int nstage;
  int radix[MAX_STAGES];
  int ns[MAX_STAGES];
  cpx *tw[MAX_STAGES];    /* tw[s][k*(p-1) + r-1] = w^(r k) over Ns*p */
  cpx *roots[MAX_STAGES]; /* generic radix roots exp(sign 2 pi i q / p) */
  /* Bluestein data (blue != 0). */
  int blue;
  int m;
  cpx *chirp;
  cpx *bfft;
  struct fft1d *mf;
  struct fft1d *mb;
} fft1d;

static fft1d *fft1d_create(int n, int sign);
void fc_shim_fft1d_exec(const fft1d *p, const cpx *in, cpx *out, cpx *scratch);

static void fft1d_destroy(fft1d *p) {
  if (!p) return;
  for (int s = 0; s < p->nstage; ++s) {
    free(p->tw[s]);
    free(p->roots[s]);
  }
  free(p->chirp);
  free(p->bfft);
  fft1d_destroy(p->mf);
  fft1d_destroy(p->mb);
  free(p);
}

/* Scratch (in complex elements) needed by fft1d_exec_b with B transforms. */
static size_t fft1d_scratch_b(const fft1d *p, int B) {
  if (p->blue) return 4 * (size_t)p->m;
  return 2 * (size_t)p->n * B;
}

static size_t fft1d_scratch(const fft1d *p) { return fft1d_scratch_b(p, 1); }

static int factorize(int n, int *fac, int *nf) {
  /* Returns 0 if every prime factor is <= MAX_GENERIC_RADIX. */
  int k = 0;
  while (n % 4 == 0) {
    fac[k++] = 4;
    n /= 4;
  }
  while (n % 2 == 0) {
    fac[k++] = 2;
    n /= 2;
  }
  for (int p = 3; p <= MAX_GENERIC_RADIX && n > 1; p += 2) {
    while (n % p == 0) {
      fac[k++] = p;
      n /= p;
    }
  }
  *nf = k;
  return n == 1 ? 0 : 1;
}

static fft1d *fft1d_create(int n, int sign) {
  fft1d *p = (fft1d *)calloc(1, sizeof(fft1d));
  p->n = n;
  p->sign = sign;
  int fac[MAX_STAGES];
  int nf = 0;
  if (n > 1 && factorize(n, fac, &nf)) {
    /* Bluestein: X_k = c_k sum_j (x_j c_j) conj(c_{k-j}), c_j = e^{s pi i j^2/n}. */
    p->blue = 1;
    int m = 1;
    while (m < 2 * n - 1) m <<= 1;
    p->m = m;
    p->chirp = (cpx *)malloc(sizeof(cpx) * n);
    for (int j = 0; j < n; ++j) {
      long long j2 = (long long)j * j % (2LL * n);
      p->chirp[j] = unit_root(sign, j2, 2LL * n);
    }
    p->mf = fft1d_create(m, -1);
    p->mb = fft1d_create(m, +1);
    cpx *b = (cpx *)calloc(m, sizeof(cpx));
    for (int j = 0; j < n; ++j) {
      b[j] = cconj(p->chirp[j]);
      if (j > 0) b[m - j] = cconj(p->chirp[j]);
    }
    p->bfft = (cpx *)malloc(sizeof(cpx) * m);
    cpx *scr = (cpx *)malloc(sizeof(cpx) * fft1d_scratch(p->mf));
    fc_shim_fft1d_exec(p->mf, b, p->bfft, scr);
    for (int j = 0; j < m; ++j) {
      p->bfft[j].re /= m;
      p->bfft[j].im /= m;
    }
    free(scr);
    free(b);
    return p;
  }
  p->nstage = nf;
  int Ns = 1;
  for (int s = 0; s < nf; ++s) {
    int r = fac[s];
    p->radix[s] = r;
    p->ns[s] = Ns;
    if (Ns > 1) {
      p->tw[s] = (cpx *)malloc(sizeof(cpx) * (size_t)Ns * (r - 1));
      for (int k = 0; k < Ns; ++k)
        for (int q = 1; q < r; ++q)
          p->tw[s][(size_t)k * (r - 1) + q - 1] =
              unit_root(sign, (long long)q * k, (long long)Ns * r);
    }
    if (r != 2 && r != 3 && r != 4) {
      p->roots[s] = (cpx *)malloc(sizeof(cpx) * r);
      for (int q = 0; q < r; ++q) p->roots[s][q] = unit_root(sign, q, r);
    }
    Ns *= r;
  }
  return p;
}

/* One Stockham pass of radix r over B interleaved transforms: element i of
 * transform b is at x[i*B + b].  Reads x, writes y. */
static void stockham_pass(int n, int r, int Ns, const cpx *tw,
                          const cpx *roots, int sign, const cpx *x, cpx *y,
                          int B) {
  const int np = n / r;
  const int ng = np / Ns;
  const double s3 = 0.86602540378443864676 * sign; /* sign * sqrt(3)/2 */
  for (int g = 0; g < ng; ++g) {
    for (int k = 0; k < Ns; ++k) {
      const int j = g * Ns + k;
      const int base = g * Ns * r + k;
      const cpx *t = tw + (size_t)k * (r - 1);
      if (r == 2) {
        const cpx w1 = Ns > 1 ? t[0] : (cpx){1.0, 0.0};
        const cpx *x0 = x + (size_t)j * B, *x1 = x + (size_t)(j + np) * B;
        cpx *y0 = y + (size_t)base * B, *y1 = y + (size_t)(base + Ns) * B;
        for (int b = 0; b < B; ++b) {
          cpx v1 = Ns > 1 ? cmul(x1[b], w1) : x1[b];
          y0[b] = cadd(x0[b], v1);
          y1[b] = csub(x0[b], v1);
        }
      } else if (r == 4) {
        cpx w1 = {1.0, 0.0}, w2 = w1, w3 = w1;
        if (Ns > 1) {
          w1 = t[0];
          w2 = t[1];
          w3 = t[2];
        }
        const cpx *x0 = x + (size_t)j * B, *x1 = x + (size_t)(j + np) * B;
        const cpx *x2 = x + (size_t)(j + 2 * np) * B;
        const cpx *x3 = x + (size_t)(j + 3 * np) * B;
        cpx *y0 = y + (size_t)base * B, *y1 = y + (size_t)(base + Ns) * B;
        cpx *y2 = y + (size_t)(base + 2 * Ns) * B;
        cpx *y3 = y + (size_t)(base + 3 * Ns) * B;
        for (int b = 0; b < B; ++b) {
          cpx v0 = x0[b], v1 = x1[b], v2 = x2[b], v3 = x3[b];
          if (Ns > 1) {
            v1 = cmul(v1, w1);
            v2 = cmul(v2, w2);
            v3 = cmul(v3, w3);
          }
          cpx a0 = cadd(v0, v2);
          cpx a1 = csub(v0, v2);
          cpx a2 = cadd(v1, v3);
          cpx d = csub(v1, v3);
          /* (sign * i) * d */
          cpx sd = {-sign * d.im, sign * d.re};
          y0[b] = cadd(a0, a2);
          y2[b] = csub(a0, a2);
          y1[b] = cadd(a1, sd);
          y3[b] = csub(a1, sd);
        }
      } else if (r == 3) {
        cpx w1 = {1.0, 0.0}, w2 = w1;
        if (Ns > 1) {
          w1 = t[0];
          w2 = t[1];
        }
        const cpx *x0 = x + (size_t)j * B, *x1 = x + (size_t)(j + np) * B;
        const cpx *x2 = x + (size_t)(j + 2 * np) * B;
        cpx *y0 = y + (size_t)base * B, *y1 = y + (size_t)(base + Ns) * B;
        cpx *y2 = y + (size_t)(base + 2 * Ns) * B;
        for (int b = 0; b < B; ++b) {
          cpx v0 = x0[b], v1 = x1[b], v2 = x2[b];
          if (Ns > 1) {
            v1 = cmul(v1, w1);
            v2 = cmul(v2, w2);
          }
          cpx tt = cadd(v1, v2);
          cpx d = csub(v1, v2);
          cpx m = {v0.re - 0.5 * tt.re, v0.im - 0.5 * tt.im};
          cpx sd = {-s3 * d.im, s3 * d.re};
          y0[b] = cadd(v0, tt);
          y1[b] = cadd(m, sd);
          y2[b] = csub(m, sd);
        }
      } else {
        cpx v[MAX_GENERIC_RADIX + 1];
        for (int b = 0; b < B; ++b) {
          for (int q = 0; q < r; ++q) v[q] = x[(size_t)(j + q * np) * B + b];
          if (Ns > 1)
            for (int q = 1; q < r; ++q) v[q] = cmul(v[q], t[q - 1]);
          for (int q = 0; q < r; ++q) {
            cpx acc = v[0];
            for (int u = 1; u < r; ++u)
              acc = cadd(acc, cmul(v[u], roots[(u * q) % r]));
            y[(size_t)(base + q * Ns) * B + b] = acc;
          }
        }
      }
    }
  }
}

/* out = DFT(in) for B interleaved transforms (layout [n][B]); in and out
 * may alias.  scratch: B * fft1d_scratch(p) elements. */
static void fft1d_exec_b(const fft1d *p, const cpx *in, cpx *out,
                         cpx *scratch, int B) {
  const int n = p->n;
  if (n == 1) {
    if (in != out) memcpy(out, in, sizeof(cpx) * B);
    return;
  }
  if (p->blue) {
    for (int b = 0; b < B; ++b) {
      /* Bluestein runs one transform at a time on a contiguous copy. */
      const int m = p->m;
      cpx *a = scratch;
      cpx *A = scratch + m;
      cpx *tmp = scratch + 2 * m; /* 2m for the inner Stockham */
      for (int j = 0; j < n; ++j) a[j] = cmul(in[(size_t)j * B + b], p->chirp[j]);
      for (int j = n; j < m; ++j) a[j].re = a[j].im = 0.0;
      fft1d_exec_b(p->mf, a, A, tmp, 1);
      for (int j = 0; j < m; ++j) A[j] = cmul(A[j], p->bfft[j]);
      fft1d_exec_b(p->mb, A, a, tmp, 1);
      for (int k = 0; k < n; ++k) out[(size_t)k * B + b] = cmul(a[k], p->chirp[k]);
    }
    return;
  }
  const int K = p->nstage;
  cpx *bufs[2] = {out, scratch};
  const cpx *src = in;
  if (in == out && (K % 2 == 1)) {
    memcpy(scratch + (size_t)n * B, in, sizeof(cpx) * (size_t)n * B);
    src = scratch + (size_t)n * B;
  }
  for (int s = 0; s < K; ++s) {
    cpx *dst = bufs[(K - 1 - s) % 2];
    stockham_pass(n, p->radix[s], p->ns[s], p->tw[s], p->roots[s], p->sign,
                  src, dst, B);
    src = dst;
  }
}

void fc_shim_fft1d_exec(const fft1d *p, const cpx *in, cpx *out,
                        cpx *scratch) {
  fft1d_exec_b(p, in, out, scratch, 1);
}

/* ------------------------------------------------------------------------- */
/* Plans                                                                     */
/* ------------------------------------------------------------------------- */

enum { KIND_R2C = 0, KIND_C2R = 1, KIND_C2C = 2 };

struct fc_shim_plan_s {
  int kind;
  int rank;
  int n[3];
  int howmany;
  /* r2c / c2r: strides of the real and complex arrays per dimension. */
  long rs[3], cs[3];
  long rdist, cdist;
  /* c2c: strides of the input and output arrays. */
  long is[3], os[3];
  long idist, odist;
  int sign;
  void *in;
  void *out;
  fft1d *f[3];    /* complex plans for dims 0..rank-2 (and all dims, c2c) */
  fft1d *last;    /* last-dim plan: half length (even) or full (odd) */
  cpx *rtw;       /* e^{-2 pi i k / n}, k <= n/2, even last dim */
  int half;
};

static void strides_from_embed(int rank, const int *n, const int *embed,
                               int last_override, long stride, long *out) {
  long acc = stride;
  for (int d = rank - 1; d >= 0; --d) {
    out[d] = acc;
    int extent = embed ? embed[d] : (d == rank - 1 && last_override > 0
                                          ? last_override
                                          : n[d]);
    acc *= extent;
  }
}

static fftw_plan make_real_plan(int kind, int rank, const int *n, int howmany,
                                void *in, const int *inembed, int istride,
                                int idist, void *out, const int *onembed,
                                int ostride, int odist) {
  if (rank < 1 || rank > 3) {
    fprintf(stderr, "fftw shim: unsupported rank %d\n", rank);
    return NULL;
  }
  fftw_plan p = (fftw_plan)calloc(1, sizeof(struct fc_shim_plan_s));
  p->kind = kind;
  p->rank = rank;
  for (int d = 0; d < rank; ++d) p->n[d] = n[d];
  p->howmany = howmany;
  const int nh = n[rank - 1] / 2 + 1;
  if (kind == KIND_R2C) {
    strides_from_embed(rank, n, inembed, 0, istride, p->rs);
    strides_from_embed(rank, n, onembed, nh, ostride, p->cs);
    p->rdist = idist;
    p->cdist = odist;
    p->sign = -1;
  } else {
    strides_from_embed(rank, n, inembed, nh, istride, p->cs);
    strides_from_embed(rank, n, onembed, 0, ostride, p->rs);
    p->cdist = idist;
    p->rdist = odist;
    p->sign = +1;
  }
  p->in = in;
  p->out = out;
  for (int d = 0; d < rank - 1; ++d) p->f[d] = fft1d_create(n[d], p->sign);
  const int nl = n[rank - 1];
  p->half = (nl % 2 == 0) && nl >= 2;
  if (p->half) {
    p->last = fft1d_create(nl / 2, p->sign);
    p->rtw = (cpx *)malloc(sizeof(cpx) * (nl / 2 + 1));
    for (int k = 0; k <= nl / 2; ++k) p->rtw[k] = unit_root(-1, k, nl);
  } else {
    p->last = fft1d_create(nl, p->sign);
  }
  return p;
}

fftw_plan fftw_plan_many_dft_r2c(int rank, const int *n, int howmany,
                                 double *in, const int *inembed, int istride,
                                 int idist, fftw_complex *out,
                                 const int *onembed, int ostride, int odist,
                                 unsigned flags) {
  (void)flags;
  return make_real_plan(KIND_R2C, rank, n, howmany, in, inembed, istride,
                        idist, out, onembed, ostride, odist);
}

fftw_plan fftw_plan_many_dft_c2r(int rank, const int *n, int howmany,
                                 fftw_complex *in, const int *inembed,
                                 int istride, int idist, double *out,
                                 const int *onembed, int ostride, int odist,
                                 unsigned flags) {
  (void)flags;
  return make_real_plan(KIND_C2R, rank, n, howmany, in, inembed, istride,
                        idist, out, onembed, ostride, odist);
}

fftw_plan fftw_plan_many_dft(int rank, const int *n, int howmany,
                             fftw_complex *in, const int *inembed, int istride,
                             int idist, fftw_complex *out, const int *onembed,
                             int ostride, int odist, int sign,
                             unsigned flags) {
  (void)flags;
  if (rank < 1 || rank > 3) {
    fprintf(stderr, "fftw shim: unsupported rank %d\n", rank);
    return NULL;
  }
  fftw_plan p = (fftw_plan)calloc(1, sizeof(struct fc_shim_plan_s));
  p->kind = KIND_C2C;
  p->rank = rank;
  for (int d = 0; d < rank; ++d) p->n[d] = n[d];
  p->howmany = howmany;
  strides_from_embed(rank, n, inembed, 0, istride, p->is);
  strides_from_embed(rank, n, onembed, 0, ostride, p->os);
  p->idist = idist;
  p->odist = odist;
  p->sign = sign < 0 ? -1 : +1;
  p->in = in;
  p->out = out;
  for (int d = 0; d < rank; ++d) p->f[d] = fft1d_create(n[d], p->sign);
  return p;
}

void fftw_destroy_plan(fftw_plan p) {
  if (!p) return;
  for (int d = 0; d < 3; ++d) fft1d_destroy(p->f[d]);
  fft1d_destroy(p->last);
  free(p->rtw);
  free(p);
}

/* ------------------------------------------------------------------------- */
/* Strided batches of complex transforms                                     */
/* ------------------------------------------------------------------------- */

/* Transforms t = 0..count-1 of length f->n: element i of transform t lives at
 * in[t*dist + i*s] and goes to out[t*dist + i*s].  Adjacent transforms are
 * gathered in blocks, interleaved, so that small dist values read whole cache
 * lines and the butterflies run across the block. */
static void many_c2c(const fft1d *f, long s, int count, long dist,
                     const cpx *in, cpx *out) {
  const int n = f->n;
  cpx *blk = (cpx *)malloc(sizeof(cpx) * (size_t)BLOCK * n);
  cpx *scr = (cpx *)malloc(sizeof(cpx) * fft1d_scratch_b(f, BLOCK));
  for (int t0 = 0; t0 < count; t0 += BLOCK) {
    const int nb = count - t0 < BLOCK ? count - t0 : BLOCK;
    for (int i = 0; i < n; ++i)
      for (int b = 0; b < nb; ++b)
        blk[(size_t)i * nb + b] = in[(t0 + b) * dist + i * s];
    fft1d_exec_b(f, blk, blk, scr, nb);
    for (int i = 0; i < n; ++i)
      for (int b = 0; b < nb; ++b)
        out[(t0 + b) * dist + i * s] = blk[(size_t)i * nb + b];
  }
  free(scr);
  free(blk);
}

/* Complex DFT along dimension d of an array with the given extents and
 * strides (in place when in == out). */
static void c2c_along(const fft1d *f, int rank, const int *ext, const long *is,
                      const long *os, int d, const cpx *in, cpx *out) {
  /* Choose the "batch" dimension: the last dimension unless d is last. */
  int bd = (d == rank - 1) ? (rank >= 2 ? rank - 2 : -1) : rank - 1;
  if (bd < 0) {
    many_c2c(f, is[d], 1, 0, in, out);
    return;
  }
  if (is[d] != os[d] || is[bd] != os[bd]) {
    fprintf(stderr, "fftw shim: mismatched strides in c2c_along\n");
    abort();
  }
  /* Iterate over the remaining dimension (at most one for rank 3). */
  int od = -1;
  for (int e = 0; e < rank; ++e)
    if (e != d && e != bd) od = e;
  const int no = od >= 0 ? ext[od] : 1;
  for (int io = 0; io < no; ++io) {
    const long ioff = od >= 0 ? io * is[od] : 0;
    const long ooff = od >= 0 ? io * os[od] : 0;
    many_c2c(f, is[d], ext[bd], is[bd], in + ioff, out + ooff);
  }
}

/* ------------------------------------------------------------------------- */
/* Real transforms along the last dimension                                  */
/* ------------------------------------------------------------------------- */

/* Real transforms of nb rows along the last dimension.  Row b starts at
 * x + b*xr (element stride xs) and its n/2+1 outputs at X + b*Xr (stride
 * Xs).  Input and output rows may alias: every row is read before any output
 * row is written. */
static void r2c_rows(const struct fc_shim_plan_s *p, const double *x, long xr,
                     long xs, cpx *X, long Xr, long Xs, int nb, cpx *buf,
                     cpx *scr) {
  const int n = p->n[p->rank - 1];
  if (p->half) {
    const int h = n / 2;
    cpx *z = buf;
    cpx *Z = buf + (size_t)h * nb;
    for (int j = 0; j < h; ++j)
      for (int b = 0; b < nb; ++b) {
        z[(size_t)j * nb + b].re = x[b * xr + (2 * j) * xs];
        z[(size_t)j * nb + b].im = x[b * xr + (2 * j + 1) * xs];
      }
    fft1d_exec_b(p->last, z, Z, scr, nb);
    for (int k = 0; k <= h; ++k) {
      const cpx w = p->rtw[k];
      const cpx *Zk = Z + (size_t)(k % h) * nb;
      const cpx *Zm = Z + (size_t)((h - k) % h) * nb;
      for (int b = 0; b < nb; ++b) {
        cpx a = Zk[b];
        cpx c = cconj(Zm[b]);
        cpx E = {0.5 * (a.re + c.re), 0.5 * (a.im + c.im)};
        /* O = (a - c) / (2i) = -i (a - c) / 2 */
        cpx D = csub(a, c);
        cpx O = {0.5 * D.im, -0.5 * D.re};
        X[b * Xr + k * Xs] = cadd(E, cmul(w, O));
      }
    }
  } else {
    cpx *z = buf;
    cpx *Z = buf + (size_t)n * nb;
    for (int j = 0; j < n; ++j)
      for (int b = 0; b < nb; ++b) {
        z[(size_t)j * nb + b].re = x[b * xr + j * xs];
        z[(size_t)j * nb + b].im = 0.0;
      }
    fft1d_exec_b(p->last, z, Z, scr, nb);
    for (int k = 0; k <= n / 2; ++k)
      for (int b = 0; b < nb; ++b) X[b * Xr + k * Xs] = Z[(size_t)k * nb + b];
  }
}

/* Inverse of r2c_rows (unnormalised).  The DC and Nyquist terms of a
 * Hermitian sequence are real, so their imaginary parts are ignored. */
static void c2r_rows(const struct fc_shim_plan_s *p, const cpx *X, long Xr,
                     long Xs, double *x, long xr, long xs, int nb, cpx *buf,
                     cpx *scr) {
  const int n = p->n[p->rank - 1];
  if (p->half) {
    const int h = n / 2;
    cpx *Xc = buf;                         /* (h+1) * nb */
    cpx *Z = buf + (size_t)(h + 1) * nb;   /* h * nb */
    cpx *z = Z + (size_t)h * nb;           /* h * nb */
    for (int k = 0; k <= h; ++k)
      for (int b = 0; b < nb; ++b) Xc[(size_t)k * nb + b] = X[b * Xr + k * Xs];
    for (int b = 0; b < nb; ++b) {
      Xc[b].im = 0.0;
      Xc[(size_t)h * nb + b].im = 0.0;
    }
    for (int k = 0; k < h; ++k) {
      const cpx w = cconj(p->rtw[k]); /* e^{+2 pi i k/n} */
      for (int b = 0; b < nb; ++b) {
        cpx a = Xc[(size_t)k * nb + b];
        cpx c = cconj(Xc[(size_t)(h - k) * nb + b]);
        cpx E = cadd(a, c);
        cpx O = cmul(csub(a, c), w);
        Z[(size_t)k * nb + b].re = E.re - O.im;
        Z[(size_t)k * nb + b].im = E.im + O.re;
      }
    }
    fft1d_exec_b(p->last, Z, z, scr, nb);
    for (int j = 0; j < h; ++j)
      for (int b = 0; b < nb; ++b) {
        x[b * xr + (2 * j) * xs] = z[(size_t)j * nb + b].re;
        x[b * xr + (2 * j + 1) * xs] = z[(size_t)j * nb + b].im;
      }
  } else {
    cpx *Y = buf;
    cpx *y = buf + (size_t)n * nb;
    for (int b = 0; b < nb; ++b) {
      Y[b].re = X[b * Xr].re;
      Y[b].im = 0.0;
    }
    for (int k = 1; k <= n / 2; ++k)
      for (int b = 0; b < nb; ++b) {
        Y[(size_t)k * nb + b] = X[b * Xr + k * Xs];
        Y[(size_t)(n - k) * nb + b] = cconj(Y[(size_t)k * nb + b]);
      }
    fft1d_exec_b(p->last, Y, y, scr, nb);
    for (int j = 0; j < n; ++j)
      for (int b = 0; b < nb; ++b) x[b * xr + j * xs] = y[(size_t)j * nb + b].re;
  }
}

static void exec_real(const struct fc_shim_plan_s *p, double *r, cpx *c) {
  const int rank = p->rank;
  const int nl = p->n[rank - 1];
  int cext[3];
  for (int d = 0; d < rank; ++d) cext[d] = p->n[d];
  cext[rank - 1] = nl / 2 + 1;
  cpx *buf = (cpx *)malloc(sizeof(cpx) * (3 * (size_t)nl + 4) * BLOCK);
  cpx *scr = (cpx *)malloc(sizeof(cpx) * fft1d_scratch_b(p->last, BLOCK));
  /* Rows: outer index i0 (rank 3 only) and a blocked row index i1. */
  const int n0 = rank == 3 ? p->n[0] : 1;
  const int n1 = rank >= 2 ? p->n[rank - 2] : 1;
  const long rr = rank >= 2 ? p->rs[rank - 2] : 0;
  const long cr = rank >= 2 ? p->cs[rank - 2] : 0;
  for (int b = 0; b < p->howmany; ++b) {
    double *x = r + b * p->rdist;
    cpx *X = c + b * p->cdist;
    if (p->kind == KIND_C2R)
      for (int d = 0; d <= rank - 2; ++d)
        c2c_along(p->f[d], rank, cext, p->cs, p->cs, d, X, X);
    for (int i0 = 0; i0 < n0; ++i0) {
      const long ro = rank == 3 ? i0 * p->rs[0] : 0;
      const long co = rank == 3 ? i0 * p->cs[0] : 0;
      for (int i1 = 0; i1 < n1; i1 += BLOCK) {
        const int nb = n1 - i1 < BLOCK ? n1 - i1 : BLOCK;
        if (p->kind == KIND_R2C)
          r2c_rows(p, x + ro + i1 * rr, rr, p->rs[rank - 1], X + co + i1 * cr,
                   cr, p->cs[rank - 1], nb, buf, scr);
        else
          c2r_rows(p, X + co + i1 * cr, cr, p->cs[rank - 1], x + ro + i1 * rr,
                   rr, p->rs[rank - 1], nb, buf, scr);
      }
    }
    if (p->kind == KIND_R2C)
      for (int d = rank - 2; d >= 0; --d)
        c2c_along(p->f[d], rank, cext, p->cs, p->cs, d, X, X);
  }
  free(scr);
  free(buf);
}

static void exec_c2c(const struct fc_shim_plan_s *p, cpx *in, cpx *out) {
  const int rank = p->rank;
  if (rank == 1) {
    if (in != out && (p->is[0] != p->os[0] || p->idist != p->odist)) {
      fprintf(stderr, "fftw shim: out-of-place rank-1 c2c needs equal layouts\n");
      abort();
    }
    many_c2c(p->f[0], p->is[0], p->howmany, p->idist, in, out);
    return;
  }
  for (int b = 0; b < p->howmany; ++b) {
    const cpx *x = in + b * p->idist;
    cpx *y = out + b * p->odist;
    int ext[3];
    for (int d = 0; d < rank; ++d) ext[d] = p->n[d];
    if (x != y) {
      /* Copy to the output layout first, then transform in place. */
      long tot = 1;
      for (int d = 0; d < rank; ++d) tot *= ext[d];
      for (long lin = 0; lin < tot; ++lin) {
        long rem = lin;
        long io = 0, oo = 0;
        for (int d = rank - 1; d >= 0; --d) {
          long id = rem % ext[d];
          rem /= ext[d];
          io += id * p->is[d];
          oo += id * p->os[d];
        }
        y[oo] = x[io];
      }
    }
    for (int d = rank - 1; d >= 0; --d)
      c2c_along(p->f[d], rank, ext, p->os, p->os, d, y, y);
  }
}

void fftw_execute(const fftw_plan p) {
  if (!p) return;
  if (p->kind == KIND_R2C)
    exec_real(p, (double *)p->in, (cpx *)p->out);
  else if (p->kind == KIND_C2R)
    exec_real(p, (double *)p->out, (cpx *)p->in);
  else
    exec_c2c(p, (cpx *)p->in, (cpx *)p->out);
}

void fftw_execute_dft_r2c(const fftw_plan p, double *in, fftw_complex *out) {
  exec_real(p, in, (cpx *)out);
}

void fftw_execute_dft_c2r(const fftw_plan p, fftw_complex *in, double *out) {
  exec_real(p, out, (cpx *)in);
}

void fftw_execute_dft(const fftw_plan p, fftw_complex *in, fftw_complex *out) {
  exec_c2c(p, (cpx *)in, (cpx *)out);
}

void fftw_cleanup(void) {}
void fftw_cleanup_threads(void) {}
int fftw_init_threads(void) { return 1; }
void fftw_plan_with_nthreads(int nthreads) { (void)nthreads; }

/* The shim keeps no wisdom; these mirror FFTW's return conventions. */
int fftw_import_wisdom_from_filename(const char *filename) {
  FILE *f = fopen(filename, "r");
  if (!f) return 0;
  fclose(f);
  return 1;
}

int fftw_export_wisdom_to_filename(const char *filename) {
  FILE *f = fopen(filename, "w");
  if (!f) return 0;
  fprintf(f, "(fftw-3.3-shim-wisdom)\n");
  fclose(f);
  return 1;
}

void fftw_forget_wisdom(void) {}
