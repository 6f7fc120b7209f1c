/*
 * ORACLE — test infrastructure only.
 *
 * A plain-C CPU restatement of the Lucas-Lehmer squaring step of CUDALucas
 * v2.06 (IBDWT in FP64), used as the checker for the CUDA engine and as the
 * timed host-core baseline.  The loops over independent butterflies, pairs
 * and carry blocks can be split over several host threads
 * (oracle_set_threads, POSIX threads); every output word is computed by the
 * same arithmetic whatever the thread count, so results do not depend on it.  Only tests/, the smoke check
 * and bench.py's cpu_baseline leg may load it; the product never does.
 *
 * Each function names the reference code it follows (file:line within the
 * CUDALucas project).  The one substitution is the FFT: the reference calls
 * cuFFT (a closed library, CUDALucas.cu:1239/1888/1890, both CUFFT_INVERSE,
 * i.e. exponent sign +1, unnormalised); here it is a mixed-radix (2,3,4,5,7)
 * Stockham FFT with the same sign and scaling.  Because the rounded integer
 * digits do not depend on the last bits of the FFT output, the digit vectors
 * produced here match the reference's whenever no roundoff approaches 0.5.
 *
 * Parity pin: the Res64 values this oracle produces after 10000 iterations
 * are checked against the self-test table of CUDALucas.cu:2673-2729 and
 * against exact big-integer arithmetic (oracle/exact.py).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct { double re, im; } cplx;

/* ------------------------------------------------------ host threads -- */
/* par_for(count, fn, arg): fn(arg, lo, hi, slot) over [0, count) split into
 * contiguous ranges, one per thread (slot = range index < g_threads). */
#define ORACLE_MAX_THREADS 256
static int g_threads = 1;
typedef void (*range_fn)(void *arg, int lo, int hi, int slot);
typedef struct { range_fn fn; void *arg; int lo, hi, slot; } par_job;

static void *par_run(void *p) {
  par_job *j = (par_job *)p;
  j->fn(j->arg, j->lo, j->hi, j->slot);
  return NULL;
}

static void par_for(int count, range_fn fn, void *arg) {
  int t = g_threads < count ? g_threads : count;
  if (t <= 1) { fn(arg, 0, count, 0); return; }
  pthread_t th[ORACLE_MAX_THREADS];
  par_job jobs[ORACLE_MAX_THREADS];
  int started[ORACLE_MAX_THREADS];
  for (int i = 0; i < t; i++) {
    jobs[i].fn = fn; jobs[i].arg = arg; jobs[i].slot = i;
    jobs[i].lo = (int)((long long)count * i / t);
    jobs[i].hi = (int)((long long)count * (i + 1) / t);
    started[i] = i > 0 && pthread_create(&th[i], NULL, par_run, &jobs[i]) == 0;
    if (i > 0 && !started[i]) par_run(&jobs[i]);  /* no thread: run it here */
  }
  par_run(&jobs[0]);
  for (int i = 1; i < t; i++) if (started[i]) pthread_join(th[i], NULL);
}

/* ------------------------------------------------------------------ FFT -- */
/* Mixed-radix Stockham FFT, exponent sign +1 (cuFFT's CUFFT_INVERSE),
 * unnormalised.  Twiddles are computed in long double and rounded once. */
typedef struct {
  int len;
  int nst;
  int radix[64];
  cplx *tw;      /* tw[e] = exp(+2 pi i e / len) */
  cplx *tmp;
} fft_plan;

static int fft_plan_init(fft_plan *p, int len) {
  int m = len, k = 0;
  static const int rs[] = {4, 2, 3, 5, 7};
  memset(p, 0, sizeof(*p));
  p->len = len;
  while (m > 1) {
    int found = 0;
    for (int i = 0; i < 5; i++) {
      if (m % rs[i] == 0) { p->radix[k++] = rs[i]; m /= rs[i]; found = 1; break; }
    }
    if (!found) return -1;
  }
  p->nst = k;
  p->tw = (cplx *)malloc(sizeof(cplx) * (size_t)len);
  p->tmp = (cplx *)malloc(sizeof(cplx) * (size_t)len);
  if (!p->tw || !p->tmp) return -1;
  for (int e = 0; e < len; e++) {
    long double a = 2.0L * 3.14159265358979323846264338327950288L * (long double)e / (long double)len;
    p->tw[e].re = (double)cosl(a);
    p->tw[e].im = (double)sinl(a);
  }
  return 0;
}

static void fft_plan_free(fft_plan *p) { free(p->tw); free(p->tmp); }

static inline cplx cmul(cplx a, cplx b) {
  cplx r = {a.re * b.re - a.im * b.im, a.re * b.im + a.im * b.re};
  return r;
}

/* one Stockham stage: butterflies j in [lo, hi) */
typedef struct { const fft_plan *p; const cplx *in; cplx *out; int R, m, ns; } fft_stage;

static void fft_stage_range(void *arg, int lo, int hi, int slot) {
  const fft_stage *st = (const fft_stage *)arg;
  const fft_plan *p = st->p;
  const int L = p->len, R = st->R, m = st->m, ns = st->ns;
  const cplx *in = st->in;
  cplx *out = st->out;
  cplx v[7], w[7];
  (void)slot;
  for (int j = lo; j < hi; j++) {
    int k = j % ns;
    for (int r = 0; r < R; r++) {
      v[r] = in[j + r * m];
      if (r && k) v[r] = cmul(v[r], p->tw[(size_t)r * k * (L / (ns * R)) % L]);
    }
    if (R == 2) {
      w[0].re = v[0].re + v[1].re; w[0].im = v[0].im + v[1].im;
      w[1].re = v[0].re - v[1].re; w[1].im = v[0].im - v[1].im;
    } else if (R == 4) {
      /* sign +1: multiply by +i on the odd difference */
      cplx s0 = {v[0].re + v[2].re, v[0].im + v[2].im}, d0 = {v[0].re - v[2].re, v[0].im - v[2].im};
      cplx s1 = {v[1].re + v[3].re, v[1].im + v[3].im}, d1 = {v[1].re - v[3].re, v[1].im - v[3].im};
      w[0].re = s0.re + s1.re; w[0].im = s0.im + s1.im;
      w[2].re = s0.re - s1.re; w[2].im = s0.im - s1.im;
      w[1].re = d0.re - d1.im; w[1].im = d0.im + d1.re;
      w[3].re = d0.re + d1.im; w[3].im = d0.im - d1.re;
    } else {
      /* direct DFT_R for the odd radices 3, 5, 7 */
      for (int a = 0; a < R; a++) {
        cplx acc = v[0];
        for (int c = 1; c < R; c++) {
          cplx t = cmul(v[c], p->tw[(size_t)((a * c) % R) * (L / R)]);
          acc.re += t.re; acc.im += t.im;
        }
        w[a] = acc;
      }
    }
    int base = (j / ns) * ns * R + k;
    for (int r = 0; r < R; r++) out[base + r * ns] = w[r];
  }
}

/* in-place, sign +1 */
static void fft_exec(fft_plan *p, cplx *x) {
  int L = p->len, ns = 1;
  cplx *in = x, *out = p->tmp;
  for (int s = 0; s < p->nst; s++) {
    fft_stage st = {p, in, out, p->radix[s], L / p->radix[s], ns};
    par_for(st.m, fft_stage_range, &st);
    ns *= st.R;
    cplx *t = in; in = out; out = t;
  }
  if (in != x) memcpy(x, in, sizeof(cplx) * (size_t)L);
}

/* -------------------------------------------------------------- context -- */
typedef struct {
  int q, n, b, qn;
  int sc;                 /* log2 of rcb block size, CUDALucas.cu:1875-1880 */
  int bigcarry;           /* BigCarry=1 selects rcbl/splicel */
  double *x;              /* g_x */
  double *ct;             /* g_ct, CUDALucas.cu:1149 */
  double *ttp;            /* g_ttp: [32 x (ttp,ttmp) col][n/32 x (ttp,ttmp) grp] */
  unsigned *s;            /* g_s: [n/32 x (big-word bits, weight>=2 bits)] */
  unsigned *size1;        /* host g_size1 (big-word bitmap) */
  double *ttp1;           /* splice weights, CUDALucas.cu:1222-1237 */
  double ttpinc[2];
  int *xint;
  int *data;
  long long *carry;
  float err;
  int offset;
  fft_plan plan;
} oracle_ctx;

/* write_gpu_data, CUDALucas.cu:1125-1252 */
static void write_tables(oracle_ctx *c) {
  int q = c->q, n = c->n, b = c->b;
  double d = 2.0 / (double)n;
  double ttp_col[32], ttmp_col[32];
  double *ttp_grp = (double *)malloc(sizeof(double) * (size_t)(n / 32));
  double *ttmp_grp = (double *)malloc(sizeof(double) * (size_t)(n / 32));
  unsigned *s1 = (unsigned *)malloc(sizeof(unsigned) * (size_t)(n / 32));
  int i, j;
  (void)q;
  /* CUDALucas.cu:1149 ct[j] = 0.5 cospi(j*2/n) */
  for (j = (n >> 2) - 1; j > 0; j--)
    c->ct[j] = 0.5 * (double)cosl(3.14159265358979323846264338327950288L * (long double)(j * d));
  c->ct[0] = 0;
  d *= 0.5;
  /* column data, CUDALucas.cu:1154-1164 */
  i = 0;
  for (j = 0; j < 32; j++) {
    ttp_col[j] = exp2(i * d);
    ttmp_col[j] = exp2(-i * d) * 2.0 * d;
    if (j & 1) ttmp_col[j] = -ttmp_col[j];
    i -= b;
    if (i < 0) i += n;
  }
  /* group data, CUDALucas.cu:1166-1174 (64-bit product to avoid overflow) */
  {
    long long ii = 0;
    for (j = 0; j < n / 32; j++) {
      ttp_grp[j] = exp2((double)ii * d);
      ttmp_grp[j] = exp2(-(double)ii * d);
      ii -= (long long)b * 32;
      while (ii < 0) ii += n;
    }
  }
  for (j = 0; j < 32; j++) { c->ttp[j * 2] = ttp_col[j]; c->ttp[j * 2 + 1] = ttmp_col[j]; }
  for (j = 0; j < n / 32; j++) { c->ttp[j * 2 + 64] = ttp_grp[j]; c->ttp[j * 2 + 65] = ttmp_grp[j]; }
  /* CUDALucas.cu:1188-1192 */
  c->ttpinc[0] = exp2((n - b) * d);
  c->ttpinc[1] = exp2(-b * d);
  /* big-word and weight>=2 bitmaps, CUDALucas.cu:1194-1220 */
  {
    double comp1 = exp2(b * d) - 0.000000001;
    double comp2 = 2.0 * comp1;
    for (j = 0; j < n / 32; j++) {
      c->size1[j] = 0;
      s1[j] = 0;
      for (i = 31; i >= 0; i--) {
        double dd = ttp_col[i] * ttp_grp[j];
        c->size1[j] <<= 1;
        s1[j] <<= 1;
        if (dd >= 2.0) {
          s1[j]++;
          if (dd < comp2) c->size1[j]++;
        } else if (dd < comp1) c->size1[j]++;
      }
    }
    for (j = 0; j < n / 32; j++) { c->s[j * 2] = c->size1[j]; c->s[j * 2 + 1] = s1[j]; }
  }
  /* splice weights: weight of the first word of each rcb block with the
   * big-word flag in the sign bit (CUDALucas.cu:1222-1237, indexed directly
   * by block here instead of through the g_ttp1 pointer offset). */
  {
    int bw = 1 << c->sc, nb = n / bw;
    for (j = 0; j < nb; j++) {
      int w = j * bw;
      double t = ttp_grp[w >> 5];  /* column 0 has weight 1 */
      if (c->size1[w >> 5] & 1) t = -t;
      c->ttp1[j] = t;
    }
  }
  free(ttp_grp); free(ttmp_grp); free(s1);
}

static inline int big_word(const oracle_ctx *c, int j) { return (c->size1[j >> 5] >> (j & 31)) & 1; }

oracle_ctx *oracle_create(int q, int n, int bigcarry) {
  oracle_ctx *c = (oracle_ctx *)calloc(1, sizeof(oracle_ctx));
  if (!c) return NULL;
  if (n % 1024 || q <= n) { free(c); return NULL; }
  c->q = q; c->n = n; c->b = q % n; c->qn = q / n; c->bigcarry = bigcarry;
  /* CUDALucas.cu:1875-1880 (B1=10240, B2=49152, B3=98304) */
  c->sc = n >= 98304 ? 10 : n >= 49152 ? 9 : n >= 10240 ? 8 : 7;
  c->x = (double *)calloc((size_t)n, sizeof(double));
  c->ct = (double *)calloc((size_t)n / 4, sizeof(double));
  c->ttp = (double *)calloc((size_t)n / 16 + 64, sizeof(double));
  c->s = (unsigned *)calloc((size_t)n / 16, sizeof(unsigned));
  c->size1 = (unsigned *)calloc((size_t)n / 32, sizeof(unsigned));
  c->ttp1 = (double *)calloc((size_t)(n >> c->sc), sizeof(double));
  c->xint = (int *)calloc((size_t)n, sizeof(int));
  c->data = (int *)calloc((size_t)(2 * (n >> c->sc)), sizeof(int));
  c->carry = (long long *)calloc((size_t)(n >> c->sc), sizeof(long long));
  if (fft_plan_init(&c->plan, n / 2)) { free(c); return NULL; }
  write_tables(c);
  return c;
}

void oracle_destroy(oracle_ctx *c) {
  if (!c) return;
  free(c->x); free(c->ct); free(c->ttp); free(c->s); free(c->size1); free(c->ttp1);
  free(c->xint); free(c->data); free(c->carry);
  fft_plan_free(&c->plan);
  free(c);
}

/* apply_weights, CUDALucas.cu:216-249 */
typedef struct { oracle_ctx *c; const int *in; } weights_job;

static void apply_weights_range(void *arg, int lo, int hi, int slot) {
  oracle_ctx *c = ((weights_job *)arg)->c;
  const int *in = ((weights_job *)arg)->in;
  (void)slot;
  for (int idx = lo; idx < hi; idx++) {
    int grp = idx >> 5, col = idx & 31;
    double tc = c->ttp[col << 1];
    if (c->s[grp * 2 + 1] & (1u << col)) tc *= 0.5;
    c->x[idx] = (double)in[idx] * c->ttp[grp * 2 + 64] * tc;
  }
}

static void apply_weights(oracle_ctx *c, const int *in) {
  weights_job job = {c, in};
  par_for(c->n, apply_weights_range, &job);
}

/* init_x, CUDALucas.cu:1254-1278, with the offset supplied by the caller
 * instead of rand() % q.  digits == NULL starts a fresh test at 4*2^offset. */
void oracle_init(oracle_ctx *c, const int *digits, int offset) {
  int n = c->n, q = c->q;
  if (!digits) {
    int bit = (offset + 2) % q;
    int digit = (int)(((long long)bit * n) / q);
    int sd = (int)(((long long)digit * q + n - 1) / n);
    memset(c->xint, 0, sizeof(int) * (size_t)n);
    c->xint[digit] = 1 << (bit - sd);
  } else {
    memcpy(c->xint, digits, sizeof(int) * (size_t)n);
  }
  c->offset = offset;
  c->err = 0;
  apply_weights(c, c->xint);
}

/* square, CUDALucas.cu:255-314 */
static void square_range(void *arg, int lo, int hi, int slot) {
  oracle_ctx *c = (oracle_ctx *)arg;
  int n = c->n, nc0 = n >> 2;
  double *a = c->x, *ct = c->ct;
  (void)slot;
  /* pair jj touches words 2jj, 2jj+1, n-2jj, n-2jj+1 only: independent */
  for (int jj = lo; jj < hi; jj++) {
    int j = jj, nc;
    double wkr, wki, xr, xi, yr, aj, aj1, ak, ak1;
    if (j) {
      wkr = 0.5 - ct[nc0 - j];
      wki = ct[j];
      j <<= 1;
      nc = n - j;
      aj = a[j]; aj1 = a[1 + j]; ak = a[nc]; ak1 = a[1 + nc];
      xr = aj - ak; xi = aj1 + ak1;
      yr = wkr * xr - wki * xi;
      xi = wkr * xi + wki * xr;
      aj -= yr; aj1 -= xi; ak += yr; ak1 -= xi;
      xr = (aj - aj1) * (aj + aj1);
      xi = 2.0 * aj * aj1;
      yr = (ak - ak1) * (ak + ak1);
      ak = 2.0 * ak * ak1;
      aj1 = xr - yr;
      ak1 = xi + ak;
      aj = wkr * aj1 + wki * ak1;
      aj1 = wkr * ak1 - wki * aj1;
      a[j] = xr - aj;
      a[1 + j] = aj1 - xi;
      a[nc] = yr + aj;
      a[1 + nc] = aj1 - ak;
    } else {
      j = n >> 1;
      aj = a[0]; aj1 = a[1];
      xi = aj - aj1; aj += aj1;
      xi *= xi; aj *= aj;
      aj1 = 0.5 * (xi - aj);
      a[0] = aj + aj1;
      a[1] = aj1;
      xr = a[j]; xi = a[1 + j];
      a[j] = (xr + xi) * (xr - xi);
      a[1 + j] = -2.0 * xr * xi;
    }
  }
}

static void square(oracle_ctx *c) { par_for(c->n >> 2, square_range, c); }

/* rcb / rcbl, CUDALucas.cu:322-484 and :536-679.  The 128-thread block is
 * simulated one row of 128 words at a time; `wide` selects the 64-bit carry
 * arithmetic of rcbl, otherwise carries are truncated to int as in rcb. */
typedef struct {
  oracle_ctx *c;
  int report, digit, bit;
  float err[ORACLE_MAX_THREADS];
} rcb_job;

/* the blocks are independent: each writes its own words and its own
 * outgoing carry, which splice applies afterwards */
static void rcb_range(void *arg, int lo, int hi, int slot) {
  rcb_job *job = (rcb_job *)arg;
  oracle_ctx *c = job->c;
  const int report = job->report, digit = job->digit, bit = job->bit;
  const int TT = 128;
  int sc = c->sc, nblk = c->n >> sc;
  long long carry[257];
  float err = 0;
  for (int blk = lo; blk < hi; blk++) {
    long long cfns = 0;
    float ferr_max = 0;
    for (int row = 0; row < (1 << sc) / TT; row++) {
      long long bigint[128], val[128];
      int nb[128];
      for (int t = 0; t < TT; t++) {
        int index = (blk << sc) + row * TT + t;
        int grp = index >> 5, col = index & 31;
        double ttmp = c->ttp[grp * 2 + 65] * c->ttp[col * 2 + 1];
        if (c->s[grp * 2 + 1] & (1u << col)) ttmp *= 2.0;  /* ttmp_col[col+32] = 2*ttmp_col */
        int numbits = c->qn + ((c->s[grp * 2] >> col) & 1);
        double tval = c->x[index] * ttmp;
        double trint = nearbyint(tval);  /* cvt.rni: round half to even */
        float ferr = fabsf((float)(tval - trint));
        if (ferr > ferr_max) ferr_max = ferr;
        bigint[t] = (long long)trint;
        if (index == digit) bigint[t] -= bit;
        if (t == 0) bigint[t] += cfns;
        nb[t] = numbits;
      }
      if (c->bigcarry) {
        for (int t = 0; t < TT; t++) {
          long long mask = (long long)(~0ULL << nb[t]);
          carry[t + 1] = bigint[t] >> nb[t];
          val[t] = bigint[t] & ~mask;
        }
        for (int t = 0; t < TT; t++) {
          long long mask = (long long)(~0ULL << nb[t]);
          if (t) val[t] += carry[t];
          long long sh = val[t] - (mask >> 1);
          val[t] -= sh & mask;
          carry[t] = sh >> nb[t];
        }
        for (int t = 0; t < TT; t++) if (t) val[t] += carry[t - 1];
        cfns = carry[TT] + carry[TT - 1];
      } else {
        int ic[257], iv[128];
        for (int t = 0; t < TT; t++) {
          int mask = -1 << nb[t];
          ic[t + 1] = (int)(bigint[t] >> nb[t]);
          iv[t] = ((int)bigint[t]) & ~mask;
        }
        for (int t = 0; t < TT; t++) {
          int mask = -1 << nb[t];
          if (t) iv[t] += ic[t];
          int sh = iv[t] - (mask >> 1);
          ic[t] = sh >> nb[t];
          iv[t] -= sh & mask;
        }
        for (int t = 0; t < TT; t++) { if (t) iv[t] += ic[t - 1]; val[t] = iv[t]; }
        cfns = ic[TT] + ic[TT - 1];
      }
      for (int t = 0; t < TT; t++) {
        int index = (blk << sc) + row * TT + t;
        int grp = index >> 5, col = index & 31;
        double tc = c->ttp[col << 1];
        if (c->s[grp * 2 + 1] & (1u << col)) tc *= 0.5;
        double ttp = c->ttp[grp * 2 + 64] * tc;
        c->x[index] = (double)val[t] * ttp;
        if (report) c->xint[index] = (int)val[t];
        if (row == 0 && t < 2) c->data[(blk << 1) + t] = (int)val[t];
      }
    }
    if (ferr_max > err) err = ferr_max;
    c->carry[(blk + 1) % nblk] = c->bigcarry ? cfns : (long long)(int)cfns;
  }
  job->err[slot] = err;
}

static void rcb(oracle_ctx *c, int report, int digit, int bit) {
  rcb_job job;
  job.c = c; job.report = report; job.digit = digit; job.bit = bit;
  for (int i = 0; i < ORACLE_MAX_THREADS; i++) job.err[i] = 0;
  par_for(c->n >> c->sc, rcb_range, &job);
  for (int i = 0; i < ORACLE_MAX_THREADS; i++)
    if (job.err[i] > c->err) c->err = job.err[i];
}

/* splice / splicel, CUDALucas.cu:486-534 and :681-721 */
typedef struct { oracle_ctx *c; int report; } splice_job;

static void splice_range(void *arg, int lo, int hi, int slot) {
  oracle_ctx *c = ((splice_job *)arg)->c;
  const int report = ((splice_job *)arg)->report;
  int bw = 1 << c->sc;
  (void)slot;
  for (int blk = lo; blk < hi; blk++) {
    int j = blk * bw;
    int numbits = c->qn;
    double temp = c->ttp1[blk];
    long long t0 = (long long)c->data[2 * blk] + c->carry[blk];
    long long t1 = c->data[2 * blk + 1];
    if (temp < 0.0) { numbits++; temp = -temp; }
    if (!c->bigcarry) t0 = (int)t0;
    {
      long long mask = (long long)(~0ULL << numbits);
      long long sh = t0 - (mask >> 1);
      t0 = t0 - (sh & mask);
      t1 += sh >> numbits;
    }
    c->x[j] = (double)t0 * temp;
    temp *= c->ttpinc[numbits == c->qn];
    c->x[j + 1] = (double)t1 * temp;
    if (report) { c->xint[j] = (int)t0; c->xint[j + 1] = (int)t1; }
  }
}

static void splice(oracle_ctx *c, int report) {
  splice_job job = {c, report};
  par_for(c->n >> c->sc, splice_range, &job);
}

/* lucas_square, CUDALucas.cu:1869-1986 */
float oracle_square(oracle_ctx *c, int report) {
  int q = c->q, n = c->n;
  c->offset = (int)((2LL * c->offset) % q);
  int bit = (c->offset + 1) % q;
  int digit = (int)(((long long)bit * n) / q);
  int sd = (int)(((long long)digit * q + n - 1) / n);
  bit = 1 << (bit - sd);
  fft_exec(&c->plan, (cplx *)c->x);
  square(c);
  fft_exec(&c->plan, (cplx *)c->x);
  rcb(c, report, digit, bit);
  splice(c, report);
  return c->err;
}

/* iters calls of lucas_square; digits are written on the last one. */
float oracle_step(oracle_ctx *c, int iters, int report_last) {
  float e = 0;
  c->err = 0;
  for (int i = 0; i < iters; i++) e = oracle_square(c, report_last && i == iters - 1);
  return e;
}

/* Host threads for the parallel loops (1 = the plain single-threaded run);
 * returns the count in effect. */
int oracle_set_threads(int t) {
  if (t >= 1) g_threads = t < ORACLE_MAX_THREADS ? t : ORACLE_MAX_THREADS;
  return g_threads;
}

void oracle_digits(const oracle_ctx *c, int *out) { memcpy(out, c->xint, sizeof(int) * (size_t)c->n); }
void oracle_weighted(const oracle_ctx *c, double *out) { memcpy(out, c->x, sizeof(double) * (size_t)c->n); }
int oracle_offset(const oracle_ctx *c) { return c->offset; }
void oracle_set_offset(oracle_ctx *c, int o) { c->offset = o; }
int oracle_big_word(const oracle_ctx *c, int j) { return big_word(c, j); }

/* ---------------------------------------------------- residue helpers -- */
/* size(), CUDALucas.cu:1280 -- big-word test from the exact definition */
static int word_is_big(int q, int n, int j) {
  long long b = q % n;
  long long e = (-(long long)j * b) % n;
  if (e < 0) e += n;
  return e < b;
}

/* find_residue, CUDALucas.cu:1491-1534 */
uint64_t oracle_find_residue(const int *x_int, int q, int n, int offset) {
  int j, k = 0, digit, bit, qn = q / n, carry = 0, lo = 1 << qn, hi = lo << 1, tx, temp;
  uint64_t residue = 0;
  digit = (int)(((long long)offset * n) / q);
  bit = offset - (int)(((long long)digit * q + n - 1) / n);
  j = (n + digit - 1) % n;
  while (x_int[j] == 0 && j != digit) { j--; if (j < 0) j += n; }
  if (j == digit && x_int[digit] == 0) return 0;
  else if (x_int[j] < 0) carry = -1;
  for (j = 0; j < 10; j++) {
    tx = x_int[digit] + carry;
    temp = word_is_big(q, n, digit) ? hi : lo;
    if (tx < 0) { tx += temp; carry = -1; } else carry = 0;
    residue += (uint64_t)tx << k;
    k += qn + word_is_big(q, n, digit);
    if (j == 0) { k -= bit; residue >>= bit; }
    if (k >= 64) break;
    digit++;
    if (digit == n) digit = 0;
  }
  return residue;
}

/* standardize_digits, CUDALucas.cu:1465-1489 */
int oracle_standardize_digits(int *x_int, int q, int n) {
  int j, qn = q / n, carry = 0, temp, lo = 1 << qn, hi = lo << 1;
  j = n - 1;
  while (x_int[j] == 0 && j) j--;
  if (j == 0 && x_int[0] == 0) return 1;
  else if (x_int[j] < 0) carry = -1;
  for (j = 0; j < n; j++) {
    x_int[j] += carry;
    temp = word_is_big(q, n, j) ? hi : lo;
    if (x_int[j] < 0) { x_int[j] += temp; carry = -1; } else carry = 0;
  }
  return 0;
}

/* pack_bits, CUDALucas.cu:1594-1614 */
void oracle_pack_bits(const int *x_int, unsigned *packed, int q, int n) {
  unsigned long long t2 = 0;
  int j = 0, k = 0, qn = q / n;
  for (int i = 0; i < n; i++) {
    unsigned long long t1 = (unsigned long long)(long long)x_int[i];
    t2 += t1 << k;
    k += qn + word_is_big(q, n, i);
    if (k >= 32) { packed[j] = (unsigned)t2; t2 >>= 32; k -= 32; j++; }
  }
  packed[j] = (unsigned)t2;
}

/* unpack_bits, CUDALucas.cu:1285-1311 */
void oracle_unpack_bits(int *x_int, const unsigned *packed, int q, int n) {
  unsigned long long t1, t2 = 0;
  int i, j = 0, k = 0, qn = q / n, mask1 = ~(-1 << (qn + 1)), mask2 = mask1 >> 1, mask;
  for (i = 0; i < n; i++) {
    int sz = word_is_big(q, n, i);
    if (k < qn + sz) { t1 = packed[j]; t2 += t1 << k; k += 32; j++; }
    mask = sz ? mask1 : mask2;
    x_int[i] = ((int)t2) & mask;
    t2 >>= (qn + sz);
    k -= (qn + sz);
  }
}

/* balance_digits, CUDALucas.cu:1313-1342 */
void oracle_balance_digits(int *x, int q, int n) {
  int half_low = 1 << (q / n - 1), low = half_low << 1, high = low << 1, upper, adj, carry = 0;
  for (int j = 0; j < n; j++) {
    if (word_is_big(q, n, j)) { upper = low; adj = high; } else { upper = half_low; adj = low; }
    x[j] += carry;
    carry = 0;
    if (x[j] >= upper) { x[j] -= adj; carry = 1; }
  }
  x[0] += carry;
}

/* checkpoint_checksum, CUDALucas.cu:1712-1733 */
unsigned oracle_checkpoint_checksum(const char *string, int chars) {
  unsigned chksum = 0;
  for (int i = 0; i < chars; i++)
    for (int j = 7; j >= 0; j--) {
      if ((chksum >> 31) == (((unsigned)(string[i] >> j)) & 1)) chksum <<= 1;
      else chksum = (chksum << 1) ^ 0x04C11DB7;
    }
  return chksum;
}

/* ch_sum, CUDALucas.cu:1735-1743 */
unsigned oracle_ch_sum(const unsigned *x_packed, int q) {
  int end = (q + 31) / 32;
  unsigned sum = 0;
  for (int j = 0; j < end + 9; j++) sum += x_packed[j];
  return sum;
}
