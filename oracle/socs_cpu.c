/*
 * FP64 CPU restatement of the reference's per-image imaging loop.
 *
 * TEST INFRASTRUCTURE: the oracle and the timed CPU baseline, never the
 * product.  Follows, in plain C with POSIX threads:
 *   - Fft2D (crates/highuvlith-core/src/math/fft2d.rs:96-170): row pass (all
 *     rows, or only the listed non-zero rows), transpose, column pass,
 *     transpose back; forward unnormalised, inverse x 1/N^2;
 *   - Mask::spectrum's raster path (mask.rs:630-635): forward FFT of the
 *     raster times the separable pixel transfer sinc(pi m / N);
 *   - socs_intensity (aerial.rs:1682-1721): kernels split into at most 16
 *     fixed contiguous groups (workspace cap 256 MiB), each group summed
 *     sequentially on its own thread, group images added in index order;
 *   - normalize + apply_flare (aerial.rs:1727-1748).
 * The reference calls rustfft; this file carries its own iterative radix-2
 * complex FFT with a precomputed twiddle table (same transform, different
 * constant factor).
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef struct {
  double re, im;
} cplx;

typedef struct {
  int n, lg;
  cplx* tw; /* exp(-2 pi i t / n), t < n/2 */
  int* rev;
} fft_plan;

static void plan_init(fft_plan* p, int n) {
  p->n = n;
  p->lg = 0;
  while ((1 << p->lg) < n) p->lg++;
  p->tw = (cplx*)malloc(sizeof(cplx) * (n / 2 + 1));
  p->rev = (int*)malloc(sizeof(int) * n);
  for (int t = 0; t < n / 2; ++t) {
    const double a = -2.0 * M_PI * t / n;
    p->tw[t].re = cos(a);
    p->tw[t].im = sin(a);
  }
  for (int i = 0; i < n; ++i) {
    int r = 0;
    for (int b = 0; b < p->lg; ++b)
      if (i & (1 << b)) r |= 1 << (p->lg - 1 - b);
    p->rev[i] = r;
  }
}

static void plan_free(fft_plan* p) {
  free(p->tw);
  free(p->rev);
}

/* In-place radix-2 DIT FFT of one length-n sequence; dir -1 forward, +1 inverse (no scaling). */
static void fft1(const fft_plan* p, cplx* x, int dir) {
  const int n = p->n;
  for (int i = 0; i < n; ++i) {
    const int j = p->rev[i];
    if (j > i) {
      cplx t = x[i];
      x[i] = x[j];
      x[j] = t;
    }
  }
  for (int len = 2; len <= n; len <<= 1) {
    const int half = len >> 1, step = n / len;
    for (int s = 0; s < n; s += len) {
      for (int k = 0; k < half; ++k) {
        cplx w = p->tw[k * step];
        if (dir > 0) w.im = -w.im;
        cplx* a = &x[s + k];
        cplx* b = &x[s + k + half];
        const double tr = b->re * w.re - b->im * w.im;
        const double ti = b->re * w.im + b->im * w.re;
        b->re = a->re - tr;
        b->im = a->im - ti;
        a->re += tr;
        a->im += ti;
      }
    }
  }
}

static void transpose(const cplx* src, cplx* dst, int rows, int cols) {
  const int T = 32;
  for (int ib = 0; ib < rows; ib += T)
    for (int jb = 0; jb < cols; jb += T)
      for (int i = ib; i < ib + T && i < rows; ++i)
        for (int j = jb; j < jb + T && j < cols; ++j) dst[(size_t)j * rows + i] = src[(size_t)i * cols + j];
}

/* 2-D transform of an n x n row-major array; rows == NULL: all rows. */
static void fft2(const fft_plan* p, cplx* data, cplx* tmp, int dir, const int* rows, int nrows) {
  const int n = p->n;
  if (rows) {
    for (int r = 0; r < nrows; ++r) fft1(p, data + (size_t)rows[r] * n, dir);
  } else {
    for (int r = 0; r < n; ++r) fft1(p, data + (size_t)r * n, dir);
  }
  transpose(data, tmp, n, n);
  for (int r = 0; r < n; ++r) fft1(p, tmp + (size_t)r * n, dir);
  transpose(tmp, data, n, n);
}

typedef struct {
  const fft_plan* plan;
  int n, nk, ns, k0, k1;
  const int64_t* support;
  const cplx* values; /* nk x ns */
  const double* eig;  /* raw eigenvalues */
  const cplx* ms;     /* spectrum at the support */
  const int* rows;
  int nrows;
  double* acc; /* n x n */
} group_job;

static void* run_group(void* arg) {
  group_job* g = (group_job*)arg;
  const int n = g->n;
  const size_t nn = (size_t)n * n;
  cplx* buf = (cplx*)malloc(sizeof(cplx) * nn);
  cplx* tmp = (cplx*)malloc(sizeof(cplx) * nn);
  memset(g->acc, 0, sizeof(double) * nn);
  const double inv = 1.0 / (double)nn;
  for (int k = g->k0; k < g->k1; ++k) {
    memset(buf, 0, sizeof(cplx) * nn);
    const cplx* u = g->values + (size_t)k * g->ns;
    for (int t = 0; t < g->ns; ++t) {
      const cplx a = u[t], m = g->ms[t];
      buf[g->support[t]].re = a.re * m.re - a.im * m.im;
      buf[g->support[t]].im = a.re * m.im + a.im * m.re;
    }
    fft2(g->plan, buf, tmp, +1, g->rows, g->nrows);
    const double lam = g->eig[k];
    for (size_t i = 0; i < nn; ++i) {
      const double re = buf[i].re * inv, im = buf[i].im * inv;
      g->acc[i] += lam * (re * re + im * im);
    }
  }
  free(buf);
  free(tmp);
  return NULL;
}

/*
 * One aerial image of a raster (n x n doubles, real transmittance) with a
 * sparse kernel set.  pixel_transfer selects Mask::spectrum semantics.
 * divisor <= 0 keeps the image absolute.  Returns 0 on success.
 */
int socs_cpu_image(int n, const double* raster, int pixel_transfer, int nk, int ns, const int64_t* support,
                   const double* values_ri, const double* eig, double divisor, double flare, int max_threads,
                   double* out) {
  fft_plan plan;
  plan_init(&plan, n);
  const size_t nn = (size_t)n * n;
  cplx* spec = (cplx*)malloc(sizeof(cplx) * nn);
  cplx* tmp = (cplx*)malloc(sizeof(cplx) * nn);
  for (size_t i = 0; i < nn; ++i) {
    spec[i].re = raster[i];
    spec[i].im = 0.0;
  }
  fft2(&plan, spec, tmp, -1, NULL, 0);
  if (pixel_transfer) {
    double* tr = (double*)malloc(sizeof(double) * n);
    for (int k = 0; k < n; ++k) {
      const int m = k < n / 2 ? k : k - n;
      const double u = M_PI * m / n;
      tr[k] = fabs(u) < 1e-6 ? 1.0 - u * u / 6.0 : sin(u) / u;
    }
    for (int i = 0; i < n; ++i)
      for (int j = 0; j < n; ++j) {
        const double f = tr[i] * tr[j];
        spec[(size_t)i * n + j].re *= f;
        spec[(size_t)i * n + j].im *= f;
      }
    free(tr);
  }
  cplx* ms = (cplx*)malloc(sizeof(cplx) * ns);
  for (int t = 0; t < ns; ++t) ms[t] = spec[support[t]];
  /* distinct rows present in the support, in order */
  int* rows = (int*)malloc(sizeof(int) * n);
  int nrows = 0;
  for (int t = 0; t < ns; ++t) {
    const int r = (int)(support[t] / n);
    if (nrows == 0 || rows[nrows - 1] != r) {
      int seen = 0;
      for (int q = 0; q < nrows; ++q)
        if (rows[q] == r) seen = 1;
      if (!seen) rows[nrows++] = r;
    }
  }
  /* fixed groups: at most 16, bounded by a 256 MiB workspace */
  const size_t per_group = nn * (sizeof(double) + sizeof(cplx));
  int max_groups = (int)((256u << 20) / (per_group ? per_group : 1));
  if (max_groups < 1) max_groups = 1;
  if (max_groups > 16) max_groups = 16;
  if (max_threads > 0 && max_groups > max_threads) max_groups = max_threads;
  int groups_req = nk < max_groups ? nk : max_groups;
  if (groups_req < 1) groups_req = 1;
  const int per = (nk + groups_req - 1) / groups_req;
  const int groups = (nk + per - 1) / per;
  group_job* jobs = (group_job*)calloc(groups, sizeof(group_job));
  pthread_t* th = (pthread_t*)calloc(groups, sizeof(pthread_t));
  double* accs = (double*)malloc(sizeof(double) * nn * groups);
  for (int g = 0; g < groups; ++g) {
    jobs[g] = (group_job){&plan, n, nk, ns, g * per, (g + 1) * per < nk ? (g + 1) * per : nk, support,
                          (const cplx*)values_ri, eig, ms, rows, nrows, accs + nn * g};
    pthread_create(&th[g], NULL, run_group, &jobs[g]);
  }
  for (int g = 0; g < groups; ++g) pthread_join(th[g], NULL);
  for (size_t i = 0; i < nn; ++i) {
    double s = accs[i];
    for (int g = 1; g < groups; ++g) s += accs[nn * g + i];
    out[i] = s;
  }
  if (divisor > 0)
    for (size_t i = 0; i < nn; ++i) out[i] /= divisor;
  if (flare > 0) {
    double mean = 0;
    for (size_t i = 0; i < nn; ++i) mean += out[i];
    mean /= (double)nn;
    for (size_t i = 0; i < nn; ++i) out[i] = out[i] * (1.0 - flare) + flare * mean;
  }
  free(accs);
  free(th);
  free(jobs);
  free(rows);
  free(ms);
  free(tmp);
  free(spec);
  plan_free(&plan);
  return 0;
}

/* Batch throughput driver: `threads` workers pull images from a shared
 * counter; each image runs the per-image loop above with one kernel group
 * per worker (the reference engine is Send + Sync and images of independent
 * clips are computed concurrently, imaging_validation.rs:720-750). */
typedef struct {
  int n, count, pixel_transfer, nk, ns;
  const uint8_t* rasters;
  const int64_t* support;
  const double* values_ri;
  const double* eig;
  double divisor, flare;
  float* out;
  int next;
  pthread_mutex_t mu;
} batch_job;

static void* batch_worker(void* arg) {
  batch_job* b = (batch_job*)arg;
  const size_t nn = (size_t)b->n * b->n;
  double* raster = (double*)malloc(sizeof(double) * nn);
  double* img = (double*)malloc(sizeof(double) * nn);
  for (;;) {
    pthread_mutex_lock(&b->mu);
    const int i = b->next++;
    pthread_mutex_unlock(&b->mu);
    if (i >= b->count) break;
    for (size_t p = 0; p < nn; ++p) raster[p] = (double)b->rasters[(size_t)i * nn + p];
    socs_cpu_image(b->n, raster, b->pixel_transfer, b->nk, b->ns, b->support, b->values_ri, b->eig, b->divisor,
                   b->flare, 1, img);
    if (b->out)
      for (size_t p = 0; p < nn; ++p) b->out[(size_t)i * nn + p] = (float)img[p];
  }
  free(raster);
  free(img);
  return NULL;
}

int socs_cpu_batch(int n, int count, const uint8_t* rasters, int pixel_transfer, int nk, int ns,
                   const int64_t* support, const double* values_ri, const double* eig, double divisor,
                   double flare, int threads, float* out) {
  batch_job b = {n, count, pixel_transfer, nk, ns, rasters, support, values_ri, eig, divisor, flare, out, 0};
  pthread_mutex_init(&b.mu, NULL);
  if (threads < 1) threads = 1;
  if (threads > count) threads = count;
  pthread_t* th = (pthread_t*)calloc(threads, sizeof(pthread_t));
  for (int t = 0; t < threads; ++t) pthread_create(&th[t], NULL, batch_worker, &b);
  for (int t = 0; t < threads; ++t) pthread_join(th[t], NULL);
  free(th);
  pthread_mutex_destroy(&b.mu);
  return 0;
}
