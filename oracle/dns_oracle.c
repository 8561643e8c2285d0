/*
 * dns_oracle.c -- CPU oracle for the finite-volume step (TEST INFRASTRUCTURE).
 *
 * This file restates, in plain C with OpenMP, the single-rank path of the
 * DistributedNavierStokes FV solver.  It is used only as the checker of the
 * CUDA library (tests/, __graft_entry__.smoke) and as the timed CPU baseline
 * of bench.py.  Each function cites the reference file:line it follows and
 * keeps the reference's operation order (no FMA contraction: built with
 * -ffp-contract=off), so that it reproduces what the Julia code computes on
 * the same inputs up to the rounding of the FFT library.
 *
 * Parity status: the reference is Julia and no Julia toolchain exists where
 * this project is built or run, and the reference ships no golden vectors.
 * The oracle is pinned by re-running the reference's own known-answer and
 * identity tests (test/serialtests.jl, test/mpitests.jl) against it, and its
 * FFTs against numpy.fft (see tests/test_oracle.py).
 */
#include "dns_oracle.h"

#include <complex.h>
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#undef I /* the loops below use I, J, K as the reference's cell indices */
#define IU _Complex_I
typedef double _Complex cplx;

/* ------------------------------------------------------------------ FFT -- */
/* Recursive mixed-radix decimation-in-time Cooley-Tukey, any length.  The
 * reference calls FFTW (CPU) / cuFFT (GPU) through AbstractFFTs
 * (src/poisson.jl:80-83,115-116); this is an independent restatement of the
 * DFT with those conventions (forward exp(-2 pi i jk/n), inverse scaled 1/n). */

typedef struct {
  int n;
  int nf;
  int f[64];
  cplx *w; /* w[t] = exp(-2 pi i t / n) */
} fftplan;

static double cospi_ld(long double x) { return (double)cosl(x * 3.141592653589793238462643383279502884L); }

/* exp(-2 pi i t/n) with the angle reduced to the first octant, evaluated in
 * long double and rounded once. */
static cplx unit_root(long t, long n) {
  t %= n;
  if (t < 0) t += n;
  /* angle = 2 pi t / n; use symmetry: work with 8t vs n octants */
  long double x = (long double)t / (long double)n; /* in [0,1) turns */
  long double c = cosl(2.0L * 3.141592653589793238462643383279502884L * x);
  long double s = sinl(2.0L * 3.141592653589793238462643383279502884L * x);
  /* exact values at quarter turns */
  if (4 * t == n) { c = 0; s = 1; }
  else if (2 * t == n) { c = -1; s = 0; }
  else if (4 * t == 3 * n) { c = 0; s = -1; }
  else if (t == 0) { c = 1; s = 0; }
  return (double)c - IU * (double)s;
}

static void plan_init(fftplan *p, int n) {
  p->n = n;
  p->nf = 0;
  int m = n;
  while (m % 4 == 0) { p->f[p->nf++] = 4; m /= 4; }
  while (m % 2 == 0) { p->f[p->nf++] = 2; m /= 2; }
  for (int q = 3; q <= m; q += 2)
    while (m % q == 0) { p->f[p->nf++] = q; m /= q; }
  p->w = (cplx *)malloc(sizeof(cplx) * (size_t)(n > 0 ? n : 1));
  for (int t = 0; t < n; t++) p->w[t] = unit_root(t, n);
}

static void plan_free(fftplan *p) { free(p->w); p->w = NULL; }

/* DFT of in[0], in[is], ..., in[(n-1)is] into out[0..n-1] (contiguous).
 * Twiddle W_n^t = p->w[t * tws]; n * tws == p->n. */
static void fft_rec(const fftplan *p, int lev, const cplx *in, long is,
                    cplx *out, int n, int tws, int inv) {
  if (n == 1) { out[0] = in[0]; return; }
  int r = p->f[lev];
  int m = n / r;
  for (int q = 0; q < r; q++)
    fft_rec(p, lev + 1, in + q * is, is * r, out + (long)q * m, m, tws * r, inv);
  cplx tmp[r];
  int N0 = p->n;
  for (int k = 0; k < m; k++) {
    for (int q = 0; q < r; q++) {
      long t = ((long)q * k % n) * tws;
      cplx w = p->w[t % N0];
      if (inv) w = conj(w);
      tmp[q] = out[(long)q * m + k] * w;
    }
    for (int s2 = 0; s2 < r; s2++) {
      cplx acc = 0;
      for (int q = 0; q < r; q++) {
        long t = (long)((q * s2) % r) * (N0 / r);
        cplx w = p->w[t];
        if (inv) w = conj(w);
        acc += tmp[q] * w;
      }
      out[k + (long)s2 * m] = acc;
    }
  }
}

/* one strided complex line, in place, via a scratch line */
static void fft_line(const fftplan *p, cplx *x, long stride, int inv, cplx *scr,
                     cplx *scr2) {
  int n = p->n;
  for (int i = 0; i < n; i++) scr[i] = x[i * stride];
  fft_rec(p, 0, scr, 1, scr2, n, 1, inv);
  if (inv) {
    double s = 1.0 / n;
    for (int i = 0; i < n; i++) x[i * stride] = scr2[i] * s;
  } else {
    for (int i = 0; i < n; i++) x[i * stride] = scr2[i];
  }
}

/* real forward transform of one contiguous line of even length n via the
 * half-length complex transform; out has n/2+1 entries, stride ostride. */
static void rfft_line(const fftplan *half, const cplx *wn, const double *x,
                      int n, cplx *out, long ostride, cplx *scr, cplx *scr2) {
  int m = n / 2;
  for (int j = 0; j < m; j++) scr[j] = x[2 * j] + IU * x[2 * j + 1];
  fft_rec(half, 0, scr, 1, scr2, m, 1, 0);
  for (int k = 0; k <= m; k++) {
    cplx zk = scr2[k % m];
    cplx zc = conj(scr2[(m - k) % m]);
    cplx e = 0.5 * (zk + zc);
    cplx o = -0.5 * IU * (zk - zc);
    out[k * ostride] = e + wn[k] * o;
  }
}

/* inverse of rfft_line, normalised 1/n; imaginary parts of the k = 0 and
 * k = n/2 inputs are ignored (FFTW c2r semantics). */
static void irfft_line(const fftplan *half, const cplx *wn, const cplx *in,
                       long istride, int n, double *x, cplx *scr, cplx *scr2) {
  int m = n / 2;
  for (int k = 0; k < m; k++) {
    cplx a = in[k * istride];
    cplx b = conj(in[(m - k) * istride]);
    if (k == 0) { a = creal(a); b = creal(in[m * istride]); }
    cplx e = 0.5 * (a + b);
    cplx o = 0.5 * (a - b) * conj(wn[k]);
    scr[k] = e + IU * o;
  }
  fft_rec(half, 0, scr, 1, scr2, m, 1, 1);
  double s = 1.0 / m;
  for (int j = 0; j < m; j++) {
    x[2 * j] = creal(scr2[j]) * s;
    x[2 * j + 1] = cimag(scr2[j]) * s;
  }
}

void dnso_cfft(int n, int howmany, int inverse, cplx *data) {
  fftplan p;
  plan_init(&p, n);
#pragma omp parallel
  {
    cplx *s1 = (cplx *)malloc(sizeof(cplx) * n), *s2 = (cplx *)malloc(sizeof(cplx) * n);
#pragma omp for
    for (int h = 0; h < howmany; h++) fft_line(&p, data + (long)h * n, 1, inverse, s1, s2);
    free(s1); free(s2);
  }
  plan_free(&p);
}

static cplx *make_wn(int n) {
  cplx *w = (cplx *)malloc(sizeof(cplx) * (n / 2 + 1));
  for (int k = 0; k <= n / 2; k++) w[k] = unit_root(k, n);
  return w;
}

void dnso_rfft(int n, int howmany, const double *in, cplx *out) {
  fftplan p;
  plan_init(&p, n / 2);
  cplx *wn = make_wn(n);
#pragma omp parallel
  {
    cplx *s1 = (cplx *)malloc(sizeof(cplx) * n), *s2 = (cplx *)malloc(sizeof(cplx) * n);
#pragma omp for
    for (int h = 0; h < howmany; h++)
      rfft_line(&p, wn, in + (long)h * n, n, out + (long)h * (n / 2 + 1), 1, s1, s2);
    free(s1); free(s2);
  }
  free(wn);
  plan_free(&p);
}

void dnso_irfft(int n, int howmany, const cplx *in, double *out) {
  fftplan p;
  plan_init(&p, n / 2);
  cplx *wn = make_wn(n);
#pragma omp parallel
  {
    cplx *s1 = (cplx *)malloc(sizeof(cplx) * n), *s2 = (cplx *)malloc(sizeof(cplx) * n);
#pragma omp for
    for (int h = 0; h < howmany; h++)
      irfft_line(&p, wn, in + (long)h * (n / 2 + 1), 1, n, out + (long)h * n, s1, s2);
    free(s1); free(s2);
  }
  free(wn);
  plan_free(&p);
}

/* ---------------------------------------------------------------- setup -- */

struct dnso {
  int nx, ny, nz, wall, imexy;
  int NX, NY, NZ; /* ghosted extents */
  double dx, dz, dymin, visc, f[3], epsy;
  double *dy, *dyu;           /* ny+2 */
  double *lam1, *lam2, *lam3; /* nkx, ny, nz */
  double *ay, *by, *cy;       /* ny (wall) */
  double *at, *bt, *ct, *an, *bn, *cn;
  int nkx;
  double *r;   /* nx*ny*nz */
  cplx *ah;    /* nkx*ny*nz, kx fastest (the reference's âx/âz/ây) */
  double *work;
  double *yb1, *yb2, *yb3; /* imex y-line buffers, nx*ny*nz */
  fftplan px_half, pz, py;
  cplx *wnx;
};

#define IDX(s, I, J, K) ((long)(I) + (long)(s)->NX * ((long)(J) + (long)(s)->NY * (long)(K)))

void dnso_set_threads(int n) {
#ifdef _OPENMP
  omp_set_num_threads(n);
#else
  (void)n;
#endif
}

/* modλ (src/poisson.jl:12): 2 (cospi(2(k-1)/n) - 1) / Δ^2 for k = 1.. */
static double modlam(int k1, int n, double d) {
  double x = (double)(2 * (k1 - 1)) / (double)n; /* Julia: 2 * (k - 1) / n */
  double c = cospi_ld((long double)x);
  if (k1 - 1 == 0) c = 1.0;
  else if (4 * (k1 - 1) == n || 4 * (k1 - 1) == 3 * n) c = 0.0;
  else if (2 * (k1 - 1) == n) c = -1.0;
  return 2 * (c - 1) / (d * d);
}

dnso_t *dnso_create(int nx, int ny, int nz, int wall, int implicit, double Lx,
                    double Lz, const double *yf, double visc, double fx,
                    double fy, double fz) {
  if (nx < 2 || ny < 2 || nz < 1 || (nx % 2) != 0) return NULL;
  if (implicit && !wall) return NULL; /* src/ydiffusion.jl:56 */
  dnso_t *s = (dnso_t *)calloc(1, sizeof(dnso_t));
  s->nx = nx; s->ny = ny; s->nz = nz; s->wall = wall; s->imexy = implicit;
  s->NX = nx + 2; s->NY = ny + 2; s->NZ = nz + 2;
  s->visc = visc; s->f[0] = fx; s->f[1] = fy; s->f[2] = fz;
  s->epsy = implicit ? 0.0 : 1.0; /* src/setup.jl:108 */
  /* griddata (src/setup.jl:148-193), w = 1 */
  s->dx = Lx / nx;
  s->dz = Lz / nz;
  int w = 1;
  double *yfe = (double *)calloc(ny + 2 * w + 1, sizeof(double));
  for (int j = 0; j <= ny; j++) yfe[w + j] = yf[j];
  for (int m = 1; m <= w; m++) {
    if (!wall) {
      yfe[w - m] = yf[0] - (yf[ny] - yf[ny - m]);
      yfe[w + ny + m] = yf[ny] + (yf[m] - yf[0]);
    } else {
      yfe[w - m] = 2 * yf[0] - yf[m];
      yfe[w + ny + m] = 2 * yf[ny] - yf[ny - m];
    }
  }
  int ne = ny + 2 * w; /* cells 1-w .. ny+w */
  s->dy = (double *)malloc(sizeof(double) * ne);
  s->dyu = (double *)malloc(sizeof(double) * ne);
  double *yce = (double *)malloc(sizeof(double) * ne);
  for (int J = 0; J < ne; J++) {
    s->dy[J] = yfe[J + 1] - yfe[J];
    yce[J] = (yfe[J] + yfe[J + 1]) / 2;
  }
  for (int J = 0; J < ne - 1; J++) s->dyu[J] = yce[J + 1] - yce[J];
  s->dyu[ne - 1] = s->dy[ne - 1];
  s->dymin = s->dy[w];
  for (int J = w; J < w + ny; J++)
    if (s->dy[J] < s->dymin) s->dymin = s->dy[J];
  free(yce);
  free(yfe);

  /* plan_poisson (src/poisson.jl:56-120) */
  s->nkx = nx / 2 + 1;
  s->lam1 = (double *)malloc(sizeof(double) * s->nkx);
  s->lam3 = (double *)malloc(sizeof(double) * nz);
  s->lam2 = (double *)malloc(sizeof(double) * ny);
  for (int k = 1; k <= s->nkx; k++) s->lam1[k - 1] = modlam(k, nx, s->dx);
  for (int k = 1; k <= nz; k++) s->lam3[k - 1] = modlam(k, nz, s->dz);
  for (int k = 1; k <= ny; k++) s->lam2[k - 1] = modlam(k, ny, s->dy[w]);
  s->ay = (double *)calloc(ny, sizeof(double));
  s->by = (double *)calloc(ny, sizeof(double));
  s->cy = (double *)calloc(ny, sizeof(double));
  if (wall) {
    for (int j = 1; j <= ny; j++) {
      double a = j == 1 ? 0.0 : 1 / (s->dy[j - 1 + w] * s->dyu[j - 2 + w]);
      double c = j == ny ? 0.0 : 1 / (s->dy[j - 1 + w] * s->dyu[j - 1 + w]);
      s->ay[j - 1] = a; s->cy[j - 1] = c; s->by[j - 1] = -(a + c);
    }
  }
  /* ydiffusion_coefficients (src/ydiffusion.jl:31-51); Julia Δye[j+w] is
   * our dy[j-1+w] (1-based vs 0-based) */
  s->at = (double *)calloc(ny, sizeof(double));
  s->bt = (double *)calloc(ny, sizeof(double));
  s->ct = (double *)calloc(ny, sizeof(double));
  s->an = (double *)calloc(ny, sizeof(double));
  s->bn = (double *)calloc(ny, sizeof(double));
  s->cn = (double *)calloc(ny, sizeof(double));
  for (int j = 1; j <= ny; j++) {
    double a = 1 / (s->dy[j - 1 + w] * s->dyu[j - 2 + w]);
    double c = 1 / (s->dy[j - 1 + w] * s->dyu[j - 1 + w]);
    s->at[j - 1] = j == 1 ? 0.0 : a;
    s->ct[j - 1] = j == ny ? 0.0 : c;
    s->bt[j - 1] = j == 1 ? -(c + 2 * a) : j == ny ? -(a + 2 * c) : -(a + c);
  }
  for (int j = 1; j <= ny - 1; j++) {
    double a = 1 / (s->dyu[j - 1 + w] * s->dy[j - 1 + w]);
    double c = 1 / (s->dyu[j - 1 + w] * s->dy[j + w]);
    s->an[j - 1] = j == 1 ? 0.0 : a;
    s->cn[j - 1] = j == ny - 1 ? 0.0 : c;
    s->bn[j - 1] = -(a + c);
  }
  long ncell = (long)nx * ny * nz;
  s->r = (double *)calloc(ncell, sizeof(double));
  s->ah = (cplx *)calloc((long)s->nkx * ny * nz, sizeof(cplx));
  s->work = (double *)calloc((long)s->nkx * ny * nz, sizeof(double));
  if (implicit) {
    s->yb1 = (double *)calloc(ncell, sizeof(double));
    s->yb2 = (double *)calloc(ncell, sizeof(double));
    s->yb3 = (double *)calloc(ncell, sizeof(double));
  }
  plan_init(&s->px_half, nx / 2);
  plan_init(&s->pz, nz);
  plan_init(&s->py, ny);
  s->wnx = make_wn(nx);
  return s;
}

void dnso_destroy(dnso_t *s) {
  if (!s) return;
  free(s->dy); free(s->dyu); free(s->lam1); free(s->lam2); free(s->lam3);
  free(s->ay); free(s->by); free(s->cy);
  free(s->at); free(s->bt); free(s->ct); free(s->an); free(s->bn); free(s->cn);
  free(s->r); free(s->ah); free(s->work);
  free(s->yb1); free(s->yb2); free(s->yb3);
  plan_free(&s->px_half); plan_free(&s->pz); plan_free(&s->py);
  free(s->wnx);
  free(s);
}

void dnso_grid(const dnso_t *s, double *dx, double *dz, double *dy, double *dyu,
               double *dymin) {
  *dx = s->dx; *dz = s->dz; *dymin = s->dymin;
  memcpy(dy, s->dy, sizeof(double) * (s->ny + 2));
  memcpy(dyu, s->dyu, sizeof(double) * (s->ny + 2));
}

void dnso_poisson_coeffs(const dnso_t *s, double *lam1, double *lam2,
                         double *lam3, double *ay, double *by, double *cy) {
  memcpy(lam1, s->lam1, sizeof(double) * s->nkx);
  memcpy(lam2, s->lam2, sizeof(double) * s->ny);
  memcpy(lam3, s->lam3, sizeof(double) * s->nz);
  memcpy(ay, s->ay, sizeof(double) * s->ny);
  memcpy(by, s->by, sizeof(double) * s->ny);
  memcpy(cy, s->cy, sizeof(double) * s->ny);
}

void dnso_ydiff_coeffs(const dnso_t *s, double *at, double *bt, double *ct,
                       double *an, double *bn, double *cn) {
  size_t b = sizeof(double) * s->ny;
  memcpy(at, s->at, b); memcpy(bt, s->bt, b); memcpy(ct, s->ct, b);
  memcpy(an, s->an, b); memcpy(bn, s->bn, b); memcpy(cn, s->cn, b);
}

/* ------------------------------------------------------------------ halo -- */

/* exchange_halo! on a single rank (src/halo.jl:81-126): dimensions in the
 * order x, y, z; periodic dims copy full-extent slabs (so edges and corners
 * follow), the wall dim uses fill_wall! (src/halo.jl:26-45). */
void dnso_fill_halo(const dnso_t *s, double *phi, int stag) {
  int NX = s->NX, NY = s->NY, NZ = s->NZ, nx = s->nx, ny = s->ny, nz = s->nz;
  /* x: periodic */
#pragma omp parallel for
  for (int K = 0; K < NZ; K++)
    for (int J = 0; J < NY; J++) {
      phi[IDX(s, 0, J, K)] = phi[IDX(s, nx, J, K)];
      phi[IDX(s, nx + 1, J, K)] = phi[IDX(s, 1, J, K)];
    }
  /* y */
  if (!s->wall) {
#pragma omp parallel for
    for (int K = 0; K < NZ; K++)
      for (int I = 0; I < NX; I++) {
        phi[IDX(s, I, 0, K)] = phi[IDX(s, I, ny, K)];
        phi[IDX(s, I, ny + 1, K)] = phi[IDX(s, I, 1, K)];
      }
  } else if (stag == 1) {
    /* wall-normal: wall faces (J = 0 and J = ny) zero, ghost ny+1
     * antisymmetric about the top wall face */
#pragma omp parallel for
    for (int K = 0; K < NZ; K++)
      for (int I = 0; I < NX; I++) {
        phi[IDX(s, I, 0, K)] = 0.0;
        phi[IDX(s, I, ny, K)] = 0.0;
        phi[IDX(s, I, ny + 1, K)] = -1 * phi[IDX(s, I, ny - 1, K)];
      }
  } else {
    double sg = stag == 3 ? 1.0 : -1.0;
#pragma omp parallel for
    for (int K = 0; K < NZ; K++)
      for (int I = 0; I < NX; I++) {
        phi[IDX(s, I, 0, K)] = sg * phi[IDX(s, I, 1, K)];
        phi[IDX(s, I, ny + 1, K)] = sg * phi[IDX(s, I, ny, K)];
      }
  }
  /* z: periodic */
#pragma omp parallel for
  for (int J = 0; J < NY; J++)
    for (int I = 0; I < NX; I++) {
      phi[IDX(s, I, J, 0)] = phi[IDX(s, I, J, nz)];
      phi[IDX(s, I, J, nz + 1)] = phi[IDX(s, I, J, 1)];
    }
}

static void fill_halo3(const dnso_t *s, double *ux, double *uy, double *uz) {
  dnso_fill_halo(s, ux, 0);
  dnso_fill_halo(s, uy, 1);
  dnso_fill_halo(s, uz, 2);
}

/* ------------------------------------------------------------- operators -- */

/* divergence_kernel! (src/operators.jl:10-26) */
void dnso_divergence(const dnso_t *s, const double *ux, const double *uy,
                     const double *uz, double *r) {
  int nx = s->nx, ny = s->ny, nz = s->nz;
#pragma omp parallel for
  for (int k = 1; k <= nz; k++)
    for (int j = 1; j <= ny; j++)
      for (int i = 1; i <= nx; i++) {
        long c = IDX(s, i, j, k);
        r[(i - 1) + (long)nx * ((j - 1) + (long)ny * (k - 1))] =
            (ux[c] - ux[IDX(s, i - 1, j, k)]) / s->dx +
            (uy[c] - uy[IDX(s, i, j - 1, k)]) / s->dy[j] +
            (uz[c] - uz[IDX(s, i, j, k - 1)]) / s->dz;
      }
}

/* momentum_kernel! (src/operators.jl:44-145); launch range = ranges.p,
 * u.y updated only for J <= jymax (ny-1 with walls, ny periodic) */
void dnso_momentum(const dnso_t *s, double *qx, double *qy, double *qz,
                   const double *ux, const double *uy, const double *uz,
                   double A, double dt) {
  int nx = s->nx, ny = s->ny, nz = s->nz;
  int jymax = s->wall ? ny - 1 : ny;
  double dx = s->dx, dz = s->dz, nu = s->visc, ey = s->epsy;
  const double *Dy = s->dy, *Dyu = s->dyu;
#pragma omp parallel for
  for (int K = 1; K <= nz; K++)
    for (int J = 1; J <= ny; J++)
      for (int I = 1; I <= nx; I++) {
#define UX(a, b, c) ux[IDX(s, a, b, c)]
#define UY(a, b, c) uy[IDX(s, a, b, c)]
#define UZ(a, b, c) uz[IDX(s, a, b, c)]
        long id = IDX(s, I, J, K);
        /* x momentum */
        double uce = (UX(I, J, K) + UX(I + 1, J, K)) / 2;
        double ucw = (UX(I - 1, J, K) + UX(I, J, K)) / 2;
        double vn = (UY(I, J, K) + UY(I + 1, J, K)) / 2;
        double un = (UX(I, J, K) + UX(I, J + 1, K)) / 2;
        double vs = (UY(I, J - 1, K) + UY(I + 1, J - 1, K)) / 2;
        double us = (UX(I, J - 1, K) + UX(I, J, K)) / 2;
        double wt = (UZ(I, J, K) + UZ(I + 1, J, K)) / 2;
        double ut = (UX(I, J, K) + UX(I, J, K + 1)) / 2;
        double wb = (UZ(I, J, K - 1) + UZ(I + 1, J, K - 1)) / 2;
        double ub = (UX(I, J, K - 1) + UX(I, J, K)) / 2;
        double conv = (uce * uce - ucw * ucw) / dx + (vn * un - vs * us) / Dy[J] +
                      (wt * ut - wb * ub) / dz;
        double diff =
            (UX(I + 1, J, K) - 2 * UX(I, J, K) + UX(I - 1, J, K)) / (dx * dx) +
            ey * ((UX(I, J + 1, K) - UX(I, J, K)) / Dyu[J] -
                  (UX(I, J, K) - UX(I, J - 1, K)) / Dyu[J - 1]) / Dy[J] +
            (UX(I, J, K + 1) - 2 * UX(I, J, K) + UX(I, J, K - 1)) / (dz * dz);
        qx[id] = A * qx[id] + dt * (-conv + nu * diff + s->f[0]);

        /* y momentum */
        double ue = (UX(I, J, K) * Dy[J] + UX(I, J + 1, K) * Dy[J + 1]) / (2 * Dyu[J]);
        double ve = (UY(I, J, K) + UY(I + 1, J, K)) / 2;
        double uw = (UX(I - 1, J, K) * Dy[J] + UX(I - 1, J + 1, K) * Dy[J + 1]) / (2 * Dyu[J]);
        double vw = (UY(I - 1, J, K) + UY(I, J, K)) / 2;
        double vcn = (UY(I, J, K) + UY(I, J + 1, K)) / 2;
        double vcs = (UY(I, J - 1, K) + UY(I, J, K)) / 2;
        double wtv = (UZ(I, J, K) * Dy[J] + UZ(I, J + 1, K) * Dy[J + 1]) / (2 * Dyu[J]);
        double vt = (UY(I, J, K) + UY(I, J, K + 1)) / 2;
        double wbv = (UZ(I, J, K - 1) * Dy[J] + UZ(I, J + 1, K - 1) * Dy[J + 1]) / (2 * Dyu[J]);
        double vb = (UY(I, J, K - 1) + UY(I, J, K)) / 2;
        conv = (ue * ve - uw * vw) / dx + (vcn * vcn - vcs * vcs) / Dyu[J] +
               (wtv * vt - wbv * vb) / dz;
        diff = (UY(I + 1, J, K) - 2 * UY(I, J, K) + UY(I - 1, J, K)) / (dx * dx) +
               ey * ((UY(I, J + 1, K) - UY(I, J, K)) / Dy[J + 1] -
                     (UY(I, J, K) - UY(I, J - 1, K)) / Dy[J]) / Dyu[J] +
               (UY(I, J, K + 1) - 2 * UY(I, J, K) + UY(I, J, K - 1)) / (dz * dz);
        if (J <= jymax) qy[id] = A * qy[id] + dt * (-conv + nu * diff + s->f[1]);

        /* z momentum */
        ue = (UX(I, J, K) + UX(I, J, K + 1)) / 2;
        double we = (UZ(I, J, K) + UZ(I + 1, J, K)) / 2;
        uw = (UX(I - 1, J, K) + UX(I - 1, J, K + 1)) / 2;
        double ww = (UZ(I - 1, J, K) + UZ(I, J, K)) / 2;
        double vnw = (UY(I, J, K) + UY(I, J, K + 1)) / 2;
        double wn = (UZ(I, J, K) + UZ(I, J + 1, K)) / 2;
        double vsw = (UY(I, J - 1, K) + UY(I, J - 1, K + 1)) / 2;
        double ws = (UZ(I, J - 1, K) + UZ(I, J, K)) / 2;
        double wct = (UZ(I, J, K) + UZ(I, J, K + 1)) / 2;
        double wcb = (UZ(I, J, K - 1) + UZ(I, J, K)) / 2;
        conv = (ue * we - uw * ww) / dx + (vnw * wn - vsw * ws) / Dy[J] +
               (wct * wct - wcb * wcb) / dz;
        diff = (UZ(I + 1, J, K) - 2 * UZ(I, J, K) + UZ(I - 1, J, K)) / (dx * dx) +
               ey * ((UZ(I, J + 1, K) - UZ(I, J, K)) / Dyu[J] -
                     (UZ(I, J, K) - UZ(I, J - 1, K)) / Dyu[J - 1]) / Dy[J] +
               (UZ(I, J, K + 1) - 2 * UZ(I, J, K) + UZ(I, J, K - 1)) / (dz * dz);
        qz[id] = A * qz[id] + dt * (-conv + nu * diff + s->f[2]);
#undef UX
#undef UY
#undef UZ
      }
}

/* active-DOF upper bound in y for component c (src/setup.jl:132-138) */
static int jhi(const dnso_t *s, int c) { return (c == 1 && s->wall) ? s->ny - 1 : s->ny; }

/* pgrad{x,y,z}_kernel! (src/operators.jl:180-196) on ranges[c] */
void dnso_pressuregrad(const dnso_t *s, double *phi, const double *p, int c,
                       double sc) {
  int nx = s->nx, nz = s->nz, jh = jhi(s, c);
#pragma omp parallel for
  for (int K = 1; K <= nz; K++)
    for (int J = 1; J <= jh; J++)
      for (int I = 1; I <= nx; I++) {
        long id = IDX(s, I, J, K);
        if (c == 0) phi[id] -= sc * (p[IDX(s, I + 1, J, K)] - p[id]) / s->dx;
        else if (c == 1) phi[id] -= sc * (p[IDX(s, I, J + 1, K)] - p[id]) / s->dyu[J];
        else phi[id] -= sc * (p[IDX(s, I, J, K + 1)] - p[id]) / s->dz;
      }
}

/* --------------------------------------------------------------- poisson -- */

/* thomas_kernel! (src/poisson.jl:14-41) on one (kx, kz) line; x stride nkx */
static void thomas_line(const dnso_t *s, cplx *x, double *cp, long st, double lam) {
  int ny = s->ny;
  const double *ay = s->ay, *by = s->by, *cy = s->cy;
  double beta = lam == 0 ? 1.0 : by[0] + lam;
  cp[0] = (lam == 0 ? 0.0 : cy[0]) / beta;
  x[0] = (lam == 0 ? 0.0 : x[0]) / beta;
  for (int j = 1; j < ny; j++) {
    beta = (by[j] + lam) - ay[j] * cp[(j - 1) * st];
    cp[j * st] = cy[j] / beta;
    x[j * st] = (x[j * st] - ay[j] * x[(j - 1) * st]) / beta;
  }
  for (int j = ny - 2; j >= 0; j--) x[j * st] -= cp[j * st] * x[(j + 1) * st];
}

/* poisson! (src/poisson.jl:147-161): rfft x -> fft z -> solve y -> ifft z ->
 * irfft x.  On one rank every transpose! is an identity copy
 * (src/transpose.jl:96-102), so all stages address one kx-fastest buffer. */
void dnso_poisson(dnso_t *s, const double *rin, double *p) {
  int nx = s->nx, ny = s->ny, nz = s->nz, nkx = s->nkx;
  cplx *ah = s->ah;
  long sj = nkx, sk = (long)nkx * ny;
#pragma omp parallel
  {
    int nmax = nx > ny ? nx : ny;
    if (nz > nmax) nmax = nz;
    cplx *s1 = (cplx *)malloc(sizeof(cplx) * (nmax + 2));
    cplx *s2 = (cplx *)malloc(sizeof(cplx) * (nmax + 2));
    /* rfft along x */
#pragma omp for collapse(2)
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        rfft_line(&s->px_half, s->wnx, rin + (long)nx * (j + (long)ny * k), nx,
                  ah + j * sj + k * sk, 1, s1, s2);
    /* fft along z */
#pragma omp for collapse(2)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nkx; i++) fft_line(&s->pz, ah + i + j * sj, sk, 0, s1, s2);
    /* solve_y! (src/poisson.jl:122-140) */
    if (s->wall) {
#pragma omp for collapse(2)
      for (int k = 0; k < nz; k++)
        for (int i = 0; i < nkx; i++)
          thomas_line(s, ah + i + k * sk, s->work + i + k * sk, sj,
                      s->lam1[i] + s->lam3[k]);
    } else {
#pragma omp for collapse(2)
      for (int k = 0; k < nz; k++)
        for (int i = 0; i < nkx; i++) fft_line(&s->py, ah + i + k * sk, sj, 0, s1, s2);
      /* modedivide_kernel! (src/poisson.jl:43-49) */
#pragma omp for collapse(2)
      for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
          for (int i = 0; i < nkx; i++) {
            double lam = s->lam1[i] + s->lam2[j] + s->lam3[k];
            cplx *x = ah + i + j * sj + k * sk;
            *x = lam == 0 ? 0.0 : *x / lam;
          }
#pragma omp for collapse(2)
      for (int k = 0; k < nz; k++)
        for (int i = 0; i < nkx; i++) fft_line(&s->py, ah + i + k * sk, sj, 1, s1, s2);
    }
    /* ifft along z */
#pragma omp for collapse(2)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nkx; i++) fft_line(&s->pz, ah + i + j * sj, sk, 1, s1, s2);
    /* irfft along x, copybox into the interior of p */
    double *line = (double *)malloc(sizeof(double) * nx);
#pragma omp for collapse(2)
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++) {
        irfft_line(&s->px_half, s->wnx, ah + j * sj + k * sk, 1, nx, line, s1, s2);
        for (int i = 0; i < nx; i++) p[IDX(s, i + 1, j + 1, k + 1)] = line[i];
      }
    free(line);
    free(s1);
    free(s2);
  }
}

/* project! (src/timestep.jl:25-31) */
void dnso_project(dnso_t *s, double *ux, double *uy, double *uz, double *psi) {
  dnso_divergence(s, ux, uy, uz, s->r);
  dnso_poisson(s, s->r, psi);
  dnso_fill_halo(s, psi, 3);
  dnso_pressuregrad(s, ux, psi, 0, 1.0);
  dnso_pressuregrad(s, uy, psi, 1, 1.0);
  dnso_pressuregrad(s, uz, psi, 2, 1.0);
  fill_halo3(s, ux, uy, uz);
}

/* ------------------------------------------------------------ ydiffusion -- */

/* interior copies (copybox!, src/pack.jl:68-78) */
static void copy_out(const dnso_t *s, const double *phi, double *buf) {
  int nx = s->nx, ny = s->ny, nz = s->nz;
#pragma omp parallel for
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
        buf[i + (long)nx * (j + (long)ny * k)] = phi[IDX(s, i + 1, j + 1, k + 1)];
}
static void copy_in(const dnso_t *s, double *phi, const double *buf) {
  int nx = s->nx, ny = s->ny, nz = s->nz;
#pragma omp parallel for
  for (int k = 0; k < nz; k++)
    for (int j = 0; j < ny; j++)
      for (int i = 0; i < nx; i++)
        phi[IDX(s, i + 1, j + 1, k + 1)] = buf[i + (long)nx * (j + (long)ny * k)];
}

/* imex_update! (src/ydiffusion.jl:119-154) with imexrhs_kernel! (:71-91) and
 * imexsolve_kernel! (:94-109) */
void dnso_imex_update(dnso_t *s, double *ux, double *uy, double *uz,
                      const double *qx, const double *qy, const double *qz,
                      const double *p, double B, double alpha, double dt) {
  int nx = s->nx, ny = s->ny, nz = s->nz;
  double th = alpha * dt * s->visc / 2;
  double *u[3] = {ux, uy, uz};
  const double *q[3] = {qx, qy, qz};
  for (int c = 0; c < 3; c++) {
    const double *a = c == 1 ? s->an : s->at, *b = c == 1 ? s->bn : s->bt,
                 *cc = c == 1 ? s->cn : s->ct;
    copy_out(s, u[c], s->yb1); /* uⁿ lines */
    int jh = jhi(s, c);
#pragma omp parallel for
    for (int K = 1; K <= nz; K++)
      for (int J = 1; J <= jh; J++)
        for (int I = 1; I <= nx; I++) {
          long id = IDX(s, I, J, K);
          u[c][id] = u[c][id] + B * q[c][id];
        }
    dnso_pressuregrad(s, u[c], p, c, alpha * dt);
    copy_out(s, u[c], s->yb2); /* v lines */
    double *rhs = s->yb3, *vt = s->yb2, *ut = s->yb1, *cp = s->yb1;
#pragma omp parallel for collapse(2)
    for (int k = 0; k < nz; k++)
      for (int i = 0; i < nx; i++) {
        long o = i + (long)nx * (long)ny * k, st = nx;
        rhs[o] = vt[o] + th * (b[0] * ut[o] + cc[0] * ut[o + st]);
        for (int j = 1; j < ny - 1; j++)
          rhs[o + j * st] = vt[o + j * st] + th * (a[j] * ut[o + (j - 1) * st] +
                                                   b[j] * ut[o + j * st] +
                                                   cc[j] * ut[o + (j + 1) * st]);
        rhs[o + (ny - 1) * st] =
            vt[o + (ny - 1) * st] +
            th * (a[ny - 1] * ut[o + (ny - 2) * st] + b[ny - 1] * ut[o + (ny - 1) * st]);
      }
#pragma omp parallel for collapse(2)
    for (int k = 0; k < nz; k++)
      for (int i = 0; i < nx; i++) {
        long o = i + (long)nx * (long)ny * k, st = nx;
        double *x = rhs + o, *cpl = cp + o;
        double beta = 1 - th * b[0];
        cpl[0] = -th * cc[0] / beta;
        x[0] = x[0] / beta;
        for (int j = 1; j < ny; j++) {
          beta = (1 - th * b[j]) + th * a[j] * cpl[(j - 1) * st];
          cpl[j * st] = -th * cc[j] / beta;
          x[j * st] = (x[j * st] + th * a[j] * x[(j - 1) * st]) / beta;
        }
        for (int j = ny - 2; j >= 0; j--) x[j * st] -= cpl[j * st] * x[(j + 1) * st];
      }
    copy_in(s, u[c], rhs);
  }
}

/* ------------------------------------------------------------- timestep -- */

static const double RK_A[3] = {0.0, -5.0 / 9.0, -153.0 / 128.0};
static const double RK_B[3] = {1.0 / 3.0, 15.0 / 16.0, 8.0 / 15.0};
static const double RK_AL[3] = {1.0 / 3.0, 5.0 / 12.0, 1.0 / 4.0};

/* step! (src/timestep.jl:41-63) */
void dnso_step(dnso_t *s, double *ux, double *uy, double *uz, double *p,
               double *qx, double *qy, double *qz, double *delta, double dt) {
  int nx = s->nx, ny = s->ny, nz = s->nz;
  double *u[3] = {ux, uy, uz}, *q[3] = {qx, qy, qz};
  for (int st = 0; st < 3; st++) {
    double A = RK_A[st], B = RK_B[st], al = RK_AL[st];
    dnso_momentum(s, qx, qy, qz, ux, uy, uz, A, dt);
    if (s->imexy) {
      dnso_imex_update(s, ux, uy, uz, qx, qy, qz, p, B, al, dt);
      fill_halo3(s, ux, uy, uz);
      dnso_project(s, ux, uy, uz, delta);
      double adt = al * dt;
#pragma omp parallel for
      for (int K = 1; K <= nz; K++)
        for (int J = 1; J <= ny; J++)
          for (int I = 1; I <= nx; I++) {
            long id = IDX(s, I, J, K);
            p[id] = p[id] + delta[id] / adt;
          }
      dnso_fill_halo(s, p, 3);
    } else {
      for (int c = 0; c < 3; c++) {
        int jh = jhi(s, c);
#pragma omp parallel for
        for (int K = 1; K <= nz; K++)
          for (int J = 1; J <= jh; J++)
            for (int I = 1; I <= nx; I++) {
              long id = IDX(s, I, J, K);
              u[c][id] = u[c][id] + B * q[c][id];
            }
      }
      fill_halo3(s, ux, uy, uz);
      dnso_project(s, ux, uy, uz, p);
    }
  }
}

static double maxabs_interior(const dnso_t *s, const double *phi) {
  double m = 0;
#pragma omp parallel for reduction(max : m)
  for (int K = 1; K <= s->nz; K++)
    for (int J = 1; J <= s->ny; J++)
      for (int I = 1; I <= s->nx; I++) {
        double v = fabs(phi[IDX(s, I, J, K)]);
        if (v > m) m = v;
      }
  return m;
}

/* cfl_timestep (src/timestep.jl:69-80) */
double dnso_cfl(const dnso_t *s, const double *ux, const double *uy,
                const double *uz, double cfl) {
  const double eps = 2.220446049250313e-16;
  double c1 = s->dx / (maxabs_interior(s, ux) + eps);
  double c2 = s->dymin / (maxabs_interior(s, uy) + eps);
  double c3 = s->dz / (maxabs_interior(s, uz) + eps);
  double conv = fmin(fmin(c1, c2), c3);
  double invdy2 = s->imexy ? 0.0 : 1 / (s->dymin * s->dymin);
  double diff = 1 / (2 * s->visc * (1 / (s->dx * s->dx) + invdy2 + 1 / (s->dz * s->dz)) + eps);
  return fmin(cfl * conv, cfl * diff);
}

double dnso_maxdiv(dnso_t *s, const double *ux, const double *uy, const double *uz) {
  dnso_divergence(s, ux, uy, uz, s->r);
  long n = (long)s->nx * s->ny * s->nz;
  double m = 0;
#pragma omp parallel for reduction(max : m)
  for (long i = 0; i < n; i++) {
    double v = fabs(s->r[i]);
    if (v > m) m = v;
  }
  return m;
}

/* kinetic_energy (src/fields.jl:45-60): host loop in k, j, i order */
double dnso_kinetic_energy(const dnso_t *s, const double *ux, const double *uy,
                           const double *uz) {
  const double *u[3] = {ux, uy, uz};
  double e = 0;
  for (int c = 0; c < 3; c++) {
    const double *D2 = c == 1 ? s->dyu : s->dy;
    int jh = jhi(s, c);
    for (int K = 1; K <= s->nz; K++)
      for (int J = 1; J <= jh; J++)
        for (int I = 1; I <= s->nx; I++) {
          double v = u[c][IDX(s, I, J, K)];
          e += v * v * s->dx * D2[J] * s->dz / 2;
        }
  }
  return e;
}

/* ---------------------------------------------------------------- stats -- */

/* sample_channelstats! (src/stats.jl:39-58): plane sums over (x, z) */
void dnso_channel_sample(const dnso_t *s, const double *ux, const double *uy,
                         const double *uz, double *acc) {
  int nx = s->nx, ny = s->ny, nz = s->nz, nf = s->wall ? ny - 1 : ny;
  double *Uc = acc, *Wc = acc + ny, *uuc = acc + 2 * ny, *wwc = acc + 3 * ny;
  double *Vf = acc + 4 * ny, *vvf = Vf + nf, *Uf = vvf + nf, *uvf = Uf + nf;
  for (int J = 1; J <= ny; J++) {
    double a = 0, b = 0, c = 0, d = 0;
    for (int K = 1; K <= nz; K++)
      for (int I = 1; I <= nx; I++) {
        double x = ux[IDX(s, I, J, K)], z = uz[IDX(s, I, J, K)];
        a += x; b += z; c += x * x; d += z * z;
      }
    Uc[J - 1] += a; Wc[J - 1] += b; uuc[J - 1] += c; wwc[J - 1] += d;
  }
  for (int J = 1; J <= nf; J++) {
    double a = 0, b = 0, c = 0, d = 0;
    for (int K = 1; K <= nz; K++)
      for (int I = 1; I <= nx; I++) {
        double v = uy[IDX(s, I, J, K)];
        double uf = (ux[IDX(s, I, J, K)] + ux[IDX(s, I, J + 1, K)]) / 2;
        double vf = (uy[IDX(s, I, J, K)] + uy[IDX(s, I + 1, J, K)]) / 2;
        a += v; b += v * v; c += uf; d += uf * vf;
      }
    Vf[J - 1] += a; vvf[J - 1] += b; Uf[J - 1] += c; uvf[J - 1] += d;
  }
}

/* sample_spectrum! + binshells! (src/stats.jl:120-157) */
void dnso_spectrum_sample(dnso_t *s, const double *ux, const double *uy,
                          const double *uz, double *E, int nbins) {
  int nx = s->nx, ny = s->ny, nz = s->nz, nkx = s->nkx;
  const double *u[3] = {ux, uy, uz};
  long sj = nkx, sk = (long)nkx * ny;
  double N2 = (double)nx * ny * nz;
  N2 = N2 * N2;
  for (int c = 0; c < 3; c++) {
    copy_out(s, u[c], s->r);
#pragma omp parallel
    {
      int nmax = nx > ny ? nx : ny;
      if (nz > nmax) nmax = nz;
      cplx *s1 = (cplx *)malloc(sizeof(cplx) * (nmax + 2));
      cplx *s2 = (cplx *)malloc(sizeof(cplx) * (nmax + 2));
#pragma omp for collapse(2)
      for (int k = 0; k < nz; k++)
        for (int j = 0; j < ny; j++)
          rfft_line(&s->px_half, s->wnx, s->r + (long)nx * (j + (long)ny * k), nx,
                    s->ah + j * sj + k * sk, 1, s1, s2);
#pragma omp for collapse(2)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nkx; i++) fft_line(&s->pz, s->ah + i + j * sj, sk, 0, s1, s2);
#pragma omp for collapse(2)
      for (int k = 0; k < nz; k++)
        for (int i = 0; i < nkx; i++) fft_line(&s->py, s->ah + i + k * sk, sj, 0, s1, s2);
      free(s1);
      free(s2);
    }
    for (int k = 0; k < nz; k++)
      for (int j = 0; j < ny; j++)
        for (int i = 0; i < nkx; i++) {
          int kx = i;
          int ky = j > ny / 2 ? j - ny : j;
          int kz = k > nz / 2 ? k - nz : k;
          int kap = (int)lround(sqrt((double)(kx * kx + ky * ky + kz * kz)));
          double wgt = (0 < kx && 2 * kx < nx) ? 2.0 : 1.0;
          cplx a = s->ah[i + j * sj + k * sk];
          double a2 = creal(a) * creal(a) + cimag(a) * cimag(a);
          if (kap < nbins) E[kap] += wgt * a2 / 2 / N2;
        }
  }
}

/* ---------------------------------------------------------------- noise -- */

static uint64_t splitmix64(uint64_t x) {
  uint64_t z = x + 0x9e3779b97f4a7c15ULL;
  z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
  z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
  return z ^ (z >> 31);
}

void dnso_noise(const dnso_t *s, double *phi, int c, unsigned long long seed,
                double amp) {
  int nx = s->nx, ny = s->ny, nz = s->nz, jh = jhi(s, c);
  for (int K = 1; K <= nz; K++)
    for (int J = 1; J <= jh; J++)
      for (int I = 1; I <= nx; I++) {
        uint64_t key = (((uint64_t)c * nz + (K - 1)) * ny + (J - 1)) * nx + (I - 1);
        uint64_t r = splitmix64((uint64_t)seed + key);
        double U = ((double)(r >> 11) + 0.5) * 0x1p-53;
        phi[IDX(s, I, J, K)] += amp * (2 * U - 1);
      }
}
