/*
 * gfd_oracle.c -- TEST INFRASTRUCTURE, NOT PRODUCT CODE.
 *
 * A plain-C CPU restatement of GPAW's real-space finite-difference path, used
 * only as the checker for the CUDA library (tests, smoke check, and the CPU
 * baseline leg of the benchmark).  Nothing in the product links or calls it.
 *
 * Algorithms restated (reference paths are relative to the GPAW source tree):
 *   halo fill   c/bc.c:138-250 (bc_unpack1: zero everything, paste interior,
 *               periodic self-copy of the opposite slab times phases[d]; with
 *               cfd==0 later axes include earlier halos, so corners carry the
 *               product of phases, c/bc.c:108-112)
 *   stencil     c/bmgs/fd.c:16-51   out[g] = sum_c coefs[c] * padded[g+off[c]]
 *   relaxation  c/bmgs/relax.c:7-73 lexicographic Gauss-Seidel (method 1) or
 *               weighted Jacobi (any other method); coefs[0] is the diagonal
 *   restriction c/bmgs/restrict.c:18-154  three separable 1-D passes (z, y, x)
 *   interpolate c/bmgs/interpolate.c:19-168 three separable 1-D passes with skip
 *   band loops  c/operators.c:109-157 (apply), c/operators.c:49-91 (relax),
 *               c/transformers.c:54-123 (transformer apply)
 *
 * Complex arrays are interleaved (re, im) doubles.  Phases are given as 12
 * doubles: phase_cd[c][d] = (re, im) at index 4*c + 2*d.  The low halo on
 * axis c gets phase_cd[c][1], the high halo gets phase_cd[c][0]
 * (c/bc.c:234-249: slab d is copied to the opposite side times phases[d]).
 *
 * Periodic axes must hold at least as many points as the halo is wide; the
 * reference's self-copy is only a plain wrap under that condition.
 */
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#include <pthread.h>

#define ORC_OK 0
#define ORC_EINVAL 1
#define ORC_ENOMEM 2

/* ------------------------------------------------------------------------ */
/* Halo-padded copy of one band.                                            */
/* ------------------------------------------------------------------------ */

typedef struct {
  int64_t n[3];     /* interior points per axis */
  int64_t lo[3];    /* halo width below the interior */
  int64_t hi[3];    /* halo width above the interior */
  int periodic[3];  /* 1: wrap with phase, 0: zero halo */
} halo_spec;

static int64_t padded_len(const halo_spec* h, int a) {
  return h->n[a] + h->lo[a] + h->hi[a];
}

/* Map padded coordinate t (0-based in the padded axis) to an interior index.
 * Returns 0 when the point is a zero halo point.  *which is -1 for no wrap,
 * 1 for the low halo (takes phase_cd[c][1]) and 0 for the high halo. */
static int map_axis(const halo_spec* h, int a, int64_t t, int64_t* src, int* which) {
  int64_t u = t - h->lo[a];
  *which = -1;
  if (u >= 0 && u < h->n[a]) { *src = u; return 1; }
  if (!h->periodic[a]) return 0;
  if (u < 0) { *src = u + h->n[a]; *which = 1; }
  else       { *src = u - h->n[a]; *which = 0; }
  return 1;
}

static void fill_padded(const halo_spec* h, int nc, const double* in, double* buf,
                        const double* ph) {
  int64_t m0 = padded_len(h, 0), m1 = padded_len(h, 1), m2 = padded_len(h, 2);
  for (int64_t i0 = 0; i0 < m0; i0++) {
    int64_t s0 = 0; int w0 = -1;
    int ok0 = map_axis(h, 0, i0, &s0, &w0);
    for (int64_t i1 = 0; i1 < m1; i1++) {
      int64_t s1 = 0; int w1 = -1;
      int ok1 = map_axis(h, 1, i1, &s1, &w1);
      double* dst = buf + ((i0 * m1 + i1) * m2) * nc;
      for (int64_t i2 = 0; i2 < m2; i2++) {
        int64_t s2 = 0; int w2 = -1;
        int ok2 = map_axis(h, 2, i2, &s2, &w2);
        if (!(ok0 && ok1 && ok2)) {
          for (int q = 0; q < nc; q++) dst[i2 * nc + q] = 0.0;
          continue;
        }
        const double* v = in + ((s0 * h->n[1] + s1) * h->n[2] + s2) * nc;
        if (nc == 1 || ph == NULL) {
          for (int q = 0; q < nc; q++) dst[i2 * nc + q] = v[q];
          continue;
        }
        /* Apply the phase of each wrapped axis in axis order, the order in
         * which the reference's sequential axis passes multiply them in. */
        double re = v[0], im = v[1];
        int w[3] = {w0, w1, w2};
        for (int c = 0; c < 3; c++) {
          if (w[c] < 0) continue;
          double pr = ph[4 * c + 2 * w[c]], pi = ph[4 * c + 2 * w[c] + 1];
          double nr = pr * re - pi * im;
          double ni = pr * im + pi * re;
          re = nr; im = ni;
        }
        dst[i2 * nc] = re;
        dst[i2 * nc + 1] = im;
      }
    }
  }
}

static int check_halo(const halo_spec* h) {
  for (int a = 0; a < 3; a++) {
    if (h->n[a] < 0 || h->lo[a] < 0 || h->hi[a] < 0) return ORC_EINVAL;
    if (h->periodic[a] && h->n[a] > 0 && (h->lo[a] > h->n[a] || h->hi[a] > h->n[a]))
      return ORC_EINVAL;
  }
  return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* Band-parallel driver: bands are split across pthreads in contiguous      */
/* chunks, as the reference's GPAW_OMP workers do (c/operators.c:116-124).  */
/* ------------------------------------------------------------------------ */

typedef void (*band_fn)(void* ctx, int64_t band, double* scratch);

typedef struct {
  band_fn fn;
  void* ctx;
  int64_t b0, b1;
  size_t scratch_doubles;
  int status;
} band_job;

static void* band_worker(void* arg) {
  band_job* j = (band_job*)arg;
  double* scratch = NULL;
  if (j->scratch_doubles) {
    scratch = (double*)malloc(j->scratch_doubles * sizeof(double));
    if (!scratch) { j->status = ORC_ENOMEM; return NULL; }
  }
  for (int64_t b = j->b0; b < j->b1; b++) j->fn(j->ctx, b, scratch);
  free(scratch);
  j->status = ORC_OK;
  return NULL;
}

static int run_bands(band_fn fn, void* ctx, int64_t nbands, size_t scratch_doubles,
                     int nthreads) {
  if (nbands <= 0) return ORC_OK;
  if (nthreads < 1) nthreads = 1;
  if (nthreads > nbands) nthreads = (int)nbands;
  band_job* jobs = (band_job*)calloc((size_t)nthreads, sizeof(band_job));
  pthread_t* th = (pthread_t*)calloc((size_t)nthreads, sizeof(pthread_t));
  if (!jobs || !th) { free(jobs); free(th); return ORC_ENOMEM; }
  int64_t per = nbands / nthreads, rem = nbands % nthreads, start = 0;
  for (int t = 0; t < nthreads; t++) {
    int64_t cnt = per + (t < rem ? 1 : 0);
    jobs[t].fn = fn; jobs[t].ctx = ctx;
    jobs[t].b0 = start; jobs[t].b1 = start + cnt;
    jobs[t].scratch_doubles = scratch_doubles;
    start += cnt;
  }
  for (int t = 1; t < nthreads; t++) pthread_create(&th[t], NULL, band_worker, &jobs[t]);
  band_worker(&jobs[0]);
  int status = jobs[0].status;
  for (int t = 1; t < nthreads; t++) {
    pthread_join(th[t], NULL);
    if (jobs[t].status) status = jobs[t].status;
  }
  free(jobs); free(th);
  return status;
}

/* ------------------------------------------------------------------------ */
/* Stencil apply  (c/bmgs/fd.c, c/operators.c:109-157)                      */
/* ------------------------------------------------------------------------ */

typedef struct {
  halo_spec h;
  int nc;
  int P;
  const double* coefs;
  int64_t* flat;        /* flat offsets on the padded grid */
  const double* in;
  double* out;
  const double* ph;
} fd_ctx;

static void fd_band(void* vctx, int64_t b, double* buf) {
  fd_ctx* c = (fd_ctx*)vctx;
  const halo_spec* h = &c->h;
  int64_t ng = h->n[0] * h->n[1] * h->n[2];
  int64_t m1 = padded_len(h, 1), m2 = padded_len(h, 2);
  fill_padded(h, c->nc, c->in + b * ng * c->nc, buf, c->ph);
  double* out = c->out + b * ng * c->nc;
  for (int64_t i0 = 0; i0 < h->n[0]; i0++)
    for (int64_t i1 = 0; i1 < h->n[1]; i1++)
      for (int64_t i2 = 0; i2 < h->n[2]; i2++) {
        int64_t g = ((i0 + h->lo[0]) * m1 + (i1 + h->lo[1])) * m2 + (i2 + h->lo[2]);
        double* o = out + ((i0 * h->n[1] + i1) * h->n[2] + i2) * c->nc;
        if (c->nc == 1) {
          double x = 0.0;
          for (int p = 0; p < c->P; p++) x += buf[g + c->flat[p]] * c->coefs[p];
          o[0] = x;
        } else {
          double xr = 0.0, xi = 0.0;
          for (int p = 0; p < c->P; p++) {
            const double* a = buf + 2 * (g + c->flat[p]);
            xr += a[0] * c->coefs[p];
            xi += a[1] * c->coefs[p];
          }
          o[0] = xr; o[1] = xi;
        }
      }
}

static int stencil_setup(int P, const int64_t* off, const int64_t n[3], const int periodic[3],
                         halo_spec* h, int64_t** flat_out) {
  int64_t mp = 0;
  for (int p = 0; p < 3 * P; p++) {
    int64_t a = off[p] < 0 ? -off[p] : off[p];
    if (a > mp) mp = a;
  }
  for (int a = 0; a < 3; a++) {
    h->n[a] = n[a]; h->lo[a] = mp; h->hi[a] = mp; h->periodic[a] = periodic[a] ? 1 : 0;
  }
  if (check_halo(h)) return ORC_EINVAL;
  int64_t m1 = padded_len(h, 1), m2 = padded_len(h, 2);
  int64_t* flat = (int64_t*)malloc(sizeof(int64_t) * (size_t)(P > 0 ? P : 1));
  if (!flat) return ORC_ENOMEM;
  for (int p = 0; p < P; p++) flat[p] = (off[3 * p] * m1 + off[3 * p + 1]) * m2 + off[3 * p + 2];
  *flat_out = flat;
  return ORC_OK;
}

int orc_fd_apply(int P, const double* coefs, const int64_t* offsets, const int64_t n[3],
                 const int periodic[3], int nc, int64_t nbands, const double* in,
                 double* out, const double* phases, int nthreads) {
  fd_ctx c;
  int st = stencil_setup(P, offsets, n, periodic, &c.h, &c.flat);
  if (st) return st;
  c.nc = nc; c.P = P; c.coefs = coefs; c.in = in; c.out = out;
  c.ph = (nc == 2) ? phases : NULL;
  size_t scratch = (size_t)(padded_len(&c.h, 0) * padded_len(&c.h, 1) * padded_len(&c.h, 2)) * nc;
  st = run_bands(fd_band, &c, nbands, scratch, nthreads);
  free(c.flat);
  return st;
}

/* ------------------------------------------------------------------------ */
/* Relaxation  (c/bmgs/relax.c, c/operators.c:49-91) -- real arrays only    */
/* ------------------------------------------------------------------------ */

int orc_relax(int method, int P, const double* coefs, const int64_t* offsets,
              const int64_t n[3], const int periodic[3], double* phi, const double* rho,
              int nsweeps, double w) {
  halo_spec h;
  int64_t* flat = NULL;
  int st = stencil_setup(P, offsets, n, periodic, &h, &flat);
  if (st) return st;
  int64_t m0 = padded_len(&h, 0), m1 = padded_len(&h, 1), m2 = padded_len(&h, 2);
  double* buf = (double*)malloc(sizeof(double) * (size_t)(m0 * m1 * m2));
  if (!buf) { free(flat); return ORC_ENOMEM; }
  const double inv_diag = 1.0 / coefs[0];
  for (int s = 0; s < nsweeps; s++) {
    fill_padded(&h, 1, phi, buf, NULL);
    for (int64_t i0 = 0; i0 < n[0]; i0++)
      for (int64_t i1 = 0; i1 < n[1]; i1++)
        for (int64_t i2 = 0; i2 < n[2]; i2++) {
          int64_t g = ((i0 + h.lo[0]) * m1 + (i1 + h.lo[1])) * m2 + (i2 + h.lo[2]);
          int64_t q = (i0 * n[1] + i1) * n[2] + i2;
          double x = 0.0;
          for (int p = 1; p < P; p++) x += buf[g + flat[p]] * coefs[p];
          if (method == 1) {
            /* Gauss-Seidel: later points in the sweep see this update. */
            double v = (rho[q] - x) * inv_diag;
            phi[q] = v;
            buf[g] = v;
          } else {
            phi[q] = (1.0 - w) * phi[q] + w * (rho[q] - x) / coefs[0];
          }
        }
  }
  free(buf); free(flat);
  return ORC_OK;
}

/* ------------------------------------------------------------------------ */
/* Restriction and interpolation (c/bmgs/restrict.c, interpolate.c,         */
/* c/transformers.c:54-123).  Weights are the Lagrange weights of the       */
/* reference for K = 2, 4, 6, 8 taps.                                       */
/* ------------------------------------------------------------------------ */

static const double LAGRANGE_W[4][4] = {
  {0.5, 0.0, 0.0, 0.0},
  {0.5625, -0.0625, 0.0, 0.0},
  {0.58593750, -0.09765625, 0.01171875, 0.0},
  {0.59814453125, -0.11962890625, 0.02392578125, -0.00244140625},
};

/* One restriction tap sum along a line with unit spacing `st` between
 * consecutive fine points:  0.5*(a0 + w1*(a[+1]+a[-1]) + w2*(a[+3]+a[-3]) ...) */
static inline double rst_tap(const double* a, int64_t st, int nn) {
  const double* w = LAGRANGE_W[nn - 1];
  double x = a[0];
  for (int k = 0; k < nn; k++) x += w[k] * (a[(2 * k + 1) * st] + a[-(2 * k + 1) * st]);
  return 0.5 * x;
}

/* Interpolated value between a[0] and a[st]. */
static inline double ip_tap(const double* a, int64_t st, int nn) {
  const double* w = LAGRANGE_W[nn - 1];
  double x = 0.0;
  for (int m = 0; m < nn; m++) {
    double t = w[m] * (a[-m * st] + a[(1 + m) * st]);
    x = (m == 0) ? t : x + t;
  }
  return x;
}

typedef struct {
  halo_spec h;     /* input grid with its transformer padding */
  int nc;
  int nn;          /* K / 2 */
  int interpolate;
  int64_t skip[3][2];
  int64_t nout[3];
  const double* in;
  double* out;
  const double* ph;
} tr_ctx;

/* 1-D restriction of every line along axis `ax` of the array `a` with
 * shape s[3] (all axes padded or already reduced), into b of shape r[3]
 * where r[ax] = (s[ax] - (4nn-3)) / 2. */
static void restrict_axis(const double* a, const int64_t s[3], double* b, const int64_t r[3],
                          int ax, int nn, int nc) {
  int64_t st_a[3] = {s[1] * s[2], s[2], 1};
  int64_t st_b[3] = {r[1] * r[2], r[2], 1};
  int64_t first = 2 * nn - 1;   /* K - 1: first fine point with a full left wing */
  for (int64_t i0 = 0; i0 < r[0]; i0++)
    for (int64_t i1 = 0; i1 < r[1]; i1++)
      for (int64_t i2 = 0; i2 < r[2]; i2++) {
        int64_t idx[3] = {i0, i1, i2};
        int64_t src[3] = {i0, i1, i2};
        src[ax] = first + 2 * idx[ax];
        int64_t ga = src[0] * st_a[0] + src[1] * st_a[1] + src[2] * st_a[2];
        int64_t gb = i0 * st_b[0] + i1 * st_b[1] + i2 * st_b[2];
        for (int q = 0; q < nc; q++)
          b[gb * nc + q] = rst_tap(a + ga * nc + q, st_a[ax] * nc, nn);
      }
}

/* 1-D interpolation along axis `ax`: the line has s[ax] padded coarse
 * points; ncore = s[ax] - (2nn-1) + skip1 steps each give an even (copy)
 * and an odd (interpolated) output, minus the skipped first even / last odd. */
static void interp_axis(const double* a, const int64_t s[3], double* b, const int64_t r[3],
                        int ax, int nn, int nc, const int64_t skip[2]) {
  int64_t st_a[3] = {s[1] * s[2], s[2], 1};
  int64_t st_b[3] = {r[1] * r[2], r[2], 1};
  int64_t base = nn - 1;
  for (int64_t i0 = 0; i0 < r[0]; i0++)
    for (int64_t i1 = 0; i1 < r[1]; i1++)
      for (int64_t i2 = 0; i2 < r[2]; i2++) {
        int64_t idx[3] = {i0, i1, i2};
        int64_t f = idx[ax] + skip[0];   /* output index before skipping */
        int64_t i = f / 2;               /* coarse step */
        int64_t src[3] = {i0, i1, i2};
        src[ax] = base + i;
        int64_t ga = src[0] * st_a[0] + src[1] * st_a[1] + src[2] * st_a[2];
        int64_t gb = i0 * st_b[0] + i1 * st_b[1] + i2 * st_b[2];
        for (int q = 0; q < nc; q++) {
          const double* p = a + ga * nc + q;
          b[gb * nc + q] = (f % 2 == 0) ? p[0] : ip_tap(p, st_a[ax] * nc, nn);
        }
      }
}

static void tr_band(void* vctx, int64_t b, double* scratch) {
  tr_ctx* c = (tr_ctx*)vctx;
  const halo_spec* h = &c->h;
  int64_t s[3] = {padded_len(h, 0), padded_len(h, 1), padded_len(h, 2)};
  int64_t ngin = h->n[0] * h->n[1] * h->n[2];
  int64_t ngout = c->nout[0] * c->nout[1] * c->nout[2];
  double* pad = scratch;
  double* t1 = pad + s[0] * s[1] * s[2] * c->nc;
  fill_padded(h, c->nc, c->in + b * ngin * c->nc, pad, c->ph);
  double* out = c->out + b * ngout * c->nc;
  if (!c->interpolate) {
    int64_t e = 4 * c->nn - 3;
    int64_t r1[3] = {s[0], s[1], (s[2] - e) / 2};
    int64_t r2[3] = {s[0], (s[1] - e) / 2, r1[2]};
    int64_t r3[3] = {(s[0] - e) / 2, r2[1], r2[2]};
    double* t2 = t1 + r1[0] * r1[1] * r1[2] * c->nc;
    restrict_axis(pad, s, t1, r1, 2, c->nn, c->nc);
    restrict_axis(t1, r1, t2, r2, 1, c->nn, c->nc);
    restrict_axis(t2, r2, out, r3, 0, c->nn, c->nc);
  } else {
    int64_t e = 2 * c->nn - 1;
    int64_t len[3];
    for (int a = 0; a < 3; a++) len[a] = 2 * (s[a] - e + c->skip[a][1]) - c->skip[a][0] - c->skip[a][1];
    int64_t r1[3] = {s[0], s[1], len[2]};
    int64_t r2[3] = {s[0], len[1], len[2]};
    int64_t r3[3] = {len[0], len[1], len[2]};
    double* t2 = t1 + r1[0] * r1[1] * r1[2] * c->nc;
    interp_axis(pad, s, t1, r1, 2, c->nn, c->nc, c->skip[2]);
    interp_axis(t1, r1, t2, r2, 1, c->nn, c->nc, c->skip[1]);
    interp_axis(t2, r2, out, r3, 0, c->nn, c->nc, c->skip[0]);
  }
}

/* pad[6], skip[6] as (axis, side) pairs; periodic[3]; nc 1 (real) or 2. */
int orc_transform(int interpolate, int K, const int64_t nin[3], const int64_t pad[6],
                  const int64_t skip[6], const int periodic[3], int nc, int64_t nbands,
                  const double* in, double* out, const double* phases, int nthreads) {
  if (K != 2 && K != 4 && K != 6 && K != 8) return ORC_EINVAL;
  tr_ctx c;
  memset(&c, 0, sizeof(c));
  c.nc = nc; c.nn = K / 2; c.interpolate = interpolate;
  c.in = in; c.out = out; c.ph = (nc == 2) ? phases : NULL;
  for (int a = 0; a < 3; a++) {
    c.h.n[a] = nin[a]; c.h.lo[a] = pad[2 * a]; c.h.hi[a] = pad[2 * a + 1];
    c.h.periodic[a] = periodic[a] ? 1 : 0;
    c.skip[a][0] = interpolate ? skip[2 * a] : 0;
    c.skip[a][1] = interpolate ? skip[2 * a + 1] : 0;
  }
  if (check_halo(&c.h)) return ORC_EINVAL;
  int64_t s[3], t1 = 0, t2 = 0;
  for (int a = 0; a < 3; a++) s[a] = padded_len(&c.h, a);
  if (!interpolate) {
    int64_t e = 4 * c.nn - 3;
    for (int a = 0; a < 3; a++) {
      if (s[a] < e || (s[a] - e) % 2) return ORC_EINVAL;
      c.nout[a] = (s[a] - e) / 2;
    }
    t1 = s[0] * s[1] * c.nout[2];
    t2 = s[0] * c.nout[1] * c.nout[2];
  } else {
    int64_t e = 2 * c.nn - 1;
    for (int a = 0; a < 3; a++) {
      c.nout[a] = 2 * (s[a] - e + c.skip[a][1]) - c.skip[a][0] - c.skip[a][1];
      if (c.nout[a] < 0) return ORC_EINVAL;
    }
    t1 = s[0] * s[1] * c.nout[2];
    t2 = s[0] * c.nout[1] * c.nout[2];
  }
  size_t scratch = (size_t)(s[0] * s[1] * s[2] + t1 + t2) * nc;
  return run_bands(tr_band, &c, nbands, scratch, nthreads);
}

/* Output shape of a transform, for the caller's allocation. */
int orc_transform_shape(int interpolate, int K, const int64_t nin[3], const int64_t pad[6],
                        const int64_t skip[6], int64_t nout[3]) {
  int nn = K / 2;
  for (int a = 0; a < 3; a++) {
    int64_t s = nin[a] + pad[2 * a] + pad[2 * a + 1];
    if (!interpolate) nout[a] = (s - (4 * nn - 3)) / 2;
    else nout[a] = 2 * (s - (2 * nn - 1) + skip[2 * a + 1]) - skip[2 * a] - skip[2 * a + 1];
  }
  return ORC_OK;
}
