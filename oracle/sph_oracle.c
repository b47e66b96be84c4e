/*
 * sph_oracle.c -- FP64 CPU restatement of CUDAsph's per-step SPH + self-gravity
 * pipeline.
 *
 * THIS FILE IS TEST INFRASTRUCTURE.  It is the checker that the CUDA library in
 * cudasph_b200/ is compared against; only tests/, __graft_entry__.smoke() and
 * the cpu_baseline leg of bench.py load it.  The product never links it.
 *
 * Every routine restates one loop of the reference (3gx/CUDAsph) in double
 * precision and cites the reference file:line it follows.  Arithmetic is plain
 * IEEE double, compiled with -ffp-contract=off so that the neighbour predicate
 * ds2 = (dx*dx + dy*dy) + dz*dz, ds2 < range*range is bit-identical to the
 * non-contracted form the GPU kernels use.
 *
 * Deliberate departures from the reference:
 *   - double instead of float everywhere (the reference device code is FP32);
 *   - the divergence/curl weight uses m_j, not m_i (dev_density_loop.cu:64 has
 *     m_i; identical for equal masses);
 *   - the EOS closed-form quartic root is polished by Newton iterations;
 *   - the hard neighbour count n_ngb is the count at the final range
 *     (dev_solve_range.cu:408 can differ from it by one through round-off);
 *   - the Psi (softening grad-h) term in the hydro force is switchable; it is
 *     only meaningful with the h-dependent spline softening;
 *   - Plummer softening is offered next to the reference spline softening.
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_PI 3.141592653589793
#define ORC_IPI 0.318309886183791

typedef struct {
  double n_target;   /* DESIRED_NGB, dev_solve_range.cu:14 (24 in the reference) */
  double rel_err;    /* CUDA_calls.cpp:4 (1e-3) */
  int max_iter;      /* MAX_ITER, dev_solve_range.cu:15 (20) */
  double f_scale;    /* dev_solve_range.cu:92 (0.1) */
  double av_alpha;   /* CUDA_calls.cpp:13 */
  double av_beta;    /* CUDA_calls.cpp:14 */
  double gamma;      /* dev_art_visc.cu:15 (5/3) */
  int eos_mode;      /* 0 ideal gas, 1 ideal gas + radiation (dev_compute_pressure.cu) */
  int soft_mode;     /* 0 spline softening at range (sph_grav_kernel.cu:14-111), 1 Plummer */
  double eps;        /* Plummer softening length */
  int use_psi;       /* include the Psi term of dev_hydro_dots.cu:69-70 */
  double cn1, cn2;   /* compute_timestep.cpp:4-5 */
  double G;          /* gravitational constant (1 in the reference's solar units) */
} orc_params;

/* ------------------------------------------------------------------ */
/* Kernel functions: dev_sph_kernels.cu:7-99 (M4 cubic spline family)   */
/* ------------------------------------------------------------------ */

/* dev_sph_kernels.cu:7-16 */
double orc_w(double u) {
  if (u < 0) return ORC_IPI;
  if (u < 1) return ORC_IPI * (1 - 1.5 * u * u + 0.75 * u * u * u);
  if (u < 2) return ORC_IPI * 0.25 * (2 - u) * (2 - u) * (2 - u);
  return 0;
}
/* dev_sph_kernels.cu:18-20 (4*pi*u^2*w(u)) */
double orc_diw(double u) { return 4.0 * ORC_PI * u * u * orc_w(u); }
/* dev_sph_kernels.cu:22-34, the integral of diw */
double orc_iw(double u) {
  if (u < 0) return 0;
  if (u < 1) {
    double u3 = u * u * u;
    return 4 * (u3 / 3.0 - 0.3 * u3 * u * u + 0.125 * u3 * u3);
  }
  if (u < 2) {
    double u3 = u * u * u;
    return 4 * (-1.0 / 60 + 2.0 / 3 * u3 - 0.75 * u3 * u + 0.3 * u3 * u * u - u3 * u3 / 24.0);
  }
  return 1;
}
/* dev_sph_kernels.cu:36-48: smooth neighbour-count weight */
double orc_ig(double u) { return orc_iw(4.0 * (1.0 - fabs(u - 1.0))); }
/* dev_sph_kernels.cu:50-60 */
double orc_digdh(double u) {
  if (u <= 0) return 0;
  if (u < 1) return 4.0 * u * orc_diw(4.0 * u);
  if (u < 2) return -4.0 * u * orc_diw(4.0 * (2 - u));
  return 0;
}
/* dev_sph_kernels.cu:62-72 */
double orc_dig(double u) {
  if (u <= 0) return 0;
  if (u < 1) return 4.0 / u * orc_diw(4.0 * u);
  if (u < 2) return -4.0 / u * orc_diw(4.0 * (2 - u));
  return 0;
}
/* dev_sph_kernels.cu:74-81: (1/u) dW/du */
double orc_dw(double u) {
  if (u < 1) return ORC_IPI * (-3 + 2.25 * u);
  if (u < 2) return -ORC_IPI * 0.75 * (2 - u) * (2 - u) / u;
  return 0;
}
/* dev_sph_kernels.cu:83-90 */
double orc_dwdh(double u) {
  if (u < 1) return ORC_IPI * (-3 + 7.5 * u * u - 4.5 * u * u * u);
  if (u < 2) return ORC_IPI * (-6 + 12 * u - 7.5 * u * u + 1.5 * u * u * u);
  return 0;
}
/* dev_sph_kernels.cu:92-99 */
double orc_dphidh(double u) {
  double u2 = u * u;
  if (u < 1) return 1.4 - 2 * u2 + 1.5 * u2 * u2 - 0.6 * u2 * u2 * u;
  if (u < 2) return 1.6 - 4 * u2 + 4 * u2 * u - 1.5 * u2 * u2 + 0.2 * u2 * u2 * u;
  return 0;
}

/* Evaluate one kernel function over an array (known-answer tests). */
void orc_kernel_eval(int which, int n, const double *u, double *out) {
  for (int i = 0; i < n; i++) {
    double v = u[i], r = 0;
    switch (which) {
      case 0: r = orc_w(v); break;
      case 1: r = orc_dw(v); break;
      case 2: r = orc_dwdh(v); break;
      case 3: r = orc_dphidh(v); break;
      case 4: r = orc_iw(v); break;
      case 5: r = orc_ig(v); break;
      case 6: r = orc_dig(v); break;
      case 7: r = orc_digdh(v); break;
      case 8: r = orc_diw(v); break;
    }
    out[i] = r;
  }
}

/* The exact neighbour predicate of dev_find_ngb.cu:66-67 / dev_solve_range.cu:
 * 331-332 in double, without contraction: (dx*dx + dy*dy) + dz*dz. */
static inline double ds2_of(double dx, double dy, double dz) {
  double a = dx * dx;
  double b = dy * dy;
  double c = dz * dz;
  return (a + b) + c;
}

/* ------------------------------------------------------------------ */
/* Uniform-grid neighbour index (exact: a conservative cell scan, then   */
/* the predicate above).  Candidates come out in ascending particle id.  */
/* ------------------------------------------------------------------ */
typedef struct {
  int n, nc[3];
  double lo[3], cell;
  int *start, *idx; /* cell start offsets (ncell+1), particle ids sorted by cell then id */
} orc_grid;

static void grid_build(orc_grid *g, int n, const double *x, const double *y, const double *z, double cell) {
  const double *p[3] = {x, y, z};
  g->n = n;
  for (int d = 0; d < 3; d++) {
    double lo = p[d][0], hi = p[d][0];
    for (int i = 1; i < n; i++) { if (p[d][i] < lo) lo = p[d][i]; if (p[d][i] > hi) hi = p[d][i]; }
    g->lo[d] = lo;
    double ext = hi - lo;
    int k = (int)(ext / cell) + 1;
    if (k < 1) k = 1;
    if (k > 256) k = 256;
    g->nc[d] = k;
  }
  double ext = 0;
  for (int d = 0; d < 3; d++) {
    double hi = p[d][0];
    for (int i = 1; i < n; i++) if (p[d][i] > hi) hi = p[d][i];
    double e = (hi - g->lo[d]) / g->nc[d];
    if (e > ext) ext = e;
  }
  g->cell = ext > 0 ? ext * (1 + 1e-12) : 1.0;
  long nct = (long)g->nc[0] * g->nc[1] * g->nc[2];
  g->start = (int *)calloc(nct + 1, sizeof(int));
  g->idx = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
  int *cid = (int *)malloc(sizeof(int) * (n > 0 ? n : 1));
  for (int i = 0; i < n; i++) {
    int c[3];
    for (int d = 0; d < 3; d++) {
      int k = (int)((p[d][i] - g->lo[d]) / g->cell);
      if (k < 0) k = 0;
      if (k >= g->nc[d]) k = g->nc[d] - 1;
      c[d] = k;
    }
    cid[i] = (c[2] * g->nc[1] + c[1]) * g->nc[0] + c[0];
    g->start[cid[i] + 1]++;
  }
  for (long c = 0; c < nct; c++) g->start[c + 1] += g->start[c];
  int *fill = (int *)malloc(sizeof(int) * nct);
  memcpy(fill, g->start, sizeof(int) * nct);
  for (int i = 0; i < n; i++) g->idx[fill[cid[i]]++] = i; /* ids ascending within a cell */
  free(fill);
  free(cid);
}
static void grid_free(orc_grid *g) { free(g->start); free(g->idx); }

static int cmp_int(const void *a, const void *b) {
  int x = *(const int *)a, y = *(const int *)b;
  return (x > y) - (x < y);
}

/* All j with ds2 < R*R (ascending j) into buf; returns the count.  buf grows. */
static int grid_query(const orc_grid *g, const double *x, const double *y, const double *z,
                      double xi, double yi, double zi, double R, int **buf, int *cap, double **dbuf) {
  double q[3] = {xi, yi, zi};
  int lo[3], hi[3];
  for (int d = 0; d < 3; d++) {
    double a = (q[d] - R - g->lo[d]) / g->cell, b = (q[d] + R - g->lo[d]) / g->cell;
    int ka = (int)floor(a) - 1, kb = (int)floor(b) + 1;
    if (ka < 0) ka = 0;
    if (kb > g->nc[d] - 1) kb = g->nc[d] - 1;
    lo[d] = ka; hi[d] = kb;
  }
  double R2 = R * R;
  int cnt = 0;
  for (int cz = lo[2]; cz <= hi[2]; cz++)
    for (int cy = lo[1]; cy <= hi[1]; cy++)
      for (int cx = lo[0]; cx <= hi[0]; cx++) {
        int c = (cz * g->nc[1] + cy) * g->nc[0] + cx;
        for (int k = g->start[c]; k < g->start[c + 1]; k++) {
          int j = g->idx[k];
          double d2 = ds2_of(xi - x[j], yi - y[j], zi - z[j]);
          if (d2 < R2) {
            if (cnt == *cap) {
              *cap = *cap * 2 + 64;
              *buf = (int *)realloc(*buf, sizeof(int) * *cap);
              *dbuf = (double *)realloc(*dbuf, sizeof(double) * *cap);
            }
            (*buf)[cnt++] = j;
          }
        }
      }
  qsort(*buf, cnt, sizeof(int), cmp_int);
  for (int k = 0; k < cnt; k++) {
    int j = (*buf)[k];
    (*dbuf)[k] = ds2_of(xi - x[j], yi - y[j], zi - z[j]);
  }
  return cnt;
}

/* ------------------------------------------------------------------ */
/* h solve: dev_solve_range.cu:17-172                                   */
/* ------------------------------------------------------------------ */

/* compute_ngb, dev_solve_range.cu:17-89, over a candidate list (ascending j,
 * squared distances d2[]).  Returns f = sum ig - N, the Newton step dx, and
 * the hard count. */
static void compute_ngb(const double *d2, int nc, double w, const orc_params *p,
                        double *f_out, double *dx_out, double *cnt_out) {
  double f = 0, g = 0, c = 0;
  double w2 = w * w;
  for (int k = 0; k < nc; k++) {
    if (d2[k] < w2) {
      double u = 2 * sqrt(d2[k]) / w;
      f += orc_ig(u);
      g -= orc_digdh(u);
      c += 1;
    }
  }
  f -= p->n_target;
  g *= 1.0 / w;
  double dx;
  if (g != 0) dx = f / g;
  else dx = (f < 0) ? -w : +w;
  *f_out = f; *dx_out = dx; *cnt_out = c;
}

typedef struct {
  const orc_grid *g;
  const double *x, *y, *z;
  double xi, yi, zi;
  double R;       /* radius of the current candidate list */
  int nc, cap;
  int *buf;
  double *d2;
} cand_list;

static void cand_ensure(cand_list *cl, double w) {
  if (w <= cl->R && cl->nc >= 0) return;
  double R = w * 1.25;
  cl->nc = grid_query(cl->g, cl->x, cl->y, cl->z, cl->xi, cl->yi, cl->zi, R, &cl->buf, &cl->cap, &cl->d2);
  cl->R = R;
}

static void eval_ngb(cand_list *cl, double w, const orc_params *p, double *f, double *dx, double *cnt) {
  cand_ensure(cl, w);
  compute_ngb(cl->d2, cl->nc, w, p, f, dx, cnt);
}

/* dev_bracket_root, dev_solve_range.cu:93-135 */
static void bracket_root(cand_list *cl, double w, const orc_params *p, double *xl_out, double *xr_out,
                         double *cnt_out, int *nevals) {
  double f, dx, cnt;
  eval_ngb(cl, w, p, &f, &dx, &cnt); (*nevals)++;
  if (fabs(dx) < p->rel_err * w) {
    *xl_out = w - 0.5 * fabs(dx); *xr_out = w + 0.5 * fabs(dx); *cnt_out = cnt;
    return;
  }
  if (fabs(dx) > p->f_scale * w) dx = (dx < 0) ? -p->f_scale * w : p->f_scale * w;
  double x_left = w, f_try = f;
  int iter = 0;
  while ((f_try * f >= 0) && (iter++ < p->max_iter)) {
    x_left = w;
    f_try = f;
    w -= dx;
    eval_ngb(cl, w, p, &f, &dx, &cnt); (*nevals)++;
    if (fabs(dx) < p->rel_err * w) {
      *xl_out = w - 0.5 * fabs(dx); *xr_out = w + 0.5 * fabs(dx); *cnt_out = cnt;
      return;
    }
    if (fabs(dx) > p->f_scale * w) dx = (dx < 0) ? -p->f_scale * w : p->f_scale * w;
  }
  if (x_left < w) { *xl_out = x_left; *xr_out = w; }
  else { *xl_out = w; *xr_out = x_left; }
  *cnt_out = cnt;
}

/* solve_range, dev_solve_range.cu:137-172 */
static double solve_range_one(cand_list *cl, double w, const orc_params *p, int *nevals) {
  double rx, ry, rz;
  bracket_root(cl, w, p, &rx, &ry, &rz, nevals);
  w = 0.5 * (rx + ry);
  double dx = 0, f, cnt;
  if (fabs(rx - ry) > p->rel_err * w) {
    int iter = 0, keep = 1;
    while (keep && (iter++ < p->max_iter)) {
      w -= dx;
      if ((w - ry) * (w - rx) >= 0) {
        dx = 0.5 * (ry - rx);
        w = 0.5 * (rx + ry);
      }
      eval_ngb(cl, w, p, &f, &dx, &cnt); (*nevals)++;
      if (f < 0) rx = w;
      else ry = w;
      keep = fabs(dx) > p->rel_err * w;
    }
  }
  return w;
}

/* dev_solve_range kernel, dev_solve_range.cu:174-189, for targets tgt[0..nt)
 * (NULL: every particle, t = i): range_out[t] <- the solution started from
 * range_in[i], over all n particles as candidates (ascending index), for every
 * target with range > 0.  n_ngb[t] is the hard count at the final range. */
static void solve_targets(int nt, const int *tgt, int n, const double *x, const double *y, const double *z,
                          const double *range_in, double *range_out, int *n_ngb, int *nevals_out,
                          const orc_params *p) {
  if (n <= 0 || nt <= 0) return;
  double cell = 0;
  for (int i = 0; i < n; i++) cell += range_in[i];
  cell = cell / n;
  if (!(cell > 0)) cell = 1;
  orc_grid g;
  grid_build(&g, n, x, y, z, cell);
#pragma omp parallel
  {
    cand_list cl;
    memset(&cl, 0, sizeof(cl));
    cl.g = &g; cl.x = x; cl.y = y; cl.z = z;
#pragma omp for schedule(dynamic, 64)
    for (int t = 0; t < nt; t++) {
      const int i = tgt ? tgt[t] : t;
      int ne = 0;
      double w = range_in[i];
      if (w > 0) {
        cl.xi = x[i]; cl.yi = y[i]; cl.zi = z[i];
        cl.nc = -1; cl.R = -1;
        w = solve_range_one(&cl, w, p, &ne);
        double f, dx, cnt;
        cand_ensure(&cl, w);
        compute_ngb(cl.d2, cl.nc, w, p, &f, &dx, &cnt);
        n_ngb[t] = (int)cnt;
      } else {
        w = 0;
        n_ngb[t] = 0;
      }
      range_out[t] = w;
      if (nevals_out) nevals_out[t] = ne;
    }
    free(cl.buf);
    free(cl.d2);
  }
  grid_free(&g);
}

/* every particle, range updated in place */
void orc_solve_range(int n, const double *x, const double *y, const double *z, double *range,
                     int *n_ngb, int *nevals_out, const orc_params *p) {
  solve_targets(n, NULL, n, x, y, z, range, range, n_ngb, nevals_out, p);
}

/* a sample of targets (the full-size parity checks): range_out, n_ngb and
 * nevals_out have nt entries */
void orc_solve_range_tgt(int nt, const int *tgt, int n, const double *x, const double *y, const double *z,
                         const double *range0, double *range_out, int *n_ngb, int *nevals_out,
                         const orc_params *p) {
  solve_targets(nt, tgt, n, x, y, z, range0, range_out, n_ngb, nevals_out, p);
}

/* ------------------------------------------------------------------ */
/* find_ngb: dev_find_ngb.cu:13-87 (exact set, ascending j)              */
/* counts[i] = #{j : ds2 < range_i^2}; if list != NULL, writes CSR lists   */
/* at offsets[i] (offsets has n+1 entries and is filled here).            */
/* ------------------------------------------------------------------ */
long long orc_find_ngb(int n, const double *x, const double *y, const double *z, const double *range,
                       int *counts, long long *offsets, int *list) {
  if (n <= 0) { if (offsets) offsets[0] = 0; return 0; }
  double cell = 0;
  for (int i = 0; i < n; i++) cell += range[i];
  cell = cell / n;
  if (!(cell > 0)) cell = 1;
  orc_grid g;
  grid_build(&g, n, x, y, z, cell);
  if (!list) {
#pragma omp parallel
    {
      int cap = 0, *buf = NULL;
      double *db = NULL;
#pragma omp for schedule(dynamic, 64)
      for (int i = 0; i < n; i++)
        counts[i] = range[i] > 0 ? grid_query(&g, x, y, z, x[i], y[i], z[i], range[i], &buf, &cap, &db) : 0;
      free(buf); free(db);
    }
    long long tot = 0;
    for (int i = 0; i < n; i++) { if (offsets) offsets[i] = tot; tot += counts[i]; }
    if (offsets) offsets[n] = tot;
    grid_free(&g);
    return tot;
  }
#pragma omp parallel
  {
    int cap = 0, *buf = NULL;
    double *db = NULL;
#pragma omp for schedule(dynamic, 64)
    for (int i = 0; i < n; i++) {
      int c = range[i] > 0 ? grid_query(&g, x, y, z, x[i], y[i], z[i], range[i], &buf, &cap, &db) : 0;
      counts[i] = c;
      memcpy(list + offsets[i], buf, sizeof(int) * c);
    }
    free(buf); free(db);
  }
  grid_free(&g);
  return offsets[n];
}

/* find_ngb for targets tgt[0..nt) at ranges range_t[t] (exact sets over all n
 * particles, ascending index).  Same two-call protocol as orc_find_ngb:
 * list == NULL fills counts and offsets (nt + 1 entries). */
long long orc_find_ngb_tgt(int nt, const int *tgt, int n, const double *x, const double *y, const double *z,
                           const double *range_t, int *counts, long long *offsets, int *list) {
  if (n <= 0 || nt <= 0) { if (offsets) offsets[0] = 0; return 0; }
  double cell = 0;
  for (int t = 0; t < nt; t++) cell += range_t[t];
  cell = cell / nt;
  if (!(cell > 0)) cell = 1;
  orc_grid g;
  grid_build(&g, n, x, y, z, cell);
#pragma omp parallel
  {
    int cap = 0, *buf = NULL;
    double *db = NULL;
#pragma omp for schedule(dynamic, 16)
    for (int t = 0; t < nt; t++) {
      const int i = tgt[t];
      int c = range_t[t] > 0 ? grid_query(&g, x, y, z, x[i], y[i], z[i], range_t[t], &buf, &cap, &db) : 0;
      counts[t] = c;
      if (list) memcpy(list + offsets[t], buf, sizeof(int) * c);
    }
    free(buf); free(db);
  }
  grid_free(&g);
  if (!list) {
    long long tot = 0;
    for (int t = 0; t < nt; t++) { offsets[t] = tot; tot += counts[t]; }
    offsets[nt] = tot;
  }
  return offsets[nt];
}

/* ------------------------------------------------------------------ */
/* Density loop: dev_density_loop.cu:29-86                              */
/* ------------------------------------------------------------------ */
/* targets tgt[0..nt) (NULL: every particle, t = i); list t at offsets[t],
 * outputs at t */
static void density_targets(int nt, const int *tgt, const double *x, const double *y, const double *z,
                            const double *range, const double *vx, const double *vy, const double *vz,
                            const double *m, const long long *offsets, const int *list,
                            double *rho, double *divv, double *curlv, double *omega, double *psi) {
#pragma omp parallel for schedule(dynamic, 64)
  for (int t = 0; t < nt; t++) {
    const int i = tgt ? tgt[t] : t;
    double dens = 0, om = 0, ps = 0, sdig = 0, div = 0, cx = 0, cy = 0, cz = 0;
    double w = range[i];
    for (long long k = offsets[t]; k < offsets[t + 1]; k++) {
      int j = list[k];
      double dx = x[i] - x[j], dy = y[i] - y[j], dz = z[i] - z[j];
      double u = 2 * sqrt(ds2_of(dx, dy, dz)) / w;
      dens += m[j] * orc_w(u);
      om += m[j] * orc_dwdh(u);
      ps += m[j] * orc_dphidh(u);
      sdig -= orc_digdh(u);
      double dvx = vx[i] - vx[j], dvy = vy[i] - vy[j], dvz = vz[i] - vz[j];
      double wt = m[j] * orc_dw(u);
      div += wt * (dx * dvx + dy * dvy + dz * dvz);
      cx += wt * (dy * dvz - dz * dvy);
      cy += wt * (dz * dvx - dx * dvz);
      cz += wt * (dx * dvy - dy * dvx);
    }
    double h = 0.5 * w;
    if (w > 0 && offsets[t + 1] > offsets[t]) {
      double h3 = h * h * h, h5 = h3 * h * h;
      if (sdig != 0) {
        om *= 1.0 / h3 / sdig;
        ps *= 1.0 / h / sdig;
      } else {
        om = ps = 0;
      }
      dens *= 1.0 / h3;
      div *= 1.0 / dens / h5;
      double c = sqrt(cx * cx + cy * cy + cz * cz) / dens / h5;
      rho[t] = dens; divv[t] = div; curlv[t] = c; omega[t] = om; psi[t] = ps;
    } else {
      rho[t] = 0; divv[t] = 0; curlv[t] = 0; omega[t] = 0; psi[t] = 0;
    }
  }
}

void orc_density(int n, const double *x, const double *y, const double *z, const double *range,
                 const double *vx, const double *vy, const double *vz, const double *m,
                 const long long *offsets, const int *list,
                 double *rho, double *divv, double *curlv, double *omega, double *psi) {
  density_targets(n, NULL, x, y, z, range, vx, vy, vz, m, offsets, list, rho, divv, curlv, omega, psi);
}

/* a sample of targets: lists and outputs indexed by t (orc_find_ngb_tgt's CSR) */
void orc_density_tgt(int nt, const int *tgt, const double *x, const double *y, const double *z,
                     const double *range, const double *vx, const double *vy, const double *vz, const double *m,
                     const long long *offsets, const int *list,
                     double *rho, double *divv, double *curlv, double *omega, double *psi) {
  density_targets(nt, tgt, x, y, z, range, vx, vy, vz, m, offsets, list, rho, divv, curlv, omega, psi);
}

/* ------------------------------------------------------------------ */
/* EOS: dev_compute_pressure.cu:3-111                                   */
/* ------------------------------------------------------------------ */
#define ORC_DENSITY_UNIT 5.89994031541978
#define ORC_ENERGY_UNIT 1.90698842928778e+15
#define ORC_PRESSURE_UNIT 1.1251117914994e+16
#define ORC_AMU 1.66054e-24
#define ORC_BOLTZMANN 1.380658e-16
#define ORC_RAD_CONST 7.56591414984829e-15

/* Positive root of x^4 + q x + r = 0 (q > 0, r < 0): the closed form of
 * dev_compute_pressure.cu:3-49 (Ferrari / resolvent cubic), then Newton
 * polish on the quartic, safeguarded from the upper bound min(-r/q, (-r)^1/4). */
double orc_quartic_root(double q, double r) {
  double kh = 0.5 * 0.125 * q * q;
  double disc = kh * kh - r * r * r / 27.0;
  double s = sqrt(disc);
  double p1 = kh + s, p2 = kh - s;
  double y = cbrt(p1) - cbrt(fabs(p2));
  double b2 = sqrt(2.0 * y);
  double c2 = y - 0.5 * q / b2;
  double x = 0.5 * (sqrt(b2 * b2 - 4 * c2) - b2);
  if (p1 == -p2) x = pow(-r - q * pow(-r - q * pow(-r, 0.25), 0.25), 0.25);
  if (p2 > 0) x = -(r + r * r * r * r / (q * q * q * q)) / q;
  double ub = -r / q, ub2 = pow(-r, 0.25);
  if (ub2 < ub) ub = ub2;
  if (!(x > 0) || !(x <= ub) || !isfinite(x)) x = ub;
  for (int it = 0; it < 8; it++) {
    double x3 = x * x * x;
    double f = x3 * x + q * x + r;
    double fp = 4 * x3 + q;
    double xn = x - f / fp;
    if (!(xn > 0)) xn = 0.5 * x;
    if (xn == x) break;
    x = xn;
  }
  return x;
}

/* get_pressure, dev_compute_pressure.cu:83-96; inputs in code units */
double orc_pressure_one(double rho, double u, double mu, const orc_params *p) {
  if (p->eos_mode == 0) return (p->gamma - 1) * rho * u;
  if (!(rho > 0) || !(mu > 0)) return 0;
  double density = rho * ORC_DENSITY_UNIT;
  double energy = u * ORC_ENERGY_UNIT;
  double mean_mu = mu * ORC_AMU;
  double tb = 1.0e6;
  double r = -density * (energy / (tb * tb)) / (ORC_RAD_CONST * tb * tb);
  double q = (ORC_BOLTZMANN / ORC_RAD_CONST) / (p->gamma - 1) * density / (((mean_mu * tb) * tb) * tb);
  double T = tb * orc_quartic_root(q, r);
  double pg = density * ((ORC_BOLTZMANN * T) / mean_mu);
  double pr = (((ORC_RAD_CONST / 3.0 * T) * T) * T) * T;
  return (pg + pr) / ORC_PRESSURE_UNIT;
}

void orc_pressure(int n, const double *rho, const double *u, const double *mu, double *P, const orc_params *p) {
#pragma omp parallel for
  for (int i = 0; i < n; i++) P[i] = orc_pressure_one(rho[i], u[i], mu[i], p);
}

/* ------------------------------------------------------------------ */
/* Artificial viscosity: dev_art_visc.cu:8-32                            */
/* ------------------------------------------------------------------ */
static void art_visc(double range_i, double range_j, double ds, double drdv,
                     double rho_i, double P_i, double div_i, double curl_i,
                     double rho_j, double P_j, double div_j, double curl_j,
                     const orc_params *p, double *visc, double *vsig) {
  double ci = sqrt(p->gamma * P_i / rho_i);
  double cj = sqrt(p->gamma * P_j / rho_j);
  double av = 0, vs = ci + cj;
  if (drdv < 0) {
    vs -= p->av_beta * drdv / ds;
    av = drdv / ((ci + cj) * ds);
    double bi = fabs(div_i) / (fabs(div_i) + curl_i + 0.0001 * ci / (0.5 * range_i));
    double bj = fabs(div_j) / (fabs(div_j) + curl_j + 0.0001 * cj / (0.5 * range_j));
    av *= (bi + bj);
    av = (P_i / (rho_i * rho_i) + P_j / (rho_j * rho_j)) * (-p->av_alpha * av + p->av_beta * av * av);
  }
  *visc = av;
  *vsig = vs;
}

/* ------------------------------------------------------------------ */
/* Hydro derivatives: dev_hydro_dots.cu:25-113 (i-side) plus the j-side  */
/* scatter of sph_accelerations.cpp:106-114 (add_ngb_acc).               */
/* ngb_acc (optional, same layout as list) receives m_i * acc per pair.   */
/* ------------------------------------------------------------------ */
void orc_hydro(int n, const double *x, const double *y, const double *z, const double *range,
               const double *vx, const double *vy, const double *vz, const double *m,
               const double *rho, const double *P, const double *divv, const double *curlv,
               const double *omega, const double *psi,
               const long long *offsets, const int *list,
               double *ax, double *ay, double *az, double *du, double *vsig, double *ngb_acc,
               const orc_params *p) {
  double *nacc = ngb_acc;
  if (!nacc) nacc = (double *)malloc(sizeof(double) * (offsets[n] > 0 ? offsets[n] : 1));
#pragma omp parallel for schedule(dynamic, 64)
  for (int i = 0; i < n; i++) {
    double axi = 0, ayi = 0, azi = 0, udot = 0, vmax = 0;
    double hi = 0.5 * range[i];
    double prho2 = (rho[i] > 0) ? P[i] / (rho[i] * rho[i]) : 0;
    double h2 = hi * hi, h5 = h2 * h2 * hi;
    double psi_i = p->use_psi ? psi[i] : 0;
    for (long long k = offsets[i]; k < offsets[i + 1]; k++) {
      int j = list[k];
      double dx = x[i] - x[j], dy = y[i] - y[j], dz = z[i] - z[j];
      double dvx = vx[i] - vx[j], dvy = vy[i] - vy[j], dvz = vz[i] - vz[j];
      double ds = sqrt(ds2_of(dx, dy, dz));
      double u = ds / hi;
      double drdv = dx * dvx + dy * dvy + dz * dvz;
      double visc, vs;
      art_visc(range[i], range[j], ds, drdv, rho[i], P[i], divv[i], curlv[i], rho[j], P[j], divv[j],
               curlv[j], p, &visc, &vs);
      if (vs > vmax) vmax = vs;
      double dwu = orc_dw(u), digu = orc_dig(u);
      double acc = (prho2 + 0.5 * visc) * dwu / h5;
      acc -= (prho2 * omega[i] + 0.5 * psi_i) / m[j] * digu / h2;
      axi -= m[j] * acc * dx;
      ayi -= m[j] * acc * dy;
      azi -= m[j] * acc * dz;
      nacc[k] = m[i] * acc;
      double ud = m[j] * (prho2 + 0.5 * visc) * dwu / h5;
      ud -= prho2 * omega[i] * digu / h2;
      udot += ud * drdv;
    }
    ax[i] = axi; ay[i] = ayi; az[i] = azi; du[i] = udot; vsig[i] = vmax;
  }
  /* j-side, sph_accelerations.cpp:106-114: dots_j += ngb_acc * (x_i - x_j).
   * Serial in ascending i for a deterministic sum. */
  for (int i = 0; i < n; i++) {
    for (long long k = offsets[i]; k < offsets[i + 1]; k++) {
      int j = list[k];
      double a = nacc[k];
      ax[j] += a * (x[i] - x[j]);
      ay[j] += a * (y[i] - y[j]);
      az[j] += a * (z[i] - z[j]);
    }
  }
  if (!ngb_acc) free(nacc);
}

/* orc_hydro's result for targets tgt[0..nt) over the whole state, each pair
 * found by scanning all n particles in ascending index:
 *   i-side, dev_hydro_dots.cu:25-84: every j with ds2 < range_i^2 (i's own
 *     list, in list order), giving a_i, du_i and vsig_i;
 *   j-side, sph_accelerations.cpp:106-114: every j with ds2 < range_j^2 (i is
 *     in j's list), adding m_j acc_ji (x_j - x_i), acc_ji evaluated with j as
 *     the list owner exactly as the i-side loop does for its own pairs.
 * The per-particle inputs (range, rho, P, div v, curl v, omega, psi) of all n
 * are taken as given: this checks the hydro loop on a sample of a state whose
 * per-particle fields are checked separately. */
void orc_hydro_tgt(int nt, const int *tgt, int n, const double *x, const double *y, const double *z,
                   const double *range, const double *vx, const double *vy, const double *vz, const double *m,
                   const double *rho, const double *P, const double *divv, const double *curlv,
                   const double *omega, const double *psi,
                   double *ax, double *ay, double *az, double *du, double *vsig, const orc_params *p) {
#pragma omp parallel for schedule(dynamic, 4)
  for (int t = 0; t < nt; t++) {
    const int i = tgt[t];
    double axi = 0, ayi = 0, azi = 0, udot = 0, vmax = 0;
    double sx = 0, sy = 0, sz = 0; /* j-side, summed apart and added at the end */
    const double hi = 0.5 * range[i];
    const double prho2 = (rho[i] > 0) ? P[i] / (rho[i] * rho[i]) : 0;
    const double h2 = hi * hi, h5 = h2 * h2 * hi;
    const double psi_i = p->use_psi ? psi[i] : 0;
    const double ri2 = range[i] * range[i];
    for (int j = 0; j < n; j++) {
      const double dx = x[i] - x[j], dy = y[i] - y[j], dz = z[i] - z[j];
      const double d2 = ds2_of(dx, dy, dz);
      const int own = d2 < ri2, other = d2 < range[j] * range[j];
      if (!own && !other) continue;
      const double dvx = vx[i] - vx[j], dvy = vy[i] - vy[j], dvz = vz[i] - vz[j];
      const double ds = sqrt(d2);
      const double drdv = dx * dvx + dy * dvy + dz * dvz;
      if (own) {
        double visc, vs;
        art_visc(range[i], range[j], ds, drdv, rho[i], P[i], divv[i], curlv[i], rho[j], P[j], divv[j],
                 curlv[j], p, &visc, &vs);
        if (vs > vmax) vmax = vs;
        const double u = ds / hi;
        const double dwu = orc_dw(u), digu = orc_dig(u);
        double acc = (prho2 + 0.5 * visc) * dwu / h5;
        acc -= (prho2 * omega[i] + 0.5 * psi_i) / m[j] * digu / h2;
        axi -= m[j] * acc * dx;
        ayi -= m[j] * acc * dy;
        azi -= m[j] * acc * dz;
        double ud = m[j] * (prho2 + 0.5 * visc) * dwu / h5;
        ud -= prho2 * omega[i] * digu / h2;
        udot += ud * drdv;
      }
      if (other) {
        /* the pair (j, i) of j's list: the same expressions with j as owner */
        const double ex = x[j] - x[i], ey = y[j] - y[i], ez = z[j] - z[i];
        const double evx = vx[j] - vx[i], evy = vy[j] - vy[i], evz = vz[j] - vz[i];
        const double eds = sqrt(ds2_of(ex, ey, ez));
        const double edrdv = ex * evx + ey * evy + ez * evz;
        const double hj = 0.5 * range[j];
        const double prho2j = (rho[j] > 0) ? P[j] / (rho[j] * rho[j]) : 0;
        const double hj2 = hj * hj, hj5 = hj2 * hj2 * hj;
        const double psi_j = p->use_psi ? psi[j] : 0;
        double visc, vs;
        art_visc(range[j], range[i], eds, edrdv, rho[j], P[j], divv[j], curlv[j], rho[i], P[i], divv[i],
                 curlv[i], p, &visc, &vs);
        const double u = eds / hj;
        double acc = (prho2j + 0.5 * visc) * orc_dw(u) / hj5;
        acc -= (prho2j * omega[j] + 0.5 * psi_j) / m[i] * orc_dig(u) / hj2;
        const double a = m[j] * acc;
        sx += a * ex;
        sy += a * ey;
        sz += a * ez;
      }
    }
    ax[t] = axi + sx; ay[t] = ayi + sy; az[t] = azi + sz; du[t] = udot; vsig[t] = vmax;
  }
}

/* ------------------------------------------------------------------ */
/* Gravity: bodyBodyInteraction, sph_grav_kernel.cu:14-111 (spline      */
/* softening at range_i / range_j with half contributions) and Plummer.  */
/* Computes for targets tgt[0..nt) (NULL = all) against all n sources.    */
/* ------------------------------------------------------------------ */
static inline void spline_g(double u, double u2, double *gacc, double *gpot) {
  /* sph_grav_kernel.cu:53-61 polynomials of the spline-softened 1/r^2 and 1/r */
  double u3 = u2 * u;
  if (u < 0.5) {
    *gacc = (10.666666666667 + u2 * (32.0 * u - 38.4));
    *gpot = -2.8 + u2 * (5.333333333333 + u2 * (6.4 * u - 9.6));
  } else {
    *gacc = (21.333333333333 - 48.0 * u + 38.4 * u2 - 10.666666666667 * u3 - 0.066666666667 / u3);
    *gpot = -3.2 + 0.066666666667 / u + u2 * (10.666666666667 + u * (-16.0 + u * (9.6 - 2.133333333333 * u)));
  }
}

/* the sources [jlo, jhi) on targets tgt[0..nt) (NULL: every particle) */
static void gravity_sources(int nt, const int *tgt, int n, int jlo, int jhi, const double *x, const double *y,
                            const double *z, const double *m, const double *range, double *gx, double *gy,
                            double *gz, double *phi, const orc_params *p) {
  int ntot = tgt ? nt : n;
  double G = p->G;
#pragma omp parallel for schedule(dynamic, 16)
  for (int t = 0; t < ntot; t++) {
    int i = tgt ? tgt[t] : t;
    double a0 = 0, a1 = 0, a2 = 0, a3 = 0;
    double xi = x[i], yi = y[i], zi = z[i];
    if (p->soft_mode == 1) {
      double e2 = p->eps * p->eps;
      for (int j = jlo; j < jhi; j++) {
        double dx = xi - x[j], dy = yi - y[j], dz = zi - z[j];
        double r2 = dx * dx + dy * dy + dz * dz + e2;
        double inv = 1.0 / sqrt(r2);
        double s = m[j] * inv;
        double s3 = s * inv * inv;
        a0 -= dx * s3; a1 -= dy * s3; a2 -= dz * s3; a3 -= s;
      }
    } else {
      double hi2 = range[i] * range[i];
      for (int j = jlo; j < jhi; j++) {
        double dx = xi - x[j], dy = yi - y[j], dz = zi - z[j];
        double r2 = dx * dx + dy * dy + dz * dz;
        double hj2 = range[j] * range[j];
        double mj = m[j];
        if (r2 >= hi2 && r2 >= hj2) {
          if (r2 > 0) {
            double inv = 1.0 / sqrt(r2);
            double s3 = mj * inv * inv * inv;
            a0 -= dx * s3; a1 -= dy * s3; a2 -= dz * s3; a3 -= mj * inv;
          }
          continue;
        }
        double inv = r2 > 0 ? 1.0 / sqrt(r2) : 0;
        double s3h = 0.5 * mj * inv * inv * inv;
        if (r2 < hi2) {
          double u2 = r2 / hi2, h = sqrt(hi2), u = sqrt(u2), ga, gp;
          spline_g(u, u2, &ga, &gp);
          ga = 0.5 * mj * ga / (hi2 * h);
          a0 -= dx * ga; a1 -= dy * ga; a2 -= dz * ga;
          a3 += mj * gp / h;
        } else {
          a0 -= dx * s3h; a1 -= dy * s3h; a2 -= dz * s3h; a3 -= mj * inv;
        }
        if (r2 < hj2) {
          double u2 = r2 / hj2, h = sqrt(hj2), u = sqrt(u2), ga, gp;
          spline_g(u, u2, &ga, &gp);
          ga = 0.5 * mj * ga / (hj2 * h);
          a0 -= dx * ga; a1 -= dy * ga; a2 -= dz * ga;
        } else {
          a0 -= dx * s3h; a1 -= dy * s3h; a2 -= dz * s3h;
        }
      }
    }
    gx[t] = G * a0; gy[t] = G * a1; gz[t] = G * a2; phi[t] = G * a3;
  }
}

void orc_gravity(int nt, const int *tgt, int n, const double *x, const double *y, const double *z,
                 const double *m, const double *range, double *gx, double *gy, double *gz, double *phi,
                 const orc_params *p) {
  gravity_sources(nt, tgt, n, 0, n, x, y, z, m, range, gx, gy, gz, phi, p);
}

/* the contribution of the sources [jlo, jhi) only (a shard's share of the
 * pairs, whose sum over the shards is orc_gravity's result) */
void orc_gravity_src(int nt, const int *tgt, int n, int jlo, int jhi, const double *x, const double *y,
                     const double *z, const double *m, const double *range, double *gx, double *gy, double *gz,
                     double *phi, const orc_params *p) {
  if (jlo < 0) jlo = 0;
  if (jhi > n) jhi = n;
  gravity_sources(nt, tgt, n, jlo, jhi, x, y, z, m, range, gx, gy, gz, phi, p);
}

/* ------------------------------------------------------------------ */
/* Morton keys + stable order (the GPU sort's oracle).                  */
/* 21 bits per dimension from positions quantised in the bounding cube. */
/* ------------------------------------------------------------------ */
static uint64_t spread3(uint32_t v) {
  uint64_t x = v & 0x1fffff;
  x = (x | (x << 32)) & 0x1f00000000ffffULL;
  x = (x | (x << 16)) & 0x1f0000ff0000ffULL;
  x = (x | (x << 8)) & 0x100f00f00f00f00fULL;
  x = (x | (x << 4)) & 0x10c30c30c30c30c3ULL;
  x = (x | (x << 2)) & 0x1249249249249249ULL;
  return x;
}

void orc_morton_keys(int n, const double *x, const double *y, const double *z, uint64_t *keys, double *box) {
  if (n <= 0) return;
  double lo[3] = {x[0], y[0], z[0]}, hi[3] = {x[0], y[0], z[0]};
  for (int i = 1; i < n; i++) {
    if (x[i] < lo[0]) lo[0] = x[i]; if (x[i] > hi[0]) hi[0] = x[i];
    if (y[i] < lo[1]) lo[1] = y[i]; if (y[i] > hi[1]) hi[1] = y[i];
    if (z[i] < lo[2]) lo[2] = z[i]; if (z[i] > hi[2]) hi[2] = z[i];
  }
  double size = hi[0] - lo[0];
  if (hi[1] - lo[1] > size) size = hi[1] - lo[1];
  if (hi[2] - lo[2] > size) size = hi[2] - lo[2];
  double scale = size > 0 ? 2097152.0 / size : 0.0;
  if (box) { box[0] = lo[0]; box[1] = lo[1]; box[2] = lo[2]; box[3] = scale; }
  for (int i = 0; i < n; i++) {
    double c[3] = {(x[i] - lo[0]) * scale, (y[i] - lo[1]) * scale, (z[i] - lo[2]) * scale};
    uint32_t q[3];
    for (int d = 0; d < 3; d++) {
      double v = c[d];
      uint32_t k = v >= 2097151.0 ? 2097151u : (uint32_t)v;
      q[d] = k;
    }
    keys[i] = (spread3(q[0]) << 2) | (spread3(q[1]) << 1) | spread3(q[2]);
  }
}

/* ------------------------------------------------------------------ */
/* Peano-Hilbert keys: peano_hilbert_key sort_bodies.cpp:66-105 and the  */
/* float quantisation of CUDAsph::sort_bodies sort_bodies.cpp:121-160.   */
/* ------------------------------------------------------------------ */
/* The curve, level by level: the current cell is traversed in a frame f (a
   proper rotation of the cube) and a direction.  The world octant
   (bx, by, bz) has the frame-local octant f^T (2b - 1); its rank q along the
   curve is the inverse Gray code of the local (z, x, y) bits, and the key
   digit is q, or 7 - q in a reversed direction (sort_bodies.cpp:84-85).  The
   child's frame is f followed by TX[q] quarter turns about x and TY[q] about
   y (the rotations applied by rotxmap_table / rotymap_table,
   sort_bodies.cpp:87-101); the child's direction flips where REV[q] (the
   sense_table sign, :89). */
static const int PH_TX[8] = {3, 0, 0, 2, 2, 0, 0, 1};
static const int PH_TY[8] = {0, 1, 1, 2, 2, 3, 3, 0};
static const int PH_REV[8] = {1, 1, 1, 0, 0, 1, 1, 1};

static void mat3_mul(const int *a, const int *b, int *r) {
  int t[9];
  for (int i = 0; i < 3; i++)
    for (int j = 0; j < 3; j++) {
      int v = 0;
      for (int k = 0; k < 3; k++) v += a[i * 3 + k] * b[k * 3 + j];
      t[i * 3 + j] = v;
    }
  memcpy(r, t, sizeof(t));
}

uint64_t orc_peano_hilbert_key(int x, int y, int z, int bits) {
  static const int turn_x[9] = {1, 0, 0, 0, 0, 1, 0, -1, 0};
  static const int turn_y[9] = {0, 0, -1, 0, 1, 0, 1, 0, 0};
  int f[9] = {1, 0, 0, 0, 1, 0, 0, 0, 1};
  int rev = 0;
  uint64_t key = 0;
  for (int l = bits - 1; l >= 0; l--) {
    const int s[3] = {((x >> l) & 1) * 2 - 1, ((y >> l) & 1) * 2 - 1, ((z >> l) & 1) * 2 - 1};
    int loc[3] = {0, 0, 0};
    for (int i = 0; i < 3; i++)
      for (int j = 0; j < 3; j++) loc[i] += f[j * 3 + i] * s[j];
    int g = (((loc[2] + 1) / 2) << 2) | (((loc[0] + 1) / 2) << 1) | ((loc[1] + 1) / 2);
    int q = 0;
    for (; g; g >>= 1) q ^= g;
    key = (key << 3) | (uint64_t)(rev ? 7 - q : q);
    for (int k = 0; k < PH_TX[q]; k++) mat3_mul(f, turn_x, f);
    for (int k = 0; k < PH_TY[q]; k++) mat3_mul(f, turn_y, f);
    rev ^= PH_REV[q];
  }
  return key;
}

/* keys of positions as sort_bodies.cpp:121-160 computes them on its float4
   state: float bounding box, domain_fac = float(1.0 / size * 2^18), then
   (int)((pos - r_min) * domain_fac) in float, 18 bits per dimension.  box =
   {r_min.x, r_min.y, r_min.z, domain_fac}; a degenerate box (size 0) gives
   domain_fac = 0 (the reference divides by zero there). */
void orc_peano_keys(int n, const double *x, const double *y, const double *z, uint64_t *keys, double *box) {
  if (n <= 0) return;
  float lo[3] = {(float)x[0], (float)y[0], (float)z[0]}, hi[3] = {lo[0], lo[1], lo[2]};
  for (int i = 1; i < n; i++) {
    const float c[3] = {(float)x[i], (float)y[i], (float)z[i]};
    for (int d = 0; d < 3; d++) {
      if (c[d] < lo[d]) lo[d] = c[d];
      if (c[d] > hi[d]) hi[d] = c[d];
    }
  }
  float size = hi[2] - lo[2];
  if (hi[1] - lo[1] > size) size = hi[1] - lo[1];
  if (hi[0] - lo[0] > size) size = hi[0] - lo[0];
  const float fac = size > 0.f ? (float)(1.0 / size * (double)(1 << 18)) : 0.f;
  if (box) { box[0] = lo[0]; box[1] = lo[1]; box[2] = lo[2]; box[3] = fac; }
  for (int i = 0; i < n; i++) {
    const float dx = (float)x[i] - lo[0], dy = (float)y[i] - lo[1], dz = (float)z[i] - lo[2];
    const float sx = dx * fac, sy = dy * fac, sz = dz * fac;
    keys[i] = orc_peano_hilbert_key((int)sx, (int)sy, (int)sz, 18);
  }
}

typedef struct { uint64_t k; int i; } kv_t;
static int cmp_kv(const void *a, const void *b) {
  const kv_t *x = (const kv_t *)a, *y = (const kv_t *)b;
  if (x->k < y->k) return -1;
  if (x->k > y->k) return 1;
  return (x->i > y->i) - (x->i < y->i);
}
/* order[r] = index of the r-th smallest key (ties by index: a stable sort). */
void orc_sort_order(int n, const uint64_t *keys, int *order) {
  kv_t *a = (kv_t *)malloc(sizeof(kv_t) * (n > 0 ? n : 1));
  for (int i = 0; i < n; i++) { a[i].k = keys[i]; a[i].i = i; }
  qsort(a, n, sizeof(kv_t), cmp_kv);
  for (int i = 0; i < n; i++) order[i] = a[i].i;
  free(a);
}

/* ------------------------------------------------------------------ */
/* Whole step: step.cpp:13-147                                          */
/* ------------------------------------------------------------------ */
typedef struct {
  int n;
  double *x, *y, *z, *range;
  double *vx, *vy, *vz, *m;
  double *rho, *P, *u, *mu;
  double *divv, *curlv, *omega, *psi;
  double *ax, *ay, *az, *du;
  double *gx, *gy, *gz, *phi;
  double *vsig;
  int *n_ngb;
  double dt, time;
  int iteration;
  /* diagnostics of the last step (system_statistics.cpp:4-84, step.cpp:99-117) */
  double stats[16];
} orc_state;

/* compute_timestep.cpp:3-25 */
double orc_timestep(int n, const double *range, const double *vsig, const double *u, const double *du,
                    const orc_params *p) {
  double dt_min = 1.0e30;
  for (int i = 0; i < n; i++) {
    double dtv = p->cn1 * fabs(range[i] / vsig[i]);
    double dte = p->cn2 * fabs(u[i] / du[i]);
    double d = 1.0 / (1.0 / dtv + 1.0 / dte);
    if (d < dt_min) dt_min = d;
  }
  return dt_min;
}

/* system_statistics.cpp:4-84 plus the force/torque sums of step.cpp:99-117.
 * st: [0]W [1]T [2]U [3]E [4..6]J [7..9]Rcm [10..12]Vcm [13]Mtot [14..15]unused */
void orc_statistics(const orc_state *s, double *st) {
  int n = s->n;
  double W = 0, T = 0, U = 0, Jx = 0, Jy = 0, Jz = 0, M = 0, cx = 0, cy = 0, cz = 0, vx = 0, vy = 0, vz = 0;
  for (int i = 0; i < n; i++) {
    double m = s->m[i];
    M += m;
    cx += m * s->x[i]; cy += m * s->y[i]; cz += m * s->z[i];
    vx += m * s->vx[i]; vy += m * s->vy[i]; vz += m * s->vz[i];
    Jx += m * (s->y[i] * s->vz[i] - s->z[i] * s->vy[i]);
    Jy += m * (s->z[i] * s->vx[i] - s->x[i] * s->vz[i]);
    Jz += m * (s->x[i] * s->vy[i] - s->y[i] * s->vx[i]);
    U += m * s->u[i];
    W += 0.5 * m * s->phi[i];
    T += 0.5 * m * (s->vx[i] * s->vx[i] + s->vy[i] * s->vy[i] + s->vz[i] * s->vz[i]);
  }
  st[0] = W; st[1] = T; st[2] = U; st[3] = T + U + W;
  st[4] = Jx; st[5] = Jy; st[6] = Jz;
  st[7] = M > 0 ? cx / M : 0; st[8] = M > 0 ? cy / M : 0; st[9] = M > 0 ? cz / M : 0;
  st[10] = M > 0 ? vx / M : 0; st[11] = M > 0 ? vy / M : 0; st[12] = M > 0 ? vz / M : 0;
  st[13] = M;
}

/* One full step.  Returns 0 on success. */
int orc_step(orc_state *s, const orc_params *p) {
  int n = s->n;
  double dt = s->dt, dth = 0.5 * dt;
  double *ovx = (double *)malloc(sizeof(double) * n * 4);
  double *ovy = ovx + n, *ovz = ovy + n, *ou = ovz + n;
  s->iteration++;
  /* predictor, step.cpp:38-61 */
  for (int i = 0; i < n; i++) {
    s->x[i] += s->vx[i] * dt;
    s->y[i] += s->vy[i] * dt;
    s->z[i] += s->vz[i] * dt;
    ovx[i] = s->vx[i]; ovy[i] = s->vy[i]; ovz[i] = s->vz[i];
    s->vx[i] += s->ax[i] * dth;
    s->vy[i] += s->ay[i] * dth;
    s->vz[i] += s->az[i] * dth;
    ou[i] = s->u[i];
    s->u[i] += s->du[i] * dth;
  }
  /* sph_accelerations, sph_accelerations.cpp:3-121 */
  orc_solve_range(n, s->x, s->y, s->z, s->range, s->n_ngb, NULL, p);
  long long *off = (long long *)malloc(sizeof(long long) * (n + 1));
  int *cnt = (int *)malloc(sizeof(int) * n);
  long long tot = orc_find_ngb(n, s->x, s->y, s->z, s->range, cnt, off, NULL);
  int *list = (int *)malloc(sizeof(int) * (tot > 0 ? tot : 1));
  orc_find_ngb(n, s->x, s->y, s->z, s->range, cnt, off, list);
  for (int i = 0; i < n; i++) s->n_ngb[i] = cnt[i];
  orc_density(n, s->x, s->y, s->z, s->range, s->vx, s->vy, s->vz, s->m, off, list, s->rho, s->divv, s->curlv,
              s->omega, s->psi);
  orc_pressure(n, s->rho, s->u, s->mu, s->P, p);
  orc_hydro(n, s->x, s->y, s->z, s->range, s->vx, s->vy, s->vz, s->m, s->rho, s->P, s->divv, s->curlv,
            s->omega, s->psi, off, list, s->ax, s->ay, s->az, s->du, s->vsig, NULL, p);
  /* CUDA_gravity + add, step.cpp:96-103 */
  orc_gravity(0, NULL, n, s->x, s->y, s->z, s->m, s->range, s->gx, s->gy, s->gz, s->phi, p);
  for (int i = 0; i < n; i++) {
    s->ax[i] += s->gx[i];
    s->ay[i] += s->gy[i];
    s->az[i] += s->gz[i];
  }
  s->time += dt;
  orc_statistics(s, s->stats);
  /* compute_timestep + kick, step.cpp:128-134 */
  double dtn = orc_timestep(n, s->range, s->vsig, s->u, s->du, p);
  for (int i = 0; i < n; i++) {
    double f = 0.5 * dtn + dth;
    s->vx[i] = ovx[i] + s->ax[i] * f;
    s->vy[i] = ovy[i] + s->ay[i] * f;
    s->vz[i] = ovz[i] + s->az[i] * f;
    s->u[i] = ou[i] + s->du[i] * f;
  }
  s->dt = dtn;
  free(list); free(cnt); free(off); free(ovx);
  return 0;
}

int orc_num_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}
