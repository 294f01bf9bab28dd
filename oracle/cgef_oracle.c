/*
 * cgef_oracle.c -- CPU FP64 restatement of the coarse-graining hot path of
 * jbphyswx/CoarseGrainingEnergyFluxes.jl.  TEST INFRASTRUCTURE ONLY: this file is the
 * checker that the CUDA library is compared against, and the CPU baseline that bench.py
 * times.  Nothing in the product links it.
 *
 * Every function names the reference lines it restates.  Arrays are the reference's
 * column-major (Nx, Ny) layout, i.e. C row-major [ny][nx] with the x (longitude) index
 * fastest; indices are 0-based here (the reference's are 1-based).
 *
 * Geometry that the reference takes from the un-vendored FlowGeometries.jl package is
 * restated from the reference's own documentation:
 *   distance : great-circle, haversine form (src/Filtering.jl:264-265, docs/src/theory.md:304)
 *   area     : R^2 cos(phi) dlambda dphi        (docs/src/theory.md:307, CHANGELOG.md:553)
 *   frames   : east/north/up basis              (src/Diagnostics.jl:612-615)
 *   stencil  : 3-node, ReduceInRun at mask edges (src/Derivatives.jl:19-31, CHANGELOG.md:243-259)
 * Those conventions are not pinned by any reference test value ("parity unpinned").
 */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>
#ifdef _OPENMP
#include <omp.h>
#endif

#define ORC_CART 0
#define ORC_SPHERE 1
#define ORC_TOPHAT 0
#define ORC_GAUSSIAN 1
#define ORC_ZEROFILL 0
#define ORC_DEFORMABLE 1
#define ORC_ENGINE_BANDED 1
#define ORC_ENGINE_SEPARABLE 2
#define ORC_ENGINE_PREFIXSUM 3

/* Kernels.jl:307 */
static const double GAUSSIAN_TRUNCATION_TOL = 1e-10;
/* Filtering.jl:1633 (and every apply path): normalisation threshold */
static const double NORM_EPS = 1e-15;

typedef struct {
  int geometry;
  int nx, ny;
  double x0, dx, y0, dy; /* uniform axes, x_i = fma(i, dx, x0) */
  double R;
  int periodic_x, periodic_y;
  const uint8_t* mask; /* ny*nx, or NULL = all active */
} orc_grid;

static inline double gx_coord(const orc_grid* g, int i) { return fma((double)i, g->dx, g->x0); }
static inline double gy_coord(const orc_grid* g, int j) { return fma((double)j, g->dy, g->y0); }
static inline int is_active(const orc_grid* g, int i, int j) {
  return g->mask == NULL ? 1 : (g->mask[(int64_t)j * g->nx + i] != 0);
}
static inline int mod_n(int a, int n) { int r = a % n; return r < 0 ? r + n : r; }

/* ------------------------------------------------------------------------------------
 * Kernels (Kernels.jl:318-324 weights, :354-359 radii)
 * ------------------------------------------------------------------------------------ */
double orc_kernel_weight(int kernel, double alpha, double d, double ell) {
  if (kernel == ORC_TOPHAT) return d <= ell / 2.0 ? 1.0 : 0.0;
  double q = d / ell;
  return exp(-alpha * (q * q));
}

double orc_kernel_radius(int kernel, double alpha, double ell) {
  if (kernel == ORC_TOPHAT) return ell / 2.0;
  return ell * sqrt(-log(GAUSSIAN_TRUNCATION_TOL) / alpha);
}

/* Great-circle distance, haversine form; Cartesian Euclidean. */
double orc_distance(const orc_grid* g, double x1, double y1, double x2, double y2) {
  if (g->geometry == ORC_CART) {
    double a = x2 - x1, b = y2 - y1;
    return sqrt(a * a + b * b);
  }
  double sdp = sin((y2 - y1) / 2.0), sdl = sin((x2 - x1) / 2.0);
  double h = sdp * sdp + cos(y1) * cos(y2) * sdl * sdl;
  if (h > 1.0) h = 1.0;
  return 2.0 * g->R * asin(sqrt(h));
}

/* Cell measure: R^2 cos(phi) dlambda dphi on the sphere, dx dy on the plane. */
double orc_area(const orc_grid* g, int i, int j) {
  (void)i;
  if (g->geometry == ORC_CART) return g->dx * g->dy;
  return g->R * g->R * cos(gy_coord(g, j)) * g->dx * g->dy;
}

/* ------------------------------------------------------------------------------------
 * Banded footprint (Filtering.jl:636-732).  CSR over bands: band b owns entries
 * ptr[b]..ptr[b+1]-1 with offsets (di, dj) and weight w = kernel(d) * area(row).
 * Cartesian: one translation-invariant band; sphere: one band per latitude row.
 * ------------------------------------------------------------------------------------ */
typedef struct {
  int nbands;
  int64_t nentries;
  int* di;
  int* dj;
  double* w;
  int64_t* ptr;
} orc_footprint;

/* Longitude half-width (in cells) that certainly contains every column of row phi2 lying
 * within rad of (0, phi1): the acos bound plus a two-cell margin, capped at the ring.  Only
 * used to bound the candidate scan; inclusion is decided by the distance test itself, so
 * the entry set equals the reference's as long as this window covers the disk. */
static int sphere_row_window(const orc_grid* g, double phi1, double phi2, double rad, int cap) {
  double c1 = cos(phi1), c2 = cos(phi2);
  double num = cos(rad / g->R) - sin(phi1) * sin(phi2);
  double den = c1 * c2;
  if (den <= 0.0) return cap;
  double c = num / den;
  if (c <= -1.0) return cap;
  if (c > 1.0) return 2 < cap ? 2 : cap;
  double dl = acos(c);
  double w = floor(dl / fabs(g->dx)) + 2.0;
  if (w > (double)cap) return cap;
  return (int)w;
}

/* rows: NULL, or ny flags; bands of unflagged rows are left empty (the row-subset oracle, which
 * evaluates only the target rows a test compares). */
static void footprint_build(const orc_grid* g, int kernel, double alpha, double ell, orc_footprint* fp,
                            int fill, const uint8_t* rows) {
  double rad = orc_kernel_radius(kernel, alpha, ell);
  int64_t n = 0;
  if (g->geometry == ORC_CART) {
    /* Filtering.jl:654-674 */
    int di_lim = g->dx > 0 ? (int)ceil(rad / g->dx) : 0;
    int dj_lim = g->dy > 0 ? (int)ceil(rad / g->dy) : 0;
    double A = g->dx * g->dy;
    if (fill) fp->ptr[0] = 0;
    for (int ddj = -dj_lim; ddj <= dj_lim; ++ddj)
      for (int ddi = -di_lim; ddi <= di_lim; ++ddi) {
        double a = ddi * g->dx, b = ddj * g->dy;
        double d = sqrt(a * a + b * b);
        if (d <= rad) {
          if (fill) {
            fp->di[n] = ddi;
            fp->dj[n] = ddj;
            fp->w[n] = orc_kernel_weight(kernel, alpha, d, ell) * A;
          }
          ++n;
        }
      }
    if (fill) fp->ptr[1] = n;
    fp->nbands = 1;
    fp->nentries = n;
    return;
  }
  /* Filtering.jl:675-731 */
  int nx = g->nx, ny = g->ny;
  int dj_lim = g->dy > 0 ? (int)ceil(rad / (g->R * g->dy)) : 0;
  int half = nx / 2;
  if (fill) fp->ptr[0] = 0;
  for (int j = 0; j < ny; ++j) {
    if (rows && !rows[j]) {
      if (fill) fp->ptr[j + 1] = n;
      continue;
    }
    double phi = gy_coord(g, j);
    /* The band's window: capped at one turn (Filtering.jl:692), and asymmetric by one when it
     * closes the ring (Filtering.jl:711-713).  The band closes the ring when some row it
     * reaches needs the full half-turn. */
    int band_closed = 0;
    for (int ddj = -dj_lim; ddj <= dj_lim; ++ddj) {
      int jj = j + ddj;
      if (jj < 0 || jj >= ny) continue;
      if (sphere_row_window(g, phi, gy_coord(g, jj), rad, half) >= half) band_closed = 1;
    }
    for (int ddj = -dj_lim; ddj <= dj_lim; ++ddj) {
      int jj = j + ddj;
      if (jj < 0 || jj >= ny) continue;
      double phi2 = gy_coord(g, jj);
      double A = orc_area(g, 0, jj);
      int win = band_closed ? half : sphere_row_window(g, phi, phi2, rad, half);
      int lo = -win;
      int hi = (band_closed && 2 * half + 1 > nx) ? half - 1 : win;
      for (int ddi = lo; ddi <= hi; ++ddi) {
        double d = orc_distance(g, 0.0, phi, (double)ddi * g->dx, phi2);
        if (d <= rad) {
          if (fill) {
            fp->di[n] = ddi;
            fp->dj[n] = ddj;
            fp->w[n] = orc_kernel_weight(kernel, alpha, d, ell) * A;
          }
          ++n;
        }
      }
    }
    if (fill) fp->ptr[j + 1] = n;
  }
  fp->nbands = ny;
  fp->nentries = n;
}

/* Band-by-band apply for K fields sharing one traversal (Filtering.jl:2550-2598).  Inactive
 * targets are 0; ZeroFill keeps masked sources in the denominator, Deformable drops them. */
static void footprint_apply_row(const orc_grid* g, const orc_footprint* fp, int strategy, int K,
                                const double* const* fields, double* const* outs, int j, double* acc_ws,
                                double* acc_wn) {
  int nx = g->nx, ny = g->ny;
  int b = fp->nbands == 1 ? 0 : j;
  int64_t lo = fp->ptr[b], hi = fp->ptr[b + 1];
  for (int i = 0; i < nx; ++i) {
    int64_t o = (int64_t)j * nx + i;
    if (!is_active(g, i, j)) {
      for (int m = 0; m < K; ++m) outs[m][o] = 0.0;
      continue;
    }
    for (int m = 0; m < K; ++m) acc_ws[m] = acc_wn[m] = 0.0;
    for (int64_t k = lo; k < hi; ++k) {
      int jj = j + fp->dj[k];
      if (jj < 0 || jj >= ny) {
        if (!g->periodic_y) continue;
        jj = mod_n(jj, ny);
      }
      int ii = i + fp->di[k];
      if (ii < 0 || ii >= nx) {
        if (!g->periodic_x) continue;
        ii = mod_n(ii, nx);
      }
      int act = is_active(g, ii, jj);
      double w = fp->w[k];
      int64_t s = (int64_t)jj * nx + ii;
      if (strategy == ORC_ZEROFILL) {
        for (int m = 0; m < K; ++m) acc_wn[m] += w;
        if (act)
          for (int m = 0; m < K; ++m) acc_ws[m] += w * fields[m][s];
      } else if (act) {
        for (int m = 0; m < K; ++m) {
          acc_wn[m] += w;
          acc_ws[m] += w * fields[m][s];
        }
      }
    }
    for (int m = 0; m < K; ++m) outs[m][o] = acc_wn[m] > NORM_EPS ? acc_ws[m] / acc_wn[m] : 0.0;
  }
}

/* rows: NULL, or ny flags; unflagged rows are not evaluated and read 0. */
static void footprint_apply(const orc_grid* g, const orc_footprint* fp, int strategy, int K,
                            const double* const* fields, double* const* outs, int nthreads, const uint8_t* rows) {
#ifdef _OPENMP
  if (nthreads <= 0) nthreads = omp_get_max_threads();
#pragma omp parallel num_threads(nthreads)
  {
    double* acc = (double*)malloc(sizeof(double) * 2 * (K > 0 ? K : 1));
#pragma omp for schedule(dynamic, 1)
    for (int j = 0; j < g->ny; ++j) {
      if (rows && !rows[j]) {
        for (int m = 0; m < K; ++m) memset(outs[m] + (int64_t)j * g->nx, 0, sizeof(double) * g->nx);
        continue;
      }
      footprint_apply_row(g, fp, strategy, K, fields, outs, j, acc, acc + K);
    }
    free(acc);
  }
#else
  (void)nthreads;
  double* acc = (double*)malloc(sizeof(double) * 2 * (K > 0 ? K : 1));
  for (int j = 0; j < g->ny; ++j) {
    if (rows && !rows[j]) {
      for (int m = 0; m < K; ++m) memset(outs[m] + (int64_t)j * g->nx, 0, sizeof(double) * g->nx);
      continue;
    }
    footprint_apply_row(g, fp, strategy, K, fields, outs, j, acc, acc + K);
  }
  free(acc);
#endif
}

/* ------------------------------------------------------------------------------------
 * Separable Gaussian, Cartesian (Filtering.jl:1172-1191, 1211-1280, 1341-1349,
 * 1391-1463, 1472-1524).  Square truncation, lim = ceil(rad / step) per axis.
 * ------------------------------------------------------------------------------------ */
typedef struct {
  int di_lim, dj_lim;
  double* gx; /* 2*di_lim+1 */
  double* gy; /* 2*dj_lim+1 */
  double* px; /* nx, ZeroFill profiles (or NULL) */
  double* py; /* ny */
  double* invrenorm; /* ny*nx, Deformable on a masked grid (or NULL) */
} orc_separable;

static void sep_row_pass(const double* src, double* dst, const double* gxw, int lim, int periodic, int nx,
                         int ny) {
  for (int j = 0; j < ny; ++j) {
    const double* s = src + (int64_t)j * nx;
    double* d = dst + (int64_t)j * nx;
    for (int i = 0; i < nx; ++i) d[i] = 0.0;
    for (int ddi = -lim; ddi <= lim; ++ddi) {
      double w = gxw[ddi + lim];
      for (int i = 0; i < nx; ++i) {
        int ii = i + ddi;
        if (ii < 0 || ii >= nx) {
          if (!periodic) continue;
          ii = mod_n(ii, nx);
        }
        d[i] += w * s[ii];
      }
    }
  }
}

static void sep_col_pass(const double* src, double* dst, const double* gyw, int lim, int periodic, int nx,
                         int ny) {
  for (int j = 0; j < ny; ++j) {
    double* d = dst + (int64_t)j * nx;
    for (int i = 0; i < nx; ++i) d[i] = 0.0;
    for (int ddj = -lim; ddj <= lim; ++ddj) {
      int jj = j + ddj;
      if (jj < 0 || jj >= ny) {
        if (!periodic) continue;
        jj = mod_n(jj, ny);
      }
      double w = gyw[ddj + lim];
      const double* s = src + (int64_t)jj * nx;
      for (int i = 0; i < nx; ++i) d[i] += w * s[i];
    }
  }
}

static double* sep_profile(int lim, const double* gw, int n, int periodic) {
  double* p = (double*)malloc(sizeof(double) * n);
  for (int i = 0; i < n; ++i) {
    double s = 0.0;
    for (int dd = -lim; dd <= lim; ++dd) {
      int ii = i + dd;
      if ((ii >= 0 && ii < n) || periodic) s += gw[dd + lim];
    }
    p[i] = s;
  }
  return p;
}

static void separable_build(const orc_grid* g, double alpha, double ell, int strategy, orc_separable* sp) {
  double rad = orc_kernel_radius(ORC_GAUSSIAN, alpha, ell);
  sp->di_lim = g->dx > 0 ? (int)ceil(rad / g->dx) : 0;
  sp->dj_lim = g->dy > 0 ? (int)ceil(rad / g->dy) : 0;
  sp->gx = (double*)malloc(sizeof(double) * (2 * sp->di_lim + 1));
  sp->gy = (double*)malloc(sizeof(double) * (2 * sp->dj_lim + 1));
  for (int k = -sp->di_lim; k <= sp->di_lim; ++k)
    sp->gx[k + sp->di_lim] = orc_kernel_weight(ORC_GAUSSIAN, alpha, fabs((double)k * g->dx), ell);
  for (int k = -sp->dj_lim; k <= sp->dj_lim; ++k)
    sp->gy[k + sp->dj_lim] = orc_kernel_weight(ORC_GAUSSIAN, alpha, fabs((double)k * g->dy), ell);
  int nx = g->nx, ny = g->ny;
  int fully_active = 1;
  if (g->mask)
    for (int64_t k = 0; k < (int64_t)nx * ny; ++k)
      if (!g->mask[k]) { fully_active = 0; break; }
  sp->px = sp->py = sp->invrenorm = NULL;
  if (fully_active || strategy == ORC_ZEROFILL) {
    sp->px = sep_profile(sp->di_lim, sp->gx, nx, g->periodic_x);
    sp->py = sep_profile(sp->dj_lim, sp->gy, ny, g->periodic_y);
  } else {
    double* mf = (double*)malloc(sizeof(double) * nx * ny);
    double* tmp = (double*)malloc(sizeof(double) * nx * ny);
    double* den = (double*)malloc(sizeof(double) * nx * ny);
    for (int64_t k = 0; k < (int64_t)nx * ny; ++k) mf[k] = g->mask[k] ? 1.0 : 0.0;
    sep_row_pass(mf, tmp, sp->gx, sp->di_lim, g->periodic_x, nx, ny);
    sep_col_pass(tmp, den, sp->gy, sp->dj_lim, g->periodic_y, nx, ny);
    for (int64_t k = 0; k < (int64_t)nx * ny; ++k) den[k] = den[k] > NORM_EPS ? 1.0 / den[k] : 0.0;
    sp->invrenorm = den;
    free(mf);
    free(tmp);
  }
}

static void separable_apply(const orc_grid* g, const orc_separable* sp, const double* field, double* out) {
  int nx = g->nx, ny = g->ny;
  int64_t n = (int64_t)nx * ny;
  double* mi = (double*)malloc(sizeof(double) * n);
  double* rp = (double*)malloc(sizeof(double) * n);
  for (int64_t k = 0; k < n; ++k) mi[k] = (g->mask == NULL || g->mask[k]) ? field[k] : 0.0;
  sep_row_pass(mi, rp, sp->gx, sp->di_lim, g->periodic_x, nx, ny);
  sep_col_pass(rp, out, sp->gy, sp->dj_lim, g->periodic_y, nx, ny);
  if (sp->invrenorm) {
    for (int64_t k = 0; k < n; ++k) out[k] *= sp->invrenorm[k];
  } else {
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        double den = sp->px[i] * sp->py[j];
        int64_t o = (int64_t)j * nx + i;
        out[o] = den > NORM_EPS ? out[o] / den : 0.0;
      }
  }
  if (g->mask)
    for (int64_t k = 0; k < n; ++k)
      if (!g->mask[k]) out[k] = 0.0;
  free(mi);
  free(rp);
}

/* ------------------------------------------------------------------------------------
 * Prefix-sum exact top-hat (Filtering.jl:780-806, 833-907, 916-1097).
 * ------------------------------------------------------------------------------------ */
typedef struct {
  double rad;
  int dj_lim, nrep, ne, use_mask_den;
  double x_period, y_period;
  double* wx; /* nx */
  double* wy; /* ny */
  double* xe; /* ne */
  int* src; /* ne */
  double* prefix_wx; /* ne+1 */
  double* prefix_den; /* (ne+1)*ny or NULL */
} orc_prefix;

/* Connectivity.metric_band: longitude (axis-1) half-width of the support at row offset
 * y_t -> y_s, in axis-1 coordinate units; negative when the row is out of reach
 * (Filtering.jl:761-765, 1004-1005). */
double orc_metric_band(const orc_grid* g, double y_t, double y_s, double rad) {
  if (g->geometry == ORC_CART) {
    double dy = y_s - y_t;
    double r2 = rad * rad - dy * dy;
    return r2 < 0.0 ? -1.0 : sqrt(r2);
  }
  double c1 = cos(y_t), c2 = cos(y_s);
  double num = cos(rad / g->R) - sin(y_t) * sin(y_s);
  double den = c1 * c2;
  if (den <= 0.0) return num <= 0.0 ? M_PI : -1.0;
  double c = num / den;
  if (c > 1.0) return -1.0;
  if (c < -1.0) return M_PI;
  return acos(c);
}

static void prefix_build(const orc_grid* g, double ell, int strategy, orc_prefix* pp) {
  int nx = g->nx, ny = g->ny;
  pp->rad = orc_kernel_radius(ORC_TOPHAT, 0.0, ell);
  pp->x_period = (g->periodic_x && nx > 1) ? nx * g->dx : 0.0;
  pp->y_period = (g->periodic_y && ny > 1) ? ny * g->dy : 0.0;
  pp->wx = (double*)malloc(sizeof(double) * nx);
  pp->wy = (double*)malloc(sizeof(double) * ny);
  for (int i = 0; i < nx; ++i) pp->wx[i] = g->dx;
  for (int j = 0; j < ny; ++j)
    pp->wy[j] = g->geometry == ORC_CART ? g->dy : g->R * g->R * cos(gy_coord(g, j)) * g->dy;
  double dy_phys = g->geometry == ORC_CART ? g->dy : g->R * g->dy;
  int lim = (isfinite(dy_phys) && dy_phys > 0) ? (int)ceil(pp->rad / dy_phys) : 0;
  pp->dj_lim = lim < ny - 1 ? lim : ny - 1;
  pp->nrep = (g->periodic_x && nx > 1) ? 3 : 1;
  pp->ne = pp->nrep * nx;
  pp->xe = (double*)malloc(sizeof(double) * pp->ne);
  pp->src = (int*)malloc(sizeof(int) * pp->ne);
  for (int r = 0; r < pp->nrep; ++r)
    for (int t = 0; t < nx; ++t) {
      int k = r * nx + t;
      pp->xe[k] = gx_coord(g, t) + (pp->nrep == 3 ? (double)(r - 1) * pp->x_period : 0.0);
      pp->src[k] = t;
    }
  pp->prefix_wx = (double*)malloc(sizeof(double) * (pp->ne + 1));
  pp->prefix_wx[0] = 0.0;
  for (int k = 0; k < pp->ne; ++k) pp->prefix_wx[k + 1] = pp->prefix_wx[k] + pp->wx[pp->src[k]];
  int masked = 0;
  if (g->mask)
    for (int64_t k = 0; k < (int64_t)nx * ny; ++k)
      if (!g->mask[k]) { masked = 1; break; }
  pp->prefix_den = NULL;
  pp->use_mask_den = 0;
  if (strategy == ORC_DEFORMABLE && masked) {
    pp->prefix_den = (double*)malloc(sizeof(double) * (pp->ne + 1) * ny);
    for (int j = 0; j < ny; ++j) {
      double* P = pp->prefix_den + (int64_t)j * (pp->ne + 1);
      double acc = 0.0;
      P[0] = 0.0;
      for (int k = 0; k < pp->ne; ++k) {
        int i = pp->src[k];
        acc += is_active(g, i, j) ? pp->wx[i] : 0.0;
        P[k + 1] = acc;
      }
    }
    pp->use_mask_den = 1;
  }
}

static void prefix_apply(const orc_grid* g, const orc_prefix* pp, const double* field, double* out) {
  int nx = g->nx, ny = g->ny, ne = pp->ne;
  int64_t pitch = ne + 1;
  double* Pn = (double*)malloc(sizeof(double) * pitch * ny);
  double* den = (double*)malloc(sizeof(double) * (int64_t)nx * ny);
  /* prefixsum_fill_numerator_row! (Filtering.jl:894-907) */
  for (int j = 0; j < ny; ++j) {
    double* P = Pn + (int64_t)j * pitch;
    double acc = 0.0;
    P[0] = 0.0;
    for (int k = 0; k < ne; ++k) {
      int i = pp->src[k];
      acc += is_active(g, i, j) ? field[(int64_t)j * nx + i] * pp->wx[i] : 0.0;
      P[k + 1] = acc;
    }
  }
  const double* Pd = pp->prefix_den;
  const double* Pwx = pp->prefix_wx;
  int use_mask_den = pp->use_mask_den;
  int uniform_fast = !g->periodic_x && ne == nx && g->dx > 0;
  for (int j = 0; j < ny; ++j) {
    double y_t = gy_coord(g, j);
    double* o = out + (int64_t)j * nx;
    double* dn = den + (int64_t)j * nx;
    for (int i = 0; i < nx; ++i) o[i] = dn[i] = 0.0;
    int nb = 2 * pp->dj_lim + 1 < ny ? 2 * pp->dj_lim + 1 : ny;
    for (int b = 0; b < nb; ++b) {
      int jj_raw = j - pp->dj_lim + b;
      if (!(g->periodic_y || (jj_raw >= 0 && jj_raw < ny))) continue;
      int jj = mod_n(jj_raw, ny);
      double dyv = gy_coord(g, jj) - y_t;
      if (g->periodic_y && pp->y_period > 0.0) dyv -= pp->y_period * round(dyv / pp->y_period);
      double hw = orc_metric_band(g, y_t, y_t + dyv, pp->rad);
      if (hw < 0.0) continue;
      double wyj = pp->wy[jj];
      const double* Pr = Pn + (int64_t)jj * pitch;
      const double* Pdr = use_mask_den ? Pd + (int64_t)jj * pitch : NULL;
      if (g->periodic_x && ne > nx && 2.0 * hw >= pp->x_period) {
        double num_all = Pr[nx] - Pr[0];
        double den_all = use_mask_den ? (Pdr[nx] - Pdr[0]) : (Pwx[nx] - Pwx[0]);
        for (int i = 0; i < nx; ++i) {
          o[i] += wyj * num_all;
          dn[i] += wyj * den_all;
        }
      } else if (uniform_fast) {
        int w = 0;
        while ((w + 1) * g->dx <= hw) ++w;
        for (int i = 0; i < nx; ++i) {
          int lo = i - w < 0 ? 0 : i - w;          /* 0-based first index */
          int hi = i + w > nx - 1 ? nx - 1 : i + w; /* 0-based last index */
          o[i] += wyj * (Pr[hi + 1] - Pr[lo]);
          dn[i] += wyj * (use_mask_den ? (Pdr[hi + 1] - Pdr[lo]) : (Pwx[hi + 1] - Pwx[lo]));
        }
      } else {
        int lo = 0, hi = -1; /* 0-based two pointers over xe */
        for (int t = 0; t < nx; ++t) {
          int i = pp->src[t];
          double xc = gx_coord(g, i);
          double xlo = xc - hw, xhi = xc + hw;
          while (lo <= ne - 1 && pp->xe[lo] < xlo) ++lo;
          while (hi < ne - 1 && pp->xe[hi + 1] <= xhi) ++hi;
          if (hi >= lo) {
            o[i] += wyj * (Pr[hi + 1] - Pr[lo]);
            dn[i] += wyj * (use_mask_den ? (Pdr[hi + 1] - Pdr[lo]) : (Pwx[hi + 1] - Pwx[lo]));
          }
        }
      }
    }
    for (int i = 0; i < nx; ++i) o[i] = (is_active(g, i, j) && dn[i] > NORM_EPS) ? o[i] / dn[i] : 0.0;
  }
  free(Pn);
  free(den);
}

/* ------------------------------------------------------------------------------------
 * Plan: kernel x geometry dispatch (Filtering.jl:636-749, 1121-1141, 1533-1561):
 * Gaussian on Cartesian -> separable; top-hat anywhere -> prefix sum; else banded.
 * ------------------------------------------------------------------------------------ */
typedef struct {
  orc_grid g;
  int kernel, strategy, engine;
  double alpha, ell;
  orc_footprint fp;
  orc_separable sp;
  orc_prefix pp;
  uint8_t* mask_copy;
  uint8_t* rows; /* banded: NULL, or ny flags of the target rows evaluated (orc_plan_new_rows) */
} orc_plan;

int orc_default_engine(int geometry, int kernel) {
  if (kernel == ORC_TOPHAT) return ORC_ENGINE_PREFIXSUM;
  if (geometry == ORC_CART) return ORC_ENGINE_SEPARABLE;
  return ORC_ENGINE_BANDED;
}

/* rows: NULL (every target row), or ny flags: a banded plan then builds and evaluates only the
 * flagged target rows' bands, and every other row of a filter output reads 0.  compute_Pi!'s
 * strain at row j reads the filtered velocities of rows j-2..j+2, so its Pi is the full plan's
 * wherever those five rows are flagged.  This keeps footprints of thousands of kilometres on the
 * full 0.25-degree sphere within seconds of CPU time for the rows a test compares. */
orc_plan* orc_plan_new_rows(int geometry, int nx, int ny, double x0, double dx, double y0, double dy, double R,
                            int periodic_x, int periodic_y, const uint8_t* mask, int kernel, double alpha,
                            double ell, int strategy, int engine, const uint8_t* rows) {
  orc_plan* p = (orc_plan*)calloc(1, sizeof(orc_plan));
  if (rows) {
    p->rows = (uint8_t*)malloc((size_t)ny);
    memcpy(p->rows, rows, (size_t)ny);
  }
  p->g.geometry = geometry;
  p->g.nx = nx;
  p->g.ny = ny;
  p->g.x0 = x0;
  p->g.dx = dx;
  p->g.y0 = y0;
  p->g.dy = dy;
  p->g.R = R;
  p->g.periodic_x = periodic_x;
  p->g.periodic_y = periodic_y;
  if (mask) {
    p->mask_copy = (uint8_t*)malloc((size_t)nx * ny);
    memcpy(p->mask_copy, mask, (size_t)nx * ny);
  }
  p->g.mask = p->mask_copy;
  p->kernel = kernel;
  p->alpha = alpha;
  p->ell = ell;
  p->strategy = strategy;
  p->engine = engine > 0 ? engine : orc_default_engine(geometry, kernel);
  if (p->engine == ORC_ENGINE_BANDED) {
    footprint_build(&p->g, kernel, alpha, ell, &p->fp, 0, p->rows);
    p->fp.di = (int*)malloc(sizeof(int) * (p->fp.nentries + 1));
    p->fp.dj = (int*)malloc(sizeof(int) * (p->fp.nentries + 1));
    p->fp.w = (double*)malloc(sizeof(double) * (p->fp.nentries + 1));
    p->fp.ptr = (int64_t*)malloc(sizeof(int64_t) * (p->fp.nbands + 1));
    footprint_build(&p->g, kernel, alpha, ell, &p->fp, 1, p->rows);
  } else if (p->engine == ORC_ENGINE_SEPARABLE) {
    separable_build(&p->g, alpha, ell, strategy, &p->sp);
  } else {
    prefix_build(&p->g, ell, strategy, &p->pp);
  }
  return p;
}

orc_plan* orc_plan_new(int geometry, int nx, int ny, double x0, double dx, double y0, double dy, double R,
                       int periodic_x, int periodic_y, const uint8_t* mask, int kernel, double alpha,
                       double ell, int strategy, int engine) {
  return orc_plan_new_rows(geometry, nx, ny, x0, dx, y0, dy, R, periodic_x, periodic_y, mask, kernel, alpha, ell,
                           strategy, engine, NULL);
}

void orc_plan_free(orc_plan* p) {
  if (!p) return;
  free(p->rows);
  free(p->fp.di);
  free(p->fp.dj);
  free(p->fp.w);
  free(p->fp.ptr);
  free(p->sp.gx);
  free(p->sp.gy);
  free(p->sp.px);
  free(p->sp.py);
  free(p->sp.invrenorm);
  free(p->pp.wx);
  free(p->pp.wy);
  free(p->pp.xe);
  free(p->pp.src);
  free(p->pp.prefix_wx);
  free(p->pp.prefix_den);
  free(p->mask_copy);
  free(p);
}

int orc_plan_engine(const orc_plan* p) { return p->engine; }
int64_t orc_plan_nentries(const orc_plan* p) { return p->engine == ORC_ENGINE_BANDED ? p->fp.nentries : 0; }
int orc_plan_nbands(const orc_plan* p) { return p->engine == ORC_ENGINE_BANDED ? p->fp.nbands : 0; }
void orc_plan_footprint(const orc_plan* p, int* di, int* dj, double* w, int64_t* ptr) {
  if (p->engine != ORC_ENGINE_BANDED) return;
  memcpy(di, p->fp.di, sizeof(int) * p->fp.nentries);
  memcpy(dj, p->fp.dj, sizeof(int) * p->fp.nentries);
  memcpy(w, p->fp.w, sizeof(double) * p->fp.nentries);
  memcpy(ptr, p->fp.ptr, sizeof(int64_t) * (p->fp.nbands + 1));
}
void orc_plan_separable_lims(const orc_plan* p, int* lims) {
  lims[0] = p->sp.di_lim;
  lims[1] = p->sp.dj_lim;
}

/* filter_apply_batch! (Filtering.jl:3360-3375): K fields through one plan. */
void orc_filter_batch(const orc_plan* p, int K, const double* const* fields, double* const* outs, int nthreads) {
  if (p->engine == ORC_ENGINE_BANDED) {
    footprint_apply(&p->g, &p->fp, p->strategy, K, fields, outs, nthreads, p->rows);
  } else if (p->engine == ORC_ENGINE_SEPARABLE) {
    for (int m = 0; m < K; ++m) separable_apply(&p->g, &p->sp, fields[m], outs[m]);
  } else {
    for (int m = 0; m < K; ++m) prefix_apply(&p->g, &p->pp, fields[m], outs[m]);
  }
}

/* ------------------------------------------------------------------------------------
 * Derivatives (Derivatives.jl:26-51, 131-144): 3-node first derivative with ReduceInRun.
 * For an active cell the run of active neighbours along the axis decides the stencil:
 * centred (f+ - f-)/2h with both neighbours; 3-node one-sided when only one side has two
 * active neighbours (also the bounded domain end, CHANGELOG.md:257-259); 2-node one-sided
 * in a run of two; 0 in a run of one.  Masked cells are 0.  Periodic axes wrap.
 * Sphere: d/dx = (d/dlambda)/(R cos phi), 0 where |cos phi| < sqrt(eps) (CHANGELOG.md:243-246);
 * d/dy = (d/dphi)/R.
 * ------------------------------------------------------------------------------------ */
static inline int axis_neighbor(int p, int off, int n, int periodic) {
  int q = p + off;
  if (q < 0 || q >= n) {
    if (!periodic || n < 2) return -1;
    q = mod_n(q, n);
  }
  return q;
}

static double stencil_1d(const double* f, const uint8_t* act, int p, int n, int stride, int periodic, double h) {
  /* act: per-point activity along the line (indexed like f with the stride) */
#define F(q) f[(int64_t)(q) * stride]
#define A(q) ((q) >= 0 && act[(int64_t)(q) * stride])
  int m1 = axis_neighbor(p, -1, n, periodic), p1 = axis_neighbor(p, 1, n, periodic);
  int am1 = A(m1), ap1 = A(p1);
  if (am1 && ap1) return (F(p1) - F(m1)) / (2.0 * h);
  if (ap1) {
    int p2 = axis_neighbor(p, 2, n, periodic);
    if (A(p2) && p2 != p) return (-3.0 * F(p) + 4.0 * F(p1) - F(p2)) / (2.0 * h);
    return (F(p1) - F(p)) / h;
  }
  if (am1) {
    int m2 = axis_neighbor(p, -2, n, periodic);
    if (A(m2) && m2 != p) return (3.0 * F(p) - 4.0 * F(m1) + F(m2)) / (2.0 * h);
    return (F(p) - F(m1)) / h;
  }
  return 0.0;
#undef F
#undef A
}

static uint8_t* activity(const orc_grid* g) {
  int64_t n = (int64_t)g->nx * g->ny;
  uint8_t* a = (uint8_t*)malloc((size_t)n);
  for (int64_t k = 0; k < n; ++k) a[k] = g->mask ? (g->mask[k] != 0) : 1;
  return a;
}

void orc_ddx_grid(const orc_grid* g, const double* f, double* out) {
  int nx = g->nx, ny = g->ny;
  uint8_t* a = activity(g);
  for (int j = 0; j < ny; ++j) {
    double scale = 1.0;
    if (g->geometry == ORC_SPHERE) {
      double c = cos(gy_coord(g, j));
      scale = fabs(c) < sqrt(2.220446049250313e-16) ? 0.0 : 1.0 / (g->R * c);
    }
    for (int i = 0; i < nx; ++i) {
      int64_t o = (int64_t)j * nx + i;
      if (!a[o] || nx < 2) { out[o] = 0.0; continue; }
      double d = stencil_1d(f + (int64_t)j * nx, a + (int64_t)j * nx, i, nx, 1, g->periodic_x, g->dx);
      out[o] = d * scale;
    }
  }
  free(a);
}

void orc_ddy_grid(const orc_grid* g, const double* f, double* out) {
  int nx = g->nx, ny = g->ny;
  uint8_t* a = activity(g);
  double scale = g->geometry == ORC_SPHERE ? 1.0 / g->R : 1.0;
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      int64_t o = (int64_t)j * nx + i;
      if (!a[o] || ny < 2) { out[o] = 0.0; continue; }
      double d = stencil_1d(f + i, a + i, j, ny, nx, g->periodic_y, g->dy);
      out[o] = d * scale;
    }
  free(a);
}

void orc_ddx(const orc_plan* p, const double* f, double* out) { orc_ddx_grid(&p->g, f, out); }
void orc_ddy(const orc_plan* p, const double* f, double* out) { orc_ddy_grid(&p->g, f, out); }

/* ------------------------------------------------------------------------------------
 * Frame rotations on the sphere (Diagnostics.jl:555-573, 596-610, 612-650).
 * ------------------------------------------------------------------------------------ */
static inline void to_planetary(double u, double v, double lam, double phi, double* X, double* Y, double* Z) {
  double sl = sin(lam), cl = cos(lam), sp = sin(phi), cp = cos(phi);
  *X = -sl * u - sp * cl * v;
  *Y = cl * u - sp * sl * v;
  *Z = cp * v;
}

/* ------------------------------------------------------------------------------------
 * compute_Pi! (Diagnostics.jl:389-416, 472-702).  Outputs Pi = mask ? -(Sxx txx + 2 Sxy txy
 * + Syy tyy) : 0 (no rho0, Diagnostics.jl:689-699); the optional buffers receive the local
 * filtered velocities, the local SFS stress and the strain.
 * ------------------------------------------------------------------------------------ */
int orc_compute_pi(const orc_plan* p, const double* u, const double* v, double* Pi, double* ubar, double* vbar,
                   double* txx_o, double* txy_o, double* tyy_o, double* sxx_o, double* sxy_o, double* syy_o,
                   int nthreads) {
  const orc_grid* g = &p->g;
  int nx = g->nx, ny = g->ny;
  int64_t n = (int64_t)nx * ny;
  double* buf = (double*)calloc((size_t)n * 20, sizeof(double));
  double* uf = buf;
  double* vf = buf + n;
  double* txx = buf + 2 * n;
  double* txy = buf + 3 * n;
  double* tyy = buf + 4 * n;
  double* sxx = buf + 5 * n;
  double* sxy = buf + 6 * n;
  double* syy = buf + 7 * n;
  double* scr = buf + 8 * n;
  if (g->geometry == ORC_CART) {
    /* Diagnostics.jl:485-548 */
    double* uu = buf + 9 * n;
    double* uv = buf + 10 * n;
    double* vv = buf + 11 * n;
    double* fuu = buf + 12 * n;
    double* fuv = buf + 13 * n;
    double* fvv = buf + 14 * n;
    const double* in2[2] = {u, v};
    double* out2[2] = {uf, vf};
    orc_filter_batch(p, 2, in2, out2, nthreads);
    for (int64_t k = 0; k < n; ++k) {
      uu[k] = u[k] * u[k];
      uv[k] = u[k] * v[k];
      vv[k] = v[k] * v[k];
    }
    const double* in3[3] = {uu, uv, vv};
    double* out3[3] = {fuu, fuv, fvv};
    orc_filter_batch(p, 3, in3, out3, nthreads);
    for (int64_t k = 0; k < n; ++k) {
      txx[k] = fuu[k] - uf[k] * uf[k];
      txy[k] = fuv[k] - uf[k] * vf[k];
      tyy[k] = fvv[k] - vf[k] * vf[k];
    }
    orc_ddx_grid(g, uf, sxx);
    orc_ddy_grid(g, uf, sxy);
    orc_ddx_grid(g, vf, scr);
    orc_ddy_grid(g, vf, syy);
    for (int64_t k = 0; k < n; ++k) sxy[k] = 0.5 * (sxy[k] + scr[k]);
  } else {
    /* Diagnostics.jl:550-681 */
    double* X = buf + 9 * n;
    double* Y = buf + 10 * n;
    double* Z = buf + 11 * n;
    double* fX = buf + 12 * n;
    double* fY = buf + 13 * n;
    double* fZ = buf + 14 * n;
    double* P[6];
    double* fP[6];
    for (int q = 0; q < 6; ++q) P[q] = (double*)malloc(sizeof(double) * n);
    for (int q = 0; q < 6; ++q) fP[q] = (double*)malloc(sizeof(double) * n);
    for (int j = 0; j < ny; ++j)
      for (int i = 0; i < nx; ++i) {
        int64_t k = (int64_t)j * nx + i;
        if (is_active(g, i, j))
          to_planetary(u[k], v[k], gx_coord(g, i), gy_coord(g, j), &X[k], &Y[k], &Z[k]);
        else
          X[k] = Y[k] = Z[k] = 0.0;
      }
    const double* in3[3] = {X, Y, Z};
    double* out3[3] = {fX, fY, fZ};
    orc_filter_batch(p, 3, in3, out3, nthreads);
    for (int64_t k = 0; k < n; ++k) {
      P[0][k] = X[k] * X[k];
      P[1][k] = X[k] * Y[k];
      P[2][k] = X[k] * Z[k];
      P[3][k] = Y[k] * Y[k];
      P[4][k] = Y[k] * Z[k];
      P[5][k] = Z[k] * Z[k];
    }
    orc_filter_batch(p, 6, (const double* const*)P, fP, nthreads);
    for (int j = 0; j < ny; ++j) {
      double phi = gy_coord(g, j), sp = sin(phi), cp = cos(phi);
      for (int i = 0; i < nx; ++i) {
        int64_t k = (int64_t)j * nx + i;
        if (!is_active(g, i, j)) {
          uf[k] = vf[k] = txx[k] = txy[k] = tyy[k] = 0.0;
          continue;
        }
        double lam = gx_coord(g, i), sl = sin(lam), cl = cos(lam);
        double e[3] = {-sl, cl, 0.0};
        double nn[3] = {-sp * cl, -sp * sl, cp};
        double ub[3] = {fX[k], fY[k], fZ[k]};
        uf[k] = e[0] * ub[0] + e[1] * ub[1] + e[2] * ub[2];
        vf[k] = nn[0] * ub[0] + nn[1] * ub[1] + nn[2] * ub[2];
        double t[3][3];
        t[0][0] = fP[0][k] - ub[0] * ub[0];
        t[0][1] = t[1][0] = fP[1][k] - ub[0] * ub[1];
        t[0][2] = t[2][0] = fP[2][k] - ub[0] * ub[2];
        t[1][1] = fP[3][k] - ub[1] * ub[1];
        t[1][2] = t[2][1] = fP[4][k] - ub[1] * ub[2];
        t[2][2] = fP[5][k] - ub[2] * ub[2];
        double te[3], tn[3];
        for (int a = 0; a < 3; ++a) {
          te[a] = t[a][0] * e[0] + t[a][1] * e[1] + t[a][2] * e[2];
          tn[a] = t[a][0] * nn[0] + t[a][1] * nn[1] + t[a][2] * nn[2];
        }
        txx[k] = e[0] * te[0] + e[1] * te[1] + e[2] * te[2];
        txy[k] = e[0] * tn[0] + e[1] * tn[1] + e[2] * tn[2];
        tyy[k] = nn[0] * tn[0] + nn[1] * tn[1] + nn[2] * tn[2];
      }
    }
    orc_ddx_grid(g, uf, sxx);
    orc_ddy_grid(g, uf, sxy);
    orc_ddx_grid(g, vf, scr);
    orc_ddy_grid(g, vf, syy);
    for (int j = 0; j < ny; ++j) {
      double phi = gy_coord(g, j), sp = sin(phi), cp = cos(phi);
      double tan_fact = fabs(cp) > 1e-12 ? sp / (g->R * cp) : 0.0;
      for (int i = 0; i < nx; ++i) {
        int64_t k = (int64_t)j * nx + i;
        if (!is_active(g, i, j)) continue;
        sxx[k] -= vf[k] * tan_fact;
        sxy[k] = 0.5 * (sxy[k] + scr[k] + uf[k] * tan_fact);
      }
    }
    for (int q = 0; q < 6; ++q) {
      free(P[q]);
      free(fP[q]);
    }
  }
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      int64_t k = (int64_t)j * nx + i;
      Pi[k] = is_active(g, i, j) ? -(sxx[k] * txx[k] + 2.0 * sxy[k] * txy[k] + syy[k] * tyy[k]) : 0.0;
    }
  if (ubar) memcpy(ubar, uf, sizeof(double) * n);
  if (vbar) memcpy(vbar, vf, sizeof(double) * n);
  if (txx_o) memcpy(txx_o, txx, sizeof(double) * n);
  if (txy_o) memcpy(txy_o, txy, sizeof(double) * n);
  if (tyy_o) memcpy(tyy_o, tyy, sizeof(double) * n);
  if (sxx_o) memcpy(sxx_o, sxx, sizeof(double) * n);
  if (sxy_o) memcpy(sxy_o, sxy, sizeof(double) * n);
  if (syy_o) memcpy(syy_o, syy, sizeof(double) * n);
  free(buf);
  return 0;
}

/* ------------------------------------------------------------------------------------
 * compute_Pi! with the vertical velocity w (the 2.5-D path, Diagnostics.jl:254-260, 483-681).
 * Cartesian: u, v, w and the products uu, uv, vv, uw, vw, ww are filtered; tau_xz, tau_yz, tau_zz
 * follow; S_xz = 1/2 dwbar/dx, S_yz = 1/2 dwbar/dy, S_zz = 0 (Diagnostics.jl:540-548).  Sphere: the
 * planetary velocity includes w along the local up vector (vector_to_cartesian), the local filtered
 * velocity gains wbar = up . Ubar (vector_from_cartesian), tau is rotated to east/north/up in full
 * (tau_er, tau_nr, tau_rr too) and S_er = 1/2 dwbar/dx, S_nr = 1/2 dwbar/dy, S_rr = 0, with the metric
 * division of the derivatives but no curvature terms (Diagnostics.jl:658-667).
 * Pi = -(Sxx txx + 2 Sxy txy + Syy tyy + 2 Sxz txz + 2 Syz tyz + Szz tzz) on active cells
 * (Diagnostics.jl:463-465, 689-699).  outs (each n values, NULL skips one): ubar, vbar, wbar, txx,
 * txy, tyy, txz, tyz, tzz, sxx, sxy, syy, sxz, syz.
 * ------------------------------------------------------------------------------------ */
int orc_compute_pi_w(const orc_plan* p, const double* u, const double* v, const double* w, double* Pi,
                     double* const* outs, int nthreads) {
  const orc_grid* g = &p->g;
  int nx = g->nx, ny = g->ny;
  int64_t n = (int64_t)nx * ny;
  double* in[9];
  double* f[9];
  for (int q = 0; q < 9; ++q) {
    in[q] = (double*)calloc((size_t)n, sizeof(double));
    f[q] = (double*)calloc((size_t)n, sizeof(double));
  }
  double* loc = (double*)calloc((size_t)n * 14, sizeof(double));
  double *ub = loc, *vb = loc + n, *wb = loc + 2 * n, *txx = loc + 3 * n, *txy = loc + 4 * n, *tyy = loc + 5 * n,
         *txz = loc + 6 * n, *tyz = loc + 7 * n, *tzz = loc + 8 * n, *sxx = loc + 9 * n, *sxy = loc + 10 * n,
         *syy = loc + 11 * n, *sxz = loc + 12 * n, *syz = loc + 13 * n;
  double* scr = (double*)calloc((size_t)n, sizeof(double));
  int sphere = g->geometry == ORC_SPHERE;
  /* the three velocity components: (u, v, w) on the plane, planetary (X, Y, Z) on the sphere */
  for (int j = 0; j < ny; ++j)
    for (int i = 0; i < nx; ++i) {
      int64_t k = (int64_t)j * nx + i;
      if (!is_active(g, i, j)) continue;
      if (sphere) {
        double lam = gx_coord(g, i), phi = gy_coord(g, j);
        double sl = sin(lam), cl = cos(lam), sp = sin(phi), cp = cos(phi);
        in[0][k] = -sl * u[k] - sp * cl * v[k] + cp * cl * w[k];
        in[1][k] = cl * u[k] - sp * sl * v[k] + cp * sl * w[k];
        in[2][k] = cp * v[k] + sp * w[k];
      } else {
        in[0][k] = u[k];
        in[1][k] = v[k];
        in[2][k] = w[k];
      }
    }
  /* products: 00, 01, 02, 11, 12, 22 */
  for (int64_t k = 0; k < n; ++k) {
    in[3][k] = in[0][k] * in[0][k];
    in[4][k] = in[0][k] * in[1][k];
    in[5][k] = in[0][k] * in[2][k];
    in[6][k] = in[1][k] * in[1][k];
    in[7][k] = in[1][k] * in[2][k];
    in[8][k] = in[2][k] * in[2][k];
  }
  orc_filter_batch(p, 3, (const double* const*)in, f, nthreads);
  orc_filter_batch(p, 6, (const double* const*)(in + 3), f + 3, nthreads);
  for (int j = 0; j < ny; ++j) {
    double phi = gy_coord(g, j), sp = sin(phi), cp = cos(phi);
    for (int i = 0; i < nx; ++i) {
      int64_t k = (int64_t)j * nx + i;
      if (!is_active(g, i, j)) continue;
      double U[3] = {f[0][k], f[1][k], f[2][k]};
      double T[3][3];
      T[0][0] = f[3][k] - U[0] * U[0];
      T[0][1] = T[1][0] = f[4][k] - U[0] * U[1];
      T[0][2] = T[2][0] = f[5][k] - U[0] * U[2];
      T[1][1] = f[6][k] - U[1] * U[1];
      T[1][2] = T[2][1] = f[7][k] - U[1] * U[2];
      T[2][2] = f[8][k] - U[2] * U[2];
      if (!sphere) {
        ub[k] = U[0];
        vb[k] = U[1];
        wb[k] = U[2];
        txx[k] = T[0][0];
        txy[k] = T[0][1];
        tyy[k] = T[1][1];
        txz[k] = T[0][2];
        tyz[k] = T[1][2];
        tzz[k] = T[2][2];
        continue;
      }
      double lam = gx_coord(g, i), sl = sin(lam), cl = cos(lam);
      double e[3] = {-sl, cl, 0.0};
      double nn[3] = {-sp * cl, -sp * sl, cp};
      double r[3] = {cp * cl, cp * sl, sp};
      ub[k] = e[0] * U[0] + e[1] * U[1] + e[2] * U[2];
      vb[k] = nn[0] * U[0] + nn[1] * U[1] + nn[2] * U[2];
      wb[k] = r[0] * U[0] + r[1] * U[1] + r[2] * U[2];
      double te[3], tn[3], tr[3];
      for (int a = 0; a < 3; ++a) {
        te[a] = T[a][0] * e[0] + T[a][1] * e[1] + T[a][2] * e[2];
        tn[a] = T[a][0] * nn[0] + T[a][1] * nn[1] + T[a][2] * nn[2];
        tr[a] = T[a][0] * r[0] + T[a][1] * r[1] + T[a][2] * r[2];
      }
      txx[k] = e[0] * te[0] + e[1] * te[1] + e[2] * te[2];
      txy[k] = e[0] * tn[0] + e[1] * tn[1] + e[2] * tn[2];
      tyy[k] = nn[0] * tn[0] + nn[1] * tn[1] + nn[2] * tn[2];
      txz[k] = e[0] * tr[0] + e[1] * tr[1] + e[2] * tr[2];
      tyz[k] = nn[0] * tr[0] + nn[1] * tr[1] + nn[2] * tr[2];
      tzz[k] = r[0] * tr[0] + r[1] * tr[1] + r[2] * tr[2];
    }
  }
  orc_ddx_grid(g, ub, sxx);
  orc_ddy_grid(g, ub, sxy);
  orc_ddx_grid(g, vb, scr);
  orc_ddy_grid(g, vb, syy);
  orc_ddx_grid(g, wb, sxz);
  orc_ddy_grid(g, wb, syz);
  for (int j = 0; j < ny; ++j) {
    double phi = gy_coord(g, j), sp = sin(phi), cp = cos(phi);
    double tan_fact = sphere && fabs(cp) > 1e-12 ? sp / (g->R * cp) : 0.0;
    for (int i = 0; i < nx; ++i) {
      int64_t k = (int64_t)j * nx + i;
      if (!is_active(g, i, j)) {
        Pi[k] = 0.0;
        continue;
      }
      if (sphere) {
        sxx[k] -= vb[k] * tan_fact;
        sxy[k] = 0.5 * (sxy[k] + scr[k] + ub[k] * tan_fact);
      } else {
        sxy[k] = 0.5 * (sxy[k] + scr[k]);
      }
      sxz[k] = 0.5 * sxz[k];
      syz[k] = 0.5 * syz[k];
      double szz = 0.0;
      Pi[k] = -(sxx[k] * txx[k] + 2.0 * sxy[k] * txy[k] + syy[k] * tyy[k] + 2.0 * sxz[k] * txz[k] +
                2.0 * syz[k] * tyz[k] + szz * tzz[k]);
    }
  }
  double* src[14] = {ub, vb, wb, txx, txy, tyy, txz, tyz, tzz, sxx, sxy, syy, sxz, syz};
  for (int q = 0; q < 14; ++q)
    if (outs && outs[q]) memcpy(outs[q], src[q], sizeof(double) * n);
  for (int q = 0; q < 9; ++q) {
    free(in[q]);
    free(f[q]);
  }
  free(loc);
  free(scr);
  return 0;
}

/* ------------------------------------------------------------------------------------
 * Energies (Diagnostics.jl:1051-1059 active_area, 1086-1134 energy_from_filtered,
 * 1144-1217 cumulative_energy!, 1319-1333 spectral_density!).
 * ------------------------------------------------------------------------------------ */
double orc_active_area(const orc_plan* p) {
  const orc_grid* g = &p->g;
  double total = 0.0;
  for (int j = 0; j < g->ny; ++j)
    for (int i = 0; i < g->nx; ++i)
      if (is_active(g, i, j)) total += orc_area(g, i, j);
  return total;
}

double orc_energy_from_filtered(const orc_plan* p, const double* uf, const double* vf, double total_area) {
  const orc_grid* g = &p->g;
  double e = 0.0;
  for (int j = 0; j < g->ny; ++j)
    for (int i = 0; i < g->nx; ++i) {
      if (!is_active(g, i, j)) continue;
      int64_t k = (int64_t)j * g->nx + i;
      double v2 = uf[k] * uf[k] + vf[k] * vf[k];
      e += v2 * orc_area(g, i, j);
    }
  return 0.5 * e / total_area;
}

/* cumulative_energy!: filters u, v as scalars (local components) per scale. */
double orc_cumulative_energy_one(const orc_plan* p, const double* u, const double* v, int nthreads) {
  int64_t n = (int64_t)p->g.nx * p->g.ny;
  double* uf = (double*)malloc(sizeof(double) * n);
  double* vf = (double*)malloc(sizeof(double) * n);
  const double* in2[2] = {u, v};
  double* out2[2] = {uf, vf};
  orc_filter_batch(p, 2, in2, out2, nthreads);
  double e = orc_energy_from_filtered(p, uf, vf, orc_active_area(p));
  free(uf);
  free(vf);
  return e;
}

void orc_spectral_density(const double* C, const double* k, int n, double* g) {
  if (n < 2) {
    for (int i = 0; i < n; ++i) g[i] = 0.0;
    return;
  }
  for (int i = 0; i < n; ++i) {
    if (i == 0)
      g[i] = (C[1] - C[0]) / (k[1] - k[0]);
    else if (i == n - 1)
      g[i] = (C[n - 1] - C[n - 2]) / (k[n - 1] - k[n - 2]);
    else
      g[i] = (C[i + 1] - C[i - 1]) / (k[i + 1] - k[i - 1]);
  }
}

int orc_max_threads(void) {
#ifdef _OPENMP
  return omp_get_max_threads();
#else
  return 1;
#endif
}

/* Grid coordinates exactly as every routine above evaluates them. */
void orc_coords(const orc_plan* p, double* x, double* y) {
  for (int i = 0; i < p->g.nx; ++i) x[i] = gx_coord(&p->g, i);
  for (int j = 0; j < p->g.ny; ++j) y[j] = gy_coord(&p->g, j);
}

/* Entry count of the banded footprint (the counting pass of footprint_build, rows in parallel):
 * the benchmark's cost model for extrapolating a timed subset of scales. */
int64_t orc_count_entries(int geometry, int nx, int ny, double x0, double dx, double y0, double dy, double R,
                          int periodic_x, int periodic_y, int kernel, double alpha, double ell) {
  orc_grid g = {geometry, nx, ny, x0, dx, y0, dy, R, periodic_x, periodic_y, NULL};
  if (geometry == ORC_CART) {
    orc_footprint fp;
    footprint_build(&g, kernel, alpha, ell, &fp, 0, NULL);
    return fp.nentries;
  }
  double rad = orc_kernel_radius(kernel, alpha, ell);
  int dj_lim = dy > 0 ? (int)ceil(rad / (R * dy)) : 0;
  int half = nx / 2;
  int64_t total = 0;
#pragma omp parallel for schedule(dynamic, 4) reduction(+ : total)
  for (int j = 0; j < ny; ++j) {
    double phi = gy_coord(&g, j);
    int closed = 0;
    for (int ddj = -dj_lim; ddj <= dj_lim; ++ddj) {
      int jj = j + ddj;
      if (jj < 0 || jj >= ny) continue;
      if (sphere_row_window(&g, phi, gy_coord(&g, jj), rad, half) >= half) closed = 1;
    }
    for (int ddj = -dj_lim; ddj <= dj_lim; ++ddj) {
      int jj = j + ddj;
      if (jj < 0 || jj >= ny) continue;
      double phi2 = gy_coord(&g, jj);
      int win = closed ? half : sphere_row_window(&g, phi, phi2, rad, half);
      int lo = -win, hi = (closed && 2 * half + 1 > nx) ? half - 1 : win;
      for (int ddi = lo; ddi <= hi; ++ddi)
        if (orc_distance(&g, 0.0, phi, (double)ddi * dx, phi2) <= rad) ++total;
    }
  }
  return total;
}
