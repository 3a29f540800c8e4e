/*
 * CPU oracle (FP64, plain C) for the Peridigm LPS / critical-stretch / Verlet /
 * contact path. TEST INFRASTRUCTURE ONLY: called by tests/, smoke() and the
 * CPU-baseline leg of bench.py as the checker; never linked by the product.
 * Each function names the reference file:line it restates. Compiled with
 * -ffp-contract=off so every product and sum rounds like the reference's
 * scalar C++ build (no fused multiply-add).
 */
#include "pd_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>
#include <string.h>

/* ---------------------------------------------------------------------------
 * Influence functions: src/core/Peridigm_InfluenceFunction.hpp:69-87.
 * ------------------------------------------------------------------------- */
double pdo_influence(int kind, double zeta, double horizon) {
  if (kind == PDO_INFLUENCE_PARABOLIC) {
    if (zeta > horizon) return 0.0;
    double s = zeta / horizon;
    return s < 0.5 ? 1.0 : -4.0 * s * s + 4.0 * s;
  }
  if (kind == PDO_INFLUENCE_GAUSSIAN) {
    double h2 = horizon * horizon * 0.4 * 0.4;
    double xi2 = zeta * zeta;
    return exp(-xi2 / h2);
  }
  return 1.0;
}

/* ---------------------------------------------------------------------------
 * FinitePlane (src/io/pdneigh/BondFilter.cxx:59-106) as used by
 * FinitePlaneFilter::filterBonds (:123-150): p0 is the owner, p1 the neighbor.
 * ua = cross(ub, n) with the component order of UTILITIES::Cross
 * (src/io/utilities/Vector3D.h:119-128); dot as UTILITIES::Dot (:112-116).
 * ------------------------------------------------------------------------- */
int pdo_plane_cuts_bond(const pdo_plane* pl, const double* p0, const double* p1) {
  const double* n = pl->normal;
  const double* r0 = pl->lower_left;
  const double* ub = pl->bottom_unit;
  double ua[3];
  ua[0] = -ub[2] * n[1] + ub[1] * n[2];
  ua[1] = ub[2] * n[0] - ub[0] * n[2];
  ua[2] = -ub[1] * n[0] + ub[0] * n[1];
  double a = pl->side_length, b = pl->bottom_length;

  double numerator = (r0[0] - p0[0]) * n[0] + (r0[1] - p0[1]) * n[1] + (r0[2] - p0[2]) * n[2];
  double denominator = (p1[0] - p0[0]) * n[0] + (p1[1] - p0[1]) * n[1] + (p1[2] - p0[2]) * n[2];
  double t;
  if (fabs(denominator) < 1.0e-14)
    t = DBL_MAX;
  else
    t = numerator / denominator;
  if (!(t >= 0.0 && t <= 1.0)) return 0;
  double xx[3];
  xx[0] = p0[0] + t * (p1[0] - p0[0]);
  xx[1] = p0[1] + t * (p1[1] - p0[1]);
  xx[2] = p0[2] + t * (p1[2] - p0[2]);
  /* bondIntersect with the FinitePlaneFilter tolerance 1e-15 (BondFilter.h:122). */
  double zero = 1.0e-15, one = 1.0 + zero;
  double dr[3] = {xx[0] - r0[0], xx[1] - r0[1], xx[2] - r0[2]};
  double aa = dr[0] * ua[0] + dr[1] * ua[1] + dr[2] * ua[2];
  double bb = dr[0] * ub[0] + dr[1] * ub[1] + dr[2] * ub[2];
  return (-zero < aa && aa / a < one && -zero < bb && bb / b < one) ? 1 : 0;
}

/* ---------------------------------------------------------------------------
 * Uniform cell grid used by both searches (candidate generation only; the
 * predicate decides membership, so the grid changes no result).
 * ------------------------------------------------------------------------- */
typedef struct {
  double lo[3];
  double c;
  int64_t dims[3];
  int64_t ncell;
  int64_t* start; /* [ncell+1] */
  int64_t* idx;   /* [n] point ids, ascending within a cell */
} cells_t;

static int64_t cell_coord(const cells_t* g, double v, int k) {
  int64_t q = (int64_t)floor((v - g->lo[k]) / g->c);
  if (q < 0) q = 0;
  if (q >= g->dims[k]) q = g->dims[k] - 1;
  return q;
}

static void cells_build(cells_t* g, int64_t n, const double* x, double reach) {
  double lo[3] = {DBL_MAX, DBL_MAX, DBL_MAX}, hi[3] = {-DBL_MAX, -DBL_MAX, -DBL_MAX};
  for (int64_t i = 0; i < n; ++i)
    for (int k = 0; k < 3; ++k) {
      if (x[3 * i + k] < lo[k]) lo[k] = x[3 * i + k];
      if (x[3 * i + k] > hi[k]) hi[k] = x[3 * i + k];
    }
  if (n == 0) lo[0] = lo[1] = lo[2] = hi[0] = hi[1] = hi[2] = 0.0;
  double c = reach * 1.0001 + 1e-300;
  for (;;) {
    int64_t tot = 1;
    for (int k = 0; k < 3; ++k) {
      g->dims[k] = (int64_t)floor((hi[k] - lo[k]) / c) + 1;
      tot *= g->dims[k];
    }
    if (tot <= 4 * n + 64) break;
    c *= 1.5;
  }
  for (int k = 0; k < 3; ++k) g->lo[k] = lo[k];
  g->c = c;
  g->ncell = g->dims[0] * g->dims[1] * g->dims[2];
  g->start = (int64_t*)calloc((size_t)g->ncell + 1, sizeof(int64_t));
  g->idx = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
  int64_t* cid = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n > 0 ? n : 1));
  for (int64_t i = 0; i < n; ++i) {
    int64_t a = cell_coord(g, x[3 * i], 0), b = cell_coord(g, x[3 * i + 1], 1),
            cc = cell_coord(g, x[3 * i + 2], 2);
    cid[i] = (cc * g->dims[1] + b) * g->dims[0] + a;
    g->start[cid[i] + 1]++;
  }
  for (int64_t q = 0; q < g->ncell; ++q) g->start[q + 1] += g->start[q];
  int64_t* fillp = (int64_t*)malloc(sizeof(int64_t) * (size_t)g->ncell);
  memcpy(fillp, g->start, sizeof(int64_t) * (size_t)g->ncell);
  for (int64_t i = 0; i < n; ++i) g->idx[fillp[cid[i]]++] = i;
  free(fillp);
  free(cid);
}

static void cells_free(cells_t* g) {
  free(g->start);
  free(g->idx);
}

static int cmp_i32(const void* a, const void* b) {
  int32_t x = *(const int32_t*)a, y = *(const int32_t*)b;
  return (x > y) - (x < y);
}

/* Candidates of point i within the 27 cells around p, filtered by
 * ZoltanSearchTree::FindPointsWithinRadius's predicate
 * (src/io/Peridigm_ZoltanSearchTree.cpp:238-245): dx = x_cand - p, keep when
 * dx*dx+dy*dy+dz*dz <= R2, R2 = r*r; then self exclusion
 * (BondFilterDefault, src/io/pdneigh/BondFilter.cxx:108-121) and the plane
 * filters. Writes the ascending list (NeighborhoodList.cxx:705) into out. */
static int64_t gather_row(const cells_t* g, const double* x, int64_t i, const double* p,
                          double r, const pdo_plane* planes, int n_planes, int32_t* out,
                          int64_t cap) {
  double R2 = r * r;
  int64_t c0 = cell_coord(g, p[0], 0), c1 = cell_coord(g, p[1], 1), c2 = cell_coord(g, p[2], 2);
  int64_t cnt = 0;
  for (int64_t zc = c2 - 1; zc <= c2 + 1; ++zc) {
    if (zc < 0 || zc >= g->dims[2]) continue;
    for (int64_t yc = c1 - 1; yc <= c1 + 1; ++yc) {
      if (yc < 0 || yc >= g->dims[1]) continue;
      for (int64_t xc = c0 - 1; xc <= c0 + 1; ++xc) {
        if (xc < 0 || xc >= g->dims[0]) continue;
        int64_t q = (zc * g->dims[1] + yc) * g->dims[0] + xc;
        for (int64_t s = g->start[q]; s < g->start[q + 1]; ++s) {
          int64_t j = g->idx[s];
          if (j == i) continue;
          double dx = (x[3 * j] - p[0]);
          double dy = (x[3 * j + 1] - p[1]);
          double dz = (x[3 * j + 2] - p[2]);
          if (!(dx * dx + dy * dy + dz * dz <= R2)) continue;
          int cut = 0;
          for (int f = 0; f < n_planes && !cut; ++f) cut = pdo_plane_cuts_bond(&planes[f], p, &x[3 * j]);
          if (cut) continue;
          if (out && cnt < cap) out[cnt] = (int32_t)j;
          cnt++;
        }
      }
    }
  }
  if (out) qsort(out, (size_t)(cnt < cap ? cnt : cap), sizeof(int32_t), cmp_i32);
  return cnt;
}

static double max_of(int64_t n, const double* h) {
  double m = 0.0;
  for (int64_t i = 0; i < n; ++i)
    if (h[i] > m) m = h[i];
  return m;
}

/* NeighborhoodList::buildNeighborhoodList, first pass (NeighborhoodList.cxx:638-681). */
int64_t pdo_neighbor_count(int64_t n, const double* x, const double* horizon,
                           const pdo_plane* planes, int n_planes, int32_t* counts) {
  cells_t g;
  cells_build(&g, n, x, max_of(n, horizon));
  int64_t tot = 0;
  for (int64_t i = 0; i < n; ++i) {
    int64_t c = gather_row(&g, x, i, &x[3 * i], horizon[i], planes, n_planes, NULL, 0);
    counts[i] = (int32_t)c;
    tot += c;
  }
  cells_free(&g);
  return tot;
}

/* NeighborhoodList::buildNeighborhoodList, second pass (NeighborhoodList.cxx:686-748). */
void pdo_neighbor_fill(int64_t n, const double* x, const double* horizon,
                       const pdo_plane* planes, int n_planes, const int64_t* row, int32_t* col) {
  cells_t g;
  cells_build(&g, n, x, max_of(n, horizon));
  for (int64_t i = 0; i < n; ++i)
    gather_row(&g, x, i, &x[3 * i], horizon[i], planes, n_planes, col + row[i], row[i + 1] - row[i]);
  cells_free(&g);
}

/* ---------------------------------------------------------------------------
 * Weighted volume: MATERIAL_EVALUATION::computeWeightedVolume
 * (src/materials/material_utilities.cxx:161-188, loop :501-520).
 * ------------------------------------------------------------------------- */
void pdo_weighted_volume(int64_t n, const double* x, const double* vol, const int64_t* row,
                         const int32_t* col, int influence, double horizon, double* m) {
  for (int64_t p = 0; p < n; ++p) {
    const double* X = &x[3 * p];
    double acc = 0.0;
    for (int64_t b = row[p]; b < row[p + 1]; ++b) {
      int64_t j = col[b];
      double dx = x[3 * j] - X[0], dy = x[3 * j + 1] - X[1], dz = x[3 * j + 2] - X[2];
      double z2 = dx * dx + dy * dy + dz * dz;
      double d = sqrt(z2);
      acc += pdo_influence(influence, d, horizon) * (z2)*vol[j];
    }
    m[p] = acc;
  }
}

/* ---------------------------------------------------------------------------
 * CriticalStretchDamageModel::computeDamage
 * (src/damage/Peridigm_CriticalStretchDamageModel.cpp:108-184): copy N->NP1
 * (:131), break when (|Y|-|X|)/|X| > s_c (strict, :155-158), keep the max
 * (:159-161), node damage = mean bond damage (:170-183). s_c is the owner's.
 * ------------------------------------------------------------------------- */
static double dist3(double a1, double a2, double a3, double b1, double b2, double b3) {
  return sqrt((a1 - b1) * (a1 - b1) + (a2 - b2) * (a2 - b2) + (a3 - b3) * (a3 - b3));
}

void pdo_damage_critical_stretch(int64_t n, const double* x, const double* y, const int64_t* row,
                                 const int32_t* col, const double* s_c, const double* dmg_n,
                                 double* dmg_np1, double* node_damage) {
  int64_t nb = row[n];
  if (dmg_np1 != dmg_n) memcpy(dmg_np1, dmg_n, sizeof(double) * (size_t)nb);
  for (int64_t i = 0; i < n; ++i) {
    for (int64_t b = row[i]; b < row[i + 1]; ++b) {
      int64_t j = col[b];
      double d0 = dist3(x[3 * i], x[3 * i + 1], x[3 * i + 2], x[3 * j], x[3 * j + 1], x[3 * j + 2]);
      double d1 = dist3(y[3 * i], y[3 * i + 1], y[3 * i + 2], y[3 * j], y[3 * j + 1], y[3 * j + 2]);
      double rel = (d1 - d0) / d0;
      double trial = 0.0;
      if (rel > s_c[i]) trial = 1.0;
      if (trial > dmg_np1[b]) dmg_np1[b] = trial;
    }
  }
  if (node_damage) {
    for (int64_t i = 0; i < n; ++i) {
      int64_t k = row[i + 1] - row[i];
      double tot = 0.0;
      for (int64_t b = row[i]; b < row[i + 1]; ++b) tot += dmg_np1[b];
      node_damage[i] = k > 0 ? tot / (double)k : 0.0;
    }
  }
}

/* ---------------------------------------------------------------------------
 * Dilatation: MATERIAL_EVALUATION::computeDilatation<double>
 * (src/materials/material_utilities.cxx:235-289), thermal term off.
 * ------------------------------------------------------------------------- */
void pdo_dilatation(int64_t n, const double* x, const double* y, const double* m,
                    const double* vol, const double* dmg, const int64_t* row, const int32_t* col,
                    int influence, double horizon, double* theta) {
  for (int64_t p = 0; p < n; ++p) {
    const double* X = &x[3 * p];
    const double* Y = &y[3 * p];
    double th = 0.0;
    for (int64_t b = row[p]; b < row[p + 1]; ++b) {
      int64_t j = col[b];
      double X_dx = x[3 * j] - X[0], X_dy = x[3 * j + 1] - X[1], X_dz = x[3 * j + 2] - X[2];
      double z2 = X_dx * X_dx + X_dy * X_dy + X_dz * X_dz;
      double Y_dx = y[3 * j] - Y[0], Y_dy = y[3 * j + 1] - Y[1], Y_dz = y[3 * j + 2] - Y[2];
      double dY = Y_dx * Y_dx + Y_dy * Y_dy + Y_dz * Y_dz;
      double d = sqrt(z2);
      double e = sqrt(dY);
      e -= d;
      double omega = pdo_influence(influence, d, horizon);
      th += 3.0 * omega * (1.0 - dmg[b]) * d * e * vol[j] / m[p];
    }
    theta[p] = th;
  }
}

/* ---------------------------------------------------------------------------
 * LPS force state: MATERIAL_EVALUATION::computeInternalForceLinearElastic<double>
 * (src/materials/elastic.cxx:55-146), scatter form (:125-130), partial stress
 * and thermal terms off. K and mu are the owner's (per point; the reference
 * has one value per block). f is zeroed first as in
 * ElasticMaterial::computeForce (Peridigm_ElasticMaterial.cpp:149).
 * ------------------------------------------------------------------------- */
void pdo_force_lps(int64_t n, const double* x, const double* y, const double* m,
                   const double* vol, const double* theta, const double* dmg, const int64_t* row,
                   const int32_t* col, const double* K, const double* mu, int influence,
                   double horizon, double* f) {
  memset(f, 0, sizeof(double) * 3 * (size_t)n);
  for (int64_t p = 0; p < n; ++p) {
    const double* X = &x[3 * p];
    const double* Y = &y[3 * p];
    double alpha = 15.0 * mu[p] / m[p];
    double selfV = vol[p];
    for (int64_t b = row[p]; b < row[p + 1]; ++b) {
      int64_t j = col[b];
      double cellV = vol[j];
      double X_dx = x[3 * j] - X[0], X_dy = x[3 * j + 1] - X[1], X_dz = x[3 * j + 2] - X[2];
      double zeta = sqrt(X_dx * X_dx + X_dy * X_dy + X_dz * X_dz);
      double Y_dx = y[3 * j] - Y[0], Y_dy = y[3 * j + 1] - Y[1], Y_dz = y[3 * j + 2] - Y[2];
      double dY = sqrt(Y_dx * Y_dx + Y_dy * Y_dy + Y_dz * Y_dz);
      double e = dY - zeta;
      double omega = pdo_influence(influence, zeta, horizon);
      double c1 = omega * theta[p] * (3.0 * K[p] / m[p] - alpha / 3.0);
      double t = (1.0 - dmg[b]) * (c1 * zeta + (1.0 - dmg[b]) * omega * alpha * e);
      double fx = t * Y_dx / dY, fy = t * Y_dy / dY, fz = t * Y_dz / dY;
      f[3 * p + 0] += fx * cellV;
      f[3 * p + 1] += fy * cellV;
      f[3 * p + 2] += fz * cellV;
      f[3 * j + 0] -= fx * selfV;
      f[3 * j + 1] -= fy * selfV;
      f[3 * j + 2] -= fz * selfV;
    }
  }
}

/* ---------------------------------------------------------------------------
 * Elastic bond-based force: MATERIAL_EVALUATION::computeInternalForceElasticBondBased<double>
 * (src/materials/elastic_bond_based.cxx:55-124), scatter form (:118-123),
 * constant 18K/(pi h^4) in 3D (:77) or 12K/(pi H h^3) for plane strain/stress
 * (:75); K is the owner's. f is zeroed first as in
 * ElasticBondBasedMaterial::computeForce (Peridigm_ElasticBondBasedMaterial.cpp:116).
 * ------------------------------------------------------------------------- */
void pdo_force_bond_based(int64_t n, const double* x, const double* y, const double* vol,
                          const double* dmg, const int64_t* row, const int32_t* col, const double* K,
                          double horizon, int plane, double height, double* f) {
  const double pi = 3.14159265358979323846;
  memset(f, 0, sizeof(double) * 3 * (size_t)n);
  for (int64_t p = 0; p < n; ++p) {
    const double* X = &x[3 * p];
    const double* Y = &y[3 * p];
    double c = plane ? 12.0 * K[p] / (pi * height * horizon * horizon * horizon)
                     : 18.0 * K[p] / (pi * horizon * horizon * horizon * horizon);
    for (int64_t b = row[p]; b < row[p + 1]; ++b) {
      int64_t j = col[b];
      double zeta = sqrt((x[3 * j] - X[0]) * (x[3 * j] - X[0]) + (x[3 * j + 1] - X[1]) * (x[3 * j + 1] - X[1]) +
                         (x[3 * j + 2] - X[2]) * (x[3 * j + 2] - X[2]));
      double dY = sqrt((y[3 * j] - Y[0]) * (y[3 * j] - Y[0]) + (y[3 * j + 1] - Y[1]) * (y[3 * j + 1] - Y[1]) +
                       (y[3 * j + 2] - Y[2]) * (y[3 * j + 2] - Y[2]));
      double stretch = (dY - zeta) / zeta;
      double t = 0.5 * (1.0 - dmg[b]) * stretch * c;
      double fx = t * (y[3 * j] - Y[0]) / dY, fy = t * (y[3 * j + 1] - Y[1]) / dY, fz = t * (y[3 * j + 2] - Y[2]) / dY;
      f[3 * p + 0] += fx * vol[j];
      f[3 * p + 1] += fy * vol[j];
      f[3 * p + 2] += fz * vol[j];
      f[3 * j + 0] -= fx * vol[p];
      f[3 * j + 1] -= fy * vol[p];
      f[3 * j + 2] -= fz * vol[p];
    }
  }
}

/* ---------------------------------------------------------------------------
 * Linear LPS ("Linear LPS Partial Volume" without partial volumes or improved
 * quadrature): the loops of PeridigmNS::LinearLPSPVMaterial::precompute
 * (src/materials/Peridigm_LinearLPSPVMaterial.cpp:231-292) and ::computeForce
 * (:295-394), which the material runs (not the functions of
 * linear_lps_pv.cxx, which square sqrt(|zeta|^2) instead of using |zeta|^2).
 *   theta_i = 3/m_i * sum omega (1-d) zeta.(u_j - u_i) V_j
 *   f = (1-d) (t1 zeta + t2 (zeta zeta^T)(u_j - u_i)),
 *   t1 = (9K - 15mu) omega theta_i / (3 m_i), t2 = 15mu omega / (m_i |zeta|^2),
 *   f_i += f V_j, f_j -= f V_i (scatter). omega is the bond's influence
 *   value (computeAndStoreInfluenceFunctionValues, material_utilities.cxx:55-84).
 * ------------------------------------------------------------------------- */
static double lin_omega(int influence, const double* X, const double* XN, double horizon) {
  double d = sqrt((X[0] - XN[0]) * (X[0] - XN[0]) + (X[1] - XN[1]) * (X[1] - XN[1]) + (X[2] - XN[2]) * (X[2] - XN[2]));
  return pdo_influence(influence, d, horizon);
}

void pdo_dilatation_linear_lps(int64_t n, const double* x, const double* y, const double* m, const double* vol,
                               const double* dmg, const int64_t* row, const int32_t* col, int influence,
                               double horizon, double* theta) {
  for (int64_t p = 0; p < n; ++p) {
    const double* xs = &x[3 * p];
    const double* ys = &y[3 * p];
    double th = 0.0;
    for (int64_t b = row[p]; b < row[p + 1]; ++b) {
      int64_t j = col[b];
      const double* xn = &x[3 * j];
      const double* yn = &y[3 * j];
      double zeta[3], u[3], un[3];
      for (int i = 0; i < 3; ++i) {
        zeta[i] = xn[i] - xs[i];
        u[i] = ys[i] - xs[i];
        un[i] = yn[i] - xn[i];
      }
      double omega = lin_omega(influence, xs, xn, horizon);
      double dot = zeta[0] * (un[0] - u[0]) + zeta[1] * (un[1] - u[1]) + zeta[2] * (un[2] - u[2]);
      th += omega * (1.0 - dmg[b]) * dot * vol[j];
    }
    if (row[p + 1] > row[p]) th *= 3.0 / m[p];
    theta[p] = th;
  }
}

void pdo_force_linear_lps(int64_t n, const double* x, const double* y, const double* m, const double* vol,
                          const double* theta, const double* dmg, const int64_t* row, const int32_t* col,
                          const double* K, const double* mu, int influence, double horizon, double* f) {
  memset(f, 0, sizeof(double) * 3 * (size_t)n);
  for (int64_t p = 0; p < n; ++p) {
    const double* xs = &x[3 * p];
    const double* ys = &y[3 * p];
    for (int64_t b = row[p]; b < row[p + 1]; ++b) {
      int64_t j = col[b];
      const double* xn = &x[3 * j];
      const double* yn = &y[3 * j];
      double zeta[3], u[3], un[3], mv[3];
      for (int i = 0; i < 3; ++i) {
        zeta[i] = xn[i] - xs[i];
        u[i] = ys[i] - xs[i];
        un[i] = yn[i] - xn[i];
      }
      double z2 = zeta[0] * zeta[0] + zeta[1] * zeta[1] + zeta[2] * zeta[2];
      double omega = lin_omega(influence, xs, xn, horizon);
      double t1 = (9.0 * K[p] - 15.0 * mu[p]) * omega * (theta[p]) / (3.0 * (m[p]));
      double t2 = 15.0 * mu[p] * omega / ((m[p]) * z2);
      for (int i = 0; i < 3; ++i)
        mv[i] = (zeta[i] * zeta[0]) * (un[0] - u[0]) + (zeta[i] * zeta[1]) * (un[1] - u[1]) +
                (zeta[i] * zeta[2]) * (un[2] - u[2]);
      double fx = (1.0 - dmg[b]) * (t1 * zeta[0] + t2 * mv[0]);
      double fy = (1.0 - dmg[b]) * (t1 * zeta[1] + t2 * mv[1]);
      double fz = (1.0 - dmg[b]) * (t1 * zeta[2] + t2 * mv[2]);
      f[3 * p + 0] += fx * vol[j];
      f[3 * p + 1] += fy * vol[j];
      f[3 * p + 2] += fz * vol[j];
      f[3 * j + 0] -= fx * vol[p];
      f[3 * j + 1] -= fy * vol[p];
      f[3 * j + 2] -= fz * vol[p];
    }
  }
}

/* ---------------------------------------------------------------------------
 * Stable time step: PeridigmNS::ComputeCriticalTimeStep
 * (src/core/Peridigm_CriticalTimeStep.cpp:52-130), constant horizon, owner K.
 * ------------------------------------------------------------------------- */
double pdo_critical_time_step(int64_t n, const double* x, const double* vol, const int64_t* row,
                              const int32_t* col, const double* K, const double* rho,
                              double horizon) {
  const double pi = 3.14159265358979323846;
  double best = 1.0e50;
  for (int64_t i = 0; i < n; ++i) {
    double spring = 18.0 * K[i] / (pi * horizon * horizon * horizon * horizon);
    double X0 = x[3 * i], X1 = x[3 * i + 1], X2 = x[3 * i + 2];
    double den = 0.0;
    for (int64_t b = row[i]; b < row[i + 1]; ++b) {
      int64_t j = col[b];
      double d = sqrt((X0 - x[3 * j]) * (X0 - x[3 * j]) + (X1 - x[3 * j + 1]) * (X1 - x[3 * j + 1]) +
                      (X2 - x[3 * j + 2]) * (X2 - x[3 * j + 2]));
      den += vol[j] * spring / d;
    }
    double cts = 1.0e50;
    if (row[i + 1] > row[i]) cts = sqrt(2.0 * rho[i] / den);
    if (cts < best) best = cts;
  }
  return best;
}

/* ---------------------------------------------------------------------------
 * Contact search: ContactManager::contactSearch
 * (src/core/Peridigm_ContactManager.cpp:696-748): all points within the search
 * radius of the current coordinates (Zoltan predicate, self excluded), minus
 * every pair in the bond family (broken bonds included, :741).
 * ------------------------------------------------------------------------- */
static int in_sorted_row(const int32_t* a, int64_t len, int32_t v) {
  int64_t lo = 0, hi = len;
  while (lo < hi) {
    int64_t mid = (lo + hi) / 2;
    if (a[mid] < v) lo = mid + 1; else hi = mid;
  }
  return lo < len && a[lo] == v;
}

static int64_t contact_row(const cells_t* g, const double* y, int64_t i, double r,
                           const int64_t* brow, const int32_t* bcol, int32_t* out, int64_t cap) {
  int32_t* tmp = NULL;
  int64_t c = gather_row(g, y, i, &y[3 * i], r, NULL, 0, NULL, 0);
  tmp = (int32_t*)malloc(sizeof(int32_t) * (size_t)(c > 0 ? c : 1));
  gather_row(g, y, i, &y[3 * i], r, NULL, 0, tmp, c);
  int64_t k = 0;
  for (int64_t s = 0; s < c; ++s) {
    if (in_sorted_row(bcol + brow[i], brow[i + 1] - brow[i], tmp[s])) continue;
    if (out && k < cap) out[k] = tmp[s];
    k++;
  }
  free(tmp);
  return k;
}

int64_t pdo_contact_count(int64_t n, const double* y, double r_search, const int64_t* brow,
                          const int32_t* bcol, int32_t* counts) {
  cells_t g;
  cells_build(&g, n, y, r_search);
  int64_t tot = 0;
  for (int64_t i = 0; i < n; ++i) {
    counts[i] = (int32_t)contact_row(&g, y, i, r_search, brow, bcol, NULL, 0);
    tot += counts[i];
  }
  cells_free(&g);
  return tot;
}

void pdo_contact_fill(int64_t n, const double* y, double r_search, const int64_t* brow,
                      const int32_t* bcol, const int64_t* crow, int32_t* ccol) {
  cells_t g;
  cells_build(&g, n, y, r_search);
  for (int64_t i = 0; i < n; ++i)
    contact_row(&g, y, i, r_search, brow, bcol, ccol + crow[i], crow[i + 1] - crow[i]);
  cells_free(&g);
}

/* ---------------------------------------------------------------------------
 * Short-range contact force: ShortRangeForceContactModel::computeForce
 * (src/contact/Peridigm_ShortRangeForceContactModel.cpp:98-261), scatter form,
 * both the friction (:146-244) and the normal-only (:245-255) branches. The
 * horizon in c = 9k/(pi h^4) is the owner's block horizon
 * (ContactManager::initialize, Peridigm_ContactManager.cpp:241-249).
 * ------------------------------------------------------------------------- */
void pdo_contact_force(int64_t n, const double* y, const double* v, const double* vol,
                       const int64_t* crow, const int32_t* ccol, double r_contact,
                       double k_spring, double friction, const double* horizon_pt, double* fc) {
  const double pi = 3.14159265358979323846;
  double rc2 = r_contact * r_contact;
  memset(fc, 0, sizeof(double) * 3 * (size_t)n);
  for (int64_t i = 0; i < n; ++i) {
    if (crow[i + 1] == crow[i]) continue;
    double X[3] = {y[3 * i], y[3 * i + 1], y[3 * i + 2]};
    double V[3] = {v[3 * i], v[3 * i + 1], v[3 * i + 2]};
    double nodeVol = vol[i];
    double h = horizon_pt[i];
    for (int64_t b = crow[i]; b < crow[i + 1]; ++b) {
      int64_t j = ccol[b];
      double d2 = (X[0] - y[3 * j]) * (X[0] - y[3 * j]) + (X[1] - y[3 * j + 1]) * (X[1] - y[3 * j + 1]) +
                  (X[2] - y[3 * j + 2]) * (X[2] - y[3 * j + 2]);
      if (!(d2 < rc2)) continue;
      double dist = dist3(X[0], X[1], X[2], y[3 * j], y[3 * j + 1], y[3 * j + 2]);
      double c = 9.0 * k_spring / (pi * h * h * h * h);
      double temp = c * (r_contact - dist) / h;
      double nbVol = vol[j];
      if (friction != 0.0) {
        double nrm[3], cdn, ndn, cvp[3], nvp[3], vcm[3], cvr[3], nvr[3], ncf[3], nnf[3];
        for (int k = 0; k < 3; ++k) nrm[k] = (y[3 * j + k] - X[k]) / dist;
        cdn = V[0] * nrm[0] + V[1] * nrm[1] + V[2] * nrm[2];
        ndn = v[3 * j] * nrm[0] + v[3 * j + 1] * nrm[1] + v[3 * j + 2] * nrm[2];
        for (int k = 0; k < 3; ++k) {
          cvp[k] = V[k] - cdn * nrm[k];
          nvp[k] = v[3 * j + k] - ndn * nrm[k];
        }
        for (int k = 0; k < 3; ++k) vcm[k] = 0.5 * (cvp[k] + nvp[k]);
        for (int k = 0; k < 3; ++k) {
          cvr[k] = cvp[k] - vcm[k];
          nvr[k] = nvp[k] - vcm[k];
        }
        double ncvr = sqrt(cvr[0] * cvr[0] + cvr[1] * cvr[1] + cvr[2] * cvr[2]);
        double nnvr = sqrt(nvr[0] * nvr[0] + nvr[1] * nvr[1] + nvr[2] * nvr[2]);
        for (int k = 0; k < 3; ++k) {
          ncf[k] = -(temp * nbVol * (y[3 * j + k] - X[k]) / dist);
          nnf[k] = (temp * nodeVol * (y[3 * j + k] - X[k]) / dist);
        }
        double nncf = sqrt(ncf[0] * ncf[0] + ncf[1] * ncf[1] + ncf[2] * ncf[2]);
        double nnnf = sqrt(nnf[0] * nnf[0] + nnf[1] * nnf[1] + nnf[2] * nnf[2]);
        for (int k = 0; k < 3; ++k) {
          double cff = ncvr != 0.0 ? -friction * nncf * cvr[k] / ncvr : 0.0;
          double nff = nnvr != 0.0 ? -friction * nnnf * nvr[k] / nnvr : 0.0;
          fc[3 * i + k] += ncf[k] + cff;
          fc[3 * j + k] += nnf[k] + nff;
        }
      } else {
        for (int k = 0; k < 3; ++k) {
          fc[3 * i + k] -= temp * nbVol * (y[3 * j + k] - X[k]) / dist;
          fc[3 * j + k] += temp * nodeVol * (y[3 * j + k] - X[k]) / dist;
        }
      }
    }
  }
}

/* ---------------------------------------------------------------------------
 * Explicit run: Peridigm::executeExplicit (src/core/Peridigm.cpp:1290-1593)
 * with ModelEvaluator::evalModel's order damage -> force -> contact
 * (src/core/Peridigm_ModelEvaluator.cpp:57-131) and DirichletIncrementBC on
 * the velocity (src/core/Peridigm_BoundaryCondition.cpp:202-241, wired with
 * coeff 0 / deltaTCoeff 1 at Peridigm_BoundaryAndInitialConditionManager.cpp:109-117).
 * ------------------------------------------------------------------------- */
typedef struct {
  int64_t* crow;
  int32_t* ccol;
} contact_list;

static void contact_rebuild(const pdo_explicit* p, const double* y, contact_list* cl) {
  int64_t n = p->n;
  int32_t* counts = (int32_t*)malloc(sizeof(int32_t) * (size_t)(n > 0 ? n : 1));
  pdo_contact_count(n, y, p->r_search, p->row, p->col, counts);
  free(cl->crow);
  free(cl->ccol);
  cl->crow = (int64_t*)malloc(sizeof(int64_t) * (size_t)(n + 1));
  cl->crow[0] = 0;
  for (int64_t i = 0; i < n; ++i) cl->crow[i + 1] = cl->crow[i] + counts[i];
  cl->ccol = (int32_t*)malloc(sizeof(int32_t) * (size_t)(cl->crow[n] > 0 ? cl->crow[n] : 1));
  pdo_contact_fill(n, y, p->r_search, p->row, p->col, cl->crow, cl->ccol);
  free(counts);
}

static void eval_model(const pdo_explicit* p, const double* y, const double* v, const double* m,
                       const double* dmg_n, double* dmg_np1, double* node_damage, double* theta,
                       double* f, double* fc, const contact_list* cl) {
  int64_t n = p->n;
  if (p->damage_on)
    pdo_damage_critical_stretch(n, p->x, y, p->row, p->col, p->s_c, dmg_n, dmg_np1, node_damage);
  else
    memcpy(dmg_np1, dmg_n, sizeof(double) * (size_t)p->row[n]);
  if (p->material == 1) {
    memset(theta, 0, sizeof(double) * (size_t)n);
    pdo_force_bond_based(n, p->x, y, p->vol, dmg_np1, p->row, p->col, p->K, p->horizon, p->plane, p->height, f);
  } else {
    pdo_dilatation(n, p->x, y, m, p->vol, dmg_np1, p->row, p->col, p->influence, p->horizon, theta);
    pdo_force_lps(n, p->x, y, m, p->vol, theta, dmg_np1, p->row, p->col, p->K, p->mu, p->influence,
                  p->horizon, f);
  }
  if (p->contact_on)
    pdo_contact_force(n, y, v, p->vol, cl->crow, cl->ccol, p->r_contact, p->k_spring, p->friction,
                      p->contact_horizon, fc);
  else
    memset(fc, 0, sizeof(double) * 3 * (size_t)n);
}

int pdo_explicit_run(const pdo_explicit* p, double* u, double* v, double* a, double* f,
                     double* fc, double* theta, double* node_damage, double* bond_damage) {
  int64_t n = p->n, nb = p->row[n];
  size_t n3 = 3 * (size_t)n;
  double* y = (double*)malloc(sizeof(double) * (n3 > 0 ? n3 : 1));
  double* m = (double*)malloc(sizeof(double) * (size_t)(n > 0 ? n : 1));
  double* dmg_np1 = (double*)malloc(sizeof(double) * (size_t)(nb > 0 ? nb : 1));
  double* ftot = (double*)malloc(sizeof(double) * (n3 > 0 ? n3 : 1));
  contact_list cl = {NULL, NULL};
  double dt = p->dt, dt2 = dt / 2.0;

  pdo_weighted_volume(n, p->x, p->vol, p->row, p->col, p->influence, p->horizon, m);
  for (size_t k = 0; k < n3; ++k) y[k] = p->x[k] + u[k];
  if (p->contact_on) contact_rebuild(p, y, &cl);

  /* Initial evaluation (Peridigm.cpp:1393-1423); its damage is not committed. */
  eval_model(p, y, v, m, bond_damage, dmg_np1, node_damage, theta, f, fc, &cl);
  for (size_t k = 0; k < n3; ++k) {
    ftot[k] = f[k] + fc[k];
    a[k] = ftot[k];
    a[k] += 0.0;
    a[k] /= p->rho[k / 3];
  }

  double tc = p->t0, tp;
  for (int step = 1; step <= p->nsteps; ++step) {
    tp = tc;
    tc = p->t0 + (step * dt);
    if (p->contact_on && p->search_freq > 0 && step % p->search_freq == 0) contact_rebuild(p, y, &cl);
    for (size_t k = 0; k < n3; ++k) v[k] = v[k] + dt2 * a[k];
    if (p->bc_mask && tc != tp) {
      for (int64_t i = 0; i < n; ++i) {
        if (!p->bc_mask[i]) continue;
        for (int c = 0; c < 3; ++c) {
          if (!(p->bc_mask[i] >> c & 1)) continue;
          const size_t k = 3 * (size_t)i + c;
          double cur, prev;
          if (p->bc_vals) {
            cur = p->bc_vals[(size_t)step * n3 + k];
            prev = p->bc_vals[(size_t)(step - 1) * n3 + k];
          } else {
            cur = p->bc_a[k] * tc + p->bc_b[k];
            prev = p->bc_a[k] * tp + p->bc_b[k];
          }
          /* a zero increment takes the previous value from the displacement
             field (Peridigm_BoundaryCondition.cpp:137-142) */
          if (cur - prev == 0.0) prev = u[k];
          v[k] = 0.0 * (cur - prev) + 1.0 * (cur - prev) * (1.0 / (tc - tp));
        }
      }
    }
    for (size_t k = 0; k < n3; ++k) y[k] = p->x[k] + u[k] + dt * v[k];
    for (size_t k = 0; k < n3; ++k) u[k] = u[k] + dt * v[k];
    eval_model(p, y, v, m, bond_damage, dmg_np1, node_damage, theta, f, fc, &cl);
    for (size_t k = 0; k < n3; ++k) {
      ftot[k] = f[k] + fc[k];
      a[k] = ftot[k];
      a[k] += 0.0;
      a[k] /= p->rho[k / 3];
    }
    for (size_t k = 0; k < n3; ++k) v[k] = v[k] + dt2 * a[k];
    memcpy(bond_damage, dmg_np1, sizeof(double) * (size_t)nb); /* updateState */
  }
  /* f reports the total force density (internal + contact), as the
   * mothership force vector does after Peridigm.cpp:1567. */
  memcpy(f, ftot, sizeof(double) * n3);
  free(y);
  free(m);
  free(dmg_np1);
  free(ftot);
  free(cl.crow);
  free(cl.ccol);
  return 0;
}

/* ---------------------------------------------------------------------------
 * Linearized LPS force (directional derivative of pdo_force_lps along w).
 * With de = Yhat.(w_j - w_p) and dYhat = ((w_j - w_p) - Yhat de)/|Y|:
 *   dtheta_p = sum 3 omega (1-d) zeta de V_j / m_p
 *   dt = (1-d) (omega dtheta_p (3K/m - alpha/3) zeta + (1-d) omega alpha de)
 *   f_p += (dt Yhat + t dYhat) V_j,  f_j -= (dt Yhat + t dYhat) V_p
 * (the scatter of elastic.cxx:119-130 differentiated term by term).
 * ------------------------------------------------------------------------- */
void pdo_lps_jv(int64_t n, const double* x, const double* y, const double* m, const double* vol,
                const double* theta, const double* dmg, const int64_t* row, const int32_t* col,
                const double* K, const double* mu, int influence, double horizon, const double* w,
                double* df) {
  double* dth = (double*)calloc((size_t)(n > 0 ? n : 1), sizeof(double));
  for (int64_t p = 0; p < n; ++p) {
    double acc = 0.0;
    for (int64_t b = row[p]; b < row[p + 1]; ++b) {
      int64_t j = col[b];
      double X[3], Y[3], dw[3];
      for (int k = 0; k < 3; ++k) {
        X[k] = x[3 * j + k] - x[3 * p + k];
        Y[k] = y[3 * j + k] - y[3 * p + k];
        dw[k] = w[3 * j + k] - w[3 * p + k];
      }
      double zeta = sqrt(X[0] * X[0] + X[1] * X[1] + X[2] * X[2]);
      double dY = sqrt(Y[0] * Y[0] + Y[1] * Y[1] + Y[2] * Y[2]);
      double de = (Y[0] * dw[0] + Y[1] * dw[1] + Y[2] * dw[2]) / dY;
      double omega = pdo_influence(influence, zeta, horizon);
      acc += 3.0 * omega * (1.0 - dmg[b]) * zeta * de * vol[j] / m[p];
    }
    dth[p] = acc;
  }
  memset(df, 0, sizeof(double) * 3 * (size_t)n);
  for (int64_t p = 0; p < n; ++p) {
    double alpha = 15.0 * mu[p] / m[p];
    double q = 3.0 * K[p] / m[p] - alpha / 3.0;
    for (int64_t b = row[p]; b < row[p + 1]; ++b) {
      int64_t j = col[b];
      double X[3], Y[3], dw[3];
      for (int k = 0; k < 3; ++k) {
        X[k] = x[3 * j + k] - x[3 * p + k];
        Y[k] = y[3 * j + k] - y[3 * p + k];
        dw[k] = w[3 * j + k] - w[3 * p + k];
      }
      double zeta = sqrt(X[0] * X[0] + X[1] * X[1] + X[2] * X[2]);
      double dY = sqrt(Y[0] * Y[0] + Y[1] * Y[1] + Y[2] * Y[2]);
      double e = dY - zeta;
      double de = (Y[0] * dw[0] + Y[1] * dw[1] + Y[2] * dw[2]) / dY;
      double omega = pdo_influence(influence, zeta, horizon);
      double d1 = 1.0 - dmg[b];
      double c1 = omega * theta[p] * q;
      double t = d1 * (c1 * zeta + d1 * omega * alpha * e);
      double dt = d1 * (omega * dth[p] * q * zeta + d1 * omega * alpha * de);
      for (int k = 0; k < 3; ++k) {
        double yh = Y[k] / dY;
        double dyh = (dw[k] - yh * de) / dY;
        double g = dt * yh + t * dyh;
        df[3 * p + k] += g * vol[j];
        df[3 * j + k] -= g * vol[p];
      }
    }
  }
  free(dth);
}
