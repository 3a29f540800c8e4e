/* CPU restatement of the quasi-static block-Jacobi CG step, for the CPU
 * baseline of the quasi-static solve.
 *
 * TEST / MEASUREMENT INFRASTRUCTURE ONLY: bench.py's cpu_baseline of the
 * quasi-static leg times these functions on the host cores; nothing in the
 * product calls them.
 *
 * The reference assembles the full Sacado AD Jacobian (ElasticMaterial::
 * computeAutomaticDifferentiationJacobian, Peridigm_ElasticMaterial.cpp:258-383)
 * and runs Belos CG on it (Peridigm.cpp:2551-2573) with the "Block 3x3"
 * preconditioner (:1603-1646). Its 2-hop stencil (about 900 neighbors per
 * point) does not fit a 60^3 cube in host memory, so this is the matrix-free
 * restatement of the same operator K = -d(V f)/du of the LPS force:
 * per-bond geometry at the current state, then per product the dilatation
 * increment pass and the force increment pass (gather form, one owner per
 * iteration, the owners split over POSIX threads), the inverse 3x3 diagonal
 * blocks and the CG vector updates. The formulas are those of the LPS linearisation in
 * pd_oracle.c (pdo_lps_jv) arranged per owner.
 *
 * Layout: x, y [3n] model and current coordinates; vol [n]; m [n] weighted
 * volume; theta [n] dilatation at y; K, mu [n]; row [n+1], col [nb]; dmg [nb]
 * (0/1); fixed [n] (bit c: dof c prescribed). Influence function "One".
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <string.h>

/* ---- a minimal parallel for over [0, n) on POSIX threads ---------------- */
static int g_threads = 1;
void pdq_set_threads(int t) { g_threads = t > 0 ? (t > 256 ? 256 : t) : 1; }

typedef void (*range_fn)(int64_t lo, int64_t hi, void* arg, double* red);
typedef struct {
  range_fn fn;
  void* arg;
  int64_t lo, hi;
  double red[4];
} task_t;

static void* run_task(void* p) {
  task_t* t = (task_t*)p;
  t->fn(t->lo, t->hi, t->arg, t->red);
  return NULL;
}

/* Runs fn on T contiguous ranges; red_out[k] (nred <= 4) = sum of the ranges' red[k]. */
static void par_for(int64_t n, range_fn fn, void* arg, double* red_out, int nred) {
  const int T = g_threads;
  task_t tasks[256];
  pthread_t th[256];
  for (int t = 0; t < T; ++t) {
    tasks[t].fn = fn;
    tasks[t].arg = arg;
    tasks[t].lo = n * t / T;
    tasks[t].hi = n * (t + 1) / T;
    memset(tasks[t].red, 0, sizeof(tasks[t].red));
  }
  for (int t = 1; t < T; ++t) pthread_create(&th[t], NULL, run_task, &tasks[t]);
  run_task(&tasks[0]);
  for (int t = 1; t < T; ++t) pthread_join(th[t], NULL);
  for (int k = 0; k < nred; ++k) {
    red_out[k] = 0.0;
    for (int t = 0; t < T; ++t) red_out[k] += tasks[t].red[k];
  }
}

typedef struct {
  int64_t n;
  const int64_t* row;
  const int32_t* col;
  const uint8_t* dmg;
  const double *x, *y, *vol, *m, *theta, *K, *mu;
  const uint8_t* fixed;
  double *g, *gc, *dinv;
  const double* p;
  double *dth, *q, *r, *x_it, *z, *pp, *pw;
  double alpha, beta;
} qs_args;

/* g[4b] = (Y/|Y|, V_j zeta), gc[2b] = (V_j T/|Y|, V_j (alpha_i + alpha_j)),
 * T = zeta (theta_i q_i + theta_j q_j) + (alpha_i + alpha_j) e;
 * q = 3K/m - alpha/3, alpha = 15 mu/m (elastic.cxx:99,119). */
static void geom_range(int64_t lo, int64_t hi, void* a, double* red) {
  const qs_args* A = (const qs_args*)a;
  const int64_t* row = A->row;
  const int32_t* col = A->col;
  const uint8_t* dmg = A->dmg;
  const double *x = A->x, *y = A->y, *vol = A->vol, *m = A->m, *theta = A->theta, *K = A->K, *mu = A->mu;
  double *g = A->g, *gc = A->gc;
  (void)red;
  for (int64_t i = lo; i < hi; ++i) {
    const double ai = 15.0 * mu[i] / m[i], qi = 3.0 * K[i] / m[i] - ai / 3.0;
    for (int64_t b = row[i]; b < row[i + 1]; ++b) {
      double* gb = g + 4 * b;
      double* cb = gc + 2 * b;
      if (dmg[b]) {
        gb[0] = gb[1] = gb[2] = gb[3] = 0.0;
        cb[0] = cb[1] = 0.0;
        continue;
      }
      const int64_t j = col[b];
      const double aj = 15.0 * mu[j] / m[j], qj = 3.0 * K[j] / m[j] - aj / 3.0;
      const double X0 = x[3 * j] - x[3 * i], X1 = x[3 * j + 1] - x[3 * i + 1], X2 = x[3 * j + 2] - x[3 * i + 2];
      const double Y0 = y[3 * j] - y[3 * i], Y1 = y[3 * j + 1] - y[3 * i + 1], Y2 = y[3 * j + 2] - y[3 * i + 2];
      const double zeta = sqrt(X0 * X0 + X1 * X1 + X2 * X2);
      const double dY = sqrt(Y0 * Y0 + Y1 * Y1 + Y2 * Y2);
      const double e = dY - zeta;
      const double T = zeta * (theta[i] * qi + theta[j] * qj) + (ai + aj) * e;
      gb[0] = Y0 / dY;
      gb[1] = Y1 / dY;
      gb[2] = Y2 / dY;
      gb[3] = vol[j] * zeta;
      cb[0] = vol[j] * T / dY;
      cb[1] = vol[j] * (ai + aj);
    }
  }
}

void pdq_bond_geom(int64_t n, const int64_t* row, const int32_t* col, const uint8_t* dmg, const double* x,
                   const double* y, const double* vol, const double* m, const double* theta, const double* K,
                   const double* mu, double* g, double* gc) {
  qs_args A = {0};
  A.n = n, A.row = row, A.col = col, A.dmg = dmg, A.x = x, A.y = y, A.vol = vol, A.m = m, A.theta = theta;
  A.K = K, A.mu = mu, A.g = g, A.gc = gc;
  par_for(n, geom_range, &A, NULL, 0);
}

/* Inverse 3x3 diagonal blocks of K (prescribed rows and columns: identity),
 * dinv [9n] row-major: D_i = -V_i d(f_i)/d(u_i). */
static void bj_range(int64_t lo, int64_t hi, void* a, double* red) {
  const qs_args* Q = (const qs_args*)a;
  const int64_t* row = Q->row;
  const int32_t* col = Q->col;
  const double *g = Q->g, *gc = Q->gc, *vol = Q->vol, *m = Q->m, *K = Q->K, *mu = Q->mu;
  const uint8_t* fixed = Q->fixed;
  double* dinv = Q->dinv;
  (void)red;
  for (int64_t i = lo; i < hi; ++i) {
    const double ai = 15.0 * mu[i] / m[i], qi = 3.0 * K[i] / m[i] - ai / 3.0;
    double D[9] = {0, 0, 0, 0, 0, 0, 0, 0, 0}, hv[3] = {0, 0, 0};
    for (int64_t b = row[i]; b < row[i + 1]; ++b) {
      const double* gb = g + 4 * b;
      const double* cb = gc + 2 * b;
      if (gb[3] == 0.0) continue;
      const int64_t j = col[b];
      const double zeta = gb[3] / vol[j];
      const double aj = 15.0 * mu[j] / m[j], qj = 3.0 * K[j] / m[j] - aj / 3.0;
      const double a = cb[1] + 3.0 * zeta * zeta * vol[j] * (qj / m[j]) * vol[i];  /* dt/de with the neighbor's theta term */
      for (int r = 0; r < 3; ++r) {
        hv[r] += gb[3] * gb[r];
        for (int c = 0; c < 3; ++c) D[3 * r + c] += (a - cb[0]) * gb[r] * gb[c] + (r == c ? cb[0] : 0.0);
      }
    }
    const double s = 3.0 * qi / m[i];
    double A[9];
    for (int r = 0; r < 3; ++r)
      for (int c = 0; c < 3; ++c) A[3 * r + c] = vol[i] * (D[3 * r + c] + s * hv[r] * hv[c]);
    for (int c = 0; c < 3; ++c)
      if ((fixed[i] >> c) & 1)
        for (int k = 0; k < 3; ++k) A[3 * c + k] = A[3 * k + c] = (k == c) ? 1.0 : 0.0;
    const double c00 = A[4] * A[8] - A[5] * A[7], c01 = A[5] * A[6] - A[3] * A[8], c02 = A[3] * A[7] - A[4] * A[6];
    const double id = 1.0 / (A[0] * c00 + A[1] * c01 + A[2] * c02);
    double* o = dinv + 9 * i;
    o[0] = c00 * id;
    o[1] = (A[2] * A[7] - A[1] * A[8]) * id;
    o[2] = (A[1] * A[5] - A[2] * A[4]) * id;
    o[3] = c01 * id;
    o[4] = (A[0] * A[8] - A[2] * A[6]) * id;
    o[5] = (A[2] * A[3] - A[0] * A[5]) * id;
    o[6] = c02 * id;
    o[7] = (A[1] * A[6] - A[0] * A[7]) * id;
    o[8] = (A[0] * A[4] - A[1] * A[3]) * id;
  }
}

void pdq_block_jacobi(int64_t n, const int64_t* row, const int32_t* col, const double* g, const double* gc,
                      const double* vol, const double* m, const double* K, const double* mu, const uint8_t* fixed,
                      double* dinv) {
  qs_args A = {0};
  A.n = n, A.row = row, A.col = col, A.g = (double*)g, A.gc = (double*)gc, A.vol = vol, A.m = m, A.K = K, A.mu = mu;
  A.fixed = fixed, A.dinv = dinv;
  par_for(n, bj_range, &A, NULL, 0);
}

/* q = K p on the free dofs (prescribed rows: q = p, prescribed columns
 * dropped: the passes read p with its prescribed components zeroed, pw). */
static void mask_range(int64_t lo, int64_t hi, void* a, double* red) {
  const qs_args* Q = (const qs_args*)a;
  (void)red;
  for (int64_t i = lo; i < hi; ++i)
    for (int c = 0; c < 3; ++c) Q->pw[3 * i + c] = ((Q->fixed[i] >> c) & 1) ? 0.0 : Q->p[3 * i + c];
}

static void dth_range(int64_t lo, int64_t hi, void* a, double* red) {
  const qs_args* Q = (const qs_args*)a;
  const double *p = Q->pw, *g = Q->g, *m = Q->m, *K = Q->K, *mu = Q->mu;
  (void)red;
  for (int64_t i = lo; i < hi; ++i) {
    double acc = 0.0;
    for (int64_t b = Q->row[i]; b < Q->row[i + 1]; ++b) {
      const double* gb = g + 4 * b;
      const int64_t j = Q->col[b];
      acc += gb[3] * (gb[0] * (p[3 * j] - p[3 * i]) + gb[1] * (p[3 * j + 1] - p[3 * i + 1]) +
                      gb[2] * (p[3 * j + 2] - p[3 * i + 2]));
    }
    const double ai = 15.0 * mu[i] / m[i], qi = 3.0 * K[i] / m[i] - ai / 3.0;
    Q->dth[i] = 3.0 * (qi / m[i]) * acc; /* q_i times the dilatation increment */
  }
}

/* red[0] += p.q */
static void df_range(int64_t lo, int64_t hi, void* a, double* red) {
  const qs_args* Q = (const qs_args*)a;
  const double *p = Q->pw, *g = Q->g, *gc = Q->gc, *dth = Q->dth;
  double pq = 0.0;
  for (int64_t i = lo; i < hi; ++i) {
    double d[3] = {0.0, 0.0, 0.0};
    for (int64_t b = Q->row[i]; b < Q->row[i + 1]; ++b) {
      const double* gb = g + 4 * b;
      const double* cb = gc + 2 * b;
      const int64_t j = Q->col[b];
      const double w0 = p[3 * j] - p[3 * i], w1 = p[3 * j + 1] - p[3 * i + 1], w2 = p[3 * j + 2] - p[3 * i + 2];
      const double de = gb[0] * w0 + gb[1] * w1 + gb[2] * w2;
      const double sy = gb[3] * (dth[i] + dth[j]) + (cb[1] - cb[0]) * de;
      d[0] += sy * gb[0] + cb[0] * w0;
      d[1] += sy * gb[1] + cb[0] * w1;
      d[2] += sy * gb[2] + cb[0] * w2;
    }
    for (int c = 0; c < 3; ++c) {
      const double qv = ((Q->fixed[i] >> c) & 1) ? Q->p[3 * i + c] : -Q->vol[i] * d[c];
      Q->q[3 * i + c] = qv;
      pq += Q->p[3 * i + c] * qv;
    }
  }
  red[0] = pq;
}

static double tangent(qs_args* A, const double* p) {
  double pq = 0.0;
  A->p = p;
  par_for(A->n, mask_range, A, NULL, 0);
  par_for(A->n, dth_range, A, NULL, 0);
  par_for(A->n, df_range, A, &pq, 1);
  return pq;
}

void pdq_tangent(int64_t n, const int64_t* row, const int32_t* col, const double* g, const double* gc,
                 const double* vol, const double* m, const double* K, const double* mu, const uint8_t* fixed,
                 const double* p, double* dth, double* q) {
  qs_args A = {0};
  A.n = n, A.row = row, A.col = col, A.g = (double*)g, A.gc = (double*)gc, A.vol = vol, A.m = m, A.K = K, A.mu = mu;
  A.fixed = fixed, A.dth = dth, A.q = q, A.pw = dth + n; /* dth: 4n doubles (increments, masked p) */
  tangent(&A, p);
}

/* z = D^-1 r; with alpha != 0 first x += alpha p, r -= alpha q; red = (r.z, r.r) */
static void precond_range(int64_t lo, int64_t hi, void* a, double* red) {
  const qs_args* Q = (const qs_args*)a;
  double rz = 0.0, rr = 0.0;
  for (int64_t i = lo; i < hi; ++i) {
    if (Q->alpha != 0.0)
      for (int c = 0; c < 3; ++c) {
        Q->x_it[3 * i + c] += Q->alpha * Q->pp[3 * i + c];
        Q->r[3 * i + c] -= Q->alpha * Q->q[3 * i + c];
      }
    const double* d = Q->dinv + 9 * i;
    const double* r = Q->r + 3 * i;
    for (int c = 0; c < 3; ++c) {
      const double zc = d[3 * c] * r[0] + d[3 * c + 1] * r[1] + d[3 * c + 2] * r[2];
      Q->z[3 * i + c] = zc;
      rz += r[c] * zc;
      rr += r[c] * r[c];
    }
  }
  red[0] = rz;
  red[1] = rr;
}

/* p = z + beta p (beta = 0: p = z) */
static void update_p_range(int64_t lo, int64_t hi, void* a, double* red) {
  const qs_args* Q = (const qs_args*)a;
  (void)red;
  for (int64_t k = 3 * lo; k < 3 * hi; ++k) Q->pp[k] = Q->z[k] + Q->beta * Q->pp[k];
}

/* `iters` iterations of block-Jacobi preconditioned CG on K x = r, from x = 0
 * (r is overwritten with the residual, x with the iterate); work [13n]
 * scratch. Returns the last relative residual |r|/|r0|. */
double pdq_bj_cg(int64_t n, const int64_t* row, const int32_t* col, const double* g, const double* gc,
                 const double* vol, const double* m, const double* K, const double* mu, const uint8_t* fixed,
                 const double* dinv, double* r, double* x, int iters, double* work) {
  const int64_t nn = 3 * n;
  qs_args A = {0};
  A.n = n, A.row = row, A.col = col, A.g = (double*)g, A.gc = (double*)gc, A.vol = vol, A.m = m, A.K = K, A.mu = mu;
  A.fixed = fixed, A.dinv = (double*)dinv, A.r = r, A.x_it = x;
  A.z = work, A.pp = work + nn, A.q = work + 2 * nn, A.dth = work + 3 * nn, A.pw = work + 3 * nn + n;
  memset(x, 0, sizeof(double) * (size_t)nn);
  double red[2];
  A.alpha = 0.0;
  par_for(n, precond_range, &A, red, 2);
  double rz = red[0];
  const double r0 = red[1];
  A.beta = 0.0;
  memset(A.pp, 0, sizeof(double) * (size_t)nn);
  par_for(n, update_p_range, &A, NULL, 0);
  double rel = 1.0;
  for (int it = 0; it < iters && r0 > 0.0; ++it) {
    const double pq = tangent(&A, A.pp);
    if (!(pq > 0.0)) break;
    A.alpha = rz / pq;
    par_for(n, precond_range, &A, red, 2);
    rel = sqrt(red[1] / r0);
    if (!(red[0] > 0.0)) break;  /* converged to zero */
    A.beta = red[0] / rz;
    rz = red[0];
    par_for(n, update_p_range, &A, NULL, 0);
  }
  return rel;
}
