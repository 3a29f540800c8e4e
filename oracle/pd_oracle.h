/*
 * CPU oracle for the Peridigm LPS / critical-stretch / Verlet / contact path.
 *
 * TEST INFRASTRUCTURE ONLY. This is a plain-C, FP64 restatement of the
 * reference algorithm, used by tests/, by __graft_entry__.smoke() and by the
 * CPU-baseline leg of bench.py as the checker. The product library never links
 * or calls it.
 *
 * Parity is pinned: tests/test_oracle_golden.py checks these functions against
 * the reference's unit-test known answers (utPeridigm_ElasticMaterial.cpp),
 * against the gold Exodus files of the reference's verification/regression
 * tests (stored as fixtures under tests/golden/), and against the reference's
 * own LPS kernels compiled from its sources into oracle/_ref/libpdref.so.
 *
 * Bond families are CSR: row[n+1] (int64) and col[nb] (int32), each row sorted
 * ascending like the reference's neighbor list (NeighborhoodList.cxx:705).
 * Vectors are interleaved xyz (3*i+k) as in Peridigm's Epetra vectors.
 */
#ifndef PD_ORACLE_H
#define PD_ORACLE_H
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { PDO_INFLUENCE_ONE = 0, PDO_INFLUENCE_PARABOLIC = 1, PDO_INFLUENCE_GAUSSIAN = 2 };

/* Rectangular_Plane bond filter (BondFilter.h FinitePlane, Peridigm_Discretization.cpp:158-175). */
typedef struct {
  double normal[3];
  double lower_left[3];
  double bottom_unit[3];
  double bottom_length;
  double side_length;
} pdo_plane;

double pdo_influence(int kind, double zeta, double horizon);
int pdo_plane_cuts_bond(const pdo_plane* pl, const double* p0, const double* p1);

/* Neighbor search (ZoltanSearchTree::FindPointsWithinRadius + NeighborhoodList +
 * BondFilterDefault/FinitePlaneFilter). Two calls: count fills counts[n]
 * and returns the total; fill writes row/col. */
int64_t pdo_neighbor_count(int64_t n, const double* x, const double* horizon,
                           const pdo_plane* planes, int n_planes, int32_t* counts);
void pdo_neighbor_fill(int64_t n, const double* x, const double* horizon,
                       const pdo_plane* planes, int n_planes, const int64_t* row, int32_t* col);

void pdo_weighted_volume(int64_t n, const double* x, const double* vol, const int64_t* row,
                         const int32_t* col, int influence, double horizon, double* m);
void pdo_damage_critical_stretch(int64_t n, const double* x, const double* y, const int64_t* row,
                                 const int32_t* col, const double* s_c, const double* dmg_n,
                                 double* dmg_np1, double* node_damage);
void pdo_dilatation(int64_t n, const double* x, const double* y, const double* m,
                    const double* vol, const double* dmg, const int64_t* row, const int32_t* col,
                    int influence, double horizon, double* theta);
void pdo_force_bond_based(int64_t n, const double* x, const double* y, const double* vol,
                          const double* dmg, const int64_t* row, const int32_t* col, const double* K,
                          double horizon, int plane, double height, double* f);
void pdo_dilatation_linear_lps(int64_t n, const double* x, const double* y, const double* m, const double* vol,
                               const double* dmg, const int64_t* row, const int32_t* col, int influence,
                               double horizon, double* theta);
void pdo_force_linear_lps(int64_t n, const double* x, const double* y, const double* m, const double* vol,
                          const double* theta, const double* dmg, const int64_t* row, const int32_t* col,
                          const double* K, const double* mu, int influence, double horizon, double* f);
void pdo_force_lps(int64_t n, const double* x, const double* y, const double* m,
                   const double* vol, const double* theta, const double* dmg, const int64_t* row,
                   const int32_t* col, const double* K, const double* mu, int influence,
                   double horizon, double* f);
double pdo_critical_time_step(int64_t n, const double* x, const double* vol, const int64_t* row,
                              const int32_t* col, const double* K, const double* rho,
                              double horizon);

/* Contact search over current coordinates y, excluding every pair that is in
 * the bond family (ContactManager::contactSearch). */
int64_t pdo_contact_count(int64_t n, const double* y, double r_search, const int64_t* brow,
                          const int32_t* bcol, int32_t* counts);
void pdo_contact_fill(int64_t n, const double* y, double r_search, const int64_t* brow,
                      const int32_t* bcol, const int64_t* crow, int32_t* ccol);
void pdo_contact_force(int64_t n, const double* y, const double* v, const double* vol,
                       const int64_t* crow, const int32_t* ccol, double r_contact,
                       double k_spring, double friction, const double* horizon_pt, double* fc);

/* Directional derivative of the LPS force density (the linearization the
 * reference's tangent assembles by automatic differentiation,
 * Peridigm_ElasticMaterial.cpp:258-383): df = (d f / d u) w, scatter form
 * mirroring elastic.cxx. theta, m at the configuration y. */
void pdo_lps_jv(int64_t n, const double* x, const double* y, const double* m, const double* vol,
                const double* theta, const double* dmg, const int64_t* row, const int32_t* col,
                const double* K, const double* mu, int influence, double horizon, const double* w,
                double* df);

/* Whole explicit run (Peridigm::executeExplicit). */
typedef struct {
  int64_t n;
  const double* x;       /* [3n] */
  const double* vol;     /* [n] */
  const double* rho;     /* [n] */
  const double* K;       /* [n] */
  const double* mu;      /* [n] */
  const int64_t* row;    /* [n+1] */
  const int32_t* col;    /* [nb] */
  int influence;
  double horizon;
  int damage_on;
  const double* s_c;     /* [n] critical stretch of the owner */
  int contact_on;
  double r_search;
  int search_freq;
  double r_contact;
  double k_spring;
  double friction;
  const double* contact_horizon; /* [n] horizon of each point's block */
  const uint8_t* bc_mask; /* [n] bit k: coordinate k has a prescribed displacement */
  const double* bc_a;     /* [3n] prescribed displacement u(t) = a*t + b */
  const double* bc_b;     /* [3n] */
  /* [(nsteps+1) x 3n] or NULL: the prescribed displacement of each dof at
   * t0 + k dt (row k), for prescribed values that are not a*t + b (an
   * expression of x, y, z, t evaluated by the caller); replaces bc_a/bc_b */
  const double* bc_vals;
  double dt;
  double t0;
  int nsteps;
  int material;           /* 0: LPS (elastic), 1: elastic bond based */
  int plane;              /* bond based: plane strain/stress constant */
  double height;
} pdo_explicit;

/* State in/out: u, v [3n]; outputs a, f (force density incl. contact), fc,
 * theta, node damage [n], bond damage [nb] (0/1 doubles). */
int pdo_explicit_run(const pdo_explicit* p, double* u, double* v, double* a, double* f,
                     double* fc, double* theta, double* node_damage, double* bond_damage);

#ifdef __cplusplus
}
#endif
#endif
