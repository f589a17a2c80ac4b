/*
 * oracle.h -- TEST INFRASTRUCTURE. Not part of the product.
 *
 * CPU restatement of the reference contact-solve hot path, used only as the
 * checker by tests/, __graft_entry__.smoke() and the cpu_baseline leg of
 * bench.py. The product (solfec-1.0_b200/) never links or calls it.
 *
 * Pinning: the restated solver is compared against the reference's own
 * GAUSS_SEIDEL_Solve compiled from its sources (oracle/_ref, built by
 * oracle/Makefile) and against committed golden vectors produced by that build
 * (tests/golden/, script tests/golden/make_golden.py).
 *
 * Layout conventions (shared with the product's C ABI):
 *  - 3x3 matrices are column-major, A[3*j+i] = A(i,j) (alg.h:948-953);
 *  - row arrays are indexed by row (contact) in the caller's list order;
 *  - off-diagonal blocks of row i are adjptr[i]..adjptr[i+1]-1 with the
 *    neighbour row in adjcol[] and the 9 entries of W_ij in Woff[9*k..].
 */
#ifndef ORC_ORACLE_H
#define ORC_ORACLE_H

#include <stdint.h>

/* reference THROW codes (err.h enum values) reported by a FAILURE_EXIT solve */
#define ORC_ERR_GAUSS_SEIDEL_DIAGONAL_DIVERGED 44
#define ORC_ERR_GAUSS_SEIDEL_DIVERGED 45

/* Restatement of the serial GAUSS_SEIDEL_Solve (bgs.c:913-1069) over a flat
 * local-dynamics description; same argument list as ref_gs_solve in
 * oracle/ref/ref_harness.c so a test can call either. Returns 0, or the THROW
 * code a FAILURE_EXIT solve raised. */
int orc_gs_solve (int n, const int *adjptr, const int *adjcol, const double *Woff,
                  const double *W, const double *A, const double *rho, const double *B, const double *V,
                  const double *gap, const double *friction, const double *restitution, const double *cohesion,
                  double *R, double *U, double *conmerit,
                  double free_energy, int dynamic, double step,
                  double epsilon, int maxiter, double meritval, int failure,
                  double diagepsilon, int diagmaxiter, int diagsolver, int reverse,
                  int *out_iters, int *out_error, double *out_merit,
                  double *rerhist, double *merhist, int *out_ncallbacks);

/* Restatement of MERIT_Function (mrf.c:35-185) with update_U = 1: recomputes U
 * for every row and returns the merit value; conmerit (may be NULL) receives
 * the per-constraint merit. */
double orc_merit (int n, const int *adjptr, const int *adjcol, const double *Woff,
                  const double *W, const double *A, const double *B, const double *V,
                  const double *gap, const double *friction, const double *restitution, const double *cohesion,
                  const double *R, double *U, double *conmerit, double free_energy, int dynamic, double step);

/* One diagonal block solve (dbs.c:492-550, CONTACT + SIGNORINI_COULOMB). */
int orc_diagonal_solve (int diagsolver, double diagepsilon, int diagmaxiter, int dynamic, double step,
                        double friction, double restitution, double cohesion, double gap, double rho,
                        const double *W, const double *B, const double *V, double *U, double *R);

/* ---------------- local dynamics assembly (ldy.c, bod.c) ---------------- */

/* Number of off-diagonal blocks LOCDYN_Insert (ldy.c:492-568) creates for the
 * contact list: per row, per non-obstacle body of the row, one block per other
 * row touching that body. Fills adjptr[ncon+1]. */
int64_t orc_count_blocks (int nbod, const int *obstacle, int ncon, const int *master, const int *slave, int *adjptr);

/* Restatement of update_V_and_B (ldy.c:364-474) and LOCDYN_Update_Begin
 * (ldy.c:626-876) for rigid bodies and obstacles (bod.c:216-258,1817-1871).
 * Body arrays: rot[9] (column-major rotation), x0[3] (referential mass centre),
 * jinv[9] (inverse referential inertia), minv (1/mass), velo[6] ([Omega; v] at
 * t+h after the free step) and velo0[6] (at t), obstacle flag.
 * Contact arrays: master, slave (-1 = none), mpnt[3]/spnt[3] referential
 * points, base[9] local frame (normal = third column).
 * Outputs per row W[9], A[9], rho, B[3], V[3]; blocks adjcol, adjbod (shared
 * body), Woff[9] in the order adjptr from orc_count_blocks; free energy.
 * Block order inside a row: master-body neighbours then slave-body neighbours,
 * each by ascending row index. Returns 0, or -1 for an unsupported input
 * (self-contact master == slave). */
int orc_assemble (int nbod, const double *rot, const double *x0, const double *jinv, const double *minv,
                  const double *velo, const double *velo0, const int *obstacle,
                  int ncon, const int *master, const int *slave, const double *mpnt, const double *spnt,
                  const double *base, double step,
                  double *W, double *A, double *rho, double *B, double *V, double *free_energy,
                  const int *adjptr, int *adjcol, int *adjbod, double *Woff);

/* ---------------- contact-graph colouring ---------------- */

/* Counter-based priority of row i for a colouring seed (shared definition with
 * the device Jones-Plassmann kernel). */
uint64_t orc_jp_priority (uint64_t seed, int i);
int orc_colour_ordered (int n, const int *adjptr, const int *adjcol, const int *order, int maxcolours, int *colour);

/* Greedy colouring in decreasing priority order: each row takes the smallest
 * colour not used by an already coloured neighbour. This is the fixed point of
 * Jones-Plassmann with smallest-available-colour selection, so the device
 * kernel must reproduce it bit for bit. Returns the number of colours, or -1
 * when more than maxcolours are needed. */
int orc_colour (int n, const int *adjptr, const int *adjcol, uint64_t seed, int maxcolours, int *colour);

/* ---------------- sphere contact update and detection (oracle_detect.c) ---------------- */

/* gjk_sphere_sphere (gjk.c:560-584): gap of two spheres and their closest points. */
double orc_gjk_sphere_sphere (const double *a, double ra, const double *b, double rb, double *p, double *q);

/* localbase (dom.c:133-151): column-major frame with the normal as third column. */
void orc_localbase (const double *n, double *loc);

/* Current sphere centres: BODY_Cur_Point of the referential centres (bod.c:1702-1716). */
void orc_sphere_centres (int nsph, const int *sbody, const double *sref, const double *rot, const double *x,
                         const double *x0, double *cur);

/* The contact part of DOM_Update_Begin for spheres (see oracle_detect.c): the
 * previous contacts (key = i << 32 | j of the sphere pair, i < j; slave_lo = 1
 * when sphere i is the slave; their R and U, may be NULL) are updated with
 * their roles kept, new pairs are detected, new contacts with duplicate points
 * are sparsified. mat[2 * (s1 * nsurf + s2) + {0, 1}] = friction, restitution.
 * Returns the number of contacts (those beyond cap are counted, not written),
 * or -1 for two coincident sphere centres. */
int orc_detect_spheres (int nsph, const int *sbody, const double *sref, const double *rad, const int *surf,
                        int nbod, const double *rot, const double *x, const double *x0, const int *obst,
                        int nsurf, const double *mat,
                        int nprev, const long long *prevkey, const int *prevslave_lo, const double *prevR,
                        const double *prevU, int cap,
                        long long *key, int *slave_lo, int *master, int *slave, double *point, double *mpnt,
                        double *spnt, double *base, double *gap, double *friction, double *restitution,
                        double *R0, double *U0, int *isnew);

/* gjk_convex_point (gjk.c:510-556): distance from p to the hull of the na
 * vertices a[3 na], nearest hull point q. */
double orc_gjk_convex_point (const double *a, int na, const double *p, double *q);

/* gjk (gjk.c:340-391): distance of the hulls of two vertex sets, nearest points
 * p (on a) and q (on b). */
double orc_gjk_polytopes (const double *a, int na, const double *b, int nb, double *p, double *q);

/* computeplanes (cvx.c:72-89) with CONVEX_Planes' layout (cvx.c:1412-1427):
 * per face its unit normal and its first vertex, pla[6 nfac]. */
void orc_convex_planes (int nfac, const int *fac, const double *cur, double *pla);

/* orc_detect_spheres with convex obstacles as well: per convex c its body,
 * referential vertices cvert[3 (cvptr[c] .. cvptr[c+1]-1)], faces fac[cfptr[c] ..]
 * (per face its vertex count, then the convex's vertex indices) and a surface
 * id per face csurf[csptr[c] .. csptr[c+1]-1]. A sphere i and convex c form the
 * pair key i << 32 | (nsph + c) (detect_convex_sphere, goc.c:308-349; the
 * convex is the slave). Returns -2 for a convex without surface faces. */
int orc_detect (int nsph, const int *sbody, const double *sref, const double *rad, const int *surf,
                int nconv, const int *cbody, const int *cvptr, const double *cvert, const int *cfptr, const int *fac,
                const int *csptr, const int *csurf,
                int nbod, const double *rot, const double *x, const double *x0, const int *obst,
                int nsurf, const double *mat,
                int nprev, const long long *prevkey, const int *prevslave_lo, const double *prevR,
                const double *prevU, int cap,
                long long *key, int *slave_lo, int *master, int *slave, double *point, double *mpnt,
                double *spnt, double *base, double *gap, double *friction, double *restitution,
                double *R0, double *U0, int *isnew);

#endif
