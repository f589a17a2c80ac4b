/*
 * solfec_b200.h -- drop-in C ABI for Solfec-1.0's contact-solve path on B200.
 *
 * Replaces, one to one:
 *   GAUSS_SEIDEL_Create       bgs.h:114-116 (bgs.c:443-472)   -> b2gs_create
 *   GAUSS_SEIDEL_Solve        bgs.h:119     (bgs.c:913-1069)  -> b2gs_solve
 *   GAUSS_SEIDEL_Failure      bgs.h:122     (bgs.c:1073)      -> b2gs_failure_string
 *   GAUSS_SEIDEL_Diagsolver   bgs.h:125     (bgs.c:1086)      -> b2gs_diagsolver_string
 *   GAUSS_SEIDEL_Error        bgs.h:128     (bgs.c:1100)      -> b2gs_error_string
 *   GAUSS_SEIDEL_Reverse      bgs.h:131     (bgs.c:1114)      -> b2gs_reverse_string
 *   GAUSS_SEIDEL_Variant      bgs.h:134     (bgs.c:1126)      -> b2gs_variant_string
 *   GAUSS_SEIDEL_Write_State  bgs.h:137     (bgs.c:1139)      -> b2gs_write_state
 *   GAUSS_SEIDEL_Destroy      bgs.h:140     (bgs.c:1158)      -> b2gs_destroy
 *   LOCDYN_Create             ldy.h:93      (ldy.c:477)       -> b2gs_locdyn_create
 *   LOCDYN_Update_Begin       ldy.h:103     (ldy.c:626-876)   -> b2gs_locdyn_update_begin
 *   LOCDYN_Destroy            ldy.h:127     (ldy.c:1196)      -> b2gs_locdyn_destroy
 * plus flat accessors for the state the reference keeps in CON records
 * (con->R, con->U, con->merit, dom->merit; dom.h:79-92).
 *
 * The structs here are flat arrays (no linked lists); a Solfec build binds
 * them by walking its LOCDYN/DOM lists once per step.
 * Only CONTACT constraints with SIGNORINI_COULOMB materials on RIG/OBS bodies
 * are on this path; anything else is rejected with B2GS_EUNSUPPORTED.
 */
#ifndef SOLFEC_B200_H
#define SOLFEC_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* GSERROR (bgs.h:31-37) */
enum b2gs_error { B2GS_OK = 0, B2GS_DIVERGED, B2GS_DIAGONAL_DIVERGED, B2GS_DIAGONAL_FAILED };
/* GSFAIL (bgs.h:39-44) */
enum b2gs_failure { B2GS_FAILURE_CONTINUE = 0, B2GS_FAILURE_EXIT, B2GS_FAILURE_CALLBACK };
/* GSONOFF (bgs.h:46-50) */
enum b2gs_onoff { B2GS_OFF = 0, B2GS_ON };
/* GSVARIANT (bgs.h:52-57); the parallel variants only matter for MPI builds */
enum b2gs_variant { B2GS_FULL = 0, B2GS_MIDDLE_JACOBI, B2GS_BOUNDARY_JACOBI };
/* DIAS (dbs.h:27-33) */
enum b2gs_dias { B2GS_PROJECTED_GRADIENT = 0, B2GS_DE_SAXCE_FENG, B2GS_SEMISMOOTH_NEWTON, B2GS_PROJECTED_NEWTON };
/* arithmetic of the sweeps (no reference counterpart: the reference is FP64) */
enum b2gs_precision { B2GS_FP64 = 0, B2GS_MIXED = 1 };

/* THROW codes of a FAILURE_EXIT solve: the reference err.h values */
#define B2GS_ERR_GAUSS_SEIDEL_DIAGONAL_DIVERGED 44
#define B2GS_ERR_GAUSS_SEIDEL_DIVERGED 45

/* negative statuses: device-layer errors (b2_device.h codes) */
#define B2GS_EUNSUPPORTED (-5)

typedef void (*b2gs_callback) (void *data);

typedef struct b2gs_solver b2gs_solver;   /* struct gs (bgs.h:64-111) */
typedef struct b2gs_locdyn b2gs_locdyn;   /* struct locdyn (ldy.h:81-90) + constraint R/U */

/* Rigid bodies (bod.c:53-74): rot[9] column-major rotation, x0[3] referential
 * mass centre, jinv[9] inverse referential inertia (column-major), minv = 1/m,
 * velo[6] = [Omega (referential); v (spatial)] after the free step (t+h),
 * velo0[6] the same at t, obstacle != 0 for OBS bodies. */
typedef struct b2gs_bodies {
  int nbod;
  const double *rot, *x0, *jinv, *minv, *velo, *velo0;
  const int *obstacle;
  int on_device;  /* pointers are device pointers */
} b2gs_bodies;

/* Contacts (dom.h:77-129): master/slave body index (slave -1 = none),
 * referential points mpnt[3]/spnt[3], local frame base[9] (column-major,
 * normal = third column, from slave to master), gap, friction, restitution,
 * and cohesion = SURFACE_MATERIAL_Cohesion_Get(mat) * area (dbs.c:500). */
typedef struct b2gs_contacts {
  int ncon;
  const int *master, *slave;
  const double *mpnt, *spnt, *base, *gap, *friction, *restitution, *cohesion;
  int on_device;
} b2gs_contacts;

/* ---- solver (GAUSS_SEIDEL) ---- */

/* GAUSS_SEIDEL_Create: defaults reverse OFF, variant FULL, nomerit 0,
 * precision FP64. Pass diagepsilon <= 0 / diagmaxiter <= 0 for the defaults
 * the Python constructor applies (lng.c:4335-4342). */
b2gs_solver* b2gs_create (double epsilon, int maxiter, double meritval, int failure,
                          double diagepsilon, int diagmaxiter, int diagsolver,
                          void *data, b2gs_callback callback);

/* GAUSS_SEIDEL_Solve: returns 0; a THROW code (B2GS_ERR_*) when the failure
 * action is EXIT and the reference would have thrown; a negative device
 * status on a device error. */
int b2gs_solve (b2gs_solver *gs, b2gs_locdyn *ldy);

const char* b2gs_failure_string (b2gs_solver *gs);
const char* b2gs_diagsolver_string (b2gs_solver *gs);
const char* b2gs_error_string (b2gs_solver *gs);
const char* b2gs_reverse_string (b2gs_solver *gs);
const char* b2gs_variant_string (b2gs_solver *gs);
void b2gs_destroy (b2gs_solver *gs);

/* GAUSS_SEIDEL_Write_State: the labelled values the reference writes
 * (GSITERS); here written as "GSITERS <iters>\n" into buf. */
int b2gs_write_state (b2gs_solver *gs, char *buf, int buflen);

/* field access (the Python getset table, lng.c:4624-4640) */
int b2gs_get_iters (b2gs_solver *gs);
int b2gs_get_error (b2gs_solver *gs);
const double* b2gs_get_rerhist (b2gs_solver *gs);   /* iters values */
const double* b2gs_get_merhist (b2gs_solver *gs);   /* iters values */
const int* b2gs_get_itershist (b2gs_solver *gs, int *count);
void b2gs_set_itershist (b2gs_solver *gs, int on);  /* itershistcount >= 0 collects */
void b2gs_set_reverse (b2gs_solver *gs, int onoff);
void b2gs_set_variant (b2gs_solver *gs, int variant);
void b2gs_set_nomerit (b2gs_solver *gs, int nomerit);
void b2gs_set_params (b2gs_solver *gs, double epsilon, int maxiter, double meritval, double diagepsilon, int diagmaxiter);
void b2gs_set_precision (b2gs_solver *gs, int precision);
void b2gs_set_grid (b2gs_solver *gs, int blocks);      /* persistent grid size (0 = automatic) */
void b2gs_set_stage_blocks (b2gs_solver *gs, int blocks); /* staging window per warp (0 = automatic) */
/* device options of the next solve (b2dev_solve_opts of b2_device.h), e.g. for b2dev_solve_batch */
struct b2dev_solve_opts;
int b2gs_get_opts (b2gs_solver *gs, struct b2dev_solve_opts *opts);
int b2gs_get_iters_mixed (b2gs_solver *gs);           /* FP32 iterations of the last mixed solve */
double b2gs_get_solve_ms (b2gs_solver *gs);           /* device time of the last solve */
double b2gs_get_merit_input (b2gs_solver *gs);        /* merit of the reactions the last solve started from */
/* the device report of the last solve (struct b2dev_solve_report of b2_device.h) */
int b2gs_get_report (b2gs_solver *gs, void *report, int nbytes);

/* ---- local dynamics (LOCDYN) and constraint state ---- */

b2gs_locdyn* b2gs_locdyn_create (int device, void *stream);
void b2gs_locdyn_destroy (b2gs_locdyn *ldy);

/* LOCDYN_Update_Begin for rigid bodies: update_V_and_B, W_ii, rho, A, free
 * energy and W_ij, then the colour-sorted device layout. New contacts start
 * from R = U = 0 (mem.c:64-86); call b2gs_locdyn_set_state to warm start. */
int b2gs_locdyn_update_begin (b2gs_locdyn *ldy, const b2gs_bodies *bod, const b2gs_contacts *con,
                              double step, int dynamic);

/* LOCDYN_Update_Begin again on the device-resident bodies of the last
 * b2gs_locdyn_update_begin, as moved by b2dev_rigid_step_begin (same contacts:
 * referential points, frames, gaps and materials are kept). */
int b2gs_locdyn_update_begin_resident (b2gs_locdyn *ldy, double step, int dynamic);

/* ---- interchange formats of the local dynamics (host/b2io.c) ---- */

/* LOCDYN_W_MatrixMarket (ldy.c:1005-1052): W as a 3n x 3n coordinate matrix,
 * rows in list order, the diagonal block then the row's off-diagonal blocks
 * in their list order, "%.15g". From host arrays in caller order (W[9n],
 * adjptr[n+1], adjcol[K], Woff[9K]), or from the device after assembly. */
int b2gs_write_w_matrix_market (const char *path, int n, const double *W, const int *adjptr, const int *adjcol,
                                const double *Woff);
int b2gs_locdyn_w_matrix_market (b2gs_locdyn *ldy, const char *path);

/* LOCDYN_Dump (ldy.c:892-1002): one line per row with its spatial point,
 * body ids, frame, W, B, V, U, R ("%.6g"), then " => " each neighbour with
 * the neighbour's blocks summed, neighbours in the reference's dump order.
 * point[3n] (spatial contact points), master_id/slave_id[n] (body ids; -1
 * for none) and base[9n] come from the caller; the device version reads W, B,
 * V, the blocks and the current R, U from the device. */
int b2gs_write_locdyn_dump (const char *path, int n, const double *point, const int *master_id, const int *slave_id,
                            const double *base, const double *W, const double *B, const double *V, const double *U,
                            const double *R, const int *adjptr, const int *adjcol, const double *Woff);
int b2gs_locdyn_dump (b2gs_locdyn *ldy, const char *path, const double *point, const int *master_id,
                      const int *slave_id, const double *base);

/* An assembled local dynamics as the reference solver reads it: rows in list
 * order with W[9], A[9], rho, B[3], V[3], gap, friction, restitution,
 * cohesion; blocks of row i at adjptr[i]..adjptr[i+1]-1 (adjcol = neighbour
 * row, Woff 9 doubles). */
int b2gs_locdyn_set (b2gs_locdyn *ldy, int n, const double *W, const double *A, const double *rho,
                     const double *B, const double *V, const double *gap, const double *friction,
                     const double *restitution, const double *cohesion, const int *adjptr, const int *adjcol,
                     const double *Woff, double free_energy, double step, int dynamic, int on_device);

int b2gs_locdyn_set_state (b2gs_locdyn *ldy, const double *R, const double *U, int on_device);
int b2gs_locdyn_get_state (b2gs_locdyn *ldy, double *R, double *U, double *conmerit, int on_device);
double b2gs_locdyn_merit (b2gs_locdyn *ldy);                    /* dom->merit after the last solve */
int b2gs_locdyn_sizes (b2gs_locdyn *ldy, int *n, long long *nblocks, int *ncolours, double *free_energy);
int b2gs_locdyn_order (b2gs_locdyn *ldy, int *order);           /* caller row swept at each position */
void b2gs_locdyn_set_colour_seed (b2gs_locdyn *ldy, uint64_t seed);
void* b2gs_locdyn_device (b2gs_locdyn *ldy);                    /* its b2dev_ctx (b2_device.h) */
const char* b2gs_last_error (void);

#ifdef __cplusplus
}
#endif

#endif
