/*
 * b2_device.h -- thin C ABI of the sm_100a device layer (libsolfec_b200.so).
 *
 * The host code in C (solfec-1.0_b200/host/b2gs.c, declared in solfec_b200.h)
 * drives the GPU only through these entry points: plain pointers, sizes and
 * integer status codes, no C++ or torch types. Every function returns
 * B2DEV_OK (0) or a negative B2DEV_E* code; b2dev_last_error() gives the text.
 *
 * A context holds one local-dynamics problem resident in HBM in the layout the
 * kernels stream (rows sorted by colour, 3x3 off-diagonal blocks in a CSR of
 * nine coefficient planes, R/U double-buffered), plus the CUDA stream all its
 * work is queued on. It is the device mirror of the reference LOCDYN (ldy.h:81-90)
 * together with the R/U state of its constraints (dom.h:79-81).
 *
 * Pointer arguments are host pointers unless the call takes an `on_device`
 * flag that is non-zero, in which case they are device pointers on the
 * context's device.
 */
#ifndef B2_DEVICE_H
#define B2_DEVICE_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum b2dev_status {
  B2DEV_OK = 0,
  B2DEV_EINVAL = -1,        /* invalid argument or size */
  B2DEV_ECUDA = -2,         /* CUDA runtime error (out of memory, launch failure) */
  B2DEV_ETIMEOUT = -3,      /* a bounded device-side wait gave up */
  B2DEV_ECOLOURS = -4,      /* the contact graph needs more colours than supported */
  B2DEV_EUNSUPPORTED = -5,  /* input outside the rigid contact path (e.g. self-contact) */
  B2DEV_ESTATE = -6         /* call out of order (e.g. solve before assembly) */
};

enum b2dev_precision { B2DEV_FP64 = 0, B2DEV_MIXED = 1 };

typedef struct b2dev_ctx b2dev_ctx;

/* Options of one solve; meaning as struct gs (bgs.h:64-111). */
typedef struct b2dev_solve_opts {
  double epsilon, meritval, diagepsilon;
  int maxiter, diagmaxiter, diagsolver, failure, reverse, nomerit;
  int precision;   /* b2dev_precision; MIXED = FP32 off-diagonal sweeps + closing FP64 refinement */
  int grid;        /* persistent grid size in blocks; 0 = chosen from occupancy and size */
  int stage_blocks; /* off-diagonal blocks staged per warp window; 0 = the largest tile if it fits */
} b2dev_solve_opts;

/* Outcome of one solve. Histories are written to caller buffers of maxiter. */
typedef struct b2dev_solve_report {
  int iters;                /* iterations (gs->iters) */
  int thrown;               /* FAILURE_EXIT raised (reference THROW) */
  int last_fail_kind;       /* 0 none, 1 DIAGONAL_DIVERGED, 2 DIAGONAL_FAILED (last failing row) */
  int nfailures;            /* diagonal failures over the returned iterations */
  int sweeps;               /* sweeps run (includes discarded speculative sweeps) */
  int iters_mixed;          /* iterations spent in FP32 sweeps (mixed precision) */
  double merit;             /* merit of the returned iterate (dom->merit) */
  double error;             /* relative error of the returned iterate */
  double merit_input;       /* merit of the initial reactions (0 without merit) */
  float ms_device;          /* device time of the solve (CUDA events) */
  float ms_kernel[2];       /* solver kernel time per launch: [0] FP64 or mixed FP32 phase, [1] FP64 refinement */
  int sweeps_launch[2];     /* sweeps run by each launch */
  int grid;                 /* persistent grid size (blocks) of the last launch */
} b2dev_solve_report;

const char* b2dev_last_error(void);

/* Create a context on a CUDA device; stream may be NULL (a stream is created)
 * or a cudaStream_t to queue all work on. */
b2dev_ctx* b2dev_create(int device, void* stream);
void b2dev_destroy(b2dev_ctx* ctx);
void* b2dev_stream(b2dev_ctx* ctx);

/* Rigid bodies and contacts of one step (layout documented in solfec_b200.h,
 * b2gs_bodies / b2gs_contacts). */
int b2dev_upload_scene(b2dev_ctx* ctx, int nbod, const double* rot, const double* x0, const double* jinv,
                       const double* minv, const double* velo, const double* velo0, const int* obstacle,
                       int ncon, const int* master, const int* slave, const double* mpnt, const double* spnt,
                       const double* base, const double* gap, const double* friction, const double* restitution,
                       const double* cohesion, int on_device);

/* LOCDYN_Update_Begin: assemble W_ii, A, rho, B, V, free energy and the
 * off-diagonal blocks of the uploaded scene, colour the contact graph and lay
 * the rows out colour by colour. */
int b2dev_assemble(b2dev_ctx* ctx, double step, int dynamic, uint64_t colour_seed);

/* Rigid time integration on either side of the solve (bod.c:1313-1493,
 * BODY_Dynamic_Step_Begin / BODY_Dynamic_Step_End for RIG and OBS bodies): the
 * uploaded body arrays (rotation, velocities) are updated in place, so the
 * next b2dev_assemble reads them without a host round trip.
 *   b2dev_rigid_setup: referential inertia J[9] (column-major), mass, current
 *     mass centre x[3] and scheme per body (0 = RIG_POS, 1 = RIG_NEG, the
 *     reference's default, 2 = RIG_IMP, NEW3's Newton solve of bod.c:163-209;
 *     NULL = all RIG_NEG). A failed NEW3 solve (singular Jacobian, or 50
 *     Newton steps, where the reference stops the program) is reported by
 *     the next b2dev_rigid_step_begin or b2dev_rigid_get.
 *   b2dev_rigid_flags: BODY_* flags per body (bod.h:140-152); BODY_DISABLE_ROTATION
 *     (4) zeroes the angular velocity at both ends of the step (bod.c:1337-1340,
 *     1450-1453); NULL clears them.
 *   b2dev_rigid_step_begin: velo0 <- velo, half step of position and rotation,
 *     free velocity with gravity (m g) and the bodies' point loads at
 *     t + step/2 (loads: [nbod][9] linear force, spatial torque, referential
 *     torque, as rig_point_forces_accumulate sums them; NULL = none).
 *   b2dev_rigid_step_end: the reactions of the last solve (rig_constraints_force; a scene
 *     without contacts needs no solve),
 *     velocity, second half step, rotation update of the scheme.
 *   b2dev_rigid_get: rot[9], x[3], velo[6], velo0[6] per body (any may be NULL). */
int b2dev_rigid_setup(b2dev_ctx* ctx, const double* J, const double* mass, const double* x, const int* scheme,
                      int on_device);
int b2dev_rigid_flags(b2dev_ctx* ctx, const int* flags, int on_device);
int b2dev_rigid_step_begin(b2dev_ctx* ctx, double step, const double* gravity, const double* loads, int on_device);
int b2dev_rigid_step_end(b2dev_ctx* ctx, double step);
int b2dev_rigid_get(b2dev_ctx* ctx, double* rot, double* x, double* velo, double* velo0, int on_device);

/* The bilateral constraints' part of DOM_Update_Begin (dom.c:3716-3732) on
 * the device bodies, after b2dev_rigid_step_begin and before the assembly:
 * RIGLNK rows get base, gap and the solver's local link vector Z[0..2] from
 * the current link (update_riglnk, dom.c:524-550; Z[3] is the link length);
 * FIXDIR rows with a slave body move their master point under the slave's
 * and take the base from the master's current image of the referential
 * direction in Z[0..2] (update_fixdir, dom.c:487-500). A row without a
 * slave (slave < 0) links to the spatial point spnt. The other kinds and
 * contacts are left as they are. Needs b2dev_rigid_setup; does nothing
 * before b2dev_set_kinds has given bilateral rows. */
int b2dev_update_constraints(b2dev_ctx* ctx);

/* Bilateral constraints of a scene with contact detection (the reference's
 * FIX_POINT, FIX_DIRECTION, SET_VELOCITY, PUT_RIGID_LINK: dom.c:3272-3427),
 * n of them with kind 1-5 (dom.h:98), master and slave body (slave -1: none,
 * spnt then a spatial point), referential points mpnt[3]/spnt[3], base[9]
 * (FIXPNT the identity, FIXDIR and VELODIR the frame of the direction,
 * VELODIR3 the caller's frame; RIGLNK and FIXDIR with a slave are refreshed
 * by b2dev_update_constraints) and Z[4] as b2dev_set_kinds takes it (RIGLNK:
 * Z[3] the link length; FIXDIR with a slave: Z[0..2] the master's
 * referential direction). Host arrays. Every b2dev_detect_spheres lists them
 * after the detected contacts (rows ncon .. ncon + n - 1 of the local
 * dynamics, ncon as it reports), with their kinds set and their reactions
 * carried from the previous detection; b2dev_get_contacts and
 * b2dev_get_contact_area list the contacts only. Calling it again replaces
 * them (n = 0 removes them); uploading a scene removes them. */
int b2dev_constraints_setup(b2dev_ctx* ctx, int n, const int* kind, const int* master, const int* slave,
                            const double* mpnt, const double* spnt, const double* base, const double* Z);

/* Contact update and detection between spheres held by the uploaded bodies:
 * the contact part of DOM_Update_Begin (dom.c:3700-3790) for sphere pairs, on
 * the device bodies (rotation of b2dev_upload_scene, mass centre of
 * b2dev_rigid_setup, both as moved by the b2dev_rigid_* steps).
 *   b2dev_spheres_setup: per sphere its body, referential centre[3], radius
 *     and surface id (0 .. nsurf-1; with nsph = 0 the arrays may be NULL); material[2 * (s1 * nsurf + s2) + {0, 1}]
 *     = friction, restitution of a surface pair (SPSET_Find resolved by the
 *     caller; the table must be symmetric; host memory).
 *   b2dev_detect_spheres: the contacts of the last detection are updated with
 *     their master and slave kept (update_contact, dom.c:430-484) and dropped
 *     where the spheres separated; every other pair of spheres of different
 *     bodies, not both obstacles, whose gap (gjk.c:560-584) is below
 *     GEOMETRIC_EPSILON becomes a new contact (detect_sphere_sphere,
 *     goc.c:421-456; insert_contact, dom.c:315-330), and so does every sphere
 *     within r + GEOMETRIC_EPSILON of a convex of b2dev_convexes_setup
 *     (detect_convex_sphere, goc.c:308-349); new contacts with a
 *     duplicate point are removed (sparsify_contacts, dom.c:2956-3054). The
 *     result replaces the scene's contacts, listed by pair (sphere i, then its
 *     partner j > i, a convex c counting as nsph + c) ascending; *ncon and *nnew (either may be NULL) receive the number of
 *     contacts and of new ones. Updated contacts carry their R and U from the
 *     last solve, new ones start from zero.
 *   b2dev_detect_carry_state: after b2dev_assemble of the detected contacts,
 *     sets the solver state to the carried R and U (b2dev_set_state).
 *   b2dev_get_contacts: the detected contacts (any pointer may be NULL):
 *     bodies, spatial point[3], referential points[3], base[9], gap, friction,
 *     restitution, sphere-pair key (i << 32 | j), slave_lo (1 when sphere i is
 *     the slave), new flag, carried R[3] and U[3].
 *   b2dev_sphere_centres: the current sphere centres[3] of the last detection. */
int b2dev_spheres_setup(b2dev_ctx* ctx, int nsph, const int* body, const double* centre, const double* radius,
                        const int* surface, int nsurf, const double* material, int on_device);
int b2dev_detect_spheres(b2dev_ctx* ctx, int* ncon, int* nnew);
/* Convex obstacles (and other convex shapes) the spheres collide with
 * (detect_convex_sphere, goc.c:308-349; the convex is the slave): per convex c
 * its body, referential vertices vert[3 (vptr[c] .. vptr[c+1]-1)], faces
 * fac[fptr[c] ..] (per face its vertex count, then indices into the convex's
 * vertices, counter-clockwise seen from outside) and a surface id per face
 * surf[sptr[c] .. sptr[c+1]-1] (-INT_MAX marks internal faces, as MESH_Convex
 * does). A sphere i and a convex c form the pair key i << 32 | (nsph + c).
 * Host memory; validated here. nconv = 0 removes them. */
int b2dev_convexes_setup(b2dev_ctx* ctx, int nconv, const int* body, const int* vptr, const double* vert,
                         const int* fptr, const int* fac, const int* sptr, const int* surf);
/* Convex-convex contacts (detect_convex_convex and update_convex_convex,
 * goc.c:280-306 and 527-553, with cvi.c, hul.c and tri.c): b2dev_detect_spheres
 * also pairs the convexes of b2dev_convexes_setup with one another (bodies
 * different, not both obstacles; a convex c counts as object nsph + c, the
 * pair key is (nsph + c1) << 32 | (nsph + c2) with c1 < c2). The lower convex
 * is the reference's first object: the slave, whose outward normal the
 * contact takes. Each pair is one contact at the area centre of the surface of
 * the two convexes' intersection, with its normal, gap, area and surface pair;
 * a pair with more than 32 face planes together is an error. Convexes of one
 * body within GEOMETRIC_EPSILON of each other when set up are adjacent
 * (cvx.c:575-589) for the sparsification.
 *   b2dev_contact_sparsify: CONTACT_SPARSIFY (lng.c:8875-8899) threshold in
 *     [0, 1] (default 0.01), minarea >= 0 (0), mindist >= 0
 *     (GEOMETRIC_EPSILON), used by sparsify_contacts (dom.c:2956-3054): a new
 *     contact of area below minarea goes; one of area below threshold times
 *     that of another contact of the same two bodies goes when their objects
 *     are adjacent; otherwise one within 2 mindist (max-norm) of another
 *     contact's point goes when that one is old or later in key order.
 *   b2dev_get_contact_area: the area of every detected contact (1 for sphere
 *     contacts, goc.c:341 and 436). */
int b2dev_contact_sparsify(b2dev_ctx* ctx, double threshold, double minarea, double mindist);
/* Detection controls of the reference's Python interface:
 *   b2dev_exclude_bodies: CONTACT_EXCLUDE_BODIES (lng.c:8817-8852): body pairs
 *     pairs[2k], pairs[2k+1] (0 .. nbod-1) never make contacts (the nobody set
 *     of the broad-phase filter, box.c:116-118); replaces earlier pairs.
 *   b2dev_exclude_surfaces: CONTACT_EXCLUDE_SURFACES (lng.c:8855-8872): no new
 *     contact is created for the surface pairs (either order; dom.c:379-389);
 *     contacts that exist are updated as before. Replaces earlier pairs.
 *   b2dev_unphysical_penetration: UNPHYSICAL_PENETRATION (lng.c:9175-9191),
 *     depth > 0: a detection that finds a contact with gap <= -depth fails with
 *     an error, where the reference stops (dom.c:374, 461, 3792). */
int b2dev_exclude_bodies(b2dev_ctx* ctx, int npairs, const int* pairs);
int b2dev_exclude_surfaces(b2dev_ctx* ctx, int npairs, const int* pairs);
int b2dev_unphysical_penetration(b2dev_ctx* ctx, double depth);
int b2dev_get_contact_area(b2dev_ctx* ctx, double* area, int on_device);
int b2dev_detect_carry_state(b2dev_ctx* ctx);
int b2dev_get_contacts(b2dev_ctx* ctx, int* master, int* slave, double* point, double* mpnt, double* spnt,
                       double* base, double* gap, double* friction, double* restitution, long long* key,
                       int* slave_lo, int* isnew, double* R0, double* U0, int on_device);
int b2dev_sphere_centres(b2dev_ctx* ctx, double* cur, int on_device);

/* Load an already assembled local dynamics (rows in caller order, blocks of
 * row i at adjptr[i]..adjptr[i+1]-1, Woff 9 doubles per block), colour it and
 * lay it out; the same data the reference solver reads from LOCDYN. */
int b2dev_upload_locdyn(b2dev_ctx* ctx, int n, const double* W, const double* A, const double* rho,
                        const double* B, const double* V, const double* gap, const double* friction,
                        const double* restitution, const double* cohesion, const int* adjptr, const int* adjcol,
                        const double* Woff, double free_energy, double step, int dynamic, uint64_t colour_seed,
                        int on_device);

/* Constraint kinds of the current problem's rows (caller order), as dom.h:98
 * numbers them: 0 CONTACT, 1 FIXPNT, 2 FIXDIR, 3 VELODIR, 4 VELODIR3, 5 RIGLNK
 * (SPRING, whose force comes from a Python callback, is not supported). The
 * solve treats them as DIAGONAL_BLOCK_Solver (dbs.c:328-550) and
 * MERIT_Function (mrf.c:88-137) do. Z[4 i ..] per row: VELODIR the prescribed
 * normal velocity Z[0]; VELODIR3 the prescribed velocity Z[0..2]; RIGLNK the
 * link vector in the row's local frame (base^T Z, as riglnk computes it) in
 * Z[0..2] and the link length in Z[3]; the row's gap is RIGLNK's merit gap. n
 * must be the problem's row count; kind NULL makes every row a contact again.
 * Uploading a scene or local dynamics, or a detection, resets the kinds. */
int b2dev_set_kinds(b2dev_ctx* ctx, int n, const int* kind, const double* Z, int on_device);

/* Reactions and relative velocities (3 per row, caller order): initial
 * values before a solve, results after it. conmerit (may be NULL) receives
 * the per-constraint merit of the last merit evaluation. */
int b2dev_set_state(b2dev_ctx* ctx, const double* R, const double* U, int on_device);
int b2dev_get_state(b2dev_ctx* ctx, double* R, double* U, double* conmerit, int on_device);

/* Run the Gauss-Seidel solve on the resident problem. rerhist / merhist may
 * be NULL or host buffers of opts->maxiter doubles. */
int b2dev_solve(b2dev_ctx* ctx, const b2dev_solve_opts* opts, b2dev_solve_report* rep, double* rerhist,
                double* merhist);

/* Introspection: sizes, processing order and the assembled data (caller order). */
int b2dev_sizes(b2dev_ctx* ctx, int* n, long long* nblocks, int* ncolours, double* free_energy);
int b2dev_get_order(b2dev_ctx* ctx, int* order);         /* order[p] = caller row swept p-th */
int b2dev_get_colours(b2dev_ctx* ctx, int* colour);      /* colour per caller row */
int b2dev_get_locdyn(b2dev_ctx* ctx, double* W, double* A, double* rho, double* B, double* V,
                     int* adjptr, int* adjcol, double* Woff, double* free_energy);

/* Events-timed device duration of the last b2dev_assemble (assembly +
 * colouring + layout), in milliseconds. */
float b2dev_last_assemble_ms(b2dev_ctx* ctx);

/* Number of this library's kernels launched on the context so far. */
long long b2dev_launch_count(b2dev_ctx* ctx);

/* Tracing: record, for every row, the inputs and outputs of its diagonal
 * solve in sweep `sweep` (0-based; -1 switches tracing off) of the next
 * solves; b2dev_get_trace copies the last record out in caller row order,
 * 16 doubles per row: B'[3], U in[3], R in[3], U out[3], R out[3], failure kind. */
int b2dev_trace_sweep(b2dev_ctx* ctx, int sweep);
int b2dev_get_trace(b2dev_ctx* ctx, double* out);

/* Contact-graph colouring that allocates nothing. No counterpart in the
 * reference (it sweeps rows in list order and never colours them).
 *
 * For callers that must not allocate device memory: code running while a
 * CUDA stream is being captured into a graph, solvers embedded in a host
 * application whose device memory is owned by its own allocator or memory
 * pool, and real-time loops where cudaMalloc/cudaFree would synchronise the
 * device. It runs the same Jones-Plassmann kernel as b2dev_assemble /
 * b2dev_upload_locdyn, on the given stream, and gives the same colours for
 * the same seed; its scratch is a fixed array inside the library (one flag per
 * row plus a control block, at most 1,048,576 rows, about 4 MB held on every
 * GPU that loads the library until the process exits).
 *
 * Device pointers: adjptr[n+1], adjcol[adjptr[n]] (the graph, as in
 * b2dev_upload_locdyn), colour[n] (output), info[4] (output, may be NULL:
 * timeout flag, colour-overflow flag, number of colours, rounds). n above the
 * maximum is rejected with B2DEV_EINVAL before anything is queued.
 * The first call on a device looks up the array's device address and the
 * kernel's residency; make that first call before any stream capture. That
 * set-up is kept for the life of the process: a cudaDeviceReset of the device
 * afterwards invalidates it, so a process that resets a device must not call
 * this entry point for that device again. Every
 * call shares the one array, so calls whose work overlaps on the GPU (other
 * streams, other threads) race: queue them on one stream or serialise them. */
int b2dev_colour_noalloc(int device, void* stream, int n, const int* adjptr, const int* adjcol, uint64_t seed,
                         int* colour, int* info);

/* One diagonal block solve (dbs.c:492-550 with the FAILURE_CONTINUE fallback
 * chain of bgs.c:976-1003) per caller-given row, on the device: W[9], B[3]
 * (the local free velocity B' including the off-diagonal sum), V[3], rho,
 * gap, friction, restitution, cohesion per row; U and R (3 per row) are read
 * as the starting point and overwritten; kind[i] = 0 ok, 1 diverged,
 * 2 failed. Host arrays. */
int b2dev_diag_solve_batch(b2dev_ctx* ctx, int n, int diagsolver, int failure, double diagepsilon, int diagmaxiter,
                           int dynamic, double step, const double* W, const double* B, const double* V,
                           const double* rho, const double* gap, const double* friction, const double* restitution,
                           const double* cohesion, double* U, double* R, int* kind);

/* Colouring priority of the next layouts: list_order = 1 (default) colours in
 * the greedy order of the caller's row list; 0 uses the seeded priorities of
 * the colour_seed argument (b2gs_locdyn_set_colour_seed selects 0). Both are
 * reproduced bit for bit by the host greedy colouring in that order. A layout
 * whose contact graph equals the previous one reuses its colours
 * (b2dev_colour_reuse_count counts the reuses). */
int b2dev_set_colour_order(b2dev_ctx* ctx, int list_order);
long long b2dev_colour_reuse_count(b2dev_ctx* ctx);

/* ---- batches of independent problems --------------------------------------
 *
 * No counterpart in the reference (one GAUSS_SEIDEL_Solve per call,
 * bgs.c:913). Many small scenes are solved by one persistent launch: the
 * caller uploads the union of their bodies and contacts (contacts of problem k
 * are caller rows row_offsets[k] .. row_offsets[k+1]-1 and touch only that
 * problem's bodies), and every problem keeps its own stopping decision,
 * merit, histories and failure bookkeeping, with the reference semantics
 * (bgs.c:1028-1069). */
typedef struct b2dev_batch_report {
  int iters, thrown, last_fail_kind, nfailures;
  double merit, error, merit_input;
  double ms_to_decision;  /* device time from the launch's start to this problem's final decision */
  int rows;               /* contacts of the problem */
} b2dev_batch_report;

/* Problems of the next b2dev_assemble (nprob = 1: one problem, offsets unused). */
int b2dev_set_problems(b2dev_ctx* ctx, int nprob, const int* row_offsets);
/* free energy of every problem (ldy.c:739), nprob doubles */
int b2dev_problem_free_energy(b2dev_ctx* ctx, double* out);
/* Rows per tile (1..32) of the current layout: smaller tiles give more
 * parallel work to small problems. Until it is set here (or by the batch
 * autotuner, which keeps its choice), a single problem of at most 16,384
 * rows gets 8 rows per tile and a larger one 32. Results do not depend on it. */
int b2dev_set_tile_rows(b2dev_ctx* ctx, int rows);
int b2dev_tile_rows(b2dev_ctx* ctx);
/* Limit, in seconds, of every bounded wait of the solver kernels on a flag
 * that another warp sets (0 restores the default of 2 s). A wait that runs
 * out ends the launch and the solve returns B2DEV_ETIMEOUT; the context keeps
 * its state and stays usable. No counterpart in the reference (its solver
 * never waits on another thread); meant for tests of that path. */
int b2dev_set_wait_limit(b2dev_ctx* ctx, double seconds);

/* Solve every problem (FP64 sweeps). use_graph: capture the launch sequence
 * into a CUDA graph and replay it while its arguments are unchanged.
 * reps[nprob]; rerhist/merhist NULL or nprob * opts->maxiter doubles;
 * total (may be NULL): iterations and merit maxima, sweeps, device time. */
int b2dev_solve_batch(b2dev_ctx* ctx, const b2dev_solve_opts* opts, b2dev_batch_report* reps, double* rerhist,
                      double* merhist, b2dev_solve_report* total, int use_graph);

/* Autotuner of the batched solve: one timed solve of the current problems per
 * combination of rows per tile {32, 16, 8}, staging window {automatic, 128
 * blocks} and persistent grid {full residency, 3/4, 1/2}, each from the
 * current initial state (restored afterwards). The fastest rows per tile stay
 * in the layout; pass grid and stage_blocks in the options of later solves. */
typedef struct b2dev_tune_result {
  int tile_rows, grid, stage_blocks, ntrials;
  float ms;                                  /* device time of the fastest trial */
  int trial_rows[32], trial_grid[32], trial_stage[32];
  float trial_ms[32];
} b2dev_tune_result;
int b2dev_autotune_batch(b2dev_ctx* ctx, const b2dev_solve_opts* opts, b2dev_tune_result* res);

/* ---- learned warm start --------------------------------------------------
 *
 * No counterpart in the reference, which starts each solve from the reactions
 * of the previous step (con->R, zero for new contacts: mem.c:64-86). A small
 * network (BF16 MLP 32 -> 128 -> 128 -> 16, GELU, FP32 accumulation; 25
 * per-contact features plus a constant input, 3 outputs used) predicts the
 * change of each contact's reaction from local quantities; the plain start
 * remains the fallback, chosen by the merit function (mrf.c:35-185).
 * Training and inference run on sm_100a tensor cores (tcgen05.mma with TMEM
 * accumulators). Parameter vector (FP32, b2dev_mlp_nparams() values):
 * W1[128][32] (column 25 = bias of layer 1), W2[128][128], b2[128],
 * W3[16][128] (rows 3..15 zero), b3[16]. */
typedef struct b2dev_mlp b2dev_mlp;

typedef struct b2dev_nn_report {
  double merit_nn;     /* merit of the network's initial reactions */
  double merit_plain;  /* merit of the reactions held before (previous step) */
  int used_nn;         /* 1: the network's reactions became the initial iterate */
  float ms;            /* device time: features, network, the two merit passes */
} b2dev_nn_report;

int b2dev_mlp_nparams(void);
/* stream NULL: the network gets its own stream */
int b2dev_mlp_create(int device, void* stream, b2dev_mlp** out);
void b2dev_mlp_destroy(b2dev_mlp* net);
/* host arrays of b2dev_mlp_nparams() floats; set also clears the Adam moments */
int b2dev_mlp_set_params(b2dev_mlp* net, const float* params);
int b2dev_mlp_get_params(b2dev_mlp* net, float* params);
/* Mean-squared loss over the 3 outputs and its gradient with respect to every
 * parameter, over all nrows samples (device arrays feat[nrows][32],
 * target[nrows][3]); grad (host, nparams) and loss (host) out. */
int b2dev_mlp_grad(b2dev_mlp* net, int nrows, const float* feat, const float* target, float* grad, double* loss);
/* Adam (beta 0.9/0.999, eps 1e-8) over `epochs` passes of minibatches of
 * batch_tiles x 128 samples in a seeded random order; epoch_loss (host,
 * `epochs` values, may be NULL) = mean loss per sample of each epoch. */
int b2dev_mlp_train(b2dev_mlp* net, int nrows, const float* feat, const float* target, int epochs, int batch_tiles,
                    double lr, uint64_t seed, double* epoch_loss);
/* network outputs out[nrows][3] for features feat[nrows][32] (device arrays) */
int b2dev_mlp_forward(b2dev_mlp* net, int nrows, const float* feat, float* out);
/* Features of every row of the context's problem with its current reactions
 * as the previous-step reactions, in caller order (device arrays):
 * feat[n][32], scale[n] (= rho v_s: the prediction is R_prev + scale y) and
 * rprev[n][3]. Used to build training sets. */
int b2dev_nn_features(b2dev_ctx* ctx, float* feat, double* scale, double* rprev);
/* Replace the context's initial reactions by the network's prediction when
 * its merit is below accept_ratio (0 < accept_ratio <= 1) times the merit of
 * the reactions held (the previous step's); otherwise, and whenever the
 * prediction's merit is higher, the plain start stays. U is left as it is. */
int b2dev_nn_warm_start(b2dev_ctx* ctx, b2dev_mlp* net, double accept_ratio, b2dev_nn_report* rep);

#ifdef __cplusplus
}
#endif

#endif
