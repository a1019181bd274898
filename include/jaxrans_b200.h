/* jaxrans_b200: the pseudo-transient Newton-Krylov hot path of JAX-RANS on NVIDIA B200.
 *
 * A C ABI (plain pointers and sizes) over hand-written sm_100a CUDA kernels.  A plan is
 * a batch of cases (each one canvas: the grid's blocks and their ghost rings) with every
 * static table the kernels read, the device work buffers and the solver state; every
 * launch advances all cases of the batch at once, and a single case is a batch of one.
 * Fields are variable-major (nvar, NI*NJ) FP64 arrays, nvar = 4 (Euler, laminar) or 5
 * (SA).  Arrays that span a batch hold the cases back to back in case order (a case's
 * offsets from jr_case_sizes); for a single case they are that case's arrays.
 *
 * Every function returns 0 on success or a JR_E* code; jr_last_error() gives a message.
 * Functions taking device pointers run on the plan's stream and do not synchronise it
 * unless stated; functions taking host pointers copy in/out and synchronise.
 *
 * The reference (giovannicatalani/jax-rans, src/jaxrans) has no FFI: each entry point
 * below replaces a Python/JAX function, cited beside it, that a binding would call.
 */
#ifndef JAXRANS_B200_H
#define JAXRANS_B200_H

#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define JR_OK 0
#define JR_EINVAL 1      /* a bad argument */
#define JR_ENOMEM 2      /* a device allocation failed */
#define JR_ECUDA 3       /* a CUDA error (message in jr_last_error) */
#define JR_EMISMATCH 4   /* buffers that do not fit the plan */
#define JR_ETIMEOUT 5    /* a device-side wait gave up (a case's status has JR_STATUS_WAIT_LIMIT) */

/* Bits of a case's status word (jr_state_get, jr_case_state_get): the last Newton step's
 * outcome.  JR_STATUS_WAIT_LIMIT stays set until the case's state is set again. */
#define JR_STATUS_NONFINITE 1         /* a non-finite value met in a reduction */
#define JR_STATUS_REJECTED 2          /* the last Newton step was rejected */
#define JR_STATUS_GMRES_BREAKDOWN 4   /* an Arnoldi vector of zero norm */
#define JR_STATUS_WAIT_LIMIT 8        /* the line solve's staged copy was not seen to land in time */

typedef struct jr_plan jr_plan;

/* Everything a plan is built from (host memory; copied by jr_plan_create). */
typedef struct jr_plan_desc {
  int32_t NI, NJ, nvar;
  const uint8_t* interior;      /* NI*NJ */
  const double* volume;         /* NI*NJ */
  const double* faces_i;        /* 2 x (NI+1) x NJ: sx plane, sy plane */
  const double* faces_j;        /* 2 x NI x (NJ+1) */
  const double* centres;        /* 2 x (NI+2) x (NJ+2): cell centres with one reflected ghost ring */
  const double* distance;       /* NI*NJ wall distance (SA), or NULL */
  const int32_t* neighbours;    /* NI*NJ */
  int32_t n_ghost[2];           /* two gather stages */
  const int32_t* ghost[2];
  const int32_t* source[2];
  const int32_t* kind[2];       /* 0 copy, 1 slip wall, 2 no-slip wall, 3 symmetry, 4 far field, 5 inflow, 6 outflow */
  const double* geom[2];        /* 4 per record: nx, ny, mx, my */
  int32_t n_walls;
  const int32_t* wall_cell;
  const int32_t* wall_family;
  const int32_t* wall_face;
  const double* wall_into;
  const double* wall_mid;       /* 2 per wall face */
  int32_t n_chains, chain_L;
  const int32_t* chain_cells;   /* [k * n_chains + c], -1 past the end */
  const int32_t* chain_len;
  const int32_t* chain_up_face;
  const int32_t* chain_up_sign;
  const int32_t* chain_down_face;
  const int32_t* chain_down_sign;
  /* physics */
  double gamma, mu_inf, sutherland, c_cr1, kappa;   /* mu_inf 0: inviscid; sutherland < 0: constant viscosity */
  int32_t flux, limiter, far_field;                  /* flux 0 hllc 1 roe; limiter 0 none 1 minmod 2 van_albada
                                                        3 van_albada_smooth 4 kappa; far field 0 uniform 1 point vortex */
  double q_inf[5];
  double quarter_chord[2];
  /* implicit solver */
  double cfl, cfl_max, cfl_growth, cfl_cutback, cfl_min;
  double krylov_tol, krylov_success, max_relative_update;   /* max_relative_update <= 0: none */
  int32_t krylov_subspace, krylov_restarts, preconditioner; /* preconditioner 0 none, 1 line_j (the reference's
                                                               split 4x4 + scalar SA chains), 2 line_j_coupled
                                                               (the SA row coupled to the mean flow: 5x5 blocks) */
  int32_t precision;                                        /* 0 fp64, 1 mixed (fp32 line factor and Krylov basis) */
  double force_length, moment_centre[2];
} jr_plan_desc;

/* Build a plan (device copies of every table, work buffers, a stream). */
int jr_plan_create(const jr_plan_desc* desc, jr_plan** out);
/* A plan of n_cases cases advanced together (a polar of angles of attack, a batch of
 * requests).  The cases may differ in grid, flow and CFL settings but must share nvar,
 * viscous or not, precision, krylov_subspace, krylov_restarts and preconditioner.
 * Replaces the jax.vmap of one Newton step over the freestreams of a polar
 * (src/jaxrans/polar.py:80-121): each case keeps its own state, CFL ramp, rejections
 * and history, and the cases never interact. */
int jr_batch_create(const jr_plan_desc* descs, int32_t n_cases, jr_plan** out);
int jr_plan_cases(const jr_plan* plan);
/* Case c's canvas cells and face entries and its offsets in batch-long arrays (a field's
 * offset is nvar * canvas_offset). */
int jr_case_sizes(const jr_plan* plan, int32_t c, int64_t* n_canvas, int64_t* n_faces, int64_t* canvas_offset,
                  int64_t* face_offset);
/* Take case c out of (enabled 0) or back into (1) every launch: a free slot of a serving
 * batch.  Its state and scalars stay as they are. */
int jr_case_enable(jr_plan* plan, int32_t c, int32_t enabled);
/* New freestream primitives q_inf (nvar values: rho, u, v, p[, nu_hat]) for case c: the
 * far-field state and the freestream of the force coefficients.  Replaces at_alpha and
 * freestream_primitive (src/jaxrans/polar.py:75-77, src/jaxrans/core/state.py:107-121):
 * the angle of attack or Mach number enters the solver only through this vector. */
int jr_case_set_inflow(jr_plan* plan, int32_t c, const double* q_inf);
/* Overwrite case c (a slot) with a new case of the same shape: same canvas, ghost, wall
 * and chain tables' sizes (a grid of the same size and topology, another section or
 * flow) and the plan's shared solver settings.  Static tables, physics and settings are
 * replaced in place -- nothing is allocated -- and the slot's state is left for
 * jr_case_state_set; JR_EMISMATCH when the shapes differ.  Replaces building a new case
 * and its residual operator (src/jaxrans/case/loader.py:349-373,
 * src/jaxrans/numerics/residual.py:273-334) for every request a server admits. */
int jr_case_load(jr_plan* plan, int32_t c, const jr_plan_desc* desc);
int jr_plan_destroy(jr_plan* plan);
const char* jr_last_error(void);
/* Number of canvas cells NI*NJ and of face entries (NI+1)*NJ + NI*(NJ+1), summed over
 * the cases of the plan. */
int jr_plan_sizes(const jr_plan* plan, int64_t* n_canvas, int64_t* n_faces);
/* The plan's CUDA stream (a cudaStream_t), for callers that order their own work on it. */
void* jr_plan_stream(jr_plan* plan);
/* Issue the plan's work on a caller's cudaStream_t (an XLA FFI handler passes XLA's);
 * NULL returns to the plan's own stream.  The stream in use is drained first, unless it
 * is already the one asked for (then the call does nothing). */
int jr_plan_set_stream(jr_plan* plan, void* stream);
int jr_synchronize(jr_plan* plan);

/* R(U): the residual on the canvas, where(interior, net flux, U - U_inf); second order,
 * or first order when first_order != 0.  Replaces make_residual(...).residual
 * (src/jaxrans/numerics/residual.py:273-334, residual() at :324-327).  Device pointers. */
int jr_residual(jr_plan* plan, const double* U, double* R, int first_order);

/* R(U) as jr_residual computes it, for callers that cannot allocate device memory when
 * they call: a handler running inside another framework's step, whose allocator owns the
 * device's memory and where a cudaMalloc or cudaFree would also synchronise the device.
 * The call's scratch (its case table, the ghost-filled canvas, the tile partial sums) is
 * a static device array of 8 MiB (8388608 bytes) inside the library, held by every GPU
 * that loads it, so the call allocates nothing and writes no work buffer of the plan; a
 * plan that needs more scratch is refused with JR_EINVAL.  The first call on a device
 * looks up the array's address there (set-up): make it with the plan's device current
 * and before any stream capture.  The address is kept for the life of the process, so a
 * cudaDeviceReset (which re-creates the device's context) makes it stale: do not use the
 * library across a device reset.  Every call on a device shares the one array, which
 * keeps the last call's contents (the canvas part is cleared by each call): calls whose
 * work overlaps on the GPU -- on other streams, or for other plans -- race on it.  No
 * counterpart in the reference, which has no FFI and allocates through XLA.  Device
 * pointers. */
int jr_residual_noalloc(jr_plan* plan, const double* U, double* R, int first_order);

/* dR1/dU . v: the exact tangent of the first-order residual at U.  The call linearises
 * the residual at U (each face's flux derivatives and each cell's SA source derivatives,
 * by forward-mode duals, into the plan's linearisation buffer) and applies that
 * linearisation to v, as a Newton step does once per step and once per Arnoldi step.
 * Replaces jax.linearize(jacobian_source.residual, U) and its jvp
 * (src/jaxrans/solvers/implicit.py:104-108).  Device pointers. */
int jr_jvp(jr_plan* plan, const double* U, const double* v, double* Jv);

/* The volume-weighted L2 norm of row `variable` of the field R over each case's block
 * cells, sqrt(sum V R^2 / sum V), computed on the device (a fixed-order sum); out (host)
 * receives one value per case.  Replaces ResidualOperator.norm
 * (src/jaxrans/numerics/residual.py:237-240).  R: device pointer; synchronises. */
int jr_norm(jr_plan* plan, const double* R, int32_t variable, double* out);

/* lambda on every canvas face, i-faces then j-faces (length n_faces).  Replaces
 * ResidualOperator.wave_speeds / face_wave_speeds (src/jaxrans/numerics/residual.py:169-192). */
int jr_wave_speeds(jr_plan* plan, const double* U, double* lam);

/* Factor the line_j preconditioner at (U, cfl) and apply it: z = M^-1 r (the coupled
 * form takes its SA coupling at the same U, which must stay valid until the apply).  Replaces
 * get_preconditioner("line_j")(...)(U, lambdas, cfl) and its solve
 * (src/jaxrans/solvers/preconditioners.py:291-306).  Device pointers. */
int jr_precond_factor(jr_plan* plan, const double* U, double cfl);
int jr_precond_apply(jr_plan* plan, const double* r, double* z);

/* The solver state: U (device or host copy in/out), CFL and the previous |R|.
 * Replaces ImplicitState (src/jaxrans/solvers/implicit.py:35-51).  jr_state_set gives
 * every case the same CFL and |R|; jr_state_get fills one cfl, residual_norm and status
 * per case (any may be NULL).  The jr_case_ forms read or write case c alone. */
int jr_state_set(jr_plan* plan, const double* U_host, double cfl, double residual_norm);
int jr_state_get(jr_plan* plan, double* U_host, double* cfl, double* residual_norm, int32_t* status);
int jr_case_state_set(jr_plan* plan, int32_t c, const double* U_host, double cfl, double residual_norm);
int jr_case_state_get(jr_plan* plan, int32_t c, double* U_host, double* cfl, double* residual_norm,
                      int32_t* status);
/* Device pointer to the plan's own state U (nvar x NI*NJ), valid until jr_plan_destroy. */
double* jr_state_device(jr_plan* plan);
/* The state from a device buffer (a restart with the inputs already in HBM). */
int jr_state_set_device(jr_plan* plan, const double* U_device, double cfl, double residual_norm);
/* Kernels one captured Newton step launches when every Krylov cycle runs (each cycle is a
 * conditional node of the graph, skipped on the device once no case needs it). */
int jr_graph_kernels(jr_plan* plan, int64_t* kernels_per_step);
/* Kernels the Newton steps of this plan have launched so far, the skipped cycles not
 * counted (the device counts the cycles it ran).  Synchronises.  Instrumentation with no
 * counterpart in the reference. */
int jr_launch_count(jr_plan* plan, int64_t* kernels);
/* Average device time (ms, CUDA events on the plan's stream, reps launches each, after one
 * untimed launch) of the hot kernels at the plan's state, out[0..6]: the residual tile, the
 * J.v tile (the tangent pass over the linearisation), the tangent ghost fill, the
 * line-solve apply, the line factor, one CGS2 orthogonalisation against the full basis
 * (three passes), and the linearisation (once per Newton step).  Replaces the timing loop
 * of the reference's scripts/benchmark.py:40-47,88-108 for these pieces. */
int jr_time_kernels(jr_plan* plan, int32_t reps, double* ms_out);

/* n_steps pseudo-transient Newton steps on the plan's state, one captured CUDA graph per
 * step for the whole batch; history (host, n_steps x n_cases, step-major) receives each
 * case's |R| before each step.  Synchronises once; JR_ETIMEOUT if a case's status has
 * JR_STATUS_WAIT_LIMIT (the steps ran; that case's last solves are not to be trusted).
 * Replaces make_newton_step (src/jaxrans/solvers/implicit.py:84-168) run as the
 * driver's block (src/jaxrans/solvers/driver.py:87-104). */
int jr_newton_steps(jr_plan* plan, int32_t n_steps, double* history);

/* The same step count without synchronising: history_device (n_steps x n_cases doubles
 * on the device) receives the norms.  For timing with events on the plan's stream. */
int jr_newton_steps_async(jr_plan* plan, int32_t n_steps, double* history_device);

/* The exit test of case c on the device (the driver's per-case test,
 * src/jaxrans/solvers/driver.py:161-190, with the force settling of
 * src/jaxrans/simulation.py:259-272), run by jr_monitor_blocks after every block:
 * non-finite (a NaN or Inf norm or force coefficient), converged (the block's last |R| <=
 * tol x the running peak), stalled (every |R| of the block equal), settled (CL, CD and CM
 * each varying by less than forces_tol over the last quarter of the blocks, at least four
 * there; forces_tol <= 0: no such test), max_iters after max_blocks blocks (1..1024).
 * release != 0: the case leaves the launches when it stops (a single-case plan is left
 * enabled for later calls).  Resets the case's monitor and enables the case. */
int jr_monitor_set(jr_plan* plan, int32_t c, double tol, double forces_tol, int32_t max_blocks, int32_t release);
/* n_blocks blocks of block_iters Newton steps of every enabled case, each block followed on
 * the device by the forces and the exit test of every monitored case; one synchronisation
 * at the end instead of one per block.  history (host, n_blocks * block_iters x n_cases,
 * step-major, at most 4096 steps) receives each case's |R| before each step; rows after
 * a case stopped are not its.  JR_ETIMEOUT as jr_newton_steps.  Replaces the driver's
 * host loop over blocks (src/jaxrans/solvers/driver.py:161-190). */
int jr_monitor_blocks(jr_plan* plan, int32_t n_blocks, int32_t block_iters, double* history);
/* Case c's monitor: reason (0 running, 1 converged, 2 settled, 3 max_iters, 4 non_finite,
 * 5 stalled), blocks run, the running peak of |R|, and (may be NULL) the force samples,
 * blocks x 3 (CL, CD, CM after each block). */
int jr_monitor_get(jr_plan* plan, int32_t c, int32_t* reason, int32_t* blocks, double* peak, double* coefficients);

/* The plan's autotuner: times the line factor and the line solve with each block size the
 * longest chain allows (64, 128, 256 threads per chain, reps launches each, at the plan's
 * state), and the solve in each form (its factor read level by level from global memory,
 * or, forms s = 1..4, staged into shared memory by one bulk asynchronous copy from level
 * s-1 of the longest chain, where that fits), and keeps the fastest; chosen (3 values,
 * may be NULL) receives the factor's threads, the solve's threads and the solve's form.  Results do not depend on the schedule (each
 * row's arithmetic is the same).  The tile shape of the residual is not tuned: it sets
 * the order of the residual norm's partial sums.  Overwrites the plan's preconditioner
 * factor (the next Newton step makes its own).  Replaces the reference's reliance on
 * XLA's own kernel choices; no counterpart function. */
int jr_autotune(jr_plan* plan, int32_t reps, int32_t* chosen);

/* Sets the line-solve schedule the autotuner would pick: factor_threads and apply_threads
 * in {64, 128, 256} (4 x apply_threads at least the longest chain's even rows), and
 * apply_stage the solve's form, 0 to 4 (JR_EINVAL where the staged part does not fit
 * one block's shared memory).  Results do not depend on it.  A staged copy that
 * fails sets JR_STATUS_WAIT_LIMIT in its case's status (kept until the case's state is set again); it is
 * not expected.  No counterpart in the reference. */
int jr_line_schedule(jr_plan* plan, int32_t factor_threads, int32_t apply_threads, int32_t apply_stage);

/* A check of the device's bounded waits, with no plan: one block waits, tries times (each
 * up to about 1 us), on an mbarrier that no copy completes.  The wait must run out:
 * returns JR_ETIMEOUT with status (may be NULL) = JR_STATUS_WAIT_LIMIT, and the context
 * stays usable.  Device 0's current context, default stream.  No counterpart in the
 * reference. */
int jr_wait_limit_check(int32_t tries, int32_t* status);

/* Force coefficients at the plan's state (or at U if not NULL, a device pointer): out
 * (host, 6 per case) = cl, cd, cm, cd_friction, fx, fy.  Replaces force_coefficients
 * (src/jaxrans/post/forces.py:108-161).  Synchronises. */
int jr_forces(jr_plan* plan, const double* U, double* out);

/* Wall loads per wall face, every case's faces back to back in the plan's wall order, 5
 * values a face (host out): gauge pressure, the area vector into the fluid (x, y), the
 * viscous force on the body (x, y) -- the inputs of the surface distributions (cp, cf).
 * At the plan's state, or at U (device) if not NULL.  Replaces wall_loads
 * (src/jaxrans/post/forces.py:48-68).  Synchronises. */
int jr_wall_loads(jr_plan* plan, const double* U, double* out);

/* ---- 3D (a wing's C-H block: config 5's path) -------------------------------------- */

typedef struct jr_plan3d jr_plan3d;

/* One 3D case: its canvas (NI x NJ x NK, k fastest; the block's cells with a ring of 2
 * ghost cells, as src/jaxrans/mesh/atlas3d.py:119-210 lays it out) and physics.  Fields
 * are variable-major, nvar = 5 (rho, rho u, rho v, rho w, E) or 6 (+ rho nu~, SA-noft2). */
typedef struct jr_plan3d_desc {
  int32_t NI, NJ, NK, nvar;
  const uint8_t* interior;      /* NI*NJ*NK */
  const double* volume;         /* NI*NJ*NK */
  const double* faces[3];       /* family a: 3 planes (x, y, z) of (NI+(a==0)) (NJ+(a==1)) (NK+(a==2)) */
  const double* centres;        /* 3 planes of (NI+2)(NJ+2)(NK+2): centres with one ring beyond the canvas */
  const double* distance;       /* NI*NJ*NK wall distance (SA), or NULL */
  int32_t n_stages;             /* the ghost fill's gather stages, in order (every pass), at most 12 */
  const int32_t* stage_records; /* n_stages counts; the records below are stage after stage */
  const int32_t* ghost;         /* per record: the ghost cell, its source cell, the kind */
  const int32_t* source;
  const int32_t* kind;          /* 0 copy, 1 slip wall, 2 no-slip wall, 3 symmetry, 4 far field */
  const double* normal;         /* 3 per record: the outward unit normal of the boundary face */
  double gamma, mu_inf, sutherland, kappa;   /* mu_inf 0: inviscid; sutherland < 0: constant viscosity */
  int32_t flux, limiter;        /* as jr_plan_desc */
  double q_inf[6];              /* primitive freestream (rho, u, v, w, p[, nu~ / nu_inf]) */
  const int32_t* neighbours;    /* NI*NJ*NK: the partner across a block face, or the cell itself */
  int32_t n_chains, chain_L;    /* line chains along each block's wall-normal index */
  const int32_t* chain_cells;   /* [chain * chain_L + k], -1 past the chain's end */
  const int32_t* chain_up_face; /* link k -> k+1: flat index into the three face families, concatenated */
  const int32_t* chain_up_sign; /* +1 / -1 the link face vector out of / into cell k, 0 no link */
  /* implicit solver (as jr_plan_desc; preconditioner 0 none, 1 line_j) */
  double cfl_max, cfl_growth, cfl_cutback, cfl_min;
  double krylov_tol, krylov_success, max_relative_update;   /* max_relative_update <= 0: none */
  int32_t krylov_subspace, krylov_restarts, preconditioner;   /* 0 none, 1 line_j, 2 line_j coupled (6x6) */
  /* wall faces (the forces) */
  int32_t n_walls;
  const int32_t* wall_cell;     /* the block cell on the face */
  const int32_t* wall_family;   /* the face's family (normal index axis) */
  const int32_t* wall_face;     /* its index within the family's canvas faces */
  const double* wall_into;      /* +1 where the family's vector points into the fluid, else -1 */
  const double* wall_mid;       /* 3 per face: the mean of its four nodes */
  /* 0: the line factor and apply in FP64; 1: in FP32 (the mixed form; Krylov vectors,
   * residual, J.v and update stay FP64) */
  int32_t line_precision;
  double c_cr1;                 /* QCR2000's c_cr1 on the SA model's stress (0: off; TMR's 0.3) */
} jr_plan3d_desc;

/* Build a 3D plan (device copies of the tables, work buffers, a stream).  Every record
 * index is checked against the canvas.  No counterpart function in the reference (its
 * atlas is built in build_atlas_3d, src/jaxrans/mesh/atlas3d.py:119). */
int jr_plan3d_create(const jr_plan3d_desc* desc, jr_plan3d** out);
int jr_plan3d_destroy(jr_plan3d* plan);
/* R(U) on the canvas (device pointers, nvar x canvas): the net flux on block cells,
 * U - U_inf elsewhere; first_order 1: the first-order residual.  Replaces
 * make_residual(...).residual (src/jaxrans/numerics/residual.py:273-334) for a 3D atlas.
 * Synchronises. */
int jr_residual3d(jr_plan3d* plan, const double* U, double* R, int32_t first_order);
/* Jv = dR1/dU . v, exact (forward-mode tangents; device pointers).  Replaces
 * jax.linearize of the first-order residual (src/jaxrans/solvers/implicit.py:104-116).
 * Synchronises. */
int jr_jvp3d(jr_plan3d* plan, const double* U, const double* v, double* Jv);
/* lambda on every canvas face (device pointers), the three families back to
 * back (family a: (NI+(a==0)) (NJ+(a==1)) (NK+(a==2)) faces): |V.S| + a|S| at the face-averaged
 * state plus the thin-layer viscous term.  Replaces face_wave_speeds
 * (src/jaxrans/numerics/residual.py:169-192) on a 3D atlas.  Synchronises. */
int jr_wave_speeds3d(jr_plan3d* plan, const double* U, double* lam);
/* z = M^-1 r of line_j at (U, cfl) (device pointers): the 5x5 mean-flow chains and the
 * scalar SA chains along each block's wall-normal index, solved by block Thomas; cells
 * on no chain copied.  Replaces get_preconditioner("line_j")(...)(U, lambdas, cfl) and
 * its solve (src/jaxrans/solvers/preconditioners.py:209-306) on a 3D atlas.  Synchronises. */
int jr_precondition3d(jr_plan3d* plan, const double* U, double cfl, const double* r, double* z);
/* n_steps pseudo-transient Newton steps on U (device, nvar x canvas, updated in place)
 * from *cfl and the previous |R| *residual_norm (both host, updated); history (host,
 * n_steps) receives |R| before each step.  GMRES(krylov_subspace) with krylov_restarts
 * cycles, CGS2, Givens least squares, the relaxation, acceptance test and CFL ramp of
 * src/jaxrans/solvers/implicit.py:54-168, driven from the host over device kernels (it
 * synchronises for the scalars: three times per Arnoldi step).  Replaces make_newton_step run as the
 * driver's block on a 3D atlas. */
int jr_newton_steps3d(jr_plan3d* plan, double* U, int32_t n_steps, double* cfl, double* residual_norm,
                      double* history);
/* Force coefficients of a 3D case at U (device): out (host, 4) = cl, cd, cm, cd_friction
 * -- lift and drag in the plane of incidence (x-z) per q_inf * area, the pitching moment
 * of pressure and friction about centre (3 values) per q_inf * area * length; the
 * friction from the laminar viscous flux at the wall.  Replaces force_coefficients
 * (src/jaxrans/post/forces.py:108-161) on a 3D atlas.  Synchronises. */
int jr_forces3d(jr_plan3d* plan, const double* U, double area, double length, const double* centre, double* out);
/* The loads on every wall face of a 3D case at U (device): out (host, n_walls x 7) = the
 * gauge pressure, the face's area vector into the fluid (3), the laminar viscous force on
 * the body (3) -- wall_loads (src/jaxrans/post/forces.py:48-68), for the surface
 * distributions (src/jaxrans/post/forces.py:229-246).  Synchronises. */
int jr_wall_loads3d(jr_plan3d* plan, const double* U, double* out);
/* The wall distance of points (device, n_points x 3) to the nearest of n_faces wall faces
 * (device, n_faces x 4 x 3: the corners round each face, taken as a bilinear patch):
 * out (device, n_points).  Faces ranked by the distance to their two triangles, then the
 * exact patch distance over the 16 nearest (src/jaxrans/mesh/wall3d.py:131-158,
 * wall_distance_3d); infinite with no faces.  For the SA model's plan; synchronises. */
int jr_wall_distance3d(const double* points, int64_t n_points, const double* faces, int32_t n_faces, double* out);
/* Kernels the 3D plan entry points (residual, J.v, wave speeds, line solve, Newton steps,
 * forces) have launched since the library was loaded (counted on the host). */
int jr_launches3d(int64_t* out);
/* Average milliseconds per call, over `reps` calls after one untimed call, with CUDA events
 * on the plan's stream, at U (device): ms (host, 3) = the residual R2 (ghost stages,
 * face phase, cell phase), the J.v of R1 along U itself, and the line preconditioner
 * (factor and solve) at CFL 25.  Synchronises; allocates two work vectors for the call.
 * No counterpart in the reference (its scripts/benchmark.py times the jitted calls). */
int jr_time_kernels3d(jr_plan3d* plan, const double* U, int32_t reps, double* ms);

#ifdef __cplusplus
}
#endif

#endif /* JAXRANS_B200_H */
