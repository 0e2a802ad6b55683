/*
 * cufil.h -- C ABI of the B200 mobility engine for the cilia/filament Stokes
 * simulator racksa/CUFCM_FIL.
 *
 * The reference exposes its hot path as the abstract C++ class
 * `mobility_solver` (src/cilia/mobility/mobility_solver.hpp:19-128) whose
 * back-ends (rpy_mobility_solver, fcm_mobility_solver) implement pure virtual
 * staging/evaluation methods (mobility_solver.hpp:26-46) and whose generic
 * layer assembles and solves the implicit saddle-point system
 * (mobility_solver.hpp:81-111).  This header replaces that class with plain C
 * entry points: opaque handles, plain pointers and sizes, int status codes.
 * Every entry point cites the reference method it stands in for.
 *
 * Layouts follow the reference's host buffers exactly
 * (mobility_solver.hpp:53-63, rpy_mobility_solver.cu:61-67):
 *   x_segs [3*n_seg]  segment centres, AoS (x,y,z)
 *   f_segs [6*n_seg]  segment force + torque, AoS (fx,fy,fz,tx,ty,tz)
 *   v_segs [6*n_seg]  segment velocity + angular velocity, AoS
 *   x_blobs, f_blobs, v_blobs [3*n_blob]  blob centres / forces / velocities
 * Segment order is swimmer -> filament -> segment
 * (id = n*NFIL*NSEG + m*NSEG + k, mobility_solver.cpp:432).
 *
 * Error convention: every function returns CF_OK (0) or a CF_E* code and
 * never exits or aborts; cf_last_error() gives a thread-local message.
 * A handle is not thread-safe; distinct handles are independent.
 */
#ifndef CUFIL_H
#define CUFIL_H

#include <stddef.h>
#include <stdint.h>

#if defined(__GNUC__)
#define CF_API __attribute__((visibility("default")))
#else
#define CF_API
#endif

#ifdef __cplusplus
extern "C" {
#endif

/* ---------------------------------------------------------------- status */
#define CF_OK 0
#define CF_EINVAL 1          /* bad argument or size */
#define CF_ENOMEM 2          /* device or pinned allocation failed */
#define CF_ECUDA 3           /* CUDA runtime / driver error */
#define CF_NOT_CONVERGED 4   /* GMRES stopped at its iteration cap */
#define CF_NONFINITE 5       /* NaN/Inf met in inputs or iterates */
#define CF_TIMEOUT 6         /* a bounded device wait gave up */
#define CF_ENOTSUP 7         /* configuration not supported */

/* Thread-local message for the last failing call on this thread. */
CF_API const char *cf_last_error(void);
/* ABI version: major*10000 + minor*100 + patch. */
CF_API int cf_version(void);

/* ============================================================ mobility ==
 * Back-end of mobility_solver: staging + block products of the RPY grand
 * mobility matrix (rpy_mobility_solver.{hpp,cu}; kernels cuda_functions.cu).
 */
typedef struct cf_mobility cf_mobility;

typedef struct cf_mobility_config {
    int n_seg;          /* NSWIM*NFIL*NSEG segments (may be 0) */
    int n_blob;         /* NSWIM*NBLOB rigid-body blobs (may be 0) */
    int wall;           /* 1: no-slip wall z=0, Swan-Brady (INFINITE_PLANE_WALL);
                           0: unbounded RPY (cuda_functions.cu:205-356) */
    int seg_dof;        /* 3: segments carry forces only (PRESCRIBED_CILIA);
                           6: forces + torques, velocities + angular velocities */
    double seg_radius;  /* RSEG (config.hpp); the wall formula assumes 1 */
    double blob_radius; /* RBLOB */
    double mu;          /* MU; the wall formula assumes 1 */
    int device;         /* CUDA device ordinal */
} cf_mobility_config;

/* allocate_host_memory + allocate_device_memory (rpy_mobility_solver.cu:54-117) */
CF_API int cf_mobility_create(const cf_mobility_config *cfg, cf_mobility **out);
/* free_host_memory + free_device_memory (rpy_mobility_solver.cu:14-52) */
CF_API int cf_mobility_destroy(cf_mobility *h);

/* copy_{segment,blob}_{positions,forces}_to_device (rpy_mobility_solver.cu:119-175) */
CF_API int cf_copy_segment_positions_to_device(cf_mobility *h, const float *x_segs);
CF_API int cf_copy_segment_forces_to_device(cf_mobility *h, const float *f_segs);
CF_API int cf_copy_blob_positions_to_device(cf_mobility *h, const float *x_blobs);
CF_API int cf_copy_blob_forces_to_device(cf_mobility *h, const float *f_blobs);
/* copy_{segment,blob}_velocities_to_host (rpy_mobility_solver.cu:177-205);
 * these wait for the engine's stream. */
CF_API int cf_copy_segment_velocities_to_host(cf_mobility *h, float *v_segs);
CF_API int cf_copy_blob_velocities_to_host(cf_mobility *h, float *v_blobs);
/* wait_for_device (rpy_mobility_solver.cu:247-256) */
CF_API int cf_wait_for_device(cf_mobility *h);

/* evaluate_*_mobility (rpy_mobility_solver.cu:258-338; kernels
 * cuda_functions.cu:362-757).  Write/accumulate semantics mirror the kernels:
 *   segment_segment  V_seg  = M_ss F_seg                       (Mss_mult)
 *   segment_blob     V_seg += M_sb F_blob                      (Msb_mult)
 *   blob_blob        V_blob = M_bb F_blob                      (Mbb_mult)
 *   blob_segment     V_blob += M_bs F_seg  if seg_dof == 3,
 *                    V_blob  = M_bs F_seg  if seg_dof == 6     (Mbs_mult)
 *   full             V_seg = M_ss F_seg + M_sb F_blob,
 *                    V_blob = M_bb F_blob + M_bs F_seg
 * All are asynchronous on the engine's stream. */
CF_API int cf_evaluate_segment_segment_mobility(cf_mobility *h);
CF_API int cf_evaluate_segment_blob_mobility(cf_mobility *h);
CF_API int cf_evaluate_blob_blob_mobility(cf_mobility *h);
CF_API int cf_evaluate_blob_segment_mobility(cf_mobility *h);
CF_API int cf_evaluate_full_mobility(cf_mobility *h);

/* One synchronous host call: positions + forces in, velocities out
 * (read_positions_and_forces + evaluate_full_mobility + copy_*_to_host).
 * Any of the blob pointers may be NULL when n_blob == 0. */
CF_API int cf_apply_mobility(cf_mobility *h, const float *x_segs, const float *x_blobs,
                      const float *f_segs, const float *f_blobs,
                      float *v_segs, float *v_blobs);

/* Same product on device-resident buffers in the same AoS layouts (no host
 * copies), enqueued on `stream` (a cudaStream_t; NULL is the legacy default
 * stream, as everywhere in CUDA).  Asynchronous. */
CF_API int cf_apply_mobility_device(cf_mobility *h, const float *d_x_segs, const float *d_x_blobs,
                             const float *d_f_segs, const float *d_f_blobs,
                             float *d_v_segs, float *d_v_blobs, void *stream);

/* Wall segment-segment product V_seg = M_ss F_seg (3-dof segments, the
 * product of cf_evaluate_segment_segment_mobility with wall = 1, seg_dof = 3)
 * on device buffers in the AoS layouts above, for callers that cannot allocate
 * device memory (inside stream capture, or under a host that owns all device
 * memory through its own allocator).  No counterpart in the reference.  It
 * allocates nothing: its scratch is a fixed array inside this library (about
 * 2.3 MB per GPU that loads it, held until the process exits), so n_seg is
 * limited to 8192 (larger values give CF_EINVAL).  The first call on a device
 * resolves that array's device address; make it before any stream capture.
 * Asynchronous on `stream` (NULL: the legacy default stream).  All calls share
 * the one array, so calls that overlap on the GPU race: serialise them (one
 * stream, or events).  It uses the split-source tile kernel, not the symmetric
 * kernel of cf_evaluate_segment_segment_mobility, so the two agree to the
 * mobility tolerance (1e-5 relative L2), not bit for bit.  It never
 * synchronises, so a bounded device wait that gives up cannot be returned as
 * CF_TIMEOUT: every entry of d_v_segs is then a quiet NaN instead. */
CF_API int cf_rpy_wall_segments_noalloc(const float *d_x_segs, const float *d_f_segs, float *d_v_segs, int n_seg,
                                        void *stream);

/* Test hook, no counterpart in the reference: the number of tries of the first
 * bounded wait with which later launches of the staged tile kernel wait for
 * their sources (process-wide; the default and the maximum are the full
 * limit).  0 makes every such wait give up at once: the block still drains its
 * copies with the full limit, skips its sum, and the product reports
 * CF_TIMEOUT (handle path) or NaN outputs (cf_rpy_wall_segments_noalloc).
 * Restore the default with cf_set_wait_limit(~0u). */
CF_API int cf_set_wait_limit(unsigned limit);

/* ================================================================ fcm ==
 * Fast force-coupling method in a triply periodic box: the reference's cuFCM
 * FCM_solver (src/cufcm/CUFCM_SOLVER.cu:20-727) for translating particles
 * (ROTATION 0): spread -> FFT Stokes solve -> gather + near-field and self
 * corrections.  Positions, forces and velocities are [3N] AoS float arrays. */
typedef struct cf_fcm cf_fcm;

typedef struct cf_fcm_config {
    int n;                    /* particles N */
    double rh;                /* hydrodynamic radius; FCM width sigma = rh/sqrt(pi) */
    double alpha, beta, eta;  /* grid Gaussian Sigma = alpha*dx, support ngd = round(alpha*beta) (<= 32),
                                 correction radius Rc = eta*alpha*dx (simulation_info keys) */
    int nx, ny, nz;           /* FFT grid (nx even) */
    double boxsize;           /* Lx; Ly = boxsize*ny/nx, Lz = boxsize*nz/nx */
    int device;
} cf_fcm_config;

/* FCM_solver::FCM_solver: derived parameters, buffers, cuFFT plans (CUFCM_SOLVER.cu:20-248) */
CF_API int cf_fcm_create(const cf_fcm_config *cfg, cf_fcm **out);
CF_API int cf_fcm_destroy(cf_fcm *h);
/* FCM_solver::hydrodynamic_solver on host arrays (synchronous) */
CF_API int cf_fcm_apply(cf_fcm *h, const float *Y, const float *F, float *V);
/* Same on device arrays, ordered after the work already on `stream` (NULL: legacy default stream). */
CF_API int cf_fcm_apply_device(cf_fcm *h, const float *d_Y, const float *d_F, float *d_V, void *stream);
/* fcm_mobility_solver::evaluate_full_mobility (fcm_mobility_solver.cu:463-502): the first n_seg particles are
 * segments (x_segs [3n_seg], f_segs [6n_seg] of which the forces are used, v_segs [6n_seg] with zero angular
 * slots), the rest blobs (x_blobs, f_blobs, v_blobs [3(N-n_seg)]). */
CF_API int cf_fcm_apply_segments_blobs(cf_fcm *h, int n_seg, const float *x_segs, const float *x_blobs,
                                       const float *f_segs, const float *f_blobs, float *v_segs, float *v_blobs);
/* Stage timing with CUDA events (off by default): after an apply, ms[6] =
 * [grid clear, hash + sort + cell list, spread, FFT + solve + inverse FFT,
 *  gather, corrections + scatter]. */
CF_API int cf_fcm_set_timing(cf_fcm *h, int enable);
CF_API int cf_fcm_stage_times(cf_fcm *h, float *ms);
/* Derived parameters: [ngd, dx, sigma, Sigma, Rc, Mx, My, Mz, self mobility] */
CF_API int cf_fcm_info(cf_fcm *h, double *info);

/* ========================================================== flow field ==
 * Flow velocities at field points from saved segment and blob forces: the
 * reference's flow-field post-processor (src/flow_field/flow_field_evaluator.cu,
 * flow_velocities :13-217, prefactor 1/(8 pi mu) :545-557).  Per flow point:
 * a Stokeslet per segment force with Blake's image system of a wall at z = 0
 * when the data has no blobs (n_blob_per_body == 0), a rotlet per segment
 * torque, a Stokeslet per blob force, and with remove_net_force minus a
 * Stokeslet of every source's force at its body's position.  Layouts are the
 * reference's: x_flow [3 n_flow], x_segs [3 n_seg], f_segs [6 n_seg] (force,
 * torque), x_blobs / f_blobs [3 n_blob], x_bodies [3 n_bodies] with segment j
 * on body j / n_seg_per_body and blob k on body k / n_blob_per_body.  A flow
 * point on a source gives non-finite values, as in the reference. */
typedef struct cf_flow cf_flow;
typedef struct cf_flow_config {
    int max_flow, max_seg, max_blob, max_bodies;  /* capacities */
    double mu;                                     /* MU */
    int remove_net_force;                          /* REMOVE_NET_FORCE_STOKESLET */
    int device;
} cf_flow_config;
CF_API int cf_flow_create(const cf_flow_config *cfg, cf_flow **out);
CF_API int cf_flow_destroy(cf_flow *h);
/* Host arrays in, host velocities out (synchronous). */
CF_API int cf_flow_velocities(cf_flow *h, const float *x_flow, int n_flow, const float *x_segs, const float *f_segs,
                              int n_seg, int n_seg_per_body, const float *x_blobs, const float *f_blobs, int n_blob,
                              int n_blob_per_body, const float *x_bodies, float *v_flow);
/* Same on device arrays, asynchronous on `stream` (NULL: the legacy default stream). */
CF_API int cf_flow_velocities_device(cf_flow *h, const float *d_x_flow, int n_flow, const float *d_x_segs,
                                     const float *d_f_segs, int n_seg, int n_seg_per_body, const float *d_x_blobs,
                                     const float *d_f_blobs, int n_blob, int n_blob_per_body,
                                     const float *d_x_bodies, float *d_v_flow, void *stream);

/* ========================================================== simulation ==
 * Generic layer of mobility_solver for prescribed-shape cilia above a no-slip
 * wall (CILIA_TYPE 3, BODY_OR_SURFACE_TYPE 0, MOBILITY_TYPE 1,
 * SOLVER_TYPE 1 with right preconditioning): beat kinematics
 * (filament::initial_guess, filament.cpp:1336-1500), RHS assembly
 * (mobility_solver.cpp:284-634), block-diagonal preconditioner
 * (apply_preconditioner_new, :1102-1594), saddle-point product
 * (system_matrix_mult_new, :1887-2185) and GMRES (solve_linear_system,
 * :2187-2669), all device-resident.
 *
 * Saddle vector layout (wall, PRESCRIBED_BODY_VELOCITIES, mobility_solver.cpp:361,373):
 *   [ 3*N_s segment constraint forces lambda | N_fil phase rates | N_fil angle rates ]
 * where the rate blocks are present when dynamic_phase / dynamic_angle are set.
 */
typedef struct cf_sim cf_sim;

#define CF_BEAT_FULFORD_BLAKE 1          /* SHAPE_SEQUENCE 1 */
#define CF_BEAT_FULFORD_BLAKE_ORIGINAL 4 /* SHAPE_SEQUENCE 4 */

#define CF_PRECOND_NONE 0
#define CF_PRECOND_BLOCK_DIAG 1          /* apply_preconditioner_new */
#define CF_PRECOND_LEARNED 2             /* per-filament MLP (flexible GMRES) */
#define CF_PRECOND_LINE 3                /* block-Jacobi over line patches along the beat direction */
#define CF_PRECOND_LEARNED_LINE 4        /* line patches + per-filament MLP correction (flexible GMRES) */

typedef struct cf_sim_config {
    int n_fil;              /* NFIL (one swimmer: the wall) */
    int n_seg;              /* NSEG segments per filament */
    double seg_sep;         /* SEG_SEP; DL = SEG_SEP*RSEG, RSEG = 1 */
    int beat;               /* CF_BEAT_* */
    int dynamic_phase;      /* DYNAMIC_PHASE_EVOLUTION */
    int dynamic_angle;      /* DYNAMIC_SHAPE_ROTATION */
    double dt;              /* DT = PERIOD/STEPS_PER_PERIOD */
    double spring_factor;   /* TORSIONAL_SPRING_MAGNITUDE_FACTOR */
    double gmres_tol;       /* LINEAR_SYSTEM_TOL (relative residual) */
    int gmres_max_iter;     /* MAX_LINEAR_SYSTEM_ITER (capped at system size) */
    int precond;            /* CF_PRECOND_* */
    /* Base positions [3*n_fil] and per-filament natural frequency [n_fil]. */
    const double *base_pos;
    const double *omega0;
    /* Initial phase and shape-rotation angle [n_fil] each (psi.dat). */
    const double *phase0;
    const double *angle0;
    /* Reference generalised forces over one period (input/forcing/*.dat). */
    const double *gen_phase_force_refs; int n_gen_phase_refs;
    const double *gen_angle_force_refs; int n_gen_angle_refs;
    /* Reference arclength parameters [rows*cols] (rows = phases over one period,
     * cols = segments); NULL selects the bisection of
     * filament::find_fitted_shape_s (WRITE_GENERALISED_FORCES mode). */
    const double *s_values_ref; int s_ref_rows; int s_ref_cols;
    /* Bisection tolerance on the length fraction, times NSEG (0 selects the
     * reference's 0.1, filament.cpp:1143). */
    double s_tol_factor;
    int device;
    /* CF_PRECOND_LINE: filaments per patch (runs of equal base x, consecutive
     * in y, the beat direction of the wall frame; at most 32, 0 selects 32) and
     * the number of steps between refreshes of the patch inverses (0 selects 1). */
    int line_patch;
    int precond_refresh;
} cf_sim_config;

CF_API int cf_sim_create(const cf_sim_config *cfg, cf_sim **out);
CF_API int cf_sim_destroy(cf_sim *s);

/* One implicit step nt: filament::initial_guess (phase/angle update when
 * nt > 0, kinematics) + mobility_solver::compute_velocities (RHS, GMRES with
 * warm start).  iters/relres may be NULL.  Returns CF_NOT_CONVERGED when GMRES
 * met its cap (the iterate is still stored, as the reference does). */
CF_API int cf_sim_step(cf_sim *s, int nt, int *iters, double *relres);
/* Same without waiting for the result: iteration count and residual are
 * recorded on the device and read by cf_sim_last_solve. */
CF_API int cf_sim_step_async(cf_sim *s, int nt);
CF_API int cf_sim_last_solve(cf_sim *s, int *iters, double *relres);
/* Copy of the filament state [n_fil] each (any pointer may be NULL). */
CF_API int cf_sim_get_state(cf_sim *s, double *phase, double *angle, double *phase_dot, double *angle_dot);
/* Segment positions [3*N_s] and constraint forces [6*N_s] in the reference's
 * host layouts (x_segs_host / f_segs_host). */
CF_API int cf_sim_get_segments(cf_sim *s, float *x_segs, float *f_segs);
/* One step with its host traffic in a single call: uploads the filament state
 * (any *_in may be NULL: keep the device state), runs step nt, and returns the
 * new state [n_fil] each, the segment positions x_segs [3*N_s] and constraint
 * forces f_segs [6*N_s] (reference layouts), iterations and residual (any
 * output may be NULL), with one synchronisation.  Same status as cf_sim_step. */
CF_API int cf_sim_step_io(cf_sim *s, int nt, const double *phase_in, const double *angle_in,
                          const double *phase_dot_in, const double *angle_dot_in, double *phase_out,
                          double *angle_out, double *phase_dot_out, double *angle_dot_out, float *x_segs,
                          float *f_segs, int *iters, double *relres);
/* Velocity directions K_phase, K_angle [3*N_s] each (vel_dir_phase/angle). */
CF_API int cf_sim_get_directions(cf_sim *s, double *k_phase, double *k_angle);
/* Arclength parameters of the current kinematics [n_fil*n_seg] (s_to_use). */
CF_API int cf_sim_get_arclengths(cf_sim *s, double *s_values);
/* The engine's stream of this handle (a cudaStream_t). */
CF_API int cf_sim_stream(cf_sim *s, void **stream);
/* Overwrites the filament state [n_fil] each from host memory (any pointer may
 * be NULL); the rates are also the GMRES warm start.  Asynchronous. */
CF_API int cf_sim_set_state(cf_sim *s, const double *phase, const double *angle, const double *phase_dot,
                            const double *angle_dot);
/* The saddle-point solution [system size]: constraint forces and rates of the
 * last step, which seed the next step's GMRES (mobility_solver.cpp:2298-2388).
 * Saved with cf_sim_get_state it checkpoints the whole trajectory state;
 * cf_sim_set_solution also sets the filament rates from its rate rows. */
CF_API int cf_sim_get_solution(cf_sim *s, double *sol);
CF_API int cf_sim_set_solution(cf_sim *s, const double *sol);
/* GMRES iterations of step nt are kept at index nt % 4096; copies the first n. */
CF_API int cf_sim_iteration_log(cf_sim *s, int *iters, int n);
/* Kernels launched by one step that ran `iters` GMRES iterations. */
CF_API int cf_sim_launches_per_step(cf_sim *s, int iters);
/* Size of the saddle-point system. */
CF_API int cf_sim_system_size(cf_sim *s);
/* Kinematics only (filament::initial_guess). */
CF_API int cf_sim_initial_guess(cf_sim *s, int nt);
/* assemble_rhs (mobility_solver.cpp:284-634) for the current state. */
CF_API int cf_sim_assemble_rhs(cf_sim *s, int nt, double *rhs);
/* apply_preconditioner_new: out = P^{-1} in (host vectors, system size). */
CF_API int cf_sim_apply_preconditioner(cf_sim *s, const double *in, double *out);
/* system_matrix_mult_new: out = A in (host vectors, system size). */
CF_API int cf_sim_system_matvec(cf_sim *s, const double *in, double *out);
/* solve_linear_system (mobility_solver.cpp:2187-2669) on a caller's right-hand
 * side: GMRES with the handle's preconditioner on A x = rhs for the current
 * geometry (that of the last cf_sim_step or cf_sim_initial_guess; CF_EINVAL
 * before either), x_inout the initial guess on entry (discarded, as the
 * reference does, when its residual exceeds |rhs|) and the solution on return.
 * tol is the relative residual target, max_iter at most the handle's
 * gmres_max_iter.  As in the reference, the solution also becomes the warm
 * start of the next step and its rate rows the filament rates.  Status as
 * cf_sim_step (CF_NOT_CONVERGED at the cap with the iterate returned); the
 * iteration log of the steps is not touched. */
CF_API int cf_sim_solve(cf_sim *s, const double *rhs, double *x_inout, double tol, int max_iter, int *iters,
                        double *relres);

/* The reference's data files, appended as its main loop appends them every
 * PLOT_FREQUENCY_IN_STEPS steps (cilia_sim_main.cu:624-718,
 * mobility_solver.cpp:3150-3279): <prefix>_seg_states.dat (segment centres),
 * _body_states.dat (the wall case's fixed body), _true_states.dat
 * ("step period phases angles", what pyfile/find_periodic and
 * pyfile/bisection read), _seg_vels.dat (M applied to the constraint forces,
 * six slots per segment) and _seg_forces.dat (six slots per segment), each
 * line led by save_step.  Call after a step. */
CF_API int cf_sim_write_data(cf_sim *s, int save_step, double period, const char *prefix);
/* <prefix>_fil_references.dat (filament base positions,
 * swimmer.cpp:1114-1127) and <prefix>.par (cilia_sim_main.cu:178-232). */
CF_API int cf_sim_write_config(cf_sim *s, const char *prefix, int total_steps);
/* The initial-condition file in the reference's psi.dat layout
 * (filament.cpp:310-340): two header values (the sweep drivers write the
 * spring constant and the period there; header may be NULL), then n_fil
 * phases, then n_fil shape-rotation angles.  A file with fewer values gives
 * CF_EINVAL (the reference silently keeps its defaults).  No GPU needed. */
CF_API int cf_read_ic(const char *path, int n_fil, double *header, double *phase, double *angle);

/* Launch shapes of the iteration kernels: choice[5] = {pair-kernel CTAs per
 * SM, dot-product row chunk, dot-product blocks per SM, update blocks per SM,
 * update tile rows (32, 64, 128 or 256)}.
 * cf_sim_autotune times the candidates on the handle's current state (basis
 * index k_hint, <= 0: half the last step's iterations) and keeps the fastest;
 * only scratch buffers are written.  choice may be NULL. */
CF_API int cf_sim_autotune(cf_sim *s, int k_hint, int *choice);
/* CF_PRECOND_LINE: rebuilds the patch inverses for the current kinematics
 * (asynchronous, on the handle's stream); no counterpart in the reference,
 * whose preconditioner has no set-up.  cf_sim_precond_info reports the patch
 * count, the largest patch system, the FLOPs of one rebuild (2 n^3 per patch)
 * and the bytes one application moves; any pointer may be NULL. */
CF_API int cf_sim_refresh_preconditioner(cf_sim *s);
CF_API int cf_sim_precond_info(cf_sim *s, int *n_patches, int *max_n, double *refresh_flops, double *apply_bytes);
CF_API int cf_sim_set_tuning(cf_sim *s, const int *choice);
CF_API int cf_sim_get_tuning(cf_sim *s, int *choice);

/* ------------------------------------------------------------------------
 * cf_mlp: the per-filament network of the learned preconditioner
 * (CF_PRECOND_LEARNED).  No counterpart in the reference.  A fully connected
 * network in -> hidden -> hidden -> out with ReLU, FP32 master weights, BF16
 * tensor-core GEMMs with FP32 accumulation, trained by the library's own
 * backward and Adam kernels on the mean squared error.  Tensors are device
 * pointers to row-major FP32 [n x in] / [n x out]; n <= max_batch.
 * Parameters, flat: W1 [in x H], b1 [H], W2 [H x H], b2 [H], W3 [H x out], b3 [out].
 * ------------------------------------------------------------------------ */
typedef struct cf_mlp cf_mlp;

CF_API int cf_mlp_create(int in_dim, int hidden, int out_dim, int max_batch, unsigned long long seed, int device,
                         cf_mlp **out);
CF_API int cf_mlp_destroy(cf_mlp *h);
CF_API long long cf_mlp_num_params(cf_mlp *h);
/* y = net(x) on `stream` (NULL: the network's own stream). */
CF_API int cf_mlp_forward(cf_mlp *h, const float *x, int n, float *y, void *stream);
/* Loss and flat gradient (host, num_params floats; either may be NULL) of one batch. */
CF_API int cf_mlp_gradients(cf_mlp *h, const float *x, const float *t, int n, float *grads, double *loss);
/* One Adam step (beta 0.9 / 0.999) on one batch; loss may be NULL (then no synchronisation). */
CF_API int cf_mlp_train_step(cf_mlp *h, const float *x, const float *t, int n, float lr, double *loss);
CF_API int cf_mlp_get_params(cf_mlp *h, float *params);
CF_API int cf_mlp_set_params(cf_mlp *h, const float *params);
CF_API int cf_mlp_stream(cf_mlp *h, void **stream);
/* Versioned checkpoint of a trained network and its correction weight alpha
 * (cf_sim_set_network_weight), for reuse across runs.  The reference keeps no
 * learned state, so the file layout is this library's own: a 56-byte header
 * (magic "CFPRECN", version 1, widths, alpha, parameter count, FNV-1a hash of
 * the parameters) and the FP32 parameters.  cf_precond_load creates a new
 * cf_mlp (max_batch rows, on `device`); a file with a wrong magic, version,
 * width, size or hash gives CF_EINVAL and creates nothing.  weight may be NULL. */
CF_API int cf_precond_save(cf_mlp *net, double weight, const char *path);
CF_API int cf_precond_load(const char *path, int max_batch, int device, cf_mlp **out, double *weight);

/* Learned preconditioner (CF_PRECOND_LEARNED, flexible GMRES): the
 * block-diagonal preconditioner plus a per-filament network correction
 * z_m = P_bd(r)_m + s_m net(features_m(r)); no counterpart in the reference.
 * Features per filament, scaled by s_m = |(r_m, rbar_m)|: its 3*nseg force
 * rows and 2 rate rows, the mean force rows of its neighbours along the
 * lattice line (rbar_m), then its segment positions relative to its base over
 * the filament length (unscaled): 9*nseg + 2 values; the correction has
 * 3*nseg + 2.  cf_sim_learned_dims gives both widths.
 * cf_sim_set_network attaches a cf_mlp of those widths (batch >= n_fil); the
 * handle keeps the pointer, the caller keeps ownership.
 * CF_PRECOND_LEARNED_LINE puts the same correction on top of the line
 * patches, z_m = P_line(r)_m + s_m net(...).
 * cf_sim_collect_pairs runs step nt of a CF_PRECOND_BLOCK_DIAG or
 * CF_PRECOND_LINE handle and, after each of its first max_pairs Arnoldi
 * products w = A z, writes the features of w and the target
 * (z_m - P(w)_m) / s_m (P the handle's preconditioner) of every filament into
 * the device arrays x [max_pairs*n_fil][in] and t [max_pairs*n_fil][out];
 * rows = the number written.  cf_sim_features: features of a host vector
 * (system size) into host x [n_fil][in]. */
CF_API int cf_sim_learned_dims(cf_sim *s, int *n_in, int *n_out);
CF_API int cf_sim_set_network(cf_sim *s, cf_mlp *net);
/* Weight of the network correction, z_m = P_bd(r)_m + alpha s_m net(...), in [0, 4] (default 1). */
CF_API int cf_sim_set_network_weight(cf_sim *s, double alpha);
CF_API int cf_sim_collect_pairs(cf_sim *s, int nt, int max_pairs, float *x, float *t, int *rows);
CF_API int cf_sim_features(cf_sim *s, const double *v, float *x);

/* ------------------------------------------------------------------------
 * Batches of independent arrays (periodic-orbit / bisection sweeps): many
 * wall arrays of uneven size stepped together, one graph launch per step for
 * the whole batch.  Each array is described by its own cf_sim_config; every
 * field except n_fil, base_pos, omega0, phase0 and angle0 must equal array
 * 0's.  Per-filament arrays (state) are concatenated array by array.  Each
 * array runs its own GMRES (own Krylov basis, Hessenberg matrix and stopping
 * test); arrays that stopped are masked out of the remaining iterations, so
 * every array gets the result its own cf_sim would give.
 * ------------------------------------------------------------------------ */
typedef struct cf_batch cf_batch;

CF_API int cf_batch_create(const cf_sim_config *cfgs, int n_arrays, cf_batch **out);
CF_API int cf_batch_destroy(cf_batch *b);
/* Arrays, filaments and segments in the batch; sizes[n_arrays] = system sizes (may be NULL). */
CF_API int cf_batch_shape(cf_batch *b, int *n_arrays, int *n_fil, int *n_seg, int *sizes);
/* One implicit step nt of every array; iters/relres [n_arrays] may be NULL.
 * Returns CF_NONFINITE if any array met a non-finite value, else
 * CF_NOT_CONVERGED if any array stopped at its cap. */
CF_API int cf_batch_step(cf_batch *b, int nt, int *iters, double *relres);
CF_API int cf_batch_step_async(cf_batch *b, int nt);
/* Result of the last solve per array (status: 1 converged, 2 cap, 3 non-finite,
 * 4 initial guess good, 5 zero right-hand side); any pointer may be NULL. */
CF_API int cf_batch_last_solve(cf_batch *b, int *iters, double *relres, int *status);
CF_API int cf_batch_get_state(cf_batch *b, double *phase, double *angle, double *phase_dot, double *angle_dot);
CF_API int cf_batch_set_state(cf_batch *b, const double *phase, const double *angle, const double *phase_dot,
                              const double *angle_dot);
/* Segment positions [3*N_s total], FP64, array by array. */
CF_API int cf_batch_get_segments(cf_batch *b, double *x_segs);
/* Saddle-point solution of one array [its system size]. */
CF_API int cf_batch_get_solution(cf_batch *b, int array, double *sol);
CF_API int cf_batch_iteration_log(cf_batch *b, int array, int *iters, int n);
CF_API int cf_batch_stream(cf_batch *b, void **stream);
/* Kernels launched by one step whose GMRES loop ran loop_iters iterations
 * (the largest iteration count in the batch). */
CF_API int cf_batch_launches_per_step(cf_batch *b, int loop_iters);
CF_API int cf_batch_autotune(cf_batch *b, int k_hint, int *choice);
CF_API int cf_batch_set_tuning(cf_batch *b, const int *choice);
CF_API int cf_batch_get_tuning(cf_batch *b, int *choice);

/* ------------------------------------------------------------------------
 * A free rigid body carrying prescribed cilia (the reference's swimmer with
 * PRESCRIBED_CILIA, BODY_VELOCITY_TYPE 0, unbounded fluid; one swimmer,
 * dynamic phase and shape-rotation angle).  Replaces the body branches of
 * mobility_solver::system_matrix_mult_new / apply_preconditioner_new
 * (mobility_solver.cpp:1887-2105, 1244-1475), swimmer::make_precon_mat
 * (swimmer.cpp:1175-1349) and the explicit body update of
 * cilia_sim_main.cu:700-716.  Saddle layout: [3 n_fil n_seg segment forces |
 * 3 n_blob blob forces | V, Omega | n_fil phase rates | n_fil angle rates].
 * All radii are 1 (RSEG = RBLOB = 1), MU = 1.
 * ------------------------------------------------------------------------ */
typedef struct cf_swim cf_swim;

typedef struct cf_swim_config {
    int n_fil, n_seg, n_blob;
    double seg_sep;            /* SEG_SEP; DL = SEG_SEP */
    int beat;                  /* CF_BEAT_FULFORD_BLAKE or CF_BEAT_FULFORD_BLAKE_ORIGINAL */
    double dt;
    double spring_factor;      /* TORSIONAL_SPRING_MAGNITUDE_FACTOR */
    double gmres_tol;
    int gmres_max_iter;
    /* Body frame: filament bases [3*n_fil] and outward directions [3*n_fil]
     * (swimmer::filament_references, normal_refs), blob positions [3*n_blob]
     * (rigid_body::blob_references). */
    const double *fil_refs;
    const double *fil_dirs;
    const double *blob_refs;
    /* Initial body position [3] and orientation [4, scalar first]; NULL: 0 and identity. */
    const double *body_x0;
    const double *body_q0;
    const double *omega0;      /* [n_fil]; NULL: 2 pi */
    const double *phase0;      /* [n_fil]; NULL: 0 */
    const double *angle0;      /* [n_fil]; NULL: 0 */
    const double *gen_phase_force_refs; int n_gen_phase_refs;
    const double *gen_angle_force_refs; int n_gen_angle_refs;
    const double *s_values_ref; int s_ref_rows; int s_ref_cols;
    double s_tol_factor;
    int device;
} cf_swim_config;

CF_API int cf_swim_create(const cf_swim_config *cfg, cf_swim **out);
CF_API int cf_swim_destroy(cf_swim *h);
/* One step nt: body frame, kinematics (phase and angle advance when nt > 0),
 * the body's preconditioner matrix, GMRES (warm start from the last solution),
 * then the body update x += dt V, q = lie_exp(dt Omega) q. */
CF_API int cf_swim_step(cf_swim *h, int nt, int *iters, double *relres);
/* Phase, angle and their rates [n_fil] each; body position [3] and
 * orientation [4] of the next step; body velocity [6] (V, Omega) of the last step. */
CF_API int cf_swim_get_state(cf_swim *h, double *phase, double *angle, double *phase_dot, double *angle_dot,
                             double *body_x, double *body_q, double *body_v);
/* Segment [3 n_fil n_seg] and blob [3 n_blob] positions and forces of the last step (FP64). */
CF_API int cf_swim_get_particles(cf_swim *h, double *x_segs, double *x_blobs, double *f_segs, double *f_blobs);
/* Velocity directions vel_dir_phase, vel_dir_angle [3 n_fil n_seg] each of the last step. */
CF_API int cf_swim_get_directions(cf_swim *h, double *k_phase, double *k_angle);
/* A x and P x (host vectors of the system size) for the geometry of the last step. */
CF_API int cf_swim_system_matvec(cf_swim *h, const double *in, double *out);
CF_API int cf_swim_apply_preconditioner(cf_swim *h, const double *in, double *out);
CF_API int cf_swim_system_size(cf_swim *h);

/* ------------------------------------------------------------------------
 * Instability-driven elastic cilia on a no-slip wall (the reference's
 * CILIA_TYPE 0 with INFINITE_PLANE_WALL): one implicit step (backward Euler at
 * step 0, BDF2 after) solved by Broyden's method around the 6x6 wall mobility.
 * Replaces filament::initial_guess / internal_forces_and_torques /
 * invert_approx_jacobian / update (filament.cpp:1336-2206),
 * mobility_solver::compute_errors (mobility_solver.cpp:2760-2860), the
 * barrier forces (cuda_functions.cu:1825-1919) and broyden_solver
 * (broyden_solver.cpp:26-131), driven as cilia_sim_main.cu:405-560 drives them.
 * MU = RSEG = 1.  Filaments start straight along +z from their bases.
 * ------------------------------------------------------------------------ */
typedef struct cf_elastic cf_elastic;

typedef struct cf_elastic_config {
    int n_fil, n_seg;              /* 13 <= n_seg <= 24 */
    double seg_sep;                /* DL = SEG_SEP (> 2) */
    const double *base_pos;        /* [3 n_fil] */
    double dt;                     /* DT = PERIOD / STEPS_PER_PERIOD */
    double dimensionless_force;    /* DIMENSIONLESS_FORCE (0: 220); F_end = it KB / (DL^2 NSEG^2) */
    double kb, kt;                 /* KB, KT (0: 1800) */
    double repulsion_factor;       /* REPULSIVE_FORCE_FACTOR (0: 2) */
    double broyden_tol;            /* TOL (0: 1e-4) */
    int max_broyden_iter;          /* MAX_BROYDEN_ITER (0: 400) */
    double jacobian_confidence;    /* JACOBIAN_CONFIDENCE_FACTOR (0: 0.1) */
    /* Step-0 perturbation forces on segments 4 and 12 (CILIA_IC_TYPE): 0 = (0.01 F_end, 0, 0) on
     * segment 4 only; 1 = that plus (0, 0.01 F_end, 0) on segment 12; 2 = perturbations
     * [n_fil][2][3] given (the reference draws them at random for its types 2 and 3). */
    int ic_type;
    const double *perturbations;
    int device;
} cf_elastic_config;

CF_API int cf_elastic_create(const cf_elastic_config *cfg, cf_elastic **out);
CF_API int cf_elastic_destroy(cf_elastic *h);
/* One step nt (0-based); broyden_iters may be NULL.  CF_NOT_CONVERGED when Broyden's method used
 * all its iterations (the reference stops the run there), CF_NONFINITE when it diverged. */
CF_API int cf_elastic_step(cf_elastic *h, int nt, int *broyden_iters);
/* Segment positions [3N], orientations [4N] (scalar first) and the internal forces and torques
 * [6N] of the last evaluation, FP64; any pointer may be NULL. */
CF_API int cf_elastic_get_segments(cf_elastic *h, double *x, double *q, double *f);
/* The approximate inverse Jacobian [6 n_seg x 6 n_seg, row-major] of filament m as last prepared. */
CF_API int cf_elastic_get_jacobian_inverse(cf_elastic *h, int m, double *jinv);
/* Initial guess and first evaluation of step nt with the Jacobian prepared, no Broyden iteration;
 * err_out [6N] (may be NULL) receives the residual.  For checking the stages. */
CF_API int cf_elastic_first_evaluation(cf_elastic *h, int nt, double *err_out);
CF_API int cf_elastic_stats(cf_elastic *h, int *last, int *max_iters, long long *total, int *steps);
CF_API int cf_elastic_system_size(cf_elastic *h);

/* One 64 x 64 x 64 tile product D = A^T B (A [k][m], B [k][n], D [m][n], host arrays, FP32) on the
 * 5th-generation tensor cores as the line patches' refresh computes its tiles: three TF32 products
 * (operands split into a TF32 high part and an FP32 remainder), FP32 accumulation in tensor memory.
 * wait_limit: tries of the bounded wait for the products (0: default).  For checking. */
CF_API int cf_tc_tile_product(const float *A, const float *B, float *D, unsigned wait_limit);

#ifdef __cplusplus
}
#endif
#endif /* CUFIL_H */
