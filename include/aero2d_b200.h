/*
 * aero2d_b200 — C ABI of the batched 2-D Euler solver path of aero2d, for B200 (sm_100a).
 *
 * The reference (Bulbulator72/Aero2d) is Python + JAX and binds no native
 * code; each entry point below replaces one JAX computation of its Euler path
 * and is called through ctypes from the Python classes aero2d_b200.euler and
 * aero2d_b200.implicit, which keep the reference's class names, arguments and
 * error behaviour.  Conventions:
 *   - every function returns an int status (A2D_OK = 0); no C++ exception
 *     crosses the ABI; a2d_last_error() describes the last failure of the
 *     calling thread;
 *   - the caller owns all device memory: it allocates the grid-metrics blob
 *     and the plan workspace (sizes from the *_bytes queries) and passes
 *     plain device pointers; the library allocates no device memory;
 *   - `stream` is a cudaStream_t passed as void* (NULL = legacy default stream);
 *   - arrays handed in and out use the reference's layouts: node coordinates
 *     x[i][j] (ni x nj, i along the contour, j from the wall outward), states
 *     U[4][ni][nc] per case (conserved rho, rho u, rho v, E), per-case freestream
 *     primitives winf[4] = (rho, u, v, p).
 * A plan is used by one host thread at a time (one plan per GUI worker or
 * request loop); distinct plans are independent.
 */
#ifndef AERO2D_B200_H
#define AERO2D_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define A2D_OK 0
#define A2D_ERR_ARG 1      /* invalid argument (sizes, null pointers, unbound plan) */
#define A2D_ERR_CUDA 2     /* a CUDA call failed */
#define A2D_ERR_STATE 3    /* call out of order (plan not bound, no step taken) */

#define A2D_FP64 0         /* every stage in FP64 */
#define A2D_MIXED 1        /* JVP, face Jacobians and Krylov basis in FP32; residual,
                              factorisation, Gram-Schmidt, norms, update in FP64 */

/* vector slots of a bound plan (packed over the cases of the plan) */
#define A2D_VEC_U 0        /* conserved state */
#define A2D_VEC_R 1        /* residual output of a2d_residual */
#define A2D_VEC_V 2        /* direction input of a2d_jvp / a2d_precond_apply */
#define A2D_VEC_JV 3       /* output of a2d_jvp / a2d_precond_apply */
#define A2D_VEC_DU 4       /* Newton update of the last step */

typedef struct a2d_plan a2d_plan;

/* Solver settings; names follow EulerSolver (aero2d/euler.py:219-221) and
 * ImplicitEuler (aero2d/implicit.py:68-70) and their solve() arguments. */
typedef struct a2d_params {
  int gmres_restart;      /* ImplicitEuler gmres_restart (<= 64)            default 50   */
  int jacobi_sweeps;      /* ImplicitEuler jacobi_sweeps                    default 4    */
  double gmres_tol;       /* ImplicitEuler gmres_tol                        default 0.01 */
  double cfl0;            /* ImplicitEuler cfl0                             default 10   */
  double cfl_max;         /* ImplicitEuler cfl_max                          default 300  */
  double max_update;      /* ImplicitEuler max_update                       default 0.2  */
  double tol;             /* ImplicitEuler.solve tol (residual drop)        default 1e-8 */
  double cfl;             /* EulerSolver cfl (explicit CFL, local_dt)       default 2.5  */
  double irs_eps;         /* EulerSolver irs_eps                            default 0.6  */
  double lim_k;           /* EulerSolver lim_k                              default 0.02 */
  int order;              /* EulerSolver order (1 or 2)                     default 2    */
  int vortex_correction;  /* EulerSolver vortex_correction                  default 1    */
  int precision;          /* A2D_FP64 or A2D_MIXED                          default FP64 */
  int retire;             /* 1: a case stops stepping once done; 0: all cases step
                             until every case is done (the reference loop) default 1    */
  int max_iter;           /* capacity of the per-step history               default 200  */
  int use_graph;          /* replay each Newton step as one CUDA graph      default 1    */
} a2d_params;

int a2d_version(void);
const char* a2d_last_error(void);
void a2d_default_params(a2d_params* params);

/* ---- O-grid generation on the device (aero2d/grid.py:34-81 ogrid, growth ratio) ----
 * a2d_grid_spacing: host; spacing[k] = ds0 * r**k for k < nj - 1, r from 200 bisection steps
 * (grid.py:34-41, :52-53).  a2d_grid_build: n grids at once, one CTA each (grid.py:50-81):
 * ring device [n][ni][2] contour points (trailing-edge point once, 3 <= ni <= 1024), spacing
 * device [n][nj-1], outputs x, y device [n][ni][nj] and min_area device [n] (the smallest cell
 * area; <= 0 is the reference's inverted-grid RuntimeError, grid.py:78-80).  Layers 0..nj-2 are
 * bitwise the reference's marching; the outer circle uses the device's atan2/cos/sin. */
int a2d_grid_spacing(int nj, double ds0, double radius, double* spacing);
int a2d_grid_build(int n, int ni, int nj, const double* ring, const double* spacing, int normal_smoothing,
                   double* x, double* y, double* min_area, void* stream);

/* ---- grid metrics (aero2d/euler.py:44-60 compute_metrics, :230-233 xf/yf) ---- */
int a2d_metrics_bytes(int ni, int nj, size_t* bytes);
/* x, y: device FP64 node coordinates [ni][nj]; metrics: device blob of a2d_metrics_bytes */
int a2d_metrics_build(int ni, int nj, const double* x, const double* y, void* metrics, void* stream);

/* ---- plans: a batch of cases (the vmap axis of euler.py:393 / implicit.py:204-210) ---- */
/* ni[k], nc[k]: cells of case k; metrics[k]: its metrics blob; winf: [ncases][4] host FP64 */
int a2d_plan_create(int ncases, const int* ni, const int* nc, const void* const* metrics,
                    const double* winf, const a2d_params* params, a2d_plan** plan);
int a2d_plan_workspace_bytes(const a2d_plan* plan, size_t* bytes);
int a2d_plan_bind(a2d_plan* plan, void* workspace, size_t bytes, void* stream);
int a2d_plan_destroy(a2d_plan* plan);
int a2d_plan_ncases(const a2d_plan* plan);

/* ---- launch-configuration knobs, chosen per (grid sizes, precision) by the autotuner
 * (aero2d_b200.autotune); no counterpart in the reference.  Results do not depend on
 * them: every variant computes the same arithmetic in the same order. ---- */
#define A2D_JVP_TILE_32x8 0     /* tile shape (i x j cells) of the FP32 JVP stencil; FP64 plans */
#define A2D_JVP_TILE_32x16 1    /* always use 32 x 8 */
#define A2D_JVP_TILE_64x4 2
#define A2D_JVP_TILE_16x16 3
#define A2D_SWEEP_LANES 0       /* line sweep: one warp per half line group, a lane per line   */
#define A2D_SWEEP_ROWS 1        /* line sweep: four warps per half line group, a warp per block row */
#define A2D_SWEEP_PAIRS 2       /* line sweep: two warps per half line group, two lanes per line */
#define A2D_SWEEP_HALVES 3      /* line sweep: a cluster of two CTAs per line group, one per half,  */
                                /* a warp per block row, the halves meeting in distributed shared  */
                                /* memory                                                           */
/* a new plan starts with A2D_JVP_TILE_32x16 and A2D_SWEEP_HALVES (FP64 plans: A2D_SWEEP_LANES);
 * A2D_SWEEP_ROWS and A2D_SWEEP_HALVES are refused on FP64 plans (A2D_ERR_ARG) */
/* any time, bound or not; a change re-captures the Newton step's graph at the next step */
int a2d_plan_set_tuning(a2d_plan* plan, int jvp_tile, int sweep_variant, void* stream);
int a2d_plan_get_tuning(const a2d_plan* plan, int* jvp_tile, int* sweep_variant);

/* vector I/O in the reference layout [4][ni][nc] of one case (device pointers) */
int a2d_vec_set(a2d_plan* plan, int slot, int case_index, const double* src, void* stream);
int a2d_vec_get(const a2d_plan* plan, int slot, int case_index, double* dst, void* stream);
/* primitives (rho, u, v, p) = cons_to_prim of a slot's vector of one case (euler.py:66-71),
 * in the reference layout [4][ni][nc]: the W that EulerSolver.residual returns (euler.py:260) */
int a2d_vec_get_prim(const a2d_plan* plan, int slot, int case_index, double* dst, void* stream);

/* ---- point operations (aero2d/euler.py) ---- */
/* U of every case := prim_to_cons(winf) (init_state, euler.py:383-384); resets the Newton state */
int a2d_init_freestream(a2d_plan* plan, void* stream);
/* resets the Newton state (CFL, histories, flags) and keeps U (warm start U0) */
int a2d_reset(a2d_plan* plan, void* stream);
/* R := residual(U, winf, circ) (euler.py:259-287); circ: device [ncases] or NULL for
 * Gamma(U) = Cl(U) M / 2 as ImplicitEuler._res does (implicit.py:160-167) */
int a2d_residual(a2d_plan* plan, const double* circ, void* stream);
/* JV := d residual(U, winf, Gamma(U)) / dU . V  (implicit.py:179-181, jax.jvp) */
int a2d_jvp(a2d_plan* plan, void* stream);
/* forces (euler.py:318-331): coef [ncases][3] = Cl, Cd, Cm; cp: wall Cp of all cases
 * concatenated (ni per case), may be NULL; device pointers */
int a2d_forces(a2d_plan* plan, double* coef, double* cp, void* stream);
/* builds the line preconditioner at U with the per-case CFL (implicit.py:81-128) */
int a2d_precond_setup(a2d_plan* plan, void* stream);
/* JV := M(V), the line-Jacobi application (implicit.py:150-157) */
int a2d_precond_apply(a2d_plan* plan, void* stream);
/* local time steps of case case_index from primitives W (device [4][ni][nc], reference layout):
 * dt [ni][nc] = params.cfl * vol / (lambda_i + lambda_j) (EulerSolver.local_dt, euler.py:289-296) */
int a2d_local_dt(const a2d_plan* plan, int case_index, const double* W, double* dt, void* stream);
/* sets the pseudo-time CFL of every case (host array [ncases]) */
int a2d_set_cfl(a2d_plan* plan, const double* cfl, void* stream);

/* ---- the Newton-Krylov solver (aero2d/implicit.py:169-253) ---- */
/* one pseudo-transient Newton step of every live case, with the per-case
 * rollback / freeze / SER-CFL logic of ImplicitEuler.solve on the device */
int a2d_newton_step(a2d_plan* plan, void* stream);
/* up to max_steps steps; stops when no case is live (retire=1) or every case is
 * done (retire=0); *steps receives the number of steps taken; synchronises */
int a2d_newton_run(a2d_plan* plan, int max_steps, int* steps, void* stream);
/* per-case results to host arrays (any may be NULL), length ncases:
 * nsteps, converged-to-tol flag, frozen flag, last finite residual norm, r0 */
int a2d_case_status(const a2d_plan* plan, int* nsteps, int* done, int* frozen, double* lastrn,
                    double* r0, void* stream);
/* per-case scalars of the last step to a host array [ncases][8]: residual norm (NaN if the
 * step failed), step length omega, CFL of the next step, r0, circulation, ||M(b - A x0)||,
 * Arnoldi vectors used, 1 if the step was committed */
int a2d_case_scalars(const a2d_plan* plan, double* out, void* stream);
/* forces of every case at the current U to host arrays: coef [ncases][3] = Cl, Cd, Cm
 * (euler.py:318-331), cp [sum of ni] or NULL; synchronises */
int a2d_case_forces(a2d_plan* plan, double* coef, double* cp, void* stream);
/* restarts the listed cases (host index list) with new freestreams winf [n][4]: U := the
 * freestream state unless keep_state (then the current U is the start, as U0 of
 * implicit.py:194-253), Newton state reset as a2d_reset, the cases live again; the
 * other cases are untouched.  With keep_state a case that has stepped keeps its residual
 * reference r0 (the previous point's), so params.tol keeps its absolute level and the
 * SER CFL ramp starts at once; a2d_reset after U0 instead takes r0 from the first
 * residual, as the reference does.  The slot recycling of a served batch. */
int a2d_case_restart(a2d_plan* plan, int n, const int* cases, const double* winf, int keep_state, void* stream);
/* stops the listed cases (host index list) from stepping until they are restarted */
int a2d_case_retire(a2d_plan* plan, int n, const int* cases, void* stream);
/* points the listed cases at other grids of their size: metrics[q] is a device blob of
 * a2d_metrics_build with case cases[q]'s ni, nc (kept alive by the caller while in use);
 * a new airfoil for a served slot, followed by a2d_case_restart (cold) */
int a2d_case_set_grid(a2d_plan* plan, int n, const int* cases, const void* const* metrics, void* stream);

/* ---- continuous-batching service: served polar sweeps ----
 * A fixed set of slots, in classes by grid size (ni, nc).  A request is a sequence of
 * freestreams (e.g. the points of an alpha sweep) on one grid of a class's size, solved one
 * after another in one slot, each point from the previous point's state when `continuation`
 * is set (alpha continuation), else from the freestream; a point ends when it converges (drop
 * below params.tol), freezes, or reaches params.max_iter steps.  Before every Newton step,
 * queued requests are admitted in arrival order into free slots of their class.  No
 * counterpart exists in the reference (its callers loop over ImplicitEuler.solve); the C
 * ABI's own serving entry points. */
typedef struct a2d_service a2d_service;
/* one class: ni, nc cells of the grid (as a2d_plan_create); metrics: its blob (a2d_metrics_build) */
int a2d_service_create(int ni, int nc, const void* metrics, int slots, const a2d_params* params,
                       a2d_service** service);
/* nclasses classes of distinct sizes: slots[c] slots of ni[c] x nc[c] cells each, metrics[c]
 * the class's default grid (used by a2d_service_submit and by requests without a grid) */
int a2d_service_create_ragged(int nclasses, const int* ni, const int* nc, const void* const* metrics,
                              const int* slots, const a2d_params* params, a2d_service** service);
/* the same with the slots split into `lanes` plans (at most the largest class's slot count):
 * slot q of each class goes to lane q mod lanes; a Newton step of every busy lane runs on the
 * lane's own stream, forked from and joined back into the caller's, so that the lanes'
 * kernels overlap on the GPU.  Results do not depend on the lane count (lanes = 1: one plan
 * stepped on the caller's stream, as a2d_service_create_ragged) */
int a2d_service_create_lanes(int nclasses, const int* ni, const int* nc, const void* const* metrics,
                             const int* slots, int lanes, const a2d_params* params, a2d_service** service);
int a2d_service_workspace_bytes(const a2d_service* service, size_t* bytes);
int a2d_service_bind(a2d_service* service, void* workspace, size_t bytes, void* stream);
/* a request on the first class's default grid; winf: host [npoints][4]; *id receives the
 * request id (> 0) */
int a2d_service_submit(a2d_service* service, int npoints, const double* winf, int continuation, long long* id);
/* a request on its own grid of ni x nc cells (a class's size): metrics is its device blob,
 * kept alive by the caller until the request's result is taken (NULL: the class's default) */
int a2d_service_submit_grid(a2d_service* service, int ni, int nc, const void* metrics, int npoints,
                            const double* winf, int continuation, long long* id);
/* admits queued requests, takes one Newton step of the busy slots and collects the
 * points that ended; *busy receives the busy slots before the step; synchronises */
int a2d_service_step(a2d_service* service, int* busy, void* stream);
/* ids of requests finished since the last poll (at most max_ids) */
int a2d_service_poll(a2d_service* service, long long* ids, int max_ids, int* n);
/* a finished request's results to host arrays: coef [npoints][3], cp [npoints][ni] or NULL,
 * converged [npoints], nsteps [npoints]; releases the request */
int a2d_service_result(a2d_service* service, long long id, double* coef, double* cp, int* converged, int* nsteps);
/* a finished request's per-point residual drop (last finite residual norm / r0) to a host
 * array [npoints]: a point reached params.tol when its drop is below it (the reference's own
 * converged flag above asks only three orders, aero2d/implicit.py:252); call before
 * a2d_service_result, which releases the request */
int a2d_service_result_drop(a2d_service* service, long long id, double* drop);
int a2d_service_pending(a2d_service* service, int* queued, int* running);
/* the service's first lane's plan (borrowed; it lives as long as the service; with one lane
 * its slots are the service's in class order), for a2d_plan_set_tuning and the measurement
 * calls.  Stepping a lane's plan directly, outside a2d_service_step, is only safe while no
 * request is queued or running */
int a2d_service_plan(a2d_service* service, a2d_plan** plan);
/* the number of lanes, and one lane's plan (borrowed), case count and the service slot of
 * each of its cases (slots: an array of nslots, or NULL) */
int a2d_service_lanes(const a2d_service* service, int* lanes);
int a2d_service_lane(a2d_service* service, int lane, a2d_plan** plan, int* nslots, int* slots);
/* kernel launches of one Newton step of all lanes' plans (counted in their captured graphs; 0
 * before the first step) and the Newton steps the service has taken since bind */
int a2d_service_stats(a2d_service* service, int* kernels_per_step, long long* newton_steps);
int a2d_service_destroy(a2d_service* service);
/* per-step histories to host arrays [steps][ncases] (residual norm, Cl); steps <= max_iter */
int a2d_history(const a2d_plan* plan, int steps, double* rn, double* cl, void* stream);

/* sweep-factor entries (G, C, P, Q) that the mixed-precision factorisation stored saturated
 * since bind (or the last reset): entries beyond the FP16 range (|v| > 65504, or not finite) are
 * stored as +-65504; FP64 plans never saturate.  *count to host; reset != 0 zeroes the counter;
 * synchronises.  No counterpart in the reference (it factors in the solver dtype) */
int a2d_factor_saturations(a2d_plan* plan, unsigned long long* count, int reset, void* stream);
/* number of cases still stepping (retire=1) or not yet done (retire=0); synchronises */
int a2d_live_count(a2d_plan* plan, int* n, void* stream);
/* kernel launches of one Newton step (counted in the captured graph; 0 before the
 * first step), Newton steps taken since the last reset, and the bytes of the case
 * tables that a2d_plan_bind copies to the device */
int a2d_plan_stats(const a2d_plan* plan, int* kernels_per_step, int* steps_taken, size_t* table_bytes);

/* ---- measurement ---- */
#define A2D_K_JVP 0        /* linearised residual stencil on the whole batch            */
#define A2D_K_SWEEP 1      /* one coupled line-Jacobi sweep (right-hand side + both     */
                           /* block-Thomas recurrences, fused)                          */
#define A2D_K_SWEEP_FIRST 2 /* the first sweep of a preconditioner application         */
#define A2D_K_DOTS 3       /* Gram-Schmidt pass 1: projections on restart/2 vectors     */
#define A2D_K_UPDATE 4     /* Gram-Schmidt pass 3: subtraction, next basis vector       */
#define A2D_K_RESIDUAL 5   /* FP64 residual stencil                                     */
#define A2D_K_FACEJAC 6    /* first-order face Jacobian blocks                          */
#define A2D_K_FACTOR 7     /* block-Thomas factorisation                                */
#define A2D_K_PROJECT 8    /* Gram-Schmidt pass 2: subtraction and re-projection        */
/* times `reps` back-to-back launches of one kernel on the plan's current data with CUDA
 * events on `stream`, for every case of the plan; *ms receives the mean per launch.
 * Overwrites scratch vectors only (not U). Synchronises. */
int a2d_time_kernel(a2d_plan* plan, int which, int reps, float* ms, void* stream);

/* ---- explicit RK4 + implicit residual smoothing (aero2d/euler.py:334-346) ---- */
/* n RK iterations of every case, each followed by circ := Cl M / 2 (euler.py:398-404);
 * res: device [ncases], the RK residual of the last iteration.  With a coarse level
 * (a2d_plan_set_coarse) each iteration is one FAS V-cycle (euler.py:368-381) through all
 * levels, every level bound */
int a2d_rk_iterate(a2d_plan* plan, int n, double* res, void* stream);
/* FAS multigrid (euler.py:241-250, 349-381): `coarse` holds the same cases, in the same
 * order, on grids of every other node (ni/2 x nc/2 cells; its params give its order, 1 in
 * the reference); NULL unlinks.  Levels chain: the coarse plan may have its own coarse level */
int a2d_plan_set_coarse(a2d_plan* plan, a2d_plan* coarse);
/* R := smooth(R) in place on the residual slot (euler.py:298-312) */
int a2d_smooth(a2d_plan* plan, void* stream);
/* per-case circulation slot used by a2d_rk_iterate: host array [ncases] */
int a2d_set_circulation(a2d_plan* plan, const double* circ, void* stream);

/* ---- residual without device allocation ---- */
/* No counterpart in the reference: an entry point for callers that cannot call cudaMalloc
 * (a host application whose memory manager owns all device memory and does not let a plugin
 * allocate, or a loop that must not allocate while it runs).  It computes, for ncases cases
 * on one grid, R = residual(U, winf, circ) exactly as a2d_residual does and the per-case
 * residual norm rnorm[k] = sqrt(mean((R_rho / vol)^2)) that the Newton loop tests for
 * convergence.  It allocates nothing: besides the caller's buffers it uses one file-scope
 * device array of about 0.86 MB, which every GPU that loads the library holds until the process
 * exits; the first call on a device looks up that array's address (and a call looks it up again
 * when the device's current context has changed since, e.g. after cudaDeviceReset), so make the
 * first call on each device, and the first after such a change, before any stream capture.  Calls share the array, so calls whose kernels overlap
 * on the GPU race.  Limits: ncases <= 64, 4 <= ni <= 512, 2 <= nj - 1 <= 128; larger batches are
 * rejected with A2D_ERR_ARG.
 *   metrics: the grid's blob from a2d_metrics_build; U, R: device [ncases][4][nj-1][ni]
 *   (component, wall-normal, circumferential: the library's internal layout, i fastest);
 *   winf: device [ncases][4]; circ: device [ncases] or NULL for Gamma(U) = Cl(U) M / 2;
 *   params: host, NULL for defaults (lim_k, order, vortex_correction are used);
 *   rnorm: device [ncases]. */
int a2d_residual_norms_static(const void* metrics, int ni, int nj, int ncases, const double* U,
                              const double* winf, const double* circ, const a2d_params* params,
                              double* R, double* rnorm, void* stream);

/* point-wise HLLC flux of n faces (euler.py:79-121): WL, WR [4][n], S [2][n], F [4][n]
 * device FP64 arrays */
int a2d_hllc_flux(int n, const double* WL, const double* WR, const double* S, double* F, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* AERO2D_B200_H */
