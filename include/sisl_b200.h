/*
 * sisl_b200.h -- C ABI of the B200 (sm_100a) SISL timestep.
 *
 * Drop-in boundary for the semi-implicit semi-Lagrangian core of the Suetes
 * regional 3-D model (reference: suetes/regional3d/steppers.py,
 * suetes/regional3d/euler.py, suetes/regional3d/operators.py).  The
 * reference is pure Python/JAX and has no FFI of its own; each entry point
 * below names the reference call it replaces (file:line in the reference
 * project).  A jax.ffi / ctypes binding maps those Python calls onto these
 * functions; no torch or C++ type crosses this boundary.
 *
 * Conventions
 *  - Every array argument is a DEVICE pointer on the current CUDA device,
 *    of the core's precision (SISL_F32 or SISL_F64) unless stated.
 *  - Field layout: a field of stagger s has the extents of the reference
 *    array, (ex, ey, ez) = (nx + [s==U], ny + [s==V], nz + [s==W]), stored
 *    x-fastest: element (i, j, k) at offset i + ex * (j + ey * k).  This is
 *    the Fortran order of the reference's (ex, ey, ez) array (numpy
 *    np.asfortranarray / a torch tensor permuted to (ez, ey, ex) contiguous).
 *    2-D horizontal arrays use i + ex * j.
 *  - Thermodynamic state is passed in perturbation form: pi_p = pi - pi_bg,
 *    th_p = th_v - theta_bg.
 *  - Streams are cudaStream_t passed as void*; NULL is the legacy stream.
 *  - Outputs are caller-allocated; scratch comes from a caller-provided
 *    workspace of sisl_workspace_bytes() bytes (256-byte aligned
 *    recommended; an absent, short or not 16-byte aligned workspace returns
 *    SISL_ERR_WORKSPACE before any launch).
 *  - Return value: SISL_OK, a negative error code, or SISL_NOT_CONVERGED
 *    (the GMRES iteration limit was hit; outputs are still written, as in
 *    the reference, which discards GMRES's status at steppers.py:466).
 *  - A core is not re-entrant: calls that share a core must be serialised
 *    (they share its pinned host scratch).
 */
#ifndef SISL_B200_H
#define SISL_B200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

enum { SISL_F32 = 0, SISL_F64 = 1 };
enum { SISL_LOC_M = 0, SISL_LOC_U = 1, SISL_LOC_V = 2, SISL_LOC_W = 3 };
enum { SISL_GMRES_BATCHED = 0, SISL_GMRES_INCREMENTAL = 1 };
enum {
  SISL_WS_STEP = 0, SISL_WS_GMRES = 1, SISL_WS_DEPARTURE = 2, SISL_WS_EXPLICIT = 3, SISL_WS_OPERATOR = 4,
  SISL_WS_FFSL = 5, SISL_WS_STEP_VJP = 6, SISL_WS_EXPLICIT_VJP = 7, SISL_WS_FFSL_VJP = 8,
  SISL_WS_SPLIT = 9, SISL_WS_SPLIT_VJP = 10
};
enum {
  SISL_RELAX_U = 1, SISL_RELAX_V = 2, SISL_RELAX_W = 4, SISL_RELAX_TH = 8, SISL_RELAX_PI = 16
};
/* kernel classes for sisl_timing_select */
enum {
  SISL_K_NONE = 0, SISL_K_MATVEC = 1, SISL_K_PRECOND = 2, SISL_K_DOTS = 3, SISL_K_UPDATE = 4,
  SISL_K_SL = 5, SISL_K_EXPLICIT = 6, SISL_K_OTHER = 7
};
enum {
  SISL_STAGGER_AVG = 0, SISL_STAGGER_DIFF = 1
};

#define SISL_OK 0
#define SISL_NOT_CONVERGED 1
#define SISL_ERR_ARG (-1)
#define SISL_ERR_CUDA (-2)
#define SISL_ERR_WORKSPACE (-3)
#define SISL_ERR_NONFINITE (-4)
#define SISL_ERR_SCRATCH_LIMIT (-5)

/* Grid extents and spacing: RegionalGrid3D(nx, ny, nz, dx, dy, dz, ...)
 * (geometry.py:141) plus CGridOperator3D's periodic axes (operators.py:16). */
typedef struct SislGrid {
  int32_t nx, ny, nz;
  int32_t periodic_x, periodic_y;
  int32_t dtype;
  double dx, dy, dz;
} SislGrid;

/* Physical constants and SISL/GMRES settings: build_dynamical_core kwargs
 * (steppers.py:37-53), the constants dict and SISLStepper3D's arguments. */
typedef struct SislParams {
  double dt, alpha;
  double g, cp, Rd, cvd, p0;
  double pi_scale;         /* 1000 (steppers.py:396) */
  double nu_div, nu_h;     /* Euler3D.nu_div, Euler3D.nu_h (euler.py:62-67) */
  double solver_tol, solver_atol;
  int32_t solver_maxiter;  /* restart cycles */
  int32_t solver_restart;  /* Krylov dimension, <= 128 */
  int32_t solve_method;    /* SISL_GMRES_* */
  int32_t use_limiter;
  int32_t departure_iterations; /* 2 (steppers.py:318) */
  int32_t refine;          /* float32 cores: 1 = also build the float64 coefficients and run GMRES with
                              float64 iterative refinement (sisl_core_set_refinement); no counterpart in
                              the reference, whose GMRES runs wholly in the state precision */
} SislParams;

/* float64 background and metrics (device pointers, device layout):
 * Euler3D.theta_bg / pi_bg / tau_damp (euler.py:76-121) and
 * RegionalGrid3D.Z_m, dz_m_full, dz_w_full, z_xi_w, z_eta_w, m_factors,
 * f_u, f_v, dm_dx_m, dm_dy_m (geometry.py:190-261).  rho_bg: the
 * background density at mass points, or NULL for the equation of state
 * p0 / (Rd theta_bg) pi_bg^(cvd/Rd) (the background the step builds,
 * steppers.py:769-775; Euler3D.precompute_bg, euler.py:127-160, accepts any
 * density).  Read only during sisl_core_create. */
typedef struct SislBackground {
  const double *theta_bg, *pi_bg, *Z_m, *dz_m_full, *dz_w_full, *z_xi_w, *z_eta_w, *tau_damp;
  const double *m_m, *m_u, *m_v, *f_u, *f_v, *dm_dx_m, *dm_dy_m;
  const double* rho_bg;
} SislBackground;

typedef struct SislCore SislCore;

typedef struct SislSolveInfo {
  int32_t cycles;          /* restart cycles run */
  int32_t arnoldi_steps;   /* matvec + preconditioner applications inside cycles */
  int32_t converged;       /* 1 when ||M(b - A x)|| <= atol */
  int32_t pad;
  double residual_norm;    /* final preconditioned residual norm */
  double atol;             /* max(tol * ||b||, solver_atol) */
  double b_norm;
} SislSolveInfo;

/* Prognostic state + SISL history (the state pytree of steppers.py:69-80,
 * 1003-1071) in perturbation form. */
typedef struct SislState {
  void *u, *v, *w, *eta_dot, *pi_p, *th_p, *rho;
  void *u_prev, *v_prev, *w_prev, *eta_dot_prev, *tend_th_prev;
  double is_first_step;
} SislState;

/* Lateral relaxation applied as bc_fn (steppers.py:1042):
 * f <- (1 - mask) f + mask * exterior on horizontal masks (precision of the
 * core), e.g. the x relaxation of schaer_mountain_3d/run.py:104-126. */
typedef struct SislRelaxation {
  int32_t fields;          /* SISL_RELAX_* bitmask */
  int32_t pad;
  const void *mask_m, *mask_u, *mask_v;
  double ext[5];           /* exterior u, v, w, th_p, pi_p */
  const void* ext_field[5];/* optional 3-D exterior fields, override ext[] */
} SislRelaxation;

typedef struct SislStepInfo {
  SislSolveInfo solve[2];
  int64_t kernel_launches;
} SislStepInfo;

/* The last CUDA failure recorded by this thread (call, error name and
 * text), or "" (no reference counterpart: diagnostics of SISL_ERR_CUDA). */
const char* sisl_last_error(void);
int sisl_version(void);
const char* sisl_status_string(int status);
size_t sisl_field_elems(const SislGrid* grid, int loc);

/* Build the derived coefficient set of Euler3D.precompute_bg (euler.py:127-160)
 * and VerticalPreconditioner.precompute_banded (steppers.py:153-185) once. */
int sisl_core_create(const SislGrid* grid, const SislParams* params, const SislBackground* bg, void* stream,
                     SislCore** out);
int sisl_core_destroy(SislCore* core);
/* Replace the GMRES settings of SemiImplicitSolver3D(solver_tol,
 * solver_maxiter, solver_restart) (steppers.py:384-399) on an existing core. */
int sisl_core_set_solver(SislCore* core, double tol, double atol, int maxiter, int restart, int method);
/* Settings of the transposed (adjoint) solve, the bwd_solve of
 * steppers.py:473-481: tol <= 0 uses the forward solver_tol and method < 0
 * the forward SISL_GMRES_* variant (both as the reference does);
 * normalize_rhs = 1 (the default) solves for the cotangent scaled to unit
 * norm and rescales the result.  GMRES takes a preconditioned residual below
 * machine epsilon as zero (_safe_normalize); unnormalised, a cotangent of
 * small norm then stops after one cycle at a relative accuracy of
 * eps / ||M b||.  normalize_rhs = 0 reproduces that behaviour. */
int sisl_core_set_adjoint(SislCore* core, double tol, int normalize_rhs, int method);
/* Switch float64 iterative refinement of a float32 core's GMRES on or off
 * (on needs a core created with SislParams.refine = 1).  The solution and
 * right-hand side are held in float64 and every restart cycle starts from
 * the residual b - A x of the float64 operator; the Krylov cycle itself
 * (basis, matvec, preconditioner, Gram-Schmidt) stays in float32.  Without
 * it the float32 residual floor (~1e-7 relative) stalls tolerances below
 * about 1e-6.  No counterpart in the reference. */
int sisl_core_set_refinement(SislCore* core, int on);
size_t sisl_workspace_bytes(const SislCore* core, int what);

/* Euler3D.linear_operator(state_prime, bg, dt, alpha) (euler.py:374-439).
 * in/out: u, v, w, pi_p, eta_dot (physical). */
int sisl_linear_operator(SislCore* core, const void* const in[5], void* const out[5], void* ws, size_t ws_bytes,
                         void* stream);
/* SemiImplicitSolver3D.solve.A_fn (steppers.py:439-461): the matvec on the
 * scaled solver vector (u, v, w, pi * pi_scale, eta_dot * dz_w_full). */
int sisl_helmholtz_matvec(SislCore* core, const void* const in[5], void* const out[5], void* stream);
/* VerticalPreconditioner.__call__ (steppers.py:187-253) on the scaled vector.
 * out must not alias in (except u, v). */
int sisl_precond_apply(SislCore* core, const void* const in[5], void* const out[5], void* stream);
/* SemiImplicitSolver3D.solve(rhs_prime, bg, x0) (steppers.py:401-496):
 * physical rhs (u, v, w, pi_p, eta_dot) and x0 (NULL: x0 = rhs as in the
 * reference); x may alias x0. */
int sisl_gmres_solve(SislCore* core, const void* const rhs[5], const void* const x0[5], void* const x[5],
                     void* ws, size_t ws_bytes, void* stream, SislSolveInfo* info);
/* Exact transpose of A_fn (steppers.py:439-461), the matvec_T that
 * jax.lax.custom_linear_solve hands to bwd_solve (steppers.py:473-481).
 * ws: sisl_workspace_bytes(core, SISL_WS_OPERATOR) bytes; out must not alias in. */
int sisl_helmholtz_matvec_t(SislCore* core, const void* const in[5], void* const out[5], void* ws,
                            size_t ws_bytes, void* stream);
/* jax.linear_transpose(M_fn) of the column preconditioner (steppers.py:474-476).
 * out must not alias in. */
int sisl_precond_apply_t(SislCore* core, const void* const in[5], void* const out[5], void* stream);
/* bwd_solve of SemiImplicitSolver3D.solve (steppers.py:473-485): the cotangent
 * of the physical rhs from the cotangent of the physical solution, by GMRES on
 * A^T with preconditioner M^T and the settings of sisl_core_set_adjoint.
 * x0 NULL starts from zero as bwd_solve does; otherwise x0 (in the units of
 * bbar) is the initial guess, e.g. the previous step's result in a backward
 * sweep (same solution within the tolerance, fewer cycles). */
int sisl_gmres_solve_transpose(SislCore* core, const void* const xbar[5], const void* const x0[5],
                               void* const bbar[5], void* ws, size_t ws_bytes, void* stream, SislSolveInfo* info);
/* SemiLagrangianAdvector3D.compute_departure_indices(state, loc, iterations)
 * (steppers.py:318-360); coords[3] have the extents of stagger loc. */
int sisl_departure(SislCore* core, int loc, const void* u, const void* v, const void* eta_dot, int iterations,
                   void* const coords[3], void* ws, size_t ws_bytes, void* stream);
/* tensor_product_interp_3d(field, coords, use_limiter) (operators.py:146-209)
 * for any field shape and any coordinate-array shape (both x-fastest). */
int sisl_tricubic(int dtype, const int32_t src_shape[3], const void* field, const int32_t dst_shape[3],
                  const void* const coords[3], void* out, int use_limiter, void* stream);
/* VJP of tensor_product_interp_3d with respect to the field (operators.py:146-209;
 * the departure coordinates are stop-gradiented, steppers.py:764-767):
 * grad += scale * J^T cot, accumulated with atomics; field is read only with
 * the limiter, whose clip and min/max chains route the cotangent as lax.min
 * and lax.max do (ties split in half). */
int sisl_tricubic_vjp(int dtype, const int32_t src_shape[3], const void* field, const int32_t dst_shape[3],
                      const void* const coords[3], const void* cot, void* grad, int use_limiter, double scale,
                      void* stream);
/* Deterministic sisl_tricubic_vjp (same arguments and result, operators.py:
 * 146-209 under jax.vjp): every contribution is summed as a fixed-point
 * integer (scale 2^e chosen on the device from the largest |scale * cot|
 * and the densest stencil base, so no sum can overflow), then added to grad
 * with one rounding per element, so the gradient is the same bits on every
 * run (float atomics round in arrival order).  ws: 256-byte aligned,
 * sisl_tricubic_vjp_workspace_bytes(dtype, src_shape) bytes (one 64-bit
 * word per field element in float32; two in float64, the integer part and
 * a 32-bit fraction, so double contributions keep their precision). */
size_t sisl_tricubic_vjp_workspace_bytes(int dtype, const int32_t src_shape[3]);
int sisl_tricubic_vjp_deterministic(int dtype, const int32_t src_shape[3], const void* field,
                                    const int32_t dst_shape[3], const void* const coords[3], const void* cot,
                                    void* grad, int use_limiter, double scale, void* ws, size_t ws_bytes,
                                    void* stream);
/* CGridOperator3D.avg / .diff (operators.py:37-132) along one axis of an
 * x-fastest field of shape in_shape: to_face = 1 maps centres to faces
 * (n -> n+1, edge-padded or periodic), 0 faces to centres (n+1 -> n);
 * mult: optional 2-D (x-fastest) multiplier at the output stagger (the map
 * factor of diff).  transpose = 1 applies the transpose (src: output-shaped
 * cotangent, dst: input-shaped), with stop_grad dropping the padded copies
 * as jax.lax.stop_gradient does (operators.py:45-61). */
int sisl_stagger(int dtype, int op, const int32_t in_shape[3], int axis, int to_face, int periodic, int stop_grad,
                 int transpose, double inv_delta, const void* mult, const void* src, void* dst, void* stream);
/* map_coordinates(field, coords, order=1, mode='nearest'), the trilinear
 * gather of SemiLagrangianAdvector3D.advect_linear (steppers.py:362-367). */
int sisl_trilinear(int dtype, const int32_t src_shape[3], const void* field, const int32_t dst_shape[3],
                   const void* const coords[3], void* out, void* stream);
/* FluxFormAdvector.advect_1d(scalar_1d, cfl_inter_1d, periodic)
 * (steppers.py:552-594) on nlines independent lines: scalar is (nlines, n)
 * and cfl (nlines, n + 1), line-major; float64 workspace of
 * sisl_ffsl_lines_workspace_bytes(n, nlines) bytes. */
size_t sisl_ffsl_lines_workspace_bytes(int n, int nlines);
/* VJP of sisl_ffsl_lines: scalar_bar (n per line) and, where non-NULL,
 * cfl_bar (n + 1 per line), written, from out_bar, in the layouts of
 * sisl_ffsl_lines; float64 scratch of sisl_ffsl_lines_vjp_workspace_bytes. */
size_t sisl_ffsl_lines_vjp_workspace_bytes(int n, int nlines);
int sisl_ffsl_lines_vjp(int dtype, int n, int nlines, const void* scalar, const void* cfl, int periodic,
                        const void* out_bar, void* scalar_bar, void* cfl_bar, void* ws, size_t ws_bytes,
                        void* stream);
int sisl_ffsl_lines(int dtype, int n, int nlines, const void* scalar, const void* cfl, int periodic, void* out,
                    void* ws, size_t ws_bytes, void* stream);
/* Allocation-free sisl_ffsl_lines; no counterpart in the reference.
 * For callers that cannot call cudaMalloc while they run: a stream in
 * global-mode graph capture, a host model that allots this library only
 * buffers pre-sized from its own pool, an FFI handler registered without a
 * workspace.  The float64 scratch is a fixed device array of
 * SISL_FFSL_NOALLOC_MAX_DOUBLES doubles (8 MiB), held by every GPU that loads
 * the library until exit; a call needs (n + 1) * nlines doubles of it and
 * returns SISL_ERR_SCRATCH_LIMIT above that.  Nothing is allocated.  The
 * first call on a device looks up the array's device address (with that
 * device current), so make it before any stream capture.  All calls share
 * the one array: calls that overlap on the GPU (other streams, other host
 * threads) race and must be serialised by the caller. */
#define SISL_FFSL_NOALLOC_MAX_DOUBLES (1 << 20)
int sisl_ffsl_lines_noalloc(int dtype, int n, int nlines, const void* scalar, const void* cfl, int periodic,
                            void* out, void* stream);
/* Euler3D.metric_curvature_tendencies(u, v) (euler.py:188-206): the
 * map-curvature accelerations at the u faces (out_u) and v faces (out_v),
 * device layout.  No workspace. */
int sisl_metric_curvature(SislCore* core, const void* u, const void* v, void* out_u, void* out_v, void* stream);
/* Euler3D.get_tendencies(state_prime, bg, is_explicit) (euler.py:208-372):
 * is_explicit = 0 gives the linear tendencies of the implicit operator.
 * Same arguments as sisl_explicit_tendencies. */
int sisl_tendencies(SislCore* core, int is_explicit, const void* const state_prime[6], void* const tend[6],
                    void* const phys_diff[4], void* ws, size_t ws_bytes, void* stream);
/* Euler3D.get_tendencies(state_prime, bg, is_explicit=True) (euler.py:208-372)
 * and nonlinear_pi_tendency (euler.py:162-186).
 * state_prime: u, v, w, pi_p, eta_dot, th_p.
 * tend: u, v, w, pi (linear part), th_v, nonlinear pi; phys_diff: u, v, w, th_v. */
int sisl_explicit_tendencies(SislCore* core, const void* const state_prime[6], void* const tend[6],
                             void* const phys_diff[4], void* ws, size_t ws_bytes, void* stream);
/* VJP of sisl_explicit_tendencies: state_prime_bar (u, v, w, pi_p, eta_dot,
 * th_p; written) from the cotangents of tend (6) and phys_diff (4; the
 * array or any entry NULL: zero), with the reference's stop_gradient on
 * padded stagger copies (operators.py:37-63).
 * ws: sisl_workspace_bytes(core, SISL_WS_EXPLICIT_VJP) bytes. */
int sisl_explicit_tendencies_vjp(SislCore* core, const void* const state_prime[6], const void* const tend_bar[6],
                                 const void* const phys_diff_bar[4], void* const state_prime_bar[6], void* ws,
                                 size_t ws_bytes, void* stream);
/* FluxFormAdvector.advect_3d_split(field, state, bg) (steppers.py:596-647):
 * mass-conserving split transport of a mass-point density by u, v, eta_dot. */
int sisl_ffsl_advect(SislCore* core, const void* field, const void* u, const void* v, const void* eta_dot, void* out,
                     void* ws, size_t ws_bytes, void* stream);
/* VJP of sisl_ffsl_advect (XLA's reverse of steppers.py:552-647):
 * field_bar and, where non-NULL, u_bar, v_bar, eta_dot_bar (written) from
 * out_bar.  The clipped departure interfaces pass half the cotangent at an
 * exact tie (jnp.clip is maximum then minimum) and none beyond it.
 * ws: sisl_workspace_bytes(core, SISL_WS_FFSL_VJP) bytes. */
int sisl_ffsl_advect_vjp(SislCore* core, const void* field, const void* u, const void* v, const void* eta_dot,
                         const void* out_bar, void* field_bar, void* u_bar, void* v_bar, void* eta_dot_bar, void* ws,
                         size_t ws_bytes, void* stream);
/* Equation of state rho = p0 / (Rd th_v) pi^(cvd/Rd) (steppers.py:1055-1056)
 * from perturbation th_p, pi_p. */
int sisl_eos(SislCore* core, const void* th_p, const void* pi_p, void* rho, void* stream);
/* SISLStepper3D.step(state, t, forcing, bc_fn) (steppers.py:720-1073) with
 * bc_fn = identity (relax NULL) or a lateral relaxation.  in and out must not
 * overlap, except that out->*_prev may equal the matching in field. */
int sisl_step(SislCore* core, const SislState* in, const SislState* out, const SislRelaxation* relax, void* ws,
              size_t ws_bytes, void* stream, SislStepInfo* info);
/* sisl_step that also copies the physical solution (u, v, w, pi_p, eta_dot)
 * of each of its two implicit solves into solves[0..4] and solves[5..9]
 * (NULL entries skipped): the residuals a checkpointed VJP recomputation
 * reuses instead of solving again (jax.checkpoint of the step,
 * steppers.py:792-850). */
int sisl_step_taped(SislCore* core, const SislState* in, const SislState* out, const SislRelaxation* relax,
                    void* const solves[10], void* ws, size_t ws_bytes, void* stream, SislStepInfo* info);
/* SISLStepper3D.step with a physics suite (steppers.py:720-1073 with
 * Euler3D.get_tendencies' physics call, euler.py:347-366): phys_tend holds
 * the suite's explicit tendencies of u (u faces), v (v faces), w (w levels)
 * and th_v (mass points), NULL entries zero; they join the tendencies and
 * their phys_diff share exactly as the reference adds them.  The suite's
 * state updates, tracer transport and the caller's bc_fn follow on the
 * caller's side (sisl_ffsl_advect for tracers); relax may be NULL.  solves
 * as for sisl_step_taped (may be NULL). */
int sisl_step_physics(SislCore* core, const SislState* in, const SislState* out, const SislRelaxation* relax,
                      const void* const phys_tend[4], void* const solves[10], void* ws, size_t ws_bytes,
                      void* stream, SislStepInfo* info);
/* Split-explicit core (SplitExplicitStepper3D, steppers.py:1076-1737).
 * sisl_split_diagnose: eta_dot and the kinematic w boundaries of a state
 * (_diagnose_eta_dot, steppers.py:1272-1310); w_out may alias w.
 * sisl_split_step: the three RK3 stages with their acoustic sub-cycles
 * (ns acoustic steps in the last stage, round(ns/3) and round(ns/2) in the
 * first two; off-centring alpha) from a diagnosed state in (u, v, w,
 * eta_dot, pi_p, th_p) to out (same fields; rho is copied through, the
 * history fields are not used).  tau_damp: the Rayleigh damping rate at w
 * levels (Euler3D.tau_damp), in the core's precision and layout.
 * phys_tend: the physics suite's tendencies of u, v, w, th_v at the step
 * start (NULL entries, or NULL, for none); eps_l: the flux noise gate of
 * the upwind advection (constants 'eps_l', default 1e-12).  The suite's
 * updates, tracer transport, bc_fn, the final diagnosis and the equation of
 * state follow on the caller's side (steppers.py:1233-1270).  out must not
 * alias in.  ws: sisl_workspace_bytes(core, SISL_WS_SPLIT) bytes. */
int sisl_split_diagnose(SislCore* core, const void* u, const void* v, const void* w, void* eta_out, void* w_out,
                        void* stream);
int sisl_split_step(SislCore* core, const SislState* in, const SislState* out, int ns, double alpha, double eps_l,
                    const void* tau_damp, const void* const phys_tend[4], void* ws, size_t ws_bytes, void* stream);
/* Cotangents through sisl_split_diagnose (_diagnose_eta_dot,
 * steppers.py:1272-1310, as XLA differentiates it: the kinematic ground
 * value reads padded winds and carries none): from the cotangents of w_out
 * and eta_out, w_in_bar is written (may equal w_out_bar) and u_bar, v_bar
 * are accumulated.  ws: sisl_workspace_bytes(core, SISL_WS_SPLIT_VJP)
 * bytes (scratch of the fixed-point scatter). */
int sisl_split_diagnose_vjp(SislCore* core, const void* w_out_bar, const void* eta_bar, void* u_bar, void* v_bar,
                            void* w_in_bar, void* ws, size_t ws_bytes, void* stream);
/* Cotangent of sisl_split_step's input state from the cotangent of its
 * output (the VJP of SplitExplicitStepper3D's three RK3 stages,
 * steppers.py:1117-1231 and 1272-1737, as XLA differentiates them: the
 * padded copies of centre-to-face staggers and the sign of the upwind flux
 * carry no cotangent).  in, ns, alpha, eps_l, tau_damp: as given to
 * sisl_split_step (no physics tendencies); out_bar: cotangents of u, v, w,
 * eta_dot, pi_p, th_p (NULL members zero); in_bar receives the cotangents
 * of the same input fields and must not alias in or out_bar.  The first two
 * stage states are recomputed; the acoustic sub-steps are linear, so their
 * transposes need no recorded intermediates.  deterministic = 1: every
 * scatter sums in fixed point (the same bits on every run, two passes per
 * scatter kernel); 0: float atomic adds (one pass; the last bits depend on
 * the order the adds land).  ws: sisl_workspace_bytes(core,
 * SISL_WS_SPLIT_VJP) bytes. */
int sisl_split_step_vjp(SislCore* core, const SislState* in, const SislState* out_bar, const SislState* in_bar,
                        int ns, double alpha, double eps_l, const void* tau_damp, int deterministic, void* ws,
                        size_t ws_bytes, void* stream);
/* Cotangent of one step's input state from the cotangent of its output
 * (the VJP of SISLStepper3D.step under jax.checkpoint, steppers.py:720-1073,
 * 792-850, with the reference's stop_gradient on the departure points and
 * on padded stagger copies).  in, relax: the step's input and bc_fn as given
 * to sisl_step_taped; solves: that call's ten recorded solutions.
 * out_bar: cotangents of the output fields, NULL members are zero (the
 * history members u_prev .. tend_th_prev included).  in_bar: u, v, w,
 * eta_dot, pi_p, th_p receive the cotangents of the input state; rho and
 * the history members, where given, are zeroed (no cotangent).  The two
 * transposed solves follow sisl_core_set_adjoint and report in
 * info->solve[0..1].  in_bar must not overlap in, solves or out_bar.
 * ws: sisl_workspace_bytes(core, SISL_WS_STEP_VJP) bytes.  Every scatter
 * of the sweep (the six semi-Lagrangian interpolation VJPs and the explicit
 * and corrector stencil transposes) sums in fixed point and the Laplacian
 * transposes are gathers, so the cotangents are the same bits on every
 * run. */
int sisl_step_vjp(SislCore* core, const SislState* in, void* const solves[10], const SislRelaxation* relax,
                  const SislState* out_bar, const SislState* in_bar, void* ws, size_t ws_bytes, void* stream,
                  SislStepInfo* info);

/* CUDA graph of one step of n members (n >= 1; member m advances ins[m]
 * into outs[m] on core m with workspace ws[m]), captured once for these
 * buffers and replayed by sisl_step_graph_launch with no host
 * synchronisation.  Members are parallel branches of the graph; each GMRES
 * restart loop is a conditional WHILE node whose condition a kernel sets on
 * the device (rnorm > atol and cycles < maxiter), so a replay runs exactly
 * the cycles the host loop of sisl_step would.  The replay of lax.scan's
 * jitted step (steppers.py:692-714) in one launch; the ensemble launch of
 * the many-member configuration.  Cores must be distinct and have no timing
 * class selected; relax may be NULL (or hold NULL entries). */
/* Launch shapes of the Helmholtz kernels: stencil block variants (0-3:
 * 32x4x2, 32x8x1, 32x2x4, 64x4x1 threads; the matvec also 4 and 5: 32x8
 * columns of two or four levels per thread, 6-8: 32x4 columns marching
 * up the levels of 1, 2 or 4 z chunks with the vertical neighbours carried
 * in registers) of the matvec and of its transpose, and column
 * variants (0-2: tiles of 256 threads / 32 columns,
 * 128 / 16, 256 / 64; 3: one thread per column marching up and down the
 * precomputed factorisation, 128 columns per block) of the preconditioner
 * and of its transpose; the preconditioner also 4: the 256 / 32 tile with
 * its loads issued in batches of four items and the face sums of u and v
 * staged in shared memory, 5 and 6: one thread per column (64 columns per
 * block) marching with every level's loads issued two levels ahead, 6 with
 * L2 evict-last hints on the values the downward sweep reads again, 7: the
 * march fed by cp.async copies into a six-level shared-memory ring (32
 * columns per block); the
 * transpose also 4: the 256 / 32 tile with its loads issued in batches of
 * four items. */
typedef struct SislTuning {
  int32_t matvec_block, precond_tile, matvec_t_block, precond_t_tile;
  float us[4];  /* microseconds per launch of the chosen shapes (sisl_autotune only) */
} SislTuning;
/* Project autotuner (no reference counterpart): time every candidate shape
 * on this core's grid with CUDA events and keep the fastest in the core;
 * results are bitwise the same for every shape.  ws: sisl_workspace_bytes(
 * core, SISL_WS_GMRES) bytes; synchronises stream; not during a capture. */
int sisl_autotune(SislCore* core, void* ws, size_t ws_bytes, void* stream, SislTuning* out);
int sisl_autotune_query(const SislCore* core, SislTuning* out);
/* Apply stored launch shapes (e.g. a cached sisl_autotune result). */
int sisl_core_set_tuning(SislCore* core, const SislTuning* tuning);
typedef struct SislStepGraph SislStepGraph;
int sisl_step_graph_create(int n, SislCore* const* cores, const SislState* ins, const SislState* outs,
                           const SislRelaxation* const* relax, void* const* ws, const size_t* ws_bytes,
                           void* stream, SislStepGraph** out);
/* sisl_step_graph_create whose members also record their two solve
 * outputs, as sisl_step_taped: solves holds 10 pointers per member (member
 * m at solves[10 m ..]), NULL entries skipped; solves may be NULL. */
int sisl_step_graph_create_taped(int n, SislCore* const* cores, const SislState* ins, const SislState* outs,
                                 const SislRelaxation* const* relax, void* const* solves, void* const* ws,
                                 const size_t* ws_bytes, void* stream, SislStepGraph** out);
/* sisl_step_graph_create_taped with the members' solves grouped (no
 * reference counterpart; the batched ensemble launch): the explicit,
 * corrector and finalisation segments of every member stay parallel
 * branches, but each of the step's two solves runs as ONE restarted GMRES
 * over all members, every Krylov phase (matvec, preconditioner,
 * projections, update, small solves) a single launch that walks a
 * member/block table, and one device-decided WHILE node per solve that
 * loops while any member continues (convergence per member).  A member's
 * share of each grouped launch is its own launch's partition, so every
 * member's step is the same bits as with sisl_step_graph_create.  Members
 * share the dtype, GMRES restart and method and the refinement switch, and
 * have nz >= 2 (SISL_ERR_ARG otherwise). */
int sisl_step_graph_create_grouped(int n, SislCore* const* cores, const SislState* ins, const SislState* outs,
                                   const SislRelaxation* const* relax, void* const* solves, void* const* ws,
                                   const size_t* ws_bytes, void* stream, SislStepGraph** out);
/* The reverse sweep of a step (sisl_step_vjp) of n members as one CUDA graph:
 * member m maps out_bars[m] to in_bars[m] with its input ins[m] and the ten
 * recorded solutions solves[10 m ..]; the transposed GMRES loops are
 * device-decided conditional nodes, so a launch needs no host
 * synchronisation (the command-buffer form of the step's VJP).  ws[m]:
 * sisl_workspace_bytes(cores[m], SISL_WS_STEP_VJP) bytes.  Statistics of
 * the transposed solves: sisl_step_graph_info; release with
 * sisl_step_graph_destroy. */
int sisl_step_vjp_graph_create(int n, SislCore* const* cores, const SislState* ins, void* const* solves,
                               const SislRelaxation* const* relax, const SislState* out_bars,
                               const SislState* in_bars, void* const* ws, const size_t* ws_bytes, void* stream,
                               SislStepGraph** out);
/* sisl_step_vjp_graph_create with the members' transposed solves grouped as
 * in sisl_step_graph_create_grouped (one GMRES on A^T over all members per
 * solve, every Krylov phase one launch); every member's cotangents are the
 * same bits.  Members share the dtype, restart, the transposed solves'
 * GMRES method and the refinement switch. */
int sisl_step_vjp_graph_create_grouped(int n, SislCore* const* cores, const SislState* ins, void* const* solves,
                                       const SislRelaxation* const* relax, const SislState* out_bars,
                                       const SislState* in_bars, void* const* ws, const size_t* ws_bytes,
                                       void* stream, SislStepGraph** out);
int sisl_step_graph_launch(SislStepGraph* graph, void* stream);
/* Solve statistics of the last replay for one member (synchronises stream);
 * returns SISL_NOT_CONVERGED / SISL_ERR_NONFINITE like sisl_step. */
int sisl_step_graph_info(SislStepGraph* graph, int member, SislStepInfo* info, void* stream);
int sisl_step_graph_destroy(SislStepGraph* graph);

/* Instrumentation (no reference counterpart): number of kernels this library
 * launched, and CUDA-event timing of one kernel class inside GMRES (events
 * recorded around each launch on the launching stream; read after the
 * stream is synchronised) with the algorithmic bytes those launches move
 * (each distinct array touched once). */
int64_t sisl_kernel_launches(void);
int sisl_timing_select(SislCore* core, int kernel_class);
int sisl_timing_read(SislCore* core, double* total_ms, int64_t* launches, double* alg_bytes);

#ifdef __cplusplus
}
#endif

#endif /* SISL_B200_H */
