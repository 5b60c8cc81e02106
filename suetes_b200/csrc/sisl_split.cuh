// Split-explicit RK3 core (SplitExplicitStepper3D, steppers.py:1076-1737):
// argument struct and launchers.  The slow tendencies reuse the explicit
// kernel (mode 1); these kernels add the 3rd-order upwind flux advection,
// the forward-backward acoustic sub-step with its vertically implicit
// column solve, and the eta_dot diagnosis.
#pragma once

#include "sisl_core.cuh"

namespace sisl {

template <typename T>
struct SplitArgs {
  const T *u0, *v0, *w0, *p0, *th0;  // state at the start of the step (pi', th')
  const T *uc, *vc, *wc, *pc, *ec;   // state at the start of the stage
  T *upp, *vpp, *wpp, *ppp;          // acoustic perturbations u'', v'', w'', pi''
  T *uh, *vh;                        // midpoint winds of the acoustic sub-step
  T *gx0, *gy0;                      // horizontal pressure gradients of the old pi''
  // the corrector's gradients of the new pi'' (NULL: not kept); the next
  // sub-step's predictor takes them as its gx0, gy0 (same pi'', same bits)
  // when gx0_ready is set instead of forming them again
  T *gx1, *gy1;
  const T *sfu, *sfv, *sfw, *sfp, *sfth;  // slow forcings
  const T* tau;                      // tau_damp at w levels
  T *cpr, *dpr;                      // Thomas scratch (mass points)
  T dtau, alpha, nu_div;
  int gx0_ready;
};

// eta_dot and the kinematic w boundaries of a state (steppers.py:1272-1310);
// w_out may alias w_in.
template <typename T>
void launch_split_diag(const Dims& d, const Coef<T>& c, const T* u, const T* v, const T* w_in, T* eta_out,
                       T* w_out, cudaStream_t st);
// upwind flux advection of th', u_m, v_m, w_m at mass points (steppers.py:1312-1465)
template <typename T>
void launch_split_adv(const Dims& d, const Coef<T>& c, const T* u, const T* v, const T* w, const T* eta,
                      const T* th, T eps_l, T* const* adv4, cudaStream_t st);
// slow forcings: explicit tendencies (f[0..5] of the explicit kernel's
// mode 1) plus the advection averaged to the staggers
template <typename T>
void launch_split_slow(const Dims& d, const T* const* tend6, const T* const* adv4, T* const* sf5, cudaStream_t st);
template <typename T>
void launch_split_init(const Dims& d, const SplitArgs<T>& a, cudaStream_t st);
template <typename T>
void launch_split_predict(const Dims& d, const Coef<T>& c, const SplitArgs<T>& a, cudaStream_t st);
template <typename T>
void launch_split_column(const Dims& d, const Coef<T>& c, const SplitArgs<T>& a, cudaStream_t st);
// the corrected u'', v'' go to upp2, vpp2 (the caller swaps the buffers)
template <typename T>
void launch_split_correct(const Dims& d, const Coef<T>& c, const SplitArgs<T>& a, T* upp2, T* vpp2,
                          cudaStream_t st);
// stage state: x = x_stage + x'' (u, v, w, pi'), th' = th'_0 + dtau ns S_th, eta copied
template <typename T>
void launch_split_end(const Dims& d, const SplitArgs<T>& a, int nsteps, T* u, T* v, T* w, T* eta, T* p, T* th,
                      cudaStream_t st);
// a += b over n elements (hyperdiffusion of the stage plus that of the step start)
template <typename T>
void launch_split_axpy(size_t n, const T* b, T* a, cudaStream_t st);

// ---------------------------------------------------------------------------
// Reverse sweep (sisl_step_vjp.cu).  Every acoustic sub-step is linear in
// the state (its matrices are background coefficients), so its transposes
// need no recorded intermediates; the slow tendencies are re-formed at the
// recomputed stage-start states.  Scatters go through a fixed-point sink
// when det_scratch is given (det_scatter_scratch_bytes), so the cotangents
// are the same bits on every run.
// ---------------------------------------------------------------------------
template <typename T>
struct SplitBar {
  T *upp, *vpp;              // u'', v'' at the sub-step start (accumulated)
  const T *upp2, *vpp2;      // u'', v'' after the corrector
  T *wpp, *ppp;              // w'', pi'' (in place: after -> before)
  T *uh, *vh, *gx0, *gy0;    // midpoint winds and old pressure gradients
  T *sfu, *sfv, *sfw, *sfp;  // slow forcings (accumulated)
  T *uc, *vc, *wc;           // stage-start state (accumulated)
  T *u0, *v0;                // step start (accumulated: the boundary faces)
  T *s1, *s2;                // column scratch at mass points
  const T* tau;              // tau_damp at w levels
  T dtau, alpha, nu_div;
};
// w, eta_dot cotangents of split_diag into w (in place), u, v (accumulated);
// eta_dot's cotangent is consumed (zeroed)
template <typename T>
void launch_split_diag_vjp(const Dims& d, const Coef<T>& c, T* wb, T* eb, T* ub, T* vb, void* det_scratch,
                           cudaStream_t st);
// the reverse of one acoustic sub-step: corrector, column, predictor
template <typename T>
void launch_split_substep_vjp(const Dims& d, const Coef<T>& c, const SplitBar<T>& b, void* det_scratch,
                              cudaStream_t st);
// split_end^T: out6 (u, v, w, eta, pi, th cotangents of the stage state) ->
// stage-start c6 (accumulated; th into the step start's th0b), u'', v'', w'',
// pi'' (written) and the th' slow forcing (written, times dtau nsteps)
template <typename T>
void launch_split_end_vjp(const Dims& d, const T* const* out6, T* const* c6, T* th0b, T* upp, T* vpp, T* wpp,
                          T* ppp, T* sfth, T dtns, cudaStream_t st);
// split_init^T: u'' = u0 - uc, ... (accumulated into the step start s6 and the stage start c6)
template <typename T>
void launch_split_init_vjp(const Dims& d, const T* upp, const T* vpp, const T* wpp, const T* ppp, T* const* s6,
                           T* const* c6, cudaStream_t st);
// split_slow^T: sf5 -> tend6 (written) and adv4 (accumulated)
template <typename T>
void launch_split_slow_vjp(const Dims& d, const T* const* sf5, T* const* tend6, T* const* adv4, void* det_scratch,
                           cudaStream_t st);
// split_adv^T at the stage-start state: adv4 -> u, v, w, eta_dot, th' (accumulated)
template <typename T>
void launch_split_adv_vjp(const Dims& d, const Coef<T>& c, const T* u, const T* v, const T* w, const T* eta,
                          const T* th, T eps_l, const T* const* adv4, T* ub, T* vb, T* wb, T* eb, T* thb,
                          void* det_scratch, cudaStream_t st);

}  // namespace sisl
