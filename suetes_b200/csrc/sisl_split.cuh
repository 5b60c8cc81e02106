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
  const T *sfu, *sfv, *sfw, *sfp, *sfth;  // slow forcings
  const T* tau;                      // tau_damp at w levels
  T *cpr, *dpr;                      // Thomas scratch (mass points)
  T dtau, alpha, nu_div;
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

}  // namespace sisl
