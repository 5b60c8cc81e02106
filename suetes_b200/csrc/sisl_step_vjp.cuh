// Argument structs and launchers of the reverse sweep of the SISL step.
#pragma once

#include "sisl_explicit.cuh"

namespace sisl {

// Cotangents of the explicit kernel's outputs (ExplicitOut, same modes);
// a null pointer is a zero cotangent.
template <typename T>
struct ExplicitBar {
  const T* f[7];
  const T* pd[4];  // mode 1 only: cotangents of the phys_diff outputs
};

// Accumulated cotangents of the explicit kernel's inputs.  hyper: cotangents
// of the hyperdiffusion tendencies at mass points (null when nu_h == 0).
template <typename T>
struct StateBar {
  T *u, *v, *w, *eta, *pi, *th;
  T* hyper[4];
};

// Cotangents around the predictor-corrector right-hand side (CorrectorIn).
template <typename T>
struct CorrectorBar {
  const T* b[5];                              // cotangent of the solve's right-hand side u, v, w, pi, eta
  T *rhs_u, *rhs_v, *rhs_w, *rhs_pi, *reta;   // accumulated
  T* th;                                      // theta' predictor
  T* pg;                                      // pi' of the guess
  T *gu, *gv, *geta;                          // guess of the nonlinear continuity
  T *ug, *vg;                                 // winds of the map curvature
};

// Reverse of the finalisation (divergence damping, relaxation, EOS).
template <typename T>
struct FinalizeBar {
  const T *th2, *pi2;                             // theta' predictor and pi' of the second solve
  const T *u, *v, *w, *eta, *pi, *th, *rho;       // cotangents of the step outputs (null: zero)
  T *x2u, *x2v, *x2w, *x2pi, *x2eta, *th2b;       // written
  Relax<T> relax;
};

template <typename T>
void launch_explicit_vjp(const Dims& d, const Coef<T>& c, const ExplicitIn<T>& in, const ExplicitBar<T>& bi,
                         const StateBar<T>& bo, int mode, cudaStream_t st);
template <typename T>
void launch_corrector_vjp(const Dims& d, const Coef<T>& c, const CorrectorIn<T>& in, const CorrectorBar<T>& cb,
                          cudaStream_t st);
template <typename T>
void launch_corrector_theta_vjp(const Dims& d, const Coef<T>& c, const T* thn_bar, T* tha_bar, T* tth_bar,
                                T* w_now_bar, T* w_next_bar, cudaStream_t st);
template <typename T>
void launch_fixup_vjp(const Dims& d, T* ru_bar, T* rv_bar, T* u_bar, T* v_bar, T* reta_bar, cudaStream_t st);
template <typename T>
void launch_finalize_vjp(const Dims& d, const Coef<T>& c, const FinalizeBar<T>& fb, T* div_bar, cudaStream_t st);
// out (state cotangents, accumulated) += hyperdiffusion^T(hyp_bar); hyp_bar
// and the temporaries are overwritten.
template <typename T>
void launch_hyper_vjp(const Dims& d, const Coef<T>& c, PtrTable<T> hyp_bar, PtrTable<T> gx4, PtrTable<T> gy4,
                      PtrTable<T> tmp4, T* u_bar, T* v_bar, T* w_bar, T* th_bar, cudaStream_t st);

}  // namespace sisl
