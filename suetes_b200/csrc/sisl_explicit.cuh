// Argument structs and launchers of the explicit-step kernels.
#pragma once

#include "sisl_core.cuh"

namespace sisl {

template <typename T>
struct ExplicitIn {
  const T *u, *v, *w, *eta, *pi, *th;  // pi' and th' (perturbations)
  const T* hyper[4];                   // hyperdiffusion tendencies of u, v, w, th' at mass points, or null
  const T* extra[4];                   // physics-suite tendencies of u, v, w (own staggers), th (mass), or null
};
// mode 0: f = {u_in, v_in, w_in, pi_in, th_in, tend_th, residual_n}
// mode 1: f = {tend_u, tend_v, tend_w, tend_pi, tend_th, nl_pi, -}, pd = phys_diff u, v, w, th
template <typename T>
struct ExplicitOut {
  T* f[7];
  T* pd[4];
};

template <typename T>
struct CorrectorIn {
  const T *rhs_u, *rhs_v, *rhs_w, *rhs_pi;  // advected right-hand sides
  const T* th_next;                         // theta' predictor
  const T* pg;                              // pi' of the current guess
  const T *gu, *gv, *geta;                  // current guess (nonlinear continuity)
  const T *ug, *vg;                         // winds for curvature / kinematic bottom
};

enum RelaxFields { RELAX_U = 1, RELAX_V = 2, RELAX_W = 4, RELAX_TH = 8, RELAX_PI = 16 };

// Lateral relaxation f <- (1 - mask) f + mask ext on horizontal masks.
template <typename T>
struct Relax {
  int on;                    // RelaxFields bitmask
  const T *mask_m, *mask_u, *mask_v;
  T ext[5];                  // exterior values of u, v, w, th', pi' (perturbation form)
  const T* ext_field[5];     // optional 3-D exterior fields (override ext[])
};

template <typename T>
struct FinalizeArgs {
  const T *u_in, *v_in;      // solved winds
  T *u_out, *v_out;          // damped + relaxed winds
  const T* div;              // horizontal divergence, or null when nu_div == 0
  T *w_io, *th_io, *pi_io;   // relaxed in place
  T* rho_out;                // EOS density, or null
  Relax<T> relax;
};

// gxy8: scratch of the face gradients (p[0..3] u faces, p[4..7] v faces) of
// the two-pass Laplacian
template <typename T>
void launch_hyper(const Dims& d, const Coef<T>& c, const T* u, const T* v, const T* w, const T* th,
                  PtrTable<T> tmp4, PtrTable<T> out4, PtrTable<T> gxy8, cudaStream_t st);
template <typename T>
void launch_explicit(const Dims& d, const Coef<T>& c, const ExplicitIn<T>& in, const ExplicitOut<T>& out, int mode,
                     cudaStream_t st);
// map-curvature accelerations at the u and v faces (euler.py:188-206)
template <typename T>
void launch_curvature(const Dims& d, const Coef<T>& c, const T* u, const T* v, T* ou, T* ov, cudaStream_t st);
template <typename T>
void launch_corrector_theta(const Dims& d, const Coef<T>& c, const T* th_adv, const T* tth, const T* w_now,
                            const T* w_next, T* th_next, cudaStream_t st);
template <typename T>
void launch_corrector_rhs(const Dims& d, const Coef<T>& c, const CorrectorIn<T>& in, Vec5<T> out, cudaStream_t st);
template <typename T>
void launch_hdiv(const Dims& d, const Coef<T>& c, const T* u, const T* v, T* div, cudaStream_t st);
template <typename T>
void launch_finalize(const Dims& d, const Coef<T>& c, const FinalizeArgs<T>& fa, cudaStream_t st);

}  // namespace sisl
