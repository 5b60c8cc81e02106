// Argument structs and launchers of the reverse sweep of the SISL step.
#pragma once

#include "sisl_explicit.cuh"
#include "sisl_split.cuh"

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

// Deterministic scatter of the explicit and corrector VJP kernels: the
// fields a launch accumulates into are registered in a DetSink; a first run
// of the kernel records each field's largest |contribution| (mode 1), a
// second adds every contribution as a fixed-point integer (mode 2: one
// 64-bit word per element in float32, an integer and a 32-bit fraction word
// in float64), and a finish kernel adds the sums to the fields with one
// rounding per element.  Integer sums do not depend on the order the
// atomics land, so the cotangents are the same bits on every run.  Mode 0:
// plain float atomic adds.
constexpr int DET_FIELDS = 16;
template <typename T>
struct DetSink {
  int mode, n;
  T* dst[DET_FIELDS];
  unsigned len[DET_FIELDS];
  unsigned long long* acc[DET_FIELDS];
  unsigned* gmax;  // DET_FIELDS words: float bits of the largest |contribution| per field
};
// scratch of a deterministic scatter into up to DET_FIELDS fields of at most
// (nx+1)(ny+1)(nz+1) elements
size_t det_scatter_scratch_bytes(const Dims& d, int elem_bytes);

// det_scratch: NULL for float atomics, else det_scatter_scratch_bytes(d, sizeof(T))
// bytes (256-byte aligned) for the deterministic scatter
template <typename T>
void launch_explicit_vjp(const Dims& d, const Coef<T>& c, const ExplicitIn<T>& in, const ExplicitBar<T>& bi,
                         const StateBar<T>& bo, int mode, void* det_scratch, cudaStream_t st);
template <typename T>
void launch_corrector_vjp(const Dims& d, const Coef<T>& c, const CorrectorIn<T>& in, const CorrectorBar<T>& cb,
                          void* det_scratch, cudaStream_t st);
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
