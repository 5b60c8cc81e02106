// Coefficient sets and host-side launch wrappers shared by the SISL kernels.
#pragma once

#include "sisl_common.cuh"

namespace sisl {

// Background / metric inputs in float64 (device pointers, device layout).
// Names follow the reference: theta_bg, pi_bg (euler.py:76-112), Z_m,
// dz_m_full, dz_w_full, z_xi_w, z_eta_w (geometry.py:232-261), tau_damp
// (euler.py:117-121), map factors, Coriolis and map-factor gradients
// (geometry.py:190-209).
struct Base64 {
  const double *theta_bg, *pi_bg, *Z_m, *dz_m, *dz_w, *z_xi_w, *z_eta_w, *tau;
  const double *m_m, *m_u, *m_v, *f_u, *f_v, *dmdx, *dmdy;
  const double* rho;  // background density, NULL: the equation of state of theta_bg, pi_bg
};

// Physical and solver scalars.
struct Scalars {
  double dt, alpha, g, cp, Rd, cvd, p0, ps, nu_div, nu_h;
};

// Derived coefficient arrays in working precision T.  Every array is
// computed once per core in float64 from Base64 and cast.
template <typename T>
struct Coef {
  // mass points
  const T *thb;    // theta_bg
  const T *pib;    // pi_bg
  const T *cpidz;  // C_pi / dz_m_full  (C_pi = Rd/cvd * pi/(rho theta), euler.py:157)
  const T *dthm;   // avg_w->m( d theta_bg/dz )  (euler.py:321-322)
  const T *lpi;    // alpha dt C_pi / dz_m  (steppers.py:180)
  const T *zxm, *zem;  // avg_u->m z_xi_u, avg_v->m z_eta_v (diffusion.py:117,125)
  const T *dzm;        // dz_m_full (geometry.py:242)
  // u faces
  const T *thu, *zxu, *rdu;  // th_v_u, z_xi_u (incl. m_u), rho_u dz_u / m_u
  // v faces
  const T *thv, *zev, *rdv;
  // w levels
  const T *thw, *rhow, *idzw, *dzw, *damp, *zxw, *zew;  // damp = 1 + dt tau
  // horizontal 2-D
  const T *mm, *mu, *mv, *fu, *fv, *dmdx, *dmdy;
  // column Helmholtz system of the preconditioner, factorised once
  // (steppers.py:171-185): lower(k) = -L_pi(k) P(k), and the Thomas factors
  // c'(k) and 1/pivot(k) of T = L U (mass levels); rho_w th_w, the w
  // back-substitution factor adt cp th_w / (dz_w (1 + dt tau)) and
  // 1/(1 + dt tau) (w levels)
  const T *tlo, *tcp, *tinv, *rtw, *pbw, *idamp;
  Scalars s;
};

enum CoefId {
  C_THB, C_PIB, C_CPIDZ, C_DTHM, C_LPI, C_ZXM, C_ZEM, C_DZM,
  C_THU, C_ZXU, C_RDU, C_THV, C_ZEV, C_RDV,
  C_THW, C_RHOW, C_IDZW, C_DZW, C_DAMP, C_ZXW, C_ZEW,
  C_MM, C_MU, C_MV, C_FU, C_FV, C_DMDX, C_DMDY,
  C_TLO, C_TCP, C_TINV, C_RTW, C_PBW, C_IDAMP,
  C_COUNT
};
int coef_loc(int id);      // LOC_* of a 3-D coefficient, or -1 for 2-D
size_t coef_elems(const Dims& d, int id);

template <typename T>
struct PtrTable {
  T* p[C_COUNT];
};

template <typename T>
Coef<T> make_coef(T* const* arrays, const Scalars& s);

// ---- preparation ----
template <typename T>
void launch_prepare(const Dims& d, const Scalars& s, const Base64& b, PtrTable<T> out, cudaStream_t st);

// ---- linear algebra on the 5-field solver vector (u, v, w, pi*ps, eta*dz_w) ----
// All five fields are passed as separate pointers.
template <typename T>
struct Vec5 {
  T* f[5];
};
template <typename T>
struct CVec5 {
  const T* f[5];
};

// out = A(x * xs) or out = b - A(x * xs) (residual mode, when b != nullptr)
template <typename T>
void launch_matvec(const Dims& d, const Coef<T>& c, CVec5<T> x, const double* xscale, CVec5<T> b,
                   Vec5<T> out, const int* active, cudaStream_t st);
template <typename T>
void launch_precond(const Dims& d, const Coef<T>& c, CVec5<T> r, Vec5<T> out, const int* active,
                    cudaStream_t st);

// transposes for the adjoint solve (sisl_adjoint.cu): out = A^T(y * ys), or
// out = b - A^T(y * ys); gzm_tmp is a mass-point scratch field.  out = M^T y.
template <typename T>
void launch_matvec_t(const Dims& d, const Coef<T>& c, CVec5<T> y, const double* yscale, CVec5<T> b, Vec5<T> out,
                     T* gzm_tmp, const int* active, cudaStream_t st);
template <typename T>
void launch_precond_t(const Dims& d, const Coef<T>& c, CVec5<T> y, Vec5<T> out, const int* active,
                      cudaStream_t st);

// grad += scale * (d tricubic / d field)^T cot  (coordinates carry no cotangent)
template <typename T>
void launch_tricubic_vjp(int sx, int sy, int sz, int dx, int dy, int dz, const T* field, const T* const* coords3,
                         const T* cot, T* grad, int use_limiter, T scale, cudaStream_t st);

// the same, deterministic: contributions summed as fixed-point integers in
// scratch (tricubic_vjp_det_scratch_bytes of the field shape and element
// size), so the result is bitwise reproducible
size_t tricubic_vjp_det_scratch_bytes(int sx, int sy, int sz, int elem_bytes);
// relative = 1: coords3 hold split-form offsets of the destination points
// (source and destination shapes equal)
template <typename T>
void launch_tricubic_vjp_det(int sx, int sy, int sz, int dx, int dy, int dz, const T* field,
                             const T* const* coords3, const T* cot, T* grad, int use_limiter, T scale, void* scratch,
                             int relative, cudaStream_t st);

// staggered average / difference along one axis and its transpose (sisl_stagger.cu)
template <typename T>
void launch_stagger(const int in_shape[3], int axis, int to_face, int periodic, int stop_grad, int transpose, T c0,
                    T c1, const T* mult, const T* src, T* dst, cudaStream_t st);

// ---- semi-Lagrangian ----
// vel.p[3*loc + 0..2] = index velocities (u m/dx, v m/dy, eta_dot) at stagger loc
template <typename T>
void launch_traj_velocity(const Dims& d, const Coef<T>& c, const T* u, const T* v, const T* eta, const T* up,
                          const T* vp, const T* etap, int extrapolate, PtrTable<T> vel, cudaStream_t st);
// relative = 1: the coordinates are written as split-form offsets -alpha
// (the point is index + offset), relative = 0 as index - alpha
template <typename T>
void launch_departure(const Dims& d, int loc, double dt, const T* const* vel3, int iterations,
                      T* const* coords3, int relative, cudaStream_t st);
// tricubic of a (sx, sy, sz) field at the points of a (dx, dy, dz) coordinate array
template <typename T>
void launch_tricubic_ext(int sx, int sy, int sz, int dx, int dy, int dz, const T* field, const T* const* coords3,
                         T* out, int use_limiter, T scale, cudaStream_t st);
template <typename T>
void launch_trilinear_ext(int sx, int sy, int sz, int dx, int dy, int dz, const T* field, const T* const* coords3,
                          T* out, cudaStream_t st);
// fused: departure point of every `loc` point, then tricubic of nf <= 2 fields
template <typename T>
void launch_sl_advect(const Dims& d, int loc, double dt, const T* const* vel3, int iterations, int nf,
                      const T* const* fields, T* const* outs, const T* scales, int use_limiter,
                      cudaStream_t st);

// ---- FFSL and EOS (sisl_ffsl.cu) ----
size_t ffsl_scratch_doubles(const Dims& d);
template <typename T>
int launch_ffsl(const Dims& d, const Coef<T>& c, const T* field, const T* u, const T* v, const T* eta, T* out,
                T* tmp0, T* tmp1, double* M, cudaStream_t st);
template <typename T>
int launch_ffsl_vjp(const Dims& d, const Coef<T>& c, const T* field, const T* u, const T* v, const T* eta,
                    const T* out_bar, T* field_bar, T* u_bar, T* v_bar, T* eta_bar, T* const* tmp, double* M,
                    double* Mb, cudaStream_t st);
template <typename T>
void launch_ffsl_lines_vjp(int N, int nlines, const T* scalar, const T* cfl, const T* out_bar, T* scalar_bar,
                           T* cfl_bar, double* M, double* Mb, int periodic, cudaStream_t st);
template <typename T>
void launch_ffsl_lines(int N, int nlines, const T* scalar, const T* cfl, T* out, double* M, int periodic,
                       cudaStream_t st);
template <typename T>
void launch_eos(const Dims& d, const Coef<T>& c, const T* th, const T* pi, T* rho, cudaStream_t st);

// ---- GMRES building blocks (sisl_gmres.cu) ----
struct GState;
struct GHostView;
template <typename T>
void gm_dots(const T* Vb, size_t stride, int m, const T* w, size_t n, double* partial, GState* gs, int mode,
             int gated, cudaStream_t st);
template <typename T>
void gm_update(const T* Vb, size_t stride, int m, T* w, size_t n, double sign, double* partial, GState* gs,
               int mode, int gated, int limit_kdone, cudaStream_t st);
template <typename T>
void gm_update_x64(const T* Vb, size_t stride, int m, double* x, size_t n, const GState* gs, cudaStream_t st);
void gm_setup(GState* gs, double eps, double tol, double atol_in, int restart, int method, cudaStream_t st);
void gm_init_tol(GState* gs, cudaStream_t st);
struct GDevInfo;
void gm_gate(GState* gs, cudaGraphConditionalHandle h, int maxiter, int after_cycle, cudaStream_t st);
void gm_info(const GState* gs, GDevInfo* o, cudaStream_t st);
void gm_begin_cycle(GState* gs, cudaStream_t st);
void gm_small_solve(GState* gs, int restart, cudaStream_t st);
void gm_snapshot(const GState* gs, GHostView* v, cudaStream_t st);

}  // namespace sisl
