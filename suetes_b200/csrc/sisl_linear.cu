// Helmholtz matvec and column (Thomas) preconditioner on the scaled solver
// vector (u, v, w, pi * pi_scale, eta_dot * dz_w_full).
//
// Matvec: Euler3D.linear_operator (euler.py:374-439) with the linear
// tendencies of get_tendencies(is_explicit=False) (euler.py:208-318),
// wrapped in the scaling of SemiImplicitSolver3D.solve.A_fn
// (steppers.py:439-461).  One fused pass: every output of the five fields at
// a point of the (nx+1, ny+1, nz+1) union box is produced by one thread.
//
// Preconditioner: VerticalPreconditioner.__call__ (steppers.py:187-253), one
// thread per (i, j) column: kinematic forcing, Helmholtz RHS, Thomas forward
// and back substitution with the factorisation prepared once per core, then
// the w and eta_dot back-substitution.
#include "sisl_core.cuh"

namespace sisl {
namespace {

template <typename T>
struct MV {
  const Dims& d;
  const Coef<T>& c;
  const T* __restrict__ xp;
  T sp;  // xscale / pi_scale
  __device__ __forceinline__ T P(int i, int j, int k) const { return ld(xp, im(d, i, j, k)) * sp; }
  // d pi / dz at w level k, edge-padded (euler.py:252)
  __device__ __forceinline__ T gzw(int i, int j, int k) const {
    int kl, kr;
    level_pair(k, d.nz, kl, kr);
    return (P(i, j, kr) - P(i, j, kl)) * ld(c.idzw, iw(d, i, j, k));
  }
  __device__ __forceinline__ T gzm(int i, int j, int k) const {
    return T(0.5) * (gzw(i, j, k) + gzw(i, j, k + 1));
  }
};

template <typename T>
__global__ void __launch_bounds__(256) matvec_kernel(Dims d, Coef<T> c, CVec5<T> x, const double* xscale,
                                                     CVec5<T> b, Vec5<T> out, const int* active) {
  if (active && *active == 0) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i > nx || j > ny || k > nz) return;
  const T xs = xscale ? (T)(*xscale) : T(1);
  const T adt = (T)(c.s.alpha * c.s.dt);
  const T cp = (T)c.s.cp;
  const T a = (T)c.s.alpha;
  const T ps = (T)c.s.ps;
  MV<T> mv{d, c, x.f[3], xs / ps};
  const T* __restrict__ xu = x.f[0];
  const T* __restrict__ xv = x.f[1];
  const T* __restrict__ xw = x.f[2];
  const T* __restrict__ xW = x.f[4];
  const T idx = (T)(1.0 / d.dx), idy = (T)(1.0 / d.dy);

  // ---------------- u faces ----------------
  if (j < ny && k < nz) {
    const int p = iu(d, i, j, k);
    T L;
    if (!d.px && (i == 0 || i == nx)) {
      L = ld(xu, p) * xs;  // locked open boundary (euler.py:414-415)
    } else {
      const int ic = (d.px && i == nx) ? 0 : i;  // periodic endpoint copy (euler.py:412)
      const int pc = iu(d, ic, j, k);
      int l, r;
      face_pair(ic, nx, d.px, l, r);
      const T gpx = (mv.P(r, j, k) - mv.P(l, j, k)) * idx * ld(c.mu, h_u(d, ic, j));
      const T gpzu = T(0.5) * (mv.gzm(l, j, k) + mv.gzm(r, j, k));
      const T vml = T(0.5) * (ld(xv, iv(d, l, j, k)) + ld(xv, iv(d, l, j + 1, k))) * xs;
      const T vmr = T(0.5) * (ld(xv, iv(d, r, j, k)) + ld(xv, iv(d, r, j + 1, k))) * xs;
      const T vat = T(0.5) * (vml + vmr);
      const T tend = -cp * ld(c.thu, pc) * (gpx - ld(c.zxu, pc) * gpzu) + ld(c.fu, h_u(d, ic, j)) * vat;
      L = ld(xu, pc) * xs - adt * tend;
    }
    if (b.f[0]) L = ld(b.f[0], p) - L;
    out.f[0][p] = L;
  }
  // ---------------- v faces ----------------
  if (i < nx && k < nz) {
    const int p = iv(d, i, j, k);
    T L;
    if (!d.py && (j == 0 || j == ny)) {
      L = ld(xv, p) * xs;
    } else {
      const int jc = (d.py && j == ny) ? 0 : j;
      const int pc = iv(d, i, jc, k);
      int l, r;
      face_pair(jc, ny, d.py, l, r);
      const T gpy = (mv.P(i, r, k) - mv.P(i, l, k)) * idy * ld(c.mv, h_v(d, i, jc));
      const T gpzv = T(0.5) * (mv.gzm(i, l, k) + mv.gzm(i, r, k));
      const T uml = T(0.5) * (ld(xu, iu(d, i, l, k)) + ld(xu, iu(d, i + 1, l, k))) * xs;
      const T umr = T(0.5) * (ld(xu, iu(d, i, r, k)) + ld(xu, iu(d, i + 1, r, k))) * xs;
      const T uat = T(0.5) * (uml + umr);
      const T tend = -cp * ld(c.thv, pc) * (gpy - ld(c.zev, pc) * gpzv) - ld(c.fv, h_v(d, i, jc)) * uat;
      L = ld(xv, pc) * xs - adt * tend;
    }
    if (b.f[1]) L = ld(b.f[1], p) - L;
    out.f[1][p] = L;
  }
  // ---------------- w levels: w and eta_dot rows ----------------
  if (i < nx && j < ny) {
    const int p = iw(d, i, j, k);
    T Lw, Le;
    if (k == 0 || k == nz) {
      Lw = ld(xw, p) * xs;                          // euler.py:426-427
      Le = ld(xW, p) * xs * ld(c.idzw, p);          // eta_dot = W / dz_w (euler.py:436-437)
    } else {
      const T tend = -cp * ld(c.thw, p) * mv.gzw(i, j, k);
      Lw = ld(c.damp, p) * ld(xw, p) * xs - adt * tend;
      // u, v averaged to w (euler.py:404-407)
      const T umk = T(0.5) * (ld(xu, iu(d, i, j, k)) + ld(xu, iu(d, i + 1, j, k)));
      const T umkm = T(0.5) * (ld(xu, iu(d, i, j, k - 1)) + ld(xu, iu(d, i + 1, j, k - 1)));
      const T vmk = T(0.5) * (ld(xv, iv(d, i, j, k)) + ld(xv, iv(d, i, j + 1, k)));
      const T vmkm = T(0.5) * (ld(xv, iv(d, i, j, k - 1)) + ld(xv, iv(d, i, j + 1, k - 1)));
      const T uw = T(0.5) * (umkm + umk) * xs;
      const T vw = T(0.5) * (vmkm + vmk) * xs;
      const T mw = ld(c.mm, h_m(d, i, j));
      Le = a * (ld(xW, p) * xs + mw * (uw * ld(c.zxw, p) + vw * ld(c.zew, p)) - ld(xw, p) * xs);
    }
    if (b.f[2]) { Lw = ld(b.f[2], p) - Lw; Le = ld(b.f[4], p) - Le; }
    out.f[2][p] = Lw;
    out.f[4][p] = Le;
  }
  // ---------------- mass points: pi row ----------------
  if (i < nx && j < ny && k < nz) {
    const int p = im(d, i, j, k);
    const T fx0 = ld(xu, iu(d, i, j, k)) * ld(c.rdu, iu(d, i, j, k)) * ld(c.thu, iu(d, i, j, k));
    const T fx1 = ld(xu, iu(d, i + 1, j, k)) * ld(c.rdu, iu(d, i + 1, j, k)) * ld(c.thu, iu(d, i + 1, j, k));
    const T fy0 = ld(xv, iv(d, i, j, k)) * ld(c.rdv, iv(d, i, j, k)) * ld(c.thv, iv(d, i, j, k));
    const T fy1 = ld(xv, iv(d, i, j + 1, k)) * ld(c.rdv, iv(d, i, j + 1, k)) * ld(c.thv, iv(d, i, j + 1, k));
    const int w0 = iw(d, i, j, k), w1 = iw(d, i, j, k + 1);
    const T fz0 = (k == 0) ? T(0) : ld(xW, w0) * ld(c.rhow, w0) * ld(c.thw, w0);
    const T fz1 = (k + 1 == nz) ? T(0) : ld(xW, w1) * ld(c.rhow, w1) * ld(c.thw, w1);
    const T m = ld(c.mm, h_m(d, i, j));
    const T divh = m * m * ((fx1 - fx0) * idx + (fy1 - fy0) * idy);
    const T tend = -ld(c.cpidz, p) * (xs * (divh + (fz1 - fz0)));
    T L = ld(x.f[3], p) * xs - adt * ps * tend;
    if (b.f[3]) L = ld(b.f[3], p) - L;
    out.f[3][p] = L;
  }
}

// ---------------------------------------------------------------------------
// Column preconditioner.  Intermediate column values are parked in the
// output arrays between the forward and the backward sweep:
//   out.w   <- rhs_w                 (w back-substitution input)
//   out.eta <- rhs_eta / alpha - kin (eta back-substitution input)
//   out.pi  <- Thomas d'             (then overwritten with the solution)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(128) precond_kernel(Dims d, Coef<T> c, CVec5<T> r, Vec5<T> out,
                                                      const int* active) {
  if (active && *active == 0) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i > nx || j > ny) return;
  const T* __restrict__ ru = r.f[0];
  const T* __restrict__ rv = r.f[1];
  // u and v pass straight through (steppers.py:247-249)
  if (j < ny && out.f[0] != ru)
    for (int k = 0; k < nz; ++k) out.f[0][iu(d, i, j, k)] = ld(ru, iu(d, i, j, k));
  if (i < nx && out.f[1] != rv)
    for (int k = 0; k < nz; ++k) out.f[1][iv(d, i, j, k)] = ld(rv, iv(d, i, j, k));
  if (i >= nx || j >= ny) return;

  const T* __restrict__ rw = r.f[2];
  const T* __restrict__ rp = r.f[3];
  const T* __restrict__ rW = r.f[4];
  T* __restrict__ ow = out.f[2];
  T* __restrict__ op = out.f[3];
  T* __restrict__ oW = out.f[4];
  const T a = (T)c.s.alpha;
  const T inva = T(1) / a;
  const T ips = (T)(1.0 / c.s.ps);
  const T ps = (T)c.s.ps;
  const T adtcp = (T)(c.s.alpha * c.s.dt * c.s.cp);
  const T mw = ld(c.mm, h_m(d, i, j));

  // u, v at mass level k averaged in x / y (the u->m and v->m halves)
  auto um = [&](int k) { return T(0.5) * (ld(ru, iu(d, i, j, k)) + ld(ru, iu(d, i + 1, j, k))); };
  auto vm = [&](int k) { return T(0.5) * (ld(rv, iv(d, i, j, k)) + ld(rv, iv(d, i, j + 1, k))); };

  // ---- forward sweep: w levels 0..nz and mass levels 0..nz-1 ----
  T um_prev = um(0), vm_prev = vm(0);
  T wt_lo = T(0);  // w_tilde at level 0 is zero (steppers.py:218)
  T dprev = T(0);
  for (int k = 0; k < nz; ++k) {
    // w level k+1 (interior when k+1 < nz)
    const int pw1 = iw(d, i, j, k + 1);
    T wt_hi = T(0);
    T um_k1 = um_prev, vm_k1 = vm_prev;
    if (k + 1 < nz) {
      um_k1 = um(k + 1);
      vm_k1 = vm(k + 1);
      const T uw = T(0.5) * (um_prev + um_k1);
      const T vw = T(0.5) * (vm_prev + vm_k1);
      const T kin = mw * (uw * ld(c.zxw, pw1) + vw * ld(c.zew, pw1));
      const T rwv = ld(rw, pw1);
      const T rWv = ld(rW, pw1);
      const T damp = ld(c.damp, pw1);
      const T wck = rwv / damp + rWv * inva - kin;
      wt_hi = ld(c.rhow, pw1) * ld(c.thw, pw1) * wck;
      ow[pw1] = rwv;
      oW[pw1] = rWv * inva - kin;
    }
    const int pm = im(d, i, j, k);
    const T rhs = ld(rp, pm) * ips - ld(c.lpi, pm) * (wt_hi - wt_lo);
    const T dk = (k == 0 ? rhs : rhs - ld(c.tlow, pm) * dprev) * ld(c.tinv, pm);
    op[pm] = dk;
    dprev = dk;
    wt_lo = wt_hi;
    um_prev = um_k1;
    vm_prev = vm_k1;
  }
  // ---- back substitution ----
  T x_hi = dprev;  // x at mass level nz-1
  op[im(d, i, j, nz - 1)] = x_hi * ps;
  for (int k = nz - 2; k >= 0; --k) {
    const int pm = im(d, i, j, k);
    const T xk = op[pm] - ld(c.tcp, pm) * x_hi;
    op[pm] = xk * ps;
    // w level k+1 lies between mass levels k and k+1
    const int pw = iw(d, i, j, k + 1);
    const T grad = (x_hi - xk) * ld(c.idzw, pw);
    const T wv = (ow[pw] - adtcp * ld(c.thw, pw) * grad) / ld(c.damp, pw);
    ow[pw] = wv;
    oW[pw] = oW[pw] + wv;
    x_hi = xk;
  }
  // boundary rows (steppers.py:237-238, 244-245)
  const int p0 = iw(d, i, j, 0), pn = iw(d, i, j, nz);
  ow[p0] = ld(rw, p0);
  ow[pn] = ld(rw, pn);
  oW[p0] = ld(rW, p0) * ld(c.dzw, p0);
  oW[pn] = ld(rW, pn) * ld(c.dzw, pn);
}

}  // namespace

template <typename T>
void launch_matvec(const Dims& d, const Coef<T>& c, CVec5<T> x, const double* xscale, CVec5<T> b,
                   Vec5<T> out, const int* active, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  dim3 grd((d.nx + 1 + 31) / 32, (d.ny + 1 + 3) / 4, (d.nz + 1 + 1) / 2);
  matvec_kernel<T><<<grd, blk, 0, st>>>(d, c, x, xscale, b, out, active);
}

template <typename T>
void launch_precond(const Dims& d, const Coef<T>& c, CVec5<T> r, Vec5<T> out, const int* active,
                    cudaStream_t st) {
  dim3 blk(32, 4);
  dim3 grd((d.nx + 1 + 31) / 32, (d.ny + 1 + 3) / 4);
  precond_kernel<T><<<grd, blk, 0, st>>>(d, c, r, out, active);
}

template void launch_matvec<float>(const Dims&, const Coef<float>&, CVec5<float>, const double*, CVec5<float>,
                                   Vec5<float>, const int*, cudaStream_t);
template void launch_matvec<double>(const Dims&, const Coef<double>&, CVec5<double>, const double*,
                                    CVec5<double>, Vec5<double>, const int*, cudaStream_t);
template void launch_precond<float>(const Dims&, const Coef<float>&, CVec5<float>, Vec5<float>, const int*,
                                    cudaStream_t);
template void launch_precond<double>(const Dims&, const Coef<double>&, CVec5<double>, Vec5<double>,
                                     const int*, cudaStream_t);

}  // namespace sisl
