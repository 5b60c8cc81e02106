// Explicit part of the SISL step: old-time tendencies with hyperdiffusion,
// the departure-side right-hand sides, the predictor-corrector right-hand
// sides, divergence damping, lateral relaxation and the equation of state.
//
// * Euler3D.get_tendencies(is_explicit=True)   euler.py:208-372
// * Euler3D.nonlinear_pi_tendency               euler.py:162-186
// * Euler3D.metric_curvature_tendencies         euler.py:188-206
// * HyperFilter (horizontal part, nu_v = 0)     diffusion.py:93-173
// * RHS assembly                                steppers.py:801-842
// * predictor-corrector right-hand sides        steppers.py:911-983
// * divergence damping, EOS                     steppers.py:1022-1031, 1055-1056
//
// Thermodynamic fields are carried in perturbation form: pi' = pi - pi_bg and
// th' = th_v - theta_bg, so float32 never subtracts two O(1) numbers.
#include "sisl_explicit.cuh"
#include "sisl_explicit_dev.cuh"

namespace sisl {
namespace {

using namespace dev;

dim3 box_grid(int ex, int ey, int ez, dim3 blk) {
  return dim3((ex + blk.x - 1) / blk.x, (ey + blk.y - 1) / blk.y, (ez + blk.z - 1) / blk.z);
}

// ---------------------------------------------------------------------------
// hyperdiffusion: mass-point copies of u, v, w, th' (diffusion.py:141-151)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void hyper_src_kernel(Dims d, const T* __restrict__ u, const T* __restrict__ v,
                                 const T* __restrict__ w, const T* __restrict__ th, PtrTable<T> out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= d.nx || j >= d.ny || k >= d.nz) return;
  const int p = im(d, i, j, k);
  out.p[0][p] = T(0.5) * (ld(u, iu(d, i, j, k)) + ld(u, iu(d, i + 1, j, k)));
  out.p[1][p] = T(0.5) * (ld(v, iv(d, i, j, k)) + ld(v, iv(d, i, j + 1, k)));
  out.p[2][p] = T(0.5) * (ld(w, iw(d, i, j, k)) + ld(w, iw(d, i, j, k + 1)));
  out.p[3][p] = ld(th, p);
}

// The Cartesian horizontal Laplacian (diffusion.py:93-129) in two passes:
// the terrain-following gradients at every u face and v face once
// (hyper_grad_kernel, HLap::Gx/Gy), then the divergence of the stored
// gradients (hyper_div_kernel), instead of re-forming twelve face
// gradients per point (the one-pass form this replaced computed the same
// values in registers; the fields agree bitwise).
template <typename T>
__global__ void hyper_grad_kernel(Dims d, Coef<T> c, PtrTable<T> src, PtrTable<T> gxy) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int kz = blockIdx.z * blockDim.z + threadIdx.z;
  const int f = kz / d.nz, k = kz % d.nz;
  if (i > d.nx || j > d.ny || f >= 4) return;
  HLap<T> L{d, c, src.p[f]};
  if (j < d.ny) gxy.p[f][iu(d, i, j, k)] = L.Gx(i, j, k);
  if (i < d.nx) gxy.p[4 + f][iv(d, i, j, k)] = L.Gy(i, j, k);
}

template <typename T>
__global__ void hyper_div_kernel(Dims d, Coef<T> c, PtrTable<T> gxy, PtrTable<T> dst, T scale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int kz = blockIdx.z * blockDim.z + threadIdx.z;
  const int f = kz / d.nz, k = kz % d.nz;
  if (i >= d.nx || j >= d.ny || f >= 4) return;
  const int nz = d.nz;
  const T* __restrict__ gx = gxy.p[f];
  const T* __restrict__ gy = gxy.p[4 + f];
  const int kl = max(k - 1, 0), kh = min(k + 1, nz - 1);
  const int lv[3] = {kl, k, kh};
  T gxm[3], gym[3], gx0 = T(0), gx1 = T(0), gy0 = T(0), gy1 = T(0);
#pragma unroll
  for (int q = 0; q < 3; ++q) {
    const T a0 = ld(gx, iu(d, i, j, lv[q])), a1 = ld(gx, iu(d, i + 1, j, lv[q]));
    const T b0 = ld(gy, iv(d, i, j, lv[q])), b1 = ld(gy, iv(d, i, j + 1, lv[q]));
    gxm[q] = T(0.5) * (a0 + a1);
    gym[q] = T(0.5) * (b0 + b1);
    if (q == 1) { gx0 = a0; gx1 = a1; gy0 = b0; gy1 = b1; }
  }
  auto lvl = [&](int kk) { return kk == kl ? 0 : (kk == k ? 1 : 2); };
  int al, ar, bl, br;
  level_pair(k, nz, al, ar);
  level_pair(k + 1, nz, bl, br);
  const T iz0 = ld(c.idzw, iw(d, i, j, k)), iz1 = ld(c.idzw, iw(d, i, j, k + 1));
  const T ex0 = (gxm[lvl(ar)] - gxm[lvl(al)]) * iz0, ex1 = (gxm[lvl(br)] - gxm[lvl(bl)]) * iz1;
  const T ey0 = (gym[lvl(ar)] - gym[lvl(al)]) * iz0, ey1 = (gym[lvl(br)] - gym[lvl(bl)]) * iz1;
  const T m = ld(c.mm, h_m(d, i, j));
  const int p = im(d, i, j, k);
  const T divx = m * (gx1 - gx0) * (T)(1.0 / d.dx) - ld(c.zxm, p) * T(0.5) * (ex0 + ex1);
  const T divy = m * (gy1 - gy0) * (T)(1.0 / d.dy) - ld(c.zem, p) * T(0.5) * (ey0 + ey1);
  dst.p[f][p] = scale * (divx + divy);
}

// ---------------------------------------------------------------------------
// explicit tendencies.  mode 0: step inputs (u_in, v_in, w_in, pi_in, th_in,
// tend_th, residual_n); mode 1: raw tendencies for the operator API.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) explicit_kernel(Dims d, Coef<T> c, ExplicitIn<T> in, ExplicitOut<T> out,
                                                       int mode) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i > nx || j > ny || k > nz) return;
  const T dt = (T)c.s.dt, a = (T)c.s.alpha, cp = (T)c.s.cp, g = (T)c.s.g;
  const T oma = T(1) - a;
  Grad<T> G{d, c, in.pi};
  Winds<T> W{d, c, in.u, in.v};
  const T* __restrict__ th = in.th;
  const bool hyp = in.hyper[0] != nullptr && mode != 2;
  const T lin = (mode == 2) ? T(0) : T(1);  // mode 2: linear tendencies (euler.py:240-247, 281-282)

  if (j < ny && k < nz) {  // u faces
    int l, r;
    face_pair(i, nx, d.px, l, r);
    const int p = iu(d, i, j, k);
    const T thp = lin * T(0.5) * (ld(th, im(d, l, j, k)) + ld(th, im(d, r, j, k)));
    const T vat = T(0.5) * (W.vm(l, j, k) + W.vm(r, j, k));
    const T met = lin * T(0.5) * (W.metric_m(l, j, k) + W.metric_m(r, j, k)) * vat;
    T pd = hyp ? T(0.5) * (ld(in.hyper[0], im(d, l, j, k)) + ld(in.hyper[0], im(d, r, j, k))) : T(0);
    if (mode != 2 && in.extra[0]) pd += ld(in.extra[0], p);  // physics tendencies join phys_diff (euler.py:347-366)
    const T tend = -cp * (ld(c.thu, p) + thp) * G.gx(i, j, k) + ld(c.fu, h_u(d, i, j)) * vat + met + pd;
    if (mode == 0) {
      out.f[0][p] = ld(in.u, p) + dt * (oma * tend + a * pd);
    } else {
      out.f[0][p] = tend;
      if (out.pd[0]) out.pd[0][p] = pd;
    }
  }
  if (i < nx && k < nz) {  // v faces
    int l, r;
    face_pair(j, ny, d.py, l, r);
    const int p = iv(d, i, j, k);
    const T thp = lin * T(0.5) * (ld(th, im(d, i, l, k)) + ld(th, im(d, i, r, k)));
    const T uat = T(0.5) * (W.um(i, l, k) + W.um(i, r, k));
    const T met = -lin * T(0.5) * (W.metric_m(i, l, k) + W.metric_m(i, r, k)) * uat;
    T pd = hyp ? T(0.5) * (ld(in.hyper[1], im(d, i, l, k)) + ld(in.hyper[1], im(d, i, r, k))) : T(0);
    if (mode != 2 && in.extra[1]) pd += ld(in.extra[1], p);
    const T tend = -cp * (ld(c.thv, p) + thp) * G.gy(i, j, k) - ld(c.fv, h_v(d, i, j)) * uat + met + pd;
    if (mode == 0) {
      out.f[1][p] = ld(in.v, p) + dt * (oma * tend + a * pd);
    } else {
      out.f[1][p] = tend;
      if (out.pd[1]) out.pd[1][p] = pd;
    }
  }
  if (i < nx && j < ny) {  // w levels
    int kl, kr;
    level_pair(k, nz, kl, kr);
    const int p = iw(d, i, j, k);
    const T thp = lin * T(0.5) * (ld(th, im(d, i, j, kl)) + ld(th, im(d, i, j, kr)));
    const T thw = ld(c.thw, p);
    T pd = hyp ? T(0.5) * (ld(in.hyper[2], im(d, i, j, kl)) + ld(in.hyper[2], im(d, i, j, kr))) : T(0);
    if (mode != 2 && in.extra[2]) pd += ld(in.extra[2], p);
    const T tend = -cp * (thw + thp) * G.gzw(i, j, k) + g * (thp / thw) + pd;
    if (mode == 0) {
      out.f[2][p] = ld(in.w, p) + dt * (oma * tend + a * pd);
      // residual_n = dz_w eta + u_w z_xi_w + v_w z_eta_w - w  (steppers.py:837-842)
      out.f[6][p] = ld(c.dzw, p) * ld(in.eta, p) + W.uw(i, j, k) * ld(c.zxw, p) + W.vw(i, j, k) * ld(c.zew, p) -
                    ld(in.w, p);
    } else {
      out.f[2][p] = tend;
      if (out.pd[2]) out.pd[2][p] = pd;
    }
  }
  if (i < nx && j < ny && k < nz) {  // mass points
    const int p = im(d, i, j, k);
    auto thu_lin = [&](int a_, int b_, int c_) { return ld(c.thu, iu(d, a_, b_, c_)); };
    auto thv_lin = [&](int a_, int b_, int c_) { return ld(c.thv, iv(d, a_, b_, c_)); };
    auto thw_lin = [&](int a_, int b_, int c_) { return ld(c.thw, iw(d, a_, b_, c_)); };
    auto thu_nl = [&](int a_, int b_, int c_) { return avg_mu(d, th, a_, b_, c_); };
    auto thv_nl = [&](int a_, int b_, int c_) { return avg_mv(d, th, a_, b_, c_); };
    auto thw_nl = [&](int a_, int b_, int c_) { return avg_mw(d, th, a_, b_, c_); };
    const T tpi = divergence(d, c, in.u, in.v, in.eta, i, j, k, thu_lin, thv_lin, thw_lin);
    const T nlpi = (mode == 2) ? T(0) : divergence(d, c, in.u, in.v, in.eta, i, j, k, thu_nl, thv_nl, thw_nl);
    const T wm = T(0.5) * (ld(in.w, iw(d, i, j, k)) + ld(in.w, iw(d, i, j, k + 1)));
    T pd = hyp ? ld(in.hyper[3], p) : T(0);
    if (mode != 2 && in.extra[3]) pd += ld(in.extra[3], p);
    const T tth = -wm * ld(c.dthm, p) + pd;
    if (mode == 0) {
      out.f[3][p] = ld(in.pi, p) + oma * dt * (tpi + nlpi);
      out.f[4][p] = ld(th, p) + oma * dt * tth;
      out.f[5][p] = tth;
    } else {
      out.f[3][p] = tpi;
      out.f[4][p] = tth;
      out.f[5][p] = nlpi;
      if (out.pd[3]) out.pd[3][p] = pd;
    }
  }
}

// ---------------------------------------------------------------------------
// predictor-corrector (steppers.py:911-983)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void corrector_theta_kernel(Dims d, Coef<T> c, const T* __restrict__ th_adv, const T* __restrict__ tth,
                                       const T* __restrict__ w_now, const T* __restrict__ w_next, T* th_next) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= d.nx || j >= d.ny || k >= d.nz) return;
  const int p = im(d, i, j, k);
  const T wm = T(0.5) * (ld(w_now, iw(d, i, j, k)) + ld(w_now, iw(d, i, j, k + 1)));
  const T wmn = T(0.5) * (ld(w_next, iw(d, i, j, k)) + ld(w_next, iw(d, i, j, k + 1)));
  const T adt = (T)(c.s.alpha * c.s.dt);
  th_next[p] = ld(th_adv, p) + adt * (ld(tth, p) + (wm - wmn) * ld(c.dthm, p));
}

template <typename T>
__global__ void __launch_bounds__(256) corrector_rhs_kernel(Dims d, Coef<T> c, CorrectorIn<T> in, Vec5<T> out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i > nx || j > ny || k > nz) return;
  const T adt = (T)(c.s.alpha * c.s.dt);
  const T cad = (T)(c.s.cp * c.s.alpha * c.s.dt);
  const T g = (T)c.s.g;
  Grad<T> G{d, c, in.pg};
  Winds<T> WG{d, c, in.ug, in.vg};
  const T* __restrict__ th = in.th_next;
  if (j < ny && k < nz) {
    int l, r;
    face_pair(i, nx, d.px, l, r);
    const int p = iu(d, i, j, k);
    const T thp = T(0.5) * (ld(th, im(d, l, j, k)) + ld(th, im(d, r, j, k)));
    const T vat = T(0.5) * (WG.vm(l, j, k) + WG.vm(r, j, k));
    const T met = T(0.5) * (WG.metric_m(l, j, k) + WG.metric_m(r, j, k)) * vat;
    out.f[0][p] = ld(in.rhs_u, p) - cad * thp * G.gx(i, j, k) + adt * met;
  }
  if (i < nx && k < nz) {
    int l, r;
    face_pair(j, ny, d.py, l, r);
    const int p = iv(d, i, j, k);
    const T thp = T(0.5) * (ld(th, im(d, i, l, k)) + ld(th, im(d, i, r, k)));
    const T uat = T(0.5) * (WG.um(i, l, k) + WG.um(i, r, k));
    const T met = -T(0.5) * (WG.metric_m(i, l, k) + WG.metric_m(i, r, k)) * uat;
    out.f[1][p] = ld(in.rhs_v, p) - cad * thp * G.gy(i, j, k) + adt * met;
  }
  if (i < nx && j < ny) {
    const int p = iw(d, i, j, k);
    T val;
    if (k == 0) {  // kinematic bottom boundary from the latest solver guess (steppers.py:974-983)
      val = ld(c.mm, h_m(d, i, j)) * (WG.uw(i, j, 0) * ld(c.zxw, p) + WG.vw(i, j, 0) * ld(c.zew, p));
    } else if (k == nz) {
      val = T(0);
    } else {
      const T thp = T(0.5) * (ld(th, im(d, i, j, k - 1)) + ld(th, im(d, i, j, k)));
      val = ld(in.rhs_w, p) + adt * (g * (thp / ld(c.thw, p))) - cad * thp * G.gzw(i, j, k);
    }
    out.f[2][p] = val;
  }
  if (i < nx && j < ny && k < nz) {
    const int p = im(d, i, j, k);
    auto thu_nl = [&](int a_, int b_, int c_) { return avg_mu(d, th, a_, b_, c_); };
    auto thv_nl = [&](int a_, int b_, int c_) { return avg_mv(d, th, a_, b_, c_); };
    auto thw_nl = [&](int a_, int b_, int c_) { return avg_mw(d, th, a_, b_, c_); };
    const T nl = divergence(d, c, in.gu, in.gv, in.geta, i, j, k, thu_nl, thv_nl, thw_nl);
    out.f[3][p] = ld(in.rhs_pi, p) + adt * nl;
  }
}

// ---------------------------------------------------------------------------
// finalisation: divergence damping (steppers.py:1022-1031), relaxation
// blend (the bc_fn of the mountain-wave runs, schaer_mountain_3d/run.py:104-126),
// EOS (steppers.py:1055-1056)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void hdiv_kernel(Dims d, Coef<T> c, const T* __restrict__ u, const T* __restrict__ v, T* div) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= d.nx || j >= d.ny || k >= d.nz) return;
  const T m = ld(c.mm, h_m(d, i, j));
  const T dux = (ld(u, iu(d, i + 1, j, k)) - ld(u, iu(d, i, j, k))) * (T)(1.0 / d.dx) * m;
  const T dvy = (ld(v, iv(d, i, j + 1, k)) - ld(v, iv(d, i, j, k))) * (T)(1.0 / d.dy) * m;
  div[im(d, i, j, k)] = dux + dvy;
}

template <typename T>
__device__ __forceinline__ T blend(T val, const T* mask, int h, T ext) {
  if (!mask) return val;
  const T m = ld(mask, h);
  return (T(1) - m) * val + m * ext;
}

template <typename T>
__global__ void __launch_bounds__(256) finalize_kernel(Dims d, Coef<T> c, FinalizeArgs<T> fa) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i > nx || j > ny || k > nz) return;
  const T nud = (T)(c.s.nu_div * c.s.dt);
  const Relax<T>& R = fa.relax;
  if (j < ny && k < nz) {
    const int p = iu(d, i, j, k);
    T val = ld(fa.u_in, p);
    if (fa.div) {
      int l, r;
      face_pair(i, nx, d.px, l, r);
      val += nud * (ld(fa.div, im(d, r, j, k)) - ld(fa.div, im(d, l, j, k))) * (T)(1.0 / d.dx) *
             ld(c.mu, h_u(d, i, j));
    }
    if (R.on & RELAX_U) val = blend(val, R.mask_u, h_u(d, i, j), R.ext_field[0] ? ld(R.ext_field[0], p) : R.ext[0]);
    fa.u_out[p] = val;
  }
  if (i < nx && k < nz) {
    const int p = iv(d, i, j, k);
    T val = ld(fa.v_in, p);
    if (fa.div) {
      int l, r;
      face_pair(j, ny, d.py, l, r);
      val += nud * (ld(fa.div, im(d, i, r, k)) - ld(fa.div, im(d, i, l, k))) * (T)(1.0 / d.dy) *
             ld(c.mv, h_v(d, i, j));
    }
    if (R.on & RELAX_V) val = blend(val, R.mask_v, h_v(d, i, j), R.ext_field[1] ? ld(R.ext_field[1], p) : R.ext[1]);
    fa.v_out[p] = val;
  }
  if (i < nx && j < ny) {
    const int p = iw(d, i, j, k);
    if (R.on & RELAX_W)
      fa.w_io[p] = blend(fa.w_io[p], R.mask_m, h_m(d, i, j), R.ext_field[2] ? ld(R.ext_field[2], p) : R.ext[2]);
  }
  if (i < nx && j < ny && k < nz) {
    const int p = im(d, i, j, k);
    T th = fa.th_io[p], pi = fa.pi_io[p];
    if (R.on & RELAX_TH) th = blend(th, R.mask_m, h_m(d, i, j), R.ext_field[3] ? ld(R.ext_field[3], p) : R.ext[3]);
    if (R.on & RELAX_PI) pi = blend(pi, R.mask_m, h_m(d, i, j), R.ext_field[4] ? ld(R.ext_field[4], p) : R.ext[4]);
    fa.th_io[p] = th;
    fa.pi_io[p] = pi;
    if (fa.rho_out) {
      const T thf = th + ld(c.thb, p), pif = pi + ld(c.pib, p);
      fa.rho_out[p] = (T)c.s.p0 / ((T)c.s.Rd * thf) * pow(pif, (T)(c.s.cvd / c.s.Rd));
    }
  }
}

}  // namespace

template <typename T>
void launch_hyper(const Dims& d, const Coef<T>& c, const T* u, const T* v, const T* w, const T* th,
                  PtrTable<T> tmp4, PtrTable<T> out4, PtrTable<T> gxy8, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  hyper_src_kernel<T><<<box_grid(d.nx, d.ny, d.nz, blk), blk, 0, st>>>(d, u, v, w, th, out4);
  const dim3 gg = box_grid(d.nx + 1, d.ny + 1, 4 * d.nz, blk), gd = box_grid(d.nx, d.ny, 4 * d.nz, blk);
  hyper_grad_kernel<T><<<gg, blk, 0, st>>>(d, c, out4, gxy8);
  hyper_div_kernel<T><<<gd, blk, 0, st>>>(d, c, gxy8, tmp4, T(1));
  hyper_grad_kernel<T><<<gg, blk, 0, st>>>(d, c, tmp4, gxy8);
  hyper_div_kernel<T><<<gd, blk, 0, st>>>(d, c, gxy8, out4, (T)(-c.s.nu_h));
}

template <typename T>
void launch_explicit(const Dims& d, const Coef<T>& c, const ExplicitIn<T>& in, const ExplicitOut<T>& out, int mode,
                     cudaStream_t st) {
  dim3 blk(32, 4, 2);
  explicit_kernel<T><<<box_grid(d.nx + 1, d.ny + 1, d.nz + 1, blk), blk, 0, st>>>(d, c, in, out, mode);
}

template <typename T>
void launch_corrector_theta(const Dims& d, const Coef<T>& c, const T* th_adv, const T* tth, const T* w_now,
                            const T* w_next, T* th_next, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  corrector_theta_kernel<T><<<box_grid(d.nx, d.ny, d.nz, blk), blk, 0, st>>>(d, c, th_adv, tth, w_now, w_next,
                                                                            th_next);
}

template <typename T>
void launch_corrector_rhs(const Dims& d, const Coef<T>& c, const CorrectorIn<T>& in, Vec5<T> out, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  corrector_rhs_kernel<T><<<box_grid(d.nx + 1, d.ny + 1, d.nz + 1, blk), blk, 0, st>>>(d, c, in, out);
}

template <typename T>
void launch_hdiv(const Dims& d, const Coef<T>& c, const T* u, const T* v, T* div, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  hdiv_kernel<T><<<box_grid(d.nx, d.ny, d.nz, blk), blk, 0, st>>>(d, c, u, v, div);
}

// Euler3D.metric_curvature_tendencies (euler.py:188-206): the map-curvature
// accelerations metric_u v_at_u at the u faces and -metric_v u_at_v at the
// v faces, metric = v_m dm/dx - u_m dm/dy at mass points averaged to the
// faces (edge padded) -- the term the explicit kernel adds to its u and v
// tendencies, on its own.  One thread per (i, j, k) of the union box.
template <typename T>
__global__ void curvature_kernel(Dims d, Coef<T> c, const T* __restrict__ u, const T* __restrict__ v,
                                 T* __restrict__ ou, T* __restrict__ ov) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const int nx = d.nx, ny = d.ny;
  if (i > nx || j > ny || k >= d.nz) return;
  const Winds<T> W{d, c, u, v};
  if (j < ny) {
    int l, r;
    face_pair(i, nx, d.px, l, r);
    const T vat = T(0.5) * (W.vm(l, j, k) + W.vm(r, j, k));
    ou[iu(d, i, j, k)] = T(0.5) * (W.metric_m(l, j, k) + W.metric_m(r, j, k)) * vat;
  }
  if (i < nx) {
    int l, r;
    face_pair(j, ny, d.py, l, r);
    const T uat = T(0.5) * (W.um(i, l, k) + W.um(i, r, k));
    ov[iv(d, i, j, k)] = -(T(0.5) * (W.metric_m(i, l, k) + W.metric_m(i, r, k))) * uat;
  }
}

template <typename T>
void launch_curvature(const Dims& d, const Coef<T>& c, const T* u, const T* v, T* ou, T* ov, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  curvature_kernel<T><<<box_grid(d.nx + 1, d.ny + 1, d.nz, blk), blk, 0, st>>>(d, c, u, v, ou, ov);
}

template <typename T>
void launch_finalize(const Dims& d, const Coef<T>& c, const FinalizeArgs<T>& fa, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  finalize_kernel<T><<<box_grid(d.nx + 1, d.ny + 1, d.nz + 1, blk), blk, 0, st>>>(d, c, fa);
}

#define SISL_INST_EX(T)                                                                                        \
  template void launch_hyper<T>(const Dims&, const Coef<T>&, const T*, const T*, const T*, const T*,           \
                                PtrTable<T>, PtrTable<T>, PtrTable<T>, cudaStream_t);                          \
  template void launch_explicit<T>(const Dims&, const Coef<T>&, const ExplicitIn<T>&, const ExplicitOut<T>&,   \
                                   int, cudaStream_t);                                                         \
  template void launch_corrector_theta<T>(const Dims&, const Coef<T>&, const T*, const T*, const T*, const T*, \
                                          T*, cudaStream_t);                                                   \
  template void launch_corrector_rhs<T>(const Dims&, const Coef<T>&, const CorrectorIn<T>&, Vec5<T>,         \
                                        cudaStream_t);                                                         \
  template void launch_hdiv<T>(const Dims&, const Coef<T>&, const T*, const T*, T*, cudaStream_t);             \
  template void launch_finalize<T>(const Dims&, const Coef<T>&, const FinalizeArgs<T>&, cudaStream_t);       \
  template void launch_curvature<T>(const Dims&, const Coef<T>&, const T*, const T*, T*, T*, cudaStream_t);
SISL_INST_EX(float)
SISL_INST_EX(double)

}  // namespace sisl
