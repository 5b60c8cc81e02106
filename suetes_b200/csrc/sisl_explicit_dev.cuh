// Point stencils shared by the explicit kernels and their adjoints
// (sisl_explicit.cu, sisl_step_vjp.cu): pressure gradients, winds at mass
// points and map curvature, face averages, the Exner flux divergence and the
// Cartesian horizontal Laplacian of the hyperdiffusion.
#pragma once

#include "sisl_core.cuh"

namespace sisl {
namespace dev {

// pressure-gradient pieces of a mass field q (physical pi' or a guess)
template <typename T>
struct Grad {
  const Dims& d;
  const Coef<T>& c;
  const T* __restrict__ q;
  __device__ __forceinline__ T Q(int i, int j, int k) const { return ld(q, im(d, i, j, k)); }
  __device__ __forceinline__ T gzw(int i, int j, int k) const {  // d q/dz at w level k (euler.py:252)
    int kl, kr;
    level_pair(k, d.nz, kl, kr);
    return (Q(i, j, kr) - Q(i, j, kl)) * ld(c.idzw, iw(d, i, j, k));
  }
  __device__ __forceinline__ T gzm(int i, int j, int k) const { return T(0.5) * (gzw(i, j, k) + gzw(i, j, k + 1)); }
  // Cartesian x-gradient at u face i: m_u dq/dxi - z_xi_u avg(dq/dz)  (euler.py:250-261)
  __device__ __forceinline__ T gx(int i, int j, int k) const {
    int l, r;
    face_pair(i, d.nx, d.px, l, r);
    const T g = (Q(r, j, k) - Q(l, j, k)) * (T)(1.0 / d.dx) * ld(c.mu, h_u(d, i, j));
    return g - ld(c.zxu, iu(d, i, j, k)) * T(0.5) * (gzm(l, j, k) + gzm(r, j, k));
  }
  __device__ __forceinline__ T gy(int i, int j, int k) const {
    int l, r;
    face_pair(j, d.ny, d.py, l, r);
    const T g = (Q(i, r, k) - Q(i, l, k)) * (T)(1.0 / d.dy) * ld(c.mv, h_v(d, i, j));
    return g - ld(c.zev, iv(d, i, j, k)) * T(0.5) * (gzm(i, l, k) + gzm(i, r, k));
  }
};

// horizontal winds at mass points and the map-curvature factor (euler.py:188-206)
template <typename T>
struct Winds {
  const Dims& d;
  const Coef<T>& c;
  const T* __restrict__ u;
  const T* __restrict__ v;
  __device__ __forceinline__ T um(int i, int j, int k) const {
    return T(0.5) * (ld(u, iu(d, i, j, k)) + ld(u, iu(d, i + 1, j, k)));
  }
  __device__ __forceinline__ T vm(int i, int j, int k) const {
    return T(0.5) * (ld(v, iv(d, i, j, k)) + ld(v, iv(d, i, j + 1, k)));
  }
  __device__ __forceinline__ T metric_m(int i, int j, int k) const {
    return vm(i, j, k) * ld(c.dmdx, h_m(d, i, j)) - um(i, j, k) * ld(c.dmdy, h_m(d, i, j));
  }
  // w-level averages of u, v (avg_u->m then avg_m->w, edge padded)
  __device__ __forceinline__ T uw(int i, int j, int k) const {
    int kl, kr;
    level_pair(k, d.nz, kl, kr);
    return T(0.5) * (um(i, j, kl) + um(i, j, kr));
  }
  __device__ __forceinline__ T vw(int i, int j, int k) const {
    int kl, kr;
    level_pair(k, d.nz, kl, kr);
    return T(0.5) * (vm(i, j, kl) + vm(i, j, kr));
  }
};

// averages of a mass field to the faces
template <typename T>
__device__ __forceinline__ T avg_mu(const Dims& d, const T* __restrict__ f, int i, int j, int k) {
  int l, r;
  face_pair(i, d.nx, d.px, l, r);
  return T(0.5) * (ld(f, im(d, l, j, k)) + ld(f, im(d, r, j, k)));
}
template <typename T>
__device__ __forceinline__ T avg_mv(const Dims& d, const T* __restrict__ f, int i, int j, int k) {
  int l, r;
  face_pair(j, d.ny, d.py, l, r);
  return T(0.5) * (ld(f, im(d, i, l, k)) + ld(f, im(d, i, r, k)));
}
template <typename T>
__device__ __forceinline__ T avg_mw(const Dims& d, const T* __restrict__ f, int i, int j, int k) {
  int kl, kr;
  level_pair(k, d.nz, kl, kr);
  return T(0.5) * (ld(f, im(d, i, j, kl)) + ld(f, im(d, i, j, kr)));
}

// -C_pi/dz_m (m^2 (dFx/dx + dFy/dy) + dFz) for fluxes
//   Fx = ux rdu thx, Fy = vy rdv thy, Fz = eta dz_w rho_w thz (zero on lid/ground)
// where the face thetas come from `thsel` (euler.py:298-318, 172-186).
template <typename T, typename ThU, typename ThV, typename ThW>
__device__ __forceinline__ T divergence(const Dims& d, const Coef<T>& c, const T* __restrict__ u,
                                        const T* __restrict__ v, const T* __restrict__ eta, int i, int j, int k,
                                        ThU thu, ThV thv, ThW thw) {
  const int u0 = iu(d, i, j, k), u1 = iu(d, i + 1, j, k);
  const int v0 = iv(d, i, j, k), v1 = iv(d, i, j + 1, k);
  const T fx0 = ld(u, u0) * ld(c.rdu, u0) * thu(i, j, k);
  const T fx1 = ld(u, u1) * ld(c.rdu, u1) * thu(i + 1, j, k);
  const T fy0 = ld(v, v0) * ld(c.rdv, v0) * thv(i, j, k);
  const T fy1 = ld(v, v1) * ld(c.rdv, v1) * thv(i, j + 1, k);
  const int w0 = iw(d, i, j, k), w1 = iw(d, i, j, k + 1);
  const T fz0 = (k == 0) ? T(0) : ld(eta, w0) * ld(c.dzw, w0) * ld(c.rhow, w0) * thw(i, j, k);
  const T fz1 = (k + 1 == d.nz) ? T(0) : ld(eta, w1) * ld(c.dzw, w1) * ld(c.rhow, w1) * thw(i, j, k + 1);
  const T m = ld(c.mm, h_m(d, i, j));
  const T divh = m * m * ((fx1 - fx0) * (T)(1.0 / d.dx) + (fy1 - fy0) * (T)(1.0 / d.dy));
  return -ld(c.cpidz, im(d, i, j, k)) * (divh + (fz1 - fz0));
}

// Terrain-following face gradients of a mass field, the first pass of the
// Cartesian horizontal Laplacian (diffusion.py:93-129).
template <typename T>
struct HLap {
  const Dims& d;
  const Coef<T>& c;
  const T* __restrict__ f;
  __device__ __forceinline__ T F(int i, int j, int k) const { return ld(f, im(d, i, j, k)); }
  __device__ __forceinline__ T dzw(int i, int j, int k) const {
    int kl, kr;
    level_pair(k, d.nz, kl, kr);
    return (F(i, j, kr) - F(i, j, kl)) * ld(c.idzw, iw(d, i, j, k));
  }
  __device__ __forceinline__ T dzm(int i, int j, int k) const { return T(0.5) * (dzw(i, j, k) + dzw(i, j, k + 1)); }
  __device__ __forceinline__ T Gx(int fi, int j, int k) const {  // at u face fi
    int l, r;
    face_pair(fi, d.nx, d.px, l, r);
    const T dxi = (F(r, j, k) - F(l, j, k)) * (T)(1.0 / d.dx) * ld(c.mu, h_u(d, fi, j));
    return dxi - ld(c.zxu, iu(d, fi, j, k)) * T(0.5) * (dzm(l, j, k) + dzm(r, j, k));
  }
  __device__ __forceinline__ T Gy(int i, int fj, int k) const {  // at v face fj
    int l, r;
    face_pair(fj, d.ny, d.py, l, r);
    const T deta = (F(i, r, k) - F(i, l, k)) * (T)(1.0 / d.dy) * ld(c.mv, h_v(d, i, fj));
    return deta - ld(c.zev, iv(d, i, fj, k)) * T(0.5) * (dzm(i, l, k) + dzm(i, r, k));
  }
};

}  // namespace dev
}  // namespace sisl
