// Coefficient preparation: every derived background/metric array the step
// needs, computed once in float64 from the reference-named inputs and cast to
// the working precision.  Follows euler.py:127-160 (precompute_bg),
// euler.py:254-255 / 320-322 (z_xi_u, z_eta_v, d theta_bg / dz),
// diffusion.py:117,125 (z_xi_m, z_eta_m) and steppers.py:153-185
// (precompute_banded: L_pi and the Thomas factorisation of the column
// Helmholtz system, once per core).
#include "sisl_core.cuh"

#include <math.h>

namespace sisl {

int coef_loc(int id) {
  switch (id) {
    case C_THB: case C_PIB: case C_CPIDZ: case C_DTHM: case C_LPI: case C_ZXM: case C_ZEM: case C_DZM:
    case C_TLO: case C_TCP: case C_TINV:
      return LOC_M;
    case C_THU: case C_ZXU: case C_RDU: return LOC_U;
    case C_THV: case C_ZEV: case C_RDV: return LOC_V;
    case C_THW: case C_RHOW: case C_IDZW: case C_DZW: case C_DAMP: case C_ZXW: case C_ZEW:
    case C_RTW: case C_PBW: case C_IDAMP:
      return LOC_W;
    default: return -1;
  }
}

size_t coef_elems(const Dims& d, int id) {
  int loc = coef_loc(id);
  if (loc >= 0) return field_size(d, loc);
  switch (id) {
    case C_MU: case C_FU: return (size_t)(d.nx + 1) * d.ny;
    case C_MV: case C_FV: return (size_t)d.nx * (d.ny + 1);
    default: return (size_t)d.nx * d.ny;
  }
}

template <typename T>
Coef<T> make_coef(T* const* a, const Scalars& s) {
  Coef<T> c;
  c.thb = a[C_THB]; c.pib = a[C_PIB]; c.cpidz = a[C_CPIDZ]; c.dthm = a[C_DTHM]; c.lpi = a[C_LPI];
  c.zxm = a[C_ZXM]; c.zem = a[C_ZEM]; c.dzm = a[C_DZM];
  c.thu = a[C_THU]; c.zxu = a[C_ZXU]; c.rdu = a[C_RDU];
  c.thv = a[C_THV]; c.zev = a[C_ZEV]; c.rdv = a[C_RDV];
  c.thw = a[C_THW]; c.rhow = a[C_RHOW]; c.idzw = a[C_IDZW]; c.dzw = a[C_DZW]; c.damp = a[C_DAMP];
  c.zxw = a[C_ZXW]; c.zew = a[C_ZEW];
  c.mm = a[C_MM]; c.mu = a[C_MU]; c.mv = a[C_MV]; c.fu = a[C_FU]; c.fv = a[C_FV];
  c.dmdx = a[C_DMDX]; c.dmdy = a[C_DMDY];
  c.tlo = a[C_TLO]; c.tcp = a[C_TCP]; c.tinv = a[C_TINV];
  c.rtw = a[C_RTW]; c.pbw = a[C_PBW]; c.idamp = a[C_IDAMP];
  c.s = s;
  return c;
}

namespace {

__device__ __forceinline__ double rho_of(const Scalars& s, double th, double pi) {
  return s.p0 / (s.Rd * th) * pow(pi, s.cvd / s.Rd);  // steppers.py:770-771
}
// background density at mass point p: the caller's, else the equation of state
__device__ __forceinline__ double rho_at(const Scalars& s, const Base64& b, int p) {
  return b.rho ? b.rho[p] : rho_of(s, b.theta_bg[p], b.pi_bg[p]);
}

// One thread per point of the (nx+1, ny+1, nz+1) union box.
template <typename T>
__global__ void prep_points(Dims d, Scalars s, Base64 b, PtrTable<T> out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i > nx || j > ny || k > nz) return;

  // ---- mass points ----
  if (i < nx && j < ny && k < nz) {
    const int p = im(d, i, j, k);
    const double th = b.theta_bg[p], pi = b.pi_bg[p];
    const double rho = rho_at(s, b, p);
    const double cpi = (s.Rd / s.cvd) * (pi / (rho * th));
    const double dzm = b.dz_m[p];
    out.p[C_THB][p] = (T)th;
    out.p[C_PIB][p] = (T)pi;
    out.p[C_CPIDZ][p] = (T)(cpi / dzm);
    out.p[C_DZM][p] = (T)dzm;
    out.p[C_LPI][p] = (T)(s.alpha * s.dt * cpi / dzm);
    // d theta_bg / dz at the two bounding w levels, averaged to the cell
    double dtw[2];
    for (int q = 0; q < 2; ++q) {
      int kl, kr;
      level_pair(k + q, nz, kl, kr);
      dtw[q] = (b.theta_bg[im(d, i, j, kr)] - b.theta_bg[im(d, i, j, kl)]) / d.dz *
               (d.dz / b.dz_w[iw(d, i, j, k + q)]);
    }
    out.p[C_DTHM][p] = (T)(0.5 * (dtw[0] + dtw[1]));
    // z_xi_m = avg_u->m of z_xi_u; z_eta_m likewise
    double zx[2], ze[2];
    for (int q = 0; q < 2; ++q) {
      int l, r;
      face_pair(i + q, nx, d.px, l, r);
      zx[q] = (b.Z_m[im(d, r, j, k)] - b.Z_m[im(d, l, j, k)]) / d.dx * b.m_u[h_u(d, i + q, j)];
      face_pair(j + q, ny, d.py, l, r);
      ze[q] = (b.Z_m[im(d, i, r, k)] - b.Z_m[im(d, i, l, k)]) / d.dy * b.m_v[h_v(d, i, j + q)];
    }
    out.p[C_ZXM][p] = (T)(0.5 * (zx[0] + zx[1]));
    out.p[C_ZEM][p] = (T)(0.5 * (ze[0] + ze[1]));
  }
  // ---- u faces ----
  if (j < ny && k < nz) {
    int l, r;
    face_pair(i, nx, d.px, l, r);
    const int pl = im(d, l, j, k), pr = im(d, r, j, k);
    const double th = 0.5 * (b.theta_bg[pl] + b.theta_bg[pr]);
    const double rho = 0.5 * (rho_at(s, b, pl) + rho_at(s, b, pr));
    const double dzu = 0.5 * (b.dz_m[pl] + b.dz_m[pr]);
    const double mu = b.m_u[h_u(d, i, j)];
    const int p = iu(d, i, j, k);
    out.p[C_THU][p] = (T)th;
    out.p[C_ZXU][p] = (T)((b.Z_m[pr] - b.Z_m[pl]) / d.dx * mu);
    out.p[C_RDU][p] = (T)(rho * dzu / mu);
  }
  // ---- v faces ----
  if (i < nx && k < nz) {
    int l, r;
    face_pair(j, ny, d.py, l, r);
    const int pl = im(d, i, l, k), pr = im(d, i, r, k);
    const double th = 0.5 * (b.theta_bg[pl] + b.theta_bg[pr]);
    const double rho = 0.5 * (rho_at(s, b, pl) + rho_at(s, b, pr));
    const double dzv = 0.5 * (b.dz_m[pl] + b.dz_m[pr]);
    const double mv = b.m_v[h_v(d, i, j)];
    const int p = iv(d, i, j, k);
    out.p[C_THV][p] = (T)th;
    out.p[C_ZEV][p] = (T)((b.Z_m[pr] - b.Z_m[pl]) / d.dy * mv);
    out.p[C_RDV][p] = (T)(rho * dzv / mv);
  }
  // ---- w levels ----
  if (i < nx && j < ny) {
    int kl, kr;
    level_pair(k, nz, kl, kr);
    const int pl = im(d, i, j, kl), pr = im(d, i, j, kr);
    const int p = iw(d, i, j, k);
    const double th = 0.5 * (b.theta_bg[pl] + b.theta_bg[pr]);
    const double rho = 0.5 * (rho_at(s, b, pl) + rho_at(s, b, pr));
    const double dzw = b.dz_w[p];
    out.p[C_THW][p] = (T)th;
    out.p[C_RHOW][p] = (T)rho;
    out.p[C_IDZW][p] = (T)(1.0 / dzw);
    out.p[C_DZW][p] = (T)dzw;
    out.p[C_DAMP][p] = (T)(1.0 + s.dt * b.tau[p]);
    out.p[C_IDAMP][p] = (T)(1.0 / (1.0 + s.dt * b.tau[p]));
    out.p[C_RTW][p] = (T)(rho * th);
    out.p[C_PBW][p] = (T)(s.alpha * s.dt * s.cp * th / dzw / (1.0 + s.dt * b.tau[p]));
    out.p[C_ZXW][p] = (T)b.z_xi_w[p];
    out.p[C_ZEW][p] = (T)b.z_eta_w[p];
  }
  // ---- 2-D ----
  if (k == 0) {
    if (i < nx && j < ny) {
      const int h = h_m(d, i, j);
      out.p[C_MM][h] = (T)b.m_m[h];
      out.p[C_DMDX][h] = (T)b.dmdx[h];
      out.p[C_DMDY][h] = (T)b.dmdy[h];
    }
    if (j < ny) {
      const int h = h_u(d, i, j);
      out.p[C_MU][h] = (T)b.m_u[h];
      out.p[C_FU][h] = (T)b.f_u[h];
    }
    if (i < nx) {
      const int h = h_v(d, i, j);
      out.p[C_MV][h] = (T)b.m_v[h];
      out.p[C_FV][h] = (T)b.f_v[h];
    }
  }
}

// Column Helmholtz system of VerticalPreconditioner.precompute_banded
// (steppers.py:153-185), one thread per column in float64:
//   P(K) = adt cp th_w / (dz_w (1 + dt tau)) rho_w th_w (0 on ground and lid)
//   L(k) = adt C_pi / dz_m,  lower = -L(k) P(k),  upper = -L(k) P(k+1),
//   main = 1 - lower - upper;  Thomas: pivot(k) = main(k) - lower(k) c'(k-1),
//   c'(k) = upper(k) / pivot(k).
template <typename T>
__global__ void prep_thomas(Dims d, Scalars s, Base64 b, PtrTable<T> out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i >= nx || j >= ny) return;
  auto Pw = [&](int K) -> double {
    if (K <= 0 || K >= nz) return 0.0;
    const int pl = im(d, i, j, K - 1), pr = im(d, i, j, K);
    const double th = 0.5 * (b.theta_bg[pl] + b.theta_bg[pr]);
    const double rho = 0.5 * (rho_at(s, b, pl) + rho_at(s, b, pr));
    const int pw = iw(d, i, j, K);
    return s.alpha * s.dt * s.cp * th / (b.dz_w[pw] * (1.0 + s.dt * b.tau[pw])) * rho * th;
  };
  double cprev = 0.0, Pk = Pw(0);
  for (int k = 0; k < nz; ++k) {
    const int p = im(d, i, j, k);
    const double th = b.theta_bg[p], pi = b.pi_bg[p];
    const double cpi = (s.Rd / s.cvd) * (pi / (rho_at(s, b, p) * th));
    const double L = s.alpha * s.dt * cpi / b.dz_m[p];
    const double Pk1 = Pw(k + 1);
    const double lower = -L * Pk, upper = -L * Pk1;
    const double piv = (1.0 - lower - upper) - lower * cprev;
    cprev = upper / piv;
    out.p[C_TLO][p] = (T)lower;
    out.p[C_TCP][p] = (T)cprev;
    out.p[C_TINV][p] = (T)(1.0 / piv);
    Pk = Pk1;
  }
}

}  // namespace

template <typename T>
void launch_prepare(const Dims& d, const Scalars& s, const Base64& b, PtrTable<T> out, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  dim3 grd((d.nx + 1 + blk.x - 1) / blk.x, (d.ny + 1 + blk.y - 1) / blk.y, (d.nz + 1 + blk.z - 1) / blk.z);
  prep_points<T><<<grd, blk, 0, st>>>(d, s, b, out);
  prep_thomas<T><<<dim3((d.nx + 127) / 128, d.ny), 128, 0, st>>>(d, s, b, out);
}

template Coef<float> make_coef<float>(float* const*, const Scalars&);
template Coef<double> make_coef<double>(double* const*, const Scalars&);
template void launch_prepare<float>(const Dims&, const Scalars&, const Base64&, PtrTable<float>, cudaStream_t);
template void launch_prepare<double>(const Dims&, const Scalars&, const Base64&, PtrTable<double>, cudaStream_t);

}  // namespace sisl
