// Helmholtz matvec and column (Thomas) preconditioner on the scaled solver
// vector (u, v, w, pi * pi_scale, eta_dot * dz_w_full).
//
// Matvec: Euler3D.linear_operator (euler.py:374-439) with the linear
// tendencies of get_tendencies(is_explicit=False) (euler.py:208-318),
// wrapped in the scaling of SemiImplicitSolver3D.solve.A_fn
// (steppers.py:439-461).  One fused pass: every output of the five fields at
// a point of the (nx+1, ny+1, nz+1) union box is produced by one thread.
// Mass and w points share the plane layout, so im(i, j, k) == iw(i, j, k).
//
// Preconditioner: VerticalPreconditioner.__call__ (steppers.py:187-253) on
// tiles of 32 columns: kinematic forcing and Helmholtz RHS, the Thomas
// recurrences with the factorisation prepared once per core, then the w and
// eta_dot back-substitution.
#include "sisl_group.cuh"

namespace sisl {
namespace {

// ---------------------------------------------------------------------------
// Matvec, one thread per point of the (nx+1, ny+1, nz+1) union box.  The
// vertical pressure gradient averaged to mass level k is formed once per
// needed column -- own (i, j), X = (i-1, j), Y = (i, j-1), wrapped on
// periodic axes -- from three pi' loads and two 1/dz_w loads with
// branch-free edge padding (euler.py:252, 257).  The own column is the
// right-hand column of u face i and v face j; on a periodic axis the face-0
// thread also writes the duplicate face n (euler.py:412, 417).
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T gz_mass(const T* __restrict__ p, const T* __restrict__ iz, int base, int k, int nz,
                                     int plane, T sp) {
  const int kl = k > 0 ? k - 1 : 0, kh = k + 1 < nz ? k + 1 : nz - 1;
  const T Pl = mul_rn(ld(p, base + kl * plane), sp), P0 = mul_rn(ld(p, base + k * plane), sp),
          Ph = mul_rn(ld(p, base + kh * plane), sp);
  const T g0 = mul_rn(k == 0 ? Ph - P0 : P0 - Pl, ld(iz, base + k * plane));
  const T g1 = mul_rn(k + 1 == nz ? P0 - Pl : Ph - P0, ld(iz, base + (k + 1) * plane));
  return mul_rn(T(0.5), g0 + g1);
}

// Every value the five rows of one union-box point read.  Values that one
// thread forms and carries or shares (scaled pressures, vertical gradients,
// vertical fluxes) are rounded on their own before they get here, so the
// rows give the same bits whichever kernel shape gathered the inputs.
template <typename T>
struct MvIn {
  T PO, PX, PY, gmO, gmX, gmY;                  // scaled pi' at mass level km, d/dz at km (own, i-1, j-1)
  T xu_f, thu, zxu, mu_f, fu_f;                 // u face (i, j, km)
  T xv_f, thv, zev, mv_f, fv_f;                 // v face (i, j, km)
  T vX0, vX1, vO0, vO1, uY0, uY1, uO0, uO1;     // neighbouring faces at km
  T xw_k, xW_k, idzw_k, damp, thw, zxw, zew, gzw;  // w level k (interior rows at the clamped level)
  T uwa, uwb, uwc, uwd, vwa, vwb, vwc, vwd, mw;  // winds at the levels around w level k
  T rdu0, rdu1, thu0, thu1, rdv0, rdv1, thv0, thv1;  // flux factors of the own cell's faces at km
  T fz0, fz1, cpidz, xp_k;                      // vertical fluxes (rounded), C_pi/dz_m, own pi' at km
};

// The five rows of one point (euler.py:374-439 through steppers.py:439-461),
// L = (Lu, Lv, Lw, Le, Lp): the expressions of matvec_point, term for term.
template <typename T>
__device__ __forceinline__ void mv_rows(const Dims& d, const Coef<T>& c, const MvIn<T>& q, T xs, bool u_lock,
                                        bool v_lock, bool wb, T (&L)[5]) {
  const T adt = (T)(c.s.alpha * c.s.dt), cp = (T)c.s.cp, a = (T)c.s.alpha, ps = (T)c.s.ps;
  const T idx = (T)(1.0 / d.dx), idy = (T)(1.0 / d.dy);
  const T vat = T(0.25) * (q.vX0 + q.vX1 + q.vO0 + q.vO1) * xs;
  const T tend_u = -cp * q.thu * ((q.PO - q.PX) * idx * q.mu_f - q.zxu * T(0.5) * (q.gmX + q.gmO)) + q.fu_f * vat;
  L[0] = u_lock ? q.xu_f * xs : q.xu_f * xs - adt * tend_u;
  const T uat = T(0.25) * (q.uY0 + q.uY1 + q.uO0 + q.uO1) * xs;
  const T tend_v = -cp * q.thv * ((q.PO - q.PY) * idy * q.mv_f - q.zev * T(0.5) * (q.gmY + q.gmO)) - q.fv_f * uat;
  L[1] = v_lock ? q.xv_f * xs : q.xv_f * xs - adt * tend_v;
  L[2] = wb ? q.xw_k * xs : q.damp * q.xw_k * xs + adt * cp * q.thw * q.gzw;
  const T uw = T(0.25) * (q.uwa + q.uwb + q.uwc + q.uwd) * xs, vw = T(0.25) * (q.vwa + q.vwb + q.vwc + q.vwd) * xs;
  L[3] = wb ? q.xW_k * xs * q.idzw_k : a * (q.xW_k * xs + q.mw * (uw * q.zxw + vw * q.zew) - q.xw_k * xs);
  const T fx0 = q.uO0 * q.rdu0 * q.thu0, fx1 = q.uO1 * q.rdu1 * q.thu1;
  const T fy0 = q.vO0 * q.rdv0 * q.thv0, fy1 = q.vO1 * q.rdv1 * q.thv1;
  const T divh = q.mw * q.mw * ((fx1 - fx0) * idx + (fy1 - fy0) * idy);
  L[4] = q.xp_k * xs + adt * ps * q.cpidz * (xs * (divh + (q.fz1 - q.fz0)));
}

// Stores of one point's rows (residual mode out = b - L when b is given);
// on a periodic axis the face-0 thread also writes the duplicate face n
// (euler.py:412, 417).
template <typename T>
__device__ __forceinline__ void mv_store(const Dims& d, const CVec5<T>& b, const Vec5<T>& out, int i, int j, int k,
                                         const T (&L)[5]) {
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  const bool do_u = (k < nz) && (j < ny) && !(d.px && i == nx);
  const bool do_v = (k < nz) && (i < nx) && !(d.py && j == ny);
  const bool own = (i < nx && j < ny);
  if (do_u) {
    const int p = iu(d, i, j, k);
    out.f[0][p] = b.f[0] ? ld(b.f[0], p) - L[0] : L[0];
    if (d.px && i == 0) {
      const int pn = iu(d, nx, j, k);
      out.f[0][pn] = b.f[0] ? ld(b.f[0], pn) - L[0] : L[0];
    }
  }
  if (do_v) {
    const int p = iv(d, i, j, k);
    out.f[1][p] = b.f[1] ? ld(b.f[1], p) - L[1] : L[1];
    if (d.py && j == 0) {
      const int pn = iv(d, i, ny, k);
      out.f[1][pn] = b.f[1] ? ld(b.f[1], pn) - L[1] : L[1];
    }
  }
  if (own) {
    const int pw = i + nx * (j + ny * k);
    out.f[2][pw] = b.f[2] ? ld(b.f[2], pw) - L[2] : L[2];
    out.f[4][pw] = b.f[4] ? ld(b.f[4], pw) - L[3] : L[3];
    if (k < nz) out.f[3][pw] = b.f[3] ? ld(b.f[3], pw) - L[4] : L[4];
  }
}

// Branch-free load phase: every index is clamped into its array, all values
// are loaded unconditionally (one memory round trip per thread), the five
// rows are formed with selects, and only the stores are predicated.
// All rows of one point of the union box (the matvec_kernel body).
template <typename T>
__device__ __forceinline__ void matvec_point(const Dims& d, const Coef<T>& c, const CVec5<T>& x, const T xs,
                                             const CVec5<T>& b, const Vec5<T>& out, int i, int j, int k) {
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  const T adt = (T)(c.s.alpha * c.s.dt), cp = (T)c.s.cp, a = (T)c.s.alpha, ps = (T)c.s.ps;
  const T sp = xs / ps;
  const T idx = (T)(1.0 / d.dx), idy = (T)(1.0 / d.dy);
  const int pm = nx * ny, pu = (nx + 1) * ny, pv = nx * (ny + 1);
  const T* __restrict__ xu = x.f[0];
  const T* __restrict__ xv = x.f[1];
  const T* __restrict__ xw = x.f[2];
  const T* __restrict__ xp = x.f[3];
  const T* __restrict__ xW = x.f[4];
  // clamped coordinates: mass columns ic < nx, jc < ny; mass levels km < nz
  const int ic = min(i, nx - 1), jc = min(j, ny - 1), km = min(k, nz - 1);
  const int il = (ic == 0) ? nx - 1 : ic - 1;   // left column of face i (wraps when periodic)
  const int jl = (jc == 0) ? ny - 1 : jc - 1;
  const int hO = ic + nx * jc, hX = il + nx * jc, hY = ic + nx * jl;
  const int iuc = min(i, nx);  // u face index (valid for u arrays)
  const int jvc = min(j, ny);
  // ---- loads (unconditional, in bounds) ----
  const T gmO = gz_mass(xp, c.idzw, hO, km, nz, pm, sp);
  const T gmX = gz_mass(xp, c.idzw, hX, km, nz, pm, sp);
  const T gmY = gz_mass(xp, c.idzw, hY, km, nz, pm, sp);
  const T PO = mul_rn(ld(xp, hO + km * pm), sp), PX = mul_rn(ld(xp, hX + km * pm), sp),
          PY = mul_rn(ld(xp, hY + km * pm), sp);
  const int pU = iuc + (nx + 1) * (jc + ny * km);        // u face (i, jc, km)
  const int pV = ic + nx * (jvc + (ny + 1) * km);        // v face (ic, j, km)
  const int uO = ic + (nx + 1) * (jc + ny * km);         // u face (ic, jc, km): own cell west face
  const int uY = ic + (nx + 1) * (jl + ny * km);
  const int vO = ic + nx * (jc + (ny + 1) * km);         // v face (ic, jc, km): own cell south face
  const int vX = il + nx * (jc + (ny + 1) * km);
  const T xu_f = ld(xu, pU), xv_f = ld(xv, pV);
  const T thu = ld(c.thu, pU), zxu = ld(c.zxu, pU), thv = ld(c.thv, pV), zev = ld(c.zev, pV);
  const T mu_f = ld(c.mu, iuc + (nx + 1) * jc), fu_f = ld(c.fu, iuc + (nx + 1) * jc);
  const T mv_f = ld(c.mv, ic + nx * jvc), fv_f = ld(c.fv, ic + nx * jvc);
  const T vX0 = ld(xv, vX), vX1 = ld(xv, vX + nx), vO0 = ld(xv, vO), vO1 = ld(xv, vO + nx);
  const T uY0 = ld(xu, uY), uY1 = ld(xu, uY + 1), uO0 = ld(xu, uO), uO1 = ld(xu, uO + 1);
  // w level k (clamped into the interior rows for the stencil loads)
  const int kw = min(max(k, 1), nz - 1);
  const int pw = hO + k * pm, pwi = hO + kw * pm;
  const T xw_k = ld(xw, pw), xW_k = ld(xW, pw), idzw_k = ld(c.idzw, pw);
  const T damp = ld(c.damp, pwi), thw = ld(c.thw, pwi), zxw = ld(c.zxw, pwi), zew = ld(c.zew, pwi);
  const T Pw1 = mul_rn(ld(xp, hO + kw * pm), sp), Pw0 = mul_rn(ld(xp, hO + (kw - 1) * pm), sp);
  const int uw1 = ic + (nx + 1) * (jc + ny * kw), uw0 = uw1 - pu;
  const int vw1 = ic + nx * (jc + (ny + 1) * kw), vw0 = vw1 - pv;
  const T uwa = ld(xu, uw0), uwb = ld(xu, uw0 + 1), uwc = ld(xu, uw1), uwd = ld(xu, uw1 + 1);
  const T vwa = ld(xv, vw0), vwb = ld(xv, vw0 + nx), vwc = ld(xv, vw1), vwd = ld(xv, vw1 + nx);
  const T mw = ld(c.mm, hO);
  // pi row at mass level km
  const int pmk = hO + km * pm;
  const T rdu0 = ld(c.rdu, uO), rdu1 = ld(c.rdu, uO + 1), thu0 = ld(c.thu, uO), thu1 = ld(c.thu, uO + 1);
  const T rdv0 = ld(c.rdv, vO), rdv1 = ld(c.rdv, vO + nx), thv0 = ld(c.thv, vO), thv1 = ld(c.thv, vO + nx);
  const int pz0 = hO + km * pm, pz1 = hO + min(km + 1, nz - 1) * pm;
  const T W0 = ld(xW, pz0), rw0 = ld(c.rhow, pz0), tw0 = ld(c.thw, pz0);
  const T W1 = ld(xW, pz1), rw1 = ld(c.rhow, pz1), tw1 = ld(c.thw, pz1);
  const T cpidz = ld(c.cpidz, pmk), xp_k = ld(xp, pmk);
  // ---- rows ----
  // u face (i, j, k): locked on an open boundary (euler.py:414-415)
  const bool u_lock = !d.px && (i == 0 || i == nx);
  const T vat = T(0.25) * (vX0 + vX1 + vO0 + vO1) * xs;
  const T tend_u = -cp * thu * ((PO - PX) * idx * mu_f - zxu * T(0.5) * (gmX + gmO)) + fu_f * vat;
  const T Lu = u_lock ? xu_f * xs : xu_f * xs - adt * tend_u;
  const bool v_lock = !d.py && (j == 0 || j == ny);
  const T uat = T(0.25) * (uY0 + uY1 + uO0 + uO1) * xs;
  const T tend_v = -cp * thv * ((PO - PY) * idy * mv_f - zev * T(0.5) * (gmY + gmO)) - fv_f * uat;
  const T Lv = v_lock ? xv_f * xs : xv_f * xs - adt * tend_v;
  // w and eta_dot rows at w level k; identity rows on the ground and lid (euler.py:426-437)
  const bool wb = (k == 0 || k == nz);
  const T gzw = mul_rn(Pw1 - Pw0, idzw_k);
  const T Lw = wb ? xw_k * xs : damp * xw_k * xs + adt * cp * thw * gzw;
  const T uw = T(0.25) * (uwa + uwb + uwc + uwd) * xs, vw = T(0.25) * (vwa + vwb + vwc + vwd) * xs;
  const T Le = wb ? xW_k * xs * idzw_k : a * (xW_k * xs + mw * (uw * zxw + vw * zew) - xw_k * xs);
  // pi row (euler.py:298-318 through linear_operator)
  const T fx0 = uO0 * rdu0 * thu0, fx1 = uO1 * rdu1 * thu1;
  const T fy0 = vO0 * rdv0 * thv0, fy1 = vO1 * rdv1 * thv1;
  const T fz0 = (km == 0) ? T(0) : mul_rn(mul_rn(W0, rw0), tw0);
  const T fz1 = (km + 1 == nz) ? T(0) : mul_rn(mul_rn(W1, rw1), tw1);
  const T divh = mw * mw * ((fx1 - fx0) * idx + (fy1 - fy0) * idy);
  const T Lp = xp_k * xs + adt * ps * cpidz * (xs * (divh + (fz1 - fz0)));
  // ---- stores ----
  const bool do_u = (k < nz) && (j < ny) && !(d.px && i == nx);
  const bool do_v = (k < nz) && (i < nx) && !(d.py && j == ny);
  const bool own = (i < nx && j < ny);
  if (do_u) {
    const int p = iu(d, i, j, k);
    out.f[0][p] = b.f[0] ? ld(b.f[0], p) - Lu : Lu;
    if (d.px && i == 0) {  // duplicate periodic face (euler.py:412)
      const int pn = iu(d, nx, j, k);
      out.f[0][pn] = b.f[0] ? ld(b.f[0], pn) - Lu : Lu;
    }
  }
  if (do_v) {
    const int p = iv(d, i, j, k);
    out.f[1][p] = b.f[1] ? ld(b.f[1], p) - Lv : Lv;
    if (d.py && j == 0) {
      const int pn = iv(d, i, ny, k);
      out.f[1][pn] = b.f[1] ? ld(b.f[1], pn) - Lv : Lv;
    }
  }
  if (own) {
    out.f[2][pw] = b.f[2] ? ld(b.f[2], pw) - Lw : Lw;
    out.f[4][pw] = b.f[4] ? ld(b.f[4], pw) - Le : Le;
    if (k < nz) out.f[3][pw] = b.f[3] ? ld(b.f[3], pw) - Lp : Lp;
  }
}

// One thread per point, or LV consecutive levels of a column per thread (the
// loads the levels share -- pressure at k+-1, the w-level winds, 1/dz_w --
// are then common subexpressions; the scaled pressures and the vertical
// gradients and fluxes two levels share are rounded on their own, so every
// shape gives bitwise the same rows).  float: 6 resident blocks of 256
// (<= 40 registers, no spills) for one level per thread, 4 for several
// (a 3-block budget for four levels measured slower); double 4 and 3.
template <typename T, int LV>
__global__ void __launch_bounds__(256, sizeof(T) == 4 ? (LV == 1 ? 6 : 4) : (LV == 1 ? 4 : 3)) matvec_kernel(Dims d, Coef<T> c, CVec5<T> x,
                                                                            const double* xscale,
                                                     CVec5<T> b, Vec5<T> out, const int* active) {
  if (active && *active == 0) return;
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k0 = (blockIdx.z * blockDim.z + threadIdx.z) * LV;
  if (i > d.nx || j > d.ny) return;
  const T xs = xscale ? (T)(*xscale) : T(1);
#pragma unroll
  for (int l = 0; l < LV; ++l)
    if (k0 + l <= d.nz) matvec_point(d, c, x, xs, b, out, i, j, k0 + l);
}

// cp.async helpers (global -> shared, asynchronous, per thread)
__device__ __forceinline__ void cp_async4(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 4;" ::"r"(s), "l"(gmem) : "memory");
}
__device__ __forceinline__ void cp_async8(void* smem, const void* gmem) {
  const unsigned s = (unsigned)__cvta_generic_to_shared(smem);
  asm volatile("cp.async.ca.shared.global [%0], [%1], 8;" ::"r"(s), "l"(gmem) : "memory");
}
template <typename T>
__device__ __forceinline__ void cp_async_t(T* smem, const T* gmem) {
  if (sizeof(T) == 4) cp_async4(smem, gmem);
  else cp_async8(smem, gmem);
}
__device__ __forceinline__ void cp_async_commit() { asm volatile("cp.async.commit_group;" ::: "memory"); }
template <int N>
__device__ __forceinline__ void cp_async_wait() { asm volatile("cp.async.wait_group %0;" ::"n"(N) : "memory"); }

// ---------------------------------------------------------------------------
// Column march: one thread per (i, j) column of the union box marching up
// the levels of its z chunk (blockIdx.z of gridDim.z chunks).  Vertical
// neighbours are carried in registers instead of reloaded: the scaled
// pressures, the vertical gradients G(k) = (P(k) - P(k-1)) / dz_w(k) of the
// own, i-1 and j-1 columns (the mass-level gradient is their average), the
// vertical flux and the winds one level down.  The loads a level needs
// first (pressures, 1/dz_w, the flux terms) are issued two levels ahead and
// the rest one level ahead, so each thread keeps ~50 loads in flight.  The
// rows are mv_rows on the same rounded inputs as matvec_point: bitwise the
// other shapes.  Needs nz >= 2.
// ---------------------------------------------------------------------------
template <typename T>
struct MvA {  // first-needed loads of level k: pi' (mass level min(k, nz-1)) and
  T pO, pX, pY, izO, izX, izY, W, rw, tw;  // 1/dz_w of the three columns, eta_dot rho_w th_w (w level k)
};
template <typename T>
struct MvB {  // the rest of level k (faces at mass level min(k, nz-1), w-level terms at k)
  T uO0, uO1, uY0, uY1, vO0, vO1, vX0, vX1, zxu, zev, rdu0, rdu1, thu0, thu1, rdv0, rdv1, thv0, thv1;
  T xw, damp, zxw, zew, cpidz;
};

// block (bx, by, bz) of a (., ., gz) grid of 32 x 4 threads
template <typename T>
__device__ __forceinline__ void matvec_march_block(const Dims& d, const Coef<T>& c, const CVec5<T>& x,
                                                   const double* xscale, const CVec5<T>& b, const Vec5<T>& out,
                                                   int bx, int by, int bz, int gz) {
  const int i = bx * blockDim.x + threadIdx.x;
  const int j = by * blockDim.y + threadIdx.y;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i > nx || j > ny) return;
  const int kA = (int)((long)bz * (nz + 1) / gz);
  const int kB = (int)((long)(bz + 1) * (nz + 1) / gz);
  if (kA >= kB) return;
  const T xs = xscale ? (T)(*xscale) : T(1);
  const T sp = xs / (T)c.s.ps;
  const int pm = nx * ny, pu = (nx + 1) * ny, pv = nx * (ny + 1);
  const T* __restrict__ xu = x.f[0];
  const T* __restrict__ xv = x.f[1];
  const T* __restrict__ xw = x.f[2];
  const T* __restrict__ xp = x.f[3];
  const T* __restrict__ xW = x.f[4];
  const int ic = min(i, nx - 1), jc = min(j, ny - 1);
  const int il = (ic == 0) ? nx - 1 : ic - 1;
  const int jl = (jc == 0) ? ny - 1 : jc - 1;
  const int hO = ic + nx * jc, hX = il + nx * jc, hY = ic + nx * jl;
  const int iuc = min(i, nx), jvc = min(j, ny);
  const int uO = ic + (nx + 1) * jc, uY = ic + (nx + 1) * jl, pU = iuc + (nx + 1) * jc;
  const int vO = ic + nx * jc, vX = il + nx * jc, pV = ic + nx * jvc;
  auto lev_a = [&](int k) {
    MvA<T> a;
    const int km = min(k, nz - 1);
    a.pO = ld(xp, hO + km * pm);
    a.pX = ld(xp, hX + km * pm);
    a.pY = ld(xp, hY + km * pm);
    a.izO = ld(c.idzw, hO + k * pm);
    a.izX = ld(c.idzw, hX + k * pm);
    a.izY = ld(c.idzw, hY + k * pm);
    a.W = ld(xW, hO + k * pm);
    a.rw = ld(c.rhow, hO + k * pm);
    a.tw = ld(c.thw, hO + k * pm);
    return a;
  };
  auto lev_b = [&](int k) {
    MvB<T> e;
    const int km = min(k, nz - 1);
    const int ou = km * pu, ov = km * pv;
    e.uO0 = ld(xu, uO + ou);
    e.uO1 = ld(xu, uO + ou + 1);
    e.uY0 = ld(xu, uY + ou);
    e.uY1 = ld(xu, uY + ou + 1);
    e.vO0 = ld(xv, vO + ov);
    e.vO1 = ld(xv, vO + ov + nx);
    e.vX0 = ld(xv, vX + ov);
    e.vX1 = ld(xv, vX + ov + nx);
    e.zxu = ld(c.zxu, pU + ou);
    e.zev = ld(c.zev, pV + ov);
    e.rdu0 = ld(c.rdu, uO + ou);
    e.rdu1 = ld(c.rdu, uO + ou + 1);
    e.thu0 = ld(c.thu, uO + ou);
    e.thu1 = ld(c.thu, uO + ou + 1);
    e.rdv0 = ld(c.rdv, vO + ov);
    e.rdv1 = ld(c.rdv, vO + ov + nx);
    e.thv0 = ld(c.thv, vO + ov);
    e.thv1 = ld(c.thv, vO + ov + nx);
    e.xw = ld(xw, hO + k * pm);
    e.damp = ld(c.damp, hO + k * pm);
    e.zxw = ld(c.zxw, hO + k * pm);
    e.zew = ld(c.zew, hO + k * pm);
    e.cpidz = ld(c.cpidz, hO + km * pm);
    return e;
  };
  const T mu_f = ld(c.mu, iuc + (nx + 1) * jc), fu_f = ld(c.fu, iuc + (nx + 1) * jc);
  const T mv_f = ld(c.mv, ic + nx * jvc), fv_f = ld(c.fv, ic + nx * jvc);
  const T mw = ld(c.mm, hO);
  const bool u_lock = !d.px && (i == 0 || i == nx), v_lock = !d.py && (j == 0 || j == ny);
  const bool ui = i < nx, vj = j < ny;
  // carried state at level kA
  MvA<T> a0 = lev_a(kA), a1 = lev_a(min(kA + 1, nz));
  MvB<T> b0 = lev_b(kA);
  T P0O = mul_rn(a0.pO, sp), P0X = mul_rn(a0.pX, sp), P0Y = mul_rn(a0.pY, sp);
  T PmO = P0O, PmX = P0X, PmY = P0Y;  // scaled pi' one level down
  T GO, GX, GY, fz0;
  T uw_a, uw_b, vw_a, vw_b;  // own-cell faces one level down
  if (kA == 0) {
    GO = mul_rn(mul_rn(a1.pO, sp) - P0O, a0.izO);
    GX = mul_rn(mul_rn(a1.pX, sp) - P0X, a0.izX);
    GY = mul_rn(mul_rn(a1.pY, sp) - P0Y, a0.izY);
    fz0 = T(0);
    uw_a = b0.uO0, uw_b = b0.uO1, vw_a = b0.vO0, vw_b = b0.vO1;
  } else {
    const MvA<T> am = lev_a(kA - 1);
    const MvB<T> bm = lev_b(kA - 1);
    PmO = mul_rn(am.pO, sp), PmX = mul_rn(am.pX, sp), PmY = mul_rn(am.pY, sp);
    GO = mul_rn(P0O - PmO, a0.izO);
    GX = mul_rn(P0X - PmX, a0.izX);
    GY = mul_rn(P0Y - PmY, a0.izY);
    fz0 = mul_rn(mul_rn(a0.W, a0.rw), a0.tw);
    uw_a = bm.uO0, uw_b = bm.uO1, vw_a = bm.vO0, vw_b = bm.vO1;
  }
  for (int k = kA; k < kB; ++k) {
    const MvA<T> a2 = lev_a(min(k + 2, nz));  // prefetch
    const MvB<T> b1 = lev_b(min(k + 1, nz));
    // next level's scaled pressures and gradients (the lid gradient repeats
    // the top pair of mass levels, as the edge padding of gz_mass)
    const T P1O = mul_rn(a1.pO, sp), P1X = mul_rn(a1.pX, sp), P1Y = mul_rn(a1.pY, sp);
    const bool top = (k + 1 >= nz);
    const T G1O = mul_rn(top ? P0O - PmO : P1O - P0O, a1.izO);
    const T G1X = mul_rn(top ? P0X - PmX : P1X - P0X, a1.izX);
    const T G1Y = mul_rn(top ? P0Y - PmY : P1Y - P0Y, a1.izY);
    const T fz1 = top ? T(0) : mul_rn(mul_rn(a1.W, a1.rw), a1.tw);
    MvIn<T> q;
    q.PO = P0O;
    q.PX = P0X;
    q.PY = P0Y;
    q.gmO = mul_rn(T(0.5), GO + G1O);
    q.gmX = mul_rn(T(0.5), GX + G1X);
    q.gmY = mul_rn(T(0.5), GY + G1Y);
    q.xu_f = ui ? b0.uO0 : b0.uO1;
    q.thu = ui ? b0.thu0 : b0.thu1;
    q.zxu = b0.zxu;
    q.mu_f = mu_f;
    q.fu_f = fu_f;
    q.xv_f = vj ? b0.vO0 : b0.vO1;
    q.thv = vj ? b0.thv0 : b0.thv1;
    q.zev = b0.zev;
    q.mv_f = mv_f;
    q.fv_f = fv_f;
    q.vX0 = b0.vX0;
    q.vX1 = b0.vX1;
    q.vO0 = b0.vO0;
    q.vO1 = b0.vO1;
    q.uY0 = b0.uY0;
    q.uY1 = b0.uY1;
    q.uO0 = b0.uO0;
    q.uO1 = b0.uO1;
    q.xw_k = b0.xw;
    q.xW_k = a0.W;
    q.idzw_k = a0.izO;
    q.damp = b0.damp;
    q.thw = a0.tw;
    q.zxw = b0.zxw;
    q.zew = b0.zew;
    q.gzw = GO;
    q.uwa = uw_a;
    q.uwb = uw_b;
    q.uwc = b0.uO0;
    q.uwd = b0.uO1;
    q.vwa = vw_a;
    q.vwb = vw_b;
    q.vwc = b0.vO0;
    q.vwd = b0.vO1;
    q.mw = mw;
    q.rdu0 = b0.rdu0;
    q.rdu1 = b0.rdu1;
    q.thu0 = b0.thu0;
    q.thu1 = b0.thu1;
    q.rdv0 = b0.rdv0;
    q.rdv1 = b0.rdv1;
    q.thv0 = b0.thv0;
    q.thv1 = b0.thv1;
    q.fz0 = fz0;
    q.fz1 = fz1;
    q.cpidz = b0.cpidz;
    q.xp_k = a0.pO;
    T L[5];
    mv_rows(d, c, q, xs, u_lock, v_lock, k == 0 || k == nz, L);
    mv_store(d, b, out, i, j, k, L);
    // one level up
    uw_a = b0.uO0, uw_b = b0.uO1, vw_a = b0.vO0, vw_b = b0.vO1;
    PmO = P0O, PmX = P0X, PmY = P0Y;
    P0O = P1O, P0X = P1X, P0Y = P1Y;
    GO = G1O, GX = G1X, GY = G1Y;
    fz0 = fz1;
    a0 = a1;
    a1 = a2;
    b0 = b1;
  }
}
template <typename T>
__global__ void __launch_bounds__(128, sizeof(T) == 4 ? 4 : 2) matvec_march_kernel(Dims d, Coef<T> c, CVec5<T> x,
                                                                                  const double* xscale, CVec5<T> b,
                                                                                  Vec5<T> out, const int* active) {
  if (active && *active == 0) return;
  matvec_march_block<T>(d, c, x, xscale, b, out, blockIdx.x, blockIdx.y, blockIdx.z, gridDim.z);
}

// ---------------------------------------------------------------------------
// Column-tile preconditioner: a block owns 32 consecutive columns (same j).
//   A1: every thread takes (w level k, column) pairs and forms w_tilde
//       (steppers.py:215-219), the acoustic coupling P = K_w rho_w th_w
//       (steppers.py:171-177) and the eta_dot/alpha - kin term (parked in
//       the eta_dot output), each once;
//   A2: the Helmholtz RHS (steppers.py:223) and L_pi (steppers.py:180) at
//       every mass level from the shared w_tilde;
//   B: one thread per column solves its tridiagonal system
//      (lower = -L_pi P_k, upper = -L_pi P_k+1, main = 1 - lower - upper;
//      steppers.py:183-185, 227) with the Thomas factorisation prepared once
//      per core (prep_thomas), in shared memory;
//   C: every thread writes w, eta_dot and pi (steppers.py:231-251).
// The banded system is strictly diagonally dominant, so no pivoting.
// Shared memory per block: (5 nz + 1) * columns values of T.
// ---------------------------------------------------------------------------

template <typename T>
struct PrecondW {  // w-level quantities of one column at one level
  T wt, ep;
};

// w_tilde and the eta_dot/alpha - kin term at w level k (zero on the ground
// and the lid: the loads use a clamped interior level and the results are
// masked).  The arithmetic is term for term the one of precond_march_kernel,
// so every column variant gives bitwise the same result.
template <typename T>
__device__ __forceinline__ PrecondW<T> precond_wlevel(const Dims& d, const Coef<T>& c, const T* __restrict__ ru,
                                                     const T* __restrict__ rv, const T* __restrict__ rw,
                                                     const T* __restrict__ rW, int i, int j, int k, T inva) {
  const int nx = d.nx, ny = d.ny;
  const int kc = min(max(k, 1), d.nz - 1);
  const T on = (k > 0 && k < d.nz) ? T(1) : T(0);
  const int p = i + nx * j + kc * nx * ny;
  const int u1 = iu(d, i, j, kc), u0 = u1 - (nx + 1) * ny;
  const int v1 = iv(d, i, j, kc), v0 = v1 - nx * (ny + 1);
  const T su_lo = ld(ru, u0) + ld(ru, u0 + 1), su_hi = ld(ru, u1) + ld(ru, u1 + 1);
  const T sv_lo = ld(rv, v0) + ld(rv, v0 + nx), sv_hi = ld(rv, v1) + ld(rv, v1 + nx);
  const T mq = T(0.25) * ld(c.mm, i + nx * j);
  const T kin = mq * ((su_lo + su_hi) * ld(c.zxw, p) + (sv_lo + sv_hi) * ld(c.zew, p));
  const T ep = ld(rW, p) * inva - kin;
  PrecondW<T> o;
  o.ep = on * ep;
  o.wt = on * (ld(c.rtw, p) * (ld(rw, p) * ld(c.idamp, p) + ep));
  return o;
}

template <typename T, int PT, int PC>
__global__ void __launch_bounds__(PT) precond_tile_kernel(Dims d, Coef<T> c, CVec5<T> r, Vec5<T> out,
                                                          const int* active) {
  if (active && *active == 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sm = reinterpret_cast<T*>(smem_raw);
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  T* s_x = sm;                    // [nz][PC]    rhs -> d' -> x
  T* s_W = s_x + nz * PC;         // [nz+1][PC]  w_tilde at w levels
  T* s_lo = s_W + (nz + 1) * PC;  // [nz][PC]    lower
  T* s_iv = s_lo + nz * PC;       // [nz][PC]    1 / pivot
  T* s_cp = s_iv + nz * PC;       // [nz][PC]    c'
  const int i0 = blockIdx.x * PC;
  const int j = blockIdx.y;
  const int tid = threadIdx.x;
  const T* __restrict__ ru = r.f[0];
  const T* __restrict__ rv = r.f[1];
  const T* __restrict__ rw = r.f[2];
  const T* __restrict__ rp = r.f[3];
  const T* __restrict__ rW = r.f[4];
  T* __restrict__ ow = out.f[2];
  T* __restrict__ op = out.f[3];
  T* __restrict__ oW = out.f[4];
  const T inva = T(1) / (T)c.s.alpha;
  const T ips = (T)(1.0 / c.s.ps);
  const T ps = (T)c.s.ps;
  const int pm = nx * ny;

  // u and v pass straight through (steppers.py:247-249) unless aliased
  if (out.f[0] != ru) {
    const int ncol = min(PC + (i0 + PC >= nx ? 1 : 0), nx + 1 - i0);
    for (int q = tid; q < ncol * nz; q += PT) {
      const int k = q / ncol, ii = i0 + q % ncol;
      out.f[0][iu(d, ii, j, k)] = ld(ru, iu(d, ii, j, k));
    }
  }
  if (out.f[1] != rv) {
    const int ncol = min(PC, nx - i0);
    const int nj = (j == ny - 1) ? 2 : 1;  // the last block row also copies face ny
    for (int q = tid; q < ncol * nz * nj; q += PT) {
      const int jj = j + q / (ncol * nz), rem = q % (ncol * nz);
      const int k = rem / ncol, ii = i0 + rem % ncol;
      out.f[1][iv(d, ii, jj, k)] = ld(rv, iv(d, ii, jj, k));
    }
  }

  // ---- A1: the w-level quantities once per (level, column) ----
#pragma unroll 2
  for (int q = tid; q < (nz + 1) * PC; q += PT) {
    const int k = q / PC, l = q % PC, i = min(i0 + l, nx - 1);
    const PrecondW<T> w = precond_wlevel(d, c, ru, rv, rw, rW, i, j, k, inva);
    s_W[q] = w.wt;
    if (i0 + l < nx && k > 0 && k < nz) oW[i + nx * j + k * pm] = w.ep;  // eta_dot / alpha - kin, completed in C
  }
  __syncthreads();
  // ---- A2: Helmholtz right-hand side (steppers.py:223) and the factorisation ----
  for (int q = tid; q < nz * PC; q += PT) {
    const int k = q / PC, l = q % PC, i = min(i0 + l, nx - 1);
    const int p = i + nx * j + k * pm;
    s_x[q] = ld(rp, p) * ips - ld(c.lpi, p) * (s_W[q + PC] - s_W[q]);
    s_lo[q] = ld(c.tlo, p);
    s_iv[q] = ld(c.tinv, p);
    s_cp[q] = ld(c.tcp, p);
  }
  __syncthreads();
  // ---- B: Thomas with the prepared factorisation, one thread per column ----
  if (tid < PC) {
    const int l = tid;
    T dprev = T(0);
    for (int k = 0; k < nz; ++k) {
      const int q = k * PC + l;
      dprev = (s_x[q] - s_lo[q] * dprev) * s_iv[q];
      s_x[q] = dprev;
    }
    T xh = dprev;
    for (int k = nz - 2; k >= 0; --k) {
      const int q = k * PC + l;
      xh = s_x[q] - s_cp[q] * xh;
      s_x[q] = xh;
    }
  }
  __syncthreads();
  // ---- C: back substitution for w, eta_dot and the scaled pi ----
#pragma unroll 2
  for (int q = tid; q < (nz + 1) * PC; q += PT) {
    const int k = q / PC, l = q % PC, i = i0 + l;
    if (i >= nx) continue;
    const int p = i + nx * j + k * pm;
    if (k == 0 || k == nz) {  // boundary rows (steppers.py:237-238, 244-245)
      ow[p] = ld(rw, p);
      oW[p] = ld(rW, p) * ld(c.dzw, p);
    } else {
      const T wv = ld(rw, p) * ld(c.idamp, p) - ld(c.pbw, p) * (s_x[q] - s_x[q - PC]);
      ow[p] = wv;
      oW[p] = oW[p] + wv;
    }
    if (k < nz) op[p] = s_x[q] * ps;
  }
}

// The same tile with its global loads batched: every thread issues PU
// items' loads before it computes any of them, so each phase waits on one
// or two rounds of memory latency instead of one per item.  The horizontal
// wind sums over faces (i, i+1) and (j, j+1) are staged per mass level
// first (A0, into the buffers the factorisation fills later), so the
// w-level phase reads six arrays instead of fifteen values.  Arithmetic is
// term for term that of precond_wlevel and precond_tile_kernel: results
// are bitwise those of every other column variant.
template <typename T, int PT, int PC, int PU>
__global__ void __launch_bounds__(PT) precond_tile_batched_kernel(Dims d, Coef<T> c, CVec5<T> r, Vec5<T> out,
                                                                  const int* active) {
  if (active && *active == 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sm = reinterpret_cast<T*>(smem_raw);
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  T* s_x = sm;                    // [nz][PC]    rhs -> d' -> x
  T* s_W = s_x + nz * PC;         // [nz+1][PC]  w_tilde at w levels
  T* s_lo = s_W + (nz + 1) * PC;  // [nz][PC]    u face sum (A0-A1), then lower
  T* s_iv = s_lo + nz * PC;       // [nz][PC]    v face sum (A0-A1), then 1 / pivot
  T* s_cp = s_iv + nz * PC;       // [nz][PC]    c'
  const int i0 = blockIdx.x * PC;
  const int j = blockIdx.y;
  const int tid = threadIdx.x;
  const T* __restrict__ ru = r.f[0];
  const T* __restrict__ rv = r.f[1];
  const T* __restrict__ rw = r.f[2];
  const T* __restrict__ rp = r.f[3];
  const T* __restrict__ rW = r.f[4];
  T* __restrict__ ow = out.f[2];
  T* __restrict__ op = out.f[3];
  T* __restrict__ oW = out.f[4];
  const T inva = T(1) / (T)c.s.alpha;
  const T ips = (T)(1.0 / c.s.ps);
  const T ps = (T)c.s.ps;
  const int pm = nx * ny;
  const int nm = nz * PC, nw = (nz + 1) * PC;

  if (out.f[0] != ru) {
    const int ncol = min(PC + (i0 + PC >= nx ? 1 : 0), nx + 1 - i0);
    for (int q = tid; q < ncol * nz; q += PT) {
      const int k = q / ncol, ii = i0 + q % ncol;
      out.f[0][iu(d, ii, j, k)] = ld(ru, iu(d, ii, j, k));
    }
  }
  if (out.f[1] != rv) {
    const int ncol = min(PC, nx - i0);
    const int nj = (j == ny - 1) ? 2 : 1;
    for (int q = tid; q < ncol * nz * nj; q += PT) {
      const int jj = j + q / (ncol * nz), rem = q % (ncol * nz);
      const int k = rem / ncol, ii = i0 + rem % ncol;
      out.f[1][iv(d, ii, jj, k)] = ld(rv, iv(d, ii, jj, k));
    }
  }

  // ---- A0: face sums of u and v per mass level ----
  for (int q0 = tid; q0 < nm; q0 += PU * PT) {
    T a0[PU], a1[PU], b0[PU], b1[PU];
#pragma unroll
    for (int u = 0; u < PU; ++u) {
      const int q = q0 + u * PT;
      if (q < nm) {
        const int k = q / PC, i = min(i0 + q % PC, nx - 1);
        const int pu = iu(d, i, j, k), pv = iv(d, i, j, k);
        a0[u] = ld(ru, pu);
        a1[u] = ld(ru, pu + 1);
        b0[u] = ld(rv, pv);
        b1[u] = ld(rv, pv + nx);
      }
    }
#pragma unroll
    for (int u = 0; u < PU; ++u) {
      const int q = q0 + u * PT;
      if (q < nm) {
        s_lo[q] = a0[u] + a1[u];
        s_iv[q] = b0[u] + b1[u];
      }
    }
  }
  __syncthreads();
  // ---- A1: the w-level quantities (precond_wlevel) ----
  for (int q0 = tid; q0 < nw; q0 += PU * PT) {
    T zx[PU], ze[PU], wW[PU], rt[PU], ww[PU], id[PU], mq[PU];
#pragma unroll
    for (int u = 0; u < PU; ++u) {
      const int q = q0 + u * PT;
      if (q < nw) {
        const int k = q / PC, i = min(i0 + q % PC, nx - 1);
        const int kc = min(max(k, 1), nz - 1);
        const int p = i + nx * j + kc * pm;
        zx[u] = ld(c.zxw, p);
        ze[u] = ld(c.zew, p);
        wW[u] = ld(rW, p);
        rt[u] = ld(c.rtw, p);
        ww[u] = ld(rw, p);
        id[u] = ld(c.idamp, p);
        mq[u] = ld(c.mm, i + nx * j);
      }
    }
#pragma unroll
    for (int u = 0; u < PU; ++u) {
      const int q = q0 + u * PT;
      if (q < nw) {
        const int k = q / PC, l = q % PC, i = min(i0 + l, nx - 1);
        const int kc = min(max(k, 1), nz - 1);
        const T on = (k > 0 && k < nz) ? T(1) : T(0);
        const int ql = (kc - 1) * PC + l, qh = kc * PC + l;
        const T m4 = T(0.25) * mq[u];
        const T kin = m4 * ((s_lo[ql] + s_lo[qh]) * zx[u] + (s_iv[ql] + s_iv[qh]) * ze[u]);
        const T ep = wW[u] * inva - kin;
        s_W[q] = on * (rt[u] * (ww[u] * id[u] + ep));
        if (i0 + l < nx && k > 0 && k < nz) oW[i + nx * j + k * pm] = on * ep;
      }
    }
  }
  __syncthreads();
  // ---- A2: Helmholtz right-hand side and the factorisation ----
  for (int q0 = tid; q0 < nm; q0 += PU * PT) {
    T pp[PU], lp[PU], tl[PU], ti[PU], tc[PU];
#pragma unroll
    for (int u = 0; u < PU; ++u) {
      const int q = q0 + u * PT;
      if (q < nm) {
        const int k = q / PC, i = min(i0 + q % PC, nx - 1);
        const int p = i + nx * j + k * pm;
        pp[u] = ld(rp, p);
        lp[u] = ld(c.lpi, p);
        tl[u] = ld(c.tlo, p);
        ti[u] = ld(c.tinv, p);
        tc[u] = ld(c.tcp, p);
      }
    }
#pragma unroll
    for (int u = 0; u < PU; ++u) {
      const int q = q0 + u * PT;
      if (q < nm) {
        s_x[q] = pp[u] * ips - lp[u] * (s_W[q + PC] - s_W[q]);
        s_lo[q] = tl[u];
        s_iv[q] = ti[u];
        s_cp[q] = tc[u];
      }
    }
  }
  __syncthreads();
  // ---- B: Thomas with the prepared factorisation, one thread per column ----
  if (tid < PC) {
    const int l = tid;
    T dprev = T(0);
    for (int k = 0; k < nz; ++k) {
      const int q = k * PC + l;
      dprev = (s_x[q] - s_lo[q] * dprev) * s_iv[q];
      s_x[q] = dprev;
    }
    T xh = dprev;
    for (int k = nz - 2; k >= 0; --k) {
      const int q = k * PC + l;
      xh = s_x[q] - s_cp[q] * xh;
      s_x[q] = xh;
    }
  }
  __syncthreads();
  // ---- C: back substitution for w, eta_dot and the scaled pi ----
  T ww[PU], id[PU], pb[PU];
  auto c_load = [&](int q0) {
#pragma unroll
    for (int u = 0; u < PU; ++u) {
      const int q = q0 + u * PT;
      const int k = q / PC, i = i0 + q % PC;
      if (q < nw && i < nx) {
        const int p = i + nx * j + k * pm;
        ww[u] = ld(rw, p);
        const bool edge = (k == 0 || k == nz);
        id[u] = edge ? ld(rW, p) : ld(c.idamp, p);
        pb[u] = edge ? ld(c.dzw, p) : ld(c.pbw, p);
      }
    }
  };
  auto c_store = [&](int q0) {
#pragma unroll
    for (int u = 0; u < PU; ++u) {
      const int q = q0 + u * PT;
      const int k = q / PC, i = i0 + q % PC;
      if (q < nw && i < nx) {
        const int p = i + nx * j + k * pm;
        if (k == 0 || k == nz) {
          ow[p] = ww[u];
          oW[p] = id[u] * pb[u];
        } else {
          const T wv = ww[u] * id[u] - pb[u] * (s_x[q] - s_x[q - PC]);
          ow[p] = wv;
          oW[p] = oW[p] + wv;
        }
        if (k < nz) op[p] = s_x[q] * ps;
      }
    }
  };
  for (int q0 = tid; q0 < nw; q0 += PU * PT) {
    c_load(q0);
    c_store(q0);
  }
}

}  // namespace

template <typename T>
void launch_matvec(const Dims& d, const Coef<T>& c, CVec5<T> x, const double* xscale, CVec5<T> b,
                   Vec5<T> out, const int* active, cudaStream_t st) {
  if (d.tune_mv >= 6 && d.nz >= 2) {  // column march in 1, 2 or 4 z chunks
    const dim3 blk(32, 4, 1);
    dim3 grd((d.nx + 1 + 31) / 32, (d.ny + 1 + 3) / 4, d.tune_mv == 7 ? 2 : (d.tune_mv == 8 ? 4 : 1));
    matvec_march_kernel<T><<<grd, blk, 0, st>>>(d, c, x, xscale, b, out, active);
    return;
  }
  if (d.tune_mv == 4 || d.tune_mv == 5) {  // two or four levels per thread
    const dim3 blk(32, 8, 1);
    const int lv = d.tune_mv == 4 ? 2 : 4;
    dim3 grd((d.nx + 1 + 31) / 32, (d.ny + 1 + 7) / 8, (d.nz + lv) / lv);
    if (lv == 2) matvec_kernel<T, 2><<<grd, blk, 0, st>>>(d, c, x, xscale, b, out, active);
    else matvec_kernel<T, 4><<<grd, blk, 0, st>>>(d, c, x, xscale, b, out, active);
    return;
  }
  const dim3 blk = stencil_block(d.tune_mv);
  dim3 grd((d.nx + 1 + blk.x - 1) / blk.x, (d.ny + 1 + blk.y - 1) / blk.y, (d.nz + 1 + blk.z - 1) / blk.z);
  matvec_kernel<T, 1><<<grd, blk, 0, st>>>(d, c, x, xscale, b, out, active);
}

// ---------------------------------------------------------------------------
// Column march: one thread per (i, j) column, NT consecutive columns per
// block so every level's loads are coalesced across the warp.  Upward over
// the mass levels it forms w_tilde and the eta_dot/alpha - kin term at the
// w level above (parked in the eta_dot output), the Helmholtz RHS and the
// forward elimination d'(k) = (rhs - lower d'(k-1)) / pivot with the
// factorisation prepared once per core (prep_thomas); d' stays in shared
// memory.  Downward it back-substitutes x(k) = d'(k) - c'(k) x(k+1) and
// writes pi, w and eta_dot at the w level between x(k) and x(k+1).
// Shared memory per block: nz * NT values of T.
// ---------------------------------------------------------------------------
template <typename T, int NT>
__global__ void __launch_bounds__(NT) precond_march_kernel(Dims d, Coef<T> c, CVec5<T> r, Vec5<T> out,
                                                           const int* active) {
  if (active && *active == 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* s_d = reinterpret_cast<T*>(smem_raw);  // [nz][NT]
  const int t = threadIdx.x;
  const int i = blockIdx.x * NT + t, j = blockIdx.y;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i >= nx) return;
  const int pm = nx * ny, h = i + nx * j;
  const int pu = (nx + 1) * ny, pv = nx * (ny + 1);
  const T inva = T(1) / (T)c.s.alpha, ips = (T)(1.0 / c.s.ps), ps = (T)c.s.ps;
  const T* __restrict__ ru = r.f[0];
  const T* __restrict__ rv = r.f[1];
  const T* __restrict__ rw = r.f[2];
  const T* __restrict__ rp = r.f[3];
  const T* __restrict__ rW = r.f[4];
  T* __restrict__ ow = out.f[2];
  T* __restrict__ op = out.f[3];
  T* __restrict__ oW = out.f[4];
  const T mq = T(0.25) * ld(c.mm, h);
  const int ub = iu(d, i, j, 0), vb = iv(d, i, j, 0);
  // u over faces i, i+1 and v over faces j, j+1 at mass level k
  auto su = [&](int k) { const int q = ub + k * pu; return ld(ru, q) + ld(ru, q + 1); };
  auto sv = [&](int k) { const int q = vb + k * pv; return ld(rv, q) + ld(rv, q + nx); };
  T su_lo = su(0), sv_lo = sv(0);
  T wt_lo = T(0), dprev = T(0);
#pragma unroll 4
  for (int k = 0; k < nz; ++k) {
    const int p = h + k * pm;
    T wt_hi = T(0);
    if (k + 1 < nz) {  // interior w level k + 1 (steppers.py:211-219)
      const int pw = p + pm;
      const T su_hi = su(k + 1), sv_hi = sv(k + 1);
      const T kin = mq * ((su_lo + su_hi) * ld(c.zxw, pw) + (sv_lo + sv_hi) * ld(c.zew, pw));
      const T ep = ld(rW, pw) * inva - kin;
      wt_hi = ld(c.rtw, pw) * (ld(rw, pw) * ld(c.idamp, pw) + ep);
      oW[pw] = ep;
      su_lo = su_hi;
      sv_lo = sv_hi;
    }
    const T rhs = ld(rp, p) * ips - ld(c.lpi, p) * (wt_hi - wt_lo);  // steppers.py:223
    dprev = (rhs - ld(c.tlo, p) * dprev) * ld(c.tinv, p);
    s_d[k * NT + t] = dprev;
    wt_lo = wt_hi;
  }
  T xh = dprev;
  op[h + (nz - 1) * pm] = xh * ps;
#pragma unroll 4
  for (int k = nz - 2; k >= 0; --k) {  // steppers.py:227-245
    const int p = h + k * pm;
    const T x = s_d[k * NT + t] - ld(c.tcp, p) * xh;
    op[p] = x * ps;
    const int pw = p + pm;
    const T wv = ld(rw, pw) * ld(c.idamp, pw) - ld(c.pbw, pw) * (xh - x);
    ow[pw] = wv;
    oW[pw] = oW[pw] + wv;
    xh = x;
  }
  ow[h] = ld(rw, h);  // ground and lid rows (steppers.py:237-238, 244-245)
  oW[h] = ld(rW, h) * ld(c.dzw, h);
  const int ptop = h + nz * pm;
  ow[ptop] = ld(rw, ptop);
  oW[ptop] = ld(rW, ptop) * ld(c.dzw, ptop);
}

template <typename T, int NT>
void launch_precond_march(const Dims& d, const Coef<T>& c, CVec5<T> r, Vec5<T> out, const int* active,
                          cudaStream_t st) {
  const size_t smem = (size_t)d.nz * NT * sizeof(T);
  static SmemLimit attr_bytes;  // per instantiation
  ensure_smem_limit((const void*)precond_march_kernel<T, NT>, attr_bytes, smem);
  // u and v pass straight through (steppers.py:247-249) unless aliased
  if (out.f[0] != r.f[0])
    cudaMemcpyAsync(out.f[0], r.f[0], sizeof(T) * field_size(d, LOC_U), cudaMemcpyDeviceToDevice, st);
  if (out.f[1] != r.f[1])
    cudaMemcpyAsync(out.f[1], r.f[1], sizeof(T) * field_size(d, LOC_V), cudaMemcpyDeviceToDevice, st);
  precond_march_kernel<T, NT><<<dim3((d.nx + NT - 1) / NT, d.ny), NT, smem, st>>>(d, c, r, out, active);
}

// ---------------------------------------------------------------------------
// Pipelined column march: one thread per (i, j) column, NT consecutive
// columns per block (coalesced rows), the arithmetic of precond_march_kernel
// term for term (bitwise every other column variant).  Every level's global
// loads are issued two levels ahead of their use (a three-deep register
// ring), so a thread keeps about thirty loads in flight while the serial
// Thomas recurrence runs: with one thread per column the grid holds only
// nx * ny threads, and that memory-level parallelism per thread is what
// keeps HBM busy.  d' stays in shared memory (nz * NT values).  HINT = 1
// marks the values the downward sweep reads again (the eta_dot/alpha - kin
// term parked in the eta_dot output, the w right-hand side and 1/(1+dt tau))
// evict-last in L2 and the one-pass streams evict-first, so the re-reads
// can hit L2 instead of HBM.
// ---------------------------------------------------------------------------
__device__ __forceinline__ uint64_t l2_policy_evict_last() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_last.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ uint64_t l2_policy_evict_first() {
  uint64_t p;
  asm volatile("createpolicy.fractional.L2::evict_first.b64 %0, 1.0;" : "=l"(p));
  return p;
}
__device__ __forceinline__ float ld_hint(const float* q, uint64_t pol) {
  float v;
  asm volatile("ld.global.nc.L2::cache_hint.f32 %0, [%1], %2;" : "=f"(v) : "l"(q), "l"(pol));
  return v;
}
__device__ __forceinline__ double ld_hint(const double* q, uint64_t pol) {
  double v;
  asm volatile("ld.global.nc.L2::cache_hint.f64 %0, [%1], %2;" : "=d"(v) : "l"(q), "l"(pol));
  return v;
}
__device__ __forceinline__ void st_hint(float* q, float v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.f32 [%0], %1, %2;" ::"l"(q), "f"(v), "l"(pol) : "memory");
}
__device__ __forceinline__ void st_hint(double* q, double v, uint64_t pol) {
  asm volatile("st.global.L2::cache_hint.f64 [%0], %1, %2;" ::"l"(q), "d"(v), "l"(pol) : "memory");
}

template <typename T, int HINT>
__device__ __forceinline__ T ldp(const T* __restrict__ q, int i, uint64_t pol) {
  if (HINT) return ld_hint(q + i, pol);
  return ld(q, i);
}

template <typename T>
struct PcUp {  // inputs of upward step k: faces at mass level k + 1, w level k + 1, mass level k
  T u0, u1, v0, v1, zx, ze, W, rt, w, id, p, l, lo, inv;
};
template <typename T>
struct PcDown {  // inputs of downward step k: mass level k, w level k + 1
  T cp, w, id, pb, ep;
};

template <typename T, int NT, int HINT>
__device__ __forceinline__ void precond_pipe_block(const Dims& d, const Coef<T>& c, const CVec5<T>& r,
                                                   const Vec5<T>& out, int bx, int by) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* s_d = reinterpret_cast<T*>(smem_raw);  // [nz][NT]
  const int t = threadIdx.x;
  const int i = bx * NT + t, j = by;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i >= nx) return;
  const int pm = nx * ny, h = i + nx * j;
  const int pu = (nx + 1) * ny, pv = nx * (ny + 1);
  const T inva = T(1) / (T)c.s.alpha, ips = (T)(1.0 / c.s.ps), ps = (T)c.s.ps;
  const T* __restrict__ ru = r.f[0];
  const T* __restrict__ rv = r.f[1];
  const T* __restrict__ rw = r.f[2];
  const T* __restrict__ rp = r.f[3];
  const T* __restrict__ rW = r.f[4];
  T* __restrict__ ow = out.f[2];
  T* __restrict__ op = out.f[3];
  T* __restrict__ oW = out.f[4];
  const uint64_t keep = HINT ? l2_policy_evict_last() : 0, once = HINT ? l2_policy_evict_first() : 0;
  const T mq = T(0.25) * ld(c.mm, h);
  const int ub = iu(d, i, j, 0), vb = iv(d, i, j, 0);
  // loads of upward step k (indices clamped in bounds; values beyond the
  // column are never used)
  auto up = [&](int k) {
    PcUp<T> a;
    const int kf = min(k + 1, nz - 1), kw = min(k + 1, nz);
    const int qu = ub + kf * pu, qv = vb + kf * pv, pw = h + kw * pm, p = h + k * pm;
    a.u0 = ldp<T, HINT>(ru, qu, once);
    a.u1 = ldp<T, HINT>(ru, qu + 1, once);
    a.v0 = ldp<T, HINT>(rv, qv, once);
    a.v1 = ldp<T, HINT>(rv, qv + nx, once);
    a.zx = ldp<T, HINT>(c.zxw, pw, once);
    a.ze = ldp<T, HINT>(c.zew, pw, once);
    a.W = ldp<T, HINT>(rW, pw, once);
    a.rt = ldp<T, HINT>(c.rtw, pw, once);
    a.w = ldp<T, HINT>(rw, pw, keep);
    a.id = ldp<T, HINT>(c.idamp, pw, keep);
    a.p = ldp<T, HINT>(rp, p, once);
    a.l = ldp<T, HINT>(c.lpi, p, once);
    a.lo = ldp<T, HINT>(c.tlo, p, once);
    a.inv = ldp<T, HINT>(c.tinv, p, once);
    return a;
  };
  T su_lo = ld(ru, ub) + ld(ru, ub + 1), sv_lo = ld(rv, vb) + ld(rv, vb + nx);
  T wt_lo = T(0), dprev = T(0);
  PcUp<T> a = up(0), b = up(min(1, nz - 1));
  for (int k = 0; k < nz; ++k) {
    const PcUp<T> cnext = up(min(k + 2, nz - 1));
    T wt_hi = T(0);
    if (k + 1 < nz) {  // interior w level k + 1 (steppers.py:211-219)
      const T su_hi = a.u0 + a.u1, sv_hi = a.v0 + a.v1;
      const T kin = mq * ((su_lo + su_hi) * a.zx + (sv_lo + sv_hi) * a.ze);
      const T ep = a.W * inva - kin;
      wt_hi = a.rt * (a.w * a.id + ep);
      if (HINT) st_hint(oW + h + (k + 1) * pm, ep, keep);
      else oW[h + (k + 1) * pm] = ep;
      su_lo = su_hi;
      sv_lo = sv_hi;
    }
    const T rhs = a.p * ips - a.l * (wt_hi - wt_lo);  // steppers.py:223
    dprev = (rhs - a.lo * dprev) * a.inv;
    s_d[k * NT + t] = dprev;
    wt_lo = wt_hi;
    a = b;
    b = cnext;
  }
  // downward: x(k) = d'(k) - c'(k) x(k+1), then w and eta_dot at w level k+1
  auto down = [&](int k) {
    PcDown<T> e;
    const int p = h + k * pm, pw = p + pm;
    e.cp = ldp<T, HINT>(c.tcp, p, once);
    e.w = ldp<T, HINT>(rw, pw, keep);
    e.id = ldp<T, HINT>(c.idamp, pw, keep);
    e.pb = ldp<T, HINT>(c.pbw, pw, once);
    e.ep = oW[pw];
    return e;
  };
  T xh = dprev;
  op[h + (nz - 1) * pm] = xh * ps;
  if (nz >= 2) {
    PcDown<T> e = down(nz - 2), f = down(max(nz - 3, 0));
    for (int k = nz - 2; k >= 0; --k) {  // steppers.py:227-245
      const PcDown<T> gnext = down(max(k - 2, 0));
      const int p = h + k * pm, pw = p + pm;
      const T x = s_d[k * NT + t] - e.cp * xh;
      op[p] = x * ps;
      const T wv = e.w * e.id - e.pb * (xh - x);
      ow[pw] = wv;
      oW[pw] = e.ep + wv;
      xh = x;
      e = f;
      f = gnext;
    }
  }
  ow[h] = ld(rw, h);  // ground and lid rows (steppers.py:237-238, 244-245)
  oW[h] = ld(rW, h) * ld(c.dzw, h);
  const int ptop = h + nz * pm;
  ow[ptop] = ld(rw, ptop);
  oW[ptop] = ld(rW, ptop) * ld(c.dzw, ptop);
}
template <typename T, int NT, int HINT>
__global__ void __launch_bounds__(NT) precond_pipe_kernel(Dims d, Coef<T> c, CVec5<T> r, Vec5<T> out,
                                                          const int* active) {
  if (active && *active == 0) return;
  precond_pipe_block<T, NT, HINT>(d, c, r, out, blockIdx.x, blockIdx.y);
}

// ---------------------------------------------------------------------------
// Asynchronous-copy column march: the one-thread-per-column arithmetic of
// precond_pipe_kernel, but every level's inputs are copied global -> shared
// with cp.async (each thread its own values, S - 1 levels ahead, one copy
// group per level), so the loads in flight hold no registers and each
// thread reads back only what it copied itself (no block barrier).
// Shared memory per block: (nz + 16 S) * NT values of T.
// ---------------------------------------------------------------------------
template <typename T, int NT, int S>
__global__ void __launch_bounds__(NT) precond_async_kernel(Dims d, Coef<T> c, CVec5<T> r, Vec5<T> out,
                                                           const int* active) {
  if (active && *active == 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nz = d.nz;
  T* s_d = reinterpret_cast<T*>(smem_raw);  // [nz][NT]
  T* ring = s_d + nz * NT;                   // [S][16][NT]
  const int t = threadIdx.x;
  const int i = blockIdx.x * NT + t, j = blockIdx.y;
  const int nx = d.nx, ny = d.ny;
  if (i >= nx) return;
  const int pm = nx * ny, h = i + nx * j;
  const int pu = (nx + 1) * ny, pv = nx * (ny + 1);
  const T inva = T(1) / (T)c.s.alpha, ips = (T)(1.0 / c.s.ps), ps = (T)c.s.ps;
  const T* __restrict__ ru = r.f[0];
  const T* __restrict__ rv = r.f[1];
  const T* __restrict__ rw = r.f[2];
  const T* __restrict__ rp = r.f[3];
  const T* __restrict__ rW = r.f[4];
  T* __restrict__ ow = out.f[2];
  T* __restrict__ op = out.f[3];
  T* __restrict__ oW = out.f[4];
  const T mq = T(0.25) * ld(c.mm, h);
  const int ub = iu(d, i, j, 0), vb = iv(d, i, j, 0);
  // the 14 inputs of upward step k into ring slot `slot` (clamped in bounds)
  auto issue_up = [&](int k, int slot) {
    k = min(k, nz - 1);
    const int kf = min(k + 1, nz - 1), kw = min(k + 1, nz);
    const int qu = ub + kf * pu, qv = vb + kf * pv, pw = h + kw * pm, p = h + k * pm;
    T* q = ring + slot * 16 * NT + t;
    cp_async_t(q + 0 * NT, ru + qu);
    cp_async_t(q + 1 * NT, ru + qu + 1);
    cp_async_t(q + 2 * NT, rv + qv);
    cp_async_t(q + 3 * NT, rv + qv + nx);
    cp_async_t(q + 4 * NT, c.zxw + pw);
    cp_async_t(q + 5 * NT, c.zew + pw);
    cp_async_t(q + 6 * NT, rW + pw);
    cp_async_t(q + 7 * NT, c.rtw + pw);
    cp_async_t(q + 8 * NT, rw + pw);
    cp_async_t(q + 9 * NT, c.idamp + pw);
    cp_async_t(q + 10 * NT, rp + p);
    cp_async_t(q + 11 * NT, c.lpi + p);
    cp_async_t(q + 12 * NT, c.tlo + p);
    cp_async_t(q + 13 * NT, c.tinv + p);
  };
  T su_lo = ld(ru, ub) + ld(ru, ub + 1), sv_lo = ld(rv, vb) + ld(rv, vb + nx);
  T wt_lo = T(0), dprev = T(0);
#pragma unroll
  for (int q = 0; q < S - 1; ++q) {
    issue_up(q, q);
    cp_async_commit();
  }
  for (int k = 0; k < nz; ++k) {
    issue_up(k + S - 1, (k + S - 1) % S);
    cp_async_commit();
    cp_async_wait<S - 1>();  // level k's group has landed
    const T* a = ring + (k % S) * 16 * NT + t;
    T wt_hi = T(0);
    if (k + 1 < nz) {  // interior w level k + 1 (steppers.py:211-219)
      const T su_hi = a[0 * NT] + a[1 * NT], sv_hi = a[2 * NT] + a[3 * NT];
      const T kin = mq * ((su_lo + su_hi) * a[4 * NT] + (sv_lo + sv_hi) * a[5 * NT]);
      const T ep = a[6 * NT] * inva - kin;
      wt_hi = a[7 * NT] * (a[8 * NT] * a[9 * NT] + ep);
      oW[h + (k + 1) * pm] = ep;
      su_lo = su_hi;
      sv_lo = sv_hi;
    }
    const T rhs = a[10 * NT] * ips - a[11 * NT] * (wt_hi - wt_lo);  // steppers.py:223
    dprev = (rhs - a[12 * NT] * dprev) * a[13 * NT];
    s_d[k * NT + t] = dprev;
    wt_lo = wt_hi;
  }
  cp_async_wait<0>();  // the ring is reused below
  // downward: x(k) = d'(k) - c'(k) x(k+1), then w and eta_dot at w level k+1
  auto issue_down = [&](int k, int slot) {
    k = max(k, 0);
    const int p = h + k * pm, pw = p + pm;
    T* q = ring + slot * 16 * NT + t;
    cp_async_t(q + 0 * NT, c.tcp + p);
    cp_async_t(q + 1 * NT, rw + pw);
    cp_async_t(q + 2 * NT, c.idamp + pw);
    cp_async_t(q + 3 * NT, c.pbw + pw);
    cp_async_t(q + 4 * NT, oW + pw);  // this thread's own eta_dot/alpha - kin of the upward sweep
  };
  T xh = dprev;
  op[h + (nz - 1) * pm] = xh * ps;
  if (nz >= 2) {
#pragma unroll
    for (int q = 0; q < S - 1; ++q) {
      issue_down(nz - 2 - q, q);
      cp_async_commit();
    }
    for (int k = nz - 2, n = 0; k >= 0; --k, ++n) {  // steppers.py:227-245
      issue_down(k - (S - 1), (n + S - 1) % S);
      cp_async_commit();
      cp_async_wait<S - 1>();
      const T* e = ring + (n % S) * 16 * NT + t;
      const int p = h + k * pm, pw = p + pm;
      const T x = s_d[k * NT + t] - e[0 * NT] * xh;
      op[p] = x * ps;
      const T wv = e[1 * NT] * e[2 * NT] - e[3 * NT] * (xh - x);
      ow[pw] = wv;
      oW[pw] = e[4 * NT] + wv;
      xh = x;
    }
    cp_async_wait<0>();
  }
  ow[h] = ld(rw, h);  // ground and lid rows (steppers.py:237-238, 244-245)
  oW[h] = ld(rW, h) * ld(c.dzw, h);
  const int ptop = h + nz * pm;
  ow[ptop] = ld(rw, ptop);
  oW[ptop] = ld(rW, ptop) * ld(c.dzw, ptop);
}

template <typename T, int NT, int S>
void launch_precond_async(const Dims& d, const Coef<T>& c, CVec5<T> r, Vec5<T> out, const int* active,
                          cudaStream_t st) {
  const size_t smem = (size_t)(d.nz + 16 * S) * NT * sizeof(T);
  static SmemLimit attr_bytes;  // per instantiation
  ensure_smem_limit((const void*)precond_async_kernel<T, NT, S>, attr_bytes, smem);
  if (out.f[0] != r.f[0])
    cudaMemcpyAsync(out.f[0], r.f[0], sizeof(T) * field_size(d, LOC_U), cudaMemcpyDeviceToDevice, st);
  if (out.f[1] != r.f[1])
    cudaMemcpyAsync(out.f[1], r.f[1], sizeof(T) * field_size(d, LOC_V), cudaMemcpyDeviceToDevice, st);
  precond_async_kernel<T, NT, S><<<dim3((d.nx + NT - 1) / NT, d.ny), NT, smem, st>>>(d, c, r, out, active);
}

template <typename T, int NT, int HINT>
void launch_precond_pipe(const Dims& d, const Coef<T>& c, CVec5<T> r, Vec5<T> out, const int* active,
                         cudaStream_t st) {
  const size_t smem = (size_t)d.nz * NT * sizeof(T);
  static SmemLimit attr_bytes;  // per instantiation
  ensure_smem_limit((const void*)precond_pipe_kernel<T, NT, HINT>, attr_bytes, smem);
  // u and v pass straight through (steppers.py:247-249) unless aliased
  if (out.f[0] != r.f[0])
    cudaMemcpyAsync(out.f[0], r.f[0], sizeof(T) * field_size(d, LOC_U), cudaMemcpyDeviceToDevice, st);
  if (out.f[1] != r.f[1])
    cudaMemcpyAsync(out.f[1], r.f[1], sizeof(T) * field_size(d, LOC_V), cudaMemcpyDeviceToDevice, st);
  precond_pipe_kernel<T, NT, HINT><<<dim3((d.nx + NT - 1) / NT, d.ny), NT, smem, st>>>(d, c, r, out, active);
}

template <typename T, int PT, int PC>
void launch_precond_tile(const Dims& d, const Coef<T>& c, CVec5<T> r, Vec5<T> out, const int* active,
                         cudaStream_t st) {
  const size_t smem = (size_t)(5 * d.nz + 1) * PC * sizeof(T);
  static SmemLimit attr_bytes;  // per instantiation
  ensure_smem_limit((const void*)precond_tile_kernel<T, PT, PC>, attr_bytes, smem);
  dim3 grd((d.nx + PC - 1) / PC, d.ny);
  precond_tile_kernel<T, PT, PC><<<grd, PT, smem, st>>>(d, c, r, out, active);
}

template <typename T, int PT, int PC, int PU>
void launch_precond_tile_batched(const Dims& d, const Coef<T>& c, CVec5<T> r, Vec5<T> out, const int* active,
                                 cudaStream_t st) {
  const size_t smem = (size_t)(5 * d.nz + 1) * PC * sizeof(T);
  static SmemLimit attr_bytes;  // per instantiation
  ensure_smem_limit((const void*)precond_tile_batched_kernel<T, PT, PC, PU>, attr_bytes, smem);
  dim3 grd((d.nx + PC - 1) / PC, d.ny);
  precond_tile_batched_kernel<T, PT, PC, PU><<<grd, PT, smem, st>>>(d, c, r, out, active);
}

template <typename T>
void launch_precond(const Dims& d, const Coef<T>& c, CVec5<T> r, Vec5<T> out, const int* active,
                    cudaStream_t st) {
  int v = d.tune_pc;
  if (v == 2 && (size_t)(5 * d.nz + 1) * 64 * sizeof(T) > 200 * 1024) v = 0;  // 64-column tile too large
  switch (v) {
    case 1: launch_precond_tile<T, 128, 16>(d, c, r, out, active, st); break;
    case 2: launch_precond_tile<T, 256, 64>(d, c, r, out, active, st); break;
    case 3: launch_precond_march<T, 128>(d, c, r, out, active, st); break;
    case 4: launch_precond_tile_batched<T, 256, 32, 4>(d, c, r, out, active, st); break;
    case 5: launch_precond_pipe<T, 64, 0>(d, c, r, out, active, st); break;
    case 6: launch_precond_pipe<T, 64, 1>(d, c, r, out, active, st); break;
    case 7: launch_precond_async<T, 32, 6>(d, c, r, out, active, st); break;
    default: launch_precond_tile<T, 256, 32>(d, c, r, out, active, st); break;
  }
}

// ---------------------------------------------------------------------------
// grouped matvec and preconditioner over ensemble members (sisl_group.cuh):
// flat block b runs block (b - first[m]) of member m's column march
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T* gvec_l(const GroupMember<T>& g, int v) {
  return g.vec + (size_t)v * g.npad;
}

// mode 0: Arnoldi step j (gated), V_j scaled by s_j -> V_{j+1} (u, v) | z;
// mode 1: b - A x -> V_0 (u, v) | z; mode 2 (U = double): b64 - A64 x64 -> r64
template <typename T, typename U>
__global__ void __launch_bounds__(128, sizeof(U) == 4 ? 3 : 2) group_matvec_kernel(GroupMember<T>* mem,
                                                                                  const int* __restrict__ first,
                                                                                  int M, int mode, int j) {
  const int b = blockIdx.x;
  const int mi = group_find(first, M, b);
  const GroupMember<T>& g = mem[mi];
  if (!g.running) return;
  if (mode == 0 && g.gs->active == 0) return;
  const int gx = (g.d.nx + 1 + 31) / 32, gy = (g.d.ny + 1 + 3) / 4;
  const int t = b - first[mi];
  const int bz = t / (gx * gy), rr = t - bz * (gx * gy), by = rr / gx, bx = rr - by * gx;
  // the scale pointer stays a run-time value in every mode (a literal null
  // would let the compiler fold x * 1 and contract the rows into other FMAs
  // than the standalone kernel's, changing the last bits)
  const double* xsp = (mode == 0) ? &g.gs->s[j] : nullptr;
  if constexpr (sizeof(U) == sizeof(T)) {
    const T* src = gvec_l(g, mode == 0 ? GV_V0 + j : GV_X);
    T* tgt = gvec_l(g, mode == 0 ? GV_V0 + j + 1 : GV_V0);
    T* z = gvec_l(g, GV_Z);
    const T* bv = gvec_l(g, GV_B);
    CVec5<T> x, bb;
    Vec5<T> out;
    for (int q = 0; q < 5; ++q) {
      x.f[q] = src + g.off[q];
      bb.f[q] = (mode == 1) ? bv + g.off[q] : nullptr;
      out.f[q] = (q < 2 ? tgt : z) + g.off[q];
    }
    matvec_march_block<T>(g.d, g.c, x, xsp, bb, out, bx, by, bz, 1);
  } else {
    CVec5<double> x, bb;
    Vec5<double> out;
    for (int q = 0; q < 5; ++q) {
      x.f[q] = g.x64 + g.off[q];
      bb.f[q] = g.b64 + g.off[q];
      out.f[q] = g.r64 + g.off[q];
    }
    matvec_march_block<double>(g.d, g.c64, x, xsp, bb, out, bx, by, bz, 1);
  }
}

// mode 0: target V_t: u, v already there, w, pi, eta_dot from z (gated when
// t >= 1); mode 1: M b -> V_1 (u, v copied by the caller)
template <typename T, int NT>
__global__ void __launch_bounds__(NT) group_precond_kernel(GroupMember<T>* mem, const int* __restrict__ first, int M,
                                                           int mode, int tv, int gated) {
  const int b = blockIdx.x;
  const int mi = group_find(first, M, b);
  const GroupMember<T>& g = mem[mi];
  if (!g.running || (gated && g.gs->active == 0)) return;
  const int gx = (g.d.nx + NT - 1) / NT;
  const int t = b - first[mi];
  const int by = t / gx, bx = t - by * gx;
  T* tgt = gvec_l(g, mode == 0 ? GV_V0 + tv : GV_V0 + 1);
  const T* src = (mode == 0) ? gvec_l(g, GV_Z) : gvec_l(g, GV_B);
  CVec5<T> r;
  Vec5<T> out;
  for (int q = 0; q < 5; ++q) {
    r.f[q] = (q < 2 && mode == 0 ? tgt : src) + g.off[q];
    out.f[q] = tgt + g.off[q];
  }
  precond_pipe_block<T, NT, 1>(g.d, g.c, r, out, bx, by);
}

// ---------------------------------------------------------------------------
// grouped host wrappers
// ---------------------------------------------------------------------------
constexpr int GROUP_PC_NT = 64;
int group_matvec_blocks(const Dims& d) { return ((d.nx + 1 + 31) / 32) * ((d.ny + 1 + 3) / 4); }
int group_precond_blocks(const Dims& d) { return ((d.nx + GROUP_PC_NT - 1) / GROUP_PC_NT) * d.ny; }

template <typename T>
void grp_matvec(const GroupLaunch<T>& g, int mode, int j, cudaStream_t st) {
  const int nb = g.blocks(GT_MV);
  if (mode == 2) {
    if constexpr (sizeof(T) == 4) group_matvec_kernel<T, double><<<nb, dim3(32, 4), 0, st>>>(g.mem, g.row(GT_MV), g.M, 2, 0);
    return;
  }
  group_matvec_kernel<T, T><<<nb, dim3(32, 4), 0, st>>>(g.mem, g.row(GT_MV), g.M, mode, j);
}

template <typename T>
void grp_precond(const GroupLaunch<T>& g, int mode, int t, int gated, cudaStream_t st) {
  int nz_max = 1;
  for (int m = 0; m < g.M; ++m) nz_max = nz_max > g.nz_h[m] ? nz_max : g.nz_h[m];
  const size_t smem = (size_t)nz_max * GROUP_PC_NT * sizeof(T);
  static SmemLimit attr_bytes;
  ensure_smem_limit((const void*)group_precond_kernel<T, GROUP_PC_NT>, attr_bytes, smem);
  group_precond_kernel<T, GROUP_PC_NT><<<g.blocks(GT_PC), GROUP_PC_NT, smem, st>>>(g.mem, g.row(GT_PC), g.M, mode, t,
                                                                                   gated);
}

template void grp_matvec<float>(const GroupLaunch<float>&, int, int, cudaStream_t);
template void grp_matvec<double>(const GroupLaunch<double>&, int, int, cudaStream_t);
template void grp_precond<float>(const GroupLaunch<float>&, int, int, int, cudaStream_t);
template void grp_precond<double>(const GroupLaunch<double>&, int, int, int, cudaStream_t);

template void launch_matvec<float>(const Dims&, const Coef<float>&, CVec5<float>, const double*, CVec5<float>,
                                   Vec5<float>, const int*, cudaStream_t);
template void launch_matvec<double>(const Dims&, const Coef<double>&, CVec5<double>, const double*,
                                    CVec5<double>, Vec5<double>, const int*, cudaStream_t);
template void launch_precond<float>(const Dims&, const Coef<float>&, CVec5<float>, Vec5<float>, const int*,
                                    cudaStream_t);
template void launch_precond<double>(const Dims&, const Coef<double>&, CVec5<double>, Vec5<double>,
                                     const int*, cudaStream_t);

}  // namespace sisl
