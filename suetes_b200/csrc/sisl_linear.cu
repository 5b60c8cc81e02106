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
#include "sisl_core.cuh"

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
  const T Pl = ld(p, base + kl * plane) * sp, P0 = ld(p, base + k * plane) * sp, Ph = ld(p, base + kh * plane) * sp;
  const T g0 = (k == 0 ? Ph - P0 : P0 - Pl) * ld(iz, base + k * plane);
  const T g1 = (k + 1 == nz ? P0 - Pl : Ph - P0) * ld(iz, base + (k + 1) * plane);
  return T(0.5) * (g0 + g1);
}

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
  const T adt = (T)(c.s.alpha * c.s.dt), cp = (T)c.s.cp, a = (T)c.s.alpha, ps = (T)c.s.ps;
  const T sp = xs / ps;
  const T idx = (T)(1.0 / d.dx), idy = (T)(1.0 / d.dy);
  const int pm = nx * ny;
  const T* __restrict__ xu = x.f[0];
  const T* __restrict__ xv = x.f[1];
  const T* __restrict__ xw = x.f[2];
  const T* __restrict__ xp = x.f[3];
  const T* __restrict__ xW = x.f[4];
  const bool own = (i < nx && j < ny);
  const int il = (i == 0) ? nx - 1 : i - 1;
  const int jl = (j == 0) ? ny - 1 : j - 1;
  const int hO = i + nx * j;  // own column (valid when own)
  T gmO = T(0);
  if (own && k < nz) gmO = gz_mass(xp, c.idzw, hO, k, nz, pm, sp);

  if (k < nz) {
    // ---- u face (i, j, k) ----
    if (j < ny && !(d.px && i == nx)) {
      const int p = iu(d, i, j, k);
      T L;
      if (!d.px && (i == 0 || i == nx)) {
        L = ld(xu, p) * xs;  // locked open boundary (euler.py:414-415)
      } else {
        const int hX = il + nx * j;
        const T gmX = gz_mass(xp, c.idzw, hX, k, nz, pm, sp);
        const T gpx = (ld(xp, hO + k * pm) - ld(xp, hX + k * pm)) * sp * idx * ld(c.mu, h_u(d, i, j));
        const int vr = iv(d, i, j, k), vl = iv(d, il, j, k);
        const T vat = T(0.25) * (ld(xv, vl) + ld(xv, vl + nx) + ld(xv, vr) + ld(xv, vr + nx)) * xs;
        const T tend = -cp * ld(c.thu, p) * (gpx - ld(c.zxu, p) * T(0.5) * (gmX + gmO)) + ld(c.fu, h_u(d, i, j)) * vat;
        L = ld(xu, p) * xs - adt * tend;
      }
      out.f[0][p] = b.f[0] ? ld(b.f[0], p) - L : L;
      if (d.px && i == 0) {
        const int pn = iu(d, nx, j, k);
        out.f[0][pn] = b.f[0] ? ld(b.f[0], pn) - L : L;
      }
    }
    // ---- v face (i, j, k) ----
    if (i < nx && !(d.py && j == ny)) {
      const int p = iv(d, i, j, k);
      T L;
      if (!d.py && (j == 0 || j == ny)) {
        L = ld(xv, p) * xs;
      } else {
        const int hY = i + nx * jl;
        const T gmY = gz_mass(xp, c.idzw, hY, k, nz, pm, sp);
        const T gpy = (ld(xp, hO + k * pm) - ld(xp, hY + k * pm)) * sp * idy * ld(c.mv, h_v(d, i, j));
        const int ur = iu(d, i, j, k), ul = iu(d, i, jl, k);
        const T uat = T(0.25) * (ld(xu, ul) + ld(xu, ul + 1) + ld(xu, ur) + ld(xu, ur + 1)) * xs;
        const T tend = -cp * ld(c.thv, p) * (gpy - ld(c.zev, p) * T(0.5) * (gmY + gmO)) - ld(c.fv, h_v(d, i, j)) * uat;
        L = ld(xv, p) * xs - adt * tend;
      }
      out.f[1][p] = b.f[1] ? ld(b.f[1], p) - L : L;
      if (d.py && j == 0) {
        const int pn = iv(d, i, ny, k);
        out.f[1][pn] = b.f[1] ? ld(b.f[1], pn) - L : L;
      }
    }
  }
  if (!own) return;
  // ---- w level k: w and eta_dot rows ----
  const int pw = hO + k * pm;
  T Lw, Le;
  if (k == 0 || k == nz) {
    Lw = ld(xw, pw) * xs;                      // euler.py:426-427
    Le = ld(xW, pw) * xs * ld(c.idzw, pw);     // eta_dot = W / dz_w (euler.py:436-437)
  } else {
    const T gzw = (ld(xp, hO + k * pm) - ld(xp, hO + (k - 1) * pm)) * sp * ld(c.idzw, pw);
    Lw = ld(c.damp, pw) * ld(xw, pw) * xs + adt * cp * ld(c.thw, pw) * gzw;
    const int u1 = iu(d, i, j, k), u0 = u1 - (nx + 1) * ny;
    const int v1 = iv(d, i, j, k), v0 = v1 - nx * (ny + 1);
    const T uw = T(0.25) * (ld(xu, u0) + ld(xu, u0 + 1) + ld(xu, u1) + ld(xu, u1 + 1)) * xs;
    const T vw = T(0.25) * (ld(xv, v0) + ld(xv, v0 + nx) + ld(xv, v1) + ld(xv, v1 + nx)) * xs;
    Le = a * (ld(xW, pw) * xs + ld(c.mm, hO) * (uw * ld(c.zxw, pw) + vw * ld(c.zew, pw)) - ld(xw, pw) * xs);
  }
  if (b.f[2]) { Lw = ld(b.f[2], pw) - Lw; Le = ld(b.f[4], pw) - Le; }
  out.f[2][pw] = Lw;
  out.f[4][pw] = Le;
  if (k == nz) return;
  // ---- mass point: pi row ----
  const int u0 = iu(d, i, j, k), v0 = iv(d, i, j, k);
  const T fx0 = ld(xu, u0) * ld(c.rdu, u0) * ld(c.thu, u0);
  const T fx1 = ld(xu, u0 + 1) * ld(c.rdu, u0 + 1) * ld(c.thu, u0 + 1);
  const T fy0 = ld(xv, v0) * ld(c.rdv, v0) * ld(c.thv, v0);
  const T fy1 = ld(xv, v0 + nx) * ld(c.rdv, v0 + nx) * ld(c.thv, v0 + nx);
  const T fz0 = (k == 0) ? T(0) : ld(xW, pw) * ld(c.rhow, pw) * ld(c.thw, pw);
  const int pw1 = pw + pm;
  const T fz1 = (k + 1 == nz) ? T(0) : ld(xW, pw1) * ld(c.rhow, pw1) * ld(c.thw, pw1);
  const T m = ld(c.mm, hO);
  const T divh = m * m * ((fx1 - fx0) * idx + (fy1 - fy0) * idy);
  const T tend = -ld(c.cpidz, pw) * (xs * (divh + (fz1 - fz0)));
  const T L = ld(xp, pw) * xs - adt * ps * tend;
  out.f[3][pw] = b.f[3] ? ld(b.f[3], pw) - L : L;
}

// ---------------------------------------------------------------------------
// Column-tile preconditioner: a block owns 32 consecutive columns (same j).
//   A: all threads compute w_tilde and the eta partial at the interior w
//      levels and the Helmholtz RHS at the mass levels, and stage the Thomas
//      coefficients, into shared memory (coalesced, fully parallel loads);
//   B: warp 0 runs the forward/backward recurrences of its 32 columns from
//      shared memory;
//   C: all threads write w, eta_dot and pi from the solution.
// Shared memory per block: (6 nz + 2) * 32 values of T.
// ---------------------------------------------------------------------------
constexpr int PT = 256;  // threads per block
constexpr int PC = 32;   // columns per block

template <typename T>
__global__ void __launch_bounds__(PT) precond_tile_kernel(Dims d, Coef<T> c, CVec5<T> r, Vec5<T> out,
                                                          const int* active) {
  if (active && *active == 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sm = reinterpret_cast<T*>(smem_raw);
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  T* s_x = sm;                        // [nz][PC]  rhs -> d' -> x
  T* s_low = s_x + nz * PC;           // [nz][PC]
  T* s_inv = s_low + nz * PC;         // [nz][PC]
  T* s_cp = s_inv + nz * PC;          // [nz][PC]
  T* s_wt = s_cp + nz * PC;           // [nz+1][PC]  w_tilde at w levels
  T* s_ep = s_wt + (nz + 1) * PC;     // [nz+1][PC]  eta_dot / alpha - kin
  const int i0 = blockIdx.x * PC;
  const int j = blockIdx.y;
  const int tid = threadIdx.x;
  const T* __restrict__ ru = r.f[0];
  const T* __restrict__ rv = r.f[1];
  const T* __restrict__ rw = r.f[2];
  const T* __restrict__ rp = r.f[3];
  const T* __restrict__ rW = r.f[4];
  const T a = (T)c.s.alpha;
  const T inva = T(1) / a;
  const T ips = (T)(1.0 / c.s.ps);
  const T ps = (T)c.s.ps;
  const T adtcp = (T)(c.s.alpha * c.s.dt * c.s.cp);

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

  // ---- A1: interior w levels ----
#pragma unroll 4
  for (int q = tid; q < (nz + 1) * PC; q += PT) {
    const int k = q / PC, l = q % PC, i = i0 + l;
    T wt = T(0), ep = T(0);
    if (i < nx && k > 0 && k < nz) {
      const int p = iw(d, i, j, k);
      const T um0 = T(0.5) * (ld(ru, iu(d, i, j, k - 1)) + ld(ru, iu(d, i + 1, j, k - 1)));
      const T um1 = T(0.5) * (ld(ru, iu(d, i, j, k)) + ld(ru, iu(d, i + 1, j, k)));
      const T vm0 = T(0.5) * (ld(rv, iv(d, i, j, k - 1)) + ld(rv, iv(d, i, j + 1, k - 1)));
      const T vm1 = T(0.5) * (ld(rv, iv(d, i, j, k)) + ld(rv, iv(d, i, j + 1, k)));
      const T kin = ld(c.mm, h_m(d, i, j)) * (T(0.5) * (um0 + um1) * ld(c.zxw, p) + T(0.5) * (vm0 + vm1) * ld(c.zew, p));
      ep = ld(rW, p) * inva - kin;
      wt = ld(c.rhow, p) * ld(c.thw, p) * (ld(rw, p) / ld(c.damp, p) + ep);
    }
    s_wt[q] = wt;
    s_ep[q] = ep;
  }
  __syncthreads();
  // ---- A2: Helmholtz RHS at mass levels and the Thomas coefficients ----
#pragma unroll 4
  for (int q = tid; q < nz * PC; q += PT) {
    const int k = q / PC, l = q % PC, i = i0 + l;
    if (i < nx) {
      const int p = im(d, i, j, k);
      s_x[q] = ld(rp, p) * ips - ld(c.lpi, p) * (s_wt[q + PC] - s_wt[q]);
      s_low[q] = ld(c.tlow, p);
      s_inv[q] = ld(c.tinv, p);
      s_cp[q] = ld(c.tcp, p);
    }
  }
  __syncthreads();
  // ---- B: recurrences, one lane per column ----
  if (tid < PC) {
    const int l = tid;
    T dprev = s_x[l] * s_inv[l];
    s_x[l] = dprev;
#pragma unroll 8
    for (int k = 1; k < nz; ++k) {
      const int q = k * PC + l;
      dprev = (s_x[q] - s_low[q] * dprev) * s_inv[q];
      s_x[q] = dprev;
    }
    T xh = dprev;
#pragma unroll 8
    for (int k = nz - 2; k >= 0; --k) {
      const int q = k * PC + l;
      xh = s_x[q] - s_cp[q] * xh;
      s_x[q] = xh;
    }
  }
  __syncthreads();
  // ---- C: back substitution for w, eta_dot and the scaled pi ----
#pragma unroll 4
  for (int q = tid; q < (nz + 1) * PC; q += PT) {
    const int k = q / PC, l = q % PC, i = i0 + l;
    if (i >= nx) continue;
    const int p = iw(d, i, j, k);
    if (k == 0 || k == nz) {  // boundary rows (steppers.py:237-238, 244-245)
      out.f[2][p] = ld(rw, p);
      out.f[4][p] = ld(rW, p) * ld(c.dzw, p);
    } else {
      const T grad = (s_x[q] - s_x[q - PC]) * ld(c.idzw, p);
      const T wv = (ld(rw, p) - adtcp * ld(c.thw, p) * grad) / ld(c.damp, p);
      out.f[2][p] = wv;
      out.f[4][p] = s_ep[q] + wv;
    }
    if (k < nz) out.f[3][im(d, i, j, k)] = s_x[q] * ps;
  }
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
  const size_t smem = (size_t)(6 * d.nz + 2) * PC * sizeof(T);
  static size_t attr_bytes = 0;  // per instantiation
  if (smem > 48 * 1024 && smem > attr_bytes) {
    cudaFuncSetAttribute(precond_tile_kernel<T>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    attr_bytes = smem;
  }
  dim3 grd((d.nx + PC - 1) / PC, d.ny);
  precond_tile_kernel<T><<<grd, PT, smem, st>>>(d, c, r, out, active);
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
