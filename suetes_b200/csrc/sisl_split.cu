// Split-explicit RK3 core (SplitExplicitStepper3D, steppers.py:1076-1737).
//
// One RK3 stage is: the explicit tendencies of the stage state (the explicit
// kernel, mode 1) plus the 3rd-order upwind flux advection of th', u_m,
// v_m, w_m (split_adv_kernel) averaged to the staggers (split_slow_kernel);
// then n acoustic sub-steps of three kernels: the horizontal predictor to
// the midpoint (split_predict_kernel), the vertically implicit pi''/w''
// column solve (split_column_kernel, one thread per column, Thomas in the
// float arithmetic of the tridiagonal solve), and the centred corrector with
// the backward w damping (split_correct_kernel); split_end_kernel assembles
// the stage state and split_diag_kernel diagnoses eta_dot and the kinematic
// w boundaries.  Every kernel is one thread per output point (columns for
// the solve) and HBM-bound.
#include "sisl_explicit_dev.cuh"
#include "sisl_split.cuh"

namespace sisl {
namespace {

using dev::Grad;
using dev::Winds;

dim3 box(int ex, int ey, int ez, dim3 blk) {
  return dim3((ex + blk.x - 1) / blk.x, (ey + blk.y - 1) / blk.y, (ez + blk.z - 1) / blk.z);
}

// m_w (u_w z_xi_w + v_w z_eta_w) at w level k of column (i, j)  (steppers.py:1296-1300)
template <typename T>
__device__ __forceinline__ T kinematic(const Dims& d, const Coef<T>& c, const Winds<T>& W, int i, int j, int k) {
  const int p = iw(d, i, j, k);
  return ld(c.mm, h_m(d, i, j)) * (W.uw(i, j, k) * ld(c.zxw, p) + W.vw(i, j, k) * ld(c.zew, p));
}

template <typename T>
__global__ void split_diag_kernel(Dims d, Coef<T> c, const T* __restrict__ u, const T* __restrict__ v,
                                  const T* w_in, T* eta_out, T* w_out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= d.nx || j >= d.ny || k > d.nz) return;
  const Winds<T> W{d, c, u, v};
  const int p = iw(d, i, j, k);
  if (k == 0) {
    w_out[p] = kinematic(d, c, W, i, j, 0);  // flow glides over the slope
    eta_out[p] = T(0);
  } else if (k == d.nz) {
    w_out[p] = T(0);
    eta_out[p] = T(0);
  } else {
    const T wv = w_in[p];
    w_out[p] = wv;
    eta_out[p] = (wv - kinematic(d, c, W, i, j, k)) / ld(c.dzw, p);
  }
}


// flux * q_face of the 3rd-order upwind-biased face value (steppers.py:1312-1360)
template <typename T>
__device__ __forceinline__ T upwind_flux(T qm2, T qm1, T q0, T qp1, T F, T eps_l) {
  const T q4 = T(7.0 / 12.0) * (q0 + qm1) - T(1.0 / 12.0) * (qp1 + qm2);
  const T qb = T(1.0 / 12.0) * ((qp1 - qm2) - T(3) * (q0 - qm1));
  const T cf = (fabs(F) < eps_l) ? T(0) : F;
  const T sg = (cf > T(0)) ? T(1) : ((cf < T(0)) ? T(-1) : T(0));
  return F * (q4 + sg * qb);
}

// the four advected fields at mass point (i, j, k): th', u_m, v_m, w_m
template <typename T>
struct AdvFields {
  const Dims& d;
  const T* __restrict__ u;
  const T* __restrict__ v;
  const T* __restrict__ w;
  const T* __restrict__ th;
  __device__ __forceinline__ T at(int f, int i, int j, int k) const {
    switch (f) {
      case 0: return ld(th, im(d, i, j, k));
      case 1: return T(0.5) * (ld(u, iu(d, i, j, k)) + ld(u, iu(d, i + 1, j, k)));
      case 2: return T(0.5) * (ld(v, iv(d, i, j, k)) + ld(v, iv(d, i, j + 1, k)));
      default: return T(0.5) * (ld(w, iw(d, i, j, k)) + ld(w, iw(d, i, j, k + 1)));
    }
  }
};

// Blocks of AX x AY mass points of one level.  For each of the four fields
// the block forms the field's values at the (AX + 4) x (AY + 4) cells of its
// x and y stencils once into shared memory (indices wrapped or clamped as
// the point form wraps them), instead of five times per point and axis; the
// z stencil is read per point.
constexpr int AX = 32, AY = 8;

template <typename T>
__global__ void __launch_bounds__(AX * AY) split_adv_kernel(Dims d, Coef<T> c, const T* __restrict__ u,
                                                            const T* __restrict__ v, const T* __restrict__ w,
                                                            const T* __restrict__ eta, const T* __restrict__ th,
                                                            T eps_l, PtrTable<T> out) {
  __shared__ T Qt[AY + 4][AX + 4];
  const int i0 = blockIdx.x * AX, j0 = blockIdx.y * AY, k = blockIdx.z;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = i0 + tx, j = j0 + ty;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  const bool live = i < nx && j < ny;
  const AdvFields<T> F{d, u, v, w, th};
  const T dx = (T)d.dx, dy = (T)d.dy;
  T mm = T(0), U0 = T(0), U1 = T(0), V0 = T(0), V1 = T(0), W0 = T(0), W1 = T(0), zfac = T(0);
  T dU = T(0), dV = T(0), dW = T(0);
  int zk[5];
  if (live) {
    mm = ld(c.mm, h_m(d, i, j));
    // U = u / m_u, V = v / m_v, W = eta dz_w at the cell's faces (steppers.py:1397-1399)
    U0 = ld(u, iu(d, i, j, k)) / ld(c.mu, h_u(d, i, j));
    U1 = ld(u, iu(d, i + 1, j, k)) / ld(c.mu, h_u(d, i + 1, j));
    V0 = ld(v, iv(d, i, j, k)) / ld(c.mv, h_v(d, i, j));
    V1 = ld(v, iv(d, i, j + 1, k)) / ld(c.mv, h_v(d, i, j + 1));
    W0 = ld(eta, iw(d, i, j, k)) * ld(c.dzw, iw(d, i, j, k));
    W1 = ld(eta, iw(d, i, j, k + 1)) * ld(c.dzw, iw(d, i, j, k + 1));
    const T dzm = ld(c.dzm, im(d, i, j, k));
    zfac = (T)d.dz / dzm;
    dU = (U1 - U0) / dx * mm;
    dV = (V1 - V0) / dy * mm;
    dW = (W1 - W0) / (T)d.dz * zfac;
  }
#pragma unroll
  for (int o = 0; o < 5; ++o) zk[o] = min(max(k - 2 + o, 0), nz - 1);
  const int t = tx + AX * ty;
#pragma unroll 1
  for (int f = 0; f < 4; ++f) {
    for (int q = t; q < (AX + 4) * (AY + 4); q += AX * AY) {
      const int x = q % (AX + 4), y = q / (AX + 4);
      Qt[y][x] = F.at(f, wrap_or_clamp(i0 - 2 + x, nx, d.px), wrap_or_clamp(j0 - 2 + y, ny, d.py), k);
    }
    __syncthreads();
    if (live) {
      T qx[5], qy[5], qz[5];
#pragma unroll
      for (int o = 0; o < 5; ++o) {
        qx[o] = Qt[ty + 2][tx + o];
        qy[o] = Qt[ty + o][tx + 2];
        qz[o] = (o == 2) ? Qt[ty + 2][tx + 2] : F.at(f, i, j, zk[o]);
      }
      const T q = qx[2];
      // faces i (q at i-2..i+1) and i+1 (q at i-1..i+2)
      const T ax = (upwind_flux(qx[1], qx[2], qx[3], qx[4], U1, eps_l) -
                    upwind_flux(qx[0], qx[1], qx[2], qx[3], U0, eps_l)) / dx * mm;
      const T ay = (upwind_flux(qy[1], qy[2], qy[3], qy[4], V1, eps_l) -
                    upwind_flux(qy[0], qy[1], qy[2], qy[3], V0, eps_l)) / dy * mm;
      const T az = (upwind_flux(qz[1], qz[2], qz[3], qz[4], W1, eps_l) -
                    upwind_flux(qz[0], qz[1], qz[2], qz[3], W0, eps_l)) / (T)d.dz * zfac;
      out.p[f][im(d, i, j, k)] = -(mm * mm) * (ax - q * dU + ay - q * dV) - (az - q * dW);
    }
    __syncthreads();  // the next field refills the tile
  }
}

// slow forcings: tend6 = {tend_u, tend_v, tend_w, tend_pi, tend_th, nl_pi};
// adv4 at mass points averaged to the u faces, v faces and w levels
template <typename T>
__global__ void split_slow_kernel(Dims d, PtrTable<T> t, PtrTable<T> sf) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i > nx || j > ny || k > nz) return;
  // t.p[0..5]: explicit tendencies; t.p[6..9]: advection of th', u_m, v_m, w_m
  if (j < ny && k < nz) {
    int l, r;
    face_pair(i, nx, d.px, l, r);
    const int p = iu(d, i, j, k);
    sf.p[0][p] = t.p[0][p] + T(0.5) * (t.p[7][im(d, l, j, k)] + t.p[7][im(d, r, j, k)]);
  }
  if (i < nx && k < nz) {
    int l, r;
    face_pair(j, ny, d.py, l, r);
    const int p = iv(d, i, j, k);
    sf.p[1][p] = t.p[1][p] + T(0.5) * (t.p[8][im(d, i, l, k)] + t.p[8][im(d, i, r, k)]);
  }
  if (i < nx && j < ny) {
    int l, r;
    level_pair(k, nz, l, r);
    const int p = iw(d, i, j, k);
    sf.p[2][p] = t.p[2][p] + T(0.5) * (t.p[9][im(d, i, j, l)] + t.p[9][im(d, i, j, r)]);
    if (k < nz) {
      const int q = im(d, i, j, k);
      sf.p[3][q] = t.p[3][q] + t.p[5][q];
      sf.p[4][q] = t.p[4][q] + t.p[6][q];
    }
  }
}

template <typename T>
__global__ void split_init_kernel(Dims d, SplitArgs<T> a) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i > nx || j > ny || k > nz) return;
  if (j < ny && k < nz) {
    const int p = iu(d, i, j, k);
    a.upp[p] = a.u0[p] - a.uc[p];
  }
  if (i < nx && k < nz) {
    const int p = iv(d, i, j, k);
    a.vpp[p] = a.v0[p] - a.vc[p];
  }
  if (i < nx && j < ny) {
    const int p = iw(d, i, j, k);
    a.wpp[p] = a.w0[p] - a.wc[p];
    if (k < nz) a.ppp[p] = a.p0[p] - a.pc[p];
  }
}

// horizontal divergence of the total winds (stage + u'') at a cell
template <typename T>
__device__ __forceinline__ T cell_div(const Dims& d, const Coef<T>& c, const T* uc, const T* up, const T* vc,
                                      const T* vp, int i, int j, int k) {
  const T mm = ld(c.mm, h_m(d, i, j));
  const int u0 = iu(d, i, j, k), v0 = iv(d, i, j, k);
  const T du = ((uc[u0 + 1] + up[u0 + 1]) - (uc[u0] + up[u0])) / (T)d.dx * mm;
  const T dv = ((vc[v0 + d.nx] + vp[v0 + d.nx]) - (vc[v0] + vp[v0])) / (T)d.dy * mm;
  return du + dv;
}

// Blocks of the predictor and corrector: SX x SY faces of one level.
constexpr int SX = 32, SY = 8;

// The horizontal divergence of the total winds (stage + perturbation) of the
// cells (i0 - 1 + x, j0 - 1 + y), x <= SX, y <= SY, at level k, into Dt.
// Cell indices beyond the grid wrap on a periodic axis and are clamped on an
// open one, so every interior face (i, j) of the block finds the two cells
// of its divergence-damping gradient at tile columns i - i0, i - i0 + 1
// (rows j - j0, j - j0 + 1), as face_pair gives them, and the periodic
// duplicate face n its wrapped pair; the open boundary faces take no
// gradient (the divergence-damping gradient, steppers.py:1528-1538).  One cell divergence per cell of the tile instead of two per
// face and axis.
template <typename T>
__device__ __forceinline__ void div_tile(const Dims& d, const Coef<T>& c, const T* uc, const T* up, const T* vc,
                                         const T* vp, int i0, int j0, int k, T (*Dt)[SX + 1]) {
  const int t = threadIdx.x + SX * threadIdx.y;
  for (int q = t; q < (SX + 1) * (SY + 1); q += SX * SY) {
    const int x = q % (SX + 1), y = q / (SX + 1);
    const int ci = wrap_or_clamp(i0 - 1 + x, d.nx, d.px), cj = wrap_or_clamp(j0 - 1 + y, d.ny, d.py);
    Dt[y][x] = cell_div(d, c, uc, up, vc, vp, ci, cj, k);
  }
}

// PART 1 of the acoustic sub-step (steppers.py:1561-1579): u'' and v'' to
// the midpoint; the boundary faces take the step-start winds (open) or the
// first face (periodic duplicate).  The pressure gradient of the old pi''
// is formed here on the first sub-step of a stage and taken from the
// previous corrector (gx0_ready) on the others.
template <typename T>
__global__ void __launch_bounds__(SX * SY) split_predict_kernel(Dims d, Coef<T> c, SplitArgs<T> a) {
  __shared__ T Dt[SY + 1][SX + 1];
  const int i0 = blockIdx.x * SX, j0 = blockIdx.y * SY, k = blockIdx.z;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = i0 + tx, j = j0 + ty;
  const int nx = d.nx, ny = d.ny;
  div_tile<T>(d, c, a.uc, a.upp, a.vc, a.vpp, i0, j0, k, Dt);
  __syncthreads();
  if (i > nx || j > ny) return;
  const T cp = (T)c.s.cp, hdt = T(0.5) * a.dtau;
  const Grad<T> G{d, c, a.ppp};
  if (j < ny) {
    const int p = iu(d, i, j, k);
    const int ie = (d.px && i == nx) ? 0 : i, pe = iu(d, ie, j, k);
    T val;
    if (!d.px && (i == 0 || i == nx)) {
      val = a.u0[p] - a.uc[p];
    } else {
      T g0;
      if (a.gx0_ready) {
        g0 = a.gx0[p];
      } else {
        g0 = G.gx(ie, j, k);
        a.gx0[p] = g0;
      }
      const T dgx = (Dt[ty + 1][tx + 1] - Dt[ty + 1][tx]) / (T)d.dx * ld(c.mu, h_u(d, ie, j));
      const T rhs = a.sfu[pe] - cp * ld(c.thu, pe) * g0 + a.nu_div * dgx;
      val = a.upp[pe] + hdt * rhs;
    }
    a.uh[p] = val;
  }
  if (i < nx) {
    const int p = iv(d, i, j, k);
    const int je = (d.py && j == ny) ? 0 : j, pe = iv(d, i, je, k);
    T val;
    if (!d.py && (j == 0 || j == ny)) {
      val = a.v0[p] - a.vc[p];
    } else {
      T g0;
      if (a.gx0_ready) {
        g0 = a.gy0[p];
      } else {
        g0 = G.gy(i, je, k);
        a.gy0[p] = g0;
      }
      const T dgy = (Dt[ty + 1][tx + 1] - Dt[ty][tx + 1]) / (T)d.dy * ld(c.mv, h_v(d, i, je));
      const T rhs = a.sfv[pe] - cp * ld(c.thv, pe) * g0 + a.nu_div * dgy;
      val = a.vpp[pe] + hdt * rhs;
    }
    a.vh[p] = val;
  }
}

// PART 2 (steppers.py:1584-1605, 1635-1737): the vertically implicit
// acoustic column.  Upward: the explicit w'' (kept in place for the
// correction), the off-centred eta_dot flux, the explicit pi'' increment
// and the forward sweep of the tridiagonal solve for delta pi; downward:
// the back substitution, pi'' += delta pi and the w'' correction by the
// gradient of delta pi.  One thread per column; cpr/dpr hold the sweep.
template <typename T>
__global__ void __launch_bounds__(128) split_column_kernel(Dims d, Coef<T> c, SplitArgs<T> a, T a2cp, T adcp) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i >= nx || j >= ny) return;
  const T al = a.alpha, dtau = a.dtau, cp = (T)c.s.cp;
  const Winds<T> W{d, c, a.uh, a.vh};
  const Grad<T> G{d, c, a.ppp};
  const T mm = ld(c.mm, h_m(d, i, j));
  const T dx = (T)d.dx, dy = (T)d.dy;
  const T wsfc = kinematic(d, c, W, i, j, 0);
  T fz_lo = T(0), gam_lo = T(0), cprev = T(0), dprev = T(0);
#pragma unroll 4
  for (int k = 0; k < nz; ++k) {
    T fz_hi = T(0), gam_hi = T(0);
    if (k + 1 < nz) {
      const int pw = iw(d, i, j, k + 1);
      const T thw = ld(c.thw, pw), rw = ld(c.rhow, pw);
      const T wold = a.wpp[pw];
      const T wex = wold + dtau * (a.sfw[pw] - cp * thw * G.gzw(i, j, k + 1));
      const T wav = (T(1) - al) * wold + al * wex;
      fz_hi = (wav - kinematic(d, c, W, i, j, k + 1)) * rw * thw;
      gam_hi = a2cp * thw * rw * thw / ld(c.dzw, pw);
      a.wpp[pw] = wex;
    }
    const int p = im(d, i, j, k);
    const T dzm = ld(c.dzm, p), cpidz = ld(c.cpidz, p);
    const int u0 = iu(d, i, j, k), v0 = iv(d, i, j, k);
    const T fx0 = a.uh[u0] * ld(c.rdu, u0) * ld(c.thu, u0);
    const T fx1 = a.uh[u0 + 1] * ld(c.rdu, u0 + 1) * ld(c.thu, u0 + 1);
    const T fy0 = a.vh[v0] * ld(c.rdv, v0) * ld(c.thv, v0);
    const T fy1 = a.vh[v0 + nx] * ld(c.rdv, v0 + nx) * ld(c.thv, v0 + nx);
    const T div_h = mm * ((fx1 - fx0) / dx * mm / dzm + (fy1 - fy0) / dy * mm / dzm);
    const T div_z = (fz_hi - fz_lo) / dzm;
    const T rhs = dtau * (a.sfp[p] - cpidz * dzm * (div_h + div_z));
    const T lower = -cpidz * gam_lo, upper = -cpidz * gam_hi;
    const T mainv = T(1) - lower - upper;
    T cpk, dpk;
    if (k == 0) {
      const T inv = T(1) / mainv;
      cpk = upper * inv;
      dpk = rhs * inv;
    } else {
      const T inv = T(1) / (mainv - lower * cprev);
      cpk = upper * inv;
      dpk = (rhs - lower * dprev) * inv;
    }
    a.cpr[p] = cpk;
    a.dpr[p] = dpk;
    cprev = cpk;
    dprev = dpk;
    fz_lo = fz_hi;
    gam_lo = gam_hi;
  }
  T xh = dprev;
  {
    const int p = im(d, i, j, nz - 1);
    a.ppp[p] = a.ppp[p] + xh;
  }
#pragma unroll 4
  for (int k = nz - 2; k >= 0; --k) {
    const int p = im(d, i, j, k);
    const T x = a.dpr[p] - a.cpr[p] * xh;
    const int pw = iw(d, i, j, k + 1);
    a.wpp[pw] = a.wpp[pw] - adcp * ld(c.thw, pw) * ((xh - x) * ld(c.idzw, pw));
    a.ppp[p] = a.ppp[p] + x;
    xh = x;
  }
  a.wpp[iw(d, i, j, 0)] = wsfc;
  a.wpp[iw(d, i, j, nz)] = T(0);
}

// The same column solve on tiles of PC columns (one block per tile and
// row j) so that every thread works outside the recurrence: A1 the w-level
// terms (explicit w'', the eta_dot flux, the coupling gamma) and A2 the
// right-hand sides at every (level, column) pair, B one warp runs the
// Thomas sweeps in shared memory, forming each row (lower, upper, main)
// from gamma and C_pi / dz_m, C the pi'' and w'' updates.  Arithmetic is
// term for term that of split_column_kernel.  Shared memory: (4 nz + 2) PC
// values (c' overwrites the eta_dot fluxes once the right-hand sides are
// formed).
template <typename T, int PT, int PC>
__global__ void __launch_bounds__(PT) split_column_tile_kernel(Dims d, Coef<T> c, SplitArgs<T> a, T a2cp,
                                                               T adcp) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sm = reinterpret_cast<T*>(smem_raw);
  const int nx = d.nx, nz = d.nz;
  T* s_fz = sm;                      // [nz+1][PC]  eta_dot flux -> c'
  T* s_gam = s_fz + (nz + 1) * PC;   // [nz+1][PC]  gamma
  T* s_x = s_gam + (nz + 1) * PC;    // [nz][PC]    rhs -> d' -> delta pi
  T* s_cz = s_x + nz * PC;           // [nz][PC]    C_pi / dz_m
  const int i0 = blockIdx.x * PC, j = blockIdx.y, tid = threadIdx.x;
  const T al = a.alpha, dtau = a.dtau, cp = (T)c.s.cp;
  const T dx = (T)d.dx, dy = (T)d.dy;
  const Winds<T> W{d, c, a.uh, a.vh};
  const Grad<T> G{d, c, a.ppp};
  for (int q = tid; q < (nz + 1) * PC; q += PT) {  // A1
    const int k = q / PC, i = i0 + q % PC;
    T fz = T(0), gam = T(0);
    if (i < nx && k > 0 && k < nz) {
      const int pw = iw(d, i, j, k);
      const T thw = ld(c.thw, pw), rw = ld(c.rhow, pw);
      const T wold = a.wpp[pw];
      const T wex = wold + dtau * (a.sfw[pw] - cp * thw * G.gzw(i, j, k));
      const T wav = (T(1) - al) * wold + al * wex;
      fz = (wav - kinematic(d, c, W, i, j, k)) * rw * thw;
      gam = a2cp * thw * rw * thw / ld(c.dzw, pw);
      a.wpp[pw] = wex;
    }
    s_fz[q] = fz;
    s_gam[q] = gam;
  }
  __syncthreads();
  for (int q = tid; q < nz * PC; q += PT) {  // A2
    const int k = q / PC, i = i0 + q % PC;
    if (i >= nx) {  // a trivial row: lower = upper = 0, main = 1
      s_x[q] = T(0);
      s_cz[q] = T(0);
      continue;
    }
    const int p = im(d, i, j, k);
    const T mm = ld(c.mm, h_m(d, i, j));
    const T dzm = ld(c.dzm, p), cpidz = ld(c.cpidz, p);
    const int u0 = iu(d, i, j, k), v0 = iv(d, i, j, k);
    const T fx0 = a.uh[u0] * ld(c.rdu, u0) * ld(c.thu, u0);
    const T fx1 = a.uh[u0 + 1] * ld(c.rdu, u0 + 1) * ld(c.thu, u0 + 1);
    const T fy0 = a.vh[v0] * ld(c.rdv, v0) * ld(c.thv, v0);
    const T fy1 = a.vh[v0 + nx] * ld(c.rdv, v0 + nx) * ld(c.thv, v0 + nx);
    const T div_h = mm * ((fx1 - fx0) / dx * mm / dzm + (fy1 - fy0) / dy * mm / dzm);
    const T div_z = (s_fz[q + PC] - s_fz[q]) / dzm;
    s_x[q] = dtau * (a.sfp[p] - cpidz * dzm * (div_h + div_z));
    s_cz[q] = cpidz;
  }
  __syncthreads();
  if (tid < PC) {  // B
    T cprev = T(0), dprev = T(0);
    for (int k = 0; k < nz; ++k) {
      const int q = k * PC + tid;
      const T cpidz = s_cz[q];
      const T lower = -cpidz * s_gam[q], upper = -cpidz * s_gam[q + PC];
      const T mainv = T(1) - lower - upper;
      T cpk, dpk;
      if (k == 0) {
        const T inv = T(1) / mainv;
        cpk = upper * inv;
        dpk = s_x[q] * inv;
      } else {
        const T inv = T(1) / (mainv - lower * cprev);
        cpk = upper * inv;
        dpk = (s_x[q] - lower * dprev) * inv;
      }
      s_fz[q] = cpk;
      s_x[q] = dpk;
      cprev = cpk;
      dprev = dpk;
    }
    T xh = dprev;
    for (int k = nz - 2; k >= 0; --k) {
      const int q = k * PC + tid;
      xh = s_x[q] - s_fz[q] * xh;
      s_x[q] = xh;
    }
  }
  __syncthreads();
  for (int q = tid; q < (nz + 1) * PC; q += PT) {  // C
    const int k = q / PC, i = i0 + q % PC;
    if (i >= nx) continue;
    const int pw = iw(d, i, j, k);
    if (k == 0) {
      a.wpp[pw] = kinematic(d, c, W, i, j, 0);
    } else if (k == nz) {
      a.wpp[pw] = T(0);
    } else {
      a.wpp[pw] = a.wpp[pw] - adcp * ld(c.thw, pw) * ((s_x[q] - s_x[q - PC]) * ld(c.idzw, pw));
    }
    if (k < nz) a.ppp[pw] = a.ppp[pw] + s_x[q];
  }
}

// PART 3 (steppers.py:1607-1626): the centred corrector of u'', v'' into
// upp2/vpp2 (read u'' from upp/vpp), and the backward damping of w''.  The
// gradients of the new pi'' go to gx1/gy1 for the next predictor.
template <typename T>
__global__ void __launch_bounds__(SX * SY) split_correct_kernel(Dims d, Coef<T> c, SplitArgs<T> a,
                                                                T* __restrict__ upp2, T* __restrict__ vpp2) {
  __shared__ T Dt[SY + 1][SX + 1];
  const int i0 = blockIdx.x * SX, j0 = blockIdx.y * SY, k = blockIdx.z;
  const int tx = threadIdx.x, ty = threadIdx.y;
  const int i = i0 + tx, j = j0 + ty;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (k < nz) div_tile<T>(d, c, a.uc, a.uh, a.vc, a.vh, i0, j0, k, Dt);
  __syncthreads();
  if (i > nx || j > ny) return;
  const T cp = (T)c.s.cp, dtau = a.dtau;
  const Grad<T> G{d, c, a.ppp};
  if (j < ny && k < nz) {
    const int p = iu(d, i, j, k);
    T val;
    if (!d.px && (i == 0 || i == nx)) {
      val = a.u0[p] - a.uc[p];
    } else {
      const int ie = (d.px && i == nx) ? 0 : i, pe = iu(d, ie, j, k);
      const T g1 = G.gx(ie, j, k);
      if (a.gx1) a.gx1[p] = g1;
      const T dgx = (Dt[ty + 1][tx + 1] - Dt[ty + 1][tx]) / (T)d.dx * ld(c.mu, h_u(d, ie, j));
      val = a.upp[pe] + dtau * (a.sfu[pe] - T(0.5) * cp * ld(c.thu, pe) * (a.gx0[pe] + g1) + a.nu_div * dgx);
    }
    upp2[p] = val;
  }
  if (i < nx && k < nz) {
    const int p = iv(d, i, j, k);
    T val;
    if (!d.py && (j == 0 || j == ny)) {
      val = a.v0[p] - a.vc[p];
    } else {
      const int je = (d.py && j == ny) ? 0 : j, pe = iv(d, i, je, k);
      const T g1 = G.gy(i, je, k);
      if (a.gy1) a.gy1[p] = g1;
      const T dgy = (Dt[ty + 1][tx + 1] - Dt[ty][tx + 1]) / (T)d.dy * ld(c.mv, h_v(d, i, je));
      val = a.vpp[pe] + dtau * (a.sfv[pe] - T(0.5) * cp * ld(c.thv, pe) * (a.gy0[pe] + g1) + a.nu_div * dgy);
    }
    vpp2[p] = val;
  }
  if (i < nx && j < ny) {
    const int p = iw(d, i, j, k);
    const T wc = a.wc[p];
    a.wpp[p] = (wc + a.wpp[p]) / (T(1) + dtau * ld(a.tau, p)) - wc;
  }
}

template <typename T>
__global__ void split_end_kernel(Dims d, SplitArgs<T> a, T dtns, T* u, T* v, T* w, T* eta, T* pp, T* th) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i > nx || j > ny || k > nz) return;
  if (j < ny && k < nz) {
    const int p = iu(d, i, j, k);
    u[p] = a.uc[p] + a.upp[p];
  }
  if (i < nx && k < nz) {
    const int p = iv(d, i, j, k);
    v[p] = a.vc[p] + a.vpp[p];
  }
  if (i < nx && j < ny) {
    const int p = iw(d, i, j, k);
    w[p] = a.wc[p] + a.wpp[p];
    eta[p] = a.ec[p];
    if (k < nz) {
      pp[p] = a.pc[p] + a.ppp[p];
      th[p] = a.th0[p] + dtns * a.sfth[p];
    }
  }
}

template <typename T>
__global__ void split_axpy_kernel(size_t n, const T* __restrict__ b, T* a) {
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x)
    a[q] = a[q] + b[q];
}

}  // namespace

template <typename T>
void launch_split_diag(const Dims& d, const Coef<T>& c, const T* u, const T* v, const T* w_in, T* eta_out,
                       T* w_out, cudaStream_t st) {
  const dim3 blk(32, 4, 2);
  split_diag_kernel<T><<<box(d.nx, d.ny, d.nz + 1, blk), blk, 0, st>>>(d, c, u, v, w_in, eta_out, w_out);
}

template <typename T>
void launch_split_adv(const Dims& d, const Coef<T>& c, const T* u, const T* v, const T* w, const T* eta,
                      const T* th, T eps_l, T* const* adv4, cudaStream_t st) {
  const dim3 blk(AX, AY, 1);
  PtrTable<T> o{};
  for (int q = 0; q < 4; ++q) o.p[q] = adv4[q];
  split_adv_kernel<T><<<box(d.nx, d.ny, d.nz, blk), blk, 0, st>>>(d, c, u, v, w, eta, th, eps_l, o);
}

template <typename T>
void launch_split_slow(const Dims& d, const T* const* tend6, const T* const* adv4, T* const* sf5, cudaStream_t st) {
  const dim3 blk(32, 4, 2);
  PtrTable<T> t{}, s{};
  for (int q = 0; q < 6; ++q) t.p[q] = const_cast<T*>(tend6[q]);
  for (int q = 0; q < 4; ++q) t.p[6 + q] = const_cast<T*>(adv4[q]);
  for (int q = 0; q < 5; ++q) s.p[q] = sf5[q];
  split_slow_kernel<T><<<box(d.nx + 1, d.ny + 1, d.nz + 1, blk), blk, 0, st>>>(d, t, s);
}

template <typename T>
void launch_split_init(const Dims& d, const SplitArgs<T>& a, cudaStream_t st) {
  const dim3 blk(32, 4, 2);
  split_init_kernel<T><<<box(d.nx + 1, d.ny + 1, d.nz + 1, blk), blk, 0, st>>>(d, a);
}

template <typename T>
void launch_split_predict(const Dims& d, const Coef<T>& c, const SplitArgs<T>& a, cudaStream_t st) {
  const dim3 blk(SX, SY, 1);
  split_predict_kernel<T><<<box(d.nx + 1, d.ny + 1, d.nz, blk), blk, 0, st>>>(d, c, a);
}

template <typename T>
void launch_split_column(const Dims& d, const Coef<T>& c, const SplitArgs<T>& a, cudaStream_t st) {
  const double ad = (double)a.alpha * (double)a.dtau;
  const T a2cp = (T)(ad * ad * c.s.cp), adcp = (T)(ad * c.s.cp);
  constexpr int PT = 256, PC = 32;
  const size_t smem = (size_t)(4 * d.nz + 2) * PC * sizeof(T);
  if (smem <= 200 * 1024) {  // tiles of 32 columns; the one-thread-per-column march beyond
    static SmemLimit attr_bytes;  // per instantiation
    ensure_smem_limit((const void*)split_column_tile_kernel<T, PT, PC>, attr_bytes, smem);
    split_column_tile_kernel<T, PT, PC><<<dim3((d.nx + PC - 1) / PC, d.ny), PT, smem, st>>>(d, c, a, a2cp, adcp);
    return;
  }
  split_column_kernel<T><<<dim3((d.nx + 127) / 128, d.ny), 128, 0, st>>>(d, c, a, a2cp, adcp);
}

template <typename T>
void launch_split_correct(const Dims& d, const Coef<T>& c, const SplitArgs<T>& a, T* upp2, T* vpp2,
                          cudaStream_t st) {
  const dim3 blk(SX, SY, 1);
  split_correct_kernel<T><<<box(d.nx + 1, d.ny + 1, d.nz + 1, blk), blk, 0, st>>>(d, c, a, upp2, vpp2);
}

template <typename T>
void launch_split_end(const Dims& d, const SplitArgs<T>& a, int nsteps, T* u, T* v, T* w, T* eta, T* p, T* th,
                      cudaStream_t st) {
  const dim3 blk(32, 4, 2);
  const T dtns = (T)((double)a.dtau * nsteps);
  split_end_kernel<T><<<box(d.nx + 1, d.ny + 1, d.nz + 1, blk), blk, 0, st>>>(d, a, dtns, u, v, w, eta, p, th);
}

template <typename T>
void launch_split_axpy(size_t n, const T* b, T* a, cudaStream_t st) {
  split_axpy_kernel<T><<<(unsigned)std::min<size_t>((n + 255) / 256, 148 * 16), 256, 0, st>>>(n, b, a);
}

#define SISL_INST_SPLIT(T)                                                                                       \
  template void launch_split_diag<T>(const Dims&, const Coef<T>&, const T*, const T*, const T*, T*, T*,        \
                                     cudaStream_t);                                                           \
  template void launch_split_adv<T>(const Dims&, const Coef<T>&, const T*, const T*, const T*, const T*,       \
                                    const T*, T, T* const*, cudaStream_t);                                    \
  template void launch_split_slow<T>(const Dims&, const T* const*, const T* const*, T* const*, cudaStream_t); \
  template void launch_split_init<T>(const Dims&, const SplitArgs<T>&, cudaStream_t);                         \
  template void launch_split_predict<T>(const Dims&, const Coef<T>&, const SplitArgs<T>&, cudaStream_t);      \
  template void launch_split_column<T>(const Dims&, const Coef<T>&, const SplitArgs<T>&, cudaStream_t);       \
  template void launch_split_correct<T>(const Dims&, const Coef<T>&, const SplitArgs<T>&, T*, T*,             \
                                        cudaStream_t);                                                        \
  template void launch_split_end<T>(const Dims&, const SplitArgs<T>&, int, T*, T*, T*, T*, T*, T*,            \
                                    cudaStream_t);                                                            \
  template void launch_split_axpy<T>(size_t, const T*, T*, cudaStream_t);
SISL_INST_SPLIT(float)
SISL_INST_SPLIT(double)

}  // namespace sisl
