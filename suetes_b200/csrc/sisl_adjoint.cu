// Transposed Helmholtz matvec A^T and transposed preconditioner M^T on the
// scaled solver vector, in gather form (no atomics, deterministic).
//
// The reference differentiates SemiImplicitSolver3D.solve through
// jax.lax.custom_linear_solve (steppers.py:483-485): the cotangent solve is
// gmres(A^T, g, M=M^T) (steppers.py:473-481) where A^T is the exact transpose
// of A_fn traced without the edge-padding stop_gradient (steppers.py:463) and
// M^T = jax.linear_transpose(M_fn).  Both transposes are written out here from
// the forward rows of sisl_linear.cu:
//
//  u face (interior or periodic face 0; the periodic face n row copies face 0)
//    L_u = u - adt [ -cp thu ((P_r - P_l) m_u/dx - zxu (gzm_l + gzm_r)/2)
//                   + f_u (v_l,j + v_l,j+1 + v_r,j + v_r,j+1)/4 ]
//  v face analogous with -f_v * (u ...)/4
//  w level (interior)   L_w = damp w + adt cp thw gzw
//  eta row (interior)   L_e = a (W + m (uw zxw + vw zew) - w)
//  boundary rows        L_u = u, L_v = v, L_w = w, L_e = W / dz_w
//  pi row               L_p = p + adt ps cpidz (m^2 (dFx/dx + dFy/dy) + dFz)
//  with P = p / ps, gzw(k) = (P(kr) - P(kl)) / dz_w(k) on the padded level
//  pair, gzm(k) = (gzw(k) + gzw(k+1)) / 2, Fx = u rdu thu, Fz = W rhow thw.
#include "sisl_group.cuh"

namespace sisl {
namespace {

dim3 box_grid(int ex, int ey, int ez, dim3 blk) {
  return dim3((ex + blk.x - 1) / blk.x, (ey + blk.y - 1) / blk.y, (ez + blk.z - 1) / blk.z);
}

// Is u face f computed (not locked, not the periodic duplicate)?
__device__ __forceinline__ bool face_live(int f, int n, int periodic) {
  return periodic ? (f < n) : (f > 0 && f < n);
}

// cotangent of the u row at face f as seen by its computation (the periodic
// face n row is a copy of face 0)
template <typename T>
__device__ __forceinline__ T ybar_u(const Dims& d, const T* __restrict__ yu, T ys, int f, int j, int k) {
  T y = ld(yu, iu(d, f, j, k)) * ys;
  if (d.px && f == 0) y += ld(yu, iu(d, d.nx, j, k)) * ys;
  return y;
}
template <typename T>
__device__ __forceinline__ T ybar_v(const Dims& d, const T* __restrict__ yv, T ys, int i, int f, int k) {
  T y = ld(yv, iv(d, i, f, k)) * ys;
  if (d.py && f == 0) y += ld(yv, iv(d, i, d.ny, k)) * ys;
  return y;
}

// Stage 1: gbar_zm(i, j, k) = sum over the live faces whose gradient reads
// column (i, j) at mass level k of -adt cp th zx / 2 * ybar.
template <typename T>
__device__ __forceinline__ void at_gzm_block(const Dims& d, const Coef<T>& c, const T* __restrict__ yu, const T* __restrict__ yv, const double* yscale, T* __restrict__ gzm, int bx, int by, int bz) {
  const int i = bx * blockDim.x + threadIdx.x;
  const int j = by * blockDim.y + threadIdx.y;
  const int k = bz * blockDim.z + threadIdx.z;
  const int nx = d.nx, ny = d.ny;
  if (i >= nx || j >= ny || k >= d.nz) return;
  const T ys = yscale ? (T)(*yscale) : T(1);
  const T coef = -(T)(c.s.alpha * c.s.dt * c.s.cp) * T(0.5);
  T g = T(0);
  // u faces: column i is the right column of face i and the left column of face i+1
  // (periodic: the left column of face 0 is nx-1)
  if (face_live(i, nx, d.px)) {
    const int p = iu(d, i, j, k);
    g += coef * ld(c.thu, p) * ld(c.zxu, p) * ybar_u(d, yu, ys, i, j, k);
  }
  {
    const int f = (i + 1 < nx) ? i + 1 : (d.px ? 0 : -1);
    if (f >= 0 && face_live(f, nx, d.px)) {
      const int p = iu(d, f, j, k);
      g += coef * ld(c.thu, p) * ld(c.zxu, p) * ybar_u(d, yu, ys, f, j, k);
    }
  }
  if (face_live(j, ny, d.py)) {
    const int p = iv(d, i, j, k);
    g += coef * ld(c.thv, p) * ld(c.zev, p) * ybar_v(d, yv, ys, i, j, k);
  }
  {
    const int f = (j + 1 < ny) ? j + 1 : (d.py ? 0 : -1);
    if (f >= 0 && face_live(f, ny, d.py)) {
      const int p = iv(d, i, f, k);
      g += coef * ld(c.thv, p) * ld(c.zev, p) * ybar_v(d, yv, ys, i, f, k);
    }
  }
  gzm[im(d, i, j, k)] = g;
}
template <typename T>
__global__ void at_gzm_kernel(Dims d, Coef<T> c, const T* __restrict__ yu, const T* __restrict__ yv, const double* yscale,
                              T* __restrict__ gzm, const int* active) {
  if (active && *active == 0) return;
  at_gzm_block<T>(d, c, yu, yv, yscale, gzm, blockIdx.x, blockIdx.y, blockIdx.z);
}

// Stage 2: every input cotangent at a union-box point.
template <typename T>
__device__ __forceinline__ void at_main_block(const Dims& d, const Coef<T>& c, const CVec5<T>& y, const double* yscale, const T* __restrict__ gzm, const CVec5<T>& b, const Vec5<T>& out, int bx, int by, int bz) {
  const int i = bx * blockDim.x + threadIdx.x;
  const int j = by * blockDim.y + threadIdx.y;
  const int k = bz * blockDim.z + threadIdx.z;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i > nx || j > ny || k > nz) return;
  const T ys = yscale ? (T)(*yscale) : T(1);
  const T adt = (T)(c.s.alpha * c.s.dt), cp = (T)c.s.cp, a = (T)c.s.alpha, ps = (T)c.s.ps;
  const T idx = (T)(1.0 / d.dx), idy = (T)(1.0 / d.dy);
  const T* __restrict__ yu = y.f[0];
  const T* __restrict__ yv = y.f[1];
  const T* __restrict__ yw = y.f[2];
  const T* __restrict__ yp = y.f[3];
  const T* __restrict__ ye = y.f[4];
  // q(cell) = adt ps cpidz ybar_p: the weight of the flux divergence of a cell
  auto qcell = [&](int ci, int cj, int ck) {
    const int p = im(d, ci, cj, ck);
    return adt * ps * ld(c.cpidz, p) * ld(yp, p) * ys;
  };
  // ---------------- xbar_u at face (i, j, k) ----------------
  if (j < ny && k < nz) {
    const int p = iu(d, i, j, k);
    T g = T(0);
    // diagonal: every u row reads its own face; on a periodic axis the row n is a
    // copy of row 0, so face 0 also collects the row-n cotangent and face n none
    if (d.px) {
      if (i < nx) g += ybar_u(d, yu, ys, i, j, k);
    } else {
      g += ld(yu, p) * ys;
    }
    // Coriolis: v face (ii, jj) averages u faces ii, ii+1 (read directly, the
    // periodic duplicate included) on rows jj and jj-1 (wrapped when periodic)
    const T w4 = adt * T(0.25);
    for (int ii = i - 1; ii <= i; ++ii) {
      if (ii < 0 || ii >= nx) continue;
      for (int dj = 0; dj <= 1; ++dj) {
        int jj = j + dj;
        if (d.py && jj == ny) jj = 0;
        if (!face_live(jj, ny, d.py)) continue;
        g += w4 * ld(c.fv, h_v(d, ii, jj)) * ybar_v(d, yv, ys, ii, jj, k);
      }
    }
    // kinematic term of the eta rows of cells i' in {i-1, i} at w levels k, k+1
    for (int di = -1; di <= 0; ++di) {
      const int ii = i + di;
      if (ii < 0 || ii >= nx) continue;
      for (int kk = k; kk <= k + 1; ++kk) {
        if (kk <= 0 || kk >= nz) continue;
        const int pw = iw(d, ii, j, kk);
        g += a * T(0.25) * ld(c.mm, h_m(d, ii, j)) * ld(c.zxw, pw) * ld(ye, pw) * ys;
      }
    }
    // flux of the pi rows: face i is the east face of cell i-1 and the west face of cell i
    {
      const T m_f = ld(c.rdu, p) * ld(c.thu, p) * idx;
      T acc = T(0);
      if (i - 1 >= 0) { const T m = ld(c.mm, h_m(d, i - 1, j)); acc += m * m * qcell(i - 1, j, k); }
      if (i < nx) { const T m = ld(c.mm, h_m(d, i, j)); acc -= m * m * qcell(i, j, k); }
      g += m_f * acc;
    }
    T r = g;
    if (b.f[0]) r = ld(b.f[0], p) - r;
    out.f[0][p] = r;
  }
  // ---------------- xbar_v at face (i, j, k) ----------------
  if (i < nx && k < nz) {
    const int p = iv(d, i, j, k);
    T g = T(0);
    if (d.py) {
      if (j < ny) g += ybar_v(d, yv, ys, i, j, k);
    } else {
      g += ld(yv, p) * ys;
    }
    // Coriolis: u face (ii, jj) averages v faces jj, jj+1 (read directly) on
    // columns ii and ii-1 (wrapped when periodic)
    const T w4 = -adt * T(0.25);
    for (int jj = j - 1; jj <= j; ++jj) {
      if (jj < 0 || jj >= ny) continue;
      for (int di = 0; di <= 1; ++di) {
        int ii = i + di;
        if (d.px && ii == nx) ii = 0;
        if (!face_live(ii, nx, d.px)) continue;
        g += w4 * ld(c.fu, h_u(d, ii, jj)) * ybar_u(d, yu, ys, ii, jj, k);
      }
    }
    for (int dj = -1; dj <= 0; ++dj) {
      const int jj = j + dj;
      if (jj < 0 || jj >= ny) continue;
      for (int kk = k; kk <= k + 1; ++kk) {
        if (kk <= 0 || kk >= nz) continue;
        const int pw = iw(d, i, jj, kk);
        g += a * T(0.25) * ld(c.mm, h_m(d, i, jj)) * ld(c.zew, pw) * ld(ye, pw) * ys;
      }
    }
    {
      const T m_f = ld(c.rdv, p) * ld(c.thv, p) * idy;
      T acc = T(0);
      if (j - 1 >= 0) { const T m = ld(c.mm, h_m(d, i, j - 1)); acc += m * m * qcell(i, j - 1, k); }
      if (j < ny) { const T m = ld(c.mm, h_m(d, i, j)); acc -= m * m * qcell(i, j, k); }
      g += m_f * acc;
    }
    T r = g;
    if (b.f[1]) r = ld(b.f[1], p) - r;
    out.f[1][p] = r;
  }
  if (i >= nx || j >= ny) return;
  // ---------------- xbar_w and xbar_W at w level k ----------------
  {
    const int p = iw(d, i, j, k);
    const bool inner = (k > 0 && k < nz);
    const T ye_k = ld(ye, p) * ys, yw_k = ld(yw, p) * ys;
    T gw = inner ? ld(c.damp, p) * yw_k - a * ye_k : yw_k;
    T gW = inner ? a * ye_k : ld(c.idzw, p) * ye_k;
    if (inner) gW += ld(c.rhow, p) * ld(c.thw, p) * (qcell(i, j, k - 1) - qcell(i, j, k));
    if (b.f[2]) { gw = ld(b.f[2], p) - gw; gW = ld(b.f[4], p) - gW; }
    out.f[2][p] = gw;
    out.f[4][p] = gW;
  }
  if (k >= nz) return;
  // ---------------- xbar_p at mass point (i, j, k) ----------------
  {
    const int p = im(d, i, j, k);
    T gP = T(0);  // cotangent of P = p / ps
    // horizontal gradients: column (i, j) is the right column of face i and the
    // left column of face i+1 (periodic: of face 0 when i = nx-1)
    if (face_live(i, nx, d.px)) {
      const int pu = iu(d, i, j, k);
      gP += adt * cp * ld(c.thu, pu) * ld(c.mu, h_u(d, i, j)) * idx * ybar_u(d, yu, ys, i, j, k);
    }
    {
      const int f = (i + 1 < nx) ? i + 1 : (d.px ? 0 : -1);
      if (f >= 0 && face_live(f, nx, d.px)) {
        const int pu = iu(d, f, j, k);
        gP -= adt * cp * ld(c.thu, pu) * ld(c.mu, h_u(d, f, j)) * idx * ybar_u(d, yu, ys, f, j, k);
      }
    }
    if (face_live(j, ny, d.py)) {
      const int pv = iv(d, i, j, k);
      gP += adt * cp * ld(c.thv, pv) * ld(c.mv, h_v(d, i, j)) * idy * ybar_v(d, yv, ys, i, j, k);
    }
    {
      const int f = (j + 1 < ny) ? j + 1 : (d.py ? 0 : -1);
      if (f >= 0 && face_live(f, ny, d.py)) {
        const int pv = iv(d, i, f, k);
        gP -= adt * cp * ld(c.thv, pv) * ld(c.mv, h_v(d, i, f)) * idy * ybar_v(d, yv, ys, i, f, k);
      }
    }
    // vertical gradient: gbar_zw(kk) idzw(kk) with the padded level pairs
    auto gzwbar = [&](int kk) -> T {  // times idzw
      const int pw = iw(d, i, j, kk);
      T g = T(0);
      if (kk - 1 >= 0) g += T(0.5) * ld(gzm, im(d, i, j, kk - 1));
      if (kk < nz) g += T(0.5) * ld(gzm, im(d, i, j, kk));
      if (kk > 0 && kk < nz) g += adt * cp * ld(c.thw, pw) * ld(yw, pw) * ys;
      return g * ld(c.idzw, pw);
    };
    if (k >= 1) gP += gzwbar(k);
    if (k + 1 <= nz - 1) gP -= gzwbar(k + 1);
    if (k == 1) gP += gzwbar(0);
    if (k == 0) gP -= gzwbar(0);
    if (k == nz - 1) gP += gzwbar(nz);
    if (k == nz - 2) gP -= gzwbar(nz);
    T r = ld(yp, p) * ys + gP / ps;
    if (b.f[3]) r = ld(b.f[3], p) - r;
    out.f[3][p] = r;
  }
}
template <typename T>
__global__ void __launch_bounds__(256) at_main_kernel(Dims d, Coef<T> c, CVec5<T> y, const double* yscale,
                                                      const T* __restrict__ gzm, CVec5<T> b, Vec5<T> out,
                                                      const int* active) {
  if (active && *active == 0) return;
  at_main_block<T>(d, c, y, yscale, gzm, b, out, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ---------------------------------------------------------------------------
// M^T, column part, on tiles of 32 columns (same j) like the forward
// preconditioner.  With ybar the output cotangent (ybar_pi = y_pi * ps on
// the unscaled pressure):
//   G(K)   = -adt cp thw (yw + yW) idzw / damp at interior w levels, else 0
//   pibar  = ybar_pi + G(k) - G(k+1)
//   z      = T^-T pibar   (T: the Helmholtz tridiagonal of the forward)
//   out_pi = z / ps,   divbar = -L_pi z
//   wtbar(K) = divbar(K-1) - divbar(K),  epbar = yW + rho_w thw wtbar
//   out_W  = epbar / alpha,  out_w = (yw + epbar) / damp  (interior levels)
//   out_W  = yW dz_w,        out_w = yw                   (ground and lid)
// With the factorisation T = L U of prep_thomas, T^T z = pibar is
// U^T w = pibar (upward) then L^T z = w (downward), the arithmetic of
// pt_march_kernel term for term (every column variant is bitwise equal).
// A: every thread takes (level, column) pairs and forms pibar and stages
//    the factors; B: one thread per column runs both sweeps in shared
//    memory; C: every thread writes pi, w and eta_dot.
// Shared memory per block: 4 nz * columns values of T.
// ---------------------------------------------------------------------------

// rounded products that the compiler may not fuse into a following add, so
// that the column variants of M^T round identically

template <typename T, int TPT, int TPC>
__global__ void __launch_bounds__(TPT) pt_column_kernel(Dims d, Coef<T> c, CVec5<T> y, Vec5<T> out,
                                                        const int* active) {
  if (active && *active == 0) return;
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sm = reinterpret_cast<T*>(smem_raw);
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  T* s_x = sm;                // [nz][TPC]  pibar -> w -> z
  T* s_cp = s_x + nz * TPC;   // [nz][TPC]  c'
  T* s_lo = s_cp + nz * TPC;  // [nz][TPC]  lower
  T* s_iv = s_lo + nz * TPC;  // [nz][TPC]  1 / pivot
  const int i0 = blockIdx.x * TPC;
  const int j = blockIdx.y;
  const int tid = threadIdx.x;
  const int pm = nx * ny;
  const T ps = (T)c.s.ps, ips = (T)(1.0 / c.s.ps), inva = T(1) / (T)c.s.alpha;
  const T* __restrict__ yw = y.f[2];
  const T* __restrict__ yp = y.f[3];
  const T* __restrict__ yW = y.f[4];
  T* __restrict__ ow = out.f[2];
  T* __restrict__ op = out.f[3];
  T* __restrict__ oW = out.f[4];
  // G(K) = -adt cp thw (yw + yW) idzw / damp at interior w levels
  auto Gw = [&](int i, int K) -> T {
    const int kc = min(max(K, 1), nz - 1);
    const int pw = i + nx * j + kc * pm;
    const T g = -ld(c.pbw, pw) * (ld(yw, pw) + ld(yW, pw));
    return (K > 0 && K < nz) ? g : T(0);
  };
  // ---- A: pibar and the factorisation ----
  for (int q = tid; q < nz * TPC; q += TPT) {
    const int k = q / TPC, l = q % TPC, i = min(i0 + l, nx - 1);
    const int p = i + nx * j + k * pm;
    s_x[q] = ld(yp, p) * ps + Gw(i, k) - Gw(i, k + 1);
    s_cp[q] = ld(c.tcp, p);
    s_lo[q] = ld(c.tlo, p);
    s_iv[q] = ld(c.tinv, p);
  }
  __syncthreads();
  // ---- B: U^T w = pibar upward, L^T z = w downward, one thread per column ----
  if (tid < TPC) {
    const int l = tid;
    T wprev = T(0), cprev = T(0);
    for (int k = 0; k < nz; ++k) {
      const int q = k * TPC + l;
      wprev = s_x[q] - cprev * wprev;
      s_x[q] = wprev;
      cprev = s_cp[q];
    }
    T zh = T(0), loh = T(0);
    for (int k = nz - 1; k >= 0; --k) {
      const int q = k * TPC + l;
      zh = (s_x[q] - loh * zh) * s_iv[q];
      s_x[q] = zh;
      loh = s_lo[q];
    }
  }
  __syncthreads();
  // ---- C: pi, w and eta_dot cotangents ----
  for (int q = tid; q < (nz + 1) * TPC; q += TPT) {
    const int k = q / TPC, l = q % TPC, i = i0 + l;
    if (i >= nx) continue;
    const int p = i + nx * j + k * pm;
    if (k < nz) op[p] = s_x[q] * ips;
    if (k == 0 || k == nz) {
      ow[p] = ld(yw, p);
      oW[p] = ld(yW, p) * ld(c.dzw, p);
    } else {
      const T dvl = mul_rn(-ld(c.lpi, p - pm), s_x[q - TPC]), dv = mul_rn(-ld(c.lpi, p), s_x[q]);
      const T ep = ld(yW, p) + ld(c.rtw, p) * (dvl - dv);
      oW[p] = ep * inva;
      ow[p] = (ld(yw, p) + ep) * ld(c.idamp, p);
    }
  }
}

// The same tile with its global loads batched: every thread issues PU
// items' loads before it computes any of them (the forward tile's
// batching).  Arithmetic is term for term that of pt_column_kernel, so the
// results are bitwise those of every other column variant.
template <typename T, int TPT, int TPC, int PU>
__device__ __forceinline__ void pt_column_batched_block(const Dims& d, const Coef<T>& c, const CVec5<T>& y, const Vec5<T>& out, int bx, int by, int bz) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* sm = reinterpret_cast<T*>(smem_raw);
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  T* s_x = sm;                // [nz][TPC]  pibar -> w -> z
  T* s_cp = s_x + nz * TPC;   // [nz][TPC]  c'
  T* s_lo = s_cp + nz * TPC;  // [nz][TPC]  lower
  T* s_iv = s_lo + nz * TPC;  // [nz][TPC]  1 / pivot
  const int i0 = bx * TPC;
  const int j = by;
  const int tid = threadIdx.x;
  const int pm = nx * ny;
  const int nm = nz * TPC, nw = (nz + 1) * TPC;
  const T ps = (T)c.s.ps, ips = (T)(1.0 / c.s.ps), inva = T(1) / (T)c.s.alpha;
  const T* __restrict__ yw = y.f[2];
  const T* __restrict__ yp = y.f[3];
  const T* __restrict__ yW = y.f[4];
  T* __restrict__ ow = out.f[2];
  T* __restrict__ op = out.f[3];
  T* __restrict__ oW = out.f[4];
  (void)ny;
  // ---- A: pibar and the factorisation ----
  for (int q0 = tid; q0 < nm; q0 += PU * TPT) {
    T a_p[PU], a_b0[PU], a_w0[PU], a_W0[PU], a_b1[PU], a_w1[PU], a_W1[PU], a_cp[PU], a_lo[PU], a_iv[PU];
#pragma unroll
    for (int u = 0; u < PU; ++u) {
      const int q = q0 + u * TPT;
      if (q < nm) {
        const int k = q / TPC, i = min(i0 + q % TPC, nx - 1);
        const int p = i + nx * j + k * pm;
        const int p0 = i + nx * j + min(max(k, 1), nz - 1) * pm;
        const int p1 = i + nx * j + min(max(k + 1, 1), nz - 1) * pm;
        a_p[u] = ld(yp, p);
        a_b0[u] = ld(c.pbw, p0);
        a_w0[u] = ld(yw, p0);
        a_W0[u] = ld(yW, p0);
        a_b1[u] = ld(c.pbw, p1);
        a_w1[u] = ld(yw, p1);
        a_W1[u] = ld(yW, p1);
        a_cp[u] = ld(c.tcp, p);
        a_lo[u] = ld(c.tlo, p);
        a_iv[u] = ld(c.tinv, p);
      }
    }
#pragma unroll
    for (int u = 0; u < PU; ++u) {
      const int q = q0 + u * TPT;
      if (q < nm) {
        const int k = q / TPC;
        const T g0 = -a_b0[u] * (a_w0[u] + a_W0[u]);
        const T g1 = -a_b1[u] * (a_w1[u] + a_W1[u]);
        const T G0 = (k > 0 && k < nz) ? g0 : T(0);
        const T G1 = (k + 1 > 0 && k + 1 < nz) ? g1 : T(0);
        s_x[q] = a_p[u] * ps + G0 - G1;
        s_cp[q] = a_cp[u];
        s_lo[q] = a_lo[u];
        s_iv[q] = a_iv[u];
      }
    }
  }
  __syncthreads();
  // ---- B: U^T w = pibar upward, L^T z = w downward, one thread per column ----
  if (tid < TPC) {
    const int l = tid;
    T wprev = T(0), cprev = T(0);
    for (int k = 0; k < nz; ++k) {
      const int q = k * TPC + l;
      wprev = s_x[q] - cprev * wprev;
      s_x[q] = wprev;
      cprev = s_cp[q];
    }
    T zh = T(0), loh = T(0);
    for (int k = nz - 1; k >= 0; --k) {
      const int q = k * TPC + l;
      zh = (s_x[q] - loh * zh) * s_iv[q];
      s_x[q] = zh;
      loh = s_lo[q];
    }
  }
  __syncthreads();
  // ---- C: pi, w and eta_dot cotangents ----
  for (int q0 = tid; q0 < nw; q0 += PU * TPT) {
    T c_w[PU], c_W[PU], c_a[PU], c_b[PU], c_r[PU], c_d[PU];
#pragma unroll
    for (int u = 0; u < PU; ++u) {
      const int q = q0 + u * TPT;
      const int k = q / TPC, i = i0 + q % TPC;
      if (q < nw && i < nx) {
        const int p = i + nx * j + k * pm;
        c_w[u] = ld(yw, p);
        c_W[u] = ld(yW, p);
        if (k == 0 || k == nz) {
          c_d[u] = ld(c.dzw, p);
        } else {
          c_a[u] = ld(c.lpi, p - pm);
          c_b[u] = ld(c.lpi, p);
          c_r[u] = ld(c.rtw, p);
          c_d[u] = ld(c.idamp, p);
        }
      }
    }
#pragma unroll
    for (int u = 0; u < PU; ++u) {
      const int q = q0 + u * TPT;
      const int k = q / TPC, i = i0 + q % TPC;
      if (q < nw && i < nx) {
        const int p = i + nx * j + k * pm;
        if (k < nz) op[p] = s_x[q] * ips;
        if (k == 0 || k == nz) {
          ow[p] = c_w[u];
          oW[p] = c_W[u] * c_d[u];
        } else {
          const T dvl = mul_rn(-c_a[u], s_x[q - TPC]), dv = mul_rn(-c_b[u], s_x[q]);
          const T ep = c_W[u] + c_r[u] * (dvl - dv);
          oW[p] = ep * inva;
          ow[p] = (c_w[u] + ep) * c_d[u];
        }
      }
    }
  }
}
template <typename T, int TPT, int TPC, int PU>
__global__ void __launch_bounds__(TPT) pt_column_batched_kernel(Dims d, Coef<T> c, CVec5<T> y, Vec5<T> out,
                                                                const int* active) {
  if (active && *active == 0) return;
  pt_column_batched_block<T, TPT, TPC, PU>(d, c, y, out, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ---------------------------------------------------------------------------
// M^T, horizontal part: out_u = y_u + sum of the kinematic cotangent
// kinbar = -alpha out_W over the interior w levels of the adjacent cells.
template <typename T>
__device__ __forceinline__ void pt_uv_block(const Dims& d, const Coef<T>& c, const CVec5<T>& y, const Vec5<T>& out, int bx, int by, int bz) {
  const int i = bx * blockDim.x + threadIdx.x;
  const int j = by * blockDim.y + threadIdx.y;
  const int k = bz * blockDim.z + threadIdx.z;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i > nx || j > ny || k >= nz) return;
  const T qa = -(T)c.s.alpha * T(0.25);
  const T* __restrict__ oW = out.f[4];
  if (j < ny) {
    const int p = iu(d, i, j, k);
    T g = ld(y.f[0], p);
    for (int ii = i - 1; ii <= i; ++ii) {
      if (ii < 0 || ii >= nx) continue;
      const T m = ld(c.mm, h_m(d, ii, j));
      for (int K = k; K <= k + 1; ++K) {
        if (K <= 0 || K >= nz) continue;
        const int pw = iw(d, ii, j, K);
        g += qa * m * ld(c.zxw, pw) * oW[pw];
      }
    }
    out.f[0][p] = g;
  }
  if (i < nx) {
    const int p = iv(d, i, j, k);
    T g = ld(y.f[1], p);
    for (int jj = j - 1; jj <= j; ++jj) {
      if (jj < 0 || jj >= ny) continue;
      const T m = ld(c.mm, h_m(d, i, jj));
      for (int K = k; K <= k + 1; ++K) {
        if (K <= 0 || K >= nz) continue;
        const int pw = iw(d, i, jj, K);
        g += qa * m * ld(c.zew, pw) * oW[pw];
      }
    }
    out.f[1][p] = g;
  }
}
template <typename T>
__global__ void __launch_bounds__(256) pt_uv_kernel(Dims d, Coef<T> c, CVec5<T> y, Vec5<T> out, const int* active) {
  if (active && *active == 0) return;
  pt_uv_block<T>(d, c, y, out, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ---------------------------------------------------------------------------
// Tricubic VJP (cotangent of the field; the departure points carry none,
// steppers.py:764-767): every destination point scatters its cotangent with
// the 64 Catmull-Rom weights of tensor_product_interp_3d
// (operators.py:146-209).  With the limiter, jnp.clip(f, lo, hi) and the
// min/max chains over the 8 cell corners in the reference order route the
// cotangent as lax.min/lax.max do: all of it to the strictly smaller
// (larger) operand, half to each on a tie.
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void cr_w(T t, T (&w)[4]) {
  w[0] = t * (T(-0.5) + t * (T(1) - T(0.5) * t));
  w[1] = T(1) + t * t * (T(-2.5) + T(1.5) * t);
  w[2] = t * (T(0.5) + t * (T(2) - T(1.5) * t));
  w[3] = t * t * (T(-0.5) + T(0.5) * t);
}

__device__ __forceinline__ void atomic_acc(float* a, float v) { atomicAdd(a, v); }
__device__ __forceinline__ void atomic_acc(double* a, double v) { atomicAdd(a, v); }

// Scatter targets of the tricubic VJP.  AtomicAcc adds into the gradient
// with float atomics (the sum's rounding depends on the order the atomics
// land).  FixedAcc adds each contribution as a fixed-point integer v * 2^e:
// integer addition is associative, so the sum -- and the gradient formed
// from it -- is the same bits on every run.  float: one 64-bit word per
// element.  double: two words, the integer part of v * 2^e and its fraction
// in 2^fb units, summed separately (the fraction sums carry into the result
// when it is formed), so double contributions keep their precision.
template <typename T>
struct AtomicAcc {
  T* g;
  __device__ __forceinline__ void add(int i, T v) const { atomic_acc(g + i, v); }
};
template <typename T>
struct FixedAcc;
template <>
struct FixedAcc<float> {
  unsigned long long* acc;
  size_t n;
  double s;  // 2^e (v * s is exact in double)
  __device__ __forceinline__ void add(int i, float v) const {
    atomicAdd(acc + i, (unsigned long long)__double2ll_rn((double)v * s));
  }
};
template <>
struct FixedAcc<double> {
  unsigned long long* acc;  // [0, n): integer parts, [n, 2n): fractions
  size_t n;
  double s;   // 2^e
  double fs;  // 2^fb
  __device__ __forceinline__ void add(int i, double v) const {
    const double y = v * s;
    double h = floor(y);
    double r = rint((y - h) * fs);  // y - h is exact; r in [0, 2^fb]
    if (r == fs) { h += 1.0; r = 0.0; }
    atomicAdd(acc + i, (unsigned long long)(long long)h);
    atomicAdd(acc + n + i, (unsigned long long)r);
  }
};

// Header of the fixed-point scratch: the largest |scale * cot| (as the bits
// of a float rounded up, which order like the values) and the largest
// number of destination points whose stencil base is one source cell.
struct DetHdr {
  unsigned int gmax_bits;
  int max_count;
};

// The fixed-point exponent.  A target sums contributions of points whose
// stencil base lies in a 4x4x4 box of cells (64 cells of at most max_count
// points each), a point giving one target at most 27 weights (clamping
// folds up to three stencil rows per axis) plus 8 limiter corners, each of
// magnitude <= gmax: below 2^12 * max_count terms, so the integer sums stay
// below 2^61.
__device__ __forceinline__ int det_exponent(const DetHdr* h) {
  const float gmax = __uint_as_float(h->gmax_bits);
  int eg, ec;
  frexpf(gmax, &eg);                         // gmax < 2^eg
  frexpf((float)max(h->max_count, 1), &ec);  // count < 2^ec
  return 61 - 12 - ec - eg;
}
// fraction bits of the double accumulator: sums of 2^12 * count fractions
// below 2^fb each stay below 2^63
__device__ __forceinline__ int det_fraction_bits(const DetHdr* h) {
  int ec;
  frexpf((float)max(h->max_count, 1), &ec);
  return min(32, 63 - 12 - ec);
}

template <typename T>
__device__ __forceinline__ FixedAcc<T> make_fixed_acc(unsigned long long* acc, size_t n, const DetHdr* h);
template <>
__device__ __forceinline__ FixedAcc<float> make_fixed_acc<float>(unsigned long long* acc, size_t n, const DetHdr* h) {
  return FixedAcc<float>{acc, n, ldexp(1.0, det_exponent(h))};
}
template <>
__device__ __forceinline__ FixedAcc<double> make_fixed_acc<double>(unsigned long long* acc, size_t n,
                                                                   const DetHdr* h) {
  return FixedAcc<double>{acc, n, ldexp(1.0, det_exponent(h)), ldexp(1.0, det_fraction_bits(h))};
}

// share of the cotangent of op(a, b) that goes to a: 1, 0 or 1/2 on a tie
template <typename T>
__device__ __forceinline__ T share_min(T a, T b) { return a < b ? T(1) : (a > b ? T(0) : T(0.5)); }
template <typename T>
__device__ __forceinline__ T share_max(T a, T b) { return a > b ? T(1) : (a < b ? T(0) : T(0.5)); }

// Stencil bases and fractions of destination point (i, j, k): from the
// absolute coordinates (clamped, floored) or, REL, from split-form offsets
// (cubic_base; source and destination shapes equal).
template <typename T, int REL>
__device__ __forceinline__ void vjp_base(int i, int j, int k, int p, int sx, int sy, int sz,
                                         const T* __restrict__ cx, const T* __restrict__ cy,
                                         const T* __restrict__ cz, int& x0, int& y0, int& z0, T& tx, T& ty,
                                         T& tz) {
  if (REL) {
    cubic_base(i, ld(cx, p), sx, x0, tx);
    cubic_base(j, ld(cy, p), sy, y0, ty);
    cubic_base(k, ld(cz, p), sz, z0, tz);
  } else {
    const T x = fmin(fmax(ld(cx, p), T(0)), (T)(sx - 1));
    const T y = fmin(fmax(ld(cy, p), T(0)), (T)(sy - 1));
    const T z = fmin(fmax(ld(cz, p), T(0)), (T)(sz - 1));
    x0 = (int)floor(x), y0 = (int)floor(y), z0 = (int)floor(z);
    tx = x - (T)x0, ty = y - (T)y0, tz = z - (T)z0;
  }
}

template <typename T, typename Acc, int REL = 0>
__device__ __forceinline__ void tricubic_vjp_point(int sx, int sy, int sz, int dx, int dy, int dz,
                                                   const T* __restrict__ f, const T* __restrict__ cx,
                                                   const T* __restrict__ cy, const T* __restrict__ cz,
                                                   const T* __restrict__ cot, const Acc& grad, int limiter,
                                                   T scale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= dx || j >= dy || k >= dz) return;
  const int p = i + dx * (j + dy * k);
  const T g = scale * ld(cot, p);
  if (g == T(0)) return;
  int x0, y0, z0;
  T tx, ty, tz;
  vjp_base<T, REL>(i, j, k, p, sx, sy, sz, cx, cy, cz, x0, y0, z0, tx, ty, tz);
  T wx[4], wy[4], wz[4];
  cr_w(tx, wx);
  cr_w(ty, wy);
  cr_w(tz, wz);
  const int ix[4] = {max(x0 - 1, 0), x0, min(x0 + 1, sx - 1), min(x0 + 2, sx - 1)};
  const int iy[4] = {max(y0 - 1, 0), y0, min(y0 + 1, sy - 1), min(y0 + 2, sy - 1)};
  const int iz[4] = {max(z0 - 1, 0), z0, min(z0 + 1, sz - 1), min(z0 + 2, sz - 1)};
  const int plane = sx * sy;
  T gf = g;
  if (limiter) {
    T fi = T(0);
#pragma unroll
    for (int a = 0; a < 4; ++a) {
      T syv = T(0);
#pragma unroll
      for (int b = 0; b < 4; ++b) {
        const int row = ix[a] + sx * iy[b];
        T szv = T(0);
#pragma unroll
        for (int q = 0; q < 4; ++q) szv += wz[q] * ld(f, row + plane * iz[q]);
        syv += wy[b] * szv;
      }
      fi += wx[a] * syv;
    }
    const int x1 = min(x0 + 1, sx - 1), y1 = min(y0 + 1, sy - 1), z1 = min(z0 + 1, sz - 1);
    // corners in the reference order (operators.py:200-201)
    const int cidx[8] = {x0 + sx * (y0 + sy * z0), x1 + sx * (y0 + sy * z0), x0 + sx * (y1 + sy * z0),
                         x1 + sx * (y1 + sy * z0), x0 + sx * (y0 + sy * z1), x1 + sx * (y0 + sy * z1),
                         x0 + sx * (y1 + sy * z1), x1 + sx * (y1 + sy * z1)};
    T nb[8], mn[8], mx[8];
#pragma unroll
    for (int s = 0; s < 8; ++s) nb[s] = ld(f, cidx[s]);
    mn[0] = mx[0] = nb[0];
#pragma unroll
    for (int s = 1; s < 8; ++s) {
      mn[s] = fmin(mn[s - 1], nb[s]);
      mx[s] = fmax(mx[s - 1], nb[s]);
    }
    // jnp.clip(f, lo, hi) = minimum(hi, maximum(lo, f))
    const T lo = mn[7], hi = mx[7];
    const T v1 = fmax(lo, fi);
    const T a1 = share_max(fi, lo);  // to f
    const T a2 = share_min(v1, hi);  // to maximum(lo, f)
    gf = g * a2 * a1;
    T glo = g * a2 * (T(1) - a1), ghi = g * (T(1) - a2);
    T gn[8];
#pragma unroll
    for (int s = 0; s < 8; ++s) gn[s] = T(0);
#pragma unroll
    for (int s = 7; s >= 1; --s) {
      const T wl = share_min(mn[s - 1], nb[s]);
      gn[s] += glo * (T(1) - wl);
      glo *= wl;
      const T wh = share_max(mx[s - 1], nb[s]);
      gn[s] += ghi * (T(1) - wh);
      ghi *= wh;
    }
    gn[0] += glo + ghi;
#pragma unroll
    for (int s = 0; s < 8; ++s)
      if (gn[s] != T(0)) grad.add(cidx[s], gn[s]);
    if (gf == T(0)) return;
  }
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    const T ga = gf * wx[a];
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int row = ix[a] + sx * iy[b];
      const T gb = ga * wy[b];
#pragma unroll
      for (int q = 0; q < 4; ++q) grad.add(row + plane * iz[q], gb * wz[q]);
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256) tricubic_vjp_kernel(int sx, int sy, int sz, int dx, int dy, int dz,
                                                           const T* __restrict__ f, const T* __restrict__ cx,
                                                           const T* __restrict__ cy, const T* __restrict__ cz,
                                                           const T* __restrict__ cot, T* grad, int limiter,
                                                           T scale) {
  tricubic_vjp_point(sx, sy, sz, dx, dy, dz, f, cx, cy, cz, cot, AtomicAcc<T>{grad}, limiter, scale);
}

// Deterministic VJP, pass 1: per destination point with a cotangent, count
// it in the source cell of its stencil base (cnt) and keep the running
// maxima of the counts and of |scale * cot| in the header.
template <typename T, int REL>
__global__ void __launch_bounds__(256) tricubic_vjp_count_kernel(int sx, int sy, int sz, int dx, int dy, int dz,
                                                                 const T* __restrict__ cx, const T* __restrict__ cy,
                                                                 const T* __restrict__ cz, const T* __restrict__ cot,
                                                                 T scale, int* cnt, DetHdr* hdr) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  float amax = 0.f;
  int cmax = 0;
  if (i < dx && j < dy && k < dz) {
    const int p = i + dx * (j + dy * k);
    const T g = scale * ld(cot, p);
    if (g != T(0)) {
      int x0, y0, z0;
      T tx, ty, tz;
      vjp_base<T, REL>(i, j, k, p, sx, sy, sz, cx, cy, cz, x0, y0, z0, tx, ty, tz);
      const int b = x0 + sx * (y0 + sy * z0);
      cmax = atomicAdd(cnt + b, 1) + 1;
      amax = __double2float_ru(fabs((double)g));
    }
  }
  for (int o = 16; o > 0; o >>= 1) {  // blockDim.x = 32: a warp is one x row
    amax = fmaxf(amax, __shfl_down_sync(0xffffffffu, amax, o));
    cmax = max(cmax, __shfl_down_sync(0xffffffffu, cmax, o));
  }
  if (threadIdx.x == 0 && cmax > 0) {
    atomicMax(&hdr->gmax_bits, __float_as_uint(amax));
    atomicMax(&hdr->max_count, cmax);
  }
}

// pass 2: the scatter in fixed point (acc zeroed beforehand)
template <typename T, int REL>
__global__ void __launch_bounds__(256) tricubic_vjp_fixed_kernel(int sx, int sy, int sz, int dx, int dy, int dz,
                                                                 const T* __restrict__ f, const T* __restrict__ cx,
                                                                 const T* __restrict__ cy, const T* __restrict__ cz,
                                                                 const T* __restrict__ cot, unsigned long long* acc,
                                                                 const DetHdr* hdr, int limiter, T scale) {
  if (hdr->max_count == 0) return;  // no cotangent at all
  const FixedAcc<T> a = make_fixed_acc<T>(acc, (size_t)sx * sy * sz, hdr);
  tricubic_vjp_point<T, FixedAcc<T>, REL>(sx, sy, sz, dx, dy, dz, f, cx, cy, cz, cot, a, limiter, scale);
}

// pass 3: grad += acc * 2^-e (one rounding per element, in a fixed order)
template <typename T>
__global__ void tricubic_vjp_finish_kernel(size_t n, const unsigned long long* __restrict__ acc,
                                           const DetHdr* hdr, T* __restrict__ grad) {
  if (hdr->max_count == 0) return;
  const double inv = ldexp(1.0, -det_exponent(hdr));
  const double finv = sizeof(T) == 8 ? ldexp(1.0, -det_fraction_bits(hdr)) : 0.0;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n; q += (size_t)gridDim.x * blockDim.x) {
    double v = (double)(long long)acc[q];
    if (sizeof(T) == 8) v += (double)acc[n + q] * finv;
    if (v != 0.0) grad[q] = grad[q] + (T)(v * inv);
  }
}

}  // namespace

// grad += scale * (d tricubic / d field)^T cot
template <typename T>
void launch_tricubic_vjp(int sx, int sy, int sz, int dx, int dy, int dz, const T* field, const T* const* coords3,
                         const T* cot, T* grad, int use_limiter, T scale, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  tricubic_vjp_kernel<T><<<box_grid(dx, dy, dz, blk), blk, 0, st>>>(sx, sy, sz, dx, dy, dz, field, coords3[0],
                                                                    coords3[1], coords3[2], cot, grad,
                                                                    use_limiter, scale);
}
size_t tricubic_vjp_det_scratch_bytes(int sx, int sy, int sz, int elem_bytes) {
  return 256 + (elem_bytes == 8 ? 2 : 1) * sizeof(unsigned long long) * (size_t)sx * sy * sz;
}

// Deterministic grad += scale * (d tricubic / d field)^T cot with the
// fixed-point scratch of tricubic_vjp_det_scratch_bytes (256-byte aligned).
template <typename T>
void launch_tricubic_vjp_det(int sx, int sy, int sz, int dx, int dy, int dz, const T* field,
                             const T* const* coords3, const T* cot, T* grad, int use_limiter, T scale, void* scratch,
                             int relative, cudaStream_t st) {
  DetHdr* hdr = (DetHdr*)scratch;
  unsigned long long* acc = (unsigned long long*)((char*)scratch + 256);
  const size_t n = (size_t)sx * sy * sz;
  dim3 blk(32, 4, 2);
  cudaMemsetAsync(scratch, 0, 256 + sizeof(int) * n, st);  // header and the counts (in acc's memory)
  const dim3 grd = box_grid(dx, dy, dz, blk);
  if (relative)
    tricubic_vjp_count_kernel<T, 1><<<grd, blk, 0, st>>>(sx, sy, sz, dx, dy, dz, coords3[0], coords3[1],
                                                         coords3[2], cot, scale, (int*)acc, hdr);
  else
    tricubic_vjp_count_kernel<T, 0><<<grd, blk, 0, st>>>(sx, sy, sz, dx, dy, dz, coords3[0], coords3[1],
                                                         coords3[2], cot, scale, (int*)acc, hdr);
  cudaMemsetAsync(acc, 0, (sizeof(T) == 8 ? 2 : 1) * sizeof(unsigned long long) * n, st);
  if (relative)
    tricubic_vjp_fixed_kernel<T, 1><<<grd, blk, 0, st>>>(sx, sy, sz, dx, dy, dz, field, coords3[0], coords3[1],
                                                         coords3[2], cot, acc, hdr, use_limiter, scale);
  else
    tricubic_vjp_fixed_kernel<T, 0><<<grd, blk, 0, st>>>(sx, sy, sz, dx, dy, dz, field, coords3[0], coords3[1],
                                                         coords3[2], cot, acc, hdr, use_limiter, scale);
  const size_t nb = (n + 255) / 256;
  tricubic_vjp_finish_kernel<T><<<(unsigned)(nb < 148 * 16 ? nb : 148 * 16), 256, 0, st>>>(n, acc, hdr, grad);
}
template void launch_tricubic_vjp_det<float>(int, int, int, int, int, int, const float*, const float* const*,
                                             const float*, float*, int, float, void*, int, cudaStream_t);
template void launch_tricubic_vjp_det<double>(int, int, int, int, int, int, const double*, const double* const*,
                                              const double*, double*, int, double, void*, int, cudaStream_t);
template void launch_tricubic_vjp<float>(int, int, int, int, int, int, const float*, const float* const*,
                                         const float*, float*, int, float, cudaStream_t);
template void launch_tricubic_vjp<double>(int, int, int, int, int, int, const double*, const double* const*,
                                          const double*, double*, int, double, cudaStream_t);

// out = M^T y (out must not alias y).
// M^T as a column march (one thread per column, NT columns per block) with
// the factorisation T = L U of prep_thomas: T^T z = pibar is U^T w = pibar
// upward (w(k) = pibar(k) - c'(k-1) w(k-1), w kept in shared memory), then
// L^T z = w downward (z(k) = (w(k) - lower(k+1) z(k+1)) / pivot(k)), where
// the w and eta_dot cotangents of the w level between z(k) and z(k+1) are
// formed.  Shared memory per block: nz * NT values of T.
template <typename T, int NT>
__device__ __forceinline__ void pt_march_block(const Dims& d, const Coef<T>& c, const CVec5<T>& y, const Vec5<T>& out, int bx, int by, int bz) {
  extern __shared__ __align__(16) unsigned char smem_raw[];
  T* s_w = reinterpret_cast<T*>(smem_raw);  // [nz][NT]
  const int t = threadIdx.x;
  const int i = bx * NT + t, j = by;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i >= nx) return;
  const int pm = nx * ny, h = i + nx * j;
  const T ps = (T)c.s.ps, ips = (T)(1.0 / c.s.ps), inva = T(1) / (T)c.s.alpha;
  const T* __restrict__ yw = y.f[2];
  const T* __restrict__ yp = y.f[3];
  const T* __restrict__ yW = y.f[4];
  T* __restrict__ ow = out.f[2];
  T* __restrict__ op = out.f[3];
  T* __restrict__ oW = out.f[4];
  T G_lo = T(0), wprev = T(0), cprev = T(0);
#pragma unroll 4
  for (int k = 0; k < nz; ++k) {
    const int p = h + k * pm;
    T G_hi = T(0);
    if (k + 1 < nz) {
      const int pw = p + pm;
      G_hi = -ld(c.pbw, pw) * (ld(yw, pw) + ld(yW, pw));
    }
    const T pib = ld(yp, p) * ps + G_lo - G_hi;
    const T wv = pib - cprev * wprev;
    s_w[k * NT + t] = wv;
    wprev = wv;
    cprev = ld(c.tcp, p);
    G_lo = G_hi;
  }
  T zh = T(0), loh = T(0), dvh = T(0);
#pragma unroll 4
  for (int k = nz - 1; k >= 0; --k) {
    const int p = h + k * pm;
    const T z = (s_w[k * NT + t] - loh * zh) * ld(c.tinv, p);
    op[p] = z * ips;
    const T dv = mul_rn(-ld(c.lpi, p), z);
    if (k + 1 < nz) {
      const int pw = p + pm;
      const T ep = ld(yW, pw) + ld(c.rtw, pw) * (dv - dvh);
      oW[pw] = ep * inva;
      ow[pw] = (ld(yw, pw) + ep) * ld(c.idamp, pw);
    }
    zh = z;
    loh = ld(c.tlo, p);
    dvh = dv;
  }
  ow[h] = ld(yw, h);
  oW[h] = ld(yW, h) * ld(c.dzw, h);
  const int ptop = h + nz * pm;
  ow[ptop] = ld(yw, ptop);
  oW[ptop] = ld(yW, ptop) * ld(c.dzw, ptop);
}
template <typename T, int NT>
__global__ void __launch_bounds__(NT) pt_march_kernel(Dims d, Coef<T> c, CVec5<T> y, Vec5<T> out,
                                                      const int* active) {
  if (active && *active == 0) return;
  pt_march_block<T, NT>(d, c, y, out, blockIdx.x, blockIdx.y, blockIdx.z);
}

// ---------------------------------------------------------------------------
// grouped transposed operators over ensemble members (sisl_group.cuh): flat
// block b runs block (b - first[m]) of member m's standalone launch
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T* gvec_a(const GroupMember<T>& g, int v) {
  return g.vec + (size_t)v * g.npad;
}
// block (bx, by, bz) of a box of ex x ey x . points covered by blockDim-shaped blocks
__device__ __forceinline__ void group_box(int t, int ex, int ey, int& bx, int& by, int& bz) {
  const int gx = (ex + (int)blockDim.x - 1) / (int)blockDim.x, gy = (ey + (int)blockDim.y - 1) / (int)blockDim.y;
  bz = t / (gx * gy);
  const int r = t - bz * (gx * gy);
  by = r / gx;
  bx = r - by * gx;
}

// stage 0: at_gzm (mass points), stage 1: at_main (union box).  mode 0
// Arnoldi step j (gated): V_j scaled by s_j -> z; mode 1 b - A^T x -> z;
// mode 2 (U = double): b64 - A64^T x64 -> r64
template <typename T, typename U>
__global__ void __launch_bounds__(256) group_at_kernel(GroupMember<T>* mem, const int* __restrict__ first, int M,
                                                       int stage, int mode, int j) {
  const int b = blockIdx.x;
  const int mi = group_find(first, M, b);
  const GroupMember<T>& g = mem[mi];
  if (!g.running) return;
  if (mode == 0 && g.gs->active == 0) return;
  int bx, by, bz;
  group_box(b - first[mi], stage ? g.d.nx + 1 : g.d.nx, stage ? g.d.ny + 1 : g.d.ny, bx, by, bz);
  // scale and right-hand side pointers stay run-time values in every mode,
  // so the rows contract into the same FMAs as the standalone kernels'
  const double* ysp = (mode == 0) ? &g.gs->s[j] : nullptr;
  if constexpr (sizeof(U) == sizeof(T)) {
    const T* src = gvec_a(g, mode == 0 ? GV_V0 + j : GV_X);
    CVec5<T> y, bb;
    Vec5<T> out;
    const T* bv = gvec_a(g, GV_B);
    T* z = gvec_a(g, GV_Z);
    for (int q = 0; q < 5; ++q) {
      y.f[q] = src + g.off[q];
      bb.f[q] = (mode == 1) ? bv + g.off[q] : nullptr;
      out.f[q] = z + g.off[q];
    }
    if (stage == 0) at_gzm_block<T>(g.d, g.c, y.f[0], y.f[1], ysp, g.tmp, bx, by, bz);
    else at_main_block<T>(g.d, g.c, y, ysp, g.tmp, bb, out, bx, by, bz);
  } else {
    CVec5<double> y, bb;
    Vec5<double> out;
    for (int q = 0; q < 5; ++q) {
      y.f[q] = g.x64 + g.off[q];
      bb.f[q] = (mode != 0) ? g.b64 + g.off[q] : nullptr;
      out.f[q] = g.r64 + g.off[q];
    }
    if (stage == 0) at_gzm_block<double>(g.d, g.c64, y.f[0], y.f[1], ysp, g.tmp64, bx, by, bz);
    else at_main_block<double>(g.d, g.c64, y, ysp, g.tmp64, bb, out, bx, by, bz);
  }
}

// stage 0: column tile (32 columns per block of 256, batched loads, the
// autotuner's usual choice), stage 1: u and v faces.  mode 0: z -> V_tv
// (gated when asked); mode 1: b -> V_1
template <typename T>
__global__ void __launch_bounds__(256) group_pt_kernel(GroupMember<T>* mem, const int* __restrict__ first, int M,
                                                       int stage, int mode, int tv, int gated) {
  const int b = blockIdx.x;
  const int mi = group_find(first, M, b);
  const GroupMember<T>& g = mem[mi];
  if (!g.running || (gated && g.gs->active == 0)) return;
  T* tgt = gvec_a(g, mode == 0 ? GV_V0 + tv : GV_V0 + 1);
  const T* src = gvec_a(g, mode == 0 ? GV_Z : GV_B);
  CVec5<T> y;
  Vec5<T> out;
  for (int q = 0; q < 5; ++q) {
    y.f[q] = src + g.off[q];
    out.f[q] = tgt + g.off[q];
  }
  const int t = b - first[mi];
  if (stage == 0) {
    const int gx = (g.d.nx + 31) / 32;
    const int by = t / gx;
    pt_column_batched_block<T, 256, 32, 4>(g.d, g.c, y, out, t - by * gx, by, 0);
  } else {
    int bx, by, bz;
    group_box(t, g.d.nx + 1, g.d.ny + 1, bx, by, bz);
    pt_uv_block<T>(g.d, g.c, y, out, bx, by, bz);
  }
}

int group_at_blocks(const Dims& d, int stage) {
  const dim3 blk(32, 4, 2);
  const dim3 g = stage ? box_grid(d.nx + 1, d.ny + 1, d.nz + 1, blk) : box_grid(d.nx, d.ny, d.nz, blk);
  return (int)(g.x * g.y * g.z);
}
int group_pt_blocks(const Dims& d, int stage) {
  if (stage == 0) return ((d.nx + 31) / 32) * d.ny;
  const dim3 g = box_grid(d.nx + 1, d.ny + 1, d.nz, dim3(32, 4, 2));
  return (int)(g.x * g.y * g.z);
}

template <typename T>
void grp_matvec_t(const GroupLaunch<T>& g, int mode, int j, cudaStream_t st) {
  for (int stage = 0; stage < 2; ++stage) {
    const int tb = stage ? GT_ATM : GT_ATG;
    if (mode == 2) {
      if constexpr (sizeof(T) == 4)
        group_at_kernel<T, double><<<g.blocks(tb), dim3(32, 4, 2), 0, st>>>(g.mem, g.row(tb), g.M, stage, 2, 0);
    } else {
      group_at_kernel<T, T><<<g.blocks(tb), dim3(32, 4, 2), 0, st>>>(g.mem, g.row(tb), g.M, stage, mode, j);
    }
  }
}

template <typename T>
void grp_precond_t(const GroupLaunch<T>& g, int mode, int t, int gated, cudaStream_t st) {
  int nz_max = 1;
  for (int m = 0; m < g.M; ++m) nz_max = nz_max > g.nz_h[m] ? nz_max : g.nz_h[m];
  const size_t smem = (size_t)(4 * nz_max) * 32 * sizeof(T);
  static SmemLimit attr_bytes;
  ensure_smem_limit((const void*)group_pt_kernel<T>, attr_bytes, smem);
  group_pt_kernel<T><<<g.blocks(GT_PTM), 256, smem, st>>>(g.mem, g.row(GT_PTM), g.M, 0, mode, t, gated);
  group_pt_kernel<T><<<g.blocks(GT_PTU), dim3(32, 4, 2), 0, st>>>(g.mem, g.row(GT_PTU), g.M, 1, mode, t, gated);
}

template void grp_matvec_t<float>(const GroupLaunch<float>&, int, int, cudaStream_t);
template void grp_matvec_t<double>(const GroupLaunch<double>&, int, int, cudaStream_t);
template void grp_precond_t<float>(const GroupLaunch<float>&, int, int, int, cudaStream_t);
template void grp_precond_t<double>(const GroupLaunch<double>&, int, int, int, cudaStream_t);

template <typename T, int NT>
void launch_pt_march(const Dims& d, const Coef<T>& c, CVec5<T> y, Vec5<T> out, const int* active,
                     cudaStream_t st) {
  const size_t smem = (size_t)d.nz * NT * sizeof(T);
  static SmemLimit attr_bytes;  // per instantiation
  ensure_smem_limit((const void*)pt_march_kernel<T, NT>, attr_bytes, smem);
  pt_march_kernel<T, NT><<<dim3((d.nx + NT - 1) / NT, d.ny), NT, smem, st>>>(d, c, y, out, active);
}

template <typename T, int TPT, int TPC>
void launch_pt_column(const Dims& d, const Coef<T>& c, CVec5<T> y, Vec5<T> out, const int* active,
                      cudaStream_t st) {
  const size_t smem = (size_t)(4 * d.nz) * TPC * sizeof(T);
  static SmemLimit attr_bytes;  // per instantiation
  ensure_smem_limit((const void*)pt_column_kernel<T, TPT, TPC>, attr_bytes, smem);
  pt_column_kernel<T, TPT, TPC><<<dim3((d.nx + TPC - 1) / TPC, d.ny), TPT, smem, st>>>(d, c, y, out, active);
}

template <typename T, int TPT, int TPC, int PU>
void launch_pt_column_batched(const Dims& d, const Coef<T>& c, CVec5<T> y, Vec5<T> out, const int* active,
                              cudaStream_t st) {
  const size_t smem = (size_t)(4 * d.nz) * TPC * sizeof(T);
  static SmemLimit attr_bytes;  // per instantiation
  ensure_smem_limit((const void*)pt_column_batched_kernel<T, TPT, TPC, PU>, attr_bytes, smem);
  pt_column_batched_kernel<T, TPT, TPC, PU>
      <<<dim3((d.nx + TPC - 1) / TPC, d.ny), TPT, smem, st>>>(d, c, y, out, active);
}

template <typename T>
void launch_precond_t(const Dims& d, const Coef<T>& c, CVec5<T> y, Vec5<T> out, const int* active,
                      cudaStream_t st) {
  int v = d.tune_pct;
  if (v == 2 && (size_t)(4 * d.nz) * 64 * sizeof(T) > 200 * 1024) v = 0;  // 64-column tile too large
  switch (v) {
    case 1: launch_pt_column<T, 128, 16>(d, c, y, out, active, st); break;
    case 2: launch_pt_column<T, 256, 64>(d, c, y, out, active, st); break;
    case 3: launch_pt_march<T, 128>(d, c, y, out, active, st); break;
    case 4: launch_pt_column_batched<T, 256, 32, 4>(d, c, y, out, active, st); break;
    default: launch_pt_column<T, 256, 32>(d, c, y, out, active, st); break;
  }
  const dim3 blk = stencil_block(d.tune_mvt);
  pt_uv_kernel<T><<<box_grid(d.nx + 1, d.ny + 1, d.nz, blk), blk, 0, st>>>(d, c, y, out, active);
}

template void launch_precond_t<float>(const Dims&, const Coef<float>&, CVec5<float>, Vec5<float>, const int*,
                                      cudaStream_t);
template void launch_precond_t<double>(const Dims&, const Coef<double>&, CVec5<double>, Vec5<double>, const int*,
                                       cudaStream_t);

// out = A^T (y * yscale), or out = b - A^T(...) when b is given; gzm_tmp is a
// mass-point scratch field.
template <typename T>
void launch_matvec_t(const Dims& d, const Coef<T>& c, CVec5<T> y, const double* yscale, CVec5<T> b, Vec5<T> out,
                     T* gzm_tmp, const int* active, cudaStream_t st) {
  const dim3 blk = stencil_block(d.tune_mvt);
  at_gzm_kernel<T><<<box_grid(d.nx, d.ny, d.nz, blk), blk, 0, st>>>(d, c, y.f[0], y.f[1], yscale, gzm_tmp, active);
  at_main_kernel<T><<<box_grid(d.nx + 1, d.ny + 1, d.nz + 1, blk), blk, 0, st>>>(d, c, y, yscale, gzm_tmp, b, out,
                                                                              active);
}

template void launch_matvec_t<float>(const Dims&, const Coef<float>&, CVec5<float>, const double*, CVec5<float>,
                                     Vec5<float>, float*, const int*, cudaStream_t);
template void launch_matvec_t<double>(const Dims&, const Coef<double>&, CVec5<double>, const double*, CVec5<double>,
                                      Vec5<double>, double*, const int*, cudaStream_t);

}  // namespace sisl
