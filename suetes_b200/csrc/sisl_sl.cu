// Semi-Lagrangian kernels: trajectory index velocities, midpoint departure
// points with trilinear gathers, and the 64-point Catmull-Rom tricubic.
//
// * trajectory velocities: steppers.py:748-762 (1.5 x - 0.5 x_prev after the
//   first step) and _get_index_velocities (steppers.py:276-316);
// * departure points: compute_departure_indices (steppers.py:318-360) with
//   map_coordinates(order=1, mode='nearest') (steppers.py:362-367);
// * tricubic: tensor_product_interp_3d (operators.py:146-209).
#include "sisl_core.cuh"

namespace sisl {
namespace {

struct Ext {
  int ex, ey, ez;
};
__device__ __forceinline__ Ext loc_ext(const Dims& d, int loc) {
  return Ext{ext_x(d, loc), ext_y(d, loc), ext_z(d, loc)};
}

// ---------------------------------------------------------------------------
// index velocities of every stagger, one thread per union-box point
// vel[loc*3 + 0..2] = (u * m / dx, v * m / dy, eta_dot) averaged to loc.
// ---------------------------------------------------------------------------
template <typename T>
__global__ void traj_velocity_kernel(Dims d, Coef<T> c, const T* __restrict__ u, const T* __restrict__ v,
                                     const T* __restrict__ e, const T* __restrict__ up,
                                     const T* __restrict__ vp, const T* __restrict__ ep, int extrap,
                                     PtrTable<T> vel) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i > nx || j > ny || k > nz) return;
  const T idx = (T)(1.0 / d.dx), idy = (T)(1.0 / d.dy);
  auto U = [&](int a, int b, int cc) {
    const int p = iu(d, a, b, cc);
    return extrap ? T(1.5) * ld(u, p) - T(0.5) * ld(up, p) : ld(u, p);
  };
  auto V = [&](int a, int b, int cc) {
    const int p = iv(d, a, b, cc);
    return extrap ? T(1.5) * ld(v, p) - T(0.5) * ld(vp, p) : ld(v, p);
  };
  auto E = [&](int a, int b, int cc) {
    const int p = iw(d, a, b, cc);
    return extrap ? T(1.5) * ld(e, p) - T(0.5) * ld(ep, p) : ld(e, p);
  };
  auto Um = [&](int a, int b, int cc) { return T(0.5) * (U(a, b, cc) + U(a + 1, b, cc)); };
  auto Vm = [&](int a, int b, int cc) { return T(0.5) * (V(a, b, cc) + V(a, b + 1, cc)); };
  auto Em = [&](int a, int b, int cc) { return T(0.5) * (E(a, b, cc) + E(a, b, cc + 1)); };

  // a null first pointer skips a stagger
  if (vel.p[0] && i < nx && j < ny && k < nz) {  // m
    const int p = im(d, i, j, k);
    const T m = ld(c.mm, h_m(d, i, j));
    vel.p[0][p] = Um(i, j, k) * m * idx;
    vel.p[1][p] = Vm(i, j, k) * m * idy;
    vel.p[2][p] = Em(i, j, k);
  }
  if (vel.p[3] && j < ny && k < nz) {  // u
    int l, r;
    face_pair(i, nx, d.px, l, r);
    const int p = iu(d, i, j, k);
    const T m = ld(c.mu, h_u(d, i, j));
    vel.p[3][p] = U(i, j, k) * m * idx;
    vel.p[4][p] = T(0.5) * (Vm(l, j, k) + Vm(r, j, k)) * m * idy;
    vel.p[5][p] = T(0.5) * (Em(l, j, k) + Em(r, j, k));
  }
  if (vel.p[6] && i < nx && k < nz) {  // v
    int l, r;
    face_pair(j, ny, d.py, l, r);
    const int p = iv(d, i, j, k);
    const T m = ld(c.mv, h_v(d, i, j));
    vel.p[6][p] = T(0.5) * (Um(i, l, k) + Um(i, r, k)) * m * idx;
    vel.p[7][p] = V(i, j, k) * m * idy;
    vel.p[8][p] = T(0.5) * (Em(i, l, k) + Em(i, r, k));
  }
  if (vel.p[9] && i < nx && j < ny) {  // w
    int kl, kr;
    level_pair(k, nz, kl, kr);
    const int p = iw(d, i, j, k);
    const T m = ld(c.mm, h_m(d, i, j));
    vel.p[9][p] = T(0.5) * (Um(i, j, kl) + Um(i, j, kr)) * m * idx;
    vel.p[10][p] = T(0.5) * (Vm(i, j, kl) + Vm(i, j, kr)) * m * idy;
    vel.p[11][p] = E(i, j, k);
  }
}

// map_coordinates(order=1, mode='nearest'): indices floor(c), floor(c)+1
// clipped into range; corners summed in itertools.product order.
template <typename T>
__device__ __forceinline__ T trilinear(const T* __restrict__ f, const Ext& e, T x, T y, T z) {
  const T fx = floor(x), fy = floor(y), fz = floor(z);
  const T wx = x - fx, wy = y - fy, wz = z - fz;
  const int lx = (int)fx, ly = (int)fy, lz = (int)fz;
  const int ix[2] = {min(max(lx, 0), e.ex - 1), min(max(lx + 1, 0), e.ex - 1)};
  const int iy[2] = {min(max(ly, 0), e.ey - 1), min(max(ly + 1, 0), e.ey - 1)};
  const int iz[2] = {min(max(lz, 0), e.ez - 1), min(max(lz + 1, 0), e.ez - 1)};
  const T Wx[2] = {T(1) - wx, wx}, Wy[2] = {T(1) - wy, wy}, Wz[2] = {T(1) - wz, wz};
  T acc = T(0);
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int q = 0; q < 2; ++q)
        acc += Wx[a] * Wy[b] * Wz[q] * ld(f, ix[a] + e.ex * (iy[b] + e.ey * iz[q]));
  return acc;
}

// the same gather at the split point (i + ox, j + oy, k + oz)
template <typename T>
__device__ __forceinline__ T trilinear_rel(const T* __restrict__ f, const Ext& e, int i, int j, int k, T ox, T oy,
                                           T oz) {
  int lx, ly, lz;
  T wx, wy, wz;
  linear_base(i, ox, lx, wx);
  linear_base(j, oy, ly, wy);
  linear_base(k, oz, lz, wz);
  const int ix[2] = {min(max(lx, 0), e.ex - 1), min(max(lx + 1, 0), e.ex - 1)};
  const int iy[2] = {min(max(ly, 0), e.ey - 1), min(max(ly + 1, 0), e.ey - 1)};
  const int iz[2] = {min(max(lz, 0), e.ez - 1), min(max(lz + 1, 0), e.ez - 1)};
  const T Wx[2] = {T(1) - wx, wx}, Wy[2] = {T(1) - wy, wy}, Wz[2] = {T(1) - wz, wz};
  T acc = T(0);
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int b = 0; b < 2; ++b)
#pragma unroll
      for (int q = 0; q < 2; ++q)
        acc += Wx[a] * Wy[b] * Wz[q] * ld(f, ix[a] + e.ex * (iy[b] + e.ey * iz[q]));
  return acc;
}

// Midpoint departure iteration in split form: the offsets (ox, oy, oz) =
// -alpha of the point (i, j, k) (steppers.py:318-360).
template <typename T>
__device__ __forceinline__ void departure_rel(const Ext& e, int i, int j, int k, T dt, const T* __restrict__ vx,
                                              const T* __restrict__ vy, const T* __restrict__ vz, int iters, T& ox,
                                              T& oy, T& oz) {
  const int p = i + e.ex * (j + e.ey * k);
  T ax = dt * ld(vx, p), ay = dt * ld(vy, p), az = dt * ld(vz, p);
  for (int it = 0; it < iters; ++it) {
    const T mx = T(-0.5) * ax, my = T(-0.5) * ay, mz = T(-0.5) * az;
    ax = dt * trilinear_rel(vx, e, i, j, k, mx, my, mz);
    ay = dt * trilinear_rel(vy, e, i, j, k, mx, my, mz);
    az = dt * trilinear_rel(vz, e, i, j, k, mx, my, mz);
  }
  ox = -ax;
  oy = -ay;
  oz = -az;
}

template <typename T>
__device__ __forceinline__ void departure_at(const Ext& e, int i, int j, int k, T dt, const T* __restrict__ vx,
                                             const T* __restrict__ vy, const T* __restrict__ vz, int iters,
                                             T& cx, T& cy, T& cz) {
  const int p = i + e.ex * (j + e.ey * k);
  const T X = (T)i, Y = (T)j, Z = (T)k;
  T ax = dt * ld(vx, p), ay = dt * ld(vy, p), az = dt * ld(vz, p);
  for (int it = 0; it < iters; ++it) {
    const T mx = X - T(0.5) * ax, my = Y - T(0.5) * ay, mz = Z - T(0.5) * az;
    ax = dt * trilinear(vx, e, mx, my, mz);
    ay = dt * trilinear(vy, e, mx, my, mz);
    az = dt * trilinear(vz, e, mx, my, mz);
  }
  cx = X - ax;
  cy = Y - ay;
  cz = Z - az;
}

template <typename T>
__device__ __forceinline__ void cr_weights(T t, T (&w)[4]) {
  // cubic_weight(p0..p3, t) written as weights of p0..p3 (operators.py:134-144)
  w[0] = t * (T(-0.5) + t * (T(1) - T(0.5) * t));
  w[1] = T(1) + t * t * (T(-2.5) + T(1.5) * t);
  w[2] = t * (T(0.5) + t * (T(2) - T(1.5) * t));
  w[3] = t * t * (T(-0.5) + T(0.5) * t);
}

// the 64-point Catmull-Rom sum (and the limiter) at stencil bases
// (x0, y0, z0) with fractions (tx, ty, tz)
template <typename T>
__device__ __forceinline__ T tricubic_core(const T* __restrict__ f, const Ext& e, int x0, int y0, int z0, T tx,
                                           T ty, T tz, int limiter) {
  T wx[4], wy[4], wz[4];
  cr_weights(tx, wx);
  cr_weights(ty, wy);
  cr_weights(tz, wz);
  const int ix[4] = {max(x0 - 1, 0), x0, min(x0 + 1, e.ex - 1), min(x0 + 2, e.ex - 1)};
  const int iy[4] = {max(y0 - 1, 0), y0, min(y0 + 1, e.ey - 1), min(y0 + 2, e.ey - 1)};
  const int iz[4] = {max(z0 - 1, 0), z0, min(z0 + 1, e.ez - 1), min(z0 + 2, e.ez - 1)};
  const int plane = e.ex * e.ey;
  T out = T(0);
#pragma unroll
  for (int a = 0; a < 4; ++a) {
    T sy = T(0);
#pragma unroll
    for (int b = 0; b < 4; ++b) {
      const int row = ix[a] + e.ex * iy[b];
      T sz = T(0);
#pragma unroll
      for (int q = 0; q < 4; ++q) sz += wz[q] * ld(f, row + plane * iz[q]);
      sy += wy[b] * sz;
    }
    out += wx[a] * sy;
  }
  if (limiter) {
    const int x1 = min(x0 + 1, e.ex - 1), y1 = min(y0 + 1, e.ey - 1), z1 = min(z0 + 1, e.ez - 1);
    const int xs[2] = {x0, x1}, ys[2] = {y0, y1}, zs[2] = {z0, z1};
    T lo = ld(f, x0 + e.ex * (y0 + e.ey * z0)), hi = lo;
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int b = 0; b < 2; ++b)
#pragma unroll
        for (int q = 0; q < 2; ++q) {
          const T nb = ld(f, xs[a] + e.ex * (ys[b] + e.ey * zs[q]));
          lo = fmin(lo, nb);
          hi = fmax(hi, nb);
        }
    out = fmin(fmax(out, lo), hi);
  }
  return out;
}

template <typename T>
__device__ __forceinline__ T tricubic_at(const T* __restrict__ f, const Ext& e, T x, T y, T z, int limiter) {
  x = fmin(fmax(x, T(0)), (T)(e.ex - 1));
  y = fmin(fmax(y, T(0)), (T)(e.ey - 1));
  z = fmin(fmax(z, T(0)), (T)(e.ez - 1));
  const int x0 = (int)floor(x), y0 = (int)floor(y), z0 = (int)floor(z);
  return tricubic_core(f, e, x0, y0, z0, x - (T)x0, y - (T)y0, z - (T)z0, limiter);
}

// the same at the split point (i + ox, j + oy, k + oz)
template <typename T>
__device__ __forceinline__ T tricubic_rel(const T* __restrict__ f, const Ext& e, int i, int j, int k, T ox, T oy,
                                          T oz, int limiter) {
  int x0, y0, z0;
  T tx, ty, tz;
  cubic_base(i, ox, e.ex, x0, tx);
  cubic_base(j, oy, e.ey, y0, ty);
  cubic_base(k, oz, e.ez, z0, tz);
  return tricubic_core(f, e, x0, y0, z0, tx, ty, tz, limiter);
}

// relative = 1 writes the split-form offsets -alpha instead of the points
template <typename T>
__global__ void departure_kernel(Dims d, int loc, T dt, const T* __restrict__ vx, const T* __restrict__ vy,
                                 const T* __restrict__ vz, int iters, T* cx, T* cy, T* cz, int relative) {
  const Ext e = loc_ext(d, loc);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= e.ex || j >= e.ey || k >= e.ez) return;
  T x, y, z;
  if (relative) departure_rel(e, i, j, k, dt, vx, vy, vz, iters, x, y, z);
  else departure_at(e, i, j, k, dt, vx, vy, vz, iters, x, y, z);
  const int p = i + e.ex * (j + e.ey * k);
  cx[p] = x;
  cy[p] = y;
  cz[p] = z;
}

template <typename T>
__global__ void tricubic_kernel(Ext src, Ext dst, const T* __restrict__ f, const T* __restrict__ cx,
                                const T* __restrict__ cy, const T* __restrict__ cz, T* out, int limiter,
                                T scale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= dst.ex || j >= dst.ey || k >= dst.ez) return;
  const int p = i + dst.ex * (j + dst.ey * k);
  out[p] = scale * tricubic_at(f, src, ld(cx, p), ld(cy, p), ld(cz, p), limiter);
}

template <typename T>
__global__ void trilinear_kernel(Ext src, Ext dst, const T* __restrict__ f, const T* __restrict__ cx,
                                 const T* __restrict__ cy, const T* __restrict__ cz, T* out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= dst.ex || j >= dst.ey || k >= dst.ez) return;
  const int p = i + dst.ex * (j + dst.ey * k);
  out[p] = trilinear(f, src, ld(cx, p), ld(cy, p), ld(cz, p));
}

// Departure point + tricubic of up to 2 fields sharing the stagger, in
// split coordinates.
template <typename T>
__global__ void sl_advect_kernel(Dims d, int loc, T dt, const T* __restrict__ vx, const T* __restrict__ vy,
                                 const T* __restrict__ vz, int iters, int nf, const T* __restrict__ f0,
                                 const T* __restrict__ f1, T* o0, T* o1, T s0, T s1, int limiter) {
  const Ext e = loc_ext(d, loc);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= e.ex || j >= e.ey || k >= e.ez) return;
  T ox, oy, oz;
  departure_rel(e, i, j, k, dt, vx, vy, vz, iters, ox, oy, oz);
  const int p = i + e.ex * (j + e.ey * k);
  o0[p] = s0 * tricubic_rel(f0, e, i, j, k, ox, oy, oz, limiter);
  if (nf > 1) o1[p] = s1 * tricubic_rel(f1, e, i, j, k, ox, oy, oz, limiter);
}

dim3 box_grid(int ex, int ey, int ez, dim3 blk) {
  return dim3((ex + blk.x - 1) / blk.x, (ey + blk.y - 1) / blk.y, (ez + blk.z - 1) / blk.z);
}

}  // namespace

template <typename T>
void launch_traj_velocity(const Dims& d, const Coef<T>& c, const T* u, const T* v, const T* eta, const T* up,
                          const T* vp, const T* etap, int extrapolate, PtrTable<T> vel, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  traj_velocity_kernel<T><<<box_grid(d.nx + 1, d.ny + 1, d.nz + 1, blk), blk, 0, st>>>(
      d, c, u, v, eta, up, vp, etap, extrapolate, vel);
}

template <typename T>
void launch_departure(const Dims& d, int loc, double dt, const T* const* vel3, int iterations, T* const* coords3,
                      int relative, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  departure_kernel<T><<<box_grid(ext_x(d, loc), ext_y(d, loc), ext_z(d, loc), blk), blk, 0, st>>>(
      d, loc, (T)dt, vel3[0], vel3[1], vel3[2], iterations, coords3[0], coords3[1], coords3[2], relative);
}

template <typename T>
void launch_tricubic_ext(int sx, int sy, int sz, int dx, int dy, int dz, const T* field, const T* const* coords3,
                         T* out, int use_limiter, T scale, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  tricubic_kernel<T><<<box_grid(dx, dy, dz, blk), blk, 0, st>>>(Ext{sx, sy, sz}, Ext{dx, dy, dz}, field,
                                                               coords3[0], coords3[1], coords3[2], out,
                                                               use_limiter, scale);
}

template <typename T>
void launch_trilinear_ext(int sx, int sy, int sz, int dx, int dy, int dz, const T* field, const T* const* coords3,
                          T* out, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  trilinear_kernel<T><<<box_grid(dx, dy, dz, blk), blk, 0, st>>>(Ext{sx, sy, sz}, Ext{dx, dy, dz}, field,
                                                                coords3[0], coords3[1], coords3[2], out);
}

template <typename T>
void launch_sl_advect(const Dims& d, int loc, double dt, const T* const* vel3, int iterations, int nf,
                      const T* const* fields, T* const* outs, const T* scales, int use_limiter, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  sl_advect_kernel<T><<<box_grid(ext_x(d, loc), ext_y(d, loc), ext_z(d, loc), blk), blk, 0, st>>>(
      d, loc, (T)dt, vel3[0], vel3[1], vel3[2], iterations, nf, fields[0], nf > 1 ? fields[1] : nullptr,
      outs[0], nf > 1 ? outs[1] : nullptr, scales[0], nf > 1 ? scales[1] : T(0), use_limiter);
}

#define SISL_INST_SL(T)                                                                                     \
  template void launch_traj_velocity<T>(const Dims&, const Coef<T>&, const T*, const T*, const T*, const T*, \
                                        const T*, const T*, int, PtrTable<T>, cudaStream_t);                 \
  template void launch_departure<T>(const Dims&, int, double, const T* const*, int, T* const*, int,          \
                                    cudaStream_t);                                                           \
  template void launch_tricubic_ext<T>(int, int, int, int, int, int, const T*, const T* const*, T*, int, T,  \
                                       cudaStream_t);                                                        \
  template void launch_trilinear_ext<T>(int, int, int, int, int, int, const T*, const T* const*, T*,         \
                                        cudaStream_t);                                                       \
  template void launch_sl_advect<T>(const Dims&, int, double, const T* const*, int, int, const T* const*,    \
                                    T* const*, const T*, int, cudaStream_t);
SISL_INST_SL(float)
SISL_INST_SL(double)

}  // namespace sisl
