// Shared device-side definitions for the SISL kernels (sm_100a).
//
// Field layout on the device: a 3-D field of stagger s has the extents of the
// reference array, (ex, ey, ez) = (nx + [s==u], ny + [s==v], nz + [s==w]),
// stored x-fastest: element (i, j, k) lives at i + ex * (j + ey * k).  This is
// the Fortran order of the reference's C-ordered (ex, ey, ez) arrays, so one
// thread per (i, j) column reads a coalesced row per level, and mass and
// w points share the same horizontal plane layout.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <atomic>
#include <mutex>

namespace sisl {

// Per-device record of the dynamic shared-memory limit a kernel has been
// raised to.  cudaFuncSetAttribute acts on the current device only, so each
// device keeps its own entry (a process may drive cores on several devices).
constexpr int SMEM_LIMIT_DEVICES = 64;
struct SmemLimit {
  std::atomic<size_t> bytes[SMEM_LIMIT_DEVICES];
};

// Raises a kernel's dynamic shared-memory limit on the current device to at
// least `bytes` (never lowers it).  Host threads that drive different cores
// call the launchers concurrently, so the check-and-set runs under one lock.
// The limit is recorded only when the attribute call succeeds; on failure
// the launch that follows reports the error.
inline void ensure_smem_limit(const void* fn, SmemLimit& limit, size_t bytes) {
  if (bytes <= 48 * 1024) return;
  int dev = 0;
  if (cudaGetDevice(&dev) != cudaSuccess) return;
  if (dev < 0 || dev >= SMEM_LIMIT_DEVICES) {  // no slot: set it every time
    cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes);
    return;
  }
  std::atomic<size_t>& current = limit.bytes[dev];
  if (bytes <= current.load()) return;
  static std::mutex m;
  std::lock_guard<std::mutex> lock(m);
  if (bytes > current.load() &&
      cudaFuncSetAttribute(fn, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)bytes) == cudaSuccess)
    current.store(bytes);
}

enum Loc { LOC_M = 0, LOC_U = 1, LOC_V = 2, LOC_W = 3 };

struct Dims {
  int nx, ny, nz;
  int px, py;          // periodic flags for x and y
  double dx, dy, dz;
  // launch shapes chosen by the autotuner (sisl_autotune): the Helmholtz
  // matvec (default 6: the column march), its transpose (stencil block), the
  // column preconditioner (default 6: the pipelined column march) and its
  // transpose (column tile)
  int tune_mv = 6, tune_pc = 6, tune_mvt = 0, tune_pct = 0;
};

// block shapes of the 3-D stencil kernels (256 threads each)
__host__ inline dim3 stencil_block(int variant) {
  switch (variant) {
    case 1: return dim3(32, 8, 1);
    case 2: return dim3(32, 2, 4);
    case 3: return dim3(64, 4, 1);
    default: return dim3(32, 4, 2);
  }
}
constexpr int N_STENCIL_BLOCKS = 4;
// the 4 blocks, 32x8 columns of 2 or 4 levels per thread, and the column
// march (32x4 columns) in 1, 2 or 4 z chunks
constexpr int N_MATVEC_SHAPES = 9;
// column variants: tiles of (threads, columns) = (256, 32), (128, 16), (256, 64),
// and the one-thread-per-column march (128 columns per block)
constexpr int N_COLUMN_TILES = 4;
// forward preconditioner only: also the (256, 32) tile with
// batched loads and staged face sums, the pipelined one-thread-per-column
// march (64 columns per block, loads two levels ahead, without and with L2
// eviction hints), and the march fed by cp.async copies into a shared ring
// (32 columns, 6 levels)
constexpr int N_PRECOND_SHAPES = 8;
// its transpose: also the (256, 32) tile with batched loads
constexpr int N_PRECOND_T_SHAPES = 5;

__host__ __device__ inline int ext_x(const Dims& d, int loc) { return d.nx + (loc == LOC_U); }
__host__ __device__ inline int ext_y(const Dims& d, int loc) { return d.ny + (loc == LOC_V); }
__host__ __device__ inline int ext_z(const Dims& d, int loc) { return d.nz + (loc == LOC_W); }
__host__ __device__ inline size_t field_size(const Dims& d, int loc) {
  return (size_t)ext_x(d, loc) * ext_y(d, loc) * ext_z(d, loc);
}

// 3-D offsets per stagger.
__device__ __forceinline__ int im(const Dims& d, int i, int j, int k) { return i + d.nx * (j + d.ny * k); }
__device__ __forceinline__ int iu(const Dims& d, int i, int j, int k) { return i + (d.nx + 1) * (j + d.ny * k); }
__device__ __forceinline__ int iv(const Dims& d, int i, int j, int k) { return i + d.nx * (j + (d.ny + 1) * k); }
__device__ __forceinline__ int iw(const Dims& d, int i, int j, int k) { return i + d.nx * (j + d.ny * k); }
// 2-D (horizontal) offsets per stagger.
__device__ __forceinline__ int h_m(const Dims& d, int i, int j) { return i + d.nx * j; }
__device__ __forceinline__ int h_u(const Dims& d, int i, int j) { return i + (d.nx + 1) * j; }
__device__ __forceinline__ int h_v(const Dims& d, int i, int j) { return i + d.nx * j; }

// Mass-to-face neighbour pair along a horizontal axis (operators.py:37-132).
// Interior face f (0 < f < n) averages/differences cells f-1 and f.  The two
// boundary faces of an open axis reuse the nearest interior face's pair (the
// edge padding of operators.py:45-61); on a periodic axis both boundary faces
// pair the last and first cells (operators.py:85-95, 123-131).
__device__ __forceinline__ void face_pair(int f, int n, int periodic, int& l, int& r) {
  if (f > 0 && f < n) { l = f - 1; r = f; return; }
  if (periodic) { l = n - 1; r = 0; return; }
  if (f == 0) { l = 0; r = 1; } else { l = n - 2; r = n - 1; }
}
// periodic or edge-clamped mass index along an axis of n cells
__device__ __forceinline__ int wrap_or_clamp(int q, int n, int periodic) {
  if (periodic) return ((q % n) + n) % n;
  return min(max(q, 0), n - 1);
}
// Mass-to-w pair along z (never periodic).
__device__ __forceinline__ void level_pair(int k, int nz, int& l, int& r) {
  if (k > 0 && k < nz) { l = k - 1; r = k; return; }
  if (k == 0) { l = 0; r = 1; } else { l = nz - 2; r = nz - 1; }
}

template <typename T>
__device__ __forceinline__ T ld(const T* __restrict__ p, int i) { return __ldg(p + i); }

// Split coordinates of a departure point: integer index i plus offset o (the
// point i + o, with o = -alpha the displacement in index units).  Forming
// i - alpha in float32 keeps only ~24 - log2(i) bits of alpha's fraction
// (about 1e-5 cell at i ~ 200, a systematic error that accumulates step
// after step); the offset keeps all of alpha's bits, and the stencil base
// and fraction follow from it exactly.
//
// Clamped Catmull-Rom stencil base x0 and fraction t of clip(i + o, 0, n - 1)
// (operators.py:172-179).
template <typename T>
__device__ __forceinline__ void cubic_base(int i, T o, int n, int& x0, T& t) {
  if (o <= (T)(-i)) { x0 = 0; t = T(0); return; }
  if (o >= (T)(n - 1 - i)) { x0 = n - 1; t = T(0); return; }
  const T fo = floor(o);
  x0 = i + (int)fo;
  t = o - fo;
}
// map_coordinates(order=1) base floor(i + o) and weight (no clamp of the
// coordinate; the caller clamps the two indices).
template <typename T>
__device__ __forceinline__ void linear_base(int i, T o, int& l, T& w) {
  o = fmin(fmax(o, T(-1e8)), T(1e8));  // keeps i + floor(o) an int for any input (indices are clamped after)
  const T fo = floor(o);
  l = i + (int)fo;
  w = o - fo;
}

// A product rounded on its own (never contracted into an FMA), for values
// that several code paths share and must round identically.
__device__ __forceinline__ float mul_rn(float a, float b) { return __fmul_rn(a, b); }
__device__ __forceinline__ double mul_rn(double a, double b) { return __dmul_rn(a, b); }

// Block-wide double-precision sum of NV values per thread; thread 0 of the
// block ends up with the totals in out[].
template <int NV>
__device__ __forceinline__ void block_sum(double (&v)[NV], double* smem /* blockDim/32 * NV */) {
  const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
  const int nw = (blockDim.x + 31) >> 5;
#pragma unroll
  for (int q = 0; q < NV; ++q) {
    double s = v[q];
    for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
    if (lane == 0) smem[warp * NV + q] = s;
  }
  __syncthreads();
  if (warp == 0) {
#pragma unroll
    for (int q = 0; q < NV; ++q) {
      double s = (lane < nw) ? smem[lane * NV + q] : 0.0;
      for (int o = 16; o > 0; o >>= 1) s += __shfl_down_sync(0xffffffffu, s, o);
      v[q] = s;
    }
  }
  __syncthreads();
}

}  // namespace sisl
