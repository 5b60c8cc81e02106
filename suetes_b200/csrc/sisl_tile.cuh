// Shared-memory halo tiles of the semi-Lagrangian gathers and scatters.
//
// A block of destination points reads (or, for the VJP, writes) the source
// field only inside the bounding box of its 4x4x4 stencils: the box of the
// block's departure cells, widened by 1 below and 2 above and clamped to
// the field.  When the box fits the block's buffer it is staged once with
// coalesced loads (x fastest) and every stencil access goes to shared
// memory; otherwise (very large Courant numbers) the block falls back to
// global memory.  The decision is uniform over the block.
#pragma once

#include <climits>

#include "sisl_common.cuh"

namespace sisl {

template <typename T>
struct TileCap {  // elements of one staged box (24 KB)
  static constexpr int n = (int)(24 * 1024 / sizeof(T));
};

struct SlBox {
  int lx, ly, lz, nx, ny, nz;
  __device__ __forceinline__ int vol() const { return (nx > 0 && ny > 0 && nz > 0) ? nx * ny * nz : 0; }
};

// Bounding box of the stencils of the block's valid points (all threads of
// the block must call it; `sb` is 6 ints of shared memory).
__device__ __forceinline__ SlBox block_box(int* sb, bool valid, int x0, int y0, int z0, int ex, int ey, int ez) {
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  if (tid == 0) {
    sb[0] = sb[1] = sb[2] = INT_MAX;
    sb[3] = sb[4] = sb[5] = INT_MIN;
  }
  __syncthreads();
  const unsigned full = 0xffffffffu;
  const int mnx = __reduce_min_sync(full, valid ? x0 : INT_MAX);
  const int mny = __reduce_min_sync(full, valid ? y0 : INT_MAX);
  const int mnz = __reduce_min_sync(full, valid ? z0 : INT_MAX);
  const int mxx = __reduce_max_sync(full, valid ? x0 : INT_MIN);
  const int mxy = __reduce_max_sync(full, valid ? y0 : INT_MIN);
  const int mxz = __reduce_max_sync(full, valid ? z0 : INT_MIN);
  if ((tid & 31) == 0) {
    atomicMin(&sb[0], mnx);
    atomicMin(&sb[1], mny);
    atomicMin(&sb[2], mnz);
    atomicMax(&sb[3], mxx);
    atomicMax(&sb[4], mxy);
    atomicMax(&sb[5], mxz);
  }
  __syncthreads();
  SlBox b;
  if (sb[0] == INT_MAX) {  // no valid point in the block
    b.lx = b.ly = b.lz = 0;
    b.nx = b.ny = b.nz = 0;
    return b;
  }
  b.lx = max(sb[0] - 1, 0);
  b.ly = max(sb[1] - 1, 0);
  b.lz = max(sb[2] - 1, 0);
  b.nx = min(sb[3] + 2, ex - 1) - b.lx + 1;
  b.ny = min(sb[4] + 2, ey - 1) - b.ly + 1;
  b.nz = min(sb[5] + 2, ez - 1) - b.lz + 1;
  return b;
}

// Stage the box of field f (x-fastest, extents ex x ey x ...) into s.
template <typename T>
__device__ __forceinline__ void stage_box(const T* __restrict__ f, int ex, int ey, const SlBox& b, T* s) {
  const int tid = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nt = blockDim.x * blockDim.y * blockDim.z;
  const int vol = b.vol();
  for (int q = tid; q < vol; q += nt) {
    const int a = q % b.nx, r = q / b.nx;
    const int c = r / b.ny, bb = r - c * b.ny;
    s[q] = ld(f, (b.lx + a) + ex * ((b.ly + bb) + ey * (b.lz + c)));
  }
  __syncthreads();
}

template <typename T>
struct BoxFetch {
  const T* s;
  SlBox b;
  __device__ __forceinline__ T operator()(int a, int bb, int c) const {
    return s[(a - b.lx) + b.nx * ((bb - b.ly) + b.ny * (c - b.lz))];
  }
};

// One fetch for both cases: a staged box (generic pointer to shared memory,
// box origin and strides) or the whole field in global memory (origin 0).
template <typename T>
struct AnyFetch {
  const T* base;
  int ox, oy, oz, sx, splane;
  __device__ __forceinline__ T operator()(int a, int bb, int c) const {
    return base[(a - ox) + sx * (bb - oy) + splane * (c - oz)];
  }
};

template <typename T>
__device__ __forceinline__ AnyFetch<T> box_or_global(bool tiled, const T* s, const SlBox& b, const T* f, int ex,
                                                     int ey) {
  if (tiled) return AnyFetch<T>{s, b.lx, b.ly, b.lz, b.nx, b.nx * b.ny};
  return AnyFetch<T>{f, 0, 0, 0, ex, ex * ey};
}

}  // namespace sisl
