// Flat vector kernels and float64 bookkeeping of the device-resident GMRES.
//
// Restates jax.scipy.sparse.linalg.gmres (jax/jaxlib >= 0.10.0; called at
// steppers.py:466 and :476): left preconditioning (Krylov space of M A), one
// classical Gram-Schmidt projection per Arnoldi step over the basis, breakdown
// when ||v|| <= eps ||M A v_k||, and either the 'batched' cycle (normal
// equations + Cholesky for the Hessenberg least-squares problem) or the
// 'incremental' cycle (Givens rotations, early exit on the rotated residual).
//
// A basis vector V_i is stored unnormalised next to its inverse norm s_i, so
// normalisation never costs a pass over memory: the matvec scales its input
// on load, projections use h_i = s_i <V_i, w>, updates use h_i s_i V_i.
// Every reduction accumulates in float64; the last block of a reduction
// kernel (ticket counter) finishes the sum and runs the scalar logic.
#include "sisl_group.cuh"

#include <math.h>

namespace sisl {
namespace {

constexpr int GT = 256;  // threads per block of the flat kernels

template <typename T> struct V16;
template <> struct V16<float> { using type = float4; static constexpr int n = 4; };
template <> struct V16<double> { using type = double2; static constexpr int n = 2; };

template <typename T>
__device__ __forceinline__ void load16(const T* p, T* r) {
  using VT = typename V16<T>::type;
  VT v = __ldg(reinterpret_cast<const VT*>(p));
  const T* q = reinterpret_cast<const T*>(&v);
#pragma unroll
  for (int e = 0; e < V16<T>::n; ++e) r[e] = q[e];
}
template <typename T>
__device__ __forceinline__ void store16(T* p, const T* r) {
  using VT = typename V16<T>::type;
  VT v;
  T* q = reinterpret_cast<T*>(&v);
#pragma unroll
  for (int e = 0; e < V16<T>::n; ++e) q[e] = r[e];
  *reinterpret_cast<VT*>(p) = v;
}

// Per-thread chunk: CH 16-byte loads (E = CH * 16/sizeof(T) elements).
constexpr int CH = 4;

__device__ __forceinline__ double warp_sum(double s) {
  for (int o = 16; o > 0; o >>= 1) s += __shfl_xor_sync(0xffffffffu, s, o);
  return s;
}

// Last-block ticket.  Returns true in exactly one block, after every other
// block's partial results are visible.
__device__ __forceinline__ bool last_block(unsigned int* counter, unsigned int nblk) {
  __shared__ bool am_last;
  __threadfence();
  __syncthreads();
  if (threadIdx.x == 0) {
    unsigned int t = atomicAdd(counter, 1u);
    am_last = (t == nblk - 1);
  }
  __syncthreads();
  if (am_last) __threadfence();
  return am_last;
}

enum DotMode { DM_PROJ = 0, DM_BNORM = 1, DM_MBNORM = 2, DM_RNORM = 3 };

// result_i = <V_i, w> for i < m and <w, w>; finished according to `mode`.
// Per tile, every warp sums its products (float64) with shuffles and lane 0
// adds them to the warp's shared slot acc[q * warps + warp]: (m + 1) x 8
// doubles per block, so shared memory never limits the resident blocks
// (registers do); the block reduces the warps' slots once at the end.
// Block `bid` of `nblk` blocks of one reduction (a member's share of a
// grouped launch, or the whole grid of a standalone one).
template <typename T>
__device__ __forceinline__ void dots_body(const T* __restrict__ Vb, size_t stride, int m, const T* __restrict__ w,
                                          size_t n, double* partial, GState* gs, int mode, int bid, int nblk) {
  extern __shared__ double acc[];  // (m + 1) * warps: per-warp sums
  const int tid = threadIdx.x, nt = blockDim.x;
  const int lane = tid & 31, wp = tid >> 5, nw = nt >> 5;
  for (int q = tid; q < (m + 1) * nw; q += nt) acc[q] = 0.0;
  __syncthreads();
  constexpr int VN = V16<T>::n;
  constexpr int E = CH * VN;
  const size_t tile = (size_t)nt * E;
  for (size_t base = (size_t)bid * tile; base < n; base += (size_t)nblk * tile) {
    T wr[E];
#pragma unroll
    for (int c = 0; c < CH; ++c) {
      const size_t off = base + ((size_t)c * nt + tid) * VN;
      if (off < n) load16(w + off, wr + c * VN);
      else
#pragma unroll
        for (int e = 0; e < VN; ++e) wr[c * VN + e] = T(0);
    }
    double sq = 0.0;
#pragma unroll
    for (int e = 0; e < E; ++e) sq += (double)wr[e] * (double)wr[e];
    sq = warp_sum(sq);
    if (lane == 0) acc[m * nw + wp] += sq;
    // two basis vectors per iteration: both chunks are in flight together
    int i = 0;
    for (; i + 1 < m; i += 2) {
      const T* __restrict__ Va = Vb + (size_t)i * stride;
      const T* __restrict__ Vc = Va + stride;
      T va[E], vc[E];
#pragma unroll
      for (int c = 0; c < CH; ++c) {
        const size_t off = base + ((size_t)c * nt + tid) * VN;
        if (off < n) {
          load16(Va + off, va + c * VN);
          load16(Vc + off, vc + c * VN);
        } else {
#pragma unroll
          for (int e = 0; e < VN; ++e) { va[c * VN + e] = T(0); vc[c * VN + e] = T(0); }
        }
      }
      double pa = 0.0, pc = 0.0;
#pragma unroll
      for (int e = 0; e < E; ++e) {
        pa += (double)va[e] * (double)wr[e];
        pc += (double)vc[e] * (double)wr[e];
      }
      pa = warp_sum(pa);
      pc = warp_sum(pc);
      if (lane == 0) {
        acc[i * nw + wp] += pa;
        acc[(i + 1) * nw + wp] += pc;
      }
    }
    if (i < m) {
      const T* __restrict__ Vi = Vb + (size_t)i * stride;
      T vr[E];
#pragma unroll
      for (int c = 0; c < CH; ++c) {
        const size_t off = base + ((size_t)c * nt + tid) * VN;
        if (off < n) load16(Vi + off, vr + c * VN);
        else
#pragma unroll
          for (int e = 0; e < VN; ++e) vr[c * VN + e] = T(0);
      }
      double p = 0.0;
#pragma unroll
      for (int e = 0; e < E; ++e) p += (double)vr[e] * (double)wr[e];
      p = warp_sum(p);
      if (lane == 0) acc[i * nw + wp] += p;
    }
  }
  __syncthreads();
  // block reduction: thread q sums the warps' slots of result q
  for (int q = tid; q <= m; q += nt) {
    double s_ = 0.0;
    for (int k = 0; k < nw; ++k) s_ += acc[q * nw + k];
    partial[(size_t)bid * (GM_MAXR + 2) + q] = s_;
  }
  if (!last_block(&gs->counter, (unsigned)nblk)) return;
  // finish: sum the partials of all blocks, one warp per result (lanes
  // stride over the blocks, so the loads are independent)
  for (int q = wp; q <= m; q += nw) {
    double s_ = 0.0;
    for (int b = lane; b < nblk; b += 32) s_ += partial[(size_t)b * (GM_MAXR + 2) + q];
    s_ = warp_sum(s_);
    if (lane == 0) acc[q] = s_;
  }
  __syncthreads();
  if (tid == 0) {
    gs->counter = 0;
    const double nrm = sqrt(acc[m]);
    if (mode == DM_PROJ) {
      for (int i = 0; i < m; ++i) gs->h[i] = gs->s[i] * acc[i];
      gs->hn0 = nrm;
    } else if (mode == DM_BNORM) {
      gs->bnorm = nrm;
    } else if (mode == DM_MBNORM) {
      gs->mbnorm = nrm;
    } else {  // DM_RNORM: _safe_normalize of the preconditioned residual
      const bool use = nrm > gs->eps;
      gs->s[0] = use ? 1.0 / nrm : 0.0;
      gs->rnorm = use ? nrm : 0.0;
    }
  }
}

template <typename T>
__global__ void dots_kernel(const T* __restrict__ Vb, size_t stride, int m, const T* __restrict__ w, size_t n,
                            double* partial, GState* gs, int mode, int gated) {
  if (gated && gs->active == 0) return;
  dots_body<T>(Vb, stride, m, w, n, partial, gs, mode, blockIdx.x, gridDim.x);
}

enum UpdMode { UM_NONE = 0, UM_ARNOLDI = 1 };

// x64 += sum_{i < min(m, kdone)} coef_i V_i with a float64 solution (the
// end-of-cycle update of GMRES with iterative refinement)
template <typename T>
__device__ __forceinline__ void update_x64_body(const T* __restrict__ Vb, size_t stride, int m,
                                                double* __restrict__ x, size_t n, const GState* gs, int bid,
                                                int nblk) {
  __shared__ double cf[GM_MAXR + 2];
  const int mm = min(m, gs->kdone);
  for (int q = threadIdx.x; q < mm; q += blockDim.x) cf[q] = gs->coef[q];
  __syncthreads();
  // CH 16-byte chunks of T per thread and tile (n is a multiple of 64: the
  // packed fields are padded), every chunk's loads in flight together; per
  // element the sum runs in the order acc = x, acc += coef_i V_i (i = 0, 1, ..)
  constexpr int VN = V16<T>::n;
  constexpr int E = CH * VN;
  const int tid = threadIdx.x, nt = blockDim.x;
  const size_t tile = (size_t)nt * E;
  for (size_t base = (size_t)bid * tile; base < n; base += (size_t)nblk * tile) {
    double acc[E];
    bool ok[CH];
#pragma unroll
    for (int c = 0; c < CH; ++c) {
      const size_t off = base + ((size_t)c * nt + tid) * VN;
      ok[c] = off < n;
#pragma unroll
      for (int e = 0; e < VN; ++e) acc[c * VN + e] = ok[c] ? x[off + e] : 0.0;
    }
    for (int i = 0; i < mm; ++i) {
      const T* __restrict__ Vi = Vb + (size_t)i * stride;
      const double ci = cf[i];
#pragma unroll
      for (int c = 0; c < CH; ++c) {
        if (!ok[c]) continue;
        const size_t off = base + ((size_t)c * nt + tid) * VN;
        T vr[VN];
        load16(Vi + off, vr);
#pragma unroll
        for (int e = 0; e < VN; ++e) acc[c * VN + e] += ci * (double)vr[e];
      }
    }
#pragma unroll
    for (int c = 0; c < CH; ++c) {
      if (!ok[c]) continue;
      const size_t off = base + ((size_t)c * nt + tid) * VN;
#pragma unroll
      for (int e = 0; e < VN; ++e) x[off + e] = acc[c * VN + e];
    }
  }
}
template <typename T>
__global__ void __launch_bounds__(256) update_x64_kernel(const T* __restrict__ Vb, size_t stride, int m,
                                                         double* __restrict__ x, size_t n, const GState* gs) {
  update_x64_body<T>(Vb, stride, m, x, n, gs, blockIdx.x, gridDim.x);
}

// w <- w + sign * sum_{i<m'} coef_i V_i with coef from gs->coef (UM_NONE,
// m' = min(m, kdone) when limit_kdone) or coef_i = h_i s_i (UM_ARNOLDI),
// then optionally finish the Arnoldi step j = m - 1.
template <typename T>
__device__ __forceinline__ void update_body(const T* __restrict__ Vb, size_t stride, int m, T* __restrict__ w,
                                            size_t n, double sign, double* partial, GState* gs, int mode,
                                            int limit_kdone, int bid, int nblk) {
  __shared__ double cf[GM_MAXR + 2];
  __shared__ double red[GT / 32];
  int mm = m;
  if (limit_kdone) mm = min(m, gs->kdone);
  for (int q = threadIdx.x; q < mm; q += blockDim.x)
    cf[q] = sign * (mode == UM_ARNOLDI ? gs->h[q] * gs->s[q] : gs->coef[q]);
  __syncthreads();
  constexpr int VN = V16<T>::n;
  constexpr int E = CH * VN;
  const size_t tile = (size_t)GT * E;
  double sq = 0.0;
  for (size_t base = (size_t)bid * tile; base < n; base += (size_t)nblk * tile) {
    T wr[E];
    bool ok[CH];
#pragma unroll
    for (int c = 0; c < CH; ++c) {
      const size_t off = base + ((size_t)c * GT + threadIdx.x) * VN;
      ok[c] = off < n;
      if (ok[c]) load16(w + off, wr + c * VN);
    }
    for (int i = 0; i < mm; ++i) {
      const T* __restrict__ Vi = Vb + (size_t)i * stride;
      const T ci = (T)cf[i];
#pragma unroll
      for (int c = 0; c < CH; ++c) {
        if (!ok[c]) continue;
        const size_t off = base + ((size_t)c * GT + threadIdx.x) * VN;
        T vr[VN];
        load16(Vi + off, vr);
#pragma unroll
        for (int e = 0; e < VN; ++e) wr[c * VN + e] += ci * vr[e];
      }
    }
#pragma unroll
    for (int c = 0; c < CH; ++c) {
      if (!ok[c]) continue;
      const size_t off = base + ((size_t)c * GT + threadIdx.x) * VN;
      store16(w + off, wr + c * VN);
#pragma unroll
      for (int e = 0; e < VN; ++e) sq += (double)wr[c * VN + e] * (double)wr[c * VN + e];
    }
  }
  if (mode != UM_ARNOLDI) return;
  sq = warp_sum(sq);
  if ((threadIdx.x & 31) == 0) red[threadIdx.x >> 5] = sq;
  __syncthreads();
  if (threadIdx.x == 0) {
    double s = 0.0;
    for (int q = 0; q < GT / 32; ++q) s += red[q];
    partial[bid] = s;
  }
  if (!last_block(&gs->counter, (unsigned)nblk)) return;
  if (threadIdx.x >= 32) return;
  double tot = 0.0;  // warp 0 sums the blocks' partials
  for (int b = threadIdx.x; b < nblk; b += 32) tot += partial[b];
  tot = warp_sum(tot);
  if (threadIdx.x != 0) return;
  gs->counter = 0;
  // ---- finish Arnoldi step j (jax _kth_arnoldi_iteration) ----
  const int j = m - 1;
  const int R = gs->restart;
  double vn1 = sqrt(tot);
  const double thresh = gs->eps * gs->hn0;
  if (vn1 > thresh) {
    gs->s[j + 1] = 1.0 / vn1;
  } else {
    gs->s[j + 1] = 0.0;
    vn1 = 0.0;
  }
  double row[GM_MAXR + 1];
  for (int q = 0; q <= R; ++q) row[q] = 0.0;
  for (int q = 0; q <= j; ++q) row[q] = gs->h[q];
  row[j + 1] = vn1;
  gs->kdone = j + 1;
  if (gs->method == 0) {  // batched: H[j, :] = h
    for (int q = 0; q <= R; ++q) gs->H[j][q] = row[q];
    if (vn1 == 0.0) { gs->breakdown = 1; gs->active = 0; }
  } else {  // incremental: rotate into R, update beta
    for (int i = 0; i < j; ++i) {
      const double c = gs->givens[i][0], s = gs->givens[i][1];
      const double x1 = row[i], y1 = row[i + 1];
      row[i] = c * x1 - s * y1;
      row[i + 1] = s * x1 + c * y1;
    }
    // _givens_rotation(a, b)
    const double a = row[j], b = row[j + 1];
    double cs, sn;
    if (b == 0.0) {
      cs = 1.0; sn = 0.0;
    } else if (fabs(a) < fabs(b)) {
      const double t = -a / b, r = 1.0 / sqrt(1.0 + t * t);
      cs = r * t; sn = r;
    } else {
      const double t = -b / a, r = 1.0 / sqrt(1.0 + t * t);
      cs = r; sn = r * t;
    }
    gs->givens[j][0] = cs;
    gs->givens[j][1] = sn;
    row[j] = cs * a - sn * b;
    row[j + 1] = sn * a + cs * b;
    for (int q = 0; q <= R; ++q) gs->H[j][q] = row[q];
    const double b0 = gs->beta[j], b1 = gs->beta[j + 1];
    gs->beta[j] = cs * b0 - sn * b1;
    gs->beta[j + 1] = sn * b0 + cs * b1;
    gs->err = fabs(gs->beta[j + 1]);
    if (!(gs->err > gs->ptol)) gs->active = 0;
  }
}
template <typename T>
__global__ void __launch_bounds__(GT) update_kernel(const T* __restrict__ Vb, size_t stride, int m,
                                                    T* __restrict__ w, size_t n, double sign, double* partial,
                                                    GState* gs, int mode, int gated, int limit_kdone) {
  if (gated && gs->active == 0) return;
  update_body<T>(Vb, stride, m, w, n, sign, partial, gs, mode, limit_kdone, blockIdx.x, gridDim.x);
}

__device__ void setup_state(GState* gs, double eps, double tol, double atol_in, int restart, int method) {
  gs->eps = eps;
  gs->tol = tol;
  gs->atol_in = atol_in;
  gs->restart = restart;
  gs->method = method;
  gs->counter = 0;
  gs->active = 1;
  gs->kdone = 0;
  gs->breakdown = 0;
  gs->cycles = 0;
  gs->steps = 0;
  for (int q = 0; q < GM_MAXR + 2; ++q) gs->s[q] = 0.0;
}
__global__ void setup_kernel(GState* gs, double eps, double tol, double atol_in, int restart, int method) {
  setup_state(gs, eps, tol, atol_in, restart, method);
}

// Graph mode: after a residual, count the finished cycle and set the WHILE
// condition: another cycle while ||M r|| > atol and cycles < maxiter.
__global__ void gate_kernel(GState* gs, cudaGraphConditionalHandle h, int maxiter, int after_cycle) {
  if (after_cycle) {
    gs->cycles += 1;
    gs->steps += gs->kdone;
  }
  const bool more = (gs->rnorm > gs->atol) && (gs->cycles < maxiter);
  cudaGraphSetConditional(h, more ? 1u : 0u);
}

__device__ void info_state(const GState* gs, GDevInfo* o) {
  o->cycles = gs->cycles;
  o->arnoldi_steps = gs->steps;
  o->converged = (gs->rnorm <= gs->atol) ? 1 : 0;
  o->pad = 0;
  o->residual_norm = gs->rnorm;
  o->atol = gs->atol;
  o->b_norm = gs->bnorm;
}
__global__ void info_kernel(const GState* gs, GDevInfo* o) { info_state(gs, o); }

__device__ void init_tol_state(GState* gs) {
  // atol = max(tol ||b||, atol); ptol = ||M b|| min(1, atol / ||b||)
  gs->atol = fmax(gs->tol * gs->bnorm, gs->atol_in);
  gs->ptol = gs->mbnorm * fmin(1.0, gs->atol / gs->bnorm);
}
__global__ void init_tol_kernel(GState* gs) { init_tol_state(gs); }

__device__ void begin_cycle_state(GState* gs) {
  const int R = gs->restart;
  for (int q = threadIdx.x; q < R * (GM_MAXR + 1); q += blockDim.x) {
    const int r = q / (GM_MAXR + 1), c = q % (GM_MAXR + 1);
    gs->H[r][c] = (r == c) ? 1.0 : 0.0;  // eye(restart, restart + 1)
  }
  for (int q = threadIdx.x; q <= R; q += blockDim.x) gs->beta[q] = 0.0;
  for (int q = threadIdx.x; q < R; q += blockDim.x) { gs->givens[q][0] = 0.0; gs->givens[q][1] = 0.0; }
  __syncthreads();
  if (threadIdx.x == 0) {
    gs->beta[0] = gs->rnorm;
    gs->err = gs->rnorm;
    gs->active = 1;
    gs->kdone = 0;
    gs->breakdown = 0;
  }
}
__global__ void begin_cycle_kernel(GState* gs) { begin_cycle_state(gs); }

// y from the cycle's small problem; coef_i = y_i s_i.
__device__ void small_solve_state(GState* gs) {
  extern __shared__ double a2[];  // R * R
  const int R = gs->restart;
  __shared__ double b2[GM_MAXR];
  __shared__ double y[GM_MAXR];
  if (gs->method == 0) {
    // _lstsq(H.T, beta): normal equations (H H^T) y = H beta, Cholesky solve
    for (int q = threadIdx.x; q < R * R; q += blockDim.x) {
      const int p = q / R, r = q % R;
      double s = 0.0;
      for (int c = 0; c <= R; ++c) s += gs->H[p][c] * gs->H[r][c];
      a2[q] = s;
    }
    for (int p = threadIdx.x; p < R; p += blockDim.x) {
      double s = 0.0;
      for (int c = 0; c <= R; ++c) s += gs->H[p][c] * gs->beta[c];
      b2[p] = s;
    }
    __syncthreads();
    // right-looking Cholesky, lower factor stored in a2
    for (int k = 0; k < R; ++k) {
      if (threadIdx.x == 0) a2[k * R + k] = sqrt(a2[k * R + k]);
      __syncthreads();
      const double dkk = a2[k * R + k];
      for (int i = k + 1 + threadIdx.x; i < R; i += blockDim.x) a2[i * R + k] /= dkk;
      __syncthreads();
      for (int q = threadIdx.x; q < (R - k - 1) * (R - k - 1); q += blockDim.x) {
        const int i = k + 1 + q / (R - k - 1), jj = k + 1 + q % (R - k - 1);
        if (jj <= i) a2[i * R + jj] -= a2[i * R + k] * a2[jj * R + k];
      }
      __syncthreads();
    }
    if (threadIdx.x == 0) {
      for (int i = 0; i < R; ++i) {  // L z = b2
        double s = b2[i];
        for (int k = 0; k < i; ++k) s -= a2[i * R + k] * y[k];
        y[i] = s / a2[i * R + i];
      }
      for (int i = R - 1; i >= 0; --i) {  // L^T y = z
        double s = y[i];
        for (int k = i + 1; k < R; ++k) s -= a2[k * R + i] * y[k];
        y[i] = s / a2[i * R + i];
      }
      for (int i = 0; i < R; ++i) gs->coef[i] = y[i] * gs->s[i];
    }
  } else {
    if (threadIdx.x == 0) {
      // back substitution with the rotated rows: sum_j R[j][i] y_j = beta_i
      const int kd = gs->kdone;
      for (int i = kd - 1; i >= 0; --i) {
        double s = gs->beta[i];
        for (int jj = i + 1; jj < kd; ++jj) s -= gs->H[jj][i] * y[jj];
        y[i] = s / gs->H[i][i];
      }
      for (int i = 0; i < R; ++i) gs->coef[i] = (i < kd) ? y[i] * gs->s[i] : 0.0;
    }
  }
}
__global__ void small_solve_kernel(GState* gs) { small_solve_state(gs); }

__global__ void snapshot_kernel(const GState* gs, GHostView* v) {
  v->rnorm = gs->rnorm;
  v->atol = gs->atol;
  v->bnorm = gs->bnorm;
  v->kdone = gs->kdone;
}

// ---------------------------------------------------------------------------
// grouped launches over ensemble members: flat block b runs block
// (b - first[m]) of member m's standalone launch (sisl_group.cuh)
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ T* gvec(const GroupMember<T>& g, int v) {
  return g.vec + (size_t)v * g.npad;
}

template <typename T>
__global__ void group_dots_kernel(GroupMember<T>* mem, const int* __restrict__ first, int M, int m, int wv,
                                  int mode, int gated) {
  const int b = blockIdx.x;
  const int mi = group_find(first, M, b);
  const GroupMember<T>& g = mem[mi];
  if (!g.running || (gated && g.gs->active == 0)) return;
  const int f0 = first[mi];
  dots_body<T>(gvec(g, GV_V0), g.npad, m, gvec(g, wv), g.npad, g.partial, g.gs, mode, b - f0, first[mi + 1] - f0);
}

// final_x = 0: Arnoldi projection of V_m out of V_0 .. V_{m-1} (gated);
// final_x = 1: x += sum coef_i V_i over the cycle's basis
template <typename T>
__global__ void __launch_bounds__(GT) group_update_kernel(GroupMember<T>* mem, const int* __restrict__ first, int M,
                                                          int m, int final_x) {
  const int b = blockIdx.x;
  const int mi = group_find(first, M, b);
  const GroupMember<T>& g = mem[mi];
  if (!g.running) return;
  const int f0 = first[mi], nb = first[mi + 1] - f0;
  if (final_x) {
    update_body<T>(gvec(g, GV_V0), g.npad, m, gvec(g, GV_X), g.npad, 1.0, g.partial, g.gs, UM_NONE, 1, b - f0, nb);
  } else {
    if (g.gs->active == 0) return;
    update_body<T>(gvec(g, GV_V0), g.npad, m, gvec(g, GV_V0 + m), g.npad, -1.0, g.partial, g.gs, UM_ARNOLDI, 0,
                   b - f0, nb);
  }
}

template <typename T>
__global__ void __launch_bounds__(256) group_update_x64_kernel(GroupMember<T>* mem, const int* __restrict__ first,
                                                               int M, int m) {
  const int b = blockIdx.x;
  const int mi = group_find(first, M, b);
  const GroupMember<T>& g = mem[mi];
  if (!g.running) return;
  const int f0 = first[mi];
  update_x64_body<T>(gvec(g, GV_V0), g.npad, m, g.x64, g.npad, g.gs, b - f0, first[mi + 1] - f0);
}

// 0: b64 = b, x64 = x, r64 = 0; 1: residual r64 -> V_0 (u, v) | z (w, pi,
// eta_dot); 2: x = x64 (after the loop: every member); 3: V_1 (u, v) = b (u, v);
// 4: transposed residual r64 -> z
template <typename T>
__global__ void __launch_bounds__(256) group_convert_kernel(GroupMember<T>* mem, const int* __restrict__ first,
                                                            int M, int mode) {
  const int b = blockIdx.x;
  const int mi = group_find(first, M, b);
  const GroupMember<T>& g = mem[mi];
  if (mode != 2 && !g.running) return;
  const size_t f0 = first[mi], nb = first[mi + 1] - f0;
  const size_t n = (mode == 3) ? g.off[2] : g.npad;
  const size_t step = nb * blockDim.x;
  T* x = gvec(g, GV_X);
  const T* bv = gvec(g, GV_B);
  T* v0 = gvec(g, GV_V0);
  T* z = gvec(g, GV_Z);
  for (size_t e = (b - f0) * (size_t)blockDim.x + threadIdx.x; e < n; e += step) {
    if (mode == 0) {
      g.b64[e] = (double)bv[e];
      g.x64[e] = (double)x[e];
      g.r64[e] = 0.0;
    } else if (mode == 1) {
      (e < g.off[2] ? v0 : z)[e] = (T)g.r64[e];
    } else if (mode == 2) {
      x[e] = (T)g.x64[e];
    } else if (mode == 4) {
      z[e] = (T)g.r64[e];
    } else {
      v0[g.npad + e] = bv[e];
    }
  }
}

// one thread per member
template <typename T>
__global__ void group_setup_kernel(GroupMember<T>* mem, int M, int R, int method, int transpose) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m >= M) return;
  GroupMember<T>& g = mem[m];
  setup_state(g.gs, g.eps, transpose ? g.tol_t : g.tol, g.atol_in, R, method);
  g.running = 1;
}
template <typename T>
__global__ void group_init_tol_kernel(GroupMember<T>* mem, int M) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < M) init_tol_state(mem[m].gs);
}
template <typename T>
__global__ void group_info_kernel(GroupMember<T>* mem, int M, int solve) {
  const int m = blockIdx.x * blockDim.x + threadIdx.x;
  if (m < M && mem[m].info[solve]) info_state(mem[m].gs, mem[m].info[solve]);
}
// one block per member
template <typename T>
__global__ void group_begin_cycle_kernel(GroupMember<T>* mem) {
  const GroupMember<T>& g = mem[blockIdx.x];
  if (g.running) begin_cycle_state(g.gs);
}
template <typename T>
__global__ void group_small_solve_kernel(GroupMember<T>* mem) {
  const GroupMember<T>& g = mem[blockIdx.x];
  if (g.running) small_solve_state(g.gs);
}
// one block: count the finished cycle of every running member, decide which
// members continue, set the WHILE condition while any does
template <typename T>
__global__ void group_gate_kernel(GroupMember<T>* mem, int M, cudaGraphConditionalHandle h, int after_cycle) {
  int any = 0;
  for (int m = threadIdx.x; m < M; m += blockDim.x) {
    GroupMember<T>& g = mem[m];
    GState* gs = g.gs;
    if (after_cycle && g.running) {
      gs->cycles += 1;
      gs->steps += gs->kdone;
    }
    const int more = g.running && (gs->rnorm > gs->atol) && (gs->cycles < g.maxiter);
    g.running = more;
    any |= more;
  }
  any = __syncthreads_or(any);
  if (threadIdx.x == 0) cudaGraphSetConditional(h, any ? 1u : 0u);
}

int flat_grid(size_t n, int elems_per_block) {
  size_t b = (n + elems_per_block - 1) / elems_per_block;
  if (b > (size_t)GM_MAXBLOCKS) b = GM_MAXBLOCKS;
  if (b < 1) b = 1;
  return (int)b;
}

// Grid of a grid-stride Krylov kernel: every block resident at once (one
// wave, no tail of a partial second wave), at most GM_MAXBLOCKS.
int resident_grid(const void* fn, int threads, size_t smem, size_t n, int elems_per_block) {
  static std::atomic<int> sms[SMEM_LIMIT_DEVICES];  // SM count per device, found once
  int dev = 0;
  cudaGetDevice(&dev);
  const bool slot = dev >= 0 && dev < SMEM_LIMIT_DEVICES;
  int ns = slot ? sms[dev].load() : 0;
  if (ns == 0) {
    if (cudaDeviceGetAttribute(&ns, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess || ns < 1) ns = 148;
    if (slot) sms[dev].store(ns);
  }
  int per_sm = 0;
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, fn, threads, smem) != cudaSuccess || per_sm < 1)
    per_sm = 1;
  size_t want = (n + elems_per_block - 1) / elems_per_block;
  size_t cap = (size_t)per_sm * ns;
  if (cap > (size_t)GM_MAXBLOCKS) cap = GM_MAXBLOCKS;
  if (want > cap) want = cap;
  if (want < 1) want = 1;
  return (int)want;
}

}  // namespace

// resident grid of the float64 solution update (tiles of 256 threads x CH 16-byte chunks)
template <typename T>
int gm_x64_blocks_t(size_t n) {
  return resident_grid((const void*)update_x64_kernel<T>, 256, 0, n, 256 * CH * V16<T>::n);
}

// ---------------------------------------------------------------------------
// host wrappers
// ---------------------------------------------------------------------------
// shared memory of the dots kernel: (m + 1) per-warp slots of 8 warps
constexpr size_t DOTS_SMEM_MAX = (size_t)(GM_MAXR + 1) * 8 * sizeof(double);
constexpr int DOTS_THREADS = 256;

template <typename T>
void gm_dots(const T* Vb, size_t stride, int m, const T* w, size_t n, double* partial, GState* gs, int mode,
             int gated, cudaStream_t st) {
  static SmemLimit attr_bytes;  // per instantiation
  ensure_smem_limit((const void*)dots_kernel<T>, attr_bytes, (size_t)DOTS_SMEM_MAX);
  const int nt = DOTS_THREADS;
  constexpr int E = CH * V16<T>::n;
  const size_t smem = (size_t)(m + 1) * (nt / 32) * sizeof(double);
  const int g = resident_grid((const void*)dots_kernel<T>, nt, smem, n, nt * E);
  dots_kernel<T><<<g, nt, smem, st>>>(Vb, stride, m, w, n, partial, gs, mode, gated);
}

template <typename T>
void gm_update(const T* Vb, size_t stride, int m, T* w, size_t n, double sign, double* partial, GState* gs,
               int mode, int gated, int limit_kdone, cudaStream_t st) {
  constexpr int E = CH * V16<T>::n;
  const int g = resident_grid((const void*)update_kernel<T>, GT, 0, n, GT * E);
  update_kernel<T><<<g, GT, 0, st>>>(Vb, stride, m, w, n, sign, partial, gs, mode, gated, limit_kdone);
}

template <typename T>
void gm_update_x64(const T* Vb, size_t stride, int m, double* x, size_t n, const GState* gs, cudaStream_t st) {
  update_x64_kernel<T><<<gm_x64_blocks_t<T>(n), 256, 0, st>>>(Vb, stride, m, x, n, gs);
}

void gm_setup(GState* gs, double eps, double tol, double atol_in, int restart, int method, cudaStream_t st) {
  setup_kernel<<<1, 1, 0, st>>>(gs, eps, tol, atol_in, restart, method);
}
void gm_init_tol(GState* gs, cudaStream_t st) { init_tol_kernel<<<1, 1, 0, st>>>(gs); }
void gm_gate(GState* gs, cudaGraphConditionalHandle h, int maxiter, int after_cycle, cudaStream_t st) {
  gate_kernel<<<1, 1, 0, st>>>(gs, h, maxiter, after_cycle);
}
void gm_info(const GState* gs, GDevInfo* o, cudaStream_t st) { info_kernel<<<1, 1, 0, st>>>(gs, o); }
void gm_begin_cycle(GState* gs, cudaStream_t st) { begin_cycle_kernel<<<1, 256, 0, st>>>(gs); }
void gm_small_solve(GState* gs, int restart, cudaStream_t st) {
  const size_t smem = (size_t)restart * restart * sizeof(double);
  static SmemLimit attr_bytes;
  ensure_smem_limit((const void*)small_solve_kernel, attr_bytes, (size_t)GM_MAXR * GM_MAXR * sizeof(double));
  small_solve_kernel<<<1, 256, smem, st>>>(gs);
}
void gm_snapshot(const GState* gs, GHostView* v, cudaStream_t st) { snapshot_kernel<<<1, 1, 0, st>>>(gs, v); }

// ---------------------------------------------------------------------------
// grouped host wrappers
// ---------------------------------------------------------------------------
template <typename T>
int gm_dots_threads(int m) {
  (void)m;
  return DOTS_THREADS;
}
template <typename T>
int gm_dots_blocks(int m, size_t n) {
  static SmemLimit attr_bytes;
  ensure_smem_limit((const void*)dots_kernel<T>, attr_bytes, (size_t)DOTS_SMEM_MAX);
  const int nt = gm_dots_threads<T>(m);
  constexpr int E = CH * V16<T>::n;
  return resident_grid((const void*)dots_kernel<T>, nt, (size_t)(m + 1) * (nt / 32) * sizeof(double), n, nt * E);
}
template <typename T>
int gm_update_blocks(size_t n) {
  constexpr int E = CH * V16<T>::n;
  return resident_grid((const void*)update_kernel<T>, GT, 0, n, GT * E);
}
int gm_x64_blocks(size_t n) { return gm_x64_blocks_t<float>(n); }
int group_convert_blocks(size_t n) { return flat_grid(n, 256 * 8) < 296 ? flat_grid(n, 256 * 8) : 296; }

template <typename T>
void grp_setup(const GroupLaunch<T>& g, int transpose, cudaStream_t st) {
  group_setup_kernel<T><<<(g.M + 127) / 128, 128, 0, st>>>(g.mem, g.M, g.R, g.method, transpose);
}
template <typename T>
void grp_dots(const GroupLaunch<T>& g, int m, int w, int mode, int gated, cudaStream_t st) {
  static SmemLimit attr_bytes;
  ensure_smem_limit((const void*)group_dots_kernel<T>, attr_bytes, (size_t)DOTS_SMEM_MAX);
  const int nt = gm_dots_threads<T>(m);
  const size_t smem = (size_t)(m + 1) * (nt / 32) * sizeof(double);
  group_dots_kernel<T><<<g.blocks(GT_DOTS0 + m), nt, smem, st>>>(g.mem, g.row(GT_DOTS0 + m), g.M, m, w, mode, gated);
}
template <typename T>
void grp_update_arnoldi(const GroupLaunch<T>& g, int m, cudaStream_t st) {
  group_update_kernel<T><<<g.blocks(GT_UPD), GT, 0, st>>>(g.mem, g.row(GT_UPD), g.M, m, 0);
}
template <typename T>
void grp_update_x(const GroupLaunch<T>& g, cudaStream_t st) {
  if (g.refine) group_update_x64_kernel<T><<<g.blocks(GT_X64), 256, 0, st>>>(g.mem, g.row(GT_X64), g.M, g.R);
  else group_update_kernel<T><<<g.blocks(GT_UPD), GT, 0, st>>>(g.mem, g.row(GT_UPD), g.M, g.R, 1);
}
template <typename T>
void grp_convert(const GroupLaunch<T>& g, int mode, cudaStream_t st) {
  group_convert_kernel<T><<<g.blocks(GT_CVT), 256, 0, st>>>(g.mem, g.row(GT_CVT), g.M, mode);
}
template <typename T>
void grp_init_tol(const GroupLaunch<T>& g, cudaStream_t st) {
  group_init_tol_kernel<T><<<(g.M + 127) / 128, 128, 0, st>>>(g.mem, g.M);
}
template <typename T>
void grp_begin_cycle(const GroupLaunch<T>& g, cudaStream_t st) {
  group_begin_cycle_kernel<T><<<g.M, 256, 0, st>>>(g.mem);
}
template <typename T>
void grp_small_solve(const GroupLaunch<T>& g, cudaStream_t st) {
  static SmemLimit attr_bytes;
  ensure_smem_limit((const void*)group_small_solve_kernel<T>, attr_bytes, (size_t)GM_MAXR * GM_MAXR * sizeof(double));
  group_small_solve_kernel<T><<<g.M, 256, (size_t)g.R * g.R * sizeof(double), st>>>(g.mem);
}
template <typename T>
void grp_gate(const GroupLaunch<T>& g, cudaGraphConditionalHandle h, int after_cycle, cudaStream_t st) {
  group_gate_kernel<T><<<1, 256, 0, st>>>(g.mem, g.M, h, after_cycle);
}
template <typename T>
void grp_info(const GroupLaunch<T>& g, int solve, cudaStream_t st) {
  group_info_kernel<T><<<(g.M + 127) / 128, 128, 0, st>>>(g.mem, g.M, solve);
}

#define SISL_GROUP_INST(T)                                                                           \
  template int gm_dots_threads<T>(int);                                                              \
  template int gm_dots_blocks<T>(int, size_t);                                                       \
  template int gm_update_blocks<T>(size_t);                                                          \
  template void grp_setup<T>(const GroupLaunch<T>&, int, cudaStream_t);                              \
  template void grp_dots<T>(const GroupLaunch<T>&, int, int, int, int, cudaStream_t);                \
  template void grp_update_arnoldi<T>(const GroupLaunch<T>&, int, cudaStream_t);                     \
  template void grp_update_x<T>(const GroupLaunch<T>&, cudaStream_t);                                \
  template void grp_convert<T>(const GroupLaunch<T>&, int, cudaStream_t);                            \
  template void grp_init_tol<T>(const GroupLaunch<T>&, cudaStream_t);                                \
  template void grp_begin_cycle<T>(const GroupLaunch<T>&, cudaStream_t);                             \
  template void grp_small_solve<T>(const GroupLaunch<T>&, cudaStream_t);                             \
  template void grp_gate<T>(const GroupLaunch<T>&, cudaGraphConditionalHandle, int, cudaStream_t);   \
  template void grp_info<T>(const GroupLaunch<T>&, int, cudaStream_t);
SISL_GROUP_INST(float)
SISL_GROUP_INST(double)
#undef SISL_GROUP_INST

template void gm_dots<float>(const float*, size_t, int, const float*, size_t, double*, GState*, int, int,
                             cudaStream_t);
template void gm_dots<double>(const double*, size_t, int, const double*, size_t, double*, GState*, int, int,
                              cudaStream_t);
template void gm_update<float>(const float*, size_t, int, float*, size_t, double, double*, GState*, int, int,
                               int, cudaStream_t);
template void gm_update<double>(const double*, size_t, int, double*, size_t, double, double*, GState*, int,
                                int, int, cudaStream_t);
template void gm_update_x64<float>(const float*, size_t, int, double*, size_t, const GState*, cudaStream_t);
template void gm_update_x64<double>(const double*, size_t, int, double*, size_t, const GState*, cudaStream_t);

}  // namespace sisl
