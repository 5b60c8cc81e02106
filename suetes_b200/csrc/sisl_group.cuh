// Grouped GMRES over an ensemble: every Krylov phase of all members' solves
// runs as ONE launch that walks a member/block table, so the small members
// of an uneven ensemble share each launch with the large ones instead of
// each issuing its own under-filled kernels.
//
// A grouped launch's flat block b belongs to member m with
// first[m] <= b < first[m + 1] and acts as block (b - first[m]) of the
// standalone launch of that member: the same per-member partition, so every
// member's reductions (and therefore its iterates and solution) are the same
// bits as its own solve's.  Convergence stays per member: `running` drops to
// 0 when a member's restart loop ends, after which its blocks return at once.
#pragma once

#include <vector>

#include "sisl_gmres.cuh"

namespace sisl {

template <typename T>
struct GroupMember {
  Dims d;
  Coef<T> c;
  Coef<double> c64;  // float64 operator of the iterative refinement (float32 cores)
  T* vec;            // (R + 4) packed vectors of npad elements: x, b, z, V_0, V_1, ..
  double *x64, *b64, *r64;
  T* tmp;            // mass-point scratch of the transposed matvec
  double* tmp64;     // its float64 counterpart (refinement)
  size_t npad;
  size_t off[5];
  GState* gs;
  double* partial;
  GDevInfo* info[2];  // statistics of the step's two solves
  double eps, tol, atol_in;
  double tol_t;      // tolerance of the transposed solves
  int maxiter;
  int running;  // 1 while this member's restart loop continues (device-written)
};

// rows of the block table: first block of every member, M + 1 entries each
enum GroupTable {
  GT_MV = 0,  // column-march matvec
  GT_PC,      // pipelined column preconditioner
  GT_UPD,     // multi-axpy (+ norm)
  GT_X64,     // float64 solution update
  GT_CVT,     // packed conversions and copies
  GT_ATG,     // transposed matvec, stage 1 (mass points)
  GT_ATM,     // transposed matvec, stage 2 (union box)
  GT_PTM,     // transposed preconditioner, 32-column tiles
  GT_PTU,     // transposed preconditioner, u and v faces
  GT_DOTS0    // GT_DOTS0 + m: projections onto m basis vectors
};
inline int group_tables(int R) { return GT_DOTS0 + R + 1; }

template <typename T>
struct GroupLaunch {
  GroupMember<T>* mem;     // device, M entries
  const int* first;        // device, group_tables(R) rows of M + 1
  std::vector<int> first_h;  // host copy
  std::vector<int> nz_h;     // members' level counts (preconditioner shared memory)
  int M = 0, R = 0, method = 0;
  bool refine = false;
  const int* row(int t) const { return first + (size_t)t * (M + 1); }
  int blocks(int t) const { return first_h[(size_t)t * (M + 1) + M]; }
};

// member owning flat block b: the largest m with first[m] <= b
__device__ __forceinline__ int group_find(const int* __restrict__ first, int M, int b) {
  int lo = 0, hi = M - 1;
  while (lo < hi) {
    const int mid = (lo + hi + 1) >> 1;
    if (__ldg(first + mid) <= b) lo = mid;
    else hi = mid - 1;
  }
  return lo;
}

// vectors a grouped kernel reads or writes, by index into the member's packed vectors
enum GroupVec { GV_X = 0, GV_B = 1, GV_Z = 2, GV_V0 = 3 };  // GV_V0 + i: basis vector i

// per-member block counts of the standalone launches
template <typename T> int gm_dots_threads(int m);
template <typename T> int gm_dots_blocks(int m, size_t n);
template <typename T> int gm_update_blocks(size_t n);
int gm_x64_blocks(size_t n);
int group_matvec_blocks(const Dims& d);
int group_precond_blocks(const Dims& d);
int group_convert_blocks(size_t n);
int group_at_blocks(const Dims& d, int stage);
int group_pt_blocks(const Dims& d, int stage);

// Krylov phases.  Every launch skips members whose `running` is 0; gated
// launches also skip members whose current cycle has stopped (gs->active).
// transpose: the tolerance of the transposed solves (tol_t)
template <typename T>
void grp_setup(const GroupLaunch<T>& g, int transpose, cudaStream_t st);
// result over basis vectors V_0 .. V_{m-1} and vector `w` (GroupVec), mode as gm_dots
template <typename T>
void grp_dots(const GroupLaunch<T>& g, int m, int w, int mode, int gated, cudaStream_t st);
// Arnoldi: V_{m} -= sum_{i<m} h_i s_i V_i and finish step m - 1 (gated);
// final: x += sum_{i<min(R, kdone)} coef_i V_i (float64 x with refinement)
template <typename T>
void grp_update_arnoldi(const GroupLaunch<T>& g, int m, cudaStream_t st);
template <typename T>
void grp_update_x(const GroupLaunch<T>& g, cudaStream_t st);
// packed conversions: 0 b64 = b, x64 = x, r64 = 0; 1 residual r64 -> V_0
// (u, v) | z (w, pi, eta); 2 x = x64; 3 V_1 (u, v) = b (u, v); 4 r64 -> z
template <typename T>
void grp_convert(const GroupLaunch<T>& g, int mode, cudaStream_t st);
template <typename T>
void grp_init_tol(const GroupLaunch<T>& g, cudaStream_t st);
template <typename T>
void grp_begin_cycle(const GroupLaunch<T>& g, cudaStream_t st);
template <typename T>
void grp_small_solve(const GroupLaunch<T>& g, cudaStream_t st);
// another cycle for member m while rnorm > atol and cycles < maxiter; the
// WHILE condition is set while any member continues
template <typename T>
void grp_gate(const GroupLaunch<T>& g, cudaGraphConditionalHandle h, int after_cycle, cudaStream_t st);
template <typename T>
void grp_info(const GroupLaunch<T>& g, int solve, cudaStream_t st);
// matvec: mode 0 Arnoldi step j: V_j scaled by s_j -> V_{j+1} (u, v) | z;
// mode 1 residual b - A x -> V_0 (u, v) | z; mode 2 float64 residual
// b64 - A64 x64 -> r64 (refinement)
template <typename T>
void grp_matvec(const GroupLaunch<T>& g, int mode, int j, cudaStream_t st);
// preconditioner after the matvec: target V_t (u, v already there), w, pi,
// eta from z; gated for the Arnoldi steps (t >= 1); mode 1: M b -> V_1
template <typename T>
void grp_precond(const GroupLaunch<T>& g, int mode, int t, int gated, cudaStream_t st);
// transposed operators.  matvec^T: mode 0 Arnoldi step j (gated), V_j
// scaled by s_j -> z; mode 1 b - A^T x -> z; mode 2 b64 - A64^T x64 -> r64.
// preconditioner^T: mode 0 z -> V_t (gated when t >= 1); mode 1 b -> V_1
template <typename T>
void grp_matvec_t(const GroupLaunch<T>& g, int mode, int j, cudaStream_t st);
template <typename T>
void grp_precond_t(const GroupLaunch<T>& g, int mode, int t, int gated, cudaStream_t st);

}  // namespace sisl
