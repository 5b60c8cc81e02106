// C ABI and host runtime of the SISL timestep: the core object (precomputed
// coefficients), workspace carving, the GMRES driver loop and the step
// orchestration of SISLStepper3D.step (steppers.py:720-1073).
#include "../../include/sisl_b200.h"

#include <atomic>
#include <cmath>
#include <cstdio>
#include <cstring>
#include <new>
#include <vector>

#include "sisl_core.cuh"
#include "sisl_explicit.cuh"
#include "sisl_group.cuh"
#include "sisl_split.cuh"
#include "sisl_step_vjp.cuh"

using namespace sisl;

static std::atomic<int64_t> g_launches{0};
static thread_local char g_last_error[256] = "";

// Record a failing CUDA call for sisl_last_error; true when e is an error.
static bool cuda_failed(cudaError_t e, const char* what) {
  if (e == cudaSuccess) return false;
  snprintf(g_last_error, sizeof(g_last_error), "%s: %s (%s)", what, cudaGetErrorName(e), cudaGetErrorString(e));
  return true;
}
static_assert(sizeof(GDevInfo) == sizeof(SislSolveInfo), "device solve statistics mirror SislSolveInfo");

struct SislCore {
  SislGrid grid;
  SislParams prm;
  Dims d;
  Scalars s;
  void* coef_mem = nullptr;
  void* coef_ptr[C_COUNT];
  GHostView* hv = nullptr;  // pinned
  int timing_class = SISL_K_NONE;
  std::vector<cudaEvent_t> ev0, ev1;
  size_t ev_used = 0;
  double timed_bytes = 0.0;  // algorithmic bytes of the timed launches
  // adjoint (transposed) solve: tolerance (<= 0: the forward solver_tol) and
  // whether the cotangent is normalised before GMRES (see sisl_core_set_adjoint)
  double adj_tol = -1.0;
  int adj_normalize = 1;
  int adj_method = -1;  // GMRES variant of the transposed solve; < 0: the forward's
  // float32 cores: float64 coefficient set for GMRES with float64 iterative
  // refinement (outer residual and solution in float64), and its switch
  void* coef64_mem = nullptr;
  void* coef64_ptr[C_COUNT];
  int refine_on = 0;
  cudaStream_t cap_side = nullptr;  // side stream for conditional-node bodies while a graph is captured
};

namespace {

size_t esize(int dtype) { return dtype == SISL_F64 ? 8 : 4; }
size_t align256(size_t x) { return (x + 255) & ~(size_t)255; }
// a workspace the entry points can carve: present, large enough, and
// 16-byte aligned -- the arrays are carved at multiples of 256 bytes from
// its start, so each keeps the start's alignment, and the kernels' 16-byte
// vector loads and stores need that much (a misaligned one would fault)
inline bool ws_bad(const void* ws, size_t have, size_t need) {
  return !ws || ((uintptr_t)ws & 15) != 0 || have < need;
}
size_t pad64(size_t x) { return (x + 63) & ~(size_t)63; }

// Scoped launch bookkeeping: counts kernels and, for the selected class,
// brackets the launch with CUDA events on the launching stream.
struct KScope {
  SislCore* c;
  cudaStream_t st;
  bool timed;
  KScope(SislCore* core, int cls, cudaStream_t s, int nkernels = 1, double bytes = 0.0)
      : c(core), st(s), timed(false) {
    g_launches += nkernels;
    if (c && c->timing_class == cls && cls != SISL_K_NONE) {
      c->timed_bytes += bytes;
      if (c->ev_used == c->ev0.size()) {
        cudaEvent_t a, b;
        cudaEventCreate(&a);
        cudaEventCreate(&b);
        c->ev0.push_back(a);
        c->ev1.push_back(b);
      }
      cudaEventRecord(c->ev0[c->ev_used], st);
      timed = true;
    }
  }
  ~KScope() {
    if (timed) {
      cudaEventRecord(c->ev1[c->ev_used], st);
      c->ev_used++;
    }
  }
};

struct Carver {
  char* base;
  size_t off = 0;
  void* take(size_t bytes) {
    off = align256(off);
    void* p = base ? base + off : nullptr;
    off += bytes;
    return p;
  }
};

int check_cuda() {
  return cuda_failed(cudaGetLastError(), "kernel launch") ? SISL_ERR_CUDA : SISL_OK;
}

template <typename T>
Coef<T> coef_of(const SislCore* c) {
  T* a[C_COUNT];
  for (int q = 0; q < C_COUNT; ++q) a[q] = (T*)c->coef_ptr[q];
  return make_coef<T>(a, c->s);
}

Coef<double> coef64_of(const SislCore* c) {
  double* a[C_COUNT];
  for (int q = 0; q < C_COUNT; ++q) a[q] = (double*)c->coef64_ptr[q];
  return make_coef<double>(a, c->s);
}

// iterative refinement applies to float32 cores holding the float64 coefficients
template <typename T>
bool refining(const SislCore* c) {
  return sizeof(T) == 4 && c->refine_on && c->coef64_mem;
}

int loc_of_field(int q) {  // solver vector field -> stagger
  static const int L[5] = {LOC_U, LOC_V, LOC_W, LOC_M, LOC_W};
  return L[q];
}

// ---------------------------------------------------------------------------
// small utility kernels
// ---------------------------------------------------------------------------
// dst = src with pi scaled by pi_mul and eta_dot by dz_w (mode 1), 1/dz_w
// (mode 2) or unchanged (mode 0); also a plain per-field scale.
template <typename T>
__global__ void scale5_kernel(Dims d, CVec5<T> src, Vec5<T> dst, T pi_mul, int eta_mode, const T* __restrict__ dzw,
                              const T* __restrict__ idzw) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i > d.nx || j > d.ny || k > d.nz) return;
  if (j < d.ny && k < d.nz) { const int p = iu(d, i, j, k); dst.f[0][p] = src.f[0][p]; }
  if (i < d.nx && k < d.nz) { const int p = iv(d, i, j, k); dst.f[1][p] = src.f[1][p]; }
  if (i < d.nx && j < d.ny) {
    const int p = iw(d, i, j, k);
    dst.f[2][p] = src.f[2][p];
    T e = src.f[4][p];
    if (eta_mode == 1) e *= dzw[p];
    else if (eta_mode == 2) e *= idzw[p];
    dst.f[4][p] = e;
  }
  if (i < d.nx && j < d.ny && k < d.nz) { const int p = im(d, i, j, k); dst.f[3][p] = src.f[3][p] * pi_mul; }
}

// zero the padding gaps of nvec contiguous solver vectors
template <typename T>
__global__ void zero_gaps_kernel(T* base, size_t npad, int nvec, size_t o0, size_t o1, size_t o2, size_t o3,
                                 size_t o4, size_t s0, size_t s1, size_t s2, size_t s3, size_t s4) {
  const size_t off[5] = {o0, o1, o2, o3, o4};
  const size_t sz[5] = {s0, s1, s2, s3, s4};
  const int v = blockIdx.x;
  if (v >= nvec) return;
  T* vb = base + (size_t)v * npad;
  for (int q = 0; q < 5; ++q) {
    const size_t end = (q < 4) ? off[q + 1] : npad;
    for (size_t e = off[q] + sz[q] + threadIdx.x; e < end; e += blockDim.x) vb[e] = T(0);
  }
}

// dst = (D) src over a packed vector; elements below `split` go to dst_lo,
// the rest to dst_hi (the u, v | w, pi, eta_dot split of the solver
// vectors).  n and split are multiples of 4 (the packed fields are padded to
// 64 elements), so every thread moves aligned groups of 4 with vector
// loads and stores; launch CONVERT_BLOCKS blocks of 256.
template <typename T>
__device__ __forceinline__ void load4(const T* p, T (&r)[4]) {
  if constexpr (sizeof(T) == 4) {
    const float4 v = __ldg(reinterpret_cast<const float4*>(p));
    r[0] = v.x; r[1] = v.y; r[2] = v.z; r[3] = v.w;
  } else {
    const double2 a = __ldg(reinterpret_cast<const double2*>(p)), b = __ldg(reinterpret_cast<const double2*>(p) + 1);
    r[0] = a.x; r[1] = a.y; r[2] = b.x; r[3] = b.y;
  }
}
template <typename T>
__device__ __forceinline__ void store4(T* p, const T (&r)[4]) {
  if constexpr (sizeof(T) == 4) {
    *reinterpret_cast<float4*>(p) = make_float4(r[0], r[1], r[2], r[3]);
  } else {
    reinterpret_cast<double2*>(p)[0] = make_double2(r[0], r[1]);
    reinterpret_cast<double2*>(p)[1] = make_double2(r[2], r[3]);
  }
}
constexpr int CONVERT_BLOCKS = 8 * 148;
template <typename S, typename D>
__global__ void __launch_bounds__(256) convert_packed_kernel(const S* __restrict__ src, D* dst_lo, D* dst_hi,
                                                             size_t split, size_t n) {
  const size_t n4 = n / 4;
  for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < n4; q += (size_t)gridDim.x * blockDim.x) {
    const size_t e = 4 * q;
    S a[4];
    load4(src + e, a);
    D b[4];
#pragma unroll
    for (int k = 0; k < 4; ++k) b[k] = (D)a[k];
    store4((e < split ? dst_lo : dst_hi) + e, b);
  }
}

// norm of a packed vector kept for the transposed solve; v *= 1/norm (mode 0)
// or v *= norm (mode 1), a zero norm leaving v unchanged
__global__ void keep_norm_kernel(const GState* gs, double* scal) { *scal = gs->bnorm; }

template <typename T>
__global__ void scale_packed_kernel(T* v, size_t n, const double* scal, int mode) {
  const double nrm = *scal;
  if (!(nrm > 0.0)) return;
  const T f = (T)(mode == 0 ? 1.0 / nrm : nrm);
  for (size_t e = blockIdx.x * (size_t)blockDim.x + threadIdx.x; e < n; e += (size_t)gridDim.x * blockDim.x)
    v[e] *= f;
}

// lateral overrides after advection (steppers.py:858-869) and the zero
// lid/ground rows of R_eta_dot (steppers.py:893)
template <typename T>
__global__ void sl_fixup_kernel(Dims d, T* rhs_u, T* rhs_v, const T* __restrict__ u0, const T* __restrict__ v0,
                                T* reta) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;  // generic 2-D index
  const int k = blockIdx.y;
  // u faces 0 and nx for every (j, k)
  if (a < d.ny && k < d.nz) {
    const int p0 = iu(d, 0, a, k), pn = iu(d, d.nx, a, k);
    if (d.px) rhs_u[pn] = rhs_u[p0];
    else { rhs_u[p0] = u0[p0]; rhs_u[pn] = u0[pn]; }
  }
  if (a < d.nx && k < d.nz) {
    const int p0 = iv(d, a, 0, k), pn = iv(d, a, d.ny, k);
    if (d.py) rhs_v[pn] = rhs_v[p0];
    else { rhs_v[p0] = v0[p0]; rhs_v[pn] = v0[pn]; }
  }
  if (k == 0) {
    for (int jj = 0; jj < d.ny; ++jj) {
      if (a < d.nx) {
        reta[iw(d, a, jj, 0)] = T(0);
        reta[iw(d, a, jj, d.nz)] = T(0);
      }
    }
  }
}

dim3 box(int ex, int ey, int ez, dim3 blk) {
  return dim3((ex + blk.x - 1) / blk.x, (ey + blk.y - 1) / blk.y, (ez + blk.z - 1) / blk.z);
}

// ---------------------------------------------------------------------------
// GMRES workspace
// ---------------------------------------------------------------------------
template <typename T>
struct GWork {
  GState* gs;
  GHostView* dview;  // device copy of the per-cycle summary
  double* partial;
  T* vec;  // (R + 4) contiguous vectors
  T* tmp;  // mass-point scratch of the transposed matvec
  double* scal;  // norm of the normalised right-hand side (transposed solve)
  // iterative refinement (float32 cores): solution, rhs and residual in float64
  bool refine = false;
  double *x64 = nullptr, *b64 = nullptr, *r64 = nullptr, *tmp64 = nullptr;
  size_t npad;
  size_t off[5], sz[5];
  int R;
  T* V(int i) const { return vec + (size_t)(3 + i) * npad; }
  T* xg() const { return vec; }
  T* bg() const { return vec + npad; }
  T* z() const { return vec + 2 * npad; }
  Vec5<T> view(T* b) const {
    Vec5<T> v;
    for (int q = 0; q < 5; ++q) v.f[q] = b + off[q];
    return v;
  }
  CVec5<T> cview(const T* b) const {
    CVec5<T> v;
    for (int q = 0; q < 5; ++q) v.f[q] = b + off[q];
    return v;
  }
  // u, v from vector a; w, pi, eta_dot from vector b
  Vec5<T> split(T* a, T* b) const {
    Vec5<T> v;
    for (int q = 0; q < 5; ++q) v.f[q] = (q < 2 ? a : b) + off[q];
    return v;
  }
};

template <typename T>
GWork<T> carve_gmres(Carver& cv, const Dims& d, int R, bool refine) {
  GWork<T> g;
  g.R = R;
  size_t o = 0;
  for (int q = 0; q < 5; ++q) {
    g.off[q] = o;
    g.sz[q] = field_size(d, loc_of_field(q));
    o += pad64(g.sz[q]);
  }
  g.npad = o;
  g.gs = (GState*)cv.take(sizeof(GState));
  g.dview = (GHostView*)cv.take(sizeof(GHostView));
  g.partial = (double*)cv.take(sizeof(double) * GM_MAXBLOCKS * (GM_MAXR + 2));
  g.vec = (T*)cv.take(sizeof(T) * g.npad * (size_t)(R + 4));
  g.tmp = (T*)cv.take(sizeof(T) * field_size(d, LOC_M));
  g.scal = (double*)cv.take(sizeof(double));
  g.refine = refine;
  if (refine) {
    g.x64 = (double*)cv.take(sizeof(double) * g.npad);
    g.b64 = (double*)cv.take(sizeof(double) * g.npad);
    g.r64 = (double*)cv.take(sizeof(double) * g.npad);
    g.tmp64 = (double*)cv.take(sizeof(double) * field_size(d, LOC_M));
  }
  return g;
}

template <typename T>
CVec5<T> cvec(const void* const p[5]) {
  CVec5<T> v;
  for (int q = 0; q < 5; ++q) v.f[q] = (const T*)p[q];
  return v;
}
template <typename T>
Vec5<T> vec(void* const p[5]) {
  Vec5<T> v;
  for (int q = 0; q < 5; ++q) v.f[q] = (T*)p[q];
  return v;
}

template <typename T>
void scale5(SislCore* c, const Coef<T>& cf, CVec5<T> src, Vec5<T> dst, T pi_mul, int eta_mode, cudaStream_t st) {
  KScope k(c, SISL_K_OTHER, st);
  dim3 blk(32, 4, 2);
  scale5_kernel<T><<<box(c->d.nx + 1, c->d.ny + 1, c->d.nz + 1, blk), blk, 0, st>>>(c->d, src, dst, pi_mul,
                                                                                   eta_mode, cf.dzw, cf.idzw);
}

template <typename T>
CVec5<T> as_const(Vec5<T> v) {
  CVec5<T> r;
  for (int q = 0; q < 5; ++q) r.f[q] = v.f[q];
  return r;
}

// Algorithmic bytes per launch (each distinct array touched once).
double matvec_bytes(const Dims& d, size_t es) {
  const double fu = field_size(d, LOC_U), fv = field_size(d, LOC_V), fw = field_size(d, LOC_W),
               fm = field_size(d, LOC_M);
  const double vec = fu + fv + 2 * fw + fm;
  // 5 inputs + 5 outputs + coefficients thu zxu rdu | thv zev rdv | thw rhow idzw damp zxw zew | cpidz
  return es * (2 * vec + 3 * fu + 3 * fv + 6 * fw + fm);
}
double precond_bytes(const Dims& d, size_t es) {
  const double fu = field_size(d, LOC_U), fv = field_size(d, LOC_V), fw = field_size(d, LOC_W),
               fm = field_size(d, LOC_M);
  const double vec = fu + fv + 2 * fw + fm;
  // 5 inputs + 3 outputs (u, v alias the matvec output) + lpi | damp rhow thw idzw zxw zew
  return es * (vec + 2 * fw + fm + fm + 6 * fw);
}

// Restarted GMRES on the packed vectors g.bg (rhs) and g.xg (initial guess).
// transpose = 1 runs the same iteration on A^T with the preconditioner M^T
// (the bwd_solve of steppers.py:473-481).
//
// Host mode (dev_info == nullptr): one device-to-host read of the residual
// summary per restart cycle decides whether another cycle runs.
// Graph mode (dev_info != nullptr, st capturing): the restart loop becomes a
// CUDA-graph conditional WHILE node whose body is one restart cycle; a gate
// kernel after every residual sets the condition (rnorm > atol and cycles <
// maxiter) on the device, and the final statistics land in *dev_info.  No
// host synchronisation: the whole solve replays inside one graph launch.
template <typename T>
int gmres_run(SislCore* c, const Coef<T>& cf, GWork<T>& g, cudaStream_t st, SislSolveInfo* info,
              int transpose = 0, GDevInfo* dev_info = nullptr) {
  const Dims& d = c->d;
  const int R = g.R;
  const size_t n = g.npad;
  const int method = (transpose && c->adj_method >= 0) ? c->adj_method : c->prm.solve_method;
  const double eps = (sizeof(T) == 8) ? 2.220446049250313e-16 : 1.1920928955078125e-07;
  GState* gs = g.gs;
  CVec5<T> none{};
  const double es = sizeof(T), vb = es * (double)n;
  const double mvb = matvec_bytes(d, sizeof(T)), pcb = precond_bytes(d, sizeof(T));
  // float64 iterative refinement: x and b held in float64, every restart's
  // residual b - A x formed with the float64 operator, the Krylov cycle in T
  const bool refine = g.refine;
  const int nconv = CONVERT_BLOCKS;
  Coef<double> cf64{};
  if (refine) {
    cf64 = coef64_of(c);
    KScope k(c, SISL_K_OTHER, st, 2);
    convert_packed_kernel<T, double><<<nconv, 256, 0, st>>>(g.bg(), g.b64, g.b64, n, n);
    convert_packed_kernel<T, double><<<nconv, 256, 0, st>>>(g.xg(), g.x64, g.x64, n, n);
    // the operator writes no padding gaps: they stay zero for the norms
    if (cudaMemsetAsync(g.r64, 0, sizeof(double) * n, st) != cudaSuccess) return SISL_ERR_CUDA;
  }
  {
    KScope k(c, SISL_K_OTHER, st);
    const double tol = (transpose && c->adj_tol > 0.0) ? c->adj_tol : c->prm.solver_tol;
    gm_setup(gs, eps, tol, c->prm.solver_atol, R, method, st);
  }
  {
    KScope k(c, SISL_K_DOTS, st);
    gm_dots<T>(g.V(0), n, 0, g.bg(), n, g.partial, gs, 1 /*BNORM*/, 0, st);
  }
  // z-space operators: forward A writes its u, v rows straight into the
  // target vector (the preconditioner passes u, v through unchanged,
  // steppers.py:247-249); the transposes go through z in full
  auto apply_A = [&](const T* x, const double* xs, CVec5<T> b, T* target, const int* act, cudaStream_t s) {
    if (transpose) launch_matvec_t<T>(d, cf, g.cview(x), xs, b, g.view(g.z()), g.tmp, act, s);
    else launch_matvec<T>(d, cf, g.cview(x), xs, b, g.split(target, g.z()), act, s);
  };
  auto apply_M = [&](const T* src_full, T* target, const int* act, cudaStream_t s) {
    if (transpose) launch_precond_t<T>(d, cf, g.cview(src_full), g.view(target), act, s);
    else launch_precond<T>(d, cf, g.cview(src_full), g.view(target), act, s);
  };
  auto apply_M_after_A = [&](T* target, const int* act, cudaStream_t s) {
    if (transpose) launch_precond_t<T>(d, cf, g.cview(g.z()), g.view(target), act, s);
    else launch_precond<T>(d, cf, as_const(g.split(target, g.z())), g.view(target), act, s);
  };
  const int na = transpose ? 2 : 1, nm = transpose ? 2 : 1;
  if (method == SISL_GMRES_INCREMENTAL) {
    {
      KScope k(c, SISL_K_PRECOND, st, nm);
      apply_M(g.bg(), g.V(1), nullptr, st);
    }
    KScope k(c, SISL_K_DOTS, st);
    gm_dots<T>(g.V(0), n, 0, g.V(1), n, g.partial, gs, 2 /*MBNORM*/, 0, st);
  }
  {
    KScope k(c, SISL_K_OTHER, st);
    gm_init_tol(gs, st);
  }
  // preconditioned residual M (b - A x), normalised into V(0)
  auto residual = [&](cudaStream_t s) {
    if (refine) {
      KScope k(c, SISL_K_MATVEC, s, na + 1);
      CVec5<double> x5, b5;
      Vec5<double> r5;
      for (int q = 0; q < 5; ++q) {
        x5.f[q] = g.x64 + g.off[q];
        b5.f[q] = g.b64 + g.off[q];
        r5.f[q] = g.r64 + g.off[q];
      }
      if (transpose) {
        launch_matvec_t<double>(d, cf64, x5, nullptr, b5, r5, g.tmp64, nullptr, s);
        convert_packed_kernel<double, T><<<nconv, 256, 0, s>>>(g.r64, g.z(), g.z(), n, n);
      } else {
        launch_matvec<double>(d, cf64, x5, nullptr, b5, r5, nullptr, s);
        convert_packed_kernel<double, T><<<nconv, 256, 0, s>>>(g.r64, g.V(0), g.z(), g.off[2], n);
      }
    } else {
      KScope k(c, SISL_K_MATVEC, s, na);
      apply_A(g.xg(), nullptr, g.cview(g.bg()), g.V(0), nullptr, s);
    }
    {
      KScope k(c, SISL_K_PRECOND, s, nm);
      apply_M_after_A(g.V(0), nullptr, s);
    }
    {
      KScope k(c, SISL_K_DOTS, s);
      gm_dots<T>(g.V(0), n, 0, g.V(0), n, g.partial, gs, 3 /*RNORM*/, 0, s);
    }
  };
  // one restart cycle: R Arnoldi steps, the small least-squares solve, x update
  auto cycle = [&](cudaStream_t s) {
    {
      KScope k(c, SISL_K_OTHER, s);
      gm_begin_cycle(gs, s);
    }
    for (int j = 0; j < R; ++j) {
      {
        KScope k(c, SISL_K_MATVEC, s, na, mvb);
        apply_A(g.V(j), &gs->s[j], none, g.V(j + 1), &gs->active, s);
      }
      {
        KScope k(c, SISL_K_PRECOND, s, nm, pcb);
        apply_M_after_A(g.V(j + 1), &gs->active, s);
      }
      {
        KScope k(c, SISL_K_DOTS, s, 1, vb * (j + 2));  // reads V_0..V_j and w
        gm_dots<T>(g.V(0), n, j + 1, g.V(j + 1), n, g.partial, gs, 0 /*PROJ*/, 1, s);
      }
      {
        KScope k(c, SISL_K_UPDATE, s, 1, vb * (j + 3));  // reads V_0..V_j, reads and writes w
        gm_update<T>(g.V(0), n, j + 1, g.V(j + 1), n, -1.0, g.partial, gs, 1 /*ARNOLDI*/, 1, 0, s);
      }
    }
    {
      KScope k(c, SISL_K_OTHER, s);
      gm_small_solve(gs, R, s);
    }
    {
      KScope k(c, SISL_K_UPDATE, s);
      if (refine) gm_update_x64<T>(g.V(0), n, R, g.x64, n, gs, s);
      else gm_update<T>(g.V(0), n, R, g.xg(), n, 1.0, g.partial, gs, 0 /*NONE*/, 0, 1, s);
    }
  };
  auto finish_x = [&]() {
    if (refine) {
      KScope k(c, SISL_K_OTHER, st);
      convert_packed_kernel<double, T><<<nconv, 256, 0, st>>>(g.x64, g.xg(), g.xg(), n, n);
    }
  };
  const int maxiter = c->prm.solver_maxiter;

  if (dev_info) {  // ---- graph mode ----
    if (!c->cap_side) return SISL_ERR_ARG;
    residual(st);
    cudaStreamCaptureStatus cs;
    cudaGraph_t gr;
    const cudaGraphNode_t* deps = nullptr;
    size_t nd = 0;
    if (cuda_failed(cudaStreamGetCaptureInfo(st, &cs, nullptr, &gr, &deps, &nd), "cudaStreamGetCaptureInfo") ||
        cs != cudaStreamCaptureStatusActive)
      return SISL_ERR_ARG;
    cudaGraphConditionalHandle h;
    if (cuda_failed(cudaGraphConditionalHandleCreate(&h, gr, 0, cudaGraphCondAssignDefault),
                    "cudaGraphConditionalHandleCreate"))
      return SISL_ERR_CUDA;
    {
      KScope k(c, SISL_K_OTHER, st);
      gm_gate(gs, h, maxiter, 0, st);
    }
    if (cuda_failed(cudaStreamGetCaptureInfo(st, &cs, nullptr, &gr, &deps, &nd), "cudaStreamGetCaptureInfo"))
      return SISL_ERR_CUDA;
    cudaGraphNodeParams np{};
    np.type = cudaGraphNodeTypeConditional;
    np.conditional.handle = h;
    np.conditional.type = cudaGraphCondTypeWhile;
    np.conditional.size = 1;
    cudaGraphNode_t node;
    if (cuda_failed(cudaGraphAddNode(&node, gr, deps, nd, &np), "cudaGraphAddNode(conditional)")) return SISL_ERR_CUDA;
    cudaGraph_t body = np.conditional.phGraph_out[0];
    if (cuda_failed(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies),
                    "cudaStreamUpdateCaptureDependencies"))
      return SISL_ERR_CUDA;
    cudaStream_t sb = c->cap_side;
    if (cuda_failed(cudaStreamBeginCaptureToGraph(sb, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed),
                    "cudaStreamBeginCaptureToGraph"))
      return SISL_ERR_CUDA;
    cycle(sb);
    residual(sb);
    {
      KScope k(c, SISL_K_OTHER, sb);
      gm_gate(gs, h, maxiter, 1, sb);
    }
    cudaGraph_t body_out = nullptr;
    if (cuda_failed(cudaStreamEndCapture(sb, &body_out), "cudaStreamEndCapture(body)")) return SISL_ERR_CUDA;
    {
      KScope k(c, SISL_K_OTHER, st);
      gm_info(gs, dev_info, st);
    }
    finish_x();
    return check_cuda();
  }

  // ---- host mode ----
  GHostView* hv = c->hv;
  auto read = [&]() -> int {
    GHostView* dv = g.dview;
    {
      KScope k(c, SISL_K_OTHER, st);
      gm_snapshot(gs, dv, st);
    }
    if (cudaMemcpyAsync(hv, dv, sizeof(GHostView), cudaMemcpyDeviceToHost, st) != cudaSuccess) return SISL_ERR_CUDA;
    if (cudaStreamSynchronize(st) != cudaSuccess) return SISL_ERR_CUDA;
    return SISL_OK;
  };
  residual(st);
  int rc = read();
  if (rc) return rc;
  int cycles = 0, steps = 0;
  while (cycles < maxiter && hv->rnorm > hv->atol) {
    cycle(st);
    residual(st);
    rc = read();
    if (rc) return rc;
    steps += hv->kdone;
    cycles++;
  }
  finish_x();
  if (info) {
    info->cycles = cycles;
    info->arnoldi_steps = steps;
    info->residual_norm = hv->rnorm;
    info->atol = hv->atol;
    info->b_norm = hv->bnorm;
    info->converged = (hv->rnorm <= hv->atol) ? 1 : 0;
  }
  if (!std::isfinite(hv->rnorm)) return SISL_ERR_NONFINITE;
  return (hv->rnorm <= hv->atol) ? SISL_OK : SISL_NOT_CONVERGED;
}

// SemiImplicitSolver3D.solve: scale, GMRES, unscale (steppers.py:401-496).
// solve_prep stages the scaled right-hand side and initial guess in the
// GMRES vectors, solve_finish unscales the solution.
template <typename T>
void solve_prep(SislCore* c, const Coef<T>& cf, GWork<T>& g, CVec5<T> rhs, const CVec5<T>* x0, cudaStream_t st) {
  {
    KScope k(c, SISL_K_OTHER, st);
    zero_gaps_kernel<T><<<g.R + 4, 256, 0, st>>>(g.vec, g.npad, g.R + 4, g.off[0], g.off[1], g.off[2], g.off[3],
                                                g.off[4], g.sz[0], g.sz[1], g.sz[2], g.sz[3], g.sz[4]);
  }
  const T ps = (T)c->s.ps;
  scale5<T>(c, cf, rhs, g.view(g.bg()), ps, 0, st);       // rhs_scaled: pi * pi_scale
  if (x0) scale5<T>(c, cf, *x0, g.view(g.xg()), ps, 1, st);  // x0 scaled: pi * ps, eta * dz_w
  else scale5<T>(c, cf, rhs, g.view(g.xg()), ps, 0, st);     // x0 = rhs_scaled
}
template <typename T>
void solve_finish(SislCore* c, const Coef<T>& cf, GWork<T>& g, Vec5<T> x, cudaStream_t st) {
  scale5<T>(c, cf, g.cview(g.xg()), x, (T)(1.0 / c->s.ps), 2, st);  // pi / ps, eta / dz_w
}
template <typename T>
int solve_physical(SislCore* c, const Coef<T>& cf, GWork<T>& g, CVec5<T> rhs, const CVec5<T>* x0, Vec5<T> x,
                   cudaStream_t st, SislSolveInfo* info, GDevInfo* dev_info = nullptr) {
  solve_prep<T>(c, cf, g, rhs, x0, st);
  int rc = gmres_run<T>(c, cf, g, st, info, 0, dev_info);
  if (rc < 0 && rc != SISL_ERR_NONFINITE) return rc;
  solve_finish<T>(c, cf, g, x, st);
  return rc;
}

// Cotangent of the physical right-hand side from the cotangent of the
// physical solution (custom_linear_solve transpose, steppers.py:473-485):
// unscale (x = S_out x_s), GMRES on A^T from a zero guess, rescale (b_s = S_in b).
// solve_t_prep stages the GMRES vectors, solve_t_finish rescales the result.
template <typename T>
int solve_t_prep(SislCore* c, const Coef<T>& cf, GWork<T>& g, CVec5<T> xbar, const CVec5<T>* x0, cudaStream_t st) {
  {
    KScope k(c, SISL_K_OTHER, st);
    zero_gaps_kernel<T><<<g.R + 4, 256, 0, st>>>(g.vec, g.npad, g.R + 4, g.off[0], g.off[1], g.off[2], g.off[3],
                                                g.off[4], g.sz[0], g.sz[1], g.sz[2], g.sz[3], g.sz[4]);
  }
  scale5<T>(c, cf, xbar, g.view(g.bg()), (T)(1.0 / c->s.ps), 2, st);  // pi / ps, eta / dz_w
  // initial guess: zero as in bwd_solve, or a caller's guess in the units of
  // the result (a warm start: the same solution within the tolerance)
  if (x0) scale5<T>(c, cf, *x0, g.view(g.xg()), (T)(1.0 / c->s.ps), 0, st);
  else if (cudaMemsetAsync(g.xg(), 0, sizeof(T) * g.npad, st) != cudaSuccess) return SISL_ERR_CUDA;
  // GMRES treats a preconditioned residual below machine epsilon as zero
  // (_safe_normalize's absolute threshold); cotangents are often far below
  // unit norm, so the right-hand side is solved at unit norm and rescaled
  if (c->adj_normalize) {
    const int nb = 2 * 148;
    KScope k(c, SISL_K_OTHER, st, 4);
    gm_setup(g.gs, 0.0, c->prm.solver_tol, c->prm.solver_atol, g.R, c->prm.solve_method, st);
    gm_dots<T>(g.V(0), g.npad, 0, g.bg(), g.npad, g.partial, g.gs, 1 /*BNORM*/, 0, st);
    keep_norm_kernel<<<1, 1, 0, st>>>(g.gs, g.scal);
    scale_packed_kernel<T><<<nb, 256, 0, st>>>(g.bg(), g.npad, g.scal, 0);
    if (x0) scale_packed_kernel<T><<<nb, 256, 0, st>>>(g.xg(), g.npad, g.scal, 0);
  }
  return SISL_OK;
}
template <typename T>
void solve_t_finish(SislCore* c, const Coef<T>& cf, GWork<T>& g, Vec5<T> bbar, cudaStream_t st) {
  if (c->adj_normalize) {
    KScope k(c, SISL_K_OTHER, st);
    scale_packed_kernel<T><<<2 * 148, 256, 0, st>>>(g.xg(), g.npad, g.scal, 1);
  }
  scale5<T>(c, cf, g.cview(g.xg()), bbar, (T)c->s.ps, 0, st);  // pi * ps
}
template <typename T>
int solve_transpose_physical(SislCore* c, const Coef<T>& cf, GWork<T>& g, CVec5<T> xbar, const CVec5<T>* x0,
                             Vec5<T> bbar, cudaStream_t st, SislSolveInfo* info, GDevInfo* dev_info = nullptr) {
  int rc = solve_t_prep<T>(c, cf, g, xbar, x0, st);
  if (rc) return rc;
  rc = gmres_run<T>(c, cf, g, st, info, 1, dev_info);
  if (rc < 0 && rc != SISL_ERR_NONFINITE) return rc;
  solve_t_finish<T>(c, cf, g, bbar, st);
  return rc;
}

// ---------------------------------------------------------------------------
// step workspace
// ---------------------------------------------------------------------------
template <typename T>
struct SWork {
  GWork<T> g;
  T* vel[12];
  T *u_in, *v_in, *w_in, *pi_in, *th_in, *tth, *res;
  T *ru, *rv, *rw, *rp, *tha, *reta;
  T *hyp[4], *htmp[4], *hgxy[8];
  T *ku, *kv, *kw, *kp;
  T *su, *sv;
  T* div;
};

template <typename T>
SWork<T> carve_step(Carver& cv, const Dims& d, int R, bool refine) {
  SWork<T> w;
  w.g = carve_gmres<T>(cv, d, R, refine);
  auto F = [&](int loc) { return (T*)cv.take(sizeof(T) * field_size(d, loc)); };
  const int vl[4] = {LOC_M, LOC_U, LOC_V, LOC_W};
  for (int l = 0; l < 4; ++l)
    for (int q = 0; q < 3; ++q) w.vel[3 * l + q] = F(vl[l]);
  w.u_in = F(LOC_U); w.v_in = F(LOC_V); w.w_in = F(LOC_W); w.pi_in = F(LOC_M); w.th_in = F(LOC_M);
  w.tth = F(LOC_M); w.res = F(LOC_W);
  w.ru = F(LOC_U); w.rv = F(LOC_V); w.rw = F(LOC_W); w.rp = F(LOC_M); w.tha = F(LOC_M); w.reta = F(LOC_W);
  for (int q = 0; q < 4; ++q) { w.hyp[q] = F(LOC_M); w.htmp[q] = F(LOC_M); }
  for (int q = 0; q < 8; ++q) w.hgxy[q] = F(q < 4 ? LOC_U : LOC_V);
  w.ku = F(LOC_U); w.kv = F(LOC_V); w.kw = F(LOC_W); w.kp = F(LOC_M);
  w.su = F(LOC_U); w.sv = F(LOC_V);
  w.div = F(LOC_M);
  return w;
}

// One step's state between its segments.  The step is issued as
// step_open, step_explicit, then for each of the two solves step_pre_solve,
// GMRES on the core's solver vectors and step_post_solve, then step_close;
// the ensemble graph interleaves the members' segments around grouped solves.
template <typename T>
struct StepRun {
  SislCore* c = nullptr;
  const SislState* in = nullptr;
  const SislState* out = nullptr;
  const SislRelaxation* relax = nullptr;
  cudaStream_t st = nullptr;
  SislStepInfo* info = nullptr;
  void* const* tape = nullptr;
  const void* const* phys = nullptr;
  Coef<T> cf{};
  SWork<T> w{};
  int64_t l0 = 0;
  int status = SISL_OK;
};

template <typename T>
int step_open(StepRun<T>& r, SislCore* c, const SislState* in, const SislState* out, const SislRelaxation* relax,
              void* ws, size_t ws_bytes, cudaStream_t st, SislStepInfo* info, void* const* tape,
              const void* const* phys) {
  r.c = c; r.in = in; r.out = out; r.relax = relax; r.st = st; r.info = info; r.tape = tape; r.phys = phys;
  r.cf = coef_of<T>(c);
  Carver cv{(char*)ws};
  r.w = carve_step<T>(cv, c->d, c->prm.solver_restart, refining<T>(c));
  if (cv.off > ws_bytes) return SISL_ERR_WORKSPACE;
  r.l0 = g_launches.load();
  r.status = SISL_OK;
  return SISL_OK;
}

// trajectory velocities, explicit tendencies, semi-Lagrangian advection
template <typename T>
void step_explicit(StepRun<T>& r) {
  SislCore* c = r.c;
  const Dims& d = c->d;
  const Coef<T>& cf = r.cf;
  SWork<T>& w = r.w;
  const SislState* in = r.in;
  cudaStream_t st = r.st;
  const T* u = (const T*)in->u;
  const T* v = (const T*)in->v;
  const T* wv = (const T*)in->w;
  const T* eta = (const T*)in->eta_dot;
  const T* pp = (const T*)in->pi_p;
  const T* th = (const T*)in->th_p;
  const double a = c->s.alpha, dt = c->s.dt;
  (void)pp;
  // 1. trajectory index velocities (steppers.py:748-762, 276-316)
  {
    PtrTable<T> vt{};
    for (int q = 0; q < 12; ++q) vt.p[q] = w.vel[q];
    const int extrap = (in->is_first_step == 1.0) ? 0 : 1;
    KScope k(c, SISL_K_SL, st);
    launch_traj_velocity<T>(d, cf, u, v, eta, (const T*)in->u_prev, (const T*)in->v_prev,
                            (const T*)in->eta_dot_prev, extrap, vt, st);
  }
  // 2. explicit tendencies with hyperdiffusion (euler.py:208-372)
  ExplicitIn<T> ein{u, v, wv, eta, (const T*)in->pi_p, th, {nullptr, nullptr, nullptr, nullptr},
                    {nullptr, nullptr, nullptr, nullptr}};
  if (r.phys)
    for (int q = 0; q < 4; ++q) ein.extra[q] = (const T*)r.phys[q];
  if (c->s.nu_h > 0.0) {
    PtrTable<T> t4{}, o4{};
    for (int q = 0; q < 4; ++q) { t4.p[q] = w.htmp[q]; o4.p[q] = w.hyp[q]; }
    KScope k(c, SISL_K_EXPLICIT, st, 5);
    PtrTable<T> g8{};
    for (int q = 0; q < 8; ++q) g8.p[q] = w.hgxy[q];
    launch_hyper<T>(d, cf, u, v, wv, th, t4, o4, g8, st);
    for (int q = 0; q < 4; ++q) ein.hyper[q] = w.hyp[q];
  }
  {
    ExplicitOut<T> eo{};
    eo.f[0] = w.u_in; eo.f[1] = w.v_in; eo.f[2] = w.w_in; eo.f[3] = w.pi_in; eo.f[4] = w.th_in;
    eo.f[5] = w.tth; eo.f[6] = w.res;
    KScope k(c, SISL_K_EXPLICIT, st);
    launch_explicit<T>(d, cf, ein, eo, 0, st);
  }
  // 3. semi-Lagrangian advection at the departure points (steppers.py:852-876)
  const int iters = c->prm.departure_iterations;
  const int lim = c->prm.use_limiter;
  {
    const T* f[2] = {w.res, w.w_in};
    T* o[2] = {w.reta, w.rw};
    const T sc[2] = {(T)(-(1.0 - a)), T(1)};
    KScope k(c, SISL_K_SL, st);
    launch_sl_advect<T>(d, LOC_W, dt, w.vel + 9, iters, 2, f, o, sc, lim, st);
  }
  {
    const T* f[1] = {w.u_in};
    T* o[1] = {w.ru};
    const T sc[1] = {T(1)};
    KScope k(c, SISL_K_SL, st);
    launch_sl_advect<T>(d, LOC_U, dt, w.vel + 3, iters, 1, f, o, sc, lim, st);
  }
  {
    const T* f[1] = {w.v_in};
    T* o[1] = {w.rv};
    const T sc[1] = {T(1)};
    KScope k(c, SISL_K_SL, st);
    launch_sl_advect<T>(d, LOC_V, dt, w.vel + 6, iters, 1, f, o, sc, lim, st);
  }
  {
    const T* f[2] = {w.pi_in, w.th_in};
    T* o[2] = {w.rp, w.tha};
    const T sc[2] = {T(1), T(1)};
    KScope k(c, SISL_K_SL, st);
    launch_sl_advect<T>(d, LOC_M, dt, w.vel + 0, iters, 2, f, o, sc, lim, st);
  }
  {
    KScope k(c, SISL_K_OTHER, st);
    const int na = (d.nx > d.ny ? d.nx : d.ny) + 1;
    sl_fixup_kernel<T><<<dim3((na + 127) / 128, d.nz), 128, 0, st>>>(d, w.ru, w.rv, u, v, w.reta);
  }
}

// 4. predictor-corrector with two implicit solves (steppers.py:911-998):
// the theta' predictor and the right-hand side of solve `it`, staged in the
// GMRES vectors with its initial guess
template <typename T>
Vec5<T> step_solution(const StepRun<T>& r) {
  const SWork<T>& w = r.w;
  Vec5<T> xs;
  xs.f[0] = w.su; xs.f[1] = w.sv; xs.f[2] = (T*)r.out->w; xs.f[3] = (T*)r.out->pi_p; xs.f[4] = (T*)r.out->eta_dot;
  return xs;
}

template <typename T>
void step_pre_solve(StepRun<T>& r, int it) {
  SislCore* c = r.c;
  const Dims& d = c->d;
  SWork<T>& w = r.w;
  const SislState* in = r.in;
  cudaStream_t st = r.st;
  const T* u = (const T*)in->u;
  const T* v = (const T*)in->v;
  const T* wv = (const T*)in->w;
  const T* eta = (const T*)in->eta_dot;
  const T* pp = (const T*)in->pi_p;
  T* ow = (T*)r.out->w;
  T* op = (T*)r.out->pi_p;
  T* oe = (T*)r.out->eta_dot;
  T* oth = (T*)r.out->th_p;
  const T* w_next = (it == 0) ? wv : ow;
  {
    KScope k(c, SISL_K_EXPLICIT, st);
    launch_corrector_theta<T>(d, r.cf, w.tha, w.tth, wv, w_next, oth, st);
  }
  CorrectorIn<T> ci;
  ci.rhs_u = w.ru; ci.rhs_v = w.rv; ci.rhs_w = w.rw; ci.rhs_pi = w.rp;
  ci.th_next = oth;
  ci.pg = (it == 0) ? pp : op;
  ci.gu = (it == 0) ? u : w.su;
  ci.gv = (it == 0) ? v : w.sv;
  ci.geta = (it == 0) ? eta : oe;
  ci.ug = (it == 0) ? w.ru : w.su;
  ci.vg = (it == 0) ? w.rv : w.sv;
  Vec5<T> rk;
  rk.f[0] = w.ku; rk.f[1] = w.kv; rk.f[2] = w.kw; rk.f[3] = w.kp; rk.f[4] = w.reta;
  {
    KScope k(c, SISL_K_EXPLICIT, st);
    launch_corrector_rhs<T>(d, r.cf, ci, rk, st);
  }
  CVec5<T> x0;
  if (it == 0) { x0.f[0] = u; x0.f[1] = v; x0.f[2] = wv; x0.f[3] = pp; x0.f[4] = eta; }
  else { x0.f[0] = w.su; x0.f[1] = w.sv; x0.f[2] = ow; x0.f[3] = op; x0.f[4] = oe; }
  solve_prep<T>(c, r.cf, w.g, as_const(rk), &x0, st);
}

// the solution of solve `it` unscaled into the step's outputs (and the tape);
// rc: the solve's status
template <typename T>
int step_post_solve(StepRun<T>& r, int it, int rc, const SislSolveInfo& si) {
  SislCore* c = r.c;
  const Dims& d = c->d;
  if (r.info) r.info->solve[it] = si;
  if (rc < 0 && rc != SISL_ERR_NONFINITE) return rc;
  const Vec5<T> xs = step_solution(r);
  solve_finish<T>(c, r.cf, r.w.g, xs, r.st);
  if (r.tape) {  // the physical solution of this solve, for the recomputation of the VJP
    static const int L5[5] = {LOC_U, LOC_V, LOC_W, LOC_M, LOC_W};
    for (int q = 0; q < 5; ++q)
      if (r.tape[5 * it + q] &&
          cudaMemcpyAsync(r.tape[5 * it + q], xs.f[q], sizeof(T) * field_size(d, L5[q]), cudaMemcpyDeviceToDevice,
                          r.st) != cudaSuccess)
        return SISL_ERR_CUDA;
  }
  if (rc != SISL_OK && r.status == SISL_OK) r.status = rc;
  return SISL_OK;
}

// 5. divergence damping, bc_fn relaxation, EOS (steppers.py:1022-1056) and
// 6. history (steppers.py:1061-1071)
template <typename T>
int step_close(StepRun<T>& r) {
  SislCore* c = r.c;
  const Dims& d = c->d;
  SWork<T>& w = r.w;
  const SislState* in = r.in;
  const SislState* out = r.out;
  const SislRelaxation* relax = r.relax;
  cudaStream_t st = r.st;
  FinalizeArgs<T> fa{};
  fa.u_in = w.su; fa.v_in = w.sv;
  fa.u_out = (T*)out->u; fa.v_out = (T*)out->v;
  fa.w_io = (T*)out->w; fa.th_io = (T*)out->th_p; fa.pi_io = (T*)out->pi_p;
  fa.rho_out = (T*)out->rho;
  fa.div = nullptr;
  if (c->s.nu_div != 0.0) {
    KScope k(c, SISL_K_OTHER, st);
    launch_hdiv<T>(d, r.cf, w.su, w.sv, w.div, st);
    fa.div = w.div;
  }
  fa.relax.on = 0;
  if (relax) {
    fa.relax.on = relax->fields;
    fa.relax.mask_m = (const T*)relax->mask_m;
    fa.relax.mask_u = (const T*)relax->mask_u;
    fa.relax.mask_v = (const T*)relax->mask_v;
    for (int q = 0; q < 5; ++q) { fa.relax.ext[q] = (T)relax->ext[q]; fa.relax.ext_field[q] = (const T*)relax->ext_field[q]; }
  }
  {
    KScope k(c, SISL_K_OTHER, st);
    launch_finalize<T>(d, r.cf, fa, st);
  }
  auto cp = [&](void* dst, const void* src, int loc) {
    if (dst && src && dst != src)
      cudaMemcpyAsync(dst, src, sizeof(T) * field_size(d, loc), cudaMemcpyDeviceToDevice, st);
  };
  cp(out->u_prev, in->u, LOC_U);
  cp(out->v_prev, in->v, LOC_V);
  cp(out->w_prev, in->w, LOC_W);
  cp(out->eta_dot_prev, in->eta_dot, LOC_W);
  cp(out->tend_th_prev, w.tth, LOC_M);
  if (r.info) r.info->kernel_launches = g_launches.load() - r.l0;
  int e = check_cuda();
  return e ? e : r.status;
}

template <typename T>
int step_impl(SislCore* c, const SislState* in, const SislState* out, const SislRelaxation* relax, void* ws,
              size_t ws_bytes, cudaStream_t st, SislStepInfo* info, void* const* tape = nullptr,
              GDevInfo* dev_info = nullptr, const void* const* phys = nullptr) {
  StepRun<T> r;
  int rc = step_open<T>(r, c, in, out, relax, ws, ws_bytes, st, info, tape, phys);
  if (rc) return rc;
  step_explicit<T>(r);
  for (int it = 0; it < 2; ++it) {
    step_pre_solve<T>(r, it);
    SislSolveInfo si{};
    rc = gmres_run<T>(c, r.cf, r.w.g, st, &si, 0, dev_info ? dev_info + it : nullptr);
    rc = step_post_solve<T>(r, it, rc, si);
    if (rc) return rc;
  }
  return step_close<T>(r);
}

// ---------------------------------------------------------------------------
// step VJP: recompute the step's explicit part from the input state and the
// recorded solutions, then run the reverse sweep
// ---------------------------------------------------------------------------
template <typename T>
struct VWork {
  T* coords[12];
  T *th1, *th2;
  T *x1b[5], *x2b[5], *bb[5];
  T *rub, *rvb, *rwb, *rpb, *reb, *thab, *tthb, *th1b, *th2b;
  T *uinb, *vinb, *winb, *pinb, *thinb, *resb;
  T *hypb[4], *gx4[4], *gy4[4], *tmp4[4];
  T* divb;
  void* det;         // fixed-point scratch of the deterministic tricubic VJPs
  char* zero_begin;  // the cotangent arrays that start at zero: [zero_begin, zero_end)
  char* zero_end;
};

template <typename T>
VWork<T> carve_vjp(Carver& cv, const Dims& d) {
  VWork<T> v;
  auto F = [&](int loc) { return (T*)cv.take(sizeof(T) * field_size(d, loc)); };
  static const int L5[5] = {LOC_U, LOC_V, LOC_W, LOC_M, LOC_W};
  for (int l = 0; l < 4; ++l)
    for (int q = 0; q < 3; ++q) v.coords[3 * l + q] = F(l);
  v.th1 = F(LOC_M); v.th2 = F(LOC_M);
  for (int q = 0; q < 5; ++q) v.bb[q] = F(L5[q]);
  for (int q = 0; q < 5; ++q) v.x2b[q] = F(L5[q]);
  for (int q = 0; q < 4; ++q) { v.gx4[q] = F(LOC_U); v.gy4[q] = F(LOC_V); v.tmp4[q] = F(LOC_M); }
  v.divb = F(LOC_M);
  v.th2b = F(LOC_M);
  {  // shared by the deterministic tricubic and stencil VJPs (they run one after another)
    const size_t a = tricubic_vjp_det_scratch_bytes(d.nx + 1, d.ny + 1, d.nz + 1, (int)sizeof(T));
    const size_t b = det_scatter_scratch_bytes(d, (int)sizeof(T));
    v.det = cv.take(a > b ? a : b);
  }
  v.zero_begin = (char*)cv.take(0);
  for (int q = 0; q < 5; ++q) v.x1b[q] = F(L5[q]);
  v.rub = F(LOC_U); v.rvb = F(LOC_V); v.rwb = F(LOC_W); v.rpb = F(LOC_M); v.reb = F(LOC_W);
  v.thab = F(LOC_M); v.th1b = F(LOC_M);
  v.uinb = F(LOC_U); v.vinb = F(LOC_V); v.winb = F(LOC_W); v.pinb = F(LOC_M); v.thinb = F(LOC_M);
  v.resb = F(LOC_W);
  for (int q = 0; q < 4; ++q) v.hypb[q] = F(LOC_M);
  v.zero_end = (char*)cv.take(0);
  v.tthb = F(LOC_M);
  return v;
}

// One reverse sweep's state between its segments: vjp_open, vjp_forward
// (recompute and the finalisation's transpose), then for the second solve
// and the first vjp_pre_solve, the transposed GMRES and vjp_post_solve,
// then vjp_close (overrides, the six interpolation VJPs, explicit^T).
template <typename T>
struct VjpRun {
  SislCore* c = nullptr;
  const SislState* in = nullptr;
  void* const* tape = nullptr;
  const SislRelaxation* relax = nullptr;
  const SislState* ob = nullptr;
  const SislState* ib = nullptr;
  cudaStream_t st = nullptr;
  SislStepInfo* info = nullptr;
  Coef<T> cf{};
  SWork<T> w{};
  VWork<T> v{};
  ExplicitIn<T> ein{};
  bool hyp = false;
  int64_t l0 = 0;
  int status = SISL_OK;
};

template <typename T>
int vjp_open(VjpRun<T>& r, SislCore* c, const SislState* in, void* const* tape, const SislRelaxation* relax,
             const SislState* ob, const SislState* ib, void* ws, size_t ws_bytes, cudaStream_t st,
             SislStepInfo* info) {
  r.c = c; r.in = in; r.tape = tape; r.relax = relax; r.ob = ob; r.ib = ib; r.st = st; r.info = info;
  r.cf = coef_of<T>(c);
  Carver cv{(char*)ws};
  r.w = carve_step<T>(cv, c->d, c->prm.solver_restart, refining<T>(c));
  r.v = carve_vjp<T>(cv, c->d);
  if (cv.off > ws_bytes) return SISL_ERR_WORKSPACE;
  r.l0 = g_launches.load();
  r.status = SISL_OK;
  return SISL_OK;
}

// cotangent initialisation, the recomputation of the forward step's explicit
// part, and the transpose of the finalisation
template <typename T>
int vjp_forward(VjpRun<T>& r) {
  SislCore* c = r.c;
  const Dims& d = c->d;
  const Coef<T>& cf = r.cf;
  SWork<T>& w = r.w;
  VWork<T>& v = r.v;
  const SislState* in = r.in;
  const SislState* ob = r.ob;
  const SislState* ib = r.ib;
  const SislRelaxation* relax = r.relax;
  cudaStream_t st = r.st;
  const T* u = (const T*)in->u;
  const T* vv = (const T*)in->v;
  const T* wv = (const T*)in->w;
  const T* eta = (const T*)in->eta_dot;
  const T* pp = (const T*)in->pi_p;
  const T* th = (const T*)in->th_p;
  const T* x1[5];
  const T* x2[5];
  for (int q = 0; q < 5; ++q) { x1[q] = (const T*)r.tape[q]; x2[q] = (const T*)r.tape[5 + q]; }
  const double dt = c->s.dt;
  auto bytes = [&](int loc) { return sizeof(T) * field_size(d, loc); };
  // cotangents of the input state: the history passes straight through
  // (u_prev' = u, ...), everything else accumulates on top
  T* ub = (T*)ib->u;
  T* vb = (T*)ib->v;
  T* wb = (T*)ib->w;
  T* eb = (T*)ib->eta_dot;
  T* pb = (T*)ib->pi_p;
  T* hb = (T*)ib->th_p;
  auto init = [&](T* dst, const void* src, int loc) -> bool {
    if (src) return cudaMemcpyAsync(dst, src, bytes(loc), cudaMemcpyDeviceToDevice, st) == cudaSuccess;
    return cudaMemsetAsync(dst, 0, bytes(loc), st) == cudaSuccess;
  };
  if (!init(ub, ob->u_prev, LOC_U) || !init(vb, ob->v_prev, LOC_V) || !init(wb, ob->w_prev, LOC_W) ||
      !init(eb, ob->eta_dot_prev, LOC_W) || !init(pb, nullptr, LOC_M) || !init(hb, nullptr, LOC_M) ||
      !init(v.tthb, ob->tend_th_prev, LOC_M))
    return SISL_ERR_CUDA;
  void* dead[6] = {ib->rho, ib->u_prev, ib->v_prev, ib->w_prev, ib->eta_dot_prev, ib->tend_th_prev};
  const int dead_loc[6] = {LOC_M, LOC_U, LOC_V, LOC_W, LOC_W, LOC_M};
  for (int q = 0; q < 6; ++q)  // no cotangent: the departure points are stop_gradient, rho is rebuilt by the EOS
    if (dead[q] && cudaMemsetAsync(dead[q], 0, bytes(dead_loc[q]), st) != cudaSuccess) return SISL_ERR_CUDA;
  if (cudaMemsetAsync(v.zero_begin, 0, (size_t)(v.zero_end - v.zero_begin), st) != cudaSuccess)
    return SISL_ERR_CUDA;

  // ---- recompute: trajectory velocities, departure points, explicit part,
  // advection and the theta' predictors (bitwise the forward step's kernels)
  {
    PtrTable<T> vt{};
    for (int q = 0; q < 12; ++q) vt.p[q] = w.vel[q];
    const int extrap = (in->is_first_step == 1.0) ? 0 : 1;
    KScope k(c, SISL_K_SL, st);
    launch_traj_velocity<T>(d, cf, u, vv, eta, (const T*)in->u_prev, (const T*)in->v_prev,
                            (const T*)in->eta_dot_prev, extrap, vt, st);
  }
  const int iters = c->prm.departure_iterations;
  const int lim = c->prm.use_limiter;
  {
    KScope k(c, SISL_K_SL, st, 4);
    // split-form offsets, as the forward's fused semi-Lagrangian kernels form them
    for (int l = 0; l < 4; ++l) launch_departure<T>(d, l, dt, w.vel + 3 * l, iters, v.coords + 3 * l, 1, st);
  }
  ExplicitIn<T>& ein = r.ein;
  ein = ExplicitIn<T>{u, vv, wv, eta, pp, th, {nullptr, nullptr, nullptr, nullptr}};
  const bool hyp = r.hyp = c->s.nu_h > 0.0;
  if (hyp) {
    PtrTable<T> t4{}, o4{};
    for (int q = 0; q < 4; ++q) { t4.p[q] = w.htmp[q]; o4.p[q] = w.hyp[q]; }
    KScope k(c, SISL_K_EXPLICIT, st, 5);
    PtrTable<T> g8{};
    for (int q = 0; q < 8; ++q) g8.p[q] = w.hgxy[q];
    launch_hyper<T>(d, cf, u, vv, wv, th, t4, o4, g8, st);
    for (int q = 0; q < 4; ++q) ein.hyper[q] = w.hyp[q];
  }
  {
    ExplicitOut<T> eo{};
    eo.f[0] = w.u_in; eo.f[1] = w.v_in; eo.f[2] = w.w_in; eo.f[3] = w.pi_in; eo.f[4] = w.th_in;
    eo.f[5] = w.tth; eo.f[6] = w.res;
    KScope k(c, SISL_K_EXPLICIT, st);
    launch_explicit<T>(d, cf, ein, eo, 0, st);
  }
  {  // ru, rv (guess winds of the first corrector) and th_adv are read back
    const T* fu[1] = {w.u_in};
    T* ou[1] = {w.ru};
    const T* fv[1] = {w.v_in};
    T* ov[1] = {w.rv};
    const T* fm[1] = {w.th_in};
    T* om[1] = {w.tha};
    const T one[1] = {T(1)};
    KScope k(c, SISL_K_SL, st, 4);
    launch_sl_advect<T>(d, LOC_U, dt, w.vel + 3, iters, 1, fu, ou, one, lim, st);
    launch_sl_advect<T>(d, LOC_V, dt, w.vel + 6, iters, 1, fv, ov, one, lim, st);
    launch_sl_advect<T>(d, LOC_M, dt, w.vel + 0, iters, 1, fm, om, one, lim, st);
    const int na = (d.nx > d.ny ? d.nx : d.ny) + 1;
    sl_fixup_kernel<T><<<dim3((na + 127) / 128, d.nz), 128, 0, st>>>(d, w.ru, w.rv, u, vv, w.reta);
  }
  {
    KScope k(c, SISL_K_EXPLICIT, st, 2);
    launch_corrector_theta<T>(d, cf, w.tha, w.tth, wv, wv, v.th1, st);
    launch_corrector_theta<T>(d, cf, w.tha, w.tth, wv, x1[2], v.th2, st);
  }

  // ---- reverse sweep
  {  // divergence damping, relaxation and EOS (steppers.py:1022-1056)
    FinalizeBar<T> fb{};
    fb.th2 = v.th2; fb.pi2 = x2[3];
    fb.u = (const T*)ob->u; fb.v = (const T*)ob->v; fb.w = (const T*)ob->w; fb.eta = (const T*)ob->eta_dot;
    fb.pi = (const T*)ob->pi_p; fb.th = (const T*)ob->th_p; fb.rho = (const T*)ob->rho;
    fb.x2u = v.x2b[0]; fb.x2v = v.x2b[1]; fb.x2w = v.x2b[2]; fb.x2pi = v.x2b[3]; fb.x2eta = v.x2b[4];
    fb.th2b = v.th2b;
    fb.relax.on = 0;
    if (relax) {
      fb.relax.on = relax->fields;
      fb.relax.mask_m = (const T*)relax->mask_m;
      fb.relax.mask_u = (const T*)relax->mask_u;
      fb.relax.mask_v = (const T*)relax->mask_v;
      for (int q = 0; q < 5; ++q) {
        fb.relax.ext[q] = (T)relax->ext[q];
        fb.relax.ext_field[q] = (const T*)relax->ext_field[q];
      }
    }
    KScope k(c, SISL_K_OTHER, st, c->s.nu_div != 0.0 ? 3 : 1);
    launch_finalize_vjp<T>(d, cf, fb, v.divb, st);
  }
  return SISL_OK;
}

// the transposed solve of the step's solve `it` staged from its solution's cotangent
template <typename T>
int vjp_pre_solve(VjpRun<T>& r, int it) {
  CVec5<T> xb;
  for (int q = 0; q < 5; ++q) xb.f[q] = it ? r.v.x2b[q] : r.v.x1b[q];
  return solve_t_prep<T>(r.c, r.cf, r.w.g, xb, nullptr, r.st);
}

// b_bar = A^-T x_bar into the corrector's cotangents (custom_linear_solve
// transpose, steppers.py:473-485), then corrector^T and predictor^T of solve it
template <typename T>
int vjp_post_solve(VjpRun<T>& r, int it, int rc, const SislSolveInfo& si) {
  SislCore* c = r.c;
  const Dims& d = c->d;
  const Coef<T>& cf = r.cf;
  SWork<T>& w = r.w;
  VWork<T>& v = r.v;
  cudaStream_t st = r.st;
  const SislState* in = r.in;
  const SislState* ib = r.ib;
  if (r.info) r.info->solve[it] = si;
  if (rc < 0 && rc != SISL_ERR_NONFINITE) return rc;
  if (rc != SISL_OK && r.status == SISL_OK) r.status = rc;
  Vec5<T> bo;
  for (int q = 0; q < 5; ++q) bo.f[q] = v.bb[q];
  solve_t_finish<T>(c, cf, w.g, bo, st);
  const T* u = (const T*)in->u;
  const T* vv = (const T*)in->v;
  const T* eta = (const T*)in->eta_dot;
  const T* pp = (const T*)in->pi_p;
  const T* x1[5];
  for (int q = 0; q < 5; ++q) x1[q] = (const T*)r.tape[q];
  T* ub = (T*)ib->u;
  T* vb = (T*)ib->v;
  T* wb = (T*)ib->w;
  T* eb = (T*)ib->eta_dot;
  T* pb = (T*)ib->pi_p;
  CorrectorIn<T> ci;
  ci.rhs_u = w.ru; ci.rhs_v = w.rv; ci.rhs_w = nullptr; ci.rhs_pi = nullptr;
  ci.th_next = it ? v.th2 : v.th1;
  ci.pg = it ? x1[3] : pp;
  ci.gu = it ? x1[0] : u;
  ci.gv = it ? x1[1] : vv;
  ci.geta = it ? x1[4] : eta;
  ci.ug = it ? x1[0] : w.ru;
  ci.vg = it ? x1[1] : w.rv;
  CorrectorBar<T> cb;
  for (int q = 0; q < 5; ++q) cb.b[q] = v.bb[q];
  cb.rhs_u = v.rub; cb.rhs_v = v.rvb; cb.rhs_w = v.rwb; cb.rhs_pi = v.rpb; cb.reta = v.reb;
  cb.th = it ? v.th2b : v.th1b;
  cb.pg = it ? v.x1b[3] : pb;
  cb.gu = it ? v.x1b[0] : ub;
  cb.gv = it ? v.x1b[1] : vb;
  cb.geta = it ? v.x1b[4] : eb;
  cb.ug = it ? v.x1b[0] : v.rub;
  cb.vg = it ? v.x1b[1] : v.rvb;
  KScope k(c, SISL_K_EXPLICIT, st, 4);  // corrector^T (max, fixed-point, finish) + predictor^T
  launch_corrector_vjp<T>(d, cf, ci, cb, v.det, st);
  // theta' predictor; the first predictor's w terms cancel (w_next = w)
  launch_corrector_theta_vjp<T>(d, cf, it ? v.th2b : v.th1b, v.thab, v.tthb, it ? wb : nullptr,
                                it ? v.x1b[2] : nullptr, st);
  return SISL_OK;
}

// lateral overrides, the six departure-point interpolation VJPs, explicit^T
// and hyperdiffusion^T
template <typename T>
int vjp_close(VjpRun<T>& r) {
  SislCore* c = r.c;
  const Dims& d = c->d;
  const Coef<T>& cf = r.cf;
  SWork<T>& w = r.w;
  VWork<T>& v = r.v;
  cudaStream_t st = r.st;
  const SislState* ib = r.ib;
  const double a = c->s.alpha;
  const int lim = c->prm.use_limiter;
  const bool hyp = r.hyp;
  const ExplicitIn<T>& ein = r.ein;
  T* ub = (T*)ib->u;
  T* vb = (T*)ib->v;
  T* wb = (T*)ib->w;
  T* eb = (T*)ib->eta_dot;
  T* pb = (T*)ib->pi_p;
  T* hb = (T*)ib->th_p;
  {  // lateral overrides, then the six departure-point interpolations
    KScope k(c, SISL_K_SL, st, 19);
    launch_fixup_vjp<T>(d, v.rub, v.rvb, ub, vb, v.reb, st);
    const T* cu[3] = {v.coords[3], v.coords[4], v.coords[5]};
    const T* cvv[3] = {v.coords[6], v.coords[7], v.coords[8]};
    const T* cwv[3] = {v.coords[9], v.coords[10], v.coords[11]};
    const T* cm[3] = {v.coords[0], v.coords[1], v.coords[2]};
    const int ux = d.nx + 1, vy = d.ny + 1, wz = d.nz + 1;
    // deterministic scatters (fixed-point sums): the cotangents are the same bits on every run
    launch_tricubic_vjp_det<T>(ux, d.ny, d.nz, ux, d.ny, d.nz, w.u_in, cu, v.rub, v.uinb, lim, T(1), v.det, 1, st);
    launch_tricubic_vjp_det<T>(d.nx, vy, d.nz, d.nx, vy, d.nz, w.v_in, cvv, v.rvb, v.vinb, lim, T(1), v.det, 1, st);
    launch_tricubic_vjp_det<T>(d.nx, d.ny, wz, d.nx, d.ny, wz, w.w_in, cwv, v.rwb, v.winb, lim, T(1), v.det, 1, st);
    launch_tricubic_vjp_det<T>(d.nx, d.ny, wz, d.nx, d.ny, wz, w.res, cwv, v.reb, v.resb, lim, (T)(-(1.0 - a)),
                               v.det, 1, st);
    launch_tricubic_vjp_det<T>(d.nx, d.ny, d.nz, d.nx, d.ny, d.nz, w.pi_in, cm, v.rpb, v.pinb, lim, T(1), v.det, 1, st);
    launch_tricubic_vjp_det<T>(d.nx, d.ny, d.nz, d.nx, d.ny, d.nz, w.th_in, cm, v.thab, v.thinb, lim, T(1), v.det,
                               1, st);
  }
  {  // explicit tendencies with hyperdiffusion (euler.py:208-372, diffusion.py:93-173)
    ExplicitBar<T> bi{};
    bi.f[0] = v.uinb; bi.f[1] = v.vinb; bi.f[2] = v.winb; bi.f[3] = v.pinb; bi.f[4] = v.thinb;
    bi.f[5] = v.tthb; bi.f[6] = v.resb;
    StateBar<T> so{ub, vb, wb, eb, pb, hb, {nullptr, nullptr, nullptr, nullptr}};
    if (hyp)
      for (int q = 0; q < 4; ++q) so.hyper[q] = v.hypb[q];
    KScope k(c, SISL_K_EXPLICIT, st, 3);  // max pass, fixed-point pass, finish
    launch_explicit_vjp<T>(d, cf, ein, bi, so, 0, v.det, st);
  }
  if (hyp) {
    PtrTable<T> h4{}, gx{}, gy{}, t4{};
    for (int q = 0; q < 4; ++q) { h4.p[q] = v.hypb[q]; gx.p[q] = v.gx4[q]; gy.p[q] = v.gy4[q]; t4.p[q] = v.tmp4[q]; }
    KScope k(c, SISL_K_EXPLICIT, st, 5);
    launch_hyper_vjp<T>(d, cf, h4, gx, gy, t4, ub, vb, wb, hb, st);
  }
  if (r.info) r.info->kernel_launches = g_launches.load() - r.l0;
  int e = check_cuda();
  return e ? e : r.status;
}

template <typename T>
int step_vjp_impl(SislCore* c, const SislState* in, void* const* tape, const SislRelaxation* relax,
                  const SislState* ob, const SislState* ib, void* ws, size_t ws_bytes, cudaStream_t st,
                  SislStepInfo* info, GDevInfo* dev_info = nullptr) {
  VjpRun<T> r;
  int rc = vjp_open<T>(r, c, in, tape, relax, ob, ib, ws, ws_bytes, st, info);
  if (rc || (rc = vjp_forward<T>(r))) return rc;
  for (int it = 1; it >= 0; --it) {
    if ((rc = vjp_pre_solve<T>(r, it))) return rc;
    SislSolveInfo si{};
    rc = gmres_run<T>(c, r.cf, r.w.g, st, &si, 1, dev_info ? dev_info + it : nullptr);
    if ((rc = vjp_post_solve<T>(r, it, rc, si))) return rc;
  }
  return vjp_close<T>(r);
}

bool valid_grid(const SislGrid* g) {
  return g && g->nx >= 2 && g->ny >= 2 && g->nz >= 2 && (g->dtype == SISL_F32 || g->dtype == SISL_F64) &&
         g->dx > 0 && g->dy > 0 && g->dz > 0 && (int64_t)(g->nx + 1) * (g->ny + 1) * (g->nz + 1) < (1LL << 31);
}

}  // namespace

// ===========================================================================
// C ABI
// ===========================================================================
namespace {

// Workspace of the split-explicit step: acoustic perturbations (two
// u''/v'' buffers swapped by the corrector), midpoint winds, the old
// pressure gradients, the slow forcings, the explicit kernel's outputs, the
// advection terms, the hyperdiffusion of the step start and of the stage,
// the Thomas sweep, and two stage states.
template <typename T>
struct SplitWork {
  T *upp, *upp2, *vpp, *vpp2, *wpp, *ppp, *uh, *vh, *gx0, *gy0, *gx1, *gy1;
  T* sf[5];
  T* tend[6];
  T* adv[4];
  T *hyp_t[4], *hyp_s[4], *htmp[4], *hgxy[8];
  T *cpr, *dpr;
  T* st[2][6];  // stage states: u, v, w, eta, pi', th'
};

template <typename T>
void carve_split(Carver& cv, const Dims& d, SplitWork<T>& w) {
  auto f = [&](int loc) { return (T*)cv.take(sizeof(T) * field_size(d, loc)); };
  w.upp = f(LOC_U); w.upp2 = f(LOC_U); w.vpp = f(LOC_V); w.vpp2 = f(LOC_V);
  w.wpp = f(LOC_W); w.ppp = f(LOC_M); w.uh = f(LOC_U); w.vh = f(LOC_V); w.gx0 = f(LOC_U); w.gy0 = f(LOC_V);
  w.gx1 = f(LOC_U); w.gy1 = f(LOC_V);
  const int sf_loc[5] = {LOC_U, LOC_V, LOC_W, LOC_M, LOC_M};
  for (int q = 0; q < 5; ++q) w.sf[q] = f(sf_loc[q]);
  const int t_loc[6] = {LOC_U, LOC_V, LOC_W, LOC_M, LOC_M, LOC_M};
  for (int q = 0; q < 6; ++q) w.tend[q] = f(t_loc[q]);
  for (int q = 0; q < 4; ++q) {
    w.adv[q] = f(LOC_M);
    w.hyp_t[q] = f(LOC_M);
    w.hyp_s[q] = f(LOC_M);
    w.htmp[q] = f(LOC_M);
  }
  for (int q = 0; q < 8; ++q) w.hgxy[q] = f(q < 4 ? LOC_U : LOC_V);
  w.cpr = f(LOC_M);
  w.dpr = f(LOC_M);
  const int s_loc[6] = {LOC_U, LOC_V, LOC_W, LOC_W, LOC_M, LOC_M};
  for (int b = 0; b < 2; ++b)
    for (int q = 0; q < 6; ++q) w.st[b][q] = f(s_loc[q]);
}

}  // namespace

namespace {

// steppers.py:1117-1231: hyperdiffusion and physics tendencies of the step
// start, then three stages of slow tendencies and acoustic sub-steps
// nstages < 3 (the reverse sweep's recomputation): stop after that many
// stages, whose states stay in the workspace (SplitWork::st)
template <typename T>
void split_step_impl(SislCore* c, const SislState* in, const SislState* out, int ns, double alpha, double eps_l,
                     const T* tau, const void* const* phys, void* ws, cudaStream_t st, int nstages = 3) {
  const Dims& d = c->d;
  const Coef<T> cf = coef_of<T>(c);
  Carver cv{(char*)ws};
  SplitWork<T> w;
  carve_split<T>(cv, d, w);
  const T* s0[6] = {(const T*)in->u, (const T*)in->v, (const T*)in->w, (const T*)in->eta_dot, (const T*)in->pi_p,
                    (const T*)in->th_p};
  T* dst_out[6] = {(T*)out->u, (T*)out->v, (T*)out->w, (T*)out->eta_dot, (T*)out->pi_p, (T*)out->th_p};
  // the HyperFilter of the step start (diff_tends); inside the stages the
  // explicit tendencies run with nu_h hidden, so their own hyperdiffusion
  // is on exactly when nu_div > 0 (euler.py:336), with the filter's nu_h
  const bool hyp_t = c->s.nu_h > 0.0, hyp_s = c->s.nu_h > 0.0 && c->s.nu_div > 0.0;
  auto table4 = [](T* const* a) {
    PtrTable<T> t{};
    for (int q = 0; q < 4; ++q) t.p[q] = a[q];
    return t;
  };
  PtrTable<T> g8{};
  for (int q = 0; q < 8; ++q) g8.p[q] = w.hgxy[q];
  if (hyp_t) {
    KScope k(c, SISL_K_EXPLICIT, st, 5);
    launch_hyper<T>(d, cf, s0[0], s0[1], s0[2], s0[5], table4(w.htmp), table4(w.hyp_t), g8, st);
  }
  const int nst[3] = {std::max(1, (int)std::nearbyint(ns / 3.0)), std::max(1, (int)std::nearbyint(ns / 2.0)), ns};
  const double dts[3] = {(c->s.dt / 3.0) / nst[0], (c->s.dt / 2.0) / nst[1], c->s.dt / nst[2]};
  const T* cur[6];
  for (int q = 0; q < 6; ++q) cur[q] = s0[q];
  for (int stage = 0; stage < nstages; ++stage) {
    T* const* dst = stage == 2 ? dst_out : w.st[stage];
    // ---- slow tendencies (steppers.py:1362-1465) ----
    const T* hyp[4] = {nullptr, nullptr, nullptr, nullptr};
    if (hyp_s) {
      KScope k(c, SISL_K_EXPLICIT, st, 5 + (hyp_t ? 4 : 0));
      launch_hyper<T>(d, cf, cur[0], cur[1], cur[2], cur[5], table4(w.htmp), table4(w.hyp_s), g8, st);
      if (hyp_t)
        for (int q = 0; q < 4; ++q) launch_split_axpy<T>(field_size(d, LOC_M), w.hyp_t[q], w.hyp_s[q], st);
      for (int q = 0; q < 4; ++q) hyp[q] = w.hyp_s[q];
    } else if (hyp_t) {
      for (int q = 0; q < 4; ++q) hyp[q] = w.hyp_t[q];
    }
    ExplicitIn<T> ein{cur[0], cur[1], cur[2], cur[3], cur[4], cur[5], {hyp[0], hyp[1], hyp[2], hyp[3]},
                      {nullptr, nullptr, nullptr, nullptr}};
    if (phys)
      for (int q = 0; q < 4; ++q) ein.extra[q] = (const T*)phys[q];
    ExplicitOut<T> eout{};
    for (int q = 0; q < 6; ++q) eout.f[q] = w.tend[q];
    {
      KScope k(c, SISL_K_EXPLICIT, st, 3);
      launch_explicit<T>(d, cf, ein, eout, 1, st);
      launch_split_adv<T>(d, cf, cur[0], cur[1], cur[2], cur[3], cur[5], (T)eps_l, w.adv, st);
      launch_split_slow<T>(d, (const T* const*)w.tend, (const T* const*)w.adv, w.sf, st);
    }
    // ---- acoustic sub-steps (steppers.py:1467-1633) ----
    SplitArgs<T> a{};
    a.u0 = s0[0]; a.v0 = s0[1]; a.w0 = s0[2]; a.p0 = s0[4]; a.th0 = s0[5];
    a.uc = cur[0]; a.vc = cur[1]; a.wc = cur[2]; a.pc = cur[4]; a.ec = cur[3];
    a.upp = w.upp; a.vpp = w.vpp; a.wpp = w.wpp; a.ppp = w.ppp;
    a.uh = w.uh; a.vh = w.vh; a.gx0 = w.gx0; a.gy0 = w.gy0; a.gx1 = w.gx1; a.gy1 = w.gy1;
    a.sfu = w.sf[0]; a.sfv = w.sf[1]; a.sfw = w.sf[2]; a.sfp = w.sf[3]; a.sfth = w.sf[4];
    a.tau = tau; a.cpr = w.cpr; a.dpr = w.dpr;
    a.dtau = (T)dts[stage]; a.alpha = (T)alpha; a.nu_div = (T)c->s.nu_div;
    T* spare_u = w.upp2;
    T* spare_v = w.vpp2;
    // algorithmic bytes, each distinct 3-D array once per kernel: init 12,
    // and per sub-step predictor 12 (16 on a stage's first sub-step, which
    // forms the pressure gradients from pi'' and the metric), column 24 (its
    // Thomas sweep written and read back once), corrector 24 (with the two
    // handed-over gradients)
    const double cellb = (double)sizeof(T) * d.nx * d.ny * d.nz;
    {
      KScope k(c, SISL_K_OTHER, st, 1 + 3 * nst[stage], cellb * (12.0 + 4.0 + 60.0 * nst[stage]));
      launch_split_init<T>(d, a, st);
      for (int n = 0; n < nst[stage]; ++n) {
        a.gx0_ready = n > 0;  // the previous corrector's gradients of this pi''
        launch_split_predict<T>(d, cf, a, st);
        launch_split_column<T>(d, cf, a, st);
        launch_split_correct<T>(d, cf, a, spare_u, spare_v, st);
        std::swap(a.upp, spare_u);
        std::swap(a.vpp, spare_v);
        std::swap(a.gx0, a.gx1);
        std::swap(a.gy0, a.gy1);
      }
    }
    {  // stage state (17 arrays) and its eta_dot diagnosis (8)
      KScope k(c, SISL_K_OTHER, st, stage < 2 ? 2 : 1, cellb * (stage < 2 ? 25.0 : 17.0));
      launch_split_end<T>(d, a, nst[stage], dst[0], dst[1], dst[2], dst[3], dst[4], dst[5], st);
      if (stage < 2) launch_split_diag<T>(d, cf, dst[0], dst[1], dst[2], dst[3], dst[2], st);
    }
    for (int q = 0; q < 6; ++q) cur[q] = dst[q];
  }
  if (nstages == 3 && out->rho && in->rho && out->rho != in->rho)
    cudaMemcpyAsync(out->rho, in->rho, sizeof(T) * field_size(d, LOC_M), cudaMemcpyDeviceToDevice, st);
}

// Reverse-sweep buffers of the split-explicit step (after SplitWork).
template <typename T>
struct SplitVjpWork {
  T* sb[2][6];  // stage-state cotangents (u, v, w, eta_dot, pi', th'), two sets
  T *upp[2], *vpp[2], *wpp, *ppp, *uh, *vh, *gx0, *gy0;
  T* sf[5];
  T* tend[6];
  T* adv[4];
  T *hyp[4], *hyp_t[4], *gx4[4], *gy4[4], *tmp4[4];
  T *s1, *s2;
  void* det;
};

template <typename T>
void carve_split_vjp(Carver& cv, const Dims& d, SplitVjpWork<T>& b) {
  auto f = [&](int loc) { return (T*)cv.take(sizeof(T) * field_size(d, loc)); };
  const int s_loc[6] = {LOC_U, LOC_V, LOC_W, LOC_W, LOC_M, LOC_M};
  for (int q = 0; q < 2; ++q)
    for (int r = 0; r < 6; ++r) b.sb[q][r] = f(s_loc[r]);
  for (int q = 0; q < 2; ++q) { b.upp[q] = f(LOC_U); b.vpp[q] = f(LOC_V); }
  b.wpp = f(LOC_W); b.ppp = f(LOC_M); b.uh = f(LOC_U); b.vh = f(LOC_V); b.gx0 = f(LOC_U); b.gy0 = f(LOC_V);
  const int sf_loc[5] = {LOC_U, LOC_V, LOC_W, LOC_M, LOC_M};
  for (int q = 0; q < 5; ++q) b.sf[q] = f(sf_loc[q]);
  const int t_loc[6] = {LOC_U, LOC_V, LOC_W, LOC_M, LOC_M, LOC_M};
  for (int q = 0; q < 6; ++q) b.tend[q] = f(t_loc[q]);
  for (int q = 0; q < 4; ++q) {
    b.adv[q] = f(LOC_M);
    b.hyp[q] = f(LOC_M);
    b.hyp_t[q] = f(LOC_M);
    b.tmp4[q] = f(LOC_M);
    b.gx4[q] = f(LOC_U);
    b.gy4[q] = f(LOC_V);
  }
  b.s1 = f(LOC_M);
  b.s2 = f(LOC_M);
  b.det = cv.take(det_scatter_scratch_bytes(d, (int)sizeof(T)));
}

// The reverse of split_step_impl (steppers.py:1117-1231 under XLA's VJP):
// recompute the first two stage states, then per stage from the last:
// eta_dot diagnosis^T, stage assembly^T, the acoustic sub-steps^T (linear:
// no recorded intermediates), their initialisation^T, the slow forcings^T,
// upwind advection^T and explicit tendencies^T at the stage start, and the
// hyperdiffusion^T of the stage and, at the end, of the step start.
template <typename T>
int split_vjp_impl(SislCore* c, const SislState* in, const SislState* ob, const SislState* ib, int ns, double alpha,
                   double eps_l, const T* tau, int deterministic, void* ws, size_t ws_bytes, cudaStream_t st) {
  const Dims& d = c->d;
  const Coef<T> cf = coef_of<T>(c);
  Carver cv{(char*)ws};
  SplitWork<T> w;
  carve_split<T>(cv, d, w);
  SplitVjpWork<T> b;
  carve_split_vjp<T>(cv, d, b);
  if (cv.off > ws_bytes) return SISL_ERR_WORKSPACE;
  if (!deterministic) b.det = nullptr;  // float atomic adds, one pass per scatter kernel
  static const int LOC6[6] = {LOC_U, LOC_V, LOC_W, LOC_W, LOC_M, LOC_M};
  auto bytes = [&](int loc) { return sizeof(T) * field_size(d, loc); };
  auto zero = [&](void* p, int loc) { return cudaMemsetAsync(p, 0, bytes(loc), st) == cudaSuccess; };
  // recompute the stage states 1 and 2 (into w.st)
  split_step_impl<T>(c, in, in, ns, alpha, eps_l, tau, nullptr, ws, st, 2);
  T* s0b[6] = {(T*)ib->u, (T*)ib->v, (T*)ib->w, (T*)ib->eta_dot, (T*)ib->pi_p, (T*)ib->th_p};
  const void* obv[6] = {ob->u, ob->v, ob->w, ob->eta_dot, ob->pi_p, ob->th_p};
  const T* s0[6] = {(const T*)in->u, (const T*)in->v, (const T*)in->w, (const T*)in->eta_dot, (const T*)in->pi_p,
                    (const T*)in->th_p};
  for (int q = 0; q < 6; ++q) {
    if (!zero(s0b[q], LOC6[q])) return SISL_ERR_CUDA;
    T* dst = b.sb[0][q];
    if (obv[q]) {
      if (cudaMemcpyAsync(dst, obv[q], bytes(LOC6[q]), cudaMemcpyDeviceToDevice, st) != cudaSuccess) return SISL_ERR_CUDA;
    } else if (!zero(dst, LOC6[q])) {
      return SISL_ERR_CUDA;
    }
  }
  const bool hyp_t = c->s.nu_h > 0.0, hyp_s = c->s.nu_h > 0.0 && c->s.nu_div > 0.0;
  if (hyp_t)
    for (int q = 0; q < 4; ++q)
      if (!zero(b.hyp_t[q], LOC_M)) return SISL_ERR_CUDA;
  const int nst[3] = {std::max(1, (int)std::nearbyint(ns / 3.0)), std::max(1, (int)std::nearbyint(ns / 2.0)), ns};
  const double dts[3] = {(c->s.dt / 3.0) / nst[0], (c->s.dt / 2.0) / nst[1], c->s.dt / nst[2]};
  const size_t nm = field_size(d, LOC_M);
  int D = 0;  // b.sb[D]: cotangents of the current stage's output
  for (int stage = 2; stage >= 0; --stage) {
    const T* const* cur = stage == 0 ? s0 : (const T* const*)w.st[stage - 1];
    T* const* Db = b.sb[D];
    T* const* Cb = b.sb[1 - D];
    for (int q = 0; q < 6; ++q)
      if (!zero(Cb[q], LOC6[q])) return SISL_ERR_CUDA;
    {
      KScope k(c, SISL_K_OTHER, st, 4);
      if (stage < 2) launch_split_diag_vjp<T>(d, cf, Db[2], Db[3], Db[0], Db[1], b.det, st);
      const T dtau = (T)dts[stage];
      const T dtns = (T)((double)dtau * nst[stage]);
      launch_split_end_vjp<T>(d, (const T* const*)Db, Cb, s0b[5], b.upp[0], b.vpp[0], b.wpp, b.ppp, b.sf[4], dtns,
                              st);
    }
    for (int q = 0; q < 4; ++q)
      if (!zero(b.sf[q], q == 0 ? LOC_U : (q == 1 ? LOC_V : (q == 2 ? LOC_W : LOC_M)))) return SISL_ERR_CUDA;
    SplitBar<T> a{};
    a.wpp = b.wpp; a.ppp = b.ppp; a.uh = b.uh; a.vh = b.vh; a.gx0 = b.gx0; a.gy0 = b.gy0;
    a.sfu = b.sf[0]; a.sfv = b.sf[1]; a.sfw = b.sf[2]; a.sfp = b.sf[3];
    a.uc = Cb[0]; a.vc = Cb[1]; a.wc = Cb[2]; a.u0 = s0b[0]; a.v0 = s0b[1];
    a.s1 = b.s1; a.s2 = b.s2; a.tau = tau;
    a.dtau = (T)dts[stage]; a.alpha = (T)alpha; a.nu_div = (T)c->s.nu_div;
    int A = 0;  // b.upp[A]: cotangent of u'' after the current sub-step
    for (int n = nst[stage] - 1; n >= 0; --n) {
      if (!zero(b.upp[1 - A], LOC_U) || !zero(b.vpp[1 - A], LOC_V) || !zero(b.uh, LOC_U) || !zero(b.vh, LOC_V) ||
          !zero(b.gx0, LOC_U) || !zero(b.gy0, LOC_V))
        return SISL_ERR_CUDA;
      a.upp2 = b.upp[A]; a.vpp2 = b.vpp[A];
      a.upp = b.upp[1 - A]; a.vpp = b.vpp[1 - A];
      KScope k(c, SISL_K_OTHER, st, 9);
      launch_split_substep_vjp<T>(d, cf, a, b.det, st);
      A = 1 - A;
    }
    {
      KScope k(c, SISL_K_OTHER, st, 6);
      launch_split_init_vjp<T>(d, b.upp[A], b.vpp[A], b.wpp, b.ppp, s0b, Cb, st);
      for (int q = 0; q < 4; ++q)
        if (!zero(b.adv[q], LOC_M)) return SISL_ERR_CUDA;
      launch_split_slow_vjp<T>(d, (const T* const*)b.sf, b.tend, b.adv, b.det, st);
      launch_split_adv_vjp<T>(d, cf, cur[0], cur[1], cur[2], cur[3], cur[5], (T)eps_l, (const T* const*)b.adv, Cb[0],
                              Cb[1], Cb[2], Cb[3], Cb[5], b.det, st);
    }
    // explicit tendencies (mode 1) at the stage start; their hyperdiffusion input
    const bool hyp = hyp_s || hyp_t;
    if (hyp)
      for (int q = 0; q < 4; ++q)
        if (!zero(b.hyp[q], LOC_M)) return SISL_ERR_CUDA;
    {
      ExplicitIn<T> ein{cur[0], cur[1], cur[2], cur[3], cur[4], cur[5], {nullptr, nullptr, nullptr, nullptr},
                        {nullptr, nullptr, nullptr, nullptr}};
      ExplicitBar<T> bi{};
      for (int q = 0; q < 6; ++q) bi.f[q] = b.tend[q];
      StateBar<T> so{Cb[0], Cb[1], Cb[2], Cb[3], Cb[4], Cb[5], {nullptr, nullptr, nullptr, nullptr}};
      if (hyp)
        for (int q = 0; q < 4; ++q) so.hyper[q] = b.hyp[q];
      KScope k(c, SISL_K_EXPLICIT, st, 3);
      launch_explicit_vjp<T>(d, cf, ein, bi, so, 1, b.det, st);
    }
    if (hyp_t && hyp) {  // hyp_s = hyper(stage) + hyp_t, or hyp_t alone
      KScope k(c, SISL_K_OTHER, st, 4);
      for (int q = 0; q < 4; ++q) launch_split_axpy<T>(nm, b.hyp[q], b.hyp_t[q], st);
    }
    if (hyp_s) {
      PtrTable<T> h4{}, gx{}, gy{}, t4{};
      for (int q = 0; q < 4; ++q) { h4.p[q] = b.hyp[q]; gx.p[q] = b.gx4[q]; gy.p[q] = b.gy4[q]; t4.p[q] = b.tmp4[q]; }
      KScope k(c, SISL_K_EXPLICIT, st, 5);
      launch_hyper_vjp<T>(d, cf, h4, gx, gy, t4, Cb[0], Cb[1], Cb[2], Cb[5], st);
    }
    if (stage == 0) {
      KScope k(c, SISL_K_OTHER, st, 6);
      for (int q = 0; q < 6; ++q) launch_split_axpy<T>(field_size(d, LOC6[q]), Cb[q], s0b[q], st);
    }
    D = 1 - D;
  }
  if (hyp_t) {
    PtrTable<T> h4{}, gx{}, gy{}, t4{};
    for (int q = 0; q < 4; ++q) { h4.p[q] = b.hyp_t[q]; gx.p[q] = b.gx4[q]; gy.p[q] = b.gy4[q]; t4.p[q] = b.tmp4[q]; }
    KScope k(c, SISL_K_EXPLICIT, st, 5);
    launch_hyper_vjp<T>(d, cf, h4, gx, gy, t4, s0b[0], s0b[1], s0b[2], s0b[5], st);
  }
  return check_cuda();
}

}  // namespace

extern "C" {

int sisl_version(void) { return 1; }

const char* sisl_last_error(void) { return g_last_error; }

const char* sisl_status_string(int s) {
  switch (s) {
    case SISL_OK: return "ok";
    case SISL_NOT_CONVERGED: return "GMRES did not reach its tolerance within maxiter restart cycles";
    case SISL_ERR_ARG: return "invalid argument";
    case SISL_ERR_CUDA: return "CUDA error";
    case SISL_ERR_WORKSPACE: return "workspace too small";
    case SISL_ERR_NONFINITE: return "non-finite residual";
    case SISL_ERR_SCRATCH_LIMIT: return "problem exceeds the fixed scratch of the allocation-free entry point";
    default: return "unknown status";
  }
}

size_t sisl_field_elems(const SislGrid* g, int loc) {
  if (!g || loc < 0 || loc > 3) return 0;
  Dims d{g->nx, g->ny, g->nz, g->periodic_x, g->periodic_y, g->dx, g->dy, g->dz};
  return field_size(d, loc);
}

int sisl_core_create(const SislGrid* grid, const SislParams* prm, const SislBackground* bg, void* stream,
                     SislCore** out) {
  if (!out || !valid_grid(grid) || !prm || !bg) return SISL_ERR_ARG;
  if (prm->solver_restart < 1 || prm->solver_restart > GM_MAXR || prm->solver_maxiter < 0) return SISL_ERR_ARG;
  if (prm->solve_method != SISL_GMRES_BATCHED && prm->solve_method != SISL_GMRES_INCREMENTAL) return SISL_ERR_ARG;
  const double* req[] = {bg->theta_bg, bg->pi_bg, bg->Z_m, bg->dz_m_full, bg->dz_w_full, bg->z_xi_w,
                         bg->z_eta_w, bg->tau_damp, bg->m_m, bg->m_u, bg->m_v, bg->f_u, bg->f_v,
                         bg->dm_dx_m, bg->dm_dy_m};
  for (const double* p : req)
    if (!p) return SISL_ERR_ARG;
  SislCore* c = new (std::nothrow) SislCore();
  if (!c) return SISL_ERR_ARG;
  c->grid = *grid;
  c->prm = *prm;
  c->d = Dims{grid->nx, grid->ny, grid->nz, grid->periodic_x ? 1 : 0, grid->periodic_y ? 1 : 0,
              grid->dx, grid->dy, grid->dz};
  c->s = Scalars{prm->dt, prm->alpha, prm->g, prm->cp, prm->Rd, prm->cvd, prm->p0, prm->pi_scale, prm->nu_div,
                 prm->nu_h};
  const size_t es = esize(grid->dtype);
  size_t total = 0, offs[C_COUNT];
  for (int q = 0; q < C_COUNT; ++q) {
    offs[q] = total;
    total += align256(es * coef_elems(c->d, q));
  }
  if (cudaMalloc(&c->coef_mem, total) != cudaSuccess) { delete c; return SISL_ERR_CUDA; }
  if (cudaMallocHost((void**)&c->hv, sizeof(GHostView)) != cudaSuccess) {
    cudaFree(c->coef_mem);
    delete c;
    return SISL_ERR_CUDA;
  }
  for (int q = 0; q < C_COUNT; ++q) c->coef_ptr[q] = (char*)c->coef_mem + offs[q];
  Base64 b{bg->theta_bg, bg->pi_bg, bg->Z_m, bg->dz_m_full, bg->dz_w_full, bg->z_xi_w, bg->z_eta_w, bg->tau_damp,
           bg->m_m, bg->m_u, bg->m_v, bg->f_u, bg->f_v, bg->dm_dx_m, bg->dm_dy_m, bg->rho_bg};
  cudaStream_t st = (cudaStream_t)stream;
  g_launches += 1;
  if (grid->dtype == SISL_F64) {
    PtrTable<double> t;
    for (int q = 0; q < C_COUNT; ++q) t.p[q] = (double*)c->coef_ptr[q];
    launch_prepare<double>(c->d, c->s, b, t, st);
  } else {
    PtrTable<float> t;
    for (int q = 0; q < C_COUNT; ++q) t.p[q] = (float*)c->coef_ptr[q];
    launch_prepare<float>(c->d, c->s, b, t, st);
  }
  if (grid->dtype == SISL_F32 && prm->refine) {  // float64 operator of the refinement
    size_t t64 = 0, o64[C_COUNT];
    for (int q = 0; q < C_COUNT; ++q) {
      o64[q] = t64;
      t64 += align256(sizeof(double) * coef_elems(c->d, q));
    }
    if (cudaMalloc(&c->coef64_mem, t64) == cudaSuccess) {
      for (int q = 0; q < C_COUNT; ++q) c->coef64_ptr[q] = (char*)c->coef64_mem + o64[q];
      PtrTable<double> t;
      for (int q = 0; q < C_COUNT; ++q) t.p[q] = (double*)c->coef64_ptr[q];
      g_launches += 1;
      launch_prepare<double>(c->d, c->s, b, t, st);
      c->refine_on = 1;
    } else {
      c->coef64_mem = nullptr;
    }
  }
  if (check_cuda() != SISL_OK || cudaStreamSynchronize(st) != cudaSuccess || (prm->refine && grid->dtype == SISL_F32 && !c->coef64_mem)) {
    cudaFree(c->coef_mem);
    if (c->coef64_mem) cudaFree(c->coef64_mem);
    cudaFreeHost(c->hv);
    delete c;
    return SISL_ERR_CUDA;
  }
  *out = c;
  return SISL_OK;
}

int sisl_core_destroy(SislCore* c) {
  if (!c) return SISL_ERR_ARG;
  for (size_t q = 0; q < c->ev0.size(); ++q) { cudaEventDestroy(c->ev0[q]); cudaEventDestroy(c->ev1[q]); }
  cudaFree(c->coef_mem);
  if (c->coef64_mem) cudaFree(c->coef64_mem);
  cudaFreeHost(c->hv);
  delete c;
  return SISL_OK;
}

size_t sisl_workspace_bytes(const SislCore* c, int what) {
  if (!c) return 0;
  Carver cv{nullptr};
  const bool f64 = c->grid.dtype == SISL_F64;
  const size_t es = esize(c->grid.dtype);
  switch (what) {
    case SISL_WS_STEP:
      if (f64) carve_step<double>(cv, c->d, c->prm.solver_restart, false);
      else carve_step<float>(cv, c->d, c->prm.solver_restart, refining<float>(c));
      break;
    case SISL_WS_GMRES:
      if (f64) carve_gmres<double>(cv, c->d, c->prm.solver_restart, false);
      else carve_gmres<float>(cv, c->d, c->prm.solver_restart, refining<float>(c));
      break;
    case SISL_WS_DEPARTURE:
      for (int l = 0; l < 4; ++l)
        for (int q = 0; q < 3; ++q) cv.take(es * field_size(c->d, l));
      break;
    case SISL_WS_EXPLICIT:
      for (int q = 0; q < 8; ++q) cv.take(es * field_size(c->d, LOC_M));
      for (int q = 0; q < 8; ++q) cv.take(es * field_size(c->d, q < 4 ? LOC_U : LOC_V));
      break;
    case SISL_WS_OPERATOR:
      for (int q = 0; q < 5; ++q) cv.take(es * field_size(c->d, loc_of_field(q)));
      break;
    case SISL_WS_FFSL:
      cv.take(es * field_size(c->d, LOC_M));
      cv.take(es * field_size(c->d, LOC_M));
      cv.take(sizeof(double) * ffsl_scratch_doubles(c->d));
      break;
    case SISL_WS_STEP_VJP:
      if (f64) {
        carve_step<double>(cv, c->d, c->prm.solver_restart, false);
        carve_vjp<double>(cv, c->d);
      } else {
        carve_step<float>(cv, c->d, c->prm.solver_restart, refining<float>(c));
        carve_vjp<float>(cv, c->d);
      }
      break;
    case SISL_WS_SPLIT:
      if (f64) {
        SplitWork<double> w;
        carve_split<double>(cv, c->d, w);
      } else {
        SplitWork<float> w;
        carve_split<float>(cv, c->d, w);
      }
      break;
    case SISL_WS_SPLIT_VJP:
      if (f64) {
        SplitWork<double> w;
        carve_split<double>(cv, c->d, w);
        SplitVjpWork<double> b;
        carve_split_vjp<double>(cv, c->d, b);
      } else {
        SplitWork<float> w;
        carve_split<float>(cv, c->d, w);
        SplitVjpWork<float> b;
        carve_split_vjp<float>(cv, c->d, b);
      }
      break;
    case SISL_WS_FFSL_VJP:
      for (int q = 0; q < 5; ++q) cv.take(es * field_size(c->d, LOC_M));
      cv.take(sizeof(double) * ffsl_scratch_doubles(c->d));
      cv.take(sizeof(double) * ffsl_scratch_doubles(c->d));
      break;
    case SISL_WS_EXPLICIT_VJP:
      for (int q = 0; q < 8; ++q) cv.take(es * field_size(c->d, LOC_M));
      for (int q = 0; q < 4; ++q) cv.take(es * field_size(c->d, LOC_U));
      for (int q = 0; q < 4; ++q) cv.take(es * field_size(c->d, LOC_V));
      cv.take(det_scatter_scratch_bytes(c->d, (int)es));
      break;
    default: return 0;
  }
  return align256(cv.off);
}

int sisl_linear_operator(SislCore* c, const void* const in[5], void* const out[5], void* ws, size_t ws_bytes,
                         void* stream) {
  if (!c || !in || !out) return SISL_ERR_ARG;
  if (ws_bad(ws, ws_bytes, sisl_workspace_bytes(c, SISL_WS_OPERATOR))) return SISL_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  Carver cv{(char*)ws};
  auto run = [&](auto tag) {
    using T = decltype(tag);
    const Coef<T> cf = coef_of<T>(c);
    Vec5<T> tmp;
    for (int q = 0; q < 5; ++q) tmp.f[q] = (T*)cv.take(sizeof(T) * field_size(c->d, loc_of_field(q)));
    scale5<T>(c, cf, cvec<T>(in), tmp, (T)c->s.ps, 1, st);
    {
      KScope k(c, SISL_K_MATVEC, st);
      launch_matvec<T>(c->d, cf, as_const(tmp), nullptr, CVec5<T>{}, vec<T>(out), nullptr, st);
    }
    // pi row back to physical units; the eta row of A_fn is already physical
    Vec5<T> o = vec<T>(out);
    scale5<T>(c, cf, as_const(o), o, (T)(1.0 / c->s.ps), 0, st);
  };
  if (c->grid.dtype == SISL_F64) run(double{});
  else run(float{});
  return check_cuda();
}

int sisl_helmholtz_matvec(SislCore* c, const void* const in[5], void* const out[5], void* stream) {
  if (!c || !in || !out) return SISL_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  KScope k(c, SISL_K_MATVEC, st);
  if (c->grid.dtype == SISL_F64)
    launch_matvec<double>(c->d, coef_of<double>(c), cvec<double>(in), nullptr, CVec5<double>{}, vec<double>(out),
                          nullptr, st);
  else
    launch_matvec<float>(c->d, coef_of<float>(c), cvec<float>(in), nullptr, CVec5<float>{}, vec<float>(out),
                         nullptr, st);
  return check_cuda();
}

int sisl_precond_apply(SislCore* c, const void* const in[5], void* const out[5], void* stream) {
  if (!c || !in || !out) return SISL_ERR_ARG;
  for (int q = 2; q < 5; ++q)
    if (in[q] == out[q]) return SISL_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  KScope k(c, SISL_K_PRECOND, st);
  if (c->grid.dtype == SISL_F64)
    launch_precond<double>(c->d, coef_of<double>(c), cvec<double>(in), vec<double>(out), nullptr, st);
  else
    launch_precond<float>(c->d, coef_of<float>(c), cvec<float>(in), vec<float>(out), nullptr, st);
  return check_cuda();
}

int sisl_gmres_solve(SislCore* c, const void* const rhs[5], const void* const x0[5], void* const x[5], void* ws,
                     size_t ws_bytes, void* stream, SislSolveInfo* info) {
  if (!c || !rhs || !x) return SISL_ERR_ARG;
  if (ws_bad(ws, ws_bytes, sisl_workspace_bytes(c, SISL_WS_GMRES))) return SISL_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  Carver cv{(char*)ws};
  int rc;
  if (c->grid.dtype == SISL_F64) {
    GWork<double> g = carve_gmres<double>(cv, c->d, c->prm.solver_restart, false);
    CVec5<double> x0v;
    if (x0) x0v = cvec<double>(x0);
    rc = solve_physical<double>(c, coef_of<double>(c), g, cvec<double>(rhs), x0 ? &x0v : nullptr, vec<double>(x),
                                st, info);
  } else {
    GWork<float> g = carve_gmres<float>(cv, c->d, c->prm.solver_restart, refining<float>(c));
    CVec5<float> x0v;
    if (x0) x0v = cvec<float>(x0);
    rc = solve_physical<float>(c, coef_of<float>(c), g, cvec<float>(rhs), x0 ? &x0v : nullptr, vec<float>(x), st,
                               info);
  }
  int e = check_cuda();
  return e ? e : rc;
}

int sisl_helmholtz_matvec_t(SislCore* c, const void* const in[5], void* const out[5], void* ws, size_t ws_bytes,
                            void* stream) {
  if (!c || !in || !out) return SISL_ERR_ARG;
  for (int q = 0; q < 5; ++q)
    if (in[q] == out[q]) return SISL_ERR_ARG;
  if (ws_bad(ws, ws_bytes, sisl_workspace_bytes(c, SISL_WS_OPERATOR))) return SISL_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  KScope k(c, SISL_K_MATVEC, st, 2);
  if (c->grid.dtype == SISL_F64)
    launch_matvec_t<double>(c->d, coef_of<double>(c), cvec<double>(in), nullptr, CVec5<double>{}, vec<double>(out),
                            (double*)ws, nullptr, st);
  else
    launch_matvec_t<float>(c->d, coef_of<float>(c), cvec<float>(in), nullptr, CVec5<float>{}, vec<float>(out),
                           (float*)ws, nullptr, st);
  return check_cuda();
}

int sisl_precond_apply_t(SislCore* c, const void* const in[5], void* const out[5], void* stream) {
  if (!c || !in || !out) return SISL_ERR_ARG;
  for (int q = 0; q < 5; ++q)
    if (in[q] == out[q]) return SISL_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  KScope k(c, SISL_K_PRECOND, st, 2);
  if (c->grid.dtype == SISL_F64)
    launch_precond_t<double>(c->d, coef_of<double>(c), cvec<double>(in), vec<double>(out), nullptr, st);
  else
    launch_precond_t<float>(c->d, coef_of<float>(c), cvec<float>(in), vec<float>(out), nullptr, st);
  return check_cuda();
}

int sisl_gmres_solve_transpose(SislCore* c, const void* const xbar[5], const void* const x0[5],
                               void* const bbar[5], void* ws, size_t ws_bytes, void* stream, SislSolveInfo* info) {
  if (!c || !xbar || !bbar) return SISL_ERR_ARG;
  if (ws_bad(ws, ws_bytes, sisl_workspace_bytes(c, SISL_WS_GMRES))) return SISL_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  Carver cv{(char*)ws};
  int rc;
  if (c->grid.dtype == SISL_F64) {
    GWork<double> g = carve_gmres<double>(cv, c->d, c->prm.solver_restart, false);
    CVec5<double> x0v;
    if (x0) x0v = cvec<double>(x0);
    rc = solve_transpose_physical<double>(c, coef_of<double>(c), g, cvec<double>(xbar), x0 ? &x0v : nullptr,
                                          vec<double>(bbar), st, info);
  } else {
    GWork<float> g = carve_gmres<float>(cv, c->d, c->prm.solver_restart, refining<float>(c));
    CVec5<float> x0v;
    if (x0) x0v = cvec<float>(x0);
    rc = solve_transpose_physical<float>(c, coef_of<float>(c), g, cvec<float>(xbar), x0 ? &x0v : nullptr,
                                         vec<float>(bbar), st, info);
  }
  int e = check_cuda();
  return e ? e : rc;
}

int sisl_departure(SislCore* c, int loc, const void* u, const void* v, const void* eta, int iterations,
                   void* const coords[3], void* ws, size_t ws_bytes, void* stream) {
  if (!c || loc < 0 || loc > 3 || !u || !v || !eta || !coords || iterations < 0) return SISL_ERR_ARG;
  if (ws_bad(ws, ws_bytes, sisl_workspace_bytes(c, SISL_WS_DEPARTURE))) return SISL_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  Carver cv{(char*)ws};
  auto run = [&](auto tag) {
    using T = decltype(tag);
    const Coef<T> cf = coef_of<T>(c);
    PtrTable<T> vt{};  // only the requested stagger's index velocities
    for (int q = 0; q < 3; ++q) vt.p[3 * loc + q] = (T*)cv.take(sizeof(T) * field_size(c->d, loc));
    {
      KScope k(c, SISL_K_SL, st);
      launch_traj_velocity<T>(c->d, cf, (const T*)u, (const T*)v, (const T*)eta, nullptr, nullptr, nullptr, 0, vt,
                              st);
    }
    T* co[3] = {(T*)coords[0], (T*)coords[1], (T*)coords[2]};
    KScope k(c, SISL_K_SL, st);
    launch_departure<T>(c->d, loc, c->s.dt, (const T* const*)(vt.p + 3 * loc), iterations, co, 0, st);
  };
  if (c->grid.dtype == SISL_F64) run(double{});
  else run(float{});
  return check_cuda();
}

int sisl_tricubic(int dtype, const int32_t src[3], const void* field, const int32_t dst[3],
                  const void* const coords[3], void* out, int use_limiter, void* stream) {
  if (!src || !dst || !field || !coords || !out) return SISL_ERR_ARG;
  for (int q = 0; q < 3; ++q)
    if (src[q] < 1 || dst[q] < 0) return SISL_ERR_ARG;
  if ((int64_t)dst[0] * dst[1] * dst[2] == 0) return SISL_OK;
  cudaStream_t st = (cudaStream_t)stream;
  KScope k(nullptr, SISL_K_SL, st);
  if (dtype == SISL_F64) {
    const double* co[3] = {(const double*)coords[0], (const double*)coords[1], (const double*)coords[2]};
    launch_tricubic_ext<double>(src[0], src[1], src[2], dst[0], dst[1], dst[2], (const double*)field, co,
                                (double*)out, use_limiter, 1.0, st);
  } else if (dtype == SISL_F32) {
    const float* co[3] = {(const float*)coords[0], (const float*)coords[1], (const float*)coords[2]};
    launch_tricubic_ext<float>(src[0], src[1], src[2], dst[0], dst[1], dst[2], (const float*)field, co,
                               (float*)out, use_limiter, 1.0f, st);
  } else {
    return SISL_ERR_ARG;
  }
  return check_cuda();
}

int sisl_tricubic_vjp(int dtype, const int32_t src[3], const void* field, const int32_t dst[3],
                      const void* const coords[3], const void* cot, void* grad, int use_limiter, double scale,
                      void* stream) {
  if (!src || !dst || !coords || !cot || !grad || (use_limiter && !field)) return SISL_ERR_ARG;
  for (int q = 0; q < 3; ++q)
    if (src[q] < 1 || dst[q] < 0) return SISL_ERR_ARG;
  if ((int64_t)dst[0] * dst[1] * dst[2] == 0) return SISL_OK;
  cudaStream_t st = (cudaStream_t)stream;
  KScope k(nullptr, SISL_K_SL, st);
  if (dtype == SISL_F64) {
    const double* co[3] = {(const double*)coords[0], (const double*)coords[1], (const double*)coords[2]};
    launch_tricubic_vjp<double>(src[0], src[1], src[2], dst[0], dst[1], dst[2], (const double*)field, co,
                                (const double*)cot, (double*)grad, use_limiter, scale, st);
  } else if (dtype == SISL_F32) {
    const float* co[3] = {(const float*)coords[0], (const float*)coords[1], (const float*)coords[2]};
    launch_tricubic_vjp<float>(src[0], src[1], src[2], dst[0], dst[1], dst[2], (const float*)field, co,
                               (const float*)cot, (float*)grad, use_limiter, (float)scale, st);
  } else {
    return SISL_ERR_ARG;
  }
  return check_cuda();
}

size_t sisl_tricubic_vjp_workspace_bytes(int dtype, const int32_t src[3]) {
  if (!src || src[0] < 1 || src[1] < 1 || src[2] < 1 || (dtype != SISL_F32 && dtype != SISL_F64)) return 0;
  return tricubic_vjp_det_scratch_bytes(src[0], src[1], src[2], dtype == SISL_F64 ? 8 : 4);
}

int sisl_tricubic_vjp_deterministic(int dtype, const int32_t src[3], const void* field, const int32_t dst[3],
                                    const void* const coords[3], const void* cot, void* grad, int use_limiter,
                                    double scale, void* ws, size_t ws_bytes, void* stream) {
  if (!src || !dst || !coords || !cot || !grad || (use_limiter && !field)) return SISL_ERR_ARG;
  if (dtype != SISL_F32 && dtype != SISL_F64) return SISL_ERR_ARG;
  for (int q = 0; q < 3; ++q)
    if (src[q] < 1 || dst[q] < 0) return SISL_ERR_ARG;
  if ((int64_t)dst[0] * dst[1] * dst[2] == 0) return SISL_OK;
  if (!ws || ((uintptr_t)ws & 255) || ws_bytes < sisl_tricubic_vjp_workspace_bytes(dtype, src))
    return SISL_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  KScope k(nullptr, SISL_K_SL, st, 3);
  if (dtype == SISL_F64) {
    const double* co[3] = {(const double*)coords[0], (const double*)coords[1], (const double*)coords[2]};
    launch_tricubic_vjp_det<double>(src[0], src[1], src[2], dst[0], dst[1], dst[2], (const double*)field, co,
                                    (const double*)cot, (double*)grad, use_limiter, scale, ws, 0, st);
  } else {
    const float* co[3] = {(const float*)coords[0], (const float*)coords[1], (const float*)coords[2]};
    launch_tricubic_vjp_det<float>(src[0], src[1], src[2], dst[0], dst[1], dst[2], (const float*)field, co,
                                   (const float*)cot, (float*)grad, use_limiter, (float)scale, ws, 0, st);
  }
  return check_cuda();
}

int sisl_stagger(int dtype, int op, const int32_t in_shape[3], int axis, int to_face, int periodic, int stop_grad,
                 int transpose, double inv_delta, const void* mult, const void* src, void* dst, void* stream) {
  if (!in_shape || !src || !dst || axis < 0 || axis > 2 || (op != SISL_STAGGER_AVG && op != SISL_STAGGER_DIFF))
    return SISL_ERR_ARG;
  for (int q = 0; q < 3; ++q)
    if (in_shape[q] < 1) return SISL_ERR_ARG;
  if (in_shape[axis] < 2) return SISL_ERR_ARG;
  if (periodic && (axis == 2 || !to_face)) periodic = 0;
  const int sh[3] = {in_shape[0], in_shape[1], in_shape[2]};
  const double c0 = op == SISL_STAGGER_AVG ? 0.5 : -inv_delta, c1 = op == SISL_STAGGER_AVG ? 0.5 : inv_delta;
  cudaStream_t st = (cudaStream_t)stream;
  KScope k(nullptr, SISL_K_EXPLICIT, st);
  if (dtype == SISL_F64)
    launch_stagger<double>(sh, axis, to_face ? 1 : 0, periodic ? 1 : 0, stop_grad ? 1 : 0, transpose ? 1 : 0, c0,
                           c1, (const double*)mult, (const double*)src, (double*)dst, st);
  else if (dtype == SISL_F32)
    launch_stagger<float>(sh, axis, to_face ? 1 : 0, periodic ? 1 : 0, stop_grad ? 1 : 0, transpose ? 1 : 0,
                          (float)c0, (float)c1, (const float*)mult, (const float*)src, (float*)dst, st);
  else
    return SISL_ERR_ARG;
  return check_cuda();
}

int sisl_trilinear(int dtype, const int32_t src[3], const void* field, const int32_t dst[3],
                   const void* const coords[3], void* out, void* stream) {
  if (!src || !dst || !field || !coords || !out) return SISL_ERR_ARG;
  for (int q = 0; q < 3; ++q)
    if (src[q] < 1 || dst[q] < 0) return SISL_ERR_ARG;
  if ((int64_t)dst[0] * dst[1] * dst[2] == 0) return SISL_OK;
  cudaStream_t st = (cudaStream_t)stream;
  KScope k(nullptr, SISL_K_SL, st);
  if (dtype == SISL_F64) {
    const double* co[3] = {(const double*)coords[0], (const double*)coords[1], (const double*)coords[2]};
    launch_trilinear_ext<double>(src[0], src[1], src[2], dst[0], dst[1], dst[2], (const double*)field, co,
                                 (double*)out, st);
  } else if (dtype == SISL_F32) {
    const float* co[3] = {(const float*)coords[0], (const float*)coords[1], (const float*)coords[2]};
    launch_trilinear_ext<float>(src[0], src[1], src[2], dst[0], dst[1], dst[2], (const float*)field, co,
                                (float*)out, st);
  } else {
    return SISL_ERR_ARG;
  }
  return check_cuda();
}

size_t sisl_ffsl_lines_workspace_bytes(int n, int nlines) {
  if (n < 1 || nlines < 1) return 0;
  return align256(sizeof(double) * (size_t)(n + 1) * nlines);
}

int sisl_ffsl_lines(int dtype, int n, int nlines, const void* scalar, const void* cfl, int periodic, void* out,
                    void* ws, size_t ws_bytes, void* stream) {
  if (n < 1 || nlines < 1 || !scalar || !cfl || !out) return SISL_ERR_ARG;
  if (ws_bad(ws, ws_bytes, sisl_ffsl_lines_workspace_bytes(n, nlines))) return SISL_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  KScope k(nullptr, SISL_K_OTHER, st);
  if (dtype == SISL_F64)
    launch_ffsl_lines<double>(n, nlines, (const double*)scalar, (const double*)cfl, (double*)out, (double*)ws,
                              periodic ? 1 : 0, st);
  else if (dtype == SISL_F32)
    launch_ffsl_lines<float>(n, nlines, (const float*)scalar, (const float*)cfl, (float*)out, (double*)ws,
                             periodic ? 1 : 0, st);
  else
    return SISL_ERR_ARG;
  return check_cuda();
}

size_t sisl_ffsl_lines_vjp_workspace_bytes(int n, int nlines) {
  if (n < 1 || nlines < 1) return 0;
  return 2 * align256(sizeof(double) * (size_t)(n + 1) * nlines);
}

int sisl_ffsl_lines_vjp(int dtype, int n, int nlines, const void* scalar, const void* cfl, int periodic,
                        const void* out_bar, void* scalar_bar, void* cfl_bar, void* ws, size_t ws_bytes,
                        void* stream) {
  if (n < 1 || nlines < 1 || !scalar || !cfl || !out_bar || !scalar_bar) return SISL_ERR_ARG;
  if (ws_bad(ws, ws_bytes, sisl_ffsl_lines_vjp_workspace_bytes(n, nlines))) return SISL_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  double* M = (double*)ws;
  double* Mb = (double*)((char*)ws + align256(sizeof(double) * (size_t)(n + 1) * nlines));
  KScope k(nullptr, SISL_K_OTHER, st);
  if (dtype == SISL_F64)
    launch_ffsl_lines_vjp<double>(n, nlines, (const double*)scalar, (const double*)cfl, (const double*)out_bar,
                                  (double*)scalar_bar, (double*)cfl_bar, M, Mb, periodic ? 1 : 0, st);
  else if (dtype == SISL_F32)
    launch_ffsl_lines_vjp<float>(n, nlines, (const float*)scalar, (const float*)cfl, (const float*)out_bar,
                                 (float*)scalar_bar, (float*)cfl_bar, M, Mb, periodic ? 1 : 0, st);
  else
    return SISL_ERR_ARG;
  return check_cuda();
}

int sisl_explicit_tendencies(SislCore* c, const void* const sp[6], void* const tend[6], void* const pd[4], void* ws,
                             size_t ws_bytes, void* stream) {
  return sisl_tendencies(c, 1, sp, tend, pd, ws, ws_bytes, stream);
}

int sisl_metric_curvature(SislCore* c, const void* u, const void* v, void* out_u, void* out_v, void* stream) {
  if (!c || !u || !v || !out_u || !out_v) return SISL_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  KScope k(c, SISL_K_EXPLICIT, st);
  if (c->grid.dtype == SISL_F64)
    launch_curvature<double>(c->d, coef_of<double>(c), (const double*)u, (const double*)v, (double*)out_u,
                             (double*)out_v, st);
  else
    launch_curvature<float>(c->d, coef_of<float>(c), (const float*)u, (const float*)v, (float*)out_u,
                            (float*)out_v, st);
  return check_cuda();
}

int sisl_tendencies(SislCore* c, int is_explicit, const void* const sp[6], void* const tend[6],
                    void* const pd[4], void* ws, size_t ws_bytes, void* stream) {
  if (!c || !sp || !tend) return SISL_ERR_ARG;
  if (ws_bad(ws, ws_bytes, sisl_workspace_bytes(c, SISL_WS_EXPLICIT))) return SISL_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  Carver cv{(char*)ws};
  auto run = [&](auto tag) {
    using T = decltype(tag);
    const Coef<T> cf = coef_of<T>(c);
    ExplicitIn<T> ein{(const T*)sp[0], (const T*)sp[1], (const T*)sp[2], (const T*)sp[4], (const T*)sp[3],
                      (const T*)sp[5], {nullptr, nullptr, nullptr, nullptr}};
    if (is_explicit && (c->s.nu_h > 0.0 || c->s.nu_div > 0.0)) {
      PtrTable<T> t4{}, o4{};
      for (int q = 0; q < 4; ++q) o4.p[q] = (T*)cv.take(sizeof(T) * field_size(c->d, LOC_M));
      for (int q = 0; q < 4; ++q) t4.p[q] = (T*)cv.take(sizeof(T) * field_size(c->d, LOC_M));
      PtrTable<T> g8{};
      for (int q = 0; q < 8; ++q) g8.p[q] = (T*)cv.take(sizeof(T) * field_size(c->d, q < 4 ? LOC_U : LOC_V));
      KScope k(c, SISL_K_EXPLICIT, st, 5);
      launch_hyper<T>(c->d, cf, ein.u, ein.v, ein.w, ein.th, t4, o4, g8, st);
      for (int q = 0; q < 4; ++q) ein.hyper[q] = o4.p[q];
    }
    ExplicitOut<T> eo{};
    for (int q = 0; q < 6; ++q) eo.f[q] = (T*)tend[q];
    for (int q = 0; q < 4; ++q) eo.pd[q] = pd ? (T*)pd[q] : nullptr;
    KScope k(c, SISL_K_EXPLICIT, st);
    launch_explicit<T>(c->d, cf, ein, eo, is_explicit ? 1 : 2, st);
  };
  if (c->grid.dtype == SISL_F64) run(double{});
  else run(float{});
  return check_cuda();
}

int sisl_step(SislCore* c, const SislState* in, const SislState* out, const SislRelaxation* relax, void* ws,
              size_t ws_bytes, void* stream, SislStepInfo* info) {
  return sisl_step_taped(c, in, out, relax, nullptr, ws, ws_bytes, stream, info);
}

int sisl_step_taped(SislCore* c, const SislState* in, const SislState* out, const SislRelaxation* relax,
                    void* const solves[10], void* ws, size_t ws_bytes, void* stream, SislStepInfo* info) {
  if (!c || !in || !out) return SISL_ERR_ARG;
  const void* need_in[] = {in->u, in->v, in->w, in->eta_dot, in->pi_p, in->th_p};
  for (const void* p : need_in)
    if (!p) return SISL_ERR_ARG;
  if (in->is_first_step != 1.0 && (!in->u_prev || !in->v_prev || !in->eta_dot_prev)) return SISL_ERR_ARG;
  const void* need_out[] = {out->u, out->v, out->w, out->eta_dot, out->pi_p, out->th_p};
  for (const void* p : need_out)
    if (!p) return SISL_ERR_ARG;
  if (ws_bad(ws, ws_bytes, sisl_workspace_bytes(c, SISL_WS_STEP))) return SISL_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  if (c->grid.dtype == SISL_F64) return step_impl<double>(c, in, out, relax, ws, ws_bytes, st, info, solves);
  return step_impl<float>(c, in, out, relax, ws, ws_bytes, st, info, solves);
}

int sisl_step_physics(SislCore* c, const SislState* in, const SislState* out, const SislRelaxation* relax,
                      const void* const phys_tend[4], void* const solves[10], void* ws, size_t ws_bytes,
                      void* stream, SislStepInfo* info) {
  if (!c || !in || !out || !phys_tend) return SISL_ERR_ARG;
  const void* need_in[] = {in->u, in->v, in->w, in->eta_dot, in->pi_p, in->th_p};
  for (const void* p : need_in)
    if (!p) return SISL_ERR_ARG;
  if (in->is_first_step != 1.0 && (!in->u_prev || !in->v_prev || !in->eta_dot_prev)) return SISL_ERR_ARG;
  const void* need_out[] = {out->u, out->v, out->w, out->eta_dot, out->pi_p, out->th_p};
  for (const void* p : need_out)
    if (!p) return SISL_ERR_ARG;
  if (ws_bad(ws, ws_bytes, sisl_workspace_bytes(c, SISL_WS_STEP))) return SISL_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  if (c->grid.dtype == SISL_F64)
    return step_impl<double>(c, in, out, relax, ws, ws_bytes, st, info, solves, nullptr, phys_tend);
  return step_impl<float>(c, in, out, relax, ws, ws_bytes, st, info, solves, nullptr, phys_tend);
}

int sisl_step_vjp(SislCore* c, const SislState* in, void* const solves[10], const SislRelaxation* relax,
                  const SislState* out_bar, const SislState* in_bar, void* ws, size_t ws_bytes, void* stream,
                  SislStepInfo* info) {
  if (!c || !in || !solves || !out_bar || !in_bar) return SISL_ERR_ARG;
  const void* need_in[] = {in->u, in->v, in->w, in->eta_dot, in->pi_p, in->th_p};
  for (const void* p : need_in)
    if (!p) return SISL_ERR_ARG;
  if (in->is_first_step != 1.0 && (!in->u_prev || !in->v_prev || !in->eta_dot_prev)) return SISL_ERR_ARG;
  for (int q = 0; q < 10; ++q)
    if (!solves[q]) return SISL_ERR_ARG;
  const void* need_bar[] = {in_bar->u, in_bar->v, in_bar->w, in_bar->eta_dot, in_bar->pi_p, in_bar->th_p};
  for (const void* p : need_bar)
    if (!p) return SISL_ERR_ARG;
  if (relax && (((relax->fields & (SISL_RELAX_W | SISL_RELAX_TH | SISL_RELAX_PI)) && !relax->mask_m) ||
                ((relax->fields & SISL_RELAX_U) && !relax->mask_u) ||
                ((relax->fields & SISL_RELAX_V) && !relax->mask_v)))
    return SISL_ERR_ARG;
  if (ws_bad(ws, ws_bytes, sisl_workspace_bytes(c, SISL_WS_STEP_VJP))) return SISL_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  if (c->grid.dtype == SISL_F64)
    return step_vjp_impl<double>(c, in, solves, relax, out_bar, in_bar, ws, ws_bytes, st, info);
  return step_vjp_impl<float>(c, in, solves, relax, out_bar, in_bar, ws, ws_bytes, st, info);
}

int sisl_explicit_tendencies_vjp(SislCore* c, const void* const sp[6], const void* const tend_bar[6],
                                 const void* const pd_bar[4], void* const sp_bar[6], void* ws, size_t ws_bytes,
                                 void* stream) {
  if (!c || !sp || !tend_bar || !sp_bar) return SISL_ERR_ARG;
  for (int q = 0; q < 6; ++q)
    if (!sp[q] || !sp_bar[q]) return SISL_ERR_ARG;
  if (ws_bad(ws, ws_bytes, sisl_workspace_bytes(c, SISL_WS_EXPLICIT_VJP))) return SISL_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  static const int LOCS[6] = {LOC_U, LOC_V, LOC_W, LOC_M, LOC_W, LOC_M};
  Carver cv{(char*)ws};
  auto run = [&](auto tag) -> int {
    using T = decltype(tag);
    const Dims& d = c->d;
    const Coef<T> cf = coef_of<T>(c);
    for (int q = 0; q < 6; ++q)
      if (cudaMemsetAsync(sp_bar[q], 0, sizeof(T) * field_size(d, LOCS[q]), st) != cudaSuccess) return SISL_ERR_CUDA;
    PtrTable<T> h4{}, gx{}, gy{}, t4{};
    for (int q = 0; q < 4; ++q) h4.p[q] = (T*)cv.take(sizeof(T) * field_size(d, LOC_M));
    for (int q = 0; q < 4; ++q) t4.p[q] = (T*)cv.take(sizeof(T) * field_size(d, LOC_M));
    for (int q = 0; q < 4; ++q) gx.p[q] = (T*)cv.take(sizeof(T) * field_size(d, LOC_U));
    for (int q = 0; q < 4; ++q) gy.p[q] = (T*)cv.take(sizeof(T) * field_size(d, LOC_V));
    void* det = cv.take(det_scatter_scratch_bytes(d, (int)sizeof(T)));  // deterministic scatter
    const bool hyp = c->s.nu_h > 0.0;
    if (hyp)
      for (int q = 0; q < 4; ++q)
        if (cudaMemsetAsync(h4.p[q], 0, sizeof(T) * field_size(d, LOC_M), st) != cudaSuccess) return SISL_ERR_CUDA;
    ExplicitIn<T> ein{(const T*)sp[0], (const T*)sp[1], (const T*)sp[2], (const T*)sp[4], (const T*)sp[3],
                      (const T*)sp[5], {nullptr, nullptr, nullptr, nullptr}};
    ExplicitBar<T> bi{};
    for (int q = 0; q < 6; ++q) bi.f[q] = (const T*)tend_bar[q];
    for (int q = 0; q < 4; ++q) bi.pd[q] = pd_bar ? (const T*)pd_bar[q] : nullptr;
    StateBar<T> so{(T*)sp_bar[0], (T*)sp_bar[1], (T*)sp_bar[2], (T*)sp_bar[4], (T*)sp_bar[3], (T*)sp_bar[5],
                   {nullptr, nullptr, nullptr, nullptr}};
    if (hyp)
      for (int q = 0; q < 4; ++q) so.hyper[q] = h4.p[q];
    {
      KScope k(c, SISL_K_EXPLICIT, st, 3);
      launch_explicit_vjp<T>(d, cf, ein, bi, so, 1, det, st);
    }
    if (hyp) {
      KScope k(c, SISL_K_EXPLICIT, st, 5);
      launch_hyper_vjp<T>(d, cf, h4, gx, gy, t4, so.u, so.v, so.w, so.th, st);
    }
    return SISL_OK;
  };
  const int rc = (c->grid.dtype == SISL_F64) ? run(double{}) : run(float{});
  if (rc) return rc;
  return check_cuda();
}

}  // extern "C"

struct SislStepGraph {
  int n = 0;
  cudaGraph_t graph = nullptr;
  cudaGraphExec_t exec = nullptr;
  GDevInfo* dinfo = nullptr;  // 2 per member, device
  void* group_mem = nullptr;  // grouped solves: member descriptors and block tables, device
  std::vector<cudaStream_t> streams;
  std::vector<cudaEvent_t> events;
};

namespace {
void destroy_graph(SislStepGraph* g) {
  if (!g) return;
  if (g->exec) cudaGraphExecDestroy(g->exec);
  if (g->graph) cudaGraphDestroy(g->graph);
  if (g->dinfo) cudaFree(g->dinfo);
  if (g->group_mem) cudaFree(g->group_mem);
  for (cudaStream_t s : g->streams) cudaStreamDestroy(s);
  for (cudaEvent_t e : g->events) cudaEventDestroy(e);
  delete g;
}

// Captures one branch per member into a new SislStepGraph: a fork on a
// private stream (the caller's may be the legacy stream, which cannot be
// captured), member m's work on its own stream with its GMRES loop bodies
// captured on a side stream, a join, then instantiation.  record(m, stream,
// dev_info) issues member m's work; dev_info holds two solve summaries.
template <typename F>
int capture_members(int n, SislCore* const* cores, F&& record, SislStepGraph** out) {
  SislStepGraph* g = new (std::nothrow) SislStepGraph();
  if (!g) return SISL_ERR_ARG;
  g_last_error[0] = 0;
  g->n = n;
  cudaStream_t st = nullptr;
  auto fail = [&](int rc) {
    cudaStreamCaptureStatus cs;
    if (st && cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
      cudaGraph_t junk = nullptr;
      cudaStreamEndCapture(st, &junk);
      if (junk) cudaGraphDestroy(junk);
    }
    for (int m = 0; m < n; ++m) cores[m]->cap_side = nullptr;
    cudaGetLastError();
    destroy_graph(g);
    return rc;
  };
  if (cuda_failed(cudaMalloc(&g->dinfo, sizeof(GDevInfo) * 2 * n), "cudaMalloc")) return fail(SISL_ERR_CUDA);
  if (cuda_failed(cudaMemset(g->dinfo, 0, sizeof(GDevInfo) * 2 * n), "cudaMemset")) return fail(SISL_ERR_CUDA);
  // member streams, side streams for the conditional bodies, fork and join events
  for (int q = 0; q < 2 * n + 1; ++q) {
    cudaStream_t s;
    if (cuda_failed(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate")) return fail(SISL_ERR_CUDA);
    g->streams.push_back(s);
  }
  st = g->streams[2 * n];
  for (int q = 0; q < n + 1; ++q) {
    cudaEvent_t e;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return fail(SISL_ERR_CUDA);
    g->events.push_back(e);
  }
  for (int m = 0; m < n; ++m)
    if (cores[m]->timing_class != SISL_K_NONE) return fail(SISL_ERR_ARG);  // no timing events inside a graph
  if (cuda_failed(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed), "cudaStreamBeginCapture"))
    return fail(SISL_ERR_CUDA);
  if (cuda_failed(cudaEventRecord(g->events[n], st), "cudaEventRecord(fork)")) return fail(SISL_ERR_CUDA);
  for (int m = 0; m < n; ++m) {
    SislCore* c = cores[m];
    cudaStream_t ms = g->streams[m];
    if (cuda_failed(cudaStreamWaitEvent(ms, g->events[n], 0), "cudaStreamWaitEvent(fork)")) return fail(SISL_ERR_CUDA);
    c->cap_side = g->streams[n + m];
    const int rc = record(m, ms, g->dinfo + 2 * m);
    c->cap_side = nullptr;
    if (rc < 0) {
      if (!g_last_error[0]) snprintf(g_last_error, sizeof(g_last_error), "member %d: status %d", m, rc);
      return fail(rc);
    }
    if (cuda_failed(cudaEventRecord(g->events[m], ms), "cudaEventRecord(join)")) return fail(SISL_ERR_CUDA);
    if (cuda_failed(cudaStreamWaitEvent(st, g->events[m], 0), "cudaStreamWaitEvent(join)")) return fail(SISL_ERR_CUDA);
  }
  if (cuda_failed(cudaStreamEndCapture(st, &g->graph), "cudaStreamEndCapture")) return fail(SISL_ERR_CUDA);
  if (cuda_failed(cudaGraphInstantiate(&g->exec, g->graph, 0), "cudaGraphInstantiate")) return fail(SISL_ERR_CUDA);
  *out = g;
  return SISL_OK;
}

// One solve of every member as grouped launches, captured on st: the
// restart loop is one conditional WHILE node (body captured on side) that
// runs while any member continues; each member's own loop state (cycles,
// convergence) lives in its GState and `running` flag.  The sequence of
// phases per member is gmres_run's (transpose: the A^T / M^T iteration of
// the custom_linear_solve transpose), so each member's result is the same
// bits as its own graph-mode solve.  slot: the step's solve index for the
// statistics.
template <typename T>
int gmres_group_run(const GroupLaunch<T>& gl, cudaStream_t st, cudaStream_t side, int slot, int transpose) {
  const int R = gl.R;
  grp_setup<T>(gl, transpose, st);
  if (gl.refine) grp_convert<T>(gl, 0, st);
  grp_dots<T>(gl, 0, GV_B, 1 /*BNORM*/, 0, st);
  if (gl.method == SISL_GMRES_INCREMENTAL) {
    if (transpose) {
      grp_precond_t<T>(gl, 1, 1, 0, st);
    } else {
      grp_convert<T>(gl, 3, st);
      grp_precond<T>(gl, 1, 1, 0, st);
    }
    grp_dots<T>(gl, 0, GV_V0 + 1, 2 /*MBNORM*/, 0, st);
  }
  grp_init_tol<T>(gl, st);
  auto residual = [&](cudaStream_t s) {
    if (transpose) {
      if (gl.refine) {
        grp_matvec_t<T>(gl, 2, 0, s);
        grp_convert<T>(gl, 4, s);
      } else {
        grp_matvec_t<T>(gl, 1, 0, s);
      }
      grp_precond_t<T>(gl, 0, 0, 0, s);
    } else {
      if (gl.refine) {
        grp_matvec<T>(gl, 2, 0, s);
        grp_convert<T>(gl, 1, s);
      } else {
        grp_matvec<T>(gl, 1, 0, s);
      }
      grp_precond<T>(gl, 0, 0, 0, s);
    }
    grp_dots<T>(gl, 0, GV_V0, 3 /*RNORM*/, 0, s);
  };
  auto cycle = [&](cudaStream_t s) {
    grp_begin_cycle<T>(gl, s);
    for (int j = 0; j < R; ++j) {
      if (transpose) {
        grp_matvec_t<T>(gl, 0, j, s);
        grp_precond_t<T>(gl, 0, j + 1, 1, s);
      } else {
        grp_matvec<T>(gl, 0, j, s);
        grp_precond<T>(gl, 0, j + 1, 1, s);
      }
      grp_dots<T>(gl, j + 1, GV_V0 + j + 1, 0 /*PROJ*/, 1, s);
      grp_update_arnoldi<T>(gl, j + 1, s);
    }
    grp_small_solve<T>(gl, s);
    grp_update_x<T>(gl, s);
  };
  residual(st);
  cudaStreamCaptureStatus cs;
  cudaGraph_t gr;
  const cudaGraphNode_t* deps = nullptr;
  size_t nd = 0;
  if (cuda_failed(cudaStreamGetCaptureInfo(st, &cs, nullptr, &gr, &deps, &nd), "cudaStreamGetCaptureInfo") ||
      cs != cudaStreamCaptureStatusActive)
    return SISL_ERR_ARG;
  cudaGraphConditionalHandle h;
  if (cuda_failed(cudaGraphConditionalHandleCreate(&h, gr, 0, cudaGraphCondAssignDefault),
                  "cudaGraphConditionalHandleCreate"))
    return SISL_ERR_CUDA;
  grp_gate<T>(gl, h, 0, st);
  if (cuda_failed(cudaStreamGetCaptureInfo(st, &cs, nullptr, &gr, &deps, &nd), "cudaStreamGetCaptureInfo"))
    return SISL_ERR_CUDA;
  cudaGraphNodeParams np{};
  np.type = cudaGraphNodeTypeConditional;
  np.conditional.handle = h;
  np.conditional.type = cudaGraphCondTypeWhile;
  np.conditional.size = 1;
  cudaGraphNode_t node;
  if (cuda_failed(cudaGraphAddNode(&node, gr, deps, nd, &np), "cudaGraphAddNode(conditional)")) return SISL_ERR_CUDA;
  cudaGraph_t body = np.conditional.phGraph_out[0];
  if (cuda_failed(cudaStreamUpdateCaptureDependencies(st, &node, 1, cudaStreamSetCaptureDependencies),
                  "cudaStreamUpdateCaptureDependencies"))
    return SISL_ERR_CUDA;
  if (cuda_failed(cudaStreamBeginCaptureToGraph(side, body, nullptr, nullptr, 0, cudaStreamCaptureModeRelaxed),
                  "cudaStreamBeginCaptureToGraph"))
    return SISL_ERR_CUDA;
  cycle(side);
  residual(side);
  grp_gate<T>(gl, h, 1, side);
  cudaGraph_t body_out = nullptr;
  if (cuda_failed(cudaStreamEndCapture(side, &body_out), "cudaStreamEndCapture(body)")) return SISL_ERR_CUDA;
  grp_info<T>(gl, slot, st);
  if (gl.refine) grp_convert<T>(gl, 2, st);
  g_launches += 1;
  return check_cuda();
}

// Grouped ensemble graph: every member's segments (open: carve its
// workspace on its stream; phase p = 0, 1, 2: its work before, between and
// after the two solves) as parallel branches, each of the two solves as one
// grouped GMRES over all members (gmres_group_run).  transpose: the solves
// are the reverse sweep's transposed ones, the step's second solve first.
template <typename T, typename Open, typename Work, typename Phase>
int capture_grouped(int n, SislCore* const* cores, int transpose, Open&& open, Work&& gwork, Phase&& phase,
                    SislStepGraph** out) {
  SislStepGraph* g = new (std::nothrow) SislStepGraph();
  if (!g) return SISL_ERR_ARG;
  g_last_error[0] = 0;
  g->n = n;
  cudaStream_t st = nullptr;
  auto fail = [&](int rc) {
    cudaStreamCaptureStatus cs;
    if (st && cudaStreamIsCapturing(st, &cs) == cudaSuccess && cs != cudaStreamCaptureStatusNone) {
      cudaGraph_t junk = nullptr;
      cudaStreamEndCapture(st, &junk);
      if (junk) cudaGraphDestroy(junk);
    }
    cudaGetLastError();
    destroy_graph(g);
    return rc;
  };
  auto method_of = [&](const SislCore* c) {
    return (transpose && c->adj_method >= 0) ? c->adj_method : c->prm.solve_method;
  };
  const SislCore* c0 = cores[0];
  const int R = c0->prm.solver_restart;
  const int method = method_of(c0);
  const bool refine = refining<T>(c0);
  for (int m = 0; m < n; ++m) {
    const SislCore* c = cores[m];
    if (c->timing_class != SISL_K_NONE) return fail(SISL_ERR_ARG);  // no timing events inside a graph
    if (c->prm.solver_restart != R || method_of(c) != method || refining<T>(c) != refine || c->d.nz < 2 || R < 1 ||
        R > GM_MAXR) {
      snprintf(g_last_error, sizeof(g_last_error),
               "grouped solve: member %d differs in restart, GMRES method or refinement, or has nz < 2", m);
      return fail(SISL_ERR_ARG);
    }
  }
  // streams: one per member, the capture stream, the loop-body stream
  for (int q = 0; q < n + 2; ++q) {
    cudaStream_t s;
    if (cuda_failed(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking), "cudaStreamCreate")) return fail(SISL_ERR_CUDA);
    g->streams.push_back(s);
  }
  st = g->streams[n];
  cudaStream_t side = g->streams[n + 1];
  for (int q = 0; q < n + 1; ++q) {
    cudaEvent_t e;
    if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return fail(SISL_ERR_CUDA);
    g->events.push_back(e);
  }
  for (int m = 0; m < n; ++m) {
    const int rc = open(m, g->streams[m]);
    if (rc) return fail(rc);
  }
  // member descriptors and block tables
  const int NT = group_tables(R);
  const size_t desc_bytes = align256(sizeof(GroupMember<T>) * n);
  const size_t tab_bytes = sizeof(int) * (size_t)NT * (n + 1);
  const size_t info_bytes = sizeof(GDevInfo) * 2 * n;
  if (cuda_failed(cudaMalloc(&g->group_mem, desc_bytes + tab_bytes), "cudaMalloc") ||
      cuda_failed(cudaMalloc(&g->dinfo, info_bytes), "cudaMalloc"))
    return fail(SISL_ERR_CUDA);
  GroupMember<T>* dmem = (GroupMember<T>*)g->group_mem;
  int* dtab = (int*)((char*)g->group_mem + desc_bytes);
  GDevInfo* dinfo = g->dinfo;
  std::vector<GroupMember<T>> hm(n);
  GroupLaunch<T> gl;
  gl.mem = dmem;
  gl.first = dtab;
  gl.M = n;
  gl.R = R;
  gl.method = method;
  gl.refine = refine;
  gl.first_h.assign((size_t)NT * (n + 1), 0);
  gl.nz_h.resize(n);
  for (int m = 0; m < n; ++m) {
    const SislCore* c = cores[m];
    const GWork<T>& w = gwork(m);
    GroupMember<T>& e = hm[m];
    std::memset(&e, 0, sizeof(e));
    e.d = c->d;
    e.c = coef_of<T>(c);
    if (refine) e.c64 = coef64_of(c);
    e.vec = w.vec;
    e.x64 = w.x64;
    e.b64 = w.b64;
    e.r64 = w.r64;
    e.tmp = w.tmp;
    e.tmp64 = w.tmp64;
    e.npad = w.npad;
    for (int q = 0; q < 5; ++q) e.off[q] = w.off[q];
    e.gs = w.gs;
    e.partial = w.partial;
    e.info[0] = dinfo + 2 * m;
    e.info[1] = dinfo + 2 * m + 1;
    e.eps = (sizeof(T) == 8) ? 2.220446049250313e-16 : 1.1920928955078125e-07;
    e.tol = c->prm.solver_tol;
    e.tol_t = (c->adj_tol > 0.0) ? c->adj_tol : c->prm.solver_tol;
    e.atol_in = c->prm.solver_atol;
    e.maxiter = c->prm.solver_maxiter;
    e.running = 0;
    gl.nz_h[m] = c->d.nz;
    const size_t np = w.npad;
    int cnt[64 + GM_MAXR];
    cnt[GT_MV] = group_matvec_blocks(c->d);
    cnt[GT_PC] = group_precond_blocks(c->d);
    cnt[GT_UPD] = gm_update_blocks<T>(np);
    cnt[GT_X64] = gm_x64_blocks(np);
    cnt[GT_CVT] = group_convert_blocks(np);
    cnt[GT_ATG] = group_at_blocks(c->d, 0);
    cnt[GT_ATM] = group_at_blocks(c->d, 1);
    cnt[GT_PTM] = group_pt_blocks(c->d, 0);
    cnt[GT_PTU] = group_pt_blocks(c->d, 1);
    for (int q = 0; q <= R; ++q) cnt[GT_DOTS0 + q] = gm_dots_blocks<T>(q, np);
    for (int t = 0; t < NT; ++t) {
      int* row = gl.first_h.data() + (size_t)t * (n + 1);
      row[m + 1] = row[m] + cnt[t];
    }
  }
  if (cuda_failed(cudaMemcpy(dmem, hm.data(), sizeof(GroupMember<T>) * n, cudaMemcpyHostToDevice), "cudaMemcpy") ||
      cuda_failed(cudaMemcpy(dtab, gl.first_h.data(), tab_bytes, cudaMemcpyHostToDevice), "cudaMemcpy") ||
      cuda_failed(cudaMemset(dinfo, 0, info_bytes), "cudaMemset"))
    return fail(SISL_ERR_CUDA);
  auto fork = [&]() -> int {
    if (cuda_failed(cudaEventRecord(g->events[n], st), "cudaEventRecord(fork)")) return SISL_ERR_CUDA;
    for (int m = 0; m < n; ++m)
      if (cuda_failed(cudaStreamWaitEvent(g->streams[m], g->events[n], 0), "cudaStreamWaitEvent(fork)"))
        return SISL_ERR_CUDA;
    return SISL_OK;
  };
  auto join = [&]() -> int {
    for (int m = 0; m < n; ++m) {
      if (cuda_failed(cudaEventRecord(g->events[m], g->streams[m]), "cudaEventRecord(join)")) return SISL_ERR_CUDA;
      if (cuda_failed(cudaStreamWaitEvent(st, g->events[m], 0), "cudaStreamWaitEvent(join)")) return SISL_ERR_CUDA;
    }
    return SISL_OK;
  };
  auto members = [&](int p) -> int {
    for (int m = 0; m < n; ++m) {
      const int rc = phase(m, p);
      if (rc < 0) {
        if (!g_last_error[0]) snprintf(g_last_error, sizeof(g_last_error), "member %d: status %d", m, rc);
        return rc;
      }
    }
    return SISL_OK;
  };
  if (cuda_failed(cudaStreamBeginCapture(st, cudaStreamCaptureModeRelaxed), "cudaStreamBeginCapture"))
    return fail(SISL_ERR_CUDA);
  int rc;
  if ((rc = fork()) || (rc = members(0)) || (rc = join()) ||
      (rc = gmres_group_run<T>(gl, st, side, transpose ? 1 : 0, transpose)) || (rc = fork()) || (rc = members(1)) ||
      (rc = join()) || (rc = gmres_group_run<T>(gl, st, side, transpose ? 0 : 1, transpose)) || (rc = fork()) ||
      (rc = members(2)) || (rc = join()))
    return fail(rc);
  if (cuda_failed(cudaStreamEndCapture(st, &g->graph), "cudaStreamEndCapture")) return fail(SISL_ERR_CUDA);
  if (cuda_failed(cudaGraphInstantiate(&g->exec, g->graph, 0), "cudaGraphInstantiate")) return fail(SISL_ERR_CUDA);
  *out = g;
  return SISL_OK;
}

// the forward step of every member with grouped solves
template <typename T>
int capture_grouped_step(int n, SislCore* const* cores, const SislState* ins, const SislState* outs,
                         const SislRelaxation* const* relax, void* const* solves, void* const* ws,
                         const size_t* ws_bytes, SislStepGraph** out) {
  std::vector<StepRun<T>> runs(n);
  const SislSolveInfo none{};
  return capture_grouped<T>(
      n, cores, 0,
      [&](int m, cudaStream_t s) {
        return step_open<T>(runs[m], cores[m], &ins[m], &outs[m], relax ? relax[m] : nullptr, ws[m], ws_bytes[m],
                            s, nullptr, solves ? solves + 10 * m : nullptr, nullptr);
      },
      [&](int m) -> const GWork<T>& { return runs[m].w.g; },
      [&](int m, int p) -> int {
        StepRun<T>& r = runs[m];
        if (p == 0) {
          step_explicit<T>(r);
          step_pre_solve<T>(r, 0);
          return SISL_OK;
        }
        const int it = p - 1;
        int rc = step_post_solve<T>(r, it, SISL_OK, none);
        if (rc) return rc;
        if (p == 1) {
          step_pre_solve<T>(r, 1);
          return SISL_OK;
        }
        rc = step_close<T>(r);
        return rc < 0 ? rc : SISL_OK;
      },
      out);
}

// the reverse sweep of every member with grouped transposed solves
template <typename T>
int capture_grouped_vjp(int n, SislCore* const* cores, const SislState* ins, void* const* solves,
                        const SislRelaxation* const* relax, const SislState* out_bars, const SislState* in_bars,
                        void* const* ws, const size_t* ws_bytes, SislStepGraph** out) {
  std::vector<VjpRun<T>> runs(n);
  const SislSolveInfo none{};
  return capture_grouped<T>(
      n, cores, 1,
      [&](int m, cudaStream_t s) {
        return vjp_open<T>(runs[m], cores[m], &ins[m], solves + 10 * m, relax ? relax[m] : nullptr, &out_bars[m],
                           &in_bars[m], ws[m], ws_bytes[m], s, nullptr);
      },
      [&](int m) -> const GWork<T>& { return runs[m].w.g; },
      [&](int m, int p) -> int {
        VjpRun<T>& r = runs[m];
        int rc;
        if (p == 0) {
          if ((rc = vjp_forward<T>(r))) return rc;
          return vjp_pre_solve<T>(r, 1);
        }
        const int it = (p == 1) ? 1 : 0;
        if ((rc = vjp_post_solve<T>(r, it, SISL_OK, none))) return rc;
        if (p == 1) return vjp_pre_solve<T>(r, 0);
        rc = vjp_close<T>(r);
        return rc < 0 ? rc : SISL_OK;
      },
      out);
}

// Argument checks shared by the graph builders: distinct cores (a core's
// side stream serves one branch), workspaces of the given kind.
int check_members(int n, SislCore* const* cores, void* const* ws, const size_t* ws_bytes, int ws_kind) {
  for (int m = 0; m < n; ++m) {
    SislCore* c = cores[m];
    if (!c || ws_bad(ws[m], ws_bytes[m], sisl_workspace_bytes(c, ws_kind))) return SISL_ERR_WORKSPACE;
    for (int q = 0; q < m; ++q)
      if (cores[q] == c) return SISL_ERR_ARG;
  }
  return SISL_OK;
}

bool step_args_ok(const SislState& a, const SislState& b) {
  const void* need[] = {a.u, a.v, a.w, a.eta_dot, a.pi_p, a.th_p, b.u, b.v, b.w, b.eta_dot, b.pi_p, b.th_p};
  for (const void* p : need)
    if (!p) return false;
  return a.is_first_step == 1.0 || (a.u_prev && a.v_prev && a.eta_dot_prev);
}
}  // namespace

extern "C" {

int sisl_step_graph_create(int n, SislCore* const* cores, const SislState* ins, const SislState* outs,
                           const SislRelaxation* const* relax, void* const* ws, const size_t* ws_bytes, void* stream,
                           SislStepGraph** out) {
  return sisl_step_graph_create_taped(n, cores, ins, outs, relax, nullptr, ws, ws_bytes, stream, out);
}

int sisl_step_graph_create_taped(int n, SislCore* const* cores, const SislState* ins, const SislState* outs,
                                 const SislRelaxation* const* relax, void* const* solves, void* const* ws,
                                 const size_t* ws_bytes, void* stream, SislStepGraph** out) {
  if (!out || n < 1 || !cores || !ins || !outs || !ws || !ws_bytes) return SISL_ERR_ARG;
  int rc = check_members(n, cores, ws, ws_bytes, SISL_WS_STEP);
  if (rc) return rc;
  for (int m = 0; m < n; ++m)
    if (!step_args_ok(ins[m], outs[m])) return SISL_ERR_ARG;
  (void)stream;  // captured on a private stream
  return capture_members(
      n, cores,
      [&](int m, cudaStream_t ms, GDevInfo* di) {
        SislCore* c = cores[m];
        const SislRelaxation* rl = relax ? relax[m] : nullptr;
        void* const* tape = solves ? solves + 10 * m : nullptr;
        return (c->grid.dtype == SISL_F64)
                   ? step_impl<double>(c, &ins[m], &outs[m], rl, ws[m], ws_bytes[m], ms, nullptr, tape, di)
                   : step_impl<float>(c, &ins[m], &outs[m], rl, ws[m], ws_bytes[m], ms, nullptr, tape, di);
      },
      out);
}

int sisl_step_graph_create_grouped(int n, SislCore* const* cores, const SislState* ins, const SislState* outs,
                                   const SislRelaxation* const* relax, void* const* solves, void* const* ws,
                                   const size_t* ws_bytes, void* stream, SislStepGraph** out) {
  if (!out || n < 1 || !cores || !ins || !outs || !ws || !ws_bytes) return SISL_ERR_ARG;
  int rc = check_members(n, cores, ws, ws_bytes, SISL_WS_STEP);
  if (rc) return rc;
  for (int m = 0; m < n; ++m) {
    if (!step_args_ok(ins[m], outs[m])) return SISL_ERR_ARG;
    if (cores[m]->grid.dtype != cores[0]->grid.dtype) return SISL_ERR_ARG;
  }
  (void)stream;  // captured on a private stream
  return (cores[0]->grid.dtype == SISL_F64)
             ? capture_grouped_step<double>(n, cores, ins, outs, relax, solves, ws, ws_bytes, out)
             : capture_grouped_step<float>(n, cores, ins, outs, relax, solves, ws, ws_bytes, out);
}

namespace {
int check_vjp_members(int n, SislCore* const* cores, const SislState* ins, void* const* solves,
                      const SislState* out_bars, const SislState* in_bars, void* const* ws, const size_t* ws_bytes) {
  if (n < 1 || !cores || !ins || !solves || !out_bars || !in_bars || !ws || !ws_bytes) return SISL_ERR_ARG;
  int rc = check_members(n, cores, ws, ws_bytes, SISL_WS_STEP_VJP);
  if (rc) return rc;
  for (int m = 0; m < n; ++m) {
    const SislState& a = ins[m];
    const SislState& ib = in_bars[m];
    const void* need[] = {a.u, a.v, a.w, a.eta_dot, a.pi_p, a.th_p, ib.u, ib.v, ib.w, ib.eta_dot, ib.pi_p, ib.th_p};
    for (const void* p : need)
      if (!p) return SISL_ERR_ARG;
    if (a.is_first_step != 1.0 && (!a.u_prev || !a.v_prev || !a.eta_dot_prev)) return SISL_ERR_ARG;
    for (int q = 0; q < 10; ++q)
      if (!solves[10 * m + q]) return SISL_ERR_ARG;
  }
  return SISL_OK;
}
}  // namespace

int sisl_step_vjp_graph_create(int n, SislCore* const* cores, const SislState* ins, void* const* solves,
                               const SislRelaxation* const* relax, const SislState* out_bars,
                               const SislState* in_bars, void* const* ws, const size_t* ws_bytes, void* stream,
                               SislStepGraph** out) {
  if (!out) return SISL_ERR_ARG;
  int rc = check_vjp_members(n, cores, ins, solves, out_bars, in_bars, ws, ws_bytes);
  if (rc) return rc;
  (void)stream;  // captured on a private stream
  return capture_members(
      n, cores,
      [&](int m, cudaStream_t ms, GDevInfo* di) {
        SislCore* c = cores[m];
        const SislRelaxation* rl = relax ? relax[m] : nullptr;
        return (c->grid.dtype == SISL_F64)
                   ? step_vjp_impl<double>(c, &ins[m], solves + 10 * m, rl, &out_bars[m], &in_bars[m], ws[m],
                                           ws_bytes[m], ms, nullptr, di)
                   : step_vjp_impl<float>(c, &ins[m], solves + 10 * m, rl, &out_bars[m], &in_bars[m], ws[m],
                                          ws_bytes[m], ms, nullptr, di);
      },
      out);
}

int sisl_step_vjp_graph_create_grouped(int n, SislCore* const* cores, const SislState* ins, void* const* solves,
                                       const SislRelaxation* const* relax, const SislState* out_bars,
                                       const SislState* in_bars, void* const* ws, const size_t* ws_bytes,
                                       void* stream, SislStepGraph** out) {
  if (!out) return SISL_ERR_ARG;
  int rc = check_vjp_members(n, cores, ins, solves, out_bars, in_bars, ws, ws_bytes);
  if (rc) return rc;
  for (int m = 0; m < n; ++m)
    if (cores[m]->grid.dtype != cores[0]->grid.dtype) return SISL_ERR_ARG;
  (void)stream;  // captured on a private stream
  return (cores[0]->grid.dtype == SISL_F64)
             ? capture_grouped_vjp<double>(n, cores, ins, solves, relax, out_bars, in_bars, ws, ws_bytes, out)
             : capture_grouped_vjp<float>(n, cores, ins, solves, relax, out_bars, in_bars, ws, ws_bytes, out);
}

int sisl_step_graph_launch(SislStepGraph* g, void* stream) {
  if (!g || !g->exec) return SISL_ERR_ARG;
  g_launches += 1;
  if (cuda_failed(cudaGraphLaunch(g->exec, (cudaStream_t)stream), "cudaGraphLaunch")) return SISL_ERR_CUDA;
  return SISL_OK;
}

int sisl_step_graph_info(SislStepGraph* g, int member, SislStepInfo* info, void* stream) {
  if (!g || !info || member < 0 || member >= g->n) return SISL_ERR_ARG;
  GDevInfo h[2];
  cudaStream_t st = (cudaStream_t)stream;
  if (cudaMemcpyAsync(h, g->dinfo + 2 * member, sizeof(h), cudaMemcpyDeviceToHost, st) != cudaSuccess ||
      cudaStreamSynchronize(st) != cudaSuccess)
    return SISL_ERR_CUDA;
  int status = SISL_OK;
  for (int q = 0; q < 2; ++q) {
    std::memcpy(&info->solve[q], &h[q], sizeof(SislSolveInfo));
    if (!std::isfinite(h[q].residual_norm)) status = SISL_ERR_NONFINITE;
    else if (!h[q].converged && status == SISL_OK) status = SISL_NOT_CONVERGED;
  }
  info->kernel_launches = 0;
  return status;
}

int sisl_step_graph_destroy(SislStepGraph* g) {
  if (!g) return SISL_ERR_ARG;
  destroy_graph(g);
  return SISL_OK;
}

int sisl_core_set_tuning(SislCore* c, const SislTuning* t) {
  if (!c || !t) return SISL_ERR_ARG;
  if (t->matvec_block < 0 || t->matvec_block >= N_MATVEC_SHAPES || t->matvec_t_block < 0 ||
      t->matvec_t_block >= N_STENCIL_BLOCKS || t->precond_tile < 0 || t->precond_tile >= N_PRECOND_SHAPES ||
      t->precond_t_tile < 0 || t->precond_t_tile >= N_PRECOND_T_SHAPES)
    return SISL_ERR_ARG;
  c->d.tune_mv = t->matvec_block;
  c->d.tune_pc = t->precond_tile;
  c->d.tune_mvt = t->matvec_t_block;
  c->d.tune_pct = t->precond_t_tile;
  return SISL_OK;
}

int sisl_autotune_query(const SislCore* c, SislTuning* out) {
  if (!c || !out) return SISL_ERR_ARG;
  std::memset(out, 0, sizeof(*out));
  out->matvec_block = c->d.tune_mv;
  out->precond_tile = c->d.tune_pc;
  out->matvec_t_block = c->d.tune_mvt;
  out->precond_t_tile = c->d.tune_pct;
  return SISL_OK;
}

}  // extern "C"

namespace {
// Time every candidate launch shape of the four tunable Helmholtz kernels on
// this core's grid (CUDA events, warm launches) and keep the fastest.
template <typename T>
int autotune_impl(SislCore* c, void* ws, cudaStream_t st, SislTuning* out) {
  Carver cv{(char*)ws};
  GWork<T> g = carve_gmres<T>(cv, c->d, c->prm.solver_restart, false);
  const Coef<T> cf = coef_of<T>(c);
  for (int q = 0; q < 3; ++q)
    if (cuda_failed(cudaMemsetAsync(g.V(q), 0, sizeof(T) * g.npad, st), "cudaMemsetAsync")) return SISL_ERR_CUDA;
  if (cuda_failed(cudaMemsetAsync(g.z(), 0, sizeof(T) * g.npad, st), "cudaMemsetAsync")) return SISL_ERR_CUDA;
  cudaEvent_t e0, e1;
  if (cuda_failed(cudaEventCreate(&e0), "cudaEventCreate") || cuda_failed(cudaEventCreate(&e1), "cudaEventCreate"))
    return SISL_ERR_CUDA;
  const int reps = 8;
  int rc = SISL_OK;
  auto time_it = [&](auto&& launch) -> float {
    launch();
    launch();
    cudaEventRecord(e0, st);
    for (int r = 0; r < reps; ++r) launch();
    cudaEventRecord(e1, st);
    float ms = 0.f;
    if (cuda_failed(cudaEventSynchronize(e1), "cudaEventSynchronize") ||
        cuda_failed(cudaEventElapsedTime(&ms, e0, e1), "cudaEventElapsedTime") || check_cuda() != SISL_OK) {
      rc = SISL_ERR_CUDA;
      return 1e30f;
    }
    return ms * 1000.f / reps;
  };
  CVec5<T> none{};
  Dims& d = c->d;
  auto pick = [&](int* field, int ncand, auto&& launch, float* us_out) {
    int best = 0;
    float tbest = 1e30f;
    for (int v = 0; v < ncand && rc == SISL_OK; ++v) {
      *field = v;
      const float t = time_it(launch);
      if (t < tbest) { tbest = t; best = v; }
    }
    *field = best;
    *us_out = tbest;
  };
  pick(&d.tune_mv, N_MATVEC_SHAPES,
       [&] { launch_matvec<T>(d, cf, g.cview(g.V(0)), nullptr, none, g.split(g.V(1), g.z()), nullptr, st); },
       &out->us[0]);
  pick(&d.tune_pc, N_PRECOND_SHAPES,
       [&] { launch_precond<T>(d, cf, as_const(g.split(g.V(1), g.z())), g.view(g.V(2)), nullptr, st); },
       &out->us[1]);
  pick(&d.tune_mvt, N_STENCIL_BLOCKS,
       [&] { launch_matvec_t<T>(d, cf, g.cview(g.V(0)), nullptr, none, g.view(g.z()), g.tmp, nullptr, st); },
       &out->us[2]);
  pick(&d.tune_pct, N_PRECOND_T_SHAPES,
       [&] { launch_precond_t<T>(d, cf, g.cview(g.z()), g.view(g.V(2)), nullptr, st); }, &out->us[3]);
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  out->matvec_block = d.tune_mv;
  out->precond_tile = d.tune_pc;
  out->matvec_t_block = d.tune_mvt;
  out->precond_t_tile = d.tune_pct;
  return rc;
}
}  // namespace

extern "C" {

int sisl_autotune(SislCore* c, void* ws, size_t ws_bytes, void* stream, SislTuning* out) {
  if (!c || !out) return SISL_ERR_ARG;
  if (ws_bad(ws, ws_bytes, sisl_workspace_bytes(c, SISL_WS_GMRES))) return SISL_ERR_WORKSPACE;
  if (c->timing_class != SISL_K_NONE) return SISL_ERR_ARG;
  std::memset(out, 0, sizeof(*out));
  cudaStream_t st = (cudaStream_t)stream;
  return c->grid.dtype == SISL_F64 ? autotune_impl<double>(c, ws, st, out) : autotune_impl<float>(c, ws, st, out);
}

int sisl_core_set_refinement(SislCore* c, int on) {
  if (!c) return SISL_ERR_ARG;
  if (on && !c->coef64_mem) return SISL_ERR_ARG;
  c->refine_on = on ? 1 : 0;
  return SISL_OK;
}

int sisl_core_set_adjoint(SislCore* c, double tol, int normalize_rhs, int method) {
  if (!c || !(tol < 1.0) || method > SISL_GMRES_INCREMENTAL) return SISL_ERR_ARG;
  c->adj_tol = tol;
  c->adj_normalize = normalize_rhs ? 1 : 0;
  c->adj_method = method < 0 ? -1 : method;
  return SISL_OK;
}

int sisl_core_set_solver(SislCore* c, double tol, double atol, int maxiter, int restart, int method) {
  if (!c || restart < 1 || restart > GM_MAXR || maxiter < 0) return SISL_ERR_ARG;
  if (method != SISL_GMRES_BATCHED && method != SISL_GMRES_INCREMENTAL) return SISL_ERR_ARG;
  c->prm.solver_tol = tol;
  c->prm.solver_atol = atol;
  c->prm.solver_maxiter = maxiter;
  c->prm.solver_restart = restart;
  c->prm.solve_method = method;
  return SISL_OK;
}

int sisl_split_diagnose(SislCore* c, const void* u, const void* v, const void* w, void* eta_out, void* w_out,
                        void* stream) {
  if (!c || !u || !v || !w || !eta_out || !w_out) return SISL_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  auto run = [&](auto tag) {
    using T = decltype(tag);
    // u, v, w, z_xi_w, z_eta_w, dz_w in; eta_dot, w out
    KScope k(c, SISL_K_OTHER, st, 1, 8.0 * sizeof(T) * c->d.nx * c->d.ny * c->d.nz);
    launch_split_diag<T>(c->d, coef_of<T>(c), (const T*)u, (const T*)v, (const T*)w, (T*)eta_out, (T*)w_out, st);
  };
  if (c->grid.dtype == SISL_F64) run(double{});
  else run(float{});
  return check_cuda();
}

int sisl_split_diagnose_vjp(SislCore* c, const void* w_out_bar, const void* eta_bar, void* u_bar, void* v_bar,
                            void* w_in_bar, void* ws, size_t ws_bytes, void* stream) {
  if (!c || !w_out_bar || !eta_bar || !u_bar || !v_bar || !w_in_bar) return SISL_ERR_ARG;
  if (w_in_bar == eta_bar || u_bar == v_bar) return SISL_ERR_ARG;
  if (ws_bad(ws, ws_bytes, sisl_workspace_bytes(c, SISL_WS_SPLIT_VJP))) return SISL_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  auto run = [&](auto tag) -> int {
    using T = decltype(tag);
    const Dims& d = c->d;
    const size_t wb = sizeof(T) * field_size(d, LOC_W);
    Carver cv{(char*)ws};
    T* eb = (T*)cv.take(wb);  // the kernel consumes (zeroes) its eta_dot cotangent: work on a copy
    void* det = cv.take(det_scatter_scratch_bytes(d, (int)sizeof(T)));
    if (w_in_bar != w_out_bar && cudaMemcpyAsync(w_in_bar, w_out_bar, wb, cudaMemcpyDeviceToDevice, st) != cudaSuccess)
      return SISL_ERR_CUDA;
    if (cudaMemcpyAsync(eb, eta_bar, wb, cudaMemcpyDeviceToDevice, st) != cudaSuccess) return SISL_ERR_CUDA;
    KScope k(c, SISL_K_OTHER, st, 3);
    launch_split_diag_vjp<T>(d, coef_of<T>(c), (T*)w_in_bar, eb, (T*)u_bar, (T*)v_bar, det, st);
    return SISL_OK;
  };
  const int rc = (c->grid.dtype == SISL_F64) ? run(double{}) : run(float{});
  return rc ? rc : check_cuda();
}

int sisl_split_step(SislCore* c, const SislState* in, const SislState* out, int ns, double alpha, double eps_l,
                    const void* tau_damp, const void* const phys_tend[4], void* ws, size_t ws_bytes, void* stream) {
  if (!c || !in || !out || !tau_damp || ns < 1 || !(alpha >= 0.0 && alpha <= 1.0) || !(eps_l >= 0.0))
    return SISL_ERR_ARG;
  const void* need_in[] = {in->u, in->v, in->w, in->eta_dot, in->pi_p, in->th_p};
  const void* need_out[] = {out->u, out->v, out->w, out->eta_dot, out->pi_p, out->th_p};
  for (const void* p : need_in)
    if (!p) return SISL_ERR_ARG;
  for (const void* p : need_out) {
    if (!p) return SISL_ERR_ARG;
    for (const void* q : need_in)
      if (p == q) return SISL_ERR_ARG;  // out must not alias in
  }
  if (ws_bad(ws, ws_bytes, sisl_workspace_bytes(c, SISL_WS_SPLIT))) return SISL_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  if (c->grid.dtype == SISL_F64)
    split_step_impl<double>(c, in, out, ns, alpha, eps_l, (const double*)tau_damp, phys_tend, ws, st);
  else
    split_step_impl<float>(c, in, out, ns, alpha, eps_l, (const float*)tau_damp, phys_tend, ws, st);
  return check_cuda();
}

int sisl_split_step_vjp(SislCore* c, const SislState* in, const SislState* out_bar, const SislState* in_bar, int ns,
                        double alpha, double eps_l, const void* tau_damp, int deterministic, void* ws,
                        size_t ws_bytes, void* stream) {
  if (!c || !in || !out_bar || !in_bar || !tau_damp || ns < 1 || !(alpha >= 0.0 && alpha <= 1.0) || !(eps_l >= 0.0))
    return SISL_ERR_ARG;
  const void* need_in[] = {in->u, in->v, in->w, in->eta_dot, in->pi_p, in->th_p};
  const void* need_bar[] = {in_bar->u, in_bar->v, in_bar->w, in_bar->eta_dot, in_bar->pi_p, in_bar->th_p};
  const void* obar[] = {out_bar->u, out_bar->v, out_bar->w, out_bar->eta_dot, out_bar->pi_p, out_bar->th_p};
  for (const void* p : need_in)
    if (!p) return SISL_ERR_ARG;
  for (const void* p : need_bar) {
    if (!p) return SISL_ERR_ARG;
    for (const void* q : need_in)
      if (p == q) return SISL_ERR_ARG;  // in_bar must not alias in or out_bar
    for (const void* q : obar)
      if (p == q) return SISL_ERR_ARG;
  }
  if (ws_bad(ws, ws_bytes, sisl_workspace_bytes(c, SISL_WS_SPLIT_VJP))) return SISL_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  if (c->grid.dtype == SISL_F64)
    return split_vjp_impl<double>(c, in, out_bar, in_bar, ns, alpha, eps_l, (const double*)tau_damp, deterministic, ws,
                                  ws_bytes, st);
  return split_vjp_impl<float>(c, in, out_bar, in_bar, ns, alpha, eps_l, (const float*)tau_damp, deterministic, ws,
                               ws_bytes, st);
}

int sisl_ffsl_advect(SislCore* c, const void* field, const void* u, const void* v, const void* eta, void* out,
                     void* ws, size_t ws_bytes, void* stream) {
  if (!c || !field || !u || !v || !eta || !out) return SISL_ERR_ARG;
  if (ws_bad(ws, ws_bytes, sisl_workspace_bytes(c, SISL_WS_FFSL))) return SISL_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  Carver cv{(char*)ws};
  auto run = [&](auto tag) {
    using T = decltype(tag);
    T* t0 = (T*)cv.take(sizeof(T) * field_size(c->d, LOC_M));
    T* t1 = (T*)cv.take(sizeof(T) * field_size(c->d, LOC_M));
    double* M = (double*)cv.take(sizeof(double) * ffsl_scratch_doubles(c->d));
    KScope k(c, SISL_K_OTHER, st, 4);
    launch_ffsl<T>(c->d, coef_of<T>(c), (const T*)field, (const T*)u, (const T*)v, (const T*)eta, (T*)out, t0, t1,
                   M, st);
  };
  if (c->grid.dtype == SISL_F64) run(double{});
  else run(float{});
  return check_cuda();
}

int sisl_ffsl_advect_vjp(SislCore* c, const void* field, const void* u, const void* v, const void* eta,
                         const void* out_bar, void* field_bar, void* u_bar, void* v_bar, void* eta_bar, void* ws,
                         size_t ws_bytes, void* stream) {
  if (!c || !field || !u || !v || !eta || !out_bar || !field_bar) return SISL_ERR_ARG;
  if (ws_bad(ws, ws_bytes, sisl_workspace_bytes(c, SISL_WS_FFSL_VJP))) return SISL_ERR_WORKSPACE;
  cudaStream_t st = (cudaStream_t)stream;
  Carver cv{(char*)ws};
  auto run = [&](auto tag) {
    using T = decltype(tag);
    T* tmp[5];
    for (int q = 0; q < 5; ++q) tmp[q] = (T*)cv.take(sizeof(T) * field_size(c->d, LOC_M));
    double* M = (double*)cv.take(sizeof(double) * ffsl_scratch_doubles(c->d));
    double* Mb = (double*)cv.take(sizeof(double) * ffsl_scratch_doubles(c->d));
    KScope k(c, SISL_K_OTHER, st, 6);
    launch_ffsl_vjp<T>(c->d, coef_of<T>(c), (const T*)field, (const T*)u, (const T*)v, (const T*)eta,
                       (const T*)out_bar, (T*)field_bar, (T*)u_bar, (T*)v_bar, (T*)eta_bar, tmp, M, Mb, st);
  };
  if (c->grid.dtype == SISL_F64) run(double{});
  else run(float{});
  return check_cuda();
}

int sisl_eos(SislCore* c, const void* th_p, const void* pi_p, void* rho, void* stream) {
  if (!c || !th_p || !pi_p || !rho) return SISL_ERR_ARG;
  cudaStream_t st = (cudaStream_t)stream;
  KScope k(c, SISL_K_OTHER, st);
  if (c->grid.dtype == SISL_F64)
    launch_eos<double>(c->d, coef_of<double>(c), (const double*)th_p, (const double*)pi_p, (double*)rho, st);
  else
    launch_eos<float>(c->d, coef_of<float>(c), (const float*)th_p, (const float*)pi_p, (float*)rho, st);
  return check_cuda();
}

int64_t sisl_kernel_launches(void) { return g_launches.load(); }

int sisl_timing_select(SislCore* c, int cls) {
  if (!c) return SISL_ERR_ARG;
  c->timing_class = cls;
  c->ev_used = 0;
  c->timed_bytes = 0.0;
  return SISL_OK;
}

int sisl_timing_read(SislCore* c, double* total_ms, int64_t* launches, double* alg_bytes) {
  if (!c) return SISL_ERR_ARG;
  double tot = 0.0;
  for (size_t q = 0; q < c->ev_used; ++q) {
    float ms = 0.f;
    if (cudaEventSynchronize(c->ev1[q]) != cudaSuccess) return SISL_ERR_CUDA;
    if (cudaEventElapsedTime(&ms, c->ev0[q], c->ev1[q]) != cudaSuccess) return SISL_ERR_CUDA;
    tot += ms;
  }
  if (total_ms) *total_ms = tot;
  if (launches) *launches = (int64_t)c->ev_used;
  if (alg_bytes) *alg_bytes = c->timed_bytes;
  return SISL_OK;
}

}  // extern "C"
