// Reverse sweep of one SISL step: the cotangent kernels of the explicit
// tendencies, the predictor-corrector right-hand sides, the theta'
// predictor, the lateral overrides, the finalisation and the
// hyperdiffusion, as XLA differentiates SISLStepper3D.step
// (steppers.py:720-1073) with the reference's stop_gradient on the padded
// copies of every centre-to-face stagger (operators.py:37-63: the edge rows
// m->u, m->v of a non-periodic axis and the levels 0 and nz of m->w carry no
// cotangent).
//
// Stencils whose transposes fan out to a handful of points (explicit and
// corrector kernels) scatter, one thread per output point, mirroring the
// forward kernels' point functions -- with a scratch buffer as fixed-point
// sums (DetSink: the same bits on every run), without one as float atomic
// adds; the two horizontal Laplacians of the hyperdiffusion are transposed
// in gather form (two passes per Laplacian: face gradients, then mass
// points).
#include "sisl_explicit_dev.cuh"
#include "sisl_step_vjp.cuh"

namespace sisl {
namespace {

using namespace dev;

dim3 box_grid(int ex, int ey, int ez, dim3 blk) {
  return dim3((ex + blk.x - 1) / blk.x, (ey + blk.y - 1) / blk.y, (ez + blk.z - 1) / blk.z);
}

// The block's copy of the launch's DetSink and its per-field state.
__shared__ __align__(16) unsigned char s_det_raw[sizeof(DetSink<double>)];
__shared__ unsigned s_det_max[DET_FIELDS];
__shared__ double s_det_scale[DET_FIELDS], s_det_frac[DET_FIELDS];

template <typename T>
__device__ __forceinline__ const DetSink<T>& det_sink() {
  return *reinterpret_cast<const DetSink<T>*>(s_det_raw);
}

// Fixed-point exponent of a field: a target element gathers fewer than 2^12
// contributions per launch, each at most gmax < 2^eg, so the integer sums
// stay below 2^61; the double fraction word carries 32 more bits.
__device__ __forceinline__ int det_field_exponent(unsigned gmax_bits) {
  int eg;
  frexpf(__uint_as_float(gmax_bits), &eg);
  return 61 - 12 - eg;
}

template <typename T>
__device__ __forceinline__ void det_begin(const DetSink<T>& sink) {
  const int t = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  const int nw = (int)(sizeof(DetSink<T>) / sizeof(unsigned));
  for (int q = t; q < nw; q += blockDim.x * blockDim.y * blockDim.z)
    reinterpret_cast<unsigned*>(s_det_raw)[q] = reinterpret_cast<const unsigned*>(&sink)[q];
  if (t < DET_FIELDS) {
    s_det_max[t] = 0u;
    if (sink.mode == 2 && t < sink.n) {
      s_det_scale[t] = ldexp(1.0, det_field_exponent(sink.gmax[t]));
      s_det_frac[t] = 4294967296.0;
    }
  }
  __syncthreads();
}

// after the point function: the block's field maxima into the launch's (mode 1)
template <typename T>
__device__ __forceinline__ void det_end() {
  const DetSink<T>& s = det_sink<T>();
  if (s.mode != 1) return;
  __syncthreads();
  const int t = threadIdx.x + blockDim.x * (threadIdx.y + blockDim.y * threadIdx.z);
  if (t < s.n && s_det_max[t]) atomicMax(s.gmax + t, s_det_max[t]);
}

// Accumulate v into field p at element i (p is the base pointer of a field;
// a pointer the sink does not list falls back to a float atomic add).  Every
// lane of a warp that reaches one call site passes the same field.
template <typename T>
__device__ __forceinline__ void radd(T* p, int i, T v) {
  const DetSink<T>& s = det_sink<T>();
  if (s.mode == 0) {
    atomicAdd(p + i, v);
    return;
  }
  int f = -1;
  for (int m = 0; m < s.n; ++m)
    if (p == s.dst[m]) {
      f = m;
      break;
    }
  if (f < 0) {
    atomicAdd(p + i, v);
    return;
  }
  if (s.mode == 1) {  // warp maximum, one shared atomic per warp and call
    const unsigned bits = __float_as_uint(__double2float_ru(fabs((double)v)));
    const unsigned mask = __activemask();
    const unsigned mx = __reduce_max_sync(mask, bits);
    if ((int)(threadIdx.x & 31) == __ffs(mask) - 1) atomicMax(&s_det_max[f], mx);
    return;
  }
  const double y = (double)v * s_det_scale[f];
  if (sizeof(T) == 4) {
    atomicAdd(s.acc[f] + i, (unsigned long long)__double2ll_rn(y));
  } else {
    double h = floor(y);
    double r = rint((y - h) * s_det_frac[f]);  // y - h is exact; r in [0, 2^32]
    if (r == s_det_frac[f]) { h += 1.0; r = 0.0; }
    atomicAdd(s.acc[f] + i, (unsigned long long)(long long)h);
    atomicAdd(s.acc[f] + s.len[f] + i, (unsigned long long)r);
  }
}

// field[q] += sum * 2^-e for every registered field (one rounding per element)
template <typename T>
__global__ void det_finish_kernel(DetSink<T> s) {
  for (int f = 0; f < s.n; ++f) {
    const unsigned gb = s.gmax[f];
    if (gb == 0u) continue;  // no contribution
    const double inv = ldexp(1.0, -det_field_exponent(gb));
    const unsigned long long* a = s.acc[f];
    T* dst = s.dst[f];
    for (size_t q = blockIdx.x * (size_t)blockDim.x + threadIdx.x; q < s.len[f];
         q += (size_t)gridDim.x * blockDim.x) {
      double v = (double)(long long)a[q];
      if (sizeof(T) == 8) v += (double)a[s.len[f] + q] * (1.0 / 4294967296.0);
      if (v != 0.0) dst[q] = dst[q] + (T)(v * inv);
    }
  }
}

// padded copies of a centre-to-face stagger (no cotangent)
__device__ __forceinline__ bool face_padded(int f, int n, int periodic) { return !periodic && (f == 0 || f == n); }
__device__ __forceinline__ bool level_padded(int k, int nz) { return k == 0 || k == nz; }

// Faces of one axis whose centre-to-face value reads mass point a and carries
// a cotangent: (face, +1) where a is the right point, (face, -1) the left.
__device__ __forceinline__ int adj_faces(int a, int n, int periodic, int* f, int* s) {
  int c = 0;
  if (a >= 1) { f[c] = a; s[c] = 1; ++c; }
  if (a + 1 <= n - 1) { f[c] = a + 1; s[c] = -1; ++c; }
  if (periodic) {
    if (a == 0) { f[c] = 0; s[c] = 1; ++c; f[c] = n; s[c] = 1; ++c; }
    if (a == n - 1) { f[c] = 0; s[c] = -1; ++c; f[c] = n; s[c] = -1; ++c; }
  }
  return c;
}

template <typename T>
__device__ __forceinline__ T opt(const T* f, int p) {
  return f ? ld(f, p) : T(0);
}

// cotangents of Grad<T> (pressure gradients) onto the mass field q
template <typename T>
struct GradAdj {
  const Dims& d;
  const Coef<T>& c;
  T* qb;
  __device__ __forceinline__ void gzw(int i, int j, int kw, T x) const {
    if (level_padded(kw, d.nz)) return;
    const T s = x * ld(c.idzw, iw(d, i, j, kw));
    radd(qb, im(d, i, j, kw), s);
    radd(qb, im(d, i, j, kw - 1), -s);
  }
  __device__ __forceinline__ void gzm(int i, int j, int k, T x) const {
    gzw(i, j, k, T(0.5) * x);
    gzw(i, j, k + 1, T(0.5) * x);
  }
  __device__ __forceinline__ void gx(int i, int j, int k, T x) const {
    if (face_padded(i, d.nx, d.px)) return;
    int l, r;
    face_pair(i, d.nx, d.px, l, r);
    const T s = x * (T)(1.0 / d.dx) * ld(c.mu, h_u(d, i, j));
    radd(qb, im(d, r, j, k), s);
    radd(qb, im(d, l, j, k), -s);
    const T y = -ld(c.zxu, iu(d, i, j, k)) * T(0.5) * x;
    gzm(l, j, k, y);
    gzm(r, j, k, y);
  }
  __device__ __forceinline__ void gy(int i, int j, int k, T x) const {
    if (face_padded(j, d.ny, d.py)) return;
    int l, r;
    face_pair(j, d.ny, d.py, l, r);
    const T s = x * (T)(1.0 / d.dy) * ld(c.mv, h_v(d, i, j));
    radd(qb, im(d, i, r, k), s);
    radd(qb, im(d, i, l, k), -s);
    const T y = -ld(c.zev, iv(d, i, j, k)) * T(0.5) * x;
    gzm(i, l, k, y);
    gzm(i, r, k, y);
  }
};

// cotangents of Winds<T> onto u, v
template <typename T>
struct WindsAdj {
  const Dims& d;
  const Coef<T>& c;
  T* ub;
  T* vb;
  __device__ __forceinline__ void um(int i, int j, int k, T x) const {
    radd(ub, iu(d, i, j, k), T(0.5) * x);
    radd(ub, iu(d, i + 1, j, k), T(0.5) * x);
  }
  __device__ __forceinline__ void vm(int i, int j, int k, T x) const {
    radd(vb, iv(d, i, j, k), T(0.5) * x);
    radd(vb, iv(d, i, j + 1, k), T(0.5) * x);
  }
  __device__ __forceinline__ void metric_m(int i, int j, int k, T x) const {
    vm(i, j, k, x * ld(c.dmdx, h_m(d, i, j)));
    um(i, j, k, -x * ld(c.dmdy, h_m(d, i, j)));
  }
  __device__ __forceinline__ void uw(int i, int j, int kw, T x) const {
    if (level_padded(kw, d.nz)) return;
    um(i, j, kw - 1, T(0.5) * x);
    um(i, j, kw, T(0.5) * x);
  }
  __device__ __forceinline__ void vw(int i, int j, int kw, T x) const {
    if (level_padded(kw, d.nz)) return;
    vm(i, j, kw - 1, T(0.5) * x);
    vm(i, j, kw, T(0.5) * x);
  }
};

// cotangents of the face averages of a mass field
template <typename T>
__device__ __forceinline__ void avg_mu_adj(const Dims& d, T* fb, int i, int j, int k, T x) {
  if (face_padded(i, d.nx, d.px)) return;
  int l, r;
  face_pair(i, d.nx, d.px, l, r);
  radd(fb, im(d, l, j, k), T(0.5) * x);
  radd(fb, im(d, r, j, k), T(0.5) * x);
}
template <typename T>
__device__ __forceinline__ void avg_mv_adj(const Dims& d, T* fb, int i, int j, int k, T x) {
  if (face_padded(j, d.ny, d.py)) return;
  int l, r;
  face_pair(j, d.ny, d.py, l, r);
  radd(fb, im(d, i, l, k), T(0.5) * x);
  radd(fb, im(d, i, r, k), T(0.5) * x);
}
template <typename T>
__device__ __forceinline__ void avg_mw_adj(const Dims& d, T* fb, int i, int j, int kw, T x) {
  if (level_padded(kw, d.nz)) return;
  radd(fb, im(d, i, j, kw - 1), T(0.5) * x);
  radd(fb, im(d, i, j, kw), T(0.5) * x);
}

// Cotangent x of divergence(...) at mass point (i, j, k).  NL: the face
// thetas are face averages of th (the nonlinear Exner tendency); otherwise
// the background th_v at the faces.
template <typename T, bool NL>
__device__ __forceinline__ void divergence_adj(const Dims& d, const Coef<T>& c, const T* __restrict__ u,
                                               const T* __restrict__ v, const T* __restrict__ eta,
                                               const T* __restrict__ th, int i, int j, int k, T x, T* ub, T* vb,
                                               T* eb, T* thb) {
  if (x == T(0)) return;
  const T s = -ld(c.cpidz, im(d, i, j, k)) * x;
  const T m = ld(c.mm, h_m(d, i, j));
  const T hx = m * m * s * (T)(1.0 / d.dx), hy = m * m * s * (T)(1.0 / d.dy);
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const T wgt = q ? hx : -hx;
    const int pu = iu(d, i + q, j, k);
    const T rd = ld(c.rdu, pu);
    if (NL) {
      radd(ub, pu, wgt * rd * avg_mu(d, th, i + q, j, k));
      avg_mu_adj(d, thb, i + q, j, k, wgt * ld(u, pu) * rd);
    } else {
      radd(ub, pu, wgt * rd * ld(c.thu, pu));
    }
  }
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const T wgt = q ? hy : -hy;
    const int pv = iv(d, i, j + q, k);
    const T rd = ld(c.rdv, pv);
    if (NL) {
      radd(vb, pv, wgt * rd * avg_mv(d, th, i, j + q, k));
      avg_mv_adj(d, thb, i, j + q, k, wgt * ld(v, pv) * rd);
    } else {
      radd(vb, pv, wgt * rd * ld(c.thv, pv));
    }
  }
#pragma unroll
  for (int q = 0; q < 2; ++q) {
    const int kw = k + q;
    if (level_padded(kw, d.nz)) continue;  // the flux is zero on the ground and the lid
    const T wgt = q ? s : -s;
    const int pw = iw(d, i, j, kw);
    const T ez = ld(c.dzw, pw) * ld(c.rhow, pw);
    if (NL) {
      radd(eb, pw, wgt * ez * avg_mw(d, th, i, j, kw));
      avg_mw_adj(d, thb, i, j, kw, wgt * ld(eta, pw) * ez);
    } else {
      radd(eb, pw, wgt * ez * ld(c.thw, pw));
    }
  }
}

// ---------------------------------------------------------------------------
// explicit tendencies (explicit_kernel modes 0 and 1)
// ---------------------------------------------------------------------------
template <typename T>
__device__ __forceinline__ void explicit_vjp_point(const Dims& d, const Coef<T>& c, const ExplicitIn<T>& in,
                                                   const ExplicitBar<T>& bi, const StateBar<T>& bo, int mode) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i > nx || j > ny || k > nz) return;
  const T dt = (T)c.s.dt, a = (T)c.s.alpha, cp = (T)c.s.cp, g = (T)c.s.g;
  const T oma = T(1) - a;
  Grad<T> G{d, c, in.pi};
  Winds<T> W{d, c, in.u, in.v};
  GradAdj<T> GA{d, c, bo.pi};
  WindsAdj<T> WA{d, c, bo.u, bo.v};
  const T* __restrict__ th = in.th;

  if (j < ny && k < nz) {  // u faces
    const int p = iu(d, i, j, k);
    const T b = opt(bi.f[0], p);
    T tb, pdb;
    if (mode == 0) {  // u_in = u + dt ((1 - a) tend + a pd), tend including pd
      if (b != T(0)) radd(bo.u, p, b);
      tb = dt * oma * b;
      pdb = dt * b;
    } else {
      tb = b;
      pdb = b + opt(bi.pd[0], p);
    }
    if (!face_padded(i, nx, d.px) && (tb != T(0) || pdb != T(0))) {
      int l, r;
      face_pair(i, nx, d.px, l, r);
      const T thp = T(0.5) * (ld(th, im(d, l, j, k)) + ld(th, im(d, r, j, k)));
      const T vat = T(0.5) * (W.vm(l, j, k) + W.vm(r, j, k));
      const T am = T(0.5) * (W.metric_m(l, j, k) + W.metric_m(r, j, k));
      // tend = -cp (th_u + th'_u) gx + f_u v_u + metric_u v_u (+ pd)
      const T tthp = -cp * G.gx(i, j, k) * tb;
      radd(bo.th, im(d, l, j, k), T(0.5) * tthp);
      radd(bo.th, im(d, r, j, k), T(0.5) * tthp);
      GA.gx(i, j, k, -cp * (ld(c.thu, p) + thp) * tb);
      const T tv = (ld(c.fu, h_u(d, i, j)) + am) * tb;
      WA.vm(l, j, k, T(0.5) * tv);
      WA.vm(r, j, k, T(0.5) * tv);
      const T tm = vat * tb;
      WA.metric_m(l, j, k, T(0.5) * tm);
      WA.metric_m(r, j, k, T(0.5) * tm);
      if (bo.hyper[0]) {
        radd(bo.hyper[0], im(d, l, j, k), T(0.5) * pdb);
        radd(bo.hyper[0], im(d, r, j, k), T(0.5) * pdb);
      }
    }
  }
  if (i < nx && k < nz) {  // v faces
    const int p = iv(d, i, j, k);
    const T b = opt(bi.f[1], p);
    T tb, pdb;
    if (mode == 0) {
      if (b != T(0)) radd(bo.v, p, b);
      tb = dt * oma * b;
      pdb = dt * b;
    } else {
      tb = b;
      pdb = b + opt(bi.pd[1], p);
    }
    if (!face_padded(j, ny, d.py) && (tb != T(0) || pdb != T(0))) {
      int l, r;
      face_pair(j, ny, d.py, l, r);
      const T thp = T(0.5) * (ld(th, im(d, i, l, k)) + ld(th, im(d, i, r, k)));
      const T uat = T(0.5) * (W.um(i, l, k) + W.um(i, r, k));
      const T am = T(0.5) * (W.metric_m(i, l, k) + W.metric_m(i, r, k));
      // tend = -cp (th_v + th'_v) gy - f_v u_v - metric_v u_v (+ pd)
      const T tthp = -cp * G.gy(i, j, k) * tb;
      radd(bo.th, im(d, i, l, k), T(0.5) * tthp);
      radd(bo.th, im(d, i, r, k), T(0.5) * tthp);
      GA.gy(i, j, k, -cp * (ld(c.thv, p) + thp) * tb);
      const T tu = (-ld(c.fv, h_v(d, i, j)) - am) * tb;
      WA.um(i, l, k, T(0.5) * tu);
      WA.um(i, r, k, T(0.5) * tu);
      const T tm = -uat * tb;
      WA.metric_m(i, l, k, T(0.5) * tm);
      WA.metric_m(i, r, k, T(0.5) * tm);
      if (bo.hyper[1]) {
        radd(bo.hyper[1], im(d, i, l, k), T(0.5) * pdb);
        radd(bo.hyper[1], im(d, i, r, k), T(0.5) * pdb);
      }
    }
  }
  if (i < nx && j < ny) {  // w levels
    const int p = iw(d, i, j, k);
    const T b = opt(bi.f[2], p);
    T tb, pdb;
    if (mode == 0) {
      if (b != T(0)) radd(bo.w, p, b);
      tb = dt * oma * b;
      pdb = dt * b;
    } else {
      tb = b;
      pdb = b + opt(bi.pd[2], p);
    }
    if (!level_padded(k, nz) && (tb != T(0) || pdb != T(0))) {
      const T thp = T(0.5) * (ld(th, im(d, i, j, k - 1)) + ld(th, im(d, i, j, k)));
      const T thw = ld(c.thw, p);
      // tend = -cp (th_w + th'_w) dpi/dz + g th'_w / th_w (+ pd)
      const T tthp = (-cp * G.gzw(i, j, k) + g / thw) * tb;
      radd(bo.th, im(d, i, j, k - 1), T(0.5) * tthp);
      radd(bo.th, im(d, i, j, k), T(0.5) * tthp);
      GA.gzw(i, j, k, -cp * (thw + thp) * tb);
      if (bo.hyper[2]) {
        radd(bo.hyper[2], im(d, i, j, k - 1), T(0.5) * pdb);
        radd(bo.hyper[2], im(d, i, j, k), T(0.5) * pdb);
      }
    }
    if (mode == 0) {  // residual_n = dz_w eta + u_w z_xi_w + v_w z_eta_w - w
      const T rb = opt(bi.f[6], p);
      if (rb != T(0)) {
        radd(bo.eta, p, ld(c.dzw, p) * rb);
        radd(bo.w, p, -rb);
        WA.uw(i, j, k, ld(c.zxw, p) * rb);
        WA.vw(i, j, k, ld(c.zew, p) * rb);
      }
    }
  }
  if (i < nx && j < ny && k < nz) {  // mass points
    const int p = im(d, i, j, k);
    T tpib, nlb, tthb, pd3b;
    if (mode == 0) {  // pi_in = pi' + (1 - a) dt (tend_pi + nl_pi), th_in = th' + (1 - a) dt tend_th
      const T pb = opt(bi.f[3], p), hb = opt(bi.f[4], p);
      if (pb != T(0)) radd(bo.pi, p, pb);
      if (hb != T(0)) radd(bo.th, p, hb);
      tpib = nlb = oma * dt * pb;
      tthb = oma * dt * hb + opt(bi.f[5], p);
      pd3b = tthb;
    } else {
      tpib = opt(bi.f[3], p);
      tthb = opt(bi.f[4], p);
      nlb = opt(bi.f[5], p);
      pd3b = tthb + opt(bi.pd[3], p);
    }
    divergence_adj<T, false>(d, c, in.u, in.v, in.eta, th, i, j, k, tpib, bo.u, bo.v, bo.eta, bo.th);
    divergence_adj<T, true>(d, c, in.u, in.v, in.eta, th, i, j, k, nlb, bo.u, bo.v, bo.eta, bo.th);
    // tend_th = -avg_w->m(w) dth_bg/dz (+ pd)
    const T tw = -ld(c.dthm, p) * tthb;
    if (tw != T(0)) {
      radd(bo.w, iw(d, i, j, k), T(0.5) * tw);
      radd(bo.w, iw(d, i, j, k + 1), T(0.5) * tw);
    }
    if (bo.hyper[3] && pd3b != T(0)) radd(bo.hyper[3], p, pd3b);
  }
}

// ---------------------------------------------------------------------------
// predictor-corrector right-hand side (corrector_rhs_kernel)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) explicit_vjp_kernel(Dims d, Coef<T> c, ExplicitIn<T> in, ExplicitBar<T> bi,
                                                           StateBar<T> bo, int mode, DetSink<T> sink) {
  det_begin(sink);
  explicit_vjp_point(d, c, in, bi, bo, mode);
  det_end<T>();
}

template <typename T>
__device__ __forceinline__ void corrector_vjp_point(const Dims& d, const Coef<T>& c, const CorrectorIn<T>& in,
                                                    const CorrectorBar<T>& cb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i > nx || j > ny || k > nz) return;
  const T adt = (T)(c.s.alpha * c.s.dt);
  const T cad = (T)(c.s.cp * c.s.alpha * c.s.dt);
  const T g = (T)c.s.g;
  Grad<T> G{d, c, in.pg};
  Winds<T> WG{d, c, in.ug, in.vg};
  GradAdj<T> GA{d, c, cb.pg};
  WindsAdj<T> WA{d, c, cb.ug, cb.vg};
  const T* __restrict__ th = in.th_next;
  if (j < ny && k < nz) {  // rhs_u - cad th'_u gx + adt metric_u v_u
    const int p = iu(d, i, j, k);
    const T b = ld(cb.b[0], p);
    if (b != T(0)) {
      radd(cb.rhs_u, p, b);
      if (!face_padded(i, nx, d.px)) {
        int l, r;
        face_pair(i, nx, d.px, l, r);
        const T thp = T(0.5) * (ld(th, im(d, l, j, k)) + ld(th, im(d, r, j, k)));
        const T vat = T(0.5) * (WG.vm(l, j, k) + WG.vm(r, j, k));
        const T am = T(0.5) * (WG.metric_m(l, j, k) + WG.metric_m(r, j, k));
        const T tthp = -cad * G.gx(i, j, k) * b;
        radd(cb.th, im(d, l, j, k), T(0.5) * tthp);
        radd(cb.th, im(d, r, j, k), T(0.5) * tthp);
        GA.gx(i, j, k, -cad * thp * b);
        const T tm = adt * vat * b, tv = adt * am * b;
        WA.metric_m(l, j, k, T(0.5) * tm);
        WA.metric_m(r, j, k, T(0.5) * tm);
        WA.vm(l, j, k, T(0.5) * tv);
        WA.vm(r, j, k, T(0.5) * tv);
      }
    }
  }
  if (i < nx && k < nz) {  // rhs_v - cad th'_v gy - adt metric_v u_v
    const int p = iv(d, i, j, k);
    const T b = ld(cb.b[1], p);
    if (b != T(0)) {
      radd(cb.rhs_v, p, b);
      if (!face_padded(j, ny, d.py)) {
        int l, r;
        face_pair(j, ny, d.py, l, r);
        const T thp = T(0.5) * (ld(th, im(d, i, l, k)) + ld(th, im(d, i, r, k)));
        const T uat = T(0.5) * (WG.um(i, l, k) + WG.um(i, r, k));
        const T am = T(0.5) * (WG.metric_m(i, l, k) + WG.metric_m(i, r, k));
        const T tthp = -cad * G.gy(i, j, k) * b;
        radd(cb.th, im(d, i, l, k), T(0.5) * tthp);
        radd(cb.th, im(d, i, r, k), T(0.5) * tthp);
        GA.gy(i, j, k, -cad * thp * b);
        const T tm = -adt * uat * b, tu = -adt * am * b;
        WA.metric_m(i, l, k, T(0.5) * tm);
        WA.metric_m(i, r, k, T(0.5) * tm);
        WA.um(i, l, k, T(0.5) * tu);
        WA.um(i, r, k, T(0.5) * tu);
      }
    }
  }
  if (i < nx && j < ny) {
    const int p = iw(d, i, j, k);
    const T be = ld(cb.b[4], p);
    if (be != T(0)) radd(cb.reta, p, be);
    // level 0 holds the kinematic bottom value, built from padded
    // (stop_gradient) averages of the guess winds: no cotangent; the lid is zero
    if (!level_padded(k, nz)) {
      const T b = ld(cb.b[2], p);
      if (b != T(0)) {
        radd(cb.rhs_w, p, b);
        const T thp = T(0.5) * (ld(th, im(d, i, j, k - 1)) + ld(th, im(d, i, j, k)));
        const T tthp = (adt * g / ld(c.thw, p) - cad * G.gzw(i, j, k)) * b;
        radd(cb.th, im(d, i, j, k - 1), T(0.5) * tthp);
        radd(cb.th, im(d, i, j, k), T(0.5) * tthp);
        GA.gzw(i, j, k, -cad * thp * b);
      }
    }
  }
  if (i < nx && j < ny && k < nz) {  // rhs_pi + adt nl_pi(guess, th')
    const int p = im(d, i, j, k);
    const T b = ld(cb.b[3], p);
    if (b != T(0)) {
      radd(cb.rhs_pi, p, b);
      divergence_adj<T, true>(d, c, in.gu, in.gv, in.geta, th, i, j, k, adt * b, cb.gu, cb.gv, cb.geta, cb.th);
    }
  }
}

template <typename T>
__global__ void __launch_bounds__(256) corrector_vjp_kernel(Dims d, Coef<T> c, CorrectorIn<T> in,
                                                            CorrectorBar<T> cb, DetSink<T> sink) {
  det_begin(sink);
  corrector_vjp_point(d, c, in, cb);
  det_end<T>();
}

// th_next = th_adv + adt (tend_th + (w_m(w_now) - w_m(w_next)) dth_bg/dz)
template <typename T>
__global__ void corrector_theta_vjp_kernel(Dims d, Coef<T> c, const T* __restrict__ tb, T* thab, T* tthb, T* wnb,
                                           T* wxb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= d.nx || j >= d.ny || k > d.nz) return;
  const T adt = (T)(c.s.alpha * c.s.dt);
  if (k < d.nz) {
    const int p = im(d, i, j, k);
    const T x = ld(tb, p);
    thab[p] += x;
    tthb[p] += adt * x;
  }
  if (wnb) {
    auto q = [&](int kk) { return adt * ld(c.dthm, im(d, i, j, kk)) * ld(tb, im(d, i, j, kk)); };
    T acc = T(0);
    if (k >= 1) acc += T(0.5) * q(k - 1);
    if (k <= d.nz - 1) acc += T(0.5) * q(k);
    const int p = iw(d, i, j, k);
    wnb[p] += acc;
    wxb[p] -= acc;
  }
}

// lateral overrides after the advection (sl_fixup_kernel): open faces take
// the old winds, a periodic axis copies face 0 onto face n, eta's ground
// and lid rows are zero
template <typename T>
__global__ void fixup_vjp_kernel(Dims d, T* rub, T* rvb, T* ub, T* vb, T* reb) {
  const int a = blockIdx.x * blockDim.x + threadIdx.x;
  const int b = blockIdx.y;
  const int k = blockIdx.z;
  if (b == 0 && a < d.ny && k < d.nz) {
    const int p0 = iu(d, 0, a, k), pn = iu(d, d.nx, a, k);
    if (d.px) {
      rub[p0] += rub[pn];
    } else {
      ub[p0] += rub[p0];
      ub[pn] += rub[pn];
      rub[p0] = T(0);
    }
    rub[pn] = T(0);
  }
  if (b == 1 && a < d.nx && k < d.nz) {
    const int p0 = iv(d, a, 0, k), pn = iv(d, a, d.ny, k);
    if (d.py) {
      rvb[p0] += rvb[pn];
    } else {
      vb[p0] += rvb[p0];
      vb[pn] += rvb[pn];
      rvb[p0] = T(0);
    }
    rvb[pn] = T(0);
  }
  if (b == 2 && a < d.nx && k < d.ny) {  // k indexes rows j here
    reb[iw(d, a, k, 0)] = T(0);
    reb[iw(d, a, k, d.nz)] = T(0);
  }
}

// ---------------------------------------------------------------------------
// finalisation (finalize_kernel, hdiv_kernel)
// ---------------------------------------------------------------------------
template <typename T>
__global__ void __launch_bounds__(256) finalize_vjp_kernel(Dims d, Coef<T> c, FinalizeBar<T> fb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i > nx || j > ny || k > nz) return;
  const Relax<T>& R = fb.relax;
  if (j < ny && k < nz) {
    const int p = iu(d, i, j, k);
    T b = opt(fb.u, p);
    if (R.on & RELAX_U) b *= T(1) - ld(R.mask_u, h_u(d, i, j));
    fb.x2u[p] = b;
  }
  if (i < nx && k < nz) {
    const int p = iv(d, i, j, k);
    T b = opt(fb.v, p);
    if (R.on & RELAX_V) b *= T(1) - ld(R.mask_v, h_v(d, i, j));
    fb.x2v[p] = b;
  }
  if (i < nx && j < ny) {
    const int p = iw(d, i, j, k);
    T b = opt(fb.w, p);
    if (R.on & RELAX_W) b *= T(1) - ld(R.mask_m, h_m(d, i, j));
    fb.x2w[p] = b;
    fb.x2eta[p] = opt(fb.eta, p);
  }
  if (i < nx && j < ny && k < nz) {
    const int p = im(d, i, j, k);
    const int h = h_m(d, i, j);
    T th = ld(fb.th2, p), pi = ld(fb.pi2, p);
    const T mth = (R.on & RELAX_TH) ? ld(R.mask_m, h) : T(0);
    const T mpi = (R.on & RELAX_PI) ? ld(R.mask_m, h) : T(0);
    if (R.on & RELAX_TH) th = (T(1) - mth) * th + mth * (R.ext_field[3] ? ld(R.ext_field[3], p) : R.ext[3]);
    if (R.on & RELAX_PI) pi = (T(1) - mpi) * pi + mpi * (R.ext_field[4] ? ld(R.ext_field[4], p) : R.ext[4]);
    T thb = opt(fb.th, p), pib = opt(fb.pi, p);
    const T rb = opt(fb.rho, p);
    if (rb != T(0)) {  // rho = p0 / (Rd th) pi^(cvd/Rd)
      const T thf = th + ld(c.thb, p), pif = pi + ld(c.pib, p);
      const T kap = (T)(c.s.cvd / c.s.Rd);
      const T rho = (T)c.s.p0 / ((T)c.s.Rd * thf) * pow(pif, kap);
      thb += rb * (-rho / thf);
      pib += rb * (kap * rho / pif);
    }
    fb.th2b[p] = (T(1) - mth) * thb;
    fb.x2pi[p] = (T(1) - mpi) * pib;
  }
}

// div_bar = nu_div dt D_face^T(damped-wind cotangents), the faces' diff of
// the divergence padded (stop_gradient) on non-periodic edges
template <typename T>
__global__ void div_t_kernel(Dims d, Coef<T> c, const T* __restrict__ ub, const T* __restrict__ vb, T* divb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= d.nx || j >= d.ny || k >= d.nz) return;
  const T nud = (T)(c.s.nu_div * c.s.dt);
  int f[4], s[4];
  T acc = T(0);
  int n = adj_faces(i, d.nx, d.px, f, s);
  for (int q = 0; q < n; ++q)
    acc += (T)s[q] * ld(c.mu, h_u(d, f[q], j)) * (T)(1.0 / d.dx) * ld(ub, iu(d, f[q], j, k));
  n = adj_faces(j, d.ny, d.py, f, s);
  for (int q = 0; q < n; ++q)
    acc += (T)s[q] * ld(c.mv, h_v(d, i, f[q])) * (T)(1.0 / d.dy) * ld(vb, iv(d, i, f[q], k));
  divb[im(d, i, j, k)] = nud * acc;
}

// winds += D_centre^T(div_bar), div = m (du/dx + dv/dy)
template <typename T>
__global__ void div_winds_t_kernel(Dims d, Coef<T> c, const T* __restrict__ divb, T* ub, T* vb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i > d.nx || j > d.ny || k >= d.nz) return;
  if (j < d.ny) {
    T acc = T(0);
    if (i >= 1) acc += ld(c.mm, h_m(d, i - 1, j)) * ld(divb, im(d, i - 1, j, k));
    if (i <= d.nx - 1) acc -= ld(c.mm, h_m(d, i, j)) * ld(divb, im(d, i, j, k));
    ub[iu(d, i, j, k)] += acc * (T)(1.0 / d.dx);
  }
  if (i < d.nx) {
    T acc = T(0);
    if (j >= 1) acc += ld(c.mm, h_m(d, i, j - 1)) * ld(divb, im(d, i, j - 1, k));
    if (j <= d.ny - 1) acc -= ld(c.mm, h_m(d, i, j)) * ld(divb, im(d, i, j, k));
    vb[iv(d, i, j, k)] += acc * (T)(1.0 / d.dy);
  }
}

// ---------------------------------------------------------------------------
// hyperdiffusion: transpose of HLap (gather form)
// ---------------------------------------------------------------------------
// cotangents of the face gradients Gx (u faces) and Gy (v faces) from the
// cotangent b of the Laplacian at mass points (times scale), four fields
template <typename T>
__global__ void __launch_bounds__(256) lap_t_faces_kernel(Dims d, Coef<T> c, PtrTable<T> bt, PtrTable<T> gxb,
                                                          PtrTable<T> gyb, T scale) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int kz = blockIdx.z * blockDim.z + threadIdx.z;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  const int f = kz / nz, k = kz % nz;
  if (i > nx || j > ny || f >= 4) return;
  const T* __restrict__ b = bt.p[f];
  auto B = [&](int a, int bb, int kk) { return scale * ld(b, im(d, a, bb, kk)); };
  // cotangent of the mass-point face average gxm (resp. gym) at level kk: the
  // vertical derivative ex(kw) = (gxm(kw) - gxm(kw-1)) / dz_w at interior
  // levels, averaged back to mass points with weight -z_xi_m / 2
  auto gmb = [&](const T* zc, int a, int bb, int kk) -> T {
    auto s = [&](int kq) { return -ld(zc, im(d, a, bb, kq)) * B(a, bb, kq); };
    const T sk = s(kk);
    T acc = T(0);
    if (kk >= 1) acc += T(0.5) * (s(kk - 1) + sk) * ld(c.idzw, iw(d, a, bb, kk));
    if (kk + 1 <= nz - 1) acc -= T(0.5) * (sk + s(kk + 1)) * ld(c.idzw, iw(d, a, bb, kk + 1));
    return acc;
  };
  if (j < ny) {  // u face i
    T acc = T(0);
    if (i >= 1) acc += ld(c.mm, h_m(d, i - 1, j)) * (T)(1.0 / d.dx) * B(i - 1, j, k) + T(0.5) * gmb(c.zxm, i - 1, j, k);
    if (i <= nx - 1) acc += -ld(c.mm, h_m(d, i, j)) * (T)(1.0 / d.dx) * B(i, j, k) + T(0.5) * gmb(c.zxm, i, j, k);
    gxb.p[f][iu(d, i, j, k)] = acc;
  }
  if (i < nx) {  // v face j
    T acc = T(0);
    if (j >= 1) acc += ld(c.mm, h_m(d, i, j - 1)) * (T)(1.0 / d.dy) * B(i, j - 1, k) + T(0.5) * gmb(c.zem, i, j - 1, k);
    if (j <= ny - 1) acc += -ld(c.mm, h_m(d, i, j)) * (T)(1.0 / d.dy) * B(i, j, k) + T(0.5) * gmb(c.zem, i, j, k);
    gyb.p[f][iv(d, i, j, k)] = acc;
  }
}

// cotangent of the Laplacian's input at mass points from the face-gradient
// cotangents (Gx, Gy padded on non-periodic edge faces: no cotangent there)
template <typename T>
__global__ void __launch_bounds__(256) lap_t_mass_kernel(Dims d, Coef<T> c, PtrTable<T> gxb, PtrTable<T> gyb,
                                                         PtrTable<T> out) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int kz = blockIdx.z * blockDim.z + threadIdx.z;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  const int f = kz / nz, k = kz % nz;
  if (i >= nx || j >= ny || f >= 4) return;
  const T* __restrict__ GX = gxb.p[f];
  const T* __restrict__ GY = gyb.p[f];
  int fx[4], sx[4], fy[4], sy[4];
  const int nfx = adj_faces(i, nx, d.px, fx, sx);
  const int nfy = adj_faces(j, ny, d.py, fy, sy);
  // cotangent of dzm (the mass-point vertical derivative) at level kk
  auto dzmb = [&](int kk) -> T {
    T acc = T(0);
    for (int q = 0; q < nfx; ++q) {
      const int p = iu(d, fx[q], j, kk);
      acc -= ld(c.zxu, p) * T(0.5) * ld(GX, p);
    }
    for (int q = 0; q < nfy; ++q) {
      const int p = iv(d, i, fy[q], kk);
      acc -= ld(c.zev, p) * T(0.5) * ld(GY, p);
    }
    return acc;
  };
  T acc = T(0);
  for (int q = 0; q < nfx; ++q)
    acc += (T)sx[q] * ld(c.mu, h_u(d, fx[q], j)) * (T)(1.0 / d.dx) * ld(GX, iu(d, fx[q], j, k));
  for (int q = 0; q < nfy; ++q)
    acc += (T)sy[q] * ld(c.mv, h_v(d, i, fy[q])) * (T)(1.0 / d.dy) * ld(GY, iv(d, i, fy[q], k));
  // dzw(kw) = (F(kw) - F(kw-1)) / dz_w at interior levels, dzm = avg of dzw
  const T m0 = dzmb(k);
  if (k >= 1) acc += T(0.5) * (dzmb(k - 1) + m0) * ld(c.idzw, iw(d, i, j, k));
  if (k + 1 <= nz - 1) acc -= T(0.5) * (m0 + dzmb(k + 1)) * ld(c.idzw, iw(d, i, j, k + 1));
  out.p[f][im(d, i, j, k)] = acc;
}

// state cotangents += transpose of the mass-point copies (hyper_src_kernel)
template <typename T>
__global__ void hyper_src_t_kernel(Dims d, PtrTable<T> s, T* ub, T* vb, T* wb, T* thb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i > nx || j > ny || k > nz) return;
  if (j < ny && k < nz) {
    T acc = T(0);
    if (i >= 1) acc += T(0.5) * ld(s.p[0], im(d, i - 1, j, k));
    if (i <= nx - 1) acc += T(0.5) * ld(s.p[0], im(d, i, j, k));
    ub[iu(d, i, j, k)] += acc;
  }
  if (i < nx && k < nz) {
    T acc = T(0);
    if (j >= 1) acc += T(0.5) * ld(s.p[1], im(d, i, j - 1, k));
    if (j <= ny - 1) acc += T(0.5) * ld(s.p[1], im(d, i, j, k));
    vb[iv(d, i, j, k)] += acc;
  }
  if (i < nx && j < ny) {
    T acc = T(0);
    if (k >= 1) acc += T(0.5) * ld(s.p[2], im(d, i, j, k - 1));
    if (k <= nz - 1) acc += T(0.5) * ld(s.p[2], im(d, i, j, k));
    wb[iw(d, i, j, k)] += acc;
  }
  if (i < nx && j < ny && k < nz) thb[im(d, i, j, k)] += ld(s.p[3], im(d, i, j, k));
}

}  // namespace

size_t det_scatter_scratch_bytes(const Dims& d, int elem_bytes) {
  const size_t n = (size_t)(d.nx + 1) * (d.ny + 1) * (d.nz + 1);
  size_t off = 256;
  for (int f = 0; f < DET_FIELDS; ++f) off += ((elem_bytes == 8 ? 2 : 1) * sizeof(unsigned long long) * n + 255) & ~(size_t)255;
  return off;
}

namespace {
// The sink of a launch: the distinct non-null destinations with their
// element counts, accumulators carved from scratch.
template <typename T>
DetSink<T> det_make(void* scratch, T* const* dst, const unsigned* len, int n) {
  DetSink<T> s{};
  s.mode = 0;
  if (!scratch) return s;
  s.gmax = (unsigned*)scratch;
  char* p = (char*)scratch + 256;
  for (int q = 0; q < n; ++q) {
    if (!dst[q]) continue;
    bool seen = false;
    for (int m = 0; m < s.n; ++m) seen = seen || s.dst[m] == dst[q];
    if (seen || s.n == DET_FIELDS) continue;
    s.dst[s.n] = dst[q];
    s.len[s.n] = len[q];
    s.acc[s.n] = (unsigned long long*)p;
    p += ((sizeof(T) == 8 ? 2 : 1) * sizeof(unsigned long long) * (size_t)len[q] + 255) & ~(size_t)255;
    s.n++;
  }
  return s;
}

// max pass, zeroed accumulators, fixed-point pass, finish (or one atomic pass)
template <typename T, typename Launch>
void det_run(DetSink<T> s, Launch&& launch, cudaStream_t st) {
  if (s.mode == 0 && !s.gmax) {
    launch(s);
    return;
  }
  cudaMemsetAsync(s.gmax, 0, sizeof(unsigned) * DET_FIELDS, st);
  s.mode = 1;
  launch(s);
  for (int f = 0; f < s.n; ++f)
    cudaMemsetAsync(s.acc[f], 0, (sizeof(T) == 8 ? 2 : 1) * sizeof(unsigned long long) * (size_t)s.len[f], st);
  s.mode = 2;
  launch(s);
  det_finish_kernel<T><<<148 * 8, 256, 0, st>>>(s);
}
}  // namespace

template <typename T>
void launch_explicit_vjp(const Dims& d, const Coef<T>& c, const ExplicitIn<T>& in, const ExplicitBar<T>& bi,
                         const StateBar<T>& bo, int mode, void* det_scratch, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  const unsigned m = (unsigned)field_size(d, LOC_M), w = (unsigned)field_size(d, LOC_W);
  T* dst[10] = {bo.u, bo.v, bo.w, bo.eta, bo.pi, bo.th, bo.hyper[0], bo.hyper[1], bo.hyper[2], bo.hyper[3]};
  const unsigned len[10] = {(unsigned)field_size(d, LOC_U), (unsigned)field_size(d, LOC_V), w, w, m, m, m, m, m, m};
  det_run<T>(det_make<T>(det_scratch, dst, len, 10), [&](const DetSink<T>& s) {
    explicit_vjp_kernel<T><<<box_grid(d.nx + 1, d.ny + 1, d.nz + 1, blk), blk, 0, st>>>(d, c, in, bi, bo, mode, s);
  }, st);
}

template <typename T>
void launch_corrector_vjp(const Dims& d, const Coef<T>& c, const CorrectorIn<T>& in, const CorrectorBar<T>& cb,
                          void* det_scratch, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  const unsigned m = (unsigned)field_size(d, LOC_M), w = (unsigned)field_size(d, LOC_W);
  const unsigned fu = (unsigned)field_size(d, LOC_U), fv = (unsigned)field_size(d, LOC_V);
  T* dst[12] = {cb.rhs_u, cb.rhs_v, cb.rhs_w, cb.rhs_pi, cb.reta, cb.th, cb.pg, cb.gu, cb.gv, cb.geta, cb.ug, cb.vg};
  const unsigned len[12] = {fu, fv, w, m, w, m, m, fu, fv, w, fu, fv};
  det_run<T>(det_make<T>(det_scratch, dst, len, 12), [&](const DetSink<T>& s) {
    corrector_vjp_kernel<T><<<box_grid(d.nx + 1, d.ny + 1, d.nz + 1, blk), blk, 0, st>>>(d, c, in, cb, s);
  }, st);
}

template <typename T>
void launch_corrector_theta_vjp(const Dims& d, const Coef<T>& c, const T* thn_bar, T* tha_bar, T* tth_bar,
                                T* w_now_bar, T* w_next_bar, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  corrector_theta_vjp_kernel<T><<<box_grid(d.nx, d.ny, d.nz + 1, blk), blk, 0, st>>>(d, c, thn_bar, tha_bar,
                                                                                   tth_bar, w_now_bar, w_next_bar);
}

template <typename T>
void launch_fixup_vjp(const Dims& d, T* ru_bar, T* rv_bar, T* u_bar, T* v_bar, T* reta_bar, cudaStream_t st) {
  const int na = (d.nx > d.ny ? d.nx : d.ny);
  const int nk = (d.nz > d.ny ? d.nz : d.ny);
  fixup_vjp_kernel<T><<<dim3((na + 127) / 128, 3, nk), 128, 0, st>>>(d, ru_bar, rv_bar, u_bar, v_bar, reta_bar);
}

template <typename T>
void launch_finalize_vjp(const Dims& d, const Coef<T>& c, const FinalizeBar<T>& fb, T* div_bar, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  finalize_vjp_kernel<T><<<box_grid(d.nx + 1, d.ny + 1, d.nz + 1, blk), blk, 0, st>>>(d, c, fb);
  if (c.s.nu_div != 0.0) {
    div_t_kernel<T><<<box_grid(d.nx, d.ny, d.nz, blk), blk, 0, st>>>(d, c, fb.x2u, fb.x2v, div_bar);
    div_winds_t_kernel<T><<<box_grid(d.nx + 1, d.ny + 1, d.nz, blk), blk, 0, st>>>(d, c, div_bar, fb.x2u, fb.x2v);
  }
}

template <typename T>
void launch_hyper_vjp(const Dims& d, const Coef<T>& c, PtrTable<T> hyp_bar, PtrTable<T> gx4, PtrTable<T> gy4,
                      PtrTable<T> tmp4, T* u_bar, T* v_bar, T* w_bar, T* th_bar, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  const dim3 gf = box_grid(d.nx + 1, d.ny + 1, 4 * d.nz, blk);
  const dim3 gm = box_grid(d.nx, d.ny, 4 * d.nz, blk);
  // hyp = -nu_h lap(lap(src)): src_bar = lap^T(lap^T(-nu_h hyp_bar))
  lap_t_faces_kernel<T><<<gf, blk, 0, st>>>(d, c, hyp_bar, gx4, gy4, (T)(-c.s.nu_h));
  lap_t_mass_kernel<T><<<gm, blk, 0, st>>>(d, c, gx4, gy4, tmp4);
  lap_t_faces_kernel<T><<<gf, blk, 0, st>>>(d, c, tmp4, gx4, gy4, T(1));
  lap_t_mass_kernel<T><<<gm, blk, 0, st>>>(d, c, gx4, gy4, hyp_bar);
  hyper_src_t_kernel<T><<<box_grid(d.nx + 1, d.ny + 1, d.nz + 1, blk), blk, 0, st>>>(d, hyp_bar, u_bar, v_bar,
                                                                                     w_bar, th_bar);
}

#define SISL_INST_VJP(T)                                                                                       \
  template void launch_explicit_vjp<T>(const Dims&, const Coef<T>&, const ExplicitIn<T>&, const ExplicitBar<T>&, \
                                       const StateBar<T>&, int, void*, cudaStream_t);                          \
  template void launch_corrector_vjp<T>(const Dims&, const Coef<T>&, const CorrectorIn<T>&,                    \
                                        const CorrectorBar<T>&, void*, cudaStream_t);                          \
  template void launch_corrector_theta_vjp<T>(const Dims&, const Coef<T>&, const T*, T*, T*, T*, T*,          \
                                              cudaStream_t);                                                   \
  template void launch_fixup_vjp<T>(const Dims&, T*, T*, T*, T*, T*, cudaStream_t);                            \
  template void launch_finalize_vjp<T>(const Dims&, const Coef<T>&, const FinalizeBar<T>&, T*, cudaStream_t);  \
  template void launch_hyper_vjp<T>(const Dims&, const Coef<T>&, PtrTable<T>, PtrTable<T>, PtrTable<T>,        \
                                    PtrTable<T>, T*, T*, T*, T*, cudaStream_t);
SISL_INST_VJP(float)
SISL_INST_VJP(double)

}  // namespace sisl
