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

// ---------------------------------------------------------------------------
// split-explicit reverse (SplitExplicitStepper3D, steppers.py:1117-1737, as
// XLA differentiates it: the padded copies of every centre-to-face stagger
// carry no cotangent, jnp.sign of the upwind flux has none)
// ---------------------------------------------------------------------------

// A pointwise write of a reverse kernel that also runs as the max pass of a
// deterministic scatter: issued only by the pass that adds the sums.
template <typename T>
__device__ __forceinline__ void wr(T* p, int i, T v) {
  if (det_sink<T>().mode != 1) p[i] = v;
}

// m_w (u_w z_xi_w + v_w z_eta_w) at w level k: cotangent x into the winds
template <typename T>
__device__ __forceinline__ void kinematic_adj(const Dims& d, const Coef<T>& c, const WindsAdj<T>& WA, int i, int j,
                                              int k, T x) {
  if (x == T(0)) return;
  const int p = iw(d, i, j, k);
  const T m = ld(c.mm, h_m(d, i, j)) * x;
  WA.uw(i, j, k, m * ld(c.zxw, p));
  WA.vw(i, j, k, m * ld(c.zew, p));
}

// horizontal divergence of (uc + up, vc + vp) at cell (i, j, k): cotangent x
template <typename T>
__device__ __forceinline__ void cell_div_adj(const Dims& d, const Coef<T>& c, T* ucb, T* upb, T* vcb, T* vpb, int i,
                                             int j, int k, T x) {
  const T mm = ld(c.mm, h_m(d, i, j));
  const int u0 = iu(d, i, j, k), v0 = iv(d, i, j, k);
  const T sx = x * mm / (T)d.dx, sy = x * mm / (T)d.dy;
  radd(ucb, u0 + 1, sx);
  radd(upb, u0 + 1, sx);
  radd(ucb, u0, -sx);
  radd(upb, u0, -sx);
  radd(vcb, v0 + d.nx, sy);
  radd(vpb, v0 + d.nx, sy);
  radd(vcb, v0, -sy);
  radd(vpb, v0, -sy);
}
// the divergence-damping gradient at u face i / v face j (never a padded face here)
template <typename T>
__device__ __forceinline__ void div_grad_x_adj(const Dims& d, const Coef<T>& c, T* ucb, T* upb, T* vcb, T* vpb, int i,
                                               int j, int k, T x) {
  if (x == T(0)) return;
  int l, r;
  face_pair(i, d.nx, d.px, l, r);
  const T s = x / (T)d.dx * ld(c.mu, h_u(d, i, j));
  cell_div_adj(d, c, ucb, upb, vcb, vpb, r, j, k, s);
  cell_div_adj(d, c, ucb, upb, vcb, vpb, l, j, k, -s);
}
template <typename T>
__device__ __forceinline__ void div_grad_y_adj(const Dims& d, const Coef<T>& c, T* ucb, T* upb, T* vcb, T* vpb, int i,
                                               int j, int k, T x) {
  if (x == T(0)) return;
  int l, r;
  face_pair(j, d.ny, d.py, l, r);
  const T s = x / (T)d.dy * ld(c.mv, h_v(d, i, j));
  cell_div_adj(d, c, ucb, upb, vcb, vpb, i, r, k, s);
  cell_div_adj(d, c, ucb, upb, vcb, vpb, i, l, k, -s);
}

// split_diag_kernel^T (steppers.py:1272-1310): one thread per w point
template <typename T>
__global__ void __launch_bounds__(256) split_diag_vjp_kernel(Dims d, Coef<T> c, T* wb, T* eb, T* ub, T* vb,
                                                             DetSink<T> sink) {
  det_begin(sink);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i < d.nx && j < d.ny && k <= d.nz) {
    const int p = iw(d, i, j, k);
    const T w_b = wb[p], e_b = eb[p];
    if (k == 0 || k == d.nz) {  // the kinematic ground value reads padded winds; the lid is zero
      wr(wb, p, T(0));
    } else {
      const T s = e_b / ld(c.dzw, p);
      wr(wb, p, w_b + s);
      const WindsAdj<T> WA{d, c, ub, vb};
      kinematic_adj(d, c, WA, i, j, k, -s);
    }
    wr(eb, p, T(0));
  }
  det_end<T>();
}

// split_correct_kernel^T (steppers.py:1607-1626): one thread per union point
template <typename T>
__global__ void __launch_bounds__(256) split_correct_vjp_kernel(Dims d, Coef<T> c, SplitBar<T> b, DetSink<T> sink) {
  det_begin(sink);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i <= nx && j <= ny && k <= nz) {
    const T cp = (T)c.s.cp, dtau = b.dtau;
    const GradAdj<T> GA{d, c, b.ppp};
    if (j < ny && k < nz) {
      const int p = iu(d, i, j, k);
      const T x = b.upp2[p];
      if (!d.px && (i == 0 || i == nx)) {
        radd(b.u0, p, x);
        radd(b.uc, p, -x);
      } else if (x != T(0)) {
        const int ie = (d.px && i == nx) ? 0 : i, pe = iu(d, ie, j, k);
        radd(b.upp, pe, x);
        radd(b.sfu, pe, dtau * x);
        const T h = -dtau * T(0.5) * cp * ld(c.thu, pe) * x;
        radd(b.gx0, pe, h);
        GA.gx(ie, j, k, h);
        div_grad_x_adj(d, c, b.uc, b.uh, b.vc, b.vh, ie, j, k, b.nu_div * dtau * x);
      }
    }
    if (i < nx && k < nz) {
      const int p = iv(d, i, j, k);
      const T x = b.vpp2[p];
      if (!d.py && (j == 0 || j == ny)) {
        radd(b.v0, p, x);
        radd(b.vc, p, -x);
      } else if (x != T(0)) {
        const int je = (d.py && j == ny) ? 0 : j, pe = iv(d, i, je, k);
        radd(b.vpp, pe, x);
        radd(b.sfv, pe, dtau * x);
        const T h = -dtau * T(0.5) * cp * ld(c.thv, pe) * x;
        radd(b.gy0, pe, h);
        GA.gy(i, je, k, h);
        div_grad_y_adj(d, c, b.uc, b.uh, b.vc, b.vh, i, je, k, b.nu_div * dtau * x);
      }
    }
    if (i < nx && j < ny) {  // w'' = (wc + w'') / (1 + dtau tau) - wc at every w level
      const int p = iw(d, i, j, k);
      const T x = b.wpp[p];
      const T f = T(1) / (T(1) + dtau * ld(b.tau, p));
      wr(b.wpp, p, x * f);
      radd(b.wc, p, x * (f - T(1)));
    }
  }
  det_end<T>();
}

// split_column_kernel^T (steppers.py:1584-1605, 1635-1737): one thread per
// column.  x (the pi'' increment) is the column solve of T x = rhs, so
// rhs_bar = T^-T x_bar, swept with the transposed bands; the w'' and eta_dot
// flux terms are re-formed per level on the way down.
template <typename T>
__global__ void __launch_bounds__(128) split_column_vjp_kernel(Dims d, Coef<T> c, SplitBar<T> b, T a2cp, T adcp,
                                                               DetSink<T> sink) {
  det_begin(sink);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i < nx && j < ny) {
    const T al = b.alpha, dtau = b.dtau, cp = (T)c.s.cp;
    const T mm = ld(c.mm, h_m(d, i, j));
    const T dx = (T)d.dx, dy = (T)d.dy;
    const GradAdj<T> GA{d, c, b.ppp};
    const WindsAdj<T> WA{d, c, b.uh, b.vh};
    auto gam = [&](int kw) -> T {  // acoustic coupling at w level kw (zero at the ground and lid)
      if (kw <= 0 || kw >= nz) return T(0);
      const int pw = iw(d, i, j, kw);
      const T thw = ld(c.thw, pw);
      return a2cp * thw * ld(c.rhow, pw) * thw / ld(c.dzw, pw);
    };
    auto wcoef = [&](int kw) -> T {  // d w''(kw) / d x(kw) = -adcp thw / dz_w (interior levels)
      if (kw <= 0 || kw >= nz) return T(0);
      const int pw = iw(d, i, j, kw);
      return adcp * ld(c.thw, pw) * ld(c.idzw, pw);
    };
    // upward: x_bar(k) and the forward sweep of T^T r = x_bar
    T cprev = T(0), dprev = T(0), g_lo = T(0), g_hi = gam(1);
    for (int k = 0; k < nz; ++k) {
      const int p = im(d, i, j, k);
      T xb = b.ppp[p];
      if (k >= 1) xb -= wcoef(k) * b.wpp[iw(d, i, j, k)];
      if (k + 1 <= nz - 1) xb += wcoef(k + 1) * b.wpp[iw(d, i, j, k + 1)];
      const T cpidz = ld(c.cpidz, p);
      const T mainv = T(1) + cpidz * (g_lo + g_hi);  // 1 - lower - upper
      const T sub = (k >= 1) ? -ld(c.cpidz, p - nx * ny) * g_lo : T(0);  // upper(k - 1)
      const T g_next = gam(k + 2);
      const T sup = (k + 1 < nz) ? -ld(c.cpidz, p + nx * ny) * g_hi : T(0);  // lower(k + 1)
      const T inv = T(1) / (mainv - sub * cprev);
      const T cpk = sup * inv, dpk = (xb - sub * dprev) * inv;
      b.s1[p] = cpk;
      b.s2[p] = dpk;
      cprev = cpk;
      dprev = dpk;
      g_lo = g_hi;
      g_hi = g_next;
    }
    // downward: r(k), then the cotangents of level k and of w level k + 1
    T rh = T(0), dh_hi = T(0);  // r(k + 1) and the div_z weight of level k + 1
    for (int k = nz - 1; k >= 0; --k) {
      const int p = im(d, i, j, k);
      const T r = (k == nz - 1) ? b.s2[p] : b.s2[p] - b.s1[p] * rh;
      radd(b.sfp, p, dtau * r);
      const T cpidz = ld(c.cpidz, p), dzm = ld(c.dzm, p);
      const T dh = -dtau * cpidz * dzm * r;  // cotangent of div_h + div_z
      // div_h = m (dFx/dx m / dz_m + dFy/dy m / dz_m), F = u_h rdu thu, v_h rdv thv
      const T e = dh * mm * mm / dzm;
      const int u0 = iu(d, i, j, k), v0 = iv(d, i, j, k);
      radd(b.uh, u0 + 1, e / dx * ld(c.rdu, u0 + 1) * ld(c.thu, u0 + 1));
      radd(b.uh, u0, -e / dx * ld(c.rdu, u0) * ld(c.thu, u0));
      radd(b.vh, v0 + nx, e / dy * ld(c.rdv, v0 + nx) * ld(c.thv, v0 + nx));
      radd(b.vh, v0, -e / dy * ld(c.rdv, v0) * ld(c.thv, v0));
      const T fz_w = dh / dzm;  // div_z = (fz(k + 1) - fz(k)) / dz_m
      if (k + 1 <= nz - 1) {    // w level k + 1: fz_bar = fz_w(k) - fz_w(k + 1)
        const int kw = k + 1, pw = iw(d, i, j, kw);
        const T thw = ld(c.thw, pw), rw = ld(c.rhow, pw);
        const T q = (fz_w - dh_hi) * rw * thw;  // cotangent of w_av - kinematic
        kinematic_adj(d, c, WA, i, j, kw, -q);
        const T wex_b = al * q + b.wpp[pw];
        const T wold_b = (T(1) - al) * q + wex_b;
        radd(b.sfw, pw, dtau * wex_b);
        GA.gzw(i, j, kw, -dtau * cp * thw * wex_b);
        wr(b.wpp, pw, wold_b);
      }
      rh = r;
      dh_hi = fz_w;
    }
    // the ground value is the kinematic one of padded winds and the lid is
    // zero: w'' there carries no cotangent back
    wr(b.wpp, iw(d, i, j, 0), T(0));
    wr(b.wpp, iw(d, i, j, nz), T(0));
  }
  det_end<T>();
}

// split_column_vjp_kernel on tiles of PC columns (one block per tile and row
// j): A forms x_bar and the transposed bands at every (level, column) pair,
// B one thread per column sweeps T^T r = x_bar in shared memory, C scatters
// the cotangents of every (level, column) pair.  Arithmetic term for term
// that of split_column_vjp_kernel, with the scatters spread over the block.
template <typename T, int PT, int PC>
__global__ void __launch_bounds__(PT) split_column_vjp_tile_kernel(Dims d, Coef<T> c, SplitBar<T> b, T a2cp, T adcp,
                                                                   DetSink<T> sink) {
  det_begin(sink);
  extern __shared__ __align__(16) unsigned char smem_raw[];
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  T* s_x = reinterpret_cast<T*>(smem_raw);  // [nz][PC] x_bar -> r
  T* s_sub = s_x + nz * PC;                  // [nz][PC] upper(k - 1)
  T* s_sup = s_sub + nz * PC;                // [nz][PC] lower(k + 1) -> c'
  T* s_mn = s_sup + nz * PC;                 // [nz][PC] main
  const int i0 = blockIdx.x * PC, j = blockIdx.y, tid = threadIdx.x;
  const T al = b.alpha, dtau = b.dtau, cp = (T)c.s.cp;
  const T dx = (T)d.dx, dy = (T)d.dy;
  auto gam = [&](int i, int kw) -> T {
    if (kw <= 0 || kw >= nz) return T(0);
    const int pw = iw(d, i, j, kw);
    const T thw = ld(c.thw, pw);
    return a2cp * thw * ld(c.rhow, pw) * thw / ld(c.dzw, pw);
  };
  auto wcoef = [&](int i, int kw) -> T {
    if (kw <= 0 || kw >= nz) return T(0);
    const int pw = iw(d, i, j, kw);
    return adcp * ld(c.thw, pw) * ld(c.idzw, pw);
  };
  for (int q = tid; q < nz * PC; q += PT) {  // A
    const int k = q / PC, i = i0 + q % PC;
    if (i >= nx) {
      s_x[q] = T(0);
      s_sub[q] = T(0);
      s_sup[q] = T(0);
      s_mn[q] = T(1);
      continue;
    }
    const int p = im(d, i, j, k);
    T xb = b.ppp[p];
    if (k >= 1) xb -= wcoef(i, k) * b.wpp[iw(d, i, j, k)];
    if (k + 1 <= nz - 1) xb += wcoef(i, k + 1) * b.wpp[iw(d, i, j, k + 1)];
    s_x[q] = xb;
    const T g_lo = gam(i, k), g_hi = gam(i, k + 1);
    s_mn[q] = T(1) + ld(c.cpidz, p) * (g_lo + g_hi);
    s_sub[q] = (k >= 1) ? -ld(c.cpidz, p - nx * ny) * g_lo : T(0);
    s_sup[q] = (k + 1 < nz) ? -ld(c.cpidz, p + nx * ny) * g_hi : T(0);
  }
  __syncthreads();
  if (tid < PC) {  // B
    T cprev = T(0), dprev = T(0);
    for (int k = 0; k < nz; ++k) {
      const int q = k * PC + tid;
      const T sub = s_sub[q];
      const T inv = T(1) / (s_mn[q] - sub * cprev);
      const T cpk = s_sup[q] * inv, dpk = (s_x[q] - sub * dprev) * inv;
      s_sup[q] = cpk;
      s_x[q] = dpk;
      cprev = cpk;
      dprev = dpk;
    }
    T rh = dprev;
    for (int k = nz - 2; k >= 0; --k) {
      const int q = k * PC + tid;
      rh = s_x[q] - s_sup[q] * rh;
      s_x[q] = rh;
    }
  }
  __syncthreads();
  const GradAdj<T> GA{d, c, b.ppp};
  const WindsAdj<T> WA{d, c, b.uh, b.vh};
  for (int q = tid; q < (nz + 1) * PC; q += PT) {  // C: level k (< nz) and w level k + 1
    const int k = q / PC, i = i0 + q % PC;
    if (i >= nx) continue;
    if (k == nz) {  // ground and lid: no cotangent back through w''
      wr(b.wpp, iw(d, i, j, 0), T(0));
      wr(b.wpp, iw(d, i, j, nz), T(0));
      continue;
    }
    const int p = im(d, i, j, k);
    const T r = s_x[q];
    radd(b.sfp, p, dtau * r);
    const T cpidz = ld(c.cpidz, p), dzm = ld(c.dzm, p);
    const T dh = -dtau * cpidz * dzm * r;
    const T mm = ld(c.mm, h_m(d, i, j));
    const T e = dh * mm * mm / dzm;
    const int u0 = iu(d, i, j, k), v0 = iv(d, i, j, k);
    radd(b.uh, u0 + 1, e / dx * ld(c.rdu, u0 + 1) * ld(c.thu, u0 + 1));
    radd(b.uh, u0, -e / dx * ld(c.rdu, u0) * ld(c.thu, u0));
    radd(b.vh, v0 + nx, e / dy * ld(c.rdv, v0 + nx) * ld(c.thv, v0 + nx));
    radd(b.vh, v0, -e / dy * ld(c.rdv, v0) * ld(c.thv, v0));
    if (k + 1 <= nz - 1) {
      const int kw = k + 1, pw = iw(d, i, j, kw);
      const int p1 = p + nx * ny;
      const T fz_lo = dh / dzm;
      const T fz_hi = (-dtau * ld(c.cpidz, p1) * ld(c.dzm, p1) * s_x[q + PC]) / ld(c.dzm, p1);
      const T thw = ld(c.thw, pw), rw = ld(c.rhow, pw);
      const T qq = (fz_lo - fz_hi) * rw * thw;
      kinematic_adj(d, c, WA, i, j, kw, -qq);
      const T wex_b = al * qq + b.wpp[pw];
      const T wold_b = (T(1) - al) * qq + wex_b;
      radd(b.sfw, pw, dtau * wex_b);
      GA.gzw(i, j, kw, -dtau * cp * thw * wex_b);
      wr(b.wpp, pw, wold_b);
    }
  }
  det_end<T>();
}

// split_predict_kernel^T (steppers.py:1561-1579): one thread per union point
template <typename T>
__global__ void __launch_bounds__(256) split_predict_vjp_kernel(Dims d, Coef<T> c, SplitBar<T> b, DetSink<T> sink) {
  det_begin(sink);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i <= nx && j <= ny && k < nz) {
    const T cp = (T)c.s.cp, hdt = T(0.5) * b.dtau;
    const GradAdj<T> GA{d, c, b.ppp};
    if (j < ny) {
      const int p = iu(d, i, j, k);
      const int ie = (d.px && i == nx) ? 0 : i, pe = iu(d, ie, j, k);
      const T x = b.uh[p];
      T g0 = b.gx0[p];
      if (!d.px && (i == 0 || i == nx)) {
        radd(b.u0, p, x);
        radd(b.uc, p, -x);
      } else if (x != T(0)) {
        radd(b.upp, pe, x);
        radd(b.sfu, pe, hdt * x);
        g0 -= hdt * cp * ld(c.thu, pe) * x;
        div_grad_x_adj(d, c, b.uc, b.upp, b.vc, b.vpp, ie, j, k, b.nu_div * hdt * x);
      }
      if (g0 != T(0)) GA.gx(ie, j, k, g0);
    }
    if (i < nx) {
      const int p = iv(d, i, j, k);
      const int je = (d.py && j == ny) ? 0 : j, pe = iv(d, i, je, k);
      const T x = b.vh[p];
      T g0 = b.gy0[p];
      if (!d.py && (j == 0 || j == ny)) {
        radd(b.v0, p, x);
        radd(b.vc, p, -x);
      } else if (x != T(0)) {
        radd(b.vpp, pe, x);
        radd(b.sfv, pe, hdt * x);
        g0 -= hdt * cp * ld(c.thv, pe) * x;
        div_grad_y_adj(d, c, b.uc, b.upp, b.vc, b.vpp, i, je, k, b.nu_div * hdt * x);
      }
      if (g0 != T(0)) GA.gy(i, je, k, g0);
    }
  }
  det_end<T>();
}

// split_end_kernel^T: pointwise
template <typename T>
__global__ void split_end_vjp_kernel(Dims d, PtrTable<T> o, PtrTable<T> cb, T* th0b, T* upp, T* vpp, T* wpp, T* ppp,
                                     T* sfth, T dtns) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i > nx || j > ny || k > nz) return;
  if (j < ny && k < nz) {
    const int p = iu(d, i, j, k);
    const T x = o.p[0][p];
    cb.p[0][p] += x;
    upp[p] = x;
  }
  if (i < nx && k < nz) {
    const int p = iv(d, i, j, k);
    const T x = o.p[1][p];
    cb.p[1][p] += x;
    vpp[p] = x;
  }
  if (i < nx && j < ny) {
    const int p = iw(d, i, j, k);
    const T x = o.p[2][p];
    cb.p[2][p] += x;
    wpp[p] = x;
    cb.p[3][p] += o.p[3][p];  // eta_dot of the stage start
    if (k < nz) {
      const T y = o.p[4][p], z = o.p[5][p];
      cb.p[4][p] += y;
      ppp[p] = y;
      th0b[p] += z;
      sfth[p] = dtns * z;
    }
  }
}

// split_init_kernel^T: u'' = u0 - uc, v'' = v0 - vc, w'' = w0 - wc, pi'' = p0 - pc
template <typename T>
__global__ void split_init_vjp_kernel(Dims d, const T* __restrict__ upp, const T* __restrict__ vpp,
                                      const T* __restrict__ wpp, const T* __restrict__ ppp, PtrTable<T> s,
                                      PtrTable<T> cb) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i > nx || j > ny || k > nz) return;
  if (j < ny && k < nz) {
    const int p = iu(d, i, j, k);
    s.p[0][p] += upp[p];
    cb.p[0][p] -= upp[p];
  }
  if (i < nx && k < nz) {
    const int p = iv(d, i, j, k);
    s.p[1][p] += vpp[p];
    cb.p[1][p] -= vpp[p];
  }
  if (i < nx && j < ny) {
    const int p = iw(d, i, j, k);
    s.p[2][p] += wpp[p];
    cb.p[2][p] -= wpp[p];
    if (k < nz) {
      s.p[4][p] += ppp[p];
      cb.p[4][p] -= ppp[p];
    }
  }
}

// split_slow_kernel^T: sf (u, v, w, pi, th) -> tend (u, v, w, pi, th, nl_pi)
// written; the advection of th', u_m, v_m, w_m accumulated (the padded
// face and level copies of the averages carry no cotangent)
template <typename T>
__global__ void __launch_bounds__(256) split_slow_vjp_kernel(Dims d, PtrTable<T> sf, PtrTable<T> t, PtrTable<T> a,
                                                             DetSink<T> sink) {
  det_begin(sink);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i <= nx && j <= ny && k <= nz) {
    if (j < ny && k < nz) {
      const int p = iu(d, i, j, k);
      const T x = sf.p[0][p];
      wr(t.p[0], p, x);
      avg_mu_adj(d, a.p[1], i, j, k, x);
    }
    if (i < nx && k < nz) {
      const int p = iv(d, i, j, k);
      const T x = sf.p[1][p];
      wr(t.p[1], p, x);
      avg_mv_adj(d, a.p[2], i, j, k, x);
    }
    if (i < nx && j < ny) {
      const int p = iw(d, i, j, k);
      const T x = sf.p[2][p];
      wr(t.p[2], p, x);
      avg_mw_adj(d, a.p[3], i, j, k, x);
      if (k < nz) {
        const T y = sf.p[3][p], z = sf.p[4][p];
        wr(t.p[3], p, y);
        wr(t.p[5], p, y);
        wr(t.p[4], p, z);
        radd(a.p[0], p, z);
      }
    }
  }
  det_end<T>();
}

// cotangent g of F (q4 + sg qb), the 3rd-order upwind-biased face flux
template <typename T>
__device__ __forceinline__ void upwind_flux_adj(T qm2, T qm1, T q0, T qp1, T F, T eps_l, T g, T& bm2, T& bm1, T& b0,
                                                T& bp1, T& bF) {
  const T q4 = T(7.0 / 12.0) * (q0 + qm1) - T(1.0 / 12.0) * (qp1 + qm2);
  const T qb = T(1.0 / 12.0) * ((qp1 - qm2) - T(3) * (q0 - qm1));
  const T cf = (fabs(F) < eps_l) ? T(0) : F;
  const T sg = (cf > T(0)) ? T(1) : ((cf < T(0)) ? T(-1) : T(0));
  bF += g * (q4 + sg * qb);
  const T t4 = g * F, tb = g * F * sg;
  b0 += T(7.0 / 12.0) * t4 - T(3.0 / 12.0) * tb;
  bm1 += T(7.0 / 12.0) * t4 + T(3.0 / 12.0) * tb;
  bp1 += -T(1.0 / 12.0) * t4 + T(1.0 / 12.0) * tb;
  bm2 += -T(1.0 / 12.0) * t4 - T(1.0 / 12.0) * tb;
}

// split_adv_kernel^T (steppers.py:1312-1465): one thread per mass point
template <typename T>
__global__ void __launch_bounds__(256) split_adv_vjp_kernel(Dims d, Coef<T> c, const T* __restrict__ u,
                                                            const T* __restrict__ v, const T* __restrict__ w,
                                                            const T* __restrict__ eta, const T* __restrict__ th,
                                                            T eps_l, PtrTable<T> ab, T* ub, T* vb, T* wb, T* eb,
                                                            T* thb, DetSink<T> sink) {
  det_begin(sink);
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  const int nx = d.nx, ny = d.ny, nz = d.nz;
  if (i < nx && j < ny && k < nz) {
    auto at = [&](int f, int a, int bq, int cz) -> T {  // the advected fields, as AdvFields::at
      switch (f) {
        case 0: return ld(th, im(d, a, bq, cz));
        case 1: return T(0.5) * (ld(u, iu(d, a, bq, cz)) + ld(u, iu(d, a + 1, bq, cz)));
        case 2: return T(0.5) * (ld(v, iv(d, a, bq, cz)) + ld(v, iv(d, a, bq + 1, cz)));
        default: return T(0.5) * (ld(w, iw(d, a, bq, cz)) + ld(w, iw(d, a, bq, cz + 1)));
      }
    };
    auto to = [&](int f, int a, int bq, int cz, T x) {  // cotangent x of at(f, a, bq, cz)
      if (x == T(0)) return;
      switch (f) {
        case 0: radd(thb, im(d, a, bq, cz), x); break;
        case 1:
          radd(ub, iu(d, a, bq, cz), T(0.5) * x);
          radd(ub, iu(d, a + 1, bq, cz), T(0.5) * x);
          break;
        case 2:
          radd(vb, iv(d, a, bq, cz), T(0.5) * x);
          radd(vb, iv(d, a, bq + 1, cz), T(0.5) * x);
          break;
        default:
          radd(wb, iw(d, a, bq, cz), T(0.5) * x);
          radd(wb, iw(d, a, bq, cz + 1), T(0.5) * x);
          break;
      }
    };
    const T mm = ld(c.mm, h_m(d, i, j));
    const T dx = (T)d.dx, dy = (T)d.dy;
    const T mu0 = ld(c.mu, h_u(d, i, j)), mu1 = ld(c.mu, h_u(d, i + 1, j));
    const T mv0 = ld(c.mv, h_v(d, i, j)), mv1 = ld(c.mv, h_v(d, i, j + 1));
    const T dz0 = ld(c.dzw, iw(d, i, j, k)), dz1 = ld(c.dzw, iw(d, i, j, k + 1));
    const T U0 = ld(u, iu(d, i, j, k)) / mu0, U1 = ld(u, iu(d, i + 1, j, k)) / mu1;
    const T V0 = ld(v, iv(d, i, j, k)) / mv0, V1 = ld(v, iv(d, i, j + 1, k)) / mv1;
    const T W0 = ld(eta, iw(d, i, j, k)) * dz0, W1 = ld(eta, iw(d, i, j, k + 1)) * dz1;
    const T dzm = ld(c.dzm, im(d, i, j, k));
    const T zfac = (T)d.dz / dzm;
    const T dU = (U1 - U0) / dx * mm, dV = (V1 - V0) / dy * mm;
    const T dW = (W1 - W0) / (T)d.dz * zfac;
    int xi[5], yj[5], zk[5];
#pragma unroll
    for (int o = 0; o < 5; ++o) {
      xi[o] = wrap_or_clamp(i - 2 + o, nx, d.px);
      yj[o] = wrap_or_clamp(j - 2 + o, ny, d.py);
      zk[o] = min(max(k - 2 + o, 0), nz - 1);
    }
    T U0b = T(0), U1b = T(0), V0b = T(0), V1b = T(0), W0b = T(0), W1b = T(0), dUb = T(0), dVb = T(0), dWb = T(0);
    const int p = im(d, i, j, k);
#pragma unroll 1
    for (int f = 0; f < 4; ++f) {
      const T o = ab.p[f][p];
      if (o == T(0)) continue;
      T qx[5], qy[5], qz[5];
#pragma unroll
      for (int q = 0; q < 5; ++q) {
        qx[q] = at(f, xi[q], j, k);
        qy[q] = at(f, i, yj[q], k);
        qz[q] = at(f, i, j, zk[q]);
      }
      const T q = qx[2];
      // out = -(m^2)(ax - q dU + ay - q dV) - (az - q dW)
      const T axb = -(mm * mm) * o, azb = -o;
      T bx[5] = {T(0), T(0), T(0), T(0), T(0)}, by[5] = {T(0), T(0), T(0), T(0), T(0)},
        bz[5] = {T(0), T(0), T(0), T(0), T(0)};
      bx[2] += (mm * mm) * (dU + dV) * o + dW * o;
      dUb += (mm * mm) * q * o;
      dVb += (mm * mm) * q * o;
      dWb += q * o;
      const T gx = axb / dx * mm, gy = axb / dy * mm, gz = azb / (T)d.dz * zfac;
      upwind_flux_adj(qx[1], qx[2], qx[3], qx[4], U1, eps_l, gx, bx[1], bx[2], bx[3], bx[4], U1b);
      upwind_flux_adj(qx[0], qx[1], qx[2], qx[3], U0, eps_l, -gx, bx[0], bx[1], bx[2], bx[3], U0b);
      upwind_flux_adj(qy[1], qy[2], qy[3], qy[4], V1, eps_l, gy, by[1], by[2], by[3], by[4], V1b);
      upwind_flux_adj(qy[0], qy[1], qy[2], qy[3], V0, eps_l, -gy, by[0], by[1], by[2], by[3], V0b);
      upwind_flux_adj(qz[1], qz[2], qz[3], qz[4], W1, eps_l, gz, bz[1], bz[2], bz[3], bz[4], W1b);
      upwind_flux_adj(qz[0], qz[1], qz[2], qz[3], W0, eps_l, -gz, bz[0], bz[1], bz[2], bz[3], W0b);
#pragma unroll
      for (int q2 = 0; q2 < 5; ++q2) {
        to(f, xi[q2], j, k, bx[q2]);
        to(f, i, yj[q2], k, by[q2]);
        to(f, i, j, zk[q2], bz[q2]);
      }
    }
    U1b += dUb / dx * mm;
    U0b -= dUb / dx * mm;
    V1b += dVb / dy * mm;
    V0b -= dVb / dy * mm;
    W1b += dWb / (T)d.dz * zfac;
    W0b -= dWb / (T)d.dz * zfac;
    if (U0b != T(0)) radd(ub, iu(d, i, j, k), U0b / mu0);
    if (U1b != T(0)) radd(ub, iu(d, i + 1, j, k), U1b / mu1);
    if (V0b != T(0)) radd(vb, iv(d, i, j, k), V0b / mv0);
    if (V1b != T(0)) radd(vb, iv(d, i, j + 1, k), V1b / mv1);
    if (W0b != T(0)) radd(eb, iw(d, i, j, k), W0b * dz0);
    if (W1b != T(0)) radd(eb, iw(d, i, j, k + 1), W1b * dz1);
  }
  det_end<T>();
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

// ---------------------------------------------------------------------------
// split-explicit reverse launchers
// ---------------------------------------------------------------------------
template <typename T>
void launch_split_diag_vjp(const Dims& d, const Coef<T>& c, T* wb, T* eb, T* ub, T* vb, void* det_scratch,
                           cudaStream_t st) {
  dim3 blk(32, 4, 2);
  T* dst[2] = {ub, vb};
  const unsigned len[2] = {(unsigned)field_size(d, LOC_U), (unsigned)field_size(d, LOC_V)};
  det_run<T>(det_make<T>(det_scratch, dst, len, 2), [&](const DetSink<T>& s) {
    split_diag_vjp_kernel<T><<<box_grid(d.nx, d.ny, d.nz + 1, blk), blk, 0, st>>>(d, c, wb, eb, ub, vb, s);
  }, st);
}

template <typename T>
void launch_split_substep_vjp(const Dims& d, const Coef<T>& c, const SplitBar<T>& b, void* det_scratch,
                              cudaStream_t st) {
  dim3 blk(32, 4, 2);
  const unsigned fu = (unsigned)field_size(d, LOC_U), fv = (unsigned)field_size(d, LOC_V);
  const unsigned fw = (unsigned)field_size(d, LOC_W), fm = (unsigned)field_size(d, LOC_M);
  {  // corrector^T
    T* dst[14] = {b.upp, b.vpp, b.sfu, b.sfv, b.gx0, b.gy0, b.ppp, b.uh, b.vh, b.uc, b.vc, b.wc, b.u0, b.v0};
    const unsigned len[14] = {fu, fv, fu, fv, fu, fv, fm, fu, fv, fu, fv, fw, fu, fv};
    det_run<T>(det_make<T>(det_scratch, dst, len, 14), [&](const DetSink<T>& s) {
      split_correct_vjp_kernel<T><<<box_grid(d.nx + 1, d.ny + 1, d.nz + 1, blk), blk, 0, st>>>(d, c, b, s);
    }, st);
  }
  {  // column^T, with the forward's alpha dtau products
    const double ad = (double)b.alpha * (double)b.dtau;
    const T a2cp = (T)(ad * ad * c.s.cp), adcp = (T)(ad * c.s.cp);
    T* dst[5] = {b.ppp, b.uh, b.vh, b.sfw, b.sfp};
    const unsigned len[5] = {fm, fu, fv, fw, fm};
    constexpr int PT = 256, PC = 32;
    const size_t smem = (size_t)(4 * d.nz) * PC * sizeof(T);
    if (smem <= 200 * 1024) {  // tiles of 32 columns; the one-thread-per-column march beyond
      static SmemLimit attr_bytes;  // per instantiation
      ensure_smem_limit((const void*)split_column_vjp_tile_kernel<T, PT, PC>, attr_bytes, smem);
      det_run<T>(det_make<T>(det_scratch, dst, len, 5), [&](const DetSink<T>& s) {
        split_column_vjp_tile_kernel<T, PT, PC>
            <<<dim3((d.nx + PC - 1) / PC, d.ny), PT, smem, st>>>(d, c, b, a2cp, adcp, s);
      }, st);
    } else {
      det_run<T>(det_make<T>(det_scratch, dst, len, 5), [&](const DetSink<T>& s) {
        split_column_vjp_kernel<T><<<dim3((d.nx + 127) / 128, d.ny), 128, 0, st>>>(d, c, b, a2cp, adcp, s);
      }, st);
    }
  }
  {  // predictor^T
    T* dst[9] = {b.upp, b.vpp, b.sfu, b.sfv, b.ppp, b.uc, b.vc, b.u0, b.v0};
    const unsigned len[9] = {fu, fv, fu, fv, fm, fu, fv, fu, fv};
    det_run<T>(det_make<T>(det_scratch, dst, len, 9), [&](const DetSink<T>& s) {
      split_predict_vjp_kernel<T><<<box_grid(d.nx + 1, d.ny + 1, d.nz, blk), blk, 0, st>>>(d, c, b, s);
    }, st);
  }
}

template <typename T>
void launch_split_end_vjp(const Dims& d, const T* const* out6, T* const* c6, T* th0b, T* upp, T* vpp, T* wpp,
                          T* ppp, T* sfth, T dtns, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  PtrTable<T> o{}, cb{};
  for (int q = 0; q < 6; ++q) {
    o.p[q] = const_cast<T*>(out6[q]);
    cb.p[q] = c6[q];
  }
  split_end_vjp_kernel<T><<<box_grid(d.nx + 1, d.ny + 1, d.nz + 1, blk), blk, 0, st>>>(d, o, cb, th0b, upp, vpp,
                                                                                     wpp, ppp, sfth, dtns);
}

template <typename T>
void launch_split_init_vjp(const Dims& d, const T* upp, const T* vpp, const T* wpp, const T* ppp, T* const* s6,
                           T* const* c6, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  PtrTable<T> s{}, cb{};
  for (int q = 0; q < 6; ++q) {
    s.p[q] = s6[q];
    cb.p[q] = c6[q];
  }
  split_init_vjp_kernel<T><<<box_grid(d.nx + 1, d.ny + 1, d.nz + 1, blk), blk, 0, st>>>(d, upp, vpp, wpp, ppp, s,
                                                                                      cb);
}

template <typename T>
void launch_split_slow_vjp(const Dims& d, const T* const* sf5, T* const* tend6, T* const* adv4, void* det_scratch,
                           cudaStream_t st) {
  dim3 blk(32, 4, 2);
  PtrTable<T> sf{}, t{}, a{};
  for (int q = 0; q < 5; ++q) sf.p[q] = const_cast<T*>(sf5[q]);
  for (int q = 0; q < 6; ++q) t.p[q] = tend6[q];
  for (int q = 0; q < 4; ++q) a.p[q] = adv4[q];
  const unsigned fm = (unsigned)field_size(d, LOC_M);
  const unsigned len[4] = {fm, fm, fm, fm};
  det_run<T>(det_make<T>(det_scratch, a.p, len, 4), [&](const DetSink<T>& s) {
    split_slow_vjp_kernel<T><<<box_grid(d.nx + 1, d.ny + 1, d.nz + 1, blk), blk, 0, st>>>(d, sf, t, a, s);
  }, st);
}

template <typename T>
void launch_split_adv_vjp(const Dims& d, const Coef<T>& c, const T* u, const T* v, const T* w, const T* eta,
                          const T* th, T eps_l, const T* const* adv4, T* ub, T* vb, T* wb, T* eb, T* thb,
                          void* det_scratch, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  PtrTable<T> a{};
  for (int q = 0; q < 4; ++q) a.p[q] = const_cast<T*>(adv4[q]);
  const unsigned fw = (unsigned)field_size(d, LOC_W), fm = (unsigned)field_size(d, LOC_M);
  T* dst[5] = {ub, vb, wb, eb, thb};
  const unsigned len[5] = {(unsigned)field_size(d, LOC_U), (unsigned)field_size(d, LOC_V), fw, fw, fm};
  det_run<T>(det_make<T>(det_scratch, dst, len, 5), [&](const DetSink<T>& s) {
    split_adv_vjp_kernel<T><<<box_grid(d.nx, d.ny, d.nz, blk), blk, 0, st>>>(d, c, u, v, w, eta, th, eps_l, a, ub,
                                                                            vb, wb, eb, thb, s);
  }, st);
}

#define SISL_INST_SPLIT_VJP(T)                                                                                 \
  template void launch_split_diag_vjp<T>(const Dims&, const Coef<T>&, T*, T*, T*, T*, void*, cudaStream_t);    \
  template void launch_split_substep_vjp<T>(const Dims&, const Coef<T>&, const SplitBar<T>&, void*,            \
                                            cudaStream_t);                                                     \
  template void launch_split_end_vjp<T>(const Dims&, const T* const*, T* const*, T*, T*, T*, T*, T*, T*, T,   \
                                        cudaStream_t);                                                         \
  template void launch_split_init_vjp<T>(const Dims&, const T*, const T*, const T*, const T*, T* const*,       \
                                         T* const*, cudaStream_t);                                             \
  template void launch_split_slow_vjp<T>(const Dims&, const T* const*, T* const*, T* const*, void*,            \
                                         cudaStream_t);                                                        \
  template void launch_split_adv_vjp<T>(const Dims&, const Coef<T>&, const T*, const T*, const T*, const T*,   \
                                        const T*, T, const T* const*, T*, T*, T*, T*, T*, void*, cudaStream_t);
SISL_INST_SPLIT_VJP(float)
SISL_INST_SPLIT_VJP(double)
#undef SISL_INST_SPLIT_VJP

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
