// Flux-form semi-Lagrangian mass transport and the equation of state.
//
// FluxFormAdvector.advect_3d_split (steppers.py:596-647) with advect_1d
// (steppers.py:552-594): cell masses rho dx dy / m^2 dz_m, one sweep per
// axis (x, y, z) remapping the cumulative mass to the departure interfaces
// with linear interpolation.  One thread per grid line; the cumulative mass
// of each line is accumulated in float64 in a line-interleaved scratch array
// (position-major, line-fastest, so neighbouring threads touch neighbouring
// words).  Periodic axes use the three-copy extension of steppers.py:569-582
// evaluated in closed form: M_ext(p) = floor(p / N) S + M(p mod N).
#include "sisl_core.cuh"

#include <mutex>

#include "../../include/sisl_b200.h"

namespace sisl {
namespace {

template <typename T>
__device__ __forceinline__ T cell_volume(const Dims& d, const Coef<T>& c, int i, int j, int k) {
  const T m = ld(c.mm, h_m(d, i, j));
  return (T)(d.dx * d.dy) / (m * m) * ld(c.dzm, im(d, i, j, k));
}

template <typename T>
__global__ void ffsl_mass_kernel(Dims d, Coef<T> c, const T* __restrict__ rho, T* mass) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= d.nx || j >= d.ny || k >= d.nz) return;
  const int p = im(d, i, j, k);
  mass[p] = ld(rho, p) * cell_volume(d, c, i, j, k);
}

template <typename T>
__global__ void ffsl_sweep_kernel(Dims d, Coef<T> c, int axis, const T* __restrict__ in, const T* __restrict__ vel,
                                  T* out, double* __restrict__ M, int periodic, double dt, int to_density) {
  const int line = blockIdx.x * blockDim.x + threadIdx.x;
  int N, nlines, a, b;
  if (axis == 0) { N = d.nx; nlines = d.ny * d.nz; a = line % d.ny; b = line / d.ny; }
  else if (axis == 1) { N = d.ny; nlines = d.nx * d.nz; a = line % d.nx; b = line / d.nx; }
  else { N = d.nz; nlines = d.nx * d.ny; a = line % d.nx; b = line / d.nx; }
  if (line >= nlines) return;
  auto cell = [&](int q) -> int {
    if (axis == 0) return im(d, q, a, b);
    if (axis == 1) return im(d, a, q, b);
    return im(d, a, b, q);
  };
  auto cfl = [&](int q) -> double {  // interface Courant number (steppers.py:614-616)
    if (axis == 0) return (double)ld(vel, iu(d, q, a, b)) * (double)ld(c.mu, h_u(d, q, a)) * dt / d.dx;
    if (axis == 1) return (double)ld(vel, iv(d, a, q, b)) * (double)ld(c.mv, h_v(d, a, q)) * dt / d.dy;
    return (double)ld(vel, iw(d, a, b, q)) * dt;
  };
  // cumulative mass M[0..N]
  double s = 0.0;
  M[line] = 0.0;
  for (int q = 0; q < N; ++q) {
    s += (double)ld(in, cell(q));
    M[(size_t)(q + 1) * nlines + line] = s;
  }
  const double S = s;
  auto Mext = [&](long long p) -> double {  // periodic three-copy cumulative mass
    const long long blk = p / N, r = p % N;
    return (double)blk * S + M[(size_t)r * nlines + line];
  };
  auto Mdep = [&](int q) -> double {
    const double c0 = cfl(q);
    if (periodic) {
      const double dep = (double)(q + N) - c0;
      const double lo = floor(dep);
      const double w = dep - lo;
      const long long L = 3LL * N + 1;
      long long i0 = (long long)lo, i1 = i0 + 1;
      i0 = i0 < 0 ? 0 : (i0 > L - 1 ? L - 1 : i0);
      i1 = i1 < 0 ? 0 : (i1 > L - 1 ? L - 1 : i1);
      return (1.0 - w) * Mext(i0) + w * Mext(i1);
    }
    double dep = (double)q - c0;
    dep = fmin(fmax(dep, 0.0), (double)N);
    const double lo = floor(dep);
    const double w = dep - lo;
    int i0 = (int)lo, i1 = i0 + 1;
    i0 = min(max(i0, 0), N);
    i1 = min(max(i1, 0), N);
    return (1.0 - w) * M[(size_t)i0 * nlines + line] + w * M[(size_t)i1 * nlines + line];
  };
  double prev = Mdep(0);
  for (int q = 0; q < N; ++q) {
    const double nxt = Mdep(q + 1);
    const int p = cell(q);
    double val = nxt - prev;
    if (to_density) {
      int i, j, k;
      if (axis == 0) { i = q; j = a; k = b; } else if (axis == 1) { i = a; j = q; k = b; } else { i = a; j = b; k = q; }
      val /= (double)cell_volume(d, c, i, j, k);
    }
    out[p] = (T)val;
    prev = nxt;
  }
}

// advect_1d (steppers.py:552-594) on nlines independent lines: scalar is
// (nlines, N) and cfl (nlines, N + 1), both line-major.
template <typename T>
__global__ void ffsl_line_kernel(int N, int nlines, const T* __restrict__ sc, const T* __restrict__ cf, T* out,
                                 double* __restrict__ M, int periodic) {
  const int line = blockIdx.x * blockDim.x + threadIdx.x;
  if (line >= nlines) return;
  const T* s_ = sc + (size_t)line * N;
  const T* c_ = cf + (size_t)line * (N + 1);
  double s = 0.0;
  M[line] = 0.0;
  for (int q = 0; q < N; ++q) {
    s += (double)s_[q];
    M[(size_t)(q + 1) * nlines + line] = s;
  }
  const double S = s;
  auto Mat = [&](long long p) -> double {
    if (!periodic) return M[(size_t)p * nlines + line];
    return (double)(p / N) * S + M[(size_t)(p % N) * nlines + line];
  };
  const long long L = periodic ? 3LL * N + 1 : (long long)N + 1;
  auto Mdep = [&](int q) -> double {
    double dep = periodic ? (double)(q + N) - (double)c_[q] : fmin(fmax((double)q - (double)c_[q], 0.0), (double)N);
    const double lo = floor(dep), w = dep - lo;
    long long i0 = (long long)lo, i1 = i0 + 1;
    i0 = i0 < 0 ? 0 : (i0 > L - 1 ? L - 1 : i0);
    i1 = i1 < 0 ? 0 : (i1 > L - 1 ? L - 1 : i1);
    return (1.0 - w) * Mat(i0) + w * Mat(i1);
  };
  double prev = Mdep(0);
  for (int q = 0; q < N; ++q) {
    const double nxt = Mdep(q + 1);
    out[(size_t)line * N + q] = (T)(nxt - prev);
    prev = nxt;
  }
}

// ---------------------------------------------------------------------------
// Reverse of advect_1d on one line (the VJP XLA forms for steppers.py:552-594):
//   Md(q) = map_coordinates(M, dep(q), order 1, nearest), out(q) = Md(q+1) - Md(q)
//   dep(q) = clip(q - cfl(q), 0, N) (open) or q + N - cfl(q) (periodic, three
//   copies); clip = maximum then minimum, so an exact tie passes half the
//   cotangent; floor() carries none.
// Md_bar(q) = out_bar(q-1) - out_bar(q); M_bar gets the interpolation weights;
// cfl_bar(q) = -clip'(q) Md_bar(q) (M(i1) - M(i0)); scalar_bar(t) = sum of
// M_bar(p) over p > t (plus the periodic total's cotangent).  M and M_bar are
// float64 line scratch, position-major and line-fastest.
// ---------------------------------------------------------------------------
template <typename ScalarAt, typename CflAt, typename OutBarAt, typename ScalarBarSet, typename CflBarSet>
__device__ __forceinline__ void advect_line_vjp(int N, int nlines, int line, int periodic, ScalarAt sc, CflAt cfl,
                                                OutBarAt ob, ScalarBarSet set_sb, CflBarSet set_cb,
                                                double* __restrict__ M, double* __restrict__ Mb) {
  auto at = [&](const double* A, long long p) -> double { return A[(size_t)p * nlines + line]; };
  double s = 0.0;
  M[line] = 0.0;
  Mb[line] = 0.0;
  for (int q = 0; q < N; ++q) {
    s += sc(q);
    M[(size_t)(q + 1) * nlines + line] = s;
    Mb[(size_t)(q + 1) * nlines + line] = 0.0;
  }
  const double S = s;
  double Sb = 0.0;
  const long long L = periodic ? 3LL * N + 1 : (long long)N + 1;
  auto Mat = [&](long long p) -> double {
    if (!periodic) return at(M, p);
    return (double)(p / N) * S + at(M, p % N);
  };
  auto Mb_add = [&](long long p, double x) {
    if (!periodic) {
      Mb[(size_t)p * nlines + line] += x;
      return;
    }
    Mb[(size_t)(p % N) * nlines + line] += x;
    Sb += (double)(p / N) * x;
  };
  for (int q = 0; q <= N; ++q) {
    const double mdb = (q >= 1 ? ob(q - 1) : 0.0) - (q <= N - 1 ? ob(q) : 0.0);
    const double c0 = cfl(q);
    double dep, cg = 1.0;
    if (periodic) {
      dep = (double)(q + N) - c0;
    } else {
      const double x = (double)q - c0;
      if (x < 0.0) { dep = 0.0; cg = 0.0; }
      else if (x == 0.0) { dep = 0.0; cg = 0.5; }
      else if (x < (double)N) { dep = x; }
      else if (x == (double)N) { dep = (double)N; cg = 0.5; }
      else { dep = (double)N; cg = 0.0; }
    }
    const double lo = floor(dep), w = dep - lo;
    long long i0 = (long long)lo, i1 = i0 + 1;
    i0 = i0 < 0 ? 0 : (i0 > L - 1 ? L - 1 : i0);
    i1 = i1 < 0 ? 0 : (i1 > L - 1 ? L - 1 : i1);
    set_cb(q, -cg * mdb * (Mat(i1) - Mat(i0)));
    if (mdb != 0.0) {
      Mb_add(i0, (1.0 - w) * mdb);
      Mb_add(i1, w * mdb);
    }
  }
  double acc = periodic ? Sb : 0.0;
  for (int q = N - 1; q >= 0; --q) {
    if (q + 1 <= N - 1 || !periodic) acc += at(Mb, q + 1);
    set_sb(q, acc);
  }
}

// one reverse x, y or z sweep of advect_3d_split; ob_density: the forward
// sweep divided by the cell volume (the z sweep); ib_density: its input was
// the density times the cell volume (the x sweep)
template <typename T>
__global__ void ffsl_sweep_vjp_kernel(Dims d, Coef<T> c, int axis, const T* __restrict__ in,
                                      const T* __restrict__ vel, const T* __restrict__ ob, T* ib, T* velb,
                                      double* __restrict__ M, double* __restrict__ Mb, int periodic, double dt,
                                      int ob_density, int ib_density) {
  const int line = blockIdx.x * blockDim.x + threadIdx.x;
  int N, nlines, a, b;
  if (axis == 0) { N = d.nx; nlines = d.ny * d.nz; a = line % d.ny; b = line / d.ny; }
  else if (axis == 1) { N = d.ny; nlines = d.nx * d.nz; a = line % d.nx; b = line / d.nx; }
  else { N = d.nz; nlines = d.nx * d.ny; a = line % d.nx; b = line / d.nx; }
  if (line >= nlines) return;
  auto ijk = [&](int q, int& i, int& j, int& k) {
    if (axis == 0) { i = q; j = a; k = b; } else if (axis == 1) { i = a; j = q; k = b; } else { i = a; j = b; k = q; }
  };
  auto cell = [&](int q) -> int {
    int i, j, k;
    ijk(q, i, j, k);
    return im(d, i, j, k);
  };
  auto vol = [&](int q) -> double {
    int i, j, k;
    ijk(q, i, j, k);
    return (double)cell_volume(d, c, i, j, k);
  };
  auto face = [&](int q) -> int {
    if (axis == 0) return iu(d, q, a, b);
    if (axis == 1) return iv(d, a, q, b);
    return iw(d, a, b, q);
  };
  auto factor = [&](int q) -> double {  // d cfl / d velocity (steppers.py:614-616)
    if (axis == 0) return (double)ld(c.mu, h_u(d, q, a)) * dt / d.dx;
    if (axis == 1) return (double)ld(c.mv, h_v(d, a, q)) * dt / d.dy;
    return dt;
  };
  advect_line_vjp(
      N, nlines, line, periodic, [&](int q) { return (double)ld(in, cell(q)); },
      [&](int q) { return (double)ld(vel, face(q)) * factor(q); },
      [&](int q) {
        const double x = (double)ld(ob, cell(q));
        return ob_density ? x / vol(q) : x;
      },
      [&](int q, double x) { ib[cell(q)] = (T)(ib_density ? x * vol(q) : x); },
      [&](int q, double x) {
        if (velb) velb[face(q)] = (T)(x * factor(q));
      },
      M, Mb);
}

// advect_1d VJP on nlines independent lines (layouts of ffsl_line_kernel)
template <typename T>
__global__ void ffsl_line_vjp_kernel(int N, int nlines, const T* __restrict__ sc, const T* __restrict__ cf,
                                     const T* __restrict__ ob, T* sb, T* cb, double* __restrict__ M,
                                     double* __restrict__ Mb, int periodic) {
  const int line = blockIdx.x * blockDim.x + threadIdx.x;
  if (line >= nlines) return;
  const size_t s0 = (size_t)line * N, c0 = (size_t)line * (N + 1);
  advect_line_vjp(
      N, nlines, line, periodic, [&](int q) { return (double)sc[s0 + q]; },
      [&](int q) { return (double)cf[c0 + q]; }, [&](int q) { return (double)ob[s0 + q]; },
      [&](int q, double x) { sb[s0 + q] = (T)x; },
      [&](int q, double x) {
        if (cb) cb[c0 + q] = (T)x;
      },
      M, Mb);
}

template <typename T>
__global__ void eos_kernel(Dims d, Coef<T> c, const T* __restrict__ th, const T* __restrict__ pi, T* rho) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= d.nx || j >= d.ny || k >= d.nz) return;
  const int p = im(d, i, j, k);
  const T thf = ld(th, p) + ld(c.thb, p), pif = ld(pi, p) + ld(c.pib, p);
  rho[p] = (T)c.s.p0 / ((T)c.s.Rd * thf) * pow(pif, (T)(c.s.cvd / c.s.Rd));  // steppers.py:1056
}

dim3 box3(const Dims& d, dim3 blk) {
  return dim3((d.nx + blk.x - 1) / blk.x, (d.ny + blk.y - 1) / blk.y, (d.nz + blk.z - 1) / blk.z);
}

}  // namespace

size_t ffsl_scratch_doubles(const Dims& d) {
  size_t x = (size_t)(d.nx + 1) * d.ny * d.nz, y = (size_t)(d.ny + 1) * d.nx * d.nz, z = (size_t)(d.nz + 1) * d.nx * d.ny;
  size_t m = x > y ? x : y;
  return m > z ? m : z;
}

// out = FFSL(field); tmp0/tmp1 are mass-point scratch fields, M the
// float64 line scratch of ffsl_scratch_doubles() entries.
template <typename T>
int launch_ffsl(const Dims& d, const Coef<T>& c, const T* field, const T* u, const T* v, const T* eta, T* out, T* tmp0,
                T* tmp1, double* M, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  ffsl_mass_kernel<T><<<box3(d, blk), blk, 0, st>>>(d, c, field, tmp0);
  const int tb = 128;
  const double dt = c.s.dt;
  ffsl_sweep_kernel<T><<<(d.ny * d.nz + tb - 1) / tb, tb, 0, st>>>(d, c, 0, tmp0, u, tmp1, M, d.px, dt, 0);
  ffsl_sweep_kernel<T><<<(d.nx * d.nz + tb - 1) / tb, tb, 0, st>>>(d, c, 1, tmp1, v, tmp0, M, d.py, dt, 0);
  ffsl_sweep_kernel<T><<<(d.nx * d.ny + tb - 1) / tb, tb, 0, st>>>(d, c, 2, tmp0, eta, out, M, 0, dt, 1);
  return 4;  // kernels launched
}

// field_bar (and u_bar, v_bar, eta_bar where non-null) of out = FFSL(field)
// from out_bar; tmp[0..4] mass-point scratch, M and Mb float64 line scratch
// of ffsl_scratch_doubles() entries each.
template <typename T>
int launch_ffsl_vjp(const Dims& d, const Coef<T>& c, const T* field, const T* u, const T* v, const T* eta,
                    const T* out_bar, T* field_bar, T* u_bar, T* v_bar, T* eta_bar, T* const* tmp, double* M,
                    double* Mb, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  const int tb = 128;
  const double dt = c.s.dt;
  T *mass = tmp[0], *mx = tmp[1], *my = tmp[2], *b1 = tmp[3], *b2 = tmp[4];
  // recompute the sweeps' inputs
  ffsl_mass_kernel<T><<<box3(d, blk), blk, 0, st>>>(d, c, field, mass);
  ffsl_sweep_kernel<T><<<(d.ny * d.nz + tb - 1) / tb, tb, 0, st>>>(d, c, 0, mass, u, mx, M, d.px, dt, 0);
  ffsl_sweep_kernel<T><<<(d.nx * d.nz + tb - 1) / tb, tb, 0, st>>>(d, c, 1, mx, v, my, M, d.py, dt, 0);
  // reverse z, y, x
  ffsl_sweep_vjp_kernel<T><<<(d.nx * d.ny + tb - 1) / tb, tb, 0, st>>>(d, c, 2, my, eta, out_bar, b1, eta_bar, M,
                                                                     Mb, 0, dt, 1, 0);
  ffsl_sweep_vjp_kernel<T><<<(d.nx * d.nz + tb - 1) / tb, tb, 0, st>>>(d, c, 1, mx, v, b1, b2, v_bar, M, Mb, d.py,
                                                                     dt, 0, 0);
  ffsl_sweep_vjp_kernel<T><<<(d.ny * d.nz + tb - 1) / tb, tb, 0, st>>>(d, c, 0, mass, u, b2, field_bar, u_bar, M,
                                                                     Mb, d.px, dt, 0, 1);
  return 6;  // kernels launched
}

template <typename T>
void launch_ffsl_lines_vjp(int N, int nlines, const T* scalar, const T* cfl, const T* out_bar, T* scalar_bar,
                           T* cfl_bar, double* M, double* Mb, int periodic, cudaStream_t st) {
  ffsl_line_vjp_kernel<T><<<(nlines + 127) / 128, 128, 0, st>>>(N, nlines, scalar, cfl, out_bar, scalar_bar, cfl_bar,
                                                                M, Mb, periodic);
}

template <typename T>
void launch_ffsl_lines(int N, int nlines, const T* scalar, const T* cfl, T* out, double* M, int periodic,
                       cudaStream_t st) {
  ffsl_line_kernel<T><<<(nlines + 127) / 128, 128, 0, st>>>(N, nlines, scalar, cfl, out, M, periodic);
}

template <typename T>
void launch_eos(const Dims& d, const Coef<T>& c, const T* th, const T* pi, T* rho, cudaStream_t st) {
  dim3 blk(32, 4, 2);
  eos_kernel<T><<<box3(d, blk), blk, 0, st>>>(d, c, th, pi, rho);
}

template int launch_ffsl<float>(const Dims&, const Coef<float>&, const float*, const float*, const float*,
                                const float*, float*, float*, float*, double*, cudaStream_t);
template int launch_ffsl<double>(const Dims&, const Coef<double>&, const double*, const double*, const double*,
                                 const double*, double*, double*, double*, double*, cudaStream_t);
template int launch_ffsl_vjp<float>(const Dims&, const Coef<float>&, const float*, const float*, const float*,
                                    const float*, const float*, float*, float*, float*, float*, float* const*,
                                    double*, double*, cudaStream_t);
template int launch_ffsl_vjp<double>(const Dims&, const Coef<double>&, const double*, const double*, const double*,
                                     const double*, const double*, double*, double*, double*, double*,
                                     double* const*, double*, double*, cudaStream_t);
template void launch_ffsl_lines_vjp<float>(int, int, const float*, const float*, const float*, float*, float*,
                                           double*, double*, int, cudaStream_t);
template void launch_ffsl_lines_vjp<double>(int, int, const double*, const double*, const double*, double*, double*,
                                            double*, double*, int, cudaStream_t);
template void launch_ffsl_lines<float>(int, int, const float*, const float*, float*, double*, int, cudaStream_t);
template void launch_ffsl_lines<double>(int, int, const double*, const double*, double*, double*, int,
                                        cudaStream_t);
template void launch_eos<float>(const Dims&, const Coef<float>&, const float*, const float*, float*, cudaStream_t);
template void launch_eos<double>(const Dims&, const Coef<double>&, const double*, const double*, double*,
                                 cudaStream_t);

}  // namespace sisl

// ---------------------------------------------------------------------------
// Allocation-free line transport.
//
// Some callers cannot call cudaMalloc while they advance a model: a stream
// in global-mode graph capture (an allocation there breaks the capture), a
// host model that hands this library only buffers it pre-sized from its own
// pool and forbids allocation inside its time loop, or an FFI handler that
// was registered without a workspace.  sisl_ffsl_lines_noalloc serves them:
// the float64 cumulative-mass scratch of the line kernel lives in the fixed
// device array below (SISL_FFSL_NOALLOC_MAX_DOUBLES doubles = 8 MiB, held on
// every GPU that loads this library until the process exits).  In host code
// the array's name is only a host-side stand-in, never a device address: the
// address is fetched with cudaGetSymbolAddress once per device (the first
// call on a device does it, with that device current) and cached.
// ---------------------------------------------------------------------------
namespace sisl {

static __device__ __align__(256) double g_ffsl_line_scratch[SISL_FFSL_NOALLOC_MAX_DOUBLES];

namespace {
std::mutex g_scratch_mutex;
constexpr int kMaxDevices = 64;
double* g_scratch_device_address[kMaxDevices] = {nullptr};

int line_scratch_address(double** out) {
  int dev = -1;
  if (cudaGetDevice(&dev) != cudaSuccess || dev < 0 || dev >= kMaxDevices) return SISL_ERR_CUDA;
  std::lock_guard<std::mutex> lock(g_scratch_mutex);
  if (g_scratch_device_address[dev] == nullptr) {
    void* p = nullptr;
    if (cudaGetSymbolAddress(&p, g_ffsl_line_scratch) != cudaSuccess) return SISL_ERR_CUDA;
    g_scratch_device_address[dev] = static_cast<double*>(p);
  }
  *out = g_scratch_device_address[dev];
  return SISL_OK;
}
}  // namespace

}  // namespace sisl

extern "C" int sisl_ffsl_lines_noalloc(int dtype, int n, int nlines, const void* scalar, const void* cfl, int periodic,
                                       void* out, void* stream) {
  using namespace sisl;
  if (n < 1 || nlines < 1 || !scalar || !cfl || !out) return SISL_ERR_ARG;
  if (dtype != SISL_F32 && dtype != SISL_F64) return SISL_ERR_ARG;
  if (((size_t)n + 1) * (size_t)nlines > (size_t)SISL_FFSL_NOALLOC_MAX_DOUBLES) return SISL_ERR_SCRATCH_LIMIT;
  double* M = nullptr;
  int rc = line_scratch_address(&M);
  if (rc != SISL_OK) return rc;
  cudaStream_t st = (cudaStream_t)stream;
  // Every scratch word a line reads is written by that line first, so the
  // previous call's contents never need clearing.
  if (dtype == SISL_F64)
    launch_ffsl_lines<double>(n, nlines, (const double*)scalar, (const double*)cfl, (double*)out, M,
                              periodic ? 1 : 0, st);
  else
    launch_ffsl_lines<float>(n, nlines, (const float*)scalar, (const float*)cfl, (float*)out, M, periodic ? 1 : 0,
                             st);
  return cudaGetLastError() == cudaSuccess ? SISL_OK : SISL_ERR_CUDA;
}
