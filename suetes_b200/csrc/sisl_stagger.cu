// Staggered two-point averages and differences of CGridOperator3D
// (operators.py:37-132) and their transposes, the building blocks of the
// differentiable step.
//
//  to-centre (u->m, v->m, w->m; n+1 -> n):  out[o] = c0 f[o] + c1 f[o+1]
//  to-face   (m->u, m->v, m->w; n -> n+1):  out[o] = c0 f[o-1] + c1 f[o], 1 <= o <= n-1
//     periodic axis (diff/avg m->u, m->v only, operators.py:86-91, 118-123):
//        out[0] = out[n] = c0 f[n-1] + c1 f[0]
//     otherwise edge padding (operators.py:37-63): out[0] = out[1], out[n] = out[n-1];
//        with stop_gradient the padded copies carry no cotangent.
//  avg: c0 = c1 = 1/2;  diff: c0 = -1/delta, c1 = 1/delta; an optional 2-D
//  multiplier at the output stagger (the map factor of diff, operators.py:100-102).
// The transposes are gathers (no atomics): every input point sums the
// outputs that read it.
#include "sisl_core.cuh"

namespace sisl {
namespace {

struct Shape3 {
  int e[3];
};

template <typename T>
__global__ void __launch_bounds__(256) stagger_kernel(Shape3 in, Shape3 out, int axis, int to_face, int periodic,
                                                      T c0, T c1, const T* __restrict__ mult,
                                                      const T* __restrict__ f, T* __restrict__ o) {
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= out.e[0] || j >= out.e[1] || k >= out.e[2]) return;
  int c[3] = {i, j, k};
  const int a = c[axis];
  const int st[3] = {1, in.e[0], in.e[0] * in.e[1]};
  const int base = i * st[0] + j * st[1] + k * st[2] - a * st[axis];
  T v;
  if (!to_face) {
    v = c0 * ld(f, base + a * st[axis]) + c1 * ld(f, base + (a + 1) * st[axis]);
  } else {
    const int n = in.e[axis];
    int l, r;
    if (a >= 1 && a <= n - 1) { l = a - 1; r = a; }
    else if (periodic) { l = n - 1; r = 0; }
    else if (a == 0) { l = 0; r = 1; }
    else { l = n - 2; r = n - 1; }
    v = c0 * ld(f, base + l * st[axis]) + c1 * ld(f, base + r * st[axis]);
  }
  if (mult) v *= ld(mult, i + out.e[0] * j);
  o[i + out.e[0] * (j + out.e[1] * k)] = v;
}

template <typename T>
__global__ void __launch_bounds__(256) stagger_t_kernel(Shape3 in, Shape3 out, int axis, int to_face,
                                                        int periodic, int stop_grad, T c0, T c1,
                                                        const T* __restrict__ mult, const T* __restrict__ g,
                                                        T* __restrict__ gin) {
  // one thread per INPUT point; g has the output shape
  const int i = blockIdx.x * blockDim.x + threadIdx.x;
  const int j = blockIdx.y * blockDim.y + threadIdx.y;
  const int k = blockIdx.z * blockDim.z + threadIdx.z;
  if (i >= in.e[0] || j >= in.e[1] || k >= in.e[2]) return;
  int c[3] = {i, j, k};
  const int a = c[axis];
  const int st[3] = {1, out.e[0], out.e[0] * out.e[1]};
  const int base = i * st[0] + j * st[1] + k * st[2] - a * st[axis];
  auto G = [&](int o) -> T {
    T v = ld(g, base + o * st[axis]);
    if (mult) {
      int cc[2] = {i, j};
      if (axis < 2) cc[axis] = o;
      v *= ld(mult, cc[0] + out.e[0] * cc[1]);
    }
    return v;
  };
  T acc = T(0);
  if (!to_face) {
    // out[o] reads f[o] (c0) and f[o+1] (c1), o in [0, n_out - 1]
    const int no = out.e[axis];
    if (a <= no - 1) acc += c0 * G(a);
    if (a >= 1) acc += c1 * G(a - 1);
  } else {
    const int n = in.e[axis];
    if (a >= 1) acc += c1 * G(a);          // out[a] reads f[a] as its right point, 1 <= a <= n-1
    if (a + 1 <= n - 1) acc += c0 * G(a + 1);  // out[a+1] reads f[a] as its left point
    if (periodic) {
      const T e = G(0) + G(n);
      if (a == 0) acc += c1 * e;
      if (a == n - 1) acc += c0 * e;
    } else if (!stop_grad) {
      if (a == 0) acc += c0 * G(0);
      if (a == 1) acc += c1 * G(0);
      if (a == n - 2) acc += c0 * G(n);
      if (a == n - 1) acc += c1 * G(n);
    }
  }
  gin[i + in.e[0] * (j + in.e[1] * k)] = acc;
}

dim3 sgrid(const Shape3& s, dim3 blk) {
  return dim3((s.e[0] + blk.x - 1) / blk.x, (s.e[1] + blk.y - 1) / blk.y, (s.e[2] + blk.z - 1) / blk.z);
}

}  // namespace

template <typename T>
void launch_stagger(const int in_shape[3], int axis, int to_face, int periodic, int stop_grad, int transpose, T c0,
                    T c1, const T* mult, const T* src, T* dst, cudaStream_t st) {
  Shape3 in{{in_shape[0], in_shape[1], in_shape[2]}};
  Shape3 out = in;
  out.e[axis] += to_face ? 1 : -1;
  dim3 blk(32, 4, 2);
  if (!transpose)
    stagger_kernel<T><<<sgrid(out, blk), blk, 0, st>>>(in, out, axis, to_face, periodic, c0, c1, mult, src, dst);
  else
    stagger_t_kernel<T><<<sgrid(in, blk), blk, 0, st>>>(in, out, axis, to_face, periodic, stop_grad, c0, c1, mult,
                                                        src, dst);
}

template void launch_stagger<float>(const int*, int, int, int, int, int, float, float, const float*, const float*,
                                    float*, cudaStream_t);
template void launch_stagger<double>(const int*, int, int, int, int, int, double, double, const double*,
                                     const double*, double*, cudaStream_t);

}  // namespace sisl
