// Forward-mode automatic differentiation for the refinement integrals: a
// dual number carries a value and its derivative along one direction, and the
// refinement quadrature is written once as a template over the scalar type,
// so that T = double gives the coefficients and T = Dual their exact
// derivative with respect to one input coordinate (a face node, the
// observation centroid, its normal or tangents).
//
// The quadrature follows the near-field refinement of the reference
// (GreenRetRefined._refine_diagonal / _refine_offdiagonal,
// mnpbem/greenfun/greenret_refined.py:122-516), with the same rules as
// refine_integrals_kernel in green.cu (28-point rule on the curved
// sub-triangles, polar rule around the centroid for the self term).
#pragma once
#include "common.cuh"

namespace bem200 {
namespace ad {

struct Dual {
  double v, d;
  __device__ __forceinline__ Dual() : v(0.0), d(0.0) {}
  __device__ __forceinline__ Dual(double a) : v(a), d(0.0) {}
  __device__ __forceinline__ Dual(double a, double b) : v(a), d(b) {}
};

__device__ __forceinline__ Dual operator+(Dual a, Dual b) { return Dual(a.v + b.v, a.d + b.d); }
__device__ __forceinline__ Dual operator-(Dual a, Dual b) { return Dual(a.v - b.v, a.d - b.d); }
__device__ __forceinline__ Dual operator-(Dual a) { return Dual(-a.v, -a.d); }
__device__ __forceinline__ Dual operator*(Dual a, Dual b) { return Dual(a.v * b.v, a.d * b.v + a.v * b.d); }
__device__ __forceinline__ Dual operator/(Dual a, Dual b) {
  const double iv = 1.0 / b.v;
  return Dual(a.v * iv, (a.d - a.v * iv * b.d) * iv);
}
__device__ __forceinline__ Dual& operator+=(Dual& a, Dual b) { a = a + b; return a; }
__device__ __forceinline__ Dual& operator*=(Dual& a, Dual b) { a = a * b; return a; }
__device__ __forceinline__ Dual dsqrt(Dual a) {
  const double s = sqrt(a.v);
  return Dual(s, s > 0 ? 0.5 * a.d / s : 0.0);
}
__device__ __forceinline__ double dsqrt(double a) { return sqrt(a); }
// max by value; the derivative follows the branch taken
__device__ __forceinline__ Dual dmax(Dual a, Dual b) { return a.v >= b.v ? a : b; }
__device__ __forceinline__ Dual dmax(Dual a, double b) { return a.v >= b ? a : Dual(b); }
__device__ __forceinline__ double dmax(double a, double b) { return fmax(a, b); }
__device__ __forceinline__ double val(double a) { return a; }
__device__ __forceinline__ double val(Dual a) { return a.v; }
__device__ __forceinline__ double der(double) { return 0.0; }
__device__ __forceinline__ double der(Dual a) { return a.d; }

template <typename T>
struct V3 {
  T x, y, z;
};
template <typename T>
__device__ __forceinline__ V3<T> mk3(T x, T y, T z) {
  V3<T> r;
  r.x = x;
  r.y = y;
  r.z = z;
  return r;
}
template <typename T>
__device__ __forceinline__ V3<T> sub(const V3<T>& a, const V3<T>& b) {
  return mk3<T>(a.x - b.x, a.y - b.y, a.z - b.z);
}
template <typename T>
__device__ __forceinline__ T dot(const V3<T>& a, const V3<T>& b) {
  return a.x * b.x + a.y * b.y + a.z * b.z;
}
template <typename T>
__device__ __forceinline__ V3<T> cross(const V3<T>& a, const V3<T>& b) {
  return mk3<T>(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
template <typename T>
__device__ __forceinline__ T norm(const V3<T>& a) {
  return dsqrt(dot(a, a));
}

// shape functions (value and d/dx, d/dy at (x, y)) of the 6-node triangle
// [v0 v1 v2 e01 e12 e20] and of the 9-node quad [v0..v3 e01 e12 e23 e30 c]
template <typename T>
__device__ __forceinline__ void tri6(const V3<T>* a, double x, double y, V3<T>& p, V3<T>& px, V3<T>& py) {
  const double l1 = x, l2 = y, l3 = 1.0 - x - y;
  const double N[6] = {l1 * (2 * l1 - 1), l2 * (2 * l2 - 1), l3 * (2 * l3 - 1), 4 * l1 * l2, 4 * l2 * l3, 4 * l3 * l1};
  const double Dx[6] = {4 * l1 - 1, 0.0, -4 * l3 + 1, 4 * l2, -4 * l2, 4 * (l3 - l1)};
  const double Dy[6] = {0.0, 4 * l2 - 1, -4 * l3 + 1, 4 * l1, 4 * (l3 - l2), -4 * l1};
  p = px = py = mk3<T>(T(0.0), T(0.0), T(0.0));
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    p.x += a[c].x * N[c]; p.y += a[c].y * N[c]; p.z += a[c].z * N[c];
    px.x += a[c].x * Dx[c]; px.y += a[c].y * Dx[c]; px.z += a[c].z * Dx[c];
    py.x += a[c].x * Dy[c]; py.y += a[c].y * Dy[c]; py.z += a[c].z * Dy[c];
  }
}

template <typename T>
__device__ __forceinline__ void quad9(const V3<T>* a, double x, double y, V3<T>& p, V3<T>& px, V3<T>& py) {
  const double N[9] = {0.25 * x * (x - 1) * y * (y - 1), 0.25 * x * (x + 1) * y * (y - 1),
                       0.25 * x * (x + 1) * y * (y + 1), 0.25 * x * (x - 1) * y * (y + 1),
                       0.5 * (1 - x * x) * y * (y - 1),  0.5 * x * (x + 1) * (1 - y * y),
                       0.5 * (1 - x * x) * y * (y + 1),  0.5 * x * (x - 1) * (1 - y * y),
                       (1 - x * x) * (1 - y * y)};
  const double Dx[9] = {0.25 * (2 * x - 1) * y * (y - 1), 0.25 * (2 * x + 1) * y * (y - 1),
                        0.25 * (2 * x + 1) * y * (y + 1), 0.25 * (2 * x - 1) * y * (y + 1),
                        -x * y * (y - 1),                 0.5 * (2 * x + 1) * (1 - y * y),
                        -x * y * (y + 1),                 0.5 * (2 * x - 1) * (1 - y * y),
                        -2 * x * (1 - y * y)};
  const double Dy[9] = {0.25 * x * (x - 1) * (2 * y - 1), 0.25 * x * (x + 1) * (2 * y - 1),
                        0.25 * x * (x + 1) * (2 * y + 1), 0.25 * x * (x - 1) * (2 * y + 1),
                        0.5 * (1 - x * x) * (2 * y - 1),  -x * (x + 1) * y,
                        0.5 * (1 - x * x) * (2 * y + 1),  -x * (x - 1) * y,
                        -2 * (1 - x * x) * y};
  p = px = py = mk3<T>(T(0.0), T(0.0), T(0.0));
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    p.x += a[c].x * N[c]; p.y += a[c].y * N[c]; p.z += a[c].z * N[c];
    px.x += a[c].x * Dx[c]; px.y += a[c].y * Dx[c]; px.z += a[c].z * Dx[c];
    py.x += a[c].x * Dy[c]; py.y += a[c].y * Dy[c]; py.z += a[c].z * Dy[c];
  }
}

// face j: kind 0 flat triangle (nodes 0-2), 1 flat quad (0-3), 2 curved
// triangle (6 nodes), 3 curved quad (9 nodes)
template <typename T>
struct Face {
  V3<T> node[9];
  int kind;
};

// polar-rule point q (self term): position and weight
template <typename T>
__device__ __forceinline__ void polar_pt(const Face<T>& f, const double* rules, int n28, int n3, int n4, int q,
                                         V3<T>& pt, T& w) {
  const double* x3 = rules + 3 * n28;
  const double* y3 = x3 + n3;
  const double* w3 = y3 + n3;
  const double* x4 = w3 + n3;
  const double* y4 = x4 + n4;
  const double* w4 = y4 + n4;
  V3<T> px, py;
  if (f.kind == 2) {
    tri6<T>(f.node, x3[q], y3[q], pt, px, py);
    w = norm(cross(px, py)) * (0.5 * w3[q]);
  } else if (f.kind == 3) {
    quad9<T>(f.node, x4[q], y4[q], pt, px, py);
    w = norm(cross(px, py)) * w4[q];
  } else if (f.kind == 0) {
    const double x = x3[q], y = y3[q], z = 1.0 - x - y;
    pt = mk3<T>(f.node[0].x * x + f.node[1].x * y + f.node[2].x * z, f.node[0].y * x + f.node[1].y * y + f.node[2].y * z,
                f.node[0].z * x + f.node[1].z * y + f.node[2].z * z);
    const T area = norm(cross(sub(f.node[1], f.node[0]), sub(f.node[2], f.node[0]))) * 0.5;
    w = area * w3[q];
  } else {
    const double x = x4[q], y = y4[q];
    const double N[4] = {0.25 * (1 - x) * (1 - y), 0.25 * (1 + x) * (1 - y), 0.25 * (1 + x) * (1 + y),
                         0.25 * (1 - x) * (1 + y)};
    const double Dx[4] = {-0.25 * (1 - y), 0.25 * (1 - y), 0.25 * (1 + y), -0.25 * (1 + y)};
    const double Dy[4] = {-0.25 * (1 - x), -0.25 * (1 + x), 0.25 * (1 + x), 0.25 * (1 - x)};
    pt = px = py = mk3<T>(T(0.0), T(0.0), T(0.0));
    for (int c = 0; c < 4; ++c) {
      pt.x += f.node[c].x * N[c]; pt.y += f.node[c].y * N[c]; pt.z += f.node[c].z * N[c];
      px.x += f.node[c].x * Dx[c]; px.y += f.node[c].y * Dx[c]; px.z += f.node[c].z * Dx[c];
      py.x += f.node[c].x * Dy[c]; py.y += f.node[c].y * Dy[c]; py.z += f.node[c].z * Dy[c];
    }
    w = norm(cross(px, py)) * w4[q];
  }
}

// 28-point-rule point q of sub-triangle s (boundary-element integration)
template <typename T>
__device__ __forceinline__ void tri_pt(const Face<T>& f, const double* rules, int n28, int s, int q, V3<T>& pt, T& w) {
  const double x = rules[q], y = rules[n28 + q], wq = rules[2 * n28 + q];
  if (f.kind >= 2) {
    V3<T> a[6];
    if (f.kind == 2) {
#pragma unroll
      for (int c = 0; c < 6; ++c) a[c] = f.node[c];
    } else {
      const int i0[6] = {0, 1, 2, 4, 5, 8};
      const int i1[6] = {2, 3, 0, 6, 7, 8};
#pragma unroll
      for (int c = 0; c < 6; ++c) a[c] = f.node[s == 0 ? i0[c] : i1[c]];
    }
    V3<T> px, py;
    tri6<T>(a, x, y, pt, px, py);
    w = norm(cross(px, py)) * (0.5 * wq);
  } else {
    const V3<T> v0 = f.node[0];
    const V3<T> v1 = (f.kind == 0 || s == 0) ? f.node[1] : f.node[2];
    const V3<T> v2 = (f.kind == 0 || s == 0) ? f.node[2] : f.node[3];
    const double z = 1.0 - x - y;
    pt = mk3<T>(v0.x * x + v1.x * y + v2.x * z, v0.y * x + v1.y * y + v2.y * z, v0.z * x + v1.z * y + v2.z * z);
    const T area = norm(cross(sub(v1, v0), sub(v2, v0))) * 0.5;
    w = area * wq;
  }
}

}  // namespace ad
}  // namespace bem200
