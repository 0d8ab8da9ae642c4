// Retarded Green-function kernels: near-field refinement (classification,
// quadrature integrals, closed-surface correction) and the per-wavelength
// assembly of G1, G2, H1, H2.  All arithmetic is FP64; outputs may be stored
// as complex128 or complex64.
//
// Reference behaviour followed (MNPBEM Python port v1.6.2):
//   refinematrix            mnpbem/greenfun/refine_utils.py:12-158
//   _refine_diagonal        mnpbem/greenfun/greenret_refined.py:122-285
//   _refine_offdiagonal     mnpbem/greenfun/greenret_refined.py:287-516
//   closed-surface terms    mnpbem/greenfun/compgreen_ret.py:192-272, :376-400
//                           mnpbem/greenfun/compgreen_stat.py:219-450
//   eval (G, F, H1, H2)     mnpbem/greenfun/greenret_refined.py:654-810
//   region connectivity     mnpbem/greenfun/compgreen_ret.py:435-505, :739-858
#include <cstdarg>
#include <cmath>
#include <atomic>
#include <mutex>
#include <unordered_map>

#include "common.cuh"

namespace bem200 {

static thread_local char g_err[1024] = {0};

void set_error(const char* fmt, ...) {
  va_list ap;
  va_start(ap, fmt);
  vsnprintf(g_err, sizeof(g_err), fmt, ap);
  va_end(ap);
}
const char* get_error() { return g_err; }

static std::atomic<unsigned long long> g_launches{0};
static thread_local bool t_count_suspended = false;
void count_launch() {
  if (!t_count_suspended) g_launches.fetch_add(1, std::memory_order_relaxed);
}
void count_launches(unsigned long long n) { g_launches.fetch_add(n, std::memory_order_relaxed); }
void count_suspend(bool on) { t_count_suspended = on; }
unsigned long long launch_count() { return g_launches.load(std::memory_order_relaxed); }

cudaError_t set_kernel_attrs(const void* kern, int smem_bytes, bool nonportable_cluster) {
  static std::mutex mu;
  static std::unordered_map<const void*, int> done;  // kernel -> largest smem limit set
  std::lock_guard<std::mutex> lock(mu);
  auto it = done.find(kern);
  if (it != done.end() && it->second >= smem_bytes) return cudaSuccess;
  cudaError_t e = cudaSuccess;
  if (smem_bytes > 0) e = cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, smem_bytes);
  if (e == cudaSuccess && nonportable_cluster)
    e = cudaFuncSetAttribute(kern, cudaFuncAttributeNonPortableClusterSizeAllowed, 1);
  if (e == cudaSuccess) done[kern] = smem_bytes;
  return e;
}

constexpr int kMaxOrder = 7;
constexpr double kEps = 2.220446049250313e-16;  // numpy finfo(float).eps
constexpr double kTwoPi = 6.283185307179586;

__device__ __forceinline__ double3 ld3(const double* p, long long i) {
  return make_double3(p[3 * i], p[3 * i + 1], p[3 * i + 2]);
}
__device__ __forceinline__ double dot3(double3 a, double3 b) { return a.x * b.x + a.y * b.y + a.z * b.z; }
__device__ __forceinline__ double3 sub3(double3 a, double3 b) {
  return make_double3(a.x - b.x, a.y - b.y, a.z - b.z);
}
__device__ __forceinline__ double3 cross3(double3 a, double3 b) {
  return make_double3(a.y * b.z - a.z * b.y, a.z * b.x - a.x * b.z, a.x * b.y - a.y * b.x);
}
__device__ __forceinline__ double norm3(double3 a) { return sqrt(a.x * a.x + a.y * a.y + a.z * a.z); }

__device__ __forceinline__ double warp_sum(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(0xffffffffu, v, o);
  return v;
}
__device__ __forceinline__ double warp_max(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

// ----------------------------------------------------------------- (a1)
// Classification of (i, j) with the algebraic distance of the reference
// (|p_i|^2 + |p_j|^2 - 2 p_i.p_j, tiny values clamped to 0).
__device__ __forceinline__ int classify_pair(double3 pi, double ni2, double radi, double3 pj, double nj2,
                                             double radj, double abs_cut, double rel_cut) {
  double dotp = fma(pi.z, pj.z, fma(pi.y, pj.y, pi.x * pj.x));
  double dsq = __dadd_rn(ni2, nj2) - 2.0 * dotp;
  if (dsq < 1e-10) dsq = 0.0;
  double d = sqrt(dsq);
  if (d == 0.0) return 2;
  double d2 = d - radj;
  double idrel = d2 / radi;
  return ((d2 < abs_cut) || (idrel < rel_cut)) ? 1 : 0;
}

__device__ __forceinline__ double sqnorm_np(double3 p) {
  // numpy sum(p * p, axis=1) over 3 entries: (x*x + y*y) + z*z without FMA
  return __dadd_rn(__dadd_rn(__dmul_rn(p.x, p.x), __dmul_rn(p.y, p.y)), __dmul_rn(p.z, p.z));
}

// one warp per row i; lanes sweep the columns
__global__ void refine_classify_kernel(int n, const double* __restrict__ pos, const double* __restrict__ rad,
                                       double abs_cut, double rel_cut, int32_t* __restrict__ row_count,
                                       const int64_t* __restrict__ row_ptr, int32_t* __restrict__ ref_row,
                                       int32_t* __restrict__ ref_col, int8_t* __restrict__ ref_kind) {
  int warp = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (warp >= n) return;
  const int i = warp;
  double3 pi = ld3(pos, i);
  double ni2 = sqnorm_np(pi);
  double radi = rad[i];
  long long base = row_ptr ? row_ptr[i] : 0;
  int count = 0;
  for (int j0 = 0; j0 < n; j0 += 32) {
    int j = j0 + lane;
    int kind = 0;
    if (j < n) {
      double3 pj = ld3(pos, j);
      kind = classify_pair(pi, ni2, radi, pj, sqnorm_np(pj), rad[j], abs_cut, rel_cut);
    }
    unsigned mask = __ballot_sync(0xffffffffu, kind != 0);
    if (row_ptr != nullptr && kind != 0) {
      int off = __popc(mask & ((1u << lane) - 1u));
      long long e = base + count + off;
      ref_row[e] = i;
      ref_col[e] = j;
      ref_kind[e] = (int8_t)kind;
    }
    count += __popc(mask);
  }
  if (row_ptr == nullptr && lane == 0) row_count[i] = count;
}

// exclusive scan of n int32 counts -> int64 row_ptr (single block)
__global__ void scan_kernel(int n, const int32_t* __restrict__ count, int64_t* __restrict__ row_ptr) {
  __shared__ long long part[1024];
  int t = threadIdx.x;
  int nt = blockDim.x;
  int chunk = (n + nt - 1) / nt;
  int lo = t * chunk, hi = min(n, lo + chunk);
  long long s = 0;
  for (int i = lo; i < hi; ++i) s += count[i];
  part[t] = s;
  __syncthreads();
  for (int o = 1; o < nt; o <<= 1) {
    long long v = (t >= o) ? part[t - o] : 0;
    __syncthreads();
    part[t] += v;
    __syncthreads();
  }
  long long run = (t == 0) ? 0 : part[t - 1];
  for (int i = lo; i < hi; ++i) {
    row_ptr[i] = run;
    run += count[i];
  }
  if (t == nt - 1) row_ptr[n] = part[nt - 1];
}

// ------------------------------------------------------------- (a2, a3)
struct FaceGeom {
  double3 node[9];
  int kind;
  double area;
};

__device__ __forceinline__ void load_face(FaceGeom& fg, const double* nodes, const int32_t* face_kind,
                                          const double* area, int j) {
  fg.kind = face_kind[j];
  fg.area = area[j];
  int nn = (fg.kind == 0) ? 3 : (fg.kind == 1 ? 4 : (fg.kind == 2 ? 6 : 9));
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    if (c < nn) fg.node[c] = ld3(nodes, 9LL * j + c);
  }
}

// 6-node triangle through nodes a[0..5]: value, d/dx, d/dy at (x, y)
__device__ __forceinline__ void tri6_eval(const double3* a, double x, double y, double3& p, double3& px,
                                          double3& py) {
  double l1 = x, l2 = y, l3 = 1.0 - x - y;
  double N[6] = {l1 * (2 * l1 - 1), l2 * (2 * l2 - 1), l3 * (2 * l3 - 1), 4 * l1 * l2, 4 * l2 * l3, 4 * l3 * l1};
  double Dx[6] = {4 * l1 - 1, 0.0, -4 * l3 + 1, 4 * l2, -4 * l2, 4 * (l3 - l1)};
  double Dy[6] = {0.0, 4 * l2 - 1, -4 * l3 + 1, 4 * l1, 4 * (l3 - l2), -4 * l1};
  p = px = py = make_double3(0, 0, 0);
#pragma unroll
  for (int c = 0; c < 6; ++c) {
    p.x += N[c] * a[c].x; p.y += N[c] * a[c].y; p.z += N[c] * a[c].z;
    px.x += Dx[c] * a[c].x; px.y += Dx[c] * a[c].y; px.z += Dx[c] * a[c].z;
    py.x += Dy[c] * a[c].x; py.y += Dy[c] * a[c].y; py.z += Dy[c] * a[c].z;
  }
}

__device__ __forceinline__ void quad9_eval(const double3* a, double x, double y, double3& p, double3& px,
                                           double3& py) {
  double N[9] = {0.25 * x * (x - 1) * y * (y - 1), 0.25 * x * (x + 1) * y * (y - 1),
                 0.25 * x * (x + 1) * y * (y + 1), 0.25 * x * (x - 1) * y * (y + 1),
                 0.5 * (1 - x * x) * y * (y - 1),  0.5 * x * (x + 1) * (1 - y * y),
                 0.5 * (1 - x * x) * y * (y + 1),  0.5 * x * (x - 1) * (1 - y * y),
                 (1 - x * x) * (1 - y * y)};
  double Dx[9] = {0.25 * (2 * x - 1) * y * (y - 1), 0.25 * (2 * x + 1) * y * (y - 1),
                  0.25 * (2 * x + 1) * y * (y + 1), 0.25 * (2 * x - 1) * y * (y + 1),
                  -x * y * (y - 1),                 0.5 * (2 * x + 1) * (1 - y * y),
                  -x * y * (y + 1),                 0.5 * (2 * x - 1) * (1 - y * y),
                  -2 * x * (1 - y * y)};
  double Dy[9] = {0.25 * x * (x - 1) * (2 * y - 1), 0.25 * x * (x + 1) * (2 * y - 1),
                  0.25 * x * (x + 1) * (2 * y + 1), 0.25 * x * (x - 1) * (2 * y + 1),
                  0.5 * (1 - x * x) * (2 * y - 1),  -x * (x + 1) * y,
                  0.5 * (1 - x * x) * (2 * y + 1),  -x * (x - 1) * y,
                  -2 * (1 - x * x) * y};
  p = px = py = make_double3(0, 0, 0);
#pragma unroll
  for (int c = 0; c < 9; ++c) {
    p.x += N[c] * a[c].x; p.y += N[c] * a[c].y; p.z += N[c] * a[c].z;
    px.x += Dx[c] * a[c].x; px.y += Dx[c] * a[c].y; px.z += Dx[c] * a[c].z;
    py.x += Dy[c] * a[c].x; py.y += Dy[c] * a[c].y; py.z += Dy[c] * a[c].z;
  }
}

// Polar-rule point q of a face (quadpol): position and weight
__device__ __forceinline__ void polar_point(const FaceGeom& fg, const double* rules, int n28, int n3, int n4,
                                            int q, double3& pt, double& w) {
  const double* x3 = rules + 3 * n28;
  const double* y3 = x3 + n3;
  const double* w3 = y3 + n3;
  const double* x4 = w3 + n3;
  const double* y4 = x4 + n4;
  const double* w4 = y4 + n4;
  double3 px, py;
  if (fg.kind == 2) {
    tri6_eval(fg.node, x3[q], y3[q], pt, px, py);
    w = w3[q] * (0.5 * norm3(cross3(px, py)));
  } else if (fg.kind == 3) {
    quad9_eval(fg.node, x4[q], y4[q], pt, px, py);
    w = w4[q] * norm3(cross3(px, py));
  } else if (fg.kind == 0) {
    double x = x3[q], y = y3[q], z = 1.0 - x - y;
    pt = make_double3(x * fg.node[0].x + y * fg.node[1].x + z * fg.node[2].x,
                      x * fg.node[0].y + y * fg.node[1].y + z * fg.node[2].y,
                      x * fg.node[0].z + y * fg.node[1].z + z * fg.node[2].z);
    w = w3[q] * fg.area;
  } else {
    double x = x4[q], y = y4[q];
    double N[4] = {0.25 * (1 - x) * (1 - y), 0.25 * (1 + x) * (1 - y), 0.25 * (1 + x) * (1 + y),
                   0.25 * (1 - x) * (1 + y)};
    double Dx[4] = {-0.25 * (1 - y), 0.25 * (1 - y), 0.25 * (1 + y), -0.25 * (1 + y)};
    double Dy[4] = {-0.25 * (1 - x), -0.25 * (1 + x), 0.25 * (1 + x), 0.25 * (1 - x)};
    pt = px = py = make_double3(0, 0, 0);
    for (int c = 0; c < 4; ++c) {
      pt.x += N[c] * fg.node[c].x; pt.y += N[c] * fg.node[c].y; pt.z += N[c] * fg.node[c].z;
      px.x += Dx[c] * fg.node[c].x; px.y += Dx[c] * fg.node[c].y; px.z += Dx[c] * fg.node[c].z;
      py.x += Dy[c] * fg.node[c].x; py.y += Dy[c] * fg.node[c].y; py.z += Dy[c] * fg.node[c].z;
    }
    w = w4[q] * norm3(cross3(px, py));
  }
}

// 28-point-rule point q of sub-triangle s of a face (quad())
__device__ __forceinline__ void tri_point(const FaceGeom& fg, const double* rules, int n28, int s, int q,
                                          double3& pt, double& w) {
  const double* x28 = rules;
  const double* y28 = rules + n28;
  const double* w28 = rules + 2 * n28;
  double x = x28[q], y = y28[q];
  if (fg.kind >= 2) {
    double3 a[6];
    if (fg.kind == 2) {
#pragma unroll
      for (int c = 0; c < 6; ++c) a[c] = fg.node[c];
    } else {
      const int i0[6] = {0, 1, 2, 4, 5, 8};
      const int i1[6] = {2, 3, 0, 6, 7, 8};
#pragma unroll
      for (int c = 0; c < 6; ++c) a[c] = fg.node[s == 0 ? i0[c] : i1[c]];
    }
    double3 px, py;
    tri6_eval(a, x, y, pt, px, py);
    w = 0.5 * w28[q] * norm3(cross3(px, py));
  } else {
    double3 v0 = fg.node[0], v1, v2;
    if (fg.kind == 0 || s == 0) {
      v1 = fg.node[1];
      v2 = fg.node[2];
    } else {
      v1 = fg.node[2];
      v2 = fg.node[3];
    }
    double z = 1.0 - x - y;
    pt = make_double3(x * v0.x + y * v1.x + z * v2.x, x * v0.y + y * v1.y + z * v2.y,
                      x * v0.z + y * v1.z + z * v2.z);
    double area = 0.5 * norm3(cross3(sub3(v1, v0), sub3(v2, v0)));
    w = w28[q] * area;
  }
}

__global__ void refine_integrals_kernel(long long nref, const int32_t* __restrict__ ref_row,
                                        const int32_t* __restrict__ ref_col, const int8_t* __restrict__ ref_kind,
                                        const double* __restrict__ pos, const double* __restrict__ nvec,
                                        const double* __restrict__ tvec1, const double* __restrict__ tvec2,
                                        const double* __restrict__ area, const double* __restrict__ nodes,
                                        const int32_t* __restrict__ face_kind, const double* __restrict__ rules,
                                        int n28, int n3, int n4, int order, double* __restrict__ gout,
                                        double* __restrict__ fout) {
  long long e = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (e >= nref) return;
  const int i = ref_row[e], j = ref_col[e], kind = ref_kind[e];
  const int no = order + 1;
  FaceGeom fg;
  load_face(fg, nodes, face_kind, area, j);
  const double3 pi = ld3(pos, i);
  const double3 ni = ld3(nvec, i);
  double sg[kMaxOrder + 1], s1[kMaxOrder + 1], s2[kMaxOrder + 1], s3[kMaxOrder + 1];
#pragma unroll
  for (int m = 0; m <= kMaxOrder; ++m) sg[m] = s1[m] = s2[m] = s3[m] = 0.0;

  if (kind == 2) {
    // polar integration around the centroid of face j (self term)
    const int npts = (fg.kind == 0 || fg.kind == 2) ? n3 : n4;
    const double3 t1 = ld3(tvec1, i), t2 = ld3(tvec2, i);
    double rmax = 0.0;
    for (int q = lane; q < npts; q += 32) {
      double3 pt;
      double w;
      polar_point(fg, rules, n28, n3, n4, q, pt, w);
      rmax = fmax(rmax, fmax(norm3(sub3(pi, pt)), kEps));
    }
    rmax = warp_max(rmax);
    const double rfloor = 1e-4 * rmax;
    for (int q = lane; q < npts; q += 32) {
      double3 pt;
      double w;
      polar_point(fg, rules, n28, n3, n4, q, pt, w);
      double3 v = sub3(pi, pt);
      double r = fmax(norm3(v), kEps);
      double ndr = dot3(ni, v), in1 = dot3(t1, v), in2 = dot3(t2, v);
      double rr = fmax(r, rfloor);
      double irr3 = 1.0 / (rr * rr * rr);
      double ir = 1.0 / r;
      double rp_m1 = ir;              // r^(m-1)
      double rp_m3 = ir * ir * ir;    // r^(m-3)
      double rp_m = 1.0;              // r^m
#pragma unroll
      for (int m = 0; m <= kMaxOrder; ++m) {
        if (m < no) {
          sg[m] += w * rp_m1;
          s1[m] += w * ndr * rp_m3;
          s2[m] += w * in1 * rp_m * irr3;
          s3[m] += w * in2 * rp_m * irr3;
        }
        rp_m1 *= r;
        rp_m3 *= r;
        rp_m *= r;
      }
    }
    double fact = 1.0;
#pragma unroll
    for (int m = 0; m <= kMaxOrder; ++m) {
      if (m > 0) fact *= m;
      if (m >= no) break;
      double a = warp_sum(sg[m]), b = warp_sum(s1[m]), c = warp_sum(s2[m]), d = warp_sum(s3[m]);
      if (lane == 0) {
        gout[e * no + m] = a / fact;
        double f1 = (m - 1) * b / fact, f2 = (m - 1) * c / fact, f3 = (m - 1) * d / fact;
        fout[(e * 3 + 0) * no + m] = ni.x * f1 + t1.x * f2 + t2.x * f3;
        fout[(e * 3 + 1) * no + m] = ni.y * f1 + t1.y * f2 + t2.y * f3;
        fout[(e * 3 + 2) * no + m] = ni.z * f1 + t1.z * f2 + t2.z * f3;
      }
    }
  } else {
    // boundary-element integration over the (curved) sub-triangles of face j
    const double3 pj = ld3(pos, j);
    const double r0 = norm3(sub3(pj, pi));
    const int nsub = (fg.kind == 1 || fg.kind == 3) ? 2 : 1;
    // s1/s2/s3 hold the x, y, z components of f
    for (int t = lane; t < nsub * n28; t += 32) {
      int s = t / n28, q = t - s * n28;
      double3 pt;
      double w;
      tri_point(fg, rules, n28, s, q, pt, w);
      double3 v = sub3(pi, pt);
      double r = fmax(norm3(v), kEps);
      double ir = 1.0 / r;
      double ir2 = ir * ir, ir3 = ir2 * ir;
      double dl = r - r0;
      double dpow = 1.0;    // dl^m
      double dprev = 0.0;   // dl^(m-1)
      double fm = 1.0;      // m!
      double fm1 = 1.0;     // (m-1)!
#pragma unroll
      for (int m = 0; m <= kMaxOrder; ++m) {
        if (m < no) {
          sg[m] += w * dpow * ir / fm;
          double fs = (m == 0) ? -ir3 : (-dpow * ir3 / fm + dprev * ir2 / fm1);
          s1[m] += w * v.x * fs;
          s2[m] += w * v.y * fs;
          s3[m] += w * v.z * fs;
        }
        dprev = dpow;
        dpow *= dl;
        fm1 = fm;
        fm *= (m + 1);
      }
    }
#pragma unroll
    for (int m = 0; m <= kMaxOrder; ++m) {
      if (m >= no) break;
      double a = warp_sum(sg[m]), b = warp_sum(s1[m]), c = warp_sum(s2[m]), d = warp_sum(s3[m]);
      if (lane == 0) {
        gout[e * no + m] = a;
        fout[(e * 3 + 0) * no + m] = b;
        fout[(e * 3 + 1) * no + m] = c;
        fout[(e * 3 + 2) * no + m] = d;
      }
    }
  }
}

// ------------------------------------------------------------------ (a4)
__device__ __forceinline__ bool in_surface(const uint64_t* closed_mask, const int32_t* pid, int i, int j) {
  uint64_t m = closed_mask[pid[j]];
  return (m >> pid[i]) & 1ull;
}

// S_j = sum_{i in surface(j), i != j} area_i F_ij with the far-field quasistatic F
__global__ void closed_colsum_kernel(int n, const int32_t* __restrict__ pid, const uint64_t* __restrict__ closed_mask,
                                     const double* __restrict__ pos, const double* __restrict__ nvec,
                                     const double* __restrict__ area, double* __restrict__ S) {
  int j = (blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  int lane = threadIdx.x & 31;
  if (j >= n) return;
  uint64_t m = closed_mask[pid[j]];
  if (m == 0) {
    if (lane == 0) S[j] = 0.0;
    return;
  }
  const double3 pj = ld3(pos, j);
  const double aj = area[j];
  double acc = 0.0;
  for (int i = lane; i < n; i += 32) {
    if (i == j || !((m >> pid[i]) & 1ull)) continue;
    double3 r = sub3(ld3(pos, i), pj);
    double d = fmax(norm3(r), kEps);
    double F = -dot3(ld3(nvec, i), r) / (d * d * d) * aj;
    acc += area[i] * F;
  }
  acc = warp_sum(acc);
  if (lane == 0) S[j] = acc;
}

// replace the far value by the refined one for refined (i, j) inside the surface
__global__ void closed_adjust_kernel(long long nref, const int32_t* __restrict__ ref_row,
                                     const int32_t* __restrict__ ref_col, const int32_t* __restrict__ pid,
                                     const uint64_t* __restrict__ closed_mask, const double* __restrict__ pos,
                                     const double* __restrict__ nvec, const double* __restrict__ area, int order,
                                     const double* __restrict__ f, double* __restrict__ S) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nref) return;
  int i = ref_row[e], j = ref_col[e];
  if (!in_surface(closed_mask, pid, i, j)) return;
  const int no = order + 1;
  double3 ni = ld3(nvec, i);
  double Fref = ni.x * f[(e * 3 + 0) * no] + ni.y * f[(e * 3 + 1) * no] + ni.z * f[(e * 3 + 2) * no];
  double Ffar = 0.0;
  if (i != j) {
    double3 r = sub3(ld3(pos, i), ld3(pos, j));
    double d = fmax(norm3(r), kEps);
    Ffar = -dot3(ni, r) / (d * d * d) * area[j];
  }
  atomicAdd(&S[j], area[i] * (Fref - Ffar));
}

__global__ void closed_apply_kernel(long long nref, const int32_t* __restrict__ ref_row,
                                    const int32_t* __restrict__ ref_col, const int8_t* __restrict__ ref_kind,
                                    const int32_t* __restrict__ pid, const uint64_t* __restrict__ closed_mask,
                                    const double* __restrict__ nvec, const double* __restrict__ area, int order,
                                    const double* __restrict__ S, double* __restrict__ f, double* __restrict__ corr) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nref) return;
  int i = ref_row[e], j = ref_col[e];
  if (i != j || ref_kind[e] != 2) return;
  if (closed_mask[pid[j]] == 0) return;
  const int no = order + 1;
  double c = -kTwoPi - S[j] / area[j];
  double3 nj = ld3(nvec, j);
  f[(e * 3 + 0) * no] += c * nj.x;
  f[(e * 3 + 1) * no] += c * nj.y;
  f[(e * 3 + 2) * no] += c * nj.z;
  if (corr) corr[j] = c;
}

__global__ void zero_kernel(double* p, long long n) {
  long long i = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (i < n) p[i] = 0.0;
}

__global__ void refine_project_kernel(long long nref, const int32_t* __restrict__ ref_row,
                                      const double* __restrict__ nvec, int order, const double* __restrict__ f,
                                      double* __restrict__ fn) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nref) return;
  const int no = order + 1;
  double3 ni = ld3(nvec, ref_row[e]);
  for (int m = 0; m < no; ++m)
    fn[e * no + m] = ni.x * f[(e * 3 + 0) * no + m] + ni.y * f[(e * 3 + 1) * no + m] + ni.z * f[(e * 3 + 2) * no + m];
}

// ------------------------------------------------------------------ (a6)
constexpr int kMaxMat = 16;
struct KTable {
  double re[kMaxMat], im[kMaxMat];
};

template <typename C>
__device__ __forceinline__ void store_c(void* base, long long idx, double re, double im) {
  reinterpret_cast<C*>(base)[idx] = cmake<C>(re, im);
}

// e^{ikd} for k = kr + i ki
__device__ __forceinline__ void phase(double kr, double ki, double d, double& pr, double& pi_) {
  double s, c;
  sincos(kr * d, &s, &c);
  double a = (ki != 0.0) ? exp(-ki * d) : 1.0;
  pr = a * c;
  pi_ = a * s;
}

// One thread per column j of a tile; the block sweeps kRowsPerBlock rows.
constexpr int kAsmThreads = 128;
constexpr int kRowsPerBlock = 8;

template <typename C>
__global__ void __launch_bounds__(kAsmThreads) green_far_kernel(
    int n, int npart, const int32_t* __restrict__ pid, const int32_t* __restrict__ blk_mat, KTable kt,
    const double* __restrict__ pos, const double* __restrict__ nvec, const double* __restrict__ area, void* G1,
    void* G2, void* H1, void* H2, long long ld) {
  const int j = blockIdx.x * kAsmThreads + threadIdx.x;
  const int i0 = blockIdx.y * kRowsPerBlock;
  __shared__ double s_pos[kRowsPerBlock][3], s_nv[kRowsPerBlock][3];
  __shared__ int s_pid[kRowsPerBlock];
  if (threadIdx.x < kRowsPerBlock && i0 + threadIdx.x < n) {
    int i = i0 + threadIdx.x;
    for (int c = 0; c < 3; ++c) {
      s_pos[threadIdx.x][c] = pos[3 * i + c];
      s_nv[threadIdx.x][c] = nvec[3 * i + c];
    }
    s_pid[threadIdx.x] = pid[i];
  }
  __syncthreads();
  if (j >= n) return;
  const double3 pj = ld3(pos, j);
  const double aj = area[j];
  const int bj = pid[j];
  const int rows = min(kRowsPerBlock, n - i0);
  for (int r = 0; r < rows; ++r) {
    const int i = i0 + r;
    const int bi = s_pid[r];
    double3 rv = make_double3(s_pos[r][0] - pj.x, s_pos[r][1] - pj.y, s_pos[r][2] - pj.z);
    const bool same_blk = (bi == bj);
    const bool diag = same_blk && (i == j);
    double d = diag ? kEps : fmax(norm3(rv), kEps);
    double ndr = s_nv[r][0] * rv.x + s_nv[r][1] * rv.y + s_nv[r][2] * rv.z;
    const int* bm = blk_mat + (bi * npart + bj) * 4;
    const double inv_d = 1.0 / d;
    const double gpre = aj * inv_d;
    const double fpre = ndr * inv_d * inv_d * aj;
    double out[8];  // G1 re/im, G2, H1, H2
#pragma unroll
    for (int q = 0; q < 8; ++q) out[q] = 0.0;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      int m = bm[t];
      if (m <= 0) continue;
      double kr = kt.re[m - 1], ki = kt.im[m - 1];
      double pr, pim;
      phase(kr, ki, d, pr, pim);
      // G = gpre e^{ikd};  F = fpre (ik - 1/d) e^{ikd},  ik = -ki + i kr
      double gr = gpre * pr, gi = gpre * pim;
      double ar = -ki - inv_d, ai = kr;
      double fr = fpre * (ar * pr - ai * pim), fi = fpre * (ar * pim + ai * pr);
      const double sgn = (t == 0 || t == 2) ? 1.0 : -1.0;
      const int oG = (t < 2) ? 0 : 2;  // G1 (terms 0, 1) or G2 (terms 2, 3)
      const int oH = (t < 2) ? 4 : 6;
      const double two_pi = (t < 2) ? kTwoPi : -kTwoPi;
      out[oG] += sgn * gr;
      out[oG + 1] += sgn * gi;
      out[oH] += sgn * (fr + (diag ? two_pi : 0.0));
      out[oH + 1] += sgn * fi;
    }
    long long idx = (long long)i * ld + j;
    if (G1) store_c<C>(G1, idx, out[0], out[1]);
    if (G2) store_c<C>(G2, idx, out[2], out[3]);
    if (H1) store_c<C>(H1, idx, out[4], out[5]);
    if (H2) store_c<C>(H2, idx, out[6], out[7]);
  }
}

template <typename C>
__global__ void green_refined_kernel(long long nref, const int32_t* __restrict__ ref_row,
                                     const int32_t* __restrict__ ref_col, int order, const double* __restrict__ g,
                                     const double* __restrict__ fn, int npart, const int32_t* __restrict__ pid,
                                     const int32_t* __restrict__ blk_mat, KTable kt, const double* __restrict__ pos,
                                     void* G1, void* G2, void* H1, void* H2, long long ld) {
  long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nref) return;
  const int i = ref_row[e], j = ref_col[e];
  const int bi = pid[i], bj = pid[j];
  const bool diag = (bi == bj) && (i == j);
  double d = diag ? kEps : fmax(norm3(sub3(ld3(pos, i), ld3(pos, j))), kEps);
  const int no = order + 1;
  const int* bm = blk_mat + (bi * npart + bj) * 4;
  double out[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) out[q] = 0.0;
  for (int t = 0; t < 4; ++t) {
    int m = bm[t];
    if (m <= 0) continue;
    double kr = kt.re[m - 1], ki = kt.im[m - 1];
    // sum_m c_m (ik)^m with ik = -ki + i kr
    double pr_ = 1.0, pi_ = 0.0, Gr = 0.0, Gi = 0.0, Fr = 0.0, Fi = 0.0;
    for (int q = 0; q < no; ++q) {
      double gq = g[e * no + q], fq = fn[e * no + q];
      Gr += gq * pr_;
      Gi += gq * pi_;
      Fr += fq * pr_;
      Fi += fq * pi_;
      double nr = pr_ * (-ki) - pi_ * kr;
      double ni = pr_ * kr + pi_ * (-ki);
      pr_ = nr;
      pi_ = ni;
    }
    double ph_r, ph_i;
    phase(kr, ki, d, ph_r, ph_i);
    double gr = Gr * ph_r - Gi * ph_i, gi = Gr * ph_i + Gi * ph_r;
    double fr = Fr * ph_r - Fi * ph_i, fi = Fr * ph_i + Fi * ph_r;
    const double sgn = (t == 0 || t == 2) ? 1.0 : -1.0;
    const int oG = (t < 2) ? 0 : 2;
    const int oH = (t < 2) ? 4 : 6;
    const double two_pi = (t < 2) ? kTwoPi : -kTwoPi;
    out[oG] += sgn * gr;
    out[oG + 1] += sgn * gi;
    out[oH] += sgn * (fr + (diag ? two_pi : 0.0));
    out[oH + 1] += sgn * fi;
  }
  long long idx = (long long)i * ld + j;
  if (G1) store_c<C>(G1, idx, out[0], out[1]);
  if (G2) store_c<C>(G2, idx, out[2], out[3]);
  if (H1) store_c<C>(H1, idx, out[4], out[5]);
  if (H2) store_c<C>(H2, idx, out[6], out[7]);
}

// ----------------------------------------------------------- d/dk of (a6)
// Derivatives of the four BEM matrices with respect to the wavenumber of one
// material `dmat` (1-based): only region terms filled with that material
// contribute (the 2 pi diagonal terms are constant).
//   far:      dG/dk = i d G,   dF/dk = -k d F_pre e^{ikd}  (F_pre = (n.r) area / d^2)
//   refined:  d/dk [sum_m c_m (ik)^m e^{ikd}] = sum_m c_m [i m (ik)^(m-1) + i d (ik)^m] e^{ikd}
template <typename C>
__global__ void __launch_bounds__(kAsmThreads) green_far_dk_kernel(
    int n, int npart, int dmat, const int32_t* __restrict__ pid, const int32_t* __restrict__ blk_mat, KTable kt,
    const double* __restrict__ pos, const double* __restrict__ nvec, const double* __restrict__ area, void* G1,
    void* G2, void* H1, void* H2, long long ld) {
  const int j = blockIdx.x * kAsmThreads + threadIdx.x;
  const int i0 = blockIdx.y * kRowsPerBlock;
  if (j >= n) return;
  const double3 pj = ld3(pos, j);
  const double aj = area[j];
  const int bj = pid[j];
  const int rows = min(kRowsPerBlock, n - i0);
  for (int r = 0; r < rows; ++r) {
    const int i = i0 + r;
    const int bi = pid[i];
    const double3 rv = sub3(ld3(pos, i), pj);
    const bool diag = (bi == bj) && (i == j);
    const double d = diag ? kEps : fmax(norm3(rv), kEps);
    const double ndr = dot3(ld3(nvec, i), rv);
    const int* bm = blk_mat + (bi * npart + bj) * 4;
    const double gpre = aj / d, fpre = ndr / (d * d) * aj;
    double out[8];
#pragma unroll
    for (int q = 0; q < 8; ++q) out[q] = 0.0;
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      if (bm[t] != dmat) continue;
      const double kr = kt.re[dmat - 1], ki = kt.im[dmat - 1];
      double pr, pim;
      phase(kr, ki, d, pr, pim);
      // dG/dk = i d gpre e^{ikd};  dF/dk = -k d fpre e^{ikd}
      const double gr = -d * gpre * pim, gi = d * gpre * pr;
      const double kdr = kr * d * fpre, kdi = ki * d * fpre;  // k d fpre
      const double fr = -(kdr * pr - kdi * pim), fi = -(kdr * pim + kdi * pr);
      const double sgn = (t == 0 || t == 2) ? 1.0 : -1.0;
      const int oG = (t < 2) ? 0 : 2, oH = (t < 2) ? 4 : 6;
      out[oG] += sgn * gr;
      out[oG + 1] += sgn * gi;
      out[oH] += sgn * fr;
      out[oH + 1] += sgn * fi;
    }
    const long long idx = (long long)i * ld + j;
    if (G1) store_c<C>(G1, idx, out[0], out[1]);
    if (G2) store_c<C>(G2, idx, out[2], out[3]);
    if (H1) store_c<C>(H1, idx, out[4], out[5]);
    if (H2) store_c<C>(H2, idx, out[6], out[7]);
  }
}

template <typename C>
__global__ void green_refined_dk_kernel(long long nref, int dmat, const int32_t* __restrict__ ref_row,
                                        const int32_t* __restrict__ ref_col, int order, const double* __restrict__ g,
                                        const double* __restrict__ fn, int npart, const int32_t* __restrict__ pid,
                                        const int32_t* __restrict__ blk_mat, KTable kt, const double* __restrict__ pos,
                                        void* G1, void* G2, void* H1, void* H2, long long ld) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nref) return;
  const int i = ref_row[e], j = ref_col[e];
  const int bi = pid[i], bj = pid[j];
  const bool diag = (bi == bj) && (i == j);
  const double d = diag ? kEps : fmax(norm3(sub3(ld3(pos, i), ld3(pos, j))), kEps);
  const int no = order + 1;
  const int* bm = blk_mat + (bi * npart + bj) * 4;
  double out[8];
#pragma unroll
  for (int q = 0; q < 8; ++q) out[q] = 0.0;
  for (int t = 0; t < 4; ++t) {
    if (bm[t] != dmat) continue;
    const double kr = kt.re[dmat - 1], ki = kt.im[dmat - 1];
    // S = sum c_m (ik)^m,  S' = sum c_m m (ik)^(m-1)   (ik = -ki + i kr)
    double pr_ = 1.0, pi_ = 0.0, qr = 0.0, qi = 0.0;  // (ik)^m and (ik)^(m-1)
    double Gr = 0, Gi = 0, Fr = 0, Fi = 0, dGr = 0, dGi = 0, dFr = 0, dFi = 0;
    for (int q = 0; q < no; ++q) {
      const double gq = g[e * no + q], fq = fn[e * no + q];
      Gr += gq * pr_;
      Gi += gq * pi_;
      Fr += fq * pr_;
      Fi += fq * pi_;
      dGr += gq * q * qr;
      dGi += gq * q * qi;
      dFr += fq * q * qr;
      dFi += fq * q * qi;
      qr = pr_;
      qi = pi_;
      const double nr = pr_ * (-ki) - pi_ * kr, ni = pr_ * kr + pi_ * (-ki);
      pr_ = nr;
      pi_ = ni;
    }
    // d/dk = i [S' + d S] e^{ikd}
    double ph_r, ph_i;
    phase(kr, ki, d, ph_r, ph_i);
    const double sgr = dGr + d * Gr, sgi = dGi + d * Gi;
    const double sfr = dFr + d * Fr, sfi = dFi + d * Fi;
    const double igr = -sgi, igi = sgr, ifr = -sfi, ifi = sfr;  // multiply by i
    const double gr = igr * ph_r - igi * ph_i, gi = igr * ph_i + igi * ph_r;
    const double fr = ifr * ph_r - ifi * ph_i, fi = ifr * ph_i + ifi * ph_r;
    const double sgn = (t == 0 || t == 2) ? 1.0 : -1.0;
    const int oG = (t < 2) ? 0 : 2, oH = (t < 2) ? 4 : 6;
    out[oG] += sgn * gr;
    out[oG + 1] += sgn * gi;
    out[oH] += sgn * fr;
    out[oH + 1] += sgn * fi;
  }
  const long long idx = (long long)i * ld + j;
  if (G1) store_c<C>(G1, idx, out[0], out[1]);
  if (G2) store_c<C>(G2, idx, out[2], out[3]);
  if (H1) store_c<C>(H1, idx, out[4], out[5]);
  if (H2) store_c<C>(H2, idx, out[6], out[7]);
}

}  // namespace bem200

using namespace bem200;

extern "C" {

int bem200_version(void) { return 100; }

uint64_t bem200_launch_count(void) { return (uint64_t)launch_count(); }

int bem200_last_error(char* buf, size_t len) {
  const char* m = get_error();
  size_t l = strlen(m);
  if (buf && len > 0) {
    size_t c = l < len - 1 ? l : len - 1;
    memcpy(buf, m, c);
    buf[c] = 0;
  }
  return (int)l;
}

int bem200_refine_count(int n, const double* pos, const double* rad, double abs_cutoff, double rel_cutoff,
                        int32_t* row_count, void* stream) {
  BEM_REQUIRE(n > 0 && pos && rad && row_count, BEM200_ERR_ARG, "refine_count: bad arguments");
  int threads = 256;
  refine_classify_kernel<<<ceil_div((long long)n * 32, threads), threads, 0, (cudaStream_t)stream>>>(
      n, pos, rad, abs_cutoff, rel_cutoff, row_count, nullptr, nullptr, nullptr, nullptr);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

int bem200_scan_i32(int n, const int32_t* count, int64_t* row_ptr, void* stream) {
  BEM_REQUIRE(n > 0 && count && row_ptr, BEM200_ERR_ARG, "scan_i32: bad arguments");
  scan_kernel<<<1, 1024, 0, (cudaStream_t)stream>>>(n, count, row_ptr);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

int bem200_refine_fill(int n, const double* pos, const double* rad, double abs_cutoff, double rel_cutoff,
                       const int64_t* row_ptr, int32_t* ref_row, int32_t* ref_col, int8_t* ref_kind,
                       void* stream) {
  BEM_REQUIRE(n > 0 && pos && rad && row_ptr && ref_row && ref_col && ref_kind, BEM200_ERR_ARG,
              "refine_fill: bad arguments");
  int threads = 256;
  refine_classify_kernel<<<ceil_div((long long)n * 32, threads), threads, 0, (cudaStream_t)stream>>>(
      n, pos, rad, abs_cutoff, rel_cutoff, nullptr, row_ptr, ref_row, ref_col, ref_kind);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

int bem200_refine_integrals(int64_t nref, const int32_t* ref_row, const int32_t* ref_col, const int8_t* ref_kind,
                            const double* pos, const double* nvec, const double* tvec1, const double* tvec2,
                            const double* area, const double* nodes, const int32_t* face_kind, const double* rules,
                            int n28, int n3, int n4, int order, double* g, double* f, void* stream) {
  BEM_REQUIRE(nref >= 0 && order >= 0 && order <= kMaxOrder, BEM200_ERR_ARG,
              "refine_integrals: order must be in [0, %d]", kMaxOrder);
  BEM_REQUIRE(n28 > 0 && n3 > 0 && n4 > 0, BEM200_ERR_ARG, "refine_integrals: empty quadrature rule");
  if (nref == 0) return BEM200_OK;
  BEM_REQUIRE(ref_row && ref_col && ref_kind && pos && nvec && tvec1 && tvec2 && area && nodes && face_kind &&
                  rules && g && f,
              BEM200_ERR_ARG, "refine_integrals: null pointer");
  int threads = 256;
  refine_integrals_kernel<<<ceil_div(nref * 32, threads), threads, 0, (cudaStream_t)stream>>>(
      nref, ref_row, ref_col, ref_kind, pos, nvec, tvec1, tvec2, area, nodes, face_kind, rules, n28, n3, n4,
      order, g, f);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

int bem200_closed_correction(int n, int npart, const int32_t* pid, const uint64_t* closed_mask, const double* pos,
                             const double* nvec, const double* area, int64_t nref, const int64_t* row_ptr,
                             const int32_t* ref_row, const int32_t* ref_col, const int8_t* ref_kind, int order,
                             double* f, double* corr, void* stream) {
  (void)row_ptr;
  BEM_REQUIRE(n > 0 && npart > 0 && npart <= 64, BEM200_ERR_ARG,
              "closed_correction: need 1 <= npart <= 64 (got %d)", npart);
  BEM_REQUIRE(pid && closed_mask && pos && nvec && area && corr, BEM200_ERR_ARG, "closed_correction: null pointer");
  cudaStream_t s = (cudaStream_t)stream;
  // corr doubles as the column-sum buffer S before it receives c_j
  closed_colsum_kernel<<<ceil_div((long long)n * 32, 256), 256, 0, s>>>(n, pid, closed_mask, pos, nvec, area, corr);
  BEM_LAUNCH_CHECK();
  if (nref > 0) {
    closed_adjust_kernel<<<ceil_div(nref, 256), 256, 0, s>>>(nref, ref_row, ref_col, pid, closed_mask, pos, nvec,
                                                            area, order, f, corr);
    BEM_LAUNCH_CHECK();
    closed_apply_kernel<<<ceil_div(nref, 256), 256, 0, s>>>(nref, ref_row, ref_col, ref_kind, pid, closed_mask,
                                                           nvec, area, order, corr, f, corr);
    BEM_LAUNCH_CHECK();
  }
  return BEM200_OK;
}

int bem200_refine_project(int64_t nref, const int32_t* ref_row, const double* nvec, int order, const double* f,
                          double* fn, void* stream) {
  if (nref == 0) return BEM200_OK;
  BEM_REQUIRE(ref_row && nvec && f && fn && order >= 0 && order <= kMaxOrder, BEM200_ERR_ARG,
              "refine_project: bad arguments");
  refine_project_kernel<<<ceil_div(nref, 256), 256, 0, (cudaStream_t)stream>>>(nref, ref_row, nvec, order, f, fn);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

int bem200_green_assemble(int n, int npart, const int32_t* pid, const int32_t* blk_mat, int nmat,
                          const double* kmat_host, const double* pos, const double* nvec, const double* area,
                          int64_t nref, const int32_t* ref_row, const int32_t* ref_col, int order, const double* g,
                          const double* fn, int out_dtype, void* G1, void* G2, void* H1, void* H2, int64_t ld,
                          void* stream) {
  BEM_REQUIRE(n > 0 && npart > 0 && ld >= n, BEM200_ERR_ARG, "green_assemble: bad sizes");
  BEM_REQUIRE(nmat > 0 && nmat <= kMaxMat && kmat_host, BEM200_ERR_ARG, "green_assemble: need 1..%d materials",
              kMaxMat);
  BEM_REQUIRE(out_dtype == BEM200_C128 || out_dtype == BEM200_C64, BEM200_ERR_ARG, "green_assemble: bad dtype");
  BEM_REQUIRE(pid && blk_mat && pos && nvec && area, BEM200_ERR_ARG, "green_assemble: null pointer");
  BEM_REQUIRE(order >= 0 && order <= kMaxOrder, BEM200_ERR_ARG, "green_assemble: bad order");
  KTable kt;
  for (int m = 0; m < kMaxMat; ++m) {
    kt.re[m] = m < nmat ? kmat_host[2 * m] : 0.0;
    kt.im[m] = m < nmat ? kmat_host[2 * m + 1] : 0.0;
  }
  cudaStream_t s = (cudaStream_t)stream;
  dim3 grid(ceil_div(n, kAsmThreads), ceil_div(n, kRowsPerBlock));
  BEM_REQUIRE(grid.y <= 65535, BEM200_ERR_ARG, "green_assemble: n too large");
  if (out_dtype == BEM200_C128)
    green_far_kernel<double2><<<grid, kAsmThreads, 0, s>>>(n, npart, pid, blk_mat, kt, pos, nvec, area, G1, G2, H1,
                                                            H2, ld);
  else
    green_far_kernel<float2><<<grid, kAsmThreads, 0, s>>>(n, npart, pid, blk_mat, kt, pos, nvec, area, G1, G2, H1,
                                                           H2, ld);
  BEM_LAUNCH_CHECK();
  if (nref > 0) {
    BEM_REQUIRE(ref_row && ref_col && g && fn, BEM200_ERR_ARG, "green_assemble: null refinement arrays");
    if (out_dtype == BEM200_C128)
      green_refined_kernel<double2><<<ceil_div(nref, 256), 256, 0, s>>>(nref, ref_row, ref_col, order, g, fn, npart,
                                                                         pid, blk_mat, kt, pos, G1, G2, H1, H2, ld);
    else
      green_refined_kernel<float2><<<ceil_div(nref, 256), 256, 0, s>>>(nref, ref_row, ref_col, order, g, fn, npart,
                                                                        pid, blk_mat, kt, pos, G1, G2, H1, H2, ld);
    BEM_LAUNCH_CHECK();
  }
  return BEM200_OK;
}

int bem200_green_assemble_dk(int n, int npart, const int32_t* pid, const int32_t* blk_mat, int nmat,
                             const double* kmat_host, int dmat, const double* pos, const double* nvec,
                             const double* area, int64_t nref, const int32_t* ref_row, const int32_t* ref_col,
                             int order, const double* g, const double* fn, void* G1, void* G2, void* H1, void* H2,
                             int64_t ld, void* stream) {
  BEM_REQUIRE(n > 0 && npart > 0 && ld >= n && nmat > 0 && nmat <= kMaxMat && kmat_host && dmat >= 1 &&
                  dmat <= nmat && pid && blk_mat && pos && nvec && area && order >= 0 && order <= kMaxOrder,
              BEM200_ERR_ARG, "green_assemble_dk: bad arguments");
  KTable kt;
  for (int m = 0; m < kMaxMat; ++m) {
    kt.re[m] = m < nmat ? kmat_host[2 * m] : 0.0;
    kt.im[m] = m < nmat ? kmat_host[2 * m + 1] : 0.0;
  }
  cudaStream_t s = (cudaStream_t)stream;
  dim3 grid(ceil_div(n, kAsmThreads), ceil_div(n, kRowsPerBlock));
  BEM_REQUIRE(grid.y <= 65535, BEM200_ERR_ARG, "green_assemble_dk: n too large");
  green_far_dk_kernel<double2><<<grid, kAsmThreads, 0, s>>>(n, npart, dmat, pid, blk_mat, kt, pos, nvec, area, G1, G2,
                                                             H1, H2, ld);
  BEM_LAUNCH_CHECK();
  if (nref > 0) {
    BEM_REQUIRE(ref_row && ref_col && g && fn, BEM200_ERR_ARG, "green_assemble_dk: null refinement arrays");
    green_refined_dk_kernel<double2><<<ceil_div(nref, 256), 256, 0, s>>>(nref, dmat, ref_row, ref_col, order, g, fn,
                                                                          npart, pid, blk_mat, kt, pos, G1, G2, H1,
                                                                          H2, ld);
    BEM_LAUNCH_CHECK();
  }
  return BEM200_OK;
}

}  // extern "C"
