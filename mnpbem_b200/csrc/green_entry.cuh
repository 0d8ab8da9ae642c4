// One entry of the BEM matrices G1, G2, H1, H2 evaluated from the face
// geometry and the near-field refinement tables, for kernels that need
// matrix entries on demand instead of a stored matrix (the H-matrix fill and
// its adaptive cross approximation).  The arithmetic is that of the assembly
// kernels in green.cu (green_far_kernel for far pairs, green_refined_kernel
// for refined pairs), term by term in the same order.
//
// Reference behaviour followed (MNPBEM Python port v1.6.2):
//   eval (G, F, H1, H2)   mnpbem/greenfun/greenret_refined.py:654-810
//   region connectivity   mnpbem/greenfun/compgreen_ret.py:435-505, :739-858
//   on-demand rows/cols   mex/acagreen/acagreen.cpp:83-149 (greenret getrow/getcol)
#pragma once

#include "common.cuh"

namespace bem200 {
namespace ge {

constexpr int kMaxMat = 16;
constexpr int kMaxOrder = 7;
constexpr double kEps = 2.220446049250313e-16;  // numpy finfo(float).eps
constexpr double kTwoPi = 6.283185307179586;

// e^{ikd} for k = kr + i ki
__device__ __forceinline__ void phase(double kr, double ki, double d, double& pr, double& pi_) {
  double s, c;
  sincos(kr * d, &s, &c);
  double a = (ki != 0.0) ? exp(-ki * d) : 1.0;
  pr = a * c;
  pi_ = a * s;
}

// Matrix `which` (0 = G1, 1 = G2, 2 = H1, 3 = H2) of a compound particle:
// region terms t = 0, 1 (G1, H1) or 2, 3 (G2, H2) of blk_mat, wavenumbers
// k[m - 1] of the materials m filling them.  Refined pairs (i, j) are found
// in the CSR tables (row_ptr, ref_col sorted by column within each row).
// Indices given to operator() are in cluster order when c2p is set.
struct GreenSource {
  int n, npart, which, order;
  const int32_t* pid;
  const int32_t* blk_mat;
  const double* pos;
  const double* nvec;
  const double* area;
  const int64_t* row_ptr;
  const int32_t* ref_col;
  const double* g;
  const double* fn;
  const int32_t* c2p;
  double kre[kMaxMat], kim[kMaxMat];

  __device__ __forceinline__ long long find_ref(int i, int j) const {
    long long lo = row_ptr[i], hi = row_ptr[i + 1];
    const long long end = hi;
    while (lo < hi) {
      const long long mid = (lo + hi) >> 1;
      if (ref_col[mid] < j)
        lo = mid + 1;
      else
        hi = mid;
    }
    return (lo < end && ref_col[lo] == j) ? lo : -1;
  }

  __device__ double2 entry(int i, int j) const {
    const int bi = pid[i], bj = pid[j];
    const bool diag = (bi == bj) && (i == j);
    const double rx = pos[3 * i] - pos[3 * j], ry = pos[3 * i + 1] - pos[3 * j + 1],
                 rz = pos[3 * i + 2] - pos[3 * j + 2];
    const double d = diag ? kEps : fmax(sqrt(rx * rx + ry * ry + rz * rz), kEps);
    const int* bm = blk_mat + (bi * npart + bj) * 4;
    const bool isH = which >= 2;
    const int t0 = (which == 0 || which == 2) ? 0 : 2;
    const long long e = row_ptr ? find_ref(i, j) : -1;
    double re = 0.0, im = 0.0;
    for (int t = t0; t < t0 + 2; ++t) {
      const int m = bm[t];
      if (m <= 0) continue;
      const double kr = kre[m - 1], ki = kim[m - 1];
      double vr, vi;
      if (e < 0) {
        const double ndr = nvec[3 * i] * rx + nvec[3 * i + 1] * ry + nvec[3 * i + 2] * rz;
        const double inv_d = 1.0 / d;
        const double aj = area[j];
        double pr, pim;
        phase(kr, ki, d, pr, pim);
        if (!isH) {
          const double gpre = aj * inv_d;
          vr = gpre * pr;
          vi = gpre * pim;
        } else {
          // F = fpre (ik - 1/d) e^{ikd},  ik = -ki + i kr
          const double fpre = ndr * inv_d * inv_d * aj;
          const double ar = -ki - inv_d, ai = kr;
          vr = fpre * (ar * pr - ai * pim);
          vi = fpre * (ar * pim + ai * pr);
        }
      } else {
        // sum_q c_q (ik)^q, then the phase e^{ikd}
        const double* c = (isH ? fn : g) + e * (order + 1);
        double pr_ = 1.0, pi_ = 0.0, Sr = 0.0, Si = 0.0;
        for (int q = 0; q <= order; ++q) {
          Sr += c[q] * pr_;
          Si += c[q] * pi_;
          const double nr = pr_ * (-ki) - pi_ * kr;
          const double ni = pr_ * kr + pi_ * (-ki);
          pr_ = nr;
          pi_ = ni;
        }
        double ph_r, ph_i;
        phase(kr, ki, d, ph_r, ph_i);
        vr = Sr * ph_r - Si * ph_i;
        vi = Sr * ph_i + Si * ph_r;
      }
      const double sgn = (t == 0 || t == 2) ? 1.0 : -1.0;
      if (isH) {
        const double two_pi = (t < 2) ? kTwoPi : -kTwoPi;
        re += sgn * (vr + (diag ? two_pi : 0.0));
      } else {
        re += sgn * vr;
      }
      im += sgn * vi;
    }
    return make_double2(re, im);
  }

  __device__ __forceinline__ double2 operator()(int ci, int cj) const {
    return c2p ? entry(c2p[ci], c2p[cj]) : entry(ci, cj);
  }
};

}  // namespace ge
}  // namespace bem200
