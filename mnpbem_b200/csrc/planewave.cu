// Plane-wave excitation and far fields on the GPU (complex128).
//
//   bem200_planewave_rhs : the BEM right-hand side b = [phi | a | alpha | De]
//                          of a plane wave, i.e. PlaneWaveRet.potential
//                          (mnpbem/simulation/planewave_ret.py:257-361) fused
//                          with BEMRet._excitation (mnpbem/bem/bem_ret.py:1360-1429)
//   bem200_farfield      : far-field amplitudes e, h on a set of directions
//                          from the surface charges and currents
//                          (mnpbem/spectrum/spectrum_ret.py:231-392)
#include "common.cuh"

namespace bem200 {

struct PolDir {
  double pol[8][3];
  double dir[8][3];
};

__device__ __forceinline__ double2 cexp_i(double2 z) {  // exp(i z)
  double s, c;
  sincos(z.x, &s, &c);
  const double a = exp(-z.y);
  return make_double2(a * c, a * s);
}

// one thread per (face, polarisation)
__global__ void planewave_rhs_kernel(int n, int p, const double* __restrict__ pos, const double* __restrict__ nvec,
                                     const int8_t* __restrict__ on_side, PolDir pd, double2 km, double k0,
                                     int eps_per_face, double2 e1s, double2 e2s, const double2* __restrict__ e1v,
                                     const double2* __restrict__ e2v, double2* __restrict__ b) {
  const long long idx = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  const long long np = (long long)n * p;
  if (idx >= np) return;
  const int i = (int)(idx / p), q = (int)(idx % p);
  const double* d = pd.dir[q];
  const double* e = pd.pol[q];
  const double3 r = make_double3(pos[3 * i], pos[3 * i + 1], pos[3 * i + 2]);
  const double3 nv = make_double3(nvec[3 * i], nvec[3 * i + 1], nvec[3 * i + 2]);
  const double rd = r.x * d[0] + r.y * d[1] + r.z * d[2];
  const double nd = nv.x * d[0] + nv.y * d[1] + nv.z * d[2];
  // ph = exp(i km r.d) / (i k0);  a = ph pol;  ap = i km (n.d) ph pol
  double2 ph = cexp_i(cscale(km, rd));
  ph = make_double2(ph.y / k0, -ph.x / k0);
  const double2 ikm_nd = make_double2(-km.y * nd, km.x * nd);
  const double2 php = cmul(ikm_nd, ph);
  const bool s1 = on_side[2 * i] != 0, s2 = on_side[2 * i + 1] != 0;
  const double2 e1 = eps_per_face ? e1v[i] : e1s, e2 = eps_per_face ? e2v[i] : e2s;
  const double ne = nv.x * e[0] + nv.y * e[1] + nv.z * e[2];
  double2* phi = b;
  double2* a = b + np;
  double2* alpha = b + 4 * np;
  double2* De = b + 7 * np;
  phi[idx] = make_double2(0, 0);
  const double f2 = s2 ? 1.0 : 0.0, f1 = s1 ? 1.0 : 0.0;
  for (int c = 0; c < 3; ++c) {
    const long long ai = ((long long)i * 3 + c) * p + q;
    a[ai] = cscale(ph, (f2 - f1) * e[c]);       // a2 - a1
    alpha[ai] = cscale(php, (f2 - f1) * e[c]);  // a2p - a1p (phi = 0 for a plane wave)
  }
  // De = -i k0 (e2 n.a2 - e1 n.a1)
  const double2 t = csub(cscale(cmul(e2, ph), f2 * ne), cscale(cmul(e1, ph), f1 * ne));
  De[idx] = make_double2(k0 * t.y, -k0 * t.x);
}

constexpr int kFFThreads = 256;
constexpr int kFFMaxPol = 4;

// One CTA per direction: A = sum_j phase_j h_j, S = sum_j phase_j s_j over the
// faces whose side towards the embedding medium is selected, phase_j =
// exp(-i km d.r_j) area_j; then e = i k0 A - i km d S, h = i km d x A.
__global__ void __launch_bounds__(kFFThreads) farfield_kernel(int n, int p, const double* __restrict__ dirs,
                                                             const double* __restrict__ pos,
                                                             const double* __restrict__ area,
                                                             const int8_t* __restrict__ on_side, double2 km, double k0,
                                                             const double2* __restrict__ W1,
                                                             const double2* __restrict__ W2, double2* __restrict__ e_out,
                                                             double2* __restrict__ h_out) {
  __shared__ double2 red[kFFThreads / 32][4 * kFFMaxPol];
  const int dI = blockIdx.x;
  const double d0 = dirs[3 * dI], d1 = dirs[3 * dI + 1], d2 = dirs[3 * dI + 2];
  double2 acc[4 * kFFMaxPol];
#pragma unroll
  for (int u = 0; u < 4 * kFFMaxPol; ++u) acc[u] = make_double2(0, 0);
  const int w4 = 4 * p;
  for (int j = threadIdx.x; j < n; j += kFFThreads) {
    const double rd = pos[3 * j] * d0 + pos[3 * j + 1] * d1 + pos[3 * j + 2] * d2;
    const double2 ph = cscale(cexp_i(cscale(km, -rd)), area[j]);
    for (int side = 0; side < 2; ++side) {
      if (!on_side[2 * j + side]) continue;
      const double2* W = (side == 0 ? W1 : W2) + (long long)j * w4;
#pragma unroll
      for (int q = 0; q < kFFMaxPol; ++q) {
        if (q >= p) break;
        acc[4 * q] = cadd(acc[4 * q], cmul(ph, W[q]));  // sigma
#pragma unroll
        for (int c = 0; c < 3; ++c)
          acc[4 * q + 1 + c] = cadd(acc[4 * q + 1 + c], cmul(ph, W[p + c * p + q]));  // h
      }
    }
  }
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
#pragma unroll
  for (int u = 0; u < 4 * kFFMaxPol; ++u) {
    double2 v = acc[u];
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
      v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    if (lane == 0) red[wid][u] = v;
  }
  __syncthreads();
  if (threadIdx.x < p) {
    const int q = threadIdx.x;
    double2 S = make_double2(0, 0), A[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
    for (int w = 0; w < kFFThreads / 32; ++w) {
      S = cadd(S, red[w][4 * q]);
      for (int c = 0; c < 3; ++c) A[c] = cadd(A[c], red[w][4 * q + 1 + c]);
    }
    const double dd[3] = {d0, d1, d2};
    const double2 ik0 = make_double2(0, k0), ikm = make_double2(-km.y, km.x);
    for (int c = 0; c < 3; ++c) {
      const double2 ev = csub(cmul(ik0, A[c]), cscale(cmul(ikm, S), dd[c]));
      e_out[((long long)dI * 3 + c) * p + q] = ev;
    }
    // d x A
    const double2 cx = csub(cscale(A[2], d1), cscale(A[1], d2));
    const double2 cy = csub(cscale(A[0], d2), cscale(A[2], d0));
    const double2 cz = csub(cscale(A[1], d0), cscale(A[0], d1));
    h_out[((long long)dI * 3 + 0) * p + q] = cmul(ikm, cx);
    h_out[((long long)dI * 3 + 1) * p + q] = cmul(ikm, cy);
    h_out[((long long)dI * 3 + 2) * p + q] = cmul(ikm, cz);
  }
}

}  // namespace bem200

using namespace bem200;

extern "C" {

int bem200_planewave_rhs(int n, int npol, const double* pos, const double* nvec, const int8_t* on_side,
                         const double* pol_host, const double* dir_host, const double* km_host, double k0,
                         int eps_per_face, const double* eps1, const double* eps2, void* b, void* stream) {
  BEM_REQUIRE(n > 0 && npol > 0 && npol <= 8 && pos && nvec && on_side && pol_host && dir_host && km_host && eps1 &&
                  eps2 && b && k0 > 0,
              BEM200_ERR_ARG, "planewave_rhs: bad arguments (1 <= npol <= 8)");
  PolDir pd;
  for (int q = 0; q < npol; ++q)
    for (int c = 0; c < 3; ++c) {
      pd.pol[q][c] = pol_host[3 * q + c];
      pd.dir[q][c] = dir_host[3 * q + c];
    }
  const double2 km = make_double2(km_host[0], km_host[1]);
  double2 e1s = make_double2(0, 0), e2s = make_double2(0, 0);
  const double2 *e1v = nullptr, *e2v = nullptr;
  if (eps_per_face) {
    e1v = (const double2*)eps1;
    e2v = (const double2*)eps2;
  } else {
    e1s = make_double2(eps1[0], eps1[1]);
    e2s = make_double2(eps2[0], eps2[1]);
  }
  const long long np = (long long)n * npol;
  planewave_rhs_kernel<<<ceil_div(np, 256), 256, 0, (cudaStream_t)stream>>>(
      n, npol, pos, nvec, on_side, pd, km, k0, eps_per_face, e1s, e2s, e1v, e2v, (double2*)b);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

int bem200_farfield(int n, int npol, int ndir, const double* dirs, const double* pos, const double* area,
                    const int8_t* on_side, const double* km_host, double k0, const void* W1, const void* W2,
                    void* e_out, void* h_out, void* stream) {
  BEM_REQUIRE(n > 0 && npol > 0 && npol <= kFFMaxPol && ndir > 0 && dirs && pos && area && on_side && km_host &&
                  W1 && W2 && e_out && h_out,
              BEM200_ERR_ARG, "farfield: bad arguments (1 <= npol <= %d)", kFFMaxPol);
  farfield_kernel<<<ndir, kFFThreads, 0, (cudaStream_t)stream>>>(n, npol, dirs, pos, area, on_side,
                                                                 make_double2(km_host[0], km_host[1]), k0,
                                                                 (const double2*)W1, (const double2*)W2,
                                                                 (double2*)e_out, (double2*)h_out);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

}  // extern "C"
