// Potentials and fields of a BEM solution at the faces, and the Cartesian
// derivatives of the retarded Green function.
//
// Reference behaviour followed (MNPBEM Python port v1.6.2):
//   GreenRetRefined.eval 'Gp', 'H1p', 'H2p'   mnpbem/greenfun/greenret_refined.py:812-864
//   CompGreenRet._eval1 (Gp keys, blocks)      mnpbem/greenfun/compgreen_ret.py:811-858
//   CompGreenRet.potential                     mnpbem/greenfun/compgreen_ret.py:976-1038
//   CompGreenRet.field                         mnpbem/greenfun/compgreen_ret.py:912-974
//   BEMRet.potential / BEMRet.field            mnpbem/bem/bem_ret.py:1833-1895
//
// For face pair (i, j) with r = pos_i - pos_j, d = |r| (eps on the diagonal)
// and the wavenumber k of the material that fills the region pair:
//   G      = area_j / d e^{ikd}
//   Gp_c   = r_c (ik - 1/d) / d^2 area_j e^{ikd}        (c = x, y, z)
//   refined pairs: G = sum_q g_q (ik)^q e^{ikd}, Gp_c = sum_q f_{c,q} (ik)^q e^{ikd}
//   H1p / H2p = Gp +/- 2 pi n_i on the diagonal of self blocks; H = n_i . Hp.
//
// Two kinds of kernels:
//   * assembly of Gp / H1p / H2p as an (n, 3, n) complex128 array (one thread
//     per column, 8 rows per CTA; refined entries overwritten by a second
//     kernel), the layout of the reference's (n1, 3, n2) arrays;
//   * the potential / field products computed without storing any n x n
//     matrix: one warp per row i sweeps the columns, evaluates G and Gp of
//     both region terms in registers and accumulates the products with the
//     surface charges and currents.  Columns of refined pairs are skipped in
//     that sweep (a per-warp bitmap in shared memory built from the row's
//     refinement list) and added from the refinement coefficients afterwards.
#include "green_entry.cuh"

namespace bem200 {
namespace fld {

using ge::kEps;
using ge::kMaxMat;
using ge::kTwoPi;
using ge::phase;

struct KTab {
  double re[kMaxMat], im[kMaxMat];
};

__device__ __forceinline__ double2 cm(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}

// ------------------------------------------------------- Gp / H1p / H2p
constexpr int kCartThreads = 128;
constexpr int kCartRows = 8;

__global__ void __launch_bounds__(kCartThreads) green_cart_far_kernel(
    int n, int npart, const int32_t* __restrict__ pid, const int32_t* __restrict__ blk, KTab kt,
    const double* __restrict__ pos, const double* __restrict__ nvec, const double* __restrict__ area, double hsign,
    double2* __restrict__ out) {
  const int j = blockIdx.x * kCartThreads + threadIdx.x;
  const int i0 = blockIdx.y * kCartRows;
  if (j >= n) return;
  const double pjx = pos[3 * j], pjy = pos[3 * j + 1], pjz = pos[3 * j + 2];
  const double aj = area[j];
  const int bj = pid[j];
  const int rows = min(kCartRows, n - i0);
  for (int r = 0; r < rows; ++r) {
    const int i = i0 + r;
    const int bi = pid[i];
    const int m = blk[bi * npart + bj];
    double2 v[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
    if (m > 0) {
      const double rx = pos[3 * i] - pjx, ry = pos[3 * i + 1] - pjy, rz = pos[3 * i + 2] - pjz;
      const bool diag = (bi == bj) && (i == j);
      const double d = diag ? kEps : fmax(sqrt(rx * rx + ry * ry + rz * rz), kEps);
      const double inv_d = 1.0 / d;
      const double kr = kt.re[m - 1], ki = kt.im[m - 1];
      double pr, pim;
      phase(kr, ki, d, pr, pim);
      const double fpre = inv_d * inv_d * aj;
      const double ar = -ki - inv_d, ai = kr;  // ik - 1/d
      const double cr = fpre * (ar * pr - ai * pim), ci = fpre * (ar * pim + ai * pr);
      v[0] = make_double2(rx * cr, rx * ci);
      v[1] = make_double2(ry * cr, ry * ci);
      v[2] = make_double2(rz * cr, rz * ci);
      if (diag)
        for (int c = 0; c < 3; ++c) v[c].x += hsign * kTwoPi * nvec[3 * i + c];
    }
    for (int c = 0; c < 3; ++c) out[((long long)i * 3 + c) * n + j] = v[c];
  }
}

__global__ void green_cart_refined_kernel(long long nref, const int32_t* __restrict__ ref_row,
                                          const int32_t* __restrict__ ref_col, int order,
                                          const double* __restrict__ f, int npart, const int32_t* __restrict__ pid,
                                          const int32_t* __restrict__ blk, KTab kt, const double* __restrict__ pos,
                                          const double* __restrict__ nvec, double hsign, int n,
                                          double2* __restrict__ out) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= nref) return;
  const int i = ref_row[e], j = ref_col[e];
  const int bi = pid[i], bj = pid[j];
  const int m = blk[bi * npart + bj];
  if (m <= 0) return;  // the far kernel wrote the zero of an unconnected block
  const bool diag = (bi == bj) && (i == j);
  const double rx = pos[3 * i] - pos[3 * j], ry = pos[3 * i + 1] - pos[3 * j + 1], rz = pos[3 * i + 2] - pos[3 * j + 2];
  const double d = diag ? kEps : fmax(sqrt(rx * rx + ry * ry + rz * rz), kEps);
  const double kr = kt.re[m - 1], ki = kt.im[m - 1];
  const int no = order + 1;
  double Sr[3] = {0, 0, 0}, Si[3] = {0, 0, 0};
  double pr_ = 1.0, pi_ = 0.0;  // (ik)^q, ik = -ki + i kr
  for (int q = 0; q < no; ++q) {
    for (int c = 0; c < 3; ++c) {
      const double fc = f[(e * 3 + c) * no + q];
      Sr[c] += fc * pr_;
      Si[c] += fc * pi_;
    }
    const double nr = pr_ * (-ki) - pi_ * kr, ni = pr_ * kr + pi_ * (-ki);
    pr_ = nr;
    pi_ = ni;
  }
  double ph_r, ph_i;
  phase(kr, ki, d, ph_r, ph_i);
  for (int c = 0; c < 3; ++c) {
    double vr = Sr[c] * ph_r - Si[c] * ph_i, vi = Sr[c] * ph_i + Si[c] * ph_r;
    if (diag) vr += hsign * kTwoPi * nvec[3 * i + c];
    out[((long long)i * 3 + c) * n + j] = make_double2(vr, vi);
  }
}

// ------------------------------------------------- potential and field
// One warp per row.  P polarisations per launch (columns q0 .. q0 + P of the
// np-wide inputs).  kField = false: potential (phi, phip, a, ap);
// kField = true: field (e, h).
constexpr int kApplyWarps = 4;
constexpr int kApplyThreads = 32 * kApplyWarps;

struct ApplyArgs {
  int n, npart, order, np, q0;
  KTab kt;
  const int32_t* pid;
  const int32_t* blk[2];  // region pair (r, 0) acts on sig1 / h1, (r, 1) on sig2 / h2
  const double* pos;
  const double* nvec;
  const double* area;
  const int64_t* row_ptr;  // refinement tables in CSR form (NULL: no refined pairs)
  const int32_t* ref_col;
  const double* g;         // (nref, order + 1)
  const double* fc;        // potential: fn (nref, order + 1); field: f (nref, 3, order + 1)
  double hsign;            // +1: H1 / H1p, -1: H2 / H2p
  double k0;               // vacuum wavenumber (field: e = i k0 A - grad phi)
  const double2* sig[2];   // (n, np)
  const double2* h[2];     // (n, 3, np)
  double2* out[4];         // potential: phi (n, np), phip, a (n, 3, np), ap; field: e (n, 3, np), h
};

template <int P, bool kField>
struct Acc {
  // potential: s[0][q] = phi, s[1][q] = phip, v[0][c][q] = a, v[1][c][q] = ap
  // field:     v[0][c][q] = e, v[1][c][q] = h
  double2 s[kField ? 1 : 2][P];
  double2 v[2][3][P];
  __device__ __forceinline__ void zero() {
#pragma unroll
    for (int a = 0; a < (kField ? 1 : 2); ++a)
#pragma unroll
      for (int q = 0; q < P; ++q) s[a][q] = make_double2(0, 0);
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int c = 0; c < 3; ++c)
#pragma unroll
        for (int q = 0; q < P; ++q) v[a][c][q] = make_double2(0, 0);
  }
};

// add the contribution of one (i, j, term): Green value G, surface derivative
// H (potential) or derivative vector Hp (field), diagonal 2 pi terms included
template <int P, bool kField>
__device__ __forceinline__ void accumulate(Acc<P, kField>& acc, const ApplyArgs& A, int t, int j, double2 G,
                                           double2 H, const double2 (&Gp)[3]) {
  const double2* sg = A.sig[t] + (long long)j * A.np + A.q0;
  const double2* hh = A.h[t] + (long long)j * 3 * A.np + A.q0;
  if (!kField) {
#pragma unroll
    for (int q = 0; q < P; ++q) {
      const double2 s = __ldg(sg + q);
      acc.s[0][q] = cadd(acc.s[0][q], cm(G, s));
      acc.s[1][q] = cadd(acc.s[1][q], cm(H, s));
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        const double2 x = __ldg(hh + c * A.np + q);
        acc.v[0][c][q] = cadd(acc.v[0][c][q], cm(G, x));
        acc.v[1][c][q] = cadd(acc.v[1][c][q], cm(H, x));
      }
    }
  } else {
    const double2 ikG = make_double2(-A.k0 * G.y, A.k0 * G.x);
#pragma unroll
    for (int q = 0; q < P; ++q) {
      const double2 s = __ldg(sg + q);
      double2 x[3];
#pragma unroll
      for (int c = 0; c < 3; ++c) x[c] = __ldg(hh + c * A.np + q);
#pragma unroll
      for (int c = 0; c < 3; ++c) {
        acc.v[0][c][q] = cadd(acc.v[0][c][q], csub(cm(ikG, x[c]), cm(Gp[c], s)));
        const int c1 = (c + 1) % 3, c2 = (c + 2) % 3;
        acc.v[1][c][q] = cadd(acc.v[1][c][q], csub(cm(Gp[c1], x[c2]), cm(Gp[c2], x[c1])));
      }
    }
  }
}

template <int P, bool kField>
__global__ void __launch_bounds__(kApplyThreads) green_apply_kernel(ApplyArgs A) {
  extern __shared__ uint32_t apply_bits[];  // kApplyWarps x words: refined columns of each warp's row
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int i = blockIdx.x * kApplyWarps + wid;
  const int words = (A.n + 31) >> 5;
  uint32_t* bits = apply_bits + (size_t)wid * words;
  if (i >= A.n) return;  // whole warps leave: no block-wide barrier follows
  for (int w = lane; w < words; w += 32) bits[w] = 0u;
  __syncwarp();
  long long e0 = 0, e1 = 0;
  if (A.row_ptr) {
    e0 = A.row_ptr[i];
    e1 = A.row_ptr[i + 1];
    for (long long e = e0 + lane; e < e1; e += 32) {
      const int j = A.ref_col[e];
      atomicOr(&bits[j >> 5], 1u << (j & 31));
    }
  }
  __syncwarp();
  const int bi = A.pid[i];
  const double pix = A.pos[3 * i], piy = A.pos[3 * i + 1], piz = A.pos[3 * i + 2];
  const double ni[3] = {A.nvec[3 * i], A.nvec[3 * i + 1], A.nvec[3 * i + 2]};
  Acc<P, kField> acc;
  acc.zero();
  // far pairs: columns whose bit is clear
  for (int j = lane; j < A.n; j += 32) {
    if ((bits[j >> 5] >> (j & 31)) & 1u) continue;
    const int bj = A.pid[j];
    const double rx = pix - A.pos[3 * j], ry = piy - A.pos[3 * j + 1], rz = piz - A.pos[3 * j + 2];
    const bool diag = (bi == bj) && (i == j);
    const double d = diag ? kEps : fmax(sqrt(rx * rx + ry * ry + rz * rz), kEps);
    const double inv_d = 1.0 / d;
    const double aj = A.area[j];
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      const int m = A.blk[t][bi * A.npart + bj];
      if (m <= 0) continue;
      const double kr = A.kt.re[m - 1], ki = A.kt.im[m - 1];
      double pr, pim;
      phase(kr, ki, d, pr, pim);
      const double2 G = make_double2(aj * inv_d * pr, aj * inv_d * pim);
      const double fpre = inv_d * inv_d * aj;
      const double ar = -ki - inv_d, ai = kr;
      const double cr = fpre * (ar * pr - ai * pim), ci = fpre * (ar * pim + ai * pr);
      double2 Gp[3] = {make_double2(rx * cr, rx * ci), make_double2(ry * cr, ry * ci), make_double2(rz * cr, rz * ci)};
      const double ndr = ni[0] * rx + ni[1] * ry + ni[2] * rz;
      double2 H = make_double2(ndr * cr, ndr * ci);
      if (diag) {
        for (int c = 0; c < 3; ++c) Gp[c].x += A.hsign * kTwoPi * ni[c];
        H.x += A.hsign * kTwoPi;
      }
      accumulate<P, kField>(acc, A, t, j, G, H, Gp);
    }
  }
  // refined pairs of row i
  const int no = A.order + 1;
  for (long long e = e0 + lane; e < e1; e += 32) {
    const int j = A.ref_col[e];
    const int bj = A.pid[j];
    const bool diag = (bi == bj) && (i == j);
    const double rx = pix - A.pos[3 * j], ry = piy - A.pos[3 * j + 1], rz = piz - A.pos[3 * j + 2];
    const double d = diag ? kEps : fmax(sqrt(rx * rx + ry * ry + rz * rz), kEps);
#pragma unroll
    for (int t = 0; t < 2; ++t) {
      const int m = A.blk[t][bi * A.npart + bj];
      if (m <= 0) continue;
      const double kr = A.kt.re[m - 1], ki = A.kt.im[m - 1];
      double gr = 0, gi = 0, cr[3] = {0, 0, 0}, ci[3] = {0, 0, 0};
      double pr_ = 1.0, pi_ = 0.0;
      for (int q = 0; q < no; ++q) {
        const double gq = A.g[e * no + q];
        gr += gq * pr_;
        gi += gq * pi_;
        if (kField) {
          for (int c = 0; c < 3; ++c) {
            const double fq = A.fc[(e * 3 + c) * no + q];
            cr[c] += fq * pr_;
            ci[c] += fq * pi_;
          }
        } else {
          const double fq = A.fc[e * no + q];
          cr[0] += fq * pr_;
          ci[0] += fq * pi_;
        }
        const double nr = pr_ * (-ki) - pi_ * kr, nim = pr_ * kr + pi_ * (-ki);
        pr_ = nr;
        pi_ = nim;
      }
      double ph_r, ph_i;
      phase(kr, ki, d, ph_r, ph_i);
      const double2 G = make_double2(gr * ph_r - gi * ph_i, gr * ph_i + gi * ph_r);
      double2 Gp[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
      double2 H = make_double2(0, 0);
      if (kField) {
        for (int c = 0; c < 3; ++c) {
          Gp[c] = make_double2(cr[c] * ph_r - ci[c] * ph_i, cr[c] * ph_i + ci[c] * ph_r);
          if (diag) Gp[c].x += A.hsign * kTwoPi * ni[c];
        }
      } else {
        // H = (n_i . f) (ik)^q e^{ikd}, + 2 pi on the diagonal
        H = make_double2(cr[0] * ph_r - ci[0] * ph_i, cr[0] * ph_i + ci[0] * ph_r);
        if (diag) H.x += A.hsign * kTwoPi;
      }
      accumulate<P, kField>(acc, A, t, j, G, H, Gp);
    }
  }
  // warp sums; lane q writes polarisation q
  auto wsum = [&](double2 v) {
#pragma unroll
    for (int o = 16; o > 0; o >>= 1) {
      v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
      v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
    }
    return v;
  };
  const long long rs = (long long)i * A.np + A.q0, rv = (long long)i * 3 * A.np + A.q0;
  if (!kField) {
#pragma unroll
    for (int a = 0; a < 2; ++a)
#pragma unroll
      for (int q = 0; q < P; ++q) {
        const double2 v = wsum(acc.s[a][q]);
        if (lane == 0) A.out[a][rs + q] = v;
      }
  }
#pragma unroll
  for (int a = 0; a < 2; ++a)
#pragma unroll
    for (int c = 0; c < 3; ++c)
#pragma unroll
      for (int q = 0; q < P; ++q) {
        const double2 v = wsum(acc.v[a][c][q]);
        if (lane == 0) A.out[kField ? a : 2 + a][rv + c * A.np + q] = v;
      }
}

template <int P, bool kField>
static int apply_launch(ApplyArgs A, cudaStream_t s) {
  auto kern = green_apply_kernel<P, kField>;
  const int words = (A.n + 31) / 32;
  const int smem = kApplyWarps * words * (int)sizeof(uint32_t);
  BEM_CUDA_CHECK(set_kernel_attrs_once(kern, smem, false));
  kern<<<ceil_div(A.n, kApplyWarps), kApplyThreads, smem, s>>>(A);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

// all polarisations in chunks of 4, 2, 1
template <bool kField>
static int apply_all(ApplyArgs A, cudaStream_t s) {
  int st = BEM200_OK;
  for (int q0 = 0; q0 < A.np && !st;) {
    A.q0 = q0;
    const int left = A.np - q0;
    if (left >= 4) {
      st = apply_launch<4, kField>(A, s);
      q0 += 4;
    } else if (left >= 2) {
      st = apply_launch<2, kField>(A, s);
      q0 += 2;
    } else {
      st = apply_launch<1, kField>(A, s);
      q0 += 1;
    }
  }
  return st;
}

static int fill_ktab(KTab& kt, int nmat, const double* kmat_host) {
  BEM_REQUIRE(nmat > 0 && nmat <= kMaxMat && kmat_host, BEM200_ERR_ARG, "green: 1 <= nmat <= %d required", kMaxMat);
  for (int m = 0; m < kMaxMat; ++m) {
    kt.re[m] = m < nmat ? kmat_host[2 * m] : 0.0;
    kt.im[m] = m < nmat ? kmat_host[2 * m + 1] : 0.0;
  }
  return BEM200_OK;
}

// shared-memory limit of the apply kernel: kApplyWarps bitmaps of n bits
constexpr int kApplyMaxN = 8 * 48 * 1024 / kApplyWarps;

}  // namespace fld
}  // namespace bem200

using namespace bem200;
using namespace bem200::fld;

extern "C" {

int bem200_green_assemble_cart(int n, int npart, const int32_t* pid, const int32_t* blk, int nmat,
                               const double* kmat_host, const double* pos, const double* nvec, const double* area,
                               int64_t nref, const int32_t* ref_row, const int32_t* ref_col, int order,
                               const double* f, int hkey, void* out, void* stream) {
  BEM_REQUIRE(n > 0 && npart > 0 && pid && blk && pos && nvec && area && out, BEM200_ERR_ARG,
              "green_assemble_cart: bad arguments");
  BEM_REQUIRE(hkey >= 0 && hkey <= 2, BEM200_ERR_ARG, "green_assemble_cart: hkey must be 0 (Gp), 1 (H1p), 2 (H2p)");
  BEM_REQUIRE(nref == 0 || (ref_row && ref_col && f && order >= 0 && order <= ge::kMaxOrder), BEM200_ERR_ARG,
              "green_assemble_cart: refinement tables missing");
  KTab kt;
  int st = fill_ktab(kt, nmat, kmat_host);
  if (st) return st;
  const double hsign = hkey == 1 ? 1.0 : (hkey == 2 ? -1.0 : 0.0);
  cudaStream_t s = (cudaStream_t)stream;
  dim3 grid(ceil_div(n, kCartThreads), ceil_div(n, kCartRows));
  BEM_REQUIRE(grid.y <= 65535, BEM200_ERR_ARG, "green_assemble_cart: n too large");
  green_cart_far_kernel<<<grid, kCartThreads, 0, s>>>(n, npart, pid, blk, kt, pos, nvec, area, hsign,
                                                      (double2*)out);
  BEM_LAUNCH_CHECK();
  if (nref > 0) {
    green_cart_refined_kernel<<<ceil_div(nref, 256), 256, 0, s>>>(nref, ref_row, ref_col, order, f, npart, pid, blk, kt,
                                                                  pos, nvec, hsign, n, (double2*)out);
    BEM_LAUNCH_CHECK();
  }
  return BEM200_OK;
}

static int apply_common(ApplyArgs& A, int n, int npart, const int32_t* pid, const int32_t* blk0, const int32_t* blk1,
                        int nmat, const double* kmat_host, const double* pos, const double* nvec, const double* area,
                        const int64_t* ref_row_ptr, const int32_t* ref_col, int order, const double* g,
                        const double* fc, int hkey, int npol, const void* sig1, const void* sig2, const void* h1,
                        const void* h2) {
  BEM_REQUIRE(n > 0 && npart > 0 && npol > 0 && pid && blk0 && blk1 && pos && nvec && area && sig1 && sig2 && h1 &&
                  h2,
              BEM200_ERR_ARG, "green potential/field: bad arguments");
  BEM_REQUIRE(n <= kApplyMaxN, BEM200_ERR_UNSUPPORTED, "green potential/field: n = %d above %d faces", n, kApplyMaxN);
  BEM_REQUIRE(hkey == 1 || hkey == 2, BEM200_ERR_ARG, "green potential/field: hkey must be 1 (H1) or 2 (H2)");
  BEM_REQUIRE(!ref_row_ptr || (ref_col && g && fc && order >= 0 && order <= ge::kMaxOrder), BEM200_ERR_ARG,
              "green potential/field: refinement tables missing");
  int st = fill_ktab(A.kt, nmat, kmat_host);
  if (st) return st;
  A.n = n;
  A.npart = npart;
  A.order = order;
  A.np = npol;
  A.q0 = 0;
  A.pid = pid;
  A.blk[0] = blk0;
  A.blk[1] = blk1;
  A.pos = pos;
  A.nvec = nvec;
  A.area = area;
  A.row_ptr = ref_row_ptr;
  A.ref_col = ref_col;
  A.g = g;
  A.fc = fc;
  A.hsign = hkey == 1 ? 1.0 : -1.0;
  A.k0 = 0.0;
  A.sig[0] = (const double2*)sig1;
  A.sig[1] = (const double2*)sig2;
  A.h[0] = (const double2*)h1;
  A.h[1] = (const double2*)h2;
  return BEM200_OK;
}

int bem200_green_potential(int n, int npart, const int32_t* pid, const int32_t* blk0, const int32_t* blk1, int nmat,
                           const double* kmat_host, const double* pos, const double* nvec, const double* area,
                           const int64_t* ref_row_ptr, const int32_t* ref_col, int order, const double* g,
                           const double* fn, int hkey, int npol, const void* sig1, const void* sig2, const void* h1,
                           const void* h2, void* phi, void* phip, void* a, void* ap, void* stream) {
  ApplyArgs A;
  int st = apply_common(A, n, npart, pid, blk0, blk1, nmat, kmat_host, pos, nvec, area, ref_row_ptr, ref_col, order,
                        g, fn, hkey, npol, sig1, sig2, h1, h2);
  if (st) return st;
  BEM_REQUIRE(phi && phip && a && ap, BEM200_ERR_ARG, "green_potential: null output");
  A.out[0] = (double2*)phi;
  A.out[1] = (double2*)phip;
  A.out[2] = (double2*)a;
  A.out[3] = (double2*)ap;
  return apply_all<false>(A, (cudaStream_t)stream);
}

int bem200_green_field(int n, int npart, const int32_t* pid, const int32_t* blk0, const int32_t* blk1, int nmat,
                       const double* kmat_host, const double* pos, const double* nvec, const double* area,
                       const int64_t* ref_row_ptr, const int32_t* ref_col, int order, const double* g, const double* f,
                       int hkey, double k0, int npol, const void* sig1, const void* sig2, const void* h1,
                       const void* h2, void* e, void* h, void* stream) {
  ApplyArgs A;
  int st = apply_common(A, n, npart, pid, blk0, blk1, nmat, kmat_host, pos, nvec, area, ref_row_ptr, ref_col, order,
                        g, f, hkey, npol, sig1, sig2, h1, h2);
  if (st) return st;
  BEM_REQUIRE(e && h, BEM200_ERR_ARG, "green_field: null output");
  A.k0 = k0;
  A.out[0] = (double2*)e;
  A.out[1] = (double2*)h;
  A.out[2] = A.out[3] = nullptr;
  return apply_all<true>(A, (cudaStream_t)stream);
}

}  // extern "C"
