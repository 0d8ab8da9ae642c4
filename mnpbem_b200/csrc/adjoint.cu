// Reverse-mode derivative of a functional of the BEM solution with respect to
// the face geometry: c = lambda^T (dA/dtheta) x for every geometry parameter
// theta at once, given the solution x = (sig1, h1 | sig2, h2) and the adjoint
// lambda = A^-T w (equation-space layout phi, a, alpha, De).  The reference has
// no gradients; the operator differentiated is the BEM operator of
// Garcia de Abajo & Howie Eqs. (19, 20) as assembled by the reference
// (mnpbem/greenfun/greenret_refined.py:654-867, compgreen_ret.py:192-272 and
// :376-400 for the closed-surface correction, bem_ret_iter.py:1362-1501 for the
// operator's structure).
//
// lambda^T A x = sum_ij  G1_ij CGa_ij + H1_ij CHa_ij - G2_ij CGb_ij - H2_ij CHb_ij
//   CGa_ij = sum_p [ lphi_i s1_j + la_i . h1_j - ik (n_i . lalpha_i) e1_j s1_j
//                    - ik lDe_i e1_j (n_i . h1_j) ]
//   CHa_ij = sum_p [ lalpha_i . h1_j + lDe_i e1_j s1_j ]      (b: s2, h2, e2)
// with G1 = G[r00] - G[r10], G2 = G[r11] - G[r01] (region terms of each
// particle block, wavenumber of the material filling them).  Far pairs:
//   G = a_j / d e^{ikd},  Gp = r phi(d) a_j,  F = n_i . Gp,
//   phi(d) = (ik - 1/d) e^{ikd} / d^2,  phi'(d) = e^{ikd} / d^2 (3/d^2 - 3ik/d - k^2)
// refined pairs: G = sum_m g_m (ik)^m e^{ikd}, Gp = sum_m f_m (ik)^m e^{ikd},
// whose coefficients g, f depend on the face nodes through the refinement
// quadrature: their derivatives are exact (dual numbers, dual.cuh).
//
// Nothing n x n (x 3) is stored: the far pairs are swept by one warp per row
// (row-side gradients: pos_i, nvec_i) and one warp per column (pos_j, area_j),
// every Green value and derivative recomputed in registers.
//
// Output: complex cotangents (c = sum of lambda^T dA x contributions) for
// pos (n, 3), nvec (n, 3), area (n), tvec1 (n, 3), tvec2 (n, 3) and the face
// nodes (n, 9, 3); the caller chains them to the vertices.
#include "dual.cuh"
#include "green_entry.cuh"

namespace bem200 {
namespace adj {

using ge::kEps;
using ge::kMaxMat;
using ge::kMaxOrder;
using ge::kTwoPi;
using ge::phase;

constexpr int kMaxPol = 4;

struct KTab {
  double re[kMaxMat], im[kMaxMat];
};

struct Args {
  int n, npol, npart, order;
  KTab kt;
  double k0;
  int eps_per_face;
  double2 e1s, e2s;
  const double2* e1d;
  const double2* e2d;
  const int32_t* pid;
  const int32_t* blk;  // (npart, npart, 4): r00, r10, r11, r01
  const uint64_t* closed_mask;
  const double* pos;
  const double* nvec;
  const double* area;
  const double* tvec1;
  const double* tvec2;
  const double* nodes;
  const int32_t* face_kind;
  const double* rules;
  int n28, n3, n4;
  long long nref;
  const int64_t* row_ptr;  // CSR of the refined pairs
  const int32_t* ref_row;
  const int32_t* ref_col;
  const int8_t* ref_kind;
  const int64_t* col_ptr;  // CSC: refined rows of every column
  const int32_t* csc_row;
  const double* g;     // (nref, order + 1)
  const double* f;     // (nref, 3, order + 1), after the closed-surface correction
  const double* corr;  // (n) closed-surface correction of each face (0 if open)
  // solution and adjoint
  const double2* W1;   // (n, 4p): s1 | h1
  const double2* W2;   // (n, 4p): s2 | h2
  const double2* lam;  // phi (n, p) | a (n, 3, p) | alpha (n, 3, p) | De (n, p)
  // outputs and scratch
  double2* gpos;
  double2* gnv;
  double2* garea;
  double2* gt1;
  double2* gt2;
  double2* gnodes;
  double2* ghat;   // (nref, order + 1)
  double2* fhat;   // (nref, 3, order + 1)
  double2* shat;   // (n): cotangent of the closed-surface sum S_j
  double2* chat;   // (n): cotangent of corr_j
  int64_t* diag_e; // (n): refined entry of the diagonal (j, j), or -1
};

__device__ __forceinline__ double2 cm(double2 a, double2 b) {
  return make_double2(a.x * b.x - a.y * b.y, a.x * b.y + a.y * b.x);
}
__device__ __forceinline__ double2 cs(double2 a, double s) { return make_double2(a.x * s, a.y * s); }
__device__ __forceinline__ double2 ca(double2 a, double2 b) { return make_double2(a.x + b.x, a.y + b.y); }
__device__ __forceinline__ double2 cneg(double2 a) { return make_double2(-a.x, -a.y); }
__device__ __forceinline__ void atomic_c(double2* p, double2 v) {
  atomicAdd(&p->x, v.x);
  atomicAdd(&p->y, v.y);
}
__device__ __forceinline__ double2 eps_of(const Args& A, int j, bool second) {
  if (!A.eps_per_face) return second ? A.e2s : A.e1s;
  return second ? A.e2d[j] : A.e1d[j];
}
__device__ __forceinline__ double2 wsum2(double2 v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.x += __shfl_xor_sync(0xffffffffu, v.x, o);
    v.y += __shfl_xor_sync(0xffffffffu, v.y, o);
  }
  return v;
}

// operator weights of pair (i, j) for family a (s1, h1, e1) or b (s2, h2, e2):
// CG, CH and dCG/dn_i (explicit normal in the operator)
struct Weights {
  double2 CG, CH, dCGdn[3];
};

__device__ __forceinline__ Weights pair_weights(const Args& A, int i, int j, bool fam_b, const double (&ni)[3]) {
  const int p = A.npol;
  const long long np = (long long)A.n * p;
  const double2* W = (fam_b ? A.W2 : A.W1) + (long long)j * 4 * p;
  const double2 e = eps_of(A, j, fam_b);
  const double2 ik = make_double2(0.0, A.k0);
  const double2* lphi = A.lam + (long long)i * p;
  const double2* la = A.lam + np + (long long)i * 3 * p;
  const double2* lal = A.lam + 4 * np + (long long)i * 3 * p;
  const double2* lDe = A.lam + 7 * np + (long long)i * p;
  Weights w;
  w.CG = w.CH = make_double2(0, 0);
  w.dCGdn[0] = w.dCGdn[1] = w.dCGdn[2] = make_double2(0, 0);
  for (int q = 0; q < p; ++q) {
    const double2 s = W[q];
    const double2 es = cm(e, s);
    double2 nla = make_double2(0, 0), nh = make_double2(0, 0);
    double2 lah = make_double2(0, 0), lalh = make_double2(0, 0);
    const double2 ld = lDe[q];
    for (int c = 0; c < 3; ++c) {
      const double2 h = W[p + c * p + q];
      const double2 lac = la[c * p + q], lalc = lal[c * p + q];
      nla = ca(nla, cs(lalc, ni[c]));
      nh = ca(nh, cs(h, ni[c]));
      lah = ca(lah, cm(lac, h));
      lalh = ca(lalh, cm(lalc, h));
      // d/dn_ic of [-ik (n.lalpha) e s - ik lDe e (n.h)]
      const double2 dd = ca(cm(lalc, es), cm(ld, cm(e, h)));
      w.dCGdn[c] = ca(w.dCGdn[c], cneg(cm(ik, dd)));
    }
    double2 cg = ca(cm(lphi[q], s), lah);
    cg = ca(cg, cneg(cm(ik, cm(nla, es))));
    cg = ca(cg, cneg(cm(ik, cm(ld, cm(e, nh)))));
    w.CG = ca(w.CG, cg);
    w.CH = ca(w.CH, ca(lalh, cm(ld, es)));
  }
  return w;
}

// the four region terms: family (0: G1/H1, 1: G2/H2) and sign in lambda^T A x
__device__ __forceinline__ int term_fam(int t) { return t < 2 ? 0 : 1; }
__device__ __forceinline__ double term_sgn(int t) { return (t == 0 || t == 3) ? 1.0 : -1.0; }

// far-pair derivative pieces of one region term (wavenumber kr + i ki):
//   dpos = CG dG/dpos_i + CH dF/dpos_i,  dn = CH Gp,  Gv = G (for the explicit
//   normal terms), val = CG G + CH F (for the area derivative: d/da_j = val / a_j)
struct FarTerm {
  double2 dpos[3], dn[3], G, val;
};

__device__ __forceinline__ FarTerm far_term(double kr, double ki, double d, const double (&r)[3], double aj,
                                            const double (&ni)[3], double2 CG, double2 CH) {
  FarTerm o;
  double pr, pim;
  phase(kr, ki, d, pr, pim);
  const double2 ph = make_double2(pr, pim);
  const double id = 1.0 / d, id2 = id * id;
  const double2 ik = make_double2(-ki, kr);
  const double2 ikm = make_double2(-ki - id, kr);  // ik - 1/d
  const double2 G = cs(ph, aj * id);
  const double2 phi = cs(cm(ikm, ph), id2);        // (ik - 1/d) e^{ikd} / d^2
  // phi' = e^{ikd} / d^2 (3/d^2 - 3ik/d - k^2)
  const double2 k2 = cm(ik, ik);                   // -k^2
  const double2 fac = make_double2(3.0 * id2 - 3.0 * ik.x * id + k2.x, -3.0 * ik.y * id + k2.y);
  const double2 dphi = cs(cm(fac, ph), id2);
  const double ndr = ni[0] * r[0] + ni[1] * r[1] + ni[2] * r[2];
  const double2 F = cs(phi, ndr * aj);
  const double2 dGdd = cm(G, ikm);                 // dG/dd
  for (int c = 0; c < 3; ++c) {
    const double u = r[c] * id;                    // dd/dpos_i
    const double2 dF = ca(cs(phi, ni[c] * aj), cs(dphi, ndr * aj * u));
    o.dpos[c] = ca(cm(CG, cs(dGdd, u)), cm(CH, dF));
    o.dn[c] = cm(CH, cs(phi, r[c] * aj));
  }
  o.G = G;
  o.val = ca(cm(CG, G), cm(CH, F));
  return o;
}

// closed-surface far term a_i Fs_ij, Fs_ij = -(n_i . r) / d^3 a_j: derivatives
// with respect to pos_i (vector), n_i (vector), a_i and a_j
struct ClosedTerm {
  double dpos[3], dn[3], da_i, da_j;
};
__device__ __forceinline__ ClosedTerm closed_term(double d, const double (&r)[3], double ai, double aj,
                                                  const double (&ni)[3]) {
  ClosedTerm o;
  const double id = 1.0 / d, id3 = id * id * id, id5 = id3 * id * id;
  const double ndr = ni[0] * r[0] + ni[1] * r[1] + ni[2] * r[2];
  const double Fs = -ndr * id3 * aj;
  for (int c = 0; c < 3; ++c) {
    o.dpos[c] = ai * aj * (-ni[c] * id3 + 3.0 * ndr * r[c] * id5);
    o.dn[c] = -ai * aj * r[c] * id3;
  }
  o.da_i = Fs;
  o.da_j = ai * Fs / aj;
  return o;
}

__device__ __forceinline__ bool in_surf(const Args& A, int i, int j) {
  return (A.closed_mask[A.pid[j]] >> A.pid[i]) & 1ull;
}

// ------------------------------------------------------------ far pairs, rows
constexpr int kWarps = 4;

__global__ void __launch_bounds__(32 * kWarps) far_rows_kernel(Args A) {
  extern __shared__ uint32_t row_bits[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int i = blockIdx.x * kWarps + wid;
  const int words = (A.n + 31) >> 5;
  uint32_t* bits = row_bits + (size_t)wid * words;
  if (i >= A.n) return;
  for (int w = lane; w < words; w += 32) bits[w] = 0u;
  __syncwarp();
  for (long long e = A.row_ptr[i] + lane; e < A.row_ptr[i + 1]; e += 32) {
    const int j = A.ref_col[e];
    atomicOr(&bits[j >> 5], 1u << (j & 31));
  }
  __syncwarp();
  const int bi = A.pid[i];
  const double pix = A.pos[3 * i], piy = A.pos[3 * i + 1], piz = A.pos[3 * i + 2];
  const double ni[3] = {A.nvec[3 * i], A.nvec[3 * i + 1], A.nvec[3 * i + 2]};
  const double ai = A.area[i];
  double2 gp[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
  double2 gn[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
  double2 ga = make_double2(0, 0);
  for (int j = lane; j < A.n; j += 32) {
    if ((bits[j >> 5] >> (j & 31)) & 1u) continue;
    if (j == i) continue;
    const int bj = A.pid[j];
    const double r[3] = {pix - A.pos[3 * j], piy - A.pos[3 * j + 1], piz - A.pos[3 * j + 2]};
    const double d = fmax(sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]), kEps);
    const double aj = A.area[j];
    const int* bm = A.blk + (bi * A.npart + bj) * 4;
    Weights wf[2];
    bool have[2] = {false, false};
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int m = bm[t];
      if (m <= 0) continue;
      const int fam = term_fam(t);
      if (!have[fam]) {
        wf[fam] = pair_weights(A, i, j, fam == 1, ni);
        have[fam] = true;
      }
      const FarTerm ft = far_term(A.kt.re[m - 1], A.kt.im[m - 1], d, r, aj, ni, wf[fam].CG, wf[fam].CH);
      const double sg = term_sgn(t);
      for (int c = 0; c < 3; ++c) {
        gp[c] = ca(gp[c], cs(ft.dpos[c], sg));
        gn[c] = ca(gn[c], cs(ca(ft.dn[c], cm(ft.G, wf[fam].dCGdn[c])), sg));
      }
    }
    if (in_surf(A, i, j)) {
      const double2 sh = A.shat[j];
      if (sh.x != 0.0 || sh.y != 0.0) {
        const ClosedTerm ct = closed_term(d, r, ai, aj, ni);
        for (int c = 0; c < 3; ++c) {
          gp[c] = ca(gp[c], cs(sh, ct.dpos[c]));
          gn[c] = ca(gn[c], cs(sh, ct.dn[c]));
        }
        ga = ca(ga, cs(sh, ct.da_i));
      }
    }
  }
  for (int c = 0; c < 3; ++c) {
    gp[c] = wsum2(gp[c]);
    gn[c] = wsum2(gn[c]);
  }
  ga = wsum2(ga);
  if (lane == 0) {
    for (int c = 0; c < 3; ++c) {
      A.gpos[3 * i + c] = ca(A.gpos[3 * i + c], gp[c]);
      A.gnv[3 * i + c] = ca(A.gnv[3 * i + c], gn[c]);
    }
    A.garea[i] = ca(A.garea[i], ga);
  }
}

// ------------------------------------------------------------ far pairs, columns
__global__ void __launch_bounds__(32 * kWarps) far_cols_kernel(Args A) {
  extern __shared__ uint32_t col_bits[];
  const int lane = threadIdx.x & 31, wid = threadIdx.x >> 5;
  const int j = blockIdx.x * kWarps + wid;
  const int words = (A.n + 31) >> 5;
  uint32_t* bits = col_bits + (size_t)wid * words;
  if (j >= A.n) return;
  for (int w = lane; w < words; w += 32) bits[w] = 0u;
  __syncwarp();
  for (long long e = A.col_ptr[j] + lane; e < A.col_ptr[j + 1]; e += 32) {
    const int i = A.csc_row[e];
    atomicOr(&bits[i >> 5], 1u << (i & 31));
  }
  __syncwarp();
  const int bj = A.pid[j];
  const double pjx = A.pos[3 * j], pjy = A.pos[3 * j + 1], pjz = A.pos[3 * j + 2];
  const double aj = A.area[j];
  const double2 sh = A.shat[j];
  double2 gp[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
  double2 ga = make_double2(0, 0);
  for (int i = lane; i < A.n; i += 32) {
    if ((bits[i >> 5] >> (i & 31)) & 1u) continue;
    if (i == j) continue;
    const int bi = A.pid[i];
    const double r[3] = {A.pos[3 * i] - pjx, A.pos[3 * i + 1] - pjy, A.pos[3 * i + 2] - pjz};
    const double d = fmax(sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]), kEps);
    const double ni[3] = {A.nvec[3 * i], A.nvec[3 * i + 1], A.nvec[3 * i + 2]};
    const int* bm = A.blk + (bi * A.npart + bj) * 4;
    Weights wf[2];
    bool have[2] = {false, false};
#pragma unroll
    for (int t = 0; t < 4; ++t) {
      const int m = bm[t];
      if (m <= 0) continue;
      const int fam = term_fam(t);
      if (!have[fam]) {
        wf[fam] = pair_weights(A, i, j, fam == 1, ni);
        have[fam] = true;
      }
      const FarTerm ft = far_term(A.kt.re[m - 1], A.kt.im[m - 1], d, r, aj, ni, wf[fam].CG, wf[fam].CH);
      const double sg = term_sgn(t);
      for (int c = 0; c < 3; ++c) gp[c] = ca(gp[c], cs(ft.dpos[c], -sg));  // d/dpos_j = -d/dpos_i
      ga = ca(ga, cs(ft.val, sg / aj));
    }
    if ((sh.x != 0.0 || sh.y != 0.0) && in_surf(A, i, j)) {
      const ClosedTerm ct = closed_term(d, r, A.area[i], aj, ni);
      for (int c = 0; c < 3; ++c) gp[c] = ca(gp[c], cs(sh, -ct.dpos[c]));
      ga = ca(ga, cs(sh, ct.da_j));
    }
  }
  for (int c = 0; c < 3; ++c) gp[c] = wsum2(gp[c]);
  ga = wsum2(ga);
  if (lane == 0) {
    for (int c = 0; c < 3; ++c) A.gpos[3 * j + c] = ca(A.gpos[3 * j + c], gp[c]);
    A.garea[j] = ca(A.garea[j], ga);
  }
}

// ------------------------------------------------------------ refined pairs
// Operator part: cotangents of the (corrected) coefficients g, f of entry e,
// the phase derivative (through d) and the normal derivatives.
__global__ void refined_op_kernel(Args A) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= A.nref) return;
  const int i = A.ref_row[e], j = A.ref_col[e];
  const int bi = A.pid[i], bj = A.pid[j];
  const bool diag = (bi == bj) && (i == j);
  const double r[3] = {A.pos[3 * i] - A.pos[3 * j], A.pos[3 * i + 1] - A.pos[3 * j + 1],
                       A.pos[3 * i + 2] - A.pos[3 * j + 2]};
  const double d = diag ? kEps : fmax(sqrt(r[0] * r[0] + r[1] * r[1] + r[2] * r[2]), kEps);
  const double ni[3] = {A.nvec[3 * i], A.nvec[3 * i + 1], A.nvec[3 * i + 2]};
  const int no = A.order + 1;
  const int* bm = A.blk + (bi * A.npart + bj) * 4;
  double2 gh[kMaxOrder + 1], fh[3][kMaxOrder + 1];
  for (int m = 0; m < no; ++m) {
    gh[m] = make_double2(0, 0);
    fh[0][m] = fh[1][m] = fh[2][m] = make_double2(0, 0);
  }
  double2 gp[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
  double2 gn[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
  Weights wf[2];
  bool have[2] = {false, false};
  for (int t = 0; t < 4; ++t) {
    const int mat = bm[t];
    if (mat <= 0) continue;
    const int fam = term_fam(t);
    if (!have[fam]) {
      wf[fam] = pair_weights(A, i, j, fam == 1, ni);
      have[fam] = true;
    }
    const double sg = term_sgn(t);
    const double kr = A.kt.re[mat - 1], ki = A.kt.im[mat - 1];
    const double2 ik = make_double2(-ki, kr);
    double pr, pim;
    phase(kr, ki, d, pr, pim);
    const double2 ph = make_double2(pr, pim);
    double2 ikm = make_double2(1, 0);  // (ik)^m
    double2 Sg = make_double2(0, 0), Sf[3] = {make_double2(0, 0), make_double2(0, 0), make_double2(0, 0)};
    const double2 CGs = cs(wf[fam].CG, sg), CHs = cs(wf[fam].CH, sg);
    for (int m = 0; m < no; ++m) {
      const double2 b = cm(ikm, ph);  // (ik)^m e^{ikd}
      gh[m] = ca(gh[m], cm(CGs, b));
      Sg = ca(Sg, cs(ikm, A.g[e * no + m]));
      for (int c = 0; c < 3; ++c) {
        fh[c][m] = ca(fh[c][m], cs(cm(CHs, b), ni[c]));
        Sf[c] = ca(Sf[c], cs(ikm, A.f[(e * 3 + c) * no + m]));
      }
      ikm = cm(ikm, ik);
    }
    const double2 G = cm(Sg, ph);
    double2 Gp[3];
    for (int c = 0; c < 3; ++c) Gp[c] = cm(Sf[c], ph);
    const double2 F = ca(ca(cs(Gp[0], ni[0]), cs(Gp[1], ni[1])), cs(Gp[2], ni[2]));
    if (!diag) {  // d/dd of e^{ikd}: ik times the value
      const double2 dv = cm(ik, ca(cm(CGs, G), cm(CHs, F)));
      for (int c = 0; c < 3; ++c) gp[c] = ca(gp[c], cs(dv, r[c] / d));
    }
    for (int c = 0; c < 3; ++c) gn[c] = ca(gn[c], ca(cm(CHs, Gp[c]), cm(G, cs(wf[fam].dCGdn[c], sg))));
  }
  for (int m = 0; m < no; ++m) {
    A.ghat[e * no + m] = gh[m];
    for (int c = 0; c < 3; ++c) A.fhat[(e * 3 + c) * no + m] = fh[c][m];
  }
  for (int c = 0; c < 3; ++c) {
    if (!diag) {
      atomic_c(&A.gpos[3 * i + c], gp[c]);
      atomic_c(&A.gpos[3 * j + c], cneg(gp[c]));
    }
    atomic_c(&A.gnv[3 * i + c], gn[c]);
  }
  if (diag) A.diag_e[j] = e;
}

// closed-surface correction of face j: corr_j = -2 pi - S_j / a_j, added as
// corr_j n_j to f[(j, j), :, 0].  chat_j = n_j . fhat[(j, j), :, 0]; the sum
// S_j gets the cotangent -chat_j / a_j; a_j and n_j get their direct parts.
__global__ void closed_prep_kernel(Args A) {
  const int j = blockIdx.x * blockDim.x + threadIdx.x;
  if (j >= A.n) return;
  const long long e = A.diag_e[j];
  A.shat[j] = make_double2(0, 0);
  if (e < 0 || A.closed_mask[A.pid[j]] == 0) return;
  const int no = A.order + 1;
  const double nj[3] = {A.nvec[3 * j], A.nvec[3 * j + 1], A.nvec[3 * j + 2]};
  double2 ch = make_double2(0, 0);
  for (int c = 0; c < 3; ++c) {
    const double2 fh0 = A.fhat[(e * 3 + c) * no];
    ch = ca(ch, cs(fh0, nj[c]));
    A.gnv[3 * j + c] = ca(A.gnv[3 * j + c], cs(fh0, A.corr[j]));
  }
  const double aj = A.area[j];
  A.chat[j] = ch;
  A.shat[j] = cs(ch, -1.0 / aj);
  // corr_j = -2 pi - S_j / a_j with S_j / a_j = -2 pi - corr_j: d/da_j (direct) = S_j / a_j^2
  A.garea[j] = ca(A.garea[j], cs(ch, (-kTwoPi - A.corr[j]) / aj));
}

// refined entries of a closed surface's sum: S_j gets a_i n_i . f_e0 (the
// uncorrected coefficient) for the refined pairs (i, j) with i on j's surface
__global__ void refined_closed_kernel(Args A) {
  const long long e = (long long)blockIdx.x * blockDim.x + threadIdx.x;
  if (e >= A.nref) return;
  const int i = A.ref_row[e], j = A.ref_col[e];
  const double2 sh = A.shat[j];
  if ((sh.x == 0.0 && sh.y == 0.0) || !in_surf(A, i, j)) return;
  const int no = A.order + 1;
  const double ni[3] = {A.nvec[3 * i], A.nvec[3 * i + 1], A.nvec[3 * i + 2]};
  const double ai = A.area[i];
  const bool diag = (i == j);
  double f0[3], nf = 0.0;
  for (int c = 0; c < 3; ++c) {
    f0[c] = A.f[(e * 3 + c) * no] - (diag ? A.corr[j] * ni[c] : 0.0);
    nf += ni[c] * f0[c];
  }
  for (int c = 0; c < 3; ++c) {
    A.fhat[(e * 3 + c) * no] = ca(A.fhat[(e * 3 + c) * no], cs(sh, ai * ni[c]));
    atomic_c(&A.gnv[3 * i + c], cs(sh, ai * f0[c]));
  }
  atomic_c(&A.garea[i], cs(sh, nf));
}

// ------------------------------------------------------------ refinement coefficients
// Derivatives of the refinement coefficients g_m, f_cm of entry e with respect
// to its inputs, contracted with their cotangents: one warp per entry, one
// dual-number evaluation of the entry's quadrature per input coordinate.
// Inputs: self terms (kind 2): pos_i, n_i, t1_i, t2_i and the nodes of face
// j; others: pos_i, pos_j and the nodes of face j.
using ad::Dual;
using ad::V3;

template <typename T>
__device__ __forceinline__ T wsumT(T v);
template <>
__device__ __forceinline__ Dual wsumT<Dual>(Dual v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) {
    v.v += __shfl_xor_sync(0xffffffffu, v.v, o);
    v.d += __shfl_xor_sync(0xffffffffu, v.d, o);
  }
  return v;
}
__device__ __forceinline__ double wmax(double v) {
#pragma unroll
  for (int o = 16; o > 0; o >>= 1) v = fmax(v, __shfl_xor_sync(0xffffffffu, v, o));
  return v;
}

__device__ __forceinline__ V3<Dual> seed3(const double* p, int dir, int first) {
  V3<Dual> v = ad::mk3<Dual>(Dual(p[0]), Dual(p[1]), Dual(p[2]));
  if (dir == first) v.x.d = 1.0;
  if (dir == first + 1) v.y.d = 1.0;
  if (dir == first + 2) v.z.d = 1.0;
  return v;
}

__global__ void refine_coef_grad_kernel(Args A) {
  const long long e = ((long long)blockIdx.x * blockDim.x + threadIdx.x) >> 5;
  const int lane = threadIdx.x & 31;
  if (e >= A.nref) return;
  const int i = A.ref_row[e], j = A.ref_col[e], kind = A.ref_kind[e];
  const int no = A.order + 1;
  const int fk = A.face_kind[j];
  const int nn = fk == 0 ? 3 : (fk == 1 ? 4 : (fk == 2 ? 6 : 9));
  const bool self = (kind == 2);
  // directions: self: pos_i (0-2), n_i (3-5), t1 (6-8), t2 (9-11), nodes (12 + 3c + x)
  //             near: pos_i (0-2), pos_j (3-5), nodes (6 + 3c + x)
  const int nbase = self ? 12 : 6;
  const int ndir = nbase + 3 * nn;
  const double* nodes = A.nodes + 27LL * j;
  for (int dir = 0; dir < ndir; ++dir) {
    ad::Face<Dual> fc;
    fc.kind = fk;
    for (int c = 0; c < nn; ++c) fc.node[c] = seed3(nodes + 3 * c, dir, nbase + 3 * c);
    const V3<Dual> pi = seed3(A.pos + 3 * i, dir, 0);
    Dual sg[kMaxOrder + 1], s1[kMaxOrder + 1], s2[kMaxOrder + 1], s3[kMaxOrder + 1];
    for (int m = 0; m <= kMaxOrder; ++m) sg[m] = s1[m] = s2[m] = s3[m] = Dual(0.0);
    double2 acc = make_double2(0, 0);
    if (self) {
      const V3<Dual> ni = seed3(A.nvec + 3 * i, dir, 3);
      const V3<Dual> t1 = seed3(A.tvec1 + 3 * i, dir, 6);
      const V3<Dual> t2 = seed3(A.tvec2 + 3 * i, dir, 9);
      const int npts = (fk == 0 || fk == 2) ? A.n3 : A.n4;
      double rmax = 0.0;
      for (int q = lane; q < npts; q += 32) {
        V3<Dual> pt;
        Dual w;
        ad::polar_pt<Dual>(fc, A.rules, A.n28, A.n3, A.n4, q, pt, w);
        rmax = fmax(rmax, fmax(ad::val(ad::norm(ad::sub(pi, pt))), kEps));
      }
      rmax = wmax(rmax);
      const double rfloor = 1e-4 * rmax;
      for (int q = lane; q < npts; q += 32) {
        V3<Dual> pt;
        Dual w;
        ad::polar_pt<Dual>(fc, A.rules, A.n28, A.n3, A.n4, q, pt, w);
        const V3<Dual> v = ad::sub(pi, pt);
        const Dual r = ad::dmax(ad::norm(v), kEps);
        const Dual ndr = ad::dot(ni, v), in1 = ad::dot(t1, v), in2 = ad::dot(t2, v);
        const Dual rr = ad::dmax(r, rfloor);
        const Dual irr3 = Dual(1.0) / (rr * rr * rr);
        const Dual ir = Dual(1.0) / r;
        Dual rp_m1 = ir, rp_m3 = ir * ir * ir, rp_m = Dual(1.0);
        for (int m = 0; m < no; ++m) {
          sg[m] += w * rp_m1;
          s1[m] += w * ndr * rp_m3;
          s2[m] += w * in1 * rp_m * irr3;
          s3[m] += w * in2 * rp_m * irr3;
          rp_m1 *= r;
          rp_m3 *= r;
          rp_m *= r;
        }
      }
      double fact = 1.0;
      for (int m = 0; m < no; ++m) {
        if (m > 0) fact *= m;
        const Dual a = wsumT(sg[m]), b = wsumT(s1[m]), c = wsumT(s2[m]), dd = wsumT(s3[m]);
        // g_m = a / m!;  f_m = n (m-1) b / m! + t1 (m-1) c / m! + t2 (m-1) dd / m!
        const double gd = a.d / fact;
        acc = ca(acc, cs(A.ghat[e * no + m], gd));
        const double cf = (m - 1) / fact;
        const Dual fx = (ni.x * b + t1.x * c + t2.x * dd) * cf;
        const Dual fy = (ni.y * b + t1.y * c + t2.y * dd) * cf;
        const Dual fz = (ni.z * b + t1.z * c + t2.z * dd) * cf;
        acc = ca(acc, cs(A.fhat[(e * 3 + 0) * no + m], fx.d));
        acc = ca(acc, cs(A.fhat[(e * 3 + 1) * no + m], fy.d));
        acc = ca(acc, cs(A.fhat[(e * 3 + 2) * no + m], fz.d));
      }
    } else {
      const V3<Dual> pj = seed3(A.pos + 3 * j, dir, 3);
      const Dual r0 = ad::norm(ad::sub(pj, pi));
      const int nsub = (fk == 1 || fk == 3) ? 2 : 1;
      for (int t = lane; t < nsub * A.n28; t += 32) {
        const int s = t / A.n28, q = t - s * A.n28;
        V3<Dual> pt;
        Dual w;
        ad::tri_pt<Dual>(fc, A.rules, A.n28, s, q, pt, w);
        const V3<Dual> v = ad::sub(pi, pt);
        const Dual r = ad::dmax(ad::norm(v), kEps);
        const Dual ir = Dual(1.0) / r;
        const Dual ir2 = ir * ir, ir3 = ir2 * ir;
        const Dual dl = r - r0;
        Dual dpow = Dual(1.0), dprev = Dual(0.0);
        double fm = 1.0, fm1 = 1.0;
        for (int m = 0; m < no; ++m) {
          sg[m] += w * dpow * ir * (1.0 / fm);
          const Dual fs = (m == 0) ? -ir3 : (-(dpow * ir3) * (1.0 / fm) + dprev * ir2 * (1.0 / fm1));
          s1[m] += w * v.x * fs;
          s2[m] += w * v.y * fs;
          s3[m] += w * v.z * fs;
          dprev = dpow;
          dpow *= dl;
          fm1 = fm;
          fm *= (m + 1);
        }
      }
      for (int m = 0; m < no; ++m) {
        const Dual a = wsumT(sg[m]), b = wsumT(s1[m]), c = wsumT(s2[m]), dd = wsumT(s3[m]);
        acc = ca(acc, cs(A.ghat[e * no + m], a.d));
        acc = ca(acc, cs(A.fhat[(e * 3 + 0) * no + m], b.d));
        acc = ca(acc, cs(A.fhat[(e * 3 + 1) * no + m], c.d));
        acc = ca(acc, cs(A.fhat[(e * 3 + 2) * no + m], dd.d));
      }
    }
    if (lane == 0) {
      double2* dst;
      if (dir < 3)
        dst = &A.gpos[3 * i + dir];
      else if (self && dir < 6)
        dst = &A.gnv[3 * i + dir - 3];
      else if (self && dir < 9)
        dst = &A.gt1[3 * i + dir - 6];
      else if (self && dir < 12)
        dst = &A.gt2[3 * i + dir - 9];
      else if (!self && dir < 6)
        dst = &A.gpos[3 * j + dir - 3];
      else
        dst = &A.gnodes[27LL * j + (dir - nbase)];
      atomic_c(dst, acc);
    }
  }
}

}  // namespace adj
}  // namespace bem200

using namespace bem200;
using namespace bem200::adj;

static size_t al256(size_t b) { return (b + 255) & ~size_t(255); }

extern "C" {

size_t bem200_shape_gradient_workspace_size(int n, int64_t nref, int order) {
  const size_t no = (size_t)order + 1;
  const size_t nr = (size_t)(nref > 0 ? nref : 1);
  return al256(sizeof(double2) * nr * no) + al256(sizeof(double2) * nr * 3 * no) + 2 * al256(sizeof(double2) * n) +
         al256(sizeof(int64_t) * n);
}

int bem200_shape_gradient(int n, int npol, int npart, const int32_t* pid, const int32_t* blk_mat, int nmat,
                          const double* kmat_host, double k0, int eps_per_face, const double* eps1,
                          const double* eps2, const uint64_t* closed_mask, const double* pos, const double* nvec,
                          const double* tvec1, const double* tvec2, const double* area, const double* nodes,
                          const int32_t* face_kind, const double* rules, int n28, int n3, int n4, int64_t nref,
                          const int64_t* ref_row_ptr, const int32_t* ref_row, const int32_t* ref_col,
                          const int8_t* ref_kind, const int64_t* csc_col_ptr, const int32_t* csc_row, int order,
                          const double* g, const double* f, const double* corr, const void* W1, const void* W2,
                          const void* lam, void* grad, void* scratch, void* stream) {
  BEM_REQUIRE(n > 0 && npol > 0 && npart > 0 && pid && blk_mat && closed_mask && pos && nvec && tvec1 && tvec2 &&
                  area && nodes && face_kind && rules && corr && W1 && W2 && lam && grad && scratch && eps1 && eps2,
              BEM200_ERR_ARG, "shape_gradient: bad arguments");
  BEM_REQUIRE(npol <= kMaxPol, BEM200_ERR_UNSUPPORTED, "shape_gradient: at most %d polarisations", kMaxPol);
  BEM_REQUIRE(nmat > 0 && nmat <= kMaxMat && kmat_host, BEM200_ERR_ARG, "shape_gradient: 1 <= nmat <= %d", kMaxMat);
  BEM_REQUIRE(order >= 0 && order <= kMaxOrder, BEM200_ERR_ARG, "shape_gradient: order above %d", kMaxOrder);
  BEM_REQUIRE(nref > 0 && ref_row_ptr && ref_row && ref_col && ref_kind && csc_col_ptr && csc_row && g && f,
              BEM200_ERR_ARG, "shape_gradient: refinement tables missing (every mesh has refined self terms)");
  BEM_REQUIRE(n <= 8 * 48 * 1024 / kWarps, BEM200_ERR_UNSUPPORTED, "shape_gradient: n = %d faces is too many", n);
  cudaStream_t s = (cudaStream_t)stream;
  Args A;
  A.n = n;
  A.npol = npol;
  A.npart = npart;
  A.order = order;
  for (int m = 0; m < kMaxMat; ++m) {
    A.kt.re[m] = m < nmat ? kmat_host[2 * m] : 0.0;
    A.kt.im[m] = m < nmat ? kmat_host[2 * m + 1] : 0.0;
  }
  A.k0 = k0;
  A.eps_per_face = eps_per_face;
  if (eps_per_face) {
    A.e1d = (const double2*)eps1;
    A.e2d = (const double2*)eps2;
    A.e1s = A.e2s = make_double2(0, 0);
  } else {
    A.e1d = A.e2d = nullptr;
    A.e1s = make_double2(eps1[0], eps1[1]);
    A.e2s = make_double2(eps2[0], eps2[1]);
  }
  A.pid = pid;
  A.blk = blk_mat;
  A.closed_mask = closed_mask;
  A.pos = pos;
  A.nvec = nvec;
  A.area = area;
  A.tvec1 = tvec1;
  A.tvec2 = tvec2;
  A.nodes = nodes;
  A.face_kind = face_kind;
  A.rules = rules;
  A.n28 = n28;
  A.n3 = n3;
  A.n4 = n4;
  A.nref = nref;
  A.row_ptr = ref_row_ptr;
  A.ref_row = ref_row;
  A.ref_col = ref_col;
  A.ref_kind = ref_kind;
  A.col_ptr = csc_col_ptr;
  A.csc_row = csc_row;
  A.g = g;
  A.f = f;
  A.corr = corr;
  A.W1 = (const double2*)W1;
  A.W2 = (const double2*)W2;
  A.lam = (const double2*)lam;
  double2* gb = (double2*)grad;
  A.gpos = gb;
  A.gnv = gb + 3 * (size_t)n;
  A.garea = gb + 6 * (size_t)n;
  A.gt1 = gb + 7 * (size_t)n;
  A.gt2 = gb + 10 * (size_t)n;
  A.gnodes = gb + 13 * (size_t)n;
  const size_t no = (size_t)order + 1;
  const size_t nr = (size_t)(nref > 0 ? nref : 1);
  char* p = (char*)scratch;
  A.ghat = (double2*)p;   p += al256(sizeof(double2) * nr * no);
  A.fhat = (double2*)p;   p += al256(sizeof(double2) * nr * 3 * no);
  A.shat = (double2*)p;   p += al256(sizeof(double2) * n);
  A.chat = (double2*)p;   p += al256(sizeof(double2) * n);
  A.diag_e = (int64_t*)p;
  BEM_CUDA_CHECK(cudaMemsetAsync(grad, 0, sizeof(double2) * 40 * (size_t)n, s));
  BEM_CUDA_CHECK(cudaMemsetAsync(A.chat, 0, sizeof(double2) * n, s));
  BEM_CUDA_CHECK(cudaMemsetAsync(A.diag_e, 0xff, sizeof(int64_t) * n, s));  // -1
  refined_op_kernel<<<ceil_div(nref, 128), 128, 0, s>>>(A);
  BEM_LAUNCH_CHECK();
  closed_prep_kernel<<<ceil_div(n, 128), 128, 0, s>>>(A);
  BEM_LAUNCH_CHECK();
  const int smem = kWarps * ((n + 31) / 32) * (int)sizeof(uint32_t);
  BEM_CUDA_CHECK(set_kernel_attrs_once(far_rows_kernel, smem, false));
  BEM_CUDA_CHECK(set_kernel_attrs_once(far_cols_kernel, smem, false));
  far_rows_kernel<<<ceil_div(n, kWarps), 32 * kWarps, smem, s>>>(A);
  BEM_LAUNCH_CHECK();
  far_cols_kernel<<<ceil_div(n, kWarps), 32 * kWarps, smem, s>>>(A);
  BEM_LAUNCH_CHECK();
  refined_closed_kernel<<<ceil_div(nref, 128), 128, 0, s>>>(A);
  BEM_LAUNCH_CHECK();
  refine_coef_grad_kernel<<<ceil_div(nref * 32, 128), 128, 0, s>>>(A);
  BEM_LAUNCH_CHECK();
  return BEM200_OK;
}

}  // extern "C"
