/*
 * bem200 -- C ABI of the B200 retarded-BEM solver library (libbem200.so).
 *
 * Every entry point takes raw device pointers (e.g. torch.Tensor.data_ptr()),
 * sizes and a CUDA stream (cudaStream_t passed as void*; NULL = default
 * stream), enqueues its work on that stream and returns a status code
 * (BEM200_OK = 0).  On failure the message is kept per host thread and read
 * with bem200_last_error().  The caller owns all memory; functions that need
 * scratch space take a workspace pointer whose size is given by the matching
 * *_workspace_size query.  No entry point keeps global mutable state, with
 * one exception: bem200_getrs_noalloc works in a fixed device buffer that the
 * library owns (see its declaration).
 *
 * Matrices are dense, row-major, complex (interleaved re/im), with leading
 * dimension `ld` in elements.  Face arrays are (n, 3) row-major float64.
 *
 * The reference interface each group replaces (MNPBEM Python port v1.6.2):
 *   refinement      -> mnpbem/greenfun/refine_utils.py:29 (refinematrix),
 *                      mnpbem/greenfun/greenret_refined.py:122, :287
 *                      (GreenRetRefined._refine_diagonal/_refine_offdiagonal),
 *                      mnpbem/greenfun/compgreen_ret.py:192, :376 (closed surface)
 *   assembly        -> mnpbem/greenfun/compgreen_ret.py:507 (CompGreenRet.eval)
 *                      and mnpbem/greenfun/greenret_refined.py:654 (eval)
 *   dense BEM       -> mnpbem/bem/bem_ret.py:293 (BEMRet.init), :1569 (solve)
 *   operator        -> mnpbem/bem/bem_ret_iter.py:1362 (BEMRetIter._afun)
 */
#ifndef BEM200_H
#define BEM200_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BEM200_OK 0
#define BEM200_ERR_ARG 1          /* invalid argument (size, pointer, option) */
#define BEM200_ERR_CUDA 2         /* CUDA runtime error */
#define BEM200_ERR_SINGULAR 3     /* exactly singular pivot met in an LU */
#define BEM200_ERR_UNSUPPORTED 4  /* configuration not implemented */
#define BEM200_ERR_TIMEOUT 5      /* a bounded device-side wait gave up */
#define BEM200_ERR_NOCONV 6       /* iterative refinement stopped above its tolerance */
#define BEM200_ERR_PIVOTING 7     /* an LU without row exchanges met a column that needs one */

#define BEM200_C128 0 /* complex double, 16 bytes per element */
#define BEM200_C64 1  /* complex float, 8 bytes per element */

/* Library version (major * 10000 + minor * 100 + patch). */
int bem200_version(void);

/* Number of device kernels this library has launched in this process. */
uint64_t bem200_launch_count(void);

/* Copies the calling thread's last error message into buf (always
 * NUL-terminated when len > 0).  Returns the length of the message. */
int bem200_last_error(char* buf, size_t len);

/* ------------------------------------------------------------------ (a1)
 * Refinement classification of all face pairs (i, j), i, j < n:
 *   kind 2 if the centroids coincide (d == 0), kind 1 if
 *   d - rad[j] < abs_cutoff or (d - rad[j]) / rad[i] < rel_cutoff, else 0,
 * with d from |p_i|^2 + |p_j|^2 - 2 p_i.p_j (values below 1e-10 -> 0).
 * Replaces refinematrix (mnpbem/greenfun/refine_utils.py:29-158).
 * Pass 1 counts refined entries per row; bem200_scan_i32 turns counts into a
 * CSR row pointer; pass 2 writes (row, col, kind) in row-major order. */
int bem200_refine_count(int n, const double* pos, const double* rad, double abs_cutoff,
                        double rel_cutoff, int32_t* row_count, void* stream);
int bem200_scan_i32(int n, const int32_t* count, int64_t* row_ptr /* n + 1 */, void* stream);
int bem200_refine_fill(int n, const double* pos, const double* rad, double abs_cutoff,
                       double rel_cutoff, const int64_t* row_ptr, int32_t* ref_row,
                       int32_t* ref_col, int8_t* ref_kind, void* stream);

/* ------------------------------------------------------------- (a2, a3)
 * Expansion coefficients of the refined entries, order+1 terms each:
 *   g[e][m]     (nref, order+1)      Green function,  G = sum_m g_m (ik)^m
 *   f[e][c][m]  (nref, 3, order+1)   Cartesian derivative, F = n_i . sum_m f_m (ik)^m
 * kind 2 entries use the polar rule on face col (quadpol), kind 1 entries the
 * 28-point rule on the (curved) sub-triangles of face col.
 * nodes (n, 9, 3) and face_kind (n) describe every face:
 *   0 flat triangle (nodes 0-2), 1 flat quad (0-3),
 *   2 curved triangle [v0 v1 v2 e01 e12 e20], 3 curved quad [v0..v3 e01 e12 e23 e30 c].
 * rules = [x28 y28 w28 | x3 y3 w3 | x4 y4 w4] with n28, n3, n4 points.
 * Replaces GreenRetRefined._refine_diagonal / _refine_offdiagonal
 * (mnpbem/greenfun/greenret_refined.py:122-516). */
int bem200_refine_integrals(int64_t nref, const int32_t* ref_row, const int32_t* ref_col,
                            const int8_t* ref_kind, const double* pos, const double* nvec,
                            const double* tvec1, const double* tvec2, const double* area,
                            const double* nodes, const int32_t* face_kind, const double* rules,
                            int n28, int n3, int n4, int order, double* g, double* f,
                            void* stream);

/* ------------------------------------------------------------------ (a4)
 * Closed-surface correction (Fuchs & Liu): for every face j of a particle
 * whose closed surface is the set of particles closed_mask[pid[j]] (bit k =
 * particle k; 0 = not closed)
 *   c_j = -2 pi - sum_{i in surface} area_i F_ij / area_j ,
 * F the quasistatic surface derivative (refined entries use n_i . f_0), and
 * f[e][:, 0] += c_j n_j for the diagonal entry e = (j, j).  c is written to
 * corr (n).  workspace: n doubles.
 * Replaces CompGreenRet._initclosed / _apply_diag_corrections
 * (mnpbem/greenfun/compgreen_ret.py:192-272, :376-400). */
int bem200_closed_correction(int n, int npart, const int32_t* pid, const uint64_t* closed_mask,
                             const double* pos, const double* nvec, const double* area,
                             int64_t nref, const int64_t* row_ptr, const int32_t* ref_row,
                             const int32_t* ref_col, const int8_t* ref_kind, int order,
                             double* f, double* corr, void* stream);

/* fn[e][m] = n_row(e) . f[e][:, m]  (the projection used by F / H1 / H2). */
int bem200_refine_project(int64_t nref, const int32_t* ref_row, const double* nvec, int order,
                          const double* f, double* fn, void* stream);

/* ------------------------------------------------------------------ (a6)
 * Per-wavelength assembly of the four BEM matrices
 *   G1 = G[r00] - G[r10], G2 = G[r11] - G[r01], H1 = H1[r00] - H1[r10],
 *   H2 = H2[r11] - H2[r01],
 * where for particle block (a, b) region pair r connects with material
 * blk_mat[(a * npart + b) * 4 + {0: r00, 1: r10, 2: r11, 3: r01}] (1-based,
 * 0 = not connected) whose wavenumber is kmat_host[2 m], kmat_host[2 m + 1]
 * (HOST array, nmat <= 16 materials).  G = area_j / d e^{ikd},
 * F = (n_i . r)(ik - 1/d) / d^2 area_j e^{ikd}, H1/H2 = F +/- 2 pi on the
 * diagonal of self blocks; refined entries take sum_m c_m (ik)^m e^{ikd}.
 * out_dtype BEM200_C128 or BEM200_C64; any output pointer may be NULL.
 * Replaces CompGreenRet.eval / _eval1 (mnpbem/greenfun/compgreen_ret.py:507,
 * :739-858) and the G1/G2/H1/H2 build of BEMRet.init (bem_ret.py:407-423). */
int bem200_green_assemble(int n, int npart, const int32_t* pid, const int32_t* blk_mat,
                          int nmat, const double* kmat_host, const double* pos,
                          const double* nvec, const double* area, int64_t nref,
                          const int32_t* ref_row, const int32_t* ref_col, int order,
                          const double* g, const double* fn, int out_dtype, void* G1, void* G2,
                          void* H1, void* H2, int64_t ld, void* stream);

/* d/dk of G1, G2, H1, H2 (complex128) for the wavenumber of material dmat
 * (1-based, <= nmat): the region terms filled with that material, far
 * entries dG/dk = i d G, dF/dk = -k d (n.r) area / d^2 e^{ikd}, refined
 * entries i sum_m c_m (m (ik)^(m-1) + d (ik)^m) e^{ikd}.  The tangent of the
 * BEM operator for derivatives with respect to a material's permittivity
 * (no counterpart call in the reference, which has no gradients). */
int bem200_green_assemble_dk(int n, int npart, const int32_t* pid, const int32_t* blk_mat, int nmat,
                             const double* kmat_host, int dmat, const double* pos, const double* nvec,
                             const double* area, int64_t nref, const int32_t* ref_row, const int32_t* ref_col,
                             int order, const double* g, const double* fn, void* G1, void* G2, void* H1, void* H2,
                             int64_t ld, void* stream);

/* ------------------------------------------------------------------ (f4)
 * Cartesian derivatives of the Green function and the potentials / fields of
 * a solution at the faces.  blk, blk0, blk1: (npart x npart) int32 material
 * index (1-based, 0 = not connected) of one region pair per particle block,
 * i.e. con[i][j] of the reference; kmat_host as in bem200_green_assemble.
 *
 * bem200_green_assemble_cart: out (n, 3, n) complex128, out[i][c][j] =
 *   Gp_c = (r_c)(ik - 1/d) / d^2 area_j e^{ikd} (refined pairs:
 *   sum_q f[e][c][q] (ik)^q e^{ikd}), plus (hkey 1: H1p) 2 pi n_i or (hkey 2:
 *   H2p) -2 pi n_i on the diagonal of self blocks (hkey 0: Gp).  f: the
 *   (nref, 3, order+1) coefficients of bem200_refine_integrals after the
 *   closed-surface correction.  Replaces CompGreenRet.eval with keys Gp, H1p,
 *   H2p (mnpbem/greenfun/compgreen_ret.py:811-858,
 *   mnpbem/greenfun/greenret_refined.py:812-864).
 *
 * bem200_green_potential: phi = G0 sig1 + G1 sig2, phip = H0 sig1 + H1 sig2,
 *   a = G0 h1 + G1 h2, ap = H0 h1 + H1 h2, with G0, H0 of region pair blk0 and
 *   G1, H1 of blk1, H the key H1 (hkey 1) or H2 (hkey 2).  sig1, sig2, phi,
 *   phip: (n, npol); h1, h2, a, ap: (n, 3, npol), complex128, device.  The
 *   matrices are never stored: entries are computed on the fly.  ref_row_ptr
 *   (n + 1, int64, NULL = none), ref_col, g, fn: refinement tables in CSR
 *   form.  Replaces CompGreenRet.potential
 *   (mnpbem/greenfun/compgreen_ret.py:976-1038).
 *
 * bem200_green_field: e = i k0 (G0 h1 + G1 h2) - Hp0 sig1 - Hp1 sig2,
 *   h = Hp0 x h1 + Hp1 x h2, Hp the key H1p (hkey 1) or H2p (hkey 2); e, h
 *   (n, 3, npol).  f: (nref, 3, order+1).  Replaces CompGreenRet.field
 *   (mnpbem/greenfun/compgreen_ret.py:912-974).  Both products support
 *   n <= 98304 faces. */
int bem200_green_assemble_cart(int n, int npart, const int32_t* pid, const int32_t* blk, int nmat,
                               const double* kmat_host, const double* pos, const double* nvec, const double* area,
                               int64_t nref, const int32_t* ref_row, const int32_t* ref_col, int order,
                               const double* f, int hkey, void* out, void* stream);
int bem200_green_potential(int n, int npart, const int32_t* pid, const int32_t* blk0, const int32_t* blk1, int nmat,
                           const double* kmat_host, const double* pos, const double* nvec, const double* area,
                           const int64_t* ref_row_ptr, const int32_t* ref_col, int order, const double* g,
                           const double* fn, int hkey, int npol, const void* sig1, const void* sig2, const void* h1,
                           const void* h2, void* phi, void* phip, void* a, void* ap, void* stream);
int bem200_green_field(int n, int npart, const int32_t* pid, const int32_t* blk0, const int32_t* blk1, int nmat,
                       const double* kmat_host, const double* pos, const double* nvec, const double* area,
                       const int64_t* ref_row_ptr, const int32_t* ref_col, int order, const double* g, const double* f,
                       int hkey, double k0, int npol, const void* sig1, const void* sig2, const void* h1,
                       const void* h2, void* e, void* h, void* stream);

/* ------------------------------------------------------------- dense LA
 * Building blocks of the dense BEM (reference: the LU / lu_solve / matmul
 * calls of mnpbem/bem/bem_ret.py:437-523, dispatched through
 * mnpbem/utils/gpu.py:145-279).  dtype BEM200_C128 or BEM200_C64; engine 0 =
 * CUDA cores, 1 = tcgen05 bf16x3 split (complex64 only); 2 is reserved for a
 * tcgen05 TF32 engine that is not built: a product that would run on the
 * tensor cores returns BEM200_ERR_UNSUPPORTED with it.  alpha, beta: HOST
 * pointers to (re, im).
 * ws/ws_bytes: scratch for the tensor-core engines
 * (bem200_gemm_workspace_size), may be NULL/0 for engine 0. */
int bem200_gemm(int dtype, int engine, int m, int n, int k, const double* alpha, const void* A, int64_t lda,
                const void* B, int64_t ldb, const double* beta, void* C, int64_t ldc, void* ws, size_t ws_bytes,
                void* stream);
size_t bem200_gemm_workspace_size(int engine, int m, int n, int k);
/* In-place P A = L U.  Rows are not moved: logical row i of P A (and of L,
 * U) is storage row rowmap[i].  ipiv[k] = logical row exchanged with row k
 * (LAPACK swap sequence, 0-based); *info = first exactly-zero pivot (1-based)
 * or 0.  All arrays are device.
 * Partial pivoting (largest |re|+|im|, first maximum on ties), LAPACK's
 * pivots, for both dtypes.  complex64 multipliers use an approximate
 * reciprocal of |pivot|^2 (last-bit differences from cgetrf's division).
 * *info = -BEM200_ERR_TIMEOUT if a bounded device-side wait of a complex64
 * panel gave up (the factors are then invalid).
 * Replaces the LU factorisations of BEMRet.init (mnpbem/bem/bem_ret.py:437-523,
 * via mnpbem/utils/gpu.py:145).
 * bem200_getrf_ex: flags BEM200_GETRF_TOURNAMENT_PIVOTING = complex64 panels
 * of more than 512 rows choose their 32 pivot rows by tournament pivoting
 * (each CTA of a cluster nominates the pivots of its own rows, one CTA
 * factors the nominees; Grigori, Demmel & Xiang, SIAM J. Matrix Anal. Appl.
 * 32, 2011): one cluster-wide exchange per panel instead of one per column,
 * pivots that may differ from LAPACK's (measured slower than partial
 * pivoting at n = 5768 on B200, so off by default).  BEM200_GETRF_PARTIAL_
 * PIVOTING (the default) is accepted and wins over it.  lookahead_nb = block
 * width of the look-ahead schedule (multiple of 32 in [64, 1024]; 0 = 128). */
#define BEM200_GETRF_PARTIAL_PIVOTING 1
#define BEM200_GETRF_TOURNAMENT_PIVOTING 2
/* BEM200_GETRF_DIAGONAL_PIVOTS: factor without the pivot search (blocked,
 * no row exchanges) and check every column against partial pivoting's choice
 * (|a_ij|_1 <= |a_jj|_1 for all i > j at step j).  A passing matrix gets
 * LAPACK's partial-pivoting factors (ipiv[k] = k, rowmap = identity); a
 * failing one sets *info = -BEM200_ERR_PIVOTING and leaves A unusable, so
 * keep a copy and factor it again without the flag.  Needs ws of
 * bem200_getrf_workspace_size bytes. */
#define BEM200_GETRF_DIAGONAL_PIVOTS 4
int bem200_getrf(int dtype, int engine, int n, void* A, int64_t ld, int32_t* rowmap, int32_t* ipiv,
                 int32_t* info, void* ws, size_t ws_bytes, void* stream);
int bem200_getrf_ex(int dtype, int engine, int n, void* A, int64_t ld, int32_t* rowmap, int32_t* ipiv,
                    int32_t* info, void* ws, size_t ws_bytes, int flags, int lookahead_nb, void* stream);
/* ws of this size lets bem200_getrf run its look-ahead schedule: panels on a
 * high-priority stream, trailing updates on a low-priority one, both forked
 * from and joined back into `stream` (same pivots and factors).  A smaller
 * (or NULL) ws selects the single-stream schedule. */
size_t bem200_getrf_workspace_size(int dtype, int engine, int n);
/* B <- A^-1 B from the getrf factors (nrhs columns, row-major B).  scratch:
 * bem200_getrs_workspace_size bytes.  *status (device int) is set to
 * BEM200_ERR_TIMEOUT if a bounded device-side wait of the blocked triangular
 * solve (nrhs <= 16) gave up; the result is then invalid.  status may be NULL,
 * but then such a timeout is recorded only in the scratch and goes
 * unnoticed: callers that need to detect it pass a status int and read it
 * after the stream completes. */
size_t bem200_getrs_workspace_size(int dtype, int n, int nrhs);
int bem200_getrs(int dtype, int engine, int n, int nrhs, const void* LU, int64_t ld, const int32_t* rowmap,
                 void* B, int64_t ldb, void* ws, size_t ws_bytes, void* scratch, int32_t* status,
                 void* stream);
/* A <- A^-1 in place (n x n, ld = n) without pivoting, for matrices whose
 * partial-pivoting LU exchanges no rows (the retarded BEM's G1, G2, Delta,
 * Sigma mostly): block Schur complement recursion (GEMMs on `engine`) with
 * Gauss-Jordan leaves.  *info (device int32) = 0, or 1 when a leaf pivot is
 * zero or not partial pivoting's choice, or the probe max|A^-1 (A v) - v| <=
 * tol max|v| for a fixed pseudo-random v fails; A is then unusable.
 * scratch: bem200_inverse_nopiv_workspace_size bytes; ws: the GEMM operand
 * workspace (bem200_gemm_workspace_size(engine, n, n, n / 2 + 64)).
 * The launch sequence (~600 kernels at n = 5768) is recorded once per
 * argument set (sizes, pointers, engine, workspace, tol) into a CUDA graph
 * and replayed on `stream` afterwards; inside the caller's own stream capture,
 * or with the environment variable BEM200_NO_GRAPHS set, the kernels are
 * launched directly.
 * Replaces the explicit inverse of BEMRet.init (mnpbem/bem/bem_ret.py:437-523,
 * Delta^-1 via lu_solve with the identity) for the mixed path. */
size_t bem200_inverse_nopiv_workspace_size(int dtype, int n);
int bem200_inverse_nopiv(int dtype, int engine, int n, void* A, int64_t ld, void* ws, size_t ws_bytes, void* scratch,
                         double tol, int32_t* info, void* stream);
/* Same solve as bem200_getrs (CUDA-core engine), for callers that cannot
 * allocate device memory: a host program linking only this library with no
 * device allocator of its own, or a caller whose device memory belongs to
 * another runtime's pool and which must not call cudaMalloc / cudaFree
 * (they synchronise the whole device).  No counterpart in the reference.
 * The scratch comes from one fixed buffer of BEM200_GETRS_NOALLOC_MAX_BYTES
 * in the library's device image (held by every GPU that loads the library
 * until exit); sizes whose scratch (bem200_getrs_workspace_size) is larger
 * are rejected with BEM200_ERR_ARG.  The call allocates nothing.  The first
 * call on a device looks up the buffer's device address (host set-up); make
 * it before any stream capture.  The address is kept per device ordinal for
 * the life of the process: it belongs to the device's primary context and is
 * stale after cudaDeviceReset or under another context on that device, so
 * use this entry point only from the primary context and not across a
 * device reset.  All calls on a GPU share the buffer: calls that overlap on
 * the GPU race, so order them (one stream, or events).  As with
 * bem200_getrs, pass status to detect a timed-out triangular solve. */
#define BEM200_GETRS_NOALLOC_MAX_BYTES (4u << 20)
int bem200_getrs_noalloc(int dtype, int n, int nrhs, const void* LU, int64_t ld, const int32_t* rowmap, void* B,
                         int64_t ldb, int32_t* status, void* stream);

/* ------------------------------------------------------------- dense BEM
 * precision 0 = complex128 throughout (the drop-in FP64 path);
 * precision 1 = mixed: complex64 factors (GEMMs on `engine`) with FP64
 * residuals and iterative refinement (bem200_bem_solve_ir).
 * precision 2 = mixed with explicit complex64 inverses G1^-1, G2^-1,
 * Delta^-1, Sigma^-1 (block Schur complement without pivoting, each checked
 * by a probe M^-1 (M v) = v): every solve and refinement sweep is then a
 * few matrix products.  bem200_bem_init returns BEM200_ERR_PIVOTING when a
 * probe fails; write the slots again and initialise with precision 1.  The
 * same workspace serves precisions 1 and 2; pass the precision the
 * workspace was initialised with to every later call.
 * The workspace (bem200_bem_workspace_size bytes) holds the factors:
 * LU(G1), LU(G2), Sigma1 = H1 G1^-1, LU(Delta), Delta^-1, LU(Sigma) + pivots
 * (precision 2: the inverses in place of the LUs).
 * bem200_bem_slots returns where G1, G2, H1, H2 must be written (dtype of the
 * precision) before bem200_bem_init, which consumes them.
 * eps: eps_per_face = 0 -> eps1/eps2 are HOST (re, im) scalars of the inside /
 * outside media; 1 -> device complex128 arrays (n) per face.
 * Replaces BEMRet.init (mnpbem/bem/bem_ret.py:293-525). */
size_t bem200_bem_workspace_size(int precision, int n);
int bem200_bem_slots(int precision, int n, void* ws, void** G1, void** G2, void** H1, void** H2);
int bem200_bem_init(int precision, int engine, int n, void* ws, int eps_per_face, const double* eps1,
                    const double* eps2, const double* nvec, double k0, void* gemm_ws, size_t gemm_ws_bytes,
                    int32_t* info_host, void* stream);
/* bem200_bem_init with the LU tiling exposed (for the project's autotuner):
 * lu_flags as bem200_getrf_ex's (BEM200_GETRF_TOURNAMENT_PIVOTING: complex64
 * factors with tournament panels; BEM200_GETRF_DIAGONAL_PIVOTS: the four
 * LUs without the pivot search, checked -- the call then returns
 * BEM200_ERR_PIVOTING when one of G1, G2, Delta, Sigma needs row exchanges,
 * and the caller writes the slots again and repeats the call without the
 * flag), lookahead_nb the block width of the
 * look-ahead LU schedule (a multiple of 32 in [64, 1024]; 0 = 128).
 * phase_ms (HOST, 4 floats, or NULL): stage timer (CUDA events on the
 * stream; the call then synchronises): LU(G1) || LU(G2) with Sigma1 || Sigma2,
 * LU(Delta), Delta^-1, Sigma build + LU(Sigma). */
int bem200_bem_init_ex(int precision, int engine, int n, void* ws, int eps_per_face, const double* eps1,
                       const double* eps2, const double* nvec, double k0, void* gemm_ws, size_t gemm_ws_bytes,
                       int lu_flags, int lookahead_nb, float* phase_ms, int32_t* info_host, void* stream);

/* Right-hand side (complex128, row-major, npol polarisations):
 *   b = [phi (n, p) | a (n, 3, p) | alpha (n, 3, p) | De (n, p)]  (8 n p values)
 * solution W1 = [sig1 (n, p) | h1 (n, 3, p)] row-interleaved as n x 4p, W2 the
 * same for (sig2, h2).  Replaces BEMRet.solve (mnpbem/bem/bem_ret.py:1569-1831,
 * Eqs. 19-20 of Garcia de Abajo & Howie, PRB 65, 115418). */
size_t bem200_bem_solve_workspace_size(int precision, int n, int npol);
int bem200_bem_solve(int precision, int engine, int n, int npol, void* ws, const void* phi, const void* a,
                     const void* alpha, const void* De, int eps_per_face, const double* eps1, const double* eps2,
                     const double* nvec, double k0, void* W1, void* W2, void* scratch, void* gemm_ws,
                     size_t gemm_ws_bytes, void* stream);
/* Device status of the factors in ws (0 = fine, BEM200_ERR_TIMEOUT = a bounded
 * wait gave up in the last solve, BEM200_ERR_SINGULAR = zero pivot); copies to
 * *host_status and synchronises the stream. */
int bem200_bem_status(int precision, int n, void* ws, int32_t* host_status, void* stream);

/* Full FP64 BEM operator r = A x (b == NULL) or r = b - A x for x = (W1, W2):
 * phi = G1 s1 - G2 s2, a = G1 h1 - G2 h2, alpha = H1 h1 - H2 h2 - ik n (G1 e1 s1
 * - G2 e2 s2), De = H1 e1 s1 - H2 e2 s2 - ik n.(G1 e1 h1 - G2 e2 h2).
 * Replaces BEMRetIter._afun (mnpbem/bem/bem_ret_iter.py:1362-1501). */
size_t bem200_bem_apply_workspace_size(int n, int npol);
int bem200_bem_apply(int n, int npol, const void* G1, const void* G2, const void* H1, const void* H2,
                     int eps_per_face, const double* eps1, const double* eps2, const double* nvec, double k0,
                     const void* W1, const void* W2, const void* b, void* r, void* scratch, void* stream);

/* Mixed-precision solve: x = M b with the complex64 factors in ws, then
 * x += M (b - A x) with the FP64 operator of G1..H2 (complex128) until
 * max|b - A x| <= tol max|b| or maxit sweeps.  *iters, *relres: HOST outputs.
 * This call synchronises the stream once per sweep to test convergence.
 * Returns BEM200_ERR_NOCONV when the refinement stops above tol: maxit
 * sweeps reached, a residual that is not finite, or a sweep that does not
 * reduce the residual (divergence).  W1, W2, *iters and *relres still hold
 * the last iterate, so a caller can continue (GMRES-IR) or report it.
 * BEM200_ERR_SINGULAR: the factors hold an exactly zero pivot;
 * BEM200_ERR_TIMEOUT: a bounded device wait of a triangular solve gave up. */
int bem200_bem_solve_ir(int engine, int n, int npol, void* ws, const void* G1, const void* G2, const void* H1,
                        const void* H2, const void* b, int eps_per_face, const double* eps1, const double* eps2,
                        const double* nvec, double k0, double tol, int maxit, void* W1, void* W2, void* scratch,
                        void* gemm_ws, size_t gemm_ws_bytes, int32_t* iters, double* relres, void* stream);
/* bem200_bem_solve_ir for a workspace of precision 1 or 2 (bem200_bem_solve_ir
 * is the precision-1 form). */
int bem200_bem_solve_ir_ex(int precision, int engine, int n, int npol, void* ws, const void* G1, const void* G2,
                           const void* H1, const void* H2, const void* b, int eps_per_face, const double* eps1,
                           const double* eps2, const double* nvec, double k0, double tol, int maxit, void* W1,
                           void* W2, void* scratch, void* gemm_ws, size_t gemm_ws_bytes, int32_t* iters,
                           double* relres, void* stream);

/* y = M b: one application of the factors in ws (built by bem200_bem_init)
 * as the preconditioner of the iterative solver.  b: right-hand-side layout,
 * y: solution layout [W1 | W2], both complex128 (8 n p values).  precision 1
 * applies the complex64 factors to b scaled to unit max-norm.  scratch:
 * bem200_bem_solve_workspace_size(precision, n, npol) bytes.  Replaces
 * BEMRetIter._mfun (mnpbem/bem/bem_ret_iter.py:1503-1634). */
int bem200_bem_precond(int precision, int engine, int n, int npol, void* ws, const void* b, int eps_per_face,
                       const double* eps1, const double* eps2, const double* nvec, double k0, void* y,
                       void* scratch, void* gemm_ws, size_t gemm_ws_bytes, void* stream);

/* Transposed solve and operator, for reverse-mode derivatives (one transposed
 * solve gives the gradient of a functional of the solution over every
 * parameter; the reference has no gradients, so these have no counterpart
 * call -- they transpose BEMRet.solve, mnpbem/bem/bem_ret.py:1569-1831, and
 * BEMRetIter._afun, mnpbem/bem/bem_ret_iter.py:1362-1501).  Pairings are
 * bilinear (no conjugation).
 * bem200_bem_solve_T: b = S^T cot with S = the factored solve of
 *   bem200_bem_solve (Eqs. 19-20): cot in the solution layout [W1 | W2]
 *   (8 n p complex128), b in the right-hand-side layout.  Every step of the
 *   solve transposed: transposed LU solves with the factors' row maps,
 *   transposed products with Delta^-1 and Sigma1.  precision 1 applies the
 *   complex64 factors once (to cot scaled to unit max-norm), the transposed
 *   counterpart of bem200_bem_precond; npol <= 4.
 * bem200_bem_apply_T: r = A^T l (w NULL) or r = w - A^T l for the FP64 BEM
 *   operator of bem200_bem_apply; l in the right-hand-side layout, w and r in
 *   the solution layout.  Refining S^T with it gives A^-T to FP64 accuracy. */
size_t bem200_bem_solve_T_workspace_size(int precision, int n, int npol);
int bem200_bem_solve_T(int precision, int engine, int n, int npol, void* ws, const void* cot, int eps_per_face,
                       const double* eps1, const double* eps2, const double* nvec, double k0, void* b, void* scratch,
                       void* stream);
size_t bem200_bem_apply_T_workspace_size(int n, int npol);
int bem200_bem_apply_T(int n, int npol, const void* G1, const void* G2, const void* H1, const void* H2,
                       int eps_per_face, const double* eps1, const double* eps2, const double* nvec, double k0,
                       const void* l, const void* w, void* r, void* scratch, void* stream);

/* bem200_shape_gradient: c = lambda^T (dA/dtheta) x contracted over every face
 * pair at once, for the geometry parameters theta of all faces: grad
 * (complex128, 40 n) = pos (n, 3) | nvec (n, 3) | area (n) | tvec1 (n, 3) |
 * tvec2 (n, 3) | face nodes (n, 9, 3).  x = (W1, W2) is the solution, lam
 * the adjoint (right-hand-side layout, e.g. from bem200_bem_solve_T), npol <=
 * 4.  Far pairs are differentiated analytically and swept by rows and by
 * columns without storing any n x n matrix; refined pairs through their
 * phase, normals and coefficients, whose derivatives with respect to the
 * face nodes and the observation frame are exact (forward-mode dual numbers
 * over the refinement quadrature); the closed-surface correction is chained
 * through its column sums.  Inputs: the assembly tables of
 * bem200_green_assemble (pid, blk_mat, kmat_host), the refinement inputs of
 * bem200_refine_integrals (nodes, face_kind, rules), the refinement tables in
 * CSR form (ref_row_ptr) and by column (csc_col_ptr (n + 1), csc_row), the
 * coefficients g and f after the closed-surface correction, corr (n) and
 * closed_mask of bem200_closed_correction.  No counterpart in the reference
 * (which has no gradients); it differentiates the assembly of
 * mnpbem/greenfun/greenret_refined.py:654-867 and compgreen_ret.py:192-400
 * within the operator of mnpbem/bem/bem_ret_iter.py:1362-1501. */
size_t bem200_shape_gradient_workspace_size(int n, int64_t nref, int order);
int bem200_shape_gradient(int n, int npol, int npart, const int32_t* pid, const int32_t* blk_mat, int nmat,
                          const double* kmat_host, double k0, int eps_per_face, const double* eps1,
                          const double* eps2, const uint64_t* closed_mask, const double* pos, const double* nvec,
                          const double* tvec1, const double* tvec2, const double* area, const double* nodes,
                          const int32_t* face_kind, const double* rules, int n28, int n3, int n4, int64_t nref,
                          const int64_t* ref_row_ptr, const int32_t* ref_row, const int32_t* ref_col,
                          const int8_t* ref_kind, const int64_t* csc_col_ptr, const int32_t* csc_row, int order,
                          const double* g, const double* f, const double* corr, const void* W1, const void* W2,
                          const void* lam, void* grad, void* scratch, void* stream);

/* x = the right-hand side b relabelled into the solution layout (phi -> sig1,
 * a -> h1, De -> sig2, alpha -> h2): the M = I "preconditioner" of the
 * unpreconditioned iteration, which pairs the two spaces as the reference's
 * packed vectors do (mnpbem/bem/bem_ret_iter.py:1196-1233). */
int bem200_bem_relabel(int n, int npol, const void* b, void* x, void* stream);

/* The two ends of the FP64 operator for operators whose four products are
 * computed elsewhere (the H-matrix path): U = [s | h | e s | e h] (n x 8p)
 * from W = [s | h] (n x 4p) with the eps of side `second` (0: eps1, 1: eps2),
 * and r = A x (b NULL) or b - A x from GU1 = G1 U1, GU2 = G2 U2, HU1 = H1 U1,
 * HU2 = H2 U2 (each n x 8p).  Replaces BEMRetIter._afun
 * (mnpbem/bem/bem_ret_iter.py:1362-1501). */
int bem200_op_prep(int n, int npol, const void* W, int eps_per_face, const double* eps1, const double* eps2,
                   int second, void* U, void* stream);
int bem200_op_combine(int n, int npol, const void* GU1, const void* GU2, const void* HU1, const void* HU2,
                      const double* nvec, double k0, const void* b, void* r, void* stream);

/* ------------------------------------------------------------- H-matrix
 * complex128 H-matrices in cluster order (reference HMatrix,
 * mnpbem/greenfun/hmatrix.py:94-541).  Blocks are (r0, m, c0, nb) int32
 * quadruples.  Dense block b is packed at D + doff[b] (m x nb row-major);
 * low-rank block b stores U (m x kcap[b]) at U + uoff[b] and V (nb x kcap[b])
 * at V + voff[b], row-major, block ~ U[:, :rank] V[:, :rank]^T.
 * bem200_hmat_permute: dst[i][j] = src[c2p[i]][c2p[j]] (n x n).
 * bem200_hmat_gather_rows: dst[i, :] = src[idx[i], :] (n x w).
 * bem200_hmat_aca: partially pivoted ACA of every low-rank block from the
 *   cluster-ordered dense matrix Mc (ld n), stopping when the new rank-1 term
 *   drops below htol times the Frobenius estimate or at rank kcap[b]
 *   (reference HMatrix._aca_block, hmatrix.py:195-336); rank[b] on the device.
 *   max_rows >= every m and nb, max_kcap >= every kcap.
 * bem200_hmat_matvec: y = H x for n x w (w <= 16) row-major x, y; T holds
 *   sum_b kcap[b] x w complex (toff[b] = prefix sum of kcap).  Block rows are
 *   added into y with atomics, so the summation order (and the last bits of
 *   y) can vary between calls (reference mtimes_vec, hmatrix.py:450-541). */
int bem200_hmat_permute(int n, const void* src, const int32_t* c2p, void* dst, void* stream);
int bem200_hmat_gather_rows(int n, int w, const void* src, const int32_t* idx, void* dst, void* stream);
int bem200_hmat_pack_dense(int nd, const int32_t* dblk, const int64_t* doff, int n, const void* Mc, void* D,
                           void* stream);
int bem200_hmat_aca(int nl, const int32_t* lblk, const int64_t* uoff, const int64_t* voff, const int32_t* kcap,
                    int n, const void* Mc, double htol, void* U, void* V, int32_t* rank, int max_rows,
                    int max_kcap, void* stream);
int bem200_hmat_matvec(int n, int w, const void* x, int nl, const int32_t* lblk, const int64_t* voff,
                       const int64_t* uoff, const int64_t* toff, const int32_t* kcap, const int32_t* rank,
                       const void* U, const void* V, void* T, int nd, const int32_t* dblk, const int64_t* doff,
                       const void* D, void* y, void* stream);

/* bem200_hmat_matvec_items: y = H x like bem200_hmat_matvec, with large blocks
 * split over several CTAs by host-built work items: vitems (l, j0) pairs
 * cover rows [j0, j0 + 128) of V_l (every low-rank block, all its rows;
 * partial V^T x added into T, which is zeroed: t_len = sum kcap x w complex),
 * bitems (b, i0) pairs cover rows [i0, i0 + 32) of block b (b < nd: dense
 * block b, else low-rank block b - nd; every row of every block). */
int bem200_hmat_matvec_items(int n, int w, const void* x, int nl, const int32_t* lblk, const int64_t* voff,
                             const int64_t* uoff, const int64_t* toff, const int32_t* kcap, const int32_t* rank,
                             const void* U, const void* V, void* T, int64_t t_len, int nd, const int32_t* dblk,
                             const int64_t* doff, const void* D, int nvitems, const int32_t* vitems, int nbitems,
                             const int32_t* bitems, void* y, void* stream);

/* bem200_hmat_compress_green: the dense leaves and the ACA of the low-rank
 * blocks of BEM matrix `which` (0 = G1, 1 = G2, 2 = H1, 3 = H2) with every
 * entry computed on demand from the Green function, so no n x n matrix is
 * stored: rows and columns of a block come from the face arrays (pos, nvec,
 * area), the region table (pid, blk_mat, kmat as in bem200_green_assemble)
 * and the refinement tables in CSR form (ref_row_ptr (n + 1) int64, ref_col,
 * g, fn; ref_row_ptr NULL = no refined pairs).  Block indices are in cluster
 * order; c2p maps them to faces.  Entries equal those of
 * bem200_green_assemble; the ACA is that of bem200_hmat_aca.  Replaces the
 * reference's densify-then-compress fill (ACACompGreenRet,
 * mnpbem/greenfun/aca_compgreen_ret.py:184-208) with the on-demand rows and
 * columns of the MEX library (mex/acagreen/acagreen.cpp:83-149). */
int bem200_hmat_compress_green(int which, int n, int npart, const int32_t* pid, const int32_t* blk_mat, int nmat,
                               const double* kmat_host, const double* pos, const double* nvec, const double* area,
                               const int64_t* ref_row_ptr, const int32_t* ref_col, int order, const double* g,
                               const double* fn, const int32_t* c2p, int nd, const int32_t* dblk,
                               const int64_t* doff, void* D, int nl, const int32_t* lblk, const int64_t* uoff,
                               const int64_t* voff, const int32_t* kcap, double htol, void* U, void* V,
                               int32_t* rank, int max_rows, int max_kcap, void* stream);

/* ------------------------------------------------------------- Krylov
 * Kernels of the restarted GMRES of the iterative solver (complex128), which
 * replaces scipy.sparse.linalg.gmres as driven by BEMIter._iter_solve
 * (mnpbem/bem/bem_iter.py:45-101).  A basis is m vectors of length len stored
 * one after the other.
 * bem200_gmres_orth: orthogonalise the vector after V_0..V_j against them
 * (classical Gram-Schmidt, two passes; j = -1: none), normalise it, and
 * return on the HOST
 * h[2 i], h[2 i + 1] = <V_i, w> (i <= j) and h[2 j + 2] = ||w|| before
 * normalisation; synchronises the stream.
 * bem200_gmres_combine: z = sum_{i < m} y_i V_i, y complex on the HOST.
 * bem200_zaxpy: y += a x, a = (re, im) on the HOST. */
size_t bem200_gmres_orth_workspace_size(int j);
int bem200_gmres_orth(int64_t len, int j, void* V, double* h_host, void* scratch, void* stream);
int bem200_gmres_combine(int64_t len, int m, const void* V, const double* y_host, void* z, void* scratch,
                         void* stream);
int bem200_zaxpy(int64_t len, const double* a, const void* x, void* y, void* stream);

/* ------------------------------------------------------------- plane wave
 * bem200_planewave_rhs: the right-hand side b (8 n p complex128, layout of
 * bem200_bem_solve) of p <= 8 plane waves exp(i km dir.r) with polarisations
 * pol (HOST arrays, p x 3), km = (re, im) the wavenumber of the embedding
 * medium (HOST); on_side (n x 2 int8) marks the face sides that touch the
 * medium.  Replaces PlaneWaveRet.potential
 * (mnpbem/simulation/planewave_ret.py:257-361) followed by BEMRet._excitation
 * (mnpbem/bem/bem_ret.py:1360-1429).
 * bem200_farfield: e, h (ndir x 3 x p complex128) far-field amplitudes on the
 * directions dirs (ndir x 3, device) from W1 = [sig1 | h1], W2 = [sig2 | h2]
 * (n x 4p); p <= 4.  Replaces SpectrumRet.farfield
 * (mnpbem/spectrum/spectrum_ret.py:231-392). */
int bem200_planewave_rhs(int n, int npol, const double* pos, const double* nvec, const int8_t* on_side,
                         const double* pol_host, const double* dir_host, const double* km_host, double k0,
                         int eps_per_face, const double* eps1, const double* eps2, void* b, void* stream);
int bem200_farfield(int n, int npol, int ndir, const double* dirs, const double* pos, const double* area,
                    const int8_t* on_side, const double* km_host, double k0, const void* W1, const void* W2,
                    void* e_out, void* h_out, void* stream);

/* dst (complex64) = src (complex128), count elements. */
int bem200_convert_c128_c64(int64_t count, const void* src, void* dst, void* stream);

#ifdef __cplusplus
}
#endif
#endif /* BEM200_H */
