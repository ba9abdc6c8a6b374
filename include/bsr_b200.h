/*
 * bsr_b200.h -- C ABI of the B200 (sm_100a) implementation of the BSR radial,
 * assembly and eigensolve hot path.
 *
 * Every entry point returns an int status (BSRG_OK = 0, negative on error) and
 * never terminates the process; bsrg_last_error() gives the message of the
 * last failure on the calling thread.  Array arguments keep the layouts of the
 * reference's Fortran arrays (column-major, the first index fastest), so a
 * Fortran ISO_C_BINDING shim can pass its module arrays through unchanged.
 * Unless an argument says "host", pointers are device pointers and the call is
 * asynchronous on the given stream (a cudaStream_t passed as void*; NULL is
 * the legacy default stream).  Memory passed in is owned by the caller; the
 * library never frees it.
 *
 * Each declaration cites the reference routine it stands behind (paths within
 * the jagot/bsr tree).
 */
#ifndef BSR_B200_H
#define BSR_B200_H

#include <stddef.h>

#ifdef __cplusplus
extern "C" {
#endif

#define BSRG_OK            0
#define BSRG_ERR_ARG      -1   /* bad argument (the reference's Stop on a range check) */
#define BSRG_ERR_CUDA     -2   /* CUDA runtime error */
#define BSRG_ERR_SOLVER   -3   /* cuSOLVER / cuBLAS error */
#define BSRG_ERR_INFO     -4   /* factorisation failed (LAPACK info /= 0 in the reference) */
#define BSRG_ERR_NOMEM    -5   /* device allocation failed */
#define BSRG_ERR_CASE     -6   /* unknown convol / SUM_AmB case */

typedef struct bsrg_basis bsrg_basis;   /* device-resident B-spline basis */
typedef struct bsrg_ctx bsrg_ctx;       /* stream + solver handles + workspace */

const char *bsrg_last_error(void);
int bsrg_version(void);

/* ---- knot grid: src/libs/BS/define_grid.f90:86 (mkgrid, grid_type 0) and
 *      :213 (mkgrid1, grid_type 1).  Host only.  t (host) must hold cap
 *      doubles; returns ns, ml, me and the adjusted h of spline_param. */
int bsrg_mkgrid(int grid_type, int ks, double z, double h, double hmax, double rmax,
                double *t, int cap, int *ns, int *ml, int *me, double *h_out);

/* ---- basis: src/libs/BS/define_spline.f90:15 (define_spline: initvb :67,
 *      initas :133, mdb1 :184, mdb2 :214, mrm.f90:2).  t is a host array of
 *      ns+ks knots; ml, me, h are spline_param's (me > 0 enables the
 *      scaling-law shortcut of moments.f90:45-61 and rk_moments.f90:74-91). */
int bsrg_define_spline(int ks, int ns, const double *t_host, int ml, int me, double h,
                       void *stream, bsrg_basis **out);
int bsrg_basis_free(bsrg_basis *b);
/* dims[0..4] = ks, ns, nv, ml, me (host) */
int bsrg_basis_dims(const bsrg_basis *b, int *dims);
/* Copy one module array to dst (device).  which: 0 gr, 1 grm, 2 grw (nv,ks);
 * 3 bsp, 4 bsq (nv+1,ks,ks); 5 bspd (nv+1,ks,ks,2); 6 sb, 7 r1, 8 rm1, 9 rm2,
 * 10 rm3, 11 db1, 12 db2 (ns,ks); 13 t (ns+ks); 14 bb (ns,ns), the full
 * overlap matrix of initas (define_spline.f90:171, Full_mat_sym); 15 bs
 * (ks,ns), facsb's banded Cholesky factor of the overlap with the r = 0
 * boundary condition (facsb.f90:2-36, DPBTRF('U') layout; BSRG_ERR_INFO with
 * the reference's message if it is not positive definite). */
int bsrg_basis_get(const bsrg_basis *b, int which, double *dst, void *stream);
/* src/libs/BS/mrm.f90:2: <B_i|r^mm|B_j> band (ns,ks) into rm (device). */
int bsrg_mrm(const bsrg_basis *b, int mm, double *rm, void *stream);

/* ---- R^k cell moments: src/libs/BS/rk_moments.f90:2 (moments.f90:2 for
 *      rkd1 = <B_i|r^k|B_j>, rkd2 = <B_i|r^-(k+1)|B_j> per interval, packed
 *      ik = ks(ks+1)/2 pairs; rk_triang :105 for the diagonal cells).
 *      rkd1, rkd2: (ik, nv); rkd: (ik, ik, nv).  Device. */
int bsrg_rk_moments(const bsrg_basis *b, int k, double *rkd1, double *rkd2, double *rkd, void *stream);

/* ---- R^k B-spline integral table: src/libs/BS/mrk_cell.f90:2.
 *      rkb(i,j,ip,jp) = R^k(B_i B_j; B_{i+ip-1} B_{j+jp-1}), stored as
 *      (ns, ns, ldp, ldp) with ldp >= ks (the reference's module array uses
 *      ldp = 2ks-1); entries with ip or jp > ks are zero.  Device.  The
 *      moments are computed into scratch that the call allocates and frees. */
int bsrg_mrk_cell(const bsrg_basis *b, int k, double *rkb, int ldp, void *stream);
/* Same, from moments already computed by bsrg_rk_moments (no allocation). */
int bsrg_mrk_cell_from_moments(const bsrg_basis *b, const double *rkd1, const double *rkd2,
                               const double *rkd, double *rkb, int ldp, void *stream);
/* ---- Breit-Pauli N^k cell moments: src/libs/BS/nk_moments.f90:2 (moments
 *      rkd1 = <B_i|r^k|B_j>, rkd2 = <B_i|r^-(k+3)|B_j>; nk_triang :105 for the
 *      diagonal cells, the r2 < r1 triangle only).  k >= -1.  Layouts as for
 *      bsrg_rk_moments.  Device. */
int bsrg_nk_moments(const bsrg_basis *b, int k, double *rkd1, double *rkd2, double *rkd, void *stream);

/* ---- N^k B-spline integral table: src/libs/BS/mnk_cell.f90:2.
 *      rkb(i,j,ip,jp) = fine * N^k(B_i B_j; B_{i+ip-1} B_{j+jp-1}) over r2 < r1,
 *      with i, ip the r1 splines (cells jv <= iv only, not symmetric);
 *      layout as bsrg_mrk_cell.  fine is spline_atomic's `fine`
 *      (0.25/137.036^2 in the reference; its TEST_BS harness sets 1).  The
 *      moments go to scratch the call allocates and frees.  Device. */
int bsrg_mnk_cell(const bsrg_basis *b, int k, double fine, double *rkb, int ldp, void *stream);

/* ---- Breit-Pauli M^k: src/libs/BS/mk_moments.f90:2 (the N^k moments, the
 *      diagonal cells symmetrised a + a^T as mk_triang :96 does) and
 *      mmk_cell.f90:2 (mrk_cell's symmetric cell sums, times fine).
 *      Layouts and fine as for the N^k calls.  Device. */
int bsrg_mk_moments(const bsrg_basis *b, int k, double *rkd1, double *rkd2, double *rkd, void *stream);
int bsrg_mmk_cell(const bsrg_basis *b, int k, double fine, double *rkb, int ldp, void *stream);

/* ---- Breit-Pauli T^k: src/libs/BS/tk_moments.f90:2 (moments k and -(k+1)
 *      of all ks*ks spline pairs with the derivative operator, 'n','d'; the
 *      diagonal cells of tk_triang :101 symmetrised) and mtk_cell.f90:2
 *      (rkb(i,j,ip,jp) with ip = ihp - ih + ks, i.e. (ns, ns, ldp, ldp),
 *      ldp >= 2ks-1; times fine/(2k+1)).  rkd1, rkd2: (ks*ks, nv); rkd:
 *      (ks*ks, ks*ks, nv).  k >= 0.  Device. */
int bsrg_tk_moments(const bsrg_basis *b, int k, double *rkd1, double *rkd2, double *rkd, void *stream);
int bsrg_mtk_cell(const bsrg_basis *b, int k, double fine, double *rkb, int ldp, void *stream);

/* ---- Breit-Pauli V^k: src/libs/BS/vk_moments.f90:2 (rkd1 = moments k+1 and
 *      rkd2 = moments -(k+2) of the ik symmetric pairs; rkd3 = moments k and
 *      rkd4 = moments -(k+3) of all ks*ks pairs with the derivative operator;
 *      diagonal cells rkd (ks*ks, ik, nv) from vk_triang :131) and
 *      mvk_cell.f90:2 (rkb(i,j,ip,jp) with ip = ihp - ih + ks over all pairs,
 *      jp = jhp - jh + 1; (ns, ns, ldp, ldp), ldp >= 2ks-1; times fine).
 *      k >= 0.  Device. */
int bsrg_vk_moments(const bsrg_basis *b, int k, double *rkd1, double *rkd2, double *rkd3, double *rkd4, double *rkd,
                    void *stream);
int bsrg_mvk_cell(const bsrg_basis *b, int k, double fine, double *rkb, int ldp, void *stream);

/* ---- Breit-Pauli W^k: src/libs/BS/wk_moments.f90:2 (the V^k layouts with
 *      rkd3 = 2 m(k,'n','d') + (k+2) m(k-1,'n','b'), rkd4 = 2 m(-(k+3),'n','d')
 *      - (k+1) m(-(k+4),'n','b'), and wk_triang's operators 2 dB/dr + k B/r and
 *      2 dB/dr - (k+3) B/r) and mwk_cell.f90:2 (mvk_cell's sums, times fine).
 *      Layouts as for V^k.  k >= 0.  Device. */
int bsrg_wk_moments(const bsrg_basis *b, int k, double *rkd1, double *rkd2, double *rkd3, double *rkd4, double *rkd,
                    void *stream);
int bsrg_mwk_cell(const bsrg_basis *b, int k, double fine, double *rkb, int ldp, void *stream);

/* ---- Breit-Pauli Q^k: src/libs/BS/qk_moments.f90:2 (W^k's moments with rkd1,
 *      rkd2 over all ks*ks pairs; diagonal cells rkd (ks*ks, ks*ks, nv)) and
 *      mqk_cell.f90:2 (every cell term added to rkb(i,j,ip,jp) and subtracted
 *      from rkb(j,i,jp,ip), in the reference's order; times fine).  rkb
 *      (ns, ns, ldp, ldp), ldp >= 2ks-1.  k >= 0.  Device. */
int bsrg_qk_moments(const bsrg_basis *b, int k, double *rkd1, double *rkd2, double *rkd3, double *rkd4, double *rkd,
                    void *stream);
int bsrg_mqk_cell(const bsrg_basis *b, int k, double fine, double *rkb, int ldp, void *stream);

/* ---- No counterpart in the reference.  bsrg_mrk_cell for callers that must
 *      not allocate device memory while they run (a serving process that has
 *      split all of its HBM among its solves at start-up; loops that cannot
 *      afford the device-wide stall a cudaMalloc/cudaFree may cause).  The
 *      interval moments go to a static device array inside the library
 *      (BSRG_NOALLOC_SCRATCH_DOUBLES doubles = 6 MiB, held by every GPU that
 *      loads the library until exit), so the call allocates nothing.  Limit:
 *      (2*ik + ik*ik)*nv <= BSRG_NOALLOC_SCRATCH_DOUBLES with ik = ks(ks+1)/2
 *      (ks = 10: nv <= 250; ks = 8: nv <= 574); larger bases get BSRG_ERR_ARG.
 *      The first call on a device looks up the array's device address and
 *      should come before any stream capture on that device; the call runs on
 *      the basis's device (switched to and back if another is current), and
 *      calls after a cudaDeviceReset of that device are not supported.  Calls
 *      share the array: calls that overlap on the GPU race and must be
 *      serialised. */
#define BSRG_NOALLOC_SCRATCH_DOUBLES 786432
int bsrg_mrk_cell_noalloc(const bsrg_basis *b, int k, double *rkb, int ldp, void *stream);

/* ---- src/libs/BS/density.f90:2.  type 's' -> d (ns,ks); 'n' -> (ns,2ks-1);
 *      'x' -> (ns,ns).  Device. */
int bsrg_density(int ns, int ks, double *d, const double *p1, const double *p2, char type, void *stream);

/* ---- src/libs/BS/convol.f90:2.  a (ns, *) receives the contraction of rkb
 *      (ns,ns,ldp,ldp) with d over electron 2 (icase 1), electron 1 (icase 2),
 *      or the exchange pairings (icase 3, 4; a is then a full (ns,ns) matrix).
 *      sym_i/sym_j in {'s','n'}; 'n' needs ldp >= 2ks-1.  Device. */
int bsrg_convol(int ns, int ks, double *a, const double *d, const double *rkb, int ldp,
                int icase, char sym_i, char sym_j, void *stream);

/* ---- src/libs/BS/bav.f90:2: y = B v (type 's', or 'n' with side 'r') or
 *      y = v B ('n', side 'l') for a band matrix b (ns, ks) ('s') or
 *      (ns, 2ks-1) ('n'), in the reference's summation order.  Device. */
int bsrg_bav(int ns, int ks, const double *b, const double *v, double *y, char type, char side, void *stream);

/* ---- src/libs/BS/bvmv.f90:2: *out = <x, A y> for the band array ar (n, k)
 *      ('s', 'a') or (n, 2k-1) ('g'), in the reference's summation order.
 *      Device (out: one double). */
int bsrg_bvmv(int n, int k, const double *ar, char type, const double *x, const double *y, double *out,
              void *stream);

/* ---- src/libs/BS/quadr.f90:2: *out = <p1 | r^m | p2> (bvmv with sb, r1,
 *      rm1, rm2 or mrm(m)).  p1, p2 (ns) and out (one double) device. */
int bsrg_quadr(const bsrg_basis *b, const double *p1, const double *p2, int m, double *out, void *stream);

/* ---- src/libs/BS/sum_amb.f90:2.  *out (device, one double) = SUM(a*b) over
 *      the storage mode sym in {'s','l','n','x'}. */
int bsrg_sum_amb(int ns, int ks, const double *a, const double *b, char sym, double *out, void *stream);

/* ---- context: stream, cuBLAS/cuSOLVER handles and a growable workspace. */
int bsrg_ctx_create(int device, void *stream, bsrg_ctx **out);
int bsrg_ctx_destroy(bsrg_ctx *c);
/* bytes of device workspace the context currently holds */
size_t bsrg_ctx_workspace_bytes(const bsrg_ctx *c);
/* Stage timing (the reference's per-stage CPU_time lines in mat_log / bsr_hd
 * logs, sub1.f90:68-202): when on, the assembly and diagonalisation calls
 * bracket each stage with CUDA events on the context stream and add the
 * elapsed device time to per-stage totals; bsrg_ctx_stage_times copies the
 * BSRG_NSTAGE totals (ms) and the counts of this library's own kernel launches
 * (library calls such as cuSOLVER's are timed but not counted), then resets
 * them.  Stages: 0 R^k cell moments, 1 direct groups, 2 exchange groups,
 * 3 one-electron / overlap / symmetrisation, 4 channel eigenproblems,
 * 5 block transforms, 6 dense eigensolve, 7 rkb expansion (mrk_cell),
 * 8 eigenpair refinement, and inside stage 6 when the library's own
 * eigensolver runs: 9 dense -> band, 10 band -> tridiagonal, 11 divide and
 * conquer, 12 stage-2 back-transformation, 13 stage-1 back-transformation.
 * bsrg_ctx_stage_flops copies (then resets) the floating-point operations the
 * library's kernels executed per stage where it counts them (block transforms,
 * the own eigensolver's stages, the refinement; 0 elsewhere). */
#define BSRG_NSTAGE 14
int bsrg_ctx_set_timing(bsrg_ctx *c, int on);
int bsrg_ctx_stage_times(bsrg_ctx *c, double *ms, int *launches, int n);
int bsrg_ctx_stage_flops(bsrg_ctx *c, double *flops, int n);

/* ---- resident R^k tables (the reference keeps one multipole's rkb in module
 *      memory, mrk_cell.f90:34-35; a serving process keeps all of them): the
 *      tables of k = 0..kmax for basis b, built once on the context's stream
 *      and kept on the device.  A context told to use them
 *      (bsrg_ctx_use_tables; NULL stops) skips the per-call table builds in
 *      bsrg_assemble / bsrg_add_two_electron for that basis.  The tables must
 *      outlive their use; several contexts may share one set. */
typedef struct bsrg_tables bsrg_tables;
int bsrg_tables_create(bsrg_ctx *c, const bsrg_basis *b, int kmax, bsrg_tables **out);
int bsrg_tables_free(bsrg_tables *t);
size_t bsrg_tables_bytes(const bsrg_tables *t);
int bsrg_ctx_use_tables(bsrg_ctx *c, const bsrg_tables *t);

/* ---- channel-block assembly of one partial wave (bsr_mat):
 *      src/bsr/BSR_MAT3/sub1.f90:72-191 (SUB1), L_data.f90:131-150 and
 *      l_core.f90:174-270 (one-electron block -1/2*hl_core, no closed shells),
 *      I_data.f90:192-218 (Case 6..9 two-electron groups: density ->
 *      convol -> UPDATE_HX), mod_intmat.f90:69,131,245 (UPDATE_HX/HL/CF).
 *
 *      H  = blockdiag(-1/2 hl_{l_ch} + E_ch sb) + sum over coefficient groups,
 *      hcc (device) has nch(nch+1)/2 blocks of (ns,ns), block ij = i(i-1)/2+j
 *      (1-based, i >= j), diagonal blocks symmetrised as in SUB1.
 *      Coefficient records (host arrays, ncoef long) are sorted by
 *      (k, type, ich, jch) exactly like the cmdata blocks of State_res:
 *        ck    multipole 0..kmax
 *        ctype 0 = direct  Rk(i . j .) (I_data jtype 6, jcase 1)
 *              1 = exchange Rk(i . . j) (I_data jtype 8, jcase 3)
 *        cich, cjch 1-based channels with cich >= cjch
 *        ca, cb 0-based orbital columns of P (ns, norb) (device)
 *        cval the angular coefficient
 *      lch, ech: host arrays of channel l and target energy (EC = 0).
 *      acf (device, (nch,nch,kmax+1)) or NULL receives UPDATE_CF's sums.
 *      scc (device) or NULL receives the overlap blocks blockdiag(sb). */
int bsrg_assemble(bsrg_ctx *c, const bsrg_basis *b, double z, int nch, const int *lch, const double *ech,
                  int norb, const double *P, int kmax, int ncoef, const int *ck, const int *ctype,
                  const int *cich, const int *cjch, const int *ca, const int *cb, const double *cval,
                  double *hcc, double *scc, double *acf);

/* ---- src/bsr/BSR_MAT3/I_data.f90:192-218 alone (I_data Case 6..9 for the
 *      Coulomb R^k integrals, icase 5): accumulates the two-electron groups into
 *      the caller's hcc blocks and, for direct groups, into acf (UPDATE_CF),
 *      without touching anything else -- the drop-in for the I_data call of
 *      State_res.  Records as for bsrg_assemble; jtype 6 and 7 records go in as
 *      type 0 and jtype 8 and 9 as type 1 (for the symmetric R^k table convol
 *      icase 2 equals icase 1 and icase 4 equals icase 3).  acf may be NULL. */
int bsrg_add_two_electron(bsrg_ctx *c, const bsrg_basis *b, int nch, int norb, const double *P, int kmax,
                          int ncoef, const int *ck, const int *ctype, const int *cich, const int *cjch,
                          const int *ca, const int *cb, const double *cval, double *hcc, double *acf);

/* ---- src/bsr/BSR_HD3/diag_hd.f90:2-340 for a block-diagonal S (diag_ovl /= 0):
 *      per-channel DSYGV on the diagonal blocks with the first l+1 splines
 *      dropped (:82-111), Egap/Edmax filter, transform of the off-diagonal
 *      blocks to the channel eigenbasis (:188-219), DSYEV('V','L') of the
 *      khm x khm matrix (:312).
 *      hcc (device) as written by bsrg_assemble; sb blocks are taken from b.
 *      lch (host).  eval (device) must hold nch*ns doubles; *khm (host) gets
 *      the dimension.  vecs (device, khm*khm, may be NULL): eigenvectors in the
 *      channel eigenbasis (the reference's a(:,:) after DSYEV); bb (device,
 *      (ns, nch*ns), may be NULL): the channel eigenbasis, columns packed.
 *      want_vectors = 0 computes eigenvalues only.
 *      With eigenvectors, and unless bsrg_ctx_set_refine turned it off, every
 *      eigenvalue is then refined in FP64 by its Rayleigh quotient,
 *      lambda + v^T (A v - lambda v) / v^T v (no counterpart in the reference:
 *      DSYEV's eigenvalues carry errors ~eps ||A||, ~1e-9 absolute when the
 *      kinetic entries reach 1e7; the quotient's error scales with
 *      |v|^T |A| |v|, which makes the eigenvalues agree per eigenvalue).  The
 *      eigenvalues stay ascending (pairs closer than the correction swap with
 *      their vectors). */
int bsrg_diag_hd(bsrg_ctx *c, const bsrg_basis *b, int nch, const int *lch, const double *hcc,
                 int itype, int ilzero, int ibzero, double edmax, double egap, int want_vectors,
                 double *eval, int *khm, double *vecs, double *bb);

/* ---- src/bsr/BSR_HD3/diag_hd.f90:2-340 for an overlap with channel-channel
 *      blocks (diag_ovl = 0, "GENERALIZED eigenvalue problem", :66-69): as
 *      bsrg_diag_hd, plus the transform of the overlap to the channel
 *      eigenbasis, C = I + bb_i^T S_ij bb_j (:127-186), DPOTRF of C (:272),
 *      DSYGST(1,'L') of A (:284), and after the eigensolve the back-transform
 *      x = L^-T y (DTRSM('Left','L','T'), :322-334).  scc (device) holds the
 *      overlap blocks in hcc's layout; its diagonal blocks are taken from b's
 *      sb, as for bsrg_diag_hd (the reference reads the same values from the
 *      overlap file).  Perturber rows (kcp > 0) are not part of this path.
 *      The refinement, when on, refines the eigenpairs of the standard
 *      problem L^-1 A L^-T.  An overlap that is not positive definite returns
 *      BSRG_ERR_INFO ("Cholesky factorization failed"). */
int bsrg_diag_hd_gen(bsrg_ctx *c, const bsrg_basis *b, int nch, const int *lch, const double *hcc,
                     const double *scc, int itype, int ilzero, int ibzero, double edmax, double egap,
                     int want_vectors, double *eval, int *khm, double *vecs, double *bb);

/* ---- src/bsr/BSR_MAT3/bs_orth.f90:2-92 (BS_ORTH, called from sub1.f90:195):
 *      orthogonality conditions of the channels.  Channel i is made orthogonal
 *      to the orbitals ort_idx[ort_ptr[i] .. ort_ptr[i+1]-1] (host, 0-based
 *      columns of P; the reference picks the bound orbitals with the channel's l
 *      that IBORT does not exempt): every block becomes
 *      H_ij -> (1 - B zz_i) H_ij (1 - zz_j B), zz_i = sum p p^T, B the full
 *      B-spline overlap.  hcc (device) is updated in place; P (device, ns x norb).
 *      Perturber blocks (kcp > 0) are outside this path. */
int bsrg_bs_orth(bsrg_ctx *c, const bsrg_basis *b, int nch, int norb, const double *P, const int *ort_ptr,
                 const int *ort_idx, double *hcc);

/* ---- No counterpart in the reference: switch the FP64 eigenpair refinement
 *      of bsrg_diag_hd on (default) or off for this context, and read the
 *      per-pair correction (refined minus raw eigenvalue) and residual norm
 *      ||A v - lambda v|| / ||v|| of the last refined bsrg_diag_hd into corr
 *      and resid (device, n <= khm doubles each, either may be NULL) on the
 *      context's stream. */
int bsrg_ctx_set_refine(bsrg_ctx *c, int on);
/* ---- No counterpart in the reference: the precision form of this context.
 *      mixed = 0: FP64 (the default).  mixed = 1: the mixed-precision form --
 *      bsrg_assemble computes the direct contraction (convol icase 1 of every
 *      direct group, I_data.f90:206) as bsrg_dgemm_ozaki's product from 8-bit
 *      digits on the tensor cores (8 digits, exact int32 accumulation: FP64
 *      accuracy).  mixed = 2: the same contraction as bsrg_dgemm_tf32x3's
 *      split-TF32 product (FP32 accumulation, ~1e-6 relative).  Everything
 *      else, the eigensolve and its refinement stay FP64. */
int bsrg_ctx_set_precision(bsrg_ctx *c, int mixed);
/* ---- No counterpart in the reference (its DSYEV call is diag_hd.f90:312):
 *      which dense eigensolver bsrg_diag_hd uses on this context.  which = 0
 *      (default): the library's two-stage solver from 7000 rows of the dense
 *      problem (where it was measured faster than cuSOLVER's syevd on a B200)
 *      and cuSOLVER's below; 1: the library's at every size up to 10240 rows;
 *      2: cuSOLVER's at every size.  Contexts that solve concurrently on
 *      several streams do better with 1: the library's solver leaves most of
 *      the GPU to the other streams where cuSOLVER's reduction serialises
 *      them.  The environment variable BSRG_EIG=own|lib overrides it. */
int bsrg_ctx_set_eigensolver(bsrg_ctx *c, int which);
int bsrg_diag_hd_refine_stats(bsrg_ctx *c, int n, double *corr, double *resid);
/* ---- No counterpart in the reference: how many bsrg_diag_hd calls on this
 *      context redid their channel problems (diag_hd.f90:82-111) on the
 *      cuSOLVER path because the library's own batched solves flagged a pair
 *      of eigenvectors as far from orthogonal (eigenvalues equal to working
 *      precision).  Host int. */
int bsrg_ctx_channel_fallbacks(const bsrg_ctx *c, int *count);

/* ---- No counterpart in the reference (it links BLAS but calls no DGEMM on
 *      this path; diag_hd.f90:188-219 transforms the blocks with hand loops):
 *      the library's FP64 tensor-core GEMM, C = alpha op(A) op(B) + beta C,
 *      column-major, for `batch` items spaced by the strides (elements).
 *      transa/transb 'N' or 'T'.  Device. */
int bsrg_dgemm(char transa, char transb, int m, int n, int k, double alpha, const double *A, long lda, long strideA,
               const double *B, long ldb, long strideB, double beta, double *C, long ldc, long strideC, int batch,
               void *stream);

/* ---- No counterpart in the reference (which assembles in FP64): the split-
 *      precision product of the mixed-precision form, on the 5th-generation
 *      tensor cores (tcgen05 kind::tf32, FP32 accumulation in tensor memory).
 *      C = alpha A B + beta C, column-major FP64 arrays (A m x k, B k x n); each
 *      operand is split into two TF32 parts and the three leading products are
 *      accumulated, ~22 significant bits per operand.  *err (device int) is set
 *      to 1 if a device-side wait ran out.  Device. */
int bsrg_dgemm_tf32x3(int m, int n, int k, double alpha, const double *A, int lda, const double *B, int ldb,
                      double beta, double *C, int ldc, int *err, void *stream);

/* ---- No counterpart in the reference (which assembles in FP64): the product
 *      of the mixed-precision form, C = alpha A B + beta C (column-major FP64,
 *      A m x k, B k x n), computed on the 5th-generation tensor cores from 8-bit
 *      integer digits with exact int32 accumulation (the Ozaki splitting): each
 *      row of A and column of B is scaled by a power of two and cut into
 *      `slices` signed 7-bit digits (6..8, 0 = 8), and the digit products of
 *      order below slices are summed.  With 8 digits the result agrees with an
 *      FP64 GEMM to ~1e-16 k max|A(i,:)| max|B(:,j)|.  k <= BSRG_OZAKI_KMAX.
 *      work (device, 256-byte aligned) holds the digits:
 *      bsrg_dgemm_ozaki_work_bytes(m, n, k, slices) bytes.  *err (device int)
 *      is set to 1 if a device-side wait ran out and to 2 if A or B holds a
 *      non-finite value (C is then undefined).  Device. */
#define BSRG_OZAKI_KMAX 16384
size_t bsrg_dgemm_ozaki_work_bytes(int m, int n, int k, int slices);
int bsrg_dgemm_ozaki(int m, int n, int k, double alpha, const double *A, int lda, const double *B, int ldb,
                     double beta, double *C, int ldc, int slices, void *work, size_t work_bytes, int *err,
                     void *stream);

/* ---- the channel solution offsets ipsol(0:nch) of the last bsrg_diag_hd on
 *      this context (module bsr_hd's ipsol, set in diag_hd.f90:100-111):
 *      channel i owns rows ipsol[i] .. ipsol[i+1]-1 of the eigenvectors. */
int bsrg_diag_hd_ipsol(bsrg_ctx *c, int nch, int *ipsol);

/* ---- src/bsr/BSR_HD3/w_out.f90:58-76 (W_OUT, the weights behind w.nnn and
 *      b_out.f90's bound-state selection): for every solution is,
 *      wt(ich, is) = sum_{j in channel ich} a(j, is)^2 in row order (device,
 *      nch x khm), iprm(:, is) the channels ordered by SORTA
 *      (libs/ZCOM/sorting_routines.f90:79-97; 1-based; device, nch x khm, may be
 *      NULL) and isol(is) = iprm(1, is), the dominant channel (device, khm).
 *      a and ipsol (host) as for bsrg_rsol_out.  Perturbers (kcp > 0) are
 *      outside this path. */
int bsrg_channel_weights(bsrg_ctx *c, int nch, const int *ipsol, int khm, const double *a, double *wt, int *isol,
                         int *iprm);

/* ---- src/bsr/BSR_HD3/rsol_out.f90:20-36: solutions in the B-spline basis
 *      v(:, is) = sum_j a(j, is) bb(:, j) channel by channel (device,
 *      (nch*ns) x khm, may be NULL) and the surface amplitudes
 *      WMAT(ich, is) = v(ich*ns, is) (device, nch x khm).  bb and a as returned
 *      by bsrg_diag_hd (bb with ns columns reserved per channel), ipsol (host)
 *      from bsrg_diag_hd_ipsol. */
int bsrg_rsol_out(bsrg_ctx *c, int ns, int nch, const int *ipsol, const double *bb, int khm, const double *a,
                  double *v, double *wmat);

/* ---- LAPACK DSYTRD (uplo 'L') as called inside DSYEV by LAP_DSYEV
 *      (src/libs/ZCOM/LAPACK_calls.f90:54-76, from diag_hd.f90:312): A (device,
 *      n x n, lower triangle) is reduced to the symmetric tridiagonal T = Q^T A Q;
 *      d (n), e (n-1) and tau (n-1) on the device; the reflectors are left in A
 *      below the subdiagonal (LAPACK layout, so DORMTR applies Q).  Uses the
 *      context's stream and workspace. */
int bsrg_dsytrd(bsrg_ctx *c, int n, double *A, int lda, double *d, double *e, double *tau);

/* ---- the tridiagonal stage of DSYEV (LAP_DSYEV, src/libs/ZCOM/LAPACK_calls.f90:54-76,
 *      from diag_hd.f90:312; DSYEV diagonalises T by DSTEQR): all eigenvalues
 *      (ascending, w) and eigenvectors (Z, ldz >= n) of the symmetric tridiagonal
 *      T = tridiag(e, d, e) by divide and conquer (LAPACK DSTEDC's algorithm).
 *      d (n), e (n-1) device, unchanged.  n <= 10240.  Uses the context's stream
 *      and workspace; reads small per-level counts back to the host. */
int bsrg_dstedc(bsrg_ctx *c, int n, const double *d, const double *e, double *w, double *Z, int ldz);

/* ---- DSYEV('V','L') as called by LAP_DSYEV (src/libs/ZCOM/LAPACK_calls.f90:54-76,
 *      from diag_hd.f90:312): all eigenvalues (w, ascending) and eigenvectors
 *      (Z, ldz) of the symmetric A (lower triangle read, lda; Z may be A).
 *      Two-stage reduction (dense -> band of width 32 -> tridiagonal), divide
 *      and conquer, back-transformation.  n <= 10240.  Device; uses the
 *      context's stream and workspace. */
int bsrg_dsyevd(bsrg_ctx *c, int n, const double *A, int lda, double *w, double *Z, int ldz);

/* ---- the reduction alone, as LAPACK's DSYTRD_2STAGE with vect = 'N' (the
 *      first half of DSYEV, LAPACK_calls.f90:54-76): the symmetric A (lower
 *      triangle, lda) is reduced through a band of width 32 to the tridiagonal
 *      T = tridiag(e, d, e) with the same eigenvalues; d (n), e (n-1) device.
 *      n <= 10240. */
int bsrg_dsytrd_2stage(bsrg_ctx *c, int n, const double *A, int lda, double *d, double *e);

/* ---- whole path for one partial wave with HOST buffers (bsr_mat SUB1 then
 *      bsr_hd SUB1_HD): knots, orbitals, coefficients in; eigenvalues out.
 *      t (ns+ks), P (ns,norb), coefficient arrays as in bsrg_assemble, all
 *      host; eval (host) must hold nch*ns doubles.  The context keeps the
 *      basis built from t (define_spline's module state) and its device
 *      buffers between calls; a call with the same ks and knots reuses them. */
int bsrg_partial_wave_solve(bsrg_ctx *c, int ks, int ns, const double *t, double z, int nch,
                            const int *lch, const double *ech, int norb, const double *P, int kmax,
                            int ncoef, const int *ck, const int *ctype, const int *cich, const int *cjch,
                            const int *ca, const int *cb, const double *cval, int want_vectors,
                            double *eval, int *khm);

#ifdef __cplusplus
}
#endif
#endif /* BSR_B200_H */
