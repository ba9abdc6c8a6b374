!======================================================================
!     bsr_gpu.f90 -- ISO_C_BINDING interface of libbsrgpu.so for the
!     BSR Fortran codes (C ABI: include/bsr_b200.h)
!----------------------------------------------------------------------
!     Interfaces for the C entry points plus wrappers named after the
!     routines they stand in for:
!
!       gpu_define_spline       after define_grid + define_spline
!       gpu_mrk_cell(k)         mrk_cell (libs/BS/mrk_cell.f90:2): fills
!                               module spline_integrals rkb from the GPU
!       gpu_mnk_cell(k), gpu_mmk_cell(k), gpu_mtk_cell(k), gpu_mvk_cell(k),
!       gpu_mwk_cell(k), gpu_mqk_cell(k)
!                               the Breit-Pauli tables mnk_cell, mmk_cell,
!                               mtk_cell, mvk_cell, mwk_cell, mqk_cell
!                               (libs/BS/m?k_cell.f90:2),
!                               with spline_atomic's fine
!       gpu_add_two_electron    the I_data Case(6..9) call for icase 5
!                               (bsr/BSR_MAT3/I_data.f90:192-218)
!       gpu_diag_hd             the eigen-solution of diag_hd for a
!                               block-diagonal overlap (bsr/BSR_HD3/
!                               diag_hd.f90:82-312)
!       gpu_w_out_weights       W_OUT's channel weights, dominant channel
!                               and SORTA order (bsr/BSR_HD3/w_out.f90:58-76)
!
!     Device memory is obtained from the CUDA runtime through its C
!     interface (cudaMalloc / cudaMemcpy / cudaFree) bound below.
!     A status /= 0 is turned into the reference's Stop with the
!     library's message, so failures read like the reference's.
!======================================================================
      Module bsr_gpu

      Use, intrinsic :: iso_c_binding
      Implicit none

      Integer(c_int), parameter :: BSRG_OK = 0
      Integer(c_int), parameter :: cudaMemcpyHostToDevice = 1
      Integer(c_int), parameter :: cudaMemcpyDeviceToHost = 2

      Type(c_ptr), save :: gpu_basis = c_null_ptr     ! bsrg_basis*
      Type(c_ptr), save :: gpu_ctx   = c_null_ptr     ! bsrg_ctx*
      Type(c_ptr), save :: d_rkb     = c_null_ptr     ! device rkb(ns,ns,2ks-1,2ks-1)
      Integer, save :: gpu_krk = -100                 ! multipole held in rkb

      Interface

       Function bsrg_last_error() bind(C, name="bsrg_last_error")
        Import :: c_ptr
        Type(c_ptr) :: bsrg_last_error
       End Function

       Function bsrg_define_spline(ks, ns, t, ml, me, h, stream, out) &
                bind(C, name="bsrg_define_spline")
        Import :: c_int, c_double, c_ptr
        Integer(c_int), value :: ks, ns, ml, me
        Real(c_double), intent(in) :: t(*)
        Real(c_double), value :: h
        Type(c_ptr), value :: stream
        Type(c_ptr), intent(out) :: out
        Integer(c_int) :: bsrg_define_spline
       End Function

       Function bsrg_mrk_cell(b, k, rkb, ldp, stream) bind(C, name="bsrg_mrk_cell")
        Import :: c_int, c_ptr
        Type(c_ptr), value :: b, rkb, stream
        Integer(c_int), value :: k, ldp
        Integer(c_int) :: bsrg_mrk_cell
       End Function

       Function bsrg_mnk_cell(b, k, fine, rkb, ldp, stream) bind(C, name="bsrg_mnk_cell")
        Import :: c_int, c_double, c_ptr
        Type(c_ptr), value :: b, rkb, stream
        Integer(c_int), value :: k, ldp
        Real(c_double), value :: fine
        Integer(c_int) :: bsrg_mnk_cell
       End Function

       Function bsrg_mmk_cell(b, k, fine, rkb, ldp, stream) bind(C, name="bsrg_mmk_cell")
        Import :: c_int, c_double, c_ptr
        Type(c_ptr), value :: b, rkb, stream
        Integer(c_int), value :: k, ldp
        Real(c_double), value :: fine
        Integer(c_int) :: bsrg_mmk_cell
       End Function

       Function bsrg_mtk_cell(b, k, fine, rkb, ldp, stream) bind(C, name="bsrg_mtk_cell")
        Import :: c_int, c_double, c_ptr
        Type(c_ptr), value :: b, rkb, stream
        Integer(c_int), value :: k, ldp
        Real(c_double), value :: fine
        Integer(c_int) :: bsrg_mtk_cell
       End Function

       Function bsrg_mvk_cell(b, k, fine, rkb, ldp, stream) bind(C, name="bsrg_mvk_cell")
        Import :: c_int, c_double, c_ptr
        Type(c_ptr), value :: b, rkb, stream
        Integer(c_int), value :: k, ldp
        Real(c_double), value :: fine
        Integer(c_int) :: bsrg_mvk_cell
       End Function

       Function bsrg_mwk_cell(b, k, fine, rkb, ldp, stream) bind(C, name="bsrg_mwk_cell")
        Import :: c_int, c_double, c_ptr
        Type(c_ptr), value :: b, rkb, stream
        Integer(c_int), value :: k, ldp
        Real(c_double), value :: fine
        Integer(c_int) :: bsrg_mwk_cell
       End Function

       Function bsrg_mqk_cell(b, k, fine, rkb, ldp, stream) bind(C, name="bsrg_mqk_cell")
        Import :: c_int, c_double, c_ptr
        Type(c_ptr), value :: b, rkb, stream
        Integer(c_int), value :: k, ldp
        Real(c_double), value :: fine
        Integer(c_int) :: bsrg_mqk_cell
       End Function

       Function bsrg_ctx_create(device, stream, out) bind(C, name="bsrg_ctx_create")
        Import :: c_int, c_ptr
        Integer(c_int), value :: device
        Type(c_ptr), value :: stream
        Type(c_ptr), intent(out) :: out
        Integer(c_int) :: bsrg_ctx_create
       End Function

       Function bsrg_add_two_electron(c, b, nch, norb, P, kmax, ncoef, ck, ctype, &
                cich, cjch, ca, cb, cval, hcc, acf) bind(C, name="bsrg_add_two_electron")
        Import :: c_int, c_double, c_ptr
        Type(c_ptr), value :: c, b, P, hcc, acf
        Integer(c_int), value :: nch, norb, kmax, ncoef
        Integer(c_int), intent(in) :: ck(*), ctype(*), cich(*), cjch(*), ca(*), cb(*)
        Real(c_double), intent(in) :: cval(*)
        Integer(c_int) :: bsrg_add_two_electron
       End Function

       Function bsrg_diag_hd(c, b, nch, lch, hcc, itype, ilzero, ibzero, edmax, egap, &
                want_vectors, eval, khm, vecs, bb) bind(C, name="bsrg_diag_hd")
        Import :: c_int, c_double, c_ptr
        Type(c_ptr), value :: c, b, hcc, eval, vecs, bb
        Integer(c_int), value :: nch, itype, ilzero, ibzero, want_vectors
        Integer(c_int), intent(in) :: lch(*)
        Real(c_double), value :: edmax, egap
        Integer(c_int), intent(out) :: khm
        Integer(c_int) :: bsrg_diag_hd
       End Function

       Function bsrg_diag_hd_gen(c, b, nch, lch, hcc, scc, itype, ilzero, ibzero, edmax, egap, &
                want_vectors, eval, khm, vecs, bb) bind(C, name="bsrg_diag_hd_gen")
        Import :: c_int, c_double, c_ptr
        Type(c_ptr), value :: c, b, hcc, scc, eval, vecs, bb
        Integer(c_int), value :: nch, itype, ilzero, ibzero, want_vectors
        Integer(c_int), intent(in) :: lch(*)
        Real(c_double), value :: edmax, egap
        Integer(c_int), intent(out) :: khm
        Integer(c_int) :: bsrg_diag_hd_gen
       End Function

       Function bsrg_channel_weights(c, nch, ipsol, khm, a, wt, isol, iprm) &
                bind(C, name="bsrg_channel_weights")
        Import :: c_int, c_ptr
        Type(c_ptr), value :: c, a, wt, isol, iprm
        Integer(c_int), value :: nch, khm
        Integer(c_int), intent(in) :: ipsol(*)
        Integer(c_int) :: bsrg_channel_weights
       End Function

       Function bsrg_dsyevd(c, n, A, lda, w, Z, ldz) bind(C, name="bsrg_dsyevd")
        Import :: c_int, c_ptr
        Type(c_ptr), value :: c, A, w, Z
        Integer(c_int), value :: n, lda, ldz
        Integer(c_int) :: bsrg_dsyevd
       End Function

       Function bsrg_ctx_set_precision(c, mixed) bind(C, name="bsrg_ctx_set_precision")
        Import :: c_int, c_ptr
        Type(c_ptr), value :: c
        Integer(c_int), value :: mixed
        Integer(c_int) :: bsrg_ctx_set_precision
       End Function

       Function bsrg_dgemm_ozaki_work_bytes(m, n, k, slices)             &
                bind(C, name="bsrg_dgemm_ozaki_work_bytes")
        Import :: c_int, c_size_t
        Integer(c_int), value :: m, n, k, slices
        Integer(c_size_t) :: bsrg_dgemm_ozaki_work_bytes
       End Function

       Function bsrg_dgemm_ozaki(m, n, k, alpha, A, lda, B, ldb, beta,    &
                C, ldc, slices, work, work_bytes, err, stream)          &
                bind(C, name="bsrg_dgemm_ozaki")
        Import :: c_int, c_ptr, c_size_t, c_double
        Integer(c_int), value :: m, n, k, lda, ldb, ldc, slices
        Real(c_double), value :: alpha, beta
        Type(c_ptr), value :: A, B, C, work, err, stream
        Integer(c_size_t), value :: work_bytes
        Integer(c_int) :: bsrg_dgemm_ozaki
       End Function

       Function cudaMalloc(p, bytes) bind(C, name="cudaMalloc")
        Import :: c_int, c_ptr, c_size_t
        Type(c_ptr) :: p
        Integer(c_size_t), value :: bytes
        Integer(c_int) :: cudaMalloc
       End Function

       Function cudaFree(p) bind(C, name="cudaFree")
        Import :: c_int, c_ptr
        Type(c_ptr), value :: p
        Integer(c_int) :: cudaFree
       End Function

       Function cudaMemcpy(dst, src, bytes, kind) bind(C, name="cudaMemcpy")
        Import :: c_int, c_ptr, c_size_t
        Type(c_ptr), value :: dst, src
        Integer(c_size_t), value :: bytes
        Integer(c_int), value :: kind
        Integer(c_int) :: cudaMemcpy
       End Function

      End Interface

      Contains

!======================================================================
      Subroutine gpu_check(rc, where)
!----------------------------------------------------------------------
!     the reference stops on errors; so does the shim, with the message
!----------------------------------------------------------------------
      Integer(c_int), intent(in) :: rc
      Character(*), intent(in) :: where
      Character(len=512), pointer :: msg
      Integer :: n
      if (rc == BSRG_OK) Return
      Call c_f_pointer(bsrg_last_error(), msg)
      n = index(msg, c_null_char) - 1
      if (n < 0) n = len(msg)
      write(*,'(a,": ",a)') where, msg(1:n)
      Stop 'bsr_gpu: GPU call failed'
      End Subroutine gpu_check

!======================================================================
      Subroutine gpu_define_spline
!----------------------------------------------------------------------
!     after define_grid / define_spline: the same basis on the GPU
!----------------------------------------------------------------------
      Use spline_param
      Use spline_grid, only: t
      Call gpu_check(bsrg_define_spline(ks, ns, t, ml, me, h, c_null_ptr, gpu_basis), &
                     'define_spline')
      if (.not. c_associated(gpu_ctx)) &
       Call gpu_check(bsrg_ctx_create(0_c_int, c_null_ptr, gpu_ctx), 'ctx_create')
      gpu_krk = -100
      End Subroutine gpu_define_spline

!======================================================================
      Subroutine gpu_mrk_cell(k)
!----------------------------------------------------------------------
!     mrk_cell(k) (mrk_cell.f90:2): module rkb filled from the GPU table
!----------------------------------------------------------------------
      Use spline_param
      Use spline_integrals
      Integer, intent(in) :: k
      Integer(c_size_t) :: bytes
      if (itype == 'aaa') Call allocate_integrals
      if (itype == 'rk ' .and. krk == k) Return
      bytes = int(ns, c_size_t) * ns * (2*ks-1) * (2*ks-1) * 8
      if (.not. c_associated(d_rkb)) Call gpu_check(cudaMalloc(d_rkb, bytes), 'cudaMalloc rkb')
      Call gpu_check(bsrg_mrk_cell(gpu_basis, k, d_rkb, 2*ks-1, c_null_ptr), 'mrk_cell')
      Call gpu_check(cudaMemcpy(c_loc(rkb), d_rkb, bytes, cudaMemcpyDeviceToHost), 'cudaMemcpy rkb')
      itype = 'rk '
      krk = k
      End Subroutine gpu_mrk_cell

!======================================================================
      Subroutine gpu_breit_cell(which, k)
!----------------------------------------------------------------------
!     m?k_cell(k) for which = 'nk ', 'mk ', 'tk ', 'vk ', 'wk ', 'qk ': module rkb
!     (ns,ns,2ks-1,2ks-1) filled from the GPU table, fine included
!----------------------------------------------------------------------
      Use spline_param
      Use spline_integrals
      Use spline_atomic, only: fine
      Character(3), intent(in) :: which
      Integer, intent(in) :: k
      Integer(c_size_t) :: bytes
      Integer(c_int) :: rc
      if (itype == 'aaa') Call allocate_integrals
      if (itype == which .and. krk == k) Return
      bytes = int(ns, c_size_t) * ns * (2*ks-1) * (2*ks-1) * 8
      if (.not. c_associated(d_rkb)) Call gpu_check(cudaMalloc(d_rkb, bytes), 'cudaMalloc rkb')
      Select case (which)
       case ('nk '); rc = bsrg_mnk_cell(gpu_basis, k, fine, d_rkb, 2*ks-1, c_null_ptr)
       case ('mk '); rc = bsrg_mmk_cell(gpu_basis, k, fine, d_rkb, 2*ks-1, c_null_ptr)
       case ('tk '); rc = bsrg_mtk_cell(gpu_basis, k, fine, d_rkb, 2*ks-1, c_null_ptr)
       case ('vk '); rc = bsrg_mvk_cell(gpu_basis, k, fine, d_rkb, 2*ks-1, c_null_ptr)
       case ('wk '); rc = bsrg_mwk_cell(gpu_basis, k, fine, d_rkb, 2*ks-1, c_null_ptr)
       case ('qk '); rc = bsrg_mqk_cell(gpu_basis, k, fine, d_rkb, 2*ks-1, c_null_ptr)
       case default; Stop 'gpu_breit_cell: unknown integral type'
      End Select
      Call gpu_check(rc, which // '_cell')
      Call gpu_check(cudaMemcpy(c_loc(rkb), d_rkb, bytes, cudaMemcpyDeviceToHost), 'cudaMemcpy rkb')
      itype = which
      krk = k
      End Subroutine gpu_breit_cell

      Subroutine gpu_mnk_cell(k)
      Integer, intent(in) :: k
      Call gpu_breit_cell('nk ', k)
      End Subroutine gpu_mnk_cell

      Subroutine gpu_mmk_cell(k)
      Integer, intent(in) :: k
      Call gpu_breit_cell('mk ', k)
      End Subroutine gpu_mmk_cell

      Subroutine gpu_mtk_cell(k)
      Integer, intent(in) :: k
      Call gpu_breit_cell('tk ', k)
      End Subroutine gpu_mtk_cell

      Subroutine gpu_mvk_cell(k)
      Integer, intent(in) :: k
      Call gpu_breit_cell('vk ', k)
      End Subroutine gpu_mvk_cell

      Subroutine gpu_mwk_cell(k)
      Integer, intent(in) :: k
      Call gpu_breit_cell('wk ', k)
      End Subroutine gpu_mwk_cell

      Subroutine gpu_mqk_cell(k)
      Integer, intent(in) :: k
      Call gpu_breit_cell('qk ', k)
      End Subroutine gpu_mqk_cell

!======================================================================
      Subroutine gpu_add_two_electron(nch, norb, pbs, kmax, ncoef, ck, ctype, &
                                      cich, cjch, ca, cb, cval, hcc, acf)
!----------------------------------------------------------------------
!     I_data Case(6..9), icase 5: the coefficient records of all R^k
!     channel-channel groups (sorted by k, type, ich, jch; type 0 for
!     jtype 6/7, 1 for jtype 8/9; orbitals 0-based) added to hcc and acf
!----------------------------------------------------------------------
      Use spline_param, only: ns
      Integer, intent(in) :: nch, norb, kmax, ncoef
      Real(8), intent(in), target :: pbs(ns, norb)
      Integer(c_int), intent(in) :: ck(*), ctype(*), cich(*), cjch(*), ca(*), cb(*)
      Real(c_double), intent(in) :: cval(*)
      Real(8), intent(inout), target :: hcc(ns, ns, nch*(nch+1)/2), acf(nch, nch, 0:kmax)
      Type(c_ptr) :: dP, dH, dA
      Integer(c_size_t) :: bp, bh, ba
      bp = int(ns, c_size_t) * norb * 8
      bh = int(ns, c_size_t) * ns * (nch*(nch+1)/2) * 8
      ba = int(nch, c_size_t) * nch * (kmax+1) * 8
      Call gpu_check(cudaMalloc(dP, bp), 'cudaMalloc P')
      Call gpu_check(cudaMalloc(dH, bh), 'cudaMalloc hcc')
      Call gpu_check(cudaMalloc(dA, ba), 'cudaMalloc acf')
      Call gpu_check(cudaMemcpy(dP, c_loc(pbs), bp, cudaMemcpyHostToDevice), 'upload P')
      Call gpu_check(cudaMemcpy(dH, c_loc(hcc), bh, cudaMemcpyHostToDevice), 'upload hcc')
      Call gpu_check(cudaMemcpy(dA, c_loc(acf), ba, cudaMemcpyHostToDevice), 'upload acf')
      Call gpu_check(bsrg_add_two_electron(gpu_ctx, gpu_basis, nch, norb, dP, kmax, ncoef, &
                     ck, ctype, cich, cjch, ca, cb, cval, dH, dA), 'I_data')
      Call gpu_check(cudaMemcpy(c_loc(hcc), dH, bh, cudaMemcpyDeviceToHost), 'download hcc')
      Call gpu_check(cudaMemcpy(c_loc(acf), dA, ba, cudaMemcpyDeviceToHost), 'download acf')
      Call gpu_check(cudaFree(dP), 'cudaFree'); Call gpu_check(cudaFree(dH), 'cudaFree')
      Call gpu_check(cudaFree(dA), 'cudaFree')
      End Subroutine gpu_add_two_electron

!======================================================================
      Subroutine gpu_diag_hd(nch, lch, hcc, itype, ilzero, ibzero, Edmax, Egap, &
                             khm, eval, a)
!----------------------------------------------------------------------
!     diag_hd steps 1, 2 and 7 (diag_hd.f90:82-312) for diag_ovl /= 0:
!     eigenvalues eval(1:khm) and eigenvectors a(1:khm,1:khm) in the
!     channel eigenbasis, as the reference leaves them after LAP_DSYEV
!----------------------------------------------------------------------
      Use spline_param, only: ns
      Integer, intent(in) :: nch, itype, ilzero, ibzero
      Integer(c_int), intent(in) :: lch(nch)
      Real(8), intent(in), target :: hcc(ns, ns, nch*(nch+1)/2)
      Real(8), intent(in) :: Edmax, Egap
      Integer, intent(out) :: khm
      Real(8), intent(out), target :: eval(nch*ns), a(*)
      Type(c_ptr) :: dH, dE, dV
      Integer(c_size_t) :: bh, be, bv
      Integer(c_int) :: k
      bh = int(ns, c_size_t) * ns * (nch*(nch+1)/2) * 8
      be = int(nch, c_size_t) * ns * 8
      bv = int(nch, c_size_t) * ns * nch * ns * 8
      Call gpu_check(cudaMalloc(dH, bh), 'cudaMalloc hcc')
      Call gpu_check(cudaMalloc(dE, be), 'cudaMalloc eval')
      Call gpu_check(cudaMalloc(dV, bv), 'cudaMalloc vectors')
      Call gpu_check(cudaMemcpy(dH, c_loc(hcc), bh, cudaMemcpyHostToDevice), 'upload hcc')
      Call gpu_check(bsrg_diag_hd(gpu_ctx, gpu_basis, nch, lch, dH, itype, ilzero, ibzero, &
                     Edmax, Egap, 1_c_int, dE, k, dV, c_null_ptr), 'diag_hd')
      khm = k
      Call gpu_check(cudaMemcpy(c_loc(eval), dE, int(khm, c_size_t) * 8, cudaMemcpyDeviceToHost), &
                     'download eval')
      Call gpu_check(cudaMemcpy(c_loc(a), dV, int(khm, c_size_t) * khm * 8, cudaMemcpyDeviceToHost), &
                     'download vectors')
      Call gpu_check(cudaFree(dH), 'cudaFree'); Call gpu_check(cudaFree(dE), 'cudaFree')
      Call gpu_check(cudaFree(dV), 'cudaFree')
      End Subroutine gpu_diag_hd

!======================================================================
      Subroutine gpu_diag_hd_gen(nch, lch, hcc, scc, itype, ilzero, ibzero, Edmax, Egap, &
                                 khm, eval, a)
!----------------------------------------------------------------------
!     diag_hd for diag_ovl = 0 (diag_hd.f90:82-334 with channel-channel
!     overlap blocks scc in hcc's layout): eigenvalues eval(1:khm) and the
!     back-transformed eigenvectors a(1:khm,1:khm) (after DTRSM, :334)
!----------------------------------------------------------------------
      Use spline_param, only: ns
      Integer, intent(in) :: nch, itype, ilzero, ibzero
      Integer(c_int), intent(in) :: lch(nch)
      Real(8), intent(in), target :: hcc(ns, ns, nch*(nch+1)/2), scc(ns, ns, nch*(nch+1)/2)
      Real(8), intent(in) :: Edmax, Egap
      Integer, intent(out) :: khm
      Real(8), intent(out), target :: eval(nch*ns), a(*)
      Type(c_ptr) :: dH, dS, dE, dV
      Integer(c_size_t) :: bh, be, bv
      Integer(c_int) :: k
      bh = int(ns, c_size_t) * ns * (nch*(nch+1)/2) * 8
      be = int(nch, c_size_t) * ns * 8
      bv = int(nch, c_size_t) * ns * nch * ns * 8
      Call gpu_check(cudaMalloc(dH, bh), 'cudaMalloc hcc')
      Call gpu_check(cudaMalloc(dS, bh), 'cudaMalloc scc')
      Call gpu_check(cudaMalloc(dE, be), 'cudaMalloc eval')
      Call gpu_check(cudaMalloc(dV, bv), 'cudaMalloc vectors')
      Call gpu_check(cudaMemcpy(dH, c_loc(hcc), bh, cudaMemcpyHostToDevice), 'upload hcc')
      Call gpu_check(cudaMemcpy(dS, c_loc(scc), bh, cudaMemcpyHostToDevice), 'upload scc')
      Call gpu_check(bsrg_diag_hd_gen(gpu_ctx, gpu_basis, nch, lch, dH, dS, itype, ilzero, ibzero, &
                     Edmax, Egap, 1_c_int, dE, k, dV, c_null_ptr), 'diag_hd_gen')
      khm = k
      Call gpu_check(cudaMemcpy(c_loc(eval), dE, int(khm, c_size_t) * 8, cudaMemcpyDeviceToHost), &
                     'download eval')
      Call gpu_check(cudaMemcpy(c_loc(a), dV, int(khm, c_size_t) * khm * 8, cudaMemcpyDeviceToHost), &
                     'download vectors')
      Call gpu_check(cudaFree(dH), 'cudaFree'); Call gpu_check(cudaFree(dS), 'cudaFree')
      Call gpu_check(cudaFree(dE), 'cudaFree'); Call gpu_check(cudaFree(dV), 'cudaFree')
      End Subroutine gpu_diag_hd_gen

!======================================================================
      Subroutine gpu_lap_dsyev(job, uplo, n, m, A, eval, info)
!----------------------------------------------------------------------
!     LAP_DSYEV (ZCOM/LAPACK_calls.f90:54-76) for job = 'V', uplo = 'L':
!     all eigenvalues and eigenvectors of A(1:n,1:n) (leading dimension
!     m) by the library's dense eigensolver; A is overwritten by the
!     eigenvectors as DSYEV leaves it.  info = 0, or the library's status.
!----------------------------------------------------------------------
      Character(1), intent(in) :: job, uplo
      Integer, intent(in) :: n, m
      Real(8), intent(inout), target :: A(m, n)
      Real(8), intent(out), target :: eval(n)
      Integer, intent(out) :: info
      Type(c_ptr) :: dA, dE
      Integer(c_size_t) :: ba, be
      if (job /= 'V' .or. uplo /= 'L') Stop 'gpu_lap_dsyev: only job = V, uplo = L'
      ba = int(m, c_size_t) * n * 8
      be = int(n, c_size_t) * 8
      Call gpu_check(cudaMalloc(dA, ba), 'cudaMalloc A')
      Call gpu_check(cudaMalloc(dE, be), 'cudaMalloc eval')
      Call gpu_check(cudaMemcpy(dA, c_loc(A), ba, cudaMemcpyHostToDevice), 'upload A')
      info = bsrg_dsyevd(gpu_ctx, n, dA, m, dE, dA, m)
      if (info == 0) then
        Call gpu_check(cudaMemcpy(c_loc(A), dA, ba, cudaMemcpyDeviceToHost), 'download vectors')
        Call gpu_check(cudaMemcpy(c_loc(eval), dE, be, cudaMemcpyDeviceToHost), 'download eval')
      end if
      Call gpu_check(cudaFree(dA), 'cudaFree'); Call gpu_check(cudaFree(dE), 'cudaFree')
      End Subroutine gpu_lap_dsyev

!======================================================================
      Subroutine gpu_w_out_weights(nch, ipsol, khm, a, WT, isol, iprm)
!----------------------------------------------------------------------
!     w_out.f90:58-76 for every solution: WT(ich,is) = SUM(a(rows of
!     ich,is)**2), iprm(:,is) from SORTA, isol(is) = iprm(1,is)
!----------------------------------------------------------------------
      Integer, intent(in) :: nch, khm
      Integer(c_int), intent(in) :: ipsol(0:nch)
      Real(8), intent(in), target :: a(khm, khm)
      Real(8), intent(out), target :: WT(nch, khm)
      Integer(c_int), intent(out), target :: isol(khm), iprm(nch, khm)
      Type(c_ptr) :: dA, dW, dI, dP
      Integer(c_size_t) :: ba, bw, bi, bp
      ba = int(khm, c_size_t) * khm * 8
      bw = int(nch, c_size_t) * khm * 8
      bi = int(khm, c_size_t) * 4
      bp = int(nch, c_size_t) * khm * 4
      Call gpu_check(cudaMalloc(dA, ba), 'cudaMalloc a')
      Call gpu_check(cudaMalloc(dW, bw), 'cudaMalloc WT')
      Call gpu_check(cudaMalloc(dI, bi), 'cudaMalloc isol')
      Call gpu_check(cudaMalloc(dP, bp), 'cudaMalloc iprm')
      Call gpu_check(cudaMemcpy(dA, c_loc(a), ba, cudaMemcpyHostToDevice), 'upload a')
      Call gpu_check(bsrg_channel_weights(gpu_ctx, nch, ipsol, khm, dA, dW, dI, dP), 'w_out weights')
      Call gpu_check(cudaMemcpy(c_loc(WT), dW, bw, cudaMemcpyDeviceToHost), 'download WT')
      Call gpu_check(cudaMemcpy(c_loc(isol), dI, bi, cudaMemcpyDeviceToHost), 'download isol')
      Call gpu_check(cudaMemcpy(c_loc(iprm), dP, bp, cudaMemcpyDeviceToHost), 'download iprm')
      Call gpu_check(cudaFree(dA), 'cudaFree'); Call gpu_check(cudaFree(dW), 'cudaFree')
      Call gpu_check(cudaFree(dI), 'cudaFree'); Call gpu_check(cudaFree(dP), 'cudaFree')
      End Subroutine gpu_w_out_weights

      End Module bsr_gpu
