! nsx_iface.f90 -- Fortran 2003 iso_c_binding interface to libnsx (include/nsx.h).
!
! For NuShellX's Fortran host code (NuLnz / NuTRL): the module gives the
! bind(C) types and interfaces of every entry point, so that Lnz_TRD's set-up
! (src/NuLnz/NuCoreX.f90:807-1367), the multiplyx/multiplya/multiplyb product
! (NuCoreX.f90:76-226) and Lnz_OP (NuCoreX.f90:240-751) can be replaced by calls
! into the B200 library.  Column-major Fortran arrays of real(8) map directly to
! the library's vector layout (blocks (2Ja,2Jb) in ascending order, each a
! d_a x d_b column-major matrix).  Compile with any Fortran 2003 compiler and
! link against nushellx_b200/libnsx.so.  (This machine has no Fortran compiler,
! so the module is not compiled here; the C header is the authoritative ABI.)
module nsx_iface
  use iso_c_binding
  implicit none

  integer(c_int), parameter :: NSX_OK = 0, NSX_E_ARG = -1, NSX_E_IO = -2, NSX_E_CUDA = -3, &
                               NSX_E_NOMEM = -4, NSX_E_NUMERIC = -5, NSX_E_NOCONV = -6
  integer(c_int), parameter :: NSX_FP64 = 0, NSX_FP32 = 1
  integer(c_int), parameter :: NSX_STAGES = 5

  type, bind(C) :: nsx_species
     integer(c_int32_t) :: nspart, minJ2, maxJ2
     type(c_ptr)        :: njt, parity
     integer(c_int32_t) :: shell_first, nshell
     integer(c_int32_t) :: nkeys
     type(c_ptr)        :: keys, val_off, vals
     integer(c_int32_t) :: words
     type(c_ptr)        :: masks
     integer(c_int32_t) :: nseg
     type(c_ptr)        :: seg_J2, seg_np, seg_npr, seg_off, seg_vals
     type(c_ptr)        :: occ          ! int16 [nspart][nshell] or c_null_ptr
  end type nsx_species

  type, bind(C) :: nsx_problem
     integer(c_int32_t) :: J2, parity
     type(nsx_species)  :: a, b
     integer(c_int32_t) :: nop
     type(c_ptr)        :: op_keys, op_vals
     real(c_double)     :: renorm
  end type nsx_problem

  type, bind(C) :: nsx_files
     type(c_ptr)        :: a, b, inter, like_a, like_b   ! NUL-terminated base names
     integer(c_int32_t) :: T2_a, nmp_a, T2_b, nmp_b
     character(kind=c_char) :: xtra
     integer(c_int32_t) :: J2, parity, nshells, nshells_p
     type(c_ptr)        :: shell_parity
  end type nsx_files

  type, bind(C) :: nsx_params
     integer(c_int32_t) :: nev, max_iter, window, keep
     real(c_double)     :: tol
     integer(c_int32_t) :: precision, pre_iter
     integer(c_int64_t) :: seed
     type(c_ptr)        :: start
     integer(c_int32_t) :: refine
  end type nsx_params

  type, bind(C) :: nsx_report
     integer(c_int32_t) :: iterations, matvecs, restarts, converged
     real(c_double)     :: seconds, matvec_seconds
     real(c_double)     :: residual(64)
  end type nsx_report

  type, bind(C) :: nsx_stats
     integer(c_int64_t) :: launches, matvecs
     integer(c_int64_t) :: stage_launches(NSX_STAGES)
     real(c_double)     :: stage_ms(NSX_STAGES), stage_bytes(NSX_STAGES), stage_flops(NSX_STAGES)
  end type nsx_stats

  type, bind(C) :: nsx_dop
     integer(c_int32_t) :: nterms
     type(c_ptr)        :: lam2, parity, eig, e, shells, u
  end type nsx_dop

  type, bind(C) :: nsx_plan_info
     integer(c_int64_t) :: y_elems, zbar_elems, zbar_tc_elems
     integer(c_int32_t) :: y_row_tiles_max, group_sources_max, fused_fp32
     integer(c_int32_t) :: slab_rows_max, slab_splits_max, slab_nl_max
     integer(c_int64_t) :: tc_tiles(4), tc_chunks_max
     integer(c_int32_t) :: fp32_path, tc_pieces
  end type nsx_plan_info

  type, bind(C) :: nsx_state
     integer(c_int32_t) :: m
     type(c_ptr)        :: V, T, next
     real(c_double)     :: beta
     integer(c_int32_t) :: iterations, restarts
  end type nsx_state

  interface
     integer(c_int) function nsx_solve_ex(h, params, resume, state_out, evals, evecs, report) &
          bind(C, name="nsx_solve_ex")
       import :: c_int, c_ptr, nsx_params, nsx_report
       type(c_ptr), value :: h
       type(nsx_params), intent(in) :: params
       type(c_ptr), value :: resume, state_out     ! nsx_state or c_null_ptr
       real(c_double), dimension(*), intent(out) :: evals
       type(c_ptr), value :: evecs
       type(nsx_report), intent(out) :: report
     end function
     integer(c_int) function nsx_write_state(h, prefix, state, evals, evecs, nev, intfile, T2) &
          bind(C, name="nsx_write_state")
       import :: c_int, c_ptr, c_char, c_int32_t, c_double, nsx_state
       type(c_ptr), value :: h
       character(kind=c_char), dimension(*), intent(in) :: prefix, intfile
       type(nsx_state), intent(in) :: state
       real(c_double), dimension(*), intent(in) :: evals
       type(c_ptr), value :: evecs
       integer(c_int32_t), value :: nev, T2
     end function
     integer(c_int) function nsx_read_state(h, prefix, state) bind(C, name="nsx_read_state")
       import :: c_int, c_ptr, c_char, nsx_state
       type(c_ptr), value :: h
       character(kind=c_char), dimension(*), intent(in) :: prefix
       type(nsx_state), intent(inout) :: state
     end function
     integer(c_int) function nsx_create_z(prob, dop, device, out) bind(C, name="nsx_create_z")
       import :: c_int, c_ptr, nsx_problem, nsx_dop
       type(nsx_problem), intent(in) :: prob
       type(nsx_dop), intent(in) :: dop
       integer(c_int), value :: device
       type(c_ptr), intent(out) :: out
     end function
     integer(c_int) function nsx_load_files_z(files, dop_path, device, out) bind(C, name="nsx_load_files_z")
       import :: c_int, c_ptr, c_char, nsx_files
       type(nsx_files), intent(in) :: files
       character(kind=c_char), dimension(*), intent(in) :: dop_path   ! NUL-terminated
       integer(c_int), value :: device
       type(c_ptr), intent(out) :: out
     end function
     ! output-block shards: rank's rows of H.v; the exchange (a bind(C) function
     ! integer(c_int) fn(user, y, n, stream), e.g. an ncclAllGather) completes each product
     integer(c_int) function nsx_create_shard(prob, device, rank, world, out) bind(C, name="nsx_create_shard")
       import :: c_int, c_ptr, c_int32_t, nsx_problem
       type(nsx_problem), intent(in) :: prob
       integer(c_int), value :: device
       integer(c_int32_t), value :: rank, world
       type(c_ptr), intent(out) :: out
     end function
     integer(c_int) function nsx_load_files_shard(files, device, rank, world, out) &
          bind(C, name="nsx_load_files_shard")
       import :: c_int, c_ptr, c_int32_t, nsx_files
       type(nsx_files), intent(in) :: files
       integer(c_int), value :: device
       integer(c_int32_t), value :: rank, world
       type(c_ptr), intent(out) :: out
     end function
     integer(c_int) function nsx_shard_info(h, rank, world, row_begin, est_flops) bind(C, name="nsx_shard_info")
       import :: c_int, c_ptr, c_int32_t, c_int64_t, c_double
       type(c_ptr), value :: h
       integer(c_int32_t), intent(out) :: rank, world
       integer(c_int64_t), dimension(*), intent(out) :: row_begin   ! world + 1
       real(c_double), dimension(*), intent(out) :: est_flops       ! world
     end function
     integer(c_int) function nsx_set_exchange(h, fn, user) bind(C, name="nsx_set_exchange")
       import :: c_int, c_ptr, c_funptr
       type(c_ptr), value :: h
       type(c_funptr), value :: fn
       type(c_ptr), value :: user
     end function
     integer(c_int) function nsx_block_flops(h, out) bind(C, name="nsx_block_flops")
       import :: c_int, c_ptr, c_double
       type(c_ptr), value :: h
       real(c_double), dimension(*), intent(out) :: out
     end function
     integer(c_int) function nsx_set_fp32_path(h, path) bind(C, name="nsx_set_fp32_path")
       import :: c_int, c_ptr, c_int32_t
       type(c_ptr), value :: h
       integer(c_int32_t), value :: path   ! 0 auto, 1 fused, 2 tensor-core, 3 SIMT
     end function
     integer(c_int) function nsx_get_plan_info(h, info) bind(C, name="nsx_get_plan_info")
       import :: c_int, c_ptr, nsx_plan_info
       type(c_ptr), value :: h
       type(nsx_plan_info), intent(out) :: info
     end function
     integer(c_int) function nsx_expectation_matrix(h, vecs, nvec, precision, out) &
          bind(C, name="nsx_expectation_matrix")
       import :: c_int, c_ptr, c_int32_t, c_double
       type(c_ptr), value :: h
       real(c_double), dimension(*), intent(in) :: vecs
       integer(c_int32_t), value :: nvec, precision
       real(c_double), dimension(*), intent(out) :: out
     end function
     integer(c_int) function nsx_xpct_files(h, xvc_path, out_prefix, precision) bind(C, name="nsx_xpct_files")
       import :: c_int, c_ptr, c_char, c_int32_t
       type(c_ptr), value :: h
       character(kind=c_char), dimension(*), intent(in) :: xvc_path, out_prefix   ! NUL-terminated
       integer(c_int32_t), value :: precision
     end function
     integer(c_int) function nsx_create(prob, device, out) bind(C, name="nsx_create")
       import :: c_int, c_ptr, nsx_problem
       type(nsx_problem), intent(in) :: prob
       integer(c_int), value :: device
       type(c_ptr), intent(out) :: out
     end function
     integer(c_int) function nsx_load_files(files, device, out) bind(C, name="nsx_load_files")
       import :: c_int, c_ptr, nsx_files
       type(nsx_files), intent(in) :: files
       integer(c_int), value :: device
       type(c_ptr), intent(out) :: out
     end function
     integer(c_int) function nsx_set_interaction(h, op_vals, nop, a_seg_vals, a_nvals, b_seg_vals, b_nvals) &
          bind(C, name="nsx_set_interaction")
       import :: c_int, c_int32_t, c_int64_t, c_double, c_ptr
       type(c_ptr), value :: h
       real(c_double), intent(in) :: op_vals(*), a_seg_vals(*), b_seg_vals(*)
       integer(c_int32_t), value :: nop
       integer(c_int64_t), value :: a_nvals, b_nvals
     end function
     integer(c_int) function nsx_file_code(i, j, k, code) bind(C, name="nsx_file_code")
       import :: c_int, c_int32_t, c_char
       integer(c_int32_t), value :: i, j, k
       character(kind=c_char), intent(out) :: code(4)
     end function
     integer(c_int64_t) function nsx_dim(h) bind(C, name="nsx_dim")
       import :: c_int64_t, c_ptr
       type(c_ptr), value :: h
     end function
     integer(c_int32_t) function nsx_nblocks(h) bind(C, name="nsx_nblocks")
       import :: c_int32_t, c_ptr
       type(c_ptr), value :: h
     end function
     integer(c_int) function nsx_blocks(h, blocks4, offsets) bind(C, name="nsx_blocks")
       import :: c_int, c_int32_t, c_int64_t, c_ptr
       type(c_ptr), value :: h
       integer(c_int32_t), intent(out) :: blocks4(*)
       integer(c_int64_t), intent(out) :: offsets(*)
     end function
     integer(c_int) function nsx_lcoef(h, mask) bind(C, name="nsx_lcoef")
       import :: c_int, c_int8_t, c_ptr
       type(c_ptr), value :: h
       integer(c_int8_t), intent(out) :: mask(*)
     end function
     real(c_double) function nsx_matvec_flops(h) bind(C, name="nsx_matvec_flops")
       import :: c_double, c_ptr
       type(c_ptr), value :: h
     end function
     integer(c_int) function nsx_matvec(h, x, y, precision, stream) bind(C, name="nsx_matvec")
       import :: c_int, c_int32_t, c_ptr
       type(c_ptr), value :: h, x, y, stream           ! x, y: device pointers
       integer(c_int32_t), value :: precision
     end function
     integer(c_int) function nsx_matvec_noalloc(h, x, y, stream) bind(C, name="nsx_matvec_noalloc")
       import :: c_int, c_ptr
       type(c_ptr), value :: h, x, y, stream           ! x, y: device pointers, FP64
     end function
     integer(c_int) function nsx_matvec_host(h, x, y, precision) bind(C, name="nsx_matvec_host")
       import :: c_int, c_int32_t, c_double, c_ptr
       type(c_ptr), value :: h
       real(c_double), intent(in) :: x(*)              ! the reference's coefR
       real(c_double), intent(out) :: y(*)             ! the reference's coefL
       integer(c_int32_t), value :: precision
     end function
     integer(c_int) function nsx_solve(h, params, evals, evecs, report) bind(C, name="nsx_solve")
       import :: c_int, c_double, c_ptr, nsx_params, nsx_report
       type(c_ptr), value :: h
       type(nsx_params), intent(in) :: params
       real(c_double), intent(out) :: evals(*)
       type(c_ptr), value :: evecs                     ! c_loc(vectors(1,1)) or c_null_ptr
       type(nsx_report), intent(out) :: report
     end function
     integer(c_int) function nsx_batch_solve(handles, n, params, evals, evecs, reports) &
          bind(C, name="nsx_batch_solve")
       import :: c_int, c_int32_t, c_ptr, nsx_params, nsx_report
       type(c_ptr), intent(in) :: handles(*)            ! one handle per problem
       integer(c_int32_t), value :: n
       type(nsx_params), intent(in) :: params(*)
       type(c_ptr), intent(in) :: evals(*)              ! c_loc of each problem's eigenvalue array
       type(c_ptr), value :: evecs                      ! c_loc of an array of n c_ptr, or c_null_ptr
       type(nsx_report), intent(out) :: reports(*)
     end function
     integer(c_int) function nsx_write_results(h, prefix, evals, evecs, nev, iterations, intfile, T2) &
          bind(C, name="nsx_write_results")
       import :: c_int, c_int32_t, c_double, c_ptr
       type(c_ptr), value :: h, prefix, intfile           ! prefix, intfile: c_loc of NUL-terminated strings
       real(c_double), intent(in) :: evals(*), evecs(*)
       integer(c_int32_t), value :: nev, iterations, T2
     end function
     integer(c_int) function nsx_stats_reset(h, timing) bind(C, name="nsx_stats_reset")
       import :: c_int, c_int32_t, c_ptr
       type(c_ptr), value :: h
       integer(c_int32_t), value :: timing
     end function
     integer(c_int) function nsx_get_stats(h, stats) bind(C, name="nsx_get_stats")
       import :: c_int, c_ptr, nsx_stats
       type(c_ptr), value :: h
       type(nsx_stats), intent(out) :: stats
     end function
     subroutine nsx_destroy(h) bind(C, name="nsx_destroy")
       import :: c_ptr
       type(c_ptr), value :: h
     end subroutine
     type(c_ptr) function nsx_last_error() bind(C, name="nsx_last_error")
       import :: c_ptr
     end function
     ! ---- learned start vector: the network (nsx_mlp_*) ----
     integer(c_int) function nsx_mlp_create(n_in, width, n_out, seed, device, net) bind(C, name="nsx_mlp_create")
       import :: c_int, c_int32_t, c_int64_t, c_ptr
       integer(c_int32_t), value :: n_in, width, n_out
       integer(c_int64_t), value :: seed
       integer(c_int), value :: device
       type(c_ptr), intent(out) :: net
     end function
     integer(c_int64_t) function nsx_mlp_param_count(net) bind(C, name="nsx_mlp_param_count")
       import :: c_int64_t, c_ptr
       type(c_ptr), value :: net
     end function
     integer(c_int) function nsx_mlp_set_params(net, params, n) bind(C, name="nsx_mlp_set_params")
       import :: c_int, c_int64_t, c_float, c_ptr
       type(c_ptr), value :: net
       real(c_float), intent(in) :: params(*)
       integer(c_int64_t), value :: n
     end function
     integer(c_int) function nsx_mlp_get_params(net, params, n) bind(C, name="nsx_mlp_get_params")
       import :: c_int, c_int64_t, c_float, c_ptr
       type(c_ptr), value :: net
       real(c_float), intent(out) :: params(*)
       integer(c_int64_t), value :: n
     end function
     integer(c_int) function nsx_mlp_forward(net, x, batch, y) bind(C, name="nsx_mlp_forward")
       import :: c_int, c_int32_t, c_float, c_ptr
       type(c_ptr), value :: net
       real(c_float), intent(in) :: x(*)
       integer(c_int32_t), value :: batch
       real(c_float), intent(out) :: y(*)
     end function
     integer(c_int) function nsx_mlp_gradients(net, x, t, batch, loss, grad) bind(C, name="nsx_mlp_gradients")
       import :: c_int, c_int32_t, c_float, c_ptr
       type(c_ptr), value :: net
       real(c_float), intent(in) :: x(*), t(*)
       integer(c_int32_t), value :: batch
       real(c_float), intent(out) :: loss
       type(c_ptr), value :: grad                      ! c_loc(g(1)) or c_null_ptr
     end function
     integer(c_int) function nsx_mlp_train(net, x, t, batch, steps, lr, loss) bind(C, name="nsx_mlp_train")
       import :: c_int, c_int32_t, c_float, c_ptr
       type(c_ptr), value :: net
       real(c_float), intent(in) :: x(*), t(*)
       integer(c_int32_t), value :: batch, steps
       real(c_float), value :: lr
       real(c_float), intent(out) :: loss
     end function
     subroutine nsx_mlp_destroy(net) bind(C, name="nsx_mlp_destroy")
       import :: c_ptr
       type(c_ptr), value :: net
     end subroutine
     type(c_ptr) function nsx_mlp_last_error() bind(C, name="nsx_mlp_last_error")
       import :: c_ptr
     end function
  end interface
end module nsx_iface
