! evp1d_cuda.F90 -- the ISO_C_BINDING module through which a Fortran host
! (CICE's ice_dyn_evp1d, integration/ice_dyn_evp1d.F90) calls the B200 EVP-1D
! solver behind include/evp1d.h.  Every interface below binds one C-ABI entry
! point of that header, argument for argument; the derived types mirror its
! structs field for field.
!
! It replaces `use bench` in dyn_evp1d_run: the subcycle loop
!     do ksub = 1,ndte
!        call stress (ee, ne, se, 1, nActive, uvel, vvel, ..., str1, ..., str8)
!        call stepu  (1, nActive, cdn_ocn, aiu, ..., nw, sw, sse, skipUcell, Tbu, Cb)
!     enddo
! (integration/ice_dyn_evp1d.F90:188-207) becomes one evp1d_run call on a
! handle made once by evp1d_init in dyn_evp1d_init (after convert_2d_1d_init,
! :108) and released by evp1d_finalize in dyn_evp1d_finalize (:326-331).
! Errors come back as codes (0 = success, EVP1D_ERR_* < 0) with a message
! from evp1d_last_error_f, where the reference stops the program.
!
! Arrays passed as c_loc(x) need the `target` attribute; Fortran logical(4)
! skip flags can be passed as they are (4 bytes, nonzero = .true.).
module evp1d_cuda
  use iso_c_binding
  implicit none
  private
  public :: evp1d_params, evp1d_fields, evp1d_grads
  public :: evp1d_set_evp_parameters, evp1d_init, evp1d_run, evp1d_finalize
  public :: evp1d_upload, evp1d_subcycles, evp1d_subcycles_inner, evp1d_download
  public :: evp1d_synchronize, evp1d_host_alloc, evp1d_host_free
  public :: evp1d_exchange_setup, evp1d_exchange_buffers, evp1d_exchange_pack
  public :: evp1d_exchange_unpack, evp1d_run_checkpointed, evp1d_adjoint
  public :: evp1d_last_error, evp1d_last_error_f

  ! evp1d_params: ice_dyn_shared's EVP parameters (src/ice.F90:80-130)
  type, bind(C) :: evp1d_params
     real(c_double) :: arlx1i, denom1, brlx, capping, e_factor, epp2i, &
                       deltaminEVP, revp, Ktens, u0, cosw, sinw, rhow
  end type

  ! evp1d_fields: the per-call arrays of dyn_evp1d_run in the 1D layout
  ! (host addresses; c_null_ptr where the header allows NULL)
  type, bind(C) :: evp1d_fields
     type(c_ptr) :: skipT, skipU
     type(c_ptr) :: stress(12)
     type(c_ptr) :: strength, Cw, aiu, uocn, vocn, waterx, watery, &
                    forcex, forcey, umassdti, fm, Tbu, uvel_init, vvel_init
     type(c_ptr) :: uvel, vvel, strintx, strinty, Cb
     type(c_ptr) :: str(8)
  end type

  ! evp1d_grads: where evp1d_adjoint writes each gradient (c_null_ptr: not
  ! wanted)
  type, bind(C) :: evp1d_grads
     type(c_ptr) :: strength, Cw, forcex, forcey
     type(c_ptr) :: uvel, vvel
     type(c_ptr) :: stress(12)
     type(c_ptr) :: uvel_init, vvel_init
  end type

  interface
     ! set_evp_parameters (src/ice.F90:109-130)
     subroutine evp1d_set_evp_parameters(p, ndte) bind(C, name="evp1d_set_evp_parameters")
       import :: evp1d_params, c_int
       type(evp1d_params), intent(inout) :: p
       integer(c_int), value :: ndte
     end subroutine

     ! the index and geometry part of dyn_evp1d_init
     ! (integration/ice_dyn_evp1d.F90:65-112); neighbour vectors 1-based
     integer(c_int) function evp1d_init(h, na, navel, ee, ne, se, nw, sw, sse, &
                                        dxT, dyT, HTE, HTN, HTEm1, HTNm1, uarear, &
                                        p, device) bind(C, name="evp1d_init")
       import :: c_ptr, c_int, c_int32_t, c_double, evp1d_params
       type(c_ptr), intent(out) :: h
       integer(c_int), value :: na, navel
       integer(c_int32_t), intent(in) :: ee(*), ne(*), se(*), nw(*), sw(*), sse(*)
       real(c_double), intent(in) :: dxT(*), dyT(*), HTE(*), HTN(*), HTEm1(*), HTNm1(*), &
                                     uarear(*)
       type(evp1d_params), intent(in) :: p
       integer(c_int), value :: device
     end function

     ! dyn_evp1d_run's subcycle loop (integration/ice_dyn_evp1d.F90:188-207)
     integer(c_int) function evp1d_run(h, ndte, io) bind(C, name="evp1d_run")
       import :: c_ptr, c_int, evp1d_fields
       type(c_ptr), value :: h
       integer(c_int), value :: ndte
       type(evp1d_fields), intent(in) :: io
     end function

     ! dyn_evp1d_finalize (integration/ice_dyn_evp1d.F90:326-331)
     integer(c_int) function evp1d_finalize(h) bind(C, name="evp1d_finalize")
       import :: c_ptr, c_int
       type(c_ptr), value :: h
     end function

     ! evp1d_run split for a caller that keeps the state on the device
     integer(c_int) function evp1d_upload(h, io) bind(C, name="evp1d_upload")
       import :: c_ptr, c_int, evp1d_fields
       type(c_ptr), value :: h
       type(evp1d_fields), intent(in) :: io
     end function
     integer(c_int) function evp1d_subcycles(h, ndte) bind(C, name="evp1d_subcycles")
       import :: c_ptr, c_int
       type(c_ptr), value :: h
       integer(c_int), value :: ndte
     end function
     integer(c_int) function evp1d_subcycles_inner(h, n) bind(C, name="evp1d_subcycles_inner")
       import :: c_ptr, c_int
       type(c_ptr), value :: h
       integer(c_int), value :: n
     end function
     integer(c_int) function evp1d_download(h, io) bind(C, name="evp1d_download")
       import :: c_ptr, c_int, evp1d_fields
       type(c_ptr), value :: h
       type(evp1d_fields), intent(in) :: io
     end function
     integer(c_int) function evp1d_synchronize(h) bind(C, name="evp1d_synchronize")
       import :: c_ptr, c_int
       type(c_ptr), value :: h
     end function

     ! page-locked host arrays (map them with c_f_pointer)
     integer(c_int) function evp1d_host_alloc(p, bytes) bind(C, name="evp1d_host_alloc")
       import :: c_ptr, c_int, c_size_t
       type(c_ptr), intent(out) :: p
       integer(c_size_t), value :: bytes
     end function
     integer(c_int) function evp1d_host_free(p) bind(C, name="evp1d_host_free")
       import :: c_ptr, c_int
       type(c_ptr), value :: p
     end function

     ! the velocity exchange of one state split into bands over GPUs (one
     ! task per band; the buffers are device memory the handle owns)
     integer(c_int) function evp1d_exchange_setup(h, ns, send_idx, nr, recv_idx) &
          bind(C, name="evp1d_exchange_setup")
       import :: c_ptr, c_int, c_int32_t
       type(c_ptr), value :: h
       integer(c_int), value :: ns
       integer(c_int32_t), intent(in) :: send_idx(*)
       integer(c_int), value :: nr
       integer(c_int32_t), intent(in) :: recv_idx(*)
     end function
     integer(c_int) function evp1d_exchange_pack(h, buf) bind(C, name="evp1d_exchange_pack")
       import :: c_ptr, c_int
       type(c_ptr), value :: h, buf          ! c_null_ptr: the handle's send buffer
     end function
     integer(c_int) function evp1d_exchange_unpack(h, buf) bind(C, name="evp1d_exchange_unpack")
       import :: c_ptr, c_int
       type(c_ptr), value :: h, buf          ! c_null_ptr: the handle's receive buffer
     end function
     integer(c_int) function evp1d_exchange_buffers(h, sendbuf, recvbuf) &
          bind(C, name="evp1d_exchange_buffers")
       import :: c_ptr, c_int
       type(c_ptr), value :: h
       type(c_ptr), intent(out) :: sendbuf, recvbuf
     end function

     ! gradients: evp1d_run recording what the reverse sweep needs
     ! (interval > 0: checkpoints every interval subcycles; <= 0: sized to
     ! device memory), then the sweep for a seed dJ/d(final u, v);
     ! lam_stress is c_null_ptr or c_loc of 12 c_ptr (each may be null)
     integer(c_int) function evp1d_run_checkpointed(h, ndte, io, interval) &
          bind(C, name="evp1d_run_checkpointed")
       import :: c_ptr, c_int, evp1d_fields
       type(c_ptr), value :: h
       integer(c_int), value :: ndte
       type(evp1d_fields), intent(in) :: io
       integer(c_int), value :: interval
     end function
     integer(c_int) function evp1d_adjoint(h, lam_uvel, lam_vvel, lam_stress, g) &
          bind(C, name="evp1d_adjoint")
       import :: c_ptr, c_int, c_double, evp1d_grads
       type(c_ptr), value :: h
       real(c_double), intent(in) :: lam_uvel(*), lam_vvel(*)
       type(c_ptr), value :: lam_stress
       type(evp1d_grads), intent(in) :: g
     end function

     ! the message of the last failed call (a C string)
     type(c_ptr) function evp1d_last_error() bind(C, name="evp1d_last_error")
       import :: c_ptr
     end function
  end interface

contains

  ! evp1d_last_error as a Fortran string
  function evp1d_last_error_f() result(msg)
    character(len=256) :: msg
    character(kind=c_char), pointer :: s(:)
    integer :: k
    call c_f_pointer(evp1d_last_error(), s, [256])
    msg = ' '
    do k = 1, 256
       if (s(k) == c_null_char) exit
       msg(k:k) = s(k)
    enddo
  end function

end module evp1d_cuda
