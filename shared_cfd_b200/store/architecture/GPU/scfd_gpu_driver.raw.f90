! The GPU time loop: on the first step the device context is built from the
! module arrays of this program (grid, connectivity, initial or restarted
! state) and the boundary descriptors of scfd_gpu_bc.f90; every step then runs
! the configured scheme through scfd_step (libscfd_b200.so).  The state comes
! back to the host on the steps before those check_convergence writes out.
! The option codes below are filled in by the generator from checkout.inp.
module scfd_gpu_driver
   use iso_c_binding
   use scfd_b200_iface
   implicit none
   type(c_ptr),save::ctx = c_null_ptr
   type(scfd_desc),save::desc
   type(scfd_stats),save::stats
   logical,save::ready = .false.
contains
   ! the value after a 25-character key of control.inp (as read_InternalLoop reads it)
   subroutine gpu_control(key, val, found)
      character(len=25),intent(in)::key
      double precision,intent(inout)::val
      logical,intent(out)::found
      character*100 buf
      found = .false.
      open(8,file="control.inp")
      do
         read(8,'(a)',end=99) buf
         if(buf(1:25) .eq. key) then
            read(buf(26:),*) val
            found = .true.
            exit
         end if
      end do
99    close(8)
   end subroutine gpu_control

   subroutine gpu_check(ierr, what)
      integer(c_int),intent(in)::ierr
      character(len=*),intent(in)::what
      character(kind=c_char)::msg(512)
      integer(c_int)::jerr
      integer k
      if(ierr .eq. 0) return
      msg = c_null_char
      if(c_associated(ctx)) jerr = scfd_last_error(ctx, msg, 512)
      print *,"Error: ",what," returned status ",ierr," (include/scfd_b200.h)"
      print *,(msg(k), k=1,80)
      stop
   end subroutine gpu_check

   subroutine gpu_init(step)
      use grbl_prmtr
      use variable
      use mod_mpi
      use scfd_gpu_chem
      use scfd_gpu_bc
      GPU_MUSCL_USE
      integer,intent(in)::step
      integer plane
      logical found
      double precision val
      double precision,allocatable::xf(:,:),rf(:,:)

      desc%abi_version = SCFD_ABI_VERSION
      desc%nplane = Nplane
      desc%ni = 0
      desc%nj = 0
      desc%ni(1:Nplane) = ni
      desc%nj(1:Nplane) = nj
      desc%ny = nY
      desc%dim = GPU_DIM
      desc%dt_mode = GPU_DT_MODE
      desc%scheme = GPU_SCHEME
      desc%recon = GPU_RECON
      desc%viscous = GPU_VISCOUS
      desc%thermo = GPU_THERMO
      desc%mu_model = 0
      desc%precision = 0
      desc%quirk_q1 = 1
      desc%il_write = 0
      desc%phi_mus = GPU_PHI
      desc%k_mus = GPU_K
      desc%kappa = GPU_KAPPA
      desc%rgas = GPU_RGAS
      desc%nu_gas = GPU_NU
      desc%suth_mu0 = 0d0
      desc%suth_t0 = 0d0
      desc%suth_s = 0d0
      desc%prandtl = 1d0
      desc%schmidt = 1d0
      desc%cfl = cfl
      desc%dt_fixed = 0d0
      ! inner-loop controls of the dual-time schemes (NR/q2d/control.part.inp defaults)
      val = 60d0
      call gpu_control('InternalLoop Max Number :', val, found)
      desc%num_internal_loop = int(val)
      desc%omega_max = 1d-1
      call gpu_control('InternalLoop Omega Max  :', desc%omega_max, found)
      desc%omega_min = 1d-3
      call gpu_control('InternalLoop Omega Min  :', desc%omega_min, found)
      desc%dq_max = 1d-2
      call gpu_control('InternalLoop Dqrate Max :', desc%dq_max, found)
      desc%res_rate_warn = 1d-5
      call gpu_control('InternalLoop ResRateWarn:', desc%res_rate_warn, found)
      desc%res_rate_err = 1d-3
      call gpu_control('InternalLoop ResRateErr :', desc%res_rate_err, found)
      desc%cfl_tau = 1d-2
      call gpu_control('InternalLoop CFL tau    :', desc%cfl_tau, found)
      desc%chem_max_substeps = 100000
      desc%pad0 = 0
      desc%reserved = 0

      call gpu_check(scfd_create(desc, ctx), "scfd_create")
      do plane=1,Nplane
         allocate(xf(0:ni(plane),0:nj(plane)), rf(0:ni(plane),0:nj(plane)))
         xf = xh(0:ni(plane),0:nj(plane),plane)
         rf = rh(0:ni(plane),0:nj(plane),plane)
         call gpu_check(scfd_set_geometry(ctx, plane, xf, rf), "scfd_set_geometry")
         deallocate(xf, rf)
      end do
      if(num_cut_copro > 0) call gpu_check(scfd_set_connectivity(ctx, cut_copro, num_cut_copro), "scfd_set_connectivity")
      call scfd_gpu_bc_set(ctx)
      call scfd_gpu_chem_set(ctx)
      call gpu_check(scfd_commit(ctx), "scfd_commit")
      call gpu_check(scfd_upload(ctx, q, w, vhi, tt), "scfd_upload")
      call gpu_check(scfd_prepare(ctx, step), "scfd_prepare")
      ready = .true.
   end subroutine gpu_init
end module scfd_gpu_driver

subroutine scfd_gpu_step(step)
   use scfd_gpu_driver
   use variable
   implicit none
   integer,intent(in)::step
   if(.not. ready) call gpu_init(step)
   call gpu_check(scfd_step(ctx, step, stats), "scfd_step")
   ! check_convergence(step+1) runs next and writes out on its OutPeriod
   if(mod(step+1, OutPeriod) .eq. 0) then
      call gpu_check(scfd_download(ctx, q, w, vhi, tt), "scfd_download")
      call gpu_check(scfd_download_qp(ctx, qp), "scfd_download_qp")
   end if
end subroutine scfd_gpu_step
