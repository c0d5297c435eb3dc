! Fortran binding of include/scfd_b200.h (libscfd_b200.so): the structures
! field for field and the entry points the GPU architecture calls.
module scfd_b200_iface
   use iso_c_binding
   implicit none
   integer(c_int32_t),parameter::SCFD_ABI_VERSION   = 1
   integer,parameter::SCFD_MAX_PLANES    = 64
   integer,parameter::SCFD_MAX_SPECIES   = 32
   integer,parameter::SCFD_MAX_REACTIONS = 256
   integer,parameter::SCFD_MAX_TRANS_SEC = 5
   integer,parameter::SCFD_BC_MAXVAL     = 2*SCFD_MAX_SPECIES+8
   integer(c_int32_t),parameter::SCFD_BC_EXTRAP = 0, SCFD_BC_FIXED = 1, SCFD_BC_OUTFLOW_P = 2, &
                                 SCFD_BC_SLIP = 3, SCFD_BC_NOSLIP = 4, SCFD_BC_FIXED_PIN = 5
   integer(c_int32_t),parameter::SCFD_SIDE_ILO = 0, SCFD_SIDE_IHI = 1, SCFD_SIDE_JLO = 2, SCFD_SIDE_JHI = 3

   type,bind(C)::scfd_desc
      integer(c_int32_t)::abi_version, nplane
      integer(c_int32_t)::ni(SCFD_MAX_PLANES), nj(SCFD_MAX_PLANES)
      integer(c_int32_t)::ny, dim, dt_mode, scheme, recon, viscous, thermo, mu_model, &
                          precision, quirk_q1, num_internal_loop, il_write
      real(c_double)    ::phi_mus, k_mus, kappa, rgas, nu_gas, suth_mu0, suth_t0, suth_s, &
                          prandtl, schmidt, cfl, dt_fixed, omega_max, omega_min, dq_max, &
                          res_rate_warn, res_rate_err
      integer(c_int32_t)::chem_max_substeps, pad0
      real(c_double)    ::cfl_tau
      integer(c_int32_t)::reserved(12)
   end type

   type,bind(C)::scfd_bc
      integer(c_int32_t)::plane, side, first, last, kind, pad
      real(c_double)    ::value(SCFD_BC_MAXVAL+2)
   end type

   type,bind(C)::scfd_stats
      real(c_double)    ::dt_grbl, tt, res, res1, omega
      integer(c_int32_t)::status, inner_iters
      integer(c_int64_t)::chem_attempts, chem_fallback_cells
      integer(c_int32_t)::res_warn, reserved(7)
   end type

   type,bind(C)::scfd_chem
      integer(c_int32_t)::ns, nr, nt, pad0
      real(c_double)    ::coeff(7,2,SCFD_MAX_SPECIES)
      real(c_double)    ::tthre(3,SCFD_MAX_SPECIES)
      real(c_double)    ::mws(SCFD_MAX_SPECIES)
      integer(c_int32_t)::rstate(2,SCFD_MAX_REACTIONS)
      integer(c_int32_t)::indnu(3,2,SCFD_MAX_REACTIONS)
      integer(c_int32_t)::numnu(2,SCFD_MAX_REACTIONS)
      integer(c_int32_t)::snu(SCFD_MAX_REACTIONS)
      integer(c_int32_t)::exist_m(SCFD_MAX_REACTIONS)
      integer(c_int32_t)::numm(SCFD_MAX_REACTIONS)
      integer(c_int32_t)::indm(SCFD_MAX_SPECIES,SCFD_MAX_REACTIONS)
      real(c_double)    ::men(SCFD_MAX_SPECIES,SCFD_MAX_REACTIONS)
      real(c_double)    ::abe(3,SCFD_MAX_REACTIONS)
      real(c_double)    ::cabe(3,SCFD_MAX_REACTIONS)
      real(c_double)    ::troe(4,SCFD_MAX_REACTIONS)
      integer(c_int32_t)::tr2th(SCFD_MAX_SPECIES)
      integer(c_int32_t)::num_sctn_trans(SCFD_MAX_SPECIES)
      real(c_double)    ::trange_trans(2,SCFD_MAX_TRANS_SEC,SCFD_MAX_SPECIES)
      real(c_double)    ::trans(4,SCFD_MAX_TRANS_SEC,SCFD_MAX_SPECIES)
      real(c_double)    ::rtol, atol
   end type

   interface
      integer(c_int) function scfd_create(desc, ctx) bind(C, name="scfd_create")
         import; type(scfd_desc),intent(in)::desc; type(c_ptr)::ctx
      end function
      integer(c_int) function scfd_destroy(ctx) bind(C, name="scfd_destroy")
         import; type(c_ptr),value::ctx
      end function
      integer(c_int) function scfd_set_geometry(ctx, plane, xh, rh) bind(C, name="scfd_set_geometry")
         import; type(c_ptr),value::ctx; integer(c_int),value::plane
         real(c_double),intent(in)::xh(*), rh(*)
      end function
      integer(c_int) function scfd_set_connectivity(ctx, recs, n) bind(C, name="scfd_set_connectivity")
         import; type(c_ptr),value::ctx; integer(c_int32_t),intent(in)::recs(11,*)
         integer(c_int),value::n
      end function
      integer(c_int) function scfd_set_bc(ctx, descs, n) bind(C, name="scfd_set_bc")
         import; type(c_ptr),value::ctx; type(scfd_bc),intent(in)::descs(*); integer(c_int),value::n
      end function
      integer(c_int) function scfd_set_chem(ctx, chem) bind(C, name="scfd_set_chem")
         import; type(c_ptr),value::ctx; type(scfd_chem),intent(in)::chem
      end function
      integer(c_int) function scfd_commit(ctx) bind(C, name="scfd_commit")
         import; type(c_ptr),value::ctx
      end function
      integer(c_int) function scfd_upload(ctx, q, w, vhi, tt) bind(C, name="scfd_upload")
         import; type(c_ptr),value::ctx
         real(c_double),intent(in)::q(*), w(*), vhi(*); real(c_double),value::tt
      end function
      integer(c_int) function scfd_prepare(ctx, step) bind(C, name="scfd_prepare")
         import; type(c_ptr),value::ctx; integer(c_int),value::step
      end function
      integer(c_int) function scfd_step(ctx, step, stats) bind(C, name="scfd_step")
         import; type(c_ptr),value::ctx; integer(c_int),value::step; type(scfd_stats)::stats
      end function
      integer(c_int) function scfd_download(ctx, q, w, vhi, tt) bind(C, name="scfd_download")
         import; type(c_ptr),value::ctx; real(c_double)::q(*), w(*), vhi(*), tt
      end function
      integer(c_int) function scfd_download_qp(ctx, qp) bind(C, name="scfd_download_qp")
         import; type(c_ptr),value::ctx; real(c_double)::qp(*)
      end function
      integer(c_int) function scfd_last_error(ctx, buf, n) bind(C, name="scfd_last_error")
         import; type(c_ptr),value::ctx; character(kind=c_char)::buf(*); integer(c_int),value::n
      end function
   end interface
end module scfd_b200_iface
