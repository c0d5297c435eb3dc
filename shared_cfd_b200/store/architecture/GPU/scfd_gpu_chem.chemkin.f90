! The Chemkin tables of module chem (filled by init_therm from chem.inp,
! MW.inp, trans.inp and control_chem.inp, species already reordered) copied
! into scfd_chem for scfd_set_chem; species indices become 0-based.
module scfd_gpu_chem
   use iso_c_binding
   use scfd_b200_iface
   implicit none
contains
   subroutine scfd_gpu_chem_set(ctx)
      use chem
      type(c_ptr),intent(in)::ctx
      type(scfd_chem),save::ch
      integer(c_int)::ierr
      integer k
      ch%ns = ns
      ch%nr = max(nr, 1)
      ch%nt = nt
      ch%pad0 = 0
      ch%coeff = 0d0; ch%tthre = 0d0; ch%mws = 0d0
      ch%rstate = 0; ch%indnu = 0; ch%numnu = 0; ch%snu = 0; ch%exist_m = 0; ch%numm = 0; ch%indm = 0
      ch%men = 0d0; ch%abe = 0d0; ch%cabe = 0d0; ch%troe = 0d0
      ch%tr2th = 0; ch%num_sctn_trans = 0; ch%trange_trans = 0d0; ch%trans = 0d0
      ch%coeff(:,:,1:ns) = coeff(:,:,1:ns)
      ch%tthre(:,1:ns) = Tthre(:,1:ns)
      ch%mws(1:ns) = MWs(1:ns)
      do k=1,nr
         ch%rstate(1,k) = Rstate(k,1)
         ch%rstate(2,k) = Rstate(k,2)
         ch%indnu(:,:,k) = IndNu(:,:,k) - 1
         ch%numnu(:,k) = NumNu(:,k)
         ch%snu(k) = snu(k)
         ch%exist_m(k) = merge(1, 0, exist_M(k))
         ch%numm(k) = NumM(k)
         ch%indm(1:ns,k) = IndM(1:ns,k) - 1
         ch%men(1:ns,k) = Men(1:ns,k)
         ch%abe(:,k) = ABE(:,k)
         ch%cabe(:,k) = cABE(:,k)
         ch%troe(:,k) = TROE(:,k)
      end do
      ch%tr2th(1:nt) = tr2th(1:nt) - 1
      ch%num_sctn_trans(1:nt) = num_sctn_trans(1:nt)
      ch%trange_trans(:,:,1:nt) = Trange_trans(:,:,1:nt)
      ch%trans(:,:,1:nt) = trans(:,:,1:nt)
      ch%rtol = rtol_user
      ch%atol = atol_user
      ierr = scfd_set_chem(ctx, ch)
      if(ierr .ne. 0) then
         print *,"Error: scfd_set_chem returned status ",ierr
         stop
      end if
   end subroutine scfd_gpu_chem_set
end module scfd_gpu_chem
