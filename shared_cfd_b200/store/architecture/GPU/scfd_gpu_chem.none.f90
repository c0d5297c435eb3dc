! no chemistry tables for this thermal model
module scfd_gpu_chem
   use iso_c_binding
   implicit none
contains
   subroutine scfd_gpu_chem_set(ctx)
      type(c_ptr),intent(in)::ctx
   end subroutine scfd_gpu_chem_set
end module scfd_gpu_chem
