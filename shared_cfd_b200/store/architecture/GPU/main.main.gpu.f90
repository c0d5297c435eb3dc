      ! one physical step of the configured scheme on the GPU (scfd_step);
      ! q, qp, w, vhi and tt come back to the host on the steps that
      ! check_convergence writes out
      call scfd_gpu_step(i)
