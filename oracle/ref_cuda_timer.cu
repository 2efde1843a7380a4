// ref_cuda_timer.cu -- times the reference's own CUDA time step on the GPU.
//
// TEST INFRASTRUCTURE ONLY (a reported baseline, not the product).  Built by
// oracle/build_ref.py together with the reference's unmodified
// src/iteration_host.cu (its kernels) and src/multiphase_lbm.cu (its host
// driver: command file, positions file, voxeliser, initial density) for one
// compiled-in lattice size.
//
// The set-up is the reference's run_gpu (src/multiphase_lbm.cu:565-593):
// prefetch of the managed density and mask, transfer_parameter,
// multiphaselbm_initialization.  Then `warmup` calls of
// multiphaselbm_iteration (src/iteration_host.cu:73-81: do_streaming,
// treat_boundary, do_collision, do_swap) and `repeats` blocks of `steps`
// calls, each block bracketed by CUDA events on the legacy default stream
// the reference launches on.  The statistics the reference computes on the
// host every statPeriod steps are not part of the step and are not run.
//
// Usage: ref_cuda_timer <commandFile> <warmup> <steps> <repeats>
// Prints one line per block: "block <r> ms_per_step <t>".
#include <cstdio>
#include <cstdlib>

#include "iteration_host.h"
#include "multiphase_lbm.h"

int main(int argc, char** argv) {
  if (argc != 5) {
    std::fprintf(stderr, "usage: %s commandFile warmup steps repeats\n", argv[0]);
    return 2;
  }
  const long warmup = std::atol(argv[2]);
  const long steps = std::atol(argv[3]);
  const long repeats = std::atol(argv[4]);
  if (warmup < 0 || steps < 1 || repeats < 1) {
    std::fprintf(stderr, "warmup >= 0, steps >= 1, repeats >= 1\n");
    return 2;
  }
  MultiphaseLBM box;
  box.read_data(argv[1]);

  const size_t nbytes_real = lx * ly * lz * sizeof(real);
  const size_t nbytes_bool = lx * ly * lz * sizeof(bool);
  int device = 0;
  cudaErrorCheck(cudaGetDevice(&device));
  cudaErrorCheck(cudaMemPrefetchAsync(box.drho, nbytes_real, device, 0));
  cudaErrorCheck(cudaMemPrefetchAsync(box.dis_fluid, nbytes_bool, device, 0));
  transfer_parameter(&box.tau, &box.G, &box.carn_star, &box.T_Tc,
                     &box.rhol_spinodal, &box.rhog_spinodal,
                     &box.inject_density, &box.rho_inject_period,
                     &box.rho_increment, &box.rhos, &box.inject_position,
                     &box.statPeriod);
  multiphaselbm_initialization(&box.drho, &box.dpsi, &box.dpressure,
                               &box.dis_fluid, &box.dcollision_f,
                               &box.dstream_f, &box.dforce);
  cudaErrorCheck(cudaDeviceSynchronize());

  const int reverse = 1;
  long step = 0;
  for (long w = 0; w < warmup; ++w, ++step)
    multiphaselbm_iteration(step, box.statPeriod, reverse, box.inject_type);
  cudaErrorCheck(cudaDeviceSynchronize());
  cudaEvent_t e0, e1;
  cudaErrorCheck(cudaEventCreate(&e0));
  cudaErrorCheck(cudaEventCreate(&e1));
  for (long r = 0; r < repeats; ++r) {
    cudaErrorCheck(cudaEventRecord(e0, 0));
    for (long k = 0; k < steps; ++k, ++step)
      multiphaselbm_iteration(step, box.statPeriod, reverse, box.inject_type);
    cudaErrorCheck(cudaEventRecord(e1, 0));
    cudaErrorCheck(cudaEventSynchronize(e1));
    cudaErrorCheck(cudaGetLastError());
    float ms = 0.f;
    cudaErrorCheck(cudaEventElapsedTime(&ms, e0, e1));
    std::printf("block %ld ms_per_step %.6f\n", r, ms / (double)steps);
    std::fflush(stdout);
  }
  cudaEventDestroy(e0);
  cudaEventDestroy(e1);
  return 0;
}
