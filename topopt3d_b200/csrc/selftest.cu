// Self-test of the bounded grid-barrier wait (grid_barrier.cuh) that the
// persistent kernels -- the coarse-grid V-cycle, the OC bisection and the
// MMA update -- cross between their phases.
//
// A small cooperative grid crosses a number of barriers.  With a block told
// to leave before its first arrival, the counter never flips, so every
// other block's wait runs out after its poll limit, sets the fault slot and
// returns: the failure is detected on the host (tpo_barrier_selftest
// returns TPO_E_CUDA and resets the counter) without trapping or hanging
// the GPU.
#include "grid_barrier.cuh"
#include "tpo_internal.h"

namespace tpo {

namespace {

__global__ void k_barrier_selftest(unsigned int *bar, double *fault, int phases,
                                   int skip, int max_polls, double *passed) {
  if ((int)blockIdx.x == skip) return;   // this block never arrives
  for (int p = 0; p < phases; ++p)
    if (!grid_barrier(bar, fault, max_polls)) return;
  if (threadIdx.x == 0) atomicAdd(passed, 1.0);
}

}  // namespace

cudaError_t launch_barrier_selftest(const Ctx &c, int blocks, int phases, int skip,
                                    int max_polls, cudaStream_t s) {
  int per_sm = 0, sms = 0, dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return e;
  e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_barrier_selftest, 64, 0);
  if (e != cudaSuccess) return e;
  e = cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, dev);
  if (e != cudaSuccess) return e;
  if (blocks > per_sm * sms) return cudaErrorCooperativeLaunchTooLarge;
  double *passed = c.scal + SC_SELFTEST;
  e = cudaMemsetAsync(passed, 0, sizeof(double), s);
  if (e != cudaSuccess) return e;
  unsigned int *bar = c.gbar;
  double *fault = c.scal + kSlotFault;
  void *args[] = {&bar, &fault, &phases, &skip, &max_polls, &passed};
  count_launch();
  return cudaLaunchCooperativeKernel((const void *)k_barrier_selftest, blocks, 64,
                                     args, 0, s);
}

}  // namespace tpo
