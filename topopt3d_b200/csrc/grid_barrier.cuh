// Grid-wide barrier for persistent kernels whose blocks are all co-resident
// (a cooperative launch): the coarse-grid V-cycle (kernels_coarse.cu) and
// the OC bisection (kernels_design.cu).
#pragma once

namespace tpo {

// polls of one grid-barrier wait before it gives up (a poll is an L2 round
// trip, so this is seconds; a phase takes microseconds)
constexpr int kBarrierPolls = 1 << 22;

// Grid-wide barrier of the persistent kernel, a sense-reversing counter:
// block 0 adds 2^31 - (blocks - 1) and every other block adds 1, so once all
// blocks have arrived bit 31 has flipped and the low bits are back where
// they started (zero), ready for the next barrier or launch.  The arrival
// is an atomic with release semantics at GPU scope, made after the block
// barrier so it covers the writes of every thread of the block; the wait
// polls with acquire loads, and the closing block barrier passes the
// acquire on to the other threads.  (A barrier on a counter of our own is
// used rather than the cooperative-groups grid sync: with the latter the
// phase after each sync ran about twice as long on B200.)  A wait that runs
// out of polls (max_polls; the persistent kernels use kBarrierPolls, the
// self-test a few thousand) sets *fault (a device scalar the host reads
// back) and returns false; the caller then returns from the kernel.
__device__ __forceinline__ bool grid_barrier(unsigned int *bar, double *fault,
                                             int max_polls = kBarrierPolls) {
  __shared__ int ok;
  __syncthreads();
  if (threadIdx.x == 0) {
    const unsigned int add = blockIdx.x == 0 ? 0x80000000u - (gridDim.x - 1) : 1u;
    unsigned int old, cur;
    asm volatile("atom.add.release.gpu.u32 %0, [%1], %2;"
                 : "=r"(old) : "l"(bar), "r"(add) : "memory");
    int polls = 0;
    ok = 1;
    do {
      asm volatile("ld.acquire.gpu.u32 %0, [%1];" : "=r"(cur) : "l"(bar) : "memory");
      if (++polls > max_polls) {
        ok = 0;
        *(volatile double *)fault = 1.0;
        break;
      }
    } while (((old ^ cur) & 0x80000000u) == 0u);
  }
  __syncthreads();
  return ok != 0;
}

}  // namespace tpo
