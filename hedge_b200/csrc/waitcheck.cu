// Failure-detection self-test (hb_op_wait_selftest): the bounded mbarrier
// wait of the tensor-core kernels, made to run out on purpose.  One CTA of
// one warp allocates tensor memory, waits with tc::mbar_wait on an mbarrier
// whose phase never completes (nothing arrives on it), raises the operator's
// device error flag when the limit passes, frees its tensor memory and
// returns; no MMA, bulk copy or other kernel is involved, so nothing is left
// in flight.
#include "common.cuh"
#include "tc.cuh"

namespace hb {

__global__ void __launch_bounds__(32, 1) wait_selftest_kernel(int* err, uint64_t limit_ns) {
  __shared__ __align__(8) uint64_t mbar;
  __shared__ uint32_t tmem_slot;
  if (threadIdx.x == 0) tc::mbar_init(&mbar, 1);
  tc::tmem_alloc(&tmem_slot, 32);
  tc::fence_before_sync();
  __syncthreads();
  tc::fence_after_sync();
  if (threadIdx.x == 0) {
    // phase 0 of an mbarrier that expects one arrival and never gets it
    if (!tc::mbar_wait(&mbar, 0u, limit_ns)) atomicCAS(err, 0, DEV_MMA_TIMEOUT);
  }
  tc::fence_before_sync();
  __syncthreads();
  tc::tmem_dealloc(tmem_slot, 32);
}

hb_status launch_wait_selftest(int* err, uint64_t limit_ns, cudaStream_t s) {
  wait_selftest_kernel<<<1, 32, 0, s>>>(err, limit_ns);
  HB_CUDA(cudaGetLastError());
  return HB_OK;
}

}  // namespace hb
