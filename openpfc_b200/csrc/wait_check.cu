// wait_check.cu -- the bounded mbarrier wait of the pipelined pass kernels,
// run on a barrier that nothing ever completes, so that its expiry path can be
// exercised on a GPU without a fault: the wait gives up after the given limit of
// %globaltimer, the CTA records the timeout bit (2) in the handle's status flag
// and returns; opfc_sync then reports OPFC_ERR_TIMEOUT and the context stays
// usable.  No copy is in flight, so nothing lands in shared memory after the
// CTA has left.
#include "kernels.cuh"

namespace opfc {

__global__ void wait_check_kernel(unsigned *flag, unsigned long long limit_ns) {
  __shared__ uint64_t bar;
  if (threadIdx.x == 0) {
    mbar_init(&bar, 1);  // one arrival expected; none is ever made
    mbar_fence_init();
  }
  __syncthreads();
  const bool ok = mbar_wait(&bar, 0, limit_ns);  // phase 0 never completes
  if (!__syncthreads_and(ok) && threadIdx.x == 0) atomicOr(flag, 2u);
}

int launch_wait_check(unsigned *flag, double limit_ms, cudaStream_t s) {
  if (!flag || !(limit_ms >= 0.1 && limit_ms <= 1000.0)) return (int)cudaErrorInvalidValue;
  wait_check_kernel<<<1, 32, 0, s>>>(flag, (unsigned long long)(limit_ms * 1e6));
  return (int)cudaGetLastError();
}

}  // namespace opfc
