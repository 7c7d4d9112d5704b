// rh_selftest.cu — exercises the bounded mbarrier wait of the pencil kernels
// on a barrier that nothing arrives on: the wait gives up after `bound` polls,
// sets the device error word and the kernel returns; the host sees
// RH_ETIMEDOUT and the context stays usable.  No fault, trap or hang.
#include <cuda_runtime.h>

#include "rh_godunov.cuh"
#include "rh_internal.h"

namespace rh {
namespace {

__global__ void wait_selftest_kernel(int* err, long long bound) {
  __shared__ __align__(8) uint64_t bar;
  __shared__ int s_abort;
  if (threadIdx.x == 0) {
    s_abort = 0;
    mbar_init(&bar, 1);  // expects one arrival; none comes
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
  }
  __syncthreads();
  bounded_mbar_wait(&bar, 0, &s_abort, err, bound);
}

}  // namespace
}  // namespace rh

using namespace rh;

extern "C" int rh_selftest_wait(long long bound) {
  Context& c = ctx();
  if (!c.inited) {
    set_error("rh_selftest_wait: rh_init first");
    return RH_ESTATE;
  }
  if (bound < 1 || bound > (1ll << 20)) {
    set_error("rh_selftest_wait: bound must be in [1, 2^20]");
    return RH_EINVAL;
  }
  wait_selftest_kernel<<<1, 32, 0, c.stream>>>(c.d_err, bound);
  RH_CUDA(cudaGetLastError());
  return rh_sync();
}
