// rh_selftest.cu — device self-tests for the test suite:
//  * the bounded mbarrier wait of the pencil kernels on a barrier that nothing
//    arrives on: the wait gives up after `bound` polls, sets the device error
//    word and the kernel returns; the host sees RH_ETIMEDOUT and the context
//    stays usable.  No fault, trap or hang;
//  * the FP64 lane reciprocal and square root of the pencil kernels (vrcp,
//    vsqrt: hardware estimates refined by Newton-Raphson steps) next to
//    CUDA's correctly rounded 1.0/x and sqrt(x), element by element.
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

__global__ void vmath_selftest_kernel(const double* __restrict__ x, long long n, double* __restrict__ out) {
  const long long i = blockIdx.x * (long long)blockDim.x + threadIdx.x;
  if (i >= n) return;
  const double v = x[i];
  out[i] = vrcp(v);
  out[n + i] = vsqrt(v);
  out[2 * n + i] = 1.0 / v;
  out[3 * n + i] = sqrt(v);
}

}  // namespace
}  // namespace rh

using namespace rh;

extern "C" int rh_selftest_vmath(const double* d_x, long long n, double* d_out) {
  Context& c = ctx();
  if (!c.inited) {
    set_error("rh_selftest_vmath: rh_init first");
    return RH_ESTATE;
  }
  if (!d_x || !d_out || n < 1) {
    set_error("rh_selftest_vmath: need device pointers and n >= 1");
    return RH_EINVAL;
  }
  vmath_selftest_kernel<<<(unsigned)((n + 255) / 256), 256, 0, c.stream>>>(d_x, n, d_out);
  RH_CUDA(cudaGetLastError());
  return rh_sync();
}

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
