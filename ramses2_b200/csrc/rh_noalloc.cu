// rh_noalloc.cu — a Courant/conservation reduction that allocates nothing.
//
// Some hosts cannot let a library call cudaMalloc: solvers whose memory
// manager owns every byte of device memory (a fixed HBM budget handed out to
// resident problems), and time-critical loops that must not take the
// device-wide synchronisation cudaMalloc/cudaFree imply.  rh_cmpdt_noalloc serves them:
// the caller passes its own device input (the oct state) and device output
// (5 doubles), and the per-block partial sums live in a file-scope device
// array of fixed size instead of library-allocated memory.
#include <cuda_runtime.h>

#include <cmath>
#include <mutex>

#include "rh_internal.h"
#include "rh_device.cuh"

namespace rh {
// Defined in rh_api.cu: per-block courant_fine partials and their reduction.
__global__ void cmpdt_kernel(const double* __restrict__ ud, const float* __restrict__ uf, int fp32,
                             const uint8_t* __restrict__ refined, long long oct0, long long noct, CflConst C,
                             double vol, double* __restrict__ partial, const uint8_t* __restrict__ refbits);
__global__ void reduce_partials_kernel(const double* __restrict__ partial, long long n, double dt0,
                                       double* __restrict__ out);
}  // namespace rh

namespace {

constexpr int kThreads = 256;                                    // cells per block (32 octs)
constexpr long long kMaxOcts = 2097152;                          // = one 256^3-cell level
constexpr long long kMaxBlocks = kMaxOcts * 8 / kThreads;        // 65,536 partials
constexpr int kMaxDevices = 64;

// Partial sums of one call: kMaxBlocks x (mass, ekin, eint, emag, dt),
// 2.6 MB held by every device that loads the library, until process exit.
static __device__ __align__(256) double g_noalloc_scratch[kMaxBlocks * 5];

std::mutex g_mu;
double* g_scratch_addr[kMaxDevices] = {};

// Device address of the scratch array on the current device (host code only
// sees a host-side stand-in under the array's name).  Looked up again on every
// call made outside stream capture, so an address cached before a device
// reset (a new context, with the array at a new address) is never used by an
// uncaptured call; a call on a stream that is being captured uses the address
// of the last uncaptured call on that device, and fails if there was none.
int scratch_address(cudaStream_t st, double** out) {
  int dev = 0;
  cudaError_t e = cudaGetDevice(&dev);
  if (e != cudaSuccess) return rh::cuda_fail(e, "cudaGetDevice");
  if (dev < 0 || dev >= kMaxDevices) {
    rh::set_error("rh_cmpdt_noalloc: device ordinal %d beyond %d", dev, kMaxDevices);
    return RH_EINVAL;
  }
  cudaStreamCaptureStatus cs = cudaStreamCaptureStatusNone;
  e = cudaStreamIsCapturing(st, &cs);
  const bool capturing = e != cudaSuccess || cs != cudaStreamCaptureStatusNone;
  if (e != cudaSuccess) (void)cudaGetLastError();  // the query's own error is not the caller's
  std::lock_guard<std::mutex> lk(g_mu);
  if (!capturing) {
    void* p = nullptr;
    e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
    if (e != cudaSuccess) return rh::cuda_fail(e, "cudaGetSymbolAddress(g_noalloc_scratch)");
    g_scratch_addr[dev] = static_cast<double*>(p);
  } else if (!g_scratch_addr[dev]) {
    rh::set_error("rh_cmpdt_noalloc: the first call on device %d must be made outside stream capture", dev);
    return RH_EINVAL;
  }
  *out = g_scratch_addr[dev];
  return RH_OK;
}

}  // namespace

extern "C" {

// Declared (with its limits and contract) in include/ramses_hydro_ext.h.
int rh_cmpdt_noalloc(const double* d_uold, int num_octs, const unsigned char* d_refined, double dx, double gamma,
                     double smallr, double smallc, double courant_factor, const double* constant_gravity,
                     double* d_out, void* stream) {
  if (!d_uold || !d_out) {
    rh::set_error("rh_cmpdt_noalloc: null device pointer");
    return RH_EINVAL;
  }
  if (num_octs < 1 || num_octs > kMaxOcts) {
    rh::set_error("rh_cmpdt_noalloc: num_octs=%d outside 1..%lld (the fixed scratch holds %lld block partials)",
                  num_octs, kMaxOcts, kMaxBlocks);
    return RH_EINVAL;
  }
  if (!(dx > 0) || !(gamma > 1) || !(smallc > 0) || !(courant_factor > 0)) {
    rh::set_error("rh_cmpdt_noalloc: need dx>0, gamma>1, smallc>0, courant_factor>0");
    return RH_EINVAL;
  }
  cudaStream_t st = static_cast<cudaStream_t>(stream);
  double* scratch = nullptr;
  int rc = scratch_address(st, &scratch);
  if (rc) return rc;
  rh::CflConst C;
  C.gamma = gamma;
  C.gm1 = gamma - 1.0;
  C.smallr = smallr;
  C.smallp = smallc * smallc / gamma;
  C.cdx_smallc = courant_factor * dx / smallc;
  C.two_cdx = 2.0 * courant_factor * dx;
  C.two_c = 2.0 * courant_factor;
  double gs = 0;
  for (int d = 0; d < 3; ++d) gs += std::fabs(constant_gravity ? constant_gravity[d] : 0.0);
  C.gsum_dx = gs * dx;
  C.k0 = C.two_cdx / (1.0 + std::sqrt(1.0 + C.two_c * 0.0001));
  C.ndim = 3;
  const long long ncell = (long long)num_octs * 8;
  const long long nblk = (ncell + kThreads - 1) / kThreads;
  rh::cmpdt_kernel<<<(unsigned)nblk, kThreads, 0, st>>>(d_uold, nullptr, 0, d_refined, 0, num_octs, C,
                                                         dx * dx * dx, scratch, nullptr);
  cudaError_t e = cudaGetLastError();
  if (e != cudaSuccess) return rh::cuda_fail(e, "cmpdt_kernel (noalloc)");
  rh::reduce_partials_kernel<<<1, 1024, 0, st>>>(scratch, nblk, dx / smallc, d_out);
  e = cudaGetLastError();
  if (e != cudaSuccess) return rh::cuda_fail(e, "reduce_partials_kernel (noalloc)");
  return RH_OK;
}

}  // extern "C"
