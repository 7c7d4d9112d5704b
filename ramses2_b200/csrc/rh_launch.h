// rh_launch.h — registry of the compiled pencil-kernel instantiations.
#pragma once
#include <cuda_runtime.h>

#include "rh_godunov.cuh"

namespace rh {

using LaunchFn = cudaError_t (*)(const LevelArgs& A, const void* S, const void* H, int nblocks, cudaStream_t st);

struct KernelKey {
  int prec, txo, tyo, slope, riemann;
};

void register_launcher(const KernelKey& k, LaunchFn fn, size_t smem, int threads);
LaunchFn find_launcher(int prec, int txo, int tyo, int slope, int riemann, size_t* smem = nullptr,
                       int* threads = nullptr);
// All registered tile shapes of a precision (for the autotuner).
int list_tiles(int prec, int* txo, int* tyo, int max);

template <typename T, int TXO, int TYO, int SLOPE, int RIEMANN>
cudaError_t launch_pencil(const LevelArgs& A, const void* S, const void* H, int nblocks, cudaStream_t st) {
  using G = Geo<T, TXO, TYO>;
  auto k = godunov_pencil_kernel<T, TXO, TYO, SLOPE, RIEMANN>;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::kSmem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  k<<<nblocks, G::NT, G::kSmem, st>>>(A, *static_cast<const StateArgs<T>*>(S),
                                      *static_cast<const HydroConst<T>*>(H));
  return cudaGetLastError();
}

template <typename T, int TXO, int TYO> struct TileRegistrar {
  TileRegistrar() {
    constexpr int P = sizeof(T) == 8 ? RH_PREC_FP64 : RH_PREC_FP32_BULK;
    using G = Geo<T, TXO, TYO>;
#define RH_REG(S, R) register_launcher({P, TXO, TYO, S, R}, &launch_pencil<T, TXO, TYO, S, R>, G::kSmem, G::NT);
    RH_REG(0, 1) RH_REG(0, 2) RH_REG(0, 3)
    RH_REG(1, 1) RH_REG(1, 2) RH_REG(1, 3)
    RH_REG(2, 1) RH_REG(2, 2) RH_REG(2, 3)
#undef RH_REG
  }
};

}  // namespace rh
