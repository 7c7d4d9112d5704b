// rh_launch.h — registry of the compiled pencil-kernel instantiations.
#pragma once
#include <cuda_runtime.h>

#include "rh_godunov.cuh"
#include "rh_godunov2.cuh"

namespace rh {

// S: StateArgs<T>*, H: HydroK<V>* of the kernel's precision.
using LaunchFn = cudaError_t (*)(const LevelArgs& A, const void* S, const void* H, int nblocks, cudaStream_t st);

// minb: CTAs per SM the register allocation is sized for (launch bounds)
// amr: variant with the coarse-fine logic (flux reset at refined cells,
// corrections to father cells of interpolated ghosts, accumulate into unew)
struct KernelKey {
  int prec, txo, tyo, minb, slope, riemann, amr;
};

void register_launcher(const KernelKey& k, LaunchFn fn, size_t smem, int threads);
LaunchFn find_launcher(int prec, int txo, int tyo, int minb, int slope, int riemann, int amr,
                       size_t* smem = nullptr, int* threads = nullptr);
// All registered tile shapes of a precision (for the autotuner).
int list_tiles(int prec, int amr, int* txo, int* tyo, int* minb, int max);

template <int TXO, int TYO, int MINB, int SLOPE, int RIEMANN, bool AMR>
cudaError_t launch_f64(const LevelArgs& A, const void* S, const void* H, int nblocks, cudaStream_t st) {
  using G = Geo<double, double, TXO, TYO, (SLOPE == 3 ? 3 : 2)>;
  auto k = godunov_pencil_kernel<double, TXO, TYO, MINB, SLOPE, RIEMANN, AMR>;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::kSmem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  k<<<nblocks, G::NT, G::kSmem, st>>>(A, *static_cast<const StateArgs<double>*>(S),
                                      *static_cast<const HydroK<double>*>(H));
  return cudaGetLastError();
}

template <int TXO, int TYO, int MINB, int SLOPE, int RIEMANN, bool AMR>
cudaError_t launch_f32x2(const LevelArgs& A, const void* S, const void* H, int nblocks, cudaStream_t st) {
  using G = Geo<float, float2, TXO, TYO, (SLOPE == 3 ? 3 : 2)>;
  auto k = godunov_pencil2_kernel<TXO, TYO, MINB, SLOPE, RIEMANN, AMR>;
  static bool attr = false;
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)G::kSmem);
    if (e != cudaSuccess) return e;
    attr = true;
  }
  k<<<nblocks, G::NT, G::kSmem, st>>>(A, *static_cast<const StateArgs<float>*>(S),
                                      *static_cast<const HydroK<float2>*>(H));
  return cudaGetLastError();
}

template <typename T, int TXO, int TYO, int MINB, bool AMR = false> struct TileRegistrar {
  TileRegistrar() {
    if constexpr (sizeof(T) == 8) {
#define RH_REG(S, R)                                                                                              \
  register_launcher({RH_PREC_FP64, TXO, TYO, MINB, S, R, AMR}, &launch_f64<TXO, TYO, MINB, S, R, AMR>,          \
                    Geo<double, double, TXO, TYO, (S == 3 ? 3 : 2)>::kSmem, Geo<double, double, TXO, TYO>::NT);
      RH_REG(0, 1) RH_REG(0, 2) RH_REG(0, 3)
      RH_REG(1, 1) RH_REG(1, 2) RH_REG(1, 3)
      RH_REG(2, 1) RH_REG(2, 2) RH_REG(2, 3)
      RH_REG(3, 1) RH_REG(3, 2) RH_REG(3, 3)
#undef RH_REG
    } else {
#define RH_REG(S, R)                                                                                              \
  register_launcher({RH_PREC_FP32_BULK, TXO, TYO, MINB, S, R, AMR}, &launch_f32x2<TXO, TYO, MINB, S, R, AMR>,   \
                    Geo<float, float2, TXO, TYO, (S == 3 ? 3 : 2)>::kSmem, Geo<float, float2, TXO, TYO>::NT);
      RH_REG(0, 1) RH_REG(0, 2) RH_REG(0, 3)
      RH_REG(1, 1) RH_REG(1, 2) RH_REG(1, 3)
      RH_REG(2, 1) RH_REG(2, 2) RH_REG(2, 3)
      RH_REG(3, 1) RH_REG(3, 2) RH_REG(3, 3)
#undef RH_REG
    }
  }
};

}  // namespace rh
