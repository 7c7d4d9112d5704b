// ref_msl_flag_driver.cpp — TEST INFRASTRUCTURE ONLY.
//
// The reference's Metal refinement-flag shader (metal/kernels/flag.metal, a
// float32 port of gpu/gpu_flag.cuf) compiled as C++ through msl_shim/; its
// hydro_flag_kernel is run one thread at a time.  Included from the reference
// checkout by the recipe (FLAG_METAL); nothing of it is copied here.
#include FLAG_METAL

extern "C" int ref_msl_hydro_flag(int* flag1, const int* nbor, const float* uold, int head_idx, int num_octs,
                                  float gamma, float smallr, float smallc2, float err_grad_d, float err_grad_p,
                                  float floor_d, float floor_p) {
  const int nblk = (num_octs + FLAG_TG_OCTS - 1) / FLAG_TG_OCTS;
  for (int b = 0; b < nblk; ++b)
    for (int t = 0; t < FLAG_TG_OCTS * 8; ++t)
      hydro_flag_kernel(flag1, nbor, uold, head_idx, num_octs, gamma, smallr, smallc2, err_grad_d, err_grad_p,
                        floor_d, floor_p, (uint)t, (uint)b);
  return 0;
}
