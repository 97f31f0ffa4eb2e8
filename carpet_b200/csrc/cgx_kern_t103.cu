// cgx_kern_t103.cu -- TMA-staged prolongation kernels, fused-multiply-add mode,
// families VC<1>, VC<3>, VC<5>, CC<0>, CC<1>, tile configuration 3 (TMA_CFGS).
#include "cgx_kern_launch.cuh"

namespace cgx {
int klaunch_tma_f1_p0_c3(int variant, const Desc *d, const CUtensorMap *maps, const int2 *tmap,
                         long long ntiles, unsigned long long *counter, int *status, cudaStream_t s) {
  switch ((variant & ~(1 << 30)) / 4) { // bit 30: failure injection
  case 0: return kern::launch_tma_family<1, VC<1>, 3>(variant, d, maps, tmap, ntiles, counter, status, s);
  case 1: return kern::launch_tma_family<1, VC<3>, 3>(variant, d, maps, tmap, ntiles, counter, status, s);
  case 2: return kern::launch_tma_family<1, VC<5>, 3>(variant, d, maps, tmap, ntiles, counter, status, s);
  case 3: return kern::launch_tma_family<1, CC<0>, 3>(variant, d, maps, tmap, ntiles, counter, status, s);
  case 4: return kern::launch_tma_family<1, CC<1>, 3>(variant, d, maps, tmap, ntiles, counter, status, s);
  }
  return set_error(CGX_EINVAL, "bad prolongation variant %d", variant);
}
} // namespace cgx
