// cgx_kern_t004.cu -- TMA-staged prolongation kernels, exact mode,
// families VC<1>, VC<3>, VC<5>, CC<0>, CC<1>, tile configuration 4 (TMA_CFGS).
#include "cgx_kern_launch.cuh"

namespace cgx {
int klaunch_tma_f0_p0_c4(int variant, const Desc *d, const CUtensorMap *maps, const int2 *tmap,
                         long long ntiles, unsigned long long *counter, int *status, cudaStream_t s) {
  switch ((variant & ~(1 << 30)) / 4) { // bit 30: failure injection
  case 0: return kern::launch_tma_family<0, VC<1>, 4>(variant, d, maps, tmap, ntiles, counter, status, s);
  case 1: return kern::launch_tma_family<0, VC<3>, 4>(variant, d, maps, tmap, ntiles, counter, status, s);
  case 2: return kern::launch_tma_family<0, VC<5>, 4>(variant, d, maps, tmap, ntiles, counter, status, s);
  case 3: return kern::launch_tma_family<0, CC<0>, 4>(variant, d, maps, tmap, ntiles, counter, status, s);
  case 4: return kern::launch_tma_family<0, CC<1>, 4>(variant, d, maps, tmap, ntiles, counter, status, s);
  }
  return set_error(CGX_EINVAL, "bad prolongation variant %d", variant);
}
} // namespace cgx
