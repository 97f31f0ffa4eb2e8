// cgx_kern_t114.cu -- TMA-staged prolongation kernels, fused-multiply-add mode,
// families CC<2>, CC<3>, CC<4>, CC<5>, ENO, tile configuration 4 (TMA_CFGS).
#include "cgx_kern_launch.cuh"

namespace cgx {
int klaunch_tma_f1_p1_c4(int variant, const Desc *d, const CUtensorMap *maps, const int2 *tmap,
                         long long ntiles, unsigned long long *counter, int *status, cudaStream_t s) {
  switch ((variant & ~(1 << 30)) / 4) { // bit 30: failure injection
  case 5: return kern::launch_tma_family<1, CC<2>, 4>(variant, d, maps, tmap, ntiles, counter, status, s);
  case 6: return kern::launch_tma_family<1, CC<3>, 4>(variant, d, maps, tmap, ntiles, counter, status, s);
  case 7: return kern::launch_tma_family<1, CC<4>, 4>(variant, d, maps, tmap, ntiles, counter, status, s);
  case 8: return kern::launch_tma_family<1, CC<5>, 4>(variant, d, maps, tmap, ntiles, counter, status, s);
  case 9: return kern::launch_tma_family<1, ENO, 4>(variant, d, maps, tmap, ntiles, counter, status, s);
  }
  return set_error(CGX_EINVAL, "bad prolongation variant %d", variant);
}
} // namespace cgx
