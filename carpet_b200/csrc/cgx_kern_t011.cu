// cgx_kern_t011.cu -- TMA-staged prolongation kernels, exact mode,
// families CC<2>, CC<3>, CC<4>, CC<5>, ENO, tile configuration 1 (TMA_CFGS).
#include "cgx_kern_launch.cuh"

namespace cgx {
int klaunch_tma_f0_p1_c1(int variant, const Desc *d, const CUtensorMap *maps, const int2 *tmap,
                         long long ntiles, unsigned long long *counter, int *status, cudaStream_t s) {
  switch ((variant & ~(1 << 30)) / 4) { // bit 30: failure injection
  case 5: return kern::launch_tma_family<0, CC<2>, 1>(variant, d, maps, tmap, ntiles, counter, status, s);
  case 6: return kern::launch_tma_family<0, CC<3>, 1>(variant, d, maps, tmap, ntiles, counter, status, s);
  case 7: return kern::launch_tma_family<0, CC<4>, 1>(variant, d, maps, tmap, ntiles, counter, status, s);
  case 8: return kern::launch_tma_family<0, CC<5>, 1>(variant, d, maps, tmap, ntiles, counter, status, s);
  case 9: return kern::launch_tma_family<0, ENO, 1>(variant, d, maps, tmap, ntiles, counter, status, s);
  }
  return set_error(CGX_EINVAL, "bad prolongation variant %d", variant);
}
} // namespace cgx
