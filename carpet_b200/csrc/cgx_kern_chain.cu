// cgx_kern_chain.cu -- the chain kernel (cgx_chain.cuh) in both
// floating-point modes, vertex-centred prolongation orders 1/3/5, tile
// configuration 1 of the TMA prolongation (TMA_CFGS).
#include "cgx_chain.cuh"

namespace cgx {
int klaunch_chain(int fp, int order, const Desc *d, const CUtensorMap *maps, const ChainTile *tiles,
                  long long ntiles, const unsigned *need, unsigned *done, int ncounters,
                  unsigned long long *ctl, int *status, cudaStream_t s) {
  constexpr int CFG = 1;
#define CGX_CHAIN_CASE(F, O)                                                                              \
  if (fp == F && order == O)                                                                              \
    return kern::launch_chain_t<F, O, CFG>(d, maps, tiles, ntiles, need, done, ncounters, ctl, status, s);
  CGX_CHAIN_CASE(0, 1) CGX_CHAIN_CASE(0, 3) CGX_CHAIN_CASE(0, 5)
  CGX_CHAIN_CASE(1, 1) CGX_CHAIN_CASE(1, 3) CGX_CHAIN_CASE(1, 5)
#undef CGX_CHAIN_CASE
  return set_error(CGX_EUNSUPPORTED, "chain: no kernel for vertex-centred order %d", order);
}
} // namespace cgx
