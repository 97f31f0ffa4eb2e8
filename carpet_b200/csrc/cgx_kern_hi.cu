// cgx_kern_hi.cu -- per-box kernels of the vertex-centred orders 7/9/11,
// both floating-point modes (their wider windows get their own kernels).
#include "cgx_kern_launch.cuh"

namespace cgx {
int klaunch_pair_hi(int fp, const Desc &d, int ntiles, int *status, cudaStream_t s) {
  return fp ? kern::launch_pair_t<1, true>(d, ntiles, status, s)
            : kern::launch_pair_t<0, true>(d, ntiles, status, s);
}
} // namespace cgx
