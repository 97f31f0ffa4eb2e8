// cgx_kern_f1.cu -- kernels of floating-point mode 1 (0: two roundings per
// multiply-add, 1: fused), orders 0-5.
#include "cgx_kern_launch.cuh"

namespace cgx {
int klaunch_pair_f1(const Desc &d, int ntiles, int *status, cudaStream_t s) {
  return kern::launch_pair_t<1, false>(d, ntiles, status, s);
}
int klaunch_map_f1(const Desc *d, const int2 *tmap, long long ntiles, unsigned long long *counter,
                  int *status, cudaStream_t s) {
  return kern::launch_map_t<1>(d, tmap, ntiles, counter, status, s);
}
int klaunch_search_f1(const Desc *d, const long long *prefix, int ndesc, long long ntiles,
                     unsigned long long *counter, int *status, cudaStream_t s) {
  return kern::launch_search_t<1>(d, prefix, ndesc, ntiles, counter, status, s);
}
int klaunch_spair_f1(const Desc &d, int ntiles, int *status, cudaStream_t s) {
  return kern::launch_spair_t<1>(d, ntiles, status, s);
}
int klaunch_stream_f1(int variant, const Desc *d, const int2 *tmap, long long ntiles,
                     unsigned long long *counter, int *status, cudaStream_t s) {
  return kern::launch_stream_map_t<1>(variant, d, tmap, ntiles, counter, status, s);
}
} // namespace cgx
