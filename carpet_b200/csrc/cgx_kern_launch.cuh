// cgx_kern_launch.cuh -- host launchers of one floating-point mode's
// kernels; included once per mode by cgx_kern_f0.cu / cgx_kern_f1.cu.
#pragma once
#include "cgx_kernels.cuh"

namespace cgx {
namespace kern {

template <int FMA, bool HIGH> int launch_pair_t(const Desc &d, int ntiles, int *status, cudaStream_t s) {
  static bool attr = false;
  const size_t smem = smem_bytes(HIGH);
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_pair<FMA, HIGH>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_error(e, "cudaFuncSetAttribute");
    attr = true;
  }
  k_pair<FMA, HIGH><<<ntiles, NTHREADS, smem, s>>>(d, status);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CGX_OK : cuda_error(e, "k_pair launch");
}

// grid of a persistent kernel: every CTA slot of the device, at most ntiles
// A launch that may begin while its stream predecessor finishes
// (programmatic dependent launch; the kernel waits with griddepcontrol
// before it touches memory).
template <class... P, class... A>
cudaError_t launch_chained(void (*kernel)(P...), int grid, int block, size_t smem, cudaStream_t s,
                           A... args) {
  cudaLaunchConfig_t cfg = {};
  cfg.gridDim = dim3((unsigned)grid);
  cfg.blockDim = dim3((unsigned)block);
  cfg.dynamicSmemBytes = smem;
  cfg.stream = s;
  cudaLaunchAttribute at[1];
  at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
  at[0].val.programmaticStreamSerializationAllowed = 1;
  cfg.attrs = at;
  cfg.numAttrs = 1;
  return cudaLaunchKernelEx(&cfg, kernel, args...);
}

template <class K>
int persistent_grid(K kernel, size_t smem, long long ntiles, int *grid, int threads = NTHREADS, int cap = 0) {
  int dev = 0, nsm = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  cudaError_t e = cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, kernel, threads, smem);
  if (e != cudaSuccess || per_sm < 1) per_sm = 1;
  if (cap > 0 && cap < per_sm) per_sm = cap;
  *grid = (int)std::min<long long>((long long)nsm * per_sm, ntiles);
  return CGX_OK;
}

template <int FMA>
int launch_map_t(const Desc *d_descs, const int2 *d_tmap, long long ntiles, unsigned long long *d_counter,
                 int *d_status, cudaStream_t s) {
  static bool attr = false;
  const size_t smem = smem_bytes(false);
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_batch_map<FMA>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_error(e, "cudaFuncSetAttribute");
    attr = true;
  }
  int grid = 0;
  persistent_grid(k_batch_map<FMA>, smem, ntiles, &grid);
  cudaError_t e = launch_chained(k_batch_map<FMA>, grid, NTHREADS, smem, s, d_descs, d_tmap, ntiles,
                                 d_counter, d_status);
  return e == cudaSuccess ? CGX_OK : cuda_error(e, "k_batch_map launch");
}

template <int FMA>
int launch_search_t(const Desc *d_descs, const long long *d_prefix, int ndesc, long long ntiles,
                    unsigned long long *d_counter, int *d_status, cudaStream_t s) {
  static bool attr = false;
  const size_t smem = smem_bytes(false);
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_batch<FMA>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_error(e, "cudaFuncSetAttribute");
    attr = true;
  }
  int grid = 0;
  persistent_grid(k_batch<FMA>, smem, ntiles, &grid);
  k_batch<FMA><<<grid, NTHREADS, smem, s>>>(d_descs, d_prefix, ndesc, ntiles, d_counter, d_status);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CGX_OK : cuda_error(e, "k_batch launch");
}

template <int FMA> int launch_spair_t(const Desc &d, int ntiles, int *status, cudaStream_t s) {
  k_spair<FMA><<<ntiles, NTHREADS, 0, s>>>(d, status);
  cudaError_t e = cudaGetLastError();
  return e == cudaSuccess ? CGX_OK : cuda_error(e, "k_spair launch");
}

template <int FMA, class F, int NTL, int TK, int CFG>
int launch_tma_v(int variant, const Desc *d_descs, const CUtensorMap *d_maps, const int2 *d_tmap,
                 long long ntiles, unsigned long long *d_counter, int *d_status, cudaStream_t s) {
  constexpr int NT = TMA_CFGS[CFG].nt;
  static bool attr = false;
  const size_t smem =
      sizeof(double) * TSmem<F, NTL, TMA_CFGS[CFG].pyc, TMA_CFGS[CFG].pd + 2>::total + 128; // + alignment slack
  if (!attr) {
    cudaError_t e = cudaFuncSetAttribute(k_tma_map<FMA, F, NTL, TK, CFG>,
                                         cudaFuncAttributeMaxDynamicSharedMemorySize, (int)smem);
    if (e != cudaSuccess) return cuda_error(e, "cudaFuncSetAttribute");
    attr = true;
  }
  int dev = 0, nsm = 0, per_sm = 0;
  cudaGetDevice(&dev);
  cudaDeviceGetAttribute(&nsm, cudaDevAttrMultiProcessorCount, dev);
  if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&per_sm, k_tma_map<FMA, F, NTL, TK, CFG>, NT, smem) !=
          cudaSuccess ||
      per_sm < 1)
    per_sm = 1;
  if (g_cta_cap[0] > 0 && g_cta_cap[0] < per_sm) per_sm = g_cta_cap[0];
  const int grid = (int)std::min<long long>((long long)nsm * per_sm, ntiles);
  cudaError_t e = launch_chained(k_tma_map<FMA, F, NTL, TK, CFG>, grid, NT, smem, s, d_descs, d_maps, d_tmap,
                                 ntiles, d_counter, d_status, variant);
  return e == cudaSuccess ? CGX_OK : cuda_error(e, "k_tma_map launch");
}

// the four time-interpolation variants of one family, in configuration CFG
template <int FMA, class F, int CFG>
int launch_tma_family(int variant, const Desc *d_descs, const CUtensorMap *d_maps, const int2 *d_tmap,
                      long long ntiles, unsigned long long *d_counter, int *d_status, cudaStream_t s) {
  switch (variant % 4) {
  case 0:
    return launch_tma_v<FMA, F, 1, T_NONE, CFG>(variant, d_descs, d_maps, d_tmap, ntiles, d_counter, d_status, s);
  case 1:
    return launch_tma_v<FMA, F, 2, T_LIN, CFG>(variant, d_descs, d_maps, d_tmap, ntiles, d_counter, d_status, s);
  case 2:
    return launch_tma_v<FMA, F, 3, T_QUAD, CFG>(variant, d_descs, d_maps, d_tmap, ntiles, d_counter, d_status, s);
  default:
    return launch_tma_v<FMA, F, 3, T_ENO, CFG>(variant, d_descs, d_maps, d_tmap, ntiles, d_counter, d_status, s);
  }
}

template <int FMA, int V>
int launch_stream_v(const Desc *d_descs, const int2 *d_tmap, long long ntiles,
                    unsigned long long *d_counter, int *d_status, cudaStream_t s) {
  int grid = 0;
  persistent_grid(k_stream_map<FMA, V>, 0, ntiles, &grid, STREAM_THREADS, g_cta_cap[1]);
  cudaError_t e = launch_chained(k_stream_map<FMA, V>, grid, STREAM_THREADS, 0, s, d_descs, d_tmap, ntiles,
                                 d_counter, d_status);
  return e == cudaSuccess ? CGX_OK : cuda_error(e, "k_stream_map launch");
}

template <int FMA>
int launch_stream_map_t(int variant, const Desc *d_descs, const int2 *d_tmap, long long ntiles,
                        unsigned long long *d_counter, int *d_status, cudaStream_t s) {
  switch (variant) {
  case SV_COPY1: return launch_stream_v<FMA, SV_COPY1>(d_descs, d_tmap, ntiles, d_counter, d_status, s);
  case SV_COPY2: return launch_stream_v<FMA, SV_COPY2>(d_descs, d_tmap, ntiles, d_counter, d_status, s);
  case SV_COPY3Q: return launch_stream_v<FMA, SV_COPY3Q>(d_descs, d_tmap, ntiles, d_counter, d_status, s);
  case SV_COPY3E: return launch_stream_v<FMA, SV_COPY3E>(d_descs, d_tmap, ntiles, d_counter, d_status, s);
  case SV_RESTRICT_VC:
    return launch_stream_v<FMA, SV_RESTRICT_VC>(d_descs, d_tmap, ntiles, d_counter, d_status, s);
  case SV_RESTRICT_CC:
    return launch_stream_v<FMA, SV_RESTRICT_CC>(d_descs, d_tmap, ntiles, d_counter, d_status, s);
  case SV_RESTRICT_CC3:
    return launch_stream_v<FMA, SV_RESTRICT_CC3>(d_descs, d_tmap, ntiles, d_counter, d_status, s);
  case SV_RESTRICT_CC5:
    return launch_stream_v<FMA, SV_RESTRICT_CC5>(d_descs, d_tmap, ntiles, d_counter, d_status, s);
  case SV_TIME:
    return launch_stream_v<FMA, SV_TIME>(d_descs, d_tmap, ntiles, d_counter, d_status, s);
  case SV_MONO:
    return launch_stream_v<FMA, SV_MONO>(d_descs, d_tmap, ntiles, d_counter, d_status, s);
  }
  return set_error(CGX_EINVAL, "bad streaming variant %d", variant);
}

} // namespace kern
} // namespace cgx
