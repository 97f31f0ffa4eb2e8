/* Stand-in for the Cactus parameter header: the CarpetLib parameters
 * the operator sources read.  OpenMP use follows cgx_shim_use_openmp. */
#ifndef CGX_SHIM_CCTK_PARAMETERS_H
#define CGX_SHIM_CCTK_PARAMETERS_H
extern "C" int cgx_shim_use_openmp;
#define DECLARE_CCTK_PARAMETERS                                              \
  const int use_openmp CCTK_ATTRIBUTE_UNUSED = cgx_shim_use_openmp;          \
  const int use_loopcontrol_in_operators CCTK_ATTRIBUTE_UNUSED = 0;          \
  const int deadbeef CCTK_ATTRIBUTE_UNUSED = 0xdeadbeef;
#endif
