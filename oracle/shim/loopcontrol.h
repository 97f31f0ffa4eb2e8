/* Stand-in for LoopControl's CCTK_LOOP3 macros: a plain OpenMP-shared
 * triple loop.  The operators are pointwise, so the loop order does not
 * change any result. */
#ifndef CGX_SHIM_LOOPCONTROL_H
#define CGX_SHIM_LOOPCONTROL_H
#define CCTK_LOOP3(name, i, j, k, imin, jmin, kmin, imax, jmax, kmax, ii, jj, kk) \
  _Pragma("omp for collapse(2)")                                              \
  for (int k = (kmin); k < (kmax); ++k)                                        \
    for (int j = (jmin); j < (jmax); ++j)                                      \
      for (int i = (imin); i < (imax); ++i)
#define CCTK_ENDLOOP3(name)
#endif
