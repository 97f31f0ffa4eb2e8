/* Stand-in for CycleClock: provides no tick counter, so CarpetLib's
 * timestat.hh falls back to its own no-op timer definitions. */
#ifndef CGX_SHIM_CYCLECLOCK_H
#define CGX_SHIM_CYCLECLOCK_H
#endif
