/* TEST INFRASTRUCTURE ONLY — link-time stand-in for sysconf() in the
 * macro-path build of the reference (oracle/Makefile, target ref_macro:
 * -Wl,--wrap=sysconf). No reference file is edited: the reference's cache
 * probe (src/common/zldsp_fft_common_system.hpp:23-124) calls sysconf(), and
 * the linker sends those calls here.
 *
 * It reports the caches of a small-cache host: L1d 48 KiB, L2 1 MiB, no L3.
 * The reference's own switch (system.hpp:132-157) then gives
 *   float:  max_l1_order 10, switch_order 14
 *   double: max_l1_order  9, switch_order 13
 * so every CFFT of order >= 14 (float) / 13 (double), and every RFFT whose
 * inner CFFT is that large, runs the reference's Cooley-Tukey DIF macro path
 * (src/common/zldsp_fft_common_execute.hpp:174-272). Every other query goes to
 * the real sysconf. */
#include <unistd.h>

extern "C" long __real_sysconf(int name);

extern "C" long __wrap_sysconf(int name) {
    switch (name) {
    case _SC_LEVEL1_DCACHE_SIZE:
        return 48L * 1024;
    case _SC_LEVEL2_CACHE_SIZE:
        return 1024L * 1024;
    case _SC_LEVEL3_CACHE_SIZE:
        return 0;
    default:
        return __real_sysconf(name);
    }
}
