/* TEST INFRASTRUCTURE ONLY — the oracle's scalar C restatement of the
 * reference's CFFT/RFFT algorithm (zldsp::fft: the micro-only Stockham path,
 * src/common/zldsp_fft_common_execute.hpp:26-144 with the passes of
 * src/common/zldsp_fft_common_radix.hpp and the RFFT pre/post steps of
 * execute.hpp:318-536; and, when zlo_set_hybrid_* selects it, the macro path
 * of execute.hpp:174-272 with the DIF stages of radix.hpp:670-843). Each
 * function cites the reference lines it follows.
 *
 * Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline leg may
 * load this library, and only to check results or as the timed CPU baseline. The
 * product (libzlfft_cuda.so) never calls it.
 *
 * Rounding follows the reference: every MulAdd / NegMulAdd of the reference
 * is an fma() here, every other operation is a separate IEEE operation, and
 * the file is compiled with -ffp-contract=off (oracle/Makefile). With
 * identical twiddle tables the output is bit-identical to the reference's
 * micro-only path, and to its macro path under the same switch (checked in
 * tests/test_oracle.py against the reference headers compiled here through
 * the Highway-API shim, the macro path through a build whose cache probe
 * reports a small-cache host).
 *
 * Pinning: the reference ships no tests or golden vectors for this path (its
 * CI accuracy scripts live in another repository), so this restatement is
 * pinned by (1) bit-equality with the reference's own code compiled here
 * (oracle/_ref/libzlref.so) and (2) an FP64 FFT (numpy.fft) plus analytic
 * known-answer tests.
 */
#define _GNU_SOURCE
#include <math.h>
#include <pthread.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

#define ZLO_F float
#define ZLO_SUF(name) name##_f32
#define ZLO_FMA fmaf
#include "zlfft_oracle_impl.h"
#undef ZLO_F
#undef ZLO_SUF
#undef ZLO_FMA

#define ZLO_F double
#define ZLO_SUF(name) name##_f64
#define ZLO_FMA fma
#include "zlfft_oracle_impl.h"
#undef ZLO_F
#undef ZLO_SUF
#undef ZLO_FMA
