/* Test infrastructure only (the oracle).  Builds liborc.so: the plain-C
 * restatement of SPAMS' omp / lasso2 coding path in double and float, see
 * sc_oracle_impl.h.  Parity of this restatement is pinned against the
 * reference itself (oracle/_ref, built by oracle/build_ref.sh) through the
 * committed fixtures in tests/golden/.  Only tests/, __graft_entry__.smoke()
 * and bench.py's CPU-baseline leg load it. */
#include <math.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#define T double
#define SUF f64
#include "sc_oracle_impl.h"
#undef T
#undef SUF

#define T float
#define SUF f32
#include "sc_oracle_impl.h"
#undef T
#undef SUF
