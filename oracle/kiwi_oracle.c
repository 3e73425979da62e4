/* CPU oracle for the KIWI kernel-integral hot path, FP64 -- TEST INFRASTRUCTURE ONLY (see kiwi_oracle.h).
 *
 * The algorithm lives in oracle_core.inc; this unit instantiates it in double, following the reference's
 * arithmetic operation by operation (build with -ffp-contract=off) so that its results are bit-identical
 * to the reference's own CPU output.  The kernel coefficient tables come from
 * kiwi_b200/csrc/kernel_tables.h, which tests/test_kernel_tables.py pins to the reference's
 * src/kernel_spec_data.cpp values.
 */
#define _GNU_SOURCE
#include "kiwi_oracle.h"

#include <math.h>
#include <stdio.h>
#include <stdlib.h>
#include <string.h>

#include "../kiwi_b200/csrc/kernel_tables.h"

#ifndef M_PI
#define M_PI 3.14159265358979323846
#endif

typedef double R;
#define R_PI M_PI
#define Q(a, b) ((double)(a) / (double)(b))
#define F_SQRT sqrt
#define F_ACOS acos
#define F_ATAN atan
#define F_LOG log
#define F_SIN sin
#define F_COS cos
#define F_FABS fabs
#define F_ATANH atanh
#define F_POW pow
#define F_FMIN fmin
#define F_FLOOR floor
#define F_SINCOS sincos
#define API(name) or_##name

#include "oracle_core.inc"
