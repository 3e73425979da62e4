/* CPU oracle for the KIWI kernel-integral hot path in __float128 -- TEST INFRASTRUCTURE ONLY.
 *
 * The same algorithm as kiwi_oracle.c (oracle_core.inc) in 113-bit arithmetic with exact rational
 * constants: the geometry (bounding boxes, cell vertices) is still formed in double exactly as the
 * reference forms it, but every integral and sum is carried with ~34 significant digits.  Its results
 * are the "truth" used to measure the error of FP64 implementations (the reference's and the GPU's):
 * the reference's formulas cancel heavily in places, so two correct FP64 implementations with different
 * libm roundings can differ by far more than an ulp, and both are judged against this.
 */
#define _GNU_SOURCE
#include <math.h>
#include <stdio.h>
#include <quadmath.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

#include "../kiwi_b200/csrc/kernel_tables.h"

typedef struct OrStats {
    int64_t bbox_pairs, sphere_pairs, skipped_outside, neg_clamped, neg_warned;
} OrStats;

typedef __float128 R;
#define R_PI M_PIq
#define Q(a, b) ((__float128)(a) / (__float128)(b))
#define F_SQRT sqrtq
#define F_ACOS acosq
#define F_ATAN atanq
#define F_LOG logq
#define F_SIN sinq
#define F_COS cosq
#define F_FABS fabsq
#define F_ATANH atanhq
#define F_POW powq
#define F_FMIN fminq
#define F_FLOOR floorq
#define F_SINCOS sincosq
#define API(name) orq_##name

#include "oracle_core.inc"
