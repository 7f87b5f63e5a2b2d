/* Test infrastructure only: the CPU oracle (see bf_oracle.h).  Instantiates the
 * type-generic body for float and double. */
#include "bf_oracle.h"

#include <float.h>
#include <math.h>
#include <stdlib.h>

/* Parameter counts, include/batchfit/models.hpp:79,103,128,160, and the reference
 * tests' own non-spectral models (Line P=2, Constant P=1, Exponential P=1). */
static unsigned bfo_pcount(int model) {
    static const unsigned counts[4] = {3, 3, 4, 8};
    if (model == BFO_LINE)
        return 2;
    if (model == BFO_CONSTANT || model == BFO_EXPONENTIAL)
        return 1;
    return counts[model];
}
static int bfo_spectral(int model) { return model >= 0 && model <= 3; }
static int bfo_known(int model) {
    return bfo_spectral(model) || model == BFO_LINE || model == BFO_CONSTANT || model == BFO_EXPONENTIAL;
}

#define REAL float
#define F(name) name##_f32
#define REAL_EPS FLT_EPSILON
#define REAL_MAX FLT_MAX
#define REAL_MIN FLT_MIN
#define EXPR(v) expf(v)
#define SQRTR(v) sqrtf(v)
#define FABSR(v) fabsf(v)
#define ISFINR(v) isfinite(v)
#define NANR NAN
#include "bf_oracle_body.h"
#undef REAL
#undef F
#undef REAL_EPS
#undef REAL_MAX
#undef REAL_MIN
#undef EXPR
#undef SQRTR
#undef FABSR
#undef ISFINR
#undef NANR
#undef BFO_LN2

#define REAL double
#define F(name) name##_f64
#define REAL_EPS DBL_EPSILON
#define REAL_MAX DBL_MAX
#define REAL_MIN DBL_MIN
#define EXPR(v) exp(v)
#define SQRTR(v) sqrt(v)
#define FABSR(v) fabs(v)
#define ISFINR(v) isfinite(v)
#define NANR ((double)NAN)
#include "bf_oracle_body.h"

void bfo_kahan_add_f32(float term, float *sum, float *correction) {
    kahan_f32(term, sum, correction);
}
