/*
 * CPU oracle for the visibility hot path (TEST INFRASTRUCTURE ONLY; see
 * oskar_oracle.h). The precision-generic body is instantiated once for
 * double and once for float.
 */
#include <math.h>
#include <stddef.h>
#include <stdint.h>
#include <stdlib.h>
#include "oskar_oracle.h"

#define ORC_PI 3.14159265358979323846264338327950288
#define ORC_OMEGA_EARTH 7.272205217e-5 /* rad/s, as the reference uses */

#define ORC_CAT_(A, B) A##_##B
#define ORC_CAT(A, B) ORC_CAT_(A, B)

/* ---- double ---- */
#define REAL double
#define ORC_T(X) ORC_CAT(X, dbl)
#define ORC_FN(X) ORC_CAT(X, d)
#define ORC_SIN sin
#define ORC_COS cos
#define ORC_EXP exp
#define ORC_SQRT sqrt
#define ORC_LOG log
#define ORC_ATAN2 atan2
#define ORC_FMOD fmod
#define ORC_KAHAN 0
#include "oskar_oracle_body.h"
#undef REAL
#undef ORC_T
#undef ORC_FN
#undef ORC_SIN
#undef ORC_COS
#undef ORC_EXP
#undef ORC_SQRT
#undef ORC_LOG
#undef ORC_ATAN2
#undef ORC_FMOD
#undef ORC_KAHAN

/* ---- float ---- */
#define REAL float
#define ORC_T(X) ORC_CAT(X, flt)
#define ORC_FN(X) ORC_CAT(X, f)
#define ORC_SIN sinf
#define ORC_COS cosf
#define ORC_EXP expf
#define ORC_SQRT sqrtf
#define ORC_LOG logf
#define ORC_ATAN2 atan2f
#define ORC_FMOD fmodf
#define ORC_KAHAN 1
#include "oskar_oracle_body.h"
