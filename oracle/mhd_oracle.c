/* Oracle: CPU restatement of the reference time step.  TEST INFRASTRUCTURE
 * ONLY (see mhd_oracle.h).  The body is instantiated for float (the
 * reference's FP32 build) and for double (Real = double). */
#include "mhd_oracle.h"

#include <math.h>
#include <stdlib.h>
#include <string.h>

#define real float
#define FN(name) name##_f32
#define R_SQRT sqrtf
#define R_FABS fabsf
#define R_FMAX fmaxf
#define R_FMIN fminf
#include "mhd_oracle_body.h"
#undef real
#undef FN
#undef R_SQRT
#undef R_FABS
#undef R_FMAX
#undef R_FMIN
#undef F_RHO
#undef F_VX
#undef F_P
#undef F_BX

#define real double
#define FN(name) name##_f64
#define R_SQRT sqrt
#define R_FABS fabs
#define R_FMAX fmax
#define R_FMIN fmin
#include "mhd_oracle_body.h"
