/*
 * CPU oracle for the Seis 2-D acoustic FD path -- TEST INFRASTRUCTURE ONLY.
 * Instantiates seis_oracle_body.h in single and double precision.  Build with
 * contraction off (oracle/Makefile) so that every operation rounds on its own.
 */
#include "seis_oracle.h"
#include <math.h>
#include <stdlib.h>
#include <string.h>

#define REAL float
#define SFX f32
#define EXPR expf
#define SQRTR sqrtf
#include "seis_oracle_body.h"
#undef REAL
#undef SFX
#undef EXPR
#undef SQRTR

#define REAL double
#define SFX f64
#define EXPR exp
#define SQRTR sqrt
#include "seis_oracle_body.h"
#undef REAL
#undef SFX
#undef EXPR
#undef SQRTR
