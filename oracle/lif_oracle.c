/*
 * TEST INFRASTRUCTURE ONLY — the CPU oracle for the GPU engine (see
 * lif_oracle.h). Instantiates lif_oracle_impl.h for the reference's float
 * build and for its double build (-DUSE_DOUBLE, src/utils/constant.h:12-16).
 */
#include <math.h>
#include <stdlib.h>
#include <string.h>

#include "lif_oracle.h"

#define REAL float
#define SFX(name) name##_f32
#define R_EXP expf
#define R_FABS fabsf
#define R_ROUND roundf
#include "lif_oracle_impl.h"
#undef REAL
#undef SFX
#undef R_EXP
#undef R_FABS
#undef R_ROUND

#define REAL double
#define SFX(name) name##_f64
#define R_EXP exp
#define R_FABS fabs
#define R_ROUND round
#include "lif_oracle_impl.h"
