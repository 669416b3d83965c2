/*
 * real.h - working precision of the CPU oracle (TEST INFRASTRUCTURE ONLY).
 *
 * Built plainly (liboracle_gm1.so) the oracle computes in binary32, one
 * operation at a time, as the reference's CPU twins do.  Built with
 * -DORACLE_F64 (liboracle_gm1_f64.so) every binary32 variable, array and
 * operation of the same source becomes binary64: the same operators in the
 * same order, evaluated in double precision - the FP64 run against which
 * each float32 prognostic field's rounding error is reported.  The
 * operators' constants keep their float32 spellings (1.0e-20f, 287.04f, ...):
 * only the arithmetic widens.  Included after the system headers.
 */
#ifndef ORACLE_REAL_H
#define ORACLE_REAL_H
#ifdef ORACLE_F64
#define float double
#define powf pow
#define expf exp
#define logf log
#define sqrtf sqrt
#define fabsf fabs
#define fminf fmin
#define fmaxf fmax
#define copysignf copysign
#define floorf floor
#define cosf cos
#define sinf sin
#endif
#endif
