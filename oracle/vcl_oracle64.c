/*
 * vcl_oracle64.c -- the C restatement (vcl_oracle.c) compiled with every
 * float as double, for the finite-difference gradient checks.  TEST
 * INFRASTRUCTURE ONLY.  Same functions and argument order as vcl_oracle.h,
 * with double arrays and double scalars wherever the header says float.
 */
#include <math.h>
#include <stdint.h>
#include <stddef.h>
#include <stdlib.h>
#include <string.h>
#define float double
#define expf exp
#define sqrtf sqrt
#define log2f log2
#define fabsf fabs
#define fminf fmin
#define fmaxf fmax
#define floorf floor
#define ceilf ceil
#define powf pow
#include "vcl_oracle.c"
