/*
 * Types shared by the CPU oracles (test infrastructure only; see
 * bn254_oracle.c).  A field element is up to FE_MAX 64-bit limbs; a field's
 * parameters carry its limb count n (BN254 Fq and Fr: 4; BLS12-381 Fq: 6,
 * Fr: 4) and limbs above n are kept zero.
 */
#ifndef MSM_ORACLE_H
#define MSM_ORACLE_H

#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

#define FE_MAX 6

typedef struct { uint64_t v[FE_MAX]; } fe;

typedef struct {
    int n;               /* 64-bit limbs */
    uint64_t m[FE_MAX];  /* modulus, little-endian 64-bit limbs */
    uint64_t inv;        /* -m^{-1} mod 2^64 */
    uint64_t r1[FE_MAX]; /* R mod m (Montgomery one), R = 2^(64 n) */
    uint64_t r2[FE_MAX]; /* R^2 mod m */
} fparams;

#endif
