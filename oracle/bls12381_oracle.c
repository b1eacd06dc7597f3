/*
 * CPU oracle for the BLS12-381 G1 multi-scalar multiplication path.
 *
 * TEST INFRASTRUCTURE ONLY, like bn254_oracle.c, whose algorithms (the
 * reference's halo2 multiexp_serial / best_multiexp, core/tests/msm_halo2.rs,
 * Jacobian formulas, the seeded generators) msm_oracle.inc restates once per
 * curve.  The reference serves BLS12-381 as its second curve: Rust operator
 * core/src/msm.rs:24-34 (381-bit points, 255-bit scalars over halo2curves'
 * bls12381), CUDA parameters core/src/common/mont/src/bls12381_fq.cuh,
 * bls12381_fr.cuh and core/src/common/curve/src/bls12381.cuh (b = 4).
 * C ABI layout: Fq in 12 little-endian u32 limbs (Montgomery, R = 2^384),
 * affine points 24 u32 (x then y), Fr in 8 u32 (Montgomery, R = 2^256).
 * The generator is the standard BLS12-381 G1 generator.
 */
#include "msm_oracle.h"

/* p = 0x1a0111ea...ffffaaab (core/src/common/mont/src/bls12381_fq.cuh:23) */
static const fparams FQ = {
    6,
    {0xb9feffffffffaaabULL, 0x1eabfffeb153ffffULL, 0x6730d2a0f6b0f624ULL, 0x64774b84f38512bfULL,
     0x4b1ba7b6434bacd7ULL, 0x1a0111ea397fe69aULL},
    0x89f3fffcfffcfffdULL,
    {0x760900000002fffdULL, 0xebf4000bc40c0002ULL, 0x5f48985753c758baULL, 0x77ce585370525745ULL,
     0x5c071a97a256ec6dULL, 0x15f65ec3fa80e493ULL},
    {0xf4df1f341c341746ULL, 0x0a76e6a609d104f1ULL, 0x8de5476c4c95b6d5ULL, 0x67eb88a9939d83c0ULL,
     0x9a793e85b519952dULL, 0x11988fe592cae3aaULL},
};

/* r = 0x73eda753...00000001 (core/src/common/mont/src/bls12381_fr.cuh:21) */
static const fparams FR = {
    4,
    {0xffffffff00000001ULL, 0x53bda402fffe5bfeULL, 0x3339d80809a1d805ULL, 0x73eda753299d7d48ULL},
    0xfffffffeffffffffULL,
    {0x00000001fffffffeULL, 0x5884b7fa00034802ULL, 0x998c4fefecbc4ff5ULL, 0x1824b159acc5056fULL},
    {0xc999e990f3f29c6dULL, 0x2b6cedcb87925c23ULL, 0x05d314967254398fULL, 0x0748d9d99f59ff11ULL},
};

#define CURVE_B 4
#define SCALAR_BITS 255
static const uint64_t GEN_X[FE_MAX] = {0xfb3af00adb22c6bbULL, 0x6c55e83ff97a1aefULL, 0xa14e3a3f171bac58ULL,
                                       0xc3688c4f9774b905ULL, 0x2695638c4fa9ac0fULL, 0x17f1d3a73197d794ULL};
static const uint64_t GEN_Y[FE_MAX] = {0x0caa232946c5e7e1ULL, 0xd03cc744a2888ae4ULL, 0x00db18cb2c04b3edULL,
                                       0xfcf5e095d5d00af6ULL, 0xa09e30ed741d8ae4ULL, 0x08b3f481e3aaa0f1ULL};

#define ORC(name) orc_bls_##name

#include "msm_oracle.inc"
