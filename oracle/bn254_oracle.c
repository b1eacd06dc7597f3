/*
 * CPU oracle for the BN254 G1 multi-scalar multiplication (MSM) path.
 *
 * TEST INFRASTRUCTURE ONLY.  Only tests/, the smoke check and the CPU-baseline
 * leg of bench.py may load this library, and only as the checker.  The CUDA
 * product path never calls into it.
 *
 * What it restates, from the reference (SJTU-Liquid/Impeller):
 *   - the CPU MSM the reference checks its GPU MSM against:
 *       core/tests/msm_halo2.rs:63-151   multiexp_serial (unsigned c-bit
 *                                        windows, c = ceil(ln n), 2^c - 1
 *                                        buckets with None/Affine/Projective
 *                                        states, running-sum reduction)
 *       core/tests/msm_halo2.rs:182-208  best_multiexp (split into
 *                                        num_threads chunks, sum the chunks)
 *     The reference runs this over halo2curves 0.6.1 (Cargo.lock:415-418),
 *     which is Rust and cannot be built here; this file is a C restatement.
 *   - the data layout of the C ABI (core/src/msm/src/msm.h:4-11): 8
 *     little-endian u32 limbs per field element, Montgomery form with
 *     R = 2^256; affine points are x then y (16 u32); the identity is (0,0)
 *     (core/src/common/curve/src/curve_xyzz.cuh:204-210).
 *   - the BN254 parameters (core/src/common/mont/src/bn254_fq.cuh:9-75,
 *     core/src/common/mont/src/bn254_fr.cuh:1-75, curve b = 3 at
 *     core/src/common/curve/src/bn254.cuh:13-31).
 *   - the window-table precompute of core/src/msm/src/msm_impl.cuh:358-371
 *     (table j holds 2^(j * shift) * P_i in affine form).
 *
 * The arithmetic here is deliberately different from the CUDA product's:
 * 64-bit limbs with 128-bit products, and Jacobian (X, Y, Z) curve
 * formulas (dbl-2009-l, add-2007-bl, madd-2007-bl from the Explicit-Formulas
 * Database) instead of the product's XYZZ formulas.  A shared mistake would
 * have to be made twice in two different ways.
 *
 * The synthetic-input generators (splitmix64 counter streams -> uniform Fr,
 * the skewed witness-like mix, P_i = r_i * G) define the seeded inputs of
 * every test and benchmark; the CUDA library carries its own copy of the
 * same definitions and tests check the two agree bit for bit.
 *
 * The field, curve, generator and MSM code lives in msm_oracle.inc and is
 * compiled once per curve: here for BN254 (symbols orc_*), in
 * bls12381_oracle.c for BLS12-381 (symbols orc_bls_*).
 */
#include "msm_oracle.h"

/* Fq: base field of BN254 G1 (core/src/common/mont/src/bn254_fq.cuh:13-17). */
static const fparams FQ = {
    4,
    {0x3c208c16d87cfd47ULL, 0x97816a916871ca8dULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL},
    0x87d20782e4866389ULL,
    {0xd35d438dc58f0d9dULL, 0x0a78eb28f5c70b3dULL, 0x666ea36f7879462cULL, 0x0e0a77c19a07df2fULL},
    {0xf32cfc5b538afa89ULL, 0xb5e71911d44501fbULL, 0x47ab1eff0a417ff6ULL, 0x06d89f71cab8351fULL},
};

/* Fr: scalar field of BN254 (core/src/common/mont/src/bn254_fr.cuh). */
static const fparams FR = {
    4,
    {0x43e1f593f0000001ULL, 0x2833e84879b97091ULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL},
    0xc2e1f593efffffffULL,
    {0xac96341c4ffffffbULL, 0x36fc76959f60cd29ULL, 0x666ea36f7879462eULL, 0x0e0a77c19a07df2fULL},
    {0x1bb8e645ae216da7ULL, 0x53fe3ab1e35c59e3ULL, 0x8c49833d53bb8085ULL, 0x0216d0b17f4e44a5ULL},
};

/* y^2 = x^3 + 3 (core/src/common/curve/src/bn254.cuh:13-31); generator (1, 2). */
#define CURVE_B 3
#define SCALAR_BITS 254
static const uint64_t GEN_X[FE_MAX] = {1};
static const uint64_t GEN_Y[FE_MAX] = {2};

#define ORC(name) orc_##name

#include "msm_oracle.inc"
