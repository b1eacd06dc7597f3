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
 * 4 x 64-bit limbs with 128-bit products, and Jacobian (X, Y, Z) curve
 * formulas (dbl-2009-l, add-2007-bl, madd-2007-bl from the Explicit-Formulas
 * Database) instead of the product's XYZZ formulas.  A shared mistake would
 * have to be made twice in two different ways.
 *
 * The synthetic-input generators (splitmix64 counter streams -> uniform Fr,
 * the skewed witness-like mix, P_i = r_i * G) define the seeded inputs of
 * every test and benchmark; the CUDA library carries its own copy of the
 * same definitions and tests check the two agree bit for bit.
 */
#include <math.h>
#include <pthread.h>
#include <stdint.h>
#include <stdlib.h>
#include <string.h>

typedef unsigned __int128 u128;

typedef struct { uint64_t v[4]; } fe;

typedef struct {
    uint64_t m[4];   /* modulus, little-endian 64-bit limbs */
    uint64_t inv;    /* -m^{-1} mod 2^64 */
    uint64_t r1[4];  /* R mod m (Montgomery one) */
    uint64_t r2[4];  /* R^2 mod m */
} fparams;

/* Fq: base field of BN254 G1 (core/src/common/mont/src/bn254_fq.cuh:13-17). */
static const fparams FQ = {
    {0x3c208c16d87cfd47ULL, 0x97816a916871ca8dULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL},
    0x87d20782e4866389ULL,
    {0xd35d438dc58f0d9dULL, 0x0a78eb28f5c70b3dULL, 0x666ea36f7879462cULL, 0x0e0a77c19a07df2fULL},
    {0xf32cfc5b538afa89ULL, 0xb5e71911d44501fbULL, 0x47ab1eff0a417ff6ULL, 0x06d89f71cab8351fULL},
};

/* Fr: scalar field of BN254 (core/src/common/mont/src/bn254_fr.cuh). */
static const fparams FR = {
    {0x43e1f593f0000001ULL, 0x2833e84879b97091ULL, 0xb85045b68181585dULL, 0x30644e72e131a029ULL},
    0xc2e1f593efffffffULL,
    {0xac96341c4ffffffbULL, 0x36fc76959f60cd29ULL, 0x666ea36f7879462eULL, 0x0e0a77c19a07df2fULL},
    {0x1bb8e645ae216da7ULL, 0x53fe3ab1e35c59e3ULL, 0x8c49833d53bb8085ULL, 0x0216d0b17f4e44a5ULL},
};

/* ------------------------------------------------------------------------ */
/* multi-precision helpers                                                   */

static inline int u256_geq(const uint64_t *a, const uint64_t *b) {
    for (int i = 3; i >= 0; i--) {
        if (a[i] != b[i]) return a[i] > b[i];
    }
    return 1;
}

static inline uint64_t u256_sub(uint64_t *r, const uint64_t *a, const uint64_t *b) {
    uint64_t borrow = 0;
    for (int i = 0; i < 4; i++) {
        u128 d = (u128)a[i] - b[i] - borrow;
        r[i] = (uint64_t)d;
        borrow = (uint64_t)(d >> 64) & 1;
    }
    return borrow;
}

static inline uint64_t u256_add(uint64_t *r, const uint64_t *a, const uint64_t *b) {
    u128 c = 0;
    for (int i = 0; i < 4; i++) {
        c += (u128)a[i] + b[i];
        r[i] = (uint64_t)c;
        c >>= 64;
    }
    return (uint64_t)c;
}

static inline int fe_is_zero(const fe *a) { return (a->v[0] | a->v[1] | a->v[2] | a->v[3]) == 0; }
static inline int fe_eq(const fe *a, const fe *b) {
    return a->v[0] == b->v[0] && a->v[1] == b->v[1] && a->v[2] == b->v[2] && a->v[3] == b->v[3];
}

/* Montgomery product a*b*R^{-1} mod m, coarsely integrated operand scanning
 * over 64-bit words; inputs and output are fully reduced. */
static void fe_mul(fe *r, const fe *a, const fe *b, const fparams *P) {
    uint64_t t[6] = {0, 0, 0, 0, 0, 0};
    for (int i = 0; i < 4; i++) {
        u128 c = 0;
        for (int j = 0; j < 4; j++) {
            c += (u128)a->v[j] * b->v[i] + t[j];
            t[j] = (uint64_t)c;
            c >>= 64;
        }
        c += t[4];
        t[4] = (uint64_t)c;
        t[5] = (uint64_t)(c >> 64);
        uint64_t m = t[0] * P->inv;
        c = (u128)m * P->m[0] + t[0];
        c >>= 64;
        for (int j = 1; j < 4; j++) {
            c += (u128)m * P->m[j] + t[j];
            t[j - 1] = (uint64_t)c;
            c >>= 64;
        }
        c += t[4];
        t[3] = (uint64_t)c;
        t[4] = t[5] + (uint64_t)(c >> 64);
    }
    uint64_t s[4];
    if (t[4] != 0 || u256_geq(t, P->m)) {
        u256_sub(s, t, P->m);
        memcpy(r->v, s, sizeof s);
    } else {
        memcpy(r->v, t, 4 * sizeof(uint64_t));
    }
}

static inline void fe_sqr(fe *r, const fe *a, const fparams *P) { fe_mul(r, a, a, P); }

static void fe_add(fe *r, const fe *a, const fe *b, const fparams *P) {
    uint64_t s[4];
    uint64_t carry = u256_add(s, a->v, b->v);
    if (carry || u256_geq(s, P->m)) u256_sub(s, s, P->m);
    memcpy(r->v, s, sizeof s);
}

static void fe_sub(fe *r, const fe *a, const fe *b, const fparams *P) {
    uint64_t s[4];
    uint64_t borrow = u256_sub(s, a->v, b->v);
    if (borrow) u256_add(s, s, P->m);
    memcpy(r->v, s, sizeof s);
}

static void fe_neg(fe *r, const fe *a, const fparams *P) {
    if (fe_is_zero(a)) {
        memset(r, 0, sizeof *r);
        return;
    }
    u256_sub(r->v, P->m, a->v);
}

static void fe_dbl(fe *r, const fe *a, const fparams *P) { fe_add(r, a, a, P); }

/* a^e for a plain (non-Montgomery) 256-bit exponent e, square-and-multiply. */
static void fe_pow(fe *r, const fe *a, const uint64_t *e, const fparams *P) {
    fe acc;
    memcpy(acc.v, P->r1, sizeof acc.v);
    fe base = *a;
    for (int i = 255; i >= 0; i--) {
        fe_sqr(&acc, &acc, P);
        if ((e[i / 64] >> (i % 64)) & 1) fe_mul(&acc, &acc, &base, P);
    }
    *r = acc;
}

/* Fermat inversion a^(m-2); inverse of zero is zero. */
static void fe_inv(fe *r, const fe *a, const fparams *P) {
    uint64_t e[4];
    uint64_t two[4] = {2, 0, 0, 0};
    u256_sub(e, P->m, two);
    fe_pow(r, a, e, P);
}

static void fe_to_mont(fe *r, const fe *a, const fparams *P) {
    fe r2;
    memcpy(r2.v, P->r2, sizeof r2.v);
    fe_mul(r, a, &r2, P);
}

static void fe_from_mont(fe *r, const fe *a, const fparams *P) {
    fe one = {{1, 0, 0, 0}};
    fe_mul(r, a, &one, P);
}

static inline void fe_load(fe *r, const uint32_t *p) {
    for (int i = 0; i < 4; i++) r->v[i] = (uint64_t)p[2 * i] | ((uint64_t)p[2 * i + 1] << 32);
}

static inline void fe_store(uint32_t *p, const fe *a) {
    for (int i = 0; i < 4; i++) {
        p[2 * i] = (uint32_t)a->v[i];
        p[2 * i + 1] = (uint32_t)(a->v[i] >> 32);
    }
}

static inline void fe_one(fe *r, const fparams *P) { memcpy(r->v, P->r1, sizeof r->v); }

/* ------------------------------------------------------------------------ */
/* G1 in Jacobian coordinates, y^2 = x^3 + 3; x = X/Z^2, y = Y/Z^3.          */

typedef struct { fe x, y; } aff;       /* Montgomery; (0,0) is the identity */
typedef struct { fe X, Y, Z; } jac;    /* Z == 0 is the identity */

static inline int aff_is_identity(const aff *a) { return fe_is_zero(&a->y); }

static inline void jac_set_identity(jac *r) { memset(r, 0, sizeof *r); }
static inline int jac_is_identity(const jac *a) { return fe_is_zero(&a->Z); }

static void jac_from_aff(jac *r, const aff *a) {
    if (aff_is_identity(a)) {
        jac_set_identity(r);
        return;
    }
    r->X = a->x;
    r->Y = a->y;
    fe_one(&r->Z, &FQ);
}

/* dbl-2009-l */
static void jac_dbl(jac *r, const jac *p) {
    if (jac_is_identity(p)) {
        *r = *p;
        return;
    }
    const fparams *F = &FQ;
    fe A, B, C, D, E, Fv, t, X3, Y3, Z3;
    fe_sqr(&A, &p->X, F);
    fe_sqr(&B, &p->Y, F);
    fe_sqr(&C, &B, F);
    fe_add(&t, &p->X, &B, F);
    fe_sqr(&t, &t, F);
    fe_sub(&t, &t, &A, F);
    fe_sub(&t, &t, &C, F);
    fe_dbl(&D, &t, F);
    fe_dbl(&E, &A, F);
    fe_add(&E, &E, &A, F);
    fe_sqr(&Fv, &E, F);
    fe_dbl(&t, &D, F);
    fe_sub(&X3, &Fv, &t, F);
    fe_sub(&t, &D, &X3, F);
    fe_mul(&Y3, &E, &t, F);
    fe_dbl(&t, &C, F);
    fe_dbl(&t, &t, F);
    fe_dbl(&t, &t, F);
    fe_sub(&Y3, &Y3, &t, F);
    fe_mul(&Z3, &p->Y, &p->Z, F);
    fe_dbl(&Z3, &Z3, F);
    r->X = X3;
    r->Y = Y3;
    r->Z = Z3;
}

/* add-2007-bl, with the identity / doubling / inverse cases handled. */
static void jac_add(jac *r, const jac *p, const jac *q) {
    if (jac_is_identity(p)) {
        *r = *q;
        return;
    }
    if (jac_is_identity(q)) {
        *r = *p;
        return;
    }
    const fparams *F = &FQ;
    fe Z1Z1, Z2Z2, U1, U2, S1, S2, H, I, J, rr, V, t, X3, Y3, Z3;
    fe_sqr(&Z1Z1, &p->Z, F);
    fe_sqr(&Z2Z2, &q->Z, F);
    fe_mul(&U1, &p->X, &Z2Z2, F);
    fe_mul(&U2, &q->X, &Z1Z1, F);
    fe_mul(&S1, &p->Y, &q->Z, F);
    fe_mul(&S1, &S1, &Z2Z2, F);
    fe_mul(&S2, &q->Y, &p->Z, F);
    fe_mul(&S2, &S2, &Z1Z1, F);
    fe_sub(&H, &U2, &U1, F);
    fe_sub(&t, &S2, &S1, F);
    if (fe_is_zero(&H)) {
        if (fe_is_zero(&t)) {
            jac_dbl(r, p);
        } else {
            jac_set_identity(r);
        }
        return;
    }
    fe_dbl(&rr, &t, F);
    fe_dbl(&I, &H, F);
    fe_sqr(&I, &I, F);
    fe_mul(&J, &H, &I, F);
    fe_mul(&V, &U1, &I, F);
    fe_sqr(&X3, &rr, F);
    fe_sub(&X3, &X3, &J, F);
    fe_dbl(&t, &V, F);
    fe_sub(&X3, &X3, &t, F);
    fe_sub(&t, &V, &X3, F);
    fe_mul(&Y3, &rr, &t, F);
    fe_mul(&t, &S1, &J, F);
    fe_dbl(&t, &t, F);
    fe_sub(&Y3, &Y3, &t, F);
    fe_add(&Z3, &p->Z, &q->Z, F);
    fe_sqr(&Z3, &Z3, F);
    fe_sub(&Z3, &Z3, &Z1Z1, F);
    fe_sub(&Z3, &Z3, &Z2Z2, F);
    fe_mul(&Z3, &Z3, &H, F);
    r->X = X3;
    r->Y = Y3;
    r->Z = Z3;
}

/* madd-2007-bl: Jacobian + affine. */
static void jac_add_aff(jac *r, const jac *p, const aff *q) {
    if (aff_is_identity(q)) {
        *r = *p;
        return;
    }
    if (jac_is_identity(p)) {
        jac_from_aff(r, q);
        return;
    }
    const fparams *F = &FQ;
    fe Z1Z1, U2, S2, H, HH, I, J, rr, V, t, X3, Y3, Z3;
    fe_sqr(&Z1Z1, &p->Z, F);
    fe_mul(&U2, &q->x, &Z1Z1, F);
    fe_mul(&S2, &q->y, &p->Z, F);
    fe_mul(&S2, &S2, &Z1Z1, F);
    fe_sub(&H, &U2, &p->X, F);
    fe_sub(&t, &S2, &p->Y, F);
    if (fe_is_zero(&H)) {
        if (fe_is_zero(&t)) {
            jac_dbl(r, p);
        } else {
            jac_set_identity(r);
        }
        return;
    }
    fe_dbl(&rr, &t, F);
    fe_sqr(&HH, &H, F);
    fe_dbl(&I, &HH, F);
    fe_dbl(&I, &I, F);
    fe_mul(&J, &H, &I, F);
    fe_mul(&V, &p->X, &I, F);
    fe_sqr(&X3, &rr, F);
    fe_sub(&X3, &X3, &J, F);
    fe_dbl(&t, &V, F);
    fe_sub(&X3, &X3, &t, F);
    fe_sub(&t, &V, &X3, F);
    fe_mul(&Y3, &rr, &t, F);
    fe_mul(&t, &p->Y, &J, F);
    fe_dbl(&t, &t, F);
    fe_sub(&Y3, &Y3, &t, F);
    fe_add(&Z3, &p->Z, &H, F);
    fe_sqr(&Z3, &Z3, F);
    fe_sub(&Z3, &Z3, &Z1Z1, F);
    fe_sub(&Z3, &Z3, &HH, F);
    r->X = X3;
    r->Y = Y3;
    r->Z = Z3;
}

static void jac_to_aff(aff *r, const jac *p) {
    if (jac_is_identity(p)) {
        memset(r, 0, sizeof *r);
        return;
    }
    fe zi, zi2, zi3;
    fe_inv(&zi, &p->Z, &FQ);
    fe_sqr(&zi2, &zi, &FQ);
    fe_mul(&zi3, &zi2, &zi, &FQ);
    fe_mul(&r->x, &p->X, &zi2, &FQ);
    fe_mul(&r->y, &p->Y, &zi3, &FQ);
}

/* Montgomery's simultaneous inversion over the Z coordinates of n points. */
static void jac_batch_to_aff(aff *out, const jac *in, size_t n) {
    fe *prefix = (fe *)malloc(sizeof(fe) * (n + 1));
    fe acc;
    fe_one(&acc, &FQ);
    for (size_t i = 0; i < n; i++) {
        prefix[i] = acc;
        if (!jac_is_identity(&in[i])) fe_mul(&acc, &acc, &in[i].Z, &FQ);
    }
    fe inv;
    fe_inv(&inv, &acc, &FQ);
    for (size_t k = n; k-- > 0;) {
        if (jac_is_identity(&in[k])) {
            memset(&out[k], 0, sizeof(aff));
            continue;
        }
        fe zi, zi2, zi3;
        fe_mul(&zi, &inv, &prefix[k], &FQ);
        fe_mul(&inv, &inv, &in[k].Z, &FQ);
        fe_sqr(&zi2, &zi, &FQ);
        fe_mul(&zi3, &zi2, &zi, &FQ);
        fe_mul(&out[k].x, &in[k].X, &zi2, &FQ);
        fe_mul(&out[k].y, &in[k].Y, &zi3, &FQ);
    }
    free(prefix);
}

/* k*P for a plain 256-bit scalar k, left-to-right double-and-add. */
static void jac_smul(jac *r, const aff *p, const uint64_t *k) {
    jac acc;
    jac_set_identity(&acc);
    for (int i = 255; i >= 0; i--) {
        jac_dbl(&acc, &acc);
        if ((k[i / 64] >> (i % 64)) & 1) jac_add_aff(&acc, &acc, p);
    }
    *r = acc;
}

static inline void aff_load(aff *a, const uint32_t *p) {
    fe_load(&a->x, p);
    fe_load(&a->y, p + 8);
}

static inline void aff_store(uint32_t *p, const aff *a) {
    fe_store(p, &a->x);
    fe_store(p + 8, &a->y);
}

static void aff_generator(aff *g) {
    fe one = {{1, 0, 0, 0}}, two = {{2, 0, 0, 0}};
    fe_to_mont(&g->x, &one, &FQ);
    fe_to_mont(&g->y, &two, &FQ);
}

static int aff_on_curve(const aff *a) {
    if (aff_is_identity(a)) return 1;
    fe three = {{3, 0, 0, 0}}, b, lhs, rhs;
    fe_to_mont(&b, &three, &FQ);
    fe_sqr(&lhs, &a->y, &FQ);
    fe_sqr(&rhs, &a->x, &FQ);
    fe_mul(&rhs, &rhs, &a->x, &FQ);
    fe_add(&rhs, &rhs, &b, &FQ);
    return fe_eq(&lhs, &rhs);
}

/* ------------------------------------------------------------------------ */
/* Exported element-wise operations (used by the parity tests).             */

enum { ORC_FQ = 0, ORC_FR = 1 };
enum {
    ORC_ADD = 0, ORC_SUB = 1, ORC_MUL = 2, ORC_SQR = 3, ORC_NEG = 4,
    ORC_TO_MONT = 5, ORC_FROM_MONT = 6, ORC_INV = 7, ORC_POW = 8
};

int orc_field_op(int field, int op, const uint32_t *a, const uint32_t *b, uint32_t *out, uint64_t count) {
    const fparams *P = field == ORC_FQ ? &FQ : field == ORC_FR ? &FR : NULL;
    if (!P) return -1;
    for (uint64_t i = 0; i < count; i++) {
        fe x, y, r;
        fe_load(&x, a + 8 * i);
        if (b) fe_load(&y, b + 8 * i);
        switch (op) {
        case ORC_ADD: fe_add(&r, &x, &y, P); break;
        case ORC_SUB: fe_sub(&r, &x, &y, P); break;
        case ORC_MUL: fe_mul(&r, &x, &y, P); break;
        case ORC_SQR: fe_sqr(&r, &x, P); break;
        case ORC_NEG: fe_neg(&r, &x, P); break;
        case ORC_TO_MONT: fe_to_mont(&r, &x, P); break;
        case ORC_FROM_MONT: fe_from_mont(&r, &x, P); break;
        case ORC_INV: fe_inv(&r, &x, P); break;
        case ORC_POW: fe_pow(&r, &x, y.v, P); break;
        default: return -2;
        }
        fe_store(out + 8 * i, &r);
    }
    return 0;
}

enum { ORC_PT_ADD = 0, ORC_PT_DBL = 1, ORC_PT_NEG = 2, ORC_PT_SMUL = 3, ORC_PT_ONCURVE = 4 };

/* Affine-in / affine-out point operations.  For ORC_PT_SMUL the second
 * operand is a plain (canonical) 256-bit scalar of 8 u32; for ORC_PT_ONCURVE
 * out[16*i] receives 1 or 0. */
int orc_point_op(int op, const uint32_t *p, const uint32_t *q, uint32_t *out, uint64_t count) {
    for (uint64_t i = 0; i < count; i++) {
        aff a, b, r;
        jac j, k;
        aff_load(&a, p + 16 * i);
        switch (op) {
        case ORC_PT_ADD:
            aff_load(&b, q + 16 * i);
            jac_from_aff(&j, &a);
            jac_add_aff(&j, &j, &b);
            jac_to_aff(&r, &j);
            break;
        case ORC_PT_DBL:
            jac_from_aff(&j, &a);
            jac_dbl(&j, &j);
            jac_to_aff(&r, &j);
            break;
        case ORC_PT_NEG:
            r.x = a.x;
            fe_neg(&r.y, &a.y, &FQ);
            if (aff_is_identity(&a)) memset(&r, 0, sizeof r);
            break;
        case ORC_PT_SMUL: {
            fe s;
            fe_load(&s, q + 8 * i);
            jac_smul(&k, &a, s.v);
            jac_to_aff(&r, &k);
            break;
        }
        case ORC_PT_ONCURVE:
            memset(&r, 0, sizeof r);
            r.x.v[0] = (uint64_t)aff_on_curve(&a);
            break;
        default:
            return -2;
        }
        aff_store(out + 16 * i, &r);
    }
    return 0;
}

/* ------------------------------------------------------------------------ */
/* Seeded synthetic inputs.                                                  */
/*
 * A stream (seed, stream id) is the splitmix64 sequence started at
 * key = mix(seed * GAMMA + mix(stream + C)); word idx is mix(key + (idx+1)*GAMMA).
 * Uniform Fr element i uses words 8i..8i+7: lo = words 0..3, hi = words 4..7,
 * value = (lo + hi * 2^256) mod r.  The skewed mix (distribution 1) draws a
 * category word from stream id + 2^32: u % 10 in {0,1} -> 0, {2,3} -> 1,
 * {4,5,6} -> (u >> 40) & 0xffff, {7,8,9} -> uniform Fr.
 */

#define GAMMA 0x9e3779b97f4a7c15ULL

static inline uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ULL;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebULL;
    return z ^ (z >> 31);
}

static inline uint64_t stream_key(uint64_t seed, uint64_t stream) {
    return mix64(seed * GAMMA + mix64(stream + 0x632be59bd9b4e019ULL));
}

static inline uint64_t stream_word(uint64_t key, uint64_t idx) { return mix64(key + (idx + 1) * GAMMA); }

static void reduce_once_r(uint64_t *x) {
    while (u256_geq(x, FR.m)) u256_sub(x, x, FR.m);
}

/* canonical (non-Montgomery) uniform Fr element number idx of a stream */
static void uniform_fr(fe *out, uint64_t key, uint64_t idx) {
    uint64_t lo[4], hi[4];
    for (int k = 0; k < 4; k++) lo[k] = stream_word(key, 8 * idx + k);
    for (int k = 0; k < 4; k++) hi[k] = stream_word(key, 8 * idx + 4 + k);
    reduce_once_r(lo);
    reduce_once_r(hi);
    fe h, r2, t, l;
    memcpy(h.v, hi, sizeof hi);
    memcpy(r2.v, FR.r2, sizeof r2.v);
    fe_mul(&t, &h, &r2, &FR); /* hi * 2^256 mod r */
    memcpy(l.v, lo, sizeof lo);
    fe_add(out, &l, &t, &FR);
}

static void gen_scalar_canonical(fe *out, uint64_t seed, uint64_t stream, int dist, uint64_t idx) {
    uint64_t key = stream_key(seed, stream);
    if (dist == 1) {
        uint64_t u = stream_word(stream_key(seed, stream + (1ULL << 32)), idx);
        uint64_t cat = u % 10;
        memset(out, 0, sizeof *out);
        if (cat < 2) return;
        if (cat < 4) {
            out->v[0] = 1;
            return;
        }
        if (cat < 7) {
            out->v[0] = (u >> 40) & 0xffff;
            return;
        }
    }
    uniform_fr(out, key, idx);
}

typedef struct {
    uint64_t seed, stream, start, n;
    int dist, mont;
    uint32_t *out;
} scal_job;

static void *scal_worker(void *arg) {
    scal_job *j = (scal_job *)arg;
    for (uint64_t i = 0; i < j->n; i++) {
        fe v, m;
        gen_scalar_canonical(&v, j->seed, j->stream, j->dist, j->start + i);
        if (j->mont) {
            fe_to_mont(&m, &v, &FR);
            fe_store(j->out + 8 * i, &m);
        } else {
            fe_store(j->out + 8 * i, &v);
        }
    }
    return NULL;
}

/* n scalars of a stream starting at element `start`; Montgomery form if mont. */
int orc_gen_scalars(uint64_t seed, uint64_t stream, int dist, uint64_t start, uint64_t n, int mont, uint32_t *out,
                    int threads) {
    if (threads < 1) threads = 1;
    if ((uint64_t)threads > n / 4096 + 1) threads = (int)(n / 4096 + 1);
    pthread_t tid[256];
    scal_job jobs[256];
    if (threads > 256) threads = 256;
    uint64_t per = (n + threads - 1) / threads;
    int launched = 0;
    for (int t = 0; t < threads; t++) {
        uint64_t s = per * t;
        if (s >= n) break;
        uint64_t e = s + per < n ? s + per : n;
        jobs[t] = (scal_job){seed, stream, start + s, e - s, dist, mont, out + 8 * s};
        pthread_create(&tid[t], NULL, scal_worker, &jobs[t]);
        launched++;
    }
    for (int t = 0; t < launched; t++) pthread_join(tid[t], NULL);
    return 0;
}

/* P_i = r_i * G with r_i the uniform Fr stream (seed, stream 0).  Computed
 * with a fixed-base comb: T[j][v] = v * 2^(8j) * G, 32 byte-indexed mixed
 * additions per point, then one simultaneous inversion per block. */
static aff *g_comb = NULL; /* [32][256] */
static pthread_mutex_t g_comb_lock = PTHREAD_MUTEX_INITIALIZER;

static void build_comb(void) {
    pthread_mutex_lock(&g_comb_lock);
    if (!g_comb) {
        aff *t = (aff *)calloc(32 * 256, sizeof(aff));
        jac *tmp = (jac *)calloc(256, sizeof(jac));
        aff g;
        aff_generator(&g);
        jac base;
        jac_from_aff(&base, &g);
        for (int j = 0; j < 32; j++) {
            jac_set_identity(&tmp[0]);
            tmp[1] = base;
            for (int v = 2; v < 256; v++) jac_add(&tmp[v], &tmp[v - 1], &base);
            jac_batch_to_aff(t + 256 * j, tmp, 256);
            for (int k = 0; k < 8; k++) jac_dbl(&base, &base);
        }
        free(tmp);
        g_comb = t;
    }
    pthread_mutex_unlock(&g_comb_lock);
}

typedef struct {
    uint64_t seed, start, n;
    uint32_t *out;
} pt_job;

static void *pt_worker(void *arg) {
    pt_job *j = (pt_job *)arg;
    const uint64_t BLK = 1024;
    jac *tmp = (jac *)malloc(sizeof(jac) * BLK);
    aff *res = (aff *)malloc(sizeof(aff) * BLK);
    uint64_t key = stream_key(j->seed, 0);
    for (uint64_t b = 0; b < j->n; b += BLK) {
        uint64_t m = j->n - b < BLK ? j->n - b : BLK;
        for (uint64_t i = 0; i < m; i++) {
            fe r;
            uniform_fr(&r, key, j->start + b + i);
            jac acc;
            jac_set_identity(&acc);
            for (int byte = 0; byte < 32; byte++) {
                unsigned v = (unsigned)((r.v[byte / 8] >> (8 * (byte % 8))) & 0xff);
                if (v) jac_add_aff(&acc, &acc, &g_comb[256 * byte + v]);
            }
            tmp[i] = acc;
        }
        jac_batch_to_aff(res, tmp, m);
        for (uint64_t i = 0; i < m; i++) aff_store(j->out + 16 * (b + i), &res[i]);
    }
    free(tmp);
    free(res);
    return NULL;
}

int orc_gen_points(uint64_t seed, uint64_t start, uint64_t n, uint32_t *out, int threads) {
    build_comb();
    if (threads < 1) threads = 1;
    if (threads > 256) threads = 256;
    if ((uint64_t)threads > n / 1024 + 1) threads = (int)(n / 1024 + 1);
    pthread_t tid[256];
    pt_job jobs[256];
    uint64_t per = (n + threads - 1) / threads;
    int launched = 0;
    for (int t = 0; t < threads; t++) {
        uint64_t s = per * t;
        if (s >= n) break;
        uint64_t e = s + per < n ? s + per : n;
        jobs[t] = (pt_job){seed, start + s, e - s, out + 16 * s};
        pthread_create(&tid[t], NULL, pt_worker, &jobs[t]);
        launched++;
    }
    for (int t = 0; t < launched; t++) pthread_join(tid[t], NULL);
    return 0;
}

/* ------------------------------------------------------------------------ */
/* The reference's CPU MSM (core/tests/msm_halo2.rs), restated.             */

/* get_at (msm_halo2.rs:74-92): c-bit unsigned digit of a little-endian
 * 32-byte canonical scalar at segment `segment`. */
static uint64_t get_at(int segment, int c, const uint8_t *bytes) {
    int skip_bits = segment * c;
    int skip_bytes = skip_bits / 8;
    if (skip_bytes >= 32) return 0;
    uint8_t v[8] = {0};
    for (int k = 0; k < 8 && skip_bytes + k < 32; k++) v[k] = bytes[skip_bytes + k];
    uint64_t tmp = 0;
    for (int k = 7; k >= 0; k--) tmp = (tmp << 8) | v[k];
    tmp >>= (skip_bits - skip_bytes * 8);
    tmp %= (1ULL << c);
    return tmp;
}

enum { B_NONE = 0, B_AFFINE = 1, B_PROJ = 2 };
typedef struct {
    int state;
    aff a;
    jac p;
} bucket;

/* multiexp_serial (msm_halo2.rs:63-151): acc += sum_i coeff_i * base_i */
static void multiexp_serial(const uint8_t *coeff_bytes, const aff *bases, size_t n, jac *acc) {
    int c;
    if (n < 4) c = 1;
    else if (n < 32) c = 3;
    else c = (int)ceil(log((double)(uint32_t)n));
    int segments = 254 / c + 1;
    size_t nb = ((size_t)1 << c) - 1;
    bucket *buckets = (bucket *)malloc(sizeof(bucket) * nb);
    for (int seg = segments - 1; seg >= 0; seg--) {
        for (int k = 0; k < c; k++) jac_dbl(acc, acc);
        for (size_t b = 0; b < nb; b++) buckets[b].state = B_NONE;
        for (size_t i = 0; i < n; i++) {
            uint64_t coeff = get_at(seg, c, coeff_bytes + 32 * i);
            if (!coeff) continue;
            bucket *bk = &buckets[coeff - 1];
            switch (bk->state) {
            case B_NONE:
                bk->state = B_AFFINE;
                bk->a = bases[i];
                break;
            case B_AFFINE:
                jac_from_aff(&bk->p, &bk->a);
                jac_add_aff(&bk->p, &bk->p, &bases[i]);
                bk->state = B_PROJ;
                break;
            default:
                jac_add_aff(&bk->p, &bk->p, &bases[i]);
                break;
            }
        }
        /* summation by parts: running sum from the top bucket down */
        jac running;
        jac_set_identity(&running);
        for (size_t b = nb; b-- > 0;) {
            if (buckets[b].state == B_AFFINE) jac_add_aff(&running, &running, &buckets[b].a);
            else if (buckets[b].state == B_PROJ) jac_add(&running, &running, &buckets[b].p);
            jac_add(acc, acc, &running);
        }
    }
    free(buckets);
}

typedef struct {
    const uint8_t *coeffs;
    const aff *bases;
    size_t n;
    jac acc;
} chunk_job;

static void *chunk_worker(void *arg) {
    chunk_job *j = (chunk_job *)arg;
    jac_set_identity(&j->acc);
    multiexp_serial(j->coeffs, j->bases, j->n, &j->acc);
    return NULL;
}

/* best_multiexp (msm_halo2.rs:182-208).  points: n affine (16 u32 each,
 * Montgomery); scalars: n Fr elements in Montgomery form (the C ABI's form);
 * out: 16 u32, canonical affine Montgomery, identity (0,0). */
int orc_msm_halo2(const uint32_t *points, const uint32_t *scalars, uint64_t n, uint32_t *out, int num_threads) {
    if (num_threads < 1) num_threads = 1;
    aff *bases = (aff *)malloc(sizeof(aff) * (n ? n : 1));
    uint8_t *coeffs = (uint8_t *)malloc(32 * (n ? n : 1));
    for (uint64_t i = 0; i < n; i++) {
        aff_load(&bases[i], points + 16 * i);
        fe s, c;
        fe_load(&s, scalars + 8 * i);
        fe_from_mont(&c, &s, &FR); /* to_repr(): canonical little-endian bytes */
        for (int k = 0; k < 32; k++) coeffs[32 * i + k] = (uint8_t)(c.v[k / 8] >> (8 * (k % 8)));
    }
    jac total;
    jac_set_identity(&total);
    if (n > (uint64_t)num_threads) {
        size_t chunk = n / num_threads;
        size_t num_chunks = (n + chunk - 1) / chunk;
        chunk_job *jobs = (chunk_job *)calloc(num_chunks, sizeof(chunk_job));
        pthread_t *tid = (pthread_t *)calloc(num_chunks, sizeof(pthread_t));
        for (size_t k = 0; k < num_chunks; k++) {
            size_t s = k * chunk;
            size_t len = s + chunk <= n ? chunk : n - s;
            jobs[k].coeffs = coeffs + 32 * s;
            jobs[k].bases = bases + s;
            jobs[k].n = len;
            pthread_create(&tid[k], NULL, chunk_worker, &jobs[k]);
        }
        for (size_t k = 0; k < num_chunks; k++) {
            pthread_join(tid[k], NULL);
            jac_add(&total, &total, &jobs[k].acc);
        }
        free(jobs);
        free(tid);
    } else {
        multiexp_serial(coeffs, bases, n, &total);
    }
    aff r;
    jac_to_aff(&r, &total);
    aff_store(out, &r);
    free(bases);
    free(coeffs);
    return 0;
}

/* Direct sum of k_i * P_i by double-and-add per term, for small n. */
int orc_msm_naive(const uint32_t *points, const uint32_t *scalars, uint64_t n, uint32_t *out) {
    jac total;
    jac_set_identity(&total);
    for (uint64_t i = 0; i < n; i++) {
        aff p;
        aff_load(&p, points + 16 * i);
        fe s, c;
        fe_load(&s, scalars + 8 * i);
        fe_from_mont(&c, &s, &FR);
        jac t;
        jac_smul(&t, &p, c.v);
        jac_add(&total, &total, &t);
    }
    aff r;
    jac_to_aff(&r, &total);
    aff_store(out, &r);
    return 0;
}

/* Window tables of core/src/msm/src/msm_impl.cuh:358-371: for j in
 * 1..n_tables-1, out[j] = 2^(j*shift) * P_i (affine, Montgomery); out[0] is a
 * copy of the input.  out holds n_tables * n points, table-major. */
int orc_precompute(const uint32_t *points, uint64_t n, uint32_t shift, uint32_t n_tables, uint32_t *out) {
    const uint64_t BLK = 1024;
    jac *tmp = (jac *)malloc(sizeof(jac) * BLK);
    aff *res = (aff *)malloc(sizeof(aff) * BLK);
    memcpy(out, points, sizeof(uint32_t) * 16 * n);
    for (uint64_t b = 0; b < n; b += BLK) {
        uint64_t m = n - b < BLK ? n - b : BLK;
        for (uint64_t i = 0; i < m; i++) {
            aff p;
            aff_load(&p, points + 16 * (b + i));
            jac_from_aff(&tmp[i], &p);
        }
        for (uint32_t j = 1; j < n_tables; j++) {
            for (uint64_t i = 0; i < m; i++)
                for (uint32_t k = 0; k < shift; k++) jac_dbl(&tmp[i], &tmp[i]);
            jac_batch_to_aff(res, tmp, m);
            for (uint64_t i = 0; i < m; i++) aff_store(out + 16 * ((uint64_t)j * n + b + i), &res[i]);
        }
    }
    free(tmp);
    free(res);
    return 0;
}
