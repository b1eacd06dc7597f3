// BN254 field and G1 arithmetic for sm_100a.
//
// Field elements are 8 little-endian 32-bit limbs in Montgomery form with
// R = 2^256, the layout of the reference's mont::Element
// (core/src/common/mont/src/field.cuh:906-1204) and of its C ABI.
// Multiplication is coarsely integrated operand scanning: per row of b, the
// products a_j*b[i] are added into the running value by lo/hi multiply-add
// pairs with carry (even j in one chain, odd j in a second), then the
// reduction factor m and the same for m*N.  Measured on B200, the
// accumulation loop runs 10% faster this way than with 64-bit mul.wide
// products added by separate ALU carry chains.  Because N < 2^254 the
// running value stays below 3N < 2^256 even for inputs in [0, 2N), so nine
// words hold every intermediate and no carry ever leaves word 8.
//
// Reduction is lazy: between operations a field value is any representative
// in [0, 2N).  For inputs below 2N the Montgomery product is below
// (4N^2 + R N) / R < 2N (as 4N < R), so it skips the final conditional
// subtraction; addition and subtraction work modulo 2N.  A value is zero mod N
// when it is 0 or N (fe_is_zero).  fe_canon gives the representative in
// [0, N); every value that leaves the arithmetic (affine results, generated
// scalars, test outputs) is canonical.
//
// Curve points use XYZZ coordinates (x = X/ZZ, y = Y/ZZZ, ZZ^3 = ZZZ^2), the
// point representation of core/src/common/curve/src/curve_xyzz.cuh:252-418,
// with the Explicit-Formulas Database's madd-2008-s, add-2008-s,
// dbl-2008-s-1 and mdbl-2008-s-1 for a = 0 (y^2 = x^3 + 3,
// core/src/common/curve/src/bn254.cuh:13-31).  ZZ == 0 marks the identity;
// an affine point with y == 0 is the identity (curve_xyzz.cuh:204-210).
#pragma once

#include <cstdint>

namespace bn254 {

typedef uint32_t u32;
typedef uint64_t u64;

struct FqP {
    static constexpr u32 M0 = 0xd87cfd47u, M1 = 0x3c208c16u, M2 = 0x6871ca8du, M3 = 0x97816a91u;
    static constexpr u32 M4 = 0x8181585du, M5 = 0xb85045b6u, M6 = 0xe131a029u, M7 = 0x30644e72u;
    static constexpr u32 INV = 0xe4866389u;  // -p^{-1} mod 2^32
    // R mod p (Montgomery one)
    static constexpr u32 R0 = 0xc58f0d9du, R1 = 0xd35d438du, R2 = 0xf5c70b3du, R3 = 0x0a78eb28u;
    static constexpr u32 R4 = 0x7879462cu, R5 = 0x666ea36fu, R6 = 0x9a07df2fu, R7 = 0x0e0a77c1u;
    // 2p
    static constexpr u32 D0 = 0xb0f9fa8eu, D1 = 0x7841182du, D2 = 0xd0e3951au, D3 = 0x2f02d522u;
    static constexpr u32 D4 = 0x0302b0bbu, D5 = 0x70a08b6du, D6 = 0xc2634053u, D7 = 0x60c89ce5u;
};

struct FrP {
    static constexpr u32 M0 = 0xf0000001u, M1 = 0x43e1f593u, M2 = 0x79b97091u, M3 = 0x2833e848u;
    static constexpr u32 M4 = 0x8181585du, M5 = 0xb85045b6u, M6 = 0xe131a029u, M7 = 0x30644e72u;
    static constexpr u32 INV = 0xefffffffu;  // -r^{-1} mod 2^32
    static constexpr u32 R0 = 0x4ffffffbu, R1 = 0xac96341cu, R2 = 0x9f60cd29u, R3 = 0x36fc7695u;
    static constexpr u32 R4 = 0x7879462eu, R5 = 0x666ea36fu, R6 = 0x9a07df2fu, R7 = 0x0e0a77c1u;
    // 2r
    static constexpr u32 D0 = 0xe0000002u, D1 = 0x87c3eb27u, D2 = 0xf372e122u, D3 = 0x5067d090u;
    static constexpr u32 D4 = 0x0302b0bau, D5 = 0x70a08b6du, D6 = 0xc2634053u, D7 = 0x60c89ce5u;
};

template <class F>
struct Fe {
    u32 l[8];
};

typedef Fe<FqP> Fq;
typedef Fe<FrP> Fr;

template <class F>
__host__ __device__ __forceinline__ Fe<F> fe_zero() {
    Fe<F> r;
#pragma unroll
    for (int i = 0; i < 8; i++) r.l[i] = 0;
    return r;
}

template <class F>
__host__ __device__ __forceinline__ Fe<F> fe_one() {
    Fe<F> r;
    r.l[0] = F::R0; r.l[1] = F::R1; r.l[2] = F::R2; r.l[3] = F::R3;
    r.l[4] = F::R4; r.l[5] = F::R5; r.l[6] = F::R6; r.l[7] = F::R7;
    return r;
}

// Zero test for a canonical value (in [0, N)).
template <class F>
__device__ __forceinline__ bool fe_is_zero_canonical(const Fe<F> &a) {
    u32 x = (a.l[0] | a.l[1]) | (a.l[2] | a.l[3]) | (a.l[4] | a.l[5]) | (a.l[6] | a.l[7]);
    return x == 0;
}

// Zero test for a value in [0, 2N): 0 or N.
template <class F>
__device__ __forceinline__ bool fe_is_zero(const Fe<F> &a) {
    u32 x = (a.l[0] | a.l[1]) | (a.l[2] | a.l[3]) | (a.l[4] | a.l[5]) | (a.l[6] | a.l[7]);
    u32 y = ((a.l[0] ^ F::M0) | (a.l[1] ^ F::M1)) | ((a.l[2] ^ F::M2) | (a.l[3] ^ F::M3)) |
            ((a.l[4] ^ F::M4) | (a.l[5] ^ F::M5)) | ((a.l[6] ^ F::M6) | (a.l[7] ^ F::M7));
    return x == 0 || y == 0;
}

// r = (t < N) ? t : t - N, for t < 2N.
template <class F>
__device__ __forceinline__ void fe_reduce_once(Fe<F> &r, const u32 t[8]) {
    u32 d[8], bw;
    asm("sub.cc.u32  %0, %9, %17;\n\t"
        "subc.cc.u32 %1, %10, %18;\n\t"
        "subc.cc.u32 %2, %11, %19;\n\t"
        "subc.cc.u32 %3, %12, %20;\n\t"
        "subc.cc.u32 %4, %13, %21;\n\t"
        "subc.cc.u32 %5, %14, %22;\n\t"
        "subc.cc.u32 %6, %15, %23;\n\t"
        "subc.cc.u32 %7, %16, %24;\n\t"
        "subc.u32    %8, 0, 0;"
        : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]),
          "=r"(bw)
        : "r"(t[0]), "r"(t[1]), "r"(t[2]), "r"(t[3]), "r"(t[4]), "r"(t[5]), "r"(t[6]), "r"(t[7]),
          "n"(F::M0), "n"(F::M1), "n"(F::M2), "n"(F::M3), "n"(F::M4), "n"(F::M5), "n"(F::M6), "n"(F::M7));
    // bw == 0xffffffff when t < N: keep t
#pragma unroll
    for (int i = 0; i < 8; i++) r.l[i] = bw ? t[i] : d[i];
}

// r = (t < 2N) ? t : t - 2N, for t < 4N.
template <class F>
__device__ __forceinline__ void fe_reduce_2n(Fe<F> &r, const u32 t[8]) {
    u32 d[8], bw;
    asm("sub.cc.u32  %0, %9, %17;\n\t"
        "subc.cc.u32 %1, %10, %18;\n\t"
        "subc.cc.u32 %2, %11, %19;\n\t"
        "subc.cc.u32 %3, %12, %20;\n\t"
        "subc.cc.u32 %4, %13, %21;\n\t"
        "subc.cc.u32 %5, %14, %22;\n\t"
        "subc.cc.u32 %6, %15, %23;\n\t"
        "subc.cc.u32 %7, %16, %24;\n\t"
        "subc.u32    %8, 0, 0;"
        : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]),
          "=r"(bw)
        : "r"(t[0]), "r"(t[1]), "r"(t[2]), "r"(t[3]), "r"(t[4]), "r"(t[5]), "r"(t[6]), "r"(t[7]),
          "n"(F::D0), "n"(F::D1), "n"(F::D2), "n"(F::D3), "n"(F::D4), "n"(F::D5), "n"(F::D6), "n"(F::D7));
#pragma unroll
    for (int i = 0; i < 8; i++) r.l[i] = bw ? t[i] : d[i];
}

// The canonical representative in [0, N) of a value in [0, 2N).
template <class F>
__device__ __forceinline__ Fe<F> fe_canon(const Fe<F> &a) {
    Fe<F> r;
    fe_reduce_once<F>(r, a.l);
    return r;
}

// Montgomery product in two accumulators.  Operand scanning over the words
// b_i keeps the running value as T = X + Y * 2^32, X holding words of weight
// 0..7 and Y words of weight 1..8.  Then a_j * b_i lands on an aligned
// register pair for every j: even j on X words (j, j+1), odd j on Y words
// (j-1, j).  Each lo/hi multiply-add pair with carry is thus one 64-bit
// multiply-add on a register pair; when the two halves of a pair straddle a
// pair boundary (one 9-word accumulator for both parities), the B200 code
// runs about 130 more instructions per product.
//
// Row i adds a * b_i and m * N (m = X_0 * (-N^{-1}) mod 2^32 makes X_0 zero)
// and divides by 2^32.  After the division X's words sit one weight lower
// (X_1 at weight 0, X_0 is zero) and Y's words at weights 0..7, so the
// arrays swap roles: the old Y becomes the new X as it is, and the old X
// becomes the new Y two words down (old X_{j+2} is new Y_j), except old X_1,
// which is added into the new X_0.  The two-word move is folded into the
// next row's odd multiply-add chain.  With inputs below 2N every partial sum
// stays below 2^288, so no carry leaves either accumulator.
//
// The row structure is the even/odd operand-scanning form of the published
// sppark mont_t multiplication (Supranational, Apache-2.0), which the
// reference's device_arith2 also uses (core/src/common/mont/src/field.cuh:526-620).

// First row: X = a_even * y, Y = a_odd * y (no accumulation).
__device__ __forceinline__ void bn_row_first(u32 (&x)[8], u32 (&y)[8], const u32 (&a)[8], u32 w) {
    asm("mul.lo.u32 %0, %16, %24;\n\tmul.hi.u32 %1, %16, %24;\n\t"
        "mul.lo.u32 %2, %18, %24;\n\tmul.hi.u32 %3, %18, %24;\n\t"
        "mul.lo.u32 %4, %20, %24;\n\tmul.hi.u32 %5, %20, %24;\n\t"
        "mul.lo.u32 %6, %22, %24;\n\tmul.hi.u32 %7, %22, %24;\n\t"
        "mul.lo.u32 %8, %17, %24;\n\tmul.hi.u32 %9, %17, %24;\n\t"
        "mul.lo.u32 %10, %19, %24;\n\tmul.hi.u32 %11, %19, %24;\n\t"
        "mul.lo.u32 %12, %21, %24;\n\tmul.hi.u32 %13, %21, %24;\n\t"
        "mul.lo.u32 %14, %23, %24;\n\tmul.hi.u32 %15, %23, %24;"
        : "=r"(x[0]), "=r"(x[1]), "=r"(x[2]), "=r"(x[3]), "=r"(x[4]), "=r"(x[5]), "=r"(x[6]), "=r"(x[7]),
          "=r"(y[0]), "=r"(y[1]), "=r"(y[2]), "=r"(y[3]), "=r"(y[4]), "=r"(y[5]), "=r"(y[6]), "=r"(y[7])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]), "r"(w));
}

// Later row, after the roles swapped: x (the old Y) += old X_1 at weight 0;
// y (the old X) = old X two words down + a_odd * w; x += a_even * w; the
// carry out of x (weight 8) into y_7.
__device__ __forceinline__ void bn_row_next(u32 (&x)[8], u32 (&y)[8], const u32 (&a)[8], u32 w) {
    asm("add.cc.u32     %0, %0, %9;\n\t"
        "madc.lo.cc.u32 %8, %17, %24, %10;\n\tmadc.hi.cc.u32 %9, %17, %24, %11;\n\t"
        "madc.lo.cc.u32 %10, %19, %24, %12;\n\tmadc.hi.cc.u32 %11, %19, %24, %13;\n\t"
        "madc.lo.cc.u32 %12, %21, %24, %14;\n\tmadc.hi.cc.u32 %13, %21, %24, %15;\n\t"
        "madc.lo.cc.u32 %14, %23, %24, 0;\n\tmadc.hi.u32    %15, %23, %24, 0;\n\t"
        "mad.lo.cc.u32  %0, %16, %24, %0;\n\tmadc.hi.cc.u32 %1, %16, %24, %1;\n\t"
        "madc.lo.cc.u32 %2, %18, %24, %2;\n\tmadc.hi.cc.u32 %3, %18, %24, %3;\n\t"
        "madc.lo.cc.u32 %4, %20, %24, %4;\n\tmadc.hi.cc.u32 %5, %20, %24, %5;\n\t"
        "madc.lo.cc.u32 %6, %22, %24, %6;\n\tmadc.hi.cc.u32 %7, %22, %24, %7;\n\t"
        "addc.u32       %15, %15, 0;"
        : "+r"(x[0]), "+r"(x[1]), "+r"(x[2]), "+r"(x[3]), "+r"(x[4]), "+r"(x[5]), "+r"(x[6]), "+r"(x[7]),
          "+r"(y[0]), "+r"(y[1]), "+r"(y[2]), "+r"(y[3]), "+r"(y[4]), "+r"(y[5]), "+r"(y[6]), "+r"(y[7])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]), "r"(w));
}

// Reduction half of a row: m = x_0 * (-N^{-1}); y += N_odd * m; x += N_even * m
// (x_0 becomes zero); the carry out of x into y_7.
template <class F>
__device__ __forceinline__ void bn_row_reduce(u32 (&x)[8], u32 (&y)[8]) {
    asm("{\n\t.reg .u32 m;\n\t"
        "mul.lo.u32     m, %0, %24;\n\t"
        "mad.lo.cc.u32  %8, m, %17, %8;\n\tmadc.hi.cc.u32 %9, m, %17, %9;\n\t"
        "madc.lo.cc.u32 %10, m, %19, %10;\n\tmadc.hi.cc.u32 %11, m, %19, %11;\n\t"
        "madc.lo.cc.u32 %12, m, %21, %12;\n\tmadc.hi.cc.u32 %13, m, %21, %13;\n\t"
        "madc.lo.cc.u32 %14, m, %23, %14;\n\tmadc.hi.u32    %15, m, %23, %15;\n\t"
        "mad.lo.cc.u32  %0, m, %16, %0;\n\tmadc.hi.cc.u32 %1, m, %16, %1;\n\t"
        "madc.lo.cc.u32 %2, m, %18, %2;\n\tmadc.hi.cc.u32 %3, m, %18, %3;\n\t"
        "madc.lo.cc.u32 %4, m, %20, %4;\n\tmadc.hi.cc.u32 %5, m, %20, %5;\n\t"
        "madc.lo.cc.u32 %6, m, %22, %6;\n\tmadc.hi.cc.u32 %7, m, %22, %7;\n\t"
        "addc.u32       %15, %15, 0;\n\t}"
        : "+r"(x[0]), "+r"(x[1]), "+r"(x[2]), "+r"(x[3]), "+r"(x[4]), "+r"(x[5]), "+r"(x[6]), "+r"(x[7]),
          "+r"(y[0]), "+r"(y[1]), "+r"(y[2]), "+r"(y[3]), "+r"(y[4]), "+r"(y[5]), "+r"(y[6]), "+r"(y[7])
        : "n"(F::M0), "n"(F::M1), "n"(F::M2), "n"(F::M3), "n"(F::M4), "n"(F::M5), "n"(F::M6), "n"(F::M7),
          "n"(F::INV));
}

// Montgomery product a*b*R^{-1} mod N in [0, 2N) for inputs in [0, 2N).
// Eight rows with the accumulators alternating; after the last (odd) row the
// value is u_0..7 + v_1..7 (v_0 is zero).  No final subtraction (lazy
// reduction).
template <class F>
__device__ __forceinline__ Fe<F> fe_mul_inline(const Fe<F> &a, const Fe<F> &b) {
    u32 u[8], v[8];
    bn_row_first(u, v, a.l, b.l[0]);
    bn_row_reduce<F>(u, v);
#pragma unroll
    for (int i = 1; i < 8; i += 2) {
        bn_row_next(v, u, a.l, b.l[i]);
        bn_row_reduce<F>(v, u);
        if (i + 1 < 8) {
            bn_row_next(u, v, a.l, b.l[i + 1]);
            bn_row_reduce<F>(u, v);
        }
    }
    Fe<F> r;
    asm("add.cc.u32  %0, %8, %16;\n\taddc.cc.u32 %1, %9, %17;\n\taddc.cc.u32 %2, %10, %18;\n\t"
        "addc.cc.u32 %3, %11, %19;\n\taddc.cc.u32 %4, %12, %20;\n\taddc.cc.u32 %5, %13, %21;\n\t"
        "addc.cc.u32 %6, %14, %22;\n\taddc.u32    %7, %15, 0;"
        : "=r"(r.l[0]), "=r"(r.l[1]), "=r"(r.l[2]), "=r"(r.l[3]), "=r"(r.l[4]), "=r"(r.l[5]), "=r"(r.l[6]),
          "=r"(r.l[7])
        : "r"(u[0]), "r"(u[1]), "r"(u[2]), "r"(u[3]), "r"(u[4]), "r"(u[5]), "r"(u[6]), "r"(u[7]), "r"(v[1]),
          "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]));
    return r;
}

// Inlined: with the carries folded into the multiply-adds a product is about
// 280 instructions, and ten inlined products per mixed addition leave the
// scheduler free to interleave independent products.  Measured on B200 this
// beats an out-of-line product by 13% on the accumulation loop (the
// out-of-line form won only for the older mul.wide + ALU-add rows, whose
// inlined copies outgrew the instruction cache).
template <class F>
__device__ __forceinline__ Fe<F> fe_mul(Fe<F> a, Fe<F> b) {
    return fe_mul_inline<F>(a, b);
}

template <class F>
__device__ __forceinline__ Fe<F> fe_sqr(const Fe<F> &a) {
    return fe_mul<F>(a, a);
}

// Leave Montgomery form: a * R^{-1} mod N, canonical, for a in [0, 2N)
// (Montgomery reduction only; the sum stays at or below N before the final
// subtraction).
template <class F>
__device__ __forceinline__ Fe<F> fe_from_mont(const Fe<F> &a) {
    u32 t[9];
#pragma unroll
    for (int i = 0; i < 8; i++) t[i] = a.l[i];
    t[8] = 0;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        u32 m = t[0] * F::INV;
        asm("mad.lo.cc.u32  %0, %9, %10, %0;\n\t"
            "madc.lo.cc.u32 %1, %9, %11, %1;\n\t"
            "madc.lo.cc.u32 %2, %9, %12, %2;\n\t"
            "madc.lo.cc.u32 %3, %9, %13, %3;\n\t"
            "madc.lo.cc.u32 %4, %9, %14, %4;\n\t"
            "madc.lo.cc.u32 %5, %9, %15, %5;\n\t"
            "madc.lo.cc.u32 %6, %9, %16, %6;\n\t"
            "madc.lo.cc.u32 %7, %9, %17, %7;\n\t"
            "addc.u32       %8, %8, 0;\n\t"
            "mad.hi.cc.u32  %1, %9, %10, %1;\n\t"
            "madc.hi.cc.u32 %2, %9, %11, %2;\n\t"
            "madc.hi.cc.u32 %3, %9, %12, %3;\n\t"
            "madc.hi.cc.u32 %4, %9, %13, %4;\n\t"
            "madc.hi.cc.u32 %5, %9, %14, %5;\n\t"
            "madc.hi.cc.u32 %6, %9, %15, %6;\n\t"
            "madc.hi.cc.u32 %7, %9, %16, %7;\n\t"
            "madc.hi.u32    %8, %9, %17, %8;"
            : "+r"(t[0]), "+r"(t[1]), "+r"(t[2]), "+r"(t[3]), "+r"(t[4]), "+r"(t[5]), "+r"(t[6]), "+r"(t[7]),
              "+r"(t[8])
            : "r"(m), "n"(F::M0), "n"(F::M1), "n"(F::M2), "n"(F::M3), "n"(F::M4), "n"(F::M5), "n"(F::M6),
              "n"(F::M7));
#pragma unroll
        for (int k = 0; k < 8; k++) t[k] = t[k + 1];
        t[8] = 0;
    }
    Fe<F> r;
    fe_reduce_once<F>(r, t);
    return r;
}

template <class F>
__device__ __forceinline__ Fe<F> fe_add(const Fe<F> &a, const Fe<F> &b) {
    u32 s[8];
    asm("add.cc.u32  %0, %8, %16;\n\t"
        "addc.cc.u32 %1, %9, %17;\n\t"
        "addc.cc.u32 %2, %10, %18;\n\t"
        "addc.cc.u32 %3, %11, %19;\n\t"
        "addc.cc.u32 %4, %12, %20;\n\t"
        "addc.cc.u32 %5, %13, %21;\n\t"
        "addc.cc.u32 %6, %14, %22;\n\t"
        "addc.u32    %7, %15, %23;"
        : "=r"(s[0]), "=r"(s[1]), "=r"(s[2]), "=r"(s[3]), "=r"(s[4]), "=r"(s[5]), "=r"(s[6]), "=r"(s[7])
        : "r"(a.l[0]), "r"(a.l[1]), "r"(a.l[2]), "r"(a.l[3]), "r"(a.l[4]), "r"(a.l[5]), "r"(a.l[6]),
          "r"(a.l[7]), "r"(b.l[0]), "r"(b.l[1]), "r"(b.l[2]), "r"(b.l[3]), "r"(b.l[4]), "r"(b.l[5]),
          "r"(b.l[6]), "r"(b.l[7]));
    Fe<F> r;
    fe_reduce_2n<F>(r, s);  // a + b < 4N < 2^256
    return r;
}

template <class F>
__device__ __forceinline__ Fe<F> fe_sub(const Fe<F> &a, const Fe<F> &b) {
    u32 d[8], bw;
    asm("sub.cc.u32  %0, %9, %17;\n\t"
        "subc.cc.u32 %1, %10, %18;\n\t"
        "subc.cc.u32 %2, %11, %19;\n\t"
        "subc.cc.u32 %3, %12, %20;\n\t"
        "subc.cc.u32 %4, %13, %21;\n\t"
        "subc.cc.u32 %5, %14, %22;\n\t"
        "subc.cc.u32 %6, %15, %23;\n\t"
        "subc.cc.u32 %7, %16, %24;\n\t"
        "subc.u32    %8, 0, 0;"
        : "=r"(d[0]), "=r"(d[1]), "=r"(d[2]), "=r"(d[3]), "=r"(d[4]), "=r"(d[5]), "=r"(d[6]), "=r"(d[7]),
          "=r"(bw)
        : "r"(a.l[0]), "r"(a.l[1]), "r"(a.l[2]), "r"(a.l[3]), "r"(a.l[4]), "r"(a.l[5]), "r"(a.l[6]),
          "r"(a.l[7]), "r"(b.l[0]), "r"(b.l[1]), "r"(b.l[2]), "r"(b.l[3]), "r"(b.l[4]), "r"(b.l[5]),
          "r"(b.l[6]), "r"(b.l[7]));
    Fe<F> r;
    // add 2N back when the subtraction borrowed (bw = 0xffffffff)
    asm("add.cc.u32  %0, %8, %16;\n\t"
        "addc.cc.u32 %1, %9, %17;\n\t"
        "addc.cc.u32 %2, %10, %18;\n\t"
        "addc.cc.u32 %3, %11, %19;\n\t"
        "addc.cc.u32 %4, %12, %20;\n\t"
        "addc.cc.u32 %5, %13, %21;\n\t"
        "addc.cc.u32 %6, %14, %22;\n\t"
        "addc.u32    %7, %15, %23;"
        : "=r"(r.l[0]), "=r"(r.l[1]), "=r"(r.l[2]), "=r"(r.l[3]), "=r"(r.l[4]), "=r"(r.l[5]), "=r"(r.l[6]),
          "=r"(r.l[7])
        : "r"(d[0]), "r"(d[1]), "r"(d[2]), "r"(d[3]), "r"(d[4]), "r"(d[5]), "r"(d[6]), "r"(d[7]),
          "r"(F::D0 & bw), "r"(F::D1 & bw), "r"(F::D2 & bw), "r"(F::D3 & bw), "r"(F::D4 & bw),
          "r"(F::D5 & bw), "r"(F::D6 & bw), "r"(F::D7 & bw));
    return r;
}

template <class F>
__device__ __forceinline__ Fe<F> fe_neg(const Fe<F> &a) {
    return fe_sub<F>(fe_zero<F>(), a);
}

template <class F>
__device__ __forceinline__ Fe<F> fe_dbl(const Fe<F> &a) {
    return fe_add<F>(a, a);
}

// a^e for a plain exponent given as 8 little-endian limbs, 4-bit fixed window.
template <class F>
__device__ __noinline__ Fe<F> fe_pow(const Fe<F> &a, const u32 e[8]) {
    Fe<F> tab[16];
    tab[0] = fe_one<F>();
    tab[1] = a;
#pragma unroll 1
    for (int i = 2; i < 16; i++) tab[i] = fe_mul<F>(tab[i - 1], a);
    Fe<F> acc = fe_one<F>();
#pragma unroll 1
    for (int nib = 63; nib >= 0; nib--) {
        acc = fe_sqr<F>(acc);
        acc = fe_sqr<F>(acc);
        acc = fe_sqr<F>(acc);
        acc = fe_sqr<F>(acc);
        u32 v = (e[nib / 8] >> (4 * (nib % 8))) & 15u;
        // table index is data-dependent; select through a loop to stay in registers
        Fe<F> sel = tab[0];
#pragma unroll
        for (int k = 1; k < 16; k++)
            if (v == (u32)k) sel = tab[k];
        acc = fe_mul<F>(acc, sel);
    }
    return acc;
}

// Fermat inversion a^(N-2); inverse of zero is zero.
template <class F>
__device__ __forceinline__ Fe<F> fe_inv(const Fe<F> &a) {
    u32 e[8] = {F::M0 - 2u, F::M1, F::M2, F::M3, F::M4, F::M5, F::M6, F::M7};
    return fe_pow<F>(a, e);
}

// Single-thread-latency inversion for the few conversions to affine form at
// the end of an MSM: binary extended Euclid on the integer representative
// (Montgomery form a = A*R) gives a^{-1} = A^{-1} R^{-1}; one Montgomery
// product with R^3 mod N turns it into A^{-1} R.  Variable time (the inputs
// are public).  Inverse of zero is zero.  The loop is bounded: every step
// shrinks u + v by at least one bit.
template <class F>
__device__ __forceinline__ bool u256_is_one(const u32 x[8]) {
    return x[0] == 1 && (x[1] | x[2] | x[3] | x[4] | x[5] | x[6] | x[7]) == 0;
}

__device__ __forceinline__ void u256_shr1(u32 x[8], u32 top) {
#pragma unroll
    for (int i = 0; i < 7; i++) x[i] = __funnelshift_r(x[i], x[i + 1], 1);
    x[7] = (x[7] >> 1) | (top << 31);
}

__device__ __forceinline__ bool u256_geq(const u32 a[8], const u32 b[8]) {
    for (int i = 7; i >= 0; i--)
        if (a[i] != b[i]) return a[i] > b[i];
    return true;
}

__device__ __forceinline__ void u256_sub(u32 a[8], const u32 b[8]) {
    asm("sub.cc.u32  %0, %0, %8;\n\t"
        "subc.cc.u32 %1, %1, %9;\n\t"
        "subc.cc.u32 %2, %2, %10;\n\t"
        "subc.cc.u32 %3, %3, %11;\n\t"
        "subc.cc.u32 %4, %4, %12;\n\t"
        "subc.cc.u32 %5, %5, %13;\n\t"
        "subc.cc.u32 %6, %6, %14;\n\t"
        "subc.u32    %7, %7, %15;"
        : "+r"(a[0]), "+r"(a[1]), "+r"(a[2]), "+r"(a[3]), "+r"(a[4]), "+r"(a[5]), "+r"(a[6]), "+r"(a[7])
        : "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]));
}

// x = x / 2 mod N for x < 2N (N odd): if x is odd, (x + N) / 2 < 3N / 2.
template <class F>
__device__ __forceinline__ void fe_half(u32 x[8]) {
    if (x[0] & 1u) {
        u32 c;
        asm("add.cc.u32  %0, %0, %9;\n\t"
            "addc.cc.u32 %1, %1, %10;\n\t"
            "addc.cc.u32 %2, %2, %11;\n\t"
            "addc.cc.u32 %3, %3, %12;\n\t"
            "addc.cc.u32 %4, %4, %13;\n\t"
            "addc.cc.u32 %5, %5, %14;\n\t"
            "addc.cc.u32 %6, %6, %15;\n\t"
            "addc.cc.u32 %7, %7, %16;\n\t"
            "addc.u32    %8, 0, 0;"
            : "+r"(x[0]), "+r"(x[1]), "+r"(x[2]), "+r"(x[3]), "+r"(x[4]), "+r"(x[5]), "+r"(x[6]), "+r"(x[7]),
              "=r"(c)
            : "n"(F::M0), "n"(F::M1), "n"(F::M2), "n"(F::M3), "n"(F::M4), "n"(F::M5), "n"(F::M6), "n"(F::M7));
        u256_shr1(x, c);
    } else {
        u256_shr1(x, 0);
    }
}

template <class F>
__device__ __noinline__ Fe<F> fe_inv_binary(const Fe<F> &a_in, const Fe<F> &r3) {
    const Fe<F> a = fe_canon<F>(a_in);
    if (fe_is_zero_canonical(a)) return a;
    u32 u[8], v[8];
    Fe<F> x1 = fe_zero<F>(), x2 = fe_zero<F>();
    x1.l[0] = 1;
#pragma unroll
    for (int i = 0; i < 8; i++) u[i] = a.l[i];
    v[0] = F::M0; v[1] = F::M1; v[2] = F::M2; v[3] = F::M3;
    v[4] = F::M4; v[5] = F::M5; v[6] = F::M6; v[7] = F::M7;
    // One shift or one subtraction per step; a valid input (0 < a < N, N
    // prime) needs at most ~4 * 254 steps.  The zero check and the step bound
    // keep a non-canonical input from looping: it yields zero.
    bool done = false;
    for (int step = 0; step < 4096; step++) {
        if (u256_is_one<F>(u) || u256_is_one<F>(v)) {
            done = true;
            break;
        }
        if ((u[0] | u[1] | u[2] | u[3] | u[4] | u[5] | u[6] | u[7]) == 0 ||
            (v[0] | v[1] | v[2] | v[3] | v[4] | v[5] | v[6] | v[7]) == 0)
            break;
        if (!(u[0] & 1u)) {
            u256_shr1(u, 0);
            fe_half<F>(x1.l);
        } else if (!(v[0] & 1u)) {
            u256_shr1(v, 0);
            fe_half<F>(x2.l);
        } else if (u256_geq(u, v)) {
            u256_sub(u, v);
            x1 = fe_sub<F>(x1, x2);
        } else {
            u256_sub(v, u);
            x2 = fe_sub<F>(x2, x1);
        }
    }
    if (!done) return fe_zero<F>();
    return fe_mul<F>(u256_is_one<F>(u) ? x1 : x2, r3);
}

template <class F>
__device__ __forceinline__ Fe<F> fe_load(const u32 *p) {
    Fe<F> r;
    const uint4 *q = reinterpret_cast<const uint4 *>(p);
    uint4 lo = q[0], hi = q[1];
    r.l[0] = lo.x; r.l[1] = lo.y; r.l[2] = lo.z; r.l[3] = lo.w;
    r.l[4] = hi.x; r.l[5] = hi.y; r.l[6] = hi.z; r.l[7] = hi.w;
    return r;
}

template <class F>
__device__ __forceinline__ void fe_store(u32 *p, const Fe<F> &a) {
    uint4 *q = reinterpret_cast<uint4 *>(p);
    q[0] = make_uint4(a.l[0], a.l[1], a.l[2], a.l[3]);
    q[1] = make_uint4(a.l[4], a.l[5], a.l[6], a.l[7]);
}

// ---------------------------------------------------------------- G1 (XYZZ)

struct Affine {
    Fq x, y;
};

struct Xyzz {
    Fq x, y, zz, zzz;
};

// Affine points come from memory in canonical form; negation keeps 0 at 0.
__device__ __forceinline__ bool affine_is_identity(const Affine &a) { return fe_is_zero_canonical(a.y); }

__device__ __forceinline__ Xyzz xyzz_identity() {
    Xyzz r;
    r.x = fe_zero<FqP>();
    r.y = fe_zero<FqP>();
    r.zz = fe_zero<FqP>();
    r.zzz = fe_zero<FqP>();
    return r;
}

__device__ __forceinline__ bool xyzz_is_identity(const Xyzz &p) { return fe_is_zero(p.zz); }

__device__ __forceinline__ Xyzz xyzz_from_affine(const Affine &a) {
    if (affine_is_identity(a)) return xyzz_identity();
    Xyzz r;
    r.x = a.x;
    r.y = a.y;
    r.zz = fe_one<FqP>();
    r.zzz = r.zz;
    return r;
}

__device__ __forceinline__ Affine affine_neg(const Affine &a) {
    Affine r;
    r.x = a.x;
    r.y = fe_neg<FqP>(a.y);
    return r;
}

__device__ __forceinline__ Xyzz xyzz_neg(const Xyzz &p) {
    Xyzz r = p;
    r.y = fe_neg<FqP>(p.y);
    return r;
}

// mdbl-2008-s-1: 2*a for an affine, non-identity a.
__device__ __forceinline__ Xyzz affine_dbl(const Affine &a) {
    Fq u = fe_dbl(a.y);
    Fq v = fe_sqr(u);
    Fq w = fe_mul(u, v);
    Fq s = fe_mul(a.x, v);
    Fq x2 = fe_sqr(a.x);
    Fq m = fe_add(fe_dbl(x2), x2);
    Xyzz r;
    r.x = fe_sub(fe_sub(fe_sqr(m), s), s);
    r.y = fe_sub(fe_mul(m, fe_sub(s, r.x)), fe_mul(w, a.y));
    r.zz = v;
    r.zzz = w;
    return r;
}

// dbl-2008-s-1 with a = 0.
__device__ __forceinline__ Xyzz xyzz_dbl(const Xyzz &p) {
    if (xyzz_is_identity(p)) return p;
    Fq u = fe_dbl(p.y);
    Fq v = fe_sqr(u);
    Fq w = fe_mul(u, v);
    Fq s = fe_mul(p.x, v);
    Fq x2 = fe_sqr(p.x);
    Fq m = fe_add(fe_dbl(x2), x2);
    Xyzz r;
    r.x = fe_sub(fe_sub(fe_sqr(m), s), s);
    r.y = fe_sub(fe_mul(m, fe_sub(s, r.x)), fe_mul(w, p.y));
    r.zz = fe_mul(v, p.zz);
    r.zzz = fe_mul(w, p.zzz);
    return r;
}

// madd-2008-s: p + q, q affine.  Handles every special case.
__device__ __forceinline__ Xyzz xyzz_add_affine(const Xyzz &p, const Affine &q) {
    if (affine_is_identity(q)) return p;
    if (xyzz_is_identity(p)) return xyzz_from_affine(q);
    Fq u2 = fe_mul(q.x, p.zz);
    Fq s2 = fe_mul(q.y, p.zzz);
    Fq P = fe_sub(u2, p.x);
    Fq R = fe_sub(s2, p.y);
    if (fe_is_zero(P)) {
        if (fe_is_zero(R)) return affine_dbl(q);
        return xyzz_identity();
    }
    Fq pp = fe_sqr(P);
    Fq ppp = fe_mul(P, pp);
    Fq Q = fe_mul(p.x, pp);
    Xyzz r;
    r.zz = fe_mul(p.zz, pp);
    r.zzz = fe_mul(p.zzz, ppp);
    Fq t = fe_mul(p.y, ppp);
    r.x = fe_sub(fe_sub(fe_sub(fe_sqr(R), ppp), Q), Q);
    r.y = fe_sub(fe_mul(R, fe_sub(Q, r.x)), t);
    return r;
}

// add-2008-s: p + q.  Handles every special case.
__device__ __forceinline__ Xyzz xyzz_add(const Xyzz &p, const Xyzz &q) {
    if (xyzz_is_identity(p)) return q;
    if (xyzz_is_identity(q)) return p;
    Fq u1 = fe_mul(p.x, q.zz);
    Fq u2 = fe_mul(q.x, p.zz);
    Fq s1 = fe_mul(p.y, q.zzz);
    Fq s2 = fe_mul(q.y, p.zzz);
    Fq P = fe_sub(u2, u1);
    Fq R = fe_sub(s2, s1);
    if (fe_is_zero(P)) {
        if (fe_is_zero(R)) return xyzz_dbl(p);
        return xyzz_identity();
    }
    Fq pp = fe_sqr(P);
    Fq ppp = fe_mul(P, pp);
    Fq Q = fe_mul(u1, pp);
    Xyzz r;
    r.zz = fe_mul(fe_mul(p.zz, q.zz), pp);
    r.zzz = fe_mul(fe_mul(p.zzz, q.zzz), ppp);
    Fq t = fe_mul(s1, ppp);
    r.x = fe_sub(fe_sub(fe_sub(fe_sqr(R), ppp), Q), Q);
    r.y = fe_sub(fe_mul(R, fe_sub(Q, r.x)), t);
    return r;
}

__device__ __forceinline__ Fq fq_r3() {
    Fq r;  // R^3 mod p
    r.l[0] = 0xda1530dfu; r.l[1] = 0xb1cd6dafu; r.l[2] = 0xa7283db6u; r.l[3] = 0x62f210e6u;
    r.l[4] = 0x0ada0afbu; r.l[5] = 0xef7f0b0cu; r.l[6] = 0x2d592544u; r.l[7] = 0x20fd6e90u;
    return r;
}

// Canonical affine form; identity -> (0, 0).  Latency-optimised (binary
// inversion): used once per MSM result.
__device__ __forceinline__ Affine xyzz_to_affine_fast(const Xyzz &p) {
    Affine r;
    if (xyzz_is_identity(p)) {
        r.x = fe_zero<FqP>();
        r.y = fe_zero<FqP>();
        return r;
    }
    Fq a = fe_inv_binary<FqP>(p.zzz, fq_r3());
    Fq b = fe_sqr(fe_mul(p.zz, a));
    r.x = fe_canon(fe_mul(p.x, b));
    r.y = fe_canon(fe_mul(p.y, a));
    return r;
}

// Canonical affine form; identity -> (0, 0).
__device__ __forceinline__ Affine xyzz_to_affine(const Xyzz &p) {
    Affine r;
    if (xyzz_is_identity(p)) {
        r.x = fe_zero<FqP>();
        r.y = fe_zero<FqP>();
        return r;
    }
    Fq a = fe_inv(p.zzz);
    Fq b = fe_sqr(fe_mul(p.zz, a));
    r.x = fe_canon(fe_mul(p.x, b));
    r.y = fe_canon(fe_mul(p.y, a));
    return r;
}

__device__ __forceinline__ Affine affine_load(const u32 *p) {
    Affine a;
    const uint4 *q = reinterpret_cast<const uint4 *>(p);
    uint4 v0 = q[0], v1 = q[1], v2 = q[2], v3 = q[3];
    a.x.l[0] = v0.x; a.x.l[1] = v0.y; a.x.l[2] = v0.z; a.x.l[3] = v0.w;
    a.x.l[4] = v1.x; a.x.l[5] = v1.y; a.x.l[6] = v1.z; a.x.l[7] = v1.w;
    a.y.l[0] = v2.x; a.y.l[1] = v2.y; a.y.l[2] = v2.z; a.y.l[3] = v2.w;
    a.y.l[4] = v3.x; a.y.l[5] = v3.y; a.y.l[6] = v3.z; a.y.l[7] = v3.w;
    return a;
}

__device__ __forceinline__ void affine_store(u32 *p, const Affine &a) {
    fe_store(p, a.x);
    fe_store(p + 8, a.y);
}

__device__ __forceinline__ Xyzz xyzz_load(const u32 *p) {
    Xyzz r;
    r.x = fe_load<FqP>(p);
    r.y = fe_load<FqP>(p + 8);
    r.zz = fe_load<FqP>(p + 16);
    r.zzz = fe_load<FqP>(p + 24);
    return r;
}

__device__ __forceinline__ void xyzz_store(u32 *p, const Xyzz &a) {
    fe_store(p, a.x);
    fe_store(p + 8, a.y);
    fe_store(p + 16, a.zz);
    fe_store(p + 24, a.zzz);
}

__device__ __forceinline__ Xyzz xyzz_shfl_down(const Xyzz &p, u32 delta, u32 mask = 0xffffffffu) {
    Xyzz r;
#pragma unroll
    for (int i = 0; i < 8; i++) {
        r.x.l[i] = __shfl_down_sync(mask, p.x.l[i], delta);
        r.y.l[i] = __shfl_down_sync(mask, p.y.l[i], delta);
        r.zz.l[i] = __shfl_down_sync(mask, p.zz.l[i], delta);
        r.zzz.l[i] = __shfl_down_sync(mask, p.zzz.l[i], delta);
    }
    return r;
}

// k * p for a small plain scalar k, left-to-right double-and-add.
__device__ __forceinline__ Xyzz xyzz_mul_u32(const Xyzz &p, u32 k) {
    Xyzz acc = xyzz_identity();
    if (k == 0) return acc;
    int top = 31 - __clz(k);
#pragma unroll 1
    for (int i = top; i >= 0; i--) {
        acc = xyzz_dbl(acc);
        if ((k >> i) & 1u) acc = xyzz_add(acc, p);
    }
    return acc;
}

}  // namespace bn254
