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

namespace ec {

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
    static constexpr int N = 8;         // limbs
    static constexpr bool LAZY = true;  // values kept in [0, 2p) (4p < 2^256)
    static constexpr u32 M[8] = {M0, M1, M2, M3, M4, M5, M6, M7};
    static constexpr u32 R[8] = {R0, R1, R2, R3, R4, R5, R6, R7};
    // R^3 mod p (binary inversion)
    static constexpr u32 RCUBE[8] = {0xda1530dfu, 0xb1cd6dafu, 0xa7283db6u, 0x62f210e6u,
                                     0x0ada0afbu, 0xef7f0b0cu, 0x2d592544u, 0x20fd6e90u};
    // R^2 mod p (conversion into Montgomery form)
    static constexpr u32 RSQ[8] = {0x538afa89u, 0xf32cfc5bu, 0xd44501fbu, 0xb5e71911u,
                                   0x0a417ff6u, 0x47ab1effu, 0xcab8351fu, 0x06d89f71u};
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
    static constexpr int N = 8;
    static constexpr bool LAZY = true;  // r < 2^254 as well
    static constexpr u32 M[8] = {M0, M1, M2, M3, M4, M5, M6, M7};
    static constexpr u32 R[8] = {R0, R1, R2, R3, R4, R5, R6, R7};
    static constexpr u32 RSQ[8] = {0xae216da7u, 0x1bb8e645u, 0xe35c59e3u, 0x53fe3ab1u,
                                   0x53bb8085u, 0x8c49833du, 0x7f4e44a5u, 0x0216d0b1u};
};

// BLS12-381 scalar field Fr: r < 2^255, so 4r > 2^256 and values stay
// canonical (every operation reduces fully).  8 limbs like BN254's fields.
struct BlsFrP {
    static constexpr u32 M0 = 0x00000001u, M1 = 0xffffffffu, M2 = 0xfffe5bfeu, M3 = 0x53bda402u;
    static constexpr u32 M4 = 0x09a1d805u, M5 = 0x3339d808u, M6 = 0x299d7d48u, M7 = 0x73eda753u;
    static constexpr u32 INV = 0xffffffffu;  // -r^{-1} mod 2^32
    static constexpr u32 R0 = 0xfffffffeu, R1 = 0x00000001u, R2 = 0x00034802u, R3 = 0x5884b7fau;
    static constexpr u32 R4 = 0xecbc4ff5u, R5 = 0x998c4fefu, R6 = 0xacc5056fu, R7 = 0x1824b159u;
    static constexpr u32 D0 = 0x00000002u, D1 = 0xfffffffeu, D2 = 0xfffcb7fdu, D3 = 0xa77b4805u;
    static constexpr u32 D4 = 0x1343b00au, D5 = 0x6673b010u, D6 = 0x533afa90u, D7 = 0xe7db4ea6u;
    static constexpr int N = 8;
    static constexpr bool LAZY = false;
    static constexpr u32 M[8] = {M0, M1, M2, M3, M4, M5, M6, M7};
    static constexpr u32 R[8] = {R0, R1, R2, R3, R4, R5, R6, R7};
    static constexpr u32 RSQ[8] = {0xf3f29c6du, 0xc999e990u, 0x87925c23u, 0x2b6cedcbu,
                                   0x7254398fu, 0x05d31496u, 0x9f59ff11u, 0x0748d9d9u};
};

// BLS12-381 base field Fq: 381-bit p in 12 limbs; 4p < 2^384, values in [0, 2p).
struct BlsFqP {
    static constexpr int N = 12;
    static constexpr bool LAZY = true;
    static constexpr u32 INV = 0xfffcfffdu;  // -p^{-1} mod 2^32
    static constexpr u32 M[12] = {0xffffaaabu, 0xb9feffffu, 0xb153ffffu, 0x1eabfffeu, 0xf6b0f624u, 0x6730d2a0u,
                                  0xf38512bfu, 0x64774b84u, 0x434bacd7u, 0x4b1ba7b6u, 0x397fe69au, 0x1a0111eau};
    static constexpr u32 D[12] = {0xffff5556u, 0x73fdffffu, 0x62a7ffffu, 0x3d57fffdu, 0xed61ec48u, 0xce61a541u,
                                  0xe70a257eu, 0xc8ee9709u, 0x869759aeu, 0x96374f6cu, 0x72ffcd34u, 0x340223d4u};
    static constexpr u32 R[12] = {0x0002fffdu, 0x76090000u, 0xc40c0002u, 0xebf4000bu, 0x53c758bau, 0x5f489857u,
                                  0x70525745u, 0x77ce5853u, 0xa256ec6du, 0x5c071a97u, 0xfa80e493u, 0x15f65ec3u};
    static constexpr u32 RCUBE[12] = {0xd94ca1e0u, 0xed48ac6bu, 0x03a7adf8u, 0x315f831eu, 0x615e29ddu, 0x9a53352au,
                                      0x921e1761u, 0x34c04e5eu, 0x65724728u, 0x2512d435u, 0x91755d4du, 0x0aa63460u};
    static constexpr u32 RSQ[12] = {0x1c341746u, 0xf4df1f34u, 0x09d104f1u, 0x0a76e6a6u, 0x4c95b6d5u, 0x8de5476cu,
                                    0x939d83c0u, 0x67eb88a9u, 0xb519952du, 0x9a793e85u, 0x92cae3aau, 0x11988fe5u};
};

// Curves: base field, scalar field, affine / XYZZ point words and the
// generator in Montgomery form.  BN254 G1: y^2 = x^3 + 3, G = (1, 2).
// BLS12-381 G1: y^2 = x^3 + 4, the standard generator
// (x = 0x17f1d3a7...db22c6bb, y = 0x08b3f481...46c5e7e1).
struct Bn254 {
    using Fq = FqP;
    using Fr = FrP;
    static constexpr u32 PW = 16, XW = 32;
    // signed-digit windows of width c (3 <= c <= 31) for scalars below r < 2^254:
    // the top digit plus its incoming carry stays at most 2^(c-1)
    __host__ __device__ static constexpr u32 windows(u32 c) { return (254u + c - 1u) / c; }
    static constexpr u32 GX[8] = {FqP::R0, FqP::R1, FqP::R2, FqP::R3, FqP::R4, FqP::R5, FqP::R6, FqP::R7};
    static constexpr u32 GY[8] = {0x8b1e1b3au, 0xa6ba871bu, 0xeb8e167bu, 0x14f1d651u,
                                  0xf0f28c58u, 0xccdd46deu, 0x340fbe5eu, 0x1c14ef83u};
};
struct Bls12381 {
    using Fq = BlsFqP;
    using Fr = BlsFrP;
    static constexpr u32 PW = 24, XW = 48;
    // the smallest W with ((r - 1) >> (c (W - 1))) + 1 <= 2^(c - 1), r the
    // group order (255 bits): ceil(255 / c), plus one for c = 3, 5, 15, 17
    __host__ __device__ static constexpr u32 windows(u32 c) {
        return c == 3 || c == 5 || c == 15 || c == 17 ? (255u + c - 1u) / c + 1u : (255u + c - 1u) / c;
    }
    static constexpr u32 GX[12] = {0xfd530c16u, 0x5cb38790u, 0x9976fff5u, 0x7817fc67u, 0x143ba1c1u, 0x154f95c7u,
                                   0xf3d0e747u, 0xf0ae6acdu, 0x21dbf440u, 0xedce6eccu, 0x9e0bfb75u, 0x12017741u};
    static constexpr u32 GY[12] = {0x0ce72271u, 0xbaac93d5u, 0x7918fd8eu, 0x8c22631au, 0x570725ceu, 0xdd595f13u,
                                   0x50405194u, 0x51ac5829u, 0xad0059c0u, 0x0e1c8c3fu, 0x5008a26au, 0x0bbc3efcu};
};

template <class F>
struct Fe {
    u32 l[F::N];
};

// A field constant (F::M, F::R, ...) as a value: device code copies it into
// a local constexpr with `constexpr Words<F::N> m = words(F::M);` and indexes
// that (the traits' arrays themselves live in host memory).
template <int N>
struct Words {
    u32 v[N];
};

template <int N>
__host__ __device__ constexpr Words<N> words(const u32 (&a)[N]) {
    Words<N> r{};
    for (int i = 0; i < N; i++) r.v[i] = a[i];
    return r;
}

typedef Fe<FqP> Fq;
typedef Fe<FrP> Fr;

template <class F>
__host__ __device__ __forceinline__ Fe<F> fe_zero() {
    Fe<F> r;
#pragma unroll
    for (int i = 0; i < F::N; i++) r.l[i] = 0;
    return r;
}

template <class F>
__host__ __device__ __forceinline__ Fe<F> fe_one() {
    constexpr Words<F::N> one = words(F::R);
    Fe<F> r;
#pragma unroll
    for (int i = 0; i < F::N; i++) r.l[i] = one.v[i];
    return r;
}

// R^3 mod N as a field element (binary inversion).
template <class F>
__device__ __forceinline__ Fe<F> fe_rcube() {
    constexpr Words<F::N> rc = words(F::RCUBE);
    Fe<F> r;
#pragma unroll
    for (int i = 0; i < F::N; i++) r.l[i] = rc.v[i];
    return r;
}

// Zero test for a canonical value (in [0, N)).
template <class F>
__device__ __forceinline__ bool fe_is_zero_canonical(const Fe<F> &a) {
    u32 x = 0;
#pragma unroll
    for (int i = 0; i < F::N; i++) x |= a.l[i];
    return x == 0;
}

// Zero test for a field value: 0 or N in the lazy range [0, 2N).
template <class F>
__device__ __forceinline__ bool fe_is_zero(const Fe<F> &a) {
    if constexpr (!F::LAZY) {
        return fe_is_zero_canonical(a);
    } else {
        constexpr Words<F::N> m = words(F::M);
        u32 x = 0, y = 0;
#pragma unroll
        for (int i = 0; i < F::N; i++) {
            x |= a.l[i];
            y |= a.l[i] ^ m.v[i];
        }
        return x == 0 || y == 0;
    }
}

}  // namespace ec

#include "field12.cuh"
#include "safegcd.cuh"

namespace ec {

// r = (t < N) ? t : t - N, for t < 2N.
template <class F>
__device__ __forceinline__ void fe_reduce_once(Fe<F> &r, const u32 *t) {
    if constexpr (F::N == 12) {
        constexpr Words<12> m = words(F::M);
        u32 d[12];
        const u32 bw = sub12(d, t, m.v);
#pragma unroll
        for (int i = 0; i < 12; i++) r.l[i] = bw ? t[i] : d[i];
        return;
    } else {
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
}

// r = (t < 2N) ? t : t - 2N, for t < 4N.
template <class F>
__device__ __forceinline__ void fe_reduce_2n(Fe<F> &r, const u32 *t) {
    if constexpr (F::N == 12) {
        constexpr Words<12> d2 = words(F::D);
        u32 d[12];
        const u32 bw = sub12(d, t, d2.v);
#pragma unroll
        for (int i = 0; i < 12; i++) r.l[i] = bw ? t[i] : d[i];
        return;
    } else {
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

// Square of an 8-word value, all 16 words: the 28 cross products a_i a_j
// (i < j) go into two accumulators of register pairs -- E on even-aligned
// pairs, O on odd-aligned ones -- so that every lo/hi multiply-add lands on
// an aligned pair; each row's chain ends on a word no earlier row wrote, or
// hands its carry to the next such word.  Then t = 2 (E + O) + sum a_i^2
// 2^(64 i).  36 products where a general product of two values takes 64.
__device__ __forceinline__ void bn_sqr_wide(u32 (&t)[16], const u32 (&a)[8]) {
    asm(
        "{\n\t.reg .u32 E2, E3, E4, E5, E6, E7, E8, E9, E10, E11, E12, E13, O1, O2, O3, O4, O5, O6, O7, O8, O9, O10, O11, O12, O13, O14;\n\t"
        "mul.lo.u32 O1, %16, %17;\n\t"
        "mul.hi.u32 O2, %16, %17;\n\t"
        "mul.lo.u32 O3, %16, %19;\n\t"
        "mul.hi.u32 O4, %16, %19;\n\t"
        "mul.lo.u32 O5, %16, %21;\n\t"
        "mul.hi.u32 O6, %16, %21;\n\t"
        "mul.lo.u32 O7, %16, %23;\n\t"
        "mul.hi.u32 O8, %16, %23;\n\t"
        "mul.lo.u32 E2, %16, %18;\n\t"
        "mul.hi.u32 E3, %16, %18;\n\t"
        "mul.lo.u32 E4, %16, %20;\n\t"
        "mul.hi.u32 E5, %16, %20;\n\t"
        "mul.lo.u32 E6, %16, %22;\n\t"
        "mul.hi.u32 E7, %16, %22;\n\t"
        "mad.lo.cc.u32 O3, %17, %18, O3;\n\t"
        "madc.hi.cc.u32 O4, %17, %18, O4;\n\t"
        "madc.lo.cc.u32 O5, %17, %20, O5;\n\t"
        "madc.hi.cc.u32 O6, %17, %20, O6;\n\t"
        "madc.lo.cc.u32 O7, %17, %22, O7;\n\t"
        "madc.hi.cc.u32 O8, %17, %22, O8;\n\t"
        "addc.u32 O9, 0, 0;\n\t"
        "mad.lo.cc.u32 E4, %17, %19, E4;\n\t"
        "madc.hi.cc.u32 E5, %17, %19, E5;\n\t"
        "madc.lo.cc.u32 E6, %17, %21, E6;\n\t"
        "madc.hi.cc.u32 E7, %17, %21, E7;\n\t"
        "madc.lo.cc.u32 E8, %17, %23, 0;\n\t"
        "madc.hi.u32 E9, %17, %23, 0;\n\t"
        "mad.lo.cc.u32 O5, %18, %19, O5;\n\t"
        "madc.hi.cc.u32 O6, %18, %19, O6;\n\t"
        "madc.lo.cc.u32 O7, %18, %21, O7;\n\t"
        "madc.hi.cc.u32 O8, %18, %21, O8;\n\t"
        "madc.lo.cc.u32 O9, %18, %23, O9;\n\t"
        "madc.hi.u32 O10, %18, %23, 0;\n\t"
        "mad.lo.cc.u32 E6, %18, %20, E6;\n\t"
        "madc.hi.cc.u32 E7, %18, %20, E7;\n\t"
        "madc.lo.cc.u32 E8, %18, %22, E8;\n\t"
        "madc.hi.cc.u32 E9, %18, %22, E9;\n\t"
        "addc.u32 E10, 0, 0;\n\t"
        "mad.lo.cc.u32 O7, %19, %20, O7;\n\t"
        "madc.hi.cc.u32 O8, %19, %20, O8;\n\t"
        "madc.lo.cc.u32 O9, %19, %22, O9;\n\t"
        "madc.hi.cc.u32 O10, %19, %22, O10;\n\t"
        "addc.u32 O11, 0, 0;\n\t"
        "mad.lo.cc.u32 E8, %19, %21, E8;\n\t"
        "madc.hi.cc.u32 E9, %19, %21, E9;\n\t"
        "madc.lo.cc.u32 E10, %19, %23, E10;\n\t"
        "madc.hi.u32 E11, %19, %23, 0;\n\t"
        "mad.lo.cc.u32 O9, %20, %21, O9;\n\t"
        "madc.hi.cc.u32 O10, %20, %21, O10;\n\t"
        "madc.lo.cc.u32 O11, %20, %23, O11;\n\t"
        "madc.hi.u32 O12, %20, %23, 0;\n\t"
        "mad.lo.cc.u32 E10, %20, %22, E10;\n\t"
        "madc.hi.cc.u32 E11, %20, %22, E11;\n\t"
        "addc.u32 E12, 0, 0;\n\t"
        "mad.lo.cc.u32 O11, %21, %22, O11;\n\t"
        "madc.hi.cc.u32 O12, %21, %22, O12;\n\t"
        "addc.u32 O13, 0, 0;\n\t"
        "mad.lo.cc.u32 E12, %21, %23, E12;\n\t"
        "madc.hi.u32 E13, %21, %23, 0;\n\t"
        "mad.lo.cc.u32 O13, %22, %23, O13;\n\t"
        "madc.hi.u32 O14, %22, %23, 0;\n\t"
        "add.cc.u32 %1, 0, O1;\n\t"
        "addc.cc.u32 %2, E2, O2;\n\t"
        "addc.cc.u32 %3, E3, O3;\n\t"
        "addc.cc.u32 %4, E4, O4;\n\t"
        "addc.cc.u32 %5, E5, O5;\n\t"
        "addc.cc.u32 %6, E6, O6;\n\t"
        "addc.cc.u32 %7, E7, O7;\n\t"
        "addc.cc.u32 %8, E8, O8;\n\t"
        "addc.cc.u32 %9, E9, O9;\n\t"
        "addc.cc.u32 %10, E10, O10;\n\t"
        "addc.cc.u32 %11, E11, O11;\n\t"
        "addc.cc.u32 %12, E12, O12;\n\t"
        "addc.cc.u32 %13, E13, O13;\n\t"
        "addc.cc.u32 %14, 0, O14;\n\t"
        "addc.u32 %15, 0, 0;\n\t"
        "add.cc.u32 %1, %1, %1;\n\t"
        "addc.cc.u32 %2, %2, %2;\n\t"
        "addc.cc.u32 %3, %3, %3;\n\t"
        "addc.cc.u32 %4, %4, %4;\n\t"
        "addc.cc.u32 %5, %5, %5;\n\t"
        "addc.cc.u32 %6, %6, %6;\n\t"
        "addc.cc.u32 %7, %7, %7;\n\t"
        "addc.cc.u32 %8, %8, %8;\n\t"
        "addc.cc.u32 %9, %9, %9;\n\t"
        "addc.cc.u32 %10, %10, %10;\n\t"
        "addc.cc.u32 %11, %11, %11;\n\t"
        "addc.cc.u32 %12, %12, %12;\n\t"
        "addc.cc.u32 %13, %13, %13;\n\t"
        "addc.cc.u32 %14, %14, %14;\n\t"
        "addc.u32 %15, %15, %15;\n\t"
        "mul.lo.u32 %0, %16, %16;\n\t"
        "mad.hi.cc.u32 %1, %16, %16, %1;\n\t"
        "madc.lo.cc.u32 %2, %17, %17, %2;\n\t"
        "madc.hi.cc.u32 %3, %17, %17, %3;\n\t"
        "madc.lo.cc.u32 %4, %18, %18, %4;\n\t"
        "madc.hi.cc.u32 %5, %18, %18, %5;\n\t"
        "madc.lo.cc.u32 %6, %19, %19, %6;\n\t"
        "madc.hi.cc.u32 %7, %19, %19, %7;\n\t"
        "madc.lo.cc.u32 %8, %20, %20, %8;\n\t"
        "madc.hi.cc.u32 %9, %20, %20, %9;\n\t"
        "madc.lo.cc.u32 %10, %21, %21, %10;\n\t"
        "madc.hi.cc.u32 %11, %21, %21, %11;\n\t"
        "madc.lo.cc.u32 %12, %22, %22, %12;\n\t"
        "madc.hi.cc.u32 %13, %22, %22, %13;\n\t"
        "madc.lo.cc.u32 %14, %23, %23, %14;\n\t"
        "madc.hi.u32 %15, %23, %23, %15;\n\t"
        "}"
        : "=r"(t[0]), "=r"(t[1]), "=r"(t[2]), "=r"(t[3]), "=r"(t[4]), "=r"(t[5]), "=r"(t[6]), "=r"(t[7]),
          "=r"(t[8]), "=r"(t[9]), "=r"(t[10]), "=r"(t[11]), "=r"(t[12]), "=r"(t[13]), "=r"(t[14]), "=r"(t[15])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]));
}

// Squaring's reduction row: the division of the running value by 2^32 (the
// role swap of bn_row_next: x becomes the old Y array, y the old X array two
// words down, old X_1 added at weight 0), the square's next word w entering
// at weight 7 (as y_6, a zero word after the shift), and the reduction row of
// bn_row_reduce, in one carry chain.
template <class F>
__device__ __forceinline__ void bn_row_reduce_word(u32 (&x)[8], u32 (&y)[8], u32 w) {
    asm("{\n\t.reg .u32 m;\n\t"
        "add.cc.u32     %0, %0, %9;\n\t"
        "mul.lo.u32     m, %0, %24;\n\t"
        "madc.lo.cc.u32 %8, m, %17, %10;\n\tmadc.hi.cc.u32 %9, m, %17, %11;\n\t"
        "madc.lo.cc.u32 %10, m, %19, %12;\n\tmadc.hi.cc.u32 %11, m, %19, %13;\n\t"
        "madc.lo.cc.u32 %12, m, %21, %14;\n\tmadc.hi.cc.u32 %13, m, %21, %15;\n\t"
        "madc.lo.cc.u32 %14, m, %23, %25;\n\tmadc.hi.u32    %15, m, %23, 0;\n\t"
        "mad.lo.cc.u32  %0, m, %16, %0;\n\tmadc.hi.cc.u32 %1, m, %16, %1;\n\t"
        "madc.lo.cc.u32 %2, m, %18, %2;\n\tmadc.hi.cc.u32 %3, m, %18, %3;\n\t"
        "madc.lo.cc.u32 %4, m, %20, %4;\n\tmadc.hi.cc.u32 %5, m, %20, %5;\n\t"
        "madc.lo.cc.u32 %6, m, %22, %6;\n\tmadc.hi.cc.u32 %7, m, %22, %7;\n\t"
        "addc.u32       %15, %15, 0;\n\t}"
        : "+r"(x[0]), "+r"(x[1]), "+r"(x[2]), "+r"(x[3]), "+r"(x[4]), "+r"(x[5]), "+r"(x[6]), "+r"(x[7]),
          "+r"(y[0]), "+r"(y[1]), "+r"(y[2]), "+r"(y[3]), "+r"(y[4]), "+r"(y[5]), "+r"(y[6]), "+r"(y[7])
        : "n"(F::M0), "n"(F::M1), "n"(F::M2), "n"(F::M3), "n"(F::M4), "n"(F::M5), "n"(F::M6), "n"(F::M7),
          "n"(F::INV), "r"(w));
}

// Montgomery square a*a*R^{-1} in [0, 2N) for 8-word fields: the full square
// (bn_sqr_wide), then eight reduction rows over it, its upper words entering
// one per row.  The same value (a^2 + m N) / R as fe_mul(a, a): m is fixed by
// a^2 mod R.  259 instructions and 36 + 64 products against 280 and 64 + 64.
template <class F>
__device__ __forceinline__ Fe<F> fe_sqr_inline(const Fe<F> &a) {
    u32 t[16];
    bn_sqr_wide(t, a.l);
    u32 u[8] = {t[0], t[1], t[2], t[3], t[4], t[5], t[6], t[7]}, v[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    bn_row_reduce<F>(u, v);
    bn_row_reduce_word<F>(v, u, t[8]);
    bn_row_reduce_word<F>(u, v, t[9]);
    bn_row_reduce_word<F>(v, u, t[10]);
    bn_row_reduce_word<F>(u, v, t[11]);
    bn_row_reduce_word<F>(v, u, t[12]);
    bn_row_reduce_word<F>(u, v, t[13]);
    bn_row_reduce_word<F>(v, u, t[14]);
    Fe<F> r;
    asm("add.cc.u32  %0, %8, %16;\n\taddc.cc.u32 %1, %9, %17;\n\taddc.cc.u32 %2, %10, %18;\n\t"
        "addc.cc.u32 %3, %11, %19;\n\taddc.cc.u32 %4, %12, %20;\n\taddc.cc.u32 %5, %13, %21;\n\t"
        "addc.cc.u32 %6, %14, %22;\n\taddc.u32    %7, %15, %23;"
        : "=r"(r.l[0]), "=r"(r.l[1]), "=r"(r.l[2]), "=r"(r.l[3]), "=r"(r.l[4]), "=r"(r.l[5]), "=r"(r.l[6]),
          "=r"(r.l[7])
        : "r"(u[0]), "r"(u[1]), "r"(u[2]), "r"(u[3]), "r"(u[4]), "r"(u[5]), "r"(u[6]), "r"(u[7]), "r"(v[1]),
          "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(t[15]));
    if constexpr (!F::LAZY) {
        const Fe<F> q = r;
        fe_reduce_once<F>(r, q.l);
    }
    return r;
}

// Montgomery product a*b*R^{-1} mod N in [0, 2N) for inputs in [0, 2N).
// Eight rows with the accumulators alternating; after the last (odd) row the
// value is u_0..7 + v_1..7 (v_0 is zero).  No final subtraction (lazy
// reduction).
template <class F>
__device__ __forceinline__ Fe<F> fe_mul_inline(const Fe<F> &a, const Fe<F> &b) {
    if constexpr (F::N == 12) {
        u32 u[12], v[12];
        bn_row_first12(u, v, a.l, b.l[0]);
        bn_row_reduce12<F>(u, v);
#pragma unroll
        for (int i = 1; i < 12; i += 2) {
            bn_row_next12(v, u, a.l, b.l[i]);
            bn_row_reduce12<F>(v, u);
            if (i + 1 < 12) {
                bn_row_next12(u, v, a.l, b.l[i + 1]);
                bn_row_reduce12<F>(u, v);
            }
        }
        Fe<F> r;
        bn_merge12(r.l, u, v);
        if constexpr (!F::LAZY) {
            const Fe<F> t = r;
            fe_reduce_once<F>(r, t.l);
        }
        return r;
    } else {
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
    if constexpr (!F::LAZY) {
        // canonical fields: inputs below N give a result below 2N
        const Fe<F> t = r;
        fe_reduce_once<F>(r, t.l);
    }
    return r;
    }
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

// Squares of 8-word values take the dedicated square (IMPELLER_SQR_AS_MUL
// selects the general product instead, for comparison builds).
template <class F>
__device__ __forceinline__ Fe<F> fe_sqr(const Fe<F> &a) {
#ifndef IMPELLER_SQR_AS_MUL
    if constexpr (F::N == 8) return fe_sqr_inline<F>(a);
    else
#endif
        return fe_mul<F>(a, a);
}

// One out-of-line copy of the product, for kernels that run only a few warps
// (the reduction tree, the final Horner and affine conversion): no other warp
// reuses their instruction cache, and an inlined point addition (about 4000
// instructions) streams through it, so a lone warp stalls on instruction
// fetch.  The point formulas below take the product as a policy.
template <class F>
__device__ __noinline__ Fe<F> fe_mul_call(Fe<F> a, Fe<F> b) {
    return fe_mul_inline<F>(a, b);
}

template <class F>
__device__ __noinline__ Fe<F> fe_sqr_call(Fe<F> a) {
    return fe_sqr<F>(a);
}

struct MulInline {
    template <class F>
    __device__ __forceinline__ static Fe<F> mul(const Fe<F> &a, const Fe<F> &b) { return fe_mul<F>(a, b); }
    template <class F>
    __device__ __forceinline__ static Fe<F> sqr(const Fe<F> &a) { return fe_sqr<F>(a); }
};
struct MulCall {
    template <class F>
    __device__ __forceinline__ static Fe<F> mul(const Fe<F> &a, const Fe<F> &b) { return fe_mul_call<F>(a, b); }
    template <class F>
    __device__ __forceinline__ static Fe<F> sqr(const Fe<F> &a) { return fe_sqr_call<F>(a); }
};

// Leave Montgomery form: a * R^{-1} mod N, canonical, for a in [0, 2N)
// (Montgomery reduction only; the sum stays at or below N before the final
// subtraction).
template <class F>
__device__ __forceinline__ Fe<F> fe_from_mont(const Fe<F> &a) {
    if constexpr (F::N == 12) {
        // a * 1 * R^{-1}: the product with the integer 1, then canonical
        Fe<F> one_int = fe_zero<F>();
        one_int.l[0] = 1;
        return fe_canon<F>(fe_mul_inline<F>(a, one_int));
    } else {
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
}

template <class F>
__device__ __forceinline__ Fe<F> fe_add(const Fe<F> &a, const Fe<F> &b) {
    if constexpr (F::N == 12) {
        u32 s[12];
        add12(s, a.l, b.l);  // a + b < 4N < 2^384
        Fe<F> r;
        if constexpr (F::LAZY) fe_reduce_2n<F>(r, s);
        else fe_reduce_once<F>(r, s);
        return r;
    } else {
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
    // a + b < 4N < 2^256 (lazy) or < 2N (canonical)
    if constexpr (F::LAZY) fe_reduce_2n<F>(r, s);
    else fe_reduce_once<F>(r, s);
    return r;
    }
}

template <class F>
__device__ __forceinline__ Fe<F> fe_sub(const Fe<F> &a, const Fe<F> &b) {
    if constexpr (F::N == 12) {
        u32 d[12];
        const u32 bw = sub12(d, a.l, b.l);
        Fe<F> r;
        constexpr Words<12> back = F::LAZY ? words(F::D) : words(F::M);
        add12_masked(r.l, d, back.v, bw);  // add 2N (N) back on borrow
        return r;
    } else {
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
    // add 2N (N for canonical fields) back when the subtraction borrowed
    constexpr u32 k0 = F::LAZY ? F::D0 : F::M0, k1 = F::LAZY ? F::D1 : F::M1, k2 = F::LAZY ? F::D2 : F::M2;
    constexpr u32 k3 = F::LAZY ? F::D3 : F::M3, k4 = F::LAZY ? F::D4 : F::M4, k5 = F::LAZY ? F::D5 : F::M5;
    constexpr u32 k6 = F::LAZY ? F::D6 : F::M6, k7 = F::LAZY ? F::D7 : F::M7;
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
          "r"(k0 & bw), "r"(k1 & bw), "r"(k2 & bw), "r"(k3 & bw), "r"(k4 & bw), "r"(k5 & bw), "r"(k6 & bw),
          "r"(k7 & bw));
    return r;
    }
}

template <class F>
__device__ __forceinline__ Fe<F> fe_neg(const Fe<F> &a) {
    return fe_sub<F>(fe_zero<F>(), a);
}

template <class F>
__device__ __forceinline__ Fe<F> fe_dbl(const Fe<F> &a) {
    return fe_add<F>(a, a);
}

// a^e for a plain exponent given as F::N little-endian limbs, 4-bit fixed window.
template <class F>
__device__ __noinline__ Fe<F> fe_pow(const Fe<F> &a, const u32 *e) {
    Fe<F> tab[16];
    tab[0] = fe_one<F>();
    tab[1] = a;
#pragma unroll 1
    for (int i = 2; i < 16; i++) tab[i] = fe_mul<F>(tab[i - 1], a);
    Fe<F> acc = fe_one<F>();
#pragma unroll 1
    for (int nib = 8 * F::N - 1; nib >= 0; nib--) {
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
    constexpr Words<F::N> m = words(F::M);
    u32 e[F::N];
    u32 borrow = 2;
#pragma unroll
    for (int i = 0; i < F::N; i++) {
        e[i] = m.v[i] - borrow;
        borrow = m.v[i] < borrow ? 1u : 0u;
    }
    return fe_pow<F>(a, e);
}

// Single-thread-latency inversion for the few conversions to affine form at
// the end of an MSM: binary extended Euclid on the integer representative
// (Montgomery form a = A*R) gives a^{-1} = A^{-1} R^{-1}; one Montgomery
// product with R^3 mod N turns it into A^{-1} R.  Variable time (the inputs
// are public).  Inverse of zero is zero.  The loop is bounded: every step
// shrinks u + v by at least one bit.
template <int N>
__device__ __forceinline__ bool un_is_one(const u32 *x) {
    u32 o = x[0] ^ 1u;
#pragma unroll
    for (int i = 1; i < N; i++) o |= x[i];
    return o == 0;
}

template <int N>
__device__ __forceinline__ bool un_is_zero(const u32 *x) {
    u32 o = 0;
#pragma unroll
    for (int i = 0; i < N; i++) o |= x[i];
    return o == 0;
}

template <int N>
__device__ __forceinline__ void un_shr1(u32 *x, u32 top) {
#pragma unroll
    for (int i = 0; i < N - 1; i++) x[i] = __funnelshift_r(x[i], x[i + 1], 1);
    x[N - 1] = (x[N - 1] >> 1) | (top << 31);
}

template <int N>
__device__ __forceinline__ bool un_geq(const u32 *a, const u32 *b) {
    for (int i = N - 1; i >= 0; i--)
        if (a[i] != b[i]) return a[i] > b[i];
    return true;
}

// a -= b (no borrow out: callers subtract the smaller value)
template <int N>
__device__ __forceinline__ void un_sub(u32 *a, const u32 *b) {
    if constexpr (N == 12) {
        u32 d[12];
        sub12(d, a, b);
#pragma unroll
        for (int i = 0; i < 12; i++) a[i] = d[i];
    } else {
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
}

// x = x / 2 mod N for x < 2N (N odd): if x is odd, (x + N) / 2 < 3N / 2.
// x * 2^-k mod N for 1 <= k <= 32 (x in [0, 2N), or [0, N) on fields
// without lazy reduction, and the result in the same range): q = -x N^-1
// mod 2^k makes x + q N divisible by 2^k.
template <class F>
__device__ __forceinline__ void fe_div2k(u32 *x, u32 k) {
    constexpr int N = F::N;
    constexpr Words<N> m = words(F::M);
    const u32 q = (x[0] * F::INV) & (k == 32 ? 0xffffffffu : ((1u << k) - 1u));
    u32 t[N + 1];
    u64 c = 0;
#pragma unroll
    for (int i = 0; i < N; i++) {
        const u64 s = (u64)q * m.v[i] + x[i] + c;
        t[i] = (u32)s;
        c = s >> 32;
    }
    t[N] = (u32)c;
    if (k == 32) {
#pragma unroll
        for (int i = 0; i < N; i++) x[i] = t[i + 1];
    } else {
#pragma unroll
        for (int i = 0; i < N; i++) x[i] = __funnelshift_r(t[i], t[i + 1], k);
    }
}

// Strip every trailing zero bit of w (nonzero), dividing x by 2 for each.
template <class F>
__device__ __forceinline__ void un_make_odd(u32 *w, u32 *x) {
    constexpr int N = F::N;
    while (w[0] == 0) {
#pragma unroll
        for (int i = 0; i < N - 1; i++) w[i] = w[i + 1];
        w[N - 1] = 0;
        fe_div2k<F>(x, 32);
    }
    const u32 k = __ffs(w[0]) - 1;
    if (k) {
#pragma unroll
        for (int i = 0; i < N - 1; i++) w[i] = __funnelshift_r(w[i], w[i + 1], k);
        w[N - 1] >>= k;
        fe_div2k<F>(x, k);
    }
}

// Invariants: x1 a = u and x2 a = v (mod N) up to the common power of two the
// halvings divide out of both sides; u and v stay odd between steps, so every
// step is one subtraction followed by all the halvings it makes possible.
// The step bound keeps a non-canonical or non-invertible input from
// looping: it yields zero.
template <class F>
__device__ __noinline__ Fe<F> fe_inv_binary(const Fe<F> &a_in, const Fe<F> &r3) {
    const Fe<F> a = fe_canon<F>(a_in);
    if (fe_is_zero_canonical(a)) return a;
    constexpr int N = F::N;
    constexpr Words<N> m = words(F::M);
    u32 u[N], v[N];
    Fe<F> x1 = fe_zero<F>(), x2 = fe_zero<F>();
    x1.l[0] = 1;
#pragma unroll
    for (int i = 0; i < N; i++) {
        u[i] = a.l[i];
        v[i] = m.v[i];
    }
    un_make_odd<F>(u, x1.l);  // v = N is odd
    for (int step = 0; step < 4096; step++) {
        if (un_is_one<N>(u)) return fe_mul<F>(x1, r3);
        if (un_is_one<N>(v)) return fe_mul<F>(x2, r3);
        if (un_geq<N>(u, v)) {
            un_sub<N>(u, v);
            if (un_is_zero<N>(u)) break;  // u == v > 1: no inverse
            x1 = fe_sub<F>(x1, x2);
            un_make_odd<F>(u, x1.l);
        } else {
            un_sub<N>(v, u);
            x2 = fe_sub<F>(x2, x1);
            un_make_odd<F>(v, x2.l);
        }
    }
    return fe_zero<F>();
}

// The same inversion by Bernstein-Yang divsteps (safegcd.cuh): batches of 30
// divsteps on the low words, one full-width update per batch; 3-4x fewer
// dependent instructions than the binary method for 254- and 381-bit moduli.
// One Montgomery product with R^3 turns A^-1 R^-1 into A^-1 R as above.
template <class F>
__device__ __noinline__ Fe<F> fe_inv_divsteps(const Fe<F> &a_in, const Fe<F> &r3) {
    const Fe<F> a = fe_canon<F>(a_in);
    constexpr Words<F::N> m = words(F::M);
    Fe<F> r;
    sg::inverse<F::N>(a.l, m.v, r.l);
    return fe_mul<F>(r, r3);
}

// 16-byte vector loads and stores (element addresses are 16-byte aligned).
template <class F>
__device__ __forceinline__ Fe<F> fe_load(const u32 *p) {
    Fe<F> r;
    const uint4 *q = reinterpret_cast<const uint4 *>(p);
#pragma unroll
    for (int k = 0; k < F::N / 4; k++) {
        const uint4 v = q[k];
        r.l[4 * k] = v.x;
        r.l[4 * k + 1] = v.y;
        r.l[4 * k + 2] = v.z;
        r.l[4 * k + 3] = v.w;
    }
    return r;
}

template <class F>
__device__ __forceinline__ void fe_store(u32 *p, const Fe<F> &a) {
    uint4 *q = reinterpret_cast<uint4 *>(p);
#pragma unroll
    for (int k = 0; k < F::N / 4; k++) q[k] = make_uint4(a.l[4 * k], a.l[4 * k + 1], a.l[4 * k + 2], a.l[4 * k + 3]);
}

// ----------------------------------------------------------- G1 (XYZZ)
//
// Templates over the base field F: BN254 G1 (F = FqP, 16-word affine, 32-word
// XYZZ) and BLS12-381 G1 (F = BlsFqP, 24 / 48 words).  Both curves are
// y^2 = x^3 + b with a = 0, the case the formulas below are written for.

template <class F>
struct AffineT {
    Fe<F> x, y;
};

template <class F>
struct XyzzT {
    Fe<F> x, y, zz, zzz;
};

typedef AffineT<FqP> Affine;
typedef XyzzT<FqP> Xyzz;

// Affine points come from memory in canonical form; negation keeps 0 at 0.
template <class F>
__device__ __forceinline__ bool affine_is_identity(const AffineT<F> &a) { return fe_is_zero_canonical(a.y); }

template <class F = FqP>
__device__ __forceinline__ XyzzT<F> xyzz_identity() {
    XyzzT<F> r;
    r.x = fe_zero<F>();
    r.y = fe_zero<F>();
    r.zz = fe_zero<F>();
    r.zzz = fe_zero<F>();
    return r;
}

template <class F>
__device__ __forceinline__ bool xyzz_is_identity(const XyzzT<F> &p) { return fe_is_zero(p.zz); }

template <class F>
__device__ __forceinline__ XyzzT<F> xyzz_from_affine(const AffineT<F> &a) {
    if (affine_is_identity(a)) return xyzz_identity<F>();
    XyzzT<F> r;
    r.x = a.x;
    r.y = a.y;
    r.zz = fe_one<F>();
    r.zzz = r.zz;
    return r;
}

template <class F>
__device__ __forceinline__ AffineT<F> affine_neg(const AffineT<F> &a) {
    AffineT<F> r;
    r.x = a.x;
    r.y = fe_neg<F>(a.y);
    return r;
}

template <class F>
__device__ __forceinline__ XyzzT<F> xyzz_neg(const XyzzT<F> &p) {
    XyzzT<F> r = p;
    r.y = fe_neg<F>(p.y);
    return r;
}

// mdbl-2008-s-1: 2*a for an affine, non-identity a.
template <class F>
__device__ __forceinline__ XyzzT<F> affine_dbl(const AffineT<F> &a) {
    Fe<F> u = fe_dbl(a.y);
    Fe<F> v = fe_sqr(u);
    Fe<F> w = fe_mul(u, v);
    Fe<F> s = fe_mul(a.x, v);
    Fe<F> x2 = fe_sqr(a.x);
    Fe<F> m = fe_add(fe_dbl(x2), x2);
    XyzzT<F> r;
    r.x = fe_sub(fe_sub(fe_sqr(m), s), s);
    r.y = fe_sub(fe_mul(m, fe_sub(s, r.x)), fe_mul(w, a.y));
    r.zz = v;
    r.zzz = w;
    return r;
}

// dbl-2008-s-1 with a = 0.
template <class F, class MUL = MulInline>
__device__ __forceinline__ XyzzT<F> xyzz_dbl(const XyzzT<F> &p) {
    if (xyzz_is_identity(p)) return p;
    Fe<F> u = fe_dbl(p.y);
    Fe<F> v = MUL::sqr(u);
    Fe<F> w = MUL::mul(u, v);
    Fe<F> s = MUL::mul(p.x, v);
    Fe<F> x2 = MUL::sqr(p.x);
    Fe<F> m = fe_add(fe_dbl(x2), x2);
    XyzzT<F> r;
    r.x = fe_sub(fe_sub(MUL::sqr(m), s), s);
    r.y = fe_sub(MUL::mul(m, fe_sub(s, r.x)), MUL::mul(w, p.y));
    r.zz = MUL::mul(v, p.zz);
    r.zzz = MUL::mul(w, p.zzz);
    return r;
}

// Jacobian coordinates (x = X / Z^2, y = Y / Z^3) for chains of doublings:
// dbl-2009-l with a = 0 costs 2 products and 5 squares against XYZZ's 6 and
// 3 (812 against 1140 32x32-bit partial products on BN254).  Z == 0 is the
// identity and stays so.
template <class F>
struct JacT {
    Fe<F> x, y, z;
};

template <class F, class MUL = MulInline>
__device__ __forceinline__ JacT<F> jac_dbl(const JacT<F> &p) {
    const Fe<F> a = MUL::sqr(p.x);
    const Fe<F> b = MUL::sqr(p.y);
    const Fe<F> c = MUL::sqr(b);
    const Fe<F> t = fe_sub(fe_sub(MUL::sqr(fe_add(p.x, b)), a), c);
    const Fe<F> d = fe_dbl(t);
    const Fe<F> e = fe_add(fe_dbl(a), a);
    JacT<F> r;
    r.x = fe_sub(MUL::sqr(e), fe_dbl(d));
    const Fe<F> c8 = fe_dbl(fe_dbl(fe_dbl(c)));
    r.y = fe_sub(MUL::mul(e, fe_sub(d, r.x)), c8);
    r.z = fe_dbl(MUL::mul(p.y, p.z));
    return r;
}

// 2^k p.  From three doublings on, through Jacobian coordinates: with
// ZZ = z^2, ZZZ = z^3, (X ZZ^2, Y ZZZ^2, ZZZ) is the same point in Jacobian
// form (Z = z ZZ), and (X, Y, Z^2, Z^3) takes it back (6 products in all).
template <class F, class MUL = MulInline>
__device__ __forceinline__ XyzzT<F> xyzz_dbl_n(const XyzzT<F> &p, u32 k) {
    if (k < 3 || xyzz_is_identity(p)) {
        XyzzT<F> r = p;
        for (u32 i = 0; i < k; i++) r = xyzz_dbl<F, MUL>(r);
        return r;
    }
    JacT<F> j;
    j.x = MUL::mul(p.x, MUL::sqr(p.zz));
    j.y = MUL::mul(p.y, MUL::sqr(p.zzz));
    j.z = p.zzz;
    for (u32 i = 0; i < k; i++) j = jac_dbl<F, MUL>(j);
    XyzzT<F> r;
    r.x = j.x;
    r.y = j.y;
    r.zz = MUL::sqr(j.z);
    r.zzz = MUL::mul(j.z, r.zz);
    return r;
}

// madd-2008-s: p + q, q affine.  Handles every special case.
template <class F>
__device__ __forceinline__ XyzzT<F> xyzz_add_affine(const XyzzT<F> &p, const AffineT<F> &q) {
    if (affine_is_identity(q)) return p;
    if (xyzz_is_identity(p)) return xyzz_from_affine(q);
    Fe<F> u2 = fe_mul(q.x, p.zz);
    Fe<F> s2 = fe_mul(q.y, p.zzz);
    Fe<F> P = fe_sub(u2, p.x);
    Fe<F> R = fe_sub(s2, p.y);
    if (fe_is_zero(P)) {
        if (fe_is_zero(R)) return affine_dbl(q);
        return xyzz_identity<F>();
    }
    Fe<F> pp = fe_sqr(P);
    Fe<F> ppp = fe_mul(P, pp);
    Fe<F> Q = fe_mul(p.x, pp);
    XyzzT<F> r;
    r.zz = fe_mul(p.zz, pp);
    r.zzz = fe_mul(p.zzz, ppp);
    Fe<F> t = fe_mul(p.y, ppp);
    r.x = fe_sub(fe_sub(fe_sub(fe_sqr(R), ppp), Q), Q);
    r.y = fe_sub(fe_mul(R, fe_sub(Q, r.x)), t);
    return r;
}

// add-2008-s: p + q.  Handles every special case.
template <class F, class MUL = MulInline>
__device__ __forceinline__ XyzzT<F> xyzz_add(const XyzzT<F> &p, const XyzzT<F> &q) {
    if (xyzz_is_identity(p)) return q;
    if (xyzz_is_identity(q)) return p;
    Fe<F> u1 = MUL::mul(p.x, q.zz);
    Fe<F> u2 = MUL::mul(q.x, p.zz);
    Fe<F> s1 = MUL::mul(p.y, q.zzz);
    Fe<F> s2 = MUL::mul(q.y, p.zzz);
    Fe<F> P = fe_sub(u2, u1);
    Fe<F> R = fe_sub(s2, s1);
    if (fe_is_zero(P)) {
        if (fe_is_zero(R)) return xyzz_dbl<F, MUL>(p);
        return xyzz_identity<F>();
    }
    Fe<F> pp = MUL::sqr(P);
    Fe<F> ppp = MUL::mul(P, pp);
    Fe<F> Q = MUL::mul(u1, pp);
    XyzzT<F> r;
    r.zz = MUL::mul(MUL::mul(p.zz, q.zz), pp);
    r.zzz = MUL::mul(MUL::mul(p.zzz, q.zzz), ppp);
    Fe<F> t = MUL::mul(s1, ppp);
    r.x = fe_sub(fe_sub(fe_sub(MUL::sqr(R), ppp), Q), Q);
    r.y = fe_sub(MUL::mul(R, fe_sub(Q, r.x)), t);
    return r;
}

__device__ __forceinline__ Fq fq_r3() { return fe_rcube<FqP>(); }

// Canonical affine form; identity -> (0, 0).  Latency-optimised (divstep
// inversion): used once per MSM result.
template <class F, class MUL = MulInline>
__device__ __forceinline__ AffineT<F> xyzz_to_affine_fast(const XyzzT<F> &p) {
    AffineT<F> r;
    if (xyzz_is_identity(p)) {
        r.x = fe_zero<F>();
        r.y = fe_zero<F>();
        return r;
    }
    Fe<F> a = fe_inv_divsteps<F>(p.zzz, fe_rcube<F>());
    Fe<F> zza = MUL::mul(p.zz, a);
    Fe<F> b = MUL::sqr(zza);
    r.x = fe_canon(MUL::mul(p.x, b));
    r.y = fe_canon(MUL::mul(p.y, a));
    return r;
}

// Canonical affine form; identity -> (0, 0).
template <class F>
__device__ __forceinline__ AffineT<F> xyzz_to_affine(const XyzzT<F> &p) {
    AffineT<F> r;
    if (xyzz_is_identity(p)) {
        r.x = fe_zero<F>();
        r.y = fe_zero<F>();
        return r;
    }
    Fe<F> a = fe_inv(p.zzz);
    Fe<F> b = fe_sqr(fe_mul(p.zz, a));
    r.x = fe_canon(fe_mul(p.x, b));
    r.y = fe_canon(fe_mul(p.y, a));
    return r;
}

template <class F = FqP>
__device__ __forceinline__ AffineT<F> affine_load(const u32 *p) {
    AffineT<F> a;
    a.x = fe_load<F>(p);
    a.y = fe_load<F>(p + F::N);
    return a;
}

template <class F>
__device__ __forceinline__ void affine_store(u32 *p, const AffineT<F> &a) {
    fe_store(p, a.x);
    fe_store(p + F::N, a.y);
}

template <class F = FqP>
__device__ __forceinline__ XyzzT<F> xyzz_load(const u32 *p) {
    XyzzT<F> r;
    r.x = fe_load<F>(p);
    r.y = fe_load<F>(p + F::N);
    r.zz = fe_load<F>(p + 2 * F::N);
    r.zzz = fe_load<F>(p + 3 * F::N);
    return r;
}

template <class F>
__device__ __forceinline__ void xyzz_store(u32 *p, const XyzzT<F> &a) {
    fe_store(p, a.x);
    fe_store(p + F::N, a.y);
    fe_store(p + 2 * F::N, a.zz);
    fe_store(p + 3 * F::N, a.zzz);
}

template <class F>
__device__ __forceinline__ XyzzT<F> xyzz_shfl_down(const XyzzT<F> &p, u32 delta, u32 mask = 0xffffffffu) {
    XyzzT<F> r;
#pragma unroll
    for (int i = 0; i < F::N; i++) {
        r.x.l[i] = __shfl_down_sync(mask, p.x.l[i], delta);
        r.y.l[i] = __shfl_down_sync(mask, p.y.l[i], delta);
        r.zz.l[i] = __shfl_down_sync(mask, p.zz.l[i], delta);
        r.zzz.l[i] = __shfl_down_sync(mask, p.zzz.l[i], delta);
    }
    return r;
}

template <class F>
__device__ __forceinline__ XyzzT<F> xyzz_shfl_xor(const XyzzT<F> &p, u32 lane_mask) {
    XyzzT<F> r;
#pragma unroll
    for (int i = 0; i < F::N; i++) {
        r.x.l[i] = __shfl_xor_sync(0xffffffffu, p.x.l[i], lane_mask);
        r.y.l[i] = __shfl_xor_sync(0xffffffffu, p.y.l[i], lane_mask);
        r.zz.l[i] = __shfl_xor_sync(0xffffffffu, p.zz.l[i], lane_mask);
        r.zzz.l[i] = __shfl_xor_sync(0xffffffffu, p.zzz.l[i], lane_mask);
    }
    return r;
}

// k * p for a small plain scalar k, left-to-right double-and-add.
template <class F>
__device__ __forceinline__ XyzzT<F> xyzz_mul_u32(const XyzzT<F> &p, u32 k) {
    XyzzT<F> acc = xyzz_identity<F>();
    if (k == 0) return acc;
    int top = 31 - __clz(k);
#pragma unroll 1
    for (int i = top; i >= 0; i--) {
        acc = xyzz_dbl(acc);
        if ((k >> i) & 1u) acc = xyzz_add(acc, p);
    }
    return acc;
}

}  // namespace ec
