// 12-limb (384-bit) field arithmetic for the BLS12-381 base field: the same
// operations as the 8-limb code beside it in bn254.cuh, with the carry
// chains and the two-accumulator Montgomery rows spelled out for 12 limbs.
// The asm bodies are generated (one line per limb pair); every function
// takes plain word arrays so bn254.cuh's templates can call it.
#pragma once

namespace ec {

// r = a - b (12 words); returns 0xffffffff on borrow, else 0.
__device__ __forceinline__ u32 sub12(u32 (&r)[12], const u32 *a, const u32 *b) {
    u32 bw;
    asm(
        "sub.cc.u32 %0, %13, %25;\n\t"
        "subc.cc.u32 %1, %14, %26;\n\t"
        "subc.cc.u32 %2, %15, %27;\n\t"
        "subc.cc.u32 %3, %16, %28;\n\t"
        "subc.cc.u32 %4, %17, %29;\n\t"
        "subc.cc.u32 %5, %18, %30;\n\t"
        "subc.cc.u32 %6, %19, %31;\n\t"
        "subc.cc.u32 %7, %20, %32;\n\t"
        "subc.cc.u32 %8, %21, %33;\n\t"
        "subc.cc.u32 %9, %22, %34;\n\t"
        "subc.cc.u32 %10, %23, %35;\n\t"
        "subc.cc.u32 %11, %24, %36;\n\t"
        "subc.u32 %12, 0, 0;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11]), "=r"(bw)
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]), "r"(a[8]), "r"(a[9]), "r"(a[10]), "r"(a[11]),
          "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]));
    return bw;
}

// r = a + b (12 words), no carry out (callers keep a + b below 2^384).
__device__ __forceinline__ void add12(u32 (&r)[12], const u32 *a, const u32 *b) {
    asm(
        "add.cc.u32 %0, %12, %24;\n\t"
        "addc.cc.u32 %1, %13, %25;\n\t"
        "addc.cc.u32 %2, %14, %26;\n\t"
        "addc.cc.u32 %3, %15, %27;\n\t"
        "addc.cc.u32 %4, %16, %28;\n\t"
        "addc.cc.u32 %5, %17, %29;\n\t"
        "addc.cc.u32 %6, %18, %30;\n\t"
        "addc.cc.u32 %7, %19, %31;\n\t"
        "addc.cc.u32 %8, %20, %32;\n\t"
        "addc.cc.u32 %9, %21, %33;\n\t"
        "addc.cc.u32 %10, %22, %34;\n\t"
        "addc.u32 %11, %23, %35;\n\t"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]), "r"(a[8]), "r"(a[9]), "r"(a[10]), "r"(a[11]),
          "r"(b[0]), "r"(b[1]), "r"(b[2]), "r"(b[3]), "r"(b[4]), "r"(b[5]), "r"(b[6]), "r"(b[7]), "r"(b[8]), "r"(b[9]), "r"(b[10]), "r"(b[11]));
}

// r = a + (mask & b) (12 words).
__device__ __forceinline__ void add12_masked(u32 (&r)[12], const u32 *a, const u32 *b, u32 mask) {
    u32 t[12];
#pragma unroll
    for (int i = 0; i < 12; i++) t[i] = b[i] & mask;
    add12(r, a, t);
}

// Rows of the two-accumulator Montgomery product (see bn254.cuh), 12 limbs.
__device__ __forceinline__ void bn_row_first12(u32 (&x)[12], u32 (&y)[12], const u32 (&a)[12], u32 w) {
    asm(
        "mul.lo.u32 %0, %24, %36;\n\tmul.hi.u32 %1, %24, %36;\n\t"
        "mul.lo.u32 %2, %26, %36;\n\tmul.hi.u32 %3, %26, %36;\n\t"
        "mul.lo.u32 %4, %28, %36;\n\tmul.hi.u32 %5, %28, %36;\n\t"
        "mul.lo.u32 %6, %30, %36;\n\tmul.hi.u32 %7, %30, %36;\n\t"
        "mul.lo.u32 %8, %32, %36;\n\tmul.hi.u32 %9, %32, %36;\n\t"
        "mul.lo.u32 %10, %34, %36;\n\tmul.hi.u32 %11, %34, %36;\n\t"
        "mul.lo.u32 %12, %25, %36;\n\tmul.hi.u32 %13, %25, %36;\n\t"
        "mul.lo.u32 %14, %27, %36;\n\tmul.hi.u32 %15, %27, %36;\n\t"
        "mul.lo.u32 %16, %29, %36;\n\tmul.hi.u32 %17, %29, %36;\n\t"
        "mul.lo.u32 %18, %31, %36;\n\tmul.hi.u32 %19, %31, %36;\n\t"
        "mul.lo.u32 %20, %33, %36;\n\tmul.hi.u32 %21, %33, %36;\n\t"
        "mul.lo.u32 %22, %35, %36;\n\tmul.hi.u32 %23, %35, %36;\n\t"
        : "=r"(x[0]), "=r"(x[1]), "=r"(x[2]), "=r"(x[3]), "=r"(x[4]), "=r"(x[5]), "=r"(x[6]), "=r"(x[7]), "=r"(x[8]), "=r"(x[9]), "=r"(x[10]), "=r"(x[11]),
          "=r"(y[0]), "=r"(y[1]), "=r"(y[2]), "=r"(y[3]), "=r"(y[4]), "=r"(y[5]), "=r"(y[6]), "=r"(y[7]), "=r"(y[8]), "=r"(y[9]), "=r"(y[10]), "=r"(y[11])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]), "r"(a[8]), "r"(a[9]), "r"(a[10]), "r"(a[11]), "r"(w));
}

__device__ __forceinline__ void bn_row_next12(u32 (&x)[12], u32 (&y)[12], const u32 (&a)[12], u32 w) {
    asm(
        "add.cc.u32 %0, %0, %13;\n\t"
        "madc.lo.cc.u32 %12, %25, %36, %14;\n\tmadc.hi.cc.u32 %13, %25, %36, %15;\n\t"
        "madc.lo.cc.u32 %14, %27, %36, %16;\n\tmadc.hi.cc.u32 %15, %27, %36, %17;\n\t"
        "madc.lo.cc.u32 %16, %29, %36, %18;\n\tmadc.hi.cc.u32 %17, %29, %36, %19;\n\t"
        "madc.lo.cc.u32 %18, %31, %36, %20;\n\tmadc.hi.cc.u32 %19, %31, %36, %21;\n\t"
        "madc.lo.cc.u32 %20, %33, %36, %22;\n\tmadc.hi.cc.u32 %21, %33, %36, %23;\n\t"
        "madc.lo.cc.u32 %22, %35, %36, 0;\n\tmadc.hi.u32 %23, %35, %36, 0;\n\t"
        "mad.lo.cc.u32 %0, %24, %36, %0;\n\tmadc.hi.cc.u32 %1, %24, %36, %1;\n\t"
        "madc.lo.cc.u32 %2, %26, %36, %2;\n\tmadc.hi.cc.u32 %3, %26, %36, %3;\n\t"
        "madc.lo.cc.u32 %4, %28, %36, %4;\n\tmadc.hi.cc.u32 %5, %28, %36, %5;\n\t"
        "madc.lo.cc.u32 %6, %30, %36, %6;\n\tmadc.hi.cc.u32 %7, %30, %36, %7;\n\t"
        "madc.lo.cc.u32 %8, %32, %36, %8;\n\tmadc.hi.cc.u32 %9, %32, %36, %9;\n\t"
        "madc.lo.cc.u32 %10, %34, %36, %10;\n\tmadc.hi.cc.u32 %11, %34, %36, %11;\n\t"
        "addc.u32 %23, %23, 0;"
        : "+r"(x[0]), "+r"(x[1]), "+r"(x[2]), "+r"(x[3]), "+r"(x[4]), "+r"(x[5]), "+r"(x[6]), "+r"(x[7]), "+r"(x[8]), "+r"(x[9]), "+r"(x[10]), "+r"(x[11]),
          "+r"(y[0]), "+r"(y[1]), "+r"(y[2]), "+r"(y[3]), "+r"(y[4]), "+r"(y[5]), "+r"(y[6]), "+r"(y[7]), "+r"(y[8]), "+r"(y[9]), "+r"(y[10]), "+r"(y[11])
        : "r"(a[0]), "r"(a[1]), "r"(a[2]), "r"(a[3]), "r"(a[4]), "r"(a[5]), "r"(a[6]), "r"(a[7]), "r"(a[8]), "r"(a[9]), "r"(a[10]), "r"(a[11]), "r"(w));
}

template <class F>
__device__ __forceinline__ void bn_row_reduce12(u32 (&x)[12], u32 (&y)[12]) {
    constexpr Words<12> M = words(F::M);
    asm(
        "{\n\t.reg .u32 m;\n\t"
        "mul.lo.u32 m, %0, %36;\n\t"
        "mad.lo.cc.u32 %12, m, %25, %12;\n\tmadc.hi.cc.u32 %13, m, %25, %13;\n\t"
        "madc.lo.cc.u32 %14, m, %27, %14;\n\tmadc.hi.cc.u32 %15, m, %27, %15;\n\t"
        "madc.lo.cc.u32 %16, m, %29, %16;\n\tmadc.hi.cc.u32 %17, m, %29, %17;\n\t"
        "madc.lo.cc.u32 %18, m, %31, %18;\n\tmadc.hi.cc.u32 %19, m, %31, %19;\n\t"
        "madc.lo.cc.u32 %20, m, %33, %20;\n\tmadc.hi.cc.u32 %21, m, %33, %21;\n\t"
        "madc.lo.cc.u32 %22, m, %35, %22;\n\tmadc.hi.u32 %23, m, %35, %23;\n\t"
        "mad.lo.cc.u32 %0, m, %24, %0;\n\tmadc.hi.cc.u32 %1, m, %24, %1;\n\t"
        "madc.lo.cc.u32 %2, m, %26, %2;\n\tmadc.hi.cc.u32 %3, m, %26, %3;\n\t"
        "madc.lo.cc.u32 %4, m, %28, %4;\n\tmadc.hi.cc.u32 %5, m, %28, %5;\n\t"
        "madc.lo.cc.u32 %6, m, %30, %6;\n\tmadc.hi.cc.u32 %7, m, %30, %7;\n\t"
        "madc.lo.cc.u32 %8, m, %32, %8;\n\tmadc.hi.cc.u32 %9, m, %32, %9;\n\t"
        "madc.lo.cc.u32 %10, m, %34, %10;\n\tmadc.hi.cc.u32 %11, m, %34, %11;\n\t"
        "addc.u32 %23, %23, 0;\n\t}"
        : "+r"(x[0]), "+r"(x[1]), "+r"(x[2]), "+r"(x[3]), "+r"(x[4]), "+r"(x[5]), "+r"(x[6]), "+r"(x[7]), "+r"(x[8]), "+r"(x[9]), "+r"(x[10]), "+r"(x[11]),
          "+r"(y[0]), "+r"(y[1]), "+r"(y[2]), "+r"(y[3]), "+r"(y[4]), "+r"(y[5]), "+r"(y[6]), "+r"(y[7]), "+r"(y[8]), "+r"(y[9]), "+r"(y[10]), "+r"(y[11])
        : "n"(M.v[0]), "n"(M.v[1]), "n"(M.v[2]), "n"(M.v[3]), "n"(M.v[4]), "n"(M.v[5]), "n"(M.v[6]), "n"(M.v[7]), "n"(M.v[8]), "n"(M.v[9]), "n"(M.v[10]), "n"(M.v[11]),
          "n"(F::INV));
}

// After the last row: value = u_0..11 + v_1..11 (v_0 is zero).
__device__ __forceinline__ void bn_merge12(u32 (&r)[12], const u32 (&u)[12], const u32 (&v)[12]) {
    asm(
        "add.cc.u32 %0, %12, %24;\n\t"
        "addc.cc.u32 %1, %13, %25;\n\t"
        "addc.cc.u32 %2, %14, %26;\n\t"
        "addc.cc.u32 %3, %15, %27;\n\t"
        "addc.cc.u32 %4, %16, %28;\n\t"
        "addc.cc.u32 %5, %17, %29;\n\t"
        "addc.cc.u32 %6, %18, %30;\n\t"
        "addc.cc.u32 %7, %19, %31;\n\t"
        "addc.cc.u32 %8, %20, %32;\n\t"
        "addc.cc.u32 %9, %21, %33;\n\t"
        "addc.cc.u32 %10, %22, %34;\n\t"
        "addc.u32 %11, %23, 0;"
        : "=r"(r[0]), "=r"(r[1]), "=r"(r[2]), "=r"(r[3]), "=r"(r[4]), "=r"(r[5]), "=r"(r[6]), "=r"(r[7]), "=r"(r[8]), "=r"(r[9]), "=r"(r[10]), "=r"(r[11])
        : "r"(u[0]), "r"(u[1]), "r"(u[2]), "r"(u[3]), "r"(u[4]), "r"(u[5]), "r"(u[6]), "r"(u[7]), "r"(u[8]), "r"(u[9]), "r"(u[10]), "r"(u[11]),
          "r"(v[1]), "r"(v[2]), "r"(v[3]), "r"(v[4]), "r"(v[5]), "r"(v[6]), "r"(v[7]), "r"(v[8]), "r"(v[9]), "r"(v[10]), "r"(v[11]));
}

}  // namespace ec

