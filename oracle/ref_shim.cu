// Host-only harness over the REFERENCE's own BN254 arithmetic.
//
// TEST INFRASTRUCTURE ONLY (oracle pinning).  Built by oracle/Makefile into
// oracle/_ref/libref_bn254.so straight from the reference's header sources,
// which stay where they are and are not copied:
//   core/src/common/mont/src/field.cuh         mont::Element host path
//                                              (host_arith::montgomery_multiplication)
//   core/src/common/mont/src/bn254_fq.cuh, bn254_fr.cuh   parameters
//   core/src/common/curve/src/curve_xyzz.cuh   PointXYZZ / PointAffine
//   core/src/common/curve/src/bn254.cuh        bn254::{Point, PointAffine, Field}
//   core/src/common/curve/src/bls12381.cuh     bls12381::{Point, PointAffine, Field}
//   core/src/common/mont/src/bls12381_fq.cuh, bls12381_fr.cuh   parameters
// The functions below only marshal u32 arrays (the C ABI layout) into those
// types and call their host operators, so the C oracle can be compared with
// the reference's own arithmetic on the same inputs.
#include "bn254.cuh"
#include "bls12381.cuh"

#include <cstdint>

using bn254::Point;
using bn254::PointAffine;
using FqE = bn254_fq::Element;
using FrE = bn254_fr::Element;
using Num = mont::Number<8>;

namespace {

template <class E>
int field_op(int op, const uint32_t *a, const uint32_t *b, uint32_t *out, uint64_t count) {
    constexpr uint64_t W = E::LIMBS;
    using N = mont::Number<E::LIMBS>;
    for (uint64_t i = 0; i < count; i++) {
        const uint32_t *pa = a + W * i;
        const uint32_t *pb = b ? b + W * i : nullptr;
        E x = E::load(pa);
        E r;
        switch (op) {
        case 0: r = x + E::load(pb); break;
        case 1: r = x - E::load(pb); break;
        case 2: r = x * E::load(pb); break;
        case 3: r = x.square(); break;
        case 4: r = x.neg(); break;
        case 5: r = E::from_number(N::load(pa)); break;
        case 6: {
            N n = x.to_number();
            n.store(out + W * i);
            continue;
        }
        case 7: r = x.invert(); break;
        case 8: r = x.pow(N::load(pb)); break;
        default: return -2;
        }
        r.store(out + W * i);
    }
    return 0;
}

template <class Pt, class Aff, class Fr>
int msm_naive(const uint32_t *points, const uint32_t *scalars, uint64_t n, uint32_t *out) {
    Pt total = Pt::identity();
    for (uint64_t i = 0; i < n; i++) {
        Aff p = Aff::load(points + Aff::N_WORDS * i);
        auto k = Fr::load(scalars + 8 * i).to_number();
        Pt acc = Pt::identity();
        for (int bit = 255; bit >= 0; bit--) {
            acc = acc.self_add();
            if ((k.limbs[bit / 32] >> (bit % 32)) & 1) acc = acc + p;
        }
        total = total + acc;
    }
    Aff r = total.is_identity() ? Aff::identity() : total.to_affine();
    r.store(out);
    return 0;
}

template <class Pt, class Aff>
int point_add(const uint32_t *p, const uint32_t *q, uint32_t *out, uint64_t count) {
    for (uint64_t i = 0; i < count; i++) {
        Aff a = Aff::load(p + Aff::N_WORDS * i);
        Aff b = Aff::load(q + Aff::N_WORDS * i);
        Pt s = a.to_point() + b;
        Aff r = s.is_identity() ? Aff::identity() : s.to_affine();
        r.store(out + Aff::N_WORDS * i);
    }
    return 0;
}

template <class Pt, class Aff>
int point_dbl(const uint32_t *p, uint32_t *out, uint64_t count) {
    for (uint64_t i = 0; i < count; i++) {
        Aff a = Aff::load(p + Aff::N_WORDS * i);
        Pt s = a.to_point().self_add();
        Aff r = s.is_identity() ? Aff::identity() : s.to_affine();
        r.store(out + Aff::N_WORDS * i);
    }
    return 0;
}

}  // namespace

extern "C" {

// Same op codes as orc_field_op in the oracle; field 0 / 1: BN254 Fq / Fr,
// 2 / 3: BLS12-381 Fq / Fr.
int ref_field_op(int field, int op, const uint32_t *a, const uint32_t *b, uint32_t *out, uint64_t count) {
    if (field == 0) return field_op<FqE>(op, a, b, out, count);
    if (field == 1) return field_op<FrE>(op, a, b, out, count);
    if (field == 2) return field_op<bls12381_fq::Element>(op, a, b, out, count);
    if (field == 3) return field_op<bls12381_fr::Element>(op, a, b, out, count);
    return -1;
}

// BLS12-381 G1: p + q (madd-2008-s) and 2p (dbl-2008-s-1), affine in and out.
int ref_bls_point_add(const uint32_t *p, const uint32_t *q, uint32_t *out, uint64_t count) {
    return point_add<bls12381::Point, bls12381::PointAffine>(p, q, out, count);
}
int ref_bls_point_dbl(const uint32_t *p, uint32_t *out, uint64_t count) {
    return point_dbl<bls12381::Point, bls12381::PointAffine>(p, out, count);
}

// out = p + q through PointXYZZ + PointAffine (madd-2008-s), then to_affine.
int ref_point_add(const uint32_t *p, const uint32_t *q, uint32_t *out, uint64_t count) {
    for (uint64_t i = 0; i < count; i++) {
        PointAffine a = PointAffine::load(p + 16 * i);
        PointAffine b = PointAffine::load(q + 16 * i);
        Point s = a.to_point() + b;
        PointAffine r = s.is_identity() ? PointAffine::identity() : s.to_affine();
        r.store(out + 16 * i);
    }
    return 0;
}

// out = 2p through PointXYZZ::self_add (dbl-2008-s-1).
int ref_point_dbl(const uint32_t *p, uint32_t *out, uint64_t count) {
    for (uint64_t i = 0; i < count; i++) {
        PointAffine a = PointAffine::load(p + 16 * i);
        Point s = a.to_point().self_add();
        PointAffine r = s.is_identity() ? PointAffine::identity() : s.to_affine();
        r.store(out + 16 * i);
    }
    return 0;
}

// sum_i k_i * P_i with the reference's host arithmetic: k_i is the scalar in
// Montgomery form (as the msm() C ABI receives it), reduced with to_number()
// like distribute_windows does (core/src/msm/src/msm_impl.cuh:52), then a
// left-to-right double-and-add per term.
int ref_msm_naive(const uint32_t *points, const uint32_t *scalars, uint64_t n, uint32_t *out) {
    return msm_naive<Point, PointAffine, FrE>(points, scalars, n, out);
}

// The same on BLS12-381 G1 (24-word affine points, 8-word Fr scalars).
int ref_bls_msm_naive(const uint32_t *points, const uint32_t *scalars, uint64_t n, uint32_t *out) {
    return msm_naive<bls12381::Point, bls12381::PointAffine, bls12381_fr::Element>(points, scalars, n, out);
}

}  // extern "C"
