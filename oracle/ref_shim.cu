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
// The functions below only marshal u32 arrays (the C ABI layout) into those
// types and call their host operators, so the C oracle can be compared with
// the reference's own arithmetic on the same inputs.
#include "bn254.cuh"

#include <cstdint>

using bn254::Point;
using bn254::PointAffine;
using FqE = bn254_fq::Element;
using FrE = bn254_fr::Element;
using Num = mont::Number<8>;

namespace {

template <class E>
int field_op(int op, const uint32_t *a, const uint32_t *b, uint32_t *out, uint64_t count) {
    for (uint64_t i = 0; i < count; i++) {
        const uint32_t *pa = a + 8 * i;
        const uint32_t *pb = b ? b + 8 * i : nullptr;
        E x = E::load(pa);
        E r;
        switch (op) {
        case 0: r = x + E::load(pb); break;
        case 1: r = x - E::load(pb); break;
        case 2: r = x * E::load(pb); break;
        case 3: r = x.square(); break;
        case 4: r = x.neg(); break;
        case 5: r = E::from_number(Num::load(pa)); break;
        case 6: {
            Num n = x.to_number();
            n.store(out + 8 * i);
            continue;
        }
        case 7: r = x.invert(); break;
        case 8: r = x.pow(Num::load(pb)); break;
        default: return -2;
        }
        r.store(out + 8 * i);
    }
    return 0;
}

}  // namespace

extern "C" {

// Same op codes as orc_field_op in bn254_oracle.c.
int ref_field_op(int field, int op, const uint32_t *a, const uint32_t *b, uint32_t *out, uint64_t count) {
    if (field == 0) return field_op<FqE>(op, a, b, out, count);
    if (field == 1) return field_op<FrE>(op, a, b, out, count);
    return -1;
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
    Point total = Point::identity();
    for (uint64_t i = 0; i < n; i++) {
        PointAffine p = PointAffine::load(points + 16 * i);
        Num k = FrE::load(scalars + 8 * i).to_number();
        Point acc = Point::identity();
        for (int bit = 255; bit >= 0; bit--) {
            acc = acc.self_add();
            if ((k.limbs[bit / 32] >> (bit % 32)) & 1) acc = acc + p;
        }
        total = total + acc;
    }
    PointAffine r = total.is_identity() ? PointAffine::identity() : total.to_affine();
    r.store(out);
    return 0;
}

}  // extern "C"
