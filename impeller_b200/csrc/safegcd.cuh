// Modular inversion by Bernstein-Yang divsteps, variable time.
//
// Used for the few conversions to affine form at the end of an MSM, where a
// single thread's latency is what counts.  The inputs are public (curve
// points), so variable time is fine.
//
// The method (D. J. Bernstein and B.-Y. Yang, "Fast constant-time gcd
// computation and modular inversion", 2019) keeps an odd f (initially the
// modulus p), a g (initially the input x) and an integer eta, and applies
// divsteps: with g odd and eta < 0, (f, g) <- (g, (g - f) / 2) and eta <-
// -eta - 1; with g odd and eta >= 0, g <- (g + f) / 2 and eta <- eta - 1;
// with g even, g <- g / 2 and eta <- eta - 1.  g reaches 0 with f = +-1.
// Divsteps look only at the low bits of f and g, so 30 of them at a time run
// on the low 32-bit words alone, collecting a 2x2 transition matrix
// T = [u v; q r] with 2^30 (f', g') = T (f, g); the full-width numbers are
// then updated once per batch.  Beside f and g the method carries d and e
// with d x = f and e x = g (mod p); they take the same matrix, divided by
// 2^30 modulo p, so at the end x^-1 = +-d.
//
// Inside a batch, runs of even steps are taken at once (count of trailing
// zeros), and consecutive odd steps that keep f are merged: while eta stays
// non-negative for the next `limit` steps, adding w f with
// w = -g / f mod 2^limit clears `limit` low bits of g, which is what those
// steps would do one by one.  |u| + |v| <= 2^30 and |q| + |r| <= 2^30 after a
// batch, so the matrix fits 32-bit signed integers (intermediate values wrap
// consistently modulo 2^32).
//
// Multi-precision numbers are signed radix-2^30: limbs 0..L-2 in [0, 2^30),
// the top limb signed.  Written for host and device so that the host build
// of this header can be checked against big-integer arithmetic.
#pragma once

#include <cstdint>

#if defined(__CUDACC__)
#define SG_HD __host__ __device__ __forceinline__
#define SG_CX __host__ __device__ constexpr
#else
#define SG_HD inline
#define SG_CX constexpr
#endif

namespace ec {
namespace sg {

static constexpr uint32_t M30 = 0x3fffffffu;

template <int L>
struct S30 {
    int32_t v[L];
};

struct Trans {
    int32_t u, v, q, r;
};

SG_HD int ctz32(uint32_t x) {
#if defined(__CUDA_ARCH__)
    return __ffs((int)x) - 1;
#else
    return __builtin_ctz(x);
#endif
}

// Limb count for an N-word (32-bit) modulus: the values stay below 2p in
// magnitude, plus a sign.
SG_CX int limbs_for(int N) { return (32 * N + 2 + 29) / 30; }

// Upper bound of batches: Bernstein-Yang's bound of (49 d + 57) / 17 divsteps
// for d-bit inputs, in batches of 30, plus one.
SG_CX int max_batches(int N) { return ((49 * 32 * N + 57) / 17 + 29) / 30 + 1; }

// 30 divsteps on the low words of f (odd) and g; returns the new eta.
SG_HD int divsteps30(int eta, uint32_t f, uint32_t g, Trans &t) {
    uint32_t u = 1, v = 0, q = 0, r = 1;
    int i = 30;
    for (;;) {
        const int z = ctz32(g | (0xffffffffu << i));  // even steps, at most i
        g >>= z;
        u <<= z;
        v <<= z;
        eta -= z;
        i -= z;
        if (i == 0) break;
        // f and g odd
        if (eta < 0) {
            uint32_t x;
            eta = -eta;
            x = f;
            f = g;
            g = 0u - x;
            x = u;
            u = q;
            q = 0u - x;
            x = v;
            v = r;
            r = 0u - x;
        }
        const int limit = (eta + 1) > i ? i : (eta + 1);
        const uint32_t m = 0xffffffffu >> (32 - limit);
        // f^-1 mod 2^32: (3f) xor 2 is right to 5 bits, each Newton step doubles that
        uint32_t fi = (3u * f) ^ 2u;
        fi *= 2u - f * fi;
        fi *= 2u - f * fi;
        fi *= 2u - f * fi;
        const uint32_t w = (0u - g * fi) & m;
        g += f * w;
        q += u * w;
        r += v * w;
    }
    t.u = (int32_t)u;
    t.v = (int32_t)v;
    t.q = (int32_t)q;
    t.r = (int32_t)r;
    return eta;
}

// (f, g) <- T (f, g) / 2^30 (exact).
template <int L>
SG_HD void update_fg(S30<L> &f, S30<L> &g, const Trans &t) {
    const int64_t u = t.u, v = t.v, q = t.q, r = t.r;
    int64_t cf = u * f.v[0] + v * g.v[0];
    int64_t cg = q * f.v[0] + r * g.v[0];
    cf >>= 30;
    cg >>= 30;
#pragma unroll
    for (int i = 1; i < L; i++) {
        cf += u * f.v[i] + v * g.v[i];
        cg += q * f.v[i] + r * g.v[i];
        f.v[i - 1] = (int32_t)(cf & M30);
        g.v[i - 1] = (int32_t)(cg & M30);
        cf >>= 30;
        cg >>= 30;
    }
    f.v[L - 1] = (int32_t)cf;
    g.v[L - 1] = (int32_t)cg;
}

// x < 0 (normalised form: the sign is the top limb's)
template <int L>
SG_HD bool s30_neg(const S30<L> &x) {
    return x.v[L - 1] < 0;
}

// x >= p for x >= 0
template <int L>
SG_HD bool s30_geq(const S30<L> &x, const S30<L> &p) {
#pragma unroll
    for (int i = L - 1; i >= 0; i--)
        if (x.v[i] != p.v[i]) return x.v[i] > p.v[i];
    return true;
}

// x += s * p for s = +-1, renormalising the limbs
template <int L>
SG_HD void s30_add_mul(S30<L> &x, const S30<L> &p, int32_t s) {
    int64_t c = 0;
#pragma unroll
    for (int i = 0; i < L - 1; i++) {
        c += (int64_t)x.v[i] + (int64_t)s * p.v[i];
        x.v[i] = (int32_t)(c & M30);
        c >>= 30;
    }
    x.v[L - 1] = (int32_t)(c + x.v[L - 1] + (int64_t)s * p.v[L - 1]);
}

// (d, e) <- T (d, e) / 2^30 mod p, for d, e in [0, p); results in [0, p).
// pinv = p^-1 mod 2^30.
template <int L>
SG_HD void update_de(S30<L> &d, S30<L> &e, const Trans &t, const S30<L> &p, uint32_t pinv) {
    const int64_t u = t.u, v = t.v, q = t.q, r = t.r;
    int64_t cd = u * d.v[0] + v * e.v[0];
    int64_t ce = q * d.v[0] + r * e.v[0];
    // md, me in [0, 2^30) make the low 30 bits of cd + md p and ce + me p zero
    const int64_t md = (int64_t)((0u - (uint32_t)cd * pinv) & M30);
    const int64_t me = (int64_t)((0u - (uint32_t)ce * pinv) & M30);
    cd += md * p.v[0];
    ce += me * p.v[0];
    cd >>= 30;
    ce >>= 30;
#pragma unroll
    for (int i = 1; i < L; i++) {
        cd += u * d.v[i] + v * e.v[i] + md * p.v[i];
        ce += q * d.v[i] + r * e.v[i] + me * p.v[i];
        d.v[i - 1] = (int32_t)(cd & M30);
        e.v[i - 1] = (int32_t)(ce & M30);
        cd >>= 30;
        ce >>= 30;
    }
    d.v[L - 1] = (int32_t)cd;
    e.v[L - 1] = (int32_t)ce;
    // (u d + v e + m p) / 2^30 lies in [-p, 2p): one correction each way
    if (s30_neg(d)) s30_add_mul(d, p, 1);
    else if (s30_geq(d, p)) s30_add_mul(d, p, -1);
    if (s30_neg(e)) s30_add_mul(e, p, 1);
    else if (s30_geq(e, p)) s30_add_mul(e, p, -1);
}

template <int L>
SG_HD bool s30_is_zero(const S30<L> &x) {
    int32_t o = 0;
#pragma unroll
    for (int i = 0; i < L; i++) o |= x.v[i];
    return o == 0;
}

// N 32-bit words (little-endian, value < 2^(32 N)) -> radix 2^30
template <int L, int N>
SG_HD S30<L> to_s30(const uint32_t *w) {
    S30<L> x;
#pragma unroll
    for (int i = 0; i < L; i++) {
        const int bit = 30 * i, k = bit >> 5, s = bit & 31;
        uint64_t lo = k < N ? w[k] : 0u;
        uint64_t hi = k + 1 < N ? w[k + 1] : 0u;
        x.v[i] = (int32_t)(((lo | (hi << 32)) >> s) & M30);
    }
    return x;
}

// radix 2^30 (non-negative, below 2^(32 N)) -> N 32-bit words
template <int L, int N>
SG_HD void from_s30(const S30<L> &x, uint32_t *w) {
#pragma unroll
    for (int k = 0; k < N; k++) {
        const int bit = 32 * k, i = bit / 30, s = bit % 30;
        uint64_t acc = (uint64_t)(uint32_t)x.v[i] >> s;
        int have = 30 - s;
        if (i + 1 < L) acc |= (uint64_t)(uint32_t)x.v[i + 1] << have;
        have += 30;
        if (have < 32 && i + 2 < L) acc |= (uint64_t)(uint32_t)x.v[i + 2] << have;
        w[k] = (uint32_t)acc;
    }
}

// p^-1 mod 2^30 for odd p0 (Newton from 5 bits)
SG_CX uint32_t inv30(uint32_t p0) {
    uint32_t x = (3u * p0) ^ 2u;
    x *= 2u - p0 * x;
    x *= 2u - p0 * x;
    x *= 2u - p0 * x;
    return x & M30;
}

// x^-1 mod p for the canonical x (N words, 0 <= x < p, p an odd prime);
// zero gives zero, as does a run that exceeds the step bound (no input in
// [0, p) does).  out: N words, canonical.
template <int N>
SG_HD void inverse(const uint32_t *x, const uint32_t *pw, uint32_t *out) {
    constexpr int L = limbs_for(N);
    const S30<L> p = to_s30<L, N>(pw);
    const uint32_t pinv = inv30(pw[0]);
    S30<L> f = p, g = to_s30<L, N>(x), d, e;
#pragma unroll
    for (int i = 0; i < L; i++) {
        d.v[i] = 0;
        e.v[i] = 0;
    }
    e.v[0] = 1;
#pragma unroll
    for (int k = 0; k < N; k++) out[k] = 0;
    if (s30_is_zero(g)) return;
    int eta = -1;
#pragma unroll 1
    for (int b = 0; b < max_batches(N); b++) {
        Trans t;
        eta = divsteps30(eta, (uint32_t)f.v[0] | ((uint32_t)f.v[1] << 30),
                         (uint32_t)g.v[0] | ((uint32_t)g.v[1] << 30), t);
        update_fg(f, g, t);
        update_de(d, e, t, p, pinv);
        if (s30_is_zero(g)) {
            // f = +-1: x^-1 = +-d
            if (s30_neg(f) && !s30_is_zero(d)) {
                S30<L> n = p;
                s30_add_mul(n, d, -1);
                d = n;
            }
            from_s30<L, N>(d, out);
            return;
        }
    }
}

}  // namespace sg
}  // namespace ec
