// Seeded synthetic inputs on the device, and element-wise field / point
// operations exported for the parity tests.
//
// The generator definitions are the ones the CPU oracle uses (splitmix64
// counter streams; uniform Fr element i = (lo + hi * 2^256) mod r from words
// 8i..8i+7; the skewed mix; P_i = r_i * G with G the curve's generator:
// (1, 2) on BN254, the standard G1 generator on BLS12-381), so the device and
// the oracle produce the same inputs bit for bit.
#include <string>

#include "../../include/impeller_msm.h"
#include "bn254.cuh"
#include "engine.h"

using namespace ec;

namespace {

#define GAMMA 0x9e3779b97f4a7c15ull

__device__ __forceinline__ u64 mix64(u64 z) {
    z = (z ^ (z >> 30)) * 0xbf58476d1ce4e5b9ull;
    z = (z ^ (z >> 27)) * 0x94d049bb133111ebull;
    return z ^ (z >> 31);
}

__device__ __forceinline__ u64 stream_key(u64 seed, u64 stream) {
    return mix64(seed * GAMMA + mix64(stream + 0x632be59bd9b4e019ull));
}

__device__ __forceinline__ u64 stream_word(u64 key, u64 idx) { return mix64(key + (idx + 1) * GAMMA); }

template <class F>
__device__ __forceinline__ Fe<F> fe_rsq() {
    constexpr Words<F::N> r2 = words(F::RSQ);
    Fe<F> r;
#pragma unroll
    for (int i = 0; i < F::N; i++) r.l[i] = r2.v[i];
    return r;
}

// canonical uniform Fr element idx of the stream with this key
template <class C>
__device__ Fe<typename C::Fr> uniform_fr(u64 key, u64 idx) {
    using FR = typename C::Fr;
    constexpr Words<8> m = words(FR::M);
    u32 lo[8], hi[8];
    for (int k = 0; k < 4; k++) {
        u64 w = stream_word(key, 8 * idx + k);
        lo[2 * k] = (u32)w;
        lo[2 * k + 1] = (u32)(w >> 32);
        u64 v = stream_word(key, 8 * idx + 4 + k);
        hi[2 * k] = (u32)v;
        hi[2 * k + 1] = (u32)(v >> 32);
    }
    while (un_geq<8>(lo, m.v)) un_sub<8>(lo, m.v);
    while (un_geq<8>(hi, m.v)) un_sub<8>(hi, m.v);
    Fe<FR> h, l;
    for (int i = 0; i < 8; i++) {
        h.l[i] = hi[i];
        l.l[i] = lo[i];
    }
    Fe<FR> t = fe_mul<FR>(h, fe_rsq<FR>());  // hi * 2^256 mod r
    return fe_canon<FR>(fe_add<FR>(l, t));
}

template <class C>
__global__ void k_gen_scalars(u32 *out, u64 n, u64 seed, u64 stream, int dist, u64 start, int mont) {
    using FR = typename C::Fr;
    const u64 key = stream_key(seed, stream);
    const u64 key_cat = stream_key(seed, stream + (1ull << 32));
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        const u64 idx = start + i;
        Fe<FR> v = fe_zero<FR>();
        bool uniform = true;
        if (dist == 1) {
            u64 u = stream_word(key_cat, idx);
            u64 cat = u % 10;
            if (cat < 7) {
                uniform = false;
                if (cat >= 2 && cat < 4) v.l[0] = 1;
                else if (cat >= 4) v.l[0] = (u32)((u >> 40) & 0xffffu);
            }
        }
        if (uniform) v = uniform_fr<C>(key, idx);
        if (mont) v = fe_canon<FR>(fe_mul<FR>(v, fe_rsq<FR>()));
        fe_store(out + 8 * i, v);
    }
}

template <class C>
__device__ __forceinline__ AffineT<typename C::Fq> generator() {
    constexpr Words<C::Fq::N> gx = words(C::GX), gy = words(C::GY);
    AffineT<typename C::Fq> g;
#pragma unroll
    for (int i = 0; i < C::Fq::N; i++) {
        g.x.l[i] = gx.v[i];
        g.y.l[i] = gy.v[i];
    }
    return g;
}

template <class C>
__global__ void k_gen_points(u32 *out, u64 n, u64 seed, u64 start) {
    using FQ = typename C::Fq;
    const u64 key = stream_key(seed, 0);
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (u64)gridDim.x * blockDim.x) {
        Fe<typename C::Fr> r = uniform_fr<C>(key, start + i);
        const AffineT<FQ> g = generator<C>();
        XyzzT<FQ> acc = xyzz_identity<FQ>();
        for (int bit = 255; bit >= 0; bit--) {
            acc = xyzz_dbl(acc);
            if ((r.l[bit >> 5] >> (bit & 31)) & 1u) acc = xyzz_add_affine(acc, g);
        }
        affine_store(out + C::PW * i, xyzz_to_affine(acc));
    }
}

template <class F>
__device__ Fe<F> test_op(int op, const Fe<F> &a, const Fe<F> &b) {
    const Fe<F> r2 = fe_rsq<F>();
    switch (op) {
    case 0: return fe_add<F>(a, b);
    case 1: return fe_sub<F>(a, b);
    case 2: return fe_mul<F>(a, b);
    case 3: return fe_sqr<F>(a);
    case 4: return fe_neg<F>(a);
    case 5: return fe_mul<F>(a, r2);
    case 6: return fe_from_mont<F>(a);
    case 7: return fe_inv<F>(a);
    case 8: return fe_pow<F>(a, b.l);
    case 9: return fe_inv_binary<F>(a, fe_mul<F>(fe_mul<F>(r2, r2), fe_one<F>()));
    default: return fe_inv_divsteps<F>(a, fe_mul<F>(fe_mul<F>(r2, r2), fe_one<F>()));
    }
}

template <class F>
__global__ void k_test_field(int op, const u32 *a, const u32 *b, u32 *out, u64 count) {
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    Fe<F> x = fe_load<F>(a + F::N * i), y = b ? fe_load<F>(b + F::N * i) : fe_zero<F>();
    fe_store(out + F::N * i, fe_canon<F>(test_op<F>(op, x, y)));
}

template <class C>
__global__ void k_test_point(int op, const u32 *p, const u32 *q, u32 *out, u64 count) {
    using FQ = typename C::Fq;
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= count) return;
    AffineT<FQ> a = affine_load<FQ>(p + C::PW * i);
    XyzzT<FQ> r;
    switch (op) {
    case 0: r = xyzz_add_affine(xyzz_from_affine(a), affine_load<FQ>(q + C::PW * i)); break;
    case 1: r = xyzz_dbl(xyzz_from_affine(a)); break;
    case 2: r = xyzz_add(xyzz_from_affine(a), xyzz_from_affine(affine_load<FQ>(q + C::PW * i))); break;
    default: {
        const u32 *k = q + 8 * i;
        XyzzT<FQ> acc = xyzz_identity<FQ>();
        for (int bit = 255; bit >= 0; bit--) {
            acc = xyzz_dbl(acc);
            if ((k[bit >> 5] >> (bit & 31)) & 1u) acc = xyzz_add_affine(acc, a);
        }
        r = acc;
    }
    }
    affine_store(out + C::PW * i, xyzz_to_affine(r));
}

// Throughput ceiling of the Montgomery product itself: four independent
// chains of base-field products per thread at full occupancy, nothing else
// in the loop.  An N-limb product is 2 N^2 + N 32x32 -> 64-bit partial
// products (N^2 for a*b, N^2 for m*p, N reduction factors): 136 for BN254's
// 8 limbs, 300 for BLS12-381's 12.
template <class F>
__global__ void k_imad_peak(u32 *out, u32 iters, u32 seed) {
    constexpr int N = F::N;
    constexpr Words<N> mod = words(F::M);
    const u32 top = (1u << (31 - __clz(mod.v[N - 1]))) - 1u;  // keeps values below p
    Fe<F> acc[4], m;
#pragma unroll
    for (int k = 0; k < N; k++) m.l[k] = seed * (threadIdx.x + 5 * k + 1) + blockIdx.x;
    m.l[N - 1] &= top;
#pragma unroll
    for (int r = 0; r < 4; r++) {
#pragma unroll
        for (int k = 0; k < N; k++) acc[r].l[k] = m.l[(k + r) % N] ^ (u32)r;
        acc[r].l[N - 1] &= top;
    }
#pragma unroll 1
    for (u32 it = 0; it < iters; it++) {
#pragma unroll
        for (int r = 0; r < 4; r++) acc[r] = fe_mul<F>(acc[r], m);
    }
    u32 v = 0;
#pragma unroll
    for (int r = 0; r < 4; r++)
#pragma unroll
        for (int k = 0; k < N; k++) v ^= acc[r].l[k];
    if (v == 0x12345678u) out[blockIdx.x * blockDim.x + threadIdx.x] = v;
}

// Dependent chains of one operation on one thread (op 0 Fq product,
// 1 XYZZ addition, 2 XYZZ doubling, 3 mixed addition), for latency numbers.
__global__ void k_op_latency(int op, u32 iters, u32 *out, long long *cycles) {
    Fq a = fe_one<FqP>();
    a.l[0] ^= 0x1234567u;
    Affine q;
    q.x = fe_one<FqP>();
    q.y = fe_add<FqP>(q.x, q.x);
    Xyzz p = xyzz_from_affine(q);
    p = xyzz_dbl(p);
    long long t0 = clock64();
    for (u32 i = 0; i < iters; i++) {
        switch (op) {
        case 0: a = fe_mul<FqP>(a, a); break;
        case 1: p = xyzz_add(p, xyzz_dbl(p)); break;
        case 2: p = xyzz_dbl(p); break;
        default: p = xyzz_add_affine(p, q); break;
        }
    }
    long long t1 = clock64();
    out[0] = a.l[0] ^ p.x.l[0];
    *cycles = t1 - t0;
}

cudaError_t launched(const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) impeller::set_error(std::string("launch of ") + what + " failed: " + cudaGetErrorString(e));
    return e;
}

template <class F>
cudaError_t imad_peak(int device, double *gops) {
    if (!gops) return cudaErrorInvalidValue;
    cudaError_t e = cudaSetDevice(device);
    if (e != cudaSuccess) return e;
    int sms = 0;
    cudaDeviceGetAttribute(&sms, cudaDevAttrMultiProcessorCount, device);
    const u32 blocks = (u32)sms * 8, threads = 256, iters = F::N == 8 ? 1u << 11 : 1u << 10;
    u32 *out = nullptr;
    if ((e = cudaMalloc(&out, (size_t)blocks * threads * 4)) != cudaSuccess) return e;
    cudaEvent_t t0, t1;
    cudaEventCreate(&t0);
    cudaEventCreate(&t1);
    k_imad_peak<F><<<blocks, threads>>>(out, iters / 8, 7u);  // warm-up
    float best = 1e30f;
    for (int rep = 0; rep < 3; rep++) {
        cudaEventRecord(t0);
        k_imad_peak<F><<<blocks, threads>>>(out, iters, 7u);
        cudaEventRecord(t1);
        cudaEventSynchronize(t1);
        float ms = 0;
        cudaEventElapsedTime(&ms, t0, t1);
        best = ms < best ? ms : best;
    }
    e = cudaGetLastError();
    cudaEventDestroy(t0);
    cudaEventDestroy(t1);
    cudaFree(out);
    if (e != cudaSuccess) return e;
    const double products = 2.0 * F::N * F::N + F::N;
    *gops = (double)blocks * threads * iters * 4.0 * products / (best * 1e-3) / 1e9;
    return cudaSuccess;
}

}  // namespace

extern "C" {

cudaError_t impeller_gen_scalars_curve(int curve, uint32_t *d_out, uint64_t n, uint64_t seed, uint64_t stream,
                                       int dist, uint64_t start, int mont, cudaStream_t s) {
    if ((!d_out && n) || (curve != IMPELLER_CURVE_BN254 && curve != IMPELLER_CURVE_BLS12381)) {
        impeller::set_error("impeller_gen_scalars: bad argument");
        return cudaErrorInvalidValue;
    }
    if (n == 0) return cudaSuccess;
    const u64 blocks = (n + 255) / 256;
    const unsigned grid = (unsigned)(blocks < 65535 ? blocks : 65535);
    if (curve == IMPELLER_CURVE_BN254)
        k_gen_scalars<Bn254><<<grid, 256, 0, s>>>(d_out, n, seed, stream, dist, start, mont);
    else
        k_gen_scalars<Bls12381><<<grid, 256, 0, s>>>(d_out, n, seed, stream, dist, start, mont);
    return launched("k_gen_scalars");
}

cudaError_t impeller_gen_scalars(uint32_t *d_out, uint64_t n, uint64_t seed, uint64_t stream, int dist,
                                 uint64_t start, int mont, cudaStream_t s) {
    return impeller_gen_scalars_curve(IMPELLER_CURVE_BN254, d_out, n, seed, stream, dist, start, mont, s);
}

cudaError_t impeller_gen_points_curve(int curve, uint32_t *d_out, uint64_t n, uint64_t seed, uint64_t start,
                                      cudaStream_t s) {
    if ((!d_out && n) || (curve != IMPELLER_CURVE_BN254 && curve != IMPELLER_CURVE_BLS12381)) {
        impeller::set_error("impeller_gen_points: bad argument");
        return cudaErrorInvalidValue;
    }
    if (n == 0) return cudaSuccess;
    const u64 blocks = (n + 127) / 128;
    const unsigned grid = (unsigned)(blocks < 65535 ? blocks : 65535);
    if (curve == IMPELLER_CURVE_BN254)
        k_gen_points<Bn254><<<grid, 128, 0, s>>>(d_out, n, seed, start);
    else
        k_gen_points<Bls12381><<<grid, 128, 0, s>>>(d_out, n, seed, start);
    return launched("k_gen_points");
}

cudaError_t impeller_gen_points(uint32_t *d_out, uint64_t n, uint64_t seed, uint64_t start, cudaStream_t s) {
    return impeller_gen_points_curve(IMPELLER_CURVE_BN254, d_out, n, seed, start, s);
}

cudaError_t impeller_imad_peak(int device, double *gops) { return imad_peak<FqP>(device, gops); }

cudaError_t impeller_imad_peak_curve(int device, unsigned int curve, double *gops) {
    if (curve == IMPELLER_CURVE_BLS12381) return imad_peak<BlsFqP>(device, gops);
    if (curve == IMPELLER_CURVE_BN254) return imad_peak<FqP>(device, gops);
    impeller::set_error("impeller_imad_peak_curve: unknown curve");
    return cudaErrorInvalidValue;
}

cudaError_t impeller_op_latency(int op, uint32_t iters, double *cycles_per_op) {
    if (!cycles_per_op || iters == 0) return cudaErrorInvalidValue;
    u32 *out = nullptr;
    long long *cyc = nullptr;
    cudaError_t e = cudaMalloc(&out, 64);
    if (e != cudaSuccess) return e;
    if ((e = cudaMalloc(&cyc, 8)) != cudaSuccess) {
        cudaFree(out);
        return e;
    }
    k_op_latency<<<1, 1>>>(op, iters, out, cyc);
    long long h = 0;
    e = cudaMemcpy(&h, cyc, 8, cudaMemcpyDeviceToHost);
    cudaFree(out);
    cudaFree(cyc);
    if (e != cudaSuccess) return e;
    *cycles_per_op = (double)h / iters;
    return cudaSuccess;
}

cudaError_t impeller_test_field_op(int field, int op, const uint32_t *d_a, const uint32_t *d_b, uint32_t *d_out,
                                   uint64_t count, cudaStream_t s) {
    if (field < 0 || field > 3 || op < 0 || op > 10 || !d_a || !d_out) {
        impeller::set_error("impeller_test_field_op: bad argument");
        return cudaErrorInvalidValue;
    }
    if (count == 0) return cudaSuccess;
    const unsigned grid = (unsigned)((count + 127) / 128);
    switch (field) {
    case 0: k_test_field<FqP><<<grid, 128, 0, s>>>(op, d_a, d_b, d_out, count); break;
    case 1: k_test_field<FrP><<<grid, 128, 0, s>>>(op, d_a, d_b, d_out, count); break;
    case 2: k_test_field<BlsFqP><<<grid, 128, 0, s>>>(op, d_a, d_b, d_out, count); break;
    default: k_test_field<BlsFrP><<<grid, 128, 0, s>>>(op, d_a, d_b, d_out, count); break;
    }
    return launched("k_test_field");
}

cudaError_t impeller_test_point_op_curve(int curve, int op, const uint32_t *d_p, const uint32_t *d_q, uint32_t *d_out,
                                         uint64_t count, cudaStream_t s) {
    if (op < 0 || op > 3 || !d_p || !d_out || (op != 1 && !d_q) ||
        (curve != IMPELLER_CURVE_BN254 && curve != IMPELLER_CURVE_BLS12381)) {
        impeller::set_error("impeller_test_point_op: bad argument");
        return cudaErrorInvalidValue;
    }
    if (count == 0) return cudaSuccess;
    const unsigned grid = (unsigned)((count + 127) / 128);
    if (curve == IMPELLER_CURVE_BN254)
        k_test_point<Bn254><<<grid, 128, 0, s>>>(op, d_p, d_q, d_out, count);
    else
        k_test_point<Bls12381><<<grid, 128, 0, s>>>(op, d_p, d_q, d_out, count);
    return launched("k_test_point");
}

cudaError_t impeller_test_point_op(int op, const uint32_t *d_p, const uint32_t *d_q, uint32_t *d_out,
                                   uint64_t count, cudaStream_t s) {
    return impeller_test_point_op_curve(IMPELLER_CURVE_BN254, op, d_p, d_q, d_out, count, s);
}

}  // extern "C"
