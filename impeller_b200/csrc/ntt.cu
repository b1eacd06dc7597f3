// Number-theoretic transform over the 8-limb fields (BN254 Fr by default),
// the drop-in for the reference's NTT library (core/src/ntt/src/ntt.h).
//
// Transform: X[k] = sum_j x[j] w^(j k), n = 2^L, in place, natural order in
// and out (what the reference's ssip_ntt / recompute_ntt compute,
// core/src/ntt/tests/test_ssip.cu:27-43).
//
// B200 layout of the work (not the reference's self-sorting stage kernels):
//   - decimation-in-frequency passes, each over a contiguous range of R index
//     bits: a CTA loads a tile of 2^(R + logC) elements (2^R points of the
//     pass's digit times C = 2^logC consecutive low indices, so every global
//     access is a run of C * 32 B) into shared memory, runs the R radix-2
//     stages there two at a time (a thread takes four elements through two
//     stages between shared-memory round trips; one Montgomery product per
//     butterfly), and writes the tile back in place.  Tiles are disjoint, so passes are in place without
//     a scratch array.  The last pass takes the lowest 11 bits (a contiguous
//     2048-element block);
//   - one reordering pass (index bit reversal) with two 16 x 16 tiles per CTA
//     (the tile of middle bits b and the tile of rev(b) swap), which also
//     reduces every value to canonical form.  When n <= 2048 the single tile
//     of the only pass is written out reversed directly.
// Work per element: L/2 Montgomery products and L additions/subtractions, so
// on B200 the transform is bound by the integer multiply-add rate (like the
// MSM's accumulation), not by HBM: a pass moves 64 B per element plus twiddle
// reads, about 10 ps per element at 6.6 TB/s, against ~8 ps of products per
// pass bit.  Values stay in the lazy [0, 2m) range between butterflies.
#include <cstdint>
#include <string>
#include <vector>

#include "../../include/impeller_ntt.h"
#include "bn254.cuh"
#include "engine.h"

using namespace ec;

namespace {

constexpr u32 TILE_LOG = 11;               // elements per pass tile: 2048 x 32 B = 64 KiB of shared memory
constexpr u32 TILE = 1u << TILE_LOG;
constexpr u32 THREADS = 256;
constexpr u32 MID_MAX = 9;                 // bits per pass above the last (C >= 4: 128 B runs)
constexpr u32 TAB_LOG = 11;                // power tables for recomputed twiddles: 2048 entries each
constexpr u32 TAB = 1u << TAB_LOG;
constexpr u32 REV_T = 4;                   // reordering tile: 16 x 16

// A logical polynomial view (PolyPtr): element i at base[(start + i) mod whole].
struct View {
    u32 *base;
    u64 start;
    u64 whole;
};

__device__ __forceinline__ u32 *at(const View &v, u64 i) {
    u64 p = v.start + i;
    if (p >= v.whole) p -= v.whole;
    return v.base + 8 * p;
}

// Shared-memory tiles hold the two 16-byte halves of the elements in two
// planes (half 0 of element e at s[e], half 1 at s[plane + e]): neighbouring
// elements then sit in neighbouring 16-byte bank groups.
template <class F>
__device__ __forceinline__ void smem_store(uint4 *s, u32 plane, u32 e, const Fe<F> &a) {
    s[e] = make_uint4(a.l[0], a.l[1], a.l[2], a.l[3]);
    s[plane + e] = make_uint4(a.l[4], a.l[5], a.l[6], a.l[7]);
}

template <class F>
__device__ __forceinline__ Fe<F> smem_load(const uint4 *s, u32 plane, u32 e) {
    const uint4 x = s[e], y = s[plane + e];
    Fe<F> a;
    a.l[0] = x.x; a.l[1] = x.y; a.l[2] = x.z; a.l[3] = x.w;
    a.l[4] = y.x; a.l[5] = y.y; a.l[6] = y.z; a.l[7] = y.w;
    return a;
}

__device__ __forceinline__ u32 brev(u32 x, u32 bits) { return bits ? __brev(x) >> (32 - bits) : 0; }

// w^e: from the caller's table (twiddle[e] = w^e), or recomputed from three
// power tables tab[t][j] = w^(j << 11t) (one or two extra products).
template <class F, bool RECOMP>
__device__ __forceinline__ Fe<F> twiddle(const u32 *tw, u32 e) {
    if (!RECOMP) return fe_load<F>(tw + 8 * (u64)e);
    Fe<F> w = fe_load<F>(tw + 8 * (e & (TAB - 1)));
    if (e >> TAB_LOG) w = fe_mul<F>(w, fe_load<F>(tw + 8 * (TAB + ((e >> TAB_LOG) & (TAB - 1)))));
    if (e >> (2 * TAB_LOG)) w = fe_mul<F>(w, fe_load<F>(tw + 8 * (2 * TAB + (e >> (2 * TAB_LOG)))));
    return w;
}

// One decimation-in-frequency pass over index bits [lo, lo + R) of an n = 2^L
// transform.  CTA tile: elements (hi, d, low0 + c) for d < 2^R, c < 2^logC,
// global index (hi << (lo + R)) | (d << lo) | (low0 + c).  Stage s (global
// bit, from lo + R - 1 down to lo) pairs d with d + 2^(s - lo):
//   a' = a + b,  b' = (a - b) * w^((i mod 2^s) << (L - 1 - s)).
// Stages go in pairs (s, s - 1); the two pairs of the lower stage share one
// twiddle.  An odd last stage runs alone.  The sums of the first stage wait
// in shared memory while its differences are multiplied, which keeps the
// kernel at 76-80 registers: three 256-thread CTAs per SM (24 warps), 7.6 %
// faster at 2^24 than holding all four values in registers (114 registers,
// two CTAs).
// rev_out (only when the tile is the whole array): write element p to
// position rev_L(p), canonical.
template <class F, bool RECOMP>
__global__ void __launch_bounds__(THREADS, 3)
k_ntt_pass(View v, const u32 *tw, u32 L, u32 lo, u32 R, u32 logC, int rev_out) {
    extern __shared__ uint4 ntt_smem[];
    const u32 tile_log = R + logC;
    const u32 tsize = 1u << tile_log;
    const u32 C = 1u << logC;
    const u32 nlb_log = lo - logC;  // low blocks per hi
    const u64 t = blockIdx.x;
    const u64 low0 = (t & ((1ull << nlb_log) - 1)) << logC;
    const u64 hi = t >> nlb_log;
    const u64 gbase = (hi << (lo + R)) | low0;

    for (u32 e = threadIdx.x; e < tsize; e += blockDim.x) {
        const u64 gi = gbase | ((u64)(e >> logC) << lo) | (e & (C - 1));
        const uint4 *p = reinterpret_cast<const uint4 *>(at(v, gi));
        ntt_smem[e] = p[0];
        ntt_smem[tsize + e] = p[1];
    }
    __syncthreads();

    int sl = (int)R - 1;
    while (sl >= 1) {
        // two stages per round (index bits sl and sl - 1 of the digit): a
        // thread loads four elements d0, d0 + h, d0 + 2h, d0 + 3h (h = 2^(sl-1))
        const u32 s = lo + (u32)sl;
        const u32 h = 1u << (sl - 1);
        const u32 hmask = h - 1;
        for (u32 qd = threadIdx.x; qd < tsize / 4; qd += blockDim.x) {
            const u32 c = qd & (C - 1);
            const u32 q = qd >> logC;
            const u32 d0 = ((q >> (sl - 1)) << (sl + 1)) | (q & hmask);
            const u32 low = (u32)(low0 + c);
            const u32 j0 = ((d0 & (2 * h - 1)) << lo) | low;  // i mod 2^s for d0 (bit sl-1 of d0 is 0)
            const u32 ex0 = j0 << (L - 1 - s), ex1 = (j0 + (h << lo)) << (L - 1 - s);
            const u32 ex2 = (((d0 & hmask) << lo) | low) << (L - s);
            const u32 e0 = (d0 << logC) | c, eh = h << logC;
            Fe<F> b0, b1;
            {
                const Fe<F> x0 = smem_load<F>(ntt_smem, tsize, e0), x2 = smem_load<F>(ntt_smem, tsize, e0 + 2 * eh);
                b0 = fe_sub<F>(x0, x2);
                smem_store<F>(ntt_smem, tsize, e0, fe_add<F>(x0, x2));  // a0, kept in place
            }
            if (ex0) b0 = fe_mul<F>(b0, twiddle<F, RECOMP>(tw, ex0));
            {
                const Fe<F> x1 = smem_load<F>(ntt_smem, tsize, e0 + eh), x3 = smem_load<F>(ntt_smem, tsize, e0 + 3 * eh);
                b1 = fe_sub<F>(x1, x3);
                smem_store<F>(ntt_smem, tsize, e0 + eh, fe_add<F>(x1, x3));  // a1
            }
            b1 = fe_mul<F>(b1, twiddle<F, RECOMP>(tw, ex1));  // ex1 != 0: bit (lo + sl - 1) of j is set
            const Fe<F> a0 = smem_load<F>(ntt_smem, tsize, e0), a1 = smem_load<F>(ntt_smem, tsize, e0 + eh);
            Fe<F> y1 = fe_sub<F>(a0, a1), y3 = fe_sub<F>(b0, b1);
            smem_store<F>(ntt_smem, tsize, e0, fe_add<F>(a0, a1));
            smem_store<F>(ntt_smem, tsize, e0 + 2 * eh, fe_add<F>(b0, b1));
            if (ex2) {
                const Fe<F> w2 = twiddle<F, RECOMP>(tw, ex2);
                y1 = fe_mul<F>(y1, w2);
                y3 = fe_mul<F>(y3, w2);
            }
            smem_store<F>(ntt_smem, tsize, e0 + eh, y1);
            smem_store<F>(ntt_smem, tsize, e0 + 3 * eh, y3);
        }
        __syncthreads();
        sl -= 2;
    }
    if (sl == 0) {
        const u32 s = lo;
        for (u32 b = threadIdx.x; b < tsize / 2; b += blockDim.x) {
            const u32 c = b & (C - 1);
            const u32 e0 = ((b >> logC) << (logC + 1)) | c, e1 = e0 + C;
            const Fe<F> x = smem_load<F>(ntt_smem, tsize, e0), y = smem_load<F>(ntt_smem, tsize, e1);
            Fe<F> dif = fe_sub<F>(x, y);
            const u32 ex = ((u32)(low0 + c)) << (L - 1 - s);
            if (ex) dif = fe_mul<F>(dif, twiddle<F, RECOMP>(tw, ex));
            smem_store<F>(ntt_smem, tsize, e0, fe_add<F>(x, y));
            smem_store<F>(ntt_smem, tsize, e1, dif);
        }
        __syncthreads();
    }

    if (rev_out) {
        for (u32 e = threadIdx.x; e < tsize; e += blockDim.x) {
            const Fe<F> a = fe_canon<F>(smem_load<F>(ntt_smem, tsize, e));
            fe_store(at(v, brev(e, L)), a);
        }
        return;
    }
    for (u32 e = threadIdx.x; e < tsize; e += blockDim.x) {
        const u64 gi = gbase | ((u64)(e >> logC) << lo) | (e & (C - 1));
        uint4 *p = reinterpret_cast<uint4 *>(at(v, gi));
        p[0] = ntt_smem[e];
        p[1] = ntt_smem[tsize + e];
    }
}

// Bit-reversal reordering of n = 2^L > 2048 elements, in place, canonical
// output.  Index i = (a, b, c): a the top 4 bits, c the low 4 bits, b the
// middle m = L - 8 bits; rev(i) = (rev4(c), rev_m(b), rev4(a)).  The CTA for
// b (with b <= rev_m(b)) holds tiles b and rev_m(b) (16 rows of 16
// consecutive elements each) and writes each into the other's place.
template <class F>
__global__ void __launch_bounds__(256) k_ntt_reverse(View v, u32 L) {
    __shared__ uint4 tl[2][16 * 17 * 2];  // 16 x 16 elements, rows padded to 17
    const u32 m = L - 2 * REV_T;
    const u32 b = blockIdx.x;
    const u32 rb = brev(b, m);
    if (rb < b) return;
    const u32 a = threadIdx.x >> 4, c = threadIdx.x & 15;
    const u32 sh = L - REV_T;
    {
        const uint4 *p = reinterpret_cast<const uint4 *>(at(v, ((u64)a << sh) | ((u64)b << REV_T) | c));
        tl[0][a * 17 + c] = p[0];
        tl[0][16 * 17 + a * 17 + c] = p[1];
        if (rb != b) {
            const uint4 *q = reinterpret_cast<const uint4 *>(at(v, ((u64)a << sh) | ((u64)rb << REV_T) | c));
            tl[1][a * 17 + c] = q[0];
            tl[1][16 * 17 + a * 17 + c] = q[1];
        }
    }
    __syncthreads();
    // destination (a, rb, c) <- source (rev4(c), b, rev4(a)), and the mirror
    const u32 src = brev(c, REV_T) * 17 + brev(a, REV_T);
    fe_store(at(v, ((u64)a << sh) | ((u64)rb << REV_T) | c), fe_canon<F>(smem_load<F>(tl[0], 16 * 17, src)));
    if (rb != b)
        fe_store(at(v, ((u64)a << sh) | ((u64)b << REV_T) | c), fe_canon<F>(smem_load<F>(tl[1], 16 * 17, src)));
}

// omegas[k] = u^(2^k), k < 33 (one thread).
template <class F>
__global__ void k_omegas(const u32 *unit, u32 *omegas, u32 count) {
    if (threadIdx.x || blockIdx.x) return;
    Fe<F> w = fe_canon<F>(fe_load<F>(unit));
    for (u32 k = 0; k < count; k++) {
        fe_store(omegas + 8 * k, fe_canon<F>(w));
        w = fe_sqr<F>(w);
    }
}

// tab[t][j] = w^(j << 11t) = prod over set bits k of j: omegas[11t + k].
template <class F>
__global__ void k_pow_tables(const u32 *omegas, u32 *tab, u32 n_omegas) {
    const u32 g = blockIdx.x * blockDim.x + threadIdx.x;
    if (g >= 3 * TAB) return;
    const u32 t = g / TAB, j = g % TAB;
    Fe<F> acc = fe_one<F>();
    for (u32 k = 0; k < TAB_LOG; k++) {
        const u32 idx = TAB_LOG * t + k;
        if (((j >> k) & 1) && idx < n_omegas) acc = fe_mul<F>(acc, fe_load<F>(omegas + 8 * idx));
    }
    fe_store(tab + 8 * g, fe_canon<F>(acc));
}

// out[i] = w^(i * step) for i < len, from the power tables.
template <class F>
__global__ void k_powers(const u32 *tab, u32 *out, u64 len, u64 step) {
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (u64)gridDim.x * blockDim.x)
        fe_store(out + 8 * i, fe_canon<F>(twiddle<F, true>(tab, (u32)(i * step))));
}

// poly[i] *= powers[((begin + i) mod plen) mod pnum]
template <class F>
__global__ void k_distribute_powers(View v, u64 len, const u32 *powers, u64 pnum, u64 begin, u64 plen) {
    const bool direct = begin == 0 && plen >= len && pnum >= len;
    for (u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x; i < len; i += (u64)gridDim.x * blockDim.x) {
        const u64 k = direct ? i : ((begin + i) % plen) % pnum;
        u32 *p = at(v, i);
        fe_store(p, fe_canon<F>(fe_mul<F>(fe_load<F>(p), fe_load<F>(powers + 8 * k))));
    }
}

}  // namespace

// ------------------------------------------------------------------ host

namespace {

using impeller::set_error;

cudaError_t launched(const char *what) {
    cudaError_t e = cudaGetLastError();
    if (e != cudaSuccess) set_error(std::string("launch of ") + what + " failed: " + cudaGetErrorString(e));
    return e;
}

#define NTT_CK(x)                                  \
    do {                                           \
        cudaError_t e_ = (x);                      \
        if (e_ != cudaSuccess) return e_;          \
    } while (0)

bool aligned16(const void *p) { return (reinterpret_cast<uintptr_t>(p) & 15) == 0; }

// PolyPtr -> View, with the reference's rules (make_slice_iter,
// core/src/common/iter/src/iter.cuh:309-316).
bool make_view(const PolyPtr &x, View &v, const char *who) {
    const u64 whole = x.whole_len ? x.whole_len : x.len;
    if (!x.ptr || !aligned16(x.ptr)) {
        set_error(std::string(who) + ": null or misaligned polynomial pointer");
        return false;
    }
    if (x.len > whole) {
        set_error(std::string(who) + ": len exceeds whole_len");
        return false;
    }
    u64 start = x.offset;
    if (x.rotate) {
        if (x.len != whole || x.offset != 0 || x.rotate >= x.len) {
            set_error(std::string(who) + ": a rotated polynomial must be whole, unsliced and rotate < len");
            return false;
        }
        start = x.len - x.rotate;
    }
    if (whole && start >= whole) {
        set_error(std::string(who) + ": offset out of range");
        return false;
    }
    v.base = x.ptr;
    v.start = start;
    v.whole = whole ? whole : 1;
    return true;
}

struct PassPlan {
    u32 lo, R, logC;
};

std::vector<PassPlan> plan_passes(u32 L) {
    std::vector<PassPlan> p;
    if (L <= TILE_LOG) {
        p.push_back({0, L, 0});
        return p;
    }
    const u32 M = L - TILE_LOG;
    const u32 np = (M + MID_MAX - 1) / MID_MAX;
    u32 cursor = L;
    for (u32 k = 0; k < np; k++) {
        const u32 R = M / np + (k < M % np ? 1 : 0);
        cursor -= R;
        p.push_back({cursor, R, TILE_LOG - R});
    }
    p.push_back({0, TILE_LOG, 0});
    return p;
}

template <class F, bool RECOMP>
cudaError_t run_ntt(const View &v, const u32 *tw, u32 L, cudaStream_t st) {
    if (L == 0) return cudaSuccess;
    auto kern = k_ntt_pass<F, RECOMP>;
    NTT_CK(cudaFuncSetAttribute(kern, cudaFuncAttributeMaxDynamicSharedMemorySize, TILE * 32));
    const std::vector<PassPlan> passes = plan_passes(L);
    const bool single = L <= TILE_LOG;
    for (const PassPlan &pp : passes) {
        const u32 tile_log = pp.R + pp.logC;
        const u64 grid = 1ull << (L - tile_log);
        kern<<<(unsigned)grid, THREADS, (size_t)32 << tile_log, st>>>(v, tw, L, pp.lo, pp.R, pp.logC, single ? 1 : 0);
        NTT_CK(launched("k_ntt_pass"));
    }
    if (!single) {
        k_ntt_reverse<F><<<1u << (L - 2 * REV_T), 256, 0, st>>>(v, L);
        NTT_CK(launched("k_ntt_reverse"));
    }
    return cudaSuccess;
}

// Power tables of w = omegas[0] (omegas[k] = w^(2^k), n_om of them, device).
template <class F>
cudaError_t pow_tables(const u32 *d_omegas, u32 n_om, u32 *d_tab, cudaStream_t st) {
    k_pow_tables<F><<<(3 * TAB + 255) / 256, 256, 0, st>>>(d_omegas, d_tab, n_om);
    return launched("k_pow_tables");
}

template <class F>
cudaError_t ntt_impl(PolyPtr x, const u32 *tw, u32 L, cudaStream_t st) {
    View v;
    if (!make_view(x, v, "ssip_ntt")) return cudaErrorInvalidValue;
    if (L > 31 || x.len != (1ull << L)) {
        set_error("ssip_ntt: len must be 2^log_len (log_len <= 31)");
        return cudaErrorInvalidValue;
    }
    if (L && (!tw || !aligned16(tw))) {
        set_error("ssip_ntt: null or misaligned twiddle table");
        return cudaErrorInvalidValue;
    }
    return run_ntt<F, false>(v, tw, L, st);
}

template <class F>
cudaError_t recompute_impl(PolyPtr x, const u32 *omegas, u32 L, cudaStream_t st) {
    View v;
    if (!make_view(x, v, "recompute_ntt")) return cudaErrorInvalidValue;
    if (L > 31 || x.len != (1ull << L)) {
        set_error("recompute_ntt: len must be 2^log_len (log_len <= 31)");
        return cudaErrorInvalidValue;
    }
    if (L == 0) return cudaSuccess;
    if (!omegas || !aligned16(omegas)) {
        set_error("recompute_ntt: null or misaligned omegas");
        return cudaErrorInvalidValue;
    }
    u32 *tab = nullptr;
    NTT_CK(cudaMallocAsync(&tab, (size_t)3 * TAB * 32, st));
    cudaError_t e = pow_tables<F>(omegas, 32, tab, st);
    if (e == cudaSuccess) e = run_ntt<F, true>(v, tab, L, st);
    cudaError_t f = cudaFreeAsync(tab, st);
    return e != cudaSuccess ? e : f;
}

// Blocking: w^(i * step) for i < count into host memory, w = *unit (host),
// and optionally omegas[0..32) = w^(2^k) into host memory.
template <class F>
cudaError_t host_powers(const u32 *unit, u64 count, u64 step, u32 *h_out, u32 *h_omegas) {
    cudaStream_t st = nullptr;
    NTT_CK(cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking));
    u32 *d = nullptr;
    const size_t tab_b = (size_t)3 * TAB * 32, om_b = 33 * 32;
    cudaError_t e = cudaMalloc(&d, 32 + om_b + tab_b + count * 32);
    if (e == cudaSuccess) {
        u32 *d_unit = d, *d_om = d + 8, *d_tab = d_om + 8 * 33, *d_out = d_tab + 3 * TAB * 8;
        e = cudaMemcpyAsync(d_unit, unit, 32, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess) {
            k_omegas<F><<<1, 1, 0, st>>>(d_unit, d_om, 33);
            e = launched("k_omegas");
        }
        if (e == cudaSuccess) e = pow_tables<F>(d_om, 33, d_tab, st);
        if (e == cudaSuccess && count) {
            const u64 blocks = (count + 255) / 256;
            k_powers<F><<<(unsigned)(blocks < 65535 ? blocks : 65535), 256, 0, st>>>(d_tab, d_out, count, step);
            e = launched("k_powers");
        }
        if (e == cudaSuccess && count) e = cudaMemcpyAsync(h_out, d_out, count * 32, cudaMemcpyDeviceToHost, st);
        if (e == cudaSuccess && h_omegas) e = cudaMemcpyAsync(h_omegas, d_om, 32 * 32, cudaMemcpyDeviceToHost, st);
        cudaError_t s = cudaStreamSynchronize(st);
        if (e == cudaSuccess) e = s;
        cudaFree(d);
    }
    cudaStreamDestroy(st);
    return e;
}

template <class F>
cudaError_t precompute_impl(u32 *twiddle, u32 len, const u32 *unit) {
    if (len == 0) return cudaSuccess;
    if (!twiddle || !unit) {
        set_error("ssip_precompute: null argument");
        return cudaErrorInvalidValue;
    }
    return host_powers<F>(unit, len, 1, twiddle, nullptr);
}

template <class F>
cudaError_t pq_omegas_impl(u32 *pq, u32 *omegas, u32 pq_deg, u32 len, const u32 *unit) {
    if (!pq || !omegas || !unit || pq_deg > 31) {
        set_error("gen_pq_omegas: bad argument");
        return cudaErrorInvalidValue;
    }
    const u64 count = pq_deg ? (1ull << pq_deg) >> 1 : 1;  // pq[0] = 1 is written even for pq_deg = 0
    return host_powers<F>(unit, count, (u64)(len >> pq_deg), pq, omegas);
}

template <class F>
cudaError_t distribute_impl(PolyPtr poly, const u32 *powers, u64 pnum, cudaStream_t st, const PolySlice *ps) {
    View v;
    if (!make_view(poly, v, "distribute_powers")) return cudaErrorInvalidValue;
    if (poly.len == 0) return cudaSuccess;
    if (!powers || !aligned16(powers) || pnum == 0) {
        set_error("distribute_powers: null, misaligned or empty powers");
        return cudaErrorInvalidValue;
    }
    u64 begin = 0, plen = poly.len;
    if (ps) {
        if (ps->len == 0 || ps->slice_len < poly.len) {
            set_error("distribute_powers: poly_slice shorter than the polynomial");
            return cudaErrorInvalidValue;
        }
        begin = ps->begin;
        plen = ps->len;
    }
    const u64 blocks = (poly.len + 255) / 256;
    k_distribute_powers<F><<<(unsigned)(blocks < 148 * 16 ? blocks : 148 * 16), 256, 0, st>>>(v, poly.len, powers,
                                                                                          pnum, begin, plen);
    return launched("k_distribute_powers");
}

#define NTT_FIELD_DISPATCH(field, fn, ...)                                  \
    switch (field) {                                                        \
    case IMPELLER_NTT_BN254_FR: return fn<FrP>(__VA_ARGS__);                \
    case IMPELLER_NTT_BN254_FQ: return fn<FqP>(__VA_ARGS__);                \
    case IMPELLER_NTT_BLS12381_FR: return fn<BlsFrP>(__VA_ARGS__);          \
    default: set_error("unknown NTT field"); return cudaErrorInvalidValue; \
    }

}  // namespace

extern "C" {

cudaError_t impeller_ntt(int field, PolyPtr x, const unsigned int *twiddle, unsigned int log_len,
                         cudaStream_t stream) {
    NTT_FIELD_DISPATCH(field, ntt_impl, x, twiddle, log_len, stream)
}

cudaError_t impeller_ntt_precompute(int field, unsigned int *twiddle, unsigned int len, const unsigned int *unit) {
    NTT_FIELD_DISPATCH(field, precompute_impl, twiddle, len, unit)
}

cudaError_t impeller_ntt_recompute(int field, PolyPtr x, const unsigned int *omegas_d, unsigned int log_len,
                                   cudaStream_t stream) {
    NTT_FIELD_DISPATCH(field, recompute_impl, x, omegas_d, log_len, stream)
}

cudaError_t impeller_ntt_gen_pq_omegas(int field, unsigned int *pq, unsigned int *omegas, unsigned int pq_deg,
                                       unsigned int len, const unsigned int *unit) {
    NTT_FIELD_DISPATCH(field, pq_omegas_impl, pq, omegas, pq_deg, len, unit)
}

cudaError_t impeller_ntt_distribute_powers(int field, PolyPtr poly, const unsigned int *powers,
                                           unsigned long long power_num, cudaStream_t stream,
                                           const PolySlice *poly_slice) {
    NTT_FIELD_DISPATCH(field, distribute_impl, poly, powers, power_num, stream, poly_slice)
}

unsigned int impeller_ntt_launches(unsigned int log_len) {
    if (log_len == 0) return 0;
    return (unsigned)plan_passes(log_len).size() + (log_len > TILE_LOG ? 1u : 0u);
}

// The reference's five symbols, on its default field (BN254 Fr).

cudaError_t ssip_ntt(PolyPtr x, const unsigned int *twiddle, unsigned int log_len, cudaStream_t stream,
                     const unsigned int max_threads_stage1_log, const unsigned int max_threads_stage2_log) {
    if (max_threads_stage1_log > 10 || max_threads_stage2_log > 10) {
        set_error("ssip_ntt: max_threads_*_log must be at most 10");
        return cudaErrorInvalidValue;
    }
    return ntt_impl<FrP>(x, twiddle, log_len, stream);
}

cudaError_t ssip_precompute(unsigned int *twiddle, unsigned int len, const unsigned int *unit) {
    return precompute_impl<FrP>(twiddle, len, unit);
}

cudaError_t recompute_ntt(PolyPtr x, const unsigned int *pq_d, unsigned int pq_deg, const unsigned int *omegas_d,
                          unsigned int log_len, cudaStream_t stream, const unsigned int max_threads_stage1_log,
                          const unsigned int max_threads_stage2_log) {
    if (max_threads_stage1_log > 10 || max_threads_stage2_log > 10 || pq_deg == 0 || !pq_d) {
        set_error("recompute_ntt: bad pq table or launch-shape argument");
        return cudaErrorInvalidValue;
    }
    return recompute_impl<FrP>(x, omegas_d, log_len, stream);
}

void gen_pq_omegas(unsigned int *pq, unsigned int *omegas, unsigned int pq_deg, unsigned int len, unsigned int *unit) {
    (void)pq_omegas_impl<FrP>(pq, omegas, pq_deg, len, unit);
}

cudaError_t distribute_powers(PolyPtr poly, const unsigned int *powers, unsigned long long power_num,
                              cudaStream_t stream, const PolySlice *poly_slice) {
    return distribute_impl<FrP>(poly, powers, power_num, stream, poly_slice);
}

}  // extern "C"
