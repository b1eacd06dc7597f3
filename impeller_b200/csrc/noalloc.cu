// MSM entry point that allocates nothing.
//
// Who needs it: callers that cannot call cudaMalloc when they need an MSM --
// runtimes whose device memory is planned ahead of time into a fixed arena
// (the reference's own compiler assigns every device byte before a proof
// runs), latency-critical paths where cudaMalloc / cudaFree would
// synchronize the device, and processes that must not grow their device
// footprint after start-up.  impeller_msm_device allocates its scratch on
// first use; this variant takes every scratch byte from a file-scope
// __device__ array instead, so a call allocates neither device nor pinned
// host memory, creates no events or streams, and calls no allocating library
// routine.
//
// The array is IMPELLER_NOALLOC_SCRATCH_BYTES (16 MiB) and every GPU that
// loads this library holds it until the process exits.  That bounds one call
// to IMPELLER_NOALLOC_MAX_N = 2^14 points (window 10: 26 digit windows of
// 512 buckets each); larger n is rejected with cudaErrorInvalidValue.
//
// The array is shared by every call on a device and keeps the last call's
// contents: the bucket counters and the heavy-bucket list are cleared at the
// start of every call; everything else is fully rewritten before it is read.
// Calls whose work overlaps on the GPU (different streams, or host threads
// racing) share that one array and race; serialize them (one stream, or
// events between streams).
//
// Set-up: the first call on a device looks up the array's device address
// with cudaGetSymbolAddress (with that device current) and caches it; make
// that first call before any stream capture.  The cached address outlives a
// cudaDeviceReset, which releases the module the array lives in, so a reset
// after the first call is not supported.  The kernels are the engine's
// own (msm_kernels.cuh), compiled into this file under their own namespace.
#include <cstdio>
#include <mutex>
#include <string>

#include "../../include/impeller_msm.h"
#include "bn254.cuh"
#include "engine.h"

namespace noalloc_copy {
#include "msm_kernels.cuh"
}

namespace {

using noalloc_copy::impeller::AccumArgs;
using noalloc_copy::impeller::FinalArgs;
using noalloc_copy::impeller::FixupArgs;
using noalloc_copy::impeller::MsmDesc;
using noalloc_copy::impeller::ReduceArgs;
using noalloc_copy::impeller::WinDesc;
using noalloc_copy::impeller::WindowSumArgs;
namespace K = noalloc_copy::impeller;

typedef uint32_t u32;

constexpr size_t SCRATCH_BYTES = (size_t)IMPELLER_NOALLOC_SCRATCH_BYTES;
constexpr u32 MAX_N = IMPELLER_NOALLOC_MAX_N;
constexpr u32 C = 10;                                  // window bits
constexpr u32 W = (254 + C - 1) / C;                   // 26 digit windows
constexpr u32 B = 1u << (C - 1);                       // 512 buckets per window
constexpr u32 NB = W * B;                              // 13312 buckets
constexpr u32 NB_PAD = (NB + K::SCAN_TILE - 1) / K::SCAN_TILE * K::SCAN_TILE;
constexpr u32 NTILES = NB_PAD / K::SCAN_TILE;
constexpr u32 E_MAX = W * MAX_N;                       // entries
constexpr u32 ACC_BLOCKS = 64, ACC_THREADS = 256, T = ACC_BLOCKS * ACC_THREADS;
constexpr u32 CHUNK = 16;                              // buckets per reduce thread
constexpr u32 RBLOCKS_PER_WIN = (B / CHUNK + K::REDUCE_BLOCK - 1) / K::REDUCE_BLOCK;
constexpr u32 NPARTS_PER_WIN = RBLOCKS_PER_WIN * K::REDUCE_WARPS;
constexpr u32 NPARTS = W * NPARTS_PER_WIN;
constexpr u32 NRBLOCKS = W * RBLOCKS_PER_WIN;

constexpr size_t up(size_t x) { return (x + 255) / 256 * 256; }
constexpr size_t O_DESC = 0;
constexpr size_t O_WINS = O_DESC + up(sizeof(MsmDesc));
constexpr size_t O_RBLK = O_WINS + up(sizeof(WinDesc) * W);
constexpr size_t O_COUNTS = O_RBLK + up(sizeof(uint2) * NRBLOCKS);
constexpr size_t O_CURSOR = O_COUNTS + up((size_t)NB_PAD * 4);
constexpr size_t O_OFFSETS = O_CURSOR + up((size_t)NB * 4);
constexpr size_t O_TILES = O_OFFSETS + up((size_t)(NB + 1) * 4);
constexpr size_t O_ENTRIES = O_TILES + up((size_t)(NTILES + 1) * 4);
constexpr size_t O_BUCKETS = O_ENTRIES + up((size_t)E_MAX * 4);
constexpr size_t O_RECB = O_BUCKETS + up((size_t)NB * 128);
constexpr size_t O_RECP = O_RECB + up((size_t)2 * T * 4);
constexpr size_t O_PARTS_V = O_RECP + up((size_t)2 * T * 128);
constexpr size_t O_PARTS_S = O_PARTS_V + up((size_t)NPARTS * 128);
constexpr size_t O_WRES = O_PARTS_S + up((size_t)NPARTS * 128);
constexpr size_t O_LONG = O_WRES + up((size_t)W * 128);
constexpr size_t O_END = O_LONG + up((size_t)(1 + T) * 4);
static_assert(O_END <= SCRATCH_BYTES, "static MSM scratch too small for IMPELLER_NOALLOC_MAX_N");

// The scratch.  In host code this name is a host-side stand-in, not a device
// address: only the address from cudaGetSymbolAddress is passed to kernels.
static __device__ __align__(256) unsigned char g_scratch[SCRATCH_BYTES];

constexpr int MAX_DEVICES = 64;
std::mutex g_mu;
void *g_addr[MAX_DEVICES] = {};

cudaError_t scratch_address(void **out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= MAX_DEVICES) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> g(g_mu);
    if (!g_addr[dev]) {
        void *p = nullptr;
        e = cudaGetSymbolAddress(&p, g_scratch);
        if (e != cudaSuccess) return e;
        g_addr[dev] = p;
    }
    *out = g_addr[dev];
    return cudaSuccess;
}

// Writes the MSM, window and reduce-block tables of one MSM of n points.
__global__ void k_noalloc_tables(unsigned char *base, const u32 *scalars, u32 n) {
    MsmDesc *d = reinterpret_cast<MsmDesc *>(base + O_DESC);
    WinDesc *w = reinterpret_cast<WinDesc *>(base + O_WINS);
    uint2 *rb = reinterpret_cast<uint2 *>(base + O_RBLK);
    const u32 t = threadIdx.x;
    if (t == 0) {
        d->scalars = scalars;
        d->n = n;
        d->c = C;
        d->n_logical = W;
        d->n_windows = W;
        d->table_stride = 0;
        d->bucket_base = 0;
        d->win_base = 0;
        d->table_base = 0;
        d->entry_base = 0;
    }
    for (u32 i = t; i < W; i += blockDim.x) {
        WinDesc x;
        x.bucket_base = i * B;
        x.nbuckets = B;
        x.chunk = CHUNK;
        x.part_base = i * NPARTS_PER_WIN;
        x.nparts = NPARTS_PER_WIN;
        x.msm = 0;
        x.pad0 = 0;
        x.pad1 = 0;
        w[i] = x;
    }
    for (u32 i = t; i < NRBLOCKS; i += blockDim.x) rb[i] = make_uint2(i / RBLOCKS_PER_WIN, i % RBLOCKS_PER_WIN);
}

cudaError_t fail(cudaError_t e, const char *what) {
    impeller::set_error(std::string("impeller_msm_device_noalloc: ") + what + ": " + cudaGetErrorString(e));
    return e;
}

#define NA_CK(x)                             \
    do {                                     \
        cudaError_t _e = (x);                \
        if (_e != cudaSuccess) return fail(_e, #x); \
    } while (0)

#define NA_LAUNCHED(name)                        \
    do {                                         \
        cudaError_t _e = cudaGetLastError();     \
        if (_e != cudaSuccess) return fail(_e, "launch of " name); \
    } while (0)

}  // namespace

extern "C" cudaError_t impeller_msm_device_noalloc(const uint32_t *d_points, const uint32_t *d_scalars, uint64_t n,
                                                   uint32_t *d_result, cudaStream_t stream) {
    if (!d_result || (n && (!d_points || !d_scalars))) {
        impeller::set_error("impeller_msm_device_noalloc: null argument");
        return cudaErrorInvalidValue;
    }
    if (n > MAX_N) {
        impeller::set_error("impeller_msm_device_noalloc: n exceeds IMPELLER_NOALLOC_MAX_N (2^14) points");
        return cudaErrorInvalidValue;
    }
    if (n == 0) {
        NA_CK(cudaMemsetAsync(d_result, 0, 64, stream));
        return cudaSuccess;
    }
    void *addr = nullptr;
    NA_CK(scratch_address(&addr));
    unsigned char *s = static_cast<unsigned char *>(addr);
    const MsmDesc *desc = reinterpret_cast<const MsmDesc *>(s + O_DESC);
    const WinDesc *wins = reinterpret_cast<const WinDesc *>(s + O_WINS);
    const uint2 *rblk = reinterpret_cast<const uint2 *>(s + O_RBLK);
    u32 *counts = reinterpret_cast<u32 *>(s + O_COUNTS);
    u32 *cursor = reinterpret_cast<u32 *>(s + O_CURSOR);
    u32 *offsets = reinterpret_cast<u32 *>(s + O_OFFSETS);
    u32 *tiles = reinterpret_cast<u32 *>(s + O_TILES);
    u32 *entries = reinterpret_cast<u32 *>(s + O_ENTRIES);
    u32 *buckets = reinterpret_cast<u32 *>(s + O_BUCKETS);
    u32 *recb = reinterpret_cast<u32 *>(s + O_RECB);
    u32 *recp = reinterpret_cast<u32 *>(s + O_RECP);
    u32 *parts_v = reinterpret_cast<u32 *>(s + O_PARTS_V);
    u32 *parts_s = reinterpret_cast<u32 *>(s + O_PARTS_S);
    u32 *wres = reinterpret_cast<u32 *>(s + O_WRES);
    u32 *longl = reinterpret_cast<u32 *>(s + O_LONG);

    k_noalloc_tables<<<1, 64, 0, stream>>>(s, d_scalars, (u32)n);
    NA_LAUNCHED("k_noalloc_tables");
    NA_CK(cudaMemsetAsync(counts, 0, (size_t)NB_PAD * 4, stream));
    const dim3 hgrid((u32)((n + 255) / 256), 1);
    K::k_histogram<K::Bn254><<<hgrid, 256, 0, stream>>>(desc, counts);
    NA_LAUNCHED("k_histogram");
    K::k_scan_reduce<<<NTILES, K::SCAN_BLOCK, 0, stream>>>(counts, tiles);
    NA_LAUNCHED("k_scan_reduce");
    K::k_scan_tiles<<<1, K::SCAN_BLOCK, 0, stream>>>(tiles, NTILES);
    NA_LAUNCHED("k_scan_tiles");
    K::k_scan_down<<<NTILES, K::SCAN_BLOCK, 0, stream>>>(counts, tiles, offsets, cursor, NB, NTILES);
    NA_LAUNCHED("k_scan_down");
    K::k_scatter<K::Bn254><<<hgrid, 256, 0, stream>>>(desc, cursor, entries);
    NA_LAUNCHED("k_scatter");
    AccumArgs aa{entries, offsets, NB, d_points, buckets, recb, recp};
    K::k_accumulate<K::Bn254><<<ACC_BLOCKS, ACC_THREADS, 0, stream>>>(aa);
    NA_LAUNCHED("k_accumulate");
    NA_CK(cudaMemsetAsync(longl, 0, 4, stream));
    FixupArgs fa{offsets, NB, T, recb, recp, buckets, longl, T};
    K::k_fixup_short<K::Bn254><<<T / 256, 256, 0, stream>>>(fa);
    NA_LAUNCHED("k_fixup_short");
    K::k_fixup_long<K::Bn254><<<64, 256, 0, stream>>>(fa, 0u);
    NA_LAUNCHED("k_fixup_long");
    ReduceArgs ra{wins, rblk, offsets, buckets, parts_v, parts_s};
    K::k_reduce<K::Bn254><<<NRBLOCKS, K::REDUCE_BLOCK, 0, stream>>>(ra);
    NA_LAUNCHED("k_reduce");
    WindowSumArgs wa{desc, wins, parts_v, parts_s, W, wres};
    K::k_window_sum<K::Bn254><<<W, K::WSUM_BLOCK, 0, stream>>>(wa);
    NA_LAUNCHED("k_window_sum");
    FinalArgs fin{desc, wres, 1, nullptr, 1, d_result};
    K::k_final<K::Bn254><<<1, 128, 0, stream>>>(fin);
    NA_LAUNCHED("k_final");
    return cudaSuccess;
}
