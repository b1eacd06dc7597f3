// MSM engine: plan layout, launch sequence, resident-SRS contexts, batches.
#include <algorithm>
#include <cmath>
#include <cstring>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

#include "../../include/impeller_msm.h"
#include "engine.h"
#include "msm_kernels.cuh"

namespace impeller {

typedef uint8_t u8;

static thread_local std::string g_err;

void set_error(const std::string &msg) { g_err = msg; }
const char *last_error() { return g_err.c_str(); }

#define CK(x)                                                                                   \
    do {                                                                                        \
        cudaError_t _e = (x);                                                                   \
        if (_e != cudaSuccess) {                                                                \
            set_error(std::string(#x) + " failed: " + cudaGetErrorString(_e));                  \
            return _e;                                                                          \
        }                                                                                       \
    } while (0)

#define CK_LAUNCH(name)                                                                         \
    do {                                                                                        \
        cudaError_t _e = cudaGetLastError();                                                    \
        if (_e != cudaSuccess) {                                                                \
            set_error(std::string("launch of " name " failed: ") + cudaGetErrorString(_e));     \
            return _e;                                                                          \
        }                                                                                       \
    } while (0)

u32 digit_windows(u32 c, u32 curve) {
    if (c < 3 || c > 31) return 0;
    return curve == CURVE_BLS12381 ? Bls12381::windows(c) : Bn254::windows(c);
}

// Launch `kern` instantiated for the plan's curve.
#define CURVE_LAUNCH(curve_id, kern, grid, block, smem, st, ...)                      \
    do {                                                                               \
        if ((curve_id) == CURVE_BLS12381)                                              \
            kern<Bls12381><<<(grid), (block), (smem), (st)>>>(__VA_ARGS__);            \
        else                                                                           \
            kern<Bn254><<<(grid), (block), (smem), (st)>>>(__VA_ARGS__);               \
    } while (0)

int sm_count(int device) {
    static std::mutex mu;
    static std::map<int, int> cache;
    std::lock_guard<std::mutex> g(mu);
    auto it = cache.find(device);
    if (it != cache.end()) return it->second;
    int v = 0;
    if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, device) != cudaSuccess || v <= 0) v = 148;
    cache[device] = v;
    return v;
}

static size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

// The sort-path rule of Plan::build, from the shapes alone.  Each MSM's
// buckets start on a multiple of FINE, so every coarse bin belongs to one
// MSM, and the count matrix holds, per MSM, its bins times its tiles of
// scalars (tiles sized by the most digit windows of any MSM): at most
// SORT_MAX_BINS bins and SORT_MAX_CELLS count cells.
bool Plan::two_level_sort(const std::vector<MsmShape> &shapes) {
    u64 nb = 0;
    u32 wmax = 1;
    for (const MsmShape &s : shapes) {
        if (s.c < 3 || s.c > 31) return false;
        wmax = std::max(wmax, digit_windows(s.c, s.curve));
    }
    const u32 tile = std::max(32u, std::min(1024u, (STAGE_ENTRIES / wmax) & ~31u));
    u64 stiles = 0, cells = 0;
    for (const MsmShape &s : shapes) {
        const u32 W = digit_windows(s.c, s.curve);
        const u32 nw = (s.n_windows == 0 || s.n_windows > W) ? W : s.n_windows;
        nb = align_up(nb, FINE);
        const u64 b0 = nb / FINE;
        nb += (u64)nw << (s.c - 1);
        const u64 tiles = (s.n + tile - 1) / tile;
        stiles += tiles;
        cells += ((nb + FINE - 1) / FINE - b0) * tiles;
    }
    const u64 nbins = (nb + FINE - 1) / FINE;
    return stiles > 0 && nbins <= SORT_MAX_BINS && cells <= SORT_MAX_CELLS;
}

bool Plan::build(Plan &p, int device, const std::vector<MsmShape> &shapes) {
    p.device = device;
    p.shapes = shapes;
    p.M = (u32)shapes.size();
    if (p.M == 0) {
        set_error("plan with no MSMs");
        return false;
    }
    const int sms = sm_count(device);
    p.curve = shapes[0].curve;
    if (p.curve != CURVE_BN254 && p.curve != CURVE_BLS12381) {
        set_error("unknown curve");
        return false;
    }
    for (const MsmShape &sh : shapes)
        if (sh.curve != p.curve) {
            set_error("every MSM of a plan must be on the same curve");
            return false;
        }
    const size_t XB = (size_t)xyzz_words(p.curve) * 4, PB = (size_t)point_words(p.curve) * 4;
    std::vector<MsmDesc> descs(p.M);
    std::vector<WinDesc> wins;
    u64 nb = 0, entries = 0;
    u32 nmax = 0;
    for (u32 m = 0; m < p.M; m++) {
        const MsmShape &s = shapes[m];
        if (s.c < 3 || s.c > 31) {
            set_error("window size must be in [3, 31]");
            return false;
        }
        const u32 W = digit_windows(s.c, p.curve);
        const u32 nw = (s.n_windows == 0 || s.n_windows > W) ? W : s.n_windows;
        const u32 n_tables = (W + nw - 1) / nw;
        const u64 B = 1ull << (s.c - 1);
        const u64 vmax = (u64)s.table_base + (u64)(n_tables - 1) * s.table_stride + s.n;
        if (n_tables > 1 && s.table_stride < s.n) {
            set_error("table stride smaller than the MSM size");
            return false;
        }
        if (vmax >= (1ull << 31)) {
            set_error("point index space (tables x length) exceeds 2^31");
            return false;
        }
        nb = align_up(nb, FINE);  // every coarse bin of the sort belongs to one MSM
        MsmDesc &d = descs[m];
        d.scalars = nullptr;
        d.n = s.n;
        d.c = s.c;
        d.n_logical = W;
        d.n_windows = nw;
        d.table_stride = s.table_stride;
        d.bucket_base = (u32)nb;
        d.win_base = (u32)wins.size();
        d.table_base = s.table_base;
        d.entry_base = (u32)entries;
        for (u32 pw = 0; pw < nw; pw++) {
            WinDesc w{};
            w.bucket_base = (u32)(nb + pw * B);
            w.nbuckets = (u32)B;
            w.msm = m;
            wins.push_back(w);
        }
        nb += nw * B;
        entries += (u64)s.n * W;
        nmax = std::max(nmax, s.n);
        if (nb >= (1ull << 31) || entries >= 0xffffffffull) {
            set_error("batch too large: bucket or entry count exceeds 32-bit indexing");
            return false;
        }
    }
    p.nb = (u32)nb;
    p.nb_pad = (u32)align_up(nb, SCAN_TILE);
    p.ntiles = p.nb_pad / SCAN_TILE;
    p.max_entries = entries;

    // reduce: chunk length L per lane, partial-sum slots per window.  Each
    // lane runs a chain of about 2L + log2 L dependent point additions, the
    // reduction tree after it about 15 per level; L is the smallest power of
    // two that keeps the lanes at most REDUCE_LANES_PER_SM per SM: beyond
    // that the lanes compete for issue slots and the chain length no longer
    // sets the time.
    const u64 target = (u64)sms * REDUCE_LANES_PER_SM;
    u32 L = 1;
    while (nb / L > target && L < (1u << 30)) L <<= 1;
    std::vector<uint2> rblocks;
    u32 nparts = 0;
    for (u32 wi = 0; wi < wins.size(); wi++) {
        WinDesc &w = wins[wi];
        w.chunk = std::min(L, w.nbuckets);
        const u32 nthreads = (w.nbuckets + w.chunk - 1) / w.chunk;
        const u32 nblocks = (nthreads + REDUCE_BLOCK - 1) / REDUCE_BLOCK;
        w.part_base = nparts;
        w.nparts = nblocks * REDUCE_WARPS;  // one partial per reduce warp
        for (u32 k = 0; k < nblocks; k++) rblocks.push_back(make_uint2(wi, k));
        nparts += w.nparts;
    }
    // reduction tree over the reduce warps' partials: levels of groups of
    // 32, appended after the level-1 slots, until each window has one
    std::vector<TreeGroup> groups;
    p.tree_first.assign(1, 0);
    {
        const u32 nw = (u32)wins.size();
        std::vector<u32> base(nw), count(nw), shift(nw);
        std::vector<bool> done(nw, false);
        for (u32 wi = 0; wi < nw; wi++) {
            base[wi] = wins[wi].part_base;
            count[wi] = wins[wi].nparts;
            shift[wi] = 31 - __builtin_clz(wins[wi].chunk) + 5;
        }
        u32 left = nw;
        while (left) {
            for (u32 wi = 0; wi < nw; wi++) {
                if (done[wi]) continue;
                const u32 ng = (count[wi] + 31) / 32;
                for (u32 g = 0; g < ng; g++)
                    groups.push_back(TreeGroup{base[wi] + 32 * g, std::min(32u, count[wi] - 32 * g),
                                               ng == 1 ? (TREE_FINAL | wi) : nparts + g, shift[wi]});
                if (ng == 1) {
                    done[wi] = true;
                    left--;
                } else {
                    base[wi] = nparts;
                    count[wi] = ng;
                    shift[wi] += 5;
                    nparts += ng;
                }
            }
            p.tree_first.push_back((u32)groups.size());
        }
    }
    p.nparts = nparts;
    p.nwins = (u32)wins.size();
    p.nrblocks = (u32)rblocks.size();

    // accumulate: persistent threads (every resident slot), at least 8 entries each
    const bool bls = p.curve == CURVE_BLS12381;
    const u32 accum_threads = bls ? AccumShape<Bls12381>::threads : AccumShape<Bn254>::threads;
    const u32 full_blocks = (u32)sms * (bls ? AccumShape<Bls12381>::per_sm : AccumShape<Bn254>::per_sm);
    const u64 want_threads = (entries + 7) / 8;
    p.accum_blocks =
        (u32)std::max<u64>(1, std::min<u64>(full_blocks, (want_threads + accum_threads - 1) / accum_threads));
    p.accum_block = accum_threads;
    const u32 T = p.accum_blocks * p.accum_block;
    p.long_cap = T;
    p.hist_grid_x = (u32)std::max<u64>(1, std::min<u64>((u64)sms * 8, (nmax + 255) / 256));

    // two-level sort: tiles of scalars small enough to stage all their
    // entries in shared memory, bins of FINE buckets, segments per bin
    u32 wmax = 1;
    for (const MsmDesc &d : descs) wmax = std::max(wmax, d.n_logical);
    p.tile_scalars = std::max(32u, std::min(1024u, (STAGE_ENTRIES / wmax) & ~31u));
    std::vector<u32> tile_first(p.M + 1);
    u64 stiles = 0;
    for (u32 m = 0; m < p.M; m++) {
        tile_first[m] = (u32)stiles;
        stiles += (descs[m].n + p.tile_scalars - 1) / p.tile_scalars;
    }
    tile_first[p.M] = (u32)stiles;
    const u64 nbins = (nb + FINE - 1) / FINE;
    // count cells: per MSM, its bins x its tiles; bin_cell[b] = first cell of bin b
    std::vector<u32> bin_cell;
    u64 cells = 0;
    if (nbins <= SORT_MAX_BINS) {
        bin_cell.assign(nbins + 1, 0);
        for (u32 m = 0; m < p.M; m++) {
            const MsmDesc &d = descs[m];
            const u64 blo = d.bucket_base / FINE;
            const u64 bhi = ((u64)d.bucket_base + ((u64)d.n_windows << (d.c - 1)) - 1) / FINE;
            const u64 tiles = tile_first[m + 1] - tile_first[m];
            for (u64 b = blo; b <= bhi; b++) {
                bin_cell[b] = (u32)std::min<u64>(cells, 0xffffffffu);
                cells += tiles;
            }
        }
        bin_cell[nbins] = (u32)std::min<u64>(cells, 0xffffffffu);
    }
    p.msd = stiles > 0 && nbins <= SORT_MAX_BINS && cells <= SORT_MAX_CELLS;
    if (p.msd) {
        p.nbins = (u32)nbins;
        p.sort_tiles = (u32)stiles;
        p.ncells = (u32)cells;
        p.cnt_pad = (u32)align_up(cells, SCAN_TILE);
        p.cscan_tiles = p.cnt_pad / SCAN_TILE;
        p.segcap = (u32)((entries + SEG_ENTRIES - 1) / SEG_ENTRIES + nbins);
    }

    // host image of the tables
    p.desc_off = 0;
    p.win_off = align_up(sizeof(MsmDesc) * p.M, 16);
    p.blk_off = p.win_off + align_up(sizeof(WinDesc) * wins.size(), 16);
    p.tf_off = p.blk_off + align_up(sizeof(uint2) * rblocks.size(), 16);
    p.bc_off = p.tf_off + align_up(sizeof(u32) * (p.M + 1), 16);
    p.tree_off = p.bc_off + align_up(sizeof(u32) * (p.msd ? p.nbins + 1 : 0), 16);
    const size_t tbytes = align_up(p.tree_off + sizeof(TreeGroup) * groups.size(), 256);
    p.tables.assign(tbytes, 0);
    std::memcpy(p.tables.data() + p.desc_off, descs.data(), sizeof(MsmDesc) * p.M);
    std::memcpy(p.tables.data() + p.win_off, wins.data(), sizeof(WinDesc) * wins.size());
    std::memcpy(p.tables.data() + p.blk_off, rblocks.data(), sizeof(uint2) * rblocks.size());
    std::memcpy(p.tables.data() + p.tf_off, tile_first.data(), sizeof(u32) * (p.M + 1));
    if (p.msd) std::memcpy(p.tables.data() + p.bc_off, bin_cell.data(), sizeof(u32) * (p.nbins + 1));
    std::memcpy(p.tables.data() + p.tree_off, groups.data(), sizeof(TreeGroup) * groups.size());

    // device scratch layout
    PlanLayout &lo = p.layout;
    size_t off = 0;
    auto take = [&](size_t bytes) {
        size_t o = off;
        off = align_up(off + bytes, 256);
        return o;
    };
    lo.o_tables = take(tbytes);
    lo.tables_bytes = tbytes;
    lo.o_counts = take(p.msd ? 0 : (size_t)p.nb_pad * 4);
    lo.o_cursor = take(p.msd ? 0 : (size_t)p.nb * 4);
    lo.o_offsets = take((size_t)(p.nb + 1) * 4);
    lo.o_tiles = take(p.msd ? 0 : (size_t)(p.ntiles + 1) * 4);
    lo.o_entries = take((size_t)std::max<u64>(entries, 1) * 4);
    const size_t ncnt = p.ncells;
    lo.o_cnt = take(p.msd ? (size_t)p.cnt_pad * 4 : 0);
    lo.o_coff = take(p.msd ? (ncnt + 1) * 4 : 0);
    lo.o_ccur = take(p.msd ? ncnt * 4 : 0);
    lo.o_ctiles = take(p.msd ? (size_t)(p.cscan_tiles + 1) * 4 : 0);
    lo.o_centry = take(p.msd ? (size_t)std::max<u64>(entries, 1) * 4 : 0);
    lo.o_cfine = take(p.msd ? (size_t)std::max<u64>(entries, 1) * 2 : 0);
    lo.o_segs = take(p.msd ? (size_t)p.segcap * 16 : 0);
    lo.o_binseg = take(p.msd ? (size_t)p.nbins * 8 : 0);
    lo.o_nsegs = take(p.msd ? 4 : 0);
    lo.o_seghist = take(p.msd ? (size_t)p.segcap * FINE * 4 : 0);
    lo.o_segcur = take(p.msd ? (size_t)p.segcap * FINE * 4 : 0);
    lo.o_buckets = take((size_t)p.nb * XB);
    lo.o_recb = take((size_t)2 * T * 4);
    lo.o_recp = take((size_t)2 * T * XB);
    lo.o_parts = take((size_t)nparts * XB);
    lo.o_parts_s = take((size_t)nparts * XB);
    lo.o_wres = take((size_t)wins.size() * XB);
    lo.o_long = take((size_t)(1 + p.long_cap) * 4);
    lo.o_carry = take((size_t)p.M * XB);
    lo.o_results = take((size_t)p.M * PB);
    lo.bytes = off;
    return true;
}

Plan::~Plan() {
    if (staging && staging != ext_staging) cudaFreeHost(staging);
    if (staged) cudaEventDestroy(staged);
    for (auto &set : prof_sets)
        for (auto e : set) cudaEventDestroy(e);
}

// sort (10 kernels two-level, 6 per-entry) + accumulate, 2 fixups, reduce,
// one per reduction-tree level, final
u32 Plan::launches() const { return (msd ? 10u : 6u) + 5u + (u32)tree_first.size() - 1u; }

const char *Plan::phase_name(int i) {
    static const char *names[NPHASE] = {"tables", "histogram", "scan", "scatter",
                                        "accumulate", "fixup", "reduce", "final"};
    return (i >= 0 && i < NPHASE) ? names[i] : "";
}

cudaError_t Plan::prof_mark(int k, cudaStream_t st) {
    if (!profiling) return cudaSuccess;
    if (k == 0) {
        if (prof_used == prof_sets.size()) {
            std::vector<cudaEvent_t> set(NPHASE + 1);
            for (auto &e : set) CK(cudaEventCreate(&e));
            prof_sets.push_back(set);
        }
        prof_used++;
    }
    CK(cudaEventRecord(prof_sets[prof_used - 1][k], st));
    return cudaSuccess;
}

cudaError_t Plan::read_profile(double *ms, u32 *runs) {
    for (int i = 0; i < NPHASE; i++) ms[i] = 0;
    for (u32 r = 0; r < prof_used; r++) {
        CK(cudaEventSynchronize(prof_sets[r][NPHASE]));
        for (int i = 0; i < NPHASE; i++) {
            float t = 0;
            CK(cudaEventElapsedTime(&t, prof_sets[r][i], prof_sets[r][i + 1]));
            ms[i] += t;
        }
    }
    if (runs) *runs = prof_used;
    prof_used = 0;
    return cudaSuccess;
}

cudaError_t Plan::stage(const u32 *const *scalars) {
    if (ext_staging && ext_cap >= tables.size()) {
        staging = ext_staging;
        if (!staged) CK(cudaEventCreateWithFlags(&staged, cudaEventDisableTiming));
    } else if (!staging) {
        CK(cudaSetDevice(device));
        CK(cudaHostAlloc(&staging, tables.size(), cudaHostAllocPortable));
        CK(cudaEventCreateWithFlags(&staged, cudaEventDisableTiming));
    } else {
        // the previous run's copy of the staging buffer must have finished
        CK(cudaEventSynchronize(staged));
    }
    std::memcpy(staging, tables.data(), tables.size());
    MsmDesc *d = reinterpret_cast<MsmDesc *>(static_cast<unsigned char *>(staging) + desc_off);
    for (u32 m = 0; m < M; m++) d[m].scalars = scalars[m];
    return cudaSuccess;
}

cudaError_t Plan::mark_staged(cudaStream_t st) {
    CK(cudaEventRecord(staged, st));
    return cudaSuccess;
}

// Scratch pointers of one plan.
struct PlanPtrs {
    const MsmDesc *desc;
    const WinDesc *wins;
    const uint2 *blk;
    const u32 *tile_first;
    u32 *counts, *cursor, *offsets, *tiles, *entries, *buckets, *recb, *recp, *parts, *parts_s, *wres, *longl;
    u32 *carry, *res;
};

static PlanPtrs plan_ptrs(const PlanLayout &L, size_t desc_off, size_t win_off, size_t blk_off, size_t tf_off,
                          void *scratch, u32 *carry_ext, u32 *results, const void *d_image = nullptr) {
    unsigned char *s = static_cast<unsigned char *>(scratch);
    const unsigned char *img = d_image ? static_cast<const unsigned char *>(d_image) : s + L.o_tables;
    PlanPtrs p;
    p.desc = reinterpret_cast<const MsmDesc *>(img + desc_off);
    p.wins = reinterpret_cast<const WinDesc *>(img + win_off);
    p.blk = reinterpret_cast<const uint2 *>(img + blk_off);
    p.tile_first = reinterpret_cast<const u32 *>(img + tf_off);
    p.counts = reinterpret_cast<u32 *>(s + L.o_counts);
    p.cursor = reinterpret_cast<u32 *>(s + L.o_cursor);
    p.offsets = reinterpret_cast<u32 *>(s + L.o_offsets);
    p.tiles = reinterpret_cast<u32 *>(s + L.o_tiles);
    p.entries = reinterpret_cast<u32 *>(s + L.o_entries);
    p.buckets = reinterpret_cast<u32 *>(s + L.o_buckets);
    p.recb = reinterpret_cast<u32 *>(s + L.o_recb);
    p.recp = reinterpret_cast<u32 *>(s + L.o_recp);
    p.parts = reinterpret_cast<u32 *>(s + L.o_parts);
    p.parts_s = reinterpret_cast<u32 *>(s + L.o_parts_s);
    p.wres = reinterpret_cast<u32 *>(s + L.o_wres);
    p.longl = reinterpret_cast<u32 *>(s + L.o_long);
    p.carry = carry_ext ? carry_ext : reinterpret_cast<u32 *>(s + L.o_carry);
    p.res = results ? results : reinterpret_cast<u32 *>(s + L.o_results);
    return p;
}

#define MARK(k)                                  \
    if ((pe = prof_mark((k), st)) != cudaSuccess) \
        return pe;

// k_coarse_scatter (kernel 0) and k_seg_scatter (kernel 1) stage entries in
// up to ~200 KB of shared memory: raise their dynamic shared-memory limit
// once per device.
static cudaError_t sort_smem(int device, u32 curve, int kernel, size_t bytes) {
    static std::mutex mu;
    static std::map<std::pair<int, int>, size_t> done;
    std::lock_guard<std::mutex> g(mu);
    size_t &have = done[std::make_pair(device, kernel * 2 + (int)curve)];
    if (have >= bytes) return cudaSuccess;
    const int b = (int)bytes;
    cudaError_t e;
    if (kernel == 1) e = cudaFuncSetAttribute(k_seg_scatter, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    else if (curve == CURVE_BLS12381)
        e = cudaFuncSetAttribute(k_coarse_scatter<Bls12381>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    else e = cudaFuncSetAttribute(k_coarse_scatter<Bn254>, cudaFuncAttributeMaxDynamicSharedMemorySize, b);
    if (e == cudaSuccess) have = bytes;
    return e;
}

// Zero n words at p and m words at q.
__global__ void k_zero_words(u32 *__restrict__ p, u32 n, u32 *__restrict__ q, u32 m) {
    for (u32 i = blockIdx.x * blockDim.x + threadIdx.x; i < n; i += gridDim.x * blockDim.x) p[i] = 0;
    if (blockIdx.x == 0 && threadIdx.x < m) q[threadIdx.x] = 0;
}

// Table image upload (unless the image is already on the device at
// d_image), counting sort, accumulation and fixups: every bucket with
// entries holds its sum in `buckets`.  No copy or memset runs on the stream
// when d_image is given, so nothing here queues behind transfers on a copy
// engine.
cudaError_t Plan::run_front(void *scratch, const u32 *points, cudaStream_t st, bool record_staged,
                            const void *d_image, u32 *bucket_out, cudaEvent_t points_ready) {
    const PlanPtrs p = plan_ptrs(layout, desc_off, win_off, blk_off, tf_off, scratch, nullptr, nullptr, d_image);
    cudaError_t pe;
    MARK(0);
    if (!d_image) {
        CK(cudaMemcpyAsync(static_cast<unsigned char *>(scratch) + layout.o_tables, staging, tables.size(),
                           cudaMemcpyHostToDevice, st));
        if (record_staged) CK(cudaEventRecord(staged, st));
    }
    if (msd) {
        unsigned char *sb = static_cast<unsigned char *>(scratch);
        u32 *cnt = reinterpret_cast<u32 *>(sb + layout.o_cnt);
        u32 *coff = reinterpret_cast<u32 *>(sb + layout.o_coff);
        u32 *ccur = reinterpret_cast<u32 *>(sb + layout.o_ccur);
        u32 *ctiles = reinterpret_cast<u32 *>(sb + layout.o_ctiles);
        const u32 ncnt = ncells;
        const unsigned char *img = d_image ? static_cast<const unsigned char *>(d_image) : sb + layout.o_tables;
        SortArgs sa{p.desc, p.tile_first, reinterpret_cast<const u32 *>(img + bc_off), M, sort_tiles, tile_scalars,
                    nbins, nb, segcap, cnt, coff,
                    reinterpret_cast<u32 *>(sb + layout.o_centry),
                    reinterpret_cast<unsigned short *>(sb + layout.o_cfine),
                    reinterpret_cast<uint4 *>(sb + layout.o_segs), reinterpret_cast<uint2 *>(sb + layout.o_binseg),
                    reinterpret_cast<u32 *>(sb + layout.o_nsegs), reinterpret_cast<u32 *>(sb + layout.o_seghist),
                    reinterpret_cast<u32 *>(sb + layout.o_segcur), p.offsets, p.entries, p.entries};
        // the scan padding of the tile counts and the long-run counter of the fixups
        k_zero_words<<<1, 256, 0, st>>>(cnt + ncnt, cnt_pad - ncnt, p.longl, 1);
        CK_LAUNCH("k_zero_words");
        MARK(1);
        CURVE_LAUNCH(curve, k_coarse_count, sort_tiles, SORT_BLOCK, nbins * 4, st, sa);
        CK_LAUNCH("k_coarse_count");
        MARK(2);
        k_scan_reduce<<<cscan_tiles, SCAN_BLOCK, 0, st>>>(cnt, ctiles);
        CK_LAUNCH("k_scan_reduce");
        k_scan_tiles<<<1, SCAN_BLOCK, 0, st>>>(ctiles, cscan_tiles);
        CK_LAUNCH("k_scan_tiles");
        k_scan_down<<<cscan_tiles, SCAN_BLOCK, 0, st>>>(cnt, ctiles, coff, ccur, ncnt, cscan_tiles);
        CK_LAUNCH("k_scan_down");
        MARK(3);
        const size_t scatter_smem = (size_t)2 * nbins * 4 + (size_t)STAGE_ENTRIES * 6;
        CK(sort_smem(device, curve, 0, scatter_smem));
        CURVE_LAUNCH(curve, k_coarse_scatter, sort_tiles, SORT_BLOCK, scatter_smem, st, sa);
        CK_LAUNCH("k_coarse_scatter");
        k_seg_plan<<<1, FINE_BLOCK, 0, st>>>(sa);
        CK_LAUNCH("k_seg_plan");
        k_seg_hist<<<segcap, FINE_BLOCK, 0, st>>>(sa);
        CK_LAUNCH("k_seg_hist");
        k_bin_scan<<<nbins, FINE_BLOCK, 0, st>>>(sa);
        CK_LAUNCH("k_bin_scan");
        const size_t seg_smem = (size_t)2 * FINE * 4 + (size_t)SEG_ENTRIES * 6;
        CK(sort_smem(device, curve, 1, seg_smem));
        k_seg_scatter<<<segcap, FINE_BLOCK, seg_smem, st>>>(sa);
        CK_LAUNCH("k_seg_scatter");
        MARK(4);
    } else {
        // the bucket counts and the long-run counter of the fixups
        k_zero_words<<<std::max(1u, std::min((nb_pad + 255) / 256, (u32)sm_count(device) * 4)), 256, 0, st>>>(
            p.counts, nb_pad, p.longl, 1);
        CK_LAUNCH("k_zero_words");
        MARK(1);

        dim3 hgrid(hist_grid_x, M);
        CURVE_LAUNCH(curve, k_histogram, hgrid, 256, 0, st, p.desc, p.counts);
        CK_LAUNCH("k_histogram");
        MARK(2);
        k_scan_reduce<<<ntiles, SCAN_BLOCK, 0, st>>>(p.counts, p.tiles);
        CK_LAUNCH("k_scan_reduce");
        k_scan_tiles<<<1, SCAN_BLOCK, 0, st>>>(p.tiles, ntiles);
        CK_LAUNCH("k_scan_tiles");
        k_scan_down<<<ntiles, SCAN_BLOCK, 0, st>>>(p.counts, p.tiles, p.offsets, p.cursor, nb, ntiles);
        CK_LAUNCH("k_scan_down");
        MARK(3);
        CURVE_LAUNCH(curve, k_scatter, hgrid, 256, 0, st, p.desc, p.cursor, p.entries);
        CK_LAUNCH("k_scatter");
        MARK(4);
    }

    if (points_ready) CK(cudaStreamWaitEvent(st, points_ready, 0));
    u32 *const buckets = bucket_out ? bucket_out : p.buckets;
    AccumArgs aa{p.entries, p.offsets, nb, points, buckets, p.recb, p.recp};
    if (bucket_out) {
        if (curve == CURVE_BLS12381) k_accumulate<Bls12381, START_CARRY><<<accum_blocks, accum_block, 0, st>>>(aa);
        else k_accumulate<Bn254, START_CARRY><<<accum_blocks, accum_block, 0, st>>>(aa);
    } else if (curve == CURVE_BLS12381) {
        k_accumulate<Bls12381, ACCUM_START_BLS><<<accum_blocks, accum_block, 0, st>>>(aa);
    } else {
        k_accumulate<Bn254, START_CONVERT><<<accum_blocks, accum_block, 0, st>>>(aa);
    }
    CK_LAUNCH("k_accumulate");
    MARK(5);

    const u32 T = accum_blocks * accum_block;
    FixupArgs fa{p.offsets, nb, T, p.recb, p.recp, buckets, p.longl, long_cap, FIXUP_WARP_MAX};
    CURVE_LAUNCH(curve, k_fixup_short, (T + 255) / 256, 256, 0, st, fa);
    CK_LAUNCH("k_fixup_short");
    const u32 wide_blocks = (u32)sm_count(device);
    CURVE_LAUNCH(curve, k_fixup_long, wide_blocks + (u32)sm_count(device) * 2, WIDE_BLOCK, 0, st, fa, wide_blocks);
    CK_LAUNCH("k_fixup_long");
    MARK(6);
    return cudaSuccess;
}

// Bucket reduction, window sums, Horner combine and affine output, over
// `buckets` (the plan's own, sparse by offsets, or dense accumulators).
cudaError_t Plan::run_tail(void *scratch, const u32 *buckets, bool dense, u32 *results, int carry_mode,
                           cudaStream_t st, u32 *carry_ext, const void *d_image) {
    const PlanPtrs p = plan_ptrs(layout, desc_off, win_off, blk_off, tf_off, scratch, carry_ext, results, d_image);
    cudaError_t pe;
    ReduceArgs ra{p.wins, p.blk, p.offsets, buckets, p.parts, p.parts_s, dense ? 1u : 0u};
    CURVE_LAUNCH(curve, k_reduce, nrblocks, REDUCE_BLOCK, 0, st, ra);
    CK_LAUNCH("k_reduce");
    MARK(7);

    const unsigned char *img = d_image ? static_cast<const unsigned char *>(d_image)
                                       : static_cast<const unsigned char *>(scratch) + layout.o_tables;
    const TreeGroup *groups = reinterpret_cast<const TreeGroup *>(img + tree_off);
    for (size_t lv = 0; lv + 1 < tree_first.size(); lv++) {
        const u32 cnt = tree_first[lv + 1] - tree_first[lv];
        TreeArgs ta{groups + tree_first[lv], cnt, p.parts, p.parts_s, p.wres};
        CURVE_LAUNCH(curve, k_reduce_tree, (cnt + TREE_WARPS - 1) / TREE_WARPS, TREE_BLOCK, 0, st, ta);
        CK_LAUNCH("k_reduce_tree");
    }
    FinalArgs fa2{p.desc, p.wres, M, carry_mode == 0 ? nullptr : p.carry, carry_mode == 2 ? 0 : 1, p.res};
    CURVE_LAUNCH(curve, k_final, (M + 31) / 32, 32, 0, st, fa2);
    CK_LAUNCH("k_final");
    MARK(8);
    return cudaSuccess;
}
#undef MARK

cudaError_t Plan::launch(void *scratch, const u32 *points, u32 *results, int carry_mode, cudaStream_t st,
                         u32 *carry_ext, bool record_staged) {
    cudaError_t e = run_front(scratch, points, st, record_staged, nullptr);
    if (e != cudaSuccess) return e;
    const u32 *buckets = reinterpret_cast<const u32 *>(static_cast<unsigned char *>(scratch) + layout.o_buckets);
    return run_tail(scratch, buckets, false, results, carry_mode, st, carry_ext, nullptr);
}

size_t Plan::image_bytes() const { return tables.size(); }

void Plan::write_image(void *dst, const u32 *const *scalars) const {
    std::memcpy(dst, tables.data(), tables.size());
    MsmDesc *d = reinterpret_cast<MsmDesc *>(static_cast<unsigned char *>(dst) + desc_off);
    for (u32 m = 0; m < M; m++) d[m].scalars = scalars[m];
}

cudaError_t Plan::launch_chunk(void *scratch, const u32 *points, u32 *acc, bool first, cudaStream_t st,
                               const void *d_image, cudaEvent_t points_ready) {
    if (first) {
        // every accumulator starts as the identity (all-zero XYZZ)
        const u64 words = (u64)nb * xyzz_words(curve);
        if (words >= (1ull << 32)) {
            set_error("bucket accumulators exceed 2^32 words");
            return cudaErrorInvalidValue;
        }
        k_zero_words<<<std::max(1u, std::min((u32)((words + 255) / 256), (u32)sm_count(device) * 8)), 256, 0, st>>>(
            acc, (u32)words, nullptr, 0);
        CK_LAUNCH("k_zero_words");
    }
    return run_front(scratch, points, st, true, d_image, acc, points_ready);
}

cudaError_t Plan::launch_chunked_tail(void *scratch, const u32 *acc, u32 *results, int carry_mode, cudaStream_t st,
                                      u32 *carry_ext, const void *d_image) {
    return run_tail(scratch, acc, true, results, carry_mode, st, carry_ext, d_image);
}

cudaError_t Plan::enqueue(void *scratch, const u32 *points, const u32 *const *scalars, u32 *results, int carry_mode,
                          cudaStream_t stream, u32 *carry_ext) {
    cudaError_t e = stage(scalars);
    if (e != cudaSuccess) return e;
    return launch(scratch, points, results, carry_mode, stream, carry_ext);
}

u32 *Plan::carry_ptr(void *scratch) const {
    return reinterpret_cast<u32 *>(static_cast<unsigned char *>(scratch) + layout.o_carry);
}

u32 *Plan::results_ptr(void *scratch) const {
    return reinterpret_cast<u32 *>(static_cast<unsigned char *>(scratch) + layout.o_results);
}

cudaError_t combine_xyzz(const u32 *d_xyzz, u32 k, u32 *d_out, cudaStream_t stream, u32 curve) {
    CURVE_LAUNCH(curve, k_combine, 1, 32, 0, stream, d_xyzz, k, d_out);
    CK_LAUNCH("k_combine");
    return cudaSuccess;
}

template <class C>
__global__ void k_precompute(u32 *points, u64 n, u32 shift, u32 n_tables) {
    using FQ = typename C::Fq;
    const u64 i = (u64)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    XyzzT<FQ> p = xyzz_from_affine(affine_load<FQ>(points + i * C::PW));
    for (u32 j = 1; j < n_tables; j++) {
        for (u32 k = 0; k < shift; k++) p = xyzz_dbl(p);
        affine_store(points + ((u64)j * n + i) * C::PW, xyzz_to_affine(p));
    }
}

cudaError_t precompute_tables(u32 *d_points, u64 n, u32 shift, u32 n_tables, cudaStream_t stream, u32 curve) {
    if (n == 0 || n_tables <= 1) return cudaSuccess;
    CURVE_LAUNCH(curve, k_precompute, (u32)((n + 127) / 128), 128, 0, stream, d_points, n, shift, n_tables);
    CK_LAUNCH("k_precompute");
    return cudaSuccess;
}

// ------------------------------------------------------------ window table

struct WindowEntry {
    u32 log2n, c, tables_c;  // best plain window; tables window (0: plain is faster)
};

static const WindowEntry k_default_table[] = {
#include "autotune_default.inc"
    {0u, 0u, 0u}};

static std::mutex g_tab_mu;
static std::vector<WindowEntry> g_window_table = [] {
    std::vector<WindowEntry> t;
    for (const WindowEntry &e : k_default_table)
        if (e.c) t.push_back(e);
    return t;
}();

// Cost model used when no measured table is loaded: W(c) windows of n
// mixed additions (10 Fq products each) plus the bucket reduction of
// W(c) * 2^(c-1) buckets (two full additions, about 45 products with the
// per-thread overhead of the chunked running sum).
static u32 model_window(u64 n) {
    u32 best = 8;
    double best_cost = 1e300;
    for (u32 c = 4; c <= 22; c++) {
        double W = digit_windows(c);
        double cost = W * ((double)n * 10.0 + std::ldexp(1.0, (int)c - 1) * 45.0);
        if (cost < best_cost) {
            best_cost = cost;
            best = c;
        }
    }
    return best;
}

static const WindowEntry *nearest_entry(u64 n) {
    if (g_window_table.empty()) return nullptr;
    const double lg = std::log2((double)n);
    const WindowEntry *best = &g_window_table[0];
    double bd = 1e300;
    for (const WindowEntry &e : g_window_table) {
        double dd = std::fabs(lg - (double)e.log2n);
        if (dd < bd) {
            bd = dd;
            best = &e;
        }
    }
    return best;
}

u32 default_window(u64 n) {
    if (n == 0) return 0;
    std::lock_guard<std::mutex> g(g_tab_mu);
    const WindowEntry *e = nearest_entry(n);
    return e ? e->c : model_window(n);
}

// The measured window table is BN254's.  On BLS12-381 (255-bit scalars) the
// windows c = 3, 5, 15, 17 need one more signed-digit window whose digits
// are only the carries out of the window below: every scalar lands in one
// bucket of that window.  Move such a choice to the neighbouring window
// without the extra one (16 for 15 and 17, which has no more windows).
u32 curve_window(u32 c, u32 curve) {
    if (curve != CURVE_BLS12381 || c < 3 || c > 31) return c;
    if (digit_windows(c, curve) == (255u + c - 1u) / c) return c;
    return c < 16 ? c + 1 : c - 1;
}

// Window of the resident tables the table recommends for MSMs of n points
// (0: plain windows are faster at that size).
u32 table_window(u64 n) {
    if (n == 0) return 0;
    std::lock_guard<std::mutex> g(g_tab_mu);
    const WindowEntry *e = nearest_entry(n);
    return e ? e->tables_c : 0;
}

}  // namespace impeller

using namespace impeller;

// -------------------------------------------------------------- contexts


u32 impeller::ctx_set_base(const impeller_ctx *ctx, u32 c) {
    for (auto &s : ctx->sets)
        if (s.first == c) return s.second;
    return NONE;
}

// With resident tables the context uses them for the sizes whose best
// (measured) tables window is one of the sets it holds; other sizes run plain.
u32 impeller::ctx_window(const impeller_ctx *ctx, u64 n) {
    const u32 ct = table_window(n);
    if (ct && ctx_set_base(ctx, ct) != NONE) return ct;
    return curve_window(default_window(n), ctx->curve);
}

static cudaError_t ctx_reserve(impeller_ctx *ctx, size_t bytes, cudaStream_t st) {
    if (bytes <= ctx->scratch_bytes) return cudaSuccess;
    CK(cudaStreamSynchronize(st));
    CK(cudaEventSynchronize(ctx->done));
    if (ctx->scratch) CK(cudaFree(ctx->scratch));
    ctx->scratch = nullptr;
    ctx->scratch_bytes = 0;
    CK(cudaMalloc(&ctx->scratch, bytes));
    ctx->scratch_bytes = bytes;
    return cudaSuccess;
}

// Shape of an MSM of n points with window c on this context: with a resident
// table set for c every digit window shares one bucket set.
MsmShape impeller::ctx_shape(const impeller_ctx *ctx, u32 n, u32 c) {
    const u32 base = ctx_set_base(ctx, c);
    if (base != NONE) return MsmShape{n, c, 1, (u32)ctx->len, base, ctx->curve};
    return MsmShape{n, c, 0, 0, 0, ctx->curve};
}

const u32 *impeller::ctx_point_base(const impeller_ctx *ctx) { return ctx->tables ? ctx->tables : ctx->points; }

static Plan *ctx_plan(impeller_ctx *ctx, u32 n, u32 c) {
    auto key = std::make_pair(n, c);
    auto it = ctx->plans.find(key);
    if (it != ctx->plans.end()) return it->second.get();
    std::unique_ptr<Plan> p(new Plan());
    if (!Plan::build(*p, ctx->device, {ctx_shape(ctx, n, c)})) return nullptr;
    Plan *raw = p.get();
    raw->set_profiling(ctx->profiling);
    ctx->plans[key] = std::move(p);
    return raw;
}

extern "C" {

const char *impeller_last_error(void) { return impeller::last_error(); }

const char *impeller_version(void) { return "impeller-b200-msm 0.1 (sm_100a)"; }

unsigned int impeller_default_window(uint64_t n) { return impeller::default_window(n); }

unsigned int impeller_default_window_curve(uint64_t n, unsigned int curve) {
    return impeller::curve_window(impeller::default_window(n), curve);
}

unsigned int impeller_table_window(uint64_t n) { return impeller::table_window(n); }

cudaError_t impeller_set_window_table(const uint32_t *log2n, const uint32_t *c, const uint32_t *tables_c,
                                      uint32_t count) {
    std::vector<WindowEntry> t;
    for (u32 i = 0; i < count; i++) {
        const u32 ct = tables_c ? tables_c[i] : 0;
        if (c[i] < 3 || c[i] > 31 || (ct && (ct < 3 || ct > 31))) {
            set_error("window table entry outside [3, 31]");
            return cudaErrorInvalidValue;
        }
        t.push_back(WindowEntry{log2n[i], c[i], ct});
    }
    std::lock_guard<std::mutex> g(g_tab_mu);
    g_window_table = t;
    return cudaSuccess;
}

cudaError_t impeller_ctx_create(impeller_ctx **out, int device, const uint32_t *points, uint64_t len,
                                int points_on_device) {
    return impeller_ctx_create_curve(out, device, points, len, points_on_device, CURVE_BN254);
}

cudaError_t impeller_ctx_create_curve(impeller_ctx **out, int device, const uint32_t *points, uint64_t len,
                                      int points_on_device, unsigned int curve) {
    if (!out || (!points && len)) {
        set_error("impeller_ctx_create: null argument");
        return cudaErrorInvalidValue;
    }
    if (curve != CURVE_BN254 && curve != CURVE_BLS12381) {
        set_error("impeller_ctx_create: unknown curve");
        return cudaErrorInvalidValue;
    }
    const u64 PB = (u64)point_words(curve) * 4;
    if (len >= (1ull << 31)) {
        set_error("impeller_ctx_create: at most 2^31 - 1 points");
        return cudaErrorInvalidValue;
    }
    std::unique_ptr<impeller_ctx> ctx(new impeller_ctx());
    ctx->device = device;
    ctx->curve = curve;
    ctx->len = len;
    CK(cudaSetDevice(device));
    CK(cudaEventCreateWithFlags(&ctx->done, cudaEventDisableTiming));
    if (points_on_device) {
        ctx->points = points;
    } else {
        u32 *d = nullptr;
        CK(cudaMalloc(&d, std::max<u64>(len, 1) * PB));
        cudaError_t e = cudaMemcpy(d, points, len * PB, cudaMemcpyHostToDevice);
        if (e != cudaSuccess) {
            cudaFree(d);
            set_error(std::string("impeller_ctx_create: upload failed: ") + cudaGetErrorString(e));
            return e;
        }
        ctx->points = d;
        ctx->owns = true;
    }
    CK(cudaMalloc(&ctx->d_result, PB));
    *out = ctx.release();
    return cudaSuccess;
}

cudaError_t impeller_ctx_destroy(impeller_ctx *ctx) {
    if (!ctx) return cudaSuccess;
    cudaSetDevice(ctx->device);
    cudaDeviceSynchronize();
    if (ctx->owns) cudaFree(const_cast<u32 *>(ctx->points));
    if (ctx->tables) cudaFree(ctx->tables);
    if (ctx->scratch) cudaFree(ctx->scratch);
    if (ctx->d_scalars) cudaFree(ctx->d_scalars);
    if (ctx->d_result) cudaFree(ctx->d_result);
    if (ctx->done) cudaEventDestroy(ctx->done);
    ctx->plans.clear();
    delete ctx;
    return cudaSuccess;
}

const uint32_t *impeller_ctx_points(const impeller_ctx *ctx) { return ctx ? ctx->points : nullptr; }

cudaError_t impeller_ctx_precompute(impeller_ctx *ctx, unsigned int c) {
    if (!ctx || c < 3 || c > 31) {
        set_error("impeller_ctx_precompute: window size must be in [3, 31]");
        return cudaErrorInvalidValue;
    }
    std::lock_guard<std::mutex> g(ctx->mu);
    if (ctx_set_base(ctx, c) != NONE) return cudaSuccess;
    CK(cudaSetDevice(ctx->device));
    CK(cudaDeviceSynchronize());
    const u32 W = digit_windows(c, ctx->curve);
    const u64 PB = (u64)point_words(ctx->curve) * 4, PW = point_words(ctx->curve);
    const u64 have = ctx->tables ? ctx->tables_points : ctx->len;  // region 0 = the points
    const u64 total = have + (u64)W * ctx->len;
    if (total >= (1ull << 31)) {
        set_error("impeller_ctx_precompute: points and window tables exceed 2^31 points");
        return cudaErrorInvalidValue;
    }
    u32 *t = nullptr;
    CK(cudaMalloc(&t, (size_t)std::max<u64>(total, 1) * PB));
    const u32 *src = ctx->tables ? ctx->tables : ctx->points;
    cudaError_t e = cudaMemcpy(t, src, have * PB, cudaMemcpyDeviceToDevice);
    u32 *set = t + (size_t)have * PW;
    if (e == cudaSuccess) e = cudaMemcpy(set, ctx->points, ctx->len * PB, cudaMemcpyDeviceToDevice);
    if (e == cudaSuccess) e = precompute_tables(set, ctx->len, c, W, 0, ctx->curve);
    if (e == cudaSuccess) e = cudaDeviceSynchronize();
    if (e != cudaSuccess) {
        cudaFree(t);
        set_error(std::string("impeller_ctx_precompute: ") + cudaGetErrorString(e));
        return e;
    }
    if (ctx->tables) cudaFree(ctx->tables);
    ctx->tables = t;
    ctx->tables_points = total;
    ctx->sets.emplace_back(c, (u32)have);
    ctx->plans.clear();
    return cudaSuccess;
}

unsigned int impeller_ctx_window(const impeller_ctx *ctx, uint64_t n) { return ctx ? ctx_window(ctx, n) : 0; }
uint64_t impeller_ctx_len(const impeller_ctx *ctx) { return ctx ? ctx->len : 0; }

static cudaError_t ctx_run_locked(impeller_ctx *ctx, const uint32_t *d_scalars, uint64_t n, unsigned int c,
                                  uint32_t *d_result, cudaStream_t stream) {
    if (n > ctx->len) {
        set_error("MSM larger than the resident point array");
        return cudaErrorInvalidValue;
    }
    if (n == 0) return cudaMemsetAsync(d_result, 0, (size_t)point_words(ctx->curve) * 4, stream);
    if (c == 0) c = ctx_window(ctx, n);
    CK(cudaSetDevice(ctx->device));
    Plan *p = ctx_plan(ctx, (u32)n, c);
    if (!p) return cudaErrorInvalidValue;
    cudaError_t e = ctx_reserve(ctx, p->scratch_bytes(), stream);
    if (e != cudaSuccess) return e;
    CK(cudaStreamWaitEvent(stream, ctx->done, 0));
    const u32 *sc[1] = {d_scalars};
    e = p->enqueue(ctx->scratch, ctx_point_base(ctx), sc, d_result, 0, stream);
    if (e != cudaSuccess) return e;
    CK(cudaEventRecord(ctx->done, stream));
    return cudaSuccess;
}

cudaError_t impeller_msm_device(impeller_ctx *ctx, const uint32_t *d_scalars, uint64_t n, unsigned int c,
                                uint32_t *d_result, cudaStream_t stream) {
    if (!ctx || (!d_scalars && n) || !d_result) {
        set_error("impeller_msm_device: null argument");
        return cudaErrorInvalidValue;
    }
    std::lock_guard<std::mutex> g(ctx->mu);
    return ctx_run_locked(ctx, d_scalars, n, c, d_result, stream);
}

cudaError_t impeller_msm_host(impeller_ctx *ctx, const uint32_t *h_scalars, uint64_t n, unsigned int c,
                              uint32_t *h_result, cudaStream_t stream) {
    if (!ctx || (!h_scalars && n) || !h_result) {
        set_error("impeller_msm_host: null argument");
        return cudaErrorInvalidValue;
    }
    std::lock_guard<std::mutex> g(ctx->mu);
    CK(cudaSetDevice(ctx->device));
    if (n > ctx->d_scalars_cap) {
        CK(cudaStreamSynchronize(stream));
        CK(cudaEventSynchronize(ctx->done));
        if (ctx->d_scalars) CK(cudaFree(ctx->d_scalars));
        ctx->d_scalars = nullptr;
        ctx->d_scalars_cap = 0;
        CK(cudaMalloc(&ctx->d_scalars, n * 32));
        ctx->d_scalars_cap = n;
    }
    // the previous run read d_scalars: order the copy after it
    CK(cudaStreamWaitEvent(stream, ctx->done, 0));
    if (n) CK(cudaMemcpyAsync(ctx->d_scalars, h_scalars, n * 32, cudaMemcpyHostToDevice, stream));
    cudaError_t e = ctx_run_locked(ctx, ctx->d_scalars, n, c, ctx->d_result, stream);
    if (e != cudaSuccess) return e;
    CK(cudaMemcpyAsync(h_result, ctx->d_result, (size_t)point_words(ctx->curve) * 4, cudaMemcpyDeviceToHost,
                       stream));
    CK(cudaStreamSynchronize(stream));
    return cudaSuccess;
}

cudaError_t impeller_ctx_profile(impeller_ctx *ctx, int enable) {
    if (!ctx) return cudaErrorInvalidValue;
    std::lock_guard<std::mutex> g(ctx->mu);
    ctx->profiling = enable != 0;
    for (auto &kv : ctx->plans) kv.second->set_profiling(ctx->profiling);
    return cudaSuccess;
}

cudaError_t impeller_ctx_profile_read(impeller_ctx *ctx, double *ms_per_phase, uint32_t nphase, uint32_t *runs) {
    if (!ctx || !ms_per_phase || nphase < (u32)Plan::NPHASE) {
        set_error("impeller_ctx_profile_read: need room for every phase");
        return cudaErrorInvalidValue;
    }
    std::lock_guard<std::mutex> g(ctx->mu);
    for (u32 i = 0; i < nphase; i++) ms_per_phase[i] = 0;
    u32 total = 0;
    for (auto &kv : ctx->plans) {
        double ms[Plan::NPHASE];
        u32 r = 0;
        cudaError_t e = kv.second->read_profile(ms, &r);
        if (e != cudaSuccess) return e;
        for (int i = 0; i < Plan::NPHASE; i++) ms_per_phase[i] += ms[i];
        total += r;
    }
    if (runs) *runs = total;
    return cudaSuccess;
}

const char *impeller_phase_name(uint32_t i) { return Plan::phase_name((int)i); }

uint32_t impeller_ctx_launches(impeller_ctx *ctx, uint64_t n, unsigned int c) {
    if (!ctx || n == 0 || n > ctx->len) return 0;
    std::lock_guard<std::mutex> g(ctx->mu);
    if (c == 0) c = ctx_window(ctx, n);
    Plan *p = ctx_plan(ctx, (u32)n, c);
    return p ? p->launches() : 0;
}

// ---------------------------------------------------------------- batches

}  // extern "C"

struct impeller_batch {
    impeller_ctx *ctx = nullptr;
    Plan plan;
    void *scratch = nullptr;
    bool graph = false;
    cudaGraph_t g = nullptr;
    cudaGraphExec_t exec = nullptr;
    cudaStream_t cap_stream = nullptr;
};

extern "C" {

cudaError_t impeller_batch_create(impeller_batch **out, impeller_ctx *ctx, const uint64_t *sizes,
                                  const unsigned int *windows, uint32_t count, uint32_t flags) {
    if (!out || !ctx || !sizes || count == 0) {
        set_error("impeller_batch_create: bad argument");
        return cudaErrorInvalidValue;
    }
    std::vector<MsmShape> shapes;
    for (u32 i = 0; i < count; i++) {
        if (sizes[i] > ctx->len || sizes[i] == 0) {
            set_error("impeller_batch_create: size 0 or larger than the resident point array");
            return cudaErrorInvalidValue;
        }
        u32 c = windows && windows[i] ? windows[i] : ctx_window(ctx, sizes[i]);
        shapes.push_back(ctx_shape(ctx, (u32)sizes[i], c));
    }
    std::unique_ptr<impeller_batch> b(new impeller_batch());
    b->ctx = ctx;
    if (!Plan::build(b->plan, ctx->device, shapes)) return cudaErrorInvalidValue;
    CK(cudaSetDevice(ctx->device));
    CK(cudaMalloc(&b->scratch, b->plan.scratch_bytes()));
    b->graph = (flags & IMPELLER_BATCH_GRAPH) != 0;
    *out = b.release();
    return cudaSuccess;
}

cudaError_t impeller_batch_destroy(impeller_batch *b) {
    if (!b) return cudaSuccess;
    cudaSetDevice(b->ctx->device);
    cudaDeviceSynchronize();
    if (b->exec) cudaGraphExecDestroy(b->exec);
    if (b->g) cudaGraphDestroy(b->g);
    if (b->cap_stream) cudaStreamDestroy(b->cap_stream);
    if (b->scratch) cudaFree(b->scratch);
    delete b;
    return cudaSuccess;
}

uint32_t impeller_batch_launches(const impeller_batch *b) { return b ? b->plan.launches() : 0; }

cudaError_t impeller_batch_profile(impeller_batch *b, int enable) {
    if (!b || (enable && b->graph)) {
        set_error("impeller_batch_profile: needs a batch created without IMPELLER_BATCH_GRAPH");
        return cudaErrorInvalidValue;
    }
    b->plan.set_profiling(enable != 0);
    return cudaSuccess;
}

cudaError_t impeller_batch_profile_read(impeller_batch *b, double *ms_per_phase, uint32_t nphase, uint32_t *runs) {
    if (!b || !ms_per_phase || nphase < (u32)Plan::NPHASE) {
        set_error("impeller_batch_profile_read: need room for every phase");
        return cudaErrorInvalidValue;
    }
    for (u32 i = 0; i < nphase; i++) ms_per_phase[i] = 0;
    return b->plan.read_profile(ms_per_phase, runs);
}

cudaError_t impeller_batch_run(impeller_batch *b, const uint32_t *const *d_scalars, uint32_t *d_results,
                               cudaStream_t stream) {
    if (!b || !d_scalars || !d_results) {
        set_error("impeller_batch_run: null argument");
        return cudaErrorInvalidValue;
    }
    CK(cudaSetDevice(b->ctx->device));
    cudaError_t e = b->plan.stage(d_scalars);
    if (e != cudaSuccess) return e;
    if (!b->graph) {
        e = b->plan.launch(b->scratch, ctx_point_base(b->ctx), nullptr, 0, stream);
        if (e != cudaSuccess) return e;
    } else {
        if (!b->exec) {
            CK(cudaStreamCreateWithFlags(&b->cap_stream, cudaStreamNonBlocking));
            CK(cudaStreamBeginCapture(b->cap_stream, cudaStreamCaptureModeThreadLocal));
            e = b->plan.launch(b->scratch, ctx_point_base(b->ctx), nullptr, 0, b->cap_stream, nullptr, false);
            cudaGraph_t g = nullptr;
            cudaError_t e2 = cudaStreamEndCapture(b->cap_stream, &g);
            if (e != cudaSuccess) return e;
            CK(e2);
            b->g = g;
            CK(cudaGraphInstantiate(&b->exec, g, 0));
        }
        CK(cudaGraphLaunch(b->exec, stream));
        e = b->plan.mark_staged(stream);
        if (e != cudaSuccess) return e;
    }
    CK(cudaMemcpyAsync(d_results, b->plan.results_ptr(b->scratch), (size_t)b->plan.M * point_words(b->plan.curve) * 4,
                       cudaMemcpyDeviceToDevice,
                       stream));
    return cudaSuccess;
}

}  // extern "C"
