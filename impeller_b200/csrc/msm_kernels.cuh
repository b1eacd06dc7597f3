// Pippenger MSM kernels for BN254 G1 on sm_100a.
//
// One pass over a batch of M MSMs that share one device-resident point array:
//
//   k_histogram   scalar (Montgomery Fr) -> canonical -> signed c-bit digits;
//                 count entries per bucket                      [HBM-bound]
//   k_scan_*      exclusive scan of the bucket counts -> bucket offsets
//   k_scatter     same digits; place (point index, sign) of every nonzero
//                 digit into its bucket's slice of `entries`     [HBM-bound]
//   k_accumulate  persistent threads walk equal slices of `entries`, one
//                 XYZZ += affine (madd-2008-s) per entry; buckets that fit in
//                 one slice are written directly, buckets cut by a slice
//                 boundary leave partial sums                  [IMAD-bound]
//   k_fixup_*     merge the partial sums of cut buckets (short runs per
//                 thread, long runs -- heavy buckets -- per warp)
//   k_reduce      per window sum_k k * S_k by chunked running sums whose
//                 cross-chunk weights come from a suffix scan
//   k_window_sum  per window (one warp): finish the window total, weight it
//                 by 2^(c * window)
//   k_final       per MSM (one warp): sum the windows, affine conversion
//
// Differences from the reference (core/src/msm/src/msm_impl.cuh): the
// reference sorts 64-bit keys with CUB radix sort (:459-463), protects the
// first bucket of each thread slice with a spin mutex (:73-105, :189-204),
// finishes the sum of the reduce blocks and the affine conversion on the host
// (:716-733, core/src/msm/src/msm.cu:37-39).  Here the sort is a counting
// sort by bucket, cut buckets are merged without locks, and every step up to
// the canonical affine result runs on the device.
#pragma once

#include "bn254.cuh"

namespace impeller {

using namespace ec;

static constexpr u32 NONE = 0xffffffffu;
static constexpr u32 SCAN_BLOCK = 256;
static constexpr u32 SCAN_PER_THREAD = 16;
static constexpr u32 SCAN_TILE = SCAN_BLOCK * SCAN_PER_THREAD;

// One MSM of a batch.  Virtual point index of digit window w of scalar i is
// table_base + (w / n_windows) * table_stride + i: window tables hold
// 2^(j*n_windows*c)*P (core/src/msm/src/msm.cuh:53-70 for the window / table
// relation); table_base selects one of several table sets kept in one array.
struct MsmDesc {
    const u32 *scalars;  // n x 8 u32, Montgomery Fr
    u32 n;
    u32 c;               // window bits
    u32 n_logical;       // ceil(254 / c) digit windows
    u32 n_windows;       // bucket sets (physical windows)
    u32 table_stride;    // points per window table
    u32 bucket_base;     // global index of bucket (window 0, weight 1)
    u32 win_base;        // global index of physical window 0
    u32 table_base;      // index of this MSM's table 0 in the point array
    u32 entry_base;      // first digit slot of this MSM (sum of n * n_logical of the earlier MSMs)
};

// One physical window of one MSM (bucket reduction unit).
struct WinDesc {
    u32 bucket_base;  // global index of the weight-1 bucket of this window
    u32 nbuckets;     // 2^(c-1)
    u32 chunk;        // buckets per reduce thread
    u32 part_base;    // first partial-sum slot of this window
    u32 nparts;       // number of partial-sum slots (reduce blocks)
    u32 msm;          // owning MSM
    u32 pad0, pad1;
};

// Signed-digit recoding of the reference (core/src/msm/src/msm_impl.cuh:22-33):
// a digit >= 2^(c-1) becomes digit - 2^c and carries into the next window.
// The top window is never recoded: for every 3 <= c <= 31, r < 2^254 keeps
// the top digit plus an incoming carry at most 2^(c-1), a valid bucket.
//
// for_each_digit calls emit(pw, table, mag, sign) for each of the n_logical
// digit windows w of a canonical scalar, lowest first (mag == 0 for a zero
// digit), with pw = w mod n_windows (the bucket set) and table = w /
// n_windows (the window table).  The scalar's limbs feed a 64-bit bit buffer
// one at a time -- the limb index is a constant in every unrolled step -- so
// a digit costs one 64-bit shift, and the window and table indices advance
// by counting instead of dividing.  Every lane runs the same windows (the
// count depends only on c and n_logical).
template <class FR, class Emit>
__device__ __forceinline__ void for_each_digit(const Fe<FR> &v, u32 c, u32 n_logical, u32 n_windows, Emit &&emit) {
    const u32 mask = (1u << c) - 1u, half = 1u << (c - 1);
    u64 buf = 0;
    u32 nbits = 0, carry = 0, w = 0, pw = 0, table = 0;
    auto step = [&](u32 raw, bool top) {
        const u32 d = raw + carry;
        if (d >= half && !top) {
            emit(pw, table, (1u << c) - d, 1u);
            carry = 1;
        } else {
            emit(pw, table, d, 0u);
            carry = 0;
        }
        w++;
        if (++pw == n_windows) {
            pw = 0;
            table++;
        }
    };
#pragma unroll
    for (int k = 0; k < FR::N; k++) {
        buf |= (u64)v.l[k] << nbits;
        nbits += 32;
        while (nbits >= c && w + 1 < n_logical) {
            step((u32)buf & mask, false);
            buf >>= c;
            nbits -= c;
        }
    }
    while (w + 1 < n_logical) {
        step((u32)buf & mask, false);
        buf >>= c;
    }
    step((u32)buf & mask, true);
}

// Lanes of a warp whose digits hit the same bucket share one atomic: heavy
// buckets (the top window in a shared bucket set, the 0 / 1 / small scalars of
// witness-like inputs) would otherwise serialize on a handful of addresses.
// Every lane of the warp runs the same number of windows, so the match is
// always taken with the full warp present.
template <class C>
__global__ void k_histogram(const MsmDesc *__restrict__ descs, u32 *__restrict__ counts) {
    const MsmDesc d = descs[blockIdx.y];
    const u32 B = 1u << (d.c - 1);
    const u32 lane = threadIdx.x & 31u;
    const u32 stride = gridDim.x * blockDim.x;
    for (u32 base = blockIdx.x * blockDim.x; base < d.n; base += stride) {
        const u32 i = base + threadIdx.x;
        const bool live = i < d.n;
        const Fe<typename C::Fr> v = live ? fe_from_mont<typename C::Fr>(fe_load<typename C::Fr>(d.scalars + 8ull * i))
                                          : fe_zero<typename C::Fr>();
        for_each_digit(v, d.c, d.n_logical, d.n_windows, [&](u32 pw, u32, u32 mag, u32) {
            const u32 key = mag ? d.bucket_base + pw * B + mag - 1 : NONE;
            const u32 peers = __match_any_sync(0xffffffffu, key);
            if (key != NONE && lane == __ffs(peers) - 1) atomicAdd(&counts[key], (u32)__popc(peers));
        });
    }
}

template <class C>
__global__ void k_scatter(const MsmDesc *__restrict__ descs, u32 *__restrict__ cursor, u32 *__restrict__ entries) {
    const MsmDesc d = descs[blockIdx.y];
    const u32 B = 1u << (d.c - 1);
    const u32 lane = threadIdx.x & 31u;
    const u32 stride = gridDim.x * blockDim.x;
    for (u32 base = blockIdx.x * blockDim.x; base < d.n; base += stride) {
        const u32 i = base + threadIdx.x;
        const bool live = i < d.n;
        const Fe<typename C::Fr> v = live ? fe_from_mont<typename C::Fr>(fe_load<typename C::Fr>(d.scalars + 8ull * i))
                                          : fe_zero<typename C::Fr>();
        for_each_digit(v, d.c, d.n_logical, d.n_windows, [&](u32 pw, u32 table, u32 mag, u32 sign) {
            const u32 key = mag ? d.bucket_base + pw * B + mag - 1 : NONE;
            const u32 peers = __match_any_sync(0xffffffffu, key);
            const u32 leader = __ffs(peers) - 1;
            u32 pos = 0;
            if (key != NONE && lane == leader) pos = atomicAdd(&cursor[key], (u32)__popc(peers));
            pos = __shfl_sync(0xffffffffu, pos, leader);
            if (key != NONE) {
                const u32 rank = __popc(peers & ((1u << lane) - 1u));
                entries[pos + rank] = ((d.table_base + table * d.table_stride + i) << 1) | sign;
            }
        });
    }
}

// ------------------------------------------------- two-level counting sort
//
// The bucket sort above costs one L2 atomic per entry in each of its two
// passes and scatters 4-byte writes over the whole entry array.  The
// two-level sort keeps every atomic in shared memory and every global write
// in runs:
//   k_coarse_count    per tile of scalars: entries per coarse bin (the top
//                     bits of the global bucket index; FINE buckets per bin),
//                     and every digit's bucket key for the scatter
//   (scan)            bin-major exclusive scan of the tile counts (per MSM
//                     its own bins x its own tiles)
//   k_coarse_scatter  per tile: the keys' entries staged in shared memory in
//                     bin order, written out as one contiguous run per bin,
//                     with the fine index (bucket within the bin) beside them
//   k_seg_plan        split every bin into segments of at most SEG_ENTRIES
//   k_seg_hist        per segment: entries per fine bucket
//   k_bin_scan        per bin: bucket offsets, and each segment's cursor per
//                     fine bucket
//   k_seg_scatter     per segment: entries staged in bucket order, written
//                     to their final slots as one run per bucket
// Order inside a bucket is irrelevant (a bucket is a sum).  Heavy buckets
// (skewed scalars) only lengthen their bin, which splits into more segments.
// Shared-memory atomics are taken per lane: a per-lane atomicAdd on a cursor
// already returns a distinct slot, and warp matching to aggregate them
// measured slower than the atomics it saves.

static constexpr u32 FINE_BITS = 10;
static constexpr u32 FINE = 1u << FINE_BITS;     // buckets per coarse bin
static constexpr u32 SORT_MAX_BINS = 8192;       // nb <= 2^23
static constexpr u64 SORT_MAX_CELLS = 1ull << 26;  // bins x scalar tiles (count matrix entries)
static constexpr u32 STAGE_ENTRIES = 16384;      // staged entries per tile
static constexpr u32 SEG_ENTRIES = 32768;        // entries per fine segment (staged whole)
static constexpr u32 SORT_BLOCK = 512;
static constexpr u32 FINE_BLOCK = 1024;
static_assert(FINE == FINE_BLOCK, "k_seg_scatter gives every bucket of a bin one thread");

struct SortArgs {
    const MsmDesc *descs;
    const u32 *tile_first;  // M + 1: first sort tile of each MSM
    const u32 *bin_cell;    // nbins + 1: first count cell of each bin; [nbins] = cells
    u32 M, ntiles, tile_scalars, nbins, nb, segcap;
    u32 *cnt;               // per MSM (bins on FINE boundaries), its bins x its tiles,
                            // bin-major: cell bin_cell[b] + (tile - tile_first[m]) (scan input, padded)
    const u32 *coff;        // exclusive scan of cnt; coff[bin_cell[nbins]] = E
    u32 *c_entry;           // entries in coarse order
    unsigned short *c_fine; // their bucket index within the bin
    uint4 *segs;            // per segment: bin, first, end
    uint2 *bin_seg;         // per bin: first segment, segment count
    u32 *nsegs;             // [0]: number of segments
    u32 *seghist;           // segcap x FINE: entries per segment and bucket
    u32 *segcur;            // segcap x FINE: each segment's first slot per bucket
    u32 *offsets;           // nb + 1 (output)
    u32 *entries;           // (output)
    u32 *keys;              // per MSM, tile and digit window: the digit's bucket (bit 31: sign) or NONE;
                            // written by k_coarse_count, read by k_coarse_scatter (may alias entries)
};

// Exclusive scan over the block (blockDim a multiple of 32, at most 1024).
__device__ __forceinline__ u32 block_scan_excl(u32 v, u32 &total, u32 *warp_tot) {
    const u32 lane = threadIdx.x & 31u, wid = threadIdx.x >> 5, nw = blockDim.x >> 5;
    u32 x = v;
#pragma unroll
    for (u32 o = 1; o < 32; o <<= 1) {
        u32 y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[wid] = x;
    __syncthreads();
    if (wid == 0) {
        u32 t = lane < nw ? warp_tot[lane] : 0;
#pragma unroll
        for (u32 o = 1; o < 32; o <<= 1) {
            u32 y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < nw) warp_tot[lane] = t;
    }
    __syncthreads();
    total = warp_tot[nw - 1];
    const u32 before = wid ? warp_tot[wid - 1] : 0;
    __syncthreads();
    return before + x - v;
}

// MSM and scalar range [start, end) of a sort tile (tiles of one MSM are
// consecutive; the largest m with tile_first[m] <= tile owns it).
__device__ __forceinline__ void sort_tile(const SortArgs &a, u32 tile, u32 &m, u32 &start, u32 &end) {
    u32 lo = 0, hi = a.M;
    while (hi - lo > 1) {
        const u32 mid = (lo + hi) >> 1;
        if (a.tile_first[mid] <= tile) lo = mid;
        else hi = mid;
    }
    m = lo;
    start = (tile - a.tile_first[m]) * a.tile_scalars;
    end = min(start + a.tile_scalars, a.descs[m].n);
}

template <class C>
__global__ void __launch_bounds__(SORT_BLOCK) k_coarse_count(SortArgs a) {
    extern __shared__ u32 hist[];  // nbins
    u32 m, start, end;
    sort_tile(a, blockIdx.x, m, start, end);
    const MsmDesc d = a.descs[m];
    const u32 B = 1u << (d.c - 1);
    // this MSM's bins
    const u32 blo = d.bucket_base >> FINE_BITS, bhi = (d.bucket_base + d.n_windows * B - 1u) >> FINE_BITS;
    for (u32 b = blo + threadIdx.x; b <= bhi; b += blockDim.x) hist[b] = 0;
    __syncthreads();
    // the tile's keys, window-major: key of window w, scalar i at w * (end - start) + i - start
    const u32 tile_n = end - start;
    u32 *kp = a.keys + d.entry_base + (size_t)start * d.n_logical;
    for (u32 base = start; base < end; base += blockDim.x) {
        const u32 i = base + threadIdx.x;
        const bool live = i < end;
        const Fe<typename C::Fr> v = live ? fe_from_mont<typename C::Fr>(fe_load<typename C::Fr>(d.scalars + 8ull * i))
                                          : fe_zero<typename C::Fr>();
        u32 *kw = kp + (i - start);
        for_each_digit(v, d.c, d.n_logical, d.n_windows, [&](u32 pw, u32, u32 mag, u32 sign) {
            u32 key = NONE;
            if (mag) {
                key = d.bucket_base + pw * B + mag - 1;
                atomicAdd(&hist[key >> FINE_BITS], 1u);
                key |= sign << 31;
            }
            if (live) *kw = key;
            kw += tile_n;
        });
    }
    __syncthreads();
    const u32 tl = blockIdx.x - a.tile_first[m];
    for (u32 b = blo + threadIdx.x; b <= bhi; b += blockDim.x) a.cnt[a.bin_cell[b] + tl] = hist[b];
}

// Shared memory: delta[nbins], cur[nbins], stage_e[STAGE_ENTRIES] (u32),
// stage_f[STAGE_ENTRIES] (u16: bucket within the bin).  A tile holds at most
// STAGE_ENTRIES entries (the plan sizes tiles by the largest window count).
// 6 staged bytes per entry keep two CTAs on an SM for plans of up to 2048
// bins.  Only the bins of the tile's MSM are touched: a batch's other MSMs
// own other bins.
template <class C>
__global__ void __launch_bounds__(SORT_BLOCK, 2) k_coarse_scatter(SortArgs a) {
    extern __shared__ u32 sm[];
    __shared__ u32 warp_tot[32];
    u32 *delta = sm, *cur = sm + a.nbins, *stage_e = sm + 2 * a.nbins;
    unsigned short *stage_f = reinterpret_cast<unsigned short *>(stage_e + STAGE_ENTRIES);
    const u32 tile = blockIdx.x;
    u32 m, start, end;
    sort_tile(a, tile, m, start, end);
    const MsmDesc d = a.descs[m];
    const u32 B = 1u << (d.c - 1);
    const u32 blo = d.bucket_base >> FINE_BITS, bhi = (d.bucket_base + d.n_windows * B - 1u) >> FINE_BITS;
    // this tile's bins: local start (exclusive scan of its counts) and the
    // distance from a local slot to the global coarse position
    const u32 per = (bhi - blo + blockDim.x) / blockDim.x;
    const u32 b0 = blo + threadIdx.x * per;
    const u32 tl = tile - a.tile_first[m];
    u32 sum = 0;
    for (u32 k = 0; k < per; k++)
        if (b0 + k <= bhi) sum += a.cnt[a.bin_cell[b0 + k] + tl];
    u32 total;
    u32 run = block_scan_excl(sum, total, warp_tot);
    for (u32 k = 0; k < per; k++) {
        const u32 b = b0 + k;
        if (b <= bhi) {
            const size_t ci = a.bin_cell[b] + tl;
            cur[b] = run;
            delta[b] = a.coff[ci] - run;
            run += a.cnt[ci];
        }
    }
    __syncthreads();
    // the keys k_coarse_count left for this tile (window-major)
    const u32 tile_n = end - start, nsets = d.n_windows;
    const u32 *kp = a.keys + d.entry_base + (size_t)start * d.n_logical;
    // Eight keys are loaded before any is placed, so that their load
    // latencies overlap (the kernel is otherwise bound by them).
    constexpr u32 KB = 8;
    for (u32 i = start + threadIdx.x; i < end; i += blockDim.x) {
        const u32 *kw = kp + (i - start);
        u32 pw = 0, table = 0;
        for (u32 w0 = 0; w0 < d.n_logical; w0 += KB) {
            u32 key[KB];
#pragma unroll
            for (u32 j = 0; j < KB; j++) key[j] = w0 + j < d.n_logical ? __ldg(kw + (size_t)(w0 + j) * tile_n) : NONE;
#pragma unroll
            for (u32 j = 0; j < KB; j++) {
                if (key[j] != NONE) {
                    const u32 bk = key[j] & 0x7fffffffu;
                    const u32 slot = atomicAdd(&cur[bk >> FINE_BITS], 1u);
                    stage_e[slot] = ((d.table_base + table * d.table_stride + i) << 1) | (key[j] >> 31);
                    stage_f[slot] = (unsigned short)(bk & (FINE - 1u));
                }
                if (++pw == nsets) {
                    pw = 0;
                    table++;
                }
            }
        }
    }
    __syncthreads();
    // one warp per bin writes the bin's run of this tile: one coalesced run
    // of entries and one of bucket indices
    const u32 lane = threadIdx.x & 31u, nw = blockDim.x >> 5;
    for (u32 b = blo + (threadIdx.x >> 5); b <= bhi; b += nw) {
        const u32 s0 = b == blo ? 0u : cur[b - 1], s1 = cur[b];
        const u32 g = delta[b];
        for (u32 s = s0 + lane; s < s1; s += 32) {
            a.c_entry[g + s] = stage_e[s];
            a.c_fine[g + s] = stage_f[s];
        }
    }
}

// One block: every bin's segments (at most SEG_ENTRIES entries each).
__global__ void __launch_bounds__(FINE_BLOCK) k_seg_plan(SortArgs a) {
    __shared__ u32 warp_tot[32];
    const u32 per = (a.nbins + blockDim.x - 1) / blockDim.x;
    const u32 b0 = threadIdx.x * per;
    u32 sum = 0;
    for (u32 k = 0; k < per; k++) {
        const u32 b = b0 + k;
        if (b < a.nbins) {
            const u32 size = a.coff[a.bin_cell[b + 1]] - a.coff[a.bin_cell[b]];
            sum += (size + SEG_ENTRIES - 1) / SEG_ENTRIES;
        }
    }
    u32 total;
    u32 run = block_scan_excl(sum, total, warp_tot);
    for (u32 k = 0; k < per; k++) {
        const u32 b = b0 + k;
        if (b < a.nbins) {
            const u32 bs = a.coff[a.bin_cell[b]], be = a.coff[a.bin_cell[b + 1]];
            const u32 ns = (be - bs + SEG_ENTRIES - 1) / SEG_ENTRIES;
            a.bin_seg[b] = make_uint2(run, ns);
            for (u32 j = 0; j < ns; j++)
                a.segs[run + j] = make_uint4(b, bs + j * SEG_ENTRIES, min(bs + (j + 1) * SEG_ENTRIES, be), 0u);
            run += ns;
        }
    }
    if (threadIdx.x == 0) a.nsegs[0] = total;
}

// Entries of a segment are read 8 bucket indices (16 bytes) at a time, four
// loads in flight per thread, so that the load latency overlaps.
__device__ __forceinline__ void hist8(u32 *hist, uint4 q) {
    atomicAdd(&hist[q.x & 0xffffu], 1u);
    atomicAdd(&hist[q.x >> 16], 1u);
    atomicAdd(&hist[q.y & 0xffffu], 1u);
    atomicAdd(&hist[q.y >> 16], 1u);
    atomicAdd(&hist[q.z & 0xffffu], 1u);
    atomicAdd(&hist[q.z >> 16], 1u);
    atomicAdd(&hist[q.w & 0xffffu], 1u);
    atomicAdd(&hist[q.w >> 16], 1u);
}

__global__ void __launch_bounds__(FINE_BLOCK) k_seg_hist(SortArgs a) {
    __shared__ u32 hist[FINE];
    if (blockIdx.x >= a.nsegs[0]) return;
    const uint4 sg = a.segs[blockIdx.x];
    for (u32 f = threadIdx.x; f < FINE; f += blockDim.x) hist[f] = 0;
    __syncthreads();
    // [y, v0) and [v1, z) one by one, [v0, v1) in aligned groups of 8
    const u32 y = sg.y, z = sg.z;
    const u32 v0 = min((y + 7u) & ~7u, z), v1 = v0 + ((z - v0) & ~7u);
    const unsigned short *cf = a.c_fine;
    if (threadIdx.x < v0 - y) atomicAdd(&hist[cf[y + threadIdx.x]], 1u);
    if (threadIdx.x < z - v1) atomicAdd(&hist[cf[v1 + threadIdx.x]], 1u);
    const uint4 *v = reinterpret_cast<const uint4 *>(cf + v0);
    const u32 nv = (v1 - v0) >> 3, bd = blockDim.x;
    u32 k = threadIdx.x;
    for (; k + 3 * bd < nv; k += 4 * bd) {
        const uint4 q0 = __ldg(v + k), q1 = __ldg(v + k + bd), q2 = __ldg(v + k + 2 * bd), q3 = __ldg(v + k + 3 * bd);
        hist8(hist, q0);
        hist8(hist, q1);
        hist8(hist, q2);
        hist8(hist, q3);
    }
    for (; k < nv; k += bd) hist8(hist, __ldg(v + k));
    __syncthreads();
    for (u32 f = threadIdx.x; f < FINE; f += blockDim.x) a.seghist[(size_t)blockIdx.x * FINE + f] = hist[f];
}

// One block per bin: per fine bucket, an exclusive scan over the bin's
// segments (their cursors) and the bucket's total; then a scan over the
// bin's buckets gives the bucket offsets.
__global__ void __launch_bounds__(FINE_BLOCK) k_bin_scan(SortArgs a) {
    __shared__ u32 warp_tot[32];
    const u32 b = blockIdx.x;
    const uint2 bs = a.bin_seg[b];
    const u32 base = a.coff[a.bin_cell[b]];
    u32 carry = base;
    for (u32 f0 = 0; f0 < FINE; f0 += blockDim.x) {
        const u32 f = f0 + threadIdx.x;
        u32 run = 0;
        for (u32 s = bs.x; s < bs.x + bs.y; s++) run += a.seghist[(size_t)s * FINE + f];
        u32 total;
        const u32 off = carry + block_scan_excl(run, total, warp_tot);
        const u32 g = b * FINE + f;
        if (g < a.nb) a.offsets[g] = off;
        // each segment's cursor: the bucket offset plus the earlier segments' counts
        u32 cur = off;
        for (u32 s = bs.x; s < bs.x + bs.y; s++) {
            a.segcur[(size_t)s * FINE + f] = cur;
            cur += a.seghist[(size_t)s * FINE + f];
        }
        carry += total;
    }
    if (b == a.nbins - 1 && threadIdx.x == 0) a.offsets[a.nb] = a.coff[a.bin_cell[a.nbins]];
}

// Shared memory: lcur[FINE], delta[FINE], stage_e[SEG_ENTRIES],
// stage_f[SEG_ENTRIES] (16-bit).  Entries are read four at a time (16 bytes
// of entries, 8 of bucket indices), two groups in flight per thread.
__device__ __forceinline__ void place1(u32 *lcur, u32 *stage_e, unsigned short *stage_f, u32 fi, u32 e) {
    const u32 slot = atomicAdd(&lcur[fi], 1u);
    stage_e[slot] = e;
    stage_f[slot] = (unsigned short)fi;
}

__device__ __forceinline__ void place4(u32 *lcur, u32 *stage_e, unsigned short *stage_f, uint2 f, uint4 e) {
    place1(lcur, stage_e, stage_f, f.x & 0xffffu, e.x);
    place1(lcur, stage_e, stage_f, f.x >> 16, e.y);
    place1(lcur, stage_e, stage_f, f.y & 0xffffu, e.z);
    place1(lcur, stage_e, stage_f, f.y >> 16, e.w);
}

__global__ void __launch_bounds__(FINE_BLOCK) k_seg_scatter(SortArgs a) {
    extern __shared__ u32 sm[];
    __shared__ u32 warp_tot[32];
    if (blockIdx.x >= a.nsegs[0]) return;
    u32 *lcur = sm, *delta = sm + FINE, *stage_e = sm + 2 * FINE;
    unsigned short *stage_f = reinterpret_cast<unsigned short *>(stage_e + SEG_ENTRIES);
    const uint4 sg = a.segs[blockIdx.x];
    const size_t h = (size_t)blockIdx.x * FINE;
    // local exclusive scan of this segment's counts (FINE == blockDim.x)
    const u32 f = threadIdx.x;
    u32 total;
    const u32 ls = block_scan_excl(a.seghist[h + f], total, warp_tot);
    lcur[f] = ls;
    delta[f] = a.segcur[h + f] - ls;
    __syncthreads();
    // [y, v0) and [v1, z) one by one, [v0, v1) in aligned groups of 4
    const u32 y = sg.y, z = sg.z;
    const u32 v0 = min((y + 3u) & ~3u, z), v1 = v0 + ((z - v0) & ~3u);
    if (threadIdx.x < v0 - y) place1(lcur, stage_e, stage_f, a.c_fine[y + threadIdx.x], a.c_entry[y + threadIdx.x]);
    if (threadIdx.x < z - v1) place1(lcur, stage_e, stage_f, a.c_fine[v1 + threadIdx.x], a.c_entry[v1 + threadIdx.x]);
    const uint2 *vf = reinterpret_cast<const uint2 *>(a.c_fine + v0);
    const uint4 *ve = reinterpret_cast<const uint4 *>(a.c_entry + v0);
    const u32 nv = (v1 - v0) >> 2, bd = blockDim.x;
    u32 k = threadIdx.x;
    for (; k + bd < nv; k += 2 * bd) {
        const uint2 f0 = __ldg(vf + k), f1 = __ldg(vf + k + bd);
        const uint4 e0 = __ldg(ve + k), e1 = __ldg(ve + k + bd);
        place4(lcur, stage_e, stage_f, f0, e0);
        place4(lcur, stage_e, stage_f, f1, e1);
    }
    for (; k < nv; k += bd) place4(lcur, stage_e, stage_f, __ldg(vf + k), __ldg(ve + k));
    __syncthreads();
    for (u32 s = threadIdx.x; s < total; s += blockDim.x) a.entries[delta[stage_f[s]] + s] = stage_e[s];
}

// ------------------------------------------------------------------- scan

__device__ __forceinline__ u32 block_exclusive_scan(u32 v, u32 &total) {
    __shared__ u32 warp_tot[SCAN_BLOCK / 32];
    const u32 lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    u32 x = v;
#pragma unroll
    for (u32 o = 1; o < 32; o <<= 1) {
        u32 y = __shfl_up_sync(0xffffffffu, x, o);
        if (lane >= o) x += y;
    }
    if (lane == 31) warp_tot[wid] = x;
    __syncthreads();
    if (wid == 0) {
        u32 t = lane < SCAN_BLOCK / 32 ? warp_tot[lane] : 0;
#pragma unroll
        for (u32 o = 1; o < 32; o <<= 1) {
            u32 y = __shfl_up_sync(0xffffffffu, t, o);
            if (lane >= o) t += y;
        }
        if (lane < SCAN_BLOCK / 32) warp_tot[lane] = t;
    }
    __syncthreads();
    total = warp_tot[SCAN_BLOCK / 32 - 1];
    u32 before = wid ? warp_tot[wid - 1] : 0;
    __syncthreads();
    return before + x - v;
}

// counts must be padded to a multiple of SCAN_TILE with zeros.
__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_reduce(const u32 *__restrict__ counts, u32 *__restrict__ tile_sums) {
    const uint4 *p = reinterpret_cast<const uint4 *>(counts + (size_t)blockIdx.x * SCAN_TILE) + threadIdx.x * 4;
    u32 s = 0;
#pragma unroll
    for (int k = 0; k < 4; k++) {
        uint4 v = p[k];
        s += v.x + v.y + v.z + v.w;
    }
    u32 total;
    block_exclusive_scan(s, total);
    if (threadIdx.x == 0) tile_sums[blockIdx.x] = total;
}

// Single block: exclusive scan of the tile sums in place; tile_sums[ntiles]
// receives the grand total.
__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_tiles(u32 *__restrict__ tile_sums, u32 ntiles) {
    u32 carry = 0;
    for (u32 base = 0; base < ntiles; base += SCAN_BLOCK) {
        u32 i = base + threadIdx.x;
        u32 v = i < ntiles ? tile_sums[i] : 0;
        u32 total;
        u32 ex = block_exclusive_scan(v, total);
        if (i < ntiles) tile_sums[i] = carry + ex;
        carry += total;
    }
    if (threadIdx.x == 0) tile_sums[ntiles] = carry;
}

__global__ void __launch_bounds__(SCAN_BLOCK) k_scan_down(const u32 *__restrict__ counts, const u32 *__restrict__ tile_sums,
                                                   u32 *__restrict__ offsets, u32 *__restrict__ cursor, u32 nb,
                                                   u32 ntiles) {
    const size_t base = (size_t)blockIdx.x * SCAN_TILE + threadIdx.x * SCAN_PER_THREAD;
    const uint4 *p = reinterpret_cast<const uint4 *>(counts + base);
    u32 v[SCAN_PER_THREAD];
#pragma unroll
    for (int k = 0; k < 4; k++) {
        uint4 q = p[k];
        v[4 * k] = q.x; v[4 * k + 1] = q.y; v[4 * k + 2] = q.z; v[4 * k + 3] = q.w;
    }
    u32 s = 0;
#pragma unroll
    for (int k = 0; k < (int)SCAN_PER_THREAD; k++) s += v[k];
    u32 total;
    u32 run = block_exclusive_scan(s, total) + tile_sums[blockIdx.x];
#pragma unroll
    for (int k = 0; k < (int)SCAN_PER_THREAD; k++) {
        size_t i = base + k;
        if (i < nb) {
            offsets[i] = run;
            cursor[i] = run;
        }
        run += v[k];
    }
    if (blockIdx.x == 0 && threadIdx.x == 0) offsets[nb] = tile_sums[ntiles];
}

// ------------------------------------------------------------- accumulate

struct AccumArgs {
    const u32 *entries;
    const u32 *offsets;  // nb + 1
    u32 nb;
    const u32 *points;   // affine, 16 u32 each
    u32 *buckets;        // XYZZ, 32 u32 each, indexed by global bucket
    u32 *rec_bucket;     // 2 per thread
    u32 *rec_point;      // 2 per thread, XYZZ
};

template <class C>
__device__ __forceinline__ AffineT<typename C::Fq> load_entry_point(const u32 *__restrict__ points, u32 e) {
    AffineT<typename C::Fq> q = affine_load<typename C::Fq>(points + (size_t)(e >> 1) * C::PW);
    if (e & 1u) q.y = fe_neg(q.y);
    return q;
}

// Thread t owns entries [t*L, min((t+1)*L, E)), L = ceil(E / T).
// A bucket whose entries all fall in one slice is written to `buckets`.
// Otherwise the slice leaves a record: slot 2t for a piece that continues a
// bucket begun in an earlier slice, slot 2t+1 for a piece whose bucket begins
// in this slice and continues in later ones.
// START_CARRY: the slice where a bucket begins starts it from the bucket's
// current value in `buckets` (a streamed call adds every chunk's points into
// accumulators that persist across its chunks; buckets without entries in
// the chunk are left as they are).
// One block of 384 threads per SM: 146 registers per thread with no spills,
// 12 warps spread evenly over the SM's four schedulers.  Measured on B200 at
// 2^22 this beats 2 x 256 threads at 128 registers (which spill) by 4%, and
// 320-, 352- and 256-thread single blocks by 8-20%.
#ifndef ACCUM_THREADS
#define ACCUM_THREADS 384
#endif
#ifndef ACCUM_BLOCKS_PER_SM
#define ACCUM_BLOCKS_PER_SM 1
#endif
// BLS12-381 (48-word XYZZ, 12-limb products) has its own block shape.
#ifndef ACCUM_THREADS_BLS
#define ACCUM_THREADS_BLS 384
#endif
#ifndef ACCUM_BLOCKS_PER_SM_BLS
#define ACCUM_BLOCKS_PER_SM_BLS 1
#endif
template <class C>
struct AccumShape {
    static constexpr u32 threads = C::XW == 32 ? ACCUM_THREADS : ACCUM_THREADS_BLS;
    static constexpr u32 per_sm = C::XW == 32 ? ACCUM_BLOCKS_PER_SM : ACCUM_BLOCKS_PER_SM_BLS;
};

// How a slice starts a bucket: START_CONVERT converts the first point (no
// addition on that branch: 5 % fewer instructions per mixed addition on
// BN254); START_IDENTITY adds every point, the first to the identity (one
// addition code path: fewer registers); START_CARRY adds every point, the
// first to the bucket's value in `buckets` (streamed chunks).
enum : int { START_CONVERT = 0, START_IDENTITY = 1, START_CARRY = 2 };
// BLS12-381 (measured at 2^22, tables c = 20): identity start 22.50 ms per
// MSM, convert 22.61 ms (its two code paths spill 44 bytes at 168 registers).
#ifndef ACCUM_START_BLS
#define ACCUM_START_BLS START_IDENTITY
#endif

template <class C, int START = START_CONVERT>
__global__ void __launch_bounds__(AccumShape<C>::threads, AccumShape<C>::per_sm) k_accumulate(AccumArgs a) {
    using FQ = typename C::Fq;
    const u32 T = gridDim.x * blockDim.x;
    const u32 t = blockIdx.x * blockDim.x + threadIdx.x;
    const u32 E = a.offsets[a.nb];
    const u32 L = (E + T - 1) / T;
    const u64 start64 = (u64)t * L;
    const u32 start = (u32)min(start64, (u64)E);
    const u32 end = (u32)min(start64 + L, (u64)E);
    a.rec_bucket[2 * t] = NONE;
    a.rec_bucket[2 * t + 1] = NONE;
    if (start >= end) return;

    // largest b with offsets[b] <= start
    u32 lo = 0, hi = a.nb;
    while (hi - lo > 1) {
        u32 mid = (lo + hi) >> 1;
        if (a.offsets[mid] <= start) lo = mid;
        else hi = mid;
    }
    u32 b = lo;
    u32 bbeg = a.offsets[b], bend = a.offsets[b + 1];
    u32 seg_end = min(bend, end);

    XyzzT<FQ> acc = xyzz_identity<FQ>();
    bool fresh = true;
    AffineT<FQ> nxt = load_entry_point<C>(a.points, a.entries[start]);
    for (u32 pos = start; pos < end; pos++) {
        AffineT<FQ> q = nxt;
        if (pos + 1 < end) nxt = load_entry_point<C>(a.points, a.entries[pos + 1]);
        // One mixed-addition code path for every entry: a bucket start only
        // picks the value the addition starts from (lanes of a warp start
        // buckets at different entries, and a second inlined addition on
        // that branch would run divergently, doubling the loop's time).
        if constexpr (START != START_CONVERT) {
            if (fresh) {
                acc = (START == START_CARRY && bbeg >= start) ? xyzz_load<FQ>(a.buckets + (size_t)b * C::XW)
                                                              : xyzz_identity<FQ>();
                fresh = false;
            }
            acc = xyzz_add_affine(acc, q);
            if (START == START_CARRY && pos + 2 == seg_end && seg_end == bend && b + 1 < a.nb)
                asm volatile("prefetch.global.L1 [%0];" ::"l"(a.buckets + (size_t)(b + 1) * C::XW));
        } else {
            if (fresh) {
                acc = xyzz_from_affine(q);
                fresh = false;
            } else {
                acc = xyzz_add_affine(acc, q);
            }
        }
        if (pos + 1 == seg_end) {
            if (bbeg >= start && bend <= end) {
                xyzz_store(a.buckets + (size_t)b * C::XW, acc);
            } else {
                u32 slot = bbeg < start ? 2 * t : 2 * t + 1;
                a.rec_bucket[slot] = b;
                xyzz_store(a.rec_point + (size_t)slot * C::XW, acc);
            }
            fresh = true;
            if (pos + 1 < end) {
                do {
                    b++;
                    bend = a.offsets[b + 1];
                } while (bend <= pos + 1);
                bbeg = a.offsets[b];
                seg_end = min(bend, end);
            }
        }
    }
}

// Long runs of up to this many pieces are merged by one warp (pieces / 32
// additions per lane, then a 5-step warp sum), longer ones by a block.
#ifndef FIXUP_WARP_MAX
#define FIXUP_WARP_MAX 256
#endif

struct FixupArgs {
    const u32 *offsets;
    u32 nb;
    u32 T;               // accumulate threads
    const u32 *rec_bucket;
    const u32 *rec_point;
    u32 *buckets;
    u32 *long_list;      // [0] = count, then owner thread ids
    u32 long_cap;
    u32 warp_max;        // longest run k_fixup_long gives one warp (0: every run)
};

// Owner of a cut bucket = the slice where the bucket begins (record 2t+1).
// The bucket continues as the first piece (record 2t') of slices t+1 .. t1.
template <class C>
__global__ void k_fixup_short(FixupArgs f) {
    using FQ = typename C::Fq;
    const u32 t = blockIdx.x * blockDim.x + threadIdx.x;
    if (t >= f.T) return;
    const u32 b = f.rec_bucket[2 * t + 1];
    if (b == NONE) return;
    const u32 E = f.offsets[f.nb];
    const u32 L = (E + f.T - 1) / f.T;
    const u32 t1 = (f.offsets[b + 1] - 1) / L;
    if (t1 - t > 4) {
        u32 k = atomicAdd(&f.long_list[0], 1u);
        if (k < f.long_cap) f.long_list[1 + k] = t;
        return;
    }
    XyzzT<FQ> acc = xyzz_load<FQ>(f.rec_point + (size_t)(2 * t + 1) * C::XW);
    for (u32 s = t + 1; s <= t1; s++) acc = xyzz_add(acc, xyzz_load<FQ>(f.rec_point + (size_t)(2 * s) * C::XW));
    xyzz_store(f.buckets + (size_t)b * C::XW, acc);
}

// Long runs (a bucket spread over more than 5 slices), in one launch:
// blocks below wide_blocks take the runs of more than warp_max pieces, one
// 128-thread block per run (every thread one piece, more only past 128;
// then a warp sum and a sum of the warps' sums: log2 of the run's length
// deep); the other blocks' warps take the shorter runs, one warp per run
// (pieces / 32 additions per lane, then a 5-step warp sum).  Both kinds run
// at the same time.  wide_blocks == 0 or warp_max == 0: every run by a warp.
static constexpr u32 WIDE_BLOCK = 128;
template <class C>
__global__ void k_fixup_long(FixupArgs f, u32 wide_blocks) {
    using FQ = typename C::Fq;
    __shared__ __align__(16) u32 part[WIDE_BLOCK / 32][C::XW];
    const u32 lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    const u32 count = min(f.long_list[0], f.long_cap);
    const u32 E = f.offsets[f.nb];
    const u32 L = (E + f.T - 1) / f.T;
    const u32 wmax = f.warp_max && wide_blocks ? f.warp_max : 0xffffffffu;
    if (blockIdx.x < wide_blocks) {
        for (u32 w = blockIdx.x; w < count; w += wide_blocks) {  // the same runs for the whole block
            const u32 t = f.long_list[1 + w];
            const u32 b = f.rec_bucket[2 * t + 1];
            const u32 pieces = (f.offsets[b + 1] - 1) / L - t + 1;  // the owner's, then slices t+1 ..
            if (pieces <= wmax) continue;
            XyzzT<FQ> acc = xyzz_identity<FQ>();
            for (u32 k = threadIdx.x; k < pieces; k += WIDE_BLOCK) {
                const size_t slot = k == 0 ? 2 * (size_t)t + 1 : 2 * (size_t)(t + k);
                acc = xyzz_add(acc, xyzz_load<FQ>(f.rec_point + slot * C::XW));
            }
            const u32 nw = min((pieces + 31) / 32, WIDE_BLOCK / 32);  // warps holding pieces
            if (wid < nw) {
#pragma unroll 1
                for (u32 o = 16; o; o >>= 1) acc = xyzz_add(acc, xyzz_shfl_down(acc, o));
                if (lane == 0) xyzz_store(&part[wid][0], acc);
            }
            __syncthreads();
            if (wid == 0) {
                XyzzT<FQ> v = lane < nw ? xyzz_load<FQ>(&part[lane][0]) : xyzz_identity<FQ>();
                u32 P = 1;
                while (P < nw) P <<= 1;
#pragma unroll 1
                for (u32 o = P >> 1; o; o >>= 1) v = xyzz_add(v, xyzz_shfl_down(v, o));
                if (lane == 0) xyzz_store(f.buckets + (size_t)b * C::XW, v);
            }
            __syncthreads();  // part is reused by the block's next run
        }
        return;
    }
    const u32 nwarps = ((gridDim.x - wide_blocks) * blockDim.x) >> 5;
    for (u32 w = ((blockIdx.x - wide_blocks) * blockDim.x + threadIdx.x) >> 5; w < count; w += nwarps) {
        const u32 t = f.long_list[1 + w];
        const u32 b = f.rec_bucket[2 * t + 1];
        const u32 t1 = (f.offsets[b + 1] - 1) / L;
        if (t1 - t + 1 > wmax) continue;  // a wide block's
        XyzzT<FQ> acc = xyzz_identity<FQ>();
        if (lane == 0) acc = xyzz_load<FQ>(f.rec_point + (size_t)(2 * t + 1) * C::XW);
        for (u32 s = t + 1 + lane; s <= t1; s += 32)
            acc = xyzz_add(acc, xyzz_load<FQ>(f.rec_point + (size_t)(2 * s) * C::XW));
#pragma unroll 1
        for (u32 o = 16; o; o >>= 1) acc = xyzz_add(acc, xyzz_shfl_down(acc, o));
        if (lane == 0) xyzz_store(f.buckets + (size_t)b * C::XW, acc);
    }
}


// ----------------------------------------------------------------- reduce
//
// Window total T = sum_{k=1..B} k * S_k.  Lane j of a window owns the weights
// (jL, (j+1)L] and forms by a running sum from the top
//   sum_j = sum_k S_k   and   sos_j = sum_k (k - jL) * S_k.
// Since sum_j j * sum_j = sum_{i>=1} suffix_i with suffix_i = sum_{j>=i} sum_j,
//   T = sum_j (sos_j + L * suffix_{j+1}),
// so each lane needs only the exclusive suffix of the chunk sums (a warp
// shuffle scan) and log2(L) doublings -- no per-lane scalar multiplication.
// Each warp leaves V_w = sum over its lanes of (sos_j + L * warp-local
// suffix_{j+1}) and S_w = sum of its chunk sums; the part owed to later warps
// of the window is 32 L * sum_w w * S_w, added by k_window_sum.

struct ReduceArgs {
    const WinDesc *wins;
    const uint2 *blocks;  // (window, block-in-window) per reduce block
    const u32 *offsets;
    const u32 *buckets;
    u32 *parts_v;         // XYZZ per reduce warp
    u32 *parts_s;         // XYZZ per reduce warp
    u32 dense;            // 1: every bucket holds a point (identity when empty); ignore offsets
};

// Products of the reduction-tree levels, which run one to a few dozen
// warps of straight-line point additions: one out-of-line copy (MulCall),
// 11 % faster than inlined at 2^19 buckets on B200.  k_final's Horner loop
// repeats one doubling, whose inlined code stays in the instruction cache:
// inlined there (8 % faster than out-of-line at window 17).  k_reduce runs
// a few warps per SM: inlined (out-of-line measured 10-19 % slower).
#ifndef TAIL_MUL_POLICY
#define TAIL_MUL_POLICY MulCall
#endif
#ifndef FINAL_MUL_POLICY
#define FINAL_MUL_POLICY MulInline
#endif
#ifndef REDUCE_MUL_POLICY
#define REDUCE_MUL_POLICY MulInline
#endif
using TailMul = TAIL_MUL_POLICY;
using FinalMul = FINAL_MUL_POLICY;
using ReduceMul = REDUCE_MUL_POLICY;

static constexpr u32 REDUCE_BLOCK = 128;
// Two 128-thread CTAs per SM (190 registers, no spills): the reduce grid
// fills fewer than two per SM at 2^19 buckets anyway; three (168 registers,
// 356 bytes of spills) measured 1-2 % slower.
#ifndef REDUCE_BLOCKS_PER_SM
#define REDUCE_BLOCKS_PER_SM 2
#endif
#ifndef REDUCE_LANES_PER_SM
#define REDUCE_LANES_PER_SM 256
#endif
static constexpr u32 REDUCE_WARPS = REDUCE_BLOCK / 32;

__device__ __forceinline__ u32 ilog2(u32 x) { return 31 - __clz(x); }

// On BLS12-381 two CTAs per SM, so that the 48-word XYZZ values fit in
// registers (254 instead of 168: spills 2 KB -> 80 B, 4 % faster).
template <class C>
__global__ void __launch_bounds__(REDUCE_BLOCK, C::XW == 32 ? REDUCE_BLOCKS_PER_SM : 2) k_reduce(ReduceArgs r) {
    using FQ = typename C::Fq;
    using Xz = XyzzT<FQ>;
    const uint2 blk = r.blocks[blockIdx.x];
    const WinDesc wd = r.wins[blk.x];
    const u32 lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    const u32 j = blk.y * REDUCE_BLOCK + threadIdx.x;
    const u32 lo = j * wd.chunk;  // weights lo+1 .. lo+chunk
    Xz sum = xyzz_identity<FQ>(), sos = xyzz_identity<FQ>();
    if (lo < wd.nbuckets) {
        const u32 hi = min(lo + wd.chunk, wd.nbuckets);
        for (u32 k = hi; k > lo; k--) {
            const u32 g = wd.bucket_base + k - 1;
            if (r.dense || r.offsets[g + 1] != r.offsets[g])
                sum = xyzz_add<FQ, ReduceMul>(sum, xyzz_load<FQ>(r.buckets + (size_t)g * C::XW));
            sos = xyzz_add<FQ, ReduceMul>(sos, sum);
        }
    }
    // inclusive suffix of `sum` inside the warp
    Xz x = sum;
#pragma unroll 1
    for (u32 o = 1; o < 32; o <<= 1) {
        Xz y = xyzz_shfl_down(x, o);
        if (lane + o < 32) x = xyzz_add<FQ, ReduceMul>(x, y);
    }
    Xz ex = xyzz_shfl_down(x, 1);
    if (lane == 31) ex = xyzz_identity<FQ>();
    ex = xyzz_dbl_n<FQ, ReduceMul>(ex, ilog2(wd.chunk));
    Xz v = xyzz_add<FQ, ReduceMul>(sos, ex);
#pragma unroll 1
    for (u32 o = 16; o; o >>= 1) v = xyzz_add<FQ, ReduceMul>(v, xyzz_shfl_down(v, o));
    if (lane == 0) {
        const size_t slot = (size_t)(wd.part_base + blk.y * REDUCE_WARPS + wid) * C::XW;
        xyzz_store(r.parts_v + slot, v);
        xyzz_store(r.parts_s + slot, x);
    }
}

struct WindowSumArgs {
    const MsmDesc *descs;
    const WinDesc *wins;
    const u32 *parts_v;
    const u32 *parts_s;
    u32 nwins;
    u32 *wres;  // XYZZ per window: the window total T
};

static constexpr u32 WSUM_BLOCK = 256;
static constexpr u32 WSUM_WARPS = WSUM_BLOCK / 32;

// One block per window: T = sum_w V_w + 32 L * sum_w w * S_w (thread t owns a
// group of g consecutive warp partials, a block-wide suffix scan gives the
// cross-group weights).  k_final weights the windows by 2^(c * window).
template <class C>
__global__ void __launch_bounds__(WSUM_BLOCK) k_window_sum(WindowSumArgs a) {
    using FQ = typename C::Fq;
    using Xz = XyzzT<FQ>;
    __shared__ __align__(16) u32 sm_a[WSUM_WARPS][C::XW];
    __shared__ __align__(16) u32 sm_b[WSUM_WARPS][C::XW];
    const u32 win = blockIdx.x;
    if (win >= a.nwins) return;
    const u32 lane = threadIdx.x & 31u, wid = threadIdx.x >> 5;
    const WinDesc wd = a.wins[win];
    u32 g = 1;
    while (g * WSUM_BLOCK < wd.nparts) g <<= 1;
    const u32 b0 = threadIdx.x * g;
    const u32 top = min(b0 + g, wd.nparts);
    // group-local weights: partial b carries weight b - b0
    Xz vsum = xyzz_identity<FQ>(), ssum = xyzz_identity<FQ>(), sos = xyzz_identity<FQ>();
    for (u32 b = top; b > b0; b--) {
        const size_t slot = (size_t)(wd.part_base + b - 1) * C::XW;
        if (b < top) sos = xyzz_add<FQ, ReduceMul>(sos, ssum);
        vsum = xyzz_add<FQ, ReduceMul>(vsum, xyzz_load<FQ>(a.parts_v + slot));
        ssum = xyzz_add<FQ, ReduceMul>(ssum, xyzz_load<FQ>(a.parts_s + slot));
    }
    // block-wide inclusive suffix of ssum: warp scan, then a scan of the warp totals
    Xz x = ssum;
#pragma unroll 1
    for (u32 o = 1; o < 32; o <<= 1) {
        Xz y = xyzz_shfl_down(x, o);
        if (lane + o < 32) x = xyzz_add<FQ, ReduceMul>(x, y);
    }
    if (lane == 0) xyzz_store(&sm_a[wid][0], x);
    __syncthreads();
    if (wid == 0) {
        Xz t = lane < WSUM_WARPS ? xyzz_load<FQ>(&sm_a[lane][0]) : xyzz_identity<FQ>();
#pragma unroll 1
        for (u32 o = 1; o < WSUM_WARPS; o <<= 1) {
            Xz y = xyzz_shfl_down(t, o);
            if (lane + o < WSUM_WARPS) t = xyzz_add<FQ, ReduceMul>(t, y);
        }
        if (lane < WSUM_WARPS) xyzz_store(&sm_b[lane][0], t);  // suffix over warps >= lane
    }
    __syncthreads();
    Xz later = wid + 1 < WSUM_WARPS ? xyzz_load<FQ>(&sm_b[wid + 1][0]) : xyzz_identity<FQ>();
    Xz ex = xyzz_shfl_down(x, 1);
    if (lane == 31) ex = xyzz_identity<FQ>();
    ex = xyzz_add<FQ, ReduceMul>(ex, later);
    ex = xyzz_dbl_n<FQ, ReduceMul>(ex, ilog2(g));
    Xz rs = xyzz_add<FQ, ReduceMul>(sos, ex);  // this group's share of sum_w w * S_w
#pragma unroll 1
    for (u32 o = 16; o; o >>= 1) {
        rs = xyzz_add<FQ, ReduceMul>(rs, xyzz_shfl_down(rs, o));
        vsum = xyzz_add<FQ, ReduceMul>(vsum, xyzz_shfl_down(vsum, o));
    }
    __syncthreads();
    if (lane == 0) {
        xyzz_store(&sm_a[wid][0], rs);
        xyzz_store(&sm_b[wid][0], vsum);
    }
    __syncthreads();
    if (wid == 0) {
        Xz r2 = lane < WSUM_WARPS ? xyzz_load<FQ>(&sm_a[lane][0]) : xyzz_identity<FQ>();
        Xz v2 = lane < WSUM_WARPS ? xyzz_load<FQ>(&sm_b[lane][0]) : xyzz_identity<FQ>();
#pragma unroll 1
        for (u32 o = WSUM_WARPS / 2; o; o >>= 1) {
            r2 = xyzz_add<FQ, ReduceMul>(r2, xyzz_shfl_down(r2, o));
            v2 = xyzz_add<FQ, ReduceMul>(v2, xyzz_shfl_down(v2, o));
        }
        if (lane == 0) {
            const u32 shift = ilog2(wd.chunk) + 5;  // 32 lanes per warp partial
            r2 = xyzz_dbl_n<FQ, ReduceMul>(r2, shift);
            xyzz_store(a.wres + (size_t)win * C::XW, xyzz_add<FQ, ReduceMul>(v2, r2));
        }
    }
}

// ------------------------------------------------------ reduction tree
//
// After k_reduce, window total T = sum_g A_g + K * sum_g g * S_g over the
// window's partials g (A = V, S of the reduce warps, K = 32 L).  One warp per
// group of 32 consecutive partials g = 32 r + j folds them into one:
//   A'_r = sum_j A_{32r+j} + K * sum_j j * S_{32r+j},   S'_r = sum_j S_{32r+j},
// so that T = sum_r A'_r + 32 K * sum_r r * S'_r: the same form with K' = 32 K.
// sum_j j * S_j = sum_{i >= 1} x_i for the inclusive suffix sums x of S.  A
// window whose partials fit one group ends there: its total is A'_0.  Every
// level is one launch over the groups of every window, so the tail runs on
// many SMs instead of one block per window.

struct TreeGroup {
    u32 in_base;   // first input partial slot
    u32 in_count;  // 1..32 partials
    u32 out;       // output partial slot, or TREE_FINAL | window
    u32 shift;     // log2 K of the input level
};
static constexpr u32 TREE_FINAL = 0x80000000u;
static constexpr u32 TREE_BLOCK = 128;
static constexpr u32 TREE_WARPS = TREE_BLOCK / 32;

struct TreeArgs {
    const TreeGroup *groups;  // this level's groups
    u32 count;
    u32 *parts_v;             // A per partial slot
    u32 *parts_s;             // S per partial slot
    u32 *wres;                // window totals
};

template <class C>
__global__ void __launch_bounds__(TREE_BLOCK, C::XW == 32 ? 2 : 1) k_reduce_tree(TreeArgs a) {
    using FQ = typename C::Fq;
    using Xz = XyzzT<FQ>;
    const u32 g = blockIdx.x * TREE_WARPS + (threadIdx.x >> 5);
    if (g >= a.count) return;  // whole warps leave together
    const u32 lane = threadIdx.x & 31u;
    const TreeGroup gr = a.groups[g];
    Xz A = xyzz_identity<FQ>(), x = xyzz_identity<FQ>();
    if (lane < gr.in_count) {
        A = xyzz_load<FQ>(a.parts_v + (size_t)(gr.in_base + lane) * C::XW);
        x = xyzz_load<FQ>(a.parts_s + (size_t)(gr.in_base + lane) * C::XW);
    }
    // Lanes at or above in_count hold the identity; P, the next power of two
    // at or above in_count, bounds every step below (a window's last group
    // is often small).
    u32 P = 1;
    while (P < gr.in_count) P <<= 1;
    // inclusive suffix sums of S
#pragma unroll 1
    for (u32 o = 1; o < P; o <<= 1) {
        Xz y = xyzz_shfl_down(x, o);
        if (lane + o < 32) x = xyzz_add<FQ, TailMul>(x, y);
    }
    Xz w = lane ? x : xyzz_identity<FQ>();
    // The sums of A and of w over the group: the first step folds lanes l
    // and l + P/2 so that lanes below P/2 carry partial sums of A and lanes
    // P/2 .. P-1 of w, then each half reduces on its own -- one addition per
    // step, not two.  Lane 0 ends with the sum of A, lane P/2 with that of w.
    const u32 half = P >> 1;
    Xz v = A;
    if (half) {
        v = xyzz_add<FQ, TailMul>(lane < half ? A : w, xyzz_shfl_xor(lane < half ? w : A, half));
#pragma unroll 1
        for (u32 o = half >> 1; o; o >>= 1) v = xyzz_add<FQ, TailMul>(v, xyzz_shfl_xor(v, o));
    }
    if (lane == half && half) v = xyzz_dbl_n<FQ, TailMul>(v, gr.shift);
    w = half ? xyzz_shfl_down(v, half) : xyzz_identity<FQ>();
    if (lane == 0) {
        A = xyzz_add<FQ, TailMul>(v, w);
        if (gr.out & TREE_FINAL) {
            xyzz_store(a.wres + (size_t)(gr.out & ~TREE_FINAL) * C::XW, A);
        } else {
            xyzz_store(a.parts_v + (size_t)gr.out * C::XW, A);
            xyzz_store(a.parts_s + (size_t)gr.out * C::XW, x);
        }
    }
}

struct FinalArgs {
    const MsmDesc *descs;
    const u32 *wres;
    u32 M;
    u32 *carry;       // optional XYZZ per MSM: added in, or written when !emit_affine
    int emit_affine;  // write canonical affine results
    u32 *results;     // one affine point (C::PW words) per MSM
};

// One thread per MSM: Horner over its windows, sum_w 2^(c w) T_w with
// c * (windows - 1) doublings (in Jacobian form between the additions),
// then the carry and the affine form.
template <class C>
__global__ void k_final(FinalArgs f) {
    using FQ = typename C::Fq;
    const u32 m = blockIdx.x * blockDim.x + threadIdx.x;
    if (m >= f.M) return;
    const MsmDesc d = f.descs[m];
    XyzzT<FQ> acc = xyzz_identity<FQ>();
    for (int w = (int)d.n_windows - 1; w >= 0; w--) {
        acc = xyzz_dbl_n<FQ, FinalMul>(acc, d.c);
        acc = xyzz_add<FQ, FinalMul>(acc, xyzz_load<FQ>(f.wres + (size_t)(d.win_base + w) * C::XW));
    }
    if (f.carry) acc = xyzz_add<FQ, FinalMul>(acc, xyzz_load<FQ>(f.carry + (size_t)m * C::XW));
    if (f.emit_affine) {
        affine_store(f.results + (size_t)m * C::PW, xyzz_to_affine_fast<FQ, FinalMul>(acc));
    } else {
        xyzz_store(f.carry + (size_t)m * C::XW, acc);
    }
}

// Sum of k XYZZ points (per-card partials) to canonical affine.
template <class C>
__global__ void k_combine(const u32 *xyzz, u32 k, u32 *out) {
    using FQ = typename C::Fq;
    if (blockIdx.x || threadIdx.x) return;
    XyzzT<FQ> acc = xyzz_identity<FQ>();
    for (u32 i = 0; i < k; i++) acc = xyzz_add<FQ, FinalMul>(acc, xyzz_load<FQ>(xyzz + (size_t)i * C::XW));
    affine_store(out, xyzz_to_affine_fast<FQ, FinalMul>(acc));
}

}  // namespace impeller
