// Host-side MSM engine: plans a batch of MSMs over one device point array,
// lays out its device scratch, and enqueues the kernel sequence on a stream.
#pragma once

#include <cuda_runtime.h>

#include <cstdint>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <utility>
#include <vector>

namespace impeller {

typedef uint32_t u32;
typedef uint64_t u64;

void set_error(const std::string &msg);
const char *last_error();

// Curves (the reference's MSM_CURVE values bn254 and bls12381).
enum : u32 { CURVE_BN254 = 0, CURVE_BLS12381 = 1 };

// Affine point and XYZZ point size in 32-bit words, per curve.
inline u32 point_words(u32 curve) { return curve == CURVE_BLS12381 ? 24u : 16u; }
inline u32 xyzz_words(u32 curve) { return curve == CURVE_BLS12381 ? 48u : 32u; }

// Shape of one MSM in a plan (every MSM of a plan is on the same curve).
struct MsmShape {
    u32 n;             // points / scalars
    u32 c;             // window bits
    u32 n_windows;     // bucket sets (physical windows); 0 -> one per digit window
    u32 table_stride;  // points per window table (used when n_windows < digit windows)
    u32 table_base;    // point index of this MSM's table 0
    u32 curve;         // CURVE_BN254 or CURVE_BLS12381
};

// Signed-digit windows of width c for the curve's scalars: the fewest that
// keep the top digit plus its incoming carry at most 2^(c-1).  BN254
// (r < 2^254): ceil(254 / c); BLS12-381 (r < 2^255): ceil(255 / c) or one
// more (c = 3, 5, 15, 17).
u32 digit_windows(u32 c, u32 curve = CURVE_BN254);
u32 default_window(u64 n);  // autotune table (or the cost model)
u32 table_window(u64 n);    // tables window the autotune table recommends (0: none)
u32 curve_window(u32 c, u32 curve);  // c moved off windows that need an extra digit window on the curve

// Device property cache.
int sm_count(int device);

struct PlanLayout {
    size_t o_tables, tables_bytes;  // descs | wins | reduce blocks | sort tiles (uploaded each run)
    size_t o_counts, o_cursor, o_offsets, o_tiles, o_entries, o_buckets;
    size_t o_recb, o_recp, o_parts, o_parts_s, o_wres, o_long, o_carry, o_results;
    // two-level sort
    size_t o_cnt, o_coff, o_ccur, o_ctiles, o_centry, o_cfine, o_segs, o_binseg, o_nsegs, o_seghist, o_segcur;
    size_t bytes;
};

class Plan {
  public:
    // Every MSM reads points[table_base + (w / n_windows) * table_stride + i].
    static bool build(Plan &p, int device, const std::vector<MsmShape> &shapes);
    // Whether a plan of these shapes would sort its entries with the
    // two-level counting sort (fast) rather than the per-entry atomic sort
    // that build() falls back to for very large batches.
    static bool two_level_sort(const std::vector<MsmShape> &shapes);
    ~Plan();

    // Enqueue one run.  scalars[m] are device pointers.  carry_mode:
    // 0 = plain (results are affine), 1 = add the XYZZ carry in and emit
    // affine, 2 = add the carry in and keep XYZZ in the carry (no affine).
    // results may be null (results stay in scratch at layout.o_results).
    // carry_ext, when given, replaces the plan's own carry slots (M XYZZ).
    cudaError_t enqueue(void *scratch, const u32 *points, const u32 *const *scalars, u32 *results, int carry_mode,
                        cudaStream_t stream, u32 *carry_ext = nullptr);
    // enqueue == stage (host: write the pinned table image with these scalar
    // pointers, after the previous run's copy of it finished) + launch
    // (stream: copy the image, run the kernels).  launch alone is what a
    // CUDA graph captures; stage before every replay.
    cudaError_t stage(const u32 *const *scalars);
    // Use a caller-owned pinned buffer for the table image instead of one
    // the plan allocates (and frees, which can synchronize the device).  The
    // caller must not reuse it while a launch of this plan may still read it.
    void set_staging(void *pinned, size_t cap) {
        ext_staging = pinned;
        ext_cap = cap;
    }
    size_t staging_bytes() const { return tables.size(); }
    // record_staged = false while capturing a CUDA graph: an event recorded
    // inside a capture cannot be waited on from the host, so the graph's
    // caller marks the staging buffer free after the graph launch instead.
    cudaError_t launch(void *scratch, const u32 *points, u32 *results, int carry_mode, cudaStream_t stream,
                       u32 *carry_ext = nullptr, bool record_staged = true);
    cudaError_t mark_staged(cudaStream_t stream);

    // Streamed accumulation, for points that arrive in chunks: each chunk
    // (this plan's MSMs over the chunk's points and scalars) sorts and
    // accumulates its points straight into `acc` (nb XYZZ, caller-owned;
    // first = set every bucket to the identity before).  launch_chunked_tail reduces `acc`
    // and emits results as launch does.  Every plan used on one `acc` must
    // have the same window structure (same c, windows and MSM count).
    // d_image: the chunk's table image (write_image) already on the device;
    // null = stage() before and upload on the stream as launch does.
    // points_ready: when given, the stream waits for it after the sort and
    // before the accumulation (the sort reads only the scalars, so it can run
    // while the chunk's points are still being copied).
    cudaError_t launch_chunk(void *scratch, const u32 *points, u32 *acc, bool first, cudaStream_t stream,
                             const void *d_image = nullptr, cudaEvent_t points_ready = nullptr);
    cudaError_t launch_chunked_tail(void *scratch, const u32 *acc, u32 *results, int carry_mode,
                                    cudaStream_t stream, u32 *carry_ext = nullptr, const void *d_image = nullptr);
    size_t acc_bytes() const { return (size_t)nb * xyzz_words(curve) * 4; }
    // The table image (descriptors with these scalar pointers, windows,
    // reduce blocks) as launch uploads it, written to host memory at dst.
    size_t image_bytes() const;
    void write_image(void *dst, const u32 *const *scalars) const;

    size_t scratch_bytes() const { return layout.bytes; }
    u32 launches() const;
    u32 *carry_ptr(void *scratch) const;
    u32 *results_ptr(void *scratch) const;

    int device = 0;
    u32 curve = CURVE_BN254;
    u32 M = 0;
    u32 nb = 0, nb_pad = 0, ntiles = 0;
    u64 max_entries = 0;
    u32 accum_blocks = 0, accum_block = 256;
    u32 nparts = 0, long_cap = 0;
    u32 hist_grid_x = 1;
    // two-level sort (msd) or per-entry atomic bucket sort
    bool msd = false;
    u32 nbins = 0, sort_tiles = 0, tile_scalars = 0, segcap = 0, cnt_pad = 0, cscan_tiles = 0, ncells = 0;
    std::vector<MsmShape> shapes;
    PlanLayout layout{};

    // Per-phase timing: when enabled, every launch records CUDA events on the
    // launching stream between phases; read_profile sums the recorded runs.
    static constexpr int NPHASE = 8;
    static const char *phase_name(int i);
    void set_profiling(bool on) { profiling = on; }
    cudaError_t read_profile(double *ms_per_phase, u32 *runs);

    Plan() = default;
    Plan(const Plan &) = delete;
    Plan &operator=(const Plan &) = delete;

  private:
    // bucket_out: accumulate into these buckets, each starting from its
    // current value (streamed chunks); null = the plan's own buckets, fresh.
    cudaError_t run_front(void *scratch, const u32 *points, cudaStream_t stream, bool record_staged,
                          const void *d_image, u32 *bucket_out = nullptr, cudaEvent_t points_ready = nullptr);
    cudaError_t run_tail(void *scratch, const u32 *buckets, bool dense, u32 *results, int carry_mode,
                         cudaStream_t stream, u32 *carry_ext, const void *d_image);

    void *staging = nullptr;     // pinned copy of the tables
    void *ext_staging = nullptr; // caller-owned staging (set_staging)
    size_t ext_cap = 0;
    cudaEvent_t staged = nullptr;
    std::vector<unsigned char> tables;  // host image of the tables
    size_t desc_off = 0, win_off = 0, blk_off = 0, tf_off = 0, bc_off = 0, tree_off = 0;
    u32 nwins = 0, nrblocks = 0;
    std::vector<u32> tree_first;  // reduction tree: first group of each level (+ total)
    bool profiling = false;
    std::vector<std::vector<cudaEvent_t>> prof_sets;  // one set of NPHASE+1 events per run
    u32 prof_used = 0;
    cudaError_t prof_mark(int k, cudaStream_t st);
};

// k_combine: sum `k` XYZZ points in device memory, write canonical affine.
cudaError_t combine_xyzz(const u32 *d_xyzz, u32 k, u32 *d_out, cudaStream_t stream, u32 curve = CURVE_BN254);

// Window tables 2^(j*shift)*P for j in 1..n_tables-1, in place after table 0.
cudaError_t precompute_tables(u32 *d_points, u64 n, u32 shift, u32 n_tables, cudaStream_t stream,
                              u32 curve = CURVE_BN254);

}  // namespace impeller

// Resident-SRS context (the C ABI's opaque impeller_ctx).
struct impeller_ctx {
    int device = 0;
    impeller::u32 curve = impeller::CURVE_BN254;
    const impeller::u32 *points = nullptr;
    impeller::u64 len = 0;
    bool owns = false;
    std::mutex mu;
    void *scratch = nullptr;
    size_t scratch_bytes = 0;
    impeller::u32 *d_scalars = nullptr;  // staging for impeller_msm_host
    impeller::u64 d_scalars_cap = 0;
    impeller::u32 *d_result = nullptr;
    cudaEvent_t done = nullptr;  // last run that used the scratch
    bool profiling = false;
    // Resident window tables: one allocation holding the points (region 0)
    // followed by table sets; the set for window c has W(c) tables of len
    // points, table j = 2^(j*c) * P, starting at point index base.
    impeller::u32 *tables = nullptr;
    impeller::u64 tables_points = 0;  // points held by `tables`
    std::vector<std::pair<impeller::u32, impeller::u32>> sets;  // (c, base)
    std::map<std::pair<impeller::u32, impeller::u32>, std::unique_ptr<impeller::Plan>> plans;
};

namespace impeller {
u32 ctx_set_base(const impeller_ctx *ctx, u32 c);            // NONE if no set for c
u32 ctx_window(const impeller_ctx *ctx, u64 n);              // window an MSM of n points uses
MsmShape ctx_shape(const impeller_ctx *ctx, u32 n, u32 c);   // plan shape on this context
const u32 *ctx_point_base(const impeller_ctx *ctx);          // points (and table sets) base
}  // namespace impeller
