// The reference's C ABI, msm() and msm_precompute(), on the B200 engine.
//
// Semantics follow core/src/msm/src/msm.cu:9-49 and the classes it drives in
// core/src/msm/src/msm_impl.cuh:
//   - buffers == NULL: write the per-card scratch size and return
//     (msm.cu:20-22, alloc_gpu at msm_impl.cuh:625-656);
//   - the len points are split into num_cards equal ranges, one per card
//     (MultiGPUMSM, msm_impl.cuh:832-844); each card splits its range into
//     `parts` chunks that are uploaded and processed in turn (MSM::run,
//     msm_impl.cuh:374-547), and runs `batch_per_run` scalar vectors per pass
//     over the uploaded points (MSM::msm, msm_impl.cuh:735-749);
//   - window j's points come from table j / n_windows (distribute_windows,
//     msm_impl.cuh:56-68);
//   - the result of each batch is written as a 16-word affine point in
//     Montgomery form, identity (0,0) (msm.cu:37-39).
// Unlike the reference, the per-part and per-card partial sums are added on
// the device, and only the canonical affine result leaves the GPU.
//
// Uploads stream: a card's points and scalars are copied in chunks on a copy
// stream while the previous chunk is sorted and accumulated on the compute
// stream; every chunk adds its bucket sums into the card's accumulators and
// the bucket reduction runs once per batch group, as the reference
// accumulates all parts into one bucket set before reducing
// (msm_impl.cuh:384-575).  With parts == 1 the whole card range stays
// resident (later batch groups reuse the points) and is streamed in chunks
// that start at 2^18 points and grow (stream_bounds); with parts > 1 each
// part is a chunk, double-buffered
// in two stages (the reference's stage_scalers / stage_points = 2 that
// get_best_config pairs with parts > 1, core/src/msm.rs:89).
#include <algorithm>
#include <cstdio>
#include <map>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "../../include/impeller_msm.h"
#include "engine.h"

using namespace impeller;

namespace {

#define CK(x)                                                                                   \
    do {                                                                                        \
        cudaError_t _e = (x);                                                                   \
        if (_e != cudaSuccess) {                                                                \
            set_error(std::string(#x) + " failed: " + cudaGetErrorString(_e));                  \
            return _e;                                                                          \
        }                                                                                       \
    } while (0)

size_t align_up(size_t x, size_t a) { return (x + a - 1) / a * a; }

struct Config {
    u32 c, W, n_windows, n_tables;
    bool debug;
    u32 curve;
    u32 PW, XW;  // affine and XYZZ point words
};

bool make_config(unsigned window_size, unsigned target_window, int debug, Config &cfg, u32 curve = CURVE_BN254) {
    if (curve != CURVE_BN254 && curve != CURVE_BLS12381) {
        set_error("unknown curve");
        return false;
    }
    if (window_size < 3 || window_size > 31) {
        set_error("window_size must be in [3, 31]");
        return false;
    }
    if (target_window == 0) {
        set_error("target_window must be at least 1");
        return false;
    }
    cfg.c = window_size;
    cfg.curve = curve;
    cfg.PW = point_words(curve);
    cfg.XW = xyzz_words(curve);
    cfg.W = digit_windows(window_size, curve);
    cfg.n_windows = std::min(cfg.W, target_window);
    cfg.n_tables = (cfg.W + cfg.n_windows - 1) / cfg.n_windows;
    cfg.debug = debug != 0;
    // The caller allocates the reference's number of window tables,
    // ceil(ceil(bits / c) / n_windows) (common/src/msm_config.rs:17-25).
    // BLS12-381 scalars need one more signed-digit window than ceil(255 / c)
    // for c = 3, 5, 15, 17; refuse a configuration whose table count would
    // then differ from the caller's.
    const u32 bits = curve == CURVE_BLS12381 ? 255u : 254u;
    const u32 ref_w = (bits + window_size - 1) / window_size;
    const u32 ref_nw = std::min(ref_w, target_window);
    const u32 ref_tables = (ref_w + ref_nw - 1) / ref_nw;
    if (ref_tables == 1) {
        // no window tables: every digit window gets its own bucket set
        cfg.n_windows = cfg.W;
        cfg.n_tables = 1;
    }
    if (ref_tables != cfg.n_tables) {
        set_error("window size " + std::to_string(window_size) + " with target window " +
                  std::to_string(target_window) +
                  " needs one more signed-digit window than the reference's table layout on this curve");
        return false;
    }
    return true;
}

// Per-card carve-out of the caller's buffer.
struct CardLayout {
    u64 card_off = 0, card_len = 0, part_len = 0;
    size_t o_points = 0, o_scalars = 0, o_carry = 0, o_results = 0, o_combine = 0, o_plan = 0, o_acc = 0;
    size_t o_images = 0, image_cap = 0, bytes = 0;  // streamed: one table image per chunk
};

// Chunk boundaries of a resident (parts == 1) range of `len` points that
// streams in: one chunk (no streaming) below 2^21 points; else a first chunk
// of 2^18 points, so that computing starts after a short upload, and chunks
// growing by 7/4, about the ratio of a chunk's compute time to its upload
// time, so that each chunk lands while the previous one is still being
// computed.  A remainder under half the next size joins the last chunk.
std::vector<u64> stream_bounds(u64 len) {
    std::vector<u64> b{0};
    if (len < (1ull << 21)) {
        b.push_back(len);
        return b;
    }
    u64 size = 1ull << 18, at = 0;
    while (at < len) {
        u64 take = std::min(size, len - at);
        if (len - at - take < size / 2) take = len - at;
        at += take;
        b.push_back(at);
        size = size * 7 / 4;
    }
    return b;
}

u32 stream_chunks(u64 len) { return (u32)stream_bounds(len).size() - 1; }

// parts > 1: each part is a chunk, in one of two buffer stages.
constexpr u32 PART_STAGES = 2;

std::vector<MsmShape> group_shapes(const Config &cfg, u32 M, u32 n, u32 part_len) {
    std::vector<MsmShape> s(M, MsmShape{n, cfg.c, cfg.n_windows, part_len, 0, cfg.curve});
    return s;
}

bool card_layout(const Config &cfg, int device, u64 len, u32 num_cards, u32 card, u32 parts, u32 batch_per_run,
                 CardLayout &L, size_t &plan_bytes) {
    const u64 per_card = (len + num_cards - 1) / num_cards;
    L.card_off = std::min<u64>(len, (u64)card * per_card);
    L.card_len = std::min<u64>(per_card, len - L.card_off);
    L.part_len = (L.card_len + parts - 1) / parts;
    if (L.part_len * cfg.n_tables >= (1ull << 31)) {
        set_error("part length times window tables exceeds 2^31 points; raise `parts`");
        return false;
    }
    plan_bytes = 0;
    size_t acc_bytes = 0, images = 0;
    if (L.part_len) {
        Plan p;
        if (!Plan::build(p, device, group_shapes(cfg, batch_per_run, (u32)L.part_len, (u32)L.part_len))) return false;
        plan_bytes = p.scratch_bytes();
        const u64 nchunks = parts > 1 ? (L.card_len + L.part_len - 1) / L.part_len : stream_chunks(L.card_len);
        if (nchunks > 1) {
            acc_bytes = p.acc_bytes();
            L.image_cap = align_up(p.image_bytes(), 256);
            images = nchunks * L.image_cap;
        }
    }
    const size_t stages = parts > 1 ? PART_STAGES : 1;
    size_t off = 0;
    auto take = [&](size_t b) {
        size_t o = off;
        off = align_up(off + b, 256);
        return o;
    };
    L.o_points = take(stages * cfg.n_tables * L.part_len * cfg.PW * 4);
    L.o_scalars = take(stages * batch_per_run * L.part_len * 32);
    L.o_carry = take((size_t)batch_per_run * cfg.XW * 4);
    L.o_results = take((size_t)batch_per_run * cfg.PW * 4);
    L.o_combine = take((size_t)num_cards * cfg.XW * 4 + cfg.PW * 4);
    L.o_plan = take(plan_bytes);
    L.o_acc = take(acc_bytes);
    L.o_images = take(images);
    L.bytes = off;
    return true;
}

// One compute stream (role 0) and one copy stream (role 1) per device, kept
// for the life of the process.
cudaStream_t device_stream(int device, int role = 0) {
    static std::mutex mu;
    static std::map<std::pair<int, int>, cudaStream_t> streams;
    std::lock_guard<std::mutex> g(mu);
    auto key = std::make_pair(device, role);
    auto it = streams.find(key);
    if (it != streams.end()) return it->second;
    cudaStream_t s = nullptr;
    if (cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking) != cudaSuccess) return nullptr;
    streams[key] = s;
    return s;
}

// Events of one streamed call, destroyed with it.
struct EventPool {
    std::vector<cudaEvent_t> ev;
    cudaEvent_t get() {
        cudaEvent_t e = nullptr;
        if (cudaEventCreateWithFlags(&e, cudaEventDisableTiming) != cudaSuccess) return nullptr;
        ev.push_back(e);
        return e;
    }
    ~EventPool() {
        for (cudaEvent_t e : ev) cudaEventDestroy(e);
    }
};

struct CardJob {
    const Config *cfg;
    int device;
    void *buffer;
    CardLayout L;
    u32 parts, batch_per_run, batches, num_cards;
    unsigned int const *const *h_points;
    unsigned int const *const *h_scalars;
    unsigned int *const *h_result;        // single card: results written directly
    std::vector<u32> partials;            // multi card: batches x 32 u32 (XYZZ)
    cudaError_t status = cudaSuccess;
    std::string error;
};

// Plans persist per device across calls (their pinned table images and
// events are the costly part to create); calls on one device are serialized.
// Each call takes a new generation; a plan used by the current call carries
// it and is never evicted, so a call may hold more plans than the cap.
struct CachedPlan {
    std::unique_ptr<Plan> plan;
    u64 gen = 0;  // generation of the last call that used it
};

struct DevicePlans {
    std::mutex mu;
    std::map<std::vector<u32>, CachedPlan> plans;
    std::vector<std::vector<u32>> order;  // oldest first
    u64 gen = 0;                          // current call
    void *host_images = nullptr;          // pinned: the chunk table images of one call
    size_t host_images_cap = 0;
};

DevicePlans &device_plans(int device) {
    static std::mutex mu;
    static std::map<int, std::unique_ptr<DevicePlans>> all;
    std::lock_guard<std::mutex> g(mu);
    auto &p = all[device];
    if (!p) p.reset(new DevicePlans());
    return *p;
}

constexpr size_t PLAN_CACHE_CAP = 32;

Plan *cached_plan(DevicePlans &D, int device, const Config &cfg, u32 M, u32 n, u32 stride) {
    std::vector<u32> key{cfg.c, cfg.n_windows, M, n, stride, cfg.curve};
    auto it = D.plans.find(key);
    if (it != D.plans.end()) {
        it->second.gen = D.gen;
        return it->second.plan.get();
    }
    if (D.plans.size() >= PLAN_CACHE_CAP) {
        // evict the oldest plan that the current call has not used
        for (size_t k = 0; k < D.order.size(); k++) {
            auto victim = D.plans.find(D.order[k]);
            if (victim->second.gen == D.gen) continue;
            D.plans.erase(victim);
            D.order.erase(D.order.begin() + k);
            break;
        }
    }
    std::unique_ptr<Plan> p(new Plan());
    if (!Plan::build(*p, device, group_shapes(cfg, M, n, stride))) return nullptr;
    Plan *raw = p.get();
    D.plans[key] = CachedPlan{std::move(p), D.gen};
    D.order.push_back(key);
    return raw;
}

cudaError_t run_card(CardJob &J) {
    const Config &cfg = *J.cfg;
    CK(cudaSetDevice(J.device));
    DevicePlans &D = device_plans(J.device);
    std::lock_guard<std::mutex> hold(D.mu);
    D.gen++;  // plans this call uses are pinned in the cache until the next call
    cudaStream_t st = device_stream(J.device, 0), cs = device_stream(J.device, 1);
    if (!st || !cs) {
        set_error("could not create a stream");
        return cudaErrorUnknown;
    }
    unsigned char *base = static_cast<unsigned char *>(J.buffer);
    u32 *d_points = reinterpret_cast<u32 *>(base + J.L.o_points);
    u32 *d_scalars = reinterpret_cast<u32 *>(base + J.L.o_scalars);
    u32 *d_carry = reinterpret_cast<u32 *>(base + J.L.o_carry);
    u32 *d_results = reinterpret_cast<u32 *>(base + J.L.o_results);
    u32 *d_acc = reinterpret_cast<u32 *>(base + J.L.o_acc);
    void *plan_scratch = base + J.L.o_plan;
    const bool multi = J.num_cards > 1;
    const u32 PW = cfg.PW, XW = cfg.XW;
    if (multi) J.partials.assign((size_t)J.batches * XW, 0);
    const u64 part_len = J.L.part_len, card_len = J.L.card_len;
    const bool staged = J.parts > 1;
    const u32 stride = (u32)part_len;  // distance between window tables in a points buffer
    const size_t point_stage = (size_t)cfg.n_tables * part_len * PW;  // u32 per stage
    EventPool events;

    // chunk k covers points [bounds[k], bounds[k + 1]) of the card range
    std::vector<u64> bounds;
    if (staged) {
        for (u64 at = 0; at < card_len; at += part_len) bounds.push_back(at);
        bounds.push_back(card_len);
    } else {
        bounds = stream_bounds(card_len);
    }
    const u32 nchunks = card_len ? (u32)bounds.size() - 1 : 0;

    bool points_resident = false;
    for (u32 g = 0; g < J.batches; g += J.batch_per_run) {
        const u32 M = std::min(J.batch_per_run, J.batches - g);
        if (card_len == 0) {
            // an empty range contributes the identity
            if (!multi)
                for (u32 b = 0; b < M; b++) std::fill(J.h_result[g + b], J.h_result[g + b] + cfg.PW, 0u);
            continue;
        }
        const int mode = multi ? 2 : 0;
        if (multi) CK(cudaMemsetAsync(d_carry, 0, (size_t)M * XW * 4, st));
        const size_t scalar_stage = (size_t)M * part_len * 8;  // u32 per stage
        cudaEvent_t t0 = nullptr, t1 = nullptr;
        if (cfg.debug) {
            cudaEventCreate(&t0);
            cudaEventCreate(&t1);
            cudaEventRecord(t0, st);
        }
        if (nchunks == 1) {
            // one chunk: upload, then the plain run
            if (!points_resident)
                for (u32 t = 0; t < cfg.n_tables; t++)
                    CK(cudaMemcpyAsync(d_points + (size_t)t * part_len * PW, J.h_points[t] + J.L.card_off * PW,
                                       card_len * PW * 4, cudaMemcpyHostToDevice, st));
            points_resident = !staged;
            std::vector<const u32 *> sc(M);
            for (u32 b = 0; b < M; b++) {
                u32 *dst = d_scalars + (size_t)b * part_len * 8;
                CK(cudaMemcpyAsync(dst, J.h_scalars[g + b] + J.L.card_off * 8, card_len * 32,
                                   cudaMemcpyHostToDevice, st));
                sc[b] = dst;
            }
            Plan *plan = cached_plan(D, J.device, cfg, M, (u32)card_len, stride);
            if (!plan) return cudaErrorInvalidValue;
            cudaError_t e = plan->enqueue(plan_scratch, d_points, sc.data(), d_results, mode, st, d_carry);
            if (e != cudaSuccess) return e;
        } else {
            // streamed: copies on cs, chunk k's compute on st once its data landed
            cudaEvent_t free_ev = events.get();
            if (!free_ev) return cudaErrorUnknown;
            CK(cudaEventRecord(free_ev, st));  // earlier work on st may still read the buffers
            CK(cudaStreamWaitEvent(cs, free_ev, 0));
            // every chunk's table image, written on the host and uploaded in one
            // copy ahead of the data (the previous call's copy has completed)
            const size_t img_bytes = (size_t)nchunks * J.L.image_cap;
            if (D.host_images_cap < img_bytes) {
                if (D.host_images) cudaFreeHost(D.host_images);
                D.host_images = nullptr;
                D.host_images_cap = 0;
                CK(cudaHostAlloc(&D.host_images, img_bytes, cudaHostAllocPortable));
                D.host_images_cap = img_bytes;
            }
            std::vector<Plan *> chunk_plan(nchunks, nullptr);
            for (u32 k = 0; k < nchunks; k++) {
                const u64 s0 = bounds[k];
                const u64 mk = bounds[k + 1] - s0;
                const u32 slot = staged ? k % PART_STAGES : 0;
                std::vector<const u32 *> sc(M);
                for (u32 b = 0; b < M; b++)
                    sc[b] = staged ? d_scalars + slot * scalar_stage + (size_t)b * part_len * 8
                                   : d_scalars + (size_t)b * part_len * 8 + s0 * 8;
                chunk_plan[k] = cached_plan(D, J.device, cfg, M, (u32)mk, stride);
                if (!chunk_plan[k]) return cudaErrorInvalidValue;
                if (chunk_plan[k]->image_bytes() > J.L.image_cap) {
                    set_error("msm: chunk table image exceeds its slot");
                    return cudaErrorInvalidValue;
                }
                chunk_plan[k]->write_image(static_cast<unsigned char *>(D.host_images) + k * J.L.image_cap, sc.data());
            }
            unsigned char *d_images = base + J.L.o_images;
            CK(cudaMemcpyAsync(d_images, D.host_images, img_bytes, cudaMemcpyHostToDevice, cs));
            std::vector<cudaEvent_t> computed(nchunks, nullptr);
            // debug: timing events per chunk (data landed, compute start, compute end)
            std::vector<cudaEvent_t> tl(cfg.debug ? 3 * nchunks : 0, nullptr);
            for (auto &e : tl) cudaEventCreate(&e);
            Plan *plan = nullptr;
            for (u32 k = 0; k < nchunks; k++) {
                const u64 s0 = bounds[k];
                const u64 mk = bounds[k + 1] - s0;
                const u32 slot = staged ? k % PART_STAGES : 0;
                if (staged && k >= PART_STAGES) CK(cudaStreamWaitEvent(cs, computed[k - PART_STAGES], 0));
                // the chunk's scalars first: its sort needs only them and runs
                // while its points are still being copied
                for (u32 b = 0; b < M; b++) {
                    u32 *dst = staged ? d_scalars + slot * scalar_stage + (size_t)b * part_len * 8
                                      : d_scalars + (size_t)b * part_len * 8 + s0 * 8;
                    CK(cudaMemcpyAsync(dst, J.h_scalars[g + b] + (J.L.card_off + s0) * 8, mk * 32,
                                       cudaMemcpyHostToDevice, cs));
                }
                cudaEvent_t scalars_landed = events.get();
                if (!scalars_landed) return cudaErrorUnknown;
                CK(cudaEventRecord(scalars_landed, cs));
                // points of this chunk: staged -> its stage buffer; resident -> in place
                u32 *pbase = staged ? d_points + slot * point_stage : d_points + s0 * PW;
                if (!points_resident)
                    for (u32 t = 0; t < cfg.n_tables; t++)
                        CK(cudaMemcpyAsync(pbase + (size_t)t * part_len * PW,
                                           J.h_points[t] + (J.L.card_off + s0) * PW, mk * PW * 4,
                                           cudaMemcpyHostToDevice, cs));
                cudaEvent_t landed = events.get();
                if (!landed) return cudaErrorUnknown;
                CK(cudaEventRecord(landed, cs));
                if (cfg.debug) cudaEventRecord(tl[3 * k], cs);
                CK(cudaStreamWaitEvent(st, scalars_landed, 0));
                if (cfg.debug) cudaEventRecord(tl[3 * k + 1], st);
                plan = chunk_plan[k];
                cudaError_t e = plan->launch_chunk(plan_scratch, pbase, d_acc, k == 0, st, d_images + k * J.L.image_cap,
                                                   landed);
                if (e != cudaSuccess) return e;
                if (cfg.debug) cudaEventRecord(tl[3 * k + 2], st);
                if (staged) {
                    computed[k] = events.get();
                    if (!computed[k]) return cudaErrorUnknown;
                    CK(cudaEventRecord(computed[k], st));
                }
            }
            points_resident = !staged;
            cudaError_t e = plan->launch_chunked_tail(plan_scratch, d_acc, d_results, mode, st, d_carry,
                                                      d_images + (size_t)(nchunks - 1) * J.L.image_cap);
            if (e != cudaSuccess) return e;
            if (cfg.debug) {
                cudaStreamSynchronize(st);
                for (u32 k = 0; k < nchunks; k++) {
                    float a = 0, b = 0, c = 0;
                    cudaEventElapsedTime(&a, t0, tl[3 * k]);
                    cudaEventElapsedTime(&b, t0, tl[3 * k + 1]);
                    cudaEventElapsedTime(&c, t0, tl[3 * k + 2]);
                    std::fprintf(stderr, "impeller msm:   chunk %u: landed %.3f ms, compute %.3f .. %.3f ms\n", k, a, b, c);
                }
                for (auto &ev : tl) cudaEventDestroy(ev);
            }
        }
        if (cfg.debug) {
            cudaEventRecord(t1, st);
            cudaEventSynchronize(t1);
            float ms = 0;
            cudaEventElapsedTime(&ms, t0, t1);
            std::fprintf(stderr, "impeller msm: card %d group %u n=%llu batch=%u chunks=%u: %.3f ms\n", J.device, g,
                         (unsigned long long)card_len, M, nchunks, ms);
            cudaEventDestroy(t0);
            cudaEventDestroy(t1);
        }
        if (!multi) {
            for (u32 b = 0; b < M; b++)
                CK(cudaMemcpyAsync(J.h_result[g + b], d_results + (size_t)b * PW, PW * 4, cudaMemcpyDeviceToHost,
                                   st));
        } else {
            CK(cudaMemcpyAsync(J.partials.data() + (size_t)g * XW, d_carry, (size_t)M * XW * 4, cudaMemcpyDeviceToHost,
                               st));
        }
        CK(cudaStreamSynchronize(st));
    }
    CK(cudaStreamSynchronize(st));
    return cudaSuccess;
}

}  // namespace

extern "C" {

unsigned int impeller_msm_n_precompute(unsigned int window_size, unsigned int target_window) {
    return impeller_msm_n_precompute_curve(IMPELLER_CURVE_BN254, window_size, target_window);
}

unsigned int impeller_msm_n_precompute_curve(unsigned int curve, unsigned int window_size,
                                             unsigned int target_window) {
    Config cfg;
    if (!make_config(window_size, target_window, 0, cfg, curve)) return 0;
    return cfg.n_tables;
}

cudaError_t impeller_msm_cfg(unsigned int window_size, unsigned int target_window, int debug, void *const *buffers,
                             unsigned long *buffer_sizes, unsigned long long len, unsigned int batch_per_run,
                             unsigned int parts, unsigned int stage_scalers, unsigned int stage_points,
                             unsigned int num_cards, const unsigned int *cards, unsigned int const *const *h_points,
                             unsigned int batches, unsigned int const *const *h_scaler_batch,
                             unsigned int *const *h_result) {
    return impeller_msm_cfg_curve(IMPELLER_CURVE_BN254, window_size, target_window, debug, buffers, buffer_sizes, len,
                                  batch_per_run, parts, stage_scalers, stage_points, num_cards, cards, h_points,
                                  batches, h_scaler_batch, h_result);
}

cudaError_t impeller_msm_cfg_curve(unsigned int curve, unsigned int window_size, unsigned int target_window,
                                   int debug, void *const *buffers, unsigned long *buffer_sizes,
                                   unsigned long long len, unsigned int batch_per_run, unsigned int parts,
                                   unsigned int stage_scalers, unsigned int stage_points, unsigned int num_cards,
                                   const unsigned int *cards, unsigned int const *const *h_points,
                                   unsigned int batches, unsigned int const *const *h_scaler_batch,
                                   unsigned int *const *h_result) {
    (void)stage_scalers;
    (void)stage_points;
    Config cfg;
    if (!make_config(window_size, target_window, debug, cfg, curve)) return cudaErrorInvalidValue;
    if (num_cards == 0 || !cards) {
        set_error("msm: at least one card is required");
        return cudaErrorInvalidValue;
    }
    if (parts == 0 || batch_per_run == 0) {
        set_error("msm: parts and batch_per_run must be at least 1");
        return cudaErrorInvalidValue;
    }
    std::vector<CardLayout> layouts(num_cards);
    for (u32 i = 0; i < num_cards; i++) {
        size_t pb = 0;
        if (!card_layout(cfg, (int)cards[i], len, num_cards, i, parts, batch_per_run, layouts[i], pb))
            return cudaErrorInvalidValue;
    }
    if (buffers == nullptr) {
        if (!buffer_sizes) {
            set_error("msm: size query needs buffer_sizes");
            return cudaErrorInvalidValue;
        }
        for (u32 i = 0; i < num_cards; i++) buffer_sizes[i] = (unsigned long)layouts[i].bytes;
        return cudaSuccess;
    }
    if (batches == 0) return cudaSuccess;
    if (!h_points || !h_scaler_batch || !h_result) {
        set_error("msm: null host array");
        return cudaErrorInvalidValue;
    }
    for (u32 t = 0; t < cfg.n_tables; t++)
        if (!h_points[t] && len) {
            set_error("msm: missing window table pointer");
            return cudaErrorInvalidValue;
        }
    for (u32 b = 0; b < batches; b++)
        if ((!h_scaler_batch[b] && len) || !h_result[b]) {
            set_error("msm: missing scalar or result pointer");
            return cudaErrorInvalidValue;
        }

    std::vector<CardJob> jobs(num_cards);
    for (u32 i = 0; i < num_cards; i++) {
        CardJob &J = jobs[i];
        J.cfg = &cfg;
        J.device = (int)cards[i];
        J.buffer = buffers[i];
        J.L = layouts[i];
        J.parts = parts;
        J.batch_per_run = batch_per_run;
        J.batches = batches;
        J.num_cards = num_cards;
        J.h_points = h_points;
        J.h_scalars = h_scaler_batch;
        J.h_result = h_result;
    }
    if (num_cards == 1) {
        return run_card(jobs[0]);
    }
    std::vector<std::thread> threads;
    for (u32 i = 0; i < num_cards; i++)
        threads.emplace_back([&jobs, i]() {
            jobs[i].status = run_card(jobs[i]);
            if (jobs[i].status != cudaSuccess) jobs[i].error = impeller::last_error();
        });
    for (auto &t : threads) t.join();
    for (auto &J : jobs)
        if (J.status != cudaSuccess) {
            set_error(J.error);
            return J.status;
        }
    // one exchange: each card's XYZZ partial to card 0, summed there
    CK(cudaSetDevice((int)cards[0]));
    cudaStream_t st = device_stream((int)cards[0]);
    unsigned char *base0 = static_cast<unsigned char *>(buffers[0]);
    u32 *d_comb = reinterpret_cast<u32 *>(base0 + layouts[0].o_combine);
    const u32 XW = cfg.XW, PW = cfg.PW;
    u32 *d_out = d_comb + (size_t)num_cards * XW;
    std::vector<u32> gather((size_t)num_cards * XW);
    for (u32 b = 0; b < batches; b++) {
        for (u32 i = 0; i < num_cards; i++)
            std::copy(jobs[i].partials.begin() + (size_t)b * XW, jobs[i].partials.begin() + (size_t)(b + 1) * XW,
                      gather.begin() + (size_t)i * XW);
        CK(cudaMemcpyAsync(d_comb, gather.data(), gather.size() * 4, cudaMemcpyHostToDevice, st));
        cudaError_t e = combine_xyzz(d_comb, num_cards, d_out, st, cfg.curve);
        if (e != cudaSuccess) return e;
        CK(cudaMemcpyAsync(h_result[b], d_out, PW * 4, cudaMemcpyDeviceToHost, st));
        CK(cudaStreamSynchronize(st));
    }
    return cudaSuccess;
}

cudaError_t impeller_msm_precompute_cfg(unsigned int window_size, unsigned int target_window,
                                        unsigned long long len, unsigned int *const *h_points,
                                        unsigned int max_cards) {
    return impeller_msm_precompute_cfg_curve(IMPELLER_CURVE_BN254, window_size, target_window, len, h_points,
                                             max_cards);
}

cudaError_t impeller_msm_precompute_cfg_curve(unsigned int curve, unsigned int window_size,
                                              unsigned int target_window, unsigned long long len,
                                              unsigned int *const *h_points, unsigned int max_cards) {
    Config cfg;
    if (!make_config(window_size, target_window, 0, cfg, curve)) return cudaErrorInvalidValue;
    const u64 PW = cfg.PW;
    if (cfg.n_tables == 1 || len == 0) return cudaSuccess;
    if (!h_points) {
        set_error("msm_precompute: null h_points");
        return cudaErrorInvalidValue;
    }
    int ndev = 0;
    CK(cudaGetDeviceCount(&ndev));
    const int devices = std::max(1, std::min(ndev, (int)std::max(1u, max_cards)));
    const u64 per = (len + devices - 1) / devices;
    const u32 shift = cfg.n_windows * cfg.c;
    std::vector<cudaError_t> status(devices, cudaSuccess);
    std::vector<std::string> errs(devices);
    auto work = [&](int dev) -> cudaError_t {
        const u64 off = std::min<u64>(len, (u64)dev * per);
        const u64 cnt = std::min<u64>(per, len - off);
        if (cnt == 0) return cudaSuccess;
        CK(cudaSetDevice(dev));
        cudaStream_t st = device_stream(dev);
        const u64 chunk = std::min<u64>(cnt, 1ull << 20);
        u32 *d = nullptr;
        CK(cudaMalloc(&d, (size_t)cfg.n_tables * chunk * PW * 4));
        cudaError_t e = cudaSuccess;
        for (u64 s = 0; s < cnt && e == cudaSuccess; s += chunk) {
            const u64 m = std::min<u64>(chunk, cnt - s);
            e = cudaMemcpyAsync(d, h_points[0] + (off + s) * PW, m * PW * 4, cudaMemcpyHostToDevice, st);
            if (e == cudaSuccess) e = precompute_tables(d, m, shift, cfg.n_tables, st, cfg.curve);
            for (u32 t = 1; t < cfg.n_tables && e == cudaSuccess; t++)
                e = cudaMemcpyAsync(h_points[t] + (off + s) * PW, d + (size_t)t * m * PW, m * PW * 4,
                                    cudaMemcpyDeviceToHost, st);
            if (e == cudaSuccess) e = cudaStreamSynchronize(st);
        }
        cudaFree(d);
        if (e != cudaSuccess) set_error(std::string("msm_precompute: ") + cudaGetErrorString(e));
        return e;
    };
    std::vector<std::thread> th;
    for (int d = 0; d < devices; d++)
        th.emplace_back([&, d]() {
            status[d] = work(d);
            if (status[d] != cudaSuccess) errs[d] = impeller::last_error();
        });
    for (auto &t : th) t.join();
    for (int d = 0; d < devices; d++)
        if (status[d] != cudaSuccess) {
            set_error(errs[d]);
            return status[d];
        }
    return cudaSuccess;
}

#ifndef IMPELLER_DEFAULT_WINDOW
#define IMPELLER_DEFAULT_WINDOW 16
#endif
#ifndef IMPELLER_DEFAULT_TARGET
#define IMPELLER_DEFAULT_TARGET 16
#endif

cudaError_t msm(void *const *buffers, unsigned long *buffer_sizes, unsigned long long len, unsigned int batch_per_run,
                unsigned int parts, unsigned int stage_scalers, unsigned int stage_points, unsigned int num_cards,
                const unsigned int *cards, unsigned int const *const *h_points, unsigned int batches,
                unsigned int const *const *h_scaler_batch, unsigned int *const *h_result) {
    return impeller_msm_cfg(IMPELLER_DEFAULT_WINDOW, IMPELLER_DEFAULT_TARGET, 0, buffers, buffer_sizes, len,
                            batch_per_run, parts, stage_scalers, stage_points, num_cards, cards, h_points, batches,
                            h_scaler_batch, h_result);
}

cudaError_t msm_precompute(unsigned long long len, unsigned int *const *h_points, unsigned int max_cards) {
    return impeller_msm_precompute_cfg(IMPELLER_DEFAULT_WINDOW, IMPELLER_DEFAULT_TARGET, len, h_points, max_cards);
}

}  // extern "C"
