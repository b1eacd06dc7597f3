// Continuous-batching MSM server over a resident-SRS context.
//
// Jobs (host scalars, n <= SRS length) arrive through impeller_server_submit
// from any thread.  A dispatcher thread
//   - admits pending jobs in arrival order while a batch slot is free and
//     their device footprint fits the HBM budget (jobs that can never fit are
//     refused at submit);
//   - packs the admitted jobs into one batch plan (every phase one launch for
//     the whole batch; per-job window and resident table set);
//   - runs each batch on its own stream with stream-ordered device memory, so
//     batches that are on the GPU at the same time overlap there: a new batch's
//     histogram and accumulation run beside an older batch's reduction;
//   - harvests finished batches by event, returns their memory, records each
//     job's latency from submission to result.
// The reference serves whole proofs, not single MSMs: its scheduler admits a
// proof task when CPU memory and a card are free and polls every 10 ms
// (scheduler/src/scheduler/core.rs:419-580, scheduler/src/scheduler.rs:432-489);
// the admission-by-free-memory rule is the same idea applied per MSM, on HBM.
#include <algorithm>
#include <atomic>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <memory>
#include <mutex>
#include <string>
#include <thread>
#include <unordered_map>
#include <vector>

#include "../../include/impeller_msm.h"
#include "engine.h"

using namespace impeller;

namespace {

double now_s() {
    using namespace std::chrono;
    return duration_cast<duration<double>>(steady_clock::now().time_since_epoch()).count();
}

size_t up256(size_t x) { return (x + 255) / 256 * 256; }

// Device memory a server maps for batch scratch when it starts (at most its
// HBM budget).
constexpr u64 POOL_RESERVE = 16ull << 30;

struct Job {
    const u32 *h_scalars = nullptr;
    u64 n = 0;
    u32 c = 0;
    MsmShape shape{};
    size_t bytes = 0;  // device footprint when run alone (scalars + plan scratch)
    double t_submit = 0, t_done = 0;
    bool done = false;
    cudaError_t status = cudaSuccess;
    u32 result[24] = {};  // affine result, point_words(curve) used
};

struct Batch {
    std::unique_ptr<Plan> plan;
    std::vector<u64> ids;
    cudaStream_t stream = nullptr;
    cudaEvent_t ev = nullptr;
    void *mem = nullptr;  // scalars | results | plan scratch
    size_t bytes = 0;
    u32 *h_results = nullptr;  // pinned, point_words(curve) u32 per job
    cudaError_t status = cudaSuccess;
};

}  // namespace

struct impeller_server {
    impeller_ctx *ctx = nullptr;
    u32 max_batch = 64, max_inflight = 3;
    u64 budget = 0;
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<u64> pending;
    std::unordered_map<u64, Job> jobs;
    std::vector<std::unique_ptr<Batch>> inflight;
    std::vector<cudaStream_t> streams;
    cudaMemPool_t pool = nullptr;  // batch scratch; keeps freed memory mapped for the next batch
    std::vector<u32 *> pinned;  // one result buffer per slot
    std::vector<void *> staging;  // one table-image buffer per slot
    size_t staging_cap = 0;
    u64 used = 0, peak = 0;
    u64 next_id = 1;
    bool stop = false;
    u32 inject = 0;
    std::thread worker;
    // statistics
    u64 submitted = 0, completed = 0, rejected = 0, failed = 0, batches = 0, points = 0, jobs_batched = 0;
    u64 max_concurrent = 0;
    std::vector<double> latencies_ms;
    double t_first = 0, t_last = 0;
};

namespace {

cudaError_t launch_batch(impeller_server *s, Batch &b, std::vector<Job *> &js, u32 slot) {
    const u32 M = (u32)js.size();
    std::vector<MsmShape> shapes;
    u64 scal_words = 0;
    for (Job *j : js) {
        shapes.push_back(j->shape);
        scal_words += j->n * 8;
    }
    b.plan.reset(new Plan());
    if (!Plan::build(*b.plan, s->ctx->device, shapes)) return cudaErrorInvalidValue;
    b.plan->set_staging(s->staging[slot], s->staging_cap);
    const size_t o_res = up256(scal_words * 4);
    const size_t RB = (size_t)point_words(s->ctx->curve) * 4;  // result bytes per job
    const size_t o_plan = o_res + up256((size_t)M * RB);
    b.bytes = o_plan + b.plan->scratch_bytes();
    b.stream = s->streams[slot];
    b.h_results = s->pinned[slot];
    cudaError_t e = cudaMallocFromPoolAsync(&b.mem, b.bytes, s->pool, b.stream);
    if (e != cudaSuccess) return e;
    unsigned char *base = static_cast<unsigned char *>(b.mem);
    std::vector<const u32 *> sc(M);
    u64 off = 0;
    for (u32 m = 0; m < M; m++) {
        u32 *d = reinterpret_cast<u32 *>(base) + off;
        if ((e = cudaMemcpyAsync(d, js[m]->h_scalars, js[m]->n * 32, cudaMemcpyHostToDevice, b.stream)) !=
            cudaSuccess)
            return e;
        sc[m] = d;
        off += js[m]->n * 8;
    }
    u32 *d_res = reinterpret_cast<u32 *>(base + o_res);
    if ((e = b.plan->enqueue(base + o_plan, ctx_point_base(s->ctx), sc.data(), d_res, 0, b.stream)) != cudaSuccess)
        return e;
    if ((e = cudaMemcpyAsync(b.h_results, d_res, (size_t)M * RB, cudaMemcpyDeviceToHost, b.stream)) != cudaSuccess)
        return e;
    if ((e = cudaEventRecord(b.ev, b.stream)) != cudaSuccess) return e;
    return cudaSuccess;
}

void finish_batch(impeller_server *s, Batch &b, double t) {
    const u32 PW = point_words(s->ctx->curve);
    for (size_t k = 0; k < b.ids.size(); k++) {
        Job &j = s->jobs[b.ids[k]];
        j.status = b.status;
        if (b.status == cudaSuccess) std::memcpy(j.result, b.h_results + PW * k, PW * 4);
        j.done = true;
        j.t_done = t;
        if (b.status == cudaSuccess) {
            s->completed++;
            s->points += j.n;
            s->latencies_ms.push_back((j.t_done - j.t_submit) * 1e3);
        } else {
            s->failed++;
        }
        s->t_last = std::max(s->t_last, t);
    }
    if (b.mem) cudaFreeAsync(b.mem, b.stream);
    if (b.ev) cudaEventDestroy(b.ev);
    s->used -= b.bytes;
}

void dispatcher(impeller_server *s) {
    cudaSetDevice(s->ctx->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        // harvest finished batches
        bool progressed = false;
        for (size_t i = 0; i < s->inflight.size();) {
            Batch &b = *s->inflight[i];
            cudaError_t q = b.status != cudaSuccess ? cudaSuccess : cudaEventQuery(b.ev);
            if (q == cudaErrorNotReady) {
                i++;
                continue;
            }
            if (b.status == cudaSuccess && q != cudaSuccess) b.status = q;
            finish_batch(s, b, now_s());
            s->inflight.erase(s->inflight.begin() + i);
            progressed = true;
        }
        if (progressed) s->cv_done.notify_all();
        // admit and launch
        while (s->inflight.size() < s->max_inflight && !s->pending.empty()) {
            std::vector<Job *> js;
            std::vector<u64> ids;
            std::vector<MsmShape> shapes;
            u64 bytes = 0;
            while (!s->pending.empty() && js.size() < s->max_batch) {
                Job &j = s->jobs[s->pending.front()];
                if (s->used + bytes + j.bytes > s->budget) break;
                // keep the batch on the two-level sort: a batch past its
                // limits sorts entry by entry, slower than its jobs alone
                shapes.push_back(j.shape);
                if (!js.empty() && !Plan::two_level_sort(shapes)) {
                    shapes.pop_back();
                    break;
                }
                bytes += j.bytes;
                js.push_back(&j);
                ids.push_back(s->pending.front());
                s->pending.pop_front();
            }
            if (js.empty()) break;  // wait for memory to free
            // a free slot: streams[k] is busy iff some in-flight batch uses it
            u32 slot = 0;
            for (; slot < s->max_inflight; slot++) {
                bool busy = false;
                for (auto &p : s->inflight) busy |= p->stream == s->streams[slot];
                if (!busy) break;
            }
            std::unique_ptr<Batch> b(new Batch());
            b->ids = ids;
            bool fail = s->inject > 0;
            if (fail) s->inject--;
            // launch without the lock: submit() keeps accepting jobs meanwhile
            lk.unlock();
            cudaError_t e = cudaEventCreateWithFlags(&b->ev, cudaEventDisableTiming);
            if (e == cudaSuccess) e = fail ? cudaErrorLaunchFailure : launch_batch(s, *b, js, slot);
            if (e != cudaSuccess) {
                // host-side fault injection or a failed launch: no result
                b->status = e;
                if (b->mem) cudaStreamSynchronize(s->streams[slot]);
                b->bytes = 0;
            }
            lk.lock();
            s->used += b->bytes;
            s->peak = std::max(s->peak, s->used);
            s->batches++;
            s->jobs_batched += ids.size();
            s->inflight.push_back(std::move(b));
            s->max_concurrent = std::max<u64>(s->max_concurrent, s->inflight.size());
        }
        if (s->stop && s->pending.empty() && s->inflight.empty()) break;
        // sleep until new work arrives, or briefly while batches are on the GPU
        if (s->inflight.empty())
            s->cv_work.wait(lk, [s] { return s->stop || !s->pending.empty(); });
        else
            s->cv_work.wait_for(lk, std::chrono::microseconds(50));
    }
}

}  // namespace

// Test hook: the next server creation fails at this setup step (0: none).
static std::atomic<u32> g_fail_setup_step{0};

// Records which setup step failed and why; a step named by the test hook
// fails with cudaErrorMemoryAllocation before it runs.
static cudaError_t setup_step(const char *what, cudaError_t e) {
    if (e != cudaSuccess) set_error(std::string("impeller_server_create: ") + what + ": " + cudaGetErrorString(e));
    return e;
}

static cudaError_t injected(u32 step, const char *what) {
    u32 want = step;
    if (g_fail_setup_step.compare_exchange_strong(want, 0u))
        return setup_step(what, cudaErrorMemoryAllocation);
    return cudaSuccess;
}

// Streams, pinned buffers and the scratch pool of a new server.
static cudaError_t server_setup(impeller_server *s) {
    cudaError_t e = cudaSuccess;
    const impeller_ctx *ctx = s->ctx;
    const u32 max_batch = s->max_batch, max_inflight = s->max_inflight;
    const u64 hbm_budget = s->budget;
    {
        // a pool of its own that returns nothing to the driver between batches
        // (the default pool unmaps freed memory at every synchronisation,
        // and mapping it again costs each batch time on the host)
        cudaMemPoolProps props = {};
        props.allocType = cudaMemAllocationTypePinned;
        props.location.type = cudaMemLocationTypeDevice;
        props.location.id = ctx->device;
        if ((e = injected(1, "memory pool")) != cudaSuccess) return e;
        if ((e = setup_step("memory pool", cudaMemPoolCreate(&s->pool, &props))) != cudaSuccess) return e;
        uint64_t keep = hbm_budget;
        e = cudaMemPoolSetAttribute(s->pool, cudaMemPoolAttrReleaseThreshold, &keep);
        if (setup_step("memory pool release threshold", e) != cudaSuccess) {
            cudaMemPoolDestroy(s->pool);
            s->pool = nullptr;
            return e;
        }
    }
    for (u32 i = 0; i < max_inflight; i++) {
        cudaStream_t st;
        if ((e = injected(2, "stream")) != cudaSuccess) return e;
        if ((e = setup_step("stream", cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking))) != cudaSuccess)
            return e;
        s->streams.push_back(st);
        u32 *p = nullptr;
        if ((e = injected(3, "pinned result buffer")) != cudaSuccess) return e;
        e = cudaHostAlloc(&p, (size_t)max_batch * point_words(ctx->curve) * 4, cudaHostAllocPortable);
        if (setup_step("pinned result buffer", e) != cudaSuccess) return e;
        s->pinned.push_back(p);
        void *t = nullptr;
        s->staging_cap = (size_t)max_batch * 4096 + (1u << 20);  // descriptors, windows, reduce blocks
        if ((e = setup_step("pinned staging buffer", cudaHostAlloc(&t, s->staging_cap, cudaHostAllocPortable))) !=
            cudaSuccess)
            return e;
        s->staging.push_back(t);
    }
    {
        // Map the pool's memory now: growing it on demand under load took
        // single batch launches 1-2 s (the host blocks while new memory is
        // mapped), which turned bursts into backlogs.  The pool keeps what
        // is freed (release threshold = budget), so this stays mapped.
        void *warm = nullptr;
        const size_t reserve = (size_t)std::min<u64>(s->budget, POOL_RESERVE);
        if ((e = injected(4, "pool reserve")) != cudaSuccess) return e;
        e = cudaMallocFromPoolAsync(&warm, reserve, s->pool, s->streams[0]);
        if (setup_step("pool reserve", e) != cudaSuccess) return e;
        if ((e = setup_step("pool reserve release", cudaFreeAsync(warm, s->streams[0]))) != cudaSuccess) return e;
        if ((e = setup_step("pool reserve sync", cudaStreamSynchronize(s->streams[0]))) != cudaSuccess) return e;
    }
    return cudaSuccess;
}

// Frees what server_setup made (streams idle).
static void server_release(impeller_server *s) {
    for (auto st : s->streams) {
        cudaStreamSynchronize(st);
        cudaStreamDestroy(st);
    }
    s->streams.clear();
    for (auto p : s->pinned) cudaFreeHost(p);
    s->pinned.clear();
    for (auto p : s->staging) cudaFreeHost(p);
    s->staging.clear();
    if (s->pool) cudaMemPoolDestroy(s->pool);
    s->pool = nullptr;
}

extern "C" {

cudaError_t impeller_server_create(impeller_server **out, impeller_ctx *ctx, uint32_t max_batch,
                                   uint32_t max_inflight, uint64_t hbm_budget) {
    if (!out || !ctx || max_batch == 0 || max_inflight == 0 || max_inflight > 16) {
        set_error("impeller_server_create: bad argument");
        return cudaErrorInvalidValue;
    }
    std::unique_ptr<impeller_server> s(new impeller_server());
    s->ctx = ctx;
    s->max_batch = max_batch;
    s->max_inflight = max_inflight;
    cudaError_t e = setup_step("cudaSetDevice", cudaSetDevice(ctx->device));
    if (e != cudaSuccess) return e;
    if (hbm_budget == 0) {
        size_t fr = 0, tot = 0;
        if ((e = setup_step("cudaMemGetInfo", cudaMemGetInfo(&fr, &tot))) != cudaSuccess) return e;
        const size_t reserve = (size_t)1 << 30;
        hbm_budget = fr > reserve ? fr - reserve : fr / 2;
    }
    s->budget = hbm_budget;
    if ((e = server_setup(s.get())) != cudaSuccess) {
        server_release(s.get());
        return e;
    }
    impeller_server *raw = s.release();
    raw->worker = std::thread(dispatcher, raw);
    *out = raw;
    return cudaSuccess;
}

cudaError_t impeller_server_submit(impeller_server *s, const uint32_t *h_scalars, uint64_t n, uint64_t *job_id) {
    if (!s || !job_id) return cudaErrorInvalidValue;
    if (!h_scalars || n == 0 || n > s->ctx->len) {
        std::lock_guard<std::mutex> g(s->mu);
        s->rejected++;
        set_error("impeller_server_submit: need 0 < n <= SRS length and host scalars");
        return cudaErrorInvalidValue;
    }
    Job j;
    j.h_scalars = h_scalars;
    j.n = n;
    j.c = ctx_window(s->ctx, n);
    j.shape = ctx_shape(s->ctx, (u32)n, j.c);
    Plan p;
    if (!Plan::build(p, s->ctx->device, {j.shape})) return cudaErrorInvalidValue;
    j.bytes = up256(n * 32) + 256 + p.scratch_bytes();
    std::lock_guard<std::mutex> g(s->mu);
    if (j.bytes > s->budget) {
        s->rejected++;
        set_error("impeller_server_submit: job needs more device memory than the server's HBM budget");
        return cudaErrorMemoryAllocation;
    }
    j.t_submit = now_s();
    if (s->submitted == 0) s->t_first = j.t_submit;
    const u64 id = s->next_id++;
    s->jobs.emplace(id, j);
    s->pending.push_back(id);
    s->submitted++;
    *job_id = id;
    s->cv_work.notify_one();
    return cudaSuccess;
}

static cudaError_t take_result(impeller_server *s, std::unordered_map<u64, Job>::iterator it, uint32_t *h_result,
                               double *latency_ms) {
    Job &j = it->second;
    cudaError_t st = j.status;
    if (h_result && st == cudaSuccess) std::memcpy(h_result, j.result, point_words(s->ctx->curve) * 4);
    if (latency_ms) *latency_ms = (j.t_done - j.t_submit) * 1e3;
    s->jobs.erase(it);
    s->cv_done.notify_all();  // other waiters on this id find it gone
    if (st != cudaSuccess) set_error(std::string("MSM job failed: ") + cudaGetErrorString(st));
    return st;
}

cudaError_t impeller_server_wait(impeller_server *s, uint64_t job_id, uint32_t *h_result, double *latency_ms) {
    if (!s) return cudaErrorInvalidValue;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) {
        set_error("impeller_server_wait: unknown job");
        return cudaErrorInvalidValue;
    }
    // Wake when the job is done, or gone: another wait() or poll() on the
    // same id may take (and erase) it first.
    s->cv_done.wait(lk, [&] {
        auto j = s->jobs.find(job_id);
        return j == s->jobs.end() || j->second.done;
    });
    it = s->jobs.find(job_id);
    if (it == s->jobs.end()) {
        set_error("impeller_server_wait: job already taken by another wait or poll");
        return cudaErrorInvalidValue;
    }
    return take_result(s, it, h_result, latency_ms);
}

cudaError_t impeller_server_poll(impeller_server *s, uint64_t job_id, uint32_t *h_result, double *latency_ms) {
    if (!s) return cudaErrorInvalidValue;
    std::lock_guard<std::mutex> g(s->mu);
    auto it = s->jobs.find(job_id);
    if (it == s->jobs.end()) {
        set_error("impeller_server_poll: unknown job");
        return cudaErrorInvalidValue;
    }
    if (!it->second.done) return cudaErrorNotReady;
    return take_result(s, it, h_result, latency_ms);
}

cudaError_t impeller_server_get_stats(impeller_server *s, impeller_server_stats *out) {
    if (!s || !out) return cudaErrorInvalidValue;
    std::lock_guard<std::mutex> g(s->mu);
    std::memset(out, 0, sizeof *out);
    out->submitted = s->submitted;
    out->completed = s->completed;
    out->rejected = s->rejected;
    out->failed = s->failed;
    out->batches = s->batches;
    out->points = s->points;
    out->peak_bytes = s->peak;
    out->budget_bytes = s->budget;
    out->mean_batch = s->batches ? (double)s->jobs_batched / (double)s->batches : 0.0;
    out->span_s = s->t_last > s->t_first ? s->t_last - s->t_first : 0.0;
    out->max_concurrent = s->max_concurrent;
    std::vector<double> l = s->latencies_ms;
    if (!l.empty()) {
        std::sort(l.begin(), l.end());
        auto q = [&](double f) { return l[std::min(l.size() - 1, (size_t)(f * (double)(l.size() - 1) + 0.5))]; };
        out->p50_ms = q(0.50);
        out->p99_ms = q(0.99);
        out->max_ms = l.back();
        double sum = 0;
        for (double v : l) sum += v;
        out->mean_ms = sum / (double)l.size();
    }
    return cudaSuccess;
}

cudaError_t impeller_server_fail_setup_step(uint32_t step) {
    if (step > 4) {
        set_error("impeller_server_fail_setup_step: steps are 1..4 (0 clears)");
        return cudaErrorInvalidValue;
    }
    g_fail_setup_step.store(step);
    return cudaSuccess;
}

cudaError_t impeller_server_inject_failures(impeller_server *s, uint32_t batches) {
    if (!s) return cudaErrorInvalidValue;
    std::lock_guard<std::mutex> g(s->mu);
    s->inject = batches;
    return cudaSuccess;
}

cudaError_t impeller_server_destroy(impeller_server *s) {
    if (!s) return cudaSuccess;
    {
        std::lock_guard<std::mutex> g(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(s->ctx->device);
    server_release(s);
    delete s;
    return cudaSuccess;
}

}  // extern "C"
