// rt_server.cu -- continuous-batching request server (include/relsim_cuda.h, rt_server_*).
//
// Render requests (one camera each) are admitted in arrival order while their
// output records fit a device-memory budget, and are traced in "epochs": one
// persistent tracer launch over a bundle table of row chunks taken round-robin
// from every admitted request with rows left, so a request that arrives while
// others are on the GPU joins the next epoch instead of waiting for them to
// finish.  An epoch traces one kind of request (Kerr-Schild FP64 or mixed,
// multi-source, Boyer-Lindquist) and is sized by the rays' cost, so that a
// launch of slow rays does not hold back requests of other kinds for long.
// Two epoch slots on separate streams keep the GPU busy while the
// scheduler retires one epoch and builds the next (the tail of one launch
// overlaps the start of the other).  Output records stay on the device, in a
// budget-sized arena, until a request's last chunk is done; then they are copied
// to the caller's host buffers on a copy stream and the arena range is freed.
//
// Reference counterpart: the render worker of GeodesicComputePipeline
// (geodesic_compute_pipeline.hpp:505-529) serialises whole frames on one
// executor; there is no request admission or batching in the reference.
#include <cuda_runtime.h>

#include <algorithm>
#include <chrono>
#include <cmath>
#include <condition_variable>
#include <cstdio>
#include <cstring>
#include <deque>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <vector>

#include "relsim_cuda.h"
#include "rt_internal.h"

using namespace relsim;

namespace {

using Clock = std::chrono::steady_clock;

constexpr int kFields = 14;                                          // rt_ray_out fields
constexpr size_t kFieldBytes[kFields] = {4, 4, 4, 4, 8, 8, 8, 8, 8, 8, 8, 8, 8, 8};
constexpr uint32_t kPixelBit = 1u << 14;                             // record_mask bit of the pixels
constexpr uint32_t kShadeSlots = 64;                                  // ring of per-request shading constants
// record_mask bits the shading pass needs: status, phi, r_hit, g and the pixels
constexpr uint32_t kShadeMask = (1u << 0) | (1u << 6) | (1u << 7) | (1u << 8) | kPixelBit;
constexpr int kSlots = 2;                                            // epochs in flight

// First-fit allocator over ray slots [0, capacity) of the output arena.
class RangeAllocator {
public:
    explicit RangeAllocator(uint64_t capacity = 0) { reset(capacity); }
    void reset(uint64_t capacity) {
        free_.clear();
        if (capacity) free_[0] = capacity;
        used_ = 0;
    }
    bool alloc(uint64_t n, uint64_t& base) {
        for (auto it = free_.begin(); it != free_.end(); ++it) {
            if (it->second < n) continue;
            base = it->first;
            const uint64_t rest = it->second - n;
            free_.erase(it);
            if (rest) free_[base + n] = rest;
            used_ += n;
            return true;
        }
        return false;
    }
    void release(uint64_t base, uint64_t n) {
        used_ -= n;
        auto it = free_.emplace(base, n).first;
        auto next = std::next(it);
        if (next != free_.end() && it->first + it->second == next->first) {
            it->second += next->second;
            free_.erase(next);
        }
        if (it != free_.begin()) {
            auto prev = std::prev(it);
            if (prev->first + prev->second == it->first) {
                prev->second += it->second;
                free_.erase(it);
            }
        }
    }
    uint64_t used() const { return used_; }

private:
    std::map<uint64_t, uint64_t> free_;  // base -> length
    uint64_t used_ = 0;
};

enum class ReqState { Waiting, Active, Copying, Done };

struct Request {
    uint64_t id = 0;
    rt_camera cam{};
    uint32_t row0 = 0, nrows = 0, width = 0;
    uint64_t rays = 0;
    rt_pixel_out* host_pixels = nullptr;
    rt_ray_out host_rays{};
    ReqState state = ReqState::Waiting;
    uint64_t base = 0;            // arena ray slot of the request's first ray
    uint32_t rows_issued = 0;     // rows put into an epoch
    uint64_t rays_done = 0;       // rays of finished epochs
    cudaEvent_t copy_done = nullptr;
    Clock::time_point t_submit, t_admit, t_first_launch, t_done;
    bool launched = false;
    bool admitted = false;        // holds an arena range
    rt_status status = RT_OK;
    uint32_t n_sources = 0;       // multi-source scene: its source table (0: single hole)
    MsSource sources[kMaxSources];
    // epochs trace one kind of request: Kerr-Schild FP64 (0) or mixed precision (1),
    // multi-source (2), Boyer-Lindquist Kerr-Newman (3)
    int kind() const {
        if (n_sources) return 2;
        if (cam.metric_form == RT_METRIC_BOYER_LINDQUIST) return 3;
        return static_cast<int>(cam.precision_mode);
    }
    // GPU time of one ray in units of a mixed-precision Kerr-Schild ray (measured
    // on B200: mixed 160 Mrays/s, FP64 105, Boyer-Lindquist 47; multi-source
    // about 90 / holes at rtol 1e-8, the mixed mode's tolerance, and 40 / holes
    // at 1e-10); epochs are budgeted in these units so that an epoch of slow
    // rays does not hold the GPU much longer than one of fast rays
    uint64_t cost() const {
        switch (kind()) {
            case 2: return (cam.rtol >= 1e-9 ? 2ull : 4ull) * n_sources;
            case 3: return 4;
            case RT_PRECISION_MIXED: return 1;
            default: return 2;
        }
    }
};

struct Chunk {
    Request* req;
    uint64_t rays;
};

struct Slot {
    cudaStream_t stream = nullptr;
    cudaEvent_t done = nullptr;
    BundleDesc* host_table = nullptr;   // pinned staging of the bundle table
    BundleDesc* dev_table = nullptr;
    unsigned long long* counters = nullptr;  // [0] queue, [8..] stats
    void* pass_state = nullptr;              // two-pass mixed tracer: parked state and queues
    char* pass_counters = nullptr;           // its queue counters
    MsDesc* host_ms = nullptr;               // multi-source epochs: camera table (pinned) and sources
    MsDesc* dev_ms = nullptr;
    MsSource* host_src = nullptr;
    MsSource* dev_src = nullptr;
    BlDesc* host_bl = nullptr;               // Boyer-Lindquist epochs: camera table (pinned)
    BlDesc* dev_bl = nullptr;
    std::vector<Chunk> chunks;
    bool busy = false;
};

}  // namespace

struct rt_server {
    int device = 0;
    int sm_count = 0;
    rt_server_config cfg{};
    uint32_t bytes_per_ray = 0;
    uint64_t arena_rays = 0;
    void* arena = nullptr;
    void* field_base[kFields] = {};
    rt_pixel_out* pixel_base = nullptr;
    RangeAllocator alloc;
    Slot slots[kSlots];
    cudaStream_t copy_stream = nullptr;

    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::deque<Request*> waiting;
    std::vector<Request*> active;           // admitted, not yet done
    std::deque<rt_request_done> completed;  // not yet polled
    uint64_t next_id = 1;
    bool stop = false;
    bool failed = false;
    std::string error;
    rt_server_stats stats{};
    std::thread worker;
    size_t rr = 0;       // round-robin start in `active`
    int last_kind = -1;  // kind of the last epoch launched
    // pixel shading of finished single-hole requests (rt_server_set_shading)
    bool shade_on = false;
    rt_shading shading{};
    ShadeDesc* dev_shade = nullptr;  // ring of per-request shading constants, used in copy-stream order
    uint32_t shade_next = 0;
};

namespace {

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

void fail_server(rt_server* s, const char* where, cudaError_t e) {
    s->failed = true;
    s->error = std::string(where) + ": " + cudaGetErrorString(e);
}

// Finish a request (lock held): record, free its arena range, publish.
void complete(rt_server* s, Request* r, rt_status st) {
    r->t_done = Clock::now();
    r->state = ReqState::Done;
    r->status = st;
    if (r->copy_done) cudaEventDestroy(r->copy_done);
    r->copy_done = nullptr;
    if (r->admitted) s->alloc.release(r->base, r->rays);
    rt_request_done d{};
    d.id = r->id;
    d.status = st;
    d.rays = r->rays;
    d.queue_ms = ms_between(r->t_submit, r->launched ? r->t_first_launch : r->t_done);
    d.latency_ms = ms_between(r->t_submit, r->t_done);
    s->completed.push_back(d);
    ++s->stats.requests_done;
    s->stats.rays_done += r->rays;
    s->active.erase(std::remove(s->active.begin(), s->active.end(), r), s->active.end());
    delete r;
    s->cv_done.notify_all();
}

// Admit waiting requests in arrival order while the arena has room (lock held).
void admit(rt_server* s) {
    while (!s->waiting.empty()) {
        Request* r = s->waiting.front();
        uint64_t base = 0;
        if (!s->alloc.alloc(r->rays, base)) break;  // FIFO: later requests wait behind it
        s->waiting.pop_front();
        r->base = base;
        r->admitted = true;
        r->state = ReqState::Active;
        r->t_admit = Clock::now();
        s->active.push_back(r);
        const uint64_t used = s->alloc.used() * s->bytes_per_ray;
        s->stats.peak_bytes_in_use = std::max<uint64_t>(s->stats.peak_bytes_in_use, used);
        s->stats.peak_active = std::max<uint32_t>(s->stats.peak_active, static_cast<uint32_t>(s->active.size()));
    }
}

// Copy a finished request's records to the caller's host buffers (lock held);
// with shading on, a single-hole request's pixels are shaded first, on the
// copy stream.
bool start_copy(rt_server* s, Request* r) {
    cudaStream_t cs = s->copy_stream;
    if (s->shade_on && r->n_sources == 0 && r->host_pixels) {
        ShadeDesc d;
        if (build_shade_desc(r->cam, s->shading, d)) {
            ShadeDesc* slot = s->dev_shade + (s->shade_next++ % kShadeSlots);
            // pageable descriptor: the copy is staged before the call returns; the ring slot
            // is next written kShadeSlots requests later, after this kernel in stream order
            cudaError_t e = cudaMemcpyAsync(slot, &d, sizeof d, cudaMemcpyHostToDevice, cs);
            if (e != cudaSuccess) return fail_server(s, "cudaMemcpyAsync", e), false;
            const uint64_t b = r->base;
            launch_shade(slot, static_cast<const uint32_t*>(s->field_base[0]) + b,
                         static_cast<const double*>(s->field_base[7]) + b, static_cast<const double*>(s->field_base[6]) + b,
                         static_cast<const double*>(s->field_base[8]) + b, ContOut{}, s->pixel_base + b, r->rays, cs);
            e = cudaGetLastError();
            if (e != cudaSuccess) return fail_server(s, "shade launch", e), false;
        }
    }
    void* const* hp = reinterpret_cast<void* const*>(&r->host_rays);
    for (int f = 0; f < kFields; ++f) {
        if (!hp[f]) continue;
        const char* src = static_cast<const char*>(s->field_base[f]) + r->base * kFieldBytes[f];
        cudaError_t e = cudaMemcpyAsync(hp[f], src, r->rays * kFieldBytes[f], cudaMemcpyDeviceToHost, cs);
        if (e != cudaSuccess) return fail_server(s, "cudaMemcpyAsync", e), false;
    }
    if (r->host_pixels) {
        cudaError_t e = cudaMemcpyAsync(r->host_pixels, s->pixel_base + r->base, r->rays * sizeof(rt_pixel_out),
                                        cudaMemcpyDeviceToHost, cs);
        if (e != cudaSuccess) return fail_server(s, "cudaMemcpyAsync", e), false;
    }
    cudaError_t e = cudaEventCreateWithFlags(&r->copy_done, cudaEventDisableTiming);
    if (e == cudaSuccess) e = cudaEventRecord(r->copy_done, cs);
    if (e != cudaSuccess) return fail_server(s, "cudaEventRecord", e), false;
    r->state = ReqState::Copying;
    return true;
}

// Build and launch one epoch into a free slot (lock held).  Returns false when
// there is nothing to trace.
bool launch_epoch(rt_server* s, Slot& slot) {
    // kind of this epoch: that of the oldest active request with rows left,
    // alternating with the other kinds when they have rows waiting too, so
    // that a stream of one kind does not hold back requests of another
    int kind = -1, other = -1;
    for (Request* r : s->active) {
        if (r->state != ReqState::Active || r->rows_issued >= r->nrows) continue;
        if (kind < 0) kind = r->kind();
        if (other < 0 && r->kind() != s->last_kind) other = r->kind();
    }
    if (kind < 0) return false;
    if (other >= 0) kind = other;
    s->last_kind = kind;
    const bool mixed = kind == RT_PRECISION_MIXED;
    const bool multi = kind == 2;
    const bool bl = kind == 3;
    uint32_t n_src = 0;               // sources copied into this epoch's table
    std::vector<std::pair<Request*, uint32_t>> src_at;  // request -> its first source in the table
    slot.chunks.clear();
    // An epoch holds at most epoch_rays rays (the slot's buffers) and takes rows
    // while its cost stays within epoch_rays units or it holds fewer than
    // min_epoch_rays rays; round robin over active requests, each taking about
    // chunk_rays units (at least one row) per turn.
    uint64_t total = 0;  // rays of the epoch
    uint64_t units = 0;  // their cost in mixed-ray units
    uint32_t nb = 0;
    const uint64_t epoch = s->cfg.epoch_rays;
    const uint64_t min_rays = std::min<uint64_t>(s->cfg.min_epoch_rays, epoch);
    const size_t n_active = s->active.size();
    auto open = [&] { return total < epoch && (units < epoch || total < min_rays) && nb < s->cfg.max_epoch_bundles; };
    bool progress = true;
    while (progress && open()) {
        progress = false;
        for (size_t k = 0; k < n_active && open(); ++k) {
            Request* r = s->active[(s->rr + k) % n_active];
            if (r->state != ReqState::Active || r->rows_issued >= r->nrows) continue;
            if (r->kind() != kind) continue;
            const uint64_t w = r->cost();
            const uint64_t by_units = (units < epoch) ? (epoch - units) / w : 0;
            const uint64_t by_floor = (total < min_rays) ? min_rays - total : 0;
            const uint64_t room = std::min<uint64_t>(std::max(by_units, by_floor), epoch - total);
            uint64_t fit = std::min<uint64_t>(std::max<uint64_t>(1, s->cfg.chunk_rays / w / r->width), room / r->width);
            // a row that does not fit: only as the epoch's first chunk (submit
            // guarantees width <= epoch_rays, so its rays fit the buffers)
            if (fit == 0 && nb == 0) fit = 1;
            if (fit == 0) continue;
            const uint32_t rows = static_cast<uint32_t>(std::min<uint64_t>(fit, r->nrows - r->rows_issued));
            const uint64_t n = static_cast<uint64_t>(rows) * r->width;
            if (multi) {
                uint32_t begin = UINT32_MAX;
                for (const auto& q : src_at)
                    if (q.first == r) begin = q.second;
                if (begin == UINT32_MAX) {
                    begin = n_src;
                    for (uint32_t j = 0; j < r->n_sources; ++j) slot.host_src[n_src++] = r->sources[j];
                    src_at.emplace_back(r, begin);
                }
                build_ms_bundle(r->cam, 0, r->width, r->row0 + r->rows_issued, rows, total,
                                r->base + static_cast<uint64_t>(r->rows_issued) * r->width, begin, r->n_sources,
                                slot.host_ms[nb]);
            } else if (bl) {
                build_bl_bundle(r->cam, 0, r->width, r->row0 + r->rows_issued, rows, total,
                                r->base + static_cast<uint64_t>(r->rows_issued) * r->width, slot.host_bl[nb]);
            } else {
                build_bundle(r->cam, 0, r->width, r->row0 + r->rows_issued, rows, total,
                             r->base + static_cast<uint64_t>(r->rows_issued) * r->width, slot.host_table[nb]);
            }
            if (!r->launched) {
                r->launched = true;
                r->t_first_launch = Clock::now();
            }
            r->rows_issued += rows;
            slot.chunks.push_back({r, n});
            total += n;
            units += n * w;
            ++nb;
            progress = true;
        }
    }
    s->rr = n_active ? (s->rr + 1) % n_active : 0;
    if (nb == 0) return false;
    cudaStream_t st = slot.stream;
    // the staging tables were last read by this slot's previous epoch, which is retired
    cudaError_t e;
    if (multi) {
        e = cudaMemcpyAsync(slot.dev_ms, slot.host_ms, sizeof(MsDesc) * nb, cudaMemcpyHostToDevice, st);
        if (e == cudaSuccess)
            e = cudaMemcpyAsync(slot.dev_src, slot.host_src, sizeof(MsSource) * n_src, cudaMemcpyHostToDevice, st);
    } else if (bl) {
        e = cudaMemcpyAsync(slot.dev_bl, slot.host_bl, sizeof(BlDesc) * nb, cudaMemcpyHostToDevice, st);
    } else {
        e = cudaMemcpyAsync(slot.dev_table, slot.host_table, sizeof(BundleDesc) * nb, cudaMemcpyHostToDevice, st);
    }
    if (e == cudaSuccess) e = cudaMemsetAsync(slot.counters, 0, 256, st);
    if (e != cudaSuccess) return fail_server(s, "epoch upload", e), false;
    const rt_launch_config c = resolve_launch_config(mixed ? s->cfg.launch_mixed : s->cfg.launch_fp64, mixed);
    TraceArgs args{};
    args.bundles = slot.dev_table;
    args.n_bundles = nb;
    args.refill_threshold = c.refill_threshold;
    args.claim = 32u * c.rays_per_thread;
    args.total_rays = total;
    args.queue = slot.counters;
    args.stats = slot.counters + 8;
    rt_ray_out rays{};
    void** dp = reinterpret_cast<void**>(&rays);
    for (int f = 0; f < kFields; ++f)
        if (s->cfg.record_mask & (1u << f)) dp[f] = s->field_base[f];
    args.out = OutPtrs{(s->cfg.record_mask & kPixelBit) ? s->pixel_base : nullptr, rays};
    if (multi) {
        MsArgs ma{};
        ma.bundles = slot.dev_ms;
        ma.sources = slot.dev_src;
        ma.n_bundles = nb;
        ma.refill_threshold = 32;
        ma.claim = 32;
        ma.total_rays = total;
        ma.queue = slot.counters;
        ma.stats = slot.counters + 8;
        ma.out = args.out;
        const int ms_sms = (s->cfg.multi_source_sms > 0 && s->cfg.multi_source_sms < static_cast<uint32_t>(s->sm_count))
                               ? static_cast<int>(s->cfg.multi_source_sms)
                               : s->sm_count;
        launch_ms_trace(ma, ms_trace_grid(ms_sms), st);
        e = cudaGetLastError();
    } else if (bl) {
        BlArgs ba{};
        ba.bundles = slot.dev_bl;
        ba.n_bundles = nb;
        ba.refill_threshold = c.refill_threshold;
        ba.claim = 32u * c.rays_per_thread;
        ba.total_rays = total;
        ba.queue = slot.counters;
        ba.stats = slot.counters + 8;
        ba.out = args.out;
        launch_bl_trace(ba, bl_trace_grid(s->sm_count), st);
        e = cudaGetLastError();
    } else if (mixed && c.mixed_single_kernel == 0) {
        // parked state of the epoch's rays: SoA with `total` slots in the slot's buffer
        TwoPassBuffers buf{};
        double* pd = static_cast<double*>(slot.pass_state);
        uint32_t* pu = reinterpret_cast<uint32_t*>(pd + PD_COUNT * total);
        buf.park = ParkBuf{pd, pu, total};
        buf.queues = pu + PU_COUNT * total;
        buf.counters = slot.pass_counters;
        // one band per epoch: the two epoch slots already overlap each other's tails
        e = static_cast<cudaError_t>(
            enqueue_two_pass(args, buf, s->sm_count, c.block_size, st, nullptr, nullptr, nullptr, 1));
    } else {
        launch_trace(args, static_cast<uint32_t>(s->sm_count) * c.ctas_per_sm, c.block_size, mixed,
                     c.fp64_rolled != 0, st);
        e = cudaGetLastError();
    }
    if (e == cudaSuccess) e = cudaEventRecord(slot.done, st);
    if (e != cudaSuccess) return fail_server(s, "epoch launch", e), false;
    slot.busy = true;
    ++s->stats.epochs;
    s->stats.bundles += nb;
    s->stats.peak_epoch_rays = std::max<uint64_t>(s->stats.peak_epoch_rays, total);
    return true;
}

void worker_main(rt_server* s) {
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    while (!s->stop) {
        bool did = false;
        if (!s->failed) {
            admit(s);
            // retire finished epochs
            for (Slot& slot : s->slots) {
                if (!slot.busy) continue;
                const cudaError_t q = cudaEventQuery(slot.done);
                if (q == cudaErrorNotReady) continue;
                if (q != cudaSuccess) {
                    fail_server(s, "epoch", q);
                    break;
                }
                slot.busy = false;
                did = true;
                for (const Chunk& c : slot.chunks) {
                    c.req->rays_done += c.rays;
                    if (c.req->rays_done == c.req->rays && c.req->state == ReqState::Active) start_copy(s, c.req);
                }
                slot.chunks.clear();
            }
            // retire finished copies
            for (size_t i = 0; i < s->active.size();) {
                Request* r = s->active[i];
                if (r->state == ReqState::Copying) {
                    const cudaError_t q = cudaEventQuery(r->copy_done);
                    if (q == cudaSuccess) {
                        complete(s, r, RT_OK);
                        did = true;
                        continue;
                    }
                    if (q != cudaErrorNotReady) {
                        fail_server(s, "copy", q);
                        break;
                    }
                }
                ++i;
            }
            admit(s);
            for (Slot& slot : s->slots)
                if (!slot.busy && !s->failed && launch_epoch(s, slot)) did = true;
        }
        if (s->failed) {
            // end every request with the device error; the server stays failed
            while (!s->waiting.empty()) {
                Request* r = s->waiting.front();
                s->waiting.pop_front();
                s->active.push_back(r);
                r->state = ReqState::Active;
            }
            while (!s->active.empty()) complete(s, s->active.front(), RT_ERR_DEVICE);
            s->cv_work.wait_for(lk, std::chrono::milliseconds(50));
            continue;
        }
        if (!did) {
            bool busy = false;
            for (const Slot& slot : s->slots) busy = busy || slot.busy;
            for (Request* r : s->active) busy = busy || r->state == ReqState::Copying;
            // short waits while the GPU works; sleep until a submission when idle
            if (busy) s->cv_work.wait_for(lk, std::chrono::microseconds(100));
            else s->cv_work.wait_for(lk, std::chrono::milliseconds(20));
        }
    }
}

bool record_fields_ok(const rt_server* s, const rt_ray_out* rays, const rt_pixel_out* pixels) {
    if (pixels && !(s->cfg.record_mask & kPixelBit)) return false;
    if (!rays) return true;
    void* const* hp = reinterpret_cast<void* const*>(rays);
    for (int f = 0; f < kFields; ++f)
        if (hp[f] && !(s->cfg.record_mask & (1u << f))) return false;
    for (int f = kFields; f < kRayFields; ++f)  // exit directions: not recorded by the server
        if (hp[f]) return false;
    return true;
}

}  // namespace

extern "C" {

void rt_server_config_defaults(rt_server_config* c) {
    if (!c) return;
    std::memset(c, 0, sizeof *c);
    c->memory_budget_bytes = uint64_t{1} << 30;
    c->max_requests = 4096;
    c->chunk_rays = 1u << 18;
    c->epoch_rays = 1u << 22;
    c->min_epoch_rays = 1u << 18;
    c->max_epoch_bundles = 4096;
    // class, final position, disk radius and g, plus the 32-byte pixels
    c->record_mask = (1u << 0) | (1u << 4) | (1u << 5) | (1u << 6) | (1u << 7) | (1u << 8) | kPixelBit;
}

rt_status rt_server_create(rt_server** out, int device_ordinal, const rt_server_config* cfg) {
    if (!out || !cfg) return RT_ERR_INVALID_ARG;
    *out = nullptr;
    if (cfg->chunk_rays == 0 || cfg->epoch_rays == 0 || cfg->max_epoch_bundles == 0 || cfg->max_requests == 0 ||
        (cfg->record_mask & ~((kPixelBit << 1) - 1u)) != 0)
        return RT_ERR_INVALID_ARG;
    int n = 0;
    if (cudaGetDeviceCount(&n) != cudaSuccess || device_ordinal < 0 || device_ordinal >= n) {
        cudaGetLastError();
        return RT_ERR_DEVICE;
    }
    cudaDeviceProp p{};
    if (cudaGetDeviceProperties(&p, device_ordinal) != cudaSuccess || p.major != 10 || p.minor != 0)
        return RT_ERR_DEVICE;
    if (cudaSetDevice(device_ordinal) != cudaSuccess) return RT_ERR_DEVICE;
    rt_server* s = new (std::nothrow) rt_server();
    if (!s) return RT_ERR_OOM;
    s->device = device_ordinal;
    s->sm_count = p.multiProcessorCount;
    s->cfg = *cfg;
    uint32_t bpr = (cfg->record_mask & kPixelBit) ? sizeof(rt_pixel_out) : 0;
    for (int f = 0; f < kFields; ++f)
        if (cfg->record_mask & (1u << f)) bpr += static_cast<uint32_t>(kFieldBytes[f]);
    s->bytes_per_ray = std::max<uint32_t>(bpr, 1);
    // arena: one allocation, one SoA array per recorded field, each 256-byte aligned
    s->arena_rays = cfg->memory_budget_bytes / s->bytes_per_ray;
    if (s->arena_rays < 32) {
        delete s;
        return RT_ERR_BUDGET;
    }
    s->arena_rays &= ~uint64_t{31};
    size_t bytes = 0;
    size_t offs[kFields + 1] = {};
    for (int f = 0; f <= kFields; ++f) {
        const bool on = (f < kFields) ? (cfg->record_mask & (1u << f)) != 0 : (cfg->record_mask & kPixelBit) != 0;
        offs[f] = bytes;
        if (on) bytes += ((s->arena_rays * ((f < kFields) ? kFieldBytes[f] : sizeof(rt_pixel_out)) + 255) / 256) * 256;
    }
    cudaError_t e = cudaMalloc(&s->arena, std::max<size_t>(bytes, 256));
    if (e != cudaSuccess) {
        cudaGetLastError();
        delete s;
        return RT_ERR_OOM;
    }
    for (int f = 0; f < kFields; ++f)
        if (cfg->record_mask & (1u << f)) s->field_base[f] = static_cast<char*>(s->arena) + offs[f];
    if (cfg->record_mask & kPixelBit) s->pixel_base = reinterpret_cast<rt_pixel_out*>(static_cast<char*>(s->arena) + offs[kFields]);
    s->alloc.reset(s->arena_rays);
    bool ok = cudaStreamCreateWithFlags(&s->copy_stream, cudaStreamNonBlocking) == cudaSuccess;
    for (Slot& slot : s->slots) {
        ok = ok && cudaStreamCreateWithFlags(&slot.stream, cudaStreamNonBlocking) == cudaSuccess;
        ok = ok && cudaEventCreateWithFlags(&slot.done, cudaEventDisableTiming) == cudaSuccess;
        ok = ok && cudaMallocHost(&slot.host_table, sizeof(BundleDesc) * cfg->max_epoch_bundles) == cudaSuccess;
        ok = ok && cudaMalloc(&slot.dev_table, sizeof(BundleDesc) * cfg->max_epoch_bundles) == cudaSuccess;
        ok = ok && cudaMalloc(&slot.counters, 256) == cudaSuccess;
        ok = ok && cudaMalloc(&slot.pass_state, two_pass_state_bytes(cfg->epoch_rays)) == cudaSuccess;
        ok = ok && cudaMalloc(&slot.pass_counters, kBandCounterBytes * kMaxBands) == cudaSuccess;
        ok = ok && cudaMallocHost(&slot.host_ms, sizeof(MsDesc) * cfg->max_epoch_bundles) == cudaSuccess;
        ok = ok && cudaMalloc(&slot.dev_ms, sizeof(MsDesc) * cfg->max_epoch_bundles) == cudaSuccess;
        ok = ok && cudaMallocHost(&slot.host_src, sizeof(MsSource) * kMaxSources * cfg->max_epoch_bundles) ==
                       cudaSuccess;
        ok = ok && cudaMalloc(&slot.dev_src, sizeof(MsSource) * kMaxSources * cfg->max_epoch_bundles) == cudaSuccess;
        ok = ok && cudaMallocHost(&slot.host_bl, sizeof(BlDesc) * cfg->max_epoch_bundles) == cudaSuccess;
        ok = ok && cudaMalloc(&slot.dev_bl, sizeof(BlDesc) * cfg->max_epoch_bundles) == cudaSuccess;
    }
    if (!ok) {
        cudaGetLastError();
        rt_server_destroy(s);
        return RT_ERR_DEVICE;
    }
    s->worker = std::thread(worker_main, s);
    *out = s;
    return RT_OK;
}

void rt_server_destroy(rt_server* s) {
    if (!s) return;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->cv_work.notify_all();
    if (s->worker.joinable()) s->worker.join();
    cudaSetDevice(s->device);
    for (Slot& slot : s->slots) {
        if (slot.stream) cudaStreamSynchronize(slot.stream);
        if (slot.done) cudaEventDestroy(slot.done);
        if (slot.host_table) cudaFreeHost(slot.host_table);
        if (slot.dev_table) cudaFree(slot.dev_table);
        if (slot.counters) cudaFree(slot.counters);
        if (slot.pass_state) cudaFree(slot.pass_state);
        if (slot.pass_counters) cudaFree(slot.pass_counters);
        if (slot.host_ms) cudaFreeHost(slot.host_ms);
        if (slot.dev_ms) cudaFree(slot.dev_ms);
        if (slot.host_src) cudaFreeHost(slot.host_src);
        if (slot.dev_src) cudaFree(slot.dev_src);
        if (slot.host_bl) cudaFreeHost(slot.host_bl);
        if (slot.dev_bl) cudaFree(slot.dev_bl);
        if (slot.stream) cudaStreamDestroy(slot.stream);
    }
    if (s->copy_stream) {
        cudaStreamSynchronize(s->copy_stream);
        cudaStreamDestroy(s->copy_stream);
    }
    for (Request* r : s->waiting) delete r;
    for (Request* r : s->active) {
        if (r->copy_done) cudaEventDestroy(r->copy_done);
        delete r;
    }
    if (s->arena) cudaFree(s->arena);
    if (s->dev_shade) cudaFree(s->dev_shade);
    delete s;
}

}  // extern "C"

namespace {
rt_status submit_request(rt_server* s, const rt_camera* cam, const rt_source* src, uint32_t n_src, bool multi,
                         rt_pixel_out* pixels, const rt_ray_out* rays, size_t capacity, uint64_t* id) {
    if (!s || !cam || !id) return RT_ERR_INVALID_ARG;
    *id = 0;
    if (cam->screen_width == 0 || cam->screen_height == 0 || cam->rtol <= 0.0 ||
        (cam->precision_mode != RT_PRECISION_FP64 && cam->precision_mode != RT_PRECISION_MIXED))
        return RT_ERR_INVALID_ARG;
    if (cam->metric_form == RT_METRIC_BOYER_LINDQUIST) {
        // a horizon (a^2 + Q^2 < M^2 after the spin clamp); the multi-source tracer is Kerr-Schild only
        const double m = std::max(cam->metric_mass, 1e-4);
        const double a = std::min(std::max(cam->metric_spin, -0.999 * m), 0.999 * m);
        if (multi || !std::isfinite(cam->metric_charge) || !(m * m - a * a - cam->metric_charge * cam->metric_charge > 0.0))
            return RT_ERR_INVALID_ARG;
    } else if (cam->metric_form != RT_METRIC_KERR_SCHILD) {
        return RT_ERR_INVALID_ARG;
    }
    if (multi) {
        if (n_src > RT_MAX_SOURCES - 1 || (n_src > 0 && !src)) return RT_ERR_INVALID_ARG;
        for (uint32_t i = 0; i < n_src; ++i)
            if (!(src[i].mass > 0.0) || !std::isfinite(src[i].mass) || !std::isfinite(src[i].position[0]) ||
                !std::isfinite(src[i].position[1]) || !std::isfinite(src[i].position[2]))
                return RT_ERR_INVALID_ARG;
    }
    if (!record_fields_ok(s, rays, pixels)) return RT_ERR_INVALID_ARG;
    uint32_t row0, nrows;
    row_window(*cam, row0, nrows);
    const uint64_t n = static_cast<uint64_t>(cam->screen_width) * nrows;
    if (n == 0 || capacity < n) return RT_ERR_INVALID_ARG;
    if (n > s->arena_rays) return RT_ERR_BUDGET;  // could never be admitted
    if (cam->screen_width > s->cfg.epoch_rays) return RT_ERR_INVALID_ARG;  // a row must fit one epoch
    Request* r = new (std::nothrow) Request();
    if (!r) return RT_ERR_OOM;
    r->cam = *cam;
    if (multi) {
        r->cam.precision_mode = RT_PRECISION_FP64;  // the multi-source tracer is FP64
        r->n_sources = build_ms_sources(*cam, src, n_src, r->sources);
    }
    r->row0 = row0;
    r->nrows = nrows;
    r->width = cam->screen_width;
    r->rays = n;
    r->host_pixels = pixels;
    if (rays) r->host_rays = *rays;
    r->t_submit = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (s->failed) {
            delete r;
            return RT_ERR_DEVICE;
        }
        if (s->waiting.size() + s->active.size() >= s->cfg.max_requests) {
            delete r;
            return RT_ERR_AGAIN;
        }
        r->id = s->next_id++;
        *id = r->id;
        s->waiting.push_back(r);
        ++s->stats.requests_submitted;
    }
    s->cv_work.notify_all();
    return RT_OK;
}
}  // namespace

extern "C" {

rt_status rt_server_submit(rt_server* s, const rt_camera* cam, rt_pixel_out* pixels, const rt_ray_out* rays,
                           size_t capacity, uint64_t* id) {
    return submit_request(s, cam, nullptr, 0, false, pixels, rays, capacity, id);
}

rt_status rt_server_submit_multi(rt_server* s, const rt_camera* cam, const rt_source* sources, uint32_t n_sources,
                                 rt_pixel_out* pixels, const rt_ray_out* rays, size_t capacity, uint64_t* id) {
    return submit_request(s, cam, sources, n_sources, true, pixels, rays, capacity, id);
}

rt_status rt_server_poll(rt_server* s, rt_request_done* done, uint32_t max_done, uint32_t* n_done,
                         double timeout_ms) {
    if (!s || !n_done || (max_done > 0 && !done)) return RT_ERR_INVALID_ARG;
    *n_done = 0;
    std::unique_lock<std::mutex> lk(s->mu);
    if (s->completed.empty() && timeout_ms > 0.0)
        s->cv_done.wait_for(lk, std::chrono::duration<double, std::milli>(timeout_ms),
                            [s] { return !s->completed.empty(); });
    while (*n_done < max_done && !s->completed.empty()) {
        done[(*n_done)++] = s->completed.front();
        s->completed.pop_front();
    }
    return RT_OK;
}

rt_status rt_server_get_stats(rt_server* s, rt_server_stats* out) {
    if (!s || !out) return RT_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    *out = s->stats;
    out->pending = static_cast<uint32_t>(s->waiting.size() + s->active.size());
    out->bytes_in_use = s->alloc.used() * s->bytes_per_ray;
    out->budget_bytes = s->arena_rays * s->bytes_per_ray;
    return RT_OK;
}

const char* rt_server_last_error(const rt_server* s) { return s ? s->error.c_str() : "null server"; }

rt_status rt_server_set_shading(rt_server* s, const rt_shading* sh) {
    if (!s) return RT_ERR_INVALID_ARG;
    std::lock_guard<std::mutex> lk(s->mu);
    if (!sh) {
        s->shade_on = false;
        return RT_OK;
    }
    rt_camera probe;
    rt_camera_defaults(&probe);
    ShadeDesc d;
    // no sky: the server's epochs record no exit directions
    if (sh->sky_enabled != 0u || sh->hydro_model > 1u || !build_shade_desc(probe, *sh, d) ||
        (s->cfg.record_mask & kShadeMask) != kShadeMask)
        return RT_ERR_INVALID_ARG;
    if (!s->dev_shade) {
        cudaSetDevice(s->device);
        if (cudaMalloc(&s->dev_shade, sizeof(ShadeDesc) * kShadeSlots) != cudaSuccess) {
            cudaGetLastError();
            s->dev_shade = nullptr;
            return RT_ERR_OOM;
        }
    }
    s->shading = *sh;
    s->shade_on = true;
    return RT_OK;
}

}  // extern "C"
