// Continuous-batching request loop for the range-Doppler chain (zkx_rd_server_*,
// zkx_rd_submit, zkx_rd_poll).
//
// Requests queue on the host in arrival order.  One worker thread per server takes the
// oldest pending request, fuses up to max_batch pending requests of the same shape and
// waveform with it, and admits the batch when a device slot is free (at most
// max_inflight batches queued on the GPU) and its workspace fits the HBM budget.  A
// batch is a three-stage pipeline over the server's streams:
//
//   copy-in stream   host-resident CPIs copied into the batch's workspace (device-resident
//                    CPIs are read in place)
//   compute stream   zkx_rd_execute_batch kernels, one launch per stage for the whole
//                    batch (range compression reads the CPIs through a pointer table)
//   copy-out stream  the requested outputs copied to each request's buffers, the
//                    workspace freed, then a host callback (completion, latency)
//
// so while one batch computes, the next copies in and the previous copies out, and the
// kernels of consecutive batches stay in order on one compute stream (a producer's
// output is still in L2 when its consumer runs).  The callback returns the workspace
// to the server's idle list and its bytes to the budget and wakes the worker, which admits
// more requests without waiting for the rest of the device work: requests that arrive
// while others are on the GPU join as soon as slots and memory free up.
//
// Workspaces are device blocks the server keeps: a batch takes the smallest idle block that
// is large enough, or a new one within the budget, and gives it back from its completion
// callback, when every copy and kernel that used it has finished.  After the first batches of each shape no
// allocation happens at all, and no stream ever waits for another batch's memory.
//
// Plans (replica spectrum and Doppler window, resident) are cached per (pulses,
// samples, replica length, waveform id) for the server's lifetime; a plan is built on
// the copy-in stream before the first batch that needs it.
#include <algorithm>
#include <chrono>
#include <climits>
#include <cmath>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <iterator>
#include <map>
#include <mutex>
#include <string>
#include <thread>
#include <tuple>
#include <vector>

#include "zkx_internal.h"

using namespace zkx;

namespace {

using Clock = std::chrono::steady_clock;

struct PlanKey {
    int pulses, samples, replica_length;
    uint64_t waveform;
    bool operator<(const PlanKey& o) const
    {
        return std::tie(pulses, samples, replica_length, waveform) <
               std::tie(o.pulses, o.samples, o.replica_length, o.waveform);
    }
    bool operator==(const PlanKey& o) const { return !(*this < o) && !(o < *this); }
};

struct PlanEntry {
    zkx_rd_plan plan = nullptr;
    cudaEvent_t ready = nullptr;
    int range_bins = 0, doppler_bins = 0;
};

struct Request {
    uint64_t ticket = 0;
    zkx_rd_request r{};
    bool x_on_device = false;  // read in place by the kernels
    PlanKey key{};
    Clock::time_point submitted;
    bool done = false;
    int status = ZKX_SUCCESS;
    std::string error;
};

constexpr size_t kAlign = 256;
// Host-resident cells per fused batch (two 1024 x 16384 CPIs): small CPIs batch up to max_batch,
// large ones cross the host link alone.
constexpr long long kMaxBatchCells = 1LL << 25;
// Cells per fused batch of any CPIs (one 2048 x 65536 CPI).
constexpr long long kMaxFusedCells = 1LL << 27;
size_t align_up(size_t n) { return (n + kAlign - 1) / kAlign * kAlign; }

// Workspace of one batch of `count` CPIs [P, N] (range nfft N, Doppler nfft P), of which
// `staged` are copied in from host memory.
struct Layout {
    size_t x = 0, compressed = 0, rd = 0, power = 0, threshold = 0, detections = 0,
           cumulative = 0, total = 0;
};

Layout batch_layout(int P, int N, int count, int staged, bool with_rd, bool compat)
{
    const size_t cells = (size_t)P * N, cube = (size_t)count * cells, map = cube;
    Layout l;
    size_t off = 0;
    l.x = off;          off += align_up((size_t)staged * cells * 8);
    l.compressed = off; off += align_up(cube * 8);
    l.power = off;      off += align_up(map * 4);
    l.threshold = off;  off += align_up(map * 4);
    l.detections = off; off += align_up(map);
    l.rd = off;         off += with_rd ? align_up(map * 8) : 0;
    l.cumulative = off; off += compat ? align_up(cells * 4) : 0;
    l.total = off;
    return l;
}

}  // namespace

struct zkx_rd_server_s {
    zkx_rd_server_desc d{};
    int device = 0;
    std::vector<cudaStream_t> streams;  // compute streams
    cudaStream_t copy_in = nullptr, copy_out = nullptr;
    std::vector<cudaEvent_t> free_events;  // reusable; returned by completion callbacks
    std::multimap<size_t, char*> idle;  // workspace blocks not in use, by size
    size_t held = 0;                    // bytes of every workspace block, in use or idle
    size_t budget = 0, in_use = 0, peak = 0, plan_bytes = 0;

    std::mutex mu;
    std::condition_variable work_cv;  // worker: new requests or freed capacity
    std::condition_variable done_cv;  // pollers: completions
    std::deque<Request*> pending;
    std::map<uint64_t, Request*> requests;  // every ticket not yet released by a poll
    std::map<PlanKey, PlanEntry> plans;
    std::thread worker;
    bool stop = false;
    int inflight = 0;
    uint64_t next_ticket = 1;
    unsigned next_stream = 0;

    std::vector<double> latency_us;
    uint64_t submitted = 0, completed = 0, failed = 0, batches = 0, batched_cpis = 0, refused = 0;
    Clock::time_point first_submit, last_done;
    bool have_first = false;
};

namespace {

struct Batch {
    zkx_rd_server_s* s = nullptr;
    std::vector<Request*> reqs;
    char* ws = nullptr;    // workspace block
    size_t bytes = 0;      // its size
    bool with_rd = false;  // some request of the batch wants the complex map
    int staged = 0;        // host-resident CPIs copied into the workspace
    cudaEvent_t in = nullptr, done = nullptr;
};

void finish_requests(zkx_rd_server_s* s, const std::vector<Request*>& reqs, int status,
                     const std::string& error, Clock::time_point now)
{
    for (Request* r : reqs) {
        r->done = true;
        r->status = status;
        r->error = error;
        if (status == ZKX_SUCCESS) {
            s->latency_us.push_back(
                std::chrono::duration<double, std::micro>(now - r->submitted).count());
            ++s->completed;
        } else {
            ++s->failed;
        }
    }
    s->last_done = now;
}

// Host callback after a batch's last copy: no CUDA calls allowed here.
void CUDART_CB batch_done(void* arg)
{
    Batch* b = static_cast<Batch*>(arg);
    zkx_rd_server_s* s = b->s;
    const Clock::time_point now = Clock::now();
    {
        std::lock_guard<std::mutex> lk(s->mu);
        finish_requests(s, b->reqs, ZKX_SUCCESS, std::string(), now);
        s->idle.emplace(b->bytes, b->ws);
        s->in_use -= b->bytes;
        --s->inflight;
        s->free_events.push_back(b->in);
        s->free_events.push_back(b->done);
    }
    s->work_cv.notify_all();
    s->done_cv.notify_all();
    delete b;
}

int make_plan(zkx_rd_server_s* s, const Request& r, cudaStream_t stream, PlanEntry* out)
{
    zkx_rd_desc d{};
    d.num_pulses = r.r.num_pulses;
    d.samples_per_pulse = r.r.samples_per_pulse;
    d.range_nfft = -1;
    d.doppler_nfft = -1;
    d.replica_length = r.r.replica_length;
    d.normalize = s->d.normalize;
    d.range_window = s->d.range_window;
    d.doppler_window = s->d.doppler_window;
    std::memcpy(d.guard_cells, s->d.guard_cells, sizeof d.guard_cells);
    std::memcpy(d.reference_cells, s->d.reference_cells, sizeof d.reference_cells);
    d.pfa = s->d.pfa;
    d.cfar_mode = s->d.cfar_mode;
    PlanEntry e;
    ZKX_TRY(zkx_rd_plan_create(&d, r.r.replica, nullptr, nullptr, stream, &e.plan));
    int rc = zkx_rd_plan_shape(e.plan, &e.range_bins, &e.doppler_bins);
    if (rc == ZKX_SUCCESS) {
        cudaError_t ce = cudaEventCreateWithFlags(&e.ready, cudaEventDisableTiming);
        if (ce == cudaSuccess) ce = cudaEventRecord(e.ready, stream);
        if (ce != cudaSuccess) rc = cuda_status(ce, "serving plan event");
    }
    if (rc != ZKX_SUCCESS) {
        if (e.ready) cudaEventDestroy(e.ready);
        zkx_rd_plan_destroy(e.plan);
        return rc;
    }
    *out = e;
    return ZKX_SUCCESS;
}

// Queues one batch on the three pipeline streams; on success the batch is owned by the
// copy-out stream's callback.
int issue_batch(zkx_rd_server_s* s, const PlanEntry& pe, Batch* b, const Layout& l,
                cudaStream_t compute)
{
    const Request& head = *b->reqs.front();
    const int P = head.r.num_pulses, N = head.r.samples_per_pulse;
    const size_t cube = (size_t)P * N, map = (size_t)pe.doppler_bins * pe.range_bins;
    const int count = (int)b->reqs.size();
    char* ws = b->ws;
    const void* table[kMaxRowTable];
    float2* staged = reinterpret_cast<float2*>(ws + l.x);
    int slot = 0;
    for (int i = 0; i < count; ++i) {
        const Request& q = *b->reqs[i];
        if (q.x_on_device) {
            table[i] = q.r.x;
            continue;
        }
        float2* dst = staged + (size_t)slot++ * cube;
        cudaError_t e = cudaMemcpyAsync(dst, q.r.x, cube * sizeof(float2), cudaMemcpyDefault, s->copy_in);
        if (e != cudaSuccess) return cuda_status(e, "serving input copy");
        table[i] = dst;
    }
    cudaError_t e = cudaEventRecord(b->in, s->copy_in);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(compute, b->in, 0);
    if (e != cudaSuccess) return cuda_status(e, "serving pipeline event");
    float2* rd = b->with_rd ? reinterpret_cast<float2*>(ws + l.rd) : nullptr;
    float* power = reinterpret_cast<float*>(ws + l.power);
    float* thr = reinterpret_cast<float*>(ws + l.threshold);
    uint8_t* det = reinterpret_cast<uint8_t*>(ws + l.detections);
    float* cum = s->d.cfar_mode == ZKX_CFAR_COMPAT ? reinterpret_cast<float*>(ws + l.cumulative) : nullptr;
    int rc = rd_execute_batch_ws(pe.plan, nullptr, count, ws + l.compressed, rd, power, thr, det, cum,
                                 compute, table);
    if (rc != ZKX_SUCCESS) return rc;
    e = cudaEventRecord(b->done, compute);
    if (e == cudaSuccess) e = cudaStreamWaitEvent(s->copy_out, b->done, 0);
    if (e != cudaSuccess) return cuda_status(e, "serving pipeline event");
    for (int i = 0; i < count; ++i) {
        const zkx_rd_request& q = b->reqs[i]->r;
        e = cudaMemcpyAsync(q.detections, det + i * map, map, cudaMemcpyDefault, s->copy_out);
        if (e == cudaSuccess && q.threshold)
            e = cudaMemcpyAsync(q.threshold, thr + i * map, map * 4, cudaMemcpyDefault, s->copy_out);
        if (e == cudaSuccess && q.power)
            e = cudaMemcpyAsync(q.power, power + i * map, map * 4, cudaMemcpyDefault, s->copy_out);
        if (e == cudaSuccess && q.rd)
            e = cudaMemcpyAsync(q.rd, rd + i * map, map * 8, cudaMemcpyDefault, s->copy_out);
        if (e != cudaSuccess) return cuda_status(e, "serving output copy");
    }
    ZKX_CUDA(cudaLaunchHostFunc(s->copy_out, batch_done, b));
    return ZKX_SUCCESS;
}

// Workspace blocks.  The budget bounds every byte the server holds on the device: the blocks
// of batches in flight (in_use), the idle blocks kept for reuse, and the resident plans, so
// held + plan_bytes <= budget at all times (held = in_use + the idle blocks).
//
// Block sizes are rounded up to classes 2^k * {1, 1.25, 1.5, 1.75} (at least 1 MB), so that the
// varying batch compositions of a request stream keep reusing a few blocks instead of
// allocating new ones (an allocation can stall the device).
size_t size_class(size_t need)
{
    size_t base = size_t(1) << 20;
    while (base * 2 <= need) base *= 2;
    for (size_t q = 4; q <= 8; ++q)
        if (base / 4 * q >= need) return base / 4 * q;
    return base * 2;
}

// Bytes of the budget not taken by blocks in flight and plans (idle blocks can be released).
size_t budget_room(const zkx_rd_server_s* s)
{
    const size_t taken = s->in_use + s->plan_bytes;
    return s->budget > taken ? s->budget - taken : 0;
}

// Whether a batch whose workspace needs `need` bytes can have a block now within the budget:
// an idle block large enough, or a new block once idle blocks are released.  Admission and
// acquire_block use the same rule, so an admitted batch always gets its block.
bool block_fits(const zkx_rd_server_s* s, size_t need)
{
    return s->idle.lower_bound(need) != s->idle.end() || need <= budget_room(s);
}

// A workspace block of at least `need_bytes` for a batch that block_fits admitted; called by
// the worker with the lock held, which it drops around allocation and release calls.  The
// smallest idle block that is large enough is reused, so that after the first batches the
// server holds about max_inflight blocks of the largest sizes and allocates nothing more (an
// allocation of gigabytes in the middle of a stream stalls every request behind it).
// Otherwise idle blocks are released (largest first) until a new block fits within the
// budget next to the blocks in flight; the new block takes its size class, or exactly
// `need_bytes` when the class would not fit.
int acquire_block(zkx_rd_server_s* s, std::unique_lock<std::mutex>& lk, size_t need_bytes, char** ws,
                  size_t* bytes)
{
    auto it = s->idle.lower_bound(need_bytes);
    if (it != s->idle.end()) {
        *ws = it->second;
        *bytes = it->first;
        s->idle.erase(it);
        return ZKX_SUCCESS;
    }
    const size_t room = budget_room(s);
    if (need_bytes > room) return fail(ZKX_OUT_OF_MEMORY, "serving: workspace exceeds the HBM budget");
    const size_t cls = size_class(need_bytes);
    const size_t need = cls <= room ? cls : need_bytes;
    std::vector<char*> release;
    while (s->held + need + s->plan_bytes > s->budget && !s->idle.empty()) {
        auto last = std::prev(s->idle.end());
        s->held -= last->first;
        release.push_back(last->second);
        s->idle.erase(last);
    }
    s->held += need;
    s->peak = std::max(s->peak, s->held);
    lk.unlock();
    for (char* p : release) cudaFree(p);  // waits for the device; completions need the lock
    char* p = nullptr;
    const cudaError_t e = cudaMalloc(&p, need);
    lk.lock();
    if (e != cudaSuccess) {
        s->held -= need;
        return cuda_status(e, "serving workspace");
    }
    *ws = p;
    *bytes = need;
    return ZKX_SUCCESS;
}

// An event from the free list (or a new one); called by the worker with the lock held.
int take_event(zkx_rd_server_s* s, cudaEvent_t* out)
{
    if (!s->free_events.empty()) {
        *out = s->free_events.back();
        s->free_events.pop_back();
        return ZKX_SUCCESS;
    }
    ZKX_CUDA(cudaEventCreateWithFlags(out, cudaEventDisableTiming));
    return ZKX_SUCCESS;
}

void worker_main(zkx_rd_server_s* s)
{
    cudaSetDevice(s->device);
    std::unique_lock<std::mutex> lk(s->mu);
    for (;;) {
        if (s->pending.empty()) {
            if (s->stop && s->inflight == 0) break;
            s->work_cv.wait(lk);
            continue;
        }
        if (s->inflight >= s->d.max_inflight) {
            s->work_cv.wait(lk);
            continue;
        }
        Request* head = s->pending.front();
        const cudaStream_t stream = s->streams[s->next_stream % s->streams.size()];
        auto it = s->plans.find(head->key);
        if (it == s->plans.end()) {
            PlanEntry pe;
            Request copy = *head;
            lk.unlock();
            // built on the copy-in stream, which every batch passes through first
            const int rc = make_plan(s, copy, s->copy_in, &pe);
            const std::string msg = rc == ZKX_SUCCESS ? std::string() : std::string(zkx_last_error());
            lk.lock();
            if (rc != ZKX_SUCCESS) {
                // fail every pending request of this key: they would build the same plan
                std::vector<Request*> bad;
                for (auto q = s->pending.begin(); q != s->pending.end();) {
                    if ((*q)->key == copy.key) {
                        bad.push_back(*q);
                        q = s->pending.erase(q);
                    } else {
                        ++q;
                    }
                }
                finish_requests(s, bad, rc, msg, Clock::now());
                s->done_cv.notify_all();
                continue;
            }
            s->plan_bytes += (size_t)pe.range_bins * 8 + (size_t)pe.doppler_bins * 4;
            it = s->plans.emplace(head->key, pe).first;
            // the plan's bytes count against the budget too: give back idle blocks if needed
            std::vector<char*> release;
            while (s->held + s->plan_bytes > s->budget && !s->idle.empty()) {
                auto last = std::prev(s->idle.end());
                s->held -= last->first;
                release.push_back(last->second);
                s->idle.erase(last);
            }
            if (!release.empty()) {
                lk.unlock();
                for (char* p : release) cudaFree(p);
                lk.lock();
            }
            continue;  // re-evaluate with the plan in place
        }
        const PlanEntry pe = it->second;
        const bool compat = s->d.cfar_mode == ZKX_CFAR_COMPAT;
        // the oldest request and the next pending ones of its key, while they fit
        std::vector<Request*> group;
        bool with_rd = false;
        int staged = 0;
        Layout l{};
        const long long cells = (long long)head->r.num_pulses * head->r.samples_per_pulse;
        for (Request* q : s->pending) {
            if ((int)group.size() >= s->d.max_batch) break;
            if (!(q->key == head->key)) continue;
            // a batch stays within the kernels' int indexing, and CPIs this large fill the GPU
            // on their own (their workspaces would only grow)
            if (!group.empty() && (long long)(group.size() + 1) * cells > kMaxFusedCells) break;
            // host-resident CPIs this large keep the host link busy on their own: fusing more
            // of them only makes the first ones wait for the last copy
            if (!group.empty() && !q->x_on_device && (long long)(staged + 1) * cells > kMaxBatchCells) break;
            const int st = staged + (q->x_on_device ? 0 : 1);
            const Layout trial = batch_layout(head->r.num_pulses, head->r.samples_per_pulse,
                                              (int)group.size() + 1, st, with_rd || q->r.rd, compat);
            if (!block_fits(s, trial.total)) break;
            group.push_back(q);
            with_rd = with_rd || q->r.rd;
            staged = st;
            l = trial;
        }
        if (group.empty()) {
            if (s->inflight == 0) {
                // nothing on the device will free memory: this request cannot run
                s->pending.pop_front();
                finish_requests(s, {head}, ZKX_OUT_OF_MEMORY, "serving: request exceeds the HBM budget",
                                Clock::now());
                s->done_cv.notify_all();
            } else {
                s->work_cv.wait(lk);
            }
            continue;
        }
        for (Request* q : group) s->pending.erase(std::find(s->pending.begin(), s->pending.end(), q));
        char* block = nullptr;
        size_t block_bytes = 0;
        ++s->inflight;  // holds the slot while the lock may be dropped
        int arc = acquire_block(s, lk, l.total, &block, &block_bytes);
        if (arc != ZKX_SUCCESS) {
            --s->inflight;
            finish_requests(s, group, arc, std::string(zkx_last_error()), Clock::now());
            s->done_cv.notify_all();
            continue;
        }
        s->in_use += block_bytes;
        ++s->next_stream;
        ++s->batches;
        s->batched_cpis += group.size();
        Batch* b = new Batch;
        b->s = s;
        b->reqs = group;
        b->ws = block;
        b->bytes = block_bytes;
        b->with_rd = with_rd;
        b->staged = staged;
        int rc = take_event(s, &b->in);
        if (rc == ZKX_SUCCESS) rc = take_event(s, &b->done);
        lk.unlock();
        if (rc == ZKX_SUCCESS) rc = issue_batch(s, pe, b, l, stream);
        const std::string msg = rc == ZKX_SUCCESS ? std::string() : std::string(zkx_last_error());
        if (rc != ZKX_SUCCESS) {
            // work already queued may still read the block: let it drain before reuse
            cudaStreamSynchronize(s->copy_in);
            cudaStreamSynchronize(stream);
            cudaStreamSynchronize(s->copy_out);
        }
        lk.lock();
        if (rc != ZKX_SUCCESS) {
            finish_requests(s, b->reqs, rc, msg, Clock::now());
            s->idle.emplace(b->bytes, b->ws);
            s->in_use -= b->bytes;
            --s->inflight;
            if (b->in) s->free_events.push_back(b->in);
            if (b->done) s->free_events.push_back(b->done);
            delete b;
            s->done_cv.notify_all();
        }
    }
}

int validate_request(const zkx_rd_request* r)
{
    if (!r || !r->x || !r->replica || !r->detections)
        return fail(ZKX_INVALID_ARGUMENT, "rd_submit: null pointer");
    if (r->num_pulses < 1 || r->samples_per_pulse < 1 || r->replica_length < 1)
        return fail(ZKX_INVALID_SHAPE, "rd_submit: shape must be positive");
    // the plan transforms each CPI at its own extents: powers of two up to 65536, any
    // other length up to 32768
    for (int extent : {r->samples_per_pulse, r->num_pulses})
        if (extent > 65536 || (!is_pow2(extent) && extent > kMaxBluesteinLength))
            return fail(ZKX_UNSUPPORTED_OPERATION,
                        "rd_submit: pulses and samples must be at most 32768, or powers of two up to 65536");
    if ((long long)r->num_pulses * r->samples_per_pulse > INT_MAX)
        return fail(ZKX_INVALID_SHAPE, "rd_submit: CPI exceeds kernel capacity");
    return ZKX_SUCCESS;
}

}  // namespace

extern "C" int zkx_rd_server_create(const zkx_rd_server_desc* desc, zkx_rd_server* out)
{
    if (!desc || !out) return fail(ZKX_INVALID_ARGUMENT, "rd_server_create: null pointer");
    *out = nullptr;
    zkx_rd_server_desc d = *desc;
    // 2 compute streams and batches of up to 32: on the mixed burst of device-resident CPIs
    // 8850-8950 CPIs/s against 8170-8540 with 4 streams and 16 (fewer batches interleaved on
    // the device evict each other's cubes from L2 less often)
    if (d.streams <= 0) d.streams = 2;
    if (d.max_inflight <= 0) d.max_inflight = 2 * d.streams;
    if (d.max_batch <= 0) d.max_batch = 32;
    if (d.hbm_fraction <= 0) d.hbm_fraction = 0.8;
    if (d.max_pending < 0) return fail(ZKX_INVALID_ARGUMENT, "rd_server_create: max_pending must be >= 0");
    if (d.hbm_fraction > 1 || d.streams > 64 || d.max_batch > kMaxRowTable)
        return fail(ZKX_INVALID_ARGUMENT,
                    "rd_server_create: hbm_fraction <= 1, streams <= 64 and max_batch <= 64 required");
    const bool windows_ok = d.range_window >= ZKX_WINDOW_NONE && d.range_window <= ZKX_WINDOW_HAMMING &&
                            d.doppler_window >= ZKX_WINDOW_NONE && d.doppler_window <= ZKX_WINDOW_HAMMING;
    if (!windows_ok) return fail(ZKX_INVALID_ARGUMENT, "rd_server_create: windows must be none, hann or hamming");
    if (d.cfar_mode != ZKX_CFAR_ACCURATE && d.cfar_mode != ZKX_CFAR_COMPAT)
        return fail(ZKX_INVALID_ARGUMENT, "rd_server_create: unknown CFAR mode");
    ZKX_TRY(ensure_device_ready());
    auto* s = new zkx_rd_server_s;
    s->d = d;
    auto cleanup = [&](int rc) {
        for (cudaStream_t st : s->streams) cudaStreamDestroy(st);
        if (s->copy_in) cudaStreamDestroy(s->copy_in);
        if (s->copy_out) cudaStreamDestroy(s->copy_out);
        delete s;
        return rc;
    };
    cudaError_t e = cudaGetDevice(&s->device);
    size_t free_bytes = 0, total_bytes = 0;
    if (e == cudaSuccess) e = cudaMemGetInfo(&free_bytes, &total_bytes);
    if (e != cudaSuccess) return cleanup(cuda_status(e, "rd_server_create"));
    s->budget = (size_t)(d.hbm_fraction * (double)free_bytes);
    if (d.budget_bytes) s->budget = std::min(s->budget, d.budget_bytes);
    for (int i = 0; i < d.streams; ++i) {
        cudaStream_t st;
        e = cudaStreamCreateWithFlags(&st, cudaStreamNonBlocking);
        if (e != cudaSuccess) return cleanup(cuda_status(e, "rd_server_create: stream"));
        s->streams.push_back(st);
    }
    e = cudaStreamCreateWithFlags(&s->copy_in, cudaStreamNonBlocking);
    if (e == cudaSuccess) e = cudaStreamCreateWithFlags(&s->copy_out, cudaStreamNonBlocking);
    if (e != cudaSuccess) return cleanup(cuda_status(e, "rd_server_create: stream"));
    s->worker = std::thread(worker_main, s);
    *out = s;
    return ZKX_SUCCESS;
}

extern "C" int zkx_rd_server_destroy(zkx_rd_server s)
{
    if (!s) return ZKX_SUCCESS;
    {
        std::lock_guard<std::mutex> lk(s->mu);
        s->stop = true;
    }
    s->work_cv.notify_all();
    if (s->worker.joinable()) s->worker.join();
    for (cudaStream_t st : s->streams) cudaStreamSynchronize(st);
    cudaStreamSynchronize(s->copy_in);
    cudaStreamSynchronize(s->copy_out);
    for (cudaStream_t st : s->streams) cudaStreamDestroy(st);
    cudaStreamDestroy(s->copy_in);
    cudaStreamDestroy(s->copy_out);
    for (cudaEvent_t ev : s->free_events) cudaEventDestroy(ev);
    for (auto& kv : s->plans) {
        cudaEventDestroy(kv.second.ready);
        zkx_rd_plan_destroy(kv.second.plan);
    }
    for (auto& kv : s->idle) cudaFree(kv.second);
    for (auto& kv : s->requests) delete kv.second;
    delete s;
    return ZKX_SUCCESS;
}

extern "C" int zkx_rd_submit(zkx_rd_server s, const zkx_rd_request* r, uint64_t* ticket)
{
    if (!s || !ticket) return fail(ZKX_INVALID_ARGUMENT, "rd_submit: null pointer");
    ZKX_TRY(validate_request(r));
    cudaPointerAttributes attr{};
    const cudaError_t pe = cudaPointerGetAttributes(&attr, r->x);
    if (pe != cudaSuccess) return cuda_status(pe, "rd_submit: input pointer");
    const bool on_device = attr.type == cudaMemoryTypeDevice || attr.type == cudaMemoryTypeManaged;
    const Layout one = batch_layout(r->num_pulses, r->samples_per_pulse, 1, on_device ? 0 : 1,
                                    r->rd != nullptr, s->d.cfar_mode == ZKX_CFAR_COMPAT);
    auto* q = new Request;
    q->r = *r;
    q->x_on_device = on_device;
    q->key = PlanKey{r->num_pulses, r->samples_per_pulse, r->replica_length, r->waveform_id};
    {
        std::lock_guard<std::mutex> lk(s->mu);
        if (one.total > s->budget) {
            delete q;
            return fail(ZKX_OUT_OF_MEMORY, "rd_submit: the CPI's workspace exceeds the HBM budget");
        }
        if (s->stop) {
            delete q;
            return fail(ZKX_INVALID_ARGUMENT, "rd_submit: server is shutting down");
        }
        if (s->d.max_pending > 0 && s->pending.size() >= (size_t)s->d.max_pending) {
            delete q;
            ++s->refused;
            return fail(ZKX_RESOURCE_FAILED, "rd_submit: max_pending requests are waiting for admission");
        }
        q->ticket = s->next_ticket++;
        q->submitted = Clock::now();
        if (!s->have_first) {
            s->first_submit = q->submitted;
            s->have_first = true;
        }
        ++s->submitted;
        s->requests[q->ticket] = q;
        s->pending.push_back(q);
        *ticket = q->ticket;
    }
    s->work_cv.notify_all();
    return ZKX_SUCCESS;
}

extern "C" int zkx_rd_poll(zkx_rd_server s, uint64_t ticket, int timeout_ms, int* done)
{
    if (!s || !done) return fail(ZKX_INVALID_ARGUMENT, "rd_poll: null pointer");
    *done = 0;
    std::unique_lock<std::mutex> lk(s->mu);
    auto it = s->requests.find(ticket);
    if (it == s->requests.end()) return fail(ZKX_INVALID_ARGUMENT, "rd_poll: unknown ticket");
    Request* q = it->second;
    if (!q->done && timeout_ms != 0) {
        if (timeout_ms < 0)
            s->done_cv.wait(lk, [&] { return q->done; });
        else
            s->done_cv.wait_for(lk, std::chrono::milliseconds(timeout_ms), [&] { return q->done; });
    }
    if (!q->done) return ZKX_SUCCESS;
    *done = 1;
    const int status = q->status;
    const std::string msg = q->error;
    s->requests.erase(it);
    delete q;
    if (status != ZKX_SUCCESS) return fail(status, msg);
    return ZKX_SUCCESS;
}

extern "C" int zkx_rd_server_stats_get(zkx_rd_server s, zkx_rd_server_stats* out)
{
    if (!s || !out) return fail(ZKX_INVALID_ARGUMENT, "rd_server_stats: null pointer");
    std::lock_guard<std::mutex> lk(s->mu);
    zkx_rd_server_stats st{};
    st.submitted = s->submitted;
    st.completed = s->completed;
    st.failed = s->failed;
    st.batches = s->batches;
    st.mean_batch = s->batches ? (double)s->batched_cpis / (double)s->batches : 0.0;
    if (!s->latency_us.empty()) {
        std::vector<double> v = s->latency_us;
        std::sort(v.begin(), v.end());
        auto pct = [&](double p) {
            const size_t i = (size_t)std::min<double>((double)v.size() - 1, std::ceil(p * (double)v.size()) - 1);
            return v[i];
        };
        st.p50_us = pct(0.50);
        st.p99_us = pct(0.99);
        st.max_us = v.back();
        double sum = 0;
        for (double x : v) sum += x;
        st.mean_us = sum / (double)v.size();
    }
    if (s->have_first && s->completed) {
        const double secs = std::chrono::duration<double>(s->last_done - s->first_submit).count();
        st.cpis_per_s = secs > 0 ? (double)s->completed / secs : 0.0;
    }
    st.budget_bytes = s->budget;
    st.peak_bytes = s->peak;
    st.plan_bytes = s->plan_bytes;
    st.plans = (int)s->plans.size();
    st.refused = s->refused;
    *out = st;
    return ZKX_SUCCESS;
}

extern "C" int zkx_rd_server_stats_reset(zkx_rd_server s)
{
    if (!s) return fail(ZKX_INVALID_ARGUMENT, "rd_server_stats: null pointer");
    std::lock_guard<std::mutex> lk(s->mu);
    s->latency_us.clear();
    s->submitted = s->completed = s->failed = s->batches = s->batched_cpis = s->refused = 0;
    s->have_first = false;
    s->peak = s->held;
    return ZKX_SUCCESS;
}
