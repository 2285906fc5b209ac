// serve.cu -- continuous-batching evaluation server for many GP runs.
//
// Independent GP runs (each with its own dataset) submit one generation at a
// time.  A worker thread owns all device work:
//   - admission: a request is admitted when its run's dataset is on the
//     device or fits the HBM budget (datasets of runs with nothing queued or
//     running are evicted to make room); requests that do not fit wait, later
//     requests of resident runs go ahead of them;
//   - batching: admitted requests are appended to a free pooled batch
//     ("slot") until its capacity is reached, then that batch is launched on
//     its own stream -- one persistent interpreter launch for all of them;
//   - overlap: with several slots, a batch is composed and copied while
//     earlier batches still run, and its kernels start as SMs free up;
//   - completion: a finished slot's fitness vectors are copied to the
//     callers' buffers (one device-to-host copy per batch) and waiters are
//     woken.
// Programs are copied at submission, on the caller's thread, into a pinned
// ring buffer, so a batch's host-to-device copies run asynchronously; a
// request that does not fit the ring keeps a pageable copy instead.
// Case chunking depends only on a run's own dataset, so a request's fitness
// is the same alone and in any mix.
#include <cuda_runtime.h>
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <map>
#include <memory>
#include <mutex>
#include <thread>
#include <vector>

#include "../../include/galop_b200.h"
#include "context.cuh"

namespace {

using Clock = std::chrono::steady_clock;

double ms_between(Clock::time_point a, Clock::time_point b) {
    return std::chrono::duration<double, std::milli>(b - a).count();
}

struct Run {
    int32_t id = 0;
    std::vector<float> inputs, targets;   // host copy until closed
    int64_t n_cases = 0;
    int32_t num_inputs = 0;
    galop_dataset* ds = nullptr;          // resident copy (or null)
    int64_t ds_bytes = 0;
    int outstanding = 0;                  // queued + in flight
    bool closed = false;
    Clock::time_point last_use;
};

// Page-locked staging for submitted programs.  Blocks are reserved in
// submission order and released as batches complete (roughly FIFO); space is
// reclaimed from the oldest block once it and everything before it is free.
class PinnedRing {
public:
    ~PinnedRing() { if (base_) cudaFreeHost(base_); }
    bool init(size_t bytes) {
        if (bytes == 0) return true;
        if (cudaMallocHost(&base_, bytes) != cudaSuccess) { cudaGetLastError(); base_ = nullptr; return false; }
        cap_ = bytes;
        return true;
    }
    // Reserve n bytes (256-aligned); null when full.
    char* alloc(size_t n) {
        std::lock_guard<std::mutex> lk(mu_);
        if (!base_) return nullptr;
        n = (n + 255) & ~(size_t)255;
        if (live_.empty()) front_ = head_ = 0;
        size_t off;
        if (live_.empty() || head_ > front_ || (head_ == front_ && live_.empty())) {
            if (head_ + n <= cap_) off = head_;
            else if (n <= front_) off = 0;
            else return nullptr;
        } else {
            if (head_ + n <= front_) off = head_;
            else return nullptr;
        }
        live_.push_back({off, n, false});
        head_ = off + n;
        return base_ + off;
    }
    void release(const char* p) {
        std::lock_guard<std::mutex> lk(mu_);
        for (auto& b : live_)
            if (base_ + b.off == p) { b.freed = true; break; }
        while (!live_.empty() && live_.front().freed) live_.pop_front();
        front_ = live_.empty() ? head_ : live_.front().off;
    }
private:
    struct Block { size_t off, size; bool freed; };
    std::mutex mu_;
    char* base_ = nullptr;
    size_t cap_ = 0, front_ = 0, head_ = 0;
    std::deque<Block> live_;
};

struct Request {
    int64_t id = 0;
    int32_t run = 0;
    std::vector<uint32_t> words;          // pageable copy when the ring is full
    std::vector<int64_t> offsets;
    char* pinned = nullptr;               // ring block: offsets then words
    const uint32_t* w = nullptr;
    const int64_t* o = nullptr;
    int64_t n = 0;
    float* out = nullptr;
    int32_t status = 1;                   // 1 = pending, 0 = done, < 0 = error
    int32_t batch_requests = 0;
    int64_t eff = 0;
    int64_t n_cases = 0;
    Clock::time_point submitted, launched, done;
    double device_ms = 0.0;
};

struct Slot {
    galop_batch* batch = nullptr;
    std::vector<std::shared_ptr<Request>> reqs;
    std::vector<int32_t> pops;
    std::vector<float> fitness;           // whole-batch fitness, host side
    std::vector<int64_t> eff;             // interpreted instructions per population
    bool busy = false;
};

}  // namespace

struct galop_server {
    galop_ctx* ctx = nullptr;
    galop_server_options opt{};
    std::mutex mu;
    std::condition_variable cv_work, cv_done;
    std::thread worker;
    bool stop = false;
    int32_t next_run = 1;
    int64_t next_req = 1;
    std::map<int32_t, std::unique_ptr<Run>> runs;
    std::deque<std::shared_ptr<Request>> pending;
    std::map<int64_t, std::shared_ptr<Request>> by_id;
    std::vector<Slot> slots;
    PinnedRing ring;
    int64_t slot_bytes = 0;
    int64_t resident_bytes = 0;          // datasets on the device
    int64_t completed = 0, batches = 0, case_ops = 0;
    double device_ms_total = 0.0;
    int worker_error = 0;

    void loop();
    bool make_room(int64_t bytes);
    void complete(Slot& s);
    void compose(Slot& s);
};

bool galop_server::make_room(int64_t bytes) {
    const int64_t budget = opt.hbm_budget_bytes;
    while (slot_bytes + resident_bytes + bytes > budget) {
        Run* victim = nullptr;
        for (auto& kv : runs) {
            Run* r = kv.second.get();
            if (r->ds && r->outstanding == 0 && (!victim || r->last_use < victim->last_use)) victim = r;
        }
        if (!victim) return false;
        galop_dataset_destroy(victim->ds);
        victim->ds = nullptr;
        resident_bytes -= victim->ds_bytes;
    }
    return true;
}

void galop_server::compose(Slot& s) {
    s.reqs.clear();
    s.pops.clear();
    if (galop_batch_clear(s.batch) != GALOP_OK) return;
    for (auto it = pending.begin(); it != pending.end();) {
        std::shared_ptr<Request> q = *it;
        Run* r = runs[q->run].get();
        if (!r->ds) {
            const int64_t need = (int64_t)(std::max<int64_t>(1024, (r->n_cases + 1023) / 1024 * 1024) *
                                           (std::max(r->num_inputs, 1) + 1) * sizeof(float));
            if (!make_room(need)) { ++it; continue; }      // waits for memory; later requests may fit
            if (galop_dataset_create(ctx, r->inputs.data(), r->targets.data(), r->n_cases, r->num_inputs, &r->ds) !=
                GALOP_OK) {
                q->status = GALOP_E_NOMEM;
                q->done = Clock::now();
                if (q->pinned) ring.release(q->pinned);
                q->pinned = nullptr;
                --r->outstanding;
                it = pending.erase(it);
                cv_done.notify_all();
                continue;
            }
            r->ds_bytes = galop_dataset_device_bytes(r->ds);
            resident_bytes += r->ds_bytes;
        }
        int32_t pop = -1;
        const int rc = galop_batch_append(s.batch, r->ds, q->w, q->o, q->n, &pop);
        if (rc == GALOP_E_CAPACITY) {
            if (s.reqs.empty()) {                         // can never fit a slot
                q->status = GALOP_E_CAPACITY;
                q->done = Clock::now();
                if (q->pinned) ring.release(q->pinned);
                q->pinned = nullptr;
                --r->outstanding;
                it = pending.erase(it);
                cv_done.notify_all();
                continue;
            }
            break;
        }
        if (rc != GALOP_OK) {
            q->status = rc;
            q->done = Clock::now();
            if (q->pinned) ring.release(q->pinned);
            q->pinned = nullptr;
            --r->outstanding;
            it = pending.erase(it);
            cv_done.notify_all();
            continue;
        }
        r->last_use = Clock::now();
        s.reqs.push_back(q);
        s.pops.push_back(pop);
        it = pending.erase(it);
    }
    if (s.reqs.empty()) return;
    const auto now = Clock::now();
    for (auto& q : s.reqs) {
        q->launched = now;
        q->batch_requests = (int32_t)s.reqs.size();
    }
    if (galop_batch_evaluate(s.batch, 0) != GALOP_OK) {
        for (auto& q : s.reqs) {
            q->status = GALOP_E_CUDA;
            q->done = Clock::now();
            if (q->pinned) ring.release(q->pinned);
            q->pinned = nullptr;
            --runs[q->run]->outstanding;
        }
        s.reqs.clear();
        cv_done.notify_all();
        return;
    }
    s.busy = true;
    ++batches;
}

void galop_server::complete(Slot& s) {
    galop_stats st{};
    galop_batch_last_stats(s.batch, &st);
    device_ms_total += st.total_ms;
    int64_t total = 0;
    for (auto& q : s.reqs) total += q->n;
    s.fitness.resize((size_t)std::max<int64_t>(total, 1));
    s.eff.resize(s.reqs.size());
    const int rc = galop_batch_get_fitness_all(s.batch, s.fitness.data(), s.eff.data());
    int64_t o = 0;
    const auto now = Clock::now();
    for (size_t i = 0; i < s.reqs.size(); ++i) {
        Request& q = *s.reqs[i];
        Run* r = runs[q.run].get();
        if (rc == GALOP_OK) {
            if (q.n) std::memcpy(q.out, s.fitness.data() + o, (size_t)q.n * sizeof(float));
            q.eff = s.eff[i];
            case_ops += q.eff * r->n_cases;
        }
        o += q.n;
        if (q.pinned) ring.release(q.pinned);
        q.pinned = nullptr;
        q.status = rc;
        q.device_ms = st.total_ms;
        q.done = now;
        --r->outstanding;
        r->last_use = now;
        ++completed;
    }
    s.reqs.clear();
    s.pops.clear();
    s.busy = false;
    cv_done.notify_all();
}

void galop_server::loop() {
    cudaSetDevice(ctx->device);
    std::unique_lock<std::mutex> lk(mu);
    for (;;) {
        bool progressed = false;
        for (Slot& s : slots) {
            if (s.busy && cudaStreamQuery((cudaStream_t)galop_batch_stream(s.batch)) != cudaErrorNotReady) {
                complete(s);
                progressed = true;
            }
        }
        for (Slot& s : slots) {
            if (!s.busy && !pending.empty()) {
                const size_t before = pending.size();
                compose(s);
                progressed |= pending.size() != before;
            }
        }
        // free datasets of closed runs with nothing outstanding
        for (auto it = runs.begin(); it != runs.end();) {
            Run* r = it->second.get();
            if (r->closed && r->outstanding == 0) {
                if (r->ds) {
                    galop_dataset_destroy(r->ds);
                    resident_bytes -= r->ds_bytes;
                }
                it = runs.erase(it);
                progressed = true;
            } else {
                ++it;
            }
        }
        bool busy = false;
        for (Slot& s : slots) busy |= s.busy;
        if (stop && !busy && pending.empty()) break;
        if (!progressed) {
            if (busy) {
                lk.unlock();
                std::this_thread::sleep_for(std::chrono::microseconds(50));
                lk.lock();
            } else {
                cv_work.wait_for(lk, std::chrono::milliseconds(5));
            }
        }
    }
}

extern "C" {

int galop_server_options_init(galop_server_options* o) {
    if (!o) return GALOP_E_INVALID;
    std::memset(o, 0, sizeof *o);
    o->hbm_budget_bytes = 150LL * 1000 * 1000 * 1000;
    o->slots = 4;
    o->pinned_bytes = 1LL << 30;
    o->max_pops_per_batch = 64;
    o->slot_programs = 1 << 20;
    o->slot_words = 1LL << 27;
    o->slot_items = 1LL << 23;
    return GALOP_OK;
}

int galop_server_create(galop_ctx* ctx, const galop_server_options* opt, galop_server** out) {
    if (!ctx || !out) return GALOP_E_INVALID;
    *out = nullptr;
    galop_server_options o;
    galop_server_options_init(&o);
    if (opt) o = *opt;
    if (o.slots < 1 || o.max_pops_per_batch < 1 || o.slot_programs < 1 || o.slot_words < 1 || o.slot_items < 1)
        return ctx->fail(GALOP_E_INVALID, "bad server options");
    auto* sv = new galop_server();
    sv->ctx = ctx;
    sv->opt = o;
    sv->ring.init((size_t)std::max<int64_t>(o.pinned_bytes, 0));   // without it, pageable copies
    sv->slots.resize(o.slots);
    for (Slot& s : sv->slots) {
        const int rc = galop_batch_create_pool(ctx, o.max_pops_per_batch, o.slot_programs, o.slot_words,
                                               o.slot_items, &s.batch);
        if (rc != GALOP_OK) {
            for (Slot& t : sv->slots) if (t.batch) galop_batch_destroy(t.batch);
            delete sv;
            return rc;
        }
        sv->slot_bytes += galop_batch_device_bytes(s.batch);
    }
    if (sv->slot_bytes > o.hbm_budget_bytes) {
        for (Slot& t : sv->slots) galop_batch_destroy(t.batch);
        delete sv;
        return ctx->fail(GALOP_E_CAPACITY, "slot buffers alone exceed the HBM budget");
    }
    sv->worker = std::thread([sv] { sv->loop(); });
    *out = sv;
    return GALOP_OK;
}

int galop_server_destroy(galop_server* sv) {
    if (!sv) return GALOP_OK;
    {
        std::lock_guard<std::mutex> lk(sv->mu);
        sv->stop = true;
    }
    sv->cv_work.notify_all();
    sv->worker.join();
    for (auto& kv : sv->runs)
        if (kv.second->ds) galop_dataset_destroy(kv.second->ds);
    for (Slot& s : sv->slots) galop_batch_destroy(s.batch);
    delete sv;
    return GALOP_OK;
}

int galop_server_open_run(galop_server* sv, const float* inputs, const float* targets, int64_t n_cases,
                          int32_t num_inputs, int32_t* run_id) {
    if (!sv || !run_id || n_cases < 0 || num_inputs < 0 || num_inputs > sv->ctx->isa.num_registers)
        return GALOP_E_INVALID;
    if (n_cases > 0 && (!targets || (num_inputs > 0 && !inputs))) return GALOP_E_INVALID;
    auto r = std::make_unique<Run>();
    r->inputs.assign(inputs, inputs + (size_t)n_cases * num_inputs);
    r->targets.assign(targets, targets + (size_t)n_cases);
    r->n_cases = n_cases;
    r->num_inputs = num_inputs;
    r->last_use = Clock::now();
    std::lock_guard<std::mutex> lk(sv->mu);
    r->id = sv->next_run++;
    *run_id = r->id;
    sv->runs[r->id] = std::move(r);
    return GALOP_OK;
}

int galop_server_close_run(galop_server* sv, int32_t run_id) {
    if (!sv) return GALOP_E_INVALID;
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->runs.find(run_id);
    if (it == sv->runs.end()) return GALOP_E_INVALID;
    it->second->closed = true;
    sv->cv_work.notify_all();
    return GALOP_OK;
}

int galop_server_submit(galop_server* sv, int32_t run_id, const uint32_t* words, const int64_t* offsets,
                        int64_t n_programs, float* fitness_out, int64_t* request_id) {
    if (!sv || !offsets || n_programs < 0 || !request_id || (n_programs > 0 && !fitness_out)) return GALOP_E_INVALID;
    if (offsets[0] != 0) return GALOP_E_INVALID;
    for (int64_t i = 0; i < n_programs; ++i)
        if (offsets[i + 1] < offsets[i]) return GALOP_E_INVALID;
    auto q = std::make_shared<Request>();
    const int64_t total = offsets[n_programs];
    const size_t ob = (size_t)(n_programs + 1) * sizeof(int64_t);
    const size_t bytes = ((ob + 255) & ~(size_t)255) + (size_t)total * sizeof(uint32_t);
    q->pinned = sv->ring.alloc(bytes);
    if (q->pinned) {
        std::memcpy(q->pinned, offsets, ob);
        q->o = reinterpret_cast<const int64_t*>(q->pinned);
        uint32_t* wdst = reinterpret_cast<uint32_t*>(q->pinned + ((ob + 255) & ~(size_t)255));
        if (total) std::memcpy(wdst, words, (size_t)total * sizeof(uint32_t));
        q->w = wdst;
    } else {
        q->words.assign(words, words + total);
        q->offsets.assign(offsets, offsets + n_programs + 1);
        q->w = q->words.data();
        q->o = q->offsets.data();
    }
    q->n = n_programs;
    q->out = fitness_out;
    q->run = run_id;
    q->submitted = Clock::now();
    std::lock_guard<std::mutex> lk(sv->mu);
    auto it = sv->runs.find(run_id);
    if (it == sv->runs.end() || it->second->closed) {
        if (q->pinned) sv->ring.release(q->pinned);
        return GALOP_E_INVALID;
    }
    q->id = sv->next_req++;
    *request_id = q->id;
    ++it->second->outstanding;
    sv->by_id[q->id] = q;
    sv->pending.push_back(q);
    sv->cv_work.notify_all();
    return GALOP_OK;
}

int galop_server_wait(galop_server* sv, int64_t request_id, double timeout_s, galop_request_info* info) {
    if (!sv) return GALOP_E_INVALID;
    std::unique_lock<std::mutex> lk(sv->mu);
    auto it = sv->by_id.find(request_id);
    if (it == sv->by_id.end()) return GALOP_E_INVALID;
    std::shared_ptr<Request> q = it->second;
    const auto deadline = Clock::now() + std::chrono::duration_cast<Clock::duration>(
                                             std::chrono::duration<double>(timeout_s > 0 ? timeout_s : 1e9));
    while (q->status == 1) {
        if (sv->cv_done.wait_until(lk, deadline) == std::cv_status::timeout && q->status == 1)
            return GALOP_E_TIMEOUT;
    }
    if (info) {
        info->status = q->status;
        info->batch_requests = q->batch_requests;
        info->queued_ms = q->status == 0 ? ms_between(q->submitted, q->launched) : 0.0;
        info->latency_ms = ms_between(q->submitted, q->done);
        info->device_ms = q->device_ms;
        info->eff_instructions = q->eff;
    }
    sv->by_id.erase(request_id);
    return q->status;
}

int galop_server_stats(galop_server* sv, galop_server_totals* out) {
    if (!sv || !out) return GALOP_E_INVALID;
    std::lock_guard<std::mutex> lk(sv->mu);
    out->completed = sv->completed;
    out->batches = sv->batches;
    out->pending = (int64_t)sv->pending.size();
    out->resident_bytes = sv->resident_bytes + sv->slot_bytes;
    out->case_ops = sv->case_ops;
    out->device_ms = sv->device_ms_total;
    return GALOP_OK;
}

}  // extern "C"
