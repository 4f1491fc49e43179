// server.cpp — continuous-batching prediction server over a device-resident
// forest (the serving pattern of the engine; the reference predicts one call
// at a time through Predictor::predict_into, inference/gbdt/predictor.rs:197).
//
// Requests (sample-major f32 rows, caller-owned input and output buffers in
// host or device memory: the copies go by unified addressing) are admitted
// FIFO into a device row ring as soon as it has room: the
// admission issues the request's host-to-device copy at once on one of two
// copy streams, so copies proceed while earlier batches traverse. A dispatcher
// coalesces admitted requests that sit contiguously in the ring into one
// batch per free slot (SLOTS batches in flight), makes the slot's stream
// wait for the batch's copies, runs ONE traversal launch over the ring
// span and copies each request's outputs straight back to the caller. A
// completion thread retires batches in order, frees their ring span, admits
// waiting requests and wakes the waiters. A row's prediction depends on that
// row alone (trees summed in forest order per row), so every result is
// identical whatever batch it shares.
#include <algorithm>
#include <chrono>
#include <condition_variable>
#include <cstring>
#include <deque>
#include <mutex>
#include <thread>
#include <unordered_map>
#include <vector>

#include "engine.h"

namespace bst {

namespace {

uint64_t now_ns() {
    return (uint64_t)std::chrono::duration_cast<std::chrono::nanoseconds>(
               std::chrono::steady_clock::now().time_since_epoch())
        .count();
}

}  // namespace

struct Server {
    static constexpr int SLOTS = 3;
    // Coalescing stops at one full wave of the traversal (one 768-row tile
    // per SM) unless the caller caps batches explicitly: a larger batch runs
    // in two waves and holds every request in it for both.
    static constexpr uint64_t WAVE_TILE_ROWS = 768ull;

    struct Req {
        uint64_t id = 0;
        const float* rows = nullptr;
        uint64_t n = 0;
        float* out = nullptr;
        uint64_t submit_ns = 0, done_ns = 0;
        uint64_t admit_ns = 0, dispatch_ns = 0;  // copy issued; batch launched
        int status = -1;      // -1 pending, else bst_status
        uint64_t pos = 0;     // first ring row, once admitted
        cudaEvent_t copy_start = nullptr;  // recorded before the request's copy
        cudaEvent_t copied = nullptr;      // recorded after the request's copy
    };
    struct Slot {
        DevArray<float> d_out;
        DevArray<unsigned char> scratch;  // the traversal's bin tiles
        cudaStream_t st = nullptr;
        cudaEvent_t done = nullptr;        // after the output copies
        cudaEvent_t k0 = nullptr, k1 = nullptr;  // around binning + traversal + transform
        std::vector<uint64_t> reqs;  // ticket ids, in ring order
        uint64_t rows = 0;
        bool busy = false;
    };

    const Model& m;
    uint64_t F = 0, G = 1, max_rows = 0, coalesce_rows = 0, ring_rows = 0;
    bool raw = false;
    int device = 0;

    std::mutex mu;
    std::condition_variable cv_work, cv_done, cv_inflight;
    std::unordered_map<uint64_t, Req> reqs;
    std::deque<uint64_t> pending;   // waiting for ring room
    std::deque<uint64_t> admitted;  // copy issued, not yet in a batch
    std::deque<std::pair<uint64_t, uint64_t>> live;  // ring spans (start, n) of admitted requests, in order
    std::deque<int> inflight;       // slot indices in issue order
    std::vector<cudaEvent_t> events;  // free copy events
    DevArray<float> ring;
    // host-to-device copies of the requests, in admission order; two
    // streams taking turns lowered the measured copy rate (46 -> 42 GB/s)
    // and raised the 10k req/s p99 (1.85 -> 2.15 ms), so one
    static constexpr int COPY_STREAMS = 1;
    cudaStream_t cst[COPY_STREAMS] = {nullptr};
    uint64_t copies_issued = 0;
    Slot slots[SLOTS];
    uint64_t next_id = 1;
    bool stop = false;
    int error = BST_OK;
    std::string error_msg;
    bst_server_stats stats{};
    // per-request phase record of every completed request, until drained
    // (bst_server_trace); capped so an undrained server stays bounded
    static constexpr size_t TRACE_MAX = 1u << 20;
    std::vector<bst_server_phase> trace;
    std::thread dispatcher, completer;

    cudaEvent_t take_event() {  // caller holds mu
        cudaEvent_t ev;
        if (!events.empty()) {
            ev = events.back();
            events.pop_back();
        } else {
            BST_CK(cudaEventCreate(&ev));  // timing enabled: the copy's duration is traced
        }
        return ev;
    }

    Server(const Model& model, uint64_t budget, uint64_t cap, bool raw_out) : m(model), raw(raw_out) {
        device = m.device;
        BST_CK(cudaSetDevice(device));
        F = m.n_features;
        G = m.n_groups;
        const DeviceForest& df = m.device_forest();  // forest resident before the first request
        // per row and slot: its input rows (in the ring), outputs and bin tiles
        const uint64_t per_row = (F + G) * sizeof(float) + forest_bin_bytes_per_row(df, F);
        max_rows = budget / ((uint64_t)SLOTS * std::max<uint64_t>(1, per_row));
        if (cap) max_rows = std::min(max_rows, cap);
        if (max_rows == 0)
            throw Error{BST_ERR_INVALID_ARGUMENT, "memory budget below one row per in-flight slot"};
        if (max_rows > 0xFFFFFFFFull) max_rows = 0xFFFFFFFFull;
        coalesce_rows = cap ? max_rows : std::min(max_rows, (uint64_t)sm_count() * WAVE_TILE_ROWS);
        ring_rows = (uint64_t)SLOTS * max_rows;  // the slots' input share of the budget
        ring.alloc((size_t)ring_rows * std::max<uint64_t>(1, F));
        for (auto& c : cst) BST_CK(cudaStreamCreateWithFlags(&c, cudaStreamNonBlocking));
        const size_t scratch = forest_scratch_max(df, max_rows, F);
        for (auto& s : slots) {
            s.d_out.alloc((size_t)max_rows * G);
            if (scratch) s.scratch.alloc(scratch);
            BST_CK(cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking));
            BST_CK(cudaEventCreate(&s.done));
            BST_CK(cudaEventCreate(&s.k0));
            BST_CK(cudaEventCreate(&s.k1));
        }
        stats.max_batch_rows = max_rows;
        dispatcher = std::thread([this] { dispatch_loop(); });
        completer = std::thread([this] { complete_loop(); });
    }

    ~Server() {
        {
            // drain: every queued request is dispatched and completed first
            std::unique_lock<std::mutex> lk(mu);
            cv_done.wait(lk, [&] {
                if (error != BST_OK) return true;
                if (!pending.empty() || !admitted.empty() || !inflight.empty()) return false;
                for (auto& s : slots)
                    if (s.busy) return false;
                return true;
            });
            stop = true;
        }
        cv_work.notify_all();
        cv_inflight.notify_all();
        if (dispatcher.joinable()) dispatcher.join();
        if (completer.joinable()) completer.join();
        cudaSetDevice(device);
        for (auto c : cst)
            if (c) cudaStreamSynchronize(c);
        for (auto& s : slots) {
            if (s.st) cudaStreamSynchronize(s.st);
            if (s.done) cudaEventDestroy(s.done);
            if (s.k0) cudaEventDestroy(s.k0);
            if (s.k1) cudaEventDestroy(s.k1);
            if (s.st) cudaStreamDestroy(s.st);
        }
        for (auto& kv : reqs) {
            if (kv.second.copy_start) cudaEventDestroy(kv.second.copy_start);
            if (kv.second.copied) cudaEventDestroy(kv.second.copied);
        }
        for (cudaEvent_t e : events) cudaEventDestroy(e);
        for (auto c : cst)
            if (c) cudaStreamDestroy(c);
    }

    // Ring room for n rows after the live spans (contiguous; wraps to row 0).
    bool ring_alloc(uint64_t n, uint64_t* pos) const {
        if (live.empty()) {
            *pos = 0;
            return n <= ring_rows;
        }
        const uint64_t tail = live.front().first;
        const uint64_t head = live.back().first + live.back().second;
        // wrapped when the newest span starts before the oldest: the free
        // room is then [head, tail) alone (empty when head == tail)
        if (live.back().first >= tail) {
            if (n <= ring_rows - head) {
                *pos = head;
                return true;
            }
            if (n <= tail) {
                *pos = 0;
                return true;
            }
            return false;
        }
        if (n <= tail - head) {
            *pos = head;
            return true;
        }
        return false;
    }

    // Admits waiting requests while the ring has room: issues their copies.
    // Caller holds mu.
    void admit_locked() {
        bool any = false;
        while (!pending.empty() && error == BST_OK) {
            Req& r = reqs[pending.front()];
            uint64_t pos;
            if (!ring_alloc(r.n, &pos)) break;
            r.copy_start = take_event();
            r.copied = take_event();
            r.pos = pos;
            r.admit_ns = now_ns();
            cudaStream_t cs = cst[copies_issued++ % COPY_STREAMS];
            BST_CK(cudaEventRecord(r.copy_start, cs));
            if (F)
                BST_CK(cudaMemcpyAsync(ring.p + pos * F, r.rows, sizeof(float) * r.n * F, cudaMemcpyDefault, cs));
            BST_CK(cudaEventRecord(r.copied, cs));
            live.emplace_back(pos, r.n);
            admitted.push_back(r.id);
            pending.pop_front();
            any = true;
        }
        if (any) cv_work.notify_one();
    }

    uint64_t submit(const float* rows, uint64_t n, float* out) {
        if (n > max_rows)
            throw Error{BST_ERR_INVALID_ARGUMENT, "request of " + std::to_string(n) +
                                                      " rows exceeds the per-batch budget of " +
                                                      std::to_string(max_rows) + " rows"};
        std::lock_guard<std::mutex> lk(mu);
        if (error != BST_OK) throw Error{(bst_status)error, error_msg};
        Req r;
        r.id = next_id++;
        r.rows = rows;
        r.n = n;
        r.out = out;
        r.submit_ns = now_ns();
        stats.submitted += 1;
        if (n == 0) {  // nothing to predict: complete at once
            r.status = BST_OK;
            r.done_ns = r.submit_ns;
            stats.completed += 1;
            reqs.emplace(r.id, r);
            return r.id;
        }
        reqs.emplace(r.id, r);
        pending.push_back(r.id);
        try {
            BST_CK(cudaSetDevice(device));
            admit_locked();
        } catch (const Error& e) {
            fail_all(e.code, e.msg);
        }
        return r.id;
    }

    int wait(uint64_t id, int64_t timeout_ms, uint64_t* submit_ns, uint64_t* done_ns) {
        std::unique_lock<std::mutex> lk(mu);
        if (reqs.find(id) == reqs.end()) throw Error{BST_ERR_INVALID_ARGUMENT, "unknown or already retired ticket"};
        auto ready = [&] { return reqs[id].status >= 0; };
        if (timeout_ms < 0)
            cv_done.wait(lk, ready);
        else if (!cv_done.wait_for(lk, std::chrono::milliseconds(timeout_ms), ready))
            return BST_ERR_TIMEOUT;
        const Req r = reqs[id];
        reqs.erase(id);
        if (r.status != BST_OK) {  // never returned to the pool
            if (r.copy_start) cudaEventDestroy(r.copy_start);
            if (r.copied) cudaEventDestroy(r.copied);
        }
        if (submit_ns) *submit_ns = r.submit_ns;
        if (done_ns) *done_ns = r.done_ns;
        return r.status;
    }

    void fail_all(int code, const std::string& msg) {  // caller holds mu
        if (error == BST_OK) {
            error = code;
            error_msg = msg;
        }
        for (auto c : cst)  // no copy still reads a caller's rows
            if (c) cudaStreamSynchronize(c);
        const uint64_t t = now_ns();
        for (auto& kv : reqs)
            if (kv.second.status < 0) {
                kv.second.status = code;
                kv.second.done_ns = t;
            }
        pending.clear();
        admitted.clear();
        cv_done.notify_all();
        cv_work.notify_all();
    }

    void dispatch_loop() {
        cudaSetDevice(device);
        const DeviceForest& f = m.device_forest();
        const int tr = transform_of(m.objective);
        for (;;) {
            int si = -1;
            std::vector<Req> batch;
            uint64_t rows = 0;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_work.wait(lk, [&] {
                    if (stop) return true;
                    if (admitted.empty()) return false;
                    for (int i = 0; i < SLOTS; ++i)
                        if (!slots[i].busy) return true;
                    return false;
                });
                if (stop) return;
                for (int i = 0; i < SLOTS; ++i)
                    if (!slots[i].busy) {
                        si = i;
                        break;
                    }
                // the admitted head while contiguous in the ring and within
                // the coalescing limit (a single request up to the capacity)
                while (!admitted.empty()) {
                    const Req& r = reqs[admitted.front()];
                    if (!batch.empty() && (rows + r.n > coalesce_rows || r.pos != batch.back().pos + batch.back().n))
                        break;
                    batch.push_back(r);
                    rows += r.n;
                    admitted.pop_front();
                }
                Slot& s = slots[si];
                s.busy = true;
                s.reqs.clear();
                s.rows = rows;
                const uint64_t t = now_ns();
                for (auto& r : batch) {
                    s.reqs.push_back(r.id);
                    reqs[r.id].dispatch_ns = t;
                }
                stats.batches += 1;
                stats.rows += rows;
                stats.max_rows_seen = std::max<uint64_t>(stats.max_rows_seen, rows);
            }
            Slot& s = slots[si];
            try {
                for (const Req& r : batch)  // every request's copy (the copy streams run side by side)
                    BST_CK(cudaStreamWaitEvent(s.st, r.copied, 0));
                BST_CK(cudaEventRecord(s.k0, s.st));
                forest_predict_rows(f, ring.p + batch.front().pos * F, rows, F, s.d_out.p, s.st, s.scratch.p,
                                    s.scratch.n);
                if (!raw) launch_transform(tr, s.d_out.p, (uint32_t)G, rows, s.st);
                BST_CK(cudaGetLastError());
                BST_CK(cudaEventRecord(s.k1, s.st));
                uint64_t off = 0;
                for (auto& r : batch) {
                    for (uint64_t g = 0; g < G; ++g)
                        BST_CK(cudaMemcpyAsync(r.out + g * r.n, s.d_out.p + g * rows + off, sizeof(float) * r.n,
                                               cudaMemcpyDefault, s.st));
                    off += r.n;
                }
                BST_CK(cudaEventRecord(s.done, s.st));
            } catch (const Error& e) {
                std::lock_guard<std::mutex> lk(mu);
                fail_all(e.code, e.msg);
                s.busy = false;
                continue;
            }
            {
                std::lock_guard<std::mutex> lk(mu);
                inflight.push_back(si);
            }
            cv_inflight.notify_one();
        }
    }

    void complete_loop() {
        cudaSetDevice(device);
        for (;;) {
            int si;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv_inflight.wait(lk, [&] { return !inflight.empty() || stop; });
                if (inflight.empty()) return;  // stop with nothing in flight
                si = inflight.front();
            }
            Slot& s = slots[si];
            const cudaError_t e = cudaEventSynchronize(s.done);
            std::lock_guard<std::mutex> lk(mu);
            inflight.pop_front();
            const uint64_t t = now_ns();
            if (e != cudaSuccess) {
                cudaGetLastError();
                fail_all(BST_ERR_CUDA, std::string("batch failed: ") + cudaGetErrorString(e));
            } else {
                float k_ms = 0.0f, d_ms = 0.0f;
                if (cudaEventElapsedTime(&k_ms, s.k0, s.k1) != cudaSuccess ||
                    cudaEventElapsedTime(&d_ms, s.k1, s.done) != cudaSuccess) {
                    cudaGetLastError();
                    k_ms = d_ms = 0.0f;
                }
                for (uint64_t id : s.reqs) {
                    auto it = reqs.find(id);
                    if (it == reqs.end()) continue;
                    Req& r = it->second;
                    r.status = BST_OK;
                    r.done_ns = t;
                    float c_ms = 0.0f;
                    if (r.copy_start && r.copied && cudaEventElapsedTime(&c_ms, r.copy_start, r.copied) != cudaSuccess) {
                        cudaGetLastError();
                        c_ms = 0.0f;
                    }
                    const uint64_t copy_ns = (uint64_t)((double)c_ms * 1e6);
                    stats.h2d_bytes += r.n * F * sizeof(float);
                    stats.h2d_ns += copy_ns;
                    if (trace.size() < TRACE_MAX) {
                        bst_server_phase ph;
                        ph.rows = r.n;
                        ph.batch_rows = s.rows;
                        ph.queue_ns = r.admit_ns - r.submit_ns;
                        ph.copy_ns = copy_ns;
                        ph.to_dispatch_ns = r.dispatch_ns - r.admit_ns;
                        ph.kernel_ns = (uint64_t)((double)k_ms * 1e6);
                        ph.d2h_ns = (uint64_t)((double)d_ms * 1e6);
                        ph.dispatch_to_done_ns = t - r.dispatch_ns;
                        trace.push_back(ph);
                    }
                    for (cudaEvent_t* e : {&r.copy_start, &r.copied})
                        if (*e) {
                            events.push_back(*e);
                            *e = nullptr;
                        }
                    if (!live.empty()) live.pop_front();  // batches retire in admission order
                }
                stats.completed += s.reqs.size();
                try {
                    admit_locked();
                } catch (const Error& err) {
                    fail_all(err.code, err.msg);
                }
            }
            s.busy = false;
            cv_done.notify_all();
            cv_work.notify_one();
        }
    }
};

// Load replay: requests submitted from this thread at scheduled steady-clock
// times, completions collected by a second thread, latency counted from the
// scheduled arrival (a late submission counts against the server).
void server_replay(Server& s, const float* pool, uint64_t pool_rows, uint64_t n_req, const uint64_t* arrival_ns,
                   const uint64_t* row_off, const uint64_t* n_rows, float* out, uint64_t ring, uint64_t ring_stride,
                   uint64_t* latency_ns, uint64_t* span_ns) {
    if (ring == 0) throw Error{BST_ERR_INVALID_ARGUMENT, "replay ring must hold at least one request"};
    for (uint64_t i = 0; i < n_req; ++i) {
        if (row_off[i] > pool_rows || n_rows[i] > pool_rows - row_off[i])
            throw Error{BST_ERR_INVALID_ARGUMENT, "replay request " + std::to_string(i) + " outside the row pool"};
        if (n_rows[i] * s.G > ring_stride)
            throw Error{BST_ERR_INVALID_ARGUMENT, "replay ring slot smaller than a request's output"};
        if (i && arrival_ns[i] < arrival_ns[i - 1])
            throw Error{BST_ERR_INVALID_ARGUMENT, "replay arrivals must be non-decreasing"};
    }
    std::vector<uint64_t> ticket(n_req, 0);
    std::mutex mu;
    std::condition_variable cv;
    uint64_t published = 0, completed = 0, last_done = 0;
    bool submit_done = false, wait_failed = false;
    int err = BST_OK;
    std::string err_msg;
    const uint64_t start = now_ns() + 1000000ull;  // 1 ms lead
    // the waiter retires every published ticket in order (the server holds
    // the caller's ring slots until then)
    std::thread waiter([&] {
        for (uint64_t i = 0;; ++i) {
            uint64_t id;
            {
                std::unique_lock<std::mutex> lk(mu);
                cv.wait(lk, [&] { return published > i || submit_done; });
                if (published <= i) return;
                id = ticket[i];
            }
            uint64_t sub = 0, done = 0;
            std::string msg;
            const int st = server_wait(s, id, -1, &sub, &done, &msg);
            std::lock_guard<std::mutex> lk(mu);
            if (st != BST_OK && !wait_failed) {
                wait_failed = true;
                err = st;
                err_msg = msg;
            }
            const uint64_t due = start + arrival_ns[i];
            latency_ns[i] = done > due ? done - due : 0;
            last_done = std::max(last_done, done);
            completed = i + 1;
            cv.notify_all();
        }
    });
    for (uint64_t i = 0; i < n_req; ++i) {
        const uint64_t due = start + arrival_ns[i];
        const uint64_t now = now_ns();
        if (due > now + 200000ull)  // sleep to 200 us before, then spin
            std::this_thread::sleep_for(std::chrono::nanoseconds(due - now - 200000ull));
        while (now_ns() < due) {
        }
        {
            std::unique_lock<std::mutex> lk(mu);
            cv.wait(lk, [&] { return wait_failed || i < ring || completed > i - ring; });  // output slot free
            if (wait_failed) break;
        }
        uint64_t id = 0;
        try {
            id = server_submit(s, pool + row_off[i] * s.F, n_rows[i], out + (i % ring) * ring_stride);
        } catch (const Error& e) {
            std::lock_guard<std::mutex> lk(mu);
            if (err == BST_OK) {
                err = e.code;
                err_msg = e.msg;
            }
            break;
        }
        std::lock_guard<std::mutex> lk(mu);
        ticket[i] = id;
        published = i + 1;
        cv.notify_all();
    }
    {
        std::lock_guard<std::mutex> lk(mu);
        submit_done = true;
        cv.notify_all();
    }
    waiter.join();
    if (err != BST_OK) throw Error{(bst_status)err, err_msg};
    const uint64_t first = start + (n_req ? arrival_ns[0] : 0);
    if (span_ns) *span_ns = last_done > first ? last_done - first : 0;
}

Server* server_create(const Model& m, uint64_t mem_budget_bytes, uint64_t max_batch_rows, bool raw) {
    return new Server(m, mem_budget_bytes, max_batch_rows, raw);
}
void server_destroy(Server* s) { delete s; }
uint64_t server_submit(Server& s, const float* rows, uint64_t n, float* out) { return s.submit(rows, n, out); }
int server_wait(Server& s, uint64_t id, int64_t timeout_ms, uint64_t* submit_ns, uint64_t* done_ns,
                std::string* err) {
    const int st = s.wait(id, timeout_ms, submit_ns, done_ns);
    if (st != BST_OK && err) {
        std::lock_guard<std::mutex> lk(s.mu);
        *err = st == BST_ERR_TIMEOUT ? std::string("request not finished within the timeout") : s.error_msg;
    }
    return st;
}
void server_stats(Server& s, bst_server_stats* out) {
    std::lock_guard<std::mutex> lk(s.mu);
    *out = s.stats;
}
uint64_t server_trace(Server& s, bst_server_phase* out, uint64_t max) {
    std::lock_guard<std::mutex> lk(s.mu);
    const uint64_t n = std::min<uint64_t>(max, s.trace.size());
    if (n && out) std::memcpy(out, s.trace.data(), n * sizeof(bst_server_phase));
    s.trace.erase(s.trace.begin(), s.trace.begin() + (ptrdiff_t)n);
    return n;
}

}  // namespace bst
