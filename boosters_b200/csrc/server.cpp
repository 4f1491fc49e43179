// server.cpp — continuous-batching prediction server over a device-resident
// forest (the serving pattern of the engine; the reference predicts one call
// at a time through Predictor::predict_into, inference/gbdt/predictor.rs:197).
//
// Requests (sample-major f32 rows, caller-owned input and output buffers)
// queue FIFO. A dispatcher thread coalesces the queue head into a batch that
// fits one of SLOTS in-flight slots (device input / output buffers sized by
// the memory budget), copies each request's rows straight from the caller's
// buffer into the slot's device input, runs ONE traversal launch over the
// whole batch and copies each request's outputs straight back, all on the
// slot's stream. While batch k runs, batch k + 1 forms from requests that
// arrived meanwhile and is issued on the next slot's stream, so copies and
// traversals of consecutive batches overlap on the device. A completion
// thread retires slots in order and wakes the waiters. A row's prediction
// depends on that row alone (trees summed in forest order per row), so every
// result is identical whatever batch it shares.
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

    struct Req {
        uint64_t id = 0;
        const float* rows = nullptr;
        uint64_t n = 0;
        float* out = nullptr;
        uint64_t submit_ns = 0, done_ns = 0;
        int status = -1;  // -1 pending, else bst_status
    };
    struct Slot {
        DevArray<float> d_in, d_out;
        cudaStream_t st = nullptr;
        cudaEvent_t done = nullptr;
        std::vector<uint64_t> reqs;  // ticket ids
        bool busy = false;
    };

    const Model& m;
    uint64_t F = 0, G = 1, max_rows = 0;
    bool raw = false;
    int device = 0;

    std::mutex mu;
    std::condition_variable cv_submit, cv_slot, cv_done, cv_inflight;
    std::deque<uint64_t> queue;
    std::unordered_map<uint64_t, Req> reqs;
    std::deque<int> inflight;  // slot indices in issue order
    Slot slots[SLOTS];
    uint64_t next_id = 1;
    bool stop = false;
    int error = BST_OK;
    std::string error_msg;
    bst_server_stats stats{};
    std::thread dispatcher, completer;

    Server(const Model& model, uint64_t budget, uint64_t cap, bool raw_out) : m(model), raw(raw_out) {
        device = m.device;
        BST_CK(cudaSetDevice(device));
        F = m.n_features;
        G = m.n_groups;
        const uint64_t per_row = (F + G) * sizeof(float);
        max_rows = budget / ((uint64_t)SLOTS * std::max<uint64_t>(1, per_row));
        if (cap) max_rows = std::min(max_rows, cap);
        if (max_rows == 0)
            throw Error{BST_ERR_INVALID_ARGUMENT, "memory budget below one row per in-flight slot"};
        if (max_rows > 0xFFFFFFFFull) max_rows = 0xFFFFFFFFull;
        (void)m.device_forest();  // forest resident before the first request
        for (auto& s : slots) {
            s.d_in.alloc((size_t)max_rows * std::max<uint64_t>(1, F));
            s.d_out.alloc((size_t)max_rows * G);
            BST_CK(cudaStreamCreateWithFlags(&s.st, cudaStreamNonBlocking));
            BST_CK(cudaEventCreateWithFlags(&s.done, cudaEventDisableTiming));
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
                if (!queue.empty() || !inflight.empty()) return false;
                for (auto& s : slots)
                    if (s.busy) return false;
                return true;
            });
            stop = true;
        }
        cv_submit.notify_all();
        cv_slot.notify_all();
        cv_inflight.notify_all();
        if (dispatcher.joinable()) dispatcher.join();
        if (completer.joinable()) completer.join();
        cudaSetDevice(device);
        for (auto& s : slots) {
            if (s.st) cudaStreamSynchronize(s.st);
            if (s.done) cudaEventDestroy(s.done);
            if (s.st) cudaStreamDestroy(s.st);
        }
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
        reqs.emplace(r.id, r);
        queue.push_back(r.id);
        stats.submitted += 1;
        cv_submit.notify_one();
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
        if (submit_ns) *submit_ns = r.submit_ns;
        if (done_ns) *done_ns = r.done_ns;
        return r.status;
    }

    void fail_all(int code, const std::string& msg) {  // caller holds mu
        if (error == BST_OK) {
            error = code;
            error_msg = msg;
        }
        const uint64_t t = now_ns();
        for (auto& kv : reqs)
            if (kv.second.status < 0) {
                kv.second.status = code;
                kv.second.done_ns = t;
            }
        queue.clear();
        cv_done.notify_all();
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
                cv_submit.wait(lk, [&] { return stop || !queue.empty(); });
                if (stop) return;
                cv_slot.wait(lk, [&] {
                    if (stop) return true;
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
                // admission: the queue head while the batch fits the slot
                while (!queue.empty()) {
                    const Req& r = reqs[queue.front()];
                    if (rows + r.n > max_rows) break;
                    batch.push_back(r);
                    rows += r.n;
                    queue.pop_front();
                }
                Slot& s = slots[si];
                s.busy = true;
                s.reqs.clear();
                for (auto& r : batch) s.reqs.push_back(r.id);
                stats.batches += 1;
                stats.rows += rows;
                stats.max_rows_seen = std::max<uint64_t>(stats.max_rows_seen, rows);
            }
            Slot& s = slots[si];
            try {
                uint64_t off = 0;
                for (auto& r : batch) {
                    if (r.n && F)
                        BST_CK(cudaMemcpyAsync(s.d_in.p + off * F, r.rows, sizeof(float) * r.n * F,
                                               cudaMemcpyHostToDevice, s.st));
                    off += r.n;
                }
                forest_predict_rows(f, s.d_in.p, rows, F, s.d_out.p, s.st);
                if (!raw) launch_transform(tr, s.d_out.p, (uint32_t)G, rows, s.st);
                BST_CK(cudaGetLastError());
                off = 0;
                for (auto& r : batch) {
                    for (uint64_t g = 0; g < G && r.n; ++g)
                        BST_CK(cudaMemcpyAsync(r.out + g * r.n, s.d_out.p + g * rows + off, sizeof(float) * r.n,
                                               cudaMemcpyDeviceToHost, s.st));
                    off += r.n;
                }
                BST_CK(cudaEventRecord(s.done, s.st));
            } catch (const Error& e) {
                std::lock_guard<std::mutex> lk(mu);
                fail_all(e.code, e.msg);
                s.busy = false;
                cv_slot.notify_one();
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
                for (uint64_t id : s.reqs) {
                    auto it = reqs.find(id);
                    if (it == reqs.end()) continue;
                    it->second.status = BST_OK;
                    it->second.done_ns = t;
                }
                stats.completed += s.reqs.size();
            }
            s.busy = false;
            cv_done.notify_all();
            cv_slot.notify_one();
        }
    }
};

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

}  // namespace bst
