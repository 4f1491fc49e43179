// engine.h — training and prediction orchestration of the B200 GBDT engine.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

#include <memory>
#include <mutex>
#include <string>
#include <vector>

#include "../../include/boosters_c.h"
#include "binning.h"
#include "kernels.h"

namespace bst {

struct Error {
    bst_status code;
    std::string msg;
};

void cuda_check(cudaError_t e, const char* what);
#define BST_CK(x) ::bst::cuda_check((x), #x)

// Device-memory cap of the library's own buffers: the environment variable
// BST_DEVICE_MEMORY_LIMIT (bytes, read once; unset or 0 = no cap) bounds
// the bytes all live DevArrays hold together, process-wide. An allocation
// that would pass it fails like an exhausted device (BST_ERR_OUT_OF_MEMORY)
// without calling cudaMalloc: for sharing a GPU with other allocators, and
// for exercising the out-of-memory paths without exhausting a device.
void dev_bytes_reserve(size_t bytes);  // throws Error{BST_ERR_OUT_OF_MEMORY}
void dev_bytes_release(size_t bytes);

// Device block cache: a released buffer is kept (per device, up to
// BST_DEVICE_CACHE_BYTES, default 8 GiB) and handed to a later request of
// at most its size and at least half of it, so that consecutive training
// calls, which allocate the same buffers, skip cudaMalloc / cudaFree
// (which maps and unmaps pages). A release waits for the device to be idle
// first, as cudaFree does, so no kernel still in flight can see its buffer
// reused. The cap above counts cached blocks; an allocation that would
// pass it, or that the device refuses, first frees every cached block.
// dev_alloc returns the block and its size (the request rounded up).
void* dev_alloc(size_t bytes, size_t* block_bytes);  // throws Error
void dev_free(void* p, size_t block_bytes);
void dev_cache_trim();  // frees every cached block
// Pinned host memory from a process-wide cache of blocks (pinned_free waits
// for the device to be idle, as cudaFreeHost does, then keeps the block).
void* pinned_alloc(size_t bytes);
void pinned_free(void* p);
void pinned_cache_trim();  // frees every cached pinned block

template <class T>
struct DevArray {
    T* p = nullptr;
    size_t n = 0;
    size_t block = 0;  // bytes of the underlying block
    DevArray() = default;
    DevArray(const DevArray&) = delete;
    DevArray& operator=(const DevArray&) = delete;
    ~DevArray() { release(); }
    void release() {
        if (p) dev_free(p, block);
        p = nullptr;
        n = 0;
        block = 0;
    }
    void alloc(size_t k) {
        if (k <= n && p) return;
        release();
        if (k == 0) return;
        p = static_cast<T*>(dev_alloc(k * sizeof(T), &block));
        n = k;
    }
};

// Host copy of a feature-major dataset (data/raw/dataset.rs:139).
struct HostDataset {
    uint64_t n = 0, F = 0;
    std::vector<float> x;  // [F][n] (owned copy), or
    const float* xv = nullptr;  // the caller's [F][n] array (a view)
    const float* xdata() const { return xv ? xv : x.data(); }
    std::vector<float> y;  // [n_outputs][n]
    uint32_t n_outputs = 0;
    std::vector<float> w;
    bool has_w = false;
    std::vector<uint8_t> user_cat;  // per feature
};

// Binned dataset resident on the GPU.
struct DeviceBinned {
    BinPlan plan;
    DevArray<uint8_t> rec;        // [n][plan.rec] row records
    uint8_t* bins8 = nullptr;     // u8 view: rec
    uint16_t* bins16 = nullptr;   // u16 view: rec + plan.u16_off (null without u16 columns)
    double binning_ms = 0.0;
};

// Host tree (repr/gbdt/tree.rs:32-47) plus training detail.
struct HostTree {
    std::vector<uint32_t> split_index, left, right, seg_start, seg_size, cat_words, split_bin;
    std::vector<float> threshold, leaf, gain, cover;
    std::vector<uint8_t> default_left, is_leaf, split_type;
    std::vector<double> grad_sum, hess_sum;
    std::vector<uint32_t> row_leaf;
    uint32_t group = 0;
    uint32_t alloc();
};

struct DeviceForest {
    DevArray<ForestNode> nodes;
    DevArray<uint32_t> roots, group_trees, group_off, cat_seg, cat_words;
    DevArray<float> base;
    ForestDev view{};
    // heap-ordered copy for the shared-memory traversal (trees of leaf depth
    // <= HEAP_DEPTH, features < 65536, rows binned against the forest's own
    // thresholds)
    bool heap_ok = false;
    uint32_t heap_min_F = 0;  // rows need at least this many features
    DevArray<uint2> heap_cat;
    DevArray<uint32_t> heap_nodes, heap_goff, heap_words, heap_thr_off;
    DevArray<float> heap_thr, heap_spl;
    DevArray<int32_t> heap_fcol;
    DevArray<uint8_t> heap_finfo;
    HeapForest heap{};
};
// out [n_groups][n] raw margins of sample-major rows x [n][F] (device). The
// shared-memory traversal bins the rows into scratch first: the caller's
// (scratch_bytes >= what n rows need) or stream-ordered pool memory.
void forest_predict_rows(const DeviceForest& f, const float* x, uint64_t n, uint64_t F, float* out, cudaStream_t st,
                         void* scratch = nullptr, size_t scratch_bytes = 0);
bool forest_uses_heap(const DeviceForest& f, uint64_t n, uint64_t F);
// Node-list forest of `trees` (forest order; no heap copy) into f.
void upload_node_forest(const std::vector<const HostTree*>& trees, uint32_t n_groups, const std::vector<float>& base,
                        DeviceForest& f);
// Scratch bytes enough for any batch of up to n_max rows; bin bytes per row.
size_t forest_scratch_max(const DeviceForest& f, uint64_t n_max, uint64_t F);
size_t forest_bin_bytes_per_row(const DeviceForest& f, uint64_t F);

struct Counters {
    uint64_t launches = 0;
    uint64_t hist_launches = 0, hist_rows = 0, hist_bytes = 0;
    uint64_t scan_launches = 0, partition_rows = 0;
    double hist_ms = 0;
};

struct Model {
    uint32_t n_groups = 1, n_features = 0;
    int objective = 0;
    std::vector<float> base;
    std::vector<HostTree> trees;
    std::vector<float> train_pred;
    double timings[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    Counters counters;
    // early stopping: boosting rounds run, and the round count kept (the
    // best round + 1; 0 when early stopping was off or never improved)
    uint32_t rounds_run = 0, rounds_kept = 0;
    int device = 0;
    // launch shape of the batched pipeline and how it was chosen (autotune.h)
    std::string tune_info;
    mutable std::mutex mu;
    mutable std::unique_ptr<DeviceForest> dev;
    const DeviceForest& device_forest() const;
    void build_heap_forest(DeviceForest& f) const;
};

// Incremental training on a GPU-resident binned dataset: the boosting loop of
// GBDTTrainer::train (training/gbdt/trainer.rs:242-401), a batch of rounds
// per update().
class Booster {
  public:
    Booster(const HostDataset& ds, const bst_config& cfg, uint32_t n_threads);
    ~Booster();
    void update(uint32_t rounds);
    uint32_t rounds_done() const;
    const Model& model() const;
    std::unique_ptr<Model> snapshot() const;

  private:
    struct Impl;
    std::unique_ptr<Impl> impl_;
};

void make_binned(const HostDataset& ds, const bst_config& cfg, cudaStream_t st, DeviceBinned& out);
// val (or null): the validation set of early stopping (trainer.rs:344-390).
std::unique_ptr<Model> train_model(const HostDataset& ds, const bst_config& cfg, uint32_t n_threads,
                                   const HostDataset* val = nullptr);
std::unique_ptr<Model> grow_one_tree(const HostDataset& ds, const float* grad, const float* hess,
                                     const bst_config& cfg, uint32_t n_threads);
void predict_host(const Model& m, const HostDataset& ds, bool raw, float* out);
void predict_device(const Model& m, const float* x_dev_sm, uint64_t n, uint64_t F, bool raw,
                    float* out_dev, cudaStream_t st);
int transform_of(int objective);
// Metric value of [G][n] predictions (probabilities for the log losses).
// Parameters of the quantile and Huber metrics.
struct MetricParams {
    const float* alpha = nullptr;
    uint32_t n_alpha = 0;
    float delta = 1.0f;
};
inline MetricParams metric_params(const bst_config& c) {
    MetricParams m;
    m.alpha = c.quantile_alpha;
    m.n_alpha = c.n_quantiles;
    m.delta = c.huber_delta;
    return m;
}
double metric_value(int metric, const float* p, uint32_t G, uint64_t n, const float* y, const float* w,
                    const MetricParams& mp = MetricParams());
int resolve_metric(int metric, int objective);
// Outputs (trees per round) of an objective: classes, quantiles, or one.
uint32_t n_outputs_of(const bst_config& c);
float quantile_alpha_of(const bst_config& c, uint32_t o);
// Model files (persist.cpp): .bstr.json text and .bstr bytes (uncompressed
// MessagePack); model_from_bytes reads either (binary by its magic).
std::string model_to_json(const Model& m, bool pretty);
std::vector<uint8_t> model_to_bstr(const Model& m, int compression_level);
std::unique_ptr<Model> model_from_bytes(const uint8_t* data, size_t len);
uint32_t crc32c_bytes(const uint8_t* p, size_t n);

// Continuous-batching prediction server (server.cpp). The model must outlive
// the server.
struct Server;
Server* server_create(const Model& m, uint64_t mem_budget_bytes, uint64_t max_batch_rows, bool raw);
void server_destroy(Server* s);
uint64_t server_submit(Server& s, const float* rows, uint64_t n, float* out);
int server_wait(Server& s, uint64_t id, int64_t timeout_ms, uint64_t* submit_ns, uint64_t* done_ns,
                std::string* err);
void server_stats(Server& s, bst_server_stats* out);
// Moves up to `max` phase records of completed requests (oldest first) out
// of the server's trace; returns how many.
uint64_t server_trace(Server& s, bst_server_phase* out, uint64_t max);
void server_replay(Server& s, const float* pool, uint64_t pool_rows, uint64_t n_req, const uint64_t* arrival_ns,
                   const uint64_t* row_off, const uint64_t* n_rows, float* out, uint64_t ring, uint64_t ring_stride,
                   uint64_t* latency_ns, uint64_t* span_ns);
void build_hist_tiles(const BinPlan& p, std::vector<HistTile>& tiles, uint32_t& max_smem,
                      const std::vector<uint8_t>* only = nullptr);
void build_lane_tiles(const BinPlan& p, uint32_t max_bins, std::vector<LaneTile>& tiles, uint32_t& tile_bins,
                      std::vector<uint8_t>& rest);

}  // namespace bst
