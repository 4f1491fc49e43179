// autotune.h — launch shapes of the batched tree pipeline, chosen by timing
// candidates on the first trees of a training run and kept in a cache file.
//
// A shape never changes a result: histogram sums are exact integers and the
// partition is deterministic per node, so every candidate grows the same
// trees; only their speed differs. The tuner therefore explores on the
// caller's own first trees (no extra work), interleaving candidates, and
// keeps the one with the lowest median tree time.
#pragma once
#include <cstdint>
#include <string>
#include <vector>

namespace bst {

struct TuneShape {
    uint32_t items = 2;  // (row segment, lane tile) histogram items per resident block
    uint32_t hist = 0;   // histogram kernel variant (launch_b_hist_part)
    uint32_t grid = 8;   // blocks per SM of the level kernels (partition, merge, scan, sums)
    std::string str() const;
    static bool parse(const std::string& s, TuneShape& out);
    bool operator==(const TuneShape& o) const { return items == o.items && hist == o.hist && grid == o.grid; }
};

// "name|sm_count|cc" of a CUDA device: choices are per device model.
std::string device_signature(int device);

// The cache file holds one "key<TAB>shape" line per tuned workload class.
// lookup: false when the file, the key or a parsable shape is missing.
bool tune_cache_lookup(const std::string& path, const std::string& key, TuneShape& out);
// Adds or replaces the key's line (rewrites the file through a temporary
// file and a rename, under a process-wide lock). Failures to write are
// ignored: the cache only saves exploration time.
void tune_cache_store(const std::string& path, const std::string& key, const TuneShape& s);

// Online exploration over candidate shapes: trees are assigned candidates
// round-robin after the first `skip` trees (cold caches and lazily loaded
// code: not timed); after `rounds` timed trees per candidate the candidate
// with the lowest median time wins.
class TuneExplorer {
  public:
    TuneExplorer() = default;
    TuneExplorer(std::vector<TuneShape> cands, uint32_t rounds, uint32_t skip);
    bool active() const { return !cands_.empty() && !done_; }
    bool done() const { return done_; }
    // candidate index of the next tree; *timed: whether its time counts
    uint32_t next(bool* timed);
    // time of a timed tree grown with candidate c (ms); the record that
    // completes every candidate's rounds finishes the exploration, and later
    // records are ignored
    void record(uint32_t c, float ms);
    const TuneShape& best() const { return cands_[best_]; }
    // per candidate: median ms of its timed trees (NaN before any)
    std::vector<double> medians() const;

  private:
    std::vector<TuneShape> cands_;
    std::vector<std::vector<float>> times_;
    uint32_t rounds_ = 2, skip_ = 1, issued_ = 0, best_ = 0;
    bool done_ = false;
};

}  // namespace bst
