// engine.cpp — GBDT training and prediction on one B200.
//
// The tree-growth control flow follows boosters' TreeGrower
// (training/gbdt/grower.rs:265-514) and growth policies
// (training/gbdt/expansion.rs:87-320); every data-parallel step runs as a
// kernel from kernels.cu on device-resident data. The host keeps only the
// tree under construction (a few hundred nodes) and reads back, per level,
// the partition counts and the chosen splits.
#include "engine.h"
#include "nvtx_range.h"

#include "autotune.h"

#include <algorithm>
#include <array>
#include <atomic>
#include <chrono>
#include <cmath>
#include <cstdlib>
#include <cstring>
#include <functional>
#include <limits>
#include <map>
#include <mutex>
#include <thread>
#include <unordered_map>

namespace bst {

void cuda_check(cudaError_t e, const char* what) {
    if (e != cudaSuccess) {
        cudaGetLastError();
        throw Error{e == cudaErrorMemoryAllocation ? BST_ERR_OUT_OF_MEMORY : BST_ERR_CUDA,
                    std::string(what) + ": " + cudaGetErrorString(e)};
    }
}

namespace {
std::atomic<uint64_t> g_dev_bytes{0};

uint64_t dev_memory_limit() {
    static const uint64_t limit = [] {
        const char* v = std::getenv("BST_DEVICE_MEMORY_LIMIT");
        return v ? std::strtoull(v, nullptr, 10) : 0ull;
    }();
    return limit;
}
}  // namespace

void dev_bytes_reserve(size_t bytes) {
    const uint64_t limit = dev_memory_limit();
    const uint64_t now = g_dev_bytes.fetch_add(bytes) + bytes;
    if (limit && now > limit) {
        g_dev_bytes.fetch_sub(bytes);
        throw Error{BST_ERR_OUT_OF_MEMORY, "device allocation of " + std::to_string(bytes) +
                                               " bytes would pass BST_DEVICE_MEMORY_LIMIT=" + std::to_string(limit) +
                                               " (" + std::to_string(now - bytes) + " bytes in use)"};
    }
}

void dev_bytes_release(size_t bytes) { g_dev_bytes.fetch_sub(bytes); }

namespace {

struct DevCache {
    std::mutex mu;
    std::multimap<size_t, std::pair<int, void*>> blocks;  // size -> (device, pointer)
    size_t bytes = 0;
};
DevCache& dev_cache() {
    static DevCache* c = new DevCache();  // never destroyed: no cudaFree after the runtime unloads
    return *c;
}

size_t dev_cache_max() {
    static const size_t m = [] {
        const char* v = std::getenv("BST_DEVICE_CACHE_BYTES");
        return v ? (size_t)std::strtoull(v, nullptr, 10) : (size_t)8 << 30;
    }();
    return m;
}

// 256 B .. 1 MiB: the next power of two; above: a multiple of 2 MiB
size_t dev_round(size_t b) {
    if (b <= ((size_t)1 << 20)) {
        size_t r = 256;
        while (r < b) r <<= 1;
        return r;
    }
    const size_t g = (size_t)2 << 20;
    return (b + g - 1) / g * g;
}

}  // namespace

// Pinned host blocks, kept for reuse like the device blocks: a training
// call's staging area and read-back slots would otherwise cost a
// cudaMallocHost and a (device-synchronising) cudaFreeHost each.
namespace {
struct PinnedCache {
    std::mutex mu;
    std::multimap<size_t, void*> blocks;     // free: size -> pointer
    std::unordered_map<void*, size_t> live;  // handed out: pointer -> size
    size_t bytes = 0;                        // free bytes
};
PinnedCache& pinned_cache() {
    static PinnedCache* c = new PinnedCache();  // never destroyed (see dev_cache)
    return *c;
}
constexpr size_t PINNED_CACHE_MAX = (size_t)256 << 20;
}  // namespace

void* pinned_alloc(size_t bytes) {
    const size_t r = dev_round(bytes);
    PinnedCache& c = pinned_cache();
    {
        std::lock_guard<std::mutex> lk(c.mu);
        auto it = c.blocks.lower_bound(r);
        if (it != c.blocks.end() && it->first <= 2 * r) {
            void* p = it->second;
            c.live[p] = it->first;
            c.bytes -= it->first;
            c.blocks.erase(it);
            return p;
        }
    }
    void* p = nullptr;
    BST_CK(cudaMallocHost(&p, r));
    std::lock_guard<std::mutex> lk(c.mu);
    c.live[p] = r;
    return p;
}

void pinned_free(void* p) {
    if (!p) return;
    cudaDeviceSynchronize();  // no copy into or out of the block is pending (cudaFreeHost would wait too)
    cudaGetLastError();
    PinnedCache& c = pinned_cache();
    {
        std::lock_guard<std::mutex> lk(c.mu);
        auto it = c.live.find(p);
        const size_t sz = it == c.live.end() ? 0 : it->second;
        if (it != c.live.end()) c.live.erase(it);
        if (sz && c.bytes + sz <= PINNED_CACHE_MAX) {
            c.blocks.emplace(sz, p);
            c.bytes += sz;
            return;
        }
    }
    cudaFreeHost(p);
    cudaGetLastError();
}

void pinned_cache_trim() {
    PinnedCache& c = pinned_cache();
    std::lock_guard<std::mutex> lk(c.mu);
    for (auto& e : c.blocks) cudaFreeHost(e.second);
    cudaGetLastError();
    c.blocks.clear();
    c.bytes = 0;
}

void dev_cache_trim() {
    DevCache& c = dev_cache();
    std::lock_guard<std::mutex> lk(c.mu);
    for (auto& e : c.blocks) {
        cudaFree(e.second.second);
        dev_bytes_release(e.first);
    }
    cudaGetLastError();
    c.blocks.clear();
    c.bytes = 0;
}

void* dev_alloc(size_t bytes, size_t* block_bytes) {
    const size_t r = dev_round(bytes);
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) cudaGetLastError();
    DevCache& c = dev_cache();
    {
        std::lock_guard<std::mutex> lk(c.mu);
        for (auto it = c.blocks.lower_bound(r); it != c.blocks.end() && it->first <= 2 * r; ++it)
            if (it->second.first == dev) {
                void* p = it->second.second;
                *block_bytes = it->first;
                c.bytes -= it->first;
                c.blocks.erase(it);
                return p;
            }
    }
    try {
        dev_bytes_reserve(r);
    } catch (const Error&) {
        dev_cache_trim();
        dev_bytes_reserve(r);  // throws again if the live buffers alone pass the cap
    }
    void* p = nullptr;
    cudaError_t e = cudaMalloc(&p, r);
    if (e != cudaSuccess) {
        cudaGetLastError();
        dev_cache_trim();
        e = cudaMalloc(&p, r);
    }
    if (e != cudaSuccess) {
        cudaGetLastError();
        dev_bytes_release(r);
        throw Error{e == cudaErrorMemoryAllocation ? BST_ERR_OUT_OF_MEMORY : BST_ERR_CUDA,
                    std::string("cudaMalloc of ") + std::to_string(r) + " bytes failed: " + cudaGetErrorString(e)};
    }
    *block_bytes = r;
    return p;
}

void dev_free(void* p, size_t block_bytes) {
    if (!p) return;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) cudaGetLastError();
    cudaPointerAttributes a{};
    if (cudaPointerGetAttributes(&a, p) == cudaSuccess && a.type == cudaMemoryTypeDevice) dev = a.device;
    cudaGetLastError();
    int cur = dev;
    cudaGetDevice(&cur);
    if (cur != dev) cudaSetDevice(dev);
    const cudaError_t se = cudaDeviceSynchronize();  // what cudaFree would wait for
    if (cur != dev) cudaSetDevice(cur);
    DevCache& c = dev_cache();
    {
        std::lock_guard<std::mutex> lk(c.mu);
        if (se == cudaSuccess && c.bytes + block_bytes <= dev_cache_max()) {
            c.blocks.emplace(block_bytes, std::make_pair(dev, p));
            c.bytes += block_bytes;
            return;
        }
    }
    cudaGetLastError();
    cudaFree(p);
    cudaGetLastError();
    dev_bytes_release(block_bytes);
}

// Column tiles of the histogram kernel: lanes of one 16-byte row vector
// whose bins fit one shared-memory histogram (<= 4096 bins = 64 KiB).
// only: if given, the columns to cover (others are skipped).
void build_hist_tiles(const BinPlan& p, std::vector<HistTile>& tiles, uint32_t& max_smem,
                      const std::vector<uint8_t>* only) {
    const uint32_t kMaxSmemBins = 4096;
    tiles.clear();
    const uint32_t nc = p.n_cols();
    std::vector<int> col_of8(p.s8, -1), col_of16(p.s16, -1);
    for (uint32_t c = 0; c < nc; ++c) {
        if (only && !(*only)[c]) continue;
        if (p.col_matrix[c] == 0)
            col_of8[p.col_pos[c]] = (int)c;
        else
            col_of16[p.col_pos[c]] = (int)c;
    }
    auto emit = [&](uint32_t matrix, uint32_t lanes, const std::vector<int>& col_of, uint32_t nvec) {
        for (uint32_t v = 0; v < nvec; ++v) {
            HistTile t;
            std::memset(&t, 0, sizeof(t));
            t.matrix = matrix;
            t.vec = v;
            bool open = false;
            for (uint32_t l = 0; l < lanes; ++l) {
                const int c = col_of[v * lanes + l];
                if (c < 0) continue;
                const uint32_t nb = p.col_nbins[c];
                if (open && t.smem_bins + nb > kMaxSmemBins) {
                    tiles.push_back(t);
                    std::memset(&t, 0, sizeof(t));
                    t.matrix = matrix;
                    t.vec = v;
                    open = false;
                }
                if (!open) {
                    t.c0 = l;
                    open = true;
                }
                t.lane_smem[l] = t.smem_bins;
                t.lane_hist[l] = p.col_hist_off[c];
                t.lane_nbins[l] = nb;
                t.smem_bins += nb;
                t.c1 = l + 1;
            }
            if (open) tiles.push_back(t);
        }
    };
    emit(0, 16, col_of8, p.s8 / 16);
    emit(1, 8, col_of16, p.s16 / 8);
    max_smem = 0;
    for (auto& t : tiles) max_smem = std::max(max_smem, t.smem_bins);
}

// Column-lane tiles: windows of each view of the row record, cut at the
// record's 32-byte sector boundaries (32 bytes, or 16 where a view starts or
// ends inside a sector), so that each window read touches one sector. A
// window holding a column with more than max_bins bins is left to the
// HistTile kernel: its columns are marked in `rest`.
void build_lane_tiles(const BinPlan& p, uint32_t max_bins, std::vector<LaneTile>& tiles, uint32_t& tile_bins,
                      std::vector<uint8_t>& rest) {
    tiles.clear();
    tile_bins = 0;
    const uint32_t nc = p.n_cols();
    rest.assign(nc, 0);
    for (uint32_t m = 0; m < 2; ++m) {
        const uint32_t esize = m == 0 ? 1u : 2u;
        const uint32_t view = m == 0 ? 0u : p.u16_off;  // the view's offset in the record (a multiple of 16)
        const uint32_t row_bytes = ((m == 0 ? p.f8 : p.f16) * esize + 15) / 16 * 16;
        std::vector<int> col_at(row_bytes / esize, -1);
        for (uint32_t c = 0; c < nc; ++c)
            if (p.col_matrix[c] == m) col_at[p.col_pos[c]] = (int)c;
        for (uint32_t off = 0; off < row_bytes;) {
            const uint32_t to_sector = 32u - (view + off) % 32u;  // 16 or 32
            const uint32_t width = std::min(to_sector, row_bytes - off);
            LaneTile t;
            std::memset(&t, 0, sizeof(t));
            t.esize = esize;
            t.words = width / 4;
            t.byte_off = off;
            t.rec_off = view + off;
            bool any = false, big = false;
            for (uint32_t e = 0; e < width / esize; ++e) {
                const int c = col_at[off / esize + e];
                if (c < 0) continue;
                any = true;
                const uint32_t nb = p.col_nbins[c];
                big = big || nb > max_bins;
                t.col_hist[e] = p.col_hist_off[c];
                t.col_nbins[e] = nb;
                t.n_bins = std::max(t.n_bins, nb);
            }
            if (any && big) {
                for (uint32_t e = 0; e < width / esize; ++e) {
                    const int c = col_at[off / esize + e];
                    if (c >= 0) rest[c] = 1;
                }
            } else if (any) {
                t.n_bins = std::max<uint32_t>(t.n_bins, 1);
                tile_bins = std::max(tile_bins, t.n_bins);
                tiles.push_back(t);
            }
            off += width;
        }
    }
}

namespace {

constexpr uint32_t PART_CHUNK_ROWS = 4096;
constexpr uint32_t SUM_CHUNK_ROWS = 8192;

// ---- column sampling (training/sampling/column.rs) -----------------------------
// The reference seeds its column sampler from OS entropy (grower.rs:150-151,
// column.rs:137-142), so no two of its runs draw the same columns; here the
// draws are a splitmix64 stream keyed by (seed, round, output, depth) and
// reproducible. The rule is the reference's: the tree's columns are
// ceil(n * colsample_bytree) of all, each depth's ceil(|tree| *
// colsample_bylevel) of the tree's, by a partial Fisher-Yates shuffle
// (sample_k_inplace, column.rs:266-283), kept in ascending order; a rate
// within 1e-6 of 1 samples nothing (column.rs:64-78).
uint64_t mix64(uint64_t z) {
    z = (z ^ (z >> 30)) * 0xBF58476D1CE4E5B9ull;
    z = (z ^ (z >> 27)) * 0x94D049BB133111EBull;
    return z ^ (z >> 31);
}
struct ColStream {
    uint64_t s;
    ColStream(uint64_t seed, uint32_t round, uint32_t output, uint32_t depth) {
        s = mix64(seed ^ (0x9E3779B97F4A7C15ull * (1ull + round)));
        s = mix64(s ^ (0xC2B2AE3D27D4EB4Full * (1ull + output)));
        s = mix64(s ^ (0x165667B19E3779F9ull * (1ull + depth)));
    }
    uint64_t next() {
        s += 0x9E3779B97F4A7C15ull;
        return mix64(s);
    }
};
constexpr uint32_t COL_TREE_DEPTH = 0xFFFFFFFFu;  // stream of the per-tree draw
bool col_rate_samples(float rate) { return std::fabs(rate - 1.0f) >= 1e-6f; }
size_t col_sample_count(size_t n, float rate) {
    const size_t k = (size_t)std::ceil((float)n * rate);
    return std::min(std::max<size_t>(k, 1), n);
}
void col_sample_k(std::vector<uint32_t>& v, size_t k, ColStream& rng) {
    const size_t n = v.size();
    if (k >= n) return;
    for (size_t i = 0; i < k; ++i) std::swap(v[i], v[rng.next() % (n - i) + i]);
    v.resize(k);
    std::sort(v.begin(), v.end());
}

// ---- uniform row sampling (training/sampling/row.rs:168-210) -------------------
// The reference's generator, restated: rand 0.8's SmallRng on 64-bit targets
// is Xoshiro256++, seed_from_u64 fills its state with four SplitMix64
// outputs, and gen_range(0..=i) is UniformInt::sample_single_inclusive (a
// 64x64 -> 128-bit multiply, rejecting low halves above the zone
// (range << lz(range)) - 1). sample_uniform keeps k = max(1, trunc(f32(n) *
// subsample)) rows by reservoir sampling: rows 0..k-1, then row i >= k
// replaces slot j = gen_range(0..=i) when j < k.
class RowSampler {
  public:
    explicit RowSampler(uint64_t seed) {
        for (int i = 0; i < 4; ++i) {
            seed += 0x9E3779B97F4A7C15ull;
            s_[i] = mix64(seed);
        }
    }
    // the sampled rows of the next call (one call per output and round) as a mask
    uint64_t sample(uint64_t n, float rate, std::vector<uint8_t>& mask) {
        uint64_t k = (uint64_t)((float)n * rate);
        k = std::min<uint64_t>(std::max<uint64_t>(k, 1), n);
        idx_.resize(k);
        for (uint64_t i = 0; i < k; ++i) idx_[i] = (uint32_t)i;
        for (uint64_t i = k; i < n; ++i) {
            const uint64_t j = range_inclusive(i);
            if (j < k) idx_[j] = (uint32_t)i;
        }
        mask.assign(n, 0);
        for (uint32_t r : idx_) mask[r] = 1;
        return k;
    }
    // sample_goss (row.rs:214-280) on one output's (grad, hess) pairs: code
    // 1 for the rows of the top_rate share by |grad x hess| (ties at the
    // threshold included), 2 for the other_rate x n drawn from the rest with
    // probability need / rest (rng.gen::<f32>(): the top 24 bits of the
    // upper half of a generator output, times 2^-24), whose grad / hess
    // are scaled by *mult; 0 for the rows left out. Returns the kept count.
    uint64_t goss(const float* gh, uint64_t n, float top_rate, float other_rate, std::vector<uint8_t>& code,
                  float* mult) {
        std::vector<float> mag(n);
        for (uint64_t i = 0; i < n; ++i) mag[i] = std::fabs(gh[2 * i] * gh[2 * i + 1]);
        uint64_t top_k = (uint64_t)((float)n * top_rate);
        top_k = std::min<uint64_t>(std::max<uint64_t>(top_k, 1), n - 1);
        const uint64_t other_k = std::max<uint64_t>((uint64_t)((float)n * other_rate), 1);
        std::vector<float> sorted(mag);
        std::nth_element(sorted.begin(), sorted.begin() + (n - top_k), sorted.end());
        const float threshold = sorted[n - top_k];
        *mult = (float)(n - top_k) / (float)other_k;
        uint64_t big = 0, small = 0;
        code.assign(n, 0);
        for (uint64_t i = 0; i < n; ++i) {
            if (mag[i] >= threshold) {
                code[i] = 1;
                ++big;
                continue;
            }
            const uint64_t need = other_k > small ? other_k - small : 0;
            const uint64_t top_left = top_k > big ? top_k - big : 0;
            const uint64_t rest = (n - i) > top_left ? (n - i) - top_left : 0;
            if (rest > 0) {
                const float prob = (float)need / (float)rest;
                const float u = (float)((uint32_t)(next() >> 32) >> 8) * (1.0f / 16777216.0f);
                if (u < prob) {
                    code[i] = 2;
                    ++small;
                }
            }
        }
        return big + small;
    }

  private:
    uint64_t s_[4];
    std::vector<uint32_t> idx_;
    static uint64_t rotl(uint64_t x, int k) { return (x << k) | (x >> (64 - k)); }
    uint64_t next() {  // Xoshiro256++
        const uint64_t r = rotl(s_[0] + s_[3], 23) + s_[0];
        const uint64_t t = s_[1] << 17;
        s_[2] ^= s_[0];
        s_[3] ^= s_[1];
        s_[1] ^= s_[2];
        s_[0] ^= s_[3];
        s_[2] ^= t;
        s_[3] = rotl(s_[3], 45);
        return r;
    }
    uint64_t range_inclusive(uint64_t high) {  // gen_range(0..=high), high < 2^64 - 1
        const uint64_t range = high + 1;
        const uint64_t zone = (range << __builtin_clzll(range)) - 1;
        for (;;) {
            const unsigned __int128 m = (unsigned __int128)next() * range;
            if ((uint64_t)m <= zone) return (uint64_t)(m >> 64);
        }
    }
};

float to_f32(double d) {
    const double lim = 0x1.ffffffp127;
    const double fmax = (double)std::numeric_limits<float>::max();
    if (d >= lim) return std::numeric_limits<float>::infinity();
    if (d <= -lim) return -std::numeric_limits<float>::infinity();
    if (d > fmax) return std::numeric_limits<float>::max();
    if (d < -fmax) return -std::numeric_limits<float>::max();
    return (float)d;
}

// f32::next_up as used for split thresholds (grower.rs:543-556).
float next_up(float x) {
    if (std::isnan(x) || x == std::numeric_limits<float>::infinity()) return x;
    uint32_t b;
    if (x == 0.0f) {
        b = 1;
    } else {
        std::memcpy(&b, &x, 4);
        b = x > 0.0f ? b + 1 : b - 1;
    }
    float r;
    std::memcpy(&r, &b, 4);
    return r;
}

// GainParams::compute_leaf_weight (training/gbdt/split/gain.rs:151-168).
float leaf_weight(double g, double h, const bst_config& c) {
    const double lambda = (double)c.lambda, alpha = (double)c.alpha;
    if (alpha == 0.0) return to_f32(-g / (h + lambda));
    const double ag = std::fabs(g);
    if (ag <= alpha) return 0.0f;
    const double sign = g > 0.0 ? -1.0 : 1.0;
    return to_f32(sign * (ag - alpha) / (h + lambda));
}

std::vector<uint32_t> bitset_words(const unsigned long long cats[4]) {  // categories.rs:145
    uint32_t mx = 0;
    bool any = false;
    for (uint32_t c = 0; c < 256; ++c)
        if ((cats[c >> 6] >> (c & 63)) & 1ull) {
            mx = c;
            any = true;
        }
    if (!any) return {};
    std::vector<uint32_t> w((mx >> 5) + 1, 0);
    for (uint32_t c = 0; c <= mx; ++c)
        if ((cats[c >> 6] >> (c & 63)) & 1ull) w[c >> 5] |= 1u << (c & 31);
    return w;
}

// Pinned staging area for per-level work lists.
struct Staging {
    char* p = nullptr;
    size_t cap = 0, off = 0;
    ~Staging() { pinned_free(p); }
    void reserve(size_t bytes) {
        if (bytes <= cap) return;
        pinned_free(p);
        p = nullptr;
        p = static_cast<char*>(pinned_alloc(bytes));
        cap = bytes;
        off = 0;
    }
    template <class T>
    T* take(size_t count) {
        size_t a = (off + 63) & ~size_t(63);
        size_t need = a + count * sizeof(T);
        if (need > cap) throw Error{BST_ERR_OUT_OF_MEMORY, "staging area exhausted"};
        off = need;
        return reinterpret_cast<T*>(p + a);
    }
    void reset() { off = 0; }
};

struct Timer {
    std::vector<cudaEvent_t> evs;
    std::vector<std::pair<int, size_t>> marks;  // (phase, first event index)
    size_t used = 0;
    cudaStream_t st = nullptr;
    double acc[8] = {0, 0, 0, 0, 0, 0, 0, 0};
    ~Timer() {
        for (auto e : evs) cudaEventDestroy(e);
    }
    cudaEvent_t next() {
        if (used == evs.size()) {
            cudaEvent_t e;
            BST_CK(cudaEventCreate(&e));
            evs.push_back(e);
        }
        return evs[used++];
    }
    // in_graph: record as event-record nodes of a stream capture (a plain
    // record during capture is only an internal dependency, not a timestamp)
    bool in_graph = false;
    bool broken = false;
    bool enabled = true;  // off: begin/end record nothing (no event nodes in graphs)
    void record(cudaEvent_t e) {
        if (in_graph)
            BST_CK(cudaEventRecordWithFlags(e, st, cudaEventRecordExternal));
        else
            BST_CK(cudaEventRecord(e, st));
    }
    size_t begin(int phase) {
        if (!enabled) return 0;
        size_t i = used;
        record(next());
        marks.push_back({phase, i});
        return i;
    }
    void end() {
        if (enabled) record(next());
    }
    // stream must be idle
    void collect() {
        for (auto& m : marks) {
            float ms = 0;
            BST_CK(cudaEventElapsedTime(&ms, evs[m.second], evs[m.second + 1]));
            acc[m.first] += ms;
        }
        marks.clear();
        used = 0;
    }
    void reserve(size_t k) {
        while (evs.size() < k) {
            cudaEvent_t e;
            BST_CK(cudaEventCreate(&e));
            evs.push_back(e);
        }
    }
    // For events recorded inside a CUDA graph: accumulate, keep the marks.
    // Returns false (and stops trying) if the events cannot be timed.
    bool collect_keep() {
        if (broken) return false;
        double tmp[8] = {0, 0, 0, 0, 0, 0, 0, 0};
        for (auto& m : marks) {
            float ms = 0;
            if (cudaEventElapsedTime(&ms, evs[m.second], evs[m.second + 1]) != cudaSuccess) {
                cudaGetLastError();
                broken = true;
                return false;
            }
            tmp[m.first] += ms;
        }
        for (int i = 0; i < 8; ++i) acc[i] += tmp[i];
        return true;
    }
};

enum Phase { PH_BIN = 0, PH_GRAD = 1, PH_HIST = 2, PH_SCAN = 3, PH_PART = 4, PH_LEAF = 5, PH_OTHER = 6 };

struct PNode {
    uint32_t begin = 0, count = 0;
};

struct Cand {
    uint32_t node, tree_node, depth;
    NodeSplit split;
    long long G, H;
    uint32_t count;
};

class Trainer {
  public:
    Trainer(const HostDataset& ds, const DeviceBinned& b, const bst_config& cfg, uint32_t n_threads,
            cudaStream_t st, Model& model)
        : ds_(ds), b_(b), p_(b.plan), cfg_(cfg), st_(st), m_(model) {
        n_ = p_.n;
        G_ = model.n_groups;
        n_cols_ = p_.n_cols();
        // column sampling: every node searches the same number of columns
        colsample_ = n_cols_ > 0 && (col_rate_samples(cfg.colsample_bytree) || col_rate_samples(cfg.colsample_bylevel));
        size_t searched = n_cols_;
        if (col_rate_samples(cfg.colsample_bytree)) searched = col_sample_count(searched, cfg.colsample_bytree);
        if (col_rate_samples(cfg.colsample_bylevel)) searched = col_sample_count(searched, cfg.colsample_bylevel);
        // the rayon reduction (last maximal column wins) only from 16 searched
        // columns (find.rs:125-129, utils.rs:152)
        last_wins_ = (n_threads != 1) && searched >= 16;
        leafwise_ = cfg.growth_strategy == BST_GROWTH_LEAFWISE;
        const uint32_t max_leaves = leafwise_ ? cfg.max_leaves : (1u << std::min<uint32_t>(cfg.max_depth, 31));
        // batched leaf-wise: room for speculative expansions (grow_leafwise)
        max_pnodes_ = std::max<uint32_t>(1, leafwise_ && cfg.batched ? 2 * max_leaves : max_leaves);
        timer_.st = st;
        timer_.enabled = cfg.phase_timings != 0;
        gp_.lambda = (double)cfg.lambda;
        gp_.min_gain = (double)cfg.min_gain;
        gp_.min_child_weight = (double)cfg.min_child_weight;
        gp_.min_samples_leaf = cfg.min_samples_leaf;
        gp_.max_onehot_cats = cfg.max_onehot_cats;
    }

    void start() { setup(); }

    // One tree on caller-given gradients (TreeGrower::grow, grower.rs:265).
    HostTree run_external(const float* g, const float* h) {
        external_ = true;  // caller-given gradients are used as they are (f32)
        setup_common();
        const uint64_t n = n_;
        pred_.alloc(n);
        BST_CK(cudaMemsetAsync(pred_.p, 0, sizeof(float) * n, st_));
        gh_.alloc(n);
        maxabs_.alloc(2);
        scales_.alloc(4);
        h_scales_.assign(4, 1.0);
        std::vector<float2> gh(n);
        float mg = 0.0f, mh = 0.0f;
        for (uint64_t i = 0; i < n; ++i) {
            gh[i] = make_float2(g[i], h[i]);
            if (std::fabs(g[i]) <= 3.4e38f) mg = std::max(mg, std::fabs(g[i]));
            if (std::fabs(h[i]) <= 3.4e38f) mh = std::max(mh, std::fabs(h[i]));
        }
        unsigned bits[2];
        std::memcpy(&bits[0], &mg, 4);
        std::memcpy(&bits[1], &mh, 4);
        BST_CK(cudaMemcpyAsync(gh_.p, gh.data(), sizeof(float2) * n, cudaMemcpyHostToDevice, st_));
        BST_CK(cudaMemcpyAsync(maxabs_.p, bits, sizeof(bits), cudaMemcpyHostToDevice, st_));
        launch_fixed_scales(maxabs_.p, 1, n_, scales_.p, st_);
        BST_CK(cudaMemcpyAsync(h_scales_.data(), scales_.p, sizeof(double) * 4, cudaMemcpyDeviceToHost, st_));
        BST_CK(cudaStreamSynchronize(st_));
        HostTree t = grow(0);
        m_.train_pred.resize(n);
        BST_CK(cudaMemcpy(m_.train_pred.data(), pred_.p, sizeof(float) * n, cudaMemcpyDeviceToHost));
        return t;
    }

    void run(const HostDataset* val = nullptr) {
        setup();
        if (cfg_.early_stopping_rounds <= 0) {  // None or Some(0): disabled (config.rs:366)
            rounds(cfg_.n_trees);
            m_.rounds_run = cfg_.n_trees;
            finish();
            return;
        }
        // Early stopping (trainer.rs:344-390, callback.rs:103-136): after
        // every round, the validation metric (the training metric without a
        // validation set; NaN with Metric::None) against the best so far;
        // stop once `patience` rounds passed without improvement and keep the
        // trees up to the best round. The margin accuracy is the one
        // higher-is-better metric (metrics/mod.rs:288-303).
        const uint32_t patience = (uint32_t)cfg_.early_stopping_rounds;
        const int metric = resolve_metric(cfg_.metric, cfg_.objective);
        const bool higher = metric == BST_METRIC_MARGIN_ACCURACY;
        if (metric != BST_METRIC_NONE && val) setup_validation(*val);
        bool have_best = false;
        double best = 0.0;
        uint32_t best_round = 0, cur = 0;
        size_t best_n_trees = 0;
        for (uint32_t r = 0; r < cfg_.n_trees; ++r) {
            const size_t before = m_.trees.size();
            rounds(1);
            m_.rounds_run = r + 1;
            double value = std::numeric_limits<double>::quiet_NaN();
            if (metric != BST_METRIC_NONE) value = val ? validation_value(metric, before) : train_value(metric);
            const bool improved = !have_best || (higher ? value > best : value < best);
            if (improved) {
                have_best = true;
                best = value;
                best_round = cur;
            }
            ++cur;
            if (cur - best_round > patience) break;  // Stop
            if (improved) best_n_trees = m_.trees.size();  // Improved
        }
        if (have_best) m_.rounds_kept = best_round + 1;
        const bool truncate = best_n_trees > 0 && best_n_trees < m_.trees.size();
        if (truncate) {
            std::lock_guard<std::mutex> lk(m_.mu);
            m_.trees.resize(best_n_trees);
            m_.dev.reset();
        }
        finish();
        if (truncate) predict_host(m_, ds_, true, m_.train_pred.data());  // the kept trees' predictions
    }

    // Boosting rounds (trainer.rs:242-335): gradients of every output, then
    // one tree per output.
    void rounds(uint32_t k) {
        BST_RANGE("bst.rounds");
        const int obj = cfg_.objective;
        for (uint32_t round = 0; round < k; ++round) {
            timer_.begin(PH_GRAD);
            BST_CK(cudaMemsetAsync(maxabs_.p, 0, sizeof(unsigned) * 2 * G_, st_));
            launch_gradients(obj, G_, pred_.p, y_.p, w_.p, n_, gh_.p, maxabs_.p, st_, alpha_.p, cfg_.huber_delta);
            if (rowsample_) {  // row.rs: per output, zero the rows outside the sample
                for (uint32_t o = 0; o < G_; ++o) {
                    uint8_t* dm = d_rowmask_.p + (size_t)o * n_;
                    float2* go = gh_.p + (size_t)o * n_;
                    if (!goss_) {
                        n_sampled_[o] = (uint32_t)row_sampler_->sample(n_, cfg_.subsample, h_rowmask_);
                        BST_CK(cudaMemcpyAsync(dm, h_rowmask_.data(), n_, cudaMemcpyHostToDevice,
                                               st_));  // pageable: staged before the call returns
                        launch_zero_unsampled(go, dm, n_, st_);
                    } else if (round_no_ < goss_warmup_) {  // GOSS starts at round floor(1 / learning_rate)
                        n_sampled_[o] = (uint32_t)n_;
                        BST_CK(cudaMemsetAsync(dm, 1, n_, st_));
                    } else {
                        h_gh_.resize(2 * (size_t)n_);
                        BST_CK(cudaMemcpyAsync(h_gh_.data(), go, sizeof(float2) * n_, cudaMemcpyDeviceToHost, st_));
                        BST_CK(cudaStreamSynchronize(st_));
                        float mult = 1.0f;
                        n_sampled_[o] = (uint32_t)row_sampler_->goss(h_gh_.data(), n_, cfg_.goss_top_rate,
                                                                     cfg_.goss_other_rate, h_rowmask_, &mult);
                        d_goss_code_.alloc(n_);
                        BST_CK(cudaMemcpyAsync(d_goss_code_.p, h_rowmask_.data(), n_, cudaMemcpyHostToDevice, st_));
                        launch_goss_apply(go, d_goss_code_.p, mult, dm, n_, st_);
                    }
                }
                BST_CK(cudaMemsetAsync(maxabs_.p, 0, sizeof(unsigned) * 2 * G_, st_));
                for (uint32_t o = 0; o < G_; ++o) launch_maxabs(gh_.p + (size_t)o * n_, n_, maxabs_.p + 2 * o, st_);
                m_.counters.launches += 2 * G_;
            }
            m_.counters.launches += 1;
            if (qmode_ != GRAD_F32) {  // the quantisation also writes the fixed-point scales
                launch_quantize(qmode_, G_, gh_.p, n_, maxabs_.p, cfg_.seed, round_no_, 0u, gq_.p, qscales_.p, st_,
                                scales_.p);
            } else {
                launch_fixed_scales(maxabs_.p, G_, n_, scales_.p, st_);
            }
            m_.counters.launches += 1;
            tree_round_ = round_no_;  // the round of this round's trees (column sampling)
            ++round_no_;
            timer_.end();
            if (use_batched_) {
                // device-side trees: no host round trip until a ring slot is reused
                for (uint32_t o = 0; o < G_; ++o) {
                    const uint32_t si = (uint32_t)(seq_ % RING);
                    if (slots_[si].pending) push_tree(collect_batched(si));
                    launch_batched(o, si);
                    ++seq_;
                }
                continue;
            }
            BST_CK(cudaMemcpyAsync(h_scales_.data(), scales_.p, sizeof(double) * 4 * G_, cudaMemcpyDeviceToHost, st_));
            if (qmode_ != GRAD_F32)
                BST_CK(cudaMemcpyAsync(h_qscales_.data(), qscales_.p, sizeof(double) * 4 * G_,
                                       cudaMemcpyDeviceToHost, st_));
            BST_CK(cudaStreamSynchronize(st_));
            for (uint32_t o = 0; o < G_; ++o) push_tree(grow(o), o);
        }
        if (use_batched_)
            for (uint32_t i = 0; i < RING; ++i) {
                const uint32_t si = (uint32_t)((seq_ + i) % RING);
                if (slots_[si].pending) push_tree(collect_batched(si));
            }
        BST_CK(cudaStreamSynchronize(st_));
        timer_.collect();
        for (int i = 1; i < 7; ++i) {
            m_.timings[i] += timer_.acc[i];
            timer_.acc[i] = 0.0;
        }
        m_.counters.hist_ms = m_.timings[PH_HIST];
    }

    void push_tree(HostTree&& t, uint32_t o) {
        t.group = o;
        std::lock_guard<std::mutex> lk(m_.mu);
        m_.trees.push_back(std::move(t));
        m_.dev.reset();
    }
    void push_tree(HostTree&& t) {
        const uint32_t o = t.group;
        push_tree(std::move(t), o);
    }

    // ---- early-stopping evaluation -------------------------------------------
    const HostDataset* val_ = nullptr;
    DevArray<float> val_x_, val_pred_, eval_tmp_;
    std::vector<float> eval_host_;

    void setup_validation(const HostDataset& v) {
        val_ = &v;
        const uint64_t nv = v.n;
        val_x_.alloc(std::max<uint64_t>(1, nv * v.F));
        if (nv * v.F) BST_CK(cudaMemcpy(val_x_.p, v.xdata(), sizeof(float) * nv * v.F, cudaMemcpyHostToDevice));
        std::vector<float> init((size_t)G_ * nv);
        for (uint32_t g = 0; g < G_; ++g)
            std::fill(init.begin() + (size_t)g * nv, init.begin() + (size_t)(g + 1) * nv, m_.base[g]);
        val_pred_.alloc(std::max<size_t>(1, init.size()));
        if (!init.empty())
            BST_CK(cudaMemcpy(val_pred_.p, init.data(), sizeof(float) * init.size(), cudaMemcpyHostToDevice));
    }

    // Metric of [G][n] raw margins on the device against labels y / weights
    // w (host): transformed copy (Evaluator::compute, eval.rs:150-185), read
    // back, summed on the host.
    double device_metric(int metric, const float* margins, uint64_t n, const float* y, const float* w) {
        const size_t cnt = (size_t)G_ * n;
        if (cnt == 0) return 0.0;
        eval_tmp_.alloc(cnt);
        BST_CK(cudaMemcpyAsync(eval_tmp_.p, margins, sizeof(float) * cnt, cudaMemcpyDeviceToDevice, st_));
        // every metric but the margin accuracy reads transformed predictions
        // (eval.rs:151, metrics/mod.rs:272-286)
        if (metric != BST_METRIC_MARGIN_ACCURACY)
            launch_transform(transform_of(cfg_.objective), eval_tmp_.p, G_, n, st_);
        eval_host_.resize(cnt);
        BST_CK(cudaMemcpyAsync(eval_host_.data(), eval_tmp_.p, sizeof(float) * cnt, cudaMemcpyDeviceToHost, st_));
        BST_CK(cudaStreamSynchronize(st_));
        return metric_value(metric, eval_host_.data(), G_, n, y, w, metric_params(cfg_));
    }

    double train_value(int metric) {
        return device_metric(metric, pred_.p, n_, ds_.y.data(), ds_.has_w ? ds_.w.data() : nullptr);
    }

    // Adds the trees pushed since `first` (this round's, one per output) to
    // the validation predictions (tree.predict_into, trainer.rs:339-343),
    // then the validation metric.
    double validation_value(int metric, size_t first) {
        const HostDataset& v = *val_;
        if (v.n && m_.trees.size() > first) {
            std::vector<const HostTree*> tp;
            for (size_t t = first; t < m_.trees.size(); ++t) tp.push_back(&m_.trees[t]);
            DeviceForest f;
            upload_node_forest(tp, G_, std::vector<float>(G_, 0.0f), f);
            eval_tmp_.alloc((size_t)G_ * v.n);
            launch_predict(f.view, val_x_.p, v.n, (uint32_t)v.F, 1, eval_tmp_.p, st_);
            launch_add_f32(val_pred_.p, eval_tmp_.p, (uint64_t)G_ * v.n, st_);
            BST_CK(cudaGetLastError());
            BST_CK(cudaStreamSynchronize(st_));  // f is freed on return
        }
        return device_metric(metric, val_pred_.p, v.n, v.y.data(), v.has_w ? v.w.data() : nullptr);
    }

    // Training predictions back to the model.
    void finish() {
        m_.train_pred.resize((size_t)G_ * n_);
        BST_CK(cudaMemcpy(m_.train_pred.data(), pred_.p, sizeof(float) * G_ * n_, cudaMemcpyDeviceToHost));
    }

  private:
    const HostDataset& ds_;
    const DeviceBinned& b_;
    const BinPlan& p_;
    const bst_config& cfg_;
    cudaStream_t st_;
    Model& m_;
    uint64_t n_ = 0;
    uint32_t G_ = 1, n_cols_ = 0, max_pnodes_ = 1;
    bool last_wins_ = false, leafwise_ = false;
    // column sampling: per-depth column masks of the tree being grown
    // ([depth][n_cols], depth < col_levels_), on the device in d_colmask_
    bool colsample_ = false;
    uint32_t col_levels_ = 0;
    // row sampling: per-output masks of the round's sampled rows and their counts
    bool rowsample_ = false;
    std::unique_ptr<RowSampler> row_sampler_;
    DevArray<float> alpha_;  // pinball: [G] alphas
    // GOSS row sampling: the sampler's row codes and the grad/hess read back
    bool goss_ = false;
    uint64_t goss_warmup_ = 0;
    DevArray<uint8_t> d_goss_code_;
    std::vector<float> h_gh_;
    // leaf renewing (L1 / pinball losses)
    bool renew_ = false;
    RenewDev rd_{};
    DevArray<uint32_t> rd_small_, rd_big_;
    float quantile_alpha(uint32_t o) const {
        return cfg_.objective == BST_OBJ_PINBALL ? quantile_alpha_of(cfg_, o) : 0.5f;
    }
    void setup_renew() {
        renew_ = !external_ && (cfg_.objective == BST_OBJ_ABSOLUTE || cfg_.objective == BST_OBJ_PINBALL);
        if (!renew_) return;
        const uint32_t cap = max_pnodes_ + 1;
        rd_small_.alloc((size_t)cap * (3 + 256));
        rd_.cap = cap;
        rd_.cnt = rd_small_.p;
        rd_.prefix = rd_small_.p + cap;
        rd_.rank = rd_small_.p + 2 * (size_t)cap;
        rd_.hist = rd_small_.p + 3 * (size_t)cap;
        rd_.n_rows = (uint32_t)n_;
        if (ds_.has_w) {
            rd_big_.alloc(4 * (size_t)n_);
            for (int k = 0; k < 2; ++k) {
                rd_.key[k] = rd_big_.p + (size_t)k * n_;
                rd_.row[k] = rd_big_.p + (size_t)(2 + k) * n_;
            }
        }
        if (!d_bleaves_.p) d_bleaves_.alloc((size_t)max_pnodes_ + 1);
        bd_.leaves = d_bleaves_.p;
#ifdef BST_CHECKED
        bd_.chk_rows = (uint32_t)n_;
#endif
        if (!bd_.state) {  // no columns: no histogram state was set up
            d_bstate_.alloc(1);
            bd_.state = d_bstate_.p;
        }
        if (!bd_.leaf_map) {
            const uint64_t max_lc = n_ / B_LEAF_CHUNK + max_pnodes_ + 16;
            d_leaf_map_.alloc(max_lc);
            bd_.leaf_map = d_leaf_map_.p;
            bd_.max_leaf_chunks = (uint32_t)max_lc;
        }
        if (!g_wide_) g_wide_ = sm_count() * 8;
    }
    // Host-driven growth: the grown tree's leaves renewed on the device
    // (values read back into the host tree and the prediction update).
    void renew_host_leaves(uint32_t o) {
        std::vector<BLeaf> lv;
        std::vector<uint32_t> pnodes;
        std::vector<uint2> lmap;
        for (uint32_t pnode = 0; pnode < n_pnodes_; ++pnode) {
            if (leaf_tree_node_[pnode] == 0xFFFFFFFFu) continue;
            BLeaf lf;
            lf.begin = pn_[pnode].begin;
            lf.count = pn_[pnode].count;
            lf.value = leaf_value_[pnode];
            lf.tnode = leaf_tree_node_[pnode];
            lf.chunk_off = (uint32_t)lmap.size();
            lf.buf = 0;
            for (uint32_t s = 0; s < lf.count; s += B_LEAF_CHUNK)
                lmap.push_back(make_uint2((uint32_t)lv.size(), lf.begin + s));
            lv.push_back(lf);
            pnodes.push_back(pnode);
        }
        if (lv.empty()) return;
        if (lmap.size() > bd_.max_leaf_chunks) throw Error{BST_ERR_INVALID_ARGUMENT, "leaf chunk map exceeds its buffer"};
        BState* hs = stage_.take<BState>(1);
        std::memset(hs, 0, sizeof(BState));
        hs->n_leaves = (uint32_t)lv.size();
        hs->leaf_chunks = (uint32_t)lmap.size();
        BLeaf* hl = stage_.take<BLeaf>(lv.size());
        std::copy(lv.begin(), lv.end(), hl);
        uint2* hm = stage_.take<uint2>(std::max<size_t>(1, lmap.size()));
        std::copy(lmap.begin(), lmap.end(), hm);
        upload(hs, 1, d_bstate_);
        upload(hl, lv.size(), d_bleaves_);
        upload(hm, lmap.size(), d_leaf_map_);
        BDev d = bd_;
        d.tree = nullptr;
        d.rmask = rowmask(o);
        timer_.begin(PH_LEAF);
        launch_leaf_renew(d, rd_, ridx_.p, ridx_.p, y_.p, pred_.p + (size_t)o * n_, ds_.has_w ? w_.p : nullptr,
                          quantile_alpha(o), cfg_.learning_rate, g_wide_, st_);
        timer_.end();
        m_.counters.launches += ds_.has_w ? 1 : 12;
        BST_CK(cudaMemcpyAsync(hl, d_bleaves_.p, sizeof(BLeaf) * lv.size(), cudaMemcpyDeviceToHost, st_));
        BST_CK(cudaStreamSynchronize(st_));
        for (size_t j = 0; j < lv.size(); ++j) {
            tree_.leaf[hl[j].tnode] = hl[j].value;
            leaf_value_[pnodes[j]] = hl[j].value;
        }
        stage_.reset();
    }
    DevArray<uint8_t> d_rowmask_;
    std::vector<uint8_t> h_rowmask_;
    std::vector<uint32_t> n_sampled_;
    DevArray<unsigned> d_scnt_;
    const uint8_t* rowmask(uint32_t o) const { return rowsample_ ? d_rowmask_.p + (size_t)o * n_ : nullptr; }
    uint32_t tree_output_ = 0;  // the output of the host-driven tree being grown
    uint32_t tree_round_ = 0;
    DevArray<uint8_t> d_colmask_;
    std::vector<std::vector<uint8_t>> h_colmask_;  // per ring slot (or [0]): host copies of the masks
    const uint8_t* colmask() const { return colsample_ ? d_colmask_.p : nullptr; }
    // masks of the tree (tree_round_, o) into host buffer `slot`, then to the device
    void upload_col_masks(uint32_t o, uint32_t slot) {
        if (!colsample_) return;
        std::vector<uint32_t> tree_cols(n_cols_);
        for (uint32_t c = 0; c < n_cols_; ++c) tree_cols[c] = c;
        if (col_rate_samples(cfg_.colsample_bytree)) {
            ColStream rng(cfg_.seed, tree_round_, o, COL_TREE_DEPTH);
            col_sample_k(tree_cols, col_sample_count(tree_cols.size(), cfg_.colsample_bytree), rng);
        }
        std::vector<uint8_t>& h = h_colmask_[slot];
        h.assign((size_t)col_levels_ * n_cols_, 0);
        for (uint32_t d = 0; d < col_levels_; ++d) {
            std::vector<uint32_t> lv = tree_cols;
            if (col_rate_samples(cfg_.colsample_bylevel)) {
                ColStream rng(cfg_.seed, tree_round_, o, d);
                col_sample_k(lv, col_sample_count(lv.size(), cfg_.colsample_bylevel), rng);
            }
            for (uint32_t c : lv) h[(size_t)d * n_cols_ + c] = 1;
        }
        // pageable source: the copy is staged before the call returns
        BST_CK(cudaMemcpyAsync(d_colmask_.p, h.data(), h.size(), cudaMemcpyHostToDevice, st_));
    }
    GainParamsDev gp_{};
    Timer timer_;
    Staging stage_;

    DevArray<float> pred_, y_, w_;
    DevArray<float2> gh_;
    DevArray<unsigned> maxabs_;
    DevArray<double> scales_;
    std::vector<double> h_scales_;
    DevArray<uint32_t> ridx_, tmp_, row_leaf_;
    // Q8 node histograms in HBin32 when every sum fits 32 bits (n * 127 < 2^31)
    bool hist32_ = false;
    size_t hbytes() const { return hist32_ ? sizeof(HBin32) : sizeof(HBin); }
    // the rows' gradient elements in the order of ridx_ / tmp_ (batched form):
    // the partition moves them with the row ids, the histogram reads them in place
    DevArray<uint8_t> qpos_[2];
    // column-major copy of the bins (batched form): the partition's split column
    DevArray<uint8_t> fm8_;
    DevArray<uint16_t> fm16_;
    BinsFM fm_{};
    DevArray<HBin> hist_;
    uint64_t slot_bins_ = 0;
    DevArray<HistTile> tiles_;
    uint32_t n_tiles_ = 0, tile_smem_ = 0;
    DevArray<LaneTile> lane_tiles_;
    uint32_t n_lane_tiles_ = 0, lane_bins_ = 0;
    DevArray<ScanColumn> scan_cols_;
    DevArray<HistChunk> d_schunks_;
    DevArray<ScanNode> d_scan_nodes_;
    DevArray<ColCand> d_cand_;
    DevArray<long long> d_node_tot_, d_sums_;
    DevArray<NodeSplit> d_splits_;
    DevArray<PartWork> d_pworks_;
    DevArray<PartChunk> d_pchunks_;
    DevArray<unsigned> d_cursors_;
    DevArray<LeafSeg> d_leaves_;

    // per-tree state
    std::vector<PNode> pn_;
    uint32_t n_pnodes_ = 0;
    HostTree tree_;
    std::vector<uint32_t> leaf_tree_node_;  // by partition node
    std::vector<float> leaf_value_;
    const double* scale_o_ = nullptr;  // units of the histogram sums (scan, node stats)
    double inv_g_ = 1.0, inv_h_ = 1.0;
    GradRef gr_o_{};  // histogram / node-sum source of the current output
    GradRef gx_o_{};  // exact f32 source (leaf solves in quantised mode)

    // quantised training (BST_PRECISION_Q16 / Q8)
    int qmode_ = GRAD_F32;
    bool external_ = false;
    DevArray<uint8_t> gq_;
    DevArray<double> qscales_;
    std::vector<double> h_qscales_;
    uint32_t round_no_ = 0;

    uint32_t grad_bytes() const { return qmode_ == GRAD_Q8 ? 2u : (qmode_ == GRAD_Q16 ? 4u : 8u); }
    GradRef grad_ref(uint32_t o) const {
        GradRef r{};
        r.gh = gh_.p + (size_t)o * n_;
        r.scale = scales_.p + 4 * (size_t)o;
        r.mode = qmode_;
        r.gq = qmode_ == GRAD_F32 ? nullptr : (const void*)(gq_.p + (size_t)o * n_ * (grad_bytes()));
        return r;
    }
    GradRef exact_ref(uint32_t o) const {
        GradRef r = grad_ref(o);
        r.mode = GRAD_F32;
        r.gq = nullptr;
        return r;
    }
    const double* unit_scale(uint32_t o) const {
        return (qmode_ == GRAD_F32 ? scales_.p : qscales_.p) + 4 * (size_t)o;
    }

    void setup() {
        setup_common();
        const uint64_t n = n_;
        pred_.alloc((size_t)G_ * n);
        y_.alloc(n);
        if (ds_.has_w) w_.alloc(n);
        gh_.alloc((size_t)G_ * n);
        maxabs_.alloc(2 * G_);
        scales_.alloc(4 * G_);
        h_scales_.assign(4 * G_, 1.0);
        if (qmode_ != GRAD_F32) {
            gq_.alloc((size_t)G_ * n * grad_bytes());
            qscales_.alloc(4 * G_);
            h_qscales_.assign(4 * G_, 1.0);
        }
        // targets: first output row (targets.output(0) in every objective)
        BST_CK(cudaMemcpyAsync(y_.p, ds_.y.data(), sizeof(float) * n, cudaMemcpyHostToDevice, st_));
        if (cfg_.objective == BST_OBJ_PINBALL) {  // one alpha per output
            std::vector<float> a(G_);
            for (uint32_t o = 0; o < G_; ++o) a[o] = quantile_alpha_of(cfg_, o);
            alpha_.alloc(G_);
            BST_CK(cudaMemcpy(alpha_.p, a.data(), sizeof(float) * G_, cudaMemcpyHostToDevice));
        }
        if (ds_.has_w) BST_CK(cudaMemcpyAsync(w_.p, ds_.w.data(), sizeof(float) * n, cudaMemcpyHostToDevice, st_));
        std::vector<float> init((size_t)G_ * n);
        for (uint32_t g = 0; g < G_; ++g) std::fill(init.begin() + (size_t)g * n, init.begin() + (size_t)(g + 1) * n, m_.base[g]);
        BST_CK(cudaMemcpyAsync(pred_.p, init.data(), sizeof(float) * init.size(), cudaMemcpyHostToDevice, st_));
        BST_CK(cudaStreamSynchronize(st_));
    }

    void setup_common() {
        const uint64_t n = n_;
        qmode_ = external_ ? GRAD_F32 : cfg_.precision;
        hist32_ = qmode_ == GRAD_Q8 && (uint64_t)n_ * 127ull <= 0x7FFFFFFFull;
        ridx_.alloc(n);
        tmp_.alloc(n);
        if (cfg_.record_leaves) row_leaf_.alloc(n);
        slot_bins_ = p_.total_bins;
        if (n_cols_) {
            // one histogram per partition node (the reference's LRU pool is
            // unnecessary with 180 GB of HBM); refuse sizes that cannot fit
            size_t free_b = 0, total_b = 0;
            BST_CK(cudaMemGetInfo(&free_b, &total_b));
            double need = (double)max_pnodes_ * (double)slot_bins_ * sizeof(HBin);
            if (leafwise_ && need > 0.6 * (double)free_b && max_pnodes_ > cfg_.max_leaves) {
                max_pnodes_ = std::max<uint32_t>(1, cfg_.max_leaves);  // no room to speculate
                need = (double)max_pnodes_ * (double)slot_bins_ * sizeof(HBin);
            }
            if (need > 0.6 * (double)free_b)
                throw Error{BST_ERR_UNSUPPORTED, "node histograms need " + std::to_string((uint64_t)need) +
                                                     " bytes; reduce max_depth / max_leaves or max_bins"};
            hist_.alloc((size_t)max_pnodes_ * slot_bins_);
        }
        build_tiles();
        std::vector<ScanColumn> sc(n_cols_);
        for (uint32_t c = 0; c < n_cols_; ++c)
            sc[c] = ScanColumn{p_.col_nbins[c], p_.col_hist_off[c], p_.col_cat[c], p_.col_missing[c]};
        scan_cols_.alloc(std::max<uint32_t>(1, n_cols_));
        if (n_cols_) BST_CK(cudaMemcpy(scan_cols_.p, sc.data(), sizeof(ScanColumn) * n_cols_, cudaMemcpyHostToDevice));

        const size_t max_chunks = (size_t)(n / 1024 + 2 * (size_t)max_pnodes_ + 16);
        d_schunks_.alloc(max_chunks);
        d_pchunks_.alloc(max_chunks);
        d_scan_nodes_.alloc(2 * (size_t)max_pnodes_ + 2);
        d_cand_.alloc((2 * (size_t)max_pnodes_ + 2) * std::max<uint32_t>(1, n_cols_));
        d_node_tot_.alloc(2 * (2 * (size_t)max_pnodes_ + 2));
        d_splits_.alloc(2 * (size_t)max_pnodes_ + 2);
        d_pworks_.alloc(max_pnodes_ + 1);
        d_cursors_.alloc(2 * ((size_t)max_pnodes_ + 1));
        d_sums_.alloc(2 * ((size_t)max_pnodes_ + 1));
        d_leaves_.alloc(max_pnodes_ + 1);
        stage_.reserve(max_chunks * 48 + (size_t)(max_pnodes_ + 4) * 256 + (1 << 20));
        if (n_cols_) setup_hist_state();
        n_sampled_.assign(G_, (uint32_t)n_);
        goss_ = !external_ && cfg_.goss_top_rate > 0.0f;
        goss_warmup_ = (uint64_t)(1.0f / cfg_.learning_rate);  // row.rs:112-116
        if (goss_ && n_ < 2) throw Error{BST_ERR_CONFIG, "GOSS needs at least 2 rows"};
        rowsample_ = std::fabs(cfg_.subsample - 1.0f) >= 1e-6f || goss_;  // config.rs:329-330
        if (rowsample_) {
            row_sampler_ = std::make_unique<RowSampler>(cfg_.seed);
            d_rowmask_.alloc((size_t)G_ * n_);
            d_scnt_.alloc(2 * ((size_t)max_pnodes_ + 1));
            d_bscnt_.alloc(2 * ((size_t)max_pnodes_ + 1));
            bd_.scnt = d_bscnt_.p;
        }
        if (colsample_) {  // splits happen at depths < max_depth (depth-wise) or < max_leaves (leaf-wise)
            col_levels_ = std::max<uint32_t>(1, leafwise_ ? cfg_.max_leaves : cfg_.max_depth);
            d_colmask_.alloc((size_t)col_levels_ * n_cols_);
            h_colmask_.resize(RING);
        }
        use_batched_ = cfg_.batched && !leafwise_ && n_cols_ > 0 && cfg_.max_depth <= 14;
        spec_leafwise_ = cfg_.batched && leafwise_ && n_cols_ > 0;
        if (use_batched_ || spec_leafwise_) {
            if (use_batched_) setup_batched();
            if (spec_leafwise_) setup_lw_device();
            for (auto& q : qpos_) q.alloc((size_t)n_ * grad_bytes());
            if (p_.f8) fm8_.alloc((size_t)n_ * p_.f8);
            if (p_.f16) fm16_.alloc((size_t)n_ * p_.f16);
            launch_transpose_bins(b_.bins8, p_.s8, p_.f8, b_.bins16, p_.s16, p_.f16, n_, fm8_.p, fm16_.p, st_);
            BST_CK(cudaGetLastError());
            fm_ = BinsFM{fm8_.p, fm16_.p, n_};
        }
        setup_renew();
    }

    // ---- device-side level loop, one CUDA graph per output (kernels.h) -------
    bool use_batched_ = false;
    // batched leaf-wise: speculative expansion batches, gradient elements
    // carried positionally in qpos_[0] (aligned with ridx_), split columns
    // read from the column-major bins
    bool spec_leafwise_ = false;
    BDev bd_{};
    DevArray<BState> d_bstate_;
    DevArray<BNode> d_front_[2];
    DevArray<unsigned long long> d_node_key_;
    DevArray<unsigned> d_bscnt_;  // row sampling: the level's sampled rows per side (BDev::scnt)
    DevArray<BExp> d_bexp_;
    DevArray<BTreeNode> d_btree_;
    DevArray<BLeaf> d_bleaves_;
    DevArray<BColumn> d_bcols_;
    DevArray<uint32_t> d_seg_exp_;
    DevArray<uint2> d_part_map_;    // partition chunk -> (expansion, first row)
    DevArray<uint2> d_leaf_map_;    // leaf chunk -> (leaf, first row)
    DevArray<uint8_t> d_part_;      // partial histograms of the lane tiles
    DevArray<uint32_t> d_bin_map_;  // global bin -> (lane tile, partial entry)
    DevArray<uint2> d_ent_;         // node partial entry -> (global bin, lane tile / offset)
    uint32_t n_ent_ = 0;
    DevArray<ScanNode> d_root_scan_;
    uint32_t max_tnodes_ = 0;
    // Pipelined replay: tree k is read back and converted on the host while
    // the device grows tree k+1. Each ring slot owns its own graph per output
    // (its event-record nodes then time only the launch that used the slot).
    static constexpr uint32_t RING = 2;
    struct Slot {
        BTreeNode* tree = nullptr;  // pinned
        BState* state = nullptr;    // pinned
        cudaEvent_t done = nullptr, w0 = nullptr, w1 = nullptr;
        bool pending = false;
        uint32_t o = 0;
        uint32_t cand = 0;   // tuner candidate of the tree in the slot
        bool timed = false;  // its time counts for the tuner
        std::vector<uint32_t> row_leaf;
    };
    Slot slots_[RING];
    uint64_t seq_ = 0;
    std::vector<cudaGraphExec_t> graphs_;  // [o * RING + slot]
    std::vector<std::unique_ptr<Timer>> gtimers_;
    std::vector<uint64_t> graph_launches_, graph_hist_launches_;

  public:
    ~Trainer() {
        free_lw_device();
        for (auto g : graphs_)
            if (g) cudaGraphExecDestroy(g);
        for (auto& sl : slots_) {
            pinned_free(sl.tree);
            pinned_free(sl.state);
            for (auto e : {sl.done, sl.w0, sl.w1})
                if (e) cudaEventDestroy(e);
        }
    }

  private:

    // Level state and buffers of the histogram pipeline (both growth loops).
    void setup_hist_state() {
        init_kernel_attributes();
        const uint32_t max_front = max_pnodes_;
        d_bstate_.alloc(1);
        d_bexp_.alloc(max_front / 2 + 1);
        bd_.state = d_bstate_.p;
#ifdef BST_CHECKED
        bd_.chk_rows = (uint32_t)n_;
#endif
        bd_.exp = d_bexp_.p;
        const uint64_t max_pc = n_ / B_PART_CHUNK + max_front + 16;
        d_part_map_.alloc(max_pc);
        bd_.part_map = d_part_map_.p;
        bd_.max_part_chunks = (uint32_t)max_pc;
        const uint64_t max_lc = n_ / B_LEAF_CHUNK + max_front + 16;
        d_leaf_map_.alloc(max_lc);
        bd_.leaf_map = d_leaf_map_.p;
        bd_.max_leaf_chunks = (uint32_t)max_lc;
        if (n_lane_tiles_ && p_.rec) make_record_maps(maps_, b_.rec.p, n_, p_.rec);
        // launch shapes: the built-in one, or the tuner's candidates (the
        // buffers below are sized for the candidate with the most segments)
        setup_tuning();
        uint32_t tgt_max = hist_target_for(shape_.items, shape_.hist);
        for (const TuneShape& c : tune_cands_) tgt_max = std::max(tgt_max, hist_target_for(c.items, c.hist));
        bd_.hist_seg_max = n_lane_tiles_ ? lane_segment_max(qmode_) : (uint32_t)HIST_CHUNK_MAX;
        apply_shape(shape_);
        // segments per level <= rows / segment + nodes; the segment is at least
        // min(1024, seg_max) and at least rows / hist_target rounded up
        const uint64_t min_seg = std::max<uint64_t>(
            1024, std::min<uint64_t>(bd_.hist_seg_max, (n_ + tgt_max - 1) / tgt_max));
        const uint64_t max_segs = n_ / std::min<uint64_t>(min_seg, HIST_CHUNK_MAX) + max_front + 16;
        d_seg_exp_.alloc(max_segs);
        bd_.seg_exp = d_seg_exp_.p;
        bd_.max_segs = (uint32_t)max_segs;
        if (n_lane_tiles_) {
            d_part_.alloc(max_segs * n_lane_tiles_ * (size_t)lane_part_stride() * lane_part_entry_bytes(qmode_));
            std::vector<uint32_t> bm(p_.total_bins, 0xFFFFFFFFu);
            std::vector<LaneTile> lt(n_lane_tiles_);
            BST_CK(cudaMemcpy(lt.data(), lane_tiles_.p, sizeof(LaneTile) * n_lane_tiles_, cudaMemcpyDeviceToHost));
            std::vector<uint2> ent;
            for (uint32_t t = 0; t < n_lane_tiles_; ++t) {
                const uint32_t C = lt[t].words * 4 / lt[t].esize, B = lt[t].n_bins;
                for (uint32_t e = 0; e < C; ++e)
                    for (uint32_t b = 0; b < lt[t].col_nbins[e]; ++b) {
                        bm[lt[t].col_hist[e] + b] = (t << 16) | (e * B + b);
                        ent.push_back(make_uint2(lt[t].col_hist[e] + b, (t << 16) | (e * B + b)));
                    }
            }
            n_ent_ = (uint32_t)ent.size();
            d_ent_.alloc(std::max<size_t>(1, ent.size()));
            BST_CK(cudaMemcpy(d_ent_.p, ent.data(), sizeof(uint2) * ent.size(), cudaMemcpyHostToDevice));
            d_bin_map_.alloc(p_.total_bins);
            BST_CK(cudaMemcpy(d_bin_map_.p, bm.data(), sizeof(uint32_t) * bm.size(), cudaMemcpyHostToDevice));
        } else {
            d_bin_map_.alloc(std::max<uint64_t>(1, p_.total_bins));
            BST_CK(cudaMemset(d_bin_map_.p, 0xFF, sizeof(uint32_t) * std::max<uint64_t>(1, p_.total_bins)));
        }
    }

    // ---- launch-shape autotuning (autotune.h) ----------------------------------
    RecordMaps maps_;                   // tensor maps of the row records (lane-kernel variant 3)
    TuneShape shape_;                   // the shape the current graphs use
    std::vector<TuneShape> tune_cands_; // exploration candidates (empty: none)
    TuneExplorer tuner_;
    std::string tune_key_;
    bool tune_stored_ = false;
    uint32_t g_wide_ = 0;               // level-kernel grid of the current shape

    // (row segment, lane tile) items per resident histogram block -> the
    // level's segment count target. Each item zeroes and flushes a whole
    // shared histogram, so fewer, larger items cost less, while too few
    // leave SMs idle at the end of a level.
    uint32_t hist_target_for(uint32_t items, uint32_t variant) const {
        const uint32_t blocks =
            n_lane_tiles_ ? sm_count() * lane_blocks_per_sm(qmode_, (int)variant) : sm_count() * 3u;
        const uint32_t tiles = std::max<uint32_t>(1, n_lane_tiles_ ? n_lane_tiles_ : n_tiles_);
        return std::max<uint32_t>(1, items * blocks / tiles);
    }

    void apply_shape(const TuneShape& sh) {
        const bool changed = !(sh == shape_) || g_wide_ == 0;
        shape_ = sh;
        bd_.hist_target = hist_target_for(sh.items, sh.hist);
        g_wide_ = sm_count() * sh.grid;
        if (changed)  // graphs bake the shape in: capture again on next use
            for (auto& g : graphs_)
                if (g) {
                    BST_CK(cudaGraphExecDestroy(g));  // an in-flight launch completes first
                    g = nullptr;
                }
    }

    // The built-in shape (measured on B200, 1M x 100 q8: 0.95 ms per tree
    // at three items per block, 0.88 at two or one), a cached choice, or the
    // candidates to explore on this run's first trees (batched depth-wise).
    void setup_tuning() {
        shape_ = TuneShape{};
        tune_cands_.clear();
        const bool depthwise_batched = cfg_.batched && !leafwise_ && cfg_.max_depth <= 14;
        if (!depthwise_batched) return;
        uint32_t lg = 0;
        while ((1ull << (lg + 1)) <= n_) ++lg;
        tune_key_ = device_signature(cfg_.device) + "|mode" + std::to_string(qmode_) + "|rec=" +
                    std::to_string(p_.rec) + "|u16=" + std::to_string(p_.u16_off) + "|tiles=" +
                    std::to_string(n_lane_tiles_) + "+" + std::to_string(n_tiles_) + "|log2n=" + std::to_string(lg) +
                    "|depth=" + std::to_string(cfg_.max_depth) + "|G=" + std::to_string(G_);
        const std::string path = cfg_.autotune_cache ? cfg_.autotune_cache : "";
        TuneShape cached;
        if (tune_cache_lookup(path, tune_key_, cached) && cached.hist < (uint32_t)lane_variants() &&
            (cached.hist != 3 || maps_.ok)) {
            shape_ = cached;
            m_.tune_info = shape_.str() + " (cached)";
            tune_stored_ = true;
            return;
        }
        if (!cfg_.autotune) {
            m_.tune_info = shape_.str() + " (built-in)";
            return;
        }
        // the built-in shape first; the other segment size for the cp.async
        // form, the register and TMA forms (the latter when the row records
        // have tensor maps) at the built-in segment size; then a half-size
        // level-kernel grid
        tune_cands_.push_back(shape_);
        auto cand = [&](uint32_t items, uint32_t hist) {
            TuneShape c;
            c.items = items;
            c.hist = hist;
            c.grid = 8;
            if (hist < (uint32_t)lane_variants() && (hist != 3 || maps_.ok) && !(c == shape_))
                tune_cands_.push_back(c);
        };
        cand(1, 0);
        cand(2, 1);
        cand(2, 2);
        cand(2, 3);
        TuneShape half = shape_;
        half.grid = 4;
        tune_cands_.push_back(half);
        tuner_ = TuneExplorer(tune_cands_, 2, 1);
        shape_ = tune_cands_[0];
        m_.tune_info = "exploring";
    }

    // Exploration finished: keep the winner from the next launch on, and
    // store it.
    void finish_tuning() {
        if (!tuner_.done() || tune_stored_) return;
        tune_stored_ = true;
        const TuneShape best = tuner_.best();
        apply_shape(best);
        const std::vector<double> med = tuner_.medians();
        std::string info = best.str() + " (explored:";
        for (size_t c = 0; c < med.size(); ++c) {
            char buf[64];
            std::snprintf(buf, sizeof buf, " %.3f", med[c]);
            info += " " + tune_cands_[c].str() + buf;
        }
        m_.tune_info = info + " ms/tree)";
        if (cfg_.autotune_cache) tune_cache_store(cfg_.autotune_cache, tune_key_, best);
    }

    void setup_batched() {
        init_kernel_attributes();
        const uint32_t max_front = max_pnodes_;
        max_tnodes_ = 2 * max_front;
        d_front_[0].alloc(max_front);
        d_front_[1].alloc(max_front);
        d_node_key_.alloc(max_front);
        BST_CK(cudaMemset(d_node_key_.p, 0, sizeof(unsigned long long) * max_front));
        d_btree_.alloc(max_tnodes_);
        d_bleaves_.alloc(max_front + 1);
        std::vector<BColumn> bc(n_cols_);
        for (uint32_t c = 0; c < n_cols_; ++c)
            bc[c] = BColumn{p_.col_matrix[c], p_.col_pos[c], p_.col_missing[c], p_.col_default[c]};
        d_bcols_.alloc(n_cols_);
        BST_CK(cudaMemcpy(d_bcols_.p, bc.data(), sizeof(BColumn) * n_cols_, cudaMemcpyHostToDevice));
        const ScanNode rs{0, (uint32_t)n_, 0u, 0u, 0, 0};
        d_root_scan_.alloc(1);
        BST_CK(cudaMemcpy(d_root_scan_.p, &rs, sizeof(rs), cudaMemcpyHostToDevice));
        for (auto& sl : slots_) {
            sl.tree = static_cast<BTreeNode*>(pinned_alloc(sizeof(BTreeNode) * max_tnodes_));
            sl.state = static_cast<BState*>(pinned_alloc(sizeof(BState)));
            BST_CK(cudaEventCreateWithFlags(&sl.done, cudaEventDisableTiming));
            BST_CK(cudaEventCreate(&sl.w0));
            BST_CK(cudaEventCreate(&sl.w1));
        }
        bd_.front[0] = d_front_[0].p;
        bd_.front[1] = d_front_[1].p;
        bd_.tree = d_btree_.p;
        bd_.leaves = d_bleaves_.p;
        bd_.pworks = d_pworks_.p;
        bd_.cursors = d_cursors_.p;
        bd_.scan_nodes = d_scan_nodes_.p;
        bd_.sums = d_sums_.p;
        bd_.bcols = d_bcols_.p;
        bd_.max_front = max_front;
        bd_.node_key = d_node_key_.p;
        bd_.max_tnodes = max_tnodes_;
        graphs_.assign((size_t)G_ * RING, nullptr);
        gtimers_.resize((size_t)G_ * RING);
        graph_launches_.assign((size_t)G_ * RING, 0);
        graph_hist_launches_.assign((size_t)G_ * RING, 0);
    }

    // Rows per histogram row segment for `rows` rows (the rule of k_b_children).
    uint32_t chunk_rows(uint64_t rows) const {
        const uint64_t tgt = std::max<uint32_t>(1, bd_.hist_target);
        uint64_t want = (rows + tgt - 1) / tgt;
        want = (want + 255) & ~uint64_t(255);
        return (uint32_t)std::min<uint64_t>(std::max<uint64_t>(want, 1024), bd_.hist_seg_max);
    }

    // Histograms of the smaller children described by the level state in bd_
    // (or of all rows, root): partial histograms of the lane tiles, general
    // tiles (atomic, into zeroed right slots), then the merge with the
    // subtraction trick.
    // wide: the level has at most WIDE_MERGE_NODES expanding nodes (the
    // merge splits each node's many row segments over more threads)
    static constexpr uint32_t WIDE_MERGE_NODES = 4;
    void enqueue_hist(const GradRef& gr, const uint32_t* ridx, bool root, Timer& tm, uint64_t& launches,
                      uint64_t& hist_launches, bool wide = false) {
        // resident general-tile blocks per SM: 64 registers x 256 threads
        // allow 4; the fixed-point form's 16 B/bin shared histograms allow 3
        const uint32_t g_hist = sm_count() * (qmode_ == GRAD_F32 ? 3 : 4);
        tm.begin(PH_HIST);
        if (n_lane_tiles_)
            launch_b_hist_part(bd_, lane_tiles_.p, n_lane_tiles_, ridx, gr, b_.bins8, p_.s8, b_.bins16, p_.s16,
                               d_part_.p, (int)shape_.hist, &maps_, st_);
        if (n_tiles_)
            launch_b_hist(bd_, tiles_.p, n_tiles_, tile_smem_, ridx, gr, b_.bins8, p_.s8, b_.bins16, p_.s16,
                          hist_.p, slot_bins_, g_hist, st_, hist32_);
        tm.end();
        tm.begin(PH_OTHER);
        launch_b_merge(bd_, hist_.p, slot_bins_, p_.total_bins, d_part_.p, n_lane_tiles_, d_ent_.p, n_ent_,
                       d_bin_map_.p, n_tiles_ > 0, root ? 1 : 0, qmode_, st_, hist32_, wide ? 1 : 0);
        tm.end();
        const uint32_t hist_kernels = (n_lane_tiles_ ? 1u : 0u) + (n_tiles_ ? 1u : 0u);
        launches += 2 * hist_kernels;  // builds and merges
        hist_launches += hist_kernels;
    }

    // The launch sequence of one tree for output o (captured into a graph).
    void enqueue_tree(uint32_t o, Timer& tm, uint64_t& launches, uint64_t& hist_launches) {
        const GradRef gh = grad_ref(o);
        const double* scale = unit_scale(o);
        float* pred = pred_.p + (size_t)o * n_;
        const uint32_t g_wide = g_wide_;
        LeafParams lp{(double)cfg_.lambda, (double)cfg_.alpha, (double)cfg_.min_gain, cfg_.learning_rate, 0u};
        launches = 0;
        hist_launches = 0;
        // level kernels get no more blocks than their level can have work
        // items (idle blocks would still take part in the last-block
        // hand-off): split searches 2^(d+1) nodes x column blocks,
        // partitions n / chunk + 2^d chunks, leaf kernels n / chunk + leaves
        const uint64_t cb = scan_col_blocks(n_cols_);
        auto cap = [&](uint64_t items) { return (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(g_wide, items)); };
        tm.begin(PH_OTHER);
        launch_b_root_init(bd_, ridx_.p, n_, chunk_rows(n_), st_);  // row ids, root node, root histogram state
        if (n_tiles_) BST_CK(cudaMemsetAsync(hist_.p, 0, hbytes() * slot_bins_, st_));
        tm.end();
        enqueue_hist(gh, ridx_.p, true, tm, launches, hist_launches, true);
        tm.begin(PH_SCAN);
        launch_b_scan(bd_, scan_cols_.p, n_cols_, hist_.p, slot_bins_, scale, gp_, d_cand_.p, d_node_tot_.p, 0,
                      last_wins_ ? 1 : 0, lp, 0u, cap(cb), st_, hist32_, d_root_scan_.p,
                      colmask());  // + level-0 decisions
        tm.end();
        launches += 2;  // root init, root split search
        // row indices: level d partitions R[d & 1] into R[(d + 1) & 1]
        uint32_t* R[2] = {ridx_.p, tmp_.p};
        for (uint32_t d = 0; d < cfg_.max_depth; ++d) {
            const int a = (int)(d & 1u);
            const bool need_split = d + 1 < cfg_.max_depth;
            uint32_t* rout = R[(d + 1) & 1u];
            // gradient elements move with the row ids: level 0 reads them in
            // row order (the unpermuted arrays), later levels ping-pong
            const void* qin = d == 0 ? (qmode_ == GRAD_F32 ? (const void*)gh.gh : gh.gq) : (const void*)qpos_[d & 1u].p;
            void* qout = qpos_[(d + 1) & 1u].p;  // the last level's node sums read it too
            tm.begin(PH_PART);
            launch_b_partition(bd_, R[d & 1u], rout, b_.bins8, p_.s8, b_.bins16, p_.s16, a, need_split ? 1 : 0,
                               cap(n_ / B_PART_CHUNK + (1ull << d) + 1), qin, qout, qmode_, fm_, st_);  // + children
            tm.end();
            launches += 1;
            if (need_split) {
                GradRef gl = gh;
                gl.qpos = qpos_[(d + 1) & 1u].p;
                if (n_tiles_) {  // general tiles add atomically into the zeroed right slots
                    tm.begin(PH_OTHER);
                    launch_b_zero_right(bd_, hist_.p, slot_bins_, g_wide, st_, hist32_);
                    tm.end();
                    launches += 1;
                }
                // level d expands at most 2^d nodes
                enqueue_hist(gl, rout, false, tm, launches, hist_launches, (1u << std::min(d, 31u)) <= WIDE_MERGE_NODES);
                tm.begin(PH_SCAN);
                launch_b_scan(bd_, scan_cols_.p, n_cols_, hist_.p, slot_bins_, scale, gp_, d_cand_.p,
                              d_node_tot_.p, a ^ 1, last_wins_ ? 1 : 0, lp, (d + 1) & 1u, cap((2ull << d) * cb), st_, hist32_,
                              nullptr, colsample_ ? d_colmask_.p + (size_t)(d + 1) * n_cols_ : nullptr);
                // + column reduction, next level's decisions
                tm.end();
                launches += 1;
            } else {
                tm.begin(PH_OTHER);
                GradRef gl = gh;
                gl.qpos = qpos_[(d + 1) & 1u].p;
                // + children sums, then the tree's leaves (k_b_finalize's work)
                launch_b_sums(bd_, rout, gl, a ^ 1, g_wide, st_, 1, lp, scale, cfg_.max_depth & 1u);
                tm.end();
                launches += 1;
            }
        }
        tm.begin(PH_LEAF);
        if (cfg_.max_depth == 0)  // a single leaf: no level ran the last sums
            launch_b_finalize(bd_, 0, lp, scale, 0u, st_);
        if (qmode_ != GRAD_F32) {
            // leaves solved from the exact sums of the f32 gradients (+ values)
            launch_b_leaf_sums(bd_, R[0], R[1], exact_ref(o), lp, scales_.p + 4 * (size_t)o,
                               cap(n_ / B_LEAF_CHUNK + (1ull << cfg_.max_depth) + 1), st_);
            launches += 1;
        }
        if (renew_) {
            launch_leaf_renew(bd_, rd_, R[0], R[1], y_.p, pred, ds_.has_w ? w_.p : nullptr, quantile_alpha(o),
                              cfg_.learning_rate, g_wide, st_);
            launches += ds_.has_w ? 1 : 12;
        }
        launch_b_leaf_update(bd_, R[0], R[1], pred, cfg_.record_leaves ? row_leaf_.p : nullptr,
                             cap(n_ / B_LEAF_CHUNK + (1ull << cfg_.max_depth) + 1), st_);
        tm.end();
        launches += 2;
    }

    // Enqueues the tree of output o into ring slot `si` (no host wait).
    void launch_batched(uint32_t o, uint32_t si) {
        BST_RANGE("bst.tree");  // the tree's graph launch (its kernels run after the range closes)
        Slot& sl = slots_[si];
        const size_t gi = (size_t)o * RING + si;
        sl.timed = false;
        if (tuner_.active()) {
            bool timed = false;
            const uint32_t c = tuner_.next(&timed);
            apply_shape(tune_cands_[c]);
            sl.cand = c;
            sl.timed = timed;
        }
        if (!graphs_[gi]) {
            gtimers_[gi] = std::make_unique<Timer>();
            gtimers_[gi]->st = st_;
            gtimers_[gi]->enabled = cfg_.phase_timings != 0;
            gtimers_[gi]->reserve(16 + 20 * (size_t)cfg_.max_depth);
            gtimers_[gi]->in_graph = true;
            bd_.rmask = rowmask(o);  // baked into the graph's kernels
            BST_CK(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
            try {
                enqueue_tree(o, *gtimers_[gi], graph_launches_[gi], graph_hist_launches_[gi]);
            } catch (...) {
                cudaGraph_t g = nullptr;
                cudaStreamEndCapture(st_, &g);
                if (g) cudaGraphDestroy(g);
                throw;
            }
            cudaGraph_t g = nullptr;
            BST_CK(cudaStreamEndCapture(st_, &g));
            cudaGraphExec_t ex = nullptr;
            const cudaError_t e = cudaGraphInstantiate(&ex, g, 0);
            cudaGraphDestroy(g);
            BST_CK(e);
            graphs_[gi] = ex;
        }
        upload_col_masks(o, si);  // read by the graph's split searches
        if (rowsample_) {  // the root's split search counts the sampled rows
            const ScanNode rs{0, n_sampled_[o], 0u, 0u, 0, 0};
            BST_CK(cudaMemcpyAsync(d_root_scan_.p, &rs, sizeof(rs), cudaMemcpyHostToDevice, st_));
        }
        BST_CK(cudaEventRecord(sl.w0, st_));
        BST_CK(cudaGraphLaunch(graphs_[gi], st_));
        BST_CK(cudaEventRecord(sl.w1, st_));
        BST_CK(cudaMemcpyAsync(sl.state, d_bstate_.p, sizeof(BState), cudaMemcpyDeviceToHost, st_));
        BST_CK(cudaMemcpyAsync(sl.tree, d_btree_.p, sizeof(BTreeNode) * max_tnodes_, cudaMemcpyDeviceToHost, st_));
        if (cfg_.record_leaves) {
            sl.row_leaf.resize(n_);
            BST_CK(cudaMemcpyAsync(sl.row_leaf.data(), row_leaf_.p, sizeof(uint32_t) * n_, cudaMemcpyDeviceToHost,
                                   st_));
        }
        BST_CK(cudaEventRecord(sl.done, st_));
        sl.pending = true;
        sl.o = o;
    }

    // Waits for ring slot `si` and converts its device tree to a host tree.
    HostTree collect_batched(uint32_t si) {
        Slot& sl = slots_[si];
        const uint32_t o = sl.o;
        const size_t gi = (size_t)o * RING + si;
        BST_CK(cudaEventSynchronize(sl.done));
        BST_CK(cudaGetLastError());
        sl.pending = false;
        if (sl.timed) {
            float ms = 0.0f;
            BST_CK(cudaEventElapsedTime(&ms, sl.w0, sl.w1));
            tuner_.record(sl.cand, ms);
            sl.timed = false;
            finish_tuning();
        }
        HostTree t;
        t.group = o;
        t.row_leaf = std::move(sl.row_leaf);
        sl.row_leaf = {};
        Timer& gt = *gtimers_[gi];
        if (!gt.collect_keep()) {
            // per-phase timestamps unavailable: book the whole tree as "other"
            float ms = 0;
            BST_CK(cudaEventElapsedTime(&ms, sl.w0, sl.w1));
            timer_.acc[PH_OTHER] += ms;
        }
        for (int i = 1; i < 7; ++i) {
            timer_.acc[i] += gt.acc[i];
            gt.acc[i] = 0.0;
        }
        const BState* h_bstate_ = sl.state;
        const BTreeNode* h_btree_ = sl.tree;
        if (h_bstate_->err)
            throw Error{BST_ERR_CUDA, "a histogram kernel's bounded wait for its row copies gave up; the tree is invalid"};
        const uint64_t rows = h_bstate_->hist_rows;
        m_.counters.launches += graph_launches_[gi];
        m_.counters.hist_launches += graph_hist_launches_[gi];
        m_.counters.hist_rows += rows;
        m_.counters.hist_bytes += rows * ((uint64_t)p_.f8 + 2ull * p_.f16 + grad_bytes() + 4ull);
        m_.counters.scan_launches += graph_hist_launches_[gi];
        return host_tree_from(std::move(t), h_bstate_->n_tnodes, h_btree_);
    }

    // Host tree from a device tree (grower.rs:576-650 threshold translation);
    // t carries the tree's group and row leaves.
    HostTree host_tree_from(HostTree&& t, uint32_t nt, const BTreeNode* h_btree_) {
        cat_nodes_.clear();
        for (uint32_t i = 0; i < nt; ++i) t.alloc();
        for (uint32_t i = 0; i < nt; ++i) {
            const BTreeNode& b = h_btree_[i];
            t.grad_sum[i] = b.G;
            t.hess_sum[i] = b.H;
            t.cover[i] = to_f32(b.H);
            if (b.flags & 4u) {
                t.is_leaf[i] = 1;
                t.leaf[i] = b.leaf;
                continue;
            }
            const uint32_t feat = p_.col_feature[b.col];
            t.split_index[i] = feat;
            t.left[i] = b.left;
            t.right[i] = b.right;
            t.gain[i] = b.gain;
            if (!(b.flags & 2u)) {
                t.threshold[i] = next_up(to_f32(p_.mappers[feat].bin_to_value(b.bin)));
                t.default_left[i] = (b.flags & 1u) ? 1 : 0;
                t.split_type[i] = 0;
                t.split_bin[i] = b.bin;
            } else {
                t.threshold[i] = 0.0f;
                t.default_left[i] = (b.flags & 1u) ? 0 : 1;
                t.split_type[i] = 1;
                cat_nodes_.push_back({i, bitset_words(b.cats)});
            }
        }
        tree_ = std::move(t);
        freeze_categories();
        return std::move(tree_);
    }

    void build_tiles() {
        std::vector<LaneTile> lt;
        std::vector<uint8_t> rest;
        build_lane_tiles(p_, lane_tile_max_bins(qmode_), lt, lane_bins_, rest);
        n_lane_tiles_ = (uint32_t)lt.size();
        if (n_lane_tiles_) {
            lane_tiles_.alloc(n_lane_tiles_);
            BST_CK(cudaMemcpy(lane_tiles_.p, lt.data(), sizeof(LaneTile) * n_lane_tiles_, cudaMemcpyHostToDevice));
        }
        std::vector<HistTile> tiles;
        build_hist_tiles(p_, tiles, tile_smem_, &rest);
        n_tiles_ = (uint32_t)tiles.size();
        if (n_tiles_) {
            tiles_.alloc(n_tiles_);
            BST_CK(cudaMemcpy(tiles_.p, tiles.data(), sizeof(HistTile) * n_tiles_, cudaMemcpyHostToDevice));
        }
    }

    template <class T>
    T* upload(const T* host, size_t count, DevArray<T>& dst) {
        if (count == 0) return dst.p;
        if (count > dst.n) throw Error{BST_ERR_INVALID_ARGUMENT, "work list exceeds its device buffer"};
        BST_CK(cudaMemcpyAsync(dst.p, host, sizeof(T) * count, cudaMemcpyHostToDevice, st_));
        return dst.p;
    }

    // ---- histograms (host-driven loop) -------------------------------------------
    // Uploads a level state (expanding nodes with their smaller children)
    // and runs the device histogram pipeline on it.
    void host_hist(const std::vector<BExp>& exps, bool root) {
        uint64_t rows = 0;
        for (auto& e : exps) rows += e.small_count;
        const uint32_t CH = root ? chunk_rows(n_) : chunk_rows(rows);
        BExp* he = stage_.take<BExp>(exps.size());
        std::vector<uint32_t> segs;
        uint32_t nseg = 0;
        for (size_t j = 0; j < exps.size(); ++j) {
            he[j] = exps[j];
            he[j].hist_off = nseg;
            const uint32_t nch = (exps[j].small_count + CH - 1) / CH;
            for (uint32_t q = 0; q < nch; ++q) segs.push_back((uint32_t)j);
            nseg += nch;
        }
        if (nseg > d_seg_exp_.n) throw Error{BST_ERR_INVALID_ARGUMENT, "histogram segment list exceeds its buffer"};
        BState* hs = stage_.take<BState>(1);
        std::memset(hs, 0, sizeof(BState));
        hs->n_exp = (uint32_t)exps.size();
        hs->hist_chunks = nseg;
        hs->hist_chunk = CH;
        uint32_t* hseg = stage_.take<uint32_t>(std::max<size_t>(1, segs.size()));
        std::copy(segs.begin(), segs.end(), hseg);
        upload(he, exps.size(), d_bexp_);
        upload(hs, 1, d_bstate_);
        upload(hseg, segs.size(), d_seg_exp_);
        uint64_t launches = 0, hist_launches = 0;
        enqueue_hist(gr_o_, ridx_.p, root, timer_, launches, hist_launches, exps.size() <= WIDE_MERGE_NODES);
        m_.counters.launches += launches;
        m_.counters.hist_launches += hist_launches;
        m_.counters.hist_rows += rows;
        m_.counters.hist_bytes += rows * ((uint64_t)p_.f8 + 2ull * p_.f16 + grad_bytes() + 4ull);
    }

    // ---- split scan ---------------------------------------------------------------
    void scan(const std::vector<ScanNode>& nodes, std::vector<NodeSplit>& out) {
        out.resize(nodes.size());
        if (nodes.empty()) return;
        ScanNode* h = stage_.take<ScanNode>(nodes.size());
        std::copy(nodes.begin(), nodes.end(), h);
        upload(h, nodes.size(), d_scan_nodes_);
        timer_.begin(PH_SCAN);
        launch_split_scan(d_scan_nodes_.p, (uint32_t)nodes.size(), scan_cols_.p, n_cols_, hist_.p, slot_bins_,
                          scale_o_, gp_, d_cand_.p, d_node_tot_.p, st_, hist32_, colmask());
        launch_split_reduce(d_cand_.p, d_node_tot_.p, (uint32_t)nodes.size(), n_cols_, last_wins_ ? 1 : 0,
                            d_splits_.p, st_);
        timer_.end();
        m_.counters.launches += 2;
        m_.counters.scan_launches += 1;
        NodeSplit* hs = stage_.take<NodeSplit>(nodes.size());
        BST_CK(cudaMemcpyAsync(hs, d_splits_.p, sizeof(NodeSplit) * nodes.size(), cudaMemcpyDeviceToHost, st_));
        BST_CK(cudaStreamSynchronize(st_));
        std::copy(hs, hs + nodes.size(), out.begin());
    }

    // Exact fixed-point sums of the rows of each node (no histogram).
    void node_sums(const std::vector<PNode>& nodes, std::vector<std::pair<long long, long long>>& out) {
        node_sums(nodes, gr_o_, out);
    }
    void node_sums(const std::vector<PNode>& nodes, const GradRef& gr,
                   std::vector<std::pair<long long, long long>>& out) {
        out.assign(nodes.size(), {0, 0});
        if (nodes.empty()) return;
        std::vector<HistChunk> ch;
        for (uint32_t j = 0; j < nodes.size(); ++j)
            for (uint32_t s = 0; s < nodes[j].count; s += SUM_CHUNK_ROWS)
                ch.push_back(HistChunk{j, nodes[j].begin + s, std::min(SUM_CHUNK_ROWS, nodes[j].count - s), 0u});
        BST_CK(cudaMemsetAsync(d_sums_.p, 0, sizeof(long long) * 2 * nodes.size(), st_));
        if (!ch.empty()) {
            HistChunk* h = stage_.take<HistChunk>(ch.size());
            std::copy(ch.begin(), ch.end(), h);
            upload(h, ch.size(), d_schunks_);
            timer_.begin(PH_OTHER);
            launch_node_sums(d_schunks_.p, (uint32_t)ch.size(), ridx_.p, gr, d_sums_.p, st_);
            timer_.end();
            m_.counters.launches += 1;
        }
        long long* hs = stage_.take<long long>(2 * nodes.size());
        BST_CK(cudaMemcpyAsync(hs, d_sums_.p, sizeof(long long) * 2 * nodes.size(), cudaMemcpyDeviceToHost, st_));
        BST_CK(cudaStreamSynchronize(st_));
        for (size_t j = 0; j < nodes.size(); ++j) out[j] = {hs[2 * j], hs[2 * j + 1]};
    }

    // ---- tree bookkeeping (grower.rs:484-514, 576-650) -----------------------------
    void make_leaf(const Cand& c) {
        const double g = (double)c.G * inv_g_, h = (double)c.H * inv_h_;
        const float w = leaf_weight(g, h, cfg_);
        const float v = w * cfg_.learning_rate;  // apply_learning_rate (mutable_tree.rs:258)
        tree_.is_leaf[c.tree_node] = 1;
        tree_.leaf[c.tree_node] = v;
        tree_.cover[c.tree_node] = to_f32(h);
        tree_.grad_sum[c.tree_node] = g;
        tree_.hess_sum[c.tree_node] = h;
        if (c.node >= leaf_tree_node_.size()) {
            leaf_tree_node_.resize(c.node + 1, 0xFFFFFFFFu);
            leaf_value_.resize(c.node + 1, 0.0f);
        }
        leaf_tree_node_[c.node] = c.tree_node;
        leaf_value_[c.node] = v;
    }

    // returns (tree node of the training-left child, tree node of the training-right child)
    std::pair<uint32_t, uint32_t> apply_split(const Cand& c) {
        const NodeSplit& s = c.split;
        const uint32_t col = s.col;
        const uint32_t feat = p_.col_feature[col];
        const Mapper& m = p_.mappers[feat];
        const uint32_t nd = c.tree_node;
        const double g = (double)c.G * inv_g_, h = (double)c.H * inv_h_;
        tree_.gain[nd] = s.gain;
        tree_.cover[nd] = to_f32(h);
        tree_.grad_sum[nd] = g;
        tree_.hess_sum[nd] = h;
        const uint32_t l = tree_.alloc(), r = tree_.alloc();
        tree_.split_index[nd] = feat;
        tree_.left[nd] = l;
        tree_.right[nd] = r;
        tree_.is_leaf[nd] = 0;
        const bool dl = s.flags & 1u;
        if (!(s.flags & 2u)) {
            tree_.threshold[nd] = next_up(to_f32(m.bin_to_value(s.bin)));
            tree_.default_left[nd] = dl;
            tree_.split_type[nd] = 0;
            tree_.split_bin[nd] = s.bin;
            return {l, r};
        }
        // categorical: stored bitset = categories going right at inference,
        // children swapped and default inverted (grower.rs:612-647)
        tree_.threshold[nd] = 0.0f;
        tree_.default_left[nd] = dl ? 0 : 1;
        tree_.split_type[nd] = 1;
        cat_nodes_.push_back({nd, bitset_words(s.cats)});
        return {r, l};
    }

    std::vector<std::pair<uint32_t, std::vector<uint32_t>>> cat_nodes_;

    void freeze_categories() {  // mutable_tree.rs:299-335
        const size_t nn = tree_.split_index.size();
        tree_.seg_start.assign(nn, 0);
        tree_.seg_size.assign(nn, 0);
        tree_.cat_words.clear();
        std::sort(cat_nodes_.begin(), cat_nodes_.end(),
                  [](const auto& a, const auto& b) { return a.first < b.first; });
        for (auto& cn : cat_nodes_) {
            tree_.seg_start[cn.first] = (uint32_t)tree_.cat_words.size();
            tree_.seg_size[cn.first] = (uint32_t)cn.second.size();
            tree_.cat_words.insert(tree_.cat_words.end(), cn.second.begin(), cn.second.end());
        }
        cat_nodes_.clear();
    }

    static bool expands(const Cand& c, float min_gain) {  // grower.rs:530-539
        const bool valid = (c.split.flags & 4u) && c.split.gain > -std::numeric_limits<float>::infinity();
        return valid && !(c.split.gain <= min_gain);
    }

    // Splits every parent in `par` (already accepted): partition, child
    // histograms (smaller child built, larger by subtraction) and child splits.
    void expand(std::vector<Cand>& par, const std::vector<std::pair<uint32_t, uint32_t>>& tree_children,
                const std::vector<uint32_t>& right_ids, bool need_split, std::vector<Cand>& children) {
        const size_t k = par.size();
        stage_.reset();
        // 1. partition (partition.rs:296-382)
        std::vector<PartChunk> pch;
        PartWork* pw = stage_.take<PartWork>(k);
        unsigned* cur = stage_.take<unsigned>(2 * k);
        uint64_t prow = 0;
        for (size_t j = 0; j < k; ++j) {
            const Cand& c = par[j];
            const PNode& pn = pn_[c.node];
            const uint32_t col = c.split.col;
            PartWork w;
            std::memset(&w, 0, sizeof(w));
            w.begin = pn.begin;
            w.count = pn.count;
            w.matrix = p_.col_matrix[col];
            w.pos = p_.col_pos[col];
            w.thr_bin = c.split.bin;
            w.flags = (c.split.flags & 1u) | (p_.col_missing[col] ? 2u : 0u) | ((c.split.flags & 2u) ? 4u : 0u);
            w.default_bin = p_.col_default[col];
            for (int q = 0; q < 4; ++q) w.cats[q] = c.split.cats[q];
            pw[j] = w;
            cur[2 * j] = pn.begin;
            cur[2 * j + 1] = pn.begin + pn.count;
            for (uint32_t s = 0; s < pn.count; s += PART_CHUNK_ROWS)
                pch.push_back(PartChunk{(uint32_t)j, pn.begin + s, std::min(PART_CHUNK_ROWS, pn.count - s), 0});
            prow += pn.count;
        }
        upload(pw, k, d_pworks_);
        upload(cur, 2 * k, d_cursors_);
        PartChunk* hpc = stage_.take<PartChunk>(std::max<size_t>(1, pch.size()));
        std::copy(pch.begin(), pch.end(), hpc);
        upload(hpc, pch.size(), d_pchunks_);
        timer_.begin(PH_PART);
        if (rowsample_) BST_CK(cudaMemsetAsync(d_scnt_.p, 0, sizeof(unsigned) * 2 * k, st_));
        if (spec_leafwise_) {
            launch_partition(d_pworks_.p, d_pchunks_.p, (uint32_t)pch.size(), ridx_.p, tmp_.p, d_cursors_.p,
                             b_.bins8, p_.s8, b_.bins16, p_.s16, st_, qpos_[0].p, qpos_[1].p, qmode_, fm_,
                             rowmask(tree_output_), d_scnt_.p);
            launch_copy_chunks(d_pchunks_.p, d_pworks_.p, (uint32_t)pch.size(), tmp_.p, ridx_.p, st_, qpos_[1].p,
                               qpos_[0].p, qmode_);
        } else {
            launch_partition(d_pworks_.p, d_pchunks_.p, (uint32_t)pch.size(), ridx_.p, tmp_.p, d_cursors_.p,
                             b_.bins8, p_.s8, b_.bins16, p_.s16, st_, nullptr, nullptr, 0, BinsFM{},
                             rowmask(tree_output_), d_scnt_.p);
            launch_copy_chunks(d_pchunks_.p, d_pworks_.p, (uint32_t)pch.size(), tmp_.p, ridx_.p, st_);
        }
        timer_.end();
        m_.counters.launches += pch.empty() ? 0 : 2;
        m_.counters.partition_rows += prow;
        if (spec_leafwise_ && need_split && n_cols_ > 0) {
            expand_children_on_device(par, tree_children, right_ids, children);
            return;
        }
        unsigned* hc = stage_.take<unsigned>(2 * k);
        unsigned* hsc = stage_.take<unsigned>(2 * k);
        BST_CK(cudaMemcpyAsync(hc, d_cursors_.p, sizeof(unsigned) * 2 * k, cudaMemcpyDeviceToHost, st_));
        if (rowsample_)
            BST_CK(cudaMemcpyAsync(hsc, d_scnt_.p, sizeof(unsigned) * 2 * k, cudaMemcpyDeviceToHost, st_));
        BST_CK(cudaStreamSynchronize(st_));
        std::vector<uint32_t> lc(k), rc(k);
        for (size_t j = 0; j < k; ++j) {
            const PNode pn = pn_[par[j].node];
            lc[j] = hc[2 * j] - pn.begin;
            rc[j] = pn.count - lc[j];
            pn_[par[j].node] = PNode{pn.begin, lc[j]};
            pn_[right_ids[j]] = PNode{pn.begin + lc[j], rc[j]};
        }
        stage_.reset();
        children.clear();
        children.reserve(2 * k);
        if (need_split && n_cols_ > 0) {
            // 2. smaller child into the right slot, then subtract (pool.rs:414-432)
            if (n_tiles_) {  // general tiles add atomically into zeroed right slots
                const uint32_t r_lo = *std::min_element(right_ids.begin(), right_ids.end());
                const uint32_t r_hi = *std::max_element(right_ids.begin(), right_ids.end());
                BST_CK(cudaMemsetAsync(reinterpret_cast<char*>(hist_.p) + (size_t)r_lo * slot_bins_ * hbytes(), 0,
                                       hbytes() * slot_bins_ * (size_t)(r_hi - r_lo + 1), st_));
            }
            std::vector<BExp> exps(k);
            for (size_t j = 0; j < k; ++j) {
                const bool left_small = lc[j] <= rc[j];  // grower.rs:398-402
                const uint32_t small = left_small ? par[j].node : right_ids[j];
                BExp e;
                std::memset(&e, 0, sizeof(e));
                e.left_pnode = par[j].node;
                e.right_pnode = right_ids[j];
                e.lc = lc[j];
                e.rc = rc[j];
                e.small_begin = pn_[small].begin;
                e.small_count = pn_[small].count;
                exps[j] = e;
            }
            host_hist(exps, false);
            // 3. child splits (left, right per parent)
            std::vector<ScanNode> sn;
            sn.reserve(2 * k);
            for (size_t j = 0; j < k; ++j) {  // pad: the children's depth (column masks); counts: sampled rows
                sn.push_back(ScanNode{par[j].node, rowsample_ ? hsc[2 * j] : lc[j], 0u, par[j].depth + 1, 0, 0});
                sn.push_back(ScanNode{right_ids[j], rowsample_ ? hsc[2 * j + 1] : rc[j], 0u, par[j].depth + 1, 0, 0});
            }
            std::vector<NodeSplit> res;
            scan(sn, res);
            for (size_t j = 0; j < k; ++j) {
                const uint32_t d = par[j].depth + 1;
                children.push_back(Cand{par[j].node, tree_children[j].first, d, res[2 * j], res[2 * j].tot_g,
                                        res[2 * j].tot_h, lc[j]});
                children.push_back(Cand{right_ids[j], tree_children[j].second, d, res[2 * j + 1],
                                        res[2 * j + 1].tot_g, res[2 * j + 1].tot_h, rc[j]});
            }
        } else {
            // children will not be split: only their sums are needed
            std::vector<PNode> smalls(k);
            for (size_t j = 0; j < k; ++j)
                smalls[j] = lc[j] <= rc[j] ? pn_[par[j].node] : pn_[right_ids[j]];
            std::vector<std::pair<long long, long long>> sums;
            node_sums(smalls, sums);
            for (size_t j = 0; j < k; ++j) {
                const bool left_small = lc[j] <= rc[j];
                const long long sg = sums[j].first, sh = sums[j].second;
                const long long lg = left_small ? sg : par[j].G - sg, lh = left_small ? sh : par[j].H - sh;
                const long long rg = par[j].G - lg, rh = par[j].H - lh;
                NodeSplit inv;
                std::memset(&inv, 0, sizeof(inv));
                inv.gain = -std::numeric_limits<float>::infinity();
                const uint32_t d = par[j].depth + 1;
                children.push_back(Cand{par[j].node, tree_children[j].first, d, inv, lg, lh, lc[j]});
                children.push_back(Cand{right_ids[j], tree_children[j].second, d, inv, rg, rh, rc[j]});
            }
        }
    }

    // Batched leaf-wise, after expand()'s partition: the children's counts,
    // smaller children and histogram segments come from the partition's
    // cursors on the device (k_lw_children), so the histograms and the
    // children's split search follow the partition directly; one read-back
    // (the children's splits and the cursors) per expansion batch.
    void expand_children_on_device(const std::vector<Cand>& par,
                                   const std::vector<std::pair<uint32_t, uint32_t>>& tree_children,
                                   const std::vector<uint32_t>& right_ids, std::vector<Cand>& children) {
        const size_t k = par.size();
        if (n_tiles_) {  // general tiles add atomically into zeroed right slots
            const uint32_t r_lo = *std::min_element(right_ids.begin(), right_ids.end());
            const uint32_t r_hi = *std::max_element(right_ids.begin(), right_ids.end());
            BST_CK(cudaMemsetAsync(reinterpret_cast<char*>(hist_.p) + (size_t)r_lo * slot_bins_ * hbytes(), 0,
                                   hbytes() * slot_bins_ * (size_t)(r_hi - r_lo + 1), st_));
        }
        BExp* he = stage_.take<BExp>(k);
        std::memset(he, 0, sizeof(BExp) * k);
        for (size_t j = 0; j < k; ++j) {
            he[j].left_pnode = par[j].node;
            he[j].right_pnode = right_ids[j];
            he[j].pad1 = par[j].depth + 1;  // the children's depth (column masks)
        }
        upload(he, k, d_bexp_);
        launch_lw_children(bd_, d_pworks_.p, d_cursors_.p, (uint32_t)k, d_scan_nodes_.p,
                           rowsample_ ? d_scnt_.p : nullptr, st_);
        uint64_t launches = 1, hist_launches = 0;
        enqueue_hist(gr_o_, ridx_.p, false, timer_, launches, hist_launches, k <= WIDE_MERGE_NODES);
        timer_.begin(PH_SCAN);
        launch_split_scan(d_scan_nodes_.p, (uint32_t)(2 * k), scan_cols_.p, n_cols_, hist_.p, slot_bins_, scale_o_, gp_,
                          d_cand_.p, d_node_tot_.p, st_, hist32_, colmask());
        launch_split_reduce(d_cand_.p, d_node_tot_.p, (uint32_t)(2 * k), n_cols_, last_wins_ ? 1 : 0, d_splits_.p, st_);
        timer_.end();
        NodeSplit* hs = stage_.take<NodeSplit>(2 * k);
        unsigned* hc = stage_.take<unsigned>(2 * k);
        BST_CK(cudaMemcpyAsync(hs, d_splits_.p, sizeof(NodeSplit) * 2 * k, cudaMemcpyDeviceToHost, st_));
        BST_CK(cudaMemcpyAsync(hc, d_cursors_.p, sizeof(unsigned) * 2 * k, cudaMemcpyDeviceToHost, st_));
        BST_CK(cudaStreamSynchronize(st_));
        m_.counters.launches += launches + 2;
        m_.counters.hist_launches += hist_launches;
        m_.counters.scan_launches += 1;
        children.clear();
        children.reserve(2 * k);
        uint64_t rows = 0;
        for (size_t j = 0; j < k; ++j) {
            const PNode pn = pn_[par[j].node];
            const uint32_t lc = hc[2 * j] - pn.begin, rc = pn.count - lc;
            pn_[par[j].node] = PNode{pn.begin, lc};
            pn_[right_ids[j]] = PNode{pn.begin + lc, rc};
            rows += std::min(lc, rc);
            const uint32_t d = par[j].depth + 1;
            children.push_back(Cand{par[j].node, tree_children[j].first, d, hs[2 * j], hs[2 * j].tot_g,
                                    hs[2 * j].tot_h, lc});
            children.push_back(Cand{right_ids[j], tree_children[j].second, d, hs[2 * j + 1], hs[2 * j + 1].tot_g,
                                    hs[2 * j + 1].tot_h, rc});
        }
        m_.counters.hist_rows += rows;
        m_.counters.hist_bytes += rows * ((uint64_t)p_.f8 + 2ull * p_.f16 + grad_bytes() + 4ull);
        stage_.reset();
    }

    // Quantised training: re-solve every leaf from the exact fixed-point sums
    // of its f32 gradients (the histogram sums only chose the splits).
    void exact_leaves(uint32_t o) {
        stage_.reset();  // every earlier staged copy has completed (node_sums / scan synchronise)
        std::vector<PNode> nodes;
        std::vector<uint32_t> ids;
        for (uint32_t pnode = 0; pnode < n_pnodes_; ++pnode)
            if (leaf_tree_node_[pnode] != 0xFFFFFFFFu) {
                nodes.push_back(pn_[pnode]);
                ids.push_back(pnode);
            }
        std::vector<std::pair<long long, long long>> sums;
        node_sums(nodes, gx_o_, sums);
        const double ig = h_scales_[4 * o + 2], ih = h_scales_[4 * o + 3];
        for (size_t j = 0; j < ids.size(); ++j) {
            const double g = (double)sums[j].first * ig, h = (double)sums[j].second * ih;
            const float v = leaf_weight(g, h, cfg_) * cfg_.learning_rate;
            const uint32_t tn = leaf_tree_node_[ids[j]];
            tree_.leaf[tn] = v;
            tree_.cover[tn] = to_f32(h);
            tree_.grad_sum[tn] = g;
            tree_.hess_sum[tn] = h;
            leaf_value_[ids[j]] = v;
        }
    }

    // Leaf-wise growth (expansion.rs:137-166): pop the leaf of largest
    // (gain, node id), split it, push its children, until max_leaves.
    //
    // The pops are replayed here exactly. Plain form: the device expands
    // each popped node on its own (the reference's order of work). Batched
    // form: when the popped node has not been expanded yet, it is expanded
    // together with the best other unexpanded candidates of the heap (at
    // most as many as pops remain). A node's rows, histogram and
    // split do not depend on when it is expanded, so a node that the replay
    // pops later costs no device step, and one it never pops is rolled back
    // into a leaf over its full row range. Node ids of the replay (the tie
    // rule's "node id": left child keeps the parent's, right child takes the
    // next) are tracked apart from the histogram slots, which are allocated
    // in batch order; the slot pool holds 2 * max_leaves so that speculation
    // never starves the remaining pops.
    struct Spec {
        Cand kids[2];
        uint32_t right_pnode, begin, count;
    };
    void grow_leafwise(const Cand& root, float min_gain) {
        struct HeapEnt {
            Cand c;
            uint32_t vid;
        };
        std::vector<HeapEnt> heap{{root, 0u}};
        std::unordered_map<uint32_t, Spec> spec;  // expanded, not yet popped (key: pnode)
        uint32_t n_leaves = 1, n_vid = 1;
        auto before = [](const HeapEnt& a, const HeapEnt& b) {  // a pops before b
            return a.c.split.gain > b.c.split.gain || (a.c.split.gain == b.c.split.gain && a.vid > b.vid);
        };
        auto pop = [&]() {
            size_t bi = 0;
            for (size_t i = 1; i < heap.size(); ++i)
                if (before(heap[i], heap[bi])) bi = i;
            HeapEnt e = heap[bi];
            heap.erase(heap.begin() + bi);
            return e;
        };
        while (n_leaves < cfg_.max_leaves && !heap.empty()) {
            HeapEnt e = pop();
            n_leaves += 1;
            if (!expands(e.c, min_gain)) {
                make_leaf(e.c);
                continue;
            }
            if (!spec.count(e.c.node)) {
                // slots: each later pop needs at most one more, so a batch
                // leaves >= rem free; with rem shrinking by one per pop there
                // is always room for at least this node
                const uint32_t rem = cfg_.max_leaves - n_leaves;  // pops that may follow
                const int64_t room = (int64_t)max_pnodes_ - (int64_t)n_pnodes_ - (int64_t)rem;
                if (room < 1) throw Error{BST_ERR_OUT_OF_MEMORY, "leaf-wise growth ran out of histogram slots"};
                const uint64_t batch = spec_leafwise_ ? std::min<uint64_t>((uint64_t)rem + 1, (uint64_t)room) : 1u;
                std::vector<HeapEnt> more;
                for (const HeapEnt& h : heap)
                    if (expands(h.c, min_gain) && !spec.count(h.c.node)) more.push_back(h);
                const size_t extra = std::min<size_t>(more.size(), (size_t)batch - 1);
                std::partial_sort(more.begin(), more.begin() + extra, more.end(), before);
                std::vector<Cand> par{e.c}, kids;
                for (size_t i = 0; i < extra; ++i) par.push_back(more[i].c);
                std::vector<std::pair<uint32_t, uint32_t>> tch(par.size(), {0xFFFFFFFFu, 0xFFFFFFFFu});
                std::vector<uint32_t> rid(par.size());
                std::vector<PNode> before_split(par.size());
                for (size_t j = 0; j < par.size(); ++j) {
                    rid[j] = n_pnodes_++;
                    before_split[j] = pn_[par[j].node];
                }
                expand(par, tch, rid, n_leaves < cfg_.max_leaves, kids);
                for (size_t j = 0; j < par.size(); ++j)
                    spec[par[j].node] = Spec{{kids[2 * j], kids[2 * j + 1]}, rid[j], before_split[j].begin,
                                             before_split[j].count};
            }
            auto it = spec.find(e.c.node);
            Spec sp = it->second;
            spec.erase(it);
            const std::pair<uint32_t, uint32_t> tch = apply_split(e.c);
            sp.kids[0].tree_node = tch.first;
            sp.kids[1].tree_node = tch.second;
            heap.push_back({sp.kids[0], e.vid});
            heap.push_back({sp.kids[1], n_vid++});
        }
        while (!heap.empty()) {
            const HeapEnt e = pop();
            auto it = spec.find(e.c.node);
            if (it != spec.end()) {  // expanded but never popped: one leaf over both children's rows
                pn_[e.c.node] = PNode{it->second.begin, it->second.count};
                pn_[it->second.right_pnode] = PNode{it->second.begin + it->second.count, 0u};
                spec.erase(it);
            }
            make_leaf(e.c);
        }
    }

    // ---- batched leaf-wise growth on the device (kernels.h, k_lw_replay) -----
    // The replay of the heap pops runs on the device between expansion
    // steps; the host launches LW_STEPS steps at a time as one CUDA graph and
    // reads back only whether the tree is done.
    static constexpr uint32_t LW_STEPS = 6;
    DevArray<LwState> d_lw_state_;
    DevArray<LwCand> d_lw_heap_;
    DevArray<LwSpec> d_lw_spec_;
    DevArray<uint2> d_lw_pn_;
    DevArray<NodeSplit> d_lw_child_;
    DevArray<unsigned long long> d_lw_keys_;
    DevArray<uint32_t> d_lw_ranks_;
    LwDev lw_{};
    LwState* h_lw_state_ = nullptr;  // pinned
    BState* h_lw_bstate_ = nullptr;  // pinned
    std::vector<cudaGraphExec_t> lw_graphs_;  // [output]
    std::vector<uint64_t> lw_launches_, lw_hist_launches_;
    std::vector<std::unique_ptr<Timer>> lw_timers_;  // [output]: event nodes of the step graphs

    void setup_lw_device() {
        init_kernel_attributes();
        const uint32_t mp = max_pnodes_;
        d_lw_state_.alloc(1);
        d_lw_heap_.alloc(2 * (size_t)cfg_.max_leaves + 4);
        d_lw_spec_.alloc(mp);
        d_lw_pn_.alloc(mp);
        d_lw_child_.alloc(2 * (size_t)mp + 2);
        d_lw_keys_.alloc(d_lw_heap_.n);
        d_lw_ranks_.alloc(2 * d_lw_heap_.n);
        lw_.keys = d_lw_keys_.p;
        lw_.ranks = d_lw_ranks_.p;
        lw_.st = d_lw_state_.p;
        lw_.heap = d_lw_heap_.p;
        lw_.spec = d_lw_spec_.p;
        lw_.pn = d_lw_pn_.p;
        lw_.child = d_lw_child_.p;
        lw_.heap_cap = (uint32_t)d_lw_heap_.n;
        lw_.max_pnodes = mp;
        lw_.max_leaves = cfg_.max_leaves;
        lw_.min_gain = cfg_.min_gain;
        // the device tree, its leaves and the columns' partition facts
        d_btree_.alloc(2 * (size_t)mp);
        d_bleaves_.alloc((size_t)mp + 1);
        d_node_key_.alloc(2 * (size_t)mp + 2);
        BST_CK(cudaMemset(d_node_key_.p, 0, sizeof(unsigned long long) * d_node_key_.n));
        std::vector<BColumn> bc(n_cols_);
        for (uint32_t c = 0; c < n_cols_; ++c)
            bc[c] = BColumn{p_.col_matrix[c], p_.col_pos[c], p_.col_missing[c], p_.col_default[c]};
        d_bcols_.alloc(n_cols_);
        BST_CK(cudaMemcpy(d_bcols_.p, bc.data(), sizeof(BColumn) * n_cols_, cudaMemcpyHostToDevice));
        bd_.tree = d_btree_.p;
        bd_.leaves = d_bleaves_.p;
        bd_.bcols = d_bcols_.p;
        bd_.node_key = d_node_key_.p;
        bd_.pworks = d_pworks_.p;
        bd_.cursors = d_cursors_.p;
        bd_.scan_nodes = d_scan_nodes_.p;
        bd_.sums = d_sums_.p;
        bd_.scnt = rowsample_ ? d_scnt_.p : nullptr;
        bd_.max_front = mp;
        bd_.max_tnodes = (uint32_t)d_btree_.n;
        if (!h_lw_state_) h_lw_state_ = static_cast<LwState*>(pinned_alloc(sizeof(LwState)));
        if (!h_lw_bstate_) h_lw_bstate_ = static_cast<BState*>(pinned_alloc(sizeof(BState)));
        lw_graphs_.assign(G_, nullptr);
        lw_launches_.assign(G_, 0);
        lw_hist_launches_.assign(G_, 0);
        lw_timers_.resize(G_);
        for (auto& t : lw_timers_) {
            t = std::make_unique<Timer>();
            t->st = st_;
            t->enabled = cfg_.phase_timings != 0;
            t->in_graph = true;
            t->reserve(LW_STEPS * 12 + 4);
        }
    }

    void free_lw_device() {
        for (auto g : lw_graphs_)
            if (g) cudaGraphExecDestroy(g);
        lw_graphs_.clear();
        pinned_free(h_lw_state_);
        pinned_free(h_lw_bstate_);
        h_lw_state_ = nullptr;
        h_lw_bstate_ = nullptr;
    }

    // LW_STEPS expansion steps of output o's tree: replay, partition (rows
    // copied back into the one row buffer), children and histogram segments,
    // histograms with the subtraction trick, the children's split search.
    void enqueue_lw_steps(uint32_t o, Timer& tm, uint64_t& launches, uint64_t& hist_launches) {
        LeafParams lp{(double)cfg_.lambda, (double)cfg_.alpha, (double)cfg_.min_gain, cfg_.learning_rate, 0u};
        GradRef gr = grad_ref(o);
        gr.qpos = qpos_[0].p;
        const double* scale = unit_scale(o);
        launches = 0;
        hist_launches = 0;
        for (uint32_t k = 0; k < LW_STEPS; ++k) {
            tm.begin(PH_OTHER);
            launch_lw_replay(bd_, lw_, lp, scale, st_);
            tm.end();
            tm.begin(PH_PART);
            launch_lw_partition(bd_, ridx_.p, tmp_.p, b_.bins8, p_.s8, b_.bins16, p_.s16, g_wide_, qpos_[0].p,
                                qpos_[1].p, qmode_, fm_, st_);
            tm.end();
            tm.begin(PH_OTHER);
            launch_lw_children(bd_, d_pworks_.p, d_cursors_.p, LW_K_FROM_STATE, d_scan_nodes_.p,
                               rowsample_ ? d_scnt_.p : nullptr, st_);
            if (n_tiles_) launch_b_zero_right(bd_, hist_.p, slot_bins_, g_wide_, st_, hist32_);
            tm.end();
            enqueue_hist(gr, ridx_.p, false, tm, launches, hist_launches, false);
            tm.begin(PH_SCAN);
            launch_b_scan(bd_, scan_cols_.p, n_cols_, hist_.p, slot_bins_, scale, gp_, d_cand_.p, d_node_tot_.p, 0,
                          last_wins_ ? 1 : 0, lp, 0u, g_wide_, st_, hist32_, nullptr, colmask(), lw_.child);
            tm.end();
            launches += 5 + (n_tiles_ ? 1 : 0);  // + replay, partition, copy-back, children, scan
        }
    }

    HostTree grow_lw_device(uint32_t o) {
        tree_output_ = o;
        gr_o_ = grad_ref(o);
        gr_o_.qpos = qpos_[0].p;  // histograms read the positional copy
        scale_o_ = unit_scale(o);
        bd_.rmask = rowmask(o);
        stage_.reset();
        timer_.begin(PH_OTHER);
        upload_col_masks(o, 0);
        launch_iota(ridx_.p, n_, st_);
        // identity order: the positional copy is the row-order array
        BST_CK(cudaMemcpyAsync(qpos_[0].p, qmode_ == GRAD_F32 ? (const void*)gr_o_.gh : gr_o_.gq,
                               (size_t)n_ * grad_bytes(), cudaMemcpyDeviceToDevice, st_));
        BST_CK(cudaMemsetAsync(d_lw_spec_.p, 0, sizeof(LwSpec) * d_lw_spec_.n, st_));
        timer_.end();
        // the root's histogram and split (grower.rs:288-308)
        if (n_tiles_) BST_CK(cudaMemsetAsync(hist_.p, 0, hbytes() * slot_bins_, st_));
        BExp e;
        std::memset(&e, 0, sizeof(e));
        e.rc = (uint32_t)n_;
        e.small_count = (uint32_t)n_;
        host_hist({e}, true);
        ScanNode* rs = stage_.take<ScanNode>(1);
        *rs = ScanNode{0, n_sampled_[o], 0u, 0u, 0, 0};  // sampled rows under row sampling
        upload(rs, 1, d_scan_nodes_);
        timer_.begin(PH_SCAN);
        launch_split_scan(d_scan_nodes_.p, 1, scan_cols_.p, n_cols_, hist_.p, slot_bins_, scale_o_, gp_, d_cand_.p,
                          d_node_tot_.p, st_, hist32_, colmask());
        launch_split_reduce(d_cand_.p, d_node_tot_.p, 1, n_cols_, last_wins_ ? 1 : 0, lw_.child, st_);
        timer_.end();
        launch_lw_init(bd_, lw_, (uint32_t)n_, (uint32_t)n_, st_);
        m_.counters.launches += 5;
        // expansion steps, LW_STEPS per graph launch, until the replay is done
        if (!lw_graphs_[o]) {
            BST_CK(cudaStreamBeginCapture(st_, cudaStreamCaptureModeThreadLocal));
            try {
                enqueue_lw_steps(o, *lw_timers_[o], lw_launches_[o], lw_hist_launches_[o]);
            } catch (...) {
                cudaGraph_t g = nullptr;
                cudaStreamEndCapture(st_, &g);
                if (g) cudaGraphDestroy(g);
                throw;
            }
            cudaGraph_t g = nullptr;
            BST_CK(cudaStreamEndCapture(st_, &g));
            cudaGraphExec_t ex = nullptr;
            const cudaError_t ce = cudaGraphInstantiate(&ex, g, 0);
            cudaGraphDestroy(g);
            BST_CK(ce);
            lw_graphs_[o] = ex;
        }
        // each step but the last pops at least one leaf
        const uint32_t max_launches = cfg_.max_leaves / LW_STEPS + 4;
        Timer& gt = *lw_timers_[o];
        for (uint32_t it = 0;; ++it) {
            if (it > max_launches) throw Error{BST_ERR_CUDA, "leaf-wise replay did not finish"};
            BST_CK(cudaGraphLaunch(lw_graphs_[o], st_));
            BST_CK(cudaMemcpyAsync(h_lw_state_, d_lw_state_.p, sizeof(LwState), cudaMemcpyDeviceToHost, st_));
            BST_CK(cudaStreamSynchronize(st_));
            if (gt.enabled && gt.collect_keep())
                for (int i = 1; i < 7; ++i) {
                    timer_.acc[i] += gt.acc[i];
                    gt.acc[i] = 0.0;
                }
            m_.counters.launches += lw_launches_[o];
            m_.counters.hist_launches += lw_hist_launches_[o];
            m_.counters.scan_launches += LW_STEPS;
            if (h_lw_state_->err) throw Error{BST_ERR_OUT_OF_MEMORY, "leaf-wise growth ran out of histogram slots"};
            if (h_lw_state_->done) break;
        }
        // leaves: values (quantised forms: from the exact sums of the f32
        // gradients), then the predictions of their rows (grower.rs:208-219)
        LeafParams lp{(double)cfg_.lambda, (double)cfg_.alpha, (double)cfg_.min_gain, cfg_.learning_rate, 0u};
        float* pred = pred_.p + (size_t)o * n_;
        timer_.begin(PH_LEAF);
        launch_lw_leaves(bd_, st_);
        if (qmode_ != GRAD_F32)
            launch_b_leaf_sums(bd_, ridx_.p, ridx_.p, exact_ref(o), lp, scales_.p + 4 * (size_t)o, g_wide_, st_);
        if (renew_) {
            launch_leaf_renew(bd_, rd_, ridx_.p, ridx_.p, y_.p, pred, ds_.has_w ? w_.p : nullptr, quantile_alpha(o),
                              cfg_.learning_rate, g_wide_, st_);
            m_.counters.launches += ds_.has_w ? 1 : 12;
        }
        launch_b_leaf_update(bd_, ridx_.p, ridx_.p, pred, cfg_.record_leaves ? row_leaf_.p : nullptr, g_wide_, st_);
        timer_.end();
        m_.counters.launches += qmode_ != GRAD_F32 ? 3 : 2;
        BST_CK(cudaMemcpyAsync(h_lw_bstate_, d_bstate_.p, sizeof(BState), cudaMemcpyDeviceToHost, st_));
        BST_CK(cudaStreamSynchronize(st_));
        const uint32_t nt = h_lw_bstate_->n_tnodes;
        if (nt == 0 || nt > d_btree_.n) throw Error{BST_ERR_CUDA, "device tree has an invalid node count"};
        std::vector<BTreeNode> bt(nt);
        BST_CK(cudaMemcpyAsync(bt.data(), d_btree_.p, sizeof(BTreeNode) * nt, cudaMemcpyDeviceToHost, st_));
        HostTree t;
        t.group = o;
        if (cfg_.record_leaves) {
            t.row_leaf.resize(n_);
            BST_CK(cudaMemcpyAsync(t.row_leaf.data(), row_leaf_.p, sizeof(uint32_t) * n_, cudaMemcpyDeviceToHost, st_));
        }
        BST_CK(cudaStreamSynchronize(st_));
        BST_CK(cudaGetLastError());
        m_.counters.hist_rows += h_lw_bstate_->hist_rows;
        m_.counters.hist_bytes += h_lw_bstate_->hist_rows * ((uint64_t)p_.f8 + 2ull * p_.f16 + grad_bytes() + 4ull);
        timer_.collect();
        return host_tree_from(std::move(t), nt, bt.data());
    }

    HostTree grow(uint32_t o) {
        BST_RANGE("bst.tree");
        if (spec_leafwise_) return grow_lw_device(o);
        tree_output_ = o;
        gr_o_ = grad_ref(o);
        if (spec_leafwise_) gr_o_.qpos = qpos_[0].p;  // histograms read the positional copy
        gx_o_ = exact_ref(o);
        scale_o_ = unit_scale(o);
        const std::vector<double>& hs = qmode_ == GRAD_F32 ? h_scales_ : h_qscales_;
        inv_g_ = hs[4 * o + 2];
        inv_h_ = hs[4 * o + 3];
        tree_ = HostTree();
        cat_nodes_.clear();
        leaf_tree_node_.assign(max_pnodes_, 0xFFFFFFFFu);
        leaf_value_.assign(max_pnodes_, 0.0f);
        pn_.assign(max_pnodes_ + 1, PNode{});
        pn_[0] = PNode{0, (uint32_t)n_};
        n_pnodes_ = 1;
        stage_.reset();
        timer_.begin(PH_OTHER);
        upload_col_masks(o, 0);
        launch_iota(ridx_.p, n_, st_);
        if (spec_leafwise_)  // identity order: the positional copy is the row-order array
            BST_CK(cudaMemcpyAsync(qpos_[0].p, qmode_ == GRAD_F32 ? (const void*)gr_o_.gh : gr_o_.gq,
                                   (size_t)n_ * grad_bytes(), cudaMemcpyDeviceToDevice, st_));
        timer_.end();
        m_.counters.launches += 1;
        tree_.alloc();  // root (mutable_tree.rs:80 init_root)

        // root histogram, sums and split (grower.rs:288-308)
        Cand root;
        root.node = 0;
        root.tree_node = 0;
        root.depth = 0;
        root.count = (uint32_t)n_;
        if (n_cols_ > 0) {
            if (n_tiles_) BST_CK(cudaMemsetAsync(hist_.p, 0, hbytes() * slot_bins_, st_));
            BExp e;
            std::memset(&e, 0, sizeof(e));
            e.rc = (uint32_t)n_;
            e.small_count = (uint32_t)n_;
            host_hist({e}, true);
            std::vector<NodeSplit> res;
            scan({ScanNode{0, n_sampled_[o], 0u, 0u, 0, 0}}, res);  // sampled rows under row sampling
            root.split = res[0];
            root.G = res[0].tot_g;
            root.H = res[0].tot_h;
        } else {
            std::vector<std::pair<long long, long long>> sums;
            node_sums({pn_[0]}, sums);
            std::memset(&root.split, 0, sizeof(root.split));
            root.split.gain = -std::numeric_limits<float>::infinity();
            root.G = sums[0].first;
            root.H = sums[0].second;
        }

        const float min_gain = cfg_.min_gain;
        if (!leafwise_) {
            // depth-wise (expansion.rs:137-196)
            std::vector<Cand> cur{root}, next;
            uint32_t depth = 0;
            while (depth < cfg_.max_depth && !cur.empty()) {
                std::vector<Cand> par;
                std::vector<std::pair<uint32_t, uint32_t>> tch;
                std::vector<uint32_t> rid;
                for (const Cand& c : cur) {
                    if (!expands(c, min_gain)) {
                        make_leaf(c);
                        continue;
                    }
                    tch.push_back(apply_split(c));
                    rid.push_back(n_pnodes_++);
                    par.push_back(c);
                }
                next.clear();
                if (!par.empty()) {
                    const bool need_split = depth + 1 < cfg_.max_depth;
                    expand(par, tch, rid, need_split, next);
                }
                cur.swap(next);
                ++depth;
            }
            for (const Cand& c : cur) make_leaf(c);
        } else {
            grow_leafwise(root, min_gain);
        }
        if (qmode_ != GRAD_F32) exact_leaves(o);
        if (renew_) renew_host_leaves(o);
        freeze_categories();

        // prediction update from the partition (grower.rs:208-219)
        std::vector<LeafSeg> segs;
        for (uint32_t pnode = 0; pnode < n_pnodes_; ++pnode) {
            if (pn_[pnode].count == 0) continue;
            segs.push_back(LeafSeg{pn_[pnode].begin, pn_[pnode].count, leaf_value_[pnode], leaf_tree_node_[pnode]});
        }
        std::sort(segs.begin(), segs.end(), [](const LeafSeg& a, const LeafSeg& b) { return a.begin < b.begin; });
        stage_.reset();
        LeafSeg* hl = stage_.take<LeafSeg>(std::max<size_t>(1, segs.size()));
        std::copy(segs.begin(), segs.end(), hl);
        upload(hl, segs.size(), d_leaves_);
        timer_.begin(PH_LEAF);
        launch_leaf_update(d_leaves_.p, (uint32_t)segs.size(), ridx_.p, n_, pred_.p + (size_t)o * n_,
                           cfg_.record_leaves ? row_leaf_.p : nullptr, st_);
        timer_.end();
        m_.counters.launches += 1;
        if (cfg_.record_leaves) {
            tree_.row_leaf.resize(n_);
            BST_CK(cudaMemcpyAsync(tree_.row_leaf.data(), row_leaf_.p, sizeof(uint32_t) * n_, cudaMemcpyDeviceToHost, st_));
        }
        BST_CK(cudaStreamSynchronize(st_));
        BST_CK(cudaGetLastError());
        timer_.collect();
        return std::move(tree_);
    }
};

// Objective::compute_base_score (objectives/mod.rs:278-298).
// compute_weighted_quantile (regression.rs:307-333): (value, weight) pairs
// sorted stably by value; the first value whose f32 running weight reaches
// alpha x the f32 total of the sorted weights.
static float weighted_quantile_base(const float* y, const float* w, uint64_t n, float alpha) {
    if (n == 0) return 0.0f;
    std::vector<std::pair<float, float>> v(n);
    for (uint64_t i = 0; i < n; ++i) v[i] = {y[i], w ? w[i] : 1.0f};
    std::stable_sort(v.begin(), v.end(), [](const std::pair<float, float>& a, const std::pair<float, float>& b) {
        return a.first < b.first;
    });
    float total = 0.0f;
    for (const auto& e : v) total += e.second;
    const float target = alpha * total;
    float cum = 0.0f;
    for (const auto& e : v) {
        cum += e.second;
        if (cum >= target) return e.first;
    }
    return v.back().first;
}

void base_scores(const HostDataset& ds, const bst_config& cfg, uint32_t G, std::vector<float>& out) {
    const uint64_t n = ds.n;
    const float* y = ds.y.data();
    out.assign(G, 0.0f);
    if (n == 0) return;
    auto wv = [&](uint64_t i) { return ds.has_w ? (double)ds.w[i] : 1.0; };
    const float* w = ds.has_w ? ds.w.data() : nullptr;
    if (cfg.objective == BST_OBJ_ABSOLUTE || cfg.objective == BST_OBJ_PSEUDO_HUBER) {  // regression.rs:106-118, 217-228
        out[0] = weighted_quantile_base(y, w, n, 0.5f);
    } else if (cfg.objective == BST_OBJ_PINBALL) {  // regression.rs:157-173
        for (uint32_t g = 0; g < G; ++g) out[g] = weighted_quantile_base(y, w, n, quantile_alpha_of(cfg, g));
    } else if (cfg.objective == BST_OBJ_HINGE) {  // classification.rs:119-125
        out[0] = 0.0f;
    } else if (cfg.objective == BST_OBJ_POISSON) {  // regression.rs:273-298
        double sw = 0, swy = 0;
        for (uint64_t i = 0; i < n; ++i) {
            sw = sw + wv(i);
            swy = swy + wv(i) * (double)y[i];
        }
        const double mean = sw > 0.0 ? std::fmax(swy / sw, 1e-7) : 1.0;
        out[0] = to_f32(std::log(mean));
    } else if (cfg.objective == BST_OBJ_SQUARED) {  // regression.rs:45-69
        double sw = 0, swy = 0;
        for (uint64_t i = 0; i < n; ++i) {
            sw = sw + wv(i);
            swy = swy + wv(i) * (double)y[i];
        }
        out[0] = sw > 0.0 ? to_f32(swy / sw) : 0.0f;
    } else if (cfg.objective == BST_OBJ_LOGISTIC) {  // classification.rs:54-76
        double pos = 0, tot = 0;
        for (uint64_t i = 0; i < n; ++i) {
            pos = pos + wv(i) * (double)y[i];
            tot = tot + wv(i);
        }
        double p = pos / tot;
        p = p < 1e-7 ? 1e-7 : (p > 1.0 - 1e-7 ? 1.0 - 1e-7 : p);
        out[0] = to_f32(std::log(p / (1.0 - p)));
    } else {  // classification.rs:189-222
        std::vector<double> cw(G, 0.0);
        double tot = 0;
        for (uint64_t i = 0; i < n; ++i) {
            const float yi = y[i];
            const uint64_t label = (yi > 0.0f) ? (uint64_t)yi : 0;
            if (label < G) cw[label] += wv(i);
            tot += wv(i);
        }
        for (uint32_t g = 0; g < G; ++g) {
            double p = cw[g] / tot;
            p = p < 1e-7 ? 1e-7 : (p > 1.0 - 1e-7 ? 1.0 - 1e-7 : p);
            out[g] = to_f32(std::log(p));
        }
    }
}

struct StreamGuard {
    cudaStream_t s = nullptr;
    StreamGuard() { BST_CK(cudaStreamCreateWithFlags(&s, cudaStreamNonBlocking)); }
    ~StreamGuard() {
        if (s) cudaStreamDestroy(s);
    }
};

}  // namespace

uint32_t n_outputs_of(const bst_config& c) {
    if (c.objective == BST_OBJ_SOFTMAX) return c.n_classes;
    if (c.objective == BST_OBJ_PINBALL) return c.n_quantiles;
    return 1;
}

float quantile_alpha_of(const bst_config& c, uint32_t o) {
    return c.quantile_alpha && o < c.n_quantiles ? c.quantile_alpha[o] : 0.5f;
}

int transform_of(int objective) {
    return objective == BST_OBJ_LOGISTIC ? 1 : (objective == BST_OBJ_SOFTMAX ? 2 : 0);
}

uint32_t HostTree::alloc() {
    split_index.push_back(0);
    threshold.push_back(0.0f);
    left.push_back(0);
    right.push_back(0);
    default_left.push_back(0);
    is_leaf.push_back(0);
    leaf.push_back(0.0f);
    split_type.push_back(0);
    gain.push_back(0.0f);
    cover.push_back(0.0f);
    split_bin.push_back(0xFFFFFFFFu);
    grad_sum.push_back(0.0);
    hess_sum.push_back(0.0);
    return (uint32_t)split_index.size() - 1;
}

namespace {

// Numeric bounds from the device copy of the features (k_numeric_bounds):
// the sample and the jobs go up, one block per feature sorts its sampled
// values, the bounds come back. `ready` runs before the first launch (the
// features' upload must be enqueued on the stream by then).
class DeviceBounds final : public NumericBounds {
  public:
    DeviceBounds(const float* x, uint64_t n, cudaStream_t st, std::function<void()> ready)
        : x_(x), n_(n), st_(st), ready_(std::move(ready)) {}
    void start(const std::vector<uint32_t>& sample, const std::vector<uint32_t>& features,
               const std::vector<uint8_t>& has_nan, uint32_t max_bins) override {
        ready_();
        feats_ = features;
        has_nan_ = has_nan;
        stride_ = max_bins + 2u;
        const uint32_t nj = (uint32_t)features.size();
        const uint32_t k = sample.empty() ? (uint32_t)n_ : (uint32_t)sample.size();
        if (!sample.empty()) {
            rows_.alloc(k);
            BST_CK(cudaMemcpyAsync(rows_.p, sample.data(), sizeof(uint32_t) * k, cudaMemcpyHostToDevice, st_));
        }
        std::vector<MapJob> jobs(nj);
        for (uint32_t j = 0; j < nj; ++j) jobs[j] = MapJob{features[j], has_nan[j] ? 1u : 0u};
        jobs_.alloc(nj);
        BST_CK(cudaMemcpyAsync(jobs_.p, jobs.data(), sizeof(MapJob) * nj, cudaMemcpyHostToDevice, st_));
        // jobs in batches whose sort buffers (2k words each) stay within 1 GiB
        const uint64_t per_job = 2ull * k;
        const uint32_t batch = (uint32_t)std::max<uint64_t>(1, std::min<uint64_t>(nj, (1ull << 28) / per_job));
        scratch_.alloc((size_t)batch * per_job);
        cand_.alloc((size_t)batch * max_bins);
        bounds_.alloc((size_t)nj * stride_);
        nb_.alloc(nj);
        for (uint32_t b0 = 0; b0 < nj; b0 += batch)
            launch_numeric_bounds(x_, n_, sample.empty() ? nullptr : rows_.p, k, jobs_.p + b0, std::min(batch, nj - b0),
                                  max_bins, scratch_.p, cand_.p, bounds_.p + (size_t)b0 * stride_, nb_.p + b0, st_);
        BST_CK(cudaGetLastError());
    }
    void finish(std::vector<Mapper>& mappers) override {
        const uint32_t nj = (uint32_t)feats_.size();
        std::vector<double> b((size_t)nj * stride_);
        std::vector<uint32_t> nb(nj);
        BST_CK(cudaMemcpyAsync(b.data(), bounds_.p, sizeof(double) * b.size(), cudaMemcpyDeviceToHost, st_));
        BST_CK(cudaMemcpyAsync(nb.data(), nb_.p, sizeof(uint32_t) * nj, cudaMemcpyDeviceToHost, st_));
        BST_CK(cudaStreamSynchronize(st_));
        for (uint32_t j = 0; j < nj; ++j) {
            if (nb[j] == 0 || nb[j] > stride_) throw Error{BST_ERR_CUDA, "device bin bounds out of range"};
            mappers[feats_[j]] = numeric_mapper_from_bounds(b.data() + (size_t)j * stride_, nb[j], has_nan_[j] != 0);
        }
    }

  private:
    const float* x_;
    uint64_t n_;
    cudaStream_t st_;
    std::function<void()> ready_;
    std::vector<uint32_t> feats_;
    std::vector<uint8_t> has_nan_;
    uint32_t stride_ = 0;
    DevArray<uint32_t> rows_, scratch_, nb_;
    DevArray<MapJob> jobs_;
    DevArray<double> cand_, bounds_;
};

}  // namespace

void make_binned(const HostDataset& ds, const bst_config& cfg, cudaStream_t st, DeviceBinned& out) {
    BST_RANGE("bst.binning");
    std::string err;
    const auto t0 = std::chrono::steady_clock::now();
    // Every feature goes to the device while the host analyses them: from
    // pinned memory as one asynchronous copy, from pageable memory on a
    // helper thread (such copies hold the calling thread). The numeric
    // features' bounds are then computed on the device from that copy.
    DevArray<float> x;
    std::thread uploader;
    struct Joiner {
        std::thread& t;
        ~Joiner() {
            if (t.joinable()) t.join();
        }
    } joiner{uploader};
    cudaError_t up_err = cudaSuccess;
    if (ds.n && ds.F) {
        x.alloc((size_t)ds.F * ds.n);
        cudaPointerAttributes a{};
        const bool pinned = cudaPointerGetAttributes(&a, ds.xdata()) == cudaSuccess && a.type == cudaMemoryTypeHost;
        cudaGetLastError();
        const size_t bytes = sizeof(float) * ds.F * ds.n;
        if (pinned) {
            BST_CK(cudaMemcpyAsync(x.p, ds.xdata(), bytes, cudaMemcpyHostToDevice, st));
        } else {
            int dev = 0;
            BST_CK(cudaGetDevice(&dev));
            uploader = std::thread([&x, &ds, &up_err, bytes, dev, st] {
                up_err = cudaSetDevice(dev);
                if (up_err == cudaSuccess) up_err = cudaMemcpyAsync(x.p, ds.xdata(), bytes, cudaMemcpyHostToDevice, st);
            });
        }
    }
    DeviceBounds numeric(x.p, ds.n, st, [&] {
        if (uploader.joinable()) uploader.join();
        BST_CK(up_err);
    });
    bst_status rc = plan_binning(ds.xdata(), ds.F, ds.n, ds.user_cat, cfg, numeric, out.plan, err);
    if (rc != BST_OK) throw Error{rc, err};
    if (uploader.joinable()) uploader.join();
    BST_CK(up_err);
    const BinPlan& p = out.plan;
    const uint32_t nc = p.n_cols();
    const uint64_t n = p.n;
    if (nc == 0) {
        out.binning_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
        return;
    }
    std::vector<BinColumn> cols(nc);
    std::vector<float> thr;
    std::vector<int32_t> cats;
    for (uint32_t c = 0; c < nc; ++c) {
        const Mapper& m = p.mappers[p.col_feature[c]];
        BinColumn bc;
        bc.matrix = p.col_matrix[c];
        bc.pos = p.col_pos[c];
        bc.src = p.col_feature[c];
        bc.is_cat = m.categorical;
        bc.nan_bin = m.missing == MISSING_NAN ? m.n_bins - 1 : m.default_bin;
        bc.zero_bin = m.missing == MISSING_ZERO ? m.default_bin : 0xFFFFFFFFu;
        if (m.categorical) {
            bc.off = (uint32_t)cats.size();
            bc.n_cats = (uint32_t)m.cats.size();
            bc.n_search = 0;
            cats.insert(cats.end(), m.cats.begin(), m.cats.end());
        } else {
            bc.off = (uint32_t)thr.size();
            bc.n_cats = 0;
            bc.n_search = m.n_search();
            for (uint32_t j = 0; j < bc.n_search; ++j) thr.push_back(f32_round_down(m.bounds[j]));
        }
        cols[c] = bc;
    }
    DevArray<float> d_thr;
    DevArray<int32_t> d_cats;
    DevArray<BinColumn> d_cols;
    d_cols.alloc(nc);
    BST_CK(cudaMemcpyAsync(d_cols.p, cols.data(), sizeof(BinColumn) * nc, cudaMemcpyHostToDevice, st));
    d_thr.alloc(std::max<size_t>(1, thr.size()));
    if (!thr.empty()) BST_CK(cudaMemcpyAsync(d_thr.p, thr.data(), sizeof(float) * thr.size(), cudaMemcpyHostToDevice, st));
    d_cats.alloc(std::max<size_t>(1, cats.size()));
    if (!cats.empty())
        BST_CK(cudaMemcpyAsync(d_cats.p, cats.data(), sizeof(int32_t) * cats.size(), cudaMemcpyHostToDevice, st));
    if (p.rec) out.rec.alloc((size_t)n * p.rec);
    out.bins8 = out.rec.p;
    out.bins16 = p.f16 ? reinterpret_cast<uint16_t*>(out.rec.p + p.u16_off) : nullptr;
    uint32_t max_tab = 0;
    for (const BinColumn& bc : cols) max_tab = std::max(max_tab, bc.is_cat ? bc.n_cats : bc.n_search);
    if (bin_assign_rows(p.rec, max_tab) == 0) throw Error{BST_ERR_UNSUPPORTED, "too many features for one row tile"};
    launch_bin_assign(x.p, n, d_cols.p, nc, d_thr.p, d_cats.p, out.rec.p, p.rec, p.u16_off, max_tab, st);
    BST_CK(cudaGetLastError());
    BST_CK(cudaStreamSynchronize(st));
    out.binning_ms = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

std::unique_ptr<Model> grow_one_tree(const HostDataset& ds, const float* g, const float* h, const bst_config& cfg,
                                     uint32_t n_threads) {
    BST_CK(cudaSetDevice(cfg.device));
    StreamGuard sg;
    auto model = std::make_unique<Model>();
    model->device = cfg.device;
    model->objective = BST_OBJ_SQUARED;
    model->n_groups = 1;
    model->n_features = (uint32_t)ds.F;
    model->base = {0.0f};
    DeviceBinned binned;
    make_binned(ds, cfg, sg.s, binned);
    Trainer tr(ds, binned, cfg, n_threads, sg.s, *model);
    HostTree t = tr.run_external(g, h);
    model->trees.push_back(std::move(t));
    return model;
}

std::unique_ptr<Model> train_model(const HostDataset& ds, const bst_config& cfg, uint32_t n_threads,
                                   const HostDataset* val) {
    BST_CK(cudaSetDevice(cfg.device));
    StreamGuard sg;
    auto model = std::make_unique<Model>();
    model->device = cfg.device;
    model->objective = cfg.objective;
    model->n_groups = n_outputs_of(cfg);
    model->n_features = (uint32_t)ds.F;
    DeviceBinned binned;
    make_binned(ds, cfg, sg.s, binned);
    model->timings[PH_BIN] = binned.binning_ms;
    base_scores(ds, cfg, model->n_groups, model->base);
    const auto t0 = std::chrono::steady_clock::now();
    Trainer tr(ds, binned, cfg, n_threads, sg.s, *model);
    tr.run(val);
    model->timings[7] = std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
    return model;
}

struct Booster::Impl {
    StreamGuard sg;
    DeviceBinned binned;
    std::unique_ptr<Model> model;
    std::unique_ptr<Trainer> tr;
    bst_config cfg;
    std::string tune_cache;  // owned copies: the caller's arrays may not outlive the call
    std::vector<float> alphas;
    uint32_t done = 0;
};

Booster::Booster(const HostDataset& ds, const bst_config& cfg, uint32_t n_threads) {
    BST_CK(cudaSetDevice(cfg.device));
    impl_ = std::make_unique<Impl>();
    Impl& b = *impl_;
    b.cfg = cfg;
    if (cfg.autotune_cache) b.tune_cache = cfg.autotune_cache;
    b.cfg.autotune_cache = cfg.autotune_cache ? b.tune_cache.c_str() : nullptr;
    if (cfg.quantile_alpha && cfg.n_quantiles) b.alphas.assign(cfg.quantile_alpha, cfg.quantile_alpha + cfg.n_quantiles);
    b.cfg.quantile_alpha = b.alphas.empty() ? nullptr : b.alphas.data();
    b.model = std::make_unique<Model>();
    Model& m = *b.model;
    m.device = cfg.device;
    m.objective = cfg.objective;
    m.n_groups = n_outputs_of(cfg);
    m.n_features = (uint32_t)ds.F;
    make_binned(ds, cfg, b.sg.s, b.binned);
    m.timings[PH_BIN] = b.binned.binning_ms;
    base_scores(ds, cfg, m.n_groups, m.base);
    b.tr = std::make_unique<Trainer>(ds, b.binned, b.cfg, n_threads, b.sg.s, m);
    b.tr->start();
}

Booster::~Booster() = default;

void Booster::update(uint32_t rounds) {
    BST_RANGE("bst.update");
    BST_CK(cudaSetDevice(impl_->cfg.device));
    const auto t0 = std::chrono::steady_clock::now();
    impl_->tr->rounds(rounds);
    impl_->done += rounds;
    impl_->model->timings[7] += std::chrono::duration<double, std::milli>(std::chrono::steady_clock::now() - t0).count();
}

uint32_t Booster::rounds_done() const { return impl_->done; }
const Model& Booster::model() const { return *impl_->model; }

std::unique_ptr<Model> Booster::snapshot() const {
    BST_CK(cudaSetDevice(impl_->cfg.device));
    impl_->tr->finish();
    const Model& s = *impl_->model;
    auto m = std::make_unique<Model>();
    m->n_groups = s.n_groups;
    m->n_features = s.n_features;
    m->objective = s.objective;
    m->base = s.base;
    m->trees = s.trees;
    m->train_pred = s.train_pred;
    for (int i = 0; i < 8; ++i) m->timings[i] = s.timings[i];
    m->counters = s.counters;
    m->device = s.device;
    m->tune_info = s.tune_info;
    return m;
}

// Node-list forest of `trees` (forest order) on the device: what
// launch_predict walks.
void upload_node_forest(const std::vector<const HostTree*>& trees, uint32_t n_groups, const std::vector<float>& base,
                        DeviceForest& df) {
    DeviceForest* f = &df;
    std::vector<ForestNode> nodes;
    std::vector<uint32_t> roots, cat_seg, cat_words, gt, goff(n_groups + 1, 0);
    for (const HostTree* tp : trees) {
        const HostTree& t = *tp;
        const uint32_t base_idx = (uint32_t)nodes.size();
        const uint32_t wbase = (uint32_t)cat_words.size();
        roots.push_back(base_idx);
        for (size_t i = 0; i < t.split_index.size(); ++i) {
            ForestNode fn;
            fn.word = (t.split_index[i] & 0x1FFFFFFFu) | ((uint32_t)t.is_leaf[i] << 31) |
                      ((uint32_t)t.default_left[i] << 30) | ((uint32_t)(t.split_type[i] == 1) << 29);
            fn.value = t.is_leaf[i] ? t.leaf[i] : t.threshold[i];
            fn.left = base_idx + t.left[i];
            fn.right = base_idx + t.right[i];
            nodes.push_back(fn);
            const uint32_t ss = t.seg_size.empty() ? 0 : t.seg_size[i];
            cat_seg.push_back(ss ? wbase + t.seg_start[i] : 0);
            cat_seg.push_back(ss);
        }
        cat_words.insert(cat_words.end(), t.cat_words.begin(), t.cat_words.end());
    }
    for (uint32_t g = 0; g < n_groups; ++g) {
        goff[g] = (uint32_t)gt.size();
        for (uint32_t t = 0; t < trees.size(); ++t)
            if (trees[t]->group == g) gt.push_back(t);
    }
    goff[n_groups] = (uint32_t)gt.size();
    auto up = [](auto& dst, const auto& src) {
        dst.alloc(std::max<size_t>(1, src.size()));
        if (!src.empty())
            BST_CK(cudaMemcpy(dst.p, src.data(), sizeof(src[0]) * src.size(), cudaMemcpyHostToDevice));
    };
    up(f->nodes, nodes);
    up(f->roots, roots);
    up(f->group_trees, gt);
    up(f->group_off, goff);
    up(f->cat_seg, cat_seg);
    up(f->cat_words, cat_words);
    up(f->base, base);
    f->view.nodes = f->nodes.p;
    f->view.roots = f->roots.p;
    f->view.group_trees = f->group_trees.p;
    f->view.group_off = f->group_off.p;
    f->view.cat_seg = f->cat_seg.p;
    f->view.cat_words = f->cat_words.p;
    f->view.base = f->base.p;
    f->view.n_trees = (uint32_t)trees.size();
    f->view.n_groups = n_groups;
#ifdef BST_CHECKED
    f->view.chk_nodes = (uint32_t)nodes.size();
#endif
}

const DeviceForest& Model::device_forest() const {
    std::lock_guard<std::mutex> lk(mu);
    if (dev) return *dev;
    BST_CK(cudaSetDevice(device));
    auto f = std::make_unique<DeviceForest>();
    std::vector<const HostTree*> tp;
    tp.reserve(trees.size());
    for (const HostTree& t : trees) tp.push_back(&t);
    upload_node_forest(tp, n_groups, base, *f);
    build_heap_forest(*f);
    dev = std::move(f);
    return *dev;
}

// Heap-ordered copy of the forest (1-based: children of heap position h at
// 2h, 2h + 1), every tree padded to a complete tree of depth HEAP_DEPTH,
// trees grouped by output group in forest order, with the bin columns its
// splits read (the word and column formats are those of HeapForest). A leaf
// at depth d < HEAP_DEPTH sits at its leftmost descendant's position,
// reached through padding splits (K = 0xFFFF on a NaN-as-0 column) that
// always go left. Leaves deeper than HEAP_DEPTH, a feature split both
// numerically and categorically, a NaN threshold whose split sends missing
// values left, more than 65534 distinct thresholds of one feature, more than
// HEAP_MAX_COLS columns or 65536 categorical splits, or a category set
// reaching category 65504 leave the forest on the node-list traversal.
void Model::build_heap_forest(DeviceForest& f) const {
    const uint32_t NF = n_features;
    if (NF == 0) return;
    std::vector<std::vector<float>> thr(NF);
    std::vector<uint8_t> fcat(NF, 0), fnum0(NF, 0), fnum1(NF, 0);
    uint32_t min_F = 1;  // padding splits may read feature 0
    for (const HostTree& t : trees)
        for (size_t i = 0; i < t.is_leaf.size(); ++i) {
            if (t.is_leaf[i]) continue;
            const uint32_t ft = t.split_index[i];
            if (ft >= NF) return;
            min_F = std::max(min_F, ft + 1);
            if (t.split_type[i] == 1) {
                fcat[ft] = 1;
                if (!t.seg_size.empty() && t.seg_size[i] > 2047u) return;
            } else {
                const float th = t.threshold[i];
                if (th == th)
                    thr[ft].push_back(th);
                else if (t.default_left[i])
                    return;
                (t.default_left[i] ? fnum1 : fnum0)[ft] = 1;
            }
        }
    // per feature: thresholds in NaN-padded blocks of blk = 2^lb entries
    // (the smallest power of two with n <= HEAP_SPLITTERS blk) and the
    // splitters (first threshold of blocks 1 ..)
    const float qnan = std::numeric_limits<float>::quiet_NaN();
    std::vector<float> thr_flat, spl((size_t)NF * HEAP_SPLITTERS, qnan);
    std::vector<uint32_t> thr_off(NF + 1, 0);
    std::vector<uint8_t> finfo(NF, 0);
    size_t max_thr = 0;
    bool any_cat = false;
    for (uint32_t ft = 0; ft < NF; ++ft) {
        if (fcat[ft] && (fnum0[ft] || fnum1[ft])) return;
        any_cat |= fcat[ft] != 0;
        auto& v = thr[ft];
        std::sort(v.begin(), v.end());
        v.erase(std::unique(v.begin(), v.end(), [](float a, float b) { return a == b; }), v.end());
        if (v.size() > 65534u) return;
        max_thr = std::max(max_thr, v.size());
        uint32_t lb = 4;  // blocks of at least one 16-entry window
        while (((size_t)HEAP_SPLITTERS << lb) < v.size()) ++lb;
        const size_t blk = (size_t)1 << lb;
        const size_t ns = std::max<size_t>(1, (v.size() + blk - 1) / blk);
        thr_off[ft] = (uint32_t)thr_flat.size();  // a multiple of 16 floats: aligned windows
        thr_flat.insert(thr_flat.end(), v.begin(), v.end());
        thr_flat.resize(thr_off[ft] + ns * blk, qnan);
        for (size_t j = 0; j + 1 < ns; ++j) spl[(size_t)ft * HEAP_SPLITTERS + j] = v[(j + 1) * blk];
        finfo[ft] = (uint8_t)(lb | (fcat[ft] ? 0x80u : 0u));
    }
    thr_off[NF] = (uint32_t)thr_flat.size();
    // bin columns: NaN-as-largest (numeric, default right) or categorical,
    // and NaN-as-0 (numeric, default left); padding needs one NaN-as-0 column
    std::vector<int32_t> fcol(2 * (size_t)NF, -1);
    int32_t n_cols = 0, pad_col = -1;
    for (uint32_t ft = 0; ft < NF; ++ft) {
        if (fcat[ft] || fnum0[ft]) fcol[2 * ft] = n_cols++;
        if (fnum1[ft]) {
            fcol[2 * ft + 1] = n_cols++;
            if (pad_col < 0) pad_col = fcol[2 * ft + 1];
        }
    }
    if (pad_col < 0) pad_col = fcol[1] = n_cols++;
    if ((uint32_t)n_cols > HEAP_MAX_COLS) return;
    const uint32_t pad_word = 0xFFFF0000u | (uint32_t)pad_col;

    std::vector<uint32_t> hn, goff(n_groups + 1, 0), words;
    std::vector<uint2> cat;
    uint32_t placed = 0;
    for (uint32_t g = 0; g < n_groups; ++g) {
        goff[g] = placed;
        for (const HostTree& t : trees) {
            if (t.group != g) continue;
            const size_t base = hn.size();
            hn.resize(base + HEAP_NODES, pad_word);
            hn[base] = 0;
            const uint32_t wbase = (uint32_t)words.size();
            words.insert(words.end(), t.cat_words.begin(), t.cat_words.end());
            // (tree node, heap position, depth)
            std::vector<std::array<uint32_t, 3>> stack{{0u, 1u, 0u}};
            while (!stack.empty()) {
                const auto it = stack.back();
                stack.pop_back();
                const uint32_t i = it[0], h = it[1], d = it[2];
                if (t.is_leaf[i]) {
                    uint32_t bits;
                    std::memcpy(&bits, &t.leaf[i], 4);
                    hn[base + (h << (HEAP_DEPTH - d))] = bits;  // padding splits lead left to here
                    continue;
                }
                if (d >= (uint32_t)HEAP_DEPTH) return;  // too deep: no heap copy
                const uint32_t ft = t.split_index[i];
                uint32_t w;
                if (t.split_type[i] == 1) {
                    if (cat.size() >= 65536u) return;
                    const uint32_t ss = t.seg_size.empty() ? 0 : t.seg_size[i];
                    w = ((uint32_t)cat.size() << 16) | 0x8000u | (uint32_t)fcol[2 * ft];
                    cat.push_back(make_uint2(ss ? wbase + t.seg_start[i] : 0u,
                                             ss | ((uint32_t)(t.default_left[i] != 0) << 31)));
                } else {
                    const float th = t.threshold[i];
                    const auto& v = thr[ft];
                    const uint32_t K =
                        th == th ? (uint32_t)(std::lower_bound(v.begin(), v.end(), th) - v.begin()) + 1u : 0u;
                    w = (K << 16) | (uint32_t)fcol[2 * ft + (t.default_left[i] ? 1 : 0)];
                }
                hn[base + h] = w;
                stack.push_back({t.left[i], 2 * h, d + 1});
                stack.push_back({t.right[i], 2 * h + 1, d + 1});
            }
            ++placed;
        }
    }
    static_assert(HEAP_NODES == 2u << HEAP_DEPTH, "complete tree of HEAP_DEPTH levels");
    goff[n_groups] = placed;
    auto up = [](auto& dst, const auto& src) {
        dst.alloc(std::max<size_t>(1, src.size()));
        if (!src.empty())
            BST_CK(cudaMemcpy(dst.p, src.data(), sizeof(src[0]) * src.size(), cudaMemcpyHostToDevice));
    };
    up(f.heap_nodes, hn);
    up(f.heap_goff, goff);
    up(f.heap_cat, cat);
    up(f.heap_words, words);
    up(f.heap_thr, thr_flat);
    up(f.heap_thr_off, thr_off);
    up(f.heap_spl, spl);
    up(f.heap_fcol, fcol);
    up(f.heap_finfo, finfo);
    f.heap.nodes = f.heap_nodes.p;
    f.heap.group_off = f.heap_goff.p;
    f.heap.cat = f.heap_cat.p;
    f.heap.cat_words = f.heap_words.p;
    f.heap.thr = f.heap_thr.p;
    f.heap.thr_off = f.heap_thr_off.p;
    f.heap.spl = f.heap_spl.p;
    f.heap.feat_col = f.heap_fcol.p;
    f.heap.feat_info = f.heap_finfo.p;
    f.heap.base = f.base.p;
    f.heap.n_trees = placed;
    f.heap.n_groups = n_groups;
    f.heap.n_features = NF;
    f.heap.n_cols = (uint32_t)n_cols;
    f.heap.has_cat = any_cat ? 1 : 0;
    f.heap.bins16 = (any_cat || max_thr > 255) ? 1 : 0;
    f.heap_min_F = min_F;
    f.heap_ok = true;
}

// Stream-ordered device memory for the traversal's bin tiles when the caller
// brings none: one pool per device, kept warm up to 1 GiB between calls.
static cudaMemPool_t scratch_pool() {
    static std::mutex mu;
    static std::map<int, cudaMemPool_t> pools;
    int dev = 0;
    BST_CK(cudaGetDevice(&dev));
    std::lock_guard<std::mutex> lk(mu);
    auto it = pools.find(dev);
    if (it != pools.end()) return it->second;
    cudaMemPoolProps props{};
    props.allocType = cudaMemAllocationTypePinned;
    props.location.type = cudaMemLocationTypeDevice;
    props.location.id = dev;
    cudaMemPool_t pool;
    BST_CK(cudaMemPoolCreate(&pool, &props));
    uint64_t keep = 1ull << 30;
    BST_CK(cudaMemPoolSetAttribute(pool, cudaMemPoolAttrReleaseThreshold, &keep));
    pools[dev] = pool;
    return pool;
}

bool forest_uses_heap(const DeviceForest& f, uint64_t n, uint64_t F) {
    return f.heap_ok && F >= f.heap_min_F && F <= 0xFFFFFFFFull && predict_heap_rows(f.heap, (uint32_t)F, n) > 0;
}

size_t forest_bin_bytes_per_row(const DeviceForest& f, uint64_t F) {
    return f.heap_ok && F <= 0xFFFFFFFFull ? predict_heap_scratch_max(f.heap, (uint32_t)F, 1) / (1 + PREDICT_TILE_MAX)
                                           : 0;
}

size_t forest_scratch_max(const DeviceForest& f, uint64_t n_max, uint64_t F) {
    return f.heap_ok && F <= 0xFFFFFFFFull ? predict_heap_scratch_max(f.heap, (uint32_t)F, n_max) : 0;
}

void forest_predict_rows(const DeviceForest& f, const float* x, uint64_t n, uint64_t F, float* out, cudaStream_t st,
                         void* scratch, size_t scratch_bytes) {
    if (!forest_uses_heap(f, n, F)) {
        launch_predict(f.view, x, n, (uint32_t)F, 0, out, st);
        return;
    }
    const size_t need = predict_heap_scratch(f.heap, (uint32_t)F, n);
    if (scratch && scratch_bytes >= need) {
        launch_predict_heap(f.heap, x, n, (uint32_t)F, out, scratch, st);
        return;
    }
    void* tmp = nullptr;
    BST_CK(cudaMallocFromPoolAsync(&tmp, std::max<size_t>(need, 16), scratch_pool(), st));
    launch_predict_heap(f.heap, x, n, (uint32_t)F, out, tmp, st);
    BST_CK(cudaFreeAsync(tmp, st));
}

void predict_device(const Model& m, const float* x, uint64_t n, uint64_t F, bool raw, float* out, cudaStream_t st) {
    BST_RANGE("bst.predict");
    const DeviceForest& f = m.device_forest();
    forest_predict_rows(f, x, n, F, out, st);
    if (!raw) launch_transform(transform_of(m.objective), out, m.n_groups, n, st);
    BST_CK(cudaGetLastError());
}

// Metric values of [G][n] predictions (already transformed for the
// probability metrics): RMSE (metrics/regression.rs:17-45), log loss
// (metrics/classification.rs:13-40), multiclass log loss
// (classification.rs:332-360); f64 sums in row order.
double metric_value(int metric, const float* p, uint32_t G, uint64_t n, const float* y, const float* w,
                    const MetricParams& mp) {
    if (n == 0) return 0.0;
    const double EPS = 1e-15;
    auto wv = [&](uint64_t i) { return w ? (double)w[i] : 1.0; };
    auto clampd = [](double v, double lo, double hi) { return v < lo ? lo : (v > hi ? hi : v); };
    if (metric == BST_METRIC_MAE) {  // metrics/regression.rs:55-87
        double sum = 0.0;
        for (uint32_t g = 0; g < G; ++g) {
            double sa = 0, sw = 0;
            for (uint64_t i = 0; i < n; ++i) {
                sa = sa + wv(i) * std::fabs((double)p[(uint64_t)g * n + i] - (double)y[i]);
                sw = sw + wv(i);
            }
            sum += sw > 0.0 ? sa / sw : 0.0;
        }
        return sum / (double)G;
    }
    if (metric == BST_METRIC_MAPE) {  // metrics/regression.rs:89-124
        double sa = 0, sw = 0;
        for (uint64_t i = 0; i < n; ++i) {
            const double pp = (double)p[i], l = (double)y[i];
            sa = sa + wv(i) * (std::fabs(pp - l) / std::fmax(std::fabs(l), EPS));
            sw = sw + wv(i);
        }
        return sw > 0.0 ? (sa / sw) * 100.0 : 0.0;
    }
    if (metric == BST_METRIC_QUANTILE) {  // metrics/regression.rs:126-174
        double tl = 0, tw = 0;
        for (uint32_t q = 0; q < G; ++q) {
            const double a = (double)(mp.alpha && q < mp.n_alpha ? mp.alpha[q] : 0.5f);
            double l = 0, sw = 0;
            for (uint64_t i = 0; i < n; ++i) {
                const double r = (double)y[i] - (double)p[(uint64_t)q * n + i];
                l = l + wv(i) * (r >= 0.0 ? a * r : (1.0 - a) * (-r));
                sw = sw + wv(i);
            }
            tl = tl + l;
            tw = tw + sw;
        }
        return tw > 0.0 ? tl / tw : 0.0;
    }
    if (metric == BST_METRIC_HUBER) {  // metrics/regression.rs:216-245
        const double delta = (double)mp.delta;
        double sl = 0, sw = 0;
        for (uint64_t i = 0; i < n; ++i) {
            const double r = std::fabs((double)p[i] - (double)y[i]);
            sl = sl + wv(i) * (r <= delta ? 0.5 * r * r : delta * (r - 0.5 * delta));
            sw = sw + wv(i);
        }
        return sw > 0.0 ? sl / sw : 0.0;
    }
    if (metric == BST_METRIC_POISSON) {  // metrics/regression.rs:176-210
        const double E = 1e-9;
        double sd = 0, sw = 0;
        for (uint64_t i = 0; i < n; ++i) {
            const double yy = (double)y[i], mu = std::fmax((double)p[i], E);
            sd = sd + wv(i) * (yy > E ? 2.0 * (yy * std::log(yy / mu) - (yy - mu)) : 2.0 * mu);
            sw = sw + wv(i);
        }
        return sw > 0.0 ? sd / sw : 0.0;
    }
    if (metric == BST_METRIC_MARGIN_ACCURACY) {  // metrics/classification.rs:85-118, threshold 0
        double sc = 0, sw = 0;
        for (uint64_t i = 0; i < n; ++i) {
            const float pc = p[i] >= 0.0f ? 1.0f : 0.0f;
            sc = sc + wv(i) * (std::fabs(pc - y[i]) < 0.5f ? 1.0 : 0.0);
            sw = sw + wv(i);
        }
        return sw > 0.0 ? sc / sw : 0.0;
    }
    if (metric == BST_METRIC_RMSE) {
        double sum = 0.0;
        for (uint32_t g = 0; g < G; ++g) {
            double ss = 0, sw = 0;
            for (uint64_t i = 0; i < n; ++i) {
                const double d = (double)p[(uint64_t)g * n + i] - (double)y[i];
                ss = ss + wv(i) * d * d;
                sw = sw + wv(i);
            }
            sum += sw > 0.0 ? std::sqrt(ss / sw) : 0.0;
        }
        return sum / (double)G;
    }
    if (metric == BST_METRIC_LOGLOSS) {
        double sl = 0, sw = 0;
        for (uint64_t i = 0; i < n; ++i) {
            const double pp = clampd((double)p[i], EPS, 1.0 - EPS), l = (double)y[i];
            sl = sl + wv(i) * -(l * std::log(pp) + (1.0 - l) * std::log(1.0 - pp));
            sw = sw + wv(i);
        }
        return sw > 0.0 ? sl / sw : 0.0;
    }
    if (metric == BST_METRIC_MLOGLOSS) {
        double sl = 0, sw = 0;
        for (uint64_t i = 0; i < n; ++i) {
            const float r = std::round(y[i]);
            const uint64_t c = r > 0.0f ? (uint64_t)r : 0;
            const double pp = clampd(c < G ? (double)p[c * n + i] : EPS, EPS, 1.0 - EPS);
            sl = sl + wv(i) * -std::log(pp);
            sw = sw + wv(i);
        }
        return sw > 0.0 ? sl / sw : 0.0;
    }
    return std::numeric_limits<double>::quiet_NaN();
}

// default_metric_for_objective (training/metrics/mod.rs:213-236) for
// BST_METRIC_DEFAULT.
int resolve_metric(int metric, int objective) {
    if (metric != BST_METRIC_DEFAULT) return metric;
    if (objective == BST_OBJ_LOGISTIC) return BST_METRIC_LOGLOSS;
    if (objective == BST_OBJ_SOFTMAX) return BST_METRIC_MLOGLOSS;
    if (objective == BST_OBJ_PINBALL) return BST_METRIC_QUANTILE;
    if (objective == BST_OBJ_HINGE) return BST_METRIC_MARGIN_ACCURACY;
    return BST_METRIC_RMSE;
}

void predict_host(const Model& m, const HostDataset& ds, bool raw, float* out) {
    BST_CK(cudaSetDevice(m.device));
    const DeviceForest& f = m.device_forest();
    StreamGuard sg;
    const uint64_t n = ds.n;
    if (n == 0) return;
    DevArray<float> x, o;
    x.alloc((size_t)n * ds.F);
    o.alloc((size_t)n * m.n_groups);
    BST_CK(cudaMemcpyAsync(x.p, ds.xdata(), sizeof(float) * n * ds.F, cudaMemcpyHostToDevice, sg.s));
    launch_predict(f.view, x.p, n, (uint32_t)ds.F, 1, o.p, sg.s);
    if (!raw) launch_transform(transform_of(m.objective), o.p, m.n_groups, n, sg.s);
    BST_CK(cudaGetLastError());
    BST_CK(cudaMemcpyAsync(out, o.p, sizeof(float) * n * m.n_groups, cudaMemcpyDeviceToHost, sg.s));
    BST_CK(cudaStreamSynchronize(sg.s));
}

}  // namespace bst
