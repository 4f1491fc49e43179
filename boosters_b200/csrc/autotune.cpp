// autotune.cpp — cache file and online exploration of the batched tree
// pipeline's launch shapes (autotune.h).
#include "autotune.h"

#include <cuda_runtime.h>
#include <unistd.h>

#include <algorithm>
#include <cmath>
#include <cstdio>
#include <cstdlib>
#include <fstream>
#include <map>
#include <mutex>
#include <sstream>

namespace bst {

std::string TuneShape::str() const {
    return "items=" + std::to_string(items) + ",hist=" + std::to_string(hist) + ",grid=" + std::to_string(grid);
}

bool TuneShape::parse(const std::string& s, TuneShape& out) {
    TuneShape t;
    int seen = 0;
    std::stringstream ss(s);
    std::string kv;
    while (std::getline(ss, kv, ',')) {
        const size_t eq = kv.find('=');
        if (eq == std::string::npos || eq + 1 >= kv.size()) return false;
        const std::string k = kv.substr(0, eq);
        char* end = nullptr;
        const unsigned long v = std::strtoul(kv.c_str() + eq + 1, &end, 10);
        if (!end || *end != '\0' || v > 1024) return false;
        if (k == "items")
            t.items = (uint32_t)v, seen |= 1;
        else if (k == "hist")
            t.hist = (uint32_t)v, seen |= 2;
        else if (k == "grid")
            t.grid = (uint32_t)v, seen |= 4;
        else
            return false;
    }
    if (seen != 7 || t.items == 0 || t.grid == 0) return false;
    out = t;
    return true;
}

// Computed once per device and process: cudaGetDeviceProperties takes
// milliseconds, and every training call asks.
std::string device_signature(int device) {
    static std::mutex mu;
    static std::map<int, std::string> known;
    {
        std::lock_guard<std::mutex> lk(mu);
        auto it = known.find(device);
        if (it != known.end()) return it->second;
    }
    cudaDeviceProp p{};
    if (cudaGetDeviceProperties(&p, device) != cudaSuccess) {
        cudaGetLastError();
        return "unknown";
    }
    std::string name = p.name;
    for (char& c : name)
        if (c == '\t' || c == '\n' || c == '|') c = ' ';
    name += "|" + std::to_string(p.multiProcessorCount) + "|" + std::to_string(p.major) + "." + std::to_string(p.minor);
    std::lock_guard<std::mutex> lk(mu);
    known[device] = name;
    return name;
}

namespace {
std::mutex g_cache_mu;

std::vector<std::pair<std::string, std::string>> read_lines(const std::string& path) {
    std::vector<std::pair<std::string, std::string>> out;
    std::ifstream f(path);
    std::string line;
    while (std::getline(f, line)) {
        const size_t tab = line.find('\t');
        if (tab == std::string::npos) continue;
        out.emplace_back(line.substr(0, tab), line.substr(tab + 1));
    }
    return out;
}
}  // namespace

bool tune_cache_lookup(const std::string& path, const std::string& key, TuneShape& out) {
    if (path.empty()) return false;
    std::lock_guard<std::mutex> lk(g_cache_mu);
    for (const auto& kv : read_lines(path))
        if (kv.first == key) return TuneShape::parse(kv.second, out);
    return false;
}

void tune_cache_store(const std::string& path, const std::string& key, const TuneShape& s) {
    if (path.empty()) return;
    std::lock_guard<std::mutex> lk(g_cache_mu);
    auto lines = read_lines(path);
    bool found = false;
    for (auto& kv : lines)
        if (kv.first == key) {
            kv.second = s.str();
            found = true;
        }
    if (!found) lines.emplace_back(key, s.str());
    const std::string tmp = path + ".tmp." + std::to_string((long)getpid());
    {
        std::ofstream f(tmp, std::ios::trunc);
        if (!f) return;
        for (const auto& kv : lines) f << kv.first << '\t' << kv.second << '\n';
        if (!f) {
            std::remove(tmp.c_str());
            return;
        }
    }
    if (std::rename(tmp.c_str(), path.c_str()) != 0) std::remove(tmp.c_str());
}

TuneExplorer::TuneExplorer(std::vector<TuneShape> cands, uint32_t rounds, uint32_t skip)
    : cands_(std::move(cands)), times_(cands_.size()), rounds_(std::max<uint32_t>(1, rounds)), skip_(skip) {
    if (cands_.size() <= 1) done_ = true;
}

uint32_t TuneExplorer::next(bool* timed) {
    const uint32_t i = issued_++;
    if (i < skip_) {
        *timed = false;
        return 0;
    }
    *timed = true;
    return (uint32_t)((i - skip_) % cands_.size());
}

std::vector<double> TuneExplorer::medians() const {
    std::vector<double> m(cands_.size(), NAN);
    for (size_t c = 0; c < cands_.size(); ++c) {
        std::vector<float> t = times_[c];
        if (t.empty()) continue;
        std::sort(t.begin(), t.end());
        const size_t k = t.size();
        m[c] = k % 2 ? t[k / 2] : 0.5 * ((double)t[k / 2 - 1] + t[k / 2]);
    }
    return m;
}

void TuneExplorer::record(uint32_t c, float ms) {
    if (done_ || c >= cands_.size()) return;
    times_[c].push_back(ms);
    for (const auto& t : times_)
        if (t.size() < rounds_) return;
    const std::vector<double> m = medians();
    best_ = 0;
    for (size_t k = 1; k < m.size(); ++k)
        if (m[k] < m[best_]) best_ = (uint32_t)k;
    done_ = true;
}

}  // namespace bst
