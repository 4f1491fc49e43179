// persist.cpp — the reference's model file layouts for GBDT models:
//   .bstr.json  JSON envelope {"bstr_version", "model_type", "model"}
//               (persist/json.rs:50-75) around the model schema;
//   .bstr       32-byte header (magic "BSTR", schema version u32 LE, format
//               byte, model type byte, 22 reserved zeros), a MessagePack
//               named-map payload of the same schema, and a 16-byte trailer
//               (payload length u64 LE, CRC32C u32 LE, 4 reserved zeros)
//               (persist/envelope.rs:13-221, binary.rs:52-146).
// The schema (persist/schema.rs:27-150) and its runtime conversion
// (persist/convert.rs:78-420, 700-730): per tree SoA arrays over all nodes
// (split index, f64 threshold, children with 0 meaning "leaf", default
// direction, scalar leaf values), categorical splits as sorted category
// lists of the nodes that have them, optional gains and covers; per forest
// tree groups (only with more than one group), group count and base scores;
// the output transform by name. Payloads are plain MessagePack (format byte
// 0x01) or zstd-compressed MessagePack (0x02; binary.rs:60-91, the
// reference writes zstd level 3 by default and reads any number of
// concatenated frames, zstd::decode_all). zstd comes from the system
// libzstd.so.1 through its public streaming API, loaded at first use.
#include <dlfcn.h>

#include <algorithm>
#include <charconv>
#include <cmath>
#include <cstring>
#include <fstream>
#include <limits>
#include <mutex>
#include <string>
#include <vector>

#include "engine.h"

namespace bst {

namespace {

constexpr uint32_t SCHEMA_VERSION = 2;      // envelope.rs:16
constexpr uint32_t MAX_SUPPORTED_VERSION = 2;
constexpr size_t HEADER_SIZE = 32, TRAILER_SIZE = 16;

[[noreturn]] void bad(const std::string& msg) { throw Error{BST_ERR_INVALID_ARGUMENT, "model file: " + msg}; }
[[noreturn]] void unsupported(const std::string& msg) { throw Error{BST_ERR_UNSUPPORTED, "model file: " + msg}; }

// ---- zstd (system libzstd.so.1, public API of zstd.h) -------------------------
// The buffer structs and entry points below are the library's documented
// stable interface (names and signatures only).
struct ZInBuf {
    const void* src;
    size_t size;
    size_t pos;
};
struct ZOutBuf {
    void* dst;
    size_t size;
    size_t pos;
};

struct Zstd {
    void* h = nullptr;
    void* (*create_dstream)() = nullptr;
    size_t (*free_dstream)(void*) = nullptr;
    size_t (*init_dstream)(void*) = nullptr;
    size_t (*decompress_stream)(void*, ZOutBuf*, ZInBuf*) = nullptr;
    size_t (*compress)(void*, size_t, const void*, size_t, int) = nullptr;
    size_t (*compress_bound)(size_t) = nullptr;
    unsigned (*is_error)(size_t) = nullptr;
    const char* (*error_name)(size_t) = nullptr;
    std::string load_error;
};

const Zstd& zstd() {
    static Zstd z;
    static std::once_flag once;
    std::call_once(once, [] {
        z.h = dlopen("libzstd.so.1", RTLD_NOW | RTLD_LOCAL);
        if (!z.h) {
            const char* e = dlerror();
            z.load_error = std::string("libzstd.so.1 could not be loaded: ") + (e ? e : "unknown error");
            return;
        }
        auto sym = [&](const char* name) {
            void* f = dlsym(z.h, name);
            if (!f && z.load_error.empty()) z.load_error = std::string("libzstd.so.1 lacks ") + name;
            return f;
        };
        z.create_dstream = reinterpret_cast<void* (*)()>(sym("ZSTD_createDStream"));
        z.free_dstream = reinterpret_cast<size_t (*)(void*)>(sym("ZSTD_freeDStream"));
        z.init_dstream = reinterpret_cast<size_t (*)(void*)>(sym("ZSTD_initDStream"));
        z.decompress_stream = reinterpret_cast<size_t (*)(void*, ZOutBuf*, ZInBuf*)>(sym("ZSTD_decompressStream"));
        z.compress = reinterpret_cast<size_t (*)(void*, size_t, const void*, size_t, int)>(sym("ZSTD_compress"));
        z.compress_bound = reinterpret_cast<size_t (*)(size_t)>(sym("ZSTD_compressBound"));
        z.is_error = reinterpret_cast<unsigned (*)(size_t)>(sym("ZSTD_isError"));
        z.error_name = reinterpret_cast<const char* (*)(size_t)>(sym("ZSTD_getErrorName"));
    });
    if (!z.load_error.empty()) unsupported("zstd payloads need the system zstd library (" + z.load_error + ")");
    return z;
}

// Every frame of the payload, concatenated (zstd::decode_all).
std::vector<uint8_t> zstd_decode_all(const uint8_t* p, size_t n) {
    const Zstd& z = zstd();
    void* ds = z.create_dstream();
    if (!ds) throw Error{BST_ERR_OUT_OF_MEMORY, "model file: zstd stream allocation failed"};
    std::vector<uint8_t> out;
    std::string err;
    size_t r = z.init_dstream(ds);
    if (z.is_error(r)) err = z.error_name(r);
    ZInBuf in{p, n, 0};
    size_t last = 0;
    while (err.empty() && in.pos < in.size) {
        const size_t old = out.size();
        out.resize(old + std::max<size_t>(1 << 16, n));
        ZOutBuf ob{out.data() + old, out.size() - old, 0};
        last = z.decompress_stream(ds, &ob, &in);
        out.resize(old + ob.pos);
        if (z.is_error(last)) err = z.error_name(last);
    }
    // flush what the decoder still holds of the last frame
    while (err.empty() && last != 0) {
        const size_t old = out.size();
        out.resize(old + (1 << 16));
        ZOutBuf ob{out.data() + old, out.size() - old, 0};
        last = z.decompress_stream(ds, &ob, &in);
        out.resize(old + ob.pos);
        if (z.is_error(last)) err = z.error_name(last);
        else if (last != 0 && ob.pos == 0) err = "truncated zstd frame";
    }
    z.free_dstream(ds);
    if (!err.empty()) bad("zstd decompression failed: " + err);
    return out;
}

std::vector<uint8_t> zstd_compress(const std::vector<uint8_t>& src, int level) {
    const Zstd& z = zstd();
    std::vector<uint8_t> out(z.compress_bound(src.size()));
    const size_t r = z.compress(out.data(), out.size(), src.data(), src.size(), level);
    if (z.is_error(r)) throw Error{BST_ERR_INVALID_ARGUMENT, std::string("zstd compression failed: ") + z.error_name(r)};
    out.resize(r);
    return out;
}

// ---- CRC32C (Castagnoli, reflected polynomial 0x82F63B78) --------------------
uint32_t crc32c(const uint8_t* p, size_t n) {
    static uint32_t table[256];
    static bool init = false;
    if (!init) {
        for (uint32_t i = 0; i < 256; ++i) {
            uint32_t c = i;
            for (int k = 0; k < 8; ++k) c = (c & 1u) ? (c >> 1) ^ 0x82F63B78u : c >> 1;
            table[i] = c;
        }
        init = true;
    }
    uint32_t c = 0xFFFFFFFFu;
    for (size_t i = 0; i < n; ++i) c = table[(c ^ p[i]) & 0xFFu] ^ (c >> 8);
    return c ^ 0xFFFFFFFFu;
}

// ---- the schema in memory ----------------------------------------------------
struct TreeS {
    uint32_t num_nodes = 0;
    std::vector<double> split_indices, thresholds, children_left, children_right, leaf_values;
    std::vector<uint8_t> default_left;
    std::vector<uint32_t> cat_nodes;
    std::vector<std::vector<uint32_t>> cat_sets;
    bool has_gains = false, has_covers = false, has_linear = false;
    std::vector<double> gains, covers;
};
struct ModelS {
    uint64_t num_features = 0, num_groups = 1, n_groups = 1;
    bool has_tree_groups = false;
    std::vector<double> tree_groups, base_score;
    std::vector<TreeS> trees;
    std::string output_transform = "identity";
};

const char* transform_name(int objective) {
    const int t = transform_of(objective);
    return t == 1 ? "sigmoid" : (t == 2 ? "softmax" : "identity");
}

ModelS to_schema(const Model& m) {
    ModelS s;
    s.num_features = m.n_features;
    s.num_groups = m.n_groups;
    s.n_groups = m.n_groups;
    s.base_score.assign(m.base.begin(), m.base.end());
    s.output_transform = transform_name(m.objective);
    s.has_tree_groups = m.n_groups > 1;
    for (const HostTree& t : m.trees) {
        TreeS ts;
        const size_t n = t.split_index.size();
        ts.num_nodes = (uint32_t)n;
        for (size_t i = 0; i < n; ++i) {
            const bool leaf = t.is_leaf[i] != 0;
            ts.split_indices.push_back(leaf ? 0.0 : (double)t.split_index[i]);
            ts.thresholds.push_back(leaf ? 0.0 : (double)t.threshold[i]);
            ts.children_left.push_back(leaf ? 0.0 : (double)t.left[i]);
            ts.children_right.push_back(leaf ? 0.0 : (double)t.right[i]);
            ts.default_left.push_back(leaf ? 0 : t.default_left[i]);
            ts.leaf_values.push_back(leaf ? (double)t.leaf[i] : 0.0);
            if (!leaf && t.split_type[i] == 1) {  // categories going right, ascending
                std::vector<uint32_t> cats;
                const uint32_t ss = t.seg_size.empty() ? 0 : t.seg_size[i];
                for (uint32_t w = 0; w < ss; ++w) {
                    const uint32_t word = t.cat_words[t.seg_start[i] + w];
                    for (uint32_t b = 0; b < 32; ++b)
                        if ((word >> b) & 1u) cats.push_back(w * 32 + b);
                }
                if (!cats.empty()) {
                    ts.cat_nodes.push_back((uint32_t)i);
                    ts.cat_sets.push_back(std::move(cats));
                }
            }
        }
        ts.has_gains = !t.gain.empty();
        ts.has_covers = !t.cover.empty();
        ts.gains.assign(t.gain.begin(), t.gain.end());
        ts.covers.assign(t.cover.begin(), t.cover.end());
        s.trees.push_back(std::move(ts));
        s.tree_groups.push_back((double)t.group);
    }
    return s;
}

uint32_t as_index(double v, const char* what) {
    if (!(v >= 0.0) || v > 4294967295.0 || v != std::floor(v)) bad(std::string("non-integer ") + what);
    return (uint32_t)v;
}

// convert.rs:193-420 (validation as the reference's, then the runtime tree)
std::unique_ptr<Model> from_schema(ModelS& s) {
    auto m = std::make_unique<Model>();
    if (s.n_groups == 0) bad("n_groups must be at least 1");
    if (s.num_groups != s.n_groups) bad("meta.num_groups and forest.n_groups differ");
    if (s.base_score.size() != s.n_groups) bad("forest base_score must have length n_groups");
    if (s.has_tree_groups && s.tree_groups.size() != s.trees.size())
        bad("forest tree_groups must have the same length as trees");
    if (s.num_features > 0xFFFFFFFFull || s.n_groups > 0xFFFFull) bad("sizes out of range");
    m->n_features = (uint32_t)s.num_features;
    m->n_groups = (uint32_t)s.n_groups;
    for (double b : s.base_score) m->base.push_back((float)b);
    if (s.output_transform == "identity")
        m->objective = BST_OBJ_SQUARED;
    else if (s.output_transform == "sigmoid")
        m->objective = BST_OBJ_LOGISTIC;
    else if (s.output_transform == "softmax")
        m->objective = BST_OBJ_SOFTMAX;
    else
        bad("unknown output_transform \"" + s.output_transform + "\"");
    for (size_t ti = 0; ti < s.trees.size(); ++ti) {
        TreeS& ts = s.trees[ti];
        const size_t n = ts.num_nodes;
        if (n == 0) bad("a tree needs at least one node");
        if (ts.split_indices.size() != n || ts.thresholds.size() != n || ts.children_left.size() != n ||
            ts.children_right.size() != n || ts.default_left.size() != n)
            bad("tree schema arrays must all have length num_nodes");
        if (ts.leaf_values.size() != n) bad("tree schema leaf_values must have length num_nodes");
        if (ts.has_gains && ts.gains.size() != n) bad("tree schema gains must have length num_nodes");
        if (ts.has_covers && ts.covers.size() != n) bad("tree schema covers must have length num_nodes");
        if (ts.cat_nodes.size() != ts.cat_sets.size())
            bad("categories.node_indices and categories.category_sets must have the same length");
        if (ts.has_linear) unsupported("linear leaves are not on this path");
        HostTree t;
        for (size_t i = 0; i < n; ++i) t.alloc();
        const uint32_t g = s.has_tree_groups ? as_index(s.tree_groups[ti], "tree group") : 0u;
        if (g >= m->n_groups) bad("forest tree group out of range");
        t.group = g;
        for (size_t i = 0; i < n; ++i) {
            const uint32_t l = as_index(ts.children_left[i], "child"), r = as_index(ts.children_right[i], "child");
            t.is_leaf[i] = l == 0 ? 1 : 0;  // 0 is the "no child" sentinel (convert.rs:375-377)
            t.split_index[i] = as_index(ts.split_indices[i], "split index");
            t.threshold[i] = (float)ts.thresholds[i];
            t.left[i] = l;
            t.right[i] = r;
            t.default_left[i] = ts.default_left[i];
            t.leaf[i] = (float)ts.leaf_values[i];
            if (ts.has_gains) t.gain[i] = (float)ts.gains[i];
            if (ts.has_covers) t.cover[i] = (float)ts.covers[i];
            if (!t.is_leaf[i]) {
                if (l >= n || r == 0 || r >= n) bad("child index out of range");
                if (t.split_index[i] >= m->n_features) bad("split index out of range");
            }
        }
        if (!ts.cat_nodes.empty()) {
            t.seg_start.assign(n, 0);
            t.seg_size.assign(n, 0);
            for (size_t k = 0; k < ts.cat_nodes.size(); ++k) {
                const uint32_t nd = ts.cat_nodes[k];
                if (nd >= n) bad("categories contain an out-of-bounds node index");
                if (t.is_leaf[nd]) bad("categories on a leaf");
                const auto& cats = ts.cat_sets[k];
                uint32_t mx = 0;
                for (uint32_t c : cats) mx = std::max(mx, c);
                const uint32_t words = cats.empty() ? 0 : (mx >> 5) + 1;
                t.split_type[nd] = 1;
                t.seg_start[nd] = (uint32_t)t.cat_words.size();
                t.seg_size[nd] = words;
                t.cat_words.resize(t.cat_words.size() + words, 0u);
                for (uint32_t c : cats) t.cat_words[t.seg_start[nd] + (c >> 5)] |= 1u << (c & 31u);
            }
        }
        // a tree: every node reached from the root at most once
        std::vector<uint8_t> seen(n, 0);
        std::vector<uint32_t> stack{0};
        while (!stack.empty()) {
            const uint32_t i = stack.back();
            stack.pop_back();
            if (seen[i]) bad("tree structure has a cycle or a shared child");
            seen[i] = 1;
            if (!t.is_leaf[i]) {
                stack.push_back(t.left[i]);
                stack.push_back(t.right[i]);
            }
        }
        m->trees.push_back(std::move(t));
    }
    return m;
}

// ---- JSON ---------------------------------------------------------------------
struct JsonOut {
    std::string s;
    bool pretty = false;
    int depth = 0;
    void nl() {
        if (!pretty) return;
        s += '\n';
        s.append((size_t)depth * 2, ' ');
    }
    void num(double v) {
        if (!std::isfinite(v)) {  // JSON has no non-finite numbers (written as null)
            s += "null";
            return;
        }
        char buf[32];
        const auto r = std::to_chars(buf, buf + sizeof(buf), v);
        s.append(buf, r.ptr);
        // keep floats recognisable as floats: "1" -> "1.0"
        bool has = false;
        for (const char* p = buf; p < r.ptr; ++p)
            if (*p == '.' || *p == 'e' || *p == 'n' || *p == 'i') has = true;
        if (!has) s += ".0";
    }
    void uint(uint64_t v) {
        char buf[24];
        const auto r = std::to_chars(buf, buf + sizeof(buf), v);
        s.append(buf, r.ptr);
    }
    void str(const std::string& v) {
        s += '"';
        for (char c : v) {
            if (c == '"' || c == '\\') s += '\\';
            s += c;
        }
        s += '"';
    }
    template <typename F>
    void obj(F body) {
        s += '{';
        ++depth;
        first = true;
        body();
        --depth;
        nl();
        s += '}';
        first = false;
    }
    bool first = true;
    void key(const char* k) {
        if (!first) s += ',';
        first = false;
        nl();
        str(k);
        s += pretty ? ": " : ":";
    }
    template <typename T, typename W>
    void arr(const std::vector<T>& v, W write) {
        s += '[';
        ++depth;
        for (size_t i = 0; i < v.size(); ++i) {
            if (i) s += ',';
            nl();
            write(v[i]);
        }
        --depth;
        if (!v.empty()) nl();
        s += ']';
        first = false;
    }
};

std::string write_json(const ModelS& m, bool pretty) {
    JsonOut o;
    o.pretty = pretty;
    o.obj([&] {
        o.key("bstr_version");
        o.uint(SCHEMA_VERSION);
        o.key("model_type");
        o.str("gbdt");
        o.key("model");
        o.obj([&] {
            o.key("meta");
            o.obj([&] {
                o.key("num_features");
                o.uint(m.num_features);
                o.key("num_groups");
                o.uint(m.num_groups);
            });
            o.key("forest");
            o.obj([&] {
                o.key("trees");
                o.arr(m.trees, [&](const TreeS& t) {
                    o.obj([&] {
                        o.key("num_nodes");
                        o.uint(t.num_nodes);
                        auto ints = [&](const char* k, const std::vector<double>& v) {
                            o.key(k);
                            o.arr(v, [&](double x) { o.uint((uint64_t)x); });
                        };
                        auto floats = [&](const char* k, const std::vector<double>& v) {
                            o.key(k);
                            o.arr(v, [&](double x) { o.num(x); });
                        };
                        ints("split_indices", t.split_indices);
                        floats("thresholds", t.thresholds);
                        ints("children_left", t.children_left);
                        ints("children_right", t.children_right);
                        o.key("default_left");
                        o.arr(t.default_left, [&](uint8_t b) { o.s += b ? "true" : "false"; });
                        o.key("leaf_values");
                        o.obj([&] {
                            o.key("type");
                            o.str("scalar");
                            floats("values", t.leaf_values);
                        });
                        if (!t.cat_nodes.empty()) {
                            o.key("categories");
                            o.obj([&] {
                                o.key("node_indices");
                                o.arr(t.cat_nodes, [&](uint32_t x) { o.uint(x); });
                                o.key("category_sets");
                                o.arr(t.cat_sets, [&](const std::vector<uint32_t>& c) {
                                    o.arr(c, [&](uint32_t x) { o.uint(x); });
                                });
                            });
                        }
                        if (t.has_gains) floats("gains", t.gains);
                        if (t.has_covers) floats("covers", t.covers);
                    });
                });
                if (m.has_tree_groups) {
                    o.key("tree_groups");
                    o.arr(m.tree_groups, [&](double x) { o.uint((uint64_t)x); });
                }
                o.key("n_groups");
                o.uint(m.n_groups);
                o.key("base_score");
                o.arr(m.base_score, [&](double x) { o.num(x); });
            });
            o.key("output_transform");
            o.str(m.output_transform);
        });
    });
    if (pretty) o.s += '\n';
    return o.s;
}

// Schema-directed JSON reader: objects are read key by key, unknown keys
// are skipped, number arrays parse straight into vectors.
struct JsonIn {
    const char* p;
    const char* e;
    void ws() {
        while (p < e && (*p == ' ' || *p == '\n' || *p == '\r' || *p == '\t')) ++p;
    }
    bool peek(char c) {
        ws();
        return p < e && *p == c;
    }
    void expect(char c) {
        ws();
        if (p >= e || *p != c) bad(std::string("JSON: expected '") + c + "'");
        ++p;
    }
    bool null() {
        ws();
        if (e - p >= 4 && std::memcmp(p, "null", 4) == 0) {
            p += 4;
            return true;
        }
        return false;
    }
    std::string str() {
        expect('"');
        std::string out;
        while (p < e && *p != '"') {
            char c = *p++;
            if (c == '\\') {
                if (p >= e) bad("JSON: bad escape");
                const char x = *p++;
                switch (x) {
                    case 'n': c = '\n'; break;
                    case 't': c = '\t'; break;
                    case 'r': c = '\r'; break;
                    case 'b': c = '\b'; break;
                    case 'f': c = '\f'; break;
                    case 'u': {
                        if (e - p < 4) bad("JSON: bad escape");
                        unsigned v = 0;
                        std::from_chars(p, p + 4, v, 16);
                        p += 4;
                        c = v < 128 ? (char)v : '?';
                        break;
                    }
                    default: c = x;
                }
            }
            out += c;
        }
        expect('"');
        return out;
    }
    double num() {
        ws();
        if (null()) return std::numeric_limits<double>::quiet_NaN();
        double v = 0.0;
        const auto r = std::from_chars(p, e, v);
        if (r.ec != std::errc()) bad("JSON: expected a number");
        p = r.ptr;
        return v;
    }
    bool boolean() {
        ws();
        if (e - p >= 4 && std::memcmp(p, "true", 4) == 0) {
            p += 4;
            return true;
        }
        if (e - p >= 5 && std::memcmp(p, "false", 5) == 0) {
            p += 5;
            return false;
        }
        bad("JSON: expected a boolean");
    }
    template <typename F>
    void array(F each) {
        expect('[');
        if (peek(']')) {
            ++p;
            return;
        }
        for (;;) {
            each();
            ws();
            if (p < e && *p == ',') {
                ++p;
                continue;
            }
            expect(']');
            return;
        }
    }
    template <typename F>
    void object(F field) {
        expect('{');
        if (peek('}')) {
            ++p;
            return;
        }
        for (;;) {
            const std::string k = str();
            expect(':');
            field(k);
            ws();
            if (p < e && *p == ',') {
                ++p;
                continue;
            }
            expect('}');
            return;
        }
    }
    void skip() {
        ws();
        if (p >= e) bad("JSON: unexpected end");
        if (*p == '{')
            object([&](const std::string&) { skip(); });
        else if (*p == '[')
            array([&] { skip(); });
        else if (*p == '"')
            str();
        else if (*p == 't' || *p == 'f')
            boolean();
        else
            num();
    }
    void numbers(std::vector<double>& v) {
        v.clear();
        array([&] { v.push_back(num()); });
    }
};

ModelS read_json(const char* data, size_t len) {
    JsonIn in{data, data + len};
    ModelS m;
    uint64_t version = 0;
    std::string type;
    bool have_model = false;
    in.object([&](const std::string& k) {
        if (k == "bstr_version") {
            version = (uint64_t)in.num();
        } else if (k == "model_type") {
            type = in.str();
        } else if (k == "model") {
            in.ws();
            if (!in.peek('{')) bad("\"model\" must be an object");
            have_model = true;
            in.object([&](const std::string& mk) {
                if (mk == "meta") {
                    in.object([&](const std::string& f) {
                        if (f == "num_features")
                            m.num_features = (uint64_t)in.num();
                        else if (f == "num_groups")
                            m.num_groups = (uint64_t)in.num();
                        else
                            in.skip();
                    });
                } else if (mk == "forest") {
                    in.object([&](const std::string& f) {
                        if (f == "trees") {
                            in.array([&] {
                                TreeS t;
                                in.object([&](const std::string& tk) {
                                    if (tk == "num_nodes") {
                                        t.num_nodes = (uint32_t)in.num();
                                    } else if (tk == "split_indices") {
                                        in.numbers(t.split_indices);
                                    } else if (tk == "thresholds") {
                                        in.numbers(t.thresholds);
                                    } else if (tk == "children_left") {
                                        in.numbers(t.children_left);
                                    } else if (tk == "children_right") {
                                        in.numbers(t.children_right);
                                    } else if (tk == "default_left") {
                                        in.array([&] { t.default_left.push_back(in.boolean() ? 1 : 0); });
                                    } else if (tk == "leaf_values") {
                                        std::string lt;
                                        in.object([&](const std::string& lk) {
                                            if (lk == "type") {
                                                lt = in.str();
                                            } else if (lk == "values") {
                                                in.array([&] {
                                                    if (in.peek('[')) {  // vector leaves: K = 1 only
                                                        std::vector<double> v;
                                                        in.numbers(v);
                                                        if (v.size() != 1)
                                                            unsupported("vector leaves with more than one value");
                                                        t.leaf_values.push_back(v[0]);
                                                    } else {
                                                        t.leaf_values.push_back(in.num());
                                                    }
                                                });
                                            } else {
                                                in.skip();
                                            }
                                        });
                                        if (lt != "scalar" && lt != "vector") bad("unknown leaf_values type");
                                    } else if (tk == "categories") {
                                        in.object([&](const std::string& ck) {
                                            if (ck == "node_indices") {
                                                in.array([&] { t.cat_nodes.push_back(as_index(in.num(), "node index")); });
                                            } else if (ck == "category_sets") {
                                                in.array([&] {
                                                    std::vector<uint32_t> cs;
                                                    in.array([&] { cs.push_back(as_index(in.num(), "category")); });
                                                    t.cat_sets.push_back(std::move(cs));
                                                });
                                            } else {
                                                in.skip();
                                            }
                                        });
                                    } else if (tk == "linear_coefficients") {
                                        in.object([&](const std::string& lk) {
                                            if (lk == "node_indices")
                                                in.array([&] {
                                                    in.num();
                                                    t.has_linear = true;
                                                });
                                            else
                                                in.skip();
                                        });
                                    } else if (tk == "gains") {
                                        if (!in.null()) {
                                            t.has_gains = true;
                                            in.numbers(t.gains);
                                        }
                                    } else if (tk == "covers") {
                                        if (!in.null()) {
                                            t.has_covers = true;
                                            in.numbers(t.covers);
                                        }
                                    } else {
                                        in.skip();
                                    }
                                });
                                m.trees.push_back(std::move(t));
                            });
                        } else if (f == "tree_groups") {
                            if (!in.null()) {
                                m.has_tree_groups = true;
                                in.numbers(m.tree_groups);
                            }
                        } else if (f == "n_groups") {
                            m.n_groups = (uint64_t)in.num();
                        } else if (f == "base_score") {
                            in.numbers(m.base_score);
                        } else {
                            in.skip();
                        }
                    });
                } else if (mk == "output_transform") {
                    m.output_transform = in.str();
                } else {
                    in.skip();
                }
            });
        } else {
            in.skip();
        }
    });
    if (version > MAX_SUPPORTED_VERSION) bad("unsupported schema version " + std::to_string(version));
    if (type != "gbdt") bad("model type \"" + type + "\" is not gbdt");
    if (!have_model) bad("missing \"model\"");
    return m;
}

// ---- MessagePack ------------------------------------------------------------
struct PackOut {
    std::vector<uint8_t> b;
    void u8(uint8_t v) { b.push_back(v); }
    void be(uint64_t v, int bytes) {
        for (int i = bytes - 1; i >= 0; --i) b.push_back((uint8_t)(v >> (8 * i)));
    }
    void uint(uint64_t v) {
        if (v < 128) {
            u8((uint8_t)v);
        } else if (v <= 0xFF) {
            u8(0xcc);
            be(v, 1);
        } else if (v <= 0xFFFF) {
            u8(0xcd);
            be(v, 2);
        } else if (v <= 0xFFFFFFFFull) {
            u8(0xce);
            be(v, 4);
        } else {
            u8(0xcf);
            be(v, 8);
        }
    }
    void f64(double v) {
        uint64_t bits;
        std::memcpy(&bits, &v, 8);
        u8(0xcb);
        be(bits, 8);
    }
    void boolean(bool v) { u8(v ? 0xc3 : 0xc2); }
    void str(const std::string& s) {
        const size_t n = s.size();
        if (n < 32) {
            u8((uint8_t)(0xa0 | n));
        } else if (n <= 0xFF) {
            u8(0xd9);
            be(n, 1);
        } else {
            u8(0xda);
            be(n, 2);
        }
        b.insert(b.end(), s.begin(), s.end());
    }
    void array(size_t n) {
        if (n < 16) {
            u8((uint8_t)(0x90 | n));
        } else if (n <= 0xFFFF) {
            u8(0xdc);
            be(n, 2);
        } else {
            u8(0xdd);
            be(n, 4);
        }
    }
    void map(size_t n) {
        if (n < 16) {
            u8((uint8_t)(0x80 | n));
        } else if (n <= 0xFFFF) {
            u8(0xde);
            be(n, 2);
        } else {
            u8(0xdf);
            be(n, 4);
        }
    }
};

std::vector<uint8_t> write_msgpack(const ModelS& m) {
    PackOut o;
    o.map(3);
    o.str("meta");
    o.map(2);
    o.str("num_features");
    o.uint(m.num_features);
    o.str("num_groups");
    o.uint(m.num_groups);
    o.str("forest");
    o.map(m.has_tree_groups ? 4 : 3);
    o.str("trees");
    o.array(m.trees.size());
    for (const TreeS& t : m.trees) {
        o.map(7 + (t.cat_nodes.empty() ? 0 : 1) + (t.has_gains ? 1 : 0) + (t.has_covers ? 1 : 0));
        o.str("num_nodes");
        o.uint(t.num_nodes);
        auto ints = [&](const char* k, const std::vector<double>& v) {
            o.str(k);
            o.array(v.size());
            for (double x : v) o.uint((uint64_t)x);
        };
        auto floats = [&](const char* k, const std::vector<double>& v) {
            o.str(k);
            o.array(v.size());
            for (double x : v) o.f64(x);
        };
        ints("split_indices", t.split_indices);
        floats("thresholds", t.thresholds);
        ints("children_left", t.children_left);
        ints("children_right", t.children_right);
        o.str("default_left");
        o.array(t.default_left.size());
        for (uint8_t x : t.default_left) o.boolean(x != 0);
        o.str("leaf_values");
        o.map(2);
        o.str("type");
        o.str("scalar");
        floats("values", t.leaf_values);
        if (!t.cat_nodes.empty()) {
            o.str("categories");
            o.map(2);
            o.str("node_indices");
            o.array(t.cat_nodes.size());
            for (uint32_t x : t.cat_nodes) o.uint(x);
            o.str("category_sets");
            o.array(t.cat_sets.size());
            for (const auto& cs : t.cat_sets) {
                o.array(cs.size());
                for (uint32_t x : cs) o.uint(x);
            }
        }
        if (t.has_gains) floats("gains", t.gains);
        if (t.has_covers) floats("covers", t.covers);
    }
    if (m.has_tree_groups) {
        o.str("tree_groups");
        o.array(m.tree_groups.size());
        for (double x : m.tree_groups) o.uint((uint64_t)x);
    }
    o.str("n_groups");
    o.uint(m.n_groups);
    o.str("base_score");
    o.array(m.base_score.size());
    for (double x : m.base_score) o.f64(x);
    o.str("output_transform");
    o.str(m.output_transform);
    return o.b;
}

struct PackIn {
    const uint8_t* p;
    const uint8_t* e;
    uint8_t byte() {
        if (p >= e) bad("MessagePack: unexpected end");
        return *p++;
    }
    uint64_t be(int bytes) {
        if (e - p < bytes) bad("MessagePack: unexpected end");
        uint64_t v = 0;
        for (int i = 0; i < bytes; ++i) v = (v << 8) | *p++;
        return v;
    }
    uint8_t peek() {
        if (p >= e) bad("MessagePack: unexpected end");
        return *p;
    }
    bool nil() {
        if (peek() == 0xc0) {
            ++p;
            return true;
        }
        return false;
    }
    double num() {  // any integer or float
        const uint8_t t = byte();
        if (t < 0x80) return (double)t;
        if (t >= 0xe0) return (double)(int8_t)t;
        switch (t) {
            case 0xcc: return (double)be(1);
            case 0xcd: return (double)be(2);
            case 0xce: return (double)be(4);
            case 0xcf: return (double)be(8);
            case 0xd0: return (double)(int8_t)be(1);
            case 0xd1: return (double)(int16_t)be(2);
            case 0xd2: return (double)(int32_t)be(4);
            case 0xd3: return (double)(int64_t)be(8);
            case 0xca: {
                const uint32_t bits = (uint32_t)be(4);
                float f;
                std::memcpy(&f, &bits, 4);
                return f;
            }
            case 0xcb: {
                const uint64_t bits = be(8);
                double d;
                std::memcpy(&d, &bits, 8);
                return d;
            }
            case 0xc0: return std::numeric_limits<double>::quiet_NaN();
        }
        bad("MessagePack: expected a number");
    }
    bool boolean() {
        const uint8_t t = byte();
        if (t == 0xc2) return false;
        if (t == 0xc3) return true;
        bad("MessagePack: expected a boolean");
    }
    std::string str() {
        const uint8_t t = byte();
        size_t n;
        if ((t & 0xe0) == 0xa0)
            n = t & 0x1f;
        else if (t == 0xd9)
            n = be(1);
        else if (t == 0xda)
            n = be(2);
        else if (t == 0xdb)
            n = be(4);
        else
            bad("MessagePack: expected a string");
        if ((size_t)(e - p) < n) bad("MessagePack: unexpected end");
        std::string s((const char*)p, n);
        p += n;
        return s;
    }
    size_t array() {
        const uint8_t t = byte();
        if ((t & 0xf0) == 0x90) return t & 0x0f;
        if (t == 0xdc) return be(2);
        if (t == 0xdd) return be(4);
        bad("MessagePack: expected an array");
    }
    size_t map() {
        const uint8_t t = byte();
        if ((t & 0xf0) == 0x80) return t & 0x0f;
        if (t == 0xde) return be(2);
        if (t == 0xdf) return be(4);
        bad("MessagePack: expected a map");
    }
    bool is_map() { return (peek() & 0xf0) == 0x80 || peek() == 0xde || peek() == 0xdf; }
    bool is_array() { return (peek() & 0xf0) == 0x90 || peek() == 0xdc || peek() == 0xdd; }
    bool is_str() { return (peek() & 0xe0) == 0xa0 || peek() == 0xd9 || peek() == 0xda || peek() == 0xdb; }
    void skip() {
        const uint8_t t = peek();
        if (is_map()) {
            const size_t n = map();
            for (size_t i = 0; i < 2 * n; ++i) skip();
        } else if (is_array()) {
            const size_t n = array();
            for (size_t i = 0; i < n; ++i) skip();
        } else if (is_str()) {
            str();
        } else if (t == 0xc2 || t == 0xc3) {
            boolean();
        } else if (t == 0xc4 || t == 0xc5 || t == 0xc6) {  // bin
            ++p;
            const size_t n = be(t == 0xc4 ? 1 : (t == 0xc5 ? 2 : 4));
            if ((size_t)(e - p) < n) bad("MessagePack: unexpected end");
            p += n;
        } else {
            num();
        }
    }
    void numbers(std::vector<double>& v) {
        const size_t n = array();
        v.clear();
        v.reserve(n);
        for (size_t i = 0; i < n; ++i) v.push_back(num());
    }
    template <typename F>
    void fields(F field) {
        const size_t n = map();
        for (size_t i = 0; i < n; ++i) field(str());
    }
};

ModelS read_msgpack(const uint8_t* data, size_t len) {
    PackIn in{data, data + len};
    ModelS m;
    in.fields([&](const std::string& mk) {
        if (mk == "meta") {
            in.fields([&](const std::string& f) {
                if (f == "num_features")
                    m.num_features = (uint64_t)in.num();
                else if (f == "num_groups")
                    m.num_groups = (uint64_t)in.num();
                else
                    in.skip();
            });
        } else if (mk == "forest") {
            in.fields([&](const std::string& f) {
                if (f == "trees") {
                    const size_t nt = in.array();
                    for (size_t ti = 0; ti < nt; ++ti) {
                        TreeS t;
                        in.fields([&](const std::string& tk) {
                            if (tk == "num_nodes") {
                                t.num_nodes = (uint32_t)in.num();
                            } else if (tk == "split_indices") {
                                in.numbers(t.split_indices);
                            } else if (tk == "thresholds") {
                                in.numbers(t.thresholds);
                            } else if (tk == "children_left") {
                                in.numbers(t.children_left);
                            } else if (tk == "children_right") {
                                in.numbers(t.children_right);
                            } else if (tk == "default_left") {
                                const size_t n = in.array();
                                for (size_t i = 0; i < n; ++i) t.default_left.push_back(in.boolean() ? 1 : 0);
                            } else if (tk == "leaf_values") {
                                std::string lt;
                                in.fields([&](const std::string& lk) {
                                    if (lk == "type") {
                                        lt = in.str();
                                    } else if (lk == "values") {
                                        const size_t n = in.array();
                                        for (size_t i = 0; i < n; ++i) {
                                            if (in.is_array()) {
                                                std::vector<double> v;
                                                in.numbers(v);
                                                if (v.size() != 1) unsupported("vector leaves with more than one value");
                                                t.leaf_values.push_back(v[0]);
                                            } else {
                                                t.leaf_values.push_back(in.num());
                                            }
                                        }
                                    } else {
                                        in.skip();
                                    }
                                });
                                if (lt != "scalar" && lt != "vector") bad("unknown leaf_values type");
                            } else if (tk == "categories") {
                                in.fields([&](const std::string& ck) {
                                    if (ck == "node_indices") {
                                        const size_t n = in.array();
                                        for (size_t i = 0; i < n; ++i) t.cat_nodes.push_back(as_index(in.num(), "node index"));
                                    } else if (ck == "category_sets") {
                                        const size_t n = in.array();
                                        for (size_t i = 0; i < n; ++i) {
                                            const size_t k = in.array();
                                            std::vector<uint32_t> cs;
                                            for (size_t j = 0; j < k; ++j) cs.push_back(as_index(in.num(), "category"));
                                            t.cat_sets.push_back(std::move(cs));
                                        }
                                    } else {
                                        in.skip();
                                    }
                                });
                            } else if (tk == "linear_coefficients") {
                                in.fields([&](const std::string& lk) {
                                    if (lk == "node_indices") {
                                        const size_t n = in.array();
                                        for (size_t i = 0; i < n; ++i) in.num();
                                        if (n) t.has_linear = true;
                                    } else {
                                        in.skip();
                                    }
                                });
                            } else if (tk == "gains") {
                                if (!in.nil()) {
                                    t.has_gains = true;
                                    in.numbers(t.gains);
                                }
                            } else if (tk == "covers") {
                                if (!in.nil()) {
                                    t.has_covers = true;
                                    in.numbers(t.covers);
                                }
                            } else {
                                in.skip();
                            }
                        });
                        m.trees.push_back(std::move(t));
                    }
                } else if (f == "tree_groups") {
                    if (!in.nil()) {
                        m.has_tree_groups = true;
                        in.numbers(m.tree_groups);
                    }
                } else if (f == "n_groups") {
                    m.n_groups = (uint64_t)in.num();
                } else if (f == "base_score") {
                    in.numbers(m.base_score);
                } else {
                    in.skip();
                }
            });
        } else if (mk == "output_transform") {
            // a unit variant: its name, or (other encoders) a one-key map or an index
            if (in.is_str()) {
                m.output_transform = in.str();
            } else if (in.is_map()) {
                const size_t n = in.map();
                if (n != 1) bad("output_transform");
                m.output_transform = in.str();
                in.skip();
            } else {
                const double v = in.num();
                m.output_transform = v == 1.0 ? "sigmoid" : (v == 2.0 ? "softmax" : "identity");
            }
        } else {
            in.skip();
        }
    });
    return m;
}

// level 0: plain MessagePack (0x01); 1-22: zstd at that level (0x02)
// (binary.rs:60-91; levels above 22 are rejected, binary.rs:56-59).
std::vector<uint8_t> write_bstr(const ModelS& m, int level) {
    if (level < 0 || level > 22)
        throw Error{BST_ERR_INVALID_ARGUMENT, "compression level " + std::to_string(level) + " is outside 0-22"};
    std::vector<uint8_t> payload = write_msgpack(m);
    if (level > 0) payload = zstd_compress(payload, level);
    std::vector<uint8_t> out(HEADER_SIZE, 0);
    std::memcpy(out.data(), "BSTR", 4);
    for (int i = 0; i < 4; ++i) out[4 + i] = (uint8_t)(SCHEMA_VERSION >> (8 * i));
    out[8] = level > 0 ? 0x02 : 0x01;
    out[9] = 1;  // GBDT
    out.insert(out.end(), payload.begin(), payload.end());
    const uint64_t len = payload.size();
    const uint32_t crc = crc32c(payload.data(), payload.size());
    uint8_t tr[TRAILER_SIZE] = {0};
    for (int i = 0; i < 8; ++i) tr[i] = (uint8_t)(len >> (8 * i));
    for (int i = 0; i < 4; ++i) tr[8 + i] = (uint8_t)(crc >> (8 * i));
    out.insert(out.end(), tr, tr + TRAILER_SIZE);
    return out;
}

ModelS read_bstr(const uint8_t* d, size_t n) {
    if (n < HEADER_SIZE + TRAILER_SIZE) bad("file too small");
    if (std::memcmp(d, "BSTR", 4) != 0) bad("missing BSTR magic");
    uint32_t version = 0;
    for (int i = 0; i < 4; ++i) version |= (uint32_t)d[4 + i] << (8 * i);
    if (version > MAX_SUPPORTED_VERSION) bad("unsupported schema version " + std::to_string(version));
    const uint8_t format = d[8], type = d[9];
    if (format == 0x00) bad("binary header format 0x00 (Json) is not valid for .bstr");
    if (format != 0x01 && format != 0x02) bad("unknown format byte");
    if (type != 1) bad("model type " + std::to_string(type) + " is not gbdt");
    const uint8_t* tr = d + n - TRAILER_SIZE;
    uint64_t len = 0;
    uint32_t crc = 0;
    for (int i = 0; i < 8; ++i) len |= (uint64_t)tr[i] << (8 * i);
    for (int i = 0; i < 4; ++i) crc |= (uint32_t)tr[8 + i] << (8 * i);
    const uint8_t* payload = d + HEADER_SIZE;
    const size_t plen = n - HEADER_SIZE - TRAILER_SIZE;
    if (len != plen) bad("payload length mismatch");
    if (crc32c(payload, plen) != crc) bad("checksum mismatch");
    if (format == 0x02) {
        const std::vector<uint8_t> raw = zstd_decode_all(payload, plen);
        return read_msgpack(raw.data(), raw.size());
    }
    return read_msgpack(payload, plen);
}

}  // namespace

uint32_t crc32c_bytes(const uint8_t* p, size_t n) { return crc32c(p, n); }

std::string model_to_json(const Model& m, bool pretty) { return write_json(to_schema(m), pretty); }

std::vector<uint8_t> model_to_bstr(const Model& m, int level) { return write_bstr(to_schema(m), level); }

std::unique_ptr<Model> model_from_bytes(const uint8_t* data, size_t len) {
    ModelS s = len >= 4 && std::memcmp(data, "BSTR", 4) == 0 ? read_bstr(data, len)
                                                              : read_json((const char*)data, len);
    return from_schema(s);
}

}  // namespace bst
