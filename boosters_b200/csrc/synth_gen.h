// synth_gen.h — seeded synthetic workloads, counter-based so any consumer
// (engine, checker, benchmark) regenerates identical bytes.
//
// Every cell is a pure function of (seed, stream, column, row): a splitmix64
// hash of the counter, turned into uniforms (53-bit) and normals
// (Box-Muller). `stream` selects an independent draw of rows (0 = training,
// 1 = held-out); model parameters (weights, column pairs, embeddings) depend
// on the seed only, so both streams share one ground truth.
//
// Header-only so that the engine library and the CPU checker each compile
// their own copy: a process that runs only the checker (the CPU baseline)
// never loads the engine. Functions return 0 on success, 1 on an invalid
// argument. Arrays are feature-major [F][n].
#pragma once
#include <cmath>
#include <cstdint>
#include <vector>

namespace synthgen {

inline uint64_t mix64(uint64_t x) {
    x += 0x9E3779B97F4A7C15ull;
    x = (x ^ (x >> 30)) * 0xBF58476D1CE4E5B9ull;
    x = (x ^ (x >> 27)) * 0x94D049BB133111EBull;
    return x ^ (x >> 31);
}

struct Rng {
    uint64_t key;
    Rng(uint64_t seed, uint64_t a, uint64_t b) {
        key = mix64(mix64(seed) ^ mix64(a * 0xD1342543DE82EF95ull + 0x632BE59BD9B4E019ull) ^ mix64(b + 0x2545F4914F6CDD1Dull));
    }
    uint64_t bits(uint64_t i) const { return mix64(key ^ mix64(i)); }
    double u01(uint64_t i) const { return (double)(bits(i) >> 11) * 0x1p-53; }
    double normal(uint64_t i) const {
        const double u1 = u01(2 * i), u2 = u01(2 * i + 1);
        return std::sqrt(-2.0 * std::log(1.0 - u1)) * std::cos(6.283185307179586 * u2);
    }
};

// purposes of independent sub-streams
enum : uint64_t { S_X = 1, S_NAN = 2, S_NOISE = 3, S_LABEL = 4, S_W = 5, S_PAIR = 6, S_CARD = 7, S_EMB = 8 };

inline int regression(uint64_t n, uint64_t F, uint64_t n_inf, uint64_t seed, uint64_t stream, float* x,
                      float* y) {
    if ((n && !x) || (n && !y)) return 1;
    std::vector<double> w(F, 0.0);
    const Rng rw(seed, S_W, 0);
    for (uint64_t j = 0; j < F && j < n_inf; ++j) w[j] = rw.normal(j);
#pragma omp parallel for schedule(static)
    for (int64_t f = 0; f < (int64_t)F; ++f) {
        const Rng r(seed, S_X, (stream << 32) ^ (uint64_t)f);
        for (uint64_t i = 0; i < n; ++i) x[(uint64_t)f * n + i] = (float)r.normal(i);
    }
    const Rng rn(seed, S_NOISE, stream);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        double s = 0.0;
        for (uint64_t j = 0; j < F && j < n_inf; ++j) s += (double)x[j * n + i] * w[j];
        y[i] = (float)(s + 0.1 * rn.normal((uint64_t)i));
    }
    return 0;
}

inline int binary(uint64_t n, uint64_t F, uint64_t n_nan_cols, uint64_t seed, uint64_t stream, float* x,
                  float* y) {
    if ((n && !x) || (n && !y) || F == 0) return 1;
    const Rng rp(seed, S_PAIR, 0);
    uint64_t pa[10], pb[10];
    for (int k = 0; k < 10; ++k) {
        pa[k] = rp.bits(2 * k) % F;
        pb[k] = rp.bits(2 * k + 1) % F;
    }
#pragma omp parallel for schedule(static)
    for (int64_t f = 0; f < (int64_t)F; ++f) {
        const Rng r(seed, S_X, (stream << 32) ^ (uint64_t)f);
        const Rng rm(seed, S_NAN, (stream << 32) ^ (uint64_t)f);
        const bool nan_col = (uint64_t)f < n_nan_cols;
        float* col = x + (uint64_t)f * n;
        for (uint64_t i = 0; i < n; ++i) {
            float v = (f % 2 == 0) ? (float)r.normal(i) : (float)r.u01(i);
            if (nan_col && rm.u01(i) < 0.1) v = NAN;
            col[i] = v;
        }
    }
    const Rng rn(seed, S_NOISE, stream), rl(seed, S_LABEL, stream);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        double s = 0.0;
        for (int k = 0; k < 10; ++k) {
            double a = x[pa[k] * n + i], b = x[pb[k] * n + i];
            if (std::isnan(a)) a = 0.0;
            if (std::isnan(b)) b = 0.0;
            s += a * b;
        }
        s += 0.5 * rn.normal((uint64_t)i);
        const double p = 1.0 / (1.0 + std::exp(-s));
        y[i] = rl.u01((uint64_t)i) < p ? 1.0f : 0.0f;
    }
    return 0;
}

inline int multiclass(uint64_t n, uint64_t n_num, uint64_t n_cat, uint64_t C, uint64_t seed, uint64_t stream,
                      float* x, float* y) {
    if ((n && !x) || (n && !y) || C < 2) return 1;
    const uint64_t F = n_num + n_cat;
    // cardinalities U{4..64}, Zipf(1.2) cumulative weights over ranks 1..K
    std::vector<uint32_t> card(n_cat);
    std::vector<std::vector<double>> cdf(n_cat);
    const Rng rc(seed, S_CARD, 0);
    for (uint64_t j = 0; j < n_cat; ++j) {
        card[j] = 4 + (uint32_t)(rc.bits(j) % 61);
        double tot = 0.0;
        for (uint32_t k = 1; k <= card[j]; ++k) tot += std::pow((double)k, -1.2);
        double acc = 0.0;
        for (uint32_t k = 1; k <= card[j]; ++k) {
            acc += std::pow((double)k, -1.2) / tot;
            cdf[j].push_back(acc);
        }
    }
    // class weights W [C][n_num] and embeddings E [C][n_cat][64]
    std::vector<double> W(C * n_num), E(C * n_cat * 64);
    const Rng rw(seed, S_W, 0), re(seed, S_EMB, 0);
    for (uint64_t i = 0; i < W.size(); ++i) W[i] = 0.5 * rw.normal(i);
    for (uint64_t i = 0; i < E.size(); ++i) E[i] = re.normal(i);
#pragma omp parallel for schedule(static)
    for (int64_t f = 0; f < (int64_t)F; ++f) {
        const Rng r(seed, S_X, (stream << 32) ^ (uint64_t)f);
        float* col = x + (uint64_t)f * n;
        if ((uint64_t)f < n_num) {
            for (uint64_t i = 0; i < n; ++i) col[i] = (float)r.normal(i);
        } else {
            const std::vector<double>& cd = cdf[f - n_num];
            for (uint64_t i = 0; i < n; ++i) {
                const double u = r.u01(i);
                uint32_t k = 0;
                while (k + 1 < cd.size() && u >= cd[k]) ++k;
                col[i] = (float)k;  // rank - 1
            }
        }
    }
    const Rng rg(seed, S_NOISE, stream);
#pragma omp parallel for schedule(static)
    for (int64_t i = 0; i < (int64_t)n; ++i) {
        double best = -INFINITY;
        uint64_t arg = 0;
        for (uint64_t c = 0; c < C; ++c) {
            double s = 0.0;
            for (uint64_t j = 0; j < n_num; ++j) s += W[c * n_num + j] * (double)x[j * n + i];
            for (uint64_t j = 0; j < n_cat; ++j) {
                const uint64_t v = (uint64_t)x[(n_num + j) * n + i];
                s += E[(c * n_cat + j) * 64 + v];
            }
            const double u = rg.u01((uint64_t)i * C + c);
            s += -std::log(-std::log(u < 1e-300 ? 1e-300 : u));  // Gumbel
            if (s > best) {
                best = s;
                arg = c;
            }
        }
        y[i] = (float)arg;
    }
    return 0;
}

}  // namespace synthgen
