// mappers.cu — numeric bin bounds on the device (dataset.rs:683-750).
//
// One block per numeric feature: the feature's sampled values (rows of the
// feature-major input picked by the ascending row sample, or every row) are
// filtered to the finite ones, sorted by a block-wide stable LSD radix sort
// of order-preserving 32-bit keys, reduced to their distinct values (+0.0 and
// -0.0 compare equal and are one value, as in the reference's dedup), and the
// bounds are the midpoints, in f64, between consecutive distinct values, or
// between the distinct values at the quantile positions
// floor(i / nb * (u - 1)) when there are more than nb of them, each kept only
// when it exceeds the previous bound. f64 arithmetic is the same IEEE
// sequence as the reference's (this file is compiled without contraction).
#include <float.h>
#include <math.h>

#include "kernels.h"

namespace bst {

namespace {

constexpr unsigned FULL = 0xFFFFFFFFu;
constexpr int MAP_THREADS = 1024;
constexpr int MAP_WARPS = MAP_THREADS / 32;
constexpr int MAP_ITEMS = 8;                                  // keys per thread and tile
constexpr uint32_t MAP_WARP_KEYS = 32u * MAP_ITEMS;           // keys per warp and tile
constexpr uint32_t MAP_TILE = MAP_THREADS * MAP_ITEMS;        // keys per tile
constexpr int MAP_QUARTERS = 4;                               // cross-warp scan: 4 x 8 warps
constexpr int MAP_QWARPS = MAP_WARPS / MAP_QUARTERS;

// Sign bit flipped for non-negative floats, all bits for negative ones:
// unsigned order of the keys is the numeric order of the floats (-0.0 just
// below +0.0).
__device__ __forceinline__ uint32_t float_key(float v) {
    const uint32_t u = __float_as_uint(v);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float key_float(uint32_t k) {
    const uint32_t u = (k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k;
    return __uint_as_float(u);
}

// Exclusive prefix sum of v over the block (blockDim.x = MAP_THREADS);
// *total = the block's sum. sh: MAP_WARPS + 1 words.
__device__ uint32_t map_block_scan(uint32_t v, uint32_t* sh, uint32_t* total) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    uint32_t x = v;
#pragma unroll
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t t = __shfl_up_sync(FULL, x, d);
        if (lane >= (uint32_t)d) x += t;
    }
    if (lane == 31) sh[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t y = sh[lane];
#pragma unroll
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t t = __shfl_up_sync(FULL, y, d);
            if (lane >= (uint32_t)d) y += t;
        }
        sh[lane] = y;
    }
    __syncthreads();
    const uint32_t r = (warp ? sh[warp - 1] : 0u) + x - v;
    *total = sh[MAP_WARPS - 1];
    __syncthreads();
    return r;
}

struct MapShared {
    uint32_t wcnt[MAP_WARPS][256];       // per-warp digit counts, then the warps' exclusive prefixes
    uint32_t qpre[MAP_QUARTERS][256];    // quarter sums, then the quarters' exclusive prefixes
    uint32_t base[256];                  // digit offsets of the next tile
    uint32_t cnt[256];                   // digit counts of the tile
    uint32_t dcnt[4][256];               // the keys' counts of each digit value, per digit position
    uint32_t scan[MAP_WARPS + 1];
    uint32_t w;                          // finite keys
};

// One stable pass of the LSD radix sort: the w keys of `in` by their digit
// at `shift` into `out`. Within a tile, key order is (warp, round, lane),
// which is index order; a key's place is the digit's offset + the keys of
// that digit in earlier tiles, earlier warps, earlier rounds and lower lanes.
__device__ void radix_pass(const uint32_t* __restrict__ in, uint32_t* __restrict__ out, uint32_t w, uint32_t shift,
                           MapShared& s) {
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    const uint32_t lt = (1u << lane) - 1u;
    for (uint32_t t0 = 0; t0 < w; t0 += MAP_TILE) {
        for (uint32_t d = lane; d < 256u; d += 32u) s.wcnt[warp][d] = 0;
        __syncwarp();
        uint32_t key[MAP_ITEMS], dig[MAP_ITEMS], rank[MAP_ITEMS];
        const uint32_t wb = t0 + warp * MAP_WARP_KEYS;
#pragma unroll
        for (int r = 0; r < MAP_ITEMS; ++r) {
            const uint32_t i = wb + (uint32_t)r * 32u + lane;
            const bool valid = i < w;
            key[r] = valid ? in[i] : 0u;
            dig[r] = valid ? ((key[r] >> shift) & 255u) : 256u;  // 256: no digit
            const uint32_t peers = __match_any_sync(FULL, dig[r]);
            rank[r] = valid ? s.wcnt[warp][dig[r]] + (uint32_t)__popc(peers & lt) : 0u;
            __syncwarp();
            if (valid && lane == (uint32_t)(__ffs(peers) - 1)) s.wcnt[warp][dig[r]] += (uint32_t)__popc(peers);
            __syncwarp();
        }
        __syncthreads();
        {  // exclusive prefixes over the warps of each quarter; quarter sums
            const uint32_t d = threadIdx.x & 255u, q = threadIdx.x >> 8;
            uint32_t run = 0;
            for (int k = 0; k < MAP_QWARPS; ++k) {
                const uint32_t wq = q * MAP_QWARPS + (uint32_t)k;
                const uint32_t c = s.wcnt[wq][d];
                s.wcnt[wq][d] = run;
                run += c;
            }
            s.qpre[q][d] = run;
        }
        __syncthreads();
        if (threadIdx.x < 256u) {  // quarters' exclusive prefixes; the tile's digit totals advance base
            const uint32_t d = threadIdx.x;
            uint32_t run = 0;
            for (int q = 0; q < MAP_QUARTERS; ++q) {
                const uint32_t c = s.qpre[q][d];
                s.qpre[q][d] = run;
                run += c;
            }
            s.cnt[d] = run;  // reused: this tile's count of digit d
        }
        __syncthreads();
#pragma unroll
        for (int r = 0; r < MAP_ITEMS; ++r)
            if (dig[r] < 256u)
                out[s.base[dig[r]] + s.qpre[warp / MAP_QWARPS][dig[r]] + s.wcnt[warp][dig[r]] + rank[r]] = key[r];
        __syncthreads();
        if (threadIdx.x < 256u) s.base[threadIdx.x] += s.cnt[threadIdx.x];
        __syncthreads();
    }
}

__global__ void __launch_bounds__(MAP_THREADS, 1)
k_numeric_bounds(const float* __restrict__ x, uint64_t col_stride, const uint32_t* __restrict__ rows, uint32_t k,
                 const MapJob* __restrict__ jobs, uint32_t max_bins, uint32_t* __restrict__ scratch,
                 double* __restrict__ cand, double* __restrict__ bounds, uint32_t* __restrict__ n_bounds) {
    __shared__ MapShared s;
    const uint32_t j = blockIdx.x;
    const MapJob job = jobs[j];
    const float* col = x + (uint64_t)job.col * col_stride;
    uint32_t* A = scratch + (size_t)j * 2u * k;
    uint32_t* B = A + k;
    double* bj = bounds + (size_t)j * (max_bins + 2u);
    double* cj = cand + (size_t)j * max_bins;
    const uint32_t lane = threadIdx.x & 31u;
    if (threadIdx.x == 0) s.w = 0;
    for (uint32_t i = threadIdx.x; i < 4u * 256u; i += MAP_THREADS) (&s.dcnt[0][0])[i] = 0;
    __syncthreads();
    // finite sampled values as keys, in any order (the sort fixes it)
    for (uint32_t i0 = 0; i0 < k; i0 += MAP_THREADS) {
        const uint32_t i = i0 + threadIdx.x;
        float v = 0.0f;
        bool fin = false;
        if (i < k) {
            v = col[rows ? (uint64_t)rows[i] : (uint64_t)i];
            fin = isfinite(v);
        }
        const uint32_t m = __ballot_sync(FULL, fin);
        uint32_t wbase = 0;
        if (lane == 0 && m) wbase = atomicAdd(&s.w, (uint32_t)__popc(m));
        wbase = __shfl_sync(FULL, wbase, 0);
        const uint32_t key = float_key(v);
        if (fin) A[wbase + (uint32_t)__popc(m & ((1u << lane) - 1u))] = key;
        // the four digits' counts (the same for every pass: they depend
        // only on the keys), one shared atomic per distinct digit and warp
#pragma unroll
        for (int dp = 0; dp < 4; ++dp) {
            const uint32_t dg = fin ? ((key >> (8 * dp)) & 255u) : 256u;
            const uint32_t peers = __match_any_sync(FULL, dg);
            if (fin && lane == (uint32_t)(__ffs(peers) - 1)) atomicAdd(&s.dcnt[dp][dg], (uint32_t)__popc(peers));
        }
    }
    __syncthreads();
    const uint32_t w = s.w;
    if (w == 0) {
        if (threadIdx.x == 0) {
            bj[0] = DBL_MAX;
            n_bounds[j] = 1;
        }
        return;
    }
    // stable LSD radix sort, 8-bit digits; a pass whose digit is the same
    // for every key is skipped
    const uint32_t key0 = A[0];  // any one key: the digit counts do not depend on order
    uint32_t* in = A;
    uint32_t* out = B;
    for (uint32_t shift = 0; shift < 32u; shift += 8u) {
        const uint32_t* dc = s.dcnt[shift / 8u];
        if (dc[(key0 >> shift) & 255u] == w) continue;
        if (threadIdx.x < 32u) {  // exclusive scan of the 256 counts: 8 per lane
            uint32_t c[8], sum = 0;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                c[q] = dc[lane * 8u + (uint32_t)q];
                sum += c[q];
            }
            uint32_t x = sum;
#pragma unroll
            for (int d = 1; d < 32; d <<= 1) {
                const uint32_t t = __shfl_up_sync(FULL, x, d);
                if (lane >= (uint32_t)d) x += t;
            }
            uint32_t run = x - sum;
#pragma unroll
            for (int q = 0; q < 8; ++q) {
                s.base[lane * 8u + (uint32_t)q] = run;
                run += c[q];
            }
        }
        __syncthreads();
        radix_pass(in, out, w, shift, s);
        uint32_t* t = in;
        in = out;
        out = t;
    }
    // distinct values (float equality), in order, into `out`
    uint32_t u = 0;
    for (uint32_t i0 = 0; i0 < w; i0 += MAP_THREADS) {
        const uint32_t i = i0 + threadIdx.x;
        uint32_t key = 0;
        bool first = false;
        if (i < w) {
            key = in[i];
            first = i == 0 || key_float(key) != key_float(in[i - 1]);
        }
        uint32_t tot;
        const uint32_t pos = map_block_scan(first ? 1u : 0u, s.scan, &tot);
        if (first) out[u + pos] = key;
        u += tot;
    }
    __syncthreads();
    if (u <= 1u) {  // one finite value (lo >= hi): a single bin, no NaN bin
        if (threadIdx.x == 0) {
            bj[0] = DBL_MAX;
            n_bounds[j] = 1;
        }
        return;
    }
    const uint32_t nb = w < max_bins ? w : max_bins;
    const uint32_t extra = job.has_nan ? 2u : 1u;  // the last bound (+ the NaN bin's)
    if (u <= nb) {
        for (uint32_t i = threadIdx.x; i + 1u < u; i += MAP_THREADS)
            bj[i] = ((double)key_float(out[i]) + (double)key_float(out[i + 1])) / 2.0;
        if (threadIdx.x == 0) {
            bj[u - 1] = DBL_MAX;
            if (job.has_nan) bj[u] = DBL_MAX;
            n_bounds[j] = u - 1 + extra;
        }
        return;
    }
    // quantile midpoints i = 1 .. nb - 1 (non-decreasing in i), kept when
    // above the previous one
    for (uint32_t i = 1u + threadIdx.x; i < nb; i += MAP_THREADS) {
        const double q = (double)i / (double)nb;
        uint64_t idx = (uint64_t)floor(q * (double)(u - 1u));
        if (idx > (uint64_t)(u - 2u)) idx = u - 2u;
        cj[i] = ((double)key_float(out[idx]) + (double)key_float(out[idx + 1])) / 2.0;
    }
    __syncthreads();
    uint32_t kept = 0;
    for (uint32_t i0 = 1; i0 < nb; i0 += MAP_THREADS) {
        const uint32_t i = i0 + threadIdx.x;
        const bool keep = i < nb && (i == 1u || cj[i] > cj[i - 1]);
        uint32_t tot;
        const uint32_t pos = map_block_scan(keep ? 1u : 0u, s.scan, &tot);
        if (keep) bj[kept + pos] = cj[i];
        kept += tot;
    }
    if (threadIdx.x == 0) {
        bj[kept] = DBL_MAX;
        if (job.has_nan) bj[kept + 1] = DBL_MAX;
        n_bounds[j] = kept + extra;
    }
}

}  // namespace

void launch_numeric_bounds(const float* x, uint64_t col_stride, const uint32_t* rows, uint32_t k, const MapJob* jobs,
                           uint32_t n_jobs, uint32_t max_bins, uint32_t* scratch, double* cand, double* bounds,
                           uint32_t* n_bounds, cudaStream_t st) {
    if (n_jobs == 0 || k == 0) return;
    k_numeric_bounds<<<n_jobs, MAP_THREADS, 0, st>>>(x, col_stride, rows, k, jobs, max_bins, scratch, cand, bounds,
                                                     n_bounds);
}

}  // namespace bst
