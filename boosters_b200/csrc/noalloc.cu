// noalloc.cu — split search on a device histogram that allocates no memory.
//
// For callers that cannot allocate device memory per call: a serving or
// embedding process whose device memory is already fully reserved by another
// allocator, or latency-critical code that cannot afford cudaMalloc/cudaFree
// (cudaFree synchronises the whole device and stalls every other stream).
// All working memory of this entry point lives in one file-scope
// `static __device__` array, NOALLOC_SCRATCH_BYTES long, which the CUDA
// runtime places on a GPU when this entry point is first called there and
// keeps until the process exits. The caller passes the inputs (a device
// histogram) and the output (a host bst_split).
//
// The CUDA runtime loads a library's device code and its `__device__` arrays
// onto a GPU lazily, at first use. The first call on each device therefore
// loads them (this file's kernels, the array, and the split-scan kernels it
// launches) before doing any work, so that later calls allocate nothing; a
// caller that reserves all device memory must make one call first.
#include <math.h>

#include <mutex>

#include "../../include/boosters_c.h"
#include "api_util.h"
#include "kernels.h"

namespace bst {
namespace {

// Limits of the scratch array.
constexpr uint32_t NA_MAX_BINS = 65536;  // total histogram bins (1 MiB of int64 pairs)
constexpr uint32_t NA_MAX_COLS = 1024;   // features

struct NoallocScratch {
    HBin hist[NA_MAX_BINS];             // fixed-point copy of the caller's histogram
    ScanColumn cols[NA_MAX_COLS];
    ColCand cand[NA_MAX_COLS];
    uint32_t n_bins[NA_MAX_COLS];
    int32_t is_cat[NA_MAX_COLS];
    int32_t has_missing[NA_MAX_COLS];
    long long node_tot[2];
    NodeSplit out;
    ScanNode node;
    double scale[4];
    unsigned long long maxabs[2];       // bit patterns of max |grad|, max |hess|
    double parent[2];
};

constexpr size_t NOALLOC_SCRATCH_BYTES = (sizeof(NoallocScratch) + 255) / 256 * 256;

static __device__ __align__(256) unsigned char g_noalloc_scratch[NOALLOC_SCRATCH_BYTES];

// Host-side address of g_noalloc_scratch per device (the symbol itself is a
// host stand-in, not a device address).
constexpr int NA_MAX_DEVICES = 64;
NoallocScratch* g_scratch_ptr[NA_MAX_DEVICES] = {nullptr};
std::mutex g_scratch_mu;

cudaError_t load_noalloc_kernels();

// First call on a device (with that device current): resolve the array's
// device address and load every kernel a call launches, so that no later
// call makes the runtime load (and allocate for) device code.
cudaError_t scratch_for_current_device(NoallocScratch** out) {
    int dev = 0;
    cudaError_t e = cudaGetDevice(&dev);
    if (e != cudaSuccess) return e;
    if (dev < 0 || dev >= NA_MAX_DEVICES) return cudaErrorInvalidDevice;
    std::lock_guard<std::mutex> lk(g_scratch_mu);
    if (!g_scratch_ptr[dev]) {
        void* p = nullptr;
        e = cudaGetSymbolAddress(&p, g_noalloc_scratch);
        if (e == cudaSuccess) e = load_noalloc_kernels();
        if (e == cudaSuccess) e = load_split_kernels();
        if (e != cudaSuccess) return e;
        g_scratch_ptr[dev] = reinterpret_cast<NoallocScratch*>(p);
    }
    *out = g_scratch_ptr[dev];
    return cudaSuccess;
}

// max |grad|, |hess| of the caller's histogram (NaN ignored); the accumulators
// start at zero (set by k_na_clear).
__global__ void k_na_clear(NoallocScratch* s) {
    if (threadIdx.x == 0) {
        s->maxabs[0] = 0ull;
        s->maxabs[1] = 0ull;
    }
}

__global__ void k_na_maxabs(const double* __restrict__ hist, uint32_t total, NoallocScratch* s) {
    unsigned long long mg = 0ull, mh = 0ull;
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        const double g = fabs(hist[2 * i]), h = fabs(hist[2 * i + 1]);
        if (g == g) mg = max(mg, (unsigned long long)__double_as_longlong(g));
        if (h == h) mh = max(mh, (unsigned long long)__double_as_longlong(h));
    }
    for (int o = 16; o > 0; o >>= 1) {
        mg = max(mg, __shfl_xor_sync(0xFFFFFFFFu, mg, o));
        mh = max(mh, __shfl_xor_sync(0xFFFFFFFFu, mh, o));
    }
    if ((threadIdx.x & 31) == 0) {
        atomicMax(&s->maxabs[0], mg);
        atomicMax(&s->maxabs[1], mh);
    }
}

__device__ double na_fixed_scale(double bound) {  // as fixed_scale() of bst_find_split
    if (!(bound > 0.0)) return 1.0;
    int e;
    frexp(bound, &e);
    int k = 62 - e;
    k = k < -1000 ? -1000 : (k > 1000 ? 1000 : k);
    return ldexp(1.0, k);
}

// One block: scales, parent totals, column table (prefix sum of n_bins).
__global__ void k_na_setup(uint32_t F, uint32_t total, uint32_t count, NoallocScratch* s) {
    __shared__ uint32_t off[NA_MAX_COLS];
    if (threadIdx.x == 0) {
        const double mg = __longlong_as_double((long long)s->maxabs[0]);
        const double mh = __longlong_as_double((long long)s->maxabs[1]);
        const double sg = na_fixed_scale((double)total * mg + fabs(s->parent[0]));
        const double sh = na_fixed_scale((double)total * mh + fabs(s->parent[1]));
        s->scale[0] = sg;
        s->scale[1] = sh;
        s->scale[2] = 1.0 / sg;
        s->scale[3] = 1.0 / sh;
        ScanNode nd;
        nd.slot = 0;
        nd.count = count;
        nd.flags = 1u;
        nd.pad = 0u;
        nd.pg = __double2ll_rn(s->parent[0] * sg);
        nd.ph = __double2ll_rn(s->parent[1] * sh);
        s->node = nd;
        uint32_t acc = 0;
        for (uint32_t f = 0; f < F; ++f) {
            off[f] = acc;
            acc += s->n_bins[f];
        }
    }
    __syncthreads();
    for (uint32_t f = threadIdx.x; f < F; f += blockDim.x)
        s->cols[f] = ScanColumn{s->n_bins[f], off[f], s->is_cat[f] ? 1u : 0u, s->has_missing[f] ? 1u : 0u};
}

__global__ void k_na_quantize(const double* __restrict__ hist, uint32_t total, NoallocScratch* s) {
    const double sg = s->scale[0], sh = s->scale[1];
    for (uint32_t i = blockIdx.x * blockDim.x + threadIdx.x; i < total; i += gridDim.x * blockDim.x) {
        HBin b;
        b.g = __double2ll_rn(hist[2 * i] * sg);
        b.h = __double2ll_rn(hist[2 * i + 1] * sh);
        s->hist[i] = b;
    }
}

cudaError_t load_noalloc_kernels() {
    cudaFuncAttributes a;
    cudaError_t e = cudaFuncGetAttributes(&a, k_na_clear);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, k_na_maxabs);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, k_na_setup);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, k_na_quantize);
    return e;
}

bst_status cuda_fail(cudaError_t e) {
    cudaGetLastError();
    return api_fail(BST_ERR_CUDA, cudaGetErrorString(e));
}

}  // namespace
}  // namespace bst

extern "C" bst_status bst_find_split_noalloc(const double* hist_dev, const uint32_t* n_bins,
                                             const int32_t* is_categorical, const int32_t* has_missing,
                                             uint32_t n_features, double parent_grad, double parent_hess,
                                             uint32_t parent_count, const bst_config* cfg, uint32_t n_threads,
                                             void* stream, bst_split* out) {
    using namespace bst;
    api_clear_error();
    if (!hist_dev || !n_bins || !is_categorical || !has_missing || !cfg || !out)
        return api_fail(BST_ERR_INVALID_ARGUMENT, "NULL argument");
    const bst_status rc = api_check_config(cfg, false);
    if (rc != BST_OK) return rc;
    *out = bst_split{};
    out->gain = -INFINITY;
    if (n_features == 0) return BST_OK;  // no candidate, as bst_find_split
    if (n_features > NA_MAX_COLS)
        return api_fail(BST_ERR_INVALID_ARGUMENT, "n_features exceeds the fixed working array's limit of 1024");
    uint64_t total = 0;
    for (uint32_t f = 0; f < n_features; ++f) {
        if (is_categorical[f] && n_bins[f] > 256)
            return api_fail(BST_ERR_UNSUPPORTED, "categorical features need <= 256 bins");
        total += n_bins[f];
    }
    if (total > NA_MAX_BINS)
        return api_fail(BST_ERR_INVALID_ARGUMENT, "sum(n_bins) exceeds the fixed working array's limit of 65536");
    if (total == 0) return BST_OK;
    cudaStream_t st = (cudaStream_t)stream;
    NoallocScratch* s = nullptr;
    const cudaError_t se = scratch_for_current_device(&s);
    if (se != cudaSuccess) return cuda_fail(se);
    const double parent[2] = {parent_grad, parent_hess};
    cudaError_t e = cudaSuccess;
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->n_bins, n_bins, sizeof(uint32_t) * n_features, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->is_cat, is_categorical, sizeof(int32_t) * n_features, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess)
        e = cudaMemcpyAsync(s->has_missing, has_missing, sizeof(int32_t) * n_features, cudaMemcpyHostToDevice, st);
    if (e == cudaSuccess) e = cudaMemcpyAsync(s->parent, parent, sizeof(parent), cudaMemcpyHostToDevice, st);
    if (e != cudaSuccess) return cuda_fail(e);
    const uint32_t tb = (uint32_t)total;
    const unsigned blocks = (tb + 255) / 256 < 1024 ? (tb + 255) / 256 : 1024;
    k_na_clear<<<1, 32, 0, st>>>(s);
    k_na_maxabs<<<blocks, 256, 0, st>>>(hist_dev, tb, s);
    k_na_setup<<<1, 256, 0, st>>>(n_features, tb, parent_count, s);
    k_na_quantize<<<blocks, 256, 0, st>>>(hist_dev, tb, s);
    GainParamsDev gp;
    gp.lambda = (double)cfg->lambda;
    gp.min_gain = (double)cfg->min_gain;
    gp.min_child_weight = (double)cfg->min_child_weight;
    gp.min_samples_leaf = cfg->min_samples_leaf;
    gp.max_onehot_cats = cfg->max_onehot_cats;
    launch_split_scan(&s->node, 1, s->cols, n_features, s->hist, tb, s->scale, gp, s->cand, s->node_tot, st);
    launch_split_reduce(s->cand, s->node_tot, 1, n_features, (n_threads != 1 && n_features >= 16) ? 1 : 0, &s->out, st);
    NodeSplit res;
    e = cudaMemcpyAsync(&res, &s->out, sizeof(res), cudaMemcpyDeviceToHost, st);
    if (e == cudaSuccess) e = cudaStreamSynchronize(st);
    if (e == cudaSuccess) e = cudaGetLastError();
    if (e != cudaSuccess) return cuda_fail(e);
    if (res.flags & 4u) {
        out->feature = res.col;
        out->gain = res.gain;
        out->default_left = (res.flags & 1u) ? 1 : 0;
        out->is_categorical = (res.flags & 2u) ? 1 : 0;
        out->bin = (res.flags & 2u) ? 0u : res.bin;
        for (int q = 0; q < 4; ++q) out->left_cats[q] = res.cats[q];
    }
    return BST_OK;
}
