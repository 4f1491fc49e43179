// kernels.cu — sm_100a kernels of the B200 GBDT engine.
//
// Every kernel here is HBM- or latency-bound integer/byte work with a little
// f32/f64 arithmetic; none is a dense contraction, so none uses tensor cores.
// Floating-point expressions are written in the reference's evaluation order
// and the file is compiled with -fmad=false so that no a*b+c is fused: f32
// and f64 results round exactly as the Rust CPU path does.
#include <math.h>

#include <atomic>


#include <type_traits>
#include <utility>

#include "kernels.h"

#include <cuda.h>  // CUtensorMap and the tensor-map encoder's types (the encoder itself is fetched at run time)

namespace bst {

uint32_t sm_count() {
    thread_local int dev_cached = -1;
    thread_local uint32_t sms = 1;
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) {
        cudaGetLastError();
        return sms;
    }
    if (dev != dev_cached) {
        int v = 0;
        if (cudaDeviceGetAttribute(&v, cudaDevAttrMultiProcessorCount, dev) != cudaSuccess) cudaGetLastError();
        sms = v > 0 ? (uint32_t)v : 1u;
        dev_cached = dev;
    }
    return sms;
}

// Checked build: g_check holds (violations, site, index, bound) of the first
// failed bounds test on this device. BST_IN(i, n, site) is true when i < n;
// otherwise it records the failure and is false, and the caller skips the
// access. In the normal build BST_IN is the constant true and every guarded
// access compiles exactly as unguarded code.
#ifdef BST_CHECKED
__device__ unsigned long long g_check[4];

__device__ __noinline__ bool check_fail(uint32_t site, unsigned long long i, unsigned long long n) {
    if (atomicAdd(&g_check[0], 1ull) == 0ull) {
        g_check[1] = site;
        g_check[2] = i;
        g_check[3] = n;
    }
    return false;
}
#define BST_IN(i, n, site) \
    ((unsigned long long)(i) < (unsigned long long)(n) || check_fail((site), (unsigned long long)(i), (unsigned long long)(n)))

bool check_take(int device, CheckRecord* out) {
    int prev = 0;
    if (cudaGetDevice(&prev) != cudaSuccess || cudaSetDevice(device) != cudaSuccess) {
        cudaGetLastError();
        return false;
    }
    unsigned long long h[4] = {0, 0, 0, 0};
    const unsigned long long z[4] = {0, 0, 0, 0};
    bool ok = cudaDeviceSynchronize() == cudaSuccess && cudaMemcpyFromSymbol(h, g_check, sizeof(h)) == cudaSuccess &&
              cudaMemcpyToSymbol(g_check, z, sizeof(z)) == cudaSuccess;
    if (!ok) cudaGetLastError();
    cudaSetDevice(prev);
    if (ok && out) *out = CheckRecord{h[0], h[1], h[2], h[3]};
    return ok;
}
#else
#define BST_IN(i, n, site) true

bool check_take(int, CheckRecord*) { return false; }
#endif

namespace {

constexpr unsigned FULL = 0xFFFFFFFFu;

// Programmatic dependent launch. Every kernel is launched with programmatic
// stream serialisation and begins with BST_PDL_ENTER: griddepcontrol.wait
// holds the kernel's threads until the kernel before it in the stream has
// completed and its memory writes are visible (for a kernel launched without
// the attribute it returns at once), so kernel bodies still run strictly in
// stream order. No kernel triggers its dependents early (the trigger is
// implicit at block exit): the next kernel's launch overlaps only this
// kernel's completion, and its blocks are placed on SMs as a whole grid
// (the one-wave grids count on one block per SM slot).
#define BST_PDL_ENTER() asm volatile("griddepcontrol.wait;" ::: "memory")

template <typename... P, typename... A>
inline void launch_k(void (*k)(P...), dim3 grid, dim3 block, size_t smem, cudaStream_t st, A&&... args) {
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t c = {};
    c.gridDim = grid;
    c.blockDim = block;
    c.dynamicSmemBytes = smem;
    c.stream = st;
    c.attrs = at;
    c.numAttrs = 1;
    cudaLaunchKernelEx(&c, k, std::forward<A>(args)...);  // errors: the caller's next check
}

// The same for a kernel chosen at run time (argument pointers as for
// cudaLaunchKernel).
inline void launch_kv(const void* k, dim3 grid, dim3 block, void** args, size_t smem, cudaStream_t st) {
    cudaLaunchAttribute at[1];
    at[0].id = cudaLaunchAttributeProgrammaticStreamSerialization;
    at[0].val.programmaticStreamSerializationAllowed = 1;
    cudaLaunchConfig_t c = {};
    c.gridDim = grid;
    c.blockDim = block;
    c.dynamicSmemBytes = smem;
    c.stream = st;
    c.attrs = at;
    c.numAttrs = 1;
    cudaLaunchKernelExC(&c, k, args);
}


__device__ __forceinline__ int32_t sat_i32(double v) {
    if (v != v) return 0;
    if (v >= 2147483647.0) return 2147483647;
    if (v <= -2147483648.0) return (int32_t)(-2147483647 - 1);
    return (int32_t)v;
}

__device__ __forceinline__ uint32_t sat_u32(float v) {
    if (!(v > 0.0f)) return 0u;
    if (v >= 4294967295.0f) return 0xFFFFFFFFu;
    return (uint32_t)v;
}

// f32 exp of an f32 argument. Computed in f64 and rounded once, so the result
// is the correctly rounded expf in all but a vanishing fraction of inputs
// (the CPU reference calls the platform libm expf).
__device__ __forceinline__ float exp_f32(float x) { return (float)exp((double)x); }

__device__ __forceinline__ long long quantize(float v, double scale) {
    return __double2ll_rn((double)v * scale);
}

__device__ __forceinline__ long long shfl_up_ll(long long v, int d) {
    return __shfl_up_sync(FULL, v, d);
}

}  // namespace

// ============================================================================
// K1: bin assignment (BinMapper::value_to_bin, data/binned/bin_mapper.rs:210)
// Reads the feature-major f32 matrix coalesced, writes row-major bins.
// ============================================================================

__global__ void __launch_bounds__(256)
k_bin_assign(const float* __restrict__ x, uint64_t n, const BinColumn* __restrict__ cols,
             uint32_t n_cols, const float* __restrict__ thr, const int32_t* __restrict__ cats,
             uint8_t* __restrict__ rec_out, uint32_t rec, uint32_t u16_off, uint32_t tab_cap) {
    BST_PDL_ENTER();
    // one thread per row of a tile of blockDim.x rows; the tile's records are
    // assembled in shared memory, then copied out as one contiguous run. Each
    // column's search table (thresholds or categories) is staged in shared
    // memory first, two buffers alternating, so the lanes' divergent binary
    // searches read shared memory instead of serialising in L1.
    // records are rec + 4 bytes apart in shared memory, so the lanes'
    // writes of one column (one row each) fall in different banks
    extern __shared__ __align__(16) unsigned char smem[];
    const uint32_t rows = blockDim.x;
    const uint32_t rs = rec + 4u;
    uint32_t* tabs = reinterpret_cast<uint32_t*>(smem + (size_t)rows * rs);  // 2 x tab_cap words
    const uint64_t r0 = (uint64_t)blockIdx.x * rows;
    const uint64_t rem = n - r0;
    const uint32_t valid = rem < (uint64_t)rows ? (uint32_t)rem : rows;
    const uint32_t tile_words = rows * rs / 4u;
    for (uint32_t i = threadIdx.x; i < tile_words; i += rows) reinterpret_cast<uint32_t*>(smem)[i] = 0u;
    const uint32_t t = threadIdx.x;
    const uint64_t row = r0 + t;
    unsigned char* my = smem + (size_t)t * rs;
    for (uint32_t c = 0; c < n_cols; ++c) {
        const BinColumn col = cols[c];
        const float v = t < valid ? x[(uint64_t)col.src * n + row] : 0.0f;
        uint32_t* tb = tabs + (c & 1u) * tab_cap;
        const uint32_t cnt = col.is_cat ? col.n_cats : col.n_search;
        const uint32_t* src = col.is_cat ? reinterpret_cast<const uint32_t*>(cats + col.off)
                                         : reinterpret_cast<const uint32_t*>(thr + col.off);
        for (uint32_t i = t; i < cnt; i += rows) tb[i] = src[i];
        // the table of column c - 1 (the other buffer) is no longer read
        // once every thread passes this barrier; c + 1 overwrites it
        __syncthreads();
        if (t < valid) {
            uint32_t bin;
            if (v != v) {
                bin = col.nan_bin;
            } else if (v == 0.0f && col.zero_bin != 0xFFFFFFFFu) {
                bin = col.zero_bin;
            } else if (col.is_cat) {
                const int32_t key = sat_i32((double)v);
                uint32_t lo = 0, hi = col.n_cats;
                while (lo < hi) {
                    uint32_t mid = (lo + hi) >> 1;
                    if ((int32_t)tb[mid] < key)
                        lo = mid + 1;
                    else
                        hi = mid;
                }
                bin = (lo < col.n_cats && (int32_t)tb[lo] == key) ? lo : 0u;
            } else {
                uint32_t lo = 0, hi = col.n_search;
                while (lo < hi) {
                    uint32_t mid = lo + ((hi - lo) >> 1);
                    if (v <= __uint_as_float(tb[mid]))
                        hi = mid;
                    else
                        lo = mid + 1;
                }
                bin = lo;
            }
            if (col.matrix == 0)
                my[col.pos] = (uint8_t)bin;
            else
                reinterpret_cast<uint16_t*>(my + u16_off)[col.pos] = (uint16_t)bin;
        }
    }
    __syncthreads();
    const uint32_t wpr = rec / 4u, nw = valid * wpr;  // rec is a multiple of 32
    uint32_t* dst = reinterpret_cast<uint32_t*>(rec_out + r0 * rec);
    const uint32_t* srcw = reinterpret_cast<const uint32_t*>(smem);
    for (uint32_t i = threadIdx.x; i < nw; i += rows) dst[i] = srcw[(i / wpr) * (rs / 4u) + i % wpr];
}

// Search-table words per buffer (a multiple of 4, so the tables stay 16-byte
// aligned) and rows per block: 256 down to 32 while the record tile and the
// two tables fit 160 KB.
static uint32_t bin_assign_tab_cap(uint32_t max_tab) { return ((max_tab ? max_tab : 1u) + 3u) & ~3u; }

int bin_assign_rows(uint32_t rec, uint32_t max_tab) {
    const size_t tabs = 8u * (size_t)bin_assign_tab_cap(max_tab);
    for (int rows = 256; rows >= 32; rows -= 32)
        if ((size_t)rows * (rec + 4u) + tabs <= 160 * 1024) return rows;
    return 0;
}

void launch_bin_assign(const float* x_fm, uint64_t n, const BinColumn* cols, uint32_t n_cols,
                       const float* thr, const int32_t* cats, uint8_t* rec_out, uint32_t rec, uint32_t u16_off,
                       uint32_t max_tab, cudaStream_t st) {
    if (n == 0 || n_cols == 0 || rec == 0) return;
    const int rows = bin_assign_rows(rec, max_tab);
    if (rows == 0) return;
    const uint32_t cap = bin_assign_tab_cap(max_tab);
    const uint64_t blocks = (n + rows - 1) / rows;
    const size_t smem = (size_t)rows * (rec + 4u) + 8u * (size_t)cap;
    if (smem > 48 * 1024)
        cudaFuncSetAttribute(k_bin_assign, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
    launch_k(k_bin_assign, (unsigned)blocks, rows, smem, st, x_fm, n, cols, n_cols, thr, cats, rec_out, rec, u16_off,
             cap);
}

// ============================================================================
// K3: gradients (training/objectives/regression.rs:20, classification.rs:24,141)
// ============================================================================

// |v| as an order-preserving bit pattern for the scale maxima; NaN and
// infinities do not set the scale.
__device__ __forceinline__ unsigned abs_bits(float v) {
    const float a = fabsf(v);
    return a <= 3.4e38f ? __float_as_uint(a) : 0u;
}

__device__ __forceinline__ unsigned warp_max_u32(unsigned b) {
    for (int o = 16; o > 0; o >>= 1) b = max(b, __shfl_xor_sync(FULL, b, o));
    return b;
}

// Per-output max |grad| and |hess| go to a per-block shared array (one
// shared atomic per warp), then one global atomic per block and value: a
// global atomic per warp on the same two words serialises in L2.
__global__ void k_gradients(int objective, uint32_t G, const float* __restrict__ pred,
                            const float* __restrict__ y, const float* __restrict__ w, uint64_t n,
                            float2* __restrict__ gh, unsigned* __restrict__ maxabs,
                            const float* __restrict__ alpha, float delta) {
    BST_PDL_ENTER();
    extern __shared__ unsigned smax[];  // [2G]
    const float HESS_MIN = 1e-6f;
    for (uint32_t i = threadIdx.x; i < 2 * G; i += blockDim.x) smax[i] = 0u;
    __syncthreads();
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    unsigned m0 = 0u, m1 = 0u;  // squared / logistic: this thread's maxima
    // loop trip count is warp-uniform so that the shuffles below are safe
    const uint64_t n_round = (n + 31) & ~uint64_t(31);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n_round; i += stride) {
        const bool ok = i < n;
        const float wi = (ok && w) ? w[i] : 1.0f;
        const float yi = ok ? y[i] : 0.0f;
        if (objective == 0) {  // squared
            const float p = ok ? pred[i] : 0.0f;
            const float g = wi * (p - yi);
            if (ok) {
                gh[i] = make_float2(g, wi);
                m0 = max(m0, abs_bits(g));
                m1 = max(m1, abs_bits(wi));
            }
        } else if (objective == 1) {  // logistic
            const float x = ok ? pred[i] : 0.0f;
            const float p = 1.0f / (1.0f + exp_f32(-x));
            const float g = wi * (p - yi);
            const float h = fmaxf(wi * p * (1.0f - p), HESS_MIN);
            if (ok) {
                gh[i] = make_float2(g, h);
                m0 = max(m0, abs_bits(g));
                m1 = max(m1, abs_bits(h));
            }
        } else if (objective >= 3) {
            // absolute (regression.rs:80-104), pinball (:129-155, one output
            // per alpha), pseudo-Huber (:183-215), Poisson (:243-271), hinge
            // (classification.rs:88-117); targets are output 0's
            const float inv_delta_sq = 1.0f / (delta * delta);
            for (uint32_t o = 0; o < G; ++o) {
                const float p = ok ? pred[(uint64_t)o * n + i] : 0.0f;
                float g, h;
                if (objective == 3) {
                    const float d = p - yi;
                    g = wi * (isnan(d) ? d : copysignf(1.0f, d));  // f32::signum
                    h = wi;
                } else if (objective == 4) {
                    const float a = alpha[o];
                    g = wi * ((p - yi) < 0.0f ? -a : 1.0f - a);
                    h = wi;
                } else if (objective == 5) {
                    const float r = p - yi, r_sq = r * r;
                    const float factor = 1.0f + r_sq * inv_delta_sq, sq = sqrtf(factor);
                    g = wi * r / sq;
                    h = wi / (factor * sq);
                } else if (objective == 6) {
                    const float pc = p < -30.0f ? -30.0f : (p > 30.0f ? 30.0f : p);
                    const float e = exp_f32(pc);
                    g = wi * (e - yi);
                    h = fmaxf(wi * e, HESS_MIN);
                } else {  // labels {0, 1} as {-1, +1}
                    const float yy = yi > 0.5f ? 1.0f : -1.0f, margin = yy * p;
                    g = margin < 1.0f ? -wi * yy : 0.0f;
                    h = wi;
                }
                if (ok) gh[(uint64_t)o * n + i] = make_float2(g, h);
                const unsigned bg = warp_max_u32(ok ? abs_bits(g) : 0u), bh = warp_max_u32(ok ? abs_bits(h) : 0u);
                if ((threadIdx.x & 31) == 0) {
                    if (bg) atomicMax(&smax[2 * o], bg);
                    if (bh) atomicMax(&smax[2 * o + 1], bh);
                }
            }
        } else {  // softmax
            uint64_t label = 0;
            if (ok && yi > 0.0f) label = (uint64_t)yi;  // `f32 as usize`
            float mx = -INFINITY;
            for (uint32_t c = 0; c < G; ++c) mx = fmaxf(mx, ok ? pred[(uint64_t)c * n + i] : 0.0f);
            float sum = -0.0f;
            for (uint32_t c = 0; c < G; ++c) sum = sum + exp_f32((ok ? pred[(uint64_t)c * n + i] : 0.0f) - mx);
            for (uint32_t c = 0; c < G; ++c) {
                const float pc = ok ? pred[(uint64_t)c * n + i] : 0.0f;
                const float p = exp_f32(pc - mx) / sum;
                const float ind = (c == label) ? 1.0f : 0.0f;
                const float g = wi * (p - ind);
                const float h = fmaxf(wi * p * (1.0f - p), HESS_MIN);
                if (ok) gh[(uint64_t)c * n + i] = make_float2(g, h);
                const unsigned bg = warp_max_u32(ok ? abs_bits(g) : 0u), bh = warp_max_u32(ok ? abs_bits(h) : 0u);
                if ((threadIdx.x & 31) == 0) {
                    if (bg) atomicMax(&smax[2 * c], bg);
                    if (bh) atomicMax(&smax[2 * c + 1], bh);
                }
            }
        }
    }
    if (objective == 0 || objective == 1) {
        m0 = warp_max_u32(m0);
        m1 = warp_max_u32(m1);
        if ((threadIdx.x & 31) == 0) {
            if (m0) atomicMax(&smax[0], m0);
            if (m1) atomicMax(&smax[1], m1);
        }
    }
    __syncthreads();
    for (uint32_t i = threadIdx.x; i < 2 * G; i += blockDim.x)
        if (smax[i]) atomicMax(&maxabs[i], smax[i]);
}

__global__ void k_maxabs(const float2* __restrict__ gh, uint64_t n, unsigned* __restrict__ maxabs) {
    BST_PDL_ENTER();
    __shared__ unsigned smax[2];
    if (threadIdx.x < 2) smax[threadIdx.x] = 0u;
    __syncthreads();
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    unsigned m0 = 0u, m1 = 0u;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) {
        const float2 v = gh[i];
        m0 = max(m0, abs_bits(v.x));
        m1 = max(m1, abs_bits(v.y));
    }
    m0 = warp_max_u32(m0);
    m1 = warp_max_u32(m1);
    if ((threadIdx.x & 31) == 0) {
        if (m0) atomicMax(&smax[0], m0);
        if (m1) atomicMax(&smax[1], m1);
    }
    __syncthreads();
    if (threadIdx.x < 2 && smax[threadIdx.x]) atomicMax(&maxabs[threadIdx.x], smax[threadIdx.x]);
}

void launch_maxabs(const float2* gh, uint64_t n, unsigned* maxabs, cudaStream_t st) {
    if (n == 0) return;
    uint64_t blocks = (n + 255) / 256;
    if (blocks > (uint64_t)sm_count() * 8) blocks = (uint64_t)sm_count() * 8;
    launch_k(k_maxabs, (unsigned)blocks, 256, 0, st, gh, n, maxabs);
}

void launch_gradients(int objective, uint32_t G, const float* pred, const float* y,
                      const float* w, uint64_t n, float2* gh, unsigned* maxabs,
                      cudaStream_t st, const float* alpha, float delta) {
    if (n == 0) return;
    uint64_t blocks = (n + 255) / 256;
    if (blocks > (uint64_t)sm_count() * 8) blocks = (uint64_t)sm_count() * 8;
    launch_k(k_gradients, (unsigned)blocks, 256, 2 * G * sizeof(unsigned), st, objective, G, pred, y, w, n, gh, maxabs,
                                                                          alpha, delta);
}

// Fixed-point scale of element i (output i / 2, grad or hess i % 2).
__device__ void write_fixed_scale(const unsigned* __restrict__ maxabs, uint32_t i, uint64_t n,
                                  double* __restrict__ scales) {
    const float m = __uint_as_float(maxabs[i]);
    int k = 0;
    if (m > 0.0f) {
        int e, en;
        frexp((double)m, &e);  // max|v| < 2^e
        frexp((double)n, &en);  // n < 2^en
        // |q| <= 2^B: 4096-row shared-memory partial sums fit the 32-bit
        // hi/lo split of k_hist_build, and n * 2^B < 2^62 keeps every int64
        // sum exact
        int B = HIST_QBITS;
        if (61 - en < B) B = 61 - en;
        k = B - e;
        if (k > 1000) k = 1000;
        if (k < -1000) k = -1000;
    }
    const uint32_t o = i >> 1, which = i & 1;
    scales[4 * o + which] = ldexp(1.0, k);
    scales[4 * o + 2 + which] = ldexp(1.0, -k);
}

__global__ void k_fixed_scales(const unsigned* __restrict__ maxabs, uint32_t G, uint64_t n,
                               double* __restrict__ scales) {
    BST_PDL_ENTER();
    const uint32_t i = blockIdx.x * blockDim.x + threadIdx.x;
    if (i < 2 * G) write_fixed_scale(maxabs, i, n, scales);
}

void launch_fixed_scales(const unsigned* maxabs, uint32_t G, uint64_t n, double* scales,
                         cudaStream_t st) {
    launch_k(k_fixed_scales, (2 * G + 63) / 64, 64, 0, st, maxabs, G, n, scales);
}

// ============================================================================
// K4: histogram build (HistogramBuilder, training/gbdt/histograms/ops.rs:79-127)
// Shared-memory privatised fixed-point histograms over a tile of columns,
// 128-bit row loads, one global atomic flush per non-empty bin.
// Each int64 value q (|q| <= 2^38) is split exactly into lo = q mod 2^20 and
// hi = q >> 20, accumulated with 32-bit shared atomics (several times the
// throughput of 64-bit shared atomics on B200); a block covers at most 4096
// rows, so 4096 * 2^20 < 2^32 and 4096 * 2^18 < 2^31 and the recombined
// sums hi * 2^20 + lo are exact.
// ============================================================================

constexpr int HIST_THREADS = 256;

// Shared-memory words per histogram bin: 4 for the hi/lo split of the 64-bit
// fixed-point values, 2 for quantised values (one 32-bit sum each for grad
// and hess: a block covers <= 4096 rows of |q| <= 32767, so 4096 * 32767 <
// 2^31 and the 32-bit sums are exact).
__host__ __device__ constexpr uint32_t acc_words(int mode) { return mode == GRAD_F32 ? 4u : 2u; }

template <int MODE>
struct GradLoad;
// operator()(row): the row's element by row id; at(pos, row): by its
// position in the row-id buffer when the positional copy exists.
template <>
struct GradLoad<GRAD_F32> {
    const float2* __restrict__ gh;
    const float2* __restrict__ qp;
    double sg, sh;
    __device__ explicit GradLoad(const GradRef& r)
        : gh(r.gh), qp(static_cast<const float2*>(r.qpos)), sg(r.scale[0]), sh(r.scale[1]) {}
    __device__ __forceinline__ void conv(float2 v, long long& g, long long& h) const {
        g = quantize(v.x, sg);
        h = quantize(v.y, sh);
    }
    __device__ __forceinline__ void operator()(uint32_t row, long long& g, long long& h) const { conv(gh[row], g, h); }
    __device__ __forceinline__ void at(uint32_t pos, uint32_t row, long long& g, long long& h) const {
        conv(qp ? qp[pos] : gh[row], g, h);
    }
};
template <>
struct GradLoad<GRAD_Q16> {
    const short2* __restrict__ q;
    const short2* __restrict__ qp;
    __device__ explicit GradLoad(const GradRef& r)
        : q(static_cast<const short2*>(r.gq)), qp(static_cast<const short2*>(r.qpos)) {}
    __device__ __forceinline__ void operator()(uint32_t row, long long& g, long long& h) const {
        const short2 v = q[row];
        g = v.x;
        h = v.y;
    }
    __device__ __forceinline__ void at(uint32_t pos, uint32_t row, long long& g, long long& h) const {
        const short2 v = qp ? qp[pos] : q[row];
        g = v.x;
        h = v.y;
    }
};
template <>
struct GradLoad<GRAD_Q8> {
    const char2* __restrict__ q;
    const char2* __restrict__ qp;
    __device__ explicit GradLoad(const GradRef& r)
        : q(static_cast<const char2*>(r.gq)), qp(static_cast<const char2*>(r.qpos)) {}
    __device__ __forceinline__ void operator()(uint32_t row, long long& g, long long& h) const {
        const char2 v = q[row];
        g = v.x;
        h = v.y;
    }
    __device__ __forceinline__ void at(uint32_t pos, uint32_t row, long long& g, long long& h) const {
        const char2 v = qp ? qp[pos] : q[row];
        g = v.x;
        h = v.y;
    }
};

template <int MODE>
__device__ __forceinline__ void hist_add(uint32_t* s, uint32_t S, uint32_t idx, long long qg, long long qh) {
    if constexpr (MODE == GRAD_F32) {
        const uint32_t lo_mask = (1u << HIST_LO_BITS) - 1u;
        atomicAdd(&s[idx], (uint32_t)qg & lo_mask);
        atomicAdd(&s[S + idx], (uint32_t)(qg >> HIST_LO_BITS));
        atomicAdd(&s[2 * S + idx], (uint32_t)qh & lo_mask);
        atomicAdd(&s[3 * S + idx], (uint32_t)(qh >> HIST_LO_BITS));
    } else {
        atomicAdd(&s[idx], (uint32_t)(int32_t)qg);
        atomicAdd(&s[S + idx], (uint32_t)(int32_t)qh);
    }
}

// Node-histogram element access for both bin types.
template <typename HB>
__device__ __forceinline__ HB hb_make(long long g, long long h) {
    HB r;
    r.g = (decltype(r.g))g;
    r.h = (decltype(r.h))h;
    return r;
}
__device__ __forceinline__ void hb_atomic_add(HBin* p, long long g, long long h) {
    atomicAdd(reinterpret_cast<unsigned long long*>(&p->g), (unsigned long long)g);
    atomicAdd(reinterpret_cast<unsigned long long*>(&p->h), (unsigned long long)h);
}
__device__ __forceinline__ void hb_atomic_add(HBin32* p, long long g, long long h) {
    atomicAdd(&p->g, (int)g);
    atomicAdd(&p->h, (int)h);
}

// One (row chunk, column tile) item: zero the shared histogram, accumulate,
// flush to the global histogram of chunk.slot. Block-uniform; `tile` is in
// shared memory; returns with the shared histogram free for reuse.
template <int MODE, typename HB = HBin>
__device__ void hist_item(const HistChunk& chunk, const HistTile& tile, uint32_t* sm, uint32_t S,
                          const uint32_t* __restrict__ ridx, const GradLoad<MODE>& load,
                          const uint8_t* __restrict__ bins8, uint32_t s8, const uint16_t* __restrict__ bins16,
                          uint32_t s16, HB* __restrict__ hist, uint64_t slot_bins) {
    constexpr uint32_t NW = acc_words(MODE);
    for (uint32_t i = threadIdx.x; i < S * NW / 4; i += HIST_THREADS)  // S is a multiple of 4
        reinterpret_cast<uint4*>(sm)[i] = make_uint4(0, 0, 0, 0);
    __syncthreads();

    const uint32_t c0 = tile.c0, c1 = tile.c1;
    uint32_t loff[16], lnb[16];
#pragma unroll
    for (int l = 0; l < 16; ++l) {
        loff[l] = tile.lane_smem[l];
        lnb[l] = tile.lane_nbins[l];
    }
    const bool ident = chunk.flags & 1u;
    const uint32_t count = min(chunk.count, (uint32_t)HIST_CHUNK_MAX);
    if (tile.matrix == 0) {
        const uint8_t* base = bins8 + (size_t)tile.vec * 16u;
        for (uint32_t i = threadIdx.x; i < count; i += HIST_THREADS) {
            const uint32_t p = chunk.begin + i;
            const uint32_t row = ident ? p : ridx[p];
            long long qg, qh;
            load(row, qg, qh);
            const uint4 b = *reinterpret_cast<const uint4*>(base + (size_t)row * s8);
            const uint32_t words[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
            for (int l = 0; l < 16; ++l) {
                if (l >= (int)c0 && l < (int)c1) {
                    const uint32_t bin = (words[l >> 2] >> ((l & 3) * 8)) & 0xFFu;
                    if (bin < lnb[l]) hist_add<MODE>(sm, S, loff[l] + bin, qg, qh);
                }
            }
        }
    } else {
        const uint16_t* base = bins16 + (size_t)tile.vec * 8u;
        for (uint32_t i = threadIdx.x; i < count; i += HIST_THREADS) {
            const uint32_t p = chunk.begin + i;
            const uint32_t row = ident ? p : ridx[p];
            long long qg, qh;
            load(row, qg, qh);
            const uint4 b = *reinterpret_cast<const uint4*>(base + (size_t)row * s16);
            const uint32_t words[4] = {b.x, b.y, b.z, b.w};
#pragma unroll
            for (int l = 0; l < 8; ++l) {
                if (l >= (int)c0 && l < (int)c1) {
                    const uint32_t bin = (words[l >> 1] >> ((l & 1) * 16)) & 0xFFFFu;
                    if (bin < lnb[l]) hist_add<MODE>(sm, S, loff[l] + bin, qg, qh);
                }
            }
        }
    }
    __syncthreads();
    HB* out = hist + (size_t)chunk.slot * slot_bins;
    for (uint32_t l = c0; l < c1; ++l) {
        const uint32_t so = tile.lane_smem[l], go = tile.lane_hist[l], nb = tile.lane_nbins[l];
        for (uint32_t b = threadIdx.x; b < nb; b += HIST_THREADS) {
            const uint32_t j = so + b;
            long long g, h;
            if constexpr (MODE == GRAD_F32) {
                const uint32_t glo = sm[j], ghi = sm[S + j], hlo = sm[2 * S + j], hhi = sm[3 * S + j];
                if (!(glo | ghi | hlo | hhi)) continue;
                g = (long long)(int32_t)ghi * (1ll << HIST_LO_BITS) + (long long)glo;
                h = (long long)(int32_t)hhi * (1ll << HIST_LO_BITS) + (long long)hlo;
            } else {
                const uint32_t gw = sm[j], hw = sm[S + j];
                if (!(gw | hw)) continue;
                g = (int32_t)gw;
                h = (int32_t)hw;
            }
            hb_atomic_add(&out[go + b], g, h);
        }
    }
    __syncthreads();
}

// ---- column-lane tiles ------------------------------------------------------

// Shared histogram of a lane tile: LANE_ROWS bins x 32 slots per accumulator
// plane (fixed height, so plane offsets are immediates).
constexpr uint32_t LANE_ROWS = 264;
constexpr uint32_t LANE_PART_STRIDE = LANE_ROWS * 32u;  // partial entries per item
constexpr uint32_t LANE_STAGES = 3;  // cp.async ring depth per warp
constexpr uint32_t LANE_SLOT = 48;   // bytes per lane per stage (32 + 16 pad: conflict-free 16-byte reads)
constexpr uint32_t LANE_REG_STAGES = 2;  // register ring depth per lane

constexpr uint32_t LANE_TMA_STAGES = 4;   // TMA ring depth per warp
constexpr uint32_t LANE_TMA_STAGE = 1024;  // bytes per warp and stage: 32 rows x 32 bytes

// Variants of the lane-tile kernel (the launch-shape tuner's `hist` knob):
//   0: each warp stages its rows' windows through a LANE_STAGES-deep cp.async
//      ring in shared memory; 256 threads (512 for the fixed-point form)
//   1: a LANE_REG_STAGES-deep ring of 128-bit register loads instead (no
//      staging memory: more resident blocks per SM); 256 / 512 threads
//   2: the register ring with 512-thread blocks
//   3: the windows gathered by the tensor memory accelerator (tile::gather4,
//      four rows per copy, issued by eight lanes of the warp) into a
//      LANE_TMA_STAGES-deep ring completed by mbarriers: the copies bypass
//      the load/store pipe that the shared-memory atomics need
// Every variant sums the same values into the same partials.
constexpr int LANE_VARIANTS = 4;
__host__ __device__ constexpr uint32_t lane_threads(int mode, int v) {
    return v == 2 ? 512u : (mode == GRAD_F32 ? 512u : 256u);
}
__host__ __device__ constexpr bool lane_regs(int v) { return v == 1 || v == 2; }
__host__ __device__ constexpr uint32_t lane_smem_bytes(int mode, int v) {
    return LANE_ROWS * 32u * acc_words(mode) * 4u +
           (v == 3 ? (lane_threads(mode, v) / 32u) * LANE_TMA_STAGES * (LANE_TMA_STAGE + 8u)
                   : (lane_regs(v) ? 0u : (lane_threads(mode, v) / 32u) * LANE_STAGES * 32u * LANE_SLOT));
}
// minimum resident blocks per SM asked of the compiler: a register budget
// (65536 / (threads x blocks) per thread); variant 0 keeps its 64 registers
__host__ __device__ constexpr uint32_t lane_min_blocks(int mode, int v) {
    return mode == GRAD_F32 ? 1u : (v == 0 ? 4u : (v == 1 ? 3u : 2u));
}

uint32_t lane_tile_max_bins(int) { return LANE_ROWS; }
int lane_variants() { return LANE_VARIANTS; }

uint32_t lane_segment_max(int mode) { return mode == GRAD_F32 ? (uint32_t)HIST_CHUNK_MAX : 16384u; }
uint32_t lane_part_entry_bytes(int mode) { return mode == GRAD_F32 ? 16u : 8u; }
uint32_t lane_part_stride() { return LANE_PART_STRIDE; }

template <int MODE>
struct LaneAdd;
template <>
struct LaneAdd<GRAD_F32> {  // hi/lo split of the 64-bit fixed-point values
    uint32_t glo, ghi, hlo, hhi;
    LaneAdd() = default;
    __device__ LaneAdd(long long qg, long long qh) {
        const uint32_t lo_mask = (1u << HIST_LO_BITS) - 1u;
        glo = (uint32_t)qg & lo_mask;
        ghi = (uint32_t)(qg >> HIST_LO_BITS);
        hlo = (uint32_t)qh & lo_mask;
        hhi = (uint32_t)(qh >> HIST_LO_BITS);
    }
    __device__ __forceinline__ void add(uint32_t* sm, uint32_t plane, uint32_t idx) const {
        atomicAdd(&sm[idx], glo);
        atomicAdd(&sm[plane + idx], ghi);
        atomicAdd(&sm[2 * plane + idx], hlo);
        atomicAdd(&sm[3 * plane + idx], hhi);
    }
    __device__ static void read(const uint32_t* sm, uint32_t plane, uint32_t idx, long long& g, long long& h) {
        g += (long long)(int32_t)sm[plane + idx] * (1ll << HIST_LO_BITS) + (long long)sm[idx];
        h += (long long)(int32_t)sm[3 * plane + idx] * (1ll << HIST_LO_BITS) + (long long)sm[2 * plane + idx];
    }
    // 4 consecutive slots (idx % 4 == 0) added into g[4], h[4]
    __device__ static void read4(const uint32_t* sm, uint32_t plane, uint32_t idx, long long* g, long long* h) {
        const uint4 glo = *reinterpret_cast<const uint4*>(sm + idx);
        const uint4 ghi = *reinterpret_cast<const uint4*>(sm + plane + idx);
        const uint4 hlo = *reinterpret_cast<const uint4*>(sm + 2 * plane + idx);
        const uint4 hhi = *reinterpret_cast<const uint4*>(sm + 3 * plane + idx);
        const uint32_t gl[4] = {glo.x, glo.y, glo.z, glo.w}, gh[4] = {ghi.x, ghi.y, ghi.z, ghi.w};
        const uint32_t hl[4] = {hlo.x, hlo.y, hlo.z, hlo.w}, hh[4] = {hhi.x, hhi.y, hhi.z, hhi.w};
#pragma unroll
        for (int q = 0; q < 4; ++q) {
            g[q] += (long long)(int32_t)gh[q] * (1ll << HIST_LO_BITS) + (long long)gl[q];
            h[q] += (long long)(int32_t)hh[q] * (1ll << HIST_LO_BITS) + (long long)hl[q];
        }
    }
};
template <int MODE>
struct LaneAdd {  // quantised: one 32-bit sum each
    uint32_t g, h;
    LaneAdd() = default;
    __device__ LaneAdd(long long qg, long long qh) : g((uint32_t)(int32_t)qg), h((uint32_t)(int32_t)qh) {}
    __device__ __forceinline__ void add(uint32_t* sm, uint32_t plane, uint32_t idx) const {
        atomicAdd(&sm[idx], g);
        atomicAdd(&sm[plane + idx], h);
    }
    __device__ static void read(const uint32_t* sm, uint32_t plane, uint32_t idx, long long& gs, long long& hs) {
        gs += (int32_t)sm[idx];
        hs += (int32_t)sm[plane + idx];
    }
    __device__ static void read4(const uint32_t* sm, uint32_t plane, uint32_t idx, long long* g, long long* h) {
        const uint4 a = *reinterpret_cast<const uint4*>(sm + idx);
        const uint4 b = *reinterpret_cast<const uint4*>(sm + plane + idx);
        g[0] += (int32_t)a.x;
        g[1] += (int32_t)a.y;
        g[2] += (int32_t)a.z;
        g[3] += (int32_t)a.w;
        h[0] += (int32_t)b.x;
        h[1] += (int32_t)b.y;
        h[2] += (int32_t)b.z;
        h[3] += (int32_t)b.w;
    }
};

// Rows [first, first + count) of a row segment into this block's shared
// histogram (zeroed by the caller). Each warp streams its rows' bin windows
// into a LANE_STAGES-deep ring of shared-memory stages with cp.async (issued
// LANE_STAGES - 1 iterations ahead, so the gathers overlap the atomics);
// gradients are prefetched into registers the same distance ahead.
// The window's words, rotated left by this lane's column offset, added to
// the lane's slots (shared by both staging forms).
template <int MODE, int ESIZE, int WORDS>
__device__ __forceinline__ void lane_add_window(uint32_t (&w)[WORDS], uint32_t lr, uint32_t slot0, uint32_t rq,
                                                uint32_t rs, const LaneAdd<MODE> a, uint32_t* sm) {
    constexpr uint32_t C = WORDS * 4 / ESIZE;
    constexpr uint32_t plane = LANE_ROWS * 32u;
    // rotate left by rb bytes: whole words by rq, then bytes by rs bits
#pragma unroll
    for (int st = 1; st < WORDS; st <<= 1) {
        const bool take = (rq & (uint32_t)st) != 0u;
        uint32_t t[WORDS];
#pragma unroll
        for (int q = 0; q < WORDS; ++q) t[q] = take ? w[(q + st) % WORDS] : w[q];
#pragma unroll
        for (int q = 0; q < WORDS; ++q) w[q] = t[q];
    }
    {
        uint32_t t[WORDS];
#pragma unroll
        for (int q = 0; q < WORDS; ++q) t[q] = __funnelshift_r(w[q], w[(q + 1) % WORDS], rs);
#pragma unroll
        for (int q = 0; q < WORDS; ++q) w[q] = t[q];
    }
#pragma unroll
    for (uint32_t j = 0; j < C; ++j) {
        uint32_t e;
        if (ESIZE == 1)
            e = (w[j >> 2] >> ((j & 3u) * 8u)) & 0xFFu;
        else
            e = (w[j >> 1] >> ((j & 1u) * 16u)) & 0xFFFFu;
        a.add(sm, plane, e * 32u + slot0 + ((lr + j) & (C - 1u)));
    }
}

// 16 bytes of a gathered row window: read-only path, no L1 allocation (each
// window is read once), and a 128-byte L2 fetch so that the row record's
// other windows, read by the blocks of the same row segment at about the same
// time, hit L2.
__device__ __forceinline__ uint4 ld_window16(const uint8_t* p) {
    uint4 v;
    asm volatile("ld.global.nc.L1::no_allocate.L2::128B.v4.u32 {%0, %1, %2, %3}, [%4];"
                 : "=r"(v.x), "=r"(v.y), "=r"(v.z), "=r"(v.w)
                 : "l"(p));
    return v;
}

// Register-staged form: each lane keeps LANE_REG_STAGES of its rows'
// windows in flight as 128-bit loads (the ring shifts by register moves).
template <int MODE, int ESIZE, int WORDS>
__device__ void lane_accumulate_regs(uint32_t first, uint32_t count, bool ident, const LaneTile& tile, uint32_t* sm,
                                     const uint32_t* __restrict__ ridx, const GradLoad<MODE>& load,
                                     const uint8_t* __restrict__ matrix, uint32_t stride) {
    constexpr uint32_t C = WORDS * 4 / ESIZE;
    constexpr uint32_t S = LANE_REG_STAGES;
    constexpr int V = WORDS / 4;  // 128-bit loads per window
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const uint32_t lr = lane % C, slot0 = (lane / C) * C;
    const uint32_t rb = lr * ESIZE;
    const uint32_t rq = rb >> 2, rs = (rb & 3u) * 8u;
    const uint8_t* base = matrix + tile.byte_off;
    const uint32_t step = nwarps * 32u;
    const uint32_t i0 = warp * 32u + lane;
    uint4 ring[S][V];
    LaneAdd<MODE> gring[S];
    auto fetch = [&](uint32_t i, uint4 (&dst)[V], LaneAdd<MODE>& g) {
        const uint32_t p = first + i;
        const uint32_t row = ident ? p : ridx[p];
        const uint8_t* src = base + (size_t)row * stride;
#pragma unroll
        for (int v = 0; v < V; ++v) dst[v] = ld_window16(src + 16 * v);
        long long qg, qh;
        load.at(p, row, qg, qh);
        g = LaneAdd<MODE>(qg, qh);
    };
#pragma unroll
    for (uint32_t k = 0; k + 1 < S; ++k) {
        const uint32_t i = i0 + k * step;
        if (i < count) fetch(i, ring[k], gring[k]);
    }
    for (uint32_t k = 0; warp * 32u + k * step < count; ++k) {
        {
            const uint32_t i = i0 + (k + S - 1) * step;
            if (i < count) fetch(i, ring[S - 1], gring[S - 1]);
        }
        const uint32_t i = i0 + k * step;
        if (i < count) {
            uint32_t w[WORDS];
#pragma unroll
            for (int v = 0; v < V; ++v) {
                w[4 * v] = ring[0][v].x;
                w[4 * v + 1] = ring[0][v].y;
                w[4 * v + 2] = ring[0][v].z;
                w[4 * v + 3] = ring[0][v].w;
            }
            lane_add_window<MODE, ESIZE, WORDS>(w, lr, slot0, rq, rs, gring[0], sm);
        }
#pragma unroll
        for (uint32_t q = 0; q + 1 < S; ++q) {
#pragma unroll
            for (int v = 0; v < V; ++v) ring[q][v] = ring[q + 1][v];
            gring[q] = gring[q + 1];
        }
    }
}

template <int MODE, int ESIZE, int WORDS>
__device__ void lane_accumulate(uint32_t first, uint32_t count, bool ident, const LaneTile& tile, uint32_t* sm,
                                uint8_t* stage, const uint32_t* __restrict__ ridx, const GradLoad<MODE>& load,
                                const uint8_t* __restrict__ matrix, uint32_t stride) {
    constexpr uint32_t C = WORDS * 4 / ESIZE;  // columns in the window
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const uint32_t lr = lane % C, slot0 = (lane / C) * C;
    const uint32_t rb = lr * ESIZE;  // left rotation of the window, bytes
    const uint32_t rq = rb >> 2, rs = (rb & 3u) * 8u;
    const uint8_t* base = matrix + tile.byte_off;
    const uint32_t step = nwarps * 32u;
    // this lane's slot in stage s: stage + (warp * LANE_STAGES + s) * 32 * LANE_SLOT + lane * LANE_SLOT
    uint8_t* my = stage + (size_t)warp * LANE_STAGES * 32u * LANE_SLOT + lane * LANE_SLOT;
    const uint32_t my_s = (uint32_t)__cvta_generic_to_shared(my);
    auto row_at = [&](uint32_t i) -> uint32_t {
        const uint32_t p = first + i;
        return ident ? p : ridx[p];
    };
    auto issue = [&](uint32_t row, uint32_t s) {
        const uint8_t* src = base + (size_t)row * stride;
        const uint32_t dst = my_s + s * 32u * LANE_SLOT;
#pragma unroll
        for (int v = 0; v < WORDS / 4; ++v)
            asm volatile("cp.async.cg.shared.global.L2::128B [%0], [%1], 16;" ::"r"(dst + 16u * v),
                         "l"(src + 16 * v)
                         : "memory");
    };
    const uint32_t i0 = warp * 32u + lane;
    // prologue: iterations 0 .. LANE_STAGES - 2
    LaneAdd<MODE> ring[LANE_STAGES];
#pragma unroll
    for (uint32_t k = 0; k < LANE_STAGES - 1; ++k) {
        const uint32_t i = i0 + k * step;
        ring[k] = LaneAdd<MODE>(0, 0);
        if (i < count) {
            const uint32_t row = row_at(i);
            issue(row, k);
            long long qg, qh;
            load.at(first + i, row, qg, qh);
            ring[k] = LaneAdd<MODE>(qg, qh);
        }
        asm volatile("cp.async.commit_group;" ::: "memory");
    }
    uint32_t row_next = 0;  // row id of iteration k + LANE_STAGES - 1
    {
        const uint32_t i = i0 + (LANE_STAGES - 1) * step;
        if (i < count) row_next = row_at(i);
    }
    uint32_t s_cur = 0, s_new = LANE_STAGES - 1;
    for (uint32_t k = 0; warp * 32u + k * step < count; ++k) {
        // issue iteration k + LANE_STAGES - 1
        {
            const uint32_t i = i0 + (k + LANE_STAGES - 1) * step;
            ring[LANE_STAGES - 1] = LaneAdd<MODE>(0, 0);
            if (i < count) {
                issue(row_next, s_new);
                long long qg, qh;
                load.at(first + i, row_next, qg, qh);
                ring[LANE_STAGES - 1] = LaneAdd<MODE>(qg, qh);
            }
            asm volatile("cp.async.commit_group;" ::: "memory");
            const uint32_t i2 = i + step;
            row_next = i2 < count ? row_at(i2) : 0u;
        }
        asm volatile("cp.async.wait_group %0;" ::"n"(LANE_STAGES - 1) : "memory");
        const uint32_t i = i0 + k * step;
        if (i < count) {
            uint32_t w[WORDS];
            const uint4* src = reinterpret_cast<const uint4*>(my + s_cur * 32u * LANE_SLOT);
#pragma unroll
            for (int v = 0; v < WORDS / 4; ++v) {
                const uint4 t = src[v];
                w[4 * v] = t.x;
                w[4 * v + 1] = t.y;
                w[4 * v + 2] = t.z;
                w[4 * v + 3] = t.w;
            }
            lane_add_window<MODE, ESIZE, WORDS>(w, lr, slot0, rq, rs, ring[0], sm);
        }
#pragma unroll
        for (uint32_t q = 0; q + 1 < LANE_STAGES; ++q) ring[q] = ring[q + 1];
        s_cur = s_cur + 1 == LANE_STAGES ? 0u : s_cur + 1;
        s_new = s_new + 1 == LANE_STAGES ? 0u : s_new + 1;
    }
    asm volatile("cp.async.wait_group 0;" ::: "memory");
}

// ---- TMA form (variant 3) ----------------------------------------------------
// A wait on an mbarrier gives up after this many polls (far beyond any copy's
// latency): the kernel then records the failure in BState::err, stops
// issuing, waits (bounded) for the copies it issued and returns.
constexpr uint32_t TMA_WAIT_POLLS = 1u << 24;

__device__ __forceinline__ bool mbar_wait(uint32_t bar, uint32_t parity) {
    for (uint32_t it = 0; it < TMA_WAIT_POLLS; ++it) {
        uint32_t done;
        asm volatile(
            "{\n .reg .pred p;\n mbarrier.try_wait.parity.shared::cta.b64 p, [%1], %2;\n selp.u32 %0, 1, 0, p;\n}\n"
            : "=r"(done)
            : "r"(bar), "r"(parity)
            : "memory");
        if (done) return true;
    }
    return false;
}

// Rows [first, first + count) of a row segment: per iteration a warp's 32
// rows are gathered by lanes 0-7 (four rows each) into stage s, whose
// mbarrier expects the stage's bytes; each lane then reads its row's window
// from shared memory. Stage rows are packed 4 x 32 bytes per gather, so a
// lane of an odd group of four reads its two 16-byte halves in swapped
// order (conflict-free 128-bit reads).
template <int MODE, int ESIZE, int WORDS>
__device__ bool lane_accumulate_tma(uint32_t first, uint32_t count, bool ident, const LaneTile& tile, uint32_t* sm,
                                    uint8_t* stage, uint64_t* bars, const uint32_t* __restrict__ ridx,
                                    const GradLoad<MODE>& load, const CUtensorMap* tmap, uint32_t n_rows,
                                    uint32_t* err, uint32_t& parity_bits) {
    constexpr uint32_t C = WORDS * 4 / ESIZE;
    constexpr uint32_t S = LANE_TMA_STAGES;
    constexpr uint32_t BOX = WORDS * 4;  // bytes per gathered row: 32 or 16
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5, nwarps = blockDim.x >> 5;
    const uint32_t lr = lane % C, slot0 = (lane / C) * C;
    const uint32_t rb = lr * ESIZE;
    const uint32_t rq = rb >> 2, rs = (rb & 3u) * 8u;
    const uint32_t step = nwarps * 32u;
    const uint32_t i0 = warp * 32u + lane;
    uint8_t* wstage = stage + (size_t)warp * S * LANE_TMA_STAGE;
    const uint32_t wstage_s = (uint32_t)__cvta_generic_to_shared(wstage);
    const uint32_t bar0 = (uint32_t)__cvta_generic_to_shared(bars + (size_t)warp * S);
    const int x = (int)tile.rec_off;
    const uint32_t grp = lane >> 2, in_grp = lane & 3u;
    // this lane's row in a stage: a gather group of 4 rows of BOX bytes at
    // each 128-byte boundary (the copies' destinations stay 128-byte aligned)
    const uint32_t my_off = grp * 128u + in_grp * BOX;
    const bool swap = (grp & 1u) != 0u && WORDS == 8;
    bool failed = false;
    auto row_at = [&](uint32_t i) -> uint32_t {
        const uint32_t p = first + i;
#ifdef BST_CHECKED
        const uint32_t r = i < count ? (ident ? p : ridx[p]) : n_rows;
        return (r == n_rows || BST_IN(r, n_rows, CHECK_HIST_ROW)) ? r : n_rows;
#else
        return i < count ? (ident ? p : ridx[p]) : n_rows;  // n_rows: out of range, zero-filled
#endif
    };
    // issue iteration k (rows of all lanes) into stage s
    auto issue = [&](uint32_t row, uint32_t s) {
        const uint32_t r0 = __shfl_sync(FULL, row, (4u * (lane & 7u)) + 0u);
        const uint32_t r1 = __shfl_sync(FULL, row, (4u * (lane & 7u)) + 1u);
        const uint32_t r2 = __shfl_sync(FULL, row, (4u * (lane & 7u)) + 2u);
        const uint32_t r3 = __shfl_sync(FULL, row, (4u * (lane & 7u)) + 3u);
        const uint32_t bar = bar0 + s * 8u;
        // the stage's previous contents were read by the generic proxy
        asm volatile("fence.proxy.async.shared::cta;" ::: "memory");
        __syncwarp();
        if (lane == 0)
            asm volatile("mbarrier.arrive.expect_tx.shared::cta.b64 _, [%0], %1;" ::"r"(bar), "r"(8u * 4u * BOX)
                         : "memory");
        __syncwarp();
        if (lane < 8) {
            const uint32_t dst = wstage_s + s * LANE_TMA_STAGE + lane * 128u;
            asm volatile(
                "cp.async.bulk.tensor.2d.shared::cluster.global.tile::gather4.mbarrier::complete_tx::bytes"
                " [%0], [%1, {%2, %3, %4, %5, %6}], [%7];" ::"r"(dst),
                "l"(reinterpret_cast<uint64_t>(tmap)), "r"(x), "r"(r0), "r"(r1), "r"(r2), "r"(r3), "r"(bar)
                : "memory");
        }
    };
    LaneAdd<MODE> ring[S];
    const uint32_t iters = count > warp * 32u ? (count - warp * 32u + step - 1) / step : 0u;
#pragma unroll
    for (uint32_t k = 0; k + 1 < S; ++k) {
        ring[k] = LaneAdd<MODE>(0, 0);
        if (k < iters) {
            const uint32_t i = i0 + k * step;
            const uint32_t row = row_at(i);
            issue(row, k);
            if (i < count) {
                long long qg, qh;
                load.at(first + i, row, qg, qh);
                ring[k] = LaneAdd<MODE>(qg, qh);
            }
        }
    }
    for (uint32_t k = 0; k < iters; ++k) {
        const uint32_t s_cur = k % S;
        {
            const uint32_t kn = k + S - 1;  // issue iteration kn
            ring[S - 1] = LaneAdd<MODE>(0, 0);
            if (kn < iters && !failed) {
                const uint32_t i = i0 + kn * step;
                const uint32_t row = row_at(i);
                issue(row, kn % S);
                if (i < count) {
                    long long qg, qh;
                    load.at(first + i, row, qg, qh);
                    ring[S - 1] = LaneAdd<MODE>(qg, qh);
                }
            }
        }
        if (!failed) {
            const uint32_t par = (parity_bits >> s_cur) & 1u;
            const bool ok = mbar_wait(bar0 + s_cur * 8u, par);
            if (!__all_sync(FULL, ok)) {  // warp-uniform: the issue path shuffles across the warp
                failed = true;
                if (lane == 0) atomicExch(err, 1u);
            }
            parity_bits ^= 1u << s_cur;
        }
        const uint32_t i = i0 + k * step;
        if (!failed && i < count) {
            const uint8_t* src = wstage + s_cur * LANE_TMA_STAGE + my_off;
            uint32_t w[WORDS];
            if constexpr (WORDS == 8) {
                const uint4 a = *reinterpret_cast<const uint4*>(src + (swap ? 16 : 0));
                const uint4 b = *reinterpret_cast<const uint4*>(src + (swap ? 0 : 16));
                const uint4 lo = swap ? b : a, hi = swap ? a : b;
                w[0] = lo.x; w[1] = lo.y; w[2] = lo.z; w[3] = lo.w;
                w[4] = hi.x; w[5] = hi.y; w[6] = hi.z; w[7] = hi.w;
            } else {
                const uint4 a = *reinterpret_cast<const uint4*>(src);
                w[0] = a.x; w[1] = a.y; w[2] = a.z; w[3] = a.w;
            }
            lane_add_window<MODE, ESIZE, WORDS>(w, lr, slot0, rq, rs, ring[0], sm);
        }
#pragma unroll
        for (uint32_t q = 0; q + 1 < S; ++q) ring[q] = ring[q + 1];
    }
    // after a failed wait, the copies still in flight must land before the
    // block's shared memory is reused: wait (bounded) on every stage's
    // pending phase, then report the failure (the caller stops)
    if (failed)
        for (uint32_t s = 0; s < S; ++s) mbar_wait(bar0 + s * 8u, (parity_bits >> s) & 1u);
    return !failed;
}

template <int MODE, int ESIZE, int WORDS, bool REGS>
__device__ __forceinline__ void lane_accumulate_v(uint32_t first, uint32_t count, bool ident, const LaneTile& t,
                                                  uint32_t* sm, uint8_t* stage, const uint32_t* __restrict__ ridx,
                                                  const GradLoad<MODE>& load, const uint8_t* __restrict__ m,
                                                  uint32_t stride) {
    if constexpr (REGS)
        lane_accumulate_regs<MODE, ESIZE, WORDS>(first, count, ident, t, sm, ridx, load, m, stride);
    else
        lane_accumulate<MODE, ESIZE, WORDS>(first, count, ident, t, sm, stage, ridx, load, m, stride);
}

template <int MODE, bool REGS>
__device__ __forceinline__ void lane_accumulate_any(uint32_t first, uint32_t count, bool ident, const LaneTile& t,
                                                    uint32_t* sm, uint8_t* stage, const uint32_t* __restrict__ ridx,
                                                    const GradLoad<MODE>& load, const uint8_t* __restrict__ bins8,
                                                    uint32_t s8, const uint16_t* __restrict__ bins16, uint32_t s16) {
    if (t.esize == 1) {
        if (t.words == 8)
            lane_accumulate_v<MODE, 1, 8, REGS>(first, count, ident, t, sm, stage, ridx, load, bins8, s8);
        else
            lane_accumulate_v<MODE, 1, 4, REGS>(first, count, ident, t, sm, stage, ridx, load, bins8, s8);
    } else {
        const uint8_t* m = reinterpret_cast<const uint8_t*>(bins16);
        if (t.words == 8)
            lane_accumulate_v<MODE, 2, 8, REGS>(first, count, ident, t, sm, stage, ridx, load, m, s16 * 2u);
        else
            lane_accumulate_v<MODE, 2, 4, REGS>(first, count, ident, t, sm, stage, ridx, load, m, s16 * 2u);
    }
}

__device__ __forceinline__ void load_lane_tile(LaneTile& dst, const LaneTile& src) {
    const uint32_t* s = reinterpret_cast<const uint32_t*>(&src);
    uint32_t* d = reinterpret_cast<uint32_t*>(&dst);
    for (uint32_t i = threadIdx.x; i < sizeof(LaneTile) / 4u; i += blockDim.x) d[i] = s[i];
}

// ---- row-segment partial histograms and the merge ----------------------------
// A work item is (row segment c, lane tile t): one block accumulates the
// segment's rows for the tile's columns in shared memory, then writes the
// tile's bins, copies summed, as partial[c * n_tiles + t][element * n_bins +
// bin] (column-major: a column's bins are contiguous, as in the node
// histogram) with plain stores (no global atomics: each partial has one
// writer). k_b_merge then sums a node's partials and applies the
// subtraction trick. Segments come from the level state: segment c belongs
// to expanding node seg_exp[c] and covers rows small_begin + (c - hist_off) *
// hist_chunk .. of that node's smaller child.

template <int MODE>
struct PartEntry;
template <>
struct PartEntry<GRAD_F32> {
    using T = longlong2;
    __device__ static T make(long long g, long long h) { return make_longlong2(g, h); }
};
template <int MODE>
struct PartEntry {
    using T = int2;  // per-block sums of <= 16384 quantised values fit int32
    __device__ static T make(long long g, long long h) { return make_int2((int)g, (int)h); }
};

template <int MODE>
__device__ void part_flush(const LaneTile& tile, const uint32_t* sm, typename PartEntry<MODE>::T* __restrict__ out);

template <int MODE, bool REGS>
__device__ void part_item(uint32_t first, uint32_t count, const LaneTile& tile, uint32_t* sm, uint8_t* stage,
                          const uint32_t* __restrict__ ridx, const GradLoad<MODE>& load,
                          const uint8_t* __restrict__ bins8, uint32_t s8, const uint16_t* __restrict__ bins16,
                          uint32_t s16, typename PartEntry<MODE>::T* __restrict__ out) {
    constexpr uint32_t NW = acc_words(MODE);
    constexpr uint32_t plane = LANE_ROWS * 32u;
    const uint32_t B = tile.n_bins;  // <= LANE_ROWS
    for (uint32_t w = 0; w < NW; ++w)
        for (uint32_t i = threadIdx.x; i < B * 8u; i += blockDim.x)
            reinterpret_cast<uint4*>(sm + w * plane)[i] = make_uint4(0, 0, 0, 0);
    __syncthreads();
    lane_accumulate_any<MODE, REGS>(first, count, false, tile, sm, stage, ridx, load, bins8, s8, bins16, s16);
    __syncthreads();
    part_flush<MODE>(tile, sm, out);
}

// The tile's partial histogram, copies summed, to out (column-major);
// returns with the shared histogram free for the next item.
template <int MODE>
__device__ void part_flush(const LaneTile& tile, const uint32_t* sm, typename PartEntry<MODE>::T* __restrict__ out) {
    constexpr uint32_t plane = LANE_ROWS * 32u;
    const uint32_t B = tile.n_bins;
    // thread -> (bin b, 4 consecutive elements c4..c4+3), copies summed
    const uint32_t C = tile.words * 4u / tile.esize, K = 32u / C, G4 = C / 4u;
    for (uint32_t t = threadIdx.x; t < B * G4; t += blockDim.x) {
        const uint32_t c4 = (t % G4) * 4u, b = t / G4;
        long long g[4] = {0, 0, 0, 0}, h[4] = {0, 0, 0, 0};
        for (uint32_t k = 0; k < K; ++k) LaneAdd<MODE>::read4(sm, plane, b * 32u + k * C + c4, g, h);
        // lanes t..t+G4-1 take 4 columns each of bin b: each store
        // instruction writes runs of consecutive bins (full 32-byte sectors)
#pragma unroll
        for (uint32_t q = 0; q < 4; ++q) out[(c4 + q) * B + b] = PartEntry<MODE>::make(g[q], h[q]);
    }
    __syncthreads();  // shared histogram free for the next item
}

template <int MODE, int V>
__global__ void __launch_bounds__(lane_threads(MODE, V), lane_min_blocks(MODE, V))
k_b_hist_part(BDev d, const LaneTile* __restrict__ tiles, uint32_t n_tiles, const uint32_t* __restrict__ ridx,
              GradRef gr, const uint8_t* __restrict__ bins8, uint32_t s8, const uint16_t* __restrict__ bins16,
              uint32_t s16, void* __restrict__ part) {
    BST_PDL_ENTER();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint32_t* sm = reinterpret_cast<uint32_t*>(smem_raw);
    uint8_t* stage = smem_raw + acc_words(MODE) * LANE_ROWS * 32u * 4u;
    __shared__ LaneTile tile;
    using E = typename PartEntry<MODE>::T;
    const GradLoad<MODE> load(gr);
    const uint32_t CH = d.state->hist_chunk;
    const uint64_t items = (uint64_t)d.state->hist_chunks * n_tiles;
    for (uint64_t it = blockIdx.x; it < items; it += gridDim.x) {
        const uint32_t c = (uint32_t)(it / n_tiles), t = (uint32_t)(it % n_tiles);
        const BExp e = d.exp[d.seg_exp[c]];
        const uint32_t start = e.small_begin + (c - e.hist_off) * CH;
        const uint32_t count = min(CH, e.small_begin + e.small_count - start);
#ifdef BST_CHECKED
        // the item's rows inside the row-id buffer, and every row id < rows
        bool rows_ok = count == 0 || BST_IN(start + count - 1, d.chk_rows, CHECK_HIST_ROW);
        if (rows_ok)
            for (uint32_t i = threadIdx.x; i < count; i += blockDim.x)
                rows_ok = BST_IN(ridx[start + i], d.chk_rows, CHECK_HIST_ROW) && rows_ok;
        if (!__syncthreads_and(rows_ok)) continue;
#endif
        load_lane_tile(tile, tiles[t]);
        __syncthreads();
        part_item<MODE, lane_regs(V)>(start, count, tile, sm, stage, ridx, load, bins8, s8, bins16, s16,
                                      reinterpret_cast<E*>(part) + (size_t)it * LANE_PART_STRIDE);
    }
}

// Variant 3: the lane-tile partial histograms with the TMA ring. `m32` /
// `m16`: tensor maps of the row records with 32- and 16-byte boxes.
template <int MODE>
__global__ void __launch_bounds__(lane_threads(MODE, 3), lane_min_blocks(MODE, 3))
k_b_hist_part_tma(BDev d, const LaneTile* __restrict__ tiles, uint32_t n_tiles, const uint32_t* __restrict__ ridx,
                  GradRef gr, uint32_t n_rows, void* __restrict__ part, const __grid_constant__ CUtensorMap m32,
                  const __grid_constant__ CUtensorMap m16) {
    BST_PDL_ENTER();
    extern __shared__ __align__(128) unsigned char smem_raw[];
    constexpr uint32_t NW = acc_words(MODE);
    constexpr uint32_t plane = LANE_ROWS * 32u;
    uint32_t* sm = reinterpret_cast<uint32_t*>(smem_raw);
    const uint32_t nwarps = blockDim.x >> 5;
    uint8_t* stage = smem_raw + NW * plane * 4u;  // 128-byte aligned (plane bytes are)
    uint64_t* bars = reinterpret_cast<uint64_t*>(stage + (size_t)nwarps * LANE_TMA_STAGES * LANE_TMA_STAGE);
    __shared__ LaneTile tile;
    using E = typename PartEntry<MODE>::T;
    const GradLoad<MODE> load(gr);
    const uint32_t lane = threadIdx.x & 31u, warp = threadIdx.x >> 5;
    if (lane == 0)
        for (uint32_t q = 0; q < LANE_TMA_STAGES; ++q) {
            const uint32_t b = (uint32_t)__cvta_generic_to_shared(bars + warp * LANE_TMA_STAGES + q);
            asm volatile("mbarrier.init.shared::cta.b64 [%0], 1;" ::"r"(b) : "memory");
        }
    asm volatile("fence.mbarrier_init.release.cluster;" ::: "memory");
    __syncthreads();
    uint32_t parity_bits = 0;
    const uint32_t CH = d.state->hist_chunk;
    const uint64_t items = (uint64_t)d.state->hist_chunks * n_tiles;
    __shared__ int s_fail;
    for (uint64_t it = blockIdx.x; it < items; it += gridDim.x) {
        const uint32_t c = (uint32_t)(it / n_tiles), t = (uint32_t)(it % n_tiles);
        const BExp e = d.exp[d.seg_exp[c]];
        const uint32_t start = e.small_begin + (c - e.hist_off) * CH;
        const uint32_t count = min(CH, e.small_begin + e.small_count - start);
        load_lane_tile(tile, tiles[t]);
        if (threadIdx.x == 0) s_fail = 0;
        __syncthreads();
        for (uint32_t w = 0; w < NW; ++w)
            for (uint32_t i = threadIdx.x; i < tile.n_bins * 8u; i += blockDim.x)
                reinterpret_cast<uint4*>(sm + w * plane)[i] = make_uint4(0, 0, 0, 0);
        __syncthreads();
        bool ok;
        if (tile.words == 8) {
            if (tile.esize == 1)
                ok = lane_accumulate_tma<MODE, 1, 8>(start, count, false, tile, sm, stage, bars, ridx, load, &m32,
                                                     n_rows, &d.state->err, parity_bits);
            else
                ok = lane_accumulate_tma<MODE, 2, 8>(start, count, false, tile, sm, stage, bars, ridx, load, &m32,
                                                     n_rows, &d.state->err, parity_bits);
        } else {
            if (tile.esize == 1)
                ok = lane_accumulate_tma<MODE, 1, 4>(start, count, false, tile, sm, stage, bars, ridx, load, &m16,
                                                     n_rows, &d.state->err, parity_bits);
            else
                ok = lane_accumulate_tma<MODE, 2, 4>(start, count, false, tile, sm, stage, bars, ridx, load, &m16,
                                                     n_rows, &d.state->err, parity_bits);
        }
        if (!ok) s_fail = 1;
        __syncthreads();
        if (s_fail) return;  // the tree is abandoned (BState::err is set)
        part_flush<MODE>(tile, sm, reinterpret_cast<E*>(part) + (size_t)it * LANE_PART_STRIDE);
    }
}

template <int MODE, int V>
static const void* lane_kernel() {
    return reinterpret_cast<const void*>(k_b_hist_part<MODE, V>);
}

static const void* lane_kernel_of(int mode, int v) {
    if (v < 0 || v >= LANE_VARIANTS) v = 0;
    if (v == 3) {
        if (mode == GRAD_F32) return reinterpret_cast<const void*>(k_b_hist_part_tma<GRAD_F32>);
        if (mode == GRAD_Q16) return reinterpret_cast<const void*>(k_b_hist_part_tma<GRAD_Q16>);
        return reinterpret_cast<const void*>(k_b_hist_part_tma<GRAD_Q8>);
    }
    switch (mode * LANE_VARIANTS + v) {
        case GRAD_F32 * LANE_VARIANTS + 0: return lane_kernel<GRAD_F32, 0>();
        case GRAD_F32 * LANE_VARIANTS + 1: return lane_kernel<GRAD_F32, 1>();
        case GRAD_F32 * LANE_VARIANTS + 2: return lane_kernel<GRAD_F32, 2>();
        case GRAD_Q16 * LANE_VARIANTS + 0: return lane_kernel<GRAD_Q16, 0>();
        case GRAD_Q16 * LANE_VARIANTS + 1: return lane_kernel<GRAD_Q16, 1>();
        case GRAD_Q16 * LANE_VARIANTS + 2: return lane_kernel<GRAD_Q16, 2>();
        case GRAD_Q8 * LANE_VARIANTS + 0: return lane_kernel<GRAD_Q8, 0>();
        case GRAD_Q8 * LANE_VARIANTS + 1: return lane_kernel<GRAD_Q8, 1>();
        default: return lane_kernel<GRAD_Q8, 2>();
    }
}

// Resident blocks per SM of a variant (occupancy of the built kernel:
// shared memory, registers and threads), per device and host thread.
uint32_t lane_blocks_per_sm(int mode, int v) {
    if (v < 0 || v >= LANE_VARIANTS) v = 0;
    thread_local int dev_cached = -1;
    thread_local uint32_t cache[3][LANE_VARIANTS];
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) cudaGetLastError();
    if (dev != dev_cached) {
        init_kernel_attributes();
        for (int m = 0; m < 3; ++m)
            for (int k = 0; k < LANE_VARIANTS; ++k) {
                int b = 0;
                if (cudaOccupancyMaxActiveBlocksPerMultiprocessor(&b, lane_kernel_of(m, k), (int)lane_threads(m, k),
                                                                  lane_smem_bytes(m, k)) != cudaSuccess) {
                    cudaGetLastError();
                    b = 1;
                }
                cache[m][k] = b > 0 ? (uint32_t)b : 1u;
            }
        dev_cached = dev;
    }
    return cache[mode >= 0 && mode < 3 ? mode : 0][v];
}

// cuTensorMapEncodeTiled, fetched from the driver through the runtime (no
// link against the driver library).
using EncodeTiledFn = CUresult (*)(CUtensorMap*, CUtensorMapDataType, cuuint32_t, void*, const cuuint64_t*,
                                   const cuuint64_t*, const cuuint32_t*, const cuuint32_t*, CUtensorMapInterleave,
                                   CUtensorMapSwizzle, CUtensorMapL2promotion, CUtensorMapFloatOOBfill);

static EncodeTiledFn encode_tiled() {
    static EncodeTiledFn fn = [] {
        void* p = nullptr;
        cudaDriverEntryPointQueryResult q = cudaDriverEntryPointSymbolNotFound;
        if (cudaGetDriverEntryPoint("cuTensorMapEncodeTiled", &p, cudaEnableDefault, &q) != cudaSuccess ||
            q != cudaDriverEntryPointSuccess) {
            cudaGetLastError();
            p = nullptr;
        }
        return reinterpret_cast<EncodeTiledFn>(p);
    }();
    return fn;
}

bool make_record_maps(RecordMaps& out, const uint8_t* rec, uint64_t n_rows, uint32_t rec_bytes) {
    out.ok = false;
    const EncodeTiledFn fn = encode_tiled();
    // the encoder's limits: 16-byte aligned base and row stride, rows and
    // record bytes within 32 bits
    if (!fn || !rec || n_rows == 0 || n_rows >= (1ull << 31) || rec_bytes == 0 || rec_bytes % 16 != 0 ||
        reinterpret_cast<uintptr_t>(rec) % 16 != 0)
        return false;
    const cuuint64_t dims[2] = {rec_bytes, n_rows};
    const cuuint64_t strides[1] = {rec_bytes};
    const cuuint32_t elem[2] = {1, 1};
    for (int k = 0; k < 2; ++k) {
        const cuuint32_t box[2] = {k == 0 ? 32u : 16u, 1u};
        CUtensorMap* m = reinterpret_cast<CUtensorMap*>(k == 0 ? out.box32 : out.box16);
        const CUresult r = fn(m, CU_TENSOR_MAP_DATA_TYPE_UINT8, 2, const_cast<uint8_t*>(rec), dims, strides, box, elem,
                              CU_TENSOR_MAP_INTERLEAVE_NONE, CU_TENSOR_MAP_SWIZZLE_NONE,
                              CU_TENSOR_MAP_L2_PROMOTION_L2_128B, CU_TENSOR_MAP_FLOAT_OOB_FILL_NONE);
        if (r != CUDA_SUCCESS) return false;
    }
    out.n_rows = (uint32_t)n_rows;
    out.ok = true;
    return true;
}

void launch_b_hist_part(const BDev& d, const LaneTile* tiles, uint32_t n_tiles, const uint32_t* ridx,
                        const GradRef& gr, const uint8_t* bins8, uint32_t s8, const uint16_t* bins16, uint32_t s16,
                        void* part, int variant, const RecordMaps* maps, cudaStream_t st) {
    if (n_tiles == 0) return;
    init_kernel_attributes();
    int v = variant >= 0 && variant < LANE_VARIANTS ? variant : 0;
    if (v == 3 && !(maps && maps->ok)) v = 0;  // no tensor maps: the cp.async form
    const unsigned g = sm_count() * lane_blocks_per_sm(gr.mode, v), th = lane_threads(gr.mode, v);
    const size_t smem = lane_smem_bytes(gr.mode, v);
    if (v == 3) {
        const uint32_t n_rows = maps->n_rows;
        const CUtensorMap& m32 = *reinterpret_cast<const CUtensorMap*>(maps->box32);
        const CUtensorMap& m16 = *reinterpret_cast<const CUtensorMap*>(maps->box16);
        void* targs[] = {(void*)&d,  (void*)&tiles, (void*)&n_tiles, (void*)&ridx, (void*)&gr,
                         (void*)&n_rows, (void*)&part, (void*)&m32, (void*)&m16};
        launch_kv(lane_kernel_of(gr.mode, v), dim3(g), dim3(th), targs, smem, st);  // errors: next check
        return;
    }
    void* args[] = {(void*)&d,    (void*)&tiles, (void*)&n_tiles, (void*)&ridx,   (void*)&gr,
                    (void*)&bins8, (void*)&s8,   (void*)&bins16,  (void*)&s16,    (void*)&part};
    launch_kv(lane_kernel_of(gr.mode, v), dim3(g), dim3(th), args, smem, st);  // errors: next check
}

// The subtraction trick (pool.rs:414-432) for one global bin of node e:
// larger = parent - smaller. The parent histogram lives in slot left_pnode,
// which becomes the left child's; the right child's is right_pnode. root:
// no parent, the sum goes to right_pnode.
template <typename HB>
__device__ __forceinline__ void merge_store(HB* __restrict__ hist, uint64_t slot_bins, const BExp& e, uint32_t gb,
                                            HB sm, int root) {
    if (root) {
        hist[(size_t)e.right_pnode * slot_bins + gb] = sm;
        return;
    }
    HB* L = hist + (size_t)e.left_pnode * slot_bins + gb;
    HB* R = hist + (size_t)e.right_pnode * slot_bins + gb;
    const HB p = *L;
    const HB lg = hb_make<HB>((long long)p.g - sm.g, (long long)p.h - sm.h);
    if (e.lc <= e.rc) {  // left child is the smaller (grower.rs:398-402)
        *L = sm;
        *R = lg;
    } else {
        *L = lg;
        *R = sm;
    }
}

// Lane-tile bins: one thread per (node, partial entry); ent[r] maps entry r
// of a node (tiles in order, column-major inside a tile) to its global bin
// (0xFFFFFFFF: no bin) and (tile << 16 | offset in the tile's partial
// record). Consecutive threads read consecutive partial entries and touch
// consecutive bins of the node histograms. Each thread handles MERGE_ILP
// entries at once and loads four segments' partials at a time, so that the
// dependent loads overlap (1 entry measured faster than 2 or 4: more
// threads in flight).
constexpr uint32_t MERGE_ILP = 1;

template <int MODE, typename HB>
__global__ void __launch_bounds__(256, 4)
k_b_merge(BDev d, HB* __restrict__ hist, uint64_t slot_bins, const void* __restrict__ part, uint32_t n_tiles,
          const uint2* __restrict__ ent, uint32_t n_ent, int root) {
    BST_PDL_ENTER();
    using E = typename PartEntry<MODE>::T;
    const E* P = reinterpret_cast<const E*>(part);
    const uint32_t n_exp = d.state->n_exp, n_seg = d.state->hist_chunks;
    const uint64_t n = (uint64_t)n_exp * n_ent;
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    const size_t rec = (size_t)n_tiles * LANE_PART_STRIDE;
    for (uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i0 < n; i0 += stride * MERGE_ILP) {
        uint2 m[MERGE_ILP];
        uint32_t j[MERGE_ILP], c0[MERGE_ILP], c1[MERGE_ILP];
        bool ok[MERGE_ILP];
#pragma unroll
        for (uint32_t u = 0; u < MERGE_ILP; ++u) {
            const uint64_t i = i0 + u * stride;
            ok[u] = i < n;
            j[u] = ok[u] ? (uint32_t)(i / n_ent) : 0u;
            m[u] = ok[u] ? ent[(uint32_t)(i % n_ent)] : make_uint2(0xFFFFFFFFu, 0u);
            c0[u] = d.exp[j[u]].hist_off;
            c1[u] = j[u] + 1 < n_exp ? d.exp[j[u] + 1].hist_off : n_seg;
            ok[u] = ok[u] && m[u].x != 0xFFFFFFFFu;
        }
        long long g[MERGE_ILP], h[MERGE_ILP];
        HB par[MERGE_ILP];
#pragma unroll
        for (uint32_t u = 0; u < MERGE_ILP; ++u) {
            g[u] = 0;
            h[u] = 0;
            par[u].g = par[u].h = 0;
            if (!ok[u]) continue;
            if (!root) par[u] = hist[(size_t)d.exp[j[u]].left_pnode * slot_bins + m[u].x];
            const E* p = P + (size_t)(m[u].y >> 16) * LANE_PART_STRIDE + (m[u].y & 0xFFFFu);
            uint32_t c = c0[u];
            for (; c + 4 <= c1[u]; c += 4) {  // four segments' loads in flight
                const E v0 = p[(size_t)c * rec], v1 = p[(size_t)(c + 1) * rec];
                const E v2 = p[(size_t)(c + 2) * rec], v3 = p[(size_t)(c + 3) * rec];
                g[u] += (long long)v0.x + (long long)v1.x + (long long)v2.x + (long long)v3.x;
                h[u] += (long long)v0.y + (long long)v1.y + (long long)v2.y + (long long)v3.y;
            }
            for (; c < c1[u]; ++c) {
                const E v = p[(size_t)c * rec];
                g[u] += v.x;
                h[u] += v.y;
            }
        }
#pragma unroll
        for (uint32_t u = 0; u < MERGE_ILP; ++u) {
            if (!ok[u]) continue;
            const BExp& e = d.exp[j[u]];
            const HB sm = hb_make<HB>(g[u], h[u]);
            if (root) {
                hist[(size_t)e.right_pnode * slot_bins + m[u].x] = sm;
                continue;
            }
            const HB lg = hb_make<HB>((long long)par[u].g - g[u], (long long)par[u].h - h[u]);
            const bool left_small = e.lc <= e.rc;  // grower.rs:398-402
            hist[(size_t)e.left_pnode * slot_bins + m[u].x] = left_small ? sm : lg;
            hist[(size_t)e.right_pnode * slot_bins + m[u].x] = left_small ? lg : sm;
        }
    }
}

// The same merge for levels with few expanding nodes (many row segments
// each): a block takes MW_E consecutive entries of one node and its MW_G
// warps sum every MW_G-th segment, then warp 0 adds the MW_G partial sums
// (exact integers, so the result equals k_b_merge's) and stores as
// k_b_merge does. Per-thread chains of segments / MW_G dependent loads
// instead of segments.
constexpr uint32_t MW_E = 32, MW_G = 8;

template <int MODE, typename HB>
__global__ void __launch_bounds__(MW_E * MW_G)
k_b_merge_wide(BDev d, HB* __restrict__ hist, uint64_t slot_bins, const void* __restrict__ part, uint32_t n_tiles,
               const uint2* __restrict__ ent, uint32_t n_ent, int root) {
    BST_PDL_ENTER();
    using E = typename PartEntry<MODE>::T;
    __shared__ long long s_g[MW_G][MW_E], s_h[MW_G][MW_E];
    const E* P = reinterpret_cast<const E*>(part);
    const uint32_t n_exp = d.state->n_exp, n_seg = d.state->hist_chunks;
    const uint32_t tiles = (n_ent + MW_E - 1) / MW_E;
    const uint64_t items = (uint64_t)n_exp * tiles;
    const size_t rec = (size_t)n_tiles * LANE_PART_STRIDE;
    const uint32_t el = threadIdx.x % MW_E, grp = threadIdx.x / MW_E;
    for (uint64_t it = blockIdx.x; it < items; it += gridDim.x) {
        const uint32_t j = (uint32_t)(it / tiles), r = (uint32_t)(it % tiles) * MW_E + el;
        const uint2 m = r < n_ent ? ent[r] : make_uint2(0xFFFFFFFFu, 0u);
        const bool ok = m.x != 0xFFFFFFFFu;
        const uint32_t c0 = d.exp[j].hist_off, c1 = j + 1 < n_exp ? d.exp[j + 1].hist_off : n_seg;
        long long g = 0, h = 0;
        if (ok) {
            const E* p = P + (size_t)(m.y >> 16) * LANE_PART_STRIDE + (m.y & 0xFFFFu);
            uint32_t c = c0 + grp;
            for (; c + 3 * MW_G < c1; c += 4 * MW_G) {  // four segments' loads in flight
                const E v0 = p[(size_t)c * rec], v1 = p[(size_t)(c + MW_G) * rec];
                const E v2 = p[(size_t)(c + 2 * MW_G) * rec], v3 = p[(size_t)(c + 3 * MW_G) * rec];
                g += (long long)v0.x + (long long)v1.x + (long long)v2.x + (long long)v3.x;
                h += (long long)v0.y + (long long)v1.y + (long long)v2.y + (long long)v3.y;
            }
            for (; c < c1; c += MW_G) {
                const E v = p[(size_t)c * rec];
                g += v.x;
                h += v.y;
            }
        }
        s_g[grp][el] = g;
        s_h[grp][el] = h;
        __syncthreads();
        if (grp == 0 && ok) {
#pragma unroll
            for (uint32_t q = 1; q < MW_G; ++q) {
                g += s_g[q][el];
                h += s_h[q][el];
            }
            const BExp& e = d.exp[j];
            const HB sm = hb_make<HB>(g, h);
            if (root) {
                hist[(size_t)e.right_pnode * slot_bins + m.x] = sm;
            } else {
                const HB par = hist[(size_t)e.left_pnode * slot_bins + m.x];
                const HB lg = hb_make<HB>((long long)par.g - g, (long long)par.h - h);
                const bool left_small = e.lc <= e.rc;  // grower.rs:398-402
                hist[(size_t)e.left_pnode * slot_bins + m.x] = left_small ? sm : lg;
                hist[(size_t)e.right_pnode * slot_bins + m.x] = left_small ? lg : sm;
            }
        }
        __syncthreads();  // s_g / s_h are reused by the next item
    }
}

// Bins of general tiles (built atomically into the right slot).
template <typename HB>
__global__ void k_b_merge_rest(BDev d, HB* __restrict__ hist, uint64_t slot_bins, uint32_t total_bins,
                               const uint32_t* __restrict__ bin_map, int root) {
    BST_PDL_ENTER();
    const uint32_t n_exp = d.state->n_exp;
    const uint64_t n = (uint64_t)n_exp * total_bins;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t j = (uint32_t)(i / total_bins), gb = (uint32_t)(i % total_bins);
        if (bin_map[gb] != 0xFFFFFFFFu) continue;
        const BExp e = d.exp[j];
        merge_store(hist, slot_bins, e, gb, hist[(size_t)e.right_pnode * slot_bins + gb], root);
    }
}

template <typename HB>
static void launch_b_merge_t(const BDev& d, HB* hist, uint64_t slot_bins, uint32_t total_bins, const void* part,
                             uint32_t n_lane_tiles, const uint2* ent, uint32_t n_ent, const uint32_t* bin_map,
                             bool has_rest, int root, int mode, cudaStream_t st, int wide) {
    const unsigned grid = sm_count() * 8u;
    if (n_lane_tiles) {
        if (wide) {
            if (mode == GRAD_F32)
                launch_k(k_b_merge_wide<GRAD_F32, HB>, grid, MW_E * MW_G, 0, st, d, hist, slot_bins, part, n_lane_tiles,
                                                                          ent, n_ent, root);
            else
                launch_k(k_b_merge_wide<GRAD_Q8, HB>, grid, MW_E * MW_G, 0, st, d, hist, slot_bins, part, n_lane_tiles,
                                                                         ent, n_ent, root);
        } else if (mode == GRAD_F32) {
            launch_k(k_b_merge<GRAD_F32, HB>, grid, 256, 0, st, d, hist, slot_bins, part, n_lane_tiles, ent, n_ent, root);
        } else {
            launch_k(k_b_merge<GRAD_Q8, HB>, grid, 256, 0, st, d, hist, slot_bins, part, n_lane_tiles, ent, n_ent, root);
        }
    }
    if (has_rest) launch_k(k_b_merge_rest<HB>, grid, 256, 0, st, d, hist, slot_bins, total_bins, bin_map, root);
}

void launch_b_merge(const BDev& d, void* hist, uint64_t slot_bins, uint32_t total_bins, const void* part,
                    uint32_t n_lane_tiles, const uint2* ent, uint32_t n_ent, const uint32_t* bin_map, bool has_rest,
                    int root, int mode, cudaStream_t st, int hist32, int wide) {
    if (hist32)
        launch_b_merge_t(d, static_cast<HBin32*>(hist), slot_bins, total_bins, part, n_lane_tiles, ent, n_ent, bin_map,
                         has_rest, root, mode, st, wide);
    else
        launch_b_merge_t(d, static_cast<HBin*>(hist), slot_bins, total_bins, part, n_lane_tiles, ent, n_ent, bin_map,
                         has_rest, root, mode, st, wide);
}


template <int MODE>
__global__ void __launch_bounds__(HIST_THREADS)
k_hist_build(const HistChunk* __restrict__ chunks, const HistTile* __restrict__ tiles,
             const uint32_t* __restrict__ ridx, GradRef gr, const uint8_t* __restrict__ bins8, uint32_t s8,
             const uint16_t* __restrict__ bins16, uint32_t s16, HBin* __restrict__ hist,
             uint64_t slot_bins, uint32_t n_tiles, uint32_t S) {
    BST_PDL_ENTER();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint32_t* sm = reinterpret_cast<uint32_t*>(smem_raw);
    __shared__ HistTile tile;
    // tiles vary fastest so the blocks of one row chunk run together and
    // share its gradients and row ids in L2
    const HistChunk chunk = chunks[blockIdx.x / n_tiles];
    if (threadIdx.x == 0) tile = tiles[blockIdx.x % n_tiles];
    __syncthreads();
    const GradLoad<MODE> load(gr);
    hist_item<MODE>(chunk, tile, sm, S, ridx, load, bins8, s8, bins16, s16, hist, slot_bins);
}

void launch_hist_build(const HistChunk* chunks, uint32_t n_chunks, const HistTile* tiles,
                       uint32_t n_tiles, uint32_t max_smem_bins, const uint32_t* ridx,
                       const GradRef& gr, const uint8_t* bins8, uint32_t s8,
                       const uint16_t* bins16, uint32_t s16, HBin* hist, uint64_t slot_bins,
                       cudaStream_t st) {
    if (n_chunks == 0 || n_tiles == 0) return;
    const uint32_t S = (max_smem_bins + 3u) & ~3u;
    const size_t smem = (size_t)S * acc_words(gr.mode) * sizeof(uint32_t);
    init_kernel_attributes();
    const uint64_t blocks = (uint64_t)n_tiles * n_chunks;
    if (blocks > 0x7FFFFFFFull) return;
    const unsigned g = (unsigned)blocks;
    if (gr.mode == GRAD_Q16)
        launch_k(k_hist_build<GRAD_Q16>, g, HIST_THREADS, smem, st, chunks, tiles, ridx, gr, bins8, s8, bins16, s16, hist,
                                                               slot_bins, n_tiles, S);
    else if (gr.mode == GRAD_Q8)
        launch_k(k_hist_build<GRAD_Q8>, g, HIST_THREADS, smem, st, chunks, tiles, ridx, gr, bins8, s8, bins16, s16, hist,
                                                              slot_bins, n_tiles, S);
    else
        launch_k(k_hist_build<GRAD_F32>, g, HIST_THREADS, smem, st, chunks, tiles, ridx, gr, bins8, s8, bins16, s16,
                                                               hist, slot_bins, n_tiles, S);
}

template <int MODE>
__global__ void k_node_sums(const HistChunk* __restrict__ chunks, const uint32_t* __restrict__ ridx, GradRef gr,
                            long long* __restrict__ sums) {
    BST_PDL_ENTER();
    const HistChunk c = chunks[blockIdx.x];
    const GradLoad<MODE> load(gr);
    long long ag = 0, ah = 0;
    for (uint32_t i = threadIdx.x; i < c.count; i += blockDim.x) {
        const uint32_t p = c.begin + i;
        const uint32_t row = (c.flags & 1u) ? p : ridx[p];
        long long qg, qh;
        load(row, qg, qh);
        ag += qg;
        ah += qh;
    }
    for (int o = 16; o > 0; o >>= 1) {
        ag += __shfl_xor_sync(FULL, ag, o);
        ah += __shfl_xor_sync(FULL, ah, o);
    }
    if ((threadIdx.x & 31) == 0) {
        atomicAdd(reinterpret_cast<unsigned long long*>(&sums[2 * c.slot]), (unsigned long long)ag);
        atomicAdd(reinterpret_cast<unsigned long long*>(&sums[2 * c.slot + 1]), (unsigned long long)ah);
    }
}

void launch_node_sums(const HistChunk* chunks, uint32_t n_chunks, const uint32_t* ridx, const GradRef& gr,
                      long long* sums, cudaStream_t st) {
    if (n_chunks == 0) return;
    if (gr.mode == GRAD_Q16)
        launch_k(k_node_sums<GRAD_Q16>, n_chunks, 256, 0, st, chunks, ridx, gr, sums);
    else if (gr.mode == GRAD_Q8)
        launch_k(k_node_sums<GRAD_Q8>, n_chunks, 256, 0, st, chunks, ridx, gr, sums);
    else
        launch_k(k_node_sums<GRAD_F32>, n_chunks, 256, 0, st, chunks, ridx, gr, sums);
}

// ============================================================================
// Quantised gradients (int16 / int8 training mode; no counterpart in the
// reference). Philox4x32-10 as published by Salmon, Moraes, Dror and Shaw,
// "Parallel Random Numbers: As Easy as 1, 2, 3" (SC 2011), gives each
// (row, output, round) two uniform words; q = floor(v * Q / max|v| + u).
// ============================================================================

__device__ __forceinline__ uint4 philox4x32_10(uint4 c, uint2 k) {
    const uint32_t M0 = 0xD2511F53u, M1 = 0xCD9E8D57u, W0 = 0x9E3779B9u, W1 = 0xBB67AE85u;
#pragma unroll
    for (int r = 0; r < 10; ++r) {
        const uint32_t hi0 = __umulhi(M0, c.x), lo0 = M0 * c.x;
        const uint32_t hi1 = __umulhi(M1, c.z), lo1 = M1 * c.z;
        c = make_uint4(hi1 ^ c.y ^ k.x, lo1, hi0 ^ c.w ^ k.y, lo0);
        k.x += W0;
        k.y += W1;
    }
    return c;
}

__device__ __forceinline__ int32_t stochastic_round(float v, double inv, uint32_t r, int32_t Q) {
    const double u = (double)r * 0x1p-32;
    double x = (double)v * inv;
    x = x + u;
    double f = floor(x);
    if (!(f >= (double)-Q)) f = (double)-Q;
    if (f > (double)Q) f = (double)Q;
    return (int32_t)f;
}

template <int MODE>
__global__ void k_quantize(const float2* __restrict__ gh, uint64_t n, uint32_t G, const unsigned* __restrict__ maxabs,
                           uint2 key, uint32_t round, uint32_t out0, void* __restrict__ gq,
                           double* __restrict__ qscales, double* __restrict__ fscales) {
    BST_PDL_ENTER();
    constexpr int32_t Q = MODE == GRAD_Q8 ? 127 : 32767;
    const uint64_t i0 = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i0 < 2ull * G) {
        const float m = __uint_as_float(maxabs[i0]);
        const uint32_t o = (uint32_t)(i0 >> 1), which = (uint32_t)(i0 & 1);
        qscales[4 * o + which] = m > 0.0f ? (double)Q / (double)m : 0.0;
        qscales[4 * o + 2 + which] = m > 0.0f ? (double)m / (double)Q : 0.0;
        if (fscales) write_fixed_scale(maxabs, (uint32_t)i0, n, fscales);  // the exact leaf sums' scales
    }
    const uint64_t total = n * G;
    for (uint64_t i = i0; i < total; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint32_t o = (uint32_t)(i / n), row = (uint32_t)(i % n);
        const float mg = __uint_as_float(maxabs[2 * o]), mh = __uint_as_float(maxabs[2 * o + 1]);
        const double ig = mg > 0.0f ? (double)Q / (double)mg : 0.0;
        const double ih = mh > 0.0f ? (double)Q / (double)mh : 0.0;
        const uint4 r = philox4x32_10(make_uint4(row, out0 + o, round, QUANT_STREAM), key);
        const float2 v = gh[i];
        const int32_t qg = stochastic_round(v.x, ig, r.x, Q), qh = stochastic_round(v.y, ih, r.y, Q);
        if constexpr (MODE == GRAD_Q8)
            static_cast<char2*>(gq)[i] = make_char2((signed char)qg, (signed char)qh);
        else
            static_cast<short2*>(gq)[i] = make_short2((short)qg, (short)qh);
    }
}

void launch_quantize(int mode, uint32_t G, const float2* gh, uint64_t n, const unsigned* maxabs, uint64_t seed,
                     uint32_t round, uint32_t out0, void* gq, double* qscales, cudaStream_t st,
                     double* fscales) {
    if (G == 0) return;
    const uint64_t total = n * G;
    uint64_t blocks = (total + 255) / 256;
    if (blocks > (uint64_t)sm_count() * 16) blocks = (uint64_t)sm_count() * 16;
    if (blocks < (2ull * G + 255) / 256) blocks = (2ull * G + 255) / 256;  // a thread per scale
    const uint2 key = make_uint2((uint32_t)seed, (uint32_t)(seed >> 32));
    if (mode == GRAD_Q8)
        launch_k(k_quantize<GRAD_Q8>, (unsigned)blocks, 256, 0, st, gh, n, G, maxabs, key, round, out0, gq, qscales,
                 fscales);
    else
        launch_k(k_quantize<GRAD_Q16>, (unsigned)blocks, 256, 0, st, gh, n, G, maxabs, key, round, out0, gq, qscales,
                 fscales);
}

// ============================================================================
// K6: split scan (GreedySplitter, training/gbdt/split/find.rs:113-644)
// One warp per (node, column); exact int64 prefix sums, f64 gain cast to f32,
// ties resolved by the reference's scan order.
// ============================================================================

namespace {

struct Best {
    float gain;
    uint32_t order;
    uint32_t bin;
    uint32_t flags;
};

__device__ __forceinline__ bool better(float g, uint32_t o, float bg, uint32_t bo) {
    // candidates: larger gain wins, equal gain -> earlier scan position wins
    return g > bg || (g == bg && o < bo);
}

__device__ __forceinline__ Best warp_best(Best b) {
    for (int off = 16; off > 0; off >>= 1) {
        Best o;
        o.gain = __shfl_xor_sync(FULL, b.gain, off);
        o.order = __shfl_xor_sync(FULL, b.order, off);
        o.bin = __shfl_xor_sync(FULL, b.bin, off);
        o.flags = __shfl_xor_sync(FULL, b.flags, off);
        if (better(o.gain, o.order, b.gain, b.order)) b = o;
    }
    return b;
}

__device__ __forceinline__ long long warp_incl_scan(long long v, int lane) {
    for (int d = 1; d < 32; d <<= 1) {
        long long t = shfl_up_ll(v, d);
        if (lane >= d) v += t;
    }
    return v;
}

// 32-bit form for the HBin32 histograms (every prefix of a node's bins is
// bounded by its exact total, which fits 31 bits there): one shuffle a step.
__device__ __forceinline__ int warp_incl_scan(int v, int lane) {
    for (int d = 1; d < 32; d <<= 1) {
        const int t = __shfl_up_sync(FULL, v, d);
        if (lane >= d) v += t;
    }
    return v;
}

__device__ __forceinline__ long long warp_sum(long long v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}
__device__ __forceinline__ int warp_sum(int v) {
    for (int o = 16; o > 0; o >>= 1) v += __shfl_xor_sync(FULL, v, o);
    return v;
}


struct GainCtx {
    double lambda, offset, mcw;
    uint32_t msl;
    __device__ float gain(double gl, double hl, double gr, double hr) const {
        const double sl = gl * gl / (hl + lambda);
        const double sr = gr * gr / (hr + lambda);
        return __double2float_rn(0.5 * (sl + sr) - offset);
    }
    __device__ bool valid(double hl, double hr, uint32_t cl, uint32_t cr) const {
        return hl >= mcw && hr >= mcw && cl >= msl && cr >= msl;
    }
};

__device__ __forceinline__ uint32_t sat_sub(uint32_t a, uint32_t b) { return a > b ? a - b : 0u; }

constexpr int SCAN_WARPS = 8;
constexpr int SORT_N = 256;  // categorical columns with <= 256 bins

}  // namespace

// One warp: best split of column `col` of node `node` (the node's histogram
// lives in slot nd.slot); writes cand[node * n_cols + col] and, for column 0,
// the node totals, and returns the candidate's gain (-inf: none) to every
// lane. key / cat: this warp's SORT_N-entry shared scratch. cmask (or null):
// the node's column mask (column sampling); a masked column has no
// candidate.
template <typename HB>
__device__ float scan_item(const ScanNode nd, uint32_t node, uint32_t col, const ScanColumn* __restrict__ cols,
                          uint32_t n_cols, const HB* __restrict__ hist, uint64_t slot_bins,
                          const double* __restrict__ scale, const GainParamsDev& gp, ColCand* __restrict__ cand,
                          long long* __restrict__ node_tot, double* key, uint32_t* cat,
                          const uint8_t* __restrict__ cmask) {
    const int lane = threadIdx.x & 31;
    const ScanColumn cm = cols[col];
    const HB* h = hist + (size_t)nd.slot * slot_bins + cm.hist_off;
    const double ig = scale[2], ih = scale[3];
    const uint32_t nb = cm.n_bins;
    const uint32_t pc = nd.count;

    // node totals (every column's bins sum to the same exact total)
    using TAcc = decltype(HB{}.g);  // int for HBin32: 32-bit sums
    TAcc tg_ = 0, th_ = 0;
    for (uint32_t b = lane; b < nb; b += 32) {
        tg_ += h[b].g;
        th_ += h[b].h;
    }
    long long tg = warp_sum(tg_), th = warp_sum(th_);
    if (nd.flags & 1u) {
        tg = nd.pg;
        th = nd.ph;
    }
    if (col == 0 && lane == 0) {
        node_tot[2 * node] = tg;
        node_tot[2 * node + 1] = th;
    }
    ColCand* out = cand + (size_t)node * n_cols + col;
    if (cmask && !cmask[col]) {  // not among the node's sampled columns
        if (lane == 0) {
            out->gain = -INFINITY;
            out->order = 0xFFFFFFFFu;
            out->bin = 0;
            out->flags = 0;
            out->cats[0] = out->cats[1] = out->cats[2] = out->cats[3] = 0ull;
        }
        return -INFINITY;
    }
    const double pg = (double)tg * ig, ph = (double)th * ih;
    GainCtx ctx;
    ctx.lambda = gp.lambda;
    ctx.offset = 0.5 * (pg * pg / (ph + gp.lambda)) + gp.min_gain;
    ctx.mcw = gp.min_child_weight;
    ctx.msl = gp.min_samples_leaf;

    Best best{-INFINITY, 0xFFFFFFFFu, 0u, 0u};

    if (!cm.is_cat) {
        if (nb >= 2) {
            // find.rs:286-407: forward scan (missing right), backward scan
            // (missing left) when the column has a NaN bin (the last bin).
            const bool hm = cm.has_missing != 0;
            const long long pm_g = tg - h[nb - 1].g, pm_h = th - h[nb - 1].h;  // P[nb-2]
            using Acc = decltype(HB{}.g);  // int for HBin32: 32-bit prefix scans
            Acc carry_g = 0, carry_h = 0;
            for (uint32_t base = 0; base < nb; base += 32) {
                const uint32_t b = base + lane;
                Acc vg = 0, vh = 0;
                if (b < nb) {
                    vg = h[b].g;
                    vh = h[b].h;
                }
                const Acc Pg_ = warp_incl_scan(vg, lane) + carry_g;
                const Acc Ph_ = warp_incl_scan(vh, lane) + carry_h;
                carry_g = __shfl_sync(FULL, Pg_, 31);
                carry_h = __shfl_sync(FULL, Ph_, 31);
                const long long Pg = Pg_, Ph = Ph_;
                if (b + 1 < nb) {  // forward candidate: bins <= b go left
                    const double lg = (double)Pg * ig, lh = (double)Ph * ih;
                    const double rg = (double)(tg - Pg) * ig, rh = (double)(th - Ph) * ih;
                    const uint32_t lc = b + 1, rc = sat_sub(pc, lc);
                    if (ctx.valid(lh, rh, lc, rc)) {
                        const float g = ctx.gain(lg, lh, rg, rh);
                        if (better(g, b, best.gain, best.order)) best = Best{g, b, b, 0u};
                    }
                }
                if (hm && b + 2 < nb) {  // backward candidate: bins b+1..nb-2 go right
                    const long long Rg = pm_g - Pg, Rh = pm_h - Ph;
                    const double rg = (double)Rg * ig, rh = (double)Rh * ih;
                    const double lg = (double)(tg - Rg) * ig, lh = (double)(th - Rh) * ih;
                    const uint32_t rc = nb - 2 - b, lc = sat_sub(pc, rc);
                    if (ctx.valid(lh, rh, lc, rc)) {
                        const float g = ctx.gain(lg, lh, rg, rh);
                        const uint32_t ord = 2 * nb - 3 - b;
                        if (better(g, ord, best.gain, best.order)) best = Best{g, ord, b, 1u};
                    }
                }
            }
        }
        best = warp_best(best);
        if (lane == 0) {
            out->gain = best.gain;
            out->order = best.order;
            out->bin = best.bin;
            out->flags = best.flags;
            out->cats[0] = out->cats[1] = out->cats[2] = out->cats[3] = 0ull;
        }
        return best.gain;
    }

    // categorical (find.rs:426-573)
    unsigned long long cats[4] = {0ull, 0ull, 0ull, 0ull};
    if (nb >= 2 && nb <= gp.max_onehot_cats) {
        for (uint32_t c = lane; c < nb; c += 32) {  // one category left (find.rs:472)
            const double lg = (double)h[c].g * ig, lh = (double)h[c].h * ih;
            const double rg = (double)(tg - h[c].g) * ig, rh = (double)(th - h[c].h) * ih;
            const uint32_t lc = 1, rc = sat_sub(pc, 1);
            if (ctx.valid(lh, rh, lc, rc)) {
                const float g = ctx.gain(lg, lh, rg, rh);
                if (better(g, c, best.gain, best.order)) best = Best{g, c, c, 2u};
            }
        }
        best = warp_best(best);
        if (best.gain > -INFINITY && best.bin < 256) cats[best.bin >> 6] = 1ull << (best.bin & 63);
    } else if (nb > gp.max_onehot_cats && nb <= SORT_N) {
        // sorted partition (find.rs:511-573): categories with hess > 1e-10
        // ordered by -g/(h+1e-6) ascending, ties by category (stable sort)
        uint32_t m = 0;
        for (uint32_t base = 0; base < nb; base += 32) {
            const uint32_t c = base + lane;
            bool ok = false;
            double r = 0.0;
            if (c < nb) {
                const double gg = (double)h[c].g * ig, hh = (double)h[c].h * ih;
                ok = hh > 1e-10;
                r = -gg / (hh + 1e-6);
            }
            const unsigned bal = __ballot_sync(FULL, ok);
            const uint32_t pos = m + __popc(bal & ((1u << lane) - 1u));
            if (ok) {
                key[pos] = r;
                cat[pos] = c;
            }
            m += __popc(bal);
        }
        // bitonic network over the next power of two >= m entries (the
        // (key, category) order is total, so the sorted prefix is the same
        // for any padded size)
        uint32_t sn = 2;
        while (sn < m) sn <<= 1;
        for (uint32_t i = m + lane; i < sn; i += 32) {
            key[i] = INFINITY;
            cat[i] = 0xFFFFFFFFu;
        }
        __syncwarp();
        if (m >= 2) {
            // bitonic sort of (key, cat) over sn entries
            for (uint32_t k = 2; k <= sn; k <<= 1) {
                for (uint32_t j = k >> 1; j > 0; j >>= 1) {
                    for (uint32_t i = lane; i < sn; i += 32) {
                        const uint32_t ixj = i ^ j;
                        if (ixj > i) {
                            const bool up = (i & k) == 0;
                            const double a = key[i], b = key[ixj];
                            const uint32_t ca = cat[i], cb = cat[ixj];
                            const bool a_gt_b = a > b || (a == b && ca > cb);
                            if (a_gt_b == up) {
                                key[i] = b;
                                key[ixj] = a;
                                cat[i] = cb;
                                cat[ixj] = ca;
                            }
                        }
                    }
                    __syncwarp();
                }
            }
            using Acc = decltype(HB{}.g);
            Acc carry_g = 0, carry_h = 0;
            for (uint32_t base = 0; base + 1 < m; base += 32) {
                const uint32_t i = base + lane;
                Acc vg = 0, vh = 0;
                if (i + 1 < m) {
                    const uint32_t c = cat[i];
                    vg = h[c].g;
                    vh = h[c].h;
                }
                const Acc Pg_ = warp_incl_scan(vg, lane) + carry_g;
                const Acc Ph_ = warp_incl_scan(vh, lane) + carry_h;
                carry_g = __shfl_sync(FULL, Pg_, 31);
                carry_h = __shfl_sync(FULL, Ph_, 31);
                const long long Pg = Pg_, Ph = Ph_;
                if (i + 1 < m) {
                    const double lg = (double)Pg * ig, lh = (double)Ph * ih;
                    const double rg = (double)(tg - Pg) * ig, rh = (double)(th - Ph) * ih;
                    const uint32_t lc = i + 1, rc = sat_sub(pc, lc);
                    if (ctx.valid(lh, rh, lc, rc)) {
                        const float g = ctx.gain(lg, lh, rg, rh);
                        if (better(g, i, best.gain, best.order)) best = Best{g, i, i, 2u};
                    }
                }
            }
            best = warp_best(best);
            if (best.gain > -INFINITY) {
                unsigned long long part[4] = {0ull, 0ull, 0ull, 0ull};
                for (uint32_t i = lane; i <= best.order && i < m; i += 32) {
                    const uint32_t c = cat[i];
                    if (c < 256) part[c >> 6] |= 1ull << (c & 63);
                }
                for (int q = 0; q < 4; ++q) {
                    unsigned long long v = part[q];
                    for (int o = 16; o > 0; o >>= 1) v |= __shfl_xor_sync(FULL, v, o);
                    cats[q] = v;
                }
            }
        }
    }
    if (lane == 0) {
        out->gain = best.gain;
        out->order = best.order;
        out->bin = best.bin;
        out->flags = best.gain > -INFINITY ? best.flags : 0u;
        for (int q = 0; q < 4; ++q) out->cats[q] = cats[q];
    }
    return best.gain;
}

template <typename HB>
__global__ void __launch_bounds__(SCAN_WARPS * 32)
k_split_scan(const ScanNode* __restrict__ nodes, const ScanColumn* __restrict__ cols,
             uint32_t n_cols, const HB* __restrict__ hist, uint64_t slot_bins,
             const double* __restrict__ scale, GainParamsDev gp, ColCand* __restrict__ cand,
             long long* __restrict__ node_tot, uint32_t col_blocks, const uint8_t* __restrict__ colmask) {
    BST_PDL_ENTER();
    __shared__ double s_key[SCAN_WARPS][SORT_N];
    __shared__ uint32_t s_cat[SCAN_WARPS][SORT_N];
    const int warp = threadIdx.x >> 5;
    const uint32_t col = (blockIdx.x % col_blocks) * SCAN_WARPS + warp;
    const uint32_t node = blockIdx.x / col_blocks;
    if (col >= n_cols) return;
    const ScanNode nd = nodes[node];
    scan_item(nd, node, col, cols, n_cols, hist, slot_bins, scale, gp, cand, node_tot, s_key[warp], s_cat[warp],
              colmask ? colmask + (size_t)nd.pad * n_cols : nullptr);
}

void launch_split_scan(const ScanNode* nodes, uint32_t n_nodes, const ScanColumn* cols,
                       uint32_t n_cols, const void* hist, uint64_t slot_bins,
                       const double* scale, GainParamsDev gp, ColCand* cand,
                       long long* node_tot, cudaStream_t st, int hist32, const uint8_t* colmask) {
    if (n_nodes == 0 || n_cols == 0) return;
    const uint32_t per = (n_cols + SCAN_WARPS - 1) / SCAN_WARPS;
    const uint64_t blocks = (uint64_t)per * n_nodes;
    if (blocks > 0x7FFFFFFFull) return;
    if (hist32)
        launch_k(k_split_scan<HBin32>, (unsigned)blocks, SCAN_WARPS * 32, 0, st, 
            nodes, cols, n_cols, static_cast<const HBin32*>(hist), slot_bins, scale, gp, cand, node_tot, per, colmask);
    else
        launch_k(k_split_scan<HBin>, (unsigned)blocks, SCAN_WARPS * 32, 0, st, 
            nodes, cols, n_cols, static_cast<const HBin*>(hist), slot_bins, scale, gp, cand, node_tot, per, colmask);
}

// Across columns (find.rs:180-212 sequential; :219-270 rayon reduce).
__global__ void k_split_reduce(const ColCand* __restrict__ cand, const long long* __restrict__ node_tot,
                               uint32_t n_cols, int last_wins, NodeSplit* __restrict__ out) {
    BST_PDL_ENTER();
    const uint32_t node = blockIdx.x;
    const int lane = threadIdx.x;
    float bg = -INFINITY;
    uint32_t bc = 0xFFFFFFFFu;
    const ColCand* c = cand + (size_t)node * n_cols;
    for (uint32_t i = lane; i < n_cols; i += 32) {
        const float g = c[i].gain;
        if (!(g > -INFINITY)) continue;
        if (bc == 0xFFFFFFFFu || g > bg || (last_wins && g == bg)) {
            bg = g;
            bc = i;
        }
    }
    for (int off = 16; off > 0; off >>= 1) {
        const float og = __shfl_xor_sync(FULL, bg, off);
        const uint32_t oc = __shfl_xor_sync(FULL, bc, off);
        bool take;
        if (oc == 0xFFFFFFFFu)
            take = false;
        else if (bc == 0xFFFFFFFFu)
            take = true;
        else if (og != bg)
            take = og > bg;
        else
            take = last_wins ? oc > bc : oc < bc;
        if (take) {
            bg = og;
            bc = oc;
        }
    }
    if (lane == 0) {
        NodeSplit s;
        s.tot_g = node_tot[2 * node];
        s.tot_h = node_tot[2 * node + 1];
        if (bc == 0xFFFFFFFFu) {
            s.gain = -INFINITY;
            s.col = 0;
            s.bin = 0;
            s.flags = 0;
            s.cats[0] = s.cats[1] = s.cats[2] = s.cats[3] = 0ull;
        } else {
            const ColCand& w = c[bc];
            s.gain = w.gain;
            s.col = bc;
            s.bin = w.bin;
            s.flags = (w.flags & 3u) | 4u;
            for (int q = 0; q < 4; ++q) s.cats[q] = w.cats[q];
        }
        out[node] = s;
    }
}

void launch_split_reduce(const ColCand* cand, const long long* node_tot, uint32_t n_nodes,
                         uint32_t n_cols, int last_wins, NodeSplit* out, cudaStream_t st) {
    if (n_nodes == 0) return;
    launch_k(k_split_reduce, n_nodes, 32, 0, st, cand, node_tot, n_cols, last_wins, out);
}

cudaError_t load_split_kernels() {
    cudaFuncAttributes a;
    cudaError_t e = cudaFuncGetAttributes(&a, k_split_scan<HBin>);
    if (e == cudaSuccess) e = cudaFuncGetAttributes(&a, k_split_reduce);
    return e;
}

// ============================================================================
// K7: row partition (RowPartitioner::split, training/gbdt/partition.rs:296-382)
// Left rows fill the node's range from the front, right rows from the back.
// ============================================================================

namespace {

constexpr int PART_THREADS = 256;  // 8 warps
constexpr int PART_PER = 8;        // rows per thread per pass: 2048-row passes

__device__ __forceinline__ bool part_left(const PartWork& w, uint32_t bin) {
    if ((w.flags & 2u) && bin == w.default_bin) return (w.flags & 1u) != 0;
    if (w.flags & 4u) return bin < 256 && ((w.cats[bin >> 6] >> (bin & 63)) & 1ull);
    return bin <= w.thr_bin;
}

// Rows ridx[start, start + len) of one node into tmp: left rows at the left
// cursor cur[0] (growing), right rows below the right cursor cur[1]
// (shrinking). Ranks come from a block-wide scan of ballots, so each
// 2048-row pass takes one atomic per side (same-address atomics from every
// warp serialise in L2). Block-uniform; blockDim.x == PART_THREADS.
// Q: the type of the gradient element carried with each row id (qin at the
// source position, qout at the destination), or char for none.
// fm8 / fm16 (or null): the same bins column-major ([column][n_rows]), so
// that a node's split column is gathered from one contiguous column.
template <typename Q = char>
__device__ void part_rows(const PartWork& w, uint32_t start, uint32_t len, unsigned* cur,
                          const uint32_t* __restrict__ ridx, uint32_t* __restrict__ tmp,
                          const uint8_t* __restrict__ bins8, uint32_t s8, const uint16_t* __restrict__ bins16,
                          uint32_t s16, const Q* __restrict__ qin = nullptr, Q* __restrict__ qout = nullptr,
                          const uint8_t* __restrict__ fm8 = nullptr, const uint16_t* __restrict__ fm16 = nullptr,
                          uint64_t n_rows = 0, const uint8_t* __restrict__ rmask = nullptr,
                          unsigned* __restrict__ scnt = nullptr) {
    constexpr bool CARRY = !std::is_same<Q, char>::value;
    __shared__ uint32_t s_l[PART_PER][PART_THREADS / 32], s_r[PART_PER][PART_THREADS / 32];
    __shared__ uint32_t s_base[2];
    __shared__ uint32_t s_sl[PART_THREADS / 32], s_sr[PART_THREADS / 32];  // sampled rows per side (row sampling)
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const unsigned lt = (1u << lane) - 1u;
    for (uint32_t b0 = 0; b0 < len; b0 += PART_THREADS * PART_PER) {
        uint32_t rows[PART_PER], bins[PART_PER];
        unsigned lm[PART_PER], rm[PART_PER];
        Q qv[CARRY ? PART_PER : 1];
#pragma unroll
        for (int k = 0; k < PART_PER; ++k) {
            const uint32_t i = b0 + k * PART_THREADS + threadIdx.x;
            rows[k] = i < len ? ridx[start + i] : 0u;
            if constexpr (CARRY) {
                if (i < len) qv[k] = qin[start + i];
            }
        }
#pragma unroll
        for (int k = 0; k < PART_PER; ++k) {
            const uint32_t i = b0 + k * PART_THREADS + threadIdx.x;
            bins[k] = 0u;
            if (i < len) {
                if (fm8 || fm16)
                    bins[k] = w.matrix == 0 ? (uint32_t)fm8[(size_t)w.pos * n_rows + rows[k]]
                                            : (uint32_t)fm16[(size_t)w.pos * n_rows + rows[k]];
                else
                    bins[k] = w.matrix == 0 ? (uint32_t)bins8[(size_t)rows[k] * s8 + w.pos]
                                            : (uint32_t)bins16[(size_t)rows[k] * s16 + w.pos];
            }
        }
#pragma unroll
        for (int k = 0; k < PART_PER; ++k) {
            const uint32_t i = b0 + k * PART_THREADS + threadIdx.x;
            const bool ok = i < len;
            const unsigned act = __ballot_sync(FULL, ok);
            lm[k] = __ballot_sync(FULL, ok && part_left(w, bins[k]));
            rm[k] = act & ~lm[k];
            if (lane == 0) {
                s_l[k][warp] = (uint32_t)__popc(lm[k]);
                s_r[k][warp] = (uint32_t)__popc(rm[k]);
            }
        }
        if (rmask) {  // row sampling: the children's sampled rows
            uint32_t sl = 0, sr = 0;
#pragma unroll
            for (int k = 0; k < PART_PER; ++k) {
                const uint32_t i = b0 + k * PART_THREADS + threadIdx.x;
                const unsigned smp = __ballot_sync(FULL, i < len && rmask[rows[k]] != 0);
                sl += (uint32_t)__popc(smp & lm[k]);
                sr += (uint32_t)__popc(smp & rm[k]);
            }
            if (lane == 0) {
                s_sl[warp] = sl;
                s_sr[warp] = sr;
            }
        }
        __syncthreads();
        if (rmask && warp == 1 && lane == 0) {
            uint32_t SL = 0, SR = 0;
            for (int q = 0; q < PART_THREADS / 32; ++q) {
                SL += s_sl[q];
                SR += s_sr[q];
            }
            if (SL) atomicAdd(&scnt[0], SL);
            if (SR) atomicAdd(&scnt[1], SR);
        }
        if (warp == 0) {
            // exclusive scan of the PART_PER x 8 counts in (k, warp) order:
            // lane q holds entries 2q and 2q + 1
            static_assert(PART_PER * (PART_THREADS / 32) == 64, "two counts per lane");
            uint32_t* fl = &s_l[0][0];
            uint32_t* fr = &s_r[0][0];
            const uint32_t l0 = fl[2 * lane], l1 = fl[2 * lane + 1], r0 = fr[2 * lane], r1 = fr[2 * lane + 1];
            uint32_t xl = l0 + l1, xr = r0 + r1;
            for (int o = 1; o < 32; o <<= 1) {
                const uint32_t tl = __shfl_up_sync(FULL, xl, o), tr = __shfl_up_sync(FULL, xr, o);
                if (lane >= o) {
                    xl += tl;
                    xr += tr;
                }
            }
            const uint32_t L = __shfl_sync(FULL, xl, 31), R = __shfl_sync(FULL, xr, 31);
            const uint32_t el = xl - l0 - l1, er = xr - r0 - r1;
            fl[2 * lane] = el;
            fl[2 * lane + 1] = el + l0;
            fr[2 * lane] = er;
            fr[2 * lane + 1] = er + r0;
            if (lane == 0) {
                s_base[0] = L ? atomicAdd(&cur[0], L) : 0u;
                s_base[1] = R ? atomicSub(&cur[1], R) - R : 0u;
            }
        }
        __syncthreads();
        const uint32_t lb = s_base[0], rbs = s_base[1];
#pragma unroll
        for (int k = 0; k < PART_PER; ++k) {
            const unsigned bit = 1u << lane;
            uint32_t dst = 0xFFFFFFFFu;
            if (lm[k] & bit)
                dst = lb + s_l[k][warp] + __popc(lm[k] & lt);
            else if (rm[k] & bit)
                dst = rbs + s_r[k][warp] + __popc(rm[k] & lt);
            if (dst != 0xFFFFFFFFu && BST_IN(dst - w.begin, w.count, CHECK_PART_DST)) {
                tmp[dst] = rows[k];
                if constexpr (CARRY) qout[dst] = qv[k];
            }
        }
        __syncthreads();  // s_l / s_r / s_base are reused by the next pass
    }
}

}  // namespace

template <typename Q>
__global__ void __launch_bounds__(PART_THREADS)
k_partition(const PartWork* __restrict__ works, const PartChunk* __restrict__ chunks,
            const uint32_t* __restrict__ ridx, uint32_t* __restrict__ tmp, unsigned* __restrict__ cursors,
            const uint8_t* __restrict__ bins8, uint32_t s8, const uint16_t* __restrict__ bins16, uint32_t s16,
            const Q* __restrict__ qin, Q* __restrict__ qout, BinsFM fm, const uint8_t* __restrict__ rmask,
            unsigned* __restrict__ scnt) {
    BST_PDL_ENTER();
    const PartChunk ch = chunks[blockIdx.x];
    __shared__ PartWork w;
    if (threadIdx.x == 0) w = works[ch.work];
    __syncthreads();
    part_rows<Q>(w, ch.start, ch.len, cursors + 2 * ch.work, ridx, tmp, bins8, s8, bins16, s16, qin, qout, fm.b8,
                 fm.b16, fm.n, rmask, rmask ? scnt + 2 * ch.work : nullptr);
}

void launch_partition(const PartWork* works, const PartChunk* chunks, uint32_t n_chunks,
                      const uint32_t* ridx, uint32_t* tmp, unsigned* cursors,
                      const uint8_t* bins8, uint32_t s8, const uint16_t* bins16, uint32_t s16,
                      cudaStream_t st, const void* qin, void* qout, int mode, const BinsFM& fm,
                      const uint8_t* rmask, unsigned* scnt) {
    if (n_chunks == 0) return;
    if (!qin || !qout)
        launch_k(k_partition<char>, n_chunks, PART_THREADS, 0, st, works, chunks, ridx, tmp, cursors, bins8, s8, bins16,
                                                             s16, nullptr, nullptr, fm, rmask, scnt);
    else if (mode == GRAD_Q8)
        launch_k(k_partition<char2>, n_chunks, PART_THREADS, 0, st, works, chunks, ridx, tmp, cursors, bins8, s8, bins16,
                                                              s16, static_cast<const char2*>(qin),
                                                              static_cast<char2*>(qout), fm, rmask, scnt);
    else if (mode == GRAD_Q16)
        launch_k(k_partition<short2>, n_chunks, PART_THREADS, 0, st, works, chunks, ridx, tmp, cursors, bins8, s8, bins16,
                                                               s16, static_cast<const short2*>(qin),
                                                               static_cast<short2*>(qout), fm, rmask, scnt);
    else
        launch_k(k_partition<float2>, n_chunks, PART_THREADS, 0, st, works, chunks, ridx, tmp, cursors, bins8, s8, bins16,
                                                               s16, static_cast<const float2*>(qin),
                                                               static_cast<float2*>(qout), fm, rmask, scnt);
}

template <typename Q>
__global__ void k_copy_chunks(const PartChunk* __restrict__ chunks, const uint32_t* __restrict__ src,
                              uint32_t* __restrict__ dst, const Q* __restrict__ qsrc, Q* __restrict__ qdst) {
    BST_PDL_ENTER();
    const PartChunk ch = chunks[blockIdx.x];
    for (uint32_t i = threadIdx.x; i < ch.len; i += blockDim.x) {
        dst[ch.start + i] = src[ch.start + i];
        if (qsrc) qdst[ch.start + i] = qsrc[ch.start + i];
    }
}

void launch_copy_chunks(const PartChunk* chunks, const PartWork* works, uint32_t n_chunks,
                        const uint32_t* src, uint32_t* dst, cudaStream_t st, const void* qsrc, void* qdst,
                        int mode) {
    (void)works;
    if (n_chunks == 0) return;
    if (!qsrc || !qdst)
        launch_k(k_copy_chunks<char>, n_chunks, 256, 0, st, chunks, src, dst, nullptr, nullptr);
    else if (mode == GRAD_Q8)
        launch_k(k_copy_chunks<char2>, n_chunks, 256, 0, st, chunks, src, dst, static_cast<const char2*>(qsrc),
                                                       static_cast<char2*>(qdst));
    else if (mode == GRAD_Q16)
        launch_k(k_copy_chunks<short2>, n_chunks, 256, 0, st, chunks, src, dst, static_cast<const short2*>(qsrc),
                                                        static_cast<short2*>(qdst));
    else
        launch_k(k_copy_chunks<float2>, n_chunks, 256, 0, st, chunks, src, dst, static_cast<const float2*>(qsrc),
                                                        static_cast<float2*>(qdst));
}

__global__ void k_iota(uint32_t* __restrict__ r, uint64_t n) {
    BST_PDL_ENTER();
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n;
         i += (uint64_t)gridDim.x * blockDim.x)
        r[i] = (uint32_t)i;
}

void launch_iota(uint32_t* ridx, uint64_t n, cudaStream_t st) {
    if (n == 0) return;
    uint64_t blocks = (n + 255) / 256;
    if (blocks > (uint64_t)sm_count() * 16) blocks = (uint64_t)sm_count() * 16;
    launch_k(k_iota, (unsigned)blocks, 256, 0, st, ridx, n);
}

// ============================================================================
// K8: leaf values -> predictions (grower.rs:208-219)
// ============================================================================

__global__ void k_leaf_update(const LeafSeg* __restrict__ leaves, uint32_t n_leaves,
                              const uint32_t* __restrict__ ridx, uint64_t n, float* __restrict__ pred,
                              uint32_t* __restrict__ row_leaf) {
    BST_PDL_ENTER();
    for (uint64_t p = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; p < n;
         p += (uint64_t)gridDim.x * blockDim.x) {
        uint32_t lo = 0, hi = n_leaves;  // last leaf with begin <= p
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (leaves[mid].begin <= p)
                lo = mid;
            else
                hi = mid;
        }
        const LeafSeg L = leaves[lo];
        if (p >= L.begin && p < (uint64_t)L.begin + L.count) {
            const uint32_t row = ridx[p];
            pred[row] = pred[row] + L.value;
            if (row_leaf) row_leaf[row] = L.tree_node;
        }
    }
}

void launch_leaf_update(const LeafSeg* leaves, uint32_t n_leaves, const uint32_t* ridx,
                        uint64_t n, float* pred, uint32_t* row_leaf, cudaStream_t st) {
    if (n == 0 || n_leaves == 0) return;
    uint64_t blocks = (n + 255) / 256;
    if (blocks > (uint64_t)sm_count() * 16) blocks = (uint64_t)sm_count() * 16;
    launch_k(k_leaf_update, (unsigned)blocks, 256, 0, st, leaves, n_leaves, ridx, n, pred, row_leaf);
}

// ============================================================================
// Device-side depth-wise growth: the level loop of TreeGrower::grow
// (training/gbdt/grower.rs:288-337, expansion.rs:137-196) as a fixed launch
// sequence whose sizes live in device memory (BState), so one CUDA graph
// replays a whole tree.
// ============================================================================

namespace {

// Block-wide exclusive scan (blockDim.x <= 1024); *total gets the block sum.
__device__ uint32_t block_excl_scan(uint32_t v, uint32_t* sh, uint32_t* total) {
    const int lane = threadIdx.x & 31, warp = threadIdx.x >> 5;
    const int nw = (blockDim.x + 31) >> 5;
    uint32_t x = v;
    for (int d = 1; d < 32; d <<= 1) {
        const uint32_t t = __shfl_up_sync(FULL, x, d);
        if (lane >= d) x += t;
    }
    if (lane == 31) sh[warp] = x;
    __syncthreads();
    if (warp == 0) {
        uint32_t y = lane < nw ? sh[lane] : 0u;
        for (int d = 1; d < 32; d <<= 1) {
            const uint32_t t = __shfl_up_sync(FULL, y, d);
            if (lane >= d) y += t;
        }
        if (lane < nw) sh[lane] = y;
    }
    __syncthreads();
    const uint32_t r = (warp ? sh[warp - 1] : 0u) + x - v;
    *total = sh[nw - 1];
    __syncthreads();
    return r;
}

// GainParams::compute_leaf_weight (gain.rs:151-168) x learning rate (mutable_tree.rs:258).
__device__ float leaf_value_dev(long long G, long long H, const double* scale, const LeafParams& lp) {
    const double g = (double)G * scale[2], h = (double)H * scale[3];
    float w;
    if (lp.alpha == 0.0) {
        w = __double2float_rn(-g / (h + lp.lambda));
    } else {
        const double ag = fabs(g);
        if (ag <= lp.alpha) {
            w = 0.0f;
        } else {
            const double sign = g > 0.0 ? -1.0 : 1.0;
            w = __double2float_rn(sign * (ag - lp.alpha) / (h + lp.lambda));
        }
    }
    return w * lp.learning_rate;
}

__device__ void write_leaf(BTreeNode& t, long long G, long long H, const double* scale, float v) {
    t.col = 0;
    t.bin = 0;
    t.flags = 4u;
    t.left = 0;
    t.right = 0;
    t.gain = 0.0f;
    t.leaf = v;
    t.G = (double)G * scale[2];
    t.H = (double)H * scale[3];
    t.cats[0] = t.cats[1] = t.cats[2] = t.cats[3] = 0ull;
}

}  // namespace


// Start of a depth-wise tree in one launch: row ids 0..n-1, the root node
// as the frontier, and the level state set up for the root histogram (one
// expanding node whose smaller child is all n rows, in `chunk`-row
// segments).
__global__ void k_b_root_init(BDev d, uint32_t* __restrict__ ridx, uint64_t n, uint32_t chunk) {
    BST_PDL_ENTER();
    uint32_t nseg = (uint32_t)((n + chunk - 1) / chunk);
    if (nseg > d.max_segs) nseg = d.max_segs;  // never: the buffer is sized for it
    const uint64_t stride = (uint64_t)gridDim.x * blockDim.x;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += stride) ridx[i] = (uint32_t)i;
    for (uint64_t c = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; c < nseg; c += stride) d.seg_exp[c] = 0;
    if (blockIdx.x != 0 || threadIdx.x != 0) return;
    BNode r;
    r.pnode = 0;
    r.tnode = 0;
    r.begin = 0;
    r.count = (uint32_t)n;
    r.G = 0;
    r.H = 0;
    r.split.gain = -INFINITY;
    r.split.col = 0;
    r.split.bin = 0;
    r.split.flags = 0;
    r.split.cats[0] = r.split.cats[1] = r.split.cats[2] = r.split.cats[3] = 0ull;
    r.split.tot_g = 0;
    r.split.tot_h = 0;
    d.front[0][0] = r;
    BExp e;
    e.front = 0;
    e.right_pnode = 0;
    e.tl = e.tr = 0;
    e.lc = 0;
    e.rc = (uint32_t)n;
    e.small_begin = 0;
    e.small_count = (uint32_t)n;
    e.part_off = 0;
    e.hist_off = 0;
    e.left_pnode = 0;
    e.pad1 = 0;
    d.exp[0] = e;
    BState s;
    s.n_front = 1;
    s.n_exp = 1;
    s.n_pnodes = 1;
    s.n_tnodes = 1;
    s.part_chunks = 0;
    s.hist_chunks = nseg;
    s.n_leaves = 0;
    s.leaf_chunks = 0;
    s.first_right = 1;
    s.hist_chunk = chunk;
    s.hist_rows = n;
    s.done = 0;
    s.err = 0;
    s.pad2[0] = s.pad2[1] = 0;
    *d.state = s;
}

void launch_b_root_init(const BDev& d, uint32_t* ridx, uint64_t n, uint32_t chunk, cudaStream_t st) {
    if (n == 0) return;
    uint64_t blocks = (n + 255) / 256;
    if (blocks > (uint64_t)sm_count() * 16) blocks = (uint64_t)sm_count() * 16;
    launch_k(k_b_root_init, (unsigned)blocks, 256, 0, st, d, ridx, n, chunk);
}



// Expansion decisions of one level (grower.rs:353-372, 530-539): leaves for
// the rest, right-child ids in frontier order (partition.rs:375), tree nodes
// in allocation order (mutable_tree.rs:105-164), partition work lists.
// buf: which row-index buffer holds the rows of this level's nodes (the
// leaves made here keep their rows there).
constexpr uint32_t DECIDE_THREADS = SCAN_WARPS * 32;  // the block size of its one caller, k_b_scan

__device__ void decide_body(BDev d, int a, LeafParams lp, const double* __restrict__ scale, uint32_t buf) {
    __shared__ uint32_t sh[33];
    __shared__ uint32_t s_jc[DECIDE_THREADS], s_j[DECIDE_THREADS], s_begin[DECIDE_THREADS];
    __shared__ uint32_t base_exp, base_leaf, base_chunk, first_right, tn0, nf;
    BState* s = d.state;
    if (threadIdx.x == 0) {
        nf = s->n_front;
        base_exp = 0;
        base_leaf = s->n_leaves;
        base_chunk = 0;
        first_right = s->n_pnodes;
        tn0 = s->n_tnodes;
    }
    __syncthreads();
    const BNode* A = d.front[a];
    for (uint32_t i0 = 0; i0 < nf; i0 += blockDim.x) {
        const uint32_t i = i0 + threadIdx.x;
        const bool valid = i < nf;
        BNode nd;
        if (valid) nd = A[i];
        const bool ex = valid && (nd.split.flags & 4u) && nd.split.gain > -INFINITY &&
                        !((double)nd.split.gain <= lp.min_gain);
        uint32_t te, tl, tc;
        const uint32_t je = block_excl_scan(ex ? 1u : 0u, sh, &te);
        const uint32_t jl = block_excl_scan((valid && !ex) ? 1u : 0u, sh, &tl);
        const uint32_t nch = ex ? (nd.count + B_PART_CHUNK - 1) / B_PART_CHUNK : 0u;
        const uint32_t jc = block_excl_scan(nch, sh, &tc);
        if (valid && !ex) {
            const float v = leaf_value_dev(nd.G, nd.H, scale, lp);
            write_leaf(d.tree[nd.tnode], nd.G, nd.H, scale, v);
            BLeaf lf;
            lf.begin = nd.begin;
            lf.count = nd.count;
            lf.value = v;
            lf.tnode = nd.tnode;
            lf.chunk_off = 0;
            lf.buf = buf;
            d.leaves[base_leaf + jl] = lf;
        }
        if (ex) {
            const uint32_t j = base_exp + je;
            const uint32_t tla = tn0 + 2 * j, tra = tn0 + 2 * j + 1;
            const bool cat = (nd.split.flags & 2u) != 0;
            const uint32_t col = nd.split.col;
            const BColumn bc = d.bcols[col];
            BTreeNode t;
            t.col = col;
            t.bin = nd.split.bin;
            t.flags = (nd.split.flags & 1u) | (cat ? 2u : 0u);
            t.left = tla;
            t.right = tra;
            t.gain = nd.split.gain;
            t.leaf = 0.0f;
            t.G = (double)nd.G * scale[2];
            t.H = (double)nd.H * scale[3];
            for (int q = 0; q < 4; ++q) t.cats[q] = nd.split.cats[q];
            d.tree[nd.tnode] = t;
            BExp e;
            e.front = i;
            e.right_pnode = first_right + j;
            e.tl = cat ? tra : tla;  // categorical: training-left rows go to the stored right child
            e.tr = cat ? tla : tra;
            e.lc = e.rc = e.small_begin = e.small_count = 0;
            e.part_off = base_chunk + jc;
            e.hist_off = 0;
            e.left_pnode = nd.pnode;
            e.pad1 = 0;
            d.exp[j] = e;
            PartWork w;
            w.begin = nd.begin;
            w.count = nd.count;
            w.matrix = bc.matrix;
            w.pos = bc.pos;
            w.thr_bin = nd.split.bin;
            w.flags = (nd.split.flags & 1u) | (bc.has_missing ? 2u : 0u) | (cat ? 4u : 0u);
            w.default_bin = bc.default_bin;
            w.pad = 0;
            for (int q = 0; q < 4; ++q) w.cats[q] = nd.split.cats[q];
            d.pworks[j] = w;
            d.cursors[2 * j] = nd.begin;
            d.cursors[2 * j + 1] = nd.begin + nd.count;
            if (d.rmask) d.scnt[2 * j] = d.scnt[2 * j + 1] = 0u;
        }
        // the partition's chunks of the tile's expanding nodes, so that each
        // partition block finds its node with one load (capacity: rows /
        // chunk + nodes, never exceeded), written by all threads: chunk c of
        // the tile belongs to the last thread whose first chunk is <= c
        s_jc[threadIdx.x] = jc;
        s_j[threadIdx.x] = base_exp + je;
        s_begin[threadIdx.x] = valid ? nd.begin : 0u;
        __syncthreads();
        for (uint32_t c = threadIdx.x; c < tc; c += blockDim.x) {
            uint32_t lo = 0, hi = blockDim.x;  // s_jc[lo] <= c < s_jc[hi]
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (s_jc[mid] <= c)
                    lo = mid;
                else
                    hi = mid;
            }
            const uint32_t g = base_chunk + c;
            if (g < d.max_part_chunks) d.part_map[g] = make_uint2(s_j[lo], s_begin[lo] + (c - s_jc[lo]) * B_PART_CHUNK);
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            base_exp += te;
            base_leaf += tl;
            base_chunk += tc;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        s->n_exp = base_exp;
        s->n_leaves = base_leaf;
        s->part_chunks = base_chunk;
        s->first_right = first_right;
        s->n_pnodes = first_right + base_exp;
        s->n_tnodes = tn0 + 2 * base_exp;
    }
}



// "Last block" hand-off: every block of the launch counts itself in
// state->done after a fence; the block that completes the count returns true
// (with the count reset) and may read everything the others wrote.
__device__ bool last_block(BState* s) {
    __shared__ bool last;
    __syncthreads();
    if (threadIdx.x == 0) {
        __threadfence();
        last = atomicAdd(&s->done, 1u) == gridDim.x - 1u;
        if (last) s->done = 0u;
    }
    __syncthreads();
    if (last) __threadfence();
    return last;
}

__device__ void children_body(BDev d, int a, int need_split);

// Partition of every expanding node (partition.rs:296-382) over 2048-row
// chunks (one atomic per side per chunk, part_rows) from row-index buffer
// rin into rout; the last block then derives the children (children_body).
template <typename Q>
__global__ void __launch_bounds__(PART_THREADS)
k_b_partition(BDev d, const uint32_t* __restrict__ ridx, uint32_t* __restrict__ tmp,
              const uint8_t* __restrict__ bins8, uint32_t s8, const uint16_t* __restrict__ bins16, uint32_t s16,
              int a, int need_split, const Q* __restrict__ qin, Q* __restrict__ qout, BinsFM fm) {
    BST_PDL_ENTER();
    __shared__ PartWork w;
    __shared__ uint2 s_m;
    const uint32_t total = min(d.state->part_chunks, d.max_part_chunks);
    for (uint32_t c = blockIdx.x; c < total; c += gridDim.x) {
        if (threadIdx.x == 0) {
            const uint2 m = d.part_map[c];  // (expansion, first row)
            s_m = m;
            w = d.pworks[m.x];
        }
        __syncthreads();
        const uint32_t j = s_m.x, start = s_m.y;
#ifdef BST_CHECKED
        const bool chunk_ok = BST_IN(start - w.begin, w.count, CHECK_PART_CHUNK);
        __syncthreads();  // every thread has read s_m / w before a skipped chunk's next rewrite
        if (!chunk_ok) continue;
#endif
        const uint32_t len = min(B_PART_CHUNK, w.begin + w.count - start);
        part_rows<Q>(w, start, len, d.cursors + 2 * j, ridx, tmp, bins8, s8, bins16, s16, qin, qout, fm.b8, fm.b16,
                     fm.n, d.rmask, d.rmask ? d.scnt + 2 * j : nullptr);
    }
    if (last_block(d.state)) children_body(d, a, need_split);
}

void launch_b_partition(const BDev& d, const uint32_t* rin, uint32_t* rout, const uint8_t* bins8, uint32_t s8,
                        const uint16_t* bins16, uint32_t s16, int a, int need_split, uint32_t grid,
                        const void* qin, void* qout, int mode, const BinsFM& fm, cudaStream_t st) {
    if (!qin || !qout)
        launch_k(k_b_partition<char>, grid, PART_THREADS, 0, st, d, rin, rout, bins8, s8, bins16, s16, a, need_split,
                                                           nullptr, nullptr, fm);
    else if (mode == GRAD_Q8)
        launch_k(k_b_partition<char2>, grid, PART_THREADS, 0, st, d, rin, rout, bins8, s8, bins16, s16, a, need_split,
                                                            static_cast<const char2*>(qin), static_cast<char2*>(qout),
                                                            fm);
    else if (mode == GRAD_Q16)
        launch_k(k_b_partition<short2>, grid, PART_THREADS, 0, st, d, rin, rout, bins8, s8, bins16, s16, a, need_split,
                                                             static_cast<const short2*>(qin),
                                                             static_cast<short2*>(qout), fm);
    else
        launch_k(k_b_partition<float2>, grid, PART_THREADS, 0, st, d, rin, rout, bins8, s8, bins16, s16, a, need_split,
                                                             static_cast<const float2*>(qin),
                                                             static_cast<float2*>(qout), fm);
}

// Column-major copy [f][n] of the first f columns of a row-major bin view
// (row stride s elements): 32 x 32 tiles through shared memory, coalesced on
// both sides.
template <typename T>
__global__ void k_transpose_bins(const T* __restrict__ in, uint32_t s, uint32_t f, uint64_t n,
                                 T* __restrict__ out) {
    BST_PDL_ENTER();
    __shared__ T t[32][33];
    const uint64_t r0 = (uint64_t)blockIdx.x * 32u;
    const uint32_t c0 = blockIdx.y * 32u;
    for (uint32_t k = threadIdx.y; k < 32u; k += blockDim.y) {
        const uint64_t r = r0 + k;
        const uint32_t c = c0 + threadIdx.x;
        if (r < n && c < f) t[k][threadIdx.x] = in[r * s + c];
    }
    __syncthreads();
    for (uint32_t k = threadIdx.y; k < 32u; k += blockDim.y) {
        const uint32_t c = c0 + k;
        const uint64_t r = r0 + threadIdx.x;
        if (r < n && c < f) out[(uint64_t)c * n + r] = t[threadIdx.x][k];
    }
}

void launch_transpose_bins(const uint8_t* b8, uint32_t s8, uint32_t f8, const uint16_t* b16, uint32_t s16,
                           uint32_t f16, uint64_t n, uint8_t* fm8, uint16_t* fm16, cudaStream_t st) {
    const dim3 blk(32, 8);
    if (f8 && n)
        launch_k(k_transpose_bins<uint8_t>, dim3((unsigned)((n + 31) / 32), (f8 + 31) / 32), blk, 0, st, b8, s8, f8, n, fm8);
    if (f16 && n)
        launch_k(k_transpose_bins<uint16_t>, dim3((unsigned)((n + 31) / 32), (f16 + 31) / 32), blk, 0, st, b16, s16, f16, n,
                                                                                               fm16);
}

// Children of every split: ranges from the partition cursors, smaller child
// (grower.rs:398-402), next frontier in (left, right) order, histogram or
// node-sum work over the smaller children.
// map[base + c] = the owner of segment c of a tile, for c < tc, written by
// all threads: thread t owns the segments from jc (exclusive scan over the
// tile's threads) on; the owner of c is the last thread whose jc is <= c.
// s_jc / s_own: shared arrays of blockDim entries.
__device__ void write_segment_owners(uint32_t* map, uint32_t cap, uint32_t base, uint32_t jc, uint32_t owner,
                                     uint32_t tc, uint32_t* s_jc, uint32_t* s_own) {
    s_jc[threadIdx.x] = jc;
    s_own[threadIdx.x] = owner;
    __syncthreads();
    for (uint32_t c = threadIdx.x; c < tc; c += blockDim.x) {
        uint32_t lo = 0, hi = blockDim.x;  // s_jc[lo] <= c < s_jc[hi]
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (s_jc[mid] <= c)
                lo = mid;
            else
                hi = mid;
        }
        if (base + c < cap) map[base + c] = s_own[lo];
    }
}

// The same for chunk maps of rows: map[base + c] = (owner, its first row
// + (c - its jc) x chunk rows). s_begin: a third shared array.
__device__ void write_chunk_owners(uint2* map, uint32_t cap, uint32_t base, uint32_t jc, uint32_t owner,
                                   uint32_t begin, uint32_t chunk, uint32_t tc, uint32_t* s_jc, uint32_t* s_own,
                                   uint32_t* s_begin) {
    s_jc[threadIdx.x] = jc;
    s_own[threadIdx.x] = owner;
    s_begin[threadIdx.x] = begin;
    __syncthreads();
    for (uint32_t c = threadIdx.x; c < tc; c += blockDim.x) {
        uint32_t lo = 0, hi = blockDim.x;  // s_jc[lo] <= c < s_jc[hi]
        while (hi - lo > 1) {
            const uint32_t mid = (lo + hi) >> 1;
            if (s_jc[mid] <= c)
                lo = mid;
            else
                hi = mid;
        }
        if (base + c < cap) map[base + c] = make_uint2(s_own[lo], s_begin[lo] + (c - s_jc[lo]) * chunk);
    }
}

__device__ void children_body(BDev d, int a, int need_split) {
    __shared__ uint32_t sh[33];
    __shared__ uint32_t s_jc[PART_THREADS], s_own[PART_THREADS];  // block size of its caller, k_b_partition
    __shared__ uint32_t base, n_exp, chunk;
    __shared__ unsigned long long rows;
    BState* s = d.state;
    if (threadIdx.x == 0) {
        n_exp = s->n_exp;
        base = 0;
        rows = 0ull;
    }
    __syncthreads();
    const BNode* A = d.front[a];
    BNode* B = d.front[a ^ 1];
    for (uint32_t j0 = 0; j0 < n_exp; j0 += blockDim.x) {
        const uint32_t j = j0 + threadIdx.x;
        const bool valid = j < n_exp;
        if (valid) {
            BExp e = d.exp[j];
            const BNode nd = A[e.front];
            const uint32_t lc = d.cursors[2 * j] - nd.begin, rc = nd.count - lc;
            const bool left_small = lc <= rc;
            e.lc = lc;
            e.rc = rc;
            e.small_begin = left_small ? nd.begin : nd.begin + lc;
            e.small_count = left_small ? lc : rc;
            BNode l, r;
            l.pnode = nd.pnode;
            l.tnode = e.tl;
            l.begin = nd.begin;
            l.count = lc;
            r.pnode = e.right_pnode;
            r.tnode = e.tr;
            r.begin = nd.begin + lc;
            r.count = rc;
            l.G = l.H = r.G = r.H = 0;
            l.split.gain = r.split.gain = -INFINITY;
            l.split.col = r.split.col = 0;
            l.split.bin = r.split.bin = 0;
            l.split.flags = r.split.flags = 0;
            for (int q = 0; q < 4; ++q) l.split.cats[q] = r.split.cats[q] = 0ull;
            l.split.tot_g = l.split.tot_h = r.split.tot_g = r.split.tot_h = 0;
            B[2 * j] = l;
            B[2 * j + 1] = r;
            // row sampling: the split search counts the sampled rows
            const uint32_t slc = d.rmask ? d.scnt[2 * j] : lc, src = d.rmask ? d.scnt[2 * j + 1] : rc;
            d.scan_nodes[2 * j] = ScanNode{nd.pnode, slc, 0u, 0u, 0, 0};
            d.scan_nodes[2 * j + 1] = ScanNode{e.right_pnode, src, 0u, 0u, 0, 0};
            d.exp[j] = e;
            atomicAdd(&rows, (unsigned long long)e.small_count);
        }
    }
    __syncthreads();
    if (threadIdx.x == 0) {
        // rows per histogram row segment: about hist_target segments (a
        // multiple of 256 rows in [1024, hist_seg_max]), so that the
        // persistent histogram launch has a few equal items per block; node
        // sums (last level) use HIST_CHUNK_MAX-row chunks
        uint32_t c = HIST_CHUNK_MAX;
        if (need_split) {
            const uint32_t tgt = d.hist_target ? d.hist_target : 1u;
            unsigned long long want = (rows + tgt - 1) / tgt;
            want = (want + 255ull) & ~255ull;
            c = (uint32_t)(want < 1024ull ? 1024ull : (want > d.hist_seg_max ? d.hist_seg_max : want));
        }
        chunk = c;
    }
    __syncthreads();
    for (uint32_t j0 = 0; j0 < n_exp; j0 += blockDim.x) {
        const uint32_t j = j0 + threadIdx.x;
        const bool valid = j < n_exp;
        const uint32_t nch = valid ? (d.exp[j].small_count + chunk - 1) / chunk : 0u;
        uint32_t tc;
        const uint32_t jc = block_excl_scan(nch, sh, &tc);
        if (valid) d.exp[j].hist_off = base + jc;
        // segment -> expansion (the buffer bound always holds)
        write_segment_owners(d.seg_exp, d.max_segs, base, jc, j, tc, s_jc, s_own);
        __syncthreads();
        if (threadIdx.x == 0) base += tc;
        __syncthreads();
    }
    if (!need_split)  // the node sums of k_b_sums accumulate from zero
        for (uint32_t i = threadIdx.x; i < 2 * n_exp; i += blockDim.x) d.sums[i] = 0;
    if (threadIdx.x == 0) {
        s->hist_chunks = base < d.max_segs ? base : d.max_segs;
        s->hist_chunk = chunk;
        s->n_front = 2 * n_exp;
        if (need_split) s->hist_rows += rows;
    }
}



// Children of a host-chosen expansion batch (batched leaf-wise growth):
// from the partition's cursors, each parent's child counts and smaller child
// (grower.rs:398-402), the level's histogram row segments (the layout the
// host-driven loop uploads, with the same segment size rule) and the
// children's scan nodes, so that the histograms follow the partition with no
// read-back. d.exp[j] carries the parents' left_pnode / right_pnode on entry.
__global__ void __launch_bounds__(1024) k_lw_children(BDev d, const PartWork* __restrict__ pw,
                                                     const unsigned* __restrict__ cursors, uint32_t k,
                                                     ScanNode* __restrict__ scan_nodes,
                                                     const unsigned* __restrict__ scnt) {
    BST_PDL_ENTER();
    __shared__ uint32_t sh[33];
    __shared__ uint32_t s_jc[1024], s_own[1024];
    __shared__ unsigned long long rows;
    __shared__ uint32_t chunk, base;
    const bool from_state = k == LW_K_FROM_STATE;
    if (from_state) k = d.state->n_exp;  // device-driven step (0: nothing to expand)
    if (k == 0) {
        if (threadIdx.x == 0) d.state->hist_chunks = 0;
        return;
    }
    if (threadIdx.x == 0) {
        rows = 0;
        base = 0;
    }
    __syncthreads();
    for (uint32_t j = threadIdx.x; j < k; j += blockDim.x) {
        const PartWork w = pw[j];
        const uint32_t lc = cursors[2 * j] - w.begin, rc = w.count - lc;
        BExp e = d.exp[j];
        e.lc = lc;
        e.rc = rc;
        const bool left_small = lc <= rc;
        e.small_begin = left_small ? w.begin : w.begin + lc;
        e.small_count = left_small ? lc : rc;
        d.exp[j] = e;
        // pad: the children's depth; counts: sampled rows under row sampling
        scan_nodes[2 * j] = ScanNode{e.left_pnode, scnt ? scnt[2 * j] : lc, 0u, e.pad1, 0, 0};
        scan_nodes[2 * j + 1] = ScanNode{e.right_pnode, scnt ? scnt[2 * j + 1] : rc, 0u, e.pad1, 0, 0};
        atomicAdd(&rows, (unsigned long long)e.small_count);
    }
    __syncthreads();
    if (threadIdx.x == 0) {  // rows per segment: about hist_target segments, a multiple of 256 in [1024, seg_max]
        const unsigned long long tgt = d.hist_target ? d.hist_target : 1u;
        unsigned long long want = (rows + tgt - 1) / tgt;
        want = (want + 255ull) & ~255ull;
        chunk = (uint32_t)(want < 1024ull ? 1024ull : (want > d.hist_seg_max ? d.hist_seg_max : want));
    }
    __syncthreads();
    for (uint32_t j0 = 0; j0 < k; j0 += blockDim.x) {
        const uint32_t j = j0 + threadIdx.x;
        const bool valid = j < k;
        const uint32_t nch = valid ? (d.exp[j].small_count + chunk - 1) / chunk : 0u;
        uint32_t tc;
        const uint32_t jc = block_excl_scan(nch, sh, &tc);
        if (valid) d.exp[j].hist_off = base + jc;
        write_segment_owners(d.seg_exp, d.max_segs, base, jc, j, tc, s_jc, s_own);  // segment -> expansion
        __syncthreads();
        if (threadIdx.x == 0) base += tc;
        __syncthreads();
    }
    const uint32_t total = base < d.max_segs ? base : d.max_segs;
    if (threadIdx.x == 0) {
        d.state->n_exp = k;
        d.state->hist_chunks = total;
        d.state->hist_chunk = chunk;
        if (from_state) d.state->hist_rows += rows;
    }
}

void launch_lw_children(const BDev& d, const PartWork* pw, const unsigned* cursors, uint32_t k, ScanNode* scan_nodes,
                        const unsigned* scnt, cudaStream_t st) {
    if (k == 0) return;
    launch_k(k_lw_children, 1, 1024, 0, st, d, pw, cursors, k, scan_nodes, scnt);
}

// ============================================================================
// Device-side leaf-wise growth (expansion.rs:129-213, grower.rs:265-342,
// 484-514): k_lw_replay replays the reference's heap pops on one warp; the
// level kernels expand the batches it hands out.
// ============================================================================

namespace {

__device__ __forceinline__ bool lw_expands(const NodeSplit& s, float min_gain) {  // grower.rs:530-539
    const bool valid = (s.flags & 4u) && s.gain > -INFINITY;
    return valid && !(s.gain <= min_gain);
}

// a pops before b: larger gain, ties by higher id (expansion.rs:311-319)
__device__ __forceinline__ bool lw_before(float ga, uint32_t va, float gb, uint32_t vb) {
    return ga > gb || (ga == gb && va > vb);
}

// Warp argmax over heap entries [0, n) that pass `ok`: returns the index
// (0xFFFFFFFF: none). All lanes get the result.
template <class Ok>
__device__ uint32_t lw_argmax(const LwCand* heap, uint32_t n, Ok ok) {
    const uint32_t lane = threadIdx.x & 31u;
    float bg = -INFINITY;
    uint32_t bv = 0, bi = 0xFFFFFFFFu;
    for (uint32_t i = lane; i < n; i += 32) {
        if (!ok(i)) continue;
        const float g = heap[i].split.gain;
        const uint32_t v = heap[i].vid;
        if (bi == 0xFFFFFFFFu || lw_before(g, v, bg, bv)) {
            bg = g;
            bv = v;
            bi = i;
        }
    }
    for (int o = 16; o > 0; o >>= 1) {
        const float og = __shfl_xor_sync(FULL, bg, o);
        const uint32_t ov = __shfl_xor_sync(FULL, bv, o), oi = __shfl_xor_sync(FULL, bi, o);
        if (oi != 0xFFFFFFFFu && (bi == 0xFFFFFFFFu || lw_before(og, ov, bg, bv))) {
            bg = og;
            bv = ov;
            bi = oi;
        }
    }
    return __shfl_sync(FULL, bi, 0);  // one answer for the warp, whatever the gains hold
}

// make_leaf (grower.rs:484-514): the leaf's value from its exact sums (the
// quantised forms solve it again from the f32 gradients), listed for the
// leaf kernels with the node's final row range.
__device__ void lw_make_leaf(const BDev& d, const LwDev& w, const LwCand& c, const double* scale, const LeafParams& lp,
                             uint32_t slot) {
    const float v = leaf_value_dev(c.split.tot_g, c.split.tot_h, scale, lp);
    write_leaf(d.tree[c.tnode], c.split.tot_g, c.split.tot_h, scale, v);
    const uint2 r = w.pn[c.pnode];
    BLeaf lf;
    lf.begin = r.x;
    lf.count = r.y;
    lf.value = v;
    lf.tnode = c.tnode;
    lf.chunk_off = 0;
    lf.buf = 0;
    d.leaves[slot] = lf;
}

}  // namespace

__global__ void k_lw_init(BDev d, LwDev w, uint32_t n, uint32_t root_count) {
    BST_PDL_ENTER();
    if (threadIdx.x != 0 || blockIdx.x != 0) return;
    LwCand r;
    r.split = w.child[0];
    r.pnode = 0;
    r.tnode = 0;
    r.depth = 0;
    r.count = root_count;
    r.vid = 0;
    r.pad[0] = r.pad[1] = r.pad[2] = 0;
    w.heap[0] = r;
    w.pn[0] = make_uint2(0u, n);
    LwState s;
    s.n_heap = 1;
    s.n_leaves = 1;
    s.n_vid = 1;
    s.n_batch = 0;
    s.done = 0;
    s.err = 0;
    s.n_leaf_out = 0;
    s.pad = 0;
    *w.st = s;
    BState& b = *d.state;
    b.n_front = 0;
    b.n_exp = 0;
    b.n_pnodes = 1;
    b.n_tnodes = 1;
    b.part_chunks = 0;
    b.hist_chunks = 0;
    b.n_leaves = 0;
    b.leaf_chunks = 0;
    b.first_right = 1;
    b.done = 0;
    b.err = 0;
    b.hist_rows = n;  // the root's histogram
}

void launch_lw_init(const BDev& d, const LwDev& w, uint32_t n, uint32_t root_count, cudaStream_t st) {
    launch_k(k_lw_init, 1, 32, 0, st, d, w, n, root_count);
}

// Absorbs the last step's expansions (children counts from the partition
// cursors, splits from the scan) into the speculation table, then pops
// (grower.rs:265-342) until a popped leaf needs an expansion that has not
// run: that leaf and the best other unexpanded candidates become the next
// step's batch (level state written, BState::n_exp = its size). When the
// budget or the heap runs out, every remaining candidate becomes a leaf (an
// expanded one over its whole range again) and the tree is done.
// The block stages the heap and the speculation table in shared memory
// (CACHED; both stay in global memory otherwise); warp 0 replays the pops,
// the whole block ranks the batch candidates and writes the batch, and the
// block writes heap and table back.
constexpr uint32_t LW_REPLAY_THREADS = 512;
constexpr size_t LW_REPLAY_SMEM_MAX = 200 * 1024;

// Block copy of n records, eight 16-byte loads in flight per thread.
template <typename T>
__device__ __forceinline__ void lw_copy(T* dst, const T* src, uint32_t n) {
    static_assert(sizeof(T) % 16 == 0, "16-byte records");
    constexpr uint32_t U = 8;
    const uint4* s = reinterpret_cast<const uint4*>(src);
    uint4* d = reinterpret_cast<uint4*>(dst);
    const uint32_t words = n * (uint32_t)(sizeof(T) / 16);
    for (uint32_t b = threadIdx.x; b < words; b += blockDim.x * U) {
        uint4 r[U];
#pragma unroll
        for (uint32_t u = 0; u < U; ++u) {
            const uint32_t i = b + u * blockDim.x;
            if (i < words) r[u] = s[i];
        }
#pragma unroll
        for (uint32_t u = 0; u < U; ++u) {
            const uint32_t i = b + u * blockDim.x;
            if (i < words) d[i] = r[u];
        }
    }
}

// Pop-order key of an expandable candidate: a pops before b iff key(a) >
// key(b) (larger gain, then higher id; gains are never NaN, -0 counts as 0).
__device__ __forceinline__ unsigned long long lw_key(float g, uint32_t vid) {
    if (g == 0.0f) g = 0.0f;
    uint32_t u = __float_as_uint(g);
    u = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    return ((unsigned long long)u << 32) | vid;
}

template <bool CACHED>
__global__ void __launch_bounds__(LW_REPLAY_THREADS) k_lw_replay(BDev d, LwDev w, LeafParams lp,
                                                                 const double* __restrict__ scale) {
    BST_PDL_ENTER();
    extern __shared__ __align__(16) unsigned char lw_smem[];
    __shared__ LwState sS;
    __shared__ uint32_t s_mode, s_e, s_bmax, s_np, s_nt, s_k, s_chunk_base;
    __shared__ uint32_t sh[33];
    BState& B = *d.state;
    LwState S = *w.st;
    if (S.done) {
        if (threadIdx.x == 0) {
            B.n_exp = 0;
            B.part_chunks = 0;
            B.hist_chunks = 0;
        }
        return;
    }
    LwCand* heap = w.heap;
    LwSpec* spec = w.spec;
    unsigned long long* keys = w.keys;
    uint32_t* ranks = w.ranks;  // [heap_cap] ranks, then [heap_cap] members
    if (CACHED) {
        unsigned char* p = lw_smem;
        heap = reinterpret_cast<LwCand*>(p);
        p += (size_t)w.heap_cap * sizeof(LwCand);
        spec = reinterpret_cast<LwSpec*>(p);
        p += (size_t)w.max_pnodes * sizeof(LwSpec);
        keys = reinterpret_cast<unsigned long long*>(p);
        p += (size_t)w.heap_cap * sizeof(unsigned long long);
        ranks = reinterpret_cast<uint32_t*>(p);
    }
    uint32_t* members = ranks + w.heap_cap;  // ranks: then the members' first partition chunks
    const uint32_t np0 = B.n_pnodes;
    if (CACHED) {  // partition nodes >= np0 hold no expansion yet
        lw_copy(heap, w.heap, S.n_heap);
        lw_copy(spec, w.spec, np0);
        for (uint32_t q = np0 + threadIdx.x; q < w.max_pnodes; q += blockDim.x) spec[q].valid = 0;
        __syncthreads();
    }
    // 1. the last step's children
    for (uint32_t j = threadIdx.x; j < S.n_batch; j += blockDim.x) {
        const BExp e = d.exp[j];
        const uint32_t P = e.left_pnode, R = e.right_pnode;
        const uint2 pr = w.pn[P];
        const uint32_t lc = d.cursors[2 * j] - pr.x, rc = pr.y - lc;
        LwSpec sp;
        sp.right_pnode = R;
        sp.begin = pr.x;
        sp.count = pr.y;
        sp.valid = 1;
        for (int q = 0; q < 2; ++q) {
            LwCand& k = sp.kids[q];
            k.split = w.child[2 * j + q];
            k.pnode = q ? R : P;
            k.tnode = 0;
            k.depth = e.pad1;
            k.count = q ? rc : lc;
            k.vid = 0;
            k.pad[0] = k.pad[1] = k.pad[2] = 0;
        }
        spec[P] = sp;
        w.pn[P] = make_uint2(pr.x, lc);
        w.pn[R] = make_uint2(pr.x + lc, rc);
    }
    S.n_batch = 0;
    __syncthreads();
    // 2. pops (warp 0); s_mode: 0 done, 1 batch needed, 2 out of slots
    if (threadIdx.x < 32) {
        const uint32_t lane = threadIdx.x;
        uint32_t n_pnodes = np0, n_tnodes = B.n_tnodes;
        uint32_t mode = 0;
        for (;;) {
            if (S.n_leaves >= w.max_leaves || S.n_heap == 0) break;
            const uint32_t i = lw_argmax(heap, S.n_heap, [](uint32_t) { return true; });
            const LwCand e = heap[i];
            const bool ex = lw_expands(e.split, w.min_gain);
            if (ex && !spec[e.pnode].valid) {
                // the next step: e and the best unexpanded candidates, at most
                // as many as pops remain (rem after e's pop) and as free slots
                // allow
                const uint32_t rem = w.max_leaves - (S.n_leaves + 1);
                const int64_t room = (int64_t)w.max_pnodes - (int64_t)n_pnodes - (int64_t)rem;
                const int64_t want = (int64_t)rem + 1;
                mode = room < 1 ? 2u : 1u;
                if (lane == 0) {
                    s_e = i;
                    s_bmax = room < 1 ? 0u : (uint32_t)(want < room ? want : room);
                }
                break;
            }
            // pop e
            if (lane == 0) heap[i] = heap[S.n_heap - 1];
            S.n_heap -= 1;
            S.n_leaves += 1;
            __syncwarp();
            if (!ex) {
                if (lane == 0) lw_make_leaf(d, w, e, scale, lp, S.n_leaf_out);
                S.n_leaf_out += 1;
                __syncwarp();
                continue;
            }
            // apply_split (grower.rs:576-650): children tree nodes in
            // allocation order; a categorical split sends the training-left
            // rows to the stored right child
            const LwSpec sp = spec[e.pnode];
            const uint32_t l = n_tnodes, r = n_tnodes + 1;
            const bool cat = (e.split.flags & 2u) != 0u;
            if (lane == 0) {
                spec[e.pnode].valid = 0;
                BTreeNode t;
                t.col = e.split.col;
                t.bin = e.split.bin;
                t.flags = (e.split.flags & 1u) | (cat ? 2u : 0u);
                t.left = l;
                t.right = r;
                t.gain = e.split.gain;
                t.leaf = 0.0f;
                t.G = (double)e.split.tot_g * scale[2];
                t.H = (double)e.split.tot_h * scale[3];
                for (int q = 0; q < 4; ++q) t.cats[q] = e.split.cats[q];
                d.tree[e.tnode] = t;
                LwCand k0 = sp.kids[0], k1 = sp.kids[1];
                k0.tnode = cat ? r : l;
                k1.tnode = cat ? l : r;
                k0.vid = e.vid;
                k1.vid = S.n_vid;
                heap[S.n_heap] = k0;
                heap[S.n_heap + 1] = k1;
            }
            n_tnodes = r + 1;
            S.n_vid += 1;
            S.n_heap += 2;
            __syncwarp();
        }
        if (mode == 0) {
            // 3. done: every candidate left becomes a leaf, an expanded one
            // over its whole range (its right partition node keeps no rows)
            for (uint32_t q = 0; q < S.n_heap; ++q) {
                const LwCand c = heap[q];
                if (lane == 0) {
                    const LwSpec sp = spec[c.pnode];
                    if (sp.valid) {
                        w.pn[c.pnode] = make_uint2(sp.begin, sp.count);
                        w.pn[sp.right_pnode] = make_uint2(sp.begin + sp.count, 0u);
                        spec[c.pnode].valid = 0;
                    }
                    lw_make_leaf(d, w, c, scale, lp, S.n_leaf_out);
                }
                S.n_leaf_out += 1;
                __syncwarp();
            }
            S.n_heap = 0;
            S.done = 1;
        } else if (mode == 2) {
            S.err = 1;
            S.done = 1;
        }
        if (lane == 0) {
            s_mode = mode;
            s_np = n_pnodes;
            s_nt = n_tnodes;
            sS = S;
        }
    }
    __syncthreads();
    const uint32_t mode = s_mode;
    if (mode == 1) {
        // 4. the batch: e first, then the expandable unexpanded candidates
        // in pop order (rank = how many of them pop earlier), at most bmax
        const uint32_t nh = sS.n_heap, ei = s_e, bmax = s_bmax, first_right = s_np;
        for (uint32_t q = threadIdx.x; q < nh; q += blockDim.x) {
            const LwCand& c = heap[q];
            const bool el = q != ei && lw_expands(c.split, w.min_gain) && !spec[c.pnode].valid;
            keys[q] = el ? lw_key(c.split.gain, c.vid) : 0ull;
        }
        if (threadIdx.x == 0) members[0] = ei;
        __syncthreads();
        uint32_t n_el = 0;
        for (uint32_t q = threadIdx.x; q < nh; q += blockDim.x) {
            const unsigned long long kq = keys[q];
            if (!kq) continue;
            uint32_t r = 0;
            for (uint32_t t = 0; t < nh; ++t) r += keys[t] > kq ? 1u : 0u;
            if (r + 1 < bmax) members[r + 1] = q;
            ++n_el;
        }
        uint32_t tot_el;
        block_excl_scan(n_el, sh, &tot_el);  // (synchronises: members complete)
        const uint32_t k = 1u + min(tot_el, bmax - 1u);
        if (threadIdx.x == 0) s_chunk_base = 0;
        __syncthreads();
        for (uint32_t j0 = 0; j0 < k; j0 += blockDim.x) {
            const uint32_t j = j0 + threadIdx.x;
            const bool valid = j < k;
            const LwCand* c = valid ? &heap[members[j]] : nullptr;
            const uint2 r = valid ? w.pn[c->pnode] : make_uint2(0u, 0u);
            const uint32_t nch = (r.y + B_PART_CHUNK - 1) / B_PART_CHUNK;
            uint32_t tc;
            const uint32_t off = s_chunk_base + block_excl_scan(nch, sh, &tc);
            if (valid) {
                const NodeSplit& sp = c->split;
                const bool cat = (sp.flags & 2u) != 0u;
                const BColumn bc = d.bcols[sp.col];
                BExp x;
                x.front = 0;
                x.right_pnode = first_right + j;
                x.tl = x.tr = 0;
                x.lc = x.rc = x.small_begin = x.small_count = 0;
                x.part_off = off;
                x.hist_off = 0;
                x.left_pnode = c->pnode;
                x.pad1 = c->depth + 1;  // the children's depth (column masks)
                d.exp[j] = x;
                PartWork pw;
                pw.begin = r.x;
                pw.count = r.y;
                pw.matrix = bc.matrix;
                pw.pos = bc.pos;
                pw.thr_bin = sp.bin;
                pw.flags = (sp.flags & 1u) | (bc.has_missing ? 2u : 0u) | (cat ? 4u : 0u);
                pw.default_bin = bc.default_bin;
                pw.pad = 0;
                for (int q = 0; q < 4; ++q) pw.cats[q] = sp.cats[q];
                d.pworks[j] = pw;
                d.cursors[2 * j] = r.x;
                d.cursors[2 * j + 1] = r.x + r.y;
                if (d.rmask) d.scnt[2 * j] = d.scnt[2 * j + 1] = 0u;
                ranks[j] = off;  // the member's first partition chunk
            }
            __syncthreads();
            if (threadIdx.x == 0) s_chunk_base += tc;
            __syncthreads();
        }
        // the chunk map, all threads: chunk c belongs to the last member whose
        // first chunk is <= c
        const uint32_t total = min(s_chunk_base, d.max_part_chunks);
        for (uint32_t c = threadIdx.x; c < total; c += blockDim.x) {
            uint32_t lo = 0, hi = k;  // ranks[lo] <= c < ranks[hi]
            while (hi - lo > 1) {
                const uint32_t mid = (lo + hi) >> 1;
                if (ranks[mid] <= c)
                    lo = mid;
                else
                    hi = mid;
            }
            d.part_map[c] = make_uint2(lo, w.pn[heap[members[lo]].pnode].x + (c - ranks[lo]) * B_PART_CHUNK);
        }
        if (threadIdx.x == 0) {
            sS.n_batch = k;
            s_np = first_right + k;
            B.n_exp = k;
            B.first_right = first_right;
            B.part_chunks = min(s_chunk_base, d.max_part_chunks);
            B.hist_chunks = 0;
        }
        __syncthreads();
    }
    if (threadIdx.x == 0) {
        if (mode != 1) {
            if (mode == 0) B.n_leaves = sS.n_leaf_out;
            B.n_exp = 0;
            B.part_chunks = 0;
            B.hist_chunks = 0;
        }
        B.n_pnodes = s_np;
        B.n_tnodes = s_nt;
        *w.st = sS;
    }
    if (CACHED && mode == 1) {  // the state the next step starts from
        lw_copy(w.heap, heap, sS.n_heap);
        lw_copy(w.spec, spec, s_np);
    }
}

static size_t lw_replay_smem(const LwDev& w) {
    return (size_t)w.heap_cap * (sizeof(LwCand) + sizeof(unsigned long long) + 2 * sizeof(uint32_t)) +
           (size_t)w.max_pnodes * sizeof(LwSpec);
}

void launch_lw_replay(const BDev& d, const LwDev& w, LeafParams lp, const double* scale, cudaStream_t st) {
    const size_t smem = lw_replay_smem(w);
    if (smem <= LW_REPLAY_SMEM_MAX) {  // 255 leaves: 160 KB
        init_kernel_attributes();
        launch_k(k_lw_replay<true>, 1, LW_REPLAY_THREADS, smem, st, d, w, lp, scale);
    } else {
        launch_k(k_lw_replay<false>, 1, LW_REPLAY_THREADS, 0, st, d, w, lp, scale);
    }
}

// Partition of the pending batch over its chunk map, rin -> rout (no
// children derivation: k_lw_children follows).
template <typename Q>
__global__ void __launch_bounds__(PART_THREADS)
k_lw_partition(BDev d, const uint32_t* __restrict__ ridx, uint32_t* __restrict__ tmp,
               const uint8_t* __restrict__ bins8, uint32_t s8, const uint16_t* __restrict__ bins16, uint32_t s16,
               const Q* __restrict__ qin, Q* __restrict__ qout, BinsFM fm) {
    BST_PDL_ENTER();
    __shared__ PartWork w;
    __shared__ uint2 s_m;
    const uint32_t total = min(d.state->part_chunks, d.max_part_chunks);
    for (uint32_t c = blockIdx.x; c < total; c += gridDim.x) {
        if (threadIdx.x == 0) {
            const uint2 m = d.part_map[c];
            s_m = m;
            w = d.pworks[m.x];
        }
        __syncthreads();
        const uint32_t j = s_m.x, start = s_m.y;
#ifdef BST_CHECKED
        const bool chunk_ok = BST_IN(start - w.begin, w.count, CHECK_PART_CHUNK);
        __syncthreads();  // every thread has read s_m / w before a skipped chunk's next rewrite
        if (!chunk_ok) continue;
#endif
        const uint32_t len = min(B_PART_CHUNK, w.begin + w.count - start);
        part_rows<Q>(w, start, len, d.cursors + 2 * j, ridx, tmp, bins8, s8, bins16, s16, qin, qout, fm.b8, fm.b16,
                     fm.n, d.rmask, d.rmask ? d.scnt + 2 * j : nullptr);
    }
}

// The partitioned rows (and gradient elements) back into the row buffer:
// chunk c copies its 2048 positions of its node's range.
constexpr uint32_t LW_COPY_THREADS = 256;

template <typename Q>
__global__ void __launch_bounds__(LW_COPY_THREADS) k_lw_copy_back(BDev d, const uint32_t* __restrict__ tmp, uint32_t* __restrict__ ridx,
                               const Q* __restrict__ qtmp, Q* __restrict__ q) {
    BST_PDL_ENTER();
    const uint32_t total = min(d.state->part_chunks, d.max_part_chunks);
    for (uint32_t c = blockIdx.x; c < total; c += gridDim.x) {
        const uint2 m = d.part_map[c];
        const PartWork w = d.pworks[m.x];
        const uint32_t len = min(B_PART_CHUNK, w.begin + w.count - m.y);
        // all of a thread's loads before its stores (launched with
        // LW_COPY_THREADS threads: U positions per thread cover a chunk)
        constexpr uint32_t U = B_PART_CHUNK / LW_COPY_THREADS;
        static_assert(B_PART_CHUNK % LW_COPY_THREADS == 0, "whole chunks");
        uint32_t rv[U];
        Q qv[std::is_same<Q, char>::value ? 1 : U];
#pragma unroll
        for (uint32_t u = 0; u < U; ++u) {
            const uint32_t i = threadIdx.x + u * LW_COPY_THREADS;
            if (i < len) {
                rv[u] = tmp[m.y + i];
                if constexpr (!std::is_same<Q, char>::value) qv[u] = qtmp[m.y + i];
            }
        }
#pragma unroll
        for (uint32_t u = 0; u < U; ++u) {
            const uint32_t i = threadIdx.x + u * LW_COPY_THREADS;
            if (i < len) {
                ridx[m.y + i] = rv[u];
                if constexpr (!std::is_same<Q, char>::value) q[m.y + i] = qv[u];
            }
        }
    }
}

template <typename Q>
static void lw_partition_t(const BDev& d, uint32_t* rin, uint32_t* rout, const uint8_t* bins8, uint32_t s8,
                           const uint16_t* bins16, uint32_t s16, uint32_t grid, Q* qin, Q* qout, const BinsFM& fm,
                           cudaStream_t st) {
    launch_k(k_lw_partition<Q>, grid, PART_THREADS, 0, st, d, rin, rout, bins8, s8, bins16, s16, qin, qout, fm);
    launch_k(k_lw_copy_back<Q>, grid, LW_COPY_THREADS, 0, st, d, rout, rin, qout, qin);
}

void launch_lw_partition(const BDev& d, uint32_t* rin, uint32_t* rout, const uint8_t* bins8, uint32_t s8,
                         const uint16_t* bins16, uint32_t s16, uint32_t grid, void* qin, void* qout, int mode,
                         const BinsFM& fm, cudaStream_t st) {
    if (!qin || !qout)
        lw_partition_t<char>(d, rin, rout, bins8, s8, bins16, s16, grid, nullptr, nullptr, fm, st);
    else if (mode == GRAD_Q8)
        lw_partition_t<char2>(d, rin, rout, bins8, s8, bins16, s16, grid, static_cast<char2*>(qin),
                              static_cast<char2*>(qout), fm, st);
    else if (mode == GRAD_Q16)
        lw_partition_t<short2>(d, rin, rout, bins8, s8, bins16, s16, grid, static_cast<short2*>(qin),
                               static_cast<short2*>(qout), fm, st);
    else
        lw_partition_t<float2>(d, rin, rout, bins8, s8, bins16, s16, grid, static_cast<float2*>(qin),
                               static_cast<float2*>(qout), fm, st);
}

// Leaf chunk map of the finished tree (k_b_finalize's second half) and the
// leaf sums zeroed for the quantised forms' exact leaf solve.
__global__ void __launch_bounds__(1024) k_lw_leaves(BDev d) {
    BST_PDL_ENTER();
    __shared__ uint32_t sh[33];
    __shared__ uint32_t s_jc[1024], s_own[1024], s_begin[1024];
    __shared__ uint32_t base;
    BState* s = d.state;
    const uint32_t nl = s->n_leaves;
    if (threadIdx.x == 0) base = 0;
    __syncthreads();
    for (uint32_t l0 = 0; l0 < nl; l0 += blockDim.x) {
        const uint32_t l = l0 + threadIdx.x;
        const uint32_t begin = l < nl ? d.leaves[l].begin : 0u;
        const uint32_t nch = l < nl ? (d.leaves[l].count + B_LEAF_CHUNK - 1) / B_LEAF_CHUNK : 0u;
        uint32_t tc;
        const uint32_t jc = block_excl_scan(nch, sh, &tc);
        if (l < nl) d.leaves[l].chunk_off = base + jc;
        // chunk -> (leaf, first row)
        write_chunk_owners(d.leaf_map, d.max_leaf_chunks, base, jc, l, begin, B_LEAF_CHUNK, tc, s_jc, s_own, s_begin);
        __syncthreads();
        if (threadIdx.x == 0) base += tc;
        __syncthreads();
    }
    for (uint32_t i = threadIdx.x; i < 2 * nl; i += blockDim.x) d.sums[i] = 0;
    if (threadIdx.x == 0) s->leaf_chunks = base < d.max_leaf_chunks ? base : d.max_leaf_chunks;
}

void launch_lw_leaves(const BDev& d, cudaStream_t st) { launch_k(k_lw_leaves, 1, 1024, 0, st, d); }

template <typename HB>
__global__ void k_b_zero_right(BDev d, HB* __restrict__ hist, uint64_t slot_bins) {
    BST_PDL_ENTER();
    const uint64_t n = (uint64_t)d.state->n_exp * slot_bins;
    HB* p = hist + (uint64_t)d.state->first_right * slot_bins;
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        p[i] = hb_make<HB>(0, 0);
}

void launch_b_zero_right(const BDev& d, void* hist, uint64_t slot_bins, uint32_t grid, cudaStream_t st, int hist32) {
    if (hist32)
        launch_k(k_b_zero_right<HBin32>, grid, 256, 0, st, d, static_cast<HBin32*>(hist), slot_bins);
    else
        launch_k(k_b_zero_right<HBin>, grid, 256, 0, st, d, static_cast<HBin*>(hist), slot_bins);
}

// Histograms of all smaller children of the level (one persistent launch).
template <int MODE, typename HB>
__global__ void __launch_bounds__(HIST_THREADS)
k_b_hist(BDev d, const HistTile* __restrict__ tiles, uint32_t n_tiles, uint32_t S, const uint32_t* __restrict__ ridx,
         GradRef gr, const uint8_t* __restrict__ bins8, uint32_t s8, const uint16_t* __restrict__ bins16, uint32_t s16,
         HB* __restrict__ hist, uint64_t slot_bins) {
    BST_PDL_ENTER();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint32_t* sm = reinterpret_cast<uint32_t*>(smem_raw);
    __shared__ HistTile tile;
    const GradLoad<MODE> load(gr);
    const uint32_t CH = d.state->hist_chunk;
    const uint64_t items = (uint64_t)d.state->hist_chunks * n_tiles;
    for (uint64_t it = blockIdx.x; it < items; it += gridDim.x) {
        const uint32_t c = (uint32_t)(it / n_tiles), t = (uint32_t)(it % n_tiles);
        const uint32_t j = d.seg_exp[c];
        const BExp e = d.exp[j];
        const uint32_t start = e.small_begin + (c - e.hist_off) * CH;
        const uint32_t seg_count = min(CH, e.small_begin + e.small_count - start);
        if (threadIdx.x == 0) tile = tiles[t];
        __syncthreads();
        for (uint32_t off = 0; off < seg_count; off += HIST_CHUNK_MAX) {  // block-uniform
            HistChunk ch;
            ch.slot = e.right_pnode;
            ch.begin = start + off;
            ch.count = min((uint32_t)HIST_CHUNK_MAX, seg_count - off);
            ch.flags = 0u;
            hist_item<MODE, HB>(ch, tile, sm, S, ridx, load, bins8, s8, bins16, s16, hist, slot_bins);
        }
    }
}

void launch_b_hist(const BDev& d, const HistTile* tiles, uint32_t n_tiles, uint32_t max_smem_bins,
                   const uint32_t* ridx, const GradRef& gr, const uint8_t* bins8, uint32_t s8,
                   const uint16_t* bins16, uint32_t s16, void* hist, uint64_t slot_bins, uint32_t grid,
                   cudaStream_t st, int hist32) {
    if (n_tiles == 0) return;
    const uint32_t S = (max_smem_bins + 3u) & ~3u;
    const size_t smem = (size_t)S * acc_words(gr.mode) * sizeof(uint32_t);
    init_kernel_attributes();
    HBin* h64 = static_cast<HBin*>(hist);
    HBin32* h32 = static_cast<HBin32*>(hist);
    if (gr.mode == GRAD_Q16)
        launch_k(k_b_hist<GRAD_Q16, HBin>, grid, HIST_THREADS, smem, st, d, tiles, n_tiles, S, ridx, gr, bins8, s8, bins16,
                                                                    s16, h64, slot_bins);
    else if (gr.mode == GRAD_Q8 && hist32)
        launch_k(k_b_hist<GRAD_Q8, HBin32>, grid, HIST_THREADS, smem, st, d, tiles, n_tiles, S, ridx, gr, bins8, s8, bins16,
                                                                     s16, h32, slot_bins);
    else if (gr.mode == GRAD_Q8)
        launch_k(k_b_hist<GRAD_Q8, HBin>, grid, HIST_THREADS, smem, st, d, tiles, n_tiles, S, ridx, gr, bins8, s8, bins16,
                                                                   s16, h64, slot_bins);
    else
        launch_k(k_b_hist<GRAD_F32, HBin>, grid, HIST_THREADS, smem, st, d, tiles, n_tiles, S, ridx, gr, bins8, s8, bins16,
                                                                    s16, h64, slot_bins);
}


// Orderable key of a column's candidate for the per-node atomicMax: larger
// gain first, then the column the reduction over columns (find.rs:180-270)
// keeps on a tie (the first, or the last when last_wins). 0: no candidate.
__device__ __forceinline__ unsigned long long cand_key(float g, uint32_t col, int last_wins) {
    if (g == 0.0f) g = 0.0f;  // -0 and +0 are the same gain
    uint32_t u = __float_as_uint(g);
    u = (u & 0x80000000u) ? ~u : (u | 0x80000000u);
    return ((unsigned long long)u << 32) | (last_wins ? col : ~col);
}

// Split finding of every node of the level (two children per expanding
// node) and the reduction over columns: each (node, column) warp posts its
// candidate's key to d.node_key[node]; the last block turns the winners into
// frontier b's splits (the winner's full candidate from cand), resets the
// keys, and derives the next level's decisions (rows in buffer buf).
template <typename HB>
__global__ void __launch_bounds__(SCAN_WARPS * 32, 4)
k_b_scan(BDev d, const ScanColumn* __restrict__ cols, uint32_t n_cols, const HB* __restrict__ hist,
         uint64_t slot_bins, const double* __restrict__ scale, GainParamsDev gp, ColCand* __restrict__ cand,
         long long* __restrict__ node_tot, int b, int last_wins, LeafParams lp, uint32_t buf,
         const ScanNode* __restrict__ root, const uint8_t* __restrict__ colmask, NodeSplit* __restrict__ lw_out) {
    BST_PDL_ENTER();
    __shared__ double s_key[SCAN_WARPS][SORT_N];
    __shared__ uint32_t s_cat[SCAN_WARPS][SORT_N];
    const int warp = threadIdx.x >> 5, lane = threadIdx.x & 31;
    const uint32_t n_nodes = root ? 1u : 2 * d.state->n_exp;
    const uint32_t col_blocks = (n_cols + SCAN_WARPS - 1) / SCAN_WARPS;
    const uint64_t items = (uint64_t)n_nodes * col_blocks;
    for (uint64_t it = blockIdx.x; it < items; it += gridDim.x) {
        const uint32_t node = (uint32_t)(it / col_blocks);
        const uint32_t col = (uint32_t)(it % col_blocks) * SCAN_WARPS + warp;
        if (col < n_cols) {
            const ScanNode nd = root ? root[0] : d.scan_nodes[node];
            const float g = scan_item(nd, node, col, cols, n_cols, hist, slot_bins, scale, gp, cand, node_tot,
                                      s_key[warp], s_cat[warp], colmask ? colmask + (size_t)nd.pad * n_cols : nullptr);
            if (lane == 0 && g > -INFINITY) atomicMax(&d.node_key[node], cand_key(g, col, last_wins));
        }
    }
    if (!last_block(d.state)) return;
    BNode* B = d.front[b];
    for (uint32_t node = threadIdx.x; node < n_nodes; node += blockDim.x) {
        const unsigned long long key = d.node_key[node];
        d.node_key[node] = 0ull;
        NodeSplit sp;
        sp.tot_g = node_tot[2 * node];
        sp.tot_h = node_tot[2 * node + 1];
        if (key == 0ull) {
            sp.gain = -INFINITY;
            sp.col = 0;
            sp.bin = 0;
            sp.flags = 0;
            sp.cats[0] = sp.cats[1] = sp.cats[2] = sp.cats[3] = 0ull;
        } else {
            const uint32_t col = last_wins ? (uint32_t)key : ~(uint32_t)key;
            const ColCand& w = cand[(size_t)node * n_cols + col];
            sp.gain = w.gain;
            sp.col = col;
            sp.bin = w.bin;
            sp.flags = (w.flags & 3u) | 4u;
            for (int q = 0; q < 4; ++q) sp.cats[q] = w.cats[q];
        }
        if (lw_out) {
            lw_out[node] = sp;
            continue;
        }
        B[node].split = sp;
        B[node].G = sp.tot_g;
        B[node].H = sp.tot_h;
    }
    if (lw_out) return;
    __syncthreads();
    decide_body(d, b, lp, scale, buf);
}

uint32_t scan_col_blocks(uint32_t n_cols) { return (n_cols + SCAN_WARPS - 1) / SCAN_WARPS; }

void launch_b_scan(const BDev& d, const ScanColumn* cols, uint32_t n_cols, const void* hist, uint64_t slot_bins,
                   const double* scale, GainParamsDev gp, ColCand* cand, long long* node_tot, int b, int last_wins,
                   LeafParams lp, uint32_t buf, uint32_t grid, cudaStream_t st, int hist32, const ScanNode* root,
                   const uint8_t* colmask, NodeSplit* lw_out) {
    if (hist32)
        launch_k(k_b_scan<HBin32>, grid, SCAN_WARPS * 32, 0, st, d, cols, n_cols, static_cast<const HBin32*>(hist), slot_bins,
                                                           scale, gp, cand, node_tot, b, last_wins, lp, buf, root,
                                                           colmask, lw_out);
    else
        launch_k(k_b_scan<HBin>, grid, SCAN_WARPS * 32, 0, st, d, cols, n_cols, static_cast<const HBin*>(hist), slot_bins,
                                                         scale, gp, cand, node_tot, b, last_wins, lp, buf, root,
                                                         colmask, lw_out);
}

// This thread's share of the fixed-point sums of positions [start, start +
// len) of a row-id buffer: RANGE_ILP positions per step, all row ids loaded
// before any gradient element, so the dependent gathers overlap.
constexpr uint32_t RANGE_ILP = 8;
template <int MODE>
__device__ __forceinline__ void range_sums(uint32_t start, uint32_t len, const uint32_t* __restrict__ ridx,
                                           const GradLoad<MODE>& load, long long& ag, long long& ah) {
    for (uint32_t i0 = threadIdx.x; i0 < len; i0 += blockDim.x * RANGE_ILP) {
        uint32_t rows[RANGE_ILP];
#pragma unroll
        for (uint32_t u = 0; u < RANGE_ILP; ++u) {
            const uint32_t i = i0 + u * blockDim.x;
            rows[u] = i < len ? ridx[start + i] : 0u;
        }
#pragma unroll
        for (uint32_t u = 0; u < RANGE_ILP; ++u) {
            const uint32_t i = i0 + u * blockDim.x;
            if (i < len) {
                long long qg, qh;
                load.at(start + i, rows[u], qg, qh);
                ag += qg;
                ah += qh;
            }
        }
    }
}

__device__ void children_sums_body(BDev d, int b);
__device__ void finalize_body(BDev d, int a, LeafParams lp, const double* __restrict__ scale, uint32_t buf);

// Node sums of the smaller children when the children are not split further
// (d.sums zeroed by the partition's last block); the last block then gives
// both children of every expansion their sums (frontier b).
template <int MODE>
__global__ void k_b_sums(BDev d, const uint32_t* __restrict__ ridx, GradRef gr, int b, int finalize, LeafParams lp,
                         const double* __restrict__ scale, uint32_t buf) {
    BST_PDL_ENTER();
    const uint32_t total = d.state->hist_chunks, CH = d.state->hist_chunk;
    const GradLoad<MODE> load(gr);
    for (uint32_t c = blockIdx.x; c < total; c += gridDim.x) {
        const uint32_t j = d.seg_exp[c];
        const BExp e = d.exp[j];
        const uint32_t start = e.small_begin + (c - e.hist_off) * CH;
        const uint32_t len = min(CH, e.small_begin + e.small_count - start);
        long long ag = 0, ah = 0;
        range_sums(start, len, ridx, load, ag, ah);
        for (int o = 16; o > 0; o >>= 1) {
            ag += __shfl_xor_sync(FULL, ag, o);
            ah += __shfl_xor_sync(FULL, ah, o);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(reinterpret_cast<unsigned long long*>(&d.sums[2 * j]), (unsigned long long)ag);
            atomicAdd(reinterpret_cast<unsigned long long*>(&d.sums[2 * j + 1]), (unsigned long long)ah);
        }
    }
    if (!last_block(d.state)) return;
    children_sums_body(d, b);
    if (finalize) {  // the tree's leaves (k_b_finalize) in the same block
        __syncthreads();
        finalize_body(d, b, lp, scale, buf);
    }
}

void launch_b_sums(const BDev& d, const uint32_t* ridx, const GradRef& gr, int b, uint32_t grid, cudaStream_t st,
                   int finalize, LeafParams lp, const double* scale, uint32_t buf) {
    if (gr.mode == GRAD_Q16)
        launch_k(k_b_sums<GRAD_Q16>, grid, 256, 0, st, d, ridx, gr, b, finalize, lp, scale, buf);
    else if (gr.mode == GRAD_Q8)
        launch_k(k_b_sums<GRAD_Q8>, grid, 256, 0, st, d, ridx, gr, b, finalize, lp, scale, buf);
    else
        launch_k(k_b_sums<GRAD_F32>, grid, 256, 0, st, d, ridx, gr, b, finalize, lp, scale, buf);
}

__device__ void children_sums_body(BDev d, int b) {
    const uint32_t n_exp = d.state->n_exp;
    const BNode* A = d.front[b ^ 1];
    BNode* B = d.front[b];
    for (uint32_t j = threadIdx.x; j < n_exp; j += blockDim.x) {
        const BExp e = d.exp[j];
        const BNode p = A[e.front];
        const long long sg = d.sums[2 * j], sh = d.sums[2 * j + 1];
        const bool left_small = e.lc <= e.rc;
        const long long lg = left_small ? sg : p.G - sg, lh = left_small ? sh : p.H - sh;
        B[2 * j].G = lg;
        B[2 * j].H = lh;
        B[2 * j + 1].G = p.G - lg;
        B[2 * j + 1].H = p.H - lh;
    }
}


// Remaining frontier -> leaves (grower.rs:484-514); leaf row chunks.
__device__ void finalize_body(BDev d, int a, LeafParams lp, const double* __restrict__ scale, uint32_t buf) {
    __shared__ uint32_t sh[33];
    __shared__ uint32_t s_jc[1024], s_own[1024], s_begin[1024];
    __shared__ uint32_t base, nf, n0;
    BState* s = d.state;
    if (threadIdx.x == 0) {
        nf = s->n_front;
        n0 = s->n_leaves;
        base = 0;
    }
    __syncthreads();
    const BNode* A = d.front[a];
    for (uint32_t i = threadIdx.x; i < nf; i += blockDim.x) {
        const BNode nd = A[i];
        const float v = leaf_value_dev(nd.G, nd.H, scale, lp);
        write_leaf(d.tree[nd.tnode], nd.G, nd.H, scale, v);
        BLeaf lf;
        lf.begin = nd.begin;
        lf.count = nd.count;
        lf.value = v;
        lf.tnode = nd.tnode;
        lf.chunk_off = 0;
        lf.buf = buf;
        d.leaves[n0 + i] = lf;
    }
    __syncthreads();
    const uint32_t nl = n0 + nf;
    for (uint32_t l0 = 0; l0 < nl; l0 += blockDim.x) {
        const uint32_t l = l0 + threadIdx.x;
        const uint32_t begin = l < nl ? d.leaves[l].begin : 0u;
        const uint32_t nch = l < nl ? (d.leaves[l].count + B_LEAF_CHUNK - 1) / B_LEAF_CHUNK : 0u;
        uint32_t tc;
        const uint32_t jc = block_excl_scan(nch, sh, &tc);
        if (l < nl) d.leaves[l].chunk_off = base + jc;
        // chunk -> (leaf, first row)
        write_chunk_owners(d.leaf_map, d.max_leaf_chunks, base, jc, l, begin, B_LEAF_CHUNK, tc, s_jc, s_own, s_begin);
        __syncthreads();
        if (threadIdx.x == 0) base += tc;
        __syncthreads();
    }
    // the quantised forms' leaf sums (k_b_leaf_sums) accumulate from zero
    for (uint32_t i = threadIdx.x; i < 2 * nl; i += blockDim.x) d.sums[i] = 0;
    if (threadIdx.x == 0) {
        s->n_leaves = nl;
        s->leaf_chunks = base < d.max_leaf_chunks ? base : d.max_leaf_chunks;
        s->n_front = 0;
    }
}

__global__ void __launch_bounds__(1024) k_b_finalize(BDev d, int a, LeafParams lp, const double* __restrict__ scale,
                                                    uint32_t buf) {
    BST_PDL_ENTER();
    finalize_body(d, a, lp, scale, buf);
}

void launch_b_finalize(const BDev& d, int a, LeafParams lp, const double* scale, uint32_t buf, cudaStream_t st) {
    launch_k(k_b_finalize, 1, 1024, 0, st, d, a, lp, scale, buf);
}

__device__ void leaf_values_body(BDev d, LeafParams lp, const double* __restrict__ scale);

// Quantised training: every leaf is solved from the exact fixed-point sums
// of the f32 gradients over its rows (d.sums[leaf][2], zeroed by
// k_b_finalize); the last block solves the leaf values (scale: the f32
// gradients' fixed-point scales).
__global__ void k_b_leaf_sums(BDev d, const uint32_t* __restrict__ r0, const uint32_t* __restrict__ r1, GradRef gr,
                              LeafParams lp, const double* __restrict__ scale) {
    BST_PDL_ENTER();
    const uint32_t total = d.state->leaf_chunks;
    const GradLoad<GRAD_F32> load(gr);
    for (uint32_t c = blockIdx.x; c < total; c += gridDim.x) {
        const uint2 m = d.leaf_map[c];
        const uint32_t l = m.x, start = m.y;
        const BLeaf lf = d.leaves[l];
        const uint32_t len = min(B_LEAF_CHUNK, lf.begin + lf.count - start);
        const uint32_t* ridx = lf.buf ? r1 : r0;
        long long ag = 0, ah = 0;
        range_sums(start, len, ridx, load, ag, ah);
        for (int o = 16; o > 0; o >>= 1) {
            ag += __shfl_xor_sync(FULL, ag, o);
            ah += __shfl_xor_sync(FULL, ah, o);
        }
        if ((threadIdx.x & 31) == 0) {
            atomicAdd(reinterpret_cast<unsigned long long*>(&d.sums[2 * l]), (unsigned long long)ag);
            atomicAdd(reinterpret_cast<unsigned long long*>(&d.sums[2 * l + 1]), (unsigned long long)ah);
        }
    }
    if (last_block(d.state)) leaf_values_body(d, lp, scale);
}

void launch_b_leaf_sums(const BDev& d, const uint32_t* r0, const uint32_t* r1, const GradRef& gr, LeafParams lp,
                        const double* scale, uint32_t grid, cudaStream_t st) {
    launch_k(k_b_leaf_sums, grid, 256, 0, st, d, r0, r1, gr, lp, scale);
}

__device__ void leaf_values_body(BDev d, LeafParams lp, const double* __restrict__ scale) {
    const uint32_t nl = d.state->n_leaves;
    for (uint32_t l = threadIdx.x; l < nl; l += blockDim.x) {
        const long long G = d.sums[2 * l], H = d.sums[2 * l + 1];
        const float v = leaf_value_dev(G, H, scale, lp);
        d.leaves[l].value = v;
        write_leaf(d.tree[d.leaves[l].tnode], G, H, scale, v);
    }
}

// pred[row] += leaf value over the final partition (grower.rs:208-219).
__global__ void k_b_leaf_update(BDev d, const uint32_t* __restrict__ r0, const uint32_t* __restrict__ r1,
                                float* __restrict__ pred, uint32_t* __restrict__ row_leaf) {
    BST_PDL_ENTER();
    const uint32_t total = d.state->leaf_chunks;
    for (uint32_t c = blockIdx.x; c < total; c += gridDim.x) {
        const uint2 m = d.leaf_map[c];
        if (!BST_IN(m.x, d.state->n_leaves, CHECK_LEAF_MAP)) continue;
        const BLeaf lf = d.leaves[m.x];
        const uint32_t start = m.y;
        const uint32_t len = min(B_LEAF_CHUNK, lf.begin + lf.count - start);
        const uint32_t* ridx = lf.buf ? r1 : r0;
        // RANGE_ILP rows per step: row ids, then predictions, then stores
        // (a leaf's rows are distinct, so the steps do not alias)
        for (uint32_t i0 = threadIdx.x; i0 < len; i0 += blockDim.x * RANGE_ILP) {
            uint32_t rows[RANGE_ILP];
            float pv[RANGE_ILP];
#pragma unroll
            for (uint32_t u = 0; u < RANGE_ILP; ++u) {
                const uint32_t i = i0 + u * blockDim.x;
                rows[u] = i < len ? ridx[start + i] : 0u;
#ifdef BST_CHECKED
                if (i < len && !BST_IN(rows[u], d.chk_rows, CHECK_LEAF_ROW)) rows[u] = 0u;
#endif
            }
#pragma unroll
            for (uint32_t u = 0; u < RANGE_ILP; ++u)
                pv[u] = i0 + u * blockDim.x < len ? pred[rows[u]] : 0.0f;
#pragma unroll
            for (uint32_t u = 0; u < RANGE_ILP; ++u)
                if (i0 + u * blockDim.x < len) {
                    pred[rows[u]] = pv[u] + lf.value;
                    if (row_leaf) row_leaf[rows[u]] = lf.tnode;
                }
        }
    }
}

void launch_b_leaf_update(const BDev& d, const uint32_t* r0, const uint32_t* r1, float* pred, uint32_t* row_leaf,
                          uint32_t grid, cudaStream_t st) {
    launch_k(k_b_leaf_update, grid, 256, 0, st, d, r0, r1, pred, row_leaf);
}

// ============================================================================
// Leaf renewing for the L1 and pinball losses (objectives/mod.rs:352-409)
// ============================================================================

namespace {

constexpr uint32_t RENEW_NONE = 0xFFFFFFFFu;

// Orderable key of a residual: unsigned order = value order; -0 counts as 0.
__device__ __forceinline__ uint32_t renew_key(float r) {
    if (r == 0.0f) r = 0.0f;
    const uint32_t u = __float_as_uint(r);
    return (u & 0x80000000u) ? ~u : (u | 0x80000000u);
}
__device__ __forceinline__ float renew_value(uint32_t k) {
    return __uint_as_float((k & 0x80000000u) ? (k & 0x7FFFFFFFu) : ~k);
}

__device__ __forceinline__ bool renew_sampled(const uint8_t* rmask, uint32_t row) { return !rmask || rmask[row]; }

__device__ __forceinline__ void renew_set(const BDev& d, uint32_t l, float v) {
    d.leaves[l].value = v;
    if (d.tree) d.tree[d.leaves[l].tnode].leaf = v;
}

}  // namespace

__global__ void k_renew_start(BDev d, RenewDev r) {
    BST_PDL_ENTER();
    const uint32_t nl = min(d.state->n_leaves, r.cap);
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < (uint64_t)nl * 256u;
         i += (uint64_t)gridDim.x * blockDim.x) {
        r.hist[i] = 0u;
        if (i < nl) r.cnt[i] = 0u;
    }
}

// Sampled rows per leaf: one block per leaf chunk, one atomic per block.
__global__ void k_renew_count(BDev d, RenewDev r, const uint32_t* __restrict__ r0, const uint32_t* __restrict__ r1) {
    BST_PDL_ENTER();
    __shared__ uint32_t s_cnt;
    const uint32_t total = d.state->leaf_chunks;
    for (uint32_t c = blockIdx.x; c < total; c += gridDim.x) {
        const uint2 m = d.leaf_map[c];
        if (m.x >= r.cap) continue;  // block-uniform
        const BLeaf lf = d.leaves[m.x];
        const uint32_t len = min(B_LEAF_CHUNK, lf.begin + lf.count - m.y);
        const uint32_t* ridx = lf.buf ? r1 : r0;
        if (threadIdx.x == 0) s_cnt = 0;
        __syncthreads();
        uint32_t k = 0;
        for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) k += renew_sampled(d.rmask, ridx[m.y + i]) ? 1u : 0u;
        for (int o = 16; o > 0; o >>= 1) k += __shfl_xor_sync(FULL, k, o);
        if ((threadIdx.x & 31) == 0 && k) atomicAdd(&s_cnt, k);
        __syncthreads();
        if (threadIdx.x == 0 && s_cnt) atomicAdd(&r.cnt[m.x], s_cnt);
        __syncthreads();
    }
}

// The rank to find: ceil(alpha m) - 1 clamped to [0, m - 1] (f32 product,
// utils.rs:42-44); none for an empty leaf.
__global__ void k_renew_rank(BDev d, RenewDev r, float alpha) {
    BST_PDL_ENTER();
    const uint32_t nl = min(d.state->n_leaves, r.cap);
    for (uint32_t l = blockIdx.x * blockDim.x + threadIdx.x; l < nl; l += gridDim.x * blockDim.x) {
        const uint32_t m = r.cnt[l];
        uint32_t k = RENEW_NONE;
        if (m > 0) {
            const float c = ceilf(alpha * (float)m);
            uint64_t kk = c > 0.0f ? (uint64_t)c : 0u;
            kk = kk > 0 ? kk - 1 : 0;
            k = (uint32_t)(kk < m - 1 ? kk : m - 1);
        }
        r.rank[l] = k;
        r.prefix[l] = 0u;
    }
}

// One radix-select pass: counts of the key byte at `shift` among the
// sampled rows whose higher bytes match the prefix.
__global__ void k_renew_hist(BDev d, RenewDev r, const uint32_t* __restrict__ r0, const uint32_t* __restrict__ r1,
                             const float* __restrict__ y, const float* __restrict__ pred, uint32_t shift) {
    BST_PDL_ENTER();
    __shared__ uint32_t sh[256];
    const uint32_t total = d.state->leaf_chunks;
    const uint32_t hi_mask = shift >= 24 ? 0u : (0xFFFFFFFFu << (shift + 8));
    for (uint32_t c = blockIdx.x; c < total; c += gridDim.x) {
        const uint2 m = d.leaf_map[c];
        if (m.x >= r.cap || r.rank[m.x] == RENEW_NONE) continue;  // block-uniform
        const BLeaf lf = d.leaves[m.x];
        const uint32_t len = min(B_LEAF_CHUNK, lf.begin + lf.count - m.y);
        const uint32_t* ridx = lf.buf ? r1 : r0;
        const uint32_t want = r.prefix[m.x] & hi_mask;
        for (uint32_t b = threadIdx.x; b < 256; b += blockDim.x) sh[b] = 0u;
        __syncthreads();
        for (uint32_t i = threadIdx.x; i < len; i += blockDim.x) {
            const uint32_t row = ridx[m.y + i];
            if (!renew_sampled(d.rmask, row)) continue;
            const uint32_t k = renew_key(y[row] - pred[row]);
            if ((k & hi_mask) == want) atomicAdd(&sh[(k >> shift) & 255u], 1u);
        }
        __syncthreads();
        uint32_t* h = r.hist + (size_t)m.x * 256u;
        for (uint32_t b = threadIdx.x; b < 256; b += blockDim.x)
            if (sh[b]) atomicAdd(&h[b], sh[b]);
        __syncthreads();
    }
}

// The byte of the wanted rank (one warp per leaf; lane j owns bytes 8j ..
// 8j + 7), then the counts cleared for the next pass.
__global__ void k_renew_pick(BDev d, RenewDev r, uint32_t shift) {
    BST_PDL_ENTER();
    const uint32_t nl = min(d.state->n_leaves, r.cap);
    const uint32_t lane = threadIdx.x & 31u, wpb = blockDim.x >> 5;
    for (uint32_t l = blockIdx.x * wpb + (threadIdx.x >> 5); l < nl; l += gridDim.x * wpb) {
        const uint32_t k = r.rank[l];
        if (k == RENEW_NONE) continue;  // warp-uniform
        uint32_t* h = r.hist + (size_t)l * 256u;
        uint32_t c[8], sum = 0;
#pragma unroll
        for (int q = 0; q < 8; ++q) {
            c[q] = h[lane * 8 + q];
            sum += c[q];
        }
        uint32_t incl = sum;
        for (int o = 1; o < 32; o <<= 1) {
            const uint32_t t = __shfl_up_sync(FULL, incl, o);
            if (lane >= (uint32_t)o) incl += t;
        }
        const uint32_t excl = incl - sum;
        // the lane whose bytes hold rank k: excl <= k < incl
        const unsigned owner = __ballot_sync(FULL, excl <= k && k < incl);
        if (owner) {
            const uint32_t src = (uint32_t)(__ffs(owner) - 1);
            if (lane == src) {
                uint32_t before = excl, b = 0;
#pragma unroll
                for (int q = 0; q < 8; ++q)
                    if (before + c[q] <= k) {
                        before += c[q];
                        b = (uint32_t)q + 1u;
                    } else {
                        break;
                    }
                r.prefix[l] |= ((lane * 8u + b) & 255u) << shift;
                r.rank[l] = k - before;
            }
        }
        __syncwarp();
#pragma unroll
        for (int q = 0; q < 8; ++q) h[lane * 8 + q] = 0u;
    }
}

__global__ void k_renew_apply(BDev d, RenewDev r, float lr) {
    BST_PDL_ENTER();
    const uint32_t nl = min(d.state->n_leaves, r.cap);
    for (uint32_t l = blockIdx.x * blockDim.x + threadIdx.x; l < nl; l += gridDim.x * blockDim.x)
        if (r.rank[l] != RENEW_NONE) renew_set(d, l, renew_value(r.prefix[l]) * lr);
}

// Weighted form: one block per leaf. The reference's partition is stable,
// so a leaf's rows are in ascending row order there; here they are in
// partition-chunk order. The leaf's sampled rows are compacted into key[0]
// / row[0] at the leaf's own positions (its range in the row buffer),
// sorted by row id (stable one-bit passes over the id's bits), their
// weights summed in that order, sorted stably by key (32 more passes, so
// equal keys stay in row order) and the running weight scanned.
constexpr uint32_t RENEW_W_THREADS = 1024;

// One stable split pass of a leaf's (key, row) pairs from buffer src to
// src ^ 1 by bit b of the key (or of the row id): zeros first, each side in
// its order.
__device__ void renew_split_pass(const RenewDev& r, uint32_t src, uint32_t first, uint32_t m, uint32_t b,
                                 bool by_row, uint32_t* sh, uint32_t* s_zero, uint32_t* s_base) {
    const uint32_t* ks = r.key[src] + first;
    const uint32_t* rs = r.row[src] + first;
    uint32_t* kd = r.key[src ^ 1u] + first;
    uint32_t* rd = r.row[src ^ 1u] + first;
    if (threadIdx.x == 0) *s_zero = 0;
    __syncthreads();
    uint32_t z = 0;
    for (uint32_t i = threadIdx.x; i < m; i += blockDim.x) z += (((by_row ? rs[i] : ks[i]) >> b) & 1u) ? 0u : 1u;
    for (int o = 16; o > 0; o >>= 1) z += __shfl_xor_sync(FULL, z, o);
    if ((threadIdx.x & 31) == 0 && z) atomicAdd(s_zero, z);
    if (threadIdx.x == 0) *s_base = 0;
    __syncthreads();
    const uint32_t zeros = *s_zero;
    for (uint32_t t0 = 0; t0 < m; t0 += blockDim.x) {
        const uint32_t i = t0 + threadIdx.x;
        const bool valid = i < m;
        const uint32_t k = valid ? ks[i] : 0u, row = valid ? rs[i] : 0u;
        const bool zero = valid && !(((by_row ? row : k) >> b) & 1u);
        uint32_t tz;
        const uint32_t rz = block_excl_scan(zero ? 1u : 0u, sh, &tz);
        const uint32_t base = *s_base;
        if (valid) {
            // ones before this one: (t0 - base) in earlier tiles, i - t0 - rz in this one
            const uint32_t dst = zero ? base + rz : zeros + (t0 - base) + (i - t0 - rz);
            kd[dst] = k;
            rd[dst] = row;
        }
        __syncthreads();
        if (threadIdx.x == 0) *s_base += tz;
        __syncthreads();
    }
}

__global__ void __launch_bounds__(RENEW_W_THREADS)
k_renew_weighted(BDev d, RenewDev r, const uint32_t* __restrict__ r0, const uint32_t* __restrict__ r1,
                 const float* __restrict__ y, const float* __restrict__ pred, const float* __restrict__ w, float alpha,
                 float lr) {
    BST_PDL_ENTER();
    __shared__ uint32_t sh[33];
    __shared__ float s_w[RENEW_W_THREADS];
    __shared__ uint32_t s_base, s_zero, s_hit;
    __shared__ float s_acc;
    const uint32_t nl = min(d.state->n_leaves, r.cap);
    for (uint32_t l = blockIdx.x; l < nl; l += gridDim.x) {
        const BLeaf lf = d.leaves[l];
        const uint32_t* ridx = lf.buf ? r1 : r0;
        const uint32_t first = lf.begin;  // the leaf's own range in the scratch arrays
        // 1. compaction (stable) of the sampled rows
        if (threadIdx.x == 0) s_base = 0;
        __syncthreads();
        for (uint32_t t0 = 0; t0 < lf.count; t0 += blockDim.x) {
            const uint32_t i = t0 + threadIdx.x;
            const uint32_t row = i < lf.count ? ridx[first + i] : 0u;
            const bool keep = i < lf.count && renew_sampled(d.rmask, row);
            uint32_t tot;
            const uint32_t off = s_base + block_excl_scan(keep ? 1u : 0u, sh, &tot);
            if (keep) {
                r.key[0][first + off] = renew_key(y[row] - pred[row]);
                r.row[0][first + off] = row;
            }
            __syncthreads();
            if (threadIdx.x == 0) s_base += tot;
            __syncthreads();
        }
        const uint32_t m = s_base;
        __syncthreads();
        if (m == 0) continue;  // block-uniform
        // 2. row order (the reference's partition order), then the f32 total
        // of the weights in that order
        uint32_t src = 0;
        const uint32_t row_bits = 32u - (uint32_t)__clz(max(r.n_rows, 2u) - 1u);  // row ids < n_rows
        for (uint32_t b = 0; b < row_bits; ++b) {
            renew_split_pass(r, src, first, m, b, true, sh, &s_zero, &s_base);
            src ^= 1u;
        }
        if (threadIdx.x == 0) s_acc = 0.0f;
        for (uint32_t t0 = 0; t0 < m; t0 += blockDim.x) {
            const uint32_t i = t0 + threadIdx.x;
            __syncthreads();
            s_w[threadIdx.x] = i < m ? w[r.row[src][first + i]] : 0.0f;
            __syncthreads();
            if (threadIdx.x == 0) {
                float acc = s_acc;
                const uint32_t e = min(m - t0, (uint32_t)blockDim.x);
                for (uint32_t q = 0; q < e; ++q) acc += s_w[q];
                s_acc = acc;
            }
        }
        __syncthreads();
        const float threshold = s_acc * alpha;
        // 3. stable sort by key: zeros of bit b first, each side in order
        for (uint32_t b = 0; b < 32; ++b) {
            renew_split_pass(r, src, first, m, b, false, sh, &s_zero, &s_base);
            src ^= 1u;
        }
        // 4. the first sorted row whose running weight reaches the threshold
        if (threadIdx.x == 0) {
            s_acc = 0.0f;
            s_hit = RENEW_NONE;
        }
        for (uint32_t t0 = 0; t0 < m; t0 += blockDim.x) {
            const uint32_t i = t0 + threadIdx.x;
            __syncthreads();
            if (s_hit != RENEW_NONE) break;  // block-uniform
            s_w[threadIdx.x] = i < m ? w[r.row[src][first + i]] : 0.0f;
            __syncthreads();
            if (threadIdx.x == 0) {
                float acc = s_acc;
                const uint32_t e = min(m - t0, (uint32_t)blockDim.x);
                for (uint32_t q = 0; q < e; ++q) {
                    acc += s_w[q];
                    if (acc >= threshold) {
                        s_hit = t0 + q;
                        break;
                    }
                }
                s_acc = acc;
            }
        }
        __syncthreads();
        if (threadIdx.x == 0) {
            const uint32_t j = s_hit != RENEW_NONE ? s_hit : m - 1;
            renew_set(d, l, renew_value(r.key[src][first + j]) * lr);
        }
        __syncthreads();
    }
}

void launch_leaf_renew(const BDev& d, const RenewDev& r, const uint32_t* r0, const uint32_t* r1, const float* y,
                       const float* pred, const float* w, float alpha, float lr, uint32_t grid, cudaStream_t st) {
    if (w) {
        launch_k(k_renew_weighted, grid, RENEW_W_THREADS, 0, st, d, r, r0, r1, y, pred, w, alpha, lr);
        return;
    }
    launch_k(k_renew_start, grid, 256, 0, st, d, r);
    launch_k(k_renew_count, grid, 256, 0, st, d, r, r0, r1);
    launch_k(k_renew_rank, grid, 256, 0, st, d, r, alpha);
    for (int shift = 24; shift >= 0; shift -= 8) {
        launch_k(k_renew_hist, grid, 256, 0, st, d, r, r0, r1, y, pred, (uint32_t)shift);
        launch_k(k_renew_pick, grid, 256, 0, st, d, r, (uint32_t)shift);
    }
    launch_k(k_renew_apply, grid, 256, 0, st, d, r, lr);
}

// ============================================================================
// K9: forest traversal (tree_view.rs:119-160, predictor.rs:271-302)
// One thread per row; trees summed in forest order per group in f32.
// ============================================================================

__global__ void k_predict(ForestDev f, const float* __restrict__ x,
                          uint64_t n, uint32_t n_features, int feature_major, float* __restrict__ out) {
    BST_PDL_ENTER();
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (i >= n) return;
    const uint64_t fstride = feature_major ? n : 1;
    const float* xr = feature_major ? x + i : x + i * n_features;
    for (uint32_t g = 0; g < f.n_groups; ++g) {
        float acc = f.base[g];
        for (uint32_t k = f.group_off[g]; k < f.group_off[g + 1]; ++k) {
            uint32_t nd = f.roots[f.group_trees[k]];
            for (int step = 0; step < 65536; ++step) {
                const ForestNode fn = f.nodes[nd];
                if (fn.word >> 31) {
                    acc = acc + fn.value;
                    break;
                }
                const uint32_t feat = fn.word & 0x1FFFFFFFu;
                const float v = feat < n_features ? xr[(uint64_t)feat * fstride] : NAN;
                bool left;
                if (v != v) {
                    left = (fn.word >> 30) & 1u;
                } else if ((fn.word >> 29) & 1u) {
                    const uint32_t cat = sat_u32(v);
                    const uint32_t start = f.cat_seg[2 * nd], size = f.cat_seg[2 * nd + 1];
                    const uint32_t wi = cat >> 5;
                    const bool right = wi < size && ((f.cat_words[start + wi] >> (cat & 31)) & 1u);
                    left = !right;
                } else {
                    left = v < fn.value;
                }
                nd = left ? fn.left : fn.right;
#ifdef BST_CHECKED
                if (!BST_IN(nd, f.chk_nodes, CHECK_PREDICT_NODE)) break;
#endif
            }
        }
        out[(uint64_t)g * n + i] = acc;
    }
}

void launch_predict(const ForestDev& f, const float* x, uint64_t n, uint32_t n_features,
                    int feature_major, float* out, cudaStream_t st) {
    if (n == 0) return;
    launch_k(k_predict, (unsigned)((n + 127) / 128), 128, 0, st, f, x, n, n_features, feature_major, out);
}

// ---- shared-memory traversal (heap-ordered trees of depth <= HEAP_DEPTH) ------
// Two launches. k_bin_rows bins the rows against the forest's thresholds into
// tiles of R rows in global scratch, each tile's bin columns laid out as the
// traversal reads them from shared memory. k_predict_heap copies a tile's
// columns into shared memory (cp.async) and streams the trees of each output
// group through a double-buffered shared-memory ring of PREDICT_CHUNK trees;
// each thread walks its row through PREDICT_IL trees at a time as
// independent chains of exactly HEAP_DEPTH steps and sums the leaves in
// forest order (the same f32 additions as k_predict). The forest is read
// once per row tile from L2 instead of once per row.
//
// Bin columns are R entries long. Row r of a u8 column sits at byte
// (r / 128) * 128 + 4 * (r % 32) + (r / 32) % 4, of a u16 column at byte
// (r / 64) * 128 + 4 * (r % 32) + 2 * ((r / 32) % 2): with R a multiple of
// 128, lane l of any warp reads bank l whatever column each lane asks for,
// so the bin fetch of a step is one conflict-free wavefront; and one 32-bit
// word holds rows r, r + 32 (, r + 64, r + 96) of a column, so the binning
// pass writes whole 128-byte lines.
constexpr uint32_t PREDICT_CHUNK = 16;
constexpr uint32_t PREDICT_IL = 4;
constexpr uint32_t PREDICT_SMEM = 227u * 1024u;
constexpr uint32_t PREDICT_TREE_BYTES = HEAP_NODES * 4u;
constexpr uint32_t PREDICT_RING = 2u * PREDICT_CHUNK * PREDICT_TREE_BYTES;
constexpr uint32_t PREDICT_MAX_ROWS = PREDICT_TILE_MAX;
constexpr uint32_t PREDICT_MIN_ROWS = 128;
constexpr uint32_t PREDICT_SPL_MAX_F = 256;  // splitter table in shared memory up to this many features
constexpr uint32_t BIN_NAN = 0xFFFFu;
constexpr uint32_t BIN_THREADS = 256;         // binning pass: 8 warps per block
constexpr uint32_t BIN_F = 8;                 // features staged per step of the binning pass
constexpr uint32_t BIN_XS_LD = BIN_F + 1;     // floats per staged row: odd stride

__host__ __device__ inline uint32_t predict_spl_floats(uint32_t NF) {
    return NF <= PREDICT_SPL_MAX_F ? NF * HEAP_SPLITTERS : 0u;
}

// Launch shape of the traversal: R rows per tile, the trees of each chunk
// split over S thread groups of R threads (S > 1 for small batches: each
// group walks its share of the chunk's trees and leaves the values in
// shared memory, where the row's group-0 thread adds them in forest order).
struct HeapPlan {
    uint32_t R = 0, S = 1;
    size_t smem = 0, col_bytes = 0;  // col_bytes: one tile's bin columns
};

static HeapPlan heap_plan(const HeapForest& f, uint32_t F, uint64_t n) {
    HeapPlan p;
    if (F == 0 || f.n_cols == 0 || f.n_cols > HEAP_MAX_COLS) return p;
    const uint64_t per_row = (uint64_t)f.n_cols * (f.bins16 ? 2u : 1u);
    if (PREDICT_RING + per_row * PREDICT_MIN_ROWS > PREDICT_SMEM) return p;
    uint64_t rmax = (PREDICT_SMEM - PREDICT_RING) / per_row;
    if (rmax > PREDICT_MAX_ROWS) rmax = PREDICT_MAX_ROWS;
    rmax &= ~(uint64_t)(PREDICT_MIN_ROWS - 1);
    // whole waves of one tile per SM: as few waves as the largest tile allows, the
    // rows spread evenly over them (a small batch over every SM)
    const uint64_t waves = n ? (n + sm_count() * rmax - 1) / (sm_count() * rmax) : 1;
    uint64_t r = (n + sm_count() * waves - 1) / (sm_count() * waves);
    r = (r + PREDICT_MIN_ROWS - 1) / PREDICT_MIN_ROWS * PREDICT_MIN_ROWS;
    if (r < PREDICT_MIN_ROWS) r = PREDICT_MIN_ROWS;
    if (r > rmax) r = rmax;
    uint32_t S = r <= 128 ? 4u : (r <= 384 ? 2u : 1u);
    if (S > 1 && PREDICT_RING + r * (per_row + PREDICT_CHUNK * 4u) > PREDICT_SMEM) S = 1;
    p.R = (uint32_t)r;
    p.S = S;
    p.col_bytes = (size_t)r * per_row;
    p.smem = PREDICT_RING + (S > 1 ? (size_t)PREDICT_CHUNK * 4u * r : 0) + p.col_bytes;
    return p;
}

uint32_t predict_heap_rows(const HeapForest& f, uint32_t F, uint64_t n) { return heap_plan(f, F, n).R; }

size_t predict_heap_scratch(const HeapForest& f, uint32_t F, uint64_t n) {
    const HeapPlan p = heap_plan(f, F, n);
    return p.R ? (size_t)((n + p.R - 1) / p.R) * p.col_bytes : 0;
}

size_t predict_heap_scratch_max(const HeapForest& f, uint32_t F, uint64_t n_max) {
    return (size_t)(n_max + PREDICT_MAX_ROWS) * f.n_cols * (f.bins16 ? 2u : 1u);
}

__device__ __forceinline__ void cp_async16(void* dst, const void* src) {
    const uint32_t d = (uint32_t)__cvta_generic_to_shared(dst);
    asm volatile("cp.async.cg.shared.global [%0], [%1], 16;" ::"r"(d), "l"(src) : "memory");
}

// Bin of v for one numeric feature (see HeapForest) once the splitters have
// picked block c: lb branchless steps count the block's first blk - 1
// entries <= v, one more compare the last. NaN padding is never <= v, so no
// search leaves the feature's blocks.
__device__ __forceinline__ uint32_t heap_bin_block(const float* __restrict__ t, uint32_t lb, uint32_t c, float v) {
    uint32_t k = c << lb;  // block start
    for (uint32_t s = (1u << lb) >> 1; s >= 1u; s >>= 1) k += t[k + s - 1] <= v ? s : 0u;
    return k + (t[k] <= v ? 1u : 0u);
}

// Binning pass: one warp bins 32 * RPL rows (lane l: rows l + 32 i), all
// features, PREDICT_BIN_F at a time staged through shared memory (coalesced
// loads), into the tile layout; the RPL rows of a lane fill one 32-bit word
// per column.
template <typename BinT>
__global__ void __launch_bounds__(BIN_THREADS)
k_bin_rows(HeapForest f, const float* __restrict__ x, uint64_t n, uint32_t F, uint32_t R, uint32_t FC,
           uint32_t* __restrict__ bins_g) {
    BST_PDL_ENTER();
    constexpr uint32_t RPL = 4u / (uint32_t)sizeof(BinT);
    constexpr uint32_t WR = 32u * RPL;  // rows per warp
    constexpr uint32_t BITS = 8u * (uint32_t)sizeof(BinT);
    extern __shared__ __align__(16) float bsm[];
    const uint32_t tid = threadIdx.x, lane = tid & 31u, warp = tid >> 5, nwarps = BIN_THREADS / 32u;
    const uint32_t NF = F < f.n_features ? F : f.n_features;
    const uint32_t spl_n = predict_spl_floats(NF);
    float* spl = bsm;
    float* xs = bsm + spl_n + (size_t)warp * WR * BIN_XS_LD;
    for (uint32_t i = tid; i < spl_n; i += BIN_THREADS) spl[i] = f.spl[i];
    __syncthreads();
    const uint32_t col_words = R * (uint32_t)sizeof(BinT) / 4u;
    const uint64_t n_groups = (n + WR - 1) / WR;
    const uint32_t n_fc = (NF + FC - 1) / FC;  // feature chunks: more warps for a small batch
    const uint64_t items = n_groups * n_fc;
    for (uint64_t it = (uint64_t)blockIdx.x * nwarps + warp; it < items; it += (uint64_t)gridDim.x * nwarps) {
        const uint64_t gi = it / n_fc;
        const uint32_t f0 = (uint32_t)(it - gi * n_fc) * FC, f1 = f0 + FC < NF ? f0 + FC : NF;
        const uint64_t row0 = gi * WR;
        const uint64_t tile = row0 / R;
        const uint32_t rg0 = (uint32_t)(row0 - tile * R);  // a multiple of WR
        const uint32_t nr = (uint32_t)(n - row0 < WR ? n - row0 : WR);
        uint32_t* tw = bins_g + (size_t)tile * f.n_cols * col_words + (rg0 / WR) * 32u + lane;
        for (uint32_t fg = f0; fg < f1; fg += BIN_F) {
            const uint32_t fj = fg + lane % BIN_F;
#pragma unroll 8
            for (uint32_t k = 0; k < WR * BIN_F / 32u; ++k) {
                const uint32_t row = lane / BIN_F + k * (32u / BIN_F);
                xs[row * BIN_XS_LD + lane % BIN_F] = row < nr && fj < f1 ? x[(row0 + row) * F + fj] : 0.0f;
            }
            __syncwarp();
            const uint32_t nf = f1 - fg < BIN_F ? f1 - fg : BIN_F;
            for (uint32_t j = 0; j < nf; ++j) {
                const uint32_t ft = fg + j;  // the same feature in every lane
                const int32_t c0 = f.feat_col[2 * ft], c1 = f.feat_col[2 * ft + 1];
                if (c0 < 0 && c1 < 0) continue;
                const uint32_t info = f.feat_info[ft];
                const uint32_t lb = info & 31u;
                const float* sp = spl_n ? spl + ft * HEAP_SPLITTERS : f.spl + (size_t)ft * HEAP_SPLITTERS;
                const float* t = f.thr + f.thr_off[ft];
                float v[RPL];
                uint32_t b[RPL];
#pragma unroll
                for (uint32_t i = 0; i < RPL; ++i) {
                    v[i] = xs[(lane + 32u * i) * BIN_XS_LD + j];
                    b[i] = 0;
                }
                if (!(info >> 7)) {
#pragma unroll
                    for (uint32_t s = HEAP_SPLITTERS / 2; s >= 1; s >>= 1) {
#pragma unroll
                        for (uint32_t i = 0; i < RPL; ++i) b[i] += sp[b[i] + s - 1] <= v[i] ? s : 0u;
                    }
                    if (lb == 4) {  // 16-entry blocks: fixed steps, the rows interleaved
#pragma unroll
                        for (uint32_t i = 0; i < RPL; ++i) b[i] <<= 4;
#pragma unroll
                        for (uint32_t s = 8; s >= 1; s >>= 1) {
#pragma unroll
                            for (uint32_t i = 0; i < RPL; ++i) b[i] += t[b[i] + s - 1] <= v[i] ? s : 0u;
                        }
#pragma unroll
                        for (uint32_t i = 0; i < RPL; ++i) b[i] += t[b[i]] <= v[i] ? 1u : 0u;
                    } else {
#pragma unroll
                        for (uint32_t i = 0; i < RPL; ++i) b[i] = heap_bin_block(t, lb, b[i], v[i]);
                    }
                }
                uint32_t w0 = 0, w1 = 0;
#pragma unroll
                for (uint32_t i = 0; i < RPL; ++i) {
                    uint32_t bb = b[i];
                    if (v[i] != v[i]) {
                        bb = BIN_NAN;
                    } else if (info >> 7) {
                        const uint32_t cv = sat_u32(v[i]);
                        bb = cv < 65534u ? cv : 65534u;
                    }
                    const uint32_t mask = (1u << BITS) - 1u;  // NaN: largest bin / 0
                    w0 |= (bb == BIN_NAN ? mask : bb & mask) << (BITS * i);
                    w1 |= (bb == BIN_NAN ? 0u : bb & mask) << (BITS * i);
                }
                if (c0 >= 0) tw[(size_t)c0 * col_words] = w0;
                if (c1 >= 0) tw[(size_t)c1 * col_words] = w1;
            }
            __syncwarp();
        }
    }
}

// One split step: from heap position h of tree to its chosen child. cb: this
// thread's row in bin column 0 (byte address); Rb: column stride in bytes.
template <bool CAT, typename BinT>
__device__ __forceinline__ uint32_t heap_step(const uint32_t* tree, const unsigned char* cb, uint32_t Rb,
                                              const HeapForest& f, uint32_t h) {
    const uint32_t w = tree[h];
    const uint32_t b = *reinterpret_cast<const BinT*>(cb + (w & 0x7FFFu) * Rb);
    bool left;
    if (CAT && (w & 0x8000u)) {
        const uint2 cs = f.cat[w >> 16];
        if (b == BIN_NAN) {
            left = (cs.y >> 31) != 0u;
        } else {
            const uint32_t wi = b >> 5;
            left = !(wi < (cs.y & 0x7FFFFFFFu) && ((f.cat_words[cs.x + wi] >> (b & 31u)) & 1u));
        }
    } else {
        left = b * 65536u + 65535u < w;  // bin < K (K: the word's upper half)
    }
    return 2u * h + (left ? 0u : 1u);
}

// Leaf values of trees [q0, q1) of the chunk at tb for this thread's row,
// PREDICT_IL chains at a time; emit(q, value) in tree order.
template <bool CAT, typename BinT, typename Emit>
__device__ __forceinline__ void heap_walk(const uint32_t* tb, uint32_t q0, uint32_t q1, const unsigned char* cb,
                                          uint32_t Rb, const HeapForest& f, Emit emit) {
    uint32_t q = q0;
    for (; q + PREDICT_IL <= q1; q += PREDICT_IL) {
        uint32_t h[PREDICT_IL];
#pragma unroll
        for (uint32_t u = 0; u < PREDICT_IL; ++u) h[u] = 1u;
#pragma unroll
        for (int step = 0; step < HEAP_DEPTH; ++step) {
#pragma unroll
            for (uint32_t u = 0; u < PREDICT_IL; ++u) h[u] = heap_step<CAT, BinT>(tb + (q + u) * HEAP_NODES, cb, Rb, f, h[u]);
        }
#pragma unroll
        for (uint32_t u = 0; u < PREDICT_IL; ++u) emit(q + u, __uint_as_float(tb[(q + u) * HEAP_NODES + h[u]]));
    }
    for (; q < q1; ++q) {
        const uint32_t* t = tb + q * HEAP_NODES;
        uint32_t h1 = 1u;
#pragma unroll
        for (int step = 0; step < HEAP_DEPTH; ++step) h1 = heap_step<CAT, BinT>(t, cb, Rb, f, h1);
        emit(q, __uint_as_float(t[h1]));
    }
}

template <bool CAT, typename BinT>
__global__ void __launch_bounds__(PREDICT_MAX_ROWS, 1)
k_predict_heap(HeapForest f, const unsigned char* __restrict__ bins_g, uint64_t n, uint32_t R, uint32_t S,
               float* __restrict__ out) {
    BST_PDL_ENTER();
    extern __shared__ __align__(16) unsigned char smem_raw[];
    uint32_t* ring = reinterpret_cast<uint32_t*>(smem_raw);  // [2][PREDICT_CHUNK][HEAP_NODES]
    float* lv = reinterpret_cast<float*>(smem_raw + PREDICT_RING);  // [PREDICT_CHUNK][R] when S > 1
    unsigned char* bins = smem_raw + PREDICT_RING + (S > 1 ? PREDICT_CHUNK * 4u * R : 0u);
    const uint32_t tid = threadIdx.x, lane = tid & 31u;
    const uint32_t rg = tid % R, sg = tid / R;  // row in the tile, tree group
    const uint32_t Rb = R * (uint32_t)sizeof(BinT);
    const uint32_t col_bytes = f.n_cols * Rb;
    const uint32_t roff = sizeof(BinT) == 1 ? (rg >> 7) * 128u + 4u * lane + ((rg >> 5) & 3u)
                                            : (rg >> 6) * 128u + 4u * lane + 2u * ((rg >> 5) & 1u);
    const unsigned char* cb = bins + roff;
    const uint64_t n_tiles = (n + R - 1) / R;
    for (uint64_t tile = blockIdx.x; tile < n_tiles; tile += gridDim.x) {
        const uint64_t r0 = tile * R;
        const uint32_t nr = (uint32_t)((uint64_t)R < n - r0 ? (uint64_t)R : n - r0);
        {  // the tile's bin columns; the first chunk wait below covers them
            const uint4* src = reinterpret_cast<const uint4*>(bins_g + tile * col_bytes);
            uint4* dst = reinterpret_cast<uint4*>(bins);
            for (uint32_t i = tid; i < col_bytes / 16u; i += blockDim.x) cp_async16(dst + i, src + i);
            asm volatile("cp.async.commit_group;" ::: "memory");
        }
        for (uint32_t g = 0; g < f.n_groups; ++g) {
            const uint32_t t0 = f.group_off[g], t1 = f.group_off[g + 1];
            float acc = f.base[g];
            auto issue = [&](uint32_t c, uint32_t buf) {  // chunk starting at tree t0 + c * CHUNK
                const uint32_t ta = t0 + c * PREDICT_CHUNK;
                const uint32_t nt = min(PREDICT_CHUNK, t1 - ta);
                const uint4* src = reinterpret_cast<const uint4*>(f.nodes + (size_t)ta * HEAP_NODES);
                uint4* dst = reinterpret_cast<uint4*>(ring + (size_t)buf * PREDICT_CHUNK * HEAP_NODES);
                for (uint32_t i = tid; i < nt * (PREDICT_TREE_BYTES / 16u); i += blockDim.x) cp_async16(dst + i, src + i);
                asm volatile("cp.async.commit_group;" ::: "memory");
            };
            const uint32_t n_chunks = (t1 - t0 + PREDICT_CHUNK - 1) / PREDICT_CHUNK;
            if (n_chunks) issue(0, 0);
            for (uint32_t c = 0; c < n_chunks; ++c) {
                if (c + 1 < n_chunks) {
                    issue(c + 1, (c + 1) & 1u);
                    asm volatile("cp.async.wait_group 1;" ::: "memory");
                } else {
                    asm volatile("cp.async.wait_group 0;" ::: "memory");
                }
                __syncthreads();  // chunk c (and the tile's bins) landed; the previous chunk's leaf values are summed
                const uint32_t* tb = ring + (size_t)(c & 1u) * PREDICT_CHUNK * HEAP_NODES;
                const uint32_t nt = min(PREDICT_CHUNK, t1 - (t0 + c * PREDICT_CHUNK));
                if (S == 1) {
                    heap_walk<CAT, BinT>(tb, 0, nt, cb, Rb, f, [&](uint32_t, float v) { acc = acc + v; });
                } else {
                    const uint32_t per = PREDICT_CHUNK / S;  // S divides the chunk
                    const uint32_t q0 = min(sg * per, nt), q1 = min(q0 + per, nt);
                    heap_walk<CAT, BinT>(tb, q0, q1, cb, Rb, f, [&](uint32_t q, float v) { lv[q * R + rg] = v; });
                    __syncthreads();
                    if (sg == 0)
                        for (uint32_t q = 0; q < nt; ++q) acc = acc + lv[q * R + rg];
                }
                __syncthreads();  // ring buffer (c & 1) free for chunk c + 2
            }
            if (sg == 0 && rg < nr) out[(uint64_t)g * n + r0 + rg] = acc;
        }
        asm volatile("cp.async.wait_group 0;" ::: "memory");
        __syncthreads();  // bins free for the next tile
    }
}

void launch_predict_heap(const HeapForest& f, const float* x, uint64_t n, uint32_t F, float* out, void* scratch,
                         cudaStream_t st) {
    if (n == 0) return;
    init_kernel_attributes();  // per device: the kernels' shared-memory opt-in
    const HeapPlan p = heap_plan(f, F, n);
    const uint32_t NF = F < f.n_features ? F : f.n_features;
    const uint64_t tiles = (n + p.R - 1) / p.R;
    {
        // warp items: row groups x feature chunks, about 32 warps per SM
        const uint32_t wr = f.bins16 ? 64u : 128u;
        const uint64_t groups = (n + wr - 1) / wr;
        const uint64_t want = sm_count() * 32u;
        const uint64_t fgs = (NF + BIN_F - 1) / BIN_F;
        uint64_t n_fc = groups >= want ? 1 : (want + groups - 1) / groups;
        if (n_fc > fgs) n_fc = fgs;
        if (n_fc < 1) n_fc = 1;
        const uint32_t FC = (uint32_t)((fgs + n_fc - 1) / n_fc) * BIN_F;
        const uint64_t items = groups * ((NF + FC - 1) / FC);
        const uint64_t blocks = (items + BIN_THREADS / 32u - 1) / (BIN_THREADS / 32u);
        const unsigned grid = (unsigned)(blocks < sm_count() * 4u ? blocks : sm_count() * 4u);
        const size_t smem = (predict_spl_floats(NF) + (size_t)(BIN_THREADS / 32u) * wr * BIN_XS_LD) * sizeof(float);
        if (f.bins16)
            launch_k(k_bin_rows<uint16_t>, grid, BIN_THREADS, smem, st, f, x, n, F, p.R, FC, static_cast<uint32_t*>(scratch));
        else
            launch_k(k_bin_rows<uint8_t>, grid, BIN_THREADS, smem, st, f, x, n, F, p.R, FC, static_cast<uint32_t*>(scratch));
    }
    const unsigned grid = (unsigned)(tiles < sm_count() ? tiles : sm_count());
    const unsigned threads = p.R * p.S;
    const unsigned char* bg = static_cast<const unsigned char*>(scratch);
    if (f.has_cat)
        launch_k(k_predict_heap<true, uint16_t>, grid, threads, p.smem, st, f, bg, n, p.R, p.S, out);
    else if (f.bins16)
        launch_k(k_predict_heap<false, uint16_t>, grid, threads, p.smem, st, f, bg, n, p.R, p.S, out);
    else
        launch_k(k_predict_heap<false, uint8_t>, grid, threads, p.smem, st, f, bg, n, p.R, p.S, out);
}

__global__ void k_transform(int t, float* __restrict__ p, uint32_t G, uint64_t n) {
    BST_PDL_ENTER();
    const uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x;
    if (t == 1) {
        if (i >= (uint64_t)G * n) return;
        const float x = p[i];
        const float c = x < -500.0f ? -500.0f : (x > 500.0f ? 500.0f : x);
        float r;
        if (c >= 0.0f) {
            r = 1.0f / (1.0f + exp_f32(-c));
        } else {
            const float e = exp_f32(c);
            r = e / (1.0f + e);
        }
        p[i] = r;
    } else if (t == 2) {
        if (i >= n) return;
        float mx = -INFINITY;
        for (uint32_t g = 0; g < G; ++g) mx = fmaxf(mx, p[(uint64_t)g * n + i]);
        float sum = 0.0f;
        for (uint32_t g = 0; g < G; ++g) {
            const float e = exp_f32(p[(uint64_t)g * n + i] - mx);
            p[(uint64_t)g * n + i] = e;
            sum = sum + e;
        }
        if (sum > 0.0f)
            for (uint32_t g = 0; g < G; ++g) p[(uint64_t)g * n + i] = p[(uint64_t)g * n + i] / sum;
    }
}

void launch_transform(int transform, float* out, uint32_t G, uint64_t n, cudaStream_t st) {
    if (transform == 0 || n == 0) return;
    const uint64_t total = transform == 1 ? (uint64_t)G * n : n;
    launch_k(k_transform, (unsigned)((total + 255) / 256), 256, 0, st, transform, out, G, n);
}

// Row sampling: grad/hess of the rows outside the sample become zero
// (sample_uniform, training/sampling/row.rs:168-210).
__global__ void k_zero_unsampled(float2* __restrict__ gh, const uint8_t* __restrict__ mask, uint64_t n) {
    BST_PDL_ENTER();
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        if (!mask[i]) gh[i] = make_float2(0.0f, 0.0f);
}

void launch_zero_unsampled(float2* gh, const uint8_t* mask, uint64_t n, cudaStream_t st) {
    if (n == 0) return;
    const uint64_t blocks = std::min<uint64_t>((n + 255) / 256, (uint64_t)sm_count() * 8);
    launch_k(k_zero_unsampled, (unsigned)blocks, 256, 0, st, gh, mask, n);
}

// GOSS (sampling/row.rs:214-280): code 0 leaves the tree (zero grad/hess),
// 1 is kept, 2 is kept with grad and hess scaled by `mult`; mask gets 0 / 1.
__global__ void k_goss_apply(float2* __restrict__ gh, const uint8_t* __restrict__ code, float mult,
                             uint8_t* __restrict__ mask, uint64_t n) {
    BST_PDL_ENTER();
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x) {
        const uint8_t c = code[i];
        if (c == 0) {
            gh[i] = make_float2(0.0f, 0.0f);
        } else if (c == 2) {
            const float2 v = gh[i];
            gh[i] = make_float2(v.x * mult, v.y * mult);
        }
        mask[i] = c ? 1 : 0;
    }
}

void launch_goss_apply(float2* gh, const uint8_t* code, float mult, uint8_t* mask, uint64_t n, cudaStream_t st) {
    if (n == 0) return;
    const uint64_t blocks = std::min<uint64_t>((n + 255) / 256, (uint64_t)sm_count() * 8);
    launch_k(k_goss_apply, (unsigned)blocks, 256, 0, st, gh, code, mult, mask, n);
}

__global__ void k_add_f32(float* __restrict__ a, const float* __restrict__ b, uint64_t n) {
    BST_PDL_ENTER();
    for (uint64_t i = (uint64_t)blockIdx.x * blockDim.x + threadIdx.x; i < n; i += (uint64_t)gridDim.x * blockDim.x)
        a[i] = a[i] + b[i];
}

void launch_add_f32(float* a, const float* b, uint64_t n, cudaStream_t st) {
    if (n == 0) return;
    const uint64_t blocks = std::min<uint64_t>((n + 255) / 256, (uint64_t)sm_count() * 8);
    launch_k(k_add_f32, (unsigned)blocks, 256, 0, st, a, b, n);
}

void init_kernel_attributes() {
    static std::atomic<unsigned long long> done{0ull};
    int dev = 0;
    if (cudaGetDevice(&dev) != cudaSuccess) return;
    const unsigned long long bit = dev < 64 ? (1ull << dev) : 0ull;
    if (bit && (done.load() & bit)) return;
    cudaFuncSetAttribute(k_bin_rows<uint8_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
    cudaFuncSetAttribute(k_bin_rows<uint16_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, 96 * 1024);
    cudaFuncSetAttribute(k_predict_heap<true, uint16_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PREDICT_SMEM);
    cudaFuncSetAttribute(k_predict_heap<false, uint16_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PREDICT_SMEM);
    cudaFuncSetAttribute(k_predict_heap<false, uint8_t>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)PREDICT_SMEM);
    const int hist_smem = 200 * 1024;
    cudaFuncSetAttribute(k_hist_build<GRAD_F32>, cudaFuncAttributeMaxDynamicSharedMemorySize, hist_smem);
    cudaFuncSetAttribute(k_hist_build<GRAD_Q16>, cudaFuncAttributeMaxDynamicSharedMemorySize, hist_smem);
    cudaFuncSetAttribute(k_hist_build<GRAD_Q8>, cudaFuncAttributeMaxDynamicSharedMemorySize, hist_smem);
    cudaFuncSetAttribute(k_b_hist<GRAD_F32, HBin>, cudaFuncAttributeMaxDynamicSharedMemorySize, hist_smem);
    cudaFuncSetAttribute(k_b_hist<GRAD_Q16, HBin>, cudaFuncAttributeMaxDynamicSharedMemorySize, hist_smem);
    cudaFuncSetAttribute(k_b_hist<GRAD_Q8, HBin>, cudaFuncAttributeMaxDynamicSharedMemorySize, hist_smem);
    cudaFuncSetAttribute(k_b_hist<GRAD_Q8, HBin32>, cudaFuncAttributeMaxDynamicSharedMemorySize, hist_smem);
    cudaFuncSetAttribute(k_bin_assign, cudaFuncAttributeMaxDynamicSharedMemorySize, 160 * 1024);
    for (int m = 0; m < 3; ++m)
        for (int v = 0; v < LANE_VARIANTS; ++v)
            cudaFuncSetAttribute(lane_kernel_of(m, v), cudaFuncAttributeMaxDynamicSharedMemorySize,
                                 (int)lane_smem_bytes(m, v));
    cudaFuncSetAttribute(k_lw_replay<true>, cudaFuncAttributeMaxDynamicSharedMemorySize, (int)LW_REPLAY_SMEM_MAX);
    done.fetch_or(bit);
}

}  // namespace bst
