// kernels.h — device data layout and launch wrappers of the B200 GBDT engine.
//
// HBM layout (training):
//   bins8   row-major u8  [n_rows][s8]   columns with <= 256 logical bins
//   bins16  row-major u16 [n_rows][s16]  columns with  > 256 logical bins
//   gh      float2 [n_outputs][n_rows]   (grad, hess) of the current round
//   ridx    u32 [n_rows]                 row ids grouped by partition node
//   hist    HBin [n_slots][total_bins]   one histogram per partition node,
//                                        64-bit fixed point (exact sums)
// s8 is a multiple of 16 and s16 a multiple of 8 so that every row starts
// on a 16-byte boundary and is read with 128-bit loads.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace bst {

// Histogram bin: exact 64-bit fixed-point sums of grad and hess.
struct HBin {
    long long g, h;
};

// ---- K1 bin assignment ----------------------------------------------------
struct BinColumn {
    uint32_t matrix;      // 0 = u8, 1 = u16
    uint32_t pos;         // column position inside its matrix row
    uint32_t is_cat;      // categorical mapper
    uint32_t n_search;    // numeric: searchable bounds (bin_mapper.rs:237-243)
    uint32_t off;         // offset into thr (numeric) or cats (categorical)
    uint32_t n_cats;      // categorical: number of categories
    uint32_t nan_bin;     // bin of NaN
    uint32_t zero_bin;    // bin of 0.0 when missing type is Zero, else 0xFFFFFFFF
};

// thr holds, per numeric column, the largest f32 <= each f64 upper bound, so
// `v <= bound` (f64) equals `v <= thr` (f32) for every f32 v.
// Rows per bin-assignment block for these strides (0 = row too wide).
int bin_assign_rows(uint32_t s8, uint32_t s16);
void launch_bin_assign(const float* x_fm, uint64_t n, const BinColumn* cols, uint32_t n_cols,
                       const float* thr, const int32_t* cats, uint8_t* bins8, uint32_t s8,
                       uint16_t* bins16, uint32_t s16, cudaStream_t st);

// ---- K3 gradients ---------------------------------------------------------
// maxabs [G][2] receives the bit patterns of max|grad|, max|hess| (atomicMax).
void launch_gradients(int objective, uint32_t G, const float* pred, const float* y,
                      const float* w, uint64_t n, float2* gh, unsigned* maxabs,
                      cudaStream_t st);
// Fixed-point resolution: every grad/hess becomes round(v * 2^k) with
// |q| <= 2^HIST_QBITS (and n * 2^k * max < 2^62 for the int64 sums).
constexpr int HIST_QBITS = 38;
constexpr int HIST_LO_BITS = 20;     // low part of the shared-memory split
constexpr int HIST_CHUNK_MAX = 4096; // rows per block: 4096 * 2^20 < 2^32, 4096 * 2^18 < 2^31
// scales [G][4] = (2^kg, 2^kh, 2^-kg, 2^-kh).
void launch_fixed_scales(const unsigned* maxabs, uint32_t G, uint64_t n, double* scales,
                         cudaStream_t st);

// ---- K4 histogram build -----------------------------------------------------
struct HistChunk {
    uint32_t slot;   // destination histogram slot
    uint32_t begin;  // first position in ridx
    uint32_t count;  // rows in this chunk
    uint32_t flags;  // bit0: rows are begin..begin+count (no ridx read)
};
struct HistTile {
    uint32_t matrix;    // 0 = u8, 1 = u16
    uint32_t vec;       // 16-byte vector index inside the row
    uint32_t c0, c1;    // lanes of that vector handled by this tile
    uint32_t smem_bins; // bins of those columns (shared-memory histogram size)
    uint32_t lane_smem[16];  // per lane: shared-memory bin offset
    uint32_t lane_hist[16];  // per lane: global histogram bin offset
    uint32_t lane_nbins[16]; // per lane: number of bins
};
void launch_hist_build(const HistChunk* chunks, uint32_t n_chunks, const HistTile* tiles,
                       uint32_t n_tiles, uint32_t max_smem_bins, const uint32_t* ridx,
                       const float2* gh, const double* scale, const uint8_t* bins8, uint32_t s8,
                       const uint16_t* bins16, uint32_t s16, HBin* hist, uint64_t slot_bins,
                       cudaStream_t st);

// Subtraction trick: the parent histogram lives in slot `left`, the smaller
// child was built into slot `right`. flags bit0 = left child is the smaller.
struct FinishWork {
    uint32_t left, right, flags, pad;
};
void launch_hist_finish(const FinishWork* w, uint32_t n_work, HBin* hist, uint64_t slot_bins,
                        uint32_t total_bins, cudaStream_t st);

// Exact node sums (sum of the same fixed-point values) for nodes whose
// histogram is not needed. Uses HistChunk.slot as the output index.
void launch_node_sums(const HistChunk* chunks, uint32_t n_chunks, const uint32_t* ridx,
                      const float2* gh, const double* scale, long long* sums, cudaStream_t st);

// ---- K6 split scan ----------------------------------------------------------
struct ScanColumn {
    uint32_t n_bins, hist_off, is_cat, has_missing;
};
struct ScanNode {
    uint32_t slot;   // histogram slot
    uint32_t count;  // rows in the node (parent_count of find.rs)
    uint32_t flags;  // bit0: use pg/ph as the parent totals instead of the bin sums
    uint32_t pad;
    long long pg, ph;  // explicit parent totals (fixed point)
};
struct GainParamsDev {
    double lambda;          // reg_lambda as f64
    double min_gain;        // min_gain as f64
    double min_child_weight;
    uint32_t min_samples_leaf;
    uint32_t max_onehot_cats;
};
// Per (node, column) best candidate.
struct ColCand {
    float gain;         // -inf if none
    uint32_t order;     // position in the reference's scan order (ties)
    uint32_t bin;       // numeric split bin
    uint32_t flags;     // bit0 default_left, bit1 categorical
    unsigned long long cats[4];  // categorical: bins going left
};
// Per node result.
struct NodeSplit {
    float gain;
    uint32_t col;
    uint32_t bin;
    uint32_t flags;     // bit0 default_left, bit1 categorical, bit2 valid
    unsigned long long cats[4];
    long long tot_g, tot_h;  // exact fixed-point node totals
};
void launch_split_scan(const ScanNode* nodes, uint32_t n_nodes, const ScanColumn* cols,
                       uint32_t n_cols, const HBin* hist, uint64_t slot_bins,
                       const double* scale, GainParamsDev gp, ColCand* cand,
                       long long* node_tot, cudaStream_t st);
void launch_split_reduce(const ColCand* cand, const long long* node_tot, uint32_t n_nodes,
                         uint32_t n_cols, int last_wins, NodeSplit* out, cudaStream_t st);

// ---- K7 partition -----------------------------------------------------------
struct PartWork {
    uint32_t begin, count;
    uint32_t matrix, pos;
    uint32_t thr_bin;
    uint32_t flags;        // bit0 default_left, bit1 has_missing, bit2 categorical
    uint32_t default_bin;
    uint32_t pad;
    unsigned long long cats[4];
};
struct PartChunk {
    uint32_t work, start, len, pad;
};
// cursors [n_work][2]: (left write cursor, right write cursor); initialised by
// the caller to (begin, begin + count). Rows are scattered into tmp.
void launch_partition(const PartWork* works, const PartChunk* chunks, uint32_t n_chunks,
                      const uint32_t* ridx, uint32_t* tmp, unsigned* cursors,
                      const uint8_t* bins8, uint32_t s8, const uint16_t* bins16, uint32_t s16,
                      cudaStream_t st);
void launch_copy_chunks(const PartChunk* chunks, const PartWork* works, uint32_t n_chunks,
                        const uint32_t* src, uint32_t* dst, cudaStream_t st);
void launch_iota(uint32_t* ridx, uint64_t n, cudaStream_t st);

// ---- K8 leaf values -> predictions -----------------------------------------
struct LeafSeg {
    uint32_t begin, count;
    float value;
    uint32_t tree_node;
};
// leaves sorted by begin and tiling [0, n).
void launch_leaf_update(const LeafSeg* leaves, uint32_t n_leaves, const uint32_t* ridx,
                        uint64_t n, float* pred, uint32_t* row_leaf, cudaStream_t st);

// ---- device-side depth-wise growth (one CUDA graph per tree) -----------------
// The host launches a fixed sequence of kernels per tree; every data-dependent
// size (frontier, expanding nodes, row chunks) is read from device memory, so
// the sequence is captured once and replayed for every tree.
struct BColumn {  // per effective column, for decisions and the partition
    uint32_t matrix, pos, has_missing, default_bin;
};
struct BNode {  // frontier entry
    uint32_t pnode, tnode, begin, count;
    long long G, H;
    NodeSplit split;
};
struct BTreeNode {  // tree node as grown (training semantics)
    uint32_t col, bin, flags;  // flags: bit0 default_left, bit1 categorical, bit2 leaf
    uint32_t left, right;      // children tree nodes in allocation order
    float gain, leaf;          // leaf: value x learning rate
    double G, H;
    unsigned long long cats[4];
};
struct BExp {  // an expanding node of the current level
    uint32_t front, right_pnode, tl, tr;  // tl/tr: tree nodes of the training-left/right child
    uint32_t lc, rc, small_begin, small_count;
    uint32_t part_off, hist_off, pad0, pad1;
};
struct BLeaf {
    uint32_t begin, count;
    float value;
    uint32_t tnode;
    uint32_t chunk_off, pad;
};
struct BState {
    uint32_t n_front, n_exp, n_pnodes, n_tnodes;
    uint32_t part_chunks, hist_chunks, n_leaves, leaf_chunks;
    uint32_t first_right, pad;
    unsigned long long hist_rows;  // rows visited by histogram builds of this tree
    uint32_t pad2[4];
};
struct LeafParams {
    double lambda, alpha, min_gain;
    float learning_rate;
    uint32_t pad;
};
struct BDev {  // device buffers of the level loop
    BState* state;
    BNode* front[2];
    BExp* exp;
    BTreeNode* tree;
    BLeaf* leaves;
    PartWork* pworks;
    unsigned* cursors;
    FinishWork* finish;
    ScanNode* scan_nodes;
    long long* sums;  // [max_exp][2]
    const BColumn* bcols;
    uint32_t max_front, max_tnodes;
};
constexpr uint32_t B_PART_CHUNK = 2048;
constexpr uint32_t B_LEAF_CHUNK = 4096;

// Raises the dynamic shared-memory limits of the kernels that need > 48 KiB
// (call once per device before any stream capture).
void init_kernel_attributes();
void launch_b_root(const BDev& d, uint64_t n, cudaStream_t st);
void launch_b_root_set(const BDev& d, const NodeSplit* root_split, cudaStream_t st);
// level kernels; `a` is the index of the current frontier buffer
void launch_b_decide(const BDev& d, int a, LeafParams lp, const double* scale, cudaStream_t st);
void launch_b_partition(const BDev& d, const uint32_t* ridx, uint32_t* tmp, const uint8_t* bins8, uint32_t s8,
                        const uint16_t* bins16, uint32_t s16, uint32_t grid, cudaStream_t st);
void launch_b_copy(const BDev& d, const uint32_t* tmp, uint32_t* ridx, uint32_t grid, cudaStream_t st);
void launch_b_children(const BDev& d, int a, int need_split, cudaStream_t st);
void launch_b_zero_right(const BDev& d, HBin* hist, uint64_t slot_bins, uint32_t grid, cudaStream_t st);
void launch_b_hist(const BDev& d, const HistTile* tiles, uint32_t n_tiles, uint32_t max_smem_bins,
                   const uint32_t* ridx, const float2* gh, const double* scale, const uint8_t* bins8,
                   uint32_t s8, const uint16_t* bins16, uint32_t s16, HBin* hist, uint64_t slot_bins,
                   uint32_t grid, cudaStream_t st);
void launch_b_finish(const BDev& d, HBin* hist, uint64_t slot_bins, uint32_t total_bins, uint32_t grid,
                     cudaStream_t st);
void launch_b_scan(const BDev& d, const ScanColumn* cols, uint32_t n_cols, const HBin* hist,
                   uint64_t slot_bins, const double* scale, GainParamsDev gp, ColCand* cand,
                   long long* node_tot, uint32_t grid, cudaStream_t st);
void launch_b_reduce(const BDev& d, int b, const ColCand* cand, const long long* node_tot, uint32_t n_cols,
                     int last_wins, uint32_t grid, cudaStream_t st);
void launch_b_sums(const BDev& d, const uint32_t* ridx, const float2* gh, const double* scale, uint32_t grid,
                   cudaStream_t st);
void launch_b_children_sums(const BDev& d, int b, cudaStream_t st);
void launch_b_finalize(const BDev& d, int a, LeafParams lp, const double* scale, cudaStream_t st);
void launch_b_leaf_update(const BDev& d, const uint32_t* ridx, float* pred, uint32_t* row_leaf, uint32_t grid,
                          cudaStream_t st);

// ---- K9 forest traversal ----------------------------------------------------
// Node: word0 = feature | (is_leaf << 31) | (default_left << 30) | (categorical << 29)
//       value = threshold (split) or leaf value (leaf); left/right absolute indices.
struct ForestNode {
    uint32_t word;
    float value;
    uint32_t left, right;
};
struct ForestDev {
    const ForestNode* nodes;
    const uint32_t* roots;        // per tree, absolute node index
    const uint32_t* group_trees;  // tree ids grouped by output group, forest order
    const uint32_t* group_off;    // [n_groups + 1] offsets into group_trees
    const uint32_t* cat_seg;      // per node: (start, size) pairs into cat_words
    const uint32_t* cat_words;
    const float* base;            // [n_groups]
    uint32_t n_trees, n_groups;
};
// feature_major != 0: x[f * n + i]; else sample-major x[i * n_features + f].
// out [n_groups][n] raw margins (base score + trees in forest order, f32).
void launch_predict(const ForestDev& f, const float* x, uint64_t n, uint32_t n_features,
                    int feature_major, float* out, cudaStream_t st);
// transform: 1 sigmoid, 2 softmax over [G][n]
void launch_transform(int transform, float* out, uint32_t G, uint64_t n, cudaStream_t st);

}  // namespace bst
