// kernels.h — device data layout and launch wrappers of the B200 GBDT engine.
//
// HBM layout (training):
//   rec     [n_rows][rec] bytes          one record per row: u8 bins of the
//                                        columns with <= 256 logical bins,
//                                        then (from a 16-byte boundary) u16
//                                        bins of the others
//   bins8   u8 view of rec, row stride s8 = rec bytes
//   bins16  u16 view at rec + u16_off, row stride s16 = rec / 2 elements
//   gh      float2 [n_outputs][n_rows]   (grad, hess) of the current round
//   ridx    u32 [n_rows]                 row ids grouped by partition node
//   hist    HBin [n_slots][total_bins]   one histogram per partition node,
//                                        64-bit fixed point (exact sums)
// rec is a multiple of 32 bytes: every row starts on a sector boundary and
// its aligned 16- or 32-byte windows are read with 128-bit loads, each
// within one sector.
#pragma once

#include <cuda_runtime.h>
#include <stdint.h>

namespace bst {

// Streaming multiprocessors of the current device (cached per host thread
// and device): launch grids are sized in whole waves of it.
uint32_t sm_count();

// Checked build (compiled with -DBST_CHECKED into libboosters_b200_checked.so):
// device accesses whose index is read from device memory test it against its
// bound first; a failed test is counted, the first one's site, index and
// bound are recorded, and the access is skipped or redirected to a zero-filled
// row, so a bad index becomes an error status on the host instead of a fault.
enum CheckSite : uint32_t {
    CHECK_PART_CHUNK = 1,  // partition chunk outside its expansion's rows
    CHECK_PART_DST = 2,    // partition scatter outside the node's row range
    CHECK_LEAF_MAP = 3,    // leaf chunk names a leaf past the tree's leaf count
    CHECK_LEAF_ROW = 4,    // leaf update row id >= rows
    CHECK_HIST_ROW = 5,    // histogram gather row id >= rows (tensor-map gather)
    CHECK_PREDICT_NODE = 6,  // traversal node link >= forest nodes
};
struct CheckRecord {
    unsigned long long violations, site, index, bound;
};
// Reads and clears the record of device `device`. False in the normal build
// (no record exists) or on a CUDA error.
bool check_take(int device, CheckRecord* out);

// Histogram bin: exact 64-bit fixed-point sums of grad and hess.
struct HBin {
    long long g, h;
};
// The quantised Q8 form's node histograms when every sum fits 32 bits
// (n * 127 < 2^31): half the bytes for the merge and the split scan.
struct HBin32 {
    int g, h;
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
    uint32_t src;         // the column's row in the feature-major input
};

// thr holds, per numeric column, the largest f32 <= each f64 upper bound, so
// `v <= bound` (f64) equals `v <= thr` (f32) for every f32 v.
// Rows per bin-assignment block for this record size and largest search
// table (the most thresholds or categories of a column; 0 = row too wide).
int bin_assign_rows(uint32_t rec, uint32_t max_tab);
void launch_bin_assign(const float* x_fm, uint64_t n, const BinColumn* cols, uint32_t n_cols,
                       const float* thr, const int32_t* cats, uint8_t* rec_out, uint32_t rec, uint32_t u16_off,
                       uint32_t max_tab, cudaStream_t st);

// Numeric bin bounds of sampled features (dataset.rs:683-750), one block
// per job: column `col` of x (feature-major, col_stride floats apart), its
// rows `rows[0..k)` (ascending; null = rows 0..k-1). Per job: scratch 2k
// words, cand max_bins doubles, bounds max_bins + 2 doubles (the upper
// bounds, the last one DBL_MAX, then DBL_MAX again for the NaN bin when
// has_nan and there are two or more distinct finite values) and n_bounds.
struct MapJob {
    uint32_t col;
    uint32_t has_nan;
};
void launch_numeric_bounds(const float* x, uint64_t col_stride, const uint32_t* rows, uint32_t k, const MapJob* jobs,
                           uint32_t n_jobs, uint32_t max_bins, uint32_t* scratch, double* cand, double* bounds,
                           uint32_t* n_bounds, cudaStream_t st);

// ---- K3 gradients ---------------------------------------------------------
// maxabs [G][2] receives the bit patterns of max|grad|, max|hess| (atomicMax).
// alpha: [G] pinball alphas (device); delta: the pseudo-Huber delta.
void launch_gradients(int objective, uint32_t G, const float* pred, const float* y,
                      const float* w, uint64_t n, float2* gh, unsigned* maxabs,
                      cudaStream_t st, const float* alpha = nullptr, float delta = 1.0f);
// Fixed-point resolution: every grad/hess becomes round(v * 2^k) with
// |q| <= 2^HIST_QBITS (and n * 2^k * max < 2^62 for the int64 sums).
constexpr int HIST_QBITS = 38;
constexpr int HIST_LO_BITS = 20;     // low part of the shared-memory split
constexpr int HIST_CHUNK_MAX = 4096; // rows per block: 4096 * 2^20 < 2^32, 4096 * 2^18 < 2^31
// scales [G][4] = (2^kg, 2^kh, 2^-kg, 2^-kh).
void launch_fixed_scales(const unsigned* maxabs, uint32_t G, uint64_t n, double* scales,
                         cudaStream_t st);

// Gradient source of the histogram and node-sum kernels (values = BST_PRECISION_*):
//   GRAD_F32  gh (f32 pairs) as fixed point round(v * scale[0..1]), exact int64 sums
//   GRAD_Q16  gq short2 [G][n] quantised integers (|q| <= 32767)
//   GRAD_Q8   gq char2  [G][n] quantised integers (|q| <= 127)
constexpr int GRAD_F32 = 0, GRAD_Q16 = 1, GRAD_Q8 = 2;
struct GradRef {
    const float2* gh;
    const void* gq;
    const double* scale;  // GRAD_F32: the fixed-point scales of this output
    int mode;
    // optional: the same elements (float2 / short2 / char2 by mode) permuted
    // into the order of the row-id buffer the histogram reads, so that the
    // lane-tile histogram loads them at the row's position (coalesced)
    // instead of gathering them by row id
    const void* qpos = nullptr;
};
__host__ __device__ constexpr uint32_t grad_elem_bytes(int mode) { return mode == 0 ? 8u : (mode == 1 ? 4u : 2u); }
// Stochastic rounding of every (output, row): q = floor(v * Q / max|v| + u),
// u from Philox4x32-10 with counter (row, output, round, QUANT_STREAM) and key
// (seed lo, seed hi); word 0 rounds grad, word 1 hess.
// qscales [G][4] = (Q / max|g|, Q / max|h|, max|g| / Q, max|h| / Q): the last
// two turn integer histogram sums into gradient units.
constexpr uint32_t QUANT_STREAM = 0x51A7E5EDu;
// maxabs[2] = bit patterns of max|grad|, max|hess| over finite values (atomicMax; zero it first)
void launch_maxabs(const float2* gh, uint64_t n, unsigned* maxabs, cudaStream_t st);
// (outputs are numbered from out0 in the counter)
// fscales (or null): also the fixed-point scales of launch_fixed_scales,
// which then need no launch of their own.
void launch_quantize(int mode, uint32_t G, const float2* gh, uint64_t n, const unsigned* maxabs,
                     uint64_t seed, uint32_t round, uint32_t out0, void* gq, double* qscales, cudaStream_t st,
                     double* fscales = nullptr);

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
                       const GradRef& gr, const uint8_t* bins8, uint32_t s8,
                       const uint16_t* bins16, uint32_t s16, HBin* hist, uint64_t slot_bins,
                       cudaStream_t st);

// Column-lane histogram tiles (bank-conflict-free form of K4). A tile is a
// 16- or 32-byte aligned window of a row-major bin matrix holding C = bytes /
// esize columns. Each lane of a warp takes one row, rotates the row's window
// by (lane mod C) elements and at step j adds its gradient pair to column
// (lane + j) mod C; the shared histogram keeps K = 32 / C copies of every
// column at word bin * 32 + copy * C + column, so the 32 lanes of every
// atomic hit 32 distinct banks. Columns with more than the tile's n_bins
// bins never share a window with these tiles (they use HistTile).
struct LaneTile {
    uint32_t esize;     // 1 (u8 matrix) or 2 (u16 matrix)
    uint32_t words;     // window width in 32-bit words: 4 or 8
    uint32_t byte_off;  // window start inside the row of its view, bytes (multiple of 16)
    uint32_t rec_off;   // window start inside the row record, bytes (multiple of 16)
    uint32_t n_bins;    // largest bin count of the window's columns
    uint32_t col_hist[32];   // per window element: global histogram bin offset
    uint32_t col_nbins[32];  // per window element: bins (0 = no column)
};
// Largest n_bins of a lane tile (shared-memory height).
uint32_t lane_tile_max_bins(int mode);
// Rows of a row segment at most: what one block may sum exactly in 32-bit
// shared counters (4096 for the hi/lo fixed-point split, 16384 quantised).
uint32_t lane_segment_max(int mode);
// Resident blocks per SM of lane-kernel variant v (0 .. lane_variants() - 1).
uint32_t lane_blocks_per_sm(int mode, int variant);
int lane_variants();
// Partial histograms: one record of lane_part_stride() entries per (segment,
// lane tile) item, entries of lane_part_entry_bytes(mode) bytes, column-major
// (entry = element * n_bins + bin).
uint32_t lane_part_stride();
uint32_t lane_part_entry_bytes(int mode);

// Exact node sums (sum of the same fixed-point values) for nodes whose
// histogram is not needed. Uses HistChunk.slot as the output index.
void launch_node_sums(const HistChunk* chunks, uint32_t n_chunks, const uint32_t* ridx,
                      const GradRef& gr, long long* sums, cudaStream_t st);

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
// hist: HBin, or HBin32 when hist32 != 0 (the same for the level kernels below)
// colmask (or null): [depth][n_cols] column masks (column sampling), a
// node's row chosen by its depth in ScanNode.pad
void launch_split_scan(const ScanNode* nodes, uint32_t n_nodes, const ScanColumn* cols,
                       uint32_t n_cols, const void* hist, uint64_t slot_bins,
                       const double* scale, GainParamsDev gp, ColCand* cand,
                       long long* node_tot, cudaStream_t st, int hist32 = 0, const uint8_t* colmask = nullptr);
void launch_split_reduce(const ColCand* cand, const long long* node_tot, uint32_t n_nodes,
                         uint32_t n_cols, int last_wins, NodeSplit* out, cudaStream_t st);
// Loads the split-scan kernels (HBin) onto the current device now rather than
// at their first launch (the runtime loads device code lazily).
cudaError_t load_split_kernels();

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
// Column-major copies of the bin matrices ([column][n]), or null pointers.
struct BinsFM {
    const uint8_t* b8 = nullptr;
    const uint16_t* b16 = nullptr;
    uint64_t n = 0;
};
// cursors [n_work][2]: (left write cursor, right write cursor); initialised by
// the caller to (begin, begin + count). Rows are scattered into tmp.
// qin / qout (grad_elem_bytes(mode) each, or null): each row's gradient
// element moves with its row id (positional copy); fm: the split column is
// read from the column-major bins when set.
void launch_partition(const PartWork* works, const PartChunk* chunks, uint32_t n_chunks,
                      const uint32_t* ridx, uint32_t* tmp, unsigned* cursors,
                      const uint8_t* bins8, uint32_t s8, const uint16_t* bins16, uint32_t s16,
                      cudaStream_t st, const void* qin = nullptr, void* qout = nullptr, int mode = 0,
                      const BinsFM& fm = BinsFM{}, const uint8_t* rmask = nullptr, unsigned* scnt = nullptr);
// rmask (or null): row-sampling mask [n]; then scnt [n_work][2] (zeroed by
// the caller) gets each work's sampled rows going left / right.
// copies the chunks' row ids src -> dst and, when qsrc is set, their
// positional gradient elements qsrc -> qdst
void launch_copy_chunks(const PartChunk* chunks, const PartWork* works, uint32_t n_chunks,
                        const uint32_t* src, uint32_t* dst, cudaStream_t st, const void* qsrc = nullptr,
                        void* qdst = nullptr, int mode = 0);
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
    uint32_t part_off, hist_off;
    uint32_t left_pnode;  // the node's own slot: parent histogram, then its left child's
    uint32_t pad1;
};
struct BLeaf {
    uint32_t begin, count;
    float value;
    uint32_t tnode;
    uint32_t chunk_off;
    uint32_t buf;  // row-index buffer (0 / 1) holding the leaf's rows
};
struct BState {
    uint32_t n_front, n_exp, n_pnodes, n_tnodes;
    uint32_t part_chunks, hist_chunks, n_leaves, leaf_chunks;
    uint32_t first_right;
    uint32_t hist_chunk;           // rows per histogram work item of the level
    unsigned long long hist_rows;  // rows visited by histogram builds of this tree
    uint32_t done;                 // last-block hand-off counter (zero between launches)
    uint32_t err;                  // nonzero: a bounded wait of a kernel gave up (the tree is invalid)
    uint32_t pad2[2];
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
    ScanNode* scan_nodes;
    long long* sums;  // [max_exp][2]
    uint32_t* seg_exp;  // histogram row segment -> expanding node of the level
    uint32_t max_segs;  // capacity of seg_exp (and of the partial-histogram buffer)
    const BColumn* bcols;
    uint32_t max_front, max_tnodes;
    uint32_t hist_target;   // desired histogram row segments per level
    uint32_t hist_seg_max;  // largest row segment (lane_segment_max)
    unsigned long long* node_key;  // [max_front] best candidate key per node; zero between levels
    const uint8_t* rmask;  // row sampling: the tree's sampled rows [n] (or null)
    unsigned* scnt;        // row sampling: [max_front][2] sampled rows per side of each expansion
    uint2* part_map;       // partition chunk -> (expansion, first row), written with the decisions
    uint32_t max_part_chunks;  // capacity of part_map
    uint2* leaf_map;       // leaf chunk -> (leaf, first row), written by k_b_finalize
    uint32_t max_leaf_chunks;  // capacity of leaf_map
#ifdef BST_CHECKED
    uint32_t chk_rows;  // rows of the training set (bound of every row id)
#endif
};
constexpr uint32_t B_PART_CHUNK = 2048;
constexpr uint32_t B_LEAF_CHUNK = 2048;  // rows per leaf-kernel work item (2048 measured faster than 4096)

// ---- leaf renewing (trainer.rs:283-313, objectives/mod.rs:352-409) ----------
// L1 and pinball losses: after a tree is grown, each leaf's value becomes
// the alpha-quantile of the residuals y - pred of its (sampled) rows, times
// the learning rate. Unweighted: the rank ceil(alpha m) - 1 element by value
// (utils.rs:17-53), found by a 4-pass radix select over orderable residual
// keys. Weighted: the first value, in value order (ties in partition order),
// whose f32 running weight reaches alpha x the f32 total of the weights
// summed in partition order (utils.rs:81-135): one block per leaf compacts,
// sorts (32 stable 1-bit passes) and scans. The leaves come from d.leaves /
// d.leaf_map / d.state (n_leaves, leaf_chunks); their values and, when
// d.tree is set, the device tree's leaf values are overwritten.
struct RenewDev {
    uint32_t* cnt;     // [cap] sampled rows per leaf
    uint32_t* prefix;  // [cap] key prefix found so far
    uint32_t* rank;    // [cap] rank below the prefix still to find (0xFFFFFFFF: leaf kept)
    uint32_t* hist;    // [cap][256]
    uint32_t cap;
    uint32_t* key[2];  // weighted: [n] ping-pong keys
    uint32_t* row[2];  // weighted: [n] ping-pong row ids
    uint32_t n_rows;   // weighted: rows of the dataset (row ids < n_rows)
};
void launch_leaf_renew(const BDev& d, const RenewDev& r, const uint32_t* r0, const uint32_t* r1, const float* y,
                       const float* pred, const float* w, float alpha, float learning_rate, uint32_t grid,
                       cudaStream_t st);

// ---- device-side leaf-wise growth (expansion.rs:129-213) ---------------------
// The reference pops the leaf of largest (gain, node id) from a max-heap,
// splits it and pushes its children until max_leaves. The device replays
// those pops exactly (k_lw_replay: one warp pops, the block ranks): when
// the popped leaf has not been expanded yet it stops and hands the level
// kernels a batch of the best unexpanded candidates (the popped one first,
// at most as many as pops remain); their rows, histograms and splits do not
// depend on when they are expanded (exact sums), so a later pop of a batch
// member costs no step.
struct LwCand {          // a leaf that may be split
    NodeSplit split;     // its best split; tot_g / tot_h: the node's exact sums
    uint32_t pnode, tnode, depth, count;  // partition node, tree node, depth, rows
    uint32_t vid;        // heap order id: gain ties pop the higher id first (expansion.rs:311-319)
    uint32_t pad[3];
};
struct LwSpec {          // a partition node expanded before its pop
    LwCand kids[2];      // training-left and training-right children
    uint32_t right_pnode, begin, count, valid;  // range before the split; valid: not yet popped
};
struct LwState {
    uint32_t n_heap, n_leaves, n_vid, n_batch;
    uint32_t done, err, n_leaf_out, pad;
};
struct LwDev {
    LwState* st;
    LwCand* heap;        // [heap_cap]
    LwSpec* spec;        // [max_pnodes]
    uint2* pn;           // [max_pnodes] (begin, count) of each partition node
    NodeSplit* child;    // [max_pnodes] split search results of the pending step's children (root: [0])
    unsigned long long* keys;  // [heap_cap] batch selection scratch (when the heap is not staged in shared memory)
    uint32_t* ranks;     // [2 * heap_cap] ditto
    uint32_t heap_cap, max_pnodes, max_leaves;
    float min_gain;
};
// State of a new tree: the root candidate from child[0], its rows [0, n).
void launch_lw_init(const BDev& d, const LwDev& w, uint32_t n, uint32_t root_count, cudaStream_t st);
// Replays pops until the next expansion is needed (writes that batch's level
// state) or the tree is done (leaves listed in BDev::leaves, BState::n_leaves).
void launch_lw_replay(const BDev& d, const LwDev& w, LeafParams lp, const double* scale, cudaStream_t st);
// Partition of the pending batch (rin -> rout), then the rows copied back
// into rin (leaf-wise keeps one row-index buffer); qin / qout likewise.
void launch_lw_partition(const BDev& d, uint32_t* rin, uint32_t* rout, const uint8_t* bins8, uint32_t s8,
                         const uint16_t* bins16, uint32_t s16, uint32_t grid, void* qin, void* qout, int mode,
                         const BinsFM& fm, cudaStream_t st);
// Leaf chunk map of the finished tree and zeroed leaf sums.
void launch_lw_leaves(const BDev& d, cudaStream_t st);

// Raises the dynamic shared-memory limits of the kernels that need > 48 KiB
// (call once per device before any stream capture).
void init_kernel_attributes();
// Row ids 0..n-1, the root node and the root histogram's level state of a
// depth-wise tree.
void launch_b_root_init(const BDev& d, uint32_t* ridx, uint64_t n, uint32_t chunk, cudaStream_t st);
// Column-major copy of the bin matrices (BinsFM).
void launch_transpose_bins(const uint8_t* b8, uint32_t s8, uint32_t f8, const uint16_t* b16, uint32_t s16,
                           uint32_t f16, uint64_t n, uint8_t* fm8, uint16_t* fm16, cudaStream_t st);
// Level kernels; `a` is the index of the current frontier buffer. Row indices
// alternate between two buffers: level d partitions buffer d & 1 into buffer
// (d + 1) & 1; a leaf records the buffer that holds its rows.
// partition rin -> rout, then (last block) the children of every split;
// qin / qout (grad_elem_bytes(mode) each, or null) move each row's gradient
// element with its row id; fm: the split columns are read column-major
void launch_b_partition(const BDev& d, const uint32_t* rin, uint32_t* rout, const uint8_t* bins8, uint32_t s8,
                        const uint16_t* bins16, uint32_t s16, int a, int need_split, uint32_t grid,
                        const void* qin, void* qout, int mode, const BinsFM& fm, cudaStream_t st);
void launch_b_zero_right(const BDev& d, void* hist, uint64_t slot_bins, uint32_t grid, cudaStream_t st,
                         int hist32 = 0);
void launch_b_hist(const BDev& d, const HistTile* tiles, uint32_t n_tiles, uint32_t max_smem_bins,
                   const uint32_t* ridx, const GradRef& gr, const uint8_t* bins8, uint32_t s8,
                   const uint16_t* bins16, uint32_t s16, void* hist, uint64_t slot_bins, uint32_t grid,
                   cudaStream_t st, int hist32 = 0);
// Partial histograms of every (row segment, lane tile) item of the level
// (state: n_exp, hist_chunks, hist_chunk; exp[].small_begin/small_count/
// hist_off; seg_exp).
// Tensor maps of the row records for the TMA form of the lane kernel
// (variant 3): 2D [n rows][rec bytes] u8, one-row boxes of 32 and of 16
// bytes (tile::gather4 loads four rows per copy). Built once per binned
// dataset; false when the driver cannot encode them (variant 3 unavailable).
struct RecordMaps {
    alignas(64) unsigned char box32[128];
    alignas(64) unsigned char box16[128];
    uint32_t n_rows = 0;  // the maps' row extent (a row id equal to it reads as zeros)
    bool ok = false;
};
bool make_record_maps(RecordMaps& out, const uint8_t* rec, uint64_t n_rows, uint32_t rec_bytes);
void launch_b_hist_part(const BDev& d, const LaneTile* tiles, uint32_t n_tiles, const uint32_t* ridx,
                        const GradRef& gr, const uint8_t* bins8, uint32_t s8, const uint16_t* bins16, uint32_t s16,
                        void* part, int variant, const RecordMaps* maps, cudaStream_t st);
// Sums each node's partials and applies the subtraction trick into slots
// left_pnode / right_pnode (root: one node, the sum goes to right_pnode).
// has_rest: bins of general tiles (bin_map[global bin] == 0xFFFFFFFF) were
// built atomically into the right slots.
// ent [n_ent]: per partial entry of a node (lane tiles in order, column-major
// inside each tile): (global bin or 0xFFFFFFFF, tile << 16 | offset).
// wide != 0: the layout for levels with few expanding nodes (many row
// segments per node); same result.
void launch_b_merge(const BDev& d, void* hist, uint64_t slot_bins, uint32_t total_bins, const void* part,
                    uint32_t n_lane_tiles, const uint2* ent, uint32_t n_ent, const uint32_t* bin_map, bool has_rest,
                    int root, int mode, cudaStream_t st, int hist32 = 0, int wide = 0);
// Batched leaf-wise growth: children counts, smaller children, histogram
// segments and scan nodes of k partitioned parents (d.exp[j] holds their
// slots), from the partition's cursors, on the device.
// scnt (or null): the partition's sampled-row counts (row sampling), used
// as the children's scan counts
// k == LW_K_FROM_STATE: the batch size is BState::n_exp (device-driven steps)
constexpr uint32_t LW_K_FROM_STATE = 0xFFFFFFFFu;
void launch_lw_children(const BDev& d, const PartWork* pw, const unsigned* cursors, uint32_t k, ScanNode* scan_nodes,
                        const unsigned* scnt, cudaStream_t st);
// split finding of the level's nodes and the reduction over columns into
// frontier b, then (last block) the decisions of the next level, whose rows
// are in buffer buf
// root (or null): the level is the root alone, described by *root (rows in
// buffer 0, frontier 0); colmask (or null): the level's column masks, a
// node's row chosen by ScanNode.pad (0 for the device-built levels)
// lw_out (or null): leaf-wise steps: the last block writes the 2 n_exp
// children's splits there instead of a frontier and takes no decisions
void launch_b_scan(const BDev& d, const ScanColumn* cols, uint32_t n_cols, const void* hist,
                   uint64_t slot_bins, const double* scale, GainParamsDev gp, ColCand* cand,
                   long long* node_tot, int b, int last_wins, LeafParams lp, uint32_t buf, uint32_t grid,
                   cudaStream_t st, int hist32 = 0, const ScanNode* root = nullptr,
                   const uint8_t* colmask = nullptr, NodeSplit* lw_out = nullptr);
// last level: the smaller children's sums, then (last block) both children's
// sums into frontier b and, when `finalize`, the tree's leaves from frontier b
// as launch_b_finalize(d, b, lp, scale, buf) would write them
void launch_b_sums(const BDev& d, const uint32_t* ridx, const GradRef& gr, int b, uint32_t grid, cudaStream_t st,
                   int finalize, LeafParams lp, const double* scale, uint32_t buf);
// work items of k_b_scan per node (column blocks of its warps)
uint32_t scan_col_blocks(uint32_t n_cols);
void launch_b_finalize(const BDev& d, int a, LeafParams lp, const double* scale, uint32_t buf, cudaStream_t st);
// quantised training: exact leaf sums of the f32 gradients (gr: GRAD_F32),
// then (last block) the leaf values with their fixed-point scale
void launch_b_leaf_sums(const BDev& d, const uint32_t* r0, const uint32_t* r1, const GradRef& gr, LeafParams lp,
                        const double* scale, uint32_t grid, cudaStream_t st);
void launch_b_leaf_update(const BDev& d, const uint32_t* r0, const uint32_t* r1, float* pred, uint32_t* row_leaf,
                          uint32_t grid, cudaStream_t st);

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
#ifdef BST_CHECKED
    uint32_t chk_nodes;  // entries of nodes (bound of every node link)
#endif
};
// feature_major != 0: x[f * n + i]; else sample-major x[i * n_features + f].
// out [n_groups][n] raw margins (base score + trees in forest order, f32).
void launch_predict(const ForestDev& f, const float* x, uint64_t n, uint32_t n_features,
                    int feature_major, float* out, cudaStream_t st);
// Heap-ordered forest for the shared-memory traversal: every tree padded to a
// complete tree of depth HEAP_DEPTH, HEAP_NODES 32-bit words per tree,
// 1-based (root 1, children 2h (left) and 2h + 1 (right)). Words 1 ..
// 2^HEAP_DEPTH - 1 are splits, words 2^HEAP_DEPTH .. HEAP_NODES - 1 the f32
// leaf values reached after exactly HEAP_DEPTH steps; a leaf shallower than
// that is reached through padding splits that always go left.
//
// Rows are binned against the forest's own sorted distinct thresholds of
// each feature: bin(x) = #{t <= x}, so x < t_k exactly when bin(x) < k + 1.
// Feature f's n thresholds sit at thr + thr_off[f] (a multiple of 16
// floats), padded with NaN (never <= x) to whole blocks of blk =
// 2^(feat_info[f] & 31) entries, blk the smallest power of two >= 16 with
// n <= 16 blk; spl[16 f + j] is the first threshold of block j + 1 (NaN past
// the last block), so that the bin search is a fixed sequence of compares. A split reads one bin column of the row tile: each
// feature has up to two numeric columns, one per missing-value direction
// (feat_col[2f]: NaN stored as the largest bin, which no split sends left;
// feat_col[2f + 1]: NaN stored as 0, which every split of that column sends
// left), or one categorical column (feat_col[2f]: min(category, 65534), NaN
// 0xFFFF). A numeric split word is K << 16 | column with K = rank + 1 of its
// threshold: left exactly when bin < K, i.e. bin * 65536 + 65535 < word. A
// categorical split word is index << 16 | 0x8000 | column, index into cat
// (start, size | default_left << 31) pairs over cat_words. Bins are u8 when
// no feature has more than 255 thresholds and nothing is categorical, else
// u16. Trees are grouped by output group in forest order (group_off[g] ..
// group_off[g + 1]).
constexpr int HEAP_DEPTH = 8;
constexpr uint32_t HEAP_NODES = 512;
constexpr uint32_t HEAP_MAX_COLS = 0x7FFFu;
constexpr uint32_t HEAP_SPLITTERS = 16;  // per feature, for the binning search
struct HeapForest {
    const uint32_t* nodes;
    const uint32_t* group_off;  // [n_groups + 1]
    const uint2* cat;
    const uint32_t* cat_words;
    const float* thr;           // per feature: distinct split thresholds, ascending, NaN-padded blocks
    const uint32_t* thr_off;    // [n_features + 1]
    const float* spl;           // [n_features][HEAP_SPLITTERS]
    const int32_t* feat_col;    // [2 * n_features], -1: no column
    const uint8_t* feat_info;   // [n_features]: log2(block) | categorical << 7
    const float* base;
    uint32_t n_trees, n_groups, n_features, n_cols;
    int has_cat;  // any categorical split
    int bins16;   // u16 bin columns (else u8)
};
// Rows per block of the shared-memory traversal for n rows of F features (0:
// the forest does not fit; use the node-list traversal).
uint32_t predict_heap_rows(const HeapForest& f, uint32_t n_features, uint64_t n);
// Bytes of bin-tile scratch the traversal of n rows needs; an upper bound for
// any n <= n_max.
size_t predict_heap_scratch(const HeapForest& f, uint32_t n_features, uint64_t n);
size_t predict_heap_scratch_max(const HeapForest& f, uint32_t n_features, uint64_t n_max);
constexpr uint32_t PREDICT_TILE_MAX = 768;  // largest traversal tile (rows)
// out [n_groups][n] raw margins of sample-major rows x [n][n_features];
// scratch: predict_heap_scratch bytes of device memory (16-byte aligned).
void launch_predict_heap(const HeapForest& f, const float* x, uint64_t n, uint32_t n_features, float* out,
                         void* scratch, cudaStream_t st);
// transform: 1 sigmoid, 2 softmax over [G][n]
void launch_transform(int transform, float* out, uint32_t G, uint64_t n, cudaStream_t st);
// a[i] = a[i] + b[i] (f32), i < n
void launch_add_f32(float* a, const float* b, uint64_t n, cudaStream_t st);
// gh[i] = (0, 0) where mask[i] == 0 (row sampling), i < n
void launch_zero_unsampled(float2* gh, const uint8_t* mask, uint64_t n, cudaStream_t st);
// GOSS codes (0 out, 1 kept, 2 kept and scaled by mult) applied to one
// output's grad/hess; mask [n] receives the kept rows.
void launch_goss_apply(float2* gh, const uint8_t* code, float mult, uint8_t* mask, uint64_t n, cudaStream_t st);

}  // namespace bst
