/*
 * boosters_c.h — C ABI of the B200-native GBDT engine (libboosters_b200.so).
 *
 * The entry points are the drop-in replacement for the Rust API of
 * egordm/boosters on its GBDT hot path (binning, training, prediction).
 * Every function that can fail returns a bst_status; the thread-local
 * message of the last failure is available from bst_last_error().
 * Handles are opaque, created and freed by the library. Output buffers are
 * owned by the caller. No function aborts the process.
 *
 * Array layouts follow the reference:
 *   features  feature-major  [n_features, n_samples]  f32 (NaN = missing)
 *   targets   output-major   [n_outputs,  n_samples]  f32
 *   weights                  [n_samples]              f32
 *   predictions group-major  [n_groups,   n_samples]  f32
 *
 * Reference interfaces are cited as crates/boosters/src/<file>:<line>.
 */
#ifndef BOOSTERS_C_H
#define BOOSTERS_C_H

#include <stddef.h>
#include <stdint.h>

#ifdef __cplusplus
extern "C" {
#endif

/* ------------------------------------------------------------------------ */
/* Status codes                                                             */
/* ------------------------------------------------------------------------ */

typedef int32_t bst_status;
#define BST_OK 0
#define BST_ERR_INVALID_ARGUMENT 1 /* null pointer, shape mismatch          */
#define BST_ERR_CONFIG 2           /* model/gbdt/config.rs:39 ConfigError   */
#define BST_ERR_EMPTY_DATASET 3    /* data/binned/dataset.rs:29 EmptyDataset */
#define BST_ERR_MISSING_TARGETS 4  /* model/gbdt/model.rs:127 (panics there) */
#define BST_ERR_UNSUPPORTED 5      /* feature outside the GPU engine's scope */
#define BST_ERR_CUDA 6             /* CUDA runtime error / no device        */
#define BST_ERR_OUT_OF_MEMORY 7
#define BST_ERR_TIMEOUT 8
#define BST_ERR_FORMAT 9 /* malformed model bytes                           */
#define BST_ERR_CHECK 10 /* checked build: a device bounds check failed      */

/* Message of the last failure on the calling thread ("" if none). */
const char* bst_last_error(void);
/* Library version string. */
const char* bst_version(void);
/* Device buffers released by the library (after a training call, a
 * server, a prediction) are kept per device for reuse, up to the
 * environment variable BST_DEVICE_CACHE_BYTES (default 8 GiB), and the
 * pinned host blocks of training calls up to 256 MiB; this frees both,
 * e.g. before another allocator on the same GPU needs the memory.
 * No reference counterpart. */
void bst_release_cached_memory(void);

/* ------------------------------------------------------------------------ */
/* Configuration  (model/gbdt/config.rs:111-226 GBDTConfig,                 */
/*                 data/binned/feature_analysis.rs:29-63 BinningConfig)     */
/* ------------------------------------------------------------------------ */

#define BST_OBJ_SQUARED 0  /* training/objectives/regression.rs:20       */
#define BST_OBJ_LOGISTIC 1 /* training/objectives/classification.rs:24   */
#define BST_OBJ_SOFTMAX 2  /* training/objectives/classification.rs:141  */
/* L1 loss: g = w sign(p - y), h = w; base score the weighted median; leaf
 * values renewed to the median residual of the leaf's rows
 * (objectives/mod.rs:352-409). */
#define BST_OBJ_ABSOLUTE 3 /* training/objectives/regression.rs:80       */
/* Pinball (quantile) loss, one output per alpha in quantile_alpha: g = w
 * (-alpha if p < y else 1 - alpha), h = w; base scores the weighted
 * alpha-quantiles; leaf values renewed to the alpha-quantile residual. */
#define BST_OBJ_PINBALL 4  /* training/objectives/regression.rs:129      */
#define BST_OBJ_PSEUDO_HUBER 5 /* regression.rs:183 (huber_delta)          */
#define BST_OBJ_POISSON 6  /* training/objectives/regression.rs:243      */
#define BST_OBJ_HINGE 7    /* training/objectives/classification.rs:88   */

#define BST_METRIC_DEFAULT -1 /* derived from the objective (training/metrics/mod.rs:213-232) */
#define BST_METRIC_NONE 0
#define BST_METRIC_RMSE 1
#define BST_METRIC_LOGLOSS 2
#define BST_METRIC_MLOGLOSS 3
#define BST_METRIC_MAE 4             /* metrics/regression.rs:55             */
#define BST_METRIC_MAPE 5            /* metrics/regression.rs:89             */
#define BST_METRIC_QUANTILE 6        /* metrics/regression.rs:126 (quantile_alpha) */
#define BST_METRIC_HUBER 7           /* metrics/regression.rs:216 (huber_delta) */
#define BST_METRIC_POISSON 8         /* metrics/regression.rs:176 deviance   */
#define BST_METRIC_MARGIN_ACCURACY 9 /* metrics/classification.rs:85         */

#define BST_GROWTH_DEPTHWISE 0 /* training/gbdt/expansion.rs:46 DepthWise */
#define BST_GROWTH_LEAFWISE 1  /* training/gbdt/expansion.rs:51 LeafWise  */

/* GPU extension: histogram accumulation precision.
 * FP32: f32 grad/hess accumulated exactly in 64-bit fixed point (the
 *       reference's f64 histograms, training/gbdt/histograms/ops.rs:42).
 * Q16 / Q8: grad/hess quantised per round and output to int16 / int8 with
 *       stochastic rounding (q = floor(v * Q / max|v| + u), Q = 32767 / 127,
 *       u from Philox4x32-10 keyed by `seed`, counter (row, output, round));
 *       histograms hold exact integer sums (32-bit per block, 64-bit per
 *       node), so the subtraction trick stays exact; splits are searched on
 *       the integer sums times max|v| / Q, and every leaf is solved in f64
 *       from the exact sums of its f32 grad/hess. Depth-wise and leaf-wise. */
#define BST_PRECISION_FP32 0
#define BST_PRECISION_Q16 1
#define BST_PRECISION_Q8 2

typedef struct bst_config {
    /* objective & metric */
    int32_t objective;    /* BST_OBJ_*                                      */
    uint32_t n_classes;   /* softmax only                                   */
    int32_t metric;       /* BST_METRIC_*                                   */
    /* boosting */
    uint32_t n_trees;     /* default 100                                    */
    float learning_rate;  /* default 0.3                                    */
    /* tree */
    int32_t growth_strategy; /* BST_GROWTH_*, default depth-wise            */
    uint32_t max_depth;      /* depth-wise, default 6                       */
    uint32_t max_leaves;     /* leaf-wise, default 31                       */
    uint32_t max_onehot_cats; /* default 4                                  */
    /* regularisation (training/gbdt/split/gain.rs:60-86 GainParams) */
    float lambda;           /* default 1.0                                  */
    float alpha;            /* default 0.0                                  */
    float min_child_weight; /* default 1.0                                  */
    float min_gain;         /* default 0.0                                  */
    uint32_t min_samples_leaf; /* default 1                                 */
    /* sampling                                                              */
    /* uniform row sampling (training/sampling/row.rs:168-210; the reference's
     * generator restated, seeded by `seed`): per output and round, rows
     * outside the sample get zero grad/hess. Default 1 (all rows). */
    float subsample;
    /* column sampling (training/sampling/column.rs): ceil(n * bytree) of the
     * columns per tree, ceil(that * bylevel) per depth, searched alone. The
     * reference draws them from OS entropy; the engine from a stream keyed
     * by (seed, round, output, depth), so runs repeat. Default 1 (all). */
    float colsample_bytree;
    float colsample_bylevel;
    /* binning */
    uint32_t max_bins;                   /* default 256                     */
    float sparsity_threshold;            /* default 0.9                     */
    int32_t enable_bundling;             /* default 1                       */
    uint32_t max_categorical_cardinality; /* default 0 (no auto-detect)     */
    uint64_t binning_sample_cnt;         /* default 200000                  */
    /* early stopping patience (model/gbdt/config.rs:210,366): < 0 means
     * None; None and 0 disable it. Supported by bst_gbdt_train only. */
    int32_t early_stopping_rounds;
    /* resources / reproducibility */
    uint64_t cache_size; /* default 8 (host histogram LRU of the reference) */
    uint64_t seed;       /* default 42                                      */
    int32_t verbosity;   /* default 0 (silent)                              */
    /* GPU extensions */
    int32_t precision;     /* BST_PRECISION_*, default FP32                 */
    int32_t batched;       /* 1: device-side frontier batching (default 1)  */
    int32_t cuda_graph;    /* 1: capture each boosting round in a CUDA graph */
    int32_t device;        /* CUDA device ordinal, default 0                */
    int32_t record_leaves; /* 1: keep per-tree row->leaf arrays (tests)     */
    int32_t phase_timings; /* 1: CUDA-event time of every training phase    */
                           /* (bst_model_train_timings); default 0: the     */
                           /* events cost ~0.3 ms per tree inside graphs    */
    /* Launch-shape autotuning of the batched depth-wise pipeline (histogram
     * items per block, histogram kernel variant, level-kernel grid): 1
     * (default) times candidate shapes on the run's first trees, which are
     * the same trees whatever the shape, and keeps the fastest; 0 uses the
     * built-in shape. autotune_cache (NULL: none) names a text file of
     * chosen shapes keyed by device, precision, bin layout and row count: a
     * cached choice skips the exploration, a new one is added. */
    int32_t autotune;
    const char* autotune_cache;
    /* Objective and metric parameters. quantile_alpha: n_quantiles values
     * in (0, 1) (BST_OBJ_PINBALL: one output each; BST_METRIC_QUANTILE),
     * copied at training; huber_delta > 0 (BST_OBJ_PSEUDO_HUBER,
     * BST_METRIC_HUBER), default 1. */
    const float* quantile_alpha;
    uint32_t n_quantiles;
    float huber_delta;
    /* GOSS row sampling (training/sampling/row.rs:214-280, the trainer's
     * RowSamplingParams::Goss): goss_top_rate > 0 turns it on (subsample
     * must then be 1). From round floor(1 / learning_rate) on, per output:
     * the top_rate share of rows by |grad x hess| are kept, other_rate x n
     * of the rest are drawn with the reference's adaptive probability
     * (seeded by `seed`) and their grad/hess scaled by (n - top) / other;
     * the remaining rows leave the round's tree. Default 0 / 0 (off). */
    float goss_top_rate;
    float goss_other_rate;
} bst_config;

/* Fill *cfg with the reference defaults (GBDTConfig::default(),
 * model/gbdt/config.rs:316). */
void bst_config_default(bst_config* cfg);

/* GBDTConfig::validate (model/gbdt/config.rs:252-310): returns BST_OK or
 * BST_ERR_CONFIG with the reference's message. */
bst_status bst_config_validate(const bst_config* cfg);

/* ------------------------------------------------------------------------ */
/* Dataset  (data/raw/dataset.rs:139 Dataset::from_array,                   */
/*           data/raw/dataset.rs:635 DatasetBuilder::add_categorical)       */
/* ------------------------------------------------------------------------ */

typedef struct bst_dataset bst_dataset;

/* Copies the host arrays. targets may be NULL (n_outputs ignored), weights
 * may be NULL (uniform), categorical_features lists feature indices that
 * the schema marks categorical. */
bst_status bst_dataset_create(const float* features, uint64_t n_features, uint64_t n_samples,
                              const float* targets, uint32_t n_outputs, const float* weights,
                              const uint32_t* categorical_features, uint32_t n_categorical,
                              bst_dataset** out);
/* As bst_dataset_create, but the features stay in the caller's array (no
 * copy): it must stay valid and unchanged while the dataset, and every
 * booster created from it, exists. Binning reads it directly (pinned host
 * memory gives an asynchronous device copy). Targets and weights are copied. */
bst_status bst_dataset_create_view(const float* features, uint64_t n_features, uint64_t n_samples,
                                   const float* targets, uint32_t n_outputs, const float* weights,
                                   const uint32_t* categorical_features, uint32_t n_categorical,
                                   bst_dataset** out);
void bst_dataset_free(bst_dataset* ds);
uint64_t bst_dataset_n_samples(const bst_dataset* ds);
uint64_t bst_dataset_n_features(const bst_dataset* ds);

/* ------------------------------------------------------------------------ */
/* Binned dataset  (data/binned/dataset.rs:207 BinnedDataset::from_dataset) */
/* ------------------------------------------------------------------------ */

typedef struct bst_binned bst_binned;

/* Feature analysis and bin bounds on the host, bin assignment on the GPU
 * (data/binned/dataset.rs:592-842). */
bst_status bst_binned_create(const bst_dataset* ds, const bst_config* cfg, bst_binned** out);
void bst_binned_free(bst_binned* b);
/* Effective columns (data/binned/dataset.rs:460 feature_views). */
uint32_t bst_binned_n_columns(const bst_binned* b);
/* Per effective column: source feature, bin count, categorical flag,
 * has-missing flag, default (missing) bin. Any pointer may be NULL. */
bst_status bst_binned_column_info(const bst_binned* b, uint32_t col, uint32_t* feature,
                                  uint32_t* n_bins, int32_t* is_categorical,
                                  int32_t* has_missing, uint32_t* default_bin);
/* Numeric upper bounds of a column (n_bins doubles; bin_mapper.rs:57). */
bst_status bst_binned_column_bounds(const bst_binned* b, uint32_t col, double* out);
/* Logical bin of every row of a column, copied back from the GPU. */
bst_status bst_binned_column_bins(const bst_binned* b, uint32_t col, uint16_t* out);

/* ------------------------------------------------------------------------ */
/* Training and prediction  (model/gbdt/model.rs:115 GBDTModel::train,      */
/*                           :217 predict, :238 predict_raw)                */
/* ------------------------------------------------------------------------ */

typedef struct bst_model bst_model;

/* n_threads keeps the reference's meaning for split tie-breaking:
 * 1 = sequential (first maximal feature wins), otherwise the rayon
 * reduction order (last maximal feature wins when >= 16 features,
 * training/gbdt/split/find.rs:125-129,266-269). val may be NULL; it is read
 * only with early stopping (cfg.early_stopping_rounds > 0) and a metric:
 * after every round the validation metric (without val: the training
 * metric; with BST_METRIC_NONE: NaN) is compared with the best so far, and
 * training stops once that many rounds passed without improvement, keeping
 * the trees up to the best round (training/gbdt/trainer.rs:344-401,
 * callback.rs:103-136). val then needs targets and at least the training
 * set's features. */
bst_status bst_gbdt_train(const bst_dataset* train, const bst_dataset* val,
                          const bst_config* cfg, uint32_t n_threads, bst_model** out);

/* out: caller-owned [n_groups, n_samples]. Transformed (sigmoid/softmax). */
bst_status bst_gbdt_predict(const bst_model* m, const bst_dataset* ds, uint32_t n_threads,
                            float* out);
/* out: caller-owned [n_groups, n_samples]. Raw margins. */
bst_status bst_gbdt_predict_raw(const bst_model* m, const bst_dataset* ds, uint32_t n_threads,
                                float* out);

/* Device-pointer prediction: features_dev is sample-major [n_rows,
 * n_features] f32 in device memory, out_dev is [n_groups, n_rows] f32 in
 * device memory; runs on `stream` (cudaStream_t, NULL = legacy stream)
 * without synchronising. raw != 0 skips the output transform. */
bst_status bst_gbdt_predict_device(const bst_model* m, const float* features_dev,
                                   uint64_t n_rows, uint64_t n_features, int32_t raw,
                                   float* out_dev, void* stream);

void bst_model_free(bst_model* m);
uint32_t bst_model_n_trees(const bst_model* m);
uint32_t bst_model_n_groups(const bst_model* m);
uint32_t bst_model_n_features(const bst_model* m);
/* Base scores, one per group. */
bst_status bst_model_base_scores(const bst_model* m, float* out);
/* Training predictions [n_groups, n_samples] left after the last round
 * (after early stopping: of the trees kept). */
bst_status bst_model_train_predictions(const bst_model* m, float* out);

/* Tree introspection (repr/gbdt/tree.rs:32-47 Tree SoA). */
bst_status bst_model_tree_info(const bst_model* m, uint32_t tree, uint32_t* n_nodes,
                               uint32_t* group, uint32_t* n_category_words);
/* Any pointer may be NULL; arrays have n_nodes entries. */
bst_status bst_model_tree_nodes(const bst_model* m, uint32_t tree, uint32_t* split_index,
                                float* threshold, uint32_t* left, uint32_t* right,
                                uint8_t* default_left, uint8_t* is_leaf, float* leaf_value,
                                uint8_t* split_type, float* gain, float* cover);
/* Categorical bitsets (repr/gbdt/categories.rs:29 CategoriesStorage). */
bst_status bst_model_tree_categories(const bst_model* m, uint32_t tree, uint32_t* seg_start,
                                     uint32_t* seg_size, uint32_t* words);
/* Training-time detail per node: the bin threshold chosen by the split scan
 * (0xFFFFFFFF for leaves / categorical) and the node's gradient and hessian
 * sums (f64). Any pointer may be NULL. */
bst_status bst_model_tree_train_info(const bst_model* m, uint32_t tree, uint32_t* split_bin,
                                     double* grad_sum, double* hess_sum);
/* With cfg.record_leaves: the tree node (leaf) each training row reached in
 * the row partition of that tree (training/gbdt/partition.rs:296). */
bst_status bst_model_tree_row_leaves(const bst_model* m, uint32_t tree, uint32_t* out);

/* Per-phase device timings of the last training call, in milliseconds:
 * [binning, gradients, histograms, split scan, partition, leaf update,
 *  other, total]. */
bst_status bst_model_train_timings(const bst_model* m, double* out8);
/* Work counters of the last training call: [kernel launches, histogram
 * launches, histogram row visits, histogram algorithmic bytes (rows x
 * (bin bytes per row + 12)), split-scan launches, partitioned rows]. */
bst_status bst_model_train_counters(const bst_model* m, uint64_t* out, uint32_t n);
/* The launch shape the batched pipeline trained with and how it was chosen
 * ("items=2,hist=0,grid=8 (cached)", "(built-in)", or "(explored: ...)" with
 * each candidate's median ms per tree; empty for other growth forms):
 * NUL-terminated into out[cap] (truncated), *len = its full length. */
bst_status bst_model_tune_info(const bst_model* m, char* out, uint64_t cap, uint64_t* len);

/* ------------------------------------------------------------------------ */
/* Component entry points (the reference's public building blocks)         */
/* ------------------------------------------------------------------------ */

/* BinMapper::value_to_bin (data/binned/bin_mapper.rs:210) on the GPU for one
 * mapper. missing_type: 0 None, 1 Zero, 2 NaN. For categorical mappers
 * pass the sorted category values in cats (bounds ignored). */
bst_status bst_bin_values(const double* bounds, uint32_t n_bounds, int32_t missing_type,
                          uint32_t default_bin, int32_t is_categorical, const int32_t* cats,
                          uint32_t n_cats, const float* values, uint64_t n_values,
                          uint32_t* out);

/* HistogramBuilder::build_gathered / build_contiguous
 * (training/gbdt/histograms/ops.rs:79,105) on the GPU. bins is
 * feature-major [n_features, n_samples] logical bins; rows selects the node
 * (NULL = all rows); out receives [sum(n_bins)][2] f64 (grad, hess). */
bst_status bst_histogram_build(const uint16_t* bins, const uint32_t* n_bins,
                               uint32_t n_features, uint64_t n_samples, const float* grad,
                               const float* hess, const uint32_t* rows, uint64_t n_rows,
                               double* out);

/* Incremental training: the boosting loop of GBDTTrainer::train
 * (training/gbdt/trainer.rs:242-401) over a GPU-resident binned copy of
 * `train`, a caller-chosen number of rounds per update. cfg.n_trees is
 * ignored; bst_booster_model snapshots the trees trained so far. Early
 * stopping (cfg.early_stopping_rounds > 0) is BST_ERR_UNSUPPORTED here. */
typedef struct bst_booster bst_booster;
bst_status bst_booster_create(const bst_dataset* train, const bst_config* cfg, uint32_t n_threads,
                              bst_booster** out);
bst_status bst_booster_update(bst_booster* b, uint32_t n_rounds);
uint32_t bst_booster_n_rounds(const bst_booster* b);
bst_status bst_booster_model(const bst_booster* b, bst_model** out);
/* Cumulative timings (as bst_model_train_timings) and counters (as
 * bst_model_train_counters) of every update so far. */
bst_status bst_booster_stats(const bst_booster* b, double* timings8, uint64_t* counters,
                             uint32_t n_counters);
void bst_booster_free(bst_booster* b);

/* TreeGrower::grow (training/gbdt/grower.rs:265) on caller-given gradients:
 * bins ds, grows one tree on the GPU and returns it as a one-tree model (base
 * score 0, identity transform). grad / hess have n_samples entries. */
bst_status bst_tree_grow(const bst_dataset* ds, const float* grad, const float* hess,
                         const bst_config* cfg, uint32_t n_threads, bst_model** out);

/* Model from explicit SoA trees (repr/gbdt/tree.rs:62 Tree::new and
 * repr/gbdt/forest.rs:31 Forest::push_tree). objective selects the output
 * transform. Child indices are local to the tree; the arrays are validated. */
bst_status bst_model_create(uint32_t n_groups, uint32_t n_features, int32_t objective,
                            const float* base_scores, bst_model** out);
bst_status bst_model_add_tree(bst_model* m, uint32_t group, uint32_t n_nodes,
                              const uint32_t* split_index, const float* threshold,
                              const uint32_t* left, const uint32_t* right,
                              const uint8_t* default_left, const uint8_t* is_leaf,
                              const float* leaf_value, const uint8_t* split_type,
                              const uint32_t* seg_start, const uint32_t* seg_size,
                              const uint32_t* words, uint32_t n_words);

/* A split as chosen by the split scan (training/gbdt/split/types.rs:34). */
typedef struct bst_split {
    uint32_t feature;      /* effective column                             */
    float gain;            /* -inf when invalid                            */
    int32_t default_left;
    int32_t is_categorical;
    uint32_t bin;          /* numerical: bins <= bin go left               */
    uint64_t left_cats[4]; /* categorical: bins going left (<= 256 bins)   */
} bst_split;

/* GreedySplitter::find_split (training/gbdt/split/find.rs:113) on the GPU
 * over a host histogram [sum(n_bins)][2] f64. */
bst_status bst_find_split(const double* histogram, const uint32_t* n_bins,
                          const int32_t* is_categorical, const int32_t* has_missing,
                          uint32_t n_features, double parent_grad, double parent_hess,
                          uint32_t parent_count, const bst_config* cfg, uint32_t n_threads,
                          bst_split* out);

/* The split search of bst_find_split, for callers that cannot allocate
 * device memory per call: a process whose device memory is already fully
 * reserved by another allocator, or latency-critical code that cannot afford
 * cudaMalloc/cudaFree (cudaFree synchronises the whole device). This entry
 * point has no counterpart in the reference.
 *
 * It allocates nothing. histogram_dev is a DEVICE array [sum(n_bins)][2] f64
 * (grad, hess); n_bins / is_categorical / has_missing are host arrays; the
 * result is written to the host struct *out after the work on `stream`
 * (cudaStream_t, NULL = legacy stream) has finished. Results equal those of
 * bst_find_split on the same histogram.
 *
 * Working memory is one fixed array in device global memory (about 1.1 MiB).
 * The CUDA runtime loads device code and arrays lazily: the first call on a
 * device loads this entry point's kernels and the array onto that device
 * and looks up the array's device address, which takes device memory once;
 * make that first call before the device's memory is fully reserved and
 * before any stream capture. The device then holds the array until the
 * process exits, and later calls allocate nothing.
 * Limits: n_features <= 1024 and sum(n_bins) <= 65536 (larger inputs return
 * BST_ERR_INVALID_ARGUMENT); categorical features with more than 256 bins
 * return BST_ERR_UNSUPPORTED, as in bst_find_split. Validation, n_features
 * == 0 (BST_OK, gain -inf) and error messages follow bst_find_split. Every
 * call shares the array: calls that overlap on the GPU (other streams, other
 * host threads) race and must be serialised by the caller. */
bst_status bst_find_split_noalloc(const double* histogram_dev, const uint32_t* n_bins,
                                  const int32_t* is_categorical, const int32_t* has_missing,
                                  uint32_t n_features, double parent_grad, double parent_hess,
                                  uint32_t parent_count, const bst_config* cfg, uint32_t n_threads,
                                  void* stream, bst_split* out);

/* The quantisation step of the Q16 / Q8 training modes, on the GPU, for one
 * output's host gradients (no counterpart in the reference, which trains on
 * f32 gradients only): q = floor(v * Q / max|v| + u) as documented at
 * BST_PRECISION_Q16, with max|v| over the finite values (|v| <= 3.4e38).
 * qg / qh [n] receive the integers; steps [4] = (Q / max|g|, Q / max|h|,
 * max|g| / Q, max|h| / Q), zeros for an all-zero input. */
bst_status bst_quantize_gradients(const float* grad, const float* hess, uint64_t n, int32_t precision,
                                  uint64_t seed, uint32_t round, uint32_t output, int32_t* qg,
                                  int32_t* qh, double* steps);

/* ------------------------------------------------------------------------ */
/* Model files: the reference's .bstr.json (JSON envelope bstr_version /     */
/* model_type / model, persist/json.rs:50-75) and .bstr (32-byte header,    */
/* MessagePack named-map payload, 16-byte trailer with CRC32C;              */
/* persist/envelope.rs:13-221, binary.rs:52-146) layouts of the model       */
/* schema (persist/schema.rs:27-150, convert.rs:78-420). Replace            */
/* GBDTModel::{to_bytes, to_json_bytes, from_bytes, from_json_bytes}        */
/* (packages/boosters-python/src/model/gbdt.rs:259-330) and Model::load     */
/* (persist/mod.rs:325).                                                   */
/* ------------------------------------------------------------------------ */

/* Library-allocated bytes: free with bst_buffer_free. .bstr payloads are
 * zstd-compressed MessagePack (format byte 0x02) at level 3, the reference's
 * default (persist/binary.rs:15-31, BinaryWriteOptions::default). zstd is
 * the system libzstd.so.1, loaded at first use; without it zstd payloads
 * return BST_ERR_UNSUPPORTED. */
#define BST_BSTR_DEFAULT_LEVEL 3
bst_status bst_model_to_json(const bst_model* model, int32_t pretty, uint8_t** out, uint64_t* len);
bst_status bst_model_to_bstr(const bst_model* model, uint8_t** out, uint64_t* len);
/* BinaryWriteOptions { compression_level } (persist/binary.rs:21-43): 0 =
 * plain MessagePack (format byte 0x01), 1-22 = zstd at that level (0x02);
 * other levels: BST_ERR_INVALID_ARGUMENT. */
bst_status bst_model_to_bstr_level(const bst_model* model, int32_t level, uint8_t** out, uint64_t* len);
/* Either layout (binary when the bytes start with "BSTR"). Malformed input:
 * BST_ERR_INVALID_ARGUMENT with the reason; linear or multi-value leaves:
 * BST_ERR_UNSUPPORTED. */
bst_status bst_model_from_bytes(const uint8_t* data, uint64_t len, bst_model** out);
void bst_buffer_free(void* p);
bst_status bst_model_write_json(const bst_model* model, const char* path, int32_t pretty);
bst_status bst_model_write_bstr(const bst_model* model, const char* path);
bst_status bst_model_write_bstr_level(const bst_model* model, const char* path, int32_t level);
bst_status bst_model_load(const char* path, bst_model** out);
/* CRC32C (Castagnoli) of the .bstr trailer. */
uint32_t bst_crc32c(const uint8_t* data, uint64_t len);

/* ------------------------------------------------------------------------ */
/* Serving: continuous batching over a device-resident forest (the engine's  */
/* serving loop; the reference predicts one call at a time through          */
/* Predictor::predict_into, inference/gbdt/predictor.rs:197).                */
/* ------------------------------------------------------------------------ */

typedef struct bst_server bst_server;

typedef struct bst_server_stats {
    uint64_t submitted;      /* requests accepted                            */
    uint64_t completed;      /* requests finished                            */
    uint64_t batches;        /* traversal launches                           */
    uint64_t rows;           /* rows predicted                               */
    uint64_t max_rows_seen;  /* largest batch                                */
    uint64_t max_batch_rows; /* batch capacity from the memory budget        */
    uint64_t h2d_bytes;      /* request rows copied to the device            */
    uint64_t h2d_ns;         /* device time of those copies (CUDA events)    */
} bst_server_stats;

/* Phases of one completed request, in ns: host steady-clock intervals and
 * device (CUDA event) durations. */
typedef struct bst_server_phase {
    uint64_t rows;                /* the request's rows                         */
    uint64_t batch_rows;          /* rows of the batch it shared                */
    uint64_t queue_ns;            /* submit -> copy issued (ring room)          */
    uint64_t copy_ns;             /* device time of its host->device copy       */
    uint64_t to_dispatch_ns;      /* copy issued -> its batch launched          */
    uint64_t kernel_ns;           /* device time of the batch's binning,        */
                                  /* traversal and transform                    */
    uint64_t d2h_ns;              /* device time of the batch's output copies   */
    uint64_t dispatch_to_done_ns; /* batch launched -> completion seen          */
} bst_server_phase;

/* The model stays device-resident and must outlive the server. The device
 * memory of the in-flight batches (3 slots of input + output rows) is bounded
 * by mem_budget_bytes; max_batch_rows caps a batch further (0: requests
 * coalesce up to one full wave of the traversal, 768 rows per SM, i.e.
 * 113,664 on a 148-SM B200, and a single request may fill a whole slot).
 * raw != 0: margins; else the objective's transform. */
bst_status bst_server_create(const bst_model* model, uint64_t mem_budget_bytes, uint64_t max_batch_rows,
                             int32_t raw, bst_server** out);
/* Queues n_rows sample-major rows [n_rows, n_features] f32 for prediction
 * into out [n_groups, n_rows]; both buffers are the caller's, in host or
 * device memory of the model's GPU (unified addressing tells them apart),
 * and must stay valid until bst_server_wait returns for the ticket (host
 * buffers should be pinned for asynchronous copies; device rows skip the
 * PCIe transfer). Requests larger than one batch are rejected with
 * BST_ERR_INVALID_ARGUMENT. Returns at once. */
bst_status bst_server_submit(bst_server* server, const float* rows, uint64_t n_rows, float* out,
                             uint64_t* ticket);
/* Waits for a ticket (timeout_ms < 0: no limit; BST_ERR_TIMEOUT leaves the
 * ticket valid). On return the ticket is retired; submit_ns / done_ns (may
 * be NULL) receive the server's steady-clock times of submission and of
 * completion of the request's batch. One waiter per ticket. */
bst_status bst_server_wait(bst_server* server, uint64_t ticket, int64_t timeout_ms, uint64_t* submit_ns,
                           uint64_t* done_ns);
bst_status bst_server_stats_get(bst_server* server, bst_server_stats* out);
/* Moves up to max phase records of completed requests (oldest first; the
 * server keeps at most 2^20 until they are taken) into out; *n = how many. */
bst_status bst_server_trace(bst_server* server, bst_server_phase* out, uint64_t max, uint64_t* n);
/* Load replay (capacity planning and latency measurement): submits n_req
 * requests from a native thread at steady-clock offsets arrival_ns[i]
 * (non-decreasing, from a start 1 ms after the call), request i being rows
 * [row_off[i], row_off[i] + n_rows[i]) of the sample-major pool, its
 * predictions written to out + (i % ring) * ring_stride (a slot is reused
 * once the request ring positions earlier has completed). latency_ns[i] =
 * completion of the request's batch - its scheduled arrival; *span_ns (may
 * be NULL) = last completion - first scheduled arrival. */
bst_status bst_server_replay(bst_server* server, const float* pool, uint64_t pool_rows, uint64_t n_req,
                             const uint64_t* arrival_ns, const uint64_t* row_off, const uint64_t* n_rows, float* out,
                             uint64_t ring, uint64_t ring_stride, uint64_t* latency_ns, uint64_t* span_ns);
/* Completes every queued request, then frees the server. */
void bst_server_free(bst_server* server);

/* ------------------------------------------------------------------------ */
/* Seeded synthetic workloads (host, counter-based; identical bytes for any */
/* consumer). Feature-major x [n_features, n_samples], y [n_samples].       */
/* ------------------------------------------------------------------------ */

/* Regression: x ~ N(0,1); y = x.w + 0.1 N(0,1), w ~ N(0,1) on the first
 * n_informative features and 0 elsewhere. */
bst_status bst_synth_regression(uint64_t n_samples, uint64_t n_features,
                                uint64_t n_informative, uint64_t seed, uint64_t stream,
                                float* x, float* y);
/* Binary: even columns N(0,1), odd U(0,1); columns < n_nan_cols get 10% NaN;
 * y ~ Bernoulli(sigmoid(sum of 10 pairwise products + N(0,0.5))), NaN->0 in
 * the label formula. */
bst_status bst_synth_binary(uint64_t n_samples, uint64_t n_features, uint64_t n_nan_cols,
                            uint64_t seed, uint64_t stream, float* x, float* y);
/* Multiclass with categoricals: n_numeric N(0,1) columns then n_categorical
 * columns with cardinality U{4..64} and Zipf(1.2) frequencies (values
 * 0..K-1); y = argmax_c(W_c.x_num + E_c[j][x_cat_j] + Gumbel). */
bst_status bst_synth_multiclass(uint64_t n_samples, uint64_t n_numeric, uint64_t n_categorical,
                                uint64_t n_classes, uint64_t seed, uint64_t stream, float* x,
                                float* y);

/* ------------------------------------------------------------------------ */
/* Metrics (training/metrics/regression.rs:17, classification.rs:13,332)    */
/* ------------------------------------------------------------------------ */

/* preds [n_groups, n_samples] (probabilities for logloss/mlogloss, raw
 * margins for the margin accuracy). Metric::compute (metrics/mod.rs:238-270).
 * BST_METRIC_QUANTILE needs bst_metric_ex. */
bst_status bst_metric(int32_t metric, const float* preds, uint32_t n_groups, uint64_t n_samples,
                      const float* targets, const float* weights, double* out);
/* The same with the quantile metric's alphas (one per group) and the Huber
 * metric's delta. */
bst_status bst_metric_ex(int32_t metric, const float* preds, uint32_t n_groups, uint64_t n_samples,
                         const float* targets, const float* weights, const float* quantile_alpha,
                         uint32_t n_quantiles, float huber_delta, double* out);

/* ------------------------------------------------------------------------ */
/* Checked build (no counterpart in the reference, whose debug_assert region */
/* checks in histograms/slices.rs:91-110 play this role on the CPU)          */
/* ------------------------------------------------------------------------ */

/* libboosters_b200_checked.so is the same library compiled with device-side
 * bounds checks at the accesses whose index is read from device memory (row
 * ids of the histogram gather and leaf update, partition chunks and scatter
 * destinations, leaf chunks, traversal node links). A failed check is
 * counted and its access skipped; no kernel traps. bst_gbdt_train returns
 * BST_ERR_CHECK when its kernels recorded a violation. This reads and clears
 * the record of `device`: the number of violations and the first one's site
 * (1 partition chunk, 2 partition scatter, 3 leaf chunk, 4 leaf-update row,
 * 5 histogram-gather row, 6 traversal node), index and bound. The normal
 * library returns BST_ERR_UNSUPPORTED. */
bst_status bst_check_report(int32_t device, uint64_t* violations, uint32_t* site, uint64_t* index,
                            uint64_t* bound);

#ifdef __cplusplus
}
#endif

#endif /* BOOSTERS_C_H */
