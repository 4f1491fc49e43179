/*
 * oracle.h — CPU restatement of egordm/boosters' GBDT hot path.
 *
 * TEST INFRASTRUCTURE ONLY. This library is the checker that the tests,
 * the smoke check and the CPU-baseline leg of bench.py compare the CUDA
 * engine against. The engine never links, loads or calls it.
 *
 * It follows the Rust CPU path with sequential (n_threads = 1) arithmetic:
 * f64 histogram sums in partition order, the exact LRU histogram pool and
 * the stable row partition. f32 exp is the correctly rounded value (glibc's
 * f64 exp rounded once); the reference calls the platform expf, which glibc
 * bounds by 0.502 ULP, so the two may differ in the last bit for rare inputs. The rayon tie-breaking of the
 * parallel split search is emulated when n_threads != 1, and the histogram
 * build / split search can use OpenMP threads without changing any result.
 */
#ifndef BST_ORACLE_H
#define BST_ORACLE_H

#include <stdint.h>

#include "../include/boosters_c.h"

#ifdef __cplusplus
extern "C" {
#endif

typedef struct orc_model orc_model;
typedef struct orc_binned orc_binned;

/* ---- binning (data/binned/dataset.rs:207) ---- */
int orc_bin(const float* x_fm, uint64_t n_features, uint64_t n_samples,
            const uint32_t* cat_idx, uint32_t n_cat, const bst_config* cfg, orc_binned** out);
void orc_binned_free(orc_binned* b);
uint32_t orc_binned_n_columns(const orc_binned* b);
void orc_binned_column_info(const orc_binned* b, uint32_t col, uint32_t* feature,
                            uint32_t* n_bins, int32_t* is_cat, int32_t* has_missing,
                            uint32_t* default_bin);
void orc_binned_column_bounds(const orc_binned* b, uint32_t col, double* out);
void orc_binned_column_bins(const orc_binned* b, uint32_t col, uint16_t* out);

/* BinMapper::value_to_bin for an explicit mapper (bin_mapper.rs:210). */
uint32_t orc_value_to_bin(const double* bounds, uint32_t n_bounds, int32_t missing_type,
                          uint32_t default_bin, int32_t is_cat, const int32_t* cats,
                          uint32_t n_cats, double value);

/* ---- components ---- */
double orc_gain_full(double gl, double hl, double gr, double hr, double gp, double hp,
                     float lambda, float min_gain); /* gain.rs:102 (returns the f32 value) */
float orc_leaf_weight(double g, double h, float lambda, float alpha); /* gain.rs:151 */
int orc_is_valid_split(double hl, double hr, uint32_t cl, uint32_t cr, float min_child_weight,
                       uint32_t min_samples_leaf); /* gain.rs:123 */
/* HistogramBuilder (ops.rs:79-127): bins feature-major u16; rows may be NULL. */
void orc_histogram_build(const uint16_t* bins, const uint32_t* n_bins, uint32_t n_features,
                         uint64_t n_samples, const float* grad, const float* hess,
                         const uint32_t* rows, uint64_t n_rows, double* out);
/* GreedySplitter::find_split (find.rs:113). */
void orc_find_split(const double* hist, const uint32_t* n_bins, const int32_t* is_cat,
                    const int32_t* has_missing, uint32_t n_features, double pg, double ph,
                    uint32_t pc, const bst_config* cfg, uint32_t n_threads, bst_split* out);
/* Objective gradients (objectives/mod.rs:236) for [n_outputs, n] preds. */
void orc_gradients(int32_t objective, uint32_t n_outputs, const float* preds, const float* y,
                   const float* w, uint64_t n, float* grad, float* hess);
void orc_base_score(int32_t objective, uint32_t n_outputs, const float* y, const float* w,
                    uint64_t n, float* out);
/* OutputTransform::transform_inplace (transform.rs:61); transform: 0 id, 1 sigmoid, 2 softmax */
void orc_transform(int32_t transform, float* preds, uint32_t n_groups, uint64_t n);
double orc_metric(int32_t metric, const float* preds, uint32_t n_groups, uint64_t n,
                  const float* y, const float* w);
/* The same with the objective's parameters (pinball alphas, Huber delta)
 * taken from cfg. */
void orc_gradients_cfg(const bst_config* cfg, uint32_t n_outputs, const float* preds, const float* y,
                       const float* w, uint64_t n, float* grad, float* hess);
void orc_base_score_cfg(const bst_config* cfg, uint32_t n_outputs, const float* y, const float* w, uint64_t n,
                        float* out);
double orc_metric_cfg(int32_t metric, const bst_config* cfg, const float* preds, uint32_t n_groups, uint64_t n,
                      const float* y, const float* w);
/* GOSS (sampling/row.rs:214-280): the sampler seeded by `seed`, called
 * `calls` times on g / h (scaled in place each call); mask of the last call,
 * returns its sampled count. */
uint64_t orc_goss(float* g, float* h, uint64_t n, float top_rate, float other_rate, uint64_t seed, uint32_t calls,
                  uint8_t* mask);
/* Leaf renewing's quantile (utils.rs:17-135): w NULL for the unweighted
 * rank rule, else the weighted step rule. NaN for n = 0. */
float orc_leaf_quantile(const float* v, const float* w, uint64_t n, float alpha);

/* ---- quantised gradients (the engine's int8 / int16 mode; no reference
 * counterpart). Philox4x32-10 (Salmon et al., SC 2011) and the stochastic
 * rounding q = floor(v * Q / max|v| + u), Q = 127 (Q8) or 32767 (Q16),
 * u = word / 2^32 of philox(ctr = (row, output, round, 0x51A7E5ED),
 * key = (seed lo, seed hi)): word 0 for grad, word 1 for hess.
 * steps = (Q / max|g|, Q / max|h|, max|g| / Q, max|h| / Q). */
void orc_philox4x32_10(const uint32_t ctr[4], const uint32_t key[2], uint32_t out[4]);
void orc_quantize(const float* grad, const float* hess, uint64_t n, int32_t precision, uint64_t seed,
                  uint32_t round, uint32_t output, int32_t* qg, int32_t* qh, double* steps);

/* ---- training (model/gbdt/model.rs:115) ---- */
/* Returns 0 on success, else a bst_status code. record_leaves keeps per-tree
 * row->leaf arrays. omp_threads = threads the histogram build / split search
 * may use (results are identical for any value). */
int orc_train(const float* x_fm, uint64_t n_features, uint64_t n_samples, const float* y,
              uint32_t y_rows, const float* w, const uint32_t* cat_idx, uint32_t n_cat,
              const bst_config* cfg, uint32_t n_threads, int record_leaves, int omp_threads,
              orc_model** out);
/* Same, but stop after max_trees trees (bounded CPU-baseline samples). */
int orc_train_limited(const float* x_fm, uint64_t n_features, uint64_t n_samples,
                      const float* y, uint32_t y_rows, const float* w, const uint32_t* cat_idx,
                      uint32_t n_cat, const bst_config* cfg, uint32_t n_threads,
                      int record_leaves, int omp_threads, uint32_t max_trees, orc_model** out);
void orc_model_free(orc_model* m);
uint32_t orc_model_n_trees(const orc_model* m);
uint32_t orc_model_n_groups(const orc_model* m);
void orc_model_base_scores(const orc_model* m, float* out);
void orc_model_train_predictions(const orc_model* m, float* out);
void orc_tree_info(const orc_model* m, uint32_t t, uint32_t* n_nodes, uint32_t* group,
                   uint32_t* n_cat_words);
void orc_tree_nodes(const orc_model* m, uint32_t t, uint32_t* split_index, float* threshold,
                    uint32_t* left, uint32_t* right, uint8_t* default_left, uint8_t* is_leaf,
                    float* leaf_value, uint8_t* split_type, float* gain, float* cover);
void orc_tree_categories(const orc_model* m, uint32_t t, uint32_t* seg_start,
                         uint32_t* seg_size, uint32_t* words);
void orc_tree_train_info(const orc_model* m, uint32_t t, uint32_t* split_bin, double* grad_sum,
                         double* hess_sum);
void orc_tree_row_leaves(const orc_model* m, uint32_t t, uint32_t* out);
/* Seconds spent in tree growth + prediction updates (binning excluded). */
double orc_model_train_seconds(const orc_model* m);
double orc_model_binning_seconds(const orc_model* m);
/* Seconds of tree t: its growth and prediction update (the first tree of a
 * round also carries that round's gradient computation). */
double orc_model_tree_seconds(const orc_model* m, uint32_t t);

/* ---- prediction (model/gbdt/model.rs:217-258) ---- */
int orc_predict(const orc_model* m, const float* x_fm, uint64_t n_features, uint64_t n_samples,
                int raw, float* out);
/* Sample-major rows [n, F] (the serving layout). */
int orc_predict_rows(const orc_model* m, const float* x_sm, uint64_t n_features,
                     uint64_t n_samples, int raw, int omp_threads, float* out);

/* TreeGrower::grow (training/gbdt/grower.rs:265) on given gradients: one
 * tree, returned as a one-tree model (base score 0, identity transform). */
int orc_grow_tree(const float* x_fm, uint64_t n_features, uint64_t n_samples, const float* grad,
                  const float* hess, const bst_config* cfg, uint32_t n_threads, orc_model** out);
/* Model from explicit SoA trees (repr/gbdt/tree.rs:62 Tree::new, forest.rs push_tree). */
int orc_model_create(uint32_t n_groups, uint32_t n_features, int32_t objective, const float* base,
                     orc_model** out);
int orc_model_add_tree(orc_model* m, uint32_t group, uint32_t n_nodes, const uint32_t* split_index,
                       const float* threshold, const uint32_t* left, const uint32_t* right,
                       const uint8_t* default_left, const uint8_t* is_leaf, const float* leaf_value,
                       const uint8_t* split_type, const uint32_t* seg_start, const uint32_t* seg_size,
                       const uint32_t* words, uint32_t n_words);

const char* orc_last_error(void);
void orc_config_default(bst_config* cfg);
/* seeded workloads (boosters_b200/csrc/synth_gen.h): 0 on success */
int orc_synth_regression(uint64_t n, uint64_t F, uint64_t n_inf, uint64_t seed, uint64_t stream, float* x,
                         float* y);
int orc_synth_binary(uint64_t n, uint64_t F, uint64_t n_nan_cols, uint64_t seed, uint64_t stream, float* x,
                     float* y);
int orc_synth_multiclass(uint64_t n, uint64_t n_num, uint64_t n_cat, uint64_t C, uint64_t seed, uint64_t stream,
                         float* x, float* y);

/* Row-sampling generator (test infrastructure): n raw Xoshiro256++ outputs
 * from `state`, and `draws` consecutive uniform row samples (masks
 * [draws][n]) of a sampler seeded with `seed` (training/sampling/row.rs). */
void orc_xoshiro256pp(const uint64_t state[4], uint32_t n, uint64_t* out);
void orc_row_sample(uint64_t seed, uint64_t n, float rate, uint32_t draws, uint8_t* masks);

#ifdef __cplusplus
}
#endif

#endif
