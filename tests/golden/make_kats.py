"""Writes tests/golden/kats.json: known-answer vectors of the reference's own
unit tests for the GBDT hot path, transcribed from the Rust test modules
(crates/boosters/src/..., cited per case). Run: python tests/golden/make_kats.py
"""
import json
import os

NAN = "nan"

KATS = {
    "value_to_bin": [
        # data/binned/bin_mapper.rs:349-377 test_numerical_value_to_bin
        {"src": "data/binned/bin_mapper.rs:365", "bounds": [1.0, 2.0, 3.0, 4.0], "missing": 0, "default_bin": 0,
         "values": [0.5, 1.0, 1.5, 2.0, 2.5, 3.0, 3.5], "bins": [0, 0, 1, 1, 2, 2, 3]},
        # bin_mapper.rs:414-428 test_numerical_with_nan_missing
        {"src": "data/binned/bin_mapper.rs:414", "bounds": [1.0, 2.0, 3.0, "inf"], "missing": 2, "default_bin": 3,
         "values": [NAN], "bins": [3]},
        # bin_mapper.rs:431-444 test_numerical_with_zero_missing
        {"src": "data/binned/bin_mapper.rs:431", "bounds": [1.0, 2.0, 3.0], "missing": 1, "default_bin": 0,
         "values": [0.0, 1.5], "bins": [0, 1]},
        # bin_mapper.rs:457-468 test_categorical_value_to_bin (unknown -> 0)
        {"src": "data/binned/bin_mapper.rs:457", "cats": [10, 20, 30], "missing": 0, "default_bin": 0,
         "values": [10.0, 20.0, 30.0, 99.0], "bins": [0, 1, 2, 0]},
        # bin_mapper.rs:544-553 test_is_trivial: empty mapper maps everything to bin 0
        {"src": "data/binned/bin_mapper.rs:549", "bounds": [], "missing": 0, "default_bin": 0,
         "values": [1.0, NAN], "bins": [0, 0]},
    ],
    "gain": [
        # training/gbdt/split/gain.rs:175-188 test_gain_computation (tolerance 0.01)
        {"src": "training/gbdt/split/gain.rs:175", "gl": 10.0, "hl": 5.0, "gr": -10.0, "hr": 5.0, "gp": 0.0,
         "hp": 10.0, "lambda": 1.0, "min_gain": 0.0, "expect": 16.666, "tol": 0.01},
    ],
    "valid_split": [
        # gain.rs:191-201 test_valid_split_check (min_child_weight 5, min_samples_leaf 10)
        {"src": "training/gbdt/split/gain.rs:191", "hl": 5.0, "hr": 5.0, "cl": 10, "cr": 10, "mcw": 5.0, "msl": 10,
         "expect": True},
        {"src": "training/gbdt/split/gain.rs:199", "hl": 4.0, "hr": 5.0, "cl": 10, "cr": 10, "mcw": 5.0, "msl": 10,
         "expect": False},
        {"src": "training/gbdt/split/gain.rs:200", "hl": 5.0, "hr": 5.0, "cl": 9, "cr": 10, "mcw": 5.0, "msl": 10,
         "expect": False},
    ],
    "leaf_weight": [
        # gain.rs:204-210 test_leaf_weight_no_l1
        {"src": "training/gbdt/split/gain.rs:204", "g": -10.0, "h": 5.0, "lambda": 1.0, "alpha": 0.0,
         "expect": 1.666, "tol": 0.01},
        # gain.rs:213-227 test_leaf_weight_with_l1
        {"src": "training/gbdt/split/gain.rs:220", "g": -1.0, "h": 5.0, "lambda": 1.0, "alpha": 2.0,
         "expect": 0.0, "tol": 0.0},
        {"src": "training/gbdt/split/gain.rs:224", "g": -10.0, "h": 5.0, "lambda": 1.0, "alpha": 2.0,
         "expect": 1.333, "tol": 0.01},
    ],
    "histogram": [
        # training/gbdt/histograms/ops.rs:403-428 test_build_histogram_basic
        {"src": "training/gbdt/histograms/ops.rs:403", "bins": [[0, 1, 0, 2, 1, 0]], "n_bins": [3],
         "grad": [1, 2, 3, 4, 5, 6], "hess": [0.5, 1.0, 1.5, 2.0, 2.5, 3.0], "rows": None,
         "expect": [[10.0, 5.0], [7.0, 3.5], [4.0, 2.0]]},
        # ops.rs:431-460 test_build_histogram_with_indices
        {"src": "training/gbdt/histograms/ops.rs:431", "bins": [[0, 1, 2, 0, 1, 2]], "n_bins": [3],
         "grad": [1, 2, 3, 4, 5, 6], "hess": [1, 1, 1, 1, 1, 1], "rows": [0, 2, 4],
         "expect": [[1.0, 1.0], [5.0, 1.0], [3.0, 1.0]]},
    ],
    "histogram_multi": [
        # ops.rs:486-518 test_build_histograms_multi_feature (100 rows, bins (i+k)%4, grad i)
        {"src": "training/gbdt/histograms/ops.rs:486", "n": 100, "n_features": 3, "n_bins": 4,
         "expect_f0_bin0_grad": float(sum(i for i in range(100) if i % 4 == 0))},
    ],
    "find_split": [
        # training/gbdt/split/find.rs:660-685 test_numerical_split_simple
        {"src": "training/gbdt/split/find.rs:660", "hist": [[10, 5], [5, 5], [-5, 5], [-10, 5]], "n_bins": [4],
         "is_cat": [0], "has_missing": [0], "pg": 0.0, "ph": 20.0, "pc": 20, "max_onehot_cats": 4,
         "expect_valid": True, "expect_feature": 0},
        # find.rs:688-712 test_categorical_onehot (category 1 goes left)
        {"src": "training/gbdt/split/find.rs:688", "hist": [[5, 5], [-10, 5], [5, 5]], "n_bins": [3],
         "is_cat": [1], "has_missing": [0], "pg": 0.0, "ph": 15.0, "pc": 15, "max_onehot_cats": 4,
         "expect_valid": True, "expect_feature": 0, "expect_categorical": True, "expect_left_contains": [1]},
        # find.rs:715-731 test_categorical_sorted (max_onehot_cats 2 forces the sorted strategy)
        {"src": "training/gbdt/split/find.rs:715", "hist": [[5, 3], [3, 3], [0, 3], [-3, 3], [-5, 3]],
         "n_bins": [5], "is_cat": [1], "has_missing": [0], "pg": 0.0, "ph": 15.0, "pc": 15, "max_onehot_cats": 2,
         "expect_valid": True, "expect_feature": 0, "expect_categorical": True},
        # find.rs:734-772 test_find_split_multiple_features (feature 1 strongest)
        {"src": "training/gbdt/split/find.rs:734",
         "hist": [[1, 5], [0, 5], [-1, 5], [10, 5], [0, 5], [-10, 5], [3, 5], [0, 5], [-3, 5]],
         "n_bins": [3, 3, 3], "is_cat": [0, 0, 0], "has_missing": [0, 0, 0], "pg": 0.0, "ph": 45.0, "pc": 45,
         "max_onehot_cats": 4, "expect_valid": True, "expect_feature": 1},
        # find.rs:775-792 test_invalid_single_bin
        {"src": "training/gbdt/split/find.rs:775", "hist": [[5, 5]], "n_bins": [1], "is_cat": [0],
         "has_missing": [0], "pg": 5.0, "ph": 5.0, "pc": 5, "max_onehot_cats": 4, "expect_valid": False},
    ],
    "objective": [
        # training/objectives/classification.rs:246-262 logistic_gradient_at_zero
        {"src": "training/objectives/classification.rs:246", "objective": 1, "preds": [[0.0]], "y": [1.0],
         "w": None, "grad": [[-0.5]], "hess": [[0.25]], "tol": 1e-6},
        # classification.rs:276-297 logistic_weighted
        {"src": "training/objectives/classification.rs:276", "objective": 1, "preds": [[0.0, 0.0]], "y": [1.0, 0.0],
         "w": [2.0, 0.5], "grad": [[-1.0, 0.25]], "hess": None, "tol": 1e-6},
        # regression.rs:461-473 absolute_loss_basic
        {"src": "training/objectives/regression.rs:461", "objective": 3, "preds": [[1.0, 2.0, 3.0]],
         "y": [0.5, 2.5, 2.5], "w": None, "grad": [[1.0, -1.0, 1.0]], "hess": None, "tol": 1e-6},
        # regression.rs:373-407 pinball_loss_quantiles, alpha 0.1 and 0.9
        {"src": "training/objectives/regression.rs:384", "objective": 4, "alpha": [0.1], "preds": [[1.0, 2.0]],
         "y": [2.0, 1.0], "w": None, "grad": [[-0.1, 0.9]], "hess": [[1.0, 1.0]], "tol": 1e-6},
        {"src": "training/objectives/regression.rs:397", "objective": 4, "alpha": [0.9], "preds": [[1.0, 2.0]],
         "y": [2.0, 1.0], "w": None, "grad": [[-0.9, 0.1]], "hess": [[1.0, 1.0]], "tol": 1e-6},
        # regression.rs:440-459 pinball_loss_median
        {"src": "training/objectives/regression.rs:440", "objective": 4, "alpha": [0.5], "preds": [[1.0, 2.0, 3.0]],
         "y": [0.5, 2.5, 2.5], "w": None, "grad": [[0.5, -0.5, 0.5]], "hess": None, "tol": 1e-6},
        # regression.rs:476-494 pseudo_huber_near_zero (tolerances 1e-3 / 1e-2)
        {"src": "training/objectives/regression.rs:476", "objective": 5, "delta": 1.0, "preds": [[0.01]],
         "y": [0.0], "w": None, "grad": [[0.01]], "hess": None, "tol": 1e-3},
        {"src": "training/objectives/regression.rs:493", "objective": 5, "delta": 1.0, "preds": [[0.01]],
         "y": [0.0], "w": None, "grad": None, "hess": [[1.0]], "tol": 1e-2},
        # regression.rs:496-509 poisson_loss_basic
        {"src": "training/objectives/regression.rs:496", "objective": 6, "preds": [[0.0]], "y": [2.0], "w": None,
         "grad": [[-1.0]], "hess": [[1.0]], "tol": 1e-6},
        # classification.rs:300-326 hinge_loss_margin (margin 2: grad 0; margin -0.5: grad -1)
        {"src": "training/objectives/classification.rs:314", "objective": 7, "preds": [[2.0]], "y": [1.0],
         "w": None, "grad": [[0.0]], "hess": None, "tol": 1e-6},
        {"src": "training/objectives/classification.rs:325", "objective": 7, "preds": [[-0.5]], "y": [1.0],
         "w": None, "grad": [[-1.0]], "hess": None, "tol": 1e-6},
    ],
    "base_score": [
        # classification.rs:264-274 logistic_base_score: 50% positives -> 0
        {"src": "training/objectives/classification.rs:264", "objective": 1, "n_outputs": 1, "y": [0, 0, 1, 1],
         "expect": [0.0], "tol": 1e-6},
        # classification.rs:343-365 softmax_base_score: class priors 1/2, 1/4, 1/4
        {"src": "training/objectives/classification.rs:343", "objective": 2, "n_outputs": 3, "y": [0, 0, 1, 2],
         "expect": [-0.6931472, -1.3862944, -1.3862944], "tol": 1e-5},
        # regression.rs:512-523 poisson_loss_base_score: ln(2.5)
        {"src": "training/objectives/regression.rs:512", "objective": 6, "n_outputs": 1, "y": [1, 2, 3, 4],
         "expect": [0.91629073], "tol": 1e-6},
    ],
    "leaf_quantile": [
        # utils.rs:362-456: the unweighted rank rule and the weighted step rule
        {"src": "utils.rs:377", "values": [], "weights": None, "alpha": 0.5, "expect": NAN},
        {"src": "utils.rs:364", "values": [], "weights": [], "alpha": 0.5, "expect": NAN},
        {"src": "utils.rs:384", "values": [42.0], "weights": None, "alpha": 0.5, "expect": 42.0},
        {"src": "utils.rs:392", "values": [1.0, 2.0, 3.0, 4.0, 5.0], "weights": None, "alpha": 0.5, "expect": 3.0},
        {"src": "utils.rs:401", "values": [1.0, 2.0, 3.0, 4.0], "weights": None, "alpha": 0.25, "expect": 1.0},
        {"src": "utils.rs:411", "values": [1.0, 2.0, 3.0, 4.0], "weights": None, "alpha": 0.75, "expect": 3.0},
        {"src": "utils.rs:421", "values": [5.0, 1.0, 3.0, 2.0, 4.0], "weights": None, "alpha": 0.5, "expect": 3.0},
        {"src": "utils.rs:430", "values": [1.0, 2.0, 3.0], "weights": [1.0, 2.0, 1.0], "alpha": 0.5, "expect": 2.0},
        {"src": "utils.rs:445", "values": [1.0, 10.0], "weights": [1.0, 9.0], "alpha": 0.5, "expect": 10.0},
    ],
    "partition": [
        # training/gbdt/partition.rs:391-463: f0 alternating, f1 halves; split f1 at bin 0, then f0 at bin 0
        {"src": "training/gbdt/partition.rs:391", "features": [[0, 1, 0, 1, 0, 1, 0, 1], [0, 0, 0, 0, 1, 1, 1, 1]],
         "split_feature": 1, "expect_left_rows": [0, 1, 2, 3]},
        {"src": "training/gbdt/partition.rs:437", "features": [[0, 1, 0, 1, 0, 1, 0, 1], [0, 0, 0, 0, 1, 1, 1, 1]],
         "split_feature": 0, "expect_left_rows": [0, 2, 4, 6]},
    ],
    "threshold_translation": [
        # training/gbdt/grower.rs:812-842: values [0, 1]; split bin 0; threshold = next_up(f32(0.5))
        {"src": "training/gbdt/grower.rs:812", "values": [0.0, 1.0], "upper": 0.5, "threshold_above_upper": True},
    ],
    "traversal": [
        # inference/gbdt/traversal.rs:278-330: num(0, 0.5, default L) -> leaf 1.0 / leaf 2.0
        {"src": "inference/gbdt/traversal.rs:278", "threshold": 0.5, "default_left": True,
         "values": [0.3, 0.7, NAN, 0.5], "expect": [1.0, 2.0, 1.0, 2.0]},
        # default right variant
        {"src": "inference/gbdt/traversal.rs:243", "threshold": 0.5, "default_left": False,
         "values": [NAN], "expect": [2.0]},
    ],
    "grower": [
        # training/gbdt/grower.rs:905-934 test_grower_simple_split: depth 1 -> 2 leaves
        {"src": "training/gbdt/grower.rs:905", "values": [0, 0, 0, 1, 1, 2, 2, 3, 3, 3],
         "grad": [1, 1, 1, 1, 1, -1, -1, -1, -1, -1], "hess": [1] * 10, "max_depth": 1, "expect_leaves": 2},
        # grower.rs:878-903 test_grower_single_leaf: depth 0 -> 1 leaf
        {"src": "training/gbdt/grower.rs:878", "values": [0, 0, 0, 1, 1, 2, 2, 3, 3, 3],
         "grad": [1] * 10, "hess": [1] * 10, "max_depth": 0, "expect_leaves": 1},
    ],
}

if __name__ == "__main__":
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "kats.json")
    with open(out, "w") as f:
        json.dump(KATS, f, indent=1)
    print(out)
