"""scikit-learn estimators over the GPU engine, with the parameter names and
behaviour of boosters' wrappers (packages/boosters-python/python/boosters/
sklearn/gbdt.py): ``GBDTRegressor`` and ``GBDTClassifier``.

The configuration is built from the constructor's parameters at ``fit``
time, so ``set_params`` and ``sklearn.base.clone`` work as for any
estimator. The classifier encodes labels to 0..K-1 (``classes_``), trains a
logistic model for two classes and a softmax model for more unless an
objective is given, and returns ``predict_proba`` as ``(n, n_classes)``.
``eval_set=(X_val, y_val)`` feeds early stopping. ``precision`` and
``batched`` select the engine's training form (extensions; the defaults are
the exact FP32 batched form).
"""
import numpy as np
from sklearn.base import BaseEstimator, ClassifierMixin, RegressorMixin
from sklearn.utils.validation import check_array, check_is_fitted, check_X_y

from . import Dataset, GBDTConfig, GBDTModel, GrowthStrategy, ImportanceType, Metric, Objective

__all__ = ["GBDTRegressor", "GBDTClassifier"]


class _GBDTBase(BaseEstimator):
    # objective kinds each estimator accepts (gbdt.py: _validate_objective)
    _objective_kinds = ()
    _name = ""

    def __init__(self, n_estimators=100, learning_rate=0.1, max_depth=6, min_child_weight=1.0, max_leaves=31,
                 grow_strategy=GrowthStrategy.Depthwise, colsample_bytree=1.0, subsample=1.0, gamma=0.0,
                 reg_alpha=0.0, reg_lambda=1.0, early_stopping_rounds=None, seed=42, n_threads=0, verbose=1,
                 objective=None, metric=None, precision="fp32", batched=True):
        self.n_estimators = n_estimators
        self.learning_rate = learning_rate
        self.max_depth = max_depth
        self.min_child_weight = min_child_weight
        self.max_leaves = max_leaves
        self.grow_strategy = grow_strategy
        self.colsample_bytree = colsample_bytree
        self.subsample = subsample
        self.gamma = gamma
        self.reg_alpha = reg_alpha
        self.reg_lambda = reg_lambda
        self.early_stopping_rounds = early_stopping_rounds
        self.seed = seed
        self.n_threads = n_threads
        self.verbose = verbose
        self.objective = objective
        self.metric = metric
        self.precision = precision
        self.batched = batched

    # ---- hooks of the two estimators ------------------------------------------
    def _default_objective(self):
        raise NotImplementedError

    def _default_metric(self):
        raise NotImplementedError

    def _encode_targets(self, y, fitting):
        raise NotImplementedError

    # ---- shared ----------------------------------------------------------------
    def _check_objective(self, obj):
        if not isinstance(obj, self._objective_kinds):
            raise ValueError(f"{self._name} cannot train {obj!r}; use "
                             + " or ".join(k.__qualname__ for k in self._objective_kinds))

    def _config(self, objective):
        self._check_objective(objective)
        return GBDTConfig(
            n_estimators=self.n_estimators, learning_rate=self.learning_rate, max_depth=self.max_depth,
            min_child_weight=self.min_child_weight, n_leaves=self.max_leaves, growth_strategy=self.grow_strategy,
            colsample_bytree=self.colsample_bytree, subsample=self.subsample, min_gain_to_split=self.gamma,
            l1=self.reg_alpha, l2=self.reg_lambda, early_stopping_rounds=self.early_stopping_rounds, seed=self.seed,
            verbosity=self.verbose, objective=objective,
            metric=self.metric if self.metric is not None else self._default_metric(),
            precision=self.precision, batched=self.batched)

    def fit(self, X, y, eval_set=None, sample_weight=None):
        X, y = check_X_y(X, y, dtype=np.float32)
        self.n_features_in_ = X.shape[1]
        labels = self._encode_targets(y, fitting=True)
        objective = self.objective if self.objective is not None else self._default_objective()
        train = Dataset(X, labels, weights=sample_weight)
        val = None
        if eval_set is not None:
            Xv, yv = eval_set
            val = Dataset(check_array(Xv, dtype=np.float32), self._encode_targets(np.asarray(yv), fitting=False))
        self.model_ = GBDTModel.train(train, self._config(objective), val_set=val, n_threads=self.n_threads)
        return self

    def _outputs(self, X):
        check_is_fitted(self, ["model_"])
        X = check_array(X, dtype=np.float32)
        if X.shape[1] != self.n_features_in_:
            raise ValueError(f"X has {X.shape[1]} features, the estimator was fitted with {self.n_features_in_}")
        return self.model_.predict(Dataset(X))  # (n, n_outputs), transformed

    @property
    def feature_importances_(self):
        check_is_fitted(self, ["model_"])
        return self.model_.feature_importance(ImportanceType.Gain)

    def get_feature_importance(self, importance_type=ImportanceType.Gain):
        check_is_fitted(self, ["model_"])
        return self.model_.feature_importance(importance_type)


class GBDTRegressor(RegressorMixin, _GBDTBase):
    """Gradient-boosted trees for regression (squared loss by default,
    RMSE as the early-stopping metric)."""

    _objective_kinds = (Objective.Squared,)
    _name = "GBDTRegressor"

    def _default_objective(self):
        return Objective.squared()

    def _default_metric(self):
        return Metric.rmse()

    def _encode_targets(self, y, fitting):
        return np.asarray(y, dtype=np.float32)

    def predict(self, X):
        return self._outputs(X)[:, 0]


class GBDTClassifier(ClassifierMixin, _GBDTBase):
    """Gradient-boosted trees for classification: logistic for two classes,
    softmax for more. The early-stopping metric defaults to log loss as in
    the reference; that metric reads the first output only, so multiclass
    early stopping should pass ``metric=Metric.MultiLogLoss()``."""

    _objective_kinds = (Objective.Logistic, Objective.Softmax)
    _name = "GBDTClassifier"

    def _default_objective(self):
        return Objective.logistic() if self.n_classes_ <= 2 else Objective.softmax(self.n_classes_)

    def _default_metric(self):
        return Metric.logloss()

    def _encode_targets(self, y, fitting):
        if fitting:
            self.classes_, codes = np.unique(y, return_inverse=True)
            self.n_classes_ = len(self.classes_)
            return codes.astype(np.float32)
        pos = np.searchsorted(self.classes_, y)
        pos = np.clip(pos, 0, len(self.classes_) - 1)
        if not np.all(self.classes_[pos] == y):
            raise ValueError("eval_set has labels that the training labels do not have")
        return pos.astype(np.float32)

    def predict_proba(self, X):
        p = self._outputs(X)
        if p.shape[1] == 1:  # logistic: P(class 1)
            return np.column_stack([1.0 - p[:, 0], p[:, 0]]).astype(np.float32)
        return p

    def predict(self, X):
        proba = self.predict_proba(X)
        if self.n_classes_ == 2:
            idx = (proba[:, 1] >= 0.5).astype(np.intp)
        else:
            idx = np.argmax(proba, axis=1)
        return self.classes_[idx]
