"""Autotuner of the mixed form's GEMM launches: exhaustive table and a
learned cost model.

Every batched GEMM launch of the mixed form (factor updates, pivot-block
inversion, solve products) can run as tcgen05 3xTF32 with 128 x 128 tiles or
as CUDA-core FP32 with 64 x 64 tiles; both compute the same update.  The
built-in rule takes tcgen05 everywhere (solves: from 64 right-hand sides).

* The exhaustive table times every launch in both variants (two profiled
  factor + solve passes) and picks the faster per launch.  It is the
  fallback when the model is not trusted and the judge of its mispredictions.
* The cost model is a small MLP (csrc/costmodel.cu) trained on the GPU by
  libmfgpu's own kernels on tables recorded from other matrices: from a
  launch's features and a variant it predicts log10 of the launch time, and
  the autotuner picks the variant with the lower prediction.

The model never touches the arithmetic: it only selects among variants.
"""

from __future__ import annotations

import ctypes
from dataclasses import dataclass

import numpy as np

from . import _lib as L
from .api import GpuContext

NFEAT = 11          # mfgpu_tune_features per launch
VARIANTS = (1, 2)   # 1: tcgen05 3xTF32, 2: CUDA-core FP32
NIN = NFEAT + 2     # features + variant one-hot


class CostModel:
    """libmfgpu's MLP (nin -> hidden -> hidden -> 1), on the GPU."""

    def __init__(self, nin: int = NIN, hidden: int = 32, seed: int = 0, device: int = 0):
        self._lib = L.lib()
        h = ctypes.c_void_p()
        rc = self._lib.mfgpu_mlp_create(device, nin, hidden, seed, ctypes.byref(h))
        if rc != 0:
            raise RuntimeError(f"mfgpu_mlp_create -> {rc}")
        self._h, self.nin, self.hidden = h, nin, hidden

    def _check(self, rc):
        if rc != 0:
            raise RuntimeError(self._lib.mfgpu_mlp_last_error(self._h).decode())

    @property
    def nparams(self) -> int:
        return int(self._lib.mfgpu_mlp_nparams(self._h))

    def get_params(self) -> np.ndarray:
        p = np.empty(self.nparams, np.float32)
        self._check(self._lib.mfgpu_mlp_get_params(self._h, L.ptr(p, L.f32p)))
        return p

    def set_params(self, p):
        p = np.ascontiguousarray(p, dtype=np.float32)
        self._check(self._lib.mfgpu_mlp_set_params(self._h, L.ptr(p, L.f32p)))

    def predict(self, X) -> np.ndarray:
        X = np.ascontiguousarray(X, dtype=np.float32)
        out = np.empty(len(X), np.float32)
        self._check(self._lib.mfgpu_mlp_predict(self._h, L.ptr(X, L.f32p), len(X), L.ptr(out, L.f32p)))
        return out

    def loss_grad(self, X, Y):
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        loss = ctypes.c_float()
        g = np.empty(self.nparams, np.float32)
        self._check(self._lib.mfgpu_mlp_loss_grad(self._h, L.ptr(X, L.f32p), L.ptr(Y, L.f32p), len(Y),
                                                  ctypes.byref(loss), L.ptr(g, L.f32p)))
        return float(loss.value), g

    def train(self, X, Y, iters: int = 2000, lr: float = 3e-3) -> float:
        X = np.ascontiguousarray(X, dtype=np.float32)
        Y = np.ascontiguousarray(Y, dtype=np.float32)
        loss = ctypes.c_float()
        self._check(self._lib.mfgpu_mlp_train(self._h, L.ptr(X, L.f32p), L.ptr(Y, L.f32p), len(Y), int(iters),
                                              float(lr), ctypes.byref(loss)))
        return float(loss.value)

    def __del__(self):
        if getattr(self, "_h", None):
            try:
                self._lib.mfgpu_mlp_destroy(self._h)
            except Exception:
                pass
            self._h = None


@dataclass
class LaunchTable:
    """Per tunable launch: features and device ms in each variant."""
    feats: np.ndarray      # (count, NFEAT)
    times: np.ndarray      # (count, 2): ms with tcgen05, with CUDA cores
    rule: np.ndarray       # (count,): the built-in rule's variant (1 or 2)

    @property
    def best(self) -> np.ndarray:
        return 1 + np.argmin(self.times, axis=1)

    def cost(self, choice) -> float:
        choice = np.asarray(choice)
        return float(self.times[np.arange(len(choice)), choice - 1].sum())


def tune_features(ctx: GpuContext, nrhs: int) -> np.ndarray:
    lib = ctx._lib
    n = ctypes.c_int64()
    ctx._check(lib.mfgpu_tune_features(ctx._h, nrhs, ctypes.byref(n), None, 0))
    f = np.empty((n.value, NFEAT), np.float32)
    ctx._check(lib.mfgpu_tune_features(ctx._h, nrhs, ctypes.byref(n), L.ptr(f, L.f32p), f.size))
    return f


def set_choice(ctx: GpuContext, choice):
    c = np.ascontiguousarray(choice, dtype=np.int8)
    ctx._check(ctx._lib.mfgpu_tune_set_choice(ctx._h, c.ctypes.data_as(ctypes.POINTER(ctypes.c_int8)), len(c)))


def measure(ctx: GpuContext, run, count: int, choice, repeats: int = 2) -> np.ndarray:
    """Device ms of every tunable launch under `choice` (min over repeats of a
    profiled run(); `run` issues one factor + one solve pass)."""
    set_choice(ctx, choice)
    best = np.full(count, np.inf)
    for _ in range(repeats):
        ctx.set_profiling(True)
        run()
        t = np.zeros(count)
        for r in ctx.launch_records():
            if len(r) > 6 and r[6] >= 0:
                t[r[6]] += r[3]
        ctx.set_profiling(False)
        best = np.minimum(best, t)
    return best


def rule_choice(feats: np.ndarray, nrhs: int) -> np.ndarray:
    """The library's built-in rule (mfgpu.cu: tc_worthwhile): tcgen05 when a
    launch's mean work per 128 x 128 tile is at least a full tile's over
    K = 64, CUDA cores otherwise; solve products on tcgen05 only from 64
    right-hand sides."""
    flops = np.power(10.0, feats[:, 3].astype(np.float64)) - 1.0
    tiles_tc = np.power(10.0, feats[:, 7].astype(np.float64)) - 1.0
    big = (tiles_tc > 0.5) & (flops >= 2.0 * 128 * 128 * 64 * tiles_tc * (1 - 1e-6))
    return np.where(big & ((feats[:, 2] == 0) | (nrhs >= 64)), 1, 2)


def exhaustive_table(ctx: GpuContext, run, nrhs: int, repeats: int = 2) -> LaunchTable:
    feats = tune_features(ctx, nrhs)
    count = len(feats)
    times = np.stack([measure(ctx, run, count, np.full(count, v), repeats) for v in VARIANTS], axis=1)
    set_choice(ctx, [])
    return LaunchTable(feats, times, rule_choice(feats, nrhs))


def _design(feats: np.ndarray):
    """Model inputs: every launch twice, once per variant (one-hot)."""
    n = len(feats)
    X = np.concatenate([np.repeat(feats, 2, axis=0), np.tile(np.eye(2, dtype=np.float32), (n, 1))], axis=1)
    return X


@dataclass
class Tuner:
    model: CostModel
    mu: np.ndarray
    sd: np.ndarray
    ymu: float
    ysd: float
    loss: float

    def predict_ms(self, feats: np.ndarray) -> np.ndarray:
        X = (_design(feats) - self.mu) / self.sd
        y = self.model.predict(X) * self.ysd + self.ymu
        return (10.0 ** y).reshape(-1, 2)

    def choose(self, feats: np.ndarray, rule=None, margin: float = 0.1) -> np.ndarray:
        """Variant per launch: the model's faster variant, but with a rule
        given, only where the model predicts at least `margin` of gain over
        the rule's variant (mispredictions near the crossover cost little)."""
        t = self.predict_ms(feats)
        best = 1 + np.argmin(t, axis=1)
        if rule is None:
            return best
        rule = np.asarray(rule)
        idx = np.arange(len(rule))
        gain = 1.0 - t[idx, best - 1] / t[idx, rule - 1]
        return np.where(gain >= margin, best, rule)


def train(tables, hidden: int = 32, iters: int = 3000, lr: float = 3e-3, seed: int = 0, device: int = 0) -> Tuner:
    """Fit the cost model to recorded tables: log10 ms of each (launch, variant)."""
    X = np.concatenate([_design(t.feats) for t in tables]).astype(np.float64)
    y = np.concatenate([np.log10(np.maximum(t.times, 1e-4)).ravel() for t in tables])
    mu, sd = X.mean(0), X.std(0)
    sd[sd == 0] = 1.0
    ymu, ysd = float(y.mean()), float(y.std() or 1.0)
    model = CostModel(NIN, hidden, seed, device)
    loss = model.train(((X - mu) / sd).astype(np.float32), ((y - ymu) / ysd).astype(np.float32), iters, lr)
    return Tuner(model, mu.astype(np.float32), sd.astype(np.float32), ymu, ysd, loss)


def judge(tuner: Tuner, table: LaunchTable) -> dict:
    """The model's schedule against the exhaustive table (best per launch) and
    the built-in rule, all costed with the table's measured times."""
    choice = tuner.choose(table.feats, table.rule)
    return {"launches": int(len(choice)), "mispredicted": int(np.sum(choice != table.best)),
            "model_ms": table.cost(choice), "table_ms": table.cost(table.best), "rule_ms": table.cost(table.rule),
            "choice": choice}
