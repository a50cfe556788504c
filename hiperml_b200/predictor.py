"""The learned configuration predictor (Python side of hml_predictor_*).

Training and inference run in the library's own GPU kernels
(hiperml_b200/csrc/predictor.cu); this module moves the measured data in and
out and scores a trained network the way it is used: by the regret of the
configuration it picks, t(predicted) / t(best measured) - 1.

Command line (GPU):
    python -m hiperml_b200.predictor DATA.npz OUT.txt [--train 4000]
trains on the first --train shapes of a tuning_data file, reports regret on
the rest, and saves the network.
"""
from __future__ import annotations

import argparse
import ctypes
import json
import os

import numpy as np

from . import api
from ._lib import PredictorOptions, SgemmConfig, check, lib

HERE = os.path.dirname(os.path.abspath(__file__))
DATASET = os.path.join(HERE, "data", "tune_b200.npz")
MODEL = os.path.join(HERE, "data", "predictor_b200.txt")

N_IN, N_HID = 5, 64
# FP32-accurate families: the regret is measured among these (BF16X3 is the
# fast math mode's extra choice)
FP32_ALGOS = (api.ALGO_SIMT, api.ALGO_BF16X6)

DEFAULTS = dict(epochs=400, batch=256, lr=3e-3, weight_decay=1e-4, target_clip=2.0, seed=7)


def n_params(C: int) -> int:
    return N_HID * N_IN + N_HID + N_HID * N_HID + N_HID + C * N_HID + C


def _i32(a):
    return np.ascontiguousarray(np.asarray(a), dtype=np.int32)


def _f32(a):
    return np.ascontiguousarray(np.asarray(a), dtype=np.float32)


def _ptr(a):
    return a.ctypes.data_as(ctypes.c_void_p)


def features(order, ta, tb, M, N, K) -> np.ndarray:
    f = np.zeros(N_IN, np.float32)
    check(lib.hml_predictor_features(order, ta, tb, M, N, K, _ptr(f)), "hml_predictor_features")
    return f


def configs_array(configs) -> ctypes.Array:
    arr = (SgemmConfig * len(configs))()
    for i, c in enumerate(configs):
        arr[i] = SgemmConfig(*[int(x) for x in c])
    return arr


def train(shapes, times_us, configs, order=api.COL_MAJOR, **opts) -> np.ndarray:
    """Trains the library's predictor on the GPU; returns the loss per epoch."""
    o = dict(DEFAULTS, **opts)
    sh = _i32(shapes)
    t = _f32(np.nan_to_num(times_us, nan=-1.0))
    cfg = configs_array(configs)
    hist = np.zeros(o["epochs"], np.float32)
    po = PredictorOptions(o["epochs"], o["batch"], o["lr"], o["weight_decay"], o["target_clip"],
                          o["seed"])
    check(lib.hml_predictor_train(order, _ptr(sh), _ptr(t), len(sh), cfg, len(configs),
                                  ctypes.byref(po), _ptr(hist)), "hml_predictor_train")
    return hist


def predict_batch(shapes, order=api.COL_MAJOR) -> np.ndarray:
    sh = _i32(shapes)
    out = np.zeros(len(sh), np.int32)
    check(lib.hml_predictor_predict_batch(order, _ptr(sh), len(sh), _ptr(out)),
          "hml_predictor_predict_batch")
    return out


def loss_grad(params, C, feats, targets, weights):
    p, f, t, w = _f32(params), _f32(feats), _f32(targets), _f32(weights)
    g = np.zeros_like(p)
    loss = np.zeros(1, np.float32)
    check(lib.hml_predictor_loss_grad(_ptr(p), C, _ptr(f), _ptr(t), _ptr(w), len(f), _ptr(g),
                                      _ptr(loss)), "hml_predictor_loss_grad")
    return float(loss[0]), g


def params() -> np.ndarray:
    n = ctypes.c_size_t()
    check(lib.hml_predictor_params(None, 0, ctypes.byref(n)), "hml_predictor_params")
    out = np.zeros(n.value, np.float32)
    check(lib.hml_predictor_params(_ptr(out), n.value, None), "hml_predictor_params")
    return out


def save(path):
    check(lib.hml_predictor_save(str(path).encode()), "hml_predictor_save")


def load(path):
    check(lib.hml_predictor_load(str(path).encode()), "hml_predictor_load")


def clear():
    check(lib.hml_predictor_clear(), "hml_predictor_clear")


def outputs() -> int:
    return lib.hml_predictor_outputs()


# ------------------------------------------------------------ evaluation
def targets_from_times(times_us, clip=DEFAULTS["target_clip"]):
    """(targets, weights) as the training kernels see them:
    y = min(log(t / t_best), clip) on measured entries, weight 1 there."""
    t = np.nan_to_num(np.asarray(times_us, np.float64), nan=-1.0)
    valid = t > 0
    best = np.where(valid, t, np.inf).min(axis=1, keepdims=True)
    y = np.where(valid, np.minimum(np.log(np.where(valid, t, 1.0) / best), clip), 0.0)
    return y.astype(np.float32), valid.astype(np.float32)


def allowed_mask(configs, algos=FP32_ALGOS):
    return np.isin(np.asarray(configs)[:, 0], algos)


def regret(times_us, chosen, configs, algos=FP32_ALGOS):
    """Per-shape regret t(chosen) / t(best allowed measured) - 1 (NaN where
    the chosen configuration has no measurement)."""
    t = np.nan_to_num(np.asarray(times_us, np.float64), nan=-1.0)
    ok = (t > 0) & allowed_mask(configs, algos)[None, :]
    best = np.where(ok, t, np.inf).min(axis=1)
    ch = np.asarray(chosen)
    tc = np.where(ch >= 0, t[np.arange(len(t)), np.clip(ch, 0, None)], -1.0)
    return np.where(tc > 0, tc / best - 1.0, np.nan)


def best_fixed_config(times_us, configs, algos=FP32_ALGOS):
    """The single allowed configuration with the lowest mean regret over the
    given shapes (among those measured on every shape)."""
    t = np.nan_to_num(np.asarray(times_us, np.float64), nan=-1.0)
    ok = (t > 0) & allowed_mask(configs, algos)[None, :]
    best = np.where(ok, t, np.inf).min(axis=1, keepdims=True)
    everywhere = ok.all(axis=0)
    r = np.where(ok, t / best - 1.0, np.inf).mean(axis=0)
    r[~everywhere] = np.inf
    return int(np.argmin(r))


def heuristic_choices(shapes, configs, order=api.COL_MAJOR):
    """Index (into `configs`) of what hml_sgemm_select picks with neither a
    tuned table nor a predictor loaded (-1 when outside the space, e.g. the
    GEMV route)."""
    index = {tuple(int(x) for x in c): i for i, c in enumerate(configs)}
    out = []
    for (M, N, K, ta, tb) in np.asarray(shapes):
        c = api.select(order, int(ta), int(tb), int(M), int(N), int(K))
        out.append(index.get(c.as_tuple(), -1))
    return np.asarray(out)


def summarize(r):
    r = np.asarray(r, np.float64)
    v = r[~np.isnan(r)]
    return {"mean": float(v.mean()) if len(v) else None,
            "p50": float(np.percentile(v, 50)) if len(v) else None,
            "p90": float(np.percentile(v, 90)) if len(v) else None,
            "max": float(v.max()) if len(v) else None,
            "covered": int(len(v)), "n": int(len(r))}


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("data")
    ap.add_argument("out")
    ap.add_argument("--train", type=int, default=4000)
    for k, v in DEFAULTS.items():
        ap.add_argument("--" + k.replace("_", "-"), type=type(v), default=v)
    a = ap.parse_args(argv)
    from . import tuning_data
    d = tuning_data.load(a.data)
    shapes, times, cfgs = d["shapes"], d["times_us"], d["configs"]
    tr, te = slice(0, a.train), slice(a.train, None)
    opts = {k: getattr(a, k) for k in DEFAULTS}
    hist = train(shapes[tr], times[tr], cfgs, **opts)
    pred = predict_batch(shapes[te])
    api.tune_clear()
    fixed = best_fixed_config(times[tr], cfgs)
    saved = outputs()
    clear()
    heur = heuristic_choices(shapes[te], cfgs)
    report = {
        "loss_first_last": [float(hist[0]), float(hist[-1])],
        "predictor": summarize(regret(times[te], pred, cfgs)),
        "fixed_default": summarize(regret(times[te], np.full(len(pred), fixed), cfgs)),
        "fixed_default_config": [int(x) for x in cfgs[fixed]],
        "heuristic": summarize(regret(times[te], heur, cfgs)),
    }
    print(json.dumps(report, indent=1))
    # train again (deterministic) to save the same network
    if saved:
        train(shapes[tr], times[tr], cfgs, **opts)
        save(a.out)
    return 0


if __name__ == "__main__":
    raise SystemExit(main())
