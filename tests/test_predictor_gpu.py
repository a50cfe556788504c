"""Learned configuration predictor on the GPU: the training kernels' gradients
against the float64 oracle, the inference kernel against the oracle's argmin,
and the trained network's regret against exhaustive autotuning, a fixed
default configuration and the library's heuristic (the method without the
predictor)."""
import os

import numpy as np
import pytest

import hiperml_b200 as hml
import oracle.mlp as mlp
from hiperml_b200 import predictor as pr
from hiperml_b200 import tuning_data as td

pytestmark = pytest.mark.gpu

C_SPACE = len(hml.configs())


def _he(C, seed):
    rng = np.random.default_rng(seed)
    parts = [rng.uniform(-1, 1, 64 * 5) * np.sqrt(6 / 5), np.zeros(64),
             rng.uniform(-1, 1, 64 * 64) * np.sqrt(6 / 64), rng.uniform(-0.1, 0.1, 64),
             rng.uniform(-1, 1, C * 64) * np.sqrt(6 / 64), rng.uniform(-0.5, 0.5, C)]
    return np.concatenate(parts).astype(np.float32)


def test_training_kernels_gradient_matches_oracle(cuda):
    C, n = C_SPACE, 48
    rng = np.random.default_rng(3)
    P = _he(C, 4)
    X = rng.uniform(0, 1, (n, 5)).astype(np.float32)
    Y = rng.uniform(0, 2, (n, C)).astype(np.float32)
    W = (rng.uniform(0, 1, (n, C)) < 0.8).astype(np.float32)
    L, g = pr.loss_grad(P, C, X, Y, W)
    Lr, gr = mlp.loss_grad(P.astype(np.float64), C, X, Y, W)
    assert abs(L - Lr) <= 1e-5 * Lr, (L, Lr)
    # per parameter block: FP32 sums of at most n * 64 products vs float64
    o = 0
    for name, size in (("W1", 64 * 5), ("b1", 64), ("W2", 64 * 64), ("b2", 64),
                       ("W3", C * 64), ("b3", C)):
        a, b = g[o:o + size].astype(np.float64), gr[o:o + size]
        scale = max(np.max(np.abs(b)), 1e-12)
        assert np.max(np.abs(a - b)) <= 2e-5 * scale, (name, np.max(np.abs(a - b)), scale)
        o += size


def _allow(shapes, cfgs, algos=pr.FP32_ALGOS):
    r4 = lambda x: (max(1, x) + 3) // 4 * 4
    out = np.zeros((len(shapes), len(cfgs)), bool)
    for i, (M, N, K, ta, tb) in enumerate(shapes):
        lda = r4(K if ta else M)
        ldb = r4(N if tb else K)
        ldc = r4(M)
        for j, c in enumerate(cfgs):
            out[i, j] = c.algo in algos and hml.config_check(0, ta, tb, M, N, K, lda, ldb, ldc,
                                                             c) == 0
    return out


def test_inference_kernel_matches_oracle(cuda, tmp_path):
    cfgs = hml.configs()
    C = len(cfgs)
    P = _he(C, 9)
    path = tmp_path / "m.txt"
    with open(path, "w") as f:
        f.write("#HML-B200 predictor v1\ninputs 5 hidden 64 64 outputs %d\n" % C)
        for c in cfgs:
            f.write("config " + " ".join(str(x) for x in c.as_tuple()) + "\n")
        f.write("params %d\n" % len(P) + " ".join(f"{x:.9g}" for x in P) + "\n")
    pr.load(path)
    try:
        shapes = td.sample_shapes(64, 11)
        got = pr.predict_batch(shapes)
        X = np.stack([pr.features(0, int(ta), int(tb), int(M), int(N), int(K))
                      for (M, N, K, ta, tb) in shapes])
        allow = _allow(shapes, cfgs)
        idx, s = mlp.predict(P.astype(np.float64), C, X, allow)
        for i in range(len(shapes)):
            assert got[i] >= 0 and allow[i, got[i]], (i, got[i])
            # the same choice, or a tie within FP32 rounding of the scores
            assert got[i] == idx[i] or abs(s[i, got[i]] - s[i, idx[i]]) <= 1e-5 * (
                1 + abs(s[i, idx[i]])), (i, got[i], idx[i])
    finally:
        pr.clear()


def _dataset():
    if not os.path.exists(pr.DATASET):
        pytest.skip("no measured dataset in the package")
    return td.load(pr.DATASET)


def test_predictor_regret_beats_fixed_default_and_heuristic(cuda):
    """Train on the first 4000 measured shapes, test on the last 1000: mean
    regret at most 10 %, below the best fixed configuration's and below the
    heuristic's (what hml_sgemm_ex picks without a predictor)."""
    d = _dataset()
    shapes, times, cfgs = d["shapes"], d["times_us"], d["configs"]
    n_tr = min(4000, int(0.8 * len(shapes)))
    tr, te = slice(0, n_tr), slice(n_tr, None)
    hml.tune_clear()
    hist = pr.train(shapes[tr], times[tr], cfgs)
    assert hist[-1] < 0.5 * hist[0], hist[[0, -1]]
    pred = pr.predict_batch(shapes[te])
    r_pred = pr.summarize(pr.regret(times[te], pred, cfgs))
    fixed = pr.best_fixed_config(times[tr], cfgs)
    r_fixed = pr.summarize(pr.regret(times[te], np.full(len(pred), fixed), cfgs))
    pr.clear()
    heur = pr.heuristic_choices(shapes[te], cfgs)
    r_heur = pr.summarize(pr.regret(times[te], heur, cfgs))
    print("predictor", r_pred, "fixed", r_fixed, "heuristic", r_heur)
    assert r_pred["covered"] == r_pred["n"]
    assert r_pred["mean"] <= 0.10, r_pred
    assert r_pred["mean"] < r_fixed["mean"], (r_pred, r_fixed)
    assert r_pred["mean"] < r_heur["mean"], (r_pred, r_heur)


def test_training_is_deterministic(cuda):
    d = _dataset()
    sub = slice(0, 300)
    pr.train(d["shapes"][sub], d["times_us"][sub], d["configs"], epochs=5)
    a = pr.params()
    pr.train(d["shapes"][sub], d["times_us"][sub], d["configs"], epochs=5)
    b = pr.params()
    pr.clear()
    np.testing.assert_array_equal(a, b)


def test_selection_consults_predictor(cuda):
    d = _dataset()
    pr.train(d["shapes"][:1000], d["times_us"][:1000], d["configs"], epochs=50)
    try:
        hml.tune_clear()
        for (M, N, K, ta, tb) in td.sample_shapes(16, 21):
            if M % 4 or K % 4 or N % 4:
                continue  # dense leading dimensions equal the autotuner's rounded ones
            want = pr.predict_batch(np.array([[M, N, K, ta, tb]]))[0]
            got = hml.select(0, int(ta), int(tb), int(M), int(N), int(K))
            assert got.as_tuple() == tuple(int(x) for x in d["configs"][want])
    finally:
        pr.clear()


def test_live_regret_on_unseen_shapes(cuda):
    """Fresh shapes, measured now by exhaustive autotuning over the FP32
    families; the predictor's pick is looked up in that measurement.  The
    10 % target is asserted on the 1000 held-out shapes above; on 16 live
    shapes (a sample whose mean moves with the one or two shapes in the
    held-out set's 10 % tail above 14 %, and with timing noise on kernels of
    a few microseconds) the mean must stay within 15 %."""
    d = _dataset()
    pr.train(d["shapes"], d["times_us"], d["configs"])
    try:
        shapes = td.sample_shapes(16, 99)
        pred = pr.predict_batch(shapes)
        cfgs = [tuple(int(x) for x in c) for c in d["configs"]]
        rs = []
        for (M, N, K, ta, tb), j in zip(shapes, pred):
            ents = hml.autotune(0, int(ta), int(tb), int(M), int(N), int(K),
                                families=(1 << hml.ALGO_SIMT) | (1 << hml.ALGO_BF16X6), reps=5)
            t = {c.as_tuple(): us for c, us, st in ents if st == 0 and us > 0}
            rs.append(t[cfgs[j]] / min(t.values()) - 1.0)
        hml.tune_clear()
        print("live regret", rs)
        assert np.mean(rs) <= 0.15, rs
    finally:
        pr.clear()


def _select_in_subprocess(env_value, shape):
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    M, N, K, ta, tb = (int(x) for x in shape)
    code = ("import hiperml_b200 as h; "
            f"c = h.select(0, {ta}, {tb}, {M}, {N}, {K}); "
            "print(' '.join(map(str, c.as_tuple())), h.lib.hml_predictor_outputs())")
    env = dict(os.environ)
    env.pop("HML_PREDICTOR", None)
    if env_value is not None:
        env["HML_PREDICTOR"] = env_value
    out = subprocess.run([sys.executable, "-c", code], env=env, cwd=root, capture_output=True,
                         text=True, timeout=300, check=True).stdout.split()
    return tuple(int(x) for x in out[:6]), int(out[6])


def test_library_loads_network_named_by_environment(cuda, tmp_path):
    d = _dataset()
    pr.train(d["shapes"][:500], d["times_us"][:500], d["configs"], epochs=30)
    path = tmp_path / "net.txt"
    pr.save(path)
    shape = (8192, 48, 1024, 0, 0)
    want = tuple(int(x) for x in d["configs"][pr.predict_batch(np.array([shape]))[0]])
    pr.clear()
    got, outputs = _select_in_subprocess(str(path), shape)
    assert got == want and outputs == len(d["configs"])
    _, outputs = _select_in_subprocess("none", shape)
    assert outputs == 0


def test_shipped_network_loads_by_default(cuda):
    if not os.path.exists(pr.MODEL):
        pytest.skip("no shipped network")
    _, outputs = _select_in_subprocess(None, (8192, 48, 1024, 0, 0))
    assert outputs == len(hml.configs())
