"""Learned configuration predictor: host-side parts (CPU).

The network oracle (oracle/mlp.py, float64) is pinned by central finite
differences; features, the model file format and the regret arithmetic are
checked without a GPU."""
import numpy as np
import pytest

import hiperml_b200 as hml
import oracle.mlp as mlp
from hiperml_b200 import predictor as pr
from hiperml_b200._lib import lib


def _random_net(C, seed, scale=0.5):
    rng = np.random.default_rng(seed)
    return rng.uniform(-scale, scale, pr.n_params(C))


def test_oracle_gradient_matches_finite_differences():
    C, n = 7, 9
    rng = np.random.default_rng(1)
    P = _random_net(C, 2)
    X = rng.uniform(0, 1, (n, 5))
    Y = rng.uniform(0, 2, (n, C))
    W = (rng.uniform(0, 1, (n, C)) < 0.8).astype(float)
    L, g = mlp.loss_grad(P, C, X, Y, W)
    assert abs(L - mlp.loss(P, C, X, Y, W)) < 1e-14
    h = 1e-6
    num = np.empty_like(P)
    for i in range(len(P)):
        e = np.zeros_like(P)
        e[i] = h
        num[i] = (mlp.loss(P + e, C, X, Y, W) - mlp.loss(P - e, C, X, Y, W)) / (2 * h)
    assert np.max(np.abs(num - g)) <= 1e-7 * max(1.0, np.max(np.abs(g))), np.max(np.abs(num - g))


@pytest.mark.parametrize("order,ta,tb,M,N,K", [
    (0, 0, 0, 4096, 16, 4096), (0, 1, 0, 300, 7, 50), (0, 0, 1, 65536, 256, 16384),
    (0, 1, 1, 20, 90, 33), (1, 0, 0, 500, 60, 17), (1, 1, 1, 64, 640, 2048)])
def test_features_follow_canonical_problem(order, ta, tb, M, N, K):
    f = pr.features(order, ta, tb, M, N, K)
    # storage strides -> canonical K-contiguity (column-major: A N-op has
    # unit stride along m; row-major: along k); the long dimension becomes M
    cm = order == 0
    akc = (ta == 1) if cm else (ta == 0)
    bkc = (tb == 0) if cm else (tb == 1)
    if N > M:
        M, N, akc, bkc = N, M, bkc, akc
    np.testing.assert_allclose(f, mlp.features(M, N, K, akc, bkc), rtol=1e-6, atol=1e-7)


def _write_model(path, cfgs, P, header="#HML-B200 predictor v1", hidden=(64, 64)):
    with open(path, "w") as f:
        f.write(header + "\n")
        f.write(f"inputs 5 hidden {hidden[0]} {hidden[1]} outputs {len(cfgs)}\n")
        for c in cfgs:
            f.write("config " + " ".join(str(x) for x in c.as_tuple()) + "\n")
        f.write(f"params {len(P)}\n")
        f.write(" ".join(f"{x:.9g}" for x in P) + "\n")


def test_model_file_round_trip(tmp_path):
    cfgs = hml.configs()[:3]
    P = _random_net(3, 4).astype(np.float32)
    _write_model(tmp_path / "m.txt", cfgs, P)
    pr.load(tmp_path / "m.txt")
    try:
        assert pr.outputs() == 3
        np.testing.assert_array_equal(pr.params(), P)
        pr.save(tmp_path / "n.txt")
        pr.clear()
        assert pr.outputs() == 0
        pr.load(tmp_path / "n.txt")
        np.testing.assert_array_equal(pr.params(), P)
    finally:
        pr.clear()


@pytest.mark.parametrize("bad", ["header", "hidden", "config", "count", "nan"])
def test_model_file_rejected(tmp_path, bad):
    cfgs = hml.configs()[:3]
    P = _random_net(3, 5).astype(np.float32)
    kw = {}
    if bad == "header":
        kw["header"] = "#HML-B200 predictor v9"
    elif bad == "hidden":
        kw["hidden"] = (32, 64)
    elif bad == "config":
        cfgs = list(cfgs)
        cfgs[1] = hml.SgemmConfig(1, 128, 16, 3, 4, 0)  # split 3 is not in the space
    elif bad == "count":
        P = P[:-1]
    else:
        P = P.copy()
        P[7] = np.nan
    _write_model(tmp_path / "bad.txt", cfgs, P, **kw)
    assert lib.hml_predictor_load(str(tmp_path / "bad.txt").encode()) == 5  # CONFIG_ERROR
    assert pr.outputs() == 0


def test_targets_and_regret_arithmetic():
    t = np.array([[10.0, 20.0, -1.0, 40.0], [5.0, -1.0, 4.0, 100.0]])
    y, w = pr.targets_from_times(t, clip=1.0)
    np.testing.assert_allclose(y[0], [0, np.log(2), 0, 1.0], rtol=1e-6)
    np.testing.assert_allclose(w, [[1, 1, 0, 1], [1, 0, 1, 1]])
    cfgs = np.array([[1, 128, 16, 1, 4, 0], [1, 128, 8, 1, 4, 1], [2, 128, 16, 1, 4, 0],
                     [3, 128, 16, 1, 4, 0]])
    # BF16X3 (algo 2) is outside the FP32 families: best of row 1 is 5.0
    r = pr.regret(t, np.array([1, 3]), cfgs)
    np.testing.assert_allclose(r, [1.0, 19.0])
    assert np.isnan(pr.regret(t, np.array([2, 0]), cfgs)[0])
    assert pr.best_fixed_config(t, cfgs) == 0
