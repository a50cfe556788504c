"""The measuring autotuner on a B200 (replaces the reference's online tuner,
src/hml_sgemm_kernel.cu:356-555, which times every repository kernel on the
caller's shape and keeps the fastest)."""
import numpy as np
import pytest

import hiperml_b200 as hml
from hiperml_b200._lib import lib

pytestmark = pytest.mark.gpu


def _median_us(fn, reps=20):
    import torch
    ev = [torch.cuda.Event(enable_timing=True) for _ in range(2 * reps)]
    for i in range(reps):
        ev[2 * i].record()
        fn()
        ev[2 * i + 1].record()
    torch.cuda.synchronize()
    return float(np.median([ev[2 * i].elapsed_time(ev[2 * i + 1]) * 1e3 for i in range(reps)]))


def test_autotune_records_fastest_allowed(cuda, tmp_path):
    hml.tune_clear()
    M, N, K = 8192, 64, 1024
    ents = hml.autotune(0, 0, 0, M, N, K, reps=3)
    assert len(ents) == lib.hml_sgemm_num_configs()
    ok = [(c, t) for c, t, s in ents if s == 0]
    assert len(ok) >= 50
    assert all(t > 0 for _, t in ok)
    # the recorded choice is the fastest FP32-accurate configuration measured
    allowed = [(c, t) for c, t in ok if c.algo in (hml.ALGO_SIMT, hml.ALGO_BF16X6)]
    best = min(allowed, key=lambda e: e[1])[0]
    assert lib.hml_tune_size() == 1
    assert hml.select(0, 0, 0, M, N, K).as_tuple() == best.as_tuple()
    f = tmp_path / "tuned.cfg"
    hml.tune_save(str(f))
    hml.tune_clear()
    assert hml.tune_load(str(f)) == 1
    assert hml.select(0, 0, 0, M, N, K).as_tuple() == best.as_tuple()
    hml.tune_clear()


def test_tuned_choice_not_slower_than_heuristic(cuda):
    """After tuning, hml_sgemm_ex on the shape runs within noise of the best
    configuration and no slower than the untuned heuristic's choice."""
    import torch
    hml.tune_clear()
    M, N, K = 16384, 32, 2048
    A = torch.empty(M * K, device="cuda")
    B = torch.empty(K * N, device="cuda")
    C = torch.zeros(M * N, device="cuda")
    hml.fill_random(A, 5, 0)
    hml.fill_random(B, 5, 1)
    run = lambda: hml.sgemm_ex(0, 0, 0, M, N, K, 1.0, A, M, B, K, 0.0, C, M)
    run()
    t_heur = _median_us(run)
    # the FP32-accurate families: the untuned choice may be either
    ents = hml.autotune(0, 0, 0, M, N, K,
                        families=(1 << hml.ALGO_SIMT) | (1 << hml.ALGO_BF16X6), reps=5)
    t_best = min(t for c, t, s in ents if s == 0)
    run()
    t_tuned = _median_us(run)
    hml.tune_clear()
    assert t_tuned <= t_heur * 1.10 + 2.0, (t_tuned, t_heur)
    assert t_tuned <= t_best * 1.25 + 2.0, (t_tuned, t_best)


def test_autotune_family_mask_and_bad_arguments(cuda):
    hml.tune_clear()
    ents = hml.autotune(1, 1, 0, 3000, 20, 512, families=1 << hml.ALGO_SIMT, reps=2)
    assert ents and all(c.algo == hml.ALGO_SIMT for c, _, _ in ents)
    with pytest.raises(hml.HmlError):
        hml.autotune(0, 0, 0, -1, 20, 512)
    hml.tune_clear()


def _select_child(env_tuned, shape):
    """hml.select in a fresh process (HML_TUNED as given, unset for None)."""
    import os
    import subprocess
    import sys
    root = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
    M, N, K = shape
    code = ("import hiperml_b200 as h; "
            f"c = h.select(0, 0, 0, {M}, {N}, {K}); "
            "print(' '.join(map(str, c.as_tuple())), h.lib.hml_tune_size())")
    env = dict(os.environ)
    env.pop("HML_TUNED", None)
    if env_tuned is not None:
        env["HML_TUNED"] = env_tuned
    out = subprocess.run([sys.executable, "-c", code], env=env, cwd=root, capture_output=True,
                         text=True, timeout=300, check=True).stdout.split()
    return tuple(int(x) for x in out[:6]), int(out[6])


def test_shipped_table_is_the_default_selection(cuda):
    """Without HML_TUNED the first selection loads data/tuned_b200.txt, and a
    reference workload shape gets the table's measured configuration;
    HML_TUNED=none leaves the table out."""
    import os
    path = os.path.join(os.path.dirname(hml.__file__), "data", "tuned_b200.txt")
    if not os.path.exists(path):
        pytest.skip("no shipped table")
    want, n_gemv = {}, 0
    for line in open(path):
        if line.startswith("v "):
            n_gemv += 1  # an SGEMV record
        elif not line.startswith("#"):
            key, cfg = line.split(":")
            akc, bkc, M, N, K = (int(x) for x in key.split())
            want[(akc, bkc, M, N, K)] = tuple(int(x) for x in cfg.split()[:6])
    shape = (65536, 32, 4096)
    got, size = _select_child(None, shape)  # column-major NN: A M-, B K-contiguous
    assert size == len(want) + n_gemv and got == want[(0, 1) + shape]
    _, size = _select_child("none", shape)
    assert size == 0


def test_tail_wave_split(cuda, tmp_path):
    """hml_sgemm_ex with a whole-K tensor-core choice whose grid ends in a
    wave of at most half the SMs: the rows of the whole waves are exactly
    the configuration's, the last wave's rows those of the same tile split in
    K over the idle SMs (here 4 ways), and repeated calls give the same bits."""
    import os

    import torch
    sms = torch.cuda.get_device_properties(0).multi_processor_count
    rest = 20
    M, N, K = (sms + rest) * 128, 32, 2048
    split = 1
    while split < 8 and 2 * split * rest <= sms and K // (2 * split) >= 256:
        split *= 2
    assert split > 1
    cfg = hml.SgemmConfig(hml.ALGO_BF16X6, 128, 32, 1, 6, 1)
    f = tmp_path / "tuned.txt"
    f.write_text("#HML-B200 tuning v2\n# device test sms %d\n"
                 "# akc bkc M N K : algo tile_m tile_n split_k stages variant time_us\n"
                 "0 1 %d %d %d : 3 128 32 1 6 1 1.0\n" % (sms, M, N, K))
    try:
        hml.tune_clear()
        assert hml.tune_load(str(f)) == 1
        assert hml.select(0, 0, 0, M, N, K).as_tuple() == cfg.as_tuple()
        A = torch.empty(M * K, device="cuda")
        B = torch.empty(K * N, device="cuda")
        hml.fill_random(A, 5, 0, 1)
        hml.fill_random(B, 5, 1, 1)
        C = torch.zeros(M * N, device="cuda")
        hml.sgemm_ex(0, 0, 0, M, N, K, 1.0, A, M, B, K, 0.0, C, M)
        C2 = torch.zeros(M * N, device="cuda")
        hml.sgemm_ex(0, 0, 0, M, N, K, 1.0, A, M, B, K, 0.0, C2, M)
        assert torch.equal(C, C2)
        whole = torch.zeros(M * N, device="cuda")
        hml.sgemm_ex(0, 0, 0, M, N, K, 1.0, A, M, B, K, 0.0, whole, M, config=cfg)
        split_cfg = hml.SgemmConfig(hml.ALGO_BF16X6, 128, 32, split, 6, 1)
        splitk = torch.zeros(M * N, device="cuda")
        hml.sgemm_ex(0, 0, 0, M, N, K, 1.0, A, M, B, K, 0.0, splitk, M, config=split_cfg)
        m1 = sms * 128
        got, w, sk = (t.view(N, M) for t in (C, whole, splitk))
        assert torch.equal(got[:, :m1], w[:, :m1])
        assert torch.equal(got[:, m1:], sk[:, m1:])
        assert not torch.equal(got, w)  # the tail rows did take the split path
        err = hml.error_fp64(0, 0, 0, M, N, K, 1.0, A, M, B, K, 0.0, None, C, M)
        assert err[2] <= 2 * (K + 2) * 2.0 ** -24, err
        assert hml.device_error() == 0
    finally:
        hml.tune_clear()
        hml.tune_load(os.path.join(os.path.dirname(hml.__file__), "data", "tuned_b200.txt"))
