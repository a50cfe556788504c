"""The stream-K SIMT kernel for N <= 8 with contiguous columns of A
(sgemm_stream.cu) against the oracle (GPU): both storage orders of B, ragged
M, N and K, strips shared by many CTAs (their partial sums combined by the
last CTA to arrive), repeatability, beta == 0, and the full-size N = 8 sweep
shape against FP64."""
import numpy as np
import pytest

import hiperml_b200 as hml
from hiperml_b200 import datagen as dg
from hiperml_b200._lib import SgemmConfig
from tests.gpu_util import assert_within_fp32_bound
from tests.test_sgemm_gpu import STREAM_VARIANT0, run_case

pytestmark = pytest.mark.gpu


def stream_configs():
    return [c for c in hml.configs() if c.algo == hml.ALGO_SIMT and c.variant >= STREAM_VARIANT0]


STREAM = stream_configs()
NB = sorted({c.tile_n for c in STREAM})


def cfg_for(nb, stages=None):
    cands = [c for c in STREAM if c.tile_n == nb]
    if stages is None:
        return max(cands, key=lambda c: c.stages)
    return [c for c in cands if c.stages == stages][0]


def test_stream_configs_in_space():
    assert NB == [4, 8]
    assert all(c.tile_m == 128 and c.split_k == 1 for c in STREAM)


# (order, transA, transB): A's columns contiguous in every case; B stored
# K-contiguous in the first two, N-contiguous in the last two
LAYOUTS = [(0, 0, 0), (1, 1, 1), (0, 0, 1), (1, 1, 0)]


@pytest.mark.parametrize("layout", LAYOUTS)
@pytest.mark.parametrize("nb", [4, 8])
def test_stream_layouts_and_ragged_shapes(cuda, layout, nb):
    """TMA needs A's leading dimension a multiple of 4 floats (M is), and
    B's too where B is stored N-contiguous (ldb = N).  A K-contiguous B is
    copied N-contiguous first, so any ldb works there (K = 333)."""
    order, ta, tb = layout
    cfg = cfg_for(nb)
    b_ncontig = layout in ((0, 0, 1), (1, 1, 0))
    ns = sorted({4, nb}) if b_ncontig else sorted({1, max(1, nb // 2 - 1), nb})
    shapes = [(1000, 332), (128, 32), (132, 4), (4100, 1000)]
    if not b_ncontig:
        shapes.append((1000, 333))
    for (M, K) in shapes:
        for N in ns:
            got, D, absD = run_case(M, N, K, order, ta, tb, 0.75, -0.5, config=cfg)
            assert_within_fp32_bound(got, D, absD, max(K, 1), what=f"{cfg} {layout} {M}x{N}x{K}")


@pytest.mark.parametrize("stages", [None, "min"])
def test_stream_every_ring_depth(cuda, stages):
    for nb in NB:
        depths = sorted(c.stages for c in STREAM if c.tile_n == nb)
        cfg = cfg_for(nb, depths[0] if stages == "min" else None)
        got, D, absD = run_case(2000, nb, 2500, 0, 0, 0, 1.0, 1.0, config=cfg)
        assert_within_fp32_bound(got, D, absD, 2500, what=str(cfg))


def test_stream_strips_shared_by_many_ctas(cuda):
    """Few strips and a long K: every strip is split across dozens of CTAs,
    and a CTA's range can start and end inside strips."""
    for nb in NB:
        cfg = cfg_for(nb)
        for (M, K) in ((200, 20000), (128, 40000), (700, 9000)):
            got, D, absD = run_case(M, nb, K, 0, 0, 0, 1.0, 0.0, config=cfg)
            assert_within_fp32_bound(got, D, absD, K, what=f"{cfg} {M}x{K}")


def test_stream_repeatable_and_counters_reset(cuda):
    """Partial sums are combined in CTA order whatever order the CTAs finish
    in: repeated calls give the same bits, also after calls of other shapes
    (the per-strip arrival counters are left at zero)."""
    import torch
    cfg = cfg_for(8)
    M, N, K = 900, 8, 30000
    A = torch.empty(M * K, device="cuda")
    B = torch.empty(K * N, device="cuda")
    hml.fill_random(A, 7, 0, dg.NORMAL)
    hml.fill_random(B, 7, 1, dg.NORMAL)
    outs = []
    for i in range(4):
        C = torch.zeros(M * N, device="cuda")
        hml.sgemm_ex(0, 0, 0, M, N, K, 1.0, A, M, B, K, 0.0, C, M, config=cfg)
        outs.append(C.cpu().numpy())
        # another shape in between, with other strips and counters
        got, D, absD = run_case(300 + 128 * i, 5, 7000, 0, 0, 0, 1.0, 0.0, config=cfg)
        assert_within_fp32_bound(got, D, absD, 7000)
    for o in outs[1:]:
        assert np.array_equal(o, outs[0])
    assert hml.device_error() == 0


def test_stream_beta_zero_does_not_read_c(cuda):
    import torch
    cfg = cfg_for(8)
    M, N, K = 1000, 7, 5000
    A = torch.empty(M * K, device="cuda")
    B = torch.empty(K * N, device="cuda")
    hml.fill_random(A, 8, 0, dg.UNIFORM)
    hml.fill_random(B, 8, 1, dg.UNIFORM)
    C = torch.full((M * N,), float("nan"), device="cuda")
    hml.sgemm_ex(0, 0, 0, M, N, K, 1.0, A, M, B, K, 0.0, C, M, config=cfg)
    assert torch.isfinite(C).all()


def test_stream_rejects_unsupported(cuda):
    cfg = cfg_for(8)
    # A row-major (K contiguous) is not this kernel's layout
    assert hml.config_check(1, 0, 0, 1000, 8, 64, 64, 8, 8, cfg) == 2
    # N above the tile
    assert hml.config_check(0, 0, 0, 1000, 9, 64, 1000, 64, 1000, cfg) == 2
    # no 16-wide stream tile
    wide = SgemmConfig(hml.ALGO_SIMT, 128, 16, 1, cfg.stages, cfg.variant + 1)
    assert hml.config_check(0, 0, 0, 1000, 16, 64, 1000, 64, 1000, wide) == 1
    # lda not a multiple of 4 floats: no TMA
    assert hml.config_check(0, 0, 0, 1001, 8, 64, 1001, 64, 1001, cfg) == 2
    bad = SgemmConfig(hml.ALGO_SIMT, 128, 8, 2, cfg.stages, cfg.variant)  # split_k must be 1
    assert hml.config_check(0, 0, 0, 1000, 8, 64, 1000, 64, 1000, bad) == 1


def test_stream_is_the_heuristic_for_skinny_columns(cuda):
    cfg = hml.select_algo(0, 0, 0, 65536, 8, 4096, hml.ALGO_SIMT)
    assert cfg.variant >= STREAM_VARIANT0 and cfg.tile_n == 8
    # leading dimensions TMA cannot take: the tiled kernel instead
    cfg = hml.select_algo(0, 0, 1, 1001, 5, 333, hml.ALGO_SIMT)
    assert cfg.variant < STREAM_VARIANT0
    got, D, absD = run_case(1001, 5, 333, 0, 0, 1, 1.0, 0.0, config=cfg)
    assert_within_fp32_bound(got, D, absD, 333)


@pytest.mark.parametrize("N", [4, 8])
def test_stream_full_size_fp64(cuda, N):
    """M = 65536, K = 4096 (the sweep's N = 8 shape, and N = 4), uniform and
    log-uniform magnitudes, checked in FP64 on the GPU."""
    import torch
    M, K = 65536, 4096
    cfg = cfg_for(N)
    A = torch.empty(M * K, device="cuda")
    B = torch.empty(K * N, device="cuda")
    C = torch.zeros(M * N, device="cuda")
    for dist in (dg.UNIFORM, dg.LOGUNIFORM):
        hml.fill_random(A, 2, 0, dist)
        hml.fill_random(B, 2, 1, dist)
        hml.sgemm_ex(0, 0, 0, M, N, K, 1.0, A, M, B, K, 0.0, C, M, config=cfg)
        err = hml.error_fp64(0, 0, 0, M, N, K, 1.0, A, M, B, K, 0.0, None, C, M)
        assert err[2] <= 2 * (K + 2) * 2.0 ** -24, err
        assert err[0] < 1e-5, err
