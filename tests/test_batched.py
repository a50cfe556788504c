"""Batched SGEMM argument validation (CPU: rejected before any device work)."""
import pytest

import hiperml_b200 as hml
from hiperml_b200._lib import lib


@pytest.mark.parametrize("bad", [
    (0, 0, 64, 8, 32, 1.0, 8, 10, 8, 32, 0.0, 8, 64),    # lda < M
    (0, 0, 64, 8, 32, 1.0, 8, 64, 8, 31, 0.0, 8, 64),    # ldb < K
    (0, 0, 64, 8, 32, 1.0, 8, 64, 8, 32, 0.0, 8, 63),    # ldc < M
    (0, 0, -1, 8, 32, 1.0, 8, 64, 8, 32, 0.0, 8, 64),    # negative M
    (2, 0, 64, 8, 32, 1.0, 8, 64, 8, 32, 0.0, 8, 64),    # bad transpose
    (0, 0, 64, 8, 32, 1.0, None, 64, 8, 32, 0.0, 8, 64),  # missing A
])
def test_plan_rejects_invalid_problem(bad):
    good = (0, 0, 64, 8, 32, 1.0, 8, 64, 8, 32, 0.0, 8, 64)
    with pytest.raises(hml.HmlError) as e:
        hml.BatchPlan(hml.COL_MAJOR, [good, good, bad])
    assert "invalid value" in str(e.value)
    assert b"batch problem 2" in lib.hml_last_error()
    with pytest.raises(hml.HmlError):
        hml.sgemm_batched(hml.COL_MAJOR, [bad], stream=0)


def test_plan_rejects_bad_order_and_count():
    assert lib.hml_batch_plan_create(7, None, 0, None) != 0
    import ctypes
    h = ctypes.c_void_p()
    assert lib.hml_batch_plan_create(0, None, -1, ctypes.byref(h)) == 1
    assert lib.hml_batch_plan_create(0, None, 3, ctypes.byref(h)) == 1
    assert lib.hml_batch_plan_run(None, None) == 1
    assert lib.hml_batch_plan_destroy(None) == 0
