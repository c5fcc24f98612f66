"""The autotuner (qm_plan_autotune): candidate fusion widths timed on the device, the fastest
plan returned and its choice cached per gate structure."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as orc
from quantummatter_b200.backend import FP32, FP64, DeviceState, Plan
from quantummatter_b200.errors import QuantumMatterError
from quantummatter_b200.workloads import brick_circuit

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,tol", [(FP64, 1e-12), (FP32, 2e-6)])
def test_autotuned_plan_is_a_candidate_and_matches_the_oracle(gpu_context, precision, tol):
    n = 20
    c = brick_circuit(n, 8, seed=precision)
    candidates = [3, 5, 10, 12]
    plan = Plan.autotune(gpu_context, c, precision, candidates)
    try:
        assert plan.width in candidates
        with DeviceState(gpu_context, n, precision) as st:
            plan.execute(st)
            got = st.Download()
    finally:
        plan.Dispose()
    assert np.max(np.abs(got - orc.execute(c))) <= tol
    # same structure, other angles: the cached choice, no timing
    again = Plan.autotune(gpu_context, brick_circuit(n, 8, seed=99), precision, candidates)
    try:
        assert again.width == plan.width
    finally:
        again.Dispose()


def test_autotune_rejects_invalid_widths(gpu_context):
    with pytest.raises(QuantumMatterError):
        Plan.autotune(gpu_context, brick_circuit(12, 2), FP64, [7])
