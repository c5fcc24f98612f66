"""Captured executions (qm_graph_*): a plan's launches recorded once as a CUDA graph and replayed.

A replay must evolve the state exactly as qm_plan_execute does: one replay from |0...0> equals
the oracle, and two replays equal two plan executions bit for bit.  Covered for fused-block plans
(compiled passes), dense fused gates and the per-gate path.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle as orc
from quantummatter_b200.backend import FP32, FP64, DeviceState, Plan
from quantummatter_b200.workloads import brick_circuit

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,tol", [(FP64, 1e-12), (FP32, 2e-6)])
@pytest.mark.parametrize("width", [0, 1, 4])
def test_replays_equal_plan_executions(gpu_context, width, precision, tol):
    n = 18
    c = brick_circuit(n, 6, seed=11)
    want = orc.execute(c)
    plan = Plan(gpu_context, c, precision, fusion_width=width)
    try:
        with DeviceState(gpu_context, n, precision) as st, DeviceState(gpu_context, n, precision) as ref:
            plan.execute(st)  # loads the plan's kernels before the capture
            st.Reset()
            graph = plan.capture(st)
            try:
                graph.launch()
                once = st.Download()
                prof = graph.launch(profile=True)
                twice = st.Download()
            finally:
                graph.Dispose()
            plan.execute(ref)
            plan.execute(ref)
            assert np.array_equal(twice, ref.Download())
    finally:
        plan.Dispose()
    assert np.max(np.abs(once - want)) <= tol
    assert prof.DeviceEvolutionSeconds > 0
