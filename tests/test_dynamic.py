"""Device-resident measurement and dynamic circuits against the oracle."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as orc
from circuits import random_state
from dynamic_ref import execute, layered, noisy_layered, noisy_teleportation, teleportation
from quantummatter_b200.backend import FP32, FP64, DeviceState
from quantummatter_b200.dynamic import B200DynamicSimulator
from quantummatter_b200.errors import ArgumentError, ArgumentOutOfRangeError, MassError
from quantummatter_b200.trajectories import random_doubles

pytestmark = pytest.mark.gpu


@pytest.mark.parametrize("precision,tol", [(FP64, 1e-12), (FP32, 2e-6)])
@pytest.mark.parametrize("n", [3, 10, 14])
def test_measure_and_marginals_match_the_oracle(gpu_context, n, precision, tol):
    rng = np.random.default_rng(n)
    psi = random_state(n, 7 + n) * 1.3
    with DeviceState(gpu_context, n, precision) as st:
        for trial in range(4):
            st.Upload(psi)
            qubits = [int(q) for q in rng.choice(n, size=int(rng.integers(1, min(n, 4) + 1)), replace=False)]
            for o in range(1 << len(qubits)):
                want = orc.marginal_probability(psi, qubits, o)
                assert abs(st.MarginalProbability(qubits, o) - want) <= tol
            u = float(rng.random())
            outcome, amb = st.Measure(qubits, u)
            assert not amb
            want_state, want_outcome = orc.measure(psi, qubits, u)
            assert outcome == want_outcome
            assert np.max(np.abs(st.Download() - want_state)) <= tol


def test_measure_rejects_bad_selections(gpu_context):
    with DeviceState(gpu_context, 4, FP64) as st:
        with pytest.raises(ArgumentError):
            st.Measure([], 0.5)
        with pytest.raises(ArgumentError):
            st.Measure([1, 1], 0.5)
        with pytest.raises(ArgumentOutOfRangeError):
            st.Measure([4], 0.5)
        with pytest.raises(ArgumentOutOfRangeError):
            st.MarginalProbability([0, 1], 4)
        st.Upload(np.zeros(16, complex))
        with pytest.raises(MassError):
            st.MarginalProbability([0], 0)


@pytest.mark.parametrize("build,n", [(lambda: teleportation(), 3), (lambda: layered(12, 5), 12)])
def test_run_counts_follow_the_reference(gpu_context, build, n):
    dc = build()
    shots, seed = 40, 20260101
    res = B200DynamicSimulator(gpu_context).Run(dc, shots=shots, seed=seed)
    D = dc.DrawsPerExecution()
    draws = random_doubles(seed, shots * D)
    want = {}
    for s in range(shots):
        _, classical = execute(dc, draws[s * D:(s + 1) * D])
        key = format(classical, "b").zfill(dc.ClassicalBitCount)
        want[key] = want.get(key, 0) + 1
    assert res.Ambiguous == 0
    assert res.Counts == dict(sorted(want.items()))
    assert sum(res.Counts.values()) == shots


def test_simulate_trajectory_state(gpu_context):
    dc = layered(10, 9)
    t = B200DynamicSimulator(gpu_context).SimulateTrajectory(dc, seed=3)
    state, classical = execute(dc, random_doubles(3, dc.DrawsPerExecution()))
    assert t.ClassicalRegister == classical
    assert np.max(np.abs(t.FinalState - state)) <= 1e-12


@pytest.mark.parametrize("build,n", [(lambda: noisy_teleportation(), 3), (lambda: noisy_layered(12, 6), 12)])
def test_noisy_dynamic_run_counts_follow_the_reference(gpu_context, build, n):
    """Noise placements between dynamic instructions, applied on the resident state, take the
    same branches and draws as the oracle composition over one seeded stream across shots."""
    from dynamic_ref import execute_noisy
    from quantummatter_b200.dynamic import B200NoisyDynamicSimulator
    nd = build()
    shots, seed = 40, 7
    res = B200NoisyDynamicSimulator(gpu_context).Run(nd, shots=shots, seed=seed)
    draws = random_doubles(seed, 40 * 64)
    want, k = {}, 0
    for _ in range(shots):
        _, classical, used = execute_noisy(nd, draws[k:])
        k += used
        key = format(classical, "b").zfill(nd.ClassicalBitCount)
        want[key] = want.get(key, 0) + 1
    assert res.Ambiguous == 0
    assert res.Counts == dict(sorted(want.items()))


def test_noisy_dynamic_trajectory_state(gpu_context):
    from dynamic_ref import execute_noisy
    from quantummatter_b200.dynamic import B200NoisyDynamicSimulator
    nd = noisy_layered(10, 11)
    t = B200NoisyDynamicSimulator(gpu_context).SimulateTrajectory(nd, seed=5)
    state, classical, _ = execute_noisy(nd, random_doubles(5, 256))
    assert t.ClassicalRegister == classical
    assert np.max(np.abs(t.FinalState - state)) <= 1e-12
