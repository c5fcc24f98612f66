"""Batched noise trajectories on the GPU against the oracle.

Every trajectory of a device batch must take the same Kraus branches as the oracle's
NoisyCircuit.Execute restatement on the same draws, consume the same number of draws, and end
in the same state (checked through <Z_i>, <Z_i Z_i+1> and the Born mass).  FP64 states agree
with the oracle to 1e-12; FP32 states to 2e-5, with FP64 masses and renormalisation.
"""
from __future__ import annotations

import numpy as np
import pytest

import oracle as orc
from quantummatter_b200.backend import FP32, FP64
from quantummatter_b200.circuit import QuantumCircuit
from quantummatter_b200.errors import ArgumentOutOfRangeError
from quantummatter_b200.noise import NoiseChannel, NoisyCircuit
from quantummatter_b200.observables import PauliString
from quantummatter_b200.trajectories import B200NoisySimulator, SimulationOptions, random_doubles

pytestmark = pytest.mark.gpu


def label(n: int, ops: dict[int, str]) -> PauliString:
    return PauliString("".join(ops.get(q, "I") for q in reversed(range(n))))


def z_observables(n: int) -> list[PauliString]:
    return [label(n, {q: "Z"}) for q in range(n)] + [label(n, {q: "Z", q + 1: "Z"}) for q in range(n - 1)]


def mixed_circuit(n: int, seed: int, layers: int = 3, gamma: float = 0.35, dep: float = 0.6) -> NoisyCircuit:
    """RY layers, CNOT/CZ ladders, every channel kind, p = 0 and p = 1 flips, and a damping
    repeated on one qubit (the second finds no mass in |1> after a jump)."""
    rng = np.random.default_rng(seed)
    nc = NoisyCircuit(n)
    for _ in range(layers):
        c = QuantumCircuit(n)
        for q in range(n):
            c.Ry(q, float(rng.uniform(0, 2 * np.pi)))
        c.Rz(0, 0.3)
        nc.Append(c)
        for q in range(n):
            nc.ApplyNoise(NoiseChannel.Depolarizing(dep), q)
        ladder = QuantumCircuit(n)
        for q in range(n - 1):
            ladder.CZ(q, q + 1) if q % 2 else ladder.CNot(q, q + 1)
        nc.Append(ladder)
        nc.ApplyNoise(NoiseChannel.BitFlip(0.3), 0)
        nc.ApplyNoise(NoiseChannel.PhaseFlip(1.0), n - 1)
        nc.ApplyNoise(NoiseChannel.BitFlip(1.0), n // 2)
        nc.ApplyNoise(NoiseChannel.PhaseFlip(0.4), 1)
        nc.ApplyNoise(NoiseChannel.BitFlip(0.0), 0)
        for q in range(n):
            nc.ApplyNoise(NoiseChannel.AmplitudeDamping(gamma), q)
        nc.ApplyNoise(NoiseChannel.AmplitudeDamping(gamma), 0)
    return nc


def oracle_rows(nc: NoisyCircuit, draws: np.ndarray, observables):
    values, masses, used, branches = [], [], [], []
    for row in draws:
        state, u, br = orc.trajectory(nc, row)
        values.append([orc.expectation(state, o) for o in observables])
        masses.append(np.vdot(state, state).real)
        used.append(u)
        branches.append(br)
    return np.array(values), np.array(masses), np.array(used), np.array(branches)


@pytest.mark.parametrize("precision,tol", [(FP64, 1e-12), (FP32, 2e-5)])
@pytest.mark.parametrize("n", [3, 5, 10, 13])
def test_batch_matches_the_oracle(gpu_context, n, precision, tol):
    nc = mixed_circuit(n, 100 + n)
    T = 12
    draws = np.random.default_rng(n).random((T, nc.MaxDraws()))
    obs = z_observables(n)
    sim = B200NoisySimulator(gpu_context, precision=precision)
    res = sim.RunBatch(nc, draws, obs, branches=True)
    values, masses, used, branches = oracle_rows(nc, draws, obs)
    ok = res.ambiguous == 0
    if precision == FP64:
        assert ok.all()
    assert ok.sum() >= T - 1
    assert np.array_equal(res.consumed[ok], used[ok])
    assert np.array_equal(res.branches[ok], branches[ok])
    assert np.max(np.abs(res.values[ok] - values[ok])) <= tol
    assert np.max(np.abs(res.masses[ok] - masses[ok]) / masses[ok]) <= tol
    # every branch kind occurred
    flat = res.branches[ok].ravel()
    assert {-1, 0, 1, 2, 3} <= set(np.unique(flat).tolist())
    assert res.stats["mass_passes"] >= 3 * (1 if n <= 8 else 2)


def test_results_do_not_depend_on_the_batch(gpu_context):
    nc = mixed_circuit(10, 7, layers=2)
    draws = np.random.default_rng(3).random((6, nc.MaxDraws()))
    obs = z_observables(10)
    sim = B200NoisySimulator(gpu_context)
    together = sim.RunBatch(nc, draws, obs, branches=True)
    again = sim.RunBatch(nc, draws, obs, branches=True)
    assert np.array_equal(together.values, again.values)
    for t in range(draws.shape[0]):
        alone = sim.RunBatch(nc, draws[t:t + 1], obs, branches=True)
        assert np.array_equal(alone.values[0], together.values[t])
        assert np.array_equal(alone.branches[0], together.branches[t])
        assert alone.masses[0] == together.masses[t]


def test_run_counts_follow_the_reference_draw_order(gpu_context):
    nc = mixed_circuit(4, 11, layers=2, gamma=0.8)
    shots, seed = 48, 20260101
    counts = B200NoisySimulator(gpu_context).Run(nc, shots=shots, seed=seed).Counts
    r = orc.DotNetRandom(seed)
    stream = [r.NextDouble() for _ in range(shots * (nc.MaxDraws() + 1))]
    offset, want = 0, {}
    for _ in range(shots):
        state, used, _ = orc.trajectory(nc, stream[offset:])
        _, o = orc.measure_all(state, stream[offset + used])
        offset += used + 1
        key = format(o, "b").zfill(4)
        want[key] = want.get(key, 0) + 1
    assert counts == dict(sorted(want.items()))


def test_estimate_probabilities_matches_welford_on_the_oracle(gpu_context):
    nc = mixed_circuit(4, 13, layers=2)
    T, seed = 40, 5
    est = B200NoisySimulator(gpu_context).EstimateProbabilities(nc, trajectories=T, seed=seed)
    stream = random_doubles(seed, T * nc.MaxDraws())
    mean = np.zeros(16)
    m2 = np.zeros(16)
    offset = 0
    for t in range(T):
        state, used, _ = orc.trajectory(nc, stream[offset:])
        offset += used
        p = np.abs(state) ** 2 / np.vdot(state, state).real
        delta = p - mean
        mean += delta / (t + 1)
        m2 += delta * (p - mean)
    stderr = np.sqrt(np.maximum(0, m2) / (T * (T - 1)))
    assert np.max(np.abs(est.Probabilities - mean)) <= 1e-12
    assert np.max(np.abs(est.StandardErrors - stderr)) <= 1e-12
    assert est.Estimate(3).Probability == est.Probabilities[3]


def test_observable_estimates_in_reference_order(gpu_context):
    nc = mixed_circuit(12, 17, layers=2)
    obs = z_observables(12)
    res = B200NoisySimulator(gpu_context).EstimateObservables(nc, obs, trajectories=20, seed=9, branches=True)
    stream = random_doubles(9, 20 * nc.MaxDraws())
    offset = 0
    for t in range(20):
        state, used, br = orc.trajectory(nc, stream[offset:])
        offset += used
        assert np.array_equal(res.branches[t], br)
        want = np.array([orc.expectation(state, o) for o in obs])
        assert np.max(np.abs(res.values[t] - want)) <= 1e-12
    assert res.mean_values().shape == (len(obs),)


def test_too_few_draws_and_bad_channels_are_rejected(gpu_context):
    nc = mixed_circuit(9, 1, layers=1)
    sim = B200NoisySimulator(gpu_context)
    with pytest.raises(ArgumentOutOfRangeError):
        sim.RunBatch(nc, np.full((2, nc.MaxDraws() - 1), 0.5))
    with pytest.raises(ArgumentOutOfRangeError):
        sim.RunBatch(nc, np.full((2, nc.MaxDraws()), 1.0))  # draws must lie in [0,1)
    with pytest.raises(ArgumentOutOfRangeError):
        B200NoisySimulator(gpu_context, SimulationOptions(MemoryBudgetBytes=1024)).Run(nc, shots=2, seed=1)
