"""Dynamic-circuit IR and the oracle's Measure / MarginalProbability (no GPU)."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as orc
from circuits import random_state
from dynamic_ref import execute, teleportation
from quantummatter_b200.circuit import QuantumCircuit
from quantummatter_b200.dynamic import DynamicCircuit
from quantummatter_b200.errors import ArgumentError, ArgumentOutOfRangeError


def test_builder_validation():
    with pytest.raises(ArgumentOutOfRangeError):
        DynamicCircuit(3, 0)
    dc = DynamicCircuit(3, 2)
    with pytest.raises(ArgumentOutOfRangeError):
        dc.If(4, 0, QuantumCircuit(3))            # mask outside the register
    with pytest.raises(ArgumentOutOfRangeError):
        dc.If(1, 2, QuantumCircuit(3))            # value outside the mask
    with pytest.raises(ArgumentError):
        dc.Append(QuantumCircuit(2))
    with pytest.raises(ArgumentError):
        dc.Measure([0, 1], [0])
    with pytest.raises(ArgumentError):
        dc.Measure([0, 0], [0, 1])
    with pytest.raises(ArgumentOutOfRangeError):
        dc.Measure([0], [2])
    with pytest.raises(ArgumentOutOfRangeError):
        dc.Reset(3)
    dc.Append(QuantumCircuit(3).H(0)).Measure([0], [1]).Reset(0)
    assert dc.StepCount == 3 and dc.DrawsPerExecution() == 2


def dense_measure(psi, qubits, u):
    """Independent model: full-basis CDF draw, projection onto the selected bits."""
    p = np.abs(psi) ** 2
    total = p.sum()
    basis = int(np.searchsorted(np.cumsum(p), u * total, side="right"))
    mask = sum(1 << q for q in qubits)
    idx = np.arange(psi.size)
    keep = (idx & mask) == (basis & mask)
    out = np.where(keep, psi, 0)
    out = out / np.sqrt(np.sum(np.abs(out) ** 2))
    outcome = sum(((basis >> q) & 1) << k for k, q in enumerate(qubits))
    return out, outcome


@pytest.mark.parametrize("seed", range(6))
def test_oracle_measure_and_marginals_match_a_dense_model(seed):
    n = 6
    rng = np.random.default_rng(seed)
    psi = random_state(n, seed) * 1.7
    qubits = [int(q) for q in rng.choice(n, size=int(rng.integers(1, 4)), replace=False)]
    u = float(rng.random())
    got, outcome = orc.measure(psi, qubits, u)
    want, want_outcome = dense_measure(psi, qubits, u)
    assert outcome == want_outcome
    assert np.max(np.abs(got - want)) <= 1e-12
    p = np.abs(psi) ** 2
    for o in range(1 << len(qubits)):
        sel = sum(((o >> k) & 1) << q for k, q in enumerate(qubits))
        mask = sum(1 << q for q in qubits)
        want_p = p[(np.arange(psi.size) & mask) == sel].sum() / p.sum()
        assert abs(orc.marginal_probability(psi, qubits, o) - want_p) <= 1e-13


def test_bell_pair_measurement_known_answers():
    bell = np.zeros(4, complex)
    bell[0] = bell[3] = 2 ** -0.5
    for u, bit in ((0.25, 0), (0.75, 1)):
        state, outcome = orc.measure(bell, [0], u)
        assert outcome == bit
        assert abs(state[3 * bit] - 1) < 1e-15 and np.sum(np.abs(state) ** 2) == pytest.approx(1)
    assert orc.marginal_probability(bell, [0, 1], 1) == 0  # |01> has no support
    assert orc.marginal_probability(bell, [1, 0], 3) == pytest.approx(0.5)


def test_teleportation_moves_the_state():
    """The teleported qubit's Z statistics equal those of the input state for every branch."""
    dc = teleportation(theta=1.1, phi=0.4)
    for draws in ([0.1, 0.3, 0.2, 0.5], [0.9, 0.8, 0.7, 0.5], [0.4, 0.6, 0.3, 0.5]):
        state, classical = execute(dc, draws[:3] + [0.0])
        assert 0 <= classical < 8
    # before the final measurement, qubit 2 holds Ry(1.1)Rz(0.4)|0>: P(1) = sin^2(0.55)
    dc2 = DynamicCircuit(3, 3)
    for step in teleportation().Steps[:-1]:
        dc2._steps.append(step)
    state, _ = execute(dc2, [0.3, 0.7, 0.2])
    assert orc.marginal_probability(state, [2], 1) == pytest.approx(np.sin(0.55) ** 2, abs=1e-12)


def test_noisy_dynamic_builder():
    """NoisyDynamicCircuit validates each instruction before taking it; channels are checked as
    NoisyCircuit.ApplyNoise checks them, and a rejected instruction changes nothing."""
    from quantummatter_b200.dynamic import MeasurementStep, NoiseStep, NoisyDynamicCircuit, UnitaryStep
    from quantummatter_b200.noise import NoiseChannel
    nd = NoisyDynamicCircuit(3, 2)
    nd.Append(QuantumCircuit(3).H(0)).ApplyNoise(NoiseChannel.Depolarizing(0.1), 2).Measure([0], [1])
    assert nd.StepCount == 3
    kinds = [type(s) for s in nd.Steps]
    assert kinds == [UnitaryStep, NoiseStep, MeasurementStep]
    with pytest.raises(ArgumentOutOfRangeError):
        nd.ApplyNoise(NoiseChannel.BitFlip(0.1), 3)
    with pytest.raises(ArgumentError):
        nd.ApplyNoise(None, 0)
    with pytest.raises(ArgumentError):
        nd.Append(QuantumCircuit(2).H(0))
    with pytest.raises(ArgumentOutOfRangeError):
        nd.If(4, 0, QuantumCircuit(3))
    assert nd.StepCount == 3
    with pytest.raises(ArgumentOutOfRangeError):
        NoisyDynamicCircuit(0, 1)


def test_noisy_dynamic_reference_composition_consumes_draws_like_the_reference():
    """The oracle composition takes no draw for p = 0 and for a flip with p = 1."""
    from dynamic_ref import execute_noisy, noisy_teleportation
    nd = noisy_teleportation()
    draws = np.random.default_rng(4).random(64)
    _, _, used = execute_noisy(nd, draws)
    # depolarizing, damping (both branches carry mass here), two measurements, reset, flip 0.25
    assert used == 6
