"""DynamicCircuit.Execute (src/QuantumMatter.Core/Dynamic/DynamicCircuit.cs:77-112) on the oracle:
the reference semantics the device simulator is checked against (test infrastructure)."""
from __future__ import annotations

import numpy as np

import oracle as orc
from quantummatter_b200.circuit import QuantumCircuit
from quantummatter_b200.dynamic import DynamicCircuit, MeasurementStep, UnitaryStep


def execute(circuit: DynamicCircuit, draws) -> tuple[np.ndarray, int]:
    state = orc.zero_state(circuit.QubitCount)
    classical, k = 0, 0
    for step in circuit.Steps:
        if isinstance(step, UnitaryStep):
            if (classical & step.Mask) == step.Value:
                state = orc.execute(step.Circuit, state)
        elif isinstance(step, MeasurementStep):
            state, outcome = orc.measure(state, step.Qubits, draws[k])
            k += 1
            written = 0
            for bit, cb in enumerate(step.ClassicalBits):
                written |= ((outcome >> bit) & 1) << cb
            classical = (classical & ~step.WriteMask) | written
        else:
            state, outcome = orc.measure(state, [step.Qubit], draws[k])
            k += 1
            if outcome != 0:
                state = orc.execute(QuantumCircuit(circuit.QubitCount).X(step.Qubit), state)
    return state, classical


def teleportation(theta: float = 1.1, phi: float = 0.4) -> DynamicCircuit:
    """Teleports Ry(theta)Rz(phi)|0> from qubit 0 to qubit 2, with a reset of qubit 0 and a final
    measurement of qubit 2 into classical bit 2."""
    dc = DynamicCircuit(3, 3)
    dc.Append(QuantumCircuit(3).Ry(0, theta).Rz(0, phi).H(1).CNot(1, 2).CNot(0, 1).H(0))
    dc.Measure([0, 1], [0, 1])
    dc.If(2, 2, QuantumCircuit(3).X(2))
    dc.If(1, 1, QuantumCircuit(3).Z(2))
    dc.Reset(0)
    dc.Measure([2], [2])
    return dc


def layered(n: int, seed: int) -> DynamicCircuit:
    """Random rotations and CNOT ladders with mid-circuit measurements of several qubits and
    conditioned segments."""
    rng = np.random.default_rng(seed)
    dc = DynamicCircuit(n, 4)
    for layer in range(3):
        c = QuantumCircuit(n)
        for q in range(n):
            c.Ry(q, float(rng.uniform(0, 6.28))).Rz(q, float(rng.uniform(0, 6.28)))
        for q in range(layer % 2, n - 1, 2):
            c.CNot(q, q + 1)
        dc.Append(c)
        qs = [int(x) for x in rng.choice(n, size=2, replace=False)]
        dc.Measure(qs, [layer % 4, (layer + 1) % 4])
        dc.If(1 << (layer % 4), 1 << (layer % 4), QuantumCircuit(n).H(int(rng.integers(n))).CNot(0, n - 1))
        dc.Reset(int(rng.integers(n)))
    return dc


def execute_noisy(circuit, draws) -> tuple[np.ndarray, int, int]:
    """NoisyDynamicCircuit execution (NoisyDynamicCircuit.cs:80-100) on the oracle: the dynamic
    steps as above and every noise placement through the oracle's CpuNoiseChannelBackend, each
    consuming its draws where the reference does.  Returns (state, classical, draws used)."""
    from quantummatter_b200.dynamic import NoiseStep, ResetStep
    state = orc.zero_state(circuit.QubitCount)
    classical, k = 0, 0
    for step in circuit.Steps:
        if isinstance(step, UnitaryStep):
            if (classical & step.Mask) == step.Value:
                state = orc.execute(step.Circuit, state)
        elif isinstance(step, MeasurementStep):
            state, outcome = orc.measure(state, step.Qubits, draws[k])
            k += 1
            written = 0
            for bit, cb in enumerate(step.ClassicalBits):
                written |= ((outcome >> bit) & 1) << cb
            classical = (classical & ~step.WriteMask) | written
        elif isinstance(step, ResetStep):
            state, outcome = orc.measure(state, [step.Qubit], draws[k])
            k += 1
            if outcome != 0:
                state = orc.execute(QuantumCircuit(circuit.QubitCount).X(step.Qubit), state)
        else:
            assert isinstance(step, NoiseStep)
            state, used = orc.noise_apply(int(step.Channel.Kind), step.Channel.Probability, step.Target, state,
                                          draws[k:k + 1])
            k += used
    return state, classical, k


def noisy_teleportation():
    """Teleportation with a channel of every kind placed inside it, including p = 1 (a flip that
    takes no draw) and p = 0 (no draw, no work)."""
    from quantummatter_b200.dynamic import NoisyDynamicCircuit
    from quantummatter_b200.noise import NoiseChannel
    nd = NoisyDynamicCircuit(3, 3)
    nd.Append(QuantumCircuit(3).Ry(0, 1.1).Rz(0, 0.4).H(1).CNot(1, 2))
    nd.ApplyNoise(NoiseChannel.Depolarizing(0.3), 2)
    nd.Append(QuantumCircuit(3).CNot(0, 1).H(0))
    nd.ApplyNoise(NoiseChannel.AmplitudeDamping(0.4), 0)
    nd.Measure([0, 1], [0, 1])
    nd.ApplyNoise(NoiseChannel.PhaseFlip(0.0), 1)
    nd.If(2, 2, QuantumCircuit(3).X(2))
    nd.If(1, 1, QuantumCircuit(3).Z(2))
    nd.ApplyNoise(NoiseChannel.BitFlip(1.0), 0)
    nd.Reset(0)
    nd.ApplyNoise(NoiseChannel.BitFlip(0.25), 2)
    nd.Measure([2], [2])
    return nd


def noisy_layered(n: int, seed: int):
    """Random rotations, CNOT ladders, mid-circuit measurements and resets with damping and
    depolarizing channels between them."""
    from quantummatter_b200.dynamic import NoisyDynamicCircuit
    from quantummatter_b200.noise import NoiseChannel
    rng = np.random.default_rng(seed)
    nd = NoisyDynamicCircuit(n, 4)
    for layer in range(3):
        c = QuantumCircuit(n)
        for q in range(n):
            c.Ry(q, float(rng.uniform(0, 6.28))).Rz(q, float(rng.uniform(0, 6.28)))
        for q in range(layer % 2, n - 1, 2):
            c.CNot(q, q + 1)
        nd.Append(c)
        nd.ApplyNoise(NoiseChannel.AmplitudeDamping(0.3), int(rng.integers(n)))
        nd.ApplyNoise(NoiseChannel.Depolarizing(0.5), int(rng.integers(n)))
        qs = [int(x) for x in rng.choice(n, size=2, replace=False)]
        nd.Measure(qs, [layer % 4, (layer + 1) % 4])
        nd.If(1 << (layer % 4), 1 << (layer % 4), QuantumCircuit(n).H(int(rng.integers(n))).CNot(0, n - 1))
        nd.Reset(int(rng.integers(n)))
    return nd
