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
