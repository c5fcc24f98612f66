"""Seeded random circuits over QuantumMatter's whole gate set (test infrastructure)."""
from __future__ import annotations

import math

import numpy as np

from quantummatter_b200.circuit import GateKind, GateOperation, QuantumCircuit, SingleQubitUnitary

SINGLE = [GateKind.H, GateKind.X, GateKind.Y, GateKind.Z, GateKind.S, GateKind.T, GateKind.Rx, GateKind.Ry,
          GateKind.Rz, GateKind.I, GateKind.Sdg, GateKind.Tdg, GateKind.Phase]
ANGLED = {GateKind.Rx, GateKind.Ry, GateKind.Rz, GateKind.Phase}


def random_unitary(rng: np.random.Generator) -> SingleQubitUnitary:
    z = rng.normal(size=(2, 2)) + 1j * rng.normal(size=(2, 2))
    q, r = np.linalg.qr(z)
    q = q * (np.diag(r) / np.abs(np.diag(r)))
    return SingleQubitUnitary.Create(q[0, 0], q[0, 1], q[1, 0], q[1, 1])


def random_circuit(qubits: int, gates: int, seed: int) -> QuantumCircuit:
    rng = np.random.default_rng(seed)
    c = QuantumCircuit(qubits)
    for _ in range(gates):
        r = rng.random()
        t = int(rng.integers(qubits))
        others = [q for q in range(qubits) if q != t]
        if r < 0.45 or not others:
            k = SINGLE[int(rng.integers(len(SINGLE)))]
            angle = float(rng.uniform(-2 * math.pi, 2 * math.pi)) if k in ANGLED else 0.0
            c.AppendValidated(GateOperation(k, t, -1, angle))
        elif r < 0.55:
            c.U(t, random_unitary(rng))
        elif r < 0.70:
            k = SINGLE[int(rng.integers(len(SINGLE)))]
            angle = float(rng.uniform(-2 * math.pi, 2 * math.pi)) if k in ANGLED else 0.0
            c.Controlled(k, int(rng.choice(others)), t, angle)
        elif r < 0.78:
            c.ControlledU(int(rng.choice(others)), t, random_unitary(rng))
        elif r < 0.88:
            c.CNot(int(rng.choice(others)), t)
        elif r < 0.95:
            c.Swap(int(rng.choice(others)), t)
        elif len(others) >= 2:
            a, b = rng.choice(others, size=2, replace=False)
            c.Toffoli(int(a), int(b), t)
    return c


def random_state(qubits: int, seed: int) -> np.ndarray:
    rng = np.random.default_rng(seed)
    v = rng.normal(size=1 << qubits) + 1j * rng.normal(size=1 << qubits)
    return (v / np.linalg.norm(v)).astype(np.complex128)


def circuit_to_arrays(c: QuantumCircuit) -> dict:
    ops = c.Operations
    u = np.zeros((len(ops), 8))
    for i, o in enumerate(ops):
        if o.Unitary is not None:
            m = o.Unitary
            u[i] = [m.M00.real, m.M00.imag, m.M01.real, m.M01.imag, m.M10.real, m.M10.imag, m.M11.real, m.M11.imag]
    return {
        "kind": np.array([int(o.Kind) for o in ops], dtype=np.int32),
        "target": np.array([o.Target for o in ops], dtype=np.int32),
        "control": np.array([o.Control for o in ops], dtype=np.int32),
        "second": np.array([o.SecondControl for o in ops], dtype=np.int32),
        "angle": np.array([o.Angle for o in ops], dtype=np.float64),
        "unitary": u,
    }


def circuit_from_arrays(qubits: int, d: dict) -> QuantumCircuit:
    c = QuantumCircuit(qubits)
    for i in range(len(d["kind"])):
        u = None
        if int(d["kind"][i]) == GateKind.Unitary:
            m = d["unitary"][i]
            u = SingleQubitUnitary(complex(m[0], m[1]), complex(m[2], m[3]), complex(m[4], m[5]), complex(m[6], m[7]))
        c.AppendValidated(GateOperation(GateKind(int(d["kind"][i])), int(d["target"][i]), int(d["control"][i]),
                                        float(d["angle"][i]), int(d["second"][i]), u))
    return c
