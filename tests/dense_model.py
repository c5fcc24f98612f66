"""Independent dense-matrix model of QuantumMatter's gate set (test infrastructure).

The reference's conformance suite checks its kernels against dense 2^n x 2^n operators
built from textbook matrices (tests/QuantumMatter.Tests/StateVectorBackendConformanceTests.cs:146-245,
ExtendedGateConformanceTests.cs:86-163).  This module is that method, written independently
of the oracle: every gate becomes a full matrix (controls as projectors), states are
multiplied by it.  Used to pin the oracle and to generate the fixtures in tests/golden/.
"""
from __future__ import annotations

import cmath
import math

import numpy as np

I2 = np.eye(2, dtype=complex)
P0 = np.array([[1, 0], [0, 0]], dtype=complex)
P1 = np.array([[0, 0], [0, 1]], dtype=complex)

# GateKind numbering (QuantumCircuit.cs:4-40)
H, X, Y, Z, S, T, RX, RY, RZ, CNOT, SWAP, I, SDG, TDG, PHASE, UNITARY, TOFFOLI = range(17)


def single_matrix(kind: int, angle: float = 0.0, unitary=None) -> np.ndarray:
    """Column-vector matrices of the reference's doc comments (QuantumCircuit.cs:6-38)."""
    h = 1 / math.sqrt(2)
    if kind == H:
        return np.array([[h, h], [h, -h]], dtype=complex)
    if kind in (X, CNOT, TOFFOLI):
        return np.array([[0, 1], [1, 0]], dtype=complex)
    if kind == Y:
        return np.array([[0, -1j], [1j, 0]], dtype=complex)
    if kind == Z:
        return np.diag([1, -1]).astype(complex)
    if kind == S:
        return np.diag([1, 1j])
    if kind == SDG:
        return np.diag([1, -1j])
    if kind == T:
        return np.diag([1, cmath.exp(1j * math.pi / 4)])
    if kind == TDG:
        return np.diag([1, cmath.exp(-1j * math.pi / 4)])
    if kind == PHASE:
        return np.diag([1, cmath.exp(1j * angle)])
    if kind == RX:
        c, s = math.cos(angle / 2), math.sin(angle / 2)
        return np.array([[c, -1j * s], [-1j * s, c]])
    if kind == RY:
        c, s = math.cos(angle / 2), math.sin(angle / 2)
        return np.array([[c, -s], [s, c]], dtype=complex)
    if kind == RZ:
        return np.diag([cmath.exp(-1j * angle / 2), cmath.exp(1j * angle / 2)])
    if kind == I:
        return I2.copy()
    if kind == UNITARY:
        return np.array([[unitary.M00, unitary.M01], [unitary.M10, unitary.M11]], dtype=complex)
    raise ValueError(kind)


def embed(op: np.ndarray, target: int, qubits: int) -> np.ndarray:
    """Operator on one qubit of an n-qubit register (qubit 0 = least significant index bit)."""
    out = np.array([[1]], dtype=complex)
    for q in reversed(range(qubits)):
        out = np.kron(out, op if q == target else I2)
    return out


def projector(bits: dict[int, int], qubits: int) -> np.ndarray:
    out = np.array([[1]], dtype=complex)
    for q in reversed(range(qubits)):
        m = I2 if q not in bits else (P1 if bits[q] else P0)
        out = np.kron(out, m)
    return out


def gate_operator(op, qubits: int) -> np.ndarray:
    """Dense operator of one GateOperation-like record."""
    kind = int(op.Kind)
    dim = 1 << qubits
    if kind == SWAP:
        a, b = op.Control, op.Target
        m = np.zeros((dim, dim), dtype=complex)
        for i in range(dim):
            ba, bb = (i >> a) & 1, (i >> b) & 1
            j = i if ba == bb else i ^ (1 << a) ^ (1 << b)
            m[j, i] = 1
        return m
    u = embed(single_matrix(kind, op.Angle, op.Unitary), op.Target, qubits)
    controls = [c for c in (op.Control, op.SecondControl) if c >= 0]
    if not controls:
        return u
    on = projector({c: 1 for c in controls}, qubits)
    return on @ u + (np.eye(dim, dtype=complex) - on)


def run(circuit, state: np.ndarray | None = None) -> np.ndarray:
    n = circuit.QubitCount
    psi = np.zeros(1 << n, dtype=complex) if state is None else np.array(state, dtype=complex)
    if state is None:
        psi[0] = 1
    for op in circuit.Operations:
        psi = gate_operator(op, n) @ psi
    return psi


def pauli_operator(labels: str) -> np.ndarray:
    mats = {"I": I2, "X": single_matrix(X), "Y": single_matrix(Y), "Z": single_matrix(Z)}
    out = np.array([[1]], dtype=complex)
    for ch in labels:  # leftmost label = highest qubit
        out = np.kron(out, mats[ch])
    return out


def expectation(psi: np.ndarray, labels: str) -> float:
    return float(np.real(np.vdot(psi, pauli_operator(labels) @ psi)) / np.real(np.vdot(psi, psi)))
