"""Seeded synthetic workloads of the benchmark configurations.

All inputs are synthetic (the reference measures on synthetic circuits only,
benchmarks/QuantumMatter.Benchmarks/CudaBenchmarks.cs:118-146).  Angles come from a
SplitMix64 stream so every run, test and benchmark sees identical circuits.
"""
from __future__ import annotations

import math

from .circuit import QuantumCircuit, u3

MASK64 = (1 << 64) - 1
DEFAULT_SEED = 20260101


class SplitMix64:
    """SplitMix64 (Steele, Lea, Flood 2014) with doubles from the top 53 bits."""

    def __init__(self, seed: int):
        self.state = seed & MASK64

    def next_u64(self) -> int:
        self.state = (self.state + 0x9E3779B97F4A7C15) & MASK64
        z = self.state
        z = ((z ^ (z >> 30)) * 0xBF58476D1CE4E5B9) & MASK64
        z = ((z ^ (z >> 27)) * 0x94D049BB133111EB) & MASK64
        return z ^ (z >> 31)

    def next_double(self) -> float:
        return (self.next_u64() >> 11) * (1.0 / (1 << 53))

    def uniform(self, lo: float, hi: float) -> float:
        return lo + (hi - lo) * self.next_double()

    def normal(self, mu: float = 0.0, sigma: float = 1.0) -> float:
        u1 = 1.0 - self.next_double()
        u2 = self.next_double()
        return mu + sigma * math.sqrt(-2.0 * math.log(u1)) * math.cos(2 * math.pi * u2)


def brick_circuit(qubits: int, depth: int, seed: int = DEFAULT_SEED) -> QuantumCircuit:
    """Random U3 + brick-pattern CNOT circuit.

    Each layer: U3(theta, phi, lambda) on every qubit with angles uniform in [0, 2pi), then
    CNOT(2i, 2i+1) on even layers and CNOT(2i+1, 2i+2) on odd layers.  20 qubits x 20 layers
    gives 400 U3 + 190 CNOT = 590 gates; 30 x 40 gives 1200 + 580 = 1780.
    """
    rng = SplitMix64(seed)
    c = QuantumCircuit(qubits)
    two_pi = 2 * math.pi
    for layer in range(depth):
        for q in range(qubits):
            theta, phi, lam = rng.uniform(0, two_pi), rng.uniform(0, two_pi), rng.uniform(0, two_pi)
            c.U(q, u3(theta, phi, lam))
        start = 0 if layer % 2 == 0 else 1
        for q in range(start, qubits - 1, 2):
            c.CNot(q, q + 1)
    return c


def gate_count(circuit: QuantumCircuit) -> int:
    return len(circuit.Operations)


def hardware_efficient_ansatz(qubits: int, layers: int = 4):
    """Layers of RY on every qubit, RZ on every qubit, then a CZ ladder (i, i+1); 2 * qubits
    parameters per layer, so P = 8 * qubits for four layers."""
    from .variational import ParameterizedCircuit
    c = ParameterizedCircuit(qubits, 2 * qubits * layers)
    p = 0
    for _ in range(layers):
        for q in range(qubits):
            c.Ry(q, p)
            p += 1
        for q in range(qubits):
            c.Rz(q, p)
            p += 1
        ladder = QuantumCircuit(qubits)
        for q in range(qubits - 1):
            ladder.CZ(q, q + 1)
        c.Append(ladder)
    return c


def xxz_chain(qubits: int, seed: int = DEFAULT_SEED):
    """Open 1D Heisenberg XXZ chain: sum_i J_i (X_i X_{i+1} + Y_i Y_{i+1} + Delta_i Z_i Z_{i+1}) + sum_i h_i Z_i
    with J ~ U[0.5, 1.5], Delta ~ U[0, 2], h ~ N(0, 0.3): 4n - 3 Pauli terms."""
    from .observables import PauliHamiltonian, PauliString, PauliTerm
    rng = SplitMix64(seed ^ (qubits * 0x9E37))

    def label(pairs: dict[int, str]) -> str:
        return "".join(pairs.get(q, "I") for q in reversed(range(qubits)))

    terms = []
    for i in range(qubits - 1):
        j, delta = rng.uniform(0.5, 1.5), rng.uniform(0.0, 2.0)
        terms.append(PauliTerm(j, PauliString(label({i: "X", i + 1: "X"}))))
        terms.append(PauliTerm(j, PauliString(label({i: "Y", i + 1: "Y"}))))
        terms.append(PauliTerm(j * delta, PauliString(label({i: "Z", i + 1: "Z"}))))
    for i in range(qubits):
        terms.append(PauliTerm(rng.normal(0.0, 0.3), PauliString(label({i: "Z"}))))
    return PauliHamiltonian(qubits, terms)


def tfim_chain(qubits: int, seed: int = DEFAULT_SEED):
    """Transverse-field Ising chain H = -sum J Z_i Z_{i+1} - sum h X_i with J, h ~ U[0.5, 1.5]."""
    from .observables import PauliHamiltonian, PauliString, PauliTerm
    rng = SplitMix64(seed ^ (qubits * 0x51ED))

    def label(pairs: dict[int, str]) -> str:
        return "".join(pairs.get(q, "I") for q in reversed(range(qubits)))

    terms = [PauliTerm(-rng.uniform(0.5, 1.5), PauliString(label({i: "Z", i + 1: "Z"}))) for i in range(qubits - 1)]
    terms += [PauliTerm(-rng.uniform(0.5, 1.5), PauliString(label({i: "X"}))) for i in range(qubits)]
    return PauliHamiltonian(qubits, terms)


def uniform_parameters(count: int, vectors: int, lo: float, hi: float, seed: int = DEFAULT_SEED):
    import numpy as np
    rng = SplitMix64(seed)
    return np.array([[rng.uniform(lo, hi) for _ in range(count)] for _ in range(vectors)], dtype=np.float64)


def noisy_ry_cz_ladder(qubits: int, depth: int, seed: int = DEFAULT_SEED, p1: float = 1e-3, p2: float = 1e-2,
                       gamma: float = 1e-3):
    """Noisy RY / CZ-ladder circuit of the trajectory workload.

    Each layer: RY(theta ~ U[0, 2pi)) on every qubit, each followed by depolarizing(p1) on its
    qubit; then CZ(i, i+1) for i = 0..n-2, each followed by depolarizing(p2) on both of its
    qubits; then amplitude damping(gamma) on every qubit.  24 qubits x 30 layers gives
    30 x (24 + 23) = 1410 gates and 30 x (24 + 46 + 24) = 2820 channel placements.
    """
    from .noise import NoiseChannel, NoisyCircuit
    rng = SplitMix64(seed)
    nc = NoisyCircuit(qubits)
    dep1, dep2, damp = NoiseChannel.Depolarizing(p1), NoiseChannel.Depolarizing(p2), NoiseChannel.AmplitudeDamping(gamma)
    two_pi = 2 * math.pi
    for _ in range(depth):
        for q in range(qubits):
            nc.Append(QuantumCircuit(qubits).Ry(q, rng.uniform(0, two_pi)))
            nc.ApplyNoise(dep1, q)
        for q in range(qubits - 1):
            nc.Append(QuantumCircuit(qubits).CZ(q, q + 1))
            nc.ApplyNoise(dep2, q)
            nc.ApplyNoise(dep2, q + 1)
        for q in range(qubits):
            nc.ApplyNoise(damp, q)
    return nc
