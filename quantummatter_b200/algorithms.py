"""Algorithm circuit builders: QFT, Grover search and Deutsch-Jozsa.

These follow the reference's decompositions gate for gate (src/QuantumMatter.Application/
Algorithms/*.cs), so a circuit built here is the circuit the reference builds and runs; what
changes is where it runs.  Their diagonal-heavy parts (the QFT's controlled-phase chains, the
oracles' CZ and Toffoli ladders) are where the fusion planner's diagonal groups pay: a chain of
commuting phases on any qubits becomes one phase per register in a pass.
"""
from __future__ import annotations

import math
from typing import Sequence

from .circuit import QuantumCircuit, SingleQubitUnitary
from .errors import ArgumentError, ArgumentOutOfRangeError

MAXIMUM_INPUT_QUBITS = 16          # BasisStatePhaseOracle.MaximumInputQubits
MAXIMUM_CIRCUIT_OPERATIONS = 1_000_000


class QuantumFourierTransform:
    """F[y, x] = exp(2 pi i x y / 2^n) / sqrt(2^n), including the bit reversal
    (QuantumFourierTransform.cs:7-96)."""

    @staticmethod
    def CreateCircuit(qubits: int, inverse: bool = False) -> QuantumCircuit:
        return QuantumFourierTransform.Append(QuantumCircuit(qubits), inverse=inverse)

    @staticmethod
    def Append(circuit: QuantumCircuit, qubits: Sequence[int] | None = None, inverse: bool = False) -> QuantumCircuit:
        if circuit is None:
            raise ArgumentError("circuit")
        register = list(range(circuit.QubitCount)) if qubits is None else [int(q) for q in qubits]
        if len(register) < 1 or len(register) > circuit.QubitCount:
            raise ArgumentError("Select a nonempty subset of the circuit's qubits.")
        if len(set(register)) != len(register) or any(not 0 <= q < circuit.QubitCount for q in register):
            raise ArgumentError("Selected qubits must be distinct and in range.")
        n = len(register)
        if inverse:
            QuantumFourierTransform._reverse(circuit, register)
            for target in range(n):
                for control in range(target):
                    circuit.CPhase(register[control], register[target], -math.ldexp(math.pi, control - target))
                circuit.H(register[target])
        else:
            for target in range(n - 1, -1, -1):
                circuit.H(register[target])
                for control in range(target - 1, -1, -1):
                    circuit.CPhase(register[control], register[target], math.ldexp(math.pi, control - target))
            QuantumFourierTransform._reverse(circuit, register)
        return circuit

    @staticmethod
    def _reverse(circuit: QuantumCircuit, register: list[int]) -> None:
        for first in range(len(register) // 2):
            circuit.Swap(register[first], register[len(register) - first - 1])


class _PhaseOracle:
    """Phase flip of one basis state of the input bits, with initially-zero scratch bits above
    them carrying a Toffoli ladder (BasisStatePhaseOracle.cs:7-80)."""

    @staticmethod
    def required_qubits(input_qubits: int) -> int:
        if not 1 <= input_qubits <= MAXIMUM_INPUT_QUBITS:
            raise ArgumentOutOfRangeError("Phase-oracle algorithms support 1 through 16 input qubits.")
        return input_qubits + max(0, input_qubits - 2)

    @staticmethod
    def operation_count(input_qubits: int, basis_index: int) -> int:
        zeros = input_qubits - bin(basis_index).count("1")
        return 2 * zeros + (1 if input_qubits <= 2 else 2 * (input_qubits - 2) + 1)

    @staticmethod
    def global_negation(circuit: QuantumCircuit) -> None:
        circuit.U(0, SingleQubitUnitary.Create(-1, 0, 0, -1))

    @staticmethod
    def _flip_zero_bits(circuit: QuantumCircuit, input_qubits: int, basis_index: int) -> None:
        for q in range(input_qubits):
            if not (basis_index >> q) & 1:
                circuit.X(q)

    @staticmethod
    def append(circuit: QuantumCircuit, input_qubits: int, basis_index: int) -> None:
        _PhaseOracle._flip_zero_bits(circuit, input_qubits, basis_index)
        if input_qubits == 1:
            circuit.Z(0)
        elif input_qubits == 2:
            circuit.CZ(0, 1)
        else:
            circuit.Toffoli(0, 1, input_qubits)
            for i in range(2, input_qubits - 1):
                circuit.Toffoli(input_qubits + i - 2, i, input_qubits + i - 1)
            circuit.CZ(2 * input_qubits - 3, input_qubits - 1)
            for i in range(input_qubits - 2, 1, -1):
                circuit.Toffoli(input_qubits + i - 2, i, input_qubits + i - 1)
            circuit.Toffoli(0, 1, input_qubits)
        _PhaseOracle._flip_zero_bits(circuit, input_qubits, basis_index)


class GroverSearch:
    """Single-solution amplitude amplification with an explicit marked index (GroverSearch.cs:6-66)."""
    MaximumInputQubits = MAXIMUM_INPUT_QUBITS
    MaximumCircuitOperations = MAXIMUM_CIRCUIT_OPERATIONS

    @staticmethod
    def RecommendedIterations(inputQubits: int) -> int:
        _PhaseOracle.required_qubits(inputQubits)
        theta = math.asin(1 / math.sqrt(1 << inputQubits))
        # Math.Round rounds half to even, as Python's round does
        return max(0, int(round(math.pi / (4 * theta) - 0.5)))

    @staticmethod
    def CreateCircuit(inputQubits: int, markedBasisIndex: int, iterations: int | None = None) -> QuantumCircuit:
        total = _PhaseOracle.required_qubits(inputQubits)
        if not 0 <= markedBasisIndex < (1 << inputQubits):
            raise ArgumentOutOfRangeError("markedBasisIndex")
        rounds = GroverSearch.RecommendedIterations(inputQubits) if iterations is None else iterations
        if rounds < 0:
            raise ArgumentOutOfRangeError("iterations")
        per_round = (_PhaseOracle.operation_count(inputQubits, markedBasisIndex) + 2 * inputQubits
                     + _PhaseOracle.operation_count(inputQubits, 0) + 1)
        if inputQubits + rounds * per_round > MAXIMUM_CIRCUIT_OPERATIONS:
            raise ArgumentOutOfRangeError("Synthesized circuit exceeds the operation limit.")
        c = QuantumCircuit(total)
        for q in range(inputQubits):
            c.H(q)
        for _ in range(rounds):
            _PhaseOracle.append(c, inputQubits, markedBasisIndex)
            for q in range(inputQubits):
                c.H(q)
            _PhaseOracle.append(c, inputQubits, 0)
            for q in range(inputQubits):
                c.H(q)
            _PhaseOracle.global_negation(c)  # the marked-zero reflection is I - 2|s><s|
        return c


class DeutschJozsa:
    """Deutsch-Jozsa with a phase oracle synthesised from a constant or balanced truth table
    (DeutschJozsa.cs:7-90)."""
    MaximumInputQubits = MAXIMUM_INPUT_QUBITS
    MaximumCircuitOperations = MAXIMUM_CIRCUIT_OPERATIONS

    @staticmethod
    def CreateCircuit(truthTable: Sequence[bool]) -> QuantumCircuit:
        if truthTable is None:
            raise ArgumentError("truthTable")
        length = len(truthTable)
        if length < 2 or length > (1 << MAXIMUM_INPUT_QUBITS) or length & (length - 1):
            raise ArgumentError("Provide a power-of-two table for 1 through 16 input qubits.")
        n = length.bit_length() - 1
        total = _PhaseOracle.required_qubits(n)
        values = [bool(v) for v in truthTable]
        ones = sum(values)
        oracle_ops = sum(_PhaseOracle.operation_count(n, i) for i, v in enumerate(values) if v)
        if ones not in (0, length, length // 2):
            raise ArgumentError("The truth table must be constant or balanced.")
        if 2 * n + (1 if ones == length else oracle_ops) > MAXIMUM_CIRCUIT_OPERATIONS:
            raise ArgumentError("Synthesized circuit exceeds the operation limit.")
        c = QuantumCircuit(total)
        for q in range(n):
            c.H(q)
        if ones == length:
            _PhaseOracle.global_negation(c)
        else:
            for i, v in enumerate(values):
                if v:
                    _PhaseOracle.append(c, n, i)
        for q in range(n):
            c.H(q)
        return c
