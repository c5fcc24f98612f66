"""Dynamic circuits with the state resident on the device.

DynamicCircuit mirrors src/QuantumMatter.Core/Dynamic/DynamicCircuit.cs: unitary segments,
segments conditioned on the classical register, measurements of ordered qubit subsets into
classical bits, and single-qubit resets (a projective measurement and a conditional X).

The reference's DynamicStateVectorSimulator (src/QuantumMatter.Application/Dynamic/
DynamicStateVectorSimulator.cs) hands every executed segment to the backend port, which with a
GPU backend means a copy of the whole state to the device and back per segment, and measures on
the host.  Here the state stays on the device for the whole trajectory: segments run as fused
plans (made once per segment and reused by every shot), measurements draw and project on the
device (qm_measure, StateVector.Observations.cs:38-97), and only the measured bits come back to
drive the classical control on the host.  Each measurement or reset consumes one draw, in
program order, from the seeded System.Random stream (or a fresh generator without a seed).
"""
from __future__ import annotations

from dataclasses import dataclass
from typing import Mapping, Sequence

import numpy as np

from .backend import FP32, FP64, B200Context, DeviceState, Plan
from .circuit import QuantumCircuit
from .errors import ArgumentError, ArgumentOutOfRangeError
from .noise import NoiseChannel, NoisyCircuit
from .trajectories import SimulationOptions, random_doubles


@dataclass(frozen=True)
class UnitaryStep:
    Circuit: QuantumCircuit
    Mask: int
    Value: int


@dataclass(frozen=True)
class MeasurementStep:
    Qubits: tuple[int, ...]
    ClassicalBits: tuple[int, ...]
    WriteMask: int


@dataclass(frozen=True)
class ResetStep:
    Qubit: int


@dataclass(frozen=True)
class NoiseStep:
    Channel: NoiseChannel
    Target: int


class SeededStream:
    """NextDouble() of System.Random(seed) in order (qm_random_doubles, fetched in chunks), or
    fresh uniform draws without a seed (Random.Shared's role)."""

    def __init__(self, seed: int | None, chunk: int = 4096):
        self._seed = seed
        self._rng = np.random.default_rng() if seed is None else None
        self._chunk = chunk
        self._buf = np.zeros(0)
        self._base = 0
        self._pos = 0

    def NextDouble(self) -> float:
        if self._rng is not None:
            return float(self._rng.random())
        i = self._pos - self._base
        if i >= self._buf.size:
            self._base = self._pos
            self._buf = random_doubles(self._seed, self._chunk, skip=self._pos)
            i = 0
        self._pos += 1
        return float(self._buf[i])


class _ArrayDraws:
    """Draws handed out in order from an array (a fixed number per shot)."""

    def __init__(self, draws: np.ndarray):
        self._draws = draws
        self._k = 0

    def NextDouble(self) -> float:
        v = float(self._draws[self._k])
        self._k += 1
        return v


def _indices(values: Sequence[int], count: int, name: str) -> int:
    mask = 0
    for v in values:
        if not isinstance(v, (int, np.integer)) or not 0 <= int(v) < count:
            raise ArgumentOutOfRangeError(name)
        bit = 1 << int(v)
        if mask & bit:
            raise ArgumentError("Indices must be distinct.")
        mask |= bit
    return mask


class DynamicCircuit:
    """A finite sequence of unitary snapshots, measurements, classical conditions and resets
    (DynamicCircuit.cs:4-112).  Each execution starts with a zero classical register."""

    def __init__(self, qubits: int, classicalBits: int):
        if not isinstance(qubits, int) or not 1 <= qubits <= 30:
            raise ArgumentOutOfRangeError("qubits")
        if not isinstance(classicalBits, int) or not 1 <= classicalBits <= 30:
            raise ArgumentOutOfRangeError("classicalBits")
        self.QubitCount = qubits
        self.ClassicalBitCount = classicalBits
        self._steps: list = []

    @property
    def StepCount(self) -> int:
        return len(self._steps)

    @property
    def Steps(self) -> tuple:
        return tuple(self._steps)

    def _circuit(self, circuit: QuantumCircuit) -> QuantumCircuit:
        if circuit is None:
            raise ArgumentError("circuit")
        if circuit.QubitCount != self.QubitCount:
            raise ArgumentError("Circuit sizes must match.")
        return circuit.Copy()

    def Append(self, circuit: QuantumCircuit) -> "DynamicCircuit":
        self._steps.append(UnitaryStep(self._circuit(circuit), 0, 0))
        return self

    def If(self, classicalMask: int, expectedValue: int, circuit: QuantumCircuit) -> "DynamicCircuit":
        c = self._circuit(circuit)
        register = (1 << self.ClassicalBitCount) - 1
        if classicalMask <= 0 or classicalMask & ~register:
            raise ArgumentOutOfRangeError("classicalMask")
        if expectedValue < 0 or expectedValue & ~classicalMask:
            raise ArgumentOutOfRangeError("expectedValue")
        self._steps.append(UnitaryStep(c, classicalMask, expectedValue))
        return self

    def Measure(self, qubits: Sequence[int], classicalBits: Sequence[int]) -> "DynamicCircuit":
        qubits, classicalBits = list(qubits), list(classicalBits)
        if len(qubits) < 1 or len(qubits) != len(classicalBits) or len(qubits) > self.QubitCount:
            raise ArgumentError("Measurement requires equally sized nonempty selections.")
        _indices(qubits, self.QubitCount, "qubits")
        write = _indices(classicalBits, self.ClassicalBitCount, "classicalBits")
        self._steps.append(MeasurementStep(tuple(int(q) for q in qubits), tuple(int(b) for b in classicalBits), write))
        return self

    def Reset(self, qubit: int) -> "DynamicCircuit":
        if not isinstance(qubit, int) or not 0 <= qubit < self.QubitCount:
            raise ArgumentOutOfRangeError("qubit")
        self._steps.append(ResetStep(qubit))
        return self

    def DrawsPerExecution(self) -> int:
        return sum(1 for s in self._steps if not isinstance(s, UnitaryStep))


@dataclass(frozen=True)
class DynamicTrajectoryResult:
    """One conditional trajectory (DynamicTrajectoryResult): final state and classical register."""
    FinalState: np.ndarray
    ClassicalBitCount: int
    ClassicalRegister: int
    Ambiguous: int = 0


@dataclass(frozen=True)
class DynamicSimulationResult:
    """DynamicSimulationResult.cs:24-39: final classical-register counts over the shots."""
    ClassicalBitCount: int
    Shots: int
    Counts: Mapping[str, int]
    Ambiguous: int = 0


class B200DynamicSimulator:
    """DynamicStateVectorSimulator with the state resident on the device."""

    def __init__(self, context: B200Context, options: SimulationOptions | None = None, precision: int = FP64):
        if context is None:
            raise ArgumentError("context")
        self.context = context
        self.options = options or SimulationOptions()
        if self.options.MemoryBudgetBytes <= 0:
            raise ArgumentOutOfRangeError("MemoryBudgetBytes")
        if precision not in (FP64, FP32):
            raise ArgumentOutOfRangeError("precision")
        self.precision = precision

    def _validate(self, circuit: DynamicCircuit) -> None:
        if circuit is None:
            raise ArgumentError("circuit")
        required = 16 << circuit.QubitCount
        if required > self.options.MemoryBudgetBytes:
            raise ArgumentOutOfRangeError(
                f"Execution requires {required} bytes; the budget is {self.options.MemoryBudgetBytes} bytes.")

    @staticmethod
    def _draws(seed: int | None, count: int) -> np.ndarray:
        if count == 0:
            return np.zeros(0)
        return random_doubles(seed, count) if seed is not None else np.random.default_rng().random(count)

    @staticmethod
    def _execute(state: DeviceState, steps, random, plans: dict | None) -> tuple[int, int]:
        """DynamicCircuit.Execute (DynamicCircuit.cs:77-112) on a resident state, with the noise
        placements of a NoisyDynamicCircuit (NoisyDynamicCircuit.cs:80-100) applied where they
        stand.  `random` (NextDouble) gives every measurement, reset and channel its draws in
        program order."""
        classical, ambiguous = 0, 0
        for i, step in enumerate(steps):
            if isinstance(step, UnitaryStep):
                if (classical & step.Mask) == step.Value:
                    if plans is not None:
                        plans[i].execute(state)
                    else:
                        state.Evolve(step.Circuit)
            elif isinstance(step, MeasurementStep):
                outcome, amb = state.Measure(step.Qubits, random.NextDouble())
                ambiguous += int(amb)
                written = 0
                for bit, cb in enumerate(step.ClassicalBits):
                    written |= ((outcome >> bit) & 1) << cb
                classical = (classical & ~step.WriteMask) | written
            elif isinstance(step, ResetStep):
                outcome, amb = state.Measure([step.Qubit], random.NextDouble())
                ambiguous += int(amb)
                if outcome != 0:
                    state.ApplyPauli(step.Qubit, 1)  # the reset's X correction
            else:
                state.ApplyNoise(step.Channel, step.Target, random)
        return classical, ambiguous

    def SimulateTrajectory(self, circuit: DynamicCircuit, seed: int | None = None) -> DynamicTrajectoryResult:
        """One conditional trajectory without any implicit terminal measurement."""
        self._validate(circuit)
        draws = self._draws(seed, circuit.DrawsPerExecution())
        with DeviceState(self.context, circuit.QubitCount, self.precision) as st:
            classical, amb = self._execute(st, circuit.Steps, _ArrayDraws(draws), None)
            state = st.Download()
        return DynamicTrajectoryResult(state, circuit.ClassicalBitCount, classical, amb)

    def Run(self, circuit: DynamicCircuit, shots: int = 1024, seed: int | None = None) -> DynamicSimulationResult:
        """Re-executes every instruction for each shot from |0...0> and counts the final classical register."""
        if shots < 1:
            raise ArgumentOutOfRangeError("shots")
        self._validate(circuit)
        D = circuit.DrawsPerExecution()
        draws = self._draws(seed, shots * D)
        plans = {i: Plan(self.context, s.Circuit, self.precision)
                 for i, s in enumerate(circuit.Steps) if isinstance(s, UnitaryStep)}
        counts: dict[int, int] = {}
        ambiguous = 0
        try:
            with DeviceState(self.context, circuit.QubitCount, self.precision) as st:
                for shot in range(shots):
                    st.Reset()
                    classical, amb = self._execute(st, circuit.Steps, _ArrayDraws(draws[shot * D:(shot + 1) * D]), plans)
                    ambiguous += amb
                    counts[classical] = counts.get(classical, 0) + 1
        finally:
            for p in plans.values():
                p.Dispose()
        labelled = {format(k, "b").zfill(circuit.ClassicalBitCount): v for k, v in counts.items()}
        return DynamicSimulationResult(circuit.ClassicalBitCount, shots, dict(sorted(labelled.items())), ambiguous)


class NoisyDynamicCircuit:
    """A dynamic program with explicit single-qubit noise placements between instructions
    (src/QuantumMatter.Core/Dynamic/NoisyDynamicCircuit.cs:7-103).  Each trajectory starts with a
    zero classical register; placements are unconditional and write no classical bits."""

    def __init__(self, qubits: int, classicalBits: int):
        DynamicCircuit(qubits, classicalBits)  # the same size validation
        self.QubitCount = qubits
        self.ClassicalBitCount = classicalBits
        self._steps: list = []

    @property
    def StepCount(self) -> int:
        return len(self._steps)

    @property
    def Steps(self) -> tuple:
        return tuple(self._steps)

    def _take(self, build) -> "NoisyDynamicCircuit":
        d = DynamicCircuit(self.QubitCount, self.ClassicalBitCount)
        build(d)  # validates; a rejected instruction changes nothing
        self._steps.extend(d.Steps)
        return self

    def Append(self, circuit: QuantumCircuit) -> "NoisyDynamicCircuit":
        return self._take(lambda d: d.Append(circuit))

    def If(self, classicalMask: int, expectedValue: int, circuit: QuantumCircuit) -> "NoisyDynamicCircuit":
        return self._take(lambda d: d.If(classicalMask, expectedValue, circuit))

    def Measure(self, qubits: Sequence[int], classicalBits: Sequence[int]) -> "NoisyDynamicCircuit":
        return self._take(lambda d: d.Measure(qubits, classicalBits))

    def Reset(self, qubit: int) -> "NoisyDynamicCircuit":
        return self._take(lambda d: d.Reset(qubit))

    def ApplyNoise(self, channel: NoiseChannel, target: int) -> "NoisyDynamicCircuit":
        NoisyCircuit(self.QubitCount).ApplyNoise(channel, target)  # validation
        self._steps.append(NoiseStep(channel, target))
        return self


class B200NoisyDynamicSimulator:
    """NoisyDynamicStateVectorSimulator (src/QuantumMatter.Application/Dynamic/
    NoisyDynamicStateVectorSimulator.cs) with the state resident on the device: segments run as
    fused plans made once per segment, measurements and resets draw and project on the device,
    channels pick their branch from the same draws as the reference (qm_state_noise_apply).  One
    seeded System.Random stream serves every shot in order."""

    def __init__(self, context: B200Context, options: SimulationOptions | None = None, precision: int = FP64):
        self._sim = B200DynamicSimulator(context, options, precision)

    def SimulateTrajectory(self, circuit: NoisyDynamicCircuit, seed: int | None = None) -> DynamicTrajectoryResult:
        """One conditional state and its classical register, without an implicit readout."""
        self._sim._validate(circuit)
        random = SeededStream(seed)
        with DeviceState(self._sim.context, circuit.QubitCount, self._sim.precision) as st:
            classical, amb = B200DynamicSimulator._execute(st, circuit.Steps, random, None)
            state = st.Download()
        return DynamicTrajectoryResult(state, circuit.ClassicalBitCount, classical, amb)

    def Run(self, circuit: NoisyDynamicCircuit, shots: int = 1024, seed: int | None = None) -> DynamicSimulationResult:
        """Re-executes every instruction for each shot from |0...0> and counts the final classical register."""
        if shots < 1:
            raise ArgumentOutOfRangeError("shots")
        self._sim._validate(circuit)
        random = SeededStream(seed)
        steps = circuit.Steps
        plans = {i: Plan(self._sim.context, s.Circuit, self._sim.precision)
                 for i, s in enumerate(steps) if isinstance(s, UnitaryStep)}
        counts: dict[int, int] = {}
        ambiguous = 0
        try:
            with DeviceState(self._sim.context, circuit.QubitCount, self._sim.precision) as st:
                for _ in range(shots):
                    st.Reset()
                    classical, amb = B200DynamicSimulator._execute(st, steps, random, plans)
                    ambiguous += amb
                    counts[classical] = counts.get(classical, 0) + 1
        finally:
            for p in plans.values():
                p.Dispose()
        labelled = {format(k, "b").zfill(circuit.ClassicalBitCount): v for k, v in counts.items()}
        return DynamicSimulationResult(circuit.ClassicalBitCount, shots, dict(sorted(labelled.items())), ambiguous)
