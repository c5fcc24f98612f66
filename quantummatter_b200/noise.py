"""Noise IR mirroring src/QuantumMatter.Core/Noise/NoiseChannel.cs and NoisyCircuit.cs."""
from __future__ import annotations

import math
from dataclasses import dataclass
from enum import IntEnum

from .circuit import QuantumCircuit
from .errors import ArgumentError, ArgumentOutOfRangeError


class NoiseKind(IntEnum):
    """NoiseChannel.cs:4-14."""
    BitFlip = 0
    PhaseFlip = 1
    Depolarizing = 2
    AmplitudeDamping = 3


@dataclass(frozen=True)
class NoiseChannel:
    """Single-qubit channel with a finite parameter in [0, 1] (NoiseChannel.cs:17-44)."""
    Kind: NoiseKind
    Probability: float

    def __post_init__(self):
        p = self.Probability
        if not isinstance(p, (int, float)) or not math.isfinite(p) or p < 0 or p > 1:
            raise ArgumentOutOfRangeError("Channel probability must be finite and in [0,1].")
        object.__setattr__(self, "Kind", NoiseKind(int(self.Kind)))
        object.__setattr__(self, "Probability", float(p))

    @staticmethod
    def BitFlip(p: float) -> "NoiseChannel":
        return NoiseChannel(NoiseKind.BitFlip, p)

    @staticmethod
    def PhaseFlip(p: float) -> "NoiseChannel":
        return NoiseChannel(NoiseKind.PhaseFlip, p)

    @staticmethod
    def Depolarizing(p: float) -> "NoiseChannel":
        return NoiseChannel(NoiseKind.Depolarizing, p)

    @staticmethod
    def AmplitudeDamping(gamma: float) -> "NoiseChannel":
        return NoiseChannel(NoiseKind.AmplitudeDamping, gamma)


@dataclass(frozen=True)
class NoisyStep:
    Circuit: QuantumCircuit | None
    Channel: NoiseChannel | None
    Target: int


class NoisyCircuit:
    """Ordered snapshots of unitary segments and channel placements (NoisyCircuit.cs:7-65)."""

    def __init__(self, qubits: int):
        if qubits < 1 or qubits > 30:
            raise ArgumentOutOfRangeError("qubits")
        self.QubitCount = qubits
        self._steps: list[NoisyStep] = []

    @property
    def StepCount(self) -> int:
        return len(self._steps)

    @property
    def Steps(self) -> tuple[NoisyStep, ...]:
        return tuple(self._steps)

    def Append(self, circuit: QuantumCircuit) -> "NoisyCircuit":
        if circuit is None:
            raise ArgumentError("circuit")
        if circuit.QubitCount != self.QubitCount:
            raise ArgumentError("Circuit sizes must match.")
        self._steps.append(NoisyStep(circuit.Copy(), None, -1))
        return self

    def ApplyNoise(self, channel: NoiseChannel, target: int) -> "NoisyCircuit":
        if channel is None:
            raise ArgumentError("channel")
        if not isinstance(target, int) or target < 0 or target >= self.QubitCount:
            raise ArgumentOutOfRangeError("target")
        self._steps.append(NoisyStep(None, channel, target))
        return self

    def Flatten(self) -> tuple[QuantumCircuit, list[tuple[NoiseChannel, int, int]]]:
        """All unitary segments as one circuit, plus (channel, target, position) placements, where
        a placement acts after the first `position` operations (the order NoisyCircuit.Execute
        applies them in)."""
        flat = QuantumCircuit(self.QubitCount)
        placements: list[tuple[NoiseChannel, int, int]] = []
        count = 0
        for step in self._steps:
            if step.Circuit is not None:
                for op in step.Circuit.Operations:
                    flat.AppendValidated(op)
                    count += 1
            else:
                placements.append((step.Channel, step.Target, count))
        return flat, placements

    def MaxDraws(self) -> int:
        """Draws one trajectory can consume: every placement with p > 0 except certain flips."""
        n = 0
        for step in self._steps:
            ch = step.Channel
            if ch is None or ch.Probability == 0:
                continue
            if ch.Kind in (NoiseKind.BitFlip, NoiseKind.PhaseFlip) and ch.Probability == 1:
                continue
            n += 1
        return n
