"""Batched noisy trajectories on the B200.

Mirrors NoisyStateVectorSimulator (src/QuantumMatter.Application/Noise/
NoisyStateVectorSimulator.cs:8-148) over qm_trajectories_run: many trajectories of one
NoisyCircuit run as the states of a device batch and every Kraus selection is taken on the
device from host draws.

Draws.  The reference evolves trajectories one after another from ONE Random: trajectory t
starts where trajectory t-1 stopped drawing.  A trajectory draws once per placement with
p > 0 (none for a certain flip) except that a damping whose jump or stay branch has zero mass
draws nothing, so the offsets are only known after the fact.  The simulator therefore hands
every trajectory the draws it would see if all earlier trajectories drew the maximum, reads
back what each consumed, and re-runs the trajectories after the first one that drew less,
from the corrected offset.  Seeded runs use the seeded System.Random stream
(qm_random_doubles); unseeded runs use a fresh numpy generator, as Random.Shared is unseeded.
"""
from __future__ import annotations

import ctypes as C
from dataclasses import dataclass, field
from typing import Mapping, Sequence

import numpy as np

from . import _lib
from ._lib import check, load
from .backend import FP32, FP64, B200Context
from .circuit import prepare
from .errors import ArgumentError, ArgumentOutOfRangeError
from .noise import NoisyCircuit
from .observables import PauliString, observable_array

DEFAULT_MEMORY_BUDGET_BYTES = 512 * 1024 * 1024  # StateVector.DefaultMemoryBudgetBytes


@dataclass(frozen=True)
class SimulationOptions:
    """SimulationOptions (src/QuantumMatter.Application/SimulationOptions.cs:6-10): the host-array budget."""
    MemoryBudgetBytes: int = DEFAULT_MEMORY_BUDGET_BYTES


@dataclass(frozen=True)
class NoisySimulationResult:
    """NoisySimulationResult (Noise/NoisySimulationResult.cs:4-16)."""
    Shots: int
    Counts: Mapping[str, int]


@dataclass(frozen=True)
class ProbabilityEstimate:
    Probability: float
    StandardError: float


class NoisyProbabilityResult:
    """NoisyProbabilityResult (Noise/NoisySimulationResult.cs:24-58)."""

    def __init__(self, qubits: int, trajectories: int, probabilities: np.ndarray, errors: np.ndarray):
        self.QubitCount = qubits
        self.Trajectories = trajectories
        self._p = probabilities
        self._e = errors

    @property
    def Length(self) -> int:
        return int(self._p.size)

    def Estimate(self, basis_index: int) -> ProbabilityEstimate:
        if not 0 <= basis_index < self.Length:
            raise ArgumentOutOfRangeError("basisIndex")
        return ProbabilityEstimate(float(self._p[basis_index]), float(self._e[basis_index]))

    @property
    def Probabilities(self) -> np.ndarray:
        return self._p.copy()

    @property
    def StandardErrors(self) -> np.ndarray:
        return self._e.copy()


@dataclass
class TrajectoryBatch:
    """Per-trajectory outputs of one batched run."""
    values: np.ndarray | None = None        # [trajectories][terms]
    masses: np.ndarray | None = None
    consumed: np.ndarray | None = None
    branches: np.ndarray | None = None      # [trajectories][placements]
    ambiguous: np.ndarray | None = None
    outcomes: np.ndarray | None = None
    probability_means: np.ndarray | None = None
    probability_stderr: np.ndarray | None = None
    stats: dict = field(default_factory=dict)
    reruns: int = 0

    def mean_values(self) -> np.ndarray:
        """Trajectory average of each term, summed with Neumaier compensation in trajectory order."""
        out = np.empty(self.values.shape[1])
        for k in range(self.values.shape[1]):
            s = 0.0
            c = 0.0
            for v in self.values[:, k]:
                v = float(v)
                t = s + v
                c += (s - t) + v if abs(s) >= abs(v) else (v - t) + s
                s = t
            out[k] = (s + c) / self.values.shape[0]
        return out


def random_doubles(seed: int, count: int, skip: int = 0) -> np.ndarray:
    """NextDouble() values skip .. skip+count-1 of System.Random(seed)."""
    out = np.empty(max(1, count), dtype=np.float64)
    check(load().qm_random_doubles(int(seed), int(skip), int(count), out.ctypes.data_as(_lib.DP)))
    return out[:count]


class _Compiled:
    """A NoisyCircuit packed for the C ABI once."""

    def __init__(self, circuit: NoisyCircuit):
        flat, placements = circuit.Flatten()
        self.qubits = circuit.QubitCount
        self.gates, self.gate_count = prepare(flat)
        self.channels = (_lib.ChannelC * max(1, len(placements)))()
        for i, (ch, target, pos) in enumerate(placements):
            self.channels[i].kind = int(ch.Kind)
            self.channels[i].target = target
            self.channels[i].probability = ch.Probability
            self.channels[i].position = pos
        self.channel_count = len(placements)
        self.max_draws = circuit.MaxDraws()


class B200NoisySimulator:
    """NoisyStateVectorSimulator over batched device trajectories (FP64 or FP32-complex states;
    Kraus renormalisation and all reductions in FP64)."""

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

    # ------------------------------------------------------------------ raw batch
    def RunBatch(self, circuit: NoisyCircuit, draws: np.ndarray, observables: Sequence[PauliString] = (),
                 branches: bool = False, outcomes: bool = False, probabilities: bool = False,
                 masses: bool = True) -> TrajectoryBatch:
        """Trajectory t consumes draws[t, :] in order.  Returns per-trajectory outputs."""
        comp = circuit if isinstance(circuit, _Compiled) else _Compiled(circuit)
        d = np.ascontiguousarray(draws, dtype=np.float64)
        if d.ndim != 2 or d.shape[0] < 1:
            raise ArgumentError("draws must be a [trajectories][draws] array")
        return self._run(comp, d, observables, branches, outcomes, probabilities, masses)

    def _run(self, comp: _Compiled, d: np.ndarray, observables, branches, outcomes, probabilities, masses):
        T, stride = d.shape
        for o in observables:
            if o.QubitCount != comp.qubits:
                raise ArgumentError("Observable and state sizes must match.")
        arr, nterms = observable_array(list(observables))
        res = TrajectoryBatch()
        outs = _lib.TrajectoryOutputs()
        keep = []

        def bind(name, array, ctype):
            keep.append(array)
            setattr(outs, name, array.ctypes.data_as(C.POINTER(ctype)))
            return array

        if nterms:
            res.values = bind("values", np.zeros((T, nterms)), C.c_double)
        if masses:
            res.masses = bind("masses", np.zeros(T), C.c_double)
        res.consumed = bind("consumed", np.zeros(T, dtype=np.int32), C.c_int32)
        res.ambiguous = bind("ambiguous", np.zeros(T, dtype=np.int32), C.c_int32)
        if branches and comp.channel_count:
            res.branches = bind("branches", np.zeros((T, comp.channel_count), dtype=np.int8), C.c_int8)
        if outcomes:
            res.outcomes = bind("outcomes", np.zeros(T, dtype=np.int64), C.c_int64)
        if probabilities:
            res.probability_means = bind("probability_means", np.zeros(1 << comp.qubits), C.c_double)
            if T >= 2:
                res.probability_stderr = bind("probability_stderr", np.zeros(1 << comp.qubits), C.c_double)
        stats = _lib.TrajectoryStats()
        check(load().qm_trajectories_run(self.context.handle, comp.qubits, self.precision, comp.gates, comp.gate_count,
                                         comp.channels, comp.channel_count, T,
                                         d.ctypes.data_as(_lib.DP) if stride else None, stride, arr, nterms,
                                         C.byref(outs), C.byref(stats)))
        res.stats = {f: getattr(stats, f) for f, _ in _lib.TrajectoryStats._fields_}
        return res

    # ------------------------------------------------------------------ reference-order draws
    @staticmethod
    def _stream(seed: int | None, count: int) -> np.ndarray:
        if seed is None:
            return np.random.default_rng().random(count)
        return random_doubles(seed, count)

    def _sequential(self, comp: _Compiled, trajectories: int, stream: np.ndarray, measure: bool,
                    observables: Sequence[PauliString] = (), branches: bool = False) -> TrajectoryBatch:
        """Runs trajectories as if they drew one after another from `stream` (trajectories * D values,
        D = the most one trajectory can draw)."""
        D = comp.max_draws + (1 if measure else 0)
        parts: list[TrajectoryBatch] = []
        start, offset, reruns = 0, 0, 0
        while start < trajectories:
            count = trajectories - start
            rows = stream[offset:offset + count * D].reshape(count, D) if D else np.zeros((count, 0))
            part = self._run(comp, rows, observables, branches, measure, False, True)
            short = np.nonzero(part.consumed != D)[0]
            keep = count if short.size == 0 else int(short[0]) + 1
            parts.append(_slice(part, keep))
            offset += int(part.consumed[:keep].sum())
            start += keep
            if start < trajectories:
                reruns += 1
        res = _concat(parts)
        res.reruns = reruns
        return res

    # ------------------------------------------------------------------ reference API
    def Run(self, circuit: NoisyCircuit, shots: int = 1024, seed: int | None = None) -> NoisySimulationResult:
        """Resets and evolves a fresh trajectory per shot, then measures it once (Run, :36-62)."""
        if shots < 1:
            raise ArgumentOutOfRangeError("shots")
        self._validate(circuit, estimating=False)
        comp = _Compiled(circuit)
        res = self._sequential(comp, shots, self._stream(seed, shots * (comp.max_draws + 1)), measure=True)
        counts: dict[str, int] = {}
        for o in res.outcomes:
            key = format(int(o), "b").zfill(circuit.QubitCount)
            counts[key] = counts.get(key, 0) + 1
        return NoisySimulationResult(shots, dict(sorted(counts.items())))

    def EstimateProbabilities(self, circuit: NoisyCircuit, trajectories: int = 1024,
                              seed: int | None = None) -> NoisyProbabilityResult:
        """Welford mean and standard error of the Born probabilities (EstimateProbabilities, :64-106)."""
        if trajectories < 2:
            raise ArgumentOutOfRangeError("trajectories")
        self._validate(circuit, estimating=True)
        comp = _Compiled(circuit)
        D = comp.max_draws
        stream = self._stream(seed, trajectories * D)
        rows = stream.reshape(trajectories, D)
        res = self._run(comp, rows, (), False, False, True, True)
        if D and np.any(res.consumed != D):
            # the device's Welford sums saw trajectories whose draws were misplaced: resolve the
            # offsets, then accumulate once more over the resolved rows
            pre = self._sequential(comp, trajectories, stream, measure=False)
            starts = np.concatenate([[0], np.cumsum(pre.consumed)[:-1]]).astype(np.int64)
            rows = np.stack([stream[s:s + D] for s in starts])
            res = self._run(comp, rows, (), False, False, True, True)
        return NoisyProbabilityResult(circuit.QubitCount, trajectories, res.probability_means, res.probability_stderr)

    def EstimateObservables(self, circuit: NoisyCircuit, observables: Sequence[PauliString],
                            trajectories: int = 1024, seed: int | None = None,
                            branches: bool = False) -> TrajectoryBatch:
        """Per-trajectory <P> of each observable at the end of every trajectory (StateVector.ExpectationValue
        after EvolveTrajectory), with the trajectory averages available from mean_values()."""
        if trajectories < 1:
            raise ArgumentOutOfRangeError("trajectories")
        self._validate(circuit, estimating=False)
        comp = _Compiled(circuit)
        return self._sequential(comp, trajectories, self._stream(seed, trajectories * comp.max_draws), measure=False,
                                observables=observables, branches=branches)

    def _validate(self, circuit: NoisyCircuit, estimating: bool) -> None:
        if circuit is None:
            raise ArgumentError("circuit")
        required = (32 if estimating else 16) << circuit.QubitCount
        if required > self.options.MemoryBudgetBytes:
            raise ArgumentOutOfRangeError(
                f"Execution requires {required} bytes; the budget is {self.options.MemoryBudgetBytes} bytes.")


def _slice(b: TrajectoryBatch, k: int) -> TrajectoryBatch:
    out = TrajectoryBatch(stats=b.stats)
    for name in ("values", "masses", "consumed", "branches", "ambiguous", "outcomes"):
        v = getattr(b, name)
        setattr(out, name, None if v is None else v[:k])
    return out


def _concat(parts: list[TrajectoryBatch]) -> TrajectoryBatch:
    out = TrajectoryBatch(stats=parts[-1].stats)
    for name in ("values", "masses", "consumed", "branches", "ambiguous", "outcomes"):
        vs = [getattr(p, name) for p in parts]
        setattr(out, name, None if vs[0] is None else np.concatenate(vs))
    return out
