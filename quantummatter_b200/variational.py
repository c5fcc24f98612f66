"""Variational layer on libqmb200, mirroring QuantumMatter's Variational namespace.

ParameterizedCircuit follows src/QuantumMatter.Core/Variational/ParameterizedCircuit.cs:5-99;
B200VariationalEnergyEvaluator has the Evaluate / EvaluateWithGradient signatures of
src/QuantumMatter.Application/Variational/VariationalEnergyEvaluator.cs:23-86 and adds a batch
form; VqeSolver is a twin of src/QuantumMatter.Application/Variational/VqeSolver.cs:27-117 that
runs its energies and gradients through the B200 evaluator.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from fractions import Fraction
from enum import IntEnum
from typing import Sequence

import numpy as np

from . import _lib
from ._lib import check, load
from .backend import FP64, B200Context
from .circuit import GateKind, GateOperation, QuantumCircuit
from .errors import ArgumentError, ArgumentOutOfRangeError
from .observables import PauliHamiltonian, terms_array


def _fma(a: float, b: float, c: float) -> float:
    """a * b + c with one rounding (Math.FusedMultiplyAdd, VqeSolver.cs:76)."""
    if not (math.isfinite(a) and math.isfinite(b) and math.isfinite(c)):
        return a * b + c
    return float(Fraction(a) * Fraction(b) + Fraction(c))


@dataclass(frozen=True)
class TemplateOperation:
    Operation: GateOperation
    ParameterIndex: int


class ParameterizedCircuit:
    """Constant segments plus parameter-indexed uncontrolled Rx/Ry/Rz rotations."""

    def __init__(self, qubits: int, parameterCount: int):
        if qubits < 1 or qubits > 30:
            raise ArgumentOutOfRangeError("qubits")
        if parameterCount < 0:
            raise ArgumentOutOfRangeError("parameterCount")
        self.QubitCount = qubits
        self.ParameterCount = parameterCount
        self._ops: list[TemplateOperation] = []
        self._rotations: list[int] = []

    @property
    def OperationCount(self) -> int:
        return len(self._ops)

    @property
    def RotationParameterIndices(self) -> tuple[int, ...]:
        return tuple(self._rotations)

    @property
    def Operations(self) -> tuple[TemplateOperation, ...]:
        return tuple(self._ops)

    def Append(self, circuit: QuantumCircuit) -> "ParameterizedCircuit":
        if circuit is None:
            raise ArgumentError("circuit")
        if circuit.QubitCount != self.QubitCount:
            raise ArgumentError("Circuit sizes must match.")
        self._ops.extend(TemplateOperation(op, -1) for op in circuit.Operations)
        return self

    def _rotation(self, kind: GateKind, target: int, parameterIndex: int) -> "ParameterizedCircuit":
        if not (0 <= target < self.QubitCount):
            raise ArgumentOutOfRangeError("target")
        if not (0 <= parameterIndex < self.ParameterCount):
            raise ArgumentOutOfRangeError("parameterIndex")
        self._ops.append(TemplateOperation(GateOperation(kind, target), parameterIndex))
        self._rotations.append(parameterIndex)
        return self

    def Rx(self, target: int, parameterIndex: int): return self._rotation(GateKind.Rx, target, parameterIndex)
    def Ry(self, target: int, parameterIndex: int): return self._rotation(GateKind.Ry, target, parameterIndex)
    def Rz(self, target: int, parameterIndex: int): return self._rotation(GateKind.Rz, target, parameterIndex)

    def _check(self, parameters: Sequence[float]) -> None:
        if len(parameters) != self.ParameterCount:
            raise ArgumentError("Binding size must match ParameterCount.")
        for p in parameters:
            if not math.isfinite(p):
                raise ArgumentOutOfRangeError("Parameters must be finite.")

    def Bind(self, parameters: Sequence[float]) -> QuantumCircuit:
        return self._bind(parameters, -1, 0.0)

    def BindWithRotationShift(self, parameters: Sequence[float], rotationIndex: int, shift: float) -> QuantumCircuit:
        if not (0 <= rotationIndex < len(self._rotations)):
            raise ArgumentOutOfRangeError("rotationIndex")
        if not math.isfinite(shift):
            raise ArgumentOutOfRangeError("shift")
        return self._bind(parameters, rotationIndex, shift)

    def _bind(self, parameters, shifted: int, shift: float) -> QuantumCircuit:
        """The shift is an extra same-axis rotation after one occurrence (ParameterizedCircuit.cs:87-88)."""
        self._check(parameters)
        out = QuantumCircuit(self.QubitCount)
        r = 0
        for t in self._ops:
            if t.ParameterIndex >= 0:
                op = t.Operation
                out.AppendValidated(GateOperation(op.Kind, op.Target, -1, float(parameters[t.ParameterIndex])))
                if r == shifted:
                    out.AppendValidated(GateOperation(op.Kind, op.Target, -1, float(shift)))
                r += 1
            else:
                out.AppendValidated(t.Operation)
        return out

    def template_array(self):
        """Packs the template into a ctypes qm_template_op array."""
        arr = (_lib.TemplateOp * max(1, len(self._ops)))()
        for i, t in enumerate(self._ops):
            o, r = t.Operation, arr[i]
            r.operation.kind, r.operation.target = int(o.Kind), o.Target
            r.operation.control, r.operation.second_control = o.Control, o.SecondControl
            r.operation.angle = o.Angle
            if o.Unitary is not None:
                u = o.Unitary
                for j, v in enumerate((u.M00.real, u.M00.imag, u.M01.real, u.M01.imag, u.M10.real, u.M10.imag,
                                       u.M11.real, u.M11.imag)):
                    r.operation.unitary[j] = v
            r.parameter = t.ParameterIndex
        return arr, len(self._ops)


@dataclass(frozen=True)
class VariationalEnergyResult:
    Energy: float
    Gradient: tuple[float, ...]


@dataclass(frozen=True)
class BatchEvaluation:
    Energies: np.ndarray
    Gradients: np.ndarray | None
    Circuits: int
    Waves: int
    BatchStates: int
    PassesPerCircuit: int
    TilePasses: int
    DeviceSeconds: float
    WallSeconds: float


class B200VariationalEnergyEvaluator:
    """Energies and parameter-shift gradients with every circuit resident on the device."""

    def __init__(self, context: B200Context, precision: int = FP64):
        if context is None:
            raise ArgumentError("context")
        self.context = context
        self.precision = precision

    def _validate(self, circuit: ParameterizedCircuit, hamiltonian: PauliHamiltonian) -> None:
        if circuit is None or hamiltonian is None:
            raise ArgumentError("circuit and hamiltonian are required")
        if circuit.QubitCount != hamiltonian.QubitCount:
            raise ArgumentError("Circuit and Hamiltonian sizes must match.")

    def EvaluateBatch(self, circuit: ParameterizedCircuit, hamiltonian: PauliHamiltonian,
                      parameters: np.ndarray, withGradient: bool = True,
                      coefficients: np.ndarray | None = None) -> BatchEvaluation:
        """Energies (and gradients) of every parameter vector.  `coefficients` ([vectors][terms])
        replaces the Hamiltonian's own coefficients per vector (same Pauli strings)."""
        self._validate(circuit, hamiltonian)
        params = np.ascontiguousarray(parameters, dtype=np.float64)
        if params.ndim == 1:
            params = params.reshape(1, -1)
        vectors, pcount = params.shape
        if pcount != circuit.ParameterCount:
            raise ArgumentError("Binding size must match ParameterCount.")
        ops, nops = circuit.template_array()
        terms, nterms = terms_array(hamiltonian.Terms)
        energies = np.zeros(vectors, dtype=np.float64)
        grads = np.zeros((vectors, max(1, pcount)), dtype=np.float64)
        stats = _lib.VqeStats()
        if coefficients is None:
            check(load().qm_vqe_evaluate(self.context.handle, circuit.QubitCount, self.precision, ops, nops, pcount,
                                         terms, nterms, params.ctypes.data_as(_lib.DP), vectors,
                                         1 if withGradient else 0, energies.ctypes.data_as(_lib.DP),
                                         grads.ctypes.data_as(_lib.DP), C.byref(stats)))
        else:
            coef = np.ascontiguousarray(coefficients, dtype=np.float64)
            if coef.shape != (vectors, nterms):
                raise ArgumentError("coefficients must be a [vectors][terms] array")
            check(load().qm_vqe_evaluate_coefficients(self.context.handle, circuit.QubitCount, self.precision, ops,
                                                      nops, pcount, terms, nterms, coef.ctypes.data_as(_lib.DP),
                                                      params.ctypes.data_as(_lib.DP), vectors,
                                                      1 if withGradient else 0, energies.ctypes.data_as(_lib.DP),
                                                      grads.ctypes.data_as(_lib.DP), C.byref(stats)))
        return BatchEvaluation(energies, grads[:, :pcount] if withGradient else None, stats.circuits, stats.waves,
                               stats.batch_states, stats.passes_per_circuit, stats.tile_passes, stats.device_seconds,
                               stats.wall_seconds)

    def EvaluateMixed(self, problems: Sequence[tuple], withGradient: bool = True) -> tuple[list, BatchEvaluation]:
        """Several (circuit, hamiltonian, parameters) problems of different sizes in one call
        (qm_vqe_evaluate_mixed): each round of waves covers every size, as one CUDA graph launch
        once the rounds are full.  Returns each problem's (energies, gradients) and the totals."""
        keep, recs, outs = [], (_lib.VqeProblem * len(problems))(), []
        for i, (circuit, hamiltonian, parameters) in enumerate(problems):
            self._validate(circuit, hamiltonian)
            params = np.ascontiguousarray(parameters, dtype=np.float64)
            if params.ndim == 1:
                params = params.reshape(1, -1)
            vectors, pcount = params.shape
            if pcount != circuit.ParameterCount:
                raise ArgumentError("Binding size must match ParameterCount.")
            ops, nops = circuit.template_array()
            terms, nterms = terms_array(hamiltonian.Terms)
            energies = np.zeros(vectors, dtype=np.float64)
            grads = np.zeros((vectors, max(1, pcount)), dtype=np.float64)
            keep += [ops, terms, params, energies, grads]
            r = recs[i]
            r.qubits, r.precision, r.operations, r.operation_count = circuit.QubitCount, self.precision, \
                C.cast(ops, C.c_void_p), nops
            r.parameter_count, r.terms, r.term_count, r.vectors = pcount, C.cast(terms, C.c_void_p), nterms, vectors
            r.coefficients, r.parameters = None, params.ctypes.data_as(_lib.DP)
            r.with_gradient, r.energies, r.gradients = 1 if withGradient else 0, energies.ctypes.data_as(_lib.DP), \
                grads.ctypes.data_as(_lib.DP)
            outs.append((energies, grads[:, :pcount] if withGradient else None))
        stats = _lib.VqeStats()
        check(load().qm_vqe_evaluate_mixed(self.context.handle, recs, len(problems), C.byref(stats)))
        total = BatchEvaluation(None, None, stats.circuits, stats.waves, stats.batch_states, stats.passes_per_circuit,
                                stats.tile_passes, stats.device_seconds, stats.wall_seconds)
        return outs, total

    def Evaluate(self, circuit: ParameterizedCircuit, hamiltonian: PauliHamiltonian,
                 parameters: Sequence[float]) -> float:
        circuit._check(parameters)
        return float(self.EvaluateBatch(circuit, hamiltonian, np.asarray(parameters, dtype=np.float64),
                                         withGradient=False).Energies[0])

    def EvaluateWithGradient(self, circuit: ParameterizedCircuit, hamiltonian: PauliHamiltonian,
                             parameters: Sequence[float]) -> VariationalEnergyResult:
        circuit._check(parameters)
        r = self.EvaluateBatch(circuit, hamiltonian, np.asarray(parameters, dtype=np.float64), withGradient=True)
        return VariationalEnergyResult(float(r.Energies[0]), tuple(float(g) for g in r.Gradients[0]))


class VqeTerminationReason(IntEnum):
    """VqeTerminationReason.cs:4-14."""
    GradientToleranceReached = 0
    IterationLimitReached = 1
    EvaluationLimitReached = 2
    LineSearchStalled = 3


@dataclass(frozen=True)
class VqeOptions:
    """VqeOptions.cs:7-28 defaults."""
    MaximumIterations: int = 200
    MaximumCircuitEvaluations: int = 100_000
    MaximumLineSearchIterations: int = 40
    GradientTolerance: float = 1e-6
    InitialStepSize: float = 1.0
    MinimumStepSize: float = 1e-12
    BacktrackingFactor: float = 0.5
    SufficientDecrease: float = 0.1

    def Validate(self) -> None:
        if self.MaximumIterations < 0 or self.MaximumCircuitEvaluations <= 0 or self.MaximumLineSearchIterations <= 0:
            raise ArgumentOutOfRangeError("limits")
        if not math.isfinite(self.GradientTolerance) or self.GradientTolerance < 0:
            raise ArgumentOutOfRangeError("GradientTolerance")
        if not math.isfinite(self.InitialStepSize) or self.InitialStepSize <= 0:
            raise ArgumentOutOfRangeError("InitialStepSize")
        if (not math.isfinite(self.MinimumStepSize) or self.MinimumStepSize <= 0
                or self.MinimumStepSize > self.InitialStepSize):
            raise ArgumentOutOfRangeError("MinimumStepSize")
        if not math.isfinite(self.BacktrackingFactor) or not 0 < self.BacktrackingFactor < 1:
            raise ArgumentOutOfRangeError("BacktrackingFactor")
        if not math.isfinite(self.SufficientDecrease) or not 0 < self.SufficientDecrease < 1:
            raise ArgumentOutOfRangeError("SufficientDecrease")


@dataclass(frozen=True)
class VqeResult:
    Parameters: tuple[float, ...]
    Energy: float
    IterationCount: int
    EnergyEvaluationCount: int
    GradientEvaluationCount: int
    CircuitEvaluationCount: int
    TerminationReason: VqeTerminationReason


class VqeSolver:
    """Steepest descent with bounded Armijo backtracking (VqeSolver.cs:27-117) on the B200 evaluator."""

    def __init__(self, evaluator: B200VariationalEnergyEvaluator, options: VqeOptions | None = None):
        if evaluator is None:
            raise ArgumentError("evaluator")
        self.evaluator = evaluator
        self.options = options or VqeOptions()
        self.options.Validate()

    def Solve(self, circuit: ParameterizedCircuit, hamiltonian: PauliHamiltonian,
              initialParameters: Sequence[float]) -> VqeResult:
        o = self.options
        if circuit.QubitCount != hamiltonian.QubitCount:
            raise ArgumentError("Circuit and Hamiltonian sizes must match.")
        if len(initialParameters) != circuit.ParameterCount:
            raise ArgumentError("Parameter count must match the circuit.")
        params = [float(p) for p in initialParameters]
        for p in params:
            if not math.isfinite(p):
                raise ArgumentOutOfRangeError("Parameters must be finite.")
        ev = self.evaluator
        energy = ev.Evaluate(circuit, hamiltonian, params)
        energies, circuits, iterations, gradients = 1, 1, 0, 0
        cost = 1 + 2 * len(circuit.RotationParameterIndices)

        def finish(reason):
            return VqeResult(tuple(params), energy, iterations, energies, gradients, circuits, reason)

        while True:
            if iterations == o.MaximumIterations:
                return finish(VqeTerminationReason.IterationLimitReached)
            if o.MaximumCircuitEvaluations - circuits < cost:
                return finish(VqeTerminationReason.EvaluationLimitReached)
            ev_result = ev.EvaluateWithGradient(circuit, hamiltonian, params)
            gradients += 1
            circuits += cost
            energy = ev_result.Energy
            g = ev_result.Gradient
            norm = max((abs(x) for x in g), default=0.0)
            if norm <= o.GradientTolerance:
                return finish(VqeTerminationReason.GradientToleranceReached)
            scaled_squares = sum((x / norm) * (x / norm) for x in g)
            step = o.InitialStepSize
            accepted = False
            for _ in range(o.MaximumLineSearchIterations):
                if circuits == o.MaximumCircuitEvaluations:
                    return finish(VqeTerminationReason.EvaluationLimitReached)
                trial = [_fma(-step, gi, pi) for gi, pi in zip(g, params)]
                finite = all(math.isfinite(x) for x in trial)
                if all(t == p for t, p in zip(trial, params)):
                    return finish(VqeTerminationReason.LineSearchStalled)
                if finite:
                    candidate = ev.Evaluate(circuit, hamiltonian, trial)
                    energies += 1
                    circuits += 1
                    if self._sufficient(energy, candidate, step, norm, scaled_squares):
                        params = trial
                        energy = candidate
                        iterations += 1
                        accepted = True
                        break
                smaller = step * o.BacktrackingFactor
                if smaller < o.MinimumStepSize or smaller >= step:
                    break
                step = smaller
            if not accepted:
                return finish(VqeTerminationReason.LineSearchStalled)

    def _sufficient(self, energy: float, candidate: float, step: float, norm: float, scaled: float) -> bool:
        """Armijo test in log space (VqeSolver.cs:109-117)."""
        if candidate >= energy:
            return False
        scale = max(abs(energy), abs(candidate))
        log_decrease = math.log(scale) + math.log(energy / scale - candidate / scale)
        log_required = (math.log(self.options.SufficientDecrease) + math.log(step) + 2 * math.log(norm)
                        + math.log(scaled))
        return log_decrease >= log_required
