"""Circuit IR mirroring QuantumMatter's Core layer, with the reference's names.

GateKind, GateOperation and QuantumCircuit follow src/QuantumMatter.Core/QuantumCircuit.cs
(:4-220); SingleQubitUnitary follows src/QuantumMatter.Core/SingleQubitUnitary.cs (:41-79).
Builders validate exactly as the reference does and raise the mirrored exceptions.
"""
from __future__ import annotations

import ctypes as C
import math
from dataclasses import dataclass
from enum import IntEnum
from typing import Iterable, Sequence

from .errors import ArgumentError, ArgumentOutOfRangeError


class GateKind(IntEnum):
    """Stable operation identifiers (QuantumCircuit.cs:4-40)."""
    H = 0
    X = 1
    Y = 2
    Z = 3
    S = 4
    T = 5
    Rx = 6
    Ry = 7
    Rz = 8
    CNot = 9
    Swap = 10
    I = 11
    Sdg = 12
    Tdg = 13
    Phase = 14
    Unitary = 15
    Toffoli = 16


class SingleQubitUnitary:
    """Immutable row-major 2x2 unitary validated at construction (SingleQubitUnitary.cs:41-63)."""

    ValidationTolerance = 1e-12

    __slots__ = ("M00", "M01", "M10", "M11")

    def __init__(self, m00: complex, m01: complex, m10: complex, m11: complex):
        object.__setattr__(self, "M00", complex(m00))
        object.__setattr__(self, "M01", complex(m01))
        object.__setattr__(self, "M10", complex(m10))
        object.__setattr__(self, "M11", complex(m11))

    def __setattr__(self, name, value):
        raise AttributeError("SingleQubitUnitary is immutable")

    @staticmethod
    def Create(m00, m01=None, m10=None, m11=None) -> "SingleQubitUnitary":
        if m01 is None:  # a 2x2 nested sequence
            rows = m00
            if len(rows) != 2 or any(len(r) != 2 for r in rows):
                raise ArgumentError("A single-qubit matrix must have exactly two rows and two columns.")
            m00, m01, m10, m11 = rows[0][0], rows[0][1], rows[1][0], rows[1][1]
        vals = [complex(v) for v in (m00, m01, m10, m11)]
        for v in vals:
            if not (math.isfinite(v.real) and math.isfinite(v.imag)):
                raise ArgumentOutOfRangeError("Matrix entries must be finite.")
        a, b, c, d = vals

        def sq(z: complex) -> float:
            return z.real * z.real + z.imag * z.imag

        first = sq(a) + sq(c)
        second = sq(b) + sq(d)
        tol = SingleQubitUnitary.ValidationTolerance
        if abs(first - 1) > tol or abs(second - 1) > tol:
            raise ArgumentError("Matrix columns must have unit norm.")
        inner = a.conjugate() * b + c.conjugate() * d
        if abs(inner) > tol:
            raise ArgumentError("Matrix columns must be orthogonal.")
        return SingleQubitUnitary(a, b, c, d)

    def Adjoint(self) -> "SingleQubitUnitary":
        return SingleQubitUnitary(self.M00.conjugate(), self.M10.conjugate(), self.M01.conjugate(),
                                  self.M11.conjugate())

    def __eq__(self, other) -> bool:
        return isinstance(other, SingleQubitUnitary) and (self.M00, self.M01, self.M10, self.M11) == (
            other.M00, other.M01, other.M10, other.M11)

    def __hash__(self) -> int:
        return hash((self.M00, self.M01, self.M10, self.M11))


def u3(theta: float, phi: float, lam: float) -> SingleQubitUnitary:
    """U3(theta, phi, lambda) = [[cos t/2, -e^{i lam} sin t/2], [e^{i phi} sin t/2, e^{i(phi+lam)} cos t/2]],
    passed to the reference as a validated custom matrix (it has no native U3)."""
    c, s = math.cos(theta / 2), math.sin(theta / 2)
    e_l = complex(math.cos(lam), math.sin(lam))
    e_p = complex(math.cos(phi), math.sin(phi))
    e_pl = complex(math.cos(phi + lam), math.sin(phi + lam))
    return SingleQubitUnitary.Create(c, -e_l * s, e_p * s, e_pl * c)


@dataclass(frozen=True)
class GateOperation:
    """GateOperation record (QuantumCircuit.cs:49-61)."""
    Kind: GateKind
    Target: int
    Control: int = -1
    Angle: float = 0.0
    SecondControl: int = -1
    Unitary: SingleQubitUnitary | None = None


_CONTROLLABLE = {GateKind.H, GateKind.X, GateKind.Y, GateKind.Z, GateKind.S, GateKind.T, GateKind.Rx, GateKind.Ry,
                 GateKind.Rz, GateKind.I, GateKind.Sdg, GateKind.Tdg, GateKind.Phase}


class QuantumCircuit:
    """Mutable, validated unitary circuit; qubit zero is the least significant index bit."""

    def __init__(self, qubits: int):
        if not isinstance(qubits, int) or qubits < 1 or qubits > 30:
            raise ArgumentOutOfRangeError("Number of qubits must be between 1 and 30.")
        self.QubitCount = qubits
        self._ops: list[GateOperation] = []

    @property
    def Operations(self) -> Sequence[GateOperation]:
        return tuple(self._ops)

    def Copy(self) -> "QuantumCircuit":
        c = QuantumCircuit(self.QubitCount)
        c._ops = list(self._ops)
        return c

    def AppendValidated(self, op: GateOperation) -> None:
        self._ops.append(op)

    def _validate(self, q: int) -> None:
        if not isinstance(q, int) or q < 0 or q >= self.QubitCount:
            raise ArgumentOutOfRangeError("qubit")

    def _add(self, kind: GateKind, target: int, control: int | None = None, angle: float = 0.0,
             second: int | None = None, unitary: SingleQubitUnitary | None = None) -> "QuantumCircuit":
        self._validate(target)
        if control is not None:
            self._validate(control)
            if control == target:
                raise ArgumentError("The two qubits must differ.")
        if second is not None:
            self._validate(second)
            if second == target or second == control:
                raise ArgumentError("All three qubits must differ.")
        if not math.isfinite(angle):
            raise ArgumentOutOfRangeError("angle")
        self._ops.append(GateOperation(kind, target, -1 if control is None else control, float(angle),
                                       -1 if second is None else second, unitary))
        return self

    # builders (QuantumCircuit.cs:136-219)
    def H(self, q): return self._add(GateKind.H, q)
    def X(self, q): return self._add(GateKind.X, q)
    def Y(self, q): return self._add(GateKind.Y, q)
    def Z(self, q): return self._add(GateKind.Z, q)
    def S(self, q): return self._add(GateKind.S, q)
    def T(self, q): return self._add(GateKind.T, q)
    def Rx(self, q, angle): return self._add(GateKind.Rx, q, angle=angle)
    def Ry(self, q, angle): return self._add(GateKind.Ry, q, angle=angle)
    def Rz(self, q, angle): return self._add(GateKind.Rz, q, angle=angle)
    def CNot(self, control, target): return self._add(GateKind.CNot, target, control)
    def Swap(self, a, b): return self._add(GateKind.Swap, b, a)
    def I(self, q): return self._add(GateKind.I, q)
    def Sdg(self, q): return self._add(GateKind.Sdg, q)
    def Tdg(self, q): return self._add(GateKind.Tdg, q)
    def Phase(self, q, angle): return self._add(GateKind.Phase, q, angle=angle)

    def Controlled(self, kind: GateKind, control: int, target: int, angle: float = 0.0) -> "QuantumCircuit":
        if kind not in _CONTROLLABLE:
            raise ArgumentOutOfRangeError("A built-in single-qubit gate is required.")
        return self._add(kind, target, control, angle)

    def CH(self, c, t): return self.Controlled(GateKind.H, c, t)
    def CY(self, c, t): return self.Controlled(GateKind.Y, c, t)
    def CZ(self, c, t): return self.Controlled(GateKind.Z, c, t)
    def CS(self, c, t): return self.Controlled(GateKind.S, c, t)
    def CT(self, c, t): return self.Controlled(GateKind.T, c, t)
    def CSdg(self, c, t): return self.Controlled(GateKind.Sdg, c, t)
    def CTdg(self, c, t): return self.Controlled(GateKind.Tdg, c, t)
    def CRx(self, c, t, angle): return self.Controlled(GateKind.Rx, c, t, angle)
    def CRy(self, c, t, angle): return self.Controlled(GateKind.Ry, c, t, angle)
    def CRz(self, c, t, angle): return self.Controlled(GateKind.Rz, c, t, angle)
    def CPhase(self, c, t, angle): return self.Controlled(GateKind.Phase, c, t, angle)

    def U(self, target: int, unitary: SingleQubitUnitary) -> "QuantumCircuit":
        if unitary is None:
            raise ArgumentError("unitary")
        return self._add(GateKind.Unitary, target, unitary=unitary)

    def ControlledU(self, control: int, target: int, unitary: SingleQubitUnitary) -> "QuantumCircuit":
        if unitary is None:
            raise ArgumentError("unitary")
        return self._add(GateKind.Unitary, target, control, unitary=unitary)

    def Toffoli(self, first: int, second: int, target: int) -> "QuantumCircuit":
        return self._add(GateKind.Toffoli, target, first, second=second)


def operations_array(ops: Iterable[GateOperation]):
    """Packs GateOperation records into a ctypes qm_operation array."""
    from ._lib import Operation
    ops = list(ops)
    arr = (Operation * max(1, len(ops)))()
    for i, o in enumerate(ops):
        r = arr[i]
        r.kind = int(o.Kind)
        r.target = o.Target
        r.control = o.Control
        r.second_control = o.SecondControl
        r.angle = o.Angle
        if o.Unitary is not None:
            u = o.Unitary
            vals = (u.M00.real, u.M00.imag, u.M01.real, u.M01.imag, u.M10.real, u.M10.imag, u.M11.real, u.M11.imag)
            for j, v in enumerate(vals):
                r.unitary[j] = v
    return arr, len(ops)


def prepare(circuit: QuantumCircuit):
    """PreparedStateVectorGate.Prepare for every operation, evaluated by libqmb200's host code."""
    from ._lib import Gate, check, load
    arr, n = operations_array(circuit.Operations)
    gates = (Gate * max(1, n))()
    check(load().qm_prepare_gates(arr, n, circuit.QubitCount, gates))
    return gates, n


def gate_record_bytes() -> int:
    from ._lib import Gate, Operation
    return C.sizeof(Gate), C.sizeof(Operation)
