"""Pauli observables mirroring src/QuantumMatter.Core/PauliString.cs and Observables/*.cs."""
from __future__ import annotations

import math
from typing import Sequence

from .errors import ArgumentError, ArgumentOutOfRangeError


class PauliString:
    """Tensor product of I, X, Y, Z with qubit zero at the right (PauliString.cs:7-29)."""

    def __init__(self, operators: str):
        if operators is None:
            raise ArgumentError("operators")
        if len(operators) < 1 or len(operators) > 30:
            raise ArgumentOutOfRangeError("A Pauli string requires 1 through 30 labels.")
        flip = sign = ycount = 0
        for qubit in range(len(operators)):
            label = operators[len(operators) - 1 - qubit]
            if label not in "IXYZ":
                raise ArgumentError("Only uppercase I, X, Y and Z labels are supported.")
            if label in "XY":
                flip |= 1 << qubit
            if label in "ZY":
                sign |= 1 << qubit
            if label == "Y":
                ycount += 1
        self.Operators = operators
        self.FlipMask = flip
        self.SignMask = sign
        self.YCount = ycount

    @property
    def QubitCount(self) -> int:
        return len(self.Operators)

    def __repr__(self) -> str:
        return f"PauliString({self.Operators!r})"


class PauliTerm:
    """Finite real coefficient times a PauliString (PauliTerm.cs:7-13)."""

    def __init__(self, coefficient: float, observable: PauliString):
        if observable is None:
            raise ArgumentError("observable")
        if not math.isfinite(coefficient):
            raise ArgumentOutOfRangeError("coefficient")
        self.Coefficient = float(coefficient)
        self.Observable = observable


class PauliHamiltonian:
    """Ordered real sum of register-sized terms; duplicates and zeros are kept (PauliHamiltonian.cs:8-26)."""

    def __init__(self, qubits: int, terms: Sequence[PauliTerm]):
        if qubits < 1 or qubits > 30:
            raise ArgumentOutOfRangeError("qubits")
        if terms is None:
            raise ArgumentError("terms")
        snap = []
        for t in terms:
            if t is None or t.Observable.QubitCount != qubits:
                raise ArgumentError("Every term must be nonnull and match the register size.")
            snap.append(t)
        self.QubitCount = qubits
        self.Terms = tuple(snap)


def terms_array(terms: Sequence[PauliTerm]):
    """Packs terms into a ctypes qm_pauli_term array."""
    from ._lib import PauliTermC
    arr = (PauliTermC * max(1, len(terms)))()
    for i, t in enumerate(terms):
        arr[i].flip_mask = t.Observable.FlipMask
        arr[i].sign_mask = t.Observable.SignMask
        arr[i].y_count = t.Observable.YCount
        arr[i].coefficient = t.Coefficient
    return arr, len(terms)


def observable_array(observables: Sequence[PauliString]):
    return terms_array([PauliTerm(1.0, o) for o in observables])

