"""QuantumMatter-B200: a B200 (sm_100a) state-vector engine behind QuantumMatter's backend ports.

The compute path is libqmb200.so (hand-written CUDA kernels behind the C ABI of
include/qm_b200.h).  This package is the host-side mirror of the reference's
Core/Infrastructure interface used by the tests and the benchmark: it loads the library
through ctypes and has no CPU fallback.
"""
from .circuit import GateKind, GateOperation, QuantumCircuit, SingleQubitUnitary, u3
from .errors import (ArgumentError, ArgumentOutOfRangeError, BudgetExceededError, DeviceError,
                     InvalidOperationError, MassError, NotSupportedError, ObjectDisposedError,
                     OperationCanceledError, PlatformNotSupportedError)
from .observables import PauliHamiltonian, PauliString, PauliTerm

__all__ = [
    "GateKind", "GateOperation", "QuantumCircuit", "SingleQubitUnitary", "u3",
    "PauliString", "PauliTerm", "PauliHamiltonian",
    "ArgumentError", "ArgumentOutOfRangeError", "BudgetExceededError", "DeviceError", "InvalidOperationError",
    "MassError", "NotSupportedError", "ObjectDisposedError", "OperationCanceledError", "PlatformNotSupportedError",
]
