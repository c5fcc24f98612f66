"""Exceptions mirroring the .NET exceptions the reference raises for each qm_status."""
from __future__ import annotations


class QuantumMatterError(Exception):
    """Base of every error raised by this package."""


class ArgumentError(QuantumMatterError, ValueError):
    """ArgumentException / ArgumentNullException."""


class ArgumentOutOfRangeError(ArgumentError):
    """ArgumentOutOfRangeException."""


class InvalidOperationError(QuantumMatterError, RuntimeError):
    """InvalidOperationException (budgets, no finite positive mass)."""


class BudgetExceededError(InvalidOperationError):
    """InvalidOperationException raised before the input is touched because a memory budget is exceeded."""


class MassError(InvalidOperationError):
    """InvalidOperationException: the state has no finite positive probability mass."""


class OperationCanceledError(QuantumMatterError):
    """OperationCanceledException."""


class ObjectDisposedError(InvalidOperationError):
    """ObjectDisposedException."""


class PlatformNotSupportedError(QuantumMatterError, OSError):
    """PlatformNotSupportedException: no CUDA device or driver."""


class NotSupportedError(QuantumMatterError, NotImplementedError):
    """NotSupportedException: unknown gate kind."""


class DeviceError(QuantumMatterError, RuntimeError):
    """A CUDA runtime failure."""


class DeviceOutOfMemoryError(DeviceError, MemoryError):
    """Device or pinned host allocation failed."""


class DeviceTimeoutError(DeviceError, TimeoutError):
    """A bounded device wait ran out."""


_BY_STATUS = {
    1: ArgumentError,
    2: BudgetExceededError,
    3: DeviceOutOfMemoryError,
    4: DeviceError,
    5: OperationCanceledError,
    6: DeviceTimeoutError,
    7: MassError,
    8: ObjectDisposedError,
    9: NotSupportedError,
    10: ArgumentOutOfRangeError,
}


def raise_for_status(status: int, message: str) -> None:
    cls = _BY_STATUS.get(status, DeviceError)
    if status == 4 and "No compatible NVIDIA CUDA device" in message:
        cls = PlatformNotSupportedError
    raise cls(f"[qm status {status}] {message}")
