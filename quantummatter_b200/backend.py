"""Backend ports of QuantumMatter on libqmb200.

B200StateVectorBackend mirrors IStateVectorBackend / CudaStateVectorBackend
(src/QuantumMatter.Core/IStateVectorBackend.cs:13,
 src/QuantumMatter.Infrastructure/CudaStateVectorBackend.cs:21-216);
B200NoiseChannelBackend mirrors INoiseChannelBackend / CpuNoiseChannelBackend
(src/QuantumMatter.Core/Noise/INoiseChannelBackend.cs:13-14,
 src/QuantumMatter.Infrastructure/CpuNoiseChannelBackend.cs:10-145);
DeviceState is the additive device-resident state the batched evaluators use.
Amplitude buffers are numpy complex128 arrays (the layout of System.Numerics.Complex[]).
"""
from __future__ import annotations

import ctypes as C
import threading
from dataclasses import dataclass
from typing import Sequence

import numpy as np

from . import _lib
from ._lib import check, load
from .circuit import QuantumCircuit, operations_array, prepare
from .errors import ArgumentError, ArgumentOutOfRangeError, ObjectDisposedError
from .observables import PauliHamiltonian, PauliString, terms_array, observable_array

FP64 = 0
FP32 = 1


class CancellationToken:
    """A cancellation flag the library polls (the role of System.Threading.CancellationToken)."""

    def __init__(self) -> None:
        self._flag = C.c_int32(0)

    def Cancel(self) -> None:
        self._flag.value = 1

    @property
    def IsCancellationRequested(self) -> bool:
        return self._flag.value != 0

    def pointer(self):
        return C.pointer(self._flag)


def _cancel_ptr(token: CancellationToken | None):
    return token.pointer() if token is not None else None


@dataclass(frozen=True)
class B200BackendOptions:
    """CudaBackendOptions (CudaBackendOptions.cs:4-21) plus the engine's fusion width."""
    DeviceIndex: int = 0
    DeviceMemoryBudgetBytes: int = 512 * 1024 * 1024
    StagingMemoryBudgetBytes: int = 512 * 1024 * 1024
    EnableProfiling: bool = False
    FusionWidth: int = 0

    def to_c(self) -> _lib.Options:
        o = _lib.Options()
        load().qm_options_default(C.byref(o))
        o.device_index = self.DeviceIndex
        o.enable_profiling = 1 if self.EnableProfiling else 0
        o.device_budget_bytes = self.DeviceMemoryBudgetBytes
        o.staging_budget_bytes = self.StagingMemoryBudgetBytes
        o.fusion_width = self.FusionWidth
        return o


@dataclass(frozen=True)
class B200DeviceInfo:
    """CudaDeviceInfo (CudaBackendOptions.cs:26)."""
    Index: int
    Name: str
    Architecture: str
    CudaDriverVersion: str
    MemoryBytes: int
    SmCount: int


@dataclass(frozen=True)
class B200ExecutionProfile:
    """CudaExecutionProfile (CudaBackendOptions.cs:35) plus transfer time and plan figures."""
    DeviceEvolutionSeconds: float
    TransferSeconds: float
    StateBytes: int
    KernelLaunches: int
    Passes: int
    PlannedBytes: int


def _profile(p: _lib.Profile) -> B200ExecutionProfile:
    return B200ExecutionProfile(p.device_seconds, p.transfer_seconds, p.state_bytes, p.kernel_launches, p.passes,
                                p.planned_bytes)


def GetDevices() -> list[B200DeviceInfo]:
    """CudaStateVectorBackend.GetDevices: an empty list means no CUDA device is visible."""
    lib = load()
    n = C.c_int32(0)
    check(lib.qm_device_count(C.byref(n)))
    out = []
    for i in range(n.value):
        info = _lib.DeviceInfo()
        check(lib.qm_device_info_get(i, C.byref(info)))
        out.append(B200DeviceInfo(i, info.name.decode(), f"SM_{info.major}{info.minor}", str(info.driver_version),
                                  info.memory_bytes, info.sm_count))
    return out


class B200Context:
    """Owns one qm_context (a device, a stream and its budgets).  Disposal is idempotent."""

    def __init__(self, options: B200BackendOptions | None = None):
        self.options = options or B200BackendOptions()
        lib = load()
        o = self.options.to_c()
        h = C.c_void_p()
        check(lib.qm_context_create(C.byref(o), C.byref(h)))
        self._h = h
        self._lock = threading.Lock()
        self._disposed = False

    @property
    def handle(self) -> C.c_void_p:
        if self._disposed:
            raise ObjectDisposedError("B200Context")
        return self._h

    def Dispose(self) -> None:
        with self._lock:
            if self._disposed:
                return
            self._disposed = True
            load().qm_context_destroy(self._h)

    close = Dispose

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.Dispose()

    def host_array(self, length: int) -> "HostArray":
        return HostArray(self, length)


class HostArray:
    """Pinned (page-locked) complex128 host array from qm_host_alloc, viewed as numpy."""

    def __init__(self, ctx: B200Context, length: int):
        self._ctx = ctx
        ptr = C.c_void_p()
        check(load().qm_host_alloc(ctx.handle, 16 * length, C.byref(ptr)))
        self._ptr = ptr
        buf = (C.c_double * (2 * length)).from_address(ptr.value)
        self.array = np.frombuffer(buf, dtype=np.complex128, count=length)

    def free(self) -> None:
        if self._ptr is not None:
            self.array = None
            load().qm_host_free(self._ctx.handle, self._ptr)
            self._ptr = None


def _check_amplitudes(amplitudes: np.ndarray) -> np.ndarray:
    if not isinstance(amplitudes, np.ndarray) or amplitudes.dtype != np.complex128 or not amplitudes.flags.c_contiguous:
        raise ArgumentError("amplitudes must be a C-contiguous complex128 numpy array")
    if not amplitudes.flags.writeable:
        raise ArgumentError("amplitudes must be writable")
    return amplitudes


class B200StateVectorBackend:
    """IStateVectorBackend on one B200: whole-circuit, in-place, synchronous evolution of a host buffer.

    Calls on one instance are serialised (the reference's SemaphoreSlim(1,1)); the buffer is
    never retained; a failure or cancellation before the commit leaves it unchanged.
    """

    def __init__(self, options: B200BackendOptions | None = None, context: B200Context | None = None):
        self._owns = context is None
        self.context = context or B200Context(options)
        self.options = self.context.options
        self.Device = GetDevices()[self.options.DeviceIndex]

    GetDevices = staticmethod(GetDevices)

    def Execute(self, circuit: QuantumCircuit, amplitudes: np.ndarray, cancellationToken: CancellationToken | None = None):
        self._execute(circuit, amplitudes, cancellationToken, None)

    def ExecuteProfiled(self, circuit: QuantumCircuit, amplitudes: np.ndarray,
                        cancellationToken: CancellationToken | None = None) -> B200ExecutionProfile:
        if not self.options.EnableProfiling:
            from .errors import InvalidOperationError
            raise InvalidOperationError("EnableProfiling must be selected when creating the CUDA backend.")
        prof = _lib.Profile()
        self._execute(circuit, amplitudes, cancellationToken, prof)
        return _profile(prof)

    def _execute(self, circuit, amplitudes, token, prof):
        if circuit is None:
            raise ArgumentError("circuit")
        amplitudes = _check_amplitudes(amplitudes)
        arr, n = operations_array(circuit.Operations)
        check(load().qm_execute_host(self.context.handle, circuit.QubitCount, arr, n,
                                     amplitudes.ctypes.data_as(C.c_void_p), amplitudes.size, _cancel_ptr(token),
                                     C.byref(prof) if prof is not None else None))

    def Dispose(self) -> None:
        if self._owns:
            self.context.Dispose()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.Dispose()


class B200NoiseChannelBackend:
    """INoiseChannelBackend on one B200 (CpuNoiseChannelBackend.cs:10-145 branch semantics).

    `random` is any object with NextDouble() (System.Random's role); draws are consumed exactly
    where the reference consumes them.
    """

    def __init__(self, options: B200BackendOptions | None = None, context: B200Context | None = None):
        self._owns = context is None
        self.context = context or B200Context(options)

    def Apply(self, channel, target: int, amplitudes: np.ndarray, random, cancellationToken=None) -> None:
        if channel is None or random is None:
            raise ArgumentError("channel and random are required")
        amplitudes = _check_amplitudes(amplitudes)
        errors: list[BaseException] = []

        def draw(_user):
            try:
                return float(random.NextDouble())
            except BaseException as exc:  # surfaced after the call returns
                errors.append(exc)
                return 0.0

        cb = _lib.NEXT_DOUBLE_FN(draw)
        rc = load().qm_noise_apply_host(self.context.handle, int(channel.Kind), float(channel.Probability), target,
                                        amplitudes.ctypes.data_as(C.c_void_p), amplitudes.size, cb, None,
                                        _cancel_ptr(cancellationToken))
        if errors:
            raise errors[0]
        check(rc)

    def Dispose(self) -> None:
        if self._owns:
            self.context.Dispose()


class Plan:
    """A fused schedule of one circuit, planned once and executed many times (qm_plan_*)."""

    def __init__(self, context: B200Context, circuit: QuantumCircuit, precision: int = FP64, fusion_width: int = 0):
        gates, n = prepare(circuit)
        h = C.c_void_p()
        check(load().qm_plan_create(context.handle, circuit.QubitCount, precision, gates, n, fusion_width, C.byref(h)))
        self._h = h
        self.context = context
        self.qubits = circuit.QubitCount
        self.precision = precision

    @classmethod
    def autotune(cls, context: B200Context, circuit: QuantumCircuit, precision: int = FP64,
                 candidates: Sequence[int] | None = None) -> "Plan":
        """The plan of the fastest candidate fusion width, timed on the device (qm_plan_autotune);
        `width` holds the choice, cached per gate structure for the process."""
        gates, n = prepare(circuit)
        h, chosen = C.c_void_p(), C.c_int32()
        cand = list(candidates or [])
        arr = (C.c_int32 * len(cand))(*cand) if cand else None
        check(load().qm_plan_autotune(context.handle, circuit.QubitCount, precision, gates, n, arr, len(cand),
                                      C.byref(h), C.byref(chosen)))
        plan = cls.__new__(cls)
        plan._h, plan.context, plan.qubits, plan.precision = h, context, circuit.QubitCount, precision
        plan.width = chosen.value
        return plan

    def stats(self) -> tuple[int, int, int]:
        passes, launches, bytes_ = C.c_int32(), C.c_int32(), C.c_int64()
        check(load().qm_plan_stats(self._h, C.byref(passes), C.byref(launches), C.byref(bytes_)))
        return passes.value, launches.value, bytes_.value

    def execute(self, state: "DeviceState", profile: bool = False) -> B200ExecutionProfile | None:
        prof = _lib.Profile() if profile else None
        check(load().qm_plan_execute(self._h, state.handle, C.byref(prof) if prof is not None else None))
        return _profile(prof) if prof is not None else None

    def capture(self, state: "DeviceState") -> "CapturedExecution":
        """One execution of this plan on `state` as a CUDA graph (qm_graph_create)."""
        return CapturedExecution(self, state)

    def Dispose(self) -> None:
        if self._h is not None:
            load().qm_plan_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.Dispose()
        except Exception:
            pass


class CapturedExecution:
    """A plan's execution on one state captured as a CUDA graph; launch() replays it in place."""

    def __init__(self, plan: Plan, state: "DeviceState"):
        h = C.c_void_p()
        check(load().qm_graph_create(plan._h, state.handle, C.byref(h)))
        self._h = h
        self.plan, self.state = plan, state

    def launch(self, profile: bool = False) -> B200ExecutionProfile | None:
        prof = _lib.Profile() if profile else None
        check(load().qm_graph_launch(self._h, C.byref(prof) if prof is not None else None))
        return _profile(prof) if prof is not None else None

    def Dispose(self) -> None:
        if self._h is not None:
            load().qm_graph_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.Dispose()
        except Exception:
            pass


class DeviceState:
    """A state vector resident in device memory (complex128 or complex64), starting at |0...0>."""

    def __init__(self, context: B200Context, qubits: int, precision: int = FP64):
        h = C.c_void_p()
        check(load().qm_state_create(context.handle, qubits, precision, C.byref(h)))
        self._h = h
        self.context = context
        self.QubitCount = qubits
        self.precision = precision
        self.Length = 1 << qubits

    @property
    def handle(self) -> C.c_void_p:
        if self._h is None:
            raise ObjectDisposedError("DeviceState")
        return self._h

    def Dispose(self) -> None:
        if self._h is not None:
            load().qm_state_destroy(self._h)
            self._h = None

    def __del__(self):
        try:
            self.Dispose()
        except Exception:
            pass

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.Dispose()

    # -- data movement
    def Reset(self) -> None:
        check(load().qm_state_reset(self.handle))

    def Upload(self, amplitudes: np.ndarray) -> None:
        a = np.ascontiguousarray(amplitudes, dtype=np.complex128)
        check(load().qm_state_upload(self.handle, a.ctypes.data_as(C.c_void_p), a.size))

    def Download(self, out: np.ndarray | None = None) -> np.ndarray:
        if out is None:
            out = np.empty(self.Length, dtype=np.complex128)
        out = _check_amplitudes(out)
        check(load().qm_state_download(self.handle, out.ctypes.data_as(C.c_void_p), out.size))
        return out

    def device_pointer(self) -> int:
        p = C.c_void_p()
        check(load().qm_state_device_pointer(self.handle, C.byref(p)))
        return p.value or 0

    # -- evolution
    def Evolve(self, circuit: QuantumCircuit, fusion_width: int = 0, profile: bool = False):
        if circuit.QubitCount != self.QubitCount:
            raise ArgumentError("Circuit and state sizes must match.")
        gates, n = prepare(circuit)
        prof = _lib.Profile() if profile else None
        check(load().qm_execute(self.handle, gates, n, fusion_width, C.byref(prof) if prof is not None else None))
        return _profile(prof) if prof is not None else None

    # -- observables
    def ExpectationValues(self, observables: Sequence[PauliString]) -> tuple[np.ndarray, float]:
        for o in observables:
            if o.QubitCount != self.QubitCount:
                raise ArgumentError("Observable and state sizes must match.")
        arr, n = observable_array(observables)
        out = np.zeros(max(1, n), dtype=np.float64)
        mass = C.c_double()
        check(load().qm_expectation_pauli(self.handle, arr, n, out.ctypes.data_as(_lib.DP), C.byref(mass)))
        return out[:n], mass.value

    def ExpectationValue(self, observable: PauliString) -> float:
        return float(self.ExpectationValues([observable])[0][0])

    def ExpectationEnergy(self, hamiltonian: PauliHamiltonian) -> float:
        if hamiltonian.QubitCount != self.QubitCount:
            raise ArgumentError("Hamiltonian and state sizes must match.")
        arr, n = terms_array(hamiltonian.Terms)
        e = C.c_double()
        check(load().qm_expectation_energy(self.handle, arr, n, C.byref(e)))
        return e.value

    # -- noise primitives
    def QubitMasses(self, target: int) -> tuple[float, float]:
        m0, m1 = C.c_double(), C.c_double()
        check(load().qm_qubit_masses(self.handle, target, C.byref(m0), C.byref(m1)))
        return m0.value, m1.value

    def ApplyPauli(self, target: int, pauli: int) -> None:
        check(load().qm_apply_pauli(self.handle, target, pauli))

    def ApplyDamping(self, target: int, jump: bool, scale: float, jump_scale: float, stay_scale: float) -> None:
        check(load().qm_apply_damping(self.handle, target, 1 if jump else 0, scale, jump_scale, stay_scale))

    def ApplyNoise(self, channel, target: int, random) -> None:
        """INoiseChannelBackend.Apply on the resident state (qm_state_noise_apply): `random` is
        any object with NextDouble(), consumed exactly where the reference consumes it."""
        if channel is None or random is None:
            raise ArgumentError("channel and random are required")
        errors: list[BaseException] = []

        def draw(_user):
            try:
                return float(random.NextDouble())
            except BaseException as exc:  # surfaced after the call returns
                errors.append(exc)
                return 0.0

        cb = _lib.NEXT_DOUBLE_FN(draw)
        rc = load().qm_state_noise_apply(self.handle, int(channel.Kind), float(channel.Probability), target, cb, None)
        if errors:
            raise errors[0]
        check(rc)

    # -- sampling
    def MeasureAll(self, u: float) -> tuple[int, bool]:
        out, amb = C.c_int64(), C.c_int32()
        check(load().qm_measure_all(self.handle, float(u), C.byref(out), C.byref(amb)))
        return out.value, bool(amb.value)

    def MarginalProbability(self, qubits: Sequence[int], outcome: int) -> float:
        """StateVector.MarginalProbability: bit k of outcome refers to qubits[k]."""
        sel = (C.c_int32 * max(1, len(qubits)))(*qubits)
        p = C.c_double()
        check(load().qm_marginal_probability(self.handle, sel, len(qubits), int(outcome), C.byref(p)))
        return p.value

    def Measure(self, qubits: Sequence[int], u: float) -> tuple[int, bool]:
        """StateVector.Measure with the draw u: projects the state on the device and returns the
        selected qubits' values (bit k = qubits[k]) and whether u sat on a CDF boundary."""
        sel = (C.c_int32 * max(1, len(qubits)))(*qubits)
        out, amb = C.c_int32(), C.c_int32()
        check(load().qm_measure(self.handle, sel, len(qubits), float(u), C.byref(out), C.byref(amb)))
        return out.value, bool(amb.value)

    def Sample(self, draws: Sequence[float]) -> tuple[np.ndarray, int]:
        d = np.ascontiguousarray(draws, dtype=np.float64)
        if d.size < 1:
            raise ArgumentOutOfRangeError("shots must be positive")
        out = np.zeros(d.size, dtype=np.int64)
        amb = C.c_int32()
        check(load().qm_sample(self.handle, d.ctypes.data_as(_lib.DP), d.size, out.ctypes.data_as(_lib.I64P),
                               C.byref(amb)))
        return out, amb.value


def jit_info() -> dict:
    """Whether passes can be compiled for their own op sequence, and process-wide counts of
    compiled kernels, failed compilations and launches of compiled passes (qm_jit_info)."""
    avail, kernels, failed, launches = C.c_int32(), C.c_int64(), C.c_int64(), C.c_int64()
    check(load().qm_jit_info(C.byref(avail), C.byref(kernels), C.byref(failed), C.byref(launches)))
    return {"available": bool(avail.value), "kernels": kernels.value, "failed": failed.value,
            "launches": launches.value}
