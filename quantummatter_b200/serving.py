"""Request serving on the B200: continuous batching under an HBM admission budget.

The reference runs one circuit at a time through its backend port (an application calls
StateVector.Evolve, ExpectationValue, StateVectorSimulator.Run or VariationalEnergyEvaluator
in sequence).  This module serves a stream of such requests concurrently on one GPU:

- ExpectationRequest: <P> of every observable on a circuit's final state
  (StateVector.ExpectationValue, StateVector.Observations.cs:107-141);
- ShotsRequest: terminal measurement samples of a circuit with a seeded draw stream
  (StateVectorSimulator.Run, StateVectorSimulator.cs:37-101);
- VqeStepRequest: one energy and parameter-shift gradient of a VQE session's ansatz
  (VariationalEnergyEvaluator.EvaluateWithGradient, VariationalEnergyEvaluator.cs:34-86) and one
  steepest-descent update of the session's parameters, which stay resident in the server
  between steps.

The server itself is the library's (qm_serve_* in include/qm_b200.h, csrc/qm_serve.cpp), so a
.NET host drives the same engine through P/Invoke:
- admission: a request reserves the bytes of its state (16 * 2^n for FP64, 8 * 2^n for FP32)
  against the server's budget; the oldest waiting request goes first, and a younger one may pass
  it only while the older one does not fit;
- batching: waiting VQE steps whose ansatz structure, Hamiltonian Pauli strings and precision
  match are evaluated as one device batch (qm_vqe_evaluate_coefficients), each with its own
  Hamiltonian coefficients and parameters; a session never has two steps in flight;
- execution: each worker thread owns a context (its own CUDA stream), so requests on different
  workers overlap on the GPU; a worker keeps the device states of recent sizes for reuse.
This module holds the request types, the Python face of the server and the plain form.
"""
from __future__ import annotations

import ctypes as C
import math
import threading
import time
from dataclasses import dataclass
from typing import Callable, Sequence

import numpy as np

from . import _lib
from ._lib import check, load
from .backend import FP32, FP64, B200Context, DeviceState
from .circuit import QuantumCircuit, operations_array
from .errors import ArgumentError, ArgumentOutOfRangeError
from .observables import PauliHamiltonian, PauliString, observable_array, terms_array
from .trajectories import random_doubles
from .variational import ParameterizedCircuit, _fma


def state_bytes(qubits: int, precision: int) -> int:
    return (8 if precision == FP32 else 16) << qubits


@dataclass
class ExpectationRequest:
    circuit: QuantumCircuit
    observables: Sequence[PauliString]
    precision: int = FP64

    @property
    def qubits(self) -> int:
        return self.circuit.QubitCount


@dataclass
class ShotsRequest:
    circuit: QuantumCircuit
    shots: int = 1000
    seed: int = 0
    precision: int = FP64

    @property
    def qubits(self) -> int:
        return self.circuit.QubitCount


class VqeSession:
    """A VQE run held by the server: ansatz, Hamiltonian and the current parameters."""

    def __init__(self, circuit: ParameterizedCircuit, hamiltonian: PauliHamiltonian, parameters: Sequence[float],
                 step_size: float = 0.1, precision: int = FP64):
        if circuit.QubitCount != hamiltonian.QubitCount:
            raise ArgumentError("Circuit and Hamiltonian sizes must match.")
        if len(parameters) != circuit.ParameterCount:
            raise ArgumentError("Parameter count must match the circuit.")
        if not (step_size > 0 and math.isfinite(step_size)):
            raise ArgumentOutOfRangeError("step_size")
        self.circuit = circuit
        self.hamiltonian = hamiltonian
        self.parameters = np.array(parameters, dtype=np.float64)
        self.step_size = float(step_size)
        self.precision = precision
        self.steps = 0
        self.coefficients = np.array([t.Coefficient for t in hamiltonian.Terms], dtype=np.float64)


@dataclass
class VqeStepRequest:
    session: VqeSession

    @property
    def qubits(self) -> int:
        return self.session.circuit.QubitCount

    @property
    def precision(self) -> int:
        return self.session.precision


@dataclass
class Response:
    kind: str
    values: np.ndarray | None = None      # expectation values
    mass: float | None = None
    outcomes: np.ndarray | None = None    # shot outcomes, in draw order
    counts: dict | None = None
    energy: float | None = None
    gradient: np.ndarray | None = None
    parameters: np.ndarray | None = None  # the session's parameters after the step
    batch: int = 1                        # requests evaluated together with this one
    submitted: float = 0.0
    started: float = 0.0
    finished: float = 0.0

    @property
    def latency(self) -> float:
        return self.finished - self.submitted


class ServeFuture:
    """A submitted request: result() waits for it and returns its Response (qm_serve_wait,
    qm_serve_take_result); the request's failure is raised there."""

    def __init__(self, server: "B200Server", request, rid: int, sizes: tuple[int, int, int]):
        self._server, self._request, self._id, self._sizes = server, request, rid, sizes
        self._lock = threading.Lock()
        self._response: Response | None = None
        self._error: BaseException | None = None

    def done(self) -> bool:
        if self._response is not None or self._error is not None:
            return True
        flag = C.c_int32()
        check(load().qm_serve_wait(self._server._h, self._id, 0.0, C.byref(flag)))
        return bool(flag.value)

    def result(self, timeout: float | None = None) -> Response:
        with self._lock:
            if self._response is None and self._error is None:
                deadline = None if timeout is None else time.perf_counter() + timeout
                flag = C.c_int32()
                while True:
                    left = 3600.0 if deadline is None else max(0.0, deadline - time.perf_counter())
                    check(load().qm_serve_wait(self._server._h, self._id, min(left, 3600.0), C.byref(flag)))
                    if flag.value:
                        break
                    if deadline is not None and time.perf_counter() >= deadline:
                        raise TimeoutError("the request has not finished")
                self._take()
        if self._error is not None:
            raise self._error
        return self._response

    def _take(self) -> None:
        nv, no, np_ = self._sizes
        values = np.zeros(max(1, nv))
        outcomes = np.zeros(max(1, no), dtype=np.int64)
        params = np.zeros(max(1, np_))
        res = _lib.ServeResult()
        check(load().qm_serve_take_result(self._server._h, self._id, C.byref(res), values.ctypes.data_as(_lib.DP), nv,
                                          outcomes.ctypes.data_as(C.POINTER(C.c_int64)), no,
                                          params.ctypes.data_as(_lib.DP), np_))
        try:
            check(res.status)
        except Exception as e:  # noqa: BLE001 - the request's own failure, raised by result()
            self._error = e
            return
        kind = {0: "expectation", 1: "shots", 2: "vqe_step"}[res.kind]
        r = Response(kind, batch=res.batch, submitted=res.submitted, started=res.started, finished=res.finished)
        if kind == "expectation":
            r.values, r.mass = values[:res.values].copy(), res.mass
        elif kind == "shots":
            r.outcomes = outcomes[:res.outcomes].copy()
            counts: dict[str, int] = {}
            for o in r.outcomes:
                k = format(int(o), "b").zfill(self._request.qubits)
                counts[k] = counts.get(k, 0) + 1
            r.counts = dict(sorted(counts.items()))
        else:
            r.energy, r.gradient = res.energy, values[:res.values].copy()
            r.parameters = params[:res.parameters].copy()
            s = self._request.session
            s.parameters = r.parameters.copy()
            s.steps += 1
        self._response = r


class B200Server:
    """The library's request server (qm_serve_*): `workers` threads, each with its own context and
    CUDA stream, admission by state bytes against `budget_bytes`, batched VQE steps."""

    def __init__(self, workers: int = 4, budget_bytes: int = 64 << 30, max_batch: int = 64,
                 context_budget_bytes: int = 32 << 30, cache_bytes: int = 8 << 30, device_index: int = 0):
        if workers < 1:
            raise ArgumentOutOfRangeError("workers")
        o = _lib.ServeOptions()
        o.device_index, o.workers, o.budget_bytes = device_index, workers, budget_bytes
        o.context_budget_bytes, o.cache_bytes, o.max_batch = context_budget_bytes, cache_bytes, max_batch
        h = C.c_void_p()
        check(load().qm_serve_create(C.byref(o), C.byref(h)))
        self._h = h
        self._sessions: dict[int, int] = {}  # id(VqeSession) -> server session
        self._session_objects: dict[int, VqeSession] = {}

    def _session(self, s: VqeSession) -> int:
        sid = self._sessions.get(id(s))
        if sid is None:
            ops, nops = s.circuit.template_array()
            arr, n = terms_array(s.hamiltonian.Terms)
            params = np.ascontiguousarray(s.parameters, dtype=np.float64)
            out = C.c_int64()
            check(load().qm_serve_session_create(self._h, s.circuit.QubitCount, s.precision, ops, nops,
                                                 s.circuit.ParameterCount, arr, n, params.ctypes.data_as(_lib.DP),
                                                 s.step_size, C.byref(out)))
            sid = self._sessions[id(s)] = out.value
            self._session_objects[id(s)] = s
        return sid

    def submit(self, request) -> ServeFuture:
        rid = C.c_int64()
        if isinstance(request, ExpectationRequest):
            ops, n = operations_array(request.circuit.Operations)
            arr, t = observable_array(list(request.observables))
            check(load().qm_serve_submit_expectation(self._h, request.qubits, request.precision, ops, n, arr, t,
                                                     C.byref(rid)))
            sizes = (t, 0, 0)
        elif isinstance(request, ShotsRequest):
            ops, n = operations_array(request.circuit.Operations)
            draws = np.ascontiguousarray(random_doubles(request.seed, request.shots), dtype=np.float64)
            check(load().qm_serve_submit_shots(self._h, request.qubits, request.precision, ops, n,
                                               draws.ctypes.data_as(_lib.DP), request.shots, C.byref(rid)))
            sizes = (0, request.shots, 0)
        elif isinstance(request, VqeStepRequest):
            sid = self._session(request.session)
            check(load().qm_serve_submit_vqe_step(self._h, sid, C.byref(rid)))
            p = request.session.circuit.ParameterCount
            sizes = (p, 0, p)
        else:
            raise ArgumentError("unknown request")
        return ServeFuture(self, request, rid.value, sizes)

    def stats(self) -> dict:
        st = _lib.ServeStats()
        check(load().qm_serve_get_stats(self._h, C.byref(st)))
        return {name: getattr(st, name) for name, _ in _lib.ServeStats._fields_}

    def close(self) -> None:
        if self._h is None:
            return
        # sessions whose last results were never taken still get their parameters back
        for key, sid in self._sessions.items():
            s = self._session_objects[key]
            params = np.zeros(max(1, s.circuit.ParameterCount))
            steps = C.c_int64()
            if load().qm_serve_session_parameters(self._h, sid, params.ctypes.data_as(_lib.DP), len(params),
                                                  C.byref(steps)) == 0 and steps.value > s.steps:
                s.parameters, s.steps = params[:s.circuit.ParameterCount].copy(), steps.value
        load().qm_serve_destroy(self._h)
        self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()

    def __del__(self):
        try:
            self.close()
        except Exception:
            pass


def serve_plain(requests: Sequence, context: B200Context,
                arrivals: Sequence[float] | None = None, clock: Callable[[], float] = time.perf_counter) -> list[Response]:
    """The plain form: one request at a time in arrival order, FP64 as given, a fresh device
    state per circuit, and a VQE step evaluated one circuit at a time (its base circuit and
    each parameter-shifted circuit bound on the host and run on a resident state)."""
    out = []
    t0 = clock()
    for i, req in enumerate(requests):
        if arrivals is not None:
            wait = t0 + arrivals[i] - clock()
            if wait > 0:
                time.sleep(wait)
        submitted = t0 + arrivals[i] if arrivals is not None else clock()
        started = clock()
        if isinstance(req, VqeStepRequest):
            s = req.session
            r = _plain_vqe(s, context)
        else:
            with DeviceState(context, req.qubits, req.precision) as st:
                st.Evolve(req.circuit)
                if isinstance(req, ExpectationRequest):
                    values, mass = st.ExpectationValues(list(req.observables))
                    r = Response("expectation", values=values, mass=mass)
                else:
                    outcomes, _ = st.Sample(random_doubles(req.seed, req.shots))
                    r = Response("shots", outcomes=outcomes)
        r.submitted, r.started, r.finished = submitted, started, clock()
        out.append(r)
    return out


def _plain_vqe(s: VqeSession, context: B200Context) -> Response:
    """Energy and occurrence-wise parameter-shift gradient, one circuit at a time on a resident state."""
    from .observables import PauliTerm
    h = PauliHamiltonian(s.hamiltonian.QubitCount,
                         [PauliTerm(float(c), t.Observable) for c, t in zip(s.coefficients, s.hamiltonian.Terms)])
    params = list(s.parameters)
    grad = np.zeros(s.circuit.ParameterCount)
    with DeviceState(context, s.circuit.QubitCount, s.precision) as st:
        st.Evolve(s.circuit.Bind(params))
        energy = st.ExpectationEnergy(h)
        for r_idx, p in enumerate(s.circuit.RotationParameterIndices):
            e = []
            for shift in (math.pi / 2, -math.pi / 2):
                st.Reset()
                st.Evolve(s.circuit.BindWithRotationShift(params, r_idx, shift))
                e.append(st.ExpectationEnergy(h))
            grad[p] += 0.5 * e[0] - 0.5 * e[1]
    new = np.array([_fma(-s.step_size, float(g), float(x)) for g, x in zip(grad, s.parameters)])
    s.parameters = new
    s.steps += 1
    return Response("vqe_step", energy=energy, gradient=grad, parameters=new.copy())
