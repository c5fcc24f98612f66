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

Admission: a request reserves the bytes of its state (16 * 2^n for FP64, 8 * 2^n for FP32)
against the server's budget and waits until the reservation fits; the oldest waiting request
goes first, and a younger one may pass it only while the older one does not fit.
Batching: waiting VQE steps whose ansatz structure, Hamiltonian Pauli strings and precision
match are evaluated as one device batch (qm_vqe_evaluate_coefficients), each with its own
Hamiltonian coefficients and parameters; a session never has two steps in flight.
Execution: each worker thread owns a B200Context (its own CUDA stream), so requests on
different workers overlap on the GPU; a worker keeps the device states of recent sizes for
reuse instead of allocating one per request.
"""
from __future__ import annotations

import math
import threading
import time
from collections import deque
from concurrent.futures import Future
from dataclasses import dataclass, field
from typing import Callable, Sequence

import numpy as np

from .backend import FP32, FP64, B200BackendOptions, B200Context, DeviceState
from .circuit import QuantumCircuit
from .errors import ArgumentError, ArgumentOutOfRangeError
from .observables import PauliHamiltonian, PauliString
from .trajectories import random_doubles
from .variational import B200VariationalEnergyEvaluator, ParameterizedCircuit, _fma


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
        self.busy = False
        # requests of sessions with the same key share a device batch
        self.key = (circuit.QubitCount, precision, _template_key(circuit),
                    tuple((t.Observable.FlipMask, t.Observable.SignMask, t.Observable.YCount) for t in hamiltonian.Terms))
        self.coefficients = np.array([t.Coefficient for t in hamiltonian.Terms], dtype=np.float64)


def _template_key(circuit: ParameterizedCircuit) -> tuple:
    ops = []
    for op in circuit.Operations:
        g = op.Operation
        u = None if g.Unitary is None else (g.Unitary.M00, g.Unitary.M01, g.Unitary.M10, g.Unitary.M11)
        ops.append((int(g.Kind), g.Target, g.Control, g.SecondControl, g.Angle if op.ParameterIndex < 0 else None,
                    op.ParameterIndex, u))
    return (circuit.ParameterCount, tuple(ops))


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


@dataclass
class _Item:
    request: object
    future: Future
    submitted: float
    bytes: int


@dataclass
class Job:
    items: list[_Item]
    bytes: int = 0
    kind: str = ""


class Scheduler:
    """Admission and batching policy (no device work; thread-unsafe, the server locks it)."""

    def __init__(self, budget_bytes: int, max_batch: int = 64, lookahead: int = 64):
        if budget_bytes <= 0:
            raise ArgumentOutOfRangeError("budget_bytes")
        self.budget = int(budget_bytes)
        self.max_batch = max_batch
        self.lookahead = lookahead
        self.reserved = 0
        self.peak_reserved = 0
        self.queue: deque[_Item] = deque()

    def push(self, item: _Item) -> None:
        if item.bytes > self.budget:
            raise ArgumentOutOfRangeError(f"the request needs {item.bytes} bytes; the budget is {self.budget} bytes")
        self.queue.append(item)

    def _fits(self, item: _Item) -> bool:
        return self.reserved + item.bytes <= self.budget

    def _ready(self, item: _Item) -> bool:
        req = item.request
        return not (isinstance(req, VqeStepRequest) and req.session.busy)

    def take(self) -> Job | None:
        """The next job: the oldest ready request that fits (younger ones pass only while the
        oldest does not fit), plus, for a VQE step, the waiting steps that share its batch key."""
        pick = None
        for idx, item in enumerate(self.queue):
            if idx >= self.lookahead:
                break
            if self._ready(item) and self._fits(item):
                pick = idx
                break
        if pick is None:
            return None
        head = self.queue[pick]
        del self.queue[pick]
        job = Job([head], head.bytes, _kind(head.request))
        if isinstance(head.request, VqeStepRequest):
            head.request.session.busy = True
            key = head.request.session.key
            rest = deque()
            while self.queue:
                item = self.queue.popleft()
                req = item.request
                if (len(job.items) < self.max_batch and isinstance(req, VqeStepRequest) and req.session.key == key
                        and self._ready(item) and self.reserved + job.bytes + item.bytes <= self.budget):
                    req.session.busy = True
                    job.items.append(item)
                    job.bytes += item.bytes
                else:
                    rest.append(item)
            self.queue = rest
        self.reserved += job.bytes
        self.peak_reserved = max(self.peak_reserved, self.reserved)
        return job

    def release(self, job: Job) -> None:
        self.reserved -= job.bytes
        for item in job.items:
            if isinstance(item.request, VqeStepRequest):
                item.request.session.busy = False


def _kind(req) -> str:
    return {ExpectationRequest: "expectation", ShotsRequest: "shots", VqeStepRequest: "vqe_step"}[type(req)]


class _Worker:
    """Executes jobs on its own context; keeps device states of recent sizes."""

    def __init__(self, context: B200Context, cache_bytes: int):
        self.context = context
        self.cache_bytes = cache_bytes
        self.states: dict[tuple[int, int], DeviceState] = {}
        self.evaluators: dict[int, B200VariationalEnergyEvaluator] = {}

    def state(self, qubits: int, precision: int) -> DeviceState:
        key = (qubits, precision)
        st = self.states.pop(key, None)
        if st is None:
            while self.states and sum(state_bytes(q, p) for q, p in self.states) + state_bytes(qubits, precision) > self.cache_bytes:
                _, old = self.states.popitem()
                old.Dispose()
            st = DeviceState(self.context, qubits, precision)
        else:
            st.Reset()
        self.states[key] = st  # most recently used last
        return st

    def run(self, job: Job) -> list[Response]:
        now = time.perf_counter()
        if job.kind == "vqe_step":
            return self._vqe(job, now)
        item = job.items[0]
        req = item.request
        st = self.state(req.qubits, req.precision)
        st.Evolve(req.circuit)
        if job.kind == "expectation":
            values, mass = st.ExpectationValues(list(req.observables))
            return [Response("expectation", values=values, mass=mass, started=now)]
        draws = random_doubles(req.seed, req.shots)
        outcomes, _ = st.Sample(draws)
        counts: dict[str, int] = {}
        for o in outcomes:
            k = format(int(o), "b").zfill(req.qubits)
            counts[k] = counts.get(k, 0) + 1
        return [Response("shots", outcomes=outcomes, counts=dict(sorted(counts.items())), started=now)]

    def _vqe(self, job: Job, now: float) -> list[Response]:
        sessions = [item.request.session for item in job.items]
        s0 = sessions[0]
        ev = self.evaluators.get(s0.precision)
        if ev is None:
            ev = self.evaluators[s0.precision] = B200VariationalEnergyEvaluator(self.context, s0.precision)
        params = np.stack([s.parameters for s in sessions])
        coef = np.stack([s.coefficients for s in sessions])
        r = ev.EvaluateBatch(s0.circuit, s0.hamiltonian, params, withGradient=True, coefficients=coef)
        out = []
        for i, s in enumerate(sessions):
            g = r.Gradients[i]
            s.parameters = np.array([_fma(-s.step_size, float(gi), float(pi)) for gi, pi in zip(g, s.parameters)])
            s.steps += 1
            out.append(Response("vqe_step", energy=float(r.Energies[i]), gradient=g.copy(),
                                parameters=s.parameters.copy(), batch=len(sessions), started=now))
        return out


class B200Server:
    """Serves requests from `workers` threads, each with its own context and stream."""

    def __init__(self, workers: int = 4, budget_bytes: int = 64 << 30, max_batch: int = 64,
                 context_budget_bytes: int = 32 << 30, cache_bytes: int = 8 << 30, device_index: int = 0,
                 contexts: Sequence[B200Context] | None = None):
        if workers < 1:
            raise ArgumentOutOfRangeError("workers")
        self.scheduler = Scheduler(budget_bytes, max_batch)
        self._cv = threading.Condition()
        self._closed = False
        own = contexts is None
        if own:
            contexts = [B200Context(B200BackendOptions(DeviceIndex=device_index,
                                                       DeviceMemoryBudgetBytes=context_budget_bytes,
                                                       StagingMemoryBudgetBytes=1 << 30))
                        for _ in range(workers)]
        self._own = own
        self._workers = [_Worker(c, cache_bytes) for c in contexts]
        self._threads = [threading.Thread(target=self._loop, args=(w,), daemon=True) for w in self._workers]
        self.completed = 0
        for t in self._threads:
            t.start()

    def submit(self, request) -> Future:
        if not isinstance(request, (ExpectationRequest, ShotsRequest, VqeStepRequest)):
            raise ArgumentError("unknown request")
        fut: Future = Future()
        item = _Item(request, fut, time.perf_counter(), state_bytes(request.qubits, request.precision))
        with self._cv:
            if self._closed:
                raise ArgumentError("the server is closed")
            self.scheduler.push(item)
            self._cv.notify_all()
        return fut

    def _loop(self, worker: _Worker) -> None:
        while True:
            with self._cv:
                job = None
                while not self._closed:
                    job = self.scheduler.take()
                    if job is not None:
                        break
                    self._cv.wait()
                if job is None:
                    return
            try:
                responses = worker.run(job)
                error = None
            except Exception as e:  # the request's caller sees the failure
                responses, error = None, e
            done = time.perf_counter()
            with self._cv:
                self.scheduler.release(job)
                self.completed += len(job.items)
                self._cv.notify_all()
            for i, item in enumerate(job.items):
                if error is not None:
                    item.future.set_exception(error)
                    continue
                r = responses[i]
                r.submitted = item.submitted
                r.finished = done
                item.future.set_result(r)

    def close(self) -> None:
        with self._cv:
            self._closed = True
            self._cv.notify_all()
        for t in self._threads:
            t.join()
        for w in self._workers:
            for st in w.states.values():
                st.Dispose()
            w.states.clear()
        if self._own:
            for w in self._workers:
                w.context.Dispose()

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


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
