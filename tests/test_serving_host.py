"""Admission and batching policy of the request server (no GPU)."""
from __future__ import annotations

from concurrent.futures import Future

import numpy as np
import pytest

from quantummatter_b200.backend import FP32, FP64
from quantummatter_b200.circuit import QuantumCircuit
from quantummatter_b200.errors import ArgumentOutOfRangeError
from quantummatter_b200.serving import (ExpectationRequest, Scheduler, ShotsRequest, VqeSession, VqeStepRequest,
                                        _Item, state_bytes)
from quantummatter_b200.workloads import hardware_efficient_ansatz, tfim_chain


def item(req, t=0.0):
    return _Item(req, Future(), t, state_bytes(req.qubits, req.precision))


def expectation(n, precision=FP64):
    return ExpectationRequest(QuantumCircuit(n).H(0), [], precision)


def session(n, seed, precision=FP64):
    c = hardware_efficient_ansatz(n, 1)
    return VqeSession(c, tfim_chain(n, seed), np.zeros(c.ParameterCount), precision=precision)


def test_reservations_never_exceed_the_budget():
    s = Scheduler(budget_bytes=state_bytes(12, FP64) * 3)
    for n in (12, 12, 11, 12, 10):
        s.push(item(expectation(n)))
    jobs = []
    while (j := s.take()) is not None:
        jobs.append(j)
        assert s.reserved <= s.budget
    # 12 + 12 + 11 fit; the fourth (12) waits, the 10-qubit one may pass it
    assert [j.items[0].request.qubits for j in jobs] == [12, 12, 11, 10]
    assert s.peak_reserved <= s.budget
    s.release(jobs[0])
    j = s.take()
    assert j.items[0].request.qubits == 12 and s.reserved <= s.budget
    assert s.take() is None


def test_oversized_requests_are_rejected():
    s = Scheduler(budget_bytes=state_bytes(10, FP64))
    with pytest.raises(ArgumentOutOfRangeError):
        s.push(item(expectation(11)))
    s.push(item(expectation(11, FP32)))  # 8 * 2^11 fits 16 * 2^10


def test_vqe_steps_batch_by_structure_and_sessions_serialise():
    s = Scheduler(budget_bytes=1 << 40, max_batch=3)
    a, b, c, d = session(6, 1), session(6, 2), session(6, 3), session(7, 4)
    e = session(6, 5, FP32)
    order = [VqeStepRequest(a), ShotsRequest(QuantumCircuit(6)), VqeStepRequest(b), VqeStepRequest(d),
             VqeStepRequest(a), VqeStepRequest(c), VqeStepRequest(e), VqeStepRequest(b)]
    for r in order:
        s.push(item(r))
    j1 = s.take()
    # a, b and c share structure and precision; a's second step waits for its first
    assert [it.request.session for it in j1.items] == [a, b, c]
    assert j1.kind == "vqe_step"
    j2 = s.take()
    assert j2.kind == "shots"
    j3 = s.take()
    assert [it.request.session for it in j3.items] == [d]
    j4 = s.take()
    assert [it.request.session for it in j4.items] == [e]  # FP32 session: its own batch
    assert s.take() is None  # a and b are busy
    s.release(j1)
    j5 = s.take()
    assert [it.request.session for it in j5.items] == [a, b]
    assert s.take() is None


def test_coefficients_differ_but_keys_match():
    a, b = session(8, 1), session(8, 2)
    assert a.key == b.key
    assert not np.array_equal(a.coefficients, b.coefficients)
