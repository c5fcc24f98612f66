"""The request server on the GPU: results in a concurrent, batched mix equal results alone."""
from __future__ import annotations

import numpy as np
import pytest

import oracle as orc
from quantummatter_b200.backend import FP32, FP64
from quantummatter_b200.observables import PauliString
from quantummatter_b200.serving import (B200Server, ExpectationRequest, ShotsRequest, VqeSession, VqeStepRequest,
                                        serve_plain, state_bytes)
from quantummatter_b200.variational import B200VariationalEnergyEvaluator
from quantummatter_b200.workloads import brick_circuit, hardware_efficient_ansatz, tfim_chain

pytestmark = pytest.mark.gpu


def observables(n, seed):
    rng = np.random.default_rng(seed)
    obs = [PauliString("".join("Z" if q == i else "I" for q in reversed(range(n)))) for i in range(n)]
    obs += [PauliString("".join(rng.choice(list("IXYZ"), size=n))) for _ in range(6)]
    return obs


def make_requests(precision=FP64):
    reqs = []
    for i, n in enumerate([9, 12, 10, 11, 12, 9]):
        reqs.append(ExpectationRequest(brick_circuit(n, 6, seed=i), observables(n, i), precision))
        reqs.append(ShotsRequest(brick_circuit(n, 5, seed=100 + i), shots=300, seed=i, precision=precision))
    return reqs


def make_sessions(precision=FP64):
    out = []
    for i, n in enumerate([10, 10, 10, 11, 10]):
        c = hardware_efficient_ansatz(n, 2)
        params = np.random.default_rng(i).uniform(-np.pi, np.pi, c.ParameterCount)
        out.append(VqeSession(c, tfim_chain(n, seed=i), params, step_size=0.05, precision=precision))
    return out


def run(server, requests, sessions, steps=2):
    futures = [server.submit(r) for r in requests]
    vqe = []
    for _ in range(steps):
        vqe.append([server.submit(VqeStepRequest(s)) for s in sessions])
    return [f.result(timeout=300) for f in futures], [[f.result(timeout=300) for f in row] for row in vqe]


@pytest.mark.parametrize("precision", [FP64, FP32])
def test_mixed_results_equal_alone(gpu_context, precision):
    reqs, sessions = make_requests(precision), make_sessions(precision)
    budget = 6 * state_bytes(12, FP64)
    with B200Server(workers=3, budget_bytes=budget, context_budget_bytes=2 << 30, cache_bytes=1 << 28) as server:
        mixed, mixed_vqe = run(server, reqs, sessions)
        stats = server.stats()
        assert 0 < stats["peak_reserved_bytes"] <= budget
        assert stats["completed"] == len(reqs) + 2 * len(sessions) and stats["max_batch"] >= 2
    assert max(r.batch for row in mixed_vqe for r in row) >= 2  # VQE steps were batched
    alone_sessions = make_sessions(precision)
    with B200Server(workers=1, budget_bytes=budget, context_budget_bytes=2 << 30) as server:
        alone = [server.submit(r).result(timeout=300) for r in reqs]
        alone_vqe = []
        for _ in range(2):
            alone_vqe.append([server.submit(VqeStepRequest(s)).result(timeout=300) for s in alone_sessions])
    for m, a in zip(mixed, alone):
        if m.kind == "expectation":
            assert np.array_equal(m.values, a.values) and m.mass == a.mass
        else:
            assert np.array_equal(m.outcomes, a.outcomes) and m.counts == a.counts
    for row_m, row_a in zip(mixed_vqe, alone_vqe):
        for m, a in zip(row_m, row_a):
            assert m.energy == a.energy
            assert np.array_equal(m.gradient, a.gradient)
            assert np.array_equal(m.parameters, a.parameters)
    for s, t in zip(sessions, alone_sessions):
        assert s.steps == t.steps == 2 and np.array_equal(s.parameters, t.parameters)


def test_served_values_match_the_oracle_and_the_plain_form(gpu_context):
    reqs = make_requests(FP64)[:4]
    sessions = make_sessions(FP64)[:2]
    with B200Server(workers=2, budget_bytes=1 << 30, context_budget_bytes=2 << 30) as server:
        served, served_vqe = run(server, reqs, sessions, steps=1)
    req = reqs[0]
    psi = orc.execute(req.circuit)
    want = np.array([orc.expectation(psi, o) for o in req.observables])
    assert np.max(np.abs(served[0].values - want)) <= 1e-12
    plain = serve_plain(reqs, gpu_context)
    for s, p in zip(served, plain):
        if s.kind == "expectation":
            assert np.array_equal(s.values, p.values)
        else:
            assert np.array_equal(s.outcomes, p.outcomes)
    # the plain VQE step (one circuit at a time) against the batched one
    fresh = make_sessions(FP64)[:2]
    for s, r in zip(fresh, served_vqe[0]):
        p = serve_plain([VqeStepRequest(s)], gpu_context)[0]
        assert abs(p.energy - r.energy) <= 1e-12
        assert np.max(np.abs(p.gradient - r.gradient)) <= 1e-11
    # and the evaluator's own coefficients give the same energy as the per-vector ones
    s = make_sessions(FP64)[0]
    e = B200VariationalEnergyEvaluator(gpu_context).EvaluateBatch(s.circuit, s.hamiltonian, s.parameters).Energies[0]
    assert e == served_vqe[0][0].energy
