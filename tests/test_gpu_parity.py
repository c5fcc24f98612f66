"""Parity of the CUDA library (through its C ABI) with the CPU oracle.  Runs on a B200.

FP64 tolerances are the reference's: 1e-12 for gate columns, 2e-12 / 3e-12 for random dense
circuits (StateVectorBackendConformanceTests.cs:146-245, CudaBackendTests.cs:145-184), 1e-12
max |delta amplitude| for the 20-qubit brick circuit, 5e-12 for energies
(VariationalEnergyTests.cs:293).  FP32 states are checked against the FP64 oracle with the
tolerance stated in each test.
"""
from __future__ import annotations

import math
import threading

import numpy as np
import pytest

import oracle as orc
from circuits import random_circuit, random_state
from conftest import golden_circuits, golden_hamiltonians, known_answers
from quantummatter_b200.backend import (FP32, FP64, B200BackendOptions, B200NoiseChannelBackend,
                                        B200StateVectorBackend, CancellationToken, DeviceState, Plan)
from quantummatter_b200.circuit import GateKind, GateOperation, QuantumCircuit
from quantummatter_b200.errors import (ArgumentError, BudgetExceededError, MassError, OperationCanceledError)
from quantummatter_b200.observables import PauliHamiltonian, PauliString, PauliTerm
from quantummatter_b200.workloads import brick_circuit

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def backend(gpu_context):
    return B200StateVectorBackend(context=gpu_context)


def run_host(backend, circuit, state=None):
    s = orc.zero_state(circuit.QubitCount) if state is None else np.array(state, dtype=np.complex128)
    backend.Execute(circuit, s)
    return s


def test_known_columns_on_every_target(backend):
    ka = known_answers()
    for name, inp, zero, one in ka["columns"]:
        for target in range(4):
            c = QuantumCircuit(4)
            spectators = 15 ^ (1 << target)
            for q in range(4):
                if q != target or inp == 1:
                    c.X(q)
            c.AppendValidated(GateOperation(GateKind[name], target, -1, ka["angle"]))
            s = run_host(backend, c)
            for index in range(16):
                expected = complex(*zero) if index == spectators else complex(*one) if index == 15 else 0
                assert abs(s[index] - expected) <= 1e-12


def test_dense_fixtures_through_the_drop_in_port(backend):
    for circuit, initial, final in golden_circuits():
        assert np.max(np.abs(run_host(backend, circuit, initial) - final)) <= 2e-12


@pytest.mark.parametrize("width", [1, 9, 10, 11, 12])
def test_random_circuits_fp64_match_the_oracle(gpu_context, width):
    for seed, n in ((0, 12), (1, 13), (2, 14)):
        c = random_circuit(n, 300, seed=900 + seed)
        psi = random_state(n, seed)
        with DeviceState(gpu_context, n, FP64) as st:
            st.Upload(psi)
            st.Evolve(c, fusion_width=width)
            got = st.Download()
        assert np.max(np.abs(got - orc.execute(c, psi))) <= 3e-12


@pytest.mark.parametrize("width", [9, 12])
def test_diagonal_heavy_circuits_match_the_oracle(gpu_context, width):
    """Groups of commuting phases and CZ/Z negates applied as one phase per register."""
    from test_abi import diagonal_heavy_circuit
    for seed, n in ((0, 12), (1, 14)):
        c = diagonal_heavy_circuit(n, 400, seed)
        psi = random_state(n, seed)
        for precision, tol in ((FP64, 3e-12), (FP32, 5e-5)):
            with DeviceState(gpu_context, n, precision) as st:
                st.Upload(psi)
                st.Evolve(c, fusion_width=width)
                got = st.Download()
            assert np.max(np.abs(got - orc.execute(c, psi))) <= tol, precision


def test_brick_20_qubits_matches_the_oracle_within_1e12(gpu_context):
    """20 qubits, depth 20: 400 U3 + 190 CNOT from |0...0>, full 2^20-amplitude vector."""
    c = brick_circuit(20, 20)
    want = orc.execute(c)
    for width in (0, 1):
        with DeviceState(gpu_context, 20, FP64) as st:
            st.Evolve(c, fusion_width=width)
            got = st.Download()
        assert np.max(np.abs(got - want)) <= 1e-12, width


def test_brick_20_qubits_fp32_error_against_fp64_oracle(gpu_context):
    c = brick_circuit(20, 20)
    want = orc.execute(c)
    with DeviceState(gpu_context, 20, FP32) as st:
        st.Evolve(c)
        got = st.Download()
    err = float(np.max(np.abs(got - want)))
    assert err <= 2e-6, err  # FP32 amplitudes after 590 gates: ~1e-7 typical


def test_plan_reuse_and_stats(gpu_context):
    c = brick_circuit(16, 10)
    p = Plan(gpu_context, c, FP64, 0)
    passes, launches, planned = p.stats()
    assert passes == launches and planned == passes * 2 * (16 << 16)
    with DeviceState(gpu_context, 16, FP64) as st:
        p.execute(st)
        p.execute(st)
        got = st.Download()
    want = orc.execute(c, orc.execute(c))
    assert np.max(np.abs(got - want)) <= 1e-12
    p.Dispose()


def test_offset_buffers_keep_their_sentinels(backend):
    """CudaBackendTests.cs:145-184: a state inside a larger array; neighbours stay untouched."""
    for n in (3, 9, 12, 17):
        c = random_circuit(n, 60, seed=n)
        psi = random_state(n, n)
        big = np.full((1 << n) + 64, 7 - 3j, dtype=np.complex128)
        view = big[32:32 + (1 << n)]
        view[:] = psi
        backend.Execute(c, view)
        assert np.all(big[:32] == 7 - 3j) and np.all(big[-32:] == 7 - 3j)
        assert np.max(np.abs(view - orc.execute(c, psi))) <= 3e-12


def test_budget_rejection_leaves_the_input_unchanged(gpu_context):
    small = B200StateVectorBackend(B200BackendOptions(DeviceMemoryBudgetBytes=1024, StagingMemoryBudgetBytes=1024))
    try:
        psi = random_state(7, 1)
        before = psi.copy()
        with pytest.raises(BudgetExceededError):
            small.Execute(QuantumCircuit(7).H(0), psi)
        assert np.array_equal(psi, before)
        ok = random_state(6, 1)
        small.Execute(QuantumCircuit(6).H(0), ok)  # 1024 bytes fit: the backend is still usable
        assert np.max(np.abs(ok - orc.execute(QuantumCircuit(6).H(0), random_state(6, 1)))) <= 1e-15
    finally:
        small.Dispose()


def test_cancellation_and_bad_length_leave_the_input_unchanged(backend):
    psi = random_state(10, 2)
    before = psi.copy()
    token = CancellationToken()
    token.Cancel()
    with pytest.raises(OperationCanceledError):
        backend.Execute(random_circuit(10, 50, 1), psi, token)
    assert np.array_equal(psi, before)
    with pytest.raises(ArgumentError):
        backend.Execute(QuantumCircuit(9).H(0), psi)
    assert np.array_equal(psi, before)


def test_concurrent_callers_on_one_backend(backend):
    """CudaBackendTests.cs:239-256: eight concurrent callers on independent buffers."""
    results, errors = {}, []

    def work(i):
        try:
            c = random_circuit(11, 80, seed=300 + i)
            psi = random_state(11, i)
            s = psi.copy()
            backend.Execute(c, s)
            results[i] = np.max(np.abs(s - orc.execute(c, psi)))
        except Exception as exc:  # pragma: no cover - reported below
            errors.append(exc)

    threads = [threading.Thread(target=work, args=(i,)) for i in range(8)]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors and len(results) == 8 and max(results.values()) <= 3e-12


def test_profiled_execution_reports_launches(gpu_context):
    b = B200StateVectorBackend(B200BackendOptions(EnableProfiling=True, FusionWidth=1))
    try:
        c = QuantumCircuit(12).H(0).I(1).X(2).CNot(2, 3).Rz(4, 0.2)
        prof = b.ExecuteProfiled(c, orc.zero_state(12))
        assert prof.KernelLaunches == 4 and prof.StateBytes == 16 << 12 and prof.DeviceEvolutionSeconds > 0
    finally:
        b.Dispose()


# ---------------------------------------------------------------- observables

def test_expectations_match_the_oracle(gpu_context):
    import itertools
    for n in (1, 2, 3, 10, 13):
        psi = random_state(n, 40 + n) * 1.3
        if n <= 3:
            labels = ["".join(p) for p in itertools.product("IXYZ", repeat=n)]
        else:
            rng = np.random.default_rng(n)
            labels = ["".join(rng.choice(list("IXYZ"), size=n)) for _ in range(40)]
        obs = [PauliString(lab) for lab in labels]
        with DeviceState(gpu_context, n, FP64) as st:
            st.Upload(psi)
            vals, mass = st.ExpectationValues(obs)
        assert abs(mass - np.vdot(psi, psi).real) <= 1e-12 * mass
        want = np.array([orc.expectation(psi, o) for o in obs])
        assert np.max(np.abs(vals - want)) <= 1e-12


def test_energies_match_fixtures_and_cancellation(gpu_context):
    for h, psi, energy, per_term in golden_hamiltonians():
        with DeviceState(gpu_context, h.QubitCount, FP64) as st:
            st.Upload(psi)
            assert abs(st.ExpectationEnergy(h) - energy) <= 5e-12
    with DeviceState(gpu_context, 1, FP64) as st:
        canceling = PauliHamiltonian(1, [PauliTerm(1e16, PauliString("I")), PauliTerm(1, PauliString("I")),
                                         PauliTerm(-1e16, PauliString("I"))])
        assert st.ExpectationEnergy(canceling) == 1
        assert st.ExpectationEnergy(PauliHamiltonian(1, [])) == 0
        st.Upload(np.array([0, 0], dtype=np.complex128))
        with pytest.raises(MassError):
            st.ExpectationEnergy(PauliHamiltonian(1, []))
        st.Upload(np.array([float("nan"), 0], dtype=np.complex128))
        with pytest.raises(MassError):
            st.ExpectationEnergy(PauliHamiltonian(1, [PauliTerm(0, PauliString("Z"))]))


# ---------------------------------------------------------------- noise

class FixedRandom:
    def __init__(self, *values):
        self.values = list(values)
        self.used = 0

    def NextDouble(self):
        v = self.values[self.used]
        self.used += 1
        return v


def test_noise_port_matches_the_oracle_and_draw_counts(gpu_context):
    nb = B200NoiseChannelBackend(context=gpu_context)
    from quantummatter_b200.noise import NoiseChannel
    for n in (1, 3, 11):
        psi = random_state(n, 70 + n)
        for t in range(n):
            for kind, p, draws in ((2, 1.0, [0.0]), (2, 1.0, [0.3]), (2, 1.0, [0.6]), (2, 1.0, [0.9]),
                                   (0, 0.5, [0.1]), (1, 0.5, [0.2]), (0, 1.0, []), (3, 0.37, [0.0]),
                                   (3, 0.37, [0.99]), (0, 0.0, [])):
                s = psi.copy()
                rnd = FixedRandom(*draws)
                nb.Apply(NoiseChannel(kind, p), t, s, rnd)
                want, used = orc.noise_apply(kind, p, t, psi, draws)
                assert rnd.used == used
                assert np.max(np.abs(s - want)) <= 2e-12


def test_device_masses_match_the_oracle(gpu_context):
    for n in (1, 5, 16):
        psi = random_state(n, 5 * n) * 0.7
        with DeviceState(gpu_context, n, FP64) as st:
            st.Upload(psi)
            for t in range(n):
                m0, m1 = st.QubitMasses(t)
                w0, w1 = orc.qubit_masses(psi, t)
                assert abs(m0 - w0) <= 1e-15 and abs(m1 - w1) <= 1e-15


# ---------------------------------------------------------------- sampling

def test_sampling_matches_the_oracle_with_the_same_draws(gpu_context):
    for n in (2, 10, 17):
        psi = random_state(n, 90 + n)
        psi[psi.size // 3: psi.size // 3 + 5] = 0  # a zero plateau
        rnd = orc.DotNetRandom(n)
        draws = [rnd.NextDouble() for _ in range(1000)]
        with DeviceState(gpu_context, n, FP64) as st:
            st.Upload(psi)
            got, ambiguous = st.Sample(draws)
        want = orc.sample(psi, draws)
        assert ambiguous == 0
        assert np.array_equal(got, want)


def test_measure_all_collapses_like_the_oracle(gpu_context):
    psi = random_state(12, 3)
    for u in (0.0, 0.31, 0.77, 0.999999):
        with DeviceState(gpu_context, 12, FP64) as st:
            st.Upload(psi)
            k, amb = st.MeasureAll(u)
            got = st.Download()
        want_state, want_k = orc.measure_all(psi, u)
        assert k == want_k and not amb
        assert np.array_equal(got, want_state)


@pytest.mark.parametrize("precision,width,tol", [(FP64, 9, 1e-12), (FP64, 11, 1e-12), (FP32, 13, 2e-5)],
                         ids=["fp64-k9", "fp64-k11", "fp32-k13"])
def test_relabeling_plans_at_other_block_widths(gpu_context, precision, width, tol):
    """Relabeling passes at explicit fusion widths: one-shot (the interpreter runs passes not yet
    compiled) and as a compiled plan, against the oracle."""
    c = random_circuit(20, 400, seed=41)
    psi = random_state(20, 3)
    want = orc.execute(c, psi)
    for compiled in (False, True):
        with DeviceState(gpu_context, 20, precision) as st:
            st.Upload(psi)
            if compiled:
                p = Plan(gpu_context, c, precision, width)
                p.execute(st)
                p.Dispose()
            else:
                st.Evolve(c, fusion_width=width)
            got = st.Download()
        assert np.max(np.abs(got - want)) <= tol, (compiled, width)


@pytest.mark.parametrize("n", [21, 24])
def test_pageable_host_buffers_match_page_locked_ones(gpu_context, n):
    """Whole-state copies from pageable host memory of 16 MiB and more move through the
    context's page-locked bounce buffers (one partial 64 MiB chunk at 21 qubits, four at 24);
    the results are bit-identical to the same calls on a page-locked buffer, for the drop-in
    port, the noise port and a device state's upload and download."""
    from quantummatter_b200.noise import NoiseChannel
    psi = random_state(n, 90 + n)
    circuit = brick_circuit(n, 2, seed=n)
    backend = B200StateVectorBackend(context=gpu_context)
    noise = B200NoiseChannelBackend(context=gpu_context)
    pinned = gpu_context.host_array(1 << n)
    try:
        results = []
        for buffer in (pinned.array, np.empty(1 << n, dtype=np.complex128)):
            buffer[:] = psi
            backend.Execute(circuit, buffer)
            noise.Apply(NoiseChannel(3, 0.37), n - 1, buffer, FixedRandom(0.5))
            with DeviceState(gpu_context, n, FP64) as st:
                st.Upload(buffer)
                out = st.Download(np.empty_like(buffer))
            results.append((buffer.copy(), out))
        (a, a_round), (b, b_round) = results
        assert np.array_equal(a, b) and np.array_equal(a_round, a) and np.array_equal(b_round, b)
        if n == 21:
            want, _ = orc.noise_apply(3, 0.37, n - 1, orc.execute(circuit, psi), [0.5])
            assert np.max(np.abs(b - want)) <= 1e-12
    finally:
        pinned.free()


# ---------------------------------------------------------------- full-size properties

def test_30_qubit_brick_round_trip_and_norm(gpu_context):
    """Size-independent checks at the 30-qubit size: the circuit followed by its inverse returns
    |0...0> and the norm stays 1.  Also runs the 28-qubit fused path against the per-gate path."""
    from test_oracle_pinning import _inverse
    c = brick_circuit(30, 40)
    with DeviceState(gpu_context, 30, FP64) as st:
        st.Evolve(c)
        _, mass = st.ExpectationValues([])
        assert abs(mass - 1) <= 1e-11
        st.Evolve(_inverse(c))
        vals, mass = st.ExpectationValues([PauliString("Z" * 30)])
        assert abs(vals[0] - 1) <= 1e-10 and abs(mass - 1) <= 1e-11
        m0, _ = st.QubitMasses(29)
        assert abs(m0 - 1) <= 1e-10
    c = brick_circuit(26, 12)
    with DeviceState(gpu_context, 26, FP64) as a, DeviceState(gpu_context, 26, FP64) as b:
        a.Evolve(c, fusion_width=0)
        b.Evolve(c, fusion_width=1)
        diff = np.max(np.abs(a.Download() - b.Download()))
    assert diff <= 1e-12


def test_30_qubit_brick_round_trip_through_compiled_plans(gpu_context):
    """The headline path at its own size: the 30-qubit brick and its inverse as plans, whose passes
    are compiled for their op sequence (rotations between deferred phases, phases carried from
    pass to pass, the next tile copied during the last exchange).  The round trip returns |0...0>
    and the norm stays 1 after the forward circuit."""
    from quantummatter_b200.backend import Plan, jit_info
    from test_oracle_pinning import _inverse
    c = brick_circuit(30, 40)
    before = jit_info()
    fwd, back = Plan(gpu_context, c, FP64), Plan(gpu_context, _inverse(c), FP64)
    try:
        with DeviceState(gpu_context, 30, FP64) as st:
            fwd.execute(st)
            _, mass = st.ExpectationValues([])
            assert abs(mass - 1) <= 1e-11
            back.execute(st)
            vals, mass = st.ExpectationValues([PauliString("Z" * 30)])
            assert abs(vals[0] - 1) <= 1e-10 and abs(mass - 1) <= 1e-11
            m0, _ = st.QubitMasses(0)
            assert abs(m0 - 1) <= 1e-10
    finally:
        fwd.Dispose()
        back.Dispose()
    after = jit_info()
    if before["available"]:
        assert after["failed"] == before["failed"] and after["launches"] > before["launches"]
