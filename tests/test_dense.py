"""Dense fused gates (fusion widths 2..6) against the oracle.

The conventional fusion scheme: gates merge into fused gates of at most k qubits, each a dense
2^m x 2^m unitary applied in one sweep of the state, with the tile staged through bulk copies.
Each width is checked against the scalar oracle (CpuStateVectorBackend restated) on random
circuits with controls, Toffolis, SWAPs and diagonals, and on the benchmark's brick circuit, at
sizes that take the single-CTA kernel (8 qubits), one tile (12), and many tiles with every
placement of the fused qubits relative to the tile's column bits (14, 20).
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle as orc
from circuits import random_circuit
from quantummatter_b200._lib import check, load
from quantummatter_b200.backend import FP32, FP64, DeviceState, Plan
from quantummatter_b200.circuit import QuantumCircuit, prepare
from quantummatter_b200.workloads import brick_circuit

QM_E_RANGE = 10


def random_state(n: int, seed: int) -> np.ndarray:
    re, im = np.random.default_rng(seed).standard_normal((2, 1 << n))
    psi = re + 1j * im
    return psi / np.linalg.norm(psi)


def plan_info(circuit: QuantumCircuit, precision: int, width: int) -> tuple[int, int, int]:
    """(status, passes, planned bytes) of qm_plan_program (host only)."""
    g, n = prepare(circuit)
    passes, ops = C.c_int32(-1), C.c_int32(-1)
    planned = C.c_int64(-1)
    rc = load().qm_plan_program(circuit.QubitCount, precision, g, n, width, C.byref(passes), None, 0, C.byref(ops),
                                None, 0, C.byref(planned))
    return rc, passes.value, planned.value


def test_widths_7_and_8_are_rejected():
    c = brick_circuit(12, 2)
    for width in (7, 8, 15, -1):
        rc, _, _ = plan_info(c, FP64, width)
        assert rc == QM_E_RANGE, width
        buf = C.create_string_buffer(256)
        load().qm_last_error(buf, 256)
        assert b"2..6" in buf.value


@pytest.mark.parametrize("width", [2, 3, 4, 5, 6])
def test_dense_plans_sweep_the_state_once_per_fused_gate(width):
    """Planned bytes: one read and one write of the state per fused gate (no gate of the brick is
    wider than two qubits), and wider fusion never needs more sweeps."""
    n = 20
    c = brick_circuit(n, 8)
    rc, passes, planned = plan_info(c, FP64, width)
    assert rc == 0 and passes == 0
    sweeps = planned // (2 * 16 << n)
    assert planned == sweeps * (2 * 16 << n)
    rc, _, narrower = plan_info(c, FP64, width - 1) if width > 2 else (0, 0, None)
    if narrower is not None:
        assert planned <= narrower
    # every fused gate of width >= 2 holds at least one CNOT and its two U3s, or is the tail
    assert sweeps <= len(c.Operations) // 2


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [(FP64, 1e-12), (FP32, 2e-6)])
@pytest.mark.parametrize("width", [2, 3, 4, 5, 6])
@pytest.mark.parametrize("n", [8, 12, 14, 20])
def test_dense_widths_match_the_oracle(gpu_context, n, width, precision, tol):
    c = random_circuit(n, 160, seed=1000 * width + n)
    psi = random_state(n, n + width)
    want = orc.execute(c, psi)
    with DeviceState(gpu_context, n, precision) as st:
        st.Upload(psi)
        st.Evolve(c, fusion_width=width)
        got = st.Download()
    assert np.max(np.abs(got - want)) <= tol


@pytest.mark.gpu
@pytest.mark.parametrize("precision,tol", [(FP64, 1e-12), (FP32, 2e-6)])
@pytest.mark.parametrize("width", [2, 4, 6])
def test_dense_brick_plan_matches_the_oracle(gpu_context, width, precision, tol):
    """The benchmark's brick structure through a persistent plan, 22 qubits (1024 tiles)."""
    n = 22
    c = brick_circuit(n, 6, seed=width)
    want = orc.execute_parallel(c)
    plan = Plan(gpu_context, c, precision, fusion_width=width)
    try:
        with DeviceState(gpu_context, n, precision) as st:
            plan.execute(st)
            got = st.Download()
    finally:
        plan.Dispose()
    assert np.max(np.abs(got - want)) <= tol


@pytest.mark.gpu
def test_dense_fused_gates_on_every_qubit_placement(gpu_context):
    """Fused gates whose qubits sit at the bottom, the top and scattered across a 16-qubit
    index, including placements where the copy run is two amplitudes."""
    n = 16
    rng = np.random.default_rng(3)
    for qubits in ([0, 1, 2, 3, 4, 5], [10, 11, 12, 13, 14, 15], [1, 3, 5, 7, 9, 11], [0, 5, 6, 12, 15],
                   [2, 3, 14], [0, 15]):
        c = QuantumCircuit(n)
        for _ in range(3):
            for q in qubits:
                c.Ry(q, float(rng.uniform(0, 6.28))).Rz(q, float(rng.uniform(0, 6.28)))
            for a, b in zip(qubits, qubits[1:]):
                c.CNot(a, b)
        psi = random_state(n, len(qubits))
        want = orc.execute(c, psi)
        for precision, tol in ((FP64, 1e-12), (FP32, 2e-6)):
            with DeviceState(gpu_context, n, precision) as st:
                st.Upload(psi)
                st.Evolve(c, fusion_width=len(qubits))
                assert np.max(np.abs(st.Download() - want)) <= tol, (qubits, precision)


def dense_launches() -> tuple[int, int]:
    """(dense fused-gate launches, of which on the tensor cores) since the library loaded."""
    a, b = C.c_int64(), C.c_int64()
    check(load().qm_dense_info(C.byref(a), C.byref(b)))
    return a.value, b.value


@pytest.mark.gpu
@pytest.mark.parametrize("width", [5, 6])
@pytest.mark.parametrize("n", [11, 12, 14, 20])
def test_tensor_core_dense_gates_match_the_oracle(gpu_context, monkeypatch, n, width):
    """Complex64 fused gates of 5 and 6 qubits on the tensor cores (tcgen05, 3xTF32 split,
    QM_DENSE_TC=1; 5-qubit gates widened by one qubit) against the oracle at the FP32 tolerance,
    with the tensor-core kernel shown to have run.  11 qubits is a single tile."""
    monkeypatch.setenv("QM_DENSE_TC", "1")
    c = random_circuit(n, 160, seed=7000 + 100 * width + n)
    psi = random_state(n, n + width + 50)
    want = orc.execute(c, psi)
    _, tc0 = dense_launches()
    with DeviceState(gpu_context, n, FP32) as st:
        st.Upload(psi)
        st.Evolve(c, fusion_width=width)
        got = st.Download()
    _, tc1 = dense_launches()
    assert tc1 > tc0
    assert np.max(np.abs(got - want)) <= 2e-6


@pytest.mark.gpu
def test_tensor_core_dense_gates_on_every_qubit_placement(gpu_context, monkeypatch):
    """Tensor-core fused gates whose qubits sit at the bottom (the tile contiguous along its
    columns), the top and scattered, and the benchmark's brick through a persistent plan."""
    monkeypatch.setenv("QM_DENSE_TC", "1")
    n = 16
    rng = np.random.default_rng(5)
    for qubits in ([0, 1, 2, 3, 4, 5], [10, 11, 12, 13, 14, 15], [1, 3, 5, 7, 9, 11], [0, 5, 6, 12, 15, 2],
                   [4, 5, 6, 7, 8]):
        c = QuantumCircuit(n)
        for _ in range(3):
            for q in qubits:
                c.Ry(q, float(rng.uniform(0, 6.28))).Rz(q, float(rng.uniform(0, 6.28)))
            for a, b in zip(qubits, qubits[1:]):
                c.CNot(a, b)
        psi = random_state(n, len(qubits) + 90)
        want = orc.execute(c, psi)
        _, tc0 = dense_launches()
        with DeviceState(gpu_context, n, FP32) as st:
            st.Upload(psi)
            st.Evolve(c, fusion_width=len(qubits))
            got = st.Download()
        assert dense_launches()[1] > tc0, qubits
        assert np.max(np.abs(got - want)) <= 2e-6, qubits
    n = 22
    c = brick_circuit(n, 6, seed=11)
    want = orc.execute_parallel(c)
    _, tc0 = dense_launches()
    plan = Plan(gpu_context, c, FP32, fusion_width=6)
    try:
        with DeviceState(gpu_context, n, FP32) as st:
            plan.execute(st)
            got = st.Download()
    finally:
        plan.Dispose()
    assert dense_launches()[1] > tc0
    assert np.max(np.abs(got - want)) <= 2e-6


@pytest.mark.gpu
@pytest.mark.parametrize("width", [5, 6])
@pytest.mark.parametrize("n", [12, 20])
def test_fp32_pipe_dense_gates_match_the_oracle(gpu_context, monkeypatch, n, width):
    """With QM_DENSE_TC=0 the complex64 gates of 5 and 6 qubits stay on the FP32 pipes (k_dense)."""
    monkeypatch.setenv("QM_DENSE_TC", "0")
    c = random_circuit(n, 160, seed=8000 + 100 * width + n)
    psi = random_state(n, n + width + 70)
    want = orc.execute(c, psi)
    launches0, tc0 = dense_launches()
    with DeviceState(gpu_context, n, FP32) as st:
        st.Upload(psi)
        st.Evolve(c, fusion_width=width)
        got = st.Download()
    launches1, tc1 = dense_launches()
    assert tc1 == tc0 and launches1 > launches0
    assert np.max(np.abs(got - want)) <= 2e-6
