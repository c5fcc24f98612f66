"""Fused passes compiled for their own op sequence (NVRTC) against the interpreter and the oracle.

Plans (qm_plan_create) run compiled passes; one-shot executions (DeviceState.Evolve) run the
interpreting pass kernel.  Both must give the oracle's state on circuits that reach every op
kind: controlled and doubly controlled gates, diagonal groups with phases and signs, SWAPs,
Toffolis, X controls on thread bits and on qubits outside the block.
"""
from __future__ import annotations

import ctypes as C
import re

import numpy as np
import pytest

import oracle as orc
from circuits import random_circuit, random_state
from quantummatter_b200._lib import check, load
from quantummatter_b200.backend import FP32, FP64, DeviceState, Plan
from quantummatter_b200.circuit import prepare
from quantummatter_b200.workloads import brick_circuit
from test_abi import diagonal_heavy_circuit


def jit_info():
    avail, kernels, failed, launches = C.c_int32(), C.c_int64(), C.c_int64(), C.c_int64()
    check(load().qm_jit_info(C.byref(avail), C.byref(kernels), C.byref(failed), C.byref(launches)))
    return avail.value, kernels.value, failed.value, launches.value


def perturbed_brick(n: int, depth: int, eps: float):
    """The brick circuit's structure with every angle moved by eps."""
    from quantummatter_b200.circuit import QuantumCircuit, u3
    from quantummatter_b200.workloads import SplitMix64
    rng, c = SplitMix64(1), QuantumCircuit(n)
    for layer in range(depth):
        for q in range(n):
            th, ph, la = (rng.uniform(0, 2 * np.pi) + eps for _ in range(3))
            c.U(q, u3(th, ph, la))
        for q in range(layer % 2, n - 1, 2):
            c.CNot(q, q + 1)
    return c


def jit_sources(c, passes):
    g, n = prepare(c)
    out = []
    for p in passes:
        ln = C.c_size_t()
        check(load().qm_jit_source(c.QubitCount, FP64, g, n, 0, p, None, 0, C.byref(ln)))
        buf = C.create_string_buffer(ln.value + 1)
        check(load().qm_jit_source(c.QubitCount, FP64, g, n, 0, p, buf, ln.value + 1, C.byref(ln)))
        out.append(buf.value.decode())
    return out


def test_generated_source_is_structural():
    """Sources hold the pass structure and the form of each rotation; the angles and every
    constant derived from them travel in the kernel's parameter block."""
    a = jit_sources(perturbed_brick(14, 4, 0.0), [0, 1])
    b = jit_sources(perturbed_brick(14, 4, 1e-9), [0, 1])
    assert a == b
    assert "qm_pass" in a[0] and "A.v[" in a[0] and "__grid_constant__ Aux A" in a[0]
    # the first pass carries its pending phases; the last multiplies them in
    assert not re.search(r"\bf\d+r = A\.v\[", a[0])
    assert re.search(r"\bf\d+r = A\.v\[", a[1])


@pytest.mark.gpu
@pytest.mark.parametrize("kind", ["random", "diagonal", "brick"])
@pytest.mark.parametrize("precision", [FP64, FP32])
def test_compiled_passes_match_the_oracle(gpu_context, kind, precision):
    avail, _, failed0, launches0 = jit_info()
    assert avail == 1
    n = 14
    if kind == "random":
        c = random_circuit(n, 300, seed=21)
    elif kind == "diagonal":
        c = diagonal_heavy_circuit(n, 300, seed=22)
    else:
        c = brick_circuit(n, 12, seed=23)
    psi = random_state(n, 5)
    want = orc.execute(c, psi)
    p = Plan(gpu_context, c, precision, 0)
    with DeviceState(gpu_context, n, precision) as st:
        st.Upload(psi)
        p.execute(st)
        compiled = st.Download()
        st.Upload(psi)
        st.Evolve(c)
        interpreted = st.Download()
    p.Dispose()
    tol = 1e-12 if precision == FP64 else 2e-5
    assert np.max(np.abs(compiled - want)) <= tol
    assert np.max(np.abs(interpreted - want)) <= tol
    _, _, failed1, launches1 = jit_info()
    assert failed1 == failed0 and launches1 > launches0  # the compiled kernels ran


@pytest.mark.gpu
def test_compiled_passes_at_scale(gpu_context):
    """A 24-qubit brick (blocks with qubits outside them) through a plan, against the oracle."""
    n = 24
    c = brick_circuit(n, 8, seed=3)
    want = orc.execute(c)
    p = Plan(gpu_context, c, FP64, 0)
    with DeviceState(gpu_context, n, FP64) as st:
        p.execute(st)
        got = st.Download()
    p.Dispose()
    assert np.max(np.abs(got - want)) <= 1e-12


@pytest.mark.gpu
def test_pipelined_passes(gpu_context):
    """From 26 qubits compiled passes copy the next tile into shared memory while computing:
    complex64 passes into a second tile, complex128 passes into the exchange tile after their
    last exchange.  The complex128 state must match the oracle's parallel path, the complex64
    one the complex128 one to FP32 rounding."""
    n = 26
    c = brick_circuit(n, 4, seed=4)
    want = orc.execute_parallel(c)
    _, _, _, launches0 = jit_info()
    out = {}
    for prec in (FP64, FP32):
        p = Plan(gpu_context, c, prec, 0)
        with DeviceState(gpu_context, n, prec) as st:
            p.execute(st)
            out[prec] = st.Download()
        p.Dispose()
    _, _, _, launches1 = jit_info()
    assert launches1 > launches0
    assert np.max(np.abs(out[FP64] - want)) <= 1e-12
    rel = np.linalg.norm(out[FP32] - out[FP64]) / np.linalg.norm(out[FP64])
    assert rel <= 1e-5


@pytest.mark.gpu
def test_pipelined_passes_as_two_teams(gpu_context, monkeypatch):
    """With QM_TEAMS=1 complex128 pipelined passes run as one 512-thread block per SM of two
    teams that hand a compute token back and forth by named barriers (blocks whose second team
    has no work item included); the state must match the oracle's parallel path."""
    monkeypatch.setenv("QM_TEAMS", "1")
    n = 26
    c = brick_circuit(n, 4, seed=5)
    want = orc.execute_parallel(c)
    g, count = prepare(c)
    ln = C.c_size_t()
    check(load().qm_jit_source(n, FP64, g, count, 0, 0, None, 0, C.byref(ln)))
    buf = C.create_string_buffer(ln.value + 1)
    check(load().qm_jit_source(n, FP64, g, count, 0, 0, buf, ln.value + 1, C.byref(ln)))
    assert b"const u32 team = threadIdx.x >>" in buf.value
    p = Plan(gpu_context, c, FP64, 0)
    try:
        with DeviceState(gpu_context, n, FP64) as st:
            p.execute(st)
            got = st.Download()
    finally:
        p.Dispose()
    assert np.max(np.abs(got - want)) <= 1e-12


def _sources(circuit, precision=FP64):
    g, n = prepare(circuit)
    out, p = [], 0
    while True:
        ln = C.c_size_t()
        if load().qm_jit_source(circuit.QubitCount, precision, g, n, 0, p, None, 0, C.byref(ln)):
            return out
        buf = C.create_string_buffer(ln.value + 1)
        check(load().qm_jit_source(circuit.QubitCount, precision, g, n, 0, p, buf, ln.value + 1, C.byref(ln)))
        out.append(buf.value.decode())
        p += 1


def test_generated_forms_of_the_benchmark_circuit(monkeypatch):
    """The 30-qubit brick's passes: every rotation pair applies its phase by three shears (7 FMAs
    per pair), the CNOTs planned as CZs leave no conditional register swap behind but those of the
    last layer, and the CZ signs are deferred into the rotations' phases.  The real-rotation
    ansatz (Ry, Rz, CZ ladders) keeps its CZs as negations, which deferral would turn into complex
    products."""
    from quantummatter_b200.workloads import hardware_efficient_ansatz, uniform_parameters
    src = _sources(brick_circuit(30, 40))
    assert len(src) == 25
    text = "\n".join(src)
    shears = text.count("const double wr = pu")
    products = len(re.findall(r"const double wr = \w+ \* x", text))
    assert shears > 9000 and products == 0
    assert text.count("double u = x") <= 8 * 14  # conditional swaps: at most the last layer's CNOTs
    monkeypatch.setenv("QM_CZ_DEFER", "0")
    negations_off = "\n".join(_sources(brick_circuit(30, 40))).count("= -x")
    monkeypatch.delenv("QM_CZ_DEFER")
    assert text.count("= -x") < negations_off
    a = hardware_efficient_ansatz(22, 4)
    bound = a.Bind(list(uniform_parameters(a.ParameterCount, 1, -3, 3, seed=1)[0]))
    on = "\n".join(_sources(bound)).count("= -x")
    monkeypatch.setenv("QM_CZ_DEFER", "0")
    assert on == "\n".join(_sources(bound)).count("= -x")
