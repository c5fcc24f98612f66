"""Fused passes compiled for their own op sequence (NVRTC) against the interpreter and the oracle.

Plans (qm_plan_create) run compiled passes; one-shot executions (DeviceState.Evolve) run the
interpreting pass kernel.  Both must give the oracle's state on circuits that reach every op
kind: controlled and doubly controlled gates, diagonal groups with phases and signs, SWAPs,
Toffolis, X controls on thread bits and on qubits outside the block.
"""
from __future__ import annotations

import ctypes as C

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


def test_generated_source_is_structural():
    """Sources depend on the pass structure, not on the angles."""
    a, na = prepare(brick_circuit(14, 4, seed=1))
    b, nb = prepare(brick_circuit(14, 4, seed=2))
    out = []
    for g, n in ((a, na), (b, nb)):
        ln = C.c_size_t()
        check(load().qm_jit_source(14, FP64, g, n, 0, 0, None, 0, C.byref(ln)))
        buf = C.create_string_buffer(ln.value + 1)
        check(load().qm_jit_source(14, FP64, g, n, 0, 0, buf, ln.value + 1, C.byref(ln)))
        out.append(buf.value.decode())
    assert out[0] == out[1]
    assert "qm_pass" in out[0] and "prog[" in out[0]


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
