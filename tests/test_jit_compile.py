"""Generated kernel sources compile for sm_100a on the CPU (nvcc cross-compiles without a GPU).

The passes compiled for their own op sequence and the tiled expectation compiled for a term list
are generated at run time and compiled with NVRTC on the GPU host; this checks a spread of them
here: random circuits (controls, Toffolis, SWAPs, X on thread bits and outside the block),
diagonal-heavy and QFT circuits, 26-qubit bricks in both precisions (the two tile pipelines),
and an XXZ term list.
"""
from __future__ import annotations

import ctypes as C
import os
import shutil
import subprocess

import pytest

from circuits import random_circuit
from quantummatter_b200._lib import check, load
from quantummatter_b200.algorithms import QuantumFourierTransform
from quantummatter_b200.backend import FP32, FP64
from quantummatter_b200.circuit import prepare
from quantummatter_b200.observables import terms_array
from quantummatter_b200.workloads import brick_circuit, xxz_chain
from test_abi import diagonal_heavy_circuit

NVCC = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"


def pass_source(circuit, precision: int, index: int) -> str:
    g, n = prepare(circuit)
    ln = C.c_size_t()
    check(load().qm_jit_source(circuit.QubitCount, precision, g, n, 0, index, None, 0, C.byref(ln)))
    buf = C.create_string_buffer(ln.value + 1)
    check(load().qm_jit_source(circuit.QubitCount, precision, g, n, 0, index, buf, ln.value + 1, C.byref(ln)))
    return buf.value.decode()


def expect_source(qubits: int, precision: int, index: int) -> str:
    arr, n = terms_array(xxz_chain(qubits).Terms)
    ln = C.c_size_t()
    check(load().qm_jit_expect_source(qubits, precision, arr, n, index, None, 0, C.byref(ln)))
    buf = C.create_string_buffer(ln.value + 1)
    check(load().qm_jit_expect_source(qubits, precision, arr, n, index, buf, ln.value + 1, C.byref(ln)))
    return buf.value.decode()


CASES = [
    ("random", lambda: pass_source(random_circuit(14, 300, seed=21), FP64, 0)),
    ("random_fp32", lambda: pass_source(random_circuit(16, 300, seed=5), FP32, 1)),
    ("diagonal", lambda: pass_source(diagonal_heavy_circuit(14, 300, seed=22), FP64, 0)),
    ("qft", lambda: pass_source(QuantumFourierTransform.CreateCircuit(20), FP64, 1)),
    ("brick26_fp64", lambda: pass_source(brick_circuit(26, 6, seed=4), FP64, 2)),
    ("brick26_fp32", lambda: pass_source(brick_circuit(26, 6, seed=4), FP32, 2)),
    ("expect_fp32", lambda: expect_source(22, FP32, 0)),
    ("expect_fp64", lambda: expect_source(20, FP64, 1)),
]


@pytest.mark.skipif(not os.path.exists(NVCC), reason="nvcc not found")
@pytest.mark.parametrize("name,make", CASES, ids=[c[0] for c in CASES])
def test_generated_source_compiles_for_sm100a(tmp_path, name, make):
    src = make()
    path = tmp_path / f"{name}.cu"
    path.write_text(src)
    res = subprocess.run([NVCC, "-gencode", "arch=compute_100a,code=sm_100a", "-O3", "-std=c++17", "-cubin",
                          "-o", str(tmp_path / f"{name}.cubin"), str(path)], capture_output=True, text=True, timeout=600)
    assert res.returncode == 0, res.stderr[-2000:]
