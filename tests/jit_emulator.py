"""TEST INFRASTRUCTURE: runs a plan's compiled passes on the CPU (tests/jit_emulator.cpp).

Each pass's generated source (qm_jit_source) is built with g++ into a small shared library and
launched on a numpy state with the pass's launch record (as the library builds it from the
planner's pass record) and its constant block (qm_jit_constants).  Passes are chained exactly as
the library chains them, so the state after the last pass is the plan's result.
"""
from __future__ import annotations

import ctypes as C
import hashlib
import os
import shutil
import subprocess
import tempfile
from pathlib import Path

import numpy as np

from quantummatter_b200._lib import FusedOpInfo, FusedPassInfo, check, load
from quantummatter_b200.backend import FP32
from quantummatter_b200.circuit import prepare

HERE = Path(__file__).resolve().parent
HARNESS = HERE / "jit_emulator.cpp"
CACHE = Path(tempfile.gettempdir()) / "qm_jit_emulator"
GXX = shutil.which("g++")
R = 4


class Launch(C.Structure):  # FusedLaunch
    _fields_ = [("outer_mask", C.c_uint32), ("thread_in", C.c_uint32), ("thread_out", C.c_uint32),
                ("op_count", C.c_int32), ("reg_in_g", C.c_uint32 * R), ("reg_out_g", C.c_uint32 * R),
                ("reg_in_l", C.c_int32 * R), ("cta_shift", C.c_int32), ("states", C.c_int32),
                ("table_slots", C.c_int32), ("pad", C.c_int32), ("ops", C.c_void_p), ("table", C.c_void_p),
                ("state_stride", C.c_uint64), ("table_stride", C.c_uint64), ("out_bit", C.c_uint8 * 16)]


def _build(src: str) -> C.CDLL:
    CACHE.mkdir(parents=True, exist_ok=True)
    key = hashlib.sha1(src.encode()).hexdigest()[:20]
    so = CACHE / f"emu_{key}.so"
    if not so.exists():
        gen = CACHE / f"emu_{key}.inc"
        gen.write_text(src)
        hist = ", reinterpret_cast<double*>(hist)" if "double* __restrict__ hist" in src else ""
        tmp = CACHE / f"emu_{key}.{os.getpid()}.so"
        res = subprocess.run([GXX, "-std=c++20", "-O1", "-shared", "-fPIC", "-pthread", "-w",
                              f'-DGENERATED="{gen}"', f"-DEMU_HIST_ARG={hist}", str(HARNESS), "-o", str(tmp)],
                             capture_output=True, text=True, timeout=900)
        if res.returncode != 0:
            raise RuntimeError(res.stderr[-3000:])
        tmp.replace(so)
    lib = C.CDLL(str(so))
    lib.emu_run.restype = C.c_int
    lib.emu_run.argtypes = [C.c_void_p, C.c_void_p, C.c_size_t, C.c_void_p, C.c_size_t, C.c_void_p, C.c_int,
                            C.c_int, C.c_int]
    return lib


def _text(fn, *args) -> bytes:
    ln = C.c_size_t()
    check(fn(*args, None, 0, C.byref(ln)))
    buf = C.create_string_buffer(ln.value + 1)
    check(fn(*args, buf, ln.value + 1, C.byref(ln)))
    return buf.raw[:ln.value]


def run_plan(circuit, precision: int, state: np.ndarray, width: int = 0, grid: int = 1) -> np.ndarray:
    """The plan's compiled passes (fusion width `width`, 0: the default) applied to a copy of
    `state` on the CPU, each launched as `grid` blocks."""
    n = circuit.QubitCount
    g, count = prepare(circuit)
    lib = load()
    P, O, pb = C.c_int32(), C.c_int32(), C.c_int64()
    check(lib.qm_plan_program(n, precision, g, count, width, C.byref(P), None, 0, C.byref(O), None, 0, C.byref(pb)))
    passes = (FusedPassInfo * max(1, P.value))()
    ops = (FusedOpInfo * max(1, O.value))()
    check(lib.qm_plan_program(n, precision, g, count, width, C.byref(P), passes, P.value, C.byref(O), ops, O.value,
                              C.byref(pb)))
    s = np.array(state, dtype=np.complex64 if precision == FP32 else np.complex128, copy=True)
    all_mask = (1 << n) - 1
    for i in range(P.value):
        p = passes[i]
        k = p.block_qubits
        src = _text(lib.qm_jit_source, n, precision, g, count, width, i).decode()
        aux = _text(lib.qm_jit_constants, n, precision, g, count, width, i)
        L = Launch()
        L.outer_mask = all_mask & ~p.block_mask
        reg_in = {p.reg_in[m] for m in range(R)}
        reg_out = {p.reg_out[m] for m in range(R)}
        for m in range(R):
            L.reg_in_l[m] = p.reg_in[m]
            L.reg_in_g[m] = 1 << p.qubits[p.reg_in[m]]
            L.reg_out_g[m] = 1 << p.qubits_out[p.reg_out[m]]
        L.thread_in = sum(1 << p.qubits[b] for b in range(k) if b not in reg_in)
        L.thread_out = sum(1 << p.qubits_out[b] for b in range(k) if b not in reg_out)
        for r in range(k - R):
            L.out_bit[r] = p.out_bit[r]
        L.op_count = p.op_count
        L.ops = C.addressof(ops) + p.op_begin * C.sizeof(FusedOpInfo)
        L.cta_shift = n - k
        L.states = 1
        auxbuf = C.create_string_buffer(aux, len(aux))
        teams = 2 if "const u32 team = threadIdx.x >>" in src else 1
        rc = _build(src).emu_run(s.ctypes.data, C.addressof(L), C.sizeof(L), auxbuf, len(aux), None,
                                 teams << (k - R), teams, grid)
        if rc:
            raise RuntimeError(f"emulator rejected pass {i}: {rc}")
    return s


def available() -> bool:
    return GXX is not None
