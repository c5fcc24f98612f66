"""TEST INFRASTRUCTURE: ctypes loader of the CPU oracle (oracle/liboracle.so).

Only tests/, __graft_entry__.smoke() and bench.py's CPU-baseline legs may import this
module.  It wraps the C restatement of QuantumMatter's scalar path (qm_oracle.c) and the
timed parallel/AVX-512 restatement (qm_cpu_parallel.cpp); see oracle/qm_oracle.h for what
each function restates and how the oracle is pinned.
"""
from __future__ import annotations

import ctypes as C
import subprocess
from pathlib import Path
from typing import Sequence

import numpy as np

HERE = Path(__file__).resolve().parent
LIB = HERE / "liboracle.so"


class Op(C.Structure):
    _fields_ = [("kind", C.c_int32), ("target", C.c_int32), ("control", C.c_int32),
                ("second_control", C.c_int32), ("angle", C.c_double), ("unitary", C.c_double * 8)]


class PGate(C.Structure):
    _fields_ = [("kernel", C.c_int32), ("target", C.c_int32), ("control_mask", C.c_uint32),
                ("swap_control", C.c_int32), ("a", C.c_double * 2), ("b", C.c_double * 2),
                ("c", C.c_double * 2), ("d", C.c_double * 2)]


class ParallelOptions(C.Structure):
    _fields_ = [("workers", C.c_int32), ("min_parallel_qubits", C.c_int32), ("simd", C.c_int32),
                ("avx512", C.c_int32), ("blocking", C.c_int32)]


class Random(C.Structure):
    _fields_ = [("seed_array", C.c_int32 * 56), ("inext", C.c_int32), ("inextp", C.c_int32)]


class Channel(C.Structure):
    _fields_ = [("kind", C.c_int32), ("target", C.c_int32), ("probability", C.c_double),
                ("position", C.c_int32), ("reserved", C.c_int32)]


_lib = None


def build() -> Path:
    res = subprocess.run(["make", "-s", "-C", str(HERE)], capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"oracle build failed:\n{res.stdout}\n{res.stderr}")
    return LIB


def load() -> C.CDLL:
    global _lib
    if _lib is not None:
        return _lib
    srcs = [HERE / "qm_oracle.c", HERE / "qm_cpu_parallel.cpp", HERE / "qm_oracle.h", HERE / "Makefile"]
    if not LIB.exists() or any(s.stat().st_mtime > LIB.stat().st_mtime for s in srcs):
        build()
    lib = C.CDLL(str(LIB))
    DP = C.POINTER(C.c_double)
    lib.qmo_validate.argtypes = [C.POINTER(Op), C.c_int32, C.c_int32]
    lib.qmo_execute.argtypes = [C.POINTER(Op), C.c_int32, C.c_int32, C.c_void_p]
    lib.qmo_execute.restype = None
    lib.qmo_prepare.argtypes = [C.POINTER(Op), C.c_int32, C.POINTER(PGate)]
    lib.qmo_apply_prepared.argtypes = [C.POINTER(PGate), C.c_int32, C.c_int32, C.c_void_p]
    lib.qmo_apply_prepared.restype = None
    lib.qmo_expectation.argtypes = [C.c_void_p, C.c_int32, C.c_uint32, C.c_uint32, C.c_int32, DP]
    lib.qmo_expectation.restype = C.c_double
    lib.qmo_energy.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_uint32), C.POINTER(C.c_uint32),
                               C.POINTER(C.c_int32), DP, C.c_int32, DP]
    lib.qmo_noise_apply.argtypes = [C.c_int32, C.c_double, C.c_int32, C.c_void_p, C.c_int32, DP, C.c_int32,
                                    C.POINTER(C.c_int32)]
    lib.qmo_qubit_masses.argtypes = [C.c_void_p, C.c_int32, C.c_int32, DP, DP]
    lib.qmo_qubit_masses.restype = None
    lib.qmo_sample.argtypes = [C.c_void_p, C.c_int32, DP, C.c_int32, C.POINTER(C.c_int64)]
    lib.qmo_measure_all.argtypes = [C.c_void_p, C.c_int32, C.c_double, C.POINTER(C.c_int64)]
    lib.qmo_random_init.argtypes = [C.POINTER(Random), C.c_int32]
    lib.qmo_random_init.restype = None
    lib.qmo_random_next_double.argtypes = [C.POINTER(Random)]
    lib.qmo_random_next_double.restype = C.c_double
    lib.qmp_execute.argtypes = [C.POINTER(ParallelOptions), C.POINTER(Op), C.c_int32, C.c_int32, C.c_void_p]
    lib.qmp_hardware_threads.restype = C.c_int32
    lib.qmo_trajectory.argtypes = [C.POINTER(Op), C.c_int32, C.POINTER(Channel), C.c_int32, C.c_int32, C.c_void_p,
                                   DP, C.c_int32, C.POINTER(C.c_int32), C.POINTER(C.c_int8)]
    _lib = lib
    return lib


def ops_array(operations) -> tuple[C.Array, int]:
    """Packs GateOperation-like records (Kind, Target, Control, Angle, SecondControl, Unitary)."""
    ops = list(operations)
    arr = (Op * max(1, len(ops)))()
    for i, o in enumerate(ops):
        r = arr[i]
        r.kind, r.target, r.control, r.second_control, r.angle = int(o.Kind), o.Target, o.Control, o.SecondControl, o.Angle
        if o.Unitary is not None:
            u = o.Unitary
            for j, v in enumerate((u.M00.real, u.M00.imag, u.M01.real, u.M01.imag, u.M10.real, u.M10.imag,
                                   u.M11.real, u.M11.imag)):
                r.unitary[j] = v
    return arr, len(ops)


def _buf(state: np.ndarray) -> C.c_void_p:
    assert state.dtype == np.complex128 and state.flags.c_contiguous
    return state.ctypes.data_as(C.c_void_p)


def zero_state(qubits: int) -> np.ndarray:
    s = np.zeros(1 << qubits, dtype=np.complex128)
    s[0] = 1
    return s


def execute(circuit, state: np.ndarray | None = None) -> np.ndarray:
    """CpuStateVectorBackend.Execute on a copy of `state` (default |0...0>)."""
    lib = load()
    s = zero_state(circuit.QubitCount) if state is None else np.array(state, dtype=np.complex128, copy=True)
    arr, n = ops_array(circuit.Operations)
    rc = lib.qmo_validate(arr, n, circuit.QubitCount)
    if rc:
        raise ValueError(f"oracle validation failed: {rc}")
    lib.qmo_execute(arr, n, circuit.QubitCount, _buf(s))
    return s


def execute_parallel(circuit, state: np.ndarray | None = None, workers: int | None = None, simd: bool = True,
                     avx512: bool = True, blocking: bool = True, min_parallel_qubits: int = 16) -> np.ndarray:
    """ParallelCpuStateVectorBackend.Execute (AVX-512, gate blocking) on a copy of `state`, in place if given."""
    lib = load()
    s = zero_state(circuit.QubitCount) if state is None else state
    arr, n = ops_array(circuit.Operations)
    o = ParallelOptions(workers or lib.qmp_hardware_threads(), min_parallel_qubits, int(simd), int(avx512),
                        int(blocking))
    rc = lib.qmp_execute(C.byref(o), arr, n, circuit.QubitCount, _buf(s))
    if rc:
        raise ValueError(f"parallel baseline failed: {rc}")
    return s


def hardware_threads() -> int:
    return int(load().qmp_hardware_threads())


def prepare(circuit) -> C.Array:
    lib = load()
    arr, n = ops_array(circuit.Operations)
    out = (PGate * max(1, n))()
    rc = lib.qmo_prepare(arr, n, out)
    if rc:
        raise ValueError(f"oracle prepare failed: {rc}")
    return out


def apply_prepared(gates, count: int, qubits: int, state: np.ndarray) -> np.ndarray:
    s = np.array(state, dtype=np.complex128, copy=True)
    load().qmo_apply_prepared(gates, count, qubits, _buf(s))
    return s


def expectation(state: np.ndarray, observable) -> float:
    """StateVector.ExpectationValue: raw sequential sum / Born mass of the same pass."""
    lib = load()
    qubits = int(np.log2(state.size))
    mass = C.c_double()
    raw = lib.qmo_expectation(_buf(np.ascontiguousarray(state)), qubits, observable.FlipMask, observable.SignMask,
                              observable.YCount, C.byref(mass))
    return raw / mass.value


def energy(state: np.ndarray, hamiltonian) -> float:
    lib = load()
    qubits = int(np.log2(state.size))
    terms = hamiltonian.Terms
    n = len(terms)
    flip = (C.c_uint32 * max(1, n))(*[t.Observable.FlipMask for t in terms])
    sign = (C.c_uint32 * max(1, n))(*[t.Observable.SignMask for t in terms])
    yc = (C.c_int32 * max(1, n))(*[t.Observable.YCount for t in terms])
    co = (C.c_double * max(1, n))(*[t.Coefficient for t in terms])
    out = C.c_double()
    rc = lib.qmo_energy(_buf(np.ascontiguousarray(state)), qubits, flip, sign, yc, co, n, C.byref(out))
    if rc:
        raise RuntimeError(f"oracle energy failed: {rc}")
    return out.value


def noise_apply(kind: int, p: float, target: int, state: np.ndarray, draws: Sequence[float]) -> tuple[np.ndarray, int]:
    """CpuNoiseChannelBackend.Apply on a copy; returns (state, draws consumed)."""
    lib = load()
    s = np.array(state, dtype=np.complex128, copy=True)
    qubits = int(np.log2(s.size))
    d = (C.c_double * max(1, len(draws)))(*draws)
    used = C.c_int32()
    rc = lib.qmo_noise_apply(kind, p, target, _buf(s), qubits, d, len(draws), C.byref(used))
    if rc:
        raise RuntimeError(f"oracle noise failed: {rc}")
    return s, used.value


def trajectory(noisy_circuit, draws: Sequence[float]) -> tuple[np.ndarray, int, np.ndarray]:
    """One NoisyCircuit.Execute trajectory from |0...0> with the given draws.
    Returns (final state, draws consumed, branch per placement)."""
    flat, placements = noisy_circuit.Flatten()
    ops, n = ops_array(flat.Operations)
    ch = (Channel * max(1, len(placements)))()
    for i, (c, target, pos) in enumerate(placements):
        ch[i].kind, ch[i].target, ch[i].probability, ch[i].position = int(c.Kind), target, c.Probability, pos
    s = zero_state(noisy_circuit.QubitCount)
    d = np.ascontiguousarray(draws, dtype=np.float64)
    dbuf = d.ctypes.data_as(C.POINTER(C.c_double)) if d.size else None
    used = C.c_int32()
    branches = np.full(max(1, len(placements)), -1, dtype=np.int8)
    rc = load().qmo_trajectory(ops, n, ch, len(placements), noisy_circuit.QubitCount, _buf(s), dbuf, int(d.size),
                               C.byref(used), branches.ctypes.data_as(C.POINTER(C.c_int8)))
    if rc:
        raise RuntimeError(f"oracle trajectory failed: {rc}")
    return s, used.value, branches[:len(placements)]


def qubit_masses(state: np.ndarray, target: int) -> tuple[float, float]:
    m0, m1 = C.c_double(), C.c_double()
    load().qmo_qubit_masses(_buf(np.ascontiguousarray(state)), int(np.log2(state.size)), target, C.byref(m0),
                            C.byref(m1))
    return m0.value, m1.value


def sample(state: np.ndarray, draws: Sequence[float]) -> np.ndarray:
    lib = load()
    d = np.ascontiguousarray(draws, dtype=np.float64)
    out = np.zeros(d.size, dtype=np.int64)
    rc = lib.qmo_sample(_buf(np.ascontiguousarray(state)), int(np.log2(state.size)),
                        d.ctypes.data_as(C.POINTER(C.c_double)), d.size, out.ctypes.data_as(C.POINTER(C.c_int64)))
    if rc:
        raise RuntimeError(f"oracle sample failed: {rc}")
    return out


def measure_all(state: np.ndarray, u: float) -> tuple[np.ndarray, int]:
    s = np.array(state, dtype=np.complex128, copy=True)
    out = C.c_int64()
    rc = load().qmo_measure_all(_buf(s), int(np.log2(s.size)), u, C.byref(out))
    if rc:
        raise RuntimeError(f"oracle measure failed: {rc}")
    return s, out.value


def marginal_probability(state: np.ndarray, qubits: Sequence[int], outcome: int) -> float:
    sel = (C.c_int32 * len(qubits))(*qubits)
    out = C.c_double()
    lib = load()
    lib.qmo_marginal_probability.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.c_int32, C.c_int32,
                                             C.POINTER(C.c_double)]
    s = np.ascontiguousarray(state, dtype=np.complex128)
    rc = lib.qmo_marginal_probability(_buf(s), int(np.log2(s.size)), sel, len(qubits), outcome, C.byref(out))
    if rc:
        raise RuntimeError(f"oracle marginal failed: {rc}")
    return out.value


def measure(state: np.ndarray, qubits: Sequence[int], u: float) -> tuple[np.ndarray, int]:
    """StateVector.Measure on a copy: (projected state, outcome)."""
    sel = (C.c_int32 * len(qubits))(*qubits)
    out = C.c_int32()
    lib = load()
    lib.qmo_measure.argtypes = [C.c_void_p, C.c_int32, C.POINTER(C.c_int32), C.c_int32, C.c_double,
                                C.POINTER(C.c_int32)]
    s = np.array(state, dtype=np.complex128, copy=True)
    rc = lib.qmo_measure(_buf(s), int(np.log2(s.size)), sel, len(qubits), u, C.byref(out))
    if rc:
        raise RuntimeError(f"oracle measure failed: {rc}")
    return s, out.value


class DotNetRandom:
    """Seeded System.Random stand-in (restated subtractive generator; see qm_oracle.c)."""

    def __init__(self, seed: int):
        self._r = Random()
        load().qmo_random_init(C.byref(self._r), seed)

    def NextDouble(self) -> float:
        return load().qmo_random_next_double(C.byref(self._r))
