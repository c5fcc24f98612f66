"""Executes a fused schedule from qm_plan_program on the CPU with numpy (test infrastructure).

The emulator follows the semantics the fused kernel implements: per pass, every CTA owns
the amplitudes whose block-qubit bits vary and whose other bits are fixed; ops act on the
block in order; a stage change only moves data between threads, so it merely changes which
local bit each register index names.  A relabeling pass writes local bit b to index bit
qubits_out[b] instead of qubits[b].  Comparing the emulated result with the oracle checks
the planner (gate placement, reordering, register and mask translation) without a GPU.
"""
from __future__ import annotations

import ctypes as C

import numpy as np

from quantummatter_b200 import _lib

OP_STAGE, OP_MATRIX, OP_MATRIX_REAL, OP_EXCHANGE, OP_DIAG, OP_NEGATE, OP_SWAP, OP_DIAG_GROUP = range(8)


def program(qubits: int, precision: int, gates, count: int, width: int):
    lib = _lib.load()
    np_, no, nbytes = C.c_int32(), C.c_int32(), C.c_int64()
    _lib.check(lib.qm_plan_program(qubits, precision, gates, count, width, C.byref(np_), None, 0, C.byref(no), None, 0,
                                   C.byref(nbytes)))
    passes = (_lib.FusedPassInfo * max(1, np_.value))()
    ops = (_lib.FusedOpInfo * max(1, no.value))()
    _lib.check(lib.qm_plan_program(qubits, precision, gates, count, width, C.byref(np_), passes, np_.value,
                                   C.byref(no), ops, no.value, C.byref(nbytes)))
    return list(passes)[:np_.value], list(ops)[:no.value], nbytes.value


def scatter(values: np.ndarray, bits) -> np.ndarray:
    """bit i of each value moved to bit bits[i]"""
    out = np.zeros_like(values)
    for i, b in enumerate(bits):
        out |= ((values >> i) & 1) << b
    return out


def deposit(values: np.ndarray, mask: int) -> np.ndarray:
    out = np.zeros_like(values)
    bit = 0
    for b in range(32):
        if mask >> b & 1:
            out |= ((values >> bit) & 1) << b
            bit += 1
    return out


def emulate(state: np.ndarray, qubits: int, passes, ops, reg_bits: int = 4) -> np.ndarray:
    s = state.copy()
    full = (1 << qubits) - 1
    for p in passes:
        k = p.block_qubits
        outer_mask = full & ~p.block_mask
        ctas = np.arange(1 << (qubits - k), dtype=np.int64)
        outer = deposit(ctas, outer_mask)
        local = np.arange(1 << k, dtype=np.int64)
        idx = outer[:, None] | deposit(local, p.block_mask)[None, :]
        blk = s[idx]
        layout = list(p.reg_in)
        assert all(b >= 3 for b in layout), "the load layout keeps the lowest qubits on thread bits"
        pending_members = 0
        for op in ops[p.op_begin:p.op_begin + p.op_count]:
            if op.code == OP_STAGE:
                layout = list(op.reg_pos)
                assert len(set(layout)) == reg_bits and all(0 <= b < k for b in layout)
                continue
            if op.code == OP_DIAG_GROUP:
                # the members follow; the kernel applies them together, the emulator one by one
                assert op.reserved >= 2
                pending_members = op.reserved
                continue
            if pending_members:
                bits = bin(op.cmask_local).count("1") + bin(op.cmask_outer).count("1")
                assert (op.code == OP_DIAG and op.cmask_local == 0 and op.cmask_outer == 0) or \
                    (op.code == OP_NEGATE and bits <= 2), "a group holds only commuting phases and negates"
                pending_members -= 1
            cta_ok = (outer & op.cmask_outer) == op.cmask_outer
            ctl = (local & op.cmask_local) == op.cmask_local
            a, b, c, d = (complex(op.coef[2 * i], op.coef[2 * i + 1]) for i in range(4))
            if op.code in (OP_MATRIX, OP_MATRIX_REAL, OP_EXCHANGE):
                lb = layout[op.reg]
                j0 = local[((local >> lb) & 1 == 0) & ctl]
                j1 = j0 | (1 << lb)
                x, y = blk[:, j0].copy(), blk[:, j1].copy()
                if op.code == OP_EXCHANGE:
                    nx, ny = y, x
                else:
                    nx, ny = a * x + b * y, c * x + d * y
                blk[np.ix_(cta_ok, j0)] = nx[cta_ok]
                blk[np.ix_(cta_ok, j1)] = ny[cta_ok]
            elif op.code == OP_SWAP:
                l1, l2 = layout[op.reg], layout[op.reg2]
                j0 = local[((local >> l1) & 1 == 1) & ((local >> l2) & 1 == 0) & ctl]
                j1 = j0 ^ (1 << l1) ^ (1 << l2)
                x, y = blk[:, j0].copy(), blk[:, j1].copy()
                blk[np.ix_(cta_ok, j0)] = y[cta_ok]
                blk[np.ix_(cta_ok, j1)] = x[cta_ok]
            elif op.code == OP_NEGATE:
                sel = local[ctl]
                blk[np.ix_(cta_ok, sel)] *= -1
            elif op.code == OP_DIAG:
                if op.local >= 0:
                    bit = np.broadcast_to(((local >> op.local) & 1).astype(bool)[None, :], blk.shape)
                else:
                    bit = np.broadcast_to(((outer & op.target_outer) != 0)[:, None], blk.shape)
                mask = cta_ok[:, None] & ctl[None, :]
                phase = np.where(bit, d, a)
                blk = np.where(mask, blk * phase, blk)
            else:
                raise AssertionError(f"unknown op {op.code}")
        assert layout == list(p.reg_out), "a pass must end in its store layout"
        q_in = [p.qubits[b] for b in range(k)]
        q_out = [p.qubits_out[b] for b in range(k)]
        assert sorted(q_out) == q_in, "a pass writes its tile back to the bits it read"
        staged = any(op.code == OP_STAGE for op in ops[p.op_begin:p.op_begin + p.op_count])
        assert q_out == q_in or staged, "a relabeling pass orders its stores after every load (a stage)"
        assert all(q_out[b] >= 3 for b in layout), "the store layout keeps the lowest index bits on thread bits"
        threads = [q_out[b] for b in range(k) if b not in layout]
        out_bit = [p.out_bit[r] for r in range(k - reg_bits)]
        assert sorted(out_bit) == sorted(threads) and out_bit[:3] == [0, 1, 2], "store ranks cover the thread bits"
        s[outer[:, None] | scatter(local, q_out)[None, :]] = blk
    return s
