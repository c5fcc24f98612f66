"""Partitioned batch workloads over two gloo ranks on the host (no GPU).

The per-unit work runs on a stand-in that evolves each trajectory on the oracle; what is under
test is the partitioning, the all-gather of per-unit results and the cross-rank draw-offset
rounds, which must reproduce the strictly sequential single-process result exactly.
"""
from __future__ import annotations

import datetime
import multiprocessing as mp
import socket

import numpy as np
import pytest

from quantummatter_b200.distributed import partition


def free_port() -> int:
    with socket.socket() as s:
        s.bind(("127.0.0.1", 0))
        return s.getsockname()[1]


def test_partition_covers_every_unit_once():
    for total in (0, 1, 5, 16, 17):
        for world in (1, 2, 3, 8):
            parts = [partition(total, world, r) for r in range(world)]
            assert parts[0][0] == 0 and parts[-1][1] == total
            assert all(parts[r][1] == parts[r + 1][0] for r in range(world - 1))
            sizes = [hi - lo for lo, hi in parts]
            assert max(sizes) - min(sizes) <= 1


def noisy_circuit():
    from quantummatter_b200.circuit import QuantumCircuit
    from quantummatter_b200.noise import NoiseChannel, NoisyCircuit
    nc = NoisyCircuit(3)
    rng = np.random.default_rng(4)
    for _ in range(2):
        c = QuantumCircuit(3)
        for q in range(3):
            c.Ry(q, float(rng.uniform(0, 6.28)))
        c.CZ(0, 1).CNot(1, 2)
        nc.Append(c)
        for q in range(3):
            nc.ApplyNoise(NoiseChannel.Depolarizing(0.5), q)
            nc.ApplyNoise(NoiseChannel.AmplitudeDamping(0.9), q)
        nc.ApplyNoise(NoiseChannel.AmplitudeDamping(0.9), 0)
    return nc


def observables():
    from quantummatter_b200.observables import PauliString
    return [PauliString("IIZ"), PauliString("IZZ"), PauliString("XIX")]


class OracleRunner:
    """RunBatch on the oracle: trajectory t consumes rows[t] in order."""

    def RunBatch(self, circuit, rows, observables):
        import oracle as orc
        from quantummatter_b200.trajectories import TrajectoryBatch
        T = rows.shape[0]
        res = TrajectoryBatch(values=np.zeros((T, len(observables))), masses=np.zeros(T),
                              consumed=np.zeros(T, dtype=np.int32))
        for t in range(T):
            state, used, _ = orc.trajectory(circuit, rows[t])
            res.values[t] = [orc.expectation(state, o) for o in observables]
            res.masses[t] = np.vdot(state, state).real
            res.consumed[t] = used
        return res


class SumEvaluator:
    """Stand-in evaluator: energy = sum of the parameters, gradient = index-weighted parameters."""

    def EvaluateBatch(self, circuit, hamiltonian, params, withGradient=True):
        from types import SimpleNamespace
        e = params.sum(axis=1)
        g = params * np.arange(1, params.shape[1] + 1) if withGradient else None
        return SimpleNamespace(Energies=e, Gradients=g)


def _rank(rank, world, port, trajectories, queue):
    import torch.distributed as dist

    from quantummatter_b200.distributed import trajectory_values, vqe_batch
    from quantummatter_b200.trajectories import random_doubles
    dist.init_process_group("gloo", init_method=f"tcp://127.0.0.1:{port}", rank=rank, world_size=world,
                            timeout=datetime.timedelta(seconds=120))
    try:
        nc = noisy_circuit()
        stream = random_doubles(31, trajectories * nc.MaxDraws())
        out = trajectory_values(OracleRunner(), nc, observables(), trajectories, stream, dist)
        params = np.arange(7 * 4, dtype=np.float64).reshape(7, 4) / 10
        e, g = vqe_batch(SumEvaluator(), None, None, params, dist)
        queue.put((rank, out, e, g))
    finally:
        dist.destroy_process_group()


def test_two_ranks_reproduce_the_sequential_run():
    trajectories = 9
    port = free_port()
    ctx = mp.get_context("spawn")
    queue = ctx.Queue()
    procs = [ctx.Process(target=_rank, args=(r, 2, port, trajectories, queue)) for r in range(2)]
    for p in procs:
        p.start()
    results = [queue.get(timeout=300) for _ in range(2)]
    for p in procs:
        p.join(timeout=60)
        assert p.exitcode == 0
    import oracle as orc
    from quantummatter_b200.trajectories import random_doubles
    nc = noisy_circuit()
    stream = random_doubles(31, trajectories * nc.MaxDraws())
    offset, want_v, want_c = 0, [], []
    for _ in range(trajectories):
        state, used, _ = orc.trajectory(nc, stream[offset:])
        want_v.append([orc.expectation(state, o) for o in observables()])
        want_c.append(used)
        offset += used
    assert min(want_c) < nc.MaxDraws()  # some trajectories drew less: replay rounds happened
    params = np.arange(7 * 4, dtype=np.float64).reshape(7, 4) / 10
    for rank, out, e, g in results:
        assert list(out["consumed"]) == want_c
        assert np.array_equal(out["values"], np.array(want_v))
        assert out["rounds"] >= 2
        assert np.array_equal(e, params.sum(axis=1))
        assert np.array_equal(g, params * np.arange(1, 5))
