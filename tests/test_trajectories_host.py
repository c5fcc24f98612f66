"""Host-side logic of the batched trajectory runner (no GPU).

- the library's seeded System.Random stream against the oracle's restatement;
- NoisyCircuit flattening and draw bounds;
- the oracle's whole-trajectory restatement against its own channel-by-channel form;
- the reference-order draw bookkeeping of B200NoisySimulator (speculate, read back what each
  trajectory consumed, re-run the rest from the corrected offset), driven by a stand-in batch
  runner that evolves every trajectory on the oracle.
"""
from __future__ import annotations

import ctypes as C

import numpy as np
import pytest

import oracle as orc
from quantummatter_b200 import _lib
from quantummatter_b200.circuit import QuantumCircuit
from quantummatter_b200.noise import NoiseChannel, NoisyCircuit
from quantummatter_b200.trajectories import B200NoisySimulator, TrajectoryBatch, random_doubles


def test_struct_layouts():
    assert C.sizeof(_lib.ChannelC) == 24
    assert C.sizeof(_lib.TrajectoryOutputs) == 64
    assert C.sizeof(_lib.TrajectoryStats) == 40


@pytest.mark.parametrize("seed", [0, 1, 42, 20260101, -7, 2**31 - 1, -2**31])
def test_seeded_stream_matches_the_oracle(seed):
    r = orc.DotNetRandom(seed)
    want = np.array([r.NextDouble() for _ in range(300)])
    assert np.array_equal(random_doubles(seed, 300), want)
    assert np.array_equal(random_doubles(seed, 100, skip=200), want[200:])


def test_known_first_draw_of_seed_42():
    # Random(42).NextDouble() is 0.668106465911542 on .NET's seeded generator
    assert abs(random_doubles(42, 1)[0] - 0.668106465911542) < 1e-15


def sample_circuit(n: int, seed: int, layers: int = 3, gamma: float = 0.35, dep: float = 0.6) -> NoisyCircuit:
    rng = np.random.default_rng(seed)
    nc = NoisyCircuit(n)
    for _ in range(layers):
        c = QuantumCircuit(n)
        for q in range(n):
            c.Ry(q, float(rng.uniform(0, 2 * np.pi)))
        nc.Append(c)
        for q in range(n):
            nc.ApplyNoise(NoiseChannel.Depolarizing(dep), q)
        ladder = QuantumCircuit(n)
        for q in range(n - 1):
            ladder.CZ(q, q + 1) if q % 2 else ladder.CNot(q, q + 1)
        nc.Append(ladder)
        nc.ApplyNoise(NoiseChannel.BitFlip(0.3), 0)
        nc.ApplyNoise(NoiseChannel.PhaseFlip(1.0), n - 1)
        nc.ApplyNoise(NoiseChannel.BitFlip(0.0), 0)
        for q in range(n):
            nc.ApplyNoise(NoiseChannel.AmplitudeDamping(gamma), q)
        nc.ApplyNoise(NoiseChannel.AmplitudeDamping(gamma), 0)  # twice in a row: zero mass after a jump
    return nc


def test_flatten_and_draw_bound():
    nc = sample_circuit(4, 1, layers=2)
    flat, placements = nc.Flatten()
    assert len(flat.Operations) == 2 * (4 + 3)
    assert len(placements) == 2 * (4 + 3 + 5)
    assert [p for _, _, p in placements[:4]] == [4, 4, 4, 4]
    # the certain phase flip and the p = 0 flip take no draw
    assert nc.MaxDraws() == 2 * (4 + 1 + 5)


def test_oracle_trajectory_matches_channel_by_channel():
    nc = sample_circuit(4, 2)
    draws = random_doubles(9, nc.MaxDraws())
    state, used, branches = orc.trajectory(nc, draws)
    s = orc.zero_state(4)
    k = 0
    for step in nc.Steps:
        if step.Circuit is not None:
            s = orc.execute(step.Circuit, s)
        elif step.Channel.Probability != 0:
            s, u = orc.noise_apply(int(step.Channel.Kind), step.Channel.Probability, step.Target, s, draws[k:])
            k += u
    assert used == k
    assert np.array_equal(state, s)
    assert set(np.unique(branches)) <= {-1, 0, 1, 2, 3}


class OracleBatchSimulator(B200NoisySimulator):
    """Stand-in for the device batch: each trajectory runs on the oracle with its row of draws."""

    def __init__(self):
        self.precision = 0
        self.calls = 0

    def _run(self, comp, d, observables, branches, outcomes, probabilities, masses):
        self.calls += 1
        T = d.shape[0]
        res = TrajectoryBatch(consumed=np.zeros(T, dtype=np.int32), outcomes=np.zeros(T, dtype=np.int64) if outcomes else None,
                              masses=np.zeros(T), ambiguous=np.zeros(T, dtype=np.int32))
        for t in range(T):
            state, used, _ = orc.trajectory(self.noisy, d[t])
            assert used <= d.shape[1]
            if outcomes:
                _, res.outcomes[t] = orc.measure_all(state, d[t][used])
                used += 1
            res.consumed[t] = used
            res.masses[t] = np.vdot(state, state).real
        return res


def test_reference_order_draws_with_replays():
    nc = sample_circuit(3, 5, layers=2, gamma=0.9)
    sim = OracleBatchSimulator()
    sim.noisy = nc
    from quantummatter_b200.trajectories import _Compiled
    comp = _Compiled.__new__(_Compiled)
    comp.max_draws = nc.MaxDraws()
    shots = 24
    stream = random_doubles(77, shots * (comp.max_draws + 1))
    res = sim._sequential(comp, shots, stream, measure=True)
    # the same shots drawn strictly one after another from the stream
    offset = 0
    want_outcomes, want_consumed = [], []
    for _ in range(shots):
        state, used, _ = orc.trajectory(nc, stream[offset:])
        _, o = orc.measure_all(state, stream[offset + used])
        want_outcomes.append(o)
        want_consumed.append(used + 1)
        offset += used + 1
    assert list(res.consumed) == want_consumed
    assert list(res.outcomes) == want_outcomes
    # with gamma = 0.9 some dampings find a zero branch, so some trajectories drew less
    assert min(want_consumed) < comp.max_draws + 1
    assert res.reruns >= 1 and sim.calls == res.reruns + 1
