"""Admission and batching policy of the library's request server (no GPU).

The policy is the header qm_serve_policy.h that qm_serve.cpp runs; tests/serve_policy_test.cpp
exercises it scenario by scenario, compiled here with g++.
"""
from __future__ import annotations

import shutil
import subprocess
from pathlib import Path

import numpy as np
import pytest

from quantummatter_b200.backend import FP64
from quantummatter_b200.serving import VqeSession
from quantummatter_b200.workloads import hardware_efficient_ansatz, tfim_chain

ROOT = Path(__file__).resolve().parents[1]
GXX = shutil.which("g++")


@pytest.fixture(scope="module")
def policy_run(tmp_path_factory):
    exe = tmp_path_factory.mktemp("policy") / "serve_policy_test"
    res = subprocess.run([GXX, "-std=c++17", "-O1", "-Wall", "-I", str(ROOT / "include"),
                          "-I", str(ROOT / "quantummatter_b200" / "csrc"), str(ROOT / "tests" / "serve_policy_test.cpp"),
                          "-o", str(exe)], capture_output=True, text=True, timeout=300)
    assert res.returncode == 0, res.stderr[-2000:]
    run = subprocess.run([str(exe)], capture_output=True, text=True, timeout=60)
    return run


@pytest.mark.skipif(GXX is None, reason="g++ not found")
@pytest.mark.parametrize("scenario", ["reservations_never_exceed_the_budget", "oversized_requests_are_rejected",
                                      "vqe_steps_batch_by_key_and_sessions_serialise",
                                      "keys_ignore_coefficients_and_parameters", "drain_returns_waiting_requests"])
def test_policy_scenario(policy_run, scenario):
    assert policy_run.returncode == 0, policy_run.stdout + policy_run.stderr
    assert f"ok {scenario}" in policy_run.stdout


def test_sessions_keep_their_coefficients():
    c = hardware_efficient_ansatz(8, 1)
    a = VqeSession(c, tfim_chain(8, 1), np.zeros(c.ParameterCount), precision=FP64)
    b = VqeSession(c, tfim_chain(8, 2), np.zeros(c.ParameterCount), precision=FP64)
    assert not np.array_equal(a.coefficients, b.coefficients)
    assert [t.Observable.FlipMask for t in a.hamiltonian.Terms] == [t.Observable.FlipMask for t in b.hamiltonian.Terms]
