"""Generates the golden fixtures in tests/golden/ (run from the repository root):

    python tests/golden/make_golden.py

known_answers.json  analytic answers the reference's test suite asserts, as data:
                    gate matrix columns on |0> and |1> (StateVectorBackendConformanceTests.cs:14-70,
                    angle pi for the rotations), single-qubit Pauli eigenvalues and two-qubit Bell
                    correlations (StateObservationTests.cs:158-190), depolarizing branch boundaries
                    (NoiseChannelTests.cs:52-64).
dense_random.npz    seeded random circuits over the whole gate set on 1-5 qubits from random
                    normalised input states, with the final states of the independent dense-matrix
                    model (tests/dense_model.py) -- the reference's dense-oracle method
                    (StateVectorBackendConformanceTests.cs:146-245).
hamiltonians.npz    seeded Pauli Hamiltonians on 1-4 qubits, random states and dense energies
                    (PauliHamiltonianTests.cs:10-38).

Nothing here uses the C oracle or the CUDA library, so the fixtures pin both independently.
"""
from __future__ import annotations

import json
import math
import sys
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
ROOT = HERE.parents[1]
sys.path.insert(0, str(ROOT))
sys.path.insert(0, str(ROOT / "tests"))

import dense_model as dm  # noqa: E402
from circuits import circuit_to_arrays, random_circuit, random_state  # noqa: E402


def known_answers() -> dict:
    r = math.sqrt(0.5)
    # (kind, input basis, amplitude of |0>, amplitude of |1>) as [re, im] pairs
    cols = [
        ("H", 0, [r, 0], [r, 0]), ("H", 1, [r, 0], [-r, 0]),
        ("X", 0, [0, 0], [1, 0]), ("X", 1, [1, 0], [0, 0]),
        ("Y", 0, [0, 0], [0, 1]), ("Y", 1, [0, -1], [0, 0]),
        ("Z", 0, [1, 0], [0, 0]), ("Z", 1, [0, 0], [-1, 0]),
        ("S", 0, [1, 0], [0, 0]), ("S", 1, [0, 0], [0, 1]),
        ("T", 0, [1, 0], [0, 0]), ("T", 1, [0, 0], [r, r]),
        ("Rx", 0, [0, 0], [0, -1]), ("Rx", 1, [0, -1], [0, 0]),
        ("Ry", 0, [0, 0], [1, 0]), ("Ry", 1, [-1, 0], [0, 0]),
        ("Rz", 0, [0, -1], [0, 0]), ("Rz", 1, [0, 0], [0, 1]),
        ("I", 0, [1, 0], [0, 0]), ("I", 1, [0, 0], [1, 0]),
        ("Sdg", 0, [1, 0], [0, 0]), ("Sdg", 1, [0, 0], [0, -1]),
        ("Tdg", 0, [1, 0], [0, 0]), ("Tdg", 1, [0, 0], [r, -r]),
        ("Phase", 0, [1, 0], [0, 0]), ("Phase", 1, [0, 0], [-1, 0]),
    ]
    # single-qubit eigenstates: (labels, eigenvalue, preparation) and Bell-state correlations
    eig = [("X", 1, "H"), ("Y", 1, "H,S"), ("Y", -1, "H,Sdg"), ("Z", -1, "X"), ("Z", 1, "")]
    bell = [("XX", 1), ("YY", -1), ("ZZ", 1), ("ZI", 0), ("IZ", 0)]
    # complete depolarization (p = 1): draw -> Pauli branch (0 identity, 1 X, 2 Y, 3 Z)
    depol = [(0.0, 1), (0.25, 2), (0.5, 3), (0.75, 0)]
    return {"columns": cols, "angle": math.pi, "eigen": eig, "bell": bell, "depolarizing_p1": depol}


def dense_random() -> dict:
    out = {}
    idx = 0
    for qubits in range(1, 6):
        for seed in range(3):
            c = random_circuit(qubits, 40 + 10 * qubits, seed=1000 * qubits + seed)
            psi0 = random_state(qubits, seed=7 + 100 * qubits + seed)
            final = dm.run(c, psi0)
            for k, v in circuit_to_arrays(c).items():
                out[f"c{idx}_{k}"] = v
            out[f"c{idx}_qubits"] = np.int32(qubits)
            out[f"c{idx}_initial"] = psi0
            out[f"c{idx}_final"] = final.astype(np.complex128)
            idx += 1
    out["count"] = np.int32(idx)
    return out


def hamiltonians() -> dict:
    rng = np.random.default_rng(424242)
    out = {}
    idx = 0
    for qubits in range(1, 5):
        for _ in range(3):
            nterms = int(rng.integers(1, 7))
            labels = ["".join(rng.choice(list("IXYZ"), size=qubits)) for _ in range(nterms)]
            coeffs = rng.normal(size=nterms)
            coeffs[rng.random(nterms) < 0.2] = 0.0
            psi = random_state(qubits, seed=int(rng.integers(1 << 30)))
            # an unnormalised state: energies are normalised by the Born mass
            psi = psi * (0.5 + rng.random())
            energy = sum(c * dm.expectation(psi, lab) for c, lab in zip(coeffs, labels) if c != 0)
            out[f"h{idx}_qubits"] = np.int32(qubits)
            out[f"h{idx}_labels"] = np.array(labels)
            out[f"h{idx}_coeffs"] = coeffs
            out[f"h{idx}_state"] = psi.astype(np.complex128)
            out[f"h{idx}_energy"] = np.float64(energy)
            out[f"h{idx}_per_term"] = np.array([dm.expectation(psi, lab) for lab in labels])
            idx += 1
    out["count"] = np.int32(idx)
    return out


def main() -> None:
    (HERE / "known_answers.json").write_text(json.dumps(known_answers(), indent=1) + "\n")
    np.savez_compressed(HERE / "dense_random.npz", **dense_random())
    np.savez_compressed(HERE / "hamiltonians.npz", **hamiltonians())
    print("wrote", sorted(p.name for p in HERE.iterdir() if p.suffix in (".json", ".npz")))


if __name__ == "__main__":
    main()
