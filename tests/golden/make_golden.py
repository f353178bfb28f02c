"""Generates tests/golden/known_answers.json and tests/golden/circuits.json.

known_answers.json holds the known-answer checks that the reference's own
self-checking demo suites and docstrings state (each entry cites its source
file:line inside the SmoQ.jl tree); the values are the analytic answers those
sources assert, not outputs of this project's code.

circuits.json holds the shared random benchmark circuits of
SmoQ.jl_benchmarks/benchmark_random_circuit_sampling: the reference generates
them with Python's random.Random(42) by the algorithm in its
generate_circuits.py:25-87 (1000 gates per N, 70 % single-qubit gates drawn
from H X Y Z S T RX RY RZ, two-qubit gates CNOT/CZ on distinct qubits,
rotation angles uniform in [0, 2*pi) printed with 15 decimals).  The
algorithm is restated here and re-run; `--verify DIR` compares the result
line by line with the reference's committed circuit_N*.txt files.

    python tests/golden/make_golden.py [--verify <circuits dir>]
"""
import json
import math
import os
import random
import sys

HERE = os.path.dirname(os.path.abspath(__file__))


def gen_circuits(seed=42, n_gates=1000, n_range=range(2, 22, 2), single_ratio=0.7):
    single = ["H", "X", "Y", "Z", "S", "T", "RX", "RY", "RZ"]
    two = ["CNOT", "CZ"]
    rot = {"RX", "RY", "RZ"}
    rng = random.Random(seed)
    out = {}
    for n in n_range:
        lines = []
        for _ in range(n_gates):
            if rng.random() < single_ratio or n == 1:
                g = rng.choice(single)
                q = rng.randint(0, n - 1)
                if g in rot:
                    th = rng.uniform(0, 2 * 3.141592653589793)
                    lines.append(f"{g} {q} {th:.15f}")
                else:
                    lines.append(f"{g} {q}")
            else:
                g = rng.choice(two)
                q1 = rng.randint(0, n - 1)
                q2 = rng.randint(0, n - 2)
                if q2 >= q1:
                    q2 += 1
                lines.append(f"{g} {q1} {q2}")
        out[n] = lines
    return out


def known_answers():
    r2 = 1 / math.sqrt(2)
    ka = {
        # demo_parametrized_gates.jl:146-153 -- R(theta)|0> analytic, tol 1e-10
        "rotations_on_zero": {
            "source": "scripts_variational_quantum_circuits/demo_parametrized_gates.jl:146-153",
            "tol": 1e-10,
            "cases": [
                {"gate": "ry", "theta": math.pi / 2, "psi": [[r2, 0], [r2, 0]]},
                {"gate": "ry", "theta": math.pi, "psi": [[0, 0], [1, 0]]},
                {"gate": "rx", "theta": math.pi / 2, "psi": [[r2, 0], [0, -r2]]},
                {"gate": "rx", "theta": math.pi, "psi": [[0, 0], [0, -1]]},
                {"gate": "rz", "theta": math.pi / 2, "psi": [[math.cos(math.pi / 4), -math.sin(math.pi / 4)], [0, 0]]},
            ],
        },
        # demo_parametrized_gates.jl:208-244 / test_summary.txt:226-227 -- H^N|0> = uniform
        "hadamard_all_uniform": {"source": "scripts_variational_quantum_circuits/demo_parametrized_gates.jl:208-244",
                                 "N": [10, 12], "fidelity": 1.0, "tol": 1e-10},
        # demo_parametrized_gates.jl:496-518 -- Ry(pi/2)^2 == Ry(pi) on every qubit
        "ry_half_squared": {"source": "scripts_variational_quantum_circuits/demo_parametrized_gates.jl:496-518",
                            "N": [10, 14], "fidelity": 1.0, "tol": 1e-10},
        # demo_parametrized_gates.jl:529-550 -- norm after Ry(pi/4) on all qubits
        "norm_after_ry": {"source": "scripts_variational_quantum_circuits/demo_parametrized_gates.jl:529-550",
                          "N": [16, 18], "theta": math.pi / 4, "norm": 1.0, "tol": 1e-10},
        # cpuQuantumStateObservables.jl:166-173, 298-304 -- Bell state (|00>+|11>)/sqrt2
        "bell": {"source": "utils/cpu/cpuQuantumStateObservables.jl:166-173,298-304",
                 "z1": 0.0, "zz": 1.0, "xx": 1.0, "yy": -1.0},
        # cpuQuantumStateObservables.jl:823-835 -- GHZ_3 (|000>+|111>)/sqrt2.  The
        # docstring claims <Z1Z2Z3> = 1, but its own _expect_pauli_Z_string loop
        # (:900-930) gives 0 (|111> has odd parity); the fixture keeps the value the
        # reference's code computes.  <XXX> = 1 as the docstring states (the
        # mixed-string loop at :948 returns half of it, 0.5).
        "ghz3": {"source": "utils/cpu/cpuQuantumStateObservables.jl:823-835,900-930",
                 "zzz": 0.0, "x1z2": 0.0, "xxx": 1.0, "xxx_reference_mixed_loop": 0.5},
        # cpuQuantumStateObservables.jl:368-375 -- |+>|+>: <XX> = 1
        "plus_plus_xx": {"source": "utils/cpu/cpuQuantumStateObservables.jl:368-375", "xx": 1.0},
        # demo_VQC_base_test.jl:119-136 -- parameter shift vs central FD (eps 1e-5), tol 1e-4
        "ps_vs_fd": {"source": "scripts_variational_quantum_circuits/demo_VQC_base_test.jl:119-136",
                     "eps": 1e-5, "tol": 1e-4},
        # demo_parametrized_gates.jl:1040-1057 -- psi vs rho observables, tol 1e-12
        "psi_vs_rho_observables": {"source": "scripts_variational_quantum_circuits/demo_parametrized_gates.jl:1040-1057",
                                   "tol": 1e-12},
    }
    return ka


def main():
    ka = known_answers()
    with open(os.path.join(HERE, "known_answers.json"), "w") as f:
        json.dump(ka, f, indent=1)
    circ = gen_circuits()
    with open(os.path.join(HERE, "circuits.json"), "w") as f:
        json.dump({str(k): v for k, v in circ.items()}, f)
    if "--verify" in sys.argv:
        d = sys.argv[sys.argv.index("--verify") + 1]
        bad = 0
        for n, lines in circ.items():
            with open(os.path.join(d, f"circuit_N{n:02d}.txt")) as f:
                ref = [l.strip() for l in f if l.strip() and not l.startswith("#")]
            if ref != lines:
                bad += 1
                print(f"N={n}: MISMATCH")
            else:
                print(f"N={n}: identical ({len(lines)} gates)")
        sys.exit(1 if bad else 0)


if __name__ == "__main__":
    main()
