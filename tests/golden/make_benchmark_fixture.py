"""Known answers of the reference's benchmark.dat (converged ground states,
m = hbar = 1) as a fixture: the harmonic-trap block (V = x^2 / 2) and the
harmonic + Gaussian barrier block (V = x^2 / 2 + b^2 exp(-x^2 / 2c^2),
b = 3, c = 0.5).  The ring block is left out (its ring length is not given).

    python tests/golden/make_benchmark_fixture.py [path/to/benchmark.dat]

The default path is benchmark.dat of the reference tree named by
$MCTDHB_REFERENCE, else of the `reference` folder beside this repository.
"""
import json
import os
import sys


def parse(path):
    blocks, cur = {"harmonic": [], "barrier": []}, None
    for ln in open(path):
        if "HARMONIC TRAP TESTS" in ln:
            cur = "harmonic"
        elif "GAUSSIAN BARRIER" in ln:
            cur = "barrier"
        elif "RING" in ln:
            cur = None
        if cur is None or not ln.strip() or ln.lstrip().startswith("#"):
            continue
        t = ln.split()
        row = {"npar": int(t[0]), "norb": int(t[1]), "g": float(t[2]), "e_per_n": float(t[3]),
               "sqrt_r2": float(t[4]), "condensate": float(t[-1].rstrip("%")) / 100.0}
        blocks[cur].append(row)
    return blocks


if __name__ == "__main__":
    repo = os.path.dirname(os.path.dirname(os.path.dirname(os.path.abspath(__file__))))
    ref = os.environ.get("MCTDHB_REFERENCE") or os.path.join(os.path.dirname(repo), "reference")
    src = sys.argv[1] if len(sys.argv) > 1 else os.path.join(ref, "benchmark.dat")
    out = os.path.join(os.path.dirname(os.path.abspath(__file__)), "benchmark_known_answers.json")
    with open(out, "w") as f:
        json.dump({"source": "benchmark.dat of the reference", **parse(src)}, f, indent=1)
    print(out)
