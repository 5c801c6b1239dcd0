"""Generate the golden fixtures of tests/golden/ from the reference itself.

Runs each case of tests/golden_cases.py through ESyS-Particle's own hot-path
classes (oracle/_ref/libesys_ref.so, built from the reference sources by
`make -C oracle ref`) and stores every particle field, pair set, pair state,
wall and bond-break record as <case>.npz.

    python tests/golden/make_golden.py
"""
import os
import subprocess
import sys

import numpy as np

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(os.path.dirname(HERE))
sys.path[:0] = [os.path.join(ROOT, "oracle"), os.path.join(ROOT, "tests")]

import golden_cases  # noqa: E402
import oracle  # noqa: E402


def main():
    subprocess.run(["make", "-s", "-j8", "-C", os.path.join(ROOT, "oracle"), "ref"], check=True)
    for name in golden_cases.CASES:
        sim = golden_cases.run(name, lambda *a: oracle.OracleSim("ref", *a))
        out = golden_cases.collect(name, sim)
        np.savez_compressed(os.path.join(HERE, name + ".npz"), **out)
        print(name, {k: v.shape for k, v in out.items()})


if __name__ == "__main__":
    main()
