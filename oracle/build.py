"""Build recipe for the oracle's C restatement (test infrastructure only).

Compiles ``oracle/kernels.c`` into ``oracle/_build/liboracle.so`` with gcc
and OpenMP. The output directory is git-ignored; the built library travels
with the working tree like the CUDA library does.
"""

import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "kernels.c")
OUT_DIR = os.path.join(HERE, "_build")
OUT = os.path.join(OUT_DIR, "liboracle.so")


def build(force=False, verbose=False):
    """Compile the oracle library if it is missing or older than its source."""
    os.makedirs(OUT_DIR, exist_ok=True)
    if (
        not force
        and os.path.exists(OUT)
        and os.path.getmtime(OUT) >= os.path.getmtime(SRC)
    ):
        return OUT
    cmd = [
        "gcc",
        "-O2",
        "-fPIC",
        "-shared",
        "-fopenmp",
        "-ffp-contract=off",
        "-o",
        OUT,
        SRC,
        "-lm",
    ]
    if verbose:
        print(" ".join(cmd))
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force=True, verbose=True))
