"""Compile the oracle's C restatement (test infrastructure only).

Outputs oracle/_build/libbnzoracle.so (MHD, MFIELD=1) and
oracle/_build/libbnzoracle_hydro.so (hydro, MFIELD=0).  The flags keep IEEE
double arithmetic in source order (no contraction into FMA, no fast-math) so
the restated kernels match the reference's compiled kernels bit for bit.
"""
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
OUT = os.path.join(HERE, "_build")
CFLAGS = ["-std=gnu11", "-O2", "-ffp-contract=off", "-fno-fast-math", "-fPIC", "-fopenmp",
          "-Wall", "-Wno-unknown-pragmas"]


def build(quiet=False):
    os.makedirs(OUT, exist_ok=True)
    src = os.path.join(HERE, "bnz_oracle.c")
    for mfield, name in ((1, "libbnzoracle.so"), (0, "libbnzoracle_hydro.so")):
        lib = os.path.join(OUT, name)
        cmd = ["gcc"] + CFLAGS + ["-DORC_MFIELD=%d" % mfield, "-shared", "-o", lib, src, "-lm"]
        subprocess.run(cmd, check=True)
        if not quiet:
            print("oracle: built", lib)
    return True


if __name__ == "__main__":
    sys.exit(0 if build() else 1)
