"""Build recipe of the CPU oracle (test infrastructure): oracle.cpp -> _build/liboracle.so.

Strict IEEE evaluation (-ffp-contract=off) and a portable x86-64-v3 target so the library
built here also loads on the GPU hosts.
"""
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "oracle.cpp")
OUT = os.path.join(HERE, "_build", "liboracle.so")


def build(force: bool = False) -> str:
    os.makedirs(os.path.dirname(OUT), exist_ok=True)
    hdr = os.path.join(HERE, "..", "include", "icefem_b200.h")
    deps = [SRC, hdr] + glob.glob(os.path.join(HERE, "*.inc"))
    if not force and os.path.exists(OUT) and os.path.getmtime(OUT) >= max(os.path.getmtime(p) for p in deps):
        return OUT
    cmd = ["g++", "-std=c++17", "-O3", "-march=x86-64-v3", "-ffp-contract=off", "-fPIC", "-shared",
           "-pthread", "-Wall", "-Wno-unused-variable", "-o", OUT, SRC]
    subprocess.run(cmd, check=True)
    return OUT


if __name__ == "__main__":
    print(build(force="--force" in sys.argv))
