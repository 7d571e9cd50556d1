"""Build the CPU oracle (test infrastructure only) into oracle/liboracle.so.

The oracle is a C++/OpenMP restatement of the chemrust-scf ChFSI path used
by tests/, __graft_entry__.smoke() and bench.py's CPU baseline.  It is built
for x86-64-v3 (AVX2/FMA) so the binary built here also runs on the GPU host.
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
SRC = os.path.join(HERE, "oracle.cpp")
LIB = os.path.join(HERE, "liboracle.so")


def build(verbose=False):
    if os.path.exists(LIB) and os.path.getmtime(LIB) >= os.path.getmtime(SRC):
        return LIB
    cmd = ["g++", "-std=c++17", "-O3", "-march=x86-64-v3", "-fopenmp", "-shared", "-fPIC",
           SRC, "-o", LIB]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
    if verbose:
        print(" ".join(cmd))
    return LIB


if __name__ == "__main__":
    print(build(True))
