"""Build the CPU oracle (test infrastructure only) into oracle/liboracle.so.

The oracle is a C++/OpenMP restatement of the chemrust-scf ChFSI path used
by tests/, __graft_entry__.smoke() and bench.py's CPU baseline.  The seeded
generator of the synthetic systems (chemrust-scf_b200/csrc/system.cpp,
plain C++) is compiled in as well, so that the CPU side builds its inputs
without the CUDA library.  Built for x86-64-v3 (AVX2/FMA) so the binary
built here also runs on the GPU host.
"""
import os
import subprocess

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
SRC = os.path.join(HERE, "oracle.cpp")
GEN = os.path.join(ROOT, "chemrust-scf_b200", "csrc", "system.cpp")
DEPS = [SRC, GEN, os.path.join(ROOT, "chemrust-scf_b200", "csrc", "system.hpp"),
        os.path.join(ROOT, "include", "chfsi.h")]
LIB = os.path.join(HERE, "liboracle.so")


def build(verbose=False):
    if os.path.exists(LIB) and all(os.path.getmtime(LIB) >= os.path.getmtime(d) for d in DEPS):
        return LIB
    inc = ["-I", os.path.join(ROOT, "include"), "-I", os.path.join(ROOT, "chemrust-scf_b200", "csrc")]
    gen_obj = os.path.join(HERE, "_system_gen.o")
    # the generator with the CUDA library's own host flags (no -march: the
    # same rounding, so both sides see bit-identical systems)
    cmds = [["g++", "-std=c++17", "-O3", "-fPIC", "-fopenmp"] + inc + ["-c", GEN, "-o", gen_obj],
            ["g++", "-std=c++17", "-O3", "-march=x86-64-v3", "-fopenmp", "-shared", "-fPIC"] + inc +
            [SRC, gen_obj, "-o", LIB]]
    for cmd in cmds:
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("oracle build failed:\n" + r.stdout + r.stderr)
        if verbose:
            print(" ".join(cmd))
    os.remove(gen_obj)
    return LIB


if __name__ == "__main__":
    print(build(True))
