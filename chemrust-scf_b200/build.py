"""Build the B200 ChFSI library (and, for tests, the CPU oracle) in-tree.

    python chemrust-scf_b200/build.py            # library + oracle
    python chemrust-scf_b200/build.py --lib      # library only

The library is compiled for sm_100a only (nvcc -gencode
arch=compute_100a,code=sm_100a) and linked into
chemrust-scf_b200/libchfsi_b200.so.  The oracle (test infrastructure) is
built by oracle/build_oracle.py.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libchfsi_b200.so")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
CUDA_FLAGS = [
    "-std=c++17", "-O3", "-lineinfo",
    "-gencode", "arch=compute_100a,code=sm_100a",
    "-Xcompiler", "-fPIC", "-Xcompiler", "-fopenmp",
    "-I", INCLUDE, "-I", CSRC,
]
CXX_FLAGS = ["-std=c++17", "-O3", "-fPIC", "-fopenmp", "-I", INCLUDE, "-I", CSRC,
             "-I", "/usr/local/cuda/include"]


def _sources():
    cu = sorted(f for f in os.listdir(CSRC) if f.endswith(".cu"))
    cpp = sorted(f for f in os.listdir(CSRC) if f.endswith(".cpp"))
    return cu, cpp


def _headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".hpp", ".cuh", ".h"))]
    hs += [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE)]
    return hs


def _stale(obj, src, headers):
    if not os.path.exists(obj):
        return True
    t = os.path.getmtime(obj)
    return any(os.path.getmtime(p) > t for p in [src] + headers)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("command failed: %s\n%s%s" % (" ".join(cmd), r.stdout, r.stderr))
    return r


def build_library(verbose=False):
    os.makedirs(BUILD, exist_ok=True)
    cu, cpp = _sources()
    headers = _headers()
    jobs, objs = [], []
    for f in cu:
        src, obj = os.path.join(CSRC, f), os.path.join(BUILD, f + ".o")
        objs.append(obj)
        if _stale(obj, src, headers):
            jobs.append([NVCC] + CUDA_FLAGS + ["-c", src, "-o", obj])
    for f in cpp:
        src, obj = os.path.join(CSRC, f), os.path.join(BUILD, f + ".o")
        objs.append(obj)
        if _stale(obj, src, headers):
            jobs.append(["g++"] + CXX_FLAGS + ["-c", src, "-o", obj])
    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        for cmd, _ in zip(jobs, ex.map(_run, jobs)):
            if verbose:
                print(" ".join(cmd))
    if jobs or not os.path.exists(LIB) or any(os.path.getmtime(o) > os.path.getmtime(LIB) for o in objs):
        cmd = [NVCC, "-shared", "-gencode", "arch=compute_100a,code=sm_100a", "-o", LIB] + objs + \
              ["-Xcompiler", "-fopenmp", "-lgomp"]
        _run(cmd)
        if verbose:
            print(" ".join(cmd))
    return LIB


def main():
    verbose = "-v" in sys.argv
    print(build_library(verbose))
    if "--lib" not in sys.argv:
        sys.path.insert(0, os.path.join(ROOT, "oracle"))
        import build_oracle  # noqa: E402
        print(build_oracle.build(verbose))


if __name__ == "__main__":
    main()
