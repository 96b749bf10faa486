"""Builds libcurfil_b200.so in-tree with nvcc for sm_100a (B200).

Each csrc/*.cu is compiled to an object under curfil_b200/_build/ (skipped when up to date),
then linked into curfil_b200/libcurfil_b200.so with the CUDA runtime linked statically.
"""
import concurrent.futures
import glob
import os
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libcurfil_b200.so")
NVCC = os.environ.get("NVCC", "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC,-O2", "-ccbin", "g++",
         "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include")]


def _headers():
    return glob.glob(os.path.join(CSRC, "*.h")) + glob.glob(os.path.join(CSRC, "*.cuh")) + \
        glob.glob(os.path.join(ROOT, "include", "*.h"))


def _compile(src, extra):
    obj = os.path.join(BUILD, os.path.basename(src) + ".o")
    newest_dep = max([os.path.getmtime(src)] + [os.path.getmtime(h) for h in _headers()])
    if os.path.exists(obj) and os.path.getmtime(obj) >= newest_dep:
        return obj, None
    cmd = [NVCC] + ARCH + FLAGS + extra + ["-c", src, "-o", obj]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        return obj, "compile failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr)
    return obj, None


def build(verbose=False, extra=()):
    os.makedirs(BUILD, exist_ok=True)
    sources = sorted(glob.glob(os.path.join(CSRC, "*.cu")))
    extra = list(extra)
    with concurrent.futures.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        results = list(ex.map(lambda s: _compile(s, extra), sources))
    errors = [e for _, e in results if e]
    if errors:
        raise RuntimeError("\n".join(errors))
    objs = [o for o, _ in results]
    if not os.path.exists(LIB) or os.path.getmtime(LIB) < max(os.path.getmtime(o) for o in objs):
        cmd = [NVCC] + ARCH + ["-shared", "-Xcompiler", "-fPIC", "-ccbin", "g++", "-o", LIB] + objs + ["-lpthread", "-lz"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed: %s\n%s\n%s" % (" ".join(cmd), r.stdout, r.stderr))
    if verbose:
        print("built", LIB)
    return LIB


def ptxas_report(source):
    """Registers / spills / shared memory of one source file (nvcc -Xptxas -v)."""
    cmd = [NVCC] + ARCH + FLAGS + ["-Xptxas", "-v", "-c", os.path.join(CSRC, source), "-o", os.devnull]
    r = subprocess.run(cmd, capture_output=True, text=True)
    return r.stdout + r.stderr


if __name__ == "__main__":
    if len(sys.argv) > 1 and sys.argv[1] == "ptxas":
        print(ptxas_report(sys.argv[2]))
    else:
        build(verbose=True)
