"""Build libxmatch_b200.so (sm_100a) in-tree.

    python xmatch_b200/build.py         # (the package itself needs the library to import)

Every CUDA source is compiled for sm_100a only; host code is compiled with
-ffp-contract=off so host-side FP64 formulas (RA half-width, thresholds)
round exactly like their written form.
"""
import os
import subprocess
import sys
from concurrent.futures import ThreadPoolExecutor

HERE = os.path.dirname(os.path.abspath(__file__))
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(HERE, "_build")
LIB = os.path.join(HERE, "libxmatch_b200.so")
CLI = os.path.join(HERE, "bin", "xmatch")

NVCC = os.environ.get("NVCC", "nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC,-ffp-contract=off,-O2",
                  "-Xptxas", "-warn-spills", "--expt-relaxed-constexpr", "-I" + os.path.join(HERE, "..", "include")]
CXXFLAGS = ["-O2", "-fPIC", "-std=c++17", "-ffp-contract=off", "-Wall", "-I" + os.path.join(HERE, "..", "include")]

CU_SOURCES = ["xm_scan.cu", "xm_build.cu", "xm_match.cu", "xm_batch.cu", "xm_api.cu", "xm_serve.cu"]
CXX_SOURCES = ["xm_io.cpp"]


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError("compile failed: " + cmd[-1])
    return r.stdout + r.stderr


def _stale(out, srcs):
    if not os.path.exists(out):
        return True
    t = os.path.getmtime(out)
    return any(os.path.getmtime(s) > t for s in srcs)


def build(verbose=False, force=False):
    os.makedirs(BUILD, exist_ok=True)
    headers = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".h", ".cuh"))]
    headers.append(os.path.join(HERE, "..", "include", "xmatch.h"))
    jobs = []
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            jobs.append([NVCC] + NVFLAGS + ["-c", s, "-o", o])
    for src in CXX_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(BUILD, src + ".o")
        objs.append(o)
        if force or _stale(o, [s] + headers):
            jobs.append(["g++"] + CXXFLAGS + ["-c", s, "-o", o])
    with ThreadPoolExecutor(max_workers=min(8, max(1, len(jobs)))) as ex:
        outs = list(ex.map(_run, jobs))
    if verbose:
        for o in outs:
            if o.strip():
                print(o)
    if force or jobs or _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs + ["-lpthread"])
    # command-line driver (xm_cli.cpp) linked against the library, found next to it at run time
    cli_src = os.path.join(CSRC, "xm_cli.cpp")
    if force or _stale(CLI, [cli_src, LIB] + headers):
        os.makedirs(os.path.dirname(CLI), exist_ok=True)
        _run(["g++"] + CXXFLAGS + [cli_src, "-o", CLI, "-L" + HERE, "-lxmatch_b200", "-Wl,-rpath,$ORIGIN/..",
                                   "-lpthread"])
    return LIB


if __name__ == "__main__":
    build(verbose="-v" in sys.argv, force="-f" in sys.argv)
    print(LIB)
