"""Build the sedi_b200 native library and tools in-tree for sm_100a.

    python -m sedi_b200.build            # library + CLI
    python -m sedi_b200.build --clean

Outputs (git-ignored, shipped with the tree):
    sedi_b200/_lib/libsedi_b200.so   C ABI declared in include/sedi_b200.h
    sedi_b200/_lib/sedi              command-line driver (reference CLI)
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
REPO = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
OUT = os.path.join(HERE, "_lib")
OBJ = os.path.join(OUT, "obj")
LIB = os.path.join(OUT, "libsedi_b200.so")
CLI = os.path.join(OUT, "sedi")

NVCC = os.environ.get("NVCC", shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVFLAGS = ARCH + ["-lineinfo", "-O3", "-std=c++17", "--extended-lambda", "-Xcompiler", "-fPIC",
                  "-I" + os.path.join(REPO, "include")]

CU_SOURCES = ["plain.cu", "batched.cu", "rng.cu", "capi.cu", "noalloc.cu", "serve.cu", "selftest.cu", "slab.cu"]


def _run(cmd):
    r = subprocess.run(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout)
        raise SystemExit("build failed")
    return r.stdout


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def build(verbose=False, ptxas_info=False):
    os.makedirs(OBJ, exist_ok=True)
    headers = [os.path.join(CSRC, h) for h in os.listdir(CSRC) if h.endswith((".cuh", ".h"))]
    headers.append(os.path.join(REPO, "include", "sedi_b200.h"))
    jobs = []
    objs = []
    for src in CU_SOURCES:
        s = os.path.join(CSRC, src)
        o = os.path.join(OBJ, src + ".o")
        objs.append(o)
        if _stale(o, [s] + headers):
            extra = ["-Xptxas", "-v"] if ptxas_info else []
            jobs.append([NVCC] + NVFLAGS + extra + ["-c", s, "-o", o])
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        for out in ex.map(_run, jobs):
            if verbose and out:
                print(out)
    if _stale(LIB, objs):
        _run([NVCC] + ARCH + ["-shared", "-o", LIB] + objs)
    cli_src = os.path.join(CSRC, "sedi_cli.cc")
    if os.path.exists(cli_src) and _stale(CLI, [cli_src, LIB] + headers):
        _run(["g++", "-std=c++17", "-O2", "-I" + os.path.join(REPO, "include"), cli_src, "-o", CLI,
              "-L" + OUT, "-lsedi_b200", "-Wl,-rpath,$ORIGIN"])
    return LIB


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--clean", action="store_true")
    ap.add_argument("-v", action="store_true")
    ap.add_argument("--ptxas", action="store_true")
    a = ap.parse_args()
    if a.clean and os.path.isdir(OUT):
        shutil.rmtree(OUT)
    print(build(verbose=a.v or a.ptxas, ptxas_info=a.ptxas))


if __name__ == "__main__":
    main()
