"""Build libpoisson_recon_b200.so in-tree with nvcc for sm_100a (B200).

    python -m poissonreconstruction_b200.build [--force] [-j N]

Objects go to _build/ at the repository root; the shared library is written next to
this file, where the Python wrapper and the tests load it.
"""
import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

HERE = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(HERE)
CSRC = os.path.join(HERE, "csrc")
BUILD = os.path.join(ROOT, "_build")
LIB = os.path.join(HERE, "libpoisson_recon_b200.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xptxas", "-O3",
              "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include")]


def nvcc():
    for cand in (os.environ.get("NVCC"), "/usr/local/cuda/bin/nvcc", shutil.which("nvcc")):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


CXX_FLAGS = ["-O3", "-std=c++17", "-fPIC", "-Wall", "-I", os.path.join(ROOT, "include")]
CLI_SRC = os.path.join(HERE, "cli", "poisson_recon_cli.cpp")
CLI = os.path.join(HERE, "poisson-recon")


def sources():
    """Library sources: CUDA (.cu, nvcc) and host-only C++ (.cpp, g++)."""
    return sorted(os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cu", ".cpp")))


def headers():
    hs = [os.path.join(CSRC, f) for f in os.listdir(CSRC) if f.endswith((".cuh", ".inc", ".h"))]
    hs.append(os.path.join(ROOT, "include", "poisson_recon.h"))
    return hs


def _stale(target, deps):
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps)


def compile_one(src, force, extra):
    obj = os.path.join(BUILD, os.path.splitext(os.path.basename(src))[0] + ".o")
    if force or _stale(obj, [src] + headers()):
        if src.endswith(".cpp"):
            cmd = [os.environ.get("CXX_HOST", "g++")] + CXX_FLAGS + ["-c", src, "-o", obj]
        else:
            cmd = [nvcc()] + ARCH + NVCC_FLAGS + extra + ["-c", src, "-o", obj]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("nvcc failed for %s:\n%s\n%s" % (src, " ".join(cmd), r.stderr))
        if r.stderr.strip():
            sys.stderr.write(r.stderr)
    return obj


def build(force=False, jobs=None, extra=()):
    os.makedirs(BUILD, exist_ok=True)
    srcs = sources()
    with cf.ThreadPoolExecutor(max_workers=jobs or min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: compile_one(s, force, list(extra)), srcs))
    if force or _stale(LIB, objs):
        cmd = [nvcc()] + ARCH + ["-shared", "-o", LIB] + objs + ["-lcudart_static", "-lrt", "-ldl", "-lpthread"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("link failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    build_cli(force)
    return LIB


def build_cli(force=False):
    """The `poisson-recon` command (the crate's CLI, src/main.rs), linked against the library."""
    if force or _stale(CLI, [CLI_SRC, LIB, os.path.join(ROOT, "include", "poisson_recon.h")]):
        cmd = [os.environ.get("CXX_HOST", "g++"), "-O2", "-std=c++17", "-Wall", "-I", os.path.join(ROOT, "include"),
               CLI_SRC, "-o", CLI, "-L" + HERE, "-lpoisson_recon_b200", "-Wl,-rpath,$ORIGIN"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError("CLI build failed:\n%s\n%s" % (" ".join(cmd), r.stderr))
    return CLI


def main():
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", type=int, default=None)
    ap.add_argument("--ptxas-verbose", action="store_true")
    a = ap.parse_args()
    extra = ["-Xptxas", "-v"] if a.ptxas_verbose else []
    print(build(force=a.force or a.ptxas_verbose, jobs=a.j, extra=extra))


if __name__ == "__main__":
    main()
