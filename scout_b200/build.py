"""Build recipe for scout-b200 (in-tree, no JIT cache).

Outputs
  scout_b200/lib/libscout.so   host C++ (OpenMP) + sm_100a CUDA kernels + both C ABIs
  bin/scout_{mis,coloring,bfs,cc}  drop-in CLIs with the reference's 5 positional arguments
  oracle/liboracle.so          CPU checker used by the tests (test infrastructure)
  oracle/_ref/*                the reference's own binaries, compiled from its sources by
                               oracle/build_ref.sh when the reference tree is present

Usage: python -m scout_b200.build [--force] [--no-ref]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys

ROOT = os.path.dirname(os.path.dirname(os.path.abspath(__file__)))
PKG = os.path.join(ROOT, "scout_b200")
CSRC = os.path.join(PKG, "csrc")
LIBDIR = os.path.join(PKG, "lib")
OBJDIR = os.path.join(ROOT, "_build")
BINDIR = os.path.join(ROOT, "bin")
ORACLE = os.path.join(ROOT, "oracle")
INCLUDE = os.path.join(ROOT, "include")

NVCC = os.environ.get("NVCC", "nvcc")
CXX = os.environ.get("CXX", "g++")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
CXXFLAGS = ["-O3", "-std=c++17", "-fPIC", "-fopenmp", "-Wall", "-Wno-unused-function", f"-I{INCLUDE}"]
NVFLAGS = ARCH + ["-O3", "-std=c++17", "-lineinfo", "-Xcompiler", "-fPIC", "-Xcompiler", "-fopenmp",
                  "--expt-relaxed-constexpr", f"-I{INCLUDE}", "-Xptxas", "-warn-spills"]


def _sources(sub: str, ext: str) -> list[str]:
    d = os.path.join(CSRC, sub)
    if not os.path.isdir(d):
        return []
    return sorted(os.path.join(d, f) for f in os.listdir(d) if f.endswith(ext))


def _headers() -> list[str]:
    hs = [os.path.join(INCLUDE, f) for f in os.listdir(INCLUDE) if f.endswith(".h")]
    for sub in ("host", "cuda", "cli"):
        d = os.path.join(CSRC, sub)
        if os.path.isdir(d):
            hs += [os.path.join(d, f) for f in os.listdir(d) if f.endswith((".hpp", ".cuh", ".h"))]
    return hs


def _stale(target: str, deps: list[str]) -> bool:
    if not os.path.exists(target):
        return True
    t = os.path.getmtime(target)
    return any(os.path.getmtime(d) > t for d in deps if os.path.exists(d))


def _run(cmd: list[str]) -> None:
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(" ".join(cmd) + "\n" + r.stdout + r.stderr)
        raise RuntimeError(f"build step failed: {os.path.basename(cmd[-1])}")
    if r.stderr.strip():
        sys.stderr.write(r.stderr)


def _compile(src: str, force: bool) -> str:
    obj = os.path.join(OBJDIR, os.path.basename(src) + ".o")
    if force or _stale(obj, [src] + _headers()):
        if src.endswith(".cu"):
            _run([NVCC] + NVFLAGS + ["-c", src, "-o", obj])
        else:
            _run([CXX] + CXXFLAGS + ["-c", src, "-o", obj])
    return obj


def build_lib(force: bool = False) -> str:
    os.makedirs(OBJDIR, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = _sources("host", ".cpp") + _sources("cuda", ".cu")
    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 4)) as ex:
        objs = list(ex.map(lambda s: _compile(s, force), srcs))
    lib = os.path.join(LIBDIR, "libscout.so")
    if force or _stale(lib, objs):
        # cudart is linked statically so the library does not depend on which libcudart the
        # host process (for instance torch) has already loaded.
        _run([NVCC] + ARCH + ["-shared", "-cudart", "static", "-o", lib] + objs + ["-Xcompiler", "-fopenmp", "-lgomp"])
    return lib


def build_cli(force: bool = False) -> list[str]:
    src = os.path.join(CSRC, "cli", "scout_main.cpp")
    if not os.path.exists(src):
        return []
    os.makedirs(BINDIR, exist_ok=True)
    lib = os.path.join(LIBDIR, "libscout.so")
    outs = []
    for p in ("mis", "coloring", "bfs", "cc"):
        out = os.path.join(BINDIR, f"scout_{p}")
        if force or _stale(out, [src, lib] + _headers()):
            flags = [f for f in CXXFLAGS if f != "-fopenmp"]   # the CLI itself has no OpenMP region
            _run([CXX] + flags + [f"-DSCOUT_PROBLEM_NAME=\"{p}\"", src, "-o", out, f"-L{LIBDIR}", "-lscout",
                                     f"-Wl,-rpath,{LIBDIR}", "-Wl,-rpath,$ORIGIN/../scout_b200/lib"])
        outs.append(out)
    return outs


def build_oracle(force: bool = False) -> str:
    srcs = [os.path.join(ORACLE, f) for f in ("oracle.cpp", "cpu_recompute.cpp")]
    out = os.path.join(ORACLE, "liboracle.so")
    if force or _stale(out, srcs):
        os.makedirs(OBJDIR, exist_ok=True)
        objs = []
        for src in srcs:   # OpenMP at compile time, libgomp named at link time
            obj = os.path.join(OBJDIR, "oracle_" + os.path.basename(src) + ".o")
            _run([CXX, "-O2", "-std=c++17", "-fPIC", "-fopenmp", "-Wall", "-c", src, "-o", obj])
            objs.append(obj)
        _run([CXX, "-shared"] + objs + ["-l:libgomp.so.1", "-o", out])
    return out


def reference_dir() -> str:
    """The reference tree: $SCOUT_REFERENCE_DIR, else a `reference` directory beside the
    repository root (absent on machines that only run the prebuilt files)."""
    return os.environ.get("SCOUT_REFERENCE_DIR") or os.path.join(os.path.dirname(ROOT), "reference")


def build_reference(force: bool = False) -> None:
    """Compiles the reference's binaries from its own sources (checker only)."""
    script = os.path.join(ORACLE, "build_ref.sh")
    ref = reference_dir()
    if not (os.path.exists(script) and os.path.isdir(ref)):
        return
    env = dict(os.environ, SCOUT_REFERENCE_DIR=ref, FORCE="1" if force else "0")
    r = subprocess.run(["bash", script], env=env, capture_output=True, text=True)
    if r.returncode != 0:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("oracle/build_ref.sh failed")


def build_all(force: bool = False, reference: bool = True) -> None:
    build_lib(force)
    build_cli(force)
    build_oracle(force)
    if reference:
        build_reference(force)


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--no-ref", action="store_true")
    a = ap.parse_args()
    if shutil.which(NVCC) is None:
        raise SystemExit("nvcc not found")
    build_all(a.force, not a.no_ref)
    print("built", os.path.join(LIBDIR, "libscout.so"))


if __name__ == "__main__":
    main()
