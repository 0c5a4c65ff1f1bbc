"""Compile the CUDA library in-tree for sm_100a.

Produces ``particlebase_b200/lib/libparticlebase_b200.so`` from the sources in
``particlebase_b200/csrc`` with nvcc (no JIT, no torch extension cache), so the
built library travels with the source tree.  Objects go to
``particlebase_b200/_build``.

    python -m particlebase_b200.build [--force] [--verbose]
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import hashlib
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
BUILD = os.path.join(PKG, "_build")
LIBDIR = os.path.join(PKG, "lib")
LIB = os.path.join(LIBDIR, "libparticlebase_b200.so")

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-Xcompiler", "-O3",
              "--expt-relaxed-constexpr", "-I", os.path.join(ROOT, "include"), "-I", CSRC]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def host_cxx() -> str:
    # The image's default CXX may lack OpenMP/spec files; nvcc only needs a
    # plain C++17 host compiler.
    for cand in ("/usr/bin/g++", shutil.which("g++")):
        if cand and os.path.exists(cand):
            return cand
    return "g++"


def sources() -> list[str]:
    out = []
    for f in sorted(os.listdir(CSRC)):
        if f.endswith((".cu", ".cpp")):
            out.append(os.path.join(CSRC, f))
    return out


def _digest(paths: list[str], extra: str) -> str:
    """Content digest of the sources and flags, with paths taken relative to
    the repository, so that a copy of the tree elsewhere keeps its build."""
    h = hashlib.sha256(extra.replace(ROOT, "<root>").encode())
    for p in paths:
        with open(p, "rb") as fh:
            h.update(os.path.relpath(p, ROOT).encode())
            h.update(fh.read())
    return h.hexdigest()


def _headers() -> list[str]:
    hs = [os.path.join(CSRC, f) for f in sorted(os.listdir(CSRC)) if f.endswith((".cuh", ".h"))]
    inc = os.path.join(ROOT, "include", "pb")
    hs += [os.path.join(inc, f) for f in sorted(os.listdir(inc))]
    return hs


def build(force: bool = False, verbose: bool = False) -> str:
    os.makedirs(BUILD, exist_ok=True)
    os.makedirs(LIBDIR, exist_ok=True)
    srcs = sources()
    stamp = os.path.join(BUILD, "stamp")
    dig = _digest(srcs + _headers(), " ".join(ARCH + NVCC_FLAGS))
    if not force and os.path.exists(LIB) and os.path.exists(stamp):
        with open(stamp) as fh:
            if fh.read().strip() == dig:
                return LIB
    cc = nvcc()
    ccbin = ["-ccbin", host_cxx()]

    def compile_one(src: str) -> str:
        obj = os.path.join(BUILD, os.path.basename(src) + ".o")
        cmd = [cc, *ccbin, *ARCH, *NVCC_FLAGS, "-c", src, "-o", obj]
        if src.endswith(".cpp"):
            cmd = [cc, *ccbin, *NVCC_FLAGS, "-x", "c++", "-c", src, "-o", obj]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
            print(" ".join(cmd), flush=True)
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"nvcc failed for {src}:\n{r.stdout}\n{r.stderr}")
        if verbose and r.stderr:
            print(r.stderr, flush=True)
        return obj

    with cf.ThreadPoolExecutor(max_workers=min(8, os.cpu_count() or 1)) as ex:
        objs = list(ex.map(compile_one, srcs))
    tmp = LIB + ".tmp"
    cmd = [cc, *ccbin, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"]
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError(f"link failed:\n{r.stdout}\n{r.stderr}")
    os.replace(tmp, LIB)
    with open(stamp, "w") as fh:
        fh.write(dig)
    return LIB


SHIM = os.path.join(PKG, "shim")
DRIVERS = os.path.join(SHIM, "_drivers")
MD_DRIVERS = ("testMD1", "testMD2", "testMD3", "testMD4", "testMD4n", "calcgr1")


def reference_dir() -> str:
    """The reference checkout: PB_REFERENCE_DIR, else a `reference` directory
    beside this repository."""
    return os.environ.get("PB_REFERENCE_DIR",
                          os.path.normpath(os.path.join(ROOT, os.pardir, "reference")))


def build_drivers(names=MD_DRIVERS, ref_dir: str | None = None, force: bool = False) -> list[str]:
    """Compile the reference's MD drivers, unmodified, against the drop-in
    classes in shim/ and this library.  Each driver source is reached through a
    symlink in shim/_drivers, so its quoted includes ("CUDAenv.hh", ...) find
    the shim headers rather than the headers next to the original file.
    Returns the built executables (none when the reference checkout is absent)."""
    ref = ref_dir or reference_dir()
    if not os.path.isdir(ref):
        return []
    build()
    os.makedirs(DRIVERS, exist_ok=True)
    cc = nvcc()
    shim_dig = _digest(sorted(os.path.join(dp, f) for dp, _, fs in os.walk(SHIM)
                              if "_drivers" not in dp for f in fs if f.endswith((".hh", ".h", ".hpp"))), LIB)

    def one(name: str) -> str | None:
        src = os.path.join(ref, name + ".cu")
        if not os.path.exists(src):
            return None
        link = os.path.join(DRIVERS, name + ".cu")
        if os.path.islink(link) or os.path.exists(link):
            os.remove(link)
        os.symlink(src, link)
        exe = os.path.join(DRIVERS, name)
        stamp = exe + ".stamp"
        dig = _digest([src], shim_dig)
        if not force and os.path.exists(exe) and os.path.exists(stamp) and open(stamp).read() == dig:
            os.remove(link)
            return exe
        cmd = [cc, "-ccbin", host_cxx(), *ARCH, "-O2", "-std=c++17", "-DREAL=float",
               "-I", SHIM, "-I", os.path.join(ROOT, "include"), link, "-o", exe,
               "-L", LIBDIR, "-lparticlebase_b200", "-Xlinker", "-rpath", "-Xlinker",
               "$ORIGIN/../../lib"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        os.remove(link)  # the executable is what ships; the link points outside the tree
        if r.returncode != 0:
            raise RuntimeError(f"driver {name} failed to build:\n{r.stdout}\n{r.stderr}")
        with open(stamp, "w") as fh:
            fh.write(dig)
        return exe

    with cf.ThreadPoolExecutor(max_workers=4) as ex:
        out = [x for x in ex.map(one, names) if x]
    return out


def main(argv=None) -> int:
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--drivers", action="store_true",
                    help="also compile the reference MD drivers against the drop-in classes")
    a = ap.parse_args(argv)
    print(build(force=a.force, verbose=a.verbose))
    if a.drivers:
        for exe in build_drivers(force=a.force):
            print(exe)
    return 0


if __name__ == "__main__":
    sys.exit(main())
