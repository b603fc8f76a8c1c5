"""Build libmbforce.so (the C-ABI CUDA library) in-tree with nvcc for sm_100a.

    python -m akitsushima_b200.build          # build if sources changed
    python -m akitsushima_b200.build --force  # rebuild
"""
import argparse
import glob
import os
import shutil
import subprocess
import sys

PKG = os.path.dirname(os.path.abspath(__file__))
ROOT = os.path.dirname(PKG)
CSRC = os.path.join(PKG, "csrc")
LIB = os.path.join(PKG, "libmbforce.so")
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path():
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found")


def sources():
    return sorted(glob.glob(os.path.join(CSRC, "*.cu")))


def _deps():
    return (sources() + glob.glob(os.path.join(CSRC, "*.cuh"))
            + [os.path.join(ROOT, "include", "mbforce.h")])


def up_to_date():
    if not os.path.exists(LIB):
        return False
    t = os.path.getmtime(LIB)
    return all(os.path.getmtime(p) <= t for p in _deps())


def build(force=False, verbose=False, extra=(), out=None):
    """Compile every .cu of csrc/ into one shared library (parallel objects).
    ``extra`` adds nvcc flags (e.g. -DMBF_CHECKS for the bounds-checked
    debugging build); ``out`` writes the library elsewhere."""
    lib_path = out or LIB
    if not force and out is None and up_to_date():
        return LIB
    nvcc = nvcc_path()
    objdir = os.path.join(PKG, "_build" if out is None else "_build_alt")
    os.makedirs(objdir, exist_ok=True)
    flags = ARCH + ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC",
                    "--expt-relaxed-constexpr", "-I" + os.path.join(ROOT, "include")]
    flags += list(extra)
    if verbose:
        flags += ["-Xptxas", "-v"]
    procs, objs = [], []
    for src in sources():
        obj = os.path.join(objdir, os.path.basename(src)[:-3] + ".o")
        objs.append(obj)
        procs.append((src, subprocess.Popen([nvcc, *flags, "-c", src, "-o", obj],
                                            stdout=subprocess.PIPE,
                                            stderr=subprocess.STDOUT, text=True)))
    failed = []
    for src, p in procs:
        out, _ = p.communicate()
        if verbose or p.returncode:
            sys.stderr.write(out)
        if p.returncode:
            failed.append(src)
    if failed:
        raise RuntimeError("nvcc failed on " + ", ".join(os.path.basename(f) for f in failed))
    tmp = lib_path + ".tmp"
    subprocess.run([nvcc, *ARCH, "-shared", "-o", tmp, *objs, "-lcudart"], check=True)
    os.replace(tmp, lib_path)
    return lib_path


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-v", "--verbose", action="store_true")
    ap.add_argument("--checks", action="store_true", help="bounds-checked debugging build")
    ap.add_argument("--out", default=None, help="library path (default: in the package)")
    a = ap.parse_args()
    print(build(force=a.force, verbose=a.verbose, extra=["-DMBF_CHECKS"] if a.checks else (),
                out=a.out))
