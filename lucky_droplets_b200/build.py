"""Build the CUDA library liblucky_droplets.so in-tree for sm_100a.

    python -m lucky_droplets_b200.build [--force] [--jobs N] [--verbose]

Every .cu under csrc/ is compiled separately (in parallel) with
``nvcc -gencode arch=compute_100a,code=sm_100a -O3 -lineinfo`` and linked into
``lucky_droplets_b200/liblucky_droplets.so``; objects go to ``_build/`` at the repository root.
A unit is recompiled when it or any header under csrc/ or include/ is newer than its object.
"""
import argparse
import concurrent.futures as cf
import os
import pathlib
import shutil
import subprocess
import sys

PKG = pathlib.Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = ROOT / "_build"
LIB = PKG / "liblucky_droplets.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + ["-O3", "-std=c++17", "--expt-relaxed-constexpr", "-lineinfo",
                     "-Xcompiler", "-fPIC", "-Xcompiler", "-fvisibility=hidden",
                     "-I", str(INCLUDE), "-I", str(CSRC)]


def nvcc():
    exe = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not os.path.exists(exe):
        raise RuntimeError("nvcc not found")
    return exe


def _headers():
    return list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))


def _stale(obj, src, newest_header):
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return src.stat().st_mtime > t or newest_header > t


def _compile(src, obj, extra, verbose):
    cmd = [nvcc()] + NVCC_FLAGS + extra + ["-c", str(src), "-o", str(obj)]
    if verbose:
        print(" ".join(cmd), flush=True)
    r = subprocess.run(cmd, capture_output=True, text=True)
    out = "\n".join(l for l in (r.stdout + r.stderr).splitlines()
                    if "Warning: The 'compute_" not in l)
    if r.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name}:\n{out}")
    return out


def build(force=False, jobs=None, verbose=False, ptxas_verbose=False):
    """Compile and link the library; returns its path."""
    BUILD.mkdir(exist_ok=True)
    sources = sorted(CSRC.glob("*.cu"))
    newest_header = max((h.stat().st_mtime for h in _headers()), default=0.0)
    objs, todo = [], []
    for src in sources:
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if force or _stale(obj, src, newest_header):
            todo.append((src, obj))
    extra = ["-Xptxas", "-v"] if ptxas_verbose else []
    if todo:
        jobs = jobs or os.cpu_count() or 4
        with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
            futs = {ex.submit(_compile, s, o, extra, verbose): s for s, o in todo}
            for f in cf.as_completed(futs):
                out = f.result()
                if ptxas_verbose and out:
                    print(f"== {futs[f].name}\n{out}")
    if todo or not LIB.exists():
        tmp = LIB.with_suffix(".so.tmp")
        cmd = [nvcc()] + ARCH + ["-shared", "-o", str(tmp)] + [str(o) for o in objs] + ["-lcudart"]
        r = subprocess.run(cmd, capture_output=True, text=True)
        if r.returncode != 0:
            raise RuntimeError(f"link failed:\n{r.stdout}{r.stderr}")
        os.replace(tmp, LIB)
    return LIB


def main(argv=None):
    ap = argparse.ArgumentParser()
    ap.add_argument("--force", action="store_true")
    ap.add_argument("--jobs", type=int, default=None)
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--ptxas-verbose", action="store_true")
    a = ap.parse_args(argv)
    path = build(force=a.force, jobs=a.jobs, verbose=a.verbose, ptxas_verbose=a.ptxas_verbose)
    print(path)


if __name__ == "__main__":
    sys.exit(main())
