"""Build the in-tree native libraries of the path.

* ``libostc.so``  — the product: sm_100a CUDA kernels + C ABI (csrc/) and the
  C++20 host helpers (host/), built with nvcc / g++ directly (no JIT cache,
  so the library travels with the repository snapshot).

Compiled objects go to ``<repo>/_build``; the shared library lands next to
this file. An object is rebuilt when its source or a header it includes is
newer than it (the compilers' dependency files), the library when an object
is newer than it.
"""
from __future__ import annotations

import os
import shutil
import subprocess
from pathlib import Path

PKG = Path(__file__).resolve().parent
REPO = PKG.parent
BUILD = REPO / "_build"
LIB = PKG / "libostc.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ["-O3", "-std=c++20", "-lineinfo", "-Xcompiler", "-fPIC", "--expt-relaxed-constexpr"]


def _nvcc() -> str:
    for cand in (shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and os.path.exists(cand):
            return cand
    raise RuntimeError("nvcc not found: the CUDA toolkit is required to build libostc.so")


def _sources():
    cu = sorted((PKG / "csrc").glob("*.cu"))
    cpp = sorted((PKG / "host").glob("*.cpp"))
    hdr = sorted((PKG / "csrc").glob("*.cuh")) + sorted((REPO / "include").glob("*.h"))
    return cu, cpp, hdr


def _stale(target: Path, deps) -> bool:
    if not target.exists():
        return True
    t = target.stat().st_mtime
    return any(d.stat().st_mtime > t for d in deps)


def _run(cmd):
    r = subprocess.run(cmd, capture_output=True, text=True)
    if r.returncode != 0:
        raise RuntimeError("build failed: %s\n%s\n%s" % (" ".join(map(str, cmd)), r.stdout, r.stderr))
    return r


def _deps(dfile: Path):
    """the files a make-style dependency file (nvcc -MD / g++ -MD) lists"""
    if not dfile.exists():
        return None
    text = dfile.read_text().replace("\\\n", " ")
    out = []
    for line in text.splitlines():
        if ":" not in line:
            continue
        for tok in line.split(":", 1)[1].split():
            out.append(Path(tok))
    return out


def _obj_stale(obj: Path, src: Path, dfile: Path, force: bool) -> bool:
    if force or not obj.exists():
        return True
    deps = _deps(dfile)
    if deps is None:
        return True
    t = obj.stat().st_mtime
    return any((not d.exists()) or d.stat().st_mtime > t for d in [src] + deps)


def build_lib(force: bool = False, verbose: bool = False) -> Path:
    """Compiles the objects whose source or any header they include changed
    (dependency files written by the compilers next to the objects), then
    links libostc.so when an object is newer than it."""
    cu, cpp, hdr = _sources()
    BUILD.mkdir(exist_ok=True)
    nvcc = _nvcc()
    objs = []
    jobs = []
    for src in cu:
        obj = BUILD / (src.stem + ".o")
        dfile = BUILD / (src.stem + ".d")
        objs.append(obj)
        if not _obj_stale(obj, src, dfile, force):
            continue
        cmd = [nvcc, *ARCH, *NVCC_FLAGS, "-MD", "-MF", str(dfile), "-c", str(src), "-o", str(obj)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        jobs.append((cmd, obj))
    for src in cpp:
        obj = BUILD / (src.stem + "_host.o")
        dfile = BUILD / (src.stem + "_host.d")
        objs.append(obj)
        if not _obj_stale(obj, src, dfile, force):
            continue
        cmd = ["g++", "-O3", "-std=c++20", "-fPIC", "-MD", "-MF", str(dfile), "-c", str(src), "-o", str(obj)]
        jobs.append((cmd, obj))
    procs = [(subprocess.Popen(c, stdout=subprocess.PIPE, stderr=subprocess.PIPE, text=True), c, o) for c, o in jobs]
    for p, c, o in procs:
        out, err = p.communicate()
        if p.returncode != 0:
            raise RuntimeError("build failed: %s\n%s\n%s" % (" ".join(map(str, c)), out, err))
        if verbose and err:
            print(err)
    if not force and LIB.exists() and not jobs and not _stale(LIB, objs + [Path(__file__)]):
        return LIB
    tmp = LIB.with_suffix(".so.tmp")
    _run([nvcc, *ARCH, "-shared", "-o", str(tmp), *map(str, objs), "-lcudart"])
    os.replace(tmp, LIB)
    return LIB


if __name__ == "__main__":
    import sys

    print(build_lib(force="--force" in sys.argv, verbose="-v" in sys.argv))
