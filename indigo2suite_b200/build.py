"""Build recipe of the engine's shared library (sm_100a only).

Compiles indigo2suite_b200/csrc/* with nvcc into indigo2suite_b200/libi2b200.so,
in-tree, so the library travels with the source tree. Object files go to
indigo2suite_b200/_build/ and are rebuilt only when a source or header changes.
"""
from __future__ import annotations

import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
INCLUDE = PKG.parent / "include"
BUILD = PKG / "_build"
LIB = PKG / "libi2b200.so"

SOURCES = [
    "engine.cu",
    "resident.cu",
    "selector.cu",
    "batch.cu",
    "gen_device.cu",
    "graph_host.cpp",
]

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = ARCH + [
    "-O3",
    "-std=c++17",
    "-lineinfo",
    "-Xcompiler", "-fPIC,-fopenmp,-O3",
    "-I", str(INCLUDE),
    "--expt-relaxed-constexpr",
]


def nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found")


def _headers() -> list[Path]:
    return list(CSRC.glob("*.cuh")) + list(CSRC.glob("*.h")) + list(INCLUDE.glob("*.h"))


def _stale(obj: Path, src: Path, flags_file: Path) -> bool:
    if not obj.exists():
        return True
    t = obj.stat().st_mtime
    return any(p.stat().st_mtime > t for p in [src, *_headers(), Path(__file__), flags_file])


def build(verbose: bool = False, defines=(), out: Path | None = None, build_dir: Path | None = None) -> Path:
    """Compile the library. `defines` (NAME=VALUE strings) override the
    engine's compile-time tuning constants (for example I2_EB_MIN_BLOCKS);
    such builds should go to their own `out` and `build_dir`."""
    lib = Path(out) if out else LIB
    bdir = Path(build_dir) if build_dir else BUILD
    bdir.mkdir(parents=True, exist_ok=True)
    dflags = [f"-D{d}" for d in defines]
    flags_file = bdir / "defines.txt"
    if not flags_file.exists() or flags_file.read_text() != " ".join(dflags):
        flags_file.write_text(" ".join(dflags))
    objs = []
    procs = []
    for name in SOURCES:
        src = CSRC / name
        obj = bdir / (name + ".o")
        objs.append(obj)
        if _stale(obj, src, flags_file):
            cmd = [nvcc(), *NVCC_FLAGS, *dflags, "-c", str(src), "-o", str(obj)]
            if verbose:
                print(" ".join(cmd), flush=True)
            procs.append((name, subprocess.Popen(cmd, stdout=subprocess.PIPE, stderr=subprocess.STDOUT)))
    failed = []
    for name, p in procs:
        out, _ = p.communicate()
        if p.returncode != 0:
            failed.append((name, out.decode(errors="replace")))
        elif verbose and out:
            print(out.decode(errors="replace"))
    if failed:
        msg = "\n".join(f"--- {n}\n{o}" for n, o in failed)
        raise RuntimeError("nvcc failed:\n" + msg)
    if procs or not lib.exists() or any(o.stat().st_mtime > lib.stat().st_mtime for o in objs):
        cmd = [nvcc(), *ARCH, "-shared", "-Xcompiler", "-fPIC,-fopenmp", "-o", str(lib),
               *[str(o) for o in objs], "-lgomp"]
        if verbose:
            print(" ".join(cmd), flush=True)
        subprocess.run(cmd, check=True)
    return lib


if __name__ == "__main__":
    import argparse

    ap = argparse.ArgumentParser()
    ap.add_argument("-v", action="store_true")
    ap.add_argument("-D", action="append", default=[], metavar="NAME=VALUE")
    ap.add_argument("--out", default=None)
    ap.add_argument("--build-dir", default=None)
    a = ap.parse_args()
    print(build(verbose=a.v, defines=a.D, out=a.out, build_dir=a.build_dir))
