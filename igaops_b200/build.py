"""Builds ``libigab200.so`` (all CUDA kernels + the C ABI) for sm_100a, in-tree.

Usage: ``python -m igaops_b200.build [--force] [-j N] [--verbose]``.

Each ``.cu`` file under ``igaops_b200/csrc`` compiles to one object; the
fused matrix-free instantiation unit ``mf_inst.cu`` compiles once per
(dimension, element type, band width).  Objects compile in parallel, then
link into ``igaops_b200/_lib/libigab200.so``.  Nothing is JIT-compiled at
import time and there is no fallback build.
"""
from __future__ import annotations

import argparse
import concurrent.futures as cf
import hashlib
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
INCLUDE = ROOT / "include"
BUILD = ROOT / "_build" / "obj"
LIBDIR = PKG / "_lib"
LIBNAME = "libigab200.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
NVCC_FLAGS = [
    "-std=c++17",
    "-O3",
    "-lineinfo",
    "-Xcompiler",
    "-fPIC",
    "--expt-relaxed-constexpr",
    f"-I{INCLUDE}",
    f"-I{CSRC}",
]

# (D, dtype tag, C++ type, band width) instances of the fused kernels
MF_INSTANCES = [
    (d, tn, t, w)
    for d in (2, 3)
    for tn, t in (("f64", "double"), ("f32", "float"))
    for w in (3, 4, 5, 6)
]


def nvcc() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found; the CUDA toolkit is required to build libigab200")
    return cand


def _units():
    units = []
    headers = sorted(CSRC.glob("*.cuh")) + [INCLUDE / "igab200.h"]
    for src in sorted(CSRC.glob("*.cu")):
        if src.name == "mf_inst.cu":
            for d, tn, t, w in MF_INSTANCES:
                defs = [
                    f"-DIGA_INST_D={d}",
                    f"-DIGA_INST_TN={tn}",
                    f"-DIGA_INST_T={t}",
                    f"-DIGA_INST_W={w}",
                ]
                units.append((src, BUILD / f"mf_inst_{d}d_{tn}_w{w}.o", defs))
        else:
            units.append((src, BUILD / (src.stem + ".o"), []))
    return units, headers


def _digest(src: Path, headers, defs) -> str:
    h = hashlib.sha256()
    h.update(" ".join(NVCC_FLAGS + ARCH + defs).encode())
    h.update(src.read_bytes())
    for hd in headers:
        h.update(hd.read_bytes())
    return h.hexdigest()


def _compile(src: Path, obj: Path, defs, headers, force: bool, verbose: bool):
    stamp = obj.with_suffix(".sha")
    dig = _digest(src, headers, defs)
    if not force and obj.exists() and stamp.exists() and stamp.read_text() == dig:
        return obj, False, ""
    cmd = [nvcc()] + NVCC_FLAGS + ARCH + defs + ["-c", str(src), "-o", str(obj)]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    res = subprocess.run(cmd, capture_output=True, text=True)
    if res.returncode != 0:
        raise RuntimeError(f"nvcc failed for {src.name} {defs}:\n{res.stderr}")
    stamp.write_text(dig)
    return obj, True, res.stderr


def build(force: bool = False, jobs: int | None = None, verbose: bool = False) -> Path:
    BUILD.mkdir(parents=True, exist_ok=True)
    LIBDIR.mkdir(parents=True, exist_ok=True)
    units, headers = _units()
    jobs = jobs or max(1, os.cpu_count() or 1)
    objs, changed = [], False
    with cf.ThreadPoolExecutor(max_workers=jobs) as ex:
        futs = [ex.submit(_compile, s, o, d, headers, force, verbose) for s, o, d in units]
        for f in futs:
            obj, did, log = f.result()
            objs.append(obj)
            changed |= did
            if verbose and log:
                sys.stderr.write(log)
    lib = LIBDIR / LIBNAME
    if changed or not lib.exists() or force:
        tmp = lib.with_suffix(".so.tmp")
        cmd = [nvcc(), "-shared"] + ARCH + ["-o", str(tmp)] + [str(o) for o in objs]
        res = subprocess.run(cmd, capture_output=True, text=True)
        if res.returncode != 0:
            raise RuntimeError(f"link failed:\n{res.stderr}")
        os.replace(tmp, lib)
    return lib


def main(argv=None):
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--force", action="store_true")
    ap.add_argument("-j", "--jobs", type=int, default=None)
    ap.add_argument("--verbose", action="store_true")
    args = ap.parse_args(argv)
    lib = build(force=args.force, jobs=args.jobs, verbose=args.verbose)
    print(lib)


if __name__ == "__main__":
    main()
