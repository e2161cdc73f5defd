"""Build the native pieces in-tree.

``build_library()`` compiles the CUDA sources under ``csrc/`` for sm_100a into
``legendre_b200/liblegendre_b200.so`` (plain ``nvcc``; no PyTorch extension
machinery, the library exports a C ABI only).  ``build_oracle()`` compiles
the CPU restatement used by the tests into ``oracle/liblegendre_oracle.so``.

Run ``python legendre_b200/build.py`` to build both (by path: importing the
package first would load a possibly stale library).
"""
from __future__ import annotations

import concurrent.futures
import hashlib
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
LIB = PKG / "liblegendre_b200.so"
ORACLE_DIR = ROOT / "oracle"
ORACLE_LIB = ORACLE_DIR / "liblegendre_oracle.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]

# Translation units and their floating-point contraction policy.  The FP64
# reference-order kernels must not contract a*b+c (the reference is Rust,
# which never does); units holding only freely restructured FP32 kernels may.
SOURCES = [
    ("lg_kernels.cu", ["-fmad=false"]),
    ("lg_modelc.cu", ["-fmad=false"]),
    ("lg_modelc_f32.cu", []),
    ("lg_abi.cu", ["-fmad=false"]),
    ("lg_amr_host.cu", ["-fmad=false"]),
    ("lg_amr.cu", ["-fmad=false"]),
    ("lg_adjoint.cu", []),      # not bit-matched to anything: contraction allowed
    ("lg_ensemble.cu", ["-fmad=false"]),
    ("lg_observe.cu", ["-fmad=false"]),
    ("lg_peaks.cu", []),        # microbenchmarks of explicit fma / integer chains
]


def _nvcc() -> str:
    for cand in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if cand and Path(cand).exists():
            return cand
    raise RuntimeError("nvcc not found; the CUDA toolkit is required to build legendre_b200")


def _digest(deps, extra: str) -> str:
    # source names relative to the repository root, so that a copy of the
    # tree at another path (with its built libraries) is not stale
    h = hashlib.sha256(extra.encode())
    for d in sorted(Path(p).resolve().relative_to(ROOT).as_posix() for p in deps):
        h.update(d.encode())
        h.update((ROOT / d).read_bytes())
    return h.hexdigest()


def _stale(target: Path, deps, extra: str = "") -> bool:
    # content hash of the sources beside the target: robust to copies that
    # do not preserve modification times
    stamp = target.with_name(target.name + ".srchash")
    if not target.exists() or not stamp.exists():
        return True
    return stamp.read_text().strip() != _digest(deps, extra)


def _stamp(target: Path, deps, extra: str = "") -> None:
    target.with_name(target.name + ".srchash").write_text(_digest(deps, extra) + "\n")


def build_library(force: bool = False, verbose: bool = False) -> Path:
    deps = [CSRC / s for s, _ in SOURCES] + list(CSRC.glob("*.h")) + list(CSRC.glob("*.cuh"))
    deps.append(ROOT / "include" / "legendre_b200.h")
    extra = repr(SOURCES) + repr(ARCH)
    if not force and not _stale(LIB, deps, extra):
        return LIB
    nvcc = _nvcc()
    objdir = PKG / "_build"
    objdir.mkdir(exist_ok=True)
    cmds, objs = [], []
    for src, flags in SOURCES:
        obj = objdir / (Path(src).stem + ".o")
        cmd = [nvcc, "-O3", "-std=c++17", *ARCH, "-lineinfo", "-Xcompiler", "-fPIC", *flags,
               "-I", str(ROOT / "include"), "-c", str(CSRC / src), "-o", str(obj)]
        if verbose:
            cmd.insert(1, "-Xptxas=-v")
        cmds.append(cmd)
        objs.append(str(obj))
    with concurrent.futures.ThreadPoolExecutor(max_workers=len(cmds)) as pool:
        list(pool.map(_run, cmds))
    _run([nvcc, "-shared", *ARCH, *objs, "-o", str(LIB)])
    _stamp(LIB, deps, extra)
    return LIB


def build_oracle(force: bool = False) -> Path:
    srcs = [ORACLE_DIR / "legendre_oracle.cpp", ORACLE_DIR / "legendre_oracle_amr.cpp"]
    deps = srcs + [ORACLE_DIR / "legendre_oracle.h", ORACLE_DIR / "oracle_core.hpp"]
    # -ffp-contract=off: no a*b+c is fused except the reference's mul_add
    # sites (std::fma).  Without -ffast-math GCC reassociates no
    # floating-point operation at any level, so -O3 gives the bits of -O2
    # (the golden fixtures check it).  No -march=native: the library travels
    # to hosts with other CPUs.
    flags = ["-O3", "-std=c++17", "-ffp-contract=off", "-fopenmp", "-fPIC", "-shared"]
    if not force and not _stale(ORACLE_LIB, deps, repr(flags)):
        return ORACLE_LIB
    cxx = shutil.which("g++") or "g++"
    _run([cxx, *flags, *map(str, srcs), "-o", str(ORACLE_LIB)])
    _stamp(ORACLE_LIB, deps, repr(flags))
    return ORACLE_LIB


def _run(cmd):
    proc = subprocess.run(cmd, capture_output=True, text=True)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError("build step failed: " + " ".join(cmd))
    if proc.stderr.strip():
        sys.stderr.write(proc.stderr)


if __name__ == "__main__":
    force = "--force" in sys.argv
    print(build_library(force=force, verbose="-v" in sys.argv))
    print(build_oracle(force=force))
