"""Build libpscb200.so in-tree with nvcc for sm_100a.

    python -m particuology_hydraulic_penalty_b200.build [--verbose]

The shared library holds every CUDA kernel of the package and its C ABI
(``include/psc_b200.h``).  It is written next to this file so that it travels
with the source tree; ``ctypes`` loads it from there.
"""

from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
LIB = PKG / "libpscb200.so"
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc_path() -> str:
    cand = shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    if not Path(cand).exists():
        raise RuntimeError("nvcc not found (CUDA toolkit required to build libpscb200.so)")
    return cand


def sources() -> list[Path]:
    return sorted(CSRC.glob("*.cu"))


def needs_rebuild() -> bool:
    if not LIB.exists():
        return True
    t = LIB.stat().st_mtime
    deps = list(CSRC.glob("*.cu")) + list(CSRC.glob("*.cuh")) + [PKG.parent / "include" / "psc_b200.h"]
    return any(p.stat().st_mtime > t for p in deps if p.exists())


def build(verbose: bool = False, force: bool = False) -> Path:
    if not force and not needs_rebuild():
        return LIB
    cmd = [
        nvcc_path(), *ARCH, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
        "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off", "-shared",
        "-I", str(PKG.parent / "include"),
        "-o", str(LIB) + ".tmp", *map(str, sources()),
    ]
    if verbose:
        cmd.insert(1, "-Xptxas=-v")
    env = dict(os.environ)
    proc = subprocess.run(cmd, cwd=str(PKG), capture_output=True, text=True, env=env)
    if proc.returncode != 0:
        sys.stderr.write(proc.stdout + proc.stderr)
        raise RuntimeError("nvcc failed building libpscb200.so")
    if verbose:
        sys.stderr.write(proc.stdout + proc.stderr)
    os.replace(str(LIB) + ".tmp", LIB)
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--verbose", action="store_true", help="print ptxas register / spill report")
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args()
    print(build(verbose=args.verbose, force=args.force))


if __name__ == "__main__":
    main()
