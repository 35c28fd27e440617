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
import tempfile
from concurrent.futures import ThreadPoolExecutor
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


def _run(cmd: list[str]) -> subprocess.CompletedProcess:
    return subprocess.run(cmd, cwd=str(PKG), capture_output=True, text=True, env=dict(os.environ))


def build(verbose: bool = False, force: bool = False) -> Path:
    """Compile every ``csrc/*.cu`` to an object in parallel (no device code crosses files, so no
    relocatable device code is needed), then link the shared library."""
    if not force and not needs_rebuild():
        return LIB
    flags = [
        *ARCH, "-O3", "-lineinfo", "-std=c++17", "--expt-relaxed-constexpr",
        "-Xcompiler", "-fPIC", "-Xcompiler", "-ffp-contract=off",
        "-I", str(PKG.parent / "include"),
    ]
    if verbose:
        flags.insert(0, "-Xptxas=-v")
    objdir = Path(tempfile.mkdtemp(prefix="pscb200_build_"))
    try:
        srcs = sources()
        objs = [objdir / (s.stem + ".o") for s in srcs]
        jobs = [[nvcc_path(), *flags, "-c", str(s), "-o", str(o)] for s, o in zip(srcs, objs)]
        with ThreadPoolExecutor(max_workers=max(1, min(len(jobs), os.cpu_count() or 1))) as pool:
            results = list(pool.map(_run, jobs))
        failed = [(s, r) for s, r in zip(srcs, results) if r.returncode != 0]
        for s, r in zip(srcs, results):
            if verbose or r.returncode != 0:
                sys.stderr.write(f"== {s.name}\n{r.stdout}{r.stderr}")
        if failed:
            raise RuntimeError("nvcc failed on " + ", ".join(s.name for s, _ in failed))
        link = _run([nvcc_path(), *ARCH, "-shared", "-Xcompiler", "-fPIC", "-o", str(LIB) + ".tmp",
                     *map(str, objs)])
        if link.returncode != 0:
            sys.stderr.write(link.stdout + link.stderr)
            raise RuntimeError("nvcc failed linking libpscb200.so")
        os.replace(str(LIB) + ".tmp", LIB)
    finally:
        shutil.rmtree(objdir, ignore_errors=True)
    return LIB


def main() -> None:
    ap = argparse.ArgumentParser(description=__doc__)
    ap.add_argument("--verbose", action="store_true", help="print ptxas register / spill report")
    ap.add_argument("--force", action="store_true")
    args = ap.parse_args()
    print(build(verbose=args.verbose, force=args.force))


if __name__ == "__main__":
    main()
