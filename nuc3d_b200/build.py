"""Build libnuc3d_b200.so in-tree with nvcc for sm_100a.

    python -m nuc3d_b200.build [--verbose]

kernels_exact.cu is compiled with -fmad=false (reference operation order);
kernels_fast.cu with FMA contraction; nuc3d_abi.cu is the C ABI.
"""
from __future__ import annotations

import argparse
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
ROOT = PKG.parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
LIB = PKG / "libnuc3d_b200.so"
PROBE_LIB = PKG / "libnuc3d_probe.so"

ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]
COMMON = ["-O3", "-lineinfo", "-std=c++17", "-Xcompiler", "-fPIC", "-I", str(ROOT / "include"),
          "-I", str(CSRC)]
UNITS = {
    "kernels_exact.cu": ["-fmad=false"],
    "kernels_fast.cu": ["-fmad=true"],
    "nuc3d_abi.cu": [],
    "nuc3d_noalloc.cu": [],
    "sensor_train.cu": [],
}


def nvcc() -> str:
    for c in (os.environ.get("NVCC"), shutil.which("nvcc"), "/usr/local/cuda/bin/nvcc"):
        if c and Path(c).exists():
            return c
    raise RuntimeError("nvcc not found")


def _stale(out: Path, deps) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(Path(d).stat().st_mtime > t for d in deps)


def build(verbose: bool = False, force: bool = False, defines=(), out: Path | None = None,
          build_dir: Path | None = None) -> Path:
    """Compile the library; `defines` (e.g. ["NUC3D_SWEEP_MINB=3"]) select tile options,
    `out`/`build_dir` put a variant build elsewhere."""
    global BUILD, LIB
    if out is not None:
        LIB = Path(out)
    if build_dir is not None:
        BUILD = Path(build_dir)
    BUILD.mkdir(parents=True, exist_ok=True)
    headers = sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + [ROOT / "include" / "nuc3d_gpu.h"]
    cc = nvcc()
    procs, objs = [], []
    for unit, extra in UNITS.items():
        src = CSRC / unit
        obj = BUILD / (src.stem + ".o")
        objs.append(obj)
        if force or _stale(obj, [src, *headers, Path(__file__)]):
            cmd = [cc, *ARCH, *COMMON, *extra, *[f"-D{d}" for d in defines], "-c", str(src),
                   "-o", str(obj)]
            if verbose:
                cmd.insert(1, "-Xptxas=-v")
                print(" ".join(cmd), flush=True)
            procs.append((unit, subprocess.Popen(cmd, stdout=subprocess.PIPE,
                                                 stderr=subprocess.STDOUT, text=True)))
    failed = []
    for unit, p in procs:
        log, _ = p.communicate()
        if log and (verbose or p.returncode):
            print(log, end="", flush=True)
        if p.returncode:
            failed.append(unit)
    if failed:
        raise RuntimeError(f"nvcc failed for {failed}")
    if force or procs or not LIB.exists():
        cmd = [cc, *ARCH, "-shared", "-o", str(LIB), *map(str, objs), "-lcudart_static", "-lrt",
               "-ldl", "-lpthread"]
        subprocess.run(cmd, check=True)
    probe_src = CSRC / "probe.cu"
    if out is None and (force or _stale(PROBE_LIB, [probe_src, Path(__file__)])):
        subprocess.run([cc, *ARCH, "-O3", "-std=c++17", "-Xcompiler", "-fPIC", "-shared",
                        str(probe_src), "-o", str(PROBE_LIB), "-lcudart_static", "-lrt", "-ldl",
                        "-lpthread"], check=True)
    return LIB


if __name__ == "__main__":
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(a.verbose, a.force))
    sys.exit(0)
