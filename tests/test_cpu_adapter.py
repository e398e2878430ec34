"""The C++ adapter the integration guide shows a NUC3d maintainer (GpuBlockData, GpuRK3) compiles
against the reference's own headers and links against the reference's objects and
libnuc3d_b200.so: the drop-in classes override the reference's virtual interfaces
(EulerData3D::solve, integration::integrationAll) with the signatures they have there.
Compile and link only; nothing runs.  Needs the reference sources and oracle/_ref/obj
(built by `make -C oracle ref`)."""
import os
import re
import shutil
import subprocess
import tempfile
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
REF = Path(os.environ.get("NUC3D_REF_SRC", "/root/reference/src"))
OBJ = ROOT / "oracle" / "_ref" / "obj"
LIB = ROOT / "nuc3d_b200" / "libnuc3d_b200.so"

MAIN = r"""
int main(int argc, char **) {
  if (argc > 1000) {  // never runs: makes the linker resolve every virtual of both classes
    nuc3d_config cfg{};
    const int t[6] = {-1, -1, -1, -1, -1, -1}, id[6] = {1, 1, 1, 1, 1, 1};
    nuc3d_gpu_adapter::GpuBlock g(cfg, 8, 8, 8, t, id, nullptr);
    nuc3d_gpu_adapter::GpuBlockData d(8, 8, 8, 5, g);
    d.upload_metrics();
    nuc3d_gpu_adapter::GpuRK3 r(g);
    nuc3d::integration *ip = &r;
    nuc3d::EulerData3D *ep = &d;
    return ip != nullptr && ep != nullptr;
  }
  return 0;
}
"""


def _adapter_source() -> str:
    text = (ROOT / "INTEGRATION.md").read_text()
    blocks = re.findall(r"```cpp\n(.*?)```", text, re.S)
    src = [b for b in blocks if "class GpuRK3" in b]
    assert src, "the integration guide has no GpuRK3 adapter block"
    return src[0]


def test_adapter_compiles_and_links_against_the_reference():
    if not (REF / "euler3d.h").exists():
        pytest.skip("reference sources not present")
    objs = sorted(p for p in OBJ.glob("*.o") if p.name not in ("NUC3d.o", "ref_taps.o"))
    if not objs or not LIB.exists():
        pytest.skip("reference objects or the library not built")
    cxx = shutil.which("g++") or "/opt/gcc/bin/g++"
    with tempfile.TemporaryDirectory() as d:
        src = Path(d) / "adapter.cpp"
        src.write_text(_adapter_source() + MAIN)
        exe = Path(d) / "adapter"
        cmd = [cxx, "-std=c++11", "-O0", "-w", "-I", str(ROOT / "oracle" / "mpi_shim"),
               "-I", str(REF), "-I", str(ROOT / "include"), str(src), *map(str, objs),
               str(LIB), f"-Wl,-rpath,{LIB.parent}", "-ldl", "-lpthread", "-lm", "-o", str(exe)]
        r = subprocess.run(cmd, capture_output=True, text=True)
        assert r.returncode == 0, r.stderr[-4000:]
        assert exe.exists()
