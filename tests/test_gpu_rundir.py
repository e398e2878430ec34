"""A reference run directory, unchanged, runs on the GPU and writes the reference's restart files.

The directory is written by oracle.refrun (exactly what the reference reads), the
reference runs in it and saves flowData/NUC3d_step_<s>_ID_<r>.bin and, with
SimutaneousData 1 and postStep 1, appends its enstrophy / kinetic-energy line to
enstrophy.dat every step; nuc3d_b200.run runs the same directory and both its restart
files and its enstrophy.dat must be byte-identical (reference-order build)."""
import math
import os
import shutil
import subprocess
import tempfile
from pathlib import Path

import numpy as np
import pytest

from oracle import refrun as R


def _case(multi: bool):
    x, y, z = R.box_nodes(16, 12, 8, hi=(2.0 * math.pi,) * 3)
    params = {"Reynolds": 1600.0, "Mach": 0.1, "Pt": 0.72, "Gamma": 1.4, "T_ref": 110.4,
              "T_inf": 288.0, "T_wall": 1.0}
    if not multi:
        return R.Case(model="NavierStokes3d", riemann="LF", schemes=("weno5js",) * 3,
                      params=params, benchmark=2, nodes=[(x, y, z)], bc_topo=[R.PERIODIC_SELF])
    sl = [(slice(None), slice(None), slice(0, 9)), (slice(None), slice(None), slice(8, 17))]
    nodes = [(x[s], y[s], z[s]) for s in sl]
    topo = [["1 1", "1 0", "0 3", "0 2", "0 5", "0 4"], ["0 1", "0 0", "1 3", "1 2", "1 5", "1 4"]]
    return R.Case(model="NavierStokes3d", riemann="LF", schemes=("weno5js",) * 3, params=params,
                  benchmark=2, nodes=nodes, bc_topo=topo)


@pytest.mark.gpu
@pytest.mark.parametrize("multi", [False, True])
def test_run_directory_restart_files_identical(multi):
    from nuc3d_b200 import rundir as RD
    case = _case(multi)
    case.post_q = True
    tmp = Path(tempfile.mkdtemp(prefix="nuc3d_rundir_"))
    try:
        R.write_case(case, tmp)
        io = (tmp / "inp/IOController.in").read_text()
        io = io.replace("endStep 1000000000", "endStep 4").replace("saveStep 1000000000", "saveStep 2")
        io = io.replace("Binary no", "Binary yes").replace("postStep 0", "postStep 1")
        (tmp / "inp/IOController.in").write_text(io)
        ref = tmp / "ref"
        shutil.copytree(tmp, ref, ignore=shutil.ignore_patterns("ref"))
        env = dict(os.environ, NUC_SHIM_NP=str(case.nranks))
        p = subprocess.run([str(R.ref_binary("nuc3d_ref"))], cwd=ref, env=env,
                           capture_output=True, text=True, timeout=600)
        assert p.returncode == 0, p.stdout[-2000:] + p.stderr[-2000:]
        RD.run(tmp, quiet=True)
        for step in (2, 4):
            for r in range(case.nranks):
                a = (ref / f"flowData/NUC3d_step_{step}_ID_{r}.bin").read_bytes()
                b = (tmp / f"flowData/NUC3d_step_{step}_ID_{r}.bin").read_bytes()
                assert a == b, (step, r)
        a = (ref / "enstrophy.dat").read_text()
        b = (tmp / "enstrophy.dat").read_text()
        assert len(a.splitlines()) == 4 and a == b, (a, b)
        # restart from the step-2 files (block::initial reads them, src/block.cpp:785-855;
        # metrics then come from the GPU) and run to step 4: same bytes as the continuous run
        io = (tmp / "inp/IOController.in").read_text().replace("startStep 0", "startStep 2")
        (tmp / "inp/IOController.in").write_text(io)
        for r in range(case.nranks):
            (tmp / f"flowData/NUC3d_step_4_ID_{r}.bin").unlink()
        RD.run(tmp, quiet=True)
        for r in range(case.nranks):
            a = (ref / f"flowData/NUC3d_step_4_ID_{r}.bin").read_bytes()
            b = (tmp / f"flowData/NUC3d_step_4_ID_{r}.bin").read_bytes()
            assert a == b, ("restart", r)
    finally:
        shutil.rmtree(tmp, ignore_errors=True)
