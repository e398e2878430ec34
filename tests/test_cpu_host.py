"""CPU tests: host-side metrics, the C ABI symbol table, golden fixture sanity."""
import ctypes
import re
from pathlib import Path

import numpy as np
import pytest

from tests import golden_cases as G

ROOT = Path(__file__).resolve().parents[1]


def test_metrics_bitwise_reference():
    """nuc3d_b200.metrics reproduces block::getJacobians bit for bit."""
    from nuc3d_b200.metrics import metrics_from_nodes
    g = G.load("tgv_ns_weno5js_lf")
    m = metrics_from_nodes(*G.nodes(g))
    assert np.array_equal(m["jac"], g.metrics_jac)
    for nm in ("xi_xyz", "eta_xyz", "zeta_xyz", "dxyz"):
        assert np.array_equal(m[nm], g.data[f"metrics_{nm}"]), nm


def test_metrics_reject_untiled_mesh():
    from nuc3d_b200.metrics import metrics_from_nodes
    from oracle.refrun import box_nodes
    with pytest.raises(ValueError):
        metrics_from_nodes(*box_nodes(10, 8, 8))


def test_library_exports_header_symbols():
    lib_path = ROOT / "nuc3d_b200" / "libnuc3d_b200.so"
    if not lib_path.exists():
        pytest.skip("library not built")
    lib = ctypes.CDLL(str(lib_path))
    header = (ROOT / "include" / "nuc3d_gpu.h").read_text()
    names = set(re.findall(r"\b(nuc3d_[a-z_]+)\s*\(", header))
    assert len(names) >= 20
    missing = [n for n in sorted(names) if not hasattr(lib, n)]
    assert not missing, missing


def test_golden_fixtures_consistent():
    for name in G.names():
        g = G.load(name)
        n = int(g.cfg["nsteps"])
        assert g.dt.shape == (n,) and g.time.shape == (n,)
        assert np.isclose(g.time[-1], g.dt.sum(), rtol=1e-14)
        nx, ny, nz = g.cfg["shape"]
        assert g.q0.shape == (5, nz, ny, nx) == g.qn.shape == g.rhs.shape
        assert np.all(np.isfinite(g.qn))
        if "libm_max_rel_diff" in g.data:
            # hccs weights (eps 1e-40) amplify glibc pow rounding the most: 7e-12
            assert g.libm_max_rel_diff[0] < 1e-10


@pytest.mark.parametrize("ivs,vis,code", [
    (("weno3js",) * 3, ("cd6",) * 3, 5),              # cd6 reaches 3 > bufferSize 2
    (("upwind1st", "weno5js", "weno5js"), ("cd2",) * 3, None),  # cd2 reaches 1: allowed
    (("weno5js",) * 3, ("cd8", "cd6", "cd6"), 5),     # cd8 reaches 4 > bufferSize 3
    (("hccs77",) * 3, ("cd8",) * 3, None),            # cd8 reaches 4 = hccs77's bufferSize
    (("weno5js",) * 3, ("cd4",) * 3, 1),              # unknown name
])
def test_create_rejects_undefined_viscous_pairs(ivs, vis, code):
    """Navier-Stokes contexts whose viscous stencil reaches past the reconstruction's
    bufferSize are refused (the reference reads outside its arrays there); the check runs
    before any CUDA call, so it holds on a machine without a GPU."""
    import nuc3d_b200 as nb
    lib = nb.load_library()
    cfg = nb.Config(scheme_ivs=ivs, scheme_vis=vis, model="NavierStokes3d")._c()
    ctx = ctypes.c_void_p()
    rc = lib.nuc3d_create(ctypes.byref(cfg), 0, ctypes.byref(ctx))
    if code is None:
        assert rc != 5 and rc != 1, lib.nuc3d_last_error()
        if rc == 0:
            lib.nuc3d_destroy(ctx)
    else:
        assert rc == code, (rc, lib.nuc3d_last_error())
