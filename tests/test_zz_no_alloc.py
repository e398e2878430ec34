"""nuc3d_rhs_noalloc: the right-hand side for callers that cannot allocate device memory.

Some callers cannot call cudaMalloc where they evaluate the right-hand side: host
frameworks that own every device buffer, time-critical loops where an allocation could
stall.  For them the
library has one entry point that allocates nothing: the caller passes its own device
buffers for the state, the metrics and the output, and the library's working memory is a
fixed 8 MiB static device array.  These tests call it through the C ABI and check that it
returns exactly what the allocating entry point (nuc3d_rhs on a context) returns, twice in
a row, and that it refuses what it cannot do.  This file is collected last on purpose.
"""
import ctypes

import numpy as np
import pytest

from tests import golden_cases as G

CASES = ["sphere_euler_weno5z_ausm_outlet", "wavy_euler_weno5js_lf", "mixed_euler_lf_outlet_symm"]


def _int6(x):
    return (ctypes.c_int * 6)(*[int(v) for v in x])


def _call(lib, cfg_c, shape, bc, dev, rhs, dt, stream):
    t, i, v = bc
    vals = np.ascontiguousarray(v, dtype=np.float64).reshape(30)
    nx, ny, nz = shape
    return lib.nuc3d_rhs_noalloc(
        ctypes.byref(cfg_c), 0, nx, ny, nz, _int6(t), _int6(i),
        vals.ctypes.data_as(ctypes.POINTER(ctypes.c_double)),
        dev["q"].data_ptr(), dev["jac"].data_ptr(), dev["xi"].data_ptr(), dev["eta"].data_ptr(),
        dev["zeta"].data_ptr(), dev["dxyz"].data_ptr(), rhs.data_ptr(),
        ctypes.byref(dt) if dt is not None else None, ctypes.c_void_p(stream))


@pytest.mark.gpu
@pytest.mark.parametrize("exact", [True, False])
@pytest.mark.parametrize("name", CASES)
def test_noalloc_matches_allocating_rhs(name, exact):
    import torch
    import nuc3d_b200 as nb

    g = G.load(name)
    s = G.solver(g, exact=exact)
    dt_ref = s.rhs()
    rhs_ref = s.get_rhs(0)
    s.close()
    if exact:
        assert np.array_equal(rhs_ref, g.rhs)

    m = nb.metrics_from_nodes(*G.nodes(g))
    cuda = lambda a: torch.from_numpy(np.ascontiguousarray(a, dtype=np.float64)).cuda()  # noqa: E731
    dev = {"q": cuda(g.q0), "jac": cuda(m["jac"]), "xi": cuda(m["xi_xyz"]),
           "eta": cuda(m["eta_xyz"]), "zeta": cuda(m["zeta_xyz"]), "dxyz": cuda(m["dxyz"])}
    lib = nb.load_library()
    cfg_c = G.nuc3d_config(g, exact)._c()
    stream = torch.cuda.current_stream().cuda_stream
    for _ in range(2):
        rhs = torch.full_like(dev["q"], float("nan"))
        dt = ctypes.c_double()
        rc = _call(lib, cfg_c, g.cfg["shape"], G.bc_arrays(g), dev, rhs, dt, stream)
        assert rc == 0, lib.nuc3d_last_error().decode()
        got = rhs.cpu().numpy()
        if exact:
            assert dt.value == dt_ref
            assert np.array_equal(got, rhs_ref), float(np.nanmax(np.abs(got - rhs_ref)))
        else:
            # the allocating path runs the pipelined sweeps, this one the one-tile-per-CTA
            # sweeps; the throughput build contracts FMAs per kernel: round-off apart
            assert abs(dt.value - dt_ref) <= 1e-11 * dt_ref
            err = float(np.max(np.abs(got - rhs_ref)) / np.max(np.abs(rhs_ref)))
            assert err < 1e-11, err


def test_noalloc_rejects_what_it_cannot_do():
    """Argument checks run before any CUDA call, so this needs no GPU."""
    import nuc3d_b200 as nb

    try:
        lib = nb.load_library()
    except ImportError:
        pytest.skip("library not built")
    g = G.load("sphere_euler_weno5z_ausm_outlet")
    dummy = {k: type("P", (), {"data_ptr": lambda self: 1})() for k in
             ("q", "jac", "xi", "eta", "zeta", "dxyz")}
    rhs = dummy["q"]
    ns = G.nuc3d_config(g)._c()
    ns.model = b"NavierStokes3d"
    assert _call(lib, ns, (16, 16, 16), G.bc_arrays(g), dummy, rhs, None, 0) == nb.NUC3D_ENOTSUP
    big = G.nuc3d_config(g)._c()
    rc = _call(lib, big, (512, 512, 512), G.bc_arrays(g), dummy, rhs, None, 0)
    assert rc == nb.NUC3D_EINVAL
    assert b"8 MiB" in lib.nuc3d_last_error()
