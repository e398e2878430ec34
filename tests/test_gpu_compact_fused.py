"""The throughput build's fused compact sweep (compact_line_kernel: one CTA per line, each
(variable, split) system solved by one warp with the partition method and cyclic
reduction) against the reference's Thomas solve (src/crweno5.cpp:207-218,
src/hccs.cpp:253-264): the reference itself through the golden fixtures, the
reference-order build (Thomas in the reference's operation order) on larger grids, and the
throughput build's own three-kernel path.  The operation order differs from Thomas, so the
bar is round-off: 1e-11 relative max-norm against the reference after the fixtures' steps
and between the two throughput paths (the nonlinear weights carry round-off differences
of one solve into the next)."""
import numpy as np
import pytest

from tests import golden_cases as G

COMPACT = ["crweno5_euler_lf_periodic", "hccs_ns_ausm_bc", "mixed_compact_ausmp"]


def rel_max(a, b):
    return float(np.max(np.abs(a - b)) / np.max(np.abs(b)))


def _expected_dirs(g):
    return sum(1 << d for d, s in enumerate(g.cfg["schemes"]) if s in ("crweno5", "hccs"))


@pytest.mark.gpu
@pytest.mark.parametrize("name", COMPACT)
def test_fused_against_reference(name):
    g = G.load(name)
    s = G.solver(g, exact=False)
    assert s.compact_solver() == _expected_dirs(g)
    s.step(int(g.cfg["nsteps"]))
    assert rel_max(s.get_q(0), g.qn) < 1e-11
    s.close()


@pytest.mark.gpu
@pytest.mark.parametrize("name", COMPACT)
def test_fused_against_three_kernels(name):
    g = G.load(name)
    out = []
    for fused in (True, False):
        s = G.solver(g, exact=False)
        s.set_compact_solver(fused)
        assert s.compact_solver() == (_expected_dirs(g) if fused else 0)
        s.step(int(g.cfg["nsteps"]))
        out.append((s.get_q(0), s.time_dt(), s.residual()))
        s.close()
    (qa, (ta, dta), ra), (qb, (tb, dtb), rb) = out
    assert rel_max(qa, qb) < 1e-11
    assert abs(dta - dtb) <= 1e-12 * dtb and abs(ra - rb) <= 1e-8 * max(abs(rb), 1e-300)


def _pulse(shape, scheme, exact, fused=True, nblocks=1):
    """A smooth pressure pulse (the spherical blast's discontinuity makes the compact
    schemes oscillate into negative pressure within a few steps at 256 cells per line,
    in the reference too: it resets the energy of 1144 cells in 4 steps at 64^3)."""
    import nuc3d_b200 as nb
    from nuc3d_b200 import cases as C
    q, m = C.gaussian_pulse(shape)
    s = nb.Solver(nb.Config(scheme_ivs=(scheme,) * 3, riemann="AUSM", model="Euler3d", mach=1.0,
                            exact=exact))
    if nblocks == 1:
        b = s.add_block(*shape, *C.outlet_faces())
        s.set_metrics(b, m["jac"], m["xi_xyz"], m["eta_xyz"], m["zeta_xyz"], m["dxyz"])
        s.finalize()
        s.set_q(b, q)
    else:  # two blocks cut along xi
        h = shape[0] // 2
        t0, i0 = [-1, 1, -1, -1, -1, -1], [1, 0, 1, 1, 1, 1]
        t1, i1 = [0, -1, -1, -1, -1, -1], [1, 1, 1, 1, 1, 1]
        s.add_block(h, shape[1], shape[2], t0, i0)
        s.add_block(shape[0] - h, shape[1], shape[2], t1, i1)
        for b, sl in enumerate((slice(0, h), slice(h, shape[0]))):
            mm = {k: np.ascontiguousarray(v[..., sl]) for k, v in m.items() if k != "dxyz"}
            s.set_metrics(b, mm["jac"], mm["xi_xyz"], mm["eta_xyz"], mm["zeta_xyz"])
        s.finalize()
        s.set_q(0, np.ascontiguousarray(q[..., :h]))
        s.set_q(1, np.ascontiguousarray(q[..., h:]))
    if not exact:
        s.set_compact_solver(fused)
    return s


def _err_vs_exact(shape, scheme, steps, nblocks=1):
    """Relative max-norm distance from the reference-order build after `steps` steps of
    the throughput build's three-kernel path and of its fused path."""
    out = {}
    for key, exact, fused in (("exact", True, False), ("three", False, False), ("fused", False, True)):
        s = _pulse(shape, scheme, exact, fused, nblocks)
        if key == "fused":
            ts = 4 if scheme == "hccs" else 3
            assert s.compact_solver() == sum(1 << d for d in range(3) if shape[d] <= 256
                                             and shape[d] - 2 * ts + 1 >= 2)
        s.step(steps)
        out[key] = [s.get_q(b) for b in range(nblocks)]
        s.close()
    err = {k: max(rel_max(a, b) for a, b in zip(out[k], out["exact"])) for k in ("three", "fused")}
    return err["three"], err["fused"]


@pytest.mark.gpu
@pytest.mark.parametrize("scheme,shape", [("crweno5", (256, 24, 20)), ("crweno5", (96, 8, 9)),
                                          ("hccs", (256, 24, 20)), ("hccs", (96, 10, 11))])
def test_fused_line_lengths(scheme, shape):
    """Lines of 256 cells (the longest fused system: 32 lanes x 8 rows), of 24 and 20
    (a few lanes of 2-3 rows) and of the shortest lines a block may have (8, 9 for crweno5;
    10, 11 for hccs: 2 bfsize + 2 cells; one lane).  The bar is the throughput build's own
    three-kernel path: hccs's switch theta (its weights' epsilon is 1e-40) turns the
    round-off of any operation order into differences up to 1e-8 after 3 steps here, and
    up to 2e-5 on a 64^3 block, with Thomas as with the fused solve."""
    three, fused = _err_vs_exact(shape, scheme, 3)
    assert fused <= max(1e-11, 4.0 * three), (fused, three)


@pytest.mark.gpu
def test_fused_two_blocks_and_long_lines():
    """Two blocks of one context (the line's halo from the neighbour block), and a grid
    whose xi lines exceed 256 cells (xi stays on the three-kernel path)."""
    for shape, nb_ in (((128, 32, 24), 2), ((320, 16, 16), 1)):
        three, fused = _err_vs_exact(shape, "crweno5", 2, nb_)
        assert fused <= max(1e-11, 4.0 * three), (shape, fused, three)
