"""bench.py's host-side pieces, without a GPU: the clock record's parsing (median SM clock,
throttle reasons), the reference's rank split, the algorithmic flop tally the roofline
divides by, and the whole-job rate."""
import os
import tempfile

import pytest

import bench


def _summary(lines):
    c = bench.ClockSampler(0)
    c.p = object()  # stands in for the nvidia-smi process: summary() reads the file only
    c.out = tempfile.NamedTemporaryFile("w+", suffix=".csv", delete=False)
    c.out.write("\n".join(lines) + "\n")
    c.out.flush()
    name = c.out.name
    s = c.summary()
    assert not os.path.exists(name)  # the record is removed once read
    return s


def test_clock_summary_median_and_reasons():
    rows = [
        "0, 1965, 1965, 480.5, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
        "0, 1950, 1965, 990.1, 0x0000000000000004, Not Active, Not Active, Not Active, Active",
        "0, 1965, 1965, 500.0, 0x0000000000000000, Not Active, Not Active, Not Active, Not Active",
    ]
    s = _summary(rows)
    assert s["sm_mhz"] == 1965.0 and s["sm_max_mhz"] == 1965.0
    assert s["reasons"] == ["sw_power_cap"] and s["samples"] == 3
    assert s["power_w_max"] == pytest.approx(990.1)


def test_clock_summary_flags_thermal_and_hw_slowdown():
    rows = [
        "0, 1200, 1965, 700.0, 0x0000000000000048, Active, Not Active, Active, Not Active",
        "0, 1210, 1965, 700.0, 0x0000000000000048, Not Active, Active, Not Active, Not Active",
        "0, [N/A], [N/A], [N/A], [N/A], [N/A], [N/A], [N/A], [N/A]",
    ]
    s = _summary(rows)
    assert s["reasons"] == ["hw_slowdown", "hw_thermal_slowdown", "sw_thermal_slowdown"]
    assert s["sm_mhz"] == pytest.approx(1205.0) and s["samples"] == 3


def test_clock_summary_without_sampler():
    assert bench.ClockSampler(0).summary() is None


@pytest.mark.parametrize("shape,nranks,parts", [
    ((256, 256, 256), 16, [4, 2, 2]),
    ((64, 64, 64), 8, [2, 2, 2]),
    ((256, 256, 256), 1, [1, 1, 1]),
    ((48, 48, 48), 128, [4, 4, 4]),  # halving stops where a block would drop below 12 cells
])
def test_decompose(shape, nranks, parts):
    got = bench.decompose(shape, nranks)
    assert got == parts
    for d in range(3):
        ext = shape[d] // got[d]
        assert ext * got[d] == shape[d] and ext % 4 == 0


def test_sweep_flops_tally():
    F = bench.FLOPS
    faces = 10 * F["weno5z"] + 5 * F["combine"] + 5 * F["difference"]
    assert bench.sweep_flops_per_cell(0) == F["AUSM"] + faces + F["con2prim"] == 878
    assert bench.sweep_flops_per_cell(1) == bench.sweep_flops_per_cell(2) == F["AUSM"] + faces + 5 == 837
    # Navier-Stokes: the direction's cd6 differences of 4 viscous fluxes and their subtraction
    assert bench.sweep_flops_per_cell(1, ns=True) - bench.sweep_flops_per_cell(1) == 4 * 8 + 4
    assert bench.sweep_flops_per_cell(0, scheme="weno7js", riemann="LF") == 60 + 10 * 146 + 10 + 46


def test_whole_job_rate():
    # 256^3 cells, 20 steps in 237.2 ms on one rank: 1414.6 Mcell-RK3-steps/s
    assert bench.whole_job_rate(1, 256 ** 3, 20, 237.2) == pytest.approx(1414.605, rel=1e-6)
    # N ranks, the slowest rank's time: N times the cells over the same time
    assert bench.whole_job_rate(4, 256 ** 3, 20, 237.2) == pytest.approx(4 * 1414.605, rel=1e-6)
