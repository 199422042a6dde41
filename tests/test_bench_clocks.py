"""The bench's clock record (CPU): the summary of nvidia-smi samples taken during the timed
region, which decides whether a run saw a slowdown."""
import bench

U = "GPU-0f1e"


def _line(sm, smax, reasons=("Not Active",) * 4, uuid=U):
    return ", ".join([uuid, str(sm), str(smax), "650.12", "0x0000000000000000", *reasons])


def test_median_clock_and_no_reason():
    out = bench.Clocks.summarize([_line(1965, 1965), _line(1950, 1965), _line(1965, 1965)], U)
    assert out == {"sm_mhz": 1965.0, "sm_max_mhz": 1965.0, "reasons": [], "samples": 3}


def test_active_reasons_are_reported_by_name():
    lines = [_line(1300, 1965, ("Not Active", "Not Active", "Not Active", "Active")),
             _line(1200, 1965, ("Active", "Not Active", "Not Active", "Active"))]
    out = bench.Clocks.summarize(lines, U)
    assert out["reasons"] == ["hw_slowdown", "sw_power_cap"] and out["sm_mhz"] == 1250.0


def test_other_gpus_and_malformed_lines_are_ignored():
    lines = [_line(900, 1965, uuid="GPU-other"), "garbage", "", _line(1965, 1965)]
    out = bench.Clocks.summarize(lines, U)
    assert out["samples"] == 1 and out["sm_mhz"] == 1965.0
    assert bench.Clocks.summarize(lines, None)["samples"] == 2


def test_unavailable_fields_and_no_samples():
    out = bench.Clocks.summarize([_line("[N/A]", "[N/A]")], U)
    assert out["sm_mhz"] is None and out["sm_max_mhz"] is None and out["samples"] == 1
    assert bench.Clocks.summarize([], U) is None
