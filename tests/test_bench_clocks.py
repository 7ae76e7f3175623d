"""The bench's clock record: nvidia-smi samples are summarised only from inside
the timed region (samples taken while the sampler starts, before the region,
are left out), throttle reasons seen there are reported, and unparsable lines
are skipped.  Host logic only, on canned nvidia-smi output."""

import datetime
import time


def _line(when: datetime.datetime, sm: int, power_cap: bool) -> str:
    stamp = when.strftime("%Y/%m/%d %H:%M:%S.%f")[:-3]
    cap = "Active" if power_cap else "Not Active"
    return f"{stamp}, {sm}, 1965, 900.00, 0x0000000000000004, Not Active, Not Active, Not Active, {cap}"


def test_only_samples_inside_the_timed_region_count():
    import bench

    c = bench.ClockSampler(0)
    now = time.time()
    c.t0, c.t1 = now, now + 1.0
    at = lambda s: datetime.datetime.fromtimestamp(now + s)  # noqa: E731
    c.out = "\n".join([
        _line(at(-0.3), 345, False),  # idle GPU while the sampler starts
        _line(at(0.1), 1965, False),
        _line(at(0.5), 1950, True),
        _line(at(0.9), 1965, False),
        _line(at(1.4), 600, False),  # after the region
        "not a sample",
    ])
    got = c.summary()
    assert got["samples"] == 3 and got["window"] == "timed region"
    assert got["sm_mhz"] == 1965 and got["sm_max_mhz"] == 1965
    assert got["reasons"] == ["sw_power_cap"]


def test_unstamped_samples_fall_back_to_the_whole_run():
    import bench

    c = bench.ClockSampler(0)
    c.t0, c.t1 = 0.0, 1.0
    c.out = "n/a, 1965, 1965, 900.00, 0x0, Not Active, Active, Not Active, Not Active"
    got = c.summary()
    assert got["samples"] == 1 and got["window"] == "whole sampler run"
    assert got["reasons"] == ["hw_thermal_slowdown"]


def test_no_output_gives_no_clock():
    import bench

    got = bench.ClockSampler(0).summary()
    assert got["samples"] == 0 and got["sm_mhz"] is None
