"""Host logic of the bench's multi-job sections, on the CPU: the FIFO queue the
plain arm's latencies come from, the per-job seeds, the seeded job lists of
configs 3 and 5, the oracle restatement of the synthetic-input stream, and the
rule that profiler figures are reported only for the kernel sources they were
captured from."""

import json

import numpy as np


def test_fifo_latencies_single_server_queue():
    import bench

    # idle server: each job's latency is its own service time
    lat, span = bench.fifo_latencies([0.0, 10.0, 20.0], [1.0, 2.0, 3.0])
    assert lat == [1.0, 2.0, 3.0] and span == 23.0
    # a burst: later jobs wait for the earlier ones, in arrival order
    lat, span = bench.fifo_latencies([0.0, 0.5, 1.0], [2.0, 2.0, 1.0])
    assert lat == [2.0, 3.5, 4.0] and span == 5.0
    # random check against an event-by-event simulation
    rng = np.random.default_rng(5)
    arr = np.cumsum(rng.exponential(1.0, 200))
    sv = rng.exponential(0.9, 200)
    lat, _ = bench.fifo_latencies(arr, sv)
    free_at = 0.0
    for a, s, got in zip(arr, sv, lat):
        start = a if a >= free_at else free_at
        free_at = start + s
        assert abs(got - (free_at - a)) < 1e-9


def test_job_seeds_are_distinct_and_config_specific():
    import bench

    s3 = [bench.job_seed(3, j) for j in range(10000)]
    s5 = [bench.job_seed(5, j) for j in range(10000)]
    assert len(set(s3)) == 10000 and len(set(s5)) == 10000 and not set(s3) & set(s5)
    assert all(0 <= s < 2**64 for s in s3)


def test_job_lists_match_the_configurations():
    import bench

    b = bench._jobs(0x5EED0003, 256, 12, 20, 4, 200, [1, 2, 3])
    assert len(b) == 256 and all(12 <= lg <= 20 and 4 <= p <= 200 and r in (1, 2, 3) for lg, p, r in b)
    s = bench._jobs(0x5EED0005, 10000, 12, 22, 8, 300, [3])
    assert all(12 <= lg <= 22 and 8 <= p <= 300 and r == 3 for lg, p, r in s)
    assert {lg for lg, _, _ in s} == set(range(12, 23))  # the whole size range, lg_n 22 included


def test_fill_field_stream_is_uniform_in_the_field(oracle):
    x = oracle.fill_field(0x5EED0005, 1 << 18)
    assert x.dtype == np.uint64 and (x < np.uint64(oracle.P)).all()
    # the top quarter of the field appears (values above 3p/4)
    assert (x > np.uint64(3 * (oracle.P // 4))).mean() > 0.2
    # deterministic in (seed, count), and different seeds give different streams
    assert np.array_equal(x, oracle.fill_field(0x5EED0005, 1 << 18))
    assert not np.array_equal(x, oracle.fill_field(0x5EED0006, 1 << 18))


def test_profile_figures_only_for_the_sources_they_were_captured_from(tmp_path, monkeypatch):
    import bench

    f = tmp_path / "fig.json"
    monkeypatch.setattr(bench, "PROFILE_FIGURES", f)
    assert bench.profile_figures() == {}
    f.write_text(json.dumps({"sources_sha256": "0" * 64, "kernels": {"k": {"dram_bytes_per_launch": 1}}}))
    assert bench.profile_figures() == {}  # stale: captured from other sources
    f.write_text(json.dumps({"sources_sha256": bench.kernel_sources_sha256(),
                             "kernels": {"k": {"dram_bytes_per_launch": 1}}}))
    assert bench.profile_figures()["kernels"]["k"]["dram_bytes_per_launch"] == 1


def test_profile_figures_written_from_a_launch_list(tmp_path):
    """The figures file is derived from ncu's CSV launch list of one fused step
    (LDE passes, then the Merkle kernels) plus the plain path's transpose."""
    import csv

    import bench

    cols = ["ID", "Process ID", "Process Name", "Host Name", "Kernel Name", "Context", "Stream", "Block Size",
            "Grid Size", "Device", "CC", "Section Name", "Metric Name", "Metric Unit", "Metric Value"]
    launches = ["ntt_column_fixed<9, 3, 6, 0>(PassArgs)", "ntt_leaves_fixed<9, 3>(PassArgs)",
                "merkle_leaves_hex(...)", "merkle_level(...)", "ntt_column_fixed<9, 3, 6, 0>(PassArgs)",
                "transpose_rev_kernel<true>(...)"]
    path = tmp_path / "figures.csv"
    with open(path, "w", newline="") as f:
        w = csv.writer(f)
        w.writerow(cols)
        for i, name in enumerate(launches):
            for m, v in [("dram__bytes_read.sum", 1000 * (i + 1)), ("dram__bytes_write.sum", 10),
                         ("smsp__inst_executed.sum", 2 ** 20), ("gpu__time_duration.sum", 5)]:
                w.writerow([i, 1, "python", "h", name, 1, 7, "(256, 1, 1)", "(8, 1, 1)", 0, "10.0", "", m, "", f"{v:,}"])
    out = tmp_path / "fig.json"
    fig = bench.write_profile_figures(path, out)
    k = fig["kernels"]
    assert k["lde_leaves 135x2^15 rate 3"]["dram_bytes_per_launch"] == 1010 + 2010
    assert k["merkle poseidon 262144x135 cap 4"]["dram_bytes_per_launch"] == 3010 + 4010
    assert k["transpose_rev 135x2^18"]["dram_bytes_per_launch"] == 6010
    assert abs(k["lde_leaves 135x2^15 rate 3"]["thread_inst_per_elem"] - 2 * 2 ** 20 * 32 / (135 << 18)) < 1e-9
    assert json.loads(out.read_text())["sources_sha256"] == bench.kernel_sources_sha256()
