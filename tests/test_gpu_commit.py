"""GPU parity of the commit-level extensions: the fused LDE -> leaves pass, the
single commit, the batched commit and the commit server, each bit-exact
against the drop-in entry points / the oracle, alone and in the mix."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def zk():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import zeknox_b200 as zk

    zk.init_coset(0, 24, 7)
    return zk


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


@pytest.mark.parametrize("lg_n,rate,b", [(4, 1, 3), (9, 3, 17), (10, 2, 135), (12, 3, 33), (15, 3, 135),
                                         (17, 2, 5), (18, 3, 7), (8, 1, 200), (20, 3, 3), (21, 3, 2)])
def test_lde_leaves_equals_lde_then_transpose(zk, oracle, lg_n, rate, b):
    import torch

    x = _dev(oracle.field_elems(300 + lg_n, b << lg_n)).view(b, 1 << lg_n)
    fused = zk.lde_leaves(x, rate)
    two_step = zk.transpose_rev(zk.lde(x, rate))
    torch.cuda.synchronize()
    assert torch.equal(fused.view(torch.int64), two_step.view(torch.int64))


@pytest.mark.parametrize("ht", [0, 3, 1])
def test_commit_vs_oracle(zk, oracle, ht):
    import torch

    lg_n, rate, b, ch = 9, 3, 135, 4
    x = oracle.field_elems(55 + ht, b << lg_n)
    out = zk.commit(_dev(x).view(b, 1 << lg_n), rate, ch, ht)
    torch.cuda.synchronize()
    leaves = oracle.transpose_rev(oracle.batch_lde(x, lg_n, rate, b), lg_n + rate, b)
    d, c = oracle.merkle_fill(leaves, b, ch, ht)
    assert np.array_equal(out.leaves.cpu().numpy().reshape(-1), leaves)
    assert np.array_equal(out.digests.cpu().numpy().reshape(-1), d)
    assert np.array_equal(out.cap.cpu().numpy().reshape(-1), c)


def _mixed_jobs(oracle, n_jobs, seed):
    """Shapes drawn like the batched workload (log size, width, rate), scaled down."""
    rng = np.random.default_rng(seed)
    jobs = []
    for i in range(n_jobs):
        lg_n = int(rng.integers(4, 13))
        b = int(rng.integers(4, 201))
        rate = int(rng.integers(1, 4))
        ch = int(min(4, lg_n + rate - 1))
        ht = [0, 3, 1][i % 3]
        jobs.append((oracle.field_elems(seed * 1000 + i, b << lg_n).reshape(b, 1 << lg_n), rate, ch, ht))
    return jobs


def test_commit_batch_equals_individual_commits(zk, oracle):
    import torch

    jobs = _mixed_jobs(oracle, 24, 7)
    alone, batch = [], []
    for x, r, ch, ht in jobs:
        d = _dev(x)
        alone.append(zk.commit(d, r, ch, ht))
        batch.append((d, r, ch, ht, zk.CommitBuffers(x.shape[1] << r, x.shape[0], ch)))
    zk.commit_batch(batch, n_streams=4)
    torch.cuda.synchronize()
    for a, (_, _, _, _, o) in zip(alone, batch):
        assert torch.equal(a.cap.view(torch.int64), o.cap.view(torch.int64))
        assert torch.equal(a.digests.view(torch.int64), o.digests.view(torch.int64))
        assert torch.equal(a.leaves.view(torch.int64), o.leaves.view(torch.int64))


def test_server_results_same_alone_and_in_the_mix(zk, oracle):
    """Every cap from the server (jobs overlapping on 4 slots under a small HBM
    budget, so some queue) equals the same job committed alone."""
    import torch

    jobs = _mixed_jobs(oracle, 30, 11)
    want = []
    for x, r, ch, ht in jobs:
        want.append(zk.commit(_dev(x), r, ch, ht).cap.cpu().numpy())
    torch.cuda.synchronize()
    biggest = max(x.nbytes * ((1 << r) * 2 + 1) for x, r, _, _ in jobs)
    with zk.Server(hbm_budget_bytes=3 * biggest, slots=4) as srv:
        tickets = [srv.submit(x, r, ch, ht) for x, r, ch, ht in jobs]
        for t, w in zip(tickets, want):
            cap, lat = srv.wait(t)
            assert np.array_equal(cap, w) and lat > 0
        # the tree stays on the device until released
        lp, dp, cp = srv.result_ptrs(tickets[0])
        assert lp and cp
        st = srv.stats()
        assert st["completed"] == len(jobs) and st["p99_s"] >= st["p50_s"] > 0
        assert st["hbm_peak"] <= 3 * biggest
        for t in tickets:
            srv.release(t)
        assert srv.stats()["hbm_in_use"] == 0


def test_server_rejects_job_over_budget(zk, oracle):
    x = oracle.field_elems(1, 8 << 10).reshape(8, 1 << 10)
    with zk.Server(hbm_budget_bytes=1 << 16, slots=2) as srv:
        t = srv.submit(x, 3, 4, 0)
        with pytest.raises(zk.ZeknoxError):
            srv.wait(t)
        srv.release(t)


def test_server_wait_any_returns_each_job_once(zk, oracle):
    """wait_any hands out every finished ticket exactly once, then None; the
    caps equal the jobs committed alone."""
    import torch

    jobs = _mixed_jobs(oracle, 12, 23)
    want = [zk.commit(_dev(x), r, ch, ht).cap.cpu().numpy() for x, r, ch, ht in jobs]
    torch.cuda.synchronize()
    with zk.Server(hbm_budget_bytes=4 << 30, slots=3) as srv:
        tickets = [srv.submit(x, r, ch, ht) for x, r, ch, ht in jobs]
        seen = []
        while len(seen) < len(jobs):
            t = srv.wait_any(timeout_ms=60000)
            assert t is not None
            seen.append(t)
            cap, _ = srv.wait(t)
            assert np.array_equal(cap, want[tickets.index(t)])
            srv.release(t)
        assert sorted(seen) == sorted(tickets)
        assert srv.wait_any(timeout_ms=0) is None
        assert srv.stats()["hbm_in_use"] == 0


def test_server_equal_jobs_submitted_together_run_in_fifo_order(zk, oracle):
    """Jobs of one size submitted together leave one another no slack past
    their FIFO finish times: they run one at a time in arrival order, so
    completions come back in submission order."""
    import torch

    x = oracle.field_elems(2929, 24 << 13).reshape(24, 1 << 13)
    want = zk.commit(_dev(x), 3, 4, 0).cap.cpu().numpy()
    torch.cuda.synchronize()
    with zk.Server(hbm_budget_bytes=4 << 30, slots=4) as srv:
        tickets = [srv.submit(x, 3, 4, 0) for _ in range(8)]
        order = [srv.wait_any(timeout_ms=60000) for _ in tickets]
        assert order == tickets
        for t in tickets:
            assert np.array_equal(srv.wait(t)[0], want)
            srv.release(t)
        assert srv.stats()["hbm_in_use"] == 0


def test_server_short_job_runs_beside_a_long_one(zk, oracle):
    """A short job submitted right behind a long one fits in the long job's
    slack: it is admitted at once, beside it, and finishes first."""
    with zk.Server(hbm_budget_bytes=16 << 30, slots=4) as srv:
        big = srv.submit_seeded(11, 20, 64, 3, 4)   # 64 x 2^20 -> 2^23 leaves: tens of ms
        small = srv.submit_seeded(12, 8, 4, 1, 2)   # 4 x 2^8 -> 2^9 leaves
        first = srv.wait_any(timeout_ms=60000)
        second = srv.wait_any(timeout_ms=60000)
        assert (first, second) == (small, big)
        for t in (big, small):
            srv.wait(t)
            srv.release(t)


def test_fill_field_matches_the_oracle_stream(zk, oracle):
    import torch

    out = torch.empty(100003, dtype=torch.uint64, device="cuda")
    zk.fill_field(out, 0x5EED0005)
    torch.cuda.synchronize()
    assert np.array_equal(out.cpu().numpy(), oracle.fill_field(0x5EED0005, 100003))


def test_server_seeded_jobs_equal_commits_of_their_inputs(zk, oracle):
    """A seeded job commits fill_field(seed) generated on the device at
    admission: its cap equals the commit of that input made alone, and (small
    shapes) the oracle's commit of the same stream."""
    import torch

    shapes = [(9, 2, 17, 2), (12, 3, 40, 4), (15, 1, 9, 4), (10, 3, 135, 3), (14, 2, 200, 4)]
    with zk.Server(hbm_budget_bytes=4 << 30, slots=4) as srv:
        tickets = [srv.submit_seeded(7000 + k, lg_n, b, r, ch) for k, (lg_n, r, b, ch) in enumerate(shapes)]
        for k, ((lg_n, r, b, ch), t) in enumerate(zip(shapes, tickets)):
            cap, _ = srv.wait(t)
            x = torch.empty((b, 1 << lg_n), dtype=torch.uint64, device="cuda")
            zk.fill_field(x, 7000 + k)
            alone = zk.commit(x, r, ch, 0).cap.cpu().numpy()
            assert np.array_equal(cap, alone)
            if b << lg_n <= 1 << 16:
                xs = oracle.fill_field(7000 + k, b << lg_n)
                leaves = oracle.transpose_rev(oracle.batch_lde(xs, lg_n, r, b), lg_n + r, b)
                _, want = oracle.merkle_fill(leaves, b, ch, oracle.HASH_POSEIDON)
                assert np.array_equal(cap.reshape(-1), want)
            srv.release(t)


@pytest.mark.parametrize("at_allocation", [1, 2, 4])
def test_server_injected_allocation_failure_frees_and_keeps_serving(zk, oracle, at_allocation):
    """Host-side fault injection: one job's at_allocation-th device allocation
    fails.  That job reports the error; what it had allocated is freed and its
    budget returned (hbm_in_use back to 0), and the jobs around it complete
    with the caps they have alone."""
    import torch

    jobs = [(9, 3, 20, 2), (11, 2, 33, 3), (10, 3, 7, 4), (12, 1, 60, 4)]
    with zk.Server(hbm_budget_bytes=1 << 30, slots=2) as srv:
        first = srv.submit_seeded(8100, jobs[0][0], jobs[0][2], jobs[0][1], jobs[0][3])
        srv.wait(first)
        srv.inject_failure(1, at_allocation)
        tickets = [srv.submit_seeded(8101 + k, lg_n, b, r, ch) for k, (lg_n, r, b, ch) in enumerate(jobs[1:])]
        with pytest.raises(zk.ZeknoxError, match="injected allocation failure"):
            srv.wait(tickets[0])
        for k, t in enumerate(tickets[1:], start=1):
            lg_n, r, b, ch = jobs[k + 1]
            x = torch.empty((b, 1 << lg_n), dtype=torch.uint64, device="cuda")
            zk.fill_field(x, 8101 + k)
            assert np.array_equal(srv.wait(t)[0], zk.commit(x, r, ch, 0).cap.cpu().numpy())
        for t in [first, *tickets]:
            srv.release(t)
        st = srv.stats()
        assert st["hbm_in_use"] == 0 and st["completed"] == 3


def test_commit_batch_graph_replays_bit_exact(zk, oracle):
    """A batch captured into a CUDA graph reproduces the individual commits,
    and commits new coefficients written into the same inputs on replay."""
    import torch

    jobs = _mixed_jobs(oracle, 10, 31)
    items = []
    for x, r, ch, ht in jobs:
        d = _dev(x)
        b, n = d.shape
        items.append((d, r, ch, ht, zk.CommitBuffers(n << r, b, ch)))
    g = zk.CommitGraph(items)
    for round_ in range(2):
        if round_:  # new values in the captured input buffers
            for k, (d, r, ch, ht, o) in enumerate(items):
                d.copy_(_dev(oracle.field_elems(900 + k, d.numel()).reshape(d.shape)))
        g.replay()
        torch.cuda.synchronize()
        for d, r, ch, ht, o in items:
            alone = zk.commit(d, r, ch, ht)
            torch.cuda.synchronize()
            assert torch.equal(alone.cap.view(torch.int64), o.cap.view(torch.int64))
            assert torch.equal(alone.digests.view(torch.int64), o.digests.view(torch.int64))
            assert torch.equal(alone.leaves.view(torch.int64), o.leaves.view(torch.int64))


def test_autotuner_choices_keep_outputs_bit_exact(zk, oracle):
    """Tuning the LDE -> leaves stage changes only how it runs: commits of the
    tuned shapes equal the untuned ones, and a tuned shape is not re-timed."""
    import torch

    zk.autotune_reset()
    for lg_n, rate, b in [(12, 3, 33), (15, 3, 135), (19, 3, 5), (21, 3, 2)]:
        x = _dev(oracle.field_elems(4400 + lg_n, b << lg_n)).view(b, 1 << lg_n)
        before = zk.commit(x, rate, 4, 0)
        torch.cuda.synchronize()
        assert zk.autotune(lg_n, rate, b) >= 1
        assert zk.autotune(lg_n, rate, b) == 0
        after = zk.commit(x, rate, 4, 0)
        torch.cuda.synchronize()
        assert torch.equal(before.leaves.view(torch.int64), after.leaves.view(torch.int64))
        assert torch.equal(before.cap.view(torch.int64), after.cap.view(torch.int64))
    zk.autotune_reset()


@pytest.mark.parametrize("lg_n,rate,b", [(10, 3, 135), (11, 3, 135), (12, 2, 9), (13, 3, 40), (12, 1, 200)])
def test_threads_per_hash_tuning_keeps_trees_bit_exact(zk, oracle, lg_n, rate, b):
    """Trees of up to 2^16 leaves also get their Poseidon leaf kernel (six, two
    or one thread per hash) by measurement; whichever wins, the forest equals
    the oracle's."""
    import torch

    zk.autotune_reset()
    x = oracle.field_elems(4500 + lg_n + b, b << lg_n)
    assert zk.autotune(lg_n, rate, b) >= 3  # at least the three leaf layouts
    out = zk.commit(_dev(x).view(b, 1 << lg_n), rate, 4, 0)
    torch.cuda.synchronize()
    lde = oracle.batch_lde(x, lg_n, rate, b)
    leaves = oracle.transpose_rev(lde, lg_n + rate, b)
    dig, cap = oracle.merkle_fill(leaves, b, 4, oracle.HASH_POSEIDON)
    assert np.array_equal(out.cap.cpu().numpy().reshape(-1), cap)
    assert np.array_equal(out.digests.cpu().numpy().reshape(-1)[:dig.size], dig)
    zk.autotune_reset()


def test_drop_in_abi_from_several_host_threads(zk, oracle):
    """zeknox's Rust tests run concurrently (cargo's test threads): the drop-in
    calls made from four host threads at once, on host buffers, give the same
    LDE and caps as the oracle (the per-device streams and tables are shared)."""
    import threading

    import torch

    shapes = [(9, 2, 20, 2), (10, 3, 7, 3), (8, 1, 33, 1), (11, 2, 3, 4)]  # lg_n, rate, batches, cap height
    want = []
    for k, (lg_n, rate, b, ch) in enumerate(shapes):
        x = oracle.field_elems(7100 + k, b << lg_n)
        lde = oracle.batch_lde(x, lg_n, rate, b)
        leaves = oracle.transpose_rev(lde, lg_n + rate, b)
        _, cap = oracle.merkle_fill(leaves, b, ch, oracle.HASH_POSEIDON)
        want.append((x, lde, cap))
    errors = []

    def worker(k):
        try:
            torch.cuda.set_device(0)
            lg_n, rate, b, ch = shapes[k]
            x, lde_want, cap_want = want[k]
            N = 1 << (lg_n + rate)
            nd, nc = 2 * (N - (1 << ch)), 1 << ch
            for _ in range(3):
                cfg = zk.NTTConfig.default()
                cfg.batches, cfg.extension_rate_bits, cfg.with_coset = b, rate, True
                lde = np.zeros(b * N, dtype=np.uint64)
                zk.lde_batch(0, lde.ctypes.data, x.ctypes.data, lg_n, cfg)  # host in, host out
                if not np.array_equal(lde, lde_want):
                    errors.append((k, "lde"))
                d_lde = torch.from_numpy(lde).cuda()
                d_leaves = torch.empty_like(d_lde)
                tcfg = zk.TransposeConfig.default()
                tcfg.batches, tcfg.are_inputs_on_device, tcfg.are_outputs_on_device = b, True, True
                zk.transpose_rev_batch(0, d_leaves.data_ptr(), d_lde.data_ptr(), lg_n + rate, tcfg)
                dig = torch.zeros(max(nd, 1) * 4, dtype=torch.uint64, device="cuda")
                cap = torch.zeros(nc * 4, dtype=torch.uint64, device="cuda")
                zk.fill_digests_buf_linear_gpu_with_gpu_ptr(dig.data_ptr(), cap.data_ptr(), d_leaves.data_ptr(), nd,
                                                            nc, N, b, ch, zk.HashPoseidon, 0)
                torch.cuda.synchronize()
                if not np.array_equal(cap.cpu().numpy(), cap_want):
                    errors.append((k, "cap"))
        except Exception as e:  # noqa: BLE001 - reported below
            errors.append((k, repr(e)))

    threads = [threading.Thread(target=worker, args=(k,)) for k in range(len(shapes))]
    for t in threads:
        t.start()
    for t in threads:
        t.join()
    assert not errors, errors
