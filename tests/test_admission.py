"""The served commits' admission rule (zeknox_b200/csrc/admission.h), on the
CPU: the function the server's dispatcher calls, built here with g++ through
a small C shim.  Checked: first in, first out when the delay budgets are
zero; shortest first among the jobs that may start; memory held back for the
oldest job while it waits; and, over random arrival / start / completion
sequences, that no job's delay budget is overdrawn, that admitted bytes never
exceed the HBM budget, and that the oldest job starts whenever nothing runs
and its memory is free."""

import ctypes
import random
import shutil
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parent.parent


@pytest.fixture(scope="module")
def shim(tmp_path_factory):
    gxx = shutil.which("g++")
    if gxx is None:
        pytest.skip("g++ not available")
    out = tmp_path_factory.mktemp("admission") / "libadmission_shim.so"
    subprocess.run([gxx, "-std=c++17", "-O2", "-shared", "-fPIC", "-I", str(ROOT / "zeknox_b200" / "csrc"),
                    str(ROOT / "tests" / "admission_shim.cpp"), "-o", str(out)], check=True)
    lib = ctypes.CDLL(str(out))
    D, U = ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_uint64)
    lib.shim_pick.argtypes = [D, D, U, ctypes.c_size_t, D, ctypes.c_size_t, ctypes.c_uint64, ctypes.c_uint64]
    lib.shim_pick.restype = ctypes.c_long
    lib.shim_charge.argtypes = [D, D, U, ctypes.c_size_t, D, ctypes.c_size_t, ctypes.c_long]
    lib.shim_charge.restype = None
    return lib


def _arr(ctype, xs):
    return (ctype * max(1, len(xs)))(*xs)


def pick(lib, queue, running, in_use, budget):
    """queue: [(est, budget_s, bytes)] in submission order; running: [budget_s]."""
    est = _arr(ctypes.c_double, [j[0] for j in queue])
    bud = _arr(ctypes.c_double, [j[1] for j in queue])
    byt = _arr(ctypes.c_uint64, [j[2] for j in queue])
    run = _arr(ctypes.c_double, running)
    return lib.shim_pick(est, bud, byt, len(queue), run, len(running), in_use, budget)


def charge(lib, queue, running, q):
    est = _arr(ctypes.c_double, [j[0] for j in queue])
    bud = _arr(ctypes.c_double, [j[1] for j in queue])
    byt = _arr(ctypes.c_uint64, [j[2] for j in queue])
    run = _arr(ctypes.c_double, running)
    lib.shim_charge(est, bud, byt, len(queue), run, len(running), q)
    return [bud[i] for i in range(len(queue))], [run[i] for i in range(len(running))]


def test_fifo_when_budgets_are_zero(shim):
    queue = [(5.0, 0.0, 10), (0.1, 0.0, 10), (0.01, 0.0, 10)]
    assert pick(shim, queue, [], 0, 100) == 0  # the oldest, even though it is the longest
    assert pick(shim, queue[1:], [0.0], 10, 100) == -1  # nothing starts beside a running job


def test_shortest_first_among_the_jobs_that_fit_every_budget(shim):
    # running job: 1.0 s of budget left; queue: a long job (budget 0.25) and two short ones
    queue = [(5.0, 0.25, 10), (0.3, 0.015, 10), (0.2, 0.01, 10), (0.005, 0.0, 10)]
    # q0 exceeds the running job's budget; q1 exceeds q0's 0.25; q2 exceeds q1's 0.015; q3 fits all
    assert pick(shim, queue, [1.0], 10, 100) == 3
    queue = [(5.0, 0.25, 10), (0.2, 0.5, 10), (0.1, 0.5, 10)]
    assert pick(shim, queue, [1.0], 10, 100) == 2  # both fit: the shorter
    bud, run = charge(shim, queue, [1.0], 2)
    assert run == [pytest.approx(0.9)] and bud == [pytest.approx(0.15), pytest.approx(0.4), 0.5]


def test_memory_is_held_back_for_the_oldest_job(shim):
    queue = [(1.0, 1.0, 30), (0.01, 0.0, 10)]
    assert pick(shim, queue, [10.0], 80, 100) == -1  # 10 more would leave the oldest's 30 no room
    assert pick(shim, queue, [10.0], 60, 100) == 1  # both fit: the shorter, within the oldest's budget
    assert pick(shim, [(1.0, 1.0, 30), (2.0, 0.0, 10)], [10.0], 60, 100) == 0  # the other exceeds its budget
    assert pick(shim, [(1.0, 1.0, 200)], [], 0, 100) == -1  # larger than the budget (the server fails it)


@pytest.mark.parametrize("seed,frac", [(1, 0.05), (2, 0.05), (3, 0.2), (4, 0.0)])
def test_random_sequences_keep_the_invariants(shim, seed, frac):
    rng = random.Random(seed)
    BUDGET = 1000
    queue, running, in_use, started = [], [], 0, []  # running: [id, budget_s, bytes]
    next_id = 0
    for _ in range(3000):
        op = rng.random()
        if op < 0.45:  # arrival
            est = rng.choice([rng.uniform(0.001, 0.02), rng.uniform(0.05, 0.5), rng.uniform(1.0, 3.0)])
            queue.append([next_id, est, frac * est, rng.choice([5, 20, 100, 400, 800])])
            next_id += 1
        elif op < 0.7 and running:  # a completion
            i = rng.randrange(len(running))
            in_use -= running[i][2]
            running.pop(i)
        else:  # the dispatcher runs once
            q = pick(shim, [(j[1], j[2], j[3]) for j in queue], [r[1] for r in running], in_use, BUDGET)
            if q < 0:
                # nothing may start: then something runs, or the oldest job's memory is not free
                assert running or not queue or in_use + queue[0][3] > BUDGET
                continue
            bud, run = charge(shim, [(j[1], j[2], j[3]) for j in queue], [r[1] for r in running], q)
            for j, b in zip(queue, bud):
                j[2] = b
            for r, b in zip(running, run):
                r[1] = b
            job = queue.pop(q)
            if frac == 0.0:
                assert q == 0 and not running  # strict FIFO, one job at a time
            running.append([job[0], job[2], job[3]])
            in_use += job[3]
            started.append(job[0])
        # invariants after every step
        assert in_use <= BUDGET
        assert all(j[2] >= -1e-12 for j in queue) and all(r[1] >= -1e-12 for r in running)
    assert len(started) > 100
    if frac == 0.0:
        assert started == sorted(started)
