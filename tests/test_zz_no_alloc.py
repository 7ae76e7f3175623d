"""GPU test of zk_lde_noalloc, the LDE entry point that allocates nothing.

It exists for callers that cannot call cudaMalloc where they run the LDE:
provers held to a pre-reserved memory budget or their own arena (the regular
entry points grow the CUDA memory pool), and hot paths that forbid allocation
calls because they can synchronise the device.  It keeps its NTT
intermediate and tables in one static device array instead.  Here its output
is compared, bit for bit, with the regular stream-ordered entry point
(zk_lde_async) on two calls in a row, with the default coset generator and
with another one installed by init_coset; the test also checks the size
limit, that its launches are counted, and that a call leaves the device's
free memory unchanged.

The file is named so that pytest collects it last; it passes alone in a
fresh process and after the other tests.
"""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def zk():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import zeknox_b200 as zk

    torch.cuda.set_device(0)
    return zk


def _rand(seed, count):
    from oracle import oracle as O

    return O.field_elems(seed, count)


def _run(zk, fn, coeffs, lg_n, rate, batches, inverse, coset):
    import torch

    d_in = torch.from_numpy(coeffs).cuda()
    d_out = torch.zeros(batches << (lg_n + rate), dtype=torch.uint64, device="cuda")
    stream = torch.cuda.current_stream().cuda_stream
    zk.capi.check(fn(d_out.data_ptr(), d_in.data_ptr(), lg_n, rate, batches, int(inverse), int(coset), stream))
    torch.cuda.synchronize()
    return d_out.cpu().numpy()


SHAPES = [
    (15, 3, 5, False, True),   # two shared-memory passes, zero-extension skip
    (9, 2, 11, False, True),   # one pass
    (13, 3, 3, True, True),    # inverse direction, coset applied on output
    (19, 3, 2, False, False),  # the largest accepted size (2^22 points)
]


@pytest.mark.parametrize("lg_n,rate,batches,inverse,coset", SHAPES)
def test_noalloc_matches_regular_entry_point(zk, lg_n, rate, batches, inverse, coset):
    L = zk.capi.LIB
    for call in range(2):  # two calls in a row: the shared array must not leak state between calls
        x = _rand(900 + 17 * lg_n + call, batches << lg_n)
        got = _run(zk, L.zk_lde_noalloc, x, lg_n, rate, batches, inverse, coset)
        want = _run(zk, L.zk_lde_async, x, lg_n, rate, batches, inverse, coset)
        assert np.array_equal(got, want), (lg_n, rate, batches, inverse, coset, call)


@pytest.mark.parametrize("lg_n,rate,batches,inverse", [(15, 3, 4, False), (12, 2, 3, True)])
def test_noalloc_uses_the_installed_coset_generator(zk, lg_n, rate, batches, inverse):
    """init_coset installs the generator of every coset LDE on the device; the
    allocation-free path must follow it exactly as zk_lde_async does."""
    from oracle import oracle as O

    L = zk.capi.LIB
    try:
        zk.init_coset(0, lg_n + rate, 3)
        x = _rand(4242 + lg_n, batches << lg_n)
        got = _run(zk, L.zk_lde_noalloc, x, lg_n, rate, batches, inverse, True)
        want = _run(zk, L.zk_lde_async, x, lg_n, rate, batches, inverse, True)
        assert np.array_equal(got, want)
        if not inverse:  # and it is the coset 3 * <w_N>, not 7 * <w_N>
            assert np.array_equal(got, O.batch_lde(x, lg_n, rate, batches, coset_gen=3).reshape(got.shape))
    finally:
        zk.init_coset(0, 22, 7)
    x = _rand(4343 + lg_n, batches << lg_n)
    got = _run(zk, L.zk_lde_noalloc, x, lg_n, rate, batches, inverse, True)
    assert np.array_equal(got, _run(zk, L.zk_lde_async, x, lg_n, rate, batches, inverse, True))


def test_noalloc_counts_launches_and_leaves_free_memory_unchanged(zk):
    import torch

    L = zk.capi.LIB
    x = _rand(77, 6 << 14)
    _run(zk, L.zk_lde_noalloc, x, 14, 3, 6, False, True)  # first call on the device: resolves the array
    d_in = torch.from_numpy(x).cuda()
    d_out = torch.zeros(6 << 17, dtype=torch.uint64, device="cuda")
    s = torch.cuda.current_stream().cuda_stream
    torch.cuda.synchronize()
    free0, _ = torch.cuda.mem_get_info()
    alloc0 = torch.cuda.memory_allocated()
    n0 = L.zk_kernel_launches()
    zk.capi.check(L.zk_lde_noalloc(d_out.data_ptr(), d_in.data_ptr(), 14, 3, 6, 0, 1, s))
    torch.cuda.synchronize()
    n1 = L.zk_kernel_launches()
    free1, _ = torch.cuda.mem_get_info()
    assert free1 == free0 and torch.cuda.memory_allocated() == alloc0
    assert n1 - n0 == 5  # three table fills and two transform passes


def test_noalloc_rejects_sizes_beyond_the_static_array(zk):
    import torch

    L = zk.capi.LIB
    d = torch.zeros(8, dtype=torch.uint64, device="cuda")
    r = L.zk_lde_noalloc(d.data_ptr(), d.data_ptr(), 20, 3, 1, 0, 1, torch.cuda.current_stream().cuda_stream)
    assert r.code == 2 and not r.message  # cudaErrorMemoryAllocation, no message allocated
    r = L.zk_lde_noalloc(d.data_ptr(), d.data_ptr(), 0, 3, 1, 0, 1, torch.cuda.current_stream().cuda_stream)
    assert r.code == 1 and not r.message
    assert isinstance(r, zk.capi.RustError) and ctypes.sizeof(r) == 16
