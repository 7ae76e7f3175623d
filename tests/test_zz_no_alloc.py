"""GPU test of zk_lde_noalloc, the LDE entry point that allocates nothing.

It exists for callers that cannot call cudaMalloc where they run the LDE:
work being captured into a CUDA graph (allocation is not capturable), provers
held to a pre-reserved memory budget or arena, and hot paths that forbid
allocation.  It keeps its NTT intermediate and tables in one static device
array instead.  Here its output is compared, bit for bit, with the regular
stream-ordered entry point (zk_lde_async) on two calls in a row; it also
checks the size limit (lg_n + rate_bits <= 22).

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
    zk.init_coset(0, 22, 7)  # the regular path uses the installed coset generator; make it the standard one
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


@pytest.mark.parametrize("lg_n,rate,batches,inverse,coset", [
    (15, 3, 5, False, True),   # two shared-memory passes, zero-extension skip
    (9, 2, 11, False, True),   # one pass
    (13, 3, 3, True, True),    # inverse direction, coset applied on output
    (19, 3, 2, False, False),  # the largest accepted size (2^22 points)
])
def test_noalloc_matches_regular_entry_point(zk, lg_n, rate, batches, inverse, coset):
    L = zk.capi.LIB
    for call in range(2):  # two calls in a row: the shared array must not leak state between calls
        x = _rand(900 + 17 * lg_n + call, batches << lg_n)
        got = _run(zk, L.zk_lde_noalloc, x, lg_n, rate, batches, inverse, coset)
        want = _run(zk, L.zk_lde_async, x, lg_n, rate, batches, inverse, coset)
        assert np.array_equal(got, want), (lg_n, rate, batches, inverse, coset, call)


def test_noalloc_rejects_sizes_beyond_the_static_array(zk):
    import torch

    L = zk.capi.LIB
    d = torch.zeros(8, dtype=torch.uint64, device="cuda")
    r = L.zk_lde_noalloc(d.data_ptr(), d.data_ptr(), 20, 3, 1, 0, 1, torch.cuda.current_stream().cuda_stream)
    assert r.code == 2 and not r.message  # cudaErrorMemoryAllocation, no message allocated
    r = L.zk_lde_noalloc(d.data_ptr(), d.data_ptr(), 0, 3, 1, 0, 1, torch.cuda.current_stream().cuda_stream)
    assert r.code == 1 and not r.message
    assert isinstance(r, zk.capi.RustError) and ctypes.sizeof(r) == 16
