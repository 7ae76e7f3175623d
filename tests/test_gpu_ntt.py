"""GPU parity: NTT / coset LDE / bit-reversing transpose through the C ABI,
bit-exact against the oracle (and against zeknox's own sm_100a build when
oracle/_ref/libzkref_gpu.so was built)."""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu


@pytest.fixture(scope="module")
def zk():
    import torch

    assert torch.cuda.is_available(), "GPU tests need a CUDA device"
    import zeknox_b200 as zk

    return zk


def _dev(a):
    import torch

    return torch.from_numpy(np.ascontiguousarray(a)).cuda()


def _host(t):
    import torch

    torch.cuda.synchronize()
    return t.cpu().numpy()


def _cfg(zk, batches, rate=0, in_dev=False, out_dev=False, coset=False, salt=0):
    c = zk.NTTConfig.default()
    c.batches = batches
    c.extension_rate_bits = rate
    c.are_inputs_on_device = in_dev
    c.are_outputs_on_device = out_dev
    c.with_coset = coset
    c.salt_size = salt
    return c


LDE_CASES = [(1, 1, 1), (2, 1, 3), (4, 2, 5), (6, 3, 2), (9, 1, 4), (10, 3, 3), (11, 2, 2), (12, 1, 2),
             (13, 3, 2), (15, 3, 4), (16, 3, 1), (20, 1, 1), (21, 3, 1), (22, 3, 1)]


@pytest.mark.parametrize("lg_n,rate,batches", LDE_CASES)
def test_lde_host_buffers(zk, oracle, lg_n, rate, batches):
    x = oracle.field_elems(1000 + lg_n * 10 + rate, batches << lg_n)
    out = np.zeros(batches << (lg_n + rate), dtype=np.uint64)
    zk.lde_batch(0, out.ctypes.data, x.ctypes.data, lg_n, _cfg(zk, batches, rate, coset=True))
    assert np.array_equal(out, oracle.batch_lde(x, lg_n, rate, batches))


@pytest.mark.parametrize("lg_n,rate,batches,inverse,coset", [
    (5, 2, 3, False, False), (5, 2, 3, True, True), (5, 2, 3, True, False), (12, 2, 2, True, True),
    (14, 3, 3, False, False), (14, 3, 3, True, True)])
def test_lde_device_buffers_and_directions(zk, oracle, lg_n, rate, batches, inverse, coset):
    x = oracle.field_elems(2000 + lg_n, batches << lg_n)
    d_in = _dev(x)
    d_out = _dev(np.zeros(batches << (lg_n + rate), dtype=np.uint64))
    zk.lde_batch(0, d_out.data_ptr(), d_in.data_ptr(), lg_n, _cfg(zk, batches, rate, True, True, coset),
                 zk.INVERSE if inverse else zk.FORWARD)
    exp = oracle.batch_lde(x, lg_n, rate, batches, inverse=inverse, with_coset=coset)
    assert np.array_equal(_host(d_out), exp)
    assert np.array_equal(_host(d_in), x)  # input untouched


@pytest.mark.parametrize("in_dev,out_dev,batches,pinned", [(False, False, 19, False), (False, True, 33, False),
                                                            (True, False, 16, False), (False, False, 135, False),
                                                            (False, True, 64, True), (False, False, 45, True)])
def test_lde_grouped_host_copies(zk, oracle, in_dev, out_dev, batches, pinned):
    """Host buffers with >= 16 polynomials go through the grouped copy/compute
    pipeline (4 groups, or 8 from 32 polynomials, alternating between two
    compute streams; uneven last group included; pageable or pinned host
    memory); the result is the same LDE."""
    import torch

    lg_n, rate = 9, 2
    x = oracle.field_elems(4000 + batches, batches << lg_n)
    exp = oracle.batch_lde(x, lg_n, rate, batches)
    if in_dev:
        src = _dev(x)
    elif pinned:
        src = torch.from_numpy(x).pin_memory()
    else:
        src = x
    src_ptr = src.data_ptr() if (in_dev or pinned) else src.ctypes.data
    if out_dev:
        out = _dev(np.zeros(batches << (lg_n + rate), dtype=np.uint64))
    elif pinned:
        out = torch.zeros(batches << (lg_n + rate), dtype=torch.uint64).pin_memory()
    else:
        out = np.zeros_like(exp)
    out_ptr = out.data_ptr() if (out_dev or pinned) else out.ctypes.data
    zk.lde_batch(0, out_ptr, src_ptr, lg_n, _cfg(zk, batches, rate, in_dev, out_dev, True))
    got = _host(out) if out_dev else (out.numpy() if pinned else out)
    assert np.array_equal(got, exp)


def test_lde_mixed_host_device(zk, oracle):
    lg_n, rate, b = 11, 2, 3
    x = oracle.field_elems(3, b << lg_n)
    exp = oracle.batch_lde(x, lg_n, rate, b)
    d_out = _dev(np.zeros(b << (lg_n + rate), dtype=np.uint64))
    zk.lde_batch(0, d_out.data_ptr(), x.ctypes.data, lg_n, _cfg(zk, b, rate, False, True, True))
    assert np.array_equal(_host(d_out), exp)
    out = np.zeros_like(exp)
    d_in = _dev(x)
    zk.lde_batch(0, out.ctypes.data, d_in.data_ptr(), lg_n, _cfg(zk, b, rate, True, False, True))
    assert np.array_equal(out, exp)


@pytest.mark.parametrize("b,out_dev", [(2, False), (33, False), (20, True)])
def test_lde_salt_rows(zk, oracle, b, out_dev):
    # ntt.cu:541-545: salt_size extra rows of random field elements after the LDE rows
    # (33 and 20 polynomials: salt behind the grouped copy pipeline, host or device output)
    lg_n, rate, salt = 8, 2, 3
    x = oracle.field_elems(4 + b, b << lg_n)
    N = 1 << (lg_n + rate)
    if out_dev:
        d_out = _dev(np.zeros((b + salt) * N, dtype=np.uint64))
        zk.lde_batch(0, d_out.data_ptr(), x.ctypes.data, lg_n, _cfg(zk, b, rate, out_dev=True, coset=True, salt=salt))
        out = _host(d_out)
    else:
        out = np.zeros((b + salt) * N, dtype=np.uint64)
        zk.lde_batch(0, out.ctypes.data, x.ctypes.data, lg_n, _cfg(zk, b, rate, coset=True, salt=salt))
    assert np.array_equal(out[: b * N], oracle.batch_lde(x, lg_n, rate, b))
    s = out[b * N:]
    assert (s < np.uint64(oracle.P)).all() and len(np.unique(s)) > 0.99 * s.size


def test_lde_invalid_args(zk):
    with pytest.raises(zk.ZeknoxError) as e:
        zk.lde_batch(0, 0, 0, 0, _cfg(zk, 1, 1))
    assert e.value.code == 1
    with pytest.raises(zk.ZeknoxError):
        zk.lde_batch(0, 0, 0, 4, _cfg(zk, 1, 0))


NTT_CASES = [1, 2, 5, 11, 12, 13, 17, 18, 23]


@pytest.mark.parametrize("lg", NTT_CASES)
@pytest.mark.parametrize("coset", [False, True])
def test_batch_ntt_forward_inverse(zk, oracle, lg, coset):
    batches = 3 if lg <= 18 else 1
    x = oracle.field_elems(500 + lg, batches << lg)
    a = x.copy()
    zk.ntt_batch(0, a.ctypes.data, lg, _cfg(zk, batches, coset=coset))
    assert np.array_equal(a, oracle.batch_ntt(x, lg, False, batches, coset))
    d = _dev(x)
    zk.intt_batch(0, d.data_ptr(), lg, _cfg(zk, batches, in_dev=True, out_dev=True, coset=coset))
    assert np.array_equal(_host(d), oracle.batch_ntt(x, lg, True, batches, coset))


def test_ntt_three_pass_vs_oracle(zk, oracle):
    lg = 25  # three shared-memory passes
    x = oracle.field_elems(25, 1 << lg)
    d = _dev(x)
    zk.ntt_batch(0, d.data_ptr(), lg, _cfg(zk, 1, in_dev=True, out_dev=True, coset=True))
    assert np.array_equal(_host(d), oracle.batch_ntt(x, lg, False, 1, True))


def test_ntt_roundtrip_large(zk, oracle):
    # size-independent property at 2^26: iNTT(NTT(x)) == x
    lg, b = 26, 1
    x = oracle.field_elems(77, b << lg)
    d = _dev(x)
    zk.ntt_batch(0, d.data_ptr(), lg, _cfg(zk, b, in_dev=True, out_dev=True))
    zk.intt_batch(0, d.data_ptr(), lg, _cfg(zk, b, in_dev=True, out_dev=True))
    assert np.array_equal(_host(d), x)


def test_init_coset_other_generator(zk, oracle):
    lg = 10
    zk.init_coset(0, lg, 11)
    try:
        x = oracle.field_elems(8, 2 << lg)
        a = x.copy()
        zk.ntt_batch(0, a.ctypes.data, lg, _cfg(zk, 2, coset=True))
        assert np.array_equal(a, oracle.batch_ntt(x, lg, False, 2, True, 11))
    finally:
        zk.init_coset(0, 20, 7)


@pytest.mark.parametrize("lg,batches", [(0, 1), (1, 3), (5, 7), (10, 135), (13, 16), (18, 135), (6, 1000), (4, 200),
                                        (7, 193), (7, 1), (8, 2), (9, 385), (11, 64)])
def test_transpose_rev(zk, oracle, lg, batches):
    x = oracle.field_elems(9 + lg, batches << lg)
    out = np.zeros_like(x)
    c = zk.TransposeConfig.default()
    c.batches = batches
    zk.transpose_rev_batch(0, out.ctypes.data, x.ctypes.data, lg, c)
    assert np.array_equal(out, oracle.transpose_rev(x, lg, batches))
    d_in, d_out = _dev(x), _dev(np.zeros_like(x))
    c.are_inputs_on_device = c.are_outputs_on_device = True
    zk.transpose_rev_batch(0, d_out.data_ptr(), d_in.data_ptr(), lg, c)
    assert np.array_equal(_host(d_out), out)


@pytest.mark.parametrize("lg,batches", [(12, 135), (7, 3)])
def test_transpose_rev_input_only_8_byte_aligned(zk, oracle, lg, batches):
    """A device input 8 bytes past a 16-byte boundary takes the 8-byte-load
    form of the transpose; the output must not change."""
    x = oracle.field_elems(31 + lg, batches << lg)
    c = zk.TransposeConfig.default()
    c.batches = batches
    c.are_inputs_on_device = c.are_outputs_on_device = True
    d_in = _dev(np.concatenate([np.zeros(1, dtype=np.uint64), x]))
    assert (d_in.data_ptr() + 8) % 16 == 8
    d_out = _dev(np.zeros_like(x))
    zk.transpose_rev_batch(0, d_out.data_ptr(), d_in.data_ptr() + 8, lg, c)
    assert np.array_equal(_host(d_out), oracle.transpose_rev(x, lg, batches))


def test_lde_multi_gpu_entry(zk, oracle):
    lg_n, rate, b = 10, 2, 5
    x = oracle.field_elems(12, b << lg_n)
    d_out = _dev(np.zeros(b << (lg_n + rate), dtype=np.uint64))
    zk.lde_batch_multi_gpu(d_out.data_ptr(), x.ctypes.data, 1, _cfg(zk, b, rate, coset=True), lg_n, x.size,
                           b << (lg_n + rate))
    assert np.array_equal(_host(d_out), oracle.batch_lde(x, lg_n, rate, b))


# ---------------------------------------------- zeknox's own sm_100a build
def _ref_gpu():
    from oracle.oracle import HERE

    so = HERE / "_ref" / "libzkref_gpu.so"
    if not so.exists():
        pytest.skip("zeknox sm_100a build not present (oracle/build_ref.sh)")
    from zeknox_b200.capi import NTTConfig, RustError, TransposeConfig

    L = ctypes.CDLL(str(so))
    vp, sz, u32, u64 = ctypes.c_void_p, ctypes.c_size_t, ctypes.c_uint32, ctypes.c_uint64
    L.init_twiddle_factors.argtypes = [sz, sz]
    L.init_twiddle_factors.restype = RustError
    L.init_coset.argtypes = [sz, sz, u64]
    L.init_coset.restype = RustError
    L.compute_batched_lde.argtypes = [sz, vp, vp, u32, ctypes.c_int, NTTConfig]
    L.compute_batched_lde.restype = RustError
    L.compute_batched_ntt.argtypes = [sz, vp, u32, ctypes.c_int, NTTConfig]
    L.compute_batched_ntt.restype = RustError
    L.compute_transpose_rev.argtypes = [sz, vp, vp, u32, TransposeConfig]
    L.compute_transpose_rev.restype = RustError
    L.fill_digests_buf_linear_gpu_with_gpu_ptr.argtypes = [vp, vp, vp, u64, u64, u64, u64, u64, u64, u64]
    L.fill_digests_buf_linear_gpu_with_gpu_ptr.restype = None
    return L


@pytest.mark.parametrize("lg_n,rate,batches", [(4, 1, 2), (12, 3, 5), (15, 3, 8)])
def test_lde_vs_zeknox_sm100_build(zk, oracle, lg_n, rate, batches):
    R = _ref_gpu()
    lg = lg_n + rate
    assert R.init_twiddle_factors(0, lg).code == 0
    assert R.init_coset(0, lg, 7).code == 0
    x = oracle.field_elems(42 + lg, batches << lg_n)
    ref_out = np.zeros(batches << lg, dtype=np.uint64)
    c = _cfg(zk, batches, rate, coset=True)
    assert R.compute_batched_lde(0, ref_out.ctypes.data, x.ctypes.data, lg_n, 0, c).code == 0
    out = np.zeros_like(ref_out)
    zk.lde_batch(0, out.ctypes.data, x.ctypes.data, lg_n, c)
    assert np.array_equal(out, ref_out)


def test_transpose_vs_zeknox_sm100_build(zk, oracle):
    R = _ref_gpu()
    lg, b = 14, 135
    x = oracle.field_elems(5, b << lg)
    c = zk.TransposeConfig.default()
    c.batches = b
    ref_out, out = np.zeros_like(x), np.zeros_like(x)
    assert R.compute_transpose_rev(0, ref_out.ctypes.data, x.ctypes.data, lg, c).code == 0
    zk.transpose_rev_batch(0, out.ctypes.data, x.ctypes.data, lg, c)
    assert np.array_equal(out, ref_out)


def test_empty_inputs_are_no_ops(zk):
    """Zero polynomials (and zero jobs / queries for the extensions) are valid
    calls that do nothing: null buffers are accepted, nothing is launched."""
    import torch

    before = zk.capi.LIB.zk_kernel_launches()
    cfg = _cfg(zk, 0, 0)
    zk.ntt_batch(0, 0, 10, cfg)
    zk.intt_batch(0, 0, 10, cfg)
    zk.lde_batch(0, 0, 0, 10, _cfg(zk, 0, 2, coset=True))
    zk.lde_batch(0, 0, 0, 10, _cfg(zk, 0, 2, in_dev=True, out_dev=True, coset=True))
    tcfg = zk.TransposeConfig.default()
    tcfg.batches, tcfg.are_inputs_on_device, tcfg.are_outputs_on_device = 0, True, True
    zk.transpose_rev_batch(0, 0, 0, 10, tcfg)
    zk.capi.check(zk.capi.LIB.zk_commit_batch(None, 0, 4, None))
    leaves = torch.zeros((16, 4), dtype=torch.uint64, device="cuda")
    digests, _ = zk.merkle_tree(leaves, 2, 0)
    rows, sib = zk.merkle_open(leaves, digests, 2, torch.zeros(0, dtype=torch.int64))
    torch.cuda.synchronize()
    assert rows.shape == (0, 4) and sib.shape[0] == 0
    # only the tree above launched kernels
    assert zk.capi.LIB.zk_kernel_launches() - before <= 8
