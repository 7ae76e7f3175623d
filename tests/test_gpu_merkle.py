"""GPU parity: Merkle digests and caps (Poseidon, Poseidon2, Keccak) through
the C ABI, bit-exact against zeknox's known answers, its CPU path's outputs
(tests/golden/) and the oracle; large trees through size-independent checks."""

import ctypes

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

HASHES = {"poseidon": 0, "poseidon2": 3, "keccak": 1, "monolith": 4, "poseidonbn128": 2}


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


def gpu_tree(zk, leaves, leaf_size, cap_height, ht, digests_init=None, cap_init=None):
    """fill_digests_buf_linear_gpu_with_gpu_ptr on device copies of the buffers."""
    nl = leaves.size // leaf_size
    nd, nc = 2 * (nl - (1 << cap_height)), 1 << cap_height
    d_leaves = _dev(leaves)
    d_dig = _dev(np.zeros(max(nd, 1) * 4, dtype=np.uint64) if digests_init is None else digests_init)
    d_cap = _dev(np.zeros(nc * 4, dtype=np.uint64) if cap_init is None else cap_init)
    zk.fill_digests_buf_linear_gpu_with_gpu_ptr(d_dig.data_ptr(), d_cap.data_ptr(), d_leaves.data_ptr(), nd, nc,
                                                nl, leaf_size, cap_height, ht, 0)
    return _host(d_dig), _host(d_cap)


def test_hash_one_kats(zk, golden):
    # one leaf, cap_height 0 -> cap[0] = H(leaf) (merkle.cu:178-181)
    k = golden["kat"]["poseidon_hash_one"]
    leaf = np.array(k["leaf"], dtype=np.uint64)
    for size, exp in k["expected"].items():
        _, cap = gpu_tree(zk, leaf[: int(size)].copy(), int(size), 0, 0)
        assert cap.tolist() == exp, size
    fib = [0, 1]
    for _ in range(10):
        fib.append(fib[-1] + fib[-2])
    _, cap = gpu_tree(zk, np.array(fib, dtype=np.uint64), 12, 0, 3)
    assert cap.tolist() == golden["kat"]["poseidon2_hash_one_fib12"]["expected"]
    kk = golden["kat"]["keccak_hash_one"]
    data = np.array(kk["data"], dtype=np.uint64)
    for size in range(1, 7):
        _, cap = gpu_tree(zk, data[:size].copy(), size, 0, 1)
        assert cap.tolist() == kk["expected"][str(size)], size
    mk = golden["kat"]["monolith_hash_one"]
    _, cap = gpu_tree(zk, np.array(mk["input"], dtype=np.uint64), 12, 0, 4)
    assert cap.tolist() == mk["expected"]
    bk = golden["kat"]["poseidon_bn128_hash_one"]
    _, cap = gpu_tree(zk, np.array(bk["input"], dtype=np.uint64), 12, 0, 2)
    assert cap.tolist() == bk["expected"]


def test_go_merkle_caps(zk, golden):
    k = golden["kat"]["go_merkle_caps"]
    leaf = np.array(k["leaf"], dtype=np.uint64)
    for case in k["cases"]:
        nl, nc = case["n_leaves"], case["n_caps"]
        _, cap = gpu_tree(zk, np.tile(leaf, nl), leaf.size, nc.bit_length() - 1, 0)
        for j in range(nc):
            assert cap[4 * j:4 * j + 4].tolist() == case["cap"]


def _fixture_shapes(golden):
    for key in sorted(k[:-len("_seed")] for k in golden["merkle"] if k.endswith("_seed")):
        name, shape, ch = key.split("_")
        nl, ls = map(int, shape.split("x"))
        yield key, HASHES[name], nl, ls, int(ch[1:])


def test_vs_reference_cpu_fixtures(zk, oracle, golden):
    for key, ht, nl, ls, ch in _fixture_shapes(golden):
        leaves = oracle.field_elems(int(golden["merkle"][key + "_seed"][0]), nl * ls)
        d, c = gpu_tree(zk, leaves, ls, ch, ht)
        assert np.array_equal(c, golden["merkle"][key + "_cap"]), key
        if (nl >> ch) > 1 and nl != (1 << ch):
            assert np.array_equal(d, golden["merkle"][key + "_digests"]), key


@pytest.mark.parametrize("ht", [0, 3, 1, 4, 2])
@pytest.mark.parametrize("nl,ls,ch", [(4096, 135, 4), (2048, 8, 0), (1024, 17, 10), (8192, 5, 3), (64, 200, 5),
                                     (1 << 16, 24, 0), (1 << 16, 9, 6), (1 << 15, 12, 12), (1 << 14, 135, 4),
                                     (1 << 14, 3, 2), (1 << 14, 13, 14),
                                     # wrappers/rust/tests/merkle_tree.rs:161-223 (4096 x 7, cap 1); the
                                     # hand-built 4-leaf trees of native/tests/tests.cu:338-375; short
                                     # leaves (no permutation) on the small-tree kernels; cap == leaves
                                     (4096, 7, 1), (4, 7, 0), (4, 7, 1), (2, 9, 0), (8192, 4, 2),
                                     (8192, 1, 0), (1 << 13, 135, 13),
                                     # one thread per leaf with 128 leaves per subtree, and short leaves
                                     (1 << 15, 9, 8), (1 << 15, 4, 6)])
def test_vs_oracle(zk, oracle, ht, nl, ls, ch):
    leaves = oracle.field_elems(ht * 1000 + nl + ls, nl * ls)
    d, c = gpu_tree(zk, leaves, ls, ch, ht)
    d2, c2 = oracle.merkle_fill(leaves, ls, ch, ht)
    assert np.array_equal(c, c2) and np.array_equal(d, d2)


def test_cpu_entry_point(zk, oracle):
    """fill_digests_buf_linear_cpu: host buffers, same tree."""
    nl, ls, ch = 1024, 135, 4
    leaves = oracle.field_elems(99, nl * ls)
    nd, nc = 2 * (nl - 16), 16
    d = np.zeros(nd * 4, dtype=np.uint64)
    c = np.zeros(nc * 4, dtype=np.uint64)
    zk.fill_digests_buf_linear_cpu(d.ctypes.data, c.ctypes.data, leaves.ctypes.data, nd, nc, nl, ls, ch, 0)
    d2, c2 = oracle.merkle_fill(leaves, ls, ch, 0)
    assert np.array_equal(c, c2) and np.array_equal(d, d2)


def test_multigpu_entry_point(zk, oracle):
    nl, ls, ch = 512, 20, 2
    leaves = oracle.field_elems(98, nl * ls)
    nd, nc = 2 * (nl - 4), 4
    dl, dd, dc = _dev(leaves), _dev(np.zeros(nd * 4, dtype=np.uint64)), _dev(np.zeros(nc * 4, dtype=np.uint64))
    zk.fill_digests_buf_linear_multigpu_with_gpu_ptr(dd.data_ptr(), dc.data_ptr(), dl.data_ptr(), nd, nc, nl, ls,
                                                     ch, 3)
    d2, c2 = oracle.merkle_fill(leaves, ls, ch, 3)
    assert np.array_equal(_host(dc), c2) and np.array_equal(_host(dd), d2)


def test_keccak_short_leaves_keep_untouched_words(zk, oracle):
    # keccak.cu:118-121: fewer than 4 words are copied, the rest of the digest is left as it was
    nl, ls, ch = 8, 2, 3  # cap == leaves
    leaves = oracle.field_elems(5, nl * ls)
    init = np.full(nl * 4, 0xABCDEF, dtype=np.uint64)
    _, cap = gpu_tree(zk, leaves, ls, ch, 1, cap_init=init.copy())
    exp = init.copy()
    oracle.merkle_fill(leaves, ls, ch, 1, cap=exp)
    assert np.array_equal(cap, exp)


def test_invalid_sizes_and_unsupported_hash(zk, oracle):
    leaves = oracle.field_elems(6, 64 * 9)
    dl = _dev(leaves)
    dd, dc = _dev(np.zeros(120 * 4, dtype=np.uint64)), _dev(np.full(4 * 4, 7, dtype=np.uint64))
    with pytest.raises(zk.ZeknoxError):  # digests size inconsistent with leaves / cap
        zk.fill_digests_buf_linear_gpu_with_gpu_ptr(dd.data_ptr(), dc.data_ptr(), dl.data_ptr(), 100, 4, 64, 9, 2, 0)
    for ht in (5, 6):  # no such hasher: nothing written
        with pytest.raises(zk.ZeknoxError):
            zk.fill_digests_buf_linear_gpu_with_gpu_ptr(dd.data_ptr(), dc.data_ptr(), dl.data_ptr(), 120, 4, 64, 9, 2,
                                                        ht)
    assert (_host(dc) == 7).all()


@pytest.mark.parametrize("ht", [0, 3, 1, 4, 2])
def test_full_size_tree_properties(zk, oracle, ht):
    """2^20 leaves x 135 (the hash-sweep shape): every cap entry, 4096 random
    internal nodes and 512 random leaf digests re-derived with the oracle."""
    import torch

    nl, ls, ch = 1 << 20, 135, 4
    g = torch.Generator(device="cuda").manual_seed(1234 + ht)
    # values below 2^62 < p are canonical field elements
    raw = torch.randint(0, 2**62, (nl, ls), generator=g, device="cuda", dtype=torch.int64)
    leaves_t = raw.view(torch.uint64)
    digests, cap = zk.merkle_tree(leaves_t, ch, ht)
    torch.cuda.synchronize()
    d = digests.cpu().numpy().reshape(-1, 4)
    c = cap.cpu().numpy().reshape(-1, 4)
    ls_sub, ds = nl >> ch, 2 * (nl >> ch) - 2
    rng = np.random.default_rng(ht)
    for s in range(1 << ch):
        assert np.array_equal(c[s], oracle.hash_two(ht, d[s * ds], d[s * ds + 1]))
    for _ in range(4096):
        s, i = rng.integers(1 << ch), rng.integers(ds - ls_sub)
        b = s * ds
        assert np.array_equal(d[b + i], oracle.hash_two(ht, d[b + 2 * i + 2], d[b + 2 * i + 3]))
    leaf_rows = rng.integers(nl, size=512)
    host_leaves = raw[torch.from_numpy(leaf_rows).cuda()].cpu().numpy().view(np.uint64)
    for row, li in zip(host_leaves, leaf_rows):
        s, j = divmod(int(li), ls_sub)
        assert np.array_equal(d[s * ds + ds - ls_sub + j], oracle.hash_one(ht, row))


# ---------------------------------------------- zeknox's own sm_100a build
@pytest.mark.parametrize("ht", [0, 3, 1, 4, 2])
def test_vs_zeknox_sm100_build(zk, oracle, ht):
    from oracle.oracle import HERE

    so = HERE / "_ref" / "libzkref_gpu.so"
    if not so.exists():
        pytest.skip("zeknox sm_100a build not present (oracle/build_ref.sh)")
    R = ctypes.CDLL(str(so))
    vp, u64 = ctypes.c_void_p, ctypes.c_uint64
    R.fill_digests_buf_linear_gpu_with_gpu_ptr.argtypes = [vp, vp, vp, u64, u64, u64, u64, u64, u64, u64]
    R.fill_digests_buf_linear_gpu_with_gpu_ptr.restype = None
    nl, ls, ch = 8192, 135, 4
    leaves = oracle.field_elems(77 + ht, nl * ls)
    nd, nc = 2 * (nl - 16), 16
    dl, dd, dc = _dev(leaves), _dev(np.zeros(nd * 4, dtype=np.uint64)), _dev(np.zeros(nc * 4, dtype=np.uint64))
    import torch

    torch.cuda.synchronize()
    R.fill_digests_buf_linear_gpu_with_gpu_ptr(dd.data_ptr(), dc.data_ptr(), dl.data_ptr(), nd, nc, nl, ls, ch, ht, 0)
    ref_d, ref_c = _host(dd), _host(dc)
    d, c = gpu_tree(zk, leaves, ls, ch, ht)
    assert np.array_equal(c, ref_c) and np.array_equal(d, ref_d)


# ------------------------------------------------- opening proofs (resident tree)
def _verify_path(oracle, ht, row, sib, index, cap, cap_height, n_leaves):
    """Plonky2's MerkleProof check: hash the leaf, fold the siblings bottom-up
    (the running digest is the left input when its index bit is 0), compare
    with the cap entry the path ends at."""
    cur = oracle.hash_one(ht, row)
    for lvl, s in enumerate(sib):
        cur = oracle.hash_two(ht, cur, s) if ((index >> lvl) & 1) == 0 else oracle.hash_two(ht, s, cur)
    depth = (n_leaves >> cap_height).bit_length() - 1
    return np.array_equal(cur, cap[index >> depth])


@pytest.mark.parametrize("ht,nl,ls,ch", [(0, 1 << 12, 135, 4), (3, 1 << 11, 24, 0), (1, 1 << 10, 7, 3),
                                         (4, 1 << 9, 16, 2), (2, 256, 9, 1), (0, 64, 12, 6)])
def test_opening_paths_verify_against_cap(zk, oracle, ht, nl, ls, ch):
    import torch

    leaves = oracle.field_elems(500 + ht * 13 + nl, nl * ls)
    lt = _dev(leaves).view(nl, ls)
    digests, cap = zk.merkle_tree(lt, ch, ht)
    rng = np.random.default_rng(ht + nl)
    q = rng.integers(0, nl, size=64)
    rows, sib = zk.merkle_open(lt, digests, ch, torch.from_numpy(q))
    torch.cuda.synchronize()
    rows, sib, capn = rows.cpu().numpy(), sib.cpu().numpy(), cap.cpu().numpy()
    depth = (nl >> ch).bit_length() - 1
    assert sib.shape == (64, depth, 4)
    for k, i in enumerate(q):
        assert np.array_equal(rows[k], leaves[i * ls:(i + 1) * ls])
        assert _verify_path(oracle, ht, rows[k], sib[k], int(i), capn, ch, nl), (ht, int(i))


def test_opening_out_of_range_index(zk, oracle):
    import torch

    nl, ls, ch = 128, 9, 2
    leaves = oracle.field_elems(77, nl * ls)
    lt = _dev(leaves).view(nl, ls)
    digests, _ = zk.merkle_tree(lt, ch, 0)
    rows, sib = zk.merkle_open(lt, digests, ch, torch.tensor([5, nl, 127]))
    torch.cuda.synchronize()
    rows, sib = rows.cpu().numpy(), sib.cpu().numpy()
    assert (rows[1] == np.uint64(2**64 - 1)).all() and (sib[1] == np.uint64(2**64 - 1)).all()
    assert np.array_equal(rows[0], leaves[5 * ls:6 * ls]) and np.array_equal(rows[2], leaves[127 * ls:128 * ls])


# ---------------------------------------- Monolith: Bars need canonical inputs
def _monolith_mds_row():
    import re
    from pathlib import Path

    h = (Path(__file__).resolve().parents[1] / "zeknox_b200" / "csrc" / "zk_constants.h").read_text()
    m = re.search(r"#define ZK_MONOLITH_MDS_ROW_LIST \\\n(.*?)\nZK_CONST_TABLE", h, re.S)
    return [int(x, 16) for x in re.findall(r"0x[0-9a-f]+", m.group(1))]


def _leaves_with_small_bar_inputs(oracle, count, seed):
    """8-word leaves (one Monolith permutation each) whose first concrete
    layer (round constants zero) outputs values below 2^32 - 1 on lanes 0-3,
    the lanes that go through the Bars next.  Such a value also has the 64-bit
    form v + p, and Bars (a byte-wise map, not a field operation) give another
    result on that form: the input must be canonical.  Solved as
    M[0..3][0..3] x[0..3] = v - M[0..3][4..7] x[4..7] (mod p)."""
    P = oracle.P
    row = _monolith_mds_row()
    M = [[row[(c - r) % 12] for c in range(12)] for r in range(12)]
    rng = np.random.default_rng(seed)
    A = [[M[r][c] for c in range(4)] for r in range(4)]

    def solve(b):  # Gaussian elimination mod p on the 4 x 4 system
        m = [A[r][:] + [b[r]] for r in range(4)]
        for col in range(4):
            piv = next(r for r in range(col, 4) if m[r][col] % P)
            m[col], m[piv] = m[piv], m[col]
            inv = pow(m[col][col], P - 2, P)
            m[col] = [v * inv % P for v in m[col]]
            for r in range(4):
                if r != col and m[r][col]:
                    f = m[r][col]
                    m[r] = [(a - f * b2) % P for a, b2 in zip(m[r], m[col])]
        return [m[r][4] for r in range(4)]

    rows = []
    for _ in range(count):
        tail = [int(v) for v in rng.integers(0, P, size=4, dtype=np.uint64)]
        small = [int(v) for v in rng.integers(0, 2**32 - 1, size=4)]
        rhs = [(small[r] - sum(M[r][4 + k] * tail[k] for k in range(4))) % P for r in range(4)]
        rows.append(solve(rhs) + tail)
    return np.array(rows, dtype=np.uint64).reshape(-1)


def test_monolith_bars_on_small_values_match_the_cpu_path(zk, oracle):
    """Regression for a case where zeknox's own GPU build and its CPU path
    disagree: a concrete-layer output below 2^32 - 1 that reaches the Bars.
    This library follows the CPU path (and zeknox's known answer): leaf digests
    equal the oracle's and, when built, zeknox's CPU hash."""
    nl, ls = 64, 8
    leaves = _leaves_with_small_bar_inputs(oracle, nl, 0x5EED)
    d, c = gpu_tree(zk, leaves, ls, 6, 4)  # cap height 6: the cap is the 64 leaf hashes
    R = oracle.ref()
    for i in range(nl):
        row = leaves[i * ls:(i + 1) * ls]
        want = oracle.hash_one(4, row)
        assert np.array_equal(c.reshape(-1, 4)[i], want), i
        if R is not None:
            ref = np.zeros(4, dtype=np.uint64)
            R.zkref_hash_one(4, row.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)), ls,
                             ref.ctypes.data_as(ctypes.POINTER(ctypes.c_uint64)))
            assert np.array_equal(ref, want), i
