"""GPU parity: the FRI commit phase over the resident commitment (folding over
GF(p^2), the shifted-coset LDE written as leaves, the per-round Merkle trees,
query openings), bit-exact against the oracle on small cases and, at larger
sizes, through the FRI verifier's own relations (every opened leaf row folds
to the next round's value at that position, the last round folds to the final
polynomial, every opening path hashes up to its round's cap)."""

import numpy as np
import pytest

pytestmark = pytest.mark.gpu

P = 0xFFFFFFFF00000001


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


def _challenge(i, cap):
    # A deterministic stand-in for the transcript: two words of the cap.
    cap = np.asarray(cap).reshape(-1)
    return (int(cap[0]) % P, int(cap[(i + 5) % cap.size]) % P)


@pytest.mark.parametrize("lg_n,arity_bits", [(1, 1), (4, 4), (6, 6), (10, 1), (10, 3), (16, 4), (17, 5), (20, 4)])
def test_fold_matches_oracle(zk, oracle, lg_n, arity_bits):
    n = 1 << lg_n
    c = oracle.field_elems(9000 + lg_n * 7 + arity_bits, 2 * n).reshape(2, n)
    for beta in [(0, 0), (1, 0), (0, 1), (P - 1, P - 1), (0x1234567890ABCDEF, 0x0FEDCBA987654321)]:
        want = oracle.fri_fold(c, arity_bits, beta)
        got = _host(zk.fri_fold(_dev(c), arity_bits, beta))
        assert np.array_equal(got, want), (lg_n, arity_bits, beta)


@pytest.mark.parametrize("lg_n,arity_bits", [(3, 3), (12, 2), (15, 4)])
def test_fold_interleaved_input(zk, oracle, lg_n, arity_bits):
    n = 1 << lg_n
    c = oracle.field_elems(9100 + lg_n, 2 * n).reshape(2, n)
    beta = (31337, 271828)
    want = oracle.fri_fold(c, arity_bits, beta)
    got = _host(zk.fri_fold(_dev(np.ascontiguousarray(c.T)), arity_bits, beta, interleaved=True))
    assert np.array_equal(got, want)


def test_fold_rejects_bad_arguments(zk, oracle):
    import torch

    c = _dev(oracle.field_elems(1, 2 * 64).reshape(2, 64))
    for ab, beta in [(0, (1, 0)), (7, (1, 0)), (2, (P, 0)), (2, (0, P + 5))]:
        out = torch.empty((2, 64), dtype=torch.uint64, device="cuda")
        err = zk.capi.LIB.zk_fri_fold_async(out.data_ptr(), c.data_ptr(), 64, ab, beta[0], beta[1], 0, None)
        assert err.code != 0, (ab, beta)
    out = torch.empty((2, 8), dtype=torch.uint64, device="cuda")
    assert zk.capi.LIB.zk_fri_fold_async(out.data_ptr(), c.data_ptr(), 48, 2, 1, 0, 0, None).code != 0
    assert zk.capi.LIB.zk_fri_fold_async(out.data_ptr(), c.data_ptr(), 2, 2, 1, 0, 0, None).code != 0


@pytest.mark.parametrize("b,lg_n,rate,shift", [(2, 9, 3, 7 ** 16), (2, 12, 1, 0x123456789), (5, 10, 2, 7 ** 256),
                                               (1, 13, 3, P - 2), (2, 15, 3, 7 ** 4096)])
def test_lde_leaves_on_a_shifted_coset(zk, oracle, b, lg_n, rate, shift):
    shift %= P
    c = oracle.field_elems(9200 + lg_n + b, b << lg_n)
    want = oracle.transpose_rev(oracle.batch_lde(c, lg_n, rate, b, coset_gen=shift), lg_n + rate, b)
    got = _host(zk.lde_leaves_coset(_dev(c.reshape(b, -1)), rate, shift))
    assert np.array_equal(got.reshape(-1), want)


@pytest.mark.parametrize("lg_n,rate,arities,cap_h,ht", [(10, 3, [4, 3, 2], 2, 0), (8, 1, [1, 1, 1, 1], 0, 0),
                                                        (9, 2, [3, 3], 1, 3), (11, 3, [4, 4], 3, 1)])
def test_fri_commit_matches_oracle(zk, oracle, lg_n, rate, arities, cap_h, ht):
    n = 1 << lg_n
    c = oracle.field_elems(9300 + lg_n, 2 * n).reshape(2, n)
    rounds, final = oracle.fri_commit(c, rate, arities, cap_h, _challenge, ht)
    com = zk.fri_commit(_dev(c), rate, arities, cap_h, _challenge, ht)
    assert len(com.rounds) == len(rounds)
    for i, (g, w) in enumerate(zip(com.rounds, rounds)):
        assert g.shift == w["shift"] and g.beta == w["beta"], i
        assert np.array_equal(_host(g.leaves), w["leaves"]), i
        assert np.array_equal(_host(g.digests).reshape(-1)[:w["digests"].size], w["digests"]), i
        assert np.array_equal(_host(g.cap).reshape(-1), w["cap"]), i
    assert np.array_equal(_host(com.final_poly), final)


def _check_rounds(oracle, com, rate_bits, rows_per_round, positions):
    """The FRI verifier's fold relation on the given leaf positions of every round."""
    for i, rnd in enumerate(com.rounds):
        leaves = rows_per_round[i]
        n_rows, width = leaves.shape
        lg_N = (n_rows * width // 2).bit_length() - 1
        for j in positions(n_rows):
            y, v = oracle.fri_fold_from_leaf(leaves[j], j, lg_N, rnd.shift, rnd.arity_bits, rnd.beta)
            if i + 1 < len(com.rounds):
                nxt = rows_per_round[i + 1].reshape(-1, 2)[j]
                assert v == (int(nxt[0]), int(nxt[1])), (i, j)
            else:
                assert v == oracle.ext_poly_eval(_host(com.final_poly), y), (i, j)


def test_fri_commit_large_folds_consistently(zk, oracle):
    """135-column-commit scale: 2^15 GF(p^2) coefficients, rate 3 (2^18 points),
    arity 16 three times, cap height 4; the final polynomial has 8 coefficients."""
    lg_n, rate, arities, cap_h = 15, 3, [4, 4, 4], 4
    n = 1 << lg_n
    c = oracle.field_elems(9400, 2 * n).reshape(2, n)
    com = zk.fri_commit(_dev(c), rate, arities, cap_h, _challenge)
    assert tuple(com.final_poly.shape) == (2, n >> 12)
    rows = [_host(r.leaves) for r in com.rounds]
    rng = np.random.default_rng(4)
    _check_rounds(oracle, com, rate, rows,
                  lambda m: sorted(set([0, m - 1] + rng.integers(0, m, size=12).tolist())))
    # Round 0's leaves are the LDE of the input on the 7-coset; the caps of the
    # two smaller rounds are recomputed by the oracle from the GPU's leaves.
    want0 = oracle.transpose_rev(oracle.batch_lde(c.reshape(-1), lg_n, rate, 2), lg_n + rate, 2)
    assert np.array_equal(rows[0].reshape(-1), want0)
    for r, lv in zip(com.rounds[1:], rows[1:]):
        _, cap = oracle.merkle_fill(lv.reshape(-1), lv.shape[1], cap_h, 0)
        assert np.array_equal(_host(r.cap).reshape(-1), cap)


def test_fri_open_paths_verify(zk, oracle):
    import torch

    lg_n, rate, arities, cap_h = 12, 3, [3, 2, 2], 2
    n = 1 << lg_n
    c = oracle.field_elems(9500, 2 * n).reshape(2, n)
    com = zk.fri_commit(_dev(c), rate, arities, cap_h, _challenge)
    q = np.random.default_rng(5).integers(0, n << rate, size=24)
    opened = zk.fri_open(com, torch.from_numpy(q))
    torch.cuda.synchronize()
    shift = 0
    for rnd, (rows, sib) in zip(com.rounds, opened):
        shift += rnd.arity_bits
        rows, sib, cap = rows.cpu().numpy(), sib.cpu().numpy(), rnd.cap.cpu().numpy()
        leaves = _host(rnd.leaves)
        nl = leaves.shape[0]
        for k, x in enumerate(q):
            i = int(x) >> shift
            assert np.array_equal(rows[k], leaves[i])
            cur = oracle.hash_one(0, rows[k])
            for lvl, s in enumerate(sib[k]):
                cur = oracle.hash_two(0, cur, s) if ((i >> lvl) & 1) == 0 else oracle.hash_two(0, s, cur)
            depth = (nl >> cap_h).bit_length() - 1
            assert np.array_equal(cur, cap[i >> depth]), (shift, i)
