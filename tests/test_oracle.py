"""CPU tests: the oracle (oracle/oracle.c) pinned against zeknox's own
known-answer vectors and its CPU Merkle outputs (tests/golden/), plus
independent restatements of the NTT / LDE / transpose semantics at small sizes.
"""

import numpy as np
import pytest

P = 0xFFFFFFFF00000001
HASHES = {"poseidon": 0, "poseidon2": 3, "keccak": 1, "monolith": 4, "poseidonbn128": 2}


def test_constants_are_canonical(oracle):
    import re
    from pathlib import Path

    hdr = (Path(__file__).resolve().parents[1] / "zeknox_b200/csrc/zk_constants.h").read_text()
    for name in ("ZK_POSEIDON_RC", "ZK_POSEIDON2_RC", "ZK_POSEIDON2_DIAG"):
        body = hdr.split(f"#define {name}_LIST")[1].split("ZK_CONST_TABLE")[0]
        vals = [int(v, 16) for v in re.findall(r"0x([0-9a-f]+)ull", body)]
        assert len(vals) in (12, 360) and all(v < P for v in vals)


def test_field_params(oracle):
    # native/ff/gl64_params.hpp:12-87 spot values: OMEGA[1] = p-1, OMEGA[6] = 2^39,
    # OMEGA[32], OMEGA_INV[2], DOMAIN_SIZE_INV[1].
    L = oracle.lib()
    assert L.orc_omega(1) == P - 1
    assert L.orc_omega(6) == 1 << 39
    assert L.orc_omega(32) == 0x185629DCDA58878C
    assert L.orc_omega_inv(2) == 0xFFFEFFFF00000001
    assert L.orc_domain_size_inv(1) == 0x7FFFFFFF80000001
    for lg in (1, 5, 18, 32):
        w = L.orc_omega(lg)
        assert pow(w, 1 << lg, P) == 1 and pow(w, 1 << (lg - 1), P) == P - 1


def test_poseidon_kat(oracle, golden):
    k = golden["kat"]["poseidon_hash_one"]
    leaf = np.array(k["leaf"], dtype=np.uint64)
    for size, exp in k["expected"].items():
        assert oracle.hash_one(0, leaf[: int(size)]).tolist() == exp, size


def test_poseidon2_kat(oracle, golden):
    fib = [0, 1]
    for _ in range(10):
        fib.append(fib[-1] + fib[-2])
    got = oracle.hash_one(3, np.array(fib, dtype=np.uint64)).tolist()
    assert got == golden["kat"]["poseidon2_hash_one_fib12"]["expected"]


def test_keccak_kat(oracle, golden):
    k = golden["kat"]["keccak_hash_one"]
    data = np.array(k["data"], dtype=np.uint64)
    out = np.zeros(4, dtype=np.uint64)  # sizes < 4 copy into a zeroed digest, as tests.cu does
    for size in range(1, 7):
        oracle.hash_one(1, data[:size], out)
        assert out.tolist() == k["expected"][str(size)], size


def test_monolith_kat(oracle, golden):
    k = golden["kat"]["monolith_hash_one"]
    got = oracle.hash_one(4, np.array(k["input"], dtype=np.uint64)).tolist()
    assert got == k["expected"]


def test_poseidon_bn128_kat(oracle, golden):
    k = golden["kat"]["poseidon_bn128_hash_one"]
    got = oracle.hash_one(2, np.array(k["input"], dtype=np.uint64)).tolist()
    assert got == k["expected"]


def test_go_merkle_caps(oracle, golden):
    k = golden["kat"]["go_merkle_caps"]
    leaf = np.array(k["leaf"], dtype=np.uint64)
    for case in k["cases"]:
        nl, nc = case["n_leaves"], case["n_caps"]
        leaves = np.tile(leaf, nl)
        _, cap = oracle.merkle_fill(leaves, leaf.size, nc.bit_length() - 1, 0)
        for j in range(nc):
            assert cap[4 * j:4 * j + 4].tolist() == case["cap"]


def _shapes(golden):
    keys = sorted(k[:-len("_seed")] for k in golden["merkle"] if k.endswith("_seed"))
    for key in keys:
        name, shape, ch = key.split("_")
        nl, ls = map(int, shape.split("x"))
        yield key, HASHES[name], nl, ls, int(ch[1:])


def test_merkle_vs_reference_cpu_fixtures(oracle, golden):
    n = 0
    for key, ht, nl, ls, ch in _shapes(golden):
        seed = int(golden["merkle"][key + "_seed"][0])
        leaves = oracle.field_elems(seed, nl * ls)
        d, c = oracle.merkle_fill(leaves, ls, ch, ht)
        assert np.array_equal(c, golden["merkle"][key + "_cap"]), key
        if (nl >> ch) > 1 and nl != (1 << ch):  # zeknox's CPU path writes digests only then
            assert np.array_equal(d, golden["merkle"][key + "_digests"]), key
        n += 1
    assert n >= 60


@pytest.mark.skipif("not __import__('oracle.oracle', fromlist=['x']).ref_available()")
def test_oracle_vs_live_reference_cpu(oracle):
    """When zeknox's CPU build is present (this container), compare live on fresh seeds."""
    for ht in (0, 1, 2, 3, 4):
        for nl, ls, ch in ((64, 135, 2), (128, 11, 3), (32, 5, 0)):
            leaves = oracle.field_elems(1000 + ht * 7 + nl, nl * ls)
            d, c = oracle.merkle_fill(leaves, ls, ch, ht)
            d2, c2 = oracle.ref_merkle_fill(leaves, ls, ch, ht)
            assert np.array_equal(c, c2) and np.array_equal(d, d2)


# ---------------------------------------------------------------- NTT
def _dft(x, w):
    n = len(x)
    return [sum(int(x[i]) * pow(w, i * k, P) for i in range(n)) % P for k in range(n)]


@pytest.mark.parametrize("lg", [1, 2, 3, 5, 7])
def test_ntt_raw_matches_naive_dft(oracle, lg):
    x = oracle.field_elems(77 + lg, 1 << lg)
    w = pow(7, (P - 1) >> lg, P)
    assert oracle.ntt_raw(x, lg).tolist() == _dft(x, w)
    assert oracle.ntt_raw(x, lg, inverse=True).tolist() == _dft(x, pow(w, P - 2, P))


@pytest.mark.parametrize("lg,batches", [(1, 3), (4, 2), (10, 3), (13, 2)])
def test_batch_ntt_roundtrip(oracle, lg, batches):
    # wrappers/rust/tests/ntt.rs:84-108: iNTT(NTT(x)) = x
    x = oracle.field_elems(5 + lg, batches << lg)
    y = oracle.batch_ntt(x, lg, False, batches)
    assert np.array_equal(oracle.batch_ntt(y, lg, True, batches), x)


@pytest.mark.parametrize("lg_n,rate", [(1, 1), (3, 2), (6, 3), (9, 1)])
def test_lde_is_coset_evaluation(oracle, lg_n, rate):
    """out[b][k] = poly_b(g * w_N^k): the coset LDE of wrappers/rust/tests/ntt.rs:394-479."""
    b = 2
    c = oracle.field_elems(9 + lg_n, b << lg_n)
    out = oracle.batch_lde(c, lg_n, rate, b).reshape(b, -1)
    N = 1 << (lg_n + rate)
    w = pow(7, (P - 1) >> (lg_n + rate), P)
    for row in range(b):
        coeffs = [int(v) for v in c[row << lg_n:(row + 1) << lg_n]]
        for k in list(range(min(N, 16))) + [N - 1]:
            x = 7 * pow(w, k, P) % P
            acc = 0
            for a in reversed(coeffs):
                acc = (acc * x + a) % P
            assert int(out[row, k]) == acc


def test_inverse_lde_semantics(oracle):
    # ntt.cu:531-535 + :137-143: zero-extend, inverse transform, x coset^i, x N^-1
    lg_n, rate, b = 4, 2, 2
    c = oracle.field_elems(31, b << lg_n)
    out = oracle.batch_lde(c, lg_n, rate, b, inverse=True).reshape(b, -1)
    N = 1 << (lg_n + rate)
    winv = pow(pow(7, (P - 1) >> (lg_n + rate), P), P - 2, P)
    ninv = pow(N, P - 2, P)
    for row in range(b):
        ext = [int(v) for v in c[row << lg_n:(row + 1) << lg_n]] + [0] * (N - (1 << lg_n))
        ref = _dft(ext, winv)
        assert out[row].tolist() == [ref[i] * pow(7, i, P) % P * ninv % P for i in range(N)]


def test_transpose_rev_semantics(oracle):
    # wrappers/rust/tests/utils.rs:15-27: transpose then swap rows i <-> rev(i)
    lg, b = 5, 3
    x = oracle.field_elems(3, b << lg)
    out = oracle.transpose_rev(x, lg, b).reshape(1 << lg, b)
    m = x.reshape(b, 1 << lg)
    for k in range(1 << lg):
        r = int(format(k, f"0{lg}b")[::-1], 2)
        assert out[r].tolist() == m[:, k].tolist()


# ---------------------------------------------------------------- FRI oracle
def test_fri_fold_oracle_matches_definition(oracle):
    """The C fold (Horner) against sum_t beta^t c[j a + t] in Python integers."""
    n = 128
    c = oracle.field_elems(77, 2 * n).reshape(2, n)
    for ab, beta in [(1, (3, 5)), (3, (oracle.P - 1, 2)), (5, (0x1234567890ABCDEF, 0))]:
        got = oracle.fri_fold(c, ab, beta)
        a = 1 << ab
        for j in range(n >> ab):
            acc = (0, 0)
            for t in range(a):
                acc = oracle.ext_add(acc, oracle.ext_mul(oracle.ext_pow(beta, t), (int(c[0, j * a + t]), int(c[1, j * a + t]))))
            assert (int(got[0, j]), int(got[1, j])) == acc


def test_fri_extension_field_is_a_field(oracle):
    """X^2 - 7 is irreducible over GF(p) (7 is a non-residue): x^(p^2-1) = 1 and
    the inverse x^(p^2-2) really inverts."""
    P = oracle.P
    assert pow(7, (P - 1) // 2, P) == P - 1
    for x in [(1, 1), (0, 1), (12345, 67890), (P - 1, 3)]:
        assert oracle.ext_pow(x, P * P - 1) == (1, 0)
        assert oracle.ext_mul(x, oracle.ext_pow(x, P * P - 2)) == (1, 0)


@pytest.mark.parametrize("lg_n,rate,arities,cap_h", [(9, 2, [2, 3, 1], 1), (8, 3, [4], 2), (10, 1, [1, 1, 2, 3], 0)])
def test_fri_oracle_rounds_fold_consistently(oracle, lg_n, rate, arities, cap_h):
    """Every leaf row of a round, interpolated at beta as the FRI verifier does,
    gives the next round's value at that position (the final polynomial after the
    last round): the fold, the shifted-coset LDE and the bit-reversed leaf layout
    agree with each other."""
    P = oracle.P

    def challenge(i, cap):
        return (int(cap[0]) % P, int(cap[(1 + i) % cap.size]) % P)

    c = oracle.field_elems(300 + lg_n, 2 << lg_n).reshape(2, -1)
    rounds, final = oracle.fri_commit(c, rate, arities, cap_h, challenge)
    assert final.shape == (2, (1 << lg_n) >> sum(arities))
    for i, (r, ab) in enumerate(zip(rounds, arities)):
        lg_N = (r["leaves"].size // 2).bit_length() - 1
        m = r["leaves"].shape[0]
        for j in sorted({0, 1, m // 3, m - 1}):
            y, v = oracle.fri_fold_from_leaf(r["leaves"][j], j, lg_N, r["shift"], ab, r["beta"])
            if i + 1 < len(rounds):
                nxt = rounds[i + 1]["leaves"].reshape(-1, 2)[j]
                assert v == (int(nxt[0]), int(nxt[1])), (i, j)
            else:
                assert v == oracle.ext_poly_eval(final, y), (i, j)
