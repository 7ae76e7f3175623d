"""Regenerate the golden fixtures in this directory (run where the zeknox
sources are available; the committed fixtures are what the tests read).

kat.json
    Known-answer vectors transcribed from zeknox's own tests, with the file and
    line each one comes from (parsed from those files, not typed in):
    Poseidon hash_one sizes 1..9 (native/tests/tests.cu:279-292), Poseidon2
    Fibonacci input (tests.cu:409-428), Keccak sizes 1..6 (tests.cu:164-173),
    Monolith hash_one of 0..11 (tests.cu:201-203), Poseidon-BN128 hash_one
    (tests.cu:492-501) and the Go Merkle caps
    (wrappers/go/lib/lib_test.go:194-213).

merkle_ref_cpu.npz
    Digests and caps produced by zeknox's own C++ CPU Merkle path
    (fill_digests_buf_linear_cpu, native/merkle/merkle.cpp:126-161, compiled by
    oracle/build_ref.sh) on SplitMix64-seeded leaves, for each hasher over a set
    of shapes covering the special cases of merkle.cu:178-212.

Usage: python tests/golden/make_golden.py [zeknox-root]
"""

import json
import os
import re
import sys
from pathlib import Path

import numpy as np

ROOT = Path(__file__).resolve().parents[2]
sys.path.insert(0, str(ROOT))
from oracle import oracle as O  # noqa: E402

# (n_leaves, leaf_size, cap_height): cap == leaves, L_s == 1, L_s == 2, general,
# short leaves (< 4 and == 4 elements), one chunk, ragged last chunk, config-1 width.
MERKLE_SHAPES = [
    (8, 7, 3), (16, 9, 4), (8, 7, 2), (16, 7, 1), (64, 135, 2), (256, 9, 0), (1024, 16, 4),
    (32, 4, 1), (32, 3, 1), (128, 8, 3), (512, 13, 2), (256, 135, 4),
]
HASHES = {"poseidon": O.HASH_POSEIDON, "poseidon2": O.HASH_POSEIDON2, "keccak": O.HASH_KECCAK,
          "monolith": O.HASH_MONOLITH, "poseidonbn128": O.HASH_POSEIDON_BN128}


def _u64s(txt):
    return [int(t.rstrip("ul").rstrip("ULL"), 0) for t in re.findall(r"0x[0-9a-fA-F]+|\d+", txt)]


def parse_kats(zk: Path) -> dict:
    tests = (zk / "native/tests/tests.cu").read_text().splitlines()
    gotest = (zk / "wrappers/go/lib/lib_test.go").read_text().splitlines()

    def block(lines, start, stop):
        return "\n".join(lines[start - 1:stop])

    kat = {}
    # Poseidon: leaf at tests.cu:279, expected[11][4] at :281-292.
    leaf = _u64s(block(tests, 279, 279).split("=", 1)[1])
    exp = [_u64s(l) for l in tests[281:292] if "{" in l]
    kat["poseidon_hash_one"] = {"source": "native/tests/tests.cu:279-292", "leaf": leaf,
                                "expected": {str(k): exp[k] for k in range(1, 10)}}
    # Poseidon2: Fibonacci input, expected digest asserted at tests.cu:425-428.
    p2 = [int(m, 16) for m in re.findall(r"h1\[\d\] == (0x[0-9a-fA-F]+)", block(tests, 424, 429))]
    kat["poseidon2_hash_one_fib12"] = {"source": "native/tests/tests.cu:405-428", "expected": p2}
    # Keccak: data at :164, expected[7][4] at :166-173.
    data = _u64s(block(tests, 164, 164).split("=", 1)[1])
    kexp = [_u64s(l) for l in tests[166:173] if "{" in l]
    kat["keccak_hash_one"] = {"source": "native/tests/tests.cu:164-173", "data": data,
                              "expected": {str(s): kexp[s] for s in range(1, 7)}}
    # Monolith: input at tests.cu:203, expected digest at :204.
    mono_in = _u64s(block(tests, 203, 203).split("=", 1)[1])
    mono_exp = _u64s(block(tests, 204, 204).split("=", 1)[1])
    kat["monolith_hash_one"] = {"source": "native/tests/tests.cu:201-204", "input": mono_in, "expected": mono_exp}
    # Poseidon-BN128: input at tests.cu:494-499, expected digest at :501.
    bn_in = _u64s(block(tests, 494, 499).split("=", 1)[1])
    bn_exp = _u64s(block(tests, 501, 501).split("=", 1)[1])
    kat["poseidon_bn128_hash_one"] = {"source": "native/tests/tests.cu:492-501", "input": bn_in, "expected": bn_exp}
    # Go caps: leaf at lib_test.go:195, three (nLeaves, nCaps, expHash) cases.
    gl = _u64s(block(gotest, 195, 195).split("{", 1)[1])
    cases = []
    body = block(gotest, 196, 213)
    for nl, nc, eh in re.findall(r"nLeaves :?= (\d+).*?nCaps :?= (\w+).*?expHash :?= \[\]uint64\{([^}]*)\}", body, re.S):
        nl = int(nl)
        nc = nl if nc == "nLeaves" else int(nc)
        cases.append({"n_leaves": nl, "n_caps": nc, "cap": _u64s(eh)})
    kat["go_merkle_caps"] = {"source": "wrappers/go/lib/lib_test.go:194-213", "leaf": gl, "cases": cases}
    assert len(cases) == 3 and len(exp) >= 10 and len(kexp) == 7 and len(p2) == 4
    assert len(mono_in) == 12 and len(mono_exp) == 4
    assert len(bn_in) == 12 and len(bn_exp) == 4
    return kat


def merkle_fixtures() -> dict:
    out = {}
    for name, ht in HASHES.items():
        for i, (nl, ls, ch) in enumerate(MERKLE_SHAPES):
            seed = 0x5EED0000 + 100 * ht + i
            leaves = O.field_elems(seed, nl * ls)
            d, c = O.ref_merkle_fill(leaves, ls, ch, ht)
            key = f"{name}_{nl}x{ls}_c{ch}"
            out[key + "_seed"] = np.array([seed], dtype=np.uint64)
            out[key + "_digests"] = d
            out[key + "_cap"] = c
    return out


def main():
    src = sys.argv[1] if len(sys.argv) > 1 else os.environ.get("ZEKNOX_SRC")
    if not src:
        sys.exit("usage: make_golden.py <zeknox source tree>   (or set ZEKNOX_SRC)")
    zk = Path(src)
    here = Path(__file__).resolve().parent
    (here / "kat.json").write_text(json.dumps(parse_kats(zk), indent=1) + "\n")
    np.savez_compressed(here / "merkle_ref_cpu.npz", **merkle_fixtures())
    print("wrote", here / "kat.json", here / "merkle_ref_cpu.npz")


if __name__ == "__main__":
    main()
