"""Generate ``zk_constants.h``: the round-constant tables of the three hashers.

The hashers are defined by their constants, so these tables must hold the same
values as zeknox's (which are Plonky2's Goldilocks Poseidon / Poseidon2
parameters):

* Poseidon: 360 round constants and the 12-entry MDS circulant + diagonal,
  read from ``native/poseidon/poseidon.hpp`` (``ALL_ROUND_CONSTANTS`` at
  poseidon.hpp:803, ``MDS_MATRIX_CIRC`` / ``MDS_MATRIX_DIAG`` at :35-36).
* Poseidon2: 360 round constants (12 per round, zero lanes for the internal
  rounds) and the 12-entry internal diagonal, read from
  ``native/poseidon2/poseidon2.cu`` (``RC12`` at :26, ``MATRIX_DIAG_12`` at :8).
* Monolith (width 12, 6 rounds): the 7 x 12 round constants and the 12 x 12
  circulant matrix, read from ``native/monolith/monolith.cu``
  (``MONOLITH_ROUND_CONSTANTS`` at monolith.cu:11, ``MONOLITH_MAT_12`` at :103);
  only the matrix's first row is kept, after checking that it is circulant.
* Poseidon-BN128 (circomlib Poseidon over the BN254 scalar field, t = 5, in
  its optimised form): round constants C[100], sparse matrices S[540], MDS
  M[5][5] and the pre-sparse matrix P[5][5], each a 4 x 64-bit Montgomery
  value, read from ``native/poseidon/poseidon_bn128_constants.h`` (:16, :119,
  :662, :700).
* Keccak-f[1600]: the 24 iota constants and the rho rotation offsets are not
  copied; they are computed here from the FIPS 202 definitions (the rc(t) LFSR
  with polynomial x^8+x^6+x^5+x^4+1, and offsets (t+1)(t+2)/2 along the
  (x, y) -> (y, 2x+3y) walk).

The header is committed; this script is only re-run when the tables change.
It reads the zeknox sources from the directory given on the command line.
"""

import re
import sys
from pathlib import Path


def _table(text: str, name: str) -> list:
    m = re.search(name + r"\s*(?:\[[^\]]*\]\s*)+=\s*\{(.*?)\};", text, re.S)
    if m is None:
        raise SystemExit(f"table {name} not found")
    body = re.sub(r"//[^\n]*", "", m.group(1))
    # The CUDA/C++ variants of a table share one initializer between #ifdef
    # branches: drop preprocessor lines and the alternative declaration.
    body = "\n".join(
        ln for ln in body.splitlines()
        if not ln.strip().startswith("#") and "u64" not in ln and "=" not in ln
    )
    vals = []
    for tok in re.findall(r"0x[0-9a-fA-F]+|\d+", body):
        vals.append(int(tok, 16) if tok.lower().startswith("0x") else int(tok))
    return vals


def keccak_round_constants() -> list:
    """FIPS 202 Algorithm 5/6: RC[ir] bit (2^j - 1) = rc(j + 7*ir)."""

    def rc(t: int) -> int:
        if t % 255 == 0:
            return 1
        r = 0b10000000  # R = 10000000 (bit 0 is the leftmost bit)
        for _ in range(t % 255):
            # R = 0 || R; then R[0]^=R[8], R[4]^=R[8], R[5]^=R[8], R[6]^=R[8]; R = Trunc8(R)
            bits = [0] + [(r >> (7 - i)) & 1 for i in range(8)]
            b8 = bits[8]
            bits[0] ^= b8
            bits[4] ^= b8
            bits[5] ^= b8
            bits[6] ^= b8
            r = 0
            for i in range(8):
                r |= bits[i] << (7 - i)
        return (r >> 7) & 1

    out = []
    for ir in range(24):
        v = 0
        for j in range(7):
            if rc(j + 7 * ir):
                v |= 1 << ((1 << j) - 1)
        out.append(v)
    return out


def keccak_rho_offsets() -> list:
    """Rotation offset of lane (x, y), lane index x + 5y (FIPS 202 Algorithm 2)."""
    off = [0] * 25
    x, y = 1, 0
    for t in range(24):
        off[x + 5 * y] = ((t + 1) * (t + 2) // 2) % 64
        x, y = y, (2 * x + 3 * y) % 5
    return off


def main() -> None:
    src = Path(sys.argv[1])
    out = Path(sys.argv[2]) if len(sys.argv) > 2 else Path(__file__).with_name("zk_constants.h")
    pos = (src / "poseidon/poseidon.hpp").read_text()
    p2 = (src / "poseidon2/poseidon2.cu").read_text()
    mono = (src / "monolith/monolith.cu").read_text()
    bn = (src / "poseidon/poseidon_bn128_constants.h").read_text()

    rc = _table(pos, "ALL_ROUND_CONSTANTS")
    circ = _table(pos, "MDS_MATRIX_CIRC")
    diag = _table(pos, "MDS_MATRIX_DIAG")
    p2_rc = _table(p2, "RC12")
    p2_diag = _table(p2, "MATRIX_DIAG_12_GOLDILOCKS")
    assert len(rc) == 360 and len(circ) == 12 and len(diag) == 12
    assert len(p2_rc) == 360 and len(p2_diag) == 12
    mono_rc = _table(mono, "MONOLITH_ROUND_CONSTANTS")
    mono_mat = _table(mono, "MONOLITH_MAT_12")
    assert len(mono_rc) == 84 and len(mono_mat) == 144
    mono_row = mono_mat[:12]
    bn_c, bn_s = _table(bn, "CONST u64 C"), _table(bn, "CONST u64 S")
    bn_m, bn_p = _table(bn, "CONST u64 M"), _table(bn, "CONST u64 P")
    assert len(bn_c) == 400 and len(bn_s) == 2160 and len(bn_m) == 100 and len(bn_p) == 100
    assert all(mono_mat[12 * r + c] == mono_row[(c - r) % 12] for r in range(12) for c in range(12)), "not circulant"
    kc = keccak_round_constants()
    rho = keccak_rho_offsets()
    # Known first / last iota constants of Keccak-f[1600].
    assert kc[0] == 0x1 and kc[1] == 0x8082 and kc[23] == 0x8000000080008008

    def arr(name, vals, per_line=4):
        # A list macro (usable in __constant__ / constexpr initializers of
        # device code) plus a plain array built from it.
        lines = []
        for i in range(0, len(vals), per_line):
            lines.append("    " + ", ".join(f"0x{v:016x}ull" for v in vals[i:i + per_line]))
        body = ", \\\n".join(lines)
        return (f"#define {name}_LIST \\\n{body}\n"
                f"ZK_CONST_TABLE uint64_t {name}[{len(vals)}] = {{{name}_LIST}};\n")

    h = [
        "// Generated by gen_constants.py. Round constants of the Goldilocks hashers.",
        "// Poseidon / Poseidon2 tables hold Plonky2's parameters (the values zeknox",
        "// uses); the Keccak-f[1600] tables are computed from FIPS 202.",
        "#pragma once",
        "#include <stdint.h>",
        "#ifndef ZK_CONST_TABLE",
        "#define ZK_CONST_TABLE static const",
        "#endif",
        "",
        "// Poseidon, width 12, x^7, 4 + 22 + 4 rounds; 12 constants per round.",
        arr("ZK_POSEIDON_RC", rc),
        "// MDS = circulant(row 0 below) + diag(8, 0, ..., 0); row r, column c uses",
        "// ZK_POSEIDON_MDS_CIRC[(c - r) mod 12].",
        arr("ZK_POSEIDON_MDS_CIRC", circ),
        arr("ZK_POSEIDON_MDS_DIAG", diag),
        "// Poseidon2, width 12: 4 external + 22 internal + 4 external rounds;",
        "// 12 constants per round (internal rounds use lane 0 only).",
        arr("ZK_POSEIDON2_RC", p2_rc),
        "// Internal-layer diagonal: x_i <- x_i * D_i + sum(x).",
        arr("ZK_POSEIDON2_DIAG", p2_diag),
        "// Monolith, width 12: round constants of the 7 concrete layers (rows 0 and 6 are zero).",
        arr("ZK_MONOLITH_RC", mono_rc),
        "// Monolith concrete layer: circulant, row r column c uses ZK_MONOLITH_MDS_ROW[(c - r) mod 12].",
        arr("ZK_MONOLITH_MDS_ROW", mono_row),
        "// Poseidon-BN128 (t = 5), Montgomery form, 4 little-endian 64-bit limbs per value:",
        "// round constants C[100], sparse matrices S[540] (9 per partial round), M[5][5], P[5][5].",
        arr("ZK_BN128_C", bn_c),
        arr("ZK_BN128_S", bn_s),
        arr("ZK_BN128_M", bn_m),
        arr("ZK_BN128_P", bn_p),
        "// Keccak-f[1600] iota constants (24 rounds).",
        arr("ZK_KECCAK_RC", kc),
        "// Rho rotation offsets per lane (index x + 5y).",
        "#define ZK_KECCAK_RHO_LIST " + ", ".join(str(v) for v in rho),
        "ZK_CONST_TABLE int ZK_KECCAK_RHO[25] = {ZK_KECCAK_RHO_LIST};",
        "",
    ]
    out.write_text("\n".join(h))
    print(f"wrote {out}")


if __name__ == "__main__":
    main()
