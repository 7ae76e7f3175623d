"""ORACLE -- test infrastructure only.

ctypes front end of ``liboracle.so`` (the C restatement in oracle.c) and of
zeknox's own CPU build in ``_ref/libzkref_cpu.so`` (built by build_ref.sh when
the zeknox sources are present).  Only tests/, ``__graft_entry__.smoke()`` and
the bench's cpu_baseline / reference legs import this module, and only as the
checker or the timed CPU baseline: the product never routes through it.
"""

from __future__ import annotations

import ctypes
import os
import subprocess
from pathlib import Path

import numpy as np

HERE = Path(__file__).resolve().parent
_LIB = None
_REF = None

HASH_POSEIDON, HASH_KECCAK, HASH_POSEIDON_BN128, HASH_POSEIDON2, HASH_MONOLITH = 0, 1, 2, 3, 4
P = 0xFFFFFFFF00000001

_u64p = ctypes.POINTER(ctypes.c_uint64)


def _ptr(a: np.ndarray):
    assert a.dtype == np.uint64 and a.flags["C_CONTIGUOUS"]
    return a.ctypes.data_as(_u64p)


def build() -> Path:
    """Compile liboracle.so (plain C, gcc) if it is missing or stale."""
    so = HERE / "liboracle.so"
    src = [HERE / "oracle.c", HERE.parent / "zeknox_b200" / "csrc" / "zk_constants.h"]
    if not so.exists() or any(s.stat().st_mtime > so.stat().st_mtime for s in src):
        subprocess.run(["make", "-s", "-C", str(HERE), "liboracle.so"], check=True)
    return so


def lib():
    global _LIB
    if _LIB is None:
        _LIB = ctypes.CDLL(str(build()))
        L = _LIB
        u64, u32, c_int, vp = ctypes.c_uint64, ctypes.c_uint32, ctypes.c_int, ctypes.c_void_p
        for name in ("orc_add", "orc_sub", "orc_mul", "orc_pow"):
            getattr(L, name).argtypes = [u64, u64]
            getattr(L, name).restype = u64
        for name in ("orc_omega", "orc_omega_inv", "orc_domain_size_inv"):
            getattr(L, name).argtypes = [ctypes.c_uint]
            getattr(L, name).restype = u64
        L.orc_poseidon_permute.argtypes = [_u64p]
        L.orc_poseidon2_permute.argtypes = [_u64p]
        L.orc_monolith_permute.argtypes = [_u64p]
        L.orc_keccak256.argtypes = [vp, ctypes.c_size_t, vp]
        L.orc_hash_one.argtypes = [c_int, _u64p, u64, _u64p]
        L.orc_hash_one.restype = c_int
        L.orc_hash_two.argtypes = [c_int, _u64p, _u64p, _u64p]
        L.orc_hash_two.restype = c_int
        L.orc_merkle_fill.argtypes = [_u64p, _u64p, _u64p, u64, u64, u64, u64, u64, c_int]
        L.orc_merkle_fill.restype = c_int
        L.orc_ntt_raw.argtypes = [_u64p, ctypes.c_uint, c_int]
        L.orc_batch_ntt.argtypes = [_u64p, ctypes.c_uint, c_int, ctypes.c_uint, c_int, u64]
        L.orc_batch_lde.argtypes = [_u64p, _u64p, ctypes.c_uint, ctypes.c_uint, c_int, ctypes.c_uint, c_int, u64]
        L.orc_transpose_rev.argtypes = [_u64p, _u64p, ctypes.c_uint, ctypes.c_uint]
        L.orc_fri_fold.argtypes = [_u64p, _u64p, u64, ctypes.c_uint, u64, u64]
    return _LIB


def ref_available() -> bool:
    return (HERE / "_ref" / "libzkref_cpu.so").exists()


def ref():
    """zeknox's own CPU path (compiled from its sources), or None if not built."""
    global _REF
    if _REF is None and ref_available():
        _REF = ctypes.CDLL(str(HERE / "_ref" / "libzkref_cpu.so"))
        u64, vp = ctypes.c_uint64, ctypes.c_void_p
        _REF.fill_digests_buf_linear_cpu.argtypes = [vp, vp, vp, u64, u64, u64, u64, u64, u64]
        _REF.fill_digests_buf_linear_cpu.restype = None
        _REF.zkref_hash_one.argtypes = [ctypes.c_int, _u64p, u64, _u64p]
        _REF.zkref_hash_two.argtypes = [ctypes.c_int, _u64p, _u64p, _u64p]
    return _REF


# ---------------------------------------------------------------- data
def splitmix64(seed: int, n: int) -> np.ndarray:
    """SplitMix64 stream (Steele, Lea, Flood 2014), vectorised."""
    idx = np.arange(1, n + 1, dtype=np.uint64)
    with np.errstate(over="ignore"):
        z = np.uint64(seed) + idx * np.uint64(0x9E3779B97F4A7C15)
        z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
        z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
        z = z ^ (z >> np.uint64(31))
    return z


def field_elems(seed: int, n: int) -> np.ndarray:
    """n uniform canonical field elements: SplitMix64 words rejection-sampled to [0, p)."""
    out = np.empty(0, dtype=np.uint64)
    s = seed
    while out.size < n:
        z = splitmix64(s, n - out.size + 64)
        out = np.concatenate([out, z[z < np.uint64(P)]])
        s = (s * 0x9E3779B97F4A7C15 + 1) & 0xFFFFFFFFFFFFFFFF
    return np.ascontiguousarray(out[:n])


def fill_field(seed: int, n: int) -> np.ndarray:
    """The product's synthetic-input stream (zk_fill_field_async, the salt rows'
    generator, ntt.cu salt_kernel), restated: element i is the first
    z(seed, i + j n), j = 0, 1, ..., below p, with z(s, c) = SplitMix64's
    output function of s + (c + 1) * 0x9E3779B97F4A7C15."""
    out = np.empty(n, dtype=np.uint64)
    todo = np.arange(n, dtype=np.uint64)
    ctr = todo.copy()
    while todo.size:
        with np.errstate(over="ignore"):
            z = np.uint64(seed) + (ctr + np.uint64(1)) * np.uint64(0x9E3779B97F4A7C15)
            z = (z ^ (z >> np.uint64(30))) * np.uint64(0xBF58476D1CE4E5B9)
            z = (z ^ (z >> np.uint64(27))) * np.uint64(0x94D049BB133111EB)
            z = z ^ (z >> np.uint64(31))
        ok = z < np.uint64(P)
        out[todo[ok]] = z[ok]
        todo, ctr = todo[~ok], ctr[~ok] + np.uint64(n)
    return out


# ---------------------------------------------------------------- hashing
def hash_one(ht: int, leaf: np.ndarray, out: np.ndarray | None = None) -> np.ndarray:
    leaf = np.ascontiguousarray(leaf, dtype=np.uint64)
    out = np.zeros(4, dtype=np.uint64) if out is None else out
    if lib().orc_hash_one(ht, _ptr(leaf), leaf.size, _ptr(out)) != 0:
        raise ValueError(f"unsupported hash type {ht}")
    return out


def hash_two(ht: int, left: np.ndarray, right: np.ndarray) -> np.ndarray:
    out = np.zeros(4, dtype=np.uint64)
    l = np.ascontiguousarray(left, dtype=np.uint64)
    r = np.ascontiguousarray(right, dtype=np.uint64)
    if lib().orc_hash_two(ht, _ptr(l), _ptr(r), _ptr(out)) != 0:
        raise ValueError(f"unsupported hash type {ht}")
    return out


def permute(ht: int, state: np.ndarray) -> np.ndarray:
    st = np.ascontiguousarray(state, dtype=np.uint64).copy()
    assert st.size == 12
    perm = {HASH_POSEIDON: lib().orc_poseidon_permute, HASH_POSEIDON2: lib().orc_poseidon2_permute,
            HASH_MONOLITH: lib().orc_monolith_permute}[ht]
    perm(_ptr(st))
    return st


def merkle_sizes(n_leaves: int, cap_height: int):
    n_caps = 1 << cap_height
    return 2 * (n_leaves - n_caps), n_caps


def merkle_fill(leaves: np.ndarray, leaf_size: int, cap_height: int, ht: int,
                digests: np.ndarray | None = None, cap: np.ndarray | None = None):
    """Digests + cap in zeknox's linear layout (merkle/merkle.cu:166-244)."""
    leaves = np.ascontiguousarray(leaves, dtype=np.uint64).reshape(-1)
    n_leaves = leaves.size // leaf_size
    n_digests, n_caps = merkle_sizes(n_leaves, cap_height)
    if digests is None:
        digests = np.zeros(max(n_digests, 1) * 4, dtype=np.uint64)
    if cap is None:
        cap = np.zeros(n_caps * 4, dtype=np.uint64)
    rc = lib().orc_merkle_fill(_ptr(digests), _ptr(cap), _ptr(leaves), n_digests, n_caps, n_leaves,
                               leaf_size, cap_height, ht)
    if rc != 0:
        raise ValueError(f"unsupported hash type {ht}")
    return digests, cap


def ref_merkle_fill(leaves: np.ndarray, leaf_size: int, cap_height: int, ht: int):
    """zeknox's own fill_digests_buf_linear_cpu (merkle/merkle.cpp:126-161)."""
    R = ref()
    if R is None:
        raise RuntimeError("zeknox CPU build not available (oracle/build_ref.sh)")
    leaves = np.ascontiguousarray(leaves, dtype=np.uint64).reshape(-1)
    n_leaves = leaves.size // leaf_size
    n_digests, n_caps = merkle_sizes(n_leaves, cap_height)
    digests = np.zeros(max(n_digests, 1) * 4, dtype=np.uint64)
    cap = np.zeros(n_caps * 4, dtype=np.uint64)
    R.fill_digests_buf_linear_cpu(digests.ctypes.data, cap.ctypes.data, leaves.ctypes.data, n_digests,
                                  n_caps, n_leaves, leaf_size, cap_height, ht)
    return digests, cap


# ---------------------------------------------------------------- NTT
def ntt_raw(a: np.ndarray, lg: int, inverse: bool = False) -> np.ndarray:
    out = np.ascontiguousarray(a, dtype=np.uint64).copy()
    lib().orc_ntt_raw(_ptr(out), lg, int(inverse))
    return out


def batch_ntt(inout: np.ndarray, lg: int, inverse: bool, batches: int, with_coset: bool = False,
              coset_gen: int = 7) -> np.ndarray:
    out = np.ascontiguousarray(inout, dtype=np.uint64).copy()
    assert out.size == batches << lg
    lib().orc_batch_ntt(_ptr(out), lg, int(inverse), batches, int(with_coset), coset_gen)
    return out


def batch_lde(inp: np.ndarray, lg_n: int, rate_bits: int, batches: int, inverse: bool = False,
              with_coset: bool = True, coset_gen: int = 7) -> np.ndarray:
    inp = np.ascontiguousarray(inp, dtype=np.uint64)
    assert inp.size == batches << lg_n
    out = np.empty(batches << (lg_n + rate_bits), dtype=np.uint64)
    lib().orc_batch_lde(_ptr(out), _ptr(inp), lg_n, rate_bits, int(inverse), batches, int(with_coset), coset_gen)
    return out


def transpose_rev(inp: np.ndarray, lg_n: int, batches: int) -> np.ndarray:
    inp = np.ascontiguousarray(inp, dtype=np.uint64)
    assert inp.size == batches << lg_n
    out = np.empty_like(inp)
    lib().orc_transpose_rev(_ptr(out), _ptr(inp), lg_n, batches)
    return out


def set_threads(n: int) -> None:
    os.environ["OMP_NUM_THREADS"] = str(n)


# ---------------------------------------------------------------- FRI
# GF(p^2) = GF(p)[X]/(X^2 - 7) in Python integers (pairs (real, X part)), and
# the FRI commit phase over it, restating the published algorithm of Plonky2's
# prover (okx/plonky2 rev 9a917ba2, fri/prover.rs fri_committed_trees; a git
# dependency of zeknox's Rust wrapper, wrappers/rust/Cargo.toml:43-44, absent
# here).  Parity against Plonky2 is unpinned; the checks below are the FRI
# verifier's own consistency relations.
EXT_W = 7


def ext_mul(a, b):
    return ((a[0] * b[0] + EXT_W * a[1] * b[1]) % P, (a[0] * b[1] + a[1] * b[0]) % P)


def ext_add(a, b):
    return ((a[0] + b[0]) % P, (a[1] + b[1]) % P)


def ext_scale(a, c: int):
    return (a[0] * c % P, a[1] * c % P)


def ext_pow(a, e: int):
    r = (1, 0)
    while e:
        if e & 1:
            r = ext_mul(r, a)
        a = ext_mul(a, a)
        e >>= 1
    return r


def fri_fold(coeffs: np.ndarray, arity_bits: int, beta) -> np.ndarray:
    """(2, n) split GF(p^2) coefficients -> (2, n >> arity_bits): sum_t beta^t c[j a + t]."""
    c = np.ascontiguousarray(coeffs, dtype=np.uint64).reshape(2, -1)
    n = c.shape[1]
    out = np.empty((2, n >> arity_bits), dtype=np.uint64)
    lib().orc_fri_fold(_ptr(out), _ptr(c), n, arity_bits, int(beta[0]), int(beta[1]))
    return out


def fri_round_leaves(coeffs: np.ndarray, rate_bits: int, shift: int, arity_bits: int) -> np.ndarray:
    """Evaluations of the (2, n) coefficients on shift * <w_N>, N = n 2^rate_bits,
    in bit-reversed order, as rows of 2^arity_bits interleaved (real, X) pairs."""
    c = np.ascontiguousarray(coeffs, dtype=np.uint64).reshape(2, -1)
    lg_n = c.shape[1].bit_length() - 1
    lde = batch_lde(c.reshape(-1), lg_n, rate_bits, 2, coset_gen=shift)
    leaves = transpose_rev(lde, lg_n + rate_bits, 2)  # (N, 2), bit-reversed rows
    return leaves.reshape(-1, 2 << arity_bits)


def fri_commit(coeffs: np.ndarray, rate_bits: int, arity_bits, cap_height: int, challenge, ht: int = HASH_POSEIDON,
               shift: int = 7):
    """The commit phase: per round, leaves / digests / cap, the challenge drawn from
    the cap by `challenge(round, cap)`, the fold; then the final coefficients.
    Returns (rounds, final (2, n_final)); rounds[i] = dict(leaves, digests, cap, beta, shift)."""
    cur = np.ascontiguousarray(coeffs, dtype=np.uint64).reshape(2, -1)
    rounds = []
    for i, ab in enumerate(arity_bits):
        leaves = fri_round_leaves(cur, rate_bits, shift, ab)
        dig, cap = merkle_fill(leaves.reshape(-1), leaves.shape[1], cap_height, ht)
        beta = challenge(i, cap)
        rounds.append(dict(leaves=leaves, digests=dig, cap=cap, beta=beta, shift=shift))
        cur = fri_fold(cur, ab, beta)
        shift = pow(shift, 1 << ab, P)
    return rounds, cur


def _bitrev(x: int, bits: int) -> int:
    return int(format(x, f"0{bits}b")[::-1], 2) if bits else 0


def fri_fold_from_leaf(row: np.ndarray, j: int, lg_N: int, shift: int, arity_bits: int, beta):
    """The folded polynomial's value at y = x0^a, computed from one leaf row of a
    round (the a evaluations at x0 * zeta^u, zeta = w_a) as the FRI verifier
    does: interpolate P_i on the coset x0 <zeta> and combine its parts with the
    powers of beta.  Returns (y, value)."""
    a = 1 << arity_bits
    m = _bitrev(j, lg_N - arity_bits)
    x0 = shift * pow(omega(lg_N), m, P) % P
    zeta_inv = pow(omega(arity_bits), P - 2, P) if arity_bits else 1
    e = [None] * a
    for t in range(a):  # row position t holds natural offset u = rev(t)
        e[_bitrev(t, arity_bits)] = (int(row[2 * t]), int(row[2 * t + 1]))
    a_inv = pow(a, P - 2, P)
    x0_inv = pow(x0, P - 2, P)
    acc = (0, 0)
    bpow = (1, 0)
    for t in range(a):
        q = (0, 0)  # Q_t(y) x0^t * a
        for u in range(a):
            q = ext_add(q, ext_scale(e[u], pow(zeta_inv, t * u, P)))
        q = ext_scale(q, a_inv * pow(x0_inv, t, P) % P)
        acc = ext_add(acc, ext_mul(bpow, q))
        bpow = ext_mul(bpow, (int(beta[0]), int(beta[1])))
    return pow(x0, a, P), acc


def ext_poly_eval(coeffs: np.ndarray, x: int):
    """Value at the base-field point x of the (2, n) split GF(p^2) polynomial."""
    c = np.ascontiguousarray(coeffs, dtype=np.uint64).reshape(2, -1)
    r0 = r1 = 0
    for k in range(c.shape[1] - 1, -1, -1):
        r0 = (r0 * x + int(c[0, k])) % P
        r1 = (r1 * x + int(c[1, k])) % P
    return (r0, r1)


def omega(lg: int) -> int:
    return pow(7, (P - 1) >> lg, P)
