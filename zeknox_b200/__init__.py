"""zeknox-b200: zeknox's Goldilocks polynomial-commitment path on one B200.

The product is libzeknox.so (C ABI in include/zeknox.h, CUDA kernels for
sm_100a in csrc/).  This package loads it through ctypes (:mod:`.capi`, which
mirrors zeknox's Rust/Go wrapper functions) and adds tensor-level helpers used
by the tests and the benchmark.  PyTorch only provides device memory and
streams here.
"""

from __future__ import annotations

from . import capi
from .capi import (  # noqa: F401
    FORWARD,
    INVERSE,
    HashKeccak,
    HashMonolith,
    HashPoseidon,
    HashPoseidon2,
    HashPoseidonBN128,
    NTTConfig,
    TransposeConfig,
    ZeknoxError,
    fill_digests_buf_linear_cpu,
    fill_digests_buf_linear_gpu_with_gpu_ptr,
    fill_digests_buf_linear_multigpu_with_gpu_ptr,
    get_number_of_gpus,
    init_coset,
    init_cuda,
    init_cuda_degree,
    init_twiddle_factors,
    intt_batch,
    lde_batch,
    lde_batch_multi_gpu,
    list_devices_info,
    ntt_batch,
    transpose_rev_batch,
)

P = 0xFFFFFFFF00000001


def _stream_ptr(stream) -> int:
    import torch

    s = stream if stream is not None else torch.cuda.current_stream()
    return int(s.cuda_stream)


def lde(coeffs, rate_bits: int, *, inverse: bool = False, with_coset: bool = True, out=None, stream=None):
    """Coset LDE of the rows of a (B, 2^lg_n) uint64 CUDA tensor -> (B, 2^(lg_n+rate_bits)).

    Stream-ordered on `stream` (default: the current torch stream)."""
    import torch

    assert coeffs.dtype == torch.uint64 and coeffs.is_cuda and coeffs.is_contiguous() and coeffs.dim() == 2
    b, n = coeffs.shape
    lg_n = n.bit_length() - 1
    assert n == 1 << lg_n
    if out is None:
        out = torch.empty((b, n << rate_bits), dtype=torch.uint64, device=coeffs.device)
    capi.check(capi.LIB.zk_lde_async(out.data_ptr(), coeffs.data_ptr(), lg_n, rate_bits, b, int(inverse),
                                     int(with_coset), _stream_ptr(stream)))
    return out


def transpose_rev(mat, out=None, stream=None):
    """(B, 2^lg) -> (2^lg, B) with rows bit-reversed: out[rev(k)][b] = mat[b][k]."""
    import torch

    assert mat.dtype == torch.uint64 and mat.is_cuda and mat.is_contiguous() and mat.dim() == 2
    b, n = mat.shape
    lg = n.bit_length() - 1
    assert n == 1 << lg
    if out is None:
        out = torch.empty((n, b), dtype=torch.uint64, device=mat.device)
    capi.check(capi.LIB.zk_transpose_rev_async(out.data_ptr(), mat.data_ptr(), lg, b, _stream_ptr(stream)))
    return out


def lde_leaves(coeffs, rate_bits: int, out=None, stream=None):
    """Forward coset LDE of (B, 2^lg_n) written as leaves: (2^(lg_n+rate_bits), B),
    out[rev(k)][b] = LDE_b[k] (compute_batched_lde + compute_transpose_rev, fused)."""
    import torch

    assert coeffs.dtype == torch.uint64 and coeffs.is_cuda and coeffs.is_contiguous() and coeffs.dim() == 2
    b, n = coeffs.shape
    lg_n = n.bit_length() - 1
    assert n == 1 << lg_n
    if out is None:
        out = torch.empty((n << rate_bits, b), dtype=torch.uint64, device=coeffs.device)
    capi.check(capi.LIB.zk_lde_leaves_async(out.data_ptr(), coeffs.data_ptr(), lg_n, rate_bits, b, _stream_ptr(stream)))
    return out


def lde_leaves_coset(coeffs, rate_bits: int, coset_gen: int, out=None, stream=None):
    """lde_leaves on the coset coset_gen * <w_N> (zk_lde_leaves_coset_async)."""
    import torch

    assert coeffs.dtype == torch.uint64 and coeffs.is_cuda and coeffs.is_contiguous() and coeffs.dim() == 2
    b, n = coeffs.shape
    lg_n = n.bit_length() - 1
    assert n == 1 << lg_n
    if out is None:
        out = torch.empty((n << rate_bits, b), dtype=torch.uint64, device=coeffs.device)
    capi.check(capi.LIB.zk_lde_leaves_coset_async(out.data_ptr(), coeffs.data_ptr(), lg_n, rate_bits, b,
                                                  coset_gen % P, _stream_ptr(stream)))
    return out


class CommitBuffers:
    """Device outputs of one commit: leaves (N, B), digests (2(N - 2^cap), 4), cap (2^cap, 4)."""

    def __init__(self, n_leaves: int, width: int, cap_height: int, device="cuda"):
        import torch

        nd, nc = merkle_sizes(n_leaves, cap_height)
        self.leaves = torch.empty((n_leaves, width), dtype=torch.uint64, device=device)
        self.digests = torch.empty((max(nd, 1), 4), dtype=torch.uint64, device=device)
        self.cap = torch.empty((nc, 4), dtype=torch.uint64, device=device)


def commit(coeffs, rate_bits: int, cap_height: int, hash_type: int = HashPoseidon, out: CommitBuffers | None = None,
           stream=None) -> CommitBuffers:
    """LDE -> leaves -> Merkle forest of (B, 2^lg_n) coefficients (zk_commit_async)."""
    b, n = coeffs.shape
    lg_n = n.bit_length() - 1
    if out is None:
        out = CommitBuffers(n << rate_bits, b, cap_height, coeffs.device)
    capi.check(capi.LIB.zk_commit_async(coeffs.data_ptr(), lg_n, rate_bits, b, cap_height, hash_type,
                                        out.leaves.data_ptr(), out.digests.data_ptr(), out.cap.data_ptr(),
                                        _stream_ptr(stream)))
    return out


def commit_batch(items, n_streams: int = 4, stream=None):
    """items: list of (coeffs, rate_bits, cap_height, hash_type, CommitBuffers); one zk_commit_batch call."""
    import ctypes

    arr = (capi.ZkCommitJob * len(items))()
    for i, (c, r, ch, ht, o) in enumerate(items):
        b, n = c.shape
        arr[i] = capi.ZkCommitJob(c.data_ptr(), n.bit_length() - 1, r, b, ch, ht, o.leaves.data_ptr(),
                                  o.digests.data_ptr(), o.cap.data_ptr())
    capi.check(capi.LIB.zk_commit_batch(ctypes.cast(arr, ctypes.POINTER(capi.ZkCommitJob)), len(items), n_streams,
                                        _stream_ptr(stream)))


def autotune(lg_n: int, rate_bits: int, batches: int) -> int:
    """Tune the LDE -> leaves stage for this shape (zk_autotune_commit); returns
    the number of candidates timed (0: already tuned or nothing to choose)."""
    import ctypes

    n = ctypes.c_int32()
    capi.check(capi.LIB.zk_autotune_commit(lg_n, rate_bits, batches, ctypes.byref(n)))
    return n.value


def autotune_reset():
    capi.check(capi.LIB.zk_autotune_reset())


class CommitGraph:
    """A batch of commits (commit_batch items) captured once into a CUDA graph.

    The first, uncaptured run builds the device tables and warms the memory
    pool; replay() then re-runs the whole batch (every LDE, transpose-to-leaves
    and Merkle launch of every job, forked over the internal streams) as one
    graph launch on the same buffers, so new coefficient values written into
    the input tensors are committed by the next replay."""

    def __init__(self, items, n_streams: int = 4):
        import torch

        self.items = items
        commit_batch(items, n_streams)
        torch.cuda.synchronize()
        self.graph = torch.cuda.CUDAGraph()
        side = torch.cuda.Stream()
        side.wait_stream(torch.cuda.current_stream())
        with torch.cuda.stream(side):
            with torch.cuda.graph(self.graph, stream=side):
                commit_batch(items, n_streams, stream=side)
        torch.cuda.current_stream().wait_stream(side)

    def replay(self):
        self.graph.replay()


class Server:
    """Commit server (zk_server_*): continuous batching under an HBM budget."""

    def __init__(self, hbm_budget_bytes: int, slots: int = 4, device: int = 0):
        import ctypes

        self._h = ctypes.c_void_p()
        capi.check(capi.LIB.zk_server_create(device, hbm_budget_bytes, slots, ctypes.byref(self._h)))
        self._keep = {}

    def submit(self, host_coeffs, rate_bits: int, cap_height: int, hash_type: int = HashPoseidon) -> int:
        """host_coeffs: (B, 2^lg_n) uint64 numpy array or pinned CPU tensor, kept alive until wait()."""
        import ctypes

        import numpy as np

        if isinstance(host_coeffs, np.ndarray):
            b, n = host_coeffs.shape
            ptr = host_coeffs.ctypes.data
        else:
            b, n = host_coeffs.shape
            ptr = host_coeffs.data_ptr()
        t = ctypes.c_uint64()
        capi.check(capi.LIB.zk_server_submit(self._h, ptr, n.bit_length() - 1, rate_bits, b, cap_height, hash_type,
                                             ctypes.byref(t)))
        self._keep[t.value] = (host_coeffs, cap_height)
        return t.value

    def submit_seeded(self, seed: int, lg_n: int, batches: int, rate_bits: int, cap_height: int,
                      hash_type: int = HashPoseidon) -> int:
        """A job whose (batches, 2^lg_n) coefficients are fill_field(seed), generated on the device at admission."""
        import ctypes

        t = ctypes.c_uint64()
        capi.check(capi.LIB.zk_server_submit_seeded(self._h, seed, lg_n, rate_bits, batches, cap_height, hash_type,
                                                    ctypes.byref(t)))
        self._keep[t.value] = (None, cap_height)
        return t.value

    def job_times(self, ticket: int):
        """-> (seconds queued, seconds from start to the cap on the host) of a completed job."""
        import ctypes

        q, r = ctypes.c_double(), ctypes.c_double()
        capi.check(capi.LIB.zk_server_job_times(self._h, ticket, ctypes.byref(q), ctypes.byref(r)))
        return q.value, r.value

    def inject_failure(self, n_jobs: int, at_allocation: int):
        """Test hook: the next n_jobs admitted jobs fail at their at_allocation-th device allocation."""
        capi.check(capi.LIB.zk_server_inject_failure(self._h, n_jobs, at_allocation))

    def wait(self, ticket: int):
        """-> (cap as a (2^cap_height, 4) uint64 array, latency in seconds)."""
        import ctypes

        import numpy as np

        _, ch = self._keep[ticket]
        cap = np.zeros((1 << ch, 4), dtype=np.uint64)
        lat = ctypes.c_double()
        capi.check(capi.LIB.zk_server_wait(self._h, ticket, cap.ctypes.data, ctypes.byref(lat)))
        return cap, lat.value

    def wait_any(self, timeout_ms: int | None = None):
        """Next completed (or failed) ticket in completion order, each returned once; None when no job is
        pending or the timeout (milliseconds; None = no limit) passes first."""
        import ctypes

        t = ctypes.c_uint64()
        capi.check(capi.LIB.zk_server_wait_any(self._h, 0xFFFFFFFF if timeout_ms is None else int(timeout_ms),
                                               ctypes.byref(t)))
        return t.value or None

    def result_ptrs(self, ticket: int):
        import ctypes

        l, d, c = ctypes.c_void_p(), ctypes.c_void_p(), ctypes.c_void_p()
        capi.check(capi.LIB.zk_server_result(self._h, ticket, ctypes.byref(l), ctypes.byref(d), ctypes.byref(c)))
        return l.value, d.value, c.value

    def release(self, ticket: int):
        capi.check(capi.LIB.zk_server_release(self._h, ticket))
        self._keep.pop(ticket, None)

    def stats(self) -> dict:
        import ctypes

        st = capi.ZkServerStats()
        capi.check(capi.LIB.zk_server_stats(self._h, ctypes.byref(st)))
        return {f: getattr(st, f) for f, _ in st._fields_}

    def close(self):
        if self._h:
            capi.check(capi.LIB.zk_server_destroy(self._h))
            self._h = None

    def __enter__(self):
        return self

    def __exit__(self, *exc):
        self.close()


def fill_field(out, seed: int, stream=None):
    """Fill a uint64 CUDA tensor with field elements uniform in [0, p) from `seed` (zk_fill_field_async)."""
    import torch

    assert out.dtype == torch.uint64 and out.is_cuda and out.is_contiguous()
    capi.check(capi.LIB.zk_fill_field_async(out.data_ptr(), out.numel(), seed & (2**64 - 1), _stream_ptr(stream)))
    return out


def merkle_sizes(n_leaves: int, cap_height: int):
    n_caps = 1 << cap_height
    return 2 * (n_leaves - n_caps), n_caps


def merkle_tree(leaves, cap_height: int, hash_type: int = HashPoseidon, digests=None, cap=None, stream=None):
    """Digests and cap of a (L, w) uint64 CUDA tensor of leaves, zeknox linear layout."""
    import torch

    assert leaves.dtype == torch.uint64 and leaves.is_cuda and leaves.is_contiguous() and leaves.dim() == 2
    n_leaves, w = leaves.shape
    n_digests, n_caps = merkle_sizes(n_leaves, cap_height)
    if digests is None:
        digests = torch.zeros((max(n_digests, 1), 4), dtype=torch.uint64, device=leaves.device)
    if cap is None:
        cap = torch.zeros((n_caps, 4), dtype=torch.uint64, device=leaves.device)
    capi.check(capi.LIB.zk_merkle_async(digests.data_ptr(), cap.data_ptr(), leaves.data_ptr(), n_digests, n_caps,
                                        n_leaves, w, cap_height, hash_type, _stream_ptr(stream)))
    return digests, cap


def merkle_open(leaves, digests, cap_height: int, indices, stream=None):
    """Opening proofs on a resident forest: for each leaf index, its leaf row and
    the sibling digests from the leaf level up to the level below the cap
    (Plonky2's MerkleProof order).  -> (rows (Q, w), siblings (Q, depth, 4)) CUDA
    tensors; the path of leaf i ends at cap entry i >> (log2(L) - cap_height)."""
    import torch

    assert leaves.dtype == torch.uint64 and leaves.is_cuda and leaves.is_contiguous() and leaves.dim() == 2
    n_leaves, w = leaves.shape
    idx = indices.to(device=leaves.device, dtype=torch.int64).contiguous().view(torch.uint64)
    q = idx.numel()
    depth = (n_leaves >> cap_height).bit_length() - 1
    rows = torch.empty((q, w), dtype=torch.uint64, device=leaves.device)
    sib = torch.empty((q, depth, 4), dtype=torch.uint64, device=leaves.device)
    capi.check(capi.LIB.zk_merkle_open_async(leaves.data_ptr(), digests.data_ptr(), n_leaves, w, cap_height,
                                             idx.data_ptr(), q, rows.data_ptr(), sib.data_ptr(), _stream_ptr(stream)))
    return rows, sib


# ---------------------------------------------------------------- FRI
def fri_fold(coeffs, arity_bits: int, beta, *, interleaved: bool = False, out=None, stream=None):
    """One FRI folding step over GF(p^2) = GF(p)[X]/(X^2 - 7) (zk_fri_fold_async).

    coeffs: (2, n) split (real parts, X parts) or, with `interleaved`, (n, 2)
    (real, X) pairs, uint64 CUDA tensor.  -> (2, n >> arity_bits) split:
    out[j] = sum_t beta^t coeffs[j 2^arity_bits + t], beta = (real, X part)."""
    import torch

    assert coeffs.dtype == torch.uint64 and coeffs.is_cuda and coeffs.is_contiguous() and coeffs.dim() == 2
    n = coeffs.shape[0] if interleaved else coeffs.shape[1]
    assert coeffs.shape == ((n, 2) if interleaved else (2, n))
    if out is None:
        out = torch.empty((2, n >> arity_bits), dtype=torch.uint64, device=coeffs.device)
    capi.check(capi.LIB.zk_fri_fold_async(out.data_ptr(), coeffs.data_ptr(), n, arity_bits, int(beta[0]) % P,
                                          int(beta[1]) % P, int(interleaved), _stream_ptr(stream)))
    return out


class FriRound:
    """One committed FRI round: leaves (N_i >> arity_bits, 2^(arity_bits+1)) rows of
    interleaved GF(p^2) evaluations in bit-reversed order, its Merkle forest, the
    coset shift it was evaluated on and the challenge drawn from its cap."""

    def __init__(self, leaves, digests, cap, arity_bits: int, shift: int):
        self.leaves, self.digests, self.cap = leaves, digests, cap
        self.arity_bits, self.shift = arity_bits, shift
        self.beta = None


class FriCommitment:
    def __init__(self, rounds, final_poly, cap_height: int):
        self.rounds, self.final_poly, self.cap_height = rounds, final_poly, cap_height


def fri_commit(coeffs, rate_bits: int, arity_bits, cap_height: int, challenge, hash_type: int = HashPoseidon,
               shift: int = 7, stream=None) -> FriCommitment:
    """The FRI commit phase over a resident polynomial (Plonky2's prover loop).

    coeffs: (2, n) split GF(p^2) coefficients on the device.  For each arity in
    `arity_bits`: the values on the current coset (shift, then shift^arity, ...)
    at rate `rate_bits` are written as leaves (zk_lde_leaves_coset_async,
    2 polynomials) and committed (zk_merkle_async); `challenge(round, cap)`
    (host callback, cap a (2^cap_height, 4) numpy array) returns beta; the
    coefficients are folded by beta (zk_fri_fold_async).  The final folded
    coefficients are returned on the device as `final_poly` (2, n / prod arity)."""
    import torch

    assert coeffs.dim() == 2 and coeffs.shape[0] == 2
    cur = coeffs
    rounds = []
    for i, ab in enumerate(arity_bits):
        n = cur.shape[1]
        leaves = lde_leaves_coset(cur, rate_bits, shift, stream=stream)
        view = leaves.view((n << rate_bits) >> ab, 2 << ab)
        dig, cap = merkle_tree(view, cap_height, hash_type, stream=stream)
        rnd = FriRound(view, dig, cap, ab, shift)
        s = stream if stream is not None else torch.cuda.current_stream()
        s.synchronize()
        rnd.beta = challenge(i, cap.cpu().numpy())
        rounds.append(rnd)
        cur = fri_fold(cur, ab, rnd.beta, stream=stream)
        shift = pow(shift, 1 << ab, P)
    return FriCommitment(rounds, cur, cap_height)


def fri_open(commitment: FriCommitment, indices, stream=None):
    """Query openings of every FRI round for indices into the first round's
    evaluation domain: round i opens leaf x >> (sum of the arity bits up to and
    including round i), as the FRI query phase does.  -> list of (rows, siblings)."""
    import torch

    idx = torch.as_tensor(indices, dtype=torch.int64).cpu()
    out = []
    shift = 0
    for rnd in commitment.rounds:
        shift += rnd.arity_bits
        out.append(merkle_open(rnd.leaves, rnd.digests, commitment.cap_height, idx >> shift, stream=stream))
    return out
