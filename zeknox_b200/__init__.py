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
