"""ctypes binding of libzeknox.so (include/zeknox.h).

Mirrors zeknox's language wrappers: the Rust crate (wrappers/rust/src/lib.rs:
``ntt_batch``, ``intt_batch``, ``lde_batch``, ``transpose_rev_batch``,
``init_twiddle_factors_rs``, ``init_coset_rs``, ``fill_digests_buf_linear_*``)
and the Go package (wrappers/go/lib/lib.go).  Calls that return a RustError
raise :class:`ZeknoxError` on a non-zero code, as the wrappers turn the code
into an error value.

There is no fallback: if libzeknox.so is missing or cannot be loaded, importing
this module raises.
"""

from __future__ import annotations

import ctypes
from pathlib import Path

PKG = Path(__file__).resolve().parent
LIB_PATH = PKG / "libzeknox.so"

HashPoseidon, HashKeccak, HashPoseidonBN128, HashPoseidon2, HashMonolith = 0, 1, 2, 3, 4
FORWARD, INVERSE = 0, 1


class ZeknoxError(RuntimeError):
    def __init__(self, code: int, message: str | None):
        super().__init__(f"zeknox error {code}: {message or ''}")
        self.code = code
        self.message = message


class RustError(ctypes.Structure):
    _fields_ = [("code", ctypes.c_int), ("message", ctypes.c_void_p)]


class NTTConfig(ctypes.Structure):
    """native/ntt/ntt.h:43-54 (wrappers/rust/src/types.rs:30-43)."""

    _fields_ = [
        ("batches", ctypes.c_uint32),
        ("order", ctypes.c_int),
        ("ntt_type", ctypes.c_int),
        ("extension_rate_bits", ctypes.c_uint32),
        ("are_inputs_on_device", ctypes.c_bool),
        ("are_outputs_on_device", ctypes.c_bool),
        ("with_coset", ctypes.c_bool),
        ("is_multi_gpu", ctypes.c_bool),
        ("salt_size", ctypes.c_uint32),
    ]

    @classmethod
    def default(cls) -> "NTTConfig":
        # wrappers/rust/src/types.rs:45-59
        return cls(batches=1, order=0, ntt_type=0, extension_rate_bits=0, are_inputs_on_device=False,
                   are_outputs_on_device=False, with_coset=False, is_multi_gpu=False, salt_size=0)


class TransposeConfig(ctypes.Structure):
    """native/ntt/ntt.h:56-61."""

    _fields_ = [("batches", ctypes.c_uint32), ("are_inputs_on_device", ctypes.c_bool),
                ("are_outputs_on_device", ctypes.c_bool)]

    @classmethod
    def default(cls) -> "TransposeConfig":
        return cls(batches=1, are_inputs_on_device=False, are_outputs_on_device=False)


class ZkCommitJob(ctypes.Structure):
    """include/zeknox.h ZkCommitJob (device buffers of one commit)."""

    _fields_ = [("d_coeffs", ctypes.c_void_p), ("lg_n", ctypes.c_uint32), ("rate_bits", ctypes.c_uint32),
                ("batches", ctypes.c_uint32), ("cap_height", ctypes.c_uint32), ("hash_type", ctypes.c_uint32),
                ("d_leaves", ctypes.c_void_p), ("d_digests", ctypes.c_void_p), ("d_cap", ctypes.c_void_p)]


class ZkServerStats(ctypes.Structure):
    _fields_ = [("completed", ctypes.c_uint64), ("queued", ctypes.c_uint64), ("max_queue", ctypes.c_uint64),
                ("p50_s", ctypes.c_double), ("p99_s", ctypes.c_double), ("max_s", ctypes.c_double),
                ("elems", ctypes.c_double), ("elems_per_s", ctypes.c_double), ("hbm_in_use", ctypes.c_uint64),
                ("hbm_peak", ctypes.c_uint64), ("ahead", ctypes.c_uint64),
                ("alloc_max_s", ctypes.c_double), ("pool_reserved_start", ctypes.c_uint64),
                ("pool_reserved_high", ctypes.c_uint64)]


assert ctypes.sizeof(NTTConfig) == 24 and ctypes.sizeof(TransposeConfig) == 8


def _load() -> ctypes.CDLL:
    if not LIB_PATH.exists():
        raise ImportError(f"{LIB_PATH} is not built; run `python zeknox_b200/build.py`")
    lib = ctypes.CDLL(str(LIB_PATH))
    vp, u32, u64, sz = ctypes.c_void_p, ctypes.c_uint32, ctypes.c_uint64, ctypes.c_size_t
    sig = {
        "get_number_of_gpus": (RustError, [ctypes.POINTER(ctypes.c_size_t)]),
        "list_devices_info": (RustError, []),
        "init_cuda": (None, []),
        "init_cuda_degree": (None, [u32]),
        "init_cuda_degree_and_generator": (None, [u32, u64]),
        "init_twiddle_factors": (RustError, [sz, sz]),
        "init_coset": (RustError, [sz, sz, u64]),
        "compute_batched_ntt": (RustError, [sz, vp, u32, ctypes.c_int, NTTConfig]),
        "compute_batched_lde": (RustError, [sz, vp, vp, u32, ctypes.c_int, NTTConfig]),
        "compute_batched_lde_multi_gpu": (RustError, [vp, vp, u32, ctypes.c_int, NTTConfig, u32, sz, sz]),
        "compute_transpose_rev": (RustError, [sz, vp, vp, u32, TransposeConfig]),
        "compute_naive_transpose_rev": (RustError, [sz, vp, vp, u32, TransposeConfig]),
        "fill_digests_buf_linear_gpu_with_gpu_ptr": (None, [vp, vp, vp, u64, u64, u64, u64, u64, u64, u64]),
        "fill_digests_buf_linear_multigpu_with_gpu_ptr": (None, [vp, vp, vp, u64, u64, u64, u64, u64, u64]),
        "fill_digests_buf_linear_cpu": (None, [vp, vp, vp, u64, u64, u64, u64, u64, u64]),
        "zk_last_error": (RustError, []),
        "zk_kernel_launches": (u64, []),
        "zk_lde_async": (RustError, [vp, vp, u32, u32, u32, u32, u32, vp]),
        "zk_transpose_rev_async": (RustError, [vp, vp, u32, u32, vp]),
        "zk_merkle_async": (RustError, [vp, vp, vp, u64, u64, u64, u64, u64, u64, vp]),
        "zk_merkle_open_async": (RustError, [vp, vp, u64, u64, u64, vp, u64, vp, vp, vp]),
        "zk_lde_noalloc": (RustError, [vp, vp, u32, u32, u32, u32, u32, vp]),
        "zk_lde_leaves_async": (RustError, [vp, vp, u32, u32, u32, vp]),
        "zk_lde_leaves_coset_async": (RustError, [vp, vp, u32, u32, u32, u64, vp]),
        "zk_fri_fold_async": (RustError, [vp, vp, u64, u32, u64, u64, u32, vp]),
        "zk_commit_async": (RustError, [vp, u32, u32, u32, u32, u32, vp, vp, vp, vp]),
        "zk_commit_batch": (RustError, [ctypes.POINTER(ZkCommitJob), u32, u32, vp]),
        "zk_server_create": (RustError, [ctypes.c_int32, u64, u32, ctypes.POINTER(vp)]),
        "zk_server_submit": (RustError, [vp, vp, u32, u32, u32, u32, u32, ctypes.POINTER(u64)]),
        "zk_server_wait": (RustError, [vp, u64, vp, ctypes.POINTER(ctypes.c_double)]),
        "zk_server_wait_any": (RustError, [vp, u32, ctypes.POINTER(u64)]),
        "zk_autotune_commit": (RustError, [u32, u32, u32, ctypes.POINTER(ctypes.c_int32)]),
        "zk_autotune_reset": (RustError, []),
        "zk_server_result": (RustError, [vp, u64, ctypes.POINTER(vp), ctypes.POINTER(vp), ctypes.POINTER(vp)]),
        "zk_server_release": (RustError, [vp, u64]),
        "zk_server_stats": (RustError, [vp, ctypes.POINTER(ZkServerStats)]),
        "zk_server_destroy": (RustError, [vp]),
        "zk_server_submit_seeded": (RustError, [vp, u64, u32, u32, u32, u32, u32, ctypes.POINTER(u64)]),
        "zk_server_inject_failure": (RustError, [vp, u32, u32]),
        "zk_fill_field_async": (RustError, [vp, u64, u64, vp]),
        "zk_server_job_times": (RustError, [vp, u64, ctypes.POINTER(ctypes.c_double), ctypes.POINTER(ctypes.c_double)]),
    }
    for name, (res, args) in sig.items():
        f = getattr(lib, name)
        f.restype = res
        f.argtypes = args
    return lib


LIB = _load()
_libc = ctypes.CDLL(None)
_libc.free.argtypes = [ctypes.c_void_p]


def check(err: RustError) -> None:
    """Raise on a non-zero RustError; frees the message (the caller owns it)."""
    if err.code == 0:
        if err.message:
            _libc.free(err.message)
        return
    msg = ctypes.string_at(err.message).decode(errors="replace") if err.message else None
    if err.message:
        _libc.free(err.message)
    raise ZeknoxError(err.code, msg)


def check_last() -> None:
    """Raise the failure recorded by the last void entry point on this thread, if any."""
    check(LIB.zk_last_error())


# ---- wrapper-style API (wrappers/rust/src/lib.rs:98-251) ----
def get_number_of_gpus() -> int:
    n = ctypes.c_size_t(0)
    check(LIB.get_number_of_gpus(ctypes.byref(n)))
    return n.value


def list_devices_info() -> None:
    check(LIB.list_devices_info())


def init_twiddle_factors(device_id: int, lg_n: int) -> None:
    check(LIB.init_twiddle_factors(device_id, lg_n))


def init_coset(device_id: int, lg_n: int, coset_gen: int) -> None:
    check(LIB.init_coset(device_id, lg_n, coset_gen))


def init_cuda() -> None:
    LIB.init_cuda()


def init_cuda_degree(max_degree: int) -> None:
    LIB.init_cuda_degree(max_degree)


def ntt_batch(device_id: int, inout: int, lg_n: int, cfg: NTTConfig) -> None:
    check(LIB.compute_batched_ntt(device_id, inout, lg_n, FORWARD, cfg))


def intt_batch(device_id: int, inout: int, lg_n: int, cfg: NTTConfig) -> None:
    check(LIB.compute_batched_ntt(device_id, inout, lg_n, INVERSE, cfg))


def lde_batch(device_id: int, output: int, input: int, lg_n: int, cfg: NTTConfig, direction: int = FORWARD) -> None:
    check(LIB.compute_batched_lde(device_id, output, input, lg_n, direction, cfg))


def lde_batch_multi_gpu(output: int, input: int, num_gpu: int, cfg: NTTConfig, lg_n: int, total_in: int,
                        total_out: int, direction: int = FORWARD) -> None:
    check(LIB.compute_batched_lde_multi_gpu(output, input, num_gpu, direction, cfg, lg_n, total_in, total_out))


def transpose_rev_batch(device_id: int, output: int, input: int, lg_n: int, cfg: TransposeConfig) -> None:
    check(LIB.compute_transpose_rev(device_id, output, input, lg_n, cfg))


def fill_digests_buf_linear_gpu_with_gpu_ptr(digests: int, cap: int, leaves: int, n_digests: int, n_caps: int,
                                             n_leaves: int, leaf_size: int, cap_height: int, hash_type: int,
                                             gpu_id: int = 0) -> None:
    LIB.fill_digests_buf_linear_gpu_with_gpu_ptr(digests, cap, leaves, n_digests, n_caps, n_leaves, leaf_size,
                                                 cap_height, hash_type, gpu_id)
    check_last()


def fill_digests_buf_linear_multigpu_with_gpu_ptr(digests: int, cap: int, leaves: int, n_digests: int, n_caps: int,
                                                  n_leaves: int, leaf_size: int, cap_height: int,
                                                  hash_type: int) -> None:
    LIB.fill_digests_buf_linear_multigpu_with_gpu_ptr(digests, cap, leaves, n_digests, n_caps, n_leaves, leaf_size,
                                                      cap_height, hash_type)
    check_last()


def fill_digests_buf_linear_cpu(digests: int, cap: int, leaves: int, n_digests: int, n_caps: int, n_leaves: int,
                                leaf_size: int, cap_height: int, hash_type: int) -> None:
    LIB.fill_digests_buf_linear_cpu(digests, cap, leaves, n_digests, n_caps, n_leaves, leaf_size, cap_height,
                                    hash_type)
    check_last()
