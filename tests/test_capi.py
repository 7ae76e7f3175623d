"""CPU tests of the drop-in boundary: libzeknox.so loads, exports every entry
point include/zeknox.h declares (and the libzeknox.a archive defines them),
the ABI structs have zeknox's layout, and host-side validation works without a
GPU.  No kernel is launched here."""

import ctypes
import re
import subprocess
from pathlib import Path

import pytest

ROOT = Path(__file__).resolve().parents[1]
HEADER = ROOT / "include" / "zeknox.h"

# The symbols zeknox's own headers declare for this path (native/lib.h:21-51,
# native/merkle/merkle.h:30-62, native/lib.cu:141 for init_cuda_degree_and_generator).
ZEKNOX_SYMBOLS = {
    "get_number_of_gpus", "list_devices_info", "init_cuda", "init_cuda_degree", "init_cuda_degree_and_generator",
    "init_twiddle_factors", "init_coset", "compute_batched_ntt", "compute_batched_lde",
    "compute_batched_lde_multi_gpu", "compute_transpose_rev", "compute_naive_transpose_rev",
    "fill_digests_buf_linear_gpu_with_gpu_ptr", "fill_digests_buf_linear_multigpu_with_gpu_ptr",
    "fill_digests_buf_linear_cpu",
}


def declared():
    return set(re.findall(r"ZK_EXTERN\s+[A-Za-z_][A-Za-z0-9_]*\s+\**\s*([A-Za-z_][A-Za-z0-9_]*)\s*\(", HEADER.read_text()))


def test_header_declares_zeknox_abi():
    assert ZEKNOX_SYMBOLS <= declared()


def test_library_loads_and_exports_every_declared_symbol():
    import zeknox_b200.capi as capi

    for name in declared():
        assert hasattr(capi.LIB, name), name
    out = subprocess.run(["nm", "-D", "--defined-only", str(capi.LIB_PATH)], capture_output=True, text=True).stdout
    exported = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert declared() <= exported
    # only the C ABI is exported
    assert exported <= declared() | {"_init", "_fini"}


def test_static_archive_defines_the_abi():
    ar = ROOT / "zeknox_b200" / "libzeknox.a"
    out = subprocess.run(["nm", "--defined-only", str(ar)], capture_output=True, text=True).stdout
    defined = {ln.split()[-1] for ln in out.splitlines() if " T " in ln}
    assert declared() <= defined


def test_struct_layouts():
    from zeknox_b200.capi import NTTConfig, RustError, TransposeConfig

    assert ctypes.sizeof(NTTConfig) == 24 and NTTConfig.salt_size.offset == 20
    assert NTTConfig.are_inputs_on_device.offset == 16 and NTTConfig.is_multi_gpu.offset == 19
    assert ctypes.sizeof(TransposeConfig) == 8 and TransposeConfig.are_outputs_on_device.offset == 5
    assert ctypes.sizeof(RustError) == 16


def test_c_header_compiles_as_c_and_matches_layout(tmp_path):
    src = tmp_path / "t.c"
    src.write_text('#include "zeknox.h"\n#include <stddef.h>\n'
                   "#ifdef __cplusplus\n#define _Static_assert static_assert\n#endif\n"
                   "_Static_assert(sizeof(NTT_Config) == 24, \"cfg\");\n"
                   "_Static_assert(offsetof(NTT_Config, salt_size) == 20, \"salt\");\n"
                   "_Static_assert(sizeof(NTT_TransposeConfig) == 8, \"tcfg\");\n"
                   "_Static_assert(sizeof(RustError) == 16, \"err\");\n"
                   "int main(void) { return 0; }\n")
    subprocess.run(["gcc", "-std=c11", "-Wall", "-Werror", "-I", str(ROOT / "include"), "-c", str(src), "-o",
                    str(tmp_path / "t.o")], check=True)
    subprocess.run(["g++", "-std=c++17", "-Wall", "-Werror", "-x", "c++", "-I", str(ROOT / "include"), "-c",
                    str(src), "-o", str(tmp_path / "t2.o")], check=True)


def test_c_program_links_and_runs_against_both_libraries(tmp_path):
    """A C caller (what the Go wrapper's cgo build is) links the shared library
    alone, or the static archive plus the static CUDA runtime, and calls into
    it: get_number_of_gpus answers without a device (0 here) or with one."""
    import shutil

    cuda_lib = Path("/usr/local/cuda/lib64")
    if not (cuda_lib / "libcudart_static.a").exists() or shutil.which("gcc") is None:
        pytest.skip("static CUDA runtime or gcc not available")
    src = tmp_path / "t.c"
    src.write_text('#include <stdio.h>\n#include <stdlib.h>\n#include "zeknox.h"\n'
                   "int main(void) {\n  size_t n = 99;\n  RustError e = get_number_of_gpus(&n);\n"
                   '  printf("%d %zu\\n", e.code, n);\n  free(e.message);\n  return e.code != 0;\n}\n')
    pkg = ROOT / "zeknox_b200"
    exe_static, exe_shared = tmp_path / "t_static", tmp_path / "t_shared"
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe_static),
                    str(pkg / "libzeknox.a"), "-L", str(cuda_lib), "-lcudart_static", "-lstdc++", "-ldl", "-lrt",
                    "-lpthread", "-lm"], check=True)
    subprocess.run(["gcc", "-std=c11", "-I", str(ROOT / "include"), str(src), "-o", str(exe_shared), "-L", str(pkg),
                    "-lzeknox", f"-Wl,-rpath,{pkg}"], check=True)
    for exe in (exe_static, exe_shared):
        out = subprocess.run([str(exe)], check=True, capture_output=True, text=True).stdout.split()
        assert out[0] == "0" and int(out[1]) >= 0


def test_host_validation_without_gpu():
    import zeknox_b200 as zk

    # argument checks that zeknox performs before touching the device (ntt.cu:255-256, :478-481)
    cfg = zk.NTTConfig.default()
    with pytest.raises(zk.ZeknoxError) as e:
        zk.ntt_batch(0, 0, 0, cfg)
    assert e.value.code == 1
    cfg.extension_rate_bits = 0
    with pytest.raises(zk.ZeknoxError) as e:
        zk.lde_batch(0, 0, 0, 5, cfg)
    assert e.value.code == 1 and "invalid args" in e.value.message
    # FRI fold: arguments are checked before anything is launched
    L = zk.capi.LIB
    assert L.zk_fri_fold_async(None, None, 64, 2, 1, 0, 0, None).code == 1  # null buffers
    fake = ctypes.c_void_p(16)  # never dereferenced: every call below fails its checks first
    for n_in, ab, b0, b1 in [(64, 0, 1, 0), (64, 7, 1, 0), (48, 2, 1, 0), (2, 2, 1, 0), (64, 2, 2**64 - 1, 0),
                             (64, 2, 0, 0xFFFFFFFF00000001)]:
        err = L.zk_fri_fold_async(fake, ctypes.c_void_p(32), n_in, ab, b0, b1, 0, None)
        assert err.code == 1, (n_in, ab, b0, b1)
    assert L.zk_fri_fold_async(fake, fake, 64, 2, 1, 0, 0, None).code == 1  # in place
    assert L.zk_fri_fold_async(fake, ctypes.c_void_p(40), 64, 2, 1, 0, 1, None).code == 1  # misaligned pairs
    n = zk.get_number_of_gpus()
    assert n >= 0
    if n == 0:  # no device: the calls fail with an error code instead of crashing
        with pytest.raises(zk.ZeknoxError):
            zk.init_twiddle_factors(0, 10)
