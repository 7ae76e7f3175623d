"""Build libzeknox.so / libzeknox.a (the C ABI of include/zeknox.h) for sm_100a.

    python zeknox_b200/build.py [--verbose]

Objects go to zeknox_b200/_build/, the libraries next to this file, so they
travel with the source tree.  nvcc cross-compiles without a GPU.
"""

from __future__ import annotations

import argparse
import concurrent.futures as cf
import os
import shutil
import subprocess
import sys
from pathlib import Path

PKG = Path(__file__).resolve().parent
CSRC = PKG / "csrc"
BUILD = PKG / "_build"
SO = PKG / "libzeknox.so"
AR = PKG / "libzeknox.a"
PROBE = PKG / "libzkprobe.so"  # measurement aid for bench.py (INT32 issue rate), not the product ABI
SOURCES = ["runtime.cu", "ntt.cu", "merkle.cu", "fri.cu", "capi.cu", "noalloc.cu", "serve.cu"]
ARCH = ["-gencode", "arch=compute_100a,code=sm_100a"]


def nvcc() -> str:
    cand = os.environ.get("NVCC") or shutil.which("nvcc") or "/usr/local/cuda/bin/nvcc"
    return cand


def _flags(verbose: bool) -> list[str]:
    f = ["-std=c++17", "-O3", "-lineinfo", *ARCH, "-Xcompiler", "-fPIC,-fvisibility=hidden",
         "--expt-relaxed-constexpr", "-I", str(PKG.parent / "include")]
    if verbose:
        f += ["-Xptxas", "-v"]
    return f


def _deps() -> list[Path]:
    return sorted(CSRC.glob("*.cu")) + sorted(CSRC.glob("*.cuh")) + sorted(CSRC.glob("*.h")) + \
        [PKG.parent / "include" / "zeknox.h"]


def _stale(out: Path) -> bool:
    if not out.exists():
        return True
    t = out.stat().st_mtime
    return any(p.stat().st_mtime > t for p in _deps())


def build(verbose: bool = False, force: bool = False) -> Path:
    if not force and not _stale(SO) and not _stale(AR) and not _stale(PROBE):
        return SO
    BUILD.mkdir(exist_ok=True)
    cmds = []
    for src in SOURCES:
        obj = BUILD / (Path(src).stem + ".o")
        cmds.append([nvcc(), *_flags(verbose), "-c", str(CSRC / src), "-o", str(obj)])
    cmds.append([nvcc(), *_flags(verbose), "-shared", "-cudart", "static", str(CSRC / "probe.cu"), "-o",
                 str(PROBE)])

    def run(cmd):
        r = subprocess.run(cmd, capture_output=True, text=True)
        return cmd, r

    objs = [str(BUILD / (Path(s).stem + ".o")) for s in SOURCES]
    with cf.ThreadPoolExecutor(max_workers=len(cmds)) as ex:
        for cmd, r in ex.map(run, cmds):
            if verbose or r.returncode:
                sys.stderr.write(r.stdout + r.stderr)
            if r.returncode:
                raise RuntimeError(f"nvcc failed: {' '.join(cmd)}")
    # Exported symbols are exactly the extern "C" ones (default visibility is
    # hidden; the C ABI is marked visible through the version script).
    vs = BUILD / "exports.map"
    vs.write_text("{ global: " + " ".join(f"{s};" for s in exported_symbols()) + " local: *; };\n")
    link = [nvcc(), *ARCH, "-shared", "-o", str(SO), *objs, "-cudart", "static",
            "-Xlinker", f"--version-script={vs}", "-Xlinker", "-Bsymbolic"]
    r = subprocess.run(link, capture_output=True, text=True)
    if r.returncode:
        sys.stderr.write(r.stdout + r.stderr)
        raise RuntimeError("link failed")
    if AR.exists():
        AR.unlink()
    subprocess.run(["ar", "rcs", str(AR), *objs], check=True)
    return SO


def exported_symbols() -> list[str]:
    """Every function include/zeknox.h declares (parsed from the header)."""
    import re

    hdr = (PKG.parent / "include" / "zeknox.h").read_text()
    return sorted(set(re.findall(r"ZK_EXTERN\s+[A-Za-z_][A-Za-z0-9_]*\s+\**\s*([A-Za-z_][A-Za-z0-9_]*)\s*\(", hdr)))


def main() -> None:
    ap = argparse.ArgumentParser()
    ap.add_argument("--verbose", action="store_true")
    ap.add_argument("--force", action="store_true")
    a = ap.parse_args()
    print(build(verbose=a.verbose, force=a.force))


if __name__ == "__main__":
    main()
